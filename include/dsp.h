/*
 * dsp.h — C ABI of the B200 DISORT spectral engine (libdsp.so).
 *
 * One call solves a whole spectral loop: many independent (column, band)
 * instances of the DISORT boundary-value problem, in FP64, on one GPU.
 *
 * The entry points replace these reference interfaces (DisORT++):
 *   dsp_flux_bands_solve     <- solveFluxSpectralBandsImpl<N> / DisortFluxSolver<N>::solve
 *                               (src/python_bindings.cpp:170-211, src/FluxSolver.hpp:49);
 *                               also solveFluxSpectralImpl<N> (src/python_bindings.cpp:148-168):
 *                               a single-wavenumber loop is the same call with
 *                               wavenumber_low == wavenumber_high per instance
 *   dsp_general_bands_solve  <- solveSpectralBands / DisortSolver::solve
 *                               (src/python_bindings.cpp:108-127, src/DisortSolver.hpp:87)
 *
 * Conventions
 *  - Plain pointers and sizes only; no exceptions cross this boundary.
 *  - Every array is given as (pointer, instance stride in elements).  A stride of 0
 *    means "shared by all instances", which is how the reference's base config plus
 *    optional per-band override lists (SpectralOverrides, python_bindings.cpp:51-82)
 *    map onto one batch.
 *  - Buffers are caller owned.  With DSP_FLAG_DEVICE_POINTERS every pointer in the
 *    batch and the output is device memory and the call is stream ordered (no host
 *    synchronisation).  Without it every pointer is host memory; the context stages
 *    the copies through its own device buffers and the call returns after the results
 *    are back in host memory.
 *  - Output arrays are instance-major: out[i * (num_layers + 1) + level], level 0 =
 *    top of atmosphere (or bottom with DSP_FLAG_INDEX_FROM_BOTTOM, as the reference).
 *  - Per-instance status codes (dsp_status) go to out->status when it is non-NULL.
 *    The reference throws std::invalid_argument for what is DSP_ERR_INVALID_INPUT
 *    here; an invalid instance gets NaN outputs and its status, the others are solved.
 *  - A context is used by one host thread at a time.
 */
#ifndef DSP_H
#define DSP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSP_API_VERSION 3

typedef enum dsp_status {
  DSP_OK = 0,
  DSP_ERR_INVALID_INPUT = 1, /* a validate() rule failed (DisortFluxConfig.cpp:43-143) */
  DSP_ERR_SINGULAR = 2,      /* zero pivot in a linear solve (BandSolver.hpp:76-78 skips it) */
  DSP_ERR_NONFINITE = 3,     /* a non-finite output value */
  DSP_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  DSP_ERR_CUDA = 5,          /* a CUDA runtime error; see dsp_context_last_error */
  DSP_ERR_UNSUPPORTED = 6,   /* option outside the engine (e.g. spherical beam) */
  DSP_ERR_NO_MEMORY = 7,     /* device or pinned allocation failed */
  DSP_ERR_EIGEN = 8,         /* neither symmetric factorisation of the layer eigenproblem exists */
  DSP_ERR_NOT_INITIALIZED = 9
} dsp_status;

/* batch flags */
#define DSP_FLAG_THERMAL            (1u << 0) /* use_thermal_emission */
#define DSP_FLAG_DELTA_M_PLUS       (1u << 1) /* use_delta_m_plus */
#define DSP_FLAG_DIFFUSION_LOWER_BC (1u << 2) /* use_diffusion_lower_bc */
#define DSP_FLAG_INDEX_FROM_BOTTOM  (1u << 3) /* index_from_bottom (layer/level arrays reversed) */
#define DSP_FLAG_DEVICE_POINTERS    (1u << 4) /* every pointer is device memory */
#define DSP_FLAG_SPHERICAL_BEAM     (1u << 5) /* use_spherical_beam */
#define DSP_FLAG_TEMPERATURE_JAC    (1u << 6) /* compute_temperature_jacobian: use dsp_flux_bands_solve_jac */
/*
 * Henyey-Greenstein fast path (flux batches): phase_function_moments holds ONE
 * asymmetry factor g per layer ([L] per instance) instead of [L][pmom_count]
 * moments, and the engine forms the moments g^k, k = 0 .. pmom_count-1, on the
 * device with the products of setHenyeyGreenstein (fillHenyeyGreenstein,
 * src/PhaseFunction.cpp:6-19), so the result equals the moment path fed with
 * those moments bit for bit.  Cuts the upload of a host-buffer solve by a factor
 * of about pmom_count on the moment array.
 */
#define DSP_FLAG_HG_G               (1u << 7)

/* A strided double array: element (instance i, index k) = ptr[i * stride + k]. */
typedef struct dsp_darray {
  const double* ptr;
  int64_t stride; /* 0: one copy shared by all instances */
} dsp_darray;

/*
 * Flux-only batch (DisortFluxConfig fields, DisortFluxConfig.hpp:15-93).
 * All instances share num_streams and num_layers, like one reference spectral loop.
 */
typedef struct dsp_flux_batch {
  int32_t n_inst;
  int32_t num_streams;            /* N: 4, 6, 8, 10, 12, 14, 16, 32 or 64 */
  int32_t num_layers;             /* L >= 1 */
  int32_t num_phase_func_moments; /* the config's num_phase_func_moments */
  int32_t pmom_count;             /* doubles per layer in phase_function_moments (>= nmomNstr()+1) */
  uint32_t flags;

  dsp_darray wavenumber_low;          /* [1] per instance */
  dsp_darray wavenumber_high;         /* [1] */
  dsp_darray delta_tau;               /* [L] */
  dsp_darray single_scat_albedo;      /* [L] */
  dsp_darray phase_function_moments;  /* [L][pmom_count] */
  dsp_darray temperature;             /* [L+1] (thermal only; may be NULL otherwise) */
  dsp_darray surface_albedo;          /* [1] */
  dsp_darray emissivity_top;          /* [1] */
  dsp_darray direct_beam_flux;        /* [1] */
  dsp_darray direct_beam_mu;          /* [1] */
  dsp_darray isotropic_flux_top;      /* [1] */
  dsp_darray isotropic_flux_bottom;   /* [1] */
  dsp_darray temperature_top;         /* [1] */
  dsp_darray temperature_bottom;      /* [1] */
  /* pseudo-spherical beam (DSP_FLAG_SPHERICAL_BEAM; may be NULL otherwise) */
  dsp_darray level_altitudes;         /* [L+1], top down, the units of bottom_radius */
  dsp_darray bottom_radius;           /* [1] */
} dsp_flux_batch;

/* FluxResult (FluxResult.hpp:14-22): each array is [n_inst][L+1]. */
typedef struct dsp_flux_out {
  double* flux_direct_beam;
  double* flux_down;
  double* flux_up;
  double* flux_tau_divergence;
  double* mean_intensity;
  double* mean_intensity_down;
  double* mean_intensity_up;
  double* mean_intensity_direct_beam;
  int32_t* status; /* [n_inst] or NULL */
} dsp_flux_out;

/*
 * Temperature Jacobians of a flux solve (FluxResult's *_temperature_jac fields,
 * FluxResult.hpp; computeThermalJacobian, src/FluxSolver.cpp:1294-1497).  Each
 * array is [n_inst][L+1][L+2]: row = output level (indexed like the fluxes),
 * column = level temperature 0..L (reversed with the levels under
 * DSP_FLAG_INDEX_FROM_BOTTOM), then the surface temperature (temperature_bottom)
 * in column L+1.  Units: output per kelvin.  Without DSP_FLAG_THERMAL every entry
 * is zero (the reference returns empty Jacobians there).
 */
typedef struct dsp_flux_jac_out {
  double* flux_up;
  double* flux_down;
  double* mean_intensity;
  double* mean_intensity_down;
  double* mean_intensity_up;
  double* flux_divergence;
} dsp_flux_jac_out;

/*
 * General batch (DisortConfig, DisortConfig.hpp:119-243): the full DisortSolver
 * with Fourier azimuth modes and intensities at user optical depths, polar
 * angles and azimuths.  Plane-parallel or pseudo-spherical beam geometry,
 * Lambertian or bidirectional (BRDF) surface.
 * Instances may differ in num_streams and num_layers: instance i owns layers
 * layer_offset[i] .. layer_offset[i+1]-1 of the layer arrays (CSR) and levels
 * layer_offset[i] + i .. layer_offset[i+1] + i of the level arrays.
 */
#define DSP_GFLAG_USER_TAU         (1u << 8)  /* use_user_tau (else outputs at the layer boundaries) */
#define DSP_GFLAG_USER_MU          (1u << 9)  /* use_user_mu */
#define DSP_GFLAG_ONLY_FLUXES      (1u << 10) /* comp_only_fluxes */
/*
 * intensity_corr_buras with the Nakajima-Tanaka method (intensity_corr_nakajima,
 * or no tabulated phase function): after the mode loop the intensities get the
 * TMS/IMS corrections where DisortSolver applies them (delta-M scaling, a beam,
 * scattering; DisortSolver.cpp:352-368, 3274-3530) and, over a BRDF surface,
 * the correction of the reflected beam (delta-M+ off; :376-391, 3751-3810).
 * Fluxes and azimuthal averages are unchanged.
 */
#define DSP_GFLAG_INTENSITY_CORR   (1u << 11)
/*
 * With DSP_GFLAG_INTENSITY_CORR: the Buras-Emde method instead
 * (intensity_corr_buras without intensity_corr_nakajima and with a tabulated
 * phase function, DisortSolver.cpp:362-367, 3532-3749): the exact single
 * scattering from the tabulated phase function, the secondary scattering from
 * its residual after the delta-M truncation.  Needs num_phase_func_angles >= 2,
 * mu_phase_function (increasing cosines) and phase_function.
 */
#define DSP_GFLAG_INTENSITY_CORR_BE (1u << 12)

typedef struct dsp_general_batch {
  int32_t n_inst;
  uint32_t flags;                 /* DSP_FLAG_* and DSP_GFLAG_* */
  const int32_t* num_streams;     /* [n_inst] */
  const int32_t* num_layers;      /* [n_inst] */
  const int64_t* layer_offset;    /* [n_inst+1] */
  const int32_t* num_phase_func_moments; /* [n_inst] */
  int32_t pmom_count;             /* doubles per layer in phase_function_moments */
  int32_t num_user_tau;           /* ntau (with DSP_GFLAG_USER_TAU), else ignored */
  int32_t num_user_mu;            /* numu (with DSP_GFLAG_USER_MU) */
  int32_t num_phi;                /* nphi */
  double accuracy_fourier_series; /* azimuthal convergence criterion (0: all modes) */

  const double* delta_tau;              /* [total layers] */
  const double* single_scat_albedo;     /* [total layers] */
  const double* phase_function_moments; /* [total layers][pmom_count] */
  const double* temperature;            /* [total layers + n_inst] (thermal only) */
  dsp_darray tau_user;                  /* [ntau] per instance or shared */
  dsp_darray mu_user;                   /* [numu], ascending */
  dsp_darray phi_user;                  /* [nphi], degrees */
  dsp_darray wavenumber_low, wavenumber_high, surface_albedo, emissivity_top, direct_beam_flux,
      direct_beam_mu, direct_beam_phi, isotropic_flux_top, isotropic_flux_bottom, temperature_top,
      temperature_bottom; /* [1] each */
  /* pseudo-spherical beam (DSP_FLAG_SPHERICAL_BEAM; may be NULL otherwise) */
  const double* level_altitudes;        /* [total layers + n_inst], top down, levels like temperature */
  dsp_darray bottom_radius;             /* [1] */
  /*
   * Bidirectional surface (DisortFlags::use_lambertian_surface = false with
   * DisortFlags::brdf_type, DisortConfig::brdf; DisortSolver.cpp:2582-2936).
   * brdf_type 0 (DSP_BRDF_LAMBERTIAN, what a zero-initialised batch gives) keeps
   * the Lambertian surface of surface_albedo.  Otherwise surface_albedo is not
   * read and brdf_params holds DSP_BRDF_PARAMS doubles per instance (stride 0:
   * shared), in the order of the reference's spec struct:
   *   DSP_BRDF_RPV       rho0, k, theta, sigma, t1, t2, scale   (RpvBrdfSpec)
   *   DSP_BRDF_COX_MUNK  u10, pcl, xsal, refractive_index, do_shadow (0 or 1)
   *   DSP_BRDF_AMBRALS   iso, vol, geo                          (AmbralsBrdfSpec)
   *   DSP_BRDF_HAPKE     b0, hh, w                              (HapkeBrdfSpec)
   * The surface's Fourier coefficients are formed on the device at every
   * azimuth mode with the reference's 100-node azimuth quadrature.
   */
  int32_t brdf_type;
  dsp_darray brdf_params;               /* [DSP_BRDF_PARAMS] */
  /* tabulated phase function (DisortConfig::mu_phase_function, ::phase_function),
     read with DSP_GFLAG_INTENSITY_CORR_BE only */
  int32_t num_phase_func_angles;
  dsp_darray mu_phase_function;         /* [num_phase_func_angles] per instance or shared */
  const double* phase_function;         /* [total layers][num_phase_func_angles], layers like delta_tau */
} dsp_general_batch;

/* brdf_type values: the BrdfType enum of DisortConfig.hpp */
#define DSP_BRDF_LAMBERTIAN 0
#define DSP_BRDF_RPV        1
#define DSP_BRDF_COX_MUNK   2
#define DSP_BRDF_AMBRALS    3
#define DSP_BRDF_HAPKE      4
#define DSP_BRDF_PARAMS     8

/*
 * Temperature Jacobians of a general solve (DisortResult's *_temperature_jac,
 * computeThermalJacobian, src/DisortSolver.cpp:2130-2358): each array is
 * [n_inst][ntau_out][ndof_out]; row = output optical depth (indexed like the
 * fluxes), column = level temperature 0..L_i, then the surface temperature in
 * column L_i + 1 (columns past it are untouched).  ndof_out >= max L_i + 2.
 */
typedef struct dsp_general_jac_out {
  double* flux_up;
  double* flux_down;
  double* mean_intensity;
  double* mean_intensity_down;
  double* mean_intensity_up;
  double* flux_divergence;
  int32_t ndof_out;
} dsp_general_jac_out;

/* DisortResult (DisortResult.hpp:16-125) for the general batch. */
typedef struct dsp_general_out {
  double* flux[8];                /* FluxResult order, each [n_inst][ntau_out] */
  double* intensity;              /* [n_inst][ntau_out][numu_out][nphi] */
  double* intensity_azimuth_avg;  /* [n_inst][ntau_out][numu_out] */
  int32_t* status;                /* [n_inst] or NULL */
  int32_t ntau_out;               /* output row stride: >= ntau (or >= max L+1 without user taus) */
  int32_t numu_out;               /* output stride: >= numu (or >= max N without user angles) */
} dsp_general_out;

typedef struct dsp_context_s* dsp_context;

/* Library / context management. `stream` is a cudaStream_t (NULL = legacy default). */
int32_t dsp_api_version(void);
const char* dsp_status_string(dsp_status s);
dsp_status dsp_context_create(int32_t device, void* stream, dsp_context* out);
dsp_status dsp_context_destroy(dsp_context ctx);
dsp_status dsp_context_set_stream(dsp_context ctx, void* stream);
const char* dsp_context_last_error(dsp_context ctx);

/*
 * Device bytes a DSP_FLAG_DEVICE_POINTERS flux solve of this batch needs as
 * workspace (the context allocates and caches it on first use).
 */
int64_t dsp_flux_workspace_bytes(const dsp_flux_batch* batch);

/*
 * Per-kernel device timing (instrumentation; no reference counterpart).  When
 * enabled, every kernel launch of the context is bracketed by CUDA events on the
 * context's stream; totals accumulate until reset.  Names are static strings.
 */
dsp_status dsp_context_set_timing(dsp_context ctx, int32_t enable);
dsp_status dsp_context_timing_reset(dsp_context ctx);
int32_t dsp_context_timing_count(dsp_context ctx);
dsp_status dsp_context_timing_get(dsp_context ctx, int32_t idx, const char** name, double* total_ms,
                                  int64_t* launches);

/*
 * Debug options of a context (no reference counterpart).  With
 * DSP_DEBUG_POISON_SCRATCH every chunk's workspace is filled with NaN (all bits
 * set) before its kernels run, so that a kernel reading scratch it did not
 * write shows up as NaN outputs.  Costs one memset of the workspace per chunk.
 */
#define DSP_DEBUG_POISON_SCRATCH 1u
dsp_status dsp_context_set_debug(dsp_context ctx, uint32_t flags);

/*
 * Launch schedules (no reference counterpart; the reference has one code path
 * per solver).  An entry applies to instances with num_streams == N and
 * min_layers <= num_layers <= max_layers; the first matching entry wins, and
 * without one the built-in choice stands.  Fields (0 = built-in choice):
 *   layer_stage  flux path, N <= 16: 1 = three one-thread-per-task launches
 *                (register-resident eigensolver), 2 = one team per layer task
 *                (shared-memory eigensolver);
 *   layer_cta    threads per CTA of the one-thread-per-task launches: 64 or 128;
 *   persistent   general path: 1 = boundary-value and intensity kernels run
 *                as resident grids that take instances from a queue ordered by
 *                descending layer count (size class), 2 = one CTA or team per
 *                instance in index order.
 * dsp_context_load_schedule_file reads entries as text lines
 *   "N min_layers max_layers layer_stage layer_cta persistent"
 * ('#' starts a comment), as written by the autotuner (disort_b200/autotune.py),
 * and replaces the context's table; DSP_ERR_INVALID_INPUT on a malformed file.
 */
typedef struct dsp_schedule {
  int32_t num_streams, min_layers, max_layers;
  int32_t layer_stage, layer_cta, persistent;
} dsp_schedule;
dsp_status dsp_context_set_schedule(dsp_context ctx, const dsp_schedule* entries, int32_t count);
dsp_status dsp_context_load_schedule_file(dsp_context ctx, const char* path);
int32_t dsp_context_schedule_count(dsp_context ctx);

/*
 * A spectral loop as one CUDA graph (no reference counterpart): the whole
 * device-pointer flux solve of `batch` into `out` (DSP_FLAG_DEVICE_POINTERS
 * required; not with DSP_FLAG_TEMPERATURE_JAC) captured once and replayed by
 * dsp_graph_launch on any stream of `device`.  Replays read the batch's device
 * arrays and write `out` at the addresses given here, so a caller refreshes the
 * inputs in place between launches.  The graph owns a private context (its
 * workspace addresses are part of the graph); creation runs the solve once
 * eagerly, then captures it.  Destroy only after the last launch has completed
 * (synchronize its stream first).
 */
typedef struct dsp_graph_s* dsp_graph;
dsp_status dsp_flux_graph_create(int32_t device, const dsp_flux_batch* batch, const dsp_flux_out* out,
                                 dsp_graph* graph);
dsp_status dsp_graph_launch(dsp_graph graph, void* stream);
dsp_status dsp_graph_destroy(dsp_graph graph);

/* Flux-only spectral-band solve (DisortFluxSolver<N> over every instance). */
dsp_status dsp_flux_bands_solve(dsp_context ctx, const dsp_flux_batch* batch,
                                const dsp_flux_out* out);

/*
 * Flux solve with temperature Jacobians (DisortFluxSolver<N>::solve with
 * compute_temperature_jacobian, src/FluxSolver.cpp:1294-1497): the fluxes of
 * dsp_flux_bands_solve plus `jac`.  The batch flag DSP_FLAG_TEMPERATURE_JAC is
 * implied; dsp_flux_bands_solve itself rejects that flag.
 */
dsp_status dsp_flux_bands_solve_jac(dsp_context ctx, const dsp_flux_batch* batch,
                                    const dsp_flux_out* out, const dsp_flux_jac_out* jac);

/* General spectral-band solve (DisortSolver::solve over every instance). */
dsp_status dsp_general_bands_solve(dsp_context ctx, const dsp_general_batch* batch,
                                   const dsp_general_out* out);

/*
 * General solve with temperature Jacobians (DisortSolver::solve with
 * compute_temperature_jacobian, src/DisortSolver.cpp:2130-2358).  The batch flag
 * DSP_FLAG_TEMPERATURE_JAC is implied; dsp_general_bands_solve rejects it.
 */
dsp_status dsp_general_bands_solve_jac(dsp_context ctx, const dsp_general_batch* batch,
                                       const dsp_general_out* out, const dsp_general_jac_out* jac);

/*
 * Albedo and transmissivity of the medium (ibcnd = Special; DisortSolver::solve
 * with computeAlbTrans, src/DisortSolver.cpp:52-58, 169-176, 4025-4358):
 * isotropic illumination of unit intensity from the top, and for more than
 * one layer from the bottom, of each instance with a black surface.  Reads
 * num_streams, num_layers, layer_offset, num_phase_func_moments, delta_tau,
 * single_scat_albedo, phase_function_moments, surface_albedo (the spherical
 * albedo correction), DSP_FLAG_DELTA_M_PLUS, DSP_FLAG_INDEX_FROM_BOTTOM and,
 * with DSP_GFLAG_USER_MU, the num_user_mu positive cosines of mu_user (else
 * the N/2 quadrature cosines); sources, optical depths and azimuths are not
 * read.  Host pointers only.  Outputs per instance: albedo_medium and
 * transmissivity_medium at the cosines [n_inst][numu_out], the spherical
 * albedo and transmissivity [n_inst] (zero unless surface_albedo > 0).
 */
typedef struct dsp_albtrans_out {
  double* albedo_medium;
  double* transmissivity_medium;
  double* spherical_albedo;
  double* spherical_transmissivity;
  int32_t* status;                  /* [n_inst] or NULL */
  int32_t numu_out;                 /* >= num_user_mu (or max N/2 without user angles) */
} dsp_albtrans_out;
dsp_status dsp_general_bands_albtrans(dsp_context ctx, const dsp_general_batch* batch,
                                      const dsp_albtrans_out* out);

/*
 * Flux solve without any allocation (no counterpart in the reference: DisORT++
 * solves on the CPU and allocates freely).  For callers that must not let a
 * library allocate device memory -- applications that hand the GPU to their own
 * pooled allocator, or that forbid allocation after start-up.  It runs the same
 * kernels as dsp_flux_bands_solve with a workspace compiled into libdsp.so: a
 * 32 MiB device array (dsp_noalloc_scratch_bytes()) that each GPU loading the
 * library keeps until exit.  Needs no context; all batch and output pointers
 * must be device memory (DSP_FLAG_DEVICE_POINTERS).  The kernels are queued on
 * `stream` (a cudaStream_t, NULL = legacy default) and not waited for; the small
 * copies of the quadrature tables and of the defaults of absent scalar inputs come
 * from pageable host memory, which the driver stages before the call returns.  An
 * instance whose workspace exceeds the array is rejected with DSP_ERR_NO_MEMORY
 * before anything is queued; larger batches reuse the array in several launches.
 * All calls share the array and it keeps the last call's contents: calls that may
 * overlap on the GPU race and must be serialised by the caller.  Every call looks
 * up the array's address on the current device (cudaGetSymbolAddress), so no
 * per-device state outlives a device reset.
 */
int64_t dsp_noalloc_scratch_bytes(void);
dsp_status dsp_flux_bands_solve_noalloc(const dsp_flux_batch* batch, const dsp_flux_out* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DSP_H */
