// dsp_general.cu — dsp_general_bands_solve: the general solver (DisortSolver::
// solve, DisortSolver.cpp:21-399) over a ragged batch of instances.
//
// Instances are grouped by stream count (one kernel instantiation per N), the
// groups cut into chunks that fit the workspace, and each chunk runs
//   gen_setup_kernel, then for every azimuth mode m the layer kernel (eigen-
//   systems, particular solutions, user-angle interpolation), the boundary-
//   value kernel (solution coefficients; fluxes at m = 0) and the intensity
//   kernel (Fourier accumulation and the convergence test).
// Instances whose series has ended (last mode, or converged) skip the later
// mode launches on the device.
#include "dsp_host.hpp"
#include "flux_bvp_tile.cuh"
#include "flux_bvp_reg.cuh"
#include "flux_jac.cuh"
#include "flux_layer.cuh"
#include "flux_sph.cuh"
#include "gen_brdf.cuh"
#include "gen_intcor.cuh"
#include "gen_kernels.cuh"

using namespace dsp;
using namespace dsp_host;

namespace {

// Per-mode constant tables for N streams: N copies of the tab_* layout whose
// Legendre block holds P_l^m(mu_i) of mode m (rows l < m zero).  The rows are
// produced by running the reference's per-mode recurrence in sequence, each
// mode seeding P_m^m from row m-1 of the previous mode (Legendre.cpp:89-119).
bool build_mode_tables(int N, std::vector<double>& out) {
  std::vector<double> base;
  if (!build_tables(N, base)) return false;
  const int T = tab_size(N);
  out.assign((size_t)T * N, 0.0);
  const double* mu = base.data() + tab_mu(N);
  std::vector<double> y((size_t)N * N, 0.0);
  for (int m = 0; m < N; ++m) {
    for (int i = 0; i < N; ++i) {
      if (m == 0) {
        y[0 * N + i] = 1.0;
        y[1 * N + i] = mu[i];
        for (int l = 2; l < N; ++l)
          y[l * N + i] = ((2.0 * l - 1.0) * mu[i] * y[(l - 1) * N + i] - (l - 1.0) * y[(l - 2) * N + i]) / l;
      } else {
        y[m * N + i] = -std::sqrt((1.0 - 1.0 / (2.0 * m)) * (1.0 - mu[i] * mu[i])) * y[(m - 1) * N + i];
        if (m + 1 < N) y[(m + 1) * N + i] = std::sqrt(2.0 * m + 1.0) * mu[i] * y[m * N + i];
        for (int l = m + 2; l < N; ++l) {
          const double tmp1 = std::sqrt(static_cast<double>((l - m) * (l + m)));
          const double tmp2 = std::sqrt(static_cast<double>((l - m - 1) * (l + m - 1)));
          y[l * N + i] = ((2.0 * l - 1.0) * mu[i] * y[(l - 1) * N + i] - tmp2 * y[(l - 2) * N + i]) / tmp1;
        }
      }
    }
    double* t = out.data() + (size_t)m * T;
    std::memcpy(t, base.data(), sizeof(double) * tab_ylm(N));
    for (int l = m; l < N; ++l)
      for (int i = 0; i < N; ++i) t[tab_ylm(N) + l * N + i] = y[l * N + i];
  }
  return true;
}

dsp_status get_mode_tables(dsp_context ctx, int N, const double** out) {
  auto it = ctx->mode_tables.find(N);
  if (it != ctx->mode_tables.end()) {
    *out = it->second;
    return DSP_OK;
  }
  std::vector<double> tab;
  if (!build_mode_tables(N, tab)) return fail(ctx, DSP_ERR_EIGEN, "Gauss quadrature did not converge");
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, tab.size() * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(mode tables)");
  e = cudaMemcpy(d, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpy(mode tables)");
  ctx->mode_tables[N] = d;
  *out = d;
  return DSP_OK;
}

// The azimuth quadrature of the bidirectional surface (DisortSolver.cpp:484-496):
// the 100-node Gauss rule on (0, 1) of the reference's gaussianQuadrature,
// mirrored to 200 nodes, [gmu 200 | gwt 200]; uploaded once per context.
dsp_status get_brdf_quadrature(dsp_context ctx, const double** out) {
  if (ctx->brdf_q) {
    *out = ctx->brdf_q;
    return DSP_OK;
  }
  const int n = 100;
  std::vector<double> q(400, 0.0);
  for (int i = 1; i <= n; ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (n + 0.5)), z1, pp;
    int iter = 0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (++iter > 10) return fail(ctx, DSP_ERR_EIGEN, "BRDF azimuth quadrature did not converge");
    } while (std::fabs(z - z1) > 3.0e-14);
    q[i - 1] = 0.5 * (1.0 + z);
    q[200 + i - 1] = 1.0 / ((1.0 - z * z) * pp * pp);
  }
  for (int i = 0; i < n; ++i) {
    q[n + i] = -q[i];
    q[200 + n + i] = q[200 + i];
  }
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, q.size() * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(BRDF quadrature)");
  e = cudaMemcpy(d, q.data(), q.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return cuda_fail(ctx, e, "cudaMemcpy(BRDF quadrature)");
  }
  ctx->brdf_q = d;
  *out = d;
  return DSP_OK;
}

// The mode-m layer and boundary-value launches of a chunk; JAC: their
// temperature-Jacobian forms (mode 0 with Jacobians asked for); SPH: with the
// pseudo-spherical beam, whose particular solution of the mode is formed
// between the two.
// Resident CTAs of a kernel on the whole GPU (persistent launches).
template <class K>
int resident_ctas(dsp_context ctx, K kernel, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * ctx->sm_count;
}

// `order`/`head` (persistent boundary-value launch): the chunk's slots by
// descending layer count and this mode's queue counter; null: one CTA or team
// per slot.
template <int N, bool JAC, bool SPH>
void launch_general_mode(dsp_context ctx, const FluxParams& p, long long layers, cudaStream_t s, const int* order,
                         int* head) {
  using LC = LCfg<N, true>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(flux_layer_kernel<N, true, JAC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)LC::smem_bytes());
    if constexpr (N > 16)
      cudaFuncSetAttribute(flux_bvp_tile_kernel<N, true, JAC, SPH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)TCfg<N>::smem_bytes());
    if constexpr (SPH)
      cudaFuncSetAttribute(flux_sph_source_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SCfg<N>::smem_bytes());
    attr = true;
  }
  if (layers > 0) {
    KernelTimer kt(ctx, "gen_layer_kernel");
    flux_layer_kernel<N, true, JAC><<<(unsigned)((layers + LC::TPC - 1) / LC::TPC), LC::CTA, LC::smem_bytes(), s>>>(p);
  }
  if constexpr (SPH) {
    if (layers > 0) {
      using C = SCfg<N>;
      KernelTimer kt(ctx, "gen_sph_source_kernel");
      flux_sph_source_kernel<N, true><<<(unsigned)((layers + C::WPC - 1) / C::WPC), 32 * C::WPC, C::smem_bytes(), s>>>(p);
    }
  }
  if constexpr (N <= 16) {
    using C = RCfg<N>;
    KernelTimer kt(ctx, "gen_bvp_kernel");
    const int slots = (p.n + C::TPC - 1) / C::TPC;
    if (order) {
      static const int cap = resident_ctas(ctx, gen_bvp_reg_persistent_kernel<N, JAC, SPH>, C::CTA, C::smem_bytes());
      gen_bvp_reg_persistent_kernel<N, JAC, SPH><<<slots < cap ? slots : cap, C::CTA, C::smem_bytes(), s>>>(p, order,
                                                                                                          head);
    } else {
      flux_bvp_reg_kernel<N, true, JAC, SPH><<<slots, C::CTA, C::smem_bytes(), s>>>(p);
    }
  } else {
    using C = TCfg<N>;
    KernelTimer kt(ctx, "gen_bvp_kernel");
    if (order) {
      static bool pattr = false;
      if (!pattr) {
        cudaFuncSetAttribute(gen_bvp_tile_persistent_kernel<N, JAC, SPH>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes());
        pattr = true;
      }
      static const int cap = resident_ctas(ctx, gen_bvp_tile_persistent_kernel<N, JAC, SPH>, C::CTA, C::smem_bytes());
      gen_bvp_tile_persistent_kernel<N, JAC, SPH><<<p.n < cap ? p.n : cap, C::CTA, C::smem_bytes(), s>>>(p, order,
                                                                                                        head);
    } else {
      flux_bvp_tile_kernel<N, true, JAC, SPH><<<p.n, C::CTA, C::smem_bytes(), s>>>(p);
    }
  }
}

template <int N, bool SPH>
dsp_status launch_general_chunk(dsp_context ctx, FluxParams p, long long layers, int maxm, const double* tabs,
                                const JacView* jv, const int* order, int* heads) {
  cudaStream_t s = ctx->stream;
  p.tables = tabs;
  {
    KernelTimer kt(ctx, "gen_setup_kernel");
    gen_setup_kernel<<<(p.n + 3) / 4, 128, 0, s>>>(p);
  }
  if constexpr (SPH) {
    // Chapman factors and the beam transmission through the spherical shells
    KernelTimer kt(ctx, "gen_sph_chapman_kernel");
    flux_sph_chapman_kernel<true><<<(p.n + 3) / 4, 128, 0, s>>>(p);
  }
  // Jacobian records only when there is a thermal source to differentiate
  const bool jrecs = jv && (p.flags & DSP_FLAG_THERMAL);
  for (int m = 0; m <= maxm; ++m) {
    p.g.m = m;
    p.tables = tabs + (size_t)m * tab_size(N);
    int* head = order ? heads + m : nullptr;
    if (p.g.brdf) {
      // the surface's Fourier coefficients of this mode, before the boundary-value problem
      KernelTimer kt(ctx, "gen_brdf_kernel");
      gen_brdf_kernel<N><<<p.n, 128, 0, s>>>(p);
    }
    if (m == 0 && jrecs) launch_general_mode<N, true, SPH>(ctx, p, layers, s, order, head);
    else launch_general_mode<N, false, SPH>(ctx, p, layers, s, order, head);
    if (m == 0 && jv) {
      // the Jacobians use the mode-0 elimination before the next mode replaces it
      using C = JCfg<N>;
      static bool attr = false;
      if (!attr) {
        cudaFuncSetAttribute(flux_jac_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)C::smem_bytes());
        attr = true;
      }
      KernelTimer kt(ctx, "gen_jac_kernel");
      flux_jac_kernel<N, true><<<p.n, C::KB, C::smem_bytes(), s>>>(p, *jv);
    }
    if (p.g.numu > 0) {
      KernelTimer kt(ctx, "gen_intensity_kernel");
      gen_intensity_kernel<N><<<(p.n + 3) / 4, 128, 0, s>>>(p);
    }
  }
  if ((p.flags & DSP_GFLAG_INTENSITY_CORR) && p.g.numu > 0) {
    // after the whole Fourier sum: the intensity corrections
    KernelTimer kt(ctx, "gen_intcor_kernel");
    gen_intcor_kernel<N><<<p.n, 128, 0, s>>>(p);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "general kernel launch");
  return DSP_OK;
}

template <int N>
dsp_status launch_general_n(dsp_context ctx, const FluxParams& p, long long layers, int maxm, const double* tabs,
                            const JacView* jv, const int* order, int* heads) {
  if (p.flags & DSP_FLAG_SPHERICAL_BEAM)
    return launch_general_chunk<N, true>(ctx, p, layers, maxm, tabs, jv, order, heads);
  return launch_general_chunk<N, false>(ctx, p, layers, maxm, tabs, jv, order, heads);
}

dsp_status launch_general(dsp_context ctx, int N, const FluxParams& p, long long layers, int maxm,
                          const double* tabs, const JacView* jv, const int* order, int* heads) {
  switch (N) {
    case 4: return launch_general_n<4>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 6: return launch_general_n<6>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 8: return launch_general_n<8>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 10: return launch_general_n<10>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 12: return launch_general_n<12>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 14: return launch_general_n<14>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 16: return launch_general_n<16>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 32: return launch_general_n<32>(ctx, p, layers, maxm, tabs, jv, order, heads);
    case 64: return launch_general_n<64>(ctx, p, layers, maxm, tabs, jv, order, heads);
  }
  return fail(ctx, DSP_ERR_UNSUPPORTED, "unsupported num_streams");
}

// Highest azimuth mode of an instance, as gen_setup_kernel decides it (host
// copy, used only to skip mode launches no instance of a chunk needs).
int host_naz(int N, uint32_t fl, bool do_int, double fbeam, double umu0, int numu_in, const double* um) {
  if (!do_int) return 0;
  const bool user_mu = (fl & DSP_GFLAG_USER_MU) != 0, only = (fl & DSP_GFLAG_ONLY_FLUXES) != 0;
  const int numu = (user_mu && !only) ? numu_in : N;
  auto at = [&](int k) { return (user_mu && !only && um && k < numu) ? um[k] : 0.0; };
  const bool indep = (fbeam == 0.0) || (std::fabs(1.0 - umu0) < 1.e-5) || only ||
                     (numu == 1 && std::fabs(1.0 - at(1)) < 1.e-5) || (numu == 1 && std::fabs(1.0 + at(1)) < 1.e-5) ||
                     (numu == 2 && std::fabs(1.0 + at(1)) < 1.e-5 && std::fabs(1.0 - at(2)) < 1.e-5);
  return indep ? 0 : N - 1;
}

// Instances the kernels do not take (num_streams outside the supported set)
// get NaN outputs, like every instance that fails validation.
__global__ void gen_fill_nan_kernel(const int* ids, int count, int ntau, int numu, int nphi, int ntau_out,
                                    int numu_out, double* const* flux, double* inten, double* iavg) {
  const int k = blockIdx.x;
  if (k >= count) return;
  const long long i = ids[k];
  const double qnan = __longlong_as_double(0x7ff8000000000000ll);
  for (int lu = threadIdx.x; lu < ntau; lu += blockDim.x) {
    for (int f = 0; f < 8; ++f) flux[f][i * ntau_out + lu] = qnan;
    for (int iu = 0; iu < numu; ++iu) {
      const long long o2 = (i * ntau_out + lu) * numu_out + iu;
      if (iavg) iavg[o2] = qnan;
      if (inten)
        for (int j = 0; j < nphi; ++j) inten[o2 * nphi + j] = qnan;
    }
  }
}

struct DevFlux {
  double* f[8];
};

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

dsp_status general_solve(dsp_context ctx, const dsp_general_batch* bin, const dsp_general_out* out,
                         const dsp_general_jac_out* jac);

}  // namespace

extern "C" dsp_status dsp_general_bands_solve(dsp_context ctx, const dsp_general_batch* bin,
                                              const dsp_general_out* out) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  NvtxRange r("dsp_general_bands_solve");
  if (bin && (bin->flags & DSP_FLAG_TEMPERATURE_JAC))
    return fail(ctx, DSP_ERR_UNSUPPORTED, "temperature Jacobians are computed by dsp_general_bands_solve_jac");
  return general_solve(ctx, bin, out, nullptr);
}

extern "C" dsp_status dsp_general_bands_solve_jac(dsp_context ctx, const dsp_general_batch* bin,
                                                  const dsp_general_out* out, const dsp_general_jac_out* jac) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  NvtxRange r("dsp_general_bands_solve_jac");
  if (!jac || !jac->flux_up || !jac->flux_down || !jac->mean_intensity || !jac->mean_intensity_down ||
      !jac->mean_intensity_up || !jac->flux_divergence)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "every Jacobian output array is required");
  return general_solve(ctx, bin, out, jac);
}

// ibcnd = Special (computeAlbTrans, DisortSolver.cpp:4025-4163) from two solves
// of the general path on the GPU: isotropic unit illumination from the top,
// then from the bottom, with a black surface, no other source and the user
// cosines mirrored to [-mu reversed | +mu] (DisortSolver.cpp:52-58, 852-865).
// The albedo of the medium is the upward intensity at the top under the top
// illumination; the transmissivity is the downward one at the bottom (one
// layer) or the upward one at the top under the bottom illumination; both
// include the boundary's own term, which is the reference's exp(-tau/mu).  The
// spherical albedo and transmissivity are the corresponding fluxes / pi
// (albTransSpherical, :4295-4358).
extern "C" dsp_status dsp_general_bands_albtrans(dsp_context ctx, const dsp_general_batch* bin,
                                                 const dsp_albtrans_out* out) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  NvtxRange r("dsp_general_bands_albtrans");
  if (!bin || !out || !out->albedo_medium || !out->transmissivity_medium || !out->spherical_albedo ||
      !out->spherical_transmissivity)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "null batch or albedo/transmissivity output");
  const dsp_general_batch& b = *bin;
  if (b.flags & DSP_FLAG_DEVICE_POINTERS)
    return fail(ctx, DSP_ERR_UNSUPPORTED, "dsp_general_bands_albtrans takes host pointers");
  const int n = b.n_inst;
  if (n < 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "n_inst must be >= 0");
  if (n == 0) return DSP_OK;
  if (!b.num_streams || !b.num_layers || !b.layer_offset)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "num_streams, num_layers and layer_offset are required");
  const bool user_mu = (b.flags & DSP_GFLAG_USER_MU) != 0;
  if (user_mu && (b.num_user_mu <= 0 || !b.mu_user.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "num_user_mu must be positive when use_user_mu=true");
  int maxL = 0;
  for (int i = 0; i < n; ++i) {
    maxL = std::max(maxL, b.num_layers[i]);
    if (!user_mu && b.num_streams[i] != b.num_streams[0])
      return fail(ctx, DSP_ERR_INVALID_INPUT, "without user angles every instance needs the same num_streams");
  }
  const int half = user_mu ? b.num_user_mu : b.num_streams[0] / 2;
  if (out->numu_out < half) return fail(ctx, DSP_ERR_INVALID_INPUT, "numu_out is smaller than the number of angles");
  // the mirrored cosines, shared or per instance
  const int nu2 = 2 * half;
  std::vector<double> umu2;
  const bool shared_mu = !user_mu || b.mu_user.stride == 0;
  const int nlist = shared_mu ? 1 : n;
  umu2.resize((size_t)nlist * nu2);
  for (int k = 0; k < nlist; ++k) {
    double* d = umu2.data() + (size_t)k * nu2;
    std::vector<double> pos(half);
    if (user_mu) {
      for (int iu = 0; iu < half; ++iu) pos[iu] = b.mu_user.ptr[b.mu_user.stride * k + iu];
    } else {
      std::vector<double> tab;
      if (!build_tables(b.num_streams[0], tab)) return fail(ctx, DSP_ERR_EIGEN, "Gauss quadrature did not converge");
      for (int iu = 0; iu < half; ++iu) pos[iu] = tab[tab_mu(b.num_streams[0]) + iu];
      std::sort(pos.begin(), pos.end());
    }
    for (int iu = 0; iu < half; ++iu) {
      d[half + iu] = pos[iu];
      d[iu] = -pos[half - 1 - iu];
    }
  }
  static const double one = 1.0, zero = 0.0, phi0 = 0.0;
  dsp_general_batch g = b;
  g.flags = (b.flags & (DSP_FLAG_DELTA_M_PLUS | DSP_FLAG_INDEX_FROM_BOTTOM)) | DSP_GFLAG_USER_MU;
  g.temperature = nullptr;
  g.level_altitudes = nullptr;
  g.num_user_tau = 0;
  g.tau_user = {nullptr, 0};
  g.num_user_mu = nu2;
  g.mu_user = {umu2.data(), shared_mu ? 0 : (int64_t)nu2};
  g.num_phi = 1;
  g.phi_user = {&phi0, 0};
  g.accuracy_fourier_series = 0.0;
  g.surface_albedo = {&zero, 0};
  g.direct_beam_flux = {&zero, 0};
  g.brdf_type = DSP_BRDF_LAMBERTIAN;
  g.num_phase_func_angles = 0;
  const int ntau = maxL + 1;
  const size_t nf = (size_t)n * ntau;
  std::vector<double> fl[2][8], iavg[2], inten(nf * nu2);
  std::vector<int32_t> st[2];
  const bool need_bot = maxL > 1;
  for (int pass = 0; pass < (need_bot ? 2 : 1); ++pass) {
    g.isotropic_flux_top = {pass == 0 ? &one : &zero, 0};
    g.isotropic_flux_bottom = {pass == 0 ? &zero : &one, 0};
    dsp_general_out o{};
    for (int f = 0; f < 8; ++f) {
      fl[pass][f].assign(nf, 0.0);
      o.flux[f] = fl[pass][f].data();
    }
    iavg[pass].assign(nf * nu2, 0.0);
    st[pass].assign(n, 0);
    o.intensity = inten.data();
    o.intensity_azimuth_avg = iavg[pass].data();
    o.status = st[pass].data();
    o.ntau_out = ntau;
    o.numu_out = nu2;
    const dsp_status e = general_solve(ctx, &g, &o, nullptr);
    if (e != DSP_OK) return e;
  }
  const bool ifb = (b.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  for (int i = 0; i < n; ++i) {
    const int L = b.num_layers[i];
    int32_t s0 = st[0][i];
    if (L > 1 && st[1][i] > s0) s0 = st[1][i];
    if (out->status) out->status[i] = s0;
    const size_t top = (size_t)i * ntau + (ifb ? L : 0), bot = (size_t)i * ntau + (ifb ? 0 : L);
    double* am = out->albedo_medium + (size_t)out->numu_out * i;
    double* tm = out->transmissivity_medium + (size_t)out->numu_out * i;
    for (int iu = 0; iu < half; ++iu) {
      // without user angles the reference orders the cosines as its quadrature
      // (descending); the solve above took them ascending
      const int up = user_mu ? half + iu : nu2 - 1 - iu, dn = user_mu ? half - 1 - iu : iu;
      am[iu] = iavg[0][top * nu2 + up];
      tm[iu] = L == 1 ? iavg[0][bot * nu2 + dn] : iavg[1][top * nu2 + up];
    }
    const double alb = b.surface_albedo.ptr ? b.surface_albedo.ptr[b.surface_albedo.stride * i] : 0.0;
    double sa = 0.0, stt = 0.0;
    if (alb > 0.0) {
      // FluxResult order: flux_down is [1], flux_up [2]
      const int pass = L == 1 ? 0 : 1;
      const double up = fl[pass][2][top] / M_PI, dn = fl[pass][1][bot] / M_PI;
      sa = L == 1 ? up : dn;
      stt = L == 1 ? dn : up;
      const double corr = alb / (1.0 - alb * sa);
      for (int iu = 0; iu < half; ++iu) {
        am[iu] += corr * stt * tm[iu];
        tm[iu] += corr * sa * tm[iu];
      }
    }
    out->spherical_albedo[i] = sa;
    out->spherical_transmissivity[i] = stt;
  }
  return DSP_OK;
}

namespace {

// The general solve behind both entry points; `jac` (may be null) adds the
// temperature Jacobians of mode 0.
dsp_status general_solve(dsp_context ctx, const dsp_general_batch* bin, const dsp_general_out* out,
                         const dsp_general_jac_out* jac) {
  if (!bin || !out) return fail(ctx, DSP_ERR_INVALID_INPUT, "null batch or output");
  const dsp_general_batch& b = *bin;
  const int n = b.n_inst;
  if (n < 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "n_inst must be >= 0");
  if (n == 0) return DSP_OK;
  const uint32_t fl = b.flags;
  if (fl & DSP_FLAG_HG_G)
    return fail(ctx, DSP_ERR_UNSUPPORTED, "the Henyey-Greenstein g fast path is a flux-batch option");
  const bool thermal = (fl & DSP_FLAG_THERMAL) != 0;
  const bool spherical = (fl & DSP_FLAG_SPHERICAL_BEAM) != 0;
  const bool user_tau = (fl & DSP_GFLAG_USER_TAU) != 0, user_mu = (fl & DSP_GFLAG_USER_MU) != 0;
  const bool only_fluxes = (fl & DSP_GFLAG_ONLY_FLUXES) != 0;
  const bool do_int = user_mu && !only_fluxes;
  const bool dev = (fl & DSP_FLAG_DEVICE_POINTERS) != 0;
  if (!b.num_streams || !b.num_layers || !b.layer_offset || !b.num_phase_func_moments || !b.delta_tau ||
      !b.single_scat_albedo || !b.phase_function_moments)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "num_streams, num_layers, layer_offset, num_phase_func_moments, "
                                            "delta_tau, single_scat_albedo and phase_function_moments are required");
  if (thermal && !b.temperature) return fail(ctx, DSP_ERR_INVALID_INPUT, "thermal emission needs temperature");
  if (spherical && (!b.level_altitudes || !b.bottom_radius.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "the spherical beam needs level_altitudes and bottom_radius");
  if (b.pmom_count < 1) return fail(ctx, DSP_ERR_INVALID_INPUT, "pmom_count must be >= 1");
  if (user_tau && (b.num_user_tau <= 0 || !b.tau_user.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "use_user_tau needs num_user_tau > 0 and tau_user");
  if (user_mu && (b.num_user_mu <= 0 || !b.mu_user.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "num_user_mu must be positive when use_user_mu=true");
  if (!only_fluxes && (b.num_phi <= 0 || !b.phi_user.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "num_phi must be positive when comp_only_fluxes=false");
  if (b.accuracy_fourier_series < 0.0)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "accuracy_fourier_series must be non-negative (0 = disabled)");
  const bool brdf = b.brdf_type != DSP_BRDF_LAMBERTIAN;
  if (b.brdf_type < DSP_BRDF_LAMBERTIAN || b.brdf_type > DSP_BRDF_HAPKE)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "bidirReflectivity: unknown BRDF type");
  if (brdf && !b.brdf_params.ptr)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "a bidirectional surface needs brdf_params");
  // the Buras-Emde correction reads the tabulated phase function
  const bool becorr = (fl & DSP_GFLAG_INTENSITY_CORR) && (fl & DSP_GFLAG_INTENSITY_CORR_BE) && do_int;
  const int na = becorr ? b.num_phase_func_angles : 0;
  if (becorr && (na < 2 || !b.mu_phase_function.ptr || !b.phase_function))
    return fail(ctx, DSP_ERR_INVALID_INPUT,
                "the Buras-Emde correction needs num_phase_func_angles >= 2, mu_phase_function and phase_function");
  for (int f = 0; f < 8; ++f)
    if (!out->flux[f]) return fail(ctx, DSP_ERR_INVALID_INPUT, "every flux output array is required");
  if (do_int && (!out->intensity || !out->intensity_azimuth_avg))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "intensity outputs are required when use_user_mu=true");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  cudaStream_t s = ctx->stream;
  dsp_status st;

  // ---- host view of the per-instance metadata -------------------------------
  std::vector<int32_t> hN(n), hL(n);
  std::vector<int64_t> hoff(n + 1);
  if (dev) {
    e = cudaMemcpyAsync(hN.data(), b.num_streams, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hL.data(), b.num_layers, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hoff.data(), b.layer_offset, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "metadata copy");
  } else {
    std::memcpy(hN.data(), b.num_streams, n * sizeof(int32_t));
    std::memcpy(hL.data(), b.num_layers, n * sizeof(int32_t));
    std::memcpy(hoff.data(), b.layer_offset, (n + 1) * sizeof(int64_t));
  }
  int maxN = 4, maxL = 0;
  for (int i = 0; i < n; ++i) {
    if (hL[i] > 0 && hoff[i + 1] - hoff[i] != hL[i])
      return fail(ctx, DSP_ERR_INVALID_INPUT, "layer_offset does not match num_layers");
    if (hN[i] > maxN && supported_nstr(hN[i])) maxN = hN[i];
    if (hL[i] > maxL) maxL = hL[i];
  }
  const int ntau_need = user_tau ? b.num_user_tau : maxL + 1;
  const int numu_eff = do_int ? b.num_user_mu : 0;
  if (out->ntau_out < ntau_need)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "ntau_out is smaller than the number of output levels");
  if (do_int && out->numu_out < b.num_user_mu)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "numu_out is smaller than num_user_mu");
  const int64_t total_layers = hoff[n];
  const int nphi = only_fluxes ? (b.num_phi > 0 ? b.num_phi : 0) : b.num_phi;
  const int64_t ntau_o = out->ntau_out, numu_o = out->numu_out;
  // Jacobian columns: the largest L + 2 (the replay's column stride), the output stride
  const int jdof = maxL + 2;
  if (jac && jac->ndof_out < jdof)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "ndof_out is smaller than num_layers + 2");
  const int64_t jdof_o = jac ? jac->ndof_out : 0;

  // ---- stage inputs --------------------------------------------------------
  static const double kDefaults[11] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0, 0.0};
  const dsp_darray* sc[11] = {&b.wavenumber_low, &b.wavenumber_high, &b.surface_albedo, &b.emissivity_top,
                              &b.direct_beam_flux, &b.direct_beam_mu, &b.direct_beam_phi, &b.isotropic_flux_top,
                              &b.isotropic_flux_bottom, &b.temperature_top, &b.temperature_bottom};
  const dsp_darray* lists[3] = {&b.tau_user, &b.mu_user, &b.phi_user};
  const int list_n[3] = {user_tau ? b.num_user_tau : 0, user_mu ? b.num_user_mu : 0, nphi};
  auto darray_elems = [&](const dsp_darray& a, int64_t per) -> size_t {
    return a.stride == 0 ? (size_t)per : (size_t)((n - 1) * a.stride + per);
  };
  const double* d_dtau;
  const double* d_ssa;
  const double* d_pmom;
  const double* d_temp = nullptr;
  const double* d_zalt = nullptr;
  dsp_darray d_rbot = b.bottom_radius;
  dsp_darray d_bpar = b.brdf_params;
  dsp_darray d_mup = b.mu_phase_function;
  const double* d_phasef = b.phase_function;
  const int32_t* d_L;
  const int64_t* d_off;
  const int32_t* d_nmom;
  dsp_darray dsc[11], dlists[3];
  {
    size_t need = 0;
    if (!dev) {
      need += align256(n * sizeof(int32_t)) * 2 + align256((n + 1) * sizeof(int64_t));
      need += align256(total_layers * sizeof(double)) * 2 + align256(total_layers * b.pmom_count * sizeof(double));
      if (thermal) need += align256((total_layers + n) * sizeof(double));
      if (spherical)
        need += align256((total_layers + n) * sizeof(double)) + align256(darray_elems(b.bottom_radius, 1) * sizeof(double));
      if (brdf) need += align256(darray_elems(b.brdf_params, DSP_BRDF_PARAMS) * sizeof(double));
      if (becorr)
        need += align256(darray_elems(b.mu_phase_function, na) * sizeof(double)) +
                align256((size_t)total_layers * na * sizeof(double));
      for (int k = 0; k < 3; ++k)
        if (lists[k]->ptr && list_n[k] > 0) need += align256(darray_elems(*lists[k], list_n[k]) * sizeof(double));
    }
    for (int k = 0; k < 11; ++k)
      need += (!sc[k]->ptr) ? 256 : (dev ? 0 : align256(darray_elems(*sc[k], 1) * sizeof(double)));
    if ((st = ensure(ctx, &ctx->stage_in, &ctx->stage_in_bytes, need + 256, "input staging")) != DSP_OK) return st;
    char* cur = static_cast<char*>(ctx->stage_in);
    auto put = [&](const void* src, size_t bytes) -> const void* {
      void* dst = cur;
      if (bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
      cur += align256(bytes);
      return dst;
    };
    e = cudaSuccess;
    if (dev) {
      d_L = b.num_layers;
      d_off = b.layer_offset;
      d_nmom = b.num_phase_func_moments;
      d_dtau = b.delta_tau;
      d_ssa = b.single_scat_albedo;
      d_pmom = b.phase_function_moments;
      d_temp = thermal ? b.temperature : nullptr;
      d_zalt = spherical ? b.level_altitudes : nullptr;
      for (int k = 0; k < 3; ++k) dlists[k] = *lists[k];
    } else {
      d_L = static_cast<const int32_t*>(put(b.num_layers, n * sizeof(int32_t)));
      d_off = static_cast<const int64_t*>(put(b.layer_offset, (n + 1) * sizeof(int64_t)));
      d_nmom = static_cast<const int32_t*>(put(b.num_phase_func_moments, n * sizeof(int32_t)));
      d_dtau = static_cast<const double*>(put(b.delta_tau, total_layers * sizeof(double)));
      d_ssa = static_cast<const double*>(put(b.single_scat_albedo, total_layers * sizeof(double)));
      d_pmom = static_cast<const double*>(put(b.phase_function_moments, total_layers * b.pmom_count * sizeof(double)));
      if (thermal) d_temp = static_cast<const double*>(put(b.temperature, (total_layers + n) * sizeof(double)));
      if (spherical) {
        d_zalt = static_cast<const double*>(put(b.level_altitudes, (total_layers + n) * sizeof(double)));
        d_rbot.ptr =
            static_cast<const double*>(put(b.bottom_radius.ptr, darray_elems(b.bottom_radius, 1) * sizeof(double)));
      }
      if (brdf)
        d_bpar.ptr = static_cast<const double*>(
            put(b.brdf_params.ptr, darray_elems(b.brdf_params, DSP_BRDF_PARAMS) * sizeof(double)));
      if (becorr) {
        d_mup.ptr = static_cast<const double*>(
            put(b.mu_phase_function.ptr, darray_elems(b.mu_phase_function, na) * sizeof(double)));
        d_phasef = static_cast<const double*>(put(b.phase_function, (size_t)total_layers * na * sizeof(double)));
      }
      for (int k = 0; k < 3; ++k) {
        dlists[k] = *lists[k];
        if (lists[k]->ptr && list_n[k] > 0)
          dlists[k].ptr = static_cast<const double*>(
              put(lists[k]->ptr, darray_elems(*lists[k], list_n[k]) * sizeof(double)));
      }
    }
    for (int k = 0; k < 11; ++k) {
      dsc[k] = *sc[k];
      if (!sc[k]->ptr) {  // absent scalar: the DisortConfig default
        dsc[k].ptr = static_cast<const double*>(put(&kDefaults[k], sizeof(double)));
        dsc[k].stride = 0;
      } else if (!dev) {
        dsc[k].ptr = static_cast<const double*>(put(sc[k]->ptr, darray_elems(*sc[k], 1) * sizeof(double)));
      }
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(input)");
  }

  // ---- outputs: zeroed, then written by the kernels -----------------------------
  const size_t flux_elems = (size_t)n * ntau_o;
  const size_t int_elems = (out->intensity && nphi > 0) ? (size_t)n * ntau_o * numu_o * nphi : 0;
  const size_t iavg_elems = out->intensity_azimuth_avg ? (size_t)n * ntau_o * numu_o : 0;
  double* dflux[8];
  double* dint = nullptr;
  double* diavg = nullptr;
  int32_t* dstatus = nullptr;
  const size_t jac_elems = jac ? (size_t)n * ntau_o * jdof_o : 0;
  double* djac[6] = {};
  double* const hjac[6] = {jac ? jac->flux_up : nullptr, jac ? jac->flux_down : nullptr,
                           jac ? jac->mean_intensity : nullptr, jac ? jac->mean_intensity_down : nullptr,
                           jac ? jac->mean_intensity_up : nullptr, jac ? jac->flux_divergence : nullptr};
  {
    const size_t need = (dev ? 0 : 8 * align256(flux_elems * 8) + align256(int_elems * 8) + align256(iavg_elems * 8) +
                                       6 * align256(jac_elems * 8)) +
                        2 * align256(n * sizeof(int32_t)) + align256(8 * sizeof(double*));
    if ((st = ensure(ctx, &ctx->stage_out, &ctx->stage_out_bytes, need, "output staging")) != DSP_OK) return st;
    char* cur = static_cast<char*>(ctx->stage_out);
    for (int f = 0; f < 8; ++f) {
      if (dev) dflux[f] = out->flux[f];
      else {
        dflux[f] = reinterpret_cast<double*>(cur);
        cur += align256(flux_elems * 8);
      }
    }
    if (dev) {
      dint = int_elems ? out->intensity : nullptr;
      diavg = iavg_elems ? out->intensity_azimuth_avg : nullptr;
    } else {
      if (int_elems) dint = reinterpret_cast<double*>(cur);
      cur += align256(int_elems * 8);
      if (iavg_elems) diavg = reinterpret_cast<double*>(cur);
      cur += align256(iavg_elems * 8);
    }
    for (int f = 0; f < 6 && jac; ++f) {
      if (dev) djac[f] = hjac[f];
      else {
        djac[f] = reinterpret_cast<double*>(cur);
        cur += align256(jac_elems * 8);
      }
    }
    dstatus = (dev && out->status) ? out->status : reinterpret_cast<int32_t*>(cur);
    cur += align256(n * sizeof(int32_t));
    double** dfp = reinterpret_cast<double**>(cur);
    cur += align256(8 * sizeof(double*));
    int32_t* dskip = reinterpret_cast<int32_t*>(cur);
    e = cudaMemcpyAsync(dfp, dflux, sizeof(dflux), cudaMemcpyHostToDevice, s);
    for (int f = 0; f < 8 && e == cudaSuccess; ++f) e = cudaMemsetAsync(dflux[f], 0, flux_elems * 8, s);
    if (e == cudaSuccess && dint) e = cudaMemsetAsync(dint, 0, int_elems * 8, s);
    if (e == cudaSuccess && diavg) e = cudaMemsetAsync(diavg, 0, iavg_elems * 8, s);
    for (int f = 0; f < 6 && jac && e == cudaSuccess; ++f) e = cudaMemsetAsync(djac[f], 0, jac_elems * 8, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "output initialisation");

    // status: 0, or the verdict on instances no kernel takes
    std::vector<int32_t> hst(n, 0);
    std::vector<int32_t> skip;
    for (int i = 0; i < n; ++i) {
      if (hN[i] < 4 || hN[i] % 2 != 0) hst[i] = DSP_ERR_INVALID_INPUT;
      else if (!supported_nstr(hN[i])) hst[i] = DSP_ERR_UNSUPPORTED;
      if (hst[i]) skip.push_back(i);
    }
    e = cudaMemcpyAsync(dstatus, hst.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // hst leaves scope
    if (e != cudaSuccess) return cuda_fail(ctx, e, "status initialisation");
    if (!skip.empty()) {
      e = cudaMemcpyAsync(dskip, skip.data(), skip.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) {
        gen_fill_nan_kernel<<<(unsigned)skip.size(), 64, 0, s>>>(dskip, (int)skip.size(), (int)ntau_need,
                                                                  numu_eff, nphi, (int)ntau_o, (int)numu_o, dfp,
                                                                  dint, diavg);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // skip leaves scope
      if (e != cudaSuccess) return cuda_fail(ctx, e, "unsupported-instance fill");
    }
  }

  // ---- groups by stream count, chunks by workspace --------------------------------
  struct Chunk {
    int N;
    std::vector<int32_t> ids;
    std::vector<int64_t> inst_off, lay_off;
    int64_t inst_doubles = 0, layers = 0;
    int64_t surf_doubles = 0;  // bidirectional surface tables, one per slot
    int64_t be_doubles = 0;    // Buras-Emde tables, one per slot (all of one NT)
    int maxm = 0;
    // persistent boundary-value launches: the slots by descending layer count
    std::vector<int32_t> order;
  };
  std::vector<Chunk> chunks;
  size_t budget = workspace_budget();
  {
    size_t freeb = 0, totalb = 0;
    if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && freeb / 2 < budget + ctx->ws_bytes)
      budget = (freeb + ctx->ws_bytes) / 2;
  }
  const double* h_fbeam = (!dev && b.direct_beam_flux.ptr) ? b.direct_beam_flux.ptr : nullptr;
  const double* h_umu0 = (!dev && b.direct_beam_mu.ptr) ? b.direct_beam_mu.ptr : nullptr;
  const double* h_mu = (!dev && user_mu) ? b.mu_user.ptr : nullptr;
  // with Jacobians of a thermal solve, per layer: P/Q, multiplier records and
  // the replayed right-hand side values [N][jdof]
  const bool jrecs = jac && thermal;
  auto jac_per_layer = [&](int N) -> int64_t {
    return jrecs ? (int64_t)jpq_stride(N) + jrec_stride(N) + (int64_t)N * jdof : 0;
  };
  // with the pseudo-spherical beam: the spherical record of every layer
  auto sph_per_layer = [&](int N) -> int64_t { return spherical ? (int64_t)sph_stride(N) : 0; };
  for (int N : kSupported) {
    const int64_t lstride = glrec_stride(N, numu_eff);
    const int64_t per_layer = lstride + brec_stride(N) + N + sph_per_layer(N) + jac_per_layer(N);
    Chunk c;
    c.N = N;
    size_t bytes = 0;
    auto flush = [&]() {
      if (!c.ids.empty()) {
        c.lay_off.push_back(c.layers);
        chunks.push_back(std::move(c));
      }
      c = Chunk();
      c.N = N;
      bytes = 0;
    };
    for (int i = 0; i < n; ++i) {
      if (hN[i] != N) continue;
      const int L = hL[i] > 0 ? hL[i] : 0;
      const int NT = user_tau ? b.num_user_tau : L + 1;
      const int64_t rec = GenLayout::make(L, N, NT).stride + (brdf ? brdf_stride(N, numu_eff) : 0) +
                          (becorr ? becor_stride(ntau_need, na) : 0);
      const size_t ib = (size_t)(rec + (int64_t)L * per_layer) * sizeof(double);
      if (!c.ids.empty() && bytes + ib > budget) flush();
      c.ids.push_back(i);
      c.inst_off.push_back(c.inst_doubles);
      c.lay_off.push_back(c.layers);
      c.inst_doubles += GenLayout::make(L, N, NT).stride;
      if (brdf) c.surf_doubles += brdf_stride(N, numu_eff);
      if (becorr) c.be_doubles += becor_stride(ntau_need, na);
      c.layers += L;
      bytes += ib;
      int naz = N - 1;
      if (!dev)
        naz = host_naz(N, fl, do_int, h_fbeam ? h_fbeam[b.direct_beam_flux.stride * i] : 0.0,
                       h_umu0 ? h_umu0[b.direct_beam_mu.stride * i] : 0.5, b.num_user_mu,
                       h_mu ? h_mu + b.mu_user.stride * i : nullptr);
      else if (!do_int) naz = 0;
      if (naz > c.maxm) c.maxm = naz;
    }
    flush();
  }
  if (chunks.empty()) goto copy_back;
  // the size-class queue of each chunk the schedule runs persistently
  for (Chunk& c : chunks) {
    const int meanL = c.ids.empty() ? 0 : (int)(c.layers / (int64_t)c.ids.size());
    if (find_schedule(ctx, c.N, meanL).persistent != 1) continue;
    c.order.resize(c.ids.size());
    for (size_t k = 0; k < c.ids.size(); ++k) c.order[k] = (int32_t)k;
    std::stable_sort(c.order.begin(), c.order.end(),
                     [&](int32_t a, int32_t b) { return hL[c.ids[a]] > hL[c.ids[b]]; });
  }
  {
    // chunk index arrays, one upload
    size_t meta_need = 0, ws_need = 0;
    for (const Chunk& c : chunks) {
      meta_need += align256(c.ids.size() * 4) + align256(c.ids.size() * 8) + align256((c.ids.size() + 1) * 8) +
                   align256(c.layers * 4) + align256(c.order.size() * 4) + align256((c.maxm + 1) * 4);
      const int64_t lstride = glrec_stride(c.N, numu_eff);
      const size_t w =
          (size_t)(c.inst_doubles + c.surf_doubles + c.be_doubles +
                   c.layers * (lstride + brec_stride(c.N) + c.N + sph_per_layer(c.N) + jac_per_layer(c.N))) *
          sizeof(double);
      if (w > ws_need) ws_need = w;
    }
    if ((st = ensure(ctx, &ctx->meta, &ctx->meta_bytes, meta_need, "chunk index")) != DSP_OK) return st;
    if ((st = ensure(ctx, &ctx->ws, &ctx->ws_bytes, ws_need + 1024, "workspace")) != DSP_OK) return st;
    std::vector<char> hmeta(meta_need);
    std::vector<size_t> moff(chunks.size());
    {
      size_t o = 0;
      for (size_t k = 0; k < chunks.size(); ++k) {
        const Chunk& c = chunks[k];
        moff[k] = o;
        const size_t nc = c.ids.size();
        std::memcpy(hmeta.data() + o, c.ids.data(), nc * 4);
        o += align256(nc * 4);
        std::memcpy(hmeta.data() + o, c.inst_off.data(), nc * 8);
        o += align256(nc * 8);
        std::memcpy(hmeta.data() + o, c.lay_off.data(), (nc + 1) * 8);
        o += align256((nc + 1) * 8);
        int32_t* li = reinterpret_cast<int32_t*>(hmeta.data() + o);
        for (size_t ci = 0; ci < nc; ++ci)
          for (int64_t l = c.lay_off[ci]; l < c.lay_off[ci + 1]; ++l) li[l] = (int32_t)ci;
        o += align256(c.layers * 4);
        if (!c.order.empty()) std::memcpy(hmeta.data() + o, c.order.data(), c.order.size() * 4);
        o += align256(c.order.size() * 4);
        o += align256((c.maxm + 1) * 4);  // queue counters, one per mode, zero
      }
    }
    e = cudaMemcpyAsync(ctx->meta, hmeta.data(), meta_need, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // hmeta leaves scope
    if (e != cudaSuccess) return cuda_fail(ctx, e, "chunk index upload");

    FluxParams p;
    std::memset(&p, 0, sizeof(p));
    p.pc = b.pmom_count;
    p.flags = fl;
    p.pk = planck_consts();
    p.status = dstatus;
    DArr* pa[11] = {&p.wlo, &p.whi, &p.alb, &p.emis, &p.fbeam, &p.umu0, &p.g.phi0, &p.fisot, &p.fisob, &p.ttop, &p.tbot};
    for (int k = 0; k < 11; ++k) {
      pa[k]->p = dsc[k].ptr;
      pa[k]->s = dsc[k].stride;
    }
    GenView& g = p.g;
    g.numu = numu_eff;
    g.numu_in = user_mu ? b.num_user_mu : 0;
    g.nphi = nphi;
    g.ntau_out = (int)ntau_o;
    g.numu_out = (int)numu_o;
    g.user_tau = user_tau ? b.num_user_tau : 0;
    g.accur = b.accuracy_fourier_series;
    g.Ls = d_L;
    g.in_off = reinterpret_cast<const long long*>(d_off);
    g.nmoms = d_nmom;
    g.dtau = d_dtau;
    g.ssa = d_ssa;
    g.pmom = d_pmom;
    g.temp = d_temp;
    g.zalt = d_zalt;
    p.rbot.p = d_rbot.ptr;
    p.rbot.s = d_rbot.stride;
    g.utau = {dlists[0].ptr, dlists[0].stride};
    g.umu = {dlists[1].ptr, dlists[1].stride};
    g.phi = {dlists[2].ptr, dlists[2].stride};
    for (int f = 0; f < 8; ++f) g.out_flux[f] = dflux[f];
    g.out_int = dint;
    g.out_iavg = diavg;
    g.brdf_type = b.brdf_type;
    g.brdf_par.p = brdf ? d_bpar.ptr : nullptr;
    g.brdf_par.s = d_bpar.stride;
    g.brdf_q = nullptr;
    if (brdf && (st = get_brdf_quadrature(ctx, &g.brdf_q)) != DSP_OK) return st;
    g.nangles = na;
    g.mup.p = becorr ? d_mup.ptr : nullptr;
    g.mup.s = d_mup.stride;
    g.phasef = becorr ? d_phasef : nullptr;
    g.becor_ld = becor_stride(ntau_need, na);
    for (size_t k = 0; k < chunks.size(); ++k) {
      const Chunk& c = chunks[k];
      const size_t nc = c.ids.size();
      char* mb = static_cast<char*>(ctx->meta) + moff[k];
      g.ids = reinterpret_cast<const int*>(mb);
      mb += align256(nc * 4);
      g.inst_off = reinterpret_cast<const long long*>(mb);
      mb += align256(nc * 8);
      g.lay_off = reinterpret_cast<const long long*>(mb);
      mb += align256((nc + 1) * 8);
      g.layer_inst = reinterpret_cast<const int*>(mb);
      mb += align256(c.layers * 4);
      const int* order = c.order.empty() ? nullptr : reinterpret_cast<const int*>(mb);
      mb += align256(c.order.size() * 4);
      int* heads = reinterpret_cast<int*>(mb);
      g.lstride = glrec_stride(c.N, numu_eff);
      p.n = (int)nc;
      p.N = c.N;
      double* w = static_cast<double*>(ctx->ws);
      p.inst_rec = w;
      p.layer_rec = w + c.inst_doubles;
      p.bvp_rec = p.layer_rec + c.layers * g.lstride;
      g.cc = p.bvp_rec + c.layers * brec_stride(c.N);
      // after the solution coefficients: the spherical records
      p.sph = spherical ? g.cc + c.layers * c.N : nullptr;
      JacView jv;
      if (jac) {
        // then P/Q, multipliers, replayed values
        double* jb = g.cc + c.layers * (c.N + sph_per_layer(c.N));
        p.jac_pq = jrecs ? jb : nullptr;
        p.jac_rec = jrecs ? jb + c.layers * jpq_stride(c.N) : nullptr;
        jv.cv = jrecs ? p.jac_rec + c.layers * jrec_stride(c.N) : nullptr;
        jv.ndof = jdof;
        jv.ndof_out = (int)jdof_o;
        for (int f = 0; f < 6; ++f) jv.out[f] = djac[f];
      }
      // after every per-layer area: the surface tables of the chunk's slots
      double* const wend = static_cast<double*>(ctx->ws) + c.inst_doubles +
                           c.layers * (g.lstride + brec_stride(c.N) + c.N + sph_per_layer(c.N) + jac_per_layer(c.N));
      g.brdf = brdf ? wend : nullptr;
      g.becor = becorr ? wend + c.surf_doubles : nullptr;
      const double* tabs = nullptr;
      if ((st = get_mode_tables(ctx, c.N, &tabs)) != DSP_OK) return st;
      if (ctx->debug & DSP_DEBUG_POISON_SCRATCH) {
        const size_t wb = (size_t)(c.inst_doubles + c.surf_doubles + c.be_doubles +
                                   c.layers * (g.lstride + brec_stride(c.N) + c.N + sph_per_layer(c.N) +
                                               jac_per_layer(c.N))) *
                          sizeof(double);
        e = cudaMemsetAsync(ctx->ws, 0xFF, wb, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "scratch poison");
      }
      if ((st = launch_general(ctx, c.N, p, c.layers, c.maxm, tabs, jac ? &jv : nullptr, order, heads)) != DSP_OK)
        return st;
    }
  }

copy_back:
  if (dev) return DSP_OK;
  for (int f = 0; f < 8; ++f) {
    e = cudaMemcpyAsync(out->flux[f], dflux[f], flux_elems * 8, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(output)");
  }
  if (dint) {
    e = cudaMemcpyAsync(out->intensity, dint, int_elems * 8, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(intensity)");
  }
  if (diavg) {
    e = cudaMemcpyAsync(out->intensity_azimuth_avg, diavg, iavg_elems * 8, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(intensity_azimuth_avg)");
  }
  for (int f = 0; f < 6 && jac; ++f) {
    e = cudaMemcpyAsync(hjac[f], djac[f], jac_elems * 8, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(jacobian)");
  }
  std::vector<int32_t> hs_tmp;
  int32_t* hs = out->status;
  if (!hs) {
    hs_tmp.resize(n);
    hs = hs_tmp.data();
  }
  e = cudaMemcpyAsync(hs, dstatus, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(status)");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "general solve");
  return DSP_OK;
}

}  // namespace
