// dsp_device.cuh — shared device-side definitions of the B200 DISORT engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dsp.h"

// Phase markers for cycle-count instrumentation builds; no-ops otherwise.
#ifndef DSP_PHASE_BEGIN
#define DSP_PHASE_BEGIN
#endif
#ifndef DSP_PHASE
#define DSP_PHASE(k)
#endif
#ifndef DSP_PHASE_END
#define DSP_PHASE_END
#endif

namespace dsp {

__host__ __device__ constexpr int pow2ceil(int x) { return x <= 1 ? 1 : 2 * pow2ceil((x + 1) / 2); }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int round4(int x) { return (x + 3) & ~3; }

struct DArr {
  const double* p;
  long long s;
  __device__ __forceinline__ double operator()(long long i, long long k = 0) const { return p[i * s + k]; }
  __device__ __forceinline__ const double* row(long long i) const { return p + i * s; }
};

// Constants of the reference's Planck routine, computed on the host with libm
// exactly as Planck.cpp:18-31 does, so the device uses bit-identical values.
struct PlanckConsts {
  double vmax, sigdpi, conc, c1;
};

// Per-stream-count constant tables (host-computed, FluxSolver.cpp:257-290, :126,
// :442-445): mu[N], wt[N], dsim[NN], dinv[NN], ylm[N][N] = P_l(mu_i) at [l*N+i].
struct Tables {
  const double* base;
  __device__ __forceinline__ const double* mu() const { return base; }
};
__host__ __device__ constexpr int tab_mu(int) { return 0; }
__host__ __device__ constexpr int tab_wt(int N) { return N; }
__host__ __device__ constexpr int tab_dsim(int N) { return 2 * N; }
__host__ __device__ constexpr int tab_dinv(int N) { return 2 * N + N / 2; }
__host__ __device__ constexpr int tab_ylm(int N) { return 3 * N; }
__host__ __device__ constexpr int tab_size(int N) { return 3 * N + N * N; }

// Instance record (doubles) written by the setup kernel.
struct InstLayout {
  int hdr, dtau_s, ssa_s, fsc, sig, mode, tau_s, tauc, btr, pkag, yb, stride;
  __host__ __device__ static InstLayout make(int L, int N) {
    InstLayout o;
    o.hdr = 0;
    o.dtau_s = 16;
    o.ssa_s = o.dtau_s + L;
    o.fsc = o.ssa_s + L;
    o.sig = o.fsc + L;
    o.mode = o.sig + L;
    o.tau_s = o.mode + L;
    o.tauc = o.tau_s + L + 1;
    o.btr = o.tauc + L + 1;
    o.pkag = o.btr + L + 1;
    o.yb = o.pkag + L + 1;
    o.stride = round4(o.yb + N + 1);
    return o;
  }
};
// header slots (the general solver also uses H_NAZ .. H_NT)
enum { H_NCUT = 0, H_LYRCUT, H_PTOP, H_PBOT, H_PBOTD, H_DELTAM, H_DMPLUS, H_FBEAM, H_UMU0, H_ALB,
       H_FISOT, H_FISOB, H_NAZ, H_KCONV, H_DONE, H_NT, H_NSLOTS };
static_assert(H_NSLOTS <= 16, "instance header is 16 doubles");

// General-solver instance record: the InstLayout fields for (L, N), then the
// output optical depths utau[NT], their scaled values utaus[NT] and the layer
// of each, lyr[NT] (NT = user taus, or L + 1 levels).
struct GenLayout {
  InstLayout il;
  int utau, utaus, lyr, stride;
  __host__ __device__ static GenLayout make(int L, int N, int NT) {
    GenLayout g;
    g.il = InstLayout::make(L, N);
    g.utau = g.il.stride;
    g.utaus = g.utau + NT;
    g.lyr = g.utaus + NT;
    g.stride = round4(g.lyr + NT);
    return g;
  }
};

// Layer record (doubles) written by the layer kernel:
// G[N][N] | eig[N] | zb[N] | z0[N] | z1[N] | xr0 | xr1
__host__ __device__ constexpr int lrec_G(int) { return 0; }
__host__ __device__ constexpr int lrec_eig(int N) { return N * N; }
__host__ __device__ constexpr int lrec_zb(int N) { return N * N + N; }
__host__ __device__ constexpr int lrec_z0(int N) { return N * N + 2 * N; }
__host__ __device__ constexpr int lrec_z1(int N) { return N * N + 3 * N; }
__host__ __device__ constexpr int lrec_xr(int N) { return N * N + 4 * N; }
__host__ __device__ constexpr int lrec_stride(int N) { return round4(N * N + 4 * N + 2); }
// Elimination record (doubles) written by the BVP kernels, per layer: the N
// pivot rows [U | V | c] of U x_l + V x_{l+1} = c and the pivot reciprocals.
// N <= 16: rows of 2N + 2 ([U | V | c | 1/pivot]); N >= 32: rows of 2N + 1
// ([U | V | c]), then 1 / pivot [N].
__host__ __device__ constexpr int brec_stride(int N) { return round4(N * (2 * N + 2)); }

// Pseudo-spherical beam record of the flux path, per layer: the slope Z1 of the
// beam particular solution Z(tau) = exp(-xba tau) (Z0 + Z1 tau) (Z0 is the layer
// record's zb), its attenuation xba, and the layer's Chapman factor
// (computeBeamSourceSpherical, FluxSolver.cpp:650-738; :391-419).
__host__ __device__ constexpr int sph_stride(int N) { return round4(N + 2); }
__host__ __device__ constexpr int sph_xba(int N) { return N; }
__host__ __device__ constexpr int sph_ch(int N) { return N + 1; }

// Temperature-Jacobian records of the flux path (compute_temperature_jacobian).
// Per layer, written by the layer stage: P[NN] | Q[NN], the thermal particular
// solution per unit Planck intercept and slope: with P and Q the solution of
// computeIsotropicSource is Z1 = xr1 P / 2 in both hemispheres and
// Z0 = (xr0 P +/- xr1 Q) / 2 (z0's upper / lower hemisphere order), so the
// derivatives with respect to a layer's top and bottom level Planck values
// (FluxSolver.cpp:789-829) follow from the derivatives of xr0 and xr1.
__host__ __device__ constexpr int jpq_stride(int N) { return N; }
// Per layer, written by the boundary-value kernels: the multiplier applied to
// every panel slot at every pivot column, [N][3N/2] (0 where the slot was not a
// candidate or the column was skipped as singular), then the pivot slot of each
// column [N] (as doubles).  Together with the pivot rows of the elimination
// record they replay the band LU on further right-hand sides.
__host__ __device__ constexpr int jrec_stride(int N) { return round4(N * (3 * (N / 2)) + N); }

// General-solver layer record: the flux layer record, then the eigenvectors
// and sources at the user polar angles of the current mode:
// GU[numu][N] | zbu[numu] | z0u[numu] | z1u[numu]
__host__ __device__ constexpr int glrec_gu(int N) { return lrec_stride(N); }
__host__ __device__ constexpr int glrec_stride(int N, int numu) { return round4(lrec_stride(N) + numu * (N + 3)); }

// Per-launch view of a general (DisortSolver) chunk.  Instances are addressed by
// chunk slot ci; ids[ci] is the batch index (inputs, outputs, status).
struct GenView {
  int m;                       // azimuth mode of this launch
  int numu;                    // user polar angles (0: no intensities)
  int numu_in;                 // num_user_mu of the batch (validated when use_user_mu)
  int nphi, ntau_out, numu_out;
  int user_tau;                // number of user optical depths (0: the L + 1 levels)
  double accur;
  const int* ids;              // [n] batch instance of each slot
  const long long* inst_off;   // [n] instance record offsets (doubles)
  const long long* lay_off;    // [n+1] chunk-local first layer of each slot
  const int* layer_inst;       // [layers] slot of each chunk-local layer
  const int* Ls;               // batch num_layers
  const long long* in_off;     // batch layer_offset (CSR)
  const int* nmoms;            // batch num_phase_func_moments
  const double *dtau, *ssa, *pmom, *temp;  // CSR inputs
  const double* zalt;          // level altitudes, laid out like temp (pseudo-spherical beam only)
  DArr utau, umu, phi, phi0;
  long long lstride;           // layer record stride (glrec_stride)
  double* cc;                  // [layers][N] boundary-value solution of the mode
  double* out_flux[8];         // [batch][ntau_out]
  double* out_int;             // [batch][ntau_out][numu_out][nphi]
  double* out_iavg;            // [batch][ntau_out][numu_out]
  // bidirectional surface (brdf_type != 0): the model's parameters per batch
  // instance, the 200-node azimuth quadrature [gmu | gwt], and per chunk slot
  // the mode's surface table (brdf_stride doubles, written by gen_brdf_kernel)
  int brdf_type;
  DArr brdf_par;
  const double* brdf_q;
  double* brdf;
  // Buras-Emde intensity correction: the tabulated phase function and, per
  // chunk slot, its residual-phase tables (becor_stride doubles)
  int nangles;
  DArr mup;
  const double* phasef;  // [batch layers][nangles], CSR like dtau
  double* becor;
  long long becor_ld;    // doubles per slot: becor_stride of the batch's largest NT
};

// Per-slot tables of the Buras-Emde correction for NT output depths
// (applyNewIntensityCorrection / prepDoubleScatIntegr, DisortSolver.cpp:3568-3640,
// 3812-3876): the residual phase function P''[NT][na], the integration grid
// mu_eq[NT][nf] and its signs [NT][nf], and the normalisation [NT].
constexpr int BE_NF = 100;
__host__ __device__ constexpr long long becor_stride(int NT, int na) {
  return ((long long)NT * (na + 2 * BE_NF + 1) + 3) & ~3ll;
}

// Surface table of one chunk slot for the current azimuth mode
// (computeSurfaceBidir, DisortSolver.cpp:2582-2708): rows r = 0..NN-1 are the
// quadrature angles, r = NN + iu the user polar angles; each row holds
// [beam reflectance | diffuse reflectance of incoming stream 0..NN-1 |
//  directional emissivity (mode 0) | the intensity kernel's reflected-field sum].
// After the rows, kept across the modes: the beam reflectance at each user angle
// for every mode run, [numu][N] (zero for modes not run), which the BRDF
// intensity correction sums (DisortSolver.cpp:306-313, 3783-3787).
__host__ __device__ constexpr int brdf_row(int N) { return N / 2 + 3; }
__host__ __device__ constexpr int brdf_beam_modes(int N, int numu) { return (N / 2 + numu) * brdf_row(N); }
__host__ __device__ constexpr int brdf_stride(int N, int numu) {
  return round4(brdf_beam_modes(N, numu) + numu * N);
}

struct FluxParams {
  int n;          // instances in this launch
  int N, L, pc, nmom;
  uint32_t flags;
  DArr wlo, whi, dtau, ssa, pmom, temp, alb, emis, fbeam, umu0, fisot, fisob, ttop, tbot, zalt, rbot;
  const double* tables;  // tab_* layout for N
  PlanckConsts pk;
  double* inst_rec;
  double* layer_rec;
  double* bvp_rec;
  InstLayout il;
  double* out[8];
  int32_t* status;
  GenView g;  // general-solver launches only
  double* sph = nullptr;      // [n][L][sph_stride], general: [layers][sph_stride] (pseudo-spherical beam only)
  double* jac_pq = nullptr;   // [n][L][jpq_stride] (temperature-Jacobian launches only)
  double* jac_rec = nullptr;  // [n][L][jrec_stride] (temperature-Jacobian launches only)
};

// The temperature-Jacobian launch of a flux chunk: the right-hand side values
// of the replayed elimination, per instance [L][N][ndof], and the six outputs
// [batch][L+1][ndof] (already offset to the chunk's first instance).
struct JacView {
  int ndof;         // flux path: L + 2 degrees of freedom (level temperatures 0..L,
                    // surface); general path: the largest L + 2 of the batch
  double* cv;       // [n][L][N][ndof] (general path: [chunk layers][N][ndof])
  double* out[6];   // flux_up, flux_down, mean_intensity, _down, _up, flux_divergence
  int ndof_out;     // general path: column stride of out (>= L + 2 of every instance)
};

// P_l^m(x) for l = m..lmax into y[l * stride] (rows l < m set to 0), the
// recurrence of Legendre.cpp:67-120.  For m > 0 the reference seeds P_m^m with
// the value its previous-mode call left in row m-1; that chain is the product
// below, evaluated in the same order.
__device__ __forceinline__ void legendre_column(int m, double x, int lmax, double* y, int stride) {
  for (int l = 0; l < m && l <= lmax; ++l) y[l * stride] = 0.0;
  if (m == 0) {
    y[0] = 1.0;
    if (lmax >= 1) y[stride] = x;
    double y2 = 1.0, y1 = x;
    for (int l = 2; l <= lmax; ++l) {
      const double v = ((2.0 * l - 1.0) * x * y1 - (l - 1.0) * y2) / l;
      y[l * stride] = v;
      y2 = y1;
      y1 = v;
    }
    return;
  }
  double pmm = 1.0;
  for (int k = 1; k <= m; ++k) pmm = -sqrt((1.0 - 1.0 / (2.0 * k)) * (1.0 - x * x)) * pmm;
  if (m <= lmax) y[m * stride] = pmm;
  const double pm1 = sqrt(2.0 * m + 1.0) * x * pmm;
  if (m + 1 <= lmax) y[(m + 1) * stride] = pm1;
  double y2 = pmm, y1 = pm1;
  for (int l = m + 2; l <= lmax; ++l) {
    const double tmp1 = sqrt(static_cast<double>((l - m) * (l + m)));
    const double tmp2 = sqrt(static_cast<double>((l - m - 1) * (l + m - 1)));
    const double v = ((2.0 * l - 1.0) * x * y1 - tmp2 * y2) / tmp1;
    y[l * stride] = v;
    y2 = y1;
    y1 = v;
  }
}

// Team helpers.  A team is TEAM consecutive threads; TEAM < 32 lives inside a
// warp (synchronised by __syncwarp on its own lanes), TEAM >= 32 is the whole CTA.
template <int TEAM>
__device__ __forceinline__ unsigned team_mask() {
  if constexpr (TEAM >= 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << TEAM) - 1u) << (lane & ~(unsigned)(TEAM - 1));
  }
}

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if constexpr (TEAM >= 32) {
    __syncthreads();
  } else {
    __syncwarp(team_mask<TEAM>());
  }
}

// Arg-max of (v, i) over the team, ties to the smaller index; result to all.
// `red` is team-private shared scratch of 2*(TEAM/32) doubles (unused for TEAM <= 32).
template <int TEAM>
__device__ __forceinline__ void team_argmax(double& v, int& idx, double* red) {
  constexpr int W = TEAM < 32 ? TEAM : 32;
  const unsigned m = team_mask<TEAM>();
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) {
    const double ov = __shfl_xor_sync(m, v, off, W);
    const int oi = __shfl_xor_sync(m, idx, off, W);
    if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
  }
  if constexpr (TEAM > 32) {
    constexpr int NW = TEAM / 32;
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
      red[w] = v;
      reinterpret_cast<int*>(red + NW)[w] = idx;
    }
    __syncthreads();
    v = red[0];
    idx = reinterpret_cast<int*>(red + NW)[0];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
      const double ov = red[k];
      const int oi = reinterpret_cast<int*>(red + NW)[k];
      if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
    __syncthreads();
  }
}

// Arg-max of a >= 0 over the candidate lanes of a full warp, ties to the lowest
// lane; 32 when no lane is a candidate.  Non-negative doubles order like their
// bit patterns, so the maximum is two 32-bit warp reductions (high words, then
// the low words of the lanes that tie on the high word) and the winner is the
// lowest lane of the ballot of exact matches.  `zero` reports a maximum of 0.
// 1/x without branches: the hardware approximation (rcp.approx.ftz.f64)
// refined by two Newton-Raphson steps y <- y + y (1 - x y), each about doubling
// the correct bits (Muller et al., Handbook of Floating-Point Arithmetic, 2nd
// ed., section 4.7); within an ulp or two of 1/x for normal x.  Subnormal x
// flush to zero (result +-inf); the pivots it serves are never that small in a
// solvable system.
__device__ __forceinline__ double rcp_newton(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

__device__ __forceinline__ int warp_argmax_nonneg(double a, bool cand, bool& zero) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(a));
  const unsigned hi = cand ? static_cast<unsigned>(b >> 32) : 0u;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const bool tie = cand && hi == mhi;
  const unsigned lo = tie ? static_cast<unsigned>(b) : 0u;
  const unsigned mlo = __reduce_max_sync(0xffffffffu, lo);
  const unsigned win = __ballot_sync(0xffffffffu, tie && static_cast<unsigned>(b) == mlo);
  zero = (mhi | mlo) == 0u;
  return win ? __ffs(win) - 1 : 32;
}

// Team copy of nd doubles from global to shared memory: 16-byte cp.async
// (LDGSTS) chunks when both ends are 16-byte aligned and nd is even, plain
// loads and stores otherwise.  The copies are waited for with cp_async_wait
// and made visible to the team by the next team barrier.  Plain (coherent)
// loads: the source may have been written by this kernel.
template <int TEAM>
__device__ __forceinline__ void team_copy_async(double* dst, const double* src, int nd, int t) {
  const bool al = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15u) == 0 && (nd & 1) == 0;
  if (al) {
    const unsigned s0 = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    for (int k = t; k < nd / 2; k += TEAM)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s0 + 16u * k), "l"(src + 2 * k) : "memory");
  } else {
    for (int k = t; k < nd; k += TEAM) dst[k] = src[k];
  }
}
// Team copy of `rows` rows of `cols` doubles (cols even) from global memory
// (row stride sstride) into shared memory (row stride dstride), 16-byte cp.async
// chunks when both layouts keep every chunk 16-byte aligned, plain loads and
// stores otherwise; waited for like team_copy_async.
template <int TEAM>
__device__ __forceinline__ void team_copy_rows_async(double* dst, int dstride, const double* src, int sstride,
                                                     int rows, int cols, int t) {
  const bool al = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15u) == 0 &&
                  ((dstride | sstride | cols) & 1) == 0;
  const int cpr = cols / 2;
  if (al) {
    const unsigned s0 = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    for (int k = t; k < rows * cpr; k += TEAM) {
      const int r = k / cpr, c2 = k - r * cpr;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s0 + 8u * (unsigned)(r * dstride + 2 * c2)),
                   "l"(src + (long long)r * sstride + 2 * c2)
                   : "memory");
    }
  } else {
    for (int k = t; k < rows * cols; k += TEAM) {
      const int r = k / cols, c = k - r * cols;
      dst[r * dstride + c] = src[(long long)r * sstride + c];
    }
  }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's most recent groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void set_status(int32_t* status, int i, int code) {
  if (status) atomicMax(status + i, code);
}

}  // namespace dsp
