// flux_sph.cuh — the pseudo-spherical beam of the flux path (use_spherical_beam).
//
// Replaces the spherical branches of disortSet (Chapman factors and beam
// transmission, FluxSolver.cpp:391-419 with chapmanImpl :1503-1566) and
// computeBeamSourceSpherical (:650-738).  Two launches between the setup
// kernel and the boundary-value kernel of a flux chunk:
//  - flux_sph_chapman_kernel, one warp per instance, lanes over layers: the
//    slant depths at each layer's top and middle through the spherical shells,
//    the Chapman factor ch = tau_mid / slant_mid and the transmission
//    exp(-slant) at each level, over the layers of the absorption loop;
//  - flux_sph_source_kernel, one warp per layer: the particular solution
//    Z(tau) = exp(-xba tau) (Z0 + Z1 tau) of a source linear in tau after
//    removing the attenuation xba = 1 / ch, from the N x N system
//    I + xba M - C, assembled in shared memory and factored with partial
//    pivoting as the reference does (with its dithering of xba near a
//    quadrature angle or a near-singular system).
// Z0 replaces the layer record's plane-parallel zb; Z1, xba and ch go to the
// layer's spherical record (sph_stride).
// The general solver (DisortSolver.cpp:740-790, 1396-1530) runs the same two
// kernels in their GEN form: the Chapman factors once per chunk after its
// setup, the particular solution once per azimuth mode after the layer kernel.
#pragma once

#include "dsp_device.cuh"

namespace dsp {

// chapmanImpl (FluxSolver.cpp:1503-1566): slant optical depth from the top to a
// point tau_frac of the way up from the bottom of layer lc (1-based); zd(j) is
// the altitude of level j, dt(j) the optical depth of layer j (1-based).
template <class ZD, class DT>
__device__ double chapman_slant(int lc, double tau_frac, ZD zd, DT dt, int num_layers, double r, double mu0) {
  constexpr double PI = 3.14159265358979323846;
  const double DEG = PI / 180.0;
  const double zenang = acos(mu0) * 180.0 / PI;
  const double zenrad = zenang * DEG;
  const double xp = r + zd(lc) + (zd(lc - 1) - zd(lc)) * tau_frac;
  const double xpsinz = xp * sin(zenrad);
  if (zenang > 90.0 && xpsinz < r) return 1.0e+20;
  int id = lc;
  if (zenang > 90.0)
    for (int j = lc; j <= num_layers; ++j)
      if (xpsinz < (zd(j - 1) + r) && xpsinz >= (zd(j) + r)) id = j;
  double sum = 0.0;
  for (int j = 1; j <= id; ++j) {
    double fact = 1.0, fact2 = 1.0;
    if (j > lc) fact = 2.0;
    else if (j == lc && lc == id && zenang > 90.0) fact2 = -1.0;
    const double rj = r + zd(j - 1);
    double rjp1 = r + zd(j);
    if (j == lc && id == lc) rjp1 = xp;
    const double dhj = zd(j - 1) - zd(j);
    double dsj;
    if (id > lc && j == id) dsj = sqrt(rj * rj - xpsinz * xpsinz);
    else dsj = sqrt(rj * rj - xpsinz * xpsinz) - fact2 * sqrt(rjp1 * rjp1 - xpsinz * xpsinz);
    sum += dt(j) * fact * dsj / dhj;
  }
  if (id > lc) {
    const double dhj = zd(lc - 1) - zd(lc);
    const double dsj = sqrt(xp * xp - xpsinz * xpsinz) - sqrt((zd(lc) + r) * (zd(lc) + r) - xpsinz * xpsinz);
    sum += dt(lc) * dsj / dhj;
  }
  return sum;
}

// One warp per instance (4 per CTA).  GEN: the general solver's chunk
// addressing (ragged layers; one spherical record per layer task of the chunk;
// level altitudes laid out like the level temperatures).
template <bool GEN = false>
__global__ void __launch_bounds__(128) flux_sph_chapman_kernel(FluxParams p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = blockIdx.x * 4 + warp;
  if (slot >= p.n) return;
  int i, L;
  double* rec;
  InstLayout il;
  const double* zin;
  double* sph0;
  if constexpr (GEN) {
    i = p.g.ids[slot];
    L = p.g.Ls[i];
    il = InstLayout::make(L, p.N);
    rec = p.inst_rec + p.g.inst_off[slot];
    zin = p.g.zalt + p.g.in_off[i] + i;
    sph0 = p.sph + p.g.lay_off[slot] * sph_stride(p.N);
  } else {
    i = slot;
    L = p.L;
    il = p.il;
    rec = p.inst_rec + (long long)i * p.il.stride;
    zin = p.zalt.row(i);
    sph0 = p.sph + (long long)i * L * sph_stride(p.N);
  }
  if (p.status && p.status[i] == DSP_ERR_INVALID_INPUT) return;
  const int N = p.N;
  const double fbeam = rec[H_FBEAM], mu0 = rec[H_UMU0];
  if (!(fbeam > 0.0)) return;
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  const double r = p.rbot(i);
  const double* dts = rec + il.dtau_s;
  const double* taus = rec + il.tau_s;
  // the layers of the absorption loop (FluxSolver.cpp:312-331; DisortSolver.cpp:
  // 749-790): the transmission is computed down to that cut even without a
  // layer cut
  int ncut_abs = L;
  if (lane == 0) {
    double abstau = 0.0;
    for (int lc = 0; lc < L; ++lc) {
      if (abstau < 10.0) ncut_abs = lc + 1;
      const int lin = ifb ? L - 1 - lc : lc;
      const double w = GEN ? p.g.ssa[p.g.in_off[i] + lin] : p.ssa.row(i)[lin];
      const double d = GEN ? p.g.dtau[p.g.in_off[i] + lin] : p.dtau.row(i)[lin];
      abstau += (1.0 - w) * d;
    }
  }
  ncut_abs = __shfl_sync(0xffffffffu, ncut_abs, 0);
  auto zd = [&](int j) { return zin[ifb ? L - j : j]; };
  auto dt = [&](int j) { return dts[j - 1]; };
  for (int lc = lane; lc < L; lc += 32) {
    double* sr = sph0 + (long long)lc * sph_stride(N);
    if (lc < ncut_abs) {
      const double taup_mid = taus[lc] + dts[lc] / 2.0;
      const double chtau_mid = chapman_slant(lc + 1, 0.5, zd, dt, L, r, mu0);
      sr[sph_ch(N)] = taup_mid / chtau_mid;
      rec[il.btr + lc + 1] = exp(-chapman_slant(lc + 1, 0.0, zd, dt, L, r, mu0));
    } else {
      sr[sph_ch(N)] = 0.0;  // as on a freshly constructed reference solver
    }
  }
}

template <int N>
struct SCfg {
  static constexpr int NN = N / 2;
  static constexpr int WPC = 4;             // layer tasks (warps) per CTA
  static constexpr int LDA = N + 1;         // padded row stride of the system
  // per warp (doubles): A[N][LDA], gl[N], zj[N], b[N], z1[N], piv[N] (as ints in doubles)
  static constexpr int O_A = 0, O_GL = N * LDA, O_ZJ = O_GL + N, O_B = O_ZJ + N, O_Z1 = O_B + N,
                       O_PIV = O_Z1 + N, WARP_SMEM = round4(O_PIV + N);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)WPC * WARP_SMEM; }
};

// GEN: one azimuth mode of the general solver (P_l^m tables of the mode; the
// source coefficients zj, with the (2 - delta_m0) factor, are read from the
// particular-solution slot where the layer kernel left them).
template <int N, bool GEN = false>
__global__ void __launch_bounds__(128) flux_sph_source_kernel(FluxParams p) {
  using C = SCfg<N>;
  constexpr int NN = C::NN, LDA = C::LDA;
  constexpr double PI = 3.14159265358979323846;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long task = (long long)blockIdx.x * C::WPC + warp;
  int i, lc, Lin;
  const double* rec;
  InstLayout il;
  double* lrec;
  const double* pml;
  if constexpr (GEN) {
    if (task >= p.g.lay_off[p.n]) return;
    const int ci = p.g.layer_inst[task];
    i = p.g.ids[ci];
    lc = (int)(task - p.g.lay_off[ci]);
    Lin = p.g.Ls[i];
    il = InstLayout::make(Lin, N);
    rec = p.inst_rec + p.g.inst_off[ci];
    lrec = p.layer_rec + task * p.g.lstride;
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? Lin - 1 - lc : lc;
    pml = p.g.pmom + (p.g.in_off[i] + lin) * (long long)p.pc;
  } else {
    if (task >= (long long)p.n * p.L) return;
    i = (int)(task / p.L);
    lc = (int)(task % p.L);
    Lin = p.L;
    il = p.il;
    rec = p.inst_rec + (long long)i * p.il.stride;
    lrec = p.layer_rec + task * lrec_stride(N);
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? p.L - 1 - lc : lc;
    pml = p.pmom.row(i) + (long long)lin * p.pc;
  }
  if (p.status && p.status[i] == DSP_ERR_INVALID_INPUT) return;
  const double fbeam = rec[H_FBEAM];
  if (!(fbeam > 0.0) || lc >= (int)rec[H_NCUT]) return;
  if constexpr (GEN) {
    if (p.g.m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  }
  double* sm = smem + warp * C::WARP_SMEM;
  double* A = sm + C::O_A;
  double* gl = sm + C::O_GL;
  double* zj = sm + C::O_ZJ;
  double* bv = sm + C::O_B;
  double* z1 = sm + C::O_Z1;
  int* piv = reinterpret_cast<int*>(sm + C::O_PIV);
  const double* mu = p.tables + tab_mu(N);
  const double* Y = p.tables + tab_ylm(N);  // Y[l * N + i] = P_l^m(mu_i)
  const double* taus = rec + il.tau_s;
  const double* btr = rec + il.btr;
  double* sr = p.sph + task * sph_stride(N);

  // scaled phase coefficients g'_k (disortSet, FluxSolver.cpp:336-386;
  // DisortSolver.cpp:663-747, where P_0 is normalised to 1)
  {
    const double ws = rec[il.ssa_s + lc];
    const int mode = (int)rec[il.mode + lc];
    const double f = rec[il.fsc + lc], sig = rec[il.sig + lc];
    for (int k = lane; k < N; k += 32) {
      const double pk = (GEN && k == 0) ? 1.0 : pml[k];
      double g;
      if (mode == 0) g = (2.0 * k + 1.0) * ws * pk;
      else if (mode == 1) g = (2.0 * k + 1.0) * ws * (pk - f) / (1.0 - f);
      else {
        const double kd = (double)k;
        g = (2.0 * k + 1.0) * ws * (pk - f * exp(-kd * kd / (2.0 * sig))) / (1.0 - f);
      }
      gl[k] = g;
    }
  }
  __syncwarp();
  // source coefficients zj (FluxSolver.cpp:660-667) and the phase matrix C:
  // rows iq < NN from the quadrature sums, the other half by symmetry
  if constexpr (GEN) {
    for (int iq = lane; iq < NN; iq += 32) {
      zj[iq] = lrec[lrec_zb(N) + NN + iq];
      zj[NN + iq] = lrec[lrec_zb(N) + NN - 1 - iq];
    }
  } else {
    const double* yb = rec + il.yb;
    for (int iq = lane; iq < N; iq += 32) {
      double s = 0.0;
      for (int k = 0; k < N; ++k) s += gl[k] * Y[k * N + iq] * yb[k];
      zj[iq] = fbeam * s / (4.0 * PI);
    }
  }
  const double* wt = p.tables + tab_wt(N);
  for (int e = lane; e < NN * N; e += 32) {
    const int iq = e / N, jq = e % N;
    double s = 0.0;
    for (int l = 0; l < N; ++l) s += (gl[l] * Y[l * N + iq]) * Y[l * N + jq];
    const double c = (s * 0.5) * wt[jq];
    A[iq * LDA + jq] = -c;
    if (jq < NN) A[(NN + iq) * LDA + NN + jq] = -c;
    else A[(NN + iq) * LDA + jq - NN] = -c;
  }
  __syncwarp();
  // attenuation xba = 1 / ch with the reference's guards and dithering
  const double big = sqrt(1.79769313486231570815e+308) / 1.0e10;
  double xba = 1.0 / sr[sph_ch(N)];
  if (fabs(xba) > big && taus[lc + 1] > 1.0) xba = 0.0;
  if (fabs(xba * taus[lc + 1]) > log(big)) xba = 0.0;
  if (fabs(xba) > 1.0e-5)
    for (int iq = 0; iq < NN; ++iq)
      if (fabs((fabs(xba) - 1.0 / mu[iq]) / xba) < 0.05) {
        xba *= 1.001;
        break;
      }
  // Frobenius norm of I + xba M - C (its reciprocal is the reference's
  // conditioning estimate, FluxSolver.cpp:707-718)
  double fro = 0.0;
  for (int e = lane; e < N * N; e += 32) {
    const int r = e / N, c = e % N;
    const double v = A[r * LDA + c] + (r == c ? 1.0 + xba * mu[r] : 0.0);
    fro += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
  if (1.0 / sqrt(fro) < 1.0e-4) {
    if (xba == 0.0) xba = 5.0e-9;
    xba *= 1.00000005;
  }
  for (int r = lane; r < N; r += 32) A[r * LDA + r] += 1.0 + xba * mu[r];
  // linear-in-tau source after removing the attenuation
  const double q0a = btr[lc], q2a = btr[lc + 1];
  const double deltat = taus[lc + 1] - taus[lc];
  for (int iq = lane; iq < N; iq += 32) {
    const double q0 = q0a * zj[iq], q2 = q2a * zj[iq];
    const double x1 = (q2 * exp(xba * taus[lc + 1]) - q0 * exp(xba * taus[lc])) / deltat;
    z1[iq] = x1;
    bv[iq] = q0 * exp(xba * taus[lc]) - x1 * taus[lc];
  }
  __syncwarp();
  // LU with partial pivoting (row swaps; ties keep the first row)
  for (int k = 0; k < N; ++k) {
    double best = -1.0;
    int bi = k;
    for (int r = k + lane; r < N; r += 32) {
      const double v = fabs(A[r * LDA + k]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) piv[k] = bi;
    if (bi != k)
      for (int c = lane; c < N; c += 32) {
        const double t = A[k * LDA + c];
        A[k * LDA + c] = A[bi * LDA + c];
        A[bi * LDA + c] = t;
      }
    __syncwarp();
    const double akk = A[k * LDA + k];
    if (akk != 0.0)
      for (int r = k + 1 + lane; r < N; r += 32) {
        const double lik = A[r * LDA + k] / akk;
        A[r * LDA + k] = lik;
        for (int c = k + 1; c < N; ++c) A[r * LDA + c] -= lik * A[k * LDA + c];
      }
    __syncwarp();
  }
  // Z1 = A^{-1} xb1, then Z0 = A^{-1} (xb0 + mu Z1), in lane 0
  if (lane == 0) {
    auto solve = [&](double* b) {
      for (int k = 0; k < N; ++k)
        if (piv[k] != k) {
          const double t = b[k];
          b[k] = b[piv[k]];
          b[piv[k]] = t;
        }
      for (int r = 1; r < N; ++r) {
        double s = b[r];
        for (int c = 0; c < r; ++c) s -= A[r * LDA + c] * b[c];
        b[r] = s;
      }
      for (int r = N - 1; r >= 0; --r) {
        double s = b[r];
        for (int c = r + 1; c < N; ++c) s -= A[r * LDA + c] * b[c];
        b[r] = s / A[r * LDA + r];
      }
    };
    solve(z1);
    for (int iq = 0; iq < N; ++iq) bv[iq] += mu[iq] * z1[iq];
    solve(bv);
  }
  __syncwarp();
  for (int iq = lane; iq < NN; iq += 32) {
    lrec[lrec_zb(N) + NN + iq] = bv[iq];
    lrec[lrec_zb(N) + NN - 1 - iq] = bv[iq + NN];
    sr[NN + iq] = z1[iq];
    sr[NN - 1 - iq] = z1[iq + NN];
  }
  if (lane == 0) sr[sph_xba(N)] = xba;
}

}  // namespace dsp
