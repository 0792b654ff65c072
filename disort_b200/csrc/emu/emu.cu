// emu.cu — libdsp_emu.so: the flux emulator's MLP on the tcgen05 tensor cores.
//
// Training step (batch B, layers i = 1..nl, H_0 = X):
//   forward   Z_i = H_{i-1} W_i^T + b_i,  H_i = GELU(Z_i)  (last layer: P = Z_nl)
//   loss      sum over heads h of w_mh * mean_k (P_mhk - Y_mk)^2, averaged over m
//             (the gradient); the reported epoch loss is the same sum with the
//             82 outputs summed rather than averaged
//   backward  dZ_nl from the loss (fused into the output GEMM's epilogue),
//             dW_i = dZ_i^T H_{i-1},  dZ_{i-1} = (dZ_i W_i) * GELU'(Z_{i-1}),
//             db_i = column sums of dZ_i
//   update    fused Adam on FP32 master weights, writing the BF16 copies W_i and
//             W_i^T the next step's GEMMs read.
// Every GEMM is C = A B^T with K-major BF16 operands (tc_gemm.cuh); the
// transposed operands of the backward GEMMs (H_i^T, dZ_i^T, X^T) are written by
// the producing epilogues, so no GEMM needs an MN-major operand.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../../include/dsp_emu.h"
#include "tc_gemm.cuh"

using bf16 = __nv_bfloat16;
using namespace dsp_tc;

namespace {

constexpr int STAGES = 4;
constexpr int DW_SPLITS = 8;

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---------------------------------------------------------------- epilogues
struct EpiStore {  // C = acc
  float* C;
  int M, N;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (col0 + j < N) C[(long long)row * N + col0 + j] = v[j];
  }
};

struct EpiStoreBias {  // C = acc + b, columns < N only
  float* C;
  const float* bias;
  int M, N;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (col0 + j < N) C[(long long)row * N + col0 + j] = v[j] + bias[col0 + j];
  }
};

struct EpiHidden {  // Z = acc + b; H = GELU(Z); optional Z (FP32) and H^T
  const float* bias;
  float* Z;
  bf16* H;
  bf16* Ht;
  int M, N;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
    float z[16];
    __align__(16) bf16 h[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      z[j] = v[j] + bias[col0 + j];
      h[j] = __float2bfloat16(gelu_f(z[j]));
    }
    const long long o = (long long)row * N + col0;
    if (Z) {
#pragma unroll
      for (int j = 0; j < 16; j += 4)
        *reinterpret_cast<float4*>(Z + o + j) = make_float4(z[j], z[j + 1], z[j + 2], z[j + 3]);
    }
    *reinterpret_cast<uint4*>(H + o) = *reinterpret_cast<const uint4*>(h);
    *reinterpret_cast<uint4*>(H + o + 8) = *reinterpret_cast<const uint4*>(h + 8);
    if (Ht) {
#pragma unroll
      for (int j = 0; j < 16; ++j) Ht[(long long)(col0 + j) * M + row] = h[j];
    }
  }
};

struct EpiOut {  // P = acc + b; training: dZ = dLoss/dP (BF16, and transposed), loss sum
  const float* bias;
  float* P;
  const float* Y;   // [M][nout]
  const float* hw;  // [M][nheads] or null
  bf16* dZ;
  bf16* dZt;
  float* loss;
  int M, N, nout, nheads;
  float gscale;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
    float lsum = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int n = col0 + j;
      if (n >= N) continue;
      const float p = v[j] + bias[n];
      if (P) P[(long long)row * N + n] = p;
      if (dZ) {
        float g = 0.0f;
        if (n < nheads * nout) {
          const int h = n / nout, k = n - h * nout;
          const float d = p - Y[(long long)row * nout + k];
          const float w = hw ? hw[(long long)row * nheads + h] : 1.0f;
          g = gscale * w * d;
          lsum += w * d * d;
        }
        const bf16 gb = __float2bfloat16(g);
        dZ[(long long)row * N + n] = gb;
        dZt[(long long)n * M + row] = gb;
      }
    }
    if (dZ && loss) {
      // one atomic per warp when the whole warp holds rows (training batches are
      // multiples of 128 rows); otherwise one per thread
      if (__activemask() == 0xffffffffu) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum);
      } else {
        atomicAdd(loss, lsum);
      }
    }
  }
};

struct EpiBwdX {  // dZ_prev = acc * GELU'(Z_prev), BF16 and transposed
  const float* Zp;
  bf16* dZ;
  bf16* dZt;
  int M, N;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
    const long long o = (long long)row * N + col0;
    __align__(16) bf16 g[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) g[j] = __float2bfloat16(v[j] * gelu_grad_f(Zp[o + j]));
    *reinterpret_cast<uint4*>(dZ + o) = *reinterpret_cast<const uint4*>(g);
    *reinterpret_cast<uint4*>(dZ + o + 8) = *reinterpret_cast<const uint4*>(g + 8);
#pragma unroll
    for (int j = 0; j < 16; ++j) dZt[(long long)(col0 + j) * M + row] = g[j];
  }
};

struct EpiDW {  // dW += acc (split-K partial sums)
  float* dW;
  int M, N;
  __device__ void apply(int row, int col0, const float (&v)[16], int) const {
    if (row >= M) return;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (col0 + j < N) atomicAdd(dW + (long long)row * N + col0 + j, v[j]);
  }
};

// ---------------------------------------------------------------- small kernels
__global__ void gather_rows_kernel(const bf16* X, const float* Y, const float* HW, const int64_t* perm, bf16* Xp,
                                   float* Yp, float* HWp, int64_t n, int in_pad, int nout, int nheads) {
  const int64_t r = blockIdx.x;
  if (r >= n) return;
  const int64_t src = perm[r];
  const uint4* xs = reinterpret_cast<const uint4*>(X + src * in_pad);
  uint4* xd = reinterpret_cast<uint4*>(Xp + r * in_pad);
  for (int k = threadIdx.x; k < in_pad / 8; k += blockDim.x) xd[k] = xs[k];
  for (int k = threadIdx.x; k < nout; k += blockDim.x) Yp[r * nout + k] = Y[src * nout + k];
  if (HW)
    for (int k = threadIdx.x; k < nheads; k += blockDim.x) HWp[r * nheads + k] = HW[src * nheads + k];
}

// dst[c][r] = src[r][c] for an R x C BF16 block (32 x 32 tiles)
__global__ void transpose_bf16_kernel(const bf16* src, bf16* dst, int R, int C) {
  __shared__ bf16 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < R && c < C) t[k][threadIdx.x] = src[(long long)r * C + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < R && c < C) dst[(long long)c * R + r] = t[threadIdx.x][k];
  }
}

// db[n] = sum_m dZt[n][m]: one warp per n
__global__ void bias_grad_kernel(const bf16* dZt, float* db, int N, int M) {
  const int n = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = lane; m < M; m += 32) s += __bfloat162float(dZt[(long long)n * M + m]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) db[n] = s;
}

// Adam on FP32 masters [rows][cols]; entries outside [rows_real) x [cols_real)
// are padding and stay zero.  Writes the BF16 copy (and its transpose).
__global__ void adam_kernel(float* W, float* m, float* v, const float* g, bf16* Wb, bf16* Wt, int rows, int cols,
                            int rows_real, int cols_real, float lr, float bc1, float bc2) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)rows * cols) return;
  const int r = (int)(idx / cols), c = (int)(idx % cols);
  float w = W[idx];
  if (r < rows_real && c < cols_real) {
    const float gi = g[idx];
    const float mi = 0.9f * m[idx] + 0.1f * gi;
    const float vi = 0.999f * v[idx] + 0.001f * gi * gi;
    m[idx] = mi;
    v[idx] = vi;
    w -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    W[idx] = w;
  }
  if (Wb) Wb[idx] = __float2bfloat16(w);
  if (Wt) Wt[(long long)c * rows + r] = __float2bfloat16(w);
}

__global__ void to_bf16_kernel(const float* W, bf16* Wb, bf16* Wt, int rows, int cols) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)rows * cols) return;
  const int r = (int)(idx / cols), c = (int)(idx % cols);
  const bf16 b = __float2bfloat16(W[idx]);
  Wb[idx] = b;
  if (Wt) Wt[(long long)c * rows + r] = b;
}

// gate: one warp per row
__global__ void gate_kernel(const float* raw, int raw_stride, int n_in, const float* lo, const float* hi,
                            const float* preds, int pstride, int nout, const float* mu, const float* sd,
                            const float* scale, const float* add, float eps, float rel_tol, float floor_frac,
                            int64_t rows, float* flux, int32_t* fallback, int32_t* idx, int32_t* count) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (r >= rows) return;
  bool out = false;
  for (int f = lane; f < n_in; f += 32) {
    const float x = raw[r * raw_stride + f];
    if (!(x >= lo[f] && x <= hi[f])) out = true;
  }
  out = __any_sync(0xffffffffu, out);
  const float sc = scale ? scale[r] : 1.0f;
  auto head = [&](int h, int k) {
    const float a = add ? add[r * nout + k] : 0.0f;
    return sc * (expf(preds[r * pstride + h * nout + k] * sd[k] + mu[k]) - eps) + a;
  };
  float fmax_ = 0.0f, dmax = 0.0f;
  for (int k = lane; k < nout; k += 32) {
    const float fm = 0.5f * (head(0, k) + head(1, k));
    flux[r * nout + k] = fm;
    fmax_ = fmaxf(fmax_, fabsf(fm));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) fmax_ = fmaxf(fmax_, __shfl_xor_sync(0xffffffffu, fmax_, off));
  const float fl = floor_frac * fmax_;
  for (int k = lane; k < nout; k += 32) {
    const float f0 = head(0, k), f1 = head(1, k);
    const float fm = 0.5f * (f0 + f1);
    dmax = fmaxf(dmax, fabsf(f0 - f1) / fmaxf(fabsf(fm), fl));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
  const bool fb = out || !(dmax <= rel_tol);
  if (lane == 0) {
    fallback[r] = fb ? 1 : 0;
    if (fb) idx[atomicAdd(count, 1)] = (int32_t)r;
  }
}

// ---------------------------------------------------------------- tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// BF16 row-major [rows][cols] (cols a multiple of 8, base 16-byte aligned),
// 64-column x box_rows boxes with the 128-byte swizzle.
bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || (cols % 8) != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int bn_for(int n) { return (n % 128 == 0) ? 128 : 64; }

template <int BN, class Epi>
cudaError_t launch_gemm_bn(const CUtensorMap& A, const CUtensorMap& B, int a_row0, int b_row0, int M, int N, int K,
                           int splits, const Epi& epi, int* err, cudaStream_t s) {
  using C = GemmCfg<BN, STAGES>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc_gemm_tn_kernel<BN, STAGES, Epi>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes());
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int kt = (K + 63) / 64;
  const int per = (kt + splits - 1) / splits;
  dim3 grid((M + 127) / 128, (N + BN - 1) / BN, splits);
  tc_gemm_tn_kernel<BN, STAGES, Epi><<<grid, 128, C::smem_bytes(), s>>>(A, B, a_row0, b_row0, kt, per, epi, err);
  return cudaGetLastError();
}

template <class Epi>
cudaError_t launch_gemm(const CUtensorMap& A, const CUtensorMap& B, int a_row0, int b_row0, int M, int N, int K,
                        int splits, const Epi& epi, int* err, cudaStream_t s) {
  if (bn_for(N) == 128) return launch_gemm_bn<128>(A, B, a_row0, b_row0, M, N, K, splits, epi, err, s);
  return launch_gemm_bn<64>(A, B, a_row0, b_row0, M, N, K, splits, epi, err, s);
}

inline int pad64(int x) { return (x + 63) / 64 * 64; }

struct Layer {
  int in_pad = 0, out_pad = 0, in_real = 0, out_real = 0;
  float *W = nullptr, *b = nullptr, *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr, *dW = nullptr,
        *db = nullptr;
  bf16 *Wb = nullptr, *Wt = nullptr;
  CUtensorMap mapW, mapWt;
};

}  // namespace

struct dsp_emu_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  dsp_emu_config cfg{};
  int in_pad = 0, out_pad = 0, hid = 0, nl = 0, B = 0;
  std::vector<Layer> L;
  std::vector<void*> allocs;
  // training activations (batch B); index i: output of layer i (0-based), i < nl-1 hidden
  std::vector<float*> Z;
  std::vector<bf16*> H, Ht, dZ, dZt;
  bf16 *X0t = nullptr, *dZo = nullptr, *dZot = nullptr;
  float* P = nullptr;
  float* loss_d = nullptr;
  int* err_d = nullptr;
  float* grad_flat = nullptr;  // contiguous dW/db of all layers
  int64_t nparams = 0;
  std::vector<CUtensorMap> mapH, mapHt, mapdZ, mapdZt;
  CUtensorMap mapX0t, mapdZo, mapdZot;
  // data
  int64_t n = 0;
  bf16 *X = nullptr, *Xp = nullptr;
  float *Y = nullptr, *Yp = nullptr, *HW = nullptr, *HWp = nullptr;
  int64_t* perm_d = nullptr;
  CUtensorMap mapX, mapXp;
  int64_t t = 0;  // Adam step
  // inference buffers
  int64_t cap = 0;
  bf16 *Ia = nullptr, *Ib = nullptr;
  CUtensorMap mapIa, mapIb;
};

namespace {

dsp_status efail(dsp_emu e, dsp_status st, const std::string& m) {
  if (e) e->err = m;
  return st;
}

template <class T>
T* dalloc(dsp_emu e, size_t count) {
  void* p = nullptr;
  if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, count * sizeof(T));
  e->allocs.push_back(p);
  return static_cast<T*>(p);
}

dsp_status check_err(dsp_emu e, cudaError_t ce, const char* where) {
  if (ce != cudaSuccess) return efail(e, DSP_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(ce));
  return DSP_OK;
}

dsp_status read_err_flag(dsp_emu e) {
  int h = 0;
  cudaError_t ce = cudaMemcpyAsync(&h, e->err_d, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "emulator");
  if (h) return efail(e, DSP_ERR_TIMEOUT, "a tensor-core GEMM wait ran out (error flag set)");
  return DSP_OK;
}

// forward + backward of one batch (rows a_row0.. of the map `xmap`, targets Yb, weights HWb)
dsp_status train_pass(dsp_emu e, const CUtensorMap& xmap, const bf16* xsrc, int a_row0, const float* Yb,
                      const float* HWb) {
  cudaStream_t s = e->stream;
  const int B = e->B, nl = e->nl;
  cudaError_t ce;
  // X^T of the batch for dW_1
  {
    dim3 blk(32, 8), grd((e->in_pad + 31) / 32, (B + 31) / 32);
    transpose_bf16_kernel<<<grd, blk, 0, s>>>(xsrc + (int64_t)a_row0 * e->in_pad, e->X0t, B, e->in_pad);
  }
  // forward
  for (int i = 0; i < nl; ++i) {
    Layer& l = e->L[i];
    const CUtensorMap& am = (i == 0) ? xmap : e->mapH[i - 1];
    const int r0 = (i == 0) ? a_row0 : 0;
    if (i < nl - 1) {
      EpiHidden ep{l.b, e->Z[i], e->H[i], e->Ht[i], B, l.out_pad};
      ce = launch_gemm(am, l.mapW, r0, 0, B, l.out_pad, l.in_pad, 1, ep, e->err_d, s);
    } else {
      EpiOut ep{l.b, e->P, Yb, HWb, e->dZo, e->dZot, e->loss_d, B, l.out_pad, e->cfg.n_out, e->cfg.n_heads,
                2.0f / (float)(e->cfg.n_out * B)};
      ce = launch_gemm(am, l.mapW, r0, 0, B, l.out_pad, l.in_pad, 1, ep, e->err_d, s);
    }
    if (ce != cudaSuccess) return check_err(e, ce, "forward GEMM");
  }
  // backward
  ce = cudaMemsetAsync(e->grad_flat, 0, e->nparams * sizeof(float), s);
  if (ce != cudaSuccess) return check_err(e, ce, "gradient reset");
  for (int i = nl - 1; i >= 0; --i) {
    Layer& l = e->L[i];
    const CUtensorMap& dzt = (i == nl - 1) ? e->mapdZot : e->mapdZt[i];
    const CUtensorMap& xt = (i == 0) ? e->mapX0t : e->mapHt[i - 1];
    EpiDW ew{l.dW, l.out_pad, l.in_pad};
    ce = launch_gemm(dzt, xt, 0, 0, l.out_pad, l.in_pad, B, DW_SPLITS, ew, e->err_d, s);
    if (ce != cudaSuccess) return check_err(e, ce, "weight-gradient GEMM");
    const bf16* dzt_ptr = (i == nl - 1) ? e->dZot : e->dZt[i];
    bias_grad_kernel<<<(l.out_pad + 7) / 8, 256, 0, s>>>(dzt_ptr, l.db, l.out_pad, B);
    if (i > 0) {
      const CUtensorMap& dz = (i == nl - 1) ? e->mapdZo : e->mapdZ[i];
      EpiBwdX ex{e->Z[i - 1], e->dZ[i - 1], e->dZt[i - 1], B, l.in_pad};
      ce = launch_gemm(dz, l.mapWt, 0, 0, B, l.in_pad, l.out_pad, 1, ex, e->err_d, s);
      if (ce != cudaSuccess) return check_err(e, ce, "input-gradient GEMM");
    }
  }
  return DSP_OK;
}

dsp_status adam_step(dsp_emu e, float lr) {
  cudaStream_t s = e->stream;
  e->t += 1;
  const float bc1 = 1.0f - std::pow(0.9f, (float)e->t), bc2 = 1.0f - std::pow(0.999f, (float)e->t);
  for (Layer& l : e->L) {
    const long long nw = (long long)l.out_pad * l.in_pad;
    adam_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(l.W, l.mW, l.vW, l.dW, l.Wb, l.Wt, l.out_pad, l.in_pad,
                                                            l.out_real, l.in_real, lr, bc1, bc2);
    adam_kernel<<<(l.out_pad + 255) / 256, 256, 0, s>>>(l.b, l.mb, l.vb, l.db, nullptr, nullptr, l.out_pad, 1,
                                                       l.out_real, 1, lr, bc1, bc2);
  }
  return check_err(e, cudaGetLastError(), "adam");
}

dsp_status refresh_bf16(dsp_emu e) {
  for (Layer& l : e->L) {
    const long long nw = (long long)l.out_pad * l.in_pad;
    to_bf16_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, e->stream>>>(l.W, l.Wb, l.Wt, l.out_pad, l.in_pad);
  }
  return check_err(e, cudaGetLastError(), "weight conversion");
}

}  // namespace

extern "C" {

dsp_status dsp_emu_create(int32_t device, void* stream, const dsp_emu_config* cfg, dsp_emu* out) {
  if (!cfg || !out) return DSP_ERR_INVALID_INPUT;
  *out = nullptr;
  if (cfg->n_in <= 0 || cfg->hidden <= 0 || cfg->hidden % 128 != 0 || cfg->n_hidden_layers < 1 || cfg->n_out <= 0 ||
      cfg->n_heads < 1 || cfg->batch <= 0 || cfg->batch % 128 != 0)
    return DSP_ERR_INVALID_INPUT;
  if (cudaSetDevice(device) != cudaSuccess) return DSP_ERR_CUDA;
  if (!encode_fn()) return DSP_ERR_UNSUPPORTED;
  dsp_emu e = new dsp_emu_s();
  e->device = device;
  e->stream = static_cast<cudaStream_t>(stream);
  e->cfg = *cfg;
  e->in_pad = pad64(cfg->n_in);
  e->out_pad = pad64(cfg->n_out * cfg->n_heads);
  e->hid = cfg->hidden;
  e->nl = cfg->n_hidden_layers + 1;
  e->B = cfg->batch;
  const int nl = e->nl, B = e->B;
  e->L.resize(nl);
  int64_t np = 0;
  for (int i = 0; i < nl; ++i) {
    Layer& l = e->L[i];
    l.in_pad = (i == 0) ? e->in_pad : e->hid;
    l.in_real = (i == 0) ? cfg->n_in : e->hid;
    l.out_pad = (i == nl - 1) ? e->out_pad : e->hid;
    l.out_real = (i == nl - 1) ? cfg->n_out * cfg->n_heads : e->hid;
    np += (int64_t)l.out_pad * l.in_pad + l.out_pad;
  }
  e->nparams = np;
  e->grad_flat = dalloc<float>(e, np);
  bool ok = e->grad_flat != nullptr;
  int64_t off = 0;
  std::mt19937_64 rng(cfg->seed);
  std::vector<float> hw;
  for (int i = 0; i < nl && ok; ++i) {
    Layer& l = e->L[i];
    const size_t nw = (size_t)l.out_pad * l.in_pad;
    l.W = dalloc<float>(e, nw);
    l.b = dalloc<float>(e, l.out_pad);
    l.mW = dalloc<float>(e, nw);
    l.vW = dalloc<float>(e, nw);
    l.mb = dalloc<float>(e, l.out_pad);
    l.vb = dalloc<float>(e, l.out_pad);
    l.Wb = dalloc<bf16>(e, nw);
    l.Wt = dalloc<bf16>(e, nw);
    l.dW = e->grad_flat + off;
    l.db = l.dW + nw;
    off += nw + l.out_pad;
    ok = l.W && l.b && l.mW && l.vW && l.mb && l.vb && l.Wb && l.Wt;
    if (!ok) break;
    // He-normal for the GELU layers, 1/sqrt(fan_in) for the output layer
    const float sdv = (i < nl - 1) ? std::sqrt(2.0f / l.in_real) : std::sqrt(1.0f / l.in_real);
    std::normal_distribution<float> nd(0.0f, sdv);
    hw.assign(nw, 0.0f);
    for (int r = 0; r < l.out_real; ++r)
      for (int c = 0; c < l.in_real; ++c) hw[(size_t)r * l.in_pad + c] = nd(rng);
    ok = cudaMemcpy(l.W, hw.data(), nw * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && make_map(&l.mapW, l.Wb, l.out_pad, l.in_pad, bn_for(l.out_pad));
    ok = ok && make_map(&l.mapWt, l.Wt, l.in_pad, l.out_pad, bn_for(l.in_pad));
  }
  // activations
  for (int i = 0; i < nl - 1 && ok; ++i) {
    e->Z.push_back(dalloc<float>(e, (size_t)B * e->hid));
    e->H.push_back(dalloc<bf16>(e, (size_t)B * e->hid));
    e->Ht.push_back(dalloc<bf16>(e, (size_t)B * e->hid));
    e->dZ.push_back(dalloc<bf16>(e, (size_t)B * e->hid));
    e->dZt.push_back(dalloc<bf16>(e, (size_t)B * e->hid));
    ok = e->Z.back() && e->H.back() && e->Ht.back() && e->dZ.back() && e->dZt.back();
    if (!ok) break;
    CUtensorMap mh, mht, mdz, mdzt;
    ok = make_map(&mh, e->H[i], B, e->hid, 128) && make_map(&mht, e->Ht[i], e->hid, B, bn_for(e->hid)) &&
         make_map(&mdz, e->dZ[i], B, e->hid, 128) && make_map(&mdzt, e->dZt[i], e->hid, B, 128);
    e->mapH.push_back(mh);
    e->mapHt.push_back(mht);
    e->mapdZ.push_back(mdz);
    e->mapdZt.push_back(mdzt);
  }
  if (ok) {
    e->X0t = dalloc<bf16>(e, (size_t)e->in_pad * B);
    e->dZo = dalloc<bf16>(e, (size_t)B * e->out_pad);
    e->dZot = dalloc<bf16>(e, (size_t)e->out_pad * B);
    e->P = dalloc<float>(e, (size_t)B * e->out_pad);
    e->loss_d = dalloc<float>(e, 1);
    e->err_d = dalloc<int>(e, 1);
    ok = e->X0t && e->dZo && e->dZot && e->P && e->loss_d && e->err_d;
    ok = ok && make_map(&e->mapX0t, e->X0t, e->in_pad, B, bn_for(e->in_pad)) &&
         make_map(&e->mapdZo, e->dZo, B, e->out_pad, 128) && make_map(&e->mapdZot, e->dZot, e->out_pad, B, 128);
  }
  if (ok) ok = refresh_bf16(e) == DSP_OK && cudaStreamSynchronize(e->stream) == cudaSuccess;
  if (!ok) {
    dsp_emu_destroy(e);
    return DSP_ERR_NO_MEMORY;
  }
  *out = e;
  return DSP_OK;
}

dsp_status dsp_emu_destroy(dsp_emu e) {
  if (!e) return DSP_ERR_INVALID_INPUT;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  for (void* p : e->allocs) cudaFree(p);
  delete e;
  return DSP_OK;
}

const char* dsp_emu_last_error(dsp_emu e) { return e ? e->err.c_str() : ""; }

int32_t dsp_emu_input_stride(dsp_emu e) { return e ? e->in_pad : 0; }

dsp_status dsp_emu_set_data(dsp_emu e, const uint16_t* feats, const float* targets, const float* head_weights,
                            int64_t n) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (!feats || !targets || n < e->B) return efail(e, DSP_ERR_INVALID_INPUT, "need at least one full batch of rows");
  cudaSetDevice(e->device);
  if (e->n != n) {
    // data buffers are replaced, not grown in place
    for (void* p : {(void*)e->X, (void*)e->Xp, (void*)e->Y, (void*)e->Yp, (void*)e->HW, (void*)e->HWp,
                    (void*)e->perm_d}) {
      if (!p) continue;
      cudaFree(p);
      e->allocs.erase(std::remove(e->allocs.begin(), e->allocs.end(), p), e->allocs.end());
    }
    e->X = dalloc<bf16>(e, (size_t)n * e->in_pad);
    e->Xp = dalloc<bf16>(e, (size_t)n * e->in_pad);
    e->Y = dalloc<float>(e, (size_t)n * e->cfg.n_out);
    e->Yp = dalloc<float>(e, (size_t)n * e->cfg.n_out);
    e->HW = dalloc<float>(e, (size_t)n * e->cfg.n_heads);
    e->HWp = dalloc<float>(e, (size_t)n * e->cfg.n_heads);
    e->perm_d = dalloc<int64_t>(e, (size_t)n);
    if (!e->X || !e->Xp || !e->Y || !e->Yp || !e->HW || !e->HWp || !e->perm_d)
      return efail(e, DSP_ERR_NO_MEMORY, "training-set buffers");
    e->n = n;
    if (!make_map(&e->mapX, e->X, n, e->in_pad, 128) || !make_map(&e->mapXp, e->Xp, n, e->in_pad, 128))
      return efail(e, DSP_ERR_CUDA, "tensor map of the training set");
  }
  cudaError_t ce = cudaMemcpyAsync(e->X, feats, (size_t)n * e->in_pad * 2, cudaMemcpyDeviceToDevice, e->stream);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(e->Y, targets, (size_t)n * e->cfg.n_out * 4, cudaMemcpyDeviceToDevice, e->stream);
  if (ce == cudaSuccess) {
    if (head_weights)
      ce = cudaMemcpyAsync(e->HW, head_weights, (size_t)n * e->cfg.n_heads * 4, cudaMemcpyDeviceToDevice, e->stream);
    else {
      std::vector<float> ones((size_t)n * e->cfg.n_heads, 1.0f);
      ce = cudaMemcpyAsync(e->HW, ones.data(), ones.size() * 4, cudaMemcpyHostToDevice, e->stream);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    }
  }
  return check_err(e, ce, "training-set upload");
}

dsp_status dsp_emu_train(dsp_emu e, int32_t epochs, float lr, float lr_min, uint64_t shuffle_seed, float* epoch_loss) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (!e->X || epochs < 0) return efail(e, DSP_ERR_INVALID_INPUT, "no training set");
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  const int64_t nb = e->n / e->B;
  const int64_t total = nb * epochs;
  std::vector<int64_t> perm(e->n);
  std::mt19937_64 rng(shuffle_seed);
  int64_t step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    cudaError_t ce = cudaMemcpyAsync(e->perm_d, perm.data(), perm.size() * 8, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);  // perm is reused next epoch
    if (ce != cudaSuccess) return check_err(e, ce, "shuffle upload");
    gather_rows_kernel<<<(unsigned)e->n, 64, 0, s>>>(e->X, e->Y, e->HW, e->perm_d, e->Xp, e->Yp, e->HWp, e->n,
                                                     e->in_pad, e->cfg.n_out, e->cfg.n_heads);
    cudaMemsetAsync(e->loss_d, 0, sizeof(float), s);
    for (int64_t b = 0; b < nb; ++b, ++step) {
      const float cs = 0.5f * (1.0f + std::cos(3.14159265358979f * (float)step / (float)std::max<int64_t>(1, total)));
      const float lr_t = lr_min + (lr - lr_min) * cs;
      dsp_status st = train_pass(e, e->mapXp, e->Xp, (int)(b * e->B), e->Yp + b * e->B * e->cfg.n_out,
                                 e->HWp + b * e->B * e->cfg.n_heads);
      if (st != DSP_OK) return st;
      if ((st = adam_step(e, lr_t)) != DSP_OK) return st;
    }
    float l = 0.0f;
    ce = cudaMemcpyAsync(&l, e->loss_d, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return check_err(e, ce, "training");
    if (epoch_loss) epoch_loss[ep] = l / (float)(nb * e->B);
    dsp_status st = read_err_flag(e);
    if (st != DSP_OK) return st;
  }
  return DSP_OK;
}

dsp_status dsp_emu_gradients(dsp_emu e, float* grads, float* loss) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (!e->X || !grads) return efail(e, DSP_ERR_INVALID_INPUT, "no training set");
  cudaSetDevice(e->device);
  cudaMemsetAsync(e->loss_d, 0, sizeof(float), e->stream);
  dsp_status st = train_pass(e, e->mapX, e->X, 0, e->Y, e->HW);
  if (st != DSP_OK) return st;
  cudaError_t ce = cudaMemcpyAsync(grads, e->grad_flat, e->nparams * 4, cudaMemcpyDeviceToDevice, e->stream);
  if (ce == cudaSuccess && loss) ce = cudaMemcpyAsync(loss, e->loss_d, 4, cudaMemcpyDeviceToDevice, e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "gradients");
  return read_err_flag(e);
}

dsp_status dsp_emu_forward(dsp_emu e, const uint16_t* feats, int64_t rows, float* preds) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (!feats || !preds || rows < 0) return efail(e, DSP_ERR_INVALID_INPUT, "null features or predictions");
  if (rows == 0) return DSP_OK;
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  const int64_t chunk = 65536;
  if (e->cap < chunk) {
    e->Ia = dalloc<bf16>(e, (size_t)chunk * e->hid);
    e->Ib = dalloc<bf16>(e, (size_t)chunk * e->hid);
    if (!e->Ia || !e->Ib) return efail(e, DSP_ERR_NO_MEMORY, "inference buffers");
    if (!make_map(&e->mapIa, e->Ia, chunk, e->hid, 128) || !make_map(&e->mapIb, e->Ib, chunk, e->hid, 128))
      return efail(e, DSP_ERR_CUDA, "inference tensor maps");
    e->cap = chunk;
  }
  CUtensorMap mx;
  if (!make_map(&mx, feats, rows, e->in_pad, 128)) return efail(e, DSP_ERR_INVALID_INPUT, "feature tensor map");
  for (int64_t r0 = 0; r0 < rows; r0 += chunk) {
    const int m = (int)std::min<int64_t>(chunk, rows - r0);
    bf16* nxt = e->Ib;
    bf16* cur = e->Ia;
    const CUtensorMap* mc = &e->mapIa;
    const CUtensorMap* mn = &e->mapIb;
    for (int i = 0; i < e->nl; ++i) {
      Layer& l = e->L[i];
      const CUtensorMap& am = (i == 0) ? mx : *mc;
      const int a0 = (i == 0) ? (int)r0 : 0;
      cudaError_t ce;
      if (i < e->nl - 1) {
        EpiHidden ep{l.b, nullptr, nxt, nullptr, m, l.out_pad};
        ce = launch_gemm(am, l.mapW, a0, 0, m, l.out_pad, l.in_pad, 1, ep, e->err_d, s);
        std::swap(cur, nxt);
        std::swap(mc, mn);
      } else {
        // predictions of the real head outputs only: compact [rows][n_heads*n_out]
        const int nreal = e->cfg.n_heads * e->cfg.n_out;
        EpiStoreBias eb{preds + r0 * (int64_t)nreal, l.b, m, nreal};
        ce = launch_gemm(am, l.mapW, a0, 0, m, l.out_pad, l.in_pad, 1, eb, e->err_d, s);
      }
      if (ce != cudaSuccess) return check_err(e, ce, "inference GEMM");
    }
  }
  return read_err_flag(e);
}

int64_t dsp_emu_param_count(dsp_emu e) { return e ? e->nparams : 0; }

dsp_status dsp_emu_layer_dims(dsp_emu e, int32_t layer, int32_t* in_pad, int32_t* out_pad) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (layer < 0 || layer >= e->nl) return DSP_ERR_INVALID_INPUT;
  if (in_pad) *in_pad = e->L[layer].in_pad;
  if (out_pad) *out_pad = e->L[layer].out_pad;
  return DSP_OK;
}

dsp_status dsp_emu_get_params(dsp_emu e, float* host) {
  if (!e || !host) return DSP_ERR_INVALID_INPUT;
  cudaSetDevice(e->device);
  int64_t off = 0;
  for (Layer& l : e->L) {
    const size_t nw = (size_t)l.out_pad * l.in_pad;
    cudaMemcpyAsync(host + off, l.W, nw * 4, cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(host + off + nw, l.b, l.out_pad * 4, cudaMemcpyDeviceToHost, e->stream);
    off += nw + l.out_pad;
  }
  return check_err(e, cudaStreamSynchronize(e->stream), "get_params");
}

dsp_status dsp_emu_set_params(dsp_emu e, const float* host) {
  if (!e || !host) return DSP_ERR_INVALID_INPUT;
  cudaSetDevice(e->device);
  int64_t off = 0;
  for (Layer& l : e->L) {
    const size_t nw = (size_t)l.out_pad * l.in_pad;
    cudaMemcpyAsync(l.W, host + off, nw * 4, cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(l.b, host + off + nw, l.out_pad * 4, cudaMemcpyHostToDevice, e->stream);
    off += nw + l.out_pad;
  }
  cudaError_t ce = cudaStreamSynchronize(e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "set_params");
  dsp_status st = refresh_bf16(e);
  if (st != DSP_OK) return st;
  return check_err(e, cudaStreamSynchronize(e->stream), "set_params");
}

dsp_status dsp_emu_gemm_bf16(dsp_emu e, const uint16_t* A, const uint16_t* B, float* Cm, int32_t M, int32_t N,
                             int32_t K) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (!A || !B || !Cm || M <= 0 || N <= 0 || K <= 0 || K % 8 != 0)
    return efail(e, DSP_ERR_INVALID_INPUT, "GEMM shape");
  cudaSetDevice(e->device);
  CUtensorMap ma, mb;
  if (!make_map(&ma, A, M, K, 128) || !make_map(&mb, B, N, K, bn_for(N)))
    return efail(e, DSP_ERR_INVALID_INPUT, "GEMM tensor maps");
  EpiStore ep{Cm, M, N};
  cudaError_t ce = launch_gemm(ma, mb, 0, 0, M, N, K, 1, ep, e->err_d, e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "GEMM launch");
  return read_err_flag(e);
}

dsp_status dsp_emu_wait_selftest(dsp_emu e, int64_t cycles) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (cycles <= 0 || cycles > (1ll << 31)) return efail(e, DSP_ERR_INVALID_INPUT, "cycles out of (0, 2^31]");
  cudaSetDevice(e->device);
  int h = 0;
  cudaError_t ce = cudaMemcpyAsync(&h, e->err_d, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "wait self-test");
  if (h) return efail(e, DSP_ERR_TIMEOUT, "the error flag was already set");
  dsp_tc::wait_selftest_kernel<<<1, 32, 0, e->stream>>>(e->err_d, (long long)cycles);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return check_err(e, ce, "wait self-test launch");
  const dsp_status st = read_err_flag(e);
  // the self-test's own timeout leaves the emulator usable: clear the flag it set
  ce = cudaMemsetAsync(e->err_d, 0, sizeof(int), e->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "wait self-test");
  return st;
}

dsp_status dsp_emu_gate(dsp_emu e, const float* raw, int32_t raw_stride, const float* lo, const float* hi,
                        const float* preds, const float* mu, const float* sd, const float* scale, const float* add,
                        float eps, float rel_tol, float floor_frac, int64_t rows, float* flux, int32_t* fallback,
                        int32_t* idx, int32_t* n_fallback) {
  if (!e) return DSP_ERR_NOT_INITIALIZED;
  if (e->cfg.n_heads != 2) return efail(e, DSP_ERR_UNSUPPORTED, "the gate compares two heads");
  if (!raw || !lo || !hi || !preds || !mu || !sd || !flux || !fallback || !idx || !n_fallback)
    return efail(e, DSP_ERR_INVALID_INPUT, "null gate argument");
  cudaSetDevice(e->device);
  cudaError_t ce = cudaMemsetAsync(n_fallback, 0, sizeof(int32_t), e->stream);
  if (ce != cudaSuccess) return check_err(e, ce, "gate");
  if (rows == 0) return DSP_OK;
  gate_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, e->stream>>>(
      raw, raw_stride, e->cfg.n_in, lo, hi, preds, e->cfg.n_heads * e->cfg.n_out, e->cfg.n_out, mu, sd, scale, add,
      eps, rel_tol, floor_frac, rows, flux, fallback, idx, n_fallback);
  return check_err(e, cudaGetLastError(), "gate");
}

}  // extern "C"
