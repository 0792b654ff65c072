// tc_gemm.cuh — BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the
// flux emulator: C[M x N] = A[M x K] * B[N x K]^T, A and B row-major with K
// contiguous ("TN"), FP32 accumulation in tensor memory, a fused epilogue.
//
// One CTA computes a 128 x BN tile with four warps:
//   warp 0 lane 0  TMA producer: 128 x 64 (A) and BN x 64 (B) BF16 boxes with the
//                  128-byte swizzle into a STAGES-deep shared-memory ring;
//   warp 1         allocates BN tensor-memory columns; lane 0 issues
//                  tcgen05.mma (M = 128, N = BN, K = 16 per instruction) and
//                  releases each stage with tcgen05.commit;
//   all warps      epilogue: warp w reads accumulator rows 32w..32w+31 with
//                  tcgen05.ld and hands 16-column slices to the epilogue functor.
// blockIdx.z splits K (the epilogue then accumulates atomically).
//
// Every wait on an mbarrier is bounded (about one second of clock64 cycles);
// a wait that runs out sets the CTA's abort flag, which makes the other roles
// stop issuing work, drains the copies already in flight (again bounded), frees
// tensor memory and reports the failure through *err.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dsp_tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false when the phase did not complete within `limit` cycles
// (~2^31 by default, about a second) or another role of the CTA has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          long long limit = (1ll << 31)) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// Self-test of the bounded wait: one mbarrier that nothing arrives on (no copy
// or MMA is issued against it), waited on by every thread with a short limit.
// The wait runs out and the CTA reports it through the error flag the GEMMs use.
static __global__ void __launch_bounds__(32) wait_selftest_kernel(int* err, long long limit) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0, &abort_flag, limit) ? 1 : 0) != 0;
  if (threadIdx.x == 0 && !ok) atomicExch(err, 1);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 128-byte swizzle: 8-row core groups 1024 bytes apart (SBO), leading offset
// unused for swizzled K-major (encoded 1), descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t sdesc_k_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);  // start address, bits [0,14)
  d |= (uint64_t)1 << 16;                  // leading byte offset (16 B units)
  d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset, bits [32,46)
  d |= (uint64_t)1 << 46;                  // version
  d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D = F32, A = B = BF16,
// both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int n) {
  return (1u << 4)                        // D format F32
         | (1u << 7)                      // A format BF16
         | (1u << 10)                     // B format BF16
         | ((uint32_t)(n >> 3) << 17)     // N >> 3
         | ((uint32_t)(128 >> 4) << 24);  // M >> 4
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN, int STAGES>
struct GemmCfg {
  static_assert(BN == 64 || BN == 128 || BN == 256, "tile N");
  static constexpr int BM = 128, BK = 64;
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  // ring + barriers (full, empty, done) + tmem slot + flags, plus 1 KB for alignment
  static constexpr size_t smem_bytes() { return (size_t)STAGES * STAGE_BYTES + 1024 + 256; }
};

// Epilogue functors receive (row, col0, v[16], split): accumulator row `row`
// of the output, columns col0..col0+15.  Rows/columns past the problem are the
// functor's to skip.
template <int BN, int STAGES, class Epi>
__global__ void __launch_bounds__(128, 1)
    tc_gemm_tn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int a_row0,
                      int b_row0, int k_tiles, int k_tiles_per_split, Epi epi, int* err) {
  using C = GemmCfg<BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  volatile int* consumed = abort_flag + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * C::BM, n0 = blockIdx.y * BN;
  const int kt0 = blockIdx.z * k_tiles_per_split;
  int nk = k_tiles - kt0;
  if (nk > k_tiles_per_split) nk = k_tiles_per_split;
  if (nk < 0) nk = 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    *consumed = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      int issued = 0;
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES;
        if (i >= STAGES && !mbar_wait(empty + s, ((i / STAGES) - 1) & 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        mbar_arrive_expect_tx(full + s, C::STAGE_BYTES);
        uint8_t* st = smem + s * C::STAGE_BYTES;
        tma_load_2d(st, &tmA, full + s, (kt0 + i) * C::BK, a_row0 + m0);
        tma_load_2d(st + C::A_BYTES, &tmB, full + s, (kt0 + i) * C::BK, b_row0 + n0);
        issued = i + 1;
      }
      // copies issued but never consumed (abort): wait for them to land
      for (int i = *consumed; i < issued; ++i) {
        const long long t0 = clock64();
        while (!mbar_try_wait(full + i % STAGES, (i / STAGES) & 1) && clock64() - t0 < (1ll << 31)) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      constexpr uint32_t idesc = idesc_bf16_f32(BN);
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES;
        if (!mbar_wait(full + s, (i / STAGES) & 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        *consumed = i + 1;
        tc_fence_after();
        const uint32_t a_addr = smem_u32(smem + s * C::STAGE_BYTES);
        const uint32_t b_addr = a_addr + C::A_BYTES;
#pragma unroll
        for (int kk = 0; kk < C::BK / 16; ++kk)
          umma_bf16(tmem, sdesc_k_sw128(a_addr + kk * 32), sdesc_k_sw128(b_addr + kk * 32), idesc,
                    (i > 0 || kk > 0) ? 1u : 0u);
        umma_commit(empty + s);
      }
      umma_commit(done);  // arrives once every MMA issued above has completed
    }
  }
  __syncwarp();
  // ---- epilogue ----
  const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0, abort_flag) ? 1 : 0) != 0;
  tc_fence_after();
  if (ok && nk > 0 && !*abort_flag) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      __syncwarp();
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      epi.apply(row, n0 + c, v, blockIdx.z);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS));
  if (threadIdx.x == 0 && (*abort_flag || !ok)) atomicExch(err, 1);
}

}  // namespace dsp_tc
