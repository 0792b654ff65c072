// phase_clock.cuh — cycle accounting by phase of the flux path's kernels
// (tracing build only; force-included into dsp_capi.cu by
// `python -m disort_b200.build --phase-clock`).
//
// The kernels mark phase boundaries with DSP_PHASE(k), k in 0..29; a marker
// adds the clock64() cycles since the previous marker of the thread to slot
// k % 10 of a per-thread accumulator, and DSP_PHASE_END adds lane 0's
// accumulators of each warp to a device array read by dsp_phase_read.  The
// totals are warp-time per phase, summed over warps: their shares show where a
// warp's time goes, not the SM's issue slots.  The accumulators cost registers
// and the markers instructions, so the tracing build runs slower than the
// product build.
#pragma once

__device__ unsigned long long g_dsp_phase[16];

#define DSP_PHASE_BEGIN                      \
  long long dsp_phase_t0_ = clock64();       \
  long long dsp_phase_acc_[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#define DSP_PHASE(k)                                         \
  {                                                          \
    const long long dsp_phase_t_ = clock64();                \
    dsp_phase_acc_[(k) % 10] += dsp_phase_t_ - dsp_phase_t0_; \
    dsp_phase_t0_ = dsp_phase_t_;                            \
  }
#define DSP_PHASE_END                                                              \
  if ((threadIdx.x & 31u) == 0u) {                                                 \
    for (int q_ = 0; q_ < 10; ++q_)                                                \
      atomicAdd(&g_dsp_phase[q_], static_cast<unsigned long long>(dsp_phase_acc_[q_])); \
  }

// Copies the 16 accumulators to `out` (host memory); returns a cudaError_t.
extern "C" int dsp_phase_read(unsigned long long* out) {
  return static_cast<int>(cudaMemcpyFromSymbol(out, g_dsp_phase, sizeof(unsigned long long) * 16));
}
// Zeroes the accumulators; returns a cudaError_t.
extern "C" int dsp_phase_reset(void) {
  const unsigned long long z[16] = {};
  return static_cast<int>(cudaMemcpyToSymbol(g_dsp_phase, z, sizeof(z)));
}
