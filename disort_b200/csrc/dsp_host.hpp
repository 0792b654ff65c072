// dsp_host.hpp — host-side internals of libdsp.so shared by its translation
// units: the context, per-kernel timing, workspace growth, error reporting and
// the per-stream-count constant tables.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dsp.h"
#include "dsp_device.cuh"

using namespace dsp;

struct dsp_context_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  int sm_count = 148;
  // device buffers owned by the context
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void* stage_in = nullptr;
  size_t stage_in_bytes = 0;
  void* stage_out = nullptr;
  size_t stage_out_bytes = 0;
  std::map<int, double*> tables;
  std::map<int, std::vector<double>> host_tables;  // host copies of `tables`
  std::map<int, double*> mode_tables;  // general solver: one table per azimuth mode
  double* brdf_q = nullptr;            // general solver: the BRDF azimuth quadrature [gmu 200 | gwt 200]
  void* meta = nullptr;                // general solver: chunk index arrays
  double* flux_defaults = nullptr;     // defaults of absent flux-batch scalars (device, uploaded once)
  size_t meta_bytes = 0;
  // host-buffer solves: copy streams and events of the copy/compute pipeline
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaStream_t s_c2 = nullptr;  // second solve stream of the host-buffer pipeline
  std::vector<cudaEvent_t> pipe_ev;
  // optional per-kernel timing
  bool timing = false;
  uint32_t debug = 0;  // DSP_DEBUG_* flags
  std::vector<dsp_schedule> schedule;  // launch schedules, first match wins
  struct Pending {
    int kernel;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> free_events;
  std::vector<std::string> knames;
  std::vector<double> kms;
  std::vector<int64_t> kcount;
};

namespace dsp_host {
// The schedule entry for (N, L); a zeroed entry (built-in choices) if none matches.
inline dsp_schedule find_schedule(dsp_context c, int N, int L) {
  for (const dsp_schedule& e : c->schedule)
    if (e.num_streams == N && e.min_layers <= L && L <= e.max_layers) return e;
  dsp_schedule z{};
  z.num_streams = N;
  return z;
}

inline cudaEvent_t take_event(dsp_context c) {
  if (!c->free_events.empty()) {
    cudaEvent_t e = c->free_events.back();
    c->free_events.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

inline int kernel_id(dsp_context c, const char* name) {
  for (size_t k = 0; k < c->knames.size(); ++k)
    if (c->knames[k] == name) return (int)k;
  c->knames.push_back(name);
  c->kms.push_back(0.0);
  c->kcount.push_back(0);
  return (int)c->knames.size() - 1;
}

// Brackets one launch with events when timing is on.
// An NVTX range over a host scope (an entry-point call, a chunk, a launch):
// header-only NVTX v3, a no-op unless a profiler's injection library is loaded.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// One launch: its NVTX range, and with timing on a pair of CUDA events around it.
struct KernelTimer {
  dsp_context c;
  cudaStream_t s;
  int id = -1;
  cudaEvent_t a = nullptr, b = nullptr;
  NvtxRange range;
  KernelTimer(dsp_context ctx, const char* name, cudaStream_t st = nullptr)
      : c(ctx), s(st ? st : ctx->stream), range(name) {
    if (!c->timing) return;
    id = kernel_id(c, name);
    a = take_event(c);
    b = take_event(c);
    cudaEventRecord(a, s);
  }
  ~KernelTimer() {
    if (id < 0) return;
    cudaEventRecord(b, s);
    c->pending.push_back({id, a, b});
  }
};

inline void drain_timing(dsp_context c) {
  for (auto& p : c->pending) {
    float ms = 0.f;
    cudaEventSynchronize(p.b);
    cudaEventElapsedTime(&ms, p.a, p.b);
    c->kms[p.kernel] += ms;
    c->kcount[p.kernel] += 1;
    c->free_events.push_back(p.a);
    c->free_events.push_back(p.b);
  }
  c->pending.clear();
}
}  // namespace dsp_host

namespace dsp_host {

inline constexpr int kSupported[] = {4, 6, 8, 10, 12, 14, 16, 32, 64};

inline bool supported_nstr(int n) {
  for (int s : kSupported)
    if (s == n) return true;
  return false;
}

inline dsp_status fail(dsp_context ctx, dsp_status st, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return st;
}

inline dsp_status cuda_fail(dsp_context ctx, cudaError_t e, const char* where) {
  return fail(ctx, DSP_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

inline dsp_status ensure(dsp_context ctx, void** buf, size_t* have, size_t need, const char* what) {
  if (*have >= need) return DSP_OK;
  if (*buf) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
  }
  size_t alloc = need + need / 8 + (1 << 20);
  cudaError_t e = cudaMalloc(buf, alloc);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, DSP_ERR_NO_MEMORY, std::string("cudaMalloc of ") + what + " failed");
  }
  *have = alloc;
  return DSP_OK;
}

// Gauss-Legendre nodes/weights on (0,1) by Newton iteration (the reference's
// gaussianQuadrature, FluxSolver.cpp:257-290) and the m = 0 Legendre table at
// the nodes (Legendre.cpp:74-88).  Computed on the host so the device and the
// reference use the same values.
inline bool build_tables(int N, std::vector<double>& tab) {
  const int NN = N / 2;
  tab.assign(tab_size(N), 0.0);
  double* mu = tab.data() + tab_mu(N);
  double* wt = tab.data() + tab_wt(N);
  for (int i = 1; i <= NN; ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (NN + 0.5));
    double z1, pp;
    int iter = 0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= NN; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = NN * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (++iter > 10) return false;
    } while (std::fabs(z - z1) > 3.0e-14);
    mu[i - 1] = 0.5 * (1.0 + z);
    wt[i - 1] = 1.0 / ((1.0 - z * z) * pp * pp);
  }
  for (int i = 0; i < NN; ++i) {
    mu[NN + i] = -mu[i];
    wt[NN + i] = wt[i];
  }
  for (int iq = 0; iq < NN; ++iq) {
    tab[tab_dsim(N) + iq] = std::sqrt(wt[iq] * mu[iq]);
    tab[tab_dinv(N) + iq] = 1.0 / tab[tab_dsim(N) + iq];
  }
  double* y = tab.data() + tab_ylm(N);
  for (int i = 0; i < N; ++i) {
    y[0 * N + i] = 1.0;
    y[1 * N + i] = mu[i];
  }
  for (int l = 2; l < N; ++l)
    for (int i = 0; i < N; ++i)
      y[l * N + i] = ((2.0 * l - 1.0) * mu[i] * y[(l - 1) * N + i] - (l - 1.0) * y[(l - 2) * N + i]) / l;
  return true;
}

inline dsp_status get_tables(dsp_context ctx, int N, const double** out) {
  auto it = ctx->tables.find(N);
  if (it != ctx->tables.end()) {
    *out = it->second;
    return DSP_OK;
  }
  std::vector<double> tab;
  if (!build_tables(N, tab)) return fail(ctx, DSP_ERR_EIGEN, "Gauss quadrature did not converge");
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, tab.size() * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(tables)");
  e = cudaMemcpy(d, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpy(tables)");
  ctx->tables[N] = d;
  ctx->host_tables[N] = tab;
  *out = d;
  return DSP_OK;
}

inline PlanckConsts planck_consts() {
  PlanckConsts pk;
  pk.vmax = std::log(DBL_MAX);
  pk.sigdpi = 5.67032E-8 / M_PI;
  pk.conc = 15.0 / std::pow(M_PI, 4.0);
  pk.c1 = 1.1911e-8;
  return pk;
}

struct Sizes {
  size_t inst, layer, bvp;  // doubles per instance
  size_t per_inst_bytes() const { return (inst + layer + bvp) * sizeof(double) + sizeof(int32_t); }
};

inline Sizes sizes_for(int N, int L) {
  Sizes s;
  s.inst = InstLayout::make(L, N).stride;
  s.layer = (size_t)L * lrec_stride(N);
  s.bvp = (size_t)L * brec_stride(N);
  return s;
}

inline size_t workspace_budget() {
  const char* e = std::getenv("DSP_WORKSPACE_MB");
  size_t mb = e ? (size_t)std::strtoull(e, nullptr, 10) : 16384;
  if (mb < 16) mb = 16;
  return mb << 20;
}

}  // namespace dsp_host
