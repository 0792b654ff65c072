// dsp_capi.cu — the C ABI of libdsp.so (include/dsp.h): contexts, timing, and
// the staging, chunking and kernel launches of a flux spectral-band solve.  The
// general solve lives in dsp_general.cu; shared host internals in dsp_host.hpp.
#include <cuda_runtime.h>

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
#include "dsp_host.hpp"
#include "flux_bvp_tile.cuh"
#include "flux_bvp_reg.cuh"
#include "flux_jac.cuh"
#include "flux_layer.cuh"
#include "flux_setup.cuh"
#include "flux_sph.cuh"

using namespace dsp;
using namespace dsp_host;

namespace {

// One chunk of a flux solve.  JAC: the temperature-Jacobian forms of the layer
// and boundary-value kernels (they also write the P/Q and multiplier records),
// then flux_jac_kernel with the view `jv`.
template <int N, bool JAC, bool SPH>
dsp_status launch_flux_chunk(dsp_context ctx, const FluxParams& p, cudaStream_t s, const JacView* jv) {
  {
    KernelTimer kt(ctx, "flux_setup_kernel", s);
    flux_setup_kernel<<<(p.n + 3) / 4, 128, 0, s>>>(p);
  }
  if constexpr (SPH) {
    KernelTimer kt(ctx, "flux_sph_chapman_kernel", s);
    flux_sph_chapman_kernel<false><<<(p.n + 3) / 4, 128, 0, s>>>(p);
  }
  {
    static bool attr = false;
    if (!attr) {
      flux_layer_set_attrs<N, JAC>();
      attr = true;
    }
    // the schedule for (N, L) may pick the layer stage's form and CTA size
    const dsp_schedule sch = find_schedule(ctx, N, p.L);
    const bool split = sch.layer_stage == 0 ? layer_split<N>() : sch.layer_stage == 1;
    flux_layer_launch<N, JAC>(
        p, ctx->host_tables.at(N).data(), s,
        [&](const char* name, auto&& launch) {
          KernelTimer kt(ctx, name, s);
          launch();
        },
        split, sch.layer_cta ? sch.layer_cta : 128);
  }
  if constexpr (SPH) {
    // the spherical particular solution replaces the layer stage's plane-parallel one
    using C = SCfg<N>;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(flux_sph_source_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)C::smem_bytes());
      attr = true;
    }
    const long long tasks = (long long)p.n * p.L;
    KernelTimer kt(ctx, "flux_sph_source_kernel", s);
    flux_sph_source_kernel<N><<<(unsigned)((tasks + C::WPC - 1) / C::WPC), 32 * C::WPC, C::smem_bytes(), s>>>(p);
  }
  if constexpr (N <= 16) {
    using C = RCfg<N>;
    const size_t sm = C::smem_bytes();
    const int grid = (p.n + C::TPC - 1) / C::TPC;
    KernelTimer kt(ctx, "flux_bvp_kernel", s);
    flux_bvp_reg_kernel<N, false, JAC, SPH><<<grid, C::CTA, sm, s>>>(p);
  } else {
    using C = TCfg<N>;
    const size_t sm = C::smem_bytes();
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(flux_bvp_tile_kernel<N, false, JAC, SPH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
      attr = true;
    }
    const int grid = (p.n + C::TPC - 1) / C::TPC;
    KernelTimer kt(ctx, "flux_bvp_kernel", s);
    flux_bvp_tile_kernel<N, false, JAC, SPH><<<grid, C::CTA, sm, s>>>(p);
  }
  if (jv) {
    using C = JCfg<N>;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(flux_jac_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes());
      attr = true;
    }
    KernelTimer kt(ctx, "flux_jac_kernel", s);
    flux_jac_kernel<N><<<p.n, C::KB, C::smem_bytes(), s>>>(p, *jv);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "flux kernel launch");
  return DSP_OK;
}

// Instances the boundary-value kernel of N streams keeps resident on the whole
// GPU at once (one wave).
template <int N>
int64_t bvp_wave_n(int sm_count) {
  int blocks = 0;
  if constexpr (N <= 16) {
    using C = RCfg<N>;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, flux_bvp_reg_kernel<N>, C::CTA, C::smem_bytes());
    return (int64_t)std::max(blocks, 1) * C::TPC * sm_count;
  } else {
    using C = TCfg<N>;
    cudaFuncSetAttribute(flux_bvp_tile_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, flux_bvp_tile_kernel<N>, C::CTA, C::smem_bytes());
    return (int64_t)std::max(blocks, 1) * C::TPC * sm_count;
  }
}

int64_t bvp_wave(int N, int sm_count) {
  switch (N) {
    case 4: return bvp_wave_n<4>(sm_count);
    case 6: return bvp_wave_n<6>(sm_count);
    case 8: return bvp_wave_n<8>(sm_count);
    case 10: return bvp_wave_n<10>(sm_count);
    case 12: return bvp_wave_n<12>(sm_count);
    case 14: return bvp_wave_n<14>(sm_count);
    case 16: return bvp_wave_n<16>(sm_count);
    case 32: return bvp_wave_n<32>(sm_count);
    case 64: return bvp_wave_n<64>(sm_count);
  }
  return sm_count;
}

template <int N>
dsp_status launch_flux_n(dsp_context ctx, const FluxParams& p, cudaStream_t s, const JacView* jv) {
  // Jacobian records are only needed when there is a thermal source to differentiate
  const bool jac = jv && (p.flags & DSP_FLAG_THERMAL);
  const bool sph = (p.flags & DSP_FLAG_SPHERICAL_BEAM) != 0;
  if (sph) return jac ? launch_flux_chunk<N, true, true>(ctx, p, s, jv) : launch_flux_chunk<N, false, true>(ctx, p, s, jv);
  return jac ? launch_flux_chunk<N, true, false>(ctx, p, s, jv) : launch_flux_chunk<N, false, false>(ctx, p, s, jv);
}

dsp_status launch_flux(dsp_context ctx, int N, const FluxParams& p, cudaStream_t s, const JacView* jv) {
  switch (N) {
    case 4: return launch_flux_n<4>(ctx, p, s, jv);
    case 6: return launch_flux_n<6>(ctx, p, s, jv);
    case 8: return launch_flux_n<8>(ctx, p, s, jv);
    case 10: return launch_flux_n<10>(ctx, p, s, jv);
    case 12: return launch_flux_n<12>(ctx, p, s, jv);
    case 14: return launch_flux_n<14>(ctx, p, s, jv);
    case 16: return launch_flux_n<16>(ctx, p, s, jv);
    case 32: return launch_flux_n<32>(ctx, p, s, jv);
    case 64: return launch_flux_n<64>(ctx, p, s, jv);
  }
  return fail(ctx, DSP_ERR_UNSUPPORTED, "unsupported num_streams");
}

// the batch arrays of dsp_flux_batch, in field order
constexpr int kFluxArrays = 16;
// scalar fields, which take the DisortFluxConfig default when absent
constexpr bool kScalarField[kFluxArrays] = {true, true, false, false, false, false, true, true,
                                            true, true, true, true, true, true, false, true};

// elements of one instance's value for each batch array, in field order
void per_inst_counts(const dsp_flux_batch* b, int64_t cnt[kFluxArrays]) {
  const int L = b->num_layers;
  const int64_t pm = (b->flags & DSP_FLAG_HG_G) ? (int64_t)L : (int64_t)L * b->pmom_count;
  const int64_t c[kFluxArrays] = {1, 1, L, L, pm, L + 1, 1, 1, 1, 1, 1, 1, 1, 1, L + 1, 1};
  for (int k = 0; k < kFluxArrays; ++k) cnt[k] = c[k];
}

dsp_darray* batch_arrays(dsp_flux_batch* b) { return &b->wavenumber_low; }

dsp_status flux_solve(dsp_context ctx, const dsp_flux_batch* batch_in, const dsp_flux_out* out,
                      const dsp_flux_jac_out* jac);

}  // namespace

extern "C" {

int32_t dsp_api_version(void) { return DSP_API_VERSION; }

const char* dsp_status_string(dsp_status s) {
  switch (s) {
    case DSP_OK: return "OK";
    case DSP_ERR_INVALID_INPUT: return "INVALID_INPUT";
    case DSP_ERR_SINGULAR: return "SINGULAR";
    case DSP_ERR_NONFINITE: return "NONFINITE";
    case DSP_ERR_TIMEOUT: return "TIMEOUT";
    case DSP_ERR_CUDA: return "CUDA_ERROR";
    case DSP_ERR_UNSUPPORTED: return "UNSUPPORTED";
    case DSP_ERR_NO_MEMORY: return "NO_MEMORY";
    case DSP_ERR_EIGEN: return "EIGEN";
    case DSP_ERR_NOT_INITIALIZED: return "NOT_INITIALIZED";
  }
  return "UNKNOWN";
}

dsp_status dsp_context_create(int32_t device, void* stream, dsp_context* out) {
  if (!out) return DSP_ERR_INVALID_INPUT;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DSP_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return DSP_ERR_INVALID_INPUT;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return DSP_ERR_CUDA;
  dsp_context c = new dsp_context_s();
  c->device = device;
  c->stream = static_cast<cudaStream_t>(stream);
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return DSP_OK;
}

dsp_status dsp_context_destroy(dsp_context ctx) {
  if (!ctx) return DSP_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  drain_timing(ctx);
  for (cudaEvent_t e : ctx->free_events) cudaEventDestroy(e);
  if (ctx->s_in) cudaStreamSynchronize(ctx->s_in);
  if (ctx->s_out) cudaStreamSynchronize(ctx->s_out);
  if (ctx->s_c2) cudaStreamSynchronize(ctx->s_c2);
  for (cudaEvent_t e : ctx->pipe_ev) cudaEventDestroy(e);
  if (ctx->s_in) cudaStreamDestroy(ctx->s_in);
  if (ctx->s_out) cudaStreamDestroy(ctx->s_out);
  if (ctx->s_c2) cudaStreamDestroy(ctx->s_c2);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->stage_in) cudaFree(ctx->stage_in);
  if (ctx->stage_out) cudaFree(ctx->stage_out);
  for (auto& kv : ctx->tables) cudaFree(kv.second);
  for (auto& kv : ctx->mode_tables) cudaFree(kv.second);
  if (ctx->brdf_q) cudaFree(ctx->brdf_q);
  if (ctx->meta) cudaFree(ctx->meta);
  if (ctx->flux_defaults) cudaFree(ctx->flux_defaults);
  delete ctx;
  return DSP_OK;
}

dsp_status dsp_context_set_stream(dsp_context ctx, void* stream) {
  if (!ctx) return DSP_ERR_INVALID_INPUT;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return DSP_OK;
}

const char* dsp_context_last_error(dsp_context ctx) { return ctx ? ctx->last_error.c_str() : ""; }

dsp_status dsp_context_set_timing(dsp_context ctx, int32_t enable) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  ctx->timing = enable != 0;
  return DSP_OK;
}

dsp_status dsp_context_set_debug(dsp_context ctx, uint32_t flags) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  if (flags & ~DSP_DEBUG_POISON_SCRATCH) return fail(ctx, DSP_ERR_INVALID_INPUT, "unknown debug flag");
  ctx->debug = flags;
  return DSP_OK;
}

dsp_status dsp_context_set_schedule(dsp_context ctx, const dsp_schedule* entries, int32_t count) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  if (count < 0 || (count > 0 && !entries)) return fail(ctx, DSP_ERR_INVALID_INPUT, "schedule entries");
  for (int32_t k = 0; k < count; ++k) {
    const dsp_schedule& e = entries[k];
    if (e.min_layers > e.max_layers || e.layer_stage < 0 || e.layer_stage > 2 || e.persistent < 0 ||
        e.persistent > 2 || (e.layer_cta != 0 && e.layer_cta != 64 && e.layer_cta != 128))
      return fail(ctx, DSP_ERR_INVALID_INPUT, "schedule entry " + std::to_string(k) + " out of range");
  }
  ctx->schedule.assign(entries, entries + count);
  return DSP_OK;
}

dsp_status dsp_context_load_schedule_file(dsp_context ctx, const char* path) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  if (!path) return fail(ctx, DSP_ERR_INVALID_INPUT, "null path");
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(ctx, DSP_ERR_INVALID_INPUT, std::string("cannot open ") + path);
  std::vector<dsp_schedule> v;
  char line[512];
  int ln = 0;
  bool bad = false;
  while (std::fgets(line, sizeof(line), f)) {
    ++ln;
    if (char* h = std::strchr(line, '#')) *h = '\0';
    dsp_schedule e{};
    char extra = 0;
    const int got = std::sscanf(line, "%d %d %d %d %d %d %c", &e.num_streams, &e.min_layers, &e.max_layers,
                                &e.layer_stage, &e.layer_cta, &e.persistent, &extra);
    if (got <= 0) continue;  // blank or comment line
    if (got != 6) {
      bad = true;
      break;
    }
    v.push_back(e);
  }
  std::fclose(f);
  if (bad) return fail(ctx, DSP_ERR_INVALID_INPUT, std::string(path) + ": line " + std::to_string(ln) +
                                                       " is not 'N min_layers max_layers layer_stage layer_cta persistent'");
  return dsp_context_set_schedule(ctx, v.data(), (int32_t)v.size());
}

int32_t dsp_context_schedule_count(dsp_context ctx) { return ctx ? (int32_t)ctx->schedule.size() : 0; }

dsp_status dsp_context_timing_reset(dsp_context ctx) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  drain_timing(ctx);
  for (auto& v : ctx->kms) v = 0.0;
  for (auto& v : ctx->kcount) v = 0;
  return DSP_OK;
}

int32_t dsp_context_timing_count(dsp_context ctx) {
  if (!ctx) return 0;
  drain_timing(ctx);
  return (int32_t)ctx->knames.size();
}

dsp_status dsp_context_timing_get(dsp_context ctx, int32_t idx, const char** name, double* total_ms,
                                  int64_t* launches) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  drain_timing(ctx);
  if (idx < 0 || idx >= (int32_t)ctx->knames.size()) return DSP_ERR_INVALID_INPUT;
  if (name) *name = ctx->knames[idx].c_str();
  if (total_ms) *total_ms = ctx->kms[idx];
  if (launches) *launches = ctx->kcount[idx];
  return DSP_OK;
}

int64_t dsp_flux_workspace_bytes(const dsp_flux_batch* b) {
  if (!b || b->num_layers <= 0 || !supported_nstr(b->num_streams)) return -1;
  Sizes s = sizes_for(b->num_streams, b->num_layers);
  if (b->flags & DSP_FLAG_HG_G) s.inst += (size_t)round4(b->num_layers * b->pmom_count);
  if (b->flags & DSP_FLAG_SPHERICAL_BEAM) s.bvp += (size_t)b->num_layers * sph_stride(b->num_streams);
  return (int64_t)s.per_inst_bytes() * (int64_t)b->n_inst;
}

dsp_status dsp_flux_bands_solve(dsp_context ctx, const dsp_flux_batch* batch_in, const dsp_flux_out* out) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  NvtxRange r("dsp_flux_bands_solve");
  if (batch_in && (batch_in->flags & DSP_FLAG_TEMPERATURE_JAC))
    return fail(ctx, DSP_ERR_UNSUPPORTED, "temperature Jacobians are computed by dsp_flux_bands_solve_jac");
  return flux_solve(ctx, batch_in, out, nullptr);
}

dsp_status dsp_flux_bands_solve_jac(dsp_context ctx, const dsp_flux_batch* batch_in, const dsp_flux_out* out,
                                    const dsp_flux_jac_out* jac) {
  if (!ctx) return DSP_ERR_NOT_INITIALIZED;
  NvtxRange r("dsp_flux_bands_solve_jac");
  if (!jac || !jac->flux_up || !jac->flux_down || !jac->mean_intensity || !jac->mean_intensity_down ||
      !jac->mean_intensity_up || !jac->flux_divergence)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "every Jacobian output array is required");
  return flux_solve(ctx, batch_in, out, jac);
}

}  // extern "C"

namespace {

// The flux solve behind both entry points; `jac` (may be null) adds the
// temperature Jacobians.
dsp_status flux_solve(dsp_context ctx, const dsp_flux_batch* batch_in, const dsp_flux_out* out,
                      const dsp_flux_jac_out* jac) {
  if (!batch_in || !out) return fail(ctx, DSP_ERR_INVALID_INPUT, "null batch or output");
  dsp_flux_batch b = *batch_in;
  const int n = b.n_inst, N = b.num_streams, L = b.num_layers;
  if (n < 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "n_inst must be >= 0");
  if (n == 0) return DSP_OK;
  if (L <= 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "num_layers must be > 0");
  if (N < 4 || N % 2 != 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "num_streams must be even and >= 4");
  if (!supported_nstr(N))
    return fail(ctx, DSP_ERR_UNSUPPORTED, "Unsupported num_streams=" + std::to_string(N) +
                                              ". Supported values: 4, 6, 8, 10, 12, 14, 16, 32, 64");
  if (b.num_phase_func_moments < 0) return fail(ctx, DSP_ERR_INVALID_INPUT, "num_phase_func_moments must be >= 0");
  const int nmomnstr = b.num_phase_func_moments > N ? b.num_phase_func_moments : N;
  if (b.pmom_count < nmomnstr + 1)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "phase_function_moments size < nmomNstr()+1");
  const bool thermal = (b.flags & DSP_FLAG_THERMAL) != 0;
  const bool spherical = (b.flags & DSP_FLAG_SPHERICAL_BEAM) != 0;
  if (spherical && (!b.level_altitudes.ptr || !b.bottom_radius.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "the spherical beam needs level_altitudes and bottom_radius");
  if (!b.delta_tau.ptr || !b.single_scat_albedo.ptr || !b.phase_function_moments.ptr)
    return fail(ctx, DSP_ERR_INVALID_INPUT, "delta_tau, single_scat_albedo and phase_function_moments are required");
  if (thermal && (!b.temperature.ptr || !b.wavenumber_low.ptr || !b.wavenumber_high.ptr))
    return fail(ctx, DSP_ERR_INVALID_INPUT, "thermal emission needs temperature and wavenumber bands");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  cudaStream_t s = ctx->stream;
  const bool dev = (b.flags & DSP_FLAG_DEVICE_POINTERS) != 0;
  const int64_t nlev = L + 1;
  dsp_status st;

  // scalar defaults for absent per-instance scalars (DisortFluxConfig.hpp:30-44)
  static const double kDefaults[kFluxArrays] = {0, 0, 0, 0, 0, 0, 0.0, 1.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int64_t cnt[kFluxArrays];
  per_inst_counts(&b, cnt);

  // absent scalars read the DisortFluxConfig defaults from a device copy made once
  if (!ctx->flux_defaults) {
    e = cudaMalloc(&ctx->flux_defaults, sizeof(kDefaults));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->flux_defaults, kDefaults, sizeof(kDefaults), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (ctx->flux_defaults) cudaFree(ctx->flux_defaults);
      ctx->flux_defaults = nullptr;
      return cuda_fail(ctx, e, "flux defaults");
    }
  }
  // ---- stage host inputs into device memory --------------------------------
  dsp_darray* arr = batch_arrays(&b);
  const double* host_in[kFluxArrays] = {};  // per-instance host arrays still to be copied
  {
    size_t need = 0;
    for (int k = 0; k < kFluxArrays; ++k) {
      size_t elems;
      if (!arr[k].ptr) elems = 0;
      else if (dev) elems = 0;
      else elems = arr[k].stride == 0 ? (size_t)cnt[k] : (size_t)((n - 1) * arr[k].stride + cnt[k]);
      need += ((elems * sizeof(double) + 255) / 256) * 256;
    }
    if ((st = ensure(ctx, &ctx->stage_in, &ctx->stage_in_bytes, need + 256, "input staging")) != DSP_OK) return st;
    char* cur = static_cast<char*>(ctx->stage_in);
    for (int k = 0; k < kFluxArrays; ++k) {
      if (!arr[k].ptr) {
        if (kScalarField[k]) {  // absent scalar: the DisortFluxConfig default
          arr[k].ptr = ctx->flux_defaults + k;
          arr[k].stride = 0;
        }
        continue;
      }
      if (dev) continue;
      const size_t elems = arr[k].stride == 0 ? (size_t)cnt[k] : (size_t)((n - 1) * arr[k].stride + cnt[k]);
      if (arr[k].stride == 0) {  // shared by every instance: copied now
        e = cudaMemcpyAsync(cur, arr[k].ptr, elems * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(input)");
      } else {  // per instance: copied piece by piece below
        host_in[k] = arr[k].ptr;
      }
      arr[k].ptr = reinterpret_cast<const double*>(cur);
      cur += ((elems * sizeof(double) + 255) / 256) * 256;
    }
  }
  // ---- outputs -----------------------------------------------------------
  const int ndof = L + 2;  // Jacobian columns: level temperatures 0..L, surface
  double* dout[8];
  double* djac[6] = {};
  double* const hjac[6] = {jac ? jac->flux_up : nullptr, jac ? jac->flux_down : nullptr,
                           jac ? jac->mean_intensity : nullptr, jac ? jac->mean_intensity_down : nullptr,
                           jac ? jac->mean_intensity_up : nullptr, jac ? jac->flux_divergence : nullptr};
  int32_t* dstatus = nullptr;
  {
    double* host_out[8] = {out->flux_direct_beam, out->flux_down, out->flux_up, out->flux_tau_divergence,
                           out->mean_intensity, out->mean_intensity_down, out->mean_intensity_up,
                           out->mean_intensity_direct_beam};
    for (int f = 0; f < 8; ++f)
      if (!host_out[f]) return fail(ctx, DSP_ERR_INVALID_INPUT, "every output array is required");
    const size_t arr_bytes = ((size_t)n * nlev * sizeof(double) + 255) / 256 * 256;
    const size_t jac_bytes = jac ? ((size_t)n * nlev * ndof * sizeof(double) + 255) / 256 * 256 : 0;
    const size_t st_bytes = ((size_t)n * sizeof(int32_t) + 255) / 256 * 256;
    const size_t need = (dev ? 0 : 8 * arr_bytes + 6 * jac_bytes) + st_bytes;
    if ((st = ensure(ctx, &ctx->stage_out, &ctx->stage_out_bytes, need, "output staging")) != DSP_OK) return st;
    char* cur = static_cast<char*>(ctx->stage_out);
    for (int f = 0; f < 8; ++f) {
      if (dev) dout[f] = host_out[f];
      else {
        dout[f] = reinterpret_cast<double*>(cur);
        cur += arr_bytes;
      }
    }
    if (jac)
      for (int f = 0; f < 6; ++f) {
        if (dev) djac[f] = hjac[f];
        else {
          djac[f] = reinterpret_cast<double*>(cur);
          cur += jac_bytes;
        }
      }
    dstatus = (dev && out->status) ? out->status : reinterpret_cast<int32_t*>(cur);
  }
  e = cudaMemsetAsync(dstatus, 0, (size_t)n * sizeof(int32_t), s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemsetAsync(status)");

  const double* tables = nullptr;
  if ((st = get_tables(ctx, N, &tables)) != DSP_OK) return st;

  // ---- workspace and chunking -------------------------------------------
  // with DSP_FLAG_HG_G every instance also holds its formed moments [L][pc]
  const bool hg = (b.flags & DSP_FLAG_HG_G) != 0;
  const size_t hg_doubles = hg ? (size_t)round4(L * b.pmom_count) : 0;  // keeps the records 32-byte aligned
  Sizes sz = sizes_for(N, L);
  sz.inst += hg_doubles;
  // with Jacobians of a thermal solve: P/Q and multiplier records, and the
  // replayed right-hand side values [L][N][ndof]
  const bool jrecs = jac && thermal;
  const size_t jpq_d = jrecs ? (size_t)L * jpq_stride(N) : 0;
  const size_t jrec_d = jrecs ? (size_t)L * jrec_stride(N) : 0;
  const size_t jcv_d = jrecs ? (size_t)L * N * ndof : 0;
  // with the pseudo-spherical beam: the spherical record of every layer
  const size_t sph_d = spherical ? (size_t)L * sph_stride(N) : 0;
  sz.bvp += jpq_d + jrec_d + jcv_d + sph_d;
  const size_t inst_doubles = sz.inst + sz.layer + sz.bvp;
  size_t budget = workspace_budget();
  size_t freeb = 0, totalb = 0;
  if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && freeb / 2 < budget + ctx->ws_bytes)
    budget = (freeb + ctx->ws_bytes) / 2;
  int64_t chunk = (int64_t)(budget / sz.per_inst_bytes());
  if (chunk < 1) chunk = 1;
  if (chunk > n) chunk = n;

  FluxParams p0;
  p0.N = N;
  p0.L = L;
  p0.pc = b.pmom_count;
  p0.nmom = b.num_phase_func_moments;
  p0.flags = b.flags;
  p0.tables = tables;
  p0.pk = planck_consts();
  p0.il = InstLayout::make(L, N);
  // solves instances [r0, r1) on stream `cs`, `ch` at a time, in the workspace at `wsb`
  auto run_range = [&](int64_t r0, int64_t r1, cudaStream_t cs, double* wsb, int64_t ch) -> dsp_status {
    FluxParams p = p0;
    DArr* pa[kFluxArrays] = {&p.wlo, &p.whi, &p.dtau, &p.ssa, &p.pmom, &p.temp, &p.alb, &p.emis,
                             &p.fbeam, &p.umu0, &p.fisot, &p.fisob, &p.ttop, &p.tbot, &p.zalt, &p.rbot};
    for (int64_t off = r0; off < r1; off += ch) {
      const int64_t m = (r1 - off < ch) ? (r1 - off) : ch;
      p.n = (int)m;
      if (ctx->debug & DSP_DEBUG_POISON_SCRATCH) {
        const cudaError_t pe = cudaMemsetAsync(wsb, 0xFF, (size_t)m * inst_doubles * sizeof(double), cs);
        if (pe != cudaSuccess) return cuda_fail(ctx, pe, "scratch poison");
      }
      for (int k = 0; k < kFluxArrays; ++k) {
        pa[k]->p = arr[k].ptr ? arr[k].ptr + arr[k].stride * off : nullptr;
        pa[k]->s = arr[k].stride;
      }
      p.inst_rec = wsb;
      p.layer_rec = wsb + (size_t)m * sz.inst;
      p.bvp_rec = p.layer_rec + (size_t)m * sz.layer;
      for (int f = 0; f < 8; ++f) p.out[f] = dout[f] + off * nlev;
      p.status = dstatus + off;
      // the spherical and Jacobian areas follow the elimination records of the chunk
      double* xbase = p.bvp_rec + (size_t)m * (sz.bvp - jpq_d - jrec_d - jcv_d - sph_d);
      p.sph = spherical ? xbase : nullptr;
      JacView jv;
      if (jac) {
        double* jbase = xbase + (size_t)m * sph_d;
        p.jac_pq = jrecs ? jbase : nullptr;
        p.jac_rec = jrecs ? jbase + (size_t)m * jpq_d : nullptr;
        jv.cv = jrecs ? jbase + (size_t)m * (jpq_d + jrec_d) : nullptr;
        jv.ndof = ndof;
        for (int f = 0; f < 6; ++f) jv.out[f] = djac[f] + off * nlev * ndof;
      }
      if (hg) {  // g per layer -> moments at the end of the instance-record area
        double* mom = wsb + (size_t)m * (sz.inst - hg_doubles);
        const long long rows = m * (long long)L;
        const long long threads = rows * p.pc;
        {
          KernelTimer kt(ctx, "hg_moments_kernel", cs);
          hg_moments_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, cs>>>(p.pmom, rows, L, p.pc, mom);
        }
        p.pmom.p = mom;
        p.pmom.s = (long long)L * p.pc;
      }
      dsp_status rs = launch_flux(ctx, N, p, cs, jac ? &jv : nullptr);
      if (rs != DSP_OK) return rs;
    }
    return DSP_OK;
  };
  if (dev) {
    const size_t ws_need = (size_t)chunk * inst_doubles * sizeof(double) + 1024;
    if ((st = ensure(ctx, &ctx->ws, &ctx->ws_bytes, ws_need, "workspace")) != DSP_OK) return st;
    return run_range(0, n, s, static_cast<double*>(ctx->ws), chunk);
  }

  // ---- host buffers: copies overlapped with the solves ----------------------
  // The batch is cut into pieces of whole boundary-value waves (the instances
  // that kernel keeps resident at once), about a quarter of the batch each, the
  // remainder last.  Piece k's inputs go up on a copy stream, it is solved on
  // one of two solve streams (alternating, each with its own half of the
  // workspace) and its outputs come back on a second copy stream, so the next
  // piece's kernels fill the GPU while a piece's last wave drains.  (With
  // pageable host memory the copies do not overlap, but the results are the same.)
  double* host_out[8] = {out->flux_direct_beam, out->flux_down, out->flux_up, out->flux_tau_divergence,
                         out->mean_intensity, out->mean_intensity_down, out->mean_intensity_up,
                         out->mean_intensity_direct_beam};
  std::vector<int32_t> hst;
  int32_t* hs = out->status;
  if (!hs) {
    hst.resize(n);
    hs = hst.data();
  }
  constexpr int kMaxPieces = 8;
  const int64_t wave = std::max<int64_t>(1, bvp_wave(N, ctx->sm_count));
  const int64_t waves = (n + wave - 1) / wave;
  int64_t piece = wave * std::max<int64_t>(1, waves / 4);
  while ((n + piece - 1) / piece > kMaxPieces - 1) piece += wave;
  piece = std::min<int64_t>(piece, n);
  // the first piece is one wave when the others are larger: the solves start
  // after a shorter upload
  const int64_t first = std::min<int64_t>(piece, wave);
  const int pieces = 1 + (int)((n - first + piece - 1) / piece);
  // two workspace halves when they fit the budget, else one stream and `chunk`
  const bool dual = pieces > 1 && piece <= chunk / 2;
  const int64_t ch = dual ? piece : chunk;
  const size_t half = (size_t)ch * inst_doubles;
  const size_t ws_need = (dual ? 2 : 1) * half * sizeof(double) + 1024;
  if ((st = ensure(ctx, &ctx->ws, &ctx->ws_bytes, ws_need, "workspace")) != DSP_OK) return st;
  if (!ctx->s_in) {
    e = cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->s_c2, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy streams");
  }
  while ((int)ctx->pipe_ev.size() < 2 * kMaxPieces + 1) {
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pipeline events");
    ctx->pipe_ev.push_back(ev);
  }
  cudaEvent_t* ev_in = ctx->pipe_ev.data();
  cudaEvent_t* ev_done = ev_in + kMaxPieces;
  cudaEvent_t ev_start = ctx->pipe_ev[2 * kMaxPieces];
  // the staging areas and the workspace may still be used by earlier work on
  // the context's stream (and the status memset above runs there)
  e = cudaEventRecord(ev_start, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_in, ev_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_c2, ev_start, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pipeline start");
  double* const ws0 = static_cast<double*>(ctx->ws);
  for (int k = 0; k < pieces; ++k) {
    const int64_t r0 = k == 0 ? 0 : first + piece * (k - 1), r1 = std::min<int64_t>(n, first + piece * k);
    cudaStream_t cs = (dual && (k & 1)) ? ctx->s_c2 : s;
    for (int a = 0; a < kFluxArrays; ++a) {
      if (!host_in[a]) continue;
      const int64_t e0 = r0 * arr[a].stride, e1 = (r1 - 1) * arr[a].stride + cnt[a];
      e = cudaMemcpyAsync(const_cast<double*>(arr[a].ptr) + e0, host_in[a] + e0, (size_t)(e1 - e0) * sizeof(double),
                          cudaMemcpyHostToDevice, ctx->s_in);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(input)");
    }
    e = cudaEventRecord(ev_in[k], ctx->s_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ev_in[k], 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pipeline input");
    if ((st = run_range(r0, r1, cs, ws0 + ((dual && (k & 1)) ? half : 0), ch)) != DSP_OK) return st;
    e = cudaEventRecord(ev_done[k], cs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_out, ev_done[k], 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pipeline output");
    for (int f = 0; f < 8; ++f) {
      e = cudaMemcpyAsync(host_out[f] + r0 * nlev, dout[f] + r0 * nlev, (size_t)(r1 - r0) * nlev * sizeof(double),
                          cudaMemcpyDeviceToHost, ctx->s_out);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(output)");
    }
    e = cudaMemcpyAsync(hs + r0, dstatus + r0, (size_t)(r1 - r0) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                        ctx->s_out);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(status)");
    if (jac)
      for (int f = 0; f < 6; ++f) {
        const int64_t per = nlev * ndof;
        e = cudaMemcpyAsync(hjac[f] + r0 * per, djac[f] + r0 * per, (size_t)(r1 - r0) * per * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->s_out);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(jacobian)");
      }
  }
  // later work on the context's stream sees the whole solve
  e = cudaEventRecord(ev_start, ctx->s_c2);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev_start, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->s_out);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "flux solve");
  return DSP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// CUDA graph of a device-pointer flux solve (no reference counterpart)
// ---------------------------------------------------------------------------
struct dsp_graph_s {
  dsp_context ctx = nullptr;  // private: its workspace addresses are baked into the graph
  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

extern "C" dsp_status dsp_flux_graph_create(int32_t device, const dsp_flux_batch* batch, const dsp_flux_out* out,
                                            dsp_graph* g) {
  if (!batch || !out || !g) return DSP_ERR_INVALID_INPUT;
  *g = nullptr;
  if (!(batch->flags & DSP_FLAG_DEVICE_POINTERS) || (batch->flags & DSP_FLAG_TEMPERATURE_JAC)) return DSP_ERR_INVALID_INPUT;
  dsp_graph_s* gr = new dsp_graph_s;
  gr->device = device;
  auto bail = [&](dsp_status st) {
    if (gr->exec) cudaGraphExecDestroy(gr->exec);
    if (gr->graph) cudaGraphDestroy(gr->graph);
    if (gr->ctx) dsp_context_destroy(gr->ctx);
    if (gr->cs) cudaStreamDestroy(gr->cs);
    delete gr;
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&gr->cs, cudaStreamNonBlocking) != cudaSuccess)
    return bail(DSP_ERR_CUDA);
  dsp_status st = dsp_context_create(device, gr->cs, &gr->ctx);
  if (st != DSP_OK) return bail(st);
  // a first solve sizes the workspace and uploads the tables, so that the
  // captured solve consists of memsets and kernel launches only
  if ((st = flux_solve(gr->ctx, batch, out, nullptr)) != DSP_OK) return bail(st);
  if (cudaStreamSynchronize(gr->cs) != cudaSuccess) return bail(DSP_ERR_CUDA);
  if (cudaStreamBeginCapture(gr->cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) return bail(DSP_ERR_CUDA);
  st = flux_solve(gr->ctx, batch, out, nullptr);
  const cudaError_t ec = cudaStreamEndCapture(gr->cs, &gr->graph);
  if (st != DSP_OK) return bail(st);
  if (ec != cudaSuccess || !gr->graph) return bail(DSP_ERR_CUDA);
  if (cudaGraphInstantiate(&gr->exec, gr->graph, 0) != cudaSuccess) return bail(DSP_ERR_CUDA);
  *g = gr;
  return DSP_OK;
}

extern "C" dsp_status dsp_graph_launch(dsp_graph g, void* stream) {
  if (!g) return DSP_ERR_INVALID_INPUT;
  if (cudaSetDevice(g->device) != cudaSuccess) return DSP_ERR_CUDA;
  return cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? DSP_OK : DSP_ERR_CUDA;
}

extern "C" dsp_status dsp_graph_destroy(dsp_graph g) {
  if (!g) return DSP_ERR_INVALID_INPUT;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->cs);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->ctx) dsp_context_destroy(g->ctx);
  if (g->cs) cudaStreamDestroy(g->cs);
  delete g;
  return DSP_OK;
}
