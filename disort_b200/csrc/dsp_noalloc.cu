// dsp_noalloc.cu — a flux solve that performs no device or host allocation.
//
// Some callers cannot let a library allocate GPU memory: a host application
// that hands the whole device to its own pooled allocator (and must account for
// every byte), or an embedding that forbids allocation after start-up.  For
// them, dsp_flux_bands_solve_noalloc runs the same kernels as
// dsp_flux_bands_solve, but its workspace is a fixed array compiled into the
// library (g_noalloc_scratch, 32 MiB of device memory that every GPU which loads
// libdsp.so keeps until the process exits), and it needs no dsp_context (a
// context owns allocations).  Inputs and outputs are the caller's device buffers.
//
// Rules of use:
//  - Every pointer in the batch and in the output must be device memory; the
//    batch must carry DSP_FLAG_DEVICE_POINTERS.
//  - One instance's workspace must fit in the array (a 60-layer, 16-stream
//    instance needs about 0.4 MB; the limit is reached near 330 layers at 64
//    streams); larger instances are rejected with DSP_ERR_NO_MEMORY before any
//    work is queued.  Bigger batches run as several launches that reuse the array.
//  - The array is shared by every call on a device and keeps the last call's
//    contents; the per-instance status words are cleared at the start of each
//    launch.  Calls that can overlap on the GPU (different streams, or
//    different host threads without ordering) race on the array; serialise them.
//  - Every call looks up the array's device address on the current device with
//    cudaGetSymbolAddress (no allocation, not a stream operation), so a device
//    reset or a new primary context between calls is harmless, and sets the
//    kernel attributes of its stream count.
//  - Every call copies the quadrature tables and the defaults of absent scalar
//    inputs from pageable host memory into the array; such copies are staged by
//    the driver before the call returns, so the call is not fully asynchronous
//    with respect to the host.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/dsp.h"
#include "dsp_device.cuh"
#include "flux_bvp_tile.cuh"
#include "flux_bvp_reg.cuh"
#include "flux_layer.cuh"
#include "flux_setup.cuh"

using namespace dsp;

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
// The workspace.  In host code this name is only a stand-in symbol, never a
// device address: the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

const int kSupported[] = {4, 6, 8, 10, 12, 14, 16, 32, 64};

// Quadrature / Legendre tables as the reference builds them (FluxSolver.cpp:257-290, :126).
bool tables_for(int N, std::vector<double>& tab) {
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
    y[i] = 1.0;
    y[N + i] = mu[i];
  }
  for (int l = 2; l < N; ++l)
    for (int i = 0; i < N; ++i)
      y[l * N + i] = ((2.0 * l - 1.0) * mu[i] * y[(l - 1) * N + i] - (l - 1.0) * y[(l - 2) * N + i]) / l;
  return true;
}

template <int N>
void set_attrs() {
  flux_layer_set_attrs<N>();
  if constexpr (N > 16)
    cudaFuncSetAttribute(flux_bvp_tile_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TCfg<N>::smem_bytes());
}

template <int N>
void launch(const FluxParams& p, const double* host_tab, cudaStream_t s) {
  flux_setup_kernel<<<(p.n + 3) / 4, 128, 0, s>>>(p);
  flux_layer_launch<N>(p, host_tab, s, [](const char*, auto&& launch) { launch(); });
  if constexpr (N <= 16) {
    using C = RCfg<N>;
    flux_bvp_reg_kernel<N><<<(p.n + C::TPC - 1) / C::TPC, C::CTA, C::smem_bytes(), s>>>(p);
  } else {
    using C = TCfg<N>;
    flux_bvp_tile_kernel<N><<<(p.n + C::TPC - 1) / C::TPC, C::CTA, C::smem_bytes(), s>>>(p);
  }
}

template <int N>
void dispatch_attrs_or_launch(bool attrs, const FluxParams* p, const double* host_tab, cudaStream_t s) {
  if (attrs) set_attrs<N>();
  else launch<N>(*p, host_tab, s);
}

bool run_for(int N, bool attrs, const FluxParams* p, const double* host_tab, cudaStream_t s) {
  switch (N) {
    case 4: dispatch_attrs_or_launch<4>(attrs, p, host_tab, s); return true;
    case 6: dispatch_attrs_or_launch<6>(attrs, p, host_tab, s); return true;
    case 8: dispatch_attrs_or_launch<8>(attrs, p, host_tab, s); return true;
    case 10: dispatch_attrs_or_launch<10>(attrs, p, host_tab, s); return true;
    case 12: dispatch_attrs_or_launch<12>(attrs, p, host_tab, s); return true;
    case 14: dispatch_attrs_or_launch<14>(attrs, p, host_tab, s); return true;
    case 16: dispatch_attrs_or_launch<16>(attrs, p, host_tab, s); return true;
    case 32: dispatch_attrs_or_launch<32>(attrs, p, host_tab, s); return true;
    case 64: dispatch_attrs_or_launch<64>(attrs, p, host_tab, s); return true;
  }
  return false;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int64_t dsp_noalloc_scratch_bytes(void) { return (int64_t)kScratchBytes; }

dsp_status dsp_flux_bands_solve_noalloc(const dsp_flux_batch* batch_in, const dsp_flux_out* out, void* stream) {
  if (!batch_in || !out) return DSP_ERR_INVALID_INPUT;
  dsp_flux_batch b = *batch_in;
  const int n = b.n_inst, N = b.num_streams, L = b.num_layers;
  if (!(b.flags & DSP_FLAG_DEVICE_POINTERS)) return DSP_ERR_INVALID_INPUT;  // cannot stage host buffers
  if (n < 0 || L <= 0 || N < 4 || N % 2) return DSP_ERR_INVALID_INPUT;
  if (n == 0) return DSP_OK;
  bool ok = false;
  for (int sN : kSupported) ok = ok || sN == N;
  if (!ok) return DSP_ERR_UNSUPPORTED;
  if (b.flags & (DSP_FLAG_SPHERICAL_BEAM | DSP_FLAG_TEMPERATURE_JAC | DSP_FLAG_HG_G)) return DSP_ERR_UNSUPPORTED;
  const int nmomnstr = b.num_phase_func_moments > N ? b.num_phase_func_moments : N;
  if (b.num_phase_func_moments < 0 || b.pmom_count < nmomnstr + 1) return DSP_ERR_INVALID_INPUT;
  if (!b.delta_tau.ptr || !b.single_scat_albedo.ptr || !b.phase_function_moments.ptr) return DSP_ERR_INVALID_INPUT;
  if ((b.flags & DSP_FLAG_THERMAL) && (!b.temperature.ptr || !b.wavenumber_low.ptr || !b.wavenumber_high.ptr))
    return DSP_ERR_INVALID_INPUT;
  double* outs[8] = {out->flux_direct_beam, out->flux_down, out->flux_up, out->flux_tau_divergence,
                     out->mean_intensity, out->mean_intensity_down, out->mean_intensity_up,
                     out->mean_intensity_direct_beam};
  for (double* o : outs)
    if (!o) return DSP_ERR_INVALID_INPUT;

  // ---- scratch layout: [defaults | tables | status | inst | layer | bvp records]
  const InstLayout il = InstLayout::make(L, N);
  const size_t per_inst = (size_t)il.stride + (size_t)L * lrec_stride(N) + (size_t)L * brec_stride(N);
  const size_t head = align256(16 * sizeof(double)) + align256((size_t)tab_size(N) * sizeof(double));
  const size_t per_inst_bytes = per_inst * sizeof(double) + sizeof(int32_t);
  // room for the status words (rounded up to 256 bytes) and the records of
  // `chunk` instances; at least one instance must fit before any work is queued
  const size_t room = kScratchBytes > head + 512 ? kScratchBytes - head - 512 : 0;
  const int64_t fit = (int64_t)(room / per_inst_bytes);
  if (fit < 1) return DSP_ERR_NO_MEMORY;  // one instance is too big for the array
  const int64_t chunk = fit < n ? fit : n;

  // the array's address on the current device, looked up on every call
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
    cudaGetLastError();
    return DSP_ERR_CUDA;
  }
  unsigned char* base = static_cast<unsigned char*>(ptr);
  run_for(N, true, nullptr, nullptr, nullptr);  // kernel attributes of this stream count
  if (cudaGetLastError() != cudaSuccess) return DSP_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // defaults of absent scalar fields (DisortFluxConfig.hpp:30-44) and the tables;
  // the copies read pageable host memory, so the driver stages them before returning
  static const double kDefaults[14] = {0, 0, 0, 0, 0, 0, 0.0, 1.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0};
  double* d_def = reinterpret_cast<double*>(base);
  double* d_tab = reinterpret_cast<double*>(base + align256(16 * sizeof(double)));
  if (cudaMemcpyAsync(d_def, kDefaults, sizeof(kDefaults), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return DSP_ERR_CUDA;
  std::vector<double> tab;
  if (!tables_for(N, tab)) return DSP_ERR_EIGEN;
  if (cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return DSP_ERR_CUDA;
  dsp_darray* arr = &b.wavenumber_low;
  for (int k = 0; k < 14; ++k)
    if (!arr[k].ptr && (k <= 1 || k >= 6)) {
      arr[k].ptr = d_def + k;
      arr[k].stride = 0;
    }

  unsigned char* cur = base + head;
  int32_t* d_status = reinterpret_cast<int32_t*>(cur);
  double* d_rec = reinterpret_cast<double*>(cur + align256((size_t)chunk * sizeof(int32_t)));

  FluxParams p;
  p.N = N;
  p.L = L;
  p.pc = b.pmom_count;
  p.nmom = b.num_phase_func_moments;
  p.flags = b.flags;
  p.tables = d_tab;
  p.pk.vmax = std::log(DBL_MAX);
  p.pk.sigdpi = 5.67032E-8 / M_PI;
  p.pk.conc = 15.0 / std::pow(M_PI, 4.0);
  p.pk.c1 = 1.1911e-8;
  p.il = il;
  DArr* pa[14] = {&p.wlo, &p.whi, &p.dtau, &p.ssa, &p.pmom, &p.temp, &p.alb,
                  &p.emis, &p.fbeam, &p.umu0, &p.fisot, &p.fisob, &p.ttop, &p.tbot};
  const int64_t nlev = L + 1;
  for (int64_t off = 0; off < n; off += chunk) {
    const int64_t m = (n - off < chunk) ? (n - off) : chunk;
    p.n = (int)m;
    for (int k = 0; k < 14; ++k) {
      pa[k]->p = arr[k].ptr ? arr[k].ptr + arr[k].stride * off : nullptr;
      pa[k]->s = arr[k].stride;
    }
    p.inst_rec = d_rec;
    p.layer_rec = d_rec + (size_t)m * il.stride;
    p.bvp_rec = p.layer_rec + (size_t)m * L * lrec_stride(N);
    for (int f = 0; f < 8; ++f) p.out[f] = outs[f] + off * nlev;
    // statuses start at zero: in the caller's array when given, else in the scratch
    p.status = out->status ? out->status + off : d_status;
    if (cudaMemsetAsync(p.status, 0, (size_t)m * sizeof(int32_t), s) != cudaSuccess) return DSP_ERR_CUDA;
    run_for(N, false, &p, tab.data(), s);
    if (cudaGetLastError() != cudaSuccess) return DSP_ERR_CUDA;
  }
  return DSP_OK;
}

}  // extern "C"
