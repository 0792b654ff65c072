// oracle_capi.cpp — C entry points of the CPU oracle (liboracle_disort.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py, never by the product.
//
// oracle_flux_bands_solve mirrors the reference spectral loop
// solveFluxSpectralBandsImpl<N> (src/python_bindings.cpp:170-190): an OpenMP
// parallel region with one solver object per thread and a static schedule
// over the bands.  It takes the same dsp_flux_batch as the GPU library, with
// host pointers.
#include <omp.h>

#include "flux_oracle.hpp"

namespace {
inline const double* at(const dsp_darray& a, int64_t i) {
  return a.ptr ? a.ptr + a.stride * i : nullptr;
}
inline double scalar(const dsp_darray& a, int64_t i, double dflt) {
  return a.ptr ? a.ptr[a.stride * i] : dflt;
}
}  // namespace

extern "C" {

int oracle_flux_bands_solve(const dsp_flux_batch* b, const dsp_flux_out* o, int nthreads) {
  if (!b || !o) return DSP_ERR_INVALID_INPUT;
  const int n = b->n_inst;
  const int L = b->num_layers;
  const int64_t nlev = L + 1;
  int worst = DSP_OK;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    oracle::FluxOracle solver;
    int local_worst = DSP_OK;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      oracle::FluxInstance c;
      c.num_layers = L;
      c.num_streams = b->num_streams;
      c.num_phase_func_moments = b->num_phase_func_moments;
      c.pmom_count = b->pmom_count;
      c.thermal = (b->flags & DSP_FLAG_THERMAL) != 0;
      c.delta_m_plus = (b->flags & DSP_FLAG_DELTA_M_PLUS) != 0;
      c.diffusion_lower_bc = (b->flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
      c.index_from_bottom = (b->flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
      c.wavenumber_low = scalar(b->wavenumber_low, i, 0.0);
      c.wavenumber_high = scalar(b->wavenumber_high, i, 0.0);
      c.surface_albedo = scalar(b->surface_albedo, i, 0.0);
      c.emissivity_top = scalar(b->emissivity_top, i, 1.0);
      c.direct_beam_flux = scalar(b->direct_beam_flux, i, 0.0);
      c.direct_beam_mu = scalar(b->direct_beam_mu, i, 0.5);
      c.isotropic_flux_top = scalar(b->isotropic_flux_top, i, 0.0);
      c.isotropic_flux_bottom = scalar(b->isotropic_flux_bottom, i, 0.0);
      c.temperature_top = scalar(b->temperature_top, i, 0.0);
      c.temperature_bottom = scalar(b->temperature_bottom, i, 0.0);
      c.delta_tau = at(b->delta_tau, i);
      c.ssa = at(b->single_scat_albedo, i);
      c.pmom = at(b->phase_function_moments, i);
      c.temperature = at(b->temperature, i);
      oracle::FluxOutput fo{o->flux_direct_beam + nlev * i, o->flux_down + nlev * i,
                            o->flux_up + nlev * i, o->flux_tau_divergence + nlev * i,
                            o->mean_intensity + nlev * i, o->mean_intensity_down + nlev * i,
                            o->mean_intensity_up + nlev * i, o->mean_intensity_direct_beam + nlev * i};
      int st;
      if ((b->flags & (DSP_FLAG_SPHERICAL_BEAM | DSP_FLAG_TEMPERATURE_JAC)) != 0) {
        st = DSP_ERR_UNSUPPORTED;
      } else if (!c.delta_tau || !c.ssa || !c.pmom) {
        st = DSP_ERR_INVALID_INPUT;
      } else {
        st = solver.solve(c, fo);
      }
      if (o->status) o->status[i] = st;
      if (st > local_worst) local_worst = st;
    }
#pragma omp critical
    if (local_worst > worst) worst = local_worst;
  }
  return worst;
}

// Gauss-Legendre nodes/weights and Legendre table as the reference builds them
// (FluxSolver.cpp:257-290 and :126); used by tests to cross-check the engine's
// per-stream constant tables.
int oracle_quadrature(int nstr, double* mu, double* w, double* ylm) {
  if (nstr < 2 || nstr % 2) return DSP_ERR_INVALID_INPUT;
  if (!oracle::gauss_quadrature(nstr / 2, mu, w)) return DSP_ERR_EIGEN;
  oracle::legendre_flat(nstr, 0, nstr, nstr - 1, mu, ylm);
  return DSP_OK;
}

double oracle_planck(double wnumlo, double wnumhi, double temp) {
  return oracle::planck_function2(wnumlo, wnumhi, temp);
}

}  // extern "C"
