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

#include "general_oracle.hpp"

namespace {
inline const double* at(const dsp_darray& a, int64_t i) {
  return a.ptr ? a.ptr + a.stride * i : nullptr;
}
inline double scalar(const dsp_darray& a, int64_t i, double dflt) {
  return a.ptr ? a.ptr[a.stride * i] : dflt;
}
}  // namespace

extern "C" {

int oracle_flux_bands_solve_jac(const dsp_flux_batch* b, const dsp_flux_out* o, const dsp_flux_jac_out* jac,
                                int nthreads);

int oracle_flux_bands_solve(const dsp_flux_batch* b, const dsp_flux_out* o, int nthreads) {
  if (b && (b->flags & DSP_FLAG_TEMPERATURE_JAC)) return DSP_ERR_UNSUPPORTED;
  return oracle_flux_bands_solve_jac(b, o, nullptr, nthreads);
}

// The flux batch with optional temperature Jacobians (jac may be null).
int oracle_flux_bands_solve_jac(const dsp_flux_batch* b, const dsp_flux_out* o, const dsp_flux_jac_out* jac,
                                int nthreads) {
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
      if (jac) {
        const int64_t js = nlev * (L + 2);
        double* const jp[6] = {jac->flux_up, jac->flux_down, jac->mean_intensity, jac->mean_intensity_down,
                               jac->mean_intensity_up, jac->flux_divergence};
        for (int f = 0; f < 6; ++f) fo.jac[f] = jp[f] + js * i;
        c.temperature_jac = true;
      }
      int st;
      c.spherical = (b->flags & DSP_FLAG_SPHERICAL_BEAM) != 0;
      c.level_altitudes = at(b->level_altitudes, i);
      c.bottom_radius = scalar(b->bottom_radius, i, 0.0);
      if (!c.delta_tau || !c.ssa || !c.pmom) {
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

// The general batch (DisortSolver::solve per instance), same static-schedule
// OpenMP loop as the flux batch.  Instances are ragged: instance i owns layers
// layer_offset[i] .. layer_offset[i+1]-1 and levels layer_offset[i] + i ..
// layer_offset[i+1] + i.
int oracle_general_bands_solve_jac(const dsp_general_batch* b, const dsp_general_out* o,
                                   const dsp_general_jac_out* jac, int nthreads);

int oracle_general_bands_solve(const dsp_general_batch* b, const dsp_general_out* o, int nthreads) {
  if (b && (b->flags & DSP_FLAG_TEMPERATURE_JAC)) return DSP_ERR_UNSUPPORTED;
  return oracle_general_bands_solve_jac(b, o, nullptr, nthreads);
}

// The general batch with optional temperature Jacobians (jac may be null).
int oracle_general_bands_solve_jac(const dsp_general_batch* b, const dsp_general_out* o,
                                   const dsp_general_jac_out* jac, int nthreads) {
  if (!b || !o || b->n_inst < 0) return DSP_ERR_INVALID_INPUT;
  const int n = b->n_inst;
  const uint32_t fl = b->flags;
  const int64_t ntau_o = o->ntau_out, numu_o = o->numu_out, nphi = b->num_phi > 0 ? b->num_phi : 0;
  int worst = DSP_OK;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    oracle::GeneralOracle solver;
    int local_worst = DSP_OK;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      oracle::GeneralInstance c;
      int st = DSP_OK;
      if (!b->num_streams || !b->num_layers || !b->layer_offset || !b->num_phase_func_moments ||
          !b->delta_tau || !b->single_scat_albedo || !b->phase_function_moments) {
        st = DSP_ERR_INVALID_INPUT;
      } else {
        const int64_t l0 = b->layer_offset[i];
        c.L = b->num_layers[i];
        c.N = b->num_streams[i];
        c.nmom = b->num_phase_func_moments[i];
        c.pc = b->pmom_count;
        c.thermal = (fl & DSP_FLAG_THERMAL) != 0;
        c.dmplus = (fl & DSP_FLAG_DELTA_M_PLUS) != 0;
        c.dlbc = (fl & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
        c.ifb = (fl & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
        c.user_tau = (fl & DSP_GFLAG_USER_TAU) != 0;
        c.user_mu = (fl & DSP_GFLAG_USER_MU) != 0;
        c.only_fluxes = (fl & DSP_GFLAG_ONLY_FLUXES) != 0;
        c.corr = (fl & DSP_GFLAG_INTENSITY_CORR) != 0;
        c.corr_be = c.corr && (fl & DSP_GFLAG_INTENSITY_CORR_BE) != 0;
        if (c.corr_be) {
          c.nangles = b->num_phase_func_angles;
          c.mup = at(b->mu_phase_function, i);
          c.phasef = b->phase_function ? b->phase_function + l0 * b->num_phase_func_angles : nullptr;
        }
        c.accur = b->accuracy_fourier_series;
        c.wlo = scalar(b->wavenumber_low, i, 0.0);
        c.whi = scalar(b->wavenumber_high, i, 0.0);
        c.alb = scalar(b->surface_albedo, i, 0.0);
        c.emis = scalar(b->emissivity_top, i, 1.0);
        c.fbeam = scalar(b->direct_beam_flux, i, 0.0);
        c.umu0 = scalar(b->direct_beam_mu, i, 0.5);
        c.phi0 = scalar(b->direct_beam_phi, i, 0.0);
        c.fisot = scalar(b->isotropic_flux_top, i, 0.0);
        c.fisob = scalar(b->isotropic_flux_bottom, i, 0.0);
        c.ttop = scalar(b->temperature_top, i, 0.0);
        c.tbot = scalar(b->temperature_bottom, i, 0.0);
        c.dtau = b->delta_tau + l0;
        c.ssa = b->single_scat_albedo + l0;
        c.pmom = b->phase_function_moments + l0 * b->pmom_count;
        c.temp = b->temperature ? b->temperature + l0 + i : nullptr;
        c.ntau = b->num_user_tau;
        c.numu = b->num_user_mu;
        c.nphi = b->num_phi;
        c.utau = at(b->tau_user, i);
        c.umu = at(b->mu_user, i);
        c.phi = at(b->phi_user, i);
        const int ntau = c.user_tau ? c.ntau : c.L + 1;
        const int numu = (c.user_mu && !c.only_fluxes) ? c.numu : c.N;
        c.spherical = (fl & DSP_FLAG_SPHERICAL_BEAM) != 0;
        c.zalt = b->level_altitudes ? b->level_altitudes + l0 + i : nullptr;
        c.radius = scalar(b->bottom_radius, i, 0.0);
        c.brdf = b->brdf_type;
        c.bp = c.brdf ? at(b->brdf_params, i) : nullptr;
        if (c.L > 0 && b->layer_offset[i + 1] - l0 != c.L) st = DSP_ERR_INVALID_INPUT;
        else if (c.brdf < 0 || c.brdf > 4 || (c.brdf && !c.bp)) st = DSP_ERR_INVALID_INPUT;
        else if (c.corr_be && (c.nangles < 2 || !c.mup || !c.phasef)) st = DSP_ERR_INVALID_INPUT;
        else if (ntau > ntau_o || numu > numu_o || c.N > 64) st = DSP_ERR_INVALID_INPUT;
        else if (jac && jac->ndof_out < c.L + 2) st = DSP_ERR_INVALID_INPUT;
        else {
          oracle::GeneralOutput go;
          for (int f = 0; f < 8; ++f) go.flux[f] = o->flux[f] + ntau_o * i;
          if (jac) {
            const int64_t js = ntau_o * jac->ndof_out;
            double* const jp[6] = {jac->flux_up, jac->flux_down, jac->mean_intensity, jac->mean_intensity_down,
                                   jac->mean_intensity_up, jac->flux_divergence};
            for (int f = 0; f < 6; ++f) go.jac[f] = jp[f] + js * i;
            go.jac_stride = jac->ndof_out;
            c.temperature_jac = true;
          }
          go.intensity = o->intensity ? o->intensity + (ntau_o * numu_o * nphi) * i : nullptr;
          go.iavg = o->intensity_azimuth_avg ? o->intensity_azimuth_avg + (ntau_o * numu_o) * i : nullptr;
          go.ntau_out = (int)ntau_o;
          go.numu_out = (int)numu_o;
          if (!c.only_fluxes && c.user_mu && (!go.intensity || !go.iavg)) st = DSP_ERR_INVALID_INPUT;
          else st = solver.solve(c, go);
        }
      }
      if (o->status) o->status[i] = st;
      if (st > local_worst) local_worst = st;
    }
#pragma omp critical
    if (local_worst > worst) worst = local_worst;
  }
  return worst;
}

// ibcnd = Special per instance (computeAlbTrans restated in general_oracle.hpp)
int oracle_general_bands_albtrans(const dsp_general_batch* b, const dsp_albtrans_out* o, int nthreads) {
  if (!b || !o || b->n_inst < 0) return DSP_ERR_INVALID_INPUT;
  const int n = b->n_inst;
  const uint32_t fl = b->flags;
  int worst = DSP_OK;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    oracle::GeneralOracle solver;
    int local_worst = DSP_OK;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      oracle::GeneralInstance c;
      int st = DSP_OK;
      if (!b->num_streams || !b->num_layers || !b->layer_offset || !b->num_phase_func_moments ||
          !b->delta_tau || !b->single_scat_albedo || !b->phase_function_moments) {
        st = DSP_ERR_INVALID_INPUT;
      } else {
        const int64_t l0 = b->layer_offset[i];
        c.special = true;
        c.L = b->num_layers[i];
        c.N = b->num_streams[i];
        c.nmom = b->num_phase_func_moments[i];
        c.pc = b->pmom_count;
        c.dmplus = (fl & DSP_FLAG_DELTA_M_PLUS) != 0;
        c.ifb = (fl & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
        c.user_mu = (fl & DSP_GFLAG_USER_MU) != 0;
        c.alb = scalar(b->surface_albedo, i, 0.0);
        c.dtau = b->delta_tau + l0;
        c.ssa = b->single_scat_albedo + l0;
        c.pmom = b->phase_function_moments + l0 * b->pmom_count;
        c.numu = b->num_user_mu;
        c.umu = at(b->mu_user, i);
        const int half = c.user_mu ? c.numu : c.N / 2;
        if (c.L > 0 && b->layer_offset[i + 1] - l0 != c.L) st = DSP_ERR_INVALID_INPUT;
        else if (half > o->numu_out || c.N > 64) st = DSP_ERR_INVALID_INPUT;
        else {
          oracle::GeneralOutput go;
          std::vector<double> f8((size_t)8 * (c.L + 1));
          for (int f = 0; f < 8; ++f) go.flux[f] = f8.data() + (size_t)f * (c.L + 1);
          go.intensity = go.iavg = nullptr;
          go.ntau_out = c.L + 1;
          go.numu_out = 2 * half;
          go.albtrans[0] = o->albedo_medium + (size_t)o->numu_out * i;
          go.albtrans[1] = o->transmissivity_medium + (size_t)o->numu_out * i;
          go.albtrans[2] = o->spherical_albedo + i;
          go.albtrans[3] = o->spherical_transmissivity + i;
          st = solver.solve(c, go);
        }
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

double oracle_planck_deriv(double wnumlo, double wnumhi, double temp) {
  return oracle::planck_function_deriv2(wnumlo, wnumhi, temp);
}

}  // extern "C"
