/* Drop-in GPU interaction for pawan; see cuda_interaction.h. */
#include "cuda_interaction.h"

#include <cstring>

namespace pawan {

__cuda::__cuda(__wake *W, double nu, int precision, int device)
    : __interaction(), _precision(precision), _device(device) {
  _nu = nu;
  addWake(W);
}

__cuda::__cuda(__wake *W1, __wake *W2, double nu, int precision, int device)
    : __interaction(), _precision(precision), _device(device) {
  _nu = nu;
  addWake(W1);
  addWake(W2);
}

__cuda::~__cuda() {
  if (_sys) pawan_system_destroy(_sys);
  if (_ctx) pawan_ctx_destroy(_ctx);
}

void __cuda::check(int status, const char *what) const {
  if (status == PAWAN_OK) return;
  std::string msg = std::string("pawan_b200: ") + what + ": " + pawan_status_name(status);
  if (_ctx) msg += std::string(" (") + pawan_ctx_last_error(_ctx) + ")";
  throw std::runtime_error(msg);
}

void __cuda::addWake(__wake *W) {
  __interaction::addWake(W);
  _wakes.push_back(W);
  if (_sys) {  // the wake set changed: rebuild the device system on next use
    pawan_system_destroy(_sys);
    _sys = nullptr;
  }
  _particles_uploaded = false;
}

void __cuda::setViscosity(double nu) {
  _nu = nu;
  if (_sys) check(pawan_system_set_nu(_sys, nu), "set_nu");
}

void __cuda::setKernel(int kernel) {
  _kernel = kernel;
  if (_sys) check(pawan_system_set_kernel(_sys, kernel), "set_kernel");
}

void __cuda::ensure_system() {
  if (!_ctx) check(pawan_ctx_create(_device, &_ctx), "context");
  if (_sys) return;
  std::vector<size_t> counts;
  for (auto *w : _wakes) counts.push_back(w->_numParticles);
  check(pawan_system_create(_ctx, counts.size(), counts.data(), _nu, _precision, &_sys),
        "system_create");
  check(pawan_system_set_kernel(_sys, _kernel), "set_kernel");
}

// The wakes' matrices are row-major N x 3 (wake.cpp:10-21); copy rows so a
// non-unit tda would still be honoured.
static void gather_rows(const gsl_matrix *m, double *out) {
  for (size_t i = 0; i < m->size1; ++i) std::memcpy(out + 3 * i, m->data + i * m->tda, 3 * sizeof(double));
}

static void scatter_rows(const double *in, gsl_matrix *m) {
  for (size_t i = 0; i < m->size1; ++i) std::memcpy(m->data + i * m->tda, in + 3 * i, 3 * sizeof(double));
}

void __cuda::upload() {
  ensure_system();
  size_t n = 0;
  for (auto *w : _wakes) n += w->_numParticles;
  if (!_particles_uploaded) {
    std::vector<double> pos(3 * n), vor(3 * n), rad(n), vol(n);
    size_t o = 0;
    for (auto *w : _wakes) {
      gather_rows(w->_position, pos.data() + 3 * o);
      gather_rows(w->_vorticity, vor.data() + 3 * o);
      for (size_t i = 0; i < w->_numParticles; ++i) {
        rad[o + i] = gsl_vector_get(w->_radius, i);
        vol[o + i] = gsl_vector_get(w->_volume, i);
      }
      o += w->_numParticles;
    }
    check(pawan_system_set_particles(_sys, pos.data(), vor.data(), rad.data(), vol.data()),
          "set_particles");
    _particles_uploaded = true;
    return;
  }
  // state layout per wake [x | alpha] (wake.cpp:110-120)
  std::vector<double> state(6 * n);
  size_t o = 0;
  for (auto *w : _wakes) {
    const size_t c = w->_numParticles;
    gather_rows(w->_position, state.data() + 6 * o);
    gather_rows(w->_vorticity, state.data() + 6 * o + 3 * c);
    o += c;
  }
  check(pawan_system_set_states(_sys, state.data(), state.size()), "set_states");
}

void __cuda::download() {
  size_t n = 0;
  for (auto *w : _wakes) n += w->_numParticles;
  std::vector<double> state(6 * n);
  check(pawan_system_get_states(_sys, state.data(), state.size()), "get_states");
  size_t o = 0;
  for (auto *w : _wakes) {
    const size_t c = w->_numParticles;
    scatter_rows(state.data() + 6 * o, w->_position);
    scatter_rows(state.data() + 6 * o + 3 * c, w->_vorticity);
    o += c;
  }
}

void __cuda::interact() {
  upload();
  check(pawan_system_solve(_sys), "solve");
  for (size_t k = 0; k < _wakes.size(); ++k) {
    __wake *w = _wakes[k];
    const size_t c = w->_numParticles;
    std::vector<double> u(3 * c), da(3 * c);
    check(pawan_system_get_wake_rates(_sys, k, u.data(), da.data()), "get_wake_rates");
    scatter_rows(u.data(), w->_velocity);
    scatter_rows(da.data(), w->_retvorcity);
  }
}

void __cuda::influence() {
  upload();
  size_t n = 0;
  for (auto *w : _wakes) n += w->_numParticles;
  std::vector<double> k(3 * n);
  check(pawan_system_influence(_sys, k.data(), k.size()), "influence");
  size_t o = 0;
  for (auto *w : _wakes) {
    scatter_rows(k.data() + 3 * o, w->_vorticityfield);
    o += w->_numParticles;
  }
}

void __cuda::diagnose() {
  upload();
  double out[11];
  check(pawan_system_diagnose(_sys, out, 1), "diagnose");
  for (int d = 0; d < 3; ++d) {
    gsl_vector_set(_totalVorticity, d, out[d]);
    gsl_vector_set(_linearImpulse, d, out[3 + d]);
    gsl_vector_set(_angularImpulse, d, out[6 + d]);
  }
  _enstrophy = out[9];
  _helicity = out[10];
  OUTT("Total Vorticity", _totalVorticity);
  OUTT("Linear Impulse", _linearImpulse);
  OUTT("Angular Impulse", _angularImpulse);
  OUT("Helicity", _helicity);
  OUT("Enstrophy", _enstrophy);
}

double __cuda::kineticEnergy() {
  upload();
  double ke = 0.0;
  check(pawan_system_kinetic_energy(_sys, &ke), "kinetic_energy");
  _kineticEnergy = ke;
  return ke;
}

void __cuda_rk4::integrate(__system *S, __io *IO) {
  __cuda *C = dynamic_cast<__cuda *>(S);
  if (!C) {
    __rk4::integrate(S, IO);
    return;
  }
  C->upload();
  FILE *f = IO->create_binary_file(".wake");
  if (!f) throw std::runtime_error("pawan_b200: cannot create the .wake file (does its directory exist?)");
  const int st = pawan_system_integrate_file(C->device_system(), _t, _n, f, PAWAN_INTEGRATE_RK4);
  std::fclose(f);
  if (st != PAWAN_OK) throw std::runtime_error("pawan_b200: integrate failed");
  C->download();
}

void __cuda_rk4::step(const double &dt, __system *S, gsl_vector *state) {
  __cuda *C = dynamic_cast<__cuda *>(S);
  if (!C) {
    __rk4::step(dt, S, state);
    return;
  }
  if (state->stride != 1) throw std::runtime_error("pawan_b200: state vector must be contiguous");
  // state -> wakes -> device; one device-resident RK4 step; device -> state, wakes
  S->setStates(state);
  C->upload();
  pawan_system *sys = C->device_system();
  if (pawan_system_rk4(sys, dt, 1) != PAWAN_OK) throw std::runtime_error("pawan_b200: rk4 step failed");
  if (pawan_system_get_states(sys, state->data, state->size) != PAWAN_OK)
    throw std::runtime_error("pawan_b200: get_states failed");
  S->setStates(state);
}

}  // namespace pawan
