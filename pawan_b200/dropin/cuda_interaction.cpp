/* Drop-in GPU interaction for pawan; see cuda_interaction.h. */
#include "cuda_interaction.h"

#include <algorithm>
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

size_t __cuda::numParticles() const {
  size_t n = 0;
  for (auto *w : _wakes) n += w->_numParticles;
  return n;
}

void __cuda::gatherPositions(double *out) const {
  for (auto *w : _wakes) {
    gather_rows(w->_position, out);
    out += 3 * w->_numParticles;
  }
}

void __cuda::gatherVorticity(double *out) const {
  for (auto *w : _wakes) {
    gather_rows(w->_vorticity, out);
    out += 3 * w->_numParticles;
  }
}

void __cuda::scatterField(const double *field) {
  for (auto *w : _wakes) {
    scatter_rows(field, w->_vorticityfield);
    field += 3 * w->_numParticles;
  }
}

void __cuda::influenceColumns(size_t ncols, const double *alpha, double *field) {
  ensure_system();
  check(pawan_system_influence_columns(_sys, ncols, alpha, field, ncols * 3 * numParticles()),
        "influence_columns");
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

namespace {
// Host memory bound of one batch of resolve columns (strengths + fields).
constexpr size_t kResolveBatchBytes = size_t(512) << 20;

struct ResolveBuffers {
  gsl_vector *states = nullptr, *vrxfield = nullptr, *result = nullptr;
  gsl_matrix *influence = nullptr;
  gsl_permutation *p = nullptr;
  FILE *f = nullptr;
  ~ResolveBuffers() {
    if (f) std::fclose(f);
    if (p) gsl_permutation_free(p);
    if (influence) gsl_matrix_free(influence);
    if (result) gsl_vector_free(result);
    if (vrxfield) gsl_vector_free(vrxfield);
    if (states) gsl_vector_free(states);
  }
};
}  // namespace

void __cuda_resolve::rebuild(__interaction *IN, __io *IO) {
  __cuda *C = dynamic_cast<__cuda *>(IN);
  if (!C) {
    __resolve::rebuild(IN, IO);
    return;
  }
  const size_t S = IN->_size;
  const size_t per = 3 * C->numParticles();
  ResolveBuffers b;
  b.states = gsl_vector_calloc(S);
  b.influence = gsl_matrix_calloc(S, S);
  b.f = IO->create_binary_file(".wakeinfluence");
  if (!b.f) throw std::runtime_error("pawan_b200: cannot create the .wakeinfluence file");
  double t = 0.0;
  std::fwrite(&t, sizeof(double), 1, b.f);
  IN->write(b.f);
  IN->getStates(b.states);
  std::vector<double> orig(S);
  for (size_t i = 0; i < S; ++i) orig[i] = gsl_vector_get(b.states, i);
  const double tStart = TIME();
  OUT("Calculating influence matrix of all particles.");
  const size_t batch = std::max<size_t>(1, kResolveBatchBytes / (2 * per * sizeof(double)));
  std::vector<double> base(per), pos(per), alpha, field;
  size_t i = 0;
  while (i < S) {
    // Columns [first, i): each sets its state entry to 1 (the reference's
    // loop, resolve.cpp:19-31), while the positions stay those of `first`.
    const size_t first = i;
    alpha.clear();
    while (i < S && i - first < batch) {
      gsl_vector_set(b.states, i, 1.0);
      IN->setStates(b.states);
      C->gatherPositions(pos.data());
      if (i == first) {
        base = pos;
      } else if (std::memcmp(pos.data(), base.data(), per * sizeof(double)) != 0) {
        gsl_vector_set(b.states, i, orig[i]);  // column i starts the next batch
        break;
      }
      alpha.resize((i - first + 1) * per);
      C->gatherVorticity(alpha.data() + (i - first) * per);
      OUT("\ti", i);
      gsl_vector_set(b.states, i, 0.0);
      t += 1.0;
      std::fwrite(&t, sizeof(double), 1, b.f);
      IN->write(b.f);  // x, alpha, s: what the reference writes after the column's resolve
      ++i;
    }
    const size_t nc = i - first;
    // Replay the columns' states: the positions of the batch go to the device
    // with the first, and each column's field is read through getRates with the
    // state vector exactly as the reference has it at that column.
    for (size_t j = first; j < i; ++j) gsl_vector_set(b.states, j, orig[j]);
    gsl_vector_set(b.states, first, 1.0);
    IN->setStates(b.states);
    C->upload();
    field.resize(nc * per);
    C->influenceColumns(nc, alpha.data(), field.data());
    for (size_t j = first; j < i; ++j) {
      if (j > first) {
        gsl_vector_set(b.states, j, 1.0);
        IN->setStates(b.states);
      }
      C->scatterField(field.data() + (j - first) * per);
      gsl_vector_view column = gsl_matrix_column(b.influence, j);
      IN->getRates(&column.vector);
      gsl_vector_set(b.states, j, 0.0);
    }
  }
  std::fclose(b.f);
  b.f = nullptr;
  OUT("Calculating expected vorticity field.");
  b.vrxfield = gsl_vector_calloc(S);
  IN->getIdealRates(b.vrxfield);
  OUT("Solving vorticity strengths.");
  b.result = gsl_vector_calloc(S);
  int s = 0;
  b.p = gsl_permutation_alloc(S);
  gsl_linalg_LU_decomp(b.influence, b.p, &s);
  gsl_linalg_LU_solve(b.influence, b.p, b.vrxfield, b.result);
  const double tEnd = TIME();
  OUT("Total Time (s)", tEnd - tStart);
  OUT("Applying new vorticity strengths.");
  IN->setStates(b.result);
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
