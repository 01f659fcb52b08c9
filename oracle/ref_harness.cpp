// Test infrastructure (oracle).  A C-ABI harness around the reference's OWN,
// unmodified C++ classes, compiled from their sources by oracle/Makefile
// against the project's GSL-API shim (oracle/gslshim).  Nothing in the product
// links this; only tests, the smoke check and bench.py's CPU-baseline leg do.
//
// What it exposes, and the reference code each entry drives:
//   refh_create            builds __wake objects from arrays and an __interaction
//                          (serial, src/interaction/interaction.cpp:11-39) or
//                          __parallel (OpenMP, src/interaction/parallel.cpp:10-11)
//                          holding them, with the viscosity set through the
//                          protected member _nu (interaction.h:24)
//   refh_solve             __interaction::solve (interaction.cpp:41-43, 95-108)
//   refh_get/set_states,   __interaction::getStates/setStates/getRates
//   refh_get_rates         (interaction.cpp:204-229, wake.cpp:87-120)
//   refh_rk4_step          __rk4::step (src/integration/rk4.cpp:12-76)
//   refh_euler_step        __integration::step (src/integration/integration.cpp:37-45)
//   refh_integrate         __integration::integrate (integration.cpp:16-35), which
//                          writes data/temp.wake under the current directory
//   refh_diagnose          __interaction::diagnose (interaction.cpp:49-93)
//   refh_kinetic_energy    calculateKineticEnergy (interaction.cpp:351-383)
//   refh_write_frame       one .wake frame: t, then __interaction::write
//                          (interaction.cpp:197-202, wake.cpp:68-73)
//   refh_vring_create      a __vring(R, core, layers) (src/wake/vring.cpp:51-104)
//                          in a serial __interaction
//   refh_influence         __interaction::resolve -> influence (interaction.cpp:45-47,
//                          110-155): every wake's _vorticityfield
//   refh_resolve           __resolve::rebuild (src/resolve/resolve.cpp:10-57), which
//                          writes data/temp.wakeinfluence under the current directory
#include <omp.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "src/integration/integration.h"
#include "src/integration/rk4.h"
#include "src/interaction/interaction.h"
#include "src/interaction/parallel.h"
#include "src/io/io.h"
#include "src/resolve/resolve.h"
#include "src/wake/vring.h"
#include "src/wake/wake.h"

namespace {

// A __wake filled from plain arrays.  The base constructor allocates a
// one-particle wake (wake.cpp:23-35); it is released and re-created with n.
class ArrayWake : public pawan::__wake {
 public:
  ArrayWake(size_t n, const double *pos, const double *vor, const double *rad, const double *vol) {
    gsl_matrix_free(_position);
    gsl_matrix_free(_velocity);
    gsl_matrix_free(_vorticity);
    gsl_matrix_free(_retvorcity);
    gsl_vector_free(_radius);
    gsl_vector_free(_volume);
    gsl_vector_free(_birthstrength);
    gsl_matrix_free(_vorticityfield);
    create_particles((int)n);
    for (size_t i = 0; i < n; ++i) {
      for (size_t d = 0; d < 3; ++d) {
        gsl_matrix_set(_position, i, d, pos[3 * i + d]);
        gsl_matrix_set(_vorticity, i, d, vor[3 * i + d]);
      }
      gsl_vector_set(_radius, i, rad[i]);
      gsl_vector_set(_volume, i, vol[i]);
      gsl_vector_set(_birthstrength, i, 0.0);
    }
  }
};

class SerialSystem : public pawan::__interaction {
 public:
  explicit SerialSystem(double nu) : pawan::__interaction() { _nu = nu; }
  double kinetic_energy(const std::vector<pawan::__wake *> &W) {
    double ke = 0.0;
    for (size_t i = 0; i < W.size(); ++i) {
      ke += calculateKineticEnergy(W[i]);
      for (size_t j = i + 1; j < W.size(); ++j) ke += calculateKineticEnergy(W[i], W[j]);
    }
    return ke;
  }
  void read_diagnostics(double *out) const {
    for (int d = 0; d < 3; ++d) {
      out[d] = gsl_vector_get(_totalVorticity, d);
      out[3 + d] = gsl_vector_get(_linearImpulse, d);
      out[6 + d] = gsl_vector_get(_angularImpulse, d);
    }
    out[9] = _enstrophy;
    out[10] = _helicity;
  }
};

class ParallelSystem : public pawan::__parallel {
 public:
  ParallelSystem(pawan::__wake *W, double nu) : pawan::__parallel(W) { _nu = nu; }
};

class StepRK4 : public pawan::__rk4 {
 public:
  StepRK4() : pawan::__rk4(1.0, 1) {}
  void run(double dt, pawan::__system *S, gsl_vector *state) { step(dt, S, state); }
};

class StepEuler : public pawan::__integration {
 public:
  StepEuler() : pawan::__integration(1.0, 1) {}
  void run(double dt, pawan::__system *S, gsl_vector *state) { step(dt, S, state); }
};

struct Handle {
  std::vector<pawan::__wake *> wakes;
  SerialSystem *serial = nullptr;
  ParallelSystem *parallel = nullptr;
  pawan::__interaction *sys() {
    return serial ? static_cast<pawan::__interaction *>(serial)
                  : static_cast<pawan::__interaction *>(parallel);
  }
};

}  // namespace

extern "C" {

void *refh_create(int n_wakes, const size_t *counts, const double *pos, const double *vor,
                  const double *rad, const double *vol, double nu, int use_parallel) {
  Handle *h = new Handle();
  size_t off = 0;
  for (int w = 0; w < n_wakes; ++w) {
    h->wakes.push_back(new ArrayWake(counts[w], pos + 3 * off, vor + 3 * off, rad + off, vol + off));
    off += counts[w];
  }
  if (use_parallel) {
    h->parallel = new ParallelSystem(h->wakes[0], nu);
    for (int w = 1; w < n_wakes; ++w) h->parallel->addWake(h->wakes[w]);
  } else {
    h->serial = new SerialSystem(nu);
    for (int w = 0; w < n_wakes; ++w) h->serial->addWake(h->wakes[w]);
  }
  return h;
}

void refh_destroy(void *p) {
  Handle *h = static_cast<Handle *>(p);
  delete h->serial;
  delete h->parallel;
  for (auto *w : h->wakes) delete w;
  delete h;
}

size_t refh_size(void *p) { return static_cast<Handle *>(p)->sys()->_size; }

void refh_set_states(void *p, const double *state) {
  Handle *h = static_cast<Handle *>(p);
  gsl_vector_const_view v = gsl_vector_const_view_array(state, h->sys()->_size);
  h->sys()->setStates(&v.vector);
}

void refh_get_states(void *p, double *state) {
  Handle *h = static_cast<Handle *>(p);
  gsl_vector_view v = gsl_vector_view_array(state, h->sys()->_size);
  h->sys()->getStates(&v.vector);
}

void refh_solve(void *p) { static_cast<Handle *>(p)->sys()->solve(); }

void refh_get_rates(void *p, double *rate) {
  Handle *h = static_cast<Handle *>(p);
  gsl_vector_view v = gsl_vector_view_array(rate, h->sys()->_size);
  h->sys()->getRates(&v.vector);
}

// Copies W->_velocity and W->_retvorcity (N x 3 each) of wake w.
void refh_get_wake_rates(void *p, int w, double *vel, double *retvor) {
  pawan::__wake *W = static_cast<Handle *>(p)->wakes[w];
  for (size_t i = 0; i < W->_numParticles; ++i)
    for (size_t d = 0; d < 3; ++d) {
      vel[3 * i + d] = gsl_matrix_get(W->_velocity, i, d);
      retvor[3 * i + d] = gsl_matrix_get(W->_retvorcity, i, d);
    }
}

// Runs nsteps of __rk4::step on `state` (length _size, reference layout).
void refh_rk4_step(void *p, double dt, size_t nsteps, double *state) {
  Handle *h = static_cast<Handle *>(p);
  gsl_vector_view v = gsl_vector_view_array(state, h->sys()->_size);
  StepRK4 rk;
  for (size_t i = 0; i < nsteps; ++i) rk.run(dt, h->sys(), &v.vector);
}

void refh_euler_step(void *p, double dt, size_t nsteps, double *state) {
  Handle *h = static_cast<Handle *>(p);
  gsl_vector_view v = gsl_vector_view_array(state, h->sys()->_size);
  StepEuler eu;
  for (size_t i = 0; i < nsteps; ++i) eu.run(dt, h->sys(), &v.vector);
}

// __rk4(T, n).integrate(S, IO): writes data/temp.wake relative to the cwd.
void refh_integrate(void *p, double T, size_t n) {
  Handle *h = static_cast<Handle *>(p);
  pawan::__io io;
  pawan::__rk4 rk(T, n);
  rk.integrate(h->sys(), &io);
}

// out: totalVorticity[3], linearImpulse[3], angularImpulse[3], enstrophy, helicity.
// Serial systems only: the OpenMP overrides of total vorticity and angular
// impulse read uninitialised accumulators (parallel.cpp:161,175).
int refh_diagnose(void *p, double *out) {
  Handle *h = static_cast<Handle *>(p);
  if (!h->serial) return 1;
  h->serial->diagnose();
  h->serial->read_diagnostics(out);
  return 0;
}

double refh_kinetic_energy(void *p) {
  Handle *h = static_cast<Handle *>(p);
  if (!h->serial) return 0.0;
  return h->serial->kinetic_energy(h->wakes);
}

int refh_write_frame(void *p, const char *path, double t, int append) {
  Handle *h = static_cast<Handle *>(p);
  FILE *f = std::fopen(path, append ? "ab" : "wb");
  if (!f) return 1;
  std::fwrite(&t, sizeof(double), 1, f);
  h->sys()->write(f);
  std::fclose(f);
  return 0;
}

void *refh_vring_create(double radius, double core, int layers, double nu) {
  Handle *h = new Handle();
  h->wakes.push_back(new pawan::__vring(radius, core, layers));
  h->serial = new SerialSystem(nu);
  h->serial->addWake(h->wakes[0]);
  return h;
}

size_t refh_num_particles(void *p) {
  size_t n = 0;
  for (auto *w : static_cast<Handle *>(p)->wakes) n += w->_numParticles;
  return n;
}

// Union (wake order) of positions, vorticities (N x 3), radii and volumes.
void refh_get_particles(void *p, double *pos, double *vor, double *rad, double *vol) {
  size_t o = 0;
  for (auto *W : static_cast<Handle *>(p)->wakes) {
    for (size_t i = 0; i < W->_numParticles; ++i) {
      for (size_t d = 0; d < 3; ++d) {
        pos[3 * (o + i) + d] = gsl_matrix_get(W->_position, i, d);
        vor[3 * (o + i) + d] = gsl_matrix_get(W->_vorticity, i, d);
      }
      rad[o + i] = gsl_vector_get(W->_radius, i);
      vol[o + i] = gsl_vector_get(W->_volume, i);
    }
    o += W->_numParticles;
  }
}

// __interaction::resolve() (the vorticity field), then every wake's
// _vorticityfield in wake order (N x 3).
void refh_influence(void *p, double *field) {
  Handle *h = static_cast<Handle *>(p);
  h->sys()->resolve();
  size_t o = 0;
  for (auto *W : h->wakes) {
    for (size_t i = 0; i < W->_numParticles; ++i)
      for (size_t d = 0; d < 3; ++d) field[3 * (o + i) + d] = gsl_matrix_get(W->_vorticityfield, i, d);
    o += W->_numParticles;
  }
}

// __resolve::rebuild(IN, IO), then the system's state (length _size).
void refh_resolve(void *p, double *state) {
  Handle *h = static_cast<Handle *>(p);
  pawan::__io io;
  pawan::__resolve rs;
  rs.rebuild(h->sys(), &io);
  gsl_vector_view v = gsl_vector_view_array(state, h->sys()->_size);
  h->sys()->getStates(&v.vector);
}

void refh_set_threads(int n) { omp_set_num_threads(n); }
int refh_max_threads(void) { return omp_get_max_threads(); }
double refh_wtime(void) { return omp_get_wtime(); }

}  // extern "C"
