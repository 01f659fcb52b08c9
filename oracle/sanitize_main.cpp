// Test infrastructure: drives the oracle's host code -- the reference's own
// sources on the GSL shim (through ref_harness.cpp) and the C restatement --
// built with AddressSanitizer and UndefinedBehaviorSanitizer by
// `make -C oracle sanitize`.  Any out-of-bounds access, use after free or
// undefined behaviour on these paths aborts with a report (exit status != 0).
// Memory the reference leaks by design (a gsl_vector per ENSTROPHY pair,
// src/interaction/interaction_utils.h:132) is not reported: the test runs with
// detect_leaks=0.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "restate.h"

extern "C" {
void *refh_create(int n_wakes, const size_t *counts, const double *pos, const double *vor,
                  const double *rad, const double *vol, double nu, int use_parallel);
void refh_destroy(void *p);
size_t refh_size(void *p);
void refh_solve(void *p);
void refh_get_rates(void *p, double *rate);
void refh_get_states(void *p, double *state);
void refh_rk4_step(void *p, double dt, size_t nsteps, double *state);
void refh_euler_step(void *p, double dt, size_t nsteps, double *state);
int refh_diagnose(void *p, double *out);
double refh_kinetic_energy(void *p);
void refh_influence(void *p, double *field);
void *refh_vring_create(double radius, double core, int layers, double nu);
void refh_resolve(void *p, double *state);
}

int main() {
  // two jittered rings of 24 particles each
  const size_t nw = 2, c = 24, n = nw * c;
  std::vector<double> pos(3 * n), vor(3 * n), rad(n, 0.12), vol(n, 1e-3);
  for (size_t w = 0; w < nw; ++w)
    for (size_t i = 0; i < c; ++i) {
      const double a = 2.0 * M_PI * i / c, j = 1e-3 * std::sin(7.0 * i + w);
      double *x = &pos[3 * (w * c + i)], *v = &vor[3 * (w * c + i)];
      x[0] = std::cos(a) + j;
      x[1] = std::sin(a) - j;
      x[2] = 0.5 * w + j;
      v[0] = -std::sin(a) * 0.1;
      v[1] = std::cos(a) * 0.1;
      v[2] = 0.0;
    }
  const size_t counts[2] = {c, c};
  double out[11], worst = 0.0;
  for (int par = 0; par < 2; ++par) {
    void *h = refh_create((int)nw, counts, pos.data(), vor.data(), rad.data(), vol.data(), 1e-3, par);
    const size_t sz = refh_size(h);
    std::vector<double> rates(sz), state(sz), field(3 * n);
    refh_solve(h);
    refh_get_rates(h, rates.data());
    refh_get_states(h, state.data());
    refh_rk4_step(h, 0.005, 1, state.data());
    refh_euler_step(h, 0.005, 1, state.data());
    if (!par) {
      refh_diagnose(h, out);
      refh_kinetic_energy(h);
    }
    refh_influence(h, field.data());
    refh_destroy(h);
    // the restatement on the same inputs
    std::vector<double> u(3 * n), da(3 * n);
    for (int k = 0; k < 2; ++k) {
      orc_set_kernel(k);
      orc_pairs(n, pos.data(), vor.data(), rad.data(), vol.data(), 1e-3, n, nullptr, u.data(), da.data());
      orc_influence(n, pos.data(), vor.data(), rad.data(), field.data());
      orc_enstrophy(n, pos.data(), vor.data(), rad.data());
      orc_helicity(n, pos.data(), vor.data(), rad.data());
    }
    orc_set_kernel(0);
    orc_pairs(n, pos.data(), vor.data(), rad.data(), vol.data(), 1e-3, n, nullptr, u.data(), da.data());
    for (size_t i = 0; i < 3 * n; ++i) worst = std::fmax(worst, std::fabs(u[i] - rates[i % 3 + 6 * (i / (3 * c)) * c + 3 * ((i / 3) % c)]));
  }
  void *v = refh_vring_create(1.0, 0.1, 1, 0.0);
  std::vector<double> s(refh_size(v));
  refh_resolve(v, s.data());
  refh_destroy(v);
  std::printf("sanitized oracle run ok (%g)\n", worst);
  return 0;
}
