/* Test infrastructure (oracle): FP64 restatement of pawan's pair physics,
 * RK4 step and diagnostics.  See restate.h.  Every formula below cites the
 * reference line it restates (paths relative to the pawan source tree).
 *
 * Gather form.  The reference visits each unordered pair once
 * (src/interaction/interaction.cpp:157-195), with d = x_target - x_source,
 * adds the pair's velocity and vorticity rate to the target and the mirrored
 * terms to the source (src/interaction/interaction_utils.h:363-407).
 * Writing both roles from the point of view of particle i, with j any other
 * particle and d = x_i - x_j, gives exactly the sum computed here.
 */
#include "restate.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Smoothing kernel: 0 = high-order algebraic (highorder.h, the reference's
 * default), 1 = Gaussian (gaussian.h).  Set by orc_set_kernel. */
static int g_kernel = 0;

void orc_set_kernel(int kernel) { g_kernel = kernel; }

/* gaussian.h:20-23 (ZETASIG). */
static double zeta_gauss(double rho, double sigma) {
  const double rho_bar = rho / sigma;
  return exp(-0.5 * rho_bar * rho_bar) / pow(sigma, 3.0) / pow(2.0 * M_PI, 1.5);
}

/* gaussian.h:46-59 (KERNEL): q, F and Z of one pair. */
static void kernel_qfz_gauss(double rho, double sigma, double *q, double *F, double *Z) {
  const double rho_bar = rho / sigma;
  const double sig3 = sigma * sigma * sigma;
  const double z = zeta_gauss(rho, sigma);
  const double phi = 0.25 * M_1_PI * erf(M_SQRT1_2 * rho_bar) / sig3;
  *Z = z;
  *q = (phi / rho_bar - z) / (rho_bar * rho_bar);
  *F = (z - 3.0 * (*q)) / (rho * rho);
}

/* highorder.h:20-23 (ZETASIG), or the Gaussian one. */
static double zeta(double rho, double sigma) {
  if (g_kernel == 1) return zeta_gauss(rho, sigma);
  const double rho_bar = rho / sigma;
  return 1.875 * M_1_PI / pow(rho_bar * rho_bar + 1.0, 7.5) / pow(sigma, 3);
}

/* highorder.h:48-60 (KERNEL) and :20-23 (ZETASIG): q, F and Z of one pair. */
static void kernel_qfz(double rho, double sigma, double *q, double *F, double *Z) {
  if (g_kernel == 1) {
    kernel_qfz_gauss(rho, sigma, q, F, Z);
    return;
  }
  const double rho_bar = rho / sigma;
  const double z = 1.875 * M_1_PI / pow(rho_bar * rho_bar + 1.0, 7.5) / pow(sigma, 3);
  const double rho_bar2 = rho_bar * rho_bar;
  const double sig3 = sigma * sigma * sigma;
  const double phi = 0.25 * M_1_PI * (rho_bar2 + 1.5) / pow(rho_bar2 + 1.0, 2.0) / sig3;
  *Z = z;
  *q = (phi / rho_bar - z) / rho_bar2;
  *F = (z - 3.0 * (*q)) / (rho * rho);
}

/* highorder.h:30-38 (QSIG): q alone, used by helicity. */
static double kernel_q(double rho, double sigma) {
  double q, F, Z;
  kernel_qfz(rho, sigma, &q, &F, &Z);
  return q;
}

static void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

static double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* One target i against all sources j != i.
 *   sigma = sqrt(0.5 (s_i^2 + s_j^2))                    interaction_utils.h:452
 *   u_i  += q (alpha_j x d)                               :458-459 (VELOCITY :52-58)
 *   da_i += q (alpha_i x alpha_j) + F [d.(alpha_i x alpha_j)] d     :466 (VORSTRETCH :69-100)
 *   da_i += (Z nu / (sigma^2/2)) (v_i alpha_j - v_j alpha_i)       :467 (DIFFUSION :253-286)
 * The source-role terms (:460-462 and :470-475, with d -> -d) reduce to the same
 * expressions. */
static void target_sum(size_t n, size_t i, const double *pos, const double *vor,
                       const double *rad, const double *vol, double nu, double *u,
                       double *da) {
  const double *xi = pos + 3 * i, *ai = vor + 3 * i;
  const double si = rad[i], vi = vol[i];
  double acc_u[3] = {0, 0, 0}, acc_a[3] = {0, 0, 0};
  for (size_t j = 0; j < n; ++j) {
    if (j == i) continue;
    const double *xj = pos + 3 * j, *aj = vor + 3 * j;
    const double sj = rad[j], vj = vol[j];
    double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
    const double rho = sqrt(dot3(d, d));
    const double sigma = sqrt(0.5 * (sj * sj + si * si));
    double q, F, Z;
    kernel_qfz(rho, sigma, &q, &F, &Z);
    double c[3];
    cross3(aj, d, c);
    for (int k = 0; k < 3; ++k) acc_u[k] += q * c[k];
    double ixj[3];
    cross3(ai, aj, ixj);
    const double roaxa = dot3(d, ixj);
    const double diff = Z * nu / (0.5 * sigma * sigma);
    for (int k = 0; k < 3; ++k)
      acc_a[k] += q * ixj[k] + F * roaxa * d[k] + diff * (vi * aj[k] - vj * ai[k]);
  }
  for (int k = 0; k < 3; ++k) {
    u[k] = acc_u[k];
    da[k] = acc_a[k];
  }
}

void orc_pairs(size_t n, const double *pos, const double *vor, const double *rad,
               const double *vol, double nu, size_t nt, const int64_t *targets,
               double *vel, double *dvor) {
  if (!targets) nt = n;
#pragma omp parallel for schedule(dynamic, 16)
  for (long t = 0; t < (long)nt; ++t) {
    const size_t i = targets ? (size_t)targets[t] : (size_t)t;
    target_sum(n, i, pos, vor, rad, vol, nu, vel + 3 * t, dvor + 3 * t);
  }
}

/* src/integration/rk4.cpp:12-76, in the same operation order:
 *   x1 = k1*(dt/2) + x;  x2 = k2*(dt/2) + x;  x3 = k3*dt + x;
 *   x += ((k1 + k4)*(dt/6) + (k2 + k3)*(dt/3)). */
void orc_rk4_step(size_t n, double *pos, double *vor, const double *rad, const double *vol,
                  double nu, double dt) {
  const size_t m = 3 * n;
  double *x = (double *)malloc(sizeof(double) * 2 * m);
  double *xs = (double *)malloc(sizeof(double) * 2 * m);
  double *k[4];
  for (int s = 0; s < 4; ++s) k[s] = (double *)malloc(sizeof(double) * 2 * m);
  memcpy(x, pos, sizeof(double) * m);
  memcpy(x + m, vor, sizeof(double) * m);
  memcpy(xs, x, sizeof(double) * 2 * m);
  const double c[3] = {0.5 * dt, 0.5 * dt, dt};
  for (int s = 0; s < 4; ++s) {
    orc_pairs(n, xs, xs + m, rad, vol, nu, n, NULL, k[s], k[s] + m);
    if (s < 3)
      for (size_t e = 0; e < 2 * m; ++e) xs[e] = k[s][e] * c[s] + x[e];
  }
  const double d6 = dt / 6., d3 = dt / 3.;
  for (size_t e = 0; e < 2 * m; ++e) {
    const double a = (k[0][e] + k[3][e]) * d6;
    const double b = (k[1][e] + k[2][e]) * d3;
    x[e] = x[e] + (a + b);
  }
  memcpy(pos, x, sizeof(double) * m);
  memcpy(vor, x + m, sizeof(double) * m);
  for (int s = 0; s < 4; ++s) free(k[s]);
  free(x);
  free(xs);
}

/* interaction.cpp:240-246 (sum alpha), :248-259 (1/2 sum x x alpha),
 * :261-275 (1/3 sum x x (x x alpha)). */
void orc_linear_diagnostics(size_t n, const double *pos, const double *vor, double *out) {
  double O[3] = {0, 0, 0}, I[3] = {0, 0, 0}, A[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    const double *r = pos + 3 * i, *a = vor + 3 * i;
    double rxa[3], rxrxa[3];
    cross3(r, a, rxa);
    cross3(r, rxa, rxrxa);
    for (int k = 0; k < 3; ++k) {
      O[k] += a[k];
      I[k] += rxa[k];
      A[k] += rxrxa[k];
    }
  }
  for (int k = 0; k < 3; ++k) {
    out[k] = O[k];
    out[3 + k] = I[k] * 0.5;
    out[6 + k] = A[k] * (1.0 / 3.0);
  }
}

/* Enstrophy: interaction.cpp:277-315 with ENSTROPHY (interaction_utils.h:107-156)
 * and ENST (highorder.h:69-86).  Pairs inside a wake are counted twice over
 * i<j, pairs across wakes twice over all (i,j); both equal one count per
 * ordered pair, which is how the sum is written here. */
double orc_enstrophy(size_t n, const double *pos, const double *vor, const double *rad) {
  if (g_kernel == 1) return 0.0; /* gaussian.h:67-86: ENST is a stub returning 0 */
  double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 16)
  for (long il = 0; il < (long)n; ++il) {
    const size_t i = (size_t)il;
    const double *xi = pos + 3 * i, *ai = vor + 3 * i;
    const double si = rad[i];
    double s = 5.0 * M_1_PI / 4.0 / (si * si * si) * dot3(ai, ai);
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double *xj = pos + 3 * j, *aj = vor + 3 * j;
      double x12[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      const double rho = sqrt(dot3(x12, x12));
      const double sigma = sqrt(0.5 * (si * si + rad[j] * rad[j]));
      const double rho2 = rho * rho, sig2 = sigma * sigma;
      const double p = rho2 + sig2;
      const double factor = (M_1_PI / 8.0) / sqrt(p * p * p * p * p * p * p);
      const double F1 = factor * (10.0 * sig2 * sig2 - 2.0 * rho2 * rho2 - 7.0 * sig2 * rho2);
      const double F2 = factor * (-15.0 * rho2);
      s += F1 * dot3(ai, aj) + F2 * dot3(ai, x12) * dot3(aj, x12);
    }
    total += s;
  }
  return total;
}

/* Helicity: interaction.cpp:317-349 with HELICITY (interaction_utils.h:167-190):
 * H(i,j) = q(rho, sigma) * (x_ij . (alpha_i x alpha_j)), summed over ordered pairs. */
double orc_helicity(size_t n, const double *pos, const double *vor, const double *rad) {
  double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 16)
  for (long il = 0; il < (long)n; ++il) {
    const size_t i = (size_t)il;
    const double *xi = pos + 3 * i, *ai = vor + 3 * i;
    double h = 0.0;
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double *xj = pos + 3 * j, *aj = vor + 3 * j;
      double x12[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      const double rho = sqrt(dot3(x12, x12));
      const double sigma = sqrt(0.5 * (rad[i] * rad[i] + rad[j] * rad[j]));
      double axa[3];
      cross3(ai, aj, axa);
      h += kernel_q(rho, sigma) * dot3(x12, axa);
    }
    total += h;
  }
  return total;
}

/* Kinetic energy: interaction.cpp:351-383 with KINETICENERGY
 * (interaction_utils.h:197-240).  Within a wake the reference returns
 * 2*(sum_i self_i + 2*sum_{i<j} KE_ij); across wakes 2*sum_{i,j} KE_ij. */
double orc_kinetic_energy(size_t n, const int32_t *wake_id, const double *pos,
                          const double *vor, const double *rad) {
  double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 16)
  for (long il = 0; il < (long)n; ++il) {
    const size_t i = (size_t)il;
    const double *xi = pos + 3 * i, *ai = vor + 3 * i;
    double ke = 2.0 * (M_1_PI * dot3(ai, ai) / rad[i] / 8.0);
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double *xj = pos + 3 * j, *aj = vor + 3 * j;
      double x12[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      const double rho2 = dot3(x12, x12);
      const double sigma2 = 0.5 * (rad[i] * rad[i] + rad[j] * rad[j]);
      const double e = ((rho2 + 2.0 * sigma2) * dot3(ai, aj) + dot3(x12, ai) * dot3(x12, aj)) /
                       pow(rho2 + sigma2, 1.5) / 16.0 / M_PI;
      ke += (wake_id[i] == wake_id[j] ? 2.0 : 1.0) * e;
    }
    total += ke;
  }
  return total;
}

/* Vorticity field, __interaction::influence (interaction.cpp:110-155):
 *   SELFINFLUENCE (interaction_utils.h:593-605): K_i += ZETASIG(0, s_i) alpha_i
 *   INFLUENCE (:519-556): sigma = sqrt(0.5 (s_i^2 + s_j^2)), rho = |x_i - x_j|,
 *     Z = ZETASIG(rho, sigma) (highorder.h:20-23); K_target += Z alpha_source and
 *     K_source += Z alpha_target (VORTICITY :38-43), i.e. in gather form
 *     K_i += Z alpha_j for every j != i. */
void orc_influence(size_t n, const double *pos, const double *vor, const double *rad,
                   double *field) {
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t i = 0; i < n; ++i) {
    const double *xi = pos + 3 * i;
    const double si = rad[i];
    const double zs = zeta(0.0, si);
    double k[3] = {zs * vor[3 * i], zs * vor[3 * i + 1], zs * vor[3 * i + 2]};
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double *xj = pos + 3 * j;
      const double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
      const double rho = sqrt(dot3(d, d));
      const double sj = rad[j];
      const double sigma = sqrt(0.5 * (si * si + sj * sj));
      const double z = zeta(rho, sigma);
      for (int c = 0; c < 3; ++c) k[c] += z * vor[3 * j + c];
    }
    for (int c = 0; c < 3; ++c) field[3 * i + c] = k[c];
  }
}
