/* Test infrastructure (oracle): a plain-C, FP64 restatement of pawan's hot
 * path in one-sided "gather" form.  Used only by tests, the smoke check and
 * bench.py's CPU-baseline leg, as the checker at sizes where running the
 * reference itself (oracle/_ref) would take too long.  It is validated against
 * the compiled reference in tests/test_oracle.py.
 *
 * Particle arrays are the union of a system's wakes in wake order:
 * pos/vor are N x 3 row-major, rad/vol are N.
 */
#ifndef PAWAN_ORACLE_RESTATE_H
#define PAWAN_ORACLE_RESTATE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Smoothing kernel of every function below: 0 = high-order algebraic
 * (src/interaction/highorder.h, the reference's default), 1 = Gaussian
 * (src/interaction/gaussian.h). */
void orc_set_kernel(int kernel);

/* Velocity and vorticity rate of the targets listed in `targets` (or all N when
 * targets == NULL, nt == N), summed over every source j != target. */
void orc_pairs(size_t n, const double *pos, const double *vor, const double *rad,
               const double *vol, double nu, size_t nt, const int64_t *targets,
               double *vel, double *dvor);

/* One classical RK4 step of the state [pos | vor] (both N x 3, updated in
 * place), with the stage order of the reference integrator. */
void orc_rk4_step(size_t n, double *pos, double *vor, const double *rad, const double *vol,
                  double nu, double dt);

/* out[0..2] total vorticity, out[3..5] linear impulse, out[6..8] angular impulse. */
void orc_linear_diagnostics(size_t n, const double *pos, const double *vor, double *out);

double orc_enstrophy(size_t n, const double *pos, const double *vor, const double *rad);
double orc_helicity(size_t n, const double *pos, const double *vor, const double *rad);
/* Smoothed vorticity field of every particle (N x 3):
 *   K_i = Z(0, s_i) alpha_i + sum_{j != i} Z(rho_ij, sigma_ij) alpha_j. */
void orc_influence(size_t n, const double *pos, const double *vor, const double *rad,
                   double *field);

/* wake_id[i] is the wake a particle belongs to (pairs inside one wake are
 * weighted twice as much as pairs across wakes, as the reference does). */
double orc_kinetic_energy(size_t n, const int32_t *wake_id, const double *pos,
                          const double *vor, const double *rad);

#ifdef __cplusplus
}
#endif

#endif
