/* A C program that uses the library through include/pawan_b200.h only -- the
 * way a C or Fortran code, or another language's FFI, would.  Reads a system
 * from a binary file, runs one solve (as __interaction::solve) and nsteps RK4
 * steps (as __rk4::step), and writes the rates and the final state.
 *
 *   solve_file <in> <out> <precision 0|1|2> <nsteps> <dt>
 *
 * in:  int64 n_wakes, int64 counts[n_wakes], f64 nu,
 *      f64 pos[N*3], vor[N*3], rad[N], vol[N]          (N = sum of counts)
 * out: f64 rates[6N], f64 state[6N]                    (reference layout) */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "pawan_b200.h"

static int read_all(FILE *f, void *p, size_t size, size_t count) {
  return fread(p, size, count, f) == count ? 0 : 1;
}

int main(int argc, char **argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s in out precision nsteps dt\n", argv[0]);
    return 2;
  }
  const int precision = atoi(argv[3]);
  const size_t nsteps = (size_t)atol(argv[4]);
  const double dt = atof(argv[5]);
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  int64_t nw = 0;
  if (read_all(f, &nw, sizeof nw, 1) || nw <= 0 || nw > 1024) return 4;
  size_t *counts = malloc(sizeof(size_t) * (size_t)nw);
  size_t n = 0;
  for (int64_t w = 0; w < nw; ++w) {
    int64_t c = 0;
    if (read_all(f, &c, sizeof c, 1) || c <= 0) return 4;
    counts[w] = (size_t)c;
    n += (size_t)c;
  }
  double nu = 0.0;
  double *pos = malloc(sizeof(double) * 3 * n), *vor = malloc(sizeof(double) * 3 * n);
  double *rad = malloc(sizeof(double) * n), *vol = malloc(sizeof(double) * n);
  if (read_all(f, &nu, sizeof nu, 1) || read_all(f, pos, sizeof(double), 3 * n) ||
      read_all(f, vor, sizeof(double), 3 * n) || read_all(f, rad, sizeof(double), n) ||
      read_all(f, vol, sizeof(double), n))
    return 4;
  fclose(f);

  pawan_ctx *ctx = NULL;
  pawan_system *sys = NULL;
  int st = pawan_ctx_create(0, &ctx);
  if (st != PAWAN_OK) {
    fprintf(stderr, "context: %s\n", pawan_status_name(st));
    return 5;
  }
  double *rates = malloc(sizeof(double) * 6 * n), *state = malloc(sizeof(double) * 6 * n);
  st = pawan_system_create(ctx, (size_t)nw, counts, nu, precision, &sys);
  if (st == PAWAN_OK) st = pawan_system_set_particles(sys, pos, vor, rad, vol);
  if (st == PAWAN_OK) st = pawan_system_solve(sys);
  if (st == PAWAN_OK) st = pawan_system_get_rates(sys, rates, 6 * n);
  if (st == PAWAN_OK && nsteps > 0) st = pawan_system_rk4(sys, dt, nsteps);
  if (st == PAWAN_OK) st = pawan_system_get_states(sys, state, 6 * n);
  if (st != PAWAN_OK) {
    fprintf(stderr, "pawan: %s (%s)\n", pawan_status_name(st), pawan_ctx_last_error(ctx));
    return 6;
  }
  pawan_system_destroy(sys);
  pawan_ctx_destroy(ctx);
  FILE *o = fopen(argv[2], "wb");
  if (!o || fwrite(rates, sizeof(double), 6 * n, o) != 6 * n ||
      fwrite(state, sizeof(double), 6 * n, o) != 6 * n)
    return 7;
  fclose(o);
  printf("solved %zu particles in %lld wakes\n", n, (long long)nw);
  free(counts);
  free(pos);
  free(vor);
  free(rad);
  free(vol);
  free(rates);
  free(state);
  return 0;
}
