/*
 * pic3d_main.c -- host driver in C for the B200 PIC step, in the shape of the
 * reference's main()/main_func()/fdtd() (PIC/3d_pic458_domain.c:192-289,
 * 627-952) at MPI size 1: set up the domain, initialise grid and particles,
 * run the time loop through the C ABI, and print the thrust_f diagnostics
 * every `thrust_every` steps in the reference's thrust458.txt column layout
 * (:5111-5119) to stdout. As fdtd does (:913-926), it also appends those lines
 * to thrust458.txt in `outdir` and, after every step, hands thrust_fave's
 * running mean to pic_append_thrust_ave, which writes thrust458_ave.txt and
 * restarts the mean at steps that are multiples of 500 (:5267-5280).
 *
 * usage: pic3d_main [nx ny nz np steps precision sort_every thrust_every outdir]
 * (normalized units: c = e0 = mu0 = q = m_e = dx = 1, m_i = 100)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "plasma_b200.h"

#define CHECK(call)                                                              \
  do {                                                                           \
    int rc_ = (call);                                                            \
    if (rc_ != PIC_OK) {                                                         \
      fprintf(stderr, "%s failed: %s\n", #call, pic_error_string(rc_));          \
      return 1;                                                                  \
    }                                                                            \
  } while (0)

int main(int argc, char **argv)
{
  int nx = argc > 1 ? atoi(argv[1]) : 32;
  int ny = argc > 2 ? atoi(argv[2]) : 32;
  int nz = argc > 3 ? atoi(argv[3]) : 32;
  int np = argc > 4 ? atoi(argv[4]) : 8;
  int steps = argc > 5 ? atoi(argv[5]) : 100;
  int precision = argc > 6 ? atoi(argv[6]) : 32;
  int sort_every = argc > 7 ? atoi(argv[7]) : 20;
  int thrust_every = argc > 8 ? atoi(argv[8]) : 10;
  const char *outdir = argc > 9 ? argv[9] : ".";

  pic_config cfg;
  CHECK(pic_config_default(&cfg, nx, ny, nz));
  cfg.np = np;
  cfg.precision = precision;
  cfg.dx = 1.0;
  cfg.dt = 0.5 * 6.0 / (7.0 * sqrt(3.0));
  cfg.q = 1.0; cfg.mi = 100.0; cfg.me = 1.0;
  cfg.mu0 = 1.0; cfg.e0 = 1.0; cfg.kb = 1.0; cfg.c = 1.0;
  cfg.v_drift = 0.1; cfg.n_all = 0.01; cfg.ti = 0.0025; cfg.te = 0.0025;
  cfg.coil_r = 2.0; cfg.coil_i = 32.0;
  cfg.absorb_grid = 0; cfg.absorb_grid2 = 0;
  cfg.sort_interval = sort_every;
  cfg.diag_every_step = 1;

  pic_ctx *ctx = NULL;
  CHECK(pic_create(&cfg, &ctx));
  CHECK(pic_init_grid(ctx));            /* init_grid, :272 */
  CHECK(pic_init_particle_flat(ctx));   /* init_particle_flat, :274 */
  CHECK(pic_fdtd(ctx, 0));              /* fdtd's refill before its loop, :673-674 */
  for (int c = 0; c < steps; ++c) {
    CHECK(pic_step(ctx, 1));
    if (c % thrust_every == 0) {
      double F[PIC_NUM_THRUST], E[PIC_NUM_ENERGY];
      CHECK(pic_thrust_f(ctx, F, E));
      CHECK(pic_append_thrust(ctx, outdir, c));
      printf("%d", c);
      for (int q = 0; q < PIC_NUM_THRUST; ++q) printf(" %.3E", F[q]);
      for (int q = 0; q < PIC_NUM_ENERGY; ++q) printf(" %.8E", E[q]);
      printf("\n");
    }
    CHECK(pic_append_thrust_ave(ctx, outdir, c));
  }
  long long status[8];
  int rc = pic_status(ctx, status);
  if (rc != PIC_OK)
    fprintf(stderr, "device counters: oob %lld range %lld nonfinite %lld\n", status[0], status[1], status[2]);
  long long ni = 0, ne = 0;
  CHECK(pic_particle_count(ctx, PIC_ION, &ni));
  CHECK(pic_particle_count(ctx, PIC_ELECTRON, &ne));
  fprintf(stderr, "steps %d ions %lld electrons %lld pushes %lld\n", steps, ni, ne, status[3]);
  CHECK(pic_destroy(ctx));
  return rc == PIC_OK ? 0 : 2;
}
