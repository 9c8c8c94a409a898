/*
 * pic_oracle.c -- FP64 CPU restatement of the 3D PIC time step of the reference
 * program PIC/3d_pic458_domain.c at MPI size 1 (one domain, PROCESS_Nx =
 * PROCESS_Ny = 1). TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * CPU-baseline leg of the benchmark may call it; the product never does.
 *
 * Parity pin: tests compare every function here with the reference's own code
 * compiled by oracle/build.py (oracle/_ref/libref3d_*.so) on identical inputs;
 * expressions are written in the reference's evaluation order so that the
 * deterministic pieces agree bit for bit (gcc -O2 -ffp-contract=off on both).
 * Random draws use the same project-written generator as the compiled
 * reference (oracle/shim/gsl_shim.c: Philox4x32-10 streams keyed like
 * init_particle_flat's gsl_rng_set calls, :437-446).
 *
 * Where the reference's linked-list code has accidents, this restatement
 * follows the evident intent and the differences are listed here:
 *  - del_particle_i/e (:2873-2927) leave the list cursor on the new head after
 *    deleting a head node, so the loops of sr_particle / add_*_flat / sorting
 *    skip the node after a deleted head. Every particle is examined here.
 *  - sorting (:7475-7590) loses the second node of every list for the same
 *    reason. Nothing is lost here.
 *  - thrust_f / thrust_fave (:4940-5285) stop at the last node of each list
 *    (while p->next_particle != NULL). All particles are summed here.
 *  - init_particle_flat (:412-625) creates Np*Nx*Ny*Nz/THREAD_N + 1 particles
 *    per thread: the extra one lands in ghost cell x index Nx+2 and is deleted
 *    by the add_*_flat call that fdtd makes before its loop. It is created here
 *    too (its random draws shift every later draw).
 *
 * Layout: the grid is the reference's Grid struct as 18 doubles per node in
 * grid[k][l][m] order (z fastest); particles are rows x,y,z,vx,vy,vz,n + flag.
 *
 * Parameters (or_create's double array, index: meaning, reference symbol):
 *   0 nx  1 ny  2 nz  3 np (Grid_Nx, Grid_Ny, Grid_Nz, Np)   4 thread_n (THREAD_N)
 *   5 dx  6 dt  7 q  8 mi  9 me  10 mu0  11 e0  12 kb  13 c
 *   14 V  15 Nall  16 Ti  17 Te  18 R  19 I  20 alpha  21 IMF_x 22 IMF_y 23 IMF_z
 *   24 Absorb_grid  25 Absorb_grid2  26 sigma amplitude a (init_grid :295)
 *   27 dipole cutoff radius in cells (external_current7 :4596, 210)
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "shim/gsl/gsl_shim.h"

#define NF 18
enum { G_BX, G_BY, G_BZ, G_B0X, G_B0Y, G_B0Z, G_EX, G_EY, G_EZ,
       G_JIX, G_JIY, G_JIZ, G_JEX, G_JEY, G_JEZ, G_NI, G_NE, G_PHI };

typedef struct {
  long n, cap;
  double *r;   /* rows of 7: x y z vx vy vz n */
  int *flag;
} or_species;

typedef struct {
  int nx, ny, nz, np, thread_n;
  double dx, dt, q, mi, me, mu0, e0, kb, c;
  double V, Nall, Ti, Te, R, I, alpha, imfx, imfy, imfz;
  int absorb, absorb2;
  double sigma_a, cutoff;
  int gx, gy, gz;           /* nx+4 ... */
  double *g;                /* nodes * NF */
  double *sigma;            /* (2gx)(2gy)(2gz) */
  or_species sp[2];         /* 0 ion, 1 electron */
  gsl_rng *rnd_p, *rnd_v;   /* thread 0 streams (thread_n == 1) */
  double fave[27];
} or_ctx;

#define NODE(c, k, l, m) ((((long)(k) * (c)->gy + (l)) * (c)->gz + (m)) * NF)
#define GV(c, k, l, m, f) ((c)->g[NODE(c, k, l, m) + (f)])
#define SIG(c, k, l, m) ((c)->sigma[((long)(k) * 2 * (c)->gy + (l)) * 2 * (c)->gz + (m)])

/* ------------------------------------------------------------------ setup */
or_ctx *or_create(const double *p)
{
  or_ctx *c = (or_ctx *)calloc(1, sizeof(or_ctx));
  c->nx = (int)p[0]; c->ny = (int)p[1]; c->nz = (int)p[2]; c->np = (int)p[3];
  c->thread_n = (int)p[4];
  c->dx = p[5]; c->dt = p[6]; c->q = p[7]; c->mi = p[8]; c->me = p[9];
  c->mu0 = p[10]; c->e0 = p[11]; c->kb = p[12]; c->c = p[13];
  c->V = p[14]; c->Nall = p[15]; c->Ti = p[16]; c->Te = p[17];
  c->R = p[18]; c->I = p[19]; c->alpha = p[20];
  c->imfx = p[21]; c->imfy = p[22]; c->imfz = p[23];
  c->absorb = (int)p[24]; c->absorb2 = (int)p[25]; c->sigma_a = p[26]; c->cutoff = p[27];
  c->gx = c->nx + 4; c->gy = c->ny + 4; c->gz = c->nz + 4;
  c->g = (double *)calloc((size_t)c->gx * c->gy * c->gz * NF, sizeof(double));
  c->sigma = (double *)calloc((size_t)8 * c->gx * c->gy * c->gz, sizeof(double));
  c->rnd_p = gsl_rng_alloc(gsl_rng_rand);
  c->rnd_v = gsl_rng_alloc(gsl_rng_rand);
  gsl_rng_set(c->rnd_p, 0);   /* (rank*10000 + thread*100), :444 */
  gsl_rng_set(c->rnd_v, 50);  /* (rank*10000 + thread*100 + 50), :445 */
  return c;
}

void or_destroy(or_ctx *c)
{
  if (!c) return;
  for (int s = 0; s < 2; ++s) { free(c->sp[s].r); free(c->sp[s].flag); }
  free(c->g); free(c->sigma);
  gsl_rng_free(c->rnd_p); gsl_rng_free(c->rnd_v);
  free(c);
}

long or_grid_nodes(const or_ctx *c) { return (long)c->gx * c->gy * c->gz; }
void or_get_grid(const or_ctx *c, double *out) { memcpy(out, c->g, sizeof(double) * or_grid_nodes(c) * NF); }
void or_set_grid(or_ctx *c, const double *in) { memcpy(c->g, in, sizeof(double) * or_grid_nodes(c) * NF); }
void or_get_sigma(const or_ctx *c, double *out) { memcpy(out, c->sigma, sizeof(double) * 8 * or_grid_nodes(c)); }

long long or_rng_counter(or_ctx *c, int which, long long set)
{
  gsl_rng *r = which == 0 ? c->rnd_p : c->rnd_v;
  if (set >= 0) r->counter = (uint64_t)set;
  return (long long)r->counter;
}

static void sp_reserve(or_species *s, long n)
{
  if (n <= s->cap) return;
  long cap = s->cap ? s->cap : 1024;
  while (cap < n) cap *= 2;
  s->r = (double *)realloc(s->r, sizeof(double) * 7 * cap);
  s->flag = (int *)realloc(s->flag, sizeof(int) * cap);
  s->cap = cap;
}

static void sp_push(or_species *s, double x, double y, double z, double vx, double vy,
                    double vz, double w, int flag)
{
  sp_reserve(s, s->n + 1);
  double *r = s->r + 7 * s->n;
  r[0] = x; r[1] = y; r[2] = z; r[3] = vx; r[4] = vy; r[5] = vz; r[6] = w;
  s->flag[s->n] = flag;
  s->n++;
}

long or_count(const or_ctx *c, int species) { return c->sp[species].n; }

void or_set_particles(or_ctx *c, int species, const double *rows, const int *flag, long n)
{
  or_species *s = &c->sp[species];
  s->n = 0;
  sp_reserve(s, n);
  if (n > 0) memcpy(s->r, rows, sizeof(double) * 7 * n);
  for (long i = 0; i < n; ++i) s->flag[i] = flag ? flag[i] : 1;
  s->n = n;
}

long or_get_particles(const or_ctx *c, int species, double *rows, int *flag, long cap)
{
  const or_species *s = &c->sp[species];
  long n = s->n < cap ? s->n : cap;
  if (n > 0) memcpy(rows, s->r, sizeof(double) * 7 * n);
  if (flag) for (long i = 0; i < n; ++i) flag[i] = s->flag[i];
  return s->n;
}

/* Removes particles whose mask byte is set, keeping the order of the rest. */
static void sp_compact(or_species *s, const unsigned char *dead)
{
  long w = 0;
  for (long i = 0; i < s->n; ++i) {
    if (dead[i]) continue;
    if (w != i) {
      memcpy(s->r + 7 * w, s->r + 7 * i, sizeof(double) * 7);
      s->flag[w] = s->flag[i];
    }
    w++;
  }
  s->n = w;
}

/* ------------------------------------------------------------ init_grid */
/* external_current7, PIC/3d_pic458_domain.c:4579-4634, at rank (0,0). */
static void or_dipole(or_ctx *c)
{
  const double dx = c->dx, mu0 = c->mu0, I = c->I, R = c->R, alpha = c->alpha;
  const double Pi = M_PI;
  const int cx = (1 * c->nx + 4) / 2, cy = (1 * c->ny + 4) / 2, cz = (c->nz + 4) / 2;
  for (int k = 0; k < c->gx; k++)
    for (int l = 0; l < c->gy; l++)
      for (int m = 0; m < c->gz; m++) {
        double x = (k + 0 * c->nx - cx) * dx;
        double y = (l + 0 * c->ny - cy) * dx;
        double z = (m - cz) * dx;
        double r = sqrt(x * x + y * y + z * z);
        if (r < c->cutoff * dx) {
          x = (k + 0 * c->nx - cx + 0.5) * dx;
          y = (l + 0 * c->ny - cy) * dx;
          z = (m - cz) * dx;
          r = sqrt(x * x + y * y + z * z);
          GV(c, k, l, m, G_B0X) = mu0 * I * Pi * R * R * (3. * x * y * sin(alpha) + 3. * x * z * cos(alpha)) / (4. * Pi * pow(r, 5)) + c->imfx;
          GV(c, k, l, m, G_BX) = GV(c, k, l, m, G_B0X);
          x = (k + 0 * c->nx - cx) * dx;
          y = (l + 0 * c->ny - cy + 0.5) * dx;
          z = (m - cz) * dx;
          r = sqrt(x * x + y * y + z * z);
          GV(c, k, l, m, G_B0Y) = mu0 * I * Pi * R * R * (3. * y * y * sin(alpha) + 3. * y * z * cos(alpha) - r * r * sin(alpha)) / (4. * Pi * pow(r, 5)) + c->imfy;
          GV(c, k, l, m, G_BY) = GV(c, k, l, m, G_B0Y);
          x = (k + 0 * c->nx - cx) * dx;
          y = (l + 0 * c->ny - cy) * dx;
          z = (m - cz + 0.5) * dx;
          r = sqrt(x * x + y * y + z * z);
          GV(c, k, l, m, G_B0Z) = mu0 * I * Pi * R * R * (3. * y * z * sin(alpha) + 3. * z * z * cos(alpha) - r * r * cos(alpha)) / (4. * Pi * pow(r, 5)) + c->imfz;
          GV(c, k, l, m, G_BZ) = GV(c, k, l, m, G_B0Z);
        } else {
          GV(c, k, l, m, G_BX) = c->imfx; GV(c, k, l, m, G_BY) = c->imfy; GV(c, k, l, m, G_BZ) = c->imfz;
          GV(c, k, l, m, G_B0X) = c->imfx; GV(c, k, l, m, G_B0Y) = c->imfy; GV(c, k, l, m, G_B0Z) = c->imfz;
        }
      }
}

/* Damping ramp value on the doubled sub-grid for one axis (init_grid :339-365). */
static double ramp(int idx, int n_total, int absorb)
{
  if (idx - 4 <= 2 * absorb) return (2 * absorb - (idx - 4)) / 4.;
  if (idx - 4 >= 2 * n_total - 2 * absorb) return (idx - 4 - (2 * n_total - 2 * absorb)) / 4.;
  return 0.;
}

/* init_grid, PIC/3d_pic458_domain.c:291-410 (PHI() blocks compiled out). */
void or_init_grid(or_ctx *c)
{
  memset(c->g, 0, sizeof(double) * or_grid_nodes(c) * NF);
  or_dipole(c);
  const double a = c->sigma_a;
  for (int k = 0; k < 2 * c->gx; k++)
    for (int l = 0; l < 2 * c->gy; l++)
      for (int m = 0; m < 2 * c->gz; m++) {
        const double x = ramp(k, c->nx, c->absorb);
        const double y = ramp(l, c->ny, c->absorb);
        const double z = ramp(m, c->nz, c->absorb);
        SIG(c, k, l, m) = a * (0.1 * sqrt(pow(x, 4) + pow(y, 4) + pow(z, 4))
                               + 0.01 * sqrt(pow(x, 12) + pow(y, 12) + pow(z, 12)));
      }
}

/* ---------------------------------------------------- particle sources */
/* ran_multivar_gaussian (:7956-7985) with a diagonal covariance: the Cholesky
 * factor is diag(sqrt(sigma0^2)) and dgemv adds exact zeros. */
static void maxwellian(or_ctx *c, double sig, double *v)
{
  double g[3];
  for (int j = 0; j < 3; ++j) g[j] = gsl_ran_gaussian(c->rnd_v, 1.);
  const double l = sqrt(sig * sig);
  v[0] = l * g[0] + 0.0;
  v[1] = l * g[1] + 0.0;
  v[2] = l * g[2] + c->V;
}

/* init_particle_flat, :412-625, one thread (THREAD_N = 1). */
void or_init_particle_flat(or_ctx *c)
{
  const double dx = c->dx;
  gsl_rng_set(c->rnd_p, 0);
  gsl_rng_set(c->rnd_v, 50);
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    sp->n = 0;
    const long loop = (long)c->np * c->nx * c->ny * c->nz;
    sp_reserve(sp, loop + 1);
    const double sig = s == 0 ? sqrt(c->kb * c->Ti / c->mi) : sqrt(c->kb * c->Te / c->me);
    const double w = c->Nall / c->np;
    int k = 0, l = 0, m = 0, n = 0;
    for (long j = 0; j <= loop; ++j) {
      const double x = gsl_ran_flat(c->rnd_p, 2. * dx + k * dx, 2. * dx + (k + 1) * dx);
      const double y = gsl_ran_flat(c->rnd_p, 2. * dx + l * dx, 2. * dx + (l + 1) * dx);
      const double z = gsl_ran_flat(c->rnd_p, 2. * dx + m * dx, 2. * dx + (m + 1) * dx);
      double v[3];
      maxwellian(c, sig, v);
      sp_push(sp, x, y, z, v[0], v[1], v[2], w, 1);
      if (j == loop) break;
      if (++n == c->np) { n = 0; m++; }
      if (m == c->nz) { m = 0; l++; }
      if (l == c->ny) { l = 0; k++; }
    }
  }
}

/* One refill slab of add_*_flat: cells [k0,k0+nk) x [l0,l0+nl) x [m0,m0+nm)
 * (absolute cell indices), Np/THREAD_N particles per cell, k outermost. */
static void fill_slab(or_ctx *c, or_species *sp, double sig, double w,
                      int k0, int nk, int l0, int nl, int m0, int nm)
{
  const double dx = c->dx;
  for (int k = 0; k < nk; k++)
    for (int l = 0; l < nl; l++)
      for (int m = 0; m < nm; m++)
        for (int j = 0; j < c->np / c->thread_n; j++) {
          const double x = gsl_ran_flat(c->rnd_p, (k + k0) * dx, (k + k0 + 1) * dx);
          const double y = gsl_ran_flat(c->rnd_p, (l + l0) * dx, (l + l0 + 1) * dx);
          const double z = gsl_ran_flat(c->rnd_p, (m + m0) * dx, (m + m0 + 1) * dx);
          double v[3];
          maxwellian(c, sig, v);
          sp_push(sp, x, y, z, v[0], v[1], v[2], w, 1);
        }
}

/* add_ion_flat / add_electron_flat, :5993-6404 / :6406-6818, at rank (0,0) of a
 * 1x1 layout: shell deletion, then the xy slabs, the xz slabs and the first
 * branch of the x-slab chain (myrank_x == 0 && myrank_y == 0). */
void or_add_flat(or_ctx *c)
{
  const double dx = c->dx;
  const int Nx = c->nx, Ny = c->ny, Nz = c->nz;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    unsigned char *dead = (unsigned char *)calloc((size_t)(sp->n > 0 ? sp->n : 1), 1);
    for (long i = 0; i < sp->n; ++i) {
      const double *r = sp->r + 7 * i;
      if (r[0] < 4 * dx || r[0] > Nx * dx || r[1] < 4 * dx || r[1] > Ny * dx ||
          r[2] < 4 * dx || r[2] > Nz * dx)
        dead[i] = 1;
    }
    sp_compact(sp, dead);
    free(dead);
    const double sig = s == 0 ? sqrt(c->kb * c->Ti / c->mi) : sqrt(c->kb * c->Te / c->me);
    const double w = c->Nall / c->np;
    fill_slab(c, sp, sig, w, 2, Nx, 2, Ny, 2, 2);             /* :6037-6071 z low  */
    fill_slab(c, sp, sig, w, 2, Nx, 2, Ny, Nz, 2);            /* :6073-6107 z high */
    fill_slab(c, sp, sig, w, 2, Nx, 2, 2, 4, Nz - 4);         /* :6111-6146 y low  */
    fill_slab(c, sp, sig, w, 2, Nx, Ny, 2, 4, Nz - 4);        /* :6148-6183 y high */
    fill_slab(c, sp, sig, w, 2, 2, 4, Ny - 2, 4, Nz - 4);     /* :6186-6220 x low  */
  }
}

/* ------------------------------------------------------------- fields */
/* renew_grid, :2533-2578: zero currents, densities and phi. */
void or_renew_grid(or_ctx *c)
{
  const long nn = or_grid_nodes(c);
  for (long i = 0; i < nn; ++i)
    for (int f = G_JIX; f <= G_PHI; ++f) c->g[i * NF + f] = 0.;
}

/* renew_b4_2, :2580-2611. */
void or_renew_b(or_ctx *c)
{
  const double temp = 1. / c->e0 * c->dt * 0.5 * 0.5;
  const double dth = 0.5 * c->dt;
  const double temp_24 = 1. / 24.;
  const double inv_dx = 1. / c->dx;
#define G(k, l, m, f) GV(c, k, l, m, f)
  for (int k = 2; k < c->nx + 2; k++)
    for (int l = 2; l < c->ny + 2; l++)
      for (int m = 2; m < c->nz + 2; m++) {
        double s = SIG(c, 2 * k + 1, 2 * l, 2 * m);
        G(k, l, m, G_BX) = G(k, l, m, G_B0X)
          + (1. - s * temp) / (1. + s * temp) * (G(k, l, m, G_BX) - G(k, l, m, G_B0X))
          - dth / (1. + s * temp)
          * temp_24 * (27. * (G(k, l, m, G_EZ) - G(k, l - 1, m, G_EZ) - G(k, l, m, G_EY) + G(k, l, m - 1, G_EY))
                       - (G(k, l + 1, m, G_EZ) - G(k, l - 2, m, G_EZ) - G(k, l, m + 1, G_EY) + G(k, l, m - 2, G_EY))) * inv_dx;
        s = SIG(c, 2 * k, 2 * l + 1, 2 * m);
        G(k, l, m, G_BY) = G(k, l, m, G_B0Y)
          + (1. - s * temp) / (1. + s * temp) * (G(k, l, m, G_BY) - G(k, l, m, G_B0Y))
          - dth / (1. + s * temp)
          * temp_24 * (27. * (G(k, l, m, G_EX) - G(k, l, m - 1, G_EX) - G(k, l, m, G_EZ) + G(k - 1, l, m, G_EZ))
                       - (G(k, l, m + 1, G_EX) - G(k, l, m - 2, G_EX) - G(k + 1, l, m, G_EZ) + G(k - 2, l, m, G_EZ))) * inv_dx;
        s = SIG(c, 2 * k, 2 * l, 2 * m + 1);
        G(k, l, m, G_BZ) = G(k, l, m, G_B0Z)
          + (1. - s * temp) / (1. + s * temp) * (G(k, l, m, G_BZ) - G(k, l, m, G_B0Z))
          - dth / (1. + s * temp)
          * temp_24 * (27. * (G(k, l, m, G_EY) - G(k - 1, l, m, G_EY) - G(k, l, m, G_EX) + G(k, l - 1, m, G_EX))
                       - (G(k + 1, l, m, G_EY) - G(k - 2, l, m, G_EY) - G(k, l + 1, m, G_EX) + G(k, l - 2, m, G_EX))) * inv_dx;
      }
}

/* renew_e4_2, :2613-2652. */
void or_renew_e(or_ctx *c)
{
  const double mu0 = c->mu0;
  const double temp = c->c * c->c * c->dt;
  const double temp_24 = 1. / 24.;
  const double inv_dx = 1. / c->dx;
  for (int k = 2; k < c->nx + 2; k++)
    for (int l = 2; l < c->ny + 2; l++)
      for (int m = 2; m < c->nz + 2; m++) {
        double s = SIG(c, 2 * k, 2 * l + 1, 2 * m + 1);
        G(k, l, m, G_EX) = (1. - 0.5 * mu0 * s * temp) / (1. + 0.5 * mu0 * s * temp) * G(k, l, m, G_EX)
          + temp / (1. + 0.5 * mu0 * s * temp)
          * (temp_24 * (27. * ((G(k, l + 1, m, G_BZ) - G(k, l + 1, m, G_B0Z) - G(k, l, m, G_BZ) + G(k, l, m, G_B0Z))
                               - (G(k, l, m + 1, G_BY) - G(k, l, m + 1, G_B0Y) - G(k, l, m, G_BY) + G(k, l, m, G_B0Y)))
                        - ((G(k, l + 2, m, G_BZ) - G(k, l + 2, m, G_B0Z) - G(k, l - 1, m, G_BZ) + G(k, l - 1, m, G_B0Z))
                           - (G(k, l, m + 2, G_BY) - G(k, l, m + 2, G_B0Y) - G(k, l, m - 1, G_BY) + G(k, l, m - 1, G_B0Y)))) * inv_dx
             - mu0 * (G(k, l, m, G_JIX) - G(k, l, m, G_JEX)));
        s = SIG(c, 2 * k + 1, 2 * l, 2 * m + 1);
        G(k, l, m, G_EY) = (1. - 0.5 * mu0 * s * temp) / (1. + 0.5 * mu0 * s * temp) * G(k, l, m, G_EY)
          + temp / (1. + 0.5 * mu0 * s * temp)
          * (temp_24 * (27. * ((G(k, l, m + 1, G_BX) - G(k, l, m + 1, G_B0X) - G(k, l, m, G_BX) + G(k, l, m, G_B0X))
                               - (G(k + 1, l, m, G_BZ) - G(k + 1, l, m, G_B0Z) - G(k, l, m, G_BZ) + G(k, l, m, G_B0Z)))
                        - ((G(k, l, m + 2, G_BX) - G(k, l, m + 2, G_B0X) - G(k, l, m - 1, G_BX) + G(k, l, m - 1, G_B0X))
                           - (G(k + 2, l, m, G_BZ) - G(k + 2, l, m, G_B0Z) - G(k - 1, l, m, G_BZ) + G(k - 1, l, m, G_B0Z)))) * inv_dx
             - mu0 * (G(k, l, m, G_JIY) - G(k, l, m, G_JEY)));
        s = SIG(c, 2 * k + 1, 2 * l + 1, 2 * m);
        G(k, l, m, G_EZ) = (1. - 0.5 * mu0 * s * temp) / (1. + 0.5 * mu0 * s * temp) * G(k, l, m, G_EZ)
          + temp / (1. + 0.5 * mu0 * s * temp)
          * (temp_24 * (27. * ((G(k + 1, l, m, G_BY) - G(k + 1, l, m, G_B0Y) - G(k, l, m, G_BY) + G(k, l, m, G_B0Y))
                               - (G(k, l + 1, m, G_BX) - G(k, l + 1, m, G_B0X) - G(k, l, m, G_BX) + G(k, l, m, G_B0X)))
                        - ((G(k + 2, l, m, G_BY) - G(k + 2, l, m, G_B0Y) - G(k - 1, l, m, G_BY) + G(k - 1, l, m, G_B0Y))
                           - (G(k, l + 2, m, G_BX) - G(k, l + 2, m, G_B0X) - G(k, l - 1, m, G_BX) + G(k, l - 1, m, G_B0X)))) * inv_dx
             - mu0 * (G(k, l, m, G_JIZ) - G(k, l, m, G_JEZ)));
      }
}

/* sr_b / sr_e at size 1 (:1001-1387): periodic copy of the 2-wide ghost
 * planes, x (all l, m) then y (all k, m). f0 is the first of 3 components. */
static void wrap3(or_ctx *c, int f0)
{
  const int Nx = c->nx, Ny = c->ny;
  for (int f = f0; f < f0 + 3; ++f) {
    for (int l = 0; l < c->gy; l++)
      for (int m = 0; m < c->gz; m++) {
        const double a0 = GV(c, Nx, l, m, f), a1 = GV(c, Nx + 1, l, m, f);
        GV(c, 0, l, m, f) = a0; GV(c, 1, l, m, f) = a1;
        GV(c, Nx + 2, l, m, f) = GV(c, 2, l, m, f); GV(c, Nx + 3, l, m, f) = GV(c, 3, l, m, f);
      }
    for (int k = 0; k < c->gx; k++)
      for (int m = 0; m < c->gz; m++) {
        GV(c, k, 0, m, f) = GV(c, k, Ny, m, f); GV(c, k, 1, m, f) = GV(c, k, Ny + 1, m, f);
        GV(c, k, Ny + 2, m, f) = GV(c, k, 2, m, f); GV(c, k, Ny + 3, m, f) = GV(c, k, 3, m, f);
      }
  }
}
void or_sr_b(or_ctx *c) { wrap3(c, G_BX); }
void or_sr_e(or_ctx *c) { wrap3(c, G_EX); }

/* sr_current2 at size 1 (:1805-2039): additive periodic fold of the ghost
 * planes of the 8 accumulated quantities, x first then y. */
void or_sr_current2(or_ctx *c)
{
  const int Nx = c->nx, Ny = c->ny;
  for (int f = G_JIX; f <= G_NE; ++f) {
    for (int l = 0; l < c->gy; l++)
      for (int m = 0; m < c->gz; m++) {
        GV(c, 2, l, m, f) += GV(c, Nx + 2, l, m, f);
        GV(c, 3, l, m, f) += GV(c, Nx + 3, l, m, f);
      }
    for (int l = 0; l < c->gy; l++)
      for (int m = 0; m < c->gz; m++) {
        GV(c, Nx, l, m, f) += GV(c, 0, l, m, f);
        GV(c, Nx + 1, l, m, f) += GV(c, 1, l, m, f);
      }
    for (int k = 0; k < c->gx; k++)
      for (int m = 0; m < c->gz; m++) {
        GV(c, k, 2, m, f) += GV(c, k, Ny + 2, m, f);
        GV(c, k, 3, m, f) += GV(c, k, Ny + 3, m, f);
      }
    for (int k = 0; k < c->gx; k++)
      for (int m = 0; m < c->gz; m++) {
        GV(c, k, Ny, m, f) += GV(c, k, 0, m, f);
        GV(c, k, Ny + 1, m, f) += GV(c, k, 1, m, f);
      }
  }
}

/* ------------------------------------------------------------ particles */
/* shape_func_v2, :3017-3326: trilinear gather, each component on its stagger. */
static void gather(const or_ctx *c, const double *p, double *out)
{
  const double dx = c->dx;
  const double inv_dx3 = 1. / (dx * dx * dx);
  const int kA = (int)(p[0] / dx), kB = (int)(p[0] / dx - 0.5);
  const int lA = (int)(p[1] / dx), lB = (int)(p[1] / dx - 0.5);
  const int mA = (int)(p[2] / dx), mB = (int)(p[2] / dx - 0.5);
  /* (kind per axis: A = node-aligned, B = half-shifted) for ex, by, ez, bx, ey, bz */
  const int kk[6] = {kA, kA, kB, kB, kB, kA};
  const int ll[6] = {lB, lB, lB, lA, lA, lA};
  const int mm[6] = {mB, mA, mA, mA, mB, mB};
  const int shk[6] = {0, 0, 1, 1, 1, 0}, shl[6] = {1, 1, 1, 0, 0, 0}, shm[6] = {1, 0, 0, 0, 1, 1};
  const int fld[6] = {G_EX, G_BY, G_EZ, G_BX, G_EY, G_BZ};
  double res[6];
  for (int q6 = 0; q6 < 6; ++q6) {
    const int k = kk[q6], l = ll[q6], m = mm[q6];
    const int kkk = k + 1, lll = l + 1, mmm = m + 1;
    const double kkkp = shk[q6] ? ((kkk + 0.5) * dx - p[0]) : (kkk * dx - p[0]);
    const double lllp = shl[q6] ? ((lll + 0.5) * dx - p[1]) : (lll * dx - p[1]);
    const double mmmp = shm[q6] ? ((mmm + 0.5) * dx - p[2]) : (mmm * dx - p[2]);
    const double pk = shk[q6] ? (p[0] - (k + 0.5) * dx) : (p[0] - k * dx);
    const double pl = shl[q6] ? (p[1] - (l + 0.5) * dx) : (p[1] - l * dx);
    const double pm = shm[q6] ? (p[2] - (m + 0.5) * dx) : (p[2] - m * dx);
    const int f = fld[q6];
    double a1 = GV(c, k, l, m, f) * (kkkp * lllp * mmmp) + GV(c, k, l, mmm, f) * (kkkp * lllp * pm);
    double a2 = GV(c, k, lll, m, f) * (kkkp * pl * mmmp) + GV(c, k, lll, mmm, f) * (kkkp * pl * pm);
    double a3 = GV(c, kkk, l, m, f) * (pk * lllp * mmmp) + GV(c, kkk, l, mmm, f) * (pk * lllp * pm);
    double a4 = GV(c, kkk, lll, m, f) * (pk * pl * mmmp) + GV(c, kkk, lll, mmm, f) * (pk * pl * pm);
    res[q6] = (a1 + a2 + a3 + a4) * inv_dx3;
  }
  /* out: ex ey ez bx by bz */
  out[0] = res[0]; out[1] = res[4]; out[2] = res[2];
  out[3] = res[3]; out[4] = res[1]; out[5] = res[5];
}

void or_gather(const or_ctx *c, const double *xyz, double *out6)
{
  double p[7] = {xyz[0], xyz[1], xyz[2], 0, 0, 0, 0};
  gather(c, p, out6);
}

/* cal_track4, :2804-2870 (relativistic variant; gamma of the rotation is
 * taken from u before the first electric half-kick). m < 0 for electrons. */
static void cal_track4(const or_ctx *c, double *p, double m)
{
  double f[6];
  gather(c, p, f);
  double ex = f[0], ey = f[1], ez = f[2], bx = f[3], by = f[4], bz = f[5];
  const double C = c->c;
  const double T = 0.5 * c->q * c->dt / m;
  ex += c->V * c->imfy;
  ey += -c->V * c->imfx;
  double gamma1 = C / sqrt(C * C - p[3] * p[3] - p[4] * p[4] - p[5] * p[5]);
  if (isnan(gamma1)) gamma1 = 0.;
  double ux = gamma1 * p[3], uy = gamma1 * p[4], uz = gamma1 * p[5];
  double gamma2 = C / sqrt(C * C + ux * ux + uy * uy + uz * uz);
  const double bux = gamma2 * (bx), buy = gamma2 * (by), buz = gamma2 * (bz);
  const double S = 2. * T / (1. + T * T * (bux * bux + buy * buy + buz * buz));
  ux += (ex) * T; uy += (ey) * T; uz += (ez) * T;
  const double uox = ux + T * (uy * buz - uz * buy);
  const double uoy = uy + T * (uz * bux - ux * buz);
  const double uoz = uz + T * (ux * buy - uy * bux);
  double upx = ux + S * (uoy * buz - uoz * buy);
  double upy = uy + S * (uoz * bux - uox * buz);
  double upz = uz + S * (uox * buy - uoy * bux);
  upx += (ex) * T; upy += (ey) * T; upz += (ez) * T;
  gamma2 = C / sqrt(C * C + upx * upx + upy * upy + upz * upz);
  p[3] = gamma2 * upx; p[4] = gamma2 * upy; p[5] = gamma2 * upz;
  p[0] += p[3] * c->dt * 0.5;
  p[1] += p[4] * c->dt * 0.5;
  p[2] += p[5] * c->dt * 0.5;
}

/* shape_func_{ion,electron}0_j_2, :3397-3553: J deposit (positive q n v for
 * both species; the E update takes ion minus electron). */
static void deposit_j(or_ctx *c, const double *p, int fx, int fy, int fz)
{
  const double dx = c->dx, dx3 = dx * dx * dx;
  int k = (int)(p[0] / dx), l = (int)(p[1] / dx - 0.5), m = (int)(p[2] / dx - 0.5);
  int kkk = k + 1, lll = l + 1, mmm = m + 1;
  const double qn = c->q * p[6] / dx3;
  double temp = qn * p[3];
  double kkkp = (kkk * dx - p[0]);
  double lllp = ((lll + 0.5) * dx - p[1]);
  double mmmp = ((mmm + 0.5) * dx - p[2]);
  double pk = (p[0] - k * dx);
  double pl = (p[1] - (l + 0.5) * dx);
  double pm = (p[2] - (m + 0.5) * dx);
  double tempkkkp = temp * kkkp, temppk = temp * pk;
  GV(c, k, l, m, fx) += (tempkkkp) * (lllp * mmmp);
  GV(c, k, l, mmm, fx) += (tempkkkp) * (lllp * pm);
  GV(c, k, lll, m, fx) += (tempkkkp) * (pl * mmmp);
  GV(c, k, lll, mmm, fx) += (tempkkkp) * (pl * pm);
  GV(c, kkk, l, m, fx) += (temppk) * (lllp * mmmp);
  GV(c, kkk, l, mmm, fx) += (temppk) * (lllp * pm);
  GV(c, kkk, lll, m, fx) += (temppk) * (pl * mmmp);
  GV(c, kkk, lll, mmm, fx) += (temppk) * (pl * pm);

  k = (int)(p[0] / dx - 0.5); l = (int)(p[1] / dx);
  kkk = k + 1; lll = l + 1;
  temp = qn * p[4];
  kkkp = ((kkk + 0.5) * dx - p[0]);
  lllp = (lll * dx - p[1]);
  pk = (p[0] - (k + 0.5) * dx);
  pl = (p[1] - l * dx);
  tempkkkp = temp * kkkp; temppk = temp * pk;
  GV(c, k, l, m, fy) += (tempkkkp) * (lllp * mmmp);
  GV(c, k, l, mmm, fy) += (tempkkkp) * (lllp * pm);
  GV(c, k, lll, m, fy) += (tempkkkp) * (pl * mmmp);
  GV(c, k, lll, mmm, fy) += (tempkkkp) * (pl * pm);
  GV(c, kkk, l, m, fy) += (temppk) * (lllp * mmmp);
  GV(c, kkk, l, mmm, fy) += (temppk) * (lllp * pm);
  GV(c, kkk, lll, m, fy) += (temppk) * (pl * mmmp);
  GV(c, kkk, lll, mmm, fy) += (temppk) * (pl * pm);

  l = (int)(p[1] / dx - 0.5); m = (int)(p[2] / dx);
  lll = l + 1; mmm = m + 1;
  temp = qn * p[5];
  lllp = ((lll + 0.5) * dx - p[1]);
  mmmp = (mmm * dx - p[2]);
  pl = (p[1] - (l + 0.5) * dx);
  pm = (p[2] - m * dx);
  tempkkkp = temp * kkkp; temppk = temp * pk;
  GV(c, k, l, m, fz) += (tempkkkp) * (lllp * mmmp);
  GV(c, k, l, mmm, fz) += (tempkkkp) * (lllp * pm);
  GV(c, k, lll, m, fz) += (tempkkkp) * (pl * mmmp);
  GV(c, k, lll, mmm, fz) += (tempkkkp) * (pl * pm);
  GV(c, kkk, l, m, fz) += (temppk) * (lllp * mmmp);
  GV(c, kkk, l, mmm, fz) += (temppk) * (lllp * pm);
  GV(c, kkk, lll, m, fz) += (temppk) * (pl * mmmp);
  GV(c, kkk, lll, mmm, fz) += (temppk) * (pl * pm);
}

/* shape_func_{ion,electron}0_n_2, :3333-3395: cell-centred density. */
static void deposit_n(or_ctx *c, const double *p, int f)
{
  const double dx = c->dx, dx3 = dx * dx * dx;
  const int k = (int)(p[0] / dx - 0.5), l = (int)(p[1] / dx - 0.5), m = (int)(p[2] / dx - 0.5);
  const int kkk = k + 1, lll = l + 1, mmm = m + 1;
  const double temp = p[6] / dx3;
  const double kkkp = ((kkk + 0.5) * dx - p[0]);
  const double lllp = ((lll + 0.5) * dx - p[1]);
  const double mmmp = ((mmm + 0.5) * dx - p[2]);
  const double pk = (p[0] - (k + 0.5) * dx);
  const double pl = (p[1] - (l + 0.5) * dx);
  const double pm = (p[2] - (m + 0.5) * dx);
  const double tempkkkp = temp * kkkp, temppk = temp * pk;
  GV(c, k, l, m, f) += (tempkkkp) * (lllp * mmmp);
  GV(c, k, l, mmm, f) += (tempkkkp) * (lllp * pm);
  GV(c, k, lll, m, f) += (tempkkkp) * (pl * mmmp);
  GV(c, k, lll, mmm, f) += (tempkkkp) * (pl * pm);
  GV(c, kkk, l, m, f) += (temppk) * (lllp * mmmp);
  GV(c, kkk, l, mmm, f) += (temppk) * (lllp * pm);
  GV(c, kkk, lll, m, f) += (temppk) * (pl * mmmp);
  GV(c, kkk, lll, mmm, f) += (temppk) * (pl * pm);
}

/* Deposits whose 2x2x2 stencil would leave the (N+4)^3 array are not made
 * (the reference writes past its array there, :747-749 allow x up to (N+4)dx);
 * they are counted instead. */
static long g_oob = 0;
long or_oob_count(void) { return g_oob; }

static int stencil_in_array(const or_ctx *c, const double *p)
{
  const double dx = c->dx;
  return (int)(p[0] / dx) + 1 < c->gx && (int)(p[1] / dx) + 1 < c->gy && (int)(p[2] / dx) + 1 < c->gz;
}

/* Push + J deposit loop of fdtd, :731-812. */
void or_push_j(or_ctx *c)
{
  const double dx = c->dx, dth = c->dt * 0.5;
  const double ax0 = c->absorb2 * dx, ay0 = ax0, az0 = ax0;
  const double ax1 = (1 * c->nx + 4 - c->absorb2) * dx;
  const double ay1 = (1 * c->ny + 4 - c->absorb2) * dx;
  const double az1 = (c->nz + 4 - c->absorb2) * dx;
  const double d3x = (c->nx + 4) * dx, d3y = (c->ny + 4) * dx, d3z = (c->nz + 4) * dx;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    for (long i = 0; i < sp->n; ++i) {
      double *p = sp->r + 7 * i;
      int bal = p[0] < ax0 || p[0] > ax1 || p[1] < ay0 || p[1] > ay1 || p[2] < az0 || p[2] > az1;
      if (!bal && !(p[0] >= 0. && p[1] >= 0. && p[2] >= 0. && stencil_in_array(c, p))) {
        g_oob++;  /* the gather would read outside the array: counted, pushed ballistically */
        bal = 1;
      }
      if (bal) {
        p[0] += p[3] * dth; p[1] += p[4] * dth; p[2] += p[5] * dth;
      } else {
        cal_track4(c, p, s == 0 ? c->mi : -c->me);
      }
      if (p[0] < d3x && p[0] >= 0. && p[1] < d3y && p[1] >= 0. && p[2] < d3z && p[2] >= 0.) {
        if (stencil_in_array(c, p)) {
          if (s == 0) deposit_j(c, p, G_JIX, G_JIY, G_JIZ);
          else deposit_j(c, p, G_JEX, G_JEY, G_JEZ);
        } else {
          g_oob++;
        }
      }
    }
  }
}

/* Drift + density loop of fdtd, :818-867. */
void or_drift_n(or_ctx *c)
{
  const double dx = c->dx, dth = c->dt * 0.5;
  const double d3x = (c->nx + 4) * dx, d3y = (c->ny + 4) * dx, d3z = (c->nz + 4) * dx;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    for (long i = 0; i < sp->n; ++i) {
      double *p = sp->r + 7 * i;
      p[0] += p[3] * dth; p[1] += p[4] * dth; p[2] += p[5] * dth;
      if (p[0] < d3x && p[0] >= 0. && p[1] < d3y && p[1] >= 0. && p[2] < d3z && p[2] >= 0.) {
        if (stencil_in_array(c, p)) deposit_n(c, p, s == 0 ? G_NI : G_NE);
        else g_oob++;
      }
    }
  }
}

/* sr_particle at size 1 (:2041-2531): z outside [2dx, (Nz+2)dx) is removed;
 * x >= (Nx+2)dx wraps by -Nx dx (sent to itself), x < 2dx is removed (the
 * backward packet is zeroed on rank 0, :2138-2142); then the same for y.
 * Survivors keep their order; wrapped particles move to the end of the list
 * (x crossers first, then y crossers), as sr_particle_x/_y append them. */
void or_sr_particle(or_ctx *c)
{
  const double dx = c->dx;
  const double dx2 = 2. * dx, gx2 = (c->nx + 2) * dx, gy2 = (c->ny + 2) * dx, gz2 = (c->nz + 2) * dx;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    for (int axis = 0; axis < 2; ++axis) {
      const double g2 = axis == 0 ? gx2 : gy2;
      const double shift = (axis == 0 ? c->nx : c->ny) * dx;
      long n0 = sp->n;
      unsigned char *dead = (unsigned char *)calloc((size_t)(n0 > 0 ? n0 : 1), 1);
      long nw = 0;
      double *wr = (double *)malloc(sizeof(double) * 7 * (n0 > 0 ? n0 : 1));
      int *wf = (int *)malloc(sizeof(int) * (n0 > 0 ? n0 : 1));
      for (long i = 0; i < n0; ++i) {
        double *p = sp->r + 7 * i;
        if (p[2] < gz2 && p[2] >= dx2) {
          if (p[axis] >= g2) {
            memcpy(wr + 7 * nw, p, sizeof(double) * 7);
            wr[7 * nw + axis] = p[axis] - shift;
            wf[nw++] = sp->flag[i];
            dead[i] = 1;
          } else if (p[axis] < dx2) {
            dead[i] = 1;
          }
        } else {
          dead[i] = 1;
        }
      }
      sp_compact(sp, dead);
      for (long j = 0; j < nw; ++j)
        sp_push(sp, wr[7 * j], wr[7 * j + 1], wr[7 * j + 2], wr[7 * j + 3], wr[7 * j + 4],
                wr[7 * j + 5], wr[7 * j + 6], wf[j]);
      free(dead); free(wr); free(wf);
    }
  }
}

/* sorting, :7475-7590: list re-threaded in cell order (k, l, m of the interior,
 * m fastest), stable within a cell; particles outside the interior dropped. */
void or_sort(or_ctx *c)
{
  const double dx = c->dx;
  const int Nx = c->nx, Ny = c->ny, Nz = c->nz;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    const long nc = (long)Nx * Ny * Nz;
    long *cnt = (long *)calloc((size_t)nc + 1, sizeof(long));
    long *key = (long *)malloc(sizeof(long) * (sp->n > 0 ? sp->n : 1));
    for (long i = 0; i < sp->n; ++i) {
      const double *p = sp->r + 7 * i;
      const int k = (int)(p[0] / dx) - 2, l = (int)(p[1] / dx) - 2, m = (int)(p[2] / dx) - 2;
      if (k >= 0 && k < Nx && l >= 0 && l < Ny && m >= 0 && m < Nz) {
        key[i] = ((long)k * Ny + l) * Nz + m;
        cnt[key[i] + 1]++;
      } else {
        key[i] = -1;
      }
    }
    for (long i = 0; i < nc; ++i) cnt[i + 1] += cnt[i];
    const long nout = cnt[nc];
    double *nr = (double *)malloc(sizeof(double) * 7 * (nout > 0 ? nout : 1));
    int *nf = (int *)malloc(sizeof(int) * (nout > 0 ? nout : 1));
    for (long i = 0; i < sp->n; ++i) {
      if (key[i] < 0) continue;
      const long d = cnt[key[i]]++;
      memcpy(nr + 7 * d, sp->r + 7 * i, sizeof(double) * 7);
      nf[d] = sp->flag[i];
    }
    free(sp->r); free(sp->flag);
    sp->r = nr; sp->flag = nf; sp->n = nout; sp->cap = nout > 0 ? nout : 1;
    free(cnt); free(key);
  }
}

/* -------------------------------------------------------- diagnostics */
/* Sums of thrust_f, :4963-5101 (omega_y = omega_z = 0, DIPOLE() compiled
 * out): F[27] then E[6], over all particles of each species. */
void or_thrust(const or_ctx *c, double *out)
{
  double F[27] = {0}, E[6] = {0};
  const double dx = c->dx;
  const int Nx = c->nx, Ny = c->ny, Nz = c->nz;
  for (int k = 2; k < Nx + 2; k++)
    for (int l = 2; l < Ny + 2; l++)
      for (int m = 2; m < Nz + 2; m++)
        if (k - 2 < 1 * Nx * 0.8 && k - 2 > 1 * Nx * 0.2 && l - 2 < 1 * Ny * 0.8 && l - 2 > 1 * Ny * 0.2 &&
            m - 2 < Nz * 0.8 && m - 2 > Nz * 0.2) {
          const double ex = GV(c, k, l, m, G_EX), ey = GV(c, k, l, m, G_EY), ez = GV(c, k, l, m, G_EZ);
          const double bx = GV(c, k, l, m, G_BX), by = GV(c, k, l, m, G_BY), bz = GV(c, k, l, m, G_BZ);
          E[0] += 0.5 * (ex * ex + ey * ey + ez * ez) * c->e0;
          E[1] += 0.5 * (bx * bx + by * by + bz * bz) / c->mu0;
        }
  for (int s = 0; s < 2; ++s) {
    const or_species *sp = &c->sp[s];
    const double sg = s == 0 ? 1.0 : -1.0, ms = s == 0 ? c->mi : c->me;
    const int o1 = s == 0 ? 3 : 9, o2 = s == 0 ? 15 : 21, oe = s == 0 ? 2 : 3;
    for (long i = 0; i < sp->n; ++i) {
      const double *p = sp->r + 7 * i;
      if (!(p[0] < 1 * Nx * dx * 0.8 && p[0] > 1 * Nx * dx * 0.2 && p[1] < 1 * Ny * dx * 0.8 &&
            p[1] > 1 * Ny * dx * 0.2 && p[2] < Nz * dx * 0.8 && p[2] > Nz * dx * 0.2))
        continue;
      double f[6];
      gather(c, p, f);
      const double ex = f[0], ey = f[1], ez = f[2], bx = f[3], by = f[4], bz = f[5];
      F[0] += sg * c->q * (ex + p[4] * bz - p[5] * by) * p[6] * dx * dx * dx;
      F[1] += sg * c->q * (ey + p[5] * bx - p[3] * bz) * p[6] * dx * dx * dx;
      F[2] += sg * c->q * (ez + p[3] * by - p[4] * bx) * p[6] * dx * dx * dx;
      const int flag = sp->flag[i];
      if (flag != 0) {
        const int o = flag > 0 ? o1 : o2;
        F[o + 0] += sg * c->q * ex * p[6] * dx * dx * dx;
        F[o + 1] += sg * c->q * ey * p[6] * dx * dx * dx;
        F[o + 2] += sg * c->q * ez * p[6] * dx * dx * dx;
        F[o + 3] += sg * c->q * (p[4] * bz - p[5] * by) * p[6] * dx * dx * dx;
        F[o + 4] += sg * c->q * (p[5] * bx - p[3] * bz) * p[6] * dx * dx * dx;
        F[o + 5] += sg * c->q * (p[3] * by - p[4] * bx) * p[6] * dx * dx * dx;
        E[flag > 0 ? oe : oe + 2] += 0.5 * ms * p[6] * dx * dx * dx * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
      }
    }
  }
  memcpy(out, F, sizeof(F));
  memcpy(out + 27, E, sizeof(E));
}

/* Gauss-law residual (no reference counterpart; the reference's compiled-out
 * renew_phi3 corrects it): r = div4(E) - q (ni - ne) / e0 at cell centres
 * (k+1/2, l+1/2, m+1/2), k,l,m in [2, N+2), with the 4th-order divergence
 * (27 (E[i+1]-E[i]) - (E[i+2]-E[i-1])) / (24 dx) that pairs with the curl of
 * renew_b4_2 / renew_e4_2. out: [sum r^2, sum (rho/e0)^2, max |r|, cells]. */
void or_gauss_residual(const or_ctx *c, double *out)
{
  double s2 = 0, r2 = 0, mx = 0;
  long n = 0;
  const double inv = 1.0 / (24.0 * c->dx);
  for (int k = 2; k < c->nx + 2; k++)
    for (int l = 2; l < c->ny + 2; l++)
      for (int m = 2; m < c->nz + 2; m++) {
        const double dvx = 27.0 * (GV(c, k + 1, l, m, G_EX) - GV(c, k, l, m, G_EX)) - (GV(c, k + 2, l, m, G_EX) - GV(c, k - 1, l, m, G_EX));
        const double dvy = 27.0 * (GV(c, k, l + 1, m, G_EY) - GV(c, k, l, m, G_EY)) - (GV(c, k, l + 2, m, G_EY) - GV(c, k, l - 1, m, G_EY));
        const double dvz = 27.0 * (GV(c, k, l, m + 1, G_EZ) - GV(c, k, l, m, G_EZ)) - (GV(c, k, l, m + 2, G_EZ) - GV(c, k, l, m - 1, G_EZ));
        const double div = (dvx + dvy + dvz) * inv;
        const double rho = c->q * (GV(c, k, l, m, G_NI) - GV(c, k, l, m, G_NE)) / c->e0;
        const double r = div - rho;
        s2 += r * r;
        r2 += rho * rho;
        if (fabs(r) > mx) mx = fabs(r);
        n++;
      }
  out[0] = s2; out[1] = r2; out[2] = mx; out[3] = (double)n;
}

/* ------------------------------------------------------------ one step */
/* The body of fdtd's loop, :687-949: add_flat when c_add > add_every-1 (the
 * reference: c_add > 4), sorting when c_thrust > sort_every-1 (c_thrust > 499),
 * thrust_fave's sums every step. Output and suspend files are not written. */
void or_step(or_ctx *c, int *c_add, int *c_thrust, int sort_every, int add_every)
{
  or_renew_grid(c);
  if (*c_thrust > sort_every - 1) { *c_thrust = 0; or_sort(c); }
  if (*c_add > add_every - 1) { or_add_flat(c); *c_add = 0; }
  or_renew_b(c);
  or_sr_b(c);
  or_push_j(c);
  or_renew_b(c);
  or_sr_b(c);
  or_drift_n(c);
  or_sr_current2(c);
  or_renew_e(c);
  or_sr_e(c);
  or_sr_particle(c);
  double t[33];
  or_thrust(c, t);
  for (int i = 0; i < 27; ++i) c->fave[i] += t[i] / 500.;
  (*c_add)++;
  (*c_thrust)++;
}

void or_fave(const or_ctx *c, double *out) { memcpy(out, c->fave, sizeof(c->fave)); }

/* fdtd, :627-952: one add_*_flat before the loop, then nsteps loop bodies with
 * the counters starting at zero. */
void or_fdtd(or_ctx *c, int nsteps, int sort_every, int add_every)
{
  int c_add = 0, c_thrust = 0;
  or_add_flat(c);
  for (int i = 0; i < nsteps; ++i) or_step(c, &c_add, &c_thrust, sort_every, add_every);
}
