/*
 * tangent.c -- FP64 tangent-linear (forward-mode derivative) of the oracle's
 * time step, for checking the GPU adjoint. TEST INFRASTRUCTURE ONLY, like the
 * rest of oracle/.
 *
 * It is compiled as one translation unit with the restatement (included
 * below), whose step functions it reuses:
 *  - the field updates renew_b4_2 / renew_e4_2 (:2580-2652), the ghost copies
 *    sr_b / sr_e (:1001-1387) and the fold sr_current2 (:1805-2039) are affine
 *    in (E, B, B0, J) with coefficients that depend only on sigma, so running
 *    them on a shadow grid that holds the tangents (dE, dB, dB0, dJ) gives the
 *    tangent fields exactly;
 *  - the particle loops (cal_track4 :2804-2870 with shape_func_v2 :3017-3326,
 *    the J deposit :3397-3553, the drift :818-867, sr_particle :2041-2531 and
 *    add_*_flat :5993-6818) are restated here in dual numbers (value, tangent).
 *
 * Parameters: the coil current I (the dipole moment is mu0 I pi R^2, so the
 * dipole part of B0 is proportional to I) and the drift V (every particle that
 * init_particle_flat and add_*_flat create gets vz = V + thermal, :7981).
 * Seeds apply to the state right after init_grid, init_particle_flat and the
 * first add_*_flat, where E = 0 and B = B0.
 *
 * Objective: the impulse along z delivered to the dipole,
 *   J = sum over steps of dt * F,  F = -sum_p s_p q n_p dx^3 (v x B0(x_p))_z
 * over the particles alive after sr_particle (s_p = +1 ions, -1 electrons):
 * the reaction to the Lorentz force of the dipole's own field on the plasma.
 * B0 is gathered with the shape functions of B.
 *
 * Sorting is skipped in the tangent run: it only reorders the particles.
 */
#include "pic_oracle.c"

typedef struct {
  double v, d;
} dual;

static inline dual dl(double v, double d) { dual r = {v, d}; return r; }
static inline dual dadd(dual a, dual b) { return dl(a.v + b.v, a.d + b.d); }
static inline dual dsub(dual a, dual b) { return dl(a.v - b.v, a.d - b.d); }
static inline dual dmul(dual a, dual b) { return dl(a.v * b.v, a.d * b.v + a.v * b.d); }
static inline dual dscl(dual a, double s) { return dl(a.v * s, a.d * s); }
static inline dual ddiv(dual a, dual b) { return dl(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
static inline dual dsqrt(dual a) { const double s = sqrt(a.v); return dl(s, a.d / (2. * s)); }

typedef struct {
  or_ctx *sh;        /* shadow context: its grid holds the tangent fields */
  double *tp[2];     /* per species: dx dy dz dvx dvy dvz of each particle row */
  long tcap[2];
  double dI, dV;     /* seed direction */
  double J, dJ;      /* objective and its tangent */
} or_tl;

static void tl_reserve(or_tl *t, int s, long n)
{
  if (n <= t->tcap[s]) return;
  long cap = t->tcap[s] ? t->tcap[s] : 1024;
  while (cap < n) cap *= 2;
  t->tp[s] = (double *)realloc(t->tp[s], sizeof(double) * 6 * cap);
  t->tcap[s] = cap;
}

/* Seeds the tangent of the current (initial) state for the direction (dI, dV). */
or_tl *or_tl_create(or_ctx *c, const double *params, double dI, double dV)
{
  or_tl *t = (or_tl *)calloc(1, sizeof(or_tl));
  t->sh = or_create(params);
  memcpy(t->sh->sigma, c->sigma, sizeof(double) * 8 * or_grid_nodes(c));
  t->dI = dI;
  t->dV = dV;
  const long nn = or_grid_nodes(c);
  const double imf[3] = {c->imfx, c->imfy, c->imfz};
  for (long i = 0; i < nn; ++i)
    for (int q = 0; q < 3; ++q) {
      const double db0 = c->I != 0. ? (c->g[i * NF + G_B0X + q] - imf[q]) / c->I * dI : 0.;
      t->sh->g[i * NF + G_B0X + q] = db0;
      t->sh->g[i * NF + G_BX + q] = db0;
    }
  for (int s = 0; s < 2; ++s) {
    tl_reserve(t, s, c->sp[s].n + 1);
    for (long i = 0; i < c->sp[s].n; ++i) {
      double *d = t->tp[s] + 6 * i;
      d[0] = d[1] = d[2] = d[3] = d[4] = 0.;
      d[5] = dV;
    }
  }
  return t;
}

void or_tl_destroy(or_tl *t)
{
  if (!t) return;
  or_destroy(t->sh);
  free(t->tp[0]);
  free(t->tp[1]);
  free(t);
}

void or_tl_result(const or_tl *t, double *out2) { out2[0] = t->J; out2[1] = t->dJ; }

/* Removes the tangent rows whose mask byte is set, as sp_compact removes rows. */
static void tl_compact(or_tl *t, int s, long n, const unsigned char *dead)
{
  long w = 0;
  for (long i = 0; i < n; ++i) {
    if (dead[i]) continue;
    if (w != i) memcpy(t->tp[s] + 6 * w, t->tp[s] + 6 * i, sizeof(double) * 6);
    w++;
  }
}

/* add_*_flat with tangents: the shell rows go, the refill rows get (0, dV). */
static void tl_add_flat(or_ctx *c, or_tl *t)
{
  const double dx = c->dx;
  long kept[2];
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    unsigned char *dead = (unsigned char *)calloc((size_t)(sp->n > 0 ? sp->n : 1), 1);
    long nk = 0;
    for (long i = 0; i < sp->n; ++i) {
      const double *r = sp->r + 7 * i;
      if (r[0] < 4 * dx || r[0] > c->nx * dx || r[1] < 4 * dx || r[1] > c->ny * dx ||
          r[2] < 4 * dx || r[2] > c->nz * dx)
        dead[i] = 1;
      else
        nk++;
    }
    tl_compact(t, s, sp->n, dead);
    kept[s] = nk;
    free(dead);
  }
  or_add_flat(c);
  for (int s = 0; s < 2; ++s) {
    tl_reserve(t, s, c->sp[s].n + 1);
    for (long i = kept[s]; i < c->sp[s].n; ++i) {
      double *d = t->tp[s] + 6 * i;
      d[0] = d[1] = d[2] = d[3] = d[4] = 0.;
      d[5] = t->dV;
    }
  }
}

/* One staggered component of shape_func_v2 in dual numbers: the value from
 * field f of c, the tangent from field f of the shadow and from the position
 * tangent. sh* = 1 for a half-shifted axis. */
static dual tl_gather1(const or_ctx *c, const or_ctx *sh, const dual *p, int f, int shk, int shl, int shm)
{
  const double dx = c->dx;
  const int k = shk ? (int)(p[0].v / dx - 0.5) : (int)(p[0].v / dx);
  const int l = shl ? (int)(p[1].v / dx - 0.5) : (int)(p[1].v / dx);
  const int m = shm ? (int)(p[2].v / dx - 0.5) : (int)(p[2].v / dx);
  const int kkk = k + 1, lll = l + 1, mmm = m + 1;
  const dual kkkp = dl((shk ? (kkk + 0.5) * dx : kkk * dx) - p[0].v, -p[0].d);
  const dual lllp = dl((shl ? (lll + 0.5) * dx : lll * dx) - p[1].v, -p[1].d);
  const dual mmmp = dl((shm ? (mmm + 0.5) * dx : mmm * dx) - p[2].v, -p[2].d);
  const dual pk = dl(p[0].v - (shk ? (k + 0.5) * dx : k * dx), p[0].d);
  const dual pl = dl(p[1].v - (shl ? (l + 0.5) * dx : l * dx), p[1].d);
  const dual pm = dl(p[2].v - (shm ? (m + 0.5) * dx : m * dx), p[2].d);
#define GD(kk, ll, mm) dl(GV(c, kk, ll, mm, f), GV(sh, kk, ll, mm, f))
  dual a1 = dadd(dmul(GD(k, l, m), dmul(dmul(kkkp, lllp), mmmp)), dmul(GD(k, l, mmm), dmul(dmul(kkkp, lllp), pm)));
  dual a2 = dadd(dmul(GD(k, lll, m), dmul(dmul(kkkp, pl), mmmp)), dmul(GD(k, lll, mmm), dmul(dmul(kkkp, pl), pm)));
  dual a3 = dadd(dmul(GD(kkk, l, m), dmul(dmul(pk, lllp), mmmp)), dmul(GD(kkk, l, mmm), dmul(dmul(pk, lllp), pm)));
  dual a4 = dadd(dmul(GD(kkk, lll, m), dmul(dmul(pk, pl), mmmp)), dmul(GD(kkk, lll, mmm), dmul(dmul(pk, pl), pm)));
#undef GD
  return dscl(dadd(dadd(dadd(a1, a2), a3), a4), 1. / (dx * dx * dx));
}

/* ex ey ez bx by bz at p (shape_func_v2's staggers). */
static void tl_gather(const or_ctx *c, const or_ctx *sh, const dual *p, dual *out)
{
  out[0] = tl_gather1(c, sh, p, G_EX, 0, 1, 1);
  out[1] = tl_gather1(c, sh, p, G_EY, 1, 0, 1);
  out[2] = tl_gather1(c, sh, p, G_EZ, 1, 1, 0);
  out[3] = tl_gather1(c, sh, p, G_BX, 1, 0, 0);
  out[4] = tl_gather1(c, sh, p, G_BY, 0, 1, 0);
  out[5] = tl_gather1(c, sh, p, G_BZ, 0, 0, 1);
}

/* cal_track4 in dual numbers (same operations as the restatement). */
static void tl_track(const or_ctx *c, const or_tl *t, dual *p, double m)
{
  dual f[6];
  tl_gather(c, t->sh, p, f);
  dual ex = f[0], ey = f[1], ez = f[2], bx = f[3], by = f[4], bz = f[5];
  const dual C = dl(c->c, 0.);
  const double T = 0.5 * c->q * c->dt / m;
  ex = dadd(ex, dl(c->V * c->imfy, t->dV * c->imfy));
  ey = dadd(ey, dl(-c->V * c->imfx, -t->dV * c->imfx));
  const dual CC = dmul(C, C);
  dual gamma1 = ddiv(C, dsqrt(dsub(dsub(dsub(CC, dmul(p[3], p[3])), dmul(p[4], p[4])), dmul(p[5], p[5]))));
  if (isnan(gamma1.v)) gamma1 = dl(0., 0.);
  dual ux = dmul(gamma1, p[3]), uy = dmul(gamma1, p[4]), uz = dmul(gamma1, p[5]);
  dual gamma2 = ddiv(C, dsqrt(dadd(dadd(dadd(CC, dmul(ux, ux)), dmul(uy, uy)), dmul(uz, uz))));
  const dual bux = dmul(gamma2, bx), buy = dmul(gamma2, by), buz = dmul(gamma2, bz);
  const dual S = ddiv(dl(2. * T, 0.),
                      dadd(dl(1., 0.), dscl(dadd(dadd(dmul(bux, bux), dmul(buy, buy)), dmul(buz, buz)), T * T)));
  ux = dadd(ux, dscl(ex, T)); uy = dadd(uy, dscl(ey, T)); uz = dadd(uz, dscl(ez, T));
  const dual uox = dadd(ux, dscl(dsub(dmul(uy, buz), dmul(uz, buy)), T));
  const dual uoy = dadd(uy, dscl(dsub(dmul(uz, bux), dmul(ux, buz)), T));
  const dual uoz = dadd(uz, dscl(dsub(dmul(ux, buy), dmul(uy, bux)), T));
  dual upx = dadd(ux, dmul(S, dsub(dmul(uoy, buz), dmul(uoz, buy))));
  dual upy = dadd(uy, dmul(S, dsub(dmul(uoz, bux), dmul(uox, buz))));
  dual upz = dadd(uz, dmul(S, dsub(dmul(uox, buy), dmul(uoy, bux))));
  upx = dadd(upx, dscl(ex, T)); upy = dadd(upy, dscl(ey, T)); upz = dadd(upz, dscl(ez, T));
  gamma2 = ddiv(C, dsqrt(dadd(dadd(dadd(CC, dmul(upx, upx)), dmul(upy, upy)), dmul(upz, upz))));
  p[3] = dmul(gamma2, upx); p[4] = dmul(gamma2, upy); p[5] = dmul(gamma2, upz);
  const double dth = c->dt * 0.5;
  p[0] = dadd(p[0], dscl(p[3], dth));
  p[1] = dadd(p[1], dscl(p[4], dth));
  p[2] = dadd(p[2], dscl(p[5], dth));
}

/* One staggered component of the J deposit: value into c, tangent into sh. */
static void tl_deposit1(or_ctx *c, or_ctx *sh, const dual *p, dual val, int f, int shk, int shl, int shm)
{
  const double dx = c->dx;
  const int k = shk ? (int)(p[0].v / dx - 0.5) : (int)(p[0].v / dx);
  const int l = shl ? (int)(p[1].v / dx - 0.5) : (int)(p[1].v / dx);
  const int m = shm ? (int)(p[2].v / dx - 0.5) : (int)(p[2].v / dx);
  const int kkk = k + 1, lll = l + 1, mmm = m + 1;
  const dual kkkp = dl((shk ? (kkk + 0.5) * dx : kkk * dx) - p[0].v, -p[0].d);
  const dual lllp = dl((shl ? (lll + 0.5) * dx : lll * dx) - p[1].v, -p[1].d);
  const dual mmmp = dl((shm ? (mmm + 0.5) * dx : mmm * dx) - p[2].v, -p[2].d);
  const dual pk = dl(p[0].v - (shk ? (k + 0.5) * dx : k * dx), p[0].d);
  const dual pl = dl(p[1].v - (shl ? (l + 0.5) * dx : l * dx), p[1].d);
  const dual pm = dl(p[2].v - (shm ? (m + 0.5) * dx : m * dx), p[2].d);
  const dual tk = dmul(val, kkkp), tp = dmul(val, pk);
#define ADD(kk, ll, mm, w) do { const dual w_ = (w); GV(c, kk, ll, mm, f) += w_.v; GV(sh, kk, ll, mm, f) += w_.d; } while (0)
  ADD(k, l, m, dmul(tk, dmul(lllp, mmmp)));
  ADD(k, l, mmm, dmul(tk, dmul(lllp, pm)));
  ADD(k, lll, m, dmul(tk, dmul(pl, mmmp)));
  ADD(k, lll, mmm, dmul(tk, dmul(pl, pm)));
  ADD(kkk, l, m, dmul(tp, dmul(lllp, mmmp)));
  ADD(kkk, l, mmm, dmul(tp, dmul(lllp, pm)));
  ADD(kkk, lll, m, dmul(tp, dmul(pl, mmmp)));
  ADD(kkk, lll, mmm, dmul(tp, dmul(pl, pm)));
#undef ADD
}

/* The push + J deposit loop (:731-812) with tangents. */
static void tl_push_j(or_ctx *c, or_tl *t)
{
  const double dx = c->dx, dth = c->dt * 0.5;
  const double ax0 = c->absorb2 * dx, ay0 = ax0, az0 = ax0;
  const double ax1 = (c->nx + 4 - c->absorb2) * dx;
  const double ay1 = (c->ny + 4 - c->absorb2) * dx;
  const double az1 = (c->nz + 4 - c->absorb2) * dx;
  const double d3x = (c->nx + 4) * dx, d3y = (c->ny + 4) * dx, d3z = (c->nz + 4) * dx;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    const int fj = s == 0 ? G_JIX : G_JEX;
    for (long i = 0; i < sp->n; ++i) {
      double *r = sp->r + 7 * i;
      double *d = t->tp[s] + 6 * i;
      dual p[6];
      for (int q = 0; q < 6; ++q) p[q] = dl(r[q], d[q]);
      int bal = r[0] < ax0 || r[0] > ax1 || r[1] < ay0 || r[1] > ay1 || r[2] < az0 || r[2] > az1;
      if (!bal && !(r[0] >= 0. && r[1] >= 0. && r[2] >= 0. && stencil_in_array(c, r))) bal = 1;
      if (bal) {
        for (int q = 0; q < 3; ++q) p[q] = dadd(p[q], dscl(p[3 + q], dth));
      } else {
        tl_track(c, t, p, s == 0 ? c->mi : -c->me);
      }
      for (int q = 0; q < 6; ++q) { r[q] = p[q].v; d[q] = p[q].d; }
      if (r[0] < d3x && r[0] >= 0. && r[1] < d3y && r[1] >= 0. && r[2] < d3z && r[2] >= 0. &&
          stencil_in_array(c, r)) {
        const dual qn = dl(c->q * r[6] / (dx * dx * dx), 0.);
        tl_deposit1(c, t->sh, p, dmul(qn, p[3]), fj + 0, 0, 1, 1);
        tl_deposit1(c, t->sh, p, dmul(qn, p[4]), fj + 1, 1, 0, 1);
        tl_deposit1(c, t->sh, p, dmul(qn, p[5]), fj + 2, 1, 1, 0);
      }
    }
  }
}

/* The drift (:818-867) of the tangents; the restatement does the values and
 * the density deposit. */
static void tl_drift(or_ctx *c, or_tl *t)
{
  const double dth = c->dt * 0.5;
  for (int s = 0; s < 2; ++s)
    for (long i = 0; i < c->sp[s].n; ++i) {
      double *d = t->tp[s] + 6 * i;
      d[0] += d[3] * dth; d[1] += d[4] * dth; d[2] += d[5] * dth;
    }
  or_drift_n(c);
}

/* or_sr_particle with the tangent rows moved alongside (a wrap is a shift, so
 * the tangents of a wrapped particle are unchanged). */
static void tl_sr_particle(or_ctx *c, or_tl *t)
{
  const double dx = c->dx;
  const double dx2 = 2. * dx, gx2 = (c->nx + 2) * dx, gy2 = (c->ny + 2) * dx, gz2 = (c->nz + 2) * dx;
  for (int s = 0; s < 2; ++s) {
    or_species *sp = &c->sp[s];
    for (int axis = 0; axis < 2; ++axis) {
      const double g2 = axis == 0 ? gx2 : gy2;
      const double shift = (axis == 0 ? c->nx : c->ny) * dx;
      const long n0 = sp->n;
      unsigned char *dead = (unsigned char *)calloc((size_t)(n0 > 0 ? n0 : 1), 1);
      long nw = 0;
      double *wr = (double *)malloc(sizeof(double) * 7 * (n0 > 0 ? n0 : 1));
      double *wd = (double *)malloc(sizeof(double) * 6 * (n0 > 0 ? n0 : 1));
      int *wf = (int *)malloc(sizeof(int) * (n0 > 0 ? n0 : 1));
      for (long i = 0; i < n0; ++i) {
        double *p = sp->r + 7 * i;
        if (p[2] < gz2 && p[2] >= dx2) {
          if (p[axis] >= g2) {
            memcpy(wr + 7 * nw, p, sizeof(double) * 7);
            memcpy(wd + 6 * nw, t->tp[s] + 6 * i, sizeof(double) * 6);
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
      tl_compact(t, s, n0, dead);
      sp_compact(sp, dead);
      tl_reserve(t, s, sp->n + nw + 1);
      for (long j = 0; j < nw; ++j) {
        memcpy(t->tp[s] + 6 * sp->n, wd + 6 * j, sizeof(double) * 6);
        sp_push(sp, wr[7 * j], wr[7 * j + 1], wr[7 * j + 2], wr[7 * j + 3], wr[7 * j + 4],
                wr[7 * j + 5], wr[7 * j + 6], wf[j]);
      }
      free(dead); free(wr); free(wd); free(wf);
    }
  }
}

/* F = -sum s q n dx^3 (v x B0(x))_z and its tangent. */
static dual tl_objective(const or_ctx *c, const or_tl *t)
{
  const double dx = c->dx, dx3 = dx * dx * dx;
  dual F = dl(0., 0.);
  for (int s = 0; s < 2; ++s) {
    const or_species *sp = &c->sp[s];
    const double sg = s == 0 ? 1.0 : -1.0;
    for (long i = 0; i < sp->n; ++i) {
      const double *r = sp->r + 7 * i;
      const double *d = t->tp[s] + 6 * i;
      dual p[6];
      for (int q = 0; q < 6; ++q) p[q] = dl(r[q], d[q]);
      if (!stencil_in_array(c, r)) continue;
      const dual b0x = tl_gather1(c, t->sh, p, G_B0X, 1, 0, 0);
      const dual b0y = tl_gather1(c, t->sh, p, G_B0Y, 0, 1, 0);
      const dual lz = dsub(dmul(p[3], b0y), dmul(p[4], b0x));
      F = dsub(F, dscl(lz, sg * c->q * r[6] * dx3));
    }
  }
  return F;
}

/* F of the current state (no tangents), for finite differences. */
double or_dipole_force(const or_ctx *c)
{
  const double dx = c->dx, dx3 = dx * dx * dx;
  double F = 0.;
  for (int s = 0; s < 2; ++s) {
    const or_species *sp = &c->sp[s];
    const double sg = s == 0 ? 1.0 : -1.0;
    for (long i = 0; i < sp->n; ++i) {
      const double *r = sp->r + 7 * i;
      if (!stencil_in_array(c, r)) continue;
      dual p[6];
      for (int q = 0; q < 6; ++q) p[q] = dl(r[q], 0.);
      const dual b0x = tl_gather1(c, c, p, G_B0X, 1, 0, 0);
      const dual b0y = tl_gather1(c, c, p, G_B0Y, 0, 1, 0);
      F -= sg * c->q * r[6] * dx3 * (r[3] * b0y.v - r[4] * b0x.v);
    }
  }
  return F;
}

/* The loop body of fdtd (:687-949) without sorting, with tangents, adding
 * dt * F of the new state to the objective. */
void or_tl_step(or_ctx *c, or_tl *t, int *c_add, int add_every)
{
  or_ctx *sh = t->sh;
  or_renew_grid(c);
  or_renew_grid(sh);
  if (*c_add > add_every - 1) { tl_add_flat(c, t); *c_add = 0; }
  or_renew_b(c); or_sr_b(c);
  or_renew_b(sh); or_sr_b(sh);
  tl_push_j(c, t);
  or_renew_b(c); or_sr_b(c);
  or_renew_b(sh); or_sr_b(sh);
  tl_drift(c, t);
  or_sr_current2(c); or_sr_current2(sh);
  or_renew_e(c); or_sr_e(c);
  or_renew_e(sh); or_sr_e(sh);
  tl_sr_particle(c, t);
  const dual F = tl_objective(c, t);
  t->J += c->dt * F.v;
  t->dJ += c->dt * F.d;
  (*c_add)++;
}

/* The same step without tangents (sorting skipped), objective included: the
 * forward run that central differences of the objective use. */
double or_plain_step(or_ctx *c, int *c_add, int add_every)
{
  or_renew_grid(c);
  if (*c_add > add_every - 1) { or_add_flat(c); *c_add = 0; }
  or_renew_b(c); or_sr_b(c);
  or_push_j(c);
  or_renew_b(c); or_sr_b(c);
  or_drift_n(c);
  or_sr_current2(c);
  or_renew_e(c); or_sr_e(c);
  or_sr_particle(c);
  (*c_add)++;
  return c->dt * or_dipole_force(c);
}
