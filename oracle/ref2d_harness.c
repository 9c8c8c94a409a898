/*
 * Harness appended to the define-patched reference translation unit
 * PIC2D/2d_pic278_mpi.c (oracle/ref2d_patch.sed) when oracle/build.py builds
 * the 2D compiled-reference oracle. TEST INFRASTRUCTURE ONLY: it is never
 * linked into the product library.
 *
 * The 2D reference keeps its state in main_func's locals (:201-222) and hands
 * it to every function; the harness owns that state as statics and calls the
 * reference's own functions (init_grid, init_particle, renew_grid, renew_b4,
 * renew_e4, sr_grid, sr_current, sr_density, external_current_perp,
 * renew_phi, add_ion5, add_electron5, sr_particle, del_particle_*,
 * cal_track_c4, shape_func_*, thrust_F). The particle loops that fdtd
 * (:527-1019) writes inline are driven here with fdtd's conditions and calls
 * in fdtd's order; each driver cites the lines it follows. MPI size 1
 * (PROCESS_N = 1, rank 0), one thread list (THREAD_N = 1).
 *
 * Exchange formats: particles as rows (x, z, vx, vy, vz, n) plus an int flag,
 * in list order; the grid as the Grid struct (18 doubles per node, :104-112)
 * in grid[k][m] order.
 */
int oracle_steps = 1;

static Grid hg[Grid_Nx + 4][Grid_Nz + 4];
static double hs[2 * (Grid_Nx + 4)][2 * (Grid_Nz + 4)];
static Grid_thread hgt[THREAD_N][Grid_Nx + 4][Grid_Nz + 4];
static Particle *hion[THREAD_N], *hion0[THREAD_N], *hel[THREAD_N], *hel0[THREAD_N];
static gsl_rng *hrp[THREAD_N], *hrv[THREAD_N];
static Particle hpack_f[THREAD_N][PACK_N], hpack_b[THREAD_N][PACK_N];
static int hcount_f[THREAD_N], hcount_b[THREAD_N];
static int h_add_i, h_add_e, h_c;

int ref2d_dims(int *out)
{
  out[0] = Grid_Nx; out[1] = Grid_Nz; out[2] = Np; out[3] = THREAD_N; out[4] = PROCESS_N;
  out[5] = Absorb_grid; out[6] = Absorb_grid2; out[7] = Absorb_grid3; out[8] = PACK_N;
  out[9] = (int)sizeof(Grid);
  return 10;
}

long ref2d_grid_nodes(void) { return (long)(Grid_Nx + 4) * (Grid_Nz + 4); }
void ref2d_get_grid(double *out) { memcpy(out, hg, sizeof(hg)); }
void ref2d_set_grid(const double *in) { memcpy(hg, in, sizeof(hg)); }
void ref2d_get_sigma(double *out) { memcpy(out, hs, sizeof(hs)); }
int ref2d_step_index(void) { return h_c; }

static Particle **h_list(int s) { return s == 0 ? hion : hel; }
static Particle **h_start(int s) { return s == 0 ? hion0 : hel0; }

long ref2d_count(int s)
{
  long n = 0;
  for (int t = 0; t < THREAD_N; t++)
    for (Particle *p = h_start(s)[t]; p; p = p->next_particle) n++;
  return n;
}

long ref2d_get_particles(int s, double *rows, int *flag, long cap)
{
  long n = 0;
  for (int t = 0; t < THREAD_N; t++)
    for (Particle *p = h_start(s)[t]; p; p = p->next_particle) {
      if (n < cap) {
        double *r = rows + 6 * n;
        r[0] = p->x; r[1] = p->z; r[2] = p->vx; r[3] = p->vy; r[4] = p->vz; r[5] = p->n;
        if (flag) flag[n] = p->flag;
      }
      n++;
    }
  return n;
}

/* Deposit condition of the push, drift and initial density loops
 * (:596, :711, :797): the 2x2 stencil base lies in the array. */
static int h_in_dep(const Particle *p)
{
  return p->x < (Grid_Nx + 3.) * dx && p->x >= dx && p->z < (Grid_Nz + 2.) * dx && p->z >= 2. * dx;
}

/* grid[k][m] += the thread accumulators (:609-616, :743-756, :830-837). */
static void h_reduce(int currents, int densities)
{
  for (int t = 0; t < THREAD_N; t++)
    for (int k = 0; k < Grid_Nx + 4; k++)
      for (int m = 0; m < Grid_Nz + 4; m++) {
        if (currents) {
          hg[k][m].jix0 += hgt[t][k][m].jix0; hg[k][m].jiy0 += hgt[t][k][m].jiy0;
          hg[k][m].jiz0 += hgt[t][k][m].jiz0; hg[k][m].jex0 += hgt[t][k][m].jex0;
          hg[k][m].jey0 += hgt[t][k][m].jey0; hg[k][m].jez0 += hgt[t][k][m].jez0;
        }
        if (densities) {
          hg[k][m].ni += hgt[t][k][m].ni;
          hg[k][m].ne += hgt[t][k][m].ne;
        }
      }
}

/* Density deposit of every particle of both species (:585-607, :778-828). */
static void h_deposit_n(void)
{
  for (int t = 0; t < THREAD_N; t++) {
    for (Particle *p = hion0[t]; p; p = p->next_particle)
      if (h_in_dep(p)) shape_func_ion0_n(p, t, hgt);
    for (Particle *p = hel0[t]; p; p = p->next_particle)
      if (h_in_dep(p)) shape_func_electron0_n(p, t, hgt);
  }
}

/* init_grid, init_particle and fdtd's set-up before its loop (:583-625). */
int ref2d_init(void)
{
  init_grid(hg, hs, 0, 1);
  init_particle(hion, hion0, hel, hel0, hrp, hrv, 0);
  renew_grid(hg, hgt);
  h_deposit_n();
  h_reduce(0, 1);
  sr_density(hg, 0, 1);
  sr_grid(hg, 0, 1);
  renew_phi(hg, 0, 1, 0);
  sr_grid(hg, 0, 1);
  h_add_i = h_add_e = h_c = 0;
  return 0;
}

/* The push loop (:681-741) for one species: ballistic half drift inside the
 * Absorb_grid2 margins, else cal_track_c4; J deposit inside the array. */
static void h_push(int s)
{
  const double m = s == 0 ? mi : -me;
  const double dt0 = s == 0 ? dti : dte;
  for (int t = 0; t < THREAD_N; t++)
    for (Particle *p = h_start(s)[t]; p; p = p->next_particle) {
      if (p->z < Absorb_grid2 * dx || p->z > (Grid_Nz + 4 - Absorb_grid2) * dx || p->x < Absorb_grid2 * dx ||
          p->x > (Grid_Nx + 4 - Absorb_grid2) * dx) {
        p->x += p->vx * dt0 * 0.5;
        p->z += p->vz * dt0 * 0.5;
      } else {
        cal_track_c4(p, &m, &dt0, hg);
      }
      if (h_in_dep(p)) {
        if (s == 0) {
          shape_func_ion0_jy(p, t, hgt); shape_func_ion0_jx(p, t, hgt); shape_func_ion0_jz(p, t, hgt);
        } else {
          shape_func_electron0_jy(p, t, hgt); shape_func_electron0_jx(p, t, hgt); shape_func_electron0_jz(p, t, hgt);
        }
      }
    }
}

/* The drift loop (:762-828) for one species. */
static void h_drift(int s)
{
  const double dt0 = s == 0 ? dti : dte;
  for (int t = 0; t < THREAD_N; t++)
    for (Particle *p = h_start(s)[t]; p; p = p->next_particle) {
      p->x += p->vx * dt0 * 0.5;
      p->z += p->vz * dt0 * 0.5;
      if (h_in_dep(p)) {
        if (s == 0) shape_func_ion0_n(p, t, hgt);
        else shape_func_electron0_n(p, t, hgt);
      }
    }
}

/* The exchange and removal loops (:861-960) for one species at size 1:
 * forward x crossers are packed and sent to this rank (appended shifted by
 * -Nx dx), the backward packet is emptied on rank 0 (:928-932), then the
 * particles outside [2 dx, (N+2) dx) in x or z are deleted. */
static void h_exchange(int s)
{
  Particle **lst = h_list(s), **st = h_start(s);
  for (int t = 0; t < THREAD_N; t++) {
    hcount_f[t] = hcount_b[t] = 0;
    for (Particle *p = st[t]; p; p = p->next_particle) {
      if (p->x < (Grid_Nx + 3.) * dx && p->x >= (Grid_Nx + 2.) * dx && p->z < (Grid_Nz + 2.) * dx && p->z >= 2. * dx)
        hpack_f[t][hcount_f[t]++] = *p;
      else if (p->x > dx && p->x < 2. * dx && p->z < (Grid_Nz + 2.) * dx && p->z >= 2. * dx)
        hpack_b[t][hcount_b[t]++] = *p;
    }
  }
  for (int t = 0; t < THREAD_N; t++) hcount_b[t] = 0;
  sr_particle((const Particle(*)[PACK_N])hpack_f, hcount_f, lst, st, 0, 1, 1);
  sr_particle((const Particle(*)[PACK_N])hpack_b, hcount_b, lst, st, 0, 1, -1);
  for (int t = 0; t < THREAD_N; t++) {
    lst[t] = st[t];
    while (lst[t]->next_particle != NULL) {
      const Particle *p = lst[t];
      if (p->x < 2. * dx || p->x >= (Grid_Nx + 2.) * dx || p->z >= (Grid_Nz + 2.) * dx || p->z < 2. * dx) {
        if (s == 0) del_particle_i(lst, t, st);
        else del_particle_e(lst, t, st);
      }
      lst[t] = lst[t]->next_particle;
    }
    const Particle *p = lst[t];
    if (p->x < 2. * dx || p->x >= (Grid_Nx + 2.) * dx || p->z >= (Grid_Nz + 2.) * dx || p->z < 2. * dx) {
      if (s == 0) del_particle_i(lst, t, st);
      else del_particle_e(lst, t, st);
    }
  }
}

/* One body of fdtd's loop (:627-1015) without file output; the refill runs
 * when its counter passes add_every - 1 (the reference: 249, :645-653). */
int ref2d_step(int add_every)
{
  renew_grid(hg, hgt);
  if (h_add_i > add_every - 1) { add_ion5(hion, hion0, hrp, hrv, 0, 1); h_add_i = 0; }
  if (h_add_e > add_every - 1) { add_electron5(hel, hel0, hrp, hrv, 0, 1); h_add_e = 0; }
  renew_b4(hg, hs);
  sr_grid(hg, 0, 1);
  h_push(0);
  h_push(1);
  h_reduce(1, 0);
  sr_current(hg, 0, 1);
  external_current_perp(hg, h_c, 0, 1);
  renew_b4(hg, hs);
  sr_grid(hg, 0, 1);
  h_drift(0);
  h_drift(1);
  h_reduce(0, 1);
  sr_density(hg, 0, 1);
  renew_e4(hg, hs);
  sr_grid(hg, 0, 1);
  renew_phi(hg, 0, 1, h_c);
  sr_grid(hg, 0, 1);
  h_exchange(0);
  h_exchange(1);
  h_add_i++;
  h_add_e++;
  h_c++;
  return 0;
}

/* thrust_F (:2304-2387): Fx, Fz, My of the current grid (it also appends a
 * line to pic1278-f.txt in the working directory, as the reference does). */
void ref2d_thrust(double *out3)
{
  double Fx, Fz, My;
  thrust_F(hg, 0, 1, &Fx, &Fz, &My);
  out3[0] = Fx; out3[1] = Fz; out3[2] = My;
}

/* The reference's sine transform (NR sinft, :2892-2925) of y[1..n]. */
void ref2d_sinft(int n, double *y1) { sinft(n, y1 - 1); }
