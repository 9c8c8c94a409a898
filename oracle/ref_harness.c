/*
 * Harness appended to the (define-patched) reference translation unit
 * PIC/3d_pic458_domain.c when the compiled-reference oracle is built by
 * oracle/build_ref.sh. TEST INFRASTRUCTURE ONLY: it is never linked into the
 * product library. It gives ctypes callers access to the reference's global
 * state (grid, sigma, grid_thread, the particle lists) and calls the
 * reference's own functions. Where the reference has no function for a piece
 * of its time step (the particle loops live inline in fdtd()), the loop is
 * restated here statement for statement with the line range it follows.
 *
 * Particle exchange format: rows of 7 doubles (x, y, z, vx, vy, vz, n) plus
 * an int flag per particle, in list order (thread 0 first).
 * Grid exchange format: the reference's Grid struct (18 doubles per node,
 * PIC/3d_pic458_domain.c:115-123), nodes in grid[k][l][m] order.
 */
#include <pthread.h>
#include <unistd.h>

int oracle_steps = 1;

static Particle *h_ion[THREAD_N], *h_ion_start[THREAD_N];
static Particle *h_el[THREAD_N], *h_el_start[THREAD_N];
static int h_have_particles = 0;

/* --- geometry / constants ------------------------------------------------ */
int ref_dims(int *out)
{
  out[0] = Grid_Nx; out[1] = Grid_Ny; out[2] = Grid_Nz; out[3] = Np;
  out[4] = THREAD_N; out[5] = (int)sizeof(Grid); out[6] = (int)sizeof(Particle);
  out[7] = Absorb_grid; out[8] = Absorb_grid2; out[9] = PACK_N;
  return 10;
}

int ref_consts(double *out)
{
  out[0] = q; out[1] = mi; out[2] = me; out[3] = mu0; out[4] = e0; out[5] = kb; out[6] = C;
  out[7] = dx; out[8] = dt; out[9] = V; out[10] = Nall; out[11] = Ti; out[12] = Te;
  out[13] = R; out[14] = I; out[15] = alpha; out[16] = IMF_x; out[17] = IMF_y; out[18] = IMF_z;
  return 19;
}

/* --- running reference code on a large stack ------------------------------
 * sr_particle keeps 4*THREAD_N*PACK_N Particle records on its stack
 * (PIC/3d_pic458_domain.c:2048-2051) and sorting a THREAD_N*Nx*Ny*Nz int array
 * (:7478); both can exceed a default 8 MB thread stack. */
typedef struct { void (*fn)(void *); void *arg; } h_call;
static void *h_tramp(void *p) { h_call *c = (h_call *)p; c->fn(c->arg); return NULL; }
static int h_run(void (*fn)(void *), void *arg)
{
  pthread_attr_t at;
  pthread_t th;
  h_call c = {fn, arg};
  pthread_attr_init(&at);
  pthread_attr_setstacksize(&at, (size_t)1 << 30);
  if (pthread_create(&th, &at, h_tramp, &c) != 0) return -1;
  pthread_join(th, NULL);
  pthread_attr_destroy(&at);
  return 0;
}

/* This process's rank coordinates (myrank_x, myrank_y of main :205-206); 0, 0
 * in a build with PROCESS_Nx = PROCESS_Ny = 1. */
static int h_rx(void) { int r = 0; MPI_Comm_rank(MPI_COMM_WORLD, &r); return r % PROCESS_Nx; }
static int h_ry(void) { int r = 0; MPI_Comm_rank(MPI_COMM_WORLD, &r); return r / PROCESS_Nx; }

/* --- grid access --------------------------------------------------------- */
long ref_grid_nodes(void) { return (long)(Grid_Nx + 4) * (Grid_Ny + 4) * (Grid_Nz + 4); }
void ref_get_grid(double *out) { memcpy(out, grid, sizeof(grid)); }
void ref_set_grid(const double *in) { memcpy(grid, in, sizeof(grid)); }
void ref_get_sigma(double *out) { memcpy(out, sigma, sizeof(sigma)); }
void ref_get_grid_thread(int t, double *out) { memcpy(out, grid_thread[t], sizeof(grid_thread[t])); }

static void h_init_grid(void *a) { (void)a; init_grid(h_rx(), h_ry()); }
int ref_init_grid(void) { return h_run(h_init_grid, NULL); }

/* --- RNG streams: the same seeds as init_particle_flat (:437-446) -------- */
void ref_init_rng(void)
{
  int i;
  for (i = 0; i < THREAD_N; i++) {
    if (!rnd_p[i]) rnd_p[i] = gsl_rng_alloc(gsl_rng_rand);
    if (!rnd_v[i]) rnd_v[i] = gsl_rng_alloc(gsl_rng_rand);
    if (!rnd_i[i]) rnd_i[i] = gsl_rng_alloc(gsl_rng_rand);
    gsl_rng_set(rnd_p[i], (h_ry() * PROCESS_Nx + h_rx()) * 10000 + i * 100);
    gsl_rng_set(rnd_v[i], (h_ry() * PROCESS_Nx + h_rx()) * 10000 + i * 100 + 50);
    gsl_rng_set(rnd_i[i], i * 10);
    particle_flag[i] = 1;
  }
}

/* which: 0 = position stream, 1 = velocity stream; get when set < 0 */
long long ref_rng_counter(int thread, int which, long long set)
{
  gsl_rng *r = which == 0 ? rnd_p[thread] : rnd_v[thread];
  if (!r) return -1;
  if (set >= 0) r->counter = (uint64_t)set;
  return (long long)r->counter;
}

/* --- particle lists ------------------------------------------------------ */
static void h_free_list(Particle *start)
{
  while (start) {
    Particle *n = start->next_particle;
    free(start);
    start = n;
  }
}

static void h_free_all(void)
{
  int i;
  if (!h_have_particles) return;
  for (i = 0; i < THREAD_N; i++) {
    h_free_list(h_ion_start[i]);
    h_free_list(h_el_start[i]);
    h_ion[i] = h_ion_start[i] = h_el[i] = h_el_start[i] = NULL;
  }
  h_have_particles = 0;
}

static void h_init_particles(void *a) { (void)a; init_particle_flat(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry()); }
int ref_init_particle_flat(void)
{
  h_free_all();
  h_run(h_init_particles, NULL);
  h_have_particles = 1;
  return 0;
}

/* Builds thread t's list from rows; every list must hold at least one node. */
static Particle *h_build(const double *rows, const int *flag, long n)
{
  Particle *start = NULL, *prev = NULL;
  long j;
  for (j = 0; j < n; j++) {
    Particle *p = (Particle *)malloc(sizeof(Particle));
    p->x = rows[7 * j + 0]; p->y = rows[7 * j + 1]; p->z = rows[7 * j + 2];
    p->vx = rows[7 * j + 3]; p->vy = rows[7 * j + 4]; p->vz = rows[7 * j + 5];
    p->n = rows[7 * j + 6];
    p->flag = flag ? flag[j] : 1;
    p->prev_particle = prev;
    p->next_particle = NULL;
    if (prev) prev->next_particle = p; else start = p;
    prev = p;
  }
  return start;
}

/* counts[t] rows for thread t, rows concatenated thread by thread. */
int ref_set_particles(const double *ion_rows, const int *ion_flag, const long *ion_counts,
                      const double *el_rows, const int *el_flag, const long *el_counts)
{
  int i;
  long oi = 0, oe = 0;
  h_free_all();
  for (i = 0; i < THREAD_N; i++) {
    if (ion_counts[i] < 1 || el_counts[i] < 1) return -1;
    h_ion_start[i] = h_ion[i] = h_build(ion_rows + 7 * oi, ion_flag ? ion_flag + oi : NULL, ion_counts[i]);
    h_el_start[i] = h_el[i] = h_build(el_rows + 7 * oe, el_flag ? el_flag + oe : NULL, el_counts[i]);
    oi += ion_counts[i];
    oe += el_counts[i];
  }
  h_have_particles = 1;
  return 0;
}

long ref_count(int species)
{
  int i;
  long n = 0;
  for (i = 0; i < THREAD_N; i++) {
    Particle *p = species == 0 ? h_ion_start[i] : h_el_start[i];
    for (; p; p = p->next_particle) n++;
  }
  return n;
}

long ref_get_particles(int species, double *rows, int *flag, long cap)
{
  int i;
  long n = 0;
  for (i = 0; i < THREAD_N; i++) {
    Particle *p = species == 0 ? h_ion_start[i] : h_el_start[i];
    for (; p; p = p->next_particle) {
      if (n < cap) {
        rows[7 * n + 0] = p->x; rows[7 * n + 1] = p->y; rows[7 * n + 2] = p->z;
        rows[7 * n + 3] = p->vx; rows[7 * n + 4] = p->vy; rows[7 * n + 5] = p->vz;
        rows[7 * n + 6] = p->n;
        if (flag) flag[n] = p->flag;
      }
      n++;
    }
  }
  return n;
}

/* --- pieces of one fdtd() iteration -------------------------------------- */

/* Push + J deposit loop, restated from fdtd PIC/3d_pic458_domain.c:731-812. */
static void h_push_j_list(Particle *start, int thread, int electron)
{
  const int rx = h_rx(), ry = h_ry();
  const double ax0 = Absorb_grid2 * dx - rx * Grid_Nx * dx, ay0 = Absorb_grid2 * dx - ry * Grid_Ny * dx;
  const double az0 = Absorb_grid2 * dx;
  const double ax1 = (PROCESS_Nx * Grid_Nx + 4 - Absorb_grid2) * dx - rx * Grid_Nx * dx;
  const double ay1 = (PROCESS_Ny * Grid_Ny + 4 - Absorb_grid2) * dx - ry * Grid_Ny * dx;
  const double az1 = (Grid_Nz + 4 - Absorb_grid2) * dx;
  const double d3x = (Grid_Nx + 4) * dx, d3y = (Grid_Ny + 4) * dx, d3z = (Grid_Nz + 4) * dx;
  const double dx0 = 0.;
  const double dth = dt * 0.5;
  Particle *p;
  for (p = start; p; p = p->next_particle) {
    if (p->x < ax0 || p->x > ax1 || p->y < ay0 || p->y > ay1 || p->z < az0 || p->z > az1) {
      p->x += p->vx * dth;
      p->y += p->vy * dth;
      p->z += p->vz * dth;
    } else {
      cal_track4(p, electron ? -me : mi, h_rx(), h_ry());
    }
    if (p->x < d3x && p->x >= dx0 && p->y < d3y && p->y >= dx0 && p->z < d3z && p->z >= dx0) {
      if (electron) shape_func_electron0_j_2(p, thread);
      else shape_func_ion0_j_2(p, thread);
    }
  }
}

/* Drift + density deposit loop, restated from fdtd :818-867. */
static void h_drift_n_list(Particle *start, int thread, int electron)
{
  const double d3x = (Grid_Nx + 4) * dx, d3y = (Grid_Ny + 4) * dx, d3z = (Grid_Nz + 4) * dx;
  const double dx0 = 0.;
  const double dth = dt * 0.5;
  Particle *p;
  for (p = start; p; p = p->next_particle) {
    p->x += p->vx * dth;
    p->y += p->vy * dth;
    p->z += p->vz * dth;
    if (p->x < d3x && p->x >= dx0 && p->y < d3y && p->y >= dx0 && p->z < d3z && p->z >= dx0) {
      if (electron) shape_func_electron0_n_2(p, thread);
      else shape_func_ion0_n_2(p, thread);
    }
  }
}

/* Thread-accumulator reduction, restated from fdtd :869-886 (parallel over k,
 * as there, when built with OpenMP). */
static void h_reduce_threads(void)
{
  int i, k, l, m;
  for (i = 0; i < THREAD_N; i++)
#pragma omp parallel for private(l, m)
    for (k = 0; k < Grid_Nx + 4; k++)
      for (l = 0; l < Grid_Ny + 4; l++)
        for (m = 0; m < Grid_Nz + 4; m++) {
          grid[k][l][m].jix0 += grid_thread[i][k][l][m].jix0;
          grid[k][l][m].jiy0 += grid_thread[i][k][l][m].jiy0;
          grid[k][l][m].jiz0 += grid_thread[i][k][l][m].jiz0;
          grid[k][l][m].jex0 += grid_thread[i][k][l][m].jex0;
          grid[k][l][m].jey0 += grid_thread[i][k][l][m].jey0;
          grid[k][l][m].jez0 += grid_thread[i][k][l][m].jez0;
          grid[k][l][m].ni += grid_thread[i][k][l][m].ni;
          grid[k][l][m].ne += grid_thread[i][k][l][m].ne;
        }
}

enum {
  REF_RENEW_GRID = 1, REF_RENEW_B = 2, REF_SR_B = 3, REF_PUSH_J = 4, REF_DRIFT_N = 5,
  REF_REDUCE = 6, REF_SR_CURRENT = 7, REF_RENEW_E = 8, REF_SR_E = 9, REF_SR_PARTICLE = 10,
  REF_ADD_FLAT = 11, REF_SORT = 12, REF_THRUST_F = 13, REF_FDTD = 14
};

/* Thrust/energy sums restated from thrust_f PIC/3d_pic458_domain.c:4963-5101 at
 * full precision (the reference prints them with %.3E). It uses the reference's
 * own shape_func_v2 gather; omega_y = omega_z = 0 on this path so the frame
 * velocity terms Vo* vanish, and the DIPOLE() block is compiled out (:108).
 * Like the reference's loops (while p->next_particle != NULL) the last node of
 * each list is not visited unless include_tail is set. F[27] then E[6]. */
void ref_thrust_sums(double *out, int include_tail)
{
  int i, k, l, m, s;
  double F[27], E[6];
  const int rx = h_rx(), ry = h_ry();  /* this rank's part of the sums (thrust_f :4971, :4984) */
  for (i = 0; i < 27; i++) F[i] = 0.;
  for (i = 0; i < 6; i++) E[i] = 0.;
  for (k = 2; k < Grid_Nx + 2; k++)
    for (l = 2; l < Grid_Ny + 2; l++)
      for (m = 2; m < Grid_Nz + 2; m++)
        if (rx * Grid_Nx + k - 2 < PROCESS_Nx * Grid_Nx * 0.8 && rx * Grid_Nx + k - 2 > PROCESS_Nx * Grid_Nx * 0.2 &&
            ry * Grid_Ny + l - 2 < PROCESS_Ny * Grid_Ny * 0.8 && ry * Grid_Ny + l - 2 > PROCESS_Ny * Grid_Ny * 0.2 &&
            m - 2 < Grid_Nz * 0.8 && m - 2 > Grid_Nz * 0.2) {
          E[0] += 0.5 * (grid[k][l][m].ex * grid[k][l][m].ex + grid[k][l][m].ey * grid[k][l][m].ey + grid[k][l][m].ez * grid[k][l][m].ez) * e0;
          E[1] += 0.5 * (grid[k][l][m].bx * grid[k][l][m].bx + grid[k][l][m].by * grid[k][l][m].by + grid[k][l][m].bz * grid[k][l][m].bz) / mu0;
        }
  for (s = 0; s < 2; s++) {
    const double sg = s == 0 ? 1.0 : -1.0;
    const double ms = s == 0 ? mi : me;
    const int o1 = s == 0 ? 3 : 9, o2 = s == 0 ? 15 : 21, oe = s == 0 ? 2 : 3;
    for (i = 0; i < THREAD_N; i++) {
      Particle *p = s == 0 ? h_ion_start[i] : h_el_start[i];
      for (; p && (include_tail || p->next_particle != NULL); p = p->next_particle) {
        double ex, ey, ez, bx, by, bz;
        if (!(rx * Grid_Nx * dx + p->x < PROCESS_Nx * Grid_Nx * dx * 0.8 &&
              rx * Grid_Nx * dx + p->x > PROCESS_Nx * Grid_Nx * dx * 0.2 &&
              ry * Grid_Ny * dx + p->y < PROCESS_Ny * Grid_Ny * dx * 0.8 &&
              ry * Grid_Ny * dx + p->y > PROCESS_Ny * Grid_Ny * dx * 0.2 &&
              p->z < Grid_Nz * dx * 0.8 && p->z > Grid_Nz * dx * 0.2)) continue;
        shape_func_v2(p, &ex, &ey, &ez, &bx, &by, &bz);
        F[0] += sg * q * (ex + p->vy * bz - p->vz * by) * p->n * dx * dx * dx;
        F[1] += sg * q * (ey + p->vz * bx - p->vx * bz) * p->n * dx * dx * dx;
        F[2] += sg * q * (ez + p->vx * by - p->vy * bx) * p->n * dx * dx * dx;
        if (p->flag != 0) {
          const int o = p->flag > 0 ? o1 : o2;
          F[o + 0] += sg * q * ex * p->n * dx * dx * dx;
          F[o + 1] += sg * q * ey * p->n * dx * dx * dx;
          F[o + 2] += sg * q * ez * p->n * dx * dx * dx;
          F[o + 3] += sg * q * (p->vy * bz - p->vz * by) * p->n * dx * dx * dx;
          F[o + 4] += sg * q * (p->vz * bx - p->vx * bz) * p->n * dx * dx * dx;
          F[o + 5] += sg * q * (p->vx * by - p->vy * bx) * p->n * dx * dx * dx;
          E[p->flag > 0 ? oe : oe + 2] += 0.5 * ms * p->n * dx * dx * dx * (p->vx * p->vx + p->vy * p->vy + p->vz * p->vz);
        }
      }
    }
  }
  memcpy(out, F, sizeof(F));
  memcpy(out + 27, E, sizeof(E));
}

/* One field-gather of shape_func_v2 (:3017-3326) at an arbitrary position. */
void ref_gather(const double *xyz, double *out6)
{
  Particle p;
  memset(&p, 0, sizeof(p));
  p.x = xyz[0]; p.y = xyz[1]; p.z = xyz[2];
  shape_func_v2(&p, &out6[0], &out6[1], &out6[2], &out6[3], &out6[4], &out6[5]);
}

static void h_op(void *arg)
{
  const int op = *(int *)arg;
  int i;
  switch (op) {
  case REF_RENEW_GRID: renew_grid(); break;
  case REF_RENEW_B: renew_b4_2(); break;
  case REF_SR_B: sr_b(h_rx(), h_ry()); break;
  case REF_PUSH_J:
    for (i = 0; i < THREAD_N; i++) {
      h_push_j_list(h_ion_start[i], i, 0);
      h_push_j_list(h_el_start[i], i, 1);
    }
    break;
  case REF_DRIFT_N:
    for (i = 0; i < THREAD_N; i++) {
      h_drift_n_list(h_ion_start[i], i, 0);
      h_drift_n_list(h_el_start[i], i, 1);
    }
    break;
  case REF_REDUCE: h_reduce_threads(); break;
  case REF_SR_CURRENT: sr_current2(h_rx(), h_ry()); break;
  case REF_RENEW_E: renew_e4_2(); break;
  case REF_SR_E: sr_e(h_rx(), h_ry()); break;
  case REF_SR_PARTICLE: sr_particle(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry()); break;
  case REF_ADD_FLAT:
    add_ion_flat(h_ion, h_ion_start, h_rx(), h_ry());
    add_electron_flat(h_el, h_el_start, h_rx(), h_ry());
    break;
  case REF_SORT:
    sorting(h_ion, h_ion_start);
    sorting(h_el, h_el_start);
    break;
  case REF_THRUST_F:
    thrust_f(h_rx(), h_ry(), 0, h_ion, h_ion_start, h_el, h_el_start);
    break;
  case REF_FDTD:
    fdtd(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry(), 0);
    break;
  default: break;
  }
}

int ref_op(int op) { return h_run(h_op, &op); }

/* Runs the reference's own fdtd() (PIC/3d_pic458_domain.c:627-952) for n steps:
 * add_*_flat once before the loop, then the full loop body, with its file
 * output (fdtd/thrust/suspend files) written to the current directory. */
int ref_fdtd(int nsteps)
{
  int op = REF_FDTD;
  oracle_steps = nsteps;
  return h_run(h_op, &op);
}

/* The body of fdtd's loop (:688-911) repeated nsteps times with its step
 * counters kept between calls: sorting every sort_every steps, add_*_flat every
 * add_every steps, then the push, field and exchange functions in fdtd's order.
 * The file output of :913-931 (output, thrust_f, thrust_fave, suspend_job) is
 * left out so that a timing measures the step itself. */
static int h_c_add = 0, h_c_thrust = 0;
static int h_loop_args[3];
static void h_loop(void *a)
{
  int s, i;
  (void)a;
  for (s = 0; s < h_loop_args[0]; s++) {
    renew_grid();
    if (h_c_thrust > h_loop_args[1] - 1) {
      h_c_thrust = 0;
      sorting(h_ion, h_ion_start);
      sorting(h_el, h_el_start);
    }
    if (h_c_add > h_loop_args[2] - 1) {
      add_ion_flat(h_ion, h_ion_start, h_rx(), h_ry());
      add_electron_flat(h_el, h_el_start, h_rx(), h_ry());
      h_c_add = 0;
    }
    renew_b4_2();
    sr_b(h_rx(), h_ry());
    /* one list per thread, as fdtd's parallel loops (:731, :818) */
#pragma omp parallel for num_threads(active_thread)
    for (i = 0; i < THREAD_N; i++) {
      h_push_j_list(h_ion_start[i], i, 0);
      h_push_j_list(h_el_start[i], i, 1);
    }
    renew_b4_2();
    sr_b(h_rx(), h_ry());
#pragma omp parallel for num_threads(active_thread)
    for (i = 0; i < THREAD_N; i++) {
      h_drift_n_list(h_ion_start[i], i, 0);
      h_drift_n_list(h_el_start[i], i, 1);
    }
    h_reduce_threads();
    sr_current2(h_rx(), h_ry());
    renew_e4_2();
    sr_e(h_rx(), h_ry());
    sr_particle(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry());
    h_c_add++;
    h_c_thrust++;
  }
}

int ref_loop(int nsteps, int sort_every, int add_every)
{
  h_loop_args[0] = nsteps;
  h_loop_args[1] = sort_every;
  h_loop_args[2] = add_every;
  return h_run(h_loop, NULL);
}

void ref_fave(double *out) { memcpy(out, Fave, sizeof(Fave)); }

/* Threads of the OpenMP loops (active_thread, :110, and the default team
 * size, as main_func's omp_set_num_threads(active_thread) :214 sets it);
 * returns THREAD_N, the number of particle lists. Without OpenMP every loop
 * runs on the calling thread. */
int ref_set_threads(int n)
{
  active_thread = n;
#ifdef _OPENMP
  omp_set_num_threads(n);
#endif
  return THREAD_N;
}
int ref_unmatched_sends(void) { return oracle_mpi_unmatched(); }

/* --- the reference's own file writers and reader ----------------------- */
/* suspend_job (:7629-7674) and continue_job (:7676-7911) in the working
 * directory, on the harness's particle lists. */
static void h_suspend(void *a) { (void)a; suspend_job(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry()); }
int ref_suspend(void) { return h_run(h_suspend, NULL); }
static void h_continue(void *a)
{
  (void)a;
  continue_job(h_ion, h_ion_start, h_el, h_el_start, h_rx(), h_ry());
}
int ref_continue(void)
{
  h_free_all();
  int rc = h_run(h_continue, NULL);
  h_have_particles = 1;
  return rc;
}
/* output (:4834-4883): fdtd458-0-0-<c>.dat in the working directory. */
static int h_output_c;
static void h_output(void *a) { (void)a; output(h_rx(), h_ry(), h_output_c); }
int ref_output(int c) { h_output_c = c; return h_run(h_output, NULL); }

/* renew_phi3 (:8315-8665), sr_phi (:1389-1574) and sr_e, as fdtd runs them
 * after renew_e4_2 when the PHI blocks are compiled in (:901-907). */
static void h_renew_phi3(void *a)
{
  (void)a;
#if ORACLE_PHI
  renew_phi3(h_rx(), h_ry());
  sr_phi(h_rx(), h_ry());
  sr_e(h_rx(), h_ry());
#endif
}
int ref_renew_phi3(void)
{
#if ORACLE_PHI
  return h_run(h_renew_phi3, NULL);
#else
  return -1;
#endif
}
