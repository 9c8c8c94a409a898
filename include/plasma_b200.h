/*
 * plasma_b200.h -- C ABI of the B200 (sm_100a) implementation of the 3D
 * particle-in-cell time step of PLASMAsim's PIC/3d_pic458_domain.c.
 *
 * The reference has no library interface: its step is a set of C functions over
 * global arrays, called in order from fdtd() (PIC/3d_pic458_domain.c:627-952),
 * that return 0 and exit() on failure. Each entry point below replaces one of
 * those functions (cited per declaration) for one domain at MPI size 1; the
 * state the reference keeps in globals (grid[][][] :147, sigma[][][] :148,
 * grid_thread :149, the particle lists owned by main_func :258-261) lives in an
 * opaque context instead. Every call returns a status code (PIC_OK == 0) and
 * never exits the process.
 *
 * Threading: one host thread per context at a time. All device work of a
 * context is issued on its own CUDA stream (pic_get_stream); calls return
 * when the work is queued unless they hand results back to host memory.
 *
 * Units are the caller's (the reference uses MKSA; normalized units work the
 * same way); positions are absolute, ghost cells included, as in the reference
 * (interior cell index i covers [i dx, (i+1) dx) for i in [2, N+2)).
 */
#ifndef PLASMA_B200_H
#define PLASMA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PIC_OK 0
#define PIC_ERR_ARG 1        /* invalid argument or configuration */
#define PIC_ERR_CUDA 2       /* a CUDA runtime call failed */
#define PIC_ERR_CAPACITY 3   /* particle capacity exceeded */
#define PIC_ERR_STATE 4      /* call out of order (e.g. step before init) */
#define PIC_ERR_DEVICE 5     /* device-side counters report lost work (pic_status) */
#define PIC_ERR_TOO_LARGE 6  /* input larger than a fixed-size scratch allows */
#define PIC_ERR_COMM 7       /* an exchange between ranks failed (transport error or timeout) */

#define PIC_ION 0
#define PIC_ELECTRON 1
#define PIC_BOTH (-1)

/* Number of doubles in one grid record of pic_get_grid / pic_set_grid: the
 * reference's Grid struct (PIC/3d_pic458_domain.c:115-123) in field order
 * bx by bz b0x b0y b0z ex ey ez jix0 jiy0 jiz0 jex0 jey0 jez0 ni ne phi. */
#define PIC_GRID_RECORD 18
/* Doubles per particle row of pic_set_particles / pic_get_particles:
 * x y z vx vy vz n (the reference's Particle, :134-141, without its links). */
#define PIC_PARTICLE_ROW 7
#define PIC_NUM_THRUST 27    /* F[27] of thrust_f, :4950 */
#define PIC_NUM_ENERGY 6     /* E[6] of thrust_f, :4953 */

/* Run-time form of the reference's compile-time parameters (:52-103). */
typedef struct pic_config {
  int nx, ny, nz;          /* interior cells: Grid_Nx, Grid_Ny, Grid_Nz */
  int np;                  /* macro-particles per cell per species: Np */
  int precision;           /* 32: FP32 particles/fields, FP64 reductions; 64: FP64 throughout */
  int device;              /* CUDA device ordinal */
  double dx, dt;           /* dx, dt */
  double q, mi, me;        /* q, mi, me (the reference: me = mi/100) */
  double mu0, e0, kb, c;   /* mu0, e0, kb, C */
  double v_drift;          /* V: solar-wind drift along +z */
  double n_all;            /* Nall: plasma density; particle weight n = Nall/Np */
  double ti, te;           /* Ti, Te */
  double coil_r, coil_i;   /* R, I: dipole moment I*pi*R^2 */
  double alpha;            /* alpha: moment direction (0, sin a, cos a) */
  double imf_x, imf_y, imf_z; /* IMF_x, IMF_y, IMF_z */
  int absorb_grid;         /* Absorb_grid: width of the field damping layer */
  int absorb_grid2;        /* Absorb_grid2: width of the ballistic particle layer */
  double sigma_a;          /* damping amplitude a of init_grid (:295) */
  double dipole_cutoff;    /* external_current7 radius in cells (:4596, 210) */
  int add_interval;        /* fdtd: add_*_flat every add_interval steps (5, :700) */
  int sort_interval;       /* fdtd: sorting every sort_interval steps (500, :694) */
  int diag_every_step;     /* 1: thrust_fave sums every step as fdtd does (:926) */
  int poisson_clean;       /* 1: renew_phi3 + sr_phi + sr_e after each renew_e4_2 and after the
                              first add_*_flat, as a build with the PHI blocks (:107, :676-681,
                              :901-907); 0: as the reference ships (PHI compiled out) */
  long long capacity;      /* particle slots per species; 0 sizes it for the tiled layout:
                              (1.125 (np + 3 sqrt(np) + 2) + 6) slots per cell + 65536 */
  unsigned long long seed_p; /* position stream key (init_particle_flat :444: 0) */
  unsigned long long seed_v; /* velocity stream key (:445: 50) */
  int absorb_grid3;        /* Absorb_grid3 (:97, 40): cells of each boundary left out of renew_phi3's residual */
  int procs_x, procs_y;    /* PROCESS_Nx, PROCESS_Ny (:100-101): the x-y decomposition, 1 x 1 by default;
                              nx, ny are then the cells of one rank (Grid_Nx, Grid_Ny) */
  int rank_x, rank_y;      /* myrank_x, myrank_y (:205-206) of this context */
  int plain_fields;        /* 0: renew_b4_2 / renew_e4_2 with TMA-staged stencil operands wherever the
                              row pitch (nz + 4 values) is a multiple of 16 bytes; 1: the per-node
                              kernels everywhere (same arithmetic, for comparison) */
  int slot_order;          /* 0 (default): the tiled, cell-sorted particle layout and its sort, two
                              record buffers per species; 1: particles in slot order, never sorted
                              (sorting only reorders, :7475-7590), one record buffer per species: half
                              the particle memory, the one-thread-per-particle push. Refills append
                              and removed particles leave empty slots, so the capacity bounds the
                              number of refills a run can take (the default capacity, 1.8 np per
                              cell, holds about 100 steps of refills). The adjoint needs 0 */
} pic_config;

typedef struct pic_ctx pic_ctx;

/* Domain decomposition (PROCESS_Nx x PROCESS_Ny > 1). Every exchange of the
 * reference's MPI code -- sr_b, sr_e, sr_current2, sr_particle (:1001-2555)
 * and thrust_f's MPI_Allreduce -- goes through a transport that the caller
 * provides; ranks are numbered myrank_y * procs_x + myrank_x, as main() does.
 * All ranks make the same calls in the same order (one host thread per rank).
 *  sendrecv: send `send_bytes` of device memory at `send` to rank `dest` and
 *            receive `recv_bytes` of device memory into `recv` from rank `src`
 *            (a rank may name itself); both ordered on `stream` (the context's
 *            cudaStream_t): the send reads what the stream's earlier work
 *            wrote, later work on the stream sees the received bytes.
 *  allreduce_sum_f64: in-place sum of n doubles in device memory over all
 *            ranks, ordered on `stream`; every rank gets the same bits.
 * Both return 0 on success. */
typedef struct pic_transport {
  void *user;
  int (*sendrecv)(void *user, const void *send, size_t send_bytes, int dest,
                  void *recv, size_t recv_bytes, int src, void *stream);
  int (*allreduce_sum_f64)(void *user, double *buf, int n, void *stream);
} pic_transport;

/* Installs the transport of a context whose configuration has
 * procs_x * procs_y > 1 (or a single-rank context that should exchange
 * through it instead of its in-place wraps); the transport must outlive the
 * context's use of it. */
int pic_set_transport(pic_ctx *ctx, const pic_transport *t);

/* In-process transport: the ranks are contexts of one process, each driven by
 * its own host thread, on one GPU or several; device-to-device copies ordered
 * with CUDA events, rendezvous on the host (a wait that sees no partner for
 * 60 s fails with PIC_ERR_COMM instead of blocking). */
typedef struct pic_group pic_group;
int pic_group_create(int nranks, pic_group **out);
int pic_group_destroy(pic_group *group);
int pic_group_transport(pic_group *group, int rank, pic_transport *out);
/* The host rendezvous limit of the group's exchanges in milliseconds (60 s
 * by default); an exchange whose partner does not arrive within it fails with
 * PIC_ERR_COMM, and the group is unusable afterwards. No reference
 * counterpart: MPI_Sendrecv and MPI_Allreduce (:1001-2531, :5103) block. */
int pic_group_set_timeout(pic_group *group, int ms);

/* NCCL transport: one process (or thread) per GPU. pic_nccl_unique_id fills
 * the 128-byte id on one rank; the caller shares it (e.g. through
 * torch.distributed's store) and every rank calls
 * pic_nccl_transport_create with it. libnccl.so.2 is loaded at run time. */
int pic_nccl_unique_id(unsigned char id[128]);
int pic_nccl_transport_create(const unsigned char id[128], int nranks, int rank, int device,
                              pic_transport *out);
int pic_nccl_transport_destroy(pic_transport *t);

/* Fills *cfg with the reference's own defaults (:52-103) for a one-domain run
 * of nx*ny*nz cells: MKSA constants, dx = 1.5, dt = 1.5e-9, Np = 16, ... */
int pic_config_default(pic_config *cfg, int nx, int ny, int nz);

/* Allocates all device state (replaces the static arrays :147-153 and the
 * particle lists of main_func :258-261). */
int pic_create(const pic_config *cfg, pic_ctx **out);
int pic_destroy(pic_ctx *ctx);

/* init_grid + external_current7 (:291-410, :4579-4634): zero fields, dipole
 * B0 on the staggered points, damping profile. */
int pic_init_grid(pic_ctx *ctx);
/* init_particle_flat (:412-625): Np per cell per species, uniform in the
 * cell, drifting Maxwellian, from the position/velocity random streams. */
int pic_init_particle_flat(pic_ctx *ctx);

/* renew_grid (:2533-2578): zero currents and densities. */
int pic_renew_grid(pic_ctx *ctx);
/* renew_b4_2 (:2580-2611) followed by sr_b (:1001-1193) at size 1. */
int pic_renew_b4_2(pic_ctx *ctx);
/* renew_e4_2 (:2613-2652) followed by sr_e (:1195-1387) at size 1. */
int pic_renew_e4_2(pic_ctx *ctx);
/* The push loop of fdtd (:731-812): cal_track4 (:2804-2870) with the
 * shape_func_v2 gather (:3017-3326), the ballistic branch outside the
 * Absorb_grid2 box, and shape_func_*0_j_2 (:3397-3553). */
int pic_push_deposit_j(pic_ctx *ctx, int species);
/* The drift loop of fdtd (:818-867) with shape_func_*0_n_2 (:3333-3395). */
int pic_drift_deposit_n(pic_ctx *ctx, int species);
/* The thread reduction of fdtd (:869-886) and sr_current2 (:1805-2039) at
 * size 1: additive periodic fold of the ghost planes of J and n. */
int pic_reduce_current(pic_ctx *ctx);
/* sr_particle (:2041-2531) at size 1: delete z outflow and x/y < 2 dx,
 * wrap x/y >= (N+2) dx by -N dx. */
int pic_sr_particle(pic_ctx *ctx);
/* add_ion_flat then add_electron_flat (:5993-6818) at size 1. */
int pic_add_flat(pic_ctx *ctx);
/* sorting (:7475-7590): particles in cell order, ghost-cell particles dropped. */
int pic_sort(pic_ctx *ctx);
/* thrust_f sums (:4963-5101): F[27] and E[6] in FP64 on the device. */
int pic_thrust_f(pic_ctx *ctx, double *F27, double *E6);
/* Running mean of thrust_fave (:5124-5285): Fave[27] as accumulated since the
 * last reset (the reference resets it every 500 steps after printing). */
int pic_thrust_fave(pic_ctx *ctx, double *Fave27, int reset);
/* Gauss-law residual of the current state (no reference counterpart; it is
 * what the reference's compiled-out renew_phi3 :8315 would correct):
 * out = [sum (div4 E - rho/e0)^2, sum (rho/e0)^2, max |div4 E - rho/e0|, cells]. */
int pic_gauss_residual(pic_ctx *ctx, double *out4);
/* renew_phi3 (:8315-8665) + sr_phi (:1389-1574) + sr_e at size 1, the block a
 * build with the PHI blocks runs after renew_e4_2 (:901-907): phi solves
 * lap(phi) = -(div4 E - q (ni - ne)/e0) on the cells Absorb_grid3 leaves in, by
 * sine transforms; E += the 4th-order gradient of phi. pic_config.poisson_clean
 * runs it inside pic_step and pic_fdtd. */
int pic_poisson_clean(pic_ctx *ctx);

/* nsteps iterations of fdtd's loop body (:687-949) continuing the step
 * counters; the particle work of one step runs as one fused kernel per species. */
int pic_step(pic_ctx *ctx, int nsteps);
/* fdtd (:627-952) for nsteps: one add_*_flat, then pic_step(nsteps). */
int pic_fdtd(pic_ctx *ctx, int nsteps);

/* Differentiation (no counterpart in the reference).
 *
 * Objective: the impulse along z delivered to the dipole over nsteps loop
 * bodies from the current state,
 *   J = sum over steps of dt * F,  F = -sum_p s_p q n dx^3 (v x B0(x_p))_z
 * over the particles alive after each step's sr_particle (s_p = +1 for ions,
 * -1 for electrons; B0 gathered with the shape functions of B): the reaction
 * to the Lorentz force of the dipole's own field on the plasma.
 *
 * Both calls advance the state by nsteps loop bodies of fdtd (:687-949) in a
 * slot-stable form: no sorting (it only reorders particles), a refill that
 * compacts the slots before it appends, and current sums in 64-bit fixed
 * point so that every replay of a step is bit-identical.
 *
 * pic_objective: *J after nsteps.
 * pic_adjoint: out3 = {J, dJ/dI, dJ/dV}, the gradient with respect to the coil
 * current I (the dipole moment is mu0 I pi R^2; only the dipole part of B0
 * depends on it) and the drift V (every particle created by the initial load
 * or a refill has vz = V + thermal, so the current state must be such a load:
 * call it after pic_init_grid, pic_init_particle_flat and pic_fdtd(ctx, 0)).
 * The reverse pass keeps a checkpoint every checkpoint_every steps and
 * recomputes each segment, so device memory holds nsteps/checkpoint_every
 * full states plus checkpoint_every step inputs. That memory and the
 * adjoint's work arrays stay with the context after the call, for the next
 * pic_objective / pic_adjoint to reuse, until pic_destroy. The context ends in
 * the state after the nsteps loop bodies. */
int pic_objective(pic_ctx *ctx, int nsteps, double *J);
int pic_adjoint(pic_ctx *ctx, int nsteps, int checkpoint_every, double *out3);

/* The reference's files, byte-compatible, in directory dir (NULL: the working
 * directory); rank is the file-name rank (myrank_x + myrank_y * PROCESS_Nx).
 *
 * pic_save_checkpoint: suspend_job (:7629-7674): suspend-<rank>-field.dat, the
 * Grid records of every node (z fastest), and suspend-<rank>-<t>-ion.dat /
 * -electron.dat for t < nthreads, the 80-byte Particle structs (list links
 * written as zero), the particles split in nthreads consecutive parts.
 * pic_load_checkpoint: continue_job (:7676-7911): reads those files (as the
 * reference or pic_save_checkpoint wrote them) into the context and restarts
 * the random streams from their seeds as continue_job does; continue with
 * pic_fdtd, as the reference continues with fdtd. Every particle must carry
 * the species weight Nall/Np and flag 1.
 * pic_write_output: output (:4834-4883): fdtd458-0-0-<step>.dat, 23 columns
 * per interior node.
 * pic_append_thrust: the line thrust_f appends to thrust458.txt (:5111-5119).
 * pic_append_thrust_ave: when step % 500 == 0, the line thrust_fave appends to
 * thrust458_ave.txt (:5266-5276), then the running mean restarts. */
int pic_save_checkpoint(pic_ctx *ctx, const char *dir, int rank, int nthreads);
int pic_load_checkpoint(pic_ctx *ctx, const char *dir, int rank, int nthreads);
int pic_write_output(pic_ctx *ctx, const char *dir, int step);
int pic_append_thrust(pic_ctx *ctx, const char *dir, int step);
int pic_append_thrust_ave(pic_ctx *ctx, const char *dir, int step);

/* State import/export in reference units (FP64 host arrays). */
int pic_set_particles(pic_ctx *ctx, int species, const double *rows, const int *flag,
                      long long n);
int pic_get_particles(pic_ctx *ctx, int species, double *rows, int *flag, long long cap,
                      long long *n_out);
int pic_particle_count(pic_ctx *ctx, int species, long long *n_out);
int pic_get_grid(pic_ctx *ctx, double *records);
int pic_set_grid(pic_ctx *ctx, const double *records);
/* Random-stream draw counters (position, velocity) shared by init and add. */
int pic_rng_counters(pic_ctx *ctx, long long *ctr_p, long long *ctr_v, int set);

/* Device counters: errors [0] deposits or gathers skipped because the stencil
 * left the array, [1] particles dropped with a cell outside the index range,
 * [2] non-finite velocities after a push; work [3] particle pushes made by
 * the push kernels since creation; errors [4] sr_particle packets lost to a
 * full exchange list, [5] field tiles whose TMA-staged operands did not arrive
 * within the wait limit (the tile is left unchanged), [6] refilled particles
 * lost to a full particle store (pic_step places a refill after the count it
 * holds on the device, without waiting for it); [7] reserved.
 * Returns PIC_ERR_DEVICE when any error counter is non-zero. */
int pic_status(pic_ctx *ctx, long long *counters8);
/* *staged = 1 when renew_b4_2 / renew_e4_2 run the TMA-staged stencil kernels,
 * 0 when they run the per-node kernels (pic_config.plain_fields, or a row
 * pitch that is not a multiple of 16 bytes). */
int pic_field_path(pic_ctx *ctx, int *staged);
int pic_synchronize(pic_ctx *ctx);
/* The context's cudaStream_t, for callers that time or order work around it. */
int pic_get_stream(pic_ctx *ctx, void **stream);
/* Per-phase CUDA-event timing of pic_step (no reference counterpart; the
 * reference prints wall-clock times only, :684-705). While enabled, every step
 * records event pairs on the context's stream around its phases:
 * [0] particle push (fused kernels), [1] field updates, ghost copies and folds,
 * [2] sort, [3] boundary refill, [4] per-step diagnostics. pic_read_timing
 * synchronises, returns the summed milliseconds and pairs per phase, the
 * number of kernels the context has launched since creation, and restarts. */
int pic_set_timing(pic_ctx *ctx, int enable);
int pic_read_timing(pic_ctx *ctx, double *ms8, long long *pairs8, long long *launches);

/* No counterpart in the reference. The Gauss-law residual of pic_gauss_residual
 * for callers that cannot allocate device memory (a plugin inside a host
 * application that owns every device allocation): it takes the FP32 planes
 * ex, ey, ez, ni, ne of a padded (nx+4)*(ny+4)*(nz+4) grid (z fastest) and a
 * device array out4 of 4 doubles, all owned by the caller, queues its work on
 * `stream` (a cudaStream_t, NULL for the default stream) and allocates
 * nothing: its scratch is a static device array of 2048 x 4 doubles, which
 * caps the input at 2048 * 256 * 64 = 33,554,432 interior cells (larger inputs
 * return PIC_ERR_TOO_LARGE; non-finite dx, q or e0 return PIC_ERR_ARG). Each
 * call looks the scratch address up in the calling thread's current CUDA
 * context; the first call in a context also loads the library's device code
 * into it, so make that first call before any stream capture. All calls share
 * the scratch: calls whose kernels overlap on the GPU race and must be ordered. */
int pic_gauss_residual_noalloc(const float *ex, const float *ey, const float *ez,
                               const float *ni, const float *ne, int nx, int ny, int nz,
                               double dx, double q, double e0, void *stream, double *out4);
const char *pic_error_string(int code);

/* ------------------------------------------------------------------------
 * Batched 2D runs of PIC2D/2d_pic278_mpi.c (the x-z model with the coil's
 * line currents), MPI size 1: many independent runs of uneven sizes advanced
 * together on one GPU. The reference runs one such simulation per program
 * (main :129-188, main_func :201-222, fdtd :527-1019); here a batch replaces
 * them, each run keeping the reference's step.
 * ------------------------------------------------------------------------ */

/* Run-time form of the 2D reference's compile-time parameters (:31-87). */
typedef struct pic2d_config {
  int nx, nz;              /* Grid_Nx, Grid_Nz (interior cells along x, z) */
  int np;                  /* Np: Np*Np macro-particles per cell per species */
  int add_interval;        /* add_ion5 / add_electron5 every add_interval steps (250, :645);
                              the same for every run of a batch */
  double dx, dt;           /* dx, dtf (= dti = dte) */
  double q, mi, me, mu0, e0, kb, c;
  double v_drift;          /* V: drift along +z */
  double n_all, ti, te;    /* Nall, Ti, Te; particle weight N0i = N0e = Nall/Np/Np */
  double coil_i;           /* I: the coil's two line currents +-I/dx^2 (:2238-2268) */
  double imf_x, imf_y, imf_z;
  int absorb_grid;         /* Absorb_grid: field damping layer */
  int absorb_grid2;        /* Absorb_grid2: ballistic particle margin */
  int absorb_grid3;        /* Absorb_grid3: margin left out of renew_phi's source (>= 2) */
  int sort_interval;       /* no reference counterpart: every run's particles are sorted by cell every
                              sort_interval steps (and at each refill), which changes only their order;
                              0 sorts at refills only. The same for every run of a batch; 12 by
                              default */
  double sigma_a;          /* damping amplitude a of init_grid (:228) */
  unsigned long long seed_p, seed_v;  /* position / velocity stream keys (:406-407: 0, 50) */
  long long capacity;      /* particle slots per species of this run; 0 sizes it */
} pic2d_config;

typedef struct pic2d_batch pic2d_batch;

/* Normalized-units defaults (c = e0 = mu0 = q = m_e = dx = 1, m_i = 100, dt at
 * half of the 2D stability limit of the 4th-order stencil), the reference's
 * absorb widths (32, 16, 32) and refill interval (250). */
int pic2d_config_normalized(pic2d_config *cfg, int nx, int nz, int np);
/* precision 32 (FP32 fields and particles, FP64 thrust sums) or 64. */
int pic2d_create(const pic2d_config *cfgs, int nruns, int precision, int device, pic2d_batch **out);
int pic2d_destroy(pic2d_batch *b);
/* init_grid (:224-387) and init_particle (:389-525) of every run, then fdtd's
 * set-up before its loop (:583-625: density, sr_density, sr_grid, renew_phi). */
int pic2d_init(pic2d_batch *b);
/* nsteps bodies of fdtd's loop (:627-1015) for every run; plain steps replay
 * a captured CUDA graph. */
int pic2d_step(pic2d_batch *b, int nsteps);
/* thrust_F (:2304-2387) of every run: out3[3 r + {0, 1, 2}] = Fx, Fz, My. */
int pic2d_thrust(pic2d_batch *b, double *out3);
int pic2d_particle_count(pic2d_batch *b, int run, int species, long long *n);
/* Rows x z vx vy vz n (FP64, absolute positions with ghost cells). */
int pic2d_get_particles(pic2d_batch *b, int run, int species, double *rows6, long long cap, long long *n);
/* The run's grid as the reference's Grid records (:104-112: b0x b0y b0z bx by
 * bz ex ey ez jix0 jiy0 jiz0 jex0 jey0 jez0 ni ne phi), (nx+4)*(nz+4) nodes,
 * z fastest. */
int pic2d_get_grid(pic2d_batch *b, int run, double *records);
/* No counterpart in the reference. Tunes the push tile shape on the batch's
 * next 16 steps (ordinary steps of the runs): tiles of 1, 2, 4 or 8 rows of
 * 32 cells, with 8 or 16 blocks per SM; choice2 = {tile rows, blocks}. */
int pic2d_autotune(pic2d_batch *b, int *choice2);
/* No counterpart in the reference. Sets the push tile shape that
 * pic2d_autotune chooses (tile rows 1, 2, 4 or 8; persistent blocks >= 1), e.g.
 * one tuned on an earlier batch of the same sizes. */
int pic2d_set_push_shape(pic2d_batch *b, int tile_rows, int blocks);
int pic2d_set_graph(pic2d_batch *b, int enable);
/* counters8: [0..2] device errors as pic_status, [3] particle pushes,
 * [4] steps taken, [5] kernels launched. */
int pic2d_status(pic2d_batch *b, long long *counters8);
int pic2d_get_stream(pic2d_batch *b, void **stream);

#ifdef __cplusplus
}
#endif

#endif
