// C ABI of the B200 PIC step (declarations and reference citations in
// include/plasma_b200.h). Host-side orchestration: one CUDA stream per
// context, every kernel launched on it, no host synchronisation inside a step
// except the particle count read back after a sort.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/plasma_b200.h"
#include "common.cuh"
#include "diag.cuh"
#include "fields.cuh"
#include "fields_tma.cuh"
#include "particles.cuh"
#include "tiled.cuh"
#include "push_tiled.cuh"
#include "relayout.cuh"
#include "adjoint.cuh"
#include "poisson3d.cuh"
#include "halo.cuh"

using namespace pb;


namespace {

constexpr int kThreads = 256;

struct Store {
  void* mem[2] = {nullptr, nullptr};  // double-buffered for the sort
  int cur = 0;
  long long cap = 0;
  long long count = 0;  // slots in use (live and empty); the host's copy of *count_dev unless `pending`
  int* count_dev = nullptr;
  // *count_dev has moved on without the host (a placement, a re-listing push,
  // a refill appended on the device): kernels cover the slots up to the
  // capacity and stop at *count_dev, and sync_count reads it back when the
  // host needs it
  bool pending = false;
  // a placement's spill count and non-home flag are on their way into pinned
  // memory (event `readback`); check_spill acts on them
  bool spill_pending = false;
  cudaEvent_t readback = nullptr;
  int* holes = nullptr;   // per-slot scratch: hole rows of every lane column
  int* nholes = nullptr;  // per interior cell: holes of its lane column
  int* nonhome = nullptr; // a particle outside its home cell stayed in the layout
  // a refill's shell deletion over the layout is left to the next classify pass
  bool shell_pending = false;
};

// Device blocks of the adjoint runs: each block is allocated on first need,
// handed back to `spare` when a run releases it and reused by later runs of
// the same context; pic_destroy frees them. cudaMalloc and cudaFree inside
// the adjoint's loop would stall the stream at every step.
struct DevPool {
  std::vector<std::pair<void*, size_t>> spare;
  std::vector<void*> all;
  std::map<void*, size_t> size;
};

}  // namespace

struct pic_ctx {
  pic_config cfg{};
  Geom g{};
  int prec = 32;
  size_t rsize = 4;
  cudaStream_t stream = nullptr;
  // fields: F_COUNT planes
  void* field_mem = nullptr;
  size_t plane_bytes = 0;
  double* ramps = nullptr;  // rx[2gx], ry[2gy], rz[2gz]
  // tensor maps of the staged field kernels: E (the B half-step's curl
  // operands) and DB (the E step's), each plane with its own box
  CUtensorMap tm_e[3], tm_db[3];
  bool staged = false;
  Store sp[2];
  // sort and scan scratch
  TileGeom tg{};
  // tiled layout of each species, double-buffered (the sort reads the old one)
  int* goff[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int* gmax[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int lay[2] = {0, 0};                // current layout buffer
  bool layout[2] = {false, false};    // slots [0, tiled_end) follow goff/gmax[lay]
  long long tiled_end[2] = {0, 0};
  bool tiled[2] = {false, false};     // layout holds every slot: the tiled push may run
  int* gcap = nullptr;
  int* total_dev = nullptr;
  int* append_dev = nullptr;          // end of the append region during a re-layout
  int* rank = nullptr;                // per-slot scratch: placement rank of every appended particle
  int* bucket = nullptr;              // per-slot scratch: appended particles bucketed by their new cell
  int* cnt = nullptr;
  int* offs = nullptr;
  int* cursor = nullptr;
  int* scan_tmp = nullptr;
  size_t scan_tmp_len = 0;
  long long ncells = 0;
  // diagnostics
  double* acc = nullptr;        // 33 thrust/energy sums, then 4 Gauss-law values
  unsigned long long* maxbits = nullptr;
  double* fave = nullptr;       // 27
  // Poisson cleaning (renew_phi3): two interior-sized work arrays, the sine
  // tables of the three axes and their sin^2 eigenvalue terms
  void* phi_w = nullptr;
  void* phi_sines = nullptr;
  double* phi_sin2 = nullptr;
  // decomposed runs: the transport, the ghost-plane buffers and the particle
  // packet lists of sr_particle (kMig lists of mig_cap records, counters)
  pic_transport xport{};
  bool has_xport = false;
  void* halo_buf[2] = {nullptr, nullptr};  // send, receive
  size_t halo_bytes = 0;
  void* mig = nullptr;
  int* mig_cnt = nullptr;
  int mig_cap = 0;
  unsigned long long* err = nullptr;  // ERR_COUNT
  DevPool adj_pool;                   // the adjoint's work and snapshot memory
  int* host_pin = nullptr;            // pinned read-back slots: per species the spill count, the non-home flag
  // import/export staging
  void* stage = nullptr;
  size_t stage_bytes = 0;
  int* flags = nullptr;
  int* pos = nullptr;
  size_t flags_len = 0;
  // host state
  long long ctr_p = 0, ctr_v = 0;
  int c_add = 0, c_thrust = 0;
  bool grid_ready = false;
  int since_layout = 0;         // steps since the last re-layout or full sort (both species)
  bool particles_ready = false;
  // kernel launches issued by this context, and optional per-phase event timing
  long long launches = 0;
  bool timing = false;
  struct Phase {
    std::vector<cudaEvent_t> ev;  // start/stop pairs
    size_t used = 0;
  } phase[8];
};

#define CK(x)                                                         \
  do {                                                                \
    cudaError_t e_ = (x);                                             \
    if (e_ != cudaSuccess) {                                          \
      fprintf(stderr, "plasma_b200: %s: %s\n", #x, cudaGetErrorString(e_)); \
      return PIC_ERR_CUDA;                                            \
    }                                                                 \
  } while (0)
#define CKL()                      \
  do {                             \
    ++c->launches;                 \
    CK(cudaGetLastError());        \
  } while (0)
#define CKR(x)                \
  do {                        \
    int r_ = (x);             \
    if (r_ != PIC_OK) return r_; \
  } while (0)

namespace {

template <typename real>
Fields<real> fields(pic_ctx* c) {
  Fields<real> F;
  for (int q = 0; q < F_COUNT; ++q)
    F.f[q] = (real*)((char*)c->field_mem + (size_t)q * c->plane_bytes);
  return F;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t store_bytes(long long cap, size_t rsize) { return 2 * parts_record_bytes(cap, rsize); }

template <typename real>
Parts<real> parts(pic_ctx* c, int s, int buf) {
  char* base = (char*)c->sp[s].mem[buf];
  return make_parts<real>((real*)base, (real*)(base + parts_record_bytes(c->sp[s].cap, sizeof(real))));
}

template <typename real>
Parts<real> parts(pic_ctx* c, int s) {
  return parts<real>(c, s, c->sp[s].cur);
}

int grid_blocks(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (int)b;
}

// Persistent-style grid for particle loops: enough blocks to fill the GPU.
int particle_blocks(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  const long long cap = 148LL * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

int set_count(pic_ctx* c, int s, long long n) {
  if (n != c->sp[s].count || c->sp[s].pending) c->tiled[s] = false;  // appended or imported slots break the layout
  c->sp[s].count = n;
  c->sp[s].pending = false;
  set_int_kernel<<<1, 1, 0, c->stream>>>(c->sp[s].count_dev, (int)n);
  CKL();
  return PIC_OK;
}

// Slots a kernel over species s covers: the host count, or the capacity while
// a re-layout's new count is still on its way back to the host (such kernels
// stop at *count_dev).
long long slot_bound(const pic_ctx* c, int s) { return c->sp[s].pending ? c->sp[s].cap : c->sp[s].count; }

double species_mass(const pic_ctx* c, int s) { return s == 0 ? c->cfg.mi : c->cfg.me; }
double species_weight(const pic_ctx* c) { return c->cfg.n_all / c->cfg.np; }

template <typename real>
PushConst<real> push_const(const pic_ctx* c, int s) {
  const pic_config& k = c->cfg;
  PushConst<real> pc;
  const double m = s == 0 ? k.mi : -k.me;
  pc.T = (real)(0.5 * k.q * k.dt / m);
  pc.C = (real)k.c;
  pc.C2 = (real)(k.c * k.c);
  pc.hdt = (real)(0.5 * k.dt / k.dx);
  pc.qn = (real)(k.q * species_weight(c));
  pc.nw = (real)species_weight(c);
  pc.ex_add = (real)(k.v_drift * k.imf_y);
  pc.ey_add = (real)(-k.v_drift * k.imf_x);
  const Geom& g = c->g;
  pc.bal_lx = k.absorb_grid2 - g.ox;
  pc.bal_ly = k.absorb_grid2 - g.oy;
  pc.bal_lz = k.absorb_grid2;
  pc.bal_hx = g.gnx + 4 - k.absorb_grid2 - g.ox;
  pc.bal_hy = g.gny + 4 - k.absorb_grid2 - g.oy;
  pc.bal_hz = k.nz + 4 - k.absorb_grid2;
  // interior cells are [2, n + 2) on each axis; a particle there is ballistic
  // when it lies below bal_l* or at or above bal_h* (fdtd :733-735)
  pc.bal_interior = pc.bal_lx > 2 || pc.bal_ly > 2 || pc.bal_lz > 2 || pc.bal_hx < k.nx + 2 ||
                    pc.bal_hy < k.ny + 2 || pc.bal_hz < k.nz + 2;
  pc.out = Outbox<real>{nullptr, 0, nullptr};
  if (c->has_xport && c->mig) {  // list s of the packet lists is species s's outbox
    pc.out.count = c->mig_cnt + s;
    pc.out.cap = c->mig_cap;
    pc.out.rec = (MigRec<real>*)c->mig + (size_t)s * c->mig_cap;
  }
  pc.pjx = s == 0 ? F_JIX : F_JEX;
  pc.pjy = s == 0 ? F_JIY : F_JEY;
  pc.pjz = s == 0 ? F_JIZ : F_JEZ;
  pc.pn = s == 0 ? F_NI : F_NE;
  return pc;
}

// Phases timed by pic_read_timing.
enum { PH_PUSH = 0, PH_FIELD = 1, PH_SORT = 2, PH_ADD = 3, PH_DIAG = 4, PH_COUNT = 5 };

int phase_mark(pic_ctx* c, int ph) {
  if (!c->timing) return PIC_OK;
  auto& p = c->phase[ph];
  if (p.used == p.ev.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    p.ev.push_back(e);
  }
  CK(cudaEventRecord(p.ev[p.used++], c->stream));
  return PIC_OK;
}

// Tile shape of the staged field kernels: 4 x 8 x 32 nodes in FP32 (25.6 KB
// of staged planes), 4 x 4 x 32 in FP64 (30.7 KB).
template <typename real> struct StShape;
template <> struct StShape<float> { static constexpr int TX = 4, TY = 8; };
template <> struct StShape<double> { static constexpr int TX = 4, TY = 4; };

template <typename real>
using StTile = StencilTile<real, StShape<real>::TX, StShape<real>::TY>;

// Tensor maps of planes first, first + 1, first + 2 over the whole padded
// array (z fastest), each with its plane's box of StencilTile.
template <typename real>
bool make_stencil_maps(const pic_ctx* c, PFN_cuTensorMapEncodeTiled_v12000 encode, int first, CUtensorMap* out) {
  using T = StTile<real>;
  const cuuint32_t ex[3] = {T::EX0, T::EX1, T::EX2}, ey[3] = {T::EY0, T::EY1, T::EY2};
  const cuuint64_t dims[3] = {(cuuint64_t)c->g.gz, (cuuint64_t)c->g.gy, (cuuint64_t)c->g.gx};
  const cuuint64_t strides[2] = {(cuuint64_t)c->g.gz * sizeof(real), (cuuint64_t)c->g.sx * sizeof(real)};
  const cuuint32_t estr[3] = {1, 1, 1};
  for (int q = 0; q < 3; ++q) {
    const cuuint32_t box[3] = {(cuuint32_t)kStBoxZ, ey[q], ex[q]};
    void* base = (char*)c->field_mem + (size_t)(first + q) * c->plane_bytes;
    if (encode(&out[q], sizeof(real) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
               base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

// Chooses the staged field kernels when the row pitch (gz values) is a
// multiple of 16 bytes and the driver encodes the tensor maps; the per-node
// kernels otherwise, or when the configuration asks for them.
template <typename real>
void setup_staged_fields(pic_ctx* c) {
  using T = StTile<real>;
  c->staged = false;
  if (c->cfg.plain_fields || ((size_t)c->g.gz * sizeof(real)) % 16 != 0) return;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
      q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return;
  }
  const auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  if (!make_stencil_maps<real>(c, encode, F_EX, c->tm_e) || !make_stencil_maps<real>(c, encode, F_DBX, c->tm_db))
    return;
  if (cudaFuncSetAttribute(renew_b_tma_kernel<real, StShape<real>::TX, StShape<real>::TY>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes) != cudaSuccess ||
      cudaFuncSetAttribute(renew_e_tma_kernel<real, StShape<real>::TX, StShape<real>::TY>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  c->staged = true;
}

Ramps ramps(const pic_ctx* c) {
  Ramps r;
  r.rx = c->ramps;
  r.ry = c->ramps + 2 * c->g.gx;
  r.rz = c->ramps + 2 * c->g.gx + 2 * c->g.gy;
  r.a = c->cfg.sigma_a;
  return r;
}

// ------------------------------------------------------------- fields
template <typename real>
int do_init_grid(pic_ctx* c) {
  DipoleParams d{c->cfg.mu0, c->cfg.coil_i, c->cfg.coil_r, c->cfg.alpha, c->cfg.dx,
                 c->cfg.dipole_cutoff, c->cfg.imf_x, c->cfg.imf_y, c->cfg.imf_z};
  init_fields_kernel<real><<<grid_blocks(c->g.nodes), kThreads, 0, c->stream>>>(fields<real>(c), c->g, d);
  CKL();
  return PIC_OK;
}

// ------------------------------------------------- exchanges between ranks
// Rank number of process-grid coordinates (periodic), as main() numbers them.
int rank_at(const pic_ctx* c, int rx, int ry) {
  const int px = c->cfg.procs_x, py = c->cfg.procs_y;
  return ((ry % py + py) % py) * px + ((rx % px + px) % px);
}

int xfer(pic_ctx* c, const void* send, size_t sbytes, int dest, void* recv, size_t rbytes, int src) {
  if (c->xport.sendrecv(c->xport.user, send, sbytes, dest, recv, rbytes, src, (void*)c->stream) != 0)
    return PIC_ERR_COMM;
  return PIC_OK;
}

// One transfer of two layers of every plane of s along `axis`: layers
// send_layer, +1 to rank `dest`; from rank `src` into recv_layer, +1.
template <typename real>
int halo_exchange(pic_ctx* c, const PlaneSet<real>& s, const PlaneSet<real>& aux, int axis, int send_layer, int dest,
                  int recv_layer, int src, int mode) {
  const Geom& g = c->g;
  const size_t n = (size_t)s.count * 2 * (size_t)std::max(g.gy * g.gz, g.gx * g.gz);
  if (n * sizeof(real) > c->halo_bytes) {
    cudaFree(c->halo_buf[0]);
    cudaFree(c->halo_buf[1]);
    c->halo_buf[0] = c->halo_buf[1] = nullptr;
    c->halo_bytes = 0;
    const size_t bytes = (size_t)8 * 2 * std::max(g.gy * g.gz, g.gx * g.gz) * sizeof(real);
    CK(cudaMalloc(&c->halo_buf[0], bytes));
    CK(cudaMalloc(&c->halo_buf[1], bytes));
    c->halo_bytes = bytes;
  }
  const long long elems = (long long)s.count * 2 * halo_layer_nodes(g, axis);
  real* sb = (real*)c->halo_buf[0];
  real* rb = (real*)c->halo_buf[1];
  halo_pack_kernel<real><<<grid_blocks(elems), kThreads, 0, c->stream>>>(s, g, axis, send_layer, sb);
  CKL();
  CKR(xfer(c, sb, elems * sizeof(real), dest, rb, elems * sizeof(real), src));
  halo_unpack_kernel<real><<<grid_blocks(elems), kThreads, 0, c->stream>>>(s, aux, g, axis, recv_layer, rb, mode);
  CKL();
  return PIC_OK;
}

// sr_b / sr_e / sr_phi at any size (:1001-1387, :1389-1574): per axis (x, then
// y over every x), layers N, N+1 to the next rank's ghosts 0, 1 and layers
// 2, 3 to the previous rank's ghosts N+2, N+3, periodic over the ranks.
template <typename real>
int halo_ghosts(pic_ctx* c, const PlaneSet<real>& s, const PlaneSet<real>& aux, int mode) {
  const int rx = c->cfg.rank_x, ry = c->cfg.rank_y;
  for (int axis = 0; axis < 2; ++axis) {
    const int N = axis == 0 ? c->g.nx : c->g.ny;
    const int next = axis == 0 ? rank_at(c, rx + 1, ry) : rank_at(c, rx, ry + 1);
    const int prev = axis == 0 ? rank_at(c, rx - 1, ry) : rank_at(c, rx, ry - 1);
    CKR(halo_exchange<real>(c, s, aux, axis, N, next, 0, prev, mode));
    CKR(halo_exchange<real>(c, s, aux, axis, 2, prev, N + 2, next, mode));
  }
  return PIC_OK;
}

// sr_current2 at any size (:1805-2039): per axis, ghosts N+2, N+3 added to
// the next rank's layers 2, 3; ghosts 0, 1 added to the previous rank's N, N+1.
template <typename real>
int halo_fold(pic_ctx* c, const PlaneSet<real>& s) {
  const int rx = c->cfg.rank_x, ry = c->cfg.rank_y;
  for (int axis = 0; axis < 2; ++axis) {
    const int N = axis == 0 ? c->g.nx : c->g.ny;
    const int next = axis == 0 ? rank_at(c, rx + 1, ry) : rank_at(c, rx, ry + 1);
    const int prev = axis == 0 ? rank_at(c, rx - 1, ry) : rank_at(c, rx, ry - 1);
    CKR(halo_exchange<real>(c, s, s, axis, N + 2, next, 2, prev, HALO_ADD));
    CKR(halo_exchange<real>(c, s, s, axis, 0, prev, N, next, HALO_ADD));
  }
  return PIC_OK;
}

// Particle packet lists of sr_particle: 0, 1 the species' outboxes, then the
// split and received lists of the x and y passes.
enum { MIG_OUT0 = 0, MIG_OUT1 = 1, MIG_XF, MIG_XB, MIG_YS, MIG_YF, MIG_YB, MIG_FIN, MIG_RA, MIG_RB, kMig };

template <typename real>
int ensure_mig(pic_ctx* c) {
  if (c->mig) return PIC_OK;
  const Geom& g = c->g;
  // packets of one step: at most the particles of the outer two cell layers
  // of the x and y faces; a list that overflows counts ERR_MIGRATION
  const long long face = 2LL * ((long long)g.gy * g.gz + (long long)g.gx * g.gz);
  const long long cap = std::min<long long>(face * std::max(c->cfg.np, 1) + 65536, 1LL << 30);
  c->mig_cap = (int)cap;
  CK(cudaMalloc(&c->mig, (size_t)kMig * cap * sizeof(MigRec<real>)));
  CK(cudaMalloc(&c->mig_cnt, sizeof(int) * 16));
  CK(cudaMemsetAsync(c->mig_cnt, 0, sizeof(int) * 16, c->stream));
  return PIC_OK;
}

template <typename real>
MigRec<real>* mig_list(pic_ctx* c, int q) {
  return (MigRec<real>*)c->mig + (size_t)q * c->mig_cap;
}

// sr_particle between ranks (:2041-2555) for species s, after the push has
// written the particles that left the rank's x-y interior to its outbox: the
// x pass (forward and backward packets to the x neighbours, received packets
// shifted by -/+ Nx cells), then the y pass over the particles still outside
// in y, then the settled packets appended after the particle slots.
template <typename real>
int do_migrate_species(pic_ctx* c, int s) {
  const Geom& g = c->g;
  const int rx = c->cfg.rank_x, ry = c->cfg.rank_y;
  int* cnt = c->mig_cnt;
  const size_t rec = sizeof(MigRec<real>);
  CK(cudaMemsetAsync(cnt + MIG_XF, 0, sizeof(int) * (kMig - MIG_XF), c->stream));
  int h[16];
  const int blocks = particle_blocks(c->mig_cap);
  int in_list = MIG_OUT0 + s;
  for (int axis = 0; axis < 2; ++axis) {
    const int F = axis == 0 ? MIG_XF : MIG_YF, B = axis == 0 ? MIG_XB : MIG_YB;
    const int S = axis == 0 ? MIG_YS : MIG_FIN;
    const bool lo = axis == 0 ? g.xlo : g.ylo, hi = axis == 0 ? g.xhi : g.yhi;
    // rank 0 drops its backward packets, the last rank (when it is not also
    // rank 0) its forward ones (:2137-2146, :2237-2246)
    mig_split_kernel<real><<<blocks, kThreads, 0, c->stream>>>(
        mig_list<real>(c, in_list), cnt + in_list, g, axis, lo ? 1 : 0, (hi && !lo) ? 1 : 0, mig_list<real>(c, F),
        cnt + F, mig_list<real>(c, B), cnt + B, mig_list<real>(c, S), cnt + S, c->mig_cap, c->err);
    CKL();
    const int next = axis == 0 ? rank_at(c, rx + 1, ry) : rank_at(c, rx, ry + 1);
    const int prev = axis == 0 ? rank_at(c, rx - 1, ry) : rank_at(c, rx, ry - 1);
    // counts first (the receiver sizes its copy), then the packets
    CKR(xfer(c, cnt + F, sizeof(int), next, cnt + MIG_RA, sizeof(int), prev));
    CKR(xfer(c, cnt + B, sizeof(int), prev, cnt + MIG_RB, sizeof(int), next));
    CK(cudaMemcpyAsync(h, cnt, sizeof(int) * kMig, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int nf = std::min(h[F], c->mig_cap), nb = std::min(h[B], c->mig_cap);
    const int ra = std::min(h[MIG_RA], c->mig_cap), rb = std::min(h[MIG_RB], c->mig_cap);
    CKR(xfer(c, mig_list<real>(c, F), nf * rec, next, mig_list<real>(c, MIG_RA), ra * rec, prev));
    CKR(xfer(c, mig_list<real>(c, B), nb * rec, prev, mig_list<real>(c, MIG_RB), rb * rec, next));
    const int N = axis == 0 ? g.nx : g.ny;
    // a forward packet arrives from the previous rank (:2374-2378)
    if (ra > 0) {
      mig_receive_kernel<real><<<particle_blocks(ra), kThreads, 0, c->stream>>>(
          mig_list<real>(c, MIG_RA), ra, axis, -N, mig_list<real>(c, S), cnt + S, c->mig_cap, c->err);
      CKL();
    }
    if (rb > 0) {
      mig_receive_kernel<real><<<particle_blocks(rb), kThreads, 0, c->stream>>>(
          mig_list<real>(c, MIG_RB), rb, axis, N, mig_list<real>(c, S), cnt + S, c->mig_cap, c->err);
      CKL();
    }
    in_list = S;
  }
  CK(cudaMemcpyAsync(h, cnt, sizeof(int) * kMig, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int nfin = std::min(h[MIG_FIN], c->mig_cap);
  Store& st = c->sp[s];
  if (st.count + nfin > st.cap) return PIC_ERR_CAPACITY;
  if (nfin > 0) {
    mig_append_kernel<real><<<particle_blocks(nfin), kThreads, 0, c->stream>>>(
        mig_list<real>(c, MIG_FIN), nfin, parts<real>(c, s), (int)st.count);
    CKL();
    // appended after the slots the layout and its tail cover: the slot-order
    // push handles them until the next re-layout, so the layout stays valid
    st.count += nfin;
    set_int_kernel<<<1, 1, 0, c->stream>>>(st.count_dev, (int)st.count);
    CKL();
  }
  CK(cudaMemsetAsync(cnt + MIG_OUT0 + s, 0, sizeof(int), c->stream));
  return PIC_OK;
}

template <typename real>
int do_migrate(pic_ctx* c) {
  for (int s = 0; s < 2; ++s) CKR(do_migrate_species<real>(c, s));
  return PIC_OK;
}

template <typename real>
int wrap_planes(pic_ctx* c, const int* ids, int n) {
  PlaneSet<real> s{};
  Fields<real> F = fields<real>(c);
  for (int q = 0; q < n; ++q) s.p[q] = F.f[ids[q]];
  s.count = n;
  if (c->has_xport) return halo_ghosts<real>(c, s, s, HALO_COPY);
  wrap_kernel<real><<<grid_blocks(4LL * n * c->g.gy * c->g.gz), kThreads, 0, c->stream>>>(s, c->g, 0);
  CKL();
  wrap_kernel<real><<<grid_blocks(4LL * n * c->g.gx * c->g.gz), kThreads, 0, c->stream>>>(s, c->g, 1);
  CKL();
  return PIC_OK;
}

template <typename real>
int do_renew_b(pic_ctx* c) {
  BParams p{1. / c->cfg.e0 * c->cfg.dt * 0.5 * 0.5, 0.5 * c->cfg.dt, 1.0 / (24.0 * c->cfg.dx)};
  if (c->staged) {
    constexpr int TX = StShape<real>::TX, TY = StShape<real>::TY;
    const int ty = (c->g.ny + TY - 1) / TY, tz = (c->g.nz + kStZ - 1) / kStZ, tx = (c->g.nx + TX - 1) / TX;
    renew_b_tma_kernel<real, TX, TY><<<tx * ty * tz, kStThreads, StTile<real>::bytes, c->stream>>>(
        c->tm_e[0], c->tm_e[1], c->tm_e[2], fields<real>(c), c->g, ramps(c), p, ty, tz, c->err);
  } else {
    const long long nint = (long long)c->g.nx * c->g.ny * c->g.nz;
    renew_b_kernel<real><<<grid_blocks(nint), kThreads, 0, c->stream>>>(fields<real>(c), c->g, ramps(c), p);
  }
  CKL();
  if (c->has_xport) {
    Fields<real> F = fields<real>(c);
    PlaneSet<real> s{}, aux{};
    for (int q = 0; q < 3; ++q) {
      s.p[q] = F.f[F_BX + q];
      aux.p[q] = F.f[F_DBX + q];
      aux.p[3 + q] = F.f[F_B0X + q];
    }
    s.count = 3;
    aux.count = 6;
    return halo_ghosts<real>(c, s, aux, HALO_BTOTAL);
  }
  wrap_b_kernel<real><<<grid_blocks(12LL * c->g.gy * c->g.gz), kThreads, 0, c->stream>>>(fields<real>(c), c->g, 0);
  CKL();
  wrap_b_kernel<real><<<grid_blocks(12LL * c->g.gx * c->g.gz), kThreads, 0, c->stream>>>(fields<real>(c), c->g, 1);
  CKL();
  return PIC_OK;
}

template <typename real>
int do_renew_e(pic_ctx* c) {
  EParams p{c->cfg.c * c->cfg.c * c->cfg.dt, c->cfg.mu0, 1.0 / (24.0 * c->cfg.dx)};
  if (c->staged) {
    constexpr int TX = StShape<real>::TX, TY = StShape<real>::TY;
    const int ty = (c->g.ny + TY - 1) / TY, tz = (c->g.nz + kStZ - 1) / kStZ, tx = (c->g.nx + TX - 1) / TX;
    renew_e_tma_kernel<real, TX, TY><<<tx * ty * tz, kStThreads, StTile<real>::bytes, c->stream>>>(
        c->tm_db[0], c->tm_db[1], c->tm_db[2], fields<real>(c), c->g, ramps(c), p, ty, tz, c->err);
  } else {
    const long long nint = (long long)c->g.nx * c->g.ny * c->g.nz;
    renew_e_kernel<real><<<grid_blocks(nint), kThreads, 0, c->stream>>>(fields<real>(c), c->g, ramps(c), p);
  }
  CKL();
  static const int ids[3] = {F_EX, F_EY, F_EZ};
  return wrap_planes<real>(c, ids, 3);
}

template <typename real>
int do_fold(pic_ctx* c) {
  PlaneSet<real> s{};
  Fields<real> F = fields<real>(c);
  for (int q = 0; q < 8; ++q) s.p[q] = F.f[F_JIX + q];
  s.count = 8;
  if (c->has_xport) return halo_fold<real>(c, s);
  fold_kernel<real><<<grid_blocks(32LL * c->g.gy * c->g.gz), kThreads, 0, c->stream>>>(s, c->g, 0);
  CKL();
  fold_kernel<real><<<grid_blocks(32LL * c->g.gx * c->g.gz), kThreads, 0, c->stream>>>(s, c->g, 1);
  CKL();
  return PIC_OK;
}

// renew_phi3 + sr_phi + sr_e (:8315-8665, :1389-1574): the Gauss residual,
// three sine transforms, the eigenvalue division, three inverse transforms,
// phi on the interior, its ghost planes wrapped, E corrected and wrapped.
template <typename real>
int do_poisson(pic_ctx* c) {
  const Geom& g = c->g;
  const long long n = (long long)g.nx * g.ny * g.nz;
  const int ns[3] = {g.nx, g.ny, g.nz};
  long long soff[3];
  soff[0] = 0;
  soff[1] = (long long)g.nx * g.nx;
  soff[2] = soff[1] + (long long)g.ny * g.ny;
  const long long stotal = soff[2] + (long long)g.nz * g.nz;
  if (!c->phi_w) {
    CK(cudaMalloc(&c->phi_w, 2 * (size_t)n * sizeof(real)));
    CK(cudaMalloc(&c->phi_sines, (size_t)stotal * sizeof(real)));
    CK(cudaMalloc(&c->phi_sin2, (size_t)(g.nx + g.ny + g.nz) * sizeof(double)));
    const double Pi = 3.14159265358979323846;
    std::vector<real> S((size_t)stotal);
    std::vector<double> s2;
    for (int a = 0; a < 3; ++a) {
      const int m = ns[a];
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) S[soff[a] + (long long)i * m + j] = (real)std::sin(Pi * (double)i * (double)j / (double)m);
      for (int i = 0; i < m; ++i) {
        const double v = std::sin(Pi * (double)i / (double)m / 2.);  // :8502-8504
        s2.push_back(v * v);
      }
    }
    CK(cudaMemcpy(c->phi_sines, S.data(), S.size() * sizeof(real), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->phi_sin2, s2.data(), s2.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  real* w0 = (real*)c->phi_w;
  real* w1 = w0 + n;
  const real* S = (const real*)c->phi_sines;
  const double d24 = 24. * c->cfg.dx;
  Fields<real> F = fields<real>(c);
  phi3_rho_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(F, g, d24, c->cfg.q, c->cfg.e0,
                                                                     c->cfg.absorb_grid3, w0);
  CKL();
  auto gemm = [&](DstGemm<real> a) -> int {
    const long long tiles = (long long)((a.M + kDstTile - 1) / kDstTile) * ((a.N + kDstTile - 1) / kDstTile) * a.B;
    const int blocks = (int)std::min<long long>(tiles, 148LL * 8);
    a.sin2 = c->phi_sin2;
    a.nx = g.nx; a.ny = g.ny; a.nz = g.nz;
    a.h2 = (c->cfg.dx / 2.) * (c->cfg.dx / 2.);
    dst3_gemm_kernel<real><<<blocks, 256, 0, c->stream>>>(a);
    CKL();
    return PIC_OK;
  };
  const long long yz = (long long)g.ny * g.nz;
  // C = mul * L R / div. z: [x*y][z] x S_z; y: S_y x [y][z] per x; x: S_x x [x][y*z]
  auto zpass = [&](const real* in, real* out, double mul, double div) {
    DstGemm<real> a{};
    a.L = in; a.lm = g.nz; a.R = S + soff[2]; a.rk = g.nz; a.C = out; a.cm = g.nz;
    a.M = g.nx * g.ny; a.N = g.nz; a.K = g.nz; a.B = 1; a.mul = mul; a.div = div;
    return gemm(a);
  };
  auto ypass = [&](const real* in, real* out, double mul, double div) {
    DstGemm<real> a{};
    a.L = S + soff[1]; a.lm = g.ny; a.R = in; a.rb = yz; a.rk = g.nz; a.C = out; a.cb = yz; a.cm = g.nz;
    a.M = g.ny; a.N = g.nz; a.K = g.ny; a.B = g.nx; a.mul = mul; a.div = div;
    return gemm(a);
  };
  auto xpass = [&](const real* in, real* out, double mul, double div, int solve) {
    DstGemm<real> a{};
    a.L = S + soff[0]; a.lm = g.nx; a.R = in; a.rk = yz; a.C = out; a.cm = yz;
    a.M = g.nx; a.N = (int)yz; a.K = g.nx; a.B = 1; a.mul = mul; a.div = div; a.solve = solve;
    return gemm(a);
  };
  CKR(zpass(w0, w1, 1., 1.));                    // fft_z
  CKR(ypass(w1, w0, 1., 1.));                    // fft_y
  CKR(xpass(w0, w1, 1., 1., 1));                 // fft_x and the division by A
  CKR(xpass(w1, w0, 2., (double)g.nx, 0));       // inv_fft_x
  CKR(ypass(w0, w1, 2., (double)g.ny));          // inv_fft_y
  CKR(zpass(w1, w0, 2., (double)g.nz));          // inv_fft_z
  phi3_store_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(F, g, w0);
  CKL();
  static const int phi_id[1] = {F_PHI};
  CKR(wrap_planes<real>(c, phi_id, 1));          // sr_phi's exchange
  phi3_grad_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(F, g, d24);
  CKL();
  static const int e_ids[3] = {F_EX, F_EY, F_EZ};
  return wrap_planes<real>(c, e_ids, 3);         // sr_e
}

int do_renew_grid(pic_ctx* c) {
  // J and n planes are contiguous (F_JIX .. F_NE)
  CK(cudaMemsetAsync((char*)c->field_mem + (size_t)F_JIX * c->plane_bytes, 0,
                     (size_t)(F_NE - F_JIX + 1) * c->plane_bytes, c->stream));
  return PIC_OK;
}

// ---------------------------------------------------------- particles
// The slot-order push over slots [first, count) (global-memory atomics).
template <typename real, int MODE>
int do_push(pic_ctx* c, int s, long long first = 0) {
  // with a re-layout's count still pending, the grid covers every slot up to
  // the capacity and the kernel stops at *count_dev
  const long long end = slot_bound(c, s);
  if (end <= first) return PIC_OK;
  push_kernel<real, MODE><<<particle_blocks(end - first), kThreads, 0, c->stream>>>(
      parts<real>(c, s), (int)first, c->sp[s].count_dev, fields<real>(c), c->g, push_const<real>(c, s),
      c->err);
  CKL();
  return PIC_OK;
}

__global__ void copy_int_kernel(int* dst, const int* src) { *dst = *src; }

// The push of species s: the slots after the layout (particles a placement
// could not place) with the slot-order kernel, then the tiled kernel.
template <typename real>
int do_push_tiled(pic_ctx* c, int s) {
  if (!c->layout[s]) return do_push<real, PUSH_FUSED>(c, s);
  CKR((do_push<real, PUSH_FUSED>(c, s, c->tiled_end[s])));
  const int ntiles = c->tg.ntx * c->tg.nty * c->tg.ntz;
  TileArgs ta{c->tg, c->goff[s][c->lay[s]], c->gmax[s][c->lay[s]]};
  const bool vec = sizeof(real) == 4 && c->g.gz % 4 == 0;
  const Parts<real> P = parts<real>(c, s);
  const Fields<real> F = fields<real>(c);
  const PushConst<real> pc = push_const<real>(c, s);
  const dim3 grid(ntiles), block(kTileX * kTileY * 32);
  const size_t smem = PushSmem<real>::bytes;
  if (vec) push_tiled_kernel<real, true><<<grid, block, smem, c->stream>>>(P, ta, F, c->g, pc, c->err);
  else push_tiled_kernel<real, false><<<grid, block, smem, c->stream>>>(P, ta, F, c->g, pc, c->err);
  CKL();
  return PIC_OK;
}

template <typename real>
int do_drift_n(pic_ctx* c, int s) {
  if (c->sp[s].count == 0) return PIC_OK;
  drift_n_kernel<real><<<particle_blocks(c->sp[s].count), kThreads, 0, c->stream>>>(
      parts<real>(c, s), c->sp[s].count_dev, fields<real>(c), c->g, push_const<real>(c, s), c->err);
  CKL();
  return PIC_OK;
}

template <typename real>
int do_sr_particle(pic_ctx* c) {
  if (c->has_xport) CKR(ensure_mig<real>(c));
  for (int s = 0; s < 2; ++s) {
    if (c->sp[s].count == 0) continue;
    sr_particle_kernel<real><<<particle_blocks(c->sp[s].count), kThreads, 0, c->stream>>>(
        parts<real>(c, s), c->sp[s].count_dev, c->g, push_const<real>(c, s).out, c->err);
    CKL();
  }
  if (c->has_xport) CKR(do_migrate<real>(c));
  return PIC_OK;
}

// Exclusive scan of n ints (in place allowed when in != out is not required).
int scan_exclusive(pic_ctx* c, const int* in, int* out, long long n, int* tmp, size_t tmp_len) {
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  if ((size_t)tiles + 1 > tmp_len) return PIC_ERR_STATE;
  scan_tile_kernel<<<(unsigned)tiles, kScanThreads, 0, c->stream>>>(in, out, tmp, n);
  CKL();
  if (tiles > 1) {
    CKR(scan_exclusive(c, tmp, tmp, tiles, tmp + tiles + 1, tmp_len - (size_t)tiles - 1));
    scan_add_kernel<<<(unsigned)tiles, 256, 0, c->stream>>>(out, tmp, n);
    CKL();
  }
  return PIC_OK;
}

SourceParams source_params(const pic_ctx* c, int s, const Slab* slabs, int nslab, int init_form);
int refill_slabs(const pic_ctx* c, Slab* slabs);

// sorting (:7475-7590) into the tiled layout of tiled.cuh: count the
// particles of every interior cell (stayers of the previous layout per lane
// column, movers and appended particles per destination cell), size every
// group by its fullest lane, scan the group sizes, then write stayers in their
// previous column order and movers after them. Particles outside the interior
// are dropped, as the reference's sort drops them.
template <typename real>
int do_sort_species(pic_ctx* c, int s) {
  Store& st = c->sp[s];
  const TileGeom& tg = c->tg;
  const int old = c->lay[s], nw = 1 - old;
  const bool have = c->layout[s];
  const long long first = have ? c->tiled_end[s] : 0;   // slots outside the old layout
  int* stay = c->cnt;
  int* moved = c->offs;
  CK(cudaMemsetAsync(stay, 0, sizeof(int) * c->ncells, c->stream));
  CK(cudaMemsetAsync(moved, 0, sizeof(int) * c->ncells, c->stream));
  CK(cudaMemsetAsync(c->cursor, 0, sizeof(int) * c->ncells, c->stream));
  const int gblocks = grid_blocks((long long)tg.ngroups * 32);
  const Parts<real> P = parts<real>(c, s);
  if (have) {
    tiled_count_kernel<real><<<gblocks, kThreads, 0, c->stream>>>(P, c->g, tg, c->goff[s][old], c->gmax[s][old],
                                                                  stay, moved);
    CKL();
  }
  if (st.count > first) {
    append_count_kernel<real><<<particle_blocks(st.count - first), kThreads, 0, c->stream>>>(
        P, (int)first, st.count_dev, c->g, moved);
    CKL();
  }
  Slab slabs[5];
  refill_slabs(c, slabs);
  group_size_kernel<<<gblocks, kThreads, 0, c->stream>>>(c->g, tg, stay, moved, source_params(c, s, slabs, 5, 0),
                                                         c->gmax[s][nw], c->gcap);
  CKL();
  CKR(scan_exclusive(c, c->gcap, c->goff[s][nw], tg.ngroups, c->scan_tmp, c->scan_tmp_len));
  tiled_total_kernel<<<1, 1, 0, c->stream>>>(c->goff[s][nw], c->gcap, tg.ngroups, c->total_dev);
  CKL();
  int total = 0;
  CK(cudaMemcpyAsync(&total, c->total_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (total > st.cap) return PIC_ERR_CAPACITY;
  Parts<real> Q = parts<real>(c, s, 1 - st.cur);
  group_pad_kernel<<<gblocks, kThreads, 0, c->stream>>>(c->g, tg, stay, moved, c->goff[s][nw], c->gmax[s][nw],
                                                        Q.cell);
  CKL();
  if (have) {
    tiled_scatter_kernel<real><<<gblocks, kThreads, 0, c->stream>>>(
        P, c->g, tg, c->goff[s][old], c->gmax[s][old], c->goff[s][nw], stay, c->cursor, Q);
    CKL();
  }
  if (st.count > first) {
    append_scatter_kernel<real><<<particle_blocks(st.count - first), kThreads, 0, c->stream>>>(
        P, (int)first, st.count_dev, c->g, tg, c->goff[s][nw], stay, c->cursor, Q);
    CKL();
  }
  st.cur = 1 - st.cur;
  c->lay[s] = nw;
  CKR(set_count(c, s, total));
  CK(cudaMemsetAsync(st.nonhome, 0, sizeof(int), c->stream));
  c->layout[s] = true;
  c->tiled_end[s] = total;
  c->tiled[s] = true;
  return PIC_OK;
}

// In-place re-layout (relayout.cuh): movers and appended particles into the
// holes of their columns, which a classify pass lists (relayout_launch). It
// issues the placement, set the new count on the device and read the
// spill count back into pinned memory without waiting; check_spill acts on
// that read-back when it has landed (a full sort when many particles found no
// hole), sync_count reads the count itself when the host needs it.
__global__ void spill_count_kernel(int* count, int first, const int* nspill) { *count = first + *nspill; }

// The placement of the particles in [tiled_end, *count_dev) into the holes
// that st.holes / st.nholes list (place_launch).
template <typename real>
int place_launch(pic_ctx* c, int s) {
  Store& st = c->sp[s];
  const TileGeom& tg = c->tg;
  const int gblocks = grid_blocks((long long)tg.ngroups * 32);
  const Parts<real> P = parts<real>(c, s);
  const long long first = c->tiled_end[s];
  const Parts<real> Q = parts<real>(c, s, 1 - st.cur);
  CK(cudaMemsetAsync(c->cursor, 0, sizeof(int) * c->ncells, c->stream));
  CK(cudaMemsetAsync(c->total_dev, 0, sizeof(int), c->stream));  // spill count
  place_count_kernel<real><<<particle_blocks(st.cap - first), kThreads, 0, c->stream>>>(
      P, (int)first, st.count_dev, c->g, c->cursor, c->rank);
  CKL();
  int* off = c->offs;  // per cell: arrivals that fit, then their bucket offset
  place_fit_kernel<<<particle_blocks(c->ncells), kThreads, 0, c->stream>>>(c->cursor, st.nholes, off, c->ncells);
  CKL();
  CKR(scan_exclusive(c, off, off, c->ncells, c->scan_tmp, c->scan_tmp_len));
  place_bucket_kernel<real><<<particle_blocks(st.cap - first), kThreads, 0, c->stream>>>(
      P, (int)first, st.count_dev, c->g, st.nholes, off, c->rank, c->bucket, c->total_dev, Q);
  CKL();
  place_fill_kernel<real><<<gblocks, kThreads, 0, c->stream>>>(P, (int)first, c->g, tg, c->goff[s][c->lay[s]],
                                                               st.holes, c->cursor, st.nholes, off, c->bucket);
  CKL();
  unspill_kernel<real><<<particle_blocks(st.cap), kThreads, 0, c->stream>>>(Q, c->total_dev, P, (int)first);
  CKL();
  spill_count_kernel<<<1, 1, 0, c->stream>>>(st.count_dev, (int)first, c->total_dev);
  CKL();
  CK(cudaMemcpyAsync(c->host_pin + s, c->total_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->host_pin + 2 + s, st.nonhome, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(st.readback, c->stream));
  st.pending = true;
  st.spill_pending = true;
  c->tiled[s] = true;
  return PIC_OK;
}

// The classify pass (every slot of the layout), then the placement.
template <typename real>
int relayout_launch(pic_ctx* c, int s) {
  Store& st = c->sp[s];
  const TileGeom& tg = c->tg;
  const int gblocks = grid_blocks((long long)tg.ngroups * 32);
  const Parts<real> P = parts<real>(c, s);
  CK(cudaMemsetAsync(st.nonhome, 0, sizeof(int), c->stream));
  copy_int_kernel<<<1, 1, 0, c->stream>>>(c->append_dev, st.count_dev);
  CKL();
  classify_kernel<real><<<gblocks, kThreads, 0, c->stream>>>(P, c->g, tg, c->goff[s][c->lay[s]],
                                                             c->gmax[s][c->lay[s]], (int)st.cap, st.holes,
                                                             st.nholes, c->append_dev, st.nonhome,
                                                             st.shell_pending ? 1 : 0);
  CKL();
  st.shell_pending = false;
  clamp_count_kernel<<<1, 1, 0, c->stream>>>(c->append_dev, (int)st.cap, st.count_dev);
  CKL();
  return place_launch<real>(c, s);
}

// The host's copy of the count, read back from the device when it moved on.
int sync_count(pic_ctx* c, int s) {
  Store& st = c->sp[s];
  if (!st.pending) return PIC_OK;
  int n = 0;
  CK(cudaMemcpyAsync(&n, st.count_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  st.count = n;
  st.pending = false;
  return PIC_OK;
}

// A placement's spill count (waiting for its read-back when `wait`): many
// particles without a hole, or particles outside their home cells left in
// the layout, call for a full sort (particles without a hole are pushed in
// slot order meanwhile).
template <typename real>
int check_spill(pic_ctx* c, int s, bool wait) {
  Store& st = c->sp[s];
  if (!st.spill_pending) return PIC_OK;
  if (wait) {
    CK(cudaEventSynchronize(st.readback));
  } else {
    const cudaError_t q = cudaEventQuery(st.readback);
    if (q == cudaErrorNotReady) {
      cudaGetLastError();  // not an error: the read-back is still on its way
      return PIC_OK;
    }
    CK(q);
  }
  st.spill_pending = false;
  const long long first = c->tiled_end[s];
  if (c->host_pin[s] > first / 50 || c->host_pin[2 + s]) {
    CKR(sync_count(c, s));
    return do_sort_species<real>(c, s);
  }
  return PIC_OK;
}

// Re-layout of every species that needs one (a full sort for a species with
// no layout yet), leaving the counts pending.
template <typename real>
int relayout_species(pic_ctx* c, const bool (&which)[2]) {
  for (int s = 0; s < 2; ++s) {
    if (!which[s]) continue;
    if (c->layout[s]) {
      CKR(relayout_launch<real>(c, s));
    } else {
      CKR(sync_count(c, s));
      CKR(do_sort_species<real>(c, s));
    }
  }
  return PIC_OK;
}

template <typename real>
int resolve_counts(pic_ctx* c) {
  for (int s = 0; s < 2; ++s) {
    CKR(check_spill<real>(c, s, true));
    CKR(sync_count(c, s));
  }
  return PIC_OK;
}

template <typename real>
int do_sort(pic_ctx* c) {
  const bool both[2] = {true, true};
  CKR(relayout_species<real>(c, both));
  c->since_layout = 0;
  return resolve_counts<real>(c);
}

// Generates `total` particles of species s from the slabs into slots
// [count, count + total), drawing from the shared position/velocity streams.
// Source description of species s for the given slabs, drawing from the
// current position of the shared random streams.
SourceParams source_params(const pic_ctx* c, int s, const Slab* slabs, int nslab, int init_form) {
  SourceParams sp{};
  sp.init_form = init_form;
  long long total = 0;
  for (int q = 0; q < nslab; ++q) {
    sp.slab[q] = slabs[q];
    sp.slab[q].first = total;
    total += (long long)slabs[q].nk * slabs[q].nl * slabs[q].nm * c->cfg.np;
  }
  sp.nslab = nslab;
  sp.np = c->cfg.np;
  sp.total = total;
  const double T = s == 0 ? c->cfg.ti : c->cfg.te;
  const double sig = std::sqrt(c->cfg.kb * T / species_mass(c, s));
  sp.dx = c->cfg.dx;
  sp.lsig = std::sqrt(sig * sig);
  sp.vdrift = c->cfg.v_drift;
  sp.seed_p = c->cfg.seed_p;
  sp.seed_v = c->cfg.seed_v;
  sp.base_p = c->ctr_p;
  sp.base_v = c->ctr_v;
  sp.dst = (int)c->sp[s].count;
  return sp;
}

// add_ion_flat :6037-6220 at size 1: z slabs, y slabs, the low-x slab.
int refill_slabs(const pic_ctx* c, Slab* slabs) {
  const int Nx = c->cfg.nx, Ny = c->cfg.ny, Nz = c->cfg.nz;
  const Geom& g = c->g;
  int n = 0;
  slabs[n++] = {2, Nx, 2, Ny, 2, 2, 0};                  // z = 2, 3 (:6035-6071)
  slabs[n++] = {2, Nx, 2, Ny, Nz, 2, 0};                 // z = Nz, Nz+1 (:6072-6108)
  if (g.ylo) slabs[n++] = {2, Nx, 2, 2, 4, Nz - 4, 0};   // y = 2, 3 on the low-y ranks (:6109-6145)
  if (g.yhi) slabs[n++] = {2, Nx, Ny, 2, 4, Nz - 4, 0};  // y = Ny, Ny+1 on the high-y ranks (:6147-6183)
  // one x slab, by the first branch of the chain at :6185-6401 that holds
  if (g.xlo && g.ylo) slabs[n++] = {2, 2, 4, Ny - 2, 4, Nz - 4, 0};
  else if (g.xlo && g.yhi) slabs[n++] = {2, 2, 2, Ny - 2, 4, Nz - 4, 0};
  else if (g.xhi && g.ylo) slabs[n++] = {Nx, 2, 4, Ny - 2, 4, Nz - 4, 0};
  else if (g.xhi && g.yhi) slabs[n++] = {Nx, 2, 2, Ny - 2, 4, Nz - 4, 0};
  else if (g.xlo) slabs[n++] = {2, 2, 2, Ny, 4, Nz - 4, 0};
  else if (g.xhi) slabs[n++] = {Nx, 2, 2, Ny, 4, Nz - 4, 0};
  return n;
}

template <typename real>
int do_source(pic_ctx* c, int s, const Slab* slabs, int nslab, int init_form = 0) {
  const SourceParams sp = source_params(c, s, slabs, nslab, init_form);
  const long long total = sp.total;
  if (total == 0) return PIC_OK;
  Store& st = c->sp[s];
  if (st.count + total > st.cap) return PIC_ERR_CAPACITY;
  source_kernel<real><<<grid_blocks(total), kThreads, 0, c->stream>>>(parts<real>(c, s), sp, c->err);
  CKL();
  c->ctr_p += 3 * total;
  c->ctr_v += 6 * total;
  return set_count(c, s, st.count + total);
}

__global__ void grow_count_kernel(int* count, long long add, int cap) {
  const long long n = (long long)*count + add;
  *count = (int)(n < cap ? n : (long long)cap);
}

// do_source for a species whose count is known only on the device: the
// particles go after the device count, a slot past the capacity is not written
// (counted as ERR_STORE_FULL, which pic_status reports), and the count grows on
// the device; the host's copy stays pending.
template <typename real>
int do_source_dev(pic_ctx* c, int s, const Slab* slabs, int nslab) {
  SourceParams sp = source_params(c, s, slabs, nslab, 0);
  const long long total = sp.total;
  if (total == 0) return PIC_OK;
  Store& st = c->sp[s];
  sp.dst_dev = st.count_dev;
  sp.cap = (int)st.cap;
  source_kernel<real><<<grid_blocks(total), kThreads, 0, c->stream>>>(parts<real>(c, s), sp, c->err);
  CKL();
  grow_count_kernel<<<1, 1, 0, c->stream>>>(st.count_dev, total, (int)st.cap);
  CKL();
  c->ctr_p += 3 * total;
  c->ctr_v += 6 * total;
  return PIC_OK;
}


// add_*_flat: the shell deletion, then the refill appended (the next step's
// re-layout moves it into the layout). With `fused` (pic_step, whose re-layout
// follows in the same step), the deletion over a species' layout is left to
// that re-layout's classify pass, which reads every slot of the layout anyway;
// the slots after the layout are cleared here.
template <typename real>
int do_add_flat(pic_ctx* c, bool fused = false) {
  Slab slabs[5];
  const int nslab = refill_slabs(c, slabs);
  for (int s = 0; s < 2; ++s) {
    Store& st = c->sp[s];
    const Parts<real> P = parts<real>(c, s);
    const bool defer = fused && c->layout[s] && !c->cfg.slot_order;
    // in pic_step, with the count still on the device, nothing here needs the
    // host's copy, so the step does not wait for the device to drain (a
    // pending spill read-back is acted on at the start of a later step)
    const bool nowait = defer && st.pending;
    if (!nowait) {
      CKR(check_spill<real>(c, s, true));
      CKR(sync_count(c, s));
    }
    const long long first = defer ? c->tiled_end[s] : 0;
    if (nowait || st.count > first) {
      delete_shell_kernel<real><<<particle_blocks((nowait ? st.cap : st.count) - first), kThreads, 0, c->stream>>>(
          P, (int)first, st.count_dev, c->g);
      CKL();
    }
    if (defer) {
      st.shell_pending = true;
      c->tiled[s] = false;  // the re-layout runs this step, refill or not
    }
    // appended; the re-layout that follows places them
    CKR(nowait ? do_source_dev<real>(c, s, slabs, nslab) : do_source<real>(c, s, slabs, nslab));
  }
  return PIC_OK;
}

template <typename real>
int do_init_particles(pic_ctx* c) {
  // init_particle_flat :412-625: Np per cell over the interior, cell order
  // (k outermost, m fastest) plus the reference's extra particle, which the
  // loop places in cell (Nx, 0, 0) of the interior numbering.
  c->ctr_p = 0;
  c->ctr_v = 0;
  for (int s = 0; s < 2; ++s) {
    CKR(set_count(c, s, 0));
    c->tiled[s] = false;
    c->layout[s] = false;
    const Slab body = {2, c->cfg.nx, 2, c->cfg.ny, 2, c->cfg.nz, 0};
    const Slab extra_cell = {2 + c->cfg.nx, 1, 2, 1, 2, 1, 0};
    CKR(do_source<real>(c, s, &body, 1, 1));
    // the extra particle: one draw set from the same streams
    SourceParams sp{};
    sp.init_form = 1;
    sp.nslab = 1;
    sp.slab[0] = extra_cell;
    sp.np = 1;
    sp.total = 1;
    const double T = s == 0 ? c->cfg.ti : c->cfg.te;
    const double sig = std::sqrt(c->cfg.kb * T / species_mass(c, s));
    sp.dx = c->cfg.dx;
    sp.lsig = std::sqrt(sig * sig);
    sp.vdrift = c->cfg.v_drift;
    sp.seed_p = c->cfg.seed_p;
    sp.seed_v = c->cfg.seed_v;
    sp.base_p = c->ctr_p;
    sp.base_v = c->ctr_v;
    sp.dst = (int)c->sp[s].count;
    if (c->sp[s].count + 1 > c->sp[s].cap) return PIC_ERR_CAPACITY;
    source_kernel<real><<<1, 32, 0, c->stream>>>(parts<real>(c, s), sp, c->err);
    CKL();
    c->ctr_p += 3;
    c->ctr_v += 6;
    CKR(set_count(c, s, c->sp[s].count + 1));
  }
  return PIC_OK;
}

// -------------------------------------------------------- diagnostics
template <typename real>
int do_thrust_sums(pic_ctx* c) {
  CK(cudaMemsetAsync(c->acc, 0, sizeof(double) * 33, c->stream));
  const pic_config& k = c->cfg;
  CellBox b{};
  const int n3[3] = {c->g.gnx, c->g.gny, k.nz};  // PROCESS_N Grid_N (:4971-4973)
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = n3[a] * 0.2;
    b.hi[a] = n3[a] * 0.8;
  }
  b.e0 = k.e0;
  b.inv_mu0 = 1.0 / k.mu0;
  b.ox = c->g.ox;
  b.oy = c->g.oy;
  const long long nint = (long long)k.nx * k.ny * k.nz;
  field_energy_kernel<real><<<particle_blocks(nint), kThreads, 0, c->stream>>>(fields<real>(c), c->g, b, c->acc);
  CKL();
  for (int s = 0; s < 2; ++s) {
    if (slot_bound(c, s) == 0) continue;
    ThrustParams tp{};
    tp.xlo = (double)c->g.gnx * k.dx * 0.2; tp.xhi = (double)c->g.gnx * k.dx * 0.8;
    tp.ylo = (double)c->g.gny * k.dx * 0.2; tp.yhi = (double)c->g.gny * k.dx * 0.8;
    tp.zlo = (double)k.nz * k.dx * 0.2; tp.zhi = (double)k.nz * k.dx * 0.8;
    tp.ox = (double)c->g.ox * k.dx;
    tp.oy = (double)c->g.oy * k.dx;
    tp.dx = k.dx;
    const double sg = s == 0 ? 1.0 : -1.0;
    const double w = k.q * species_weight(c) * k.dx * k.dx * k.dx;
    const int o = s == 0 ? 3 : 9;
    for (int q = 0; q < 3; ++q) { tp.idx[q] = q; tp.scale[q] = sg * w; }
    for (int q = 0; q < 6; ++q) { tp.idx[3 + q] = o + q; tp.scale[3 + q] = sg * w; }
    tp.idx[9] = 27 + (s == 0 ? 2 : 3);
    tp.scale[9] = 0.5 * species_mass(c, s) * species_weight(c) * k.dx * k.dx * k.dx;
    thrust_particles_kernel<real><<<particle_blocks(slot_bound(c, s)), kThreads, 0, c->stream>>>(
        parts<real>(c, s), c->sp[s].count_dev, fields<real>(c), c->g, tp, c->acc);
    CKL();
  }
  // thrust_f's MPI_Allreduce of F and E over the ranks (:5103-5108)
  if (c->has_xport && c->xport.allreduce_sum_f64(c->xport.user, c->acc, 33, (void*)c->stream) != 0) return PIC_ERR_COMM;
  return PIC_OK;
}

template <typename real>
int do_gauss(pic_ctx* c, double* out4) {
  CK(cudaMemsetAsync(c->acc + 40, 0, sizeof(double) * 4, c->stream));
  CK(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned long long), c->stream));
  const long long nint = (long long)c->g.nx * c->g.ny * c->g.nz;
  gauss_kernel<real><<<particle_blocks(nint), kThreads, 0, c->stream>>>(
      fields<real>(c), c->g, 1.0 / (24.0 * c->cfg.dx), c->cfg.q / c->cfg.e0, c->acc + 40, c->maxbits);
  CKL();
  double h[4];
  unsigned long long mb = 0;
  CK(cudaMemcpyAsync(h, c->acc + 40, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&mb, c->maxbits, sizeof(mb), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double mx;
  std::memcpy(&mx, &mb, sizeof(mx));
  out4[0] = h[0];
  out4[1] = h[1];
  out4[2] = mx;
  out4[3] = h[3];
  return PIC_OK;
}

// ------------------------------------------------------------ a step
template <typename real>
int do_step(pic_ctx* c) {
  // a placement's spill count that has landed is acted on without waiting
  for (int s = 0; s < 2; ++s) CKR(check_spill<real>(c, s, false));
  CKR(phase_mark(c, PH_FIELD));
  CKR(do_renew_grid(c));
  CKR(phase_mark(c, PH_FIELD));
  if (c->c_thrust > c->cfg.sort_interval - 1) {
    c->c_thrust = 0;
    // sorting (:696-697) only reorders particles, for locality. The tiled
    // layout is already refreshed by the re-layout after every refill, so the
    // periodic sort runs only when that has not happened for half a sort
    // interval.
    if (!c->cfg.slot_order && c->since_layout >= std::max(1, c->cfg.sort_interval / 2)) {
      CKR(phase_mark(c, PH_SORT));
      CKR(do_sort<real>(c));
      CKR(phase_mark(c, PH_SORT));
    }
  }
  if (c->c_add > c->cfg.add_interval - 1) {
    CKR(phase_mark(c, PH_ADD));
    CKR(do_add_flat<real>(c, true));
    CKR(phase_mark(c, PH_ADD));
    c->c_add = 0;
  }
  CKR(phase_mark(c, PH_FIELD));
  CKR(do_renew_b<real>(c));
  CKR(phase_mark(c, PH_FIELD));
  // a re-layout after a refill or an import
  const bool which[2] = {!c->cfg.slot_order && !c->tiled[0], !c->cfg.slot_order && !c->tiled[1]};
  if (which[0] || which[1]) {
    CKR(phase_mark(c, PH_SORT));
    CKR(relayout_species<real>(c, which));
    if (which[0] && which[1]) c->since_layout = 0;
    CKR(phase_mark(c, PH_SORT));
  }
  CKR(phase_mark(c, PH_PUSH));
  if (c->has_xport) CKR(resolve_counts<real>(c));  // the exchange lists are sized from the counts
  if (c->has_xport) CKR(ensure_mig<real>(c));
  // the counts stay on the device: the push and the diagnostics cover the
  // slots up to the capacity and stop at the device count, and the host reads
  // a count back only when an entry point needs it
  for (int s = 0; s < 2; ++s) CKR(do_push_tiled<real>(c, s));
  if (c->has_xport) CKR(do_migrate<real>(c));  // sr_particle's exchange between ranks
  CKR(phase_mark(c, PH_PUSH));
  CKR(phase_mark(c, PH_FIELD));
  CKR(do_renew_b<real>(c));
  CKR(do_fold<real>(c));
  CKR(do_renew_e<real>(c));
  if (c->cfg.poisson_clean) CKR(do_poisson<real>(c));
  CKR(phase_mark(c, PH_FIELD));
  if (c->cfg.diag_every_step) {
    CKR(phase_mark(c, PH_DIAG));
    CKR(do_thrust_sums<real>(c));
    fave_accumulate_kernel<<<1, 32, 0, c->stream>>>(c->acc, c->fave, 1.0 / 500.0);
    CKL();
    CKR(phase_mark(c, PH_DIAG));
  }
  c->c_add++;
  c->c_thrust++;
  c->since_layout++;
  return PIC_OK;
}

// --------------------------------------------------------- import/export
// The staging buffer grows with an eighth of headroom, so that a particle
// count that grows by a refill between two exports does not reallocate it.
int ensure_stage(pic_ctx* c, size_t bytes) {
  if (bytes <= c->stage_bytes) return PIC_OK;
  if (c->stage) CK(cudaFree(c->stage));
  c->stage = nullptr;
  c->stage_bytes = 0;
  const size_t want = bytes + bytes / 8;
  CK(cudaMalloc(&c->stage, want));
  c->stage_bytes = want;
  return PIC_OK;
}

// Flags and positions of the export's compaction: sized once for the larger
// particle store, since the count changes every refill.
int ensure_flags(pic_ctx* c, size_t n) {
  if (n <= c->flags_len) return PIC_OK;
  if (c->flags) CK(cudaFree(c->flags));
  if (c->pos) CK(cudaFree(c->pos));
  c->flags = c->pos = nullptr;
  c->flags_len = 0;
  const size_t want = std::max<size_t>(n, (size_t)std::max(c->sp[0].cap, c->sp[1].cap));
  CK(cudaMalloc(&c->flags, sizeof(int) * want));
  CK(cudaMalloc(&c->pos, sizeof(int) * want));
  c->flags_len = want;
  return PIC_OK;
}

template <typename real>
int do_export(pic_ctx* c, int s, double* rows, long long cap, long long* n_out) {
  Store& st = c->sp[s];
  const long long n = st.count;
  if (n == 0) {
    *n_out = 0;
    return PIC_OK;
  }
  CKR(ensure_flags(c, (size_t)n));
  live_flag_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(parts<real>(c, s), (int)n, c->flags);
  CKL();
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  std::vector<int> dummy;
  int* tmp = nullptr;
  CK(cudaMalloc(&tmp, sizeof(int) * (size_t)(2 * tiles + 64)));
  int rc = scan_exclusive(c, c->flags, c->pos, n, tmp, (size_t)(2 * tiles + 64));
  if (rc != PIC_OK) {
    cudaFree(tmp);
    return rc;
  }
  int last_pos = 0, last_flag = 0;
  CK(cudaMemcpyAsync(&last_pos, c->pos + n - 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&last_flag, c->flags + n - 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaFree(tmp));
  const long long live = (long long)last_pos + last_flag;
  *n_out = live;
  if (rows == nullptr || cap <= 0 || live == 0) return PIC_OK;
  CKR(ensure_stage(c, sizeof(double) * 7 * (size_t)live));
  export_rows_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(
      parts<real>(c, s), (int)n, c->pos, c->cfg.dx, species_weight(c), (double*)c->stage);
  CKL();
  const long long ncopy = live < cap ? live : cap;
  CK(cudaMemcpyAsync(rows, c->stage, sizeof(double) * 7 * (size_t)ncopy, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

template <typename real>
int do_import(pic_ctx* c, int s, const double* rows, const int* flag, long long n) {
  Store& st = c->sp[s];
  if (n > st.cap) return PIC_ERR_CAPACITY;
  if (n > 0) {
    CKR(ensure_stage(c, sizeof(double) * 7 * (size_t)n));
    CK(cudaMemcpyAsync(c->stage, rows, sizeof(double) * 7 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    // every row carries the species' weight and flag 1: checked on the device
    // before the store changes (a host loop over the rows would read them all
    // a second time through the host's memory)
    const int* fdev = nullptr;
    if (flag) {
      CKR(ensure_flags(c, (size_t)n));
      CK(cudaMemcpyAsync(c->flags, flag, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
      fdev = c->flags;
    }
    const double w = species_weight(c);
    CK(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned long long), c->stream));
    import_check_kernel<<<particle_blocks(n), kThreads, 0, c->stream>>>((const double*)c->stage, n, w,
                                                                        1e-12 * std::fabs(w), fdev, c->maxbits);
    CKL();
    unsigned long long bad = 0;
    CK(cudaMemcpyAsync(&bad, c->maxbits, sizeof(bad), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad) return PIC_ERR_ARG;
    import_rows_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(parts<real>(c, s), (int)n,
                                                                         (const double*)c->stage, c->cfg.dx, c->err);
    CKL();
  }
  CKR(set_count(c, s, n));
  c->tiled[s] = false;
  c->layout[s] = false;
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

template <typename real>
__global__ void grid_export_kernel(Fields<real> F, int nodes, double* rec) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nodes) return;
  double* r = rec + 18 * (long long)n;
  const int map[17] = {F_BX, F_BY, F_BZ, F_B0X, F_B0Y, F_B0Z, F_EX, F_EY, F_EZ,
                       F_JIX, F_JIY, F_JIZ, F_JEX, F_JEY, F_JEZ, F_NI, F_NE};
#pragma unroll
  for (int q = 0; q < 17; ++q) r[q] = (double)F.f[map[q]][n];
  r[17] = (double)F.f[F_PHI][n];
}

template <typename real>
__global__ void grid_import_kernel(Fields<real> F, int nodes, const double* rec) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nodes) return;
  const double* r = rec + 18 * (long long)n;
  const int map[17] = {F_BX, F_BY, F_BZ, F_B0X, F_B0Y, F_B0Z, F_EX, F_EY, F_EZ,
                       F_JIX, F_JIY, F_JIZ, F_JEX, F_JEY, F_JEZ, F_NI, F_NE};
#pragma unroll
  for (int q = 0; q < 17; ++q) F.f[map[q]][n] = (real)r[q];
  F.f[F_PHI][n] = (real)r[17];
  F.f[F_DBX][n] = (real)(r[0] - r[3]);
  F.f[F_DBY][n] = (real)(r[1] - r[4]);
  F.f[F_DBZ][n] = (real)(r[2] - r[5]);
}

template <typename real>
int do_get_grid(pic_ctx* c, double* records) {
  const size_t bytes = sizeof(double) * 18 * (size_t)c->g.nodes;
  CKR(ensure_stage(c, bytes));
  grid_export_kernel<real><<<grid_blocks(c->g.nodes), kThreads, 0, c->stream>>>(fields<real>(c), c->g.nodes,
                                                                                (double*)c->stage);
  CKL();
  CK(cudaMemcpyAsync(records, c->stage, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

template <typename real>
int do_set_grid(pic_ctx* c, const double* records) {
  const size_t bytes = sizeof(double) * 18 * (size_t)c->g.nodes;
  CKR(ensure_stage(c, bytes));
  CK(cudaMemcpyAsync(c->stage, records, bytes, cudaMemcpyHostToDevice, c->stream));
  grid_import_kernel<real><<<grid_blocks(c->g.nodes), kThreads, 0, c->stream>>>(fields<real>(c), c->g.nodes,
                                                                                (const double*)c->stage);
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

#include "adjoint_run.cuh"

// nsteps slot-stable loop bodies from the current state with the objective;
// with `grad`, the reverse pass as well. out = {J, dJ/dI, dJ/dV}.
template <typename real>
int do_adjoint(pic_ctx* c, int nsteps, int every, bool grad, double* out) {
  AdjRun R;
  std::vector<AdjSnap> ck;
  std::vector<AdjSnap> last;  // the last segment's step inputs, kept by the forward sweep
  AdjSnap fin;
  auto run = [&]() -> int {
    const long long capmax = c->sp[0].cap > c->sp[1].cap ? c->sp[0].cap : c->sp[1].cap;
    // the scan serves the compaction's counts over nodes + 1 keys
    const long long scan_n = capmax > (long long)c->g.nodes + 1 ? capmax : (long long)c->g.nodes + 1;
    R.scan_len = (size_t)(2 * ((scan_n + kScanTile - 1) / kScanTile) + 64);
    CKR(adj_alloc(c, R, (void**)&R.scan_tmp, sizeof(int) * R.scan_len));
    for (int b = 0; b < 2; ++b) {
      CKR(adj_alloc(c, R, (void**)&R.skey[b], sizeof(int) * (size_t)capmax));
      CKR(adj_alloc(c, R, (void**)&R.sslot[b], sizeof(int) * (size_t)capmax));
    }
    CKR(adj_alloc(c, R, (void**)&R.kcnt, sizeof(int) * ((size_t)c->g.nodes + 1)));
    CKR(adj_alloc(c, R, (void**)&R.kpos, sizeof(int) * ((size_t)c->g.nodes + 1)));
    CKR(adj_alloc(c, R, (void**)&R.acc, sizeof(double) * 4));
    CKR(adj_alloc(c, R, (void**)&R.j64, sizeof(unsigned long long) * 3 * (size_t)c->g.nodes));
    CK(cudaMemsetAsync(R.acc, 0, sizeof(double) * 4, c->stream));
    // forward sweep, keeping a checkpoint every `every` steps and the step
    // inputs of the last segment, which the reverse pass then need not recompute
    const int last0 = ((nsteps - 1) / every) * every;
    if (grad) last.resize((size_t)(nsteps - last0));
    for (int n = 0; n < nsteps; ++n) {
      if (grad && n % every == 0) {
        ck.emplace_back();
        CKR(adj_save<real>(c, ck.back()));
      }
      AdjSnap* rec = grad && n >= last0 ? &last[(size_t)(n - last0)] : nullptr;
      CKR(adj_forward_step<real>(c, R, rec, true, n == nsteps - 1));
    }
    double h[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(h, R.acc, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out[0] = h[0];
    if (!grad) return PIC_OK;
    CKR(adj_save<real>(c, fin));
    // the final J and n planes, which the recomputed segments overwrite
    CKR(adj_alloc(c, R, &R.jn_final, 8 * c->plane_bytes));
    CK(cudaMemcpyAsync(R.jn_final, (char*)c->field_mem + (size_t)F_JIX * c->plane_bytes, 8 * c->plane_bytes,
                       cudaMemcpyDeviceToDevice, c->stream));
    // adjoint state: zero for the final state (the objective terms enter in the reverse kernels)
    for (int s = 0; s < 2; ++s)
      for (int b = 0; b < 2; ++b) {
        const size_t bytes = 6 * align256((size_t)c->sp[s].cap * sizeof(real));
        CKR(adj_alloc(c, R, &R.lam[s][b], bytes));
        CK(cudaMemsetAsync(R.lam[s][b], 0, bytes, c->stream));
      }
    CKR(adj_alloc(c, R, &R.lfield, 12 * c->plane_bytes));
    CK(cudaMemsetAsync(R.lfield, 0, 12 * c->plane_bytes, c->stream));
    CKR(adj_alloc(c, R, &R.tdb, 3 * c->plane_bytes));
    CK(cudaMemsetAsync(R.tdb, 0, 3 * c->plane_bytes, c->stream));
    CK(cudaMemsetAsync(R.acc, 0, sizeof(double) * 4, c->stream));
    for (int seg = (int)ck.size() - 1; seg >= 0; --seg) {
      const int n0 = seg * every, n1 = n0 + every < nsteps ? n0 + every : nsteps;
      std::vector<AdjSnap> rec;
      int rc = PIC_OK;
      if (n0 == last0) {
        rec.swap(last);
      } else {
        CKR(adj_restore<real>(c, ck[seg]));
        rec.resize((size_t)(n1 - n0));
        for (int n = n0; n < n1 && rc == PIC_OK; ++n) rc = adj_forward_step<real>(c, R, &rec[n - n0], false, false);
      }
      for (int n = n1 - 1; n >= n0 && rc == PIC_OK; --n) {
        rc = adj_reverse_step<real>(c, R, rec[n - n0]);
        if (rc == PIC_OK) rc = adj_unrefill<real>(c, R, rec[n - n0]);
      }
      for (auto& S : rec) snap_free(c, S);
      if (seg > 0) snap_free(c, ck[seg]);  // the first checkpoint's particles serve the drift gradient below
      if (rc != PIC_OK) return rc;
    }
    // the initial particles were created with vz = V + thermal
    for (int s = 0; s < 2; ++s) {
      const long long n = ck[0].count[s];
      if (n == 0) continue;
      const AdjPart<real> A = adj_part<real>(c, R, s, R.lcur[s]);
      drift_grad_kernel<real><<<particle_blocks(n), kThreads, 0, c->stream>>>(
          parts_at<real>(ck[0].part[s], ck[0].slots[s]), A.lv[2], 0, (int)n, R.acc);
      CKL();
    }
    CK(cudaMemcpyAsync(h, R.acc, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out[1] = h[1];
    out[2] = h[2];
    CK(cudaMemcpyAsync((char*)c->field_mem + (size_t)F_JIX * c->plane_bytes, R.jn_final, 8 * c->plane_bytes,
                       cudaMemcpyDeviceToDevice, c->stream));
    return adj_restore<real>(c, fin);
  };
  const int rc = run();
  cudaStreamSynchronize(c->stream);
  for (auto& S : ck) snap_free(c, S);
  for (auto& S : last) snap_free(c, S);
  snap_free(c, fin);
  adj_free(c, R);
  return rc;
}

// Dispatch on the context's precision.
#define DISPATCH(c, call)                      \
  ((c)->prec == 64 ? call<double> : call<float>)

// Every entry point starts here: the context's device, and, unless the entry
// point works with counts that only the device knows (pic_step, pic_fdtd),
// the particle counts that earlier steps left on the device read back.
int check_ctx(pic_ctx* c, bool resolve = true) {
  if (!c) return PIC_ERR_ARG;
  if (cudaSetDevice(c->cfg.device) != cudaSuccess) return PIC_ERR_CUDA;
  if (resolve && (c->sp[0].pending || c->sp[1].pending || c->sp[0].spill_pending || c->sp[1].spill_pending))
    CKR(DISPATCH(c, resolve_counts)(c));
  return PIC_OK;
}

double ramp_value(int idx, int n_total, int absorb) {
  if (idx - 4 <= 2 * absorb) return (2 * absorb - (idx - 4)) / 4.;
  if (idx - 4 >= 2 * n_total - 2 * absorb) return (idx - 4 - (2 * n_total - 2 * absorb)) / 4.;
  return 0.;
}

}  // namespace

// ================================================================= C ABI
extern "C" {

const char* pic_error_string(int code) {
  switch (code) {
    case PIC_OK: return "ok";
    case PIC_ERR_ARG: return "invalid argument";
    case PIC_ERR_CUDA: return "CUDA error";
    case PIC_ERR_CAPACITY: return "particle capacity exceeded";
    case PIC_ERR_STATE: return "call out of order";
    case PIC_ERR_DEVICE: return "device counters report lost work";
    case PIC_ERR_TOO_LARGE: return "input larger than the fixed-size scratch allows";
    case PIC_ERR_COMM: return "an exchange between ranks failed";
    default: return "unknown error";
  }
}

int pic_config_default(pic_config* k, int nx, int ny, int nz) {
  if (!k) return PIC_ERR_ARG;
  std::memset(k, 0, sizeof(*k));
  k->nx = nx; k->ny = ny; k->nz = nz;
  k->np = 16;
  k->precision = 32;
  k->device = 0;
  k->dx = 1.5; k->dt = 1.5e-9;
  k->q = 1.602176487e-19;
  k->mi = 1.672621637e-27;
  k->me = k->mi / 100.;
  k->mu0 = 1.25663706144e-6;
  k->e0 = 8.854187817e-12;
  k->kb = 1.3806504e-23;
  k->c = 2.99792458e8;
  k->v_drift = 1.2e7;
  k->n_all = 5e10;
  k->ti = 1e9; k->te = 1e9;
  k->coil_r = 2.;
  k->coil_i = 6.8e7;
  k->alpha = M_PI / 2.;
  k->absorb_grid = 32;
  k->absorb_grid2 = 40;
  k->sigma_a = 1e-6;
  k->dipole_cutoff = 210.;
  k->add_interval = 5;
  k->sort_interval = 500;
  k->procs_x = k->procs_y = 1;  // PROCESS_Nx x PROCESS_Ny = 1 x 1: a single domain
  k->diag_every_step = 1;
  k->poisson_clean = 0;
  k->absorb_grid3 = 40;
  k->capacity = 0;
  k->seed_p = 0;
  k->seed_v = 50;
  return PIC_OK;
}

int pic_create(const pic_config* cfg, pic_ctx** out) {
  if (!cfg || !out) return PIC_ERR_ARG;
  *out = nullptr;
  const pic_config& k = *cfg;
  if (k.nx < 5 || k.ny < 5 || k.nz < 5 || k.nx + 4 > kMaxDim || k.ny + 4 > kMaxDim || k.nz + 4 > kMaxDim)
    return PIC_ERR_ARG;
  if (k.np < 1 || !(k.dx > 0) || !(k.dt > 0) || !(k.c > 0) || !(k.mi > 0) || !(k.me > 0)) return PIC_ERR_ARG;
  if (k.precision != 32 && k.precision != 64) return PIC_ERR_ARG;
  if (k.slot_order != 0 && k.slot_order != 1) return PIC_ERR_ARG;
  if (k.add_interval < 1 || k.sort_interval < 1) return PIC_ERR_ARG;
  if (k.absorb_grid3 < 0 || (k.poisson_clean != 0 && k.poisson_clean != 1)) return PIC_ERR_ARG;
  if (k.procs_x < 1 || k.procs_y < 1 || k.rank_x < 0 || k.rank_y < 0 || k.rank_x >= k.procs_x ||
      k.rank_y >= k.procs_y)
    return PIC_ERR_ARG;
  if ((k.procs_x > 1 || k.procs_y > 1) && k.poisson_clean) return PIC_ERR_ARG;  // single domain only
  if (cudaSetDevice(k.device) != cudaSuccess) return PIC_ERR_CUDA;
  pic_ctx* c = new (std::nothrow) pic_ctx();
  if (!c) return PIC_ERR_ARG;
  c->cfg = k;
  c->prec = k.precision;
  c->rsize = k.precision == 64 ? 8 : 4;
  Geom& g = c->g;
  g.nx = k.nx; g.ny = k.ny; g.nz = k.nz;
  g.gx = k.nx + 4; g.gy = k.ny + 4; g.gz = k.nz + 4;
  g.sx = g.gy * g.gz;
  g.nodes = g.gx * g.gy * g.gz;
  g.ox = k.rank_x * k.nx;
  g.oy = k.rank_y * k.ny;
  g.gnx = k.procs_x * k.nx;
  g.gny = k.procs_y * k.ny;
  g.xlo = k.rank_x == 0;
  g.xhi = k.rank_x == k.procs_x - 1;
  g.ylo = k.rank_y == 0;
  g.yhi = k.rank_y == k.procs_y - 1;
  c->ncells = (long long)k.nx * k.ny * k.nz;
  auto fail = [&](int code) {
    pic_destroy(c);
    cudaGetLastError();  // a failed allocation must not fail the next context's launch checks
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMallocHost(&c->host_pin, sizeof(int) * 16) != cudaSuccess) return fail(PIC_ERR_CUDA);
  for (int s = 0; s < 2; ++s)
    if (cudaEventCreateWithFlags(&c->sp[s].readback, cudaEventDisableTiming) != cudaSuccess) return fail(PIC_ERR_CUDA);
  c->plane_bytes = align256((size_t)g.nodes * c->rsize);
  if (cudaMalloc(&c->field_mem, c->plane_bytes * F_COUNT) != cudaSuccess) return fail(PIC_ERR_CUDA);
  cudaMemsetAsync(c->field_mem, 0, c->plane_bytes * F_COUNT, c->stream);
  // damping ramps of init_grid (:336-365) per axis on the doubled grid
  {
    std::vector<double> h(2 * (g.gx + g.gy + g.gz));
    // k + 2 myrank_x Grid_Nx on the doubled grid of PROCESS_Nx Grid_Nx cells (:338-349)
    for (int i = 0; i < 2 * g.gx; ++i) h[i] = ramp_value(i + 2 * g.ox, g.gnx, k.absorb_grid);
    for (int i = 0; i < 2 * g.gy; ++i) h[2 * g.gx + i] = ramp_value(i + 2 * g.oy, g.gny, k.absorb_grid);
    for (int i = 0; i < 2 * g.gz; ++i) h[2 * (g.gx + g.gy) + i] = ramp_value(i, k.nz, k.absorb_grid);
    if (cudaMalloc(&c->ramps, sizeof(double) * h.size()) != cudaSuccess) return fail(PIC_ERR_CUDA);
    if (cudaMemcpy(c->ramps, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(PIC_ERR_CUDA);
  }
  if (c->prec == 64) setup_staged_fields<double>(c);
  else setup_staged_fields<float>(c);
  const bool tiled = k.slot_order == 0;
  long long cap = k.capacity;
  if (cap <= 0) {
    // the tiled layout gives every lane column room for its fullest cell plus
    // a refill reserve (refill_reserve): about np + 3 sqrt(np) + 2 slots per
    // cell, plus an eighth, plus 4; a few more for the unplaced tail. Slot
    // order keeps the initial load and the refills of about 100 steps.
    const double per_cell = tiled ? 1.125 * (k.np + 3.0 * std::sqrt((double)k.np) + 2.0) + 6.0 : 1.8 * k.np;
    cap = (long long)(per_cell * k.nx * k.ny * k.nz) + 65536;
  }
  if (cap > 0x7fffffffLL) return fail(PIC_ERR_ARG);
  for (int s = 0; s < 2; ++s) {
    c->sp[s].cap = cap;
    for (int b = 0; b < (tiled ? 2 : 1); ++b)
      if (cudaMalloc(&c->sp[s].mem[b], store_bytes(cap, c->rsize)) != cudaSuccess) return fail(PIC_ERR_CUDA);
    if (cudaMalloc(&c->sp[s].count_dev, sizeof(int)) != cudaSuccess) return fail(PIC_ERR_CUDA);
    cudaMemsetAsync(c->sp[s].count_dev, 0, sizeof(int), c->stream);
  }
  if (cudaMalloc(&c->cnt, sizeof(int) * c->ncells) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMalloc(&c->offs, sizeof(int) * c->ncells) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMalloc(&c->cursor, sizeof(int) * c->ncells) != cudaSuccess) return fail(PIC_ERR_CUDA);
  c->scan_tmp_len = (size_t)(c->ncells / kScanTile) * 2 + 64;
  if (cudaMalloc(&c->scan_tmp, sizeof(int) * c->scan_tmp_len) != cudaSuccess) return fail(PIC_ERR_CUDA);
  {
    TileGeom& t = c->tg;
    t.ntx = (k.nx + kTileX - 1) / kTileX;
    t.nty = (k.ny + kTileY - 1) / kTileY;
    t.ntz = (k.nz + kLanes - 1) / kLanes;
    t.ngroups = t.ntx * t.nty * t.ntz * kTileX * kTileY;
    for (int s = 0; s < 2; ++s) {
      for (int b = 0; b < 2; ++b) {
        if (cudaMalloc(&c->goff[s][b], sizeof(int) * t.ngroups) != cudaSuccess) return fail(PIC_ERR_CUDA);
        if (cudaMalloc(&c->gmax[s][b], sizeof(int) * t.ngroups) != cudaSuccess) return fail(PIC_ERR_CUDA);
      }
    }
    if (cudaMalloc(&c->gcap, sizeof(int) * t.ngroups) != cudaSuccess) return fail(PIC_ERR_CUDA);
    if (cudaMalloc(&c->total_dev, sizeof(int)) != cudaSuccess) return fail(PIC_ERR_CUDA);
    if (cudaMalloc(&c->append_dev, sizeof(int)) != cudaSuccess) return fail(PIC_ERR_CUDA);
    if (tiled) {  // re-layout scratch
      for (int s = 0; s < 2; ++s) {  // each species' hole lists live from its push to its next placement
        if (cudaMalloc(&c->sp[s].holes, sizeof(int) * (size_t)cap) != cudaSuccess) return fail(PIC_ERR_CUDA);
        if (cudaMalloc(&c->sp[s].nholes, sizeof(int) * c->ncells) != cudaSuccess) return fail(PIC_ERR_CUDA);
        if (cudaMalloc(&c->sp[s].nonhome, sizeof(int)) != cudaSuccess) return fail(PIC_ERR_CUDA);
        cudaMemsetAsync(c->sp[s].nonhome, 0, sizeof(int), c->stream);
      }
      if (cudaMalloc(&c->rank, sizeof(int) * (size_t)cap) != cudaSuccess) return fail(PIC_ERR_CUDA);
      if (cudaMalloc(&c->bucket, sizeof(int) * (size_t)cap) != cudaSuccess) return fail(PIC_ERR_CUDA);
    }
    const int pb_f = (int)PushSmem<float>::bytes, pb_d = (int)PushSmem<double>::bytes;
    if (cudaFuncSetAttribute(push_tiled_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, pb_d) !=
            cudaSuccess ||
        cudaFuncSetAttribute(push_tiled_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, pb_f) !=
            cudaSuccess ||
        cudaFuncSetAttribute(push_tiled_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, pb_f) !=
            cudaSuccess)
      return fail(PIC_ERR_CUDA);
  }
  if (cudaMalloc(&c->acc, sizeof(double) * 64) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMalloc(&c->maxbits, sizeof(unsigned long long)) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMalloc(&c->fave, sizeof(double) * 27) != cudaSuccess) return fail(PIC_ERR_CUDA);
  if (cudaMalloc(&c->err, sizeof(unsigned long long) * ERR_COUNT) != cudaSuccess) return fail(PIC_ERR_CUDA);
  cudaMemsetAsync(c->acc, 0, sizeof(double) * 64, c->stream);
  cudaMemsetAsync(c->fave, 0, sizeof(double) * 27, c->stream);
  cudaMemsetAsync(c->err, 0, sizeof(unsigned long long) * ERR_COUNT, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(PIC_ERR_CUDA);
  *out = c;
  return PIC_OK;
}

int pic_destroy(pic_ctx* c) {
  if (!c) return PIC_OK;
  cudaSetDevice(c->cfg.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->field_mem);
  cudaFree(c->ramps);
  for (void* p : c->adj_pool.all) cudaFree(p);
  if (c->host_pin) cudaFreeHost(c->host_pin);
  for (int s = 0; s < 2; ++s)
    if (c->sp[s].readback) cudaEventDestroy(c->sp[s].readback);
  for (int s = 0; s < 2; ++s) {
    cudaFree(c->sp[s].mem[0]);
    cudaFree(c->sp[s].mem[1]);
    cudaFree(c->sp[s].count_dev);
  }
  for (int s = 0; s < 2; ++s) {
    for (int b = 0; b < 2; ++b) {
      cudaFree(c->goff[s][b]);
      cudaFree(c->gmax[s][b]);
    }
  }
  cudaFree(c->gcap);
  cudaFree(c->total_dev);
  cudaFree(c->append_dev);
  for (int s = 0; s < 2; ++s) {
    cudaFree(c->sp[s].holes);
    cudaFree(c->sp[s].nholes);
    cudaFree(c->sp[s].nonhome);
  }
  cudaFree(c->rank);
  cudaFree(c->bucket);
  cudaFree(c->cnt);
  cudaFree(c->offs);
  cudaFree(c->cursor);
  cudaFree(c->scan_tmp);
  cudaFree(c->acc);
  cudaFree(c->maxbits);
  cudaFree(c->fave);
  cudaFree(c->phi_w);
  cudaFree(c->phi_sines);
  cudaFree(c->phi_sin2);
  cudaFree(c->halo_buf[0]);
  cudaFree(c->halo_buf[1]);
  cudaFree(c->mig);
  cudaFree(c->mig_cnt);
  cudaFree(c->err);
  cudaFree(c->stage);
  cudaFree(c->flags);
  cudaFree(c->pos);
  for (int p = 0; p < 8; ++p)
    for (cudaEvent_t e : c->phase[p].ev) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return PIC_OK;
}

int pic_init_grid(pic_ctx* c) {
  CKR(check_ctx(c));
  CKR(DISPATCH(c, do_init_grid)(c));
  c->grid_ready = true;
  return PIC_OK;
}

int pic_init_particle_flat(pic_ctx* c) {
  CKR(check_ctx(c));
  CKR(DISPATCH(c, do_init_particles)(c));
  c->particles_ready = true;
  return PIC_OK;
}

int pic_renew_grid(pic_ctx* c) {
  CKR(check_ctx(c));
  return do_renew_grid(c);
}

int pic_renew_b4_2(pic_ctx* c) {
  CKR(check_ctx(c));
  return DISPATCH(c, do_renew_b)(c);
}

int pic_renew_e4_2(pic_ctx* c) {
  CKR(check_ctx(c));
  return DISPATCH(c, do_renew_e)(c);
}

int pic_push_deposit_j(pic_ctx* c, int species) {
  CKR(check_ctx(c));
  if (species < -1 || species > 1) return PIC_ERR_ARG;
  for (int s = 0; s < 2; ++s) {
    if (species >= 0 && s != species) continue;
    CKR((c->prec == 64 ? do_push<double, PUSH_J>(c, s) : do_push<float, PUSH_J>(c, s)));
  }
  return PIC_OK;
}

int pic_drift_deposit_n(pic_ctx* c, int species) {
  CKR(check_ctx(c));
  if (species < -1 || species > 1) return PIC_ERR_ARG;
  for (int s = 0; s < 2; ++s) {
    if (species >= 0 && s != species) continue;
    CKR((c->prec == 64 ? do_drift_n<double>(c, s) : do_drift_n<float>(c, s)));
  }
  return PIC_OK;
}

int pic_reduce_current(pic_ctx* c) {
  CKR(check_ctx(c));
  return DISPATCH(c, do_fold)(c);
}

int pic_sr_particle(pic_ctx* c) {
  CKR(check_ctx(c));
  return DISPATCH(c, do_sr_particle)(c);
}

int pic_add_flat(pic_ctx* c) {
  CKR(check_ctx(c));
  return DISPATCH(c, do_add_flat)(c, false);
}

int pic_sort(pic_ctx* c) {
  CKR(check_ctx(c));
  if (c->cfg.slot_order) return PIC_OK;  // slot order: sorting only reorders, so there is nothing to do
  return DISPATCH(c, do_sort)(c);
}

int pic_thrust_f(pic_ctx* c, double* F27, double* E6) {
  CKR(check_ctx(c));
  CKR(DISPATCH(c, do_thrust_sums)(c));
  double h[33];
  CK(cudaMemcpyAsync(h, c->acc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (F27) std::memcpy(F27, h, sizeof(double) * 27);
  if (E6) std::memcpy(E6, h + 27, sizeof(double) * 6);
  return PIC_OK;
}

int pic_thrust_fave(pic_ctx* c, double* Fave27, int reset) {
  CKR(check_ctx(c));
  if (Fave27) {
    CK(cudaMemcpyAsync(Fave27, c->fave, sizeof(double) * 27, cudaMemcpyDeviceToHost, c->stream));
  }
  if (reset) CK(cudaMemsetAsync(c->fave, 0, sizeof(double) * 27, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

int pic_set_transport(pic_ctx* c, const pic_transport* t) {
  CKR(check_ctx(c));
  if (!t || !t->sendrecv || !t->allreduce_sum_f64) return PIC_ERR_ARG;
  if (c->cfg.poisson_clean) return PIC_ERR_STATE;
  c->xport = *t;
  c->has_xport = true;
  return PIC_OK;
}

int pic_poisson_clean(pic_ctx* c) {
  CKR(check_ctx(c));
  if (!c->grid_ready) return PIC_ERR_STATE;
  if (c->has_xport || c->cfg.procs_x * c->cfg.procs_y > 1) return PIC_ERR_STATE;  // single domain only
  return DISPATCH(c, do_poisson)(c);
}

int pic_objective(pic_ctx* c, int nsteps, double* J) {
  CKR(check_ctx(c));
  if (!J || nsteps < 0) return PIC_ERR_ARG;
  if (c->cfg.slot_order) return PIC_ERR_ARG;  // its compaction needs the second record buffer
  if (c->cfg.poisson_clean) return PIC_ERR_ARG;  // the adjoint does not differentiate the cleaning
  if (c->has_xport || c->cfg.procs_x * c->cfg.procs_y > 1) return PIC_ERR_ARG;  // single domain only
  if (!c->grid_ready) return PIC_ERR_STATE;
  double out[3] = {0, 0, 0};
  CKR(DISPATCH(c, do_adjoint)(c, nsteps, 1, false, out));
  *J = out[0];
  return PIC_OK;
}

int pic_adjoint(pic_ctx* c, int nsteps, int checkpoint_every, double* out3) {
  CKR(check_ctx(c));
  if (!out3 || nsteps < 1 || checkpoint_every < 1) return PIC_ERR_ARG;
  if (c->cfg.slot_order) return PIC_ERR_ARG;
  if (c->cfg.poisson_clean) return PIC_ERR_ARG;
  if (c->has_xport || c->cfg.procs_x * c->cfg.procs_y > 1) return PIC_ERR_ARG;
  if (!c->grid_ready) return PIC_ERR_STATE;
  double out[3] = {0, 0, 0};
  CKR(DISPATCH(c, do_adjoint)(c, nsteps, checkpoint_every, true, out));
  for (int q = 0; q < 3; ++q) out3[q] = out[q];
  return PIC_OK;
}

int pic_gauss_residual(pic_ctx* c, double* out4) {
  CKR(check_ctx(c));
  if (!out4) return PIC_ERR_ARG;
  return DISPATCH(c, do_gauss)(c, out4);
}

int pic_step(pic_ctx* c, int nsteps) {
  CKR(check_ctx(c, false));
  if (!c->grid_ready) return PIC_ERR_STATE;
  for (int i = 0; i < nsteps; ++i) CKR(DISPATCH(c, do_step)(c));
  return PIC_OK;
}

int pic_fdtd(pic_ctx* c, int nsteps) {
  CKR(check_ctx(c, false));
  if (!c->grid_ready) return PIC_ERR_STATE;
  c->c_add = 0;
  c->c_thrust = 0;
  CKR(DISPATCH(c, do_add_flat)(c, false));
  if (c->cfg.poisson_clean) CKR(DISPATCH(c, do_poisson)(c));  // :676-681
  return pic_step(c, nsteps);
}

int pic_set_particles(pic_ctx* c, int species, const double* rows, const int* flag, long long n) {
  CKR(check_ctx(c));
  if (species < 0 || species > 1 || n < 0 || (n > 0 && !rows)) return PIC_ERR_ARG;
  CKR(DISPATCH(c, do_import)(c, species, rows, flag, n));
  c->particles_ready = true;
  return PIC_OK;
}

int pic_get_particles(pic_ctx* c, int species, double* rows, int* flag, long long cap, long long* n_out) {
  CKR(check_ctx(c));
  if (species < 0 || species > 1 || !n_out) return PIC_ERR_ARG;
  CKR(DISPATCH(c, do_export)(c, species, rows, cap, n_out));
  if (flag) {
    const long long m = *n_out < cap ? *n_out : cap;
    for (long long i = 0; i < m; ++i) flag[i] = 1;
  }
  return PIC_OK;
}

int pic_particle_count(pic_ctx* c, int species, long long* n_out) {
  return pic_get_particles(c, species, nullptr, nullptr, 0, n_out);
}

int pic_get_grid(pic_ctx* c, double* records) {
  CKR(check_ctx(c));
  if (!records) return PIC_ERR_ARG;
  return DISPATCH(c, do_get_grid)(c, records);
}

int pic_set_grid(pic_ctx* c, const double* records) {
  CKR(check_ctx(c));
  if (!records) return PIC_ERR_ARG;
  CKR(DISPATCH(c, do_set_grid)(c, records));
  c->grid_ready = true;
  return PIC_OK;
}

int pic_rng_counters(pic_ctx* c, long long* ctr_p, long long* ctr_v, int set) {
  if (!c || !ctr_p || !ctr_v) return PIC_ERR_ARG;
  if (set) {
    if (*ctr_p < 0 || *ctr_v < 0) return PIC_ERR_ARG;
    c->ctr_p = *ctr_p;
    c->ctr_v = *ctr_v;
  } else {
    *ctr_p = c->ctr_p;
    *ctr_v = c->ctr_v;
  }
  return PIC_OK;
}

int pic_field_path(pic_ctx* c, int* staged) {
  CKR(check_ctx(c));
  if (!staged) return PIC_ERR_ARG;
  *staged = c->staged ? 1 : 0;
  return PIC_OK;
}

int pic_status(pic_ctx* c, long long* counters8) {
  CKR(check_ctx(c));
  unsigned long long h[ERR_COUNT];
  CK(cudaMemcpyAsync(h, c->err, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int any = 0;
  for (int q = 0; q < ERR_COUNT; ++q) {
    if (counters8) counters8[q] = (long long)h[q];
    if (q < ERR_FIRST_INFO || q == ERR_MIGRATION || q == ERR_FIELD_WAIT || q == ERR_STORE_FULL) any |= h[q] != 0;
  }
  return any ? PIC_ERR_DEVICE : PIC_OK;
}

int pic_synchronize(pic_ctx* c) {
  CKR(check_ctx(c));
  CK(cudaStreamSynchronize(c->stream));
  return PIC_OK;
}

int pic_get_stream(pic_ctx* c, void** stream) {
  if (!c || !stream) return PIC_ERR_ARG;
  *stream = (void*)c->stream;
  return PIC_OK;
}

int pic_set_timing(pic_ctx* c, int enable) {
  CKR(check_ctx(c));
  CK(cudaStreamSynchronize(c->stream));
  c->timing = enable != 0;
  for (int p = 0; p < 8; ++p) c->phase[p].used = 0;
  return PIC_OK;
}

int pic_read_timing(pic_ctx* c, double* ms8, long long* marks8, long long* launches) {
  CKR(check_ctx(c));
  CK(cudaStreamSynchronize(c->stream));
  for (int p = 0; p < 8; ++p) {
    double ms = 0.0;
    const auto& ph = c->phase[p];
    for (size_t q = 0; q + 1 < ph.used; q += 2) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ph.ev[q], ph.ev[q + 1]));
      ms += t;
    }
    if (ms8) ms8[p] = ms;
    if (marks8) marks8[p] = (long long)(ph.used / 2);
    c->phase[p].used = 0;
  }
  if (launches) *launches = c->launches;
  return PIC_OK;
}

}  // extern "C"

#include "files.cuh"
