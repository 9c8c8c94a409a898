// Host side of the adjoint run (pic_adjoint / pic_objective), included by
// api.cu after the step functions it reuses.
//
// Forward: the loop body of fdtd (:687-949) in slot-stable form: the push is
// the one-thread-per-particle fused kernel over the slots, sorting is left out
// (it only reorders particles) and the refill compacts the slots, in cell
// order, before it appends, so that a particle keeps its slot from one refill
// to the next and the compaction's slot map is all the reverse pass needs.
// The forward sweep's push also adds each step's dt * F to the objective.
//
// Reverse: checkpoint/recompute. The forward sweep keeps the full state every
// `every` steps; the reverse pass restores each segment's checkpoint, replays
// its steps while keeping each step's push input (particles after the refill,
// E, and B and DB after the first half-step), and then runs the transposed
// step backwards over the segment. Memory
// is bounded by (nsteps / every) checkpoints plus `every` step inputs.

struct AdjSnap {
  long long count[2] = {0, 0};
  long long slots[2] = {0, 0};       // record slots of part[s] (>= count[s]): the layout parts_at needs
  void* part[2] = {nullptr, nullptr};
  void* planes = nullptr;            // E, B, DB (nine consecutive planes from F_EX)
  int* map[2] = {nullptr, nullptr};  // the refill's compaction map (old slot -> new slot), or null
  long long map_n[2] = {0, 0};
  long long kept[2] = {0, 0};        // slots before the refill's appended particles
  long long ctr_p = 0, ctr_v = 0;
  int c_add = 0, c_thrust = 0;
};

struct AdjRun {
  std::vector<void*> owned;  // work blocks taken from the context's pool
  // the refill's cell sort: keys and slots (double-buffered) and the radix
  // sort's temporary storage
  int* skey[2] = {nullptr, nullptr};
  int* sslot[2] = {nullptr, nullptr};
  int* kcnt = nullptr;  // the compaction's counting sort: slots per key (nodes + 1 buckets)
  int* kpos = nullptr;  // and each key's run: start after the scan, end after the scatter
  void* jn_final = nullptr;  // J_i, J_e, n_i, n_e after the forward sweep
  void* tdb = nullptr;       // three planes: one reverse step's particle terms of dJ/dDB
  // a refill's compaction count is read back without waiting: until
  // adj_resolve, sp[s].count is an upper bound and *count_dev the count
  bool pend[2] = {false, false};
  long long pend_added[2] = {0, 0};  // particles appended after the compaction
  int* scan_tmp = nullptr;
  size_t scan_len = 0;
  void* lam[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [species][buffer]: lx[3] lv[3]
  int lcur[2] = {0, 0};
  void* lfield = nullptr;  // lE 3, lDB 3, lJ 3, W 3
  unsigned long long* j64 = nullptr;  // fixed-point J sums of one species (3 planes)
  double* acc = nullptr;   // [0] J, [1] dJ/dI, [2] dJ/dV
};

constexpr int kSnapPlanes = 9;  // F_EX .. F_DBZ

static_assert(F_EY == F_EX + 1 && F_EZ == F_EX + 2 && F_BX == F_EX + 3 && F_DBX == F_EX + 6 &&
                  F_DBZ == F_EX + 8,
              "E, B and DB planes are consecutive");

// A block of at least `bytes` from the context's pool: the smallest spare
// block that holds it, else a new one with 1/16 headroom (particle counts
// drift a little between steps) rounded to 2 MB.
int pool_get(pic_ctx* c, void** p, size_t bytes) {
  DevPool& P = c->adj_pool;
  size_t best = P.spare.size();
  for (size_t q = 0; q < P.spare.size(); ++q)
    if (P.spare[q].second >= bytes && (best == P.spare.size() || P.spare[q].second < P.spare[best].second)) best = q;
  if (best < P.spare.size()) {
    *p = P.spare[best].first;
    P.spare.erase(P.spare.begin() + (long)best);
    return PIC_OK;
  }
  const size_t want = ((bytes + bytes / 16) + ((size_t)1 << 21) - 1) & ~(((size_t)1 << 21) - 1);
  CK(cudaMalloc(p, want));
  P.all.push_back(*p);
  P.size[*p] = want;
  return PIC_OK;
}

void pool_put(pic_ctx* c, void*& p) {
  if (!p) return;
  c->adj_pool.spare.emplace_back(p, c->adj_pool.size[p]);
  p = nullptr;
}

int adj_alloc(pic_ctx* c, AdjRun& R, void** p, size_t bytes) {
  CKR(pool_get(c, p, bytes));
  R.owned.push_back(*p);
  return PIC_OK;
}

// Work memory back to the pool; the stream orders its reuse after this run.
void adj_free(pic_ctx* c, AdjRun& R) {
  for (void*& p : R.owned) pool_put(c, p);
  R.owned.clear();
}

int snap_alloc(pic_ctx* c, void** p, size_t bytes) { return pool_get(c, p, bytes); }

void snap_free(pic_ctx* c, AdjSnap& S) {
  for (int s = 0; s < 2; ++s) {
    pool_put(c, S.part[s]);
    void* m = S.map[s];
    pool_put(c, m);
    S.map[s] = nullptr;
  }
  pool_put(c, S.planes);
}

template <typename real>
Parts<real> parts_at(void* base, long long cap) {
  char* b = (char*)base;
  return make_parts<real>((real*)b, (real*)(b + parts_record_bytes(cap, sizeof(real))));
}

template <typename real>
int copy_parts(pic_ctx* c, Parts<real> dst, Parts<real> src, long long n) {
  if (n <= 0) return PIC_OK;
  CK(cudaMemcpyAsync(dst.ra, src.ra, 4 * sizeof(real) * (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(dst.rb, src.rb, 4 * sizeof(real) * (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
  return PIC_OK;
}

// The context's particles, fields (E, B, DB), random-stream counters and step
// counters into a new snapshot.
template <typename real>
int adj_save(pic_ctx* c, AdjSnap& S) {
  for (int s = 0; s < 2; ++s) {
    S.count[s] = c->sp[s].count;
    S.slots[s] = S.count[s] > 0 ? S.count[s] : 1;
    CKR(snap_alloc(c, &S.part[s], store_bytes(S.slots[s], c->rsize)));
    CKR(copy_parts<real>(c, parts_at<real>(S.part[s], S.slots[s]), parts<real>(c, s), S.count[s]));
  }
  CKR(snap_alloc(c, &S.planes, kSnapPlanes * c->plane_bytes));
  CK(cudaMemcpyAsync(S.planes, (char*)c->field_mem + (size_t)F_EX * c->plane_bytes,
                     kSnapPlanes * c->plane_bytes, cudaMemcpyDeviceToDevice, c->stream));
  S.ctr_p = c->ctr_p;
  S.ctr_v = c->ctr_v;
  S.c_add = c->c_add;
  S.c_thrust = c->c_thrust;
  return PIC_OK;
}

template <typename real>
int adj_restore(pic_ctx* c, const AdjSnap& S) {
  for (int s = 0; s < 2; ++s) {
    if (S.count[s] > c->sp[s].cap) return PIC_ERR_CAPACITY;
    CKR(copy_parts<real>(c, parts<real>(c, s), parts_at<real>(S.part[s], S.slots[s]), S.count[s]));
    CKR(set_count(c, s, S.count[s]));
    c->tiled[s] = false;
    c->layout[s] = false;
  }
  CK(cudaMemcpyAsync((char*)c->field_mem + (size_t)F_EX * c->plane_bytes, S.planes,
                     kSnapPlanes * c->plane_bytes, cudaMemcpyDeviceToDevice, c->stream));
  c->ctr_p = S.ctr_p;
  c->ctr_v = S.ctr_v;
  c->c_add = S.c_add;
  c->c_thrust = S.c_thrust;
  return PIC_OK;
}

AdjConst adj_const(const pic_ctx* c, int s) {
  const pic_config& k = c->cfg;
  AdjConst a;
  a.K = (s == 0 ? 1.0 : -1.0) * k.q * species_weight(c) * k.dx * k.dx * k.dx;
  a.dt = k.dt;
  a.inv_I = k.coil_i != 0.0 ? 1.0 / k.coil_i : 0.0;
  a.imf[0] = k.imf_x; a.imf[1] = k.imf_y; a.imf[2] = k.imf_z;
  a.jsign = s == 0 ? 1.0 : -1.0;
  return a;
}

// Bits of the compaction's sort keys: node indices and one dead key above them.
int key_bits(const pic_ctx* c) {
  int b = 1;
  while ((1LL << b) - 1 < (long long)c->g.nodes + 1) ++b;
  return b;
}

// Removes the empty slots of species s and orders the rest by cell (a stable
// counting sort on the node index, so a replayed segment gets the same order),
// recording the slot map in `map` when it is not null. Cell order keeps the
// lanes of a warp on few stencil bases, which the aggregated scatters of the
// adjoint kernels need; between refills the slots drift apart as particles
// move. The new count is set on the device and read back into pinned memory
// without waiting (adj_resolve).
template <typename real>
int adj_compact(pic_ctx* c, AdjRun& R, int s, int* map) {
  Store& st = c->sp[s];
  const long long n = st.count;
  if (n == 0) return PIC_OK;
  const int bits = key_bits(c);
  const int dead = (1 << bits) - 1;
  const int nodes = c->g.nodes;
  cell_key_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(parts<real>(c, s), (int)n, c->g, dead, R.skey[0],
                                                                     R.sslot[0]);
  CKL();
  CK(cudaMemsetAsync(R.kcnt, 0, sizeof(int) * (size_t)(nodes + 1), c->stream));
  key_count_kernel<<<grid_blocks(n), kThreads, 0, c->stream>>>(R.skey[0], (int)n, dead, nodes, R.kcnt);
  CKL();
  CKR(scan_exclusive(c, R.kcnt, R.kpos, nodes + 1, R.scan_tmp, R.scan_len));
  key_scatter_kernel<<<grid_blocks(n), kThreads, 0, c->stream>>>(R.skey[0], (int)n, dead, nodes, R.kpos, R.skey[1],
                                                                 R.sslot[1]);
  CKL();
  key_rank_kernel<<<grid_blocks(n), kThreads, 0, c->stream>>>(R.skey[1], R.sslot[1], (int)n, dead, R.kcnt, R.kpos,
                                                              R.skey[0], R.sslot[0]);
  CKL();
  cell_gather_kernel<real><<<grid_blocks(n), kThreads, 0, c->stream>>>(parts<real>(c, s), (int)n, dead, R.skey[0],
                                                                        R.sslot[0], parts<real>(c, s, 1 - st.cur),
                                                                        map, st.count_dev);
  CKL();
  CK(cudaMemcpyAsync(c->host_pin + 2 + s, st.count_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(st.readback, c->stream));
  st.cur = 1 - st.cur;
  c->tiled[s] = false;
  c->layout[s] = false;
  R.pend[s] = true;
  R.pend_added[s] = 0;
  return PIC_OK;
}

// The refill's appended particles after a pending compaction: placed from the
// device count, which they then extend; the host count stays an upper bound.
template <typename real>
int adj_source(pic_ctx* c, AdjRun& R, int s, const Slab* slabs, int nslab) {
  if (!R.pend[s]) return do_source<real>(c, s, slabs, nslab);
  SourceParams sp = source_params(c, s, slabs, nslab, 0);
  const long long total = sp.total;
  if (total == 0) return PIC_OK;
  Store& st = c->sp[s];
  if (st.count + total > st.cap) return PIC_ERR_CAPACITY;
  sp.dst_dev = st.count_dev;
  source_kernel<real><<<grid_blocks(total), kThreads, 0, c->stream>>>(parts<real>(c, s), sp, c->err);
  CKL();
  add_count_kernel<<<1, 1, 0, c->stream>>>(st.count_dev, (int)total);
  CKL();
  c->ctr_p += 3 * total;
  c->ctr_v += 6 * total;
  st.count += total;
  R.pend_added[s] += total;
  return PIC_OK;
}

// Waits for pending compaction counts and sets the host counts (and, with
// `rec`, the recorded step input's counts and kept slots).
int adj_resolve(pic_ctx* c, AdjRun& R, AdjSnap* rec) {
  for (int s = 0; s < 2; ++s) {
    if (!R.pend[s]) continue;
    Store& st = c->sp[s];
    CK(cudaEventSynchronize(st.readback));
    R.pend[s] = false;
    const long long kept = c->host_pin[2 + s];  // read back before the appends
    st.count = kept + R.pend_added[s];
    if (rec) {
      rec->kept[s] = kept;
      rec->count[s] = st.count;
    }
  }
  return PIC_OK;
}

// One slot-stable loop body; with `rec`, the step input goes into it. With
// `objective` the push adds the step's dt * F to the objective (the forward
// sweep; a recomputed step's terms are known). The density deposit runs only
// with `density` (the last step of the forward sweep): no step of the adjoint
// run reads n, and the run ends with that step's n.
template <typename real>
int adj_forward_step(pic_ctx* c, AdjRun& R, AdjSnap* rec, bool objective, bool density) {
  CKR(do_renew_grid(c));
  long long kept[2] = {c->sp[0].count, c->sp[1].count};
  if (c->c_add > c->cfg.add_interval - 1) {
    Slab slabs[5];
    refill_slabs(c, slabs);
    for (int s = 0; s < 2; ++s) {
      Store& st = c->sp[s];
      if (st.count > 0) {
        delete_shell_kernel<real><<<particle_blocks(st.count), kThreads, 0, c->stream>>>(parts<real>(c, s), 0,
                                                                                         st.count_dev, c->g);
        CKL();
      }
      int* map = nullptr;
      if (rec && st.count > 0) {
        CKR(snap_alloc(c, (void**)&map, sizeof(int) * (size_t)st.count));
        rec->map[s] = map;
        rec->map_n[s] = st.count;
      }
      CKR(adj_compact<real>(c, R, s, map));
      CKR(adj_source<real>(c, R, s, slabs, 5));
    }
    c->c_add = 0;
  }
  CKR(do_renew_b<real>(c));
  if (rec) {  // the push's inputs: particles, E at the step start, B and DB after the first half-step
    CKR(adj_save<real>(c, *rec));
    rec->kept[0] = kept[0];
    rec->kept[1] = kept[1];
  }
  const int nodes = c->g.nodes;
  Fields<real> F = fields<real>(c);
  for (int s = 0; s < 2; ++s) {
    const long long n = c->sp[s].count;  // an upper bound while a compaction count is pending
    if (n == 0) continue;
    const PushConst<real> pc = push_const<real>(c, s);
    CK(cudaMemsetAsync(R.j64, 0, sizeof(unsigned long long) * 3 * (size_t)nodes, c->stream));
    push_fixed_kernel<real><<<particle_blocks(n), kThreads, 0, c->stream>>>(
        parts<real>(c, s), c->sp[s].count_dev, F, c->g, pc, R.j64, R.j64 + nodes, R.j64 + 2 * (size_t)nodes,
        (real)(kJFixed / c->cfg.c), density ? 1 : 0, adj_const(c, s), objective ? R.acc : nullptr, c->err);
    CKL();
    jconvert_kernel<real><<<grid_blocks(nodes), kThreads, 0, c->stream>>>(
        R.j64, nodes, F.f[pc.pjx], F.f[pc.pjy], F.f[pc.pjz], c->cfg.q * species_weight(c) * c->cfg.c / kJFixed);
    CKL();
  }
  CKR(adj_resolve(c, R, rec));  // waits for the refill's counts while the GPU pushes
  CKR(do_renew_b<real>(c));
  CKR(do_fold<real>(c));
  CKR(do_renew_e<real>(c));
  c->c_add++;
  c->c_thrust++;
  return PIC_OK;
}

template <typename real>
AdjPart<real> adj_part(pic_ctx* c, AdjRun& R, int s, int buf) {
  AdjPart<real> A;
  const long long cap = c->sp[s].cap;
  char* p = (char*)R.lam[s][buf];
  for (int q = 0; q < 3; ++q) { A.lx[q] = (real*)p; p += align256((size_t)cap * sizeof(real)); }
  for (int q = 0; q < 3; ++q) { A.lv[q] = (real*)p; p += align256((size_t)cap * sizeof(real)); }
  real* lf = (real*)R.lfield;
  const size_t pl = c->plane_bytes / sizeof(real);
  for (int q = 0; q < 3; ++q) {
    A.le[q] = lf + q * pl;
    A.ldb[q] = lf + (3 + q) * pl;
    A.lj[q] = lf + (6 + q) * pl;
  }
  return A;
}

template <typename real>
AdjField<real> adj_field(pic_ctx* c, AdjRun& R) {
  AdjField<real> A;
  real* lf = (real*)R.lfield;
  const size_t pl = c->plane_bytes / sizeof(real);
  for (int q = 0; q < 3; ++q) {
    A.le[q] = lf + q * pl;
    A.ldb[q] = lf + (3 + q) * pl;
    A.lj[q] = lf + (6 + q) * pl;
    A.w[q] = lf + (9 + q) * pl;
  }
  return A;
}

template <typename real>
PlaneSet<real> plane_set(real* const* p, int n) {
  PlaneSet<real> s{};
  for (int q = 0; q < n; ++q) s.p[q] = p[q];
  s.count = n;
  return s;
}

// Transpose of renew_b4_2 + sr_b on (lE, lDB).
template <typename real>
int adj_renew_b(pic_ctx* c, AdjRun& R) {
  AdjField<real> A = adj_field<real>(c, R);
  const Geom& g = c->g;
  const double inv_I = c->cfg.coil_i != 0.0 ? 1.0 / c->cfg.coil_i : 0.0;
  wrap_b_adjoint<real><<<grid_blocks((long long)g.gx * g.gz), kThreads, 0, c->stream>>>(fields<real>(c), A, g, 1,
                                                                                         inv_I, R.acc);
  CKL();
  wrap_b_adjoint<real><<<grid_blocks((long long)g.gy * g.gz), kThreads, 0, c->stream>>>(fields<real>(c), A, g, 0,
                                                                                         inv_I, R.acc);
  CKL();
  BParams p{1. / c->cfg.e0 * c->cfg.dt * 0.5 * 0.5, 0.5 * c->cfg.dt, 1.0 / (24.0 * c->cfg.dx)};
  const long long nint = (long long)g.nx * g.ny * g.nz;
  renew_b_adjoint_point<real><<<grid_blocks(nint), kThreads, 0, c->stream>>>(A, g, ramps(c), p);
  CKL();
  renew_b_adjoint_curl<real><<<grid_blocks(g.nodes), kThreads, 0, c->stream>>>(A, g);
  CKL();
  return PIC_OK;
}

// Transpose of renew_e4_2 + sr_e and of the sr_current2 fold: lE in, lJ out.
template <typename real>
int adj_renew_e(pic_ctx* c, AdjRun& R) {
  AdjField<real> A = adj_field<real>(c, R);
  const Geom& g = c->g;
  wrap_y_adjoint<real><<<grid_blocks((long long)g.gx * g.gz), kThreads, 0, c->stream>>>(plane_set(A.le, 3), g);
  CKL();
  wrap_x_adjoint<real><<<grid_blocks((long long)g.gy * g.gz), kThreads, 0, c->stream>>>(plane_set(A.le, 3), g);
  CKL();
  CK(cudaMemsetAsync(A.lj[0], 0, 3 * c->plane_bytes, c->stream));
  EParams p{c->cfg.c * c->cfg.c * c->cfg.dt, c->cfg.mu0, 1.0 / (24.0 * c->cfg.dx)};
  const long long nint = (long long)g.nx * g.ny * g.nz;
  renew_e_adjoint_point<real><<<grid_blocks(nint), kThreads, 0, c->stream>>>(A, g, ramps(c), p);
  CKL();
  renew_e_adjoint_curl<real><<<grid_blocks(g.nodes), kThreads, 0, c->stream>>>(A, g);
  CKL();
  fold_y_adjoint<real><<<grid_blocks((long long)g.gx * g.gz), kThreads, 0, c->stream>>>(plane_set(A.lj, 3), g);
  CKL();
  fold_x_adjoint<real><<<grid_blocks((long long)g.gy * g.gz), kThreads, 0, c->stream>>>(plane_set(A.lj, 3), g);
  CKL();
  return PIC_OK;
}

// The transposed step n, given the adjoint of its output state; `in` is the
// step's recorded input.
template <typename real>
int adj_reverse_step(pic_ctx* c, AdjRun& R, const AdjSnap& in) {
  // the fields the push gathered, as recorded: E at the step start, B after the first half-step
  CK(cudaMemcpyAsync((char*)c->field_mem + (size_t)F_EX * c->plane_bytes, in.planes, kSnapPlanes * c->plane_bytes,
                     cudaMemcpyDeviceToDevice, c->stream));
  CKR(adj_renew_e<real>(c, R));
  CKR(adj_renew_b<real>(c, R));  // second B half-step
  for (int s = 0; s < 2; ++s) {
    const long long n = in.count[s];
    if (n == 0) continue;
    AdjPart<real> A = adj_part<real>(c, R, s, R.lcur[s]);
    for (int q = 0; q < 3; ++q) A.ldb[q] = (real*)((char*)R.tdb + (size_t)q * c->plane_bytes);
    push_adjoint_kernel<real><<<particle_blocks(n), kThreads, 0, c->stream>>>(
        parts_at<real>(in.part[s], in.slots[s]), (int)n, fields<real>(c), c->g, push_const<real>(c, s), A,
        adj_const(c, s), R.acc);
    CKL();
  }
  {
    AdjPart<real> T{};
    for (int q = 0; q < 3; ++q) T.ldb[q] = (real*)((char*)R.tdb + (size_t)q * c->plane_bytes);
    ldb_merge_kernel<real><<<particle_blocks(c->g.nodes), kThreads, 0, c->stream>>>(
        fields<real>(c), T, adj_field<real>(c, R), c->g.nodes, adj_const(c, 0), R.acc);
    CKL();
  }
  CKR(adj_renew_b<real>(c, R));  // first B half-step
  return PIC_OK;
}

// Transpose of the refill at the start of the recorded step: the appended
// particles were created with vz = V + thermal, and the slots before the
// compaction take the adjoints of their new slots through its map.
template <typename real>
int adj_unrefill(pic_ctx* c, AdjRun& R, const AdjSnap& in) {
  for (int s = 0; s < 2; ++s) {
    if (in.count[s] > in.kept[s]) {
      const AdjPart<real> A = adj_part<real>(c, R, s, R.lcur[s]);
      drift_grad_kernel<real><<<particle_blocks(in.count[s] - in.kept[s]), kThreads, 0, c->stream>>>(
          parts_at<real>(in.part[s], in.slots[s]), A.lv[2], (int)in.kept[s], (int)in.count[s], R.acc);
      CKL();
    }
    if (in.map[s]) {
      const int nb = 1 - R.lcur[s];
      uncompact_adjoint_kernel<real><<<grid_blocks(in.map_n[s]), kThreads, 0, c->stream>>>(
          in.map[s], (int)in.map_n[s], adj_part<real>(c, R, s, R.lcur[s]), adj_part<real>(c, R, s, nb));
      CKL();
      R.lcur[s] = nb;
    }
  }
  return PIC_OK;
}
