// Batched time steps: many independent lattices (engines built and set up
// one by one through the single-engine entry points) advanced together, with
// every phase of a step one launch over all of them.  Part of engine.cu's
// translation unit (it uses the engine internals defined there).
//
// Per step and phase the batch launches the TMA marching sweeps of
// march_tma.cuh over a tile list that concatenates the tiles of every
// lattice, one list per sweep form (CPML-free interior, CPML-free, CPML):
// entry b = (lattice, k tile, j tile, x chunk), with the lattice's sweep
// parameters and tensor maps read from a device array.  The lattice faces
// k = nz, j = ny, the TFSF pass groups and the step counters go the same way
// (block lists over all lattices).  A step of the batch is therefore
// 2 x (up to 3 sweep launches + 1 face launch + 2 TFSF launches) + 1
// launches whatever the number of lattices, the launch pattern is captured
// into CUDA graphs of whole step chunks, and small lattices share the SMs
// instead of each leaving most of them idle.  Tile lists put the largest
// lattices first so that the tail of each launch holds small tiles.
//
// Per lattice the arithmetic and its order are those of the engine's default
// sweep (split H then E, marching along x with TMA-staged planes), so a
// batched lattice follows the same step sequence as the same engine run
// alone: H sweep, H lattice faces, TFSF H groups 1 and 2, E sweep, E lattice
// faces, TFSF E groups 1 and 2, step counter.  Engines with ADE media,
// lumped sources, movies, an NF2FF surface or coefficient overrides are not
// batched (their per-step extras stay with xfd_run).
//
// By default (option `queue` = 1) the whole step is instead ONE launch of
// the persistent kernel k_batch_queue (batch_queue.cuh): the same CTA bodies
// over one device work queue that holds every tile, face block and TFSF
// block of the step of every lattice, with bounded per-lattice dependency
// waits in place of the launch boundaries; `queue` = 0 keeps the launch per
// phase and form described above.
//
// The form (`queue`), the tile shape (rows per tile, `tile_rows`: 8 or 16,
// the queue form only) and the x chunk length (planes per CTA,
// `march_ichunk`) are what the autotuner chooses: with the `autotune` option
// set to K, the next xfd_batch_run spends 1 + K of its steps on each of 12
// candidates (the queue form at rows 8 and 16, the launch per phase at rows
// 8, each at depths 8, 16, 32, 64; a warm-up step, then K steps in one graph
// timed by CUDA events) and keeps the fastest.  Tiling does not change any node's arithmetic, so the
// tuned run advances the same simulation.  Temporal blocking is not
// implemented: every launch advances one time step.

#include "batch_queue.cuh"

struct xfd_batch {
  int device = 0;
  int precision = XFD_FP64;
  std::vector<xfd_engine*> eng;  // in tile-list order (largest lattice first)
  std::string err;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  // Launch-per-phase form, option "concurrent" (default 1): the sweep-form
  // launches of a phase on `stream` and three side streams (they sweep
  // disjoint tiles), forked from and joined back into `stream`.
  bool concurrent = true;
  cudaStream_t side[3]{};
  cudaEvent_t fork_ev = nullptr, join_ev[3]{};
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  std::vector<void*> allocs;  // device tables of the current preparation
  int march_ichunk = 16;
  bool use_graph = true;
  int graph_chunk = 32;
  int autotune = 0;  // steps timed per candidate depth on the next run (0: off)
  bool ready = false;
  // Field buffer of each engine (in `eng` order) when the tables were built:
  // the tables hold that buffer's pointers and tensor maps.
  std::vector<int> cur_at_prepare;
  void* d_march = nullptr;  // MarchTmaP<T>[n]
  void* d_yee = nullptr;    // YeeP<T>[n]
  void* d_tfsf = nullptr;   // TfsfSceneD<T>[n]
  long long** d_steps = nullptr;
  int4* d_tiles = nullptr;
  // lists: CPML-free interior, CPML-free, CPML tiles meeting x layers only,
  // y only, z only, several axes
  long long tile_off[7] = {0, 0, 0, 0, 0, 0, 0};
  bool split_axes = true;
  int2* d_edge = nullptr;
  long long n_edge = 0;
  int2* d_tfb = nullptr;
  long long tfsf_off[5] = {0, 0, 0, 0, 0};  // pass groups H1, H2, E1, E2
  cudaGraphExec_t graph_exec = nullptr;
  long long graph_len = 0;
  struct Tune {
    int queue, rows, depth;
    double ms;
  };
  std::vector<Tune> tune_ms;  // candidates of the last tuning, ms per step
  // Persistent queue form (batch_queue.cuh).
  bool queue = true;
  int tile_rows = 8;             // rows per tile: kMTJ or kWideTJ
  long long queue_wait = 0;      // cycles per dependency wait (0: the stage-wait default)
  bool queue_stall_test = false; // test hook: one item waits for a count never reached
  int4* d_items = nullptr;
  int* d_need = nullptr;
  int* d_qcnt = nullptr;  // head, exits, done[n]
  int n_items = 0;
  int queue_grid = 0;
};

namespace {

xfd_status bfail(xfd_batch* b, xfd_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else g_create_error = buf;
  return s;
}

#define BATCH_TRY(b, call)                                                                   \
  do {                                                                                       \
    cudaError_t _c = (call);                                                                 \
    if (_c != cudaSuccess)                                                                   \
      return bfail((b), XFD_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_c));      \
  } while (0)

void batch_drop_graph(xfd_batch* b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  b->graph_exec = nullptr;
  b->graph_len = 0;
}

void batch_free_tables(xfd_batch* b) {
  for (void* p : b->allocs) cudaFree(p);
  b->allocs.clear();
  b->d_march = b->d_yee = b->d_tfsf = nullptr;
  b->d_steps = nullptr;
  b->d_tiles = nullptr;
  b->d_edge = nullptr;
  b->d_tfb = nullptr;
  b->d_items = nullptr;
  b->d_need = nullptr;
  b->d_qcnt = nullptr;
  b->n_items = 0;
  b->ready = false;
}

template <typename U>
xfd_status batch_upload(xfd_batch* b, U** dst, const U* src, size_t n) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(n * sizeof(U), 16);
  cudaError_t c = cudaMalloc(&p, bytes);
  if (c != cudaSuccess)
    return bfail(b, c == cudaErrorMemoryAllocation ? XFD_ERR_OUT_OF_MEMORY : XFD_ERR_CUDA,
                 "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(c));
  b->allocs.push_back(p);
  if (n) BATCH_TRY(b, cudaMemcpyAsync(p, src, n * sizeof(U), cudaMemcpyHostToDevice, b->stream));
  *dst = static_cast<U*>(p);
  return XFD_OK;
}

template <typename T>
xfd_status batch_set_smem() {
  constexpr int MS = march_stages<T>();
  constexpr int MF = march_free_stages<T>();
  const int msm = MarchGeom<T, kMTJ, 32>::smem(MS);
  const int msm_free = MarchGeom<T, kMTJ, 32>::smem(MF);
  cudaError_t c = cudaSuccess;
  auto set = [&](const void* f, int bytes) {
    if (c == cudaSuccess)
      c = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MF, false, true>, msm_free);
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MF, false, false>, msm_free);
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MS, true, false>, msm);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MF, false, true>, msm_free);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MF, false, false>, msm_free);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MS, true, false>, msm);
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 1>, msm_free);
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 2>, msm_free);
  set((const void*)k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 4>, msm_free);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 1>, msm_free);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 2>, msm_free);
  set((const void*)k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 4>, msm_free);
  set((const void*)k_batch_queue<T, kMTJ>, MarchGeom<T, kMTJ, 32>::smem(MS));
  set((const void*)k_batch_queue<T, kWideTJ>, MarchGeom<T, kWideTJ, 32>::smem(MS));
  if (c != cudaSuccess) {
    g_create_error = cudaGetErrorString(c);
    return XFD_ERR_CUDA;
  }
  return XFD_OK;
}

// Builds the per-lattice parameter arrays and the tile and block lists for
// the current x chunk length.
template <typename T>
xfd_status batch_prepare(xfd_batch* b) {
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  batch_drop_graph(b);
  batch_free_tables(b);
  if (batch_set_smem<T>() != XFD_OK)
    return bfail(b, XFD_ERR_CUDA, "batched sweep attributes: %s", g_create_error.c_str());
  const int n = (int)b->eng.size();
  std::vector<MarchTmaP<T>> mp((size_t)n);
  std::vector<YeeP<T>> yp((size_t)n);
  std::vector<TfsfSceneD<T>> ts((size_t)n);
  std::vector<long long*> steps((size_t)n);
  std::vector<int4> tiles[6];
  std::vector<int2> edge;
  std::vector<int2> tfb[4];
  // The queue form sweeps tiles of tile_rows rows; its face and TFSF items
  // are blocks of one CTA's threads.
  const int tj = b->queue ? b->tile_rows : kMTJ;
  const int qnt = 32 * tj;
  std::vector<std::array<int, 8>> qcount((size_t)n);  // items per lattice and level
  for (int s = 0; s < n; ++s) {
    xfd_engine* e = b->eng[(size_t)s];
    e->march_ichunk = b->march_ichunk;
    e->graph_dirty = true;
    xfd_status st = ensure_ready(e);
    if (st == XFD_OK && !e->tma_ready) st = build_tma_maps<T>(e);
    if (st != XFD_OK) return bfail(b, st, "lattice %d: %s", s, e->err.c_str());
    BATCH_TRY(b, cudaStreamSynchronize(e->stream));
    MarchTmaP<T> q{};
    q.p = march_params<T>(e);
    q.m = tj == kMTJ ? e->mtma[e->cur] : e->mtma_w[e->cur];
    q.err = e->d_err;
    q.wait_budget = e->stage_wait;
    int lo[3], hi[3];
    march_split(e, lo, hi, tj);
    const bool box = hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2];
    for (int a = 0; a < 3; ++a) {
      q.box_lo[a] = box ? lo[a] : 0;
      q.box_hi[a] = box ? hi[a] : 0;
    }
    const Lat& L = e->L;
    const bool in = box && lo[0] >= 1 && 32 * hi[0] <= L.nz && lo[1] >= 1 &&
                    tj * hi[1] <= L.ny && lo[2] >= 1 && hi[2] * e->march_ichunk <= L.nx;
    const int nt[3] = {(L.nz + 31) / 32, (L.ny + tj - 1) / tj,
                       (L.nx + 1 + e->march_ichunk - 1) / e->march_ichunk};
    std::array<int, 8>& qc = qcount[(size_t)s];
    qc.fill(0);
    for (int z = 0; z < nt[2]; ++z)
      for (int y = 0; y < nt[1]; ++y)
        for (int x = 0; x < nt[0]; ++x) {
          const bool inbox = box && x >= lo[0] && x < hi[0] && y >= lo[1] && y < hi[1] &&
                             z >= lo[2] && z < hi[2];
          int f = inbox ? (in ? 0 : 1) : 5;
          if (!inbox && b->split_axes) {
            const int ich = e->march_ichunk;
            f = 2 + cpml_tile_list(e, 32 * x, std::min(32 * x + 32, L.nz), tj * y,
                                   std::min(tj * y + tj, L.ny), ich * z,
                                   std::min(ich * z + ich, L.nx + 1));
          }
          tiles[f].push_back(make_int4(s, x, y, z));
          qc[0] += 1;
          qc[4] += 1;
        }
    mp[(size_t)s] = q;
    yp[(size_t)s] = yee_params<T>(e);
    const int bn = b->queue ? qnt * kQueueNodeIters : 256;  // nodes per face / TFSF block
    const long long nb = (edge_nodes(L) + bn - 1) / bn;
    for (long long k = 0; k < nb; ++k) edge.push_back(make_int2(s, (int)k));
    qc[1] = qc[5] = (int)nb;
    TfsfSceneD<T> t{};
    if (e->have_tfsf) {
      t.tf = e->tfsf;
      static const int level_of_group[4] = {2, 3, 6, 7};
      for (int g = 0; g < 4; ++g) {
        t.g[g] = e->tfsf_groups[g];
        const long long gb = (t.g[g].total + bn - 1) / bn;
        for (long long k = 0; k < gb; ++k) tfb[g].push_back(make_int2(s, (int)k));
        qc[level_of_group[g]] = (int)gb;
      }
    }
    t.L = L;
    t.fields = reinterpret_cast<T* const*>(e->d_fields[e->cur]);
    t.step = e->d_step;
    t.err = e->d_err;
    ts[(size_t)s] = t;
    steps[(size_t)s] = e->d_step;
  }
  MarchTmaP<T>* dm = nullptr;
  YeeP<T>* dy = nullptr;
  TfsfSceneD<T>* dt = nullptr;
  xfd_status st;
  if ((st = batch_upload(b, &dm, mp.data(), mp.size())) != XFD_OK) return st;
  if ((st = batch_upload(b, &dy, yp.data(), yp.size())) != XFD_OK) return st;
  if ((st = batch_upload(b, &dt, ts.data(), ts.size())) != XFD_OK) return st;
  if ((st = batch_upload(b, &b->d_steps, steps.data(), steps.size())) != XFD_OK) return st;
  std::vector<int4> all;
  for (int f = 0; f < 6; ++f) {
    b->tile_off[f] = (long long)all.size();
    all.insert(all.end(), tiles[f].begin(), tiles[f].end());
  }
  b->tile_off[6] = (long long)all.size();
  if ((st = batch_upload(b, &b->d_tiles, all.data(), all.size())) != XFD_OK) return st;
  if ((st = batch_upload(b, &b->d_edge, edge.data(), edge.size())) != XFD_OK) return st;
  b->n_edge = (long long)edge.size();
  std::vector<int2> tall;
  for (int g = 0; g < 4; ++g) {
    b->tfsf_off[g] = (long long)tall.size();
    tall.insert(tall.end(), tfb[g].begin(), tfb[g].end());
  }
  b->tfsf_off[4] = (long long)tall.size();
  if ((st = batch_upload(b, &b->d_tfb, tall.data(), tall.size())) != XFD_OK) return st;
  if (b->queue) {
    int per_sm = 0, sms = 0;
    const void* kq = tj == kMTJ ? (const void*)k_batch_queue<T, kMTJ>
                                : (const void*)k_batch_queue<T, kWideTJ>;
    const size_t qsm = tj == kMTJ ? MarchGeom<T, kMTJ, 32>::smem(march_stages<T>())
                                  : MarchGeom<T, kWideTJ, 32>::smem(march_stages<T>());
    BATCH_TRY(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kq, qnt, qsm));
    BATCH_TRY(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    if (per_sm < 1) return bfail(b, XFD_ERR_CUDA, "queue kernel does not fit on an SM");
    const int resident = per_sm * sms;
    // Items level by level (H tiles, H faces, TFSF H 1, 2, E tiles, E faces,
    // TFSF E 1, 2); tiles of a level by form, costliest first (CPML tiles
    // meeting several axes, single-axis CPML tiles, CPML-free, the interior),
    // lattices largest first within a form.  (Pipelining the queue over
    // groups of lattices, the H levels of one group between the H and E
    // levels of the one before, measured slower: 8.2 against 7.6 ms per step
    // on 96 lattices of 64^3-224^3.)
    std::vector<int4> items;
    std::vector<int> need;
    auto need_of = [&](int s, int level) {
      int c = 0;
      for (int l = 0; l < level; ++l) c += qcount[(size_t)s][(size_t)l];
      return c;
    };
    static const int form_order[6] = {5, 2, 3, 4, 1, 0};
    auto push_tiles = [&](int level, int kind0) {
      for (int f : form_order)
        for (const int4& w : tiles[f]) {
          items.push_back(make_int4(((kind0 + f) << 16) | w.x, w.y, w.z, w.w));
          need.push_back(need_of(w.x, level));
        }
    };
    auto push_blocks = [&](int level, int kind, const std::vector<int2>& blocks) {
      for (const int2& v : blocks) {
        items.push_back(make_int4((kind << 16) | v.x, v.y, 0, 0));
        need.push_back(need_of(v.x, level));
      }
    };
    push_tiles(0, kQ_H_IN);
    push_blocks(1, kQ_EDGE_H, edge);
    push_blocks(2, kQ_TFSF_H1, tfb[0]);
    push_blocks(3, kQ_TFSF_H2, tfb[1]);
    push_tiles(4, kQ_E_IN);
    push_blocks(5, kQ_EDGE_E, edge);
    push_blocks(6, kQ_TFSF_E1, tfb[2]);
    push_blocks(7, kQ_TFSF_E2, tfb[3]);
    if (b->queue_stall_test) {
      // The first item of lattice 0 that waits at all waits for more items
      // than the lattice has: a count nothing reaches, so the wait runs out.
      int total = 0;
      for (int l = 0; l < 8; ++l) total += qcount[0][(size_t)l];
      for (size_t t = 0; t < items.size(); ++t)
        if ((items[t].x & 0xffff) == 0 && need[t] > 0) {
          need[t] = total + 1;
          break;
        }
    }
    if ((st = batch_upload(b, &b->d_items, items.data(), items.size())) != XFD_OK) return st;
    if ((st = batch_upload(b, &b->d_need, need.data(), need.size())) != XFD_OK) return st;
    std::vector<int> zero((size_t)n + 2, 0);
    if ((st = batch_upload(b, &b->d_qcnt, zero.data(), zero.size())) != XFD_OK) return st;
    b->n_items = (int)items.size();
    b->queue_grid = std::max(1, std::min(b->n_items, resident));
  }
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  b->d_march = dm;
  b->d_yee = dy;
  b->d_tfsf = dt;
  b->cur_at_prepare.clear();
  for (const xfd_engine* e : b->eng) b->cur_at_prepare.push_back(e->cur);
  b->ready = true;
  return XFD_OK;
}

template <typename T>
cudaError_t batch_enqueue_queue(xfd_batch* b) {
  BatchQueueD<T> q{};
  q.march = static_cast<const MarchTmaP<T>*>(b->d_march);
  q.yee = static_cast<const YeeP<T>*>(b->d_yee);
  q.tfsf = static_cast<const TfsfSceneD<T>*>(b->d_tfsf);
  q.items = b->d_items;
  q.need = b->d_need;
  q.n_items = b->n_items;
  q.n_lattices = (int)b->eng.size();
  q.head = b->d_qcnt;
  q.exits = b->d_qcnt + 1;
  q.done = b->d_qcnt + 2;
  q.steps = b->d_steps;
  q.wait_budget = b->queue_wait > 0 ? b->queue_wait : kStageWaitDefault;
  constexpr int MS = march_stages<T>();
  if (b->tile_rows == kWideTJ)
    k_batch_queue<T, kWideTJ><<<b->queue_grid, dim3(32, kWideTJ, 1),
                                MarchGeom<T, kWideTJ, 32>::smem(MS), b->stream>>>(q);
  else
    k_batch_queue<T, kMTJ><<<b->queue_grid, dim3(32, kMTJ, 1), MarchGeom<T, kMTJ, 32>::smem(MS),
                             b->stream>>>(q);
  return cudaGetLastError();
}

template <typename T>
cudaError_t batch_enqueue_t(xfd_batch* b) {
  if (b->queue) return batch_enqueue_queue<T>(b);
  cudaStream_t s = b->stream;
  constexpr int MS = march_stages<T>();
  constexpr int MF = march_free_stages<T>();
  const size_t msm = MarchGeom<T, kMTJ, 32>::smem(MS);
  const size_t msm_free = MarchGeom<T, kMTJ, 32>::smem(MF);
  const dim3 blk(32, kMTJ, 1);
  const auto* dm = static_cast<const MarchTmaP<T>*>(b->d_march);
  const auto* dy = static_cast<const YeeP<T>*>(b->d_yee);
  const auto* dt = static_cast<const TfsfSceneD<T>*>(b->d_tfsf);
  auto n_of = [&](int f) { return (unsigned)(b->tile_off[f + 1] - b->tile_off[f]); };
  auto list = [&](int f) { return b->d_tiles + b->tile_off[f]; };
  cudaError_t cerr = cudaSuccess;
  const bool conc = b->concurrent && b->side[0];
  auto sweeps = [&](auto k_in, auto k_free, auto kx, auto ky, auto kz, auto k_cp) {
    // x-, y-, z-only CPML lists on the side streams, the rest on `stream`
    cudaStream_t sx = conc ? b->side[0] : s, sy = conc ? b->side[1] : s,
                 sz = conc ? b->side[2] : s;
    if (conc) {
      if (cerr == cudaSuccess) cerr = cudaEventRecord(b->fork_ev, s);
      for (int q = 0; q < 3 && cerr == cudaSuccess; ++q)
        cerr = cudaStreamWaitEvent(b->side[q], b->fork_ev, 0);
    }
    if (n_of(5)) k_cp<<<n_of(5), blk, msm, s>>>(dm, list(5));
    if (n_of(2)) kx<<<n_of(2), blk, msm_free, sx>>>(dm, list(2));
    if (n_of(3)) ky<<<n_of(3), blk, msm_free, sy>>>(dm, list(3));
    if (n_of(4)) kz<<<n_of(4), blk, msm_free, sz>>>(dm, list(4));
    if (n_of(1)) k_free<<<n_of(1), blk, msm_free, s>>>(dm, list(1));
    if (n_of(0)) k_in<<<n_of(0), blk, msm_free, s>>>(dm, list(0));
    if (conc) {
      for (int q = 0; q < 3 && cerr == cudaSuccess; ++q) {
        cerr = cudaEventRecord(b->join_ev[q], b->side[q]);
        if (cerr == cudaSuccess) cerr = cudaStreamWaitEvent(s, b->join_ev[q], 0);
      }
    }
  };
  auto tfsf = [&](int g) {
    const long long nb = b->tfsf_off[g + 1] - b->tfsf_off[g];
    if (nb > 0) k_tfsf_batch<T><<<(unsigned)nb, 256, 0, s>>>(dt, b->d_tfb + b->tfsf_off[g], g);
  };
  sweeps(k_march_h_tma_batch<T, kMTJ, 32, MF, false, true>,
         k_march_h_tma_batch<T, kMTJ, 32, MF, false, false>,
         k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 1>,
         k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 2>,
         k_march_h_tma_batch<T, kMTJ, 32, MF, true, false, 4>,
         k_march_h_tma_batch<T, kMTJ, 32, MS, true, false>);
  if (b->n_edge) k_edge_batch<T, false><<<(unsigned)b->n_edge, 256, 0, s>>>(dy, b->d_edge);
  tfsf(0);
  tfsf(1);
  sweeps(k_march_e_tma_batch<T, kMTJ, 32, MF, false, true>,
         k_march_e_tma_batch<T, kMTJ, 32, MF, false, false>,
         k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 1>,
         k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 2>,
         k_march_e_tma_batch<T, kMTJ, 32, MF, true, false, 4>,
         k_march_e_tma_batch<T, kMTJ, 32, MS, true, false>);
  if (b->n_edge) k_edge_batch<T, true><<<(unsigned)b->n_edge, 256, 0, s>>>(dy, b->d_edge);
  tfsf(2);
  tfsf(3);
  const int n = (int)b->eng.size();
  k_advance_batch<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(b->d_steps, n);
  if (cerr != cudaSuccess) return cerr;
  return cudaGetLastError();
}

cudaError_t batch_enqueue(xfd_batch* b) {
  return b->precision == XFD_FP64 ? batch_enqueue_t<double>(b) : batch_enqueue_t<float>(b);
}

xfd_status batch_prepare_any(xfd_batch* b) {
  return b->precision == XFD_FP64 ? batch_prepare<double>(b) : batch_prepare<float>(b);
}

xfd_status batch_build_graph(xfd_batch* b, long long len) {
  batch_drop_graph(b);
  cudaGraph_t g = nullptr;
  BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  for (long long q = 0; q < len; ++q) {
    cudaError_t c = batch_enqueue(b);
    if (c != cudaSuccess) {
      cudaGraph_t dummy = nullptr;
      cudaStreamEndCapture(b->stream, &dummy);
      if (dummy) cudaGraphDestroy(dummy);
      return bfail(b, XFD_ERR_CUDA, "batched launch during capture: %s", cudaGetErrorString(c));
    }
  }
  BATCH_TRY(b, cudaStreamEndCapture(b->stream, &g));
  cudaError_t c = cudaGraphInstantiate(&b->graph_exec, g, 0);
  cudaGraphDestroy(g);
  if (c != cudaSuccess)
    return bfail(b, XFD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(c));
  BATCH_TRY(b, cudaGraphUpload(b->graph_exec, b->stream));
  b->graph_len = len;
  return XFD_OK;
}

// Runs `n` steps of the prepared batch: graph chunks, then single steps.
xfd_status batch_steps(xfd_batch* b, long long n) {
  long long left = n;
  while (left > 0) {
    if (b->use_graph && left >= b->graph_chunk) {
      if (!b->graph_exec || b->graph_len != b->graph_chunk) {
        xfd_status s = batch_build_graph(b, b->graph_chunk);
        if (s != XFD_OK) return s;
      }
      BATCH_TRY(b, cudaGraphLaunch(b->graph_exec, b->stream));
      left -= b->graph_len;
      continue;
    }
    cudaError_t c = batch_enqueue(b);
    if (c != cudaSuccess) return bfail(b, XFD_ERR_CUDA, "batched step: %s", cudaGetErrorString(c));
    left -= 1;
  }
  return XFD_OK;
}

// Candidates of the autotuner: the queue form with tile rows 8 and 16, then
// the launch per phase and form (8 rows), each at the depths below.
constexpr int kTuneDepths[] = {8, 16, 32, 64};
constexpr int kTuneCandidates = 12;

void tune_candidate(int c, int* queue, int* rows, int* depth) {
  *queue = c < 8 ? 1 : 0;
  *rows = c < 4 ? kMTJ : c < 8 ? kWideTJ : kMTJ;
  *depth = kTuneDepths[c % 4];
}

// Times each candidate (form, tile rows, x chunk length) on 1 + K steps of
// the run (K in one graph, by CUDA events) and keeps the fastest.  Returns
// the steps consumed.
xfd_status batch_autotune(xfd_batch* b, long long* used) {
  *used = 0;
  const int K = b->autotune;
  b->tune_ms.clear();
  int best = b->march_ichunk, best_rows = b->tile_rows, best_queue = b->queue ? 1 : 0;
  double best_ms = 0;
  for (int c_i = 0; c_i < kTuneCandidates; ++c_i) {
    int queue, rows, d;
    tune_candidate(c_i, &queue, &rows, &d);
    b->queue = queue != 0;
    b->march_ichunk = d;
    b->tile_rows = rows;
    xfd_status s = batch_prepare_any(b);
    if (s != XFD_OK) return s;
    cudaError_t c = batch_enqueue(b);  // warm-up step
    if (c != cudaSuccess) return bfail(b, XFD_ERR_CUDA, "batched step: %s", cudaGetErrorString(c));
    if ((s = batch_build_graph(b, K)) != XFD_OK) return s;
    BATCH_TRY(b, cudaEventRecord(b->t0, b->stream));
    BATCH_TRY(b, cudaGraphLaunch(b->graph_exec, b->stream));
    BATCH_TRY(b, cudaEventRecord(b->t1, b->stream));
    BATCH_TRY(b, cudaEventSynchronize(b->t1));
    float ms = 0;
    BATCH_TRY(b, cudaEventElapsedTime(&ms, b->t0, b->t1));
    const double per = (double)ms / K;
    b->tune_ms.push_back({queue, rows, d, per});
    if (b->tune_ms.size() == 1 || per < best_ms) {
      best = d;
      best_rows = rows;
      best_queue = queue;
      best_ms = per;
    }
    *used += 1 + K;
  }
  b->autotune = 0;
  if (best != b->march_ichunk || best_rows != b->tile_rows || (best_queue != 0) != b->queue) {
    b->march_ichunk = best;
    b->tile_rows = best_rows;
    b->queue = best_queue != 0;
    xfd_status s = batch_prepare_any(b);
    if (s != XFD_OK) return s;
  }
  batch_drop_graph(b);
  return XFD_OK;
}

}  // namespace

extern "C" {

xfd_status xfd_batch_create(xfd_engine* const* engines, int32_t n, xfd_batch** out) {
  if (!engines || !out || n < 1) return bfail(nullptr, XFD_ERR_INVALID_ARGUMENT, "bad batch");
  if (n > 0xffff)  // queue items carry the lattice in 16 bits
    return bfail(nullptr, XFD_ERR_INVALID_ARGUMENT, "more than 65535 engines in one batch");
  *out = nullptr;
  for (int32_t s = 0; s < n; ++s) {
    const xfd_engine* e = engines[s];
    if (!e) return bfail(nullptr, XFD_ERR_INVALID_ARGUMENT, "null engine %d", s);
    if (e->device != engines[0]->device || e->precision != engines[0]->precision)
      return bfail(nullptr, XFD_ERR_INVALID_ARGUMENT,
                   "engine %d: all batched engines need one device and one precision", s);
    if (e->ade_kind >= 0 || !e->lumped_h.empty() || !e->movies.empty() || e->have_nf2ff ||
        e->have_td || e->n_ovr || e->n_hterm || e->pr_begin.size() > 1 || !e->ind_h.empty())
      return bfail(nullptr, XFD_ERR_UNSUPPORTED,
                   "engine %d: ADE media, lumped sources and inductors, movies, NF2FF, probes "
                   "and coefficient overrides are not batched", s);
    if (is_fused(e) && e->cur != 0)
      return bfail(nullptr, XFD_ERR_STATE,
                   "engine %d: fields are in the second buffer of a fused sweep", s);
    for (int32_t r = 0; r < s; ++r)
      if (engines[r] == e) return bfail(nullptr, XFD_ERR_INVALID_ARGUMENT, "engine %d twice", s);
  }
  auto b = std::make_unique<xfd_batch>();
  b->device = engines[0]->device;
  b->precision = engines[0]->precision;
  b->eng.assign(engines, engines + n);
  std::stable_sort(b->eng.begin(), b->eng.end(),
                   [](const xfd_engine* x, const xfd_engine* y) { return x->n_lat > y->n_lat; });
  cudaError_t c = cudaSetDevice(b->device);
  if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (c == cudaSuccess) c = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (c == cudaSuccess) c = cudaEventCreate(&b->t0);
  if (c == cudaSuccess) c = cudaEventCreate(&b->t1);
  if (c == cudaSuccess) c = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
  for (int q = 0; q < 3 && c == cudaSuccess; ++q) {
    c = cudaStreamCreateWithFlags(&b->side[q], cudaStreamNonBlocking);
    if (c == cudaSuccess) c = cudaEventCreateWithFlags(&b->join_ev[q], cudaEventDisableTiming);
  }
  if (c != cudaSuccess) {
    for (int q = 0; q < 3; ++q) {
      if (b->join_ev[q]) cudaEventDestroy(b->join_ev[q]);
      if (b->side[q]) cudaStreamDestroy(b->side[q]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    return bfail(nullptr, XFD_ERR_CUDA, "batch stream: %s", cudaGetErrorString(c));
  }
  *out = b.release();
  return XFD_OK;
}

void xfd_batch_destroy(xfd_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  batch_free_tables(b);
  for (int q = 0; q < 3; ++q) {
    if (b->side[q]) cudaStreamSynchronize(b->side[q]);
    if (b->join_ev[q]) cudaEventDestroy(b->join_ev[q]);
    if (b->side[q]) cudaStreamDestroy(b->side[q]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* xfd_batch_last_error(const xfd_batch* b) {
  return b ? b->err.c_str() : g_create_error.c_str();
}

xfd_status xfd_batch_run(xfd_batch* b, int64_t n) {
  if (!b) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "null batch");
  if (n < 0) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "negative step count");
  for (size_t s = 0; s < b->eng.size(); ++s) {
    const xfd_engine* e = b->eng[s];
    if (e->host_step + n > e->n_steps)
      return bfail(b, XFD_ERR_INVALID_ARGUMENT, "lattice %zu: run past n_steps (%lld + %lld > %lld)",
                   s, (long long)e->host_step, (long long)n, (long long)e->n_steps);
  }
  // A member engine run alone in a fused (ping-pong) sweep since the tables
  // were built may hold its fields in the other buffer: rebuild them.
  if (b->ready) {
    for (size_t s = 0; s < b->eng.size(); ++s) {
      if (s >= b->cur_at_prepare.size() || b->eng[s]->cur != b->cur_at_prepare[s]) {
        b->ready = false;
        break;
      }
    }
  }
  BATCH_TRY(b, cudaSetDevice(b->device));
  // Order after each engine's own queued work (uploads, earlier runs).
  for (xfd_engine* e : b->eng) {
    BATCH_TRY(b, cudaEventRecord(b->ev, e->stream));
    BATCH_TRY(b, cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  xfd_status st;
  if (!b->ready && (st = batch_prepare_any(b)) != XFD_OK) return st;
  long long left = n;
  const long long tune_steps = (long long)kTuneCandidates * (1 + (long long)b->autotune);
  if (b->autotune > 0 && left >= tune_steps) {
    long long used = 0;
    if ((st = batch_autotune(b, &used)) != XFD_OK) return st;
    left -= used;
  }
  if ((st = batch_steps(b, left)) != XFD_OK) return st;
  // Later work on each engine's stream (downloads, single runs) follows the batch.
  BATCH_TRY(b, cudaEventRecord(b->ev, b->stream));
  for (xfd_engine* e : b->eng) {
    BATCH_TRY(b, cudaStreamWaitEvent(e->stream, b->ev, 0));
    e->host_step += n;
  }
  return XFD_OK;
}

xfd_status xfd_batch_sync(xfd_batch* b) {
  if (!b) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "null batch");
  BATCH_TRY(b, cudaSetDevice(b->device));
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  for (size_t s = 0; s < b->eng.size(); ++s) {
    int err = 0;
    BATCH_TRY(b, cudaMemcpy(&err, b->eng[s]->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err & 2)
      return bfail(b, XFD_ERR_TIMEOUT, "lattice %zu: a sweep stage or queue wait ran out of time",
                   s);
    if (err)
      return bfail(b, XFD_ERR_NUMERIC, "lattice %zu: TFSF projection left the incident grid", s);
  }
  return XFD_OK;
}

xfd_status xfd_batch_get_option(const xfd_batch* b, const char* name, int64_t* value) {
  xfd_batch* m = const_cast<xfd_batch*>(b);
  if (!b || !name || !value) return bfail(m, XFD_ERR_INVALID_ARGUMENT, "null option");
  if (!strcmp(name, "graph")) *value = b->use_graph ? 1 : 0;
  else if (!strcmp(name, "graph_chunk")) *value = b->graph_chunk;
  else if (!strcmp(name, "march_ichunk")) *value = b->march_ichunk;
  else if (!strcmp(name, "autotune")) *value = b->autotune;
  else if (!strcmp(name, "march_split_axes")) *value = b->split_axes ? 1 : 0;
  else if (!strcmp(name, "queue")) *value = b->queue ? 1 : 0;
  else if (!strcmp(name, "concurrent")) *value = b->concurrent ? 1 : 0;
  else if (!strcmp(name, "tile_rows")) *value = b->tile_rows;
  else if (!strcmp(name, "queue_wait_cycles")) *value = b->queue_wait;
  else if (!strcmp(name, "queue_stall_test")) *value = b->queue_stall_test ? 1 : 0;
  else return bfail(m, XFD_ERR_INVALID_ARGUMENT, "unknown option '%s'", name);
  return XFD_OK;
}

xfd_status xfd_batch_set_option(xfd_batch* b, const char* name, int64_t value) {
  if (!b || !name) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "null option");
  if (!strcmp(name, "graph")) {
    b->use_graph = value != 0;
  } else if (!strcmp(name, "graph_chunk")) {
    if (value < 1 || value > 4096) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "graph_chunk range");
    b->graph_chunk = (int)value;
    batch_drop_graph(b);
  } else if (!strcmp(name, "march_ichunk")) {
    if (value < 1 || value > 4096) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "march_ichunk range");
    b->march_ichunk = (int)value;
    b->ready = false;
    batch_drop_graph(b);
  } else if (!strcmp(name, "autotune")) {
    if (value < 0 || value > 4096) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "autotune range");
    b->autotune = (int)value;
  } else if (!strcmp(name, "march_split_axes")) {
    b->split_axes = value != 0;
    b->ready = false;
    batch_drop_graph(b);
  } else if (!strcmp(name, "queue")) {
    b->queue = value != 0;
    b->ready = false;
    batch_drop_graph(b);
  } else if (!strcmp(name, "concurrent")) {
    b->concurrent = value != 0;
    batch_drop_graph(b);
  } else if (!strcmp(name, "tile_rows")) {
    if (value != kMTJ && value != kWideTJ)
      return bfail(b, XFD_ERR_INVALID_ARGUMENT, "tile_rows must be %d or %d", kMTJ, kWideTJ);
    if (value != kMTJ && !b->queue)
      return bfail(b, XFD_ERR_UNSUPPORTED, "tile_rows %d needs the queue form", (int)value);
    b->tile_rows = (int)value;
    b->ready = false;
    batch_drop_graph(b);
  } else if (!strcmp(name, "queue_wait_cycles")) {
    if (value < 0) return bfail(b, XFD_ERR_INVALID_ARGUMENT, "queue_wait_cycles < 0");
    b->queue_wait = value;
    batch_drop_graph(b);
  } else if (!strcmp(name, "queue_stall_test")) {
    b->queue_stall_test = value != 0;
    b->ready = false;
    batch_drop_graph(b);
  } else {
    return bfail(b, XFD_ERR_INVALID_ARGUMENT, "unknown option '%s'", name);
  }
  return XFD_OK;
}

xfd_status xfd_batch_tuning(const xfd_batch* b, int32_t* depth, double* ms_per_step,
                            int32_t capacity, int32_t* count) {
  return xfd_batch_tuning_shapes(b, nullptr, nullptr, depth, ms_per_step, capacity, count);
}

xfd_status xfd_batch_tuning_shapes(const xfd_batch* b, int32_t* queue, int32_t* rows,
                                   int32_t* depth, double* ms_per_step, int32_t capacity,
                                   int32_t* count) {
  if (!b || !count) return bfail(const_cast<xfd_batch*>(b), XFD_ERR_INVALID_ARGUMENT, "null");
  *count = (int32_t)b->tune_ms.size();
  for (int32_t q = 0; q < *count && q < capacity; ++q) {
    if (queue) queue[q] = b->tune_ms[(size_t)q].queue;
    if (rows) rows[q] = b->tune_ms[(size_t)q].rows;
    if (depth) depth[q] = b->tune_ms[(size_t)q].depth;
    if (ms_per_step) ms_per_step[q] = b->tune_ms[(size_t)q].ms;
  }
  return XFD_OK;
}

int32_t xfd_batch_launches_per_step(const xfd_batch* b) {
  if (!b || !b->ready) return 0;
  if (b->queue) return 1;
  int n = 1;  // step counters
  for (int f = 0; f < 6; ++f) n += b->tile_off[f + 1] > b->tile_off[f] ? 2 : 0;
  if (b->n_edge) n += 2;
  for (int g = 0; g < 4; ++g) n += b->tfsf_off[g + 1] > b->tfsf_off[g] ? 1 : 0;
  return n;
}

int32_t xfd_batch_size(const xfd_batch* b) { return b ? (int32_t)b->eng.size() : 0; }

void* xfd_batch_stream(xfd_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"
