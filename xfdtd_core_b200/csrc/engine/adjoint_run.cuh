// Saved states and the adjoint driver.  Part of engine.cu's translation
// unit (it uses the engine internals defined there).
//
// A saved state (xfd_checkpoint_save / _load) is a device copy of what the
// next step reads: the six field arrays of the current buffer, the CPML psi
// arrays, the ADE currents and the step counter.  Movie frames are outputs
// and are not rewound; engines with NF2FF surfaces save states but refuse to
// load them, because their running DFT sums cannot be rewound.
//
// xfd_adjoint_run: forward n steps from the current state, saving the state
// every K steps and recording the objective component over its node box
// each step; the caller's objective turns the record into J and dJ/drecord;
// the reverse pass then walks the segments from the last to the first:
// restore the segment's saved state, recompute its K steps while recording
// E over the design box (K + 1 rows: memory stays bounded by the segment),
// and run K reverse steps (k_adj_h, the sensitivity sums, k_adj_e, the
// objective's adjoint source).  The forward state at the end of the run is
// restored last, so the engine is left as a plain forward run would leave
// it.  Cost: one forward run, one recomputation, one reverse run.

namespace {

struct StateRegion {
  void* p;
  size_t bytes;
};

size_t slab_cells(const xfd_engine* e, const xfd_engine::Slab& S) {
  if (S.m == 0) return (size_t)S.n * e->L.NY * e->L.KP;
  if (S.m == 1) return (size_t)(e->L.nx + 1) * S.n * e->L.KP;
  return (size_t)(e->L.nx + 1) * e->L.NY * S.n;
}

std::vector<StateRegion> state_regions(xfd_engine* e) {
  std::vector<StateRegion> r;
  for (int c = 0; c < 6; ++c) r.push_back({e->fbuf[e->cur][c], (size_t)e->n_lat * e->wsize});
  for (const auto& S : e->slabs) {
    const size_t b = slab_cells(e, S) * e->wsize;
    for (int w = 0; w < 2; ++w) {
      r.push_back({S.psi_e[w], b});
      r.push_back({S.psi_h[psi_h_buf(e)][w], b});
    }
  }
  if (e->ade_kind >= 0) {
    const bool d = e->precision == XFD_FP64;
    const long long n = d ? e->ade64.n : e->ade32.n;
    const int np = d ? e->ade64.np : e->ade32.np;
    void* j = d ? (void*)e->ade64.j : (void*)e->ade32.j;
    void* jp = d ? (void*)e->ade64.jp : (void*)e->ade32.jp;
    void* ep = d ? (void*)e->ade64.ep : (void*)e->ade32.ep;
    r.push_back({j, (size_t)n * np * e->wsize});
    if (jp) r.push_back({jp, (size_t)n * np * e->wsize});
    if (ep) r.push_back({ep, (size_t)n * e->wsize});
  }
  if (e->ind.n > 0) r.push_back({e->ind.j, (size_t)e->ind.n * sizeof(double)});
  r.push_back({e->d_step, sizeof(long long)});
  return r;
}

size_t state_bytes(xfd_engine* e) {
  size_t b = 0;
  for (const auto& r : state_regions(e)) b += (r.bytes + 255) / 256 * 256;
  return b;
}

xfd_status state_copy(xfd_engine* e, xfd_engine::Ckpt& c, bool save) {
  size_t off = 0;
  for (const auto& r : state_regions(e)) {
    char* slot = static_cast<char*>(c.buf) + off;
    CUDA_TRY(e, cudaMemcpyAsync(save ? (void*)slot : r.p, save ? r.p : (const void*)slot, r.bytes,
                                cudaMemcpyDeviceToDevice, e->stream));
    off += (r.bytes + 255) / 256 * 256;
  }
  if (save) {
    c.step = e->host_step;
  } else {
    e->host_step = c.step;
    // Ping-pong sweeps: the other buffer gets the same fields, so that nodes
    // no kernel writes hold equal values in both (the sweeps then skip them).
    if (is_pingpong(e))
      for (int q = 0; q < 6; ++q)
        CUDA_TRY(e, cudaMemcpyAsync(e->fbuf[1 - e->cur][q], e->fbuf[e->cur][q],
                                    (size_t)e->n_lat * e->wsize, cudaMemcpyDeviceToDevice,
                                    e->stream));
  }
  return XFD_OK;
}

xfd_status ckpt_save(xfd_engine* e, xfd_engine::Ckpt& c) {
  const size_t need = state_bytes(e);
  if (c.buf && c.bytes != need) {
    CUDA_TRY(e, cudaStreamSynchronize(e->stream));
    cudaFree(c.buf);
    c.buf = nullptr;
  }
  if (!c.buf) {
    cudaError_t r = cudaMalloc(&c.buf, need);
    if (r != cudaSuccess) {
      c.buf = nullptr;
      return fail(e, r == cudaErrorMemoryAllocation ? XFD_ERR_OUT_OF_MEMORY : XFD_ERR_CUDA,
                  "checkpoint cudaMalloc(%zu): %s", need, cudaGetErrorString(r));
    }
    c.bytes = need;
  }
  return state_copy(e, c, true);
}

void ckpt_free(xfd_engine::Ckpt& c) {
  if (c.buf) cudaFree(c.buf);
  c = xfd_engine::Ckpt{};
}

// Device buffers of an adjoint run, taken in a fixed order from the
// engine's kept buffers (reused while the size matches, else reallocated)
// and zeroed on the run's stream.
struct AdjBuffers {
  xfd_engine* e;
  size_t next = 0;
};

xfd_status adj_alloc(xfd_engine* e, AdjBuffers& B, void** out, size_t bytes) {
  bytes = std::max<size_t>(bytes, 16);
  if (B.next < e->adj_bufs.size() && e->adj_sizes[B.next] != bytes) {
    CUDA_TRY(e, cudaStreamSynchronize(e->stream));
    cudaFree(e->adj_bufs[B.next]);
    e->adj_bufs[B.next] = nullptr;
  }
  if (B.next >= e->adj_bufs.size()) {
    e->adj_bufs.push_back(nullptr);
    e->adj_sizes.push_back(0);
  }
  if (!e->adj_bufs[B.next]) {
    cudaError_t r = cudaMalloc(&e->adj_bufs[B.next], bytes);
    if (r != cudaSuccess) {
      e->adj_bufs[B.next] = nullptr;
      *out = nullptr;
      return fail(e, r == cudaErrorMemoryAllocation ? XFD_ERR_OUT_OF_MEMORY : XFD_ERR_CUDA,
                  "adjoint cudaMalloc(%zu): %s", bytes, cudaGetErrorString(r));
    }
    e->adj_sizes[B.next] = bytes;
  }
  *out = e->adj_bufs[B.next++];
  CUDA_TRY(e, cudaMemsetAsync(*out, 0, bytes, e->stream));
  return XFD_OK;
}

// Tiles of the split marching sweeps (k tiles of 32, j tiles of kMTJ, x
// chunks of `ich` planes, the grid moved by shift[g] nodes) on which the
// scaled reverse step is the forward step: every node of the tile and its
// neighbours one node away lie in no CPML layer and strictly inside the
// lattice (main update range of every component), and the curl factors fe,
// fh are one value per axis there.  Per axis the shift (a multiple of 8
// nodes along k) and the run of tiles that cover the most nodes; an empty
// box when some axis has none.
void adjoint_split(const xfd_engine* e, int ich, int lo[3], int hi[3], int shift[3]) {
  const Lat& L = e->L;
  const int size[3] = {32, kMTJ, ich};
  const int n_nodes[3] = {L.nz + 1, L.ny + 1, L.nx + 1};
  const int axis_of[3] = {2, 1, 0};  // grid dimension -> lattice axis
  // k shifts in steps of 8 nodes: every TMA x coordinate stays a multiple of
  // 16 bytes for the field maps (4 or 8 bytes per value) and for the uint16
  // class map alike.
  const int step[3] = {8, 1, 1};
  for (int g = 0; g < 3; ++g) {
    const int m = axis_of[g];
    const int n_cells = n_nodes[g] - 1;
    lo[g] = hi[g] = shift[g] = 0;
    int best_len = 0;
    for (int sh = 0; sh < size[g]; sh += step[g]) {
      const int nt = (n_nodes[g] - sh + size[g] - 1) / size[g];
      auto ok = [&](int b) {
        const int a0 = sh + b * size[g] - 1;
        const int a1 = std::min(sh + (b + 1) * size[g], n_nodes[g]) - 1 + 1;
        if (a0 < 1 || a1 > n_cells - 1) return false;
        for (const auto& S : e->slabs) {
          if (S.m != m) continue;
          if (a0 < S.e_lo + S.n && S.e_lo <= a1) return false;
          if (a0 < S.h_lo + S.n && S.h_lo <= a1) return false;
        }
        // One curl factor per axis: spacings computed as differences of
        // node coordinates may differ in their last bits, so equal within
        // 1e-12 relative (the forward sweep's destination weights then stand
        // for the transpose's source weights, far below a step's rounding).
        const double f = e->fe_h[m][(size_t)a0];
        for (int x = a0; x <= a1; ++x)
          if (std::fabs(e->fe_h[m][(size_t)x] - f) > 1e-12 * std::fabs(f) ||
              std::fabs(e->fh_h[m][(size_t)x] - f) > 1e-12 * std::fabs(f))
            return false;
        return true;
      };
      for (int b = 0; b < nt;) {
        if (!ok(b)) {
          ++b;
          continue;
        }
        int c = b;
        while (c < nt && ok(c)) ++c;
        if (c - b > best_len) {
          best_len = c - b;
          lo[g] = b;
          hi[g] = c;
          shift[g] = sh;
        }
        b = c;
      }
    }
  }
}

// Fork side stream 0 from `st` / join it back (the adjoint's reverse step).
cudaError_t side_fork(xfd_engine* e, cudaStream_t st) {
  cudaError_t c = cudaEventRecord(e->fork_ev, st);
  return c == cudaSuccess ? cudaStreamWaitEvent(e->side[0], e->fork_ev, 0) : c;
}

cudaError_t side_join(xfd_engine* e, cudaStream_t st) {
  cudaError_t c = cudaEventRecord(e->join_ev[0], e->side[0]);
  return c == cudaSuccess ? cudaStreamWaitEvent(st, e->join_ev[0], 0) : c;
}

bool box_ok(const Lat& L, const int32_t s[3], const int32_t t[3]) {
  const int n[3] = {L.nx, L.ny, L.nz};
  for (int a = 0; a < 3; ++a)
    if (s[a] < 0 || t[a] <= s[a] || t[a] > n[a] + 1) return false;
  return true;
}

long long box_nodes(const int32_t s[3], const int32_t t[3]) {
  return (long long)(t[0] - s[0]) * (t[1] - s[1]) * (t[2] - s[2]);
}

template <typename T>
void set_rec(xfd_engine* e, int r, const BoxRecD<T>& d) {
  if constexpr (sizeof(T) == 8) e->rec64[r] = d; else e->rec32[r] = d;
}

template <typename T>
xfd_status adjoint_run_t(xfd_engine* e, const xfd_adjoint_desc* d, double* value, double* sens) {
  const Lat L = e->L;
  const long long N = d->n_steps, K = d->forward_only ? N : d->checkpoint_interval;
  const long long S = (N + K - 1) / K;
  const long long t0 = e->host_step;
  const long long n_obj = box_nodes(d->obj_s, d->obj_e);
  const long long n_des = box_nodes(d->design_s, d->design_e);
  cudaStream_t st = e->stream;
  AdjBuffers B{e};
  xfd_status s;
  void *rec = nullptr, *hist = nullptr, *src = nullptr, *g = nullptr, *lamp = nullptr;
  if ((s = adj_alloc(e, B, &rec, (size_t)N * n_obj * sizeof(T))) != XFD_OK) return s;
  if (d->forward_only) {
    BoxRecD<T> ro{};
    for (int q = 0; q < 3; ++q) {
      ro.s[q] = d->obj_s[q];
      ro.e[q] = d->obj_e[q];
    }
    ro.c0 = d->obj_field;
    ro.nc = 1;
    ro.n = n_obj;
    ro.base = t0;
    ro.rows = N;
    ro.dst = static_cast<T*>(rec);
    set_rec<T>(e, 0, ro);
    e->n_rec = 1;
    e->graph_dirty = true;
    s = xfd_run(e, N);
    e->n_rec = 0;
    e->graph_dirty = true;
    if (s != XFD_OK) return s;
    std::vector<T> rec_h((size_t)(N * n_obj));
    CUDA_TRY(e, cudaMemcpyAsync(rec_h.data(), rec, rec_h.size() * sizeof(T),
                                cudaMemcpyDeviceToHost, st));
    CUDA_TRY(e, cudaStreamSynchronize(st));
    std::vector<double> rec_d(rec_h.begin(), rec_h.end()), drec(rec_h.size(), 0.0);
    double J = 0.0;
    if (d->objective(d->user, N, n_obj, rec_d.data(), drec.data(), &J) != 0)
      return fail(e, XFD_ERR_NUMERIC, "objective callback failed");
    if (value) *value = J;
    return XFD_OK;
  }
  if ((s = adj_alloc(e, B, &hist, (size_t)(K + 1) * 3 * n_des * sizeof(T))) != XFD_OK) return s;
  if ((s = adj_alloc(e, B, &src, (size_t)N * n_obj * sizeof(double))) != XFD_OK) return s;
  if ((s = adj_alloc(e, B, &g, (size_t)6 * n_des * sizeof(double))) != XFD_OK) return s;
  if ((s = adj_alloc(e, B, &lamp, 6 * sizeof(void*))) != XFD_OK) return s;
  void* lam[6];
  for (int c = 0; c < 6; ++c)
    if ((s = adj_alloc(e, B, &lam[c], (size_t)e->n_lat * e->wsize)) != XFD_OK) return s;
  CUDA_TRY(e, cudaMemcpyAsync(lamp, lam, sizeof lam, cudaMemcpyHostToDevice, st));
  YeeP<T> a = yee_params<T>(e);
  for (int c = 0; c < 6; ++c) a.f[c] = static_cast<T*>(lam[c]);
  // The same scaled fields and CPML adjoints in the marching-sweep layout.
  MarchP<T> ap = march_params<T>(e);
  for (int c = 0; c < 6; ++c) ap.f[c] = static_cast<T*>(lam[c]);
  int slot_of[3] = {0, 0, 0};
  for (size_t q = 0; q < e->slabs.size(); ++q) {
    const size_t b = slab_cells(e, e->slabs[q]) * e->wsize;
    SlabAxisD<T>& A = ap.slab[e->slabs[q].m];
    const int slot = slot_of[e->slabs[q].m]++;
    for (int w = 0; w < 2; ++w) {
      void *pe = nullptr, *ph = nullptr;
      if ((s = adj_alloc(e, B, &pe, b)) != XFD_OK) return s;
      if ((s = adj_alloc(e, B, &ph, b)) != XFD_OK) return s;
      a.slab[q].psi_e[w] = static_cast<T*>(pe);
      a.slab[q].psi_h[w] = static_cast<T*>(ph);
      A.psi_e[slot][w] = static_cast<T*>(pe);
      A.psi_h_in[slot][w] = static_cast<const T*>(ph);
      A.psi_h_out[slot][w] = static_cast<T*>(ph);
    }
  }
  T* const* lam_dev = static_cast<T* const*>(lamp);
  if (e->adj_ck.size() < (size_t)S + 1) e->adj_ck.resize((size_t)S + 1);
  std::vector<xfd_engine::Ckpt>& ck = e->adj_ck;
  // Coefficient overrides as dense arrays over their bounding node box.
  OvBoxD<T> ov{};
  if (e->n_ovr) {
    for (int q = 0; q < 3; ++q) {
      ov.s[q] = INT32_MAX;
      ov.e[q] = INT32_MIN;
    }
    for (long long q = 0; q < e->n_ovr; ++q)
      for (int a2 = 0; a2 < 3; ++a2) {
        ov.s[a2] = std::min(ov.s[a2], e->ovr_node[(size_t)(3 * q + a2)]);
        ov.e[a2] = std::max(ov.e[a2], e->ovr_node[(size_t)(3 * q + a2)] + 1);
      }
    ov.n = (long long)(ov.e[0] - ov.s[0]) * (ov.e[1] - ov.s[1]) * (ov.e[2] - ov.s[2]);
    std::vector<T> hca((size_t)(3 * ov.n), T(0)), hcb((size_t)(3 * ov.n), T(0));
    for (long long q = 0; q < e->n_ovr; ++q) {
      const int32_t* x = &e->ovr_node[(size_t)(3 * q)];
      const long long p = ((long long)(x[0] - ov.s[0]) * (ov.e[1] - ov.s[1]) + (x[1] - ov.s[1])) *
                              (ov.e[2] - ov.s[2]) +
                          (x[2] - ov.s[2]);
      hca[(size_t)(e->ovr_comp[(size_t)q] * ov.n + p)] = (T)e->ovr_ca[(size_t)q];
      hcb[(size_t)(e->ovr_comp[(size_t)q] * ov.n + p)] = (T)e->ovr_cb[(size_t)q];
    }
    void *dca = nullptr, *dcb = nullptr;
    if ((s = adj_alloc(e, B, &dca, hca.size() * sizeof(T))) != XFD_OK) return s;
    if ((s = adj_alloc(e, B, &dcb, hcb.size() * sizeof(T))) != XFD_OK) return s;
    CUDA_TRY(e, cudaMemcpyAsync(dca, hca.data(), hca.size() * sizeof(T), cudaMemcpyHostToDevice,
                                st));
    CUDA_TRY(e, cudaMemcpyAsync(dcb, hcb.data(), hcb.size() * sizeof(T), cudaMemcpyHostToDevice,
                                st));
    CUDA_TRY(e, cudaStreamSynchronize(st));
    ov.ca = static_cast<const T*>(dca);
    ov.cb = static_cast<const T*>(dcb);
  }

  // Forward: state saved at the start of every segment, objective recorded.
  BoxRecD<T> ro{};
  for (int q = 0; q < 3; ++q) {
    ro.s[q] = d->obj_s[q];
    ro.e[q] = d->obj_e[q];
  }
  ro.c0 = d->obj_field;
  ro.nc = 1;
  ro.n = n_obj;
  ro.base = t0;
  ro.shift = 0;
  ro.rows = N;
  ro.dst = static_cast<T*>(rec);
  set_rec<T>(e, 0, ro);
  e->n_rec = 1;
  e->graph_dirty = true;
  // The design history of the last segment is recorded on the way, so that
  // segment needs no recomputation.
  BoxRecD<T> rd{};
  for (int q = 0; q < 3; ++q) {
    rd.s[q] = d->design_s[q];
    rd.e[q] = d->design_e[q];
  }
  rd.c0 = 0;
  rd.nc = 3;
  rd.n = n_des;
  rd.rows = K + 1;
  rd.dst = static_cast<T*>(hist);
  const unsigned db = blocks_for(3 * n_des, 256);
  for (long long q = 0; q < S; ++q) {
    if ((s = ckpt_save(e, ck[(size_t)q])) != XFD_OK) break;
    if (q == S - 1) {
      rd.base = t0 + q * K;
      rd.shift = 0;
      // E at the segment start (the buffer holding it: ping-pong sweeps alternate)
      T* const* fields = reinterpret_cast<T* const*>(e->d_fields[e->cur]);
      k_box_record<T><<<db, 256, 0, st>>>(rd, L, fields, e->d_step);
      rd.shift = 1;
      set_rec<T>(e, 1, rd);
      e->n_rec = 2;
      e->graph_dirty = true;
    }
    if ((s = xfd_run(e, std::min(K, N - q * K))) != XFD_OK) break;
  }
  e->n_rec = 0;
  e->graph_dirty = true;
  if (s != XFD_OK) return s;
  if ((s = ckpt_save(e, ck[(size_t)S])) != XFD_OK) return s;

  // Objective on the host.
  std::vector<T> rec_h((size_t)(N * n_obj));
  CUDA_TRY(e, cudaMemcpyAsync(rec_h.data(), rec, rec_h.size() * sizeof(T),
                              cudaMemcpyDeviceToHost, st));
  CUDA_TRY(e, cudaStreamSynchronize(st));
  std::vector<double> rec_d(rec_h.begin(), rec_h.end()), drec(rec_h.size(), 0.0);
  double J = 0.0;
  if (d->objective(d->user, N, n_obj, rec_d.data(), drec.data(), &J) != 0)
    return fail(e, XFD_ERR_NUMERIC, "objective callback failed");
  if (value) *value = J;
  CUDA_TRY(e, cudaMemcpyAsync(src, drec.data(), drec.size() * sizeof(double),
                              cudaMemcpyHostToDevice, st));

  // Reverse, on the scaled fields (adjoint.cuh): the CPML-free box with
  // uniform curl factors by the forward marching sweeps over tensor maps of
  // the adjoint arrays, the rest by the transpose-gather kernels.
  BoxRecD<T> rs = ro;
  const double* srcd = static_cast<const double*>(src);
  double* g0 = static_cast<double*>(g);
  double* g1 = g0 + 3 * n_des;
  const unsigned sb = blocks_for(n_obj, 256);
  AdjBox abox{};
  const int ich = e->march_ichunk;
  int alo[3], ahi[3], ash[3];
  adjoint_split(e, ich, alo, ahi, ash);
  const bool has_box = ahi[0] > alo[0] && ahi[1] > alo[1] && ahi[2] > alo[2];
  MarchTmaP<T> am{};
  if (has_box) {
    const int size[3] = {32, kMTJ, ich};
    for (int q = 0; q < 3; ++q) {
      abox.lo[q] = ash[q] + alo[q] * size[q];
      abox.hi[q] = ash[q] + ahi[q] * size[q];
      am.org[q] = alo[q];
      am.box_lo[q] = alo[q];
      am.box_hi[q] = ahi[q];
      am.shift[q] = ash[q];
    }
    abox.org_k = ash[0] % 32 ? ash[0] % 32 - 32 : 0;
    abox.org_j = ash[1] % kMTJ ? ash[1] % kMTJ - kMTJ : 0;
    am.p = ap;
    if ((s = build_march_maps<T>(e, lam, &am.m)) != XFD_OK) return s;
    am.err = e->d_err;
  }
  static_assert(kMTJ == 8, "the gather CTAs are 32 x 8 nodes, the box tiles 32 x kMTJ");
  const dim3 blk(32, 8, 1);
  const dim3 grd((unsigned)((L.nz + 1 - abox.org_k + 31) / 32),
                 (unsigned)((L.ny + 1 - abox.org_j + 7) / 8), (unsigned)(L.nx + 1));
  constexpr int MF = march_free_stages<T>();
  const size_t msm_free = MarchGeom<T, kMTJ, 32>::smem(MF);
  const dim3 gbox((unsigned)(ahi[0] - alo[0]), (unsigned)(ahi[1] - alo[1]),
                  (unsigned)(ahi[2] - alo[2]));
  const dim3 blk_m(32, kMTJ, 1);
  const OverrideD<T> ovd = ovr_of<T>(e);
  k_adj_source<T><<<sb, 256, 0, st>>>(rs, a, ov, srcd + (N - 1) * n_obj);  // dJ/dE^N
  for (long long q = S - 1; q >= 0; --q) {
    const long long base = t0 + q * K, len = std::min(K, N - q * K);
    if (q < S - 1) {  // recompute the segment, recording the design history
      if ((s = state_copy(e, ck[(size_t)q], false)) != XFD_OK) return s;
      rd.base = base;
      rd.shift = 0;
      T* const* fields = reinterpret_cast<T* const*>(e->d_fields[e->cur]);
      k_box_record<T><<<db, 256, 0, st>>>(rd, L, fields, e->d_step);  // E at the segment start
      rd.shift = 1;
      set_rec<T>(e, 0, rd);
      e->n_rec = 1;
      e->graph_dirty = true;
      s = xfd_run(e, len);
      e->n_rec = 0;
      e->graph_dirty = true;
      if (s != XFD_OK) return s;
    }
    for (long long m = len; m >= 1; --m) {
      const long long gstep = q * K + m;  // u holds cb dJ/dE^gstep
      // The box sweep (on a side stream) and the shell gather write disjoint
      // nodes and read only the other field: they run side by side.
      if (has_box) {
        CUDA_TRY(e, side_fork(e, st));
        k_march_h_tma<T, kMTJ, 32, MF, false, true><<<gbox, blk_m, msm_free, e->side[0]>>>(am);
      }
      k_adj_h<T><<<grd, blk, 0, st>>>(ap, abox);
      if (has_box) CUDA_TRY(e, side_join(e, st));
      k_adj_sens<T><<<db, 256, 0, st>>>(rd, a, ov, static_cast<const T*>(hist), (int)m, g0, g1);
      if (e->n_ovr) k_ovr_gather<T><<<blocks_for(e->n_ovr, 256), 256, 0, st>>>(ovd, lam_dev);
      if (has_box) {
        CUDA_TRY(e, side_fork(e, st));
        k_march_e_tma<T, kMTJ, 32, MF, false, true><<<gbox, blk_m, msm_free, e->side[0]>>>(am);
      }
      k_adj_e<T><<<grd, blk, 0, st>>>(ap, abox);
      if (has_box) CUDA_TRY(e, side_join(e, st));
      if (e->n_ovr)
        k_ovr_apply<T><<<blocks_for(e->n_ovr, 256), 256, 0, st>>>(ovd, lam_dev, nullptr);
      if (gstep - 1 >= 1)
        k_adj_source<T><<<sb, 256, 0, st>>>(rs, a, ov, srcd + (gstep - 2) * n_obj);
    }
    CUDA_TRY(e, cudaGetLastError());
  }
  if ((s = state_copy(e, ck[(size_t)S], false)) != XFD_OK) return s;
  CUDA_TRY(e, cudaMemcpyAsync(sens, g, (size_t)6 * n_des * sizeof(double), cudaMemcpyDeviceToHost,
                              st));
  CUDA_TRY(e, cudaStreamSynchronize(st));
  int err = 0;
  CUDA_TRY(e, cudaMemcpy(&err, e->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err & 2) return fail(e, XFD_ERR_TIMEOUT, "a sweep stage wait ran out of time");
  if (err) return fail(e, XFD_ERR_NUMERIC, "TFSF projection left the incident grid");
  return XFD_OK;
}

}  // namespace

extern "C" {

xfd_status xfd_checkpoint_save(xfd_engine* e, int32_t slot) {
  if (!e || slot < 0 || slot > 4095) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad slot");
  CUDA_TRY(e, cudaSetDevice(e->device));
  if (e->ckpts.size() <= (size_t)slot) e->ckpts.resize((size_t)slot + 1);
  return ckpt_save(e, e->ckpts[(size_t)slot]);
}

xfd_status xfd_checkpoint_load(xfd_engine* e, int32_t slot) {
  if (!e || slot < 0 || (size_t)slot >= e->ckpts.size() || !e->ckpts[(size_t)slot].buf)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "no saved state in slot %d", slot);
  // The NF2FF accumulators and the per-step sample ring are running sums over
  // the steps already taken; a state rewound under them would fold samples of
  // steps after the saved one with the phasors of earlier steps.
  if (e->have_nf2ff || e->have_td)
    return fail(e, XFD_ERR_UNSUPPORTED,
                "loading a saved state is not supported on an engine with an NF2FF surface "
                "(its running DFT sums cannot be rewound)");
  CUDA_TRY(e, cudaSetDevice(e->device));
  if (e->ckpts[(size_t)slot].bytes != state_bytes(e))
    return fail(e, XFD_ERR_STATE, "slot %d was saved with another configuration", slot);
  return state_copy(e, e->ckpts[(size_t)slot], false);
}

xfd_status xfd_checkpoint_drop(xfd_engine* e, int32_t slot) {
  if (!e || slot < 0) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad slot");
  if ((size_t)slot >= e->ckpts.size()) return XFD_OK;
  CUDA_TRY(e, cudaSetDevice(e->device));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  ckpt_free(e->ckpts[(size_t)slot]);
  return XFD_OK;
}

int64_t xfd_checkpoint_step(const xfd_engine* e, int32_t slot) {
  if (!e || slot < 0 || (size_t)slot >= e->ckpts.size()) return -1;
  return e->ckpts[(size_t)slot].step;
}

xfd_status xfd_adjoint_run(xfd_engine* e, const xfd_adjoint_desc* d, double* value,
                           double* sens) {
  if (!e || !d || (!sens && !d->forward_only) || !d->objective)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "null adjoint argument");
  if (d->n_steps < 1 || (d->checkpoint_interval < 1 && !d->forward_only))
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "adjoint needs n_steps >= 1 and an interval >= 1");
  if (e->host_step + d->n_steps > e->n_steps)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "run past n_steps (%lld + %lld > %lld)",
                (long long)e->host_step, (long long)d->n_steps, (long long)e->n_steps);
  if (d->obj_field < 0 || d->obj_field > 2 || !box_ok(e->L, d->obj_s, d->obj_e) ||
      (!d->forward_only && !box_ok(e->L, d->design_s, d->design_e)))
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad objective field or node box");
  if (e->ade_kind >= 0 || e->have_nf2ff || e->have_td || !e->movies.empty() ||
      !e->ind_h.empty() || e->n_hterm)
    return fail(e, XFD_ERR_UNSUPPORTED,
                "the adjoint covers CPML, TFSF and lumped sources; not ADE media, inductors, "
                "thin wires, NF2FF or movies");
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s = ensure_ready(e);
  if (s == XFD_OK && !e->tma_ready)
    s = e->precision == XFD_FP64 ? build_tma_maps<double>(e) : build_tma_maps<float>(e);
  if (s != XFD_OK) return s;
  return e->precision == XFD_FP64 ? adjoint_run_t<double>(e, d, value, sens)
                                  : adjoint_run_t<float>(e, d, value, sens);
}

}  // extern "C"
