// Marching split sweeps with TMA-staged planes.  Same arithmetic, ranges and
// correction order as k_march_h / k_march_e (march.cuh); the difference is
// how the per-plane inputs arrive (and that the CPML forms load the old psi
// values of a node one plane ahead): one thread of the CTA issues TMA tile
// loads (cp.async.bulk.tensor, no multicast) of the planes S-1 ahead into a
// ring of S shared-memory stages, each completing on its own mbarrier, so
// that a CTA keeps several planes of DRAM reads in flight while it computes.
// Results are stored straight from registers (coalesced rows along k).
//
// Stage contents (box origins along k are multiples of 32 elements, or that
// minus 16 bytes, so every TMA x coordinate is 16-byte aligned):
//   H sweep, plane i: E_x,E_y,E_z "halo" boxes over j0..j0+TJ, k0..k0+TK+XA-1
//                     (the +1 neighbours along j and k), H_x,H_y,H_z and the
//                     class index over the tile.  The E of plane i+1 comes
//                     from the next stage.
//   E sweep, plane i: H_x,H_y,H_z halo boxes over j0-1..j0+TJ-1,
//                     k0-XA..k0+TK-1 (the -1 neighbours), E_x,E_y,E_z and the
//                     class index over the tile.  The H of plane i-1 is the
//                     previous stage, kept until plane i is done.
// One CTA barrier per plane: a stage is refilled right after the barrier
// that follows its last use.  The (ca, cb) half-rows of the NC most frequent
// material classes (the engine numbers classes by descending node count) are
// read from a shared-memory copy.
// Out-of-range rows, columns and planes read as zeros and are never used.
// The tiles cover k < nz and j < ny; the lattice faces k = nz and j = ny hold
// only boundary nodes and are swept by k_edge_h / k_edge_e (kernels.cuh), so
// no CTA marches through a one-column or one-row remainder tile.
// Stage waits are bounded (a cycle budget); on expiry the CTA sets bit 2 of
// the engine's error word, drains its loads in flight and returns, and later
// launches that find the bit set return at once.
// The batched kernels (k_march_*_tma_batch) run the same CTA body over a tile
// list that spans many lattices, each with its parameters and tensor maps in
// device memory.
#pragma once

#include "march.cuh"
#include "tma.cuh"

namespace xfd {

struct MarchMaps {
  CUtensorMap halo[6];  // box (TK+XA) x (TJ+1) of each field component
  CUtensorMap tile[6];  // box TK x TJ
  CUtensorMap cls;      // box TK x TJ (uint16)
};

// Work split as for the fused marching sweep: CP = false forms sweep the
// box of tiles and chunks whose nodes lie in no CPML layer, with their grid
// offset by `org`; CP = true forms take the full grid and skip that box.
// IN = true (CP = false only) is for a box away from every lattice boundary:
// all nodes of its tiles have every component in range and the full main
// update, so the form carries no range tests.
// `shift` moves the tile grid by whole nodes (k by a multiple of 8 nodes, so
// that every TMA x coordinate -- field values and the uint16 class index --
// stays a multiple of 16 bytes): tile (x, y, z) starts at node
// (shift[0] + 32 x, shift[1] + TJ y, shift[2] + ichunk z).  The time step
// shifts by -size < shift <= 0 so that tile and chunk edges fall near the CPML
// layers' edges (the first tile and chunk then start below node 0: nodes
// k < 0, j < 0 are inactive, planes i < 0 are not swept); the adjoint's
// reverse sweeps shift forward to fit their box to the CPML.
template <typename T>
struct MarchTmaP {
  MarchP<T> p;
  MarchMaps m;
  int* err;
  int org[3];
  int box_lo[3], box_hi[3];
  int shift[3];
  long long wait_budget;  // stage-wait cycles (0: the default)
};

template <typename T, int TJ, int TK>
struct MarchGeom {
  static constexpr int XA = 16 / (int)sizeof(T);
  static constexpr int W = TK + XA;  // halo box width
  static constexpr int R = TJ + 1;   // halo box rows
  __host__ __device__ static constexpr int pad(int b) { return (b + 127) / 128 * 128; }
  static constexpr int HALO_B = R * W * (int)sizeof(T);
  static constexpr int TILE_B = TJ * TK * (int)sizeof(T);
  static constexpr int CLS_B = TJ * TK * 2;
  static constexpr int HALO_OFF = 0;
  static constexpr int TILE_OFF = 3 * pad(HALO_B);
  static constexpr int CLS_OFF = TILE_OFF + 3 * pad(TILE_B);
  static constexpr int STAGE = CLS_OFF + pad(CLS_B);
  static constexpr int TX_FULL = 3 * HALO_B + 3 * TILE_B + CLS_B;
  static constexpr int TX_HALO = 3 * HALO_B;
  static constexpr int NC = 64;  // classes whose (ca, cb) half-rows are cached
  static constexpr int TB = NC * 6 * (int)sizeof(T);
  __host__ __device__ static constexpr int smem(int S) { return S * STAGE + TB + 8 * S; }
};

// Copies the (ca, cb) pairs of one half of the class table (0: E, 1: H) of
// the first NC classes to shared memory.
template <typename T, int NC, int NT>
__device__ __forceinline__ void stage_half_table(T* sT, const T* tab, int n_classes, int half,
                                                 int tid) {
  const int n = min(n_classes, NC) * 6;
  for (int x = tid; x < n; x += NT) {
    const int c = x / 6;
    sT[x] = tab[(size_t)c * 12 + half * 6 + (x - c * 6)];
  }
}

// CPML psi update from an already loaded old value: psi = b psi + a diff,
// stored in place.
template <typename T>
__device__ __forceinline__ T psi_upd(T* ps, T old, T b, T a, T diff) {
  const T v = b * old + a * diff;
  *ps = v;
  return v;
}

// Ring bookkeeping shared by the TMA sweeps: bounded stage waits and the
// drain on failure.  All threads keep identical copies of parity/pending.
// Stage waits give up after `budget` cycles (the engine's "stage_wait_cycles"
// option where the kernel takes it; about 2 s by default); drain() waits for
// the loads still in flight with the default budget whatever `budget` is, so
// that no CTA exits while a bulk copy is still writing its shared memory.
constexpr long long kStageWaitDefault = 4000000000LL;  // about 2 s

struct StageRing {
  uint64_t* bars;
  uint32_t parity = 0;   // bit s: phase to wait for on stage s
  uint32_t pending = 0;  // bit s: a load into stage s is in flight
  long long budget = kStageWaitDefault;
  __device__ __forceinline__ void set_budget(long long b) {
    budget = b > 0 ? b : kStageWaitDefault;
  }

  __device__ __forceinline__ bool try_once(uint32_t a, uint32_t ph) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(ph)
        : "memory");
    return done != 0;
  }
  __device__ __forceinline__ bool test_once(uint32_t a, uint32_t ph) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(ph)
        : "memory");
    return done != 0;
  }
  __device__ bool wait(int s) {
    const uint32_t a = smem_u32(&bars[s]);
    const uint32_t ph = (parity >> s) & 1u;
    if (budget == kStageWaitDefault) {
      // try_wait may suspend the thread until the phase completes (up to a
      // system-dependent limit): no issue slots spent on polling.
      if (!try_once(a, ph)) {
        const long long t0 = clock64();
        while (!try_once(a, ph))
          if (clock64() - t0 > budget) return false;
      }
    } else {
      // A caller-set budget is kept to the cycle: non-blocking probes.
      const long long t0 = clock64();
      while (!test_once(a, ph))
        if (clock64() - t0 >= budget) return false;
    }
    parity ^= 1u << s;
    pending &= ~(1u << s);
    return true;
  }
  __device__ void drain(int S) {
    budget = kStageWaitDefault;
    for (int s = 0; s < S; ++s)
      if ((pending >> s) & 1u) wait(s);
  }
  // For a CTA that sweeps another tile next (the persistent batched kernel):
  // once no load is in flight (none is on the normal path, where every staged
  // plane was waited for) and every thread is done with the stages,
  // invalidate the barriers, so that their words can be initialised again or
  // become stage memory.
  __device__ void release(int S, int tid) {
    drain(S);
    __syncthreads();
    if (tid == 0)
      for (int s = 0; s < S; ++s) mbar_inval(&bars[s]);
  }
};

// ---------------------------------------------------------------------------
// H sweep.  Planes q = 0 .. n_planes of the chunk are staged (plane n_planes
// is i_hi, E only, when i_hi <= nx); plane q lives in stage q % S.
// ---------------------------------------------------------------------------
template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX = 7, bool REUSE = false>
__device__ __forceinline__ void march_h_cta(const MarchTmaP<T>& P, const int gx, const int gy,
                                            const int gz) {
  using G = MarchGeom<T, TJ, TK>;
  extern __shared__ __align__(128) unsigned char smem[];
  const MarchP<T>& p = P.p;
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  if (CP && gx >= P.box_lo[0] && gx < P.box_hi[0] && gy >= P.box_lo[1] && gy < P.box_hi[1] &&
      gz >= P.box_lo[2] && gz < P.box_hi[2])
    return;  // swept by the CPML-free form
  // One thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)P.err & 2))) return;
  const int k0 = gx * TK + P.shift[0], j0 = gy * TJ + P.shift[1];
  const int k = k0 + tk, j = j0 + tj;
  // A negative shift moves the first chunk (and tile) partly below node 0.
  const int i0 = gz * p.ichunk + P.shift[2];
  const int i_lo = max(i0, 0);
  const int i_hi = min(i0 + p.ichunk, L.nx + 1);
  const int n_planes = i_hi - i_lo;
  const int n_staged = n_planes + (i_hi <= L.nx ? 1 : 0);

  StageRing ring;
  ring.set_budget(P.wait_budget);
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);  // [NC][6] (ca, cb) half-rows
  ring.bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::TB);
  auto halo = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::HALO_OFF + c * G::pad(G::HALO_B));
  };
  auto tile = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::TILE_OFF + c * G::pad(G::TILE_B));
  };
  auto ctile = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::CLS_OFF);
  };
  auto issue = [&](int q) {
    const int s = q % S, i = i_lo + q;
    uint64_t* bar = &ring.bars[s];
    unsigned char* base = smem + s * G::STAGE;
    const bool e_only = q == n_planes;
    mbar_expect_tx(bar, e_only ? G::TX_HALO : G::TX_FULL);
    for (int c = 0; c < 3; ++c)
      tma_load_3d(base + G::HALO_OFF + c * G::pad(G::HALO_B), &P.m.halo[c], k0, j0, i, bar);
    if (!e_only) {
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::TILE_OFF + c * G::pad(G::TILE_B), &P.m.tile[3 + c], k0, j0, i, bar);
      tma_load_3d(base + G::CLS_OFF, &P.m.cls, k0, j0, i, bar);
    }
  };

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < S && q < n_staged; ++q) issue(q);
  for (int q = 0; q < S && q < n_staged; ++q) ring.pending |= 1u << (q % S);
  stage_half_table<T, G::NC, TJ * TK>(sT, p.tab, p.n_classes, 1, tid);

  // Per-thread constants (as k_march_h).  The faces k = nz and j = ny are
  // left to k_edge_h (kernels.cuh).
  const bool act = IN || (k >= 0 && j >= 0 && k < L.nz && j < L.ny);
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const bool jv = IN || j < L.ny, kv = IN || k < L.nz;
  const T fhj = (act && jv) ? p.fh[1][j] : T(0);
  const T fhk = (act && kv) ? p.fh[2][k] : T(0);
  int qy = 0, qz = 0;
  const int ly = (CP && (AX & 2) && act) ? layer_of(p.slab[1], j, false, qy) : -1;
  const int lz = (CP && (AX & 4) && act) ? layer_of(p.slab[2], k, false, qz) : -1;
  T ay = 0, by = 0, az = 0, bz = 0;
  T* psy[2] = {nullptr, nullptr};
  T* psz[2] = {nullptr, nullptr};
  long long psy_st = 0, psz_st = 0;
  if (ly >= 0) {
    const SlabAxisD<T>& A = p.slab[1];
    ay = A.a_h[qy][ly];
    by = A.b_h[qy][ly];
    psy_st = (long long)A.n[qy] * KP;
    for (int w = 0; w < 2; ++w) psy[w] = A.psi_h_out[qy][w] + (long long)ly * KP + k;
  }
  if (lz >= 0) {
    const SlabAxisD<T>& A = p.slab[2];
    az = A.a_h[qz][lz];
    bz = A.b_h[qz][lz];
    psz_st = (long long)L.NY * A.n[qz];
    for (int w = 0; w < 2; ++w) psz[w] = A.psi_h_out[qz][w] + (long long)j * A.n[qz] + lz;
  }
  T* Hx = p.f[3] + row;
  T* Hy = p.f[4] + row;
  T* Hz = p.f[5] + row;
  const int hq = tj * G::W + tk;  // (j, k) in a halo box
  const int tq = tj * TK + tk;    // (j, k) in a tile box

  // psi cells of the node on plane i, by slot: 0 Hx-y, 1 Hx-z, 2 Hy-x,
  // 3 Hy-z, 4 Hz-x, 5 Hz-y (CPML form only).  Old values are loaded one plane
  // ahead, so their DRAM latency overlaps the compute of the plane before.
  T pv[6] = {};
  auto load_psi = [&](int i) {
    pv[0] = ly >= 0 ? psy[1][i * psy_st] : T(0);
    pv[5] = ly >= 0 ? psy[0][i * psy_st] : T(0);
    pv[1] = lz >= 0 ? psz[0][i * psz_st] : T(0);
    pv[3] = lz >= 0 ? psz[1][i * psz_st] : T(0);
    int qx = 0;
    const int cx = (AX & 1) ? p.xl[i].x : -1;
    const int lx = (act && cx >= 0) ? (cx >> 1) : -1;
    qx = cx & 1;
    const long long ox = (long long)lx * PS + row;
    pv[2] = lx >= 0 ? p.slab[0].psi_h_out[qx][0][ox] : T(0);
    pv[4] = lx >= 0 ? p.slab[0].psi_h_out[qx][1][ox] : T(0);
  };
  if constexpr (CP) load_psi(i_lo);

  bool ok = true;
  if (n_staged > 0) ok = ring.wait(0);
  for (int q = 0; q < n_planes; ++q) {
    const int i = i_lo + q;
    const bool iv = IN || i < L.nx;
    const int sc = q % S, sn = (q + 1) % S;
    T po[6];
#pragma unroll
    for (int x = 0; x < 6; ++x) po[x] = pv[x];
    if constexpr (CP) {
      if (q + 1 < n_planes) load_psi(i + 1);
    }
    if (ok && iv) ok = ring.wait(sn);  // plane i+1 (exists when i < nx)
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // Every thread is past plane q-1: refill its stage with plane q-1+S.
    if (q >= 1 && q - 1 + S < n_staged) {
      if (tid == 0) {
        fence_proxy_async();
        issue(q - 1 + S);
      }
      ring.pending |= 1u << ((q - 1) % S);
    }
    if (act) {
      const bool main_rng = iv && jv && kv;
      const T fhi = iv ? p.fh[0][i] : T(0);
      const int cl = ctile(sc)[tq];
      const T* r = cl < G::NC ? sT + cl * 6 : p.tab + (size_t)cl * 12 + 6;
      const T* Exs = halo(sc, 0);
      const T* Eys = halo(sc, 1);
      const T* Ezs = halo(sc, 2);
      const T ex = Exs[hq], ex_k = Exs[hq + 1], ex_j = Exs[hq + G::W];
      const T ey = Eys[hq], ey_k = Eys[hq + 1];
      const T ez = Ezs[hq], ez_j = Ezs[hq + G::W];
      const T ey_n = iv ? halo(sn, 1)[hq] : T(0);
      const T ez_n = iv ? halo(sn, 2)[hq] : T(0);
      const T dEy_k = ey_k - ey, dEz_j = ez_j - ez;  // Hx
      const T dEz_i = ez_n - ez, dEx_k = ex_k - ex;  // Hy
      const T dEx_j = ex_j - ex, dEy_i = ey_n - ey;  // Hz
      const long long o = i * PS;
      int qx = 0;
      const int cx = (CP && (AX & 1)) ? p.xl[i].x : -1;
      const int lx = cx >= 0 ? (cx >> 1) : -1;
      qx = cx & 1;
      if (jv && kv) {
        const T ca = r[0], cb = r[1];
        T h = tile(sc, 0)[tq];
        if (main_rng) h = ca * h + cb * (fhk * dEy_k - fhj * dEz_j);
        if (ly >= 0) h -= cb * psi_upd(psy[1] + i * psy_st, po[0], by, ay, dEz_j);
        if (lz >= 0) h += cb * psi_upd(psz[0] + i * psz_st, po[1], bz, az, dEy_k);
        Hx[o] = h;
      }
      if (iv && kv) {
        const T ca = r[2], cb = r[3];
        T h = tile(sc, 1)[tq];
        if (main_rng) h = ca * h + cb * (fhi * dEz_i - fhk * dEx_k);
        if (lx >= 0) {
          const SlabAxisD<T>& A = p.slab[0];
          h += cb * psi_upd(A.psi_h_out[qx][0] + (long long)lx * PS + row, po[2], A.b_h[qx][lx],
                            A.a_h[qx][lx], dEz_i);
        }
        if (lz >= 0) h -= cb * psi_upd(psz[1] + i * psz_st, po[3], bz, az, dEx_k);
        Hy[o] = h;
      }
      if (iv && jv) {
        const T ca = r[4], cb = r[5];
        T h = tile(sc, 2)[tq];
        if (main_rng) h = ca * h + cb * (fhj * dEx_j - fhi * dEy_i);
        if (lx >= 0) {
          const SlabAxisD<T>& A = p.slab[0];
          h -= cb * psi_upd(A.psi_h_out[qx][1] + (long long)lx * PS + row, po[4], A.b_h[qx][lx],
                            A.a_h[qx][lx], dEy_i);
        }
        if (ly >= 0) h += cb * psi_upd(psy[0] + i * psy_st, po[5], by, ay, dEx_j);
        Hz[o] = h;
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicOr(P.err, 2);
    ring.drain(S);
  }
  if constexpr (REUSE) ring.release(S, tid);
}

// ---------------------------------------------------------------------------
// E sweep.  Staged planes q = -1 .. n_planes-1 (plane -1 = i_lo-1, H only,
// when i_lo >= 1); plane q lives in stage (q+1) % S.
// ---------------------------------------------------------------------------
template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX = 7, bool REUSE = false>
__device__ __forceinline__ void march_e_cta(const MarchTmaP<T>& P, const int gx, const int gy,
                                            const int gz) {
  using G = MarchGeom<T, TJ, TK>;
  extern __shared__ __align__(128) unsigned char smem[];
  const MarchP<T>& p = P.p;
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  if (CP && gx >= P.box_lo[0] && gx < P.box_hi[0] && gy >= P.box_lo[1] && gy < P.box_hi[1] &&
      gz >= P.box_lo[2] && gz < P.box_hi[2])
    return;  // swept by the CPML-free form
  // One thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)P.err & 2))) return;
  const int k0 = gx * TK + P.shift[0], j0 = gy * TJ + P.shift[1];
  const int k = k0 + tk, j = j0 + tj;
  // A negative shift moves the first chunk (and tile) partly below node 0.
  const int i0 = gz * p.ichunk + P.shift[2];
  const int i_lo = max(i0, 0);
  const int i_hi = min(i0 + p.ichunk, L.nx + 1);
  const int n_planes = i_hi - i_lo;
  const int q_first = i_lo >= 1 ? -1 : 0;  // first staged plane

  StageRing ring;
  ring.set_budget(P.wait_budget);
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);  // [NC][6] (ca, cb) half-rows
  ring.bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::TB);
  auto slot = [](int q) { return (q + 1) % S; };
  auto halo = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::HALO_OFF + c * G::pad(G::HALO_B));
  };
  auto tile = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::TILE_OFF + c * G::pad(G::TILE_B));
  };
  auto ctile = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::CLS_OFF);
  };
  auto issue = [&](int q) {
    const int s = slot(q), i = i_lo + q;
    uint64_t* bar = &ring.bars[s];
    unsigned char* base = smem + s * G::STAGE;
    const bool h_only = q < 0;
    mbar_expect_tx(bar, h_only ? G::TX_HALO : G::TX_FULL);
    for (int c = 0; c < 3; ++c)
      tma_load_3d(base + G::HALO_OFF + c * G::pad(G::HALO_B), &P.m.halo[3 + c], k0 - G::XA,
                  j0 - 1, i, bar);
    if (!h_only) {
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::TILE_OFF + c * G::pad(G::TILE_B), &P.m.tile[c], k0, j0, i, bar);
      tma_load_3d(base + G::CLS_OFF, &P.m.cls, k0, j0, i, bar);
    }
  };

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const int q_end = n_planes;  // one past the last staged plane
  if (tid == 0)
    for (int q = q_first; q < q_first + S && q < q_end; ++q) issue(q);
  for (int q = q_first; q < q_first + S && q < q_end; ++q) ring.pending |= 1u << slot(q);
  stage_half_table<T, G::NC, TJ * TK>(sT, p.tab, p.n_classes, 0, tid);

  // faces k = nz, j = ny: k_edge_e
  const bool act = IN || (k >= 0 && j >= 0 && k < L.nz && j < L.ny);
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const bool jv = IN || j < L.ny, kv = IN || k < L.nz;
  const bool jm = IN || (j >= 1 && jv), km = IN || (k >= 1 && kv);
  const T fej = act ? p.fe[1][j] : T(0);
  const T fek = act ? p.fe[2][k] : T(0);
  int qy = 0, qz = 0;
  const int ly = (CP && (AX & 2) && act) ? layer_of(p.slab[1], j, true, qy) : -1;
  const int lz = (CP && (AX & 4) && act) ? layer_of(p.slab[2], k, true, qz) : -1;
  T ay = 0, by = 0, az = 0, bz = 0;
  T* psy[2] = {nullptr, nullptr};
  T* psz[2] = {nullptr, nullptr};
  long long psy_st = 0, psz_st = 0;
  if (ly >= 0) {
    const SlabAxisD<T>& A = p.slab[1];
    ay = A.a_e[qy][ly];
    by = A.b_e[qy][ly];
    psy_st = (long long)A.n[qy] * KP;
    for (int w = 0; w < 2; ++w) psy[w] = A.psi_e[qy][w] + (long long)ly * KP + k;
  }
  if (lz >= 0) {
    const SlabAxisD<T>& A = p.slab[2];
    az = A.a_e[qz][lz];
    bz = A.b_e[qz][lz];
    psz_st = (long long)L.NY * A.n[qz];
    for (int w = 0; w < 2; ++w) psz[w] = A.psi_e[qz][w] + (long long)j * A.n[qz] + lz;
  }
  T* Ex = p.f[0] + row;
  T* Ey = p.f[1] + row;
  T* Ez = p.f[2] + row;
  const int hq = (tj + 1) * G::W + tk + G::XA;  // (j, k) in a halo box
  const int tq = tj * TK + tk;

  // psi cells of the node on plane i, by slot: 0 Ex-y, 1 Ex-z, 2 Ey-x,
  // 3 Ey-z, 4 Ez-x, 5 Ez-y (CPML form only), old values loaded a plane ahead.
  T pv[6] = {};
  auto load_psi = [&](int i) {
    pv[0] = ly >= 0 ? psy[1][i * psy_st] : T(0);
    pv[5] = ly >= 0 ? psy[0][i * psy_st] : T(0);
    pv[1] = lz >= 0 ? psz[0][i * psz_st] : T(0);
    pv[3] = lz >= 0 ? psz[1][i * psz_st] : T(0);
    int qx = 0;
    const int cx = (AX & 1) ? p.xl[i].y : -1;
    const int lx = (act && cx >= 0) ? (cx >> 1) : -1;
    qx = cx & 1;
    const long long ox = (long long)lx * PS + row;
    pv[2] = lx >= 0 ? p.slab[0].psi_e[qx][0][ox] : T(0);
    pv[4] = lx >= 0 ? p.slab[0].psi_e[qx][1][ox] : T(0);
  };
  if constexpr (CP) {
    if (n_planes > 0) load_psi(i_lo);
  }

  bool ok = true;
  if (q_first < 0) ok = ring.wait(slot(-1));
  for (int q = 0; q < n_planes; ++q) {
    const int i = i_lo + q;
    const int sc = slot(q), sp = slot(q - 1);
    T po[6];
#pragma unroll
    for (int x = 0; x < 6; ++x) po[x] = pv[x];
    if constexpr (CP) {
      if (q + 1 < n_planes) load_psi(i + 1);
    }
    if (ok) ok = ring.wait(sc);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // Every thread is past plane q-1, so plane q-2 is free: refill its stage.
    if (q - 2 >= q_first && q - 2 + S < q_end) {
      if (tid == 0) {
        fence_proxy_async();
        issue(q - 2 + S);
      }
      ring.pending |= 1u << slot(q - 2);
    }
    if (act) {
      const bool iv = IN || i < L.nx, i1 = IN || i >= 1;
      const bool im = i1 && iv;
      const T fei = p.fe[0][i];
      const int cl = ctile(sc)[tq];
      const T* r = cl < G::NC ? sT + cl * 6 : p.tab + (size_t)cl * 12;
      const T* Hxs = halo(sc, 0);
      const T* Hys = halo(sc, 1);
      const T* Hzs = halo(sc, 2);
      const T hx = Hxs[hq], hy = Hys[hq], hz = Hzs[hq];
      const T hx_k = Hxs[hq - 1], hx_j = Hxs[hq - G::W];
      const T hy_k = Hys[hq - 1];
      const T hz_j = Hzs[hq - G::W];
      const T hy_p = i1 ? halo(sp, 1)[hq] : T(0);
      const T hz_p = i1 ? halo(sp, 2)[hq] : T(0);
      const T dHz_j = hz - hz_j, dHy_k = hy - hy_k;  // Ex
      const T dHx_k = hx - hx_k, dHz_i = hz - hz_p;  // Ey
      const T dHy_i = hy - hy_p, dHx_j = hx - hx_j;  // Ez
      const long long o = i * PS;
      int qx = 0;
      const int cx = (CP && (AX & 1)) ? p.xl[i].y : -1;
      const int lx = cx >= 0 ? (cx >> 1) : -1;
      qx = cx & 1;
      if (iv) {
        const T ca = r[0], cb = r[1];
        T e = tile(sc, 0)[tq];
        if (jm && km) e = ca * e + cb * (fej * dHz_j - fek * dHy_k);
        if (ly >= 0) e += cb * psi_upd(psy[1] + i * psy_st, po[0], by, ay, dHz_j);
        if (lz >= 0) e -= cb * psi_upd(psz[0] + i * psz_st, po[1], bz, az, dHy_k);
        Ex[o] = e;
      }
      if (jv) {
        const T ca = r[2], cb = r[3];
        T e = tile(sc, 1)[tq];
        if (im && km) e = ca * e + cb * (fek * dHx_k - fei * dHz_i);
        if (lx >= 0) {
          const SlabAxisD<T>& A = p.slab[0];
          e -= cb * psi_upd(A.psi_e[qx][0] + (long long)lx * PS + row, po[2], A.b_e[qx][lx],
                            A.a_e[qx][lx], dHz_i);
        }
        if (lz >= 0) e += cb * psi_upd(psz[1] + i * psz_st, po[3], bz, az, dHx_k);
        Ey[o] = e;
      }
      if (kv) {
        const T ca = r[4], cb = r[5];
        T e = tile(sc, 2)[tq];
        if (im && jm) e = ca * e + cb * (fei * dHy_i - fej * dHx_j);
        if (lx >= 0) {
          const SlabAxisD<T>& A = p.slab[0];
          e += cb * psi_upd(A.psi_e[qx][1] + (long long)lx * PS + row, po[4], A.b_e[qx][lx],
                            A.a_e[qx][lx], dHy_i);
        }
        if (ly >= 0) e -= cb * psi_upd(psy[0] + i * psy_st, po[5], by, ay, dHx_j);
        Ez[o] = e;
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicOr(P.err, 2);
    ring.drain(S);
  }
  if constexpr (REUSE) ring.release(S, tid);
}

// One lattice: CTA (x, y, z) sweeps tile (x, y) and chunk z, offset by org.
template <typename T, int TJ, int TK, int S, bool CP, bool IN>
__global__ void __launch_bounds__(TJ* TK) k_march_h_tma(const __grid_constant__ MarchTmaP<T> P) {
  march_h_cta<T, TJ, TK, S, CP, IN>(P, blockIdx.x + P.org[0], blockIdx.y + P.org[1],
                                    blockIdx.z + P.org[2]);
}

template <typename T, int TJ, int TK, int S, bool CP, bool IN>
__global__ void __launch_bounds__(TJ* TK) k_march_e_tma(const __grid_constant__ MarchTmaP<T> P) {
  march_e_cta<T, TJ, TK, S, CP, IN>(P, blockIdx.x + P.org[0], blockIdx.y + P.org[1],
                                    blockIdx.z + P.org[2]);
}

// One lattice, a tile list: CTA b sweeps tile tiles[b] = (-, k tile, j tile,
// chunk).  AX names the CPML axes (bits x, y, z) whose layers the listed
// tiles can meet, so that the other axes' layer code is left out.
template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX>
__global__ void __launch_bounds__(TJ* TK)
    k_march_h_tma_list(const __grid_constant__ MarchTmaP<T> P, const int4* __restrict__ tiles) {
  const int4 w = tiles[blockIdx.x];
  march_h_cta<T, TJ, TK, S, CP, IN, AX>(P, w.y, w.z, w.w);
}

template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX>
__global__ void __launch_bounds__(TJ* TK)
    k_march_e_tma_list(const __grid_constant__ MarchTmaP<T> P, const int4* __restrict__ tiles) {
  const int4 w = tiles[blockIdx.x];
  march_e_cta<T, TJ, TK, S, CP, IN, AX>(P, w.y, w.z, w.w);
}

// Many lattices in one launch: CTA b sweeps the tile list entry
// tiles[b] = (lattice, k tile, j tile, chunk) with the parameters
// scenes[lattice] (device memory, tensor maps included).  The host builds
// the list so that every entry is a tile of the form launched (CPML-free
// interior, CPML-free, or CPML), largest lattices first.
// The thread that issues the TMA loads first acquires the lattice's tensor
// maps, which the host copied into device memory.
__device__ __forceinline__ void acquire_march_maps(const MarchMaps& m) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int c = 0; c < 6; ++c) {
      tensormap_acquire(&m.halo[c]);
      tensormap_acquire(&m.tile[c]);
    }
    tensormap_acquire(&m.cls);
  }
}

template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX = 7>
__global__ void __launch_bounds__(TJ* TK)
    k_march_h_tma_batch(const MarchTmaP<T>* __restrict__ scenes, const int4* __restrict__ tiles) {
  const int4 w = tiles[blockIdx.x];
  acquire_march_maps(scenes[w.x].m);
  march_h_cta<T, TJ, TK, S, CP, IN, AX>(scenes[w.x], w.y, w.z, w.w);
}

template <typename T, int TJ, int TK, int S, bool CP, bool IN, int AX = 7>
__global__ void __launch_bounds__(TJ* TK)
    k_march_e_tma_batch(const MarchTmaP<T>* __restrict__ scenes, const int4* __restrict__ tiles) {
  const int4 w = tiles[blockIdx.x];
  acquire_march_maps(scenes[w.x].m);
  march_e_cta<T, TJ, TK, S, CP, IN, AX>(scenes[w.x], w.y, w.z, w.w);
}

}  // namespace xfd
