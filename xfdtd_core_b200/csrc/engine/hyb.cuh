// Fused H-then-E sweep of the CPML-free interior box (sweep 7).
//
// One kernel updates H and then E of every node of the interior box in one
// pass over the fields: fields ping-pong between two buffers, so the kernel
// reads E^n, H^{n-1/2} and the class index from `in` (by TMA) and writes
// H^{n+1/2}, E^{n+1} to `out`, and no CTA ever reads a value a neighbouring CTA
// has already advanced.  DRAM traffic per node is the compulsory one: six field
// values read, six written, one uint16 class index read (50 B in FP32).
//
// A CTA of 32 x TJ compute threads (plus a helper warp) owns a 32-node (k) x
// TJ-row (j) tile and marches
// along i over a chunk of planes; tiles are 128-byte aligned along k (unless
// the march_shift option moves them by a multiple of 8 nodes).  Per
// plane i it stages, by TMA into a ring of S shared-memory stages:
//   E of plane i over rows j0-1 .. j0+TJ and nodes k0-XA .. k0+31+XA,
//   H of plane i over rows j0-1 .. j0+TJ-1 and nodes k0-XA .. k0+31,
//   the class index over rows j0-1 .. j0+TJ-1 and nodes k0-8 .. k0+31
// (XA = 16 bytes of the field type, so that every TMA x coordinate is a
// multiple of 16 bytes).  E of plane i+1 is the next stage.  Each thread then
// computes the three H components of its node (the reference's hNext,
// src/include/updator/update_scheme.h:57-62, over BasicUpdator::updateH's
// ranges, src/updator/basic_updator.cpp:23-36); the TFSF H-face corrections
// are already in the H it reads (k_tfsf_pre, kernels.cuh).  A helper warp
// issues the loads and recomputes H_x, H_z of row j0-1 and H_x, H_y of column
// k0-1 (nodes of the neighbouring tiles that the E update reads).  After one CTA barrier each thread computes the three E components
// (eNext, update_scheme.h:26-31, over BasicUpdator3D::updateE's ranges,
// src/updator/basic_updator_3d.cpp:38-69): the k-1 neighbours of H come by
// warp shuffle, the j-1 neighbours from shared memory, the i-1 neighbours are
// the thread's own H of the previous plane, kept in registers.  A chunk starts
// by recomputing H_y, H_z of its plane i_lo-1.
//
// The box is chosen by the host so that its nodes, the recomputed row j0-1,
// column k0-1 and plane i_lo-1, and the neighbours read at j0+TJ, k0+32, i_hi
// all lie away from the lattice boundaries and outside every CPML layer:
// every node takes the full main update and the kernel has no range tests.
// The CPML tiles around the box are swept by the split marching forms in
// ping-pong mode (march_tma.cuh), the lattice faces k = nz, j = ny by
// k_edge_pp (kernels.cuh).
//
// Stage waits are bounded (a cycle budget, the engine's "stage_wait_cycles"
// option); on expiry the CTA sets bit 2 of the engine's error word, drains
// its loads in flight (with the default budget) and returns.
#pragma once

#include "march_tma.cuh"

namespace xfd {

struct HybMaps {
  CUtensorMap e[3];  // E halo boxes: (32 + 2 XA) x (TJ + 2)
  CUtensorMap h[3];  // H halo boxes: (32 + XA) x (TJ + 1)
  CUtensorMap cls;   // class boxes: (32 + 8) x (TJ + 1)
};

template <typename T>
struct HybP {
  Lat L;
  T* out[6];
  const T* tab;  // n_classes x 12: (ca, cb) of Ex Ey Ez Hx Hy Hz
  int n_classes;
  const T* fe[3];
  const T* fh[3];
  int* err;
  long long wait_budget;  // stage-wait cycles (0: the default)
  HybMaps m;
  int org[3];   // first (k tile, j tile, chunk) of the box
  int shift[3];  // node of tile (0, 0, 0): k0 = 32 x + shift[0], j0, i_lo likewise
  int ichunk;
  // Tile list: CTA b sweeps tile (tiles[b].y, tiles[b].z, tiles[b].w) (k tile,
  // j tile, chunk); null: CTA (x, y, z) sweeps tile org + (x, y, z).
  const int4* tiles;
};

template <typename T, int TJ>
struct HybGeom {
  static constexpr int TK = 32;
  static constexpr int XA = 16 / (int)sizeof(T);
  static constexpr int WE = TK + 2 * XA, RE = TJ + 2;  // E boxes
  static constexpr int WH = TK + XA, RH = TJ + 1;      // H boxes
  static constexpr int WC = TK + 8, RC = TJ + 1;       // class boxes (uint16)
  __host__ __device__ static constexpr int pad(int b) { return (b + 127) / 128 * 128; }
  static constexpr int E_B = RE * WE * (int)sizeof(T);
  static constexpr int H_B = RH * WH * (int)sizeof(T);
  static constexpr int C_B = RC * WC * 2;
  static constexpr int E_OFF = 0;
  static constexpr int H_OFF = 3 * pad(E_B);
  static constexpr int C_OFF = H_OFF + 3 * pad(H_B);
  static constexpr int STAGE = C_OFF + pad(C_B);
  static constexpr int TX_FULL = 3 * E_B + 3 * H_B + C_B;
  static constexpr int TX_E = 3 * E_B;
  static constexpr int NC = 64;                          // classes cached in shared memory
  static constexpr int TB = NC * 12 * (int)sizeof(T);    // their (ca, cb) rows
  // New H for the E update: H_x, H_z of rows j0-1 .. j0+TJ-1 (32 nodes each)
  // and H_x, H_y of column k0-1 (TJ nodes), two buffers (planes alternate).
  static constexpr int HN = 2 * 2 * (RH * TK + TJ) * (int)sizeof(T);
  __host__ __device__ static constexpr int smem(int S) { return S * STAGE + TB + HN + 8 * S; }
};

// The 12 (ca, cb) values of a class as vector loads: FP32 3 x float4, FP64
// 6 x double2 (rows are 48 / 96 bytes, so 16-byte aligned), from shared memory
// for the first NC classes, else from the table in global memory.
template <typename T>
struct ClassRow {
  T v[12];
  __device__ __forceinline__ void load(const T* r) {
    if constexpr (sizeof(T) == 4) {
      const float4* q = reinterpret_cast<const float4*>(r);
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const float4 a = q[u];
        v[4 * u] = a.x;
        v[4 * u + 1] = a.y;
        v[4 * u + 2] = a.z;
        v[4 * u + 3] = a.w;
      }
    } else {
      const double2* q = reinterpret_cast<const double2*>(r);
#pragma unroll
      for (int u = 0; u < 6; ++u) {
        const double2 a = q[u];
        v[2 * u] = a.x;
        v[2 * u + 1] = a.y;
      }
    }
  }
};

// CTA: TJ compute warps (warp w owns row j0 + w of the tile, lane = k - k0)
// and one helper warp (threadIdx.y == TJ) that issues the TMA loads and
// recomputes the H values of the neighbouring tiles that the E update reads:
// H_x, H_z of row j0-1 (lane = k - k0) and H_x, H_y of column k0-1 (lanes
// 0 .. TJ-1 = j - j0).  Compute warps carry no halo work, so no warp diverges.
template <typename T, int TJ, int S>
__global__ void __launch_bounds__(32 * (TJ + 1), sizeof(T) == 8 ? 3 : 4)
    k_hyb(const __grid_constant__ HybP<T> p) {
  using G = HybGeom<T, TJ>;
  constexpr int TK = G::TK;
  extern __shared__ __align__(128) unsigned char smem[];
  const Lat L = p.L;
  const int tk = threadIdx.x, wj = threadIdx.y, tid = wj * TK + tk;
  const bool helper = wj == TJ;
  if (__syncthreads_or(tid == 0 && (*(volatile int*)p.err & 2))) return;
  int gx, gy, gz;
  if (p.tiles) {
    const int4 w = p.tiles[blockIdx.x];
    gx = w.y;
    gy = w.z;
    gz = w.w;
  } else {
    gx = blockIdx.x + p.org[0];
    gy = blockIdx.y + p.org[1];
    gz = blockIdx.z + p.org[2];
  }
  const int k0 = gx * TK + p.shift[0], j0 = gy * TJ + p.shift[1];
  const int i_lo = gz * p.ichunk + p.shift[2];
  const int i_hi = min(i_lo + p.ichunk, L.nx);
  const int n = i_hi - i_lo;  // planes updated; staged: i_lo-1 .. i_hi (n + 2)

  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);          // [NC][12]
  T* sN = reinterpret_cast<T*>(smem + S * G::STAGE + G::TB);  // new H
  StageRing ring;
  ring.set_budget(p.wait_budget);
  ring.bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::TB + G::HN);
  auto sE = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::E_OFF + c * G::pad(G::E_B));
  };
  auto sH = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::H_OFF + c * G::pad(G::H_B));
  };
  auto sC = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::C_OFF);
  };
  // New-H buffers: rows [b][0 = x, 1 = z][RH][32], columns [b][0 = x, 1 = y][TJ].
  auto nrow = [&](int b, int w) { return sN + (b * 2 + w) * (G::RH * TK); };
  auto ncol = [&](int b, int w) { return sN + 4 * (G::RH * TK) + (b * 2 + w) * TJ; };
  const int n_staged = n + 2;
  const bool issuer = helper && tk == 0;
  auto issue = [&](int u) {  // plane i_lo - 1 + u into stage u % S
    const int s = u % S, i = i_lo - 1 + u;
    uint64_t* bar = &ring.bars[s];
    unsigned char* base = smem + s * G::STAGE;
    const bool e_only = u == n + 1;
    mbar_expect_tx(bar, e_only ? G::TX_E : G::TX_FULL);
    for (int c = 0; c < 3; ++c)
      tma_load_3d(base + G::E_OFF + c * G::pad(G::E_B), &p.m.e[c], k0 - G::XA, j0 - 1, i, bar);
    if (!e_only) {
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::H_OFF + c * G::pad(G::H_B), &p.m.h[c], k0 - G::XA, j0 - 1, i, bar);
      tma_load_3d(base + G::C_OFF, &p.m.cls, k0 - 8, j0 - 1, i, bar);
    }
  };
  if (issuer) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (issuer)
    for (int u = 0; u < S && u < n_staged; ++u) issue(u);
  for (int u = 0; u < S && u < n_staged; ++u) ring.pending |= 1u << (u % S);
  for (int x = tid; x < min(p.n_classes, G::NC) * 12; x += 32 * (TJ + 1)) sT[x] = p.tab[x];

  const long long PS = (long long)L.NY * L.KP;
  // Node of this thread: compute warps own (j0 + wj, k0 + tk); the helper
  // warp's lane tk handles row-halo node (j0-1, k0+tk) and, for tk < TJ,
  // column-halo node (j0+tk, k0-1).
  const int j = helper ? j0 - 1 : j0 + wj, k = k0 + tk;
  const long long row = (long long)j * L.KP + k;
  const T fhj = p.fh[1][j], fhk = p.fh[2][k];
  const T fej = helper ? T(0) : p.fe[1][j], fek = p.fe[2][k];
  const bool col = helper && tk < TJ;
  const int jc = j0 + tk;  // column-halo row (helper lanes tk < TJ)
  const T fhj_c = col ? p.fh[1][jc] : T(0);
  const T fhk_c = p.fh[2][k0 - 1];
  // Offsets in the staged boxes: own / row-halo node, column-halo node.
  const int wr = helper ? 0 : wj + 1;  // box row of j
  const int eq = wr * G::WE + tk + G::XA;
  const int hq = wr * G::WH + tk + G::XA;
  const int cq = wr * G::WC + tk + 8;
  const int eq_c = (tk + 1) * G::WE + G::XA - 1, hq_c = (tk + 1) * G::WH + G::XA - 1,
            cq_c = (tk + 1) * G::WC + 7;
  T* const o_ex = p.out[0] + row;
  T* const o_ey = p.out[1] + row;
  T* const o_ez = p.out[2] + row;
  T* const o_hx = p.out[3] + row;
  T* const o_hy = p.out[4] + row;
  T* const o_hz = p.out[5] + row;
  __syncthreads();  // class rows staged

  auto row_of = [&](int cl) { return cl < G::NC ? sT + cl * 12 : p.tab + (size_t)cl * 12; };

  bool ok = true;
  // ---- plane i_lo - 1: H_y, H_z of the compute warps' nodes (the E update's
  // i-1 neighbours)
  T hy_prev = T(0), hz_prev = T(0);
  if (n > 0) {
    ok = ring.wait(0);
    if (ok) ok = ring.wait(1 % S);
    if (ok && !helper) {
      const int i = i_lo - 1;
      const T fhi = p.fh[0][i];
      const T* E0 = sE(0, 0);
      const T* E1 = sE(0, 1);
      const T* E2 = sE(0, 2);
      ClassRow<T> c;
      c.load(row_of(sC(0)[cq]));
      const T ex = E0[eq], ey = E1[eq], ez = E2[eq];
      T hy = c.v[8] * sH(0, 1)[hq] +
             c.v[9] * (fhi * (sE(1 % S, 2)[eq] - ez) - fhk * (E0[eq + 1] - ex));
      T hz = c.v[10] * sH(0, 2)[hq] +
             c.v[11] * (fhj * (E0[eq + G::WE] - ex) - fhi * (sE(1 % S, 1)[eq] - ey));
      hy_prev = hy;
      hz_prev = hz;
    }
  }

  for (int q = 0; q < n; ++q) {
    const int i = i_lo + q;
    const int sc = (q + 1) % S, sn = (q + 2) % S;
    if (ok) ok = ring.wait(sn);  // E of plane i+1
    const int b = q & 1;
    T hx = T(0), hy = T(0), hz = T(0), ex = T(0), ey = T(0), ez = T(0);
    ClassRow<T> c;
    if (ok) {
      const T fhi = p.fh[0][i];
      const T* E0 = sE(sc, 0);
      const T* E1 = sE(sc, 1);
      const T* E2 = sE(sc, 2);
      const T* N1 = sE(sn, 1);
      const T* N2 = sE(sn, 2);
      // H_x, H_z of this lane's node (own node, or row-halo node for the helper)
      c.load(row_of(sC(sc)[cq]));
      ex = E0[eq];
      ey = E1[eq];
      ez = E2[eq];
      hx = c.v[6] * sH(sc, 0)[hq] +
           c.v[7] * (fhk * (E1[eq + 1] - ey) - fhj * (E2[eq + G::WE] - ez));
      hz = c.v[10] * sH(sc, 2)[hq] +
           c.v[11] * (fhj * (E0[eq + G::WE] - ex) - fhi * (N1[eq] - ey));
      if (!helper)
        hy = c.v[8] * sH(sc, 1)[hq] +
             c.v[9] * (fhi * (N2[eq] - ez) - fhk * (E0[eq + 1] - ex));
      nrow(b, 0)[wr * TK + tk] = hx;
      nrow(b, 1)[wr * TK + tk] = hz;
      if (!helper) {
        const long long o = i * PS;
        o_hx[o] = hx;
        o_hy[o] = hy;
        o_hz[o] = hz;
      } else if (col) {  // H_x, H_y at (i, j0 + tk, k0-1)
        ClassRow<T> cc;
        cc.load(row_of(sC(sc)[cq_c]));
        const T ex_c = E0[eq_c], ey_c = E1[eq_c], ez_c = E2[eq_c];
        const T hxc = cc.v[6] * sH(sc, 0)[hq_c] +
                cc.v[7] * (fhk_c * (E1[eq_c + 1] - ey_c) - fhj_c * (E2[eq_c + G::WE] - ez_c));
        const T hyc = cc.v[8] * sH(sc, 1)[hq_c] +
                cc.v[9] * (fhi * (N2[eq_c] - ez_c) - fhk_c * (E0[eq_c + 1] - ex_c));
        ncol(b, 0)[tk] = hxc;
        ncol(b, 1)[tk] = hyc;
      }
    }
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // The stage of plane i (u = q + 1) is read only before this barrier (the
    // E update below works from registers and the new-H buffers), so it is
    // free now -- and at q = 0 so is that of plane i_lo - 1 (u = 0): refill
    // them with the planes S further on.
    for (int u = q == 0 ? 0 : q + 1; u <= q + 1; ++u) {
      if (u + S < n_staged) {
        if (issuer) {
          fence_proxy_async();
          issue(u + S);
        }
        ring.pending |= 1u << (u % S);
      }
    }
    // ---------------------------------------------------------- E(i)
    if (!helper) {
      const T fei = p.fe[0][i];
      const T hy_s = __shfl_up_sync(0xffffffffu, hy, 1);
      const T hx_s = __shfl_up_sync(0xffffffffu, hx, 1);
      const T hym = tk > 0 ? hy_s : ncol(b, 1)[wj];
      const T hxm_k = tk > 0 ? hx_s : ncol(b, 0)[wj];
      const T hzm_j = nrow(b, 1)[wj * TK + tk];
      const T hxm_j = nrow(b, 0)[wj * TK + tk];
      const long long o = i * PS;
      o_ex[o] = c.v[0] * ex + c.v[1] * (fej * (hz - hzm_j) - fek * (hy - hym));
      o_ey[o] = c.v[2] * ey + c.v[3] * (fek * (hx - hxm_k) - fei * (hz - hz_prev));
      o_ez[o] = c.v[4] * ez + c.v[5] * (fei * (hy - hy_prev) - fej * (hx - hxm_j));
      hy_prev = hy;
      hz_prev = hz;
    }
  }
  if (!ok && tid == 0) atomicOr(p.err, 2);
  // No CTA exits with a load in flight: wait (bounded) for every stage still
  // pending (none on the normal path, where each staged plane was waited for).
  ring.drain(S);
}

}  // namespace xfd
