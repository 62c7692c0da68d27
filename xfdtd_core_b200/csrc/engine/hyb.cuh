// Fused H-then-E sweep of the CPML-free interior box (sweep 7).
//
// One kernel updates H and then E of every node of the interior box in one
// pass over the fields: fields ping-pong between two buffers, so the kernel
// reads E^n, H^{n-1/2} and the class index from `in` (by TMA) and writes
// H^{n+1/2}, E^{n+1} to `out`, and no CTA ever reads a value a neighbouring CTA
// has already advanced.  DRAM traffic per node is the compulsory one: six field
// values read, six written, one uint16 class index read (50 B in FP32).
//
// A CTA of 32 x TJ threads owns a 32-node (k) x TJ-row (j) tile and marches
// along i over a chunk of planes; tiles are 128-byte aligned along k.  Per
// plane i it stages, by TMA into a ring of S shared-memory stages:
//   E of plane i over rows j0-1 .. j0+TJ and nodes k0-XA .. k0+31+XA,
//   H of plane i over rows j0-1 .. j0+TJ-1 and nodes k0-XA .. k0+31,
//   the class index over rows j0-1 .. j0+TJ-1 and nodes k0-8 .. k0+31
// (XA = 16 bytes of the field type, so that every TMA x coordinate is a
// multiple of 16 bytes).  E of plane i+1 is the next stage.  Each thread then
// computes the three H components of its node (the reference's hNext,
// src/include/updator/update_scheme.h:57-62, over BasicUpdator::updateH's
// ranges, src/updator/basic_updator.cpp:23-36), with the TFSF H-face
// corrections of TFSF3DCorrector::correctH (src/waveform_source/tfsf_corrector.cpp:205-232)
// applied inline; warp 0 also recomputes H_x, H_z of row j0-1 and lane 0 of
// each warp H_x, H_y of column k0-1 (nodes of the neighbouring tiles that the
// E update reads).  After one CTA barrier it computes the three E components
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
// Stage waits are bounded (a cycle budget); on expiry the CTA sets bit 2 of
// the engine's error word, drains its loads in flight and returns.
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
  TfsfD tf;
  TfsfHD tfh;
  const long long* step;
  int* err;
  HybMaps m;
  int org[3];   // first (k tile, j tile, chunk) of the box
  int ichunk;
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

// Bit 4 c + s: TFSF H pass s of component c covers rows j and nodes k (its
// i range is checked per plane).
template <typename T>
__device__ __forceinline__ uint32_t hyb_tfsf_mask(const HybP<T>& p, int j, int k) {
  uint32_t m = 0;
  for (int c = 0; c < 3; ++c)
    for (int s = 0; s < p.tfh.n[c]; ++s) {
      const TfsfHPass& Q = p.tfh.pass[c][s];
      if (j >= Q.lo[1] && j < Q.hi[1] && k >= Q.lo[2] && k < Q.hi[2]) m |= 1u << (4 * c + s);
    }
  return m;
}

// TFSF H-face corrections of component c at node (i, j, k), in the
// reference's pass order (correctTFSF, src/include/waveform_source/tfsf_corrector.h:89-229),
// over the passes of `mask`.
template <typename T>
__device__ __forceinline__ T hyb_tfsf_h(const HybP<T>& p, uint32_t mask, int c, int i, int j,
                                        int k, T h, long long t) {
  uint32_t m = (mask >> (4 * c)) & 15u;
  while (m) {
    const int s = __ffs(m) - 1;
    m &= m - 1;
    const TfsfHPass& Q = p.tfh.pass[c][s];
    if (i < Q.lo[0] || i >= Q.hi[0]) continue;
    const int xi[3] = {i + (Q.neg && Q.m == 0 ? 1 : 0), j + (Q.neg && Q.m == 1 ? 1 : 0),
                       k + (Q.neg && Q.m == 2 ? 1 : 0)};
    int e_flag = 0;
    const double v = tfsf_incident(p.tf, true, Q.dual, t, xi, &e_flag);
    if (e_flag) atomicOr(p.err, 1);
    h = (T)((double)h + v * Q.coeff);
  }
  return h;
}

template <typename T, int TJ, int S, bool TF>
__global__ void __launch_bounds__(32 * TJ) k_hyb(const __grid_constant__ HybP<T> p) {
  using G = HybGeom<T, TJ>;
  constexpr int TK = G::TK;
  extern __shared__ __align__(128) unsigned char smem[];
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  if (__syncthreads_or(tid == 0 && (*(volatile int*)p.err & 2))) return;
  const int k0 = (blockIdx.x + p.org[0]) * TK, j0 = (blockIdx.y + p.org[1]) * TJ;
  const int i_lo = (blockIdx.z + p.org[2]) * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx);
  const int n = i_hi - i_lo;  // planes updated; staged: i_lo-1 .. i_hi (n + 2)
  const int k = k0 + tk, j = j0 + tj;

  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);                  // [NC][12]
  T* sN = reinterpret_cast<T*>(smem + S * G::STAGE + G::TB);          // new H
  StageRing ring;
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
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ring.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int u = 0; u < S && u < n_staged; ++u) issue(u);
  for (int u = 0; u < S && u < n_staged; ++u) ring.pending |= 1u << (u % S);
  for (int x = tid; x < min(p.n_classes, G::NC) * 12; x += 32 * TJ) sT[x] = p.tab[x];

  const long long t = TF ? *p.step : 0;
  const long long PS = (long long)L.NY * L.KP;
  const long long row = (long long)j * L.KP + k;
  const T fhj = p.fh[1][j], fhk = p.fh[2][k];
  const T fej = p.fe[1][j], fek = p.fe[2][k];
  // Halo duties: warp 0 recomputes row j0-1 (node k), lane 0 of warp tj
  // column k0-1 (node j).
  const bool row_halo = tj == 0;
  const bool col_halo = tk == 0;
  const T fhj_r = row_halo ? p.fh[1][j0 - 1] : T(0);
  const T fhk_c = col_halo ? p.fh[2][k0 - 1] : T(0);
  // Offsets of this thread's node in the staged boxes.
  const int eq = (tj + 1) * G::WE + tk + G::XA;
  const int hq = (tj + 1) * G::WH + tk + G::XA;
  const int cq = (tj + 1) * G::WC + tk + 8;
  // Row halo node (j0-1, k): row 0 of the boxes; column halo (j, k0-1).
  const int eq_r = tk + G::XA, hq_r = tk + G::XA, cq_r = tk + 8;
  const int eq_c = (tj + 1) * G::WE + G::XA - 1, hq_c = (tj + 1) * G::WH + G::XA - 1,
            cq_c = (tj + 1) * G::WC + 7;
  // TFSF H passes that can meet this thread's node, row halo and column halo.
  const uint32_t tm = TF ? hyb_tfsf_mask(p, j, k) : 0u;
  const uint32_t tm_r = TF && row_halo ? hyb_tfsf_mask(p, j0 - 1, k) : 0u;
  const uint32_t tm_c = TF && col_halo ? hyb_tfsf_mask(p, j, k0 - 1) : 0u;
  __syncthreads();  // class rows staged

  auto coef = [&](int cl, int x) -> T {
    return cl < G::NC ? sT[cl * 12 + x] : p.tab[(size_t)cl * 12 + x];
  };

  bool ok = true;
  // ---- plane i_lo - 1: H_y, H_z of this node (the E update's i-1 neighbours)
  T hy_prev = T(0), hz_prev = T(0);
  if (n > 0) {
    ok = ring.wait(0);
    if (ok) ok = ring.wait(1 % S);
    if (ok) {
      const int i = i_lo - 1;
      const T fhi = p.fh[0][i];
      const T* E0 = sE(0, 0);
      const T* E1 = sE(0, 1);
      const T* E2 = sE(0, 2);
      const int cl = sC(0)[cq];
      const T ex = E0[eq], ey = E1[eq], ez = E2[eq];
      const T ex_k = E0[eq + 1], ex_j = E0[eq + G::WE];
      const T ez_n = sE(1 % S, 2)[eq], ey_n = sE(1 % S, 1)[eq];
      T hy = coef(cl, 8) * sH(0, 1)[hq] + coef(cl, 9) * (fhi * (ez_n - ez) - fhk * (ex_k - ex));
      T hz = coef(cl, 10) * sH(0, 2)[hq] + coef(cl, 11) * (fhj * (ex_j - ex) - fhi * (ey_n - ey));
      if (TF) {
        hy = hyb_tfsf_h(p, tm, 1, i, j, k, hy, t);
        hz = hyb_tfsf_h(p, tm, 2, i, j, k, hz, t);
      }
      hy_prev = hy;
      hz_prev = hz;
    }
  }

  for (int q = 0; q < n; ++q) {
    const int i = i_lo + q;
    const int sc = (q + 1) % S, sn = (q + 2) % S;
    if (ok) ok = ring.wait(sn);  // E of plane i+1
    // ---------------------------------------------------------- H(i)
    T hx = T(0), hy = T(0), hz = T(0);
    T ex = T(0), ey = T(0), ez = T(0);
    int cl = 0;
    const int b = q & 1;
    if (ok) {
      const T fhi = p.fh[0][i];
      const T* E0 = sE(sc, 0);
      const T* E1 = sE(sc, 1);
      const T* E2 = sE(sc, 2);
      const T* N1 = sE(sn, 1);
      const T* N2 = sE(sn, 2);
      cl = sC(sc)[cq];
      ex = E0[eq];
      ey = E1[eq];
      ez = E2[eq];
      const T dEy_k = E1[eq + 1] - ey, dEz_j = E2[eq + G::WE] - ez;
      const T dEz_i = N2[eq] - ez, dEx_k = E0[eq + 1] - ex;
      const T dEx_j = E0[eq + G::WE] - ex, dEy_i = N1[eq] - ey;
      hx = coef(cl, 6) * sH(sc, 0)[hq] + coef(cl, 7) * (fhk * dEy_k - fhj * dEz_j);
      hy = coef(cl, 8) * sH(sc, 1)[hq] + coef(cl, 9) * (fhi * dEz_i - fhk * dEx_k);
      hz = coef(cl, 10) * sH(sc, 2)[hq] + coef(cl, 11) * (fhj * dEx_j - fhi * dEy_i);
      if (TF && tm) {
        hx = hyb_tfsf_h(p, tm, 0, i, j, k, hx, t);
        hy = hyb_tfsf_h(p, tm, 1, i, j, k, hy, t);
        hz = hyb_tfsf_h(p, tm, 2, i, j, k, hz, t);
      }
      const long long o = i * PS + row;
      p.out[3][o] = hx;
      p.out[4][o] = hy;
      p.out[5][o] = hz;
      nrow(b, 0)[(tj + 1) * TK + tk] = hx;
      nrow(b, 1)[(tj + 1) * TK + tk] = hz;
      if (row_halo) {  // H_x, H_z at (i, j0-1, k)
        const int cr = sC(sc)[cq_r];
        const T ex_r = E0[eq_r], ey_r = E1[eq_r], ez_r = E2[eq_r];
        T hxr = coef(cr, 6) * sH(sc, 0)[hq_r] +
                coef(cr, 7) * (fhk * (E1[eq_r + 1] - ey_r) - fhj_r * (E2[eq_r + G::WE] - ez_r));
        T hzr = coef(cr, 10) * sH(sc, 2)[hq_r] +
                coef(cr, 11) * (fhj_r * (E0[eq_r + G::WE] - ex_r) - fhi * (N1[eq_r] - ey_r));
        if (TF && tm_r) {
          hxr = hyb_tfsf_h(p, tm_r, 0, i, j0 - 1, k, hxr, t);
          hzr = hyb_tfsf_h(p, tm_r, 2, i, j0 - 1, k, hzr, t);
        }
        nrow(b, 0)[tk] = hxr;
        nrow(b, 1)[tk] = hzr;
      }
      if (col_halo) {  // H_x, H_y at (i, j, k0-1)
        const int cc = sC(sc)[cq_c];
        const T ex_c = E0[eq_c], ey_c = E1[eq_c], ez_c = E2[eq_c];
        T hxc = coef(cc, 6) * sH(sc, 0)[hq_c] +
                coef(cc, 7) * (fhk_c * (E1[eq_c + 1] - ey_c) - fhj * (E2[eq_c + G::WE] - ez_c));
        T hyc = coef(cc, 8) * sH(sc, 1)[hq_c] +
                coef(cc, 9) * (fhi * (N2[eq_c] - ez_c) - fhk_c * (E0[eq_c + 1] - ex_c));
        if (TF && tm_c) {
          hxc = hyb_tfsf_h(p, tm_c, 0, i, j, k0 - 1, hxc, t);
          hyc = hyb_tfsf_h(p, tm_c, 1, i, j, k0 - 1, hyc, t);
        }
        ncol(b, 0)[tj] = hxc;
        ncol(b, 1)[tj] = hyc;
      }
    }
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // Every thread is past plane i-1 (stage q % S): refill it.
    if (q + S < n_staged) {
      if (tid == 0) {
        fence_proxy_async();
        issue(q + S);
      }
      ring.pending |= 1u << (q % S);
    }
    // ---------------------------------------------------------- E(i)
    {
      const T fei = p.fe[0][i];
      const T hy_k = tk > 0 ? T(0) : ncol(b, 1)[tj];
      const T hx_k = tk > 0 ? T(0) : ncol(b, 0)[tj];
      const T hy_s = __shfl_up_sync(0xffffffffu, hy, 1);
      const T hx_s = __shfl_up_sync(0xffffffffu, hx, 1);
      const T hym = tk > 0 ? hy_s : hy_k;
      const T hxm_k = tk > 0 ? hx_s : hx_k;
      const T hzm_j = nrow(b, 1)[tj * TK + tk];
      const T hxm_j = nrow(b, 0)[tj * TK + tk];
      const T ex_n = coef(cl, 0) * ex + coef(cl, 1) * (fej * (hz - hzm_j) - fek * (hy - hym));
      const T ey_n = coef(cl, 2) * ey + coef(cl, 3) * (fek * (hx - hxm_k) - fei * (hz - hz_prev));
      const T ez_n = coef(cl, 4) * ez + coef(cl, 5) * (fei * (hy - hy_prev) - fej * (hx - hxm_j));
      const long long o = i * PS + row;
      p.out[0][o] = ex_n;
      p.out[1][o] = ey_n;
      p.out[2][o] = ez_n;
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
