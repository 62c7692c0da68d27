// Fused H-then-E marching sweep with overlapped tiles and TMA-staged planes.
//
// One launch per time step advances the Yee fields from the `in` buffers
// (E^n, H^{n-1/2}) to the `out` buffers (E^{n+1}, H^{n+1/2}), with the CPML
// auxiliaries of both phases and the TFSF H-face corrections, as k_fused
// (fused.cuh) does.  What differs is the work decomposition:
//
//  * A CTA is TJ warps; warp w, lane l is node (j0-1+w, k0-1+l) of the (j,k)
//    plane.  Every thread computes H at its node; the E update, and the
//    writes of both fields, belong to the threads with w >= 1 and l >= 1.
//    Neighbouring tiles therefore overlap by one row and one column
//    (k0 = 31 bx, j0 = (TJ-1) by), the overlapped H being recomputed
//    identically from the same inputs; no thread needs a second pass.
//  * The H values E needs from the node below in k come from lane l-1 by a
//    warp shuffle, those from the row below in j through a double-buffered
//    shared array, those from plane i-1 from the thread's own registers.
//  * The CTA marches along i over a chunk of planes, starting one plane
//    early (H only) to rebuild H of plane i_lo-1.  Per plane it needs E, old
//    H and the class index of its tile: one thread issues TMA tile loads
//    (cp.async.bulk.tensor, no multicast) of the planes ahead into a ring of
//    S stages with one mbarrier each.  H of plane i also needs E of plane
//    i+1, which is the next stage (an E-only stage past the chunk's end).
//  * Two CTA barriers per plane: one before the H phase (after which the
//    stage of plane q-1 is refilled), one between the H and E phases.
//  * The CPML terms are compiled into a second form of the plane body that
//    the CTA takes only on planes or tiles meeting a slab (a CTA-uniform
//    test), so the interior runs without them; the old psi values a node
//    reads are loaded one phase ahead (H psi of plane i+1 after the H phase
//    of plane i, E psi after the E phase), so their DRAM latency overlaps
//    the compute of the other phase.  The TFSF H-face corrections are compiled
//    in only for launches of a scene that has them.
//  * The table rows of the NC most frequent material classes (the engine
//    numbers classes by descending node count) are copied to shared memory
//    once per CTA; rarer classes are read from global memory.  The shared
//    copy keeps the lookups off L1, which the stage ring mostly occupies.
//  * Box origins along k are rounded down to 16 bytes; the thread's column
//    inside a box is offset by the remainder.  Out-of-range rows, columns
//    and planes read as zeros and feed no update.
//
// Arithmetic, loop ranges and correction order follow the reference:
// BasicUpdator::updateH / BasicUpdator3D::updateE
// (src/updator/basic_updator.cpp:23-36, src/updator/basic_updator_3d.cpp:38-69),
// TFSF3DCorrector::correctH (src/waveform_source/tfsf_corrector.cpp:205-232) on H
// before the CPML terms, PMLCorrector<xyz>::correctH/correctE
// (src/include/boundary/pml_corrector.h:178-382) over each component's
// whole transverse extent, slab axes in ascending order.  CPML H psi
// ping-pong with the fields (overlapped nodes read the old psi and only the
// owning thread writes); E psi is updated in place by its owner.
//
// Stage waits are bounded (a cycle budget); on expiry the CTA sets bit 2 of
// the engine's error word, drains its loads in flight and returns, and
// launches that find the bit set return at once.
#pragma once

#include <type_traits>

#include "fused.cuh"
#include "march.cuh"
#include "march_tma.cuh"

namespace xfd {

struct FmarchMaps {
  CUtensorMap e[3];  // E of the input buffer, box (TK+XA) x (TJ+1)
  CUtensorMap h[3];  // H of the input buffer, box (TK+XA) x TJ
  CUtensorMap cls;   // class index, box (TK+8) x TJ
};

// Work split: the tiles and plane chunks that meet no CPML layer form a box
// in (tile k, tile j, chunk) index space, swept by the ANYCP = false form
// of the kernel (no CPML code at all, fewer registers) with its grid offset
// by `org`; the ANYCP = true form takes the full grid and its CTAs inside
// the box [box_lo, box_hi) return at once.
template <typename T>
struct FmarchP {
  FusedP<T> p;
  FmarchMaps m;
  int org[3];
  int box_lo[3], box_hi[3];
};

template <typename T, int TJ>
struct FmarchGeom {
  static constexpr int TK = 32;
  static constexpr int XA = 16 / (int)sizeof(T);
  static constexpr int W = TK + XA;  // field box width
  static constexpr int WC = TK + 8;  // class box width
  __host__ __device__ static constexpr int pad(int b) { return (b + 127) / 128 * 128; }
  static constexpr int EB = (TJ + 1) * W * (int)sizeof(T);
  static constexpr int HB = TJ * W * (int)sizeof(T);
  static constexpr int CB = TJ * WC * 2;
  static constexpr int E_OFF = 0;
  static constexpr int H_OFF = 3 * pad(EB);
  static constexpr int C_OFF = H_OFF + 3 * pad(HB);
  static constexpr int STAGE = C_OFF + pad(CB);
  static constexpr int TX_FULL = 3 * EB + 3 * HB + CB;
  static constexpr int TX_E = 3 * EB;
  static constexpr int XB = 2 * 2 * TJ * TK * (int)sizeof(T);  // H exchange [2][Hx,Hz][TJ][TK]
  static constexpr int NC = 128;                             // classes cached in shared memory
  static constexpr int TB = NC * 12 * (int)sizeof(T);
  __host__ __device__ static constexpr int smem(int S) {
    return S * STAGE + pad(XB) + TB + 8 * S;
  }
  // Tiles: k0 = (TK-1) bx, j0 = (TJ-1) by.
  __host__ __device__ static constexpr int tiles_k(int nz) { return (nz + 1 + TK - 2) / (TK - 1); }
  __host__ __device__ static constexpr int tiles_j(int ny) { return (ny + 1 + TJ - 2) / (TJ - 1); }
};

// TFSF H-face corrections of component c at node (i, j, k), in pass order.
template <typename T>
__device__ __forceinline__ T tfsf_h_apply(const FusedP<T>& p, int c, int i, int j, int k,
                                          long long t, T h) {
  for (int s = 0; s < p.tfh.n[c]; ++s) {
    const TfsfHPass& Q = p.tfh.pass[c][s];
    if (i < Q.lo[0] || i >= Q.hi[0] || j < Q.lo[1] || j >= Q.hi[1] || k < Q.lo[2] ||
        k >= Q.hi[2])
      continue;
    int xi[3] = {i, j, k};
    if (Q.neg) xi[Q.m] += 1;
    int e_flag = 0;
    const double v = tfsf_incident(p.tf, true, Q.dual, t, xi, &e_flag);
    if (e_flag) atomicOr(p.err, 1);
    h = (T)((double)h + v * Q.coeff);
  }
  return h;
}

// Resident CTAs per SM each form is compiled for (its register budget).
template <typename T, bool ANYCP>
constexpr int fmarch_min_blocks() {
  return ANYCP ? (sizeof(T) == 8 ? 2 : 3) : (sizeof(T) == 8 ? 3 : 5);
}

template <typename T, int TJ, int S, bool ANYCP>
__global__ void __launch_bounds__(TJ * 32, (fmarch_min_blocks<T, ANYCP>()))
    k_fmarch(const __grid_constant__ FmarchP<T> P) {
  using G = FmarchGeom<T, TJ>;
  constexpr int TK = G::TK;
  extern __shared__ __align__(128) unsigned char smem[];
  const FusedP<T>& p = P.p;
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  const int bx = blockIdx.x + P.org[0], by = blockIdx.y + P.org[1], bz = blockIdx.z + P.org[2];
  if (ANYCP && bx >= P.box_lo[0] && bx < P.box_hi[0] && by >= P.box_lo[1] &&
      by < P.box_hi[1] && bz >= P.box_lo[2] && bz < P.box_hi[2])
    return;  // swept by the CPML-free form
  // One thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)p.err & 2))) return;
  const int k0 = bx * (TK - 1), j0 = by * (TJ - 1);
  const int k = k0 - 1 + tk, j = j0 - 1 + tj;
  const int i_lo = bz * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const int i_first = i_lo > 0 ? i_lo - 1 : 0;
  const int n_planes = i_hi - i_first;                     // computed planes
  const int n_staged = n_planes + (i_hi <= L.nx ? 1 : 0);  // + E-only plane i_hi
  // Box origins along k, rounded down to 16 bytes (floor division).
  const int kx = k0 - 1;
  const int xe = (kx >= 0 ? kx / G::XA : -((-kx + G::XA - 1) / G::XA)) * G::XA;
  const int xc = (kx >= 0 ? kx / 8 : -((-kx + 7) / 8)) * 8;
  const int oe = kx - xe, oc = kx - xc;  // column offsets of k0-1 in the boxes

  StageRing ring;
  T* sX = reinterpret_cast<T*>(smem + S * G::STAGE);  // [2][2][TJ][TK]
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE + G::pad(G::XB));  // [NC][12]
  ring.bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::pad(G::XB) + G::TB);
  auto ebox = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::E_OFF + c * G::pad(G::EB));
  };
  auto hbox = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::H_OFF + c * G::pad(G::HB));
  };
  auto cbox = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::C_OFF);
  };
  auto issue = [&](int q) {
    const int s = q % S, i = i_first + q;
    uint64_t* bar = &ring.bars[s];
    unsigned char* base = smem + s * G::STAGE;
    const bool e_only = q == n_planes;
    mbar_expect_tx(bar, e_only ? G::TX_E : G::TX_FULL);
    for (int c = 0; c < 3; ++c)
      tma_load_3d(base + G::E_OFF + c * G::pad(G::EB), &P.m.e[c], xe, j0 - 1, i, bar);
    if (!e_only) {
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::H_OFF + c * G::pad(G::HB), &P.m.h[c], xe, j0 - 1, i, bar);
      tma_load_3d(base + G::C_OFF, &P.m.cls, xc, j0 - 1, i, bar);
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
  {
    const int nt = min(p.n_classes, G::NC) * 12;
    for (int x = tid; x < nt; x += TJ * TK) sT[x] = p.tab[x];
  }

  // ---------------------------------------------------------- per thread
  const bool act = j >= 0 && j <= L.ny && k >= 0 && k <= L.nz;
  const bool own = act && tj >= 1 && tk >= 1;
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = act ? (long long)j * KP + k : 0;
  const bool jv = j < L.ny, kv = k < L.nz;
  const bool jm = j >= 1 && jv, km = k >= 1 && kv;
  const T fhj = (act && jv) ? p.fh[1][j] : T(0);
  const T fhk = (act && kv) ? p.fh[2][k] : T(0);
  const T fej = act ? p.fe[1][j] : T(0);
  const T fek = act ? p.fe[2][k] : T(0);
  // CPML layers normal to y and z (H and E layers), fixed for the march.
  int qyh = 0, qzh = 0, qye = 0, qze = 0;
  const int lyh = act ? layer_of(p.slab[1], j, false, qyh) : -1;
  const int lzh = act ? layer_of(p.slab[2], k, false, qzh) : -1;
  const int lye = own ? layer_of(p.slab[1], j, true, qye) : -1;
  const int lze = own ? layer_of(p.slab[2], k, true, qze) : -1;
  const long long t = *p.step;
  const int eq = tj * G::W + oe + tk;   // node (j, k) in an E or H box
  const int cq = tj * G::WC + oc + tk;  // node (j, k) in the class box
  const int xq = tj * TK + tk;          // node (j, k) in the exchange array
  T hy_p = T(0), hz_p = T(0);           // H_y, H_z of plane i-1

  // CPML grading of the node's y and z layers, fixed for the march.
  T ahy = 0, bhy = 0, ahz = 0, bhz = 0, aey = 0, bey = 0, aez = 0, bez = 0;
  if (lyh >= 0) ahy = p.slab[1].a_h[qyh][lyh], bhy = p.slab[1].b_h[qyh][lyh];
  if (lzh >= 0) ahz = p.slab[2].a_h[qzh][lzh], bhz = p.slab[2].b_h[qzh][lzh];
  if (lye >= 0) aey = p.slab[1].a_e[qye][lye], bey = p.slab[1].b_e[qye][lye];
  if (lze >= 0) aez = p.slab[2].a_e[qze][lze], bez = p.slab[2].b_e[qze][lze];
  // psi cell offsets within a slab array on plane i: y slab [i][l][k],
  // z slab [i][j][l], x slab [l][j][k].
  auto off_y = [&](int i, int q, int l) { return ((long long)i * p.slab[1].n[q] + l) * KP + k; };
  auto off_z = [&](int i, int q, int l) {
    return ((long long)i * L.NY + j) * p.slab[2].n[q] + l;
  };
  auto off_x = [&](int l) { return (long long)l * PS + (long long)j * KP + k; };
  // The psi values the node reads on plane i, in slot order
  //   H: 0 Hx-y 1 Hx-z 2 Hy-x 3 Hy-z 4 Hz-x 5 Hz-y   (old psi_h)
  //   E: 6 Ex-y 7 Ex-z 8 Ey-x 9 Ey-z 10 Ez-x 11 Ez-y (psi_e)
  // Slabs store component A=(m+1)%3 at index 0 and B=(m+2)%3 at index 1.
  auto load_psi_h = [&](int i, T (&v)[12]) {
    const SlabAxisD<T>& X = p.slab[0];
    const SlabAxisD<T>& Y = p.slab[1];
    const SlabAxisD<T>& Z = p.slab[2];
    int qxh = 0;
    const int lxh = act ? layer_of(X, i, false, qxh) : -1;
    v[0] = lyh >= 0 ? Y.psi_h_in[qyh][1][off_y(i, qyh, lyh)] : T(0);
    v[5] = lyh >= 0 ? Y.psi_h_in[qyh][0][off_y(i, qyh, lyh)] : T(0);
    v[1] = lzh >= 0 ? Z.psi_h_in[qzh][0][off_z(i, qzh, lzh)] : T(0);
    v[3] = lzh >= 0 ? Z.psi_h_in[qzh][1][off_z(i, qzh, lzh)] : T(0);
    v[2] = lxh >= 0 ? X.psi_h_in[qxh][0][off_x(lxh)] : T(0);
    v[4] = lxh >= 0 ? X.psi_h_in[qxh][1][off_x(lxh)] : T(0);
  };
  auto load_psi_e = [&](int i, T (&v)[12]) {
    const SlabAxisD<T>& X = p.slab[0];
    const SlabAxisD<T>& Y = p.slab[1];
    const SlabAxisD<T>& Z = p.slab[2];
    int qxe = 0;
    const int lxe = (own && i >= i_lo) ? layer_of(X, i, true, qxe) : -1;
    const bool e_rd = i >= i_lo;  // E psi is read only on updated planes
    v[6] = (e_rd && lye >= 0) ? Y.psi_e[qye][1][off_y(i, qye, lye)] : T(0);
    v[11] = (e_rd && lye >= 0) ? Y.psi_e[qye][0][off_y(i, qye, lye)] : T(0);
    v[7] = (e_rd && lze >= 0) ? Z.psi_e[qze][0][off_z(i, qze, lze)] : T(0);
    v[9] = (e_rd && lze >= 0) ? Z.psi_e[qze][1][off_z(i, qze, lze)] : T(0);
    v[8] = lxe >= 0 ? X.psi_e[qxe][0][off_x(lxe)] : T(0);
    v[10] = lxe >= 0 ? X.psi_e[qxe][1][off_x(lxe)] : T(0);
  };

  // One plane: H(i) (all threads), the row/column exchange, E(i) (owners).
  // CP: the CPML terms, with the old psi values of plane i in ps; each
  // phase, once done, reloads its slots of ps for plane i+1 when `nxt`.
  // TF: the TFSF H faces.
  auto plane = [&](int i, int q, int sc, int sn, bool iv, T fhi, T fei, T (&ps)[12], bool nxt,
                   auto cp_tag, auto tf_tag) {
    constexpr bool CP = decltype(cp_tag)::value;
    constexpr bool TF = decltype(tf_tag)::value;
    const bool upd = i >= i_lo;  // E update and writes (plane i_lo-1 is H only)
    const long long o = i * PS + row;
    T* xb = sX + (q & 1) * (2 * TJ * TK);
    T hx = T(0), hy = T(0), hz = T(0);
    const T* r = nullptr;
    const SlabAxisD<T>& X = p.slab[0];
    const SlabAxisD<T>& Y = p.slab[1];
    const SlabAxisD<T>& Z = p.slab[2];
    int qxh = 0, qxe = 0;
    const int lxh = CP ? layer_of(X, i, false, qxh) : -1;
    const int lxe = CP ? layer_of(X, i, true, qxe) : -1;
    T axh = 0, bxh = 0, axe = 0, bxe = 0;
    if (CP && lxh >= 0) axh = X.a_h[qxh][lxh], bxh = X.b_h[qxh][lxh];
    if (CP && lxe >= 0) axe = X.a_e[qxe][lxe], bxe = X.b_e[qxe][lxe];
    // ---------------------------------------------------------- H(i)
    if (act) {
      const int cl = cbox(sc)[cq];
      r = cl < G::NC ? sT + cl * 12 : p.tab + (size_t)cl * 12;
      const T* Ex = ebox(sc, 0);
      const T* Ey = ebox(sc, 1);
      const T* Ez = ebox(sc, 2);
      const T ex = Ex[eq], ex_k = Ex[eq + 1], ex_j = Ex[eq + G::W];
      const T ey = Ey[eq], ey_k = Ey[eq + 1];
      const T ez = Ez[eq], ez_j = Ez[eq + G::W];
      const T ey_n = iv ? ebox(sn, 1)[eq] : T(0);
      const T ez_n = iv ? ebox(sn, 2)[eq] : T(0);
      const T dEy_k = ey_k - ey, dEz_j = ez_j - ez;  // Hx
      const T dEz_i = ez_n - ez, dEx_k = ex_k - ex;  // Hy
      const T dEx_j = ex_j - ex, dEy_i = ey_n - ey;  // Hz
      const bool main_rng = iv && jv && kv;
      const bool wr = own && upd;
      if (jv && kv) {  // Hx: i <= nx, j < ny, k < nz
        const T ca = r[6], cb = r[7];
        T h = hbox(sc, 0)[eq];
        if (main_rng) h = ca * h + cb * (fhk * dEy_k - fhj * dEz_j);
        if constexpr (TF) h = tfsf_h_apply(p, 0, i, j, k, t, h);
        if constexpr (CP) {
          if (lyh >= 0) {
            const T v = bhy * ps[0] + ahy * dEz_j;
            if (wr) Y.psi_h_out[qyh][1][off_y(i, qyh, lyh)] = v;
            h -= cb * v;
          }
          if (lzh >= 0) {
            const T v = bhz * ps[1] + ahz * dEy_k;
            if (wr) Z.psi_h_out[qzh][0][off_z(i, qzh, lzh)] = v;
            h += cb * v;
          }
        }
        hx = h;
        if (wr) p.out[3][o] = h;
      }
      if (iv && kv) {  // Hy: i < nx, j <= ny, k < nz
        const T ca = r[8], cb = r[9];
        T h = hbox(sc, 1)[eq];
        if (main_rng) h = ca * h + cb * (fhi * dEz_i - fhk * dEx_k);
        if constexpr (TF) h = tfsf_h_apply(p, 1, i, j, k, t, h);
        if constexpr (CP) {
          if (lxh >= 0) {
            const T v = bxh * ps[2] + axh * dEz_i;
            if (wr) X.psi_h_out[qxh][0][off_x(lxh)] = v;
            h += cb * v;
          }
          if (lzh >= 0) {
            const T v = bhz * ps[3] + ahz * dEx_k;
            if (wr) Z.psi_h_out[qzh][1][off_z(i, qzh, lzh)] = v;
            h -= cb * v;
          }
        }
        hy = h;
        if (wr) p.out[4][o] = h;
      }
      if (iv && jv) {  // Hz: i < nx, j < ny, k <= nz
        const T ca = r[10], cb = r[11];
        T h = hbox(sc, 2)[eq];
        if (main_rng) h = ca * h + cb * (fhj * dEx_j - fhi * dEy_i);
        if constexpr (TF) h = tfsf_h_apply(p, 2, i, j, k, t, h);
        if constexpr (CP) {
          if (lxh >= 0) {
            const T v = bxh * ps[4] + axh * dEy_i;
            if (wr) X.psi_h_out[qxh][1][off_x(lxh)] = v;
            h -= cb * v;
          }
          if (lyh >= 0) {
            const T v = bhy * ps[5] + ahy * dEx_j;
            if (wr) Y.psi_h_out[qyh][0][off_y(i, qyh, lyh)] = v;
            h += cb * v;
          }
        }
        hz = h;
        if (wr) p.out[5][o] = h;
      }
    }
    if constexpr (CP) {
      if (nxt) load_psi_h(i + 1, ps);  // in flight through the E phase
    }
    // H_x, H_z for the row above; H_y, H_x from lane k-1 by shuffle.
    xb[xq] = hx;
    xb[TJ * TK + xq] = hz;
    const T hy_k = __shfl_up_sync(0xffffffffu, hy, 1);
    const T hx_k = __shfl_up_sync(0xffffffffu, hx, 1);
    __syncthreads();
    // ---------------------------------------------------------- E(i)
    if (own && upd) {
      const T hx_j = xb[xq - TK];
      const T hz_j = xb[TJ * TK + xq - TK];
      const bool i1 = i >= 1, im = i1 && iv;
      const T dHz_j = hz - hz_j, dHy_k = hy - hy_k;  // Ex
      const T dHx_k = hx - hx_k, dHz_i = hz - hz_p;  // Ey
      const T dHy_i = hy - hy_p, dHx_j = hx - hx_j;  // Ez
      if (iv) {  // Ex: i < nx; main 1 <= j < ny, 1 <= k < nz
        const T ca = r[0], cb = r[1];
        T e = ebox(sc, 0)[eq];
        if (jm && km) e = ca * e + cb * (fej * dHz_j - fek * dHy_k);
        if constexpr (CP) {
          if (lye >= 0) {
            const T v = bey * ps[6] + aey * dHz_j;
            Y.psi_e[qye][1][off_y(i, qye, lye)] = v;
            e += cb * v;
          }
          if (lze >= 0) {
            const T v = bez * ps[7] + aez * dHy_k;
            Z.psi_e[qze][0][off_z(i, qze, lze)] = v;
            e -= cb * v;
          }
        }
        p.out[0][o] = e;
      }
      if (jv) {  // Ey: j < ny; main 1 <= i < nx, 1 <= k < nz
        const T ca = r[2], cb = r[3];
        T e = ebox(sc, 1)[eq];
        if (im && km) e = ca * e + cb * (fek * dHx_k - fei * dHz_i);
        if constexpr (CP) {
          if (lxe >= 0) {
            const T v = bxe * ps[8] + axe * dHz_i;
            X.psi_e[qxe][0][off_x(lxe)] = v;
            e -= cb * v;
          }
          if (lze >= 0) {
            const T v = bez * ps[9] + aez * dHx_k;
            Z.psi_e[qze][1][off_z(i, qze, lze)] = v;
            e += cb * v;
          }
        }
        p.out[1][o] = e;
      }
      if (kv) {  // Ez: k < nz; main 1 <= i < nx, 1 <= j < ny
        const T ca = r[4], cb = r[5];
        T e = ebox(sc, 2)[eq];
        if (im && jm) e = ca * e + cb * (fei * dHy_i - fej * dHx_j);
        if constexpr (CP) {
          if (lxe >= 0) {
            const T v = bxe * ps[10] + axe * dHy_i;
            X.psi_e[qxe][1][off_x(lxe)] = v;
            e += cb * v;
          }
          if (lye >= 0) {
            const T v = bey * ps[11] + aey * dHx_j;
            Y.psi_e[qye][0][off_y(i, qye, lye)] = v;
            e -= cb * v;
          }
        }
        p.out[2][o] = e;
      }
    }
    if constexpr (CP) {
      if (nxt) load_psi_e(i + 1, ps);  // in flight through the next H phase
    }
    hy_p = hy;
    hz_p = hz;
  };
  auto run_plane = [&](int i, int q, int sc, int sn, bool iv, T fhi, T fei, T (&ps)[12],
                       bool nxt, auto cp_tag) {
    if (p.tfh.enabled)
      plane(i, q, sc, sn, iv, fhi, fei, ps, nxt, cp_tag, std::true_type{});
    else
      plane(i, q, sc, sn, iv, fhi, fei, ps, nxt, cp_tag, std::false_type{});
  };
  // CPML layers of plane i along x (either phase), uniform over the CTA.
  auto x_cpml = [&](int i) {
    int qq;
    return layer_of(p.slab[0], i, false, qq) >= 0 || layer_of(p.slab[0], i, true, qq) >= 0;
  };
  const bool tile_cpml = __syncthreads_or(lyh >= 0 || lzh >= 0 || lye >= 0 || lze >= 0);

  bool ok = true;
  if (n_staged > 0) ok = ring.wait(0);
  // x curl factors and the psi values of the next plane, loaded one plane ahead
  T fhi_n = i_first < L.nx ? p.fh[0][i_first] : T(0);
  T fei_n = p.fe[0][i_first];
  T pf[12] = {};
  int pf_i = -1;
  for (int q = 0; q < n_planes; ++q) {
    const int i = i_first + q;
    const bool iv = i < L.nx;
    const int sc = q % S, sn = (q + 1) % S;
    const T fhi = fhi_n, fei = fei_n;
    if (q + 1 < n_planes) {
      fhi_n = i + 1 < L.nx ? p.fh[0][i + 1] : T(0);
      fei_n = p.fe[0][i + 1];
    }
    if (ok && iv) ok = ring.wait(sn);  // E of plane i+1
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
    if constexpr (ANYCP) {
      if (tile_cpml || x_cpml(i)) {  // CTA-uniform
        if (pf_i != i) {
          load_psi_h(i, pf);
          load_psi_e(i, pf);
        }
        const bool nxt = q + 1 < n_planes && (tile_cpml || x_cpml(i + 1));
        run_plane(i, q, sc, sn, iv, fhi, fei, pf, nxt, std::true_type{});
        pf_i = nxt ? i + 1 : -1;
        continue;
      }
    }
    run_plane(i, q, sc, sn, iv, fhi, fei, pf, false, std::false_type{});
  }
  if (!ok) {
    if (tid == 0) atomicOr(p.err, 2);
    ring.drain(S);
  }
}

}  // namespace xfd
