// Fused H-then-E marching sweep, two nodes per thread along k, for the
// CPML-free interior of the grid.
//
// Same step, same tiles of work and the same overlapped-tile scheme as
// k_fmarch (fmarch.cuh), with the k extent of a warp doubled: lane l of warp
// w holds nodes (j0-1+w, kb+2l) and (j0-1+w, kb+2l+1), kb = k0-2, k0 = 62 bx,
// so one warp covers 64 k nodes of which 62 (lanes 1..31) are owned and the
// tile of k_fmarch's k tiles 2 bx and 2 bx + 1 is exactly covered.  Pairs
// are read from the staged boxes and written to the field arrays as two-
// element vectors; the per-plane work of the ring (stage wait, barrier,
// refill) and of the loop is shared by two nodes.  The k-1 neighbour of the
// first node of a pair comes from lane l-1 by a warp shuffle, that of the
// second node from the thread itself.
//
// This form has no CPML terms: it is launched only on the box of tiles and
// plane chunks that meet no CPML layer (fmarch_split, engine.cu), the rest of
// the grid being swept by k_fmarch's CPML form.  TFSF H-face corrections are
// compiled in for launches of a scene that has them.
//
// Arithmetic and loop ranges: BasicUpdator::updateH / BasicUpdator3D::updateE
// (src/updator/basic_updator.cpp:23-36, src/updator/basic_updator_3d.cpp:38-69),
// TFSF3DCorrector::correctH (src/waveform_source/tfsf_corrector.cpp:205-232).
#pragma once

#include <type_traits>

#include "fmarch.cuh"

namespace xfd {

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

struct FvecMaps {
  CUtensorMap e[3];  // E of the input buffer, box (64+XA) x (TJ+1)
  CUtensorMap h[3];  // H of the input buffer, box (64+XA) x TJ
  CUtensorMap cls;   // class index, box 72 x TJ
};

template <typename T>
struct FvecP {
  FusedP<T> p;
  FvecMaps m;
  int org[3];  // first (k tile of 62, j tile, chunk) of the launch
};

template <typename T, int TJ>
struct FvecGeom {
  static constexpr int XA = 16 / (int)sizeof(T);
  static constexpr int W = 64 + XA;  // field box width
  static constexpr int WC = 72;      // class box width
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
  static constexpr int XB = 2 * 2 * TJ * 64 * (int)sizeof(T);  // [2][Hx,Hz][TJ][64]
  static constexpr int NC = 64;  // classes cached in shared memory
  static constexpr int TB = NC * 12 * (int)sizeof(T);
  __host__ __device__ static constexpr int smem(int S) {
    return S * STAGE + pad(XB) + TB + 8 * S;
  }
};

template <typename T, int TJ, int S>
__global__ void __launch_bounds__(TJ * 32, sizeof(T) == 8 ? 2 : 3)
    k_fvec(const __grid_constant__ FvecP<T> P) {
  using G = FvecGeom<T, TJ>;
  using T2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  const FusedP<T>& p = P.p;
  const Lat L = p.L;
  const int l = threadIdx.x, w = threadIdx.y, tid = w * 32 + l;
  // One thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)p.err & 2))) return;
  const int bx = blockIdx.x + P.org[0], by = blockIdx.y + P.org[1], bz = blockIdx.z + P.org[2];
  const int k0 = 62 * bx, j0 = (TJ - 1) * by;
  const int kb = k0 - 2;
  const int ka = kb + 2 * l;  // first node of the pair; the second is ka + 1
  const int j = j0 - 1 + w;
  const int i_lo = bz * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const int i_first = i_lo > 0 ? i_lo - 1 : 0;
  const int n_planes = i_hi - i_first;
  const int n_staged = n_planes + (i_hi <= L.nx ? 1 : 0);
  // Box origins along k rounded down to 16 bytes (kb >= -2, kb even).
  const int xe = (kb >= 0 ? kb / G::XA : -((-kb + G::XA - 1) / G::XA)) * G::XA;
  const int xc = (kb >= 0 ? kb / 8 : -((-kb + 7) / 8)) * 8;
  const int oe = kb - xe, oc = kb - xc;  // even: pairs stay vector-aligned

  StageRing ring;
  T* sX = reinterpret_cast<T*>(smem + S * G::STAGE);
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE + G::pad(G::XB));
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
    for (int x = tid; x < nt; x += TJ * 32) sT[x] = p.tab[x];
  }

  // ---------------------------------------------------------- per thread
  const bool jin = j >= 0 && j <= L.ny;
  bool act[2], own[2], kv[2], km[2];
  T fhk[2], fek[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = ka + e;
    act[e] = jin && k >= 0 && k <= L.nz;
    own[e] = act[e] && w >= 1 && l >= 1;
    kv[e] = k < L.nz;
    km[e] = k >= 1 && kv[e];
    fhk[e] = (act[e] && kv[e]) ? p.fh[2][k] : T(0);
    fek[e] = act[e] ? p.fe[2][k] : T(0);
  }
  const bool any_act = act[0] || act[1];
  const bool jv = j < L.ny, jm = j >= 1 && jv;
  const T fhj = (jin && jv) ? p.fh[1][j] : T(0);
  const T fej = jin ? p.fe[1][j] : T(0);
  const long long PS = (long long)L.NY * L.KP;
  const long long row = jin ? (long long)j * L.KP + ka : 0;
  const long long t = *p.step;
  const int eq = w * G::W + oe + 2 * l;    // first node of the pair in an E or H box
  const int cq = w * G::WC + oc + 2 * l;   // in the class box
  const int xq = w * 64 + 2 * l;           // in the exchange array
  T hy_p[2] = {T(0), T(0)}, hz_p[2] = {T(0), T(0)};  // H_y, H_z of plane i-1

  // Writes a pair, as one vector store when both nodes are written.
  auto put = [&](T* base, long long o, bool w0, bool w1, T v0, T v1) {
    if (w0 && w1) {
      *reinterpret_cast<T2*>(base + o) = T2{v0, v1};
    } else {
      if (w0) base[o] = v0;
      if (w1) base[o + 1] = v1;
    }
  };

  auto plane = [&](int i, int q, int sc, int sn, bool iv, T fhi, T fei, auto tf_tag) {
    constexpr bool TF = decltype(tf_tag)::value;
    const bool upd = i >= i_lo;
    const long long o = i * PS + row;
    T* xb = sX + (q & 1) * (2 * TJ * 64);
    T hx[2] = {T(0), T(0)}, hy[2] = {T(0), T(0)}, hz[2] = {T(0), T(0)};
    const T* r[2] = {nullptr, nullptr};
    // ---------------------------------------------------------- H(i)
    if (any_act) {
      const uint32_t c2 = *reinterpret_cast<const uint32_t*>(cbox(sc) + cq);
      const int cl[2] = {(int)(c2 & 0xffffu), (int)(c2 >> 16)};
#pragma unroll
      for (int e = 0; e < 2; ++e)
        r[e] = cl[e] < G::NC ? sT + cl[e] * 12 : p.tab + (size_t)cl[e] * 12;
      const T* Ex = ebox(sc, 0);
      const T* Ey = ebox(sc, 1);
      const T* Ez = ebox(sc, 2);
      const T2 ex = *reinterpret_cast<const T2*>(Ex + eq);
      const T2 exj = *reinterpret_cast<const T2*>(Ex + eq + G::W);
      const T ex2 = Ex[eq + 2];
      const T2 ey = *reinterpret_cast<const T2*>(Ey + eq);
      const T ey2 = Ey[eq + 2];
      const T2 ez = *reinterpret_cast<const T2*>(Ez + eq);
      const T2 ezj = *reinterpret_cast<const T2*>(Ez + eq + G::W);
      T2 eyn = T2{T(0), T(0)}, ezn = T2{T(0), T(0)};
      if (iv) {
        eyn = *reinterpret_cast<const T2*>(ebox(sn, 1) + eq);
        ezn = *reinterpret_cast<const T2*>(ebox(sn, 2) + eq);
      }
      const T dEy_k[2] = {ey.y - ey.x, ey2 - ey.y};
      const T dEz_j[2] = {ezj.x - ez.x, ezj.y - ez.y};
      const T dEz_i[2] = {ezn.x - ez.x, ezn.y - ez.y};
      const T dEx_k[2] = {ex.y - ex.x, ex2 - ex.y};
      const T dEx_j[2] = {exj.x - ex.x, exj.y - ex.y};
      const T dEy_i[2] = {eyn.x - ey.x, eyn.y - ey.y};
      const T2 hxo = *reinterpret_cast<const T2*>(hbox(sc, 0) + eq);
      const T2 hyo = *reinterpret_cast<const T2*>(hbox(sc, 1) + eq);
      const T2 hzo = *reinterpret_cast<const T2*>(hbox(sc, 2) + eq);
      const T hxv[2] = {hxo.x, hxo.y}, hyv[2] = {hyo.x, hyo.y}, hzv[2] = {hzo.x, hzo.y};
      bool vx[2], vy[2], vz[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (!act[e]) {
          vx[e] = vy[e] = vz[e] = false;
          continue;
        }
        const int k = ka + e;
        const T* re = r[e];
        const bool main_rng = iv && jv && kv[e];
        vx[e] = jv && kv[e];  // Hx: i <= nx, j < ny, k < nz
        vy[e] = iv && kv[e];  // Hy: i < nx, j <= ny, k < nz
        vz[e] = iv && jv;     // Hz: i < nx, j < ny, k <= nz
        if (vx[e]) {
          T h = hxv[e];
          if (main_rng) h = re[6] * h + re[7] * (fhk[e] * dEy_k[e] - fhj * dEz_j[e]);
          if constexpr (TF) h = tfsf_h_apply(p, 0, i, j, k, t, h);
          hx[e] = h;
        }
        if (vy[e]) {
          T h = hyv[e];
          if (main_rng) h = re[8] * h + re[9] * (fhi * dEz_i[e] - fhk[e] * dEx_k[e]);
          if constexpr (TF) h = tfsf_h_apply(p, 1, i, j, k, t, h);
          hy[e] = h;
        }
        if (vz[e]) {
          T h = hzv[e];
          if (main_rng) h = re[10] * h + re[11] * (fhj * dEx_j[e] - fhi * dEy_i[e]);
          if constexpr (TF) h = tfsf_h_apply(p, 2, i, j, k, t, h);
          hz[e] = h;
        }
      }
      if (upd) {
        const bool w0 = own[0], w1 = own[1];
        put(p.out[3], o, w0 && vx[0], w1 && vx[1], hx[0], hx[1]);
        put(p.out[4], o, w0 && vy[0], w1 && vy[1], hy[0], hy[1]);
        put(p.out[5], o, w0 && vz[0], w1 && vz[1], hz[0], hz[1]);
      }
    }
    // H_x, H_z for the row above; the second node's H_y, H_x to lane l+1.
    *reinterpret_cast<T2*>(xb + xq) = T2{hx[0], hx[1]};
    *reinterpret_cast<T2*>(xb + TJ * 64 + xq) = T2{hz[0], hz[1]};
    const T hy_k0 = __shfl_up_sync(0xffffffffu, hy[1], 1);
    const T hx_k0 = __shfl_up_sync(0xffffffffu, hx[1], 1);
    __syncthreads();
    // ---------------------------------------------------------- E(i)
    if ((own[0] || own[1]) && upd) {
      const T2 hxj = *reinterpret_cast<const T2*>(xb + xq - 64);
      const T2 hzj = *reinterpret_cast<const T2*>(xb + TJ * 64 + xq - 64);
      const bool i1 = i >= 1, im = i1 && iv;
      const T dHz_j[2] = {hz[0] - hzj.x, hz[1] - hzj.y};
      const T dHy_k[2] = {hy[0] - hy_k0, hy[1] - hy[0]};
      const T dHx_k[2] = {hx[0] - hx_k0, hx[1] - hx[0]};
      const T dHz_i[2] = {hz[0] - hz_p[0], hz[1] - hz_p[1]};
      const T dHy_i[2] = {hy[0] - hy_p[0], hy[1] - hy_p[1]};
      const T dHx_j[2] = {hx[0] - hxj.x, hx[1] - hxj.y};
      const T2 exo = *reinterpret_cast<const T2*>(ebox(sc, 0) + eq);
      const T2 eyo = *reinterpret_cast<const T2*>(ebox(sc, 1) + eq);
      const T2 ezo = *reinterpret_cast<const T2*>(ebox(sc, 2) + eq);
      T ex[2] = {exo.x, exo.y}, ey[2] = {eyo.x, eyo.y}, ez[2] = {ezo.x, ezo.y};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (!own[e]) continue;
        const T* re = r[e];
        // Ex: i < nx; main 1 <= j < ny, 1 <= k < nz
        if (jm && km[e]) ex[e] = re[0] * ex[e] + re[1] * (fej * dHz_j[e] - fek[e] * dHy_k[e]);
        // Ey: j < ny; main 1 <= i < nx, 1 <= k < nz
        if (im && km[e]) ey[e] = re[2] * ey[e] + re[3] * (fek[e] * dHx_k[e] - fei * dHz_i[e]);
        // Ez: k < nz; main 1 <= i < nx, 1 <= j < ny
        if (im && jm) ez[e] = re[4] * ez[e] + re[5] * (fei * dHy_i[e] - fej * dHx_j[e]);
      }
      put(p.out[0], o, own[0] && iv, own[1] && iv, ex[0], ex[1]);
      put(p.out[1], o, own[0] && jv, own[1] && jv, ey[0], ey[1]);
      put(p.out[2], o, own[0] && kv[0], own[1] && kv[1], ez[0], ez[1]);
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      hy_p[e] = hy[e];
      hz_p[e] = hz[e];
    }
  };

  bool ok = true;
  if (n_staged > 0) ok = ring.wait(0);
  T fhi_n = i_first < L.nx ? p.fh[0][i_first] : T(0);
  T fei_n = p.fe[0][i_first];
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
    if (p.tfh.enabled)
      plane(i, q, sc, sn, iv, fhi, fei, std::true_type{});
    else
      plane(i, q, sc, sn, iv, fhi, fei, std::false_type{});
  }
  if (!ok) {
    if (tid == 0) atomicOr(p.err, 2);
    ring.drain(S);
  }
}

}  // namespace xfd
