// Interior form of the TMA marching split sweeps with two rows per thread and
// a producer warp.  Same arithmetic as the CPML-free interior form of
// k_march_h_tma / k_march_e_tma (march_tma.cuh, IN = true) on the same box of
// nodes away from every CPML layer and lattice boundary, so no range tests and
// no psi terms; what changes is how the work is laid out:
//
//  * a CTA sweeps a 32 (k) x 16 (j) tile through a chunk of x planes; each of
//    its 8 consumer warps takes two adjacent rows, so the per-plane overheads
//    (stage wait, class and curl-factor lookups, addressing) are paid once per
//    two nodes and the j neighbour of the first row is the second row's value;
//  * a ninth warp only issues the TMA loads (cp.async.bulk.tensor, no
//    multicast) into a ring of S stages: stage s is filled on full[s] and
//    handed back on empty[s] when all 8 consumer warps have finished reading
//    it, so no CTA-wide barrier is taken per plane and a consumer warp runs
//    ahead of the others up to the ring's depth;
//  * the x curl factor of the next plane is loaded one plane ahead.
//
// Staged planes u = 0 .. n_planes (one more than the planes computed): for
// the H sweep plane i_lo + u (the last one E halo only), for the E sweep
// plane i_lo - 1 + u (the first one H halo only).  Computing plane c reads
// staged c and c + 1 and then releases staged c.
// Every mbarrier wait is bounded (a cycle budget of about 2 s).  A consumer
// warp that runs out sets bit 2 of the engine's error word and stops (it no
// longer releases stages); the producer that runs out waiting for a stage to
// come back sets the bit, stops issuing and waits (bounded) for the loads it
// has in flight before it exits.  Later launches that find the bit set return
// at once.
#pragma once

#include "march_tma.cuh"

namespace xfd {

constexpr int kWideTJ = 16;  // rows of a wide CTA
constexpr int kWideCW = 8;   // consumer warps (two rows each)

template <typename T, int S>
struct WideGeom {
  using G = MarchGeom<T, kWideTJ, 32>;
  static constexpr int kThreads = 32 * (kWideCW + 1);
  __host__ __device__ static constexpr int smem() { return S * G::STAGE + G::TB + 16 * S; }
};

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t ph) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(a), "r"(ph)
      : "memory");
  return done != 0;
}

// Wait for phase `ph` of `bar`, giving up after about 2 s (4e9 cycles).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t ph) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try(a, ph)) return true;
  const long long t0 = clock64();
  while (!mbar_try(a, ph))
    if (clock64() - t0 > 4000000000LL) return false;
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Producer warp body: issues staged planes 0 .. n_staged-1, refilling a stage
// once its previous plane has been released.  `issue(u, s, bar)` starts the
// loads of staged plane u into stage s.
template <int S, typename Issue>
__device__ __forceinline__ void wide_produce(uint64_t* full, uint64_t* empty, int n_staged,
                                            int* err, Issue issue) {
  if (threadIdx.x != 0) return;
  int issued = 0;
  bool ok = true;
  for (int u = 0; u < n_staged; ++u) {
    const int s = u % S;
    if (u >= S) {
      if (!mbar_wait_bounded(&empty[s], (uint32_t)((u / S - 1) & 1))) {
        ok = false;
        break;
      }
      fence_proxy_async();
    }
    issue(u, s, &full[s]);
    ++issued;
  }
  if (!ok) {
    atomicOr(err, 2);
    // Only the newest load of each stage can still be in flight.
    for (int u = issued > S ? issued - S : 0; u < issued; ++u)
      mbar_wait_bounded(&full[u % S], (uint32_t)((u / S) & 1));
  }
}

// ---------------------------------------------------------------------------
// H sweep: staged plane u = i_lo + u holds the E halo boxes (rows j0..j0+16,
// k0..k0+31+XA), the H tiles and the class tile; plane i_lo + n_planes only
// the E halo.
// ---------------------------------------------------------------------------
template <typename T, int S>
__global__ void __launch_bounds__(WideGeom<T, S>::kThreads)
    k_march_h_wide(const __grid_constant__ MarchTmaP<T> P) {
  using G = MarchGeom<T, kWideTJ, 32>;
  extern __shared__ __align__(128) unsigned char smem[];
  const MarchP<T>& p = P.p;
  const Lat L = p.L;
  const int lane = threadIdx.x, warp = threadIdx.y, tid = warp * 32 + lane;
  // One thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)P.err & 2))) return;
  const int k0 = (blockIdx.x + P.org[0]) * 32 + P.shift[0];
  const int j0 = (blockIdx.y + P.org[1]) * kWideTJ + P.shift[1];
  const int i_lo = (blockIdx.z + P.org[2]) * p.ichunk + P.shift[2];
  const int n_planes = min(p.ichunk, L.nx - i_lo);  // the box ends at or before nx
  const int n_staged = n_planes + 1;
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::TB);
  uint64_t* empty = full + S;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kWideCW);
    }
    fence_mbar_init();
  }
  stage_half_table<T, G::NC, WideGeom<T, S>::kThreads>(sT, p.tab, p.n_classes, 1, tid);
  __syncthreads();

  if (warp == kWideCW) {
    wide_produce<S>(full, empty, n_staged, P.err, [&](int u, int s, uint64_t* bar) {
      unsigned char* base = smem + s * G::STAGE;
      const int i = i_lo + u;
      const bool e_only = u == n_planes;
      mbar_expect_tx(bar, e_only ? G::TX_HALO : G::TX_FULL);
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::HALO_OFF + c * G::pad(G::HALO_B), &P.m.halo[c], k0, j0, i, bar);
      if (!e_only) {
        for (int c = 0; c < 3; ++c)
          tma_load_3d(base + G::TILE_OFF + c * G::pad(G::TILE_B), &P.m.tile[3 + c], k0, j0, i,
                      bar);
        tma_load_3d(base + G::CLS_OFF, &P.m.cls, k0, j0, i, bar);
      }
    });
    return;
  }

  // Consumer: rows j, j+1 (tile rows 2 warp, 2 warp + 1), column k.
  const int k = k0 + lane, j = j0 + 2 * warp;
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const T fhj0 = p.fh[1][j], fhj1 = p.fh[1][j + 1];
  const T fhk = p.fh[2][k];
  T* Hx = p.f[3] + row;
  T* Hy = p.f[4] + row;
  T* Hz = p.f[5] + row;
  constexpr int W = G::W;
  const int hq = 2 * warp * W + lane;   // row j, column k in a halo box
  const int tq = 2 * warp * 32 + lane;  // row j, column k in a tile box
  auto halo = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::HALO_OFF + c * G::pad(G::HALO_B));
  };
  auto tile = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::TILE_OFF + c * G::pad(G::TILE_B));
  };
  auto ctile = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::CLS_OFF);
  };

  bool ok = mbar_wait_bounded(&full[0], 0);
  T fhi_next = p.fh[0][i_lo];
  for (int c = 0; ok && c < n_planes; ++c) {
    const int i = i_lo + c;
    const int sc = c % S, sn = (c + 1) % S;
    const T fhi = fhi_next;
    if (c + 1 < n_planes) fhi_next = p.fh[0][i + 1];
    if (!mbar_wait_bounded(&full[sn], (uint32_t)(((c + 1) / S) & 1))) {
      ok = false;
      break;
    }
    const uint16_t* ct = ctile(sc);
    const int cl0 = ct[tq], cl1 = ct[tq + 32];
    const T* r0 = cl0 < G::NC ? sT + cl0 * 6 : p.tab + (size_t)cl0 * 12 + 6;
    const T* r1 = cl1 < G::NC ? sT + cl1 * 6 : p.tab + (size_t)cl1 * 12 + 6;
    const T* Exs = halo(sc, 0);
    const T* Eys = halo(sc, 1);
    const T* Ezs = halo(sc, 2);
    const T* Eyn = halo(sn, 1);
    const T* Ezn = halo(sn, 2);
    const T ex0 = Exs[hq], ex1 = Exs[hq + W], ex2 = Exs[hq + 2 * W];
    const T exk0 = Exs[hq + 1], exk1 = Exs[hq + W + 1];
    const T ey0 = Eys[hq], ey1 = Eys[hq + W];
    const T eyk0 = Eys[hq + 1], eyk1 = Eys[hq + W + 1];
    const T ez0 = Ezs[hq], ez1 = Ezs[hq + W], ez2 = Ezs[hq + 2 * W];
    const T eyn0 = Eyn[hq], eyn1 = Eyn[hq + W];
    const T ezn0 = Ezn[hq], ezn1 = Ezn[hq + W];
    const T* hx = tile(sc, 0);
    const T* hy = tile(sc, 1);
    const T* hz = tile(sc, 2);
    const T hx0 = hx[tq], hx1 = hx[tq + 32];
    const T hy0 = hy[tq], hy1 = hy[tq + 32];
    const T hz0 = hz[tq], hz1 = hz[tq + 32];
    const long long o = i * PS;
    // row j
    Hx[o] = r0[0] * hx0 + r0[1] * (fhk * (eyk0 - ey0) - fhj0 * (ez1 - ez0));
    Hy[o] = r0[2] * hy0 + r0[3] * (fhi * (ezn0 - ez0) - fhk * (exk0 - ex0));
    Hz[o] = r0[4] * hz0 + r0[5] * (fhj0 * (ex1 - ex0) - fhi * (eyn0 - ey0));
    // row j + 1
    Hx[o + KP] = r1[0] * hx1 + r1[1] * (fhk * (eyk1 - ey1) - fhj1 * (ez2 - ez1));
    Hy[o + KP] = r1[2] * hy1 + r1[3] * (fhi * (ezn1 - ez1) - fhk * (exk1 - ex1));
    Hz[o + KP] = r1[4] * hz1 + r1[5] * (fhj1 * (ex2 - ex1) - fhi * (eyn1 - ey1));
    // Every value read from stage sc has been used: hand it back.
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[sc]);
  }
  if (!ok && lane == 0) atomicOr(P.err, 2);
}

// ---------------------------------------------------------------------------
// E sweep: staged plane u = i_lo - 1 + u holds the H halo boxes (rows
// j0-1..j0+15, k0-XA..k0+31), the E tiles and the class tile; plane i_lo - 1
// only the H halo.
// ---------------------------------------------------------------------------
template <typename T, int S>
__global__ void __launch_bounds__(WideGeom<T, S>::kThreads)
    k_march_e_wide(const __grid_constant__ MarchTmaP<T> P) {
  using G = MarchGeom<T, kWideTJ, 32>;
  extern __shared__ __align__(128) unsigned char smem[];
  const MarchP<T>& p = P.p;
  const Lat L = p.L;
  const int lane = threadIdx.x, warp = threadIdx.y, tid = warp * 32 + lane;
  if (__syncthreads_or(tid == 0 && (*(volatile int*)P.err & 2))) return;
  const int k0 = (blockIdx.x + P.org[0]) * 32 + P.shift[0];
  const int j0 = (blockIdx.y + P.org[1]) * kWideTJ + P.shift[1];
  const int i_lo = (blockIdx.z + P.org[2]) * p.ichunk + P.shift[2];  // >= 1 inside the box
  const int n_planes = min(p.ichunk, L.nx - i_lo);
  const int n_staged = n_planes + 1;
  T* sT = reinterpret_cast<T*>(smem + S * G::STAGE);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::TB);
  uint64_t* empty = full + S;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kWideCW);
    }
    fence_mbar_init();
  }
  stage_half_table<T, G::NC, WideGeom<T, S>::kThreads>(sT, p.tab, p.n_classes, 0, tid);
  __syncthreads();

  if (warp == kWideCW) {
    wide_produce<S>(full, empty, n_staged, P.err, [&](int u, int s, uint64_t* bar) {
      unsigned char* base = smem + s * G::STAGE;
      const int i = i_lo - 1 + u;
      const bool h_only = u == 0;
      mbar_expect_tx(bar, h_only ? G::TX_HALO : G::TX_FULL);
      for (int c = 0; c < 3; ++c)
        tma_load_3d(base + G::HALO_OFF + c * G::pad(G::HALO_B), &P.m.halo[3 + c], k0 - G::XA,
                    j0 - 1, i, bar);
      if (!h_only) {
        for (int c = 0; c < 3; ++c)
          tma_load_3d(base + G::TILE_OFF + c * G::pad(G::TILE_B), &P.m.tile[c], k0, j0, i, bar);
        tma_load_3d(base + G::CLS_OFF, &P.m.cls, k0, j0, i, bar);
      }
    });
    return;
  }

  const int k = k0 + lane, j = j0 + 2 * warp;
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const T fej0 = p.fe[1][j], fej1 = p.fe[1][j + 1];
  const T fek = p.fe[2][k];
  T* Ex = p.f[0] + row;
  T* Ey = p.f[1] + row;
  T* Ez = p.f[2] + row;
  constexpr int W = G::W;
  const int hq = (2 * warp + 1) * W + lane + G::XA;  // row j, column k in a halo box
  const int tq = 2 * warp * 32 + lane;
  auto halo = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::HALO_OFF + c * G::pad(G::HALO_B));
  };
  auto tile = [&](int s, int c) {
    return reinterpret_cast<const T*>(smem + s * G::STAGE + G::TILE_OFF + c * G::pad(G::TILE_B));
  };
  auto ctile = [&](int s) {
    return reinterpret_cast<const uint16_t*>(smem + s * G::STAGE + G::CLS_OFF);
  };

  bool ok = mbar_wait_bounded(&full[0], 0);
  T fei_next = p.fe[0][i_lo];
  for (int c = 0; ok && c < n_planes; ++c) {
    const int i = i_lo + c;
    const int sp = c % S, sc = (c + 1) % S;  // staged c: plane i-1; staged c+1: plane i
    const T fei = fei_next;
    if (c + 1 < n_planes) fei_next = p.fe[0][i + 1];
    if (!mbar_wait_bounded(&full[sc], (uint32_t)(((c + 1) / S) & 1))) {
      ok = false;
      break;
    }
    const uint16_t* ct = ctile(sc);
    const int cl0 = ct[tq], cl1 = ct[tq + 32];
    const T* r0 = cl0 < G::NC ? sT + cl0 * 6 : p.tab + (size_t)cl0 * 12;
    const T* r1 = cl1 < G::NC ? sT + cl1 * 6 : p.tab + (size_t)cl1 * 12;
    const T* Hxs = halo(sc, 0);
    const T* Hys = halo(sc, 1);
    const T* Hzs = halo(sc, 2);
    const T hxm = Hxs[hq - W], hx0 = Hxs[hq], hx1 = Hxs[hq + W];
    const T hxk0 = Hxs[hq - 1], hxk1 = Hxs[hq + W - 1];
    const T hy0 = Hys[hq], hy1 = Hys[hq + W];
    const T hyk0 = Hys[hq - 1], hyk1 = Hys[hq + W - 1];
    const T hzm = Hzs[hq - W], hz0 = Hzs[hq], hz1 = Hzs[hq + W];
    const T hyp0 = halo(sp, 1)[hq], hyp1 = halo(sp, 1)[hq + W];
    const T hzp0 = halo(sp, 2)[hq], hzp1 = halo(sp, 2)[hq + W];
    const T* ex = tile(sc, 0);
    const T* ey = tile(sc, 1);
    const T* ez = tile(sc, 2);
    const T ex0 = ex[tq], ex1 = ex[tq + 32];
    const T ey0 = ey[tq], ey1 = ey[tq + 32];
    const T ez0 = ez[tq], ez1 = ez[tq + 32];
    const long long o = i * PS;
    // row j
    Ex[o] = r0[0] * ex0 + r0[1] * (fej0 * (hz0 - hzm) - fek * (hy0 - hyk0));
    Ey[o] = r0[2] * ey0 + r0[3] * (fek * (hx0 - hxk0) - fei * (hz0 - hzp0));
    Ez[o] = r0[4] * ez0 + r0[5] * (fei * (hy0 - hyp0) - fej0 * (hx0 - hxm));
    // row j + 1
    Ex[o + KP] = r1[0] * ex1 + r1[1] * (fej1 * (hz1 - hz0) - fek * (hy1 - hyk1));
    Ey[o + KP] = r1[2] * ey1 + r1[3] * (fek * (hx1 - hxk1) - fei * (hz1 - hzp1));
    Ez[o + KP] = r1[4] * ez1 + r1[5] * (fei * (hy1 - hyp1) - fej1 * (hx1 - hx0));
    // Plane i-1 (staged c) is no longer needed.
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[sp]);
  }
  if (!ok && lane == 0) atomicOr(P.err, 2);
}

}  // namespace xfd
