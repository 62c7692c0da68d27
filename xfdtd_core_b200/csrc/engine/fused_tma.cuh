// Pipelined fused H-then-E sweep: the per-plane inputs of k_fused (E^n of
// plane i+1 with its halo, H^{n-1/2} of plane i, the class index of plane i)
// are brought into a ring of S shared-memory stages by TMA tile loads issued
// S-2 planes ahead, so DRAM latency overlaps the compute of earlier planes.
// Arithmetic, ranges and correction order are those of k_fused (fused.cuh).
//
// TMA boxes start on 16-byte boundaries along k (k0 - 16/sizeof(T) for the
// fields, k0 - 8 for the uint16 class), wider than the tile so that the
// k0-1 .. k0+TK halo is inside; out-of-range rows and planes read zeros.
// Waits on the stage barriers are bounded by a cycle budget: on expiry the
// CTA records an error (bit 2 of the engine's error word) and drains its
// outstanding loads before returning; launches that find the bit set return.
#pragma once

#include "fused.cuh"
#include "tma.cuh"

namespace xfd {

struct TmaMaps {
  CUtensorMap e[3];  // E components of the input buffer, box (WE, TJ+2, 1)
  CUtensorMap h[3];  // H components of the input buffer, box (WE, TJ+1, 1)
  CUtensorMap cls;   // class index, box (WC, TJ+1, 1)
};

template <typename T>
struct FusedTmaP {
  FusedP<T> p;
  TmaMaps m;
};

template <typename T, int TJ, int TK>
struct TmaGeom {
  static constexpr int XA = 16 / (int)sizeof(T);  // k alignment of field boxes
  static constexpr int WE = TK + 2 * XA;          // field box width
  static constexpr int RE = TJ + 2, RH = TJ + 1;  // box rows
  static constexpr int WC = TK + 16;              // class box width (uint16)
  __host__ __device__ static constexpr int pad(int b) { return (b + 127) / 128 * 128; }
  static constexpr int EB = RE * WE * (int)sizeof(T);  // bytes of one E box
  static constexpr int HB = RH * WE * (int)sizeof(T);
  static constexpr int CB = RH * WC * 2;
  static constexpr int E_OFF = 0;
  static constexpr int H_OFF = 3 * pad(EB);
  static constexpr int C_OFF = H_OFF + 3 * pad(HB);
  static constexpr int STAGE = C_OFF + pad(CB);
  static constexpr int TX_FULL = 3 * EB + 3 * HB + CB;
  static constexpr int TX_E = 3 * EB;
  static constexpr int HJ = TJ + 1, HK = TK + 1;
  static constexpr int SH_BYTES = 2 * 3 * HJ * HK * (int)sizeof(T);
  __host__ __device__ static constexpr int smem(int S) { return S * STAGE + pad(SH_BYTES) + 8 * S; }
};

template <typename T, int TJ, int TK, int S>
__global__ void __launch_bounds__(TJ* TK) k_fused_tma(const __grid_constant__ FusedTmaP<T> P) {
  using G = TmaGeom<T, TJ, TK>;
  constexpr int NT = TJ * TK;
  constexpr int HJ = G::HJ, HK = G::HK;
  extern __shared__ __align__(128) unsigned char smem[];
  T* sH = reinterpret_cast<T*>(smem + S * G::STAGE);  // [2][3][HJ*HK]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::pad(G::SH_BYTES));
  const FusedP<T>& p = P.p;
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
  const int i_lo = blockIdx.z * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const int i_first = i_lo > 0 ? i_lo - 1 : 0;
  const int n_planes = i_hi - i_first;
  const long long t = *p.step;
  // A sweep whose stage wait timed out poisons the step sequence: later
  // launches return at once instead of waiting out their own budgets.  One
  // thread reads the error word, so that the whole CTA returns or none.
  if (__syncthreads_or(tid == 0 && (*(volatile int*)p.err & 2))) return;

  auto stage_e = [&](int s, int c) {
    return reinterpret_cast<T*>(smem + s * G::STAGE + G::E_OFF + c * G::pad(G::EB));
  };
  auto stage_h = [&](int s, int c) {
    return reinterpret_cast<T*>(smem + s * G::STAGE + G::H_OFF + c * G::pad(G::HB));
  };
  auto stage_c = [&](int s) {
    return reinterpret_cast<uint16_t*>(smem + s * G::STAGE + G::C_OFF);
  };
  // Loads for plane iteration q (plane i_first+q): E(i+1), H(i), class(i).
  auto issue = [&](int q) {
    const int s = q % S;
    const int i = i_first + q;
    mbar_expect_tx(&bars[s], G::TX_FULL);
    for (int c = 0; c < 3; ++c) {
      tma_load_3d(stage_e(s, c), &P.m.e[c], k0 - G::XA, j0 - 1, i + 1, &bars[s]);
      tma_load_3d(stage_h(s, c), &P.m.h[c], k0 - G::XA, j0 - 1, i, &bars[s]);
    }
    tma_load_3d(stage_c(s), &P.m.cls, k0 - 8, j0 - 1, i, &bars[s]);
  };

  uint32_t parity = 0;    // bit s: phase to wait for on stage s
  uint32_t pending = 0;   // bit s: a load into stage s is in flight
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    // E(i_first) into the slot of iteration -1, then iterations 0 .. S-2.
    const int sp = S - 1;
    mbar_expect_tx(&bars[sp], G::TX_E);
    for (int c = 0; c < 3; ++c)
      tma_load_3d(stage_e(sp, c), &P.m.e[c], k0 - G::XA, j0 - 1, i_first, &bars[sp]);
    for (int q = 0; q < S - 1 && q < n_planes; ++q) issue(q);
  }
  pending = (1u << (S - 1));
  for (int q = 0; q < S - 1 && q < n_planes; ++q) pending |= 1u << q;

  const long long budget = 4000000000LL;  // cycles before a wait counts as failed
  bool ok = true;
  auto wait_stage = [&](int s) {
    const long long t0 = clock64();
    const uint32_t a = smem_u32(&bars[s]);
    const uint32_t ph = (parity >> s) & 1u;
    while (true) {
      uint32_t done;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          " selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(a), "r"(ph)
          : "memory");
      if (done) break;
      if (clock64() - t0 > budget) return false;
    }
    parity ^= 1u << s;
    pending &= ~(1u << s);
    return true;
  };

  if (n_planes > 0) ok = wait_stage(S - 1);  // E(i_first)
  for (int q = 0; q < n_planes; ++q) {
    const int i = i_first + q;
    const int sc = q % S, sp = (q + S - 1) % S;
    if (ok) ok = wait_stage(sc);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    const T* Ecur[3] = {stage_e(sp, 0), stage_e(sp, 1), stage_e(sp, 2)};  // E(i)
    const T* Enxt[3] = {stage_e(sc, 0), stage_e(sc, 1), stage_e(sc, 2)};  // E(i+1)
    const int hs = i & 1;
    T* sHc = sH + hs * 3 * HJ * HK;
    T* sHp = sH + (hs ^ 1) * 3 * HJ * HK;
    // ------------------------------------------------------------ H(i)
    for (int qq = tid; qq < HJ * HK; qq += NT) {
      const int jj = qq / HK, kk = qq - jj * HK;
      const int j = j0 - 1 + jj, k = k0 - 1 + kk;
      T hv[3] = {T(0), T(0), T(0)};
      if (j >= 0 && j <= L.ny && k >= 0 && k <= L.nz) {
        const long long id = lat_index(L, i, j, k);
        const bool owned = jj >= 1 && kk >= 1 && i >= i_lo;
        const bool main_rng = i < L.nx && j < L.ny && k < L.nz;
        const int eq = jj * G::WE + kk + G::XA - 1;
        const T* row = p.tab + (size_t)stage_c(sc)[jj * G::WC + kk + 7] * 12;
        auto E0 = [&](int c) { return Ecur[c][eq]; };
        auto Ep = [&](int c, int d) {
          return d == 0 ? Enxt[c][eq] : (d == 1 ? Ecur[c][eq + G::WE] : Ecur[c][eq + 1]);
        };
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int ta = (c + 1) % 3, tb = (c + 2) % 3;
          const int xc = c == 0 ? i : (c == 1 ? j : k);
          const int nc = c == 0 ? L.nx : (c == 1 ? L.ny : L.nz);
          const int xa = ta == 0 ? i : (ta == 1 ? j : k);
          const int na = ta == 0 ? L.nx : (ta == 1 ? L.ny : L.nz);
          const int xb = tb == 0 ? i : (tb == 1 ? j : k);
          const int nb = tb == 0 ? L.nx : (tb == 1 ? L.ny : L.nz);
          if (!(xc <= nc && xa < na && xb < nb)) continue;
          const T ca = row[6 + 2 * c], cb = row[7 + 2 * c];
          T h = stage_h(sc, c)[eq];
          if (main_rng) {
            const T d_a = Ep(ta, tb) - E0(ta);
            const T d_b = Ep(tb, ta) - E0(tb);
            h = ca * h + cb * (p.fh[tb][xb] * d_a - p.fh[ta][xa] * d_b);
          }
          if (p.tfh.enabled) {
            for (int s = 0; s < p.tfh.n[c]; ++s) {
              const TfsfHPass& Q = p.tfh.pass[c][s];
              if (i < Q.lo[0] || i >= Q.hi[0] || j < Q.lo[1] || j >= Q.hi[1] || k < Q.lo[2] ||
                  k >= Q.hi[2])
                continue;
              int xi[3] = {i, j, k};
              if (Q.neg) {
                if (Q.m == 0) xi[0] += 1;
                else if (Q.m == 1) xi[1] += 1;
                else xi[2] += 1;
              }
              int e_flag = 0;
              const double v = tfsf_incident(p.tf, true, Q.dual, t, xi, &e_flag);
              if (e_flag) atomicOr(p.err, 1);
              h = (T)((double)h + v * Q.coeff);
            }
          }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            if (a == c) continue;
            const SlabAxisD<T>& SA = p.slab[a];
            const int xm = a == 0 ? i : (a == 1 ? j : k);
            const int which = (c == (a + 1) % 3) ? 0 : 1;
            const int dual = which == 0 ? (a + 2) % 3 : (a + 1) % 3;
            for (int s = 0; s < SA.count; ++s) {
              const int l = xm - SA.h_lo[s];
              if (l < 0 || l >= SA.n[s]) continue;
              const T diff = Ep(dual, a) - E0(dual);
              const long long pi = psi_idx(a, SA.n[s], L, i, j, k, l);
              const T psi = SA.b_h[s][l] * SA.psi_h_in[s][which][pi] + SA.a_h[s][l] * diff;
              if (owned) SA.psi_h_out[s][which][pi] = psi;
              h += (which == 0 ? cb : -cb) * psi;
            }
          }
          hv[c] = h;
          if (owned) p.out[3 + c][id] = h;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) sHc[c * HJ * HK + qq] = hv[c];
    }
    __syncthreads();
    // ------------------------------------------------------------ E(i)
    {
      const int j = j0 + tj, k = k0 + tk;
      if (i >= i_lo && j <= L.ny && k <= L.nz) {
        const long long id = lat_index(L, i, j, k);
        const T* row = p.tab + (size_t)stage_c(sc)[(tj + 1) * G::WC + tk + 8] * 12;
        const int hq = (tj + 1) * HK + (tk + 1);
        const int eq = (tj + 1) * G::WE + tk + G::XA;
        auto H0 = [&](int c) { return sHc[c * HJ * HK + hq]; };
        auto Hm = [&](int c, int d) {
          return d == 0 ? sHp[c * HJ * HK + hq]
                        : (d == 1 ? sHc[c * HJ * HK + hq - HK] : sHc[c * HJ * HK + hq - 1]);
        };
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int ta = (c + 1) % 3, tb = (c + 2) % 3;
          const int xc = c == 0 ? i : (c == 1 ? j : k);
          const int nc = c == 0 ? L.nx : (c == 1 ? L.ny : L.nz);
          const int xa = ta == 0 ? i : (ta == 1 ? j : k);
          const int na = ta == 0 ? L.nx : (ta == 1 ? L.ny : L.nz);
          const int xb = tb == 0 ? i : (tb == 1 ? j : k);
          const int nb = tb == 0 ? L.nx : (tb == 1 ? L.ny : L.nz);
          if (!(xc < nc && xa <= na && xb <= nb)) continue;
          const bool main_rng = xa >= 1 && xa < na && xb >= 1 && xb < nb;
          const T ca = row[2 * c], cb = row[2 * c + 1];
          T e = Ecur[c][eq];
          if (main_rng) {
            const T d_a = H0(tb) - Hm(tb, ta);
            const T d_b = H0(ta) - Hm(ta, tb);
            e = ca * e + cb * (p.fe[ta][xa] * d_a - p.fe[tb][xb] * d_b);
          }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            if (a == c) continue;
            const SlabAxisD<T>& SA = p.slab[a];
            const int xm = a == 0 ? i : (a == 1 ? j : k);
            const int which = (c == (a + 1) % 3) ? 0 : 1;
            const int dual = which == 0 ? (a + 2) % 3 : (a + 1) % 3;
            for (int s = 0; s < SA.count; ++s) {
              const int l = xm - SA.e_lo[s];
              if (l < 0 || l >= SA.n[s]) continue;
              const T diff = H0(dual) - Hm(dual, a);
              T* ps = SA.psi_e[s][which] + psi_idx(a, SA.n[s], L, i, j, k, l);
              const T psi = SA.b_e[s][l] * *ps + SA.a_e[s][l] * diff;
              *ps = psi;
              e += (which == 0 ? -cb : cb) * psi;
            }
          }
          p.out[c][id] = e;
        }
      }
    }
    __syncthreads();
    // Stage sp (E(i)) is free: refill it with the loads of iteration q+S-1.
    if (tid == 0 && q + S - 1 < n_planes) {
      fence_proxy_async();
      issue(q + S - 1);
    }
    if (q + S - 1 < n_planes) pending |= 1u << sp;
  }
  if (!ok) {
    if (tid == 0) atomicOr(p.err, 2);
    // Drain the loads still in flight into this CTA's shared memory.
    for (int s = 0; s < S; ++s)
      if ((pending >> s) & 1u) wait_stage(s);
  }
}

}  // namespace xfd
