// Fused H-then-E sweep: one kernel per time step for the Yee update, the CPML
// auxiliaries of both phases and the TFSF H-face corrections.
//
// Fields ping-pong between two buffers: the sweep reads E^n, H^{n-1/2} from
// `in` and writes E^{n+1}, H^{n+1/2} to `out`, so no CTA ever reads a value a
// neighbouring CTA has already advanced.  Each CTA owns a (TJ x TK) tile of
// the (j, k) plane and marches along i over a chunk of IC planes.  Per plane
// it stages E^n of plane i+1 (tile plus a one-node halo) in shared memory,
// computes H^{n+1/2} on the tile plus its low j/k halo (the halo nodes belong
// to the neighbouring tiles and are recomputed, identically, because the E
// update needs them), then the E^{n+1} of the tile from the staged H of
// planes i and i-1.  A chunk starts one plane early to rebuild H of plane
// i_lo-1.  Compulsory DRAM traffic per node: 6 field reads, 6 writes and the
// uint16 class index, plus the CPML psi in the slabs.
//
// CPML (PMLCorrector<xyz>::correctH/correctE, src/include/boundary/pml_corrector.h:178-382):
// H psi ping-pong with the fields (halo recomputation reads the old psi);
// E psi is updated in place (only the owning thread touches it).
// TFSF H faces (TFSF3DCorrector::correctH, src/waveform_source/tfsf_corrector.cpp:205-232)
// are applied to every H node the sweep computes, in the reference pass
// order, before the CPML term, as in Domain::run's correctH.
#pragma once

#include "kernels.cuh"

namespace xfd {

// CPML slabs normal to one axis (at most one on each side).
template <typename T>
struct SlabAxisD {
  int count;
  int n[2], e_lo[2], h_lo[2];
  const T* a_e[2];
  const T* b_e[2];
  const T* a_h[2];
  const T* b_h[2];
  T* psi_e[2][2];            // [slab][component A=(m+1)%3 / B=(m+2)%3]
  const T* psi_h_in[2][2];
  T* psi_h_out[2][2];
};

// TFSF H-face passes of one H component, in the reference's order.
struct TfsfHPass {
  int m, neg, dual;
  int lo[3], hi[3];  // field nodes corrected by the pass
  double coeff;
};

struct TfsfHD {
  int enabled;
  int n[3];
  TfsfHPass pass[3][4];
};

template <typename T>
struct FusedP {
  Lat L;
  const T* in[6];
  T* out[6];
  const uint16_t* cls;
  const T* tab;
  int n_classes;
  const T* fe[3];
  const T* fh[3];
  SlabAxisD<T> slab[3];
  TfsfD tf;
  TfsfHD tfh;
  int ichunk;
  const long long* step;
  int* err;
};

template <int A>
__device__ __forceinline__ int pick(int i, int j, int k) {
  return A == 0 ? i : (A == 1 ? j : k);
}

__device__ __forceinline__ long long psi_idx(int m, int n, const Lat& L, int i, int j, int k,
                                             int l) {
  if (m == 0) return ((long long)l * L.NY + j) * L.KP + k;
  if (m == 1) return ((long long)i * n + l) * L.KP + k;
  return ((long long)i * L.NY + j) * n + l;
}

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__(TJ* TK) k_fused(const __grid_constant__ FusedP<T> p) {
  constexpr int EJ = TJ + 2, EK = TK + 2;  // staged E: j0-1 .. j0+TJ, k0-1 .. k0+TK
  constexpr int HJ = TJ + 1, HK = TK + 1;  // staged H: j0-1 .. j0+TJ-1, k0-1 .. k0+TK-1
  constexpr int NT = TJ * TK;
  __shared__ T sE[2][3][EJ * EK];
  __shared__ T sH[2][3][HJ * HK];
  const Lat L = p.L;
  const int tk = threadIdx.x, tj = threadIdx.y, tid = tj * TK + tk;
  const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
  const int i_lo = blockIdx.z * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const int i_first = i_lo > 0 ? i_lo - 1 : 0;
  const long long t = *p.step;
  const long long sti = (long long)L.NY * L.KP;

  auto load_e = [&](int i, int slot) {
    for (int q = tid; q < EJ * EK; q += NT) {
      const int jj = q / EK, kk = q - jj * EK;
      const int j = j0 - 1 + jj, k = k0 - 1 + kk;
      const bool ok = i <= L.nx && j >= 0 && j <= L.ny && k >= 0 && k <= L.nz;
      const long long id = ok ? lat_index(L, i, j, k) : 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) sE[slot][c][q] = ok ? p.in[c][id] : T(0);
    }
  };

  load_e(i_first, i_first & 1);
  for (int i = i_first; i < i_hi; ++i) {
    const int s0 = i & 1, s1 = s0 ^ 1;
    load_e(i + 1, s1);
    __syncthreads();
    // ------------------------------------------------------------ H(i)
    for (int q = tid; q < HJ * HK; q += NT) {
      const int jj = q / HK, kk = q - jj * HK;
      const int j = j0 - 1 + jj, k = k0 - 1 + kk;
      T hv[3] = {T(0), T(0), T(0)};
      if (j >= 0 && j <= L.ny && k >= 0 && k <= L.nz) {
        const long long id = lat_index(L, i, j, k);
        const bool owned = jj >= 1 && kk >= 1 && i >= i_lo;
        const bool main_rng = i < L.nx && j < L.ny && k < L.nz;
        const T* row = p.tab + (size_t)p.cls[id] * 12;
        const int eq = jj * EK + kk;  // this node in the staged E plane
        // E_c(x + e_d): d = x -> other slot, y -> +EK, z -> +1
        auto E0 = [&](int c) { return sE[s0][c][eq]; };
        auto Ep = [&](int c, int d) {
          return d == 0 ? sE[s1][c][eq] : (d == 1 ? sE[s0][c][eq + EK] : sE[s0][c][eq + 1]);
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
          T h = p.in[3 + c][id];
          if (main_rng) {
            const T d_a = Ep(ta, tb) - E0(ta);
            const T d_b = Ep(tb, ta) - E0(tb);
            h = ca * h + cb * (p.fh[tb][xb] * d_a - p.fh[ta][xa] * d_b);
          }
          if (p.tfh.enabled) {
            for (int s = 0; s < p.tfh.n[c]; ++s) {
              const TfsfHPass& P = p.tfh.pass[c][s];
              if (i < P.lo[0] || i >= P.hi[0] || j < P.lo[1] || j >= P.hi[1] || k < P.lo[2] ||
                  k >= P.hi[2])
                continue;
              int xi[3] = {i, j, k};
              if (P.neg) {
                if (P.m == 0) xi[0] += 1;
                else if (P.m == 1) xi[1] += 1;
                else xi[2] += 1;
              }
              int e_flag = 0;
              const double v = tfsf_incident(p.tf, true, P.dual, t, xi, &e_flag);
              if (e_flag) atomicOr(p.err, 1);
              h = (T)((double)h + v * P.coeff);
            }
          }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            if (a == c) continue;
            const SlabAxisD<T>& S = p.slab[a];
            const int xm = a == 0 ? i : (a == 1 ? j : k);
            const int which = (c == (a + 1) % 3) ? 0 : 1;
            const int dual = which == 0 ? (a + 2) % 3 : (a + 1) % 3;
            for (int s = 0; s < S.count; ++s) {
              const int l = xm - S.h_lo[s];
              if (l < 0 || l >= S.n[s]) continue;
              const T diff = Ep(dual, a) - E0(dual);
              const long long pi = psi_idx(a, S.n[s], L, i, j, k, l);
              const T psi = S.b_h[s][l] * S.psi_h_in[s][which][pi] + S.a_h[s][l] * diff;
              if (owned) S.psi_h_out[s][which][pi] = psi;
              h += (which == 0 ? cb : -cb) * psi;
            }
          }
          hv[c] = h;
          if (owned) p.out[3 + c][id] = h;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) sH[s0][c][q] = hv[c];
    }
    __syncthreads();
    // ------------------------------------------------------------ E(i)
    const int j = j0 + tj, k = k0 + tk;
    if (i >= i_lo && j <= L.ny && k <= L.nz) {
      const long long id = lat_index(L, i, j, k);
      const T* row = p.tab + (size_t)p.cls[id] * 12;
      const int hq = (tj + 1) * HK + (tk + 1);  // this node in the staged H plane
      const int eq = (tj + 1) * EK + (tk + 1);
      auto H0 = [&](int c) { return sH[s0][c][hq]; };
      auto Hm = [&](int c, int d) {  // H_c(x - e_d)
        return d == 0 ? sH[s1][c][hq] : (d == 1 ? sH[s0][c][hq - HK] : sH[s0][c][hq - 1]);
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
        T e = sE[s0][c][eq];
        if (main_rng) {
          const T d_a = H0(tb) - Hm(tb, ta);
          const T d_b = H0(ta) - Hm(ta, tb);
          e = ca * e + cb * (p.fe[ta][xa] * d_a - p.fe[tb][xb] * d_b);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          if (a == c) continue;
          const SlabAxisD<T>& S = p.slab[a];
          const int xm = a == 0 ? i : (a == 1 ? j : k);
          const int which = (c == (a + 1) % 3) ? 0 : 1;
          const int dual = which == 0 ? (a + 2) % 3 : (a + 1) % 3;
          for (int s = 0; s < S.count; ++s) {
            const int l = xm - S.e_lo[s];
            if (l < 0 || l >= S.n[s]) continue;
            const T diff = H0(dual) - Hm(dual, a);
            T* ps = S.psi_e[s][which] + psi_idx(a, S.n[s], L, i, j, k, l);
            const T psi = S.b_e[s][l] * *ps + S.a_e[s][l] * diff;
            *ps = psi;
            e += (which == 0 ? -cb : cb) * psi;
          }
        }
        p.out[c][id] = e;
      }
    }
    __syncthreads();
  }
  (void)sti;
}

}  // namespace xfd
