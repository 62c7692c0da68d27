// Discrete adjoint of the time step (no counterpart in the reference, which
// has no gradient path): the exact transpose of update_h_node /
// update_e_node (kernels.cuh), CPML auxiliaries included, run backward in
// time.  The forward step is affine in the state (fields, CPML psi): TFSF
// faces and lumped sources add terms that do not depend on the state, so
// they have no adjoint terms.
//
// Notation for one forward step n -> n+1 (split H then E):
//   H update, component c at node y, ta = c+1, tb = c+2 (mod 3):
//     d_a = E_ta[y + e_tb] - E_ta[y],   d_b = E_tb[y + e_ta] - E_tb[y]
//     psi' = b_h psi + a_h d   (slab along tb: d = d_a, "which" 0, sign +;
//                               slab along ta: d = d_b, "which" 1, sign -)
//     H' = [M ? ca : 1] H + cb (M fh[tb] d_a - M fh[ta] d_b) + cb (+psi'_0 - psi'_1)
//   E update, component c at node x:
//     d_a = H_tb[x] - H_tb[x - e_ta],   d_b = H_ta[x] - H_ta[x - e_tb]
//     psi' = b_e psi + a_e d   (slab along tb: d = d_b, "which" 0, sign -;
//                               slab along ta: d = d_a, "which" 1, sign +)
//     E' = [M ? ca : 1] E + cb (M fe[ta] d_a - M fe[tb] d_b) + cb (-psi'_0 + psi'_1)
// (M: the node is in the main update range.)  The adjoint variables lam
// (fields) and lam_psi (CPML) live in arrays of the forward layout.  One
// reverse step m -> m-1 is two lattice sweeps:
//   k_adj_h: per H node, lam_psi_h <- b_h (lam_psi_h + s cb lam_H);
//            lam_H <- [M ? ca : 1] lam_H + (transposed E-update differences of lam_E)
//   k_adj_e: per E node, lam_psi_e <- b_e (lam_psi_e + s cb lam_E);
//            lam_E <- [M ? ca : 1] lam_E + (transposed H-update differences of lam_H)
// where the transposed differences are gathered from the neighbour nodes
// that read this node in the forward step (no atomics).  k_adj_h fuses the
// self part of the previous reverse step's H adjoint with this step's
// gather, so both sweeps read their neighbours' values as the exact
// transpose requires.
#pragma once

#include "kernels.cuh"

namespace xfd {

__device__ __forceinline__ bool in_lattice(const Lat& L, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i <= L.nx && j <= L.ny && k <= L.nz;
}

// Per-node E coefficient overrides (OverrideD, kernels.cuh) as dense arrays
// over their bounding node box: (ca, cb) of component c at box point p in
// ca[c n + p], cb[c n + p]; cb = 0 where the node keeps its class pair.
template <typename T>
struct OvBoxD {
  int s[3], e[3];
  long long n;  // 0: no overrides
  const T* ca;
  const T* cb;
};

template <typename T>
__device__ __forceinline__ void e_coeff(const OvBoxD<T>& ov, const T* row, int c, int i, int j,
                                        int k, T& ca, T& cb) {
  ca = row[2 * c];
  cb = row[2 * c + 1];
  if (ov.n && i >= ov.s[0] && i < ov.e[0] && j >= ov.s[1] && j < ov.e[1] && k >= ov.s[2] &&
      k < ov.e[2]) {
    const long long p =
        ((long long)(i - ov.s[0]) * (ov.e[1] - ov.s[1]) + (j - ov.s[1])) * (ov.e[2] - ov.s[2]) +
        (k - ov.s[2]);
    const T b = ov.cb[c * ov.n + p];
    if (b != T(0)) {
      cb = b;
      ca = ov.ca[c * ov.n + p];
    }
  }
}

// Adjoint of one curl difference of the E update of component c at node
// (i, j, k): want_a selects d_a (else d_b).  lam fields in a.f, lam_psi_e
// in the slabs' psi_e; zero where the node is outside the lattice or the
// component outside its range.
template <typename T>
__device__ __forceinline__ T e_diff_adj(const YeeP<T>& a, const OvBoxD<T>& ov, int i, int j, int k,
                                        int c, bool want_a) {
  const Lat& L = a.L;
  if (!in_lattice(L, i, j, k)) return T(0);
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  bool valid = true, main_rng = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d == c) {
      valid = valid && (x[d] < n[d]);
    } else {
      valid = valid && (x[d] <= n[d]);
      main_rng = main_rng && (x[d] >= 1) && (x[d] < n[d]);
    }
  }
  if (!valid) return T(0);
  const long long id = lat_index(L, i, j, k);
  const T lam = a.f[c][id];
  T ca, cb;
  e_coeff(ov, a.tab + (size_t)a.cls[id] * 12, c, i, j, k, ca, cb);
  const int ta = (c + 1) % 3, tb = (c + 2) % 3;
  T v = T(0);
  if (main_rng) v = want_a ? cb * a.fe[ta][x[ta]] * lam : -cb * a.fe[tb][x[tb]] * lam;
  for (int s = 0; s < a.n_slab; ++s) {
    const SlabD<T>& sl = a.slab[s];
    if (sl.m == c) continue;
    const int which = (c == (sl.m + 1) % 3) ? 0 : 1;  // 0: d_b (slab along tb), 1: d_a
    if ((which == 1) != want_a) continue;
    const int l = x[sl.m] - sl.e_lo;
    if (l < 0 || l >= sl.n) continue;
    const T pe = sl.psi_e[which][psi_index(sl, L, i, j, k, l)] + (which == 0 ? -cb : cb) * lam;
    v += sl.a_e[l] * pe;
  }
  return v;
}

// Adjoint of one curl difference of the H update of component c at node
// (i, j, k): want_a selects d_a (else d_b).
template <typename T>
__device__ __forceinline__ T h_diff_adj(const YeeP<T>& a, int i, int j, int k, int c, bool want_a) {
  const Lat& L = a.L;
  if (!in_lattice(L, i, j, k)) return T(0);
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  bool valid = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) valid = valid && ((d == c) ? (x[d] <= n[d]) : (x[d] < n[d]));
  if (!valid) return T(0);
  const bool main_rng = (i < L.nx) && (j < L.ny) && (k < L.nz);
  const long long id = lat_index(L, i, j, k);
  const T lam = a.f[3 + c][id];
  const T cb = a.tab[(size_t)a.cls[id] * 12 + 7 + 2 * c];
  const int ta = (c + 1) % 3, tb = (c + 2) % 3;
  T v = T(0);
  if (main_rng) v = want_a ? cb * a.fh[tb][x[tb]] * lam : -cb * a.fh[ta][x[ta]] * lam;
  for (int s = 0; s < a.n_slab; ++s) {
    const SlabD<T>& sl = a.slab[s];
    if (sl.m == c) continue;
    const int which = (c == (sl.m + 1) % 3) ? 0 : 1;  // 0: d_a (slab along tb), 1: d_b
    if ((which == 0) != want_a) continue;
    const int l = x[sl.m] - sl.h_lo;
    if (l < 0 || l >= sl.n) continue;
    const T ph = sl.psi_h[which][psi_index(sl, L, i, j, k, l)] + (which == 0 ? cb : -cb) * lam;
    v += sl.a_h[l] * ph;
  }
  return v;
}

// Reverse H sweep.  For H_q at y (r1 = q+1, r2 = q+2): H_q is the d_a
// operand of E_r1 (differenced along r2) and the d_b operand of E_r2
// (differenced along r1) in the forward E update.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_h(const __grid_constant__ YeeP<T> a,
                                               const __grid_constant__ OvBoxD<T> ov) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const Lat& L = a.L;
  if (k > L.nz || j > L.ny || i > L.nx) return;
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  const long long id = lat_index(L, i, j, k);
  const T* row = a.tab + (size_t)a.cls[id] * 12;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    bool valid = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) valid = valid && ((d == q) ? (x[d] <= n[d]) : (x[d] < n[d]));
    if (!valid) continue;
    T* Lq = a.f[3 + q];
    const T lam = Lq[id];
    const T ca = row[6 + 2 * q], cb = row[7 + 2 * q];
    for (int s = 0; s < a.n_slab; ++s) {
      const SlabD<T>& sl = a.slab[s];
      if (sl.m == q) continue;
      const int l = x[sl.m] - sl.h_lo;
      if (l < 0 || l >= sl.n) continue;
      const int which = (q == (sl.m + 1) % 3) ? 0 : 1;
      T* ps = sl.psi_h[which] + psi_index(sl, L, i, j, k, l);
      *ps = sl.b_h[l] * (*ps + (which == 0 ? cb : -cb) * lam);
    }
    const int r1 = (q + 1) % 3, r2 = (q + 2) % 3;
    int y1[3] = {i, j, k}, y2[3] = {i, j, k};
    y1[r2] += 1;  // the E_r1 node that reads H_q[y] as H_q[x - e_r2]
    y2[r1] += 1;  // the E_r2 node that reads H_q[y] as H_q[x - e_r1]
    const bool main_rng = (i < L.nx) && (j < L.ny) && (k < L.nz);
    T v = main_rng ? ca * lam : lam;
    v += e_diff_adj(a, ov, i, j, k, r1, true) - e_diff_adj(a, ov, y1[0], y1[1], y1[2], r1, true);
    v += e_diff_adj(a, ov, i, j, k, r2, false) - e_diff_adj(a, ov, y2[0], y2[1], y2[2], r2, false);
    Lq[id] = v;
  }
}

// Reverse E sweep.  For E_q at x (r1 = q+1, r2 = q+2): E_q is the d_a
// operand of H_r2 (differenced along r1) and the d_b operand of H_r1
// (differenced along r2) in the forward H update.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_e(const __grid_constant__ YeeP<T> a,
                                               const __grid_constant__ OvBoxD<T> ov) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  const Lat& L = a.L;
  if (k > L.nz || j > L.ny || i > L.nx) return;
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  const long long id = lat_index(L, i, j, k);
  const T* row = a.tab + (size_t)a.cls[id] * 12;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    bool valid = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) valid = valid && ((d == q) ? (x[d] < n[d]) : (x[d] <= n[d]));
    if (!valid) continue;
    T* Lq = a.f[q];
    const T lam = Lq[id];
    T ca, cb;
    e_coeff(ov, row, q, i, j, k, ca, cb);
    for (int s = 0; s < a.n_slab; ++s) {
      const SlabD<T>& sl = a.slab[s];
      if (sl.m == q) continue;
      const int l = x[sl.m] - sl.e_lo;
      if (l < 0 || l >= sl.n) continue;
      const int which = (q == (sl.m + 1) % 3) ? 0 : 1;
      T* ps = sl.psi_e[which] + psi_index(sl, L, i, j, k, l);
      *ps = sl.b_e[l] * (*ps + (which == 0 ? -cb : cb) * lam);
    }
    const int r1 = (q + 1) % 3, r2 = (q + 2) % 3;
    int y1[3] = {i, j, k}, y2[3] = {i, j, k};
    y1[r1] -= 1;  // the H_r2 node that reads E_q[x] as E_q[y + e_r1]
    y2[r2] -= 1;  // the H_r1 node that reads E_q[x] as E_q[y + e_r2]
    const bool main_rng = x[r1] >= 1 && x[r1] < n[r1] && x[r2] >= 1 && x[r2] < n[r2];
    T v = main_rng ? ca * lam : lam;
    v += h_diff_adj(a, y1[0], y1[1], y1[2], r2, true) - h_diff_adj(a, i, j, k, r2, true);
    v += h_diff_adj(a, y2[0], y2[1], y2[2], r1, false) - h_diff_adj(a, i, j, k, r1, false);
    Lq[id] = v;
  }
}

// A node box of the lattice and some of its field components, copied into
// row (step - base + shift) of a rows x nc x n array; rows outside [0, rows)
// are skipped.
template <typename T>
struct BoxRecD {
  int s[3], e[3];
  int c0, nc;
  long long n;
  long long base;
  int shift;
  long long rows;
  T* dst;
};

__device__ __forceinline__ void box_node(const int s[3], const int e[3], long long p, int& i,
                                         int& j, int& k) {
  const int e2 = e[2] - s[2], e1 = e[1] - s[1];
  k = s[2] + (int)(p % e2);
  p /= e2;
  j = s[1] + (int)(p % e1);
  i = s[0] + (int)(p / e1);
}

template <typename T>
__global__ void k_box_record(BoxRecD<T> r, Lat L, T* const* fields, const long long* step) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= r.n * r.nc) return;
  const long long row = *step - r.base + r.shift;
  if (row < 0 || row >= r.rows) return;
  const int cc = (int)(q / r.n);
  const long long p = q - (long long)cc * r.n;
  int i, j, k;
  box_node(r.s, r.e, p, i, j, k);
  r.dst[(row * r.nc + cc) * r.n + p] = fields[r.c0 + cc][lat_index(L, i, j, k)];
}

// Sensitivity sums over the design box: for E component c at node x,
// G0 += lam_c(x) E_c^{m-1}(x) and G1 += lam_c(x) E_c^m(x), with E^{m-1},
// E^m rows slot-1, slot of the recorded history (3 x n per row), in FP64.
template <typename T>
__global__ void k_adj_sens(BoxRecD<T> r, Lat L, T* const* lam, const T* hist, int slot,
                           double* g0, double* g1) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= r.n * 3) return;
  const int c = (int)(q / r.n);
  const long long p = q - (long long)c * r.n;
  int i, j, k;
  box_node(r.s, r.e, p, i, j, k);
  const double l = (double)lam[c][lat_index(L, i, j, k)];
  g0[q] += l * (double)hist[((long long)(slot - 1) * 3 + c) * r.n + p];
  g1[q] += l * (double)hist[((long long)slot * 3 + c) * r.n + p];
}

// Adjoint source: lam_c(x) += d[p] over the objective box (one component).
template <typename T>
__global__ void k_adj_source(BoxRecD<T> r, Lat L, T* const* lam, const double* d) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= r.n) return;
  int i, j, k;
  box_node(r.s, r.e, p, i, j, k);
  T* f = lam[r.c0];
  const long long id = lat_index(L, i, j, k);
  f[id] = (T)((double)f[id] + d[p]);
}

}  // namespace xfd
