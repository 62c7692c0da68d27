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
// (M: the node is in the main update range.)  One reverse step m -> m-1,
// on adjoint variables lam (fields) and lam_psi (CPML) in arrays of the
// forward layout, is two lattice sweeps:
//   H: lam_psi_h <- b_h (lam_psi_h + s cb lam_H)  (the previous step's H part);
//      lam_H <- [M ? ca : 1] lam_H + (transposed E-update differences of lam_E)
//   E: lam_psi_e <- b_e (lam_psi_e + s cb lam_E);
//      lam_E <- [M ? ca : 1] lam_E + (transposed H-update differences of lam_H)
// where the transposed differences are gathered from the neighbour nodes
// that read this node in the forward step (no atomics), each sweep reading
// its neighbours' values before the other sweep changes them, as the exact
// transpose requires.  The fields are held scaled, u = cb lam_E and
// w = -cb lam_H: in those variables the reverse step is node for node the
// forward step with the same (ca, cb), so on a box with no CPML and one curl
// factor per axis the forward marching sweeps (march_tma.cuh) run it
// unchanged, and the gather kernels here (k_adj_h, k_adj_e) do the exact
// transpose on the shell around that box, without class lookups at
// neighbour nodes.
#pragma once

#include "fused.cuh"
#include "kernels.cuh"
#include "march.cuh"

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

// The reverse pass runs on scaled adjoint fields u_c = cb_c lam_E,c (E
// nodes) and w_c = -cb_c lam_H,c (H nodes), with (ca, cb) the node's class
// pair.  Written in u and w the reverse step is, node for node, the forward
// step with the same (ca, cb): on a CPML-free box with uniform curl factors
// (the transposed differences weigh the source node, the forward ones the
// destination) the forward marching sweeps run it unchanged, and the gather
// kernels below do the exact transpose on the rest of the lattice.  The CPML
// adjoints lam_psi stay unscaled.
//
// Index of a psi cell of the slab in slot q along axis AX (layer l).
template <typename T, int AX>
__device__ __forceinline__ long long psi_at(const MarchP<T>& p, int q, int i, int j, int k, int l) {
  const Lat& L = p.L;
  if (AX == 0) return ((long long)l * L.NY + j) * L.KP + k;
  if (AX == 1) return ((long long)i * p.slab[1].n[q] + l) * L.KP + k;
  return ((long long)i * L.NY + j) * p.slab[2].n[q] + l;
}

// X terms (adjoint of one difference of the E update of component C at node
// (i, j, k); zero outside the lattice or the component's range):
//   X_a = M fe[ta][x_ta] u + a_e (lam_psi + u)    (d_a: slab along ta)
//   X_b = -M fe[tb][x_tb] u + a_e (lam_psi - u)   (d_b: slab along tb)
template <typename T, int C, bool WANT_A>
__device__ __forceinline__ T x_term(const MarchP<T>& p, int i, int j, int k) {
  constexpr int TA = (C + 1) % 3, TB = (C + 2) % 3, AX = WANT_A ? TA : TB;
  constexpr int W = (C == (AX + 1) % 3) ? 0 : 1;  // psi component slot of C in that slab
  const Lat& L = p.L;
  if (i < 0 || j < 0 || k < 0 || i > L.nx || j > L.ny || k > L.nz) return T(0);
  if (pick<C>(i, j, k) >= pick<C>(L.nx, L.ny, L.nz)) return T(0);
  const int xa = pick<TA>(i, j, k), xb = pick<TB>(i, j, k);
  const bool main_rng = xa >= 1 && xa < pick<TA>(L.nx, L.ny, L.nz) && xb >= 1 &&
                        xb < pick<TB>(L.nx, L.ny, L.nz);
  const T u = p.f[C][lat_index(L, i, j, k)];
  T v = main_rng ? (WANT_A ? p.fe[TA][xa] * u : -p.fe[TB][xb] * u) : T(0);
  int q;
  const int l = layer_of(p.slab[AX], pick<AX>(i, j, k), true, q);
  if (l >= 0) {
    const SlabAxisD<T>& A = p.slab[AX];
    v += A.a_e[q][l] * (A.psi_e[q][W][psi_at<T, AX>(p, q, i, j, k, l)] + (WANT_A ? u : -u));
  }
  return v;
}

// Y terms (adjoint of one difference of the H update of component C at y):
//   Y_a = -M fh[tb][y_tb] w + a_h (lam_psi - w)   (d_a: slab along tb)
//   Y_b = M fh[ta][y_ta] w + a_h (lam_psi + w)    (d_b: slab along ta)
template <typename T, int C, bool WANT_A>
__device__ __forceinline__ T y_term(const MarchP<T>& p, int i, int j, int k) {
  constexpr int TA = (C + 1) % 3, TB = (C + 2) % 3, AX = WANT_A ? TB : TA;
  constexpr int W = (C == (AX + 1) % 3) ? 0 : 1;
  const Lat& L = p.L;
  if (i < 0 || j < 0 || k < 0 || i > L.nx || j > L.ny || k > L.nz) return T(0);
  const int xa = pick<TA>(i, j, k), xb = pick<TB>(i, j, k);
  if (xa >= pick<TA>(L.nx, L.ny, L.nz) || xb >= pick<TB>(L.nx, L.ny, L.nz)) return T(0);
  const bool main_rng = pick<C>(i, j, k) < pick<C>(L.nx, L.ny, L.nz);
  const T w = p.f[3 + C][lat_index(L, i, j, k)];
  T v = main_rng ? (WANT_A ? -p.fh[TB][xb] * w : p.fh[TA][xa] * w) : T(0);
  int q;
  const int l = layer_of(p.slab[AX], pick<AX>(i, j, k), false, q);
  if (l >= 0) {
    const SlabAxisD<T>& A = p.slab[AX];
    v += A.a_h[q][l] * (A.psi_h_out[q][W][psi_at<T, AX>(p, q, i, j, k, l)] + (WANT_A ? -w : w));
  }
  return v;
}

// Node box swept by the forward marching kernels on the scaled fields (k,
// j, i ranges [lo, hi)); the gather kernels skip it.  The gather grid starts
// at node (org_k, org_j) (<= 0) so that its 32 x 8 CTAs line up with the
// box's tiles: a CTA lies wholly inside the box or wholly outside.
struct AdjBox {
  int lo[3], hi[3];
  int org_k, org_j;
};

__device__ __forceinline__ bool in_adj_box(const AdjBox& b, int i, int j, int k) {
  return k >= b.lo[0] && k < b.hi[0] && j >= b.lo[1] && j < b.hi[1] && i >= b.lo[2] &&
         i < b.hi[2];
}

// The whole CTA of a gather kernel (32 x 8 nodes of plane i) in the box.
__device__ __forceinline__ bool cta_in_adj_box(const AdjBox& b) {
  const int k0 = b.org_k + blockIdx.x * blockDim.x, j0 = b.org_j + blockIdx.y * blockDim.y;
  return in_adj_box(b, blockIdx.z, j0, k0) &&
         in_adj_box(b, blockIdx.z, j0 + blockDim.y - 1, k0 + blockDim.x - 1);
}

// Psi adjoint of component Q in the slab along axis M at node (i, j, k):
// lam_psi <- b (lam_psi + s v), s = -1 for the slab's first component.
template <typename T, int Q, int M, bool E>
__device__ __forceinline__ void psi_adj(const MarchP<T>& p, int i, int j, int k, T v) {
  constexpr int W = (Q == (M + 1) % 3) ? 0 : 1;
  int q;
  const int l = layer_of(p.slab[M], pick<M>(i, j, k), E, q);
  if (l < 0) return;
  const SlabAxisD<T>& A = p.slab[M];
  T* ps = (E ? A.psi_e[q][W] : A.psi_h_out[q][W]) + psi_at<T, M>(p, q, i, j, k, l);
  *ps = (E ? A.b_e[q][l] : A.b_h[q][l]) * (*ps + (W == 0 ? -v : v));
}

// H_Q at y (R1 = Q+1, R2 = Q+2) is the d_a operand of E_R1 (differenced
// along R2) and the d_b operand of E_R2 (differenced along R1) in the forward
// E update.  The gather (loads only) is split from the update (stores), so
// that a node's three components read before any of them is written.
template <typename T, int Q>
__device__ __forceinline__ bool adj_h_gather(const MarchP<T>& p, int i, int j, int k, long long id,
                                             T& w, T& sum) {
  constexpr int R1 = (Q + 1) % 3, R2 = (Q + 2) % 3;
  const Lat& L = p.L;
  if (pick<R1>(i, j, k) >= pick<R1>(L.nx, L.ny, L.nz) ||
      pick<R2>(i, j, k) >= pick<R2>(L.nx, L.ny, L.nz))
    return false;  // H_Q out of range
  w = p.f[3 + Q][id];
  sum = x_term<T, R1, true>(p, i, j, k) -
        x_term<T, R1, true>(p, i + (R2 == 0), j + (R2 == 1), k + (R2 == 2)) +
        x_term<T, R2, false>(p, i, j, k) -
        x_term<T, R2, false>(p, i + (R1 == 0), j + (R1 == 1), k + (R1 == 2));
  return true;
}

// Completes the previous reverse step's H adjoint (psi) and writes H_Q.
template <typename T, int Q>
__device__ __forceinline__ void adj_h_update(const MarchP<T>& p, const T* row, int i, int j, int k,
                                             long long id, bool main_rng, T w, T sum) {
  constexpr int R1 = (Q + 1) % 3, R2 = (Q + 2) % 3;
  psi_adj<T, Q, R1, false>(p, i, j, k, w);
  psi_adj<T, Q, R2, false>(p, i, j, k, w);
  p.f[3 + Q][id] = (main_rng ? row[6 + 2 * Q] * w : w) - row[7 + 2 * Q] * sum;
}

// E_Q at x (R1 = Q+1, R2 = Q+2) is the d_a operand of H_R2 (differenced
// along R1) and the d_b operand of H_R1 (differenced along R2) in the forward
// H update.  Nodes with a coefficient override take the class pair here and
// the override fix-up afterwards, as in the forward step.
template <typename T, int Q>
__device__ __forceinline__ bool adj_e_gather(const MarchP<T>& p, int i, int j, int k, long long id,
                                             T& u, T& sum) {
  constexpr int R1 = (Q + 1) % 3, R2 = (Q + 2) % 3;
  const Lat& L = p.L;
  if (pick<Q>(i, j, k) >= pick<Q>(L.nx, L.ny, L.nz)) return false;  // E_Q out of range
  u = p.f[Q][id];
  sum = y_term<T, R2, true>(p, i - (R1 == 0), j - (R1 == 1), k - (R1 == 2)) -
        y_term<T, R2, true>(p, i, j, k) +
        y_term<T, R1, false>(p, i - (R2 == 0), j - (R2 == 1), k - (R2 == 2)) -
        y_term<T, R1, false>(p, i, j, k);
  return true;
}

template <typename T, int Q>
__device__ __forceinline__ void adj_e_update(const MarchP<T>& p, const T* row, int i, int j, int k,
                                             long long id, T u, T sum) {
  constexpr int R1 = (Q + 1) % 3, R2 = (Q + 2) % 3;
  const Lat& L = p.L;
  psi_adj<T, Q, R1, true>(p, i, j, k, u);
  psi_adj<T, Q, R2, true>(p, i, j, k, u);
  const int x1 = pick<R1>(i, j, k), x2 = pick<R2>(i, j, k);
  const bool main_rng = x1 >= 1 && x1 < pick<R1>(L.nx, L.ny, L.nz) && x2 >= 1 &&
                        x2 < pick<R2>(L.nx, L.ny, L.nz);
  p.f[Q][id] = (main_rng ? row[2 * Q] * u : u) + row[2 * Q + 1] * sum;
}

// Reverse H sweep outside the box (one thread per node).
template <typename T>
__global__ void __launch_bounds__(256) k_adj_h(const __grid_constant__ MarchP<T> p,
                                               const __grid_constant__ AdjBox box) {
  if (cta_in_adj_box(box)) return;
  const int k = box.org_k + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = box.org_j + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int i = blockIdx.z;
  const Lat& L = p.L;
  if (k < 0 || j < 0 || k > L.nz || j > L.ny || i > L.nx || in_adj_box(box, i, j, k)) return;
  const long long id = lat_index(L, i, j, k);
  const T* row = p.tab + (size_t)p.cls[id] * 12;
  const bool main_rng = (i < L.nx) && (j < L.ny) && (k < L.nz);
  T w0, w1, w2, s0, s1, s2;
  const bool v0 = adj_h_gather<T, 0>(p, i, j, k, id, w0, s0);
  const bool v1 = adj_h_gather<T, 1>(p, i, j, k, id, w1, s1);
  const bool v2 = adj_h_gather<T, 2>(p, i, j, k, id, w2, s2);
  if (v0) adj_h_update<T, 0>(p, row, i, j, k, id, main_rng, w0, s0);
  if (v1) adj_h_update<T, 1>(p, row, i, j, k, id, main_rng, w1, s1);
  if (v2) adj_h_update<T, 2>(p, row, i, j, k, id, main_rng, w2, s2);
}

// Reverse E sweep outside the box (one thread per node).
template <typename T>
__global__ void __launch_bounds__(256) k_adj_e(const __grid_constant__ MarchP<T> p,
                                               const __grid_constant__ AdjBox box) {
  if (cta_in_adj_box(box)) return;
  const int k = box.org_k + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = box.org_j + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int i = blockIdx.z;
  const Lat& L = p.L;
  if (k < 0 || j < 0 || k > L.nz || j > L.ny || i > L.nx || in_adj_box(box, i, j, k)) return;
  const long long id = lat_index(L, i, j, k);
  const T* row = p.tab + (size_t)p.cls[id] * 12;
  T u0, u1, u2, s0, s1, s2;
  const bool v0 = adj_e_gather<T, 0>(p, i, j, k, id, u0, s0);
  const bool v1 = adj_e_gather<T, 1>(p, i, j, k, id, u1, s1);
  const bool v2 = adj_e_gather<T, 2>(p, i, j, k, id, u2, s2);
  if (v0) adj_e_update<T, 0>(p, row, i, j, k, id, u0, s0);
  if (v1) adj_e_update<T, 1>(p, row, i, j, k, id, u1, s1);
  if (v2) adj_e_update<T, 2>(p, row, i, j, k, id, u2, s2);
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
// G0 += lam_c(x) E_c^{m-1}(x) and G1 += lam_c(x) E_c^m(x), lam = u / cb with
// the node's own cb (override or class), E^{m-1}, E^m rows slot-1, slot of
// the recorded history (3 x n per row), in FP64.
template <typename T>
__global__ void k_adj_sens(BoxRecD<T> r, YeeP<T> a, OvBoxD<T> ov, const T* hist, int slot,
                           double* g0, double* g1) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= r.n * 3) return;
  const int c = (int)(q / r.n);
  const long long p = q - (long long)c * r.n;
  int i, j, k;
  box_node(r.s, r.e, p, i, j, k);
  const int x[3] = {i, j, k};
  const int nn[3] = {a.L.nx, a.L.ny, a.L.nz};
  if (x[c] >= nn[c]) return;  // component out of range
  const long long id = lat_index(a.L, i, j, k);
  T ca, cb;
  e_coeff(ov, a.tab + (size_t)a.cls[id] * 12, c, i, j, k, ca, cb);
  const double l = (double)a.f[c][id] / (double)cb;
  g0[q] += l * (double)hist[((long long)(slot - 1) * 3 + c) * r.n + p];
  g1[q] += l * (double)hist[((long long)slot * 3 + c) * r.n + p];
}

// Adjoint source: u_c(x) += cb(x) d[p] over the objective box (one
// component), cb the node's own (override or class).
template <typename T>
__global__ void k_adj_source(BoxRecD<T> r, YeeP<T> a, OvBoxD<T> ov, const double* d) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= r.n) return;
  int i, j, k;
  box_node(r.s, r.e, p, i, j, k);
  const long long id = lat_index(a.L, i, j, k);
  T ca, cb;
  e_coeff(ov, a.tab + (size_t)a.cls[id] * 12, r.c0, i, j, k, ca, cb);
  T* f = a.f[r.c0];
  f[id] = (T)((double)f[id] + (double)cb * d[p]);
}

}  // namespace xfd
