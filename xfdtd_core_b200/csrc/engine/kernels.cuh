// Device kernels of the B200 FDTD engine.
//
// Data layout: every field component, the uint16 material-class index and the
// per-slab CPML psi arrays are stored on the (nx+1) x (ny+1) x (nz+1) node
// lattice, k fastest, with rows padded to a pitch KP (a multiple of 32
// elements) so that a warp of 32 consecutive k reads whole 128 B (FP32) or
// 256 B (FP64) lines.  A component that is shorter than the lattice along an
// axis (Ex has nx entries along x, ...) leaves the last plane unused.
//
// The update of component c reads its (ca, cb) pair from the class table
// row of its node and the per-axis curl factors fe/fh, which fold in the cell
// size and the CPML kappa:
//   E_c = ca E_c + cb (fe_a (H_b - H_b[x_a-1]) - fe_b (H_a - H_a[x_b-1]))
//   H_c = ca H_c + cb (fh_b (E_a[x_b+1] - E_a) - fh_a (E_b[x_a+1] - E_b))
// with a = (c+1)%3, b = (c+2)%3 -- the structure of eNext/hNext in the
// reference (src/include/updator/update_scheme.h:26-62) with its coefficient
// arrays factored into class x axis terms.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace xfd {

// Programmatic dependent launch (small lattices, option "pdl"): a kernel
// launched with programmatic stream serialization may start while the kernel
// before it still runs; griddepcontrol.wait blocks until that kernel has
// finished and its writes are visible, and launch_dependents lets the next
// kernel start launching in turn.  In a kernel launched without the
// attribute both are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}


struct Lat {
  int nx, ny, nz;
  int NY;  // ny + 1
  int KP;  // k pitch
};

__host__ __device__ __forceinline__ long long lat_index(const Lat& L, int i, int j, int k) {
  return ((long long)i * L.NY + j) * L.KP + k;
}

// One CPML slab.  psi[0] belongs to the slab's tangential component A =
// (m+1)%3, psi[1] to B = (m+2)%3.  Layer l of the slab is coordinate
// lo + l along m.  psi layout: m=0 -> [l][j][k] (pitch NY*KP, KP),
// m=1 -> [i][l][k] (pitch n*KP, KP), m=2 -> [i][j][l] (pitch NY*n, n).
template <typename T>
struct SlabD {
  int m, n, e_lo, h_lo;
  const T* a_e;
  const T* b_e;
  const T* a_h;
  const T* b_h;
  T* psi_e[2];
  T* psi_h[2];
};

template <typename T>
__device__ __forceinline__ long long psi_index(const SlabD<T>& s, const Lat& L, int i, int j,
                                               int k, int l) {
  if (s.m == 0) return ((long long)l * L.NY + j) * L.KP + k;
  if (s.m == 1) return ((long long)i * s.n + l) * L.KP + k;
  return ((long long)i * L.NY + j) * s.n + l;
}

template <typename T>
struct YeeP {
  Lat L;
  T* f[6];  // Ex Ey Ez Hx Hy Hz
  const uint16_t* cls;
  const T* tab;  // n_classes x 12: (ca, cb) of Ex Ey Ez Hx Hy Hz
  const T* fe[3];
  const T* fh[3];
  int n_slab;
  SlabD<T> slab[6];
};

// ---------------------------------------------------------------------------
// H sweep.  One thread per lattice node (i, j, k); each handles Hx, Hy, Hz.
// Main update over i<nx, j<ny, k<nz (BasicUpdator::updateH,
// src/updator/basic_updator.cpp:23-36), then the CPML correction of every
// slab whose H layers contain the node (PMLCorrector<xyz>::correctH,
// src/include/boundary/pml_corrector.h:290-382) over the component's whole
// transverse extent, in slab insertion order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sel3(int m, int a, int b, int c) {
  return m == 0 ? a : (m == 1 ? b : c);
}
__device__ __forceinline__ long long sel3(int m, long long a, long long b, long long c) {
  return m == 0 ? a : (m == 1 ? b : c);
}

// `rd` (ping-pong sweeps): the buffer holding the old fields, read for the
// node's own value and its E neighbours; the result goes to p.f.  Null: in
// place.
template <typename T>
__device__ __forceinline__ void update_h_node(const YeeP<T>& p, int i, int j, int k,
                                              T* const* rd = nullptr) {
  const Lat L = p.L;
  const long long id = lat_index(L, i, j, k);
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  const long long st[3] = {(long long)L.NY * L.KP, (long long)L.KP, 1};
  const bool main_rng = (i < L.nx) && (j < L.ny) && (k < L.nz);
  const T* row = p.tab + (size_t)p.cls[id] * 12;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    bool valid = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) valid = valid && ((d == c) ? (x[d] <= n[d]) : (x[d] < n[d]));
    if (!valid) continue;
    const int ta = (c + 1) % 3, tb = (c + 2) % 3;
    T* H = p.f[3 + c];
    const T ca = row[6 + 2 * c];
    const T cb = row[7 + 2 * c];
    T h = rd ? rd[3 + c][id] : H[id];
    if (main_rng) {
      const T* Ea = rd ? rd[ta] : p.f[ta];
      const T* Eb = rd ? rd[tb] : p.f[tb];
      const T d_a = Ea[id + st[tb]] - Ea[id];
      const T d_b = Eb[id + st[ta]] - Eb[id];
      h = ca * h + cb * (p.fh[tb][x[tb]] * d_a - p.fh[ta][x[ta]] * d_b);
    }
    for (int s = 0; s < p.n_slab; ++s) {
      const SlabD<T>& sl = p.slab[s];
      if (sl.m == c) continue;
      const int l = sel3(sl.m, i, j, k) - sl.h_lo;
      if (l < 0 || l >= sl.n) continue;
      const int which = (c == (sl.m + 1) % 3) ? 0 : 1;
      // H_A differences E_B, H_B differences E_A, forward along m.
      const int dc = which == 0 ? (sl.m + 2) % 3 : (sl.m + 1) % 3;
      const T* D = rd ? rd[dc] : p.f[dc];
      const T diff = D[id + sel3(sl.m, st[0], st[1], st[2])] - D[id];
      T* ps = sl.psi_h[which] + psi_index(sl, L, i, j, k, l);
      const T psi = sl.b_h[l] * *ps + sl.a_h[l] * diff;
      *ps = psi;
      h += (which == 0 ? cb : -cb) * psi;
    }
    H[id] = h;
  }
}

// ---------------------------------------------------------------------------
// E sweep.  Main update over x_c < n_c and 1 <= x < n across
// (BasicUpdator3D::updateE, src/updator/basic_updator_3d.cpp:38-69), then
// CPML (PMLCorrector<xyz>::correctE, pml_corrector.h:178-288): layers
// [e_lo, e_lo + n) along m, whole transverse extent.
// ---------------------------------------------------------------------------
// `rd` (ping-pong sweeps): the buffer holding the old E, read for the node's
// own value; the new H neighbours and the result are in p.f.  Null: in place.
template <typename T>
__device__ __forceinline__ void update_e_node(const YeeP<T>& p, int i, int j, int k,
                                              T* const* rd = nullptr) {
  const Lat L = p.L;
  const long long id = lat_index(L, i, j, k);
  const int x[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  const long long st[3] = {(long long)L.NY * L.KP, (long long)L.KP, 1};
  const T* row = p.tab + (size_t)p.cls[id] * 12;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
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
    if (!valid) continue;
    main_rng = main_rng && valid;
    const int ta = (c + 1) % 3, tb = (c + 2) % 3;
    T* E = p.f[c];
    const T ca = row[2 * c];
    const T cb = row[2 * c + 1];
    T e = rd ? rd[c][id] : E[id];
    if (main_rng) {
      const T* Ha = p.f[3 + ta];
      const T* Hb = p.f[3 + tb];
      const T d_a = Hb[id] - Hb[id - st[ta]];
      const T d_b = Ha[id] - Ha[id - st[tb]];
      e = ca * e + cb * (p.fe[ta][x[ta]] * d_a - p.fe[tb][x[tb]] * d_b);
    }
    for (int s = 0; s < p.n_slab; ++s) {
      const SlabD<T>& sl = p.slab[s];
      if (sl.m == c) continue;
      const int l = sel3(sl.m, i, j, k) - sl.e_lo;
      if (l < 0 || l >= sl.n) continue;
      const int which = (c == (sl.m + 1) % 3) ? 0 : 1;
      // E_A differences H_B, E_B differences H_A, backward along m.
      const T* D = p.f[3 + (which == 0 ? (sl.m + 2) % 3 : (sl.m + 1) % 3)];
      const T diff = D[id] - D[id - sel3(sl.m, st[0], st[1], st[2])];
      T* ps = sl.psi_e[which] + psi_index(sl, L, i, j, k, l);
      const T psi = sl.b_e[l] * *ps + sl.a_e[l] * diff;
      *ps = psi;
      e += (which == 0 ? -cb : cb) * psi;
    }
    E[id] = e;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_update_h(const __grid_constant__ YeeP<T> p) {
  pdl_enter();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k > p.L.nz || j > p.L.ny || i > p.L.nx) return;
  update_h_node(p, i, j, k);
}

template <typename T>
__global__ void __launch_bounds__(256) k_update_e(const __grid_constant__ YeeP<T> p) {
  pdl_enter();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k > p.L.nz || j > p.L.ny || i > p.L.nx) return;
  update_e_node(p, i, j, k);
}

// The lattice faces k = nz (all i, j) and j = ny (all i, k < nz), which hold
// only boundary nodes: every component there is either out of range or
// outside its main update range, so it changes only by CPML terms.  Sweeps
// that tile k < nz, j < ny leave these faces to the two kernels below, one
// thread per node, with the arithmetic of k_update_h / k_update_e; a node in
// no CPML layer returns at once.
__host__ __device__ __forceinline__ long long edge_nodes(const Lat& L) {
  return (long long)(L.nx + 1) * (L.ny + 1) + (long long)(L.nx + 1) * L.nz;
}

// Face node t (< 2^31: two lattice faces) as (i, j, k), 32-bit decoding.
__device__ __forceinline__ void edge_node(const Lat& L, long long t, int& i, int& j, int& k) {
  const unsigned fa = (unsigned)((L.nx + 1) * (L.ny + 1));
  unsigned u = (unsigned)t;
  if (u < fa) {
    i = (int)(u / (unsigned)(L.ny + 1));
    j = (int)(u - (unsigned)i * (unsigned)(L.ny + 1));
    k = L.nz;
  } else {
    u -= fa;
    i = (int)(u / (unsigned)L.nz);
    k = (int)(u - (unsigned)i * (unsigned)L.nz);
    j = L.ny;
  }
}

template <typename T>
__device__ __forceinline__ bool in_some_layer(const YeeP<T>& p, int i, int j, int k, bool e) {
  for (int s = 0; s < p.n_slab; ++s) {
    const SlabD<T>& sl = p.slab[s];
    const int l = sel3(sl.m, i, j, k) - (e ? sl.e_lo : sl.h_lo);
    if (l >= 0 && l < sl.n) return true;
  }
  return false;
}

template <typename T, bool E>
__device__ __forceinline__ void edge_update(const YeeP<T>& p, long long t) {
  if (t >= edge_nodes(p.L)) return;
  int i, j, k;
  edge_node(p.L, t, i, j, k);
  if (!in_some_layer(p, i, j, k, E)) return;
  if (E)
    update_e_node(p, i, j, k);
  else
    update_h_node(p, i, j, k);
}

template <typename T>
__global__ void __launch_bounds__(256) k_edge_h(const __grid_constant__ YeeP<T> p) {
  edge_update<T, false>(p, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_edge_e(const __grid_constant__ YeeP<T> p) {
  edge_update<T, true>(p, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Ping-pong forms (sweep 7): a face node in a CPML layer is written to p.f
// from the old fields in `rd`.  A node in no layer never changes, and the
// engine keeps both buffers equal on such nodes (uploads and restored states
// fill both), so it is skipped as in the in-place form -- unless `copy_all`
// (a lumped element, inductor or coefficient override adds to some face
// node after the sweep), when every face node is carried over.
template <typename T, bool E>
__global__ void __launch_bounds__(256) k_edge_pp(const __grid_constant__ YeeP<T> p,
                                                 T* const* rd, bool copy_all) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= edge_nodes(p.L)) return;
  int i, j, k;
  edge_node(p.L, t, i, j, k);
  if (!copy_all && !in_some_layer(p, i, j, k, E)) return;
  if (E)
    update_e_node(p, i, j, k, rd);
  else
    update_h_node(p, i, j, k, rd);
}

// Many lattices in one launch: block b covers the 256 face nodes starting at
// blocks[b].y * 256 of lattice blocks[b].x.
template <typename T, bool E>
__global__ void __launch_bounds__(256)
    k_edge_batch(const YeeP<T>* __restrict__ scenes, const int2* __restrict__ blocks) {
  const int2 b = blocks[blockIdx.x];
  edge_update<T, E>(scenes[b.x], (long long)b.y * 256 + threadIdx.x);
}

// ---------------------------------------------------------------------------
// TFSF3D face corrections (TFSF3DCorrector, src/waveform_source/tfsf_corrector.cpp:177-232,
// correctTFSF, src/include/waveform_source/tfsf_corrector.h:89-229).  The 12
// passes of one phase go in two launches so that the passes that meet on a
// box edge (same component, different face axes) are applied in the
// reference order; within a launch no two threads touch the same node.
// The incident value is interpolated in FP64 from the 1-D grid row of the
// current step (exInc..hzInc, tfsf_corrector.cpp:16-122).
// ---------------------------------------------------------------------------
struct TfsfD {
  int bs[3];
  int aux;
  const double* e_inc;
  const double* h_inc;
  const double* p_int[3];
  const double* p_half[3];
  double te[3], th[3];
};

struct TfsfPassD {
  int axis, neg, field, is_e;
  int s[3], e[3];
  long long begin;
  double coeff;
};

struct TfsfGroupD {
  int n;
  long long total;
  TfsfPassD pass[6];
};

__device__ __forceinline__ double tfsf_incident(const TfsfD& tf, bool inc_e, int comp,
                                                long long t, const int x[3], int* err) {
  // Per axis d: the offset from the box start, one further along the
  // component axis (E incident) or along the other two (H incident); the
  // projection table is the half-step one along the component axis for E and
  // the integer one for H, and the other way round across.  Written with
  // selects so that nothing is indexed by a run-time axis (no local memory).
  double parts[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const bool along = d == comp;
    const int r = x[d] - tf.bs[d] + ((inc_e ? along : !along) ? 1 : 0);
    const bool half = inc_e ? along : !along;
    parts[d] = half ? tf.p_half[d][r] : tf.p_int[d][r];
  }
  const double proj = inc_e ? parts[0] + parts[1] + parts[2]
                            : parts[0] + parts[1] + parts[2] - 0.5;
  long long idx = (long long)proj;
  const double w = proj - (double)idx;
  const int len = inc_e ? tf.aux : tf.aux - 1;
  if (idx < 0 || idx + 1 >= len) {
    *err = 1;
    idx = idx < 0 ? 0 : (long long)len - 2;
  }
  const double* row = inc_e ? tf.e_inc + t * tf.aux : tf.h_inc + t * (tf.aux - 1);
  const double tr = inc_e ? tf.te[comp] : tf.th[comp];
  return tr * ((1 - w) * row[idx] + w * row[idx + 1]);
}

// `cls` / `tab` (H passes only): add the correction divided by the node's ca
// (sweep 7's pre-pass on the H it is about to read, see k_tfsf_pre).
template <typename T>
__device__ __forceinline__ void tfsf_node(const TfsfD& tf, const TfsfGroupD& g, const Lat& L,
                                          T* const* fields, const long long* step, int* err,
                                          long long tid, const uint16_t* cls = nullptr,
                                          const T* tab = nullptr) {
  if (tid >= g.total) return;
  int q = 0;
  while (q + 1 < g.n && tid >= g.pass[q + 1].begin) ++q;
  const TfsfPassD& P = g.pass[q];
  // A pass covers one face: far fewer than 2^31 nodes, so 32-bit decoding.
  unsigned r = (unsigned)(tid - P.begin);
  const unsigned e2 = (unsigned)(P.e[2] - P.s[2]), e1 = (unsigned)(P.e[1] - P.s[1]);
  const int k = P.s[2] + (int)(r % e2);
  r /= e2;
  const int j = P.s[1] + (int)(r % e1);
  r /= e1;
  const int i = P.s[0] + (int)r;
  const long long t = *step;
  int xi[3] = {i, j, k};
  int xf[3] = {i, j, k};
  const int m = P.axis;
  bool inc_e;
  if (P.is_e) {
    inc_e = false;  // E face reads the H incident half a cell outside
    if (P.neg) xi[m] -= 1;
  } else {
    inc_e = true;   // H face corrects the node half a cell outside
    if (P.neg) xf[m] -= 1;
  }
  const int dual = (P.field == (m + 1) % 3) ? (m + 2) % 3 : (m + 1) % 3;
  int e_flag = 0;
  const double v = tfsf_incident(tf, inc_e, dual, t, xi, &e_flag);
  if (e_flag) atomicOr(err, 1);
  T* F = fields[(P.is_e ? 0 : 3) + P.field];
  const long long id = lat_index(L, xf[0], xf[1], xf[2]);
  if (cls) {
    const double ca = (double)tab[(size_t)cls[id] * 12 + 6 + 2 * P.field];
    F[id] = (T)((double)F[id] + v * P.coeff / ca);
  } else {
    F[id] = (T)((double)F[id] + v * P.coeff);
  }
}

template <typename T>
__global__ void k_tfsf(const __grid_constant__ TfsfD tf, const __grid_constant__ TfsfGroupD g,
                       Lat L, T* const* fields, const long long* step,
                       int* err) {
  pdl_enter();
  tfsf_node<T>(tf, g, L, fields, step, err, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// TFSF H-face corrections before sweep 7 (TFSF3DCorrector::correctH,
// src/waveform_source/tfsf_corrector.cpp:205-232, in its pass order): the
// reference adds coeff v to H after updateH, H' = ca H + cb curl E + coeff v.
// Sweep 7 reads H from the input buffer in several kernels (the fused box,
// its halo recomputes, the CPML tiles), so the correction goes into that H
// first, divided by the node's ca: ca (H + coeff v / ca) + cb curl E is the
// same sum (the two differ by one rounding).  Every reader of the old H then
// sees the corrected value, and no sweep kernel carries TFSF code.  The input
// buffer's H is overwritten by the next step's sweep.
template <typename T>
__global__ void k_tfsf_pre(const __grid_constant__ TfsfD tf, const __grid_constant__ TfsfGroupD g,
                           Lat L, T* const* fields_in, const uint16_t* cls, const T* tab,
                           const long long* step, int* err) {
  tfsf_node<T>(tf, g, L, fields_in, step, err, (long long)blockIdx.x * blockDim.x + threadIdx.x,
               cls, tab);
}

// Per-lattice TFSF state for the batched launch: the incident tables, the
// four pass groups (H 1, H 2, E 1, E 2) and where the lattice's fields, step
// counter and error word live.
template <typename T>
struct TfsfSceneD {
  TfsfD tf;
  TfsfGroupD g[4];
  Lat L;
  T* const* fields;
  const long long* step;
  int* err;
};

// Pass group `group` of many lattices in one launch: block b covers the 256
// face nodes starting at blocks[b].y * 256 of lattice blocks[b].x.
template <typename T>
__global__ void __launch_bounds__(256)
    k_tfsf_batch(const TfsfSceneD<T>* __restrict__ scenes, const int2* __restrict__ blocks,
                 int group) {
  const int2 b = blocks[blockIdx.x];
  const TfsfSceneD<T>& S = scenes[b.x];
  tfsf_node<T>(S.tf, S.g[group], S.L, S.fields, S.step, S.err,
               (long long)b.y * 256 + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Lumped current sources: E += coff * waveform[t]
// (CurrentSourceCorrector::correctE, src/object/lumped_element/lumped_element_corrrector.cpp:24-37).
// ---------------------------------------------------------------------------
struct LumpedD {
  long long n;
  int n_steps;
  const long long* node;
  const int* comp;
  const int* source;
  const double* coff;
  const double* wave;  // n_sources x n_steps
};

template <typename T>
__global__ void k_lumped(LumpedD lp, T* const* fields, const long long* step) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= lp.n) return;
  const long long t = *step;
  T* E = fields[lp.comp[e]];
  const long long id = lp.node[e];
  const double w = lp.wave[(long long)lp.source[e] * lp.n_steps + t];
  E[id] = (T)((double)E[id] + lp.coff[e] * w);
}

// ---------------------------------------------------------------------------
// Lumped inductors on their compacted node list (InductorCorrector::correctE,
// src/object/lumped_element/lumped_element_corrrector.cpp:42-99): after the E
// update, E += cecjc * J, then J += cjcec * E with the corrected E.  J is an
// FP64 state in both precisions; in FP32 it advances with the stored E.
// ---------------------------------------------------------------------------
struct InductorD {
  long long n;
  const long long* node;
  const int* comp;
  const double* cecjc;
  const double* cjcec;
  double* j;
};

template <typename T>
__global__ void k_inductor(InductorD d, T* const* fields) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.n) return;
  T* E = fields[d.comp[q]];
  const long long id = d.node[q];
  const double jq = d.j[q];
  const T en = (T)((double)E[id] + d.cecjc[q] * jq);
  E[id] = en;
  d.j[q] = jq + d.cjcec[q] * (double)en;
}

// ---------------------------------------------------------------------------
// ADE on the compacted dispersive node list.  The E sweep has already
// written the plain Yee value with the ADE-overwritten (ca, cb) of the node;
// k_ade_update adds the polarisation terms and advances J
// (MLorentzUpdator::updateE/updateJ/calculateJSum/recordEPrevious,
//  src/updator/m_lor_ade_updator.cpp:21-140; Drude/Debye J updates,
//  src/updator/ade_updator/drude_ade_updator.cpp:31-39,
//  src/updator/ade_updator/debye_ade_updator.cpp:43-51).  k_ade_gather saves
// the node's field value before the E sweep (the reference's e_cur).
// ---------------------------------------------------------------------------
template <typename T>
struct AdeD {
  long long n;
  int np;
  const long long* node;
  const uint8_t* comp;
  const uint8_t* mat;
  const T* coef;  // per material: cejsum, ceep, then per pole 7 values
  T* j;           // np x n
  T* jp;          // np x n (kind 0)
  T* ep;          // n (kind 0)
  T* ec;          // n
};

template <typename T>
__global__ void k_ade_gather(AdeD<T> a, T* const* fields) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  a.ec[e] = fields[a.comp[e]][a.node[e]];
}

// fields_in (ping-pong sweeps): the buffer still holding E^n, read directly
// as e_cur; null when k_ade_gather saved it.
template <typename T, int KIND>
__global__ void k_ade_update(AdeD<T> a, T* const* fields, T* const* fields_in) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  const T* cf = a.coef + (size_t)a.mat[e] * (2 + 7 * a.np);
  T* E = fields[a.comp[e]];
  const long long id = a.node[e];
  const T e_yee = E[id];
  const T e_cur = fields_in ? fields_in[a.comp[e]][id] : a.ec[e];
  const T e_prev = (KIND == 0) ? a.ep[e] : T(0);
  T j_sum = 0;
  for (int p = 0; p < a.np; ++p) {
    const T* pc = cf + 2 + 7 * p;
    const long long q = (long long)p * a.n + e;
    if (KIND == 0) {
      j_sum += pc[5] * a.j[q] + pc[6] * a.jp[q];
    } else {
      j_sum += pc[5] * a.j[q];
    }
  }
  const T e_next = (cf[1] * e_prev + e_yee) + cf[0] * j_sum;
  E[id] = e_next;
  for (int p = 0; p < a.np; ++p) {
    const T* pc = cf + 2 + 7 * p;
    const long long q = (long long)p * a.n + e;
    if (KIND == 0) {
      const T jn = pc[2] * e_next + pc[3] * e_cur + pc[4] * e_prev + pc[0] * a.j[q] +
                   pc[1] * a.jp[q];
      a.jp[q] = a.j[q];
      a.j[q] = jn;
    } else if (KIND == 1) {
      a.j[q] = pc[0] * a.j[q] + pc[3] * (e_next + e_cur);
    } else {
      a.j[q] = pc[0] * a.j[q] + pc[3] * (e_next - e_cur);
    }
  }
  if (KIND == 0) a.ep[e] = e_cur;
}

// ---------------------------------------------------------------------------
// NF2FF.  k_nf2ff_sample writes, per Huygens node, the four signed
// surface-centre field values of the step into slot t % batch of an FP64
// sample buffer (calculateJ/calculateM, src/nffft/nffft_fd_data_update.cpp:22-122,
// with interpolateSurfaceCenter, src/include/nffft/interpolate_scheme.h:19-138);
// k_nf2ff_dft folds a full batch into the complex FP64 accumulators with the
// per-step phasors (FDPlaneData::initDFT, src/nffft/nffft_fd_data.cpp:65-76).
// ---------------------------------------------------------------------------
// Compensated accumulation across batches (a run of thousands of steps adds
// one batch partial per window to each running sum): s + x is rounded into s
// and its exact rounding error (Knuth's TwoSum, six additions, no branch) is
// added to c, so the error of the final s + c does not grow with the number
// of windows.  The _rn intrinsics keep the compiler from contracting or
// reassociating the additions.
__device__ __forceinline__ void two_sum_acc(double& s, double& c, double x) {
  const double t = __dadd_rn(s, x);
  const double bp = __dsub_rn(t, s);
  const double err = __dadd_rn(__dsub_rn(s, __dsub_rn(t, bp)), __dsub_rn(x, bp));
  c = __dadd_rn(c, err);
  s = t;
}

struct Nf2ffD {
  int nf, batch;
  int s[6][3], e[6][3];
  long long begin[7];  // node offsets per face, begin[6] = total
  long long P;
  double* sample;      // batch x 4 x P
  double2* acc;        // (nf*4) x P: running sums
  double2* comp;       // (nf*4) x P: their compensation terms (TwoSum errors);
                       // the accumulated value is acc + comp
  const double2* te;   // nf x n_steps
  const double2* th;
  int n_steps;
  double scale;
};

template <typename T>
__device__ __forceinline__ T fld(const T* F, const Lat& L, int i, int j, int k) {
  return F[lat_index(L, i, j, k)];
}

template <typename T>
__device__ double surf_e(T* const* f, const Lat& L, int m, int comp, int i, int j, int k) {
  int q[3] = {i, j, k};
  q[3 - m - comp] += 1;
  const T* E = f[comp];
  return 0.5 * ((double)fld(E, L, q[0], q[1], q[2]) + (double)fld(E, L, i, j, k));
}

template <typename T>
__device__ double surf_h(T* const* f, const Lat& L, int m, int comp, int i, int j, int k) {
  const T* H = f[3 + comp];
  if (m == 0) {
    int p1[3] = {i, j, k};
    p1[comp] += 1;
    return 0.25 * ((double)fld(H, L, p1[0], p1[1], p1[2]) + (double)fld(H, L, i, j, k) +
                   (double)fld(H, L, p1[0] - 1, p1[1], p1[2]) + (double)fld(H, L, i - 1, j, k));
  }
  if (m == 1) {
    if (comp == 2)
      return 0.25 * ((double)fld(H, L, i, j, k + 1) + (double)fld(H, L, i, j, k) +
                     (double)fld(H, L, i, j - 1, k + 1) + (double)fld(H, L, i, j - 1, k));
    return 0.25 * ((double)fld(H, L, i + 1, j, k) + (double)fld(H, L, i, j, k) +
                   (double)fld(H, L, i + 1, j - 1, k) + (double)fld(H, L, i, j - 1, k));
  }
  if (comp == 0)
    return 0.25 * ((double)fld(H, L, i + 1, j, k) + (double)fld(H, L, i, j, k) +
                   (double)fld(H, L, i, j, k - 1) + (double)fld(H, L, i + 1, j, k - 1));
  return 0.25 * ((double)fld(H, L, i, j, k) + (double)fld(H, L, i, j + 1, k) +
                 (double)fld(H, L, i, j, k - 1) + (double)fld(H, L, i, j + 1, k - 1));
}

template <typename T>
__global__ void k_nf2ff_sample(const __grid_constant__ Nf2ffD nf, Lat L, T* const* fields,
                               const long long* step) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nf.P) return;
  int d = 0;
  while (d < 5 && p >= nf.begin[d + 1]) ++d;
  // A face holds far fewer than 2^31 points: 32-bit decoding.
  unsigned r = (unsigned)(p - nf.begin[d]);
  const int* s = nf.s[d];
  const int* e = nf.e[d];
  const unsigned e2 = (unsigned)(e[2] - s[2]), e1 = (unsigned)(e[1] - s[1]);
  const int k = s[2] + (int)(r % e2);
  r /= e2;
  const int j = s[1] + (int)(r % e1);
  r /= e1;
  const int i = s[0] + (int)r;
  const int m = d / 2;
  const bool positive = (d % 2) == 1;
  const int A = (m + 1) % 3, B = (m + 2) % 3;
  const long long slot = *step % nf.batch;
  double* out = nf.sample + slot * 4 * nf.P + p;
  const double cj1 = positive ? -1.0 : 1.0, cj2 = positive ? 1.0 : -1.0;
  out[0] = cj1 * surf_h(fields, L, m, B, i, j, k);
  out[nf.P] = cj2 * surf_h(fields, L, m, A, i, j, k);
  out[2 * nf.P] = -cj1 * surf_e(fields, L, m, B, i, j, k);
  out[3 * nf.P] = -cj2 * surf_e(fields, L, m, A, i, j, k);
}

// Batch DFT: acc[f][q][p] += scale * sum_s sample[s][q][p] * phasor_q[f][t0+s].
// One thread per (q, p); phasors of the batch staged in shared memory.
template <int FCH>
__global__ void __launch_bounds__(256) k_nf2ff_dft(Nf2ffD nf, const long long* step, int nb,
                                                   long long t0_explicit) {
  extern __shared__ double2 sh[];  // [2][nf][batch]
  long long t0;
  if (nb <= 0) {
    nb = nf.batch;
    t0 = *step + 1 - nf.batch;
  } else {
    t0 = t0_explicit;
  }
  // Steps t0 .. t0+nb-1 lie in one batch window: slots slot0 .. slot0+nb-1.
  const long long slot0 = t0 % nf.batch;
  for (int x = threadIdx.x; x < nf.nf * nb; x += blockDim.x) {
    const int f = x / nb, s = x % nb;
    sh[f * nf.batch + s] = nf.th[(long long)f * nf.n_steps + t0 + s];
    sh[nf.nf * nf.batch + f * nf.batch + s] = nf.te[(long long)f * nf.n_steps + t0 + s];
  }
  __syncthreads();
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 4 * nf.P) return;
  const int q = (int)(tid / nf.P);
  const long long p = tid % nf.P;
  const double2* ph = sh + (q < 2 ? 0 : nf.nf * nf.batch);
  const double* smp = nf.sample + (slot0 * 4 + q) * nf.P + p;
  for (int f0 = 0; f0 < nf.nf; f0 += FCH) {
    double re[FCH], im[FCH];
#pragma unroll
    for (int u = 0; u < FCH; ++u) re[u] = im[u] = 0.0;
    for (int s = 0; s < nb; ++s) {
      const double v = smp[(long long)s * 4 * nf.P];
#pragma unroll
      for (int u = 0; u < FCH; ++u) {
        if (f0 + u < nf.nf) {
          const double2 z = ph[(f0 + u) * nf.batch + s];
          re[u] += v * z.x;
          im[u] += v * z.y;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < FCH; ++u) {
      if (f0 + u < nf.nf) {
        const long long o = ((long long)(f0 + u) * 4 + q) * nf.P + p;
        double2 z = nf.acc[o], c = nf.comp[o];
        two_sum_acc(z.x, c.x, __dmul_rn(nf.scale, re[u]));
        two_sum_acc(z.y, c.y, __dmul_rn(nf.scale, im[u]));
        nf.acc[o] = z;
        nf.comp[o] = c;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Movie frame: copy the monitor box of one component into frame t/interval
// (FieldMonitor::output, src/monitor/field_monitor.cpp:82-96).
// ---------------------------------------------------------------------------
struct MovieD {
  int field;
  int s[3], e[3];
  int interval;
  long long max_frames;
  void* store;
};

template <typename T>
__global__ void k_movie(const __grid_constant__ MovieD mv, Lat L, T* const* fields,
                        const long long* step) {
  const int e2 = mv.e[2] - mv.s[2], e1 = mv.e[1] - mv.s[1], e0 = mv.e[0] - mv.s[0];
  const long long n = (long long)e0 * e1 * e2;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n) return;
  const long long frame = *step / mv.interval;
  if (frame >= mv.max_frames) return;
  int i, j, k;
  if (n < (1LL << 31)) {  // 32-bit decoding (64-bit division is emulated)
    unsigned r = (unsigned)tid;
    k = mv.s[2] + (int)(r % (unsigned)e2);
    r /= (unsigned)e2;
    j = mv.s[1] + (int)(r % (unsigned)e1);
    r /= (unsigned)e1;
    i = mv.s[0] + (int)r;
  } else {
    long long r = tid;
    k = mv.s[2] + (int)(r % e2);
    r /= e2;
    j = mv.s[1] + (int)(r % e1);
    r /= e1;
    i = mv.s[0] + (int)r;
  }
  T* out = static_cast<T*>(mv.store) + frame * n + tid;
  *out = fields[mv.field][lat_index(L, i, j, k)];
}

// ---------------------------------------------------------------------------
// Per-node E coefficient overrides: nodes whose E update uses its own
// (ca, cb) instead of its material class's pair (ca0, cb0) -- for example
// the nodes around a block of per-voxel permittivities, each of which would
// otherwise need a class of its own.  The sweep applies the class pair; the
// override then rescales: E' = r E_sweep + d E_old with r = cb / cb0 and
// d = ca - r ca0, which is ca E_old + cb (curl H) for a node in the main
// range outside CPML layers (the only nodes the host overrides).  E_old is
// saved before a split sweep (k_ovr_gather) or read from the input buffer of
// a ping-pong sweep.
// ---------------------------------------------------------------------------
template <typename T>
struct OverrideD {
  long long n;
  const long long* node;  // lattice index
  const uint8_t* comp;    // 0..2
  T* r;
  T* d;
  T* eold;
};

template <typename T>
__global__ void k_ovr_prepare(OverrideD<T> o, const uint16_t* cls, const T* tab, const double* ca,
                              const double* cb) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= o.n) return;
  const T* row = tab + (size_t)cls[o.node[q]] * 12 + 2 * o.comp[q];
  const double r = cb[q] / (double)row[1];
  o.r[q] = (T)r;
  o.d[q] = (T)(ca[q] - r * (double)row[0]);
}

template <typename T>
__global__ void k_ovr_gather(OverrideD<T> o, T* const* fields) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= o.n) return;
  o.eold[q] = fields[o.comp[q]][o.node[q]];
}

template <typename T>
__global__ void k_ovr_apply(OverrideD<T> o, T* const* fields, T* const* fields_in) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= o.n) return;
  T* E = fields[o.comp[q]];
  const long long id = o.node[q];
  const T old = fields_in ? fields_in[o.comp[q]][id] : o.eold[q];
  E[id] = o.r[q] * E[id] + o.d[q] * old;
}

// ---------------------------------------------------------------------------
// NaN / Inf watchdog: a grid-stride scan of the six field buffers (padding
// included: it stays zero) that sets bit 4 of the error word on the first
// non-finite value; the host reads it at the next sync (XFD_ERR_NUMERIC).
// Nothing traps and the sweep runs on.  No counterpart in the reference,
// whose only numeric check is MLorentzEqDecision::stabilityCondition
// (src/material/dispersive_material_equation.cpp:56-98).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_watchdog(T* const* fields, long long n_lat, int* err) {
  bool bad = false;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int c = 0; c < 6; ++c) {
    const T* f = fields[c];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n_lat; q += stride)
      bad = bad || !isfinite(f[q]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(err, 4);
}

// ---------------------------------------------------------------------------
// Per-node H curl-term corrections, for coefficients that scale one curl term
// of an H node but not the other (ThinWire::correctUpdateCoefficient,
// src/object/thin_wire.cpp:42-133, multiplies chxey / chyex / chzex / chzey
// next to the wire).  The class table holds one cb per component, so the
// sweep applies the unscaled pair and this pass adds the difference:
//   H_c += da (E_a[x_b+1] - E_a) + db (E_b[x_a+1] - E_b)
// with the E of the same step (the E sweep has not run yet); a = c+1,
// b = c+2.  One entry per (node, component): no two threads write one value.
// ---------------------------------------------------------------------------
template <typename T>
struct HTermD {
  long long n;
  const long long* node;  // lattice index
  const uint8_t* comp;    // 0..2: Hx Hy Hz
  const T* da;
  const T* db;
};

template <typename T>
__global__ void k_hterm(const __grid_constant__ HTermD<T> h, Lat L, T* const* fields) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= h.n) return;
  const int c = h.comp[q], a = (c + 1) % 3, b = (c + 2) % 3;
  // lattice strides by selects (no run-time-indexed local array)
  auto stride = [&](int d) {
    return d == 0 ? (long long)L.NY * L.KP : (d == 1 ? (long long)L.KP : 1LL);
  };
  const long long id = h.node[q];
  const T* Ea = fields[a];
  const T* Eb = fields[b];
  T* H = fields[3 + c];
  H[id] += h.da[q] * (Ea[id + stride(b)] - Ea[id]) + h.db[q] * (Eb[id + stride(a)] - Eb[id]);
}

// ---------------------------------------------------------------------------
// Time-domain NF2FF (NFFFTTimeDomain::update, src/nffft/nfffft_time_domain.cpp:80-96
// -> TDPlaneData::update, src/include/nffft/nffft_td_data.h:169-240): per
// Huygens point and step, the surface-centre tangential E and H
// (interpolateSurfaceCenter, as for the frequency-domain transform) minus
// their values of the previous step, weighted by the face-cell area, are
// added to the retarded-time bins nn, nn + 1 of the far-field potentials,
// nn + f = delay + offset + t (offset 1/2 for E, 0 for H; delay = (the
// surface's largest projected distance - the point's) / (c dt), FP64 on the
// host).  Face with normal m, tangential axes A = m+1, B = m+2, sign
// s = -1 on the negative face: U[A] += s (B change), U[B] -= s (A change) for
// E; W[A] -= s (B change), W[B] += s (A change) for H.  The bins are shared
// by many points: FP64 atomics.
// ---------------------------------------------------------------------------
struct Nf2ffTdD {
  int s[6][3], e[6][3];
  long long begin[7];  // point offsets per face, begin[6] = P
  long long P;
  const double* delay;  // P
  const double* ds;     // P
  double* prev;         // 4 x P: E_a, E_b, H_a, H_b of the previous step
  double* pot;          // 6 x n_bins: W_x W_y W_z U_x U_y U_z
  long long n_bins;
};

__device__ __forceinline__ void td_add(double* row, long long n_bins, double x, double c,
                                       double ds, double delta, int* err) {
  const long long nn = (long long)floor(x);
  const double f = x - (double)nn;
  if (nn < 0 || nn + 1 >= n_bins) {
    atomicOr(err, 1);
    return;
  }
  atomicAdd(row + nn, c * (1 - f) * ds * delta);
  atomicAdd(row + nn + 1, c * f * ds * delta);
}

template <typename T>
__global__ void k_nf2ff_td(const __grid_constant__ Nf2ffTdD td, Lat L, T* const* fields,
                           const long long* step,
                           int* err) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= td.P) return;
  int d = 0;
  while (d < 5 && p >= td.begin[d + 1]) ++d;
  unsigned r = (unsigned)(p - td.begin[d]);  // one face: 32-bit decoding
  const int* s = td.s[d];
  const int* e = td.e[d];
  const unsigned e2 = (unsigned)(e[2] - s[2]), e1 = (unsigned)(e[1] - s[1]);
  const int k = s[2] + (int)(r % e2);
  r /= e2;
  const int j = s[1] + (int)(r % e1);
  r /= e1;
  const int i = s[0] + (int)r;
  const int m = d / 2;
  const double sg = (d % 2) ? 1.0 : -1.0;
  const int A = (m + 1) % 3, B = (m + 2) % 3;
  const double t = (double)*step;
  const double ds = td.ds[p];
  // E: coefficients (1, -1) times the face sign, bins at delay + 1/2 + t
  const double ea = surf_e(fields, L, m, A, i, j, k), eb = surf_e(fields, L, m, B, i, j, k);
  const double dea = ea - td.prev[p], deb = eb - td.prev[td.P + p];
  td.prev[p] = ea;
  td.prev[td.P + p] = eb;
  const double xe = (td.delay[p] + 0.5) + t;
  td_add(td.pot + (3 + A) * td.n_bins, td.n_bins, xe, sg, ds, deb, err);
  td_add(td.pot + (3 + B) * td.n_bins, td.n_bins, xe, -sg, ds, dea, err);
  // H: coefficients (-1, 1) times the face sign, bins at delay + t
  const double ha = surf_h(fields, L, m, A, i, j, k), hb = surf_h(fields, L, m, B, i, j, k);
  const double dha = ha - td.prev[2 * td.P + p], dhb = hb - td.prev[3 * td.P + p];
  td.prev[2 * td.P + p] = ha;
  td.prev[3 * td.P + p] = hb;
  const double xh = (td.delay[p] + 0.0) + t;
  td_add(td.pot + A * td.n_bins, td.n_bins, xh, -sg, ds, dhb, err);
  td_add(td.pot + B * td.n_bins, td.n_bins, xh, sg, ds, dha, err);
}

// ---------------------------------------------------------------------------
// Weighted probes: per probe and step, value = sum_q w[q] F_{comp[q]}(node q),
// one CTA per probe (FP64 block reduction), written to series[probe][t]
// (VoltageMonitor::update, src/monitor/voltage_monitor.cpp:198-235;
// CurrentMonitor::update, src/monitor/current_monitor.cpp:253-379).
// ---------------------------------------------------------------------------
struct ProbeD {
  int n_probes;
  const long long* begin;  // n_probes + 1 entry offsets
  const long long* node;   // lattice index
  const uint8_t* comp;     // 0..5
  const double* w;
  double* series;          // n_probes x n_steps
  long long n_steps;
};

template <typename T>
__global__ void __launch_bounds__(256) k_probes(const __grid_constant__ ProbeD pr, T* const* fields,
                                                const long long* step) {
  pdl_enter();
  const int q = blockIdx.x;
  double acc = 0.0;
  for (long long e = pr.begin[q] + threadIdx.x; e < pr.begin[q + 1]; e += blockDim.x)
    acc += pr.w[e] * (double)fields[pr.comp[e]][pr.node[e]];
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) v += red[wi];
    const long long t = *step;
    if (t >= 0 && t < pr.n_steps) pr.series[(long long)q * pr.n_steps + t] = v;
  }
}

__global__ void k_advance(long long* step) {
  pdl_enter();
  *step += 1;
}

// Step counters of many lattices.
__global__ void k_advance_batch(long long* const* steps, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) *steps[s] += 1;
}

}  // namespace xfd
