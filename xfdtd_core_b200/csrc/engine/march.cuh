// Marching split sweeps: the H update and the E update of one time step as
// two kernels, each CTA owning a (TJ x TK) tile of the (j, k) plane and
// marching along i over a chunk of planes.  Per plane a thread updates the
// three components of its node; the i-neighbour it needs twice (E of plane
// i+1 for H, H of plane i-1 for E) is carried in registers from the previous
// plane, and everything that does not change along i -- the curl factors of
// j and k, the CPML layers normal to y and z with their grading -- is read
// once before the march.  The CPML term of each component reuses the
// difference of its curl term along the slab's axis.
//
// Arithmetic, ranges and correction order are those of k_update_h /
// k_update_e (kernels.cuh): the main update over the reference's loop
// ranges (BasicUpdator::updateH, src/updator/basic_updator.cpp:23-36;
// BasicUpdator3D::updateE, src/updator/basic_updator_3d.cpp:38-69), then the
// CPML corrections (PMLCorrector<xyz>::correctH/correctE,
// src/include/boundary/pml_corrector.h:178-382) over each component's whole
// transverse extent, slab axes in ascending order.  CPML slabs must be at
// most one per side of an axis, with disjoint layers (checked when a slab is
// added).
#pragma once

#include "fused.cuh"

namespace xfd {

template <typename T>
struct MarchP {
  Lat L;
  T* f[6];  // Ex Ey Ez Hx Hy Hz, updated in place
  const uint16_t* cls;
  const T* tab;
  int n_classes;
  const T* fe[3];
  const T* fh[3];
  SlabAxisD<T> slab[3];  // psi_h_in == psi_h_out
  int ichunk;
  const int2* xl;  // per x plane: (layer << 1 | slab) of the H (.x) / E (.y) layers, or -1
};

// CPML layer of coordinate x along a slab axis: the layer index, or -1, and
// the slab (0/1) in q.
template <typename T>
__device__ __forceinline__ int layer_of(const SlabAxisD<T>& A, int x, bool e_layers, int& q) {
  q = 0;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    if (s < A.count) {
      const int l = x - (e_layers ? A.e_lo[s] : A.h_lo[s]);
      if (l >= 0 && l < A.n[s]) {
        q = s;
        return l;
      }
    }
  }
  return -1;
}

// One psi cell of a slab: the update psi = b psi + a diff, in place.
template <typename T>
__device__ __forceinline__ T psi_step(T* ps, T b, T a, T diff) {
  const T v = b * *ps + a * diff;
  *ps = v;
  return v;
}

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__(TJ* TK) k_march_h(const __grid_constant__ MarchP<T> p) {
  const Lat L = p.L;
  const int k = blockIdx.x * TK + threadIdx.x;
  const int j = blockIdx.y * TJ + threadIdx.y;
  if (k > L.nz || j > L.ny) return;
  const int i_lo = blockIdx.z * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const bool jv = j < L.ny, kv = k < L.nz;
  const T fhj = jv ? p.fh[1][j] : T(0);
  const T fhk = kv ? p.fh[2][k] : T(0);

  // CPML normal to y (psi [i][l][k]) and z (psi [i][j][l]): fixed for the march.
  int qy, qz;
  const int ly = layer_of(p.slab[1], j, false, qy);
  const int lz = layer_of(p.slab[2], k, false, qz);
  T ay = 0, by = 0, az = 0, bz = 0;
  T* psy[2] = {nullptr, nullptr};
  T* psz[2] = {nullptr, nullptr};
  long long psy_st = 0, psz_st = 0;
  if (ly >= 0) {
    const SlabAxisD<T>& A = p.slab[1];
    ay = A.a_h[qy][ly];
    by = A.b_h[qy][ly];
    psy_st = (long long)A.n[qy] * KP;
    for (int w = 0; w < 2; ++w) psy[w] = A.psi_h_out[qy][w] + (long long)ly * KP + k;
  }
  if (lz >= 0) {
    const SlabAxisD<T>& A = p.slab[2];
    az = A.a_h[qz][lz];
    bz = A.b_h[qz][lz];
    psz_st = (long long)L.NY * A.n[qz];
    for (int w = 0; w < 2; ++w) psz[w] = A.psi_h_out[qz][w] + (long long)j * A.n[qz] + lz;
  }

  const T* __restrict__ Ex = p.f[0] + row;
  const T* __restrict__ Ey = p.f[1] + row;
  const T* __restrict__ Ez = p.f[2] + row;
  T* __restrict__ Hx = p.f[3] + row;
  T* __restrict__ Hy = p.f[4] + row;
  T* __restrict__ Hz = p.f[5] + row;
  T ey_c = Ey[i_lo * PS];  // E_y, E_z of plane i (carried)
  T ez_c = Ez[i_lo * PS];

  for (int i = i_lo; i < i_hi; ++i) {
    const long long o = i * PS;
    const bool iv = i < L.nx;
    const bool main_rng = iv && jv && kv;
    const T fhi = iv ? p.fh[0][i] : T(0);
    const T* r = p.tab + (size_t)p.cls[row + o] * 12 + 6;
    const T ex = Ex[o];
    const T ex_k = kv ? Ex[o + 1] : T(0);
    const T ex_j = jv ? Ex[o + KP] : T(0);
    const T ey_k = kv ? Ey[o + 1] : T(0);
    const T ez_j = jv ? Ez[o + KP] : T(0);
    T ey_n = T(0), ez_n = T(0);
    if (iv) {
      ey_n = Ey[o + PS];
      ez_n = Ez[o + PS];
    }
    const T dEy_k = ey_k - ey_c, dEz_j = ez_j - ez_c;  // Hx
    const T dEz_i = ez_n - ez_c, dEx_k = ex_k - ex;    // Hy
    const T dEx_j = ex_j - ex, dEy_i = ey_n - ey_c;    // Hz

    // CPML normal to x: uniform over the plane.
    int qx;
    const int lx = layer_of(p.slab[0], i, false, qx);

    if (jv && kv) {  // Hx: i <= nx, j < ny, k < nz
      const T ca = r[0], cb = r[1];
      T h = Hx[o];
      if (main_rng) h = ca * h + cb * (fhk * dEy_k - fhj * dEz_j);
      if (ly >= 0) h -= cb * psi_step(psy[1] + i * psy_st, by, ay, dEz_j);
      if (lz >= 0) h += cb * psi_step(psz[0] + i * psz_st, bz, az, dEy_k);
      Hx[o] = h;
    }
    if (iv && kv) {  // Hy: i < nx, j <= ny, k < nz
      const T ca = r[2], cb = r[3];
      T h = Hy[o];
      if (main_rng) h = ca * h + cb * (fhi * dEz_i - fhk * dEx_k);
      if (lx >= 0) {
        const SlabAxisD<T>& A = p.slab[0];
        h += cb * psi_step(A.psi_h_out[qx][0] + (long long)lx * PS + row, A.b_h[qx][lx],
                           A.a_h[qx][lx], dEz_i);
      }
      if (lz >= 0) h -= cb * psi_step(psz[1] + i * psz_st, bz, az, dEx_k);
      Hy[o] = h;
    }
    if (iv && jv) {  // Hz: i < nx, j < ny, k <= nz
      const T ca = r[4], cb = r[5];
      T h = Hz[o];
      if (main_rng) h = ca * h + cb * (fhj * dEx_j - fhi * dEy_i);
      if (lx >= 0) {
        const SlabAxisD<T>& A = p.slab[0];
        h -= cb * psi_step(A.psi_h_out[qx][1] + (long long)lx * PS + row, A.b_h[qx][lx],
                           A.a_h[qx][lx], dEy_i);
      }
      if (ly >= 0) h += cb * psi_step(psy[0] + i * psy_st, by, ay, dEx_j);
      Hz[o] = h;
    }
    ey_c = ey_n;
    ez_c = ez_n;
  }
}

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__(TJ* TK) k_march_e(const __grid_constant__ MarchP<T> p) {
  const Lat L = p.L;
  const int k = blockIdx.x * TK + threadIdx.x;
  const int j = blockIdx.y * TJ + threadIdx.y;
  if (k > L.nz || j > L.ny) return;
  const int i_lo = blockIdx.z * p.ichunk;
  const int i_hi = min(i_lo + p.ichunk, L.nx + 1);
  const long long PS = (long long)L.NY * L.KP;
  const int KP = L.KP;
  const long long row = (long long)j * KP + k;
  const bool jv = j < L.ny, kv = k < L.nz;
  const bool j1 = j >= 1, k1 = k >= 1;
  const bool jm = j1 && jv, km = k1 && kv;  // tangential main range along j, k
  const T fej = p.fe[1][j];
  const T fek = p.fe[2][k];

  int qy, qz;
  const int ly = layer_of(p.slab[1], j, true, qy);
  const int lz = layer_of(p.slab[2], k, true, qz);
  T ay = 0, by = 0, az = 0, bz = 0;
  T* psy[2] = {nullptr, nullptr};
  T* psz[2] = {nullptr, nullptr};
  long long psy_st = 0, psz_st = 0;
  if (ly >= 0) {
    const SlabAxisD<T>& A = p.slab[1];
    ay = A.a_e[qy][ly];
    by = A.b_e[qy][ly];
    psy_st = (long long)A.n[qy] * KP;
    for (int w = 0; w < 2; ++w) psy[w] = A.psi_e[qy][w] + (long long)ly * KP + k;
  }
  if (lz >= 0) {
    const SlabAxisD<T>& A = p.slab[2];
    az = A.a_e[qz][lz];
    bz = A.b_e[qz][lz];
    psz_st = (long long)L.NY * A.n[qz];
    for (int w = 0; w < 2; ++w) psz[w] = A.psi_e[qz][w] + (long long)j * A.n[qz] + lz;
  }

  T* __restrict__ Ex = p.f[0] + row;
  T* __restrict__ Ey = p.f[1] + row;
  T* __restrict__ Ez = p.f[2] + row;
  const T* __restrict__ Hx = p.f[3] + row;
  const T* __restrict__ Hy = p.f[4] + row;
  const T* __restrict__ Hz = p.f[5] + row;
  // H_y, H_z of plane i-1 (carried)
  T hy_p = i_lo >= 1 ? Hy[(i_lo - 1) * PS] : T(0);
  T hz_p = i_lo >= 1 ? Hz[(i_lo - 1) * PS] : T(0);

  for (int i = i_lo; i < i_hi; ++i) {
    const long long o = i * PS;
    const bool iv = i < L.nx, i1 = i >= 1;
    const bool im = i1 && iv;
    const T fei = p.fe[0][i];
    const T* r = p.tab + (size_t)p.cls[row + o] * 12;
    const T hx = Hx[o], hy = Hy[o], hz = Hz[o];
    const T hx_k = k1 ? Hx[o - 1] : T(0);
    const T hx_j = j1 ? Hx[o - KP] : T(0);
    const T hy_k = k1 ? Hy[o - 1] : T(0);
    const T hz_j = j1 ? Hz[o - KP] : T(0);
    const T dHz_j = hz - hz_j, dHy_k = hy - hy_k;  // Ex
    const T dHx_k = hx - hx_k, dHz_i = hz - hz_p;  // Ey
    const T dHy_i = hy - hy_p, dHx_j = hx - hx_j;  // Ez

    int qx;
    const int lx = layer_of(p.slab[0], i, true, qx);

    if (iv) {  // Ex: i < nx, j <= ny, k <= nz; main 1 <= j < ny, 1 <= k < nz
      const T ca = r[0], cb = r[1];
      T e = Ex[o];
      if (jm && km) e = ca * e + cb * (fej * dHz_j - fek * dHy_k);
      if (ly >= 0) e += cb * psi_step(psy[1] + i * psy_st, by, ay, dHz_j);
      if (lz >= 0) e -= cb * psi_step(psz[0] + i * psz_st, bz, az, dHy_k);
      Ex[o] = e;
    }
    if (jv) {  // Ey: j < ny; main 1 <= i < nx, 1 <= k < nz
      const T ca = r[2], cb = r[3];
      T e = Ey[o];
      if (im && km) e = ca * e + cb * (fek * dHx_k - fei * dHz_i);
      if (lx >= 0) {
        const SlabAxisD<T>& A = p.slab[0];
        e -= cb * psi_step(A.psi_e[qx][0] + (long long)lx * PS + row, A.b_e[qx][lx],
                           A.a_e[qx][lx], dHz_i);
      }
      if (lz >= 0) e += cb * psi_step(psz[1] + i * psz_st, bz, az, dHx_k);
      Ey[o] = e;
    }
    if (kv) {  // Ez: k < nz; main 1 <= i < nx, 1 <= j < ny
      const T ca = r[4], cb = r[5];
      T e = Ez[o];
      if (im && jm) e = ca * e + cb * (fei * dHy_i - fej * dHx_j);
      if (lx >= 0) {
        const SlabAxisD<T>& A = p.slab[0];
        e += cb * psi_step(A.psi_e[qx][1] + (long long)lx * PS + row, A.b_e[qx][lx],
                           A.a_e[qx][lx], dHy_i);
      }
      if (ly >= 0) e -= cb * psi_step(psy[0] + i * psy_st, by, ay, dHx_j);
      Ez[o] = e;
    }
    hy_p = hy;
    hz_p = hz;
  }
}

}  // namespace xfd
