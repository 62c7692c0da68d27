// NF2FF far-field potentials from the accumulated frequency-domain surface
// currents, on the GPU: FDPlaneData::getPotential / calculatePotential
// (src/nffft/nffft_fd_data_process.cpp:15-144), called per frequency by
// NFFFTFrequencyDomain::processFarField (src/nffft/nffft_frequency_domain.cpp:103-129).
//
// For frequency f, angle (theta, phi) and potential
//   A_theta = sum_faces sum_points (J_a T_theta[a] + J_b T_theta[b]) e^{i k r.rhat} ds
//   F_phi   = same with M and T_phi,  A_phi: J and T_phi,  F_theta: M and T_theta,
// where a, b are the face's tangential axes, T the theta-hat / phi-hat
// components of the Cartesian unit vectors (cCSToSCSTransformMatrix,
// include/xfdtd/util/transform.h:25-59), r the face-centre position minus the
// origin (rVector, nffft_fd_data_process.cpp:185-200) and ds the face-cell
// area (nffft_fd_data_process.cpp:202-215).  One CTA per (angle, frequency)
// sums all surface points: per point one complex exponential and four
// complex multiply-adds, FP64 throughout, then a tree reduction.
#pragma once

#include <cuda_runtime.h>

namespace xfd {

struct FarFieldD {
  int nf, n_ang;
  long long P;               // surface points (all faces)
  long long begin[7];        // first point of each face; begin[6] = P
  int s[6][3], e[6][3];      // face boxes [s, e)
  const double2* acc;        // (nf * 4) x P: J_a, J_b, M_a, M_b per frequency
  const double2* comp;       // same shape: compensation terms, value = acc + comp
  const double* k0;          // nf: wave numbers 2 pi f / c
  const double* ang;         // n_ang x 8: T_theta[x,y,z], T_phi[x,y,z], st*cp, st*sp
  const double* cos_t;       // n_ang
  const double* node_e[3];   // e-node coordinates (n+1) per axis
  const double* node_h[3];   // cell-centre coordinates (n) per axis
  const double* size_e[3];   // cell sizes (n) per axis
  double origin[3];
  double2* out;              // nf x 4 x n_ang: a_theta, f_phi, a_phi, f_theta
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(256) k_far_field(const __grid_constant__ FarFieldD d) {
  const int ang = blockIdx.x, f = blockIdx.y;
  const double* T = d.ang + (long long)ang * 8;
  const double stcp = T[6], stsp = T[7], ct = d.cos_t[ang];
  const double k0 = d.k0[f];
  double2 acc[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) acc[r] = make_double2(0.0, 0.0);
  const double2* J = d.acc + (long long)f * 4 * d.P;
  const double2* Jc = d.comp + (long long)f * 4 * d.P;
  auto cur = [&](long long o) {
    const double2 a = J[o], c = Jc[o];
    return make_double2(a.x + c.x, a.y + c.y);
  };
  for (long long p = threadIdx.x; p < d.P; p += blockDim.x) {
    int face = 0;
    while (face < 5 && p >= d.begin[face + 1]) ++face;
    long long r = p - d.begin[face];
    const int* s = d.s[face];
    const int* e = d.e[face];
    const int e2 = e[2] - s[2], e1 = e[1] - s[1];
    const int x[3] = {s[0] + (int)(r / ((long long)e1 * e2)), s[1] + (int)((r / e2) % e1),
                      s[2] + (int)(r % e2)};
    const int m = face / 2, A = (m + 1) % 3, B = (m + 2) % 3;
    double pos[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      pos[a] = (a == m ? d.node_e[a][x[a]] : d.node_h[a][x[a]]) - d.origin[a];
    const double ds = d.size_e[A][x[A]] * d.size_e[B][x[B]];
    const double arg = pos[0] * stcp + pos[1] * stsp + pos[2] * ct;
    double sn, cs;
    sincos(k0 * arg, &sn, &cs);
    const double2 ph = make_double2(cs, sn);
    const double2 ja = cur(p), jb = cur(d.P + p), ma = cur(2 * d.P + p), mb = cur(3 * d.P + p);
    const double tta = T[A], ttb = T[B], tpa = T[3 + A], tpb = T[3 + B];
    // rows: a_theta (J, theta), f_phi (M, phi), a_phi (J, phi), f_theta (M, theta)
    const double2 src[4] = {
        make_double2(ja.x * tta + jb.x * ttb, ja.y * tta + jb.y * ttb),
        make_double2(ma.x * tpa + mb.x * tpb, ma.y * tpa + mb.y * tpb),
        make_double2(ja.x * tpa + jb.x * tpb, ja.y * tpa + jb.y * tpb),
        make_double2(ma.x * tta + mb.x * ttb, ma.y * tta + mb.y * ttb)};
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) {
      const double2 v = cmul(src[rr], ph);
      acc[rr].x += v.x * ds;
      acc[rr].y += v.y * ds;
    }
  }
  // Tree reduction: warps, then the CTA.
  __shared__ double2 red[8][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    for (int o = 16; o > 0; o >>= 1) {
      acc[rr].x += __shfl_down_sync(0xffffffffu, acc[rr].x, o);
      acc[rr].y += __shfl_down_sync(0xffffffffu, acc[rr].y, o);
    }
    if (lane == 0) red[wid][rr] = acc[rr];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int rr = threadIdx.x;
    double2 v = red[0][rr];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      v.x += red[w][rr].x;
      v.y += red[w][rr].y;
    }
    d.out[((long long)f * 4 + rr) * d.n_ang + ang] = v;
  }
}

}  // namespace xfd
