// Allocation-free NF2FF step: xfd_nf2ff_step_static.
//
// The engine's NF2FF path samples the tangential surface fields of every
// time step into a sample buffer it allocates at set-up, then folds those
// samples into the frequency-domain surface currents (k_nf2ff_sample and
// k_nf2ff_dft in kernels.cuh).  This file holds a variant of that pair for
// callers that cannot allocate device memory: an FDTD time loop embedded in
// a larger GPU application that owns all device memory through its own pool
// or a fixed arena, where an extra cudaMalloc either fails because the pool
// has already claimed the memory or synchronises the whole device in the
// middle of the caller's time loop.  Such a caller passes its own field
// arrays, phasor tables and accumulator; the one piece of scratch the step
// needs -- the four signed surface values of every Huygens point for this
// step -- lives in g_nf2ff_scratch below, a fixed array every GPU that loads
// the library holds until the process exits.
//
// The arithmetic follows the engine's kernels and the reference:
// calculateJ / calculateM (src/nffft/nffft_fd_data_update.cpp:22-122) with
// interpolateSurfaceCenter (src/include/nffft/interpolate_scheme.h:19-138) for
// the samples, and the running DFT with the per-step phasors of
// FDPlaneData::initDFT (src/nffft/nffft_fd_data.cpp:65-76), one step per call.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "xfd_engine.h"

// Sets the message xfd_last_error(NULL) returns (engine.cu).
extern "C" void xfd_internal_set_error(const char* msg);

namespace {

constexpr int kMaxPoints = XFD_NF2FF_STATIC_MAX_POINTS;
constexpr int kMaxDevices = 64;

// Four signed surface values (J_a, J_b, M_a, M_b) per Huygens point for the
// step being folded: [4][P] doubles.  Every call writes each entry it reads
// before reading it, so nothing here has to start at zero.
static __device__ __align__(256) double g_nf2ff_scratch[4 * kMaxPoints];

std::mutex g_mu;
// Device address of the scratch array per device, with the CUDA context it
// was looked up in: a cudaDeviceReset ends that context, and the next call
// (in a new context) looks the address up again.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  double* addr = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];

// Unique id of the calling thread's current context (cuCtxGetId, through the
// runtime's driver entry point: this library links only the runtime).
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
bool current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    looked_up = true;
  }
  void* ctx = nullptr;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx) return false;
  return get_id(ctx, id) == 0;
}

struct FieldView {
  const void* f[6];
  long long si[6], sj[6];  // element strides along i and j (k is contiguous)
};

struct Faces {
  int s[6][3], e[6][3];
  long long begin[7];  // first point of each face; begin[6] = P
};

template <typename T>
__device__ __forceinline__ double at(const FieldView& v, int c, int i, int j, int k) {
  return (double)static_cast<const T*>(v.f[c])[(long long)i * v.si[c] + (long long)j * v.sj[c] + k];
}

// E component `comp` at the centre of the face cell (i, j, k) normal to m.
template <typename T>
__device__ double surf_e(const FieldView& v, int m, int comp, int i, int j, int k) {
  int q[3] = {i, j, k};
  q[3 - m - comp] += 1;
  return 0.5 * (at<T>(v, comp, q[0], q[1], q[2]) + at<T>(v, comp, i, j, k));
}

// H component `comp` at the centre of the face cell (i, j, k) normal to m.
template <typename T>
__device__ double surf_h(const FieldView& v, int m, int comp, int i, int j, int k) {
  const int c = 3 + comp;
  if (m == 0) {
    int p1[3] = {i, j, k};
    p1[comp] += 1;
    return 0.25 * (at<T>(v, c, p1[0], p1[1], p1[2]) + at<T>(v, c, i, j, k) +
                   at<T>(v, c, p1[0] - 1, p1[1], p1[2]) + at<T>(v, c, i - 1, j, k));
  }
  if (m == 1) {
    if (comp == 2)
      return 0.25 * (at<T>(v, c, i, j, k + 1) + at<T>(v, c, i, j, k) +
                     at<T>(v, c, i, j - 1, k + 1) + at<T>(v, c, i, j - 1, k));
    return 0.25 * (at<T>(v, c, i + 1, j, k) + at<T>(v, c, i, j, k) +
                   at<T>(v, c, i + 1, j - 1, k) + at<T>(v, c, i, j - 1, k));
  }
  if (comp == 0)
    return 0.25 * (at<T>(v, c, i + 1, j, k) + at<T>(v, c, i, j, k) + at<T>(v, c, i, j, k - 1) +
                   at<T>(v, c, i + 1, j, k - 1));
  return 0.25 * (at<T>(v, c, i, j, k) + at<T>(v, c, i, j + 1, k) + at<T>(v, c, i, j, k - 1) +
                 at<T>(v, c, i, j + 1, k - 1));
}

// One thread per Huygens point: the four signed surface values into scratch.
template <typename T>
__global__ void k_nf2ff_sample_static(FieldView v, Faces fc, double* scratch) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long P = fc.begin[6];
  if (p >= P) return;
  int d = 0;
  while (d < 5 && p >= fc.begin[d + 1]) ++d;
  long long r = p - fc.begin[d];
  const int* s = fc.s[d];
  const int* e = fc.e[d];
  const int e2 = e[2] - s[2], e1 = e[1] - s[1];
  const int k = s[2] + (int)(r % e2);
  r /= e2;
  const int j = s[1] + (int)(r % e1);
  r /= e1;
  const int i = s[0] + (int)r;
  const int m = d / 2;
  const bool positive = (d % 2) == 1;
  const int A = (m + 1) % 3, B = (m + 2) % 3;
  const double cj1 = positive ? -1.0 : 1.0, cj2 = positive ? 1.0 : -1.0;
  double* out = scratch + p;
  out[0] = cj1 * surf_h<T>(v, m, B, i, j, k);
  out[P] = cj2 * surf_h<T>(v, m, A, i, j, k);
  out[2 * P] = -cj1 * surf_e<T>(v, m, B, i, j, k);
  out[3 * P] = -cj2 * surf_e<T>(v, m, A, i, j, k);
}

// s + x rounded into s, its exact rounding error (Knuth's TwoSum) added to c.
__device__ __forceinline__ void two_sum_acc(double& s, double& c, double x) {
  const double t = __dadd_rn(s, x);
  const double bp = __dsub_rn(t, s);
  c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, __dsub_rn(t, bp)), __dsub_rn(x, bp)));
  s = t;
}

// One thread per (q, p): acc[f][q][p] += scale * sample[q][p] * phasor_q[f][t]
// (J currents q = 0, 1 take the H-time phasors th, M currents q = 2, 3 te);
// with `comp` the addition is compensated (acc + comp is the sum).
__global__ void k_nf2ff_dft_static(const double* scratch, long long P, int nf,
                                   const double2* te, const double2* th, long long n_steps,
                                   long long t, double scale, double2* acc, double2* comp) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 4 * P) return;
  const int q = (int)(tid / P);
  const long long p = tid - q * P;
  const double v = scratch[q * P + p];
  const double2* ph = q < 2 ? th : te;
  for (int f = 0; f < nf; ++f) {
    const double2 z = ph[(long long)f * n_steps + t];
    const long long o = ((long long)f * 4 + q) * P + p;
    double2 w = acc[o];
    if (comp) {
      double2 c = comp[o];
      two_sum_acc(w.x, c.x, __dmul_rn(scale, __dmul_rn(v, z.x)));
      two_sum_acc(w.y, c.y, __dmul_rn(scale, __dmul_rn(v, z.y)));
      comp[o] = c;
    } else {
      w.x += scale * (v * z.x);
      w.y += scale * (v * z.y);
    }
    acc[o] = w;
  }
}

xfd_status fail(xfd_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  xfd_internal_set_error(buf);
  return s;
}

// The device address of the scratch array on the current device.  The
// array's name in host code is only a host-side handle, so the address is
// looked up once per device and context (with that device current) and kept.
xfd_status scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t c = cudaGetDevice(&dev);
  if (c != cudaSuccess) return fail(XFD_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(c));
  if (dev < 0 || dev >= kMaxDevices) return fail(XFD_ERR_UNSUPPORTED, "device %d", dev);
  // Make the device's primary context current (since CUDA 12 cudaSetDevice
  // initialises it), so that the context id below is the one the launches
  // will use.
  c = cudaSetDevice(dev);
  if (c != cudaSuccess) return fail(XFD_ERR_CUDA, "CUDA context: %s", cudaGetErrorString(c));
  unsigned long long ctx = 0;
  const bool have_ctx = current_context_id(&ctx);
  std::lock_guard<std::mutex> lock(g_mu);
  ScratchAddr& a = g_scratch_addr[dev];
  if (!a.addr || !have_ctx || a.ctx_id != ctx) {
    void* p = nullptr;
    c = cudaGetSymbolAddress(&p, g_nf2ff_scratch);
    if (c != cudaSuccess || !p)
      return fail(XFD_ERR_CUDA, "cudaGetSymbolAddress(NF2FF scratch): %s", cudaGetErrorString(c));
    a.addr = static_cast<double*>(p);
    a.ctx_id = have_ctx ? ctx : 0;
  }
  *out = a.addr;
  return XFD_OK;
}

}  // namespace

extern "C" xfd_status xfd_nf2ff_step_static(const xfd_nf2ff_step_desc* d, void* stream) {
  if (!d) return fail(XFD_ERR_INVALID_ARGUMENT, "null NF2FF step descriptor");
  const int n[3] = {d->nx, d->ny, d->nz};
  if (n[0] < 1 || n[1] < 1 || n[2] < 1) return fail(XFD_ERR_INVALID_ARGUMENT, "bad grid size");
  if (d->precision != XFD_FP64 && d->precision != XFD_FP32)
    return fail(XFD_ERR_INVALID_ARGUMENT, "bad precision %d", d->precision);
  if (d->n_freq < 1 || d->n_freq > XFD_NF2FF_STATIC_MAX_FREQ)
    return fail(XFD_ERR_INVALID_ARGUMENT, "n_freq %d outside 1..%d", d->n_freq,
                XFD_NF2FF_STATIC_MAX_FREQ);
  if (d->n_steps < 1 || d->step < 0 || d->step >= d->n_steps)
    return fail(XFD_ERR_INVALID_ARGUMENT, "step %lld outside 0..%lld", (long long)d->step,
                (long long)d->n_steps - 1);
  if (!d->te || !d->th || !d->acc) return fail(XFD_ERR_INVALID_ARGUMENT, "null phasors/acc");
  FieldView v{};
  for (int c = 0; c < 6; ++c) {
    if (!d->fields[c]) return fail(XFD_ERR_INVALID_ARGUMENT, "null field %d", c);
    // Reference component shapes: E_c has n along c and n+1 across,
    // H_c has n+1 along c and n across.
    long long dim[3];
    for (int a = 0; a < 3; ++a)
      dim[a] = c < 3 ? n[a] + (a != c ? 1 : 0) : n[a] + (a == c - 3 ? 1 : 0);
    v.f[c] = d->fields[c];
    v.sj[c] = dim[2];
    v.si[c] = dim[1] * dim[2];
  }
  Faces fc{};
  long long total = 0;
  for (int f = 0; f < 6; ++f) {
    fc.begin[f] = total;
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      fc.s[f][a] = d->task_s[f][a];
      fc.e[f][a] = d->task_e[f][a];
      if (fc.e[f][a] <= fc.s[f][a]) empty = true;
    }
    if (empty) {
      for (int a = 0; a < 3; ++a) fc.s[f][a] = fc.e[f][a] = 0;
      continue;
    }
    for (int a = 0; a < 3; ++a)
      if (fc.s[f][a] < 1 || fc.e[f][a] > n[a])  // stencils read one node either side
        return fail(XFD_ERR_INVALID_ARGUMENT, "NF2FF face %d out of range", f);
    total += (long long)(fc.e[f][0] - fc.s[f][0]) * (fc.e[f][1] - fc.s[f][1]) *
             (fc.e[f][2] - fc.s[f][2]);
  }
  fc.begin[6] = total;
  if (total > kMaxPoints)
    return fail(XFD_ERR_UNSUPPORTED,
                "NF2FF surface of %lld points exceeds the static scratch (%d points)", total,
                kMaxPoints);
  if (total == 0) return XFD_OK;
  double* scratch = nullptr;
  xfd_status st = scratch_on_current_device(&scratch);
  if (st != XFD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned g1 = (unsigned)((total + 255) / 256);
  if (d->precision == XFD_FP64)
    k_nf2ff_sample_static<double><<<g1, 256, 0, s>>>(v, fc, scratch);
  else
    k_nf2ff_sample_static<float><<<g1, 256, 0, s>>>(v, fc, scratch);
  const unsigned g2 = (unsigned)((4 * total + 255) / 256);
  k_nf2ff_dft_static<<<g2, 256, 0, s>>>(scratch, total, d->n_freq,
                                         reinterpret_cast<const double2*>(d->te),
                                         reinterpret_cast<const double2*>(d->th), d->n_steps,
                                         d->step, d->scale, reinterpret_cast<double2*>(d->acc),
                                         reinterpret_cast<double2*>(d->acc_comp));
  cudaError_t c = cudaGetLastError();
  if (c != cudaSuccess) return fail(XFD_ERR_CUDA, "NF2FF step launch: %s", cudaGetErrorString(c));
  return XFD_OK;
}
