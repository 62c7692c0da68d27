// C-ABI implementation of the B200 FDTD engine (include/xfd_engine.h).
//
// One engine = one simulation on one GPU.  The host hands over FP64 set-up
// data; the engine converts it to its precision (fields, class table, curl
// factors, CPML and ADE state in FP32 or FP64; TFSF tables, lumped sources and
// NF2FF phasors/accumulators always FP64), keeps everything resident in HBM
// and runs the time loop on one stream, captured into CUDA graphs of whole
// step chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "fused.cuh"
#include "fused_tma.cuh"
#include "march.cuh"
#include "march_tma.cuh"
#include "march_wide.cuh"
#include "fmarch.cuh"
#include "fvec.cuh"
#include "hyb.cuh"
#include "farfield.cuh"
#include "kernels.cuh"
#include "adjoint.cuh"
#include "xfd_engine.h"

using namespace xfd;

namespace {

thread_local std::string g_create_error;

struct MovieH {
  MovieD d;
  long long n_nodes;
  long long copied;  // frames already queued for copy-out to `host`
  void* host;        // pinned host frame store (max_frames x n_nodes)
};

struct LumpedH {
  int comp;
  std::vector<long long> node;
  std::vector<double> coff;
  std::vector<double> wave;
};

}  // namespace

constexpr int kSides = 4;  // side streams of the TMA marching sweeps

struct xfd_engine {
  int device = 0;
  int precision = XFD_FP64;
  size_t wsize = 8;
  Lat L{};
  long long n_lat = 0;  // NX * NY * KP
  int64_t n_steps = 0;
  double dt = 0;
  std::string err;
  cudaStream_t stream = nullptr;

  std::vector<void*> allocs;
  void* fbuf[2][6] = {};          // ping-pong field buffers
  void** d_fields[2] = {};        // device arrays of the 6 field pointers per buffer
  int cur = 0;                    // buffer holding the current fields
  uint16_t* cls = nullptr;
  void* tab = nullptr;
  int n_classes = 0;
  void* fe[3] = {};
  void* fh[3] = {};
  std::vector<double> fe_h[3], fh_h[3];  // host copies (fh padded to n+1)
  bool have_classes = false, have_curl = false;

  struct Slab {
    int m, neg, n, e_lo, h_lo;
    void *a_e, *b_e, *a_h, *b_h;
    void* psi_e[2];     // [component A / B]
    void* psi_h[2][2];  // [buffer][component A / B]; follows the field buffer
  };
  std::vector<Slab> slabs;

  bool have_tfsf = false;
  TfsfD tfsf{};
  TfsfGroupD tfsf_groups[4]{};  // H group 1, H group 2, E group 1, E group 2
  TfsfHD tfsf_h{};              // H passes per component for the fused sweep

  std::vector<LumpedH> lumped_h;
  LumpedD lumped{};
  bool lumped_dirty = false;

  // lumped inductors: host lists, device list with its FP64 current state
  struct InductorH {
    int comp;
    std::vector<long long> node;
    std::vector<double> cecjc, cjcec;
  };
  std::vector<InductorH> ind_h;
  InductorD ind{};
  bool ind_dirty = false;

  // per-node E coefficient overrides (device list + host copy for the adjoint)
  long long n_ovr = 0;
  OverrideD<double> ovr64{};
  OverrideD<float> ovr32{};
  std::vector<int32_t> ovr_node;  // 3 per entry
  std::vector<uint8_t> ovr_comp;
  std::vector<double> ovr_ca, ovr_cb;
  long long n_hterm = 0;  // H curl-term corrections (xfd_set_h_term_overrides)
  HTermD<double> hterm64{};
  HTermD<float> hterm32{};

  int ade_kind = -1;
  AdeD<double> ade64{};
  AdeD<float> ade32{};

  bool have_nf2ff = false;
  Nf2ffD nf2ff{};
  bool have_td = false;  // time-domain NF2FF
  Nf2ffTdD td{};
  // weighted probes: host lists, device copy rebuilt when one is added
  std::vector<long long> pr_begin{0};
  std::vector<long long> pr_node;
  std::vector<uint8_t> pr_comp;
  std::vector<double> pr_w;
  ProbeD probes{};
  bool probes_dirty = false;
  long long nf_sampled_since_flush = 0;
  long long nf_last_flush_step = 0;

  std::vector<MovieH> movies;

  long long* d_step = nullptr;
  int* d_err = nullptr;
  int64_t host_step = 0;

  // monitor copy-out: D2H of finished frames on a side stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ev = nullptr;
  // Side streams of the TMA marching sweeps: the CPML-free box and the
  // lattice-face kernel run beside the CPML form (disjoint nodes), forked
  // from and joined back into `stream` (also inside graph capture).
  cudaStream_t side[kSides]{};
  cudaEvent_t fork_ev = nullptr, join_ev[kSides]{};
  cudaEvent_t halo_ev = nullptr;  // xfd_halo_copy: this engine's queued work
  bool march_concurrent = true;
  std::vector<void*> host_allocs;

  // graph
  bool use_graph = true;
  int graph_chunk = 32;
  // 0 split, 1 fused, 2 fused + TMA, 3 split marching, 4 split marching + TMA,
  // 5 fused marching (overlapped tiles) + TMA, 6 = 5 with a two-nodes-per-
  // thread form on the CPML-free interior, 7 fused H-then-E TMA sweep of the
  // CPML-free interior box with the split marching forms on the CPML tiles
  // (ping-pong buffers)
  int kernel_mode = 7;
  int ichunk = 32;
  int march_ichunk = 16;  // planes per CTA of the marching split sweeps
  bool pdl = true;        // sweep 0: programmatic dependent launch
  // Cycles a TMA-staged sweep's stage wait may take before the CTA gives up
  // (error bit 2, XFD_ERR_TIMEOUT at the next sync); 0: about 2 s.
  long long stage_wait = 0;
  // NaN / Inf watchdog: every `watchdog` steps a scan of the six fields sets
  // error bit 4 (XFD_ERR_NUMERIC at the next sync) on a non-finite value; 0: off.
  long long watchdog = 0;
  bool tma_ready = false;
  TmaMaps tma[2]{};       // tensor maps over buffer 0 / 1 (and the class index)
  MarchMaps mtma[2]{};    // tensor maps of the TMA marching sweeps
  MarchMaps mtma_w[2]{};  // and of their two-rows-per-thread interior form
  bool march_wide = false;  // sweep the interior box with k_march_*_wide
  // Tile lists of the CPML form, by the CPML axes their tiles meet: x only,
  // y only, z only, several (lists 0..3 at mt_off[q] .. mt_off[q+1]).
  bool march_split_axes = true;
  // Stages of the single-axis CPML lists: 0 as the general CPML form, 1 as
  // the CPML-free forms (less shared memory, more CTAs per SM).
  int march_cp_stages = 1;
  // Shift the tile grid to fit the CPML layers.  Off by default: a k shift
  // that is not a multiple of 32 values leaves every tile row off the 128-byte
  // lines (TMA boxes and the warps' stores), which costs more than the larger
  // CPML-free box gains.
  bool march_shift = false;
  int4* d_mtiles = nullptr;
  size_t mtiles_cap = 0;
  int mt_off[5] = {0, 0, 0, 0, 0};
  long long mtiles_key = -1;
  int2* d_xlayer = nullptr;  // per x plane: CPML layer code of the H / E layers
  size_t xlayer_slabs = (size_t)-1;  // slab count the table was built for
  HybMaps hmaps[2]{};     // tensor maps of the fused interior sweep (sweep 7), by input buffer
  // Its box tiles, one CTA each.
  int4* d_hyb_tiles = nullptr;
  size_t hyb_tiles_cap = 0;
  int n_hyb_tiles = 0;
  long long hyb_key = -1;
  FmarchMaps fmaps[2]{};  // tensor maps of the fused marching sweep
  FvecMaps fvmaps[2]{};   // tensor maps of its two-nodes-per-thread interior form
  cudaGraphExec_t graph_exec = nullptr;
  int graph_cur = -1;
  long long graph_len = 0;
  bool graph_dirty = true;

  // Saved states (xfd_checkpoint_*): one device buffer per slot.
  struct Ckpt {
    void* buf = nullptr;
    size_t bytes = 0;
    int64_t step = -1;
  };
  std::vector<Ckpt> ckpts;
  // Device buffers and saved states of the last adjoint run, kept for the
  // next run (reused in allocation order while the sizes match).
  std::vector<void*> adj_bufs;
  std::vector<size_t> adj_sizes;
  std::vector<Ckpt> adj_ck;
  // Per-step node-box records of the adjoint (objective field, design
  // history), launched after the record phase of each step.
  BoxRecD<double> rec64[2]{};
  BoxRecD<float> rec32[2]{};
  int n_rec = 0;
};

namespace {

xfd_status fail(xfd_engine* e, xfd_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (e) e->err = buf;
  else g_create_error = buf;
  return s;
}

#define CUDA_TRY(e, call)                                                                   \
  do {                                                                                      \
    cudaError_t _c = (call);                                                                \
    if (_c != cudaSuccess)                                                                  \
      return fail((e), XFD_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_c));      \
  } while (0)

xfd_status dev_alloc(xfd_engine* e, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t c = cudaMalloc(p, bytes);
  if (c != cudaSuccess) {
    *p = nullptr;
    return fail(e, c == cudaErrorMemoryAllocation ? XFD_ERR_OUT_OF_MEMORY : XFD_ERR_CUDA,
                "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(c));
  }
  e->allocs.push_back(*p);
  c = cudaMemsetAsync(*p, 0, bytes, e->stream);
  if (c != cudaSuccess) return fail(e, XFD_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(c));
  return XFD_OK;
}

// Uploads `n` doubles, converted to the engine precision.
xfd_status upload_real(xfd_engine* e, void** dst, const double* src, size_t n) {
  xfd_status s = dev_alloc(e, dst, n * e->wsize);
  if (s != XFD_OK) return s;
  if (n == 0) return XFD_OK;
  if (e->precision == XFD_FP64) {
    CUDA_TRY(e, cudaMemcpyAsync(*dst, src, n * 8, cudaMemcpyHostToDevice, e->stream));
  } else {
    std::vector<float> tmp(src, src + n);
    CUDA_TRY(e, cudaMemcpyAsync(*dst, tmp.data(), n * 4, cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  }
  return XFD_OK;
}

template <typename U>
xfd_status upload_raw(xfd_engine* e, U** dst, const U* src, size_t n) {
  void* p = nullptr;
  xfd_status s = dev_alloc(e, &p, n * sizeof(U));
  if (s != XFD_OK) return s;
  *dst = static_cast<U*>(p);
  if (n) CUDA_TRY(e, cudaMemcpyAsync(p, src, n * sizeof(U), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

// Extent of component c (0..5) in the reference shape.
void comp_shape(const Lat& L, int c, int out[3]) {
  const int n[3] = {L.nx, L.ny, L.nz};
  const int ax = c % 3;
  const bool is_e = c < 3;
  for (int d = 0; d < 3; ++d) {
    if (is_e) out[d] = (d == ax) ? n[d] : n[d] + 1;
    else out[d] = (d == ax) ? n[d] + 1 : n[d];
  }
}

cudaMemcpy3DParms copy_parms(const xfd_engine* e, int c, void* dev, void* host, bool to_dev,
                             size_t elem) {
  int shp[3];
  comp_shape(e->L, c, shp);
  cudaMemcpy3DParms p{};
  cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)shp[2] * elem, (size_t)shp[2],
                                          (size_t)shp[1]);
  cudaPitchedPtr dp = make_cudaPitchedPtr(dev, (size_t)e->L.KP * elem, (size_t)e->L.KP,
                                          (size_t)e->L.NY);
  p.extent = make_cudaExtent((size_t)shp[2] * elem, (size_t)shp[1], (size_t)shp[0]);
  if (to_dev) {
    p.srcPtr = hp;
    p.dstPtr = dp;
    p.kind = cudaMemcpyHostToDevice;
  } else {
    p.srcPtr = dp;
    p.dstPtr = hp;
    p.kind = cudaMemcpyDeviceToHost;
  }
  return p;
}

inline bool is_fused(const xfd_engine* e) {
  return e->kernel_mode == 1 || e->kernel_mode == 2 || e->kernel_mode == 5 ||
         e->kernel_mode == 6;
}
// Sweeps whose step reads one field buffer and writes the other.
inline bool is_pingpong(const xfd_engine* e) { return is_fused(e) || e->kernel_mode == 7; }
inline bool uses_tma(const xfd_engine* e) {
  return e->kernel_mode == 2 || e->kernel_mode == 4 || e->kernel_mode == 5 ||
         e->kernel_mode == 6 || e->kernel_mode == 7;
}
// The CPML H psi buffer the next step reads: the fused sweeps ping-pong it
// with the fields; sweep 7 updates it in place (the split CPML forms) and
// keeps it in buffer 0; the in-place sweeps use the field buffer's.
inline int psi_h_buf(const xfd_engine* e) { return e->kernel_mode == 7 ? 0 : e->cur; }

template <typename T>
YeeP<T> yee_params(xfd_engine* e) {
  YeeP<T> p{};
  p.L = e->L;
  for (int c = 0; c < 6; ++c) p.f[c] = static_cast<T*>(e->fbuf[e->cur][c]);
  p.cls = e->cls;
  p.tab = static_cast<const T*>(e->tab);
  for (int a = 0; a < 3; ++a) {
    p.fe[a] = static_cast<const T*>(e->fe[a]);
    p.fh[a] = static_cast<const T*>(e->fh[a]);
  }
  p.n_slab = (int)e->slabs.size();
  for (size_t s = 0; s < e->slabs.size(); ++s) {
    const auto& S = e->slabs[s];
    auto& D = p.slab[s];
    D.m = S.m;
    D.n = S.n;
    D.e_lo = S.e_lo;
    D.h_lo = S.h_lo;
    D.a_e = static_cast<const T*>(S.a_e);
    D.b_e = static_cast<const T*>(S.b_e);
    D.a_h = static_cast<const T*>(S.a_h);
    D.b_h = static_cast<const T*>(S.b_h);
    for (int w = 0; w < 2; ++w) {
      D.psi_e[w] = static_cast<T*>(S.psi_e[w]);
      D.psi_h[w] = static_cast<T*>(S.psi_h[psi_h_buf(e)][w]);
    }
  }
  return p;
}

unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

constexpr int kTJ = 8, kTK = 32;

constexpr int kStagesF32 = 4, kStagesF64 = 3;
constexpr int kMarchStagesF32 = 6, kMarchStagesF64 = 4;
constexpr int kMTJ = 8;  // rows (warps) per CTA of the TMA marching sweeps
template <typename T>
__host__ __device__ constexpr int march_stages() {
  return sizeof(T) == 8 ? kMarchStagesF64 : kMarchStagesF32;
}
// The CPML-free forms need fewer registers, so they run more CTAs per SM;
// fewer stages keep their shared memory from capping that.
template <typename T>
__host__ __device__ constexpr int march_free_stages() { return sizeof(T) == 8 ? 3 : 4; }
// Stages of the two-rows-per-thread interior form (3 CTAs per SM in FP32,
// 2 in FP64).
template <typename T>
constexpr int march_wide_stages() { return sizeof(T) == 8 ? 4 : 5; }
constexpr int kFmStages = 4;
constexpr int kFmTJ = 8;
template <typename T>
constexpr int kFvStages() { return sizeof(T) == 8 ? 3 : 4; }
// Stages of the fused interior sweep (sweep 7): 4 CTAs per SM in FP32 and 3
// in FP64 with the shared memory these take.
template <typename T>
constexpr int hyb_stages() { return sizeof(T) == 8 ? 3 : 4; }



// Encodes one 3-D tiled map over the (nz+1, ny+1, nx+1) lattice of `base`.
template <typename EncFn>
CUresult encode_lattice(EncFn encode, CUtensorMap* m, CUtensorMapDataType dt, size_t elem,
                        void* base, const Lat& L, int box_k, int box_j) {
  const cuuint64_t dims[3] = {(cuuint64_t)L.nz + 1, (cuuint64_t)L.ny + 1, (cuuint64_t)L.nx + 1};
  const cuuint64_t strides[2] = {(cuuint64_t)L.KP * elem, (cuuint64_t)L.KP * L.NY * elem};
  const cuuint32_t box[3] = {(cuuint32_t)box_k, (cuuint32_t)box_j, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return encode(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Tensor maps for the pipelined sweep: one per field component and buffer
// (3-D: k, j, i over the logical lattice extent so out-of-range boxes read
// zeros) and one for the class index.
xfd_status tensor_map_encoder(xfd_engine* e, EncodeTiledFn* out) {
  static EncodeTiledFn encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CUDA_TRY(e, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess)
      return fail(e, XFD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  *out = encode;
  return XFD_OK;
}

// Tensor maps of the marching sweeps over six field arrays of the lattice
// layout (the engine's buffers, or the adjoint's scaled fields).
// `tj` rows per tile (halo boxes tj + 1 rows).
template <typename T>
xfd_status build_march_maps(xfd_engine* e, void* const f[6], MarchMaps* m, int tj = kMTJ) {
  EncodeTiledFn encode = nullptr;
  xfd_status st = tensor_map_encoder(e, &encode);
  if (st != XFD_OK) return st;
  const int W = 32 + 16 / (int)sizeof(T);
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int c = 0; c < 6; ++c) {
    CUresult r = encode_lattice(encode, &m->halo[c], dt, sizeof(T), f[c], e->L, W, tj + 1);
    if (r == CUDA_SUCCESS)
      r = encode_lattice(encode, &m->tile[c], dt, sizeof(T), f[c], e->L, 32, tj);
    if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (march %d): %d", c, (int)r);
  }
  CUresult r = encode_lattice(encode, &m->cls, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, e->cls, e->L, 32,
                              tj);
  if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (march class): %d", (int)r);
  return XFD_OK;
}

template <typename T>
xfd_status build_tma_maps(xfd_engine* e) {
  using G = TmaGeom<T, kTJ, kTK>;
  EncodeTiledFn encode = nullptr;
  {
    xfd_status st = tensor_map_encoder(e, &encode);
    if (st != XFD_OK) return st;
  }
  const Lat& L = e->L;
  const cuuint64_t dims[3] = {(cuuint64_t)L.nz + 1, (cuuint64_t)L.ny + 1, (cuuint64_t)L.nx + 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int b = 0; b < 2; ++b) {
    const cuuint64_t strides[2] = {(cuuint64_t)L.KP * sizeof(T),
                                   (cuuint64_t)L.KP * L.NY * sizeof(T)};
    for (int c = 0; c < 6; ++c) {
      const cuuint32_t box[3] = {(cuuint32_t)G::WE, (cuuint32_t)(c < 3 ? G::RE : G::RH), 1};
      CUtensorMap* m = c < 3 ? &e->tma[b].e[c] : &e->tma[b].h[c - 3];
      CUresult r = encode(m, dt, 3, e->fbuf[b][c], dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (field %d): %d", c, (int)r);
    }
    const cuuint64_t cstrides[2] = {(cuuint64_t)L.KP * 2, (cuuint64_t)L.KP * L.NY * 2};
    const cuuint32_t cbox[3] = {(cuuint32_t)G::WC, (cuuint32_t)G::RH, 1};
    CUresult r = encode(&e->tma[b].cls, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, e->cls, dims, cstrides,
                        cbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (class): %d", (int)r);
  }
  // Marching sweeps: halo and tile boxes of every component, class tiles.
  using MG = MarchGeom<T, kMTJ, 32>;
  for (int b = 0; b < 2; ++b) {
    xfd_status st = build_march_maps<T>(e, e->fbuf[b], &e->mtma[b]);
    if (st == XFD_OK) st = build_march_maps<T>(e, e->fbuf[b], &e->mtma_w[b], kWideTJ);
    if (st != XFD_OK) return st;
  }
  // Fused marching sweep: E (TJ+1 rows) and H (TJ rows) boxes of width
  // 32 elements + 16 bytes, class boxes of 40.
  const int fm_tj = kFmTJ;
  for (int b = 0; b < 2; ++b) {
    const int W = 32 + 16 / (int)sizeof(T);
    for (int c = 0; c < 3; ++c) {
      CUresult r = encode_lattice(encode, &e->fmaps[b].e[c], dt, sizeof(T), e->fbuf[b][c], L, W,
                                  fm_tj + 1);
      if (r == CUDA_SUCCESS)
        r = encode_lattice(encode, &e->fmaps[b].h[c], dt, sizeof(T), e->fbuf[b][3 + c], L, W,
                           fm_tj);
      if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (fmarch %d): %d", c, (int)r);
    }
    CUresult r = encode_lattice(encode, &e->fmaps[b].cls, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                                e->cls, L, 40, fm_tj);
    if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (fmarch class): %d", (int)r);
  }
  // Two-nodes-per-thread interior form: boxes (64 elements + 16 bytes) wide.
  for (int b = 0; b < 2; ++b) {
    const int W = 64 + 16 / (int)sizeof(T);
    for (int c = 0; c < 3; ++c) {
      CUresult r = encode_lattice(encode, &e->fvmaps[b].e[c], dt, sizeof(T), e->fbuf[b][c], L, W,
                                  kFmTJ + 1);
      if (r == CUDA_SUCCESS)
        r = encode_lattice(encode, &e->fvmaps[b].h[c], dt, sizeof(T), e->fbuf[b][3 + c], L, W,
                           kFmTJ);
      if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (fvec %d): %d", c, (int)r);
    }
    CUresult r = encode_lattice(encode, &e->fvmaps[b].cls, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                                e->cls, L, 72, kFmTJ);
    if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (fvec class): %d", (int)r);
  }
  CUDA_TRY(e, cudaFuncSetAttribute(k_fvec<T, kFmTJ, kFvStages<T>()>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   FvecGeom<T, kFmTJ>::smem(kFvStages<T>())));
  CUDA_TRY(e, cudaFuncSetAttribute(k_fmarch<T, kFmTJ, kFmStages, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   FmarchGeom<T, kFmTJ>::smem(kFmStages)));
  CUDA_TRY(e, cudaFuncSetAttribute(k_fmarch<T, kFmTJ, kFmStages, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   FmarchGeom<T, kFmTJ>::smem(kFmStages)));
  constexpr int S = sizeof(T) == 8 ? kStagesF64 : kStagesF32;
  CUDA_TRY(e, cudaFuncSetAttribute(k_fused_tma<T, kTJ, kTK, S>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, G::smem(S)));
  constexpr int MS = march_stages<T>();
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_h_tma<T, kMTJ, 32, MS, true, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MS)));
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_e_tma<T, kMTJ, 32, MS, true, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MS)));
  constexpr int MF = march_free_stages<T>();
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_h_tma<T, kMTJ, 32, MF, false, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MF)));
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_e_tma<T, kMTJ, 32, MF, false, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MF)));
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_h_tma<T, kMTJ, 32, MF, false, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MF)));
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_e_tma<T, kMTJ, 32, MF, false, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MF)));
  {
    auto attr = [&](const void* f) {
      return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, MG::smem(MS));
    };
    const void* fs[8] = {(const void*)k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 1>,
                         (const void*)k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 2>,
                         (const void*)k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 4>,
                         (const void*)k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 7>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 1>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 2>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 4>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 7>};
    for (const void* f : fs) CUDA_TRY(e, attr(f));
    constexpr int MF4 = march_free_stages<T>();
    const void* f4[6] = {(const void*)k_march_h_tma_list<T, kMTJ, 32, MF4, true, false, 1>,
                         (const void*)k_march_h_tma_list<T, kMTJ, 32, MF4, true, false, 2>,
                         (const void*)k_march_h_tma_list<T, kMTJ, 32, MF4, true, false, 4>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MF4, true, false, 1>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MF4, true, false, 2>,
                         (const void*)k_march_e_tma_list<T, kMTJ, 32, MF4, true, false, 4>};
    for (const void* f : f4)
      CUDA_TRY(e, cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       MG::smem(MF4)));
  }
  // Fused interior sweep (sweep 7): per input buffer, E boxes (32 + 2 XA) x
  // (kMTJ + 2), H boxes (32 + XA) x (kMTJ + 1), class boxes 40 x (kMTJ + 1).
  {
    using HG = HybGeom<T, kMTJ>;
    for (int b = 0; b < 2; ++b) {
      for (int c = 0; c < 3; ++c) {
        CUresult r = encode_lattice(encode, &e->hmaps[b].e[c], dt, sizeof(T), e->fbuf[b][c], L,
                                    HG::WE, HG::RE);
        if (r == CUDA_SUCCESS)
          r = encode_lattice(encode, &e->hmaps[b].h[c], dt, sizeof(T), e->fbuf[b][3 + c], L,
                             HG::WH, HG::RH);
        if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (hyb %d): %d", c, (int)r);
      }
      CUresult r = encode_lattice(encode, &e->hmaps[b].cls, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                                  e->cls, L, HG::WC, HG::RC);
      if (r != CUDA_SUCCESS) return fail(e, XFD_ERR_CUDA, "tensor map (hyb class): %d", (int)r);
    }
    constexpr int HS = hyb_stages<T>();
    CUDA_TRY(e, cudaFuncSetAttribute(k_hyb<T, kMTJ, HS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, HG::smem(HS)));
  }
  constexpr int MW = march_wide_stages<T>();
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_h_wide<T, MW>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   WideGeom<T, MW>::smem()));
  CUDA_TRY(e, cudaFuncSetAttribute(k_march_e_wide<T, MW>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   WideGeom<T, MW>::smem()));
  e->tma_ready = true;
  return XFD_OK;
}

template <typename T>
FusedP<T> fused_params(xfd_engine* e, int in, int out) {
  FusedP<T> p{};
  p.L = e->L;
  for (int c = 0; c < 6; ++c) {
    p.in[c] = static_cast<const T*>(e->fbuf[in][c]);
    p.out[c] = static_cast<T*>(e->fbuf[out][c]);
  }
  p.cls = e->cls;
  p.tab = static_cast<const T*>(e->tab);
  p.n_classes = e->n_classes;
  for (int a = 0; a < 3; ++a) {
    p.fe[a] = static_cast<const T*>(e->fe[a]);
    p.fh[a] = static_cast<const T*>(e->fh[a]);
  }
  for (const auto& S : e->slabs) {
    auto& A = p.slab[S.m];
    const int q = A.count++;
    A.n[q] = S.n;
    A.e_lo[q] = S.e_lo;
    A.h_lo[q] = S.h_lo;
    A.a_e[q] = static_cast<const T*>(S.a_e);
    A.b_e[q] = static_cast<const T*>(S.b_e);
    A.a_h[q] = static_cast<const T*>(S.a_h);
    A.b_h[q] = static_cast<const T*>(S.b_h);
    for (int w = 0; w < 2; ++w) {
      A.psi_e[q][w] = static_cast<T*>(S.psi_e[w]);
      A.psi_h_in[q][w] = static_cast<const T*>(S.psi_h[in][w]);
      A.psi_h_out[q][w] = static_cast<T*>(S.psi_h[out][w]);
    }
  }
  p.tf = e->tfsf;
  p.tfh = e->tfsf_h;
  p.tfh.enabled = e->have_tfsf ? 1 : 0;
  p.ichunk = e->ichunk;
  p.step = e->d_step;
  p.err = e->d_err;
  return p;
}

// Tile counts of the fused marching sweep along (k, j, chunks of i) and the
// box of tile/chunk indices whose nodes meet no CPML layer of either phase.
// A k tile bx holds nodes 31 bx - 1 .. 31 bx + 30, a j tile by holds
// (TJ-1) by - 1 .. (TJ-1) by + TJ - 2, a chunk bz computes planes
// max(bz ichunk - 1, 0) .. min((bz+1) ichunk, nx+1) - 1.
void fmarch_split(const xfd_engine* e, int nt[3], int lo[3], int hi[3]) {
  const Lat& L = e->L;
  const int tj = kFmTJ;
  nt[0] = (L.nz + 1 + 29) / 31;
  nt[1] = (L.ny + 1 + tj - 2) / (tj - 1);
  nt[2] = (L.nx + 1 + e->ichunk - 1) / e->ichunk;
  const int axis_of[3] = {2, 1, 0};  // grid dimension -> lattice axis
  for (int g = 0; g < 3; ++g) {
    const int m = axis_of[g];
    auto range = [&](int b, int& a0, int& a1) {
      if (g == 0) { a0 = 31 * b - 1; a1 = 31 * b + 30; }
      else if (g == 1) { a0 = (tj - 1) * b - 1; a1 = (tj - 1) * b + tj - 2; }
      else { a0 = std::max(b * e->ichunk - 1, 0); a1 = std::min((b + 1) * e->ichunk, L.nx + 1) - 1; }
    };
    auto is_free = [&](int b) {
      int a0, a1;
      range(b, a0, a1);
      for (const auto& S : e->slabs) {
        if (S.m != m) continue;
        if (a0 < S.e_lo + S.n && S.e_lo <= a1) return false;
        if (a0 < S.h_lo + S.n && S.h_lo <= a1) return false;
      }
      return true;
    };
    // Longest run of free indices.
    int best_lo = 0, best_len = 0;
    for (int b = 0; b < nt[g];) {
      if (!is_free(b)) { ++b; continue; }
      int c = b;
      while (c < nt[g] && is_free(c)) ++c;
      if (c - b > best_len) { best_lo = b; best_len = c - b; }
      b = c;
    }
    lo[g] = best_lo;
    hi[g] = best_lo + best_len;
  }
}

// The box of (k tile of 32, j tile of 8, chunk of march_ichunk planes) of
// the split marching sweeps whose nodes lie in no CPML layer of either phase.
// Along grid dimension g (0: k tiles of 32, 1: j tiles of tj rows, 2: chunks of
// march_ichunk x planes) with the grid shifted by sh nodes (-size < sh <= 0),
// tile b covers nodes [sh + b size, sh + (b+1) size) within the lattice.  The
// longest run [lo, hi) of tiles that meet no CPML layer of either phase;
// returns the nodes it covers.
int march_free_run(const xfd_engine* e, int g, int sh, int& lo, int& hi, int tj = kMTJ) {
  const Lat& L = e->L;
  const int size[3] = {32, tj, e->march_ichunk};
  const int n_nodes[3] = {L.nz, L.ny, L.nx + 1};
  const int axis_of[3] = {2, 1, 0};  // grid dimension -> lattice axis
  const int m = axis_of[g], z = size[g], n = n_nodes[g];
  const int nt = (n - sh + z - 1) / z;
  auto is_free = [&](int b) {
    const int a0 = std::max(sh + b * z, 0), a1 = std::min(sh + (b + 1) * z, n) - 1;
    for (const auto& S : e->slabs) {
      if (S.m != m) continue;
      if (a0 < S.e_lo + S.n && S.e_lo <= a1) return false;
      if (a0 < S.h_lo + S.n && S.h_lo <= a1) return false;
    }
    return true;
  };
  lo = hi = 0;
  int best = 0;
  for (int b = 0; b < nt;) {
    if (!is_free(b)) {
      ++b;
      continue;
    }
    int c = b;
    while (c < nt && is_free(c)) ++c;
    const int nodes = std::min(sh + c * z, n) - std::max(sh + b * z, 0);
    if (nodes > best) {
      best = nodes;
      lo = b;
      hi = c;
    }
    b = c;
  }
  return best;
}

// The CPML-free box of the unshifted tile grid of tj-row tiles (the batched
// sweeps' split).
void march_split(const xfd_engine* e, int lo[3], int hi[3], int tj = kMTJ) {
  for (int g = 0; g < 3; ++g) march_free_run(e, g, 0, lo[g], hi[g], tj);
}

// Work split of the TMA marching sweeps for the current options: the
// CPML-free box (in 8-row tiles), whether it is away from every lattice
// boundary, the 16-row tiles of the two-rows-per-thread form, and the box of
// tiles that the CPML form skips.
struct MarchLayout {
  int nt[3];                 // tiles along k, j and chunks along i
  int shift[3];              // grid shift (nodes) along k, j, i
  int lo[3], hi[3];          // CPML-free box
  bool box, in, wide;
  int wy_lo, wy_hi;          // 16-row tiles of the wide form
  int skip_lo[3], skip_hi[3];  // tiles swept by the box or wide form
};

MarchLayout march_layout(const xfd_engine* e) {
  MarchLayout m{};
  const Lat& L = e->L;
  const int size[3] = {32, kMTJ, e->march_ichunk};
  const int n_nodes[3] = {L.nz, L.ny, L.nx + 1};
  // Per axis the shift whose CPML-free run covers the most nodes (k in steps
  // of 8 nodes, so that every TMA x coordinate stays a multiple of 16 bytes
  // for the field and the uint16 class maps alike).  Sweep 7 always shifts
  // along j and i (rows and planes carry no alignment), along k only with the
  // march_shift option.
  const int step[3] = {8, 1, 1};
  const bool hyb = e->kernel_mode == 7;
  for (int g = 0; g < 3; ++g) {
    int best = -1;
    for (int sh = 0; sh > -size[g]; sh -= step[g]) {
      if (sh != 0 && !e->march_shift && !(hyb && g > 0)) break;
      int lo = 0, hi = 0;
      const int nodes = march_free_run(e, g, sh, lo, hi);
      if (nodes > best) {
        best = nodes;
        m.shift[g] = sh;
        m.lo[g] = lo;
        m.hi[g] = hi;
      }
    }
    m.nt[g] = (n_nodes[g] - m.shift[g] + size[g] - 1) / size[g];
  }
  if (hyb) {
    // The fused interior sweep has no range tests and no CPML terms: its box
    // keeps one node away from the lattice's low faces (k, j, i >= 1) and
    // below nz, ny, nx, and the nodes it recomputes below the box (row
    // j0-1, column k0-1, plane i_lo-1) lie in no H layer of that axis.
    const int upper[3] = {L.nz, L.ny, L.nx};
    const int axis_of[3] = {2, 1, 0};
    for (int g = 0; g < 3; ++g) {
      const int sh = m.shift[g];
      while (m.lo[g] * size[g] + sh < 1) ++m.lo[g];
      m.hi[g] = std::min(m.hi[g], (upper[g] - sh) / size[g]);
      while (m.hi[g] > m.lo[g]) {
        const int below = m.lo[g] * size[g] + sh - 1;
        bool in_layer = false;
        for (const auto& S : e->slabs)
          if (S.m == axis_of[g] && below >= S.h_lo && below < S.h_lo + S.n) in_layer = true;
        if (!in_layer) break;
        ++m.lo[g];
      }
    }
  }
  m.box = m.hi[0] > m.lo[0] && m.hi[1] > m.lo[1] && m.hi[2] > m.lo[2];
  // The box is away from every lattice boundary when no tile holds k = 0,
  // j = 0 or a node past nz-1 / ny-1 and no chunk holds plane 0 or nx.
  m.in = m.box && 32 * m.lo[0] + m.shift[0] >= 1 && 32 * m.hi[0] + m.shift[0] <= L.nz &&
         kMTJ * m.lo[1] + m.shift[1] >= 1 && kMTJ * m.hi[1] + m.shift[1] <= L.ny &&
         e->march_ichunk * m.lo[2] + m.shift[2] >= 1 &&
         e->march_ichunk * m.hi[2] + m.shift[2] <= L.nx;
  // The two-rows-per-thread form takes the interior box's whole pairs of
  // 8-row tiles; the CPML form sweeps the rest, an unpaired tile row included.
  m.wy_lo = (m.lo[1] + 1) / 2;
  m.wy_hi = m.hi[1] / 2;
  m.wide = m.in && e->march_wide && m.wy_hi > m.wy_lo && !hyb;
  if (hyb && !m.in) m.box = false;  // every tile goes to the CPML forms
  for (int a = 0; a < 3; ++a) {
    m.skip_lo[a] = m.box ? m.lo[a] : 0;
    m.skip_hi[a] = m.box ? m.hi[a] : 0;
  }
  if (m.wide) {
    m.skip_lo[1] = 2 * m.wy_lo;
    m.skip_hi[1] = 2 * m.wy_hi;
  }
  return m;
}

// The CPML form's tiles outside the skip box, sorted by the CPML axes whose
// layers (of either phase) their node ranges meet: lists of x-only, y-only,
// z-only and several-axis (or none) tiles, as (0, k tile, j tile, chunk).
// Whether the node range [a0, a1) along lattice axis `axis` meets a CPML
// layer of either phase.
bool meets_cpml(const xfd_engine* e, int axis, int a0, int a1) {
  for (const auto& S : e->slabs) {
    if (S.m != axis) continue;
    if (a0 < S.e_lo + S.n && S.e_lo < a1) return true;
    if (a0 < S.h_lo + S.n && S.h_lo < a1) return true;
  }
  return false;
}

// List of a CPML-form tile by the axes whose layers it meets: 0 x only,
// 1 y only, 2 z only, 3 several (or none).  Node ranges along k, j, i.
int cpml_tile_list(const xfd_engine* e, int k0, int k1, int j0, int j1, int i0, int i1) {
  const int mask = (meets_cpml(e, 0, i0, i1) ? 1 : 0) | (meets_cpml(e, 1, j0, j1) ? 2 : 0) |
                   (meets_cpml(e, 2, k0, k1) ? 4 : 0);
  return mask == 1 ? 0 : mask == 2 ? 1 : mask == 4 ? 2 : 3;
}

void march_tile_lists(const xfd_engine* e, std::vector<int4> lists[4]) {
  const MarchLayout m = march_layout(e);
  const Lat& L = e->L;
  for (int gz = 0; gz < m.nt[2]; ++gz)
    for (int gy = 0; gy < m.nt[1]; ++gy)
      for (int gx = 0; gx < m.nt[0]; ++gx) {
        if (gx >= m.skip_lo[0] && gx < m.skip_hi[0] && gy >= m.skip_lo[1] &&
            gy < m.skip_hi[1] && gz >= m.skip_lo[2] && gz < m.skip_hi[2])
          continue;
        const int ich = e->march_ichunk, sx = m.shift[2], sy = m.shift[1], sz = m.shift[0];
        int q = 3;
        if (e->march_split_axes)
          q = cpml_tile_list(e, std::max(gx * 32 + sz, 0), std::min((gx + 1) * 32 + sz, L.nz),
                             std::max(gy * kMTJ + sy, 0), std::min((gy + 1) * kMTJ + sy, L.ny),
                             std::max(gz * ich + sx, 0), std::min((gz + 1) * ich + sx, L.nx + 1));
        lists[q].push_back(make_int4(0, gx, gy, gz));
      }
}

// The box tiles of sweep 7 split by whether a TFSF H pass reaches a node
// that the tile's CTA computes: its own nodes over planes i_lo-1 .. i_hi-1,
// the recomputed row j0-1 and column k0-1.  Without TFSF every tile is in the
// first list.
xfd_status build_hyb_tiles(xfd_engine* e) {
  const MarchLayout ml = march_layout(e);
  const long long key = (long long)e->slabs.size() * 1000003LL + e->march_ichunk * 4 +
                        (e->march_shift ? 2 : 0) + (ml.box ? 1 : 0);
  if (key == e->hyb_key) return XFD_OK;
  // j tiles fastest, then k tiles, then chunks: CTAs resident together share
  // the E / H rows of their j halos through L2.
  std::vector<int4> all;
  if (ml.box)
    for (int gz = ml.lo[2]; gz < ml.hi[2]; ++gz)
      for (int gx = ml.lo[0]; gx < ml.hi[0]; ++gx)
        for (int gy = ml.lo[1]; gy < ml.hi[1]; ++gy) all.push_back(make_int4(0, gx, gy, gz));
  e->n_hyb_tiles = (int)all.size();
  if (all.size() > e->hyb_tiles_cap) {
    void* p = nullptr;
    xfd_status st = dev_alloc(e, &p, all.size() * sizeof(int4));
    if (st != XFD_OK) return st;
    e->d_hyb_tiles = static_cast<int4*>(p);
    e->hyb_tiles_cap = all.size();
  }
  if (!all.empty())
    CUDA_TRY(e, cudaMemcpy(e->d_hyb_tiles, all.data(), all.size() * sizeof(int4),
                           cudaMemcpyHostToDevice));
  e->hyb_key = key;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status build_march_tiles(xfd_engine* e) {
  const long long key = (long long)e->slabs.size() * 1000003LL + e->march_ichunk * 16 +
                        (e->kernel_mode == 7 ? 8 : 0) + (e->march_shift ? 4 : 0) +
                        (e->march_wide ? 2 : 0) + (e->march_split_axes ? 1 : 0);
  if (key == e->mtiles_key) return XFD_OK;
  std::vector<int4> lists[4];
  march_tile_lists(e, lists);
  std::vector<int4> all;
  e->mt_off[0] = 0;
  for (int q = 0; q < 4; ++q) {
    all.insert(all.end(), lists[q].begin(), lists[q].end());
    e->mt_off[q + 1] = (int)all.size();
  }
  if (all.size() > e->mtiles_cap) {
    void* p = nullptr;
    xfd_status st = dev_alloc(e, &p, all.size() * sizeof(int4));
    if (st != XFD_OK) return st;
    e->d_mtiles = static_cast<int4*>(p);
    e->mtiles_cap = all.size();
  }
  if (!all.empty())
    CUDA_TRY(e, cudaMemcpy(e->d_mtiles, all.data(), all.size() * sizeof(int4),
                           cudaMemcpyHostToDevice));
  e->mtiles_key = key;
  e->graph_dirty = true;
  return XFD_OK;
}

template <typename T>
MarchP<T> march_params(xfd_engine* e) {
  const int pb = psi_h_buf(e);
  const FusedP<T> f = fused_params<T>(e, pb, pb);
  MarchP<T> p{};
  p.L = f.L;
  for (int c = 0; c < 6; ++c) p.f[c] = static_cast<T*>(e->fbuf[e->cur][c]);
  p.cls = f.cls;
  p.tab = f.tab;
  p.n_classes = e->n_classes;
  for (int a = 0; a < 3; ++a) {
    p.fe[a] = f.fe[a];
    p.fh[a] = f.fh[a];
    p.slab[a] = f.slab[a];
  }
  p.ichunk = e->march_ichunk;
  p.xl = e->d_xlayer;
  return p;
}

long long gcd_ll(long long a, long long b) { return b == 0 ? a : gcd_ll(b, a % b); }

template <typename T>
OverrideD<T> ovr_of(const xfd_engine* e) {
  if constexpr (sizeof(T) == 8) return e->ovr64; else return e->ovr32;
}

template <typename T>
HTermD<T> hterm_of(const xfd_engine* e) {
  if constexpr (sizeof(T) == 8) return e->hterm64; else return e->hterm32;
}

// Launches one time step (host step index t decides the periodic kernels).
// Sweep 7, one step from buffer `in` to `out`: the fused box kernel (side
// stream 0) beside the CPML form's H tile lists and the H lattice faces (main
// stream, side streams 1-3); then the TFSF H passes outside the box; then,
// once the box kernel is done, the CPML form's E tile lists and the E faces.
// The CPML forms read the old fields of `in` and the new H of `out` through
// their tensor maps and write `out`; their psi stay in place (buffer 0).
template <typename T>
cudaError_t enqueue_hyb_t(xfd_engine* e, int in, int out) {
  cudaStream_t s = e->stream;
  const MarchLayout ml = march_layout(e);
  constexpr int MS = march_stages<T>();
  constexpr int MF = march_free_stages<T>();
  constexpr int HS = hyb_stages<T>();
  const size_t msm = MarchGeom<T, kMTJ, 32>::smem(MS);
  const size_t msm_free = MarchGeom<T, kMTJ, 32>::smem(MF);
  const dim3 blk_m(32, kMTJ, 1);
  T* const* fields_in = reinterpret_cast<T* const*>(e->d_fields[in]);
  MarchTmaP<T> mh{};
  mh.p = march_params<T>(e);
  for (int c = 0; c < 6; ++c) mh.p.f[c] = static_cast<T*>(e->fbuf[out][c]);
  mh.m = e->mtma[in];  // old E halo boxes, old H tiles
  mh.err = e->d_err;
  mh.wait_budget = e->stage_wait;
  for (int a = 0; a < 3; ++a) {
    mh.box_lo[a] = ml.skip_lo[a];
    mh.box_hi[a] = ml.skip_hi[a];
    mh.shift[a] = ml.shift[a];
  }
  MarchTmaP<T> me = mh;
  for (int c = 0; c < 3; ++c) {
    me.m.halo[3 + c] = e->mtma[out].halo[3 + c];  // new H halo boxes
    me.m.tile[c] = e->mtma[in].tile[c];           // old E tiles
  }
  YeeP<T> yp = yee_params<T>(e);
  for (int c = 0; c < 6; ++c) yp.f[c] = static_cast<T*>(e->fbuf[out][c]);
  const unsigned edge_blocks = (unsigned)((edge_nodes(e->L) + 255) / 256);
  cudaError_t c = cudaSuccess;
  auto fork = [&](int first) {
    if (c == cudaSuccess) c = cudaEventRecord(e->fork_ev, s);
    for (int q = first; q < kSides && c == cudaSuccess; ++q)
      c = cudaStreamWaitEvent(e->side[q], e->fork_ev, 0);
  };
  auto join = [&](int first, int last) {
    for (int q = first; q <= last && c == cudaSuccess; ++q) {
      c = cudaEventRecord(e->join_ev[q], e->side[q]);
      if (c == cudaSuccess) c = cudaStreamWaitEvent(s, e->join_ev[q], 0);
    }
  };
  auto lists = [&](const MarchTmaP<T>& P, auto kx4, auto ky4, auto kz4, auto kcp) {
    auto list = [&](auto k, int q, size_t sm) {
      const int n = e->mt_off[q + 1] - e->mt_off[q];
      cudaStream_t sq = q == 3 ? s : e->side[q + 1];
      if (n > 0 && c == cudaSuccess) k<<<n, blk_m, sm, sq>>>(P, e->d_mtiles + e->mt_off[q]);
    };
    list(kx4, 0, msm_free);
    list(ky4, 1, msm_free);
    list(kz4, 2, msm_free);
    list(kcp, 3, msm);
  };
  // TFSF H-face corrections into the H every sweep kernel reads (k_tfsf_pre).
  if (e->have_tfsf) {
    T* const* fi = reinterpret_cast<T* const*>(e->d_fields[in]);
    for (int g = 0; g < 2 && c == cudaSuccess; ++g) {
      const auto& G = e->tfsf_groups[g];
      if (G.total > 0)
        k_tfsf_pre<T><<<blocks_for(G.total, 256), 256, 0, s>>>(
            e->tfsf, G, e->L, fi, e->cls, static_cast<const T*>(e->tab), e->d_step, e->d_err);
    }
  }
  fork(0);
  if (ml.box && c == cudaSuccess) {
    HybP<T> hp{};
    hp.L = e->L;
    for (int q = 0; q < 6; ++q) hp.out[q] = static_cast<T*>(e->fbuf[out][q]);
    hp.tab = static_cast<const T*>(e->tab);
    hp.n_classes = e->n_classes;
    for (int a = 0; a < 3; ++a) {
      hp.fe[a] = static_cast<const T*>(e->fe[a]);
      hp.fh[a] = static_cast<const T*>(e->fh[a]);
      hp.org[a] = ml.lo[a];
      hp.shift[a] = ml.shift[a];
    }
    hp.err = e->d_err;
    hp.wait_budget = e->stage_wait;
    hp.m = e->hmaps[in];
    hp.ichunk = e->march_ichunk;
    const size_t hsm = HybGeom<T, kMTJ>::smem(HS);
    const dim3 blk_h(32, kMTJ + 1, 1);  // kMTJ compute warps + the helper warp
    hp.tiles = e->d_hyb_tiles;
    if (e->n_hyb_tiles > 0)
      k_hyb<T, kMTJ, HS><<<e->n_hyb_tiles, blk_h, hsm, e->side[0]>>>(hp);
  }
  lists(mh, k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 1>,
        k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 2>,
        k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 4>,
        k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 7>);
  // Lumped elements, inductors and overrides add to their nodes after the
  // sweep: if one sits on a lattice face k = nz or j = ny, those faces are
  // carried over in full.
  bool face_targets = false;
  auto on_face = [&](long long id) {
    const long long jk = id % ((long long)e->L.NY * e->L.KP);
    const int j = (int)(jk / e->L.KP), k = (int)(jk % e->L.KP);
    return j == e->L.ny || k == e->L.nz;
  };
  for (const auto& l : e->lumped_h)
    for (long long id : l.node) face_targets = face_targets || on_face(id);
  for (const auto& l : e->ind_h)
    for (long long id : l.node) face_targets = face_targets || on_face(id);
  for (size_t q = 0; q < e->ovr_node.size(); q += 3)
    face_targets = face_targets || e->ovr_node[q + 1] == e->L.ny || e->ovr_node[q + 2] == e->L.nz;
  if (c == cudaSuccess)
    k_edge_pp<T, false><<<edge_blocks, 256, 0, e->side[1]>>>(yp, fields_in, face_targets);
  join(1, kSides - 1);
  join(0, 0);  // the box kernel's new H
  fork(1);
  lists(me, k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 1>,
        k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 2>,
        k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 4>,
        k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 7>);
  if (c == cudaSuccess)
    k_edge_pp<T, true><<<edge_blocks, 256, 0, e->side[1]>>>(yp, fields_in, face_targets);
  join(1, kSides - 1);
  if (c != cudaSuccess) return c;
  return cudaGetLastError();
}

// A launch of kernel k, with programmatic stream serialization when `pdl`
// (the kernel calls pdl_enter first: kernels.cuh).
template <typename... KP, typename... A>
cudaError_t launch_k(bool pdl, void (*k)(KP...), dim3 g, dim3 b, cudaStream_t s, A&&... a) {
  if (!pdl) {
    k<<<g, b, 0, s>>>(std::forward<A>(a)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(a)...);
}

template <typename T>
cudaError_t enqueue_step_t(xfd_engine* e, long long t) {
  cudaStream_t s = e->stream;
  const bool fused = is_fused(e);
  const bool pp = is_pingpong(e);
  const int in = e->cur, out = pp ? 1 - e->cur : e->cur;
  T* const* fields = reinterpret_cast<T* const*>(e->d_fields[out]);
  T* const* fields_in = reinterpret_cast<T* const*>(e->d_fields[in]);
  AdeD<T> ad{};
  if (e->ade_kind >= 0) {
    if constexpr (sizeof(T) == 8) ad = e->ade64; else ad = e->ade32;
  }
  // Sweep 0 (small lattices): its H / E updates, TFSF passes and step
  // counter go out with programmatic dependent launch (option "pdl").
  const bool pdl = e->pdl && e->kernel_mode == 0;
  if (e->kernel_mode == 7) {
    cudaError_t c = enqueue_hyb_t<T>(e, in, out);
    if (c != cudaSuccess) return c;
  } else if (fused) {
    // H + TFSF-H + CPML-H, then E + CPML-E, in one sweep: in -> out.
    const dim3 blk(kTK, kTJ, 1);
    const dim3 grd((unsigned)((e->L.nz + 1 + kTK - 1) / kTK),
                   (unsigned)((e->L.ny + 1 + kTJ - 1) / kTJ),
                   (unsigned)((e->L.nx + 1 + e->ichunk - 1) / e->ichunk));
    if (e->kernel_mode == 5 || e->kernel_mode == 6) {
      FmarchP<T> fm{};
      fm.p = fused_params<T>(e, in, out);
      fm.m = e->fmaps[in];
      int nt[3], lo[3], hi[3];
      fmarch_split(e, nt, lo, hi);
      if (e->kernel_mode == 6) {
        // The interior in pairs of k tiles for the two-nodes-per-thread form;
        // the CPML form sweeps everything outside those pairs.
        const int v0 = (lo[0] + 1) / 2, v1 = hi[0] / 2;
        if (v1 > v0 && hi[1] > lo[1] && hi[2] > lo[2]) {
          FvecP<T> fv{};
          fv.p = fm.p;
          fv.m = e->fvmaps[in];
          fv.org[0] = v0;
          fv.org[1] = lo[1];
          fv.org[2] = lo[2];
          constexpr int FS = kFvStages<T>();
          k_fvec<T, kFmTJ, FS><<<dim3(v1 - v0, hi[1] - lo[1], hi[2] - lo[2]), dim3(32, kFmTJ, 1),
                                 FvecGeom<T, kFmTJ>::smem(FS), s>>>(fv);
          lo[0] = 2 * v0;
          hi[0] = 2 * v1;
        } else {
          hi[0] = lo[0];  // no interior form: the CPML form sweeps all
        }
        for (int a = 0; a < 3; ++a) {
          fm.box_lo[a] = lo[a];
          fm.box_hi[a] = hi[a];
          fm.org[a] = 0;
        }
        k_fmarch<T, kFmTJ, kFmStages, true>
            <<<dim3(nt[0], nt[1], nt[2]), dim3(32, kFmTJ, 1), FmarchGeom<T, kFmTJ>::smem(kFmStages),
               s>>>(fm);
      } else {
        for (int a = 0; a < 3; ++a) {
          fm.box_lo[a] = lo[a];
          fm.box_hi[a] = hi[a];
          fm.org[a] = lo[a];
        }
        const size_t sm = FmarchGeom<T, kFmTJ>::smem(kFmStages);
        const dim3 blk(32, kFmTJ, 1);
        if (hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2])
          k_fmarch<T, kFmTJ, kFmStages, false>
              <<<dim3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]), blk, sm, s>>>(fm);
        fm.org[0] = fm.org[1] = fm.org[2] = 0;
        k_fmarch<T, kFmTJ, kFmStages, true><<<dim3(nt[0], nt[1], nt[2]), blk, sm, s>>>(fm);
      }
    } else if (e->kernel_mode == 2) {
      FusedTmaP<T> tp{};
      tp.p = fused_params<T>(e, in, out);
      tp.m = e->tma[in];
      constexpr int S = sizeof(T) == 8 ? kStagesF64 : kStagesF32;
      k_fused_tma<T, kTJ, kTK, S>
          <<<grd, blk, TmaGeom<T, kTJ, kTK>::smem(S), s>>>(tp);
    } else {
      const FusedP<T> fp = fused_params<T>(e, in, out);
      k_fused<T, kTJ, kTK><<<grd, blk, 0, s>>>(fp);
    }
  } else {
    const YeeP<T> yp = yee_params<T>(e);
    const bool march = e->kernel_mode == 3 || e->kernel_mode == 4;
    const bool march_tma = e->kernel_mode == 4;
    constexpr int MS = march_stages<T>();
    MarchP<T> mp{};
    MarchTmaP<T> mtp{};
    if (march) mp = march_params<T>(e);
    if (march_tma) {
      mtp.p = mp;
      mtp.m = e->mtma[e->cur];
      mtp.err = e->d_err;
      mtp.wait_budget = e->stage_wait;
    }
    const dim3 blk(32, 8, 1);
    const dim3 grd((unsigned)((e->L.nz + 1 + 31) / 32), (unsigned)((e->L.ny + 1 + 7) / 8),
                   (unsigned)(e->L.nx + 1));
    // The TMA marching sweeps tile k < nz, j < ny (the faces k = nz, j = ny
    // go to k_edge_h / k_edge_e); the plain marching sweeps tile all nodes.
    const dim3 grd_m(grd.x, grd.y,
                     (unsigned)((e->L.nx + 1 + mp.ichunk - 1) / std::max(1, mp.ichunk)));
    const unsigned edge_blocks = (unsigned)((edge_nodes(e->L) + 255) / 256);
    MarchLayout ml{};
    if (march_tma) {
      ml = march_layout(e);
      for (int a = 0; a < 3; ++a) {
        mtp.box_lo[a] = ml.skip_lo[a];
        mtp.box_hi[a] = ml.skip_hi[a];
        mtp.shift[a] = ml.shift[a];
      }
    }
    const dim3 blk_m(32, kMTJ, 1);
    const size_t msm = MarchGeom<T, kMTJ, 32>::smem(MS);
    constexpr int MF = march_free_stages<T>();
    const size_t msm_free = MarchGeom<T, kMTJ, 32>::smem(MF);
    constexpr int MW = march_wide_stages<T>();
    // With march_concurrent, the box form runs on side[0], the face kernel on
    // side[1], and the CPML form's tile lists spread over the main stream and
    // side[1..3] (x-only after the faces, y-only, z-only, several on main).
    const bool conc = march_tma && e->march_concurrent;
    auto fork = [&]() -> cudaError_t {
      if (!conc) return cudaSuccess;
      cudaError_t c = cudaEventRecord(e->fork_ev, s);
      for (int q = 0; q < kSides && c == cudaSuccess; ++q)
        c = cudaStreamWaitEvent(e->side[q], e->fork_ev, 0);
      return c;
    };
    auto join = [&]() -> cudaError_t {
      if (!conc) return cudaSuccess;
      cudaError_t c = cudaSuccess;
      for (int q = 0; q < kSides && c == cudaSuccess; ++q) {
        c = cudaEventRecord(e->join_ev[q], e->side[q]);
        if (c == cudaSuccess) c = cudaStreamWaitEvent(s, e->join_ev[q], 0);
      }
      return c;
    };
    cudaStream_t s_box = conc ? e->side[0] : s, s_edge = conc ? e->side[1] : s;
    // kcp: the CPML form's tile-list kernels for x-only, y-only, z-only and
    // several-axis tiles.
    auto launch_march = [&](auto kfree, auto kfree_in, auto kwide, auto kx, auto ky, auto kz,
                            auto kx4, auto ky4, auto kz4, auto kcp) {
      if (ml.wide) {
        MarchTmaP<T> q = mtp;
        q.m = e->mtma_w[e->cur];
        q.org[0] = ml.lo[0];
        q.org[1] = ml.wy_lo;
        q.org[2] = ml.lo[2];
        const dim3 g(ml.hi[0] - ml.lo[0], ml.wy_hi - ml.wy_lo, ml.hi[2] - ml.lo[2]);
        kwide<<<g, dim3(32, kWideCW + 1, 1), WideGeom<T, MW>::smem(), s_box>>>(q);
      } else if (ml.box) {
        MarchTmaP<T> q = mtp;
        for (int a = 0; a < 3; ++a) q.org[a] = ml.lo[a];
        const dim3 g(ml.hi[0] - ml.lo[0], ml.hi[1] - ml.lo[1], ml.hi[2] - ml.lo[2]);
        if (ml.in)
          kfree_in<<<g, blk_m, msm_free, s_box>>>(q);
        else
          kfree<<<g, blk_m, msm_free, s_box>>>(q);
      }
      auto list = [&](auto k, int q, size_t sm) {
        const int n = e->mt_off[q + 1] - e->mt_off[q];
        cudaStream_t sq = !conc || q == 3 ? s : e->side[q + 1];
        if (n > 0) k<<<n, blk_m, sm, sq>>>(mtp, e->d_mtiles + e->mt_off[q]);
      };
      if (e->march_cp_stages == 1) {
        list(kx4, 0, msm_free);
        list(ky4, 1, msm_free);
        list(kz4, 2, msm_free);
      } else {
        list(kx, 0, msm);
        list(ky, 1, msm);
        list(kz, 2, msm);
      }
      list(kcp, 3, msm);
    };
    // H phase: updateH + CPML (fused) -> TFSF H faces.
    if (march_tma) {
      cudaError_t c = fork();
      if (c != cudaSuccess) return c;
      launch_march(k_march_h_tma<T, kMTJ, 32, MF, false, false>,
                   k_march_h_tma<T, kMTJ, 32, MF, false, true>, k_march_h_wide<T, MW>,
                   k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 1>,
                   k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 2>,
                   k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 4>,
                   k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 1>,
                   k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 2>,
                   k_march_h_tma_list<T, kMTJ, 32, MF, true, false, 4>,
                   k_march_h_tma_list<T, kMTJ, 32, MS, true, false, 7>);
      k_edge_h<T><<<edge_blocks, 256, 0, s_edge>>>(yp);
      if ((c = join()) != cudaSuccess) return c;
    }
    else if (march)
      k_march_h<T, 8, 32><<<grd_m, blk, 0, s>>>(mp);
    else if (cudaError_t c = launch_k(pdl, k_update_h<T>, grd, blk, s, yp); c != cudaSuccess)
      return c;
    if (e->n_hterm)
      k_hterm<T><<<blocks_for(e->n_hterm, 256), 256, 0, s>>>(hterm_of<T>(e), e->L, fields);
    if (e->have_tfsf) {
      for (int g = 0; g < 2; ++g) {
        const auto& G = e->tfsf_groups[g];
        if (G.total > 0)
          if (cudaError_t c = launch_k(pdl, k_tfsf<T>, dim3(blocks_for(G.total, 256)), dim3(256), s,
                                       e->tfsf, G, e->L, fields, (const long long*)e->d_step,
                                       e->d_err);
              c != cudaSuccess)
            return c;
      }
    }
    // E phase: ADE e_cur gather -> updateE + CPML.
    if (e->ade_kind >= 0) k_ade_gather<T><<<blocks_for(ad.n, 256), 256, 0, s>>>(ad, fields);
    if (e->n_ovr) k_ovr_gather<T><<<blocks_for(e->n_ovr, 256), 256, 0, s>>>(ovr_of<T>(e), fields);
    if (march_tma) {
      cudaError_t c = fork();
      if (c != cudaSuccess) return c;
      launch_march(k_march_e_tma<T, kMTJ, 32, MF, false, false>,
                   k_march_e_tma<T, kMTJ, 32, MF, false, true>, k_march_e_wide<T, MW>,
                   k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 1>,
                   k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 2>,
                   k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 4>,
                   k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 1>,
                   k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 2>,
                   k_march_e_tma_list<T, kMTJ, 32, MF, true, false, 4>,
                   k_march_e_tma_list<T, kMTJ, 32, MS, true, false, 7>);
      k_edge_e<T><<<edge_blocks, 256, 0, s_edge>>>(yp);
      if ((c = join()) != cudaSuccess) return c;
    }
    else if (march)
      k_march_e<T, 8, 32><<<grd_m, blk, 0, s>>>(mp);
    else if (cudaError_t c = launch_k(pdl, k_update_e<T>, grd, blk, s, yp); c != cudaSuccess)
      return c;
  }
  // Coefficient overrides complete the E update of their nodes.
  if (e->n_ovr)
    k_ovr_apply<T><<<blocks_for(e->n_ovr, 256), 256, 0, s>>>(ovr_of<T>(e), fields,
                                                             pp ? fields_in : nullptr);
  // ADE -> lumped -> TFSF E faces (the reference's updateE then correctE order).
  T* const* ecur = pp ? fields_in : nullptr;
  if (e->ade_kind == 0) k_ade_update<T, 0><<<blocks_for(ad.n, 256), 256, 0, s>>>(ad, fields, ecur);
  if (e->ade_kind == 1) k_ade_update<T, 1><<<blocks_for(ad.n, 256), 256, 0, s>>>(ad, fields, ecur);
  if (e->ade_kind == 2) k_ade_update<T, 2><<<blocks_for(ad.n, 256), 256, 0, s>>>(ad, fields, ecur);
  if (e->lumped.n > 0)
    k_lumped<T><<<blocks_for(e->lumped.n, 256), 256, 0, s>>>(e->lumped, fields, e->d_step);
  if (e->ind.n > 0) k_inductor<T><<<blocks_for(e->ind.n, 256), 256, 0, s>>>(e->ind, fields);
  if (e->have_tfsf) {
    for (int g = 2; g < 4; ++g) {
      const auto& G = e->tfsf_groups[g];
      if (G.total > 0)
        if (cudaError_t c = launch_k(pdl, k_tfsf<T>, dim3(blocks_for(G.total, 256)), dim3(256), s,
                                     e->tfsf, G, e->L, fields, (const long long*)e->d_step,
                                     e->d_err);
            c != cudaSuccess)
          return c;
    }
  }
  // record: monitors, then NF2FF (Domain::record, src/domain/domain.cpp:176-184).
  for (auto& mv : e->movies) {
    if (t % mv.d.interval == 0)
      k_movie<T><<<blocks_for(mv.n_nodes, 256), 256, 0, s>>>(mv.d, e->L, fields, e->d_step);
  }
  if (e->probes.n_probes)
    if (cudaError_t c = launch_k(pdl, k_probes<T>, dim3(e->probes.n_probes), dim3(256), s,
                                 e->probes, fields, (const long long*)e->d_step);
        c != cudaSuccess)
      return c;
  if (e->have_td)
    k_nf2ff_td<T><<<blocks_for(e->td.P, 256), 256, 0, s>>>(e->td, e->L, fields, e->d_step,
                                                          e->d_err);
  for (int r = 0; r < e->n_rec; ++r) {
    BoxRecD<T> rd;
    if constexpr (sizeof(T) == 8) rd = e->rec64[r]; else rd = e->rec32[r];
    k_box_record<T><<<blocks_for(rd.n * rd.nc, 256), 256, 0, s>>>(rd, e->L, fields, e->d_step);
  }
  if (e->have_nf2ff) {
    k_nf2ff_sample<T><<<blocks_for(e->nf2ff.P, 256), 256, 0, s>>>(e->nf2ff, e->L, fields,
                                                                  e->d_step);
    if ((t + 1) % e->nf2ff.batch == 0) {
      const size_t smem = (size_t)2 * e->nf2ff.nf * e->nf2ff.batch * sizeof(double2);
      k_nf2ff_dft<8><<<blocks_for(4 * e->nf2ff.P, 256), 256, smem, s>>>(e->nf2ff, e->d_step, 0,
                                                                        0);
    }
  }
  if (e->watchdog > 0 && (t + 1) % e->watchdog == 0)
    k_watchdog<T><<<4 * 148, 256, 0, s>>>(fields, e->n_lat, e->d_err);
  if (cudaError_t c = launch_k(pdl, k_advance, dim3(1), dim3(1), s, e->d_step); c != cudaSuccess)
    return c;
  e->cur = out;
  return cudaGetLastError();
}

cudaError_t enqueue_step(xfd_engine* e, long long t) {
  return e->precision == XFD_FP64 ? enqueue_step_t<double>(e, t) : enqueue_step_t<float>(e, t);
}

// Steps between identical launch patterns: lcm of every periodic kernel's
// period, replicated up to the configured chunk length.
long long pattern_period(const xfd_engine* e) {
  long long per = 1;
  for (const auto& mv : e->movies) per = per / gcd_ll(per, mv.d.interval) * mv.d.interval;
  if (e->have_nf2ff) per = per / gcd_ll(per, e->nf2ff.batch) * e->nf2ff.batch;
  if (e->watchdog > 0) per = per / gcd_ll(per, e->watchdog) * e->watchdog;
  if (is_pingpong(e) && per % 2) per *= 2;  // buffers alternate every step
  return per;
}

xfd_status ensure_ready(xfd_engine* e) {
  if (!e->have_classes) return fail(e, XFD_ERR_STATE, "material classes not set");
  if (!e->have_curl) return fail(e, XFD_ERR_STATE, "curl factors not set");
  if (uses_tma(e) && !e->tma_ready) {
    xfd_status st = e->precision == XFD_FP64 ? build_tma_maps<double>(e) : build_tma_maps<float>(e);
    if (st != XFD_OK) return st;
  }
  if (e->xlayer_slabs != e->slabs.size()) {
    // Per x plane the layer of the x-normal CPML slabs, for the H and the E
    // layers: (layer << 1) | slab, or -1 outside every slab.
    std::vector<int2> xl((size_t)e->L.nx + 1, make_int2(-1, -1));
    int q[2] = {0, 0};
    for (const auto& S : e->slabs) {
      if (S.m != 0) continue;
      const int slot = q[0]++;
      for (int l = 0; l < S.n; ++l) {
        xl[(size_t)S.h_lo + l].x = (l << 1) | slot;
        xl[(size_t)S.e_lo + l].y = (l << 1) | slot;
      }
    }
    if (!e->d_xlayer) {
      void* p = nullptr;
      xfd_status st = dev_alloc(e, &p, xl.size() * sizeof(int2));
      if (st != XFD_OK) return st;
      e->d_xlayer = static_cast<int2*>(p);
    }
    CUDA_TRY(e, cudaMemcpy(e->d_xlayer, xl.data(), xl.size() * sizeof(int2),
                           cudaMemcpyHostToDevice));
    e->xlayer_slabs = e->slabs.size();
    e->graph_dirty = true;
  }
  if (e->kernel_mode == 4 || e->kernel_mode == 7) {
    xfd_status st = build_march_tiles(e);
    if (st == XFD_OK && e->kernel_mode == 7) st = build_hyb_tiles(e);
    if (st != XFD_OK) return st;
  }
  if (e->probes_dirty) {
    // Upload the probe lists (all probes in one launch per step).
    ProbeD pd{};
    pd.n_probes = (int)e->pr_begin.size() - 1;
    pd.n_steps = e->n_steps;
    long long *db = nullptr, *dn = nullptr;
    uint8_t* dc = nullptr;
    double* dw = nullptr;
    xfd_status st;
    if ((st = upload_raw(e, &db, e->pr_begin.data(), e->pr_begin.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dn, e->pr_node.data(), e->pr_node.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dc, e->pr_comp.data(), e->pr_comp.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dw, e->pr_w.data(), e->pr_w.size())) != XFD_OK) return st;
    void* ser = nullptr;
    if ((st = dev_alloc(e, &ser, (size_t)pd.n_probes * e->n_steps * sizeof(double))) != XFD_OK)
      return st;
    // keep the series recorded so far
    if (e->probes.series && e->probes.n_probes)
      CUDA_TRY(e, cudaMemcpyAsync(ser, e->probes.series,
                                  (size_t)e->probes.n_probes * e->n_steps * sizeof(double),
                                  cudaMemcpyDeviceToDevice, e->stream));
    pd.begin = db;
    pd.node = dn;
    pd.comp = dc;
    pd.w = dw;
    pd.series = static_cast<double*>(ser);
    e->probes = pd;
    e->probes_dirty = false;
    e->graph_dirty = true;
  }
  if (e->lumped_dirty) {
    // Concatenate the current sources into one device list.
    std::vector<long long> node;
    std::vector<int> comp, src;
    std::vector<double> coff, wave;
    for (size_t q = 0; q < e->lumped_h.size(); ++q) {
      const auto& l = e->lumped_h[q];
      for (size_t n = 0; n < l.node.size(); ++n) {
        node.push_back(l.node[n]);
        comp.push_back(l.comp);
        src.push_back((int)q);
        coff.push_back(l.coff[n]);
      }
      wave.insert(wave.end(), l.wave.begin(), l.wave.end());
    }
    LumpedD d{};
    d.n = (long long)node.size();
    d.n_steps = (int)e->n_steps;
    long long* dn = nullptr;
    int *dc = nullptr, *ds = nullptr;
    double *dco = nullptr, *dw = nullptr;
    xfd_status st;
    if ((st = upload_raw(e, &dn, node.data(), node.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dc, comp.data(), comp.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &ds, src.data(), src.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dco, coff.data(), coff.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dw, wave.data(), wave.size())) != XFD_OK) return st;
    d.node = dn;
    d.comp = dc;
    d.source = ds;
    d.coff = dco;
    d.wave = dw;
    e->lumped = d;
    e->lumped_dirty = false;
  }
  if (e->ind_dirty) {
    // Concatenate the inductors; their current state starts at zero.
    std::vector<long long> node;
    std::vector<int> comp;
    std::vector<double> cecjc, cjcec;
    for (const auto& l : e->ind_h) {
      node.insert(node.end(), l.node.begin(), l.node.end());
      comp.insert(comp.end(), l.node.size(), l.comp);
      cecjc.insert(cecjc.end(), l.cecjc.begin(), l.cecjc.end());
      cjcec.insert(cjcec.end(), l.cjcec.begin(), l.cjcec.end());
    }
    InductorD d{};
    d.n = (long long)node.size();
    long long* dn = nullptr;
    int* dc = nullptr;
    double *da = nullptr, *db = nullptr, *dj = nullptr;
    const std::vector<double> zero(node.size(), 0.0);
    xfd_status st;
    if ((st = upload_raw(e, &dn, node.data(), node.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dc, comp.data(), comp.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &da, cecjc.data(), cecjc.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &db, cjcec.data(), cjcec.size())) != XFD_OK) return st;
    if ((st = upload_raw(e, &dj, zero.data(), zero.size())) != XFD_OK) return st;
    d.node = dn;
    d.comp = dc;
    d.cecjc = da;
    d.cjcec = db;
    d.j = dj;
    e->ind = d;
    e->ind_dirty = false;
  }
  return XFD_OK;
}

void drop_graph(xfd_engine* e) {
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  e->graph_exec = nullptr;
  e->graph_len = 0;
}

xfd_status build_graph(xfd_engine* e, long long t0) {
  drop_graph(e);
  const long long per = pattern_period(e);
  long long len = per;
  while (len < e->graph_chunk) len += per;
  cudaGraph_t g = nullptr;
  const int cur0 = e->cur;
  CUDA_TRY(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  for (long long s = 0; s < len; ++s) {
    cudaError_t c = enqueue_step(e, t0 + s);
    if (c != cudaSuccess) {
      e->cur = cur0;
      cudaGraph_t dummy;
      cudaStreamEndCapture(e->stream, &dummy);
      if (dummy) cudaGraphDestroy(dummy);
      return fail(e, XFD_ERR_CUDA, "kernel launch during capture: %s", cudaGetErrorString(c));
    }
  }
  e->cur = cur0;  // capture only recorded the launches
  CUDA_TRY(e, cudaStreamEndCapture(e->stream, &g));
  cudaError_t c = cudaGraphInstantiate(&e->graph_exec, g, 0);
  cudaGraphDestroy(g);
  if (c != cudaSuccess) return fail(e, XFD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(c));
  e->graph_len = len;
  e->graph_cur = cur0;
  e->graph_dirty = false;
  return XFD_OK;
}

// Queues the D2H copy of every movie frame finished so far on the copy
// stream, ordered after the compute stream's work to date, so that it
// overlaps the following steps.
xfd_status queue_frame_copies(xfd_engine* e) {
  bool any = false;
  for (auto& m : e->movies) {
    const long long done = std::min<long long>((e->host_step + m.d.interval - 1) / m.d.interval,
                                               m.d.max_frames);
    if (done > m.copied) any = true;
  }
  if (!any) return XFD_OK;
  CUDA_TRY(e, cudaEventRecord(e->copy_ev, e->stream));
  CUDA_TRY(e, cudaStreamWaitEvent(e->copy_stream, e->copy_ev, 0));
  for (auto& m : e->movies) {
    const long long done = std::min<long long>((e->host_step + m.d.interval - 1) / m.d.interval,
                                               m.d.max_frames);
    if (done <= m.copied) continue;
    const size_t per = (size_t)m.n_nodes * e->wsize;
    CUDA_TRY(e, cudaMemcpyAsync(static_cast<char*>(m.host) + m.copied * per,
                                static_cast<char*>(m.d.store) + m.copied * per,
                                (size_t)(done - m.copied) * per, cudaMemcpyDeviceToHost,
                                e->copy_stream));
    m.copied = done;
  }
  return XFD_OK;
}

xfd_status flush_nf2ff(xfd_engine* e) {
  if (!e->have_nf2ff) return XFD_OK;
  const long long pending = e->host_step - e->nf_last_flush_step;
  const long long done_batches = (e->host_step / e->nf2ff.batch) * e->nf2ff.batch;
  // Steps after the last full batch boundary are not yet folded in.
  const long long t0 = std::max(done_batches, e->nf_last_flush_step);
  const long long nb = e->host_step - t0;
  (void)pending;
  if (nb > 0) {
    const size_t smem = (size_t)2 * e->nf2ff.nf * e->nf2ff.batch * sizeof(double2);
    k_nf2ff_dft<8><<<blocks_for(4 * e->nf2ff.P, 256), 256, smem, e->stream>>>(
        e->nf2ff, e->d_step, (int)nb, t0);
    CUDA_TRY(e, cudaGetLastError());
    // Zero the folded slots so the batch-end DFT of this window adds nothing
    // for them again.
    const long long slot0 = t0 % e->nf2ff.batch;
    CUDA_TRY(e, cudaMemsetAsync(e->nf2ff.sample + slot0 * 4 * e->nf2ff.P, 0,
                                (size_t)nb * 4 * e->nf2ff.P * sizeof(double), e->stream));
  }
  e->nf_last_flush_step = e->host_step;
  return XFD_OK;
}

}  // namespace

extern "C" {

xfd_status xfd_create(const xfd_grid_desc* g, xfd_engine** out) {
  if (!g || !out) return fail(nullptr, XFD_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return fail(nullptr, XFD_ERR_INVALID_ARGUMENT, "grid too small (%d, %d, %d)", g->nx, g->ny,
                g->nz);
  if (g->precision != XFD_FP64 && g->precision != XFD_FP32)
    return fail(nullptr, XFD_ERR_INVALID_ARGUMENT, "unknown precision %d", g->precision);
  if (g->n_steps < 0) return fail(nullptr, XFD_ERR_INVALID_ARGUMENT, "negative n_steps");
  auto e = std::make_unique<xfd_engine>();
  e->device = g->device;
  cudaError_t c = cudaSetDevice(g->device);
  if (c != cudaSuccess)
    return fail(nullptr, XFD_ERR_CUDA, "cudaSetDevice(%d): %s", g->device, cudaGetErrorString(c));
  c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (c != cudaSuccess) return fail(nullptr, XFD_ERR_CUDA, "stream: %s", cudaGetErrorString(c));
  c = cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking);
  if (c == cudaSuccess) c = cudaEventCreateWithFlags(&e->copy_ev, cudaEventDisableTiming);
  for (int q = 0; q < kSides && c == cudaSuccess; ++q) {
    c = cudaStreamCreateWithFlags(&e->side[q], cudaStreamNonBlocking);
    if (c == cudaSuccess) c = cudaEventCreateWithFlags(&e->join_ev[q], cudaEventDisableTiming);
  }
  if (c == cudaSuccess) c = cudaEventCreateWithFlags(&e->fork_ev, cudaEventDisableTiming);
  if (c != cudaSuccess) {
    for (int q = 0; q < kSides; ++q) {
      if (e->side[q]) cudaStreamDestroy(e->side[q]);
      if (e->join_ev[q]) cudaEventDestroy(e->join_ev[q]);
    }
    if (e->copy_ev) cudaEventDestroy(e->copy_ev);
    if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
    cudaStreamDestroy(e->stream);
    return fail(nullptr, XFD_ERR_CUDA, "copy / side streams: %s", cudaGetErrorString(c));
  }
  e->precision = g->precision;
  e->wsize = g->precision == XFD_FP64 ? 8 : 4;
  e->n_steps = g->n_steps;
  e->dt = g->dt;
  e->L.nx = g->nx;
  e->L.ny = g->ny;
  e->L.nz = g->nz;
  e->L.NY = g->ny + 1;
  e->L.KP = ((g->nz + 1) + 31) / 32 * 32;
  e->n_lat = (long long)(g->nx + 1) * e->L.NY * e->L.KP;
  // Small lattices: the marching sweeps' CTAs (a 32 x 8 tile through 16
  // planes each) would not fill the GPU twice over, so the one-thread-per-
  // node split sweep (more, shorter CTAs) is the default there.  The
  // "kernel" option overrides the choice.
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    const long long tiles = (long long)((g->nz + 31) / 32) * ((g->ny + 7) / 8) *
                            ((g->nx + 1 + 15) / 16);
    if (tiles < 2LL * sms) e->kernel_mode = 0;
  }
  if (e->n_lat > (1LL << 40))
    return fail(nullptr, XFD_ERR_INVALID_ARGUMENT, "grid too large");
  xfd_engine* ep = e.get();
  for (int k = 0; k < 12; ++k) {
    if (dev_alloc(ep, &e->fbuf[k / 6][k % 6], (size_t)e->n_lat * e->wsize) != XFD_OK) {
      g_create_error = ep->err;
      for (void* p : ep->allocs) cudaFree(p);
      cudaStreamDestroy(ep->stream);
      return g_create_error.find("cudaMalloc") != std::string::npos ? XFD_ERR_OUT_OF_MEMORY
                                                                     : XFD_ERR_CUDA;
    }
  }
  void* df = nullptr;
  void* df2 = nullptr;
  void* ds = nullptr;
  void* de = nullptr;
  if (dev_alloc(ep, &df, 6 * sizeof(void*)) != XFD_OK ||
      dev_alloc(ep, &df2, 6 * sizeof(void*)) != XFD_OK ||
      dev_alloc(ep, &ds, sizeof(long long)) != XFD_OK || dev_alloc(ep, &de, sizeof(int)) != XFD_OK) {
    g_create_error = ep->err;
    for (void* p : ep->allocs) cudaFree(p);
    cudaStreamDestroy(ep->stream);
    return XFD_ERR_CUDA;
  }
  e->d_fields[0] = static_cast<void**>(df);
  e->d_fields[1] = static_cast<void**>(df2);
  e->d_step = static_cast<long long*>(ds);
  e->d_err = static_cast<int*>(de);
  c = cudaMemcpyAsync(e->d_fields[0], e->fbuf[0], sizeof e->fbuf[0], cudaMemcpyHostToDevice,
                      e->stream);
  if (c == cudaSuccess)
    c = cudaMemcpyAsync(e->d_fields[1], e->fbuf[1], sizeof e->fbuf[1], cudaMemcpyHostToDevice,
                        e->stream);
  if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
  if (c != cudaSuccess) {
    g_create_error = cudaGetErrorString(c);
    for (void* p : ep->allocs) cudaFree(p);
    cudaStreamDestroy(ep->stream);
    return XFD_ERR_CUDA;
  }
  *out = e.release();
  return XFD_OK;
}

void xfd_destroy(xfd_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->copy_stream) cudaStreamSynchronize(e->copy_stream);
  drop_graph(e);
  for (auto& c : e->ckpts)
    if (c.buf) cudaFree(c.buf);
  for (auto& c : e->adj_ck)
    if (c.buf) cudaFree(c.buf);
  for (void* p : e->adj_bufs) cudaFree(p);
  for (void* p : e->allocs) cudaFree(p);
  for (void* p : e->host_allocs) cudaFreeHost(p);
  if (e->copy_ev) cudaEventDestroy(e->copy_ev);
  if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
  for (int q = 0; q < kSides; ++q) {
    if (e->join_ev[q]) cudaEventDestroy(e->join_ev[q]);
    if (e->side[q]) cudaStreamDestroy(e->side[q]);
  }
  if (e->fork_ev) cudaEventDestroy(e->fork_ev);
  if (e->halo_ev) cudaEventDestroy(e->halo_ev);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

const char* xfd_last_error(const xfd_engine* e) {
  return e ? e->err.c_str() : g_create_error.c_str();
}

// Message for xfd_last_error(NULL) from entry points without an engine.
void xfd_internal_set_error(const char* msg) { g_create_error = msg; }

xfd_status xfd_set_material_classes(xfd_engine* e, const double* table, int32_t n_classes,
                                    const uint16_t* lattice_class) {
  if (!e || !table || !lattice_class || n_classes <= 0 || n_classes > 65536)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad material class arguments (n_classes=%d)",
                n_classes);
  const long long n_nodes = (long long)(e->L.nx + 1) * (e->L.ny + 1) * (e->L.nz + 1);
  for (long long q = 0; q < n_nodes; ++q) {
    if (lattice_class[q] >= n_classes)
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "class index %u at node %lld >= %d",
                  lattice_class[q], q, n_classes);
  }
  CUDA_TRY(e, cudaSetDevice(e->device));
  // Relabel the classes by descending node count, so that the classes
  // covering most nodes have the smallest indices and stay hot in cache.
  std::vector<long long> freq(n_classes, 0);
  for (long long q = 0; q < n_nodes; ++q) ++freq[lattice_class[q]];
  std::vector<int> order(n_classes);
  for (int c = 0; c < n_classes; ++c) order[c] = c;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return freq[a] > freq[b]; });
  std::vector<uint16_t> remap(n_classes);
  std::vector<double> table2((size_t)n_classes * 12);
  for (int r = 0; r < n_classes; ++r) {
    remap[order[r]] = (uint16_t)r;
    for (int x = 0; x < 12; ++x) table2[(size_t)r * 12 + x] = table[(size_t)order[r] * 12 + x];
  }
  std::vector<uint16_t> lattice2((size_t)n_nodes);
  for (long long q = 0; q < n_nodes; ++q) lattice2[q] = remap[lattice_class[q]];
  lattice_class = lattice2.data();
  xfd_status s = upload_real(e, &e->tab, table2.data(), (size_t)n_classes * 12);
  if (s != XFD_OK) return s;
  void* p = nullptr;
  if ((s = dev_alloc(e, &p, (size_t)e->n_lat * sizeof(uint16_t))) != XFD_OK) return s;
  e->cls = static_cast<uint16_t*>(p);
  cudaMemcpy3DParms prm{};
  const size_t rowb = (size_t)(e->L.nz + 1) * sizeof(uint16_t);
  prm.srcPtr = make_cudaPitchedPtr(const_cast<uint16_t*>(lattice_class), rowb,
                                   (size_t)(e->L.nz + 1), (size_t)(e->L.ny + 1));
  prm.dstPtr = make_cudaPitchedPtr(p, (size_t)e->L.KP * sizeof(uint16_t), (size_t)e->L.KP,
                                   (size_t)e->L.NY);
  prm.extent = make_cudaExtent(rowb, (size_t)(e->L.ny + 1), (size_t)(e->L.nx + 1));
  prm.kind = cudaMemcpyHostToDevice;
  CUDA_TRY(e, cudaMemcpy3DAsync(&prm, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  e->n_classes = n_classes;
  e->have_classes = true;
  e->tma_ready = false;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_set_e_overrides(xfd_engine* e, int64_t n, const int32_t* node, const int32_t* comp,
                               const double* ca, const double* cb) {
  if (!e || n < 0 || (n > 0 && (!node || !comp || !ca || !cb)))
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad override arguments");
  if (!e->have_classes) return fail(e, XFD_ERR_STATE, "set the material classes first");
  if (e->n_ovr) return fail(e, XFD_ERR_STATE, "overrides already set");
  if (n == 0) return XFD_OK;
  const int nn[3] = {e->L.nx, e->L.ny, e->L.nz};
  std::vector<long long> id((size_t)n);
  std::vector<uint8_t> cm((size_t)n);
  for (int64_t q = 0; q < n; ++q) {
    const int c = comp[q];
    const int* x = node + 3 * q;
    bool ok = c >= 0 && c <= 2 && cb[q] > 0;
    for (int d = 0; d < 3 && ok; ++d)
      ok = x[d] >= 0 && (d == c ? x[d] < nn[d] : x[d] <= nn[d]);
    if (!ok) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad override entry %lld", (long long)q);
    id[(size_t)q] = lat_index(e->L, x[0], x[1], x[2]);
    cm[(size_t)q] = (uint8_t)c;
  }
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s;
  long long* dn = nullptr;
  uint8_t* dc = nullptr;
  double *dca = nullptr, *dcb = nullptr;
  if ((s = upload_raw(e, &dn, id.data(), id.size())) != XFD_OK) return s;
  if ((s = upload_raw(e, &dc, cm.data(), cm.size())) != XFD_OK) return s;
  if ((s = upload_raw(e, &dca, ca, (size_t)n)) != XFD_OK) return s;
  if ((s = upload_raw(e, &dcb, cb, (size_t)n)) != XFD_OK) return s;
  void *r = nullptr, *d = nullptr, *old = nullptr;
  if ((s = dev_alloc(e, &r, (size_t)n * e->wsize)) != XFD_OK) return s;
  if ((s = dev_alloc(e, &d, (size_t)n * e->wsize)) != XFD_OK) return s;
  if ((s = dev_alloc(e, &old, (size_t)n * e->wsize)) != XFD_OK) return s;
  if (e->precision == XFD_FP64) {
    OverrideD<double> o{n, dn, dc, static_cast<double*>(r), static_cast<double*>(d),
                        static_cast<double*>(old)};
    k_ovr_prepare<double><<<blocks_for(n, 256), 256, 0, e->stream>>>(
        o, e->cls, static_cast<const double*>(e->tab), dca, dcb);
    e->ovr64 = o;
  } else {
    OverrideD<float> o{n, dn, dc, static_cast<float*>(r), static_cast<float*>(d),
                       static_cast<float*>(old)};
    k_ovr_prepare<float><<<blocks_for(n, 256), 256, 0, e->stream>>>(
        o, e->cls, static_cast<const float*>(e->tab), dca, dcb);
    e->ovr32 = o;
  }
  CUDA_TRY(e, cudaGetLastError());
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  e->ovr_node.assign(node, node + 3 * n);
  e->ovr_comp = cm;
  e->ovr_ca.assign(ca, ca + n);
  e->ovr_cb.assign(cb, cb + n);
  e->n_ovr = n;
  e->graph_dirty = true;
  return XFD_OK;
}

namespace {
xfd_status halo_event(xfd_engine* e) {
  if (e->halo_ev) return XFD_OK;
  CUDA_TRY(e, cudaSetDevice(e->device));
  CUDA_TRY(e, cudaEventCreateWithFlags(&e->halo_ev, cudaEventDisableTiming));
  return XFD_OK;
}
}  // namespace

xfd_status xfd_halo_copy(xfd_engine* dst, int32_t dst_plane, xfd_engine* src, int32_t src_plane,
                         int32_t n_comp, const int32_t* comps) {
  if (!dst || !src || dst == src || n_comp < 1 || n_comp > 6 || !comps)
    return fail(dst, XFD_ERR_INVALID_ARGUMENT, "bad halo copy arguments");
  if (dst->precision != src->precision || dst->L.ny != src->L.ny || dst->L.nz != src->L.nz ||
      dst->L.KP != src->L.KP)
    return fail(dst, XFD_ERR_INVALID_ARGUMENT, "halo copy between lattices of other y-z extent");
  for (int q = 0; q < n_comp; ++q) {
    const int c = comps[q];
    // planes along x: nx + 1 of E_y, E_z, H_x; nx of E_x, H_y, H_z
    const int extra = (c == 1 || c == 2 || c == 3) ? 1 : 0;
    if (c < 0 || c > 5 || dst_plane < 0 || dst_plane >= dst->L.nx + extra || src_plane < 0 ||
        src_plane >= src->L.nx + extra)
      return fail(dst, XFD_ERR_INVALID_ARGUMENT, "halo copy component %d / plane out of range", c);
  }
  xfd_status st;
  if ((st = halo_event(src)) != XFD_OK) return st;
  if ((st = halo_event(dst)) != XFD_OK) return st;
  // dst waits for the source's queued steps, copies, and the source's next
  // step waits for the copy (its in-place sweeps would overwrite the plane).
  CUDA_TRY(src, cudaSetDevice(src->device));
  CUDA_TRY(src, cudaEventRecord(src->halo_ev, src->stream));
  CUDA_TRY(dst, cudaSetDevice(dst->device));
  CUDA_TRY(dst, cudaStreamWaitEvent(dst->stream, src->halo_ev, 0));
  const size_t plane = (size_t)dst->L.NY * dst->L.KP;
  for (int q = 0; q < n_comp; ++q) {
    const int c = comps[q];
    unsigned char* d = static_cast<unsigned char*>(dst->fbuf[dst->cur][c]) +
                       (size_t)dst_plane * plane * dst->wsize;
    const unsigned char* sp = static_cast<const unsigned char*>(src->fbuf[src->cur][c]) +
                              (size_t)src_plane * plane * src->wsize;
    if (dst->device == src->device)
      CUDA_TRY(dst, cudaMemcpyAsync(d, sp, plane * dst->wsize, cudaMemcpyDeviceToDevice,
                                    dst->stream));
    else
      CUDA_TRY(dst, cudaMemcpyPeerAsync(d, dst->device, sp, src->device, plane * dst->wsize,
                                        dst->stream));
  }
  CUDA_TRY(dst, cudaEventRecord(dst->halo_ev, dst->stream));
  CUDA_TRY(src, cudaSetDevice(src->device));
  CUDA_TRY(src, cudaStreamWaitEvent(src->stream, dst->halo_ev, 0));
  return XFD_OK;
}

xfd_status xfd_plane_copy(xfd_engine* e, int32_t plane, int32_t n_comp, const int32_t* comps,
                          void* buf, int32_t into_engine) {
  if (!e || n_comp < 1 || n_comp > 6 || !comps || !buf)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad plane copy arguments");
  for (int q = 0; q < n_comp; ++q) {
    const int c = comps[q];
    const int extra = (c == 1 || c == 2 || c == 3) ? 1 : 0;  // E_y, E_z, H_x: nx + 1 planes
    if (c < 0 || c > 5 || plane < 0 || plane >= e->L.nx + extra)
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "plane copy component %d / plane out of range", c);
  }
  CUDA_TRY(e, cudaSetDevice(e->device));
  const size_t bytes = (size_t)e->L.NY * e->L.KP * e->wsize;
  for (int q = 0; q < n_comp; ++q) {
    unsigned char* f =
        static_cast<unsigned char*>(e->fbuf[e->cur][comps[q]]) + (size_t)plane * bytes;
    unsigned char* b = static_cast<unsigned char*>(buf) + (size_t)q * bytes;
    // cudaMemcpyDefault: `buf` may be device memory (of any device) or host
    // memory; stream-ordered with the engine's steps either way.
    CUDA_TRY(e, cudaMemcpyAsync(into_engine ? f : b, into_engine ? b : f, bytes, cudaMemcpyDefault,
                                e->stream));
  }
  return XFD_OK;
}

int64_t xfd_plane_values(const xfd_engine* e) {
  return e ? (int64_t)e->L.NY * e->L.KP : 0;
}

xfd_status xfd_set_h_term_overrides(xfd_engine* e, int64_t n, const int32_t* node,
                                    const int32_t* comp, const double* delta_a,
                                    const double* delta_b) {
  if (!e || n < 0 || (n > 0 && (!node || !comp || !delta_a || !delta_b)))
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad H term arguments");
  if (e->n_hterm) return fail(e, XFD_ERR_STATE, "H term corrections already set");
  if (n == 0) return XFD_OK;
  const int nn[3] = {e->L.nx, e->L.ny, e->L.nz};
  std::vector<long long> id((size_t)n);
  std::vector<uint8_t> cm((size_t)n);
  std::set<std::pair<long long, int>> seen;
  for (int64_t q = 0; q < n; ++q) {
    const int c = comp[q];
    const int* x = node + 3 * q;
    bool ok = c >= 0 && c <= 2 && std::isfinite(delta_a[q]) && std::isfinite(delta_b[q]);
    for (int d = 0; d < 3 && ok; ++d) ok = x[d] >= 0 && x[d] < nn[d];  // main H range
    if (!ok) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad H term entry %lld", (long long)q);
    id[(size_t)q] = lat_index(e->L, x[0], x[1], x[2]);
    cm[(size_t)q] = (uint8_t)c;
    if (!seen.emplace(id[(size_t)q], c).second)
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "H term entry %lld repeats a node", (long long)q);
  }
  // The correction runs between a split sweep's H and E phases.
  if (e->kernel_mode == 7) {
    xfd_status st = xfd_set_option(e, "kernel", 4);
    if (st != XFD_OK) return st;
  } else if (is_pingpong(e)) {
    xfd_status st = xfd_set_option(e, "kernel", 0);
    if (st != XFD_OK) return st;
  }
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s;
  long long* dn = nullptr;
  uint8_t* dc = nullptr;
  if ((s = upload_raw(e, &dn, id.data(), id.size())) != XFD_OK) return s;
  if ((s = upload_raw(e, &dc, cm.data(), cm.size())) != XFD_OK) return s;
  if (e->precision == XFD_FP64) {
    double *da = nullptr, *db = nullptr;
    if ((s = upload_raw(e, &da, delta_a, (size_t)n)) != XFD_OK) return s;
    if ((s = upload_raw(e, &db, delta_b, (size_t)n)) != XFD_OK) return s;
    e->hterm64 = HTermD<double>{n, dn, dc, da, db};
  } else {
    std::vector<float> fa(delta_a, delta_a + n), fb(delta_b, delta_b + n);
    float *da = nullptr, *db = nullptr;
    if ((s = upload_raw(e, &da, fa.data(), fa.size())) != XFD_OK) return s;
    if ((s = upload_raw(e, &db, fb.data(), fb.size())) != XFD_OK) return s;
    e->hterm32 = HTermD<float>{n, dn, dc, da, db};
  }
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  e->n_hterm = n;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_set_curl_factors(xfd_engine* e, const double* const fe[3],
                                const double* const fh[3]) {
  if (!e || !fe || !fh) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null curl factors");
  CUDA_TRY(e, cudaSetDevice(e->device));
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int a = 0; a < 3; ++a) {
    if (!fe[a] || !fh[a]) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null curl factor axis %d", a);
    std::vector<double> he(fe[a], fe[a] + n[a] + 1);
    std::vector<double> hh(fh[a], fh[a] + n[a]);
    hh.push_back(0.0);  // pad to n+1 so both tables share one length
    xfd_status s = upload_real(e, &e->fe[a], he.data(), he.size());
    if (s != XFD_OK) return s;
    s = upload_real(e, &e->fh[a], hh.data(), hh.size());
    if (s != XFD_OK) return s;
    e->fe_h[a] = he;
    e->fh_h[a] = hh;
  }
  e->have_curl = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_add_cpml(xfd_engine* e, const xfd_cpml_slab* sl) {
  if (!e || !sl) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null slab");
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  if (sl->axis < 0 || sl->axis > 2 || sl->thickness <= 0)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad CPML slab axis/thickness");
  if (e->slabs.size() >= 6) return fail(e, XFD_ERR_UNSUPPORTED, "at most 6 CPML slabs");
  const int m = sl->axis;
  if (sl->e_start < 1 || sl->e_start + sl->thickness > n[m] + 1 || sl->h_start < 0 ||
      sl->h_start + sl->thickness > n[m])
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "CPML layers out of the grid");
  if (!sl->a_e || !sl->b_e || !sl->a_h || !sl->b_h)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "null CPML coefficient");
  // One slab per side of an axis, layers disjoint from the other side's (the
  // reference's PML objects, one per direction).
  for (const auto& O : e->slabs) {
    if (O.m != m) continue;
    if ((O.neg != 0) == (sl->negative != 0))
      return fail(e, XFD_ERR_UNSUPPORTED, "two CPML slabs on one side of axis %d", m);
    const bool e_overlap = sl->e_start < O.e_lo + O.n && O.e_lo < sl->e_start + sl->thickness;
    const bool h_overlap = sl->h_start < O.h_lo + O.n && O.h_lo < sl->h_start + sl->thickness;
    if (e_overlap || h_overlap)
      return fail(e, XFD_ERR_UNSUPPORTED, "CPML slabs on axis %d overlap", m);
  }
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_engine::Slab S{};
  S.m = m;
  S.neg = sl->negative;
  S.n = sl->thickness;
  S.e_lo = sl->e_start;
  S.h_lo = sl->h_start;
  xfd_status s;
  if ((s = upload_real(e, &S.a_e, sl->a_e, S.n)) != XFD_OK) return s;
  if ((s = upload_real(e, &S.b_e, sl->b_e, S.n)) != XFD_OK) return s;
  if ((s = upload_real(e, &S.a_h, sl->a_h, S.n)) != XFD_OK) return s;
  if ((s = upload_real(e, &S.b_h, sl->b_h, S.n)) != XFD_OK) return s;
  long long sz;
  if (m == 0) sz = (long long)S.n * e->L.NY * e->L.KP;
  else if (m == 1) sz = (long long)(e->L.nx + 1) * S.n * e->L.KP;
  else sz = (long long)(e->L.nx + 1) * e->L.NY * S.n;
  for (int w = 0; w < 2; ++w) {
    if ((s = dev_alloc(e, &S.psi_e[w], (size_t)sz * e->wsize)) != XFD_OK) return s;
    for (int b = 0; b < 2; ++b)
      if ((s = dev_alloc(e, &S.psi_h[b][w], (size_t)sz * e->wsize)) != XFD_OK) return s;
  }
  e->slabs.push_back(S);
  e->graph_dirty = true;
  return XFD_OK;
}

// xfd_set_tfsf / xfd_set_tfsf_slab.  slab: `t` is the source on a global
// lattice of which this engine holds the x-slab whose plane 0 is global plane
// x_offset; the box's x coordinates are global, and every pass is cut to the
// nodes of this lattice that it corrects.
static xfd_status set_tfsf_impl(xfd_engine* e, const xfd_tfsf_desc* t, bool slab,
                                int x_offset) {
  if (!e || !t) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null TFSF");
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int a = 0; a < 3; ++a) {
    const bool bad = (slab && a == 0)
                         ? (t->box_s[a] < 1 || t->box_e[a] <= t->box_s[a])
                         : (t->box_s[a] < 1 || t->box_e[a] > n[a] - 1 ||
                            t->box_e[a] <= t->box_s[a]);
    if (bad) return fail(e, XFD_ERR_INVALID_ARGUMENT, "TFSF box out of the grid on axis %d", a);
    if (!t->p_int[a] || !t->p_half[a]) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null projection");
  }
  if (t->aux < 3 || !t->e_inc || !t->h_inc) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad TFSF grid");
  CUDA_TRY(e, cudaSetDevice(e->device));
  TfsfD d{};
  for (int a = 0; a < 3; ++a) {
    d.bs[a] = t->box_s[a] - (a == 0 ? x_offset : 0);  // projections index from the box start
    d.te[a] = t->te[a];
    d.th[a] = t->th[a];
  }
  d.aux = t->aux;
  xfd_status s;
  double* p = nullptr;
  if ((s = upload_raw(e, &p, t->e_inc, (size_t)e->n_steps * t->aux)) != XFD_OK) return s;
  d.e_inc = p;
  if ((s = upload_raw(e, &p, t->h_inc, (size_t)e->n_steps * (t->aux - 1))) != XFD_OK) return s;
  d.h_inc = p;
  for (int a = 0; a < 3; ++a) {
    const int sz = t->box_e[a] - t->box_s[a];
    if ((s = upload_raw(e, &p, t->p_int[a], (size_t)sz + 1)) != XFD_OK) return s;
    d.p_int[a] = p;
    if ((s = upload_raw(e, &p, t->p_half[a], (size_t)sz + 2)) != XFD_OK) return s;
    d.p_half[a] = p;
  }
  e->tfsf = d;
  // Pass table in the order of TFSF3DCorrector::correctE/correctH; group 1
  // takes each component's first face axis, group 2 its second.
  struct PassSpec { int axis, neg, field; };
  static const PassSpec h1[6] = {{0, 1, 1}, {0, 0, 1}, {1, 1, 0}, {1, 0, 0}, {0, 1, 2}, {0, 0, 2}};
  static const PassSpec h2[6] = {{2, 1, 0}, {2, 0, 0}, {1, 1, 2}, {1, 0, 2}, {2, 1, 1}, {2, 0, 1}};
  static const PassSpec e1[6] = {{0, 1, 2}, {0, 0, 2}, {2, 1, 1}, {2, 0, 1}, {2, 1, 0}, {2, 0, 0}};
  static const PassSpec e2[6] = {{1, 1, 2}, {1, 0, 2}, {0, 1, 1}, {0, 0, 1}, {1, 1, 0}, {1, 0, 0}};
  const PassSpec* groups[4] = {h1, h2, e1, e2};
  for (int g = 0; g < 4; ++g) {
    TfsfGroupD G{};
    G.n = 6;
    const bool is_e = g >= 2;
    long long begin = 0;
    for (int q = 0; q < 6; ++q) {
      const PassSpec& ps = groups[g][q];
      TfsfPassD P{};
      P.axis = ps.axis;
      P.neg = ps.neg;
      P.field = ps.field;
      P.is_e = is_e;
      const int m = ps.axis, A = (m + 1) % 3, B = (m + 2) % 3;
      for (int a = 0; a < 3; ++a) {
        P.s[a] = t->box_s[a] - (a == 0 ? x_offset : 0);
        P.e[a] = t->box_e[a] - (a == 0 ? x_offset : 0);
      }
      // offset_a / offset_b (src/include/waveform_source/tfsf_corrector.h:122-140)
      const bool off_a = (is_e && ps.field == B) || (!is_e && ps.field == A);
      if (off_a) P.e[A] += 1; else P.e[B] += 1;
      const int cs = ps.neg ? P.s[m] : P.e[m];  // the box start / end along m
      P.s[m] = cs;
      P.e[m] = cs + 1;
      if (slab) {
        // Cut along x to the nodes of this lattice the pass corrects: x of
        // the corrected node is i - 1 on a negative H face along x, else i;
        // E_x, H_y and H_z have nx values along x, the others nx + 1.  (As
        // the reference cuts its TFSF by the domain it runs on,
        // src/waveform_source/tfsf_3d.cpp:21-33.)
        const int sh = (!is_e && ps.neg && m == 0) ? 1 : 0;
        const bool cells = is_e ? ps.field == 0 : ps.field != 0;
        const int hi = (cells ? n[0] : n[0] + 1) + sh;
        const int s0 = std::max(P.s[0], sh), e0 = std::max(std::min(P.e[0], hi), s0);
        P.s[0] = s0;
        P.e[0] = e0;
      }
      const int equation_flag = is_e ? 1 : -1;
      const int different_flag = (ps.field == A) ? -1 : 1;
      const int direction_flag = ps.neg ? -1 : 1;
      const double coef = is_e ? t->ca[m] : t->cb[m];
      P.coeff = coef * (double)(equation_flag * different_flag * direction_flag);
      P.begin = begin;
      begin += (long long)(P.e[0] - P.s[0]) * (P.e[1] - P.s[1]) * (P.e[2] - P.s[2]);
      G.pass[q] = P;
    }
    G.total = begin;
    e->tfsf_groups[g] = G;
  }
  // Per-component H passes for the fused sweep, in pass order: the node the
  // pass corrects sits half a cell outside the box on a negative face.
  TfsfHD th{};
  for (int g = 0; g < 2; ++g)
    for (int q = 0; q < 6; ++q) {
      const TfsfPassD& P = e->tfsf_groups[g].pass[q];
      const int c = P.field, m = P.axis;
      TfsfHPass hp{};
      hp.m = m;
      hp.neg = P.neg;
      hp.dual = (c == (m + 1) % 3) ? (m + 2) % 3 : (m + 1) % 3;
      for (int a = 0; a < 3; ++a) {
        hp.lo[a] = P.s[a];
        hp.hi[a] = P.e[a];
      }
      if (P.neg) {
        hp.lo[m] -= 1;
        hp.hi[m] -= 1;
      }
      hp.coeff = P.coeff;
      th.pass[c][th.n[c]++] = hp;
    }
  e->tfsf_h = th;
  e->have_tfsf = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_set_tfsf(xfd_engine* e, const xfd_tfsf_desc* t) {
  return set_tfsf_impl(e, t, false, 0);
}

xfd_status xfd_set_tfsf_slab(xfd_engine* e, const xfd_tfsf_desc* t, int32_t x_offset) {
  return set_tfsf_impl(e, t, true, x_offset);
}

xfd_status xfd_add_current_source(xfd_engine* e, int32_t comp, const int32_t box_s[3],
                                  const int32_t box_e[3], const double* coff,
                                  const double* waveform) {
  if (!e || !box_s || !box_e || !coff || !waveform || comp < 0 || comp > 2)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad current source arguments");
  int shp[3];
  comp_shape(e->L, comp, shp);
  LumpedH l;
  l.comp = comp;
  for (int a = 0; a < 3; ++a) {
    if (box_s[a] < 0 || box_e[a] > shp[a] || box_e[a] <= box_s[a])
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "current source box out of range on axis %d", a);
  }
  long long q = 0;
  for (int i = box_s[0]; i < box_e[0]; ++i)
    for (int j = box_s[1]; j < box_e[1]; ++j)
      for (int k = box_s[2]; k < box_e[2]; ++k, ++q) {
        l.node.push_back(lat_index(e->L, i, j, k));
        l.coff.push_back(coff[q]);
      }
  l.wave.assign(waveform, waveform + e->n_steps);
  e->lumped_h.push_back(std::move(l));
  e->lumped_dirty = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_add_inductor(xfd_engine* e, int32_t comp, const int32_t box_s[3],
                            const int32_t box_e[3], const double* cecjc, const double* cjcec) {
  if (!e || !box_s || !box_e || !cecjc || !cjcec || comp < 0 || comp > 2)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad inductor arguments");
  if (e->ind.n > 0) return fail(e, XFD_ERR_STATE, "inductors are added before the first step");
  int shp[3];
  comp_shape(e->L, comp, shp);
  for (int a = 0; a < 3; ++a)
    if (box_s[a] < 0 || box_e[a] > shp[a] || box_e[a] <= box_s[a])
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "inductor box out of range on axis %d", a);
  xfd_engine::InductorH l;
  l.comp = comp;
  long long q = 0;
  for (int i = box_s[0]; i < box_e[0]; ++i)
    for (int j = box_s[1]; j < box_e[1]; ++j)
      for (int k = box_s[2]; k < box_e[2]; ++k, ++q) {
        l.node.push_back(lat_index(e->L, i, j, k));
        l.cecjc.push_back(cecjc[q]);
        l.cjcec.push_back(cjcec[q]);
      }
  e->ind_h.push_back(std::move(l));
  e->ind_dirty = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_set_ade(xfd_engine* e, const xfd_ade_desc* a) {
  if (!e || !a) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null ADE");
  if (a->kind < 0 || a->kind > 2 || a->n_poles <= 0 || a->n_materials <= 0 ||
      a->n_materials > 256 || a->n_entries < 0)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad ADE description");
  if (e->ade_kind >= 0) return fail(e, XFD_ERR_STATE, "ADE already set");
  CUDA_TRY(e, cudaSetDevice(e->device));
  const long long n = a->n_entries;
  std::vector<long long> node(n);
  for (long long q = 0; q < n; ++q) {
    const int c = a->comp[q];
    const int i = a->node[3 * q], j = a->node[3 * q + 1], k = a->node[3 * q + 2];
    int shp[3];
    comp_shape(e->L, c, shp);
    if (c > 2 || i < 0 || j < 0 || k < 0 || i >= shp[0] || j >= shp[1] || k >= shp[2] ||
        a->material[q] >= a->n_materials)
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad ADE entry %lld", q);
    node[q] = lat_index(e->L, i, j, k);
  }
  xfd_status s;
  long long* dn = nullptr;
  uint8_t *dc = nullptr, *dm = nullptr;
  if ((s = upload_raw(e, &dn, node.data(), (size_t)n)) != XFD_OK) return s;
  if ((s = upload_raw(e, &dc, a->comp, (size_t)n)) != XFD_OK) return s;
  if ((s = upload_raw(e, &dm, a->material, (size_t)n)) != XFD_OK) return s;
  void* coef = nullptr;
  if ((s = upload_real(e, &coef, a->mat_coeff, (size_t)a->n_materials * (2 + 7 * a->n_poles))) !=
      XFD_OK)
    return s;
  void *j = nullptr, *jp = nullptr, *ep = nullptr, *ec = nullptr;
  if ((s = dev_alloc(e, &j, (size_t)n * a->n_poles * e->wsize)) != XFD_OK) return s;
  if ((s = dev_alloc(e, &ec, (size_t)n * e->wsize)) != XFD_OK) return s;
  if (a->kind == 0) {
    if ((s = dev_alloc(e, &jp, (size_t)n * a->n_poles * e->wsize)) != XFD_OK) return s;
    if ((s = dev_alloc(e, &ep, (size_t)n * e->wsize)) != XFD_OK) return s;
  }
  if (e->precision == XFD_FP64) {
    AdeD<double> d{n, a->n_poles, dn, dc, dm, static_cast<double*>(coef), static_cast<double*>(j),
                   static_cast<double*>(jp), static_cast<double*>(ep), static_cast<double*>(ec)};
    e->ade64 = d;
  } else {
    AdeD<float> d{n, a->n_poles, dn, dc, dm, static_cast<float*>(coef), static_cast<float*>(j),
                  static_cast<float*>(jp), static_cast<float*>(ep), static_cast<float*>(ec)};
    e->ade32 = d;
  }
  e->ade_kind = a->kind;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_set_nf2ff(xfd_engine* e, const xfd_nf2ff_desc* d) {
  if (!e || !d || d->n_freq <= 0 || !d->te || !d->th || d->batch <= 0 || d->batch > 1024)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad NF2FF description");
  if (e->have_nf2ff) return fail(e, XFD_ERR_STATE, "NF2FF already set");
  CUDA_TRY(e, cudaSetDevice(e->device));
  Nf2ffD nf{};
  nf.nf = d->n_freq;
  nf.batch = d->batch;
  nf.scale = d->scale;
  nf.n_steps = (int)e->n_steps;
  long long total = 0;
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int f = 0; f < 6; ++f) {
    nf.begin[f] = total;
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      nf.s[f][a] = d->task_s[f][a];
      nf.e[f][a] = d->task_e[f][a];
      if (nf.e[f][a] <= nf.s[f][a]) empty = true;
    }
    if (empty) {
      for (int a = 0; a < 3; ++a) nf.s[f][a] = nf.e[f][a] = 0;
      continue;
    }
    for (int a = 0; a < 3; ++a) {
      // interpolation stencils read one node on either side
      if (nf.s[f][a] < 1 || nf.e[f][a] > n[a])
        return fail(e, XFD_ERR_INVALID_ARGUMENT, "NF2FF face %d out of range", f);
    }
    total += (long long)(nf.e[f][0] - nf.s[f][0]) * (nf.e[f][1] - nf.s[f][1]) *
             (nf.e[f][2] - nf.s[f][2]);
  }
  nf.begin[6] = total;
  nf.P = total;
  xfd_status s;
  void* p = nullptr;
  if ((s = dev_alloc(e, &p, (size_t)nf.batch * 4 * total * sizeof(double))) != XFD_OK) return s;
  nf.sample = static_cast<double*>(p);
  if ((s = dev_alloc(e, &p, (size_t)nf.nf * 4 * total * sizeof(double2))) != XFD_OK) return s;
  nf.acc = static_cast<double2*>(p);
  if ((s = dev_alloc(e, &p, (size_t)nf.nf * 4 * total * sizeof(double2))) != XFD_OK) return s;
  nf.comp = static_cast<double2*>(p);
  double* q = nullptr;
  if ((s = upload_raw(e, &q, d->te, (size_t)nf.nf * e->n_steps * 2)) != XFD_OK) return s;
  nf.te = reinterpret_cast<const double2*>(q);
  if ((s = upload_raw(e, &q, d->th, (size_t)nf.nf * e->n_steps * 2)) != XFD_OK) return s;
  nf.th = reinterpret_cast<const double2*>(q);
  const size_t smem = (size_t)2 * nf.nf * nf.batch * sizeof(double2);
  if (smem > 200 * 1024) return fail(e, XFD_ERR_UNSUPPORTED, "n_freq * batch too large");
  CUDA_TRY(e, cudaFuncSetAttribute(k_nf2ff_dft<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  e->nf2ff = nf;
  e->have_nf2ff = true;
  e->nf_last_flush_step = e->host_step;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_nf2ff_far_field(xfd_engine* e, const xfd_far_field_desc* d, double* out,
                               int64_t capacity) {
  if (!e || !e->have_nf2ff) return fail(e, XFD_ERR_STATE, "no NF2FF");
  if (!d || !out || !d->theta || !d->phi || !d->freqs || d->n_angles < 1)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad far-field arguments");
  const Nf2ffD& nf = e->nf2ff;
  if (d->n_freq != nf.nf)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "far field: %d frequencies, NF2FF has %d",
                d->n_freq, nf.nf);
  const long long total = (long long)nf.nf * 4 * d->n_angles;
  if (capacity < total) return fail(e, XFD_ERR_INVALID_ARGUMENT, "far-field buffer too small");
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int a = 0; a < 3; ++a)
    if (!d->node_e[a] || !d->node_h[a] || !d->size_e[a])
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "null grid axis %d", a);
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status st = flush_nf2ff(e);
  if (st != XFD_OK) return st;
  // Host tables: per angle the theta-hat / phi-hat components of x, y, z and
  // sin(theta) cos/sin(phi) (cCSToSCSTransformMatrix), per frequency 2 pi f / c.
  const int na = d->n_angles;
  std::vector<double> ang((size_t)na * 8), cos_t(na), k0(nf.nf);
  for (int q = 0; q < na; ++q) {
    const double ct = std::cos(d->theta[q]), stt = std::sin(d->theta[q]);
    const double cp = std::cos(d->phi[q]), sp = std::sin(d->phi[q]);
    double* T = &ang[(size_t)q * 8];
    T[0] = ct * cp;
    T[1] = ct * sp;
    T[2] = -1 * stt;
    T[3] = -1 * sp;
    T[4] = cp;
    T[5] = 0.0;
    T[6] = stt * cp;
    T[7] = stt * sp;
    cos_t[q] = ct;
  }
  const double pi = 3.14159265358979323846;
  const double eps0 = 8.854187817e-12, mu0 = 4 * pi * 1e-7;
  const double c0 = 1 / std::sqrt(eps0 * mu0);
  for (int f = 0; f < nf.nf; ++f) k0[f] = 2.0 * pi * d->freqs[f] / c0;
  // Temporary device copies (freed before returning).
  std::vector<void*> tmp;
  auto up = [&](const double* src, size_t count, const double** dst) -> xfd_status {
    void* p = nullptr;
    cudaError_t c = cudaMalloc(&p, count * sizeof(double));
    if (c != cudaSuccess) return fail(e, XFD_ERR_OUT_OF_MEMORY, "far field: %s", cudaGetErrorString(c));
    tmp.push_back(p);
    c = cudaMemcpyAsync(p, src, count * sizeof(double), cudaMemcpyHostToDevice, e->stream);
    if (c != cudaSuccess) return fail(e, XFD_ERR_CUDA, "far field: %s", cudaGetErrorString(c));
    *dst = static_cast<const double*>(p);
    return XFD_OK;
  };
  FarFieldD fd{};
  fd.nf = nf.nf;
  fd.n_ang = na;
  fd.P = nf.P;
  for (int f = 0; f < 7; ++f) fd.begin[f] = nf.begin[f];
  for (int f = 0; f < 6; ++f)
    for (int a = 0; a < 3; ++a) {
      fd.s[f][a] = nf.s[f][a];
      fd.e[f][a] = nf.e[f][a];
    }
  fd.acc = nf.acc;
  fd.comp = nf.comp;
  for (int a = 0; a < 3; ++a) fd.origin[a] = d->origin[a];
  xfd_status s2 = XFD_OK;
  double2* dout = nullptr;
  do {
    if ((s2 = up(ang.data(), ang.size(), &fd.ang)) != XFD_OK) break;
    if ((s2 = up(cos_t.data(), cos_t.size(), &fd.cos_t)) != XFD_OK) break;
    if ((s2 = up(k0.data(), k0.size(), &fd.k0)) != XFD_OK) break;
    for (int a = 0; a < 3 && s2 == XFD_OK; ++a) {
      if ((s2 = up(d->node_e[a], (size_t)n[a] + 1, &fd.node_e[a])) != XFD_OK) break;
      if ((s2 = up(d->node_h[a], (size_t)n[a], &fd.node_h[a])) != XFD_OK) break;
      s2 = up(d->size_e[a], (size_t)n[a], &fd.size_e[a]);
    }
    if (s2 != XFD_OK) break;
    cudaError_t c = cudaMalloc(reinterpret_cast<void**>(&dout), total * sizeof(double2));
    if (c != cudaSuccess) {
      s2 = fail(e, XFD_ERR_OUT_OF_MEMORY, "far field: %s", cudaGetErrorString(c));
      break;
    }
    tmp.push_back(dout);
    fd.out = dout;
    if (nf.P > 0) {
      k_far_field<<<dim3((unsigned)na, (unsigned)nf.nf), 256, 0, e->stream>>>(fd);
    } else {
      cudaMemsetAsync(dout, 0, total * sizeof(double2), e->stream);
    }
    c = cudaGetLastError();
    if (c == cudaSuccess)
      c = cudaMemcpyAsync(out, dout, total * sizeof(double2), cudaMemcpyDeviceToHost, e->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    if (c != cudaSuccess) s2 = fail(e, XFD_ERR_CUDA, "far field: %s", cudaGetErrorString(c));
  } while (false);
  cudaStreamSynchronize(e->stream);
  for (void* p : tmp) cudaFree(p);
  return s2;
}

xfd_status xfd_set_nf2ff_td(xfd_engine* e, const xfd_nf2ff_td_desc* d) {
  if (!e || !d || !d->delay || !d->ds || d->n_bins < 2)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad time-domain NF2FF description");
  if (e->have_td) return fail(e, XFD_ERR_STATE, "time-domain NF2FF already set");
  CUDA_TRY(e, cudaSetDevice(e->device));
  Nf2ffTdD td{};
  long long P = 0;
  const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int f = 0; f < 6; ++f) {
    td.begin[f] = P;
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      td.s[f][a] = d->task_s[f][a];
      td.e[f][a] = d->task_e[f][a];
      if (td.e[f][a] <= td.s[f][a]) empty = true;
    }
    if (empty) {
      for (int a = 0; a < 3; ++a) td.s[f][a] = td.e[f][a] = 0;
      continue;
    }
    // The interpolation reads one node on either side along the tangential axes.
    for (int a = 0; a < 3; ++a)
      if (td.s[f][a] < 1 || td.e[f][a] > n[a])
        return fail(e, XFD_ERR_INVALID_ARGUMENT, "time-domain NF2FF face %d out of range", f);
    P += (long long)(td.e[f][0] - td.s[f][0]) * (td.e[f][1] - td.s[f][1]) *
         (td.e[f][2] - td.s[f][2]);
  }
  td.begin[6] = P;
  td.P = P;
  td.n_bins = d->n_bins;
  xfd_status st;
  double *dl = nullptr, *ds = nullptr;
  if ((st = upload_raw(e, &dl, d->delay, (size_t)P)) != XFD_OK) return st;
  if ((st = upload_raw(e, &ds, d->ds, (size_t)P)) != XFD_OK) return st;
  void *prev = nullptr, *pot = nullptr;
  if ((st = dev_alloc(e, &prev, (size_t)4 * P * sizeof(double))) != XFD_OK) return st;
  if ((st = dev_alloc(e, &pot, (size_t)6 * td.n_bins * sizeof(double))) != XFD_OK) return st;
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  td.delay = dl;
  td.ds = ds;
  td.prev = static_cast<double*>(prev);
  td.pot = static_cast<double*>(pot);
  e->td = td;
  e->have_td = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_get_nf2ff_td(xfd_engine* e, double* out, int64_t capacity, int64_t* count) {
  if (!e || !count) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null argument");
  if (!e->have_td) return fail(e, XFD_ERR_STATE, "no time-domain NF2FF");
  *count = 6 * e->td.n_bins;
  if (!out) return XFD_OK;
  if (capacity < *count) return fail(e, XFD_ERR_INVALID_ARGUMENT, "buffer too small");
  CUDA_TRY(e, cudaSetDevice(e->device));
  CUDA_TRY(e, cudaMemcpyAsync(out, e->td.pot, (size_t)*count * sizeof(double),
                              cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

xfd_status xfd_add_probe(xfd_engine* e, int64_t n, const int32_t* comp, const int32_t* node,
                         const double* weight, int32_t* id) {
  if (!e || n < 0 || (n > 0 && (!comp || !node || !weight)) || !id)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad probe arguments");
  const int nn[3] = {e->L.nx, e->L.ny, e->L.nz};
  for (int64_t q = 0; q < n; ++q) {
    const int c = comp[q];
    bool ok = c >= 0 && c <= 5;
    for (int a = 0; a < 3 && ok; ++a) ok = node[3 * q + a] >= 0 && node[3 * q + a] <= nn[a];
    if (!ok) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad probe entry %lld", (long long)q);
  }
  for (int64_t q = 0; q < n; ++q) {
    e->pr_node.push_back(lat_index(e->L, node[3 * q], node[3 * q + 1], node[3 * q + 2]));
    e->pr_comp.push_back((uint8_t)comp[q]);
    e->pr_w.push_back(weight[q]);
  }
  e->pr_begin.push_back((long long)e->pr_node.size());
  *id = (int32_t)e->pr_begin.size() - 2;
  e->probes_dirty = true;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_get_probe(xfd_engine* e, int32_t id, double* out, int64_t capacity,
                         int64_t* count) {
  if (!e || !count || id < 0 || id >= (int32_t)e->pr_begin.size() - 1)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad probe id");
  *count = e->n_steps;
  if (!out) return XFD_OK;
  if (capacity < *count) return fail(e, XFD_ERR_INVALID_ARGUMENT, "buffer too small");
  CUDA_TRY(e, cudaSetDevice(e->device));
  if (!e->probes.series || id >= e->probes.n_probes) {
    std::fill(out, out + *count, 0.0);
    return XFD_OK;
  }
  CUDA_TRY(e, cudaMemcpyAsync(out, e->probes.series + (size_t)id * e->n_steps,
                              (size_t)*count * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

xfd_status xfd_get_nf2ff(xfd_engine* e, double* out, int64_t capacity, int64_t* count) {
  if (!e || !e->have_nf2ff) return fail(e, XFD_ERR_STATE, "no NF2FF");
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s = flush_nf2ff(e);
  if (s != XFD_OK) return s;
  const Nf2ffD& nf = e->nf2ff;
  const long long total = (long long)nf.nf * 4 * nf.P;
  if (count) *count = total;
  if (!out) return XFD_OK;
  if (capacity < total) return fail(e, XFD_ERR_INVALID_ARGUMENT, "NF2FF buffer too small");
  std::vector<double2> h((size_t)total), hc((size_t)total);
  CUDA_TRY(e, cudaMemcpyAsync(h.data(), nf.acc, total * sizeof(double2), cudaMemcpyDeviceToHost,
                              e->stream));
  CUDA_TRY(e, cudaMemcpyAsync(hc.data(), nf.comp, total * sizeof(double2),
                              cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  for (long long x = 0; x < total; ++x) {  // running sums + their compensation
    h[(size_t)x].x += hc[(size_t)x].x;
    h[(size_t)x].y += hc[(size_t)x].y;
  }
  // device [f][q][p] (p over all faces) -> [f][face][q][face nodes]
  long long o = 0;
  for (int f = 0; f < nf.nf; ++f)
    for (int d = 0; d < 6; ++d)
      for (int q = 0; q < 4; ++q)
        for (long long p = nf.begin[d]; p < nf.begin[d + 1]; ++p, ++o) {
          const double2 z = h[((size_t)f * 4 + q) * nf.P + p];
          out[2 * o] = z.x;
          out[2 * o + 1] = z.y;
        }
  return XFD_OK;
}

xfd_status xfd_add_movie(xfd_engine* e, int32_t field, const int32_t box_s[3],
                         const int32_t box_e[3], int32_t interval, int32_t* id) {
  if (!e || !box_s || !box_e || field < 0 || field > 5 || interval <= 0)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad movie arguments");
  int shp[3];
  comp_shape(e->L, field, shp);
  MovieH m{};
  m.d.field = field;
  m.d.interval = interval;
  long long nn = 1;
  for (int a = 0; a < 3; ++a) {
    if (box_s[a] < 0 || box_e[a] > shp[a] || box_e[a] <= box_s[a])
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "movie box out of range on axis %d", a);
    m.d.s[a] = box_s[a];
    m.d.e[a] = box_e[a];
    nn *= box_e[a] - box_s[a];
  }
  m.n_nodes = nn;
  m.d.max_frames = (e->n_steps + interval - 1) / interval;
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s = dev_alloc(e, &m.d.store, (size_t)m.d.max_frames * nn * e->wsize);
  if (s != XFD_OK) return s;
  void* h = nullptr;
  const size_t hb = std::max<size_t>((size_t)m.d.max_frames * nn * e->wsize, 16);
  cudaError_t c = cudaHostAlloc(&h, hb, cudaHostAllocDefault);
  if (c != cudaSuccess)
    return fail(e, XFD_ERR_OUT_OF_MEMORY, "pinned frame store (%zu B): %s", hb,
                cudaGetErrorString(c));
  e->host_allocs.push_back(h);
  m.host = h;
  m.copied = 0;
  e->movies.push_back(m);
  if (id) *id = (int32_t)e->movies.size() - 1;
  e->graph_dirty = true;
  return XFD_OK;
}

xfd_status xfd_get_movie_frames(xfd_engine* e, int32_t id, void* out, int64_t capacity_bytes,
                                int64_t* n_frames) {
  if (!e || id < 0 || id >= (int32_t)e->movies.size())
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad movie id");
  const auto& m = e->movies[id];
  long long frames = (e->host_step + m.d.interval - 1) / m.d.interval;
  frames = std::min(frames, m.d.max_frames);
  if (n_frames) *n_frames = frames;
  if (!out) return XFD_OK;
  const size_t bytes = (size_t)frames * m.n_nodes * e->wsize;
  if ((size_t)capacity_bytes < bytes) return fail(e, XFD_ERR_INVALID_ARGUMENT, "movie buffer too small");
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s = queue_frame_copies(e);
  if (s != XFD_OK) return s;
  CUDA_TRY(e, cudaStreamSynchronize(e->copy_stream));
  std::memcpy(out, m.host, bytes);
  return XFD_OK;
}

xfd_status xfd_upload_fields(xfd_engine* e, const void* const fields[6]) {
  if (!e || !fields) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null fields");
  CUDA_TRY(e, cudaSetDevice(e->device));
  for (int c = 0; c < 6; ++c) {
    if (!fields[c]) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null field %d", c);
    cudaMemcpy3DParms p =
        copy_parms(e, c, e->fbuf[e->cur][c], const_cast<void*>(fields[c]), true, e->wsize);
    CUDA_TRY(e, cudaMemcpy3DAsync(&p, e->stream));
  }
  // Ping-pong sweeps: the other buffer gets the same fields, so that nodes no
  // kernel writes (PEC walls, lattice-face nodes outside the CPML) hold equal
  // values in both and the sweeps need not carry them over every step.
  if (is_pingpong(e))
    for (int c = 0; c < 6; ++c)
      CUDA_TRY(e, cudaMemcpyAsync(e->fbuf[1 - e->cur][c], e->fbuf[e->cur][c],
                                  (size_t)e->n_lat * e->wsize, cudaMemcpyDeviceToDevice,
                                  e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

xfd_status xfd_download_field(xfd_engine* e, int32_t field, void* out) {
  if (!e || !out || field < 0 || field > 5) return fail(e, XFD_ERR_INVALID_ARGUMENT, "bad field");
  CUDA_TRY(e, cudaSetDevice(e->device));
  cudaMemcpy3DParms p = copy_parms(e, field, e->fbuf[e->cur][field], out, false, e->wsize);
  CUDA_TRY(e, cudaMemcpy3DAsync(&p, e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

xfd_status xfd_download_fields(xfd_engine* e, void* const fields[6]) {
  if (!e || !fields) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null fields");
  CUDA_TRY(e, cudaSetDevice(e->device));
  for (int c = 0; c < 6; ++c) {
    if (!fields[c]) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null field %d", c);
    cudaMemcpy3DParms p = copy_parms(e, c, e->fbuf[e->cur][c], fields[c], false, e->wsize);
    CUDA_TRY(e, cudaMemcpy3DAsync(&p, e->stream));
  }
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  return XFD_OK;
}

xfd_status xfd_run(xfd_engine* e, int64_t n) {
  if (!e) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null engine");
  if (n < 0) return fail(e, XFD_ERR_INVALID_ARGUMENT, "negative step count");
  if (e->host_step + n > e->n_steps)
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "run past n_steps (%lld + %lld > %lld)",
                (long long)e->host_step, (long long)n, (long long)e->n_steps);
  CUDA_TRY(e, cudaSetDevice(e->device));
  xfd_status s = ensure_ready(e);
  if (s != XFD_OK) return s;
  long long left = n;
  const long long per = pattern_period(e);
  while (left > 0) {
    const bool aligned = (e->host_step % per) == 0;
    if (e->use_graph && aligned) {
      if (e->graph_dirty || !e->graph_exec || e->graph_cur != e->cur) {
        if ((s = build_graph(e, e->host_step)) != XFD_OK) return s;
      }
      if (left >= e->graph_len) {
        CUDA_TRY(e, cudaGraphLaunch(e->graph_exec, e->stream));
        e->host_step += e->graph_len;
        if (e->graph_len % 2 && is_pingpong(e)) e->cur = 1 - e->cur;
        left -= e->graph_len;
        if ((s = queue_frame_copies(e)) != XFD_OK) return s;
        continue;
      }
    }
    cudaError_t c = enqueue_step(e, e->host_step);
    if (c != cudaSuccess) return fail(e, XFD_ERR_CUDA, "step launch: %s", cudaGetErrorString(c));
    e->host_step += 1;
    left -= 1;
  }
  return queue_frame_copies(e);
}

xfd_status xfd_sync(xfd_engine* e) {
  if (!e) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null engine");
  CUDA_TRY(e, cudaSetDevice(e->device));
  CUDA_TRY(e, cudaStreamSynchronize(e->stream));
  CUDA_TRY(e, cudaStreamSynchronize(e->copy_stream));
  int err = 0;
  CUDA_TRY(e, cudaMemcpy(&err, e->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err & 2) return fail(e, XFD_ERR_TIMEOUT, "a sweep stage wait ran out of time");
  if (err & 4) return fail(e, XFD_ERR_NUMERIC, "the watchdog found a non-finite field value");
  if (err) return fail(e, XFD_ERR_NUMERIC, "TFSF projection left the incident grid");
  return XFD_OK;
}

int64_t xfd_current_step(const xfd_engine* e) { return e ? e->host_step : -1; }

xfd_status xfd_get_option(const xfd_engine* e, const char* name, int64_t* value) {
  xfd_engine* m = const_cast<xfd_engine*>(e);
  if (!e || !name || !value) return fail(m, XFD_ERR_INVALID_ARGUMENT, "null option");
  if (!strcmp(name, "graph")) *value = e->use_graph ? 1 : 0;
  else if (!strcmp(name, "graph_chunk")) *value = e->graph_chunk;
  else if (!strcmp(name, "kernel")) *value = e->kernel_mode;
  else if (!strcmp(name, "ichunk")) *value = e->ichunk;
  else if (!strcmp(name, "march_ichunk")) *value = e->march_ichunk;
  else if (!strcmp(name, "stage_wait_cycles")) *value = e->stage_wait;
  else if (!strcmp(name, "watchdog_interval")) *value = e->watchdog;
  else if (!strcmp(name, "pdl")) *value = e->pdl ? 1 : 0;
  else if (!strcmp(name, "march_wide")) *value = e->march_wide ? 1 : 0;
  else if (!strcmp(name, "march_concurrent")) *value = e->march_concurrent ? 1 : 0;
  else if (!strcmp(name, "march_split_axes")) *value = e->march_split_axes ? 1 : 0;
  else if (!strcmp(name, "march_shift")) *value = e->march_shift ? 1 : 0;
  else if (!strcmp(name, "march_cp_stages")) *value = e->march_cp_stages;
  else return fail(m, XFD_ERR_INVALID_ARGUMENT, "unknown option '%s'", name);
  return XFD_OK;
}

xfd_status xfd_set_option(xfd_engine* e, const char* name, int64_t value) {
  if (!e || !name) return fail(e, XFD_ERR_INVALID_ARGUMENT, "null option");
  if (!strcmp(name, "graph")) {
    e->use_graph = value != 0;
  } else if (!strcmp(name, "graph_chunk")) {
    if (value < 1 || value > 4096) return fail(e, XFD_ERR_INVALID_ARGUMENT, "graph_chunk range");
    e->graph_chunk = (int)value;
  } else if (!strcmp(name, "kernel")) {
    if (value < 0 || value > 7)
      return fail(e, XFD_ERR_UNSUPPORTED, "kernel mode %lld", (long long)value);
    if (e->n_hterm && (value == 1 || value == 2 || value >= 5))
      return fail(e, XFD_ERR_UNSUPPORTED,
                  "kernel mode %lld: H curl-term corrections need a split H/E sweep (0, 3, 4)",
                  (long long)value);
    const int before = psi_h_buf(e);
    const bool was_pp = is_pingpong(e);
    e->kernel_mode = (int)value;
    const int after = psi_h_buf(e);
    if (!was_pp && is_pingpong(e)) {  // both buffers must agree on untouched nodes
      CUDA_TRY(e, cudaSetDevice(e->device));
      for (int c = 0; c < 6; ++c)
        CUDA_TRY(e, cudaMemcpyAsync(e->fbuf[1 - e->cur][c], e->fbuf[e->cur][c],
                                    (size_t)e->n_lat * e->wsize, cudaMemcpyDeviceToDevice,
                                    e->stream));
    }
    if (before != after) {  // the next step reads the H psi from another buffer
      CUDA_TRY(e, cudaSetDevice(e->device));
      for (const auto& S : e->slabs) {
        const size_t b = (S.m == 0   ? (size_t)S.n * e->L.NY * e->L.KP
                          : S.m == 1 ? (size_t)(e->L.nx + 1) * S.n * e->L.KP
                                     : (size_t)(e->L.nx + 1) * e->L.NY * S.n) *
                         e->wsize;
        for (int w = 0; w < 2; ++w)
          CUDA_TRY(e, cudaMemcpyAsync(S.psi_h[after][w], S.psi_h[before][w], b,
                                      cudaMemcpyDeviceToDevice, e->stream));
      }
    }
  } else if (!strcmp(name, "ichunk")) {
    if (value < 1 || value > 4096) return fail(e, XFD_ERR_INVALID_ARGUMENT, "ichunk range");
    e->ichunk = (int)value;
  } else if (!strcmp(name, "stage_wait_cycles")) {
    if (value < 0) return fail(e, XFD_ERR_INVALID_ARGUMENT, "stage_wait_cycles >= 0");
    e->stage_wait = value;
  } else if (!strcmp(name, "watchdog_interval")) {
    if (value < 0 || value > (1LL << 30))
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "watchdog_interval range");
    e->watchdog = value;
  } else if (!strcmp(name, "pdl")) {
    e->pdl = value != 0;
    e->graph_dirty = true;
  } else if (!strcmp(name, "march_ichunk")) {
    if (value < 1 || value > 4096)
      return fail(e, XFD_ERR_INVALID_ARGUMENT, "march_ichunk range");
    e->march_ichunk = (int)value;
  } else if (!strcmp(name, "march_wide")) {
    e->march_wide = value != 0;
  } else if (!strcmp(name, "march_concurrent")) {
    e->march_concurrent = value != 0;
  } else if (!strcmp(name, "march_split_axes")) {
    e->march_split_axes = value != 0;
  } else if (!strcmp(name, "march_shift")) {
    e->march_shift = value != 0;
  } else if (!strcmp(name, "march_cp_stages")) {
    if (value != 0 && value != 1) return fail(e, XFD_ERR_INVALID_ARGUMENT, "march_cp_stages 0 or 1");
    e->march_cp_stages = (int)value;
  } else {
    return fail(e, XFD_ERR_INVALID_ARGUMENT, "unknown option '%s'", name);
  }
  e->graph_dirty = true;
  return XFD_OK;
}

void* xfd_stream(xfd_engine* e) { return e ? (void*)e->stream : nullptr; }

int32_t xfd_launches_per_step(const xfd_engine* e) {
  if (!e) return 0;
  const bool fused = is_fused(e);
  if (e->kernel_mode == 7) {
    // box kernel, the nonempty CPML tile lists and the lattice faces of both
    // phases, the TFSF H passes outside the box, then the common tail
    const MarchLayout ml = march_layout(e);
    std::vector<int4> lists[4];
    march_tile_lists(e, lists);
    int n = 1 + 2;  // step counter, faces
    if (ml.box) n += 1;
    for (int q = 0; q < 4; ++q)
      if (!lists[q].empty()) n += 2;
    if (e->have_tfsf) n += 4;
    if (e->ade_kind >= 0) n += 1;
    if (!e->lumped_h.empty()) n += 1;
    if (!e->ind_h.empty()) n += 1;
    if (e->have_nf2ff) n += 1;
    if (e->have_td) n += 1;
    if (e->probes.n_probes) n += 1;
    if (e->watchdog == 1) n += 1;
    if (e->n_ovr) n += 1;
    return n + e->n_rec;
  }
  int n = fused ? 2 : 3;  // sweep(s) + step counter
  if (e->kernel_mode == 5 || e->kernel_mode == 6) {
    int nt[3], lo[3], hi[3];
    fmarch_split(e, nt, lo, hi);
    if (e->kernel_mode == 6) lo[0] = 2 * ((lo[0] + 1) / 2), hi[0] = 2 * (hi[0] / 2);
    if (hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2]) n += 1;  // CPML-free part
  }
  if (e->kernel_mode == 4) {
    // The two sweeps counted above become, per sweep: the lattice-face kernel
    // (k_edge_h / k_edge_e), the CPML-free box form and the CPML form's
    // nonempty tile lists.  The face kernels make up for the two.
    const MarchLayout ml = march_layout(e);
    if (ml.box) n += 2;
    std::vector<int4> lists[4];
    march_tile_lists(e, lists);
    for (int q = 0; q < 4; ++q)
      if (!lists[q].empty()) n += 2;
  }
  if (e->have_tfsf) n += fused ? 2 : 4;
  if (e->ade_kind >= 0) n += fused ? 1 : 2;
  if (!e->lumped_h.empty()) n += 1;
  if (!e->ind_h.empty()) n += 1;
  if (e->have_nf2ff) n += 1;
  if (e->have_td) n += 1;
  if (e->probes.n_probes) n += 1;
  if (e->watchdog == 1) n += 1;  // one scan per step (every K-th step otherwise)
  if (e->n_ovr) n += fused ? 1 : 2;
  if (e->n_hterm) n += 1;
  return n + e->n_rec;
}

int64_t xfd_stencil_bytes_per_step(const xfd_engine* e) {
  if (!e) return 0;
  const long long cells = (long long)e->L.nx * e->L.ny * e->L.nz;
  long long b = cells * (12LL * (long long)e->wsize + 2);
  for (const auto& s : e->slabs) {
    const int n[3] = {e->L.nx, e->L.ny, e->L.nz};
    long long slab_cells = (long long)s.n;
    for (int a = 0; a < 3; ++a)
      if (a != s.m) slab_cells *= n[a];
    b += slab_cells * 8LL * (long long)e->wsize;
  }
  return b;
}

int64_t xfd_algorithmic_bytes_per_step(const xfd_engine* e) {
  if (!e) return 0;
  const long long w = (long long)e->wsize;
  long long b = xfd_stencil_bytes_per_step(e);
  if (e->ade_kind >= 0) {
    const long long n = e->precision == XFD_FP64 ? e->ade64.n : e->ade32.n;
    const long long np = e->precision == XFD_FP64 ? e->ade64.np : e->ade32.np;
    b += n * (2 * np * w + (e->ade_kind == 0 ? 2 * np * w + 2 * w : 0));
  }
  if (e->have_tfsf)
    for (int g = 0; g < 4; ++g) b += e->tfsf_groups[g].total * 2 * w;
  if (e->have_nf2ff) {
    const Nf2ffD& nf = e->nf2ff;
    b += nf.P * 4 * 8;                                    // FP64 samples
    b += nf.P * 4LL * nf.nf * 16 * 2 / (long long)nf.batch;  // accumulators per batch
  }
  return b;
}

}  // extern "C"

#include "batch.cuh"
#include "adjoint_run.cuh"
