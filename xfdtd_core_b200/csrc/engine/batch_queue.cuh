// Persistent batched step: one launch per time step of many lattices, driven
// by a device work queue.  Part of engine.cu's translation unit (included by
// batch.cuh).
//
// The host lists every piece of work of one step of every lattice as an item
// of a level: 0 H sweep tiles, 1 H lattice faces (k = nz, j = ny), 2 / 3 TFSF
// H pass groups 1 / 2, 4 E sweep tiles, 5 E lattice faces, 6 / 7 TFSF E pass
// groups 1 / 2 -- the order of the engine's own step, which is the
// reference's updateH, correctH, updateE, correctE (Domain::run,
// src/domain/domain.cpp:88-114) -- and the queue holds them level by level.
// A grid of as many CTAs as fit on the GPU at once loops:
// thread 0 takes the next item with one atomicAdd on the queue head, and the
// CTA does it with the same CTA body as the multi-launch batch
// (march_tma.cuh, edge_update / tfsf_node of kernels.cuh), so every node gets
// the same arithmetic as the lattice run alone.
//
// Dependencies are per lattice: an item of level L waits until the items of
// its lattice at levels < L have finished (need[item] = their count, compared
// with the lattice's done counter, which each finished item increments after
// a device-scope fence).  Every item an item waits for sits earlier in the
// queue, so it was taken by a CTA that is running: the waits end without any
// co-residency assumption.  They are bounded all the same: after `wait_budget`
// cycles the CTA sets bit 2 of the lattice's error word (the stage-wait
// timeout bit), counts the item as done without doing it, and goes on; later
// items of that lattice see the bit and are skipped, and xfd_batch_sync
// reports XFD_ERR_TIMEOUT.
//
// Writes of one level are read by TMA loads (the async proxy) of a later level
// in the same launch, so each thread fences the generic and async proxies
// after each item, and the thread that issues the loads fences again after
// its wait (the first item of a CTA has no earlier accesses to order).  The
// last CTA to leave the queue resets the head and the done counters for the
// next launch and advances the lattices' step counters.
#pragma once

namespace {

// Face and TFSF items cover kQueueNodeIters nodes per thread (blocks of
// 32 x 32 x TJ nodes), so that their count, and with it the per-item cost of
// the queue (the atomic, the fences, the barriers), stays small beside the
// tiles.
constexpr int kQueueNodeIters = 32;

enum BatchItemKind : int {
  kQ_H_IN = 0, kQ_H_FREE, kQ_H_X, kQ_H_Y, kQ_H_Z, kQ_H_CP,  // H sweep tiles by form
  kQ_EDGE_H, kQ_TFSF_H1, kQ_TFSF_H2,
  kQ_E_IN, kQ_E_FREE, kQ_E_X, kQ_E_Y, kQ_E_Z, kQ_E_CP,  // E sweep tiles by form
  kQ_EDGE_E, kQ_TFSF_E1, kQ_TFSF_E2,
};

template <typename T>
struct BatchQueueD {
  const MarchTmaP<T>* march;  // per lattice (tensor maps for the queue's tile rows)
  const YeeP<T>* yee;
  const TfsfSceneD<T>* tfsf;
  const int4* items;  // (kind << 16 | lattice, k tile / block, j tile, chunk)
  const int* need;    // per item: finished items of its lattice to wait for
  int n_items;
  int n_lattices;
  int* head;   // next item
  int* exits;  // CTAs past the end of the queue
  int* done;   // per lattice: items finished in this launch
  long long* const* steps;
  long long wait_budget;  // cycles per dependency wait
};

template <typename T, int TJ>
__global__ void __launch_bounds__(32 * TJ, (sizeof(T) == 8 ? 2 : 4) * 8 / TJ)
    k_batch_queue(const __grid_constant__ BatchQueueD<T> q) {
  constexpr int NT = 32 * TJ;
  constexpr int MS = march_stages<T>();
  constexpr int MF = march_free_stages<T>();
  __shared__ int s_item;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = atomicAdd(q.head, 1);
    __syncthreads();
    const int t = s_item;
    if (t >= q.n_items) break;
    const int4 w = q.items[t];
    const int kind = w.x >> 16, s = w.x & 0xffff;
    const MarchTmaP<T>& P = q.march[s];
    if (tid == 0) {
      const int need = q.need[t];
      const volatile int* d = q.done + s;
      if (need > 0 && *d < need) {
        const long long t0 = clock64();
        while (*d < need) {
          if (clock64() - t0 >= q.wait_budget) {
            atomicOr(P.err, 2);
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
      fence_proxy_async_all();
    }
    const bool skip = __syncthreads_or(tid == 0 && (*(volatile int*)P.err & 2));
    if (!skip) {
      const bool tile = kind <= kQ_H_CP || (kind >= kQ_E_IN && kind <= kQ_E_CP);
      if (tile) acquire_march_maps(P.m);
      const long long node0 = (long long)w.y * (NT * kQueueNodeIters) + tid;
      switch (kind) {
        case kQ_H_IN: march_h_cta<T, TJ, 32, MF, false, true, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_H_FREE: march_h_cta<T, TJ, 32, MF, false, false, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_H_X: march_h_cta<T, TJ, 32, MF, true, false, 1, true>(P, w.y, w.z, w.w); break;
        case kQ_H_Y: march_h_cta<T, TJ, 32, MF, true, false, 2, true>(P, w.y, w.z, w.w); break;
        case kQ_H_Z: march_h_cta<T, TJ, 32, MF, true, false, 4, true>(P, w.y, w.z, w.w); break;
        case kQ_H_CP: march_h_cta<T, TJ, 32, MS, true, false, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_E_IN: march_e_cta<T, TJ, 32, MF, false, true, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_E_FREE: march_e_cta<T, TJ, 32, MF, false, false, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_E_X: march_e_cta<T, TJ, 32, MF, true, false, 1, true>(P, w.y, w.z, w.w); break;
        case kQ_E_Y: march_e_cta<T, TJ, 32, MF, true, false, 2, true>(P, w.y, w.z, w.w); break;
        case kQ_E_Z: march_e_cta<T, TJ, 32, MF, true, false, 4, true>(P, w.y, w.z, w.w); break;
        case kQ_E_CP: march_e_cta<T, TJ, 32, MS, true, false, 7, true>(P, w.y, w.z, w.w); break;
        case kQ_EDGE_H:
          for (int u = 0; u < kQueueNodeIters; ++u)
            edge_update<T, false>(q.yee[s], node0 + (long long)u * NT);
          break;
        case kQ_EDGE_E:
          for (int u = 0; u < kQueueNodeIters; ++u)
            edge_update<T, true>(q.yee[s], node0 + (long long)u * NT);
          break;
        default: {  // TFSF pass groups
          const TfsfSceneD<T>& S = q.tfsf[s];
          const int g = kind == kQ_TFSF_H1 ? 0 : kind == kQ_TFSF_H2 ? 1 : kind == kQ_TFSF_E1 ? 2 : 3;
          for (int u = 0; u < kQueueNodeIters; ++u)
            tfsf_node<T>(S.tf, S.g[g], S.L, S.fields, S.step, S.err, node0 + (long long)u * NT);
        }
      }
    }
    // This thread's accesses of the item (stage memory, fields) are ordered
    // before the TMA loads of later items.
    fence_proxy_async_all();
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(q.done + s, 1);
    }
  }
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(q.exits, 1) == (int)gridDim.x - 1) {
      // Every other CTA has left the queue: reset it for the next launch.
      __threadfence();
      for (int s = 0; s < q.n_lattices; ++s) {
        q.done[s] = 0;
        *q.steps[s] += 1;
      }
      *q.head = 0;
      *q.exits = 0;
      __threadfence();
    }
  }
}

}  // namespace
