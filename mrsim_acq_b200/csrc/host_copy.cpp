// host_copy.cpp — large copies between pageable host memory (the reference's Vec buffers) and the
// device, through the context's page-locked slots.  A plain cudaMemcpyAsync from pageable memory
// stages through the driver's buffers on one thread (~10 GB/s measured on the benchmark's host);
// here up to kSlots host threads each own one slot, copy their chunks of the caller's buffer into
// (out of) it and queue the DMA on the call's stream, so host copies run in parallel with each
// other and with the copy engine.  A slot's event orders its reuse: a thread refills its slot
// only after the slot's previous copy has drained.  Page-locked sources and small copies take
// the direct path.
#include <algorithm>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "mrsim_internal.h"

namespace mrsim {
namespace {

constexpr int kSlots = 8;
constexpr size_t kSlotBytes = (size_t)8 << 20;
constexpr size_t kDirectBelow = (size_t)8 << 20;

bool page_locked(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory unknown to CUDA is not an error worth keeping
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

// The context's slots, allocated on first use; false (and the direct copy) when page-locked
// memory cannot be had.
bool ensure_slots(mrsim_context* ctx) {
  if (ctx->host_pinned) return true;
  void* p = nullptr;
  if (cudaHostAlloc(&p, kSlots * kSlotBytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  std::vector<cudaEvent_t> ev(kSlots, nullptr);
  for (auto& e : ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      for (auto& f : ev)
        if (f) cudaEventDestroy(f);
      cudaFreeHost(p);
      return false;
    }
  ctx->host_pinned = p;
  ctx->host_pinned_n = kSlots * kSlotBytes;
  ctx->slot_ev = ev;
  return true;
}

int threads_for(size_t bytes) {
  const size_t chunks = (bytes + kSlotBytes - 1) / kSlotBytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return (int)std::min<size_t>({(size_t)kSlots, chunks, (size_t)hw});
}

// Runs f(t) on nt threads (t = 0 on the caller's), each with the context's device current, and
// rethrows the first error.
template <class F>
void on_threads(mrsim_context* ctx, int nt, F&& f) {
  std::vector<std::exception_ptr> err(nt);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t)
    pool.emplace_back([&, t] {
      try {
        MRSIM_CUDA(cudaSetDevice(ctx->device));
        f(t);
      } catch (...) {
        err[t] = std::current_exception();
      }
    });
  try {
    f(0);
  } catch (...) {
    err[0] = std::current_exception();
  }
  for (auto& th : pool) th.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

}  // namespace

void copy_pageable_h2d(mrsim_context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes < kDirectBelow || page_locked(src) || !ensure_slots(ctx)) {
    MRSIM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return;
  }
  const size_t chunks = (bytes + kSlotBytes - 1) / kSlotBytes;
  const int nt = threads_for(bytes);
  on_threads(ctx, nt, [&](int t) {
    char* slot = (char*)ctx->host_pinned + (size_t)t * kSlotBytes;
    for (size_t c = (size_t)t; c < chunks; c += (size_t)nt) {
      const size_t off = c * kSlotBytes, n = std::min(kSlotBytes, bytes - off);
      MRSIM_CUDA(cudaEventSynchronize(ctx->slot_ev[t]));  // the slot's previous copy has drained
      std::memcpy(slot, (const char*)src + off, n);
      MRSIM_CUDA(cudaMemcpyAsync((char*)dst + off, slot, n, cudaMemcpyHostToDevice, st));
      MRSIM_CUDA(cudaEventRecord(ctx->slot_ev[t], st));
    }
  });
}

void copy_pageable_d2h(mrsim_context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes < kDirectBelow || page_locked(dst) || !ensure_slots(ctx)) {
    MRSIM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
    return;
  }
  const size_t chunks = (bytes + kSlotBytes - 1) / kSlotBytes;
  const int nt = threads_for(bytes);
  on_threads(ctx, nt, [&](int t) {
    char* slot = (char*)ctx->host_pinned + (size_t)t * kSlotBytes;
    for (size_t c = (size_t)t; c < chunks; c += (size_t)nt) {
      const size_t off = c * kSlotBytes, n = std::min(kSlotBytes, bytes - off);
      MRSIM_CUDA(cudaEventSynchronize(ctx->slot_ev[t]));  // no earlier copy still reads the slot
      MRSIM_CUDA(cudaMemcpyAsync(slot, (const char*)src + off, n, cudaMemcpyDeviceToHost, st));
      MRSIM_CUDA(cudaEventRecord(ctx->slot_ev[t], st));
      MRSIM_CUDA(cudaEventSynchronize(ctx->slot_ev[t]));
      std::memcpy((char*)dst + off, slot, n);
    }
  });
}

}  // namespace mrsim
