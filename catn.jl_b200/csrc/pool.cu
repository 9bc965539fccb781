// libcatn_b200: process-wide cache of the device and pinned host blocks that
// networks and batches allocate (slots, input images, results, traces).
//
// Creating a network and destroying it costs a cudaMalloc and a cudaFree of
// its slot arena and a cudaMallocHost / cudaFreeHost of its input image: on a
// B200 about 10 ms to create and 30-50 ms to destroy a 10 x 10 lattice at
// Dmax 48 / chi 256, against 24 ms of contraction.  Callers that create and
// contract networks one after another (the reference's pinning loops, a
// Julia loop over disorder samples) pay that every time.  A freed block is
// kept here instead, per device and kind, and handed to the next request it
// covers (the smallest such block, at most twice the request).  At most kPoolBlocks blocks per device
// and kind are kept; an allocation that runs out of device memory frees the
// cached blocks of its device and tries again; catn_release_cached_memory()
// frees them all (a program that resets the device calls it before the
// reset: the kept addresses do not survive a reset, and nothing here can
// tell).  Blocks are handed out with their old contents: every
// user initialises what it reads (the engine resets a slot before loading an
// instance, the host image is cleared before packing).
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include <mutex>
#include <unordered_map>
#include <vector>
#include "capi_internal.h"

namespace catn_capi {

namespace {

constexpr size_t kPoolBlocks = 8;

struct Block {
  void* p;
  size_t bytes;
  int dev;
  bool host;
};

std::mutex g_pool_mu;
std::vector<Block> g_free;                  // cached blocks
std::unordered_map<void*, Block> g_live;    // blocks handed out

cudaError_t raw_alloc(void** p, size_t bytes, bool host) {
  return host ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
}
void raw_free(const Block& b) {
  if (b.host) cudaFreeHost(b.p);
  else cudaFree(b.p);
}

// Frees the cached blocks of device `dev` (all devices when dev < 0) of one
// kind, or of both kinds when `kind` < 0.  Called with the mutex held.
void drop_cached(int dev, int kind) {
  std::vector<Block> keep;
  for (const Block& b : g_free) {
    if ((dev < 0 || b.dev == dev) && (kind < 0 || (int)b.host == kind)) raw_free(b);
    else keep.push_back(b);
  }
  g_free.swap(keep);
}

}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, bool host) {
  *p = nullptr;
  if (bytes == 0) bytes = 256;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  int best = -1;
  for (size_t q = 0; q < g_free.size(); ++q) {
    const Block& b = g_free[q];
    // a block at most twice the request (plus 1 MiB): a small request never
    // takes a large block that a later large request would need
    if (b.dev == dev && b.host == host && b.bytes >= bytes && b.bytes <= 2 * bytes + (1u << 20) &&
        (best < 0 || b.bytes < g_free[best].bytes))
      best = (int)q;
  }
  if (best >= 0) {
    Block b = g_free[best];
    g_free.erase(g_free.begin() + best);
    g_live[b.p] = b;
    *p = b.p;
    return cudaSuccess;
  }
  e = raw_alloc(p, bytes, host);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();   // clear the error before retrying
    drop_cached(dev, host ? 1 : 0);
    e = raw_alloc(p, bytes, host);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  g_live[*p] = Block{*p, bytes, dev, host};
  return cudaSuccess;
}

void pool_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) return;   // not a pool block: never freed here
  const Block b = it->second;
  g_live.erase(it);
  // cudaFree / cudaFreeHost wait for the device; a cached block must not be
  // handed out while work queued before this call may still use it, so the
  // block's device is synchronised here (another device's block is freed)
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != b.dev || cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    raw_free(b);
    return;
  }
  size_t same = 0;
  for (const Block& f : g_free)
    if (f.dev == b.dev && f.host == b.host) ++same;
  if (same >= kPoolBlocks) {
    // keep the larger blocks: drop the smallest cached one if b is larger
    int small = -1;
    for (size_t q = 0; q < g_free.size(); ++q)
      if (g_free[q].dev == b.dev && g_free[q].host == b.host &&
          (small < 0 || g_free[q].bytes < g_free[small].bytes))
        small = (int)q;
    if (small < 0 || g_free[small].bytes >= b.bytes) {
      raw_free(b);
      return;
    }
    raw_free(g_free[small]);
    g_free.erase(g_free.begin() + small);
  }
  g_free.push_back(b);
}

size_t pool_cached_bytes(bool host) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  size_t s = 0;
  for (const Block& b : g_free)
    if (b.host == host) s += b.bytes;
  return s;
}

}  // namespace catn_capi

extern "C" catn_status catn_release_cached_memory(void) {
  std::lock_guard<std::mutex> lock(catn_capi::g_pool_mu);
  catn_capi::drop_cached(-1, -1);
  return CATN_OK;
}

extern "C" int64_t catn_cached_bytes(int32_t host) {
  return (int64_t)catn_capi::pool_cached_bytes(host != 0);
}
