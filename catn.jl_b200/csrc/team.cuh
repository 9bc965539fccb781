// Cooperative "team" abstraction for the CATN contraction engine.
//
// On the GPU a team is one thread block (CTA): every thread runs the same
// control logic with identical inputs, only the leader thread writes shared
// control state, and FP work is split over threads / warps.  The same source
// also compiles as plain C++ (team of one thread) for the host-side memory
// checking harness used by the CPU test-suite; that build is never part of
// the shipped library.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define CATN_HD __host__ __device__ __forceinline__
// Heavy engine routines are kept out of line so that registers are
// allocated per routine instead of for one monolithic kernel.
#define CATN_HDI __host__ __device__ __noinline__
#else
#define CATN_HD inline
#define CATN_HDI
#endif

#if defined(__CUDA_ARCH__)
#define CATN_DEVICE_PASS 1
#else
#define CATN_DEVICE_PASS 0
#endif

// CATN_LEAN = 1 (set by a translation unit before its includes) compiles the
// engine without the block Jacobi route, the blocked QR, the tensor-core
// merges and the matrix-free randomized swaps: the persistent kernel of
// launches that use none of them (FP64, svd_route != 2, rsvd != 2).
#ifndef CATN_LEAN
#define CATN_LEAN 0
#endif

namespace catn {

struct Team {
  // Shared scratch: >= 64 doubles for reductions / broadcasts, followed by a
  // larger staging area of `stage_bytes` bytes (shared memory on the GPU).
  double* red;
  char* stage;
  int stage_bytes;
  // Tensor-core staging area in shared memory and the CTA's TMEM columns
  // for the split-precision products (null / 0: none; set by the kernels
  // that allocate them, never in the host build).
  unsigned char* tcs;
  unsigned tmem;

#if CATN_DEVICE_PASS
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ int warp() const { return threadIdx.x >> 5; }
  __device__ __forceinline__ int lane() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int nwarps() const { return blockDim.x >> 5; }
  __device__ __forceinline__ int wsize() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ void wsync() const { __syncwarp(); }
  __device__ __forceinline__ double wsum(double v) const {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }
  __device__ __forceinline__ double wmax(double v) const {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
  }
  __device__ __forceinline__ int wor(int v) const { return __any_sync(0xffffffffu, v); }
#else
  int rank() const { return 0; }
  int size() const { return 1; }
  int warp() const { return 0; }
  int lane() const { return 0; }
  int nwarps() const { return 1; }
  int wsize() const { return 1; }
  void sync() const {}
  void wsync() const {}
  double wsum(double v) const { return v; }
  double wmax(double v) const { return v; }
  int wor(int v) const { return v; }
#endif
  CATN_HD bool leader() const { return rank() == 0; }

  // Sum of `v` over the whole team; every thread receives the result.
  CATN_HD double sum(double v) const {
    v = wsum(v);
    sync();
    if (lane() == 0) red[warp()] = v;
    sync();
    double s = 0.0;
    for (int w = 0; w < nwarps(); ++w) s += red[w];
    sync();
    return s;
  }
  CATN_HD double maxv(double v) const {
    v = wmax(v);
    sync();
    if (lane() == 0) red[warp()] = v;
    sync();
    double s = red[0];
    for (int w = 1; w < nwarps(); ++w) s = fmax(s, red[w]);
    sync();
    return s;
  }
  // Logical OR of `v` over the team.
  CATN_HD int any(int v) const {
    double d = sum(v ? 1.0 : 0.0);
    return d > 0.5;
  }
  // Index of the largest value (smallest index on ties) over the team's
  // (value, index) candidates; every thread receives it.  idx < 0 = none.
  CATN_HD long long argmax(double v, long long idx) const {
#if CATN_DEVICE_PASS
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, v, o);
      long long oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (oi >= 0 && (idx < 0 || ov > v || (ov == v && oi < idx))) { v = ov; idx = oi; }
    }
#endif
    sync();
    if (lane() == 0) { red[2 * warp()] = v; ((long long*)red)[2 * warp() + 1] = idx; }
    sync();
    double bv = red[0];
    long long bi = ((long long*)red)[1];
    for (int w = 1; w < nwarps(); ++w) {
      double wv = red[2 * w];
      long long wi = ((long long*)red)[2 * w + 1];
      if (wi >= 0 && (bi < 0 || wv > bv || (wv == bv && wi < bi))) { bv = wv; bi = wi; }
    }
    sync();
    return bi;
  }
  // Atomics on shared or global ints (plain operations in the host build).
#if CATN_DEVICE_PASS
  __device__ __forceinline__ int atomic_add(int* p, int v) const { return atomicAdd(p, v); }
  __device__ __forceinline__ int atomic_cas(int* p, int cmp, int val) const { return atomicCAS(p, cmp, val); }
#else
  int atomic_add(int* p, int v) const { int o = *p; *p += v; return o; }
  int atomic_cas(int* p, int cmp, int val) const { int o = *p; if (o == cmp) *p = val; return o; }
#endif
  // Exclusive prefix sum of one int per thread over the team (thread order);
  // *total receives the sum.
  CATN_HD int scan_excl(int v, int* total) const {
#if CATN_DEVICE_PASS
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane() >= o) x += y;
    }
    sync();
    int* ws = (int*)red;
    if (lane() == 31) ws[warp()] = x;
    sync();
    int base = 0, tot = 0;
    for (int w = 0; w < nwarps(); ++w) {
      if (w < warp()) base += ws[w];
      tot += ws[w];
    }
    sync();
    *total = tot;
    return base + x - v;
#else
    *total = v;
    return 0;
#endif
  }
  // Value computed by the leader, returned to every thread.
  CATN_HD long long bcast(long long v) const {
    sync();
    if (leader()) ((long long*)red)[0] = v;
    sync();
    long long r = ((long long*)red)[0];
    sync();
    return r;
  }
  CATN_HD double bcastd(double v) const {
    sync();
    if (leader()) red[0] = v;
    sync();
    double r = red[0];
    sync();
    return r;
  }
};

}  // namespace catn
