// libcatn_b200: catn_tc_matmul, the split-precision (3xTF32) tensor-core
// product of two FP64 matrices, as a standalone entry point.  It runs the
// same tcgen05 primitives (tcgen05.cuh) as the split-precision contraction,
// so that they can be checked on their own against an FP64 product.
#include <cuda_runtime.h>
#include <string>
#include "catn_b200.h"
#include "tcgen05.cuh"
#include "capi_internal.h"

using namespace catn_capi;

namespace {

constexpr int kTcBM = 128;   // rows per CTA tile (MMA M)
constexpr int kTcBN = 128;   // columns per CTA tile (MMA N, TMEM columns)
constexpr int kTcBK = 32;    // K per stage
constexpr int kTcThreads = 256;
constexpr uint32_t kTcTmemCols = 128;
constexpr int kTcTileBytes = kTcBM * kTcBK * 4;        // one FP32 operand tile (16 KiB)
constexpr int kTcStageBytes = 4 * kTcTileBytes;         // A hi, A lo, B hi, B lo
constexpr int kTcSmem = 2 * kTcStageBytes + 1024 + 64;  // two stages, alignment, barriers
constexpr long long kTcWaitPolls = 1LL << 24;

// C (M x N) = A (M x K) * B (K x N), column-major FP64, one 128 x 128 tile of
// C per CTA.  Two shared-memory stages of 32 values of K: while one thread's
// 4 x 3 MMAs of stage s run on the tensor cores (TMEM accumulator, completion
// committed to the stage's mbarrier), the threads load stage s + 1 from
// global memory into registers, wait until the MMAs of stage s - 1 have
// released the other buffer, and split the values into TF32 hi / lo parts
// there (K-major).  *err is set when a wait ran out (the tile is then not
// written).
__global__ void __launch_bounds__(kTcThreads) catn_tc_matmul_kernel(int M, int N, int K, const double* A, int lda,
                                                                     const double* B, int ldb, double* C, int ldc,
                                                                     int* err) {
#if defined(__CUDA_ARCH__)
  using namespace catn::tc;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_smem + 1023) & ~(uintptr_t)1023);
  uint64_t* bar = (uint64_t*)(base + 2 * kTcStageBytes);   // one per stage buffer
  uint32_t* tslot = (uint32_t*)(base + 2 * kTcStageBytes + 16);
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.x * kTcBM, n0 = (long long)blockIdx.y * kTcBN;
  if (tid == 0) {
    failed = 0;
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
  }
  if (warp == 0) tmem_alloc(tslot, kTcTmemCols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = idesc_tf32(kTcBM, kTcBN);
  const uint32_t sbo = kTcBK / 4 * 128;
  const int ns = (K + kTcBK - 1) / kTcBK;
  double va[16], vb[16];
  auto load = [&](int st) {
    const long long k0 = (long long)st * kTcBK;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int e = tid + kTcThreads * j;
      const int r = e & 127, k = e >> 7;   // A: consecutive rows (coalesced column reads)
      const long long gr = m0 + r, gk = k0 + k;
      va[j] = (gr < M && gk < K) ? A[gr + gk * (long long)lda] : 0.0;
      const int kb = e & 31, n = e >> 5;   // B: consecutive k
      const long long gn = n0 + n, gkb = k0 + kb;
      vb[j] = (gn < N && gkb < K) ? B[gkb + gn * (long long)ldb] : 0.0;
    }
  };
  if (ns > 0) load(0);
  int st = 0;
  for (; st < ns; ++st) {
    const int b = st & 1;
    float* a_hi = (float*)(base + b * kTcStageBytes);
    float* a_lo = a_hi + kTcBM * kTcBK;
    float* b_hi = a_lo + kTcBM * kTcBK;
    float* b_lo = b_hi + kTcBN * kTcBK;
    if (st >= 2) {
      // the MMAs of stage st - 2 read this buffer: the barrier's use number (st - 2) / 2
      const bool ok = mbar_wait(bar + b, (uint32_t)(((st - 2) >> 1) & 1), kTcWaitPolls);
      fence_after_sync();
      if (__syncthreads_or(!ok)) {
        if (tid == 0) failed = 1;
        break;
      }
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int e = tid + kTcThreads * j;
      float h, l;
      split_tf32(va[j], &h, &l);
      uint32_t o = kmajor_off(e & 127, e >> 7, kTcBK) / 4;
      a_hi[o] = h;
      a_lo[o] = l;
      split_tf32(vb[j], &h, &l);
      o = kmajor_off(e >> 5, e & 31, kTcBK) / 4;
      b_hi[o] = h;
      b_lo[o] = l;
    }
    fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
#pragma unroll
      for (int s = 0; s < kTcBK / 8; ++s) {
        const uint32_t off = (uint32_t)s * 2 * kLBO;
        const uint64_t dah = smem_desc(smem_u32(a_hi) + off, kLBO, sbo);
        const uint64_t dal = smem_desc(smem_u32(a_lo) + off, kLBO, sbo);
        const uint64_t dbh = smem_desc(smem_u32(b_hi) + off, kLBO, sbo);
        const uint64_t dbl = smem_desc(smem_u32(b_lo) + off, kLBO, sbo);
        mma_tf32(tmem, dah, dbh, idesc, (st > 0 || s > 0) ? 1u : 0u);
        mma_tf32(tmem, dah, dbl, idesc, 1u);
        mma_tf32(tmem, dal, dbh, idesc, 1u);
      }
      mma_commit(bar + b);
    }
    if (st + 1 < ns) load(st + 1);   // global latency under the MMAs just issued
  }
  // MMAs complete in issue order: the last committed stage's barrier covers all
  const int issued = st;   // stages whose MMAs were committed
  if (issued > 0) {
    const int last = issued - 1;
    const bool ok = mbar_wait(bar + (last & 1), (uint32_t)((last >> 1) & 1), kTcWaitPolls);
    fence_after_sync();
    if (__syncthreads_or(!ok) && tid == 0) failed = 1;
  }
  __syncthreads();
  if (K > 0 && !failed) {
    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), columns
    // 64 (w / 4) .. + 63 in two loads of 32
    const int q = warp & 3, half = warp >> 2;
    const long long row = m0 + q * 32 + lane;
    for (int c0 = half * 64; c0 < half * 64 + 64; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
      if (row < M)
        for (int i = 0; i < 32; ++i) {
          const long long col = n0 + c0 + i;
          if (col < N) C[row + col * (long long)ldc] = (double)v[i];
        }
    }
  } else if (K <= 0) {
    for (int e = tid; e < kTcBM * kTcBN; e += kTcThreads) {
      const long long r = m0 + e % kTcBM, c = n0 + e / kTcBM;
      if (r < M && c < N) C[r + c * (long long)ldc] = 0.0;
    }
  }
  if (failed && tid == 0) *err = 1;
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, kTcTmemCols);
#endif
}

}  // namespace

extern "C" catn_status catn_tc_matmul(int32_t M, int32_t N, int32_t K, const double* A, const double* B, double* C) {
  if (M < 0 || N < 0 || K < 0) return fail(CATN_EINVAL, "negative dimension");
  if (M == 0 || N == 0) return CATN_OK;
  if ((K > 0 && (!A || !B)) || !C) return fail(CATN_EINVAL, "NULL argument");
  const size_t sa = sizeof(double) * (size_t)M * (size_t)K, sb = sizeof(double) * (size_t)K * (size_t)N;
  const size_t sc = sizeof(double) * (size_t)M * (size_t)N;
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int* dErr = nullptr;
  catn_status st = CATN_OK;
  auto cleanup = [&]() {
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(dErr);
  };
  do {
    cudaError_t e;
    if ((e = cudaMalloc(&dA, sa ? sa : 8)) != cudaSuccess) { st = cuda_fail(e, "cudaMalloc"); break; }
    if ((e = cudaMalloc(&dB, sb ? sb : 8)) != cudaSuccess) { st = cuda_fail(e, "cudaMalloc"); break; }
    if ((e = cudaMalloc(&dC, sc)) != cudaSuccess) { st = cuda_fail(e, "cudaMalloc"); break; }
    if ((e = cudaMalloc(&dErr, sizeof(int))) != cudaSuccess) { st = cuda_fail(e, "cudaMalloc"); break; }
    if (sa && (e = cudaMemcpy(dA, A, sa, cudaMemcpyHostToDevice)) != cudaSuccess) { st = cuda_fail(e, "copy A"); break; }
    if (sb && (e = cudaMemcpy(dB, B, sb, cudaMemcpyHostToDevice)) != cudaSuccess) { st = cuda_fail(e, "copy B"); break; }
    if ((e = cudaMemset(dErr, 0, sizeof(int))) != cudaSuccess) { st = cuda_fail(e, "cudaMemset"); break; }
    if ((e = cudaFuncSetAttribute(catn_tc_matmul_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem)) !=
        cudaSuccess) { st = cuda_fail(e, "cudaFuncSetAttribute"); break; }
    dim3 grid((M + kTcBM - 1) / kTcBM, (N + kTcBN - 1) / kTcBN);
    catn_tc_matmul_kernel<<<grid, kTcThreads, kTcSmem>>>(M, N, K, dA, M, dB, K, dC, M, dErr);
    if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "launch"); break; }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) { st = cuda_fail(e, "kernel"); break; }
    int herr = 0;
    if ((e = cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) { st = cuda_fail(e, "copy err"); break; }
    if (herr) { st = fail(CATN_ETIMEOUT, "tensor-core wait timed out"); break; }
    if ((e = cudaMemcpy(C, dC, sc, cudaMemcpyDeviceToHost)) != cudaSuccess) { st = cuda_fail(e, "copy C"); break; }
  } while (0);
  cleanup();
  return st;
}
