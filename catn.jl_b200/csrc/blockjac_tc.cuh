// Split-precision (3xTF32, tcgen05) products: the pair Gram G = X_P^T X_P
// of the block Jacobi's first phase, and the two-site merges of large
// swaps.
//
// Both stream their operands through a shared-memory tile that the threads
// fill with TF32 hi / lo parts (K-major, tcgen05.cuh's layout) while one
// thread issues the MMAs of the previous tile; the global loads of the next
// tile are issued into registers before the CTA waits for the tensor core,
// so their latency overlaps the MMAs.
//   Gram:  D (128 x 32) = A (128 x K) B (K x 32), K = the pair's rows in
//          chunks of 64; A's rows 0-31 are the pair's columns and rows
//          32-127 are zero (the MMA's smallest M here is 128), B is A's
//          first 32 rows.  Accumulates in TMEM over every chunk.
//   Merge: tiles of 128 x 128 of C = A B, K in chunks of 32, read back with
//          tcgen05.ld and stored in FP64 through the caller's operand map.
// The staging area (T.tcs) and the CTA's TMEM columns (T.tmem) are set up
// by the kernel; a wait for the tensor core that runs out marks the area
// broken (later products take the FP64 path) and the caller reports failure.
#pragma once
#include "tcgen05.cuh"
#include "linalg.cuh"

namespace catn {

// Layout of the staging area (offsets in bytes from T.tcs, 1024-aligned).
constexpr int kTcOffAhi = 0;                 // 128 x 64 TF32 (Gram) / two 128 x 32 (merge)
constexpr int kTcOffAlo = 32 * 1024;
constexpr int kTcOffCtl = 64 * 1024;         // mbarrier, TMEM slot, counters
constexpr int kTcRegionBytes = 64 * 1024 + 64;
constexpr int kTcTmemCols = 128;   // Grams use columns 0-31, merges 0-127
constexpr long long kTcWaitPolls = 1LL << 22;

#if defined(__CUDACC__)
struct TcCtl {
  uint64_t bar;             // mbarrier
  unsigned tmem_slot;       // written by tcgen05.alloc
  unsigned commits;         // MMA groups committed to bar and waited for
  int broken;               // a wait ran out: no further MMAs
  int pending;              // a committed group not yet waited for
};

__device__ __forceinline__ TcCtl* tc_ctl(const Team& T) { return (TcCtl*)(T.tcs + kTcOffCtl); }

// Kernel prologue / epilogue: TMEM columns and the mbarrier.  Every thread
// of the CTA calls both.
__device__ inline void tc_setup(Team& T, unsigned char* region) {
#if defined(CATN_NO_TCGEN05)
  (void)region;
  T.tcs = nullptr;
  T.tmem = 0;
  return;
#endif
  T.tcs = region;
  TcCtl* c = tc_ctl(T);
  if (threadIdx.x == 0) {
    c->commits = 0;
    c->broken = 0;
    c->pending = 0;
    tc::mbar_init(&c->bar, 1);
  }
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&c->tmem_slot, kTcTmemCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  T.tmem = c->tmem_slot;
}
__device__ inline void tc_teardown(const Team& T) {
  if (!T.tcs) return;
  TcCtl* c = tc_ctl(T);
  __syncthreads();
  if (threadIdx.x == 0 && c->pending) {
    // a group still in flight after a failed wait: let it land (bounded)
    tc::mbar_wait(&c->bar, c->commits & 1u, kTcWaitPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(T.tmem, kTcTmemCols);
}

// Wait for the group committed last; false (and the area marked broken) when
// the wait ran out.  Every thread calls it with the same `commits`.
__device__ __forceinline__ bool tc_wait(const Team& T, unsigned* commits) {
  TcCtl* c = tc_ctl(T);
  const bool ok = tc::mbar_wait(&c->bar, *commits & 1u, kTcWaitPolls);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      c->broken = 1;
      c->pending = 1;   // the group still in flight completes phase `commits`
      c->commits = *commits;
    }
    __syncthreads();
    return false;
  }
  *commits += 1;
  tc::fence_after_sync();
  return true;
}
__device__ __forceinline__ void tc_issue_commit(const Team& T) {
  tc::mma_commit(&tc_ctl(T)->bar);
}
// Record the count of completed groups (thread 0) at the end of a routine.
__device__ __forceinline__ void tc_finish(const Team& T, unsigned commits, int pending) {
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_ctl(T)->commits = commits;
    tc_ctl(T)->pending = pending;
  }
  __syncthreads();
}

// (the TMEM base address may be 0, so the staging area marks the set-up)
__device__ __forceinline__ bool tc_ready(const Team& T) { return T.tcs && !tc_ctl(T)->broken; }

// G (32 x 32, row-major FP64) = X_P^T X_P over rows [0, m) on the tensor
// cores.  Returns false when a wait ran out.
__device__ inline bool tc_gram(const Team& T, const double* X, long long m, long long ld, const long long* cols,
                               double* G) {
  constexpr int KC = 64;
  float* ahi = (float*)(T.tcs + kTcOffAhi);
  float* alo = (float*)(T.tcs + kTcOffAlo);
  const int tid = threadIdx.x;
  unsigned commits = tc_ctl(T)->commits;
  __syncthreads();
  // rows 32..127 of A stay zero for the whole Gram
  for (int e = tid; e < (128 - 32) * KC; e += 256) {
    const int r = 32 + e / KC, k = e % KC;
    const uint32_t o = tc::kmajor_off(r, k, KC) / 4;
    ahi[o] = 0.0f;
    alo[o] = 0.0f;
  }
  const long long nch = (m + KC - 1) / KC;
  double v[8];
  auto load = [&](long long c) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 256 * j;
      const int i = e >> 6, k = e & 63;
      const long long r = c * KC + k;
      v[j] = (cols[i] >= 0 && r < m) ? ldcg(X + r + cols[i] * ld) : 0.0;
    }
  };
  load(0);
  const uint32_t idesc = tc::idesc_tf32(128, 32);
  const uint32_t sbo = KC / 4 * 128;
  const uint32_t a_hi = tc::smem_u32(ahi), a_lo = tc::smem_u32(alo);
  for (long long c = 0; c < nch; ++c) {
    if (c > 0 && !tc_wait(T, &commits)) return false;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 256 * j;
      const int i = e >> 6, k = e & 63;
      float h, l;
      tc::split_tf32(v[j], &h, &l);
      const uint32_t o = tc::kmajor_off(i, k, KC) / 4;
      ahi[o] = h;
      alo[o] = l;
    }
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < KC / 8; ++s) {
        const uint32_t off = (uint32_t)s * 2 * tc::kLBO;
        const uint64_t dh = tc::smem_desc(a_hi + off, tc::kLBO, sbo);
        const uint64_t dl = tc::smem_desc(a_lo + off, tc::kLBO, sbo);
        tc::mma_tf32(T.tmem, dh, dh, idesc, (c > 0 || s > 0) ? 1u : 0u);
        tc::mma_tf32(T.tmem, dh, dl, idesc, 1u);
        tc::mma_tf32(T.tmem, dl, dh, idesc, 1u);
      }
      tc_issue_commit(T);
    }
    if (c + 1 < nch) load(c + 1);
  }
  if (nch > 0 && !tc_wait(T, &commits)) return false;
  if ((tid >> 5) == 0) {
    float g[32];
    tc::tmem_ld32(T.tmem, g);   // lanes 0-31 = rows 0-31 of D
#pragma unroll
    for (int j = 0; j < 32; ++j) G[(tid & 31) * 32 + j] = nch > 0 ? (double)g[j] : 0.0;
  }
  tc::fence_before_sync();
  tc_finish(T, commits, 0);
  return true;
}

// C (M x N, written through the operand map `out`) = A (M x K, column-major,
// lda) * B (K x N, column-major, ldb) on the tensor cores, for the large
// two-site merges of swap! in split precision.  Tiles of 128 x 128 of C, K
// in chunks of 32; the next chunk's operands are loaded into registers while
// the MMAs of the current one run.  Loads of A and B are plain (the CTA's
// own sites).  Returns false when a wait ran out.
__device__ inline bool tc_gemm_mop(const Team& T, long long M, long long N, long long K, const double* A,
                                   long long lda, const double* B, long long ldb, const MOp& out) {
  constexpr int BM = 128, BN = 128, KC = 32;
  float* ahi = (float*)(T.tcs + kTcOffAhi);
  float* bhi = (float*)(T.tcs + kTcOffAhi + 16 * 1024);
  float* alo = (float*)(T.tcs + kTcOffAlo);
  float* blo = (float*)(T.tcs + kTcOffAlo + 16 * 1024);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned commits = tc_ctl(T)->commits;
  __syncthreads();
  const long long mt = (M + BM - 1) / BM, nt = (N + BN - 1) / BN, kc = (K + KC - 1) / KC;
  const long long iters = mt * nt * kc;
  double va[16], vb[16];
  auto load = [&](long long it) {
    const long long tile = it / kc, c = it - tile * kc;
    const long long m0 = (tile / nt) * BM, n0 = (tile % nt) * BN, k0 = c * KC;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int e = tid + 256 * j;
      const int r = e & 127, k = e >> 7;   // A: consecutive rows
      const long long gr = m0 + r, gk = k0 + k;
      va[j] = (gr < M && gk < K) ? A[gr + gk * lda] : 0.0;
      const int kb = e & 31, n = e >> 5;   // B: consecutive k
      const long long gn = n0 + n, gkb = k0 + kb;
      vb[j] = (gn < N && gkb < K) ? B[gkb + gn * ldb] : 0.0;
    }
  };
  const uint32_t idesc = tc::idesc_tf32(BM, BN);
  const uint32_t sbo = KC / 4 * 128;
  const uint32_t sa_hi = tc::smem_u32(ahi), sa_lo = tc::smem_u32(alo);
  const uint32_t sb_hi = tc::smem_u32(bhi), sb_lo = tc::smem_u32(blo);
  if (iters > 0) load(0);
  for (long long it = 0; it < iters; ++it) {
    const long long tile = it / kc, c = it - tile * kc;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int e = tid + 256 * j;
      float h, l;
      tc::split_tf32(va[j], &h, &l);
      uint32_t o = tc::kmajor_off(e & 127, e >> 7, KC) / 4;
      ahi[o] = h;
      alo[o] = l;
      tc::split_tf32(vb[j], &h, &l);
      o = tc::kmajor_off(e >> 5, e & 31, KC) / 4;
      bhi[o] = h;
      blo[o] = l;
    }
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < KC / 8; ++s) {
        const uint32_t off = (uint32_t)s * 2 * tc::kLBO;
        const uint64_t ah = tc::smem_desc(sa_hi + off, tc::kLBO, sbo), al = tc::smem_desc(sa_lo + off, tc::kLBO, sbo);
        const uint64_t bh = tc::smem_desc(sb_hi + off, tc::kLBO, sbo), bl = tc::smem_desc(sb_lo + off, tc::kLBO, sbo);
        tc::mma_tf32(T.tmem, ah, bh, idesc, (c > 0 || s > 0) ? 1u : 0u);
        tc::mma_tf32(T.tmem, ah, bl, idesc, 1u);
        tc::mma_tf32(T.tmem, al, bh, idesc, 1u);
      }
      tc_issue_commit(T);
    }
    if (it + 1 < iters) load(it + 1);
    if (!tc_wait(T, &commits)) return false;
    if (c == kc - 1) {
      // epilogue: warp w reads lanes 32 (w % 4) (rows), columns 64 (w / 4) .. + 63
      const long long m0 = (tile / nt) * BM, n0 = (tile % nt) * BN;
      const int q = warp & 3, half = warp >> 2;
      const long long row = m0 + q * 32 + lane;
      for (int c0 = half * 64; c0 < half * 64 + 64; c0 += 32) {
        float y[32];
        tc::tmem_ld32(T.tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, y);
        if (row < M) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const long long col = n0 + c0 + j;
            if (col < N) out.ref(row, col) = (double)y[j];
          }
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }
  }
  tc_finish(T, commits, 0);
  return true;
}
#endif  // __CUDACC__

}  // namespace catn
