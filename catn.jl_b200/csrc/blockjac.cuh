// Block one-sided Jacobi for the large SVDs (the block route of svd_route).
//
// The columns of X (m x n) are split into blocks of kBlockW; a round of the
// round-robin tournament over the blocks pairs every block with another, and
// one item rotates one pair of blocks (2 kBlockW columns):
//   1. G = X_P^T X_P, the pair's Gram matrix (2b x 2b), accumulated in FP64;
//   2. if some off-diagonal entry of G is above tolerance, a cyclic Jacobi
//      sweep on G (FP64, parallel order, starting from the identity) gives
//      the rotation Q, so that Q stays close to the identity and the
//      columns keep their places from round to round;
//   3. X_P <- X_P Q and V_P <- V_P Q.
// A sweep is nb - 1 rounds (nb blocks, padded to even); the SVD has
// converged when a whole sweep rotated nothing.  The arithmetic per item is
// two small GEMMs and a 32 x 32 eigen core instead of 2b(2b-1)/2 separate
// column pairs, and a sweep has nb - 1 rounds instead of n - 1, which is
// what makes the route fast on the full-rank 4096 x 4096 swaps of large
// networks: the scalar route's rounds are latency-bound.
//
// The pair Gram is exact to FP64 rounding, so singular values come out with
// absolute (not relative) accuracy ~ eps * sigma_1, the accuracy LAPACK's
// gesdd has; tiny singular values far below the largest are therefore not
// resolved to full relative precision (the scalar route resolves them).
//
// Items are claimed by whole CTAs through the shared job (JOB_BLOCK): the
// owner publishes a round, its own CTA and helper CTAs claim pairs until
// none is left, and the owner waits (bounded) for the claimed ones.
#pragma once
#include "linalg.cuh"
#include "blockjac_tc.cuh"
#include "blockqr.cuh"

namespace catn {

constexpr int kBlockW = 16;             // columns per block
constexpr int kBlockK = 2 * kBlockW;    // columns per item
// Smallest column count of the Jacobi factor that takes the block route by
// default (svd_route 2, or 0 with precision 1).  Below it the scalar rounds
// are short and the block items' fixed costs (Gram, eigen core) dominate.
constexpr int kBlockMinN = 192;
// Inner Jacobi sweeps on a pair's Gram per item.
constexpr int kBlockInnerSweeps = 2;
// Workspace (doubles) an item needs beside the GEMM stage: G, Q, four
// partial Grams, rotation parameters, column list.
constexpr int kBlockWsDoubles = 6 * kBlockK * kBlockK + 4 * kBlockK + 64;

// Column index of item column c (0 <= c < 2b) of pair (p, q), or -1 when
// the pair's block is padding or the column lies beyond n.
CATN_HD long long block_col(long long p, long long q, int c, long long n) {
  const long long blk = c < kBlockW ? p : q;
  const long long col = blk * kBlockW + (c % kBlockW);
  return col < n ? col : -1;
}

// G (k x k, row-major, k = kBlockK) = X_P^T X_P over rows [0, m).  Loads go
// through L2 (other CTAs rotated these columns in earlier rounds).
CATN_HDI inline void block_gram(const Team& T, const double* X, long long m, long long ld, const long long* cols,
                                double* G, double* part) {
#if CATN_DEVICE_PASS
  // rows staged 64 at a time as S[c][r] (ld 65); four row groups of 64
  // threads, each thread a 4 x 4 tile of G, partial Grams summed at the end
  double* S = (double*)T.stage;
  const int tid = T.rank();
  const int grp = tid >> 6, tt = tid & 63;
  const int i0 = (tt & 7) * 4, j0 = (tt >> 3) * 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  // the next chunk's 8 values per thread are loaded into registers while
  // the current one is multiplied
  double v[8];
  auto load = [&](long long r0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 256 * j;
      const int c = e >> 6, r = e & 63;
      const long long col = cols[c];
      v[j] = (col >= 0 && r0 + r < m) ? ldcg(X + (r0 + r) + col * ld) : 0.0;
    }
  };
  load(0);
  for (long long r0 = 0; r0 < m; r0 += 64) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = tid + 256 * j;
      S[(e >> 6) * 65 + (e & 63)] = v[j];
    }
    __syncthreads();
    if (r0 + 64 < m) load(r0 + 64);
    for (int r = grp; r < 64; r += 4) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = S[(i0 + q) * 65 + r];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = S[(j0 + q) * 65 + r];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) part[grp * kBlockK * kBlockK + (i0 + x) * kBlockK + (j0 + y)] = acc[x][y];
  __syncthreads();
  for (int e = tid; e < kBlockK * kBlockK; e += 256) {
    const int kk = kBlockK * kBlockK;
    G[e] = (part[e] + part[kk + e]) + (part[2 * kk + e] + part[3 * kk + e]);
  }
  __syncthreads();
#else
  (void)part;
  for (int i = 0; i < kBlockK; ++i)
    for (int j = 0; j < kBlockK; ++j) {
      double s = 0.0;
      if (cols[i] >= 0 && cols[j] >= 0)
        for (long long r = 0; r < m; ++r) s = fma(X[r + cols[i] * ld], X[r + cols[j] * ld], s);
      G[i * kBlockK + j] = s;
    }
#endif
}

// Y_P <- Y_P Q on rows [0, m) (Q row-major k x k in shared memory); one row
// per thread at a time, the row's 2b values held in registers.
CATN_HDI inline void block_rotate(const Team& T, double* Y, long long m, long long ld, const long long* cols,
                                  const double* Q) {
#if CATN_DEVICE_PASS
  for (long long r = T.rank(); r < m; r += T.size()) {
    double x[kBlockK], y[kBlockK];
#pragma unroll
    for (int c = 0; c < kBlockK; ++c) x[c] = cols[c] >= 0 ? ldcg(Y + r + cols[c] * ld) : 0.0;
#pragma unroll
    for (int j = 0; j < kBlockK; ++j) y[j] = 0.0;
#pragma unroll
    for (int i = 0; i < kBlockK; ++i) {
      const double2* qi = (const double2*)(Q + i * kBlockK);
#pragma unroll
      for (int j = 0; j < kBlockK / 2; ++j) {
        const double2 qv = qi[j];
        y[2 * j] = fma(x[i], qv.x, y[2 * j]);
        y[2 * j + 1] = fma(x[i], qv.y, y[2 * j + 1]);
      }
    }
#pragma unroll
    for (int c = 0; c < kBlockK; ++c)
      if (cols[c] >= 0) stcg(Y + r + cols[c] * ld, y[c]);
  }
  T.sync();
#else
  double x[kBlockK], y[kBlockK];
  for (long long r = 0; r < m; ++r) {
    for (int c = 0; c < kBlockK; ++c) x[c] = cols[c] >= 0 ? Y[r + cols[c] * ld] : 0.0;
    for (int j = 0; j < kBlockK; ++j) {
      double s = 0.0;
      for (int i = 0; i < kBlockK; ++i) s = fma(x[i], Q[i * kBlockK + j], s);
      y[j] = s;
    }
    for (int c = 0; c < kBlockK; ++c)
      if (cols[c] >= 0) Y[r + cols[c] * ld] = y[c];
  }
#endif
}

// Whether the pair needs rotating: some off-diagonal |G_ij| above
// max(tol sqrt(G_ii G_jj), floor sqrt(max(G_ii, G_jj))).  Every thread
// returns the same answer.
CATN_HDI inline bool block_needs_rotation(const Team& T, const double* G, double tol, double floor_abs) {
  int big = 0;
  for (int e = T.rank(); e < kBlockK * kBlockK; e += T.size()) {
    const int i = e / kBlockK, j = e - i * kBlockK;
    if (i >= j) continue;
    const double gi = G[i * kBlockK + i], gj = G[j * kBlockK + j];
    if (gi < 1e-250 || gj < 1e-250) continue;
    const double g = fabs(G[e]);
    const double thr = fmax(tol * sqrt(gi * gj), floor_abs * sqrt(fmax(gi, gj)));
    if (g > thr) big = 1;
  }
  return T.any(big) != 0;
}

// Cyclic Jacobi sweeps on the symmetric G (k x k, row-major) in parallel
// order (kBlockK / 2 disjoint rotations per step); Q accumulates them from
// the identity.  The rotation of (p, q), p < q, is jacobi_rotation's, as in
// the scalar route: columns p', q' = c p - s q, s p + c q.
// On the GPU one warp does it with G and Q in registers, lane l holding row
// l of each.  The round-robin order is kept with the players moving instead
// of the pairing: every step rotates the fixed neighbour pairs (2k, 2k+1),
// then moves each row and column one place round the circle (position 0
// fixed, the others shifted), so that after 31 steps every pair has met once
// and the layout is back where it started.  Every register index is then a
// compile-time constant and the step's code is the same for every step (the
// xor-paired form needed 31 unrolled copies, which overflowed the instruction
// cache), and rows cross lanes by shuffles only.
CATN_HD constexpr int rr_circ_of_phys(int x) { return (x & 1) ? 31 - (x >> 1) : (x >> 1); }
CATN_HD constexpr int rr_phys_of_circ(int c) { return c < 16 ? 2 * c : 2 * (31 - c) + 1; }
// physical place of the element at x after one step, and the place it came from
CATN_HD constexpr int rr_next(int x) {
  return rr_phys_of_circ(rr_circ_of_phys(x) == 0 ? 0 : (rr_circ_of_phys(x) == 31 ? 1 : rr_circ_of_phys(x) + 1));
}
CATN_HD constexpr int rr_prev(int x) {
  return rr_phys_of_circ(rr_circ_of_phys(x) == 0 ? 0 : (rr_circ_of_phys(x) == 1 ? 31 : rr_circ_of_phys(x) - 1));
}
#if CATN_DEVICE_PASS
__device__ __forceinline__ double lane_pick(const double* a, int idx) {
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < 32; ++k)
    if (k == idx) v = a[k];
  return v;
}
__device__ __forceinline__ void inner_circle_step(double* g, double* qv, int l, double tol) {
  const unsigned FULL = 0xffffffffu;
  const bool lo = (l & 1) == 0;
  const double d = lane_pick(g, l);
  const double dp = __shfl_xor_sync(FULL, d, 1);
  const double apq = lane_pick(g, l ^ 1);
  double c = 1.0, sn = 0.0;
  if (!jacobi_rotation(lo ? d : dp, lo ? dp : d, apq, tol, &c, &sn)) {
    c = 1.0;
    sn = 0.0;
  }
  // both lanes of a pair use the even lane's rotation
  const double cx = __shfl_xor_sync(FULL, c, 1), sx = __shfl_xor_sync(FULL, sn, 1);
  if (!lo) {
    c = cx;
    sn = sx;
  }
  // columns (2k, 2k+1) of this lane's rows of G and Q
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const double ck = __shfl_sync(FULL, c, 2 * k), sk = __shfl_sync(FULL, sn, 2 * k);
    const double gp = g[2 * k], gq = g[2 * k + 1];
    g[2 * k] = ck * gp - sk * gq;
    g[2 * k + 1] = sk * gp + ck * gq;
    const double qp = qv[2 * k], qq = qv[2 * k + 1];
    qv[2 * k] = ck * qp - sk * qq;
    qv[2 * k + 1] = sk * qp + ck * qq;
  }
  // rows 2k and 2k+1 of G
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const double o = __shfl_xor_sync(FULL, g[k], 1);
    g[k] = lo ? (c * g[k] - sn * o) : (sn * o + c * g[k]);
  }
  // move every column of G and Q, and every row of G, one place on
  double tg[32], tq[32];
#pragma unroll
  for (int x = 0; x < 32; ++x) {
    tg[rr_next(x)] = g[x];
    tq[rr_next(x)] = qv[x];
  }
  const int src = rr_prev(l);
#pragma unroll
  for (int x = 0; x < 32; ++x) {
    g[x] = __shfl_sync(FULL, tg[x], src);
    qv[x] = tq[x];
  }
}
#endif

CATN_HDI inline void block_inner(const Team& T, double* G, double* Q, double* rot, double tol, int sweeps,
                                 double* pad) {
  constexpr int K = kBlockK, H = kBlockK / 2;
  static_assert(K == 32, "the one-warp core holds one row per lane");
#if CATN_DEVICE_PASS
  (void)pad; (void)rot; (void)H;
  if (T.warp() == 0) {
    const int l = T.lane();
    double g[32], qv[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      g[k] = G[l * K + k];
      qv[k] = (k == l) ? 1.0 : 0.0;
    }
    for (int sw = 0; sw < sweeps; ++sw) {
#pragma unroll 1
      for (int r = 0; r < K - 1; ++r) inner_circle_step(g, qv, l, tol);
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      G[l * K + k] = g[k];
      Q[l * K + k] = qv[k];
    }
  }
  T.sync();
#else
  // the host build: the same pairs in the same order, tracked through the
  // original indices instead of moving rows and columns
  (void)pad; (void)T;
  int at[K], nat[K];
  for (int x = 0; x < K; ++x) at[x] = x;
  for (int e = 0; e < K * K; ++e) Q[e] = (e / K == e % K) ? 1.0 : 0.0;
  for (int sw = 0; sw < sweeps; ++sw) {
    for (int r = 0; r < K - 1; ++r) {
      for (int k = 0; k < H; ++k) {   // parameters from the state at the step's start
        const int p = at[2 * k], q = at[2 * k + 1];
        double c = 1.0, sn = 0.0;
        if (!jacobi_rotation(G[p * K + p], G[q * K + q], G[p * K + q], tol, &c, &sn)) {
          c = 1.0;
          sn = 0.0;
        }
        rot[3 * k] = c;
        rot[3 * k + 1] = sn;
      }
      for (int k = 0; k < H; ++k) {   // columns of G and Q
        const int p = at[2 * k], q = at[2 * k + 1];
        const double c = rot[3 * k], sn = rot[3 * k + 1];
        for (int i = 0; i < K; ++i) {
          const double gp = G[i * K + p], gq = G[i * K + q];
          G[i * K + p] = c * gp - sn * gq;
          G[i * K + q] = sn * gp + c * gq;
          const double qp = Q[i * K + p], qq = Q[i * K + q];
          Q[i * K + p] = c * qp - sn * qq;
          Q[i * K + q] = sn * qp + c * qq;
        }
      }
      for (int k = 0; k < H; ++k) {   // rows of G
        const int p = at[2 * k], q = at[2 * k + 1];
        const double c = rot[3 * k], sn = rot[3 * k + 1];
        for (int j = 0; j < K; ++j) {
          const double gp = G[p * K + j], gq = G[q * K + j];
          G[p * K + j] = c * gp - sn * gq;
          G[q * K + j] = sn * gp + c * gq;
        }
      }
      for (int x = 0; x < K; ++x) nat[rr_next(x)] = at[x];
      for (int x = 0; x < K; ++x) at[x] = nat[x];
    }
  }
#endif
}

// One item: block pair (p, q) of the round.  ws holds kBlockWsDoubles.
// With `tc` and the CTA's tensor-core area ready, the pair's Gram is a 3xTF32
// tensor-core product (blockjac_tc.cuh), else FP64.
// Returns 1 when the pair was rotated, 0 when it was left alone, -1 when a
// wait for the tensor core ran out (same in every thread).
CATN_HDI inline int block_item(const Team& T, double* X, double* V, long long m, long long n, long long ld,
                               long long p, long long q, double tol, double floor_abs, double* ws, bool tc) {
  double* G = ws;
  double* Q = G + kBlockK * kBlockK;
  double* part = Q + kBlockK * kBlockK;
  double* rot = part + 4 * kBlockK * kBlockK;
  long long* cols = (long long*)(rot + 3 * kBlockK);
  for (int c = T.rank(); c < kBlockK; c += T.size()) cols[c] = block_col(p, q, c, n);
  T.sync();
#if CATN_DEVICE_PASS
  const bool on_tc = tc && tc_ready(T);
  if (on_tc) {
    if (!tc_gram(T, X, m, ld, cols, G)) return -1;
  } else {
    block_gram(T, X, m, ld, cols, G, part);
  }
#else
  (void)tc;
  const bool on_tc = false;
  block_gram(T, X, m, ld, cols, G, part);
#endif
  if (!block_needs_rotation(T, G, tol, floor_abs)) return 0;
  block_inner(T, G, Q, rot, tol, kBlockInnerSweeps, part);
  // the rotation itself stays FP64: each column is rotated thousands of
  // times, and 3xTF32 products would leave ~2^-21 of its norm behind each time
  block_rotate(T, X, m, ld, cols, Q);
  block_rotate(T, V, n, n, cols, Q);
  return 1;
}

// The team's share of the current round of a JOB_BLOCK or JOB_PANEL job:
// the leader claims items one at a time for the whole team, which works
// them (a block pair, or a tile of trailing columns) and reports each done.
CATN_HDI inline void block_work(const Team& T, JacobiJob* J, double* ws) {
  for (;;) {
    long long item = -1;
    if (T.leader()) {
#if CATN_DEVICE_PASS
      const unsigned long long old = atomicAdd(&J->word, 1ULL);
#else
      const unsigned long long old = J->word;
      J->word = old + 1;
#endif
      const long long it = (long long)(old & 0xfffffULL);
      const long long count = (long long)((old >> 20) & 0xfffffULL);
      item = it < count ? it : -1;
      fence_gpu();
    }
    item = T.bcast(item);
    if (item < 0) return;
    double* X = (double*)ldcg_u((const unsigned long long*)&J->B);
    double* V = (double*)ldcg_u((const unsigned long long*)&J->V);
    const long long m = ldcg_i(&J->m), n = ldcg_i(&J->n), ld = ldcg_i(&J->ldb), np = ldcg_i(&J->np);
    int rot = 0;
    if (ldcg_i(&J->kind) == JOB_PANEL) {
      // 32 trailing columns of a blocked QR panel update
      long long* cols = (long long*)(ws + kPanelWsDoubles);
      const long long c0 = ldcg_i(&J->c0) + item * kPanelW;
      for (int c = T.rank(); c < kPanelW; c += T.size()) cols[c] = (c0 + c < n) ? c0 + c : -1;
      T.sync();
      panel_item(T, X, m, ld, V, (const double*)ldcg_u((const unsigned long long*)&J->W2), ldcg_i(&J->k), cols,
                 (double*)ldcg_u((const unsigned long long*)&J->nrm), ws);
    } else {
      const long long r = ldcg_i(&J->round);
      long long p, q;
      rr_pair(np, r, item, &p, &q);
      rot = block_item(T, X, V, m, n, ld, p, q, ldcg(&J->tol), ldcg(&J->tk), ws, ldcg_i(&J->tc) != 0);
    }
    fence_gpu();
    T.sync();
    if (T.leader()) {
      // bit 0: rotated; bit 1: a tensor-core wait ran out
      const int flag = rot > 0 ? 1 : (rot < 0 ? 2 : 0);
#if CATN_DEVICE_PASS
      if (flag) atomicOr(&J->rotated, flag);
      atomicAdd(&J->done, 1);
#else
      if (flag) J->rotated |= flag;
      J->done += 1;
#endif
    }
    T.sync();
  }
}

// Owner side of one round of a JOB_BLOCK job: publish `count` pairs, take
// the team's share, wait (bounded) for the rest.  Returns 1 when the wait
// ran out.
CATN_HDI inline int job_round_cta(const Team& T, JacobiJob* J, unsigned long long seq, long long count,
                                  double* ws) {
  if (T.leader()) {
    J->done = 0;
    fence_gpu();
    job_set_word(J, job_word(seq, count) + (count > 0 ? CATN_JOB_PHANTOM_CLAIMS : 0));
  }
  T.sync();
  block_work(T, J, ws);
  return job_wait_done(T, J, count);
}

// Householder QR of A (m x n, m >= n, ld lda) after sorting its columns by
// norm, largest first: A P = Q R with piv[k] the original index of column
// k, R in the upper triangle and the reflectors below it (LAPACK geqrf
// layout, tau), as qrcp_inplace leaves them.  Blocked: each panel of 32
// reflectors is factored by the team, and the trailing columns are updated
// in compact WY form, 32 columns per item, shared through J when J is set.
// Sorting instead of pivoting at every step keeps the columns graded, which
// is what the one-sided Jacobi on R^T needs (about one more sweep than full
// pivoting), with one shared round per panel instead of one per column.
// With stop_tol > 0 the factorisation ends at the first panel boundary k
// whose trailing block has Frobenius norm <= stop_tol and returns k (every
// singular value of the dropped block is below stop_tol); otherwise n.
// -2: a shared wait ran out.  work: m n + 32 m + 2048 doubles.
CATN_HDI inline long long qr_sorted_blocked(const Team& T, JacobiJob* J, double* A, long long m, long long n,
                                            long long lda, double* tau, int* piv, double* nrm, double stop_tol,
                                            double* work, double* ws) {
  constexpr int B = kPanelW;
  double* tmp = work;             // m x n
  double* Vp = tmp + m * n;       // up to m x 32
  double* G = Vp + m * B;         // 32 x 32
  double* Nm = G + B * B;         // 32 x 32
  // column norms and the descending order (stable: ties by index)
  for (long long j = T.warp(); j < n; j += T.nwarps()) {
    const double* aj = A + j * lda;
    double s2 = 0.0;
    for (long long i = T.lane(); i < m; i += T.wsize()) s2 = fma(aj[i], aj[i], s2);
    s2 = T.wsum(s2);
    if (T.lane() == 0) nrm[j] = s2;
  }
  T.sync();
  for (long long j = T.rank(); j < n; j += T.size()) {
    const double v = nrm[j];
    long long rk = 0;
    for (long long i = 0; i < n; ++i) rk += (nrm[i] > v || (nrm[i] == v && i < j)) ? 1 : 0;
    piv[rk] = (int)j;
  }
  T.sync();
  for (long long e = T.rank(); e < m * n; e += T.size()) {
    long long i, k;
    divmod(e, m, &i, &k);
    tmp[e] = A[i + (long long)piv[k] * lda];
  }
  T.sync();
  for (long long e = T.rank(); e < m * n; e += T.size()) {
    long long i, k;
    divmod(e, m, &i, &k);
    A[i + k * lda] = tmp[e];
  }
  for (long long k = T.rank(); k < n; k += T.size()) nrm[k] = 0.0;
  fence_gpu();
  T.sync();
  unsigned long long seq = 0;
  if (J) {
    seq = job_open(T, J);
    if (T.leader()) {
      J->kind = JOB_PANEL;
      fence_gpu();
      J->open = 1;
      fence_gpu();
    }
    T.sync();
  }
  long long rank = n;
  int timed_out = 0;
  for (long long k0 = 0; k0 < n && !timed_out; k0 += B) {
    const long long kb = (n - k0 < B) ? n - k0 : B, mp = m - k0;
    if (stop_tol > 0.0 && k0 > 0) {
      double rem = 0.0;
      for (long long j = k0 + T.rank(); j < n; j += T.size()) rem += ldcg(nrm + j);
      rem = T.sum(rem);
      if (rem <= stop_tol * stop_tol) {
        rank = k0;
        break;
      }
    }
    double* P = A + k0 + k0 * lda;
    if (J) {   // the panel's columns as the helpers left them, through this SM
      for (long long e = T.rank(); e < mp * kb; e += T.size()) {
        long long i, j;
        divmod(e, mp, &i, &j);
        P[i + j * lda] = ldcg(P + i + j * lda);
      }
      T.sync();
    }
    qr_inplace(T, P, mp, kb, lda, tau + k0);
    if (k0 + kb >= n) break;
    // compact WY: V explicit (unit diagonal), G = V^T V, Nm = -T
    for (long long e = T.rank(); e < mp * kb; e += T.size()) {
      long long i, j;
      divmod(e, mp, &i, &j);
      Vp[e] = (i > j) ? P[i + j * lda] : (i == j ? 1.0 : 0.0);
    }
    for (long long e = T.rank(); e < kb * kb; e += T.size()) Nm[e] = 0.0;
    T.sync();
    gemm(T, kb, kb, mp, transposed(Vp, mp), colmajor(Vp, mp), colmajor(G, kb));
    for (long long j = 0; j < kb; ++j) {
      const double tj = tau[k0 + j];
      for (long long i = T.rank(); i <= j; i += T.size()) {
        double s2 = 0.0;
        for (long long l = i; l < j; ++l) s2 = fma(Nm[i + l * kb], G[l + j * kb], s2);
        Nm[i + j * kb] = -tj * (i == j ? 1.0 : s2);
      }
      T.sync();
    }
    fence_gpu();
    T.sync();
    const long long c_first = k0 + kb;
    const long long items = (n - c_first + B - 1) / B;
    if (J) {
      if (T.leader()) {
        J->B = A + k0; J->V = Vp; J->W2 = Nm; J->nrm = nrm;
        J->m = (int)mp; J->n = (int)n; J->ldb = (int)lda; J->k = (int)kb; J->c0 = (int)c_first;
        fence_gpu();
      }
      timed_out = job_round_cta(T, J, seq, items, ws);
      ++seq;
    } else {
      long long* cols = (long long*)(ws + kPanelWsDoubles);
      for (long long it = 0; it < items; ++it) {
        for (int c = T.rank(); c < B; c += T.size()) cols[c] = (c_first + it * B + c < n) ? c_first + it * B + c : -1;
        T.sync();
        panel_item(T, A + k0, mp, lda, Vp, Nm, (int)kb, cols, nrm, ws);
      }
    }
  }
  if (J) {
    job_close(T, J, seq);
    // every column as the helpers left it, through this SM
    for (long long e = T.rank(); e < m * n; e += T.size()) {
      long long i, k;
      divmod(e, m, &i, &k);
      A[i + k * lda] = ldcg(A + i + k * lda);
    }
  }
  T.sync();
  return timed_out ? -2 : rank;
}

// Block one-sided Jacobi on X (m x n, ld) with V (n x n) accumulated, the
// rounds shared through J when J is set (else the team does every item).
// Same contract as jacobi_sweeps: returns the sweep count, -1 without
// convergence within max_sweeps, -2 when a wait for claimed items ran out.
// floor_rel > 0 adds an absolute floor floor_rel * max column norm to the
// rotation test (reduced-precision products cannot orthogonalise columns
// below their own rounding level).
CATN_HDI inline int jacobi_block(const Team& T, JacobiJob* J, double* X, long long m, long long n, long long ld,
                                 double* V, int max_sweeps, double* ws, double floor_rel, bool tc) {
  for (long long e = T.rank(); e < n * n; e += T.size()) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  T.sync();
  if (n < 2) return 0;
  double mx = 0.0;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) mx = fmax(mx, fabs(X[i + c * ld]));
  mx = T.maxv(mx);
  const double sc = mx > 0.0 ? 1.0 / mx : 1.0;
  double cmax = 0.0;
  for (long long c = T.warp(); c < n; c += T.nwarps()) {
    double s2 = 0.0;
    for (long long i = T.lane(); i < m; i += T.wsize()) {
      const double x = X[i + c * ld] * sc;
      X[i + c * ld] = x;
      s2 = fma(x, x, s2);
    }
    cmax = fmax(cmax, T.wsum(s2));
  }
  cmax = T.maxv(cmax);
  fence_gpu();
  T.sync();
  const long long nb0 = (n + kBlockW - 1) / kBlockW;
  const long long nb = (nb0 % 2) ? nb0 + 1 : nb0;
  const long long npair = nb / 2;
  const double tol = 2.220446049250313e-16 * (double)(m > 16 ? m : 16);
  const double floor_abs = floor_rel > 0.0 ? floor_rel * sqrt(cmax) : 0.0;
  // With tc the sweeps run in two phases: first the pair Grams on the tensor
  // cores (3xTF32), the rotation test at their rounding level (relative
  // 4e-6, floor 4e-7 of the largest column); then FP64 Grams with the FP64
  // test until a sweep rotates nothing, which certifies the result at the
  // FP64 level.  The rotations are FP64 in both phases.
  int phase = tc ? 0 : 1;
  auto ptol = [&](int ph) { return ph == 0 ? 4e-6 : tol; };
  auto pfloor = [&](int ph) { return ph == 0 ? 4e-7 * sqrt(cmax) : floor_abs; };
  int result = -1, timed_out = 0;
  unsigned long long seq = 0;
  if (J) {
    seq = job_open(T, J);
    if (T.leader()) {
      J->kind = JOB_BLOCK;
      J->B = X; J->V = V; J->nrm = nullptr;
      J->m = (int)m; J->n = (int)n; J->ldb = (int)ld; J->np = (int)nb;
      J->tol = ptol(phase); J->tk = pfloor(phase); J->tc = phase == 0 ? 1 : 0;
      J->rotated = 0; J->round = 0;
      fence_gpu();
      J->open = 1;
      fence_gpu();
    }
    T.sync();
  }
  for (int sweep = 0; sweep < max_sweeps && !timed_out; ++sweep) {
    int rot = 0;
    if (J) {
      if (T.leader()) J->rotated = 0;
      for (long long r = 0; r < nb - 1 && !timed_out; ++r) {
        if (T.leader()) J->round = (int)r;
        timed_out = job_round_cta(T, J, seq, npair, ws);
        ++seq;
      }
      fence_gpu();
      T.sync();
      rot = ldcg_i(&J->rotated);
      T.sync();
      if (rot & 2) timed_out = 1;
    } else {
      for (long long r = 0; r < nb - 1 && !timed_out; ++r)
        for (long long pi = 0; pi < npair && !timed_out; ++pi) {
          long long p, q;
          rr_pair(nb, r, pi, &p, &q);
          const int it = block_item(T, X, V, m, n, ld, p, q, ptol(phase), pfloor(phase), ws, phase == 0);
          if (it > 0) rot = 1;
          if (it < 0) timed_out = 1;
        }
    }
    if (!rot && phase == 0) {
      phase = 1;
      if (J && T.leader()) {
        J->tol = ptol(1); J->tk = pfloor(1); J->tc = 0;
        fence_gpu();
      }
      T.sync();
      continue;
    }
    if (!rot) {
      result = sweep + 1;
      break;
    }
  }
  if (J) job_close(T, J, seq);
  const double inv = 1.0 / sc;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) X[i + c * ld] = ldcg(X + i + c * ld) * inv;
  for (long long e = T.rank(); e < n * n; e += T.size()) V[e] = ldcg(V + e);
  T.sync();
  return timed_out ? -2 : result;
}

#if defined(__CUDACC__)
// Helper CTAs: claim work of other CTAs' shared jobs until every instance of
// the launch is finished.  The leader scans the job board (32 slots per
// warp-wide load) and the whole CTA takes the job it picked: block pairs are
// claimed by the CTA (block_work), column pairs and Householder chunks by
// each warp (job_work).  The CTA stays with the job for its next rounds.
__device__ inline void help_jobs(const Team& T, JacobiJob* board, int nslots, const int* finished, int ninst,
                                 double* ws) {
  const unsigned FULL = 0xffffffffu;
  const int lane = T.lane();
  long long idle = 0;
  while (idle < (1LL << 22)) {
    int pick = -1;
    if (T.warp() == 0) {
      if (ldcg_i(finished) >= ninst) {
        pick = -2;
      } else {
        const int nblk = (nslots + 31) / 32;
        for (int b = 0; b < nblk && pick < 0; ++b) {
          const int base = ((b + (int)blockIdx.x) % nblk) * 32;
          const int s = base + lane;
          bool ok = false;
          if (s < nslots) {
            const JacobiJob* J = board + s;
            const int open = ldcg_i(&J->open);
            const unsigned long long word = ldcg_u(&J->word);
            ok = open && (word & 0xfffffULL) < ((word >> 20) & 0xfffffULL);
          }
          const unsigned mask = __ballot_sync(FULL, ok);
          if (mask) {
            const int r = (int)blockIdx.x & 31;
            const unsigned hi = mask & (~0u << r);
            pick = base + __ffs(hi ? hi : mask) - 1;
          }
        }
      }
    }
    pick = (int)T.bcast(pick);
    if (pick == -2) return;
    if (pick < 0) {
      ++idle;
      __nanosleep(256);
      continue;
    }
    idle = 0;
    JacobiJob* J = board + pick;
    for (int t = 0; t < kJobStickPolls; ++t) {
      int state = 0;   // 0 nothing yet, 1 items, 2 closed
      if (T.leader()) {
        const int open = ldcg_i(&J->open);
        const unsigned long long word = ldcg_u(&J->word);
        state = !open ? 2 : ((word & 0xfffffULL) < ((word >> 20) & 0xfffffULL) ? 1 : 0);
      }
      state = (int)T.bcast(state);
      if (state == 2) break;
      if (state == 0) {
        __nanosleep(32);
        continue;
      }
      const int kind = ldcg_i(&J->kind);
      if (kind == JOB_BLOCK || kind == JOB_PANEL) {
        block_work(T, J, ws);
      } else {
        job_work(T, J);
        T.sync();
      }
      t = -1;
    }
  }
}
#endif

}  // namespace catn
