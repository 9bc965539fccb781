// Team-cooperative dense linear algebra for the CATN engine (FP64).
//
//  * gemm      C = A * B over general two-level strided operands, so every
//              einsum of the reference (mps_node.jl:63,85,99,150,367,504,539,
//              613) is one call with its index permutation folded into the
//              operand maps (no separate permute pass).
//  * qr_*      Householder QR (LAPACK geqrf semantics, R in the upper
//              triangle, reflectors below) and application of the thin Q to
//              a padded matrix -- the reference's `qr` + `_thin_q`
//              (linalg_utils.jl:32-37).
//  * svd       thin SVD A = U diag(S) V^T with S sorted descending, by QR
//              pre-reduction (tall inputs) and one-sided Hestenes Jacobi with
//              a round-robin pair order; the reference's `svd` (gesdd) in
//              `tsvd` (linalg_utils.jl:15-28).
#pragma once
#include "team.cuh"

namespace catn {

// Two-level index map: x -> (x % n1) * s1 + (x / n1) * s2.
// Element counts of one operation stay below 2^31, so index splits use
// 32-bit unsigned division (far cheaper than 64-bit on the GPU).
struct IMap {
  int n1;
  long long s1, s2;
  CATN_HD long long at(long long x) const {
    if (n1 == 1) return x * s2;
    const unsigned q = (unsigned)x / (unsigned)n1;
    return ((long long)((unsigned)x - q * (unsigned)n1)) * s1 + (long long)q * s2;
  }
};
// (x % n, x / n) for 0 <= x < 2^31, n > 0.
CATN_HD void divmod(long long x, long long n, long long* r, long long* q) {
  const unsigned qq = (unsigned)x / (unsigned)n;
  *q = qq;
  *r = (long long)((unsigned)x - qq * (unsigned)n);
}
CATN_HD IMap imap(int n1, long long s1, long long s2) { IMap m; m.n1 = n1; m.s1 = s1; m.s2 = s2; return m; }
// Plain column-major index: row r -> r, col c -> c*ld.
CATN_HD IMap rows_plain() { return imap(1, 0, 1); }
CATN_HD IMap cols_plain(long long ld) { return imap(1, 0, ld); }

// Matrix operand X(r, c) = p[R.at(r) + C.at(c)] * rs[r] * cs[c] (scales optional).
struct MOp {
  double* p;
  IMap R, C;
  const double* rs;
  const double* cs;
  CATN_HD double ld(long long r, long long c) const {
    double v = p[R.at(r) + C.at(c)];
    if (rs) v *= rs[r];
    if (cs) v *= cs[c];
    return v;
  }
  CATN_HD double& ref(long long r, long long c) const { return p[R.at(r) + C.at(c)]; }
};
CATN_HD MOp mop(double* p, IMap R, IMap C, const double* rs = nullptr, const double* cs = nullptr) {
  MOp o; o.p = p; o.R = R; o.C = C; o.rs = rs; o.cs = cs; return o;
}
// Plain column-major matrix with leading dimension ld.
CATN_HD MOp colmajor(double* p, long long ld) { return mop(p, rows_plain(), cols_plain(ld)); }
// Transposed view of a column-major matrix: X(r, c) = p[c + r*ld].
CATN_HD MOp transposed(double* p, long long ld) { return mop(p, cols_plain(ld), rows_plain()); }

// ---------------------------------------------------------------------------
// GEMM: C(M x N) = A(M x K) * B(K x N), overwrite (or C += A * B with accum).
// ---------------------------------------------------------------------------
constexpr int GEMM_BM = 64, GEMM_BN = 64, GEMM_BK = 16;
// Shared tiles are [BK][BM + 1] and [BK][BN + 1]: the padding keeps the
// k-fastest tile loads (operands whose k index is the unit-stride one) free
// of bank conflicts.
constexpr int GEMM_LDA = GEMM_BM + 1, GEMM_LDB = GEMM_BN + 1;
constexpr int GEMM_STAGE_BYTES = (GEMM_LDA + GEMM_LDB) * GEMM_BK * 8;

// Whether consecutive indices of the map are (mostly) consecutive addresses.
CATN_HD bool unit_stride(const IMap& m) { return m.n1 == 1 ? m.s2 == 1 : m.s1 == 1; }

CATN_HDI inline void gemm(const Team& T, long long M, long long N, long long K, const MOp& A,
                          const MOp& B, const MOp& C, bool accum = false) {
  if (M <= 0 || N <= 0) return;
#if CATN_DEVICE_PASS
  if (T.size() == 256 && M * N <= 1024 && 8 * (M * K + K * N) <= T.stage_bytes) {
    // small products: gather both operands into shared memory at once (one
    // round trip), then one output per thread (k ascending, as below)
    double* sA = (double*)T.stage;   // M x K, ld M
    double* sB = sA + M * K;         // K x N, ld K
    for (long long e = T.rank(); e < M * K; e += 256) {
      long long r, k;
      divmod(e, M, &r, &k);
      sA[e] = A.ld(r, k);
    }
    for (long long e = T.rank(); e < K * N; e += 256) {
      long long k, c;
      divmod(e, K, &k, &c);
      sB[e] = B.ld(k, c);
    }
    __syncthreads();
    for (long long e = T.rank(); e < M * N; e += 256) {
      long long r, c;
      divmod(e, M, &r, &c);
      double s = 0.0;
      for (long long k = 0; k < K; ++k) s = fma(sA[r + k * M], sB[k + c * K], s);
      C.ref(r, c) = accum ? C.ref(r, c) + s : s;
    }
    __syncthreads();
    return;
  }
  if (T.size() == 256 && T.stage_bytes >= GEMM_STAGE_BYTES && M * N >= 256) {
    double* sA = (double*)T.stage;            // [BK][LDA]
    double* sB = sA + GEMM_BK * GEMM_LDA;     // [BK][LDB]
    const int tid = T.rank();
    // tile loads: consecutive threads walk the operand's unit-stride index
    const bool a_kfast = !unit_stride(A.R) && unit_stride(A.C);
    const bool b_kfast = unit_stride(B.R) && !unit_stride(B.C);
    // 16 x 16 threads, each with the 4 x 4 outputs (tr + 16 x, tc + 16 y);
    // with a column-major C the fast thread index walks the rows, so the
    // stores are coalesced
    const bool c_rows = unit_stride(C.R);
    const int tr = c_rows ? (tid & 15) : (tid >> 4);
    const int tc = c_rows ? (tid >> 4) : (tid & 15);
    for (long long m0 = 0; m0 < M; m0 += GEMM_BM) {
      for (long long n0 = 0; n0 < N; n0 += GEMM_BN) {
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
        for (long long k0 = 0; k0 < K; k0 += GEMM_BK) {
          for (int e = tid; e < GEMM_BK * GEMM_BM; e += 256) {
            int kk, mm;
            if (a_kfast) { kk = e & (GEMM_BK - 1); mm = e / GEMM_BK; }
            else { kk = e / GEMM_BM; mm = e - kk * GEMM_BM; }
            long long r = m0 + mm, k = k0 + kk;
            sA[kk * GEMM_LDA + mm] = (r < M && k < K) ? A.ld(r, k) : 0.0;
          }
          for (int e = tid; e < GEMM_BK * GEMM_BN; e += 256) {
            int kk, nn;
            if (b_kfast) { kk = e & (GEMM_BK - 1); nn = e / GEMM_BK; }
            else { kk = e / GEMM_BN; nn = e - kk * GEMM_BN; }
            long long c = n0 + nn, k = k0 + kk;
            sB[kk * GEMM_LDB + nn] = (c < N && k < K) ? B.ld(k, c) : 0.0;
          }
          __syncthreads();
#pragma unroll 4
          for (int kk = 0; kk < GEMM_BK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = sA[kk * GEMM_LDA + tr + 16 * q];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = sB[kk * GEMM_LDB + tc + 16 * q];
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
              for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
          }
          __syncthreads();
        }
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          long long r = m0 + tr + 16 * x;
          if (r >= M) continue;
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            long long c = n0 + tc + 16 * y;
            if (c < N) C.ref(r, c) = accum ? C.ref(r, c) + acc[x][y] : acc[x][y];
          }
        }
      }
    }
    __syncthreads();
    return;
  }
#endif
  // Small problems (and the host build): one output element per thread.
  for (long long e = T.rank(); e < M * N; e += T.size()) {
    long long r, c;
    divmod(e, M, &r, &c);
    double s = 0.0;
    for (long long k = 0; k < K; ++k) s = fma(A.ld(r, k), B.ld(k, c), s);
    C.ref(r, c) = accum ? C.ref(r, c) + s : s;
  }
  T.sync();
}

// ---------------------------------------------------------------------------
// Elementwise helpers
// ---------------------------------------------------------------------------
CATN_HDI inline void copy(const Team& T, double* dst, const double* src, long long n) {
  for (long long e = T.rank(); e < n; e += T.size()) dst[e] = src[e];
  T.sync();
}
CATN_HDI inline void fill(const Team& T, double* dst, double v, long long n) {
  for (long long e = T.rank(); e < n; e += T.size()) dst[e] = v;
  T.sync();
}
CATN_HDI inline void scale(const Team& T, double* dst, double v, long long n) {
  for (long long e = T.rank(); e < n; e += T.size()) dst[e] *= v;
  T.sync();
}
// dst(rows x cols, col-major ld_d) = op(r, c)
CATN_HDI inline void materialize(const Team& T, double* dst, long long rows, long long cols,
                                 long long ldd, const MOp& op) {
  for (long long e = T.rank(); e < rows * cols; e += T.size()) {
    long long r, c;
    divmod(e, rows, &r, &c);
    dst[r + c * ldd] = op.ld(r, c);
  }
  T.sync();
}
CATN_HDI inline double sumsq(const Team& T, const double* x, long long n) {
  double s = 0.0;
  for (long long e = T.rank(); e < n; e += T.size()) s = fma(x[e], x[e], s);
  return T.sum(s);
}
CATN_HDI inline double sumv(const Team& T, const double* x, long long n) {
  double s = 0.0;
  for (long long e = T.rank(); e < n; e += T.size()) s += x[e];
  return T.sum(s);
}
CATN_HDI inline double maxabs(const Team& T, const double* x, long long n) {
  double s = 0.0;
  for (long long e = T.rank(); e < n; e += T.size()) s = fmax(s, fabs(x[e]));
  return T.maxv(s);
}

// ---------------------------------------------------------------------------
// Householder reflector H = I - tk v v^T (v = [1 at row k; v[k+1:m]]) applied
// to the columns j0 <= j < j1 of X (ld ldx); with nrm, the squared norm of
// rows k+1..m-1 of each updated column goes to nrm[j] in the same pass.
// Each warp takes NC columns at a time, so their loads are in flight together.
// ---------------------------------------------------------------------------
template <int NC>
CATN_HDI inline void house_apply_cols_n(const Team& T, const double* v, long long k, long long m, double tk,
                                        double* X, long long ldx, long long j0, long long j1, double* nrm) {
  for (long long jb = j0 + NC * T.warp(); jb < j1; jb += NC * T.nwarps()) {
    double* c[NC];
    bool on[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      on[q] = jb + q < j1;
      c[q] = X + (on[q] ? jb + q : jb) * ldx;
    }
    double w[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) w[q] = 0.0;
    if (tk != 0.0) {
      for (long long i = k + 1 + T.lane(); i < m; i += T.wsize()) {
        const double vi = v[i];
#pragma unroll
        for (int q = 0; q < NC; ++q) w[q] = fma(vi, c[q][i], w[q]);
      }
#pragma unroll
      for (int q = 0; q < NC; ++q) w[q] = (T.wsum(w[q]) + c[q][k]) * tk;
      T.wsync();
    }
    double s[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) s[q] = 0.0;
    if (tk != 0.0) {
      // two rows of every column per trip, all loads issued before the
      // stores (the columns may alias as far as the compiler knows)
      for (long long i0 = k + 1 + T.lane(); i0 < m; i0 += 2 * T.wsize()) {
        const long long i1 = i0 + T.wsize();
        const bool h1 = i1 < m;
        const double v0 = v[i0], v1 = h1 ? v[i1] : 0.0;
        double x0[NC], x1[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          x0[q] = c[q][i0];
          x1[q] = h1 ? c[q][i1] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          x0[q] = fma(-w[q], v0, x0[q]);
          x1[q] = fma(-w[q], v1, x1[q]);
          s[q] = fma(x0[q], x0[q], s[q]);
          s[q] = fma(x1[q], x1[q], s[q]);
        }
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          if (!on[q]) continue;
          c[q][i0] = x0[q];
          if (h1) c[q][i1] = x1[q];
        }
      }
    } else if (nrm) {
      for (long long i = k + 1 + T.lane(); i < m; i += T.wsize()) {
#pragma unroll
        for (int q = 0; q < NC; ++q) s[q] = fma(c[q][i], c[q][i], s[q]);
      }
    }
    if (nrm) {
#pragma unroll
      for (int q = 0; q < NC; ++q) s[q] = T.wsum(s[q]);
    }
    T.wsync();
    if (T.lane() == 0) {
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        if (!on[q]) continue;
        if (tk != 0.0) c[q][k] -= w[q];
        if (nrm) nrm[jb + q] = s[q];
      }
    }
    T.wsync();
  }
}
// Columns per warp: enough columns for every warp first, then up to four.
CATN_HDI inline void house_apply_cols(const Team& T, const double* v, long long k, long long m, double tk,
                                      double* X, long long ldx, long long j0, long long j1, double* nrm) {
  if (tk == 0.0 && !nrm) return;
  const long long per = (j1 - j0) / T.nwarps();
  if (per >= 4) house_apply_cols_n<4>(T, v, k, m, tk, X, ldx, j0, j1, nrm);
  else if (per >= 2) house_apply_cols_n<2>(T, v, k, m, tk, X, ldx, j0, j1, nrm);
  else house_apply_cols_n<1>(T, v, k, m, tk, X, ldx, j0, j1, nrm);
}

// ---------------------------------------------------------------------------
// Householder QR, m >= n, in place (LAPACK dgeqr2 semantics).
// ---------------------------------------------------------------------------
CATN_HDI inline void qr_inplace(const Team& T, double* A, long long m, long long n, long long lda,
                                double* tau) {
  for (long long k = 0; k < n; ++k) {
    double* ak = A + k * lda;
    double loc = 0.0;
    for (long long i = k + 1 + T.rank(); i < m; i += T.size()) loc = fma(ak[i], ak[i], loc);
    double xnorm2 = T.sum(loc);
    double alpha = ak[k];
    double tk = 0.0;
    if (xnorm2 > 0.0) {
      double beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
      tk = (beta - alpha) / beta;
      double sc = 1.0 / (alpha - beta);
      for (long long i = k + 1 + T.rank(); i < m; i += T.size()) ak[i] *= sc;
      T.sync();
      if (T.leader()) ak[k] = beta;
    }
    if (T.leader()) tau[k] = tk;
    T.sync();
    if (tk != 0.0 && k + 1 < n) {
      // A[k:m, j] -= tk * v * (v^T A[k:m, j]),  v = [1; A[k+1:m, k]]
      house_apply_cols(T, ak, k, m, tk, A, lda, k + 1, n, nullptr);
      T.sync();
    }
  }
}

// Householder QR with column pivoting, m >= n, in place: A P = Q R
// (LAPACK dgeqp3 semantics; partial column norms are recomputed exactly
// while each reflector is applied).  piv[k] = original index of column k.
// With stop_tol > 0 the factorisation ends at the first step k >= 1 where
// the trailing block's Frobenius norm sqrt(sum_j>=k nrm[j]) <= stop_tol and
// returns that rank k (every singular value of the dropped block is below
// stop_tol); otherwise it returns n.
CATN_HDI inline long long qrcp_inplace(const Team& T, double* A, long long m, long long n, long long lda,
                                       double* tau, int* piv, double* nrm, double stop_tol = 0.0) {
  for (long long j = T.warp(); j < n; j += T.nwarps()) {
    const double* aj = A + j * lda;
    double s = 0.0;
    for (long long i = T.lane(); i < m; i += T.wsize()) s = fma(aj[i], aj[i], s);
    s = T.wsum(s);
    if (T.lane() == 0) { nrm[j] = s; piv[j] = (int)j; }
  }
  T.sync();
  for (long long k = 0; k < n; ++k) {
    // pivot: largest remaining partial norm
    double bv = -1.0, rem = 0.0;
    long long bi = -1;
    for (long long j = k + T.rank(); j < n; j += T.size()) {
      double v = nrm[j];
      rem += v;
      if (bi < 0 || v > bv) { bv = v; bi = j; }
    }
    if (stop_tol > 0.0 && k > 0) {
      rem = T.sum(rem);
      if (rem <= stop_tol * stop_tol) return k;
    }
    long long p = T.argmax(bv, bi);
    if (p != k && p >= 0) {
      double* ak = A + k * lda;
      double* ap = A + p * lda;
      for (long long i = T.rank(); i < m; i += T.size()) {
        double t = ak[i]; ak[i] = ap[i]; ap[i] = t;
      }
      T.sync();
      if (T.leader()) {
        double t = nrm[k]; nrm[k] = nrm[p]; nrm[p] = t;
        int q = piv[k]; piv[k] = piv[p]; piv[p] = q;
      }
      T.sync();
    }
    double* ak = A + k * lda;
    double loc = 0.0;
    for (long long i = k + 1 + T.rank(); i < m; i += T.size()) loc = fma(ak[i], ak[i], loc);
    double xnorm2 = T.sum(loc);
    double alpha = ak[k];
    double tk = 0.0;
    if (xnorm2 > 0.0) {
      double beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
      tk = (beta - alpha) / beta;
      double sc = 1.0 / (alpha - beta);
      for (long long i = k + 1 + T.rank(); i < m; i += T.size()) ak[i] *= sc;
      T.sync();
      if (T.leader()) ak[k] = beta;
    }
    if (T.leader()) tau[k] = tk;
    T.sync();
    if (k + 1 < n) {
      house_apply_cols(T, ak, k, m, tk, A, lda, k + 1, n, nrm);
      T.sync();
    }
  }
  return n;
}

// C(m x ncols, ld ldc) <- Q * C with Q = H_0 ... H_{n-1} from qr_inplace.
CATN_HDI inline void qr_apply_q(const Team& T, const double* A, long long m, long long n,
                                long long lda, const double* tau, double* C, long long ncols,
                                long long ldc) {
  for (long long k = n - 1; k >= 0; --k) {
    double tk = tau[k];
    if (tk == 0.0) continue;
    house_apply_cols(T, A + k * lda, k, m, tk, C, ldc, 0, ncols, nullptr);
    T.sync();
  }
}

// qr_apply_q by panels of up to b reflectors (compact WY form): the panel
// H_k0 ... H_k0+kb-1 equals I - V T V^T with V (rows k0..m-1) unit lower
// trapezoidal and T upper triangular, T_jj = tau_j and T[0:j, j] =
// -tau_j T[0:j, 0:j] (V[:, 0:j]^T v_j).  N = -T obeys the same recurrence
// with N_jj = -tau_j, so C[k0:m] += V (N (V^T C[k0:m])): three GEMMs per
// panel instead of one pass over C per reflector.  Panels go last to first
// (Q = H_0 H_1 ... H_{n-1}).  work: (m + 2 ncols + 2 b) b doubles.
CATN_HDI inline void qr_apply_q_blocked(const Team& T, const double* A, long long m, long long n, long long lda,
                                        const double* tau, double* C, long long ncols, long long ldc, long long b,
                                        double* work) {
  double* Vp = work;           // mp x kb, ld mp
  double* G = Vp + m * b;      // kb x kb: V^T V
  double* Nm = G + b * b;      // kb x kb: -T
  double* Y = Nm + b * b;      // kb x ncols: V^T C, then Y2 = N Y
  double* Y2 = Y + b * ncols;
  for (long long p = (n + b - 1) / b - 1; p >= 0; --p) {
    const long long k0 = p * b, kb = (n - k0 < b) ? n - k0 : b, mp = m - k0;
    for (long long e = T.rank(); e < mp * kb; e += T.size()) {
      long long i, j;
      divmod(e, mp, &i, &j);
      Vp[e] = (i > j) ? A[k0 + i + (k0 + j) * lda] : (i == j ? 1.0 : 0.0);
    }
    for (long long e = T.rank(); e < kb * kb; e += T.size()) Nm[e] = 0.0;
    T.sync();
    gemm(T, kb, kb, mp, transposed(Vp, mp), colmajor(Vp, mp), colmajor(G, kb));
    for (long long j = 0; j < kb; ++j) {
      const double tj = tau[k0 + j];
      for (long long i = T.rank(); i <= j; i += T.size()) {
        double s = 0.0;
        for (long long l = i; l < j; ++l) s = fma(Nm[i + l * kb], G[l + j * kb], s);
        Nm[i + j * kb] = -tj * (i == j ? 1.0 : s);
      }
      T.sync();
    }
    gemm(T, kb, ncols, mp, transposed(Vp, mp), colmajor(C + k0, ldc), colmajor(Y, kb));
    gemm(T, kb, ncols, kb, colmajor(Nm, kb), colmajor(Y, kb), colmajor(Y2, kb));
    gemm(T, mp, ncols, kb, colmajor(Vp, mp), colmajor(Y2, kb), colmajor(C + k0, ldc), true);
  }
}

// ---------------------------------------------------------------------------
// One-sided Jacobi on B (m x n, m >= n, col-major ld ldb), accumulating V
// (n x n, ld n).  Columns of B converge to U * diag(S).  Returns the number
// of sweeps, or -1 when the sweep cap was reached.
// ---------------------------------------------------------------------------
// 1 / sqrt(x) (the host build divides).
CATN_HD double rsqrt_d(double x) {
#if CATN_DEVICE_PASS
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}

// Jacobi rotation annihilating the off-diagonal g of the 2x2 Gram block
// [[al, g], [g, be]]: returns false when the pair is already orthogonal to
// tolerance (g^2 <= tol^2 al be) or a column is numerically zero; otherwise
// c = cos, s = sin of the angle with tan = t = sign(d g) 2|g| / (|d| + r),
// d = be - al, r^2 = d^2 + 4 g^2, in half-angle form: cos 2a = |d| / r,
// c = sqrt((1 + cos 2a) / 2), s = sign(d g) |g| / (r c), t = s / c -- two
// reciprocal square roots and no division (d == 0 takes the sign of g).
CATN_HD bool jacobi_rotation(double al, double be, double g, double tol, double* c, double* s, double* t = nullptr) {
  if (al < 1e-250 || be < 1e-250) return false;
  if (!(g * g > tol * tol * al * be)) return false;
  const double d = be - al;
  const double rr = rsqrt_d(fma(d, d, 4.0 * g * g));   // 1 / r
  const double q = fma(0.5 * fabs(d), rr, 0.5);        // c^2
  const double kq = rsqrt_d(q);                          // 1 / c
  const double sv = fabs(g) * rr * kq;
  const double sg = ((d < 0.0) != (g < 0.0)) ? -sv : sv;
  *c = q * kq;
  *s = sg;
  if (t) *t = sg * kq;
  return true;
}

// Round-robin (circle method) schedule over np (even) players, player 0
// fixed: in round r (0 <= r < np-1) position k holds player
// ((k - 1 + r) mod (np - 1)) + 1 for k >= 1, and pair i joins the players at
// positions i and np-1-i.  Division-free: r < np-1 and k < np.
CATN_HD int rr_at(int np, int r, int k) {
  if (k == 0) return 0;
  int t = k - 1 + r;
  if (t >= np - 1) t -= np - 1;
  return t + 1;
}
CATN_HD void rr_pair(long long np, long long r, long long i, long long* a, long long* b) {
  *a = rr_at((int)np, (int)r, (int)i);
  *b = rr_at((int)np, (int)r, (int)(np - 1 - i));
}
// Partner of player j in round r.
CATN_HD int rr_partner(int np, int r, int j) {
  int k = 0;   // position of player j
  if (j != 0) {
    k = j - 1 - r;
    if (k < 0) k += np - 1;
    k += 1;
  }
  return rr_at(np, r, np - 1 - k);
}

CATN_HDI inline int jacobi_sweeps(const Team& T, double* B, long long m, long long n, long long ldb,
                                  double* V, int max_sweeps, double* nrm) {
  for (long long e = T.rank(); e < n * n; e += T.size()) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  T.sync();
  if (n < 2) return 0;
  // Work at unit max-abs scale so that numerically-zero columns are
  // recognised by an absolute threshold and never reach denormal range.
  double mx = 0.0;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) mx = fmax(mx, fabs(B[i + c * ldb]));
  mx = T.maxv(mx);
  const double sc = mx > 0.0 ? 1.0 / mx : 1.0;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) B[i + c * ldb] *= sc;
  T.sync();
  const long long np = (n % 2) ? n + 1 : n;
  const long long npair = np / 2;
  const double tol = 2.220446049250313e-16 * (double)(m > 16 ? m : 16);
  const int nw = T.nwarps();
  int result = -1;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    // squared column norms, recomputed each sweep; within a sweep a rotation
    // by t updates them as |b_p|^2 -= t g, |b_q|^2 += t g (Rutishauser)
    for (long long c = T.warp(); c < n; c += nw) {
      const double* bc = B + c * ldb;
      double s2 = 0.0;
      for (long long i = T.lane(); i < m; i += T.wsize()) s2 = fma(bc[i], bc[i], s2);
      s2 = T.wsum(s2);
      if (T.lane() == 0) nrm[c] = s2;
    }
    T.sync();
    int rotated = 0;
    for (long long r = 0; r < np - 1; ++r) {
      // two pairs per warp in flight, so that their memory latencies overlap
      for (long long pi = T.warp(); pi < npair; pi += 2 * nw) {
        long long p0, q0, p1 = 0, q1 = 0;
        rr_pair(np, r, pi, &p0, &q0);
        const bool h1 = pi + nw < npair;
        if (h1) rr_pair(np, r, pi + nw, &p1, &q1);
        const bool a0 = p0 < n && q0 < n, a1 = h1 && p1 < n && q1 < n;
        double* bp0 = B + p0 * ldb;
        double* bq0 = B + q0 * ldb;
        double* bp1 = B + p1 * ldb;
        double* bq1 = B + q1 * ldb;
        double g0 = 0.0, g1 = 0.0;
        for (long long i = T.lane(); i < m; i += T.wsize()) {
          if (a0) g0 = fma(bp0[i], bq0[i], g0);
          if (a1) g1 = fma(bp1[i], bq1[i], g1);
        }
        g0 = T.wsum(g0);
        g1 = T.wsum(g1);
        double c0 = 1.0, s0 = 0.0, t0 = 0.0, c1 = 1.0, s1 = 0.0, t1 = 0.0;
        const bool r0 = a0 && jacobi_rotation(nrm[p0], nrm[q0], g0, tol, &c0, &s0, &t0);
        const bool r1 = a1 && jacobi_rotation(nrm[p1], nrm[q1], g1, tol, &c1, &s1, &t1);
        if (!r0 && !r1) continue;
        rotated = 1;
        T.wsync();
        for (long long i = T.lane(); i < m; i += T.wsize()) {
          if (r0) {
            const double x = bp0[i], y = bq0[i];
            bp0[i] = c0 * x - s0 * y;
            bq0[i] = s0 * x + c0 * y;
          }
          if (r1) {
            const double x = bp1[i], y = bq1[i];
            bp1[i] = c1 * x - s1 * y;
            bq1[i] = s1 * x + c1 * y;
          }
        }
        double* vp0 = V + p0 * n;
        double* vq0 = V + q0 * n;
        double* vp1 = V + p1 * n;
        double* vq1 = V + q1 * n;
        for (long long i = T.lane(); i < n; i += T.wsize()) {
          if (r0) {
            const double x = vp0[i], y = vq0[i];
            vp0[i] = c0 * x - s0 * y;
            vq0[i] = s0 * x + c0 * y;
          }
          if (r1) {
            const double x = vp1[i], y = vq1[i];
            vp1[i] = c1 * x - s1 * y;
            vq1[i] = s1 * x + c1 * y;
          }
        }
        T.wsync();
        if (T.lane() == 0) {
          if (r0) {
            nrm[p0] -= t0 * g0;
            nrm[q0] += t0 * g0;
          }
          if (r1) {
            nrm[p1] -= t1 * g1;
            nrm[q1] += t1 * g1;
          }
        }
        T.wsync();
      }
      T.sync();
    }
    if (!T.any(rotated)) {
      result = sweep + 1;
      break;
    }
  }
  const double inv = 1.0 / sc;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) B[i + c * ldb] *= inv;
  T.sync();
  return result;
}

// Work of one CTA's large SVD opened to idle warps of other CTAs (helper
// CTAs of a batch, the other CTAs of a single-network launch).  A job runs
// in rounds; each round has `count` items that warps claim through `word` =
// (round sequence << 40) | (count << 20) | claims so far, so a claim always
// knows the count of the round it counted in.  The owner publishes a round
// only after every item of the previous one reported done, and the round's
// payload (round, k, tk, c0) is written before the round is published, so a
// valid claim may read it.  Kinds: Jacobi column pairs of one round-robin
// round (B, V, nrm); Householder reflector k applied to 4-column chunks of C
// from column c0 (reflector in column k of A), with the trailing squared
// norms recomputed into nrm when nrm is set (pivoted QR); block pairs of the
// block Jacobi route (blockjac.cuh) and 32-column tiles of a blocked QR's
// trailing update (blockqr.cuh), both claimed by whole CTAs.
enum { JOB_JACOBI = 0, JOB_HOUSE = 1, JOB_BLOCK = 2, JOB_PANEL = 3 };
constexpr int JOB_CHUNK = 4;   // columns per Householder claim
struct JacobiJob {
  unsigned long long word;
  int done, rotated, round, open;
  int kind, m, n, ldb, np, k, c0, ldc;
  int tc, pad;   // block items: products on the tensor cores (split precision)
  double tol, tk;
  double* B;     // Jacobi columns / Householder reflectors (A) / panel-update target
  double* V;     // Jacobi rotations / Householder target (C) / panel reflectors
  double* nrm;
  double* W2;    // panel update: -T of the compact WY form
};

// ---------------------------------------------------------------------------
// Shared jobs.  Every access to the shared matrices, V and the norms goes
// through L2 (ld/st .cg): an SM's L1 is not coherent with writes of other SMs.
// ---------------------------------------------------------------------------
#if CATN_DEVICE_PASS
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ void stcg(double* p, double v) { __stcg(p, v); }
__device__ __forceinline__ int ldcg_i(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long ldcg_u(const unsigned long long* p) { return __ldcg(p); }
__device__ __forceinline__ void fence_gpu() { __threadfence(); }
#else
inline double ldcg(const double* p) { return *p; }
inline void stcg(double* p, double v) { *p = v; }
inline int ldcg_i(const int* p) { return *p; }
inline unsigned long long ldcg_u(const unsigned long long* p) { return *p; }
inline void fence_gpu() {}
#endif

CATN_HD unsigned long long job_word(unsigned long long seq, long long count) {
  return (seq << 40) | ((unsigned long long)count << 20);
}

// Poll limit of the owner's wait for claimed items (a claimed item is a few
// microseconds of work; 2^24 polls of >= 64 ns is over a second).  The test
// build of the host harness sets it small.
#ifndef CATN_JOB_SPIN_CAP
#define CATN_JOB_SPIN_CAP (1LL << 24)
#endif
// Claims already counted when a round is published: always 0 in the library.
// The host harness's timeout test sets it to 1, which models a helper warp
// that claimed an item and never reported it done.
#ifndef CATN_JOB_PHANTOM_CLAIMS
#define CATN_JOB_PHANTOM_CLAIMS 0
#endif
CATN_HD void job_set_word(JacobiJob* J, unsigned long long w) {
#if CATN_DEVICE_PASS
  atomicExch(&J->word, w);
#else
  J->word = w;
#endif
}

// Rows per lane of the register-resident pair rotation (columns up to
// kPairRows warps long).
constexpr int kPairRows = 8;

// Pair pi of round r (round-robin order) on B (m x n) and V (n x n) with
// the squared norms in nrm; warp-level.  Returns whether it rotated.  With
// m, n <= kPairRows * warp size every load (both columns of B and of V, both
// norms) is issued at once and the columns stay in registers for the
// rotation, so a pair costs one L2 round trip instead of one per row block.
CATN_HDI inline bool jacobi_pair_l2(const Team& T, double* B, double* V, double* nrm, long long m, long long n,
                                    long long ldb, long long np, long long r, long long pi, double tol) {
  long long p, q;
  rr_pair(np, r, pi, &p, &q);
  if (p >= n || q >= n) return false;
  double* bp = B + p * ldb;
  double* bq = B + q * ldb;
  double* vp = V + p * n;
  double* vq = V + q * n;
  const double al = ldcg(nrm + p), be = ldcg(nrm + q);
  double c, s, t, g = 0.0;
  const long long ws = T.wsize();
  if (m <= ws * kPairRows && n <= ws * kPairRows) {
    double xp[kPairRows], xq[kPairRows], yp[kPairRows], yq[kPairRows];
#pragma unroll
    for (int e = 0; e < kPairRows; ++e) {
      const long long i = T.lane() + ws * e;
      xp[e] = i < m ? ldcg(bp + i) : 0.0;
      xq[e] = i < m ? ldcg(bq + i) : 0.0;
      yp[e] = i < n ? ldcg(vp + i) : 0.0;
      yq[e] = i < n ? ldcg(vq + i) : 0.0;
    }
#pragma unroll
    for (int e = 0; e < kPairRows; ++e) g = fma(xp[e], xq[e], g);
    g = T.wsum(g);
    if (!jacobi_rotation(al, be, g, tol, &c, &s, &t)) return false;
#pragma unroll
    for (int e = 0; e < kPairRows; ++e) {
      const long long i = T.lane() + ws * e;
      if (i < m) {
        stcg(bp + i, c * xp[e] - s * xq[e]);
        stcg(bq + i, s * xp[e] + c * xq[e]);
      }
      if (i < n) {
        stcg(vp + i, c * yp[e] - s * yq[e]);
        stcg(vq + i, s * yp[e] + c * yq[e]);
      }
    }
  } else {
    for (long long i = T.lane(); i < m; i += T.wsize()) g = fma(ldcg(bp + i), ldcg(bq + i), g);
    g = T.wsum(g);
    if (!jacobi_rotation(al, be, g, tol, &c, &s, &t)) return false;
    for (long long i = T.lane(); i < m; i += T.wsize()) {
      const double x = ldcg(bp + i), y = ldcg(bq + i);
      stcg(bp + i, c * x - s * y);
      stcg(bq + i, s * x + c * y);
    }
    for (long long i = T.lane(); i < n; i += T.wsize()) {
      const double x = ldcg(vp + i), y = ldcg(vq + i);
      stcg(vp + i, c * x - s * y);
      stcg(vq + i, s * x + c * y);
    }
  }
  T.wsync();
  if (T.lane() == 0) {
    stcg(nrm + p, al - t * g);
    stcg(nrm + q, be + t * g);
  }
  T.wsync();
  return true;
}

// Rows per lane of the register-resident reflector application (columns up
// to kHouseRows warps long below the reflector's row).
constexpr int kHouseRows = 32;

// Reflector k (v = A[k+1:m, k] with an implicit 1 at k, factor tk) applied to
// column j of C; with nrm, the squared norm of C[k+1:m, j] goes to nrm[j].
// Warp-level, through L2.  When the rows below k fit kHouseRows per lane,
// the reflector and the column are loaded at once and kept in registers for
// the dot product, the update and the norm: one L2 round trip instead of
// one per row block and pass.
CATN_HDI inline void house_col_l2(const Team& T, const double* A, long long m, long long lda, long long k, double tk,
                                  double* C, long long ldc, long long j, double* nrm) {
  const double* ak = A + k * lda;
  double* cj = C + j * ldc;
  const long long ws = T.wsize();
  if (m - (k + 1) <= ws * kHouseRows) {
    double vr[kHouseRows], cr[kHouseRows];
#pragma unroll
    for (int e = 0; e < kHouseRows; ++e) {
      const long long i = k + 1 + T.lane() + ws * e;
      vr[e] = (i < m && tk != 0.0) ? ldcg(ak + i) : 0.0;
      cr[e] = i < m ? ldcg(cj + i) : 0.0;
    }
    double w = 0.0;
    if (tk != 0.0) {
      const double ck = ldcg(cj + k);
#pragma unroll
      for (int e = 0; e < kHouseRows; ++e) w = fma(vr[e], cr[e], w);
      w = (T.wsum(w) + ck) * tk;
      T.wsync();
      if (T.lane() == 0) stcg(cj + k, ck - w);
    }
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < kHouseRows; ++e) {
      const long long i = k + 1 + T.lane() + ws * e;
      if (tk != 0.0) {
        cr[e] = fma(-w, vr[e], cr[e]);
        if (i < m) stcg(cj + i, cr[e]);
      }
      s = fma(cr[e], cr[e], s);
    }
    if (nrm) {
      s = T.wsum(s);
      if (T.lane() == 0) stcg(nrm + j, s);
    }
    T.wsync();
    return;
  }
  if (tk != 0.0) {
    double w = 0.0;
    for (long long i = k + 1 + T.lane(); i < m; i += T.wsize()) w = fma(ldcg(ak + i), ldcg(cj + i), w);
    w = (T.wsum(w) + ldcg(cj + k)) * tk;
    T.wsync();
    if (T.lane() == 0) stcg(cj + k, ldcg(cj + k) - w);
    for (long long i = k + 1 + T.lane(); i < m; i += T.wsize()) stcg(cj + i, ldcg(cj + i) - w * ldcg(ak + i));
    T.wsync();
  }
  if (nrm) {
    double s = 0.0;
    for (long long i = k + 1 + T.lane(); i < m; i += T.wsize()) {
      const double x = ldcg(cj + i);
      s = fma(x, x, s);
    }
    s = T.wsum(s);
    if (T.lane() == 0) stcg(nrm + j, s);
    T.wsync();
  }
}

// One claim on J by the calling warp: the item index in the current round,
// or -1 when the round has none left.
CATN_HDI inline long long job_claim(const Team& T, JacobiJob* J) {
#if CATN_DEVICE_PASS
  unsigned long long old = 0;
  if (T.lane() == 0) old = atomicAdd(&J->word, 1ULL);
  old = __shfl_sync(0xffffffffu, old, 0);
#else
  const unsigned long long old = J->word;
  J->word = old + 1;
#endif
  const long long item = (long long)(old & 0xfffffULL);
  const long long count = (long long)((old >> 20) & 0xfffffULL);
  if (item >= count) return -1;
  fence_gpu();
  return item;
}

// The calling warp's share of the current round of J: claims until none is
// left, reports each item done.
CATN_HDI inline void job_work(const Team& T, JacobiJob* J) {
  for (;;) {
    const long long item = job_claim(T, J);
    if (item < 0) return;
    // the job's fields through L2 as well: this SM may hold lines of an earlier job
    double* B = (double*)ldcg_u((const unsigned long long*)&J->B);
    double* V = (double*)ldcg_u((const unsigned long long*)&J->V);
    double* nrm = (double*)ldcg_u((const unsigned long long*)&J->nrm);
    bool rot = false;
    if (ldcg_i(&J->kind) == JOB_JACOBI) {
      rot = jacobi_pair_l2(T, B, V, nrm, ldcg_i(&J->m), ldcg_i(&J->n), ldcg_i(&J->ldb), ldcg_i(&J->np),
                           ldcg_i(&J->round), item, ldcg(&J->tol));
    } else {
      const long long m = ldcg_i(&J->m), lda = ldcg_i(&J->ldb), k = ldcg_i(&J->k), ldc = ldcg_i(&J->ldc);
      const long long c0 = ldcg_i(&J->c0), cend = ldcg_i(&J->n);
      const double tk = ldcg(&J->tk);
      for (long long j = c0 + item * JOB_CHUNK; j < cend && j < c0 + (item + 1) * JOB_CHUNK; ++j)
        house_col_l2(T, B, m, lda, k, tk, V, ldc, j, nrm);
    }
    fence_gpu();
    if (T.lane() == 0) {
#if CATN_DEVICE_PASS
      if (rot) atomicOr(&J->rotated, 1);
      atomicAdd(&J->done, 1);
#else
      if (rot) J->rotated = 1;
      J->done += 1;
#endif
    }
    T.wsync();
  }
}

// Owner side: open J (closed word first, then the fields the caller set,
// then `open`), returning the first round's sequence number.
CATN_HDI inline unsigned long long job_open(const Team& T, JacobiJob* J) {
  unsigned long long seq = (ldcg_u(&J->word) >> 40) + 1;
  T.sync();
  if (T.leader()) {
    job_set_word(J, job_word(seq, 0));   // closed: no claim can count
    fence_gpu();
  }
  return seq + 1;
}
// Owner side: wait (bounded) until every item of the round is reported done.
// Returns 1 when the wait ran out.
CATN_HDI inline int job_wait_done(const Team& T, JacobiJob* J, long long count) {
  int timed_out = 0;
  if (T.leader()) {
    long long spins = 0;
    while (ldcg_i(&J->done) < count) {
      if (++spins > CATN_JOB_SPIN_CAP) {   // claimed items never take this long
        timed_out = 1;
        break;
      }
#if CATN_DEVICE_PASS
      __nanosleep(64);
#endif
    }
    fence_gpu();
    T.red[0] = timed_out ? 1.0 : 0.0;
  }
  T.sync();
  timed_out = T.red[0] > 0.5;
  T.sync();
  return timed_out;
}
// Publish one round of `count` items (the leader has written its payload),
// do the team's share, wait (bounded) until every item is done.  Returns 1
// when the wait ran out.
CATN_HDI inline int job_round(const Team& T, JacobiJob* J, unsigned long long seq, long long count) {
  if (T.leader()) {
    J->done = 0;
    fence_gpu();
    job_set_word(J, job_word(seq, count) + (count > 0 ? CATN_JOB_PHANTOM_CLAIMS : 0));
  }
  T.sync();
  job_work(T, J);
  return job_wait_done(T, J, count);
}
CATN_HDI inline void job_close(const Team& T, JacobiJob* J, unsigned long long seq) {
  if (T.leader()) {
    J->open = 0;
    fence_gpu();
    job_set_word(J, job_word(seq, 0));
  }
  T.sync();
}

// jacobi_sweeps with every round's pairs claimed dynamically through J by
// the team's warps and by helper warps of other CTAs (help_jobs).  Returns
// the sweep count, -1 without convergence, -2 when a wait for claimed pairs
// ran out (the caller reports it as an error).  B and V are rewritten
// through the calling SM at the end, so later plain loads see the helpers'
// writes.
CATN_HDI inline int jacobi_sweeps_shared(const Team& T, JacobiJob* J, double* B, long long m, long long n,
                                         long long ldb, double* V, int max_sweeps, double* nrm) {
  for (long long e = T.rank(); e < n * n; e += T.size()) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  T.sync();
  if (n < 2) return 0;
  double mx = 0.0;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) mx = fmax(mx, fabs(B[i + c * ldb]));
  mx = T.maxv(mx);
  const double sc = mx > 0.0 ? 1.0 / mx : 1.0;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) B[i + c * ldb] *= sc;
  const long long np = (n % 2) ? n + 1 : n;
  const int npair = (int)(np / 2);
  const double tol = 2.220446049250313e-16 * (double)(m > 16 ? m : 16);
  unsigned long long seq = job_open(T, J);
  if (T.leader()) {
    J->kind = JOB_JACOBI;
    J->B = B; J->V = V; J->nrm = nrm;
    J->m = (int)m; J->n = (int)n; J->ldb = (int)ldb; J->np = (int)np; J->tol = tol;
    J->rotated = 0; J->round = 0;
    fence_gpu();
    J->open = 1;
    fence_gpu();
  }
  T.sync();
  int result = -1;
  int timed_out = 0;
  for (int sweep = 0; sweep < max_sweeps && !timed_out; ++sweep) {
    for (long long c = T.warp(); c < n; c += T.nwarps()) {
      const double* bc = B + c * ldb;
      double s2 = 0.0;
      for (long long i = T.lane(); i < m; i += T.wsize()) {
        const double x = ldcg(bc + i);
        s2 = fma(x, x, s2);
      }
      s2 = T.wsum(s2);
      if (T.lane() == 0) stcg(nrm + c, s2);
    }
    fence_gpu();
    T.sync();
    if (T.leader()) J->rotated = 0;
    for (long long r = 0; r < np - 1 && !timed_out; ++r) {
      if (T.leader()) J->round = (int)r;
      timed_out = job_round(T, J, seq, npair);
      ++seq;
    }
    fence_gpu();
    T.sync();
    const int rot = ldcg_i(&J->rotated);
    T.sync();
    if (!rot) {
      result = sweep + 1;
      break;
    }
  }
  job_close(T, J, seq);
  const double inv = 1.0 / sc;
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) B[i + c * ldb] = ldcg(B + i + c * ldb) * inv;
  for (long long e = T.rank(); e < n * n; e += T.size()) V[e] = ldcg(V + e);
  T.sync();
  return timed_out ? -2 : result;
}

// qrcp_inplace with each step's trailing update (and norm recomputation)
// shared through J in 4-column chunks.  Same arithmetic per column; returns
// the rank reached, or -2 when a wait ran out.  A is rewritten through the
// calling SM at the end.
CATN_HDI inline long long qrcp_shared(const Team& T, JacobiJob* J, double* A, long long m, long long n, long long lda,
                                      double* tau, int* piv, double* nrm, double stop_tol) {
  for (long long j = T.warp(); j < n; j += T.nwarps()) {
    const double* aj = A + j * lda;
    double s = 0.0;
    for (long long i = T.lane(); i < m; i += T.wsize()) s = fma(aj[i], aj[i], s);
    s = T.wsum(s);
    if (T.lane() == 0) { stcg(nrm + j, s); piv[j] = (int)j; }
  }
  fence_gpu();
  T.sync();
  unsigned long long seq = job_open(T, J);
  if (T.leader()) {
    J->kind = JOB_HOUSE;
    J->B = A; J->V = A; J->nrm = nrm;
    J->m = (int)m; J->n = (int)n; J->ldb = (int)lda; J->ldc = (int)lda;
    fence_gpu();
    J->open = 1;
    fence_gpu();
  }
  T.sync();
  long long rank = n;
  int timed_out = 0;
  for (long long k = 0; k < n && !timed_out; ++k) {
    double bv = -1.0, rem = 0.0;
    long long bi = -1;
    for (long long j = k + T.rank(); j < n; j += T.size()) {
      const double v = ldcg(nrm + j);
      rem += v;
      if (bi < 0 || v > bv) { bv = v; bi = j; }
    }
    if (stop_tol > 0.0 && k > 0) {
      rem = T.sum(rem);
      if (rem <= stop_tol * stop_tol) { rank = k; break; }
    }
    const long long p = T.argmax(bv, bi);
    double* ak = A + k * lda;
    if (p != k && p >= 0) {
      double* ap = A + p * lda;
      for (long long i = T.rank(); i < m; i += T.size()) {
        const double t = ldcg(ak + i);
        stcg(ak + i, ldcg(ap + i));
        stcg(ap + i, t);
      }
      T.sync();
      if (T.leader()) {
        const double t = ldcg(nrm + k);
        stcg(nrm + k, ldcg(nrm + p));
        stcg(nrm + p, t);
        const int q = piv[k]; piv[k] = piv[p]; piv[p] = q;
      }
      T.sync();
    }
    double loc = 0.0;
    for (long long i = k + 1 + T.rank(); i < m; i += T.size()) {
      const double x = ldcg(ak + i);
      loc = fma(x, x, loc);
    }
    const double xnorm2 = T.sum(loc);
    const double alpha = ldcg(ak + k);
    double tk = 0.0;
    if (xnorm2 > 0.0) {
      const double beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
      tk = (beta - alpha) / beta;
      const double sc = 1.0 / (alpha - beta);
      for (long long i = k + 1 + T.rank(); i < m; i += T.size()) stcg(ak + i, ldcg(ak + i) * sc);
      T.sync();
      if (T.leader()) stcg(ak + k, beta);
    }
    if (T.leader()) {
      tau[k] = tk;
      J->k = (int)k; J->tk = tk; J->c0 = (int)(k + 1);
    }
    fence_gpu();
    T.sync();
    const long long cols = n - k - 1;
    if (cols > 0) {
      timed_out = job_round(T, J, seq, (cols + JOB_CHUNK - 1) / JOB_CHUNK);
      ++seq;
    }
  }
  job_close(T, J, seq);
  for (long long c = 0; c < n; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) A[i + c * lda] = ldcg(A + i + c * lda);
  for (long long j = T.rank(); j < n; j += T.size()) nrm[j] = ldcg(nrm + j);
  T.sync();
  return timed_out ? -2 : rank;
}

// qr_apply_q with each reflector's update of C shared through J in 4-column
// chunks; returns 1 when a wait ran out.  C is rewritten through the
// calling SM at the end.
CATN_HDI inline int qr_apply_q_shared(const Team& T, JacobiJob* J, const double* A, long long m, long long n,
                                      long long lda, const double* tau, double* C, long long ncols, long long ldc) {
  fence_gpu();
  unsigned long long seq = job_open(T, J);
  if (T.leader()) {
    J->kind = JOB_HOUSE;
    J->B = (double*)A; J->V = C; J->nrm = nullptr;
    J->m = (int)m; J->n = (int)ncols; J->ldb = (int)lda; J->ldc = (int)ldc; J->c0 = 0;
    fence_gpu();
    J->open = 1;
    fence_gpu();
  }
  T.sync();
  int timed_out = 0;
  for (long long k = n - 1; k >= 0 && !timed_out; --k) {
    const double tk = tau[k];
    if (tk == 0.0) continue;
    if (T.leader()) { J->k = (int)k; J->tk = tk; }
    timed_out = job_round(T, J, seq, (ncols + JOB_CHUNK - 1) / JOB_CHUNK);
    ++seq;
  }
  job_close(T, J, seq);
  for (long long c = 0; c < ncols; ++c)
    for (long long i = T.rank(); i < m; i += T.size()) C[i + c * ldc] = ldcg(C + i + c * ldc);
  T.sync();
  return timed_out;
}

// Polls (of about 1 us each) that a helper keeps watching the job it last
// worked on for that job's next round before it scans the board again.
constexpr int kJobStickPolls = 64;

#if defined(__CUDACC__)
// Whether J is open with unclaimed items of its current round (warp-uniform:
// lane 0's view).
__device__ __forceinline__ bool job_has_items(const JacobiJob* J) {
  int open = ldcg_i(&J->open);
  unsigned long long word = ldcg_u(&J->word);
  open = __shfl_sync(0xffffffffu, open, 0);
  word = __shfl_sync(0xffffffffu, word, 0);
  return open && (word & 0xfffffULL) < ((word >> 20) & 0xfffffULL);
}

// Helper loop of launches whose jobs are all warp items (scalar Jacobi pairs
// and Householder columns): every warp scans the board, claims items and
// stays with its job independently, with no CTA barrier, until every
// instance of the launch is finished.  Launches that can publish CTA items
// (block Jacobi pairs, blocked-QR panels) use help_jobs instead.
__device__ inline void help_jacobi(const Team& T, JacobiJob* board, int nslots, const int* finished, int ninst) {
  const unsigned FULL = 0xffffffffu;
  const int w = (int)blockIdx.x * T.nwarps() + T.warp();
  const int lane = T.lane();
  long long idle = 0;
  while (idle < (1LL << 22)) {
    if (ldcg_i(finished) >= ninst) return;
    // find a job with unclaimed items: the lanes check 32 slots at once
    // (independent L2 loads), starting at a warp-specific block so that
    // helpers spread over the open jobs
    const int nblk = (nslots + 31) / 32;
    int pick = -1;
    for (int b = 0; b < nblk && pick < 0; ++b) {
      const int base = ((b + w) % nblk) * 32;
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
        const int r = w & 31;   // first candidate at or after lane r (cyclically)
        const unsigned hi = mask & (~0u << r);
        pick = base + __ffs(hi ? hi : mask) - 1;
      }
    }
    if (pick < 0) {
      ++idle;
      __nanosleep(256);
      continue;
    }
    idle = 0;
    JacobiJob* J = board + pick;
    job_work(T, J);
    // stay with J: its owner opens the next round within microseconds
    for (int t = 0; t < kJobStickPolls; ++t) {
      if (job_has_items(J)) {
        job_work(T, J);
        t = -1;
        continue;
      }
      if (!ldcg_i(&J->open)) break;
      __nanosleep(32);
    }
  }
}
#endif

// Column norms of B (n columns), then stable descending order.
// S_out[r] = sigma of the r-th largest column, perm[r] = its column index.
CATN_HDI inline void sort_columns(const Team& T, const double* B, long long m, long long n,
                                  long long ldb, double* sig, double* S_out, int* perm) {
  for (long long j = T.warp(); j < n; j += T.nwarps()) {
    const double* bj = B + j * ldb;
    double s = 0.0;
    for (long long i = T.lane(); i < m; i += T.wsize()) s = fma(bj[i], bj[i], s);
    s = T.wsum(s);
    if (T.lane() == 0) sig[j] = sqrt(s);
  }
  T.sync();
  for (long long j = T.rank(); j < n; j += T.size()) {
    double sj = sig[j];
    long long rk = 0;
    for (long long l = 0; l < n; ++l) {
      double sl = sig[l];
      rk += (sl > sj || (sl == sj && l < j)) ? 1 : 0;
    }
    perm[rk] = (int)j;
    S_out[rk] = sj;
  }
  T.sync();
}

}  // namespace catn

namespace catn {

#if CATN_DEVICE_PASS
// ---------------------------------------------------------------------------
// Tiny SVD by one warp (nn <= NN <= 16, nn <= mm <= ME * 32 / NN <= 64): the
// same method as the team path -- pivoted Householder QR W P = Q R, one-sided
// Jacobi on X = R^T, W = (Q V') Sigma (P U')^T -- with the whole problem in
// registers.  Each column is spread over LPC = 32 / NN lanes (lane = column +
// NN * part holds the rows part + LPC * e), so every lane works and the
// reductions are xor shuffles over the parts.  Pivoting tracks positions
// instead of moving columns; the Jacobi rounds pair column j with j ^ m
// (m = 1 .. NN-1, every pair once per sweep).  W (column-major, ld mm) is
// overwritten by the Householder form; outputs: Ut (mm x nn) = Q V'[:, perm],
// Vt (nn x nn) = P U'[:, perm], Sout (nn, descending).  Returns the sweep
// count (-1 when the cap was reached).  Must be called by all 32 lanes of one
// warp.
// ---------------------------------------------------------------------------

template <int NN, int ME>
__device__ __noinline__ int svd_warp_tiny(double* W, int mm, int nn, double* tau, int* piv_s, double* Ut, double* Vt,
                                          double* Sout, int max_sweeps) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int LPC = 32 / NN;                   // lanes per column
  static_assert(ME * LPC <= 64 && ME >= 1, "rows per lane");   // this lane: rows part + LPC*e, e < ME (mm <= ME*LPC)
  constexpr int XE = NN >= LPC ? NN / LPC : 1;   // rows of X per lane
  constexpr int RP = NN < LPC ? NN : LPC;        // parts holding rows of X
  const int lane = threadIdx.x & 31;
  const int col = lane & (NN - 1), part = lane / NN;
  const bool ocol = col < nn;
  // ---- pivoted Householder QR, this lane's rows i = part + LPC*e of column col
  double a[ME];
#pragma unroll
  for (int e = 0; e < ME; ++e) {
    const int i = part + LPC * e;
    a[e] = (ocol && i < mm) ? W[i + col * mm] : 0.0;
  }
  // nrm: squared norm of the rows >= k, lo: of the rows > k (k = 0 here)
  double nrm = 0.0, lo = 0.0;
#pragma unroll
  for (int e = 0; e < ME; ++e) {
    const double t = a[e] * a[e];
    nrm += t;
    if (part + LPC * e > 0) lo += t;
  }
#pragma unroll
  for (int o = NN; o < 32; o <<= 1) {
    nrm += __shfl_xor_sync(FULL, nrm, o);
    lo += __shfl_xor_sync(FULL, lo, o);
  }
  int cur = col;   // position of this column in the pivoted order
  double tau_k = 0.0;   // lane k keeps tau[k]
  for (int k = 0; k < nn; ++k) {
    // pivot: largest remaining norm, smallest position on ties (a total
    // order, NaN below every number, so every lane reaches the same answer)
    const bool cand = ocol && cur >= k;
    double bv = cand ? (nrm == nrm ? nrm : -0.5) : -1.0;
    int bc = cand ? (cur << 8) | col : (64 << 8);
#pragma unroll
    for (int o = 1; o < NN; o <<= 1) {
      const double ov = __shfl_xor_sync(FULL, bv, o);
      const int oc = __shfl_xor_sync(FULL, bc, o);
      if (ov > bv || (ov == bv && oc < bc)) { bv = ov; bc = oc; }
    }
    const int pc = bc >> 8;
    if (ocol && pc != k && pc < nn) {
      if (cur == pc) cur = k;
      else if (cur == k) cur = pc;
    }
    const int gk = pc < nn ? (bc & 255) : 0;   // lane of the column now at position k
    // (pc >= nn cannot happen for k < nn: some column is always a candidate)
    double mine = 0.0;
#pragma unroll
    for (int e = 0; e < ME; ++e)
      if (part + LPC * e == k) mine = a[e];
    const double loc = __shfl_sync(FULL, lo, gk);
    const double alpha = __shfl_sync(FULL, mine, gk + NN * (k & (LPC - 1)));
    double tk = 0.0;
    if (loc > 0.0) {
      // |beta| = sqrt(alpha^2 + loc), beta = -sign(alpha) |beta|,
      // tau = (beta - alpha) / beta = 1 + |alpha| / |beta|, scale = 1 / (alpha - beta)
      const double q = fma(alpha, alpha, loc);
      const double rq = rsqrt(q);
      const double nb = q * rq;
      const double beta = alpha < 0.0 ? nb : -nb;
      tk = fma(fabs(alpha), rq, 1.0);
      const double sc = 1.0 / (alpha - beta);
      if (ocol && cur == k) {
#pragma unroll
        for (int e = 0; e < ME; ++e) {
          const int i = part + LPC * e;
          if (i > k) a[e] *= sc;
          else if (i == k) a[e] = beta;
        }
      }
    }
    if (lane == k) tau_k = tk;
    const bool act = ocol && cur > k;
    if (tk != 0.0) {
      double vk[ME];
#pragma unroll
      for (int e = 0; e < ME; ++e) vk[e] = 0.0;
      double w = 0.0;
      double w2 = 0.0;
#pragma unroll
      for (int e = 0; e < ME; ++e) {
        const int i = part + LPC * e;
        const double t = __shfl_sync(FULL, a[e], gk + NN * part);
        vk[e] = i > k ? t : (i == k ? 1.0 : 0.0);
        if (e & 1) w2 = fma(vk[e], a[e], w2);
        else w = fma(vk[e], a[e], w);
      }
      w += w2;
#pragma unroll
      for (int o = NN; o < 32; o <<= 1) w += __shfl_xor_sync(FULL, w, o);
      if (act) {
        w *= tk;
#pragma unroll
        for (int e = 0; e < ME; ++e) {
          a[e] = fma(-w, vk[e], a[e]);
        }
      }
    }
    // squared norms of the rows > k and > k+1 of the remaining columns
    double sn = 0.0, sl = 0.0;
#pragma unroll
    for (int e = 0; e < ME; ++e) {
      const int i = part + LPC * e;
      const double t = a[e] * a[e];
      if (i > k) sn += t;
      if (i > k + 1) sl += t;
    }
#pragma unroll
    for (int o = NN; o < 32; o <<= 1) {
      sn += __shfl_xor_sync(FULL, sn, o);
      sl += __shfl_xor_sync(FULL, sl, o);
    }
    if (act) { nrm = sn; lo = sl; }
  }
  // Householder form into W (column order of the pivoted matrix), pivots
#pragma unroll
  for (int e = 0; e < ME; ++e) {
    const int i = part + LPC * e;
    if (ocol && i < mm) W[i + cur * mm] = a[e];
  }
  if (ocol && part == 0) piv_s[cur] = col;
  if (lane < nn) tau[lane] = tau_k;
  __syncwarp();
  // ---- one-sided Jacobi on X = R^T; lane holds rows i = part + LPC*e of column col
  double x[XE], v[XE];
#pragma unroll
  for (int e = 0; e < XE; ++e) {
    const int i = part + LPC * e;
    x[e] = (ocol && i < nn && i >= col) ? W[col + i * mm] : 0.0;
    v[e] = (i == col) ? 1.0 : 0.0;
  }
  double mx = 0.0;
#pragma unroll
  for (int e = 0; e < XE; ++e) mx = fmax(mx, fabs(x[e]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
  const double sc = mx > 0.0 ? 1.0 / mx : 1.0;
#pragma unroll
  for (int e = 0; e < XE; ++e) x[e] *= sc;
  const double tol = 2.220446049250313e-16 * 16.0;
  int result = -1;
  for (int sweep = 0; sweep < max_sweeps && nn > 1; ++sweep) {
    int rotated = 0;
    // round m pairs column j with j ^ m: every pair once per sweep
    for (int m = 1; m < NN; ++m) {
      int partner = col ^ m;
      if (!ocol || partner >= nn) partner = -1;
      const int src = partner >= 0 ? partner + NN * part : lane;
      double px[XE];
      double ao = 0.0, ap = 0.0, g = 0.0;
#pragma unroll
      for (int e = 0; e < XE; ++e) {
        px[e] = __shfl_sync(FULL, x[e], src);
        ao = fma(x[e], x[e], ao);
        ap = fma(px[e], px[e], ap);
        g = fma(x[e], px[e], g);
      }
#pragma unroll
      for (int o = NN; o < NN * RP; o <<= 1) {
        ao += __shfl_xor_sync(FULL, ao, o);
        ap += __shfl_xor_sync(FULL, ap, o);
        g += __shfl_xor_sync(FULL, g, o);
      }
      bool doit = false, low = false;
      double c = 1.0, s = 0.0;
      if (partner >= 0) {
        low = col < partner;
        if (jacobi_rotation(low ? ao : ap, low ? ap : ao, g, tol, &c, &s)) {
          doit = true;
          rotated = 1;
        }
      }
      if (__any_sync(FULL, doit)) {
        const double sl = low ? -s : s;
#pragma unroll
        for (int e = 0; e < XE; ++e) {
          const double pv = __shfl_sync(FULL, v[e], src);
          if (doit) {
            x[e] = fma(sl, px[e], c * x[e]);
            v[e] = fma(sl, pv, c * v[e]);
          }
        }
      }
    }
    if (!__any_sync(FULL, rotated)) {
      result = sweep + 1;
      break;
    }
  }
  if (nn <= 1) result = 0;
  // singular values, descending order
  double sg = 0.0;
#pragma unroll
  for (int e = 0; e < XE; ++e) sg = fma(x[e], x[e], sg);
#pragma unroll
  for (int o = NN; o < NN * RP; o <<= 1) sg += __shfl_xor_sync(FULL, sg, o);
  sg = __shfl_sync(FULL, ocol ? sqrt(sg) / sc : -1.0, col);   // lanes outside the RP parts take part 0's
  int rank = 0;
  for (int l = 0; l < nn; ++l) {
    const double sl = __shfl_sync(FULL, sg, l);
    rank += (sl > sg || (sl == sg && l < col)) ? 1 : 0;
  }
  if (ocol) {
    if (part == 0) Sout[rank] = sg;
#pragma unroll
    for (int e = 0; e < XE; ++e) {
      const int i = part + LPC * e;
      if (i < nn) Vt[piv_s[i] + rank * nn] = (sg > 0.0) ? (x[e] / sc) / sg : 0.0;
    }
  }
  // Ut[:, rank] = Q [v; 0], reflectors from W
  double u[ME];
#pragma unroll
  for (int e = 0; e < ME; ++e) u[e] = 0.0;
#pragma unroll
  for (int e = 0; e < XE; ++e) u[e] = v[e];
  for (int k = nn - 1; k >= 0; --k) {
    const double tk = tau[k];
    if (tk != 0.0) {
      double vk[ME];
#pragma unroll
      for (int e = 0; e < ME; ++e) vk[e] = 0.0;
      double w = 0.0, w2 = 0.0;
#pragma unroll
      for (int e = 0; e < ME; ++e) {
        const int i = part + LPC * e;
        vk[e] = i > k ? (i < mm ? W[i + k * mm] : 0.0) : (i == k ? 1.0 : 0.0);
        if (e & 1) w2 = fma(vk[e], u[e], w2);
        else w = fma(vk[e], u[e], w);
      }
      w += w2;
#pragma unroll
      for (int o = NN; o < 32; o <<= 1) w += __shfl_xor_sync(FULL, w, o);
      w *= tk;
#pragma unroll
      for (int e = 0; e < ME; ++e) {
        u[e] = fma(-w, vk[e], u[e]);
      }
    }
  }
  if (ocol) {
#pragma unroll
    for (int e = 0; e < ME; ++e) {
      const int i = part + LPC * e;
      if (i < mm) Ut[i + rank * mm] = u[e];
    }
  }
  __syncwarp();
  return result;
}

// Dispatch on the column count (NN = next power of two) and the rows per lane.
__device__ __forceinline__ int svd_warp_tiny_any(double* W, int mm, int nn, double* tau, int* piv, double* Ut,
                                                 double* Vt, double* S, int max_sweeps) {
  if (nn <= 2)
    return mm <= 16 ? svd_warp_tiny<2, 1>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps)
                    : svd_warp_tiny<2, 4>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps);
  if (nn <= 4)
    return mm <= 8    ? svd_warp_tiny<4, 1>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps)
           : mm <= 16 ? svd_warp_tiny<4, 2>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps)
                      : svd_warp_tiny<4, 8>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps);
  if (nn <= 8)
    return mm <= 16 ? svd_warp_tiny<8, 4>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps)
                    : svd_warp_tiny<8, 16>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps);
  return mm <= 32 ? svd_warp_tiny<16, 16>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps)
                  : svd_warp_tiny<16, 32>(W, mm, nn, tau, piv, Ut, Vt, S, max_sweeps);
}
#endif

}  // namespace catn
