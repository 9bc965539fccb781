// Trailing update of the blocked Householder QR (qr_sorted_blocked in
// blockjac.cuh): one item applies a panel's reflectors, in compact WY form
// Q = H_k0 ... H_k0+kb-1 = I - V T V^T (Nm = -T), as Q^T to a tile of 32
// trailing columns,
//     C <- Q^T C = C + V (Nm^T (V^T C)),
// and records the squared norms of the updated columns below the panel (the
// next panels' stop test).  V (mp x kb, unit lower trapezoidal, ld mp) and Nm
// (kb x kb, ld kb) are in global memory, written by the owner; C is the
// matrix from the panel's first row on.  Items are claimed by whole CTAs
// through the shared job (JOB_PANEL) like the block Jacobi's pairs.
#pragma once
#include "linalg.cuh"

namespace catn {

constexpr int kPanelW = 32;   // reflectors per panel and columns per trailing item

// Y (kb x 32, row-major, zero past kb) = V^T C_tile over rows [0, mp).
CATN_HDI inline void panel_cross_gram(const Team& T, const double* V, long long mp, int kb, const double* Cm,
                                      long long ldc, const long long* cols, double* Y, double* part, double* S2) {
#if CATN_DEVICE_PASS
  double* S1 = (double*)T.stage;   // [32][65]: V rows staged
  const int tid = T.rank();
  const int grp = tid >> 6, tt = tid & 63;
  const int i0 = (tt & 7) * 4, j0 = (tt >> 3) * 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (long long r0 = 0; r0 < mp; r0 += 64) {
    for (int e = tid; e < kPanelW * 64; e += 256) {
      const int c = e >> 6, r = e & 63;
      const bool in = r0 + r < mp;
      S1[c * 65 + r] = (in && c < kb) ? ldcg(V + (r0 + r) + c * mp) : 0.0;
      S2[c * 65 + r] = (in && cols[c] >= 0) ? ldcg(Cm + (r0 + r) + cols[c] * ldc) : 0.0;
    }
    __syncthreads();
    for (int r = grp; r < 64; r += 4) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = S1[(i0 + q) * 65 + r];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = S2[(j0 + q) * 65 + r];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  constexpr int KK = kPanelW * kPanelW;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) part[grp * KK + (i0 + x) * kPanelW + (j0 + y)] = acc[x][y];
  __syncthreads();
  for (int e = tid; e < KK; e += 256) Y[e] = (part[e] + part[KK + e]) + (part[2 * KK + e] + part[3 * KK + e]);
  __syncthreads();
#else
  (void)part; (void)S2;
  for (int i = 0; i < kPanelW; ++i)
    for (int j = 0; j < kPanelW; ++j) {
      double s = 0.0;
      if (i < kb && cols[j] >= 0)
        for (long long r = 0; r < mp; ++r) s = fma(V[r + i * mp], Cm[r + cols[j] * ldc], s);
      Y[i * kPanelW + j] = s;
    }
#endif
}

// One trailing item: the 32 columns cols[] (-1: absent) of C (mp rows).
// ws holds 4 K + 2 K + 2080 + 64 doubles (K = 32 x 32).
CATN_HDI inline void panel_item(const Team& T, double* Cm, long long mp, long long ldc, const double* V,
                                const double* Nm, int kb, const long long* cols, double* nrm, double* ws) {
  constexpr int K = kPanelW;
  double* Y = ws;
  double* Y2 = Y + K * K;
  double* part = Y2 + K * K;
  double* S2 = part + 4 * K * K;
  double* nsq = S2 + K * 65;   // [8 warps][32] partial squared norms
  panel_cross_gram(T, V, mp, kb, Cm, ldc, cols, Y, part, S2);
  // Y2 = Nm^T Y (Nm kb x kb, column-major, ld kb; global): the factorisation
  // applies the panel's reflectors H_0 first, i.e. Q^T = I - V T^T V^T
  for (int e = T.rank(); e < K * K; e += T.size()) {
    const int i = e / K, j = e - i * K;
    double s = 0.0;
    if (i < kb)
      for (int l = 0; l < kb; ++l) s = fma(ldcg(Nm + l + (long long)i * kb), Y[l * K + j], s);
    Y2[e] = s;
  }
  T.sync();
  // C += V Y2, row by row, in two halves of 16 columns; squared norms of
  // the updated rows below the panel (local rows >= kb)
  for (int h = 0; h < 2; ++h) {
    double loc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) loc[j] = 0.0;
    for (long long r = T.rank(); r < mp; r += T.size()) {
      double v[K];
#pragma unroll
      for (int i = 0; i < K; ++i) v[i] = (i < kb) ? ldcg(V + r + (long long)i * mp) : 0.0;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int c = 16 * h + j;
        if (cols[c] < 0) continue;
        double* p = Cm + r + cols[c] * ldc;
        double x = ldcg(p);
#pragma unroll
        for (int i = 0; i < K; ++i) x = fma(v[i], Y2[i * K + c], x);
        stcg(p, x);
        if (r >= kb) loc[j] = fma(x, x, loc[j]);
      }
    }
#if CATN_DEVICE_PASS
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double s = T.wsum(loc[j]);
      if (T.lane() == 0) nsq[T.warp() * 16 + j] = s;
    }
    T.sync();
    if (T.rank() < 16) {
      double s = 0.0;
      for (int w = 0; w < T.nwarps(); ++w) s += nsq[w * 16 + T.rank()];
      const long long col = cols[16 * h + T.rank()];
      if (col >= 0) stcg(nrm + col, s);
    }
    T.sync();
#else
    (void)nsq;
    for (int j = 0; j < 16; ++j)
      if (cols[16 * h + j] >= 0) nrm[cols[16 * h + j]] = loc[j];
#endif
  }
  T.sync();
}

// Workspace (doubles) of panel_item.
constexpr int kPanelWsDoubles = 6 * kPanelW * kPanelW + kPanelW * 65 + 8 * 16 + 64;

}  // namespace catn
