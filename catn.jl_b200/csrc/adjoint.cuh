// Adjoint of contraction! (reverse mode over the tape of one gradient run).
//
// A gradient run contracts the network exactly as a plain run does, with the
// site heap append-only and every site-writing operation recorded (engine.cuh,
// TapeRec).  backward() then walks the records last to first and accumulates
// d lnZ / d(site version) into the shadow heap; the gradients of the sites
// loaded from the input image are the result, in the image's own layout, and
// the host maps them to d lnZ / d w and d lnZ / d h (host_image.h).
//
// Every SVD on the path splits a matrix across one bond, A ~ Q diag(S) P^T
// (k kept values), and everything downstream of the split is invariant under
// an orthogonal change of basis on that bond (the contraction value does not
// see it, and lnZ is the log of that value).  With that invariance the
// 1/(s_j^2 - s_i^2) terms of the general SVD adjoint cancel exactly, leaving
//   orthonormal Q, loaded factor P S:   Abar = Q (P S)bar^T + (I - Q Q^T) Qbar S^-1 P^T
//   balanced split Q S^1/2, P S^1/2 (the bond cut): X_ij = (Gi_ij s_j + Gj_ji s_i)
//     / ((s_i + s_j) sqrt(s_i s_j)) in place of the F-term matrix,
// which stay finite for degenerate singular values.  Kept values below
// 1e-10 s_1 (noise kept by the absolute cutoff: their directions enter the
// outputs with weight s or sqrt(s) but their singular vectors are rounding)
// are treated like the discarded ones, as exactly zero, which is the usual
// tensor-network practice for the truncated part.
#pragma once
#include "engine.cuh"

namespace catn {

// Re-carve the arena for a gradient run: scratch 20 %, tape records 4 %,
// then the append-only heap and its shadow (38 % each).  Call after make_ctx
// and before load_instance.
CATN_HDI inline void tape_enable(Ctx& C, long long arena_bytes) {
  const long long cap = arena_bytes & ~255LL;
  const long long sc = (cap / 5) & ~255LL;
  const long long rb = (cap / 25) & ~255LL;
  const long long H = ((cap - sc - rb) / 2) & ~255LL;
  C.sp_lo = 0;
  C.sp = 0;
  C.sp_hi = sc;
  C.sp_peak = 0;
  C.rec = (TapeRec*)(C.base + sc);
  C.rcap = rb / (long long)sizeof(TapeRec);
  C.nrec = 0;
  C.h_lo0 = C.h_lo1 = sc + rb;
  C.hsize = H;
  C.half = 0;
  C.hb = C.h_lo0;
  C.he = C.h_lo0 + H;
  C.h_peak = 0;
  C.gshift = H;
  C.tape = 1;
}

CATN_HD double* gptr(const Ctx& C, long long off) { return (double*)(C.base + off + C.gshift); }
// Transposed view of an operand.
CATN_HD MOp tview(const MOp& a) { return mop(a.p, a.C, a.R, a.cs, a.rs); }

// 1/s and 1/sqrt(s) over the kept values, zero below 1e-10 s_1.
CATN_HDI inline void inv_kept(const Team& T, long long k, const double* S, double* inv, double* isq) {
  double s1 = 0.0;
  for (long long e = T.rank(); e < k; e += T.size()) s1 = fmax(s1, fabs(S[e]));
  s1 = T.maxv(s1);
  const double thr = 1e-10 * s1;
  for (long long e = T.rank(); e < k; e += T.size()) {
    const bool live = S[e] > thr && S[e] > 0.0;
    inv[e] = live ? 1.0 / S[e] : 0.0;
    if (isq) isq[e] = live ? 1.0 / sqrt(S[e]) : 0.0;
  }
  T.sync();
}

// A (rows x cols) ~ Q diag(S) P^T with Q orthonormal (rows x k); given
// Qb = dL/dQ (rows x k, plain) and Plb = dL/d(P S) (cols x k):
//   Abar (+)= Q Plb^T + (Qb - Q (Q^T Qb)) S^-1 P^T.
CATN_HDI inline void split_bwd(Ctx& C, long long rows, long long cols, long long k, const MOp& Q, const double* S,
                               const MOp& P, const double* Qb, const MOp& Plb, const MOp& Aout, bool accum) {
  const Team& T = C.T;
  double* J = spush(C, k * k);
  double* inv = spush(C, k);
  double* Y = spush(C, rows * k);
  if (failed(C)) return;
  inv_kept(T, k, S, inv, nullptr);
  gemm(T, k, k, rows, tview(Q), colmajor((double*)Qb, rows), colmajor(J, k));
  gemm(T, rows, k, k, Q, colmajor(J, k), colmajor(Y, rows));
  for (long long e = T.rank(); e < rows * k; e += T.size()) {
    long long r, i;
    divmod(e, rows, &r, &i);
    Y[e] = (Qb[e] - Y[e]) * inv[i];
  }
  T.sync();
  gemm(T, rows, cols, k, Q, tview(Plb), Aout, accum);
  gemm(T, rows, cols, k, colmajor(Y, rows), tview(P), Aout, true);
}

// ---------------------------------------------------------------------------
// one backward routine per record type
// ---------------------------------------------------------------------------
// cano_to! right step: site (m x n) = U diag(S) V^T; new site = U[:, 1:k]
// (orthonormal); new next = R * next with R = (S V^T)[1:k, :].
CATN_HDI inline void bwd_cano_r(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long m = (long long)r.a[0] * r.a[1], n = r.a[2], k = r.a[3], N2 = (long long)r.a[4] * r.a[5];
  const double* S = dptr(C, r.o[4]);
  double* Vp = dptr(C, r.o[5]);
  double* Gn = gptr(C, r.o[3]);
  double* Rb = spush(C, k * n);
  if (failed(C)) return;
  gemm(T, k, n, N2, colmajor(Gn, k), transposed(dptr(C, r.o[1]), n), colmajor(Rb, k));   // Rbar = Gn next^T
  gemm(T, n, N2, k, mop(Vp, rows_plain(), cols_plain(n), nullptr, S), colmajor(Gn, k), colmajor(gptr(C, r.o[1]), n),
       true);                                                                                // next_bar += R^T Gn
  split_bwd(C, m, n, k, colmajor(dptr(C, r.o[2]), m), S, colmajor(Vp, n), gptr(C, r.o[2]), transposed(Rb, k),
            colmajor(gptr(C, r.o[0]), m), true);
}

// cano_to! left step: Mt = site^T ((d dr) x dl) = U diag(S) V^T; new site =
// U[:, 1:k]^T (orthonormal); new prev = prev * (V S)[:, 1:k].
CATN_HDI inline void bwd_cano_l(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long dl = r.a[0], m = (long long)r.a[1] * r.a[2], k = r.a[3], P = (long long)r.a[4] * r.a[5];
  const double* S = dptr(C, r.o[4]);
  double* Vp = dptr(C, r.o[5]);
  double* Gp = gptr(C, r.o[3]);
  double* Bb = spush(C, dl * k);
  double* Ub = spush(C, m * k);
  if (failed(C)) return;
  gemm(T, dl, k, P, transposed(dptr(C, r.o[1]), P), colmajor(Gp, P), colmajor(Bb, dl));   // (V S)bar = prev^T Gp
  gemm(T, P, dl, k, colmajor(Gp, P), mop(Vp, cols_plain(dl), rows_plain(), S, nullptr),
       colmajor(gptr(C, r.o[1]), P), true);                                                 // prev_bar += Gp (V S)^T
  materialize(T, Ub, m, k, m, transposed(gptr(C, r.o[2]), k));
  split_bwd(C, m, dl, k, transposed(dptr(C, r.o[2]), k), S, colmajor(Vp, dl), Ub, colmajor(Bb, dl),
            transposed(gptr(C, r.o[0]), dl), true);
}

// swap!: W = ein"ijk,kab->iajb"(tl, tr), M = reshape(W, d0 d1, d2 d3)
// = U diag(S) V^T; i < j: lo = U, hi = S V^T; i > j: lo = U S, hi = V^T.
CATN_HDI inline void bwd_swap(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long d0 = r.a[0], d1 = r.a[1], d2 = r.a[2], d3 = r.a[3], kk = r.a[4], k = r.a[5];
  const long long m = d0 * d1, n = d2 * d3;
  const double* S = dptr(C, r.o[4]);
  double* Mb = spush(C, m * n);
  if (failed(C)) return;
  if (r.a[6]) {
    // Q = U (lo), loaded factor V S = hi^T
    split_bwd(C, m, n, k, colmajor(dptr(C, r.o[2]), m), S, colmajor(dptr(C, r.o[5]), n), gptr(C, r.o[2]),
              transposed(gptr(C, r.o[3]), k), colmajor(Mb, m), false);
  } else {
    // transposed problem M^T = V diag(S) U^T: Q = V = hi^T, loaded factor U S = lo
    double* Vb = spush(C, n * k);
    if (failed(C)) return;
    materialize(T, Vb, n, k, n, transposed(gptr(C, r.o[3]), k));
    split_bwd(C, n, m, k, transposed(dptr(C, r.o[3]), k), S, colmajor(dptr(C, r.o[5]), m), Vb,
              colmajor(gptr(C, r.o[2]), m), transposed(Mb, m), false);
  }
  // Mbar seen with rows (i + d0 j) and columns (a + d1 b)
  const MOp Mx = mop(Mb, imap((int)d0, 1, m), imap((int)d1, d0, m * d2));
  gemm(T, d0 * d2, kk, d1 * d3, Mx, mop(dptr(C, r.o[1]), imap(1, 0, kk), rows_plain()),
       colmajor(gptr(C, r.o[0]), d0 * d2), true);
  gemm(T, kk, d1 * d3, d0 * d2, mop(dptr(C, r.o[0]), imap(1, 0, d0 * d2), rows_plain()), Mx,
       colmajor(gptr(C, r.o[1]), kk), true);
}

// reverse!: new[c + dr (b + d a)] = old[a + dl (b + d c)].
CATN_HDI inline void bwd_reverse(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long dl = r.a[0], d = r.a[1], dr = r.a[2], tot = dl * d * dr;
  double* go = gptr(C, r.o[0]);
  const double* gn = gptr(C, r.o[1]);
  for (long long e = T.rank(); e < tot; e += T.size()) {
    long long a, rest, b, c;
    divmod(e, dl, &a, &rest);
    divmod(rest, d, &b, &c);
    go[e] += gn[c + dr * (b + d * a)];
  }
  T.sync();
}

// merge!: fused (dl da x db dr) = a (dl da x k) * b (k x db dr).
CATN_HDI inline void bwd_merge(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long rows = (long long)r.a[0] * r.a[1], k = r.a[2], cols = (long long)r.a[3] * r.a[4];
  const double* gf = gptr(C, r.o[2]);
  gemm(T, rows, k, cols, colmajor((double*)gf, rows), transposed(dptr(C, r.o[1]), k), colmajor(gptr(C, r.o[0]), rows),
       true);
  gemm(T, k, cols, rows, transposed(dptr(C, r.o[0]), rows), colmajor((double*)gf, rows),
       colmajor(gptr(C, r.o[1]), k), true);
}

// eat! (a): lnZ += log|vi . vj|.
CATN_HDI inline void bwd_eat_a(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  if (!r.flag) return;
  const long long d = r.a[0];
  const double* vi = dptr(C, r.o[0]);
  const double* vj = dptr(C, r.o[1]);
  double* gi = gptr(C, r.o[0]);
  double* gj = gptr(C, r.o[1]);
  const double rinv = 1.0 / r.v[0];
  for (long long e = T.rank(); e < d; e += T.size()) {
    gi[e] += vj[e] * rinv;
    gj[e] += vi[e] * rinv;
  }
  T.sync();
}

// eat! (b): new = prev * (last * tj).
CATN_HDI inline void bwd_eat_b(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long Dl = r.a[0], dd = r.a[1], ne = r.a[2];
  double* last = dptr(C, r.o[0]);
  double* tj = dptr(C, r.o[1]);
  double* prev = dptr(C, r.o[2]);
  double* gn = gptr(C, r.o[3]);
  double* v = spush(C, Dl);
  double* vb = spush(C, Dl);
  if (failed(C)) return;
  gemm(T, Dl, 1, dd, colmajor(last, Dl), colmajor(tj, dd), colmajor(v, Dl));
  gemm(T, ne, Dl, 1, colmajor(gn, ne), transposed(v, 1), colmajor(gptr(C, r.o[2]), ne), true);
  gemm(T, Dl, 1, ne, transposed(prev, ne), colmajor(gn, ne), colmajor(vb, Dl));
  gemm(T, Dl, dd, 1, colmajor(vb, Dl), transposed(tj, 1), colmajor(gptr(C, r.o[0]), Dl), true);
  gemm(T, dd, 1, Dl, transposed(last, Dl), colmajor(vb, Dl), colmajor(gptr(C, r.o[1]), dd), true);
}

// eat! (c): new = prev * (last * hj).
CATN_HDI inline void bwd_eat_c(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long Dl = r.a[0], dd = r.a[1], Dr = r.a[2], pr = r.a[3];
  double* last = dptr(C, r.o[0]);
  double* hj = dptr(C, r.o[1]);
  double* prev = dptr(C, r.o[2]);
  double* gn = gptr(C, r.o[3]);
  double* mat = spush(C, Dl * Dr);
  double* mb = spush(C, Dl * Dr);
  if (failed(C)) return;
  gemm(T, Dl, Dr, dd, colmajor(last, Dl), colmajor(hj, dd), colmajor(mat, Dl));
  gemm(T, pr, Dl, Dr, colmajor(gn, pr), transposed(mat, Dl), colmajor(gptr(C, r.o[2]), pr), true);
  gemm(T, Dl, Dr, pr, transposed(prev, pr), colmajor(gn, pr), colmajor(mb, Dl));
  gemm(T, Dl, dd, Dr, colmajor(mb, Dl), transposed(hj, dd), colmajor(gptr(C, r.o[0]), Dl), true);
  gemm(T, dd, Dr, Dl, transposed(last, Dl), colmajor(mb, Dl), colmajor(gptr(C, r.o[1]), dd), true);
}

// Division by the norm: y = x / nrm(x), lnZ += log nrm(x).
CATN_HDI inline void bwd_norm(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long len = r.a[0];
  const double nrm = r.v[0], inv = 1.0 / nrm;
  const double* x = dptr(C, r.o[0]);
  const double* y = dptr(C, r.o[1]);
  const double* gy = gptr(C, r.o[1]);
  double* gx = gptr(C, r.o[0]);
  double c = 0.0;
  for (long long e = T.rank(); e < len; e += T.size()) c = fma(y[e], gy[e], c);
  c = T.sum(c);
  if (r.a[1] == 1) {   // 2-norm: d nrm / dx = y
    for (long long e = T.rank(); e < len; e += T.size()) gx[e] += (gy[e] + (1.0 - c) * y[e]) * inv;
    T.sync();
    return;
  }
  // max-abs norm: d nrm / dx = sign(x_m) e_m at the first largest |x_m|
  double best = -1.0;
  long long bi = -1;
  for (long long e = T.rank(); e < len; e += T.size())
    if (fabs(x[e]) > best) { best = fabs(x[e]); bi = e; }
  bi = T.argmax(best, bi);
  for (long long e = T.rank(); e < len; e += T.size()) gx[e] += gy[e] * inv;
  T.sync();
  if (T.leader() && bi >= 0) gx[bi] += (1.0 - c) * (x[bi] < 0.0 ? -1.0 : 1.0) * inv;
  T.sync();
}

// cut_bondim_opt!: P = mati matj^T ~ Uf diag(S) Vf^T (k = myd kept), new Ai
// from Fi = Uf sqrt(S), new Aj from Fj = Vf sqrt(S).  With Gi = Fi^T Fi_bar
// and Gj = Fj^T Fj_bar (k x k), the adjoint of P is
//   Pbar = Uf X Vf^T + (Ubar - Uf J) S^-1 Vf^T + Uf S^-1 (Vbar - Vf K)^T,
//   X_ij = (Gi_ij s_j + Gj_ji s_i) / ((s_i + s_j) sqrt(s_i s_j)),
//   Ubar = Fi_bar sqrt(S), J = Uf^T Ubar, Vbar and K alike,
// applied to mati and matj in factored form (P itself is never formed).
CATN_HDI inline void bwd_cut(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  const long long dl = r.a[0], d = r.a[1], dr = r.a[2], dl2 = r.a[3], dr2 = r.a[4], k = r.a[5];
  const long long da = dl * dr, db = dl2 * dr2;
  const double* S = dptr(C, r.o[4]);
  double* inv = spush(C, k);
  double* isq = spush(C, k);
  double* Gi = spush(C, k * k);
  double* Gj = spush(C, k * k);
  double* J = spush(C, k * k);
  double* K = spush(C, k * k);
  double* X = spush(C, k * k);
  double* Zi = spush(C, da * k);
  double* Zj = spush(C, db * k);
  double* Bi = spush(C, k * d);
  double* Bj = spush(C, k * d);
  double* Q = spush(C, k * d);
  if (failed(C)) return;
  inv_kept(T, k, S, inv, isq);
  const MOp mati = mop(dptr(C, r.o[0]), imap((int)dl, 1, dl * d), cols_plain(dl));
  const MOp matj = mop(dptr(C, r.o[1]), imap((int)dl2, 1, dl2 * d), cols_plain(dl2));
  const MOp gmati = mop(gptr(C, r.o[0]), imap((int)dl, 1, dl * d), cols_plain(dl));
  const MOp gmatj = mop(gptr(C, r.o[1]), imap((int)dl2, 1, dl2 * d), cols_plain(dl2));
  const MOp Fi = mop(dptr(C, r.o[2]), imap((int)dl, 1, dl * k), cols_plain(dl));
  const MOp Fj = mop(dptr(C, r.o[3]), imap((int)dl2, 1, dl2 * k), cols_plain(dl2));
  const MOp Fib = mop(gptr(C, r.o[2]), imap((int)dl, 1, dl * k), cols_plain(dl));
  const MOp Fjb = mop(gptr(C, r.o[3]), imap((int)dl2, 1, dl2 * k), cols_plain(dl2));
  const MOp Uf = mop(Fi.p, Fi.R, Fi.C, nullptr, isq);
  const MOp Vf = mop(Fj.p, Fj.R, Fj.C, nullptr, isq);
  gemm(T, k, k, da, tview(Fi), Fib, colmajor(Gi, k));
  gemm(T, k, k, db, tview(Fj), Fjb, colmajor(Gj, k));
  for (long long e = T.rank(); e < k * k; e += T.size()) {
    long long i, j;
    divmod(e, k, &i, &j);
    const double si = S[i], sj = S[j];
    // J = Uf^T Ubar = S^-1/2 Gi S^1/2, K = S^-1/2 Gj S^1/2
    J[e] = Gi[e] * isq[i] * sqrt(sj);
    K[e] = Gj[e] * isq[i] * sqrt(sj);
    // (Gi_ij s_j + Gj_ji s_i) / ((s_i + s_j) sqrt(s_i s_j)), zero for noise-level values
    X[e] = (isq[i] > 0.0 && isq[j] > 0.0) ? (Gi[e] * sj + Gj[j + k * i] * si) * isq[i] * isq[j] / (si + sj) : 0.0;
  }
  T.sync();
  // Zi = Ubar - Uf J, Zj = Vbar - Vf K
  gemm(T, da, k, k, Uf, colmajor(J, k), colmajor(Zi, da));
  gemm(T, db, k, k, Vf, colmajor(K, k), colmajor(Zj, db));
  for (long long e = T.rank(); e < da * k; e += T.size()) {
    long long x, i;
    divmod(e, da, &x, &i);
    Zi[e] = Fib.ld(x, i) * sqrt(S[i]) - Zi[e];
  }
  for (long long e = T.rank(); e < db * k; e += T.size()) {
    long long x, i;
    divmod(e, db, &x, &i);
    Zj[e] = Fjb.ld(x, i) * sqrt(S[i]) - Zj[e];
  }
  T.sync();
  gemm(T, k, d, da, tview(Uf), mati, colmajor(Bi, k));   // Bi = Uf^T mati
  gemm(T, k, d, db, tview(Vf), matj, colmajor(Bj, k));   // Bj = Vf^T matj
  // mati_bar += Uf (X Bj + inv Zj^T matj) + (Zi inv) Bj
  gemm(T, k, d, k, colmajor(X, k), colmajor(Bj, k), colmajor(Q, k));
  gemm(T, k, d, db, mop(Zj, cols_plain(db), rows_plain(), inv, nullptr), matj, colmajor(Q, k), true);
  gemm(T, da, d, k, Uf, colmajor(Q, k), gmati, true);
  gemm(T, da, d, k, mop(Zi, rows_plain(), cols_plain(da), nullptr, inv), colmajor(Bj, k), gmati, true);
  // matj_bar += Vf (X^T Bi + inv Zi^T mati) + (Zj inv) Bi
  gemm(T, k, d, k, transposed(X, k), colmajor(Bi, k), colmajor(Q, k));
  gemm(T, k, d, da, mop(Zi, cols_plain(da), rows_plain(), inv, nullptr), mati, colmajor(Q, k), true);
  gemm(T, db, d, k, Vf, colmajor(Q, k), gmatj, true);
  gemm(T, db, d, k, mop(Zj, rows_plain(), cols_plain(db), nullptr, inv), colmajor(Bi, k), gmatj, true);
}

// network_lognorm: lnZ += log|sum(x)|.
CATN_HDI inline void bwd_logz(Ctx& C, const TapeRec& r) {
  const Team& T = C.T;
  double* g = gptr(C, r.o[0]);
  const double zi = 1.0 / r.v[0];
  for (long long e = T.rank(); e < r.a[0]; e += T.size()) g[e] += zi;
  T.sync();
}

// Zero the shadow of every heap byte written so far.
CATN_HDI inline void shadow_zero(Ctx& C) {
  const Team& T = C.T;
  double* g = gptr(C, C.h_lo0);
  const long long len = (C.hb - C.h_lo0) / 8;
  for (long long e = T.rank(); e < len; e += T.size()) g[e] = 0.0;
  T.sync();
}

// Walk the records last to first, accumulating into the shadow heap.
CATN_HDI inline void backward_walk(Ctx& C) {
  for (long long q = C.nrec - 1; q >= 0 && !failed(C); --q) {
    const TapeRec r = C.rec[q];
    const long long mark = C.sp;
    switch (r.op) {
      case OP_CANO_R: bwd_cano_r(C, r); break;
      case OP_CANO_L: bwd_cano_l(C, r); break;
      case OP_SWAP: bwd_swap(C, r); break;
      case OP_REVERSE: bwd_reverse(C, r); break;
      case OP_MERGE: bwd_merge(C, r); break;
      case OP_EAT_A: bwd_eat_a(C, r); break;
      case OP_EAT_B: bwd_eat_b(C, r); break;
      case OP_EAT_C: bwd_eat_c(C, r); break;
      case OP_NORM: bwd_norm(C, r); break;
      case OP_CUT: bwd_cut(C, r); break;
      case OP_LOGZ: bwd_logz(C, r); break;
      default: fail_all(C, CATN_ESTATE); break;
    }
    C.sp = mark;
  }
}

// Walk the whole tape backwards from d lnZ = 1.
CATN_HDI inline void backward(Ctx& C) {
  shadow_zero(C);
  backward_walk(C);
}

// ---------------------------------------------------------------------------
// Checkpointed gradient runs (ckpt_interval K > 0)
// ---------------------------------------------------------------------------
// The forward pass runs in segments of K steps, each from a packed state: the
// live sites laid out contiguously from the working heap's first byte in node
// / position order (the layout load_instance writes), together with the
// slot's graph bookkeeping and the loop state.  Before a segment runs, that
// state is saved in the checkpoint store; the segment then runs with the tape
// on, and its end state is packed for the next one.  The backward pass takes
// the segments last to first.  The last one's records are still in place;
// every earlier one is restored from its checkpoint and recomputed with the
// tape on, i.e. the same arithmetic on the same layout, so the values and
// records are bit-identical to the forward pass.  The shadow of its end
// state's live sites is seeded with the gradient carried back from the next
// segment, its records are walked, and the gradient of its packed start state
// becomes the carry for the segment before (written over that checkpoint's
// own site data, which is not needed again).  Every site gradient
// accumulates the same contributions in the same order as on the whole tape,
// so the result equals the ckpt_interval = 0 run bit for bit.  Memory: the
// scratch stack, one segment's records, the append-only heap of one segment
// and its shadow, and one checkpoint (bookkeeping + live sites) per K steps.
struct CkptHdr {
  LoopState S;
  long long prev;         // store offset of the checkpoint before (-1: none)
  long long meta_bytes;   // bookkeeping (below)
  long long data_bytes;   // packed live sites
  long long sp;
  int rsvd_calls, pad;
};

// Where the slot's bookkeeping lives.  A checkpoint keeps the node headers,
// the edge entries and their free stack, the control words, the logdim
// cache, the site references and neighbour lists of each node up to its
// counts, and the edge map as one flag per entry (the (n+1)^2 map holds
// either -1 or the id of an alive entry of that pair, so the flags "entry e
// is the one mapped" rebuild it exactly); the per-step scratch lists and the
// work counters are not saved.
struct CkptStore {
  long long lo, top, hi;   // byte offsets in the arena
  long long last;          // offset of the newest checkpoint (-1: none)
  long long nodes;         // slot bytes [0, nodes): node headers
  long long ent0, ent1;    // slot bytes [ent0, ent1): edge entries and free stack
  long long ctl0, ctl1;    // slot bytes [ctl0, ctl1): control words
  long long ldc0, ldc1;    // slot bytes [ldc0, ldc1): logdim cache
};

CATN_HD long long ckpt_hdr_bytes() { return al256((long long)sizeof(CkptHdr)); }
CATN_HD long long ckpt_fixed_bytes(const Ctx& C, const CkptStore& K) {
  return al256(K.nodes) + al256(K.ent1 - K.ent0) + al256(K.ctl1 - K.ctl0) + al256(K.ldc1 - K.ldc0) +
         al256(4LL * C.ecap);
}
CATN_HD double* ckpt_data(const Ctx& C, long long at) {
  const CkptHdr* h = (const CkptHdr*)(C.base + at);
  return (double*)(C.base + at + ckpt_hdr_bytes() + h->meta_bytes);
}

// Arena of a checkpointed gradient run: scratch 20 %, records 2 %, the
// checkpoint store 40 %, then the append-only heap of one segment and its
// shadow (19 % each).  Call after make_ctx and before load_instance.
CATN_HDI inline void tape_enable_ckpt(Ctx& C, const SlotLayout& L, long long arena_bytes, CkptStore& K) {
  const long long cap = arena_bytes & ~255LL;
  const long long sc = (cap / 5) & ~255LL;
  const long long rb = (cap / 50) & ~255LL;
  const long long st = (cap * 2 / 5) & ~255LL;
  const long long H = ((cap - sc - rb - st) / 2) & ~255LL;
  C.sp_lo = 0;
  C.sp = 0;
  C.sp_hi = sc;
  C.sp_peak = 0;
  C.rec = (TapeRec*)(C.base + sc);
  C.rcap = rb / (long long)sizeof(TapeRec);
  C.nrec = 0;
  K.lo = K.top = sc + rb;
  K.hi = sc + rb + st;
  K.last = -1;
  K.nodes = L.off_site - L.off_node;
  K.ent0 = L.off_ent - L.off_node;
  K.ent1 = L.off_emap - L.off_node;
  K.ctl0 = L.off_ctl - L.off_node;
  K.ctl1 = L.off_pairs - L.off_node;
  K.ldc0 = L.off_ldc - L.off_node;
  K.ldc1 = L.off_arena - L.off_node;
  C.h_lo0 = C.h_lo1 = K.hi;
  C.hsize = H;
  C.half = 0;
  C.hb = C.h_lo0;
  C.he = C.h_lo0 + H;
  C.h_peak = 0;
  C.gshift = H;
  C.tape = 1;
}

// Team copy of `bytes` (a multiple of 8, both ends 8-byte aligned).
CATN_HDI inline void copy_bytes(const Team& T, char* dst, const char* src, long long bytes) {
  long long* d = (long long*)dst;
  const long long* s = (const long long*)src;
  for (long long e = T.rank(); e < bytes / 8; e += T.size()) d[e] = s[e];
}

// Copy each node's site references and neighbour entries (up to its counts)
// between the slot and a packed area (`save`: slot -> packed).  Every thread
// walks the node counts alike; thread r moves the nodes k = r + 1 (mod team).
CATN_HDI inline void ckpt_lists(Ctx& C, SiteRef* ps, int* pn, bool save) {
  const Team& T = C.T;
  long long os = 0, on = 0;
  for (int k = 1; k <= C.n; ++k) {
    const int ns = C.node[k].nsites, nn = C.node[k].nnbr;
    if ((k - 1) % T.size() == T.rank()) {
      for (int p = 1; p <= ns; ++p) {
        if (save) ps[os + p - 1] = sref(C, k, p);
        else sref(C, k, p) = ps[os + p - 1];
      }
      for (int p = 1; p <= nn; ++p) {
        if (save) pn[on + p - 1] = nbref(C, k, p);
        else nbref(C, k, p) = pn[on + p - 1];
      }
    }
    os += ns;
    on += nn;
  }
}

// Save the current state as a new checkpoint: the live sites packed into the
// store, their references rewritten to the packed layout at the heap's first
// byte, then the bookkeeping and the loop state.  The working heap is
// reloaded from the packed copy (the next segment starts from it).
CATN_HDI inline void ckpt_save(Ctx& C, CkptStore& K, const LoopState& S) {
  const Team& T = C.T;
  long long data = 0, nsite = 0, nnbr = 0;
  for (int k = 1; k <= C.n; ++k) {
    for (int p = 1; p <= C.node[k].nsites; ++p) data += al256(sbytes(sref(C, k, p)));
    nsite += C.node[k].nsites;
    nnbr += C.node[k].nnbr;
  }
  const long long meta = ckpt_fixed_bytes(C, K) + al256(nsite * (long long)sizeof(SiteRef)) + al256(4 * nnbr);
  const long long need = ckpt_hdr_bytes() + meta + data;
  if (K.top + need > K.hi || data > C.hsize) {
    fail_all(C, CATN_ENOMEM);
    return;
  }
  const long long at = K.top;
  char* m = C.base + at + ckpt_hdr_bytes();
  double* dst = (double*)(m + meta);
  T.sync();
  long long cur = 0;
  for (int k = 1; k <= C.n; ++k)
    for (int p = 1; p <= C.node[k].nsites; ++p) {
      const SiteRef s = sref(C, k, p);
      const long long sz = (long long)s.dl * s.d * s.dr;
      const double* src = dptr(C, s.off);
      for (long long e = T.rank(); e < sz; e += T.size()) dst[cur / 8 + e] = src[e];
      cur += al256(8 * sz);
    }
  T.sync();
  if (T.leader()) {
    long long c2 = C.h_lo0;
    for (int k = 1; k <= C.n; ++k)
      for (int p = 1; p <= C.node[k].nsites; ++p) {
        SiteRef& s = sref(C, k, p);
        s.off = c2;
        c2 += al256(sbytes(s));
      }
    CkptHdr h;
    h.S = S;
    h.prev = K.last;
    h.meta_bytes = meta;
    h.data_bytes = data;
    h.sp = C.sp;
    h.rsvd_calls = C.rsvd_calls;
    h.pad = 0;
    *(CkptHdr*)(C.base + at) = h;
  }
  T.sync();
  const char* slot = (const char*)C.node;
  copy_bytes(T, m, slot, K.nodes);
  m += al256(K.nodes);
  copy_bytes(T, m, slot + K.ent0, K.ent1 - K.ent0);
  m += al256(K.ent1 - K.ent0);
  copy_bytes(T, m, slot + K.ctl0, K.ctl1 - K.ctl0);
  m += al256(K.ctl1 - K.ctl0);
  copy_bytes(T, m, slot + K.ldc0, K.ldc1 - K.ldc0);
  m += al256(K.ldc1 - K.ldc0);
  int* flag = (int*)m;
  for (long long e = T.rank(); e < C.ecap; e += T.size()) {
    const EdgeEnt E = C.ent[e];
    flag[e] = (E.alive && emap_at(C, E.i, E.j) == (int)e) ? 1 : 0;
  }
  m += al256(4LL * C.ecap);
  ckpt_lists(C, (SiteRef*)m, (int*)(m + al256(nsite * (long long)sizeof(SiteRef))), true);
  copy_bytes(T, C.base + C.h_lo0, (const char*)dst, data);
  T.sync();
  K.last = at;
  K.top += need;
  C.hb = C.h_lo0 + data;
  C.nrec = 0;
}

// Restore checkpoint `at` (bookkeeping, packed sites, loop state) into the
// slot and the working heap; the tape restarts empty.
CATN_HDI inline void ckpt_restore(Ctx& C, const CkptStore& K, long long at, LoopState& S) {
  const Team& T = C.T;
  T.sync();
  const CkptHdr h = *(const CkptHdr*)(C.base + at);
  char* slot = (char*)C.node;
  const char* m = C.base + at + ckpt_hdr_bytes();
  copy_bytes(T, slot, m, K.nodes);
  m += al256(K.nodes);
  copy_bytes(T, slot + K.ent0, m, K.ent1 - K.ent0);
  m += al256(K.ent1 - K.ent0);
  copy_bytes(T, slot + K.ctl0, m, K.ctl1 - K.ctl0);
  m += al256(K.ctl1 - K.ctl0);
  copy_bytes(T, slot + K.ldc0, m, K.ldc1 - K.ldc0);
  m += al256(K.ldc1 - K.ldc0);
  const int* flag = (const int*)m;
  m += al256(4LL * C.ecap);
  const long long nn = (long long)C.n + 1;
  for (long long e = T.rank(); e < nn * nn; e += T.size()) C.emap[e] = -1;
  T.sync();   // node counts and entries in place before the lists and the map
  for (long long e = T.rank(); e < C.ecap; e += T.size())
    if (flag[e]) emap_at(C, C.ent[e].i, C.ent[e].j) = (int)e;
  long long nsite = 0;
  for (int k = 1; k <= C.n; ++k) nsite += C.node[k].nsites;
  ckpt_lists(C, (SiteRef*)m, (int*)(m + al256(nsite * (long long)sizeof(SiteRef))), false);
  copy_bytes(T, C.base + C.h_lo0, (const char*)ckpt_data(C, at), h.data_bytes);
  T.sync();
  S = h.S;
  C.hb = C.h_lo0 + h.data_bytes;
  C.sp = h.sp;
  C.rsvd_calls = h.rsvd_calls;
  C.nrec = 0;
}

// Seed the shadow of the live sites (node / position order) from `carry`,
// the gradient of the same sites packed as in a checkpoint.
CATN_HDI inline void ckpt_seed(Ctx& C, const double* carry) {
  const Team& T = C.T;
  long long cur = 0;
  for (int k = 1; k <= C.n; ++k)
    for (int p = 1; p <= C.node[k].nsites; ++p) {
      const SiteRef s = sref(C, k, p);
      const long long sz = (long long)s.dl * s.d * s.dr;
      double* g = gptr(C, s.off);
      for (long long e = T.rank(); e < sz; e += T.size()) g[e] = carry[cur / 8 + e];
      cur += al256(8 * sz);
    }
  T.sync();
}

// Forward pass in segments of K steps, then the backward pass segment by
// segment.  Returns the forward outputs; the gradients of the loaded sites
// are left in the shadow of the heap's first bytes (the load layout).
CATN_HDI inline ContractOut contract_grad_ckpt(Ctx& C, CkptStore& K, int interval) {
  const Team& T = C.T;
  LoopState S;
  contract_begin(C, S);
  if (!failed(C)) ckpt_save(C, K, S);
  while (!failed(C)) {
    int steps = 0;
    bool more = true;
    while (steps < interval && (more = contract_step(C, S))) ++steps;
    if (failed(C)) break;
    if (!more) {
      contract_end(C, S);
      break;
    }
    ckpt_save(C, K, S);
  }
  const ContractOut O = S.O;
  if (failed(C)) return O;
  const int jacmax = C.ctl[CTL_JACMAX];
  // the last segment's records and heap are in place
  shadow_zero(C);
  backward_walk(C);
  long long at = K.last;
  while (!failed(C)) {
    const CkptHdr h = *(const CkptHdr*)(C.base + at);
    if (h.prev < 0) break;   // the first checkpoint: the load layout
    // the gradient of this segment's start state is the carry for the one before
    double* carry = ckpt_data(C, at);
    copy_bytes(T, (char*)carry, (const char*)gptr(C, C.h_lo0), h.data_bytes);
    T.sync();
    ckpt_restore(C, K, h.prev, S);
    for (int q = 0; q < interval && !failed(C); ++q)
      if (!contract_step(C, S) && !failed(C)) fail_all(C, CATN_ESTATE);   // the recomputation must retrace
    if (failed(C)) break;
    shadow_zero(C);
    ckpt_seed(C, carry);
    backward_walk(C);
    at = h.prev;
  }
  T.sync();
  if (T.leader() && C.ctl[CTL_JACMAX] < jacmax) C.ctl[CTL_JACMAX] = jacmax;
  T.sync();
  return O;
}

// Gradients of the sites loaded from the image (MPS form), written in the
// image's data layout at `gimg + D.data_off`.
CATN_HDI inline void site_gradients_out(Ctx& C, const InstDesc& D, const long long* img64, double* gimg) {
  const Team& T = C.T;
  const long long* hdr = img64 + D.hdr_off;
  const long long* dims = img64 + D.dim_off;
  double* out = gimg + D.data_off;
  long long sidx = 0, doff = 0, cur = C.heap_first;
  for (int k = 1; k <= C.n; ++k) {
    const int ns = (int)hdr[4 * (k - 1)];
    for (int p = 1; p <= ns; ++p, ++sidx) {
      const long long sz = dims[3 * sidx] * dims[3 * sidx + 1] * dims[3 * sidx + 2];
      const double* g = gptr(C, cur);
      for (long long e = T.rank(); e < sz; e += T.size()) out[doff + e] = g[e];
      doff += sz;
      cur += al256(8 * sz);
    }
  }
  T.sync();
}

// Load, contract with the tape on, run the adjoint and report one instance.
CATN_HDI inline void run_instance_grad(const Team& T, char* slot, const SlotLayout& L, const InstDesc& D,
                                       const long long* i64, const int* i32, const double* dat, catn_result* res,
                                       double* gimg, double* sws, long long sws_doubles,
                                       const JobLink* jl = nullptr) {
  Ctx C = make_ctx(T, slot, L, D.P, D.n, sws, sws_doubles);
  C.multigraph = D.multigraph;
  C.rsvd_min = D.rsvd_min;
  if (jl) {
    C.job = jl->job;
    C.qhead = jl->qhead;
    C.ninst = jl->ninst;
    C.job_min_n = jl->min_n;
    C.job_pool = jl->pool;
    C.job_min_qr = jl->min_qr;
    C.block_min_n = jl->block_min_n;
    C.blocked_qr_min_n = jl->blocked_qr_min_n;
  }
  reset_slot(C);
  const int interval = D.P.ckpt_interval;
  CkptStore K;
  if (interval > 0)
    tape_enable_ckpt(C, L, L.arena_bytes, K);
  else
    tape_enable(C, L.arena_bytes);
  if (D.kind != 0) fail_all(C, CATN_EINVAL);   // gradients of MPS-form inputs only
  if (!failed(C)) load_instance(C, D, i64, i32, dat);
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = -1; O.nsteps = 0;
  const long long t0 = clk();
  if (!failed(C) && interval > 0) {
    O = contract_grad_ckpt(C, K, interval);   // forward, recomputation and backward
    prof_add(C, PROF_TOTAL, (double)(clk() - t0));
  } else if (!failed(C)) {
    O = contract(C);
    prof_add(C, PROF_TOTAL, (double)(clk() - t0));
    if (!failed(C)) backward(C);
  }
  if (!failed(C)) site_gradients_out(C, D, i64, gimg);
  T.sync();
  if (T.leader()) {
    res->lnZ = O.lnZ;
    res->err = O.err;
    res->psi = O.psi;
    res->sign = O.sign;
    res->maxdim = O.maxdim;
    res->status = C.ctl[CTL_STATUS] ? C.ctl[CTL_STATUS] : C.status;
    res->nsteps = O.nsteps;
    res->jacobi_max = C.ctl[CTL_JACMAX];
    res->arena_peak = C.h_lo0 + 2 * C.h_peak;
    res->flops = C.acct[0];
    res->bytes = C.acct[1];
    for (int q = 0; q < PROF_SLOTS; ++q) res->prof[q] = C.acct[2 + q];
  }
  T.sync();
}

}  // namespace catn
