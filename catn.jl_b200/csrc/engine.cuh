// CATN contraction engine: the reference's `contraction!` loop and every MPS
// operation it reaches, as team-cooperative code.  One team (one CTA on the
// GPU) owns one network ("instance") and runs it start to finish.
//
// Execution discipline: every thread of the team runs the same control flow
// on the same data (all control decisions are uniform).  Shared control
// state lives in the slot's global memory; only the leader thread writes it,
// always followed by a team barrier before anyone reads it again.  FP work is
// split over the team (linalg.cuh).
//
// Reference map (CATN.jl v0.1.0):
//   tsvd ...................... linalg_utils.jl:15-28       -> svd_full + keep_rule
//   raw2mps ................... mps_node.jl:31-50           -> raw2mps
//   cano_to!/left_canonical! .. mps_node.jl:72-106          -> cano_to
//   swap!/move!/move2tail!/move2head! mps_node.jl:126-229  -> swap, move, ...
//   reverse! .................. mps_node.jl:238-244         -> reverse_node
//   find/add/delete_neighbor .. mps_node.jl:257-287         -> nb_find, ...
//   logdim .................... mps_node.jl:299-311         -> logdim
//   lognorm / network_lognorm . mps_node.jl:319-328, tensor_network.jl:489-501
//   compress!/compress_opt! ... mps_node.jl:356-447         -> compress_node
//   eat! ...................... mps_node.jl:463-575         -> eat
//   merge! .................... mps_node.jl:595-622         -> merge_dup
//   dim_after_merge/count_*/select_* tensor_network.jl:152-316
//   cut_bondim_opt! ........... tensor_network.jl:399-477   -> cut_bond
//   contraction! .............. tensor_network.jl:556-717   -> contract
#pragma once
#include "linalg.cuh"
#include "catn_layout.h"

namespace catn {

struct Ctx {
  Team T;
  catn_params P;
  int n;        // number of nodes (ids 1..n)
  int maxs;     // site / neighbour capacity per node
  NodeHdr* node;
  SiteRef* site;
  int* nbr;
  EdgeEnt* ent;
  int ecap;
  int* bhead;
  int* btail;
  int* bcnt;
  int* emap;
  int* ctl;
  int* pairs;   // 2 * pcap ints of scratch (pair lists, reverse offsets)
  int pcap;
  int* list;    // lcap ints: node-id lists for the bucket updates
  int* tmp;     // 2 * maxs + 8 ints: neighbour snapshot and duplicates
  char* base;
  long long cap;
  long long* ameta;  // [0] bump, [1..NCLS] free heads, [NCLS+1] peak
  int* trace;
  int trace_cap;
};

// ---------------------------------------------------------------------------
// status
// ---------------------------------------------------------------------------
CATN_HD void set_status_leader(Ctx& C, int code) {
  if (C.ctl[CTL_STATUS] == 0) C.ctl[CTL_STATUS] = code;
}
CATN_HDI inline void set_status(Ctx& C, int code) {
  C.T.sync();
  if (C.T.leader()) set_status_leader(C, code);
  C.T.sync();
}
CATN_HD int failed(const Ctx& C) { return C.ctl[CTL_STATUS] != 0; }

// ---------------------------------------------------------------------------
// arena: power-of-two classes, per-class free lists, bump allocation
// ---------------------------------------------------------------------------
CATN_HD int size_class(long long bytes) {
  int c = 0;
  long long s = 64;
  while (s < bytes) { s <<= 1; ++c; }
  return c;
}

// Leader-only allocation (no barrier).  Returns -1 and sets the status on failure.
CATN_HD long long aalloc_leader(Ctx& C, long long bytes) {
  if (bytes <= 0) bytes = 8;
  int c = size_class(bytes);
  long long off = -1;
  if (c < CATN_NCLS) {
    if (C.ameta[1 + c] >= 0) {
      off = C.ameta[1 + c];
      C.ameta[1 + c] = *(long long*)(C.base + off);
    } else {
      long long sz = 64LL << c;
      if (C.ameta[0] + sz <= C.cap) {
        off = C.ameta[0];
        C.ameta[0] += sz;
        if (C.ameta[0] > C.ameta[CATN_NCLS + 1]) C.ameta[CATN_NCLS + 1] = C.ameta[0];
      }
    }
  }
  if (off < 0) set_status_leader(C, CATN_ENOMEM);
  return off;
}
CATN_HD void afree_leader(Ctx& C, long long off, long long bytes) {
  if (off < 0) return;
  if (bytes <= 0) bytes = 8;
  int c = size_class(bytes);
  *(long long*)(C.base + off) = C.ameta[1 + c];
  C.ameta[1 + c] = off;
}
// Team allocation: every thread receives the offset.
CATN_HDI inline long long aalloc(Ctx& C, long long bytes) {
  long long off = 0;
  C.T.sync();
  if (C.T.leader()) off = aalloc_leader(C, bytes);
  return C.T.bcast(off);
}
// Team free: the block must no longer be in use by any thread.
CATN_HDI inline void afree(Ctx& C, long long off, long long bytes) {
  C.T.sync();
  if (C.T.leader()) afree_leader(C, off, bytes);
  C.T.sync();
}
CATN_HD double* dptr(const Ctx& C, long long off) { return (double*)(C.base + off); }
CATN_HD int* iptr(const Ctx& C, long long off) { return (int*)(C.base + off); }

// ---------------------------------------------------------------------------
// node / site / neighbour accessors (positions are 1-based)
// ---------------------------------------------------------------------------
CATN_HD SiteRef& sref(const Ctx& C, int k, int pos) {
  return C.site[(long long)k * C.maxs + (pos - 1)];
}
CATN_HD int& nbref(const Ctx& C, int k, int pos) { return C.nbr[(long long)k * C.maxs + (pos - 1)]; }
CATN_HD long long sbytes(const SiteRef& s) { return 8LL * s.dl * s.d * s.dr; }
CATN_HD SiteRef mksite(int dl, int d, int dr, long long off) {
  SiteRef s; s.dl = dl; s.d = d; s.dr = dr; s.pad = 0; s.off = off; return s;
}

// find_neighbor (mps_node.jl:257-260): first match, 1-based, 0 = absent.
CATN_HD int nb_find(const Ctx& C, int k, int j) {
  int nn = C.node[k].nnbr;
  for (int p = 1; p <= nn; ++p)
    if (nbref(C, k, p) == j) return p;
  return 0;
}
// Leader-only neighbour edits.
CATN_HD void nb_delete_at_leader(Ctx& C, int k, int pos) {
  int nn = C.node[k].nnbr;
  for (int p = pos; p < nn; ++p) nbref(C, k, p) = nbref(C, k, p + 1);
  C.node[k].nnbr = nn - 1;
}
CATN_HD void nb_insert_at_leader(Ctx& C, int k, int pos, int v) {
  int nn = C.node[k].nnbr;
  if (nn >= C.maxs) { set_status_leader(C, CATN_ENOMEM); return; }
  for (int p = nn; p >= pos; --p) nbref(C, k, p + 1) = nbref(C, k, p);
  nbref(C, k, pos) = v;
  C.node[k].nnbr = nn + 1;
}
CATN_HD void site_delete_at_leader(Ctx& C, int k, int pos) {
  int ns = C.node[k].nsites;
  for (int p = pos; p < ns; ++p) sref(C, k, p) = sref(C, k, p + 1);
  C.node[k].nsites = ns - 1;
}

// logdim (mps_node.jl:299-311): left fold of log2(phys dim).
CATN_HD double logdim_all(const Ctx& C, int k) {
  int ns = C.node[k].nsites;
  double s = 0.0;
  for (int p = 1; p <= ns; ++p) {
    double v = log2((double)sref(C, k, p).d);
    s = (p == 1) ? v : s + v;
  }
  return s;
}
CATN_HD double logdim_at(const Ctx& C, int k, int p) { return log2((double)sref(C, k, p).d); }

// ---------------------------------------------------------------------------
// thin SVD with ownership of the input buffer
// ---------------------------------------------------------------------------
struct Svd {
  long long U, S, V;   // arena offsets: U (m x p), S (p), V (n x p), column-major
  long long m, n, p;
};

CATN_HDI inline void svd_free(Ctx& C, const Svd& R) {
  afree(C, R.U, 8 * R.m * R.p);
  afree(C, R.S, 8 * R.p);
  afree(C, R.V, 8 * R.n * R.p);
}

// SVD of the m x n column-major matrix in arena buffer `a` (allocated with
// `a_bytes`), which is consumed.  S is sorted descending.
//
// Method (Drmac-Veselic preconditioned one-sided Jacobi): pivoted
// Householder QR  W P = Q R  of the tall orientation W (A or A^T), then
// one-sided Jacobi on X = R^T, X V' = U' Sigma, giving R = V' Sigma U'^T and
// W = (Q V') Sigma (P U')^T.  The pivoted, transposed triangle converges in
// a handful of sweeps even for strongly graded spectra.
CATN_HDI inline Svd svd_full(Ctx& C, long long a, long long a_bytes, long long m, long long n) {
  const Team& T = C.T;
  Svd R;
  R.m = m; R.n = n; R.p = 0; R.U = R.S = R.V = -1;
  const bool wide = m < n;
  const long long mm = wide ? n : m, nn = wide ? m : n;
  long long work = a, work_bytes = a_bytes;
  if (wide) {
    work = aalloc(C, 8 * mm * nn);
    if (work < 0) { afree(C, a, a_bytes); return R; }
    materialize(T, dptr(C, work), mm, nn, mm, transposed(dptr(C, a), m));
    afree(C, a, a_bytes);
    work_bytes = 8 * mm * nn;
  }
  long long tau = aalloc(C, 8 * nn);
  long long piv = aalloc(C, 4 * nn);
  long long nrm = aalloc(C, 8 * nn);
  long long X = aalloc(C, 8 * nn * nn);
  long long Vb = aalloc(C, 8 * nn * nn);
  long long sig = aalloc(C, 8 * nn);
  long long Sout = aalloc(C, 8 * nn);
  long long perm = aalloc(C, 4 * nn);
  if (tau < 0 || piv < 0 || nrm < 0 || X < 0 || Vb < 0 || sig < 0 || Sout < 0 || perm < 0) return R;
  qrcp_inplace(T, dptr(C, work), mm, nn, mm, dptr(C, tau), iptr(C, piv), dptr(C, nrm));
  {
    const double* W = dptr(C, work);
    double* Xp = dptr(C, X);
    for (long long e = T.rank(); e < nn * nn; e += T.size()) {
      long long i = e % nn, j = e / nn;
      Xp[e] = (j <= i) ? W[j + i * mm] : 0.0;   // X = R^T
    }
    T.sync();
  }
  int sweeps = jacobi_sweeps(T, dptr(C, X), nn, nn, nn, dptr(C, Vb), 60);
  if (T.leader()) {
    if (sweeps < 0) set_status_leader(C, CATN_ENOCONV);
    else if (sweeps > C.ctl[CTL_JACMAX]) C.ctl[CTL_JACMAX] = sweeps;
  }
  sort_columns(T, dptr(C, X), nn, nn, nn, dptr(C, sig), dptr(C, Sout), iptr(C, perm));
  long long Ut = aalloc(C, 8 * mm * nn);   // left vectors of W: Q V'[:, perm]
  long long Vt = aalloc(C, 8 * nn * nn);   // right vectors of W: P U'[:, perm]
  if (Ut < 0 || Vt < 0) return R;
  {
    const double* Xp = dptr(C, X);
    const double* Sp = dptr(C, Sout);
    const int* pp = iptr(C, perm);
    const int* pv = iptr(C, piv);
    const double* Vp = dptr(C, Vb);
    double* Up = dptr(C, Ut);
    double* Wp = dptr(C, Vt);
    for (long long e = T.rank(); e < mm * nn; e += T.size()) {
      long long r = e % mm, c = e / mm;
      Up[e] = (r < nn) ? Vp[r + (long long)pp[c] * nn] : 0.0;
    }
    for (long long e = T.rank(); e < nn * nn; e += T.size()) {
      long long i = e % nn, c = e / nn;
      double s = Sp[c];
      double v = (s > 0.0) ? Xp[i + (long long)pp[c] * nn] / s : 0.0;
      Wp[(long long)pv[i] + c * nn] = v;
    }
    T.sync();
  }
  qr_apply_q(T, dptr(C, work), mm, nn, mm, dptr(C, tau), dptr(C, Ut), nn, mm);
  afree(C, tau, 8 * nn);
  afree(C, piv, 4 * nn);
  afree(C, nrm, 8 * nn);
  afree(C, X, 8 * nn * nn);
  afree(C, Vb, 8 * nn * nn);
  afree(C, sig, 8 * nn);
  afree(C, perm, 4 * nn);
  afree(C, work, work_bytes);
  R.p = nn;
  R.S = Sout;
  if (!wide) {
    R.U = Ut;   // m x p
    R.V = Vt;   // n x p
  } else {
    R.U = Vt;   // m x m
    R.V = Ut;   // n x m
  }
  return R;
}

// tsvd keep rule (linalg_utils.jl:22-26): nkeep = count(S > cutoff), 0 -> 1,
// capped by maxdim; returns the discarded sum of singular values.
CATN_HDI inline int keep_rule(Ctx& C, const Svd& R, double cutoff, long long maxdim, double* disc) {
  const Team& T = C.T;
  const double* S = dptr(C, R.S);
  double cnt = 0.0;
  for (long long e = T.rank(); e < R.p; e += T.size()) cnt += (S[e] > cutoff) ? 1.0 : 0.0;
  long long count = (long long)(T.sum(cnt) + 0.5);
  long long nkeep = count == 0 ? 1 : count;
  if (nkeep > maxdim) nkeep = maxdim;
  if (nkeep > R.p) nkeep = R.p;
  double d = 0.0;
  for (long long e = nkeep + T.rank(); e < R.p; e += T.size()) d += S[e];
  *disc = T.sum(d);
  return (int)nkeep;
}
// cano_to! keep rule (mps_node.jl:80-81): count(S > cutoff), all when none pass.
CATN_HDI inline int keep_all_if_none(Ctx& C, const Svd& R, double cutoff) {
  const Team& T = C.T;
  const double* S = dptr(C, R.S);
  double cnt = 0.0;
  for (long long e = T.rank(); e < R.p; e += T.size()) cnt += (S[e] > cutoff) ? 1.0 : 0.0;
  long long count = (long long)(T.sum(cnt) + 0.5);
  return (int)(count == 0 ? R.p : count);
}

// ---------------------------------------------------------------------------
// cano_to! (mps_node.jl:72-104)
// ---------------------------------------------------------------------------
CATN_HDI inline void cano_to(Ctx& C, int k, int idx) {
  const Team& T = C.T;
  NodeHdr h = C.node[k];
  if (idx == 0) idx = h.nsites;
  if (h.cano == idx) return;
  if (h.cano < idx) {
    for (int i = h.cano; i < idx; ++i) {
      if (failed(C)) return;
      SiteRef s = sref(C, k, i), nx = sref(C, k, i + 1);
      long long m = (long long)s.dl * s.d, n = s.dr;
      Svd R = svd_full(C, s.off, sbytes(s), m, n);
      if (R.p == 0) return;
      int nkeep = keep_all_if_none(C, R, C.P.cutoff);
      long long ni = aalloc(C, 8 * m * nkeep);
      long long nn2 = aalloc(C, 8LL * nkeep * nx.d * nx.dr);
      if (ni < 0 || nn2 < 0) return;
      copy(T, dptr(C, ni), dptr(C, R.U), m * nkeep);
      // next <- (S V^H)[1:nkeep, :] * next
      gemm(T, nkeep, (long long)nx.d * nx.dr, n,
           mop(dptr(C, R.V), imap(1, 0, n), rows_plain(), dptr(C, R.S), nullptr),
           colmajor(dptr(C, nx.off), n), colmajor(dptr(C, nn2), nkeep));
      svd_free(C, R);
      afree(C, nx.off, sbytes(nx));
      if (T.leader()) {
        sref(C, k, i) = mksite(s.dl, s.d, nkeep, ni);
        sref(C, k, i + 1) = mksite(nkeep, nx.d, nx.dr, nn2);
        C.node[k].cano = i + 1;
      }
      T.sync();
    }
  } else {
    for (int i = h.cano; i > idx; --i) {
      if (failed(C)) return;
      SiteRef s = sref(C, k, i), pv = sref(C, k, i - 1);
      const long long dl = s.dl, m = (long long)s.d * s.dr;
      long long w = aalloc(C, 8 * m * dl);
      if (w < 0) return;
      // Mt = permutedims(site, (2,3,1)) as (d*dr) x dl = transpose of the dl x (d*dr) view
      materialize(T, dptr(C, w), m, dl, m, transposed(dptr(C, s.off), dl));
      afree(C, s.off, sbytes(s));
      Svd R = svd_full(C, w, 8 * m * dl, m, dl);
      if (R.p == 0) return;
      int nkeep = keep_all_if_none(C, R, C.P.cutoff);
      long long ni = aalloc(C, 8 * m * nkeep);
      long long np = aalloc(C, 8LL * pv.dl * pv.d * nkeep);
      if (ni < 0 || np < 0) return;
      // new site = permutedims(reshape(U[:, 1:nkeep], d, dr, nkeep), (3,1,2)) = U^T
      materialize(T, dptr(C, ni), nkeep, m, nkeep, transposed(dptr(C, R.U), m));
      // prev <- prev * (S V^H)^T
      gemm(T, (long long)pv.dl * pv.d, nkeep, dl, colmajor(dptr(C, pv.off), (long long)pv.dl * pv.d),
           mop(dptr(C, R.V), rows_plain(), cols_plain(dl), nullptr, dptr(C, R.S)),
           colmajor(dptr(C, np), (long long)pv.dl * pv.d));
      svd_free(C, R);
      afree(C, pv.off, sbytes(pv));
      if (T.leader()) {
        sref(C, k, i) = mksite(nkeep, s.d, s.dr, ni);
        sref(C, k, i - 1) = mksite(pv.dl, pv.d, nkeep, np);
        C.node[k].cano = i - 1;
      }
      T.sync();
    }
  }
}

// ---------------------------------------------------------------------------
// swap! (mps_node.jl:126-178)
// ---------------------------------------------------------------------------
CATN_HDI inline double swap(Ctx& C, int k, int i, int j) {
  const Team& T = C.T;
  NodeHdr h = C.node[k];
  int dij = i - j;
  if ((dij != 1 && dij != -1) || i < 1 || j < 1 || i > h.nsites || j > h.nsites) {
    set_status(C, CATN_ESTATE);
    return 0.0;
  }
  if (h.cano != i && h.cano != j) {
    int ai = h.cano - i, aj = h.cano - j;
    ai = ai < 0 ? -ai : ai;
    aj = aj < 0 ? -aj : aj;
    cano_to(C, k, ai < aj ? i : j);
    if (failed(C)) return 0.0;
  }
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  SiteRef tl = sref(C, k, lo), tr = sref(C, k, hi);
  const long long d0 = tl.dl, d1 = tr.d, d2 = tl.d, d3 = tr.dr, kk = tl.dr;
  const long long m = d0 * d1, n = d2 * d3;
  long long Mb = aalloc(C, 8 * m * n);
  if (Mb < 0) return 0.0;
  // W = ein"ijk,kab->iajb"(tl, tr); M = reshape(W, d0*d1, d2*d3)
  gemm(T, d0 * d2, d1 * d3, kk, colmajor(dptr(C, tl.off), d0 * d2), colmajor(dptr(C, tr.off), kk),
       mop(dptr(C, Mb), imap((int)d0, 1, d0 * d1), imap((int)d1, d0, d0 * d1 * d2)));
  afree(C, tl.off, sbytes(tl));
  afree(C, tr.off, sbytes(tr));
  const bool rsvd_route = C.P.swapopt && ((m > 7000 && n > 7000) || m > 20000 || n > 20000);
  Svd R = svd_full(C, Mb, 8 * m * n, m, n);
  if (R.p == 0) return 0.0;
  double err = 0.0;
  int myd;
  if (rsvd_route) {
    // The reference's randomized route keeps min(chi, rank) vectors with no
    // cutoff and reports zero error (mps_node.jl:154-156); the exact top-chi
    // subspace it approximates is used here.
    myd = (int)(R.p < C.P.chi ? R.p : C.P.chi);
  } else {
    myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &err);
  }
  long long nl = aalloc(C, 8 * m * myd);
  long long nr = aalloc(C, 8 * n * myd);
  if (nl < 0 || nr < 0) return err;
  if (i < j) {
    copy(T, dptr(C, nl), dptr(C, R.U), m * myd);
    materialize(T, dptr(C, nr), myd, n, myd,
                mop(dptr(C, R.V), imap(1, 0, n), rows_plain(), dptr(C, R.S), nullptr));
  } else {
    materialize(T, dptr(C, nl), m, myd, m,
                mop(dptr(C, R.U), rows_plain(), cols_plain(m), nullptr, dptr(C, R.S)));
    materialize(T, dptr(C, nr), myd, n, myd, mop(dptr(C, R.V), imap(1, 0, n), rows_plain()));
  }
  svd_free(C, R);
  if (T.leader()) {
    sref(C, k, lo) = mksite((int)d0, (int)d1, myd, nl);
    sref(C, k, hi) = mksite(myd, (int)d2, (int)d3, nr);
    C.node[k].cano = j;
    int t = nbref(C, k, i);
    nbref(C, k, i) = nbref(C, k, j);
    nbref(C, k, j) = t;
  }
  T.sync();
  return err;
}

// move! / move2tail! / move2head! (mps_node.jl:186-229)
CATN_HDI inline double move(Ctx& C, int k, int a, int b) {
  double err = 0.0;
  if (a == b) return err;
  if (b > a) {
    for (int idx = a; idx < b && !failed(C); ++idx) err += swap(C, k, idx, idx + 1);
  } else {
    for (int idx = a; idx > b && !failed(C); --idx) err += swap(C, k, idx, idx - 1);
  }
  return err;
}
CATN_HDI inline double move2tail(Ctx& C, int k, int idx) {
  double err = 0.0;
  int n = C.node[k].nsites;
  if (idx == n) {
    cano_to(C, k, n);
    return err;
  }
  for (int q = idx; q < n && !failed(C); ++q) err += swap(C, k, q, q + 1);
  cano_to(C, k, n);
  return err;
}
CATN_HDI inline double move2head(Ctx& C, int k, int idx) {
  double err = move(C, k, idx, 1);
  cano_to(C, k, 1);
  return err;
}

// reverse! (mps_node.jl:238-244): reversed site order, each site (3,2,1)-permuted.
CATN_HDI inline void reverse_node(Ctx& C, int k) {
  const Team& T = C.T;
  NodeHdr h = C.node[k];
  if (h.nsites <= 1) return;
  const int ns = h.nsites;
  long long* offs = (long long*)(C.pairs);   // scratch: new offsets per site
  T.sync();
  if (T.leader()) {
    for (int p = 1; p <= ns; ++p) offs[p - 1] = aalloc_leader(C, sbytes(sref(C, k, p)));
  }
  T.sync();
  if (failed(C)) return;
  for (int p = 1; p <= ns; ++p) {
    SiteRef s = sref(C, k, p);
    const double* src = dptr(C, s.off);
    double* dst = dptr(C, offs[p - 1]);
    const long long dl = s.dl, d = s.d, dr = s.dr, tot = dl * d * dr;
    for (long long e = T.rank(); e < tot; e += T.size()) {
      long long a = e % dl, rest = e / dl, b = rest % d, c = rest / d;
      dst[c + dr * (b + d * a)] = src[e];
    }
  }
  T.sync();
  if (T.leader()) {
    for (int p = 1; p <= ns; ++p) afree_leader(C, sref(C, k, p).off, sbytes(sref(C, k, p)));
    for (int p = 1; p <= ns / 2; ++p) {
      SiteRef a = sref(C, k, p), b = sref(C, k, ns + 1 - p);
      sref(C, k, p) = b;
      sref(C, k, ns + 1 - p) = a;
    }
    for (int p = 1; p <= ns; ++p) {
      SiteRef s = sref(C, k, p);
      sref(C, k, p) = mksite(s.dr, s.d, s.dl, offs[ns - p]);
    }
    int nn = C.node[k].nnbr;
    for (int p = 1; p <= nn / 2; ++p) {
      int t = nbref(C, k, p);
      nbref(C, k, p) = nbref(C, k, nn + 1 - p);
      nbref(C, k, nn + 1 - p) = t;
    }
    C.node[k].cano = ns + 1 - h.cano;
  }
  T.sync();
}

// Free every site of node k and empty its lists (clear!, mps_node.jl:335-339).
CATN_HDI inline void clear_node(Ctx& C, int k) {
  C.T.sync();
  if (C.T.leader()) {
    int ns = C.node[k].nsites;
    for (int p = 1; p <= ns; ++p) afree_leader(C, sref(C, k, p).off, sbytes(sref(C, k, p)));
    C.node[k].nsites = 0;
    C.node[k].nnbr = 0;
  }
  C.T.sync();
}

CATN_HDI inline double norm_of(Ctx& C, const double* x, long long n) {
  if (C.P.norm_method == 1) return sqrt(sumsq(C.T, x, n));
  if (C.P.norm_method == 2) return maxabs(C.T, x, n);
  return 1.0;
}

// ---------------------------------------------------------------------------
// merge! (mps_node.jl:595-622)
// ---------------------------------------------------------------------------
CATN_HDI inline double merge_dup(Ctx& C, int k, int j, bool cross) {
  const Team& T = C.T;
  int idx1 = 0, idx2 = 0, found = 0;
  {
    int nn = C.node[k].nnbr;
    for (int p = 1; p <= nn; ++p) {
      if (nbref(C, k, p) == j) {
        if (found == 0) idx1 = p;
        else if (found == 1) idx2 = p;
        ++found;
      }
    }
  }
  if (found != 2) {
    set_status(C, CATN_ESTATE);
    return 0.0;
  }
  int target = cross ? idx1 : idx1 + 1;
  double err = move(C, k, idx2, target);
  if (failed(C)) return err;
  T.sync();
  if (T.leader()) nb_delete_at_leader(C, k, target);
  T.sync();
  cano_to(C, k, idx1);
  if (failed(C)) return err;
  SiteRef a = sref(C, k, idx1), b = sref(C, k, idx1 + 1);
  long long rows = (long long)a.dl * a.d, cols = (long long)b.d * b.dr;
  long long f = aalloc(C, 8 * rows * cols);
  if (f < 0) return err;
  gemm(T, rows, cols, a.dr, colmajor(dptr(C, a.off), rows), colmajor(dptr(C, b.off), a.dr),
       colmajor(dptr(C, f), rows));
  afree(C, a.off, sbytes(a));
  afree(C, b.off, sbytes(b));
  if (T.leader()) {
    sref(C, k, idx1) = mksite(a.dl, a.d * b.d, b.dr, f);
    site_delete_at_leader(C, k, idx1 + 1);
  }
  T.sync();
  cano_to(C, k, idx1);
  return err;
}

// ---------------------------------------------------------------------------
// eat! (mps_node.jl:463-575).  Returns lognorm; adds swap errors to *err and
// multiplies the phase into *phase.
// ---------------------------------------------------------------------------
CATN_HDI inline double eat(Ctx& C, int ki, int kj, int idx, int idxi, double* err, double* phase) {
  const Team& T = C.T;
  const double cutoff = C.P.cutoff;
  NodeHdr hi = C.node[ki];
  if (hi.nsites == 1) {
    // (a) both leaves: non-conjugating dot product
    if (C.node[kj].nsites != 1) { set_status(C, CATN_ESTATE); return 0.0; }
    SiteRef si = sref(C, ki, 1), sj = sref(C, kj, 1);
    long long d = si.d;
    double loc = 0.0;
    const double* vi = dptr(C, si.off);
    const double* vj = dptr(C, sj.off);
    for (long long e = T.rank(); e < d; e += T.size()) loc = fma(vi[e], vj[e], loc);
    double r = T.sum(loc);
    double absr = fabs(r);
    T.sync();
    if (T.leader()) {
      afree_leader(C, si.off, sbytes(si));
      C.node[ki].nsites = 0;
      nb_delete_at_leader(C, ki, idx);
    }
    T.sync();
    if (absr <= cutoff) return 0.0;
    *phase *= (r / absr);
    return log(absr);
  }
  *err += move2tail(C, ki, idx);
  if (failed(C)) return 0.0;
  hi = C.node[ki];
  SiteRef last = sref(C, ki, hi.nsites);   // (dl, d, 1)
  SiteRef prev = sref(C, ki, hi.nsites - 1);
  if (C.node[kj].nsites == 1) {
    // (b) j is a leaf
    SiteRef tj = sref(C, kj, 1);
    long long vbuf = aalloc(C, 8LL * last.dl);
    long long nt = aalloc(C, 8LL * prev.dl * prev.d);
    if (vbuf < 0 || nt < 0) return 0.0;
    gemm(T, last.dl, 1, last.d, colmajor(dptr(C, last.off), last.dl), colmajor(dptr(C, tj.off), last.d),
         colmajor(dptr(C, vbuf), last.dl));
    gemm(T, (long long)prev.dl * prev.d, 1, prev.dr, colmajor(dptr(C, prev.off), (long long)prev.dl * prev.d),
         colmajor(dptr(C, vbuf), prev.dr), colmajor(dptr(C, nt), (long long)prev.dl * prev.d));
    afree(C, vbuf, 8LL * last.dl);
    const long long ne = (long long)prev.dl * prev.d;
    double nrm = norm_of(C, dptr(C, nt), ne);
    afree(C, last.off, sbytes(last));
    afree(C, prev.off, sbytes(prev));
    if (T.leader()) {
      sref(C, ki, hi.nsites - 1) = mksite(prev.dl, prev.d, 1, nt);
      C.node[ki].cano = C.node[ki].cano - 1;
      C.node[ki].nsites = hi.nsites - 1;
      C.node[ki].nnbr = C.node[ki].nnbr - 1;
    }
    T.sync();
    if (nrm <= cutoff) return 0.0;
    scale(T, dptr(C, nt), 1.0 / nrm, ne);
    return log(nrm);
  }
  // (c) general
  *err += move2head(C, kj, idxi);
  if (failed(C)) return 0.0;
  SiteRef hj = sref(C, kj, 1);   // (1, d, drj)
  const long long Dl = last.dl, dd = last.d, Dr = hj.dr;
  long long mat = aalloc(C, 8 * Dl * Dr);
  long long nt = aalloc(C, 8LL * prev.dl * prev.d * Dr);
  if (mat < 0 || nt < 0) return 0.0;
  gemm(T, Dl, Dr, dd, colmajor(dptr(C, last.off), Dl), colmajor(dptr(C, hj.off), dd),
       colmajor(dptr(C, mat), Dl));
  gemm(T, (long long)prev.dl * prev.d, Dr, prev.dr, colmajor(dptr(C, prev.off), (long long)prev.dl * prev.d),
       colmajor(dptr(C, mat), Dl), colmajor(dptr(C, nt), (long long)prev.dl * prev.d));
  afree(C, mat, 8 * Dl * Dr);
  afree(C, last.off, sbytes(last));
  afree(C, prev.off, sbytes(prev));
  afree(C, hj.off, sbytes(hj));
  T.sync();
  if (T.leader()) {
    const int nsi = hi.nsites - 1;
    sref(C, ki, nsi) = mksite(prev.dl, prev.d, (int)Dr, nt);
    const int nsj = C.node[kj].nsites;
    if (nsi + nsj - 1 > C.maxs || C.node[ki].nnbr - 1 + C.node[kj].nnbr > C.maxs) {
      set_status_leader(C, CATN_ENOMEM);
    } else {
      for (int p = 2; p <= nsj; ++p) sref(C, ki, nsi + p - 1) = sref(C, kj, p);
      C.node[ki].nsites = nsi + nsj - 1;
      C.node[ki].cano = nsi;
      C.node[kj].nsites = 0;   // ownership of j's sites 2:end moved to i
      int nni = C.node[ki].nnbr - 1;
      const int nnj = C.node[kj].nnbr;
      for (int p = 2; p <= nnj; ++p) nbref(C, ki, nni + p - 1) = nbref(C, kj, p);
      C.node[ki].nnbr = nni + (nnj > 1 ? nnj - 1 : 0);
    }
  }
  T.sync();
  if (failed(C)) return 0.0;
  cano_to(C, ki, C.node[ki].nsites);
  if (failed(C)) return 0.0;
  SiteRef ctr = sref(C, ki, C.node[ki].cano);
  double nrm = norm_of(C, dptr(C, ctr.off), (long long)ctr.dl * ctr.d * ctr.dr);
  if (nrm <= cutoff) return 0.0;
  scale(T, dptr(C, ctr.off), 1.0 / nrm, (long long)ctr.dl * ctr.d * ctr.dr);
  return log(nrm);
}

// ---------------------------------------------------------------------------
// QR pre-reduction helper: matrix X (rows x cols) in buffer `buf` (consumed
// into Householder form when rows > cols).  Produces R (cols x cols or the
// original rows x cols) in a new buffer.
// ---------------------------------------------------------------------------
struct QRed {
  bool flag;
  long long house, house_bytes, tau;   // Householder storage (rows x cols) and tau (cols)
  long long Rb;                         // R (or the matrix itself), column-major
  long long rrows, cols, rows;
};

CATN_HDI inline QRed qr_reduce(Ctx& C, long long buf, long long buf_bytes, long long rows, long long cols) {
  const Team& T = C.T;
  QRed q;
  q.rows = rows;
  q.cols = cols;
  q.house = buf;
  q.house_bytes = buf_bytes;
  q.tau = -1;
  q.flag = rows > cols;
  if (!q.flag) {
    q.Rb = buf;
    q.rrows = rows;
    return q;
  }
  q.tau = aalloc(C, 8 * cols);
  q.Rb = aalloc(C, 8 * cols * cols);
  q.rrows = cols;
  if (q.tau < 0 || q.Rb < 0) return q;
  qr_inplace(T, dptr(C, buf), rows, cols, rows, dptr(C, q.tau));
  const double* W = dptr(C, buf);
  double* Rp = dptr(C, q.Rb);
  for (long long e = T.rank(); e < cols * cols; e += T.size()) {
    long long r = e % cols, c = e / cols;
    Rp[e] = (r <= c) ? W[r + c * rows] : 0.0;
  }
  T.sync();
  return q;
}
// Y (rrows x ncols) -> Q [Y; 0] (rows x ncols) in a new buffer (or a copy when !flag).
CATN_HDI inline long long qr_expand(Ctx& C, const QRed& q, const double* Y, long long ncols) {
  const Team& T = C.T;
  long long out = aalloc(C, 8 * q.rows * ncols);
  if (out < 0) return out;
  double* O = dptr(C, out);
  for (long long e = T.rank(); e < q.rows * ncols; e += T.size()) {
    long long r = e % q.rows, c = e / q.rows;
    O[e] = (r < q.rrows) ? Y[r + c * q.rrows] : 0.0;
  }
  T.sync();
  if (q.flag) qr_apply_q(T, dptr(C, q.house), q.rows, q.cols, q.rows, dptr(C, q.tau), O, ncols, q.rows);
  return out;
}
CATN_HDI inline void qr_release(Ctx& C, const QRed& q) {
  if (q.flag) {
    afree(C, q.tau, 8 * q.cols);
    afree(C, q.Rb, 8 * q.cols * q.cols);
  }
  afree(C, q.house, q.house_bytes);
}

// ---------------------------------------------------------------------------
// compress! / compress_opt! (mps_node.jl:356-447).  Returns the discarded sum.
// ---------------------------------------------------------------------------
CATN_HDI inline double compress_node(Ctx& C, int k, bool opt) {
  const Team& T = C.T;
  double err = 0.0;
  if (C.node[k].nsites == 0) return err;
  T.sync();
  if (T.leader()) C.node[k].cano = 1;
  T.sync();
  cano_to(C, k, C.node[k].nsites);
  const int ns = C.node[k].nsites;
  for (int jj = ns; jj >= 2 && !failed(C); --jj) {
    const int i = jj - 1;
    SiteRef tl = sref(C, k, i), tr = sref(C, k, jj);
    const long long d0 = tl.dl, d1 = tl.d, dd = tl.dr, d2 = tr.d, d3 = tr.dr;
    const long long ml = d0 * d1, nr = d2 * d3;
    long long Uo, Vo;
    int myd;
    double e;
    if (!opt) {
      long long mat = aalloc(C, 8 * ml * nr);
      if (mat < 0) return err;
      gemm(T, ml, nr, dd, colmajor(dptr(C, tl.off), ml), colmajor(dptr(C, tr.off), dd),
           colmajor(dptr(C, mat), ml));
      afree(C, tl.off, sbytes(tl));
      afree(C, tr.off, sbytes(tr));
      Svd R = svd_full(C, mat, 8 * ml * nr, ml, nr);
      if (R.p == 0) return err;
      myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &e);
      Uo = aalloc(C, 8 * ml * myd);
      Vo = aalloc(C, 8 * nr * myd);
      if (Uo < 0 || Vo < 0) return err;
      materialize(T, dptr(C, Uo), ml, myd, ml, mop(dptr(C, R.U), rows_plain(), cols_plain(ml), nullptr, dptr(C, R.S)));
      materialize(T, dptr(C, Vo), myd, nr, myd, mop(dptr(C, R.V), imap(1, 0, nr), rows_plain()));
      svd_free(C, R);
    } else {
      // matl = (d0 d1) x dd, QR when tall; matr^H = (d2 d3) x dd, QR when matr is wide
      QRed ql = qr_reduce(C, tl.off, sbytes(tl), ml, dd);
      long long trt = aalloc(C, 8 * nr * dd);
      if (trt < 0) return err;
      materialize(T, dptr(C, trt), nr, dd, nr, transposed(dptr(C, tr.off), dd));
      afree(C, tr.off, sbytes(tr));
      QRed qr = qr_reduce(C, trt, 8 * nr * dd, nr, dd);
      if (failed(C)) return err;
      // mat = Rl * Rr^H  (ql.rrows x qr.rrows)
      long long mat = aalloc(C, 8 * ql.rrows * qr.rrows);
      if (mat < 0) return err;
      gemm(T, ql.rrows, qr.rrows, dd, colmajor(dptr(C, ql.Rb), ql.rrows), transposed(dptr(C, qr.Rb), qr.rrows),
           colmajor(dptr(C, mat), ql.rrows));
      Svd R = svd_full(C, mat, 8 * ql.rrows * qr.rrows, ql.rrows, qr.rrows);
      if (R.p == 0) return err;
      myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &e);
      // U * S then Ql;  V then Qr
      long long us = aalloc(C, 8 * ql.rrows * myd);
      if (us < 0) return err;
      materialize(T, dptr(C, us), ql.rrows, myd, ql.rrows,
                  mop(dptr(C, R.U), rows_plain(), cols_plain(ql.rrows), nullptr, dptr(C, R.S)));
      long long Ufull = qr_expand(C, ql, dptr(C, us), myd);
      long long Vfull = qr_expand(C, qr, dptr(C, R.V), myd);   // first myd columns of V
      afree(C, us, 8 * ql.rrows * myd);
      svd_free(C, R);
      qr_release(C, ql);
      qr_release(C, qr);
      if (Ufull < 0 || Vfull < 0) return err;
      Uo = Ufull;
      Vo = aalloc(C, 8 * nr * myd);
      if (Vo < 0) return err;
      materialize(T, dptr(C, Vo), myd, nr, myd, transposed(dptr(C, Vfull), nr));
      afree(C, Vfull, 8 * nr * myd);
    }
    err += e;
    if (T.leader()) {
      sref(C, k, i) = mksite((int)d0, (int)d1, myd, Uo);
      sref(C, k, jj) = mksite(myd, (int)d2, (int)d3, Vo);
    }
    T.sync();
  }
  T.sync();
  if (T.leader()) C.node[k].cano = 1;
  T.sync();
  return err;
}

// ---------------------------------------------------------------------------
// cut_bondim_opt! (tensor_network.jl:399-477).  Returns the discarded sum.
// ---------------------------------------------------------------------------
CATN_HDI inline double cut_bond(Ctx& C, int i, int idx_j_in_i) {
  const Team& T = C.T;
  if (C.P.Dmax < 0) return 0.0;
  int j = nbref(C, i, idx_j_in_i);
  if (j <= 0) { set_status(C, CATN_ESTATE); return 0.0; }
  int idx_i_in_j = nb_find(C, j, i);
  if (idx_i_in_j == 0) { set_status(C, CATN_ESTATE); return 0.0; }
  cano_to(C, i, idx_j_in_i);
  cano_to(C, j, idx_i_in_j);
  if (failed(C)) return 0.0;
  SiteRef Ai = sref(C, i, idx_j_in_i), Aj = sref(C, j, idx_i_in_j);
  const long long d = Ai.d;
  const long long ri_rows = (long long)Ai.dl * Ai.dr, rj_rows = (long long)Aj.dl * Aj.dr;
  // mati = reshape(permutedims(Ai, (1,3,2)), da_l*da_r, d)
  long long mi = aalloc(C, 8 * ri_rows * d);
  long long mj = aalloc(C, 8 * rj_rows * d);
  if (mi < 0 || mj < 0) return 0.0;
  materialize(T, dptr(C, mi), ri_rows, d, ri_rows,
              mop(dptr(C, Ai.off), imap(Ai.dl, 1, (long long)Ai.dl * d), cols_plain(Ai.dl)));
  materialize(T, dptr(C, mj), rj_rows, d, rj_rows,
              mop(dptr(C, Aj.off), imap(Aj.dl, 1, (long long)Aj.dl * d), cols_plain(Aj.dl)));
  afree(C, Ai.off, sbytes(Ai));
  afree(C, Aj.off, sbytes(Aj));
  QRed qi = qr_reduce(C, mi, 8 * ri_rows * d, ri_rows, d);
  QRed qj = qr_reduce(C, mj, 8 * rj_rows * d, rj_rows, d);
  if (failed(C)) return 0.0;
  long long mg = aalloc(C, 8 * qi.rrows * qj.rrows);
  if (mg < 0) return 0.0;
  gemm(T, qi.rrows, qj.rrows, d, colmajor(dptr(C, qi.Rb), qi.rrows), transposed(dptr(C, qj.Rb), qj.rrows),
       colmajor(dptr(C, mg), qi.rrows));
  Svd R = svd_full(C, mg, 8 * qi.rrows * qj.rrows, qi.rrows, qj.rrows);
  if (R.p == 0) return 0.0;
  double disc = 0.0;
  int kept = keep_rule(C, R, C.P.cutoff, 0x7fffffffLL, &disc);
  int myd = kept < C.P.Dmax ? kept : C.P.Dmax;
  if (myd < 1) myd = 1;
  double extra = 0.0;
  {
    const double* S = dptr(C, R.S);
    double loc = 0.0;
    for (long long e = myd + T.rank(); e < kept; e += T.size()) loc += S[e];
    extra = T.sum(loc);
  }
  // sqrt(S) scaled factors
  long long sq = aalloc(C, 8LL * myd);
  long long ui = aalloc(C, 8 * qi.rrows * myd);
  long long vj = aalloc(C, 8 * qj.rrows * myd);
  if (sq < 0 || ui < 0 || vj < 0) return 0.0;
  {
    const double* S = dptr(C, R.S);
    double* q = dptr(C, sq);
    for (long long e = T.rank(); e < myd; e += T.size()) q[e] = sqrt(S[e]);
    T.sync();
  }
  materialize(T, dptr(C, ui), qi.rrows, myd, qi.rrows,
              mop(dptr(C, R.U), rows_plain(), cols_plain(qi.rrows), nullptr, dptr(C, sq)));
  materialize(T, dptr(C, vj), qj.rrows, myd, qj.rrows,
              mop(dptr(C, R.V), rows_plain(), cols_plain(qj.rrows), nullptr, dptr(C, sq)));
  svd_free(C, R);
  afree(C, sq, 8LL * myd);
  long long fi = qr_expand(C, qi, dptr(C, ui), myd);   // (da_l*da_r) x myd
  long long fj = qr_expand(C, qj, dptr(C, vj), myd);
  afree(C, ui, 8 * qi.rrows * myd);
  afree(C, vj, 8 * qj.rrows * myd);
  qr_release(C, qi);
  qr_release(C, qj);
  if (fi < 0 || fj < 0) return 0.0;
  // new site = permutedims(reshape(mat, dl, dr, myd), (1,3,2))
  long long ni = aalloc(C, 8LL * Ai.dl * myd * Ai.dr);
  long long nj = aalloc(C, 8LL * Aj.dl * myd * Aj.dr);
  if (ni < 0 || nj < 0) return 0.0;
  {
    const double* F = dptr(C, fi);
    double* O = dptr(C, ni);
    const long long dl = Ai.dl, dr = Ai.dr, tot = dl * myd * dr;
    for (long long e = T.rank(); e < tot; e += T.size()) {
      long long a = e % dl, rest = e / dl, r = rest % myd, c = rest / myd;
      O[e] = F[(a + dl * c) + ri_rows * r];
    }
    const double* G = dptr(C, fj);
    double* P2 = dptr(C, nj);
    const long long dl2 = Aj.dl, dr2 = Aj.dr, tot2 = dl2 * myd * dr2;
    for (long long e = T.rank(); e < tot2; e += T.size()) {
      long long a = e % dl2, rest = e / dl2, r = rest % myd, c = rest / myd;
      P2[e] = G[(a + dl2 * c) + rj_rows * r];
    }
    T.sync();
  }
  afree(C, fi, 8 * ri_rows * myd);
  afree(C, fj, 8 * rj_rows * myd);
  if (T.leader()) {
    sref(C, i, idx_j_in_i) = mksite(Ai.dl, myd, Ai.dr, ni);
    sref(C, j, idx_i_in_j) = mksite(Aj.dl, myd, Aj.dr, nj);
  }
  T.sync();
  return disc + extra;
}

// ---------------------------------------------------------------------------
// raw2mps (mps_node.jl:31-50): dense column-major tensor -> sites of node k.
// ---------------------------------------------------------------------------
CATN_HDI inline void raw2mps(Ctx& C, int k, const double* data, const long long* dims, int nd) {
  const Team& T = C.T;
  if (nd == 0) return;   // the reference returns an empty MPS for a 0-d tensor
  long long total = 1;
  for (int q = 0; q < nd; ++q) total *= dims[q];
  if (nd > C.maxs) { set_status(C, CATN_ENOMEM); return; }
  long long R = aalloc(C, 8 * total);
  if (R < 0) return;
  copy(T, dptr(C, R), data, total);
  long long Rbytes = 8 * total, cur = total;
  long long dleft = 1;
  for (int q = 0; q < nd - 1; ++q) {
    long long m = dleft * dims[q], n = cur / m;
    Svd S = svd_full(C, R, Rbytes, m, n);
    if (S.p == 0) return;
    double disc;
    int c = keep_rule(C, S, C.P.cutoff, C.P.chi, &disc);
    long long u = aalloc(C, 8 * m * c);
    long long r2 = aalloc(C, 8LL * c * n);
    if (u < 0 || r2 < 0) return;
    copy(T, dptr(C, u), dptr(C, S.U), m * c);
    materialize(T, dptr(C, r2), c, n, c, mop(dptr(C, S.V), imap(1, 0, n), rows_plain(), dptr(C, S.S), nullptr));
    svd_free(C, S);
    if (T.leader()) sref(C, k, q + 1) = mksite((int)dleft, (int)dims[q], c, u);
    T.sync();
    R = r2;
    Rbytes = 8LL * c * n;
    cur = (long long)c * n;
    dleft = c;
  }
  if (T.leader()) {
    sref(C, k, nd) = mksite((int)dleft, (int)dims[nd - 1], 1, R);
    C.node[k].nsites = nd;
    C.node[k].cano = nd;
  }
  T.sync();
}

// ---------------------------------------------------------------------------
// edge-cost buckets (tensor_network.jl:152-236), leader-only helpers
// ---------------------------------------------------------------------------
CATN_HD int dim_after_merge(const Ctx& C, int i, int j) {
  int idx = nb_find(C, i, j);
  double v = logdim_all(C, i) + logdim_all(C, j) - 2.0 * logdim_at(C, i, idx);
  return (int)rint(v);
}
CATN_HD int& emap_at(const Ctx& C, int i, int j) { return C.emap[(long long)i * (C.n + 1) + j]; }

CATN_HD void bucket_add_leader(Ctx& C, int cost, int i, int j) {
  if (cost < 0 || cost >= CATN_CMAX) { set_status_leader(C, CATN_ENOMEM); return; }
  int e = C.ctl[CTL_FREEENT];
  if (e < 0) { set_status_leader(C, CATN_ENOMEM); return; }
  C.ctl[CTL_FREEENT] = C.ent[e].next;
  EdgeEnt& E = C.ent[e];
  E.cost = cost; E.i = i; E.j = j; E.alive = 1; E.next = -1; E.prev = C.btail[cost];
  if (C.btail[cost] >= 0) C.ent[C.btail[cost]].next = e;
  else C.bhead[cost] = e;
  C.btail[cost] = e;
  C.bcnt[cost] += 1;
  if (cost < C.ctl[CTL_MINC]) C.ctl[CTL_MINC] = cost;
  int& m = emap_at(C, i, j);
  if (m >= 0 && C.ent[m].alive) C.ctl[CTL_ANOMALY] += 1;
  m = e;
}
CATN_HD void bucket_unlink_leader(Ctx& C, int e) {
  EdgeEnt& E = C.ent[e];
  if (E.prev >= 0) C.ent[E.prev].next = E.next; else C.bhead[E.cost] = E.next;
  if (E.next >= 0) C.ent[E.next].prev = E.prev; else C.btail[E.cost] = E.prev;
  C.bcnt[E.cost] -= 1;
  E.alive = 0;
  E.next = C.ctl[CTL_FREEENT];
  C.ctl[CTL_FREEENT] = e;
}
// filter!(pair -> pair != [i,j], edge_count[cost])
CATN_HD void bucket_remove_leader(Ctx& C, int cost, int i, int j) {
  if (cost < 0 || cost >= CATN_CMAX) return;
  int& m = emap_at(C, i, j);
  if (m >= 0 && C.ent[m].alive && C.ent[m].cost == cost && C.ent[m].i == i && C.ent[m].j == j) {
    bucket_unlink_leader(C, m);
    m = -1;
    return;
  }
  // Slow path: entries not reachable through the pair map.
  if (C.bcnt[cost] == 0) return;
  int e = C.bhead[cost];
  for (int guard = 0; e >= 0 && guard <= C.ecap; ++guard) {
    int nx = C.ent[e].next;
    if (C.ent[e].i == i && C.ent[e].j == j) {
      bucket_unlink_leader(C, e);
      if (m == e) m = -1;
    }
    e = nx;
  }
}

// Sort pairs (lexicographic) in scratch, dedupe; returns count.
CATN_HD int sort_pairs_leader(int* pr, int np) {
  // shell sort on packed 64-bit keys
  for (int gap = np / 2; gap > 0; gap /= 2) {
    for (int a = gap; a < np; ++a) {
      int ti = pr[2 * a], tj = pr[2 * a + 1];
      int b = a;
      while (b >= gap && (pr[2 * (b - gap)] > ti || (pr[2 * (b - gap)] == ti && pr[2 * (b - gap) + 1] > tj))) {
        pr[2 * b] = pr[2 * (b - gap)];
        pr[2 * b + 1] = pr[2 * (b - gap) + 1];
        b -= gap;
      }
      pr[2 * b] = ti;
      pr[2 * b + 1] = tj;
    }
  }
  int w = 0;
  for (int a = 0; a < np; ++a) {
    if (w > 0 && pr[2 * (w - 1)] == pr[2 * a] && pr[2 * (w - 1) + 1] == pr[2 * a + 1]) continue;
    pr[2 * w] = pr[2 * a];
    pr[2 * w + 1] = pr[2 * a + 1];
    ++w;
  }
  return w;
}

// count_add_nodes! (:185-197) over `list` (node ids, <=0 skipped).
CATN_HD void count_add_nodes_leader(Ctx& C, const int* list, int nl) {
  int* pr = C.pairs;
  int np = 0;
  for (int a = 0; a < nl; ++a) {
    int i = list[a];
    if (i <= 0) continue;
    int nn = C.node[i].nnbr;
    for (int p = 1; p <= nn; ++p) {
      int j = nbref(C, i, p);
      if (j <= 0) continue;
      if (np >= C.pcap) { set_status_leader(C, CATN_ENOMEM); return; }
      pr[2 * np] = i < j ? i : j;
      pr[2 * np + 1] = i < j ? j : i;
      ++np;
    }
  }
  np = sort_pairs_leader(pr, np);
  for (int a = 0; a < np; ++a) {
    int i = pr[2 * a], j = pr[2 * a + 1];
    bucket_add_leader(C, dim_after_merge(C, i, j), i, j);
  }
}
// count_remove_nodes! (:213-225)
CATN_HD void count_remove_nodes_leader(Ctx& C, const int* list, int nl) {
  for (int a = 0; a < nl; ++a) {
    int id = list[a];
    if (id <= 0) continue;
    int nn = C.node[id].nnbr;
    for (int p = 1; p <= nn; ++p) {
      int nb = nbref(C, id, p);
      if (nb <= 0) continue;
      int i = id < nb ? id : nb, j = id < nb ? nb : id;
      bucket_remove_leader(C, dim_after_merge(C, i, j), i, j);
    }
  }
}

CATN_HD int min_cost_leader(Ctx& C) {
  int c = C.ctl[CTL_MINC];
  if (c < 0) c = 0;
  while (c < CATN_CMAX && C.bcnt[c] == 0) ++c;
  C.ctl[CTL_MINC] = c;
  return c;
}

// select_edge_min_dim (:248-253) / _triangle (:262-288) / _sequentially (:300-316)
CATN_HD long long select_leader(Ctx& C, int* maxdim) {
  int sel = C.P.select;
  if (sel == 0 || sel == 1) {
    int cost = min_cost_leader(C);
    if (cost >= CATN_CMAX) { set_status_leader(C, CATN_ESTATE); return 0; }
    if (cost > *maxdim) *maxdim = cost;
    int e = C.bhead[cost];
    int bi = C.ent[e].i, bj = C.ent[e].j;
    if (sel == 1) {
      int best = -1;
      for (int guard = 0; e >= 0 && guard <= C.ecap; e = C.ent[e].next, ++guard) {
        int i = C.ent[e].i, j = C.ent[e].j;
        int nn = C.node[j].nnbr;
        int both = 0;
        for (int p = 1; p <= nn; ++p) {
          int k = nbref(C, j, p);
          if (k <= 0 || k == i) continue;
          bool dup = false;
          for (int q = 1; q < p; ++q)
            if (nbref(C, j, q) == k) { dup = true; break; }
          if (dup) continue;
          if (nb_find(C, k, i) > 0) ++both;
        }
        if (both > best) { best = both; bi = i; bj = j; }
      }
    }
    return ((long long)bi << 32) | (unsigned)bj;
  }
  // sequential: minimum i + nb, ascending node ids
  long long best = -1;
  int bs = 0x7fffffff;
  for (int i = 1; i <= C.n; ++i) {
    int nn = C.node[i].nnbr;
    for (int p = 1; p <= nn; ++p) {
      int nb = nbref(C, i, p);
      if (nb <= 0 || !(i < nb)) continue;
      if (i + nb < bs) { bs = i + nb; best = ((long long)i << 32) | (unsigned)nb; }
    }
  }
  if (best < 0) set_status_leader(C, CATN_ESTATE);
  return best < 0 ? 0 : best;
}

CATN_HDI inline int has_real_edges(Ctx& C) {
  const Team& T = C.T;
  int loc = 0;
  for (int k = 1 + T.rank(); k <= C.n && !loc; k += T.size()) {
    int nn = C.node[k].nnbr;
    for (int p = 1; p <= nn; ++p)
      if (nbref(C, k, p) > 0) { loc = 1; break; }
  }
  return T.any(loc);
}

CATN_HD unsigned fnv_step(unsigned h, int v) { return (h ^ (unsigned)v) * 16777619u; }

// ---------------------------------------------------------------------------
// contraction! (tensor_network.jl:556-717)
// ---------------------------------------------------------------------------
struct ContractOut {
  double lnZ, err, psi, sign;
  int maxdim, nsteps;
};

CATN_HDI inline ContractOut contract(Ctx& C) {
  const Team& T = C.T;
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = -1; O.nsteps = 0;
  const bool buckets = (C.P.select == 0 || C.P.select == 1);
  if (buckets) {
    T.sync();
    if (T.leader()) {
      // select_edge_init!: all node ids
      for (int k = 1; k <= C.n; ++k) C.list[k - 1] = k;
      count_add_nodes_leader(C, C.list, C.n);
    }
    T.sync();
  }
  int maxdim = -1;
  // Every step clears one node, so a network of n nodes needs fewer than n
  // steps; the cap only guards against corrupted state.
  const int step_cap = C.n + 16;
  while (!failed(C) && has_real_edges(C)) {
    if (O.nsteps > step_cap) {
      set_status(C, CATN_ESTATE);
      break;
    }
    // --- select ---
    long long pk = 0;
    int md = maxdim;
    T.sync();
    if (T.leader()) pk = select_leader(C, &md);
    pk = T.bcast(pk);
    maxdim = (int)T.bcast(md);
    if (failed(C)) break;
    int i = (int)(pk >> 32), j = (int)(pk & 0xffffffff);
    if (C.node[j].nsites > C.node[i].nsites) { int t = i; i = j; j = t; }
    // --- bookkeeping before any shape change ---
    if (buckets) {
      T.sync();
      if (T.leader()) {
        int* list = C.list;
        int nl = 0;
        list[nl++] = i;
        list[nl++] = j;
        for (int p = 1; p <= C.node[i].nnbr; ++p) list[nl++] = nbref(C, i, p);
        for (int p = 1; p <= C.node[j].nnbr; ++p) list[nl++] = nbref(C, j, p);
        count_remove_nodes_leader(C, list, nl);
      }
      T.sync();
    }
    int idx_j_in_i = nb_find(C, i, j);
    int idx_i_in_j = nb_find(C, j, i);
    int rev = 0;
    if (C.P.reverse) {
      int li = C.node[i].nnbr, lj = C.node[j].nnbr;
      if (idx_j_in_i < (li + 1) / 2) {
        reverse_node(C, i);
        idx_j_in_i = nb_find(C, i, j);
        rev |= 1;
      }
      if (idx_i_in_j >= (lj + 1) / 2) {
        reverse_node(C, j);
        idx_i_in_j = nb_find(C, j, i);
        rev |= 2;
      }
    }
    if (failed(C)) break;
    // snapshot of j's neighbours (after any reverse)
    int* neigh_j = C.tmp;
    int* dup = C.tmp + C.maxs;
    const int lnj = C.node[j].nnbr;
    T.sync();
    if (T.leader())
      for (int p = 1; p <= lnj; ++p) neigh_j[p - 1] = nbref(C, j, p);
    T.sync();
    int nd = 0;
    unsigned duph = 2166136261u;
    for (int l = 1; l <= lnj && !failed(C); ++l) {
      if (l == idx_i_in_j) continue;
      int k = neigh_j[l - 1];
      if (k <= 0) continue;
      int idx_k_in_i = nb_find(C, i, k);
      int idx_i_in_k = nb_find(C, k, i);
      int idx_j_in_k = nb_find(C, k, j);
      if (idx_j_in_k == 0) { set_status(C, CATN_ESTATE); break; }
      T.sync();
      if (T.leader()) {
        nb_delete_at_leader(C, k, idx_j_in_k);
        nb_insert_at_leader(C, k, idx_j_in_k, i);
      }
      T.sync();
      if (idx_k_in_i > 0) {
        T.sync();
        if (T.leader()) dup[nd] = k;
        T.sync();
        ++nd;
        duph = fnv_step(duph, k);
        bool cross = idx_i_in_k > idx_j_in_k;
        O.err += merge_dup(C, k, i, cross);
      }
    }
    if (failed(C)) break;
    // --- eat! ---
    double lnv = eat(C, i, j, idx_j_in_i, idx_i_in_j, &O.err, &O.psi);
    O.lnZ += lnv;
    if (failed(C)) break;
    // --- duplicates: merge into i, then cut ---
    for (int q = 0; q < nd && !failed(C); ++q) {
      int k = dup[q];
      merge_dup(C, i, k, false);   // its error is not accumulated (tensor_network.jl:662)
      int idx_k_in_i = nb_find(C, i, k);
      if (failed(C)) break;
      if (C.P.cut_bond || (C.P.Dmax > 0 && sref(C, i, idx_k_in_i).d > C.P.Dmax))
        O.err += cut_bond(C, i, idx_k_in_i);
    }
    if (failed(C)) break;
    clear_node(C, j);
    if (C.P.compress) compress_node(C, i, C.P.svdopt != 0);   // error discarded (:688-694)
    if (failed(C)) break;
    if (buckets) {
      T.sync();
      if (T.leader()) {
        int* list = C.list;
        int nl = 0;
        list[nl++] = i;
        for (int p = 1; p <= C.node[i].nnbr; ++p) list[nl++] = nbref(C, i, p);
        count_add_nodes_leader(C, list, nl);
      }
      T.sync();
    }
    const int nsi = C.node[i].nsites;
    unsigned shh = 2166136261u;
    for (int p = 1; p <= nsi; ++p) {
      int d = sref(C, i, p).d;
      if (d > maxdim) maxdim = d;
      shh = fnv_step(shh, d);
    }
    if (C.trace && O.nsteps < C.trace_cap) {
      T.sync();
      if (T.leader()) {
        int* r = C.trace + 8LL * O.nsteps;
        r[0] = i; r[1] = j; r[2] = rev; r[3] = nd; r[4] = (int)duph; r[5] = nsi; r[6] = (int)shh; r[7] = maxdim;
      }
      T.sync();
    }
    O.nsteps += 1;
  }
  // --- network_lognorm (tensor_network.jl:489-501) ---
  double lsum = 0.0, nneg = 0.0, nzero = 0.0, bad = 0.0;
  for (int k = 1 + T.rank(); k <= C.n; k += T.size()) {
    NodeHdr h = C.node[k];
    bool scalar = true;
    for (int p = 1; p <= h.nsites; ++p)
      if (sref(C, k, p).d != 1) { scalar = false; break; }
    if (!scalar || h.nsites == 0) continue;
    if (h.nsites != 1) { bad += 1.0; continue; }
    SiteRef s = sref(C, k, 1);
    const double* x = dptr(C, s.off);
    double z = 0.0;
    for (long long e = 0; e < (long long)s.dl * s.dr; ++e) z += x[e];
    lsum += log(fabs(z));
    if (z < 0) nneg += 1.0;
    if (z == 0) nzero += 1.0;
  }
  lsum = T.sum(lsum);
  nneg = T.sum(nneg);
  nzero = T.sum(nzero);
  bad = T.sum(bad);
  if (bad > 0.5) set_status(C, CATN_ESTATE);
  O.lnZ += lsum;
  O.sign = nzero > 0.5 ? 0.0 : (((long long)(nneg + 0.5)) % 2 ? -1.0 : 1.0);
  O.maxdim = maxdim;
  return O;
}

// ---------------------------------------------------------------------------
// Slot initialisation and instance loading
// ---------------------------------------------------------------------------
CATN_HDI inline Ctx make_ctx(const Team& T, char* slot, const SlotLayout& L, const catn_params& P, int n) {
  Ctx C;
  C.T = T;
  C.P = P;
  C.n = n;
  C.maxs = L.maxs;
  C.node = (NodeHdr*)(slot + L.off_node);
  C.site = (SiteRef*)(slot + L.off_site);
  C.nbr = (int*)(slot + L.off_nbr);
  C.ent = (EdgeEnt*)(slot + L.off_ent);
  C.ecap = L.ecap;
  C.bhead = (int*)(slot + L.off_bhead);
  C.btail = (int*)(slot + L.off_btail);
  C.bcnt = (int*)(slot + L.off_bcnt);
  C.emap = (int*)(slot + L.off_emap);
  C.ctl = (int*)(slot + L.off_ctl);
  C.pairs = (int*)(slot + L.off_pairs);
  C.pcap = L.pcap;
  C.list = (int*)(slot + L.off_list);
  C.tmp = (int*)(slot + L.off_tmp);
  C.ameta = (long long*)(slot + L.off_ameta);
  C.base = slot + L.off_arena;
  C.cap = L.arena_bytes;
  C.trace = nullptr;
  C.trace_cap = 0;
  return C;
}

CATN_HDI inline void reset_slot(Ctx& C) {
  const Team& T = C.T;
  const long long nn = (long long)C.n + 1;
  for (long long e = T.rank(); e < nn * nn; e += T.size()) C.emap[e] = -1;
  for (long long e = T.rank(); e < CATN_CMAX; e += T.size()) { C.bhead[e] = -1; C.btail[e] = -1; C.bcnt[e] = 0; }
  for (long long e = T.rank(); e < C.ecap; e += T.size()) {
    C.ent[e].alive = 0;
    C.ent[e].next = (e + 1 < C.ecap) ? (int)(e + 1) : -1;
  }
  for (long long e = T.rank(); e < nn; e += T.size()) { C.node[e].nsites = 0; C.node[e].nnbr = 0; C.node[e].cano = 0; C.node[e].pad = 0; }
  for (long long e = T.rank(); e < CATN_NCLS + 2; e += T.size()) C.ameta[e] = (e >= 1 && e <= CATN_NCLS) ? -1 : 0;
  for (long long e = T.rank(); e < CTL_WORDS; e += T.size()) C.ctl[e] = 0;
  T.sync();
  if (T.leader()) {
    C.ctl[CTL_FREEENT] = C.ecap > 0 ? 0 : -1;
    C.ctl[CTL_MINC] = 0;
  }
  T.sync();
}

// Load one instance from the packed input image.
CATN_HDI inline void load_instance(Ctx& C, const InstDesc& D, const long long* img64, const int* img32,
                                   const double* imgd) {
  const Team& T = C.T;
  const long long* hdr = img64 + D.hdr_off;
  const long long* dims = img64 + D.dim_off;
  const int* nbrs = img32 + D.nbr_off;
  const double* data = imgd + D.data_off;
  if (D.kind == 0) {
    // MPS form: leader allocates every site, then the team copies
    T.sync();
    if (T.leader()) {
      long long sidx = 0, nidx = 0;
      for (int k = 1; k <= C.n; ++k) {
        int ns = (int)hdr[4 * (k - 1)], nn = (int)hdr[4 * (k - 1) + 1], cano = (int)hdr[4 * (k - 1) + 2];
        if (ns > C.maxs || nn > C.maxs) { set_status_leader(C, CATN_ENOMEM); break; }
        C.node[k].nsites = ns;
        C.node[k].nnbr = nn;
        C.node[k].cano = cano;
        for (int p = 1; p <= ns; ++p, ++sidx) {
          int dl = (int)dims[3 * sidx], d = (int)dims[3 * sidx + 1], dr = (int)dims[3 * sidx + 2];
          long long off = aalloc_leader(C, 8LL * dl * d * dr);
          sref(C, k, p) = mksite(dl, d, dr, off);
        }
        for (int p = 1; p <= nn; ++p, ++nidx) nbref(C, k, p) = nbrs[nidx];
      }
    }
    T.sync();
    if (failed(C)) return;
    long long doff = 0;
    for (int k = 1; k <= C.n; ++k) {
      int ns = C.node[k].nsites;
      for (int p = 1; p <= ns; ++p) {
        SiteRef s = sref(C, k, p);
        long long sz = (long long)s.dl * s.d * s.dr;
        double* dst = dptr(C, s.off);
        for (long long e = T.rank(); e < sz; e += T.size()) dst[e] = data[doff + e];
        doff += sz;
      }
    }
    T.sync();
  } else {
    long long dpos = 0, doff = 0, nidx = 0;
    for (int k = 1; k <= C.n && !failed(C); ++k) {
      int nd = (int)hdr[4 * (k - 1)];
      if (nd > C.maxs) { set_status(C, CATN_ENOMEM); break; }
      T.sync();
      if (T.leader()) {
        C.node[k].nnbr = nd;
        for (int p = 1; p <= nd; ++p) nbref(C, k, p) = nbrs[nidx + p - 1];
      }
      T.sync();
      long long tot = 1;
      for (int q = 0; q < nd; ++q) tot *= dims[dpos + q];
      raw2mps(C, k, data + doff, dims + dpos, nd);
      nidx += nd;
      dpos += nd;
      doff += (nd == 0) ? 1 : tot;
    }
  }
}

}  // namespace catn

namespace catn {

// Load, contract and report one instance in the given slot.
CATN_HDI inline void run_instance(const Team& T, char* slot, const SlotLayout& L, const InstDesc& D,
                                  const long long* i64, const int* i32, const double* dat,
                                  catn_result* res, int* trace_base) {
  Ctx C = make_ctx(T, slot, L, D.P, D.n);
  reset_slot(C);
  if (D.trace_cap > 0 && trace_base) {
    C.trace = trace_base + D.trace_off;
    C.trace_cap = D.trace_cap;
  }
  load_instance(C, D, i64, i32, dat);
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = -1; O.nsteps = 0;
  if (!failed(C)) O = contract(C);
  T.sync();
  if (T.leader()) {
    res->lnZ = O.lnZ;
    res->err = O.err;
    res->psi = O.psi;
    res->sign = O.sign;
    res->maxdim = O.maxdim;
    res->status = C.ctl[CTL_STATUS];
    res->nsteps = O.nsteps;
    res->jacobi_max = C.ctl[CTL_JACMAX];
    res->arena_peak = C.ameta[CATN_NCLS + 1];
  }
  T.sync();
}

}  // namespace catn

namespace catn {

// mps2raw of the single surviving open-leg node (tensor_network.jl:517-523,
// mps_node.jl:52-70) into `out` (capacity `cap` doubles).  Returns the number
// of elements (0 for a closed network, -1 on error); leg sizes go to dims.
CATN_HDI inline long long result_tensor_dev(Ctx& C, double* out, long long cap, long long* dims, int* ndim) {
  const Team& T = C.T;
  int open = 0, cnt = 0;
  for (int k = 1; k <= C.n; ++k) {
    int ns = C.node[k].nsites;
    bool scalar = true;
    for (int p = 1; p <= ns; ++p)
      if (sref(C, k, p).d != 1) { scalar = false; break; }
    if (!scalar) { open = k; ++cnt; }
  }
  if (cnt == 0) { *ndim = 0; return 0; }
  if (cnt > 1) { set_status(C, CATN_ESTATE); return -1; }
  const int ns = C.node[open].nsites;
  long long total = 1;
  for (int p = 1; p <= ns; ++p) total *= sref(C, open, p).d;
  SiteRef s0 = sref(C, open, 1);
  long long rmax = s0.dr;
  for (int p = 1; p <= ns; ++p) if (sref(C, open, p).dr > rmax) rmax = sref(C, open, p).dr;
  long long cur = aalloc(C, 8 * total * rmax);
  long long nxt = aalloc(C, 8 * total * rmax);
  if (cur < 0 || nxt < 0) return -1;
  copy(T, dptr(C, cur), dptr(C, s0.off), (long long)s0.d * s0.dr);
  long long pdim = s0.d;
  for (int p = 2; p <= ns; ++p) {
    SiteRef b = sref(C, open, p);
    gemm(T, pdim, (long long)b.d * b.dr, b.dl, colmajor(dptr(C, cur), pdim), colmajor(dptr(C, b.off), b.dl),
         colmajor(dptr(C, nxt), pdim));
    long long t = cur; cur = nxt; nxt = t;
    pdim *= b.d;
  }
  if (total <= cap && out) copy(T, out, dptr(C, cur), total);
  if (T.leader()) {
    for (int p = 1; p <= ns && p <= 64; ++p) dims[p - 1] = sref(C, open, p).d;
    *ndim = ns;
  }
  T.sync();
  afree(C, cur, 8 * total * rmax);
  afree(C, nxt, 8 * total * rmax);
  return total;
}

}  // namespace catn
