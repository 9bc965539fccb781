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
//   tsvd ...................... linalg_utils.jl:15-28       -> svd_begin/svd_finish + keep_rule
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
//   dim_after_merge/count_*/select_* tensor_network.jl:152-316 -> pair_cost, count_*_team, select_team
//   cut_bondim_opt! ........... tensor_network.jl:399-477   -> cut_bond
//   contraction! .............. tensor_network.jl:556-717   -> contract
#pragma once
#include "linalg.cuh"
#include "blockjac.cuh"
#include "ising_build.cuh"
#include "catn_layout.h"

namespace catn {

// One operation of the adjoint tape (gradient runs).  Every operation that
// writes site data appends one record naming its input and output versions
// by heap byte offset (the heap is append-only on a gradient run, so an
// offset names one version for the whole run) plus what its backward needs.
enum {
  OP_CANO_R = 1,   // a: dl d dr nkeep nx.d nx.dr    o: site nx | new site, new nx | S V
  OP_CANO_L,       // a: dl d dr nkeep pv.dl pv.d    o: site pv | new site, new pv | S V
  OP_SWAP,         // a: d0 d1 d2 d3 k myd i<j       o: tl tr | lo hi | S, U or V
  OP_REVERSE,      // a: dl d dr                     o: old new
  OP_MERGE,        // a: dl da k db dr               o: a b | fused
  OP_EAT_A,        // a: d                           o: vi vj          v: r, flag: |r| > cutoff
  OP_EAT_B,        // a: Dl dd ne                    o: last tj prev | new
  OP_EAT_C,        // a: Dl dd Dr pr                 o: last hj prev | new
  OP_NORM,         // a: len method                  o: x | x / nrm    v: nrm
  OP_CUT,          // a: dl d dr dl2 dr2 myd         o: Ai Aj | new Ai, new Aj | S
  OP_LOGZ          // a: len                         o: scalar site    v: z
};
struct TapeRec {
  int op, flag;
  int a[10];
  long long o[8];
  double v[2];
};

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
  int* fstack;   // free stack of entry ids (CTL_FTOP entries)
  int* emap;
  int* ctl;
  int* pairs;   // 12 * pcap bytes of scratch (sort keys, reverse refs)
  int pcap;
  int* list;    // lcap ints: node-id lists for the bucket updates
  int* tmp;     // 2 * maxs + 8 ints: neighbour snapshot and duplicates
  char* base;   // arena
  // Scratch stack for per-operation temporaries [sp_lo, sp_hi).  Every
  // thread keeps an identical copy of the stack pointer, so pushing and
  // popping needs no barrier.
  long long sp, sp_lo, sp_hi, sp_peak;
  // Site heap: two halves of hsize bytes; allocation bumps hb inside the
  // current half, and a full half is compacted into the other one.
  long long h_lo0, h_lo1, hsize, hb, he;
  int half;
  int compactions;
  long long h_peak;
  // Shared-memory workspace for small SVDs.
  double* sws;
  long long sws_doubles;
  double* acct;   // [flops, bytes] (global, leader-updated)
  double* ldc;    // per-node logdim cache [n+1]
  long long* ldv; // cache validity [n+1]
  int status;     // uniform copy of the instance status
  int rsvd_min;   // randomized-SVD route threshold override (0: 7000 / 20000)
  int rsvd_calls; // randomized SVDs so far (selects each sketch's generator stream)
  int multigraph; // the input lists some neighbour twice
  int* trace;
  int trace_cap;
  // Adjoint tape (tape != 0 on gradient runs only): the site heap is
  // append-only, records go to rec[0, rcap), and the gradient of the double
  // at heap byte offset o lives at byte offset o + gshift (the shadow heap).
  int tape;
  TapeRec* rec;
  long long nrec, rcap, gshift;
  long long heap_first;   // first byte of the sites loaded from the image
  // Shared Jacobi (batch kernel): this CTA's job board entry, the launch's
  // work-queue head and instance count (helpers exist once the queue is
  // drained), and the smallest column count worth sharing.
  JacobiJob* job;
  const int* qhead;
  int ninst, job_min_n;
  int job_pool;        // CTAs of the launch do nothing but help: share from the start
  long long job_min_qr;   // smallest rows x columns whose Householder work is shared
  int block_min_n;     // smallest Jacobi factor (columns) on the block route
  int blocked_qr_min_n;   // smallest block-route QR (columns) taking the blocked, norm-sorted form
};

// Where a batch CTA publishes its shared Jacobi sweeps (null: never).
struct JobLink {
  JacobiJob* job;
  const int* qhead;
  int ninst, min_n;
  int pool;   // the launch has dedicated helper CTAs
  long long min_qr;
  int block_min_n;   // smallest Jacobi factor (columns) on the block route
  int blocked_qr_min_n;
  int cta_jobs;      // some instance may publish CTA items (block route): helpers claim as whole CTAs
};

// ---------------------------------------------------------------------------
// status: C.status is identical in every thread (uniform control flow);
// ctl[CTL_STATUS] is the global copy reported to the host.
// ---------------------------------------------------------------------------
CATN_HD void fail_all(Ctx& C, int code) {   // called by every thread alike
  if (C.status == 0) C.status = code;
  if (C.T.leader() && C.ctl[CTL_STATUS] == 0) C.ctl[CTL_STATUS] = code;
}
CATN_HD void fail_leader(Ctx& C, int code) {   // inside leader-only blocks
  if (C.ctl[CTL_STATUS] == 0) C.ctl[CTL_STATUS] = code;
}
// After a leader-only block that may have failed: make the status uniform.
CATN_HDI inline void refresh_status(Ctx& C) {
  C.T.sync();
  C.status = C.ctl[CTL_STATUS];
  C.T.sync();
}
CATN_HD int failed(const Ctx& C) { return C.status != 0; }

// ---------------------------------------------------------------------------
// memory
// ---------------------------------------------------------------------------
CATN_HD long long al256(long long b) { return (b + 255) & ~255LL; }

// SM clock for the per-instance cycle breakdown (0 in the host build).
CATN_HD long long clk() {
#if CATN_DEVICE_PASS
  return (long long)clock64();
#else
  return 0;
#endif
}
enum { PROF_TOTAL = 0, PROF_SVD_TINY, PROF_SVD_SMALL, PROF_SVD_LARGE, PROF_BOOK, PROF_N_TINY, PROF_N_SMALL,
       PROF_N_LARGE, PROF_SWAP_GEMM, PROF_SWAP_EPI, PROF_CANO_EPI, PROF_EAT, PROF_MERGE, PROF_CUT, PROF_REVERSE,
       PROF_CONTROL, PROF_LQR, PROF_LJAC, PROF_LAPPLY, PROF_N_BLOCK, PROF_BLOCK_SWEEPS, PROF_LJAC_COLS,
       PROF_LJAC_BLOCK, PROF_LJAC_BIG, PROF_SLOTS, PROF_COMPACT = PROF_SLOTS, PROF_N_COMPACT = PROF_SLOTS + 1 };
CATN_HD void prof_add(Ctx& C, int slot, double v) {
  if (C.T.leader()) C.acct[2 + slot] += v;
}


CATN_HD double* spush(Ctx& C, long long ndoubles) {
  long long bytes = al256(8 * (ndoubles > 0 ? ndoubles : 1));
  if (C.sp + bytes > C.sp_hi) {
    fail_all(C, CATN_ENOMEM);
    return nullptr;
  }
  double* p = (double*)(C.base + C.sp);
  C.sp += bytes;
  if (C.sp > C.sp_peak) C.sp_peak = C.sp;
  return p;
}

CATN_HD double* dptr(const Ctx& C, long long off) { return (double*)(C.base + off); }
CATN_HD SiteRef& sref(const Ctx& C, int k, int pos) {
  return C.site[(long long)k * C.maxs + (pos - 1)];
}
CATN_HD int& nbref(const Ctx& C, int k, int pos) { return C.nbr[(long long)k * C.maxs + (pos - 1)]; }
CATN_HD long long sbytes(const SiteRef& s) { return 8LL * s.dl * s.d * s.dr; }
CATN_HD SiteRef mksite(int dl, int d, int dr, long long off) {
  SiteRef s; s.dl = dl; s.d = d; s.dr = dr; s.pad = 0; s.off = off; return s;
}
CATN_HD double* sdata(const Ctx& C, const SiteRef& s) { return (double*)(C.base + s.off); }

// Move every live site into the other heap half, contiguously.
CATN_HDI inline void heap_compact(Ctx& C) {
  const Team& T = C.T;
  const long long t0 = clk();
  T.sync();
  const long long lo = C.half ? C.h_lo0 : C.h_lo1;
  long long cur = lo;
  for (int k = 1; k <= C.n; ++k) {
    const int ns = C.node[k].nsites;
    for (int p = 1; p <= ns; ++p) {
      SiteRef s = sref(C, k, p);
      const long long sz = (long long)s.dl * s.d * s.dr;
      const double* src = dptr(C, s.off);
      double* dst = dptr(C, cur);
      for (long long e = T.rank(); e < sz; e += T.size()) dst[e] = src[e];
      cur += al256(8 * sz);
    }
  }
  T.sync();
  if (T.leader()) {
    long long c2 = lo;
    for (int k = 1; k <= C.n; ++k) {
      const int ns = C.node[k].nsites;
      for (int p = 1; p <= ns; ++p) {
        SiteRef& s = sref(C, k, p);
        s.off = c2;
        c2 += al256(sbytes(s));
      }
    }
  }
  T.sync();
  C.half ^= 1;
  C.hb = cur;
  C.he = lo + C.hsize;
  C.compactions += 1;
  prof_add(C, PROF_COMPACT, (double)(clk() - t0));
  prof_add(C, PROF_N_COMPACT, 1.0);
}

// Make room for `bytes` of new sites (may compact: re-read site refs after).
// A gradient run never compacts: every version stays where it was written.
CATN_HDI inline bool heap_reserve(Ctx& C, long long bytes) {
  if (C.hb + bytes <= C.he) return true;
  if (!C.tape) heap_compact(C);
  if (C.hb + bytes <= C.he) return true;
  fail_all(C, CATN_ENOMEM);
  return false;
}
CATN_HD long long heap_take(Ctx& C, long long bytes) {
  long long off = C.hb;
  C.hb += al256(bytes);
  long long used = C.hb - (C.half ? C.h_lo1 : C.h_lo0);
  if (used > C.h_peak) C.h_peak = used;
  return off;
}

// Append one tape record (all threads call it alike; the leader writes).
CATN_HD TapeRec trec(int op) {
  TapeRec r;
  r.op = op;
  r.flag = 0;
  for (int q = 0; q < 10; ++q) r.a[q] = 0;
  for (int q = 0; q < 8; ++q) r.o[q] = -1;
  r.v[0] = r.v[1] = 0.0;
  return r;
}
CATN_HD void tape_push(Ctx& C, const TapeRec& r) {
  if (C.nrec >= C.rcap) {
    fail_all(C, CATN_ENOMEM);
    return;
  }
  if (C.T.leader()) C.rec[C.nrec] = r;
  C.nrec += 1;
}

// Algorithmic work counters.
CATN_HD void account(Ctx& C, double flops, double bytes) {
  if (C.T.leader()) {
    C.acct[0] += flops;
    C.acct[1] += bytes;
  }
}

// ---------------------------------------------------------------------------
// neighbour accessors (positions are 1-based)
// ---------------------------------------------------------------------------
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
  if (nn >= C.maxs) { fail_leader(C, CATN_ENOMEM); return; }
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
// thin SVD (workspace in shared memory when it fits, else scratch)
// ---------------------------------------------------------------------------
struct Svd {
  double* U;   // m x p, column-major
  double* S;   // p, descending
  double* V;   // n x p
  long long m, n, p;
};

// Oriented input: W (mm x nn, mm >= nn) holds A (m x n) or A^T when m < n.
struct SvdIn {
  double* W;
  long long m, n, mm, nn;
  bool wide, smem;
  double tol;      // rank-revealing stop tolerance for large inputs (0 = none)
  long long need;  // singular vectors the caller can use (the first `need`; S is always complete)
};

CATN_HD long long svd_ws_doubles(long long mm, long long nn) {
  return 2 * mm * nn + 3 * nn * nn + 8 * nn + 64;
}

// `cutoff`: the truncation cutoff the caller applies to the singular values;
// large inputs may drop a trailing block whose singular values are all below
// a quarter of it (never counted, never kept).
CATN_HDI inline SvdIn svd_begin(Ctx& C, long long m, long long n, double cutoff = 0.0) {
  SvdIn s;
  s.m = m;
  s.n = n;
  s.tol = 0.25 * cutoff;
  s.wide = m < n;
  s.mm = s.wide ? n : m;
  s.nn = s.wide ? m : n;
  s.need = 1LL << 40;
  if (s.mm * s.nn >= (1LL << 31)) {   // index arithmetic is 32-bit per operation
    fail_all(C, CATN_ENOMEM);
    s.smem = false;
    s.W = nullptr;
    return s;
  }
  s.smem = svd_ws_doubles(s.mm, s.nn) <= C.sws_doubles;
  s.W = s.smem ? C.sws : spush(C, s.mm * s.nn);
  return s;
}
// Operand map that writes A(r, c) into the oriented W.
CATN_HD MOp svd_target(const SvdIn& s) {
  return s.wide ? mop(s.W, cols_plain(s.mm), rows_plain()) : colmajor(s.W, s.mm);
}
CATN_HDI inline void svd_fill(Ctx& C, const SvdIn& s, const MOp& A) {
  const Team& T = C.T;
  for (long long e = T.rank(); e < s.mm * s.nn; e += T.size()) {
    long long r, c;
    divmod(e, s.mm, &r, &c);
    s.W[e] = s.wide ? A.ld(c, r) : A.ld(r, c);
  }
  T.sync();
}

// Whether the Jacobi sweeps on an n-column matrix in global memory go to the
// shared job: always when the launch has dedicated helper CTAs, otherwise
// once the launch's queue is drained (idle CTAs then help); the same answer
// in every thread.
// Whether p points into this CTA's shared memory (the SVD workspace or any
// other part of it).  Such an address means nothing to another CTA, so work
// on an array there is never published to helper CTAs.
CATN_HD bool cta_local(const Ctx& C, const void* p) {
#if CATN_DEVICE_PASS
  (void)C;
  return p && __isShared(p);
#else
  const double* q = (const double*)p;
  return q && q >= C.sws && q < C.sws + C.sws_doubles;
#endif
}

CATN_HDI inline bool share_jacobi(Ctx& C, long long n, const double* X, const double* V, const double* nrm) {
  if (!C.job || n < C.job_min_n || cta_local(C, X) || cta_local(C, V) || cta_local(C, nrm)) return false;
  if (C.job_pool) return true;
  long long drained = 0;
  if (C.T.leader()) drained = ldcg_i(C.qhead) >= C.ninst ? 1 : 0;
  return C.T.bcast(drained) != 0;
}

// Whether the Householder work on a rows x cols matrix in global memory goes
// to the shared job (same rule as share_jacobi, by element count); X and Y
// are the arrays the helpers would read and write.
CATN_HDI inline bool share_house(Ctx& C, long long rows, long long cols, const double* X, const double* Y) {
  if (!C.job || rows * cols < C.job_min_qr || cta_local(C, X) || cta_local(C, Y)) return false;
  if (C.job_pool) return true;
  long long drained = 0;
  if (C.T.leader()) drained = ldcg_i(C.qhead) >= C.ninst ? 1 : 0;
  return C.T.bcast(drained) != 0;
}
// Whether the one-sided Jacobi on an n-column factor X takes the block route
// (blockjac.cuh): svd_route 2, or svd_route 0 with precision 1, for factors
// of at least block_min_n columns held in global memory.  The factor and its
// rotations must lie outside the shared-memory workspace, which the block
// items use (the SVD routines place both there when 2 n^2 doubles fit).
CATN_HD bool use_block(const Ctx& C, long long n, const double* X) {
#if CATN_LEAN
  (void)C; (void)n; (void)X;
  return false;
#endif
  if (cta_local(C, X) || 2 * n * n <= C.sws_doubles || n < C.block_min_n) return false;
  return C.P.svd_route == 2 || (C.P.svd_route == 0 && C.P.precision == 1);
}
// Whether the large-SVD routes of this release are selected (block route
// available, singular vectors formed only as far as the caller uses them);
// svd_route 1, and svd_route 0 in FP64, keep the earlier arithmetic bit for bit.
CATN_HD bool new_routes(const Ctx& C) {
#if CATN_LEAN
  (void)C;
  return false;
#endif
  return C.P.svd_route == 2 || (C.P.svd_route == 0 && C.P.precision == 1);
}
// Columns of U and V an SVD of nn values forms for its caller.
CATN_HD long long vec_cols(const Ctx& C, const SvdIn& s, long long nn) {
  return (new_routes(C) && s.need < nn) ? (s.need > 0 ? s.need : 1) : nn;
}
// The shared job for a block-route Jacobi (null: the owner's team alone):
// always with dedicated helper CTAs, otherwise once the queue is drained.
CATN_HDI inline JacobiJob* block_job(Ctx& C) {
  if (!C.job) return nullptr;
  if (C.job_pool) return C.job;
  long long drained = 0;
  if (C.T.leader()) drained = ldcg_i(C.qhead) >= C.ninst ? 1 : 0;
  return C.T.bcast(drained) != 0 ? C.job : nullptr;
}
// One-sided Jacobi of X (rows x n, ld) with V accumulated, on the route the
// parameters select.  Returns jacobi_sweeps' codes.
CATN_HDI inline int jacobi_any(Ctx& C, double* X, long long rows, long long n, long long ld, double* V,
                               double* nrm) {
  const long long t0 = clk();
  int sweeps;
  const bool blk = use_block(C, n, X) && !cta_local(C, V) && !cta_local(C, nrm);
  if (blk) {
    // precision 1: rotations stop at the rounding level of FP32 products
    const double floor_rel = C.P.precision == 1 ? 1e-8 : 0.0;
    sweeps = jacobi_block(C.T, block_job(C), X, rows, n, ld, V, 60, C.sws, floor_rel, C.P.precision == 1);
    prof_add(C, PROF_N_BLOCK, 1.0);
    prof_add(C, PROF_BLOCK_SWEEPS, (double)sweeps);
  } else {
    sweeps = share_jacobi(C, n, X, V, nrm) ? jacobi_sweeps_shared(C.T, C.job, X, rows, n, ld, V, 60, nrm)
                                   : jacobi_sweeps(C.T, X, rows, n, ld, V, 60, nrm);
  }
  if (X != C.sws) {
    const double dt = (double)(clk() - t0);
    prof_add(C, PROF_LJAC, dt);
    prof_add(C, PROF_LJAC_COLS, (double)n);
    if (blk) prof_add(C, PROF_LJAC_BLOCK, dt);
    if (n >= 1024) prof_add(C, PROF_LJAC_BIG, dt);
  }
  return sweeps;
}

// Split precision: the two-site merge of a large swap (M x N >= 2^18 outputs)
// as a 3xTF32 tensor-core product (tc_gemm_mop).  Returns false when the
// caller should take the FP64 GEMM (FP64 mode, small merges, no tensor-core
// area in this kernel); a tensor-core wait that ran out fails the instance.
constexpr long long kTcMergeMinElems = 1LL << 18;
CATN_HDI inline bool merge_on_tc(Ctx& C, long long M, long long N, long long K, const double* A, const double* B,
                                 const MOp& out) {
#if CATN_DEVICE_PASS && !CATN_LEAN
  if (C.P.precision != 1 || M * N < kTcMergeMinElems || !tc_ready(C.T)) return false;
  if (!tc_gemm_mop(C.T, M, N, K, A, M, B, K, out)) fail_all(C, CATN_ETIMEOUT);
  C.T.sync();
  return true;
#else
  (void)C; (void)M; (void)N; (void)K; (void)A; (void)B; (void)out;
  return false;
#endif
}

// Blocked application of Q: panel width and the smallest m x ncols product
// that takes it (with at least two panels of reflectors; below that the
// per-reflector passes are faster).
constexpr long long kQPanel = 32;
constexpr long long kBlockedQMinElems = 8192;
// qr_apply_q, shared when large; false when a shared wait ran out.
CATN_HDI inline bool apply_q_any(Ctx& C, const double* A, long long m, long long n, long long lda, const double* tau,
                                 double* Cm, long long ncols, long long ldc) {
  if (share_house(C, m, ncols, Cm, A)) {
    if (qr_apply_q_shared(C.T, C.job, A, m, n, lda, tau, Cm, ncols, ldc)) {
      fail_all(C, CATN_ETIMEOUT);
      return false;
    }
    return true;
  }
  // large products: reflectors in panels of kQPanel (three GEMMs per panel)
  // when the scratch stack has room, one reflector at a time otherwise
  if (n >= 2 * kQPanel && m * ncols >= kBlockedQMinElems) {
    const long long need = (m + 2 * ncols + 2 * kQPanel) * kQPanel;
    if (C.sp + 8 * need + 512 <= C.sp_hi) {
      const long long mark = C.sp;
      double* work = spush(C, need);
      qr_apply_q_blocked(C.T, A, m, n, lda, tau, Cm, ncols, ldc, kQPanel, work);
      C.sp = mark;
      return true;
    }
  }
  qr_apply_q(C.T, A, m, n, lda, tau, Cm, ncols, ldc);
  return true;
}
// apply_q_any with its cycles counted (large SVDs).
CATN_HDI inline bool apply_q(Ctx& C, const double* A, long long m, long long n, long long lda, const double* tau,
                             double* Cm, long long ncols, long long ldc) {
  const long long t0 = clk();
  const bool ok = apply_q_any(C, A, m, n, lda, tau, Cm, ncols, ldc);
  prof_add(C, PROF_LAPPLY, (double)(clk() - t0));
  return ok;
}
// qrcp_inplace, shared when large; -2 when a shared wait ran out.
CATN_HDI inline long long qrcp(Ctx& C, double* A, long long m, long long n, long long lda, double* tau, int* piv,
                               double* nrm, double stop_tol) {
  const long long t0 = clk();
  long long r;
  const long long work = m * n + (long long)kPanelW * m + 2048;
  if (new_routes(C) && n >= C.blocked_qr_min_n && !cta_local(C, A) && !cta_local(C, nrm) &&
      2 * n * n > C.sws_doubles &&
      C.sp + 8 * work + 4096 <= C.sp_hi) {
    // the blocked QR: columns sorted by norm, panels of 32 reflectors
    const long long mark = C.sp;
    double* w = spush(C, work);
    r = qr_sorted_blocked(C.T, block_job(C), A, m, n, lda, tau, piv, nrm, stop_tol, w, C.sws);
    C.sp = mark;
    if (r == -2) fail_all(C, CATN_ETIMEOUT);
  } else if (share_house(C, m, n, A, nrm)) {
    r = qrcp_shared(C.T, C.job, A, m, n, lda, tau, piv, nrm, stop_tol);
    if (r == -2) fail_all(C, CATN_ETIMEOUT);
  } else {
    r = qrcp_inplace(C.T, A, m, n, lda, tau, piv, nrm, stop_tol);
  }
  if (A != C.sws) prof_add(C, PROF_LQR, (double)(clk() - t0));
  return r;
}

// Large input whose pivoted QR W P = Q R stopped at rank r (trailing block
// dropped): SVD of the r x nn top block T = [R11 R12] P^T through its
// transpose (pivoted QR + Jacobi again), then U_W = Q1 * V_T, V_W = U_T.
CATN_HDI inline Svd svd_truncated(Ctx& C, const SvdIn& s, long long r, const double* tau, const int* piv,
                                  long long t0) {
  const Team& T = C.T;
  Svd R;
  R.m = s.m; R.n = s.n; R.p = 0; R.U = R.S = R.V = nullptr;
  const long long mm = s.mm, nn = s.nn;
  double* Tt = spush(C, nn * r);
  double* tau2 = spush(C, r);
  double* nrm2 = spush(C, r);
  int* piv2 = (int*)spush(C, r / 2 + 1);
  // the Jacobi pair lives in the shared-memory workspace when it fits (the
  // large path leaves it unused): its rounds are latency-bound in global memory
  const bool jsm = 2 * r * r <= C.sws_doubles;
  double* X2 = jsm ? C.sws : spush(C, r * r);
  double* Vb2 = jsm ? C.sws + r * r : spush(C, r * r);
  double* sig2 = spush(C, r);
  double* S2 = spush(C, r);
  int* perm2 = (int*)spush(C, r / 2 + 1);
  double* Uin = spush(C, nn * r);
  double* Vin = spush(C, r * r);
  double* Uw = spush(C, mm * r);
  if (failed(C)) return R;
  for (long long e = T.rank(); e < nn * r; e += T.size()) {
    long long j, i;   // Tt[piv[j], i] = R[i, j]
    divmod(e, nn, &j, &i);
    Tt[(long long)piv[j] + nn * i] = (j >= i) ? s.W[i + j * mm] : 0.0;
  }
  T.sync();
  if (qrcp(C, Tt, nn, r, nn, tau2, piv2, nrm2, 0.0) < 0) return R;
  for (long long e = T.rank(); e < r * r; e += T.size()) {
    long long i, j;
    divmod(e, r, &i, &j);
    X2[e] = (j <= i) ? Tt[j + i * nn] : 0.0;
  }
  T.sync();
  int sweeps = jacobi_any(C, X2, r, r, r, Vb2, nrm2);
  if (sweeps < 0) fail_all(C, sweeps == -2 ? CATN_ETIMEOUT : CATN_ENOCONV);
  if (T.leader() && sweeps > C.ctl[CTL_JACMAX]) C.ctl[CTL_JACMAX] = sweeps;
  sort_columns(T, X2, r, r, r, sig2, S2, perm2);
  const long long nv = vec_cols(C, s, r);   // singular vectors formed
  for (long long e = T.rank(); e < nn * nv; e += T.size()) {
    long long rr, c;
    divmod(e, nn, &rr, &c);
    Uin[e] = (rr < r) ? Vb2[rr + (long long)perm2[c] * r] : 0.0;
  }
  for (long long e = T.rank(); e < r * nv; e += T.size()) {
    long long i, c;
    divmod(e, r, &i, &c);
    double sv = S2[c];
    Vin[(long long)piv2[i] + c * r] = (sv > 0.0) ? X2[i + (long long)perm2[c] * r] / sv : 0.0;
  }
  T.sync();
  if (!apply_q(C, Tt, nn, r, nn, tau2, Uin, nv, nn)) return R;
  for (long long e = T.rank(); e < mm * nv; e += T.size()) {
    long long rr, c;
    divmod(e, mm, &rr, &c);
    Uw[e] = (rr < r) ? Vin[rr + c * r] : 0.0;
  }
  T.sync();
  if (!apply_q(C, s.W, mm, r, mm, tau, Uw, nv, mm)) return R;
  prof_add(C, PROF_SVD_LARGE, (double)(clk() - t0));
  prof_add(C, PROF_N_LARGE, 1.0);
  R.p = r;
  R.S = S2;
  if (!s.wide) {
    R.U = Uw;
    R.V = Uin;
  } else {
    R.U = Uin;
    R.V = Uw;
  }
  return R;
}

// Drmac-Veselic preconditioned one-sided Jacobi: pivoted Householder QR
// W P = Q R, one-sided Jacobi on X = R^T (X V' = U' Sigma), so that
// W = (Q V') Sigma (P U')^T.  The pivoted, transposed triangle converges in
// a handful of sweeps even for strongly graded spectra.
CATN_HDI inline Svd svd_finish(Ctx& C, const SvdIn& s) {
  const Team& T = C.T;
  Svd R;
  R.m = s.m; R.n = s.n; R.p = 0; R.U = R.S = R.V = nullptr;
  if (failed(C) || !s.W) return R;
  const long long t0 = clk();
  const long long mm = s.mm, nn = s.nn;
  double *X, *Vb, *Ut, *Vt, *tau, *nrm, *sig, *Sout;
  int *piv, *perm;
  if (s.smem) {
    double* q = s.W + mm * nn;
    X = q; q += nn * nn;
    Vb = q; q += nn * nn;
    Vt = q; q += nn * nn;
    Ut = q; q += mm * nn;
    tau = q; q += nn;
    nrm = q; q += nn;
    sig = q; q += nn;
    Sout = q; q += nn;
    piv = (int*)q; q += (nn + 1) / 2 + 1;
    perm = (int*)q;
  } else {
    tau = spush(C, nn);
    nrm = spush(C, nn);
    piv = (int*)spush(C, (nn + 1) / 2 + 1);
    X = Vb = Vt = Ut = sig = Sout = nullptr;
    perm = nullptr;
    if (failed(C)) return R;
  }
#if CATN_DEVICE_PASS
  if (s.smem && nn <= 16 && mm <= 64) {
    // tiny problem: one warp, warp-level synchronisation only
    int sweeps = 0;
    if (T.warp() == 0)
      sweeps = svd_warp_tiny_any(s.W, (int)mm, (int)nn, tau, piv, Ut, Vt, Sout, 60);
    T.sync();
    if (T.leader()) {
      if (sweeps > C.ctl[CTL_JACMAX]) C.ctl[CTL_JACMAX] = sweeps;
      C.ctl[CTL_BCAST] = sweeps;
    }
    T.sync();
    if (C.ctl[CTL_BCAST] < 0) fail_all(C, CATN_ENOCONV);
    T.sync();
    prof_add(C, PROF_SVD_TINY, (double)(clk() - t0));
    prof_add(C, PROF_N_TINY, 1.0);
    R.p = nn;
    R.S = Sout;
    if (!s.wide) { R.U = Ut; R.V = Vt; } else { R.U = Vt; R.V = Ut; }
    return R;
  }
#endif
  double stop = 0.0;
  if (!s.smem && s.tol > 0.0) {
    // truncate only when the matrix is far above the tolerance, so that the
    // "keep everything when nothing passes the cutoff" rule never meets a
    // truncated factorisation
    double f2 = 0.0;
    for (long long e = T.rank(); e < mm * nn; e += T.size()) f2 = fma(s.W[e], s.W[e], f2);
    f2 = T.sum(f2);
    if (sqrt(f2) > 1e6 * s.tol) stop = s.tol;
  }
  const long long r = qrcp(C, s.W, mm, nn, mm, tau, piv, nrm, stop);
  if (r < 0) return R;
  if (r < nn) return svd_truncated(C, s, r, tau, piv, t0);
  if (!s.smem) {
    const bool jsm = 2 * nn * nn <= C.sws_doubles;   // Jacobi pair in shared memory when it fits
    X = jsm ? C.sws : spush(C, nn * nn);
    Vb = jsm ? C.sws + nn * nn : spush(C, nn * nn);
    Vt = spush(C, nn * nn);
    Ut = spush(C, mm * nn);
    sig = spush(C, nn);
    Sout = spush(C, nn);
    perm = (int*)spush(C, (nn + 1) / 2 + 1);
    if (failed(C)) return R;
  }
  for (long long e = T.rank(); e < nn * nn; e += T.size()) {
    long long i, j;
    divmod(e, nn, &i, &j);
    X[e] = (j <= i) ? s.W[j + i * mm] : 0.0;   // X = R^T
  }
  T.sync();
  int sweeps = jacobi_any(C, X, nn, nn, nn, Vb, nrm);
  if (sweeps < 0) fail_all(C, sweeps == -2 ? CATN_ETIMEOUT : CATN_ENOCONV);
  if (T.leader() && sweeps > C.ctl[CTL_JACMAX]) C.ctl[CTL_JACMAX] = sweeps;
  sort_columns(T, X, nn, nn, nn, sig, Sout, perm);
  const long long nv = vec_cols(C, s, nn);   // singular vectors formed
  for (long long e = T.rank(); e < mm * nv; e += T.size()) {
    long long r, c;
    divmod(e, mm, &r, &c);
    Ut[e] = (r < nn) ? Vb[r + (long long)perm[c] * nn] : 0.0;
  }
  for (long long e = T.rank(); e < nn * nv; e += T.size()) {
    long long i, c;
    divmod(e, nn, &i, &c);
    double sv = Sout[c];
    Vt[(long long)piv[i] + c * nn] = (sv > 0.0) ? X[i + (long long)perm[c] * nn] / sv : 0.0;
  }
  T.sync();
  if (!apply_q(C, s.W, mm, nn, mm, tau, Ut, nv, mm)) return R;
  prof_add(C, s.smem ? PROF_SVD_SMALL : PROF_SVD_LARGE, (double)(clk() - t0));
  prof_add(C, s.smem ? PROF_N_SMALL : PROF_N_LARGE, 1.0);
  R.p = nn;
  R.S = Sout;
  if (!s.wide) {
    R.U = Ut;
    R.V = Vt;
  } else {
    R.U = Vt;
    R.V = Ut;
  }
  return R;
}

// tsvd keep rule (linalg_utils.jl:22-26): nkeep = count(S > cutoff), 0 -> 1,
// capped by maxdim; *disc = sum of the discarded singular values.
CATN_HDI inline int keep_rule(Ctx& C, const Svd& R, double cutoff, long long maxdim, double* disc) {
  const Team& T = C.T;
  const double* S = R.S;
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
  double cnt = 0.0;
  for (long long e = T.rank(); e < R.p; e += T.size()) cnt += (R.S[e] > cutoff) ? 1.0 : 0.0;
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
      const long long mark = C.sp;
      SiteRef s = sref(C, k, i);
      const long long m = (long long)s.dl * s.d, n = s.dr;
      SvdIn in = svd_begin(C, m, n, C.P.cutoff);
      if (failed(C)) return;
      svd_fill(C, in, colmajor(sdata(C, s), m));
      Svd R = svd_finish(C, in);
      if (failed(C)) return;
      const long long te = clk();
      const int nkeep = keep_all_if_none(C, R, C.P.cutoff);
      SiteRef nx = sref(C, k, i + 1);
      const long long tb = C.tape ? al256(8LL * nkeep) + al256(8 * n * nkeep) : 0;
      if (!heap_reserve(C, al256(8 * m * nkeep) + al256(8LL * nkeep * nx.d * nx.dr) + tb)) return;
      nx = sref(C, k, i + 1);
      const long long ni = heap_take(C, 8 * m * nkeep);
      const long long nn2 = heap_take(C, 8LL * nkeep * nx.d * nx.dr);
      if (C.tape) {
        TapeRec r = trec(OP_CANO_R);
        r.a[0] = s.dl; r.a[1] = s.d; r.a[2] = s.dr; r.a[3] = nkeep; r.a[4] = nx.d; r.a[5] = nx.dr;
        r.o[0] = s.off; r.o[1] = nx.off; r.o[2] = ni; r.o[3] = nn2;
        r.o[4] = heap_take(C, 8LL * nkeep);
        r.o[5] = heap_take(C, 8 * n * nkeep);
        copy(T, dptr(C, r.o[4]), R.S, nkeep);
        copy(T, dptr(C, r.o[5]), R.V, n * nkeep);
        tape_push(C, r);
      }
      copy(T, dptr(C, ni), R.U, m * nkeep);
      // next <- (S V^H)[1:nkeep, :] * next
      gemm(T, nkeep, (long long)nx.d * nx.dr, n, mop(R.V, imap(1, 0, n), rows_plain(), R.S, nullptr),
           colmajor(sdata(C, nx), n), colmajor(dptr(C, nn2), nkeep));
      account(C, 2.0 * m * n * n + 2.0 * n * n * nx.d * nx.dr,
              8.0 * (m * n + (double)n * nx.d * nx.dr + m * nkeep + (double)nkeep * nx.d * nx.dr));
      if (T.leader()) {
        sref(C, k, i) = mksite(s.dl, s.d, nkeep, ni);
        sref(C, k, i + 1) = mksite(nkeep, nx.d, nx.dr, nn2);
        C.node[k].cano = i + 1;
      }
      T.sync();
      C.sp = mark;
      prof_add(C, PROF_CANO_EPI, (double)(clk() - te));
    }
  } else {
    for (int i = h.cano; i > idx; --i) {
      if (failed(C)) return;
      const long long mark = C.sp;
      SiteRef s = sref(C, k, i);
      const long long dl = s.dl, m = (long long)s.d * s.dr;
      // Mt = permutedims(site, (2,3,1)) as (d*dr) x dl = transpose of the dl x (d*dr) view
      SvdIn in = svd_begin(C, m, dl, C.P.cutoff);
      if (failed(C)) return;
      svd_fill(C, in, transposed(sdata(C, s), dl));
      Svd R = svd_finish(C, in);
      if (failed(C)) return;
      const long long te = clk();
      const int nkeep = keep_all_if_none(C, R, C.P.cutoff);
      SiteRef pv = sref(C, k, i - 1);
      const long long tb = C.tape ? al256(8LL * nkeep) + al256(8 * dl * nkeep) : 0;
      if (!heap_reserve(C, al256(8 * m * nkeep) + al256(8LL * pv.dl * pv.d * nkeep) + tb)) return;
      pv = sref(C, k, i - 1);
      const long long ni = heap_take(C, 8 * m * nkeep);
      const long long np = heap_take(C, 8LL * pv.dl * pv.d * nkeep);
      if (C.tape) {
        TapeRec r = trec(OP_CANO_L);
        r.a[0] = s.dl; r.a[1] = s.d; r.a[2] = s.dr; r.a[3] = nkeep; r.a[4] = pv.dl; r.a[5] = pv.d;
        r.o[0] = s.off; r.o[1] = pv.off; r.o[2] = ni; r.o[3] = np;
        r.o[4] = heap_take(C, 8LL * nkeep);
        r.o[5] = heap_take(C, 8 * dl * nkeep);
        copy(T, dptr(C, r.o[4]), R.S, nkeep);
        copy(T, dptr(C, r.o[5]), R.V, dl * nkeep);
        tape_push(C, r);
      }
      // new site = permutedims(reshape(U[:, 1:nkeep], d, dr, nkeep), (3,1,2)) = U^T
      materialize(T, dptr(C, ni), nkeep, m, nkeep, transposed(R.U, m));
      // prev <- prev * (S V^H)^T
      gemm(T, (long long)pv.dl * pv.d, nkeep, dl, colmajor(sdata(C, pv), (long long)pv.dl * pv.d),
           mop(R.V, rows_plain(), cols_plain(dl), nullptr, R.S), colmajor(dptr(C, np), (long long)pv.dl * pv.d));
      account(C, 2.0 * m * dl * dl + 2.0 * dl * dl * pv.dl * pv.d,
              8.0 * (m * dl + (double)pv.dl * pv.d * dl + m * nkeep + (double)pv.dl * pv.d * nkeep));
      if (T.leader()) {
        sref(C, k, i) = mksite(nkeep, s.d, s.dr, ni);
        sref(C, k, i - 1) = mksite(pv.dl, pv.d, nkeep, np);
        C.node[k].cano = i - 1;
      }
      T.sync();
      C.sp = mark;
      prof_add(C, PROF_CANO_EPI, (double)(clk() - te));
    }
  }
}

// ---------------------------------------------------------------------------
// Thin Q (m x min(m, c)) of the Householder QR of A (m x c, m >= c,
// overwritten by the factorisation).
CATN_HDI inline bool thin_q(Ctx& C, double* A, long long m, long long c, double* tau, double* Q) {
  const Team& T = C.T;
  qr_inplace(T, A, m, c, m, tau);
  for (long long e = T.rank(); e < m * c; e += T.size()) {
    long long r, j;
    divmod(e, m, &r, &j);
    Q[e] = (r == j) ? 1.0 : 0.0;
  }
  T.sync();
  return apply_q(C, A, m, c, m, tau, Q, c, m);
}

// The reference's randomized SVD (linalg_utils.jl:44-58) of the swap
// matrix M (m x n, the oriented input `in`), with its Gaussian sketch from
// the counter-based generator keyed by (P.seed, this instance's call
// count): G (n x p, p = min(n, 10 k)), Y = M G, ten rounds of Y <- thin Q
// of M (M^T Y), Q = thin Q of Y, B = Q^T M = Ub S Vb^T (exact), U = Q Ub;
// the first min(k, rank B) triplets.  Needs m >= p (the thin Q of a wide
// sketch is not formed; the caller takes the exact route then).
CATN_HDI inline Svd rsvd_swap(Ctx& C, const SvdIn& in, long long m, long long n, long long k) {
  const Team& T = C.T;
  Svd R;
  R.m = m; R.n = n; R.p = 0; R.U = R.S = R.V = nullptr;
  // M out of the shared-memory workspace, which the SVD of B reuses
  double* Wm = in.W;
  if (in.smem) {
    Wm = spush(C, m * n);
    if (failed(C)) return R;
    copy(T, Wm, in.W, m * n);
  }
  const MOp M = in.wide ? transposed(Wm, in.mm) : colmajor(Wm, in.mm);
  const MOp Mt = in.wide ? colmajor(Wm, in.mm) : transposed(Wm, in.mm);
  const long long p = n < 10 * k ? n : 10 * k;
  double* G = spush(C, n * p);
  double* Y = spush(C, m * p);
  double* Z = spush(C, n * p);
  double* Qm = spush(C, m * p);
  double* tau = spush(C, p);
  if (failed(C)) return R;
  const unsigned long long key = (unsigned long long)(unsigned)C.P.seed;
  const unsigned long long stream = 16ULL + (unsigned long long)C.rsvd_calls;
  C.rsvd_calls += 1;   // every thread keeps the same count
  for (long long e = T.rank(); e < n * p; e += T.size()) G[e] = disorder_normal(key, stream, (unsigned long long)e);
  T.sync();
  gemm(T, m, p, n, M, colmajor(G, n), colmajor(Y, m));
  for (int it = 0; it < 10; ++it) {
    gemm(T, n, p, m, Mt, colmajor(Y, m), colmajor(Z, n));   // Z = M^T Y
    gemm(T, m, p, n, M, colmajor(Z, n), colmajor(Y, m));    // Y = M Z
    if (!thin_q(C, Y, m, p, tau, Qm)) return R;
    copy(T, Y, Qm, m * p);
  }
  if (!thin_q(C, Y, m, p, tau, Qm)) return R;              // Q (m x p)
  SvdIn bin = svd_begin(C, p, n, 0.0);
  if (failed(C)) return R;
  gemm(T, p, n, m, transposed(Qm, m), M, svd_target(bin));  // B = Q^T M
  Svd F = svd_finish(C, bin);
  if (failed(C) || !F.U) return R;
  const long long kk = F.p < k ? F.p : k;
  double* U = spush(C, m * kk);
  if (failed(C)) return R;
  gemm(T, m, kk, p, colmajor(Qm, m), colmajor(F.U, p), colmajor(U, m));
  R.p = kk;
  R.U = U;
  R.S = F.S;
  R.V = F.V;
  return R;
}

// Matrix-free products with the swap matrix M = reshape(ein"ijk,kab->iajb"(tl,
// tr), d0 d1, d2 d3) (tl: d0 x d2 x kk, tr: kk x d1 x d3, column-major), M
// never formed: M[(i,a), (j,b)] = sum_k tl[i,j,k] tr[k,a,b], rows i + d0 a,
// columns j + d2 b.  X is (d0 kk d3 p) doubles of workspace.
// Y (m x p) = M G, G (n x p): X[(i,k), (b,c)] = sum_j tl[i,j,k] G[(j,b), c],
// then Y[(i,a), c] = sum_(k,b) X[(i,k), (b,c)] tr[k,a,b].
CATN_HDI inline void mf_apply(const Team& T, const double* tl, const double* tr, long long d0, long long d1,
                              long long d2, long long d3, long long kk, const double* G, long long p, double* X,
                              double* Y) {
  const long long m = d0 * d1, n = d2 * d3;
  gemm(T, d0 * kk, d3 * p, d2, mop((double*)tl, imap((int)d0, 1, d0 * d2), imap(1, 0, d0)),
       mop((double*)G, rows_plain(), imap((int)d3, d2, n)), colmajor(X, d0 * kk));
  gemm(T, d0 * p, d1, kk * d3, mop(X, imap((int)d0, 1, d0 * kk * d3), imap((int)kk, d0, d0 * kk)),
       mop((double*)tr, imap((int)kk, 1, kk * d1), imap(1, 0, kk)), mop(Y, imap((int)d0, 1, m), imap(1, 0, d0)));
}
// Z (n x p) = M^T Y, Y (m x p): X[(i,c), (k,b)] = sum_a Y[(i,a), c] tr[k,a,b],
// then Z[(j,b), c] = sum_(i,k) tl[i,j,k] X[(i,c), (k,b)].
CATN_HDI inline void mf_apply_t(const Team& T, const double* tl, const double* tr, long long d0, long long d1,
                                long long d2, long long d3, long long kk, const double* Y, long long p, double* X,
                                double* Z) {
  const long long m = d0 * d1, n = d2 * d3;
  gemm(T, d0 * p, kk * d3, d1, mop((double*)Y, imap((int)d0, 1, m), imap(1, 0, d0)),
       mop((double*)tr, imap(1, 0, kk), imap((int)kk, 1, kk * d1)), colmajor(X, d0 * p));
  gemm(T, d2, d3 * p, d0 * kk, mop((double*)tl, imap(1, 0, d0), imap((int)d0, 1, d0 * d2)),
       mop(X, imap((int)d0, 1, d0 * p), imap((int)d3, d0 * p * kk, d0)), mop(Z, rows_plain(), imap((int)d3, d2, n)));
}

// rsvd_swap with the products of M applied from (tl, tr) (catn_params.rsvd
// = 2): the same sketch, power iterations, thin Qs and projected SVD, for
// swap matrices too large to hold (M of (chi Dmax)^2 doubles); B = Q^T M is
// formed as (M^T Q)^T.  Its workspace is O((m + n + d0 kk d3) p).
CATN_HDI inline Svd rsvd_swap_mf(Ctx& C, const double* tl, const double* tr, long long d0, long long d1, long long d2,
                                 long long d3, long long kk, long long k) {
  const Team& T = C.T;
  const long long m = d0 * d1, n = d2 * d3;
  Svd R;
  R.m = m; R.n = n; R.p = 0; R.U = R.S = R.V = nullptr;
  const long long p = n < 10 * k ? n : 10 * k;
  double* G = spush(C, n * p);
  double* Y = spush(C, m * p);
  double* Z = spush(C, n * p);
  double* Qm = spush(C, m * p);
  double* tau = spush(C, p);
  double* X = spush(C, d0 * kk * d3 * p);
  if (failed(C)) return R;
  const unsigned long long key = (unsigned long long)(unsigned)C.P.seed;
  const unsigned long long stream = 16ULL + (unsigned long long)C.rsvd_calls;
  C.rsvd_calls += 1;   // every thread keeps the same count
  for (long long e = T.rank(); e < n * p; e += T.size()) G[e] = disorder_normal(key, stream, (unsigned long long)e);
  T.sync();
  mf_apply(T, tl, tr, d0, d1, d2, d3, kk, G, p, X, Y);
  for (int it = 0; it < 10; ++it) {
    mf_apply_t(T, tl, tr, d0, d1, d2, d3, kk, Y, p, X, Z);   // Z = M^T Y
    mf_apply(T, tl, tr, d0, d1, d2, d3, kk, Z, p, X, Y);     // Y = M Z
    if (!thin_q(C, Y, m, p, tau, Qm)) return R;
    copy(T, Y, Qm, m * p);
  }
  if (!thin_q(C, Y, m, p, tau, Qm)) return R;              // Q (m x p)
  mf_apply_t(T, tl, tr, d0, d1, d2, d3, kk, Qm, p, X, Z);   // Z = M^T Q (n x p)
  SvdIn bin = svd_begin(C, p, n, 0.0);
  if (failed(C)) return R;
  {
    const MOp Bt = svd_target(bin);   // B (p x n) = Z^T
    for (long long e = T.rank(); e < p * n; e += T.size()) {
      long long r, c;
      divmod(e, p, &r, &c);
      Bt.ref(r, c) = Z[c + n * r];
    }
    T.sync();
  }
  Svd F = svd_finish(C, bin);
  if (failed(C) || !F.U) return R;
  const long long kq = F.p < k ? F.p : k;
  double* U = spush(C, m * kq);
  if (failed(C)) return R;
  gemm(T, m, kq, p, colmajor(Qm, m), colmajor(F.U, p), colmajor(U, m));
  R.p = kq;
  R.U = U;
  R.S = F.S;
  R.V = F.V;
  return R;
}

// swap! (mps_node.jl:126-178)
// ---------------------------------------------------------------------------
CATN_HDI inline double swap(Ctx& C, int k, int i, int j) {
  const Team& T = C.T;
  NodeHdr h = C.node[k];
  int dij = i - j;
  if ((dij != 1 && dij != -1) || i < 1 || j < 1 || i > h.nsites || j > h.nsites) {
    fail_all(C, CATN_ESTATE);
    return 0.0;
  }
  if (h.cano != i && h.cano != j) {
    int ai = h.cano - i, aj = h.cano - j;
    ai = ai < 0 ? -ai : ai;
    aj = aj < 0 ? -aj : aj;
    cano_to(C, k, ai < aj ? i : j);
    if (failed(C)) return 0.0;
  }
  const long long mark = C.sp;
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  SiteRef tl = sref(C, k, lo), tr = sref(C, k, hi);
  const long long d0 = tl.dl, d1 = tr.d, d2 = tl.d, d3 = tr.dr, kk = tl.dr;
  const long long m = d0 * d1, n = d2 * d3;
  const long long rmin = C.rsvd_min > 0 ? C.rsvd_min : 7000, rbig = C.rsvd_min > 0 ? 3LL * C.rsvd_min : 20000;
  const bool rsvd_route = C.P.swapopt && ((m > rmin && n > rmin) || m > rbig || n > rbig);
  // the reference's randomized algorithm on request (forward runs, sketch no
  // wider than M); otherwise the exact top-chi subspace it approximates
  const bool randomized = rsvd_route && C.P.rsvd >= 1 && !C.tape && m >= (n < 10LL * C.P.chi ? n : 10LL * C.P.chi);
  // rsvd = 2: the same algorithm with M applied from (tl, tr), never formed
  const bool matfree = !CATN_LEAN && randomized && C.P.rsvd == 2;
  SvdIn in = SvdIn();
  if (!matfree) {
    in = svd_begin(C, m, n, rsvd_route ? 0.0 : C.P.cutoff);
    if (failed(C)) return 0.0;
    in.need = C.P.chi;   // keep_rule and the randomized route keep at most chi
  }
  // W = ein"ijk,kab->iajb"(tl, tr); M = reshape(W, d0*d1, d2*d3), written
  // straight into the SVD's oriented input.
  if (!matfree) {
    const long long tg = clk();
    MOp out = in.wide ? mop(in.W, imap((int)d0, n, 1), imap((int)d1, n * d0, d2))
                      : mop(in.W, imap((int)d0, 1, d0 * d1), imap((int)d1, d0, d0 * d1 * d2));
    if (!merge_on_tc(C, d0 * d2, d1 * d3, kk, sdata(C, tl), sdata(C, tr), out))
      gemm(T, d0 * d2, d1 * d3, kk, colmajor(sdata(C, tl), d0 * d2), colmajor(sdata(C, tr), kk), out);
    prof_add(C, PROF_SWAP_GEMM, (double)(clk() - tg));
  }
  Svd R = matfree      ? rsvd_swap_mf(C, sdata(C, tl), sdata(C, tr), d0, d1, d2, d3, kk, C.P.chi)
          : randomized ? rsvd_swap(C, in, m, n, C.P.chi)
                       : svd_finish(C, in);
  if (failed(C)) return 0.0;
  const long long te = clk();
  double err = 0.0;
  int myd;
  if (rsvd_route) {
    // The reference's randomized route keeps min(chi, rank) vectors with no
    // cutoff and reports zero error (mps_node.jl:154-156): its randomized
    // algorithm with P.rsvd = 1 (rsvd_swap), else the exact top-chi subspace
    // it approximates.
    myd = (int)(R.p < C.P.chi ? R.p : C.P.chi);
  } else {
    myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &err);
  }
  const long long tb = C.tape ? al256(8LL * myd) + al256(8 * (i < j ? n : m) * myd) : 0;
  if (!heap_reserve(C, al256(8 * m * myd) + al256(8 * n * myd) + tb)) return err;
  const long long nl = heap_take(C, 8 * m * myd);
  const long long nr = heap_take(C, 8 * n * myd);
  if (C.tape) {
    // i < j stores U verbatim and S V^H; i > j stores U S and V^H verbatim:
    // keep S and the factor that is not stored as it is
    TapeRec r = trec(OP_SWAP);
    r.a[0] = (int)d0; r.a[1] = (int)d1; r.a[2] = (int)d2; r.a[3] = (int)d3; r.a[4] = (int)kk; r.a[5] = myd;
    r.a[6] = i < j;
    r.o[0] = tl.off; r.o[1] = tr.off; r.o[2] = nl; r.o[3] = nr;
    r.o[4] = heap_take(C, 8LL * myd);
    r.o[5] = heap_take(C, 8 * (i < j ? n : m) * myd);
    copy(T, dptr(C, r.o[4]), R.S, myd);
    copy(T, dptr(C, r.o[5]), i < j ? R.V : R.U, (i < j ? n : m) * myd);
    tape_push(C, r);
  }
  if (i < j) {
    copy(T, dptr(C, nl), R.U, m * myd);
    materialize(T, dptr(C, nr), myd, n, myd, mop(R.V, imap(1, 0, n), rows_plain(), R.S, nullptr));
  } else {
    materialize(T, dptr(C, nl), m, myd, m, mop(R.U, rows_plain(), cols_plain(m), nullptr, R.S));
    materialize(T, dptr(C, nr), myd, n, myd, mop(R.V, imap(1, 0, n), rows_plain()));
  }
  account(C, 2.0 * m * n * kk + 4.0 * m * n * myd,
          8.0 * ((double)d0 * d2 * kk + (double)kk * d1 * d3 + (double)m * myd + (double)myd * n));
  if (T.leader()) {
    sref(C, k, lo) = mksite((int)d0, (int)d1, myd, nl);
    sref(C, k, hi) = mksite(myd, (int)d2, (int)d3, nr);
    C.node[k].cano = j;
    int t = nbref(C, k, i);
    nbref(C, k, i) = nbref(C, k, j);
    nbref(C, k, j) = t;
  }
  T.sync();
  C.sp = mark;
  prof_add(C, PROF_SWAP_EPI, (double)(clk() - te));
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
  const long long tr0 = clk();
  const int ns = h.nsites;
  long long total = 0;
  for (int p = 1; p <= ns; ++p) total += al256(sbytes(sref(C, k, p)));
  if (!heap_reserve(C, total)) return;
  const long long first = C.hb;
  C.hb += total;
  {
    long long used = C.hb - (C.half ? C.h_lo1 : C.h_lo0);
    if (used > C.h_peak) C.h_peak = used;
  }
  long long cur = first;
  for (int p = 1; p <= ns; ++p) {
    SiteRef s = sref(C, k, p);
    const double* src = sdata(C, s);
    double* dst = dptr(C, cur);
    const long long dl = s.dl, d = s.d, dr = s.dr, tot = dl * d * dr;
    for (long long e = T.rank(); e < tot; e += T.size()) {
      long long a, rest, b, c;
      divmod(e, dl, &a, &rest);
      divmod(rest, d, &b, &c);
      dst[c + dr * (b + d * a)] = src[e];
    }
    cur += al256(8 * tot);
  }
  T.sync();
  if (C.tape) {
    long long c2 = first;
    for (int p = 1; p <= ns; ++p) {
      const SiteRef s = sref(C, k, p);
      TapeRec r = trec(OP_REVERSE);
      r.a[0] = s.dl; r.a[1] = s.d; r.a[2] = s.dr;
      r.o[0] = s.off; r.o[1] = c2;
      tape_push(C, r);
      c2 += al256(sbytes(s));
    }
    T.sync();
  }
  if (T.leader()) {
    // old site p was copied (transposed) to `first + sum of earlier sizes`;
    // it becomes position ns + 1 - p
    SiteRef* old = (SiteRef*)C.pairs;
    for (int p = 1; p <= ns; ++p) old[p - 1] = sref(C, k, p);
    long long c2 = first;
    for (int p = 1; p <= ns; ++p) {
      const SiteRef s = old[p - 1];
      sref(C, k, ns + 1 - p) = mksite(s.dr, s.d, s.dl, c2);
      c2 += al256(sbytes(s));
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
  prof_add(C, PROF_REVERSE, (double)(clk() - tr0));
}

// clear! (mps_node.jl:335-339)
CATN_HDI inline void clear_node(Ctx& C, int k) {
  C.T.sync();
  if (C.T.leader()) {
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
    fail_all(C, CATN_ESTATE);
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
  const long long tf = clk();
  SiteRef a = sref(C, k, idx1), b = sref(C, k, idx1 + 1);
  const long long rows = (long long)a.dl * a.d, cols = (long long)b.d * b.dr;
  if (!heap_reserve(C, al256(8 * rows * cols))) return err;
  a = sref(C, k, idx1);
  b = sref(C, k, idx1 + 1);
  const long long f = heap_take(C, 8 * rows * cols);
  gemm(T, rows, cols, a.dr, colmajor(sdata(C, a), rows), colmajor(sdata(C, b), a.dr), colmajor(dptr(C, f), rows));
  if (C.tape) {
    TapeRec r = trec(OP_MERGE);
    r.a[0] = a.dl; r.a[1] = a.d; r.a[2] = a.dr; r.a[3] = b.d; r.a[4] = b.dr;
    r.o[0] = a.off; r.o[1] = b.off; r.o[2] = f;
    tape_push(C, r);
  }
  account(C, 2.0 * rows * a.dr * cols, 8.0 * ((double)rows * a.dr + (double)a.dr * cols + (double)rows * cols));
  if (T.leader()) {
    sref(C, k, idx1) = mksite(a.dl, a.d * b.d, b.dr, f);
    site_delete_at_leader(C, k, idx1 + 1);
  }
  T.sync();
  prof_add(C, PROF_MERGE, (double)(clk() - tf));
  cano_to(C, k, idx1);
  return err;
}

// Divide site (k, pos) by nrm.  A gradient run writes the quotient as a new
// recorded version (same arithmetic as the in-place scale).
CATN_HDI inline bool normalize_site(Ctx& C, int k, int pos, double nrm) {
  const Team& T = C.T;
  SiteRef s = sref(C, k, pos);
  const long long len = (long long)s.dl * s.d * s.dr;
  if (!C.tape || C.P.norm_method == 0) {
    scale(T, sdata(C, s), 1.0 / nrm, len);
    return true;
  }
  if (!heap_reserve(C, al256(8 * len))) return false;
  const long long xo = heap_take(C, 8 * len);
  const double inv = 1.0 / nrm;
  const double* x = sdata(C, s);
  double* y = dptr(C, xo);
  for (long long e = T.rank(); e < len; e += T.size()) y[e] = x[e] * inv;
  T.sync();
  TapeRec r = trec(OP_NORM);
  r.a[0] = (int)len; r.a[1] = C.P.norm_method;
  r.o[0] = s.off; r.o[1] = xo;
  r.v[0] = nrm;
  tape_push(C, r);
  if (T.leader()) sref(C, k, pos).off = xo;
  T.sync();
  return true;
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
    if (C.node[kj].nsites != 1) { fail_all(C, CATN_ESTATE); return 0.0; }
    SiteRef si = sref(C, ki, 1), sj = sref(C, kj, 1);
    long long d = si.d;
    double loc = 0.0;
    const double* vi = sdata(C, si);
    const double* vj = sdata(C, sj);
    for (long long e = T.rank(); e < d; e += T.size()) loc = fma(vi[e], vj[e], loc);
    double r = T.sum(loc);
    double absr = fabs(r);
    if (C.tape) {
      TapeRec q = trec(OP_EAT_A);
      q.a[0] = (int)d; q.o[0] = si.off; q.o[1] = sj.off; q.v[0] = r; q.flag = absr > cutoff;
      tape_push(C, q);
    }
    T.sync();
    if (T.leader()) {
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
  const long long mark = C.sp;
  if (C.node[kj].nsites == 1) {
    // (b) j is a leaf: mat = mati * matj, folded into mps[end-1]
    SiteRef last = sref(C, ki, hi.nsites), tj = sref(C, kj, 1);
    double* vbuf = spush(C, last.dl);
    if (failed(C)) return 0.0;
    gemm(T, last.dl, 1, last.d, colmajor(sdata(C, last), last.dl), colmajor(sdata(C, tj), last.d),
         colmajor(vbuf, last.dl));
    SiteRef prev = sref(C, ki, hi.nsites - 1);
    const long long ne = (long long)prev.dl * prev.d;
    if (!heap_reserve(C, al256(8 * ne))) return 0.0;
    prev = sref(C, ki, hi.nsites - 1);
    const long long nt = heap_take(C, 8 * ne);
    gemm(T, ne, 1, prev.dr, colmajor(sdata(C, prev), ne), colmajor(vbuf, prev.dr), colmajor(dptr(C, nt), ne));
    if (C.tape) {
      TapeRec q = trec(OP_EAT_B);
      q.a[0] = last.dl; q.a[1] = last.d; q.a[2] = (int)ne;
      q.o[0] = last.off; q.o[1] = tj.off; q.o[2] = prev.off; q.o[3] = nt;
      tape_push(C, q);
    }
    account(C, 2.0 * last.dl * last.d + 2.0 * ne * prev.dr, 8.0 * ((double)last.dl * last.d + ne * prev.dr + ne));
    const double nrm = norm_of(C, dptr(C, nt), ne);
    if (T.leader()) {
      sref(C, ki, hi.nsites - 1) = mksite(prev.dl, prev.d, 1, nt);
      C.node[ki].cano = C.node[ki].cano - 1;
      C.node[ki].nsites = hi.nsites - 1;
      C.node[ki].nnbr = C.node[ki].nnbr - 1;
    }
    T.sync();
    C.sp = mark;
    if (nrm <= cutoff) return 0.0;
    if (!normalize_site(C, ki, hi.nsites - 1, nrm)) return 0.0;
    return log(nrm);
  }
  // (c) general
  *err += move2head(C, kj, idxi);
  if (failed(C)) return 0.0;
  const long long tf = clk();
  SiteRef last = sref(C, ki, hi.nsites);   // (Dl, dd, 1)
  SiteRef hj = sref(C, kj, 1);              // (1, dd, Dr)
  const long long Dl = last.dl, dd = last.d, Dr = hj.dr;
  double* mat = spush(C, Dl * Dr);
  if (failed(C)) return 0.0;
  gemm(T, Dl, Dr, dd, colmajor(sdata(C, last), Dl), colmajor(sdata(C, hj), dd), colmajor(mat, Dl));
  SiteRef prev = sref(C, ki, hi.nsites - 1);
  const long long pr = (long long)prev.dl * prev.d;
  if (!heap_reserve(C, al256(8 * pr * Dr))) return 0.0;
  prev = sref(C, ki, hi.nsites - 1);
  const long long nt = heap_take(C, 8 * pr * Dr);
  gemm(T, pr, Dr, prev.dr, colmajor(sdata(C, prev), pr), colmajor(mat, Dl), colmajor(dptr(C, nt), pr));
  if (C.tape) {
    TapeRec q = trec(OP_EAT_C);
    q.a[0] = (int)Dl; q.a[1] = (int)dd; q.a[2] = (int)Dr; q.a[3] = (int)pr;
    q.o[0] = last.off; q.o[1] = hj.off; q.o[2] = prev.off; q.o[3] = nt;
    tape_push(C, q);
  }
  account(C, 2.0 * Dl * dd * Dr + 2.0 * pr * prev.dr * Dr,
          8.0 * ((double)Dl * dd + (double)dd * Dr + (double)pr * prev.dr + (double)pr * Dr));
  T.sync();
  if (T.leader()) {
    const int nsi = hi.nsites - 1;
    sref(C, ki, nsi) = mksite(prev.dl, prev.d, (int)Dr, nt);
    const int nsj = C.node[kj].nsites;
    if (nsi + nsj - 1 > C.maxs || C.node[ki].nnbr - 1 + C.node[kj].nnbr > C.maxs) {
      fail_leader(C, CATN_ENOMEM);
    } else {
      for (int p = 2; p <= nsj; ++p) sref(C, ki, nsi + p - 1) = sref(C, kj, p);
      C.node[ki].nsites = nsi + nsj - 1;
      C.node[ki].cano = nsi;
      C.node[kj].nsites = 0;   // j's sites 2:end now belong to i
      int nni = C.node[ki].nnbr - 1;
      const int nnj = C.node[kj].nnbr;
      for (int p = 2; p <= nnj; ++p) nbref(C, ki, nni + p - 1) = nbref(C, kj, p);
      C.node[ki].nnbr = nni + (nnj > 1 ? nnj - 1 : 0);
    }
  }
  refresh_status(C);
  C.sp = mark;
  prof_add(C, PROF_EAT, (double)(clk() - tf));
  if (failed(C)) return 0.0;
  cano_to(C, ki, C.node[ki].nsites);
  if (failed(C)) return 0.0;
  SiteRef ctr = sref(C, ki, C.node[ki].cano);
  const long long ce = (long long)ctr.dl * ctr.d * ctr.dr;
  const double nrm = norm_of(C, sdata(C, ctr), ce);
  if (nrm <= cutoff) return 0.0;
  if (!normalize_site(C, ki, C.node[ki].cano, nrm)) return 0.0;
  return log(nrm);
}

// ---------------------------------------------------------------------------
// QR pre-reduction (compress_opt!, cut_bondim_opt!): X (rows x cols) in a
// scratch buffer, consumed into Householder form when rows > cols.
// ---------------------------------------------------------------------------
struct QRed {
  bool flag;
  double* house;   // rows x cols (Householder form when flag)
  double* tau;
  double* Rb;      // R (cols x cols) or the matrix itself (rows x cols)
  long long rrows, cols, rows;
};

CATN_HDI inline QRed qr_reduce(Ctx& C, double* X, long long rows, long long cols) {
  const Team& T = C.T;
  QRed q;
  q.rows = rows;
  q.cols = cols;
  q.house = X;
  q.tau = nullptr;
  q.flag = rows > cols;
  q.Rb = X;
  q.rrows = rows;
  if (!q.flag) return q;
  q.tau = spush(C, cols);
  q.Rb = spush(C, cols * cols);
  q.rrows = cols;
  if (failed(C)) return q;
  qr_inplace(T, X, rows, cols, rows, q.tau);
  for (long long e = T.rank(); e < cols * cols; e += T.size()) {
    long long r, c;
    divmod(e, cols, &r, &c);
    q.Rb[e] = (r <= c) ? X[r + c * rows] : 0.0;
  }
  T.sync();
  return q;
}
// Y (rrows x ncols) -> Q [Y; 0] (rows x ncols) into `out`.
CATN_HDI inline void qr_expand(Ctx& C, const QRed& q, const double* Y, long long ncols, double* out) {
  const Team& T = C.T;
  for (long long e = T.rank(); e < q.rows * ncols; e += T.size()) {
    long long r, c;
    divmod(e, q.rows, &r, &c);
    out[e] = (r < q.rrows) ? Y[r + c * q.rrows] : 0.0;
  }
  T.sync();
  if (q.flag) qr_apply_q(T, q.house, q.rows, q.cols, q.rows, q.tau, out, ncols, q.rows);
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
    const long long mark = C.sp;
    SiteRef tl = sref(C, k, i), tr = sref(C, k, jj);
    const long long d0 = tl.dl, d1 = tl.d, dd = tl.dr, d2 = tr.d, d3 = tr.dr;
    const long long ml = d0 * d1, nr = d2 * d3;
    double* Uo = nullptr;   // ml x myd  (U * S, through Ql)
    double* Vo = nullptr;   // nr x myd  (V, through Qr)
    int myd;
    double e;
    Svd R;
    if (!opt) {
      SvdIn in = svd_begin(C, ml, nr, C.P.cutoff);
      if (failed(C)) return err;
      gemm(T, ml, nr, dd, colmajor(sdata(C, tl), ml), colmajor(sdata(C, tr), dd), svd_target(in));
      R = svd_finish(C, in);
      if (failed(C)) return err;
      myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &e);
    } else {
      double* matl = spush(C, ml * dd);
      double* matrt = spush(C, nr * dd);
      if (failed(C)) return err;
      copy(T, matl, sdata(C, tl), ml * dd);
      materialize(T, matrt, nr, dd, nr, transposed(sdata(C, tr), dd));
      QRed ql = qr_reduce(C, matl, ml, dd);
      QRed qr = qr_reduce(C, matrt, nr, dd);
      if (failed(C)) return err;
      // mat = Rl * Rr^H  (ql.rrows x qr.rrows)
      SvdIn in = svd_begin(C, ql.rrows, qr.rrows, C.P.cutoff);
      if (failed(C)) return err;
      gemm(T, ql.rrows, qr.rrows, dd, colmajor(ql.Rb, ql.rrows), transposed(qr.Rb, qr.rrows), svd_target(in));
      R = svd_finish(C, in);
      if (failed(C)) return err;
      myd = keep_rule(C, R, C.P.cutoff, C.P.chi, &e);
      double* us = spush(C, ql.rrows * myd);
      Uo = spush(C, ml * myd);
      Vo = spush(C, nr * myd);
      if (failed(C)) return err;
      materialize(T, us, ql.rrows, myd, ql.rrows, mop(R.U, rows_plain(), cols_plain(ql.rrows), nullptr, R.S));
      qr_expand(C, ql, us, myd, Uo);
      qr_expand(C, qr, R.V, myd, Vo);
    }
    err += e;
    if (!heap_reserve(C, al256(8 * ml * myd) + al256(8 * nr * myd))) return err;
    const long long ou = heap_take(C, 8 * ml * myd);
    const long long ov = heap_take(C, 8 * nr * myd);
    if (!opt) {
      materialize(T, dptr(C, ou), ml, myd, ml, mop(R.U, rows_plain(), cols_plain(ml), nullptr, R.S));
      materialize(T, dptr(C, ov), myd, nr, myd, mop(R.V, imap(1, 0, nr), rows_plain()));
    } else {
      copy(T, dptr(C, ou), Uo, ml * myd);
      materialize(T, dptr(C, ov), myd, nr, myd, transposed(Vo, nr));
    }
    account(C, 2.0 * ml * nr * dd + 4.0 * ml * nr * myd,
            8.0 * ((double)ml * dd + (double)dd * nr + (double)ml * myd + (double)myd * nr));
    if (T.leader()) {
      sref(C, k, i) = mksite((int)d0, (int)d1, myd, ou);
      sref(C, k, jj) = mksite(myd, (int)d2, (int)d3, ov);
    }
    T.sync();
    C.sp = mark;
  }
  T.sync();
  if (T.leader()) C.node[k].cano = 1;
  T.sync();
  return err;
}

// The matrix itself as a QRed without reduction (cut_bondim!).
CATN_HDI inline QRed qr_none(double* X, long long rows, long long cols) {
  QRed q;
  q.rows = rows;
  q.cols = cols;
  q.house = X;
  q.tau = nullptr;
  q.flag = false;
  q.Rb = X;
  q.rrows = rows;
  return q;
}

// ---------------------------------------------------------------------------
// cut_bondim_opt! (tensor_network.jl:399-477) with `opt`, cut_bondim!
// (tensor_network.jl:342-388) without: the plain cut neither canonicalises
// the two nodes nor pre-reduces the two matrices by QR, so its SVD takes the
// whole (da_l da_r) x (db_l db_r) product.  Returns the discarded sum.
// ---------------------------------------------------------------------------
CATN_HDI inline double cut_bond(Ctx& C, int i, int idx_j_in_i, bool opt = true) {
  const Team& T = C.T;
  if (C.P.Dmax < 0) return 0.0;
  int j = nbref(C, i, idx_j_in_i);
  if (j <= 0) { fail_all(C, CATN_ESTATE); return 0.0; }
  int idx_i_in_j = nb_find(C, j, i);
  if (idx_i_in_j == 0) { fail_all(C, CATN_ESTATE); return 0.0; }
  if (opt) {
    cano_to(C, i, idx_j_in_i);
    cano_to(C, j, idx_i_in_j);
  }
  if (failed(C)) return 0.0;
  const long long tcut = clk();
  const long long mark = C.sp;
  SiteRef Ai = sref(C, i, idx_j_in_i), Aj = sref(C, j, idx_i_in_j);
  const long long d = Ai.d;
  const long long ri_rows = (long long)Ai.dl * Ai.dr, rj_rows = (long long)Aj.dl * Aj.dr;
  // mati = reshape(permutedims(Ai, (1,3,2)), da_l*da_r, d)
  double* mi = spush(C, ri_rows * d);
  double* mj = spush(C, rj_rows * d);
  if (failed(C)) return 0.0;
  materialize(T, mi, ri_rows, d, ri_rows, mop(sdata(C, Ai), imap(Ai.dl, 1, (long long)Ai.dl * d), cols_plain(Ai.dl)));
  materialize(T, mj, rj_rows, d, rj_rows, mop(sdata(C, Aj), imap(Aj.dl, 1, (long long)Aj.dl * d), cols_plain(Aj.dl)));
  QRed qi = opt ? qr_reduce(C, mi, ri_rows, d) : qr_none(mi, ri_rows, d);
  QRed qj = opt ? qr_reduce(C, mj, rj_rows, d) : qr_none(mj, rj_rows, d);
  if (failed(C)) return 0.0;
  SvdIn in = svd_begin(C, qi.rrows, qj.rrows, C.P.cutoff);
  if (failed(C)) return 0.0;
  if (C.P.Dmax > 0) in.need = C.P.Dmax;   // the cut keeps at most Dmax vectors
  gemm(T, qi.rrows, qj.rrows, d, colmajor(qi.Rb, qi.rrows), transposed(qj.Rb, qj.rrows), svd_target(in));
  Svd R = svd_finish(C, in);
  if (failed(C)) return 0.0;
  double disc = 0.0;
  const int kept = keep_rule(C, R, C.P.cutoff, 0x7fffffffLL, &disc);
  int myd = kept < C.P.Dmax ? kept : C.P.Dmax;
  if (myd < 1) myd = 1;
  double extra = 0.0;
  {
    double loc = 0.0;
    for (long long e = myd + T.rank(); e < kept; e += T.size()) loc += R.S[e];
    extra = T.sum(loc);
  }
  double* sq = spush(C, myd);
  double* ui = spush(C, qi.rrows * myd);
  double* vj = spush(C, qj.rrows * myd);
  double* fi = spush(C, ri_rows * myd);
  double* fj = spush(C, rj_rows * myd);
  if (failed(C)) return 0.0;
  for (long long e = T.rank(); e < myd; e += T.size()) sq[e] = sqrt(R.S[e]);
  T.sync();
  materialize(T, ui, qi.rrows, myd, qi.rrows, mop(R.U, rows_plain(), cols_plain(qi.rrows), nullptr, sq));
  materialize(T, vj, qj.rrows, myd, qj.rrows, mop(R.V, rows_plain(), cols_plain(qj.rrows), nullptr, sq));
  qr_expand(C, qi, ui, myd, fi);   // (da_l*da_r) x myd
  qr_expand(C, qj, vj, myd, fj);
  const long long tb = C.tape ? al256(8LL * myd) : 0;
  if (!heap_reserve(C, al256(8LL * Ai.dl * myd * Ai.dr) + al256(8LL * Aj.dl * myd * Aj.dr) + tb)) return 0.0;
  const long long ni = heap_take(C, 8LL * Ai.dl * myd * Ai.dr);
  const long long nj = heap_take(C, 8LL * Aj.dl * myd * Aj.dr);
  if (C.tape) {
    TapeRec r = trec(OP_CUT);
    r.a[0] = Ai.dl; r.a[1] = (int)d; r.a[2] = Ai.dr; r.a[3] = Aj.dl; r.a[4] = Aj.dr; r.a[5] = myd;
    r.o[0] = Ai.off; r.o[1] = Aj.off; r.o[2] = ni; r.o[3] = nj;
    r.o[4] = heap_take(C, 8LL * myd);
    copy(T, dptr(C, r.o[4]), R.S, myd);
    tape_push(C, r);
  }
  {
    // new site = permutedims(reshape(mat, dl, dr, myd), (1,3,2))
    double* O = dptr(C, ni);
    const long long dl = Ai.dl, dr = Ai.dr, tot = dl * myd * dr;
    for (long long e = T.rank(); e < tot; e += T.size()) {
      long long a, rest, r, c;
      divmod(e, dl, &a, &rest);
      divmod(rest, myd, &r, &c);
      O[e] = fi[(a + dl * c) + ri_rows * r];
    }
    double* P2 = dptr(C, nj);
    const long long dl2 = Aj.dl, dr2 = Aj.dr, tot2 = dl2 * myd * dr2;
    for (long long e = T.rank(); e < tot2; e += T.size()) {
      long long a, rest, r, c;
      divmod(e, dl2, &a, &rest);
      divmod(rest, myd, &r, &c);
      P2[e] = fj[(a + dl2 * c) + rj_rows * r];
    }
    T.sync();
  }
  account(C, 4.0 * (double)ri_rows * d * d + 4.0 * (double)rj_rows * d * d + 2.0 * qi.rrows * qj.rrows * d +
                 4.0 * qi.rrows * qj.rrows * myd,
          8.0 * ((double)ri_rows * d + (double)rj_rows * d + (double)ri_rows * myd + (double)rj_rows * myd));
  if (T.leader()) {
    sref(C, i, idx_j_in_i) = mksite(Ai.dl, myd, Ai.dr, ni);
    sref(C, j, idx_i_in_j) = mksite(Aj.dl, myd, Aj.dr, nj);
  }
  T.sync();
  C.sp = mark;
  prof_add(C, PROF_CUT, (double)(clk() - tcut));
  return disc + extra;
}

// ---------------------------------------------------------------------------
// raw2mps (mps_node.jl:31-50): dense column-major tensor -> sites of node k.
// ---------------------------------------------------------------------------
CATN_HDI inline void raw2mps(Ctx& C, int k, const double* data, const long long* dims, int nd) {
  const Team& T = C.T;
  if (nd == 0) return;   // the reference returns an empty MPS for a 0-d tensor
  if (nd > C.maxs) { fail_all(C, CATN_ENOMEM); return; }
  const long long mark = C.sp;
  long long total = 1;
  for (int q = 0; q < nd; ++q) total *= dims[q];
  double* R = spush(C, total);
  if (failed(C)) return;
  copy(T, R, data, total);
  long long cur = total, dleft = 1;
  for (int q = 0; q < nd - 1; ++q) {
    const long long m = dleft * dims[q], n = cur / m;
    SvdIn in = svd_begin(C, m, n, C.P.cutoff);
    if (failed(C)) return;
    svd_fill(C, in, colmajor(R, m));
    Svd S = svd_finish(C, in);
    if (failed(C)) return;
    double disc;
    const int c = keep_rule(C, S, C.P.cutoff, C.P.chi, &disc);
    double* r2 = spush(C, (long long)c * n);
    if (failed(C) || !heap_reserve(C, al256(8 * m * c))) return;
    const long long u = heap_take(C, 8 * m * c);
    copy(T, dptr(C, u), S.U, m * c);
    materialize(T, r2, c, n, c, mop(S.V, imap(1, 0, n), rows_plain(), S.S, nullptr));
    if (T.leader()) sref(C, k, q + 1) = mksite((int)dleft, (int)dims[q], c, u);
    T.sync();
    // sites 1..q+1 are live from here on (compaction may move them)
    if (T.leader()) C.node[k].nsites = q + 1;
    T.sync();
    R = r2;
    cur = (long long)c * n;
    dleft = c;
  }
  if (!heap_reserve(C, al256(8 * cur))) return;
  const long long last = heap_take(C, 8 * cur);
  copy(T, dptr(C, last), R, cur);
  if (T.leader()) {
    sref(C, k, nd) = mksite((int)dleft, (int)dims[nd - 1], 1, last);
    C.node[k].nsites = nd;
    C.node[k].cano = nd;
  }
  T.sync();
  C.sp = mark;
}

// ---------------------------------------------------------------------------
// Edge-cost bookkeeping (tensor_network.jl:152-316) as an entry pool.  An
// alive entry (cost, i, j, seq) stands for pair [i, j] in bucket `cost` of the
// reference's edge_count; `seq` is its insertion rank, so bucket order is
// ascending seq and "first pair of the cheapest bucket" is the alive entry of
// least cost with the least seq.  Removal, insertion and selection are
// team-parallel.
// ---------------------------------------------------------------------------
CATN_HD int& emap_at(const Ctx& C, int i, int j) { return C.emap[(long long)i * (C.n + 1) + j]; }

// Fill the logdim cache (left fold of log2 phys dims, mps_node.jl:299-311) for
// `list` nodes and all their neighbours, in a phase of its own so that cost
// readers never race cache writers.
CATN_HDI inline void logdim_prefetch(Ctx& C, const int* list, int nl) {
  const Team& T = C.T;
  for (int a = T.warp(); a < nl; a += T.nwarps()) {
    const int x = list[a];
    if (x <= 0) continue;
    const int nn = C.node[x].nnbr;
    for (int p = T.lane(); p <= nn; p += T.wsize()) {
      const int y = (p == 0) ? x : nbref(C, x, p);
      if (y <= 0 || C.ldv[y]) continue;
      C.ldc[y] = logdim_all(C, y);
    }
  }
  T.sync();
  for (int a = T.warp(); a < nl; a += T.nwarps()) {
    const int x = list[a];
    if (x <= 0) continue;
    const int nn = C.node[x].nnbr;
    for (int p = T.lane(); p <= nn; p += T.wsize()) {
      const int y = (p == 0) ? x : nbref(C, x, p);
      if (y > 0) C.ldv[y] = 1;
    }
  }
  T.sync();
}

// dim_after_merge (tensor_network.jl:152-155) with the shared bond's phys dim
// d already known (a bond has the same phys dim at both ends):
// round(logdim(i) + logdim(j) - 2 log2(d)), ties to even.
CATN_HD int pair_cost(const Ctx& C, int i, int j, int d) {
  const double v = C.ldc[i] + C.ldc[j] - 2.0 * log2((double)d);
  return (int)rint(v);
}

// count_remove_nodes! (:213-225): every bond of every node in `list` leaves
// the bucket of its current cost.
CATN_HDI inline void count_remove_nodes_team(Ctx& C, const int* list, int nl) {
  const Team& T = C.T;
  logdim_prefetch(C, list, nl);
  int* ftop = C.ctl + CTL_FTOP;
  for (int a = T.warp(); a < nl; a += T.nwarps()) {
    const int x = list[a];
    if (x <= 0) continue;
    const int nn = C.node[x].nnbr;
    for (int p = 1 + T.lane(); p <= nn; p += T.wsize()) {
      const int y = nbref(C, x, p);
      if (y <= 0) continue;
      const int i = x < y ? x : y, j = x < y ? y : x;
      const int cost = pair_cost(C, i, j, sref(C, x, p).d);
      int& m = emap_at(C, i, j);
      const int e = m;
      if (e < 0) continue;
      EdgeEnt& E = C.ent[e];
      if (E.cost != cost || E.i != i || E.j != j) continue;
      if (T.atomic_cas(&E.alive, 1, 0) == 1) {   // exactly one remover per entry
        m = -1;
        C.fstack[T.atomic_add(ftop, 1)] = e;
      }
    }
  }
  T.sync();
}

// Bitonic sort of `pow2` 64-bit keys with one int payload, in place.
CATN_HDI inline void bitonic_sort(const Team& T, long long* key, int* val, int pow2) {
  for (int k = 2; k <= pow2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = T.rank(); t < pow2; t += T.size()) {
        const int u = t ^ j;
        if (u > t) {
          const bool up = (t & k) == 0;
          if ((key[t] > key[u]) == up) {
            const long long kk = key[t]; key[t] = key[u]; key[u] = kk;
            const int vv = val[t]; val[t] = val[u]; val[u] = vv;
          }
        }
      }
      T.sync();
    }
  }
}

// count_add_nodes! (:185-197): the bonds of `list` nodes, deduplicated and
// inserted in lexicographic order of (i, j) -- the reference's
// sort(collect(Set(...))).
CATN_HDI inline void count_add_nodes_team(Ctx& C, const int* list, int nl) {
  const Team& T = C.T;
  const long long EMPTY = 0x7fffffffffffffffLL;
  logdim_prefetch(C, list, nl);
  int local = 0;
  for (int a = T.rank(); a < nl; a += T.size())
    if (list[a] > 0) local += C.node[list[a]].nnbr;
  const int npairs = (int)(T.sum((double)local) + 0.5);
  int pow2 = 1;
  while (pow2 < npairs) pow2 <<= 1;
  // sort workspace: shared memory when it fits, else the slot's pair scratch
  long long* key;
  int* val;
  if ((long long)pow2 * 12 <= C.sws_doubles * 8) {
    key = (long long*)C.sws;
  } else if ((long long)pow2 <= (long long)C.pcap) {
    key = (long long*)C.pairs;
  } else {
    fail_all(C, CATN_ENOMEM);
    return;
  }
  val = (int*)(key + pow2);
  int* cnt = C.ctl + CTL_SPARE;
  T.sync();
  if (T.leader()) *cnt = 0;
  T.sync();
  for (int a = T.warp(); a < nl; a += T.nwarps()) {
    const int x = list[a];
    if (x <= 0) continue;
    const int nn = C.node[x].nnbr;
    for (int p = 1 + T.lane(); p <= nn; p += T.wsize()) {
      const int y = nbref(C, x, p);
      const int slot = T.atomic_add(cnt, 1);
      if (y <= 0) {
        key[slot] = EMPTY;   // open leg: sorts to the end, dropped below
        val[slot] = 0;
        continue;
      }
      const int i = x < y ? x : y, j = x < y ? y : x;
      key[slot] = ((long long)i << 32) | (long long)j;
      val[slot] = sref(C, x, p).d;
    }
  }
  T.sync();
  for (int t = npairs + T.rank(); t < pow2; t += T.size()) {
    key[t] = EMPTY;
    val[t] = 0;
  }
  T.sync();
  bitonic_sort(T, key, val, pow2);
  // unique real pairs get consecutive ranks in sorted order
  int* ftop = C.ctl + CTL_FTOP;
  const int top0 = *ftop;
  const int seq0 = C.ctl[CTL_SEQ];
  int base_rank = 0;
  for (int t0 = 0; t0 < pow2; t0 += T.size()) {
    const int t = t0 + T.rank();
    int flag = 0;
    if (t < pow2 && key[t] != EMPTY && (t == 0 || key[t] != key[t - 1])) flag = 1;
    int tot = 0;
    const int r = base_rank + T.scan_excl(flag, &tot);
    if (flag) {
      if (r >= top0) {
        fail_all(C, CATN_ENOMEM);
      } else {
        const int i = (int)(key[t] >> 32), j = (int)(key[t] & 0xffffffff);
        const int e = C.fstack[top0 - 1 - r];
        EdgeEnt& E = C.ent[e];
        E.cost = pair_cost(C, i, j, val[t]);
        E.i = i;
        E.j = j;
        E.seq = seq0 + r;
        E.alive = 1;
        int& m = emap_at(C, i, j);
        if (m >= 0 && C.ent[m].alive) T.atomic_add(C.ctl + CTL_ANOMALY, 1);
        m = e;
      }
    }
    base_rank += tot;
  }
  T.sync();
  if (T.leader()) {
    const int used = base_rank < top0 ? base_rank : top0;
    *ftop = top0 - used;
    C.ctl[CTL_SEQ] = seq0 + used;
    if (base_rank > top0) fail_leader(C, CATN_ENOMEM);
  }
  refresh_status(C);
}

// select_edge_min_dim (:248-253) / _triangle (:262-288) / _sequentially
// (:300-316), as team reductions over the entry pool / the nodes.
CATN_HDI inline long long select_team(Ctx& C, int* maxdim) {
  const Team& T = C.T;
  const int sel = C.P.select;
  if (sel == 0 || sel == 1) {
    // cheapest non-empty bucket
    double mc = 1e300;
    for (int e = T.rank(); e < C.ecap; e += T.size())
      if (C.ent[e].alive && C.ent[e].cost < mc) mc = C.ent[e].cost;
    mc = -T.maxv(-mc);
    if (mc > 1e299) { fail_all(C, CATN_ESTATE); return 0; }
    const int cost = (int)mc;
    if (cost > *maxdim) *maxdim = cost;
    double bv = -1.0;
    long long be = -1;
    for (int e = T.rank(); e < C.ecap; e += T.size()) {
      const EdgeEnt E = C.ent[e];
      if (!E.alive || E.cost != cost) continue;
      int both = 0;
      if (sel == 1) {
        const int i = E.i, j = E.j, nn = C.node[j].nnbr;
        for (int p = 1; p <= nn; ++p) {
          const int k = nbref(C, j, p);
          if (k <= 0 || k == i) continue;
          // Set semantics: a repeated neighbour counts once.  Every step merges
          // the duplicates it creates, so lists repeat only when the input does.
          if (C.multigraph) {
            bool dup = false;
            for (int q = 1; q < p; ++q)
              if (nbref(C, j, q) == k) { dup = true; break; }
            if (dup) continue;
          }
          if (nb_find(C, k, i) > 0) ++both;
        }
      }
      // largest count first, then earliest insertion
      const double key = (double)both * 2147483648.0 + (double)(0x7fffffff - E.seq);
      if (be < 0 || key > bv) { bv = key; be = e; }
    }
    const long long e = T.argmax(bv, be);
    if (e < 0) { fail_all(C, CATN_ESTATE); return 0; }
    return ((long long)C.ent[e].i << 32) | (unsigned)C.ent[e].j;
  }
  // sequential: minimum i + nb, ties by ascending node id
  double bv = -1.0;
  long long bi = -1;
  for (int i = 1 + T.rank(); i <= C.n; i += T.size()) {
    const int nn = C.node[i].nnbr;
    for (int p = 1; p <= nn; ++p) {
      const int nb = nbref(C, i, p);
      if (nb <= 0 || !(i < nb)) continue;
      const double key = -((double)(i + nb) * 4194304.0 + (double)i);
      if (bi < 0 || key > bv) { bv = key; bi = ((long long)i << 32) | (unsigned)nb; }
    }
  }
  const long long best = T.argmax(bv, bi);
  if (best < 0) { fail_all(C, CATN_ESTATE); return 0; }
  return best;
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

// Loop state of contraction! between steps (contract_begin / _step / _end).
struct LoopState {
  ContractOut O;
  int maxdim, buckets, step_cap;
};

// select_edge_init! and the loop state before the first step.
CATN_HDI inline void contract_begin(Ctx& C, LoopState& S) {
  const Team& T = C.T;
  S.O.lnZ = 0.0; S.O.err = 0.0; S.O.psi = 1.0; S.O.sign = 1.0; S.O.maxdim = -1; S.O.nsteps = 0;
  S.buckets = (C.P.select == 0 || C.P.select == 1);
  if (C.tape && C.P.compress) fail_all(C, CATN_EINVAL);   // no adjoint of the compress sweeps
  if (S.buckets) {
    // select_edge_init!: all node ids
    for (int k = 1 + T.rank(); k <= C.n; k += T.size()) C.list[k - 1] = k;
    T.sync();
    count_add_nodes_team(C, C.list, C.n);
  }
  S.maxdim = -1;
  // Every step clears one node, so a network of n nodes needs fewer than n
  // steps; the cap only guards against corrupted state.
  S.step_cap = C.n + 16;
}

// One step of the main loop (tensor_network.jl:574-707); false when no real
// edge is left or the instance failed.
CATN_HDI inline bool contract_step(Ctx& C, LoopState& S) {
  const Team& T = C.T;
  const long long tc0 = clk();
  const bool more = !failed(C) && has_real_edges(C);
  prof_add(C, PROF_CONTROL, (double)(clk() - tc0));
  if (!more) return false;
  if (S.O.nsteps > S.step_cap) {
    fail_all(C, CATN_ESTATE);
    return false;
  }
  // --- select ---
  const long long tb0 = clk();
  const long long pk = select_team(C, &S.maxdim);
  if (failed(C)) return false;
  int i = (int)(pk >> 32), j = (int)(pk & 0xffffffff);
  if (C.node[j].nsites > C.node[i].nsites) { int t = i; i = j; j = t; }
  // --- bookkeeping before any shape change ---
  if (S.buckets) {
    int* list = C.list;
    const int nl = 2 + C.node[i].nnbr + C.node[j].nnbr;
    T.sync();
    if (T.leader()) {
      int q = 0;
      list[q++] = i;
      list[q++] = j;
      for (int p = 1; p <= C.node[i].nnbr; ++p) list[q++] = nbref(C, i, p);
      for (int p = 1; p <= C.node[j].nnbr; ++p) list[q++] = nbref(C, j, p);
    }
    T.sync();
    count_remove_nodes_team(C, list, nl);
    // every node whose sites this step may change: i, j and their neighbours
    for (int q = T.rank(); q < nl; q += T.size())
      if (list[q] > 0) C.ldv[list[q]] = 0;
    T.sync();
  }
  prof_add(C, PROF_BOOK, (double)(clk() - tb0));
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
  if (failed(C)) return false;
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
    if (idx_j_in_k == 0) { fail_all(C, CATN_ESTATE); break; }
    T.sync();
    if (T.leader()) {
      nb_delete_at_leader(C, k, idx_j_in_k);
      nb_insert_at_leader(C, k, idx_j_in_k, i);
    }
    refresh_status(C);
    if (failed(C)) break;
    if (idx_k_in_i > 0) {
      T.sync();
      if (T.leader()) dup[nd] = k;
      T.sync();
      ++nd;
      duph = fnv_step(duph, k);
      bool cross = idx_i_in_k > idx_j_in_k;
      S.O.err += merge_dup(C, k, i, cross);
    }
  }
  if (failed(C)) return false;
  // --- eat! ---
  double lnv = eat(C, i, j, idx_j_in_i, idx_i_in_j, &S.O.err, &S.O.psi);
  S.O.lnZ += lnv;
  if (failed(C)) return false;
  // --- duplicates: merge into i, then cut ---
  for (int q = 0; q < nd && !failed(C); ++q) {
    int k = dup[q];
    merge_dup(C, i, k, false);   // its error is not accumulated (tensor_network.jl:662)
    int idx_k_in_i = nb_find(C, i, k);
    if (failed(C)) break;
    if (C.P.cut_bond || (C.P.Dmax > 0 && sref(C, i, idx_k_in_i).d > C.P.Dmax))
      S.O.err += cut_bond(C, i, idx_k_in_i);
  }
  if (failed(C)) return false;
  clear_node(C, j);
  if (C.P.compress) compress_node(C, i, C.P.svdopt != 0);   // error discarded (:688-694)
  if (failed(C)) return false;
  if (S.buckets) {
    const long long tb1 = clk();
    int* list = C.list;
    const int nl = 1 + C.node[i].nnbr;
    T.sync();
    if (T.leader()) {
      list[0] = i;
      for (int p = 1; p <= C.node[i].nnbr; ++p) list[p] = nbref(C, i, p);
    }
    T.sync();
    count_add_nodes_team(C, list, nl);
    prof_add(C, PROF_BOOK, (double)(clk() - tb1));
  }
  const int nsi = C.node[i].nsites;
  unsigned shh = 2166136261u;
  for (int p = 1; p <= nsi; ++p) {
    int d = sref(C, i, p).d;
    if (d > S.maxdim) S.maxdim = d;
    shh = fnv_step(shh, d);
  }
  if (C.trace && S.O.nsteps < C.trace_cap) {
    T.sync();
    if (T.leader()) {
      int* r = C.trace + 8LL * S.O.nsteps;
      r[0] = i; r[1] = j; r[2] = rev; r[3] = nd; r[4] = (int)duph; r[5] = nsi; r[6] = (int)shh; r[7] = S.maxdim;
    }
    T.sync();
  }
  S.O.nsteps += 1;
  return true;
}

// network_lognorm (tensor_network.jl:489-501) and the outputs.
CATN_HDI inline void contract_end(Ctx& C, LoopState& S) {
  const Team& T = C.T;
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
  if (C.tape) {
    // every thread walks the nodes alike so that the records are uniform
    for (int k = 1; k <= C.n; ++k) {
      NodeHdr h = C.node[k];
      if (h.nsites != 1 || sref(C, k, 1).d != 1) continue;
      SiteRef s = sref(C, k, 1);
      const double* x = dptr(C, s.off);
      double z = 0.0;
      for (long long e = 0; e < (long long)s.dl * s.dr; ++e) z += x[e];
      TapeRec r = trec(OP_LOGZ);
      r.a[0] = s.dl * s.dr; r.o[0] = s.off; r.v[0] = z;
      tape_push(C, r);
    }
  }
  lsum = T.sum(lsum);
  nneg = T.sum(nneg);
  nzero = T.sum(nzero);
  bad = T.sum(bad);
  if (bad > 0.5) fail_all(C, CATN_ESTATE);
  S.O.lnZ += lsum;
  S.O.sign = nzero > 0.5 ? 0.0 : (((long long)(nneg + 0.5)) % 2 ? -1.0 : 1.0);
  S.O.maxdim = S.maxdim;
}

CATN_HDI inline ContractOut contract(Ctx& C) {
  LoopState S;
  contract_begin(C, S);
  while (contract_step(C, S)) {
  }
  contract_end(C, S);
  return S.O;
}

// ---------------------------------------------------------------------------
// Slot initialisation and instance loading
// ---------------------------------------------------------------------------
// `sws`/`sws_doubles`: shared-memory SVD workspace of the team.
CATN_HDI inline Ctx make_ctx(const Team& T, char* slot, const SlotLayout& L, const catn_params& P, int n,
                             double* sws, long long sws_doubles) {
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
  C.fstack = (int*)(slot + L.off_fstack);
  C.emap = (int*)(slot + L.off_emap);
  C.ctl = (int*)(slot + L.off_ctl);
  C.pairs = (int*)(slot + L.off_pairs);
  C.pcap = L.pcap;
  C.list = (int*)(slot + L.off_list);
  C.tmp = (int*)(slot + L.off_tmp);
  C.acct = (double*)(slot + L.off_ameta);
  C.ldc = (double*)(slot + L.off_ldc);
  C.ldv = (long long*)(slot + L.off_ldc) + (C.n + 1);
  C.base = slot + L.off_arena;
  // arena: scratch stack (40%), two heap halves (30% each)
  const long long cap = L.arena_bytes & ~255LL;
  const long long sc = (cap * 2 / 5) & ~255LL;
  C.hsize = ((cap - sc) / 2) & ~255LL;
  C.sp_lo = 0;
  C.sp = 0;
  C.sp_hi = sc;
  C.sp_peak = 0;
  C.h_lo0 = sc;
  C.h_lo1 = sc + C.hsize;
  C.half = 0;
  C.hb = C.h_lo0;
  C.he = C.h_lo0 + C.hsize;
  C.h_peak = 0;
  C.compactions = 0;
  C.sws = sws;
  C.sws_doubles = sws_doubles;
  C.status = 0;
  C.rsvd_min = 0;
  C.rsvd_calls = 0;
  C.multigraph = 1;
  C.trace = nullptr;
  C.trace_cap = 0;
  C.tape = 0;
  C.rec = nullptr;
  C.nrec = C.rcap = C.gshift = 0;
  C.heap_first = 0;
  C.job = nullptr;
  C.qhead = nullptr;
  C.ninst = 0;
  C.job_min_n = 1 << 30;
  C.job_pool = 0;
  C.job_min_qr = 1LL << 62;
  C.block_min_n = kBlockMinN;
  C.blocked_qr_min_n = 1 << 30;
  return C;
}

CATN_HDI inline void reset_slot(Ctx& C) {
  const Team& T = C.T;
  const long long nn = (long long)C.n + 1;
  for (long long e = T.rank(); e < nn * nn; e += T.size()) C.emap[e] = -1;
  for (long long e = T.rank(); e < C.ecap; e += T.size()) {
    C.ent[e].alive = 0;
    C.fstack[e] = (int)(C.ecap - 1 - e);   // pops hand out 0, 1, 2, ...
  }
  for (long long e = T.rank(); e < nn; e += T.size()) {
    C.node[e].nsites = 0; C.node[e].nnbr = 0; C.node[e].cano = 0; C.node[e].pad = 0;
    C.ldv[e] = 0;
  }
  for (long long e = T.rank(); e < CTL_WORDS; e += T.size()) C.ctl[e] = 0;
  T.sync();
  if (T.leader()) {
    C.ctl[CTL_FTOP] = C.ecap;
    for (int q = 0; q < 2 + PROF_SLOTS + 2; ++q) C.acct[q] = 0.0;
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
    // MPS form: sites laid out contiguously in the heap (every thread
    // computes the same offsets), leader writes the refs, team copies data.
    long long total = 0, nsites = 0;
    for (int k = 1; k <= C.n; ++k) {
      const int ns = (int)hdr[4 * (k - 1)], nn = (int)hdr[4 * (k - 1) + 1];
      if (ns > C.maxs || nn > C.maxs) { fail_all(C, CATN_ENOMEM); return; }
      for (int p = 0; p < ns; ++p, ++nsites)
        total += al256(8 * dims[3 * nsites] * dims[3 * nsites + 1] * dims[3 * nsites + 2]);
    }
    if (!heap_reserve(C, total)) return;
    const long long first = C.hb;
    C.heap_first = first;
    C.hb += total;
    if (C.hb - C.h_lo0 > C.h_peak) C.h_peak = C.hb - C.h_lo0;
    if (T.leader()) {
      long long sidx = 0, nidx = 0, cur = first;
      for (int k = 1; k <= C.n; ++k) {
        const int ns = (int)hdr[4 * (k - 1)], nn = (int)hdr[4 * (k - 1) + 1], cano = (int)hdr[4 * (k - 1) + 2];
        C.node[k].nsites = ns;
        C.node[k].nnbr = nn;
        C.node[k].cano = cano;
        for (int p = 1; p <= ns; ++p, ++sidx) {
          const int dl = (int)dims[3 * sidx], d = (int)dims[3 * sidx + 1], dr = (int)dims[3 * sidx + 2];
          sref(C, k, p) = mksite(dl, d, dr, cur);
          cur += al256(8LL * dl * d * dr);
        }
        for (int p = 1; p <= nn; ++p, ++nidx) nbref(C, k, p) = nbrs[nidx];
      }
    }
    long long sidx = 0, doff = 0, cur = first;
    for (int k = 1; k <= C.n; ++k) {
      const int ns = (int)hdr[4 * (k - 1)];
      for (int p = 1; p <= ns; ++p, ++sidx) {
        const long long sz = dims[3 * sidx] * dims[3 * sidx + 1] * dims[3 * sidx + 2];
        double* dst = dptr(C, cur);
        for (long long e = T.rank(); e < sz; e += T.size()) dst[e] = data[doff + e];
        doff += sz;
        cur += al256(8 * sz);
      }
    }
    T.sync();
  } else {
    long long dpos = 0, doff = 0, nidx = 0;
    for (int k = 1; k <= C.n && !failed(C); ++k) {
      const int nd = (int)hdr[4 * (k - 1)];
      if (nd > C.maxs) { fail_all(C, CATN_ENOMEM); break; }
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

// Load, contract and report one instance in the given slot.
CATN_HDI inline void run_instance(const Team& T, char* slot, const SlotLayout& L, const InstDesc& D,
                                  const long long* i64, const int* i32, const double* dat,
                                  catn_result* res, int* trace_base, double* sws, long long sws_doubles,
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
  if (D.trace_cap > 0 && trace_base) {
    C.trace = trace_base + D.trace_off;
    C.trace_cap = D.trace_cap;
  }
  load_instance(C, D, i64, i32, dat);
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = -1; O.nsteps = 0;
  // cut_bondim! / cut_bondim_opt! calls made on the network before its
  // contraction, replayed in order (i, idx_j_in_i, opt per call); with
  // cut_only the instance stops after them and reports the discarded sum of
  // the last one as its error.
  double cut_err = 0.0;
  for (int q = 0; q < D.n_cuts && !failed(C); ++q) {
    const int* c = i32 + D.cut_off + 3LL * q;
    cut_err = cut_bond(C, c[0], c[1], c[2] != 0);
  }
  const long long t0 = clk();
  if (D.cut_only) O.err = cut_err;
  else if (!failed(C)) O = contract(C);
  prof_add(C, PROF_TOTAL, (double)(clk() - t0));
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
    res->arena_peak = C.sp_peak + 2 * C.h_peak;
    res->flops = C.acct[0];
    res->bytes = C.acct[1];
    for (int q = 0; q < PROF_SLOTS; ++q) res->prof[q] = C.acct[2 + q];
  }
  T.sync();
}

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
  if (cnt == 0) {
    if (T.leader()) *ndim = 0;
    T.sync();
    return 0;
  }
  if (cnt > 1) { fail_all(C, CATN_ESTATE); return -1; }
  const int ns = C.node[open].nsites;
  long long total = 1;
  for (int p = 1; p <= ns; ++p) total *= sref(C, open, p).d;
  SiteRef s0 = sref(C, open, 1);
  long long rmax = s0.dr;
  for (int p = 1; p <= ns; ++p) if (sref(C, open, p).dr > rmax) rmax = sref(C, open, p).dr;
  double* cur = spush(C, total * rmax);
  double* nxt = spush(C, total * rmax);
  if (failed(C)) return -1;
  copy(T, cur, sdata(C, s0), (long long)s0.d * s0.dr);
  long long pdim = s0.d;
  for (int p = 2; p <= ns; ++p) {
    SiteRef b = sref(C, open, p);
    gemm(T, pdim, (long long)b.d * b.dr, b.dl, colmajor(cur, pdim), colmajor(sdata(C, b), b.dl), colmajor(nxt, pdim));
    double* t = cur; cur = nxt; nxt = t;
    pdim *= b.d;
  }
  if (total <= cap && out) copy(T, out, cur, total);
  if (T.leader()) {
    for (int p = 1; p <= ns && p <= 64; ++p) dims[p - 1] = sref(C, open, p).d;
    *ndim = ns;
  }
  T.sync();
  return total;
}

}  // namespace catn
