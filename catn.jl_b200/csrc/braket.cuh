// Double-layer (bra-ket) networks for <psi|psi> (reference src/braket.jl),
// contracted by one CTA like every other network.
//
// A BraKet node is an MPS node whose sites carry the ket virtual legs and
// then the bra virtual legs of one site tensor; the junction bond between
// the last ket site and the first bra site is the contracted physical index.
// The ket/bra tag of a leg rides in its neighbour id (BRA flag bit), so the
// engine's swap, cano_to and compress sweeps carry it with the site exactly
// as the reference's swap! permutes `layer` in lockstep (braket.jl:556-558).
#pragma once
#include "engine.cuh"

namespace catn {

constexpr int BRA = 1 << 30;   // neighbour-id flag of a bra leg

// Sites pos0+1 .. pos0+nax of node k from R of shape (dl0, a_1, .., a_nax,
// drlast) (column-major) by left-to-right truncated SVDs over a_1 .. a_{nax-1}
// (braket.jl:120-132 and 159-169): site q = U reshaped (dleft, a_q, c), the
// last site keeps the remainder (dleft, a_nax, drlast).
CATN_HDI inline void sweep_sites(Ctx& C, int k, int pos0, const double* data, long long dl0, const long long* ax,
                                 int nax, long long drlast) {
  const Team& T = C.T;
  const long long mark = C.sp;
  long long total = dl0 * drlast;
  for (int q = 0; q < nax; ++q) total *= ax[q];
  double* R = spush(C, total);
  if (failed(C)) return;
  copy(T, R, data, total);
  long long cur = total, dleft = dl0;
  for (int q = 0; q < nax - 1; ++q) {
    const long long m = dleft * ax[q], n = cur / m;
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
    if (T.leader()) {
      sref(C, k, pos0 + q + 1) = mksite((int)dleft, (int)ax[q], c, u);
      C.node[k].nsites = pos0 + q + 1;   // live from here on (compaction may move them)
    }
    T.sync();
    R = r2;
    cur = (long long)c * n;
    dleft = c;
  }
  if (!heap_reserve(C, al256(8 * cur))) return;
  const long long last = heap_take(C, 8 * cur);
  copy(T, dptr(C, last), R, cur);
  if (T.leader()) {
    sref(C, k, pos0 + nax) = mksite((int)dleft, (int)ax[nax - 1], (int)drlast, last);
    C.node[k].nsites = pos0 + nax;
  }
  T.sync();
  C.sp = mark;
}

// braket_node (braket.jl:75-195) from the image: per node, header (deg, d),
// dims D_1..D_deg, ket neighbours, data Tk (D_1..D_deg, d) then
// Tbra (d, D_1..D_deg).
CATN_HDI inline void load_braket(Ctx& C, const InstDesc& D, const long long* img64, const int* img32,
                                 const double* imgd) {
  const Team& T = C.T;
  const long long* hdr = img64 + D.hdr_off;
  const long long* dims = img64 + D.dim_off;
  const int* nbrs = img32 + D.nbr_off;
  const double* data = imgd + D.data_off;
  long long dpos = 0, doff = 0, nidx = 0;
  for (int k = 1; k <= C.n && !failed(C); ++k) {
    const int deg = (int)hdr[4 * (k - 1)];
    const long long d = hdr[4 * (k - 1) + 1];
    if (2 * deg > C.maxs) { fail_all(C, CATN_ENOMEM); return; }
    T.sync();
    if (T.leader()) {
      C.node[k].nnbr = 2 * deg;
      for (int p = 0; p < deg; ++p) {
        nbref(C, k, p + 1) = nbrs[nidx + p];
        nbref(C, k, deg + p + 1) = nbrs[nidx + p] | BRA;
      }
    }
    T.sync();
    long long tot = d;
    for (int q = 0; q < deg; ++q) tot *= dims[dpos + q];
    sweep_sites(C, k, 0, data + doff, 1, dims + dpos, deg, d);          // ket
    sweep_sites(C, k, deg, data + doff + tot, d, dims + dpos, deg, 1);  // bra
    if (failed(C)) return;
    T.sync();
    if (T.leader()) C.node[k].cano = 1;   // left_canonical! (braket.jl:235)
    T.sync();
    cano_to(C, k, 2 * deg);
    nidx += deg;
    dpos += deg;
    doff += 2 * tot;
  }
}

// Norm of the centre after cano_to!(end), which divides the last site
// (braket.jl:730-743); returns its log, 0 when at or below the cutoff.
CATN_HDI inline double braket_finish(Ctx& C, int k) {
  cano_to(C, k, C.node[k].nsites);
  if (failed(C)) return 0.0;
  SiteRef ctr = sref(C, k, C.node[k].cano);
  const long long ce = (long long)ctr.dl * ctr.d * ctr.dr;
  const double nrm = norm_of(C, sdata(C, ctr), ce);
  if (nrm <= C.P.cutoff) return 0.0;
  scale(C.T, sdata(C, sref(C, k, C.node[k].nsites)), 1.0 / nrm, ce);
  return log(nrm);
}

// eat! (braket.jl:638-798): contract the paired ket and bra legs of the bond
// between i and j; j's remaining sites are appended to i.
CATN_HDI inline double eat_braket(Ctx& C, int ki, int kj, double* err, double* phase) {
  const Team& T = C.T;
  const int n_i = C.node[ki].nsites, n_j = C.node[kj].nsites;
  const int bi = nb_find(C, ki, kj | BRA);
  if (bi == 0) { fail_all(C, CATN_ESTATE); return 0.0; }
  *err += move(C, ki, bi, n_i);
  const int kl = nb_find(C, ki, kj);
  if (kl == 0 || failed(C)) { fail_all(C, CATN_ESTATE); return 0.0; }
  *err += move(C, ki, kl, n_i - 1);
  cano_to(C, ki, n_i);
  const int kjj = nb_find(C, kj, ki);
  if (kjj == 0 || failed(C)) { fail_all(C, CATN_ESTATE); return 0.0; }
  *err += move(C, kj, kjj, 1);
  const int bj = nb_find(C, kj, ki | BRA);
  if (bj == 0 || failed(C)) { fail_all(C, CATN_ESTATE); return 0.0; }
  *err += move(C, kj, bj, 2);
  if (failed(C)) return 0.0;
  const long long mark = C.sp;
  const SiteRef Aik = sref(C, ki, n_i - 1), Aib = sref(C, ki, n_i);
  const SiteRef Ajk = sref(C, kj, 1), Ajb = sref(C, kj, 2);
  const long long dl = Aik.dl, Dk = Aik.d, Db = Aib.d, dr = Ajb.dr;
  double* Wi = spush(C, dl * Dk * Db);
  double* Wj = spush(C, Dk * Db * dr);
  double* mat = spush(C, dl * dr);
  if (failed(C)) return 0.0;
  gemm(T, dl * Dk, Db, Aik.dr, colmajor(sdata(C, Aik), dl * Dk), colmajor(sdata(C, Aib), Aik.dr),
       colmajor(Wi, dl * Dk));
  gemm(T, Dk, Db * dr, Ajk.dr, colmajor(sdata(C, Ajk), Dk), colmajor(sdata(C, Ajb), Ajk.dr), colmajor(Wj, Dk));
  gemm(T, dl, dr, Dk * Db, colmajor(Wi, dl), colmajor(Wj, Dk * Db), colmajor(mat, dl));
  account(C, 2.0 * dl * Dk * Db * Aik.dr + 2.0 * Dk * Db * dr * Ajk.dr + 2.0 * dl * dr * Dk * Db,
          8.0 * ((double)dl * Dk * Aik.dr + (double)Aik.dr * Db + (double)Dk * Ajk.dr + (double)Ajk.dr * Db * dr));
  if (n_i == 2 && n_j == 2) {
    // (A) both nodes exhausted: a scalar
    const double z = sumv(T, mat, dl * dr);
    T.sync();
    if (T.leader()) {
      C.node[ki].nsites = 0;
      C.node[ki].nnbr = 0;
    }
    T.sync();
    C.sp = mark;
    const double az = fabs(z);
    if (az <= C.P.cutoff) return 0.0;
    *phase *= z / az;
    return log(az);
  }
  if (n_i == 2) {
    // (B) i exhausted: mat (1 x dr) prefixes j's third site
    const SiteRef s3 = sref(C, kj, 3);
    const long long cols = (long long)s3.d * s3.dr;
    if (!heap_reserve(C, al256(8 * cols))) return 0.0;
    const long long f = heap_take(C, 8 * cols);
    gemm(T, 1, cols, dr, colmajor(mat, 1), colmajor(sdata(C, sref(C, kj, 3)), dr), colmajor(dptr(C, f), 1));
    T.sync();
    if (T.leader()) {
      const int ns = n_j - 2;
      sref(C, ki, 1) = mksite(1, s3.d, s3.dr, f);
      for (int p = 2; p <= ns; ++p) sref(C, ki, p) = sref(C, kj, p + 2);
      const int nn = C.node[kj].nnbr - 2;
      for (int p = 1; p <= nn; ++p) nbref(C, ki, p) = nbref(C, kj, p + 2);
      C.node[ki].nsites = ns;
      C.node[ki].nnbr = nn;
      C.node[ki].cano = 1;
      C.node[kj].nsites = 0;
    }
    T.sync();
    C.sp = mark;
    return braket_finish(C, ki);
  }
  // (C) / (D): mat folded into i's site n_i - 2, i's last two sites dropped,
  // j's sites 3:end appended
  const SiteRef pv = sref(C, ki, n_i - 2);
  const long long pr = (long long)pv.dl * pv.d;
  if (!heap_reserve(C, al256(8 * pr * dr))) return 0.0;
  const long long f = heap_take(C, 8 * pr * dr);
  gemm(T, pr, dr, dl, colmajor(sdata(C, sref(C, ki, n_i - 2)), pr), colmajor(mat, dl), colmajor(dptr(C, f), pr));
  T.sync();
  if (T.leader()) {
    const int base = n_i - 2;
    const int add = n_j - 2;
    const int nni = C.node[ki].nnbr - 2, nnj = C.node[kj].nnbr - 2;
    if (base + add > C.maxs || nni + nnj > C.maxs) {
      fail_leader(C, CATN_ENOMEM);
    } else {
      sref(C, ki, base) = mksite(pv.dl, pv.d, (int)dr, f);
      for (int p = 1; p <= add; ++p) sref(C, ki, base + p) = sref(C, kj, p + 2);
      for (int p = 1; p <= nnj; ++p) nbref(C, ki, nni + p) = nbref(C, kj, p + 2);
      C.node[ki].nsites = base + add;
      C.node[ki].nnbr = nni + nnj;
      C.node[ki].cano = base;
      C.node[kj].nsites = 0;
    }
  }
  refresh_status(C);
  C.sp = mark;
  if (failed(C)) return 0.0;
  return braket_finish(C, ki);
}

// contraction! of a BraKet network (braket.jl:960-1078): the first remaining
// edge each step, j absorbed into i (order(i) >= order(j)), compress(_opt)!
// of i, the eaten edge removed and every edge (and neighbour id) naming j
// re-pointed to i; finally the norms of the remaining nodes.
//
// With P.braket_loops (no reference counterpart: the reference rejects
// cycles, braket.jl:405-420), a neighbour k of both i and j now holds two
// doubled bonds to i.  The re-pointed edge is dropped from the list, and the
// pair is fused as merge! fuses a duplicate bond (mps_node.jl:595-622): in k
// the ket legs, then the bra legs, each in the order (i's bond, j's bond)
// (`cross` from their positions before the re-pointing, as
// tensor_network.jl:641-650 does); then the same two fusions in i, whose
// own legs precede the ones it took from j.  After the fusions of a step, i
// is compressed once more.
CATN_HDI inline ContractOut contract_braket(Ctx& C, const int* edges0, int ne0) {
  const Team& T = C.T;
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = 0; O.nsteps = 0;
  int* E = C.pairs;   // live edge list: (i, j) pairs
  for (int e = T.rank(); e < 2 * ne0; e += T.size()) E[e] = edges0[e];
  T.sync();
  int ne = ne0;
  int maxdim = 0;
  while (ne > 0 && !failed(C)) {
    if (O.nsteps > ne0 + 4) { fail_all(C, CATN_ESTATE); break; }
    int i = E[0], j = E[1];
    if (C.node[j].nsites > C.node[i].nsites) { int t = i; i = j; j = t; }
    const double lnv = eat_braket(C, i, j, &O.err, &O.psi);
    O.lnZ += lnv;
    if (failed(C)) break;
    O.err += compress_node(C, i, C.P.svdopt != 0);
    if (failed(C)) break;
    for (int p = 1; p <= C.node[i].nsites; ++p) if (sref(C, i, p).d > maxdim) maxdim = sref(C, i, p).d;
    int* dup = C.list;   // [0] count, then (k, cross bits) pairs
    T.sync();
    if (T.leader()) {
      // drop the eaten edge, re-point the ones naming j (and j's neighbours' ids)
      int w = 0, nd = 0;
      for (int e = 0; e < ne; ++e) {
        int a = E[2 * e], b = E[2 * e + 1];
        if ((a == i && b == j) || (a == j && b == i)) continue;
        if (a == j || b == j) {
          const int other = a == j ? b : a;
          const int xk = nb_find(C, other, i), yk = nb_find(C, other, j);
          const int xb = nb_find(C, other, i | BRA), yb = nb_find(C, other, j | BRA);
          const int nn = C.node[other].nnbr;
          for (int p = 1; p <= nn; ++p) {
            const int v = nbref(C, other, p);
            if ((v & ~BRA) == j) nbref(C, other, p) = i | (v & BRA);
          }
          if (xk > 0) {   // a second doubled bond between i and other (loops only)
            dup[1 + 2 * nd] = other;
            dup[2 + 2 * nd] = (xk > yk ? 1 : 0) | (xb > yb ? 2 : 0);
            ++nd;
            continue;
          }
          if (a == j) a = i; else b = i;
        }
        E[2 * w] = a;
        E[2 * w + 1] = b;
        ++w;
      }
      dup[0] = nd;
      C.ctl[CTL_BCAST] = w;
      C.node[j].nsites = 0;
      C.node[j].nnbr = 0;
      if (nd > 0 && !C.P.braket_loops) fail_leader(C, CATN_ESTATE);
    }
    refresh_status(C);
    ne = C.ctl[CTL_BCAST];
    const int nd = dup[0];
    for (int q = 0; q < nd && !failed(C); ++q) {
      const int k = dup[1 + 2 * q], cr = dup[2 + 2 * q];
      O.err += merge_dup(C, k, i, (cr & 1) != 0);
      if (!failed(C)) O.err += merge_dup(C, k, i | BRA, (cr & 2) != 0);
      if (!failed(C)) O.err += merge_dup(C, i, k, false);
      if (!failed(C)) O.err += merge_dup(C, i, k | BRA, false);
      for (int p = 1; p <= C.node[k].nsites; ++p) if (sref(C, k, p).d > maxdim) maxdim = sref(C, k, p).d;
    }
    if (nd > 0 && !failed(C)) {
      O.err += compress_node(C, i, C.P.svdopt != 0);
      for (int p = 1; p <= C.node[i].nsites; ++p) if (sref(C, i, p).d > maxdim) maxdim = sref(C, i, p).d;
    }
    if (failed(C)) break;
    const int nsi = C.node[i].nsites;
    unsigned shh = 2166136261u, lyh = 2166136261u;
    for (int p = 1; p <= nsi; ++p) {
      shh = fnv_step(shh, sref(C, i, p).d);
      lyh = fnv_step(lyh, (nbref(C, i, p) & BRA) ? 0 : 1);
    }
    T.sync();
    if (T.leader() && C.trace && O.nsteps < C.trace_cap) {
      int* r = C.trace + 8LL * O.nsteps;
      r[0] = i; r[1] = j; r[2] = 0; r[3] = (int)lyh; r[4] = nd; r[5] = nsi; r[6] = (int)shh; r[7] = maxdim;
    }
    T.sync();
    O.nsteps += 1;
  }
  // braket_lognorm (braket.jl:915-940)
  for (int k = 1; k <= C.n && !failed(C); ++k) {
    if (C.node[k].nsites == 0) continue;
    cano_to(C, k, C.node[k].nsites);
    if (failed(C)) break;
    SiteRef ctr = sref(C, k, C.node[k].cano);
    const double nrm = norm_of(C, sdata(C, ctr), (long long)ctr.dl * ctr.d * ctr.dr);
    if (nrm > C.P.cutoff) O.lnZ += log(nrm);
  }
  O.maxdim = maxdim;
  return O;
}

// Load, contract and report one BraKet instance in the given slot.
CATN_HDI inline void run_instance_braket(const Team& T, char* slot, const SlotLayout& L, const InstDesc& D,
                                         const long long* i64, const int* i32, const double* dat, catn_result* res,
                                         int* trace_base, double* sws, long long sws_doubles) {
  Ctx C = make_ctx(T, slot, L, D.P, D.n, sws, sws_doubles);
  C.rsvd_min = D.rsvd_min;
  reset_slot(C);
  if (D.trace_cap > 0 && trace_base) {
    C.trace = trace_base + D.trace_off;
    C.trace_cap = D.trace_cap;
  }
  if (D.kind != 2 || 2LL * D.n_edges > 3LL * C.pcap) fail_all(C, CATN_EINVAL);
  if (!failed(C)) load_braket(C, D, i64, i32, dat);
  ContractOut O;
  O.lnZ = 0.0; O.err = 0.0; O.psi = 1.0; O.sign = 1.0; O.maxdim = 0; O.nsteps = 0;
  const long long t0 = clk();
  if (!failed(C)) O = contract_braket(C, i32 + D.edge_off, D.n_edges);
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

}  // namespace catn
