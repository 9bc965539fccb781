// Internal data layout shared by the host side of libcatn_b200 and the
// device engine: per-instance input images, per-CTA slot layout, and the
// control words of one running instance.
#pragma once
#include <stdint.h>
#include "catn_b200.h"

namespace catn {

constexpr int CATN_NCLS = 40;      // arena size classes: 64 B << c

struct NodeHdr {
  int nsites;
  int nnbr;
  int cano;
  int pad;
};

struct SiteRef {
  int dl, d, dr, pad;
  long long off;   // byte offset of the (dl, d, dr) column-major tensor in the arena
};

// One pair [i, j] in the bucket of its cost (the reference's edge_count).
struct EdgeEnt {
  int cost, i, j;
  int alive;   // 1 while in its bucket
  int seq;     // insertion sequence number (bucket order = ascending seq)
  int pad;
};

// Control words of a running instance.
enum {
  CTL_STATUS = 0,   // catn_status
  CTL_FTOP = 1,     // entries on the free stack
  CTL_SPARE = 2,    // scratch counter for team atomics
  CTL_JACMAX = 3,   // max Jacobi sweeps seen
  CTL_NSTEPS = 4,
  CTL_ANOMALY = 5,  // bucket bookkeeping anomaly counter (diagnostic)
  CTL_SEQ = 6,      // next insertion sequence number
  CTL_BCAST = 7,    // scratch word for team broadcasts of small results
  CTL_WORDS = 8
};

// One instance of the input image.
struct InstDesc {
  catn_params P;
  int n;            // nodes
  int kind;         // 0 = MPS form, 1 = dense tensors (raw2mps on device),
                    // 2 = BraKet <psi|psi> (braket_node on device)
  long long hdr_off;   // int64 image: per node 4 words
                       //   MPS:   nsites, nnbr, cano, 0
                       //   dense: ndims, nnbr(=ndims), 0, 0
  long long dim_off;   // int64 image: MPS: 3 per site; dense: ndims per node
  long long nbr_off;   // int32 image: neighbours, nodes in order
  long long data_off;  // double image: tensors in order
  long long data_len;
  int trace_cap;       // records of 8 int32 (0 = no trace)
  int cost;            // work estimate (real edges) used to order the queue
  int multigraph;      // some node lists the same neighbour twice
  int rsvd_min;        // randomized-SVD route threshold (catn_params.rsvd_min_dim;
                       // 0 = the reference's 7000 / 20000)
  long long trace_off; // int32 offset into the trace buffer
  long long edge_off;  // BraKet (kind 2): int32 image, edge pairs in processing order
  int n_edges;
  int n_cuts;          // cut_bondim! calls before the contraction (kinds 0, 1)
  long long cut_off;   // int32 image: 3 words per call (i, idx_j_in_i, opt)
  int cut_only;        // 1: stop after the cuts (the error of the last one)
  int pad4;
};

// Byte layout of one CTA slot (control state + arena).
struct SlotLayout {
  int nmax, maxs, ecap, pcap;
  long long off_node, off_site, off_nbr, off_ent, off_fstack, off_emap;
  long long off_ctl, off_pairs, off_list, off_tmp, off_ameta, off_ldc, off_arena;
  int lcap, pad;
  long long arena_bytes, slot_bytes;
};

inline long long align256(long long x) { return (x + 255) & ~255LL; }

inline SlotLayout make_layout(int nmax, int maxs, int ecap, long long arena_bytes) {
  SlotLayout L;
  L.nmax = nmax;
  L.maxs = maxs;
  L.ecap = ecap;
  long long pc = (long long)maxs * (maxs + 1);
  if (pc < 2LL * ecap) pc = 2LL * ecap;
  L.pcap = (int)(pc + 64);
  L.lcap = (nmax + 1 > 2 * maxs + 2 ? nmax + 1 : 2 * maxs + 2) + 16;
  L.pad = 0;
  long long o = 0;
  long long nn = (long long)nmax + 1;
  L.off_node = o;  o = align256(o + nn * (long long)sizeof(NodeHdr));
  L.off_site = o;  o = align256(o + nn * maxs * (long long)sizeof(SiteRef));
  L.off_nbr = o;   o = align256(o + nn * maxs * 4LL);
  L.off_ent = o;   o = align256(o + (long long)ecap * (long long)sizeof(EdgeEnt));
  L.off_fstack = o; o = align256(o + (long long)ecap * 4LL);   // free stack of entry ids
  L.off_emap = o;  o = align256(o + nn * nn * 4LL);
  L.off_ctl = o;   o = align256(o + CTL_WORDS * 4LL);
  L.off_pairs = o; o = align256(o + (long long)L.pcap * 12LL);
  L.off_list = o;  o = align256(o + (long long)L.lcap * 4LL);
  L.off_tmp = o;   o = align256(o + (2LL * maxs + 8) * 4LL);
  L.off_ameta = o; o = align256(o + 64 * 8LL);   // work and cycle counters
  L.off_ldc = o;   o = align256(o + nn * 16LL);   // per-node logdim cache: value + valid flag
  L.off_arena = o;
  L.arena_bytes = arena_bytes;
  L.slot_bytes = align256(o + arena_bytes);
  return L;
}

}  // namespace catn
