// Host-side construction of the packed input image that the device engine
// loads: networks in MPS form, dense-tensor networks (raw2mps on device) and
// the Ising / spin-glass builder of the reference (src/ising.jl:20-227).
#pragma once
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>
#include "catn_layout.h"
#include "ising_build.cuh"

namespace catn {

// Parameters of one Ising instance, kept on the host for the chain rule of
// the adjoint (ising_param_grad).
struct IsingSpec {
  int n = 0;
  std::vector<int> edges;
  std::vector<double> w, h;
  double beta = 0.0;
  int pos1 = 0, val1 = 0, pos2 = 0, val2 = 0;
  int inst = -1;   // index into Image::desc
};

struct Image {
  std::vector<long long> i64;
  std::vector<int> i32;
  std::vector<double> dat;
  std::vector<InstDesc> desc;
  int nmax = 0;       // largest node count
  int emax = 0;       // largest real-edge count
  int smax = 0;       // largest per-node site / neighbour count at load
  long long trace_total = 0;
  std::vector<IsingSpec> ising;   // Ising instances, in the order added
  // Site recipes of the Ising instances added with recording on
  // (ising_build.cuh), in image order.
  std::vector<IsingSiteRecipe> recipes;

  // Network in MPS form.  Returns an error message or "".
  std::string add_mps(const catn_params& P, int n, const int* site_counts, const int* nbr_counts,
                      const int* canos, const long long* site_dims, const double* site_data,
                      const int* neighbors, int trace_cap) {
    if (n < 1) return "network has no nodes";
    InstDesc D;
    std::memset(&D, 0, sizeof(D));
    D.P = P;
    D.n = n;
    D.kind = 0;
    D.hdr_off = (long long)i64.size();
    long long nsites = 0, nnb = 0;
    for (int k = 0; k < n; ++k) {
      if (site_counts[k] < 0 || nbr_counts[k] < 0) return "negative site/neighbour count";
      i64.push_back(site_counts[k]);
      i64.push_back(nbr_counts[k]);
      i64.push_back(canos[k]);
      i64.push_back(0);
      nsites += site_counts[k];
      nnb += nbr_counts[k];
      if (site_counts[k] > smax) smax = site_counts[k];
      if (nbr_counts[k] > smax) smax = nbr_counts[k];
    }
    D.dim_off = (long long)i64.size();
    long long ndata = 0;
    for (long long s = 0; s < nsites; ++s) {
      long long dl = site_dims[3 * s], d = site_dims[3 * s + 1], dr = site_dims[3 * s + 2];
      if (dl < 1 || d < 1 || dr < 1) return "site dimensions must be >= 1";
      i64.push_back(dl);
      i64.push_back(d);
      i64.push_back(dr);
      ndata += dl * d * dr;
    }
    D.nbr_off = (long long)i32.size();
    int edges2 = 0;
    for (long long q = 0; q < nnb; ++q) {
      int v = neighbors[q];
      if (v > n) return "neighbour id out of range";
      if (v > 0) ++edges2;
      i32.push_back(v);
    }
    D.data_off = (long long)dat.size();
    D.data_len = ndata;
    dat.insert(dat.end(), site_data, site_data + ndata);
    D.multigraph = has_repeats(n, nbr_counts, neighbors);
    finish(D, n, edges2 / 2 + 1, trace_cap);
    return "";
  }

  // Does any node list the same neighbour twice?
  static int has_repeats(int n, const int* counts, const int* neighbors) {
    long long pos = 0;
    for (int k = 0; k < n; ++k) {
      std::set<int> seen;
      for (int q = 0; q < counts[k]; ++q, ++pos) {
        int v = neighbors[pos];
        if (v > 0 && !seen.insert(v).second) return 1;
      }
    }
    return 0;
  }

  // Network of dense tensors; raw2mps runs on the device.
  std::string add_dense(const catn_params& P, int n, const int* ndims, const long long* dims,
                        const double* data, const int* neighbors, int trace_cap) {
    if (n < 1) return "network has no nodes";
    InstDesc D;
    std::memset(&D, 0, sizeof(D));
    D.P = P;
    D.n = n;
    D.kind = 1;
    D.hdr_off = (long long)i64.size();
    long long nd_tot = 0;
    for (int k = 0; k < n; ++k) {
      i64.push_back(ndims[k]);
      i64.push_back(ndims[k]);
      i64.push_back(0);
      i64.push_back(0);
      nd_tot += ndims[k];
      if (ndims[k] > smax) smax = ndims[k];
    }
    D.dim_off = (long long)i64.size();
    long long pos = 0, ndata = 0;
    for (int k = 0; k < n; ++k) {
      long long tot = 1;
      for (int q = 0; q < ndims[k]; ++q) {
        if (dims[pos + q] < 1) return "tensor dimensions must be >= 1";
        i64.push_back(dims[pos + q]);
        tot *= dims[pos + q];
      }
      pos += ndims[k];
      ndata += tot;   // a 0-d tensor holds one value
    }
    D.nbr_off = (long long)i32.size();
    int edges2 = 0;
    for (long long q = 0; q < nd_tot; ++q) {
      int v = neighbors[q];
      if (v > n) return "neighbour id out of range";
      if (v > 0) ++edges2;
      i32.push_back(v);
    }
    D.data_off = (long long)dat.size();
    D.data_len = ndata;
    dat.insert(dat.end(), data, data + ndata);
    D.multigraph = has_repeats(n, ndims, neighbors);
    finish(D, n, edges2 / 2 + 1, trace_cap);
    return "";
  }

  // braket_network (src/braket.jl:369-508) for real tensors: `labels` holds
  // one positive label per axis, tensors in order.  A label on one tensor is
  // that tensor's physical index (exactly one per tensor), on two tensors a
  // virtual bond; cyclic bond graphs are rejected.  Per node the image holds
  // (deg, d), the virtual dims, the ket neighbours in axis order and the
  // data Tk (virtual axes, then physical) followed by Tbra (physical, then
  // virtual); the edges follow the first appearance of their labels.
  std::string add_braket(const catn_params& P, int n, const int* ndims, const long long* dims, const double* data,
                         const int* labels, int trace_cap) {
    if (n < 1) return "braket_network: no tensors";
    std::vector<long long> aoff(n + 1, 0), doff(n + 1, 0);
    for (int k = 0; k < n; ++k) {
      if (ndims[k] < 1) return "braket_network: every tensor needs at least one index";
      aoff[k + 1] = aoff[k] + ndims[k];
      long long tot = 1;
      for (int q = 0; q < ndims[k]; ++q) {
        if (dims[aoff[k] + q] < 1) return "tensor dimensions must be >= 1";
        tot *= dims[aoff[k] + q];
      }
      doff[k + 1] = doff[k] + tot;
    }
    // label -> owners (node ids), in first-appearance order
    std::vector<int> order;
    std::vector<std::vector<int>> owners;
    std::vector<int> label_of;   // index into owners by label position
    auto find_label = [&](int l) {
      for (size_t q = 0; q < order.size(); ++q)
        if (order[q] == l) return (int)q;
      return -1;
    };
    for (int k = 0; k < n; ++k)
      for (int q = 0; q < ndims[k]; ++q) {
        const int l = labels[aoff[k] + q];
        int x = find_label(l);
        if (x < 0) {
          order.push_back(l);
          owners.push_back({});
          x = (int)order.size() - 1;
        }
        owners[x].push_back(k + 1);
        label_of.push_back(x);
      }
    for (size_t x = 0; x < order.size(); ++x)
      if (owners[x].size() > 2)
        return "braket_network: label " + std::to_string(order[x]) + " appears " +
               std::to_string(owners[x].size()) + " times (expected 1 or 2)";
    for (int k = 0; k < n; ++k) {
      int nphys = 0;
      for (int q = 0; q < ndims[k]; ++q) nphys += owners[label_of[aoff[k] + q]].size() == 1;
      if (nphys != 1)
        return "braket_network: tensor " + std::to_string(k + 1) + " has " + std::to_string(nphys) +
               " physical (open) labels, expected 1";
    }
    std::vector<int> parent(n + 1);
    for (int k = 0; k <= n; ++k) parent[k] = k;
    auto root = [&](int x) {
      while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
      return x;
    };
    std::vector<int> epairs;
    for (size_t x = 0; x < order.size(); ++x) {
      if (owners[x].size() != 2) continue;
      const int u = owners[x][0], v = owners[x][1];
      if (P.braket_loops) {
        // cycles of three or more nodes are contracted; two labels on the
        // same pair of tensors (a parallel bond) are not
        for (size_t q = 0; q + 1 < epairs.size(); q += 2)
          if ((epairs[q] == u && epairs[q + 1] == v) || (epairs[q] == v && epairs[q + 1] == u))
            return "braket_network: tensors " + std::to_string(u) + " and " + std::to_string(v) +
                   " share more than one label (parallel bonds are not supported)";
      } else {
        const int a = root(u), b = root(v);
        if (a == b)
          return "braket_network: virtual-bond graph contains a cycle — cyclic graphs are not supported in v1";
        parent[a] = b;
      }
      epairs.push_back(u);
      epairs.push_back(v);
    }
    InstDesc D;
    std::memset(&D, 0, sizeof(D));
    D.P = P;
    D.n = n;
    D.kind = 2;
    D.hdr_off = (long long)i64.size();
    std::vector<int> phys(n);
    for (int k = 0; k < n; ++k) {
      for (int q = 0; q < ndims[k]; ++q)
        if (owners[label_of[aoff[k] + q]].size() == 1) phys[k] = q;
      i64.push_back(ndims[k] - 1);
      i64.push_back(dims[aoff[k] + phys[k]]);
      i64.push_back(0);
      i64.push_back(0);
      if (2 * (ndims[k] - 1) > smax) smax = 2 * (ndims[k] - 1);
    }
    D.dim_off = (long long)i64.size();
    for (int k = 0; k < n; ++k)
      for (int q = 0; q < ndims[k]; ++q)
        if (q != phys[k]) i64.push_back(dims[aoff[k] + q]);
    D.nbr_off = (long long)i32.size();
    for (int k = 0; k < n; ++k)
      for (int q = 0; q < ndims[k]; ++q) {
        if (q == phys[k]) continue;
        const std::vector<int>& o = owners[label_of[aoff[k] + q]];
        i32.push_back(o[0] == k + 1 ? o[1] : o[0]);
      }
    D.edge_off = (long long)i32.size();
    D.n_edges = (int)(epairs.size() / 2);
    for (int v : epairs) i32.push_back(v);
    D.data_off = (long long)dat.size();
    for (int k = 0; k < n; ++k) {
      const int nd = ndims[k];
      const long long* dk = dims + aoff[k];
      std::vector<long long> stride(nd, 1), perm;
      for (int q = 1; q < nd; ++q) stride[q] = stride[q - 1] * dk[q - 1];
      for (int q = 0; q < nd; ++q)
        if (q != phys[k]) perm.push_back(q);
      perm.push_back(phys[k]);
      const long long tot = doff[k + 1] - doff[k];
      const double* src = data + doff[k];
      // Tk(i_perm0, .., i_perm(nd-1)) = Ti(...) and Tbra(p, v...) = Tk(v..., p)
      std::vector<double> tk(tot), tb(tot);
      std::vector<long long> idx(nd, 0);
      const long long d = dk[phys[k]];
      for (long long e = 0; e < tot; ++e) {
        long long so = 0;
        for (int q = 0; q < nd; ++q) so += idx[perm[q]] * stride[perm[q]];
        tk[e] = src[so];
        const long long pi = idx[perm[nd - 1]];
        tb[pi + d * (e % (tot / d))] = src[so];
        for (int q = 0; q < nd; ++q) {   // next multi-index in Tk order
          if (++idx[perm[q]] < dk[perm[q]]) break;
          idx[perm[q]] = 0;
        }
      }
      dat.insert(dat.end(), tk.begin(), tk.end());
      dat.insert(dat.end(), tb.begin(), tb.end());
    }
    D.data_len = (long long)dat.size() - D.data_off;
    finish(D, n, D.n_edges + 1, trace_cap);
    return "";
  }

  // ising_network (src/ising.jl:20-227): one site per incident edge, B =
  // exp(beta w s_i s_j) on the first endpoint, identity on the second, field
  // folded into the first (or leaf) site, degree-0 spins as 2cosh(beta h).
  // With rec_edge_base >= 0 one recipe per site goes to `recipes`, its
  // coupling and field indices offset by rec_edge_base and rec_node_base
  // (the instance's place in the batch's weights and fields).
  std::string add_ising(const catn_params& P, int n, int n_edges, const int* edges, const double* w,
                        const double* h, double beta, int pos1, int val1, int pos2, int val2,
                        int trace_cap, long long rec_edge_base = -1, long long rec_node_base = -1) {
    if (n < 1) return "ising_network: n must be >= 1";
    std::vector<int> degree(n + 1, 0);
    for (int e = 0; e < n_edges; ++e) {
      int i = edges[2 * e], j = edges[2 * e + 1];
      if (i < 1 || i > n || j < 1 || j > n) return "ising_network: edge endpoint out of range";
      degree[i] += 1;
      degree[j] += 1;
    }
    if ((pos1 != 0 && (val1 < 1 || val1 > 2)) || (pos2 != 0 && (val2 < 1 || val2 > 2)))
      return "ising_network: pinned value must be 1 or 2";
    struct Site { int dl, d, dr; double v[8]; };
    std::vector<std::vector<Site>> mps(n + 1);
    std::vector<std::vector<int>> nbr(n + 1);
    const bool record = rec_edge_base >= 0;
    std::vector<std::vector<IsingSiteRecipe>> rec(record ? n + 1 : 0);
    // the site layout build_site picks for `node` (leaf / first / last / interior)
    auto layout_of = [&](int node) -> int {
      if (degree[node] == 1) return 0;
      if (nbr[node].empty()) return 1;
      if ((int)nbr[node].size() == degree[node] - 1) return 2;
      return 3;
    };
    auto recipe = [&](int e, int node, int role, const double* own, const double* other) {
      IsingSiteRecipe r;
      std::memset(&r, 0, sizeof(r));
      r.edge = e < 0 ? -1 : (int)(rec_edge_base + e);
      r.node = (int)(rec_node_base + node - 1);
      r.inst = (int)desc.size();
      r.role = (signed char)role;
      r.layout = (signed char)(role == 2 ? 0 : layout_of(node));
      if (own) { r.s_own[0] = (signed char)own[0]; r.s_own[1] = (signed char)own[1]; }
      if (other) { r.s_other[0] = (signed char)other[0]; r.s_other[1] = (signed char)other[1]; }
      rec[node].push_back(r);
    };
    auto build_site = [&](int node, double field_diag[2], const double Q[2][2]) -> Site {
      Site s;
      std::memset(&s, 0, sizeof(s));
      int deg = degree[node];
      // F*Q with F = diag(field)
      double FQ[2][2] = {{field_diag[0] * Q[0][0], field_diag[0] * Q[0][1]},
                         {field_diag[1] * Q[1][0], field_diag[1] * Q[1][1]}};
      if (deg == 1) {
        // leaf: sum over spin_i -> (1, 2, 1)
        s.dl = 1; s.d = 2; s.dr = 1;
        s.v[0] = FQ[0][0] + FQ[1][0];
        s.v[1] = FQ[0][1] + FQ[1][1];
      } else if (nbr[node].empty()) {
        // first: reshape((F*Q)', 1, 2, 2): site[0, a, b] = (F Q)[b, a]
        s.dl = 1; s.d = 2; s.dr = 2;
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) s.v[a + 2 * b] = FQ[b][a];
      } else if ((int)nbr[node].size() == deg - 1) {
        // last: reshape(Q, 2, 2, 1): site[a, s, 0] = Q[a, s]
        s.dl = 2; s.d = 2; s.dr = 1;
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) s.v[a + 2 * b] = Q[a][b];
      } else {
        // interior: t3[a, s, b] = delta_ab Q[a, s]
        s.dl = 2; s.d = 2; s.dr = 2;
        for (int a = 0; a < 2; ++a)
          for (int sp = 0; sp < 2; ++sp) s.v[a + 2 * sp + 4 * a] = Q[a][sp];
      }
      return s;
    };
    for (int e = 0; e < n_edges; ++e) {
      int i = edges[2 * e], j = edges[2 * e + 1];
      double si[2] = {1.0, -1.0}, sj[2] = {1.0, -1.0};
      if (i == pos1) si[val1 - 1] = 0.0;
      else if (i == pos2) si[val2 - 1] = 0.0;
      if (j == pos1) sj[val1 - 1] = 0.0;
      else if (j == pos2) sj[val2 - 1] = 0.0;
      double B[2][2], I2[2][2] = {{1.0, 0.0}, {0.0, 1.0}};
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) B[a][b] = std::exp(beta * w[e] * (si[a] * sj[b]));
      double fi[2] = {std::exp(beta * h[i - 1] * si[0]), std::exp(beta * h[i - 1] * si[1])};
      if (record) recipe(e, i, 0, si, sj);
      mps[i].push_back(build_site(i, fi, B));
      nbr[i].push_back(j);
      double fj[2] = {std::exp(beta * h[j - 1] * sj[0]), std::exp(beta * h[j - 1] * sj[1])};
      if (record) recipe(e, j, 1, sj, si);
      mps[j].push_back(build_site(j, fj, I2));
      nbr[j].push_back(i);
    }
    std::vector<int> sc(n), nc(n), cn(n);
    std::vector<long long> dims;
    std::vector<double> data;
    std::vector<int> nb;
    for (int k = 1; k <= n; ++k) {
      if (degree[k] == 0) {
        Site s;
        std::memset(&s, 0, sizeof(s));
        s.dl = s.d = s.dr = 1;
        s.v[0] = std::exp(beta * h[k - 1]) + std::exp(-beta * h[k - 1]);
        mps[k].push_back(s);
        if (record) recipe(-1, k, 2, nullptr, nullptr);
      }
      sc[k - 1] = (int)mps[k].size();
      nc[k - 1] = (int)nbr[k].size();
      cn[k - 1] = (int)mps[k].size();
      for (size_t q0 = 0; q0 < mps[k].size(); ++q0) {
        const Site& s = mps[k][q0];
        if (record) rec[k][q0].dat = (long long)data.size();   // made absolute below
        dims.push_back(s.dl);
        dims.push_back(s.d);
        dims.push_back(s.dr);
        for (int q = 0; q < s.dl * s.d * s.dr; ++q) data.push_back(s.v[q]);
      }
      for (int v : nbr[k]) nb.push_back(v);
    }
    std::string err = add_mps(P, n, sc.data(), nc.data(), cn.data(), dims.data(), data.data(), nb.data(), trace_cap);
    if (err.empty() && record) {
      const long long base = desc.back().data_off;
      for (int k = 1; k <= n; ++k)
        for (IsingSiteRecipe r : rec[k]) {
          r.dat += base;
          recipes.push_back(r);
        }
    }
    if (err.empty()) {
      IsingSpec sp;
      sp.n = n;
      sp.edges.assign(edges, edges + 2 * n_edges);
      sp.w.assign(w, w + n_edges);
      sp.h.assign(h, h + n);
      sp.beta = beta;
      sp.pos1 = pos1; sp.val1 = val1; sp.pos2 = pos2; sp.val2 = val2;
      sp.inst = (int)desc.size() - 1;
      ising.push_back(sp);
    }
    return err;
  }

  // Neighbour list of node k (1-based) of the first instance, from the
  // image (MPS and dense forms; empty for BraKet images or a bad k).
  std::vector<int> neighbors_of(int k) const {
    std::vector<int> out;
    if (desc.empty() || desc[0].kind == 2 || k < 1 || k > desc[0].n) return out;
    const InstDesc& D = desc[0];
    const int col = D.kind == 0 ? 1 : 0;   // MPS: nnbr is word 1; dense: ndims (word 0)
    long long off = D.nbr_off;
    for (int q = 1; q < k; ++q) off += i64[D.hdr_off + 4 * (q - 1) + col];
    const long long nn = i64[D.hdr_off + 4 * (k - 1) + col];
    for (long long p = 0; p < nn; ++p) out.push_back(i32[off + p]);
    return out;
  }

  // The cut_bondim! calls (3 words each: i, idx_j_in_i, opt) replayed before
  // the first instance's contraction, kept at the end of the int32 image.
  void set_cuts(const std::vector<int>& cuts) {
    InstDesc& D = desc[0];
    if (D.n_cuts > 0) i32.resize((size_t)D.cut_off);
    D.cut_off = (long long)i32.size();
    D.n_cuts = (int)(cuts.size() / 3);
    i32.insert(i32.end(), cuts.begin(), cuts.end());
  }

 private:
  void finish(InstDesc& D, int n, int edges, int trace_cap) {
    // the randomized-SVD route's size threshold (0: the reference's)
    D.rsvd_min = D.P.rsvd_min_dim;
    D.trace_cap = trace_cap;
    D.cost = edges;
    D.trace_off = trace_total;
    trace_total += 8LL * trace_cap;
    desc.push_back(D);
    if (n > nmax) nmax = n;
    if (edges > emax) emax = edges;
  }
};

// d lnZ / d w_e and d lnZ / d h_k from the gradients of the sites that
// add_ising built (`gsite`: same order and layout as its data), by the chain
// rule through B = exp(beta w s_i s_j) on the first endpoint's site and the
// field factors exp(beta h s) folded into each node's first (or leaf) site.
// Follows add_ising's construction step by step.
inline void ising_param_grad(int n, int n_edges, const int* edges, const double* w, const double* h, double beta,
                             int pos1, int val1, int pos2, int val2, const double* gsite, double* dw, double* dh) {
  std::vector<int> degree(n + 1, 0);
  for (int e = 0; e < n_edges; ++e) {
    degree[edges[2 * e]] += 1;
    degree[edges[2 * e + 1]] += 1;
  }
  // one entry per site, in the order add_ising pushes them per node
  struct SiteInfo { int edge, layout; bool isB; double s[2], other[2], f[2]; };   // layout: 0 leaf 1 first 2 last 3 interior
  std::vector<std::vector<SiteInfo>> sites(n + 1);
  auto spins = [&](int k, double s[2]) {
    s[0] = 1.0;
    s[1] = -1.0;
    if (k == pos1) s[val1 - 1] = 0.0;
    else if (k == pos2) s[val2 - 1] = 0.0;
  };
  auto layout_of = [&](int k) {
    if (degree[k] == 1) return 0;
    if (sites[k].empty()) return 1;
    if ((int)sites[k].size() == degree[k] - 1) return 2;
    return 3;
  };
  for (int e = 0; e < n_edges; ++e) {
    const int i = edges[2 * e], j = edges[2 * e + 1];
    SiteInfo a, b;
    spins(i, a.s);
    spins(j, a.other);
    a.edge = e; a.isB = true; a.layout = layout_of(i);
    for (int q = 0; q < 2; ++q) a.f[q] = std::exp(beta * h[i - 1] * a.s[q]);
    sites[i].push_back(a);
    spins(j, b.s);
    spins(i, b.other);
    b.edge = e; b.isB = false; b.layout = layout_of(j);
    for (int q = 0; q < 2; ++q) b.f[q] = std::exp(beta * h[j - 1] * b.s[q]);
    sites[j].push_back(b);
  }
  for (int e = 0; e < n_edges; ++e) dw[e] = 0.0;
  for (int k = 0; k < n; ++k) dh[k] = 0.0;
  long long off = 0;
  for (int k = 1; k <= n; ++k) {
    if (degree[k] == 0) {
      dh[k - 1] += gsite[off] * beta * (std::exp(beta * h[k - 1]) - std::exp(-beta * h[k - 1]));
      off += 1;
      continue;
    }
    for (const SiteInfo& si : sites[k]) {
      const int e = si.edge;
      double Q[2][2];
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          Q[a][b] = si.isB ? std::exp(beta * w[e] * (si.s[a] * si.other[b])) : (a == b ? 1.0 : 0.0);
      double Qb[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, fb[2] = {0.0, 0.0};
      const double* G = gsite + off;
      if (si.layout == 0) {          // v[b] = sum_a f_a Q[a][b]
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            Qb[a][b] = G[b] * si.f[a];
            fb[a] += G[b] * Q[a][b];
          }
        off += 2;
      } else if (si.layout == 1) {   // v[a + 2b] = f_b Q[b][a]
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            Qb[b][a] = G[a + 2 * b] * si.f[b];
            fb[b] += G[a + 2 * b] * Q[b][a];
          }
        off += 4;
      } else if (si.layout == 2) {   // v[a + 2b] = Q[a][b]
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) Qb[a][b] = G[a + 2 * b];
        off += 4;
      } else {                       // v[a + 2 sp + 4 a] = Q[a][sp]
        for (int a = 0; a < 2; ++a)
          for (int sp = 0; sp < 2; ++sp) Qb[a][sp] = G[a + 2 * sp + 4 * a];
        off += 8;
      }
      if (si.isB) {
        double g = 0.0;
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) g += Qb[a][b] * beta * si.s[a] * si.other[b] * Q[a][b];
        dw[e] += g;
      }
      if (si.layout <= 1)
        for (int a = 0; a < 2; ++a) dh[k - 1] += fb[a] * beta * si.s[a] * si.f[a];
    }
  }
}

// Site / neighbour capacity per node: the largest order a node can reach
// is bounded by its initial order plus everything it can absorb.
inline int default_maxs(const Image& im) {
  int m = 128;
  if (im.smax + 8 > m) m = im.smax + 8;
  return m;
}

}  // namespace catn
