// Device-side rebuild of Ising / spin-glass site tensors: the values that
// the reference's ising_network forms (src/ising.jl:95-183) -- B = exp(beta
// w s_i s_j) on the first endpoint of every edge, the identity on the
// second, the field exp(beta h s) folded into the first (or leaf) site of a
// node, 2 cosh(beta h) for a degree-0 spin -- recomputed from new couplings,
// fields and beta for a batch whose lattices and pins stay fixed.  When the
// host builds a batch (host_image.h, add_ising) it records one recipe per
// site: where the site's values go, which coupling and field they use, and
// which of the four site layouts the reference chose for it.  The device then
// evaluates the recipes (catn_ising_batch_set_params) with the same
// arithmetic, expression for expression.
#pragma once
#include "team.cuh"

namespace catn {

struct IsingSiteRecipe {
  long long dat;          // index of the site's first value in the double image
  int edge;               // coupling index into the batch's weights (-1: degree-0 spin)
  int node;               // field index into the batch's fields
  int inst;               // instance (selects its beta)
  signed char role;       // 0: first endpoint of its edge (carries B), 1: second (identity),
                          // 2: degree-0 spin
  signed char layout;     // 0 leaf (1,2,1), 1 first (1,2,2), 2 last (2,2,1), 3 interior (2,2,2)
  signed char s_own[2];   // the node's spin values after pinning (+1, -1, or 0 when pinned out)
  signed char s_other[2]; // the same for the edge's other endpoint
  short pad;
};

// Site values (column-major (dl, d, dr), at most 8 entries) of recipe r for
// coupling w, field h and inverse temperature beta; returns their count.
CATN_HD int ising_site_values(const IsingSiteRecipe& r, double w, double h, double beta, double v[8]) {
  for (int q = 0; q < 8; ++q) v[q] = 0.0;
  if (r.role == 2) {
    v[0] = exp(beta * h) + exp(-beta * h);
    return 1;
  }
  const double so[2] = {(double)r.s_own[0], (double)r.s_own[1]};
  double Q[2][2] = {{1.0, 0.0}, {0.0, 1.0}};
  if (r.role == 0) {
    const double st[2] = {(double)r.s_other[0], (double)r.s_other[1]};
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b) Q[a][b] = exp(beta * w * (so[a] * st[b]));
  }
  const double F[2] = {exp(beta * h * so[0]), exp(beta * h * so[1])};
  const double FQ[2][2] = {{F[0] * Q[0][0], F[0] * Q[0][1]}, {F[1] * Q[1][0], F[1] * Q[1][1]}};
  switch (r.layout) {
    case 0:   // leaf: the node's spin summed out
      v[0] = FQ[0][0] + FQ[1][0];
      v[1] = FQ[0][1] + FQ[1][1];
      return 2;
    case 1:   // first site: (F Q)^T as (1, 2, 2)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) v[a + 2 * b] = FQ[b][a];
      return 4;
    case 2:   // last site: Q as (2, 2, 1)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) v[a + 2 * b] = Q[a][b];
      return 4;
    default:  // interior: delta_ab Q[a, s] as (2, 2, 2)
      for (int a = 0; a < 2; ++a)
        for (int sp = 0; sp < 2; ++sp) v[a + 2 * sp + 4 * a] = Q[a][sp];
      return 8;
  }
}

// Disorder generator: a standard normal from (seed, stream, index) by the
// SplitMix64 mixing function (Steele, Lea and Flood, 2014) on a Weyl
// sequence of the counter, and the Box-Muller transform (1958) of two
// 53-bit uniforms.  Counter-based, so every entry is independent of how the
// work is split over threads, and the host can recompute any entry.
CATN_HD unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
CATN_HD double disorder_normal(unsigned long long seed, unsigned long long stream, unsigned long long index) {
  const unsigned long long key = splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ULL));
  const unsigned long long a = splitmix64(key + 2 * index), b = splitmix64(key + 2 * index + 1);
  const double u1 = (double)((a >> 11) + 1) * (1.0 / 9007199254740992.0);   // (0, 1]
  const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);         // [0, 1)
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

}  // namespace catn
