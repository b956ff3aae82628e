// Host symbolic phase of the B200 sparse direct solver: fill-reducing orderings and the supernodal symbolic analysis.
// The results are bit-identical to the reference's (jwt625/applied-multiphysics packages/core/src/la/sparse.mjs
// amdOrder / ndOrder / analyze and order3d.mjs nd3Order): same permutation, elimination tree, column counts,
// relaxed supernodes and row structures. Only the host-side organisation differs (nested-dissection leaves are
// ordered in parallel worker threads; the output positions are fixed before the workers run, so the result does not
// depend on the thread count).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace amp {

struct Pattern {  // full symmetric CSR, sorted rows, diagonal present (borrowed pointers)
  int n;
  const int *rowptr;
  const int *colidx;
  int64_t nnz() const { return n ? rowptr[n] : 0; }
};

// Approximate minimum degree (sparse.mjs:297-592). perm: new -> old, length n. Returns false on internal error.
bool amd_order(const Pattern &P, double dense_factor, int *perm);
// 2D coordinate-bisection nested dissection (sparse.mjs:231-283).
void nd_order(const Pattern &P, const double *x, const double *y, int leaf, int *perm);
// 3D coordinate-bisection nested dissection with AMD leaves and separators (order3d.mjs:27-77).
void nd3_order(const Pattern &P, const double *x, const double *y, const double *z, int leaf, int *perm,
               int threads = 0);

// FNV-1a fingerprint of a pattern (sparse.mjs:908-925).
uint32_t pattern_hash(const Pattern &P);
std::string pattern_key(const Pattern &P);

struct Symbolic {
  int n = 0, nsuper = 0, maxFront = 0;
  int64_t nnzL = 0, nnzA = 0, nnzLStored = 0;
  double fill = 1, flops = 0;
  int patNnz = 0;
  uint32_t hash = 0;
  std::vector<int> perm, pinv, parent, colCount;
  std::vector<int> lowerP, lowerI, lowerSrc;
  std::vector<int> superStart, colSuper, superParent, childHead, childNext;
  std::vector<int> Sp, Si;
  std::vector<int64_t> Lxp;
  double ordering_ms = 0, symbolic_ms = 0;
};

// analyze (sparse.mjs:666-902). ordering: 0 amd, 1 nd (2D; x, y), 2 nd3 (x, y, z; leaf 2000). perm (new -> old)
// overrides the ordering when non-null.
void analyze(const Pattern &P, const int *perm, int ordering, const double *x, const double *y, const double *z,
             bool relax, Symbolic &S);

}  // namespace amp
