// Host symbolic phase (see symbolic.hpp). Every step follows the reference's published algorithm so that the
// permutation, elimination tree, column counts and supernodes are bit-identical to
// packages/core/src/la/sparse.mjs (cited per function); the code organisation is this library's own.
#include "symbolic.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <thread>

namespace amp {

// ---------------------------------------------------------------------------------------------------------------
// Approximate minimum degree on the quotient graph (sparse.mjs:297-592; Amestoy, Davis & Duff 1996 as restated in
// Davis, Direct Methods for Sparse Linear Systems, ch. 7). State layout and every update rule mirror the reference,
// including its workspace size (nnz + nnz/5 + 2n), garbage-collection trigger, hash h % n and wclear threshold 2e9.
// ---------------------------------------------------------------------------------------------------------------
namespace {

inline int flip(int i) { return -i - 2; }

class QuotientGraphAMD {
 public:
  QuotientGraphAMD(const Pattern &P, double dense_factor) : n_(P.n) {
    int64_t cnz = 0;
    for (int i = 0; i < n_; i++)
      for (int p = P.rowptr[i]; p < P.rowptr[i + 1]; p++) cnz += P.colidx[p] != i;
    nzmax_ = cnz + cnz / 5 + 2 * (int64_t)n_;
    Cp_.assign(n_ + 1, 0);
    Ci_.assign(nzmax_ + 1, 0);
    int64_t q = 0;
    for (int i = 0; i < n_; i++) {
      Cp_[i] = (int)q;
      for (int p = P.rowptr[i]; p < P.rowptr[i + 1]; p++)
        if (P.colidx[p] != i) Ci_[q++] = P.colidx[p];
    }
    Cp_[n_] = (int)q;
    cnz_ = q;
    len_.assign(n_ + 1, 0);
    for (int k = 0; k < n_; k++) len_[k] = Cp_[k + 1] - Cp_[k];
    nv_.assign(n_ + 1, 1);
    next_.assign(n_ + 1, -1);
    head_.assign(n_ + 1, -1);
    elen_.assign(n_ + 1, 0);
    degree_.assign(len_.begin(), len_.end());
    w_.assign(n_ + 1, 1);
    hhead_.assign(n_ + 1, -1);
    last_.assign(n_ + 1, -1);
    double big = dense_factor * std::sqrt((double)n_);
    if (!(big > 16.0)) big = std::isnan(big) ? big : 16.0;
    dense_ = std::isnan(big) ? big : std::min((double)(n_ - 2), big);
  }

  bool run(int *out) {
    mark_ = clear_marks(0, 0);
    elen_[n_] = -2;
    Cp_[n_] = -1;
    w_[n_] = 0;
    nv_[n_] = 0;
    classify_initial();
    while (nel_ < n_) eliminate_one();
    return postorder(out);
  }

 private:
  int64_t clear_marks(int64_t mark, int64_t lemax) {
    if (mark < 2 || (double)(mark + lemax) > 2e9) {
      for (int k = 0; k < n_; k++)
        if (w_[k] != 0) w_[k] = 1;
      return 2;
    }
    return mark;
  }

  void bucket_insert(int i, int d) {
    if (head_[d] != -1) last_[head_[d]] = i;
    next_[i] = head_[d];
    head_[d] = i;
  }

  void classify_initial() {
    for (int i = 0; i < n_; i++) {
      int d = degree_[i];
      if (d == 0) {  // empty row: eliminated at once
        elen_[i] = -2;
        nel_++;
        Cp_[i] = -1;
        w_[i] = 0;
      } else if ((double)d > dense_) {  // dense row: ordered last
        nv_[i] = 0;
        elen_[i] = -1;
        nel_++;
        Cp_[i] = flip(n_);
        nv_[n_]++;
      } else
        bucket_insert(i, d);
    }
  }

  void compact_storage() {
    for (int j = 0; j < n_; j++) {
      int p = Cp_[j];
      if (p >= 0) {
        Cp_[j] = Ci_[p];
        Ci_[p] = flip(j);
      }
    }
    int64_t q = 0;
    for (int64_t p = 0; p < cnz_;) {
      int j = flip(Ci_[p++]);
      if (j >= 0) {
        Ci_[q] = Cp_[j];
        Cp_[j] = (int)q++;
        for (int t = 0; t < len_[j] - 1; t++) Ci_[q++] = Ci_[p++];
      }
    }
    cnz_ = q;
  }

  void eliminate_one() {
    int k = -1;
    for (; mindeg_ < n_ && (k = head_[mindeg_]) == -1; mindeg_++) {
    }
    if (next_[k] != -1) last_[next_[k]] = -1;
    head_[mindeg_] = next_[k];
    const int elenk = elen_[k];
    int nvk = nv_[k];
    nel_ += nvk;
    if (elenk > 0 && cnz_ + mindeg_ >= nzmax_) compact_storage();

    // construct the new element Lk from k's elements and variables
    int dk = 0;
    nv_[k] = -nvk;
    int64_t p = Cp_[k];
    const int64_t pk1 = elenk == 0 ? p : cnz_;
    int64_t pk2 = pk1;
    for (int k1 = 1; k1 <= elenk + 1; k1++) {
      int e, ln;
      int64_t pj;
      if (k1 > elenk) {
        e = k;
        pj = p;
        ln = len_[k] - elenk;
      } else {
        e = Ci_[p++];
        pj = Cp_[e];
        ln = len_[e];
      }
      for (int k2 = 1; k2 <= ln; k2++) {
        int i = Ci_[pj++];
        int nvi = nv_[i];
        if (nvi <= 0) continue;
        dk += nvi;
        nv_[i] = -nvi;
        if (pk2 >= nzmax_) {
          std::fprintf(stderr, "amp amd: quotient graph workspace overflow\n");
          std::abort();
        }
        Ci_[pk2++] = i;
        if (next_[i] != -1) last_[next_[i]] = last_[i];
        if (last_[i] != -1)
          next_[last_[i]] = next_[i];
        else
          head_[degree_[i]] = next_[i];
      }
      if (e != k) {
        Cp_[e] = flip(k);  // element e absorbed into k
        w_[e] = 0;
      }
    }
    if (elenk != 0) cnz_ = pk2;
    degree_[k] = dk;
    Cp_[k] = (int)pk1;
    len_[k] = (int)(pk2 - pk1);
    elen_[k] = -2;

    // |Le \ Lk| for every element e adjacent to the variables of Lk
    mark_ = clear_marks(mark_, lemax_);
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci_[pk];
      int eln = elen_[i];
      if (eln <= 0) continue;
      int nvi = -nv_[i];
      int64_t wnvi = mark_ - nvi;
      for (int64_t q = Cp_[i]; q <= (int64_t)Cp_[i] + eln - 1; q++) {
        int e = Ci_[q];
        if (w_[e] >= mark_)
          w_[e] -= nvi;
        else if (w_[e] != 0)
          w_[e] = (int)(degree_[e] + wnvi);
      }
    }

    // approximate external degrees, aggressive absorption, hashing of the variables of Lk
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci_[pk];
      int64_t p1 = Cp_[i], p2 = p1 + elen_[i] - 1, pn = p1;
      int64_t h = 0;
      int d = 0;
      for (int64_t q = p1; q <= p2; q++) {
        int e = Ci_[q];
        if (w_[e] == 0) continue;
        int64_t dext = w_[e] - mark_;
        if (dext > 0) {
          d += (int)dext;
          Ci_[pn++] = e;
          h += e;
        } else {
          Cp_[e] = flip(k);
          w_[e] = 0;
        }
      }
      elen_[i] = (int)(pn - p1 + 1);
      int64_t p3 = pn, p4 = p1 + len_[i];
      for (int64_t q = p2 + 1; q < p4; q++) {
        int j = Ci_[q];
        int nvj = nv_[j];
        if (nvj <= 0) continue;
        d += nvj;
        Ci_[pn++] = j;
        h += j;
      }
      if (d == 0) {  // mass elimination
        Cp_[i] = flip(k);
        int nvi = -nv_[i];
        dk -= nvi;
        nvk += nvi;
        nel_ += nvi;
        nv_[i] = 0;
        elen_[i] = -1;
      } else {
        degree_[i] = std::min(degree_[i], d);
        Ci_[pn] = Ci_[p3];
        Ci_[p3] = Ci_[p1];
        Ci_[p1] = k;
        len_[i] = (int)(pn - p1 + 1);
        h = (h < 0 ? -h : h) % n_;
        next_[i] = hhead_[h];
        hhead_[h] = i;
        last_[i] = (int)h;
      }
    }
    degree_[k] = dk;
    lemax_ = std::max<int64_t>(lemax_, dk);
    mark_ = clear_marks(mark_ + lemax_, lemax_);

    // indistinguishable variables (supervariables) within each hash bucket
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci_[pk];
      if (nv_[i] >= 0) continue;
      int hb = last_[i];
      i = hhead_[hb];
      hhead_[hb] = -1;
      for (; i != -1 && next_[i] != -1; i = next_[i], mark_++) {
        const int ln = len_[i], eln = elen_[i];
        for (int64_t q = (int64_t)Cp_[i] + 1; q <= (int64_t)Cp_[i] + ln - 1; q++) w_[Ci_[q]] = (int)mark_;
        int jlast = i;
        for (int j = next_[i]; j != -1;) {
          bool same = len_[j] == ln && elen_[j] == eln;
          for (int64_t q = (int64_t)Cp_[j] + 1; same && q <= (int64_t)Cp_[j] + ln - 1; q++)
            if (w_[Ci_[q]] != mark_) same = false;
          if (same) {
            Cp_[j] = flip(i);
            nv_[i] += nv_[j];
            nv_[j] = 0;
            elen_[j] = -1;
            j = next_[j];
            next_[jlast] = j;
          } else {
            jlast = j;
            j = next_[j];
          }
        }
      }
    }

    // finalize Lk: restore nv, new degrees into the buckets
    int64_t q = pk1;
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci_[pk];
      int nvi = -nv_[i];
      if (nvi <= 0) continue;
      nv_[i] = nvi;
      int d = std::min(degree_[i] + dk - nvi, n_ - nel_ - nvi);
      bucket_insert(i, d);
      last_[i] = -1;
      mindeg_ = std::min(mindeg_, d);
      degree_[i] = d;
      Ci_[q++] = i;
    }
    nv_[k] = nvk;
    if ((len_[k] = (int)(q - pk1)) == 0) {
      Cp_[k] = -1;
      w_[k] = 0;
    }
    if (elenk != 0) cnz_ = q;
  }

  // postorder of the assembly tree (children in increasing order, absorbed variables before their element)
  bool postorder(int *out) {
    for (int i = 0; i < n_; i++) Cp_[i] = flip(Cp_[i]);
    std::fill(head_.begin(), head_.end(), -1);
    for (int j = n_; j >= 0; j--) {
      if (nv_[j] > 0) continue;
      if (Cp_[j] < 0) {  // the placeholder n without dense rows: the reference's no-op
        next_[j] = 0;
        continue;
      }
      next_[j] = head_[Cp_[j]];
      head_[Cp_[j]] = j;
    }
    for (int e = n_; e >= 0; e--) {
      if (nv_[e] <= 0) continue;
      if (Cp_[e] != -1) {
        next_[e] = head_[Cp_[e]];
        head_[Cp_[e]] = e;
      }
    }
    int o = 0;
    std::vector<int> &stack = w_;
    for (int i = 0; i <= n_; i++) {
      if (Cp_[i] != -1) continue;
      int top = 0;
      stack[0] = i;
      while (top >= 0) {
        int pp = stack[top];
        int ii = head_[pp];
        if (ii == -1) {
          top--;
          if (pp < n_) out[o++] = pp;
        } else {
          head_[pp] = next_[ii];
          stack[++top] = ii;
        }
      }
    }
    return o == n_;
  }

  int n_;
  int64_t nzmax_ = 0, cnz_ = 0, mark_ = 0, lemax_ = 0;
  int nel_ = 0, mindeg_ = 0;
  double dense_ = 0;
  std::vector<int> Cp_, Ci_, len_, nv_, next_, head_, elen_, degree_, w_, hhead_, last_;
};

// Stable ordering of node ids by one coordinate (the reference sorts with Array.prototype.sort, which is stable).
void sort_by_coordinate(std::vector<int> &nodes, const double *key) {
  std::stable_sort(nodes.begin(), nodes.end(), [key](int a, int b) { return key[a] < key[b]; });
}

}  // namespace

bool amd_order(const Pattern &P, double dense_factor, int *perm) {
  if (P.n == 0) return true;
  QuotientGraphAMD amd(P, dense_factor);
  return amd.run(perm);
}

// ---------------------------------------------------------------------------------------------------------------
// 2D nested dissection (sparse.mjs:231-283): split along the longer bounding-box side (ties to x), separator = nodes
// of the first half with a neighbour in the second half; order A, B, then S. Leaves keep their input order.
// ---------------------------------------------------------------------------------------------------------------
namespace {
struct Bisection {
  std::vector<int> A, S, B;
};

// One bisection step shared by the 2D and 3D orderings. axis chosen by the caller; skip_self reproduces the 2D
// test w !== v (the 3D code has none; the diagonal is on the first-half side, so both give the same sets).
void bisect(const Pattern &P, std::vector<int> &sorted, std::vector<signed char> &side, bool skip_self, Bisection &out) {
  const int len = (int)sorted.size(), half = len >> 1;
  for (int i = 0; i < len; i++) side[sorted[i]] = i < half ? 1 : 2;
  out.A.clear();
  out.S.clear();
  out.B.clear();
  for (int i = 0; i < len; i++) {
    int v = sorted[i];
    if (i >= half) {
      out.B.push_back(v);
      continue;
    }
    bool sep = false;
    for (int p = P.rowptr[v]; p < P.rowptr[v + 1] && !sep; p++) {
      int w = P.colidx[p];
      if ((!skip_self || w != v) && side[w] == 2) sep = true;
    }
    (sep ? out.S : out.A).push_back(v);
  }
  for (int v : sorted) side[v] = 0;
}

void nd2_recurse(const Pattern &P, const double *x, const double *y, int leaf, std::vector<int> nodes,
                 std::vector<signed char> &side, std::vector<int> &order) {
  if ((int)nodes.size() <= leaf) {
    order.insert(order.end(), nodes.begin(), nodes.end());
    return;
  }
  double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
  for (int v : nodes) {
    x0 = std::min(x0, x[v]);
    x1 = std::max(x1, x[v]);
    y0 = std::min(y0, y[v]);
    y1 = std::max(y1, y[v]);
  }
  sort_by_coordinate(nodes, (x1 - x0 >= y1 - y0) ? x : y);
  Bisection b;
  bisect(P, nodes, side, true, b);
  nodes.clear();
  nodes.shrink_to_fit();
  nd2_recurse(P, x, y, leaf, std::move(b.A), side, order);
  nd2_recurse(P, x, y, leaf, std::move(b.B), side, order);
  order.insert(order.end(), b.S.begin(), b.S.end());
}
}  // namespace

void nd_order(const Pattern &P, const double *x, const double *y, int leaf, int *perm) {
  std::vector<int> all(P.n), order;
  order.reserve(P.n);
  for (int i = 0; i < P.n; i++) all[i] = i;
  std::vector<signed char> side(P.n, 0);
  nd2_recurse(P, x, y, leaf, std::move(all), side, order);
  std::copy(order.begin(), order.end(), perm);
}

// ---------------------------------------------------------------------------------------------------------------
// 3D nested dissection (order3d.mjs:27-77): the recursion only fixes, for every leaf and separator, its node list and
// its slot range in the output; the AMD orderings of those induced subgraphs (subPattern :11-24: rows in node-list
// order, columns in the parent row's order, diagonal kept) then run in parallel.
// ---------------------------------------------------------------------------------------------------------------
namespace {
struct LeafTask {
  std::vector<int> nodes;
  int offset;
};

void nd3_partition(const Pattern &P, const double *C[3], int leaf, std::vector<int> nodes, int offset,
                   std::vector<signed char> &side, std::vector<LeafTask> &tasks) {
  if ((int)nodes.size() <= leaf) {
    tasks.push_back({std::move(nodes), offset});
    return;
  }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int v : nodes)
    for (int d = 0; d < 3; d++) {
      lo[d] = std::min(lo[d], C[d][v]);
      hi[d] = std::max(hi[d], C[d][v]);
    }
  int ax = 0;
  for (int d = 1; d < 3; d++)
    if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
  sort_by_coordinate(nodes, C[ax]);
  Bisection b;
  bisect(P, nodes, side, false, b);
  nodes.clear();
  nodes.shrink_to_fit();
  int na = (int)b.A.size(), nb = (int)b.B.size();
  nd3_partition(P, C, leaf, std::move(b.A), offset, side, tasks);
  nd3_partition(P, C, leaf, std::move(b.B), offset + na, side, tasks);
  tasks.push_back({std::move(b.S), offset + na + nb});
}

void order_induced_subgraph(const Pattern &P, const std::vector<int> &nodes, std::vector<int> &loc, int *out) {
  const int m = (int)nodes.size();
  for (int i = 0; i < m; i++) loc[nodes[i]] = i;
  std::vector<int> rp(m + 1, 0), cols;
  for (int i = 0; i < m; i++) {
    int v = nodes[i];
    for (int p = P.rowptr[v]; p < P.rowptr[v + 1]; p++) {
      int w = loc[P.colidx[p]];
      if (w >= 0) cols.push_back(w);
    }
    rp[i + 1] = (int)cols.size();
  }
  std::vector<int> sub(m);
  Pattern S{m, rp.data(), cols.data()};
  if (!amd_order(S, 10.0, sub.data())) {
    std::fprintf(stderr, "amp nd3: amd failed on a subgraph\n");
    std::abort();
  }
  for (int i = 0; i < m; i++) out[i] = nodes[sub[i]];
  for (int v : nodes) loc[v] = -1;
}
}  // namespace

void nd3_order(const Pattern &P, const double *x, const double *y, const double *z, int leaf, int *perm,
               int threads) {
  const double *C[3] = {x, y, z};
  std::vector<int> all(P.n);
  for (int i = 0; i < P.n; i++) all[i] = i;
  std::vector<signed char> side(P.n, 0);
  std::vector<LeafTask> tasks;
  nd3_partition(P, C, leaf, std::move(all), 0, side, tasks);
  if (threads <= 0) threads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  threads = std::min<int>(threads, (int)tasks.size());
  std::atomic<size_t> nextTask{0};
  auto worker = [&]() {
    std::vector<int> loc(P.n, -1);
    for (size_t t; (t = nextTask.fetch_add(1)) < tasks.size();)
      order_induced_subgraph(P, tasks[t].nodes, loc, perm + tasks[t].offset);
  };
  if (threads <= 1)
    worker();
  else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Fingerprint (sparse.mjs:908-925)
// ---------------------------------------------------------------------------------------------------------------
uint32_t pattern_hash(const Pattern &P) {
  uint32_t h = 0x811c9dc5u;
  auto mix = [&h](uint32_t v) {
    for (int sh = 0; sh < 32; sh += 8) {
      h ^= (v >> sh) & 0xffu;
      h *= 0x01000193u;
    }
  };
  for (int i = 0; i <= P.n; i++) mix((uint32_t)P.rowptr[i]);
  int64_t nnz = P.nnz();
  for (int64_t p = 0; p < nnz; p++) mix((uint32_t)P.colidx[p]);
  return h;
}

std::string pattern_key(const Pattern &P) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%d:%lld:%x", P.n, (long long)P.nnz(), pattern_hash(P));
  return buf;
}

// ---------------------------------------------------------------------------------------------------------------
// Supernodal symbolic analysis (sparse.mjs:666-902)
// ---------------------------------------------------------------------------------------------------------------
namespace {

// Liu's elimination tree of P A P^T with path compression (sparse.mjs:628-645).
std::vector<int> elimination_tree(const Pattern &A, const std::vector<int> &perm, const std::vector<int> &pinv) {
  const int n = A.n;
  std::vector<int> parent(n, -1), anc(n, -1);
  for (int k = 0; k < n; k++) {
    int v = perm[k];
    for (int p = A.rowptr[v]; p < A.rowptr[v + 1]; p++) {
      for (int i = pinv[A.colidx[p]]; i != -1 && i < k;) {
        int inext = anc[i];
        anc[i] = k;
        if (inext == -1) parent[i] = k;
        i = inext;
      }
    }
  }
  return parent;
}

// Depth-first postorder of a forest, children in increasing index (sparse.mjs:597-625).
std::vector<int> forest_postorder(const std::vector<int> &parent) {
  const int n = (int)parent.size();
  std::vector<int> head(n, -1), next(n, 0), stack(n), post(n);
  for (int j = n - 1; j >= 0; j--)
    if (parent[j] != -1) {
      next[j] = head[parent[j]];
      head[parent[j]] = j;
    }
  int k = 0;
  for (int j = 0; j < n; j++) {
    if (parent[j] != -1) continue;
    int top = 0;
    stack[0] = j;
    while (top >= 0) {
      int p = stack[top], i = head[p];
      if (i == -1) {
        top--;
        post[k++] = p;
      } else {
        head[p] = next[i];
        stack[++top] = i;
      }
    }
  }
  return post;
}

// Gilbert-Ng-Peyton column counts on a postordered tree (sparse.mjs:720-753).
void column_counts(int n, const std::vector<int> &parent, const std::vector<int> &lowerP, const std::vector<int> &lowerI,
                   std::vector<int> &cc) {
  cc.assign(n, 0);
  std::vector<int> first(n, -1), maxfirst(n, -1), prevleaf(n, -1), ancestor(n);
  for (int k = 0; k < n; k++) {
    cc[k] = first[k] == -1 ? 1 : 0;
    for (int j = k; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
  }
  for (int i = 0; i < n; i++) ancestor[i] = i;
  for (int j = 0; j < n; j++) {
    if (parent[j] != -1) cc[parent[j]]--;
    for (int p = lowerP[j]; p < lowerP[j + 1]; p++) {
      int i = lowerI[p];
      if (i <= j || first[j] <= maxfirst[i]) continue;  // j is not a leaf of the row subtree of i
      maxfirst[i] = first[j];
      int jprev = prevleaf[i];
      prevleaf[i] = j;
      cc[j]++;
      if (jprev == -1) continue;
      int q = jprev;
      while (q != ancestor[q]) q = ancestor[q];
      for (int s = jprev; s != q;) {
        int sp = ancestor[s];
        ancestor[s] = q;
        s = sp;
      }
      cc[q]--;  // least common ancestor
    }
    if (parent[j] != -1) ancestor[j] = parent[j];
  }
  for (int j = 0; j < n; j++)
    if (parent[j] != -1) cc[parent[j]] += cc[j];
}

// Fundamental supernodes and relaxed amalgamation (sparse.mjs:761-814). The zero-fraction arithmetic is IEEE double,
// evaluated in the reference's order.
std::vector<int> supernode_partition(int n, const std::vector<int> &parent, const std::vector<int> &cc, bool relax) {
  std::vector<int> nchild(n, 0);
  for (int j = 0; j < n; j++)
    if (parent[j] != -1) nchild[parent[j]]++;
  std::vector<int> fStart{0};
  for (int j = 1; j < n; j++)
    if (!(parent[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1)) fStart.push_back(j);
  fStart.push_back(n);
  const int nsf = (int)fStart.size() - 1;
  if (!relax || nsf <= 1) return fStart;
  std::vector<int> colSuperF(n);
  for (int s = 0; s < nsf; s++)
    for (int j = fStart[s]; j < fStart[s + 1]; j++) colSuperF[j] = s;
  struct Node {
    int first, last, parent;
    double rows, zeros, entries;
    bool alive;
  };
  std::vector<Node> sn(nsf);
  for (int s = 0; s < nsf; s++) {
    Node &a = sn[s];
    a.first = fStart[s];
    a.last = fStart[s + 1] - 1;
    a.rows = cc[fStart[s]];
    double nc = fStart[s + 1] - fStart[s];
    a.entries = nc * a.rows - (nc * (nc - 1)) / 2;
    a.zeros = 0;
    int pl = parent[a.last];
    a.parent = pl == -1 ? -1 : colSuperF[pl];
    a.alive = true;
  }
  for (int s = 0; s < nsf; s++) {
    Node &c = sn[s];
    if (c.parent == -1) continue;
    Node &p = sn[c.parent];
    if (p.first != c.last + 1) continue;  // only the parent's last child can merge (contiguous columns)
    double ncC = c.last - c.first + 1, ncP = p.last - p.first + 1;
    double nc = ncC + ncP;
    double m = ncC + p.rows;
    double stored = nc * m - (nc * (nc - 1)) / 2;
    double zeros = stored - c.entries - p.entries + c.zeros + p.zeros;
    double zf = zeros / stored;
    bool merge = nc <= 4 || (nc <= 16 && zf < 0.8) || (nc <= 48 && zf < 0.1) || zf < 0.05;
    if (!merge) continue;
    p.first = c.first;
    p.rows = m;
    p.zeros = zeros;
    p.entries += c.entries;
    c.alive = false;
  }
  std::vector<int> st;
  for (int s = 0; s < nsf; s++)
    if (sn[s].alive) st.push_back(sn[s].first);
  st.push_back(n);
  return st;
}

}  // namespace

void analyze(const Pattern &A, const int *perm_in, int ordering, const double *x, const double *y, const double *z,
             bool relax, Symbolic &S) {
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  const int n = A.n;
  S = Symbolic();
  S.n = n;
  S.patNnz = (int)A.nnz();
  S.hash = pattern_hash(A);
  if (n == 0) {
    S.lowerP.assign(1, 0);
    S.superStart.assign(1, 0);
    S.Sp.assign(1, 0);
    S.Lxp.assign(1, 0);
    return;
  }
  std::vector<int> perm0(n);
  if (perm_in)
    std::copy(perm_in, perm_in + n, perm0.begin());
  else if (ordering == 1)
    nd_order(A, x, y, 48, perm0.data());
  else if (ordering == 2)
    nd3_order(A, x, y, z, 2000, perm0.data());
  else if (!amd_order(A, 10.0, perm0.data())) {
    std::fprintf(stderr, "amp analyze: amd failed\n");
    std::abort();
  }
  auto t1 = clk::now();
  // elimination tree, then the order followed by its postorder (same fill)
  std::vector<int> pinv(n);
  for (int i = 0; i < n; i++) pinv[perm0[i]] = i;
  std::vector<int> parent0 = elimination_tree(A, perm0, pinv);
  std::vector<int> post = forest_postorder(parent0);
  S.perm.resize(n);
  std::vector<int> postInv(n);
  for (int k = 0; k < n; k++) {
    S.perm[k] = perm0[post[k]];
    postInv[post[k]] = k;
  }
  S.parent.resize(n);
  for (int k = 0; k < n; k++) {
    int p = parent0[post[k]];
    S.parent[k] = p == -1 ? -1 : postInv[p];
  }
  S.pinv.resize(n);
  for (int i = 0; i < n; i++) S.pinv[S.perm[i]] = i;
  // lower CSC of P A P^T with the CSR slot of every entry (the device assembly map)
  S.lowerP.assign(n + 1, 0);
  for (int v = 0; v < n; v++) {
    int pv = S.pinv[v];
    for (int p = A.rowptr[v]; p < A.rowptr[v + 1]; p++)
      if (S.pinv[A.colidx[p]] >= pv) S.lowerP[pv + 1]++;
  }
  for (int j = 0; j < n; j++) S.lowerP[j + 1] += S.lowerP[j];
  S.nnzA = S.lowerP[n];
  S.lowerI.resize(S.nnzA);
  S.lowerSrc.resize(S.nnzA);
  {
    std::vector<int> nxt(S.lowerP.begin(), S.lowerP.begin() + n);
    for (int v = 0; v < n; v++) {
      int pv = S.pinv[v];
      for (int p = A.rowptr[v]; p < A.rowptr[v + 1]; p++) {
        int pi = S.pinv[A.colidx[p]];
        if (pi >= pv) {
          int q = nxt[pv]++;
          S.lowerI[q] = pi;
          S.lowerSrc[q] = p;
        }
      }
    }
  }
  column_counts(n, S.parent, S.lowerP, S.lowerI, S.colCount);
  for (int j = 0; j < n; j++) {
    S.nnzL += S.colCount[j];
    S.flops += (double)S.colCount[j] * (double)S.colCount[j];
  }
  S.superStart = supernode_partition(n, S.parent, S.colCount, relax);
  const int ns = (int)S.superStart.size() - 1;
  S.nsuper = ns;
  S.colSuper.resize(n);
  for (int s = 0; s < ns; s++)
    for (int j = S.superStart[s]; j < S.superStart[s + 1]; j++) S.colSuper[j] = s;
  S.superParent.resize(ns);
  for (int s = 0; s < ns; s++) {
    int pl = S.parent[S.superStart[s + 1] - 1];
    S.superParent[s] = pl == -1 ? -1 : S.colSuper[pl];
  }
  // children linked in decreasing order (the multifrontal stack pops the last child first)
  S.childHead.assign(ns, -1);
  S.childNext.assign(ns, -1);
  for (int s = 0; s < ns; s++) {
    int P = S.superParent[s];
    if (P == -1) continue;
    S.childNext[s] = S.childHead[P];
    S.childHead[P] = s;
  }
  // row structures: own columns, then the sorted union of A's rows below and the children's rows below
  S.Sp.assign(ns + 1, 0);
  std::vector<int> rowsBuf;  // concatenated rows (in supernode order)
  rowsBuf.reserve((size_t)S.nnzA);
  std::vector<int> marker(n, -1);
  for (int s = 0; s < ns; s++) {
    const int f = S.superStart[s], l = S.superStart[s + 1] - 1;
    const size_t base = rowsBuf.size();
    for (int j = f; j <= l; j++) rowsBuf.push_back(j);
    const size_t belowStart = rowsBuf.size();
    for (int j = f; j <= l; j++)
      for (int p = S.lowerP[j]; p < S.lowerP[j + 1]; p++) {
        int i = S.lowerI[p];
        if (i > l && marker[i] != s) {
          marker[i] = s;
          rowsBuf.push_back(i);
        }
      }
    for (int c = S.childHead[s]; c != -1; c = S.childNext[c]) {
      int ncc = S.superStart[c + 1] - S.superStart[c];
      for (int r = S.Sp[c] + ncc; r < S.Sp[c + 1]; r++) {
        int i = rowsBuf[r];
        if (i > l && marker[i] != s) {
          marker[i] = s;
          rowsBuf.push_back(i);
        }
      }
    }
    std::sort(rowsBuf.begin() + belowStart, rowsBuf.end());
    int len = (int)(rowsBuf.size() - base);
    S.Sp[s + 1] = S.Sp[s] + len;
    S.maxFront = std::max(S.maxFront, len);
  }
  S.Si = std::move(rowsBuf);
  S.Lxp.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++)
    S.Lxp[s + 1] = S.Lxp[s] + (int64_t)(S.Sp[s + 1] - S.Sp[s]) * (S.superStart[s + 1] - S.superStart[s]);
  S.nnzLStored = S.Lxp[ns];
  S.fill = (double)S.nnzL / (double)S.nnzA;
  auto t2 = clk::now();
  S.ordering_ms = perm_in ? 0.0 : std::chrono::duration<double, std::milli>(t1 - t0).count();
  S.symbolic_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
}

}  // namespace amp
