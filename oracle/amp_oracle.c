/*
 * amp_oracle.c -- TEST INFRASTRUCTURE ONLY (never linked into the product library).
 *
 * A line-by-line CPU restatement, in plain C, of the reference's supernodal sparse direct solver
 * (jwt625/applied-multiphysics, packages/core/src/la/). It serves three purposes:
 *   1. the parity oracle for the symbolic analysis (bit-exact: permutation, etree, column counts, supernodes,
 *      row structures) and for the FP64 numeric factor / solves of the product;
 *   2. the JS "blocked" kernels as the scalar reference, and
 *   3. an SSE2 (__m128d, the f64x2 width of WebAssembly SIMD) restatement of the reference's WASM kernels
 *      (wasm/front-real.mjs g4/s4/g1/s1, wasm/solve-real.mjs fdiag/facc/bdiag/lfwd1/lbwd1/lfwdq/lbwdq), which is
 *      the timed single-thread CPU baseline. Per entry it applies the same operations in the same order as the
 *      scalar path, so both are bitwise identical (checked by the tests).
 *
 * Build: -O2 -ffp-contract=off, no -ffast-math (IEEE double, no fused multiply-add, correctly rounded sqrt and /).
 *
 * JavaScript semantics mirrored here:
 *   - Array.prototype.sort(cmp) is stable: a stable merge sort on the coordinate key;
 *   - typed-array .sort() is numeric ascending;
 *   - AMD's hash sum h and the mark counter are JS doubles: int64 here;
 *   - the relaxed-amalgamation arithmetic is f64, restated in double;
 *   - Lxp offsets are Float64Array values: int64 here.
 *
 * Parity status: the reference is JavaScript and no JS engine exists on this machine, so the symbolic restatement is
 * pinned by the reference's own property tests (ported in tests/) and by hand-derived traces of small cases, not by
 * executed reference output.
 */
#include <emmintrin.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n);
    abort();
  }
  return p;
}
static void *xrealloc(void *q, size_t n) {
  void *p = realloc(q, n ? n : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n);
    abort();
  }
  return p;
}
static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s ? s : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}
/* Math.max / Math.min: NaN if either argument is NaN. */
static double js_max(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }
static double js_min(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
static int *ifill(int *a, int64_t n, int v) {
  for (int64_t i = 0; i < n; i++) a[i] = v;
  return a;
}

/* ---- pattern fingerprint: sparse.mjs:908-925 ------------------------------------------------------------------ */
ORC_API uint32_t orc_fingerprint_hash(int n, const int *rowptr, const int *colidx) {
  uint32_t h = 0x811c9dc5u;
#define MIX(v)                       \
  do {                               \
    uint32_t vv = (uint32_t)(v);     \
    h ^= vv & 0xffu;                 \
    h *= 0x01000193u;                \
    h ^= (vv >> 8) & 0xffu;          \
    h *= 0x01000193u;                \
    h ^= (vv >> 16) & 0xffu;         \
    h *= 0x01000193u;                \
    h ^= vv >> 24;                   \
    h *= 0x01000193u;                \
  } while (0)
  for (int i = 0; i <= n; i++) MIX(rowptr[i]);
  int nnz = rowptr[n];
  for (int p = 0; p < nnz; p++) MIX(colidx[p]);
#undef MIX
  return h;
}

/* ---- approximate minimum degree: sparse.mjs:287-592 ----------------------------------------------------------- */
#define FLIP(i) (-(i)-2)

ORC_API int orc_amd_order(int n, const int *rowptr, const int *colidx, double denseFactor, int *out) {
  if (n == 0) return 0; /* :299 */
  int64_t cnz = 0;      /* :300-301 */
  for (int i = 0; i < n; i++)
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
      if (colidx[p] != i) cnz++;
  int64_t nzmax = cnz + cnz / 5 + 2 * (int64_t)n; /* :302 Math.floor(cnz / 5) */
  int *Cp = xcalloc(n + 1, sizeof(int));
  int *Ci = xcalloc(nzmax + 1, sizeof(int));
  int q0 = 0; /* :305-310 */
  for (int i = 0; i < n; i++) {
    Cp[i] = q0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
      if (colidx[p] != i) Ci[q0++] = colidx[p];
  }
  Cp[n] = q0;
  int *len = xcalloc(n + 1, sizeof(int)), *nv = xcalloc(n + 1, sizeof(int)), *next = xcalloc(n + 1, sizeof(int)),
      *head = xcalloc(n + 1, sizeof(int)), *elen = xcalloc(n + 1, sizeof(int)), *degree = xcalloc(n + 1, sizeof(int)),
      *w = xcalloc(n + 1, sizeof(int)), *hhead = xcalloc(n + 1, sizeof(int)), *last = xcalloc(n + 1, sizeof(int));
  for (int k = 0; k < n; k++) len[k] = Cp[k + 1] - Cp[k]; /* :320 */
  /* :321 Math.min(n - 2, Math.max(16, denseFactor * Math.sqrt(n))) */
  double dmx = js_max(16.0, denseFactor * sqrt((double)n));
  double dense = js_min((double)(n - 2), dmx);
  for (int i = 0; i <= n; i++) { /* :322-331 */
    head[i] = -1;
    last[i] = -1;
    next[i] = -1;
    hhead[i] = -1;
    nv[i] = 1;
    w[i] = 1;
    elen[i] = 0;
    degree[i] = len[i];
  }
  int64_t mark;
  /* wclear :332-338 */
#define WCLEAR(m_, lemax_, res_)                                        \
  do {                                                                  \
    int64_t mm_ = (m_);                                                 \
    if (mm_ < 2 || (double)(mm_ + (lemax_)) > 2e9) {                    \
      for (int kk_ = 0; kk_ < n; kk_++)                                 \
        if (w[kk_] != 0) w[kk_] = 1;                                    \
      (res_) = 2;                                                       \
    } else                                                              \
      (res_) = mm_;                                                     \
  } while (0)
  WCLEAR(0, 0, mark); /* :339 */
  elen[n] = -2;       /* :340-343 */
  Cp[n] = -1;
  w[n] = 0;
  nv[n] = 0;
  int nel = 0;
  for (int i = 0; i < n; i++) { /* :345-363 */
    int d = degree[i];
    if (d == 0) {
      elen[i] = -2;
      nel++;
      Cp[i] = -1;
      w[i] = 0;
    } else if ((double)d > dense) {
      nv[i] = 0;
      elen[i] = -1;
      nel++;
      Cp[i] = FLIP(n);
      nv[n]++;
    } else {
      if (head[d] != -1) last[head[d]] = i;
      next[i] = head[d];
      head[d] = i;
    }
  }
  int mindeg = 0;
  int64_t lemax = 0;
  while (nel < n) { /* :366 */
    int k = -1;     /* :368-369 */
    for (; mindeg < n && (k = head[mindeg]) == -1; mindeg++)
      ;
    if (next[k] != -1) last[next[k]] = -1; /* :370-374 */
    head[mindeg] = next[k];
    int elenk = elen[k];
    int nvk = nv[k];
    nel += nvk;
    if (elenk > 0 && cnz + mindeg >= nzmax) { /* :376-394 garbage collection */
      for (int j = 0; j < n; j++) {
        int p = Cp[j];
        if (p >= 0) {
          Cp[j] = Ci[p];
          Ci[p] = FLIP(j);
        }
      }
      int64_t q = 0;
      for (int64_t p = 0; p < cnz;) {
        int j = FLIP(Ci[p++]);
        if (j >= 0) {
          Ci[q] = Cp[j];
          Cp[j] = (int)q++;
          for (int k3 = 0; k3 < len[j] - 1; k3++) Ci[q++] = Ci[p++];
        }
      }
      cnz = q;
    }
    int dk = 0; /* :396-432 new element Lk */
    nv[k] = -nvk;
    int64_t p = Cp[k];
    int64_t pk1 = elenk == 0 ? p : cnz;
    int64_t pk2 = pk1;
    for (int k1 = 1; k1 <= elenk + 1; k1++) {
      int e;
      int64_t pj;
      int ln;
      if (k1 > elenk) {
        e = k;
        pj = p;
        ln = len[k] - elenk;
      } else {
        e = Ci[p++];
        pj = Cp[e];
        ln = len[e];
      }
      for (int k2 = 1; k2 <= ln; k2++) {
        int i = Ci[pj++];
        int nvi = nv[i];
        if (nvi <= 0) continue;
        dk += nvi;
        nv[i] = -nvi;
        if (pk2 >= nzmax) {
          fprintf(stderr, "oracle amd: workspace overflow\n");
          abort();
        }
        Ci[pk2++] = i;
        if (next[i] != -1) last[next[i]] = last[i];
        if (last[i] != -1)
          next[last[i]] = next[i];
        else
          head[degree[i]] = next[i];
      }
      if (e != k) {
        Cp[e] = FLIP(k);
        w[e] = 0;
      }
    }
    if (elenk != 0) cnz = pk2;
    degree[k] = dk;
    Cp[k] = (int)pk1;
    len[k] = (int)(pk2 - pk1);
    elen[k] = -2;
    WCLEAR(mark, lemax, mark); /* :434-446 set differences */
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci[pk];
      int eln = elen[i];
      if (eln <= 0) continue;
      int nvi = -nv[i];
      int64_t wnvi = mark - nvi;
      for (int64_t q = Cp[i]; q <= (int64_t)Cp[i] + eln - 1; q++) {
        int e = Ci[q];
        if (w[e] >= mark)
          w[e] -= nvi;
        else if (w[e] != 0)
          w[e] = (int)(degree[e] + wnvi);
      }
    }
    for (int64_t pk = pk1; pk < pk2; pk++) { /* :448-500 degree update, absorption, hashing */
      int i = Ci[pk];
      int64_t p1 = Cp[i], p2 = p1 + elen[i] - 1;
      int64_t pn = p1;
      int64_t h = 0;
      int d = 0;
      for (int64_t q = p1; q <= p2; q++) {
        int e = Ci[q];
        if (w[e] != 0) {
          int64_t dext = w[e] - mark;
          if (dext > 0) {
            d += (int)dext;
            Ci[pn++] = e;
            h += e;
          } else {
            Cp[e] = FLIP(k);
            w[e] = 0;
          }
        }
      }
      elen[i] = (int)(pn - p1 + 1);
      int64_t p3 = pn, p4 = p1 + len[i];
      for (int64_t q = p2 + 1; q < p4; q++) {
        int j = Ci[q];
        int nvj = nv[j];
        if (nvj <= 0) continue;
        d += nvj;
        Ci[pn++] = j;
        h += j;
      }
      if (d == 0) {
        Cp[i] = FLIP(k);
        int nvi = -nv[i];
        dk -= nvi;
        nvk += nvi;
        nel += nvi;
        nv[i] = 0;
        elen[i] = -1;
      } else {
        degree[i] = degree[i] < d ? degree[i] : d;
        Ci[pn] = Ci[p3];
        Ci[p3] = Ci[p1];
        Ci[p1] = k;
        len[i] = (int)(pn - p1 + 1);
        h = (h < 0 ? -h : h) % n;
        next[i] = hhead[h];
        hhead[h] = i;
        last[i] = (int)h;
      }
    }
    degree[k] = dk; /* :501-503 */
    lemax = lemax > dk ? lemax : dk;
    WCLEAR(mark + lemax, lemax, mark);
    for (int64_t pk = pk1; pk < pk2; pk++) { /* :505-532 supervariable detection */
      int i = Ci[pk];
      if (nv[i] >= 0) continue;
      int h = last[i];
      i = hhead[h];
      hhead[h] = -1;
      for (; i != -1 && next[i] != -1; i = next[i], mark++) {
        int ln = len[i], eln = elen[i];
        for (int64_t q = (int64_t)Cp[i] + 1; q <= (int64_t)Cp[i] + ln - 1; q++) w[Ci[q]] = (int)mark;
        int jlast = i;
        for (int j = next[i]; j != -1;) {
          int ok = len[j] == ln && elen[j] == eln;
          for (int64_t q = (int64_t)Cp[j] + 1; ok && q <= (int64_t)Cp[j] + ln - 1; q++)
            if (w[Ci[q]] != mark) ok = 0;
          if (ok) {
            Cp[j] = FLIP(i);
            nv[i] += nv[j];
            nv[j] = 0;
            elen[j] = -1;
            j = next[j];
            next[jlast] = j;
          } else {
            jlast = j;
            j = next[j];
          }
        }
      }
    }
    int64_t q = pk1; /* :534-555 finalize Lk */
    for (int64_t pk = pk1; pk < pk2; pk++) {
      int i = Ci[pk];
      int nvi = -nv[i];
      if (nvi <= 0) continue;
      nv[i] = nvi;
      int d = degree[i] + dk - nvi;
      int lim = n - nel - nvi;
      d = d < lim ? d : lim;
      if (head[d] != -1) last[head[d]] = i;
      next[i] = head[d];
      last[i] = -1;
      head[d] = i;
      mindeg = mindeg < d ? mindeg : d;
      degree[i] = d;
      Ci[q++] = i;
    }
    nv[k] = nvk;
    if ((len[k] = (int)(q - pk1)) == 0) {
      Cp[k] = -1;
      w[k] = 0;
    }
    if (elenk != 0) cnz = q;
  }
  for (int i = 0; i < n; i++) Cp[i] = FLIP(Cp[i]); /* :558-589 postorder of the assembly tree */
  for (int j = 0; j <= n; j++) head[j] = -1;
  for (int j = n; j >= 0; j--) {
    if (nv[j] > 0) continue;
    if (Cp[j] < 0) { /* only j = n without dense rows: JS reads head[-1] (undefined -> 0) and drops the write */
      next[j] = 0;
      continue;
    }
    next[j] = head[Cp[j]];
    head[Cp[j]] = j;
  }
  for (int e = n; e >= 0; e--) {
    if (nv[e] <= 0) continue;
    if (Cp[e] != -1) {
      next[e] = head[Cp[e]];
      head[Cp[e]] = e;
    }
  }
  int o = 0;
  for (int i = 0; i <= n; i++) {
    if (Cp[i] != -1) continue;
    int top = 0;
    w[0] = i;
    while (top >= 0) {
      int pp = w[top];
      int ii = head[pp];
      if (ii == -1) {
        top--;
        if (pp < n) out[o++] = pp;
      } else {
        head[pp] = next[ii];
        w[++top] = ii;
      }
    }
  }
  free(Cp);
  free(Ci);
  free(len);
  free(nv);
  free(next);
  free(head);
  free(elen);
  free(degree);
  free(w);
  free(hhead);
  free(last);
#undef WCLEAR
  return o == n ? 0 : -1; /* :590 */
}

/* ---- stable sort of node ids by a coordinate key (Array.prototype.sort((p, q) => key[p] - key[q])) -------------- */
static void stable_sort_by_key(int *a, int len, const double *key, int *tmp) {
  if (len < 2) return;
  int mid = len / 2;
  stable_sort_by_key(a, mid, key, tmp);
  stable_sort_by_key(a + mid, len - mid, key, tmp);
  int i = 0, j = mid, k = 0;
  while (i < mid && j < len) {
    if (key[a[j]] < key[a[i]])
      tmp[k++] = a[j++];
    else
      tmp[k++] = a[i++];
  }
  while (i < mid) tmp[k++] = a[i++];
  while (j < len) tmp[k++] = a[j++];
  memcpy(a, tmp, sizeof(int) * len);
}

/* ---- 2D coordinate-bisection nested dissection: sparse.mjs:231-283 --------------------------------------------- */
typedef struct {
  int n;
  const int *rowptr, *colidx;
  const double *x, *y, *z;
  int leaf;
  signed char *side;
  int *order;
  int no;
  int *loc; /* nd3 only */
  int *sortTmp;
} nd_ctx;

static void nd2_rec(nd_ctx *c, int *nodes, int len) {
  if (len <= c->leaf) { /* :237-240 */
    for (int i = 0; i < len; i++) c->order[c->no++] = nodes[i];
    return;
  }
  double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY; /* :241-250 */
  for (int i = 0; i < len; i++) {
    int v = nodes[i];
    if (c->x[v] < x0) x0 = c->x[v];
    if (c->x[v] > x1) x1 = c->x[v];
    if (c->y[v] < y0) y0 = c->y[v];
    if (c->y[v] > y1) y1 = c->y[v];
  }
  const double *key = (x1 - x0 >= y1 - y0) ? c->x : c->y; /* :251 */
  int *sorted = xmalloc(sizeof(int) * len);
  memcpy(sorted, nodes, sizeof(int) * len);
  stable_sort_by_key(sorted, len, key, c->sortTmp); /* :252 */
  int half = len >> 1;
  for (int i = 0; i < len; i++) c->side[sorted[i]] = i < half ? 1 : 2;
  int *A = xmalloc(sizeof(int) * len), *S = xmalloc(sizeof(int) * len), *B = xmalloc(sizeof(int) * len);
  int na = 0, ns = 0, nb = 0;
  for (int i = 0; i < len; i++) { /* :258-272 */
    int v = sorted[i];
    if (i < half) {
      int sep = 0;
      for (int p = c->rowptr[v]; p < c->rowptr[v + 1]; p++) {
        int w = c->colidx[p];
        if (w != v && c->side[w] == 2) {
          sep = 1;
          break;
        }
      }
      if (sep)
        S[ns++] = v;
      else
        A[na++] = v;
    } else
      B[nb++] = v;
  }
  for (int i = 0; i < len; i++) c->side[sorted[i]] = 0; /* :273 */
  free(sorted);
  nd2_rec(c, A, na); /* :274-276 */
  nd2_rec(c, B, nb);
  for (int i = 0; i < ns; i++) c->order[c->no++] = S[i];
  free(A);
  free(S);
  free(B);
}

ORC_API int orc_nd_order(int n, const int *rowptr, const int *colidx, const double *x, const double *y, int leaf,
                         int *perm) {
  nd_ctx c = {n, rowptr, colidx, x, y, NULL, leaf, xcalloc(n, 1), perm, 0, NULL, xmalloc(sizeof(int) * (n + 1))};
  int *all = xmalloc(sizeof(int) * (n + 1));
  for (int i = 0; i < n; i++) all[i] = i;
  nd2_rec(&c, all, n);
  free(all);
  free(c.side);
  free(c.sortTmp);
  return c.no == n ? 0 : -1;
}

/* ---- 3D coordinate-bisection ND with AMD leaves: order3d.mjs:11-77 --------------------------------------------- */
static void nd3_leaf(nd_ctx *c, const int *nodes, int m) { /* order3d.mjs:33-39 leafOrder + subPattern :11-24 */
  for (int i = 0; i < m; i++) c->loc[nodes[i]] = i;
  int *rp = xcalloc(m + 1, sizeof(int));
  int64_t cnt = 0;
  for (int i = 0; i < m; i++) {
    int v = nodes[i];
    for (int p = c->rowptr[v]; p < c->rowptr[v + 1]; p++)
      if (c->loc[c->colidx[p]] >= 0) cnt++;
  }
  int *cols = xmalloc(sizeof(int) * (cnt + 1));
  int q = 0;
  for (int i = 0; i < m; i++) {
    int v = nodes[i];
    for (int p = c->rowptr[v]; p < c->rowptr[v + 1]; p++) {
      int w = c->loc[c->colidx[p]];
      if (w >= 0) cols[q++] = w;
    }
    rp[i + 1] = q;
  }
  int *pp = xmalloc(sizeof(int) * (m + 1));
  if (orc_amd_order(m, rp, cols, 10.0, pp) != 0) {
    fprintf(stderr, "oracle nd3: amd failed\n");
    abort();
  }
  for (int i = 0; i < m; i++) c->order[c->no++] = nodes[pp[i]];
  for (int i = 0; i < m; i++) c->loc[nodes[i]] = -1;
  free(rp);
  free(cols);
  free(pp);
}

static void nd3_rec(nd_ctx *c, int *nodes, int len) {
  if (len <= c->leaf) { /* :41 */
    nd3_leaf(c, nodes, len);
    return;
  }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}; /* :42-48 */
  const double *C[3] = {c->x, c->y, c->z};
  for (int i = 0; i < len; i++) {
    int v = nodes[i];
    for (int d = 0; d < 3; d++) {
      if (C[d][v] < lo[d]) lo[d] = C[d][v];
      if (C[d][v] > hi[d]) hi[d] = C[d][v];
    }
  }
  int ax = 0; /* :49-50 strict > */
  for (int d = 1; d < 3; d++)
    if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
  const double *key = C[ax];
  int *sorted = xmalloc(sizeof(int) * len);
  memcpy(sorted, nodes, sizeof(int) * len);
  stable_sort_by_key(sorted, len, key, c->sortTmp); /* :52 */
  int half = len >> 1;
  for (int i = 0; i < len; i++) c->side[sorted[i]] = i < half ? 1 : 2;
  int *A = xmalloc(sizeof(int) * len), *S = xmalloc(sizeof(int) * len), *B = xmalloc(sizeof(int) * len);
  int na = 0, ns = 0, nb = 0;
  for (int i = 0; i < len; i++) { /* :58-70 (no w !== v test in 3D) */
    int v = sorted[i];
    if (i < half) {
      int sep = 0;
      for (int p = c->rowptr[v]; p < c->rowptr[v + 1]; p++)
        if (c->side[c->colidx[p]] == 2) {
          sep = 1;
          break;
        }
      if (sep)
        S[ns++] = v;
      else
        A[na++] = v;
    } else
      B[nb++] = v;
  }
  for (int i = 0; i < len; i++) c->side[sorted[i]] = 0; /* :71 */
  free(sorted);
  nd3_rec(c, A, na); /* :72-74 */
  nd3_rec(c, B, nb);
  nd3_leaf(c, S, ns);
  free(A);
  free(S);
  free(B);
}

ORC_API int orc_nd3_order(int n, const int *rowptr, const int *colidx, const double *x, const double *y,
                          const double *z, int leaf, int *perm) {
  nd_ctx c = {n, rowptr, colidx, x, y, z, leaf, xcalloc(n, 1), perm, 0, NULL, xmalloc(sizeof(int) * (n + 1))};
  c.loc = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1);
  int *all = xmalloc(sizeof(int) * (n + 1));
  for (int i = 0; i < n; i++) all[i] = i;
  nd3_rec(&c, all, n);
  free(all);
  free(c.side);
  free(c.loc);
  free(c.sortTmp);
  return c.no == n ? 0 : -1;
}

/* ---- symbolic analysis: sparse.mjs:596-902 --------------------------------------------------------------------- */
typedef struct {
  int n, nsuper, maxFront;
  int64_t nnzL, nnzA, nnzLStored;
  double fill, flops;
  uint32_t hash;
  int patNnz;
  int *perm, *pinv, *parent, *colCount;
  int *lowerP, *lowerI, *lowerSrc;
  int *superStart, *colSuper, *superParent, *childHead, *childNext;
  int *Sp, *Si;
  int64_t *Lxp;
} orc_sym;

static int *postorder_of(const int *parent, int n) { /* sparse.mjs:597-625 */
  int *head = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1), *next = xcalloc(n + 1, sizeof(int)),
      *stack = xcalloc(n + 1, sizeof(int)), *post = xcalloc(n + 1, sizeof(int));
  for (int j = n - 1; j >= 0; j--) {
    if (parent[j] == -1) continue;
    next[j] = head[parent[j]];
    head[parent[j]] = j;
  }
  int k = 0;
  for (int j = 0; j < n; j++) {
    if (parent[j] != -1) continue;
    int top = 0;
    stack[0] = j;
    while (top >= 0) {
      int p = stack[top];
      int i = head[p];
      if (i == -1) {
        top--;
        post[k++] = p;
      } else {
        head[p] = next[i];
        stack[++top] = i;
      }
    }
  }
  free(head);
  free(next);
  free(stack);
  return post;
}

static int *etree_of(int n, const int *rowptr, const int *colidx, const int *perm, const int *pinv) { /* :628-645 */
  int *parent = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1), *anc = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1);
  for (int k = 0; k < n; k++) {
    int v = perm[k];
    for (int p = rowptr[v]; p < rowptr[v + 1]; p++) {
      int i = pinv[colidx[p]];
      while (i != -1 && i < k) {
        int inext = anc[i];
        anc[i] = k;
        if (inext == -1) parent[i] = k;
        i = inext;
      }
    }
  }
  free(anc);
  return parent;
}

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* ordering: 0 = amd, 1 = nd (2D, needs x y); perm0 (new -> old) overrides when non-null. Returns NULL with *err set:
 * 1 = perm length (not representable here), 2 = nd needs coordinates, 3 = internal ordering error. */
ORC_API orc_sym *orc_analyze(int n, const int *rowptr, const int *colidx, const int *perm_in, int ordering,
                             const double *x, const double *y, int relax, int *err) {
  *err = 0;
  orc_sym *S = xcalloc(1, sizeof(orc_sym));
  S->n = n;
  S->hash = orc_fingerprint_hash(n, rowptr, colidx);
  S->patNnz = rowptr[n];
  if (n == 0) { /* :670-675 */
    S->lowerP = xcalloc(1, sizeof(int));
    S->superStart = xcalloc(1, sizeof(int));
    S->Sp = xcalloc(1, sizeof(int));
    S->Lxp = xcalloc(1, sizeof(int64_t));
    S->fill = 1;
    return S;
  }
  int *perm0 = xmalloc(sizeof(int) * n);
  if (perm_in)
    memcpy(perm0, perm_in, sizeof(int) * n);
  else if (ordering == 1) {
    if (!x || !y) { /* :678 */
      *err = 2;
      free(perm0);
      free(S);
      return NULL;
    }
    if (orc_nd_order(n, rowptr, colidx, x, y, 48, perm0) != 0) *err = 3;
  } else if (orc_amd_order(n, rowptr, colidx, 10.0, perm0) != 0)
    *err = 3;
  if (*err) {
    free(perm0);
    free(S);
    return NULL;
  }
  int *pinv = xmalloc(sizeof(int) * n); /* :682-696 */
  for (int i = 0; i < n; i++) pinv[perm0[i]] = i;
  int *parent0 = etree_of(n, rowptr, colidx, perm0, pinv);
  int *post = postorder_of(parent0, n);
  int *perm = xmalloc(sizeof(int) * n);
  for (int k = 0; k < n; k++) perm[k] = perm0[post[k]];
  int *postInv = xmalloc(sizeof(int) * n);
  for (int k = 0; k < n; k++) postInv[post[k]] = k;
  int *parent = xmalloc(sizeof(int) * n);
  for (int k = 0; k < n; k++) {
    int p = parent0[post[k]];
    parent[k] = p == -1 ? -1 : postInv[p];
  }
  for (int i = 0; i < n; i++) pinv[perm[i]] = i;
  free(perm0);
  free(parent0);
  free(post);
  free(postInv);
  int *lowerP = xcalloc(n + 1, sizeof(int)); /* :698-718 lower CSC with source slots */
  for (int v = 0; v < n; v++) {
    int pv = pinv[v];
    for (int p = rowptr[v]; p < rowptr[v + 1]; p++)
      if (pinv[colidx[p]] >= pv) lowerP[pv + 1]++;
  }
  for (int j = 0; j < n; j++) lowerP[j + 1] += lowerP[j];
  int nnzA = lowerP[n];
  int *lowerI = xmalloc(sizeof(int) * (nnzA + 1)), *lowerSrc = xmalloc(sizeof(int) * (nnzA + 1));
  int *nxt = xmalloc(sizeof(int) * n);
  memcpy(nxt, lowerP, sizeof(int) * n);
  for (int v = 0; v < n; v++) {
    int pv = pinv[v];
    for (int p = rowptr[v]; p < rowptr[v + 1]; p++) {
      int pi = pinv[colidx[p]];
      if (pi >= pv) {
        int q = nxt[pv]++;
        lowerI[q] = pi;
        lowerSrc[q] = p;
      }
    }
  }
  free(nxt);
  int *colCount = xcalloc(n, sizeof(int)); /* :720-753 Gilbert-Ng-Peyton column counts */
  {
    int *first = ifill(xmalloc(sizeof(int) * n), n, -1), *maxfirst = ifill(xmalloc(sizeof(int) * n), n, -1),
        *prevleaf = ifill(xmalloc(sizeof(int) * n), n, -1), *ancestor = xmalloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) {
      colCount[k] = first[k] == -1 ? 1 : 0;
      for (int j = k; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
    }
    for (int i = 0; i < n; i++) ancestor[i] = i;
    for (int j = 0; j < n; j++) {
      if (parent[j] != -1) colCount[parent[j]]--;
      for (int p = lowerP[j]; p < lowerP[j + 1]; p++) {
        int i = lowerI[p];
        if (i <= j || first[j] <= maxfirst[i]) continue;
        maxfirst[i] = first[j];
        int jprev = prevleaf[i];
        prevleaf[i] = j;
        colCount[j]++;
        if (jprev == -1) continue;
        int q = jprev;
        while (q != ancestor[q]) q = ancestor[q];
        for (int s = jprev, sp; s != q; s = sp) {
          sp = ancestor[s];
          ancestor[s] = q;
        }
        colCount[q]--;
      }
      if (parent[j] != -1) ancestor[j] = parent[j];
    }
    for (int j = 0; j < n; j++)
      if (parent[j] != -1) colCount[parent[j]] += colCount[j];
    free(first);
    free(maxfirst);
    free(prevleaf);
    free(ancestor);
  }
  int64_t nnzL = 0; /* :754-759 */
  double flops = 0;
  for (int j = 0; j < n; j++) {
    nnzL += colCount[j];
    flops += (double)colCount[j] * (double)colCount[j];
  }
  int *nchild = xcalloc(n, sizeof(int)); /* :761-766 fundamental supernodes */
  for (int j = 0; j < n; j++)
    if (parent[j] != -1) nchild[parent[j]]++;
  int *fStart = xmalloc(sizeof(int) * (n + 2));
  int nfs = 0;
  fStart[nfs++] = 0;
  for (int j = 1; j < n; j++)
    if (!(parent[j - 1] == j && colCount[j - 1] == colCount[j] + 1 && nchild[j] == 1)) fStart[nfs++] = j;
  fStart[nfs++] = n;
  int nsf = nfs - 1;
  free(nchild);
  int *colSuperF = xmalloc(sizeof(int) * n); /* :768-769 */
  for (int s = 0; s < nsf; s++)
    for (int j = fStart[s]; j < fStart[s + 1]; j++) colSuperF[j] = s;
  int *superStart; /* :773-814 relaxed amalgamation */
  int nsuper;
  if (relax && nsf > 1) {
    int *sf = xmalloc(sizeof(int) * nsf), *sl = xmalloc(sizeof(int) * nsf), *sparent = xmalloc(sizeof(int) * nsf);
    double *sm = xmalloc(sizeof(double) * nsf), *sz = xcalloc(nsf, sizeof(double)),
           *snnz = xmalloc(sizeof(double) * nsf);
    unsigned char *alive = xmalloc(nsf);
    memset(alive, 1, nsf);
    for (int s = 0; s < nsf; s++) {
      sf[s] = fStart[s];
      sl[s] = fStart[s + 1] - 1;
      sm[s] = colCount[fStart[s]];
      double nc = fStart[s + 1] - fStart[s];
      snnz[s] = nc * sm[s] - (nc * (nc - 1)) / 2;
      int pl = parent[sl[s]];
      sparent[s] = pl == -1 ? -1 : colSuperF[pl];
    }
    for (int s = 0; s < nsf; s++) {
      int P = sparent[s];
      if (P == -1 || sf[P] != sl[s] + 1) continue;
      double ncC = sl[s] - sf[s] + 1, ncP = sl[P] - sf[P] + 1;
      double nc = ncC + ncP;
      double m = ncC + sm[P];
      double stored = nc * m - (nc * (nc - 1)) / 2;
      double zeros = stored - snnz[s] - snnz[P] + sz[s] + sz[P];
      double zf = zeros / stored;
      int merge = nc <= 4 || (nc <= 16 && zf < 0.8) || (nc <= 48 && zf < 0.1) || zf < 0.05;
      if (!merge) continue;
      sf[P] = sf[s];
      sm[P] = m;
      sz[P] = zeros;
      snnz[P] += snnz[s];
      alive[s] = 0;
    }
    superStart = xmalloc(sizeof(int) * (nsf + 1));
    nsuper = 0;
    for (int s = 0; s < nsf; s++)
      if (alive[s]) superStart[nsuper++] = sf[s];
    superStart[nsuper] = n;
    free(sf);
    free(sl);
    free(sparent);
    free(sm);
    free(sz);
    free(snnz);
    free(alive);
  } else {
    superStart = xmalloc(sizeof(int) * (nsf + 1));
    memcpy(superStart, fStart, sizeof(int) * (nsf + 1));
    nsuper = nsf;
  }
  free(fStart);
  free(colSuperF);
  int *colSuper = xmalloc(sizeof(int) * n); /* :816-822 */
  for (int s = 0; s < nsuper; s++)
    for (int j = superStart[s]; j < superStart[s + 1]; j++) colSuper[j] = s;
  int *superParent = xmalloc(sizeof(int) * (nsuper + 1));
  for (int s = 0; s < nsuper; s++) {
    int pl = parent[superStart[s + 1] - 1];
    superParent[s] = pl == -1 ? -1 : colSuper[pl];
  }
  int *childHead = ifill(xmalloc(sizeof(int) * (nsuper + 1)), nsuper, -1); /* :824-832 */
  int *childNext = ifill(xmalloc(sizeof(int) * (nsuper + 1)), nsuper, -1);
  for (int s = 0; s < nsuper; s++) {
    int P = superParent[s];
    if (P == -1) continue;
    childNext[s] = childHead[P];
    childHead[P] = s;
  }
  int *Sp = xcalloc(nsuper + 1, sizeof(int)); /* :833-867 row structures */
  int **rowsOf = xmalloc(sizeof(int *) * nsuper);
  int *rowsLen = xmalloc(sizeof(int) * nsuper);
  int *marker = ifill(xmalloc(sizeof(int) * n), n, -1);
  int *below = xmalloc(sizeof(int) * (n + 1));
  int maxFront = 0;
  for (int s = 0; s < nsuper; s++) {
    int f = superStart[s], l = superStart[s + 1] - 1;
    int nb = 0;
    for (int j = f; j <= l; j++)
      for (int p = lowerP[j]; p < lowerP[j + 1]; p++) {
        int i = lowerI[p];
        if (i > l && marker[i] != s) {
          marker[i] = s;
          below[nb++] = i;
        }
      }
    for (int c = childHead[s]; c != -1; c = childNext[c]) {
      int *rc = rowsOf[c];
      int ncc = superStart[c + 1] - superStart[c];
      for (int r = ncc; r < rowsLen[c]; r++) {
        int i = rc[r];
        if (i > l && marker[i] != s) {
          marker[i] = s;
          below[nb++] = i;
        }
      }
    }
    int len = l - f + 1 + nb;
    int *rows = xmalloc(sizeof(int) * (len + 1));
    for (int j = f; j <= l; j++) rows[j - f] = j;
    memcpy(rows + (l - f + 1), below, sizeof(int) * nb);
    qsort(rows + (l - f + 1), nb, sizeof(int), cmp_int); /* :863 numeric typed-array sort */
    rowsOf[s] = rows;
    rowsLen[s] = len;
    Sp[s + 1] = Sp[s] + len;
    if (len > maxFront) maxFront = len;
  }
  free(marker);
  free(below);
  int *Si = xmalloc(sizeof(int) * ((int64_t)Sp[nsuper] + 1)); /* :868-873 */
  int64_t *Lxp = xcalloc(nsuper + 1, sizeof(int64_t));
  for (int s = 0; s < nsuper; s++) {
    memcpy(Si + Sp[s], rowsOf[s], sizeof(int) * rowsLen[s]);
    Lxp[s + 1] = Lxp[s] + (int64_t)rowsLen[s] * (superStart[s + 1] - superStart[s]);
    free(rowsOf[s]);
  }
  free(rowsOf);
  free(rowsLen);
  S->nsuper = nsuper;
  S->maxFront = maxFront;
  S->nnzL = nnzL;
  S->nnzA = nnzA;
  S->nnzLStored = Lxp[nsuper];
  S->fill = (double)nnzL / (double)nnzA;
  S->flops = flops;
  S->perm = perm;
  S->pinv = pinv;
  S->parent = parent;
  S->colCount = colCount;
  S->lowerP = lowerP;
  S->lowerI = lowerI;
  S->lowerSrc = lowerSrc;
  S->superStart = superStart;
  S->colSuper = colSuper;
  S->superParent = superParent;
  S->childHead = childHead;
  S->childNext = childNext;
  S->Sp = Sp;
  S->Si = Si;
  S->Lxp = Lxp;
  return S;
}

ORC_API void orc_sym_free(orc_sym *S) {
  if (!S) return;
  free(S->perm);
  free(S->pinv);
  free(S->parent);
  free(S->colCount);
  free(S->lowerP);
  free(S->lowerI);
  free(S->lowerSrc);
  free(S->superStart);
  free(S->colSuper);
  free(S->superParent);
  free(S->childHead);
  free(S->childNext);
  free(S->Sp);
  free(S->Si);
  free(S->Lxp);
  free(S);
}

/* Scalars of an analysis: n nsuper maxFront patNnz hash, and int64 nnzL nnzA nnzLStored; doubles fill flops. */
ORC_API void orc_sym_info(const orc_sym *S, int *ints, int64_t *longs, double *dbls) {
  ints[0] = S->n;
  ints[1] = S->nsuper;
  ints[2] = S->maxFront;
  ints[3] = S->patNnz;
  ints[4] = (int)S->hash;
  longs[0] = S->nnzL;
  longs[1] = S->nnzA;
  longs[2] = S->nnzLStored;
  dbls[0] = S->fill;
  dbls[1] = S->flops;
}

/* Pointers to the arrays of an analysis (order matches oracle.py). */
ORC_API void orc_sym_arrays(const orc_sym *S, void **out) {
  out[0] = S->perm;
  out[1] = S->pinv;
  out[2] = S->parent;
  out[3] = S->colCount;
  out[4] = S->lowerP;
  out[5] = S->lowerI;
  out[6] = S->lowerSrc;
  out[7] = S->superStart;
  out[8] = S->colSuper;
  out[9] = S->superParent;
  out[10] = S->childHead;
  out[11] = S->childNext;
  out[12] = S->Sp;
  out[13] = S->Si;
  out[14] = S->Lxp;
}

/* ---- front kernels of the JS path ("blocked"): sparse.mjs:992-1098, :1131-1158; ldlt.mjs:492-535 --------------- */

/* panelUpdate: sparse.mjs:1131-1158 */
static int panel_update(double *F, int m, int k, int c0) {
  int64_t kb = (int64_t)k * m;
  int c = c0;
  for (; c + 3 < k; c += 4) {
    int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
    double l0 = F[k + b0], l1 = F[k + b1], l2 = F[k + b2], l3 = F[k + b3];
    for (int i = k; i < m; i++) F[i + kb] -= F[i + b0] * l0 + F[i + b1] * l1 + F[i + b2] * l2 + F[i + b3] * l3;
  }
  for (; c < k; c++) {
    int64_t b0 = (int64_t)c * m;
    double l0 = F[k + b0];
    if (l0 == 0) continue;
    for (int i = k; i < m; i++) F[i + kb] -= F[i + b0] * l0;
  }
  double d = F[k + kb];
  if (!(d > 0)) return 0;
  double dk = sqrt(d);
  F[k + kb] = dk;
  double inv = 1 / dk;
  for (int i = k + 1; i < m; i++) F[i + kb] *= inv;
  return 1;
}

/* Cholesky dense partial factorization of one front, JS loops: sparse.mjs:995-1098 */
static int chol_front_js(double *F, int m, int nc) {
  int k = 0;
  for (; k + 1 < nc; k += 2) {
    int64_t ka = (int64_t)k * m, kb1 = ka + m;
    int c = 0;
    for (; c + 3 < k; c += 4) {
      int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
      double l0 = F[k + b0], l1 = F[k + b1], l2 = F[k + b2], l3 = F[k + b3];
      double e0 = F[k + 1 + b0], e1 = F[k + 1 + b1], e2 = F[k + 1 + b2], e3 = F[k + 1 + b3];
      F[k + ka] -= F[k + b0] * l0 + F[k + b1] * l1 + F[k + b2] * l2 + F[k + b3] * l3;
      for (int i = k + 1; i < m; i++) {
        double f0 = F[i + b0], f1 = F[i + b1], f2 = F[i + b2], f3 = F[i + b3];
        F[i + ka] -= f0 * l0 + f1 * l1 + f2 * l2 + f3 * l3;
        F[i + kb1] -= f0 * e0 + f1 * e1 + f2 * e2 + f3 * e3;
      }
    }
    if (!panel_update(F, m, k, c) || !panel_update(F, m, k + 1, c)) return 0;
  }
  if (k < nc && !panel_update(F, m, k, 0)) return 0;
  int j0 = nc;
  for (; j0 + 1 < m; j0 += 2) {
    int ja = j0, jbb = j0 + 1;
    int64_t ab = (int64_t)ja * m, bb = (int64_t)jbb * m;
    int c = 0;
    for (; c + 3 < nc; c += 4) {
      int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
      double a0 = F[ja + b0], a1 = F[ja + b1], a2 = F[ja + b2], a3 = F[ja + b3];
      double e0 = F[jbb + b0], e1 = F[jbb + b1], e2 = F[jbb + b2], e3 = F[jbb + b3];
      F[ja + ab] -= F[ja + b0] * a0 + F[ja + b1] * a1 + F[ja + b2] * a2 + F[ja + b3] * a3;
      for (int i = jbb; i < m; i++) {
        double f0 = F[i + b0], f1 = F[i + b1], f2 = F[i + b2], f3 = F[i + b3];
        F[i + ab] -= f0 * a0 + f1 * a1 + f2 * a2 + f3 * a3;
        F[i + bb] -= f0 * e0 + f1 * e1 + f2 * e2 + f3 * e3;
      }
    }
    for (; c < nc; c++) {
      int64_t b0 = (int64_t)c * m;
      double a0 = F[ja + b0], e0 = F[jbb + b0];
      if (a0 != 0) F[ja + ab] -= F[ja + b0] * a0;
      if (a0 == 0 && e0 == 0) continue;
      for (int i = jbb; i < m; i++) {
        double f0 = F[i + b0];
        if (a0 != 0) F[i + ab] -= f0 * a0;
        if (e0 != 0) F[i + bb] -= f0 * e0;
      }
    }
  }
  for (int j = j0; j < m; j++) {
    int64_t jb = (int64_t)j * m;
    int c = 0;
    for (; c + 3 < nc; c += 4) {
      int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
      double l0 = F[j + b0], l1 = F[j + b1], l2 = F[j + b2], l3 = F[j + b3];
      for (int i = j; i < m; i++) F[i + jb] -= F[i + b0] * l0 + F[i + b1] * l1 + F[i + b2] * l2 + F[i + b3] * l3;
    }
    for (; c < nc; c++) {
      int64_t b0 = (int64_t)c * m;
      double l0 = F[j + b0];
      if (l0 == 0) continue;
      for (int i = j; i < m; i++) F[i + jb] -= F[i + b0] * l0;
    }
  }
  return 1;
}

/* LDL^T dense partial factorization of one front, JS loops: ldlt.mjs:492-535. Returns 0 on a non-finite pivot. */
static int ldlt_front_js(double *F, int m, int nc, double *D, int f, double tau, int *nNeg, int *nPert) {
  for (int k = 0; k < nc; k++) {
    int64_t kb = (int64_t)k * m;
    int c = 0;
    for (; c + 3 < k; c += 4) {
      int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
      double w0 = F[k + b0] * D[f + c], w1 = F[k + b1] * D[f + c + 1], w2 = F[k + b2] * D[f + c + 2],
             w3 = F[k + b3] * D[f + c + 3];
      for (int i = k; i < m; i++) F[i + kb] -= F[i + b0] * w0 + F[i + b1] * w1 + F[i + b2] * w2 + F[i + b3] * w3;
    }
    for (; c < k; c++) {
      int64_t b0 = (int64_t)c * m;
      double w0 = F[k + b0] * D[f + c];
      if (w0 == 0) continue;
      for (int i = k; i < m; i++) F[i + kb] -= F[i + b0] * w0;
    }
    double d = F[k + kb];
    if (!(fabs(d) >= tau)) {
      if (!isfinite(d)) return 0;
      d = d < 0 ? -tau : tau;
      (*nPert)++;
    }
    if (d < 0) (*nNeg)++;
    D[f + k] = d;
    F[k + kb] = 1;
    double inv = 1 / d;
    for (int i = k + 1; i < m; i++) F[i + kb] *= inv;
  }
  for (int j = nc; j < m; j++) {
    int64_t jb = (int64_t)j * m;
    int c = 0;
    for (; c + 3 < nc; c += 4) {
      int64_t b0 = (int64_t)c * m, b1 = b0 + m, b2 = b1 + m, b3 = b2 + m;
      double w0 = F[j + b0] * D[f + c], w1 = F[j + b1] * D[f + c + 1], w2 = F[j + b2] * D[f + c + 2],
             w3 = F[j + b3] * D[f + c + 3];
      for (int i = j; i < m; i++) F[i + jb] -= F[i + b0] * w0 + F[i + b1] * w1 + F[i + b2] * w2 + F[i + b3] * w3;
    }
    for (; c < nc; c++) {
      int64_t b0 = (int64_t)c * m;
      double w0 = F[j + b0] * D[f + c];
      if (w0 == 0) continue;
      for (int i = j; i < m; i++) F[i + jb] -= F[i + b0] * w0;
    }
  }
  return 1;
}

/* ---- SSE2 restatement of wasm/front-real.mjs (g4, s4, g1, s1 and RealFront.front) ------------------------------ */
/* Per entry: acc - (((a0 w0 + a1 w1) + a2 w2) + a3 w3), rows two at a time, odd last row scalar (front-real.mjs:56-79,
 * 81-124). H is the front (column-major m x m), W the packed weights. */
static void k_g4(double *H, const double *W, int m, int t, int r0, int ng) {
  double *T0 = H + (int64_t)t * m, *T1 = T0 + m, *T2 = T1 + m, *T3 = T2 + m;
  const double *pa = H;
  for (int g = 0; g < ng; g++, pa += 4 * (int64_t)m, W += 16) {
    const double *A0 = pa, *A1 = A0 + m, *A2 = A1 + m, *A3 = A2 + m;
    __m128d w[16];
    for (int q = 0; q < 16; q++) w[q] = _mm_set1_pd(W[q]);
    int o = r0;
    for (; o + 2 <= m; o += 2) {
      __m128d a0 = _mm_loadu_pd(A0 + o), a1 = _mm_loadu_pd(A1 + o), a2 = _mm_loadu_pd(A2 + o),
              a3 = _mm_loadu_pd(A3 + o);
      double *T[4] = {T0, T1, T2, T3};
      for (int jj = 0; jj < 4; jj++) {
        __m128d s = _mm_mul_pd(a0, w[4 * jj]);
        s = _mm_add_pd(s, _mm_mul_pd(a1, w[4 * jj + 1]));
        s = _mm_add_pd(s, _mm_mul_pd(a2, w[4 * jj + 2]));
        s = _mm_add_pd(s, _mm_mul_pd(a3, w[4 * jj + 3]));
        _mm_storeu_pd(T[jj] + o, _mm_sub_pd(_mm_loadu_pd(T[jj] + o), s));
      }
    }
    if (o < m) {
      double *T[4] = {T0, T1, T2, T3};
      for (int jj = 0; jj < 4; jj++) {
        double s = A0[o] * W[4 * jj];
        s = s + A1[o] * W[4 * jj + 1];
        s = s + A2[o] * W[4 * jj + 2];
        s = s + A3[o] * W[4 * jj + 3];
        T[jj][o] = T[jj][o] - s;
      }
    }
  }
}
static void k_g1(double *H, const double *W, int m, int t, int r0, int ng) {
  double *T0 = H + (int64_t)t * m;
  const double *pa = H;
  for (int g = 0; g < ng; g++, pa += 4 * (int64_t)m, W += 4) {
    const double *A0 = pa, *A1 = A0 + m, *A2 = A1 + m, *A3 = A2 + m;
    __m128d w0 = _mm_set1_pd(W[0]), w1 = _mm_set1_pd(W[1]), w2 = _mm_set1_pd(W[2]), w3 = _mm_set1_pd(W[3]);
    int o = r0;
    for (; o + 2 <= m; o += 2) {
      __m128d s = _mm_mul_pd(_mm_loadu_pd(A0 + o), w0);
      s = _mm_add_pd(s, _mm_mul_pd(_mm_loadu_pd(A1 + o), w1));
      s = _mm_add_pd(s, _mm_mul_pd(_mm_loadu_pd(A2 + o), w2));
      s = _mm_add_pd(s, _mm_mul_pd(_mm_loadu_pd(A3 + o), w3));
      _mm_storeu_pd(T0 + o, _mm_sub_pd(_mm_loadu_pd(T0 + o), s));
    }
    if (o < m) {
      double s = A0[o] * W[0];
      s = s + A1[o] * W[1];
      s = s + A2[o] * W[2];
      s = s + A3[o] * W[3];
      T0[o] = T0[o] - s;
    }
  }
}
static void k_s4(double *H, const double *W, int m, int t, int r0, int c) {
  double *T[4];
  T[0] = H + (int64_t)t * m;
  for (int jj = 1; jj < 4; jj++) T[jj] = T[jj - 1] + m;
  const double *A = H + (int64_t)c * m;
  __m128d w[4];
  for (int jj = 0; jj < 4; jj++) w[jj] = _mm_set1_pd(W[jj]);
  int o = r0;
  for (; o + 2 <= m; o += 2) {
    __m128d av = _mm_loadu_pd(A + o);
    for (int jj = 0; jj < 4; jj++) _mm_storeu_pd(T[jj] + o, _mm_sub_pd(_mm_loadu_pd(T[jj] + o), _mm_mul_pd(av, w[jj])));
  }
  if (o < m)
    for (int jj = 0; jj < 4; jj++) T[jj][o] = T[jj][o] - A[o] * W[jj];
}
static void k_s1(double *H, double wv, int m, int t, int r0, int c) {
  double *T0 = H + (int64_t)t * m;
  const double *A = H + (int64_t)c * m;
  __m128d w = _mm_set1_pd(wv);
  int o = r0;
  for (; o + 2 <= m; o += 2) _mm_storeu_pd(T0 + o, _mm_sub_pd(_mm_loadu_pd(T0 + o), _mm_mul_pd(_mm_loadu_pd(A + o), w)));
  if (o < m) T0[o] = T0[o] - A[o] * wv;
}

typedef struct {
  double *H, *W;
  int m, ldlt, f;
  const double *D;
} rf_ctx;
static inline double rf_wt(const rf_ctx *x, int t, int c) {
  double v = x->H[t + (int64_t)c * x->m];
  return x->ldlt ? v * x->D[x->f + c] : v;
}
static void rf_pack4(rf_ctx *x, int t, int ng) { /* front-real.mjs:324-329 */
  for (int g = 0; g < ng; g++)
    for (int jj = 0; jj < 4; jj++)
      for (int q = 0; q < 4; q++) x->W[16 * g + 4 * jj + q] = rf_wt(x, t + jj, 4 * g + q);
}
static void rf_pack1(rf_ctx *x, int t, int ng) { /* :331-335 */
  for (int g = 0; g < ng; g++)
    for (int q = 0; q < 4; q++) x->W[4 * g + q] = rf_wt(x, t, 4 * g + q);
}
static void rf_heads(rf_ctx *x, int t, int ng, int s0, int s1) { /* :337-356 */
  double *H = x->H, *W = x->W;
  int m = x->m;
  for (int jj = 0; jj < 3; jj++) {
    int64_t tb = (int64_t)(t + jj) * m;
    for (int i = t + jj; i < t + 3; i++) {
      for (int g = 0; g < ng; g++) {
        int64_t b0 = (int64_t)4 * g * m;
        const double *wb = W + 16 * g + 4 * jj;
        H[i + tb] -= H[i + b0] * wb[0] + H[i + b0 + m] * wb[1] + H[i + b0 + 2 * m] * wb[2] + H[i + b0 + 3 * m] * wb[3];
      }
      for (int c = s0; c < s1; c++) {
        double w = rf_wt(x, t + jj, c);
        if (w != 0) H[i + tb] -= H[i + (int64_t)c * m] * w;
      }
    }
  }
}
static void rf_single(rf_ctx *x, int t, int c, double w, int r0) { /* :359-365 */
  if (w == 0) return;
  int m = x->m;
  if (m - r0 >= 8)
    k_s1(x->H, w, m, t, r0, c);
  else {
    double *H = x->H;
    int64_t tb = (int64_t)t * m, cb = (int64_t)c * m;
    for (int i = r0; i < m; i++) H[i + tb] -= H[i + cb] * w;
  }
}
static int rf_pivot(rf_ctx *x, int t, double *D, double tau, int *nNeg, int *nPert) { /* :367-389 */
  double *H = x->H;
  int m = x->m;
  int64_t tb = (int64_t)t * m;
  double d = H[t + tb];
  if (!x->ldlt) {
    if (!(d > 0)) return 0;
    double dk = sqrt(d);
    H[t + tb] = dk;
    double inv = 1 / dk;
    for (int i = t + 1; i < m; i++) H[i + tb] *= inv;
    return 1;
  }
  if (!(fabs(d) >= tau)) {
    if (!isfinite(d)) return 0;
    d = d < 0 ? -tau : tau;
    (*nPert)++;
  }
  if (d < 0) (*nNeg)++;
  D[x->f + t] = d;
  H[t + tb] = 1;
  double inv = 1 / d;
  for (int i = t + 1; i < m; i++) H[i + tb] *= inv;
  return 1;
}
/* RealFront.front: front-real.mjs:259-321 */
static int rf_front(double *H, double *W, int m, int nc, int ldlt, double *D, int f, double tau, int *nNeg,
                    int *nPert) {
  rf_ctx x = {H, W, m, ldlt, f, D};
  int k = 0;
  for (; k + 3 < nc; k += 4) {
    int ng = k >> 2;
    if (ng > 0) {
      rf_pack4(&x, k, ng);
      rf_heads(&x, k, ng, 0, 0);
      k_g4(H, W, m, k, k + 3, ng);
    }
    for (int jj = 0; jj < 4; jj++) {
      int t = k + jj;
      for (int c = k; c < t; c++) rf_single(&x, t, c, rf_wt(&x, t, c), t);
      if (!rf_pivot(&x, t, D, tau, nNeg, nPert)) return 0;
    }
  }
  for (; k < nc; k++) {
    int ng = k >> 2;
    if (ng > 0) {
      rf_pack1(&x, k, ng);
      k_g1(H, W, m, k, k, ng);
    }
    for (int c = 4 * ng; c < k; c++) rf_single(&x, k, c, rf_wt(&x, k, c), k);
    if (!rf_pivot(&x, k, D, tau, nNeg, nPert)) return 0;
  }
  int ng = nc >> 2, c4 = 4 * ng;
  int j = nc;
  for (; j + 3 < m; j += 4) {
    if (ng > 0) {
      rf_pack4(&x, j, ng);
      rf_heads(&x, j, ng, c4, nc);
      k_g4(H, W, m, j, j + 3, ng);
    } else if (c4 < nc)
      rf_heads(&x, j, 0, c4, nc);
    for (int c = c4; c < nc; c++) {
      double w0 = rf_wt(&x, j, c), w1 = rf_wt(&x, j + 1, c), w2 = rf_wt(&x, j + 2, c), w3 = rf_wt(&x, j + 3, c);
      if (w0 != 0 && w1 != 0 && w2 != 0 && w3 != 0) {
        W[0] = w0;
        W[1] = w1;
        W[2] = w2;
        W[3] = w3;
        k_s4(H, W, m, j, j + 3, c);
      } else {
        if (w0 != 0) k_s1(H, w0, m, j, j + 3, c);
        if (w1 != 0) k_s1(H, w1, m, j + 1, j + 3, c);
        if (w2 != 0) k_s1(H, w2, m, j + 2, j + 3, c);
        if (w3 != 0) k_s1(H, w3, m, j + 3, j + 3, c);
      }
    }
  }
  for (; j < m; j++) {
    if (ng > 0) {
      rf_pack1(&x, j, ng);
      k_g1(H, W, m, j, j, ng);
    }
    for (int c = c4; c < nc; c++) rf_single(&x, j, c, rf_wt(&x, j, c), j);
  }
  return 1;
}

/* ---- multifrontal driver shared by Cholesky (sparse.mjs:941-1125) and LDL^T (ldlt.mjs:450-562) ------------------ */
#define WASM_MIN_FRONT 32 /* front-real.mjs:202 */

/* kind: 0 Cholesky, 1 LDL^T. simd: 0 JS loops only ('blocked'), 1 SSE2 front kernel for m >= 32 ('wasm').
 * Returns 1 ok, 0 numerical failure. Lx has nnzLStored entries; D (LDL^T) has n. stats: nNeg, nPerturbed. */
ORC_API int orc_factor_range(const orc_sym *S, const double *values, int kind, int simd, double pivotTol, double *Lx,
                             double *D, int *stats, int s_first, int s_last);
ORC_API int orc_factor(const orc_sym *S, const double *values, int kind, int simd, double pivotTol, double *Lx,
                       double *D, int *stats) {
  return orc_factor_range(S, values, kind, simd, pivotTol, Lx, D, stats, 0, S->nsuper - 1);
}

/* The same multifrontal loop over supernodes s_first .. s_last only: a complete subtree in postorder (s_last its root,
 * s_first its first descendant). Used to time a bounded sample of a large factorization. */
ORC_API int orc_factor_range(const orc_sym *S, const double *values, int kind, int simd, double pivotTol, double *Lx,
                             double *D, int *stats, int s_first, int s_last) {
  int n = S->n, nsuper = S->nsuper, maxFront = S->maxFront;
  stats[0] = stats[1] = 0;
  if (n == 0) return 1;
  double tau = 0;
  if (kind == 1) { /* ldlt.mjs:419-424 diagScale, :458 */
    double amax = 0;
    for (int j = 0; j < n; j++)
      for (int p = S->lowerP[j]; p < S->lowerP[j + 1]; p++)
        if (S->lowerI[p] == j) {
          amax = js_max(amax, fabs(values[S->lowerSrc[p]]));
        }
    tau = pivotTol * (amax > 0 ? amax : 1);
  }
  double *F = xmalloc(sizeof(double) * (size_t)maxFront * maxFront);
  double *W = xmalloc(sizeof(double) * (8 * (size_t)maxFront + 64));
  int *rel = xcalloc(n, sizeof(int));
  size_t stackCap = 1024, top = 0;
  double *stack = xmalloc(sizeof(double) * stackCap);
  int *stackDim = xcalloc(nsuper, sizeof(int));
  size_t *stackPos = xmalloc(sizeof(size_t) * (nsuper + 1));
  int nsp = 0;
  int nNeg = 0, nPert = 0, ok = 1;
  for (int s = s_first; s <= s_last && s < nsuper && ok; s++) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f;
    int r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    for (int r = 0; r < m; r++) rel[S->Si[r0 + r]] = r;
    for (int b = 0; b < m; b++) memset(F + (int64_t)b * m + b, 0, sizeof(double) * (m - b));
    for (int c = 0; c < nc; c++) {
      int j = f + c;
      int64_t cb = (int64_t)c * m;
      for (int p = S->lowerP[j]; p < S->lowerP[j + 1]; p++) F[rel[S->lowerI[p]] + cb] += values[S->lowerSrc[p]];
    }
    for (int ch = S->childHead[s]; ch != -1; ch = S->childNext[ch]) {
      size_t off = stackPos[--nsp];
      int mu = stackDim[ch];
      int cr0 = S->Sp[ch] + (S->superStart[ch + 1] - S->superStart[ch]);
      for (int b = 0; b < mu; b++) {
        int64_t cb = (int64_t)rel[S->Si[cr0 + b]] * m;
        size_t ub = off + (size_t)b * mu;
        for (int a = b; a < mu; a++) F[rel[S->Si[cr0 + a]] + cb] += stack[ub + a];
      }
      top = off;
    }
    if (simd && m >= WASM_MIN_FRONT) {
      if (!rf_front(F, W, m, nc, kind, D, f, tau, &nNeg, &nPert)) ok = 0;
    } else if (kind == 0) {
      if (!chol_front_js(F, m, nc)) ok = 0;
    } else if (!ldlt_front_js(F, m, nc, D, f, tau, &nNeg, &nPert))
      ok = 0;
    if (!ok) break;
    memcpy(Lx + S->Lxp[s], F, sizeof(double) * (size_t)m * nc);
    int mu = m - nc;
    stackDim[s] = mu;
    if (mu > 0) {
      size_t need = top + (size_t)mu * mu;
      if (need > stackCap) {
        size_t nc2 = need > 2 * stackCap ? need : 2 * stackCap;
        double *bigger = xmalloc(sizeof(double) * nc2);
        memcpy(bigger, stack, sizeof(double) * top);
        free(stack);
        stack = bigger;
        stackCap = nc2;
      }
      for (int b = 0; b < mu; b++) {
        int64_t src = (int64_t)(nc + b) * m + nc;
        size_t dst = top + (size_t)b * mu;
        for (int a = b; a < mu; a++) stack[dst + a] = F[src + a];
      }
      stackPos[nsp++] = top;
      top = need;
    } else
      stackPos[nsp++] = top;
  }
  stats[0] = nNeg;
  stats[1] = nPert;
  free(F);
  free(W);
  free(rel);
  free(stack);
  free(stackDim);
  free(stackPos);
  return ok;
}

/* ---- Cholesky solves: sparse.mjs:1160-1305 (JS) and wasm/solve-real.mjs:451-473 (kernels) ----------------------- */
static void below_accumulate(const double *Lx, int64_t lo, int m, int nc, int mu, const double *y, int f, double *t) {
  for (int r = 0; r < mu; r++) t[r] = 0; /* sparse.mjs:1161-1176 */
  int c = 0;
  for (; c + 1 < nc; c += 2) {
    int64_t ca = lo + (int64_t)c * m + nc, cb = ca + m;
    double ya = y[f + c], yb = y[f + c + 1];
    for (int r = 0; r < mu; r++) t[r] += Lx[ca + r] * ya + Lx[cb + r] * yb;
  }
  if (c < nc) {
    int64_t ca = lo + (int64_t)c * m + nc;
    double ya = y[f + c];
    for (int r = 0; r < mu; r++) t[r] += Lx[ca + r] * ya;
  }
}
static double dot_below(const double *Lx, int64_t o, const double *t, int mu) { /* :1179-1193 */
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int r = 0;
  for (; r + 3 < mu; r += 4) {
    s0 += Lx[o + r] * t[r];
    s1 += Lx[o + r + 1] * t[r + 1];
    s2 += Lx[o + r + 2] * t[r + 2];
    s3 += Lx[o + r + 3] * t[r + 3];
  }
  for (; r < mu; r++) s0 += Lx[o + r] * t[r];
  return s0 + s1 + (s2 + s3);
}

/* SSE2 fdiag / facc / bdiag: solve-real.mjs:47-207 */
static void k_fdiag(const double *L, double *y, int m, int nc) {
  for (int c = 0; c < nc; c++) {
    const double *col = L + (int64_t)c * m;
    double yj = y[c] / col[c];
    y[c] = yj;
    __m128d vy = _mm_set1_pd(yj);
    int o = c + 1;
    for (; o + 2 <= nc; o += 2) _mm_storeu_pd(y + o, _mm_sub_pd(_mm_loadu_pd(y + o), _mm_mul_pd(_mm_loadu_pd(col + o), vy)));
    if (o < nc) y[o] = y[o] - col[o] * yj;
  }
}
static void k_facc(const double *L, const double *y, double *t, int m, int nc, int mu) {
  int o = 0;
  for (; o + 2 <= mu; o += 2) _mm_storeu_pd(t + o, _mm_setzero_pd());
  if (o < mu) t[o] = 0;
  const double *A0 = L + nc;
  int c = 0;
#define PASS(ncol)                                                                                       \
  do {                                                                                                   \
    const double *A[4];                                                                                  \
    A[0] = A0;                                                                                           \
    for (int q = 1; q < (ncol); q++) A[q] = A[q - 1] + m;                                                \
    double ys[4];                                                                                        \
    __m128d vs[4];                                                                                       \
    for (int q = 0; q < (ncol); q++) {                                                                   \
      ys[q] = y[c + q];                                                                                  \
      vs[q] = _mm_set1_pd(ys[q]);                                                                        \
    }                                                                                                    \
    int oo = 0;                                                                                          \
    for (; oo + 2 <= mu; oo += 2) {                                                                      \
      __m128d acc = _mm_loadu_pd(t + oo);                                                                \
      if ((ncol) == 1)                                                                                   \
        acc = _mm_add_pd(acc, _mm_mul_pd(_mm_loadu_pd(A[0] + oo), vs[0]));                               \
      else                                                                                               \
        for (int pp = 0; pp < (ncol); pp += 2)                                                           \
          acc = _mm_add_pd(acc, _mm_add_pd(_mm_mul_pd(_mm_loadu_pd(A[pp] + oo), vs[pp]),                 \
                                           _mm_mul_pd(_mm_loadu_pd(A[pp + 1] + oo), vs[pp + 1])));       \
      _mm_storeu_pd(t + oo, acc);                                                                        \
    }                                                                                                    \
    if (oo < mu) {                                                                                       \
      double acc = t[oo];                                                                                \
      if ((ncol) == 1)                                                                                   \
        acc = acc + A[0][oo] * ys[0];                                                                    \
      else                                                                                               \
        for (int pp = 0; pp < (ncol); pp += 2) acc = acc + (A[pp][oo] * ys[pp] + A[pp + 1][oo] * ys[pp + 1]); \
      t[oo] = acc;                                                                                       \
    }                                                                                                    \
    c += (ncol);                                                                                         \
    A0 += (int64_t)(ncol) * m;                                                                           \
  } while (0)
  while (c + 3 < nc) PASS(4);
  if (c + 1 < nc) PASS(2);
  if (c < nc) PASS(1);
#undef PASS
}
static void k_bdiag(const double *L, double *y, const double *t, int m, int nc, int mu) {
  for (int c = nc - 1; c >= 0; c--) {
    const double *col = L + (int64_t)c * m;
    double w = y[c];
    for (int o = c + 1; o < nc; o++) w = w - col[o] * y[o];
    const double *lb = col + nc;
    __m128d a01 = _mm_setzero_pd(), a23 = _mm_setzero_pd();
    int o = 0;
    for (; o + 4 <= mu; o += 4) {
      a01 = _mm_add_pd(a01, _mm_mul_pd(_mm_loadu_pd(lb + o), _mm_loadu_pd(t + o)));
      a23 = _mm_add_pd(a23, _mm_mul_pd(_mm_loadu_pd(lb + o + 2), _mm_loadu_pd(t + o + 2)));
    }
    double s[4];
    _mm_storeu_pd(s, a01);
    _mm_storeu_pd(s + 2, a23);
    for (; o < mu; o++) s[0] = s[0] + lb[o] * t[o];
    y[c] = (w - ((s[0] + s[1]) + (s[2] + s[3]))) / col[c];
  }
}

#define SOLVE_MIN_NNZL 50000 /* solve-real.mjs:414 */

/* One Cholesky solve. simd: 0 = JS solveNumeric; 1 = reference default (WASM kernels when nnzLStored >= 50000). */
ORC_API void orc_solve_chol(const orc_sym *S, const double *Lx, const double *b, double *x, int simd) {
  int n = S->n, nsuper = S->nsuper;
  if (n == 0) return;
  double *y = xmalloc(sizeof(double) * n), *t = xmalloc(sizeof(double) * (S->maxFront + 1));
  int useK = simd && S->nnzLStored >= SOLVE_MIN_NNZL;
  for (int i = 0; i < n; i++) y[i] = b[S->perm[i]];
  for (int s = 0; s < nsuper; s++) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0, mu = m - nc;
    int64_t lo = S->Lxp[s];
    if (useK)
      k_fdiag(Lx + lo, y + f, m, nc);
    else
      for (int c = 0; c < nc; c++) {
        int64_t cb = lo + (int64_t)c * m;
        double yj = (y[f + c] /= Lx[cb + c]);
        for (int r = c + 1; r < nc; r++) y[f + r] -= Lx[cb + r] * yj;
      }
    if (mu == 0) continue;
    if (useK)
      k_facc(Lx + lo, y + f, t, m, nc, mu);
    else
      below_accumulate(Lx, lo, m, nc, mu, y, f, t);
    int rb = r0 + nc;
    for (int r = 0; r < mu; r++) y[S->Si[rb + r]] -= t[r];
  }
  for (int s = nsuper - 1; s >= 0; s--) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0, mu = m - nc;
    int64_t lo = S->Lxp[s];
    int rb = r0 + nc;
    for (int r = 0; r < mu; r++) t[r] = y[S->Si[rb + r]];
    if (useK)
      k_bdiag(Lx + lo, y + f, t, m, nc, mu);
    else
      for (int c = nc - 1; c >= 0; c--) {
        int64_t cb = lo + (int64_t)c * m;
        double w = y[f + c];
        for (int r = c + 1; r < nc; r++) w -= Lx[cb + r] * y[f + r];
        y[f + c] = (w - dot_below(Lx, cb + nc, t, mu)) / Lx[cb + c];
      }
  }
  for (int i = 0; i < n; i++) x[S->perm[i]] = y[i];
  free(y);
  free(t);
}

/* ---- LDL^T solves: ldlt.mjs:565-643 (JS) and wasm/solve-real.mjs:483-534 (kernels) ------------------------------ */
/* q vectors stored one after another (b[k n + i]). simd: 1 = reference default (WASM kernels when nnzLStored >= 50000,
 * in chunks of QCAP = 8 vectors). Per entry both paths are the same arithmetic. */
#define QCAP 8
static void ldlt_solve1(const orc_sym *S, const double *Lx, const double *D, const double *b, double *x) {
  int n = S->n; /* ldlt.mjs:613-643 (lfwd1 / lbwd1 apply the same per-entry operations) */
  double *y = xmalloc(sizeof(double) * n);
  for (int i = 0; i < n; i++) y[i] = b[S->perm[i]];
  for (int s = 0; s < S->nsuper; s++) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    int64_t lo = S->Lxp[s];
    for (int c = 0; c < nc; c++) {
      int64_t cb = lo + (int64_t)c * m;
      double yj = y[f + c];
      if (yj == 0) continue;
      for (int r = c + 1; r < nc; r++) y[f + r] -= Lx[cb + r] * yj;
      for (int r = nc; r < m; r++) y[S->Si[r0 + r]] -= Lx[cb + r] * yj;
    }
  }
  for (int j = 0; j < n; j++) y[j] /= D[j];
  for (int s = S->nsuper - 1; s >= 0; s--) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    int64_t lo = S->Lxp[s];
    for (int c = nc - 1; c >= 0; c--) {
      int64_t cb = lo + (int64_t)c * m;
      double v = y[f + c];
      for (int r = c + 1; r < nc; r++) v -= Lx[cb + r] * y[f + r];
      for (int r = nc; r < m; r++) v -= Lx[cb + r] * y[S->Si[r0 + r]];
      y[f + c] = v;
    }
  }
  for (int i = 0; i < n; i++) x[S->perm[i]] = y[i];
  free(y);
}
static void ldlt_solveq(const orc_sym *S, const double *Lx, const double *D, const double *b, int q, double *x,
                        int k0, int qq) {
  int n = S->n; /* ldlt.mjs:565-611 on vectors k0 .. k0 + qq - 1 (lfwdq / lbwdq: same per-entry operations) */
  double *y = xmalloc(sizeof(double) * (size_t)n * qq), *v = xmalloc(sizeof(double) * qq);
  (void)q;
  for (int i = 0; i < n; i++) {
    int pi = S->perm[i];
    for (int k = 0; k < qq; k++) y[(size_t)i * qq + k] = b[(size_t)(k0 + k) * n + pi];
  }
  for (int s = 0; s < S->nsuper; s++) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    int64_t lo = S->Lxp[s];
    for (int c = 0; c < nc; c++) {
      int64_t cb = lo + (int64_t)c * m;
      size_t jq = (size_t)(f + c) * qq;
      for (int r = c + 1; r < m; r++) {
        double l = Lx[cb + r];
        if (l == 0) continue;
        size_t iq = (size_t)S->Si[r0 + r] * qq;
        for (int k = 0; k < qq; k++) y[iq + k] -= l * y[jq + k];
      }
    }
  }
  for (int j = 0; j < n; j++) {
    double dj = 1 / D[j];
    for (int k = 0; k < qq; k++) y[(size_t)j * qq + k] *= dj;
  }
  for (int s = S->nsuper - 1; s >= 0; s--) {
    int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    int64_t lo = S->Lxp[s];
    for (int c = nc - 1; c >= 0; c--) {
      int64_t cb = lo + (int64_t)c * m;
      size_t jq = (size_t)(f + c) * qq;
      for (int k = 0; k < qq; k++) v[k] = y[jq + k];
      for (int r = c + 1; r < m; r++) {
        double l = Lx[cb + r];
        if (l == 0) continue;
        size_t iq = (size_t)S->Si[r0 + r] * qq;
        for (int k = 0; k < qq; k++) v[k] -= l * y[iq + k];
      }
      for (int k = 0; k < qq; k++) y[jq + k] = v[k];
    }
  }
  for (int i = 0; i < n; i++) {
    int pi = S->perm[i];
    for (int k = 0; k < qq; k++) x[(size_t)(k0 + k) * n + pi] = y[(size_t)i * qq + k];
  }
  free(y);
  free(v);
}
ORC_API void orc_solve_ldlt(const orc_sym *S, const double *Lx, const double *D, const double *b, int q, double *x,
                            int simd) {
  if (S->n == 0) return;
  if (q == 1) { /* solveMany(b, 1) -> solve (ldlt.mjs:215 / solve-real.mjs ldltSolveWasm) */
    ldlt_solve1(S, Lx, D, b, x);
    return;
  }
  if (simd && S->nnzLStored >= SOLVE_MIN_NNZL) {
    for (int k0 = 0; k0 < q; k0 += QCAP) { /* solve-real.mjs:504-534: chunks of QCAP, qq = 1 still uses lfwdq */
      int qq = q - k0 < QCAP ? q - k0 : QCAP;
      ldlt_solveq(S, Lx, D, b, q, x, k0, qq);
    }
  } else
    ldlt_solveq(S, Lx, D, b, q, x, 0, q);
}

/* ---- matVec and iterative refinement: sparse.mjs:219-228, ldlt.mjs:253-275 ------------------------------------- */
ORC_API void orc_matvec(int n, const int *rowptr, const int *colidx, const double *val, const double *x, double *y) {
  for (int i = 0; i < n; i++) {
    double s = 0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) s += val[p] * x[colidx[p]];
    y[i] = s;
  }
}

/* kind 0: Cholesky factor (Lx), kind 1: LDL^T (Lx, D). Returns steps; rel residual in *rel. */
ORC_API int orc_solve_refined(const orc_sym *S, const int *rowptr, const int *colidx, const double *values,
                              const double *Lx, const double *D, int kind, const double *b, int maxSteps, double tol,
                              double *x, double *rel_out) {
  int n = S->n;
  double *r = xmalloc(sizeof(double) * (n + 1)), *dx = xmalloc(sizeof(double) * (n + 1));
  if (kind == 0)
    orc_solve_chol(S, Lx, b, x, 1);
  else
    orc_solve_ldlt(S, Lx, D, b, 1, x, 1);
  double bn = 0;
  for (int i = 0; i < n; i++) bn += b[i] * b[i];
  bn = sqrt(bn);
  if (bn == 0 || bn != bn) bn = 1; /* Math.sqrt(bn) || 1 */
  double rel = INFINITY;
  int steps = 0;
  for (; steps <= maxSteps; steps++) {
    double rn = 0;
    for (int i = 0; i < n; i++) {
      double s = b[i];
      for (int p = rowptr[i]; p < rowptr[i + 1]; p++) s -= values[p] * x[colidx[p]];
      r[i] = s;
      rn += s * s;
    }
    rel = sqrt(rn) / bn;
    if (rel < tol || steps == maxSteps) break;
    if (kind == 0)
      orc_solve_chol(S, Lx, r, dx, 1);
    else
      orc_solve_ldlt(S, Lx, D, r, 1, dx, 1);
    for (int i = 0; i < n; i++) x[i] += dx[i];
  }
  *rel_out = rel;
  free(r);
  free(dx);
  return steps;
}


/* ---- complex-symmetric supernodal LDL^T: ldlt.mjs:648-864 (ComplexSupernodalLDLT) ---------------------------------
 * A = A^T complex (no conjugation), values as two arrays (re, im) on the CSR slots. Multifrontal over the supernodal
 * tree with dense column-major complex fronts (planar: Fr, Fi), left-looking within the front: column k is updated by
 * the earlier pivot columns (update(k, k)), its pivot settled (|d| < tau -> d scaled to magnitude tau, or tau when
 * d = 0; non-finite -> failure), L(:, k) = F(:, k) / d with a unit diagonal; the update block's columns take all
 * pivot columns (update(j, j)); the update block goes on the stack. tau = pivotTol * max_i hypot(A(i, i)) (diagScale,
 * ldlt.mjs:419-424; C hypot stands for Math.hypot). Returns 1 (ok) or 0; stats[0] = nPerturbed. */
ORC_API int orc_cfactor(const orc_sym *S, const double *re, const double *im, double pivotTol, double *Lr, double *Li,
                        double *Dr, double *Di, int *stats) {
  int n = S->n, nsuper = S->nsuper, maxFront = S->maxFront;
  stats[0] = 0;
  if (n == 0) return 1;
  double amax = 0;
  for (int j = 0; j < n; j++)
    for (int p = S->lowerP[j]; p < S->lowerP[j + 1]; p++)
      if (S->lowerI[p] == j) amax = js_max(amax, hypot(re[S->lowerSrc[p]], im[S->lowerSrc[p]]));
  const double tau = pivotTol * (amax > 0 ? amax : 1);
  double *Fr = xmalloc(sizeof(double) * (size_t)maxFront * maxFront + 8);
  double *Fi = xmalloc(sizeof(double) * (size_t)maxFront * maxFront + 8);
  int *rel = xcalloc(n, sizeof(int));
  size_t cap = 1024, top = 0;
  double *sr = xmalloc(sizeof(double) * cap), *si = xmalloc(sizeof(double) * cap);
  int *stackDim = xcalloc(nsuper, sizeof(int));
  size_t *stackPos = xmalloc(sizeof(size_t) * (nsuper + 1));
  int nsp = 0, nPert = 0, ok = 1;
  for (int s = 0; s < nsuper && ok; s++) {
    const int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    for (int r = 0; r < m; r++) rel[S->Si[r0 + r]] = r;
    for (int b = 0; b < m; b++)
      for (int a = b; a < m; a++) Fr[(size_t)b * m + a] = Fi[(size_t)b * m + a] = 0.0;
    for (int c = 0; c < nc; c++) {
      const int j = f + c;
      const size_t cb = (size_t)c * m;
      for (int p = S->lowerP[j]; p < S->lowerP[j + 1]; p++) {
        const size_t at = rel[S->lowerI[p]] + cb;
        Fr[at] += re[S->lowerSrc[p]];
        Fi[at] += im[S->lowerSrc[p]];
      }
    }
    for (int ch = S->childHead[s]; ch != -1; ch = S->childNext[ch]) {
      const size_t off = stackPos[--nsp];
      const int mu = stackDim[ch];
      const int cr0 = S->Sp[ch] + (S->superStart[ch + 1] - S->superStart[ch]);
      for (int b = 0; b < mu; b++) {
        const size_t cbb = (size_t)rel[S->Si[cr0 + b]] * m, ub = off + (size_t)b * mu;
        for (int a = b; a < mu; a++) {
          const size_t at = rel[S->Si[cr0 + a]] + cbb;
          Fr[at] += sr[ub + a];
          Fi[at] += si[ub + a];
        }
      }
      top = off;
    }
    /* update(k, lim): column k (rows i >= lim) -= sum_{c < min(k, nc)} L[:, c] D[c] L[k, c] */
#define CUPDATE(K, LIM)                                              \
    do {                                                             \
      const int k_ = (K), lim_ = (LIM);                              \
      const size_t kb_ = (size_t)k_ * m;                             \
      const int cmax_ = k_ < nc ? k_ : nc;                           \
      for (int c = 0; c < cmax_; c++) {                              \
        const size_t b0 = (size_t)c * m;                             \
        const double lr = Fr[k_ + b0], li = Fi[k_ + b0];             \
        const double dr = Dr[f + c], di = Di[f + c];                 \
        const double wr = lr * dr - li * di, wi = lr * di + li * dr; \
        if (wr == 0 && wi == 0) continue;                            \
        for (int i = lim_; i < m; i++) {                             \
          const double ar = Fr[i + b0], ai = Fi[i + b0];             \
          Fr[i + kb_] -= ar * wr - ai * wi;                          \
          Fi[i + kb_] -= ar * wi + ai * wr;                          \
        }                                                            \
      }                                                              \
    } while (0)
    for (int k = 0; k < nc && ok; k++) {
      CUPDATE(k, k);
      const size_t kb = (size_t)k * m;
      double dr = Fr[k + kb], di = Fi[k + kb];
      const double mag = hypot(dr, di);
      if (!(mag >= tau)) {
        if (!isfinite(mag)) {
          ok = 0;
          break;
        }
        if (mag == 0) {
          dr = tau;
        } else {
          dr *= tau / mag;
          di *= tau / mag;
        }
        nPert++;
      }
      Dr[f + k] = dr;
      Di[f + k] = di;
      Fr[k + kb] = 1;
      Fi[k + kb] = 0;
      const double den = dr * dr + di * di, ir = dr / den, ii = -di / den;
      for (int i = k + 1; i < m; i++) {
        const double ar = Fr[i + kb], ai = Fi[i + kb];
        Fr[i + kb] = ar * ir - ai * ii;
        Fi[i + kb] = ar * ii + ai * ir;
      }
    }
    if (!ok) break;
    for (int j = nc; j < m; j++) CUPDATE(j, j);
#undef CUPDATE
    memcpy(Lr + S->Lxp[s], Fr, sizeof(double) * (size_t)m * nc);
    memcpy(Li + S->Lxp[s], Fi, sizeof(double) * (size_t)m * nc);
    const int mu = m - nc;
    stackDim[s] = mu;
    if (mu > 0) {
      const size_t need = top + (size_t)mu * mu;
      if (need > cap) {
        size_t len = need > 2 * cap ? need : 2 * cap;
        sr = xrealloc(sr, sizeof(double) * len);
        si = xrealloc(si, sizeof(double) * len);
        cap = len;
      }
      for (int b = 0; b < mu; b++) {
        const size_t src = (size_t)(nc + b) * m + nc, dst = top + (size_t)b * mu;
        for (int a = b; a < mu; a++) {
          sr[dst + a] = Fr[src + a];
          si[dst + a] = Fi[src + a];
        }
      }
      stackPos[nsp++] = top;
      top = need;
    } else {
      stackPos[nsp++] = top;
    }
  }
  free(Fr);
  free(Fi);
  free(rel);
  free(sr);
  free(si);
  free(stackDim);
  free(stackPos);
  stats[0] = nPert;
  return ok;
}

/* ComplexSupernodalLDLT.solve (ldlt.mjs:802-862, the JS path): y = P b; forward with the unit lower L column by column
 * (zero columns skipped); y /= D; backward; x = P^T y. */
ORC_API void orc_csolve(const orc_sym *S, const double *Lr, const double *Li, const double *Dr, const double *Di,
                        const double *br, const double *bi, double *xr, double *xi) {
  const int n = S->n;
  double *yr = xmalloc(sizeof(double) * (n + 1)), *yi = xmalloc(sizeof(double) * (n + 1));
  for (int i = 0; i < n; i++) {
    yr[i] = br[S->perm[i]];
    yi[i] = bi[S->perm[i]];
  }
  for (int s = 0; s < S->nsuper; s++) {
    const int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    const int64_t lo = S->Lxp[s];
    for (int c = 0; c < nc; c++) {
      const int64_t cb = lo + (int64_t)c * m;
      const double a = yr[f + c], b = yi[f + c];
      if (a == 0 && b == 0) continue;
      for (int r = c + 1; r < m; r++) {
        const double lr = Lr[cb + r], li = Li[cb + r];
        const int t = S->Si[r0 + r];
        yr[t] -= lr * a - li * b;
        yi[t] -= lr * b + li * a;
      }
    }
  }
  for (int j = 0; j < n; j++) {
    const double ar = Dr[j], ai = Di[j], den = ar * ar + ai * ai, a = yr[j], b = yi[j];
    yr[j] = (a * ar + b * ai) / den;
    yi[j] = (b * ar - a * ai) / den;
  }
  for (int s = S->nsuper - 1; s >= 0; s--) {
    const int f = S->superStart[s], nc = S->superStart[s + 1] - f, r0 = S->Sp[s], m = S->Sp[s + 1] - r0;
    const int64_t lo = S->Lxp[s];
    for (int c = nc - 1; c >= 0; c--) {
      const int64_t cb = lo + (int64_t)c * m;
      double a = yr[f + c], b = yi[f + c];
      for (int r = c + 1; r < m; r++) {
        const double lr = Lr[cb + r], li = Li[cb + r];
        const int t = S->Si[r0 + r];
        a -= lr * yr[t] - li * yi[t];
        b -= lr * yi[t] + li * yr[t];
      }
      yr[f + c] = a;
      yi[f + c] = b;
    }
  }
  for (int i = 0; i < n; i++) {
    xr[S->perm[i]] = yr[i];
    xi[S->perm[i]] = yi[i];
  }
  free(yr);
  free(yi);
}

/* ---- up-looking Cholesky (the reference's own test oracle): sparse.mjs:1379-1544 ------------------------------- */
typedef struct {
  int n;
  int *perm, *pinv, *Cp, *Ci, *srcIndex, *parent, *Lp, *Li, *mark, *s, *c;
  double *Lx, *x;
  int64_t nnzL;
} orc_up;

static int up_ereach(const orc_up *U, int k, int *mark, int *s, int stamp) { /* :1458-1473 */
  int top = U->n;
  mark[k] = stamp;
  for (int p = U->Cp[k]; p < U->Cp[k + 1]; p++) {
    int i = U->Ci[p];
    if (i > k) continue;
    int len = 0;
    for (; mark[i] != stamp; i = U->parent[i]) {
      s[len++] = i;
      mark[i] = stamp;
    }
    while (len > 0) s[--top] = s[--len];
  }
  return top;
}

ORC_API orc_up *orc_up_create(int n, const int *rowptr, const int *colidx, const int *perm) {
  orc_up *U = xcalloc(1, sizeof(orc_up)); /* :1384-1457 */
  U->n = n;
  U->perm = xmalloc(sizeof(int) * (n + 1));
  memcpy(U->perm, perm, sizeof(int) * n);
  U->pinv = xmalloc(sizeof(int) * (n + 1));
  for (int i = 0; i < n; i++) U->pinv[perm[i]] = i;
  int *cnt = xcalloc(n + 1, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) {
      int pi = U->pinv[i], pj = U->pinv[colidx[p]];
      if (pi <= pj) cnt[pj + 1]++;
    }
  for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
  U->Cp = cnt;
  int nnzC = cnt[n];
  U->Ci = xmalloc(sizeof(int) * (nnzC + 1));
  U->srcIndex = xmalloc(sizeof(int) * (nnzC + 1));
  int *next = xmalloc(sizeof(int) * (n + 1));
  memcpy(next, cnt, sizeof(int) * n);
  for (int i = 0; i < n; i++)
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) {
      int pi = U->pinv[i], pj = U->pinv[colidx[p]];
      if (pi <= pj) {
        int q = next[pj]++;
        U->Ci[q] = pi;
        U->srcIndex[q] = p;
      }
    }
  free(next);
  U->parent = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1);
  int *anc = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1);
  for (int k = 0; k < n; k++)
    for (int p = U->Cp[k]; p < U->Cp[k + 1]; p++) {
      int i = U->Ci[p];
      while (i != -1 && i < k) {
        int inext = anc[i];
        anc[i] = k;
        if (inext == -1) U->parent[i] = k;
        i = inext;
      }
    }
  free(anc);
  U->mark = xcalloc(n + 1, sizeof(int));
  U->s = xcalloc(n + 1, sizeof(int));
  int *colCount = xcalloc(n + 1, sizeof(int));
  for (int k = 0; k < n; k++) {
    int top = up_ereach(U, k, U->mark, U->s, k + 1);
    for (int q = top; q < n; q++) colCount[U->s[q]]++;
    colCount[k]++;
  }
  U->Lp = xcalloc(n + 1, sizeof(int));
  for (int k = 0; k < n; k++) U->Lp[k + 1] = U->Lp[k] + colCount[k];
  free(colCount);
  U->nnzL = U->Lp[n];
  U->Li = xmalloc(sizeof(int) * (U->nnzL + 1));
  U->Lx = xmalloc(sizeof(double) * (U->nnzL + 1));
  U->x = xcalloc(n + 1, sizeof(double));
  U->c = xcalloc(n + 1, sizeof(int));
  return U;
}
ORC_API const int *orc_up_Lp(const orc_up *U) { return U->Lp; }
ORC_API int64_t orc_up_nnzL(const orc_up *U) { return U->nnzL; }
ORC_API int orc_up_factor(orc_up *U, const double *values) { /* :1485-1521 */
  int n = U->n;
  int *mark = U->mark, *s = U->s, *c = U->c;
  double *x = U->x;
  memset(mark, 0, sizeof(int) * n);
  int stamp = 1;
  for (int k = 0; k < n; k++) c[k] = U->Lp[k];
  for (int k = 0; k < n; k++) {
    stamp++;
    int top = up_ereach(U, k, mark, s, stamp);
    for (int p = U->Cp[k]; p < U->Cp[k + 1]; p++) x[U->Ci[p]] = values[U->srcIndex[p]];
    double d = x[k];
    x[k] = 0;
    for (int q = top; q < n; q++) {
      int i = s[q];
      double lki = x[i] / U->Lx[U->Lp[i]];
      x[i] = 0;
      int ci = c[i];
      for (int p = U->Lp[i] + 1; p < ci; p++) x[U->Li[p]] -= U->Lx[p] * lki;
      d -= lki * lki;
      U->Li[ci] = k;
      U->Lx[ci] = lki;
      c[i] = ci + 1;
    }
    if (!(d > 0)) return 0;
    U->Li[c[k]] = k;
    U->Lx[c[k]] = sqrt(d);
    c[k]++;
  }
  return 1;
}
ORC_API void orc_up_solve(const orc_up *U, const double *b, double *out) { /* :1523-1543 */
  int n = U->n;
  double *y = xmalloc(sizeof(double) * (n + 1));
  for (int i = 0; i < n; i++) y[i] = b[U->perm[i]];
  for (int j = 0; j < n; j++) {
    y[j] /= U->Lx[U->Lp[j]];
    double yj = y[j];
    for (int p = U->Lp[j] + 1; p < U->Lp[j + 1]; p++) y[U->Li[p]] -= U->Lx[p] * yj;
  }
  for (int j = n - 1; j >= 0; j--) {
    double v = y[j];
    for (int p = U->Lp[j] + 1; p < U->Lp[j + 1]; p++) v -= U->Lx[p] * y[U->Li[p]];
    y[j] = v / U->Lx[U->Lp[j]];
  }
  for (int i = 0; i < n; i++) out[U->perm[i]] = y[i];
  free(y);
}
ORC_API void orc_up_free(orc_up *U) {
  if (!U) return;
  free(U->perm);
  free(U->pinv);
  free(U->Cp);
  free(U->Ci);
  free(U->srcIndex);
  free(U->parent);
  free(U->Lp);
  free(U->Li);
  free(U->Lx);
  free(U->mark);
  free(U->s);
  free(U->c);
  free(U->x);
  free(U);
}

/* ---- up-looking LDL^T (SymbolicLDLT + LDLT): ldlt.mjs:35-207 ---------------------------------------------------- */
/* Factor and one solve in one call (the tests need inertia and solutions). Returns ok; stats: nNeg, nPerturbed. */
ORC_API int orc_ldlt_up(int n, const int *rowptr, const int *colidx, const int *perm, const double *values,
                        double pivotTol, const double *b, double *x, int *stats) {
  int *pinv = xmalloc(sizeof(int) * (n + 1)); /* :41-66 */
  for (int i = 0; i < n; i++) pinv[perm[i]] = i;
  int *Cp = xcalloc(n + 1, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) {
      int pi = pinv[i], pj = pinv[colidx[p]];
      if (pi <= pj) Cp[pj + 1]++;
    }
  for (int i = 0; i < n; i++) Cp[i + 1] += Cp[i];
  int *Ci = xmalloc(sizeof(int) * (Cp[n] + 1)), *src = xmalloc(sizeof(int) * (Cp[n] + 1));
  int *next = xmalloc(sizeof(int) * (n + 1));
  memcpy(next, Cp, sizeof(int) * n);
  for (int i = 0; i < n; i++)
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) {
      int pi = pinv[i], pj = pinv[colidx[p]];
      if (pi <= pj) {
        int q = next[pj]++;
        Ci[q] = pi;
        src[q] = p;
      }
    }
  int *parent = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1), *anc = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1);
  for (int k = 0; k < n; k++) /* :68-79 */
    for (int p = Cp[k]; p < Cp[k + 1]; p++) {
      int i = Ci[p];
      while (i != -1 && i < k) {
        int inext = anc[i];
        anc[i] = k;
        if (inext == -1) parent[i] = k;
        i = inext;
      }
    }
  int *mark = ifill(xmalloc(sizeof(int) * (n + 1)), n, -1), *cnt = xcalloc(n + 1, sizeof(int)); /* :82-94 */
  for (int k = 0; k < n; k++) {
    mark[k] = k;
    for (int p = Cp[k]; p < Cp[k + 1]; p++) {
      int i = Ci[p];
      while (i < k && mark[i] != k) {
        cnt[i]++;
        mark[i] = k;
        i = parent[i];
      }
    }
  }
  int *Lp = xcalloc(n + 1, sizeof(int));
  for (int k = 0; k < n; k++) Lp[k + 1] = Lp[k] + cnt[k];
  int *Li = xmalloc(sizeof(int) * (Lp[n] + 1));
  double *Lx = xmalloc(sizeof(double) * (Lp[n] + 1)), *D = xmalloc(sizeof(double) * (n + 1)),
         *Y = xcalloc(n + 1, sizeof(double));
  int *flag = xcalloc(n + 1, sizeof(int)), *pattern = xcalloc(n + 1, sizeof(int)), *Lnz = xcalloc(n + 1, sizeof(int));
  double amax = 0; /* :133-138 */
  for (int k = 0; k < n; k++)
    for (int p = Cp[k]; p < Cp[k + 1]; p++)
      if (Ci[p] == k) {
        amax = js_max(amax, fabs(values[src[p]]));
      }
  double tau = pivotTol * (amax > 0 ? amax : 1);
  int nNeg = 0, nPert = 0, ok = 1;
  for (int k = 0; k < n && ok; k++) { /* :140-179 */
    Lnz[k] = 0;
    Y[k] = 0;
    int top = n;
    flag[k] = k;
    for (int p = Cp[k]; p < Cp[k + 1]; p++) {
      int i = Ci[p];
      Y[i] += values[src[p]];
      int len = 0;
      for (; flag[i] != k; i = parent[i]) {
        pattern[len++] = i;
        flag[i] = k;
      }
      while (len > 0) pattern[--top] = pattern[--len];
    }
    double d = Y[k];
    Y[k] = 0;
    for (; top < n; top++) {
      int i = pattern[top];
      double yi = Y[i];
      Y[i] = 0;
      int p2 = Lp[i] + Lnz[i];
      for (int p = Lp[i]; p < p2; p++) Y[Li[p]] -= Lx[p] * yi;
      double lki = yi / D[i];
      d -= lki * yi;
      Li[p2] = k;
      Lx[p2] = lki;
      Lnz[i]++;
    }
    if (!(fabs(d) >= tau)) {
      if (!isfinite(d)) {
        ok = 0;
        break;
      }
      d = d < 0 ? -tau : tau;
      nPert++;
    }
    if (d < 0) nNeg++;
    D[k] = d;
  }
  stats[0] = nNeg;
  stats[1] = nPert;
  if (ok && b && x) { /* :189-207 */
    double *y = Y;
    for (int i = 0; i < n; i++) y[i] = b[perm[i]];
    for (int j = 0; j < n; j++) {
      double yj = y[j];
      if (yj != 0)
        for (int p = Lp[j]; p < Lp[j + 1]; p++) y[Li[p]] -= Lx[p] * yj;
    }
    for (int j = 0; j < n; j++) y[j] /= D[j];
    for (int j = n - 1; j >= 0; j--) {
      double v = y[j];
      for (int p = Lp[j]; p < Lp[j + 1]; p++) v -= Lx[p] * y[Li[p]];
      y[j] = v;
    }
    for (int i = 0; i < n; i++) x[perm[i]] = y[i];
  }
  free(pinv);
  free(Cp);
  free(Ci);
  free(src);
  free(next);
  free(parent);
  free(anc);
  free(mark);
  free(cnt);
  free(Lp);
  free(Li);
  free(Lx);
  free(D);
  free(Y);
  free(flag);
  free(pattern);
  free(Lnz);
  return ok;
}
