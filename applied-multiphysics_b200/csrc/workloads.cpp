// Synthetic FEM workloads for the sparse direct solver: seeded, deterministic CSR systems (full symmetric storage,
// sorted rows, diagonal present) with DOF coordinates and right-hand sides, built the way the reference assembles its
// systems:
//   - patterns as packages/core/src/la/sparse.mjs buildPattern (:37-78), buildElementPattern (:86-110) and
//     blockPattern (:131-146); Dirichlet restriction as packages/core/src/fem/tri.mjs restrictMatrix (:192-225);
//   - P1 triangles as fem/tri.mjs triangleGeometry / assemble (:10-80), structured meshes as
//     packages/core/test/helpers/tri-grid.mjs (alternating diagonals) and tet-grid.mjs (6 Kuhn tets per hex);
//   - 3D P1 elasticity with D = dMatrix('3d', E, nu) (packages/physics/src/elastic/index.ts:50-58);
//   - lowest-order Nedelec (Whitney) edge elements after packages/core/src/fem/nedelec1.mjs.
// Random numbers: the reference tests' LCG s = s * 1664525 + 1013904223 (mod 2^32), U(0,1) = s / 2^32.
// These generators are the inputs of the tests and the benchmark; they are not part of the solve path.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#define WL_API extern "C" __attribute__((visibility("default")))

namespace {

struct Lcg {
  uint32_t s;
  explicit Lcg(uint32_t seed) : s(seed) {}
  double u01() {
    s = s * 1664525u + 1013904223u;
    return s / 4294967296.0;
  }
  double sym() { return 2.0 * u01() - 1.0; }  // U(-1, 1)
  int uniform_int(int lo, int hi) {          // U{lo..hi}
    int v = lo + (int)std::floor(u01() * (hi - lo + 1));
    return v > hi ? hi : v;
  }
  double normal() {  // Box-Muller on the LCG
    double u1 = u01(), u2 = u01();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  }
};

struct Csr {
  int n = 0;
  std::vector<int> rowptr, colidx;
};

// buildElementPattern (sparse.mjs:86-110): counting sort into rows, each row sorted ascending and unique.
Csr element_pattern(int n, const int *elem, int64_t ne, int k) {
  std::vector<int64_t> cap(n + 1, 0);
  for (int i = 0; i < n; i++) cap[i + 1] = 1;
  for (int64_t q = 0; q < ne * k; q++) cap[elem[q] + 1] += k - 1;
  for (int i = 0; i < n; i++) cap[i + 1] += cap[i];
  std::vector<int> buf(cap[n]);
  std::vector<int64_t> fill(cap.begin(), cap.begin() + n);
  for (int i = 0; i < n; i++) buf[fill[i]++] = i;
  for (int64_t e = 0; e < ne; e++)
    for (int a = 0; a < k; a++) {
      int r = elem[k * e + a];
      for (int b = 0; b < k; b++)
        if (b != a) buf[fill[r]++] = elem[k * e + b];
    }
  Csr P;
  P.n = n;
  P.rowptr.assign(n + 1, 0);
  int64_t nnz = 0;
  for (int i = 0; i < n; i++) {
    int64_t p0 = cap[i], p1 = cap[i + 1];
    std::sort(buf.begin() + p0, buf.begin() + p1);
    for (int64_t p = p0; p < p1; p++)
      if (p == p0 || buf[p] != buf[p - 1]) buf[nnz++] = buf[p];
    P.rowptr[i + 1] = (int)nnz;
  }
  buf.resize(nnz);
  P.colidx = std::move(buf);
  return P;
}

// blockPattern (sparse.mjs:131-146): DOF = node * bs + component.
Csr block_pattern(const Csr &p, int bs) {
  Csr B;
  B.n = p.n * bs;
  B.rowptr.assign(B.n + 1, 0);
  for (int i = 0; i < p.n; i++) {
    int len = (p.rowptr[i + 1] - p.rowptr[i]) * bs;
    for (int c = 0; c < bs; c++) B.rowptr[i * bs + c + 1] = len;
  }
  for (int i = 0; i < B.n; i++) B.rowptr[i + 1] += B.rowptr[i];
  B.colidx.resize(B.rowptr[B.n]);
  for (int i = 0; i < p.n; i++)
    for (int c = 0; c < bs; c++) {
      int z = B.rowptr[i * bs + c];
      for (int q = p.rowptr[i]; q < p.rowptr[i + 1]; q++)
        for (int d = 0; d < bs; d++) B.colidx[z++] = p.colidx[q] * bs + d;
    }
  return B;
}

// entryIndex (sparse.mjs:206-217): binary search in a sorted row.
inline int entry_index(const Csr &P, int i, int j) {
  int lo = P.rowptr[i], hi = P.rowptr[i + 1] - 1;
  while (lo <= hi) {
    int m = (lo + hi) >> 1;
    int c = P.colidx[m];
    if (c == j) return m;
    if (c < j)
      lo = m + 1;
    else
      hi = m - 1;
  }
  return -1;
}

}  // namespace

struct amp_workload {
  int n;
  int64_t nnz;
  int *rowptr, *colidx;
  double *values;
  double *x, *y, *z;  // DOF coordinates (z null in 2D)
  int nrhs;
  double *rhs;  // rhs[k * n + i]
};

namespace {

template <class T>
T *dup(const std::vector<T> &v) {
  T *p = (T *)std::malloc(sizeof(T) * (v.size() ? v.size() : 1));
  if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

// restrictMatrix (fem/tri.mjs:192-225) of a full pattern + values to the free DOFs; returns the workload with
// coordinates mapped and the map old -> new (-1 fixed).
amp_workload *restrict_to(const Csr &P, const std::vector<double> &val, const std::vector<char> &isFree,
                          const std::vector<double> *X, const std::vector<double> *Y, const std::vector<double> *Z,
                          std::vector<int> &map) {
  int n = P.n;
  map.assign(n, -1);
  int nf = 0;
  for (int i = 0; i < n; i++)
    if (isFree[i]) map[i] = nf++;
  std::vector<int> rowptr(nf + 1, 0);
  int64_t nnz = 0;
  for (int i = 0; i < n; i++) {
    if (map[i] < 0) continue;
    for (int p = P.rowptr[i]; p < P.rowptr[i + 1]; p++)
      if (map[P.colidx[p]] >= 0) nnz++;
    rowptr[map[i] + 1] = (int)nnz;
  }
  std::vector<int> colidx(nnz);
  std::vector<double> v(nnz);
  int64_t q = 0;
  for (int i = 0; i < n; i++) {
    if (map[i] < 0) continue;
    for (int p = P.rowptr[i]; p < P.rowptr[i + 1]; p++) {
      int c = map[P.colidx[p]];
      if (c >= 0) {
        colidx[q] = c;
        v[q] = val[p];
        q++;
      }
    }
  }
  amp_workload *W = (amp_workload *)std::calloc(1, sizeof(amp_workload));
  W->n = nf;
  W->nnz = nnz;
  W->rowptr = dup(rowptr);
  W->colidx = dup(colidx);
  W->values = dup(v);
  auto mapc = [&](const std::vector<double> *C) -> double * {
    if (!C) return nullptr;
    std::vector<double> o(nf);
    for (int i = 0; i < n; i++)
      if (map[i] >= 0) o[map[i]] = (*C)[i];
    return dup(o);
  };
  W->x = mapc(X);
  W->y = mapc(Y);
  W->z = mapc(Z);
  return W;
}

// Structured triangle grid on [0,1]^2 with N cells per side, alternating diagonals (tri-grid.mjs:30-49).
void tri_grid(int N, std::vector<double> &x, std::vector<double> &y, std::vector<int> &tri) {
  int nx = N + 1, ny = N + 1;
  x.resize(nx * ny);
  y.resize(nx * ny);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      x[i + nx * j] = (double)i / N;
      y[i + nx * j] = (double)j / N;
    }
  tri.clear();
  for (int j = 0; j + 1 < ny; j++)
    for (int i = 0; i + 1 < nx; i++) {
      int n00 = i + nx * j, n10 = n00 + 1, n01 = n00 + nx, n11 = n01 + 1;
      if ((i + j) % 2 == 0) {
        int t[6] = {n00, n10, n11, n00, n11, n01};
        tri.insert(tri.end(), t, t + 6);
      } else {
        int t[6] = {n00, n10, n01, n10, n11, n01};
        tri.insert(tri.end(), t, t + 6);
      }
    }
}

// P1 scalar stiffness sum_T A_T gradN^T (k_T I) gradN (fem/tri.mjs triangleGeometry + assemble with cxx = cyy = k).
// Also the load vector of f = 1 (A / 3 per vertex).
void p1_assemble(const Csr &P, const std::vector<double> &x, const std::vector<double> &y, const std::vector<int> &tri,
                 const std::vector<double> &kTri, std::vector<double> &val, std::vector<double> &load) {
  int64_t nt = (int64_t)tri.size() / 3;
  val.assign(P.colidx.size(), 0.0);
  load.assign(P.n, 0.0);
  for (int64_t t = 0; t < nt; t++) {
    int i = tri[3 * t], j = tri[3 * t + 1], k = tri[3 * t + 2];
    double x1 = x[i], y1 = y[i], x2 = x[j], y2 = y[j], x3 = x[k], y3 = y[k];
    double a2 = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
    double A = 0.5 * a2;
    double gx[3] = {(y2 - y3) / a2, (y3 - y1) / a2, (y1 - y2) / a2};
    double gy[3] = {(x3 - x2) / a2, (x1 - x3) / a2, (x2 - x1) / a2};
    double kk = kTri.empty() ? 1.0 : kTri[t];
    int v[3] = {i, j, k};
    for (int a = 0; a < 3; a++) {
      for (int b = 0; b < 3; b++) {
        double s = A * (gx[a] * (kk * gx[b]) + gy[a] * (kk * gy[b]));
        if (s != 0) val[entry_index(P, v[a], v[b])] += s;
      }
      load[v[a]] += A / 3.0;
    }
  }
}

amp_workload *heat2d(int N, const std::vector<double> &kTri, std::vector<double> &loadOut) {
  std::vector<double> x, y, val, load;
  std::vector<int> tri;
  tri_grid(N, x, y, tri);
  int nn = (N + 1) * (N + 1);
  Csr P = element_pattern(nn, tri.data(), (int64_t)tri.size() / 3, 3);
  p1_assemble(P, x, y, tri, kTri, val, load);
  std::vector<char> isFree(nn, 0);
  for (int j = 1; j < N; j++)
    for (int i = 1; i < N; i++) isFree[i + (N + 1) * j] = 1;
  std::vector<int> map;
  amp_workload *W = restrict_to(P, val, isFree, &x, &y, nullptr, map);
  loadOut.assign(W->n, 0.0);
  for (int i = 0; i < nn; i++)
    if (map[i] >= 0) loadOut[map[i]] = load[i];
  return W;
}

// 6 Kuhn tets per hex along monotone index paths (test/helpers/tet-grid.mjs:9-46), node id i + NX (j + NY k).
void kuhn_tets(int nx, int ny, int nz, std::vector<int> &tets) {
  static const int PERMS[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int NX = nx + 1, NY = ny + 1;
  auto id = [&](int i, int j, int k) { return i + NX * (j + NY * k); };
  tets.clear();
  tets.reserve((size_t)nx * ny * nz * 24);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (auto &p : PERMS) {
          int c[3] = {i, j, k};
          tets.push_back(id(c[0], c[1], c[2]));
          for (int ax : p) {
            c[ax]++;
            tets.push_back(id(c[0], c[1], c[2]));
          }
        }
}

// Gradients of the barycentric coordinates of a tet and its volume.
double tet_grads(const double *P0, const double *P1, const double *P2, const double *P3, double g[4][3]) {
  double a[3] = {P1[0] - P0[0], P1[1] - P0[1], P1[2] - P0[2]};
  double b[3] = {P2[0] - P0[0], P2[1] - P0[1], P2[2] - P0[2]};
  double c[3] = {P3[0] - P0[0], P3[1] - P0[1], P3[2] - P0[2]};
  double det = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
  // rows of the inverse of [a b c]^T give grad lambda_1..3
  double inv[3][3];
  inv[0][0] = (b[1] * c[2] - b[2] * c[1]) / det;
  inv[0][1] = (b[2] * c[0] - b[0] * c[2]) / det;
  inv[0][2] = (b[0] * c[1] - b[1] * c[0]) / det;
  inv[1][0] = (c[1] * a[2] - c[2] * a[1]) / det;
  inv[1][1] = (c[2] * a[0] - c[0] * a[2]) / det;
  inv[1][2] = (c[0] * a[1] - c[1] * a[0]) / det;
  inv[2][0] = (a[1] * b[2] - a[2] * b[1]) / det;
  inv[2][1] = (a[2] * b[0] - a[0] * b[2]) / det;
  inv[2][2] = (a[0] * b[1] - a[1] * b[0]) / det;
  for (int d = 0; d < 3; d++) {
    g[1][d] = inv[0][d];
    g[2][d] = inv[1][d];
    g[3][d] = inv[2][d];
    g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
  }
  return std::fabs(det) / 6.0;
}

}  // namespace

extern "C" {

WL_API void amp_wl_free(amp_workload *W) {
  if (!W) return;
  std::free(W->rowptr);
  std::free(W->colidx);
  std::free(W->values);
  std::free(W->x);
  std::free(W->y);
  std::free(W->z);
  std::free(W->rhs);
  std::free(W);
}

// 2D Poisson, P1 triangles on the unit square with N x N cells (2 triangles each, alternating diagonals), homogeneous
// Dirichlet boundary. RHS 0: load of f = 1; RHS 1: seeded U(-1, 1).
WL_API amp_workload *amp_wl_poisson2d(int N, uint32_t seed) {
  std::vector<double> load;
  amp_workload *W = heat2d(N, {}, load);
  Lcg r(seed);
  W->nrhs = 2;
  W->rhs = (double *)std::malloc(sizeof(double) * 2 * W->n);
  for (int i = 0; i < W->n; i++) W->rhs[i] = load[i];
  for (int i = 0; i < W->n; i++) W->rhs[W->n + i] = r.sym();
  return W;
}

// One member of the batched 2D heat set: N x N cells on the unit square, per-triangle conductivity lognormal(0, 1),
// Dirichlet on the whole boundary, q seeded U(-1, 1) right-hand sides.
WL_API amp_workload *amp_wl_heat2d_lognormal(int N, uint32_t seed, int q) {
  Lcg r(seed);
  std::vector<double> kTri(2 * (size_t)N * N);
  for (auto &k : kTri) k = std::exp(r.normal());
  std::vector<double> load;
  amp_workload *W = heat2d(N, kTri, load);
  W->nrhs = q;
  W->rhs = (double *)std::malloc(sizeof(double) * (size_t)q * W->n + 8);
  for (int64_t i = 0; i < (int64_t)q * W->n; i++) W->rhs[i] = r.sym();
  return W;
}

// 3D linear elasticity, P1 tets: N^3 unit cube, 6 Kuhn tets per hex, E, nu; the x = 0 face clamped; seeded U(-1, 1)
// body load per DOF (q vectors). DOF = node * 3 + component; DOF coordinates = node coordinates.
WL_API amp_workload *amp_wl_elastic3d(int N, double E, double nu, uint32_t seed, int q) {
  int NX = N + 1, nn = NX * NX * NX;
  std::vector<int> tets;
  kuhn_tets(N, N, N, tets);
  int64_t ne = (int64_t)tets.size() / 4;
  std::vector<double> X(nn), Y(nn), Z(nn);
  for (int k = 0; k < NX; k++)
    for (int j = 0; j < NX; j++)
      for (int i = 0; i < NX; i++) {
        int v = i + NX * (j + NX * k);
        X[v] = (double)i / N;
        Y[v] = (double)j / N;
        Z[v] = (double)k / N;
      }
  Csr node = element_pattern(nn, tets.data(), ne, 4);
  Csr P = block_pattern(node, 3);
  // dMatrix('3d', E, nu): Voigt [xx, yy, zz, yz, xz, xy]
  double lam = (E * nu) / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  double D[6][6] = {};
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) D[i][j] = lam;
    D[i][i] = lam + 2 * mu;
    D[i + 3][i + 3] = mu;
  }
  std::vector<double> val(P.colidx.size(), 0.0);
  for (int64_t e = 0; e < ne; e++) {
    const int *t = &tets[4 * e];
    double p[4][3];
    for (int a = 0; a < 4; a++) {
      p[a][0] = X[t[a]];
      p[a][1] = Y[t[a]];
      p[a][2] = Z[t[a]];
    }
    double g[4][3];
    double V = tet_grads(p[0], p[1], p[2], p[3], g);
    double B[6][12] = {};
    for (int a = 0; a < 4; a++) {
      double gx = g[a][0], gy = g[a][1], gz = g[a][2];
      B[0][3 * a] = gx;
      B[1][3 * a + 1] = gy;
      B[2][3 * a + 2] = gz;
      B[3][3 * a + 1] = gz;
      B[3][3 * a + 2] = gy;
      B[4][3 * a] = gz;
      B[4][3 * a + 2] = gx;
      B[5][3 * a] = gy;
      B[5][3 * a + 1] = gx;
    }
    double DB[6][12];
    for (int i = 0; i < 6; i++)
      for (int c = 0; c < 12; c++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += D[i][k] * B[k][c];
        DB[i][c] = s;
      }
    double Ke[12][12];  // exactly symmetric: upper triangle computed, lower mirrored
    for (int r = 0; r < 12; r++)
      for (int c = r; c < 12; c++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += B[k][r] * DB[k][c];
        Ke[r][c] = Ke[c][r] = V * s;
      }
    for (int r = 0; r < 12; r++) {
      int row = 3 * t[r / 3] + r % 3;
      for (int c = 0; c < 12; c++) val[entry_index(P, row, 3 * t[c / 3] + c % 3)] += Ke[r][c];
    }
  }
  int n = P.n;
  std::vector<char> isFree(n, 1);
  std::vector<double> Xd(n), Yd(n), Zd(n);
  for (int v = 0; v < nn; v++)
    for (int c = 0; c < 3; c++) {
      Xd[3 * v + c] = X[v];
      Yd[3 * v + c] = Y[v];
      Zd[3 * v + c] = Z[v];
      if (v % NX == 0) isFree[3 * v + c] = 0;
    }
  std::vector<int> map;
  amp_workload *W = restrict_to(P, val, isFree, &Xd, &Yd, &Zd, map);
  Lcg r(seed);
  W->nrhs = q;
  W->rhs = (double *)std::malloc(sizeof(double) * (size_t)q * W->n + 8);
  for (int64_t i = 0; i < (int64_t)q * W->n; i++) W->rhs[i] = r.sym();
  return W;
}

// 3D heat, P2 (tet10) Lagrange on an N^3 cube with 6 Kuhn tets per hex. The P2 DOFs are the points of the doubled
// (2N+1)^3 grid (vertices and edge midpoints). Conductivity 100 inside nsph seeded spheres of the given radius
// (centres U(0,1)^3, element centroid test), else 1. Dirichlet on x = 0 and x = 1. q seeded U(-1,1) RHS.
WL_API amp_workload *amp_wl_heat3d_p2(int N, int nsph, double radius, uint32_t seed, int q) {
  int M = 2 * N + 1;  // doubled grid points per side
  int64_t nd = (int64_t)M * M * M;
  std::vector<int> tets;
  kuhn_tets(N, N, N, tets);
  int64_t ne = (int64_t)tets.size() / 4;
  int NX = N + 1;
  auto vcoord = [&](int v, int c) {
    int i = v % NX, j = (v / NX) % NX, k = v / (NX * NX);
    return c == 0 ? i : (c == 1 ? j : k);
  };
  auto dof = [&](int I, int J, int K) { return I + M * (J + M * K); };
  static const int EP[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  std::vector<int> elem(10 * ne);
  for (int64_t e = 0; e < ne; e++) {
    const int *t = &tets[4 * e];
    for (int a = 0; a < 4; a++) elem[10 * e + a] = dof(2 * vcoord(t[a], 0), 2 * vcoord(t[a], 1), 2 * vcoord(t[a], 2));
    for (int l = 0; l < 6; l++) {
      int a = t[EP[l][0]], b = t[EP[l][1]];
      elem[10 * e + 4 + l] = dof(vcoord(a, 0) + vcoord(b, 0), vcoord(a, 1) + vcoord(b, 1), vcoord(a, 2) + vcoord(b, 2));
    }
  }
  Csr P = element_pattern((int)nd, elem.data(), ne, 10);
  Lcg r(seed);
  std::vector<double> cx(nsph), cy(nsph), cz(nsph);
  for (int s = 0; s < nsph; s++) {
    cx[s] = r.u01();
    cy[s] = r.u01();
    cz[s] = r.u01();
  }
  // 4-point degree-2 rule on the reference tet
  const double qa = 0.5854101966249685, qb = 0.1381966011250105;
  double lq[4][4];
  for (int qp = 0; qp < 4; qp++)
    for (int i = 0; i < 4; i++) lq[qp][i] = (i == qp) ? qa : qb;
  std::vector<double> val(P.colidx.size(), 0.0);
  for (int64_t e = 0; e < ne; e++) {
    const int *t = &tets[4 * e];
    double p[4][3];
    for (int a = 0; a < 4; a++)
      for (int c = 0; c < 3; c++) p[a][c] = (double)vcoord(t[a], c) / N;
    double g[4][3];
    double V = tet_grads(p[0], p[1], p[2], p[3], g);
    double ctr[3] = {0, 0, 0};
    for (int a = 0; a < 4; a++)
      for (int c = 0; c < 3; c++) ctr[c] += 0.25 * p[a][c];
    double kk = 1.0;
    for (int s = 0; s < nsph; s++) {
      double dx = ctr[0] - cx[s], dy = ctr[1] - cy[s], dz = ctr[2] - cz[s];
      if (dx * dx + dy * dy + dz * dz <= radius * radius) {
        kk = 100.0;
        break;
      }
    }
    double K[10][10] = {};
    for (int qp = 0; qp < 4; qp++) {
      const double *L = lq[qp];
      double G[10][3];
      for (int i = 0; i < 4; i++)
        for (int d = 0; d < 3; d++) G[i][d] = (4 * L[i] - 1) * g[i][d];
      for (int l = 0; l < 6; l++) {
        int i = EP[l][0], j = EP[l][1];
        for (int d = 0; d < 3; d++) G[4 + l][d] = 4 * (L[i] * g[j][d] + L[j] * g[i][d]);
      }
      for (int a = 0; a < 10; a++)
        for (int b = 0; b < 10; b++) K[a][b] += 0.25 * (G[a][0] * G[b][0] + G[a][1] * G[b][1] + G[a][2] * G[b][2]);
    }
    for (int a = 0; a < 10; a++)
      for (int b = 0; b < 10; b++) val[entry_index(P, elem[10 * e + a], elem[10 * e + b])] += kk * V * K[a][b];
  }
  std::vector<char> isFree(nd, 1);
  std::vector<double> X(nd), Y(nd), Z(nd);
  for (int K = 0; K < M; K++)
    for (int J = 0; J < M; J++)
      for (int I = 0; I < M; I++) {
        int v = dof(I, J, K);
        X[v] = 0.5 * I / N;
        Y[v] = 0.5 * J / N;
        Z[v] = 0.5 * K / N;
        if (I == 0 || I == M - 1) isFree[v] = 0;
      }
  std::vector<int> map;
  amp_workload *W = restrict_to(P, val, isFree, &X, &Y, &Z, map);
  W->nrhs = q;
  W->rhs = (double *)std::malloc(sizeof(double) * (size_t)q * W->n + 8);
  for (int64_t i = 0; i < (int64_t)q * W->n; i++) W->rhs[i] = r.sym();
  return W;
}

// 3D driven Maxwell, lowest-order Nedelec (Whitney) edges on an N^3 cube with 6 Kuhn tets per hex:
// A = K - k2 M with K_ab = V curl W_a . curl W_b (nu = 1) and M_ab = eps_r int W_a . W_b. eps_r = eps_in inside
// nbox seeded axis-aligned boxes (edge lengths U(0.1, 0.3)), else 1. PEC: edges whose midpoint lies on the cube
// surface are removed. Edge orientation low -> high node id (tet vertices ascending, local pairs 01 02 03 12 13 23).
// DOF coordinates = edge midpoints. RHS: q port-like currents, each a seeded U(-1,1) amplitude on the free edges of
// the layer 0 < x <= 1/N (next to the x = 0 face), zero elsewhere.
WL_API amp_workload *amp_wl_maxwell3d(int N, int nbox, double eps_in, double k2, uint32_t seed, int q) {
  int NX = N + 1, nn = NX * NX * NX;
  std::vector<int> tets;
  kuhn_tets(N, N, N, tets);
  int64_t ne = (int64_t)tets.size() / 4;
  auto vc = [&](int v, int c) {
    int i = v % NX, j = (v / NX) % NX, k = v / (NX * NX);
    return c == 0 ? i : (c == 1 ? j : k);
  };
  static const int EP[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  // edge ids: direction d in 7 monotone 0/1 offsets, id = d * nn + low node (sparse ids, compacted below)
  static const int DIRS[7][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  auto dir_of = [&](int a, int b) {
    int d[3] = {vc(b, 0) - vc(a, 0), vc(b, 1) - vc(a, 1), vc(b, 2) - vc(a, 2)};
    for (int q2 = 0; q2 < 7; q2++)
      if (DIRS[q2][0] == d[0] && DIRS[q2][1] == d[1] && DIRS[q2][2] == d[2]) return q2;
    return -1;
  };
  std::vector<int> eid((size_t)7 * nn, -1);
  std::vector<int> tetEdges(6 * ne);
  int nE = 0;
  std::vector<int> ea, eb;
  for (int64_t e = 0; e < ne; e++)
    for (int l = 0; l < 6; l++) {
      int a = tets[4 * e + EP[l][0]], b = tets[4 * e + EP[l][1]];
      size_t key = (size_t)dir_of(a, b) * nn + a;
      if (eid[key] < 0) {
        eid[key] = nE++;
        ea.push_back(a);
        eb.push_back(b);
      }
      tetEdges[6 * e + l] = eid[key];
    }
  Csr P = element_pattern(nE, tetEdges.data(), ne, 6);
  Lcg r(seed);
  std::vector<double> bx0(nbox), bx1(nbox), by0(nbox), by1(nbox), bz0(nbox), bz1(nbox);
  for (int s = 0; s < nbox; s++) {
    double c[3], h[3];
    for (int d = 0; d < 3; d++) c[d] = r.u01();
    for (int d = 0; d < 3; d++) h[d] = 0.05 + 0.1 * r.u01();
    bx0[s] = c[0] - h[0];
    bx1[s] = c[0] + h[0];
    by0[s] = c[1] - h[1];
    by1[s] = c[1] + h[1];
    bz0[s] = c[2] - h[2];
    bz1[s] = c[2] + h[2];
  }
  std::vector<double> val(P.colidx.size(), 0.0);
  for (int64_t e = 0; e < ne; e++) {
    const int *t = &tets[4 * e];
    double p[4][3];
    for (int a = 0; a < 4; a++)
      for (int c = 0; c < 3; c++) p[a][c] = (double)vc(t[a], c) / N;
    double g[4][3];
    double V = tet_grads(p[0], p[1], p[2], p[3], g);
    double ctr[3] = {0, 0, 0};
    for (int a = 0; a < 4; a++)
      for (int c = 0; c < 3; c++) ctr[c] += 0.25 * p[a][c];
    double eps = 1.0;
    for (int s = 0; s < nbox; s++)
      if (ctr[0] >= bx0[s] && ctr[0] <= bx1[s] && ctr[1] >= by0[s] && ctr[1] <= by1[s] && ctr[2] >= bz0[s] &&
          ctr[2] <= bz1[s]) {
        eps = eps_in;
        break;
      }
    double curl[6][3];
    for (int l = 0; l < 6; l++) {
      const double *gi = g[EP[l][0]], *gj = g[EP[l][1]];
      curl[l][0] = 2 * (gi[1] * gj[2] - gi[2] * gj[1]);
      curl[l][1] = 2 * (gi[2] * gj[0] - gi[0] * gj[2]);
      curl[l][2] = 2 * (gi[0] * gj[1] - gi[1] * gj[0]);
    }
    auto dg = [&](int i, int j) { return g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2]; };
    auto mll = [&](int i, int j) { return V * (i == j ? 2.0 : 1.0) / 20.0; };  // int lambda_i lambda_j
    for (int a = 0; a < 6; a++)
      for (int b = 0; b < 6; b++) {
        int i = EP[a][0], j = EP[a][1], k = EP[b][0], l = EP[b][1];
        double Kab = V * (curl[a][0] * curl[b][0] + curl[a][1] * curl[b][1] + curl[a][2] * curl[b][2]);
        // int (l_i g_j - l_j g_i) . (l_k g_l - l_l g_k)
        double Mab = mll(i, k) * dg(j, l) - mll(i, l) * dg(j, k) - mll(j, k) * dg(i, l) + mll(j, l) * dg(i, k);
        val[entry_index(P, tetEdges[6 * e + a], tetEdges[6 * e + b])] += Kab - k2 * eps * Mab;
      }
  }
  std::vector<char> isFree(nE, 1);
  std::vector<double> X(nE), Y(nE), Z(nE);
  for (int e = 0; e < nE; e++) {
    int sx = vc(ea[e], 0) + vc(eb[e], 0), sy = vc(ea[e], 1) + vc(eb[e], 1), sz = vc(ea[e], 2) + vc(eb[e], 2);
    X[e] = 0.5 * sx / N;
    Y[e] = 0.5 * sy / N;
    Z[e] = 0.5 * sz / N;
    if (sx == 0 || sx == 2 * N || sy == 0 || sy == 2 * N || sz == 0 || sz == 2 * N) isFree[e] = 0;
  }
  std::vector<int> map;
  amp_workload *W = restrict_to(P, val, isFree, &X, &Y, &Z, map);
  W->nrhs = q;
  W->rhs = (double *)std::calloc((size_t)q * W->n + 1, sizeof(double));
  for (int k = 0; k < q; k++)
    for (int i = 0; i < W->n; i++)
      if (W->x[i] <= 1.0 / N + 1e-12) W->rhs[(size_t)k * W->n + i] = r.sym();
  return W;
}

// Fixtures of the reference's own tests.
// grid(): 27-point pattern on an Nx x Ny x Nz node grid (la-real-front.test.mjs:15-31 with sym = 0,
// la-real-solve.test.mjs:15-31 with sym = 1), diagonal 26.5 + 0.01 (r % 7) - shift.
WL_API amp_workload *amp_wl_grid27(int Nx, int Ny, int Nz, int zeroEvery, double shift, int sym) {
  int n = Nx * Ny * Nz;
  std::vector<int> el;
  auto id = [&](int i, int j, int k) { return i + Nx * (j + Ny * k); };
  static const int O[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  for (int k = 0; k + 1 < Nz; k++)
    for (int j = 0; j + 1 < Ny; j++)
      for (int i = 0; i + 1 < Nx; i++)
        for (auto &o : O) el.push_back(id(i + o[0], j + o[1], k + o[2]));
  Csr P = element_pattern(n, el.data(), (int64_t)el.size() / 8, 8);
  amp_workload *W = (amp_workload *)std::calloc(1, sizeof(amp_workload));
  W->n = n;
  W->nnz = (int64_t)P.colidx.size();
  W->rowptr = dup(P.rowptr);
  W->colidx = dup(P.colidx);
  std::vector<double> v(P.colidx.size());
  for (int r = 0; r < n; r++)
    for (int p = P.rowptr[r]; p < P.rowptr[r + 1]; p++) {
      int c = P.colidx[p];
      if (c == r)
        v[p] = 26.5 + 0.01 * (r % 7) - shift;
      else if (zeroEvery && (r + c) % zeroEvery == 0)
        v[p] = 0;
      else {
        int hsh = sym ? ((std::min(r, c) * 31 + std::max(r, c) * 17) % 11) : ((r * 31 + c * 17) % 11);
        v[p] = -1 + 0.001 * hsh;
      }
    }
  W->values = dup(v);
  return W;
}

// hexMatrix (la-sparse.test.mjs:13-63): graded Q1 hex Laplacian, anisotropic k, x = 0 face fixed; x, y = the test's
// node coordinates (y = ys[j] + 0.37 zs[k]).
WL_API amp_workload *amp_wl_hex_q1(int nx, int ny, int nz) {
  std::vector<double> xs(nx + 1), ys(ny + 1), zs(nz + 1);
  for (int i = 0; i <= nx; i++) xs[i] = std::pow((double)i / nx, 1.3);
  for (int j = 0; j <= ny; j++) ys[j] = (double)j / ny;
  for (int k = 0; k <= nz; k++) zs[k] = 0.2 * std::pow((double)k / nz, 0.8);
  auto Nn = [&](int i, int j, int k) { return i + (nx + 1) * (j + (ny + 1) * k); };
  int n = (nx + 1) * (ny + 1) * (nz + 1);
  int ne = nx * ny * nz;
  std::vector<int> elem(8 * ne);
  std::vector<double> Ke(64 * (size_t)ne);
  const double S[2][2] = {{1, -1}, {-1, 1}}, Mm[2][2] = {{2, 1}, {1, 2}};
  int e = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++, e++) {
        double hx = xs[i + 1] - xs[i], hy = ys[j + 1] - ys[j], hz = zs[k + 1] - zs[k];
        double kx = 1 + (i % 2), ky = 0.5, kz = 3 + (k % 3);
        for (int a = 0; a < 8; a++)
          for (int b = 0; b < 8; b++) {
            int ia = a & 1, ja = (a >> 1) & 1, ka = a >> 2, ib = b & 1, jb = (b >> 1) & 1, kb = b >> 2;
            Ke[64 * e + 8 * a + b] = kx * (S[ia][ib] / hx) * (Mm[ja][jb] * hy / 6) * (Mm[ka][kb] * hz / 6) +
                                     ky * (Mm[ia][ib] * hx / 6) * (S[ja][jb] / hy) * (Mm[ka][kb] * hz / 6) +
                                     kz * (Mm[ia][ib] * hx / 6) * (Mm[ja][jb] * hy / 6) * (S[ka][kb] / hz);
          }
        for (int a = 0; a < 8; a++) elem[8 * e + a] = Nn(i + (a & 1), j + ((a >> 1) & 1), k + (a >> 2));
      }
  Csr full = element_pattern(n, elem.data(), ne, 8);
  std::vector<double> vals(full.colidx.size(), 0.0);
  for (int qq = 0; qq < ne; qq++)
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) vals[entry_index(full, elem[8 * qq + a], elem[8 * qq + b])] += Ke[64 * qq + 8 * a + b];
  std::vector<char> isFree(n, 0);
  std::vector<double> X(n), Y(n);
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        int v = Nn(i, j, k);
        X[v] = xs[i];
        Y[v] = ys[j] + 0.37 * zs[k];
        if (i > 0) isFree[v] = 1;
      }
  std::vector<int> map;
  return restrict_to(full, vals, isFree, &X, &Y, nullptr, map);
}

// chain (core-solvers.test.mjs:20-27): 1D pattern, tridiag(off, diag, off).
WL_API amp_workload *amp_wl_chain(int n, double diag, double off) {
  std::vector<int> el(2 * (size_t)(n - 1));
  for (int i = 0; i + 1 < n; i++) {
    el[2 * i] = i;
    el[2 * i + 1] = i + 1;
  }
  Csr P = element_pattern(n, el.data(), n - 1, 2);
  amp_workload *W = (amp_workload *)std::calloc(1, sizeof(amp_workload));
  W->n = n;
  W->nnz = (int64_t)P.colidx.size();
  W->rowptr = dup(P.rowptr);
  W->colidx = dup(P.colidx);
  std::vector<double> v(P.colidx.size());
  for (int r = 0; r < n; r++)
    for (int p = P.rowptr[r]; p < P.rowptr[r + 1]; p++) v[p] = P.colidx[p] == r ? diag : off;
  W->values = dup(v);
  return W;
}

// The mesh behind a workload, for on-device assembly (the inputs of assembleCells, physics/src/common/scalar.ts:96-146):
// node coordinates (dim per node), element connectivity (k nodes per element), the DOF map (system row of node v's
// component c at dofs[v bs + c], -1 for a Dirichlet DOF; the map of restrict_to) and the per-element coefficients.
//   kind 0: heat2d_lognormal(N, seed) P1 triangles, bs 1, coef = conductivity per triangle (seed 0: all 1, the
//           Poisson system);
//   kind 1: elastic3d(N, E, nu) P1 tets, bs 3, x = 0 clamped, coef = (E, nu) per tet.
// Outputs are malloc'd (free with amp_wl_free_array).
WL_API int amp_wl_mesh(int kind, int N, uint32_t seed, double E, double nu, int *nnodes, int *dim, double **coords,
                       int64_t *nelem, int *k, int **conn, int *bs, int **dofs, double **coef, int *ncoef) {
  std::vector<double> X, Y, Z;
  std::vector<int> elem;
  std::vector<char> isFree;
  std::vector<double> cf;
  int B = 1, D = 2, K = 3, nn = 0;
  if (kind == 0) {
    tri_grid(N, X, Y, elem);
    nn = (N + 1) * (N + 1);
    isFree.assign(nn, 0);
    for (int j = 1; j < N; j++)
      for (int i = 1; i < N; i++) isFree[i + (N + 1) * j] = 1;
    cf.assign(elem.size() / 3, 1.0);
    if (seed) {
      Lcg r(seed);
      for (auto &c : cf) c = std::exp(r.normal());
    }
  } else if (kind == 1) {
    const int NX = N + 1;
    nn = NX * NX * NX;
    kuhn_tets(N, N, N, elem);
    X.resize(nn);
    Y.resize(nn);
    Z.resize(nn);
    for (int kk = 0; kk < NX; kk++)
      for (int j = 0; j < NX; j++)
        for (int i = 0; i < NX; i++) {
          const int v = i + NX * (j + NX * kk);
          X[v] = (double)i / N;
          Y[v] = (double)j / N;
          Z[v] = (double)kk / N;
        }
    B = 3;
    D = 3;
    K = 4;
    isFree.assign((size_t)nn * 3, 1);
    for (int v = 0; v < nn; v++)
      if (v % NX == 0) isFree[3 * v] = isFree[3 * v + 1] = isFree[3 * v + 2] = 0;
    for (size_t e = 0; e < elem.size() / 4; e++) {
      cf.push_back(E);
      cf.push_back(nu);
    }
  } else {
    return 1;
  }
  std::vector<double> xyz((size_t)nn * D);
  for (int v = 0; v < nn; v++) {
    xyz[(size_t)D * v] = X[v];
    xyz[(size_t)D * v + 1] = Y[v];
    if (D == 3) xyz[(size_t)D * v + 2] = Z[v];
  }
  std::vector<int> map(isFree.size(), -1);
  int nf = 0;
  for (size_t i = 0; i < isFree.size(); i++)
    if (isFree[i]) map[i] = nf++;
  *nnodes = nn;
  *dim = D;
  *coords = dup(xyz);
  *nelem = (int64_t)elem.size() / K;
  *k = K;
  *conn = dup(elem);
  *bs = B;
  *dofs = dup(map);
  *coef = dup(cf);
  *ncoef = (int)cf.size();
  return 0;
}

// Pattern utilities of the reference (sparse.mjs buildPattern :37-78 for triangles is buildElementPattern with k = 3
// up to the in-row sort, which gives the same sorted unique rows). Outputs malloc'd arrays.
WL_API int amp_wl_element_pattern(int n, const int *elem, int64_t ne, int k, int **rowptr, int **colidx) {
  Csr P = element_pattern(n, elem, ne, k);
  *rowptr = dup(P.rowptr);
  *colidx = dup(P.colidx);
  return (int)P.colidx.size();
}
WL_API void amp_wl_free_array(void *p) { std::free(p); }

}  // extern "C"
