// On-device assembly of the CSR values from a mesh (the reference's assembleCells, physics/src/common/scalar.ts:96-146,
// with its element slots, la/sparse.mjs:113-185): the values are produced in HBM, so a refactorisation with new
// coefficients (a time step, a Newton step, another shift) moves only the per-element coefficients over PCIe.
//
// Two kernels:
//   k_elem_*     one thread per element computes its full nd x nd element matrix (nd = nodes x DOFs per node, local
//                index bs a + c for node a, component c) into a per-element buffer;
//   k_gather     one thread per CSR slot sums the element entries that land on it, in increasing element order: the
//                order in which the reference's element loop adds them (K[slots[...]] += Ke[...]), so the values are
//                the same bits as the host assembly in that order.
// This file is compiled without FMA contraction (-fmad=false): every product and sum rounds as in the host code.
#include <cuda_runtime.h>

#include <cstdint>

namespace amp {

// P1 triangles, scalar coefficient k per element: Ke_ab = A (gx_a (k gx_b) + gy_a (k gy_b)), the triangle geometry
// and stiffness of fem/tri.mjs:45-80 with cxx = cyy = k.
__global__ void k_elem_p1tri(int64_t ne, const int *__restrict__ conn, const double *__restrict__ xy,
                             const double *__restrict__ coef, double *__restrict__ Ke) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int i = conn[3 * e], j = conn[3 * e + 1], k = conn[3 * e + 2];
  const double x1 = xy[2 * (int64_t)i], y1 = xy[2 * (int64_t)i + 1], x2 = xy[2 * (int64_t)j],
               y2 = xy[2 * (int64_t)j + 1], x3 = xy[2 * (int64_t)k], y3 = xy[2 * (int64_t)k + 1];
  const double a2 = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
  const double A = 0.5 * a2;
  const double gx[3] = {(y2 - y3) / a2, (y3 - y1) / a2, (y1 - y2) / a2};
  const double gy[3] = {(x3 - x2) / a2, (x1 - x3) / a2, (x2 - x1) / a2};
  const double kk = coef[e];
  double *out = Ke + 9 * e;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) out[3 * a + b] = A * (gx[a] * (kk * gx[b]) + gy[a] * (kk * gy[b]));
}

// P1 tets, linear elasticity with (E, nu) per element: Ke = V B^T D B, D = dMatrix('3d', E, nu) in Voigt order
// [xx, yy, zz, yz, xz, xy] (physics/src/elastic/index.ts:50-58), B the strain-displacement matrix of the gradients of
// the barycentric coordinates. Local DOF 3 a + c. The upper triangle is computed and mirrored (Ke exactly symmetric).
__global__ void __launch_bounds__(128) k_elem_p1tet_elastic(int64_t ne, const int *__restrict__ conn,
                                                            const double *__restrict__ xyz,
                                                            const double *__restrict__ coef, double *__restrict__ Ke) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double p[4][3];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int d = 0; d < 3; d++) p[a][d] = xyz[3 * (int64_t)conn[4 * e + a] + d];
  // gradients of the barycentric coordinates and the volume
  const double av[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
  const double bv[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
  const double cv[3] = {p[3][0] - p[0][0], p[3][1] - p[0][1], p[3][2] - p[0][2]};
  const double det = av[0] * (bv[1] * cv[2] - bv[2] * cv[1]) - av[1] * (bv[0] * cv[2] - bv[2] * cv[0]) +
                     av[2] * (bv[0] * cv[1] - bv[1] * cv[0]);
  double inv[3][3];
  inv[0][0] = (bv[1] * cv[2] - bv[2] * cv[1]) / det;
  inv[0][1] = (bv[2] * cv[0] - bv[0] * cv[2]) / det;
  inv[0][2] = (bv[0] * cv[1] - bv[1] * cv[0]) / det;
  inv[1][0] = (cv[1] * av[2] - cv[2] * av[1]) / det;
  inv[1][1] = (cv[2] * av[0] - cv[0] * av[2]) / det;
  inv[1][2] = (cv[0] * av[1] - cv[1] * av[0]) / det;
  inv[2][0] = (av[1] * bv[2] - av[2] * bv[1]) / det;
  inv[2][1] = (av[2] * bv[0] - av[0] * bv[2]) / det;
  inv[2][2] = (av[0] * bv[1] - av[1] * bv[0]) / det;
  double g[4][3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    g[1][d] = inv[0][d];
    g[2][d] = inv[1][d];
    g[3][d] = inv[2][d];
    g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
  }
  const double V = fabs(det) / 6.0;
  const double E = coef[2 * e], nu = coef[2 * e + 1];
  const double lam = (E * nu) / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  double D[6][6];
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) D[i][j] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
#pragma unroll
    for (int j = 0; j < 3; j++) D[i][j] = lam;
    D[i][i] = lam + 2 * mu;
    D[i + 3][i + 3] = mu;
  }
  double B[6][12];
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int c = 0; c < 12; c++) B[i][c] = 0.0;
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const double gx = g[a][0], gy = g[a][1], gz = g[a][2];
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
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int c = 0; c < 12; c++) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) s += D[i][k] * B[k][c];
      DB[i][c] = s;
    }
  double *out = Ke + 144 * e;
#pragma unroll 1
  for (int r = 0; r < 12; r++)
#pragma unroll 1
    for (int c = r; c < 12; c++) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) s += B[k][r] * DB[k][c];
      out[12 * r + c] = out[12 * c + r] = V * s;
    }
}

// values[s] = sum of Ke[gidx[q]] for q in [gptr[s], gptr[s + 1]) (element order), from +0.
__global__ void k_gather_slots(int64_t nnz, const int64_t *__restrict__ gptr, const uint32_t *__restrict__ gidx,
                               const double *__restrict__ Ke, double *__restrict__ values) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nnz) return;
  double v = 0.0;
  for (int64_t q = gptr[s]; q < gptr[s + 1]; q++) v += Ke[gidx[q]];
  values[s] = v;
}

// kind 0: P1 triangles (scalar), kind 1: P1 tets (elasticity); returns the kernels launched
int launch_assemble_values(int kind, int64_t ne, const int *conn, const double *coords, const double *coef, double *Ke,
                           int64_t nnz, const int64_t *gptr, const uint32_t *gidx, double *values, cudaStream_t st) {
  int launched = 0;
  if (ne > 0) {
    if (kind == 0)
      k_elem_p1tri<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(ne, conn, coords, coef, Ke);
    else
      k_elem_p1tet_elastic<<<(unsigned)((ne + 127) / 128), 128, 0, st>>>(ne, conn, coords, coef, Ke);
    launched++;
  }
  if (nnz > 0) {
    k_gather_slots<<<(unsigned)((nnz + 255) / 256), 256, 0, st>>>(nnz, gptr, gidx, Ke, values);
    launched++;
  }
  return launched;
}

}  // namespace amp
