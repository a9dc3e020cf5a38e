// Device assembly of the local matrices (LMA) of the two operator families
// the solves use, by 3x3x3 Gauss quadrature on perturbed trilinear hexahedra:
//   W0 (Q1 nodal):   A = M + nu K,  M = int phi_i phi_j |J|,
//                    K = int (J^-T grad phi_i).(J^-T grad phi_j) |J|
//   W2 (RT0) / W3:   M2 = int (J v_i).(J v_j) / |J|, D_i = int sigma div v_i,
//                    A = M2 + tau D^T D
// These are the set-up kernels of the reference's FEM layer
// (compute_mass_matrix_kernel_w_scalar / _w2, compute_div_operator_kernel,
// coordinate_jacobian) for the synthetic workloads; each cell-layer is one
// thread and the arithmetic is that of lfric_core_b200/csrc/meshgen.c, so the
// host and device generators give the same matrices. The result is handed to
// lfx_lma_create as a device array, so large batches never pass through the
// host.
#include <cmath>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

__constant__ double c_rv[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

__device__ void gauss3(double* x, double* w) {
  const double d = sqrt(15.0) / 10.0;
  x[0] = 0.5 - d;
  x[1] = 0.5;
  x[2] = 0.5 + d;
  w[0] = 5.0 / 18.0;
  w[1] = 8.0 / 18.0;
  w[2] = 5.0 / 18.0;
}

__device__ void q1(const double* xi, double* phi, double (*dphi)[3]) {
  for (int v = 0; v < 8; ++v) {
    double f[3], g[3];
    for (int a = 0; a < 3; ++a) {
      f[a] = c_rv[v][a] > 0.5 ? xi[a] : 1.0 - xi[a];
      g[a] = c_rv[v][a] > 0.5 ? 1.0 : -1.0;
    }
    phi[v] = f[0] * f[1] * f[2];
    dphi[v][0] = g[0] * f[1] * f[2];
    dphi[v][1] = f[0] * g[1] * f[2];
    dphi[v][2] = f[0] * f[1] * g[2];
  }
}

__device__ void corners(int64_t c, int k, int nl, const int* vc, const double* xyz3d,
                        double X[8][3]) {
  for (int v = 0; v < 8; ++v) {
    const int64_t vid = vc[c * 4 + (v & 3)] - 1;
    const int64_t p = vid * (nl + 1) + k + (v >> 2);
    for (int a = 0; a < 3; ++a) X[v][a] = xyz3d[p * 3 + a];
  }
}

__device__ double jacobian(double X[8][3], double (*dphi)[3], double J[3][3]) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0.0;
      for (int v = 0; v < 8; ++v) s += X[v][a] * dphi[v][b];
      J[a][b] = s;
    }
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

__global__ void assemble_w0(int64_t nc3, int nl, const int* vc, const double* xyz3d, double nu,
                            double* lma) {
  double gx[3], gw[3];
  gauss3(gx, gw);
  for (int64_t ik = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ik < nc3;
       ik += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = ik / nl;
    const int k = (int)(ik % nl);
    double X[8][3], A[8][8];
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) A[i][j] = 0.0;
    corners(c, k, nl, vc, xyz3d, X);
    for (int q = 0; q < 27; ++q) {
      const double xi[3] = {gx[q % 3], gx[(q / 3) % 3], gx[q / 9]};
      const double wq = gw[q % 3] * gw[(q / 3) % 3] * gw[q / 9];
      double phi[8], dphi[8][3], J[3][3], G[3][3], Ji[3][3];
      q1(xi, phi, dphi);
      const double dj = jacobian(X, dphi, J), adj = fabs(dj);
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / dj;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / dj;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / dj;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / dj;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / dj;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / dj;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / dj;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / dj;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / dj;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          G[a][b] = Ji[a][0] * Ji[b][0] + Ji[a][1] * Ji[b][1] + Ji[a][2] * Ji[b][2];
      /* the upper triangle; the lower one is its mirror image, so the
       * local matrix is symmetric bit for bit */
      for (int i = 0; i < 8; ++i)
        for (int j = i; j < 8; ++j) {
          double kij = 0.0;
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) kij += dphi[i][a] * G[a][b] * dphi[j][b];
          A[i][j] += wq * adj * (phi[i] * phi[j] + nu * kij);
        }
    }
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) lma[ik + nc3 * (i + 8 * j)] = i <= j ? A[i][j] : A[j][i];
  }
}

__device__ void rt0(const double* xi, double v[6][3]) {
  for (int i = 0; i < 6; ++i)
    for (int a = 0; a < 3; ++a) v[i][a] = 0.0;
  v[0][0] = xi[0] - 1.0;
  v[1][1] = xi[1] - 1.0;
  v[2][0] = xi[0];
  v[3][1] = xi[1];
  v[4][2] = xi[2] - 1.0;
  v[5][2] = xi[2];
}

__global__ void assemble_w2(int64_t nc3, int nl, const int* cn, const int* vc,
                            const double* xyz3d, double tau, double* a) {
  double gx[3], gw[3];
  gauss3(gx, gw);
  for (int64_t ik = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ik < nc3;
       ik += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = ik / nl;
    const int k = (int)(ik % nl);
    double sg[6];
    for (int s = 0; s < 4; ++s) sg[s] = (c + 1 < cn[c * 4 + s]) ? 1.0 : -1.0;
    sg[4] = -1.0;
    sg[5] = 1.0;
    double X[8][3], M[6][6];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) M[i][j] = 0.0;
    corners(c, k, nl, vc, xyz3d, X);
    for (int q = 0; q < 27; ++q) {
      const double xi[3] = {gx[q % 3], gx[(q / 3) % 3], gx[q / 9]};
      const double wq = gw[q % 3] * gw[(q / 3) % 3] * gw[q / 9];
      double phi[8], dphi[8][3], J[3][3], v[6][3], Jv[6][3];
      q1(xi, phi, dphi);
      const double adj = fabs(jacobian(X, dphi, J));
      rt0(xi, v);
      for (int i = 0; i < 6; ++i)
        for (int r = 0; r < 3; ++r) Jv[i][r] = J[r][0] * v[i][0] + J[r][1] * v[i][1] + J[r][2] * v[i][2];
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
          M[i][j] += wq * sg[i] * sg[j] *
                     (Jv[i][0] * Jv[j][0] + Jv[i][1] * Jv[j][1] + Jv[i][2] * Jv[j][2]) / adj;
    }
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) a[ik + nc3 * (i + 6 * j)] = M[i][j] + tau * sg[i] * sg[j];
  }
}

struct DevBuf {
  lfx_ctx* ctx;
  void* p = nullptr;
  size_t n = 0;
  ~DevBuf() { dfree(ctx, p, n); }
};

int upload(lfx_ctx* ctx, DevBuf& b, const void* src, size_t bytes) {
  b.ctx = ctx;
  int rc = dmalloc(ctx, &b.p, bytes);
  if (rc) return rc;
  b.n = bytes;
  LFX_CK(ctx, cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyDefault, ctx->stream));
  return LFX_OK;
}

int make_ops(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, int32_t ndf, const int32_t* map,
             int64_t undf, const double* d_lma, int32_t ncolours, const int32_t* npc,
             const int32_t* cic, int32_t maxc, lfx_op** op64, lfx_op** op32) {
  lfx_op* first = nullptr;
  int rc = LFX_OK;
  if (op64) {
    rc = lfx_lma_create(ctx, ncell_2d, nlayers, ndf, ndf, map, map, undf, undf, d_lma, ncolours,
                        npc, cic, maxc, LFX_R64, op64);
    if (rc) return rc;
    first = *op64;
  }
  if (op32) {
    if (first)
      rc = lfx_lma_create_like(first, d_lma, LFX_R32, op32);
    else
      rc = lfx_lma_create(ctx, ncell_2d, nlayers, ndf, ndf, map, map, undf, undf, d_lma, ncolours,
                          npc, cic, maxc, LFX_R32, op32);
  }
  return rc;
}

}  // namespace

extern "C" {

int lfx_fem_w0_operator(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers,
                        const int32_t* verts_on_cell, int64_t nvert_2d, const double* xyz3d,
                        double nu, const int32_t* map, int64_t undf, int32_t ncolours,
                        const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                        int32_t max_cells_per_colour, lfx_op** op64, lfx_op** op32) {
  if (!ctx || !verts_on_cell || !xyz3d || !map || (!op64 && !op32)) return LFX_INVALID_ARGUMENT;
  const int64_t nc3 = (int64_t)ncell_2d * nlayers;
  DevBuf vc, xyz, lma;
  int rc = upload(ctx, vc, verts_on_cell, sizeof(int32_t) * 4 * (size_t)ncell_2d);
  if (!rc) rc = upload(ctx, xyz, xyz3d, sizeof(double) * 3 * (size_t)nvert_2d * (nlayers + 1));
  if (rc) return rc;
  lma.ctx = ctx;
  rc = dmalloc(ctx, &lma.p, sizeof(double) * 64 * (size_t)nc3);
  if (rc) return rc;
  lma.n = sizeof(double) * 64 * (size_t)nc3;
  assemble_w0<<<ctx->num_sms * 8, 128, 0, ctx->stream>>>(nc3, nlayers, (const int*)vc.p,
                                                          (const double*)xyz.p, nu, (double*)lma.p);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return make_ops(ctx, ncell_2d, nlayers, 8, map, undf, (const double*)lma.p, ncolours,
                  ncells_per_colour, cells_in_colour, max_cells_per_colour, op64, op32);
}

int lfx_fem_w2_operator(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, const int32_t* cell_next,
                        const int32_t* verts_on_cell, int64_t nvert_2d, const double* xyz3d,
                        double tau, const int32_t* map, int64_t undf, int32_t ncolours,
                        const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                        int32_t max_cells_per_colour, lfx_op** op64, lfx_op** op32) {
  if (!ctx || !cell_next || !verts_on_cell || !xyz3d || !map || (!op64 && !op32))
    return LFX_INVALID_ARGUMENT;
  const int64_t nc3 = (int64_t)ncell_2d * nlayers;
  DevBuf cn, vc, xyz, lma;
  int rc = upload(ctx, cn, cell_next, sizeof(int32_t) * 4 * (size_t)ncell_2d);
  if (!rc) rc = upload(ctx, vc, verts_on_cell, sizeof(int32_t) * 4 * (size_t)ncell_2d);
  if (!rc) rc = upload(ctx, xyz, xyz3d, sizeof(double) * 3 * (size_t)nvert_2d * (nlayers + 1));
  if (rc) return rc;
  lma.ctx = ctx;
  rc = dmalloc(ctx, &lma.p, sizeof(double) * 36 * (size_t)nc3);
  if (rc) return rc;
  lma.n = sizeof(double) * 36 * (size_t)nc3;
  assemble_w2<<<ctx->num_sms * 8, 128, 0, ctx->stream>>>(nc3, nlayers, (const int*)cn.p,
                                                          (const int*)vc.p, (const double*)xyz.p,
                                                          tau, (double*)lma.p);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return make_ops(ctx, ncell_2d, nlayers, 6, map, undf, (const double*)lma.p, ncolours,
                  ncells_per_colour, cells_in_colour, max_cells_per_colour, op64, op32);
}

}  // extern "C"
