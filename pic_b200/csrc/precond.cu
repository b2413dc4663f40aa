// precond.cu -- the preconditioner M(r) of flexible CG (pic_ife_solve with
// PIC_SOLVER_FCG_UNET): a composition of
//   1. damped-Jacobi pre-smoothing       z1 = w D^-1 r
//   2. Galerkin coarse correction        z2 = z1 + P Ac^-1 P^T (r - A z1)
//   3. learned correction (callback)     z3 = z2 + N(r - A z2)
//   4. damped-Jacobi post-smoothing      z  = z3 + w D^-1 (r - A z3)
// Each stage can be switched off.  The smoother removes the rough part of
// the error, the coarse space (bilinear P on a uniform coarse grid of spacing
// cs nodes, Ac = P^T A P assembled on the host and inverted once on the
// device, applied from a scaled FP16 copy) the global part, and the
// network what lies between -- it is trained on exactly the residuals stage 3
// sees.  The reference solver (IFE-Solver/MY_PCG.f90) is Jacobi-PCG only:
// none of this has a counterpart there.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pic_ctx.h"

// The smoothing and post-smoothing kernels (they need the solver's stencil
// operator) and the FCG kernels are in picgpu.cu; this file holds the coarse
// space.

namespace pic {

namespace {

constexpr int PC_THREADS = 256;

struct CoarseK {
  int nnx, nny, cs, ncx, ncy;
};

// rc[C] = sum over the fine nodes f of C's support of P[f,C] t[f]
// (t is 0 on Dirichlet nodes).  One block per coarse node; fixed-order
// block reduction.
__global__ void __launch_bounds__(PC_THREADS) k_pc_restrict(CoarseK c, const double *__restrict__ t,
                                                             double *__restrict__ rc) {
  const int C = blockIdx.x;
  const int I = C / c.ncy, J = C % c.ncy;
  const int i0 = max(0, (I - 1) * c.cs + 1), i1 = min(c.nnx - 1, (I + 1) * c.cs - 1);
  const int j0 = max(0, (J - 1) * c.cs + 1), j1 = min(c.nny - 1, (J + 1) * c.cs - 1);
  const int ni = i1 - i0 + 1, nj = j1 - j0 + 1;
  const double inv = 1.0 / c.cs;
  double s = 0.0;
  for (int e = threadIdx.x; e < ni * nj; e += PC_THREADS) {
    const int i = i0 + e / nj, j = j0 + e % nj;
    const double w = (1.0 - fabs((double)(i - I * c.cs)) * inv) * (1.0 - fabs((double)(j - J * c.cs)) * inv);
    s = fma(w, t[(int64_t)i * c.nny + j], s);
  }
  __shared__ double ws[PC_THREADS / 32];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int q = 0; q < PC_THREADS / 32; ++q) a += ws[q];
    rc[C] = a;
  }
}

// ec = Ainv rc, one warp per row (row-major scaled FP16 inverse, rows of ld)
__global__ void k_pc_gemv(const __half *__restrict__ ainv, int ld, double scale, const double *__restrict__ rc,
                          double *__restrict__ ec, int nc) {
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nc) return;
  const __half *a = ainv + (size_t)row * ld;
  double s = 0.0;
  for (int k = lane; k < nc; k += 32) s = fma((double)__half2float(a[k]), rc[k], s);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) ec[row] = s * scale;
}

// z (+)= P ec on unknown nodes (bilinear from the four coarse nodes around);
// with assign, z = P ec and 0 on Dirichlet nodes
__global__ void k_pc_prolong(CoarseK c, const double *__restrict__ ec, const int32_t *__restrict__ row_kind,
                             int assign, double *__restrict__ z, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  if (row_kind[n] < 0) {
    if (assign) z[n] = 0.0;
    return;
  }
  const int i = (int)(n / c.nny), j = (int)(n % c.nny);
  const int I = i / c.cs, J = j / c.cs;
  const double fx = (double)(i - I * c.cs) / c.cs, fy = (double)(j - J * c.cs) / c.cs;
  const int I1 = min(I + 1, c.ncx - 1), J1 = min(J + 1, c.ncy - 1);
  double v = (1.0 - fx) * (1.0 - fy) * ec[I * c.ncy + J];
  v = fma(fx * (1.0 - fy), ec[I1 * c.ncy + J], v);
  v = fma((1.0 - fx) * fy, ec[I * c.ncy + J1], v);
  v = fma(fx * fy, ec[I1 * c.ncy + J1], v);
  z[n] = assign ? v : z[n] + v;
}

// ---- multigrid V-cycle, one launch per operation (the persistent solver
// runs the same per-node functions between grid barriers)

__global__ void k_mg_restrict(MgLevel L, const double *__restrict__ tf, int nxf, int nyf, double w, int smoothed) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < (int64_t)L.nx * L.ny) mg_restrict_node(L, tf, nxf, nyf, w, smoothed != 0, n);
}

__global__ void k_mg_smooth(MgLevel L) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < (int64_t)L.nx * L.ny) mg_smooth_node(L, n);
}

__global__ void k_mg_post(MgLevel L, const double *__restrict__ ec, int nyc, double w) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < (int64_t)L.nx * L.ny) mg_post_node(L, ec, nyc, w, n);
}

// z (+)= P e_1 on unknown nodes of the solver's grid (z = P e_1 and 0 on
// Dirichlet nodes with assign)
__global__ void k_mg_prolong0(const double *__restrict__ e1, int ny1, const int32_t *__restrict__ row_kind, int nny,
                              int assign, double *__restrict__ z, int64_t nn) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  if (row_kind[n] < 0) {
    if (assign) z[n] = 0.0;
    return;
  }
  const int i = (int)(n / nny), j = (int)(n - (int64_t)i * nny);
  const double pe = mg_prolong(e1, ny1, i, j);
  z[n] = assign ? pe : z[n] + pe;
}

__global__ void k_pc_dinv(const double *__restrict__ diag, double *__restrict__ dinv, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nn) dinv[n] = 1.0 / diag[n];
}

template <class T>
int pc_alloc(T **p, size_t n) {
  PIC_CUDA(cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)));
  return PIC_OK;
}

int pc_vectors() {
  int rc;
  if (!g.d_pc_t && (rc = pc_alloc(&g.d_pc_t, g.nn))) return rc;
  if (!g.d_pc_y && (rc = pc_alloc(&g.d_pc_y, g.nn))) return rc;
  if (!g.d_pc_za && (rc = pc_alloc(&g.d_pc_za, g.nn))) return rc;
  if (!g.d_pc_dinv) {
    if ((rc = pc_alloc(&g.d_pc_dinv, g.nn))) return rc;
    k_pc_dinv<<<blocks_for(g.nn, PC_THREADS), PC_THREADS, 0, g.st>>>(g.d_diag, g.d_pc_dinv, g.nn);
    PIC_LAUNCHED();
  }
  return PIC_OK;
}

CoarseK coarse_k() { return CoarseK{g.m.nnx, g.m.nny, g.pc_cs, g.pc_ncx, g.pc_ncy}; }

}  // namespace

// z += P Ac^-1 P^T t (z = P Ac^-1 P^T t with assign)
int coarse_correct(const double *t, double *z, int assign) {
  CoarseK c = coarse_k();
  const int nc = c.ncx * c.ncy;
  k_pc_restrict<<<nc, PC_THREADS, 0, g.st>>>(c, t, g.d_pc_rc);
  PIC_LAUNCHED();
  k_pc_gemv<<<(nc + 7) / 8, 256, 0, g.st>>>(g.d_pc_ainv, g.pc_ainv_ld, g.pc_ainv_scale, g.d_pc_rc, g.d_pc_ec, nc);
  PIC_LAUNCHED();
  k_pc_prolong<<<blocks_for(g.nn, PC_THREADS), PC_THREADS, 0, g.st>>>(c, g.d_pc_ec, g.d_row_kind, assign, z,
                                                                        g.nn);
  PIC_LAUNCHED();
  return PIC_OK;
}

// z += P V(t) (z = P V(t) with assign): the multigrid V-cycle of t, the
// solver-grid residual after pre-smoothing (0 on Dirichlet nodes)
int mg_correct(const double *t, double *z, int assign) {
  const MgK &M = g.mg;
  const double w = g.pc_omega;
  for (int l = 1; l < M.L; ++l) {
    const MgLevel &L = M.lv[l];
    const int64_t nl = (int64_t)L.nx * L.ny;
    const double *tf = l == 1 ? t : M.lv[l - 1].t;
    const int nxf = l == 1 ? g.m.nnx : M.lv[l - 1].nx, nyf = l == 1 ? g.m.nny : M.lv[l - 1].ny;
    k_mg_restrict<<<blocks_for(nl, PC_THREADS), PC_THREADS, 0, g.st>>>(L, tf, nxf, nyf, w, l < M.L - 1 ? 1 : 0);
    PIC_LAUNCHED();
    if (l < M.L - 1) {
      k_mg_smooth<<<blocks_for(nl, PC_THREADS), PC_THREADS, 0, g.st>>>(L);
      PIC_LAUNCHED();
    }
  }
  const MgLevel &C = M.lv[M.L - 1];
  const int nc = C.nx * C.ny;
  k_pc_gemv<<<(nc + 7) / 8, 256, 0, g.st>>>(g.d_pc_ainv, g.pc_ainv_ld, g.pc_ainv_scale, C.r, C.z, nc);
  PIC_LAUNCHED();
  for (int l = M.L - 2; l >= 1; --l) {
    const MgLevel &L = M.lv[l];
    k_mg_post<<<blocks_for((int64_t)L.nx * L.ny, PC_THREADS), PC_THREADS, 0, g.st>>>(L, mg_e(M, l + 1),
                                                                                     M.lv[l + 1].ny, w);
    PIC_LAUNCHED();
  }
  k_mg_prolong0<<<blocks_for(g.nn, PC_THREADS), PC_THREADS, 0, g.st>>>(mg_e(M, 1), M.lv[1].ny, g.d_row_kind,
                                                                        g.m.nny, assign, z, g.nn);
  PIC_LAUNCHED();
  return PIC_OK;
}

namespace {

// Gauss-Jordan inversion of the dense SPD coarse operator on the device,
// without pivoting (SPD pivots stay positive), one elimination step per
// pair of launches: k_gj_pivot copies the scaled pivot row and the pivot
// column, k_gj_update eliminates column k from every other row and writes
// the new row and column k.  In-place, FP64.
__global__ void k_gj_pivot(const double *__restrict__ A, int n, int k, double *__restrict__ rowk,
                           double *__restrict__ colk, int *__restrict__ bad) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double p = A[(size_t)k * n + k];
  if (j == 0 && !(p > 0.0)) *bad = 1;
  rowk[j] = (j == k) ? 1.0 / p : A[(size_t)k * n + j] / p;
  colk[j] = A[(size_t)j * n + k];
}

__global__ void k_gj_update(double *__restrict__ A, int n, int k, const double *__restrict__ rowk,
                            const double *__restrict__ colk) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int i = (int)(e / n), j = (int)(e % n);
  double v;
  if (i == k) v = rowk[j];
  else if (j == k) v = -colk[i] * rowk[k];
  else v = fma(-colk[i], rowk[j], A[e]);
  A[e] = v;
}

// FP16 copy of the inverse, divided by `scale` so the largest entry (on the
// diagonal, as for any SPD matrix) sits near 2^14
// b (rows of ld, zero past column n) = a (n x n) / scale, in FP16
__global__ void k_to_f16(const double *__restrict__ a, __half *__restrict__ b, double inv_scale, int n, int ld) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * ld) return;
  const int64_t row = i / ld;
  const int col = (int)(i - row * ld);
  b[i] = col < n ? __float2half_rn((float)(a[row * n + col] * inv_scale)) : __float2half_rn(0.0f);
}

__global__ void k_diag_of(const double *__restrict__ a, double *__restrict__ d, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = a[(size_t)i * n + i];
}

// Inverts the dense SPD nc x nc matrix Ac on the device (Gauss-Jordan, FP64)
// and keeps the scaled FP16 copy the solver reads in g.d_pc_ainv.
int dense_inverse_f16(const std::vector<double> &Ac, int nc, const char *who) {
  int rc;
  double *d_a = nullptr, *d_row = nullptr, *d_col = nullptr;
  int *d_bad = nullptr;
  const size_t nc2 = (size_t)nc * nc;
  if ((rc = pc_alloc(&d_a, nc2))) return rc;
  if ((rc = pc_alloc(&d_row, nc)) || (rc = pc_alloc(&d_col, nc)) || (rc = pc_alloc(&d_bad, 1))) {
    cudaFree(d_a);
    return rc;
  }
  auto release = [&]() {
    cudaFree(d_a);
    cudaFree(d_row);
    cudaFree(d_col);
    cudaFree(d_bad);
  };
  int bad = 0;
  cudaError_t e = cudaMemcpyAsync(d_a, Ac.data(), nc2 * sizeof(double), cudaMemcpyHostToDevice, g.st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), g.st);
  for (int k = 0; e == cudaSuccess && k < nc; ++k) {
    k_gj_pivot<<<(nc + 255) / 256, 256, 0, g.st>>>(d_a, nc, k, d_row, d_col, d_bad);
    k_gj_update<<<(unsigned)((nc2 + 255) / 256), 256, 0, g.st>>>(d_a, nc, k, d_row, d_col);
    e = cudaPeekAtLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, g.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.st);
  if (e != cudaSuccess) {
    release();
    return cuda_fail(e, "coarse operator inversion");
  }
  if (bad) {
    release();
    set_error(std::string(who) + ": coarse operator is not positive definite");
    return PIC_ERR_SETUP;
  }
  // The per-iteration GEMV reads a scaled FP16 copy (a quarter of the FP64
  // bytes: 36 MB at 65x65 coarse nodes, so it and the solver's vectors fit in
  // L2 together) and accumulates in FP64.  A preconditioner tolerates the
  // 2^-11 relative rounding of the coarse correction; convergence is always
  // judged on the FP64 residual.
  std::vector<double> dg(nc);
  k_diag_of<<<(nc + 255) / 256, 256, 0, g.st>>>(d_a, d_row, nc);
  e = cudaMemcpyAsync(dg.data(), d_row, nc * sizeof(double), cudaMemcpyDeviceToHost, g.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.st);
  double dmax = 0.0;
  for (double v : dg) dmax = std::max(dmax, std::fabs(v));
  g.pc_ainv_scale = (dmax > 0.0) ? dmax / 16384.0 : 1.0;
  // rows padded to a multiple of 8 coefficients (16 bytes) for vector loads
  g.pc_ainv_ld = (nc + 7) & ~7;
  const size_t nld = (size_t)nc * g.pc_ainv_ld;
  rc = (e == cudaSuccess) ? pc_alloc(&g.d_pc_ainv, nld) : cuda_fail(e, "coarse inverse diagonal");
  if (!rc) {
    k_to_f16<<<(unsigned)((nld + 255) / 256), 256, 0, g.st>>>(d_a, g.d_pc_ainv, 1.0 / g.pc_ainv_scale, nc,
                                                               g.pc_ainv_ld);
    e = cudaStreamSynchronize(g.st);
    if (e != cudaSuccess) rc = cuda_fail(e, "coarse inverse copy");
  }
  release();
  if (rc) return rc;
  return PIC_OK;
}

void coarse_free() {
  if (g.d_pc_ainv) cudaFree(g.d_pc_ainv);
  if (g.d_pc_rc) cudaFree(g.d_pc_rc);
  if (g.d_pc_ec) cudaFree(g.d_pc_ec);
  g.d_pc_ainv = nullptr;
  g.d_pc_rc = g.d_pc_ec = nullptr;
  g.pc_cs = 0;
}

void mg_free() {
  for (int l = 1; l < PIC_MG_MAX_LEVELS; ++l) {
    MgLevel &L = g.mg.lv[l];
    for (void *p : {(void *)L.st, (void *)L.dinv, (void *)L.r, (void *)L.z, (void *)L.t})
      if (p) cudaFree(p);
    L = MgLevel{};
  }
  if (g.mg.L > 1 && g.d_pc_ainv) {
    cudaFree(g.d_pc_ainv);
    g.d_pc_ainv = nullptr;
  }
  g.mg.L = 0;
}

}  // namespace

// Builds Ac = P^T A P from the mesh's CSR stiffness matrix (unknowns,
// 1-based) and uploads its inverse.
int coarse_setup(const pic_mesh_desc *mesh, int coarse_cells) {
  coarse_free();
  mg_free();
  ++g.fcg_graph_gen;  // captured iterations hold the old buffers
  if (coarse_cells <= 0) return PIC_OK;
  const int ex = g.m.nnx - 1, ey = g.m.nny - 1;
  int cs = std::max(1, std::min(ex, ey) / coarse_cells);
  while (cs > 1 && (ex % cs || ey % cs)) --cs;
  const int ncx = ex / cs + 1, ncy = ey / cs + 1, nc = ncx * ncy;
  if (nc > 9000) {
    set_error("pic_coarse_setup: coarse grid too large (at most 9000 coarse nodes)");
    return PIC_ERR_ARG;
  }
  const int64_t nn = (int64_t)g.m.nnx * g.m.nny;
  const int nu = mesh->n_unknowns;
  std::vector<int64_t> node_of(nu);
  for (int64_t n = 0; n < nn; ++n)
    if (mesh->node_type[n] > 0) node_of[mesh->node_type[n] - 1] = n;
  // P rows: up to 4 (coarse index, weight) per unknown
  std::vector<int> pc((size_t)nu * 4);
  std::vector<double> pw((size_t)nu * 4);
  for (int u = 0; u < nu; ++u) {
    const int64_t n = node_of[u];
    const int i = (int)(n / g.m.nny), j = (int)(n % g.m.nny);
    const int I = i / cs, J = j / cs;
    const double fx = (double)(i - I * cs) / cs, fy = (double)(j - J * cs) / cs;
    const int I1 = std::min(I + 1, ncx - 1), J1 = std::min(J + 1, ncy - 1);
    const int cc[4] = {I * ncy + J, I1 * ncy + J, I * ncy + J1, I1 * ncy + J1};
    const double ww[4] = {(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy};
    for (int q = 0; q < 4; ++q) {
      pc[4 * (size_t)u + q] = cc[q];
      pw[4 * (size_t)u + q] = ww[q];
    }
  }
  std::vector<double> Ac((size_t)nc * nc, 0.0);
  for (int u = 0; u < nu; ++u)
    for (int64_t e = mesh->a_srow[u] - 1; e < mesh->a_srow[u + 1] - 1; ++e) {
      const int v = mesh->a_jcol[e] - 1;
      const double a = mesh->a_k[e];
      for (int p = 0; p < 4; ++p) {
        const double wp = pw[4 * (size_t)u + p];
        if (wp == 0.0) continue;
        for (int q = 0; q < 4; ++q) {
          const double wq = pw[4 * (size_t)v + q];
          if (wq == 0.0) continue;
          Ac[(size_t)pc[4 * (size_t)u + p] * nc + pc[4 * (size_t)v + q]] += wp * a * wq;
        }
      }
    }
  for (int C = 0; C < nc; ++C)  // coarse nodes without unknowns in their support
    if (Ac[(size_t)C * nc + C] == 0.0) Ac[(size_t)C * nc + C] = 1.0;
  int rc;
  if ((rc = dense_inverse_f16(Ac, nc, "pic_coarse_setup"))) return rc;
  if ((rc = pc_alloc(&g.d_pc_rc, nc))) return rc;
  if ((rc = pc_alloc(&g.d_pc_ec, nc))) return rc;
  g.pc_cs = cs;
  g.pc_ncx = ncx;
  g.pc_ncy = ncy;
  return PIC_OK;
}

namespace {

// Row of bilinear interpolation P for the node (i, j) of a grid whose
// coarser grid has nyc columns: up to 4 (coarse node, weight) pairs.
int p_row(int i, int j, int nyc, int *cc, double *ww) {
  const int I = i >> 1, J = j >> 1;
  const int nxp = (i & 1) ? 2 : 1, nyp = (j & 1) ? 2 : 1;
  const double wx = (i & 1) ? 0.5 : 1.0, wy = (j & 1) ? 0.5 : 1.0;
  int k = 0;
  for (int a = 0; a < nxp; ++a)
    for (int b = 0; b < nyp; ++b) {
      cc[k] = (I + a) * nyc + (J + b);
      ww[k] = wx * wy;
      ++k;
    }
  return k;
}

// st[k*nc + C] += wu * a * wv for the coarse pair (C, C2); false when C2 is
// not among C's 9 neighbours (the finer operator is not a 9-point stencil)
inline bool rap_add(std::vector<double> &st, int64_t nc, int nyc, int C, int C2, double v) {
  const int dI = C2 / nyc - C / nyc, dJ = C2 % nyc - C % nyc;
  if (dI < -1 || dI > 1 || dJ < -1 || dJ > 1) return false;
  st[(size_t)((dI + 1) * 3 + (dJ + 1)) * nc + C] += v;
  return true;
}

}  // namespace

// Galerkin hierarchy A_{l+1} = P^T A_l P on grids halved until at most
// max_coarse_nodes remain (each halving needs nnx-1 and nny-1 even), level 1
// from the mesh's CSR stiffness matrix over the unknowns, the coarsest level
// inverted densely.  Replaces the two-level coarse space.
int mg_setup(const pic_mesh_desc *mesh, int max_coarse) {
  coarse_free();
  mg_free();
  ++g.fcg_graph_gen;  // captured iterations hold the old buffers
  if (max_coarse <= 0) return PIC_OK;
  int nx[PIC_MG_MAX_LEVELS], ny[PIC_MG_MAX_LEVELS];
  nx[0] = g.m.nnx;
  ny[0] = g.m.nny;
  int L = 1;
  while (L < PIC_MG_MAX_LEVELS && (int64_t)nx[L - 1] * ny[L - 1] > max_coarse && (nx[L - 1] - 1) % 2 == 0 &&
         (ny[L - 1] - 1) % 2 == 0 && nx[L - 1] >= 5 && ny[L - 1] >= 5) {
    nx[L] = (nx[L - 1] - 1) / 2 + 1;
    ny[L] = (ny[L - 1] - 1) / 2 + 1;
    ++L;
  }
  if (L < 2 || (int64_t)nx[L - 1] * ny[L - 1] > 9000) {
    set_error("pic_multigrid_setup: the grid does not halve down to 9000 nodes or fewer "
              "(nnx-1 and nny-1 need enough factors of 2)");
    return PIC_ERR_ARG;
  }
  std::vector<std::vector<double>> st(L);
  std::vector<std::vector<char>> act(L);
  int cu[4], cv[4];
  double wu[4], wv[4];
  bool ok = true;
  {  // level 1 from the CSR rows of the unknowns (1-based)
    const int64_t nn = (int64_t)g.m.nnx * g.m.nny, n1 = (int64_t)nx[1] * ny[1];
    const int nu = mesh->n_unknowns, nny = g.m.nny;
    std::vector<int64_t> node_of(nu);
    for (int64_t n = 0; n < nn; ++n)
      if (mesh->node_type[n] > 0) node_of[mesh->node_type[n] - 1] = n;
    st[1].assign((size_t)9 * n1, 0.0);
    for (int u = 0; u < nu && ok; ++u) {
      const int64_t n = node_of[u];
      const int ku = p_row((int)(n / nny), (int)(n % nny), ny[1], cu, wu);
      for (int64_t e = mesh->a_srow[u] - 1; e < mesh->a_srow[u + 1] - 1 && ok; ++e) {
        const int64_t m = node_of[mesh->a_jcol[e] - 1];
        const double a = mesh->a_k[e];
        const int kv = p_row((int)(m / nny), (int)(m % nny), ny[1], cv, wv);
        for (int p = 0; p < ku; ++p)
          for (int q = 0; q < kv; ++q) ok = ok && rap_add(st[1], n1, ny[1], cu[p], cv[q], (wu[p] * a) * wv[q]);
      }
    }
  }
  for (int l = 1; l < L && ok; ++l) {
    const int64_t nl = (int64_t)nx[l] * ny[l];
    act[l].resize(nl);
    for (int64_t n = 0; n < nl; ++n) act[l][n] = st[l][4 * (size_t)nl + n] != 0.0;
    if (l + 1 == L) break;
    const int64_t nc = (int64_t)nx[l + 1] * ny[l + 1];
    st[l + 1].assign((size_t)9 * nc, 0.0);
    for (int64_t f = 0; f < nl && ok; ++f) {
      if (!act[l][f]) continue;
      const int i = (int)(f / ny[l]), j = (int)(f % ny[l]);
      const int ku = p_row(i, j, ny[l + 1], cu, wu);
      for (int k = 0; k < 9 && ok; ++k) {
        const int i2 = i + k / 3 - 1, j2 = j + k % 3 - 1;
        if (i2 < 0 || i2 >= nx[l] || j2 < 0 || j2 >= ny[l]) continue;
        const int64_t f2 = (int64_t)i2 * ny[l] + j2;
        const double a = st[l][(size_t)k * nl + f];
        if (a == 0.0 || !act[l][f2]) continue;
        const int kv = p_row(i2, j2, ny[l + 1], cv, wv);
        for (int p = 0; p < ku; ++p)
          for (int q = 0; q < kv; ++q) ok = ok && rap_add(st[l + 1], nc, ny[l + 1], cu[p], cv[q], (wu[p] * a) * wv[q]);
      }
    }
  }
  if (!ok) {
    set_error("pic_multigrid_setup: the stiffness matrix couples nodes more than one cell apart");
    return PIC_ERR_SETUP;
  }
  int rc = PIC_OK;
  for (int l = 1; l < L && !rc; ++l) {  // FP32 stencils and 1/diag, FP64 vectors
    const int64_t nl = (int64_t)nx[l] * ny[l];
    std::vector<float> s32((size_t)9 * nl), d32(nl);
    for (size_t q = 0; q < s32.size(); ++q) s32[q] = (float)st[l][q];
    for (int64_t n = 0; n < nl; ++n) d32[n] = act[l][n] ? (float)(1.0 / st[l][4 * (size_t)nl + n]) : 0.0f;
    MgLevel &V = g.mg.lv[l];
    V.nx = nx[l];
    V.ny = ny[l];
    float *dst = nullptr, *ddi = nullptr;
    if ((rc = pc_alloc(&dst, s32.size())) || (rc = pc_alloc(&ddi, (size_t)nl))) break;
    V.st = dst;
    V.dinv = ddi;
    if ((rc = pc_alloc(&V.r, (size_t)nl)) || (rc = pc_alloc(&V.z, (size_t)nl)) || (rc = pc_alloc(&V.t, (size_t)nl)))
      break;
    cudaError_t e = cudaMemcpy(dst, s32.data(), s32.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ddi, d32.data(), d32.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(V.r, 0, nl * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(V.z, 0, nl * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(V.t, 0, nl * sizeof(double));
    if (e != cudaSuccess) rc = cuda_fail(e, "pic_multigrid_setup upload");
  }
  if (!rc) {  // the coarsest operator, dense (identity rows on inactive nodes)
    const int nc = nx[L - 1] * ny[L - 1];
    std::vector<double> Ac((size_t)nc * nc, 0.0);
    const std::vector<double> &sc = st[L - 1];
    for (int C = 0; C < nc; ++C) {
      if (!act[L - 1][C]) {
        Ac[(size_t)C * nc + C] = 1.0;
        continue;
      }
      const int I = C / ny[L - 1], J = C % ny[L - 1];
      for (int k = 0; k < 9; ++k) {
        const int i2 = I + k / 3 - 1, j2 = J + k % 3 - 1;
        if (i2 < 0 || i2 >= nx[L - 1] || j2 < 0 || j2 >= ny[L - 1]) continue;
        Ac[(size_t)C * nc + (size_t)i2 * ny[L - 1] + j2] += sc[(size_t)k * nc + C];
      }
    }
    rc = dense_inverse_f16(Ac, nc, "pic_multigrid_setup");
  }
  if (rc) {
    mg_free();
    return rc;
  }
  g.mg.lv[0].nx = g.m.nnx;
  g.mg.lv[0].ny = g.m.nny;
  g.mg.L = L;
  return PIC_OK;
}

int precond_prepare() { return pc_vectors(); }

int precond_learned_on() { return (g.pc_learned && g.precond) ? 1 : 0; }

// The learned stage: y = fn(t) with the callback registered by the caller.
// Returns 1 when it fails.
int precond_callback() { return g.precond(g.d_pc_t, g.d_pc_y, g.precond_user) != 0 ? 1 : 0; }

void precond_free() {
  mg_free();
  auto F = [](void *p) {
    if (p) cudaFree(p);
  };
  F(g.d_pc_t); F(g.d_pc_y); F(g.d_pc_za); F(g.d_pc_dinv); F(g.d_pc_ainv); F(g.d_pc_rc); F(g.d_pc_ec);
}

}  // namespace pic
