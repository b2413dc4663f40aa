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

// ec = Ainv rc, one warp per row (row-major FP64 inverse)
__global__ void k_pc_gemv(const __half *__restrict__ ainv, double scale, const double *__restrict__ rc,
                          double *__restrict__ ec, int nc) {
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nc) return;
  const __half *a = ainv + (size_t)row * nc;
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
  k_pc_gemv<<<(nc + 7) / 8, 256, 0, g.st>>>(g.d_pc_ainv, g.pc_ainv_scale, g.d_pc_rc, g.d_pc_ec, nc);
  PIC_LAUNCHED();
  k_pc_prolong<<<blocks_for(g.nn, PC_THREADS), PC_THREADS, 0, g.st>>>(c, g.d_pc_ec, g.d_row_kind, assign, z,
                                                                        g.nn);
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
__global__ void k_to_f16(const double *__restrict__ a, __half *__restrict__ b, double inv_scale, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2half_rn((float)(a[i] * inv_scale));
}

__global__ void k_diag_of(const double *__restrict__ a, double *__restrict__ d, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = a[(size_t)i * n + i];
}

}  // namespace

// Builds Ac = P^T A P from the mesh's CSR stiffness matrix (unknowns,
// 1-based) and uploads its inverse.
int coarse_setup(const pic_mesh_desc *mesh, int coarse_cells) {
  if (g.d_pc_ainv) {
    cudaFree(g.d_pc_ainv);
    cudaFree(g.d_pc_rc);
    cudaFree(g.d_pc_ec);
    g.d_pc_ainv = nullptr;
    g.d_pc_rc = g.d_pc_ec = nullptr;
  }
  g.pc_cs = 0;
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
    set_error("pic_coarse_setup: coarse operator is not positive definite");
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
  rc = (e == cudaSuccess) ? pc_alloc(&g.d_pc_ainv, nc2) : cuda_fail(e, "coarse inverse diagonal");
  if (!rc) {
    k_to_f16<<<(unsigned)((nc2 + 255) / 256), 256, 0, g.st>>>(d_a, g.d_pc_ainv, 1.0 / g.pc_ainv_scale,
                                                               (int64_t)nc2);
    e = cudaStreamSynchronize(g.st);
    if (e != cudaSuccess) rc = cuda_fail(e, "coarse inverse copy");
  }
  release();
  if (rc) return rc;
  if ((rc = pc_alloc(&g.d_pc_rc, nc))) return rc;
  if ((rc = pc_alloc(&g.d_pc_ec, nc))) return rc;
  g.pc_cs = cs;
  g.pc_ncx = ncx;
  g.pc_ncy = ncy;
  return PIC_OK;
}

int precond_prepare() { return pc_vectors(); }

int precond_learned_on() { return (g.pc_learned && g.precond) ? 1 : 0; }

// The learned stage: y = fn(t) with the callback registered by the caller.
// Returns 1 when it fails.
int precond_callback() { return g.precond(g.d_pc_t, g.d_pc_y, g.precond_user) != 0 ? 1 : 0; }

void precond_free() {
  auto F = [](void *p) {
    if (p) cudaFree(p);
  };
  F(g.d_pc_t); F(g.d_pc_y); F(g.d_pc_za); F(g.d_pc_dinv); F(g.d_pc_ainv); F(g.d_pc_rc); F(g.d_pc_ec);
}

}  // namespace pic
