// mg_dev.h -- geometric multigrid V-cycle of the flexible-CG preconditioner:
// the per-node operations, shared by the persistent solver kernel
// (picgpu.cu) and the one-launch-per-operation path (precond.cu), so both
// compute the same numbers.
//
// Level 0 is the solver's own grid and operator.  Level l >= 1 is the uniform
// grid of every second node of level l-1 (nx_l = (nx_{l-1} - 1)/2 + 1), with
// the Galerkin operator A_l = P^T A_{l-1} P of bilinear interpolation P,
// assembled on the host; it is a 9-point stencil, stored per node as FP32
// coefficients st[3a+c][n] coupling node (I,J) with (I+a-1, J+c-1).  A level
// node whose support holds no unknown of the finer level is inactive:
// dinv = 0 there, and every vector stays 0 on it.  The coarsest level is
// solved with the dense FP16 inverse of its operator.
//
// One V-cycle, with damped Jacobi (weight w) as smoother, one sweep down and
// one up at every level:
//   down, l = 1..L-1:  r_l = P^T t_{l-1}, z_l = w D_l^-1 r_l (one pass)
//                      t_l = r_l - A_l z_l                          (l < L-1)
//                      z_{L-1} = A_{L-1}^-1 r_{L-1}                 (coarsest)
//   up,   l = L-2..1:  y = z_l + P e_{l+1},  e_l = y + w D_l^-1 (r_l - A_l y)
//   level 0:           zA += P e_1, then the solver's own post-smoothing.
// e_l is stored in t_l (no longer needed once r_{l+1} exists); the
// coarsest level's e is its z.
#ifndef PIC_MG_DEV_H
#define PIC_MG_DEV_H

#include <stdint.h>

namespace pic {

#define PIC_MG_MAX_LEVELS 8

struct MgLevel {
  int nx, ny;          // grid nodes
  const float *st;     // [9][nx*ny]
  const float *dinv;   // [nx*ny], 0 on inactive nodes
  double *r, *z, *t;   // [nx*ny]
};

struct MgK {
  int L;  // levels including the solver's grid (0: no multigrid)
  MgLevel lv[PIC_MG_MAX_LEVELS];
};

// (i, j) of node m, a node of the 3x3 neighbourhood of node n = (I, J) on a
// grid of ny nodes per column, without an integer division: m - n = a ny + c
// with a, c in {-1, 0, 1} (ny >= 3).
__device__ __forceinline__ void mg_nb_ij(int64_t n, int I, int J, int64_t m, int ny, int &i, int &j) {
  const int64_t d = m - n;
  const int a = d >= ny - 1 ? 1 : (d <= 1 - ny ? -1 : 0);
  i = I + a;
  j = J + (int)(d - (int64_t)a * ny);
}

// r_l[I,J] = sum over the 3x3 finer nodes around (2I, 2J) of w_x w_y t[f],
// w = 1 at the centre and 1/2 beside it (P^T of bilinear interpolation);
// fixed order, rows then columns.
template <class T>
__device__ __forceinline__ double mg_restrict(const T *__restrict__ tf, int nxf, int nyf, int I, int J) {
  const int i0 = 2 * I, j0 = 2 * J;
  double s = 0.0;
#pragma unroll
  for (int a = -1; a <= 1; ++a) {
    const int i = i0 + a;
    if (i < 0 || i >= nxf) continue;
    const double wa = a == 0 ? 1.0 : 0.5;
#pragma unroll
    for (int c = -1; c <= 1; ++c) {
      const int j = j0 + c;
      if (j < 0 || j >= nyf) continue;
      const double w = c == 0 ? wa : 0.5 * wa;
      s = fma(w, (double)tf[(int64_t)i * nyf + j], s);
    }
  }
  return s;
}

// (P e)[i,j] on the finer grid from the coarser level's e (nxc x nyc):
// bilinear, the coarse nodes i/2 (even i) or (i-1)/2 and (i+1)/2 (odd i)
__device__ __forceinline__ double mg_prolong(const double *__restrict__ e, int nyc, int i, int j) {
  const int I = i >> 1, J = j >> 1;
  const bool ox = i & 1, oy = j & 1;
  const double *p = e + (int64_t)I * nyc + J;
  if (!ox && !oy) return p[0];
  if (ox && !oy) return 0.5 * (p[0] + p[nyc]);
  if (!ox && oy) return 0.5 * (p[0] + p[1]);
  return 0.25 * ((p[0] + p[nyc]) + (p[1] + p[nyc + 1]));
}

// A_l applied at node n = (I,J) to the values v(m) of the 9 nodes around
// (coefficients toward nodes outside the grid are 0 and not read)
template <class Fv>
__device__ __forceinline__ double mg_apply(const MgLevel &L, int I, int J, Fv v) {
  const int64_t nl = (int64_t)L.nx * L.ny, n = (int64_t)I * L.ny + J;
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int i = I + a - 1;
    if (i < 0 || i >= L.nx) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int j = J + c - 1;
      if (j < 0 || j >= L.ny) continue;
      acc = fma((double)L.st[(3 * a + c) * nl + n], v((int64_t)i * L.ny + j), acc);
    }
  }
  return acc;
}

// restriction at node n of a level that is smoothed next: r = P^T t_f and
// z = w D^-1 r (0 on inactive nodes), so the down-sweep reads z at the
// neighbours instead of forming it from their r and D^-1
template <class T>
__device__ __forceinline__ void mg_restrict_node(const MgLevel &L, const T *__restrict__ tf, int nxf, int nyf,
                                                 double w, bool smoothed, int64_t n) {
  const int I = (int)n / L.ny, J = (int)n - I * L.ny;  // level grids hold < 2^31 nodes
  const double r = mg_restrict(tf, nxf, nyf, I, J);
  L.r[n] = r;
  if (smoothed) L.z[n] = (w * r) * (double)L.dinv[n];
}

// The down- and up-sweep values at node n.  Every load is issued whatever
// the node's kind and the result selected at the end (0 on inactive nodes),
// so no load waits on D^-1: the same numbers as testing D^-1 first.
// down-sweep: t = r - A z with z = w D^-1 r stored by the restriction
__device__ __forceinline__ double mg_smooth_val(const MgLevel &L, int64_t n) {
  const double dn = (double)L.dinv[n];
  const int I = (int)n / L.ny, J = (int)n - I * L.ny;
  auto z = [&](int64_t m) { return L.z[m]; };
  const double t = L.r[n] - mg_apply(L, I, J, z);
  return dn == 0.0 ? 0.0 : t;
}

// up-sweep: y = z + P e_c (0 on inactive nodes), e = y + w D^-1 (r - A y)
__device__ __forceinline__ double mg_post_val(const MgLevel &L, const double *__restrict__ ec, int nyc, double w,
                                              int64_t n) {
  const double dn = (double)L.dinv[n];
  const int I = (int)n / L.ny, J = (int)n - I * L.ny;
  auto y = [&](int64_t m) {
    int i, j;
    mg_nb_ij(n, I, J, m, L.ny, i, j);
    const double v = L.z[m] + mg_prolong(ec, nyc, i, j);
    return L.dinv[m] != 0.0f ? v : 0.0;
  };
  const double yn = y(n);
  const double e = fma(w * dn, L.r[n] - mg_apply(L, I, J, y), yn);
  return dn == 0.0 ? 0.0 : e;
}

__device__ __forceinline__ void mg_smooth_node(const MgLevel &L, int64_t n) { L.t[n] = mg_smooth_val(L, n); }

__device__ __forceinline__ void mg_post_node(const MgLevel &L, const double *__restrict__ ec, int nyc, double w,
                                             int64_t n) {
  L.t[n] = mg_post_val(L, ec, nyc, w, n);
}

// e of level l (the coarsest level's z, else its t)
__host__ __device__ __forceinline__ const double *mg_e(const MgK &M, int l) { return l == M.L - 1 ? M.lv[l].z : M.lv[l].t; }

}  // namespace pic

#endif
