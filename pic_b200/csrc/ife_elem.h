// ife_elem.h -- the Q1 immersed-finite-element interface element: its basis
// from the defining conditions, its element stiffness and its load matrix.
// Compiled for the host (the mesh builder, mesh_build.cpp) and for the
// device (the interface-element kernel of pic_mesh_build_device, ife_dev.cu)
// from this one source, so both produce the same bits (FP64, no fused
// multiply-add: the host with -ffp-contract=off, the device with
// --fmad=false).
//
//   Q1 IFE basis ................... code/IFE-Rectangular/Retangular_reference_basis_IFE.f90,
//                                    code/IFE-Rectangular/retangular_local_basis_IFE.f90
//   element stiffness .............. code/IFE-Rectangular/Generate_stiffness_matrix_local_IFE.f90:104-200,
//                                    code/IFE-Rectangular/Gauss_integration_local_stiffness_IFE.f90
//   load matrix .................... code/IFE-Rectangular/IFE_RHS_2D.f90, Linear_IFE_Basis_Coeff_2D.f90,
//                                    Inter_Tetra_Partition_2D.f90
//
// The basis is obtained by solving its defining 8x8 conditions (nodal values,
// continuity at the two cut points, equal xi*eta coefficients, flux
// continuity across the cut) instead of the reference's closed-form
// expressions; both describe the same unique basis.
#ifndef PIC_IFE_ELEM_H
#define PIC_IFE_ELEM_H

#include <math.h>

#if defined(__CUDACC__)
#define PIC_HD __host__ __device__
#else
#define PIC_HD
#endif

namespace pic {

struct IfeElem {
  int elem = 0;       // 0-based element number
  int type = 0;       // 1 corner cut, 2 opposite edges
  int ref2loc[4];     // 0-based local corner of reference vertex r
  double beta[2];     // beta1 (piece 1, holds reference vertex 1), beta2
  double D[2], E[2];  // cut points (physical)
  double a = 0, b = 0;  // reference coordinates of E (xi) and D (eta or xi)
  double coef[4][2][4];  // [ref basis][piece][c1 c2 c3 c4] in (xi, eta)
  double X[4][2];        // physical coordinates of reference vertices 1..4
};

PIC_HD inline void ife_tri_set(double T[4][3][2], int piece[4], int k, const double *a, const double *b,
                               const double *c, int p) {
  for (int d = 0; d < 2; ++d) { T[k][0][d] = a[d]; T[k][1][d] = b[d]; T[k][2][d] = c[d]; }
  piece[k] = p;
}

PIC_HD inline void ife_rowv(double *M, int r, int blk, const double *P) {
  M[r * 8 + 4 * blk + 0] = 1; M[r * 8 + 4 * blk + 1] = P[0];
  M[r * 8 + 4 * blk + 2] = P[1]; M[r * 8 + 4 * blk + 3] = P[0] * P[1];
}

// Dense Gaussian elimination with partial pivoting (n <= 8); returns false if singular.
PIC_HD inline bool solve_dense(int n, double *M, double *rhs, double *x) {
  double A[64], b[8];
  for (int k = 0; k < n * n; ++k) A[k] = M[k];
  for (int k = 0; k < n; ++k) b[k] = rhs[k];
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r * n + c]) > fabs(A[p * n + c])) p = r;
    if (A[p * n + c] == 0.0) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) {
        const double t = A[c * n + k];
        A[c * n + k] = A[p * n + k];
        A[p * n + k] = t;
      }
      const double t = b[c];
      b[c] = b[p];
      b[p] = t;
    }
    for (int r = c + 1; r < n; ++r) {
      double f = A[r * n + c] / A[c * n + c];
      if (f == 0.0) continue;
      for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = b[r];
    for (int k = r + 1; k < n; ++k) s -= A[r * n + k] * x[k];
    x[r] = s / A[r * n + r];
  }
  return true;
}

// Piece (0 or 1) holding reference vertex r.
PIC_HD inline int piece_of_ref_vertex(int type, int r) {
  if (type == 1) return r == 0 ? 0 : 1;
  return (r == 0 || r == 3) ? 0 : 1;
}

// Reference coordinates of the cut points D and E.
PIC_HD inline void ref_cut_points(const IfeElem &f, double Dref[2], double Eref[2]) {
  if (f.type == 1) {  // E on edge 1-2 (eta = 0), D on edge 1-4 (xi = 0)
    Eref[0] = f.a; Eref[1] = 0;
    Dref[0] = 0; Dref[1] = f.b;
  } else {            // E on edge 1-2 (eta = 0), D on edge 4-3 (eta = 1)
    Eref[0] = f.a; Eref[1] = 0;
    Dref[0] = f.b; Dref[1] = 1;
  }
}

// Solve the defining conditions of the Q1 IFE basis (reference coordinates).
PIC_HD inline bool build_q1_ife_basis(IfeElem &f) {
  double Dr[2], Er[2];
  ref_cut_points(f, Dr, Er);
  double Mx[2] = {0.5 * (Dr[0] + Er[0]), 0.5 * (Dr[1] + Er[1])};
  double n[2] = {Er[1] - Dr[1], Dr[0] - Er[0]};  // normal to DE
  for (int basis = 0; basis < 4; ++basis) {
    double M[64] = {0}, rhs[8] = {0}, sol[8];
    int row = 0;
    for (int v = 0; v < 4; ++v, ++row) {
      int p = piece_of_ref_vertex(f.type, v);
      const double xi = (v == 1 || v == 2) ? 1.0 : 0.0, et = (v >= 2) ? 1.0 : 0.0;  // reference square
      double *R = M + row * 8 + 4 * p;
      R[0] = 1; R[1] = xi; R[2] = et; R[3] = xi * et;
      rhs[row] = (v == basis) ? 1.0 : 0.0;
    }
    for (const double *P : {Dr, Er}) {  // continuity at D and E
      double *R = M + row * 8;
      R[0] = 1; R[1] = P[0]; R[2] = P[1]; R[3] = P[0] * P[1];
      R[4] = -1; R[5] = -P[0]; R[6] = -P[1]; R[7] = -P[0] * P[1];
      ++row;
    }
    {  // equal xi*eta coefficients -> continuity along the whole cut
      double *R = M + row * 8;
      R[3] = 1; R[7] = -1;
      ++row;
    }
    {  // flux continuity beta1 grad p1 . n = beta2 grad p2 . n at the midpoint
      double *R = M + row * 8;
      double b1 = f.beta[0], b2 = f.beta[1];
      R[1] = b1 * n[0]; R[2] = b1 * n[1]; R[3] = b1 * (Mx[1] * n[0] + Mx[0] * n[1]);
      R[5] = -b2 * n[0]; R[6] = -b2 * n[1]; R[7] = -b2 * (Mx[1] * n[0] + Mx[0] * n[1]);
      ++row;
    }
    if (!solve_dense(8, M, rhs, sol)) return false;
    for (int p = 0; p < 2; ++p)
      for (int k = 0; k < 4; ++k) f.coef[basis][p][k] = sol[4 * p + k];
  }
  return true;
}

// Value and physical gradient of reference basis `rb` at physical (x, y) on piece p.
PIC_HD inline void ife_eval(const IfeElem &f, int rb, int p, double x, double y, double *val, double *gx,
              double *gy) {
  const double x1 = f.X[0][0], y1 = f.X[0][1];
  const double x2 = f.X[1][0], y2 = f.X[1][1];
  const double x4 = f.X[3][0], y4 = f.X[3][1];
  double bottom = (x2 - x1) * (y4 - y1) - (x4 - x1) * (y2 - y1);
  double xi = ((y4 - y1) * (x - x1) - (x4 - x1) * (y - y1)) / bottom;
  double et = ((x2 - x1) * (y - y1) - (y2 - y1) * (x - x1)) / bottom;
  const double *c = f.coef[rb][p];
  double r1 = c[1] + c[3] * et, r2 = c[2] + c[3] * xi;
  if (val) *val = c[0] + c[1] * xi + c[2] * et + c[3] * xi * et;
  if (gx) *gx = r1 * (y4 - y1) / bottom + r2 * (y1 - y2) / bottom;
  if (gy) *gy = r1 * (x1 - x4) / bottom + r2 * (x2 - x1) / bottom;
}

// Sub-triangles (physical) and their piece, following the reference's split.
PIC_HD inline int ife_triangles(const IfeElem &f, double T[4][3][2], int piece[4]) {
  const double *V1 = f.X[0], *V2 = f.X[1], *V3 = f.X[2], *V4 = f.X[3];
  if (f.type == 1) {
    ife_tri_set(T, piece, 0, V1, f.D, f.E, 0);
    ife_tri_set(T, piece, 1, V4, f.D, V3, 1);
    ife_tri_set(T, piece, 2, V3, f.D, f.E, 1);
    ife_tri_set(T, piece, 3, V2, V3, f.E, 1);
  } else {
    ife_tri_set(T, piece, 0, V4, V1, f.D, 0);
    ife_tri_set(T, piece, 1, V1, f.D, f.E, 0);
    ife_tri_set(T, piece, 2, V2, f.D, f.E, 1);
    ife_tri_set(T, piece, 3, V3, V2, f.D, 1);
  }
  return 4;
}

PIC_HD inline double tri_area(const double T[3][2]) {
  double ax = T[1][0] - T[0][0], ay = T[1][1] - T[0][1];
  double bx = T[2][0] - T[0][0], by = T[2][1] - T[0][1];
  return fabs(ax * by - ay * bx) * 0.5;
}

// Element stiffness (local HT order) of an interface element: exact 3-point
// edge-midpoint quadrature of the piecewise quadratic integrand.
PIC_HD inline void ife_stiffness(const IfeElem &f, double K[4][4]) {
  for (int j = 0; j < 4; ++j)
    for (int k = 0; k < 4; ++k) K[j][k] = 0;
  double T[4][3][2];
  int piece[4];
  int nt = ife_triangles(f, T, piece);
  for (int t = 0; t < nt; ++t) {
    double A = tri_area(T[t]);
    double beta = f.beta[piece[t]];
    for (int g = 0; g < 3; ++g) {
      double x = 0.5 * (T[t][g][0] + T[t][(g + 1) % 3][0]);
      double y = 0.5 * (T[t][g][1] + T[t][(g + 1) % 3][1]);
      double gx[4], gy[4];
      for (int rb = 0; rb < 4; ++rb) ife_eval(f, rb, piece[t], x, y, nullptr, &gx[rb], &gy[rb]);
      for (int rj = 0; rj < 4; ++rj)
        for (int rk = 0; rk < 4; ++rk)
          K[f.ref2loc[rj]][f.ref2loc[rk]] += A / 3.0 * beta * (gx[rj] * gx[rk] + gy[rj] * gy[rk]);
    }
  }
}

// Axisymmetric (r = y) element stiffness of an interface element: the
// integrand is now cubic, so each sub-triangle takes a collapsed 3x3
// Gauss-Legendre rule (exact to degree 4 on the triangle), in place of the
// reference's nine-point triangle rule (Gauss_integration_local_stiffness_IFE.f90,
// delta == 1 branch): both are exact here, so they agree to rounding.
PIC_HD inline void ife_stiffness_axi(const IfeElem &f, double K[4][4]) {
  for (int j = 0; j < 4; ++j)
    for (int k = 0; k < 4; ++k) K[j][k] = 0;
  double T[4][3][2];
  int piece[4];
  int nt = ife_triangles(f, T, piece);
  const double g = sqrt(0.6);
  const double u[3] = {0.5 * (1.0 - g), 0.5, 0.5 * (1.0 + g)};
  const double w[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
  for (int t = 0; t < nt; ++t) {
    const double A = tri_area(T[t]);
    const double beta = f.beta[piece[t]];
    const double *P0 = T[t][0], *P1 = T[t][1], *P2 = T[t][2];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        // (s, q) in the unit square -> P0 + s (P1 - P0) + s q (P2 - P1), Jacobian 2 A s
        const double sa = u[a], qb = u[b];
        const double x = P0[0] + sa * (P1[0] - P0[0]) + sa * qb * (P2[0] - P1[0]);
        const double y = P0[1] + sa * (P1[1] - P0[1]) + sa * qb * (P2[1] - P1[1]);
        const double wt = w[a] * w[b] * 2.0 * A * sa * y;
        double gx[4], gy[4];
        for (int rb = 0; rb < 4; ++rb) ife_eval(f, rb, piece[t], x, y, nullptr, &gx[rb], &gy[rb]);
        for (int rj = 0; rj < 4; ++rj)
          for (int rk = 0; rk < 4; ++rk)
            K[f.ref2loc[rj]][f.ref2loc[rk]] += wt * beta * (gx[rj] * gx[rk] + gy[rj] * gy[rk]);
      }
  }
}

// Load matrix of an interface element (IFE_RHS_2D.f90) with the reference's
// piecewise-bilinear "linear IFE" interpolation (Linear_IFE_Basis_Coeff_2D.f90),
// its sub-triangles (Inter_Tetra_Partition_2D.f90) and edge-midpoint rule
// (Gauss_Nodes_Elem_2D).  Coordinates are taken relative to reference vertex 1.
PIC_HD inline bool ife_load_matrix(const IfeElem &f, double Mout[16], int axi) {
  double ox = f.X[0][0], oy = f.X[0][1];
  double v[4][2];
  for (int r = 0; r < 4; ++r) { v[r][0] = f.X[r][0] - ox; v[r][1] = f.X[r][1] - oy; }
  double I1[2] = {f.D[0] - ox, f.D[1] - oy}, I2[2] = {f.E[0] - ox, f.E[1] - oy};
  double coef[4][8];
  for (int basis = 0; basis < 4; ++basis) {
    double M[64] = {0}, rhs[8] = {0};
    if (f.type == 2) { ife_rowv(M, 0, 0, v[0]); ife_rowv(M, 3, 0, v[3]); ife_rowv(M, 1, 1, v[1]); ife_rowv(M, 2, 1, v[2]); }
    else { ife_rowv(M, 0, 0, v[0]); ife_rowv(M, 3, 1, v[3]); ife_rowv(M, 1, 1, v[1]); ife_rowv(M, 2, 1, v[2]); }
    double mid[2] = {0.5 * (I1[0] + I2[0]), 0.5 * (I1[1] + I2[1])};
    const double *pts[3] = {I1, I2, mid};
    for (int k = 0; k < 3; ++k) {
      double *R = M + (4 + k) * 8;
      R[0] = 1; R[1] = pts[k][0]; R[2] = pts[k][1]; R[3] = pts[k][0] * pts[k][1];
      R[4] = -1; R[5] = -pts[k][0]; R[6] = -pts[k][1]; R[7] = -pts[k][0] * pts[k][1];
    }
    {
      double *R = M + 7 * 8;
      double b1 = f.beta[0], b2 = f.beta[1];
      double dy = I2[1] - I1[1], dx = I2[0] - I1[0];
      double q = ((I2[1] * I2[1]) - (I1[1] * I1[1]) - (I2[0] * I2[0]) + (I1[0] * I1[0])) * 0.5;
      R[1] = b1 * dy; R[2] = -b1 * dx; R[3] = b1 * q;
      R[5] = -b2 * dy; R[6] = b2 * dx; R[7] = -b2 * q;
    }
    if (f.D[0] == f.E[0] || f.D[1] == f.E[1]) {
      double *R = M + 6 * 8;
      for (int k = 0; k < 8; ++k) R[k] = 0;
      R[3] = 1; R[7] = -1;
    }
    rhs[basis] = 1.0;
    if (!solve_dense(8, M, rhs, coef[basis])) return false;
  }
  // sub-triangles: points 1..4 = reference vertices, 5 = D, 6 = E
  const double *P[6] = {v[0], v[1], v[2], v[3], I1, I2};
  int tri1[4][4] = {{0, 4, 5, 0}, {1, 5, 2, 1}, {5, 2, 4, 1}, {2, 4, 3, 1}};
  int tri2[4][4] = {{0, 5, 3, 0}, {3, 4, 5, 0}, {5, 2, 4, 1}, {2, 5, 1, 1}};
  int (*tri)[4] = (f.type == 1) ? tri1 : tri2;
  for (int k = 0; k < 16; ++k) Mout[k] = 0;
  for (int st = 0; st < 4; ++st) {
    double T[3][2];
    for (int q = 0; q < 3; ++q) { T[q][0] = P[tri[st][q]][0]; T[q][1] = P[tri[st][q]][1]; }
    double V = tri_area(T);
    int reg = tri[st][3];
    for (int g = 0; g < 3; ++g) {
      double x = 0.5 * T[g][0] + 0.5 * T[(g + 1) % 3][0];
      double y = 0.5 * T[g][1] + 0.5 * T[(g + 1) % 3][1];
      double ps[4];
      for (int b = 0; b < 4; ++b) {
        const double *c = coef[b] + 4 * reg;
        ps[b] = c[0] + c[1] * x + c[2] * y + c[3] * x * y;
      }
      // axisymmetric (IFE_RHS_2D.f90:95): the same points, weighted by r = y
      const double rw = axi ? (y + oy) : 1.0;
      for (int rj = 0; rj < 4; ++rj)
        for (int rk = 0; rk < 4; ++rk)
          Mout[f.ref2loc[rj] * 4 + f.ref2loc[rk]] += V * (1.0 / 3.0) * ps[rj] * ps[rk] * rw;
    }
  }
  return true;
}

// Basis, stiffness (axisymmetric when axi) and load matrix of one interface
// element whose geometry (type, ref2loc, beta, D, E, a, b, X) is set.
// Returns 0, 1 for a singular basis system, 2 for a singular load system.
PIC_HD inline int ife_element_all(IfeElem &f, int axi, double K[16], double M[16]) {
  if (!build_q1_ife_basis(f)) return 1;
  double Kl[4][4];
  if (axi) ife_stiffness_axi(f, Kl);
  else ife_stiffness(f, Kl);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) K[4 * a + b] = Kl[a][b];
  if (!ife_load_matrix(f, M, axi)) return 2;
  return 0;
}

}  // namespace pic

#endif
