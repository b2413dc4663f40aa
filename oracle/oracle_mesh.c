/*
 * oracle_mesh.c -- the oracle's own restatement (FP64) of the reference's
 * setup phase: node numbering, object classification, interface-element
 * geometry, the closed-form Q1 IFE basis, element stiffness by the
 * reference's Gauss rules and its assembly into the stiffness CSR and the
 * Dirichlet block, the load matrices of the right-hand side, the dual-cell
 * volumes and the PPR patches.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/ and the CPU-baseline legs of
 * bench.py load it.  It shares no code with libpicgpu's mesh builder (it
 * neither calls nor links it): every array is derived here from the deck,
 * following the reference routine cited beside each step, so that a test
 * can compare the product's descriptor with this one entry by entry.
 *
 * Arithmetic follows the reference as compiled.  Its Gauss weights and
 * points are written as default-kind (REAL(4)) Fortran literals and then
 * stored in REAL(8) arrays (Generate_Gauss_reference.f90,
 * Generate_Gauss_reference_triangle.f90, IFE_RHS_2D.f90 gwght), so they
 * carry single-precision rounding (relative 1e-8).  or_mesh_build(...,
 * quad = OR_QUAD_AS_COMPILED) reproduces those values; OR_QUAD_EXACT uses the
 * same rules with FP64 constants, which isolates the rounding of the
 * constants from everything else when comparing with another builder.
 *
 * Reference paths are relative to PIC-IFE_GEC/ of weqwoueu/pic-.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/picgpu.h"

#define OR_QUAD_AS_COMPILED 0
#define OR_QUAD_EXACT 1

/* IFE_MAIN_PARAM.f90:40 */
#define SMALL 1.0e-12

/* ------------------------------------------------------------------ */
/* Quadrature rules                                                      */
/* ------------------------------------------------------------------ */
typedef struct {
  double w9[9], p9[9][2];     /* rectangle, Generate_Gauss_reference.f90 (9 points) */
  double w4[4], p4[4][2];     /* rectangle, 4 points                                */
  double wt9[9], pt9[9][2];   /* triangle, Generate_Gauss_reference_triangle.f90     */
  double third;               /* IFE_RHS_2D.f90 gwght = 1.0/3.0                      */
} Quad;

/* The constant expressions of the two Fortran routines, evaluated in the
 * literals' kind: float for the as-compiled rules (each operation rounded to
 * single precision, as the compiler folds them), double for the exact ones. */
#define QUAD_RULES(T, SQRT)                                                              \
  do {                                                                                  \
    const T s6 = SQRT((T)0.6), s3 = SQRT((T)3.0), i3 = (T)1.0 / s3;                     \
    const T a9[9] = {(T)64.0 / (T)81.0,   (T)100.0 / (T)324.0, (T)100.0 / (T)324.0,     \
                     (T)100.0 / (T)324.0, (T)100.0 / (T)324.0, (T)40.0 / (T)81.0,       \
                     (T)40.0 / (T)81.0,   (T)40.0 / (T)81.0,   (T)40.0 / (T)81.0};      \
    const T b9[9][2] = {{0, 0}, {s6, s6}, {s6, -s6}, {-s6, s6}, {-s6, -s6},             \
                        {0, s6}, {0, -s6}, {s6, 0}, {-s6, 0}};                           \
    const T b4[4][2] = {{i3, i3}, {i3, -i3}, {-i3, i3}, {-i3, -i3}};                    \
    const T at[9] = {(T)64.0 / (T)81.0 * (T)1 / (T)8.0,                                 \
                     (T)100.0 / (T)324.0 * ((T)1 - s6) / (T)8.0,                        \
                     (T)100.0 / (T)324.0 * ((T)1 - s6) / (T)8.0,                        \
                     (T)100.0 / (T)324.0 * ((T)1 + s6) / (T)8.0,                        \
                     (T)100.0 / (T)324.0 * ((T)1 + s6) / (T)8.0,                        \
                     (T)40.0 / (T)81.0 * (T)1 / (T)8.0,                                 \
                     (T)40.0 / (T)81.0 * (T)1 / (T)8.0,                                 \
                     (T)40.0 / (T)81.0 * ((T)1 - s6) / (T)8.0,                          \
                     (T)40.0 / (T)81.0 * ((T)1 + s6) / (T)8.0};                         \
    const T bt[9][2] = {{((T)1.0 + 0) / (T)2.0, ((T)1.0 - 0) * ((T)1.0 + 0) / (T)4.0},  \
                        {((T)1.0 + s6) / (T)2.0, ((T)1.0 + s6) * ((T)1.0 - s6) / (T)4.0}, \
                        {((T)1.0 + s6) / (T)2.0, ((T)1.0 - s6) * ((T)1.0 - s6) / (T)4.0}, \
                        {((T)1.0 - s6) / (T)2.0, ((T)1.0 + s6) * ((T)1.0 + s6) / (T)4.0}, \
                        {((T)1.0 - s6) / (T)2.0, ((T)1.0 + s6) * ((T)1.0 - s6) / (T)4.0}, \
                        {((T)1.0 + 0) / (T)2.0, ((T)1.0 + s6) / (T)4.0},               \
                        {(T)1.0 / (T)2.0, ((T)1.0 - s6) / (T)4.0},                     \
                        {((T)1.0 + s6) / (T)2.0, ((T)1.0 - s6) / (T)4.0},               \
                        {((T)1.0 - s6) / (T)2.0, ((T)1.0 + s6) / (T)4.0}};              \
    for (int g = 0; g < 9; ++g) {                                                       \
      q->w9[g] = (double)a9[g];                                                         \
      q->p9[g][0] = (double)b9[g][0];                                                   \
      q->p9[g][1] = (double)b9[g][1];                                                   \
      q->wt9[g] = (double)at[g];                                                        \
      q->pt9[g][0] = (double)bt[g][0];                                                  \
      q->pt9[g][1] = (double)bt[g][1];                                                  \
    }                                                                                   \
    for (int g = 0; g < 4; ++g) {                                                       \
      q->w4[g] = 1.0;                                                                   \
      q->p4[g][0] = (double)b4[g][0];                                                   \
      q->p4[g][1] = (double)b4[g][1];                                                   \
    }                                                                                   \
    q->third = (double)((T)1.0 / (T)3.0);                                               \
  } while (0)

static void quad_rules(Quad *q, int mode) {
  if (mode == OR_QUAD_EXACT) QUAD_RULES(double, sqrt);
  else QUAD_RULES(float, sqrtf);
}

/* ------------------------------------------------------------------ */
/* Object geometry                                                       */
/* ------------------------------------------------------------------ */

/* Update_Locate_Node_2D.f90: circle Norm_2 <= R; box within SmallValue;
 * inclined ellipse by its quadratic form, inside when form - 1 < -1e-8. */
static int node_inside(const pic_object *o, double x, double y) {
  if (o->shape == PIC_SHAPE_CIRCLE) {
    double dx = x - o->cx, dy = y - o->cy;
    return sqrt(dx * dx + dy * dy) <= o->a;
  }
  if (o->shape == PIC_SHAPE_BOX)
    return x > o->cx - SMALL && x < o->a + SMALL && y > o->cy - SMALL && y < o->b + SMALL;
  if (o->shape == PIC_SHAPE_ELLIPSE) {
    /* the deck's semi-axis a lies along `angle`: the reference's x_r along
     * its focal direction theta */
    double th = o->angle, xr = o->a, yr = o->b, xc = o->cx, yc = o->cy;
    double c = cos(th), s = sin(th);
    double tA = (c * c) / (xr * xr) + (s * s) / (yr * yr);
    double tB = (1 / (xr * xr) - 1 / (yr * yr)) * sin(2 * th);
    double tC = (s * s) / (xr * xr) + (c * c) / (yr * yr);
    double t = tA * x * x + tB * x * y + tC * y * y - (2 * tA * xc + tB * yc) * x -
               (tB * xc + 2 * tC * yc) * y + (tA * xc * xc + tB * xc * yc + tC * yc * yc);
    return t - 1.0 < -1.0e-8;
  }
  return 0;
}

/* Root classification shared by Line_Circle_Intersection_BL.f90 and
 * Line_Ellipse_Intersection_BL.f90: 1 strictly inside the segment, -1/-2 at
 * an end (the interface through a vertex), 0 outside. */
static int root_flag(double x1, double y1, double x2, double y2, const double R[2], double tol) {
  double rx1 = x1 - R[0], ry1 = y1 - R[1], rx2 = x2 - R[0], ry2 = y2 - R[1];
  double r = rx1 * rx2 + ry1 * ry2;
  if (r < -tol) return 1;
  if (fabs(r) < tol) return (rx1 * rx1 + ry1 * ry1) > (rx2 * rx2 + ry2 * ry2) ? -2 : -1;
  return 0;
}

static int pick_root(int n_root, const double r1[2], const double r2[2], double x1, double y1,
                     double x2, double y2, double tol, double out[2]) {
  int f1 = 0, f2 = 0;
  if (n_root) {
    f1 = root_flag(x1, y1, x2, y2, r1, tol);
    f2 = root_flag(x1, y1, x2, y2, r2, tol);
  }
  if (f1 != 0 && f2 == 0) { out[0] = r1[0]; out[1] = r1[1]; return f1; }
  if (f1 == 0 && f2 != 0) { out[0] = r2[0]; out[1] = r2[1]; return f2; }
  if ((f1 == -1 && f2 == -1) || (f1 == -2 && f2 == -2)) { out[0] = r1[0]; out[1] = r1[1]; return f1; }
  return 0;
}

/* Intersection of the element edge (x1,y1)-(x2,y2) (axis-aligned) with the
 * object's boundary: Line_Circle_Intersection_BL.f90,
 * Line_Ellipse_Intersection_BL.f90 (inclined branch),
 * Line_Rectangular_Intersection_BL.f90.  Returns the flag (1 = a crossing
 * inside the edge). */
static int edge_object(const pic_object *o, double x1, double y1, double x2, double y2, double P[2]) {
  double r1[2] = {0, 0}, r2[2] = {0, 0};
  int n_root = 0;
  P[0] = P[1] = 0;
  if (o->shape == PIC_SHAPE_CIRCLE) {
    double r = o->a, xc = o->cx, yc = o->cy;
    if (fabs(x1 - x2) < SMALL) {
      double dl = r * r - (x1 - xc) * (x1 - xc);
      if (dl > SMALL) { n_root = 2; r1[0] = x1; r1[1] = yc + sqrt(dl); r2[0] = x1; r2[1] = yc - sqrt(dl); }
      else if (fabs(dl) < SMALL) { n_root = 1; r1[0] = r2[0] = x1; r1[1] = r2[1] = yc; }
    }
    if (x1 != x2 && fabs(y1 - y2) < SMALL) {
      double dl = r * r - (y1 - yc) * (y1 - yc);
      if (dl > SMALL) { n_root = 2; r1[0] = xc + sqrt(dl); r1[1] = y1; r2[0] = xc - sqrt(dl); r2[1] = y1; }
      else if (fabs(dl) < SMALL) { n_root = 1; r1[0] = r2[0] = xc; r1[1] = r2[1] = y1; }
    }
    return pick_root(n_root, r1, r2, x1, y1, x2, y2, SMALL, P);
  }
  if (o->shape == PIC_SHAPE_ELLIPSE) {
    double th = o->angle, xr = o->a, yr = o->b, xc = o->cx, yc = o->cy;
    double c = cos(th), s = sin(th);
    double tA = (c * c) / (xr * xr) + (s * s) / (yr * yr);
    double tB = (1 / (xr * xr) - 1 / (yr * yr)) * sin(2 * th);
    double tC = (s * s) / (xr * xr) + (c * c) / (yr * yr);
    if (fabs(x1 - x2) < 1.0e-8) { /* vertical edge: solve for y */
      double dA = tC, dB = tB * x1 - tB * xc - 2 * tC * yc;
      double dC = tA * x1 * x1 - (2 * tA * xc + tB * yc) * x1 + (tA * xc * xc + tB * xc * yc + tC * yc * yc - 1);
      double dl = dB * dB - 4 * dA * dC;
      if (dl > 1.0e-8) {
        n_root = 2;
        r1[0] = x1; r1[1] = (-dB + sqrt(dl)) / (2 * dA);
        r2[0] = x1; r2[1] = (-dB - sqrt(dl)) / (2 * dA);
      } else if (fabs(dl) < 1.0e-8) {
        n_root = 1; r1[0] = r2[0] = x1; r1[1] = r2[1] = -dB / (2 * dA);
      }
    }
    if (x1 != x2 && fabs(y1 - y2) < 1.0e-8) { /* horizontal edge: solve for x */
      double dA = tA, dB = tB * y1 - tB * yc - 2 * tA * xc;
      double dC = tC * y1 * y1 - (2 * tC * yc + tB * xc) * y1 + (tA * xc * xc + tB * xc * yc + tC * yc * yc - 1);
      double dl = dB * dB - 4 * dA * dC;
      if (dl > 1.0e-8) {
        n_root = 2;
        r1[0] = (-dB + sqrt(dl)) / (2 * dA); r1[1] = y1;
        r2[0] = (-dB - sqrt(dl)) / (2 * dA); r2[1] = y1;
      } else if (fabs(dl) < 1.0e-8) {
        n_root = 1; r1[0] = r2[0] = -dB / (2 * dA); r1[1] = r2[1] = y1;
      }
    }
    return pick_root(n_root, r1, r2, x1, y1, x2, y2, 1.0e-8, P);
  }
  if (o->shape == PIC_SHAPE_BOX) {
    double oxn = o->cx, oxx = o->a, oyn = o->cy, oyx = o->b;
    int flag = 0;
    if (fabs(y1 - y2) < SMALL) {
      double xn = fmin(x1, x2), xx = fmax(x1, x2);
      if (!(y1 - oyn < -SMALL || y1 - oyx > SMALL)) {
        if (xn - oxn < -SMALL) { P[0] = oxn; P[1] = y1; flag = 1; }
        else if (xx - oxx > SMALL) { P[0] = oxx; P[1] = y1; flag = 1; }
      }
    }
    if (fabs(x1 - x2) < SMALL) {
      double yn = fmin(y1, y2), yx = fmax(y1, y2);
      if (!(x1 - oxn < -SMALL || x1 - oxx > SMALL)) {
        if (yn - oyn < -SMALL) { P[0] = x1; P[1] = oyn; flag = 1; }
        else if (yx - oyx > SMALL) { P[0] = x1; P[1] = oyx; flag = 1; }
      }
    }
    return flag;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Interface element information (El_Object_Intersection_info_2D_BL.f90: */
/* the case table on the four corners' labels, generic cases: no vertex  */
/* on the interface)                                                     */
/* ------------------------------------------------------------------ */
typedef struct {
  int elem;        /* 0-based element                                 */
  int type;        /* information_1(6): 1 corner cut, 2 opposite edges */
  int r2l[4];      /* information_1(11:14) pointer_reference_to_local, 0-based */
  int l2r[4];      /* information_1(7:10) pointer_local_to_reference, 0-based  */
  double beta1, beta2, D[2], E[2];
} OrIfe;

/* Case table, inside mask bit c set when local corner c+1 is inside:
 * element type, first reference vertex (local, 0-based), local edge of D and
 * of E (edge c runs from corner c to c+1), and whether beta1 is the inside
 * value.  Rows follow the reference's IF chain; the saddle masks 5 and 10
 * have no row there. */
static const struct { int type, r1, eD, eE, in1; } kCase[16] = {
    {0, 0, 0, 0, 0},  /* 0000 */
    {1, 0, 3, 0, 1},  /* I O O O */
    {1, 1, 0, 1, 1},  /* O I O O */
    {2, 3, 1, 3, 0},  /* I I O O */
    {1, 2, 1, 2, 1},  /* O O I O */
    {0, 0, 0, 0, 0},  /* I O I O saddle */
    {2, 0, 2, 0, 0},  /* O I I O */
    {1, 3, 2, 3, 0},  /* I I I O */
    {1, 3, 2, 3, 1},  /* O O O I */
    {2, 0, 2, 0, 1},  /* I O O I */
    {0, 0, 0, 0, 0},  /* O I O I saddle */
    {1, 2, 1, 2, 0},  /* I I O I */
    {2, 3, 1, 3, 1},  /* O O I I */
    {1, 1, 0, 1, 0},  /* I O I I */
    {1, 0, 3, 0, 0},  /* O I I I */
    {0, 0, 0, 0, 0},  /* 1111 */
};

/* ------------------------------------------------------------------ */
/* Closed-form Q1 IFE reference basis, Retangular_reference_basis_IFE.f90 */
/* (basis_type 1), coefficient tensor k11, k12, k21, k22 from             */
/* Function_coefficient_2D (1, 0, 0, 1 in the explicit step).  bi 1..4,   */
/* pf (piece) 1..2.  C = C1..C4 of C1 + C2 xi + C3 eta + C4 xi eta.        */
/* ------------------------------------------------------------------ */
static void ife_ref_coef(int typ, int bi, int pf, double a, double b, double R, double C[4]) {
  const double k11 = 0.0 + 1.0, k12 = 0.0 + 0.0, k21 = 0.0 + 0.0, k22 = 0.0 + 1.0;
  const double a2 = a * a, b2 = b * b, a3 = a * a * a, b3 = b * b * b;
  double C1 = 0, C2 = 0, C3 = 0, C4 = 0, bot;
  if (typ == 1) {
    bot = 2 * R * a2 * k22 - a2 * b2 * k21 - a2 * b2 * k12 + 2 * R * b2 * k11 + 2 * a * b2 * k11 + 2 * a * b2 * k12 -
          a * b3 * k11 + 2 * a2 * b * k21 + 2 * a2 * b * k22 - a3 * b * k22 - 2 * R * a * b2 * k11 -
          2 * R * a * b2 * k12 + R * a * b3 * k11 - 2 * R * a2 * b * k21 - 2 * R * a2 * b * k22 + R * a3 * b * k22 +
          R * a2 * b2 * k12 + R * a2 * b2 * k21 + 2 * R * a * b * k12 + 2 * R * a * b * k21;
    if (bi == 1) {
      if (pf == 1) {
        C1 = 1;
        C2 = (b3 * k11 - 2 * b2 * k12 - 2 * b2 * k11 - 2 * a * b * k21 - 2 * a * b * k22 - 2 * R * a2 * k22 +
              2 * R * b2 * k12 - R * b3 * k11 + a * b2 * k12 + a * b2 * k21 + a2 * b * k22 - R * a * b2 * k12 -
              R * a * b2 * k21 - R * a2 * b * k22 - 2 * R * a * b * k12 + 2 * R * a * b * k22) / bot;
        C3 = (a3 * k22 - 2 * a2 * k22 - 2 * a2 * k21 - 2 * a * b * k11 - 2 * a * b * k12 + 2 * R * a2 * k21 -
              R * a3 * k22 - 2 * R * b2 * k11 + a * b2 * k11 + a2 * b * k12 + a2 * b * k21 - R * a * b2 * k11 -
              R * a2 * b * k12 - R * a2 * b * k21 + 2 * R * a * b * k11 - 2 * R * a * b * k21) / bot;
        C4 = 2 * R * (a2 * k22 + b2 * k11 + a * b * k12 + a * b * k21) / bot;
      } else {
        C1 = 2 * R * (a2 * k22 + b2 * k11 + a * b * k12 + a * b * k21) / bot;
        C2 = -C1; C3 = -C1; C4 = C1;
      }
    } else if (bi == 2) {
      if (pf == 1) {
        C1 = 0;
        C2 = (2 * b2 * k11 - b3 * k11 + 2 * a * b * k21 + 2 * R * a2 * k22 + R * b3 * k11 + a * b2 * k12 -
              a * b2 * k21 + a2 * b * k22 - R * a * b2 * k12 + R * a * b2 * k21 - R * a2 * b * k22 +
              2 * R * a * b * k12) / bot;
        C3 = (2 * a2 * k21 - a3 * k22 + a2 * b2 * k12 + a2 * b2 * k21 + 2 * a * b * k11 - 2 * R * a2 * k21 +
              R * a3 * k22 - 3 * a * b2 * k11 + a * b3 * k11 - a2 * b * k12 - 3 * a2 * b * k21 + a3 * b * k22 +
              3 * R * a * b2 * k11 - R * a * b3 * k11 + R * a2 * b * k12 + 3 * R * a2 * b * k21 - R * a3 * b * k22 -
              R * a2 * b2 * k12 - R * a2 * b2 * k21 - 2 * R * a * b * k11) / bot;
        C4 = (2 * R * a * b2 * k12 - 2 * R * b2 * k11 - 2 * a * b2 * k12 - 2 * a2 * b * k22 - 2 * R * a2 * k22 +
              2 * R * a2 * b * k22 - 2 * R * a * b * k12 - 2 * R * a * b * k21) / bot;
      } else {
        C1 = (2 * a * b2 * k11 - a2 * b2 * k21 - a2 * b2 * k12 - a * b3 * k11 + 2 * a2 * b * k21 - a3 * b * k22 -
              2 * R * a * b2 * k11 + R * a * b3 * k11 - 2 * R * a2 * b * k21 + R * a3 * b * k22 + R * a2 * b2 * k12 +
              R * a2 * b2 * k21) / bot;
        C2 = 1 - C1; C3 = -C1; C4 = C1 - 1;
      }
    } else if (bi == 3) {
      if (pf == 1) {
        C1 = 0;
        C2 = (b3 * k11 - a2 * b2 * k12 - a2 * b2 * k21 - R * b3 * k11 + a * b2 * k12 - a * b3 * k11 +
              a * b2 * k21 + a2 * b * k22 - a3 * b * k22 - R * a * b2 * k12 + R * a * b3 * k11 - R * a * b2 * k21 -
              R * a2 * b * k22 + R * a3 * b * k22 + R * a2 * b2 * k12 + R * a2 * b2 * k21) / bot;
        C3 = (a3 * k22 - a2 * b2 * k12 - a2 * b2 * k21 - R * a3 * k22 + a * b2 * k11 - a * b3 * k11 +
              a2 * b * k12 + a2 * b * k21 - a3 * b * k22 - R * a * b2 * k11 + R * a * b3 * k11 - R * a2 * b * k12 -
              R * a2 * b * k21 + R * a3 * b * k22 + R * a2 * b2 * k12 + R * a2 * b2 * k21) / bot;
        C4 = (2 * R * a2 * k22 + 2 * R * b2 * k11 + 2 * a * b2 * k11 + 2 * a * b2 * k12 + 2 * a2 * b * k21 +
              2 * a2 * b * k22 - 2 * R * a * b2 * k11 - 2 * R * a * b2 * k12 - 2 * R * a2 * b * k21 -
              2 * R * a2 * b * k22 + 2 * R * a * b * k12 + 2 * R * a * b * k21) / bot;
      } else {
        C1 = (a2 * b2 * k12 + a2 * b2 * k21 + a * b3 * k11 + a3 * b * k22 - R * a * b3 * k11 - R * a3 * b * k22 -
              R * a2 * b2 * k12 - R * a2 * b2 * k21) / bot;
        C2 = -C1; C3 = -C1; C4 = 1 + C1;
      }
    } else {
      if (pf == 1) {
        C1 = 0;
        C2 = (2 * b2 * k12 - b3 * k11 + a2 * b2 * k12 + a2 * b2 * k21 + 2 * a * b * k22 - 2 * R * b2 * k12 +
              R * b3 * k11 - 3 * a * b2 * k12 + a * b3 * k11 - a * b2 * k21 - 3 * a2 * b * k22 + a3 * b * k22 +
              3 * R * a * b2 * k12 - R * a * b3 * k11 + R * a * b2 * k21 + 3 * R * a2 * b * k22 - R * a3 * b * k22 -
              R * a2 * b2 * k12 - R * a2 * b2 * k21 - 2 * R * a * b * k22) / bot;
        C3 = (2 * a2 * k22 - a3 * k22 + 2 * a * b * k12 + R * a3 * k22 + 2 * R * b2 * k11 + a * b2 * k11 -
              a2 * b * k12 + a2 * b * k21 - R * a * b2 * k11 + R * a2 * b * k12 - R * a2 * b * k21 +
              2 * R * a * b * k21) / bot;
        C4 = (2 * R * a * b2 * k11 - 2 * R * b2 * k11 - 2 * a * b2 * k11 - 2 * a2 * b * k21 - 2 * R * a2 * k22 +
              2 * R * a2 * b * k21 - 2 * R * a * b * k12 - 2 * R * a * b * k21) / bot;
      } else {
        C1 = (2 * a * b2 * k12 - a2 * b2 * k21 - a2 * b2 * k12 - a * b3 * k11 + 2 * a2 * b * k22 - a3 * b * k22 -
              2 * R * a * b2 * k12 + R * a * b3 * k11 - 2 * R * a2 * b * k22 + R * a3 * b * k22 + R * a2 * b2 * k12 +
              R * a2 * b2 * k21) / bot;
        C2 = -C1; C3 = 1 - C1; C4 = C1 - 1;
      }
    }
  } else {
    bot = 2 * R * k11 + a * k11 + 2 * a * k12 + b * k11 - 2 * b * k12 - a2 * k12 + a2 * k21 + 2 * a2 * k22 -
          a3 * k22 + b2 * k12 - b2 * k21 + 2 * b2 * k22 - b3 * k22 - R * a * k11 + 2 * R * a * k21 - R * b * k11 -
          2 * R * b * k21 - 4 * a * b * k22 + R * a2 * k12 - R * a2 * k21 + R * a3 * k22 - R * b2 * k12 +
          R * b2 * k21 + R * b3 * k22 + a * b2 * k22 + a2 * b * k22 - R * a * b2 * k22 - R * a2 * b * k22;
    if (bi == 1) {
      if (pf == 1) {
        C1 = 1;
        C2 = (2 * R * k12 - 2 * k12 - R * k11 - k11 + a * k12 - a * k21 - 2 * a * k22 - b * k11 + 3 * b * k12 +
              b * k21 + 2 * b * k22 + a2 * k22 - b2 * k12 + b2 * k21 - 3 * b2 * k22 + b3 * k22 - 3 * R * a * k12 -
              R * a * k21 + 2 * R * a * k22 + R * b * k11 - R * b * k12 + R * b * k21 - 2 * R * b * k22 -
              a * b * k12 - a * b * k21 + 2 * a * b * k22 - 3 * R * a2 * k22 + R * b2 * k12 - R * b2 * k21 +
              R * b2 * k22 - R * b3 * k22 - a2 * b * k22 + R * a2 * b * k22 + R * a * b * k12 + R * a * b * k21 +
              2 * R * a * b * k22) / bot;
        C3 = -1;
        C4 = (2 * R * k11 + 2 * b * k11 - 2 * b2 * k21 + 2 * R * a * k12 + 2 * R * a * k21 - 2 * R * b * k11 -
              2 * R * b * k12 - 2 * R * b * k21 + 2 * a * b * k21 + 2 * R * a2 * k22 + 2 * R * b2 * k21 +
              2 * R * b2 * k22 - 2 * R * a * b * k21 - 4 * R * a * b * k22) / bot;
      } else {
        C1 = (2 * R * k11 + b * k11 - 2 * b * k12 + b2 * k12 - b2 * k21 + 2 * b2 * k22 - b3 * k22 +
              2 * R * a * k12 + 2 * R * a * k21 - R * b * k11 - 2 * R * b * k21 + a * b * k12 + a * b * k21 -
              2 * a * b * k22 + 2 * R * a2 * k22 - R * b2 * k12 + R * b2 * k21 + R * b3 * k22 + a2 * b * k22 -
              R * a2 * b * k22 - R * a * b * k12 - R * a * b * k21 - 2 * R * a * b * k22) / bot;
        C2 = -C1;
        C3 = (2 * b2 * k21 - 2 * b * k11 - 2 * R * k11 - 2 * R * a * k12 - 2 * R * a * k21 + 2 * R * b * k11 +
              2 * R * b * k12 + 2 * R * b * k21 - 2 * a * b * k21 - 2 * R * a2 * k22 - 2 * R * b2 * k21 -
              2 * R * b2 * k22 + 2 * R * a * b * k21 + 4 * R * a * b * k22) / bot;
        C4 = -C3;
      }
    } else if (bi == 2) {
      if (pf == 1) {
        C1 = 0;
        C2 = (k11 + R * k11 + a * k12 + a * k21 + b * k11 - 3 * b * k12 - b * k21 + a2 * k22 + b2 * k12 -
              b2 * k21 + 3 * b2 * k22 - b3 * k22 + R * a * k12 + R * a * k21 - R * b * k11 + R * b * k12 -
              R * b * k21 + a * b * k12 + a * b * k21 - 4 * a * b * k22 + R * a2 * k22 - R * b2 * k12 +
              R * b2 * k21 - R * b2 * k22 + R * b3 * k22 + a2 * b * k22 - R * a2 * b * k22 - R * a * b * k12 -
              R * a * b * k21) / bot;
        C3 = 0;
        C4 = (2 * b * k12 - 2 * a * k12 - 2 * b * k11 - 2 * R * k11 - 2 * a2 * k22 + 2 * b2 * k21 - 2 * b2 * k22 -
              2 * R * a * k21 + 2 * R * b * k11 + 2 * R * b * k21 - 2 * a * b * k21 + 4 * a * b * k22 -
              2 * R * b2 * k21 + 2 * R * a * b * k21) / bot;
      } else {
        C1 = (a * k11 - a2 * k12 + a2 * k21 - a3 * k22 - R * a * k11 - a * b * k12 - a * b * k21 + R * a2 * k12 -
              R * a2 * k21 + R * a3 * k22 + a * b2 * k22 - R * a * b2 * k22 + R * a * b * k12 + R * a * b * k21) /
             bot;
        C2 = 1 - C1;
        C3 = (b * k11 - a * k11 + a2 * k12 - a2 * k21 + a3 * k22 - b2 * k12 - b2 * k21 + b3 * k22 + R * a * k11 -
              R * b * k11 + 2 * a * b * k21 - R * a2 * k12 + R * a2 * k21 - R * a3 * k22 + R * b2 * k12 +
              R * b2 * k21 - R * b3 * k22 - a * b2 * k22 - a2 * b * k22 + R * a * b2 * k22 + R * a2 * b * k22 -
              2 * R * a * b * k21) / bot;
        C4 = -C3 - 1;
      }
    } else if (bi == 3) {
      if (pf == 1) {
        C1 = 0;
        C2 = (k11 - R * k11 - a * k11 + a * k12 + a * k21 + b * k12 - b * k21 - a2 * k12 - a2 * k21 + a2 * k22 -
              a3 * k22 - b2 * k22 + R * a * k11 - R * a * k12 - R * a * k21 - R * b * k12 + R * b * k21 -
              a * b * k12 + a * b * k21 + R * a2 * k12 + R * a2 * k21 - R * a2 * k22 + R * a3 * k22 +
              R * b2 * k22 + a * b2 * k22 - R * a * b2 * k22 + R * a * b * k12 - R * a * b * k21) / bot;
        C3 = 0;
        C4 = (2 * R * k11 + 2 * a * k11 + 2 * a * k12 - 2 * b * k12 + 2 * a2 * k21 + 2 * a2 * k22 + 2 * b2 * k22 -
              2 * R * a * k11 + 2 * R * a * k21 - 2 * R * b * k21 - 2 * a * b * k21 - 4 * a * b * k22 -
              2 * R * a2 * k21 + 2 * R * a * b * k21) / bot;
      } else {
        C1 = a * (k11 - R * k11 + a * k12 + a * k21 + b * k12 - b * k21 + a2 * k22 - b2 * k22 - R * a * k12 -
                  R * a * k21 - R * b * k12 + R * b * k21 - R * a2 * k22 + R * b2 * k22) / bot;
        C2 = -C1;
        C3 = (b * k11 - a * k11 - a2 * k12 - a2 * k21 - a3 * k22 + b2 * k12 - b2 * k21 - b3 * k22 + R * a * k11 -
              R * b * k11 + 2 * a * b * k21 + R * a2 * k12 + R * a2 * k21 + R * a3 * k22 - R * b2 * k12 +
              R * b2 * k21 + R * b3 * k22 + a * b2 * k22 + a2 * b * k22 - R * a * b2 * k22 - R * a2 * b * k22 -
              2 * R * a * b * k21) / bot;
        C4 = 1 - C3;
      }
    } else {
      if (pf == 1) {
        C1 = 0;
        C2 = (2 * k12 - k11 + R * k11 - 2 * R * k12 + a * k11 - 3 * a * k12 - a * k21 + 2 * a * k22 - b * k12 +
              b * k21 - 2 * b * k22 + a2 * k12 + a2 * k21 - 3 * a2 * k22 + a3 * k22 + b2 * k22 - R * a * k11 +
              3 * R * a * k12 + R * a * k21 - 2 * R * a * k22 + R * b * k12 - R * b * k21 + 2 * R * b * k22 +
              a * b * k12 - a * b * k21 + 2 * a * b * k22 - R * a2 * k12 - R * a2 * k21 + 3 * R * a2 * k22 -
              R * a3 * k22 - R * b2 * k22 - a * b2 * k22 + R * a * b2 * k22 - R * a * b * k12 + R * a * b * k21 -
              2 * R * a * b * k22) / bot;
        C3 = 1;
        C4 = (2 * R * a * k11 - 2 * a * k11 - 2 * a2 * k21 - 2 * R * k11 - 2 * R * a * k12 - 2 * R * a * k21 +
              2 * R * b * k12 + 2 * R * b * k21 + 2 * a * b * k21 + 2 * R * a2 * k21 - 2 * R * a2 * k22 -
              2 * R * b2 * k22 - 2 * R * a * b * k21 + 4 * R * a * b * k22) / bot;
      } else {
        C1 = -a * (k11 - 2 * k12 - R * k11 + 2 * R * k12 + a * k12 + a * k21 - 2 * a * k22 + b * k12 - b * k21 +
                   2 * b * k22 + a2 * k22 - b2 * k22 - R * a * k12 - R * a * k21 + 2 * R * a * k22 - R * b * k12 +
                   R * b * k21 - 2 * R * b * k22 - R * a2 * k22 + R * b2 * k22) / bot;
        C2 = -C1;
        C3 = (2 * R * k11 + 2 * a * k11 + 2 * a2 * k21 - 2 * R * a * k11 + 2 * R * a * k12 + 2 * R * a * k21 -
              2 * R * b * k12 - 2 * R * b * k21 - 2 * a * b * k21 - 2 * R * a2 * k21 + 2 * R * a2 * k22 +
              2 * R * b2 * k22 + 2 * R * a * b * k21 - 4 * R * a * b * k22) / bot;
        C4 = -C3;
      }
    }
  }
  C[0] = C1; C[1] = C2; C[2] = C3; C[3] = C4;
}

/* Retangular_local_basis_IFE.f90: derivative (dx = 1: d/dx, else d/dy) of
 * LOCAL basis j on piece pf at physical (x, y). */
static double ife_local_deriv(const OrIfe *f, const double V[4][2], int j, int pf, double x, double y,
                              int dx) {
  const double x1 = V[f->r2l[0]][0], y1 = V[f->r2l[0]][1];
  const double x2 = V[f->r2l[1]][0], y2 = V[f->r2l[1]][1];
  const double x4 = V[f->r2l[3]][0], y4 = V[f->r2l[3]][1];
  const double bottom = (x2 - x1) * (y4 - y1) - (x4 - x1) * (y2 - y1);
  const double ks = ((y4 - y1) * (x - x1) - (x4 - x1) * (y - y1)) / bottom;
  const double et = ((x2 - x1) * (y - y1) - (y2 - y1) * (x - x1)) / bottom;
  double a, b;
  a = ((y4 - y1) * (f->E[0] - x1) - (x4 - x1) * (f->E[1] - y1)) / bottom;
  if (f->type == 1) b = ((x2 - x1) * (f->D[1] - y1) - (y2 - y1) * (f->D[0] - x1)) / bottom;
  else b = ((y4 - y1) * (f->D[0] - x1) - (x4 - x1) * (f->D[1] - y1)) / bottom;
  double C[4];
  ife_ref_coef(f->type, f->l2r[j] + 1, pf, a, b, f->beta1 / f->beta2, C);
  const double r1 = C[1] + C[3] * et, r2 = C[2] + C[3] * ks;
  if (dx) return r1 * (y4 - y1) / bottom + r2 * (y1 - y2) / bottom;
  return r1 * (x1 - x4) / bottom + r2 * (x2 - x1) / bottom;
}

/* Gauss_integration_local_stiffness_IFE.f90: one entry (trial j, test k)
 * of the xx (dx = 1) or yy part; four sub-triangles, nine points each. */
static double ife_stiff_entry(const OrIfe *f, const double V[4][2], const Quad *q, int j, int k, int dx,
                              int delta) {
  const double *P1 = V[f->r2l[0]], *P2 = V[f->r2l[1]], *P3 = V[f->r2l[2]], *P4 = V[f->r2l[3]];
  const double *T[4][3];
  int pf[4];
  if (f->type == 1) {
    T[0][0] = P1; T[0][1] = f->D; T[0][2] = f->E; pf[0] = 1;
    T[1][0] = P4; T[1][1] = f->D; T[1][2] = P3; pf[1] = 2;
    T[2][0] = P3; T[2][1] = f->D; T[2][2] = f->E; pf[2] = 2;
    T[3][0] = P2; T[3][1] = P3; T[3][2] = f->E; pf[3] = 2;
  } else {
    T[0][0] = P4; T[0][1] = P1; T[0][2] = f->D; pf[0] = 1;
    T[1][0] = P1; T[1][1] = f->D; T[1][2] = f->E; pf[1] = 1;
    T[2][0] = P2; T[2][1] = f->D; T[2][2] = f->E; pf[2] = 2;
    T[3][0] = P3; T[3][1] = P2; T[3][2] = f->D; pf[3] = 2;
  }
  double r = 0;
  for (int t = 0; t < 4; ++t) {
    /* Generate_Gauss_local_triangle.f90 */
    const double x1 = T[t][0][0], y1 = T[t][0][1], x2 = T[t][1][0], y2 = T[t][1][1];
    const double x3 = T[t][2][0], y3 = T[t][2][1];
    const double jac = fabs((x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1));
    const double beta = pf[t] == 1 ? f->beta1 : f->beta2;
    const double coef = 0.0 + beta; /* Function_coefficient_2D: Chi_p (0) + beta */
    for (int g = 0; g < 9; ++g) {
      const double w = q->wt9[g] * jac;
      const double gx = x1 + (x2 - x1) * q->pt9[g][0] + (x3 - x1) * q->pt9[g][1];
      const double gy = y1 + (y2 - y1) * q->pt9[g][0] + (y3 - y1) * q->pt9[g][1];
      const double r1 = ife_local_deriv(f, V, j, pf[t], gx, gy, dx);
      const double r2 = ife_local_deriv(f, V, k, pf[t], gx, gy, dx);
      if (delta == 0) r = r + w * coef * r1 * r2;
      else r = r + w * coef * r1 * r2 * gy;
    }
  }
  return r;
}

/* Retangular_reference_basis.f90 (basis_type 1) first derivatives and
 * Retangular_local_basis.f90's chain rule. */
static double q1_deriv(int j, double x, double y, double x0, double y0, double h1, double h2, int dx) {
  const double ks = (2 * x - 2 * x0 - h1) / h1, et = (2 * y - 2 * y0 - h2) / h2;
  double r;
  if (dx) {
    r = (j == 0) ? (-1 + et) / 4 : (j == 1) ? (1 - et) / 4 : (j == 2) ? (1 + et) / 4 : (-1 - et) / 4;
    return r * 2 / h1;
  }
  r = (j == 0) ? (-1 + ks) / 4 : (j == 1) ? (-1 - ks) / 4 : (j == 2) ? (1 + ks) / 4 : (1 - ks) / 4;
  return r * 2 / h2;
}

/* Gauss_integration_local_stiffness.f90 with Generate_Gauss_local.f90's
 * nine-point rule: one entry of the xx or yy part of a regular element. */
static double q1_stiff_entry(const Quad *q, double x0, double y0, double h1, double h2, double beta, int j,
                             int k, int dx, int delta) {
  const double jac = h1 * h2 / 4;
  double r = 0;
  for (int g = 0; g < 9; ++g) {
    const double w = q->w9[g] * jac;
    const double gx = h1 * q->p9[g][0] / 2. + x0 + h1 / 2.;
    const double gy = h2 * q->p9[g][1] / 2. + y0 + h2 / 2.;
    const double t1 = q1_deriv(j, gx, gy, x0, y0, h1, h2, dx);
    const double t2 = q1_deriv(k, gx, gy, x0, y0, h1, h2, dx);
    const double coef = 0.0 + beta;
    if (delta == 0) r = r + w * coef * t1 * t2;
    else r = r + w * coef * t1 * t2 * gy;
  }
  return r;
}

/* AGAUS.f90: Gauss elimination with full pivoting; its pivot magnitude D is
 * an implicitly typed REAL(4), so the search compares against the pivot
 * rounded to single precision.  Returns 0 when singular. */
static int agaus(double *A, double *B, int n, double *X) {
  int js[8];
  for (int k = 0; k < n - 1; ++k) {
    float d = 0.0f;
    int is = k;
    js[k] = k;
    for (int i = k; i < n; ++i)
      for (int j = k; j < n; ++j)
        if (fabs(A[i * n + j]) > (double)d) {
          d = (float)fabs(A[i * n + j]);
          js[k] = j;
          is = i;
        }
    if (d + 1.0f == 1.0f) return 0;
    if (js[k] != k)
      for (int i = 0; i < n; ++i) {
        double t = A[i * n + k]; A[i * n + k] = A[i * n + js[k]]; A[i * n + js[k]] = t;
      }
    if (is != k) {
      for (int j = k; j < n; ++j) {
        double t = A[k * n + j]; A[k * n + j] = A[is * n + j]; A[is * n + j] = t;
      }
      double t = B[k]; B[k] = B[is]; B[is] = t;
    }
    for (int j = k + 1; j < n; ++j) A[k * n + j] = A[k * n + j] / A[k * n + k];
    B[k] = B[k] / A[k * n + k];
    for (int i = k + 1; i < n; ++i) {
      for (int j = k + 1; j < n; ++j) A[i * n + j] = A[i * n + j] - A[i * n + k] * A[k * n + j];
      B[i] = B[i] - A[i * n + k] * B[k];
    }
  }
  if (fabs(A[(n - 1) * n + n - 1]) + 1.0f == 1.0f) return 0;
  X[n - 1] = B[n - 1] / A[(n - 1) * n + n - 1];
  for (int i = n - 2; i >= 0; --i) {
    double t = 0.0;
    for (int j = i + 1; j < n; ++j) t = t + A[i * n + j] * X[j];
    X[i] = B[i] - t;
  }
  js[n - 1] = n - 1;
  for (int k = n - 1; k >= 0; --k)
    if (js[k] != k) { double t = X[k]; X[k] = X[js[k]]; X[js[k]] = t; }
  return 1;
}

/* Linear_FE_Basis_Coeff_2D.f90 + FE_RHS_HW_2D.f90 with the four-point rule:
 * the load matrix of a regular element (row i, column k), r-weighted when
 * delta = 1. */
static int q1_load(const Quad *q, const double V[4][2], double h1, double h2, int delta, double M[16]) {
  double coef[4][4];
  for (int bi = 0; bi < 4; ++bi) {
    double A[16], rhs[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
      A[i * 4 + 0] = 1.0; A[i * 4 + 1] = V[i][0]; A[i * 4 + 2] = V[i][1]; A[i * 4 + 3] = V[i][0] * V[i][1];
    }
    rhs[bi] = 1.0;
    if (!agaus(A, rhs, 4, coef[bi])) return 0;
  }
  const double jac = h1 * h2 / 4;
  double gw[4], gx[4], gy[4];
  for (int g = 0; g < 4; ++g) {
    gw[g] = q->w4[g] * jac;
    gx[g] = h1 * q->p4[g][0] / 2. + V[0][0] + h1 / 2.;
    gy[g] = h2 * q->p4[g][1] / 2. + V[0][1] + h2 / 2.;
  }
  double phi[4][4];
  for (int i = 0; i < 4; ++i)
    for (int g = 0; g < 4; ++g)
      phi[i][g] = coef[i][0] + coef[i][1] * gx[g] + coef[i][2] * gy[g] + coef[i][3] * gx[g] * gy[g];
  /* hardwire(i, g) = w_g phi_i(g) [* r_g]; rho(g) = sum_k R_k phi_k(g) */
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 4; ++k) {
      double s = 0;
      for (int g = 0; g < 4; ++g) {
        double hw = delta == 0 ? gw[g] * phi[i][g] : gw[g] * phi[i][g] * gy[g];
        s = s + hw * phi[k][g];
      }
      M[i * 4 + k] = s;
    }
  return 1;
}

/* IFE_RHS_2D.f90 with Linear_IFE_Basis_Coeff_2D.f90,
 * Inter_Tetra_Partition_2D.f90, Gauss_Nodes_Elem_2D.f90, Tetra_Volume_2D.f90:
 * the load matrix of an interface element in local corner order. */
static int ife_load(const OrIfe *f, const double V[4][2], const Quad *q, int delta, double Mout[16]) {
  double v[4][2];
  for (int r = 0; r < 4; ++r) { v[r][0] = V[f->r2l[r]][0]; v[r][1] = V[f->r2l[r]][1]; }
  const double *I1 = f->D, *I2 = f->E; /* intrs(1,:) = D, intrs(2,:) = E */
  double coef[4][8];
  double M[64];
  memset(M, 0, sizeof M);
  if (f->type == 2) {
    M[0 * 8 + 1] = v[0][0]; M[0 * 8 + 2] = v[0][1]; M[0 * 8 + 3] = v[0][0] * v[0][1];
    M[3 * 8 + 1] = v[3][0]; M[3 * 8 + 2] = v[3][1]; M[3 * 8 + 3] = v[3][0] * v[3][1];
    M[1 * 8 + 5] = v[1][0]; M[1 * 8 + 6] = v[1][1]; M[1 * 8 + 7] = v[1][0] * v[1][1];
    M[2 * 8 + 5] = v[2][0]; M[2 * 8 + 6] = v[2][1]; M[2 * 8 + 7] = v[2][0] * v[2][1];
    M[0 * 8 + 0] = 1; M[3 * 8 + 0] = 1; M[1 * 8 + 4] = 1; M[2 * 8 + 4] = 1;
  } else {
    M[0 * 8 + 1] = v[0][0]; M[0 * 8 + 2] = v[0][1]; M[0 * 8 + 3] = v[0][0] * v[0][1];
    M[3 * 8 + 5] = v[3][0]; M[3 * 8 + 6] = v[3][1]; M[3 * 8 + 7] = v[3][0] * v[3][1];
    M[1 * 8 + 5] = v[1][0]; M[1 * 8 + 6] = v[1][1]; M[1 * 8 + 7] = v[1][0] * v[1][1];
    M[2 * 8 + 5] = v[2][0]; M[2 * 8 + 6] = v[2][1]; M[2 * 8 + 7] = v[2][0] * v[2][1];
    M[0 * 8 + 0] = 1; M[1 * 8 + 4] = 1; M[2 * 8 + 4] = 1; M[3 * 8 + 4] = 1;
  }
  const double mx = (I1[0] + I2[0]) / 2, my = (I1[1] + I2[1]) / 2;
  for (int r = 4; r < 7; ++r) { M[r * 8 + 0] = 1; M[r * 8 + 4] = -1; }
  M[4 * 8 + 1] = I1[0]; M[4 * 8 + 2] = I1[1]; M[4 * 8 + 3] = I1[0] * I1[1];
  M[5 * 8 + 1] = I2[0]; M[5 * 8 + 2] = I2[1]; M[5 * 8 + 3] = I2[0] * I2[1];
  M[6 * 8 + 1] = mx; M[6 * 8 + 2] = my; M[6 * 8 + 3] = mx * my;
  M[4 * 8 + 5] = -I1[0]; M[4 * 8 + 6] = -I1[1]; M[4 * 8 + 7] = -I1[0] * I1[1];
  M[5 * 8 + 5] = -I2[0]; M[5 * 8 + 6] = -I2[1]; M[5 * 8 + 7] = -I2[0] * I2[1];
  M[6 * 8 + 5] = -mx; M[6 * 8 + 6] = -my; M[6 * 8 + 7] = -(mx * my);
  const double b1 = f->beta1, b2 = f->beta2;
  const double qq = ((I2[1] * I2[1]) - (I1[1] * I1[1]) - (I2[0] * I2[0]) + (I1[0] * I1[0])) * .5;
  M[7 * 8 + 0] = 0; M[7 * 8 + 1] = b1 * (I2[1] - I1[1]); M[7 * 8 + 2] = -b1 * (I2[0] - I1[0]);
  M[7 * 8 + 3] = b1 * qq;
  M[7 * 8 + 4] = 0; M[7 * 8 + 5] = -b2 * (I2[1] - I1[1]); M[7 * 8 + 6] = b2 * (I2[0] - I1[0]);
  M[7 * 8 + 7] = -b2 * qq;
  if (I1[0] == I2[0] || I1[1] == I2[1]) {
    for (int k = 0; k < 8; ++k) M[6 * 8 + k] = 0;
    M[6 * 8 + 3] = 1; M[6 * 8 + 7] = -1;
  }
  for (int bi = 0; bi < 4; ++bi) {
    double A[64], rhs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    memcpy(A, M, sizeof A);
    rhs[bi] = 1.0;
    if (!agaus(A, rhs, 8, coef[bi])) return 0;
  }
  /* points 1..4 = reference vertices, 5 = D, 6 = E; last entry = region */
  const double *P[6] = {v[0], v[1], v[2], v[3], I1, I2};
  static const int tri1[4][4] = {{0, 4, 5, 1}, {1, 5, 2, 2}, {5, 2, 4, 2}, {2, 4, 3, 2}};
  static const int tri2[4][4] = {{0, 5, 3, 1}, {3, 4, 5, 1}, {5, 2, 4, 2}, {2, 5, 1, 2}};
  const int(*tri)[4] = f->type == 1 ? tri1 : tri2;
  for (int k = 0; k < 16; ++k) Mout[k] = 0;
  for (int st = 0; st < 4; ++st) {
    const double *A = P[tri[st][0]], *B = P[tri[st][1]], *Cc = P[tri[st][2]];
    double ax = B[0] - A[0], ay = B[1] - A[1], bx = Cc[0] - A[0], by = Cc[1] - A[1];
    const double Vol = fabs(ax * by - bx * ay) / 2.0; /* Mat_Det_2 */
    const int reg = tri[st][3];
    double gx[3], gy[3];
    gx[0] = 0.5 * A[0] + 0.5 * B[0]; gy[0] = 0.5 * A[1] + 0.5 * B[1];
    gx[1] = 0.5 * B[0] + 0.5 * Cc[0]; gy[1] = 0.5 * B[1] + 0.5 * Cc[1];
    gx[2] = 0.5 * Cc[0] + 0.5 * A[0]; gy[2] = 0.5 * Cc[1] + 0.5 * A[1];
    double psi[4][3];
    for (int b = 0; b < 4; ++b) {
      const double *c = coef[b] + 4 * (reg - 1);
      for (int g = 0; g < 3; ++g) psi[b][g] = c[0] + c[1] * gx[g] + c[2] * gy[g] + c[3] * gx[g] * gy[g];
    }
    /* vector(r2l(i)) += V * sum_g w rhs(g) psi_i(g) [* y_g], rhs(g) =
     * sum_r R(r2l(r)) psi_r(g): the matrix entry (r2l(i), r2l(r)) */
    for (int i = 0; i < 4; ++i)
      for (int r = 0; r < 4; ++r) {
        double s = 0;
        for (int g = 0; g < 3; ++g) {
          double t = delta == 0 ? q->third * psi[r][g] * psi[i][g] : q->third * psi[r][g] * gy[g] * psi[i][g];
          s = s + t;
        }
        Mout[f->r2l[i] * 4 + f->r2l[r]] += Vol * s;
      }
  }
  return 1;
}

/* ------------------------------------------------------------------ */
/* The descriptor the oracle builds (owned arrays)                       */
/* ------------------------------------------------------------------ */
typedef struct {
  pic_mesh_desc desc; /* first member: the handle is a pic_mesh_desc* */
  int32_t *node_type, *node_index, *element_index;
  double *phi_dirichlet, *cell_volume;
  int32_t *a_srow, *a_jcol, *xt_srow, *xt_jcol;
  double *a_k, *xt_k, *a_diag, *rhs_fix, *mass_q1, *ife_mass, *mass_rows;
  int32_t *patch_ptr, *patch_nodes;
  pic_object *objects;
  OrIfe *ife;
  int n_ife;
} OrMesh;

void or_mesh_free(pic_mesh_desc *d) {
  if (!d) return;
  OrMesh *S = (OrMesh *)d;
  free(S->node_type); free(S->node_index); free(S->element_index); free(S->phi_dirichlet);
  free(S->cell_volume); free(S->a_srow); free(S->a_jcol); free(S->xt_srow); free(S->xt_jcol);
  free(S->a_k); free(S->xt_k); free(S->a_diag); free(S->rhs_fix); free(S->mass_q1); free(S->ife_mass);
  free(S->mass_rows); free(S->patch_ptr); free(S->patch_nodes); free(S->objects); free(S->ife);
  free(S);
}

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* sorted, unique (Bubble_sort_new and the duplicate-skipping loops of
 * Get_PointPatch.f90) */
static int sort_unique(int32_t *v, int n) {
  if (n <= 0) return 0;
  qsort(v, (size_t)n, sizeof(int32_t), cmp_i32);
  int m = 1;
  for (int i = 1; i < n; ++i)
    if (v[i] != v[m - 1]) v[m++] = v[i];
  return m;
}

/* Returns 0, or a negative code: -1 bad deck, -2 out of memory, -3
 * geometry the reference's case table does not cover (interface through a
 * vertex, saddle, two objects in an element), -4 singular local system. */
int or_mesh_build(const pic_deck *dk, int quad, pic_mesh_desc **out) {
  if (!dk || !out) return -1;
  *out = NULL;
  const int nnx = dk->nnx, nny = dk->nny, nex = nnx - 1, ney = nny - 1;
  if (nnx < 3 || nny < 3 || !(dk->xmax > dk->xmin) || !(dk->ymax > dk->ymin) || dk->n_objects < 0 ||
      dk->n_objects > PIC_MAX_OBJECTS || (dk->delta != 0 && dk->delta != 1))
    return -1;
  const int delta = dk->delta;
  const int64_t nn = (int64_t)nnx * nny, ne = (int64_t)nex * ney;
  Quad q;
  quad_rules(&q, quad);
  OrMesh *S = calloc(1, sizeof(OrMesh));
  if (!S) return -2;
  int rc = 0;
#define NEW(p, n) do { (p) = calloc((size_t)((n) > 0 ? (n) : 1), sizeof(*(p))); if (!(p)) { rc = -2; goto fail; } } while (0)
  /* Cubic_Partition_2D.f90:30-50: x(i) = x_s + h_x*(i-1), node (i-1)*ny + j */
  const double hx = (dk->xmax - dk->xmin) / (nnx - 1), hy = (dk->ymax - dk->ymin) / (nny - 1);
  double *xs = NULL, *ys = NULL;
  NEW(xs, nnx); NEW(ys, nny);
  for (int i = 0; i < nnx; ++i) xs[i] = dk->xmin + hx * i;
  for (int j = 0; j < nny; ++j) ys[j] = dk->ymin + hy * j;
#define NODE(i, j) ((int64_t)(i) * nny + (j))
#define ELEM(i, j) ((int64_t)(i) * ney + (j))
  NEW(S->objects, dk->n_objects);
  memcpy(S->objects, dk->objects, sizeof(pic_object) * (size_t)dk->n_objects);

  /* node_index (Setup_IFE_Mesh_2D.f90:402-424 with Update_Locate_Node_2D):
   * the first object a node falls in labels it -(k+2) */
  NEW(S->node_index, nn);
  for (int64_t n = 0; n < nn; ++n) S->node_index[n] = -1;
  for (int i = 0; i < nnx; ++i)
    for (int j = 0; j < nny; ++j)
      for (int k = 0; k < dk->n_objects; ++k)
        if (S->node_index[NODE(i, j)] == -1 && node_inside(&dk->objects[k], xs[i], ys[j]))
          S->node_index[NODE(i, j)] = -(k + 2);

  /* node_type (Partition_Cube_2D.f90:24-58): Dirichlet when a Dirichlet wall
   * or a conductor holds the node, unknowns numbered in node order.  A node
   * on two Dirichlet walls takes the x wall's value. */
  NEW(S->node_type, nn);
  NEW(S->phi_dirichlet, nn);
  int32_t nu = 0;
  for (int i = 0; i < nnx; ++i)
    for (int j = 0; j < nny; ++j) {
      int64_t n = NODE(i, j);
      int dir = 0;
      double val = 0;
      if (j == 0 && dk->wall_dirichlet[2]) { dir = 1; val = dk->wall_phi[2]; }
      if (j == nny - 1 && dk->wall_dirichlet[3]) { dir = 1; val = dk->wall_phi[3]; }
      if (i == 0 && dk->wall_dirichlet[0]) { dir = 1; val = dk->wall_phi[0]; }
      if (i == nnx - 1 && dk->wall_dirichlet[1]) { dir = 1; val = dk->wall_phi[1]; }
      int lab = S->node_index[n];
      if (lab <= -2 && dk->objects[-lab - 2].conductor) { dir = 1; val = dk->objects[-lab - 2].phi; }
      S->phi_dirichlet[n] = dir ? val : 0.0;
      S->node_type[n] = dir ? -1 : ++nu;
    }

  /* element_index and the interface elements
   * (Update_Mesh_Objects_Intersection_2D.f90, El_Object_Intersection_info_2D_BL.f90) */
  NEW(S->element_index, ne);
  NEW(S->ife, ne);
  double *elem_beta = NULL;
  NEW(elem_beta, ne);
  static const int cdi[4] = {0, 1, 1, 0}, cdj[4] = {0, 0, 1, 1};
  for (int i = 0; i < nex; ++i)
    for (int j = 0; j < ney; ++j) {
      int64_t e = ELEM(i, j);
      int lab[4], obj = -1, same = 1;
      for (int c = 0; c < 4; ++c) {
        lab[c] = S->node_index[NODE(i + cdi[c], j + cdj[c])];
        if (lab[c] != lab[0]) same = 0;
        if (lab[c] <= -2) {
          if (obj >= 0 && obj != -lab[c] - 2) { rc = -3; goto fail; }
          obj = -lab[c] - 2;
        }
      }
      if (same) {
        S->element_index[e] = lab[0];
        elem_beta[e] = (lab[0] <= -2 && !dk->objects[-lab[0] - 2].conductor) ? dk->objects[-lab[0] - 2].eps : 1.0;
        continue;
      }
      const pic_object *o = &dk->objects[obj];
      if (o->conductor) { /* cut by a conductor: a plain Q1 element */
        S->element_index[e] = -1;
        elem_beta[e] = 1.0;
        continue;
      }
      double V[4][2], P[4][2];
      int mask = 0, ncut = 0;
      for (int c = 0; c < 4; ++c) {
        V[c][0] = xs[i + cdi[c]]; V[c][1] = ys[j + cdj[c]];
        if (lab[c] <= -2) mask |= 1 << c;
      }
      for (int c = 0; c < 4; ++c) {
        int d = (c + 1) & 3;
        int fl = edge_object(o, V[c][0], V[c][1], V[d][0], V[d][1], P[c]);
        if (fl < 0) { rc = -3; goto fail; } /* interface through a vertex */
        if (fl == 1) {
          ++ncut;
          if (((mask >> c) & 1) == ((mask >> d) & 1)) { rc = -3; goto fail; }
        } else if (((mask >> c) & 1) != ((mask >> d) & 1)) { rc = -3; goto fail; }
      }
      if (ncut != 2 || kCase[mask].type == 0) { rc = -3; goto fail; }
      OrIfe *f = &S->ife[S->n_ife];
      f->elem = (int)e;
      f->type = kCase[mask].type;
      for (int r = 0; r < 4; ++r) {
        f->r2l[r] = (kCase[mask].r1 + r) & 3;
        f->l2r[f->r2l[r]] = r;
      }
      f->D[0] = P[kCase[mask].eD][0]; f->D[1] = P[kCase[mask].eD][1];
      f->E[0] = P[kCase[mask].eE][0]; f->E[1] = P[kCase[mask].eE][1];
      /* beta_plus = object%Eps, beta_minus = ONE */
      f->beta1 = kCase[mask].in1 ? o->eps : 1.0;
      f->beta2 = kCase[mask].in1 ? 1.0 : o->eps;
      S->element_index[e] = ++S->n_ife;
    }

  /* Sparse_Structure.f90 / Sparse_Structure_xt (SIDG/Sparse_Structure_xt.f90):
   * each row's columns in order of first appearance over the element loop
   * (elements j fastest, corners in HT order).  The SIDG edge pass there adds
   * structural entries that stay 0 without DG areas; they are omitted. */
  {
    int32_t *cnt = NULL, *cnt_xt = NULL;
    NEW(cnt, nu + 1); NEW(cnt_xt, nu + 1);
    int32_t *vrow = NULL, *vrow_xt = NULL; /* up to 9 and 9 per row */
    NEW(vrow, (int64_t)nu * 9); NEW(vrow_xt, (int64_t)nu * 9);
    for (int i = 0; i < nex; ++i)
      for (int j = 0; j < ney; ++j) {
        int64_t nd[4];
        for (int c = 0; c < 4; ++c) nd[c] = NODE(i + cdi[c], j + cdj[c]);
        for (int a = 0; a < 4; ++a) {
          int u = S->node_type[nd[a]];
          if (u <= 0) continue;
          for (int b = 0; b < 4; ++b) {
            int v = S->node_type[nd[b]];
            if (v > 0) {
              int found = 0;
              for (int m = 0; m < cnt[u - 1]; ++m) found |= vrow[(int64_t)(u - 1) * 9 + m] == v;
              if (!found) vrow[(int64_t)(u - 1) * 9 + cnt[u - 1]++] = v;
            } else {
              int32_t id = (int32_t)(nd[b] + 1);
              int found = 0;
              for (int m = 0; m < cnt_xt[u - 1]; ++m) found |= vrow_xt[(int64_t)(u - 1) * 9 + m] == id;
              if (!found) vrow_xt[(int64_t)(u - 1) * 9 + cnt_xt[u - 1]++] = id;
            }
          }
        }
      }
    NEW(S->a_srow, nu + 1); NEW(S->xt_srow, nu + 1);
    int64_t nz = 0, nzx = 0;
    for (int u = 0; u < nu; ++u) {
      S->a_srow[u] = (int32_t)(nz + 1); nz += cnt[u];
      S->xt_srow[u] = (int32_t)(nzx + 1); nzx += cnt_xt[u];
    }
    S->a_srow[nu] = (int32_t)(nz + 1);
    S->xt_srow[nu] = (int32_t)(nzx + 1);
    NEW(S->a_jcol, nz); NEW(S->a_k, nz); NEW(S->xt_jcol, nzx); NEW(S->xt_k, nzx);
    for (int u = 0; u < nu; ++u) {
      for (int m = 0; m < cnt[u]; ++m) S->a_jcol[S->a_srow[u] - 1 + m] = vrow[(int64_t)u * 9 + m];
      for (int m = 0; m < cnt_xt[u]; ++m) S->xt_jcol[S->xt_srow[u] - 1 + m] = vrow_xt[(int64_t)u * 9 + m];
    }
    S->desc.nnz = nz;
    S->desc.nnz_xt = nzx;
    free(cnt); free(cnt_xt); free(vrow); free(vrow_xt);
  }

  /* Generate_stiffness_matrix_local_IFE.f90 called twice (IFE_Start_2D.f90:
   * 361-375: the xx part into matrix1/matrix5, the yy part into
   * matrix2/matrix6), then A = matrix1 + matrix2, A_xt = matrix5 + matrix6. */
  {
    double *a1 = NULL, *a2 = NULL, *x1 = NULL, *x2 = NULL;
    NEW(a1, S->desc.nnz); NEW(a2, S->desc.nnz); NEW(x1, S->desc.nnz_xt); NEW(x2, S->desc.nnz_xt);
    for (int part = 0; part < 2; ++part) {
      double *A = part == 0 ? a1 : a2, *X = part == 0 ? x1 : x2;
      const int dx = part == 0;
      for (int i = 0; i < nex; ++i)
        for (int j = 0; j < ney; ++j) {
          int64_t e = ELEM(i, j);
          int64_t nd[4];
          double V[4][2];
          for (int c = 0; c < 4; ++c) {
            nd[c] = NODE(i + cdi[c], j + cdj[c]);
            V[c][0] = xs[i + cdi[c]]; V[c][1] = ys[j + cdj[c]];
          }
          /* wsy add for sidg: h from the element's own corners */
          const double h1 = V[1][0] - V[0][0], h2 = V[3][1] - V[0][1];
          double K[4][4];
          int eid = S->element_index[e];
          for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
              K[a][b] = eid > 0 ? ife_stiff_entry(&S->ife[eid - 1], V, &q, a, b, dx, delta)
                                : q1_stiff_entry(&q, V[0][0], V[0][1], h1, h2, elem_beta[e], a, b, dx, delta);
          /* El_Stiff(j,k): trial j, test k; row of corner k gets El_Stiff(k, j) */
          for (int k = 0; k < 4; ++k) {
            int u = S->node_type[nd[k]];
            if (u <= 0) continue;
            for (int jj = 0; jj < 4; ++jj) {
              int v = S->node_type[nd[jj]];
              if (v > 0) {
                for (int m = S->a_srow[u - 1] - 1; m < S->a_srow[u] - 1; ++m)
                  if (S->a_jcol[m] == v) { A[m] = A[m] + K[k][jj]; break; }
              } else {
                for (int m = S->xt_srow[u - 1] - 1; m < S->xt_srow[u] - 1; ++m)
                  if (S->xt_jcol[m] == nd[jj] + 1) { X[m] = X[m] + K[k][jj]; break; }
              }
            }
          }
        }
    }
    for (int64_t m = 0; m < S->desc.nnz; ++m) S->a_k[m] = a1[m] + a2[m];
    for (int64_t m = 0; m < S->desc.nnz_xt; ++m) S->xt_k[m] = x1[m] + x2[m];
    free(a1); free(a2); free(x1); free(x2);
  }
  /* Diagonal_Preconditioner.f90 */
  NEW(S->a_diag, nu);
  for (int u = 0; u < nu; ++u)
    for (int m = S->a_srow[u] - 1; m < S->a_srow[u + 1] - 1; ++m)
      if (S->a_jcol[m] == u + 1) { S->a_diag[u] = S->a_k[m]; break; }
  NEW(S->rhs_fix, nu);

  /* load matrices (Global_RHS_PDE_2D.f90:72-138): regular elements from the
   * first element of the mesh (Cartesian; a uniform mesh has one matrix),
   * per element row on an r-z mesh; interface elements their own */
  {
    NEW(S->mass_q1, 16);
    double V[4][2];
    for (int c = 0; c < 4; ++c) { V[c][0] = xs[cdi[c]]; V[c][1] = ys[cdj[c]]; }
    if (!q1_load(&q, V, V[1][0] - V[0][0], V[3][1] - V[0][1], 0, S->mass_q1)) { rc = -4; goto fail; }
    if (delta == 1) {
      NEW(S->mass_rows, (int64_t)16 * ney);
      for (int j = 0; j < ney; ++j) {
        for (int c = 0; c < 4; ++c) { V[c][0] = xs[cdi[c]]; V[c][1] = ys[j + cdj[c]]; }
        if (!q1_load(&q, V, V[1][0] - V[0][0], V[3][1] - V[0][1], 1, S->mass_rows + 16 * (int64_t)j)) {
          rc = -4;
          goto fail;
        }
      }
    }
    NEW(S->ife_mass, (int64_t)16 * S->n_ife);
    for (int k = 0; k < S->n_ife; ++k) {
      const OrIfe *f = &S->ife[k];
      int i = f->elem / ney, j = f->elem % ney;
      for (int c = 0; c < 4; ++c) { V[c][0] = xs[i + cdi[c]]; V[c][1] = ys[j + cdj[c]]; }
      if (!ife_load(f, V, &q, delta, S->ife_mass + 16 * (int64_t)k)) { rc = -4; goto fail; }
    }
  }

  /* dual-cell volumes, SetupGrids_2D_QLL.f90:197-289 (Cell_volume_zwz(2,:)) */
  NEW(S->cell_volume, nn);
  {
    const double pi = 3.14159265358979; /* Pi_LY, SetupGrids_2D_QLL.f90:53 */
    const double xmin = dk->xmin, xmax = dk->xmax, ymin = dk->ymin, ymax = dk->ymax;
    for (int i = 0; i < nnx; ++i)
      for (int j = 0; j < nny; ++j) {
        const double x = xs[i], y = ys[j];
        /* the element the node belongs to (P_flag(5,:)): its own, or the last one on the far walls */
        const int ie = i < nex ? i : nex - 1, je = j < ney ? j : ney - 1;
        const double h1 = xs[ie + 1] - xs[ie], h2 = ys[je + 1] - ys[je];
        const int onxn = fabs(x - xmin) < SMALL, onxx = fabs(x - xmax) < SMALL;
        const int onyn = fabs(y - ymin) < SMALL, onyx = fabs(y - ymax) < SMALL;
        double v;
        if ((onxn || onxx) && (onyn || onyx)) {
          if (delta == 0) v = h1 * h2 / 4.0;
          else if (onyn) v = 2.0 * pi * (ymin + h2 / 4.0) * (h2 / 2.0) * h1 / 2.0;
          else v = 2.0 * pi * (ymax - h2 / 4.0) * (h2 / 2.0) * h1 / 2.0;
        } else if (onxn || onxx || onyn || onyx) {
          if (delta == 0) v = h1 * h2 / 2.0;
          else if (onyn) v = 2.0 * pi * (ymin + h2 / 4.0) * (h2 / 2.0) * h1;
          else if (onyx) v = 2.0 * pi * (ymax - h2 / 4.0) * (h2 / 2.0) * h1;
          else v = 2.0 * pi * y * h2 * h1 / 2.0;
        } else {
          v = delta == 0 ? h1 * h2 / 1.0 : 2.0 * pi * y * h2 * h1 / 1.0;
        }
        S->cell_volume[NODE(i, j)] = v;
      }
  }

  /* PPR patches, Get_PointPatch.f90 (its O(N^2) duplicate-node search finds
   * nothing on a conforming mesh and is skipped) */
  {
    int32_t *base = NULL, *bcnt = NULL, *kind = NULL, *pat = NULL, *pcnt = NULL;
    const int CAP = 64;
    NEW(base, nn * 16); NEW(bcnt, nn); NEW(kind, nn); NEW(pat, nn * CAP); NEW(pcnt, nn);
    for (int i = 0; i < nnx; ++i)
      for (int j = 0; j < nny; ++j) {
        int64_t n = NODE(i, j);
        const double x = xs[i], y = ys[j];
        /* ParPosition_ppr_elem.f90: the elements holding points biased by
         * hx/4 towards each quadrant (SW, SE, NE, NW) */
        int64_t ex[4] = {-1, -1, -1, -1};
        if (i > 0 && j > 0) ex[0] = ELEM(i - 1, j - 1);
        if (i < nex && j > 0) ex[1] = ELEM(i, j - 1);
        if (i < nex && j < ney) ex[2] = ELEM(i, j);
        if (i > 0 && j < ney) ex[3] = ELEM(i - 1, j);
        const int onxn = fabs(x - dk->xmin) < SMALL, onxx = fabs(x - dk->xmax) < SMALL;
        const int onyn = fabs(y - dk->ymin) < SMALL, onyx = fabs(y - dk->ymax) < SMALL;
        int64_t pe[4];
        int npe = 0;
        if ((onxn || onxx) && (onyn || onyx)) { /* corner: its one element */
          for (int c = 0; c < 4; ++c) if (ex[c] >= 0) pe[npe++] = ex[c];
          kind[n] = 2;
        } else if (onxn) { pe[npe++] = ex[1]; pe[npe++] = ex[2]; kind[n] = 2; }
        else if (onyx) { pe[npe++] = ex[0]; pe[npe++] = ex[1]; kind[n] = 2; }
        else if (onxx) { pe[npe++] = ex[0]; pe[npe++] = ex[3]; kind[n] = 2; }
        else if (onyn) { pe[npe++] = ex[3]; pe[npe++] = ex[2]; kind[n] = 2; }
        else {
          int all_in = 1, all_out = 1;
          for (int c = 0; c < 4; ++c) {
            all_in &= S->element_index[ex[c]] == -2; /* In_index */
            all_out &= S->element_index[ex[c]] == -1; /* Out_index */
          }
          if (all_in || all_out) {
            for (int c = 0; c < 4; ++c) pe[npe++] = ex[c];
            kind[n] = 1;
          } else {
            for (int c = 0; c < 4; ++c) if (S->element_index[ex[c]] < 0) pe[npe++] = ex[c];
            kind[n] = 3;
          }
        }
        int32_t tmp[16];
        int nt = 0;
        for (int k = 0; k < npe; ++k) {
          int ei = (int)(pe[k] / ney), ej = (int)(pe[k] % ney);
          for (int c = 0; c < 4; ++c) tmp[nt++] = (int32_t)(NODE(ei + cdi[c], ej + cdj[c]) + 1);
        }
        nt = sort_unique(tmp, nt);
        bcnt[n] = nt;
        memcpy(base + n * 16, tmp, sizeof(int32_t) * (size_t)nt);
        pcnt[n] = nt;
        memcpy(pat + n * CAP, tmp, sizeof(int32_t) * (size_t)nt);
      }
    /* union over the patch's nodes of their unextended patches */
    int32_t *u = NULL;
    NEW(u, 16 * 16);
    for (int pass = 0; pass < 2; ++pass)
      for (int64_t n = 0; n < nn; ++n) {
        int want = pass == 0 ? (pcnt[n] < 6 && pcnt[n] != 0) : ((kind[n] == 2 || kind[n] == 3) && pcnt[n] < 12);
        if (!want || bcnt[n] == 0) continue;
        int nu2 = 0;
        for (int k = 0; k < bcnt[n]; ++k) {
          int64_t m = base[n * 16 + k] - 1;
          for (int t = 0; t < bcnt[m]; ++t) u[nu2++] = base[m * 16 + t];
        }
        nu2 = sort_unique(u, nu2);
        if (nu2 > CAP) { rc = -3; free(u); goto fail_patch; }
        pcnt[n] = nu2;
        memcpy(pat + n * CAP, u, sizeof(int32_t) * (size_t)nu2);
      }
    free(u);
    /* nodes whose four elements are all interface elements keep an empty
     * patch: Get_PointPatch.f90 builds ab_point_patch for them but never
     * stores it, and GetEfield_SIDG_PPR.f90 skips n_node_in_one_patch = 0 */
    NEW(S->patch_ptr, nn + 1);
    int64_t tot = 0;
    for (int64_t n = 0; n < nn; ++n) { S->patch_ptr[n] = (int32_t)tot; tot += pcnt[n]; }
    S->patch_ptr[nn] = (int32_t)tot;
    NEW(S->patch_nodes, tot);
    for (int64_t n = 0; n < nn; ++n)
      memcpy(S->patch_nodes + S->patch_ptr[n], pat + n * CAP, sizeof(int32_t) * (size_t)pcnt[n]);
  fail_patch:
    free(base); free(bcnt); free(kind); free(pat); free(pcnt);
    if (rc) goto fail;
  }

  {
    pic_mesh_desc *d = &S->desc;
    d->nnx = nnx; d->nny = nny;
    d->xmin = dk->xmin; d->xmax = dk->xmax; d->ymin = dk->ymin; d->ymax = dk->ymax;
    d->delta = delta;
    d->node_type = S->node_type; d->node_index = S->node_index; d->element_index = S->element_index;
    d->phi_dirichlet = S->phi_dirichlet; d->cell_volume = S->cell_volume;
    d->n_unknowns = nu;
    d->a_srow = S->a_srow; d->a_jcol = S->a_jcol; d->a_k = S->a_k;
    d->xt_srow = S->xt_srow; d->xt_jcol = S->xt_jcol; d->xt_k = S->xt_k;
    d->a_diag = S->a_diag; d->rhs_fix = S->rhs_fix; d->mass_q1 = S->mass_q1;
    d->n_interface = S->n_ife; d->ife_mass = S->ife_mass;
    d->patch_ptr = S->patch_ptr; d->patch_nodes = S->patch_nodes;
    d->n_objects = dk->n_objects; d->objects = S->objects;
    d->mass_rows = S->mass_rows;
  }
  free(xs); free(ys); free(elem_beta);
  *out = &S->desc;
  return 0;
fail:
  free(xs); free(ys); free(elem_beta);
  or_mesh_free(&S->desc);
  return rc ? rc : -2;
#undef NEW
#undef NODE
#undef ELEM
}

/* Interface element k (1-based, element order) as the reference's
 * information_1/2 hold it: element (1-based), type, pointer_reference_to_local
 * (1-based), beta1, beta2, D, E. */
int or_mesh_interface(const pic_mesh_desc *d, int32_t k, int32_t *element, int32_t *type, int32_t *r2l,
                      double *beta, double *D, double *E) {
  const OrMesh *S = (const OrMesh *)d;
  if (!d || k < 1 || k > S->n_ife) return -1;
  const OrIfe *f = &S->ife[k - 1];
  if (element) *element = f->elem + 1;
  if (type) *type = f->type;
  if (r2l) for (int r = 0; r < 4; ++r) r2l[r] = f->r2l[r] + 1;
  if (beta) { beta[0] = f->beta1; beta[1] = f->beta2; }
  if (D) { D[0] = f->D[0]; D[1] = f->D[1]; }
  if (E) { E[0] = f->E[0]; E[1] = f->E[1]; }
  return 0;
}

/* The quadrature constants in use (for the tests): w9[9], p9 (9x2),
 * wt9[9], pt9 (9x2), w4[4], p4 (4x2), third. */
void or_quad_constants(int quad, double *out) {
  Quad q;
  quad_rules(&q, quad);
  int o = 0;
  for (int g = 0; g < 9; ++g) out[o++] = q.w9[g];
  for (int g = 0; g < 9; ++g) { out[o++] = q.p9[g][0]; out[o++] = q.p9[g][1]; }
  for (int g = 0; g < 9; ++g) out[o++] = q.wt9[g];
  for (int g = 0; g < 9; ++g) { out[o++] = q.pt9[g][0]; out[o++] = q.pt9[g][1]; }
  for (int g = 0; g < 4; ++g) out[o++] = q.w4[g];
  for (int g = 0; g < 4; ++g) { out[o++] = q.p4[g][0]; out[o++] = q.p4[g][1]; }
  out[o++] = q.third;
}
