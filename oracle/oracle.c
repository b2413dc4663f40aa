/*
 * oracle.c -- CPU restatement (FP64) of the reference's IFE-PIC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for libpicgpu: only
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py load
 * it.  The product never calls it.
 *
 * Reference: weqwoueu/pic-, project PIC-IFE_GEC (Fortran).  No Fortran
 * compiler exists on the build or GPU hosts, so the reference cannot be
 * compiled; each routine here restates the reference routine cited beside
 * it.  Where the GPU design deliberately differs (int64 fixed-point deposit,
 * Philox random numbers, canonical reduction order of dot products,
 * histogram selection of MCC candidates), the oracle applies the same
 * definition so that results compare bit for bit or to the stated tolerance.
 * Pinned against the reference's own known answers: normalisation constants
 * (OUTPUT/physics_parameter.inp:42-47), the closed-form Q1 IFE basis
 * (IFE-Rectangular/Retangular_reference_basis_IFE.f90) and the IFE
 * convergence rates of Norm_Error_{0064,0128,0256}.txt; see tests/.  The
 * axisymmetric (delta 1) branches have no reference outputs; they are
 * pinned by analytic answers in tests/: dual volumes that sum to the
 * cylinder, a manufactured solution at second order, an exact dielectric
 * slab, free streaming along the 3D straight line, and a plasma uniform in
 * volume that deposits its density.
 */
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/picgpu.h"

#define OR_KB 1.3807e-23
#define OR_QE 1.6022e-19
#define OR_ME 9.1095e-31
#define OR_EPS0 8.8542e-12
#define OR_JTOEV 1.6022e-19
#define OR_EVTOK 11605.0
#define OR_MINREAL 1.0e-15
#define OR_PI 3.141592653589793238
#define OR_FEXP 2.71828
#define OR_QSCALE 1099511627776.0
#define OR_ESCALE 4294967296.0

/* ------------------------------------------------------------------ */
/* normalisation, Input_2D.f90:362-392                                  */
/* ------------------------------------------------------------------ */
void or_reference_scales(double n_ref, double T_eV, double out[4]) {
  double T_ref = T_eV * OR_EVTOK;
  out[0] = sqrt(OR_EPS0 * OR_KB * T_ref / n_ref / OR_QE / OR_QE); /* L_ref    */
  out[1] = sqrt(OR_EPS0 * OR_ME / n_ref / OR_QE / OR_QE);         /* time_ref */
  out[2] = sqrt(OR_KB * T_ref / OR_ME);                           /* v_ref    */
  out[3] = OR_KB * T_ref / OR_QE;                                 /* Phi_ref  */
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11)                                 */
/* ------------------------------------------------------------------ */
void or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u01(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------ */
/* mesh view                                                            */
/* ------------------------------------------------------------------ */
typedef struct {
  const pic_mesh_desc *d;
  int nnx, nny, nex, ney;
  int64_t nn, ne;
  double hx, hy;
  double *xs, *ys;
} Mesh;

static void mesh_open(Mesh *m, const pic_mesh_desc *d) {
  m->d = d;
  m->nnx = d->nnx; m->nny = d->nny; m->nex = d->nnx - 1; m->ney = d->nny - 1;
  m->nn = (int64_t)d->nnx * d->nny; m->ne = (int64_t)m->nex * m->ney;
  m->hx = (d->xmax - d->xmin) / (d->nnx - 1);
  m->hy = (d->ymax - d->ymin) / (d->nny - 1);
  m->xs = (double *)malloc(sizeof(double) * d->nnx);
  m->ys = (double *)malloc(sizeof(double) * d->nny);
  for (int i = 0; i < d->nnx; ++i) m->xs[i] = d->xmin + m->hx * i; /* Cubic_Partition_2D.f90:40-48 */
  for (int j = 0; j < d->nny; ++j) m->ys[j] = d->ymin + m->hy * j;
}
static void mesh_close(Mesh *m) { free(m->xs); free(m->ys); }

/* InjectPositioning.f90:13-22 with the GetParChg_2D.f90:143-149 clamp. */
static int locate(const Mesh *m, double x, double y) {
  double rxp = (x - m->d->xmin) / m->hx, ryp = (y - m->d->ymin) / m->hy;
  int i = (int)rxp + 1, j = (int)ryp + 1;
  if (i == m->nnx) i = m->nnx - 1;
  if (j == m->nny) j = m->nny - 1;
  if (!(rxp >= 0.0) || !(ryp >= 0.0) || i < 1 || j < 1 || i > m->nex || j > m->ney) return -1;
  return (i - 1) * m->ney + (j - 1);
}

int32_t or_locate(const pic_mesh_desc *d, double x, double y) {
  Mesh m;
  mesh_open(&m, d);
  int e = locate(&m, x, y);
  mesh_close(&m);
  return e;
}

/* bilinear weights, MoveOne.f90:80-92 / GetParChg_2D.f90:788-802 */
static void weights(const Mesh *m, int e, double x, double y, double W[4], int64_t nodes[4]) {
  int i = e / m->ney, j = e % m->ney;
  double x1 = m->xs[i], x2 = m->xs[i + 1], y1 = m->ys[j], y2 = m->ys[j + 1];
  double dx = (x - x1) / (x2 - x1), dy = (y - y1) / (y2 - y1);
  double xc = 1.0 - dx, yc = 1.0 - dy;
  W[0] = xc * yc; W[1] = dx * yc; W[2] = dx * dy; W[3] = xc * dy;
  int64_t n1 = (int64_t)i * m->nny + j;
  nodes[0] = n1; nodes[1] = n1 + m->nny; nodes[2] = n1 + m->nny + 1; nodes[3] = n1 + 1;
}

/* axisymmetric (r = y) deposit weights, GetParChg_2D.f90:803-821: linear in
 * r^2 across the element, the two lower nodes scaled by beta = 0.75 in the
 * element row on the axis (R1 = dymin + y1 with dymin = ymin, as there). */
static void weights_axi(const Mesh *m, int e, double x, double y, double W[4], int64_t nodes[4]) {
  int i = e / m->ney, j = e % m->ney;
  double x1 = m->xs[i], x2 = m->xs[i + 1], y1 = m->ys[j], y4 = m->ys[j + 1];
  double dx = (x - x1) / (x2 - x1), xc = 1.0 - dx;
  double beta = (fabs(y1 - m->d->ymin) < 1e-5) ? 0.75 : 1.0;
  double R1 = m->d->ymin + y1, R2 = m->d->ymin + y4, R = y;
  double den = R2 * R2 - R1 * R1;
  W[0] = ((xc * (R2 * R2 - R * R)) / den) * beta;
  W[1] = ((dx * (R2 * R2 - R * R)) / den) * beta;
  W[2] = (dx * (R * R - R1 * R1)) / den;
  W[3] = (xc * (R * R - R1 * R1)) / den;
  int64_t n1 = (int64_t)i * m->nny + j;
  nodes[0] = n1; nodes[1] = n1 + m->nny; nodes[2] = n1 + m->nny + 1; nodes[3] = n1 + 1;
}

static int in_object(const pic_object *o, double x, double y) {
  if (o->shape == PIC_SHAPE_CIRCLE) { /* MCCInterface.f90:493-497 */
    double dx = x - o->cx, dy = y - o->cy;
    return dx * dx + dy * dy < o->a * o->a;
  }
  if (o->shape == PIC_SHAPE_BOX) /* MCCInterface.f90:487-491 */
    return x > o->cx && x < o->a && y > o->cy && y < o->b;
  if (o->shape == PIC_SHAPE_ELLIPSE) {
    double c = cos(o->angle), s = sin(o->angle);
    double u = (x - o->cx) * c + (y - o->cy) * s, v = -(x - o->cx) * s + (y - o->cy) * c;
    return (u * u) / (o->a * o->a) + (v * v) / (o->b * o->b) < 1.0;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* MoveAll -> MoveOne (IMPIC/MoveOne.f90:54-264) + Get_ParticleEField_PPR */
/* (PPR/Get_ParticleEField_PPR.f90) + AdjustParticleBoundary              */
/* (MCCInterface.f90:361-532), Cartesian, no magnetic field.              */
/* loc[p] < 0 marks absorbed particles (X = -2000 in the reference).      */
/* coef: [5][nn] = coef_ppr(2..6,:).  Returns the number absorbed.        */
/* ------------------------------------------------------------------ */
int64_t or_move_all(const pic_mesh_desc *d, int64_t n, double *x, double *y, double *vx, double *vy,
                    const double *vz, int32_t *loc, const double *efx, const double *efy,
                    const double *coef, double qm, double dt, const int32_t wall[4]) {
  (void)vz;
  Mesh m;
  mesh_open(&m, d);
  const int64_t nn = m.nn;
  int64_t lost = 0;
#pragma omp parallel for schedule(static) reduction(+ : lost)
  for (int64_t p = 0; p < n; ++p) {
    int e = loc[p];
    if (e < 0) continue;
    double W[4];
    int64_t nd[4];
    weights(&m, e, x[p], y[p], W, nd);
    double Ex, Ey;
    if (d->element_index[e] > 0) {
      double ex = 0.0, ey = 0.0;
      int cnt = 0;
      for (int c = 0; c < 4; ++c) {
        int64_t q = nd[c];
        if (d->node_index[q] == -1) {
          ++cnt;
          double xr = x[p] - m.xs[q / m.nny], yr = y[p] - m.ys[q % m.nny];
          ex = ((ex + coef[0 * nn + q]) + (2.0 * coef[2 * nn + q]) * xr) + coef[3 * nn + q] * yr;
          ey = ((ey + coef[1 * nn + q]) + (2.0 * coef[4 * nn + q]) * yr) + coef[3 * nn + q] * xr;
        }
      }
      ex = ex / (double)cnt;
      ey = ey / (double)cnt;
      Ex = -ex;
      Ey = -ey;
    } else {
      Ex = ((W[0] * efx[nd[0]] + W[1] * efx[nd[1]]) + W[2] * efx[nd[2]]) + W[3] * efx[nd[3]];
      Ey = ((W[0] * efy[nd[0]] + W[1] * efy[nd[1]]) + W[2] * efy[nd[2]]) + W[3] * efy[nd[3]];
    }
    vx[p] = vx[p] + (qm * Ex) * dt;
    vy[p] = vy[p] + (qm * Ey) * dt;
    x[p] = x[p] + dt * vx[p];
    y[p] = y[p] + dt * vy[p];
    int dead = 0;
    if (x[p] <= d->xmin) {
      if (wall[0] == PIC_WALL_REFLECT) { x[p] = d->xmin + (d->xmin - x[p]); vx[p] = -vx[p]; } else dead = 1;
    } else if (x[p] > d->xmax) {
      if (wall[1] == PIC_WALL_REFLECT) { x[p] = d->xmax - (x[p] - d->xmax); vx[p] = -vx[p]; } else dead = 1;
    } else if (y[p] < d->ymin) {
      if (wall[2] == PIC_WALL_REFLECT) { y[p] = d->ymin + (d->ymin - y[p]); vy[p] = -vy[p]; } else dead = 1;
    } else if (y[p] > d->ymax) {
      if (wall[3] == PIC_WALL_REFLECT) { y[p] = d->ymax - (y[p] - d->ymax); vy[p] = -vy[p]; } else dead = 1;
    }
    for (int k = 0; k < d->n_objects && !dead; ++k)
      if (in_object(&d->objects[k], x[p], y[p])) dead = 1;
    if (dead) { loc[p] = -1; ++lost; }
  }
  mesh_close(&m);
  return lost;
}

/* ------------------------------------------------------------------ */
/* Axisymmetric MoveOne (IMPIC/MoveOne.f90:213-263, delta == 1, no B).   */
/* x = z (axial), y = r; the velocity is held in the particle's own      */
/* frame: vx = v_z, vy = v_r, vz = v_theta (the reference keeps the      */
/* angle PO%Z and Cartesian transverse components instead; the two agree */
/* in exact arithmetic, and this form needs no angle and no cos/sin).    */
/* E_theta = 0: v_z += qm E_z dt, v_r += qm E_r dt; the transverse move  */
/* X = r + dt v_r, Y = dt v_theta (X = 0 -> hy * 1e-5 as there), r' =    */
/* |(X, Y)|, then (v_r, v_theta) rotated into the new frame by           */
/* (X, Y)/r'.  Walls and objects as or_move_all.                          */
/* ------------------------------------------------------------------ */
int64_t or_move_all_axi(const pic_mesh_desc *d, int64_t n, double *x, double *y, double *vx, double *vy,
                        double *vz, int32_t *loc, const double *efx, const double *efy, const double *coef,
                        double qm, double dt, const int32_t wall[4]) {
  Mesh m;
  mesh_open(&m, d);
  const int64_t nn = m.nn;
  int64_t lost = 0;
#pragma omp parallel for schedule(static) reduction(+ : lost)
  for (int64_t p = 0; p < n; ++p) {
    int e = loc[p];
    if (e < 0) continue;
    double W[4];
    int64_t nd[4];
    weights(&m, e, x[p], y[p], W, nd); /* the field gather is bilinear, as in Cartesian */
    double Ez, Er;
    if (d->element_index[e] > 0) {
      double ex = 0.0, ey = 0.0;
      int cnt = 0;
      for (int c = 0; c < 4; ++c) {
        int64_t q = nd[c];
        if (d->node_index[q] == -1) {
          ++cnt;
          double xr = x[p] - m.xs[q / m.nny], yr = y[p] - m.ys[q % m.nny];
          ex = ((ex + coef[0 * nn + q]) + (2.0 * coef[2 * nn + q]) * xr) + coef[3 * nn + q] * yr;
          ey = ((ey + coef[1 * nn + q]) + (2.0 * coef[4 * nn + q]) * yr) + coef[3 * nn + q] * xr;
        }
      }
      Ez = -(ex / (double)cnt);
      Er = -(ey / (double)cnt);
    } else {
      Ez = ((W[0] * efx[nd[0]] + W[1] * efx[nd[1]]) + W[2] * efx[nd[2]]) + W[3] * efx[nd[3]];
      Er = ((W[0] * efy[nd[0]] + W[1] * efy[nd[1]]) + W[2] * efy[nd[2]]) + W[3] * efy[nd[3]];
    }
    vx[p] = vx[p] + (qm * Ez) * dt;
    vy[p] = vy[p] + (qm * Er) * dt;
    double X = y[p] + dt * vy[p], Y = dt * vz[p];
    if (X == 0.0) X = m.hy * (double)1.0e-5f;
    double rn = sqrt(X * X + Y * Y), c = X / rn, s = Y / rn;
    double vr = c * vy[p] + s * vz[p], vt = c * vz[p] - s * vy[p];
    vy[p] = vr;
    vz[p] = vt;
    x[p] = x[p] + dt * vx[p];
    y[p] = rn;
    int dead = 0;
    if (x[p] <= d->xmin) {
      if (wall[0] == PIC_WALL_REFLECT) { x[p] = d->xmin + (d->xmin - x[p]); vx[p] = -vx[p]; } else dead = 1;
    } else if (x[p] > d->xmax) {
      if (wall[1] == PIC_WALL_REFLECT) { x[p] = d->xmax - (x[p] - d->xmax); vx[p] = -vx[p]; } else dead = 1;
    } else if (y[p] > d->ymax) {
      if (wall[3] == PIC_WALL_REFLECT) { y[p] = d->ymax - (y[p] - d->ymax); vy[p] = -vy[p]; } else dead = 1;
    }
    for (int k = 0; k < d->n_objects && !dead; ++k)
      if (in_object(&d->objects[k], x[p], y[p])) dead = 1;
    if (dead) { loc[p] = -1; ++lost; }
  }
  mesh_close(&m);
  return lost;
}

/* ------------------------------------------------------------------ */
/* GetParChg_2D.f90:122-911 for one species: locate (137-163), bilinear  */
/* weights accumulated per node (788-866) as int64 fixed point with      */
/* 2^-40 per unit weight and 2^-32 per unit weight*eV.                    */
/* ------------------------------------------------------------------ */
int64_t or_deposit(const pic_mesh_desc *d, int64_t n, const double *x, const double *y, const double *vx,
                   const double *vy, const double *vz, int32_t *loc, double mass, double vref,
                   int64_t *q_acc, int64_t *e_acc) {
  Mesh m;
  mesh_open(&m, d);
  int64_t bad = 0;
  /* integer sums: the node totals do not depend on the thread order */
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int64_t p = 0; p < n; ++p) {
    if (loc[p] < 0) continue;
    int e = locate(&m, x[p], y[p]);
    if (e < 0) { loc[p] = -1; ++bad; continue; }
    loc[p] = e;
    double W[4];
    int64_t nd[4];
    if (d->delta == 1) weights_axi(&m, e, x[p], y[p], W, nd);
    else weights(&m, e, x[p], y[p], W, nd);
    double energy = ((((0.5 * mass) * ((vx[p] * vx[p] + vy[p] * vy[p]) + vz[p] * vz[p])) * vref) * vref) / OR_JTOEV;
    /* Cartesian weights sum to 1: corner 2 takes the rest of the particle's
     * 2^40, so every particle deposits its charge exactly; the r-z weights
     * (0.75 below on the axis row) round each corner on its own */
    int64_t q[4];
    for (int c = 0; c < 4; ++c) q[c] = llrint(W[c] * OR_QSCALE);
    if (d->delta != 1) q[2] = ((int64_t)1 << 40) - ((q[0] + q[1]) + q[3]);
    for (int c = 0; c < 4; ++c) {
      const int64_t dq = q[c], de = llrint((W[c] * energy) * OR_ESCALE);
#pragma omp atomic
      q_acc[nd[c]] += dq;
#pragma omp atomic
      e_acc[nd[c]] += de;
    }
  }
  mesh_close(&m);
  return bad;
}

/* GetParChg_2D.f90:869-911: rho_s = Weight*qs*sum/L_ref/L_ref/n_ref/V;
 * rho accumulates over species in order; ek_s = mean energy per particle. */
void or_normalize(const pic_mesh_desc *d, int ns, const int64_t *const *q_acc, const int64_t *const *e_acc,
                  const double *wq, double L_ref, double n_ref, double *rho, double *const *rho_s,
                  double *const *ek_s) {
  int64_t nn = (int64_t)d->nnx * d->nny;
  for (int64_t i = 0; i < nn; ++i) {
    double acc = 0.0, V = d->cell_volume[i];
    for (int s = 0; s < ns; ++s) {
      double cnt = (double)q_acc[s][i] * (1.0 / OR_QSCALE);
      double es = (double)e_acc[s][i] * (1.0 / OR_ESCALE);
      /* one more 1/L_ref for delta 1 (:900-904): the dual volume is a volume */
      double t = ((wq[s] * cnt) / L_ref) / L_ref;
      if (d->delta == 1) t = t / L_ref;
      double r = (t / n_ref) / V;
      rho_s[s][i] = r;
      ek_s[s][i] = (cnt != 0.0) ? es / cnt : 0.0;
      acc = acc + r;
    }
    rho[i] = acc;
  }
}

/* ------------------------------------------------------------------ */
/* IFE_Solve_2D.f90:126-192: b = M rho - rhs_FIX - A_xt phi_D on the full */
/* node grid (Global_RHS_PDE_2D.f90:72-138 element loop; the interface   */
/* elements' load matrices come with the mesh).                           */
/* ------------------------------------------------------------------ */
void or_rhs(const pic_mesh_desc *d, const double *rho, double *b) {
  Mesh m;
  mesh_open(&m, d);
  int64_t nn = m.nn;
  for (int64_t i = 0; i < nn; ++i) b[i] = 0.0;
  for (int ei = 0; ei < m.nex; ++ei)
    for (int ej = 0; ej < m.ney; ++ej) {
      int64_t e = (int64_t)ei * m.ney + ej;
      int id = d->element_index[e];
      /* axisymmetric (Global_RHS_PDE_2D.f90:98): the element row's r-weighted matrix */
      const double *Mreg = (d->delta == 1 && d->mass_rows) ? d->mass_rows + 16 * (size_t)ej : d->mass_q1;
      const double *M = id > 0 ? d->ife_mass + 16 * (size_t)(id - 1) : Mreg;
      int64_t n1 = (int64_t)ei * m.nny + ej;
      int64_t nd[4] = {n1, n1 + m.nny, n1 + m.nny + 1, n1 + 1};
      double R[4] = {rho[nd[0]], rho[nd[1]], rho[nd[2]], rho[nd[3]]};
      for (int j = 0; j < 4; ++j) {
        if (d->node_type[nd[j]] <= 0) continue;
        const double *Mr = M + 4 * j;
        double el = ((Mr[0] * R[0] + Mr[1] * R[1]) + Mr[2] * R[2]) + Mr[3] * R[3];
        b[nd[j]] = b[nd[j]] + el;
      }
    }
  for (int64_t i = 0; i < nn; ++i) {
    int u = d->node_type[i];
    if (u <= 0) continue;
    double ebc = 0.0; /* Global_RHS_EBC_2D_bjw.f90:72-77 */
    for (int q = d->xt_srow[u - 1] - 1; q < d->xt_srow[u] - 1; ++q)
      ebc = ebc + d->phi_dirichlet[d->xt_jcol[q] - 1] * d->xt_k[q];
    double fix = d->rhs_fix ? d->rhs_fix[u - 1] : 0.0;
    b[i] = (b[i] - fix) - ebc;
  }
  mesh_close(&m);
}

/* ------------------------------------------------------------------ */
/* canonical reduction order shared with the GPU dot products           */
/* ------------------------------------------------------------------ */
#define RT 256
#define RI 4
static double butterfly_warp_seq(double *lane_vals /* [RT] */) {
  double ws[RT / 32];
  for (int w = 0; w < RT / 32; ++w) {
    double v[32], nv[32];
    for (int l = 0; l < 32; ++l) v[l] = lane_vals[32 * w + l];
    for (int off = 16; off > 0; off >>= 1) {
      for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ off];
      memcpy(v, nv, sizeof v);
    }
    ws[w] = v[0];
  }
  double s = 0.0;
  for (int w = 0; w < RT / 32; ++w) s = s + ws[w];
  return s;
}

/* sum over blocks of per-block partials (last-block reduction) */
static double final_sum(const double *part, int nb) {
  double t[RT];
  for (int th = 0; th < RT; ++th) {
    double a = 0.0;
    for (int b = th; b < nb; b += RT) a = a + part[b];
    t[th] = a;
  }
  return butterfly_warp_seq(t);
}

/* generic canonical dot: sum fma(a_n, b_n, acc) per thread */
double or_canon_dot(const double *a, const double *b, int64_t n) {
  int nb = (int)((n + RT * RI - 1) / (RT * RI));
  double *part = (double *)malloc(sizeof(double) * (nb > 0 ? nb : 1));
  /* blocks are independent; their partials are summed in block order */
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < nb; ++blk) {
    double t[RT];
    for (int th = 0; th < RT; ++th) {
      double acc = 0.0;
      for (int it = 0; it < RI; ++it) {
        int64_t i = (int64_t)blk * RT * RI + it * RT + th;
        if (i < n) acc = fma(a[i], b[i], acc);
      }
      t[th] = acc;
    }
    part[blk] = butterfly_warp_seq(t);
  }
  double s = final_sum(part, nb);
  free(part);
  return s;
}

/* CSR matvec over the full grid (MATVEC_1.f90:14-22); Dirichlet rows 0 */
static void matvec(const pic_mesh_desc *d, const int64_t *u2n, const double *v, double *y) {
  int64_t nn = (int64_t)d->nnx * d->nny;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nn; ++i) {
    int u = d->node_type[i];
    if (u <= 0) { y[i] = 0.0; continue; }
    double acc = 0.0;
    for (int q = d->a_srow[u - 1] - 1; q < d->a_srow[u] - 1; ++q) acc = fma(d->a_k[q], v[u2n[d->a_jcol[q] - 1]], acc);
    y[i] = acc;
  }
}

/* ------------------------------------------------------------------ */
/* MY_PCG.f90:56-133 (Jacobi preconditioner MSOLVE_1.f90) on full-grid   */
/* vectors; x in: warm start phi, out: phi (Dirichlet nodes from phi_D). */
/* stats: [iterations, ierr, normR, normRHS].                             */
/* ------------------------------------------------------------------ */
void or_pcg(const pic_mesh_desc *d, const double *b, double *phi, double tol, int maxit, double *stats) {
  int64_t nn = (int64_t)d->nnx * d->nny;
  int64_t *u2n = (int64_t *)malloc(sizeof(int64_t) * (d->n_unknowns > 0 ? d->n_unknowns : 1));
  for (int64_t i = 0; i < nn; ++i)
    if (d->node_type[i] > 0) u2n[d->node_type[i] - 1] = i;
  double *x = calloc(nn, 8), *r = calloc(nn, 8), *w = calloc(nn, 8), *p = calloc(nn, 8), *q = calloc(nn, 8),
         *diag = calloc(nn, 8), *tmp = calloc(nn, 8);
  for (int64_t i = 0; i < nn; ++i) {
    int u = d->node_type[i];
    x[i] = u > 0 ? phi[i] : 0.0;
    diag[i] = u > 0 ? d->a_diag[u - 1] : 1.0;
  }
  matvec(d, u2n, x, tmp);
  for (int64_t i = 0; i < nn; ++i) {
    r[i] = d->node_type[i] > 0 ? b[i] - tmp[i] : 0.0;
    w[i] = r[i] / diag[i];
  }
  double normRHS = or_canon_dot(b, b, nn), rho = or_canon_dot(r, w, nn), rho0 = 0.0, beta = 0.0, normR = 0.0;
  double tol2 = tol * tol;
  int iter = 0, ierr = 0, done = !(normRHS > 0.0);
  while (!done) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nn; ++i) p[i] = iter == 0 ? w[i] : fma(beta, p[i], w[i]);
    matvec(d, u2n, p, q);
    double pq = or_canon_dot(p, q, nn);
    if (pq == 0.0) { ierr = 3; break; }
    double alpha = rho / pq;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nn; ++i) {
      x[i] = fma(alpha, p[i], x[i]);
      r[i] = fma(-alpha, q[i], r[i]);
      w[i] = r[i] / diag[i];
    }
    normR = or_canon_dot(r, r, nn);
    rho0 = rho;
    rho = or_canon_dot(r, w, nn);
    ++iter;
    if (normR / normRHS <= tol2) done = 1;
    else if (iter >= maxit) { ierr = 1; done = 1; }
    else if (rho0 == 0.0) { ierr = 2; done = 1; }
    else beta = rho / rho0;
  }
  for (int64_t i = 0; i < nn; ++i) phi[i] = d->node_type[i] > 0 ? x[i] : d->phi_dirichlet[i];
  if (stats) { stats[0] = iter; stats[1] = ierr; stats[2] = normR; stats[3] = normRHS; }
  free(x); free(r); free(w); free(p); free(q); free(diag); free(tmp); free(u2n);
}

/* ------------------------------------------------------------------ */
/* PPR: GetEfield_SIDG_PPR.f90:153-241 with BRINV.f90 (Gauss-Jordan,    */
/* full pivoting).  coef out: [5][nn] = coef_ppr(2..6,:); efx = -coef2.  */
/* ------------------------------------------------------------------ */
static int brinv(double *a, int n) {
  int is[16], js[16];
  for (int k = 0; k < n; ++k) {
    double dmax = 0.0;
    for (int i = k; i < n; ++i)
      for (int j = k; j < n; ++j) {
        double p = fabs(a[i * n + j]);
        if (p > dmax) { dmax = p; is[k] = i; js[k] = j; }
      }
    if (dmax + 1.0 == 1.0) return 0;
    if (is[k] != k) for (int j = 0; j < n; ++j) { double t = a[k * n + j]; a[k * n + j] = a[is[k] * n + j]; a[is[k] * n + j] = t; }
    if (js[k] != k) for (int i = 0; i < n; ++i) { double t = a[i * n + k]; a[i * n + k] = a[i * n + js[k]]; a[i * n + js[k]] = t; }
    a[k * n + k] = 1.0 / a[k * n + k];
    for (int j = 0; j < n; ++j) if (j != k) a[k * n + j] = a[k * n + j] * a[k * n + k];
    for (int i = 0; i < n; ++i)
      if (i != k) for (int j = 0; j < n; ++j) if (j != k) a[i * n + j] = a[i * n + j] - a[i * n + k] * a[k * n + j];
    for (int i = 0; i < n; ++i) if (i != k) a[i * n + k] = -a[i * n + k] * a[k * n + k];
  }
  for (int k = n - 1; k >= 0; --k) {
    if (js[k] != k) for (int j = 0; j < n; ++j) { double t = a[k * n + j]; a[k * n + j] = a[js[k] * n + j]; a[js[k] * n + j] = t; }
    if (is[k] != k) for (int i = 0; i < n; ++i) { double t = a[i * n + k]; a[i * n + k] = a[i * n + is[k]]; a[i * n + is[k]] = t; }
  }
  return 1;
}

void or_ppr(const pic_mesh_desc *d, const double *phi, double *coef, double *efx, double *efy) {
  Mesh m;
  mesh_open(&m, d);
  int64_t nn = m.nn;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < nn; ++i) {
    int b0 = d->patch_ptr[i], cnt = d->patch_ptr[i + 1] - b0;
    double c[5] = {0, 0, 0, 0, 0};
    double xi = m.xs[i / m.nny], yi = m.ys[i % m.nny];
    if (cnt >= 6) {
      double *px = malloc(8 * cnt), *py = malloc(8 * cnt), *AT = malloc(8 * 6 * cnt);
      double h = 0.0;
      for (int q = 0; q < cnt; ++q) {
        int64_t k = d->patch_nodes[b0 + q] - 1;
        px[q] = m.xs[k / m.nny] - xi;
        py[q] = m.ys[k % m.nny] - yi;
        double t = fmax(fabs(px[q]), fabs(py[q]));
        if (t > h) h = t;
      }
      for (int q = 0; q < cnt; ++q) {
        double X = px[q] / h, Y = py[q] / h;
        AT[0 * cnt + q] = 1.0; AT[1 * cnt + q] = X; AT[2 * cnt + q] = Y;
        AT[3 * cnt + q] = X * X; AT[4 * cnt + q] = X * Y; AT[5 * cnt + q] = Y * Y;
      }
      double N[36];
      for (int a = 0; a < 6; ++a)
        for (int bb = 0; bb < 6; ++bb) {
          double s = 0.0;
          for (int q = 0; q < cnt; ++q) s = s + AT[a * cnt + q] * AT[bb * cnt + q];
          N[a * 6 + bb] = s;
        }
      if (brinv(N, 6)) {
        for (int a = 1; a < 6; ++a) {
          double acc = 0.0;
          for (int q = 0; q < cnt; ++q) {
            double P = 0.0;
            for (int bb = 0; bb < 6; ++bb) P = P + N[a * 6 + bb] * AT[bb * cnt + q];
            acc = fma(P, phi[d->patch_nodes[b0 + q] - 1], acc);
          }
          c[a - 1] = (a <= 2) ? acc / h : acc / (h * h);
        }
      }
      free(px); free(py); free(AT);
    }
    for (int k = 0; k < 5; ++k) coef[k * nn + i] = c[k];
    efx[i] = -c[0];
    efy[i] = -c[1];
  }
  mesh_close(&m);
}

/* ------------------------------------------------------------------ */
/* Counting sort by (element, id), dropping absorbed particles.          */
/* perm out: source index of each live particle in sorted order.         */
/* ------------------------------------------------------------------ */
static const int32_t *g_sort_loc;
static const uint32_t *g_sort_id;
static int cmp_sort(const void *a, const void *b) {
  int64_t i = *(const int64_t *)a, j = *(const int64_t *)b;
  if (g_sort_loc[i] != g_sort_loc[j]) return g_sort_loc[i] < g_sort_loc[j] ? -1 : 1;
  return g_sort_id[i] < g_sort_id[j] ? -1 : (g_sort_id[i] > g_sort_id[j]);
}
int64_t or_sort_perm(int64_t n, const int32_t *loc, const uint32_t *id, int64_t *perm) {
  int64_t m = 0;
  for (int64_t p = 0; p < n; ++p)
    if (loc[p] >= 0) perm[m++] = p;
  g_sort_loc = loc;
  g_sort_id = id;
  qsort(perm, m, sizeof(int64_t), cmp_sort);
  return m;
}

/* ------------------------------------------------------------------ */
/* MCC_jw null collision (mc/MCCPublic.F90:35-111) for one species.      */
/* ------------------------------------------------------------------ */
typedef struct {
  uint32_t ctr[4], key[2];
  uint32_t call;
  int have;
  double buf[2];
} Rng;

static double draw(Rng *r) {
  if (r->have == 0) {
    uint32_t c[4] = {r->ctr[0], r->ctr[1], r->ctr[2] | r->call, r->ctr[3]}, o[4];
    or_philox(c, r->key, o);
    r->call++;
    r->buf[0] = u01(o[0], o[1]);
    r->buf[1] = u01(o[2], o[3]);
    r->have = 2;
  }
  double u = r->buf[2 - r->have];
  r->have--;
  return u;
}

/* VelocityRandomInitializationParticleOne (base/ParticleOne.f90) */
static void rand_dir(Rng *r, double V, double v[3]) {
  double R = draw(r);
  double ct = 1.0 - 2.0 * R, st = sqrt(1.0 - ct * ct);
  R = draw(r);
  double fai = 2.0 * OR_PI * R;
  v[0] = V * ct; v[1] = V * st * cos(fai); v[2] = V * st * sin(fai);
}

/* VelocityMaxwellianInitializationParticleOne (base/ParticleOne.f90) */
static void maxwell(Rng *r, double mass, double T, double v[3]) {
  double beta = 1.0 / (OR_KB * T), R = 0.5;
  for (int it = 0; it < 64; ++it) {
    R = draw(r);
    double fa = R * R;
    R = draw(r);
    if (R < 1e-300) R = 1e-300;
    double fb = -((OR_FEXP * R) * log(R));
    if (!(fa > fb)) break;
  }
  rand_dir(r, sqrt(((-3.0 * log(R)) / beta) / mass), v);
}

typedef struct { double gx, gy, gz, gper, g, e, mr; } Rel;

/* PostCollisionVelocity (mc/TypeMCC.f90:101-133); iso=0 CosKaiVahedi, 1 IsotropicCosKai (MCCChi.f90) */
static void post(Rng *r, Rel *s, double v[3], int iso) {
  if (fabs(s->gper) < OR_MINREAL) { rand_dir(r, s->g, v); return; }
  double ct;
  if (!iso) {
    if (s->e < OR_MINREAL) ct = 1.0;
    else { double R = draw(r); ct = ((s->e + 2.0) - 2.0 * pow(s->e + 1.0, R)) / s->e; }
  } else { double R = draw(r); ct = 1.0 - 2.0 * R; }
  double fct = 1.0 - ct, st = sqrt(1.0 - ct * ct);
  double R = draw(r), aphi = 2.0 * OR_PI * R, cp = cos(aphi), sp = sin(aphi);
  double hx = s->gper * cp;
  double hy = -(s->gx * s->gy * cp + s->g * s->gz * sp) / s->gper;
  double hz = -(s->gx * s->gz * cp - s->g * s->gy * sp) / s->gper;
  v[0] = v[0] - s->mr * (s->gx * fct + hx * st);
  v[1] = v[1] - s->mr * (s->gy * fct + hy * st);
  v[2] = v[2] - s->mr * (s->gz * fct + hz * st);
}

/* VelocityUpdater (mc/TypeMCC.f90:84-99) */
static void scale(Rel *s, double v[3], double f) {
  s->gx *= f; s->gy *= f; s->gz *= f; s->gper *= f; s->g *= f;
  v[0] *= f; v[1] *= f; v[2] *= f;
}

/* Selection keys of the null-collision candidates: two 32-bit round keys
 * per (seed, step, species) from one Philox block (purpose byte 1, counter
 * word 0 = 0), and per particle two rounds of C. Wellons' lowbias32 integer
 * hash ("Prospecting for hash functions", 2018), each after an xor of a
 * round key into the id.  A bijection of the id for a fixed step. */
static uint32_t lowbias32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
static void select_round_keys(uint64_t seed, uint64_t step, int32_t species, uint32_t rk[2]) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t c[4] = {0u, (uint32_t)step, (1u << 24) | ((uint32_t)species << 16), (uint32_t)(step >> 32)}, o[4];
  or_philox(c, key, o);
  rk[0] = o[0];
  rk[1] = o[1];
}
static uint32_t select_key(uint32_t id, const uint32_t rk[2]) { return lowbias32(lowbias32(id ^ rk[0]) ^ rk[1]); }

/* the selection keys of n ids at one step (for the statistical tests) */
void or_mcc_select_keys(uint64_t seed, uint64_t step, int32_t species, int64_t n, const uint32_t *id,
                        uint32_t *out) {
  uint32_t rk[2];
  select_round_keys(seed, step, species, rk);
  for (int64_t i = 0; i < n; ++i) out[i] = select_key(id[i], rk);
}

static const uint64_t *g_key_arr;
static int cmp_key(const void *a, const void *b) {
  uint64_t x = g_key_arr[*(const int64_t *)a], y = g_key_arr[*(const int64_t *)b];
  return x < y ? -1 : (x > y);
}

/*
 * One species, one step.  v* are normalised velocities (updated in place);
 * created particles (ionisation) are written, in parent-id order, to
 * new_e (3 per event, normalised, same species) and new_ion (3 per event,
 * SI); parent slots to new_parent.  Returns the number of collisions, or -1.
 * out_counts[r] counts reaction r (0-based).
 */
int64_t or_mcc(const pic_mcc_table *t, const pic_gas *gas, double mass, double vref, uint64_t seed,
               uint64_t step, int32_t species, int64_t n, const int32_t *loc, const uint32_t *id,
               double *vx, double *vy, double *vz, int64_t *out_counts, int64_t *n_new,
               int64_t *new_parent, double *new_e, double *new_ion) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t slo = (uint32_t)step, shi = (uint32_t)(step >> 32);
  int64_t npar = 0;
  for (int64_t p = 0; p < n; ++p) npar += loc[p] >= 0;
  /* SelectParticle (MCCPublic.F90:113-146): N = INT(NPar*P) + Bernoulli(residue) */
  double xcoll = (double)npar * t->collision_ratio;
  int64_t ncoll = (int64_t)xcoll;
  double residue = xcoll - (double)ncoll;
  {
    uint32_t c[4] = {0xFFFFFFFFu, slo, (2u << 24) | ((uint32_t)species << 16), shi}, o[4];
    or_philox(c, key, o);
    if (u01(o[0], o[1]) < residue) ++ncoll;
  }
  for (int r = 0; r < t->n_reaction; ++r) out_counts[r] = 0;
  *n_new = 0;
  if (ncoll <= 0) return 0;
  /* uniform random N-subset: smallest (key, id), the key a keyed hash of
   * the id (or_mcc_select_keys) */
  uint64_t *k64 = malloc(8 * (size_t)n);
  int64_t *idx = malloc(8 * (size_t)npar);
  int64_t m = 0;
  uint32_t rk[2];
  select_round_keys(seed, step, species, rk);
  for (int64_t p = 0; p < n; ++p) {
    if (loc[p] < 0) continue;
    k64[p] = ((uint64_t)select_key(id[p], rk) << 32) | id[p];
    idx[m++] = p;
  }
  g_key_arr = k64;
  qsort(idx, m, sizeof(int64_t), cmp_key);
  int64_t nion = 0;
  int64_t *ion_par = malloc(8 * (size_t)ncoll);
  double *ion_buf = malloc(8 * 6 * (size_t)ncoll);
  for (int64_t c0 = 0; c0 < ncoll; ++c0) {
    int64_t p = idx[c0];
    Rng r;
    r.ctr[0] = id[p]; r.ctr[1] = slo; r.ctr[2] = (3u << 24) | ((uint32_t)species << 16); r.ctr[3] = shi;
    r.key[0] = key[0]; r.key[1] = key[1]; r.call = 0; r.have = 0;
    double v[3] = {vx[p] * vref, vy[p] * vref, vz[p] * vref};
    /* UpdateMCCParticleOne (TypeMCC.f90:58-82) */
    double vt[3];
    maxwell(&r, gas->mass, gas->temperature, vt);
    double miu = mass * gas->mass / (mass + gas->mass);
    Rel s;
    s.mr = gas->mass / (mass + gas->mass);
    s.gx = v[0] - vt[0]; s.gy = v[1] - vt[1]; s.gz = v[2] - vt[2];
    double gt = s.gy * s.gy + s.gz * s.gz;
    s.gper = sqrt(gt);
    double g2 = gt + s.gx * s.gx;
    s.g = sqrt(g2);
    s.e = ((0.5 * miu) * g2) / OR_JTOEV;
    /* SelectProbility (TypeMCC.f90:155-198) */
    double E = s.e, tp[PIC_MAX_REACTIONS];
    double pos = (log10(E) - t->energy_min) / t->energy_interval, cpos = ceil(pos);
    int N = (cpos < -1.0e9) ? -1000000000 : (cpos > 1.0e9 ? 1000000000 : (int)cpos);
    int nr = t->n_reaction, nsg = t->n_sigma;
    for (int j = 0; j < nr; ++j) {
      if (N < 1) tp[j] = t->probability[j];
      else if (N < nsg) {
        double S1 = (double)N - pos, S2 = 1.0 - S1;
        tp[j] = t->probability[(size_t)(N - 1) * nr + j] * S1 + t->probability[(size_t)N * nr + j] * S2;
      } else tp[j] = t->probability[(size_t)(nsg - 1) * nr + j] * E / t->energy_max;
      if (E < t->threshold[j]) tp[j] = 0.0;
    }
    double R = draw(&r);
    int ri = 0;
    for (int j = 0; j < nr; ++j) if (R < tp[j]) { ri = j + 1; break; }
    if (ri > 0) {
      out_counts[ri - 1]++;
      int type = t->reaction_type[ri - 1];
      double thr = t->threshold[ri - 1];
      if (type == 11) post(&r, &s, v, 0);                       /* MCCElectron.F90:21 */
      else if (type == 12) {                                    /* ElectronExcitation */
        double f = sqrt(1.0 - thr / s.e);
        s.e = s.e - thr;
        scale(&s, v, f);
        post(&r, &s, v, 0);
      } else if (type == 13) {                                  /* ElectronIonization */
        double v0[3] = {v[0], v[1], v[2]}, e0 = s.e, et = s.e - thr;
        double Rr = draw(&r);
        double eold = 10.0 * tan(Rr * atan(et) / 20.0);       /* CreatEnergyVehadi */
        if (fabs(eold) < OR_MINREAL) eold = OR_MINREAL;
        scale(&s, v, sqrt(eold / s.e));
        post(&r, &s, v, 0);
        double fn = sqrt((et - eold) / e0);
        ion_par[nion] = ((int64_t)id[p] << 32) | p;
        for (int q = 0; q < 3; ++q) { ion_buf[6 * nion + q] = v0[q] * fn / vref; ion_buf[6 * nion + 3 + q] = vt[q]; }
        ++nion;
      } else if (type == 101) post(&r, &s, v, 1);              /* MCCIon.F90:13-14 */
      else if (type == 103) { v[0] = vt[0]; v[1] = vt[1]; v[2] = vt[2]; } /* charge exchange */
    }
    vx[p] = v[0] / vref; vy[p] = v[1] / vref; vz[p] = v[2] / vref;
  }
  /* creations in parent-id order (MCCAddNewParticle, MCCPublic.F90:173-189) */
  int64_t *ord = malloc(8 * (size_t)(nion > 0 ? nion : 1));
  uint64_t *pk = malloc(8 * (size_t)(nion > 0 ? nion : 1));
  for (int64_t i = 0; i < nion; ++i) { ord[i] = i; pk[i] = (uint64_t)ion_par[i]; }
  g_key_arr = pk;
  qsort(ord, nion, sizeof(int64_t), cmp_key);
  for (int64_t i = 0; i < nion; ++i) {
    int64_t o = ord[i];
    new_parent[i] = ion_par[o] & 0xffffffff;
    for (int q = 0; q < 3; ++q) { new_e[3 * i + q] = ion_buf[6 * o + q]; new_ion[3 * i + q] = ion_buf[6 * o + 3 + q]; }
  }
  *n_new = nion;
  free(ord); free(pk); free(ion_par); free(ion_buf); free(k64); free(idx);
  return ncoll;
}

/* ------------------------------------------------------------------ */
/* Closed-form Q1 IFE reference basis, isotropic coefficient            */
/* (k11 = k22 = 1, k12 = k21 = 0) of Retangular_reference_basis_IFE.f90. */
/* Returns C1..C4 of basis `bi` (1..4) on piece `pf` (1..2) for element  */
/* type `typ` (1 corner cut, 2 opposite edges), ratio R = beta1/beta2.    */
/* Implemented for the entries the tests use.                             */
/* ------------------------------------------------------------------ */
int or_ife_closed_form(int typ, int bi, int pf, double a, double b, double R, double C[4]) {
  if (typ == 1) {
    double bottom = 2 * R * (a * a + b * b) + (1 - R) * a * b * (2 * b - b * b + 2 * a - a * a);
    double c1 = 2 * R * (a * a + b * b) / bottom;
    if (bi == 1 && pf == 2) { C[0] = c1; C[1] = -c1; C[2] = -c1; C[3] = c1; return 1; }
    if (bi == 1 && pf == 1) {
      C[0] = 1;
      C[1] = (b * b * b - 2 * b * b - 2 * a * b - 2 * R * a * a - R * b * b * b + (a * a) * b -
              R * (a * a) * b + 2 * R * a * b) / bottom;
      C[2] = (a * a * a - 2 * a * a - 2 * a * b - R * a * a * a - 2 * R * b * b + a * (b * b) -
              R * a * (b * b) + 2 * R * a * b) / bottom;
      C[3] = 2 * R * (a * a + b * b) / bottom;
      return 1;
    }
    if (bi == 3 && pf == 2) {
      double k = (a * (b * b * b) + (a * a * a) * b - R * a * (b * b * b) - R * (a * a * a) * b) / bottom;
      C[0] = k; C[1] = -k; C[2] = -k; C[3] = 1 + k;
      return 1;
    }
    return 0;
  }
  if (typ == 2) {
    double bottom = 2 * R + a + b - (a * a * a) - (b * b * b) + 2 * (a * a) + 2 * (b * b) - R * a - R * b +
                    R * (a * a * a) + R * (b * b * b) - 4 * a * b + a * (b * b) + (a * a) * b -
                    R * a * (b * b) - R * (a * a) * b;
    if (bi == 2 && pf == 2) {
      double c1 = (a - (a * a * a) - R * a + R * (a * a * a) + a * (b * b) - R * a * (b * b)) / bottom;
      double c3 = (b - a + (a * a * a) + (b * b * b) + R * a - R * b - R * (a * a * a) - R * (b * b * b) -
                   a * (b * b) - (a * a) * b + R * a * (b * b) + R * (a * a) * b) / bottom;
      C[0] = c1; C[1] = 1 - c1; C[2] = c3; C[3] = -c3 - 1;
      return 1;
    }
    return 0;
  }
  return 0;
}

/* Host threads the oracle's parallel loops use (OpenMP; 1 without it). */
int or_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* Diagnostics                                                          */
/* ------------------------------------------------------------------ */

/* GetParChg_2D.f90:880-904 (delta = 0): node energy density of one species,
 * Ek_tot = Weight * sum(W*E) / L_ref / L_ref / n_ref / V, from the
 * fixed-point energy sums of or_deposit. */
void or_ek_tot(const pic_mesh_desc *d, const int64_t *e_acc, double weight, double L_ref, double n_ref,
               double *ek_tot) {
  int64_t nn = (int64_t)d->nnx * d->nny;
  for (int64_t i = 0; i < nn; ++i) {
    double es = (double)e_acc[i] * (1.0 / OR_ESCALE);
    double t = ((weight * es) / L_ref) / L_ref;
    if (d->delta == 1) t = t / L_ref;
    ek_tot[i] = (t / n_ref) / d->cell_volume[i];
  }
}

/* Output_To_Tecplot_IJK_2D.f90:184-215 (Average_x): the nodes with x = x_i
 * are column i of the grid, visited in node order (j ascending); their sum
 * divided by their count, times the output scale of :220-223. */
void or_average_x(int nnx, int nny, const double *f, double scale, double *out) {
  for (int i = 0; i < nnx; ++i) {
    double s = 0.0;
    int count = 0;
    for (int j = 0; j < nny; ++j) {
      s = s + f[(int64_t)i * nny + j];
      count = count + 1;
    }
    out[i] = (s / (double)count) * scale;
  }
}

/* Output_Energy.f90:41-71: bin edges Ek_per(i+1) = Ek_max*REAL(i)/N and
 * Vk_per(i+1) = Vk_max*REAL(i-(0.5*N))/N (REAL: single precision, exact
 * here), i = 0..N; a particle counts in bin b when edge(b) < value <=
 * edge(b+1), tested against every bin as the reference does.  Energy:
 * EnergyParticleOne (base/ParticleOne.f90:235-244) times VFactor^2, / JtoeV.
 * Only live particles (loc >= 0). */
void or_energy_spectrum(int64_t n, const double *vx, const double *vy, const double *vz, const int32_t *loc,
                        double mass, double vref, int nbins, double e_max, double v_max, int64_t *count_e,
                        int64_t *count_vx) {
  double *ee = (double *)malloc(sizeof(double) * (nbins + 1));
  double *ve = (double *)malloc(sizeof(double) * (nbins + 1));
  for (int i = 0; i <= nbins; ++i) {
    ee[i] = (e_max * (double)(float)i) / (double)nbins;
    ve[i] = (v_max * (double)((float)i - 0.5f * (float)nbins)) / (double)nbins;
  }
  for (int b = 0; b < nbins; ++b) count_e[b] = count_vx[b] = 0;
  for (int64_t p = 0; p < n; ++p) {
    if (loc[p] < 0) continue;
    double e = ((((0.5 * mass) * ((vx[p] * vx[p] + vy[p] * vy[p]) + vz[p] * vz[p])) * vref) * vref) / OR_JTOEV;
    double v = vx[p];
    for (int b = 0; b < nbins; ++b) {
      if (e <= ee[b + 1] && e > ee[b]) count_e[b] += 1;
      if (v <= ve[b + 1] && v > ve[b]) count_vx[b] += 1;
    }
  }
  free(ee);
  free(ve);
}

/* OUTPUT_velocity.f90:48-103: column num = MIN(MAX(1, FLOOR(X)+1), N)
 * (0-based here); pass 1 sums vx, vy, vz and counts per column, drift =
 * sum/count (0 for an empty column); pass 2 sums (v - drift)^2, thermal =
 * sqrt(that/count).  FP64 sums in particle order (the reference's are FP32).
 * drift, thermal: [3][nbins]. */
void or_velocity_moments(int64_t n, const double *x, const double *vx, const double *vy, const double *vz,
                         const int32_t *loc, int nbins, int64_t *count, double *drift, double *thermal) {
  const double *v[3] = {vx, vy, vz};
  double *sum = (double *)calloc((size_t)3 * nbins, sizeof(double));
  for (int b = 0; b < nbins; ++b) count[b] = 0;
  for (int pass = 0; pass < 2; ++pass) {
    for (int b = 0; b < 3 * nbins; ++b) sum[b] = 0.0;
    for (int64_t p = 0; p < n; ++p) {
      if (loc[p] < 0) continue;
      double f = floor(x[p]);
      int b = (f >= 0.0) ? ((f >= (double)(nbins - 1)) ? nbins - 1 : (int)f) : 0;
      if (pass == 0) count[b] += 1;
      for (int c = 0; c < 3; ++c) {
        double t = v[c][p];
        if (pass == 1) {
          double dd = t - drift[c * nbins + b];
          t = dd * dd;
        }
        sum[c * nbins + b] = sum[c * nbins + b] + t;
      }
    }
    double *out = pass == 0 ? drift : thermal;
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < nbins; ++b) {
        double r = 0.0;
        if (count[b] != 0) {
          r = sum[c * nbins + b] / (double)count[b];
          if (pass == 1) r = sqrt(r);
        }
        out[c * nbins + b] = r;
      }
  }
  free(sum);
}
