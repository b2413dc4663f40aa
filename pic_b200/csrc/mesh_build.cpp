// mesh_build.cpp -- host-side mesh builder for the IFE-PIC step.
//
// Produces the arrays that the reference's setup phase leaves in its
// IFE_Data module, for a uniform Q1 rectangular mesh with immersed circles,
// ellipses and boxes.  Every array keeps the reference's meaning; the code is
// organised around the regular grid instead of the reference's element lists.
//
//   node/element numbering ........ code/IFE-Rectangular/Cubic_Partition_2D.f90:40-90
//   node_type (unknown numbering) . code/IFE-Rectangular/Partition_Cube_2D.f90:20-60
//   interface element geometry .... code/IFE-Rectangular/El_Object_Intersection_info_2D_BL.f90:330-980
//   Q1 IFE basis ................... code/IFE-Rectangular/Retangular_reference_basis_IFE.f90,
//                                    code/IFE-Rectangular/retangular_local_basis_IFE.f90
//   element stiffness + assembly ... code/IFE-Rectangular/Generate_stiffness_matrix_local_IFE.f90:104-200,
//                                    code/IFE-Rectangular/Gauss_integration_local_stiffness_IFE.f90
//   load (RHS) matrices ............ code/IFE-Rectangular/Global_RHS_PDE_2D.f90:72-138,
//                                    code/IFE-Rectangular/IFE_RHS_2D.f90, Linear_IFE_Basis_Coeff_2D.f90,
//                                    Inter_Tetra_Partition_2D.f90
//   dual-cell volume ............... code/Setup/SetupGrids_2D_QLL.f90:197-330
//   PPR patches .................... code/PPR/Get_PointPatch.f90
//
// The Q1 IFE basis is obtained by solving its defining 8x8 conditions (nodal
// values, continuity at the two cut points, equal xi*eta coefficients, flux
// continuity across the cut) instead of the reference's closed-form
// expressions; both describe the same unique basis, and the oracle checks the
// two against each other.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/picgpu.h"
#include "ife_elem.h"

namespace pic {
void set_error(const std::string &msg);
// ife_dev.cu: basis, stiffness and load matrix of n interface elements on the
// current CUDA device (FP64, the code of ife_elem.h); 0 or a PIC_ERR_* code
int ife_elements_device(IfeElem *elems, int n, int axi, double *K, double *M);
}
using pic::IfeElem;

namespace {


struct MeshStore {
  pic_mesh_desc desc;
  std::vector<int32_t> node_type, node_index, element_index;
  std::vector<double> phi_dirichlet, cell_volume;
  std::vector<int32_t> a_srow, a_jcol, xt_srow, xt_jcol;
  std::vector<double> a_k, xt_k, a_diag, rhs_fix, mass_q1, ife_mass, mass_rows;
  std::vector<int32_t> patch_ptr, patch_nodes;
  std::vector<pic_object> objects;
  std::vector<IfeElem> ife;
  std::vector<double> xs, ys;
};

bool inside_object(const pic_object &o, double x, double y) {
  switch (o.shape) {
    case PIC_SHAPE_CIRCLE: {
      double dx = x - o.cx, dy = y - o.cy;
      return dx * dx + dy * dy < o.a * o.a;
    }
    case PIC_SHAPE_ELLIPSE: {
      double c = std::cos(o.angle), s = std::sin(o.angle);
      double u = (x - o.cx) * c + (y - o.cy) * s;
      double v = -(x - o.cx) * s + (y - o.cy) * c;
      return (u * u) / (o.a * o.a) + (v * v) / (o.b * o.b) < 1.0;
    }
    case PIC_SHAPE_BOX:
      return x > o.cx && x < o.a && y > o.cy && y < o.b;
    default:
      return false;
  }
}

// Parameter t in (0,1) where segment P1->P2 crosses the object boundary.
bool edge_crossing(const pic_object &o, const double P1[2], const double P2[2], double *t) {
  double dx = P2[0] - P1[0], dy = P2[1] - P1[1];
  if (o.shape == PIC_SHAPE_CIRCLE || o.shape == PIC_SHAPE_ELLIPSE) {
    // f(t) = A t^2 + B t + C on the segment (ellipse in its own frame).
    double c = 1, s = 0, ia2, ib2;
    if (o.shape == PIC_SHAPE_ELLIPSE) {
      c = std::cos(o.angle);
      s = std::sin(o.angle);
      ia2 = 1.0 / (o.a * o.a);
      ib2 = 1.0 / (o.b * o.b);
    } else {
      ia2 = ib2 = 1.0 / (o.a * o.a);
    }
    double u0 = (P1[0] - o.cx) * c + (P1[1] - o.cy) * s;
    double v0 = -(P1[0] - o.cx) * s + (P1[1] - o.cy) * c;
    double du = dx * c + dy * s, dv = -dx * s + dy * c;
    double A = du * du * ia2 + dv * dv * ib2;
    double B = 2.0 * (u0 * du * ia2 + v0 * dv * ib2);
    double C = u0 * u0 * ia2 + v0 * v0 * ib2 - 1.0;
    double disc = B * B - 4 * A * C;
    if (disc < 0 || A <= 0) return false;
    double sq = std::sqrt(disc);
    // numerically stable roots
    double q = -0.5 * (B + (B >= 0 ? sq : -sq));
    double r1 = q / A, r2 = (q != 0) ? C / q : r1;
    double best = -1;
    for (double r : {r1, r2})
      if (r > 0 && r < 1) best = (best < 0) ? r : std::min(best, r);
    if (best < 0) return false;
    *t = best;
    return true;
  }
  if (o.shape == PIC_SHAPE_BOX) {
    // axis-aligned edges only: crossing where the moving coordinate meets a box side
    double cand[4] = {o.cx, o.a, o.cy, o.b};
    for (int k = 0; k < 4; ++k) {
      double num, den;
      if (k < 2) { num = cand[k] - P1[0]; den = dx; }
      else { num = cand[k] - P1[1]; den = dy; }
      if (den == 0) continue;
      double tt = num / den;
      if (tt > 0 && tt < 1) {
        double px = P1[0] + tt * dx, py = P1[1] + tt * dy;
        bool on = (k < 2) ? (py >= o.cy && py <= o.b) : (px >= o.cx && px <= o.a);
        if (on) { *t = tt; return true; }
      }
    }
    return false;
  }
  return false;
}

}  // namespace

extern "C" {

static int mesh_build(const pic_deck *deck, pic_mesh_desc **out, bool device) {
  if (!deck || !out) return PIC_ERR_ARG;
  *out = nullptr;
  const int nnx = deck->nnx, nny = deck->nny;
  if (nnx < 3 || nny < 3 || deck->xmax <= deck->xmin || deck->ymax <= deck->ymin ||
      deck->n_objects < 0 || deck->n_objects > PIC_MAX_OBJECTS) {
    pic::set_error("pic_mesh_build: bad mesh extent or object count");
    return PIC_ERR_ARG;
  }
  if (deck->delta != 0 && deck->delta != 1) {
    pic::set_error("pic_mesh_build: delta must be 0 (Cartesian) or 1 (axisymmetric)");
    return PIC_ERR_ARG;
  }
  const bool axi = deck->delta == 1;
  MeshStore *S = new (std::nothrow) MeshStore();
  if (!S) return PIC_ERR_ARG;
  const int64_t nn = (int64_t)nnx * nny;
  const int nex = nnx - 1, ney = nny - 1;
  const int64_t ne = (int64_t)nex * ney;
  // Node coordinates as in Cubic_Partition_2D.f90:40-48: x_s + h_x*(count-1).
  const double hx = (deck->xmax - deck->xmin) / (nnx - 1);
  const double hy = (deck->ymax - deck->ymin) / (nny - 1);
  S->xs.resize(nnx);
  S->ys.resize(nny);
  for (int i = 0; i < nnx; ++i) S->xs[i] = deck->xmin + hx * i;
  for (int j = 0; j < nny; ++j) S->ys[j] = deck->ymin + hy * j;
  auto X = [&](int i) { return S->xs[i]; };
  auto Y = [&](int j) { return S->ys[j]; };
  auto node = [&](int i, int j) { return (int64_t)i * nny + j; };
  auto elem = [&](int i, int j) { return (int64_t)i * ney + j; };
  S->objects.assign(deck->objects, deck->objects + deck->n_objects);

  // ---- node_index: -1 outside, -(k+2) inside object k
  S->node_index.assign(nn, -1);
  for (int i = 0; i < nnx; ++i)
    for (int j = 0; j < nny; ++j)
      for (int k = 0; k < deck->n_objects; ++k)
        if (inside_object(deck->objects[k], X(i), Y(j))) {
          if (S->node_index[node(i, j)] != -1) {
            pic::set_error("pic_mesh_build: objects overlap at a node");
            delete S;
            return PIC_ERR_SETUP;
          }
          S->node_index[node(i, j)] = -(k + 2);
        }

  // ---- node_type / Dirichlet values (Partition_Cube_2D.f90:32-58).
  // Corner nodes of two Dirichlet walls take the left/right wall value.
  S->node_type.assign(nn, 0);
  S->phi_dirichlet.assign(nn, 0.0);
  std::vector<char> dir(nn, 0);
  for (int i = 0; i < nnx; ++i)
    for (int j = 0; j < nny; ++j) {
      int64_t n = node(i, j);
      int side = -1;
      if (i == 0 && deck->wall_dirichlet[0]) side = 0;
      else if (i == nnx - 1 && deck->wall_dirichlet[1]) side = 1;
      else if (j == 0 && deck->wall_dirichlet[2]) side = 2;
      else if (j == nny - 1 && deck->wall_dirichlet[3]) side = 3;
      if (side >= 0) { dir[n] = 1; S->phi_dirichlet[n] = deck->wall_phi[side]; }
      int reg = S->node_index[n];
      if (reg <= -2 && deck->objects[-reg - 2].conductor) {
        dir[n] = 1;
        S->phi_dirichlet[n] = deck->objects[-reg - 2].phi;
      }
    }
  int32_t n_unknowns = 0;
  for (int64_t n = 0; n < nn; ++n) S->node_type[n] = dir[n] ? -1 : ++n_unknowns;

  // ---- element_index and interface elements
  S->element_index.assign(ne, -1);
  std::vector<double> elem_beta(ne, 1.0);  // permittivity of non-interface elements
  const int loc_di[4] = {0, 1, 1, 0}, loc_dj[4] = {0, 0, 1, 1};
  for (int i = 0; i < nex; ++i)
    for (int j = 0; j < ney; ++j) {
      int64_t e = elem(i, j);
      int lab[4];
      for (int c = 0; c < 4; ++c) lab[c] = S->node_index[node(i + loc_di[c], j + loc_dj[c])];
      int obj = -1;
      bool mixed = false;
      for (int c = 0; c < 4; ++c) {
        if (lab[c] != lab[0]) mixed = true;
        if (lab[c] <= -2) {
          if (obj >= 0 && obj != -lab[c] - 2) {
            pic::set_error("pic_mesh_build: two objects meet inside one element");
            delete S;
            return PIC_ERR_SETUP;
          }
          obj = -lab[c] - 2;
        }
      }
      if (!mixed) {
        S->element_index[e] = lab[0];
        elem_beta[e] = (lab[0] <= -2) ? deck->objects[-lab[0] - 2].eps : 1.0;
        if (lab[0] <= -2 && deck->objects[-lab[0] - 2].conductor) elem_beta[e] = 1.0;
        continue;
      }
      const pic_object &o = deck->objects[obj];
      if (o.conductor) {  // cut by a conductor: plain Q1 element, Dirichlet nodes inside
        S->element_index[e] = -1;
        elem_beta[e] = 1.0;
        continue;
      }
      IfeElem f;
      f.elem = (int)e;
      double P[4][2];
      bool ins[4];
      int n_in = 0;
      for (int c = 0; c < 4; ++c) {
        P[c][0] = X(i + loc_di[c]);
        P[c][1] = Y(j + loc_dj[c]);
        ins[c] = lab[c] <= -2;
        n_in += ins[c];
      }
      // cut points on local edges c -> c+1
      double cut[4][2];
      bool has_cut[4] = {false, false, false, false};
      int n_cut = 0;
      for (int c = 0; c < 4; ++c) {
        int d = (c + 1) & 3;
        if (ins[c] == ins[d]) continue;
        double t;
        if (!edge_crossing(o, P[c], P[d], &t) || t < 1e-10 || t > 1 - 1e-10) {
          char buf[160];
          snprintf(buf, sizeof buf,
                   "pic_mesh_build: interface through a vertex or not found in element %lld",
                   (long long)e + 1);
          pic::set_error(buf);
          delete S;
          return PIC_ERR_SETUP;
        }
        cut[c][0] = P[c][0] + t * (P[d][0] - P[c][0]);
        cut[c][1] = P[c][1] + t * (P[d][1] - P[c][1]);
        has_cut[c] = true;
        ++n_cut;
      }
      if (n_cut != 2) {
        pic::set_error("pic_mesh_build: element cut on more than two edges");
        delete S;
        return PIC_ERR_SETUP;
      }
      int r1;
      if (n_in == 1 || n_in == 3) {
        f.type = 1;
        r1 = 0;
        for (int c = 0; c < 4; ++c) {
          int cnt = 0;
          for (int q = 0; q < 4; ++q) cnt += (ins[q] == ins[c]);
          if (cnt == 1) r1 = c;
        }
      } else {
        f.type = 2;
        // cut edges opposite; reference edges 1-2 and 4-3 are the cut ones.
        // The reference's case table (El_Object_Intersection_info_2D_BL.f90)
        // takes local corner 1 as reference vertex 1 when edges 1-2 and 3-4
        // are cut, local corner 4 when edges 2-3 and 4-1 are.  The choice
        // fixes the sub-triangles of the load-matrix quadrature, which is not
        // exact for r-weighted integrands, so it is the reference's here.
        if (has_cut[0] && has_cut[2]) r1 = 0;
        else if (has_cut[1] && has_cut[3]) r1 = 3;
        else {
          pic::set_error("pic_mesh_build: saddle-type interface element is not supported");
          delete S;
          return PIC_ERR_SETUP;
        }
      }
      for (int r = 0; r < 4; ++r) {
        f.ref2loc[r] = (r1 + r) & 3;
        f.X[r][0] = P[f.ref2loc[r]][0];
        f.X[r][1] = P[f.ref2loc[r]][1];
      }
      // E on reference edge 1-2 (local edge r1), D on edge 1-4 (type 1) or 4-3 (type 2)
      int eE = r1, eD = (f.type == 1) ? ((r1 + 3) & 3) : ((r1 + 2) & 3);
      f.E[0] = cut[eE][0]; f.E[1] = cut[eE][1];
      f.D[0] = cut[eD][0]; f.D[1] = cut[eD][1];
      double beta_in = o.eps, beta_out = 1.0;
      f.beta[0] = ins[f.ref2loc[0]] ? beta_in : beta_out;
      f.beta[1] = ins[f.ref2loc[0]] ? beta_out : beta_in;
      {
        const double x1 = f.X[0][0], y1 = f.X[0][1], x2 = f.X[1][0], y2 = f.X[1][1];
        const double x4 = f.X[3][0], y4 = f.X[3][1];
        double bottom = (x2 - x1) * (y4 - y1) - (x4 - x1) * (y2 - y1);
        f.a = ((y4 - y1) * (f.E[0] - x1) - (x4 - x1) * (f.E[1] - y1)) / bottom;
        if (f.type == 1) f.b = ((x2 - x1) * (f.D[1] - y1) - (y2 - y1) * (f.D[0] - x1)) / bottom;
        else f.b = ((y4 - y1) * (f.D[0] - x1) - (x4 - x1) * (f.D[1] - y1)) / bottom;
      }
      S->ife.push_back(f);
      S->element_index[e] = (int32_t)S->ife.size();
    }

  // ---- the interface elements' basis, stiffness and load matrices: on the
  // CUDA device (pic_mesh_build_device) or here, with the same code
  std::vector<double> Kife(16 * S->ife.size()), Mife(16 * S->ife.size());
  if (device && !S->ife.empty()) {
    int rc = pic::ife_elements_device(S->ife.data(), (int)S->ife.size(), axi ? 1 : 0, Kife.data(), Mife.data());
    if (rc) {
      delete S;
      return rc;
    }
  } else {
    for (size_t k = 0; k < S->ife.size(); ++k) {
      const int st = pic::ife_element_all(S->ife[k], axi ? 1 : 0, &Kife[16 * k], &Mife[16 * k]);
      if (st) {
        pic::set_error(st == 1 ? "pic_mesh_build: singular IFE basis system"
                               : "pic_mesh_build: singular interface load-matrix system");
        delete S;
        return PIC_ERR_SETUP;
      }
    }
  }

  // ---- element stiffness + assembly into CSR (A over unknowns, A_xt to Dirichlet nodes)
  // Row structure: unknown/Dirichlet nodes of the 3x3 neighbourhood, ascending.
  S->a_srow.assign(n_unknowns + 1, 0);
  S->xt_srow.assign(n_unknowns + 1, 0);
  std::vector<int64_t> row_of_node(nn, -1);
  {
    int64_t cnt = 0, cnt_xt = 0;
    int32_t u = 0;
    for (int i = 0; i < nnx; ++i)
      for (int j = 0; j < nny; ++j) {
        int64_t n = node(i, j);
        if (S->node_type[n] < 0) continue;
        S->a_srow[u] = (int32_t)(cnt + 1);
        S->xt_srow[u] = (int32_t)(cnt_xt + 1);
        for (int di = -1; di <= 1; ++di)
          for (int dj = -1; dj <= 1; ++dj) {
            int ii = i + di, jj = j + dj;
            if (ii < 0 || jj < 0 || ii >= nnx || jj >= nny) continue;
            int64_t m = node(ii, jj);
            if (S->node_type[m] > 0) {
              S->a_jcol.push_back(S->node_type[m]);
              ++cnt;
            } else {
              S->xt_jcol.push_back((int32_t)(m + 1));
              ++cnt_xt;
            }
          }
        row_of_node[n] = u++;
      }
    S->a_srow[u] = (int32_t)(cnt + 1);
    S->xt_srow[u] = (int32_t)(cnt_xt + 1);
    S->a_k.assign(cnt, 0.0);
    S->xt_k.assign(cnt_xt, 0.0);
  }
  // Q1 element stiffness of an hx x hy rectangle, HT order, per unit beta.
  double Kq1[4][4];
  {
    const double Kx[4][4] = {{2, -2, -1, 1}, {-2, 2, 1, -1}, {-1, 1, 2, -2}, {1, -1, -2, 2}};
    const double Ky[4][4] = {{2, 1, -1, -2}, {1, 2, -2, -1}, {-1, -2, 2, 1}, {-2, -1, 1, 2}};
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) Kq1[a][b] = (hy / hx * Kx[a][b] + hx / hy * Ky[a][b]) / 6.0;
  }
  // Axisymmetric (r = y): the Q1 stiffness and load matrices of element row j
  // weighted by r (Gauss_integration_local_stiffness.f90:88,
  // Global_RHS_PDE_2D.f90:98), by 2x2 Gauss-Legendre, exact for these
  // degrees (quadratic x linear).  HT order: (0,0), (1,0), (1,1), (0,1).
  std::vector<double> Kaxi, Maxi;
  if (axi) {
    Kaxi.assign((size_t)16 * ney, 0.0);
    Maxi.assign((size_t)16 * ney, 0.0);
    const double gq = 0.5 / std::sqrt(3.0), t[2] = {0.5 - gq, 0.5 + gq};
    for (int j = 0; j < ney; ++j) {
      const double r0 = Y(j), hr = Y(j + 1) - Y(j);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          const double xi = t[a], et = t[b], r = r0 + hr * et, w = 0.25 * hx * hr * r;
          const double X1[4] = {1 - xi, xi, xi, 1 - xi}, R1[4] = {1 - et, 1 - et, et, et};
          const double dX[4] = {-1 / hx, 1 / hx, 1 / hx, -1 / hx}, dR[4] = {-1 / hr, -1 / hr, 1 / hr, 1 / hr};
          for (int p = 0; p < 4; ++p)
            for (int q = 0; q < 4; ++q) {
              Kaxi[16 * j + 4 * p + q] += w * (dX[p] * R1[p] * dX[q] * R1[q] + X1[p] * dR[p] * X1[q] * dR[q]);
              Maxi[16 * j + 4 * p + q] += w * (X1[p] * R1[p]) * (X1[q] * R1[q]);
            }
        }
    }
  }
  auto find_col = [&](const std::vector<int32_t> &srow, const std::vector<int32_t> &jcol,
                      int64_t r, int32_t col) -> int64_t {
    for (int64_t m = srow[r] - 1; m < srow[r + 1] - 1; ++m)
      if (jcol[m] == col) return m;
    return -1;
  };
  for (int i = 0; i < nex; ++i)
    for (int j = 0; j < ney; ++j) {
      int64_t e = elem(i, j);
      double K[4][4];
      int32_t eid = S->element_index[e];
      if (eid > 0) {
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b) K[a][b] = Kife[16 * (size_t)(eid - 1) + 4 * a + b];
      } else {
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b)
            K[a][b] = elem_beta[e] * (axi ? Kaxi[16 * j + 4 * a + b] : Kq1[a][b]);
      }
      int64_t nodes[4];
      for (int c = 0; c < 4; ++c) nodes[c] = node(i + loc_di[c], j + loc_dj[c]);
      for (int k = 0; k < 4; ++k) {
        if (S->node_type[nodes[k]] <= 0) continue;
        int64_t r = row_of_node[nodes[k]];
        for (int q = 0; q < 4; ++q) {
          if (S->node_type[nodes[q]] > 0) {
            int64_t m = find_col(S->a_srow, S->a_jcol, r, S->node_type[nodes[q]]);
            S->a_k[m] += K[k][q];
          } else {
            int64_t m = find_col(S->xt_srow, S->xt_jcol, r, (int32_t)(nodes[q] + 1));
            S->xt_k[m] += K[k][q];
          }
        }
      }
    }
  S->a_diag.assign(n_unknowns, 0.0);
  for (int32_t u = 0; u < n_unknowns; ++u)
    for (int64_t m = S->a_srow[u] - 1; m < S->a_srow[u + 1] - 1; ++m)
      if (S->a_jcol[m] == u + 1) S->a_diag[u] = S->a_k[m];
  S->rhs_fix.assign(n_unknowns, 0.0);

  // ---- load matrices
  S->mass_q1.resize(16);
  {
    const double w[4][4] = {{4, 2, 1, 2}, {2, 4, 2, 1}, {1, 2, 4, 2}, {2, 1, 2, 4}};
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) S->mass_q1[a * 4 + b] = hx * hy * w[a][b] / 36.0;
  }
  S->ife_mass = Mife;

  if (axi) S->mass_rows = Maxi;

  // ---- dual-cell volume (Cartesian): corners hx*hy/4, edges hx*hy/2, interior hx*hy
  S->cell_volume.assign(nn, 0.0);
  for (int i = 0; i < nnx; ++i)
    for (int j = 0; j < nny; ++j) {
      int ie = std::min(i, nnx - 2), je = std::min(j, nny - 2);
      double hxp = X(ie + 1) - X(ie), hyp = Y(je + 1) - Y(je);
      bool bx = (i == 0 || i == nnx - 1), by = (j == 0 || j == nny - 1);
      if (!axi) {
        double div = (bx && by) ? 4.0 : ((bx || by) ? 2.0 : 1.0);
        S->cell_volume[node(i, j)] = hxp * hyp / div;
        continue;
      }
      // axisymmetric (SetupGrids_2D_QLL.f90:233-289): rings of the dual cell,
      // r = y; on r = ymin / ymax the half cell's mean radius R +- hy/4
      const double pi = 3.14159265358979, y = Y(j);
      double v;
      if (j == 0) v = 2.0 * pi * (deck->ymin + hyp / 4.0) * (hyp / 2.0) * hxp;
      else if (j == nny - 1) v = 2.0 * pi * (deck->ymax - hyp / 4.0) * (hyp / 2.0) * hxp;
      else v = 2.0 * pi * y * hyp * hxp;
      if (bx) v = v / 2.0;  // on the z walls (and at the corners) half the cell
      S->cell_volume[node(i, j)] = v;
    }

  // ---- PPR patches (Get_PointPatch.f90)
  {
    std::vector<std::vector<int32_t>> patch(nn), base(nn);
    std::vector<int> kind(nn, 0);  // 1 interior regular, 2 boundary, 3 interface
    for (int i = 0; i < nnx; ++i)
      for (int j = 0; j < nny; ++j) {
        int64_t n = node(i, j);
        // adjacent elements: SW, SE, NE, NW (part_ex_1..4)
        int64_t ex[4] = {-1, -1, -1, -1};
        if (i > 0 && j > 0) ex[0] = elem(i - 1, j - 1);
        if (i < nex && j > 0) ex[1] = elem(i, j - 1);
        if (i < nex && j < ney) ex[2] = elem(i, j);
        if (i > 0 && j < ney) ex[3] = elem(i - 1, j);
        std::vector<int64_t> pe;
        bool boundary = (i == 0 || j == 0 || i == nnx - 1 || j == nny - 1);
        if (boundary) {
          kind[n] = 2;
          for (int c = 0; c < 4; ++c)
            if (ex[c] >= 0) pe.push_back(ex[c]);
        } else {
          bool all_in = true, all_out = true;
          for (int c = 0; c < 4; ++c) {
            all_in = all_in && S->element_index[ex[c]] == -2;
            all_out = all_out && S->element_index[ex[c]] == -1;
          }
          if (all_in || all_out) {
            kind[n] = 1;
            for (int c = 0; c < 4; ++c) pe.push_back(ex[c]);
          } else {
            kind[n] = 3;
            for (int c = 0; c < 4; ++c)
              if (S->element_index[ex[c]] < 0) pe.push_back(ex[c]);
          }
        }
        std::vector<int32_t> nodes;
        for (int64_t e : pe) {
          int ei = (int)(e / ney), ej = (int)(e % ney);
          for (int c = 0; c < 4; ++c) nodes.push_back((int32_t)node(ei + loc_di[c], ej + loc_dj[c]));
        }
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        base[n] = nodes;
        patch[n] = nodes;
      }
    auto union_of = [&](const std::vector<int32_t> &src) {
      std::vector<int32_t> u;
      for (int32_t k : src) u.insert(u.end(), base[k].begin(), base[k].end());
      std::sort(u.begin(), u.end());
      u.erase(std::unique(u.begin(), u.end()), u.end());
      return u;
    };
    for (int64_t n = 0; n < nn; ++n)  // extend patches with fewer than 6 nodes
      if (!patch[n].empty() && patch[n].size() < 6) {
        auto u = union_of(base[n]);
        if (!u.empty()) patch[n] = u;
      }
    for (int64_t n = 0; n < nn; ++n)  // boundary / interface nodes below 12 nodes
      if ((kind[n] == 2 || kind[n] == 3) && patch[n].size() < 12 && !base[n].empty()) {
        auto u = union_of(base[n]);
        if (!u.empty()) patch[n] = u;
      }
    for (int i = 0; i < nnx; ++i)  // nodes whose four elements are all interface elements
      for (int j = 0; j < nny; ++j) {
        int64_t n = node(i, j);
        if (!base[n].empty()) continue;
        std::vector<int32_t> cand;
        for (int di = -1; di <= 0; ++di)
          for (int dj = -1; dj <= 0; ++dj) {
            int ei = i + di, ej = j + dj;
            if (ei < 0 || ej < 0 || ei >= nex || ej >= ney) continue;
            for (int c = 0; c < 4; ++c) {
              int32_t m = (int32_t)node(ei + loc_di[c], ej + loc_dj[c]);
              if (base[m].empty()) continue;
              bool same = (S->node_index[n] == -1) ? (S->node_index[m] == -1)
                                                     : (S->node_index[m] == -2);
              if (same) cand.push_back(m);
            }
          }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        patch[n] = cand;
      }
    S->patch_ptr.assign(nn + 1, 0);
    for (int64_t n = 0; n < nn; ++n) {
      S->patch_ptr[n + 1] = S->patch_ptr[n] + (int32_t)patch[n].size();
      for (int32_t m : patch[n]) S->patch_nodes.push_back(m + 1);
    }
  }

  // ---- descriptor
  pic_mesh_desc &d = S->desc;
  std::memset(&d, 0, sizeof d);
  d.nnx = nnx; d.nny = nny;
  d.xmin = deck->xmin; d.xmax = deck->xmax; d.ymin = deck->ymin; d.ymax = deck->ymax;
  d.delta = deck->delta;
  d.node_type = S->node_type.data();
  d.node_index = S->node_index.data();
  d.element_index = S->element_index.data();
  d.phi_dirichlet = S->phi_dirichlet.data();
  d.cell_volume = S->cell_volume.data();
  d.n_unknowns = n_unknowns;
  d.nnz = (int64_t)S->a_k.size();
  d.a_srow = S->a_srow.data(); d.a_jcol = S->a_jcol.data(); d.a_k = S->a_k.data();
  d.nnz_xt = (int64_t)S->xt_k.size();
  d.xt_srow = S->xt_srow.data(); d.xt_jcol = S->xt_jcol.data(); d.xt_k = S->xt_k.data();
  d.a_diag = S->a_diag.data();
  d.rhs_fix = S->rhs_fix.data();
  d.mass_q1 = S->mass_q1.data();
  d.mass_rows = axi ? S->mass_rows.data() : nullptr;
  d.n_interface = (int32_t)S->ife.size();
  d.ife_mass = S->ife_mass.data();
  d.patch_ptr = S->patch_ptr.data();
  d.patch_nodes = S->patch_nodes.data();
  d.n_objects = (int32_t)S->objects.size();
  d.objects = S->objects.data();
  *out = &S->desc;
  return PIC_OK;
}

int pic_mesh_build(const pic_deck *deck, pic_mesh_desc **out) { return mesh_build(deck, out, false); }

int pic_mesh_build_device(const pic_deck *deck, pic_mesh_desc **out) { return mesh_build(deck, out, true); }

void pic_mesh_free(pic_mesh_desc *mesh) {
  if (!mesh) return;
  // desc is the first member of MeshStore
  delete reinterpret_cast<MeshStore *>(mesh);
}

int pic_mesh_interface_info(const pic_mesh_desc *mesh, int32_t k, int32_t *element,
                            int32_t *type, int32_t *ref_to_local, double *beta, double *d,
                            double *e) {
  if (!mesh) return PIC_ERR_ARG;
  const MeshStore *S = reinterpret_cast<const MeshStore *>(mesh);
  if (k < 1 || k > (int32_t)S->ife.size()) return PIC_ERR_ARG;
  const IfeElem &f = S->ife[k - 1];
  if (element) *element = f.elem + 1;
  if (type) *type = f.type;
  if (ref_to_local)
    for (int r = 0; r < 4; ++r) ref_to_local[r] = f.ref2loc[r] + 1;
  if (beta) { beta[0] = f.beta[0]; beta[1] = f.beta[1]; }
  if (d) { d[0] = f.D[0]; d[1] = f.D[1]; }
  if (e) { e[0] = f.E[0]; e[1] = f.E[1]; }
  return PIC_OK;
}

int pic_mesh_ife_basis(const pic_mesh_desc *mesh, int32_t k, int32_t basis, double x, double y,
                       double *value, double *dx, double *dy) {
  if (!mesh) return PIC_ERR_ARG;
  const MeshStore *S = reinterpret_cast<const MeshStore *>(mesh);
  if (k < 1 || k > (int32_t)S->ife.size() || basis < 0 || basis > 3) return PIC_ERR_ARG;
  const IfeElem &f = S->ife[k - 1];
  int rb = 0;
  for (int r = 0; r < 4; ++r)
    if (f.ref2loc[r] == basis) rb = r;
  // piece of (x, y): side of the cut line DE relative to reference vertex 1
  double sx = f.E[0] - f.D[0], sy = f.E[1] - f.D[1];
  double s_pt = sx * (y - f.D[1]) - sy * (x - f.D[0]);
  double s_v1 = sx * (f.X[0][1] - f.D[1]) - sy * (f.X[0][0] - f.D[0]);
  int piece = (s_pt * s_v1 >= 0) ? 0 : 1;
  pic::ife_eval(f, rb, piece, x, y, value, dx, dy);
  return PIC_OK;
}

}  // extern "C"
