/*
 * ORACLE -- test infrastructure only.  A plain-C restatement of manapy's
 * explicit finite-volume kernels, loop for loop and in the same order, used to
 * check the CUDA path and to time the reference algorithm on host cores.  It is
 * never part of the product path.
 *
 * Conventions follow the reference exactly:
 *   - ragged int tables are manapy's padded layout: row i is tab[i*w .. i*w+w-1]
 *     with the row count in the last column (tab[i*w + w-1]);
 *   - face lists (innerfaces, boundaryfaces, ...) are int32 index arrays;
 *   - 2D/3D vectors are stored [n][3] (ghost centres [n][3] in 2D, [n][4] in 3D).
 * Single-rank meshes: the halo, halo-ghost and periodic loops of the reference
 * iterate over empty tables and are omitted.
 *
 * Compiled without -ffast-math and with -ffp-contract=off, so every operation
 * is one IEEE-754 rounding in source order.
 */
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdint.h>
#include <string.h>

#define ROW(tab, w, i) ((tab) + (int64_t)(i) * (w))
#define CNT(tab, w, i) ((tab)[(int64_t)(i) * (w) + (w) - 1])

static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline double dmax(double a, double b) { return a > b ? a : b; }

/* manapy/ast/ast_utils.py:8-18 */
void or_facetocell(const double *u_face, double *u_c, const int32_t *faceid, int wf, int nc) {
  for (int i = 0; i < nc; i++) u_c[i] = 0.;
  for (int i = 0; i < nc; i++) {
    const int32_t *r = ROW(faceid, wf, i);
    for (int j = 0; j < CNT(faceid, wf, i); j++) u_c[i] += u_face[r[j]];
  }
  for (int i = 0; i < nc; i++) u_c[i] /= CNT(faceid, wf, i);
}

/* manapy/boundary/bc_utils.py:64-68 (dirichlet), :51-56 (neumann), :45-49 (nonslip),
 * :58-62 (neumannNH).  kind: 0 dirichlet, 1 neumann, 2 nonslip, 3 neumannNH */
void or_ghost_value(int kind, const double *value, const double *w_c, double *w_ghost,
                    const int32_t *cellidf, const int32_t *faces, int nfaces, const double *cst,
                    const double *dist) {
  for (int k = 0; k < nfaces; k++) {
    int i = faces[k];
    if (kind == 0) w_ghost[i] = value[i];
    else if (kind == 1) w_ghost[i] = w_c[cellidf[2 * i]];
    else if (kind == 2) w_ghost[i] = -1 * w_c[cellidf[2 * i]];
    else w_ghost[i] = w_c[cellidf[2 * i]] + cst[i] * dist[i];
  }
}

/* manapy/ast/functions2d.py:5-104 */
void or_cell_gradient_2d(const double *w_c, const double *w_ghost, const double *centerc,
                         const int32_t *cellnid, int wcn, const int32_t *ghostnid, int wgn,
                         const double *centergf, int nc, double *w_x, double *w_y, double *w_z) {
  for (int i = 0; i < nc; i++) {
    double i_xx = 0., i_yy = 0., i_xy = 0., j_xw = 0., j_yw = 0.;
    const double cx = centerc[3 * i], cy = centerc[3 * i + 1];
    const int32_t *r = ROW(cellnid, wcn, i);
    for (int j = 0; j < CNT(cellnid, wcn, i); j++) {
      int c = r[j];
      double j_x = centerc[3 * c] - cx, j_y = centerc[3 * c + 1] - cy;
      i_xx += j_x * j_x; i_yy += j_y * j_y; i_xy += (j_x * j_y);
      j_xw += (j_x * (w_c[c] - w_c[i]));
      j_yw += (j_y * (w_c[c] - w_c[i]));
    }
    const int32_t *g = ROW(ghostnid, wgn, i);
    for (int j = 0; j < CNT(ghostnid, wgn, i); j++) {
      int f = g[j];
      double j_x = centergf[3 * f] - cx, j_y = centergf[3 * f + 1] - cy;
      i_xx += j_x * j_x; i_yy += j_y * j_y; i_xy += (j_x * j_y);
      j_xw += (j_x * (w_ghost[f] - w_c[i]));
      j_yw += (j_y * (w_ghost[f] - w_c[i]));
    }
    double dia = i_xx * i_yy - i_xy * i_xy;
    w_x[i] = (i_yy * j_xw - i_xy * j_yw) / dia;
    w_y[i] = (i_xx * j_yw - i_xy * j_xw) / dia;
    w_z[i] = 0.;
  }
}

/* manapy/ast/functions3d.py:4-120 (ghost centres [nf][4]) */
void or_cell_gradient_3d(const double *w_c, const double *w_ghost, const double *centerc,
                         const int32_t *cellnid, int wcn, const int32_t *ghostnid, int wgn,
                         const double *centergf, int nc, double *w_x, double *w_y, double *w_z) {
  for (int i = 0; i < nc; i++) {
    double i_xx = 0., i_yy = 0., i_zz = 0., i_xy = 0., i_xz = 0., i_yz = 0.;
    double j_x = 0., j_y = 0., j_z = 0.;
    const double cx = centerc[3 * i], cy = centerc[3 * i + 1], cz = centerc[3 * i + 2];
    const int32_t *r = ROW(cellnid, wcn, i);
    for (int j = 0; j < CNT(cellnid, wcn, i); j++) {
      int c = r[j];
      double jx = centerc[3 * c] - cx, jy = centerc[3 * c + 1] - cy, jz = centerc[3 * c + 2] - cz;
      i_xx += jx * jx; i_yy += jy * jy; i_zz += jz * jz;
      i_xy += (jx * jy); i_xz += (jx * jz); i_yz += (jy * jz);
      j_x += (jx * (w_c[c] - w_c[i])); j_y += (jy * (w_c[c] - w_c[i])); j_z += (jz * (w_c[c] - w_c[i]));
    }
    const int32_t *g = ROW(ghostnid, wgn, i);
    for (int j = 0; j < CNT(ghostnid, wgn, i); j++) {
      int f = g[j];
      double jx = centergf[4 * f] - cx, jy = centergf[4 * f + 1] - cy, jz = centergf[4 * f + 2] - cz;
      i_xx += jx * jx; i_yy += jy * jy; i_zz += jz * jz;
      i_xy += (jx * jy); i_xz += (jx * jz); i_yz += (jy * jz);
      j_x += (jx * (w_ghost[f] - w_c[i])); j_y += (jy * (w_ghost[f] - w_c[i]));
      j_z += (jz * (w_ghost[f] - w_c[i]));
    }
    double dia = i_xx * i_yy * i_zz + 2. * i_xy * i_xz * i_yz - i_xx * (i_yz * i_yz)
                 - i_yy * (i_xz * i_xz) - i_zz * (i_xy * i_xy);
    w_x[i] = ((i_yy * i_zz - i_yz * i_yz) * j_x + (i_xz * i_yz - i_xy * i_zz) * j_y
              + (i_xy * i_yz - i_xz * i_yy) * j_z) / dia;
    w_y[i] = ((i_xz * i_yz - i_xy * i_zz) * j_x + (i_xx * i_zz - i_xz * i_xz) * j_y
              + (i_xy * i_xz - i_yz * i_xx) * j_z) / dia;
    w_z[i] = ((i_xy * i_yz - i_xz * i_yy) * j_x + (i_xy * i_xz - i_yz * i_xx) * j_y
              + (i_xx * i_yy - i_xy * i_xy) * j_z) / dia;
  }
}

/* manapy/ast/functions2d.py:280-325 (dim 2, eps 1e-8) and
 * manapy/ast/functions3d.py:364-408 (dim 3, eps 1e-10).  Faces whose name
 * selects the halo branch do not occur on a single-rank mesh. */
void or_barthlimiter(int dim, const double *w_c, const double *w_ghost, const double *w_x,
                     const double *w_y, const double *w_z, double *psi, const int32_t *cellid,
                     const int32_t *faceid, int wf, const int32_t *namef, const double *centerc,
                     const double *centerf, int nc) {
  const double eps = dim == 2 ? 1e-8 : 1e-10;
  for (int i = 0; i < nc; i++) psi[i] = 1.;
  for (int i = 0; i < nc; i++) {
    double w_max = w_c[i], w_min = w_c[i];
    const int32_t *r = ROW(faceid, wf, i);
    int n = CNT(faceid, wf, i);
    for (int j = 0; j < n; j++) {
      int f = r[j];
      int nm = namef[f];
      double a = w_c[cellid[2 * f]], b;
      if (nm == 0 || nm > 10) b = w_c[cellid[2 * f + 1]];
      else b = w_ghost[f];
      w_max = dmax(dmax(w_max, a), b);
      w_min = dmin(dmin(w_min, a), b);
    }
    for (int j = 0; j < n; j++) {
      int f = r[j];
      double r1 = centerf[3 * f] - centerc[3 * i];
      double r2 = centerf[3 * f + 1] - centerc[3 * i + 1];
      double delta2;
      if (dim == 2) delta2 = w_x[i] * r1 + w_y[i] * r2;
      else {
        double r3 = centerf[3 * f + 2] - centerc[3 * i + 2];
        delta2 = w_x[i] * r1 + w_y[i] * r2 + w_z[i] * r3;
      }
      double psi_ij = 1.;
      if (fabs(delta2) < eps) psi_ij = 1.;
      else {
        if (delta2 > 0.) psi_ij = dmin(1., (w_max - w_c[i]) / delta2);
        if (delta2 < 0.) psi_ij = dmin(1., (w_min - w_c[i]) / delta2);
      }
      psi[i] = dmin(psi[i], psi_ij);
    }
  }
}

/* manapy/ast/functions2d.py:199-276 and functions3d.py:251-362 */
void or_centertovertex(int dim, const double *w_c, const double *w_ghost, const double *centerc,
                       const int32_t *cellid, int wc, const int32_t *ghostid, int wg,
                       const double *vertexn, const double *centergf, int wgc, const double *R_x,
                       const double *R_y, const double *R_z, const double *lambda_x,
                       const double *lambda_y, const double *lambda_z, const int32_t *number,
                       int nn, double *w_n) {
  for (int i = 0; i < nn; i++) w_n[i] = 0.;
  for (int i = 0; i < nn; i++) {
    const double vx = vertexn[4 * i], vy = vertexn[4 * i + 1], vz = vertexn[4 * i + 2];
    double den;
    if (dim == 2) den = number[i] + lambda_x[i] * R_x[i] + lambda_y[i] * R_y[i];
    else den = number[i] + lambda_x[i] * R_x[i] + lambda_y[i] * R_y[i] + lambda_z[i] * R_z[i];
    const int32_t *r = ROW(cellid, wc, i);
    for (int j = 0; j < CNT(cellid, wc, i); j++) {
      int c = r[j];
      double xd = centerc[3 * c] - vx, yd = centerc[3 * c + 1] - vy;
      double alpha;
      if (dim == 2) alpha = (1. + lambda_x[i] * xd + lambda_y[i] * yd) / den;
      else {
        double zd = centerc[3 * c + 2] - vz;
        alpha = (1. + lambda_x[i] * xd + lambda_y[i] * yd + lambda_z[i] * zd) / den;
      }
      w_n[i] += alpha * w_c[c];
    }
    const int32_t *g = ROW(ghostid, wg, i);
    for (int j = 0; j < CNT(ghostid, wg, i); j++) {
      int f = g[j];
      double xd = centergf[wgc * f] - vx, yd = centergf[wgc * f + 1] - vy;
      double alpha;
      if (dim == 2) alpha = (1. + lambda_x[i] * xd + lambda_y[i] * yd) / den;
      else {
        double zd = centergf[wgc * f + 2] - vz;
        alpha = (1. + lambda_x[i] * xd + lambda_y[i] * yd + lambda_z[i] * zd) / den;
      }
      w_n[i] += alpha * w_ghost[f];
    }
  }
}

static void face_grad_2d_one(int i, int right_is_ghost, const double *w_c, const double *w_ghost,
                             const double *w_node, const int32_t *cellidf, const int32_t *nodeidf,
                             int wnf, const double *airDiamond, const double *f_1,
                             const double *f_2, const double *f_3, const double *f_4,
                             double *wx_face, double *wy_face) {
  double vi1 = w_node[ROW(nodeidf, wnf, i)[0]], vi2 = w_node[ROW(nodeidf, wnf, i)[1]];
  double vv1 = w_c[cellidf[2 * i]];
  double vv2 = right_is_ghost ? w_ghost[i] : w_c[cellidf[2 * i + 1]];
  double a = airDiamond[i];
  wx_face[i] = 1 / (2 * a) * ((vi1 + vv1) * f_1[2 * i + 1] + (vv1 + vi2) * f_2[2 * i + 1]
                              + (vi2 + vv2) * f_3[2 * i + 1] + (vv2 + vi1) * f_4[2 * i + 1]);
  wy_face[i] = -1 / (2 * a) * ((vi1 + vv1) * f_1[2 * i] + (vv1 + vi2) * f_2[2 * i]
                               + (vi2 + vv2) * f_3[2 * i] + (vv2 + vi1) * f_4[2 * i]);
}

/* manapy/ast/functions2d.py:108-196 (f_k stored [nf][2]) */
void or_face_gradient_2d(const double *w_c, const double *w_ghost, const double *w_node,
                         const int32_t *cellidf, const int32_t *nodeidf, int wnf,
                         const double *airDiamond, const double *f_1, const double *f_2,
                         const double *f_3, const double *f_4, double *wx_face, double *wy_face,
                         const int32_t *innerfaces, int ni, const int32_t *dirichletfaces, int nd,
                         const int32_t *neumannfaces, int nn) {
  for (int k = 0; k < ni; k++)
    face_grad_2d_one(innerfaces[k], 0, w_c, w_ghost, w_node, cellidf, nodeidf, wnf, airDiamond, f_1,
                     f_2, f_3, f_4, wx_face, wy_face);
  for (int k = 0; k < nd; k++)
    face_grad_2d_one(dirichletfaces[k], 1, w_c, w_ghost, w_node, cellidf, nodeidf, wnf, airDiamond,
                     f_1, f_2, f_3, f_4, wx_face, wy_face);
  for (int k = 0; k < nn; k++)
    face_grad_2d_one(neumannfaces[k], 1, w_c, w_ghost, w_node, cellidf, nodeidf, wnf, airDiamond,
                     f_1, f_2, f_3, f_4, wx_face, wy_face);
}

static void face_grad_3d_one(int i, int right_is_ghost, const double *w_c, const double *w_ghost,
                             const double *w_node, const int32_t *cellidf, const int32_t *nodeidf,
                             int wnf, const double *airDiamond, const double *normalf,
                             const double *f_1, const double *f_2, double *wx, double *wy,
                             double *wz) {
  const int32_t *nd = ROW(nodeidf, wnf, i);
  int i4 = nd[2];
  if (CNT(nodeidf, wnf, i) == 4) i4 = nd[3];
  double VA = w_node[nd[0]], VB = w_node[nd[1]], VC = w_node[nd[2]], VD = w_node[i4];
  double VL = w_c[cellidf[2 * i]];
  double VR = right_is_ghost ? w_ghost[i] : w_c[cellidf[2 * i + 1]];
  double a = airDiamond[i];
  wx[i] = (f_1[3 * i] * (VA - VC) + f_2[3 * i] * (VB - VD) + normalf[3 * i] * (VR - VL)) / a;
  wy[i] = (f_1[3 * i + 1] * (VA - VC) + f_2[3 * i + 1] * (VB - VD) + normalf[3 * i + 1] * (VR - VL)) / a;
  wz[i] = (f_1[3 * i + 2] * (VA - VC) + f_2[3 * i + 2] * (VB - VD) + normalf[3 * i + 2] * (VR - VL)) / a;
}

/* manapy/ast/functions3d.py:122-248 */
void or_face_gradient_3d(const double *w_c, const double *w_ghost, const double *w_node,
                         const int32_t *cellidf, const int32_t *nodeidf, int wnf,
                         const double *airDiamond, const double *normalf, const double *f_1,
                         const double *f_2, double *wx, double *wy, double *wz,
                         const int32_t *innerfaces, int ni, const int32_t *dirichletfaces, int nd,
                         const int32_t *neumannfaces, int nn) {
  for (int k = 0; k < ni; k++)
    face_grad_3d_one(innerfaces[k], 0, w_c, w_ghost, w_node, cellidf, nodeidf, wnf, airDiamond,
                     normalf, f_1, f_2, wx, wy, wz);
  for (int k = 0; k < nd; k++)
    face_grad_3d_one(dirichletfaces[k], 1, w_c, w_ghost, w_node, cellidf, nodeidf, wnf,
                     airDiamond, normalf, f_1, f_2, wx, wy, wz);
  for (int k = 0; k < nn; k++)
    face_grad_3d_one(neumannfaces[k], 1, w_c, w_ghost, w_node, cellidf, nodeidf, wnf, airDiamond,
                     normalf, f_1, f_2, wx, wy, wz);
}

/* manapy/solvers/advecdiff/fvm_utils.py:43-176 (dim 2) and :180-314 (dim 3),
 * inner faces then boundary faces. */
void or_explicitscheme_convective(int dim, double *rez_w, const double *w_c, const double *w_ghost,
                                  const double *u_face, const double *v_face, const double *w_face,
                                  const double *w_x, const double *w_y, const double *w_z,
                                  const double *psi, const double *centerc, const double *centerf,
                                  const int32_t *cellidf, const double *normalf,
                                  const int32_t *innerfaces, int ni, const int32_t *boundaryfaces,
                                  int nb, int nc, int order) {
  for (int i = 0; i < nc; i++) rez_w[i] = 0.;
  for (int k = 0; k < ni; k++) {
    int i = innerfaces[k];
    int l = cellidf[2 * i], r = cellidf[2 * i + 1];
    double rl0 = centerf[3 * i] - centerc[3 * l], rr0 = centerf[3 * i] - centerc[3 * r];
    double rl1 = centerf[3 * i + 1] - centerc[3 * l + 1], rr1 = centerf[3 * i + 1] - centerc[3 * r + 1];
    double dl, dr;
    if (dim == 2) {
      dl = w_x[l] * rl0 + w_y[l] * rl1;
      dr = w_x[r] * rr0 + w_y[r] * rr1;
    } else {
      double rl2 = centerf[3 * i + 2] - centerc[3 * l + 2], rr2 = centerf[3 * i + 2] - centerc[3 * r + 2];
      dl = w_x[l] * rl0 + w_y[l] * rl1 + w_z[l] * rl2;
      dr = w_x[r] * rr0 + w_y[r] * rr1 + w_z[r] * rr2;
    }
    double w_l = w_c[l] + (order - 1) * psi[l] * dl;
    double w_r = w_c[r] + (order - 1) * psi[r] * dr;
    double sign = u_face[i] * normalf[3 * i] + v_face[i] * normalf[3 * i + 1] + w_face[i] * normalf[3 * i + 2];
    double sol = sign >= 0 ? w_l : w_r;
    double flux = sign * sol;
    rez_w[l] -= flux;
    rez_w[r] += flux;
  }
  for (int k = 0; k < nb; k++) {
    int i = boundaryfaces[k];
    int l = cellidf[2 * i];
    double rl0 = centerf[3 * i] - centerc[3 * l], rl1 = centerf[3 * i + 1] - centerc[3 * l + 1];
    double dl;
    if (dim == 2) dl = w_x[l] * rl0 + w_y[l] * rl1;
    else {
      double rl2 = centerf[3 * i + 2] - centerc[3 * l + 2];
      dl = w_x[l] * rl0 + w_y[l] * rl1 + w_z[l] * rl2;
    }
    double w_l = w_c[l] + (order - 1) * psi[l] * dl;
    double w_r = w_ghost[i];
    double sign = u_face[i] * normalf[3 * i] + v_face[i] * normalf[3 * i + 1] + w_face[i] * normalf[3 * i + 2];
    double sol = sign >= 0 ? w_l : w_r;
    rez_w[l] -= sign * sol;
  }
}

/* manapy/solvers/advecdiff/fvm_utils.py:5-26 */
void or_explicitscheme_dissipative(const double *wx_face, const double *wy_face,
                                   const double *wz_face, const int32_t *cellidf,
                                   const double *normalf, const int32_t *namef, int nf,
                                   double *dissip_w, int nc, double Dxx, double Dyy, double Dzz) {
  for (int i = 0; i < nc; i++) dissip_w[i] = 0.;
  for (int i = 0; i < nf; i++) {
    double q = Dxx * wx_face[i] * normalf[3 * i] + Dyy * wy_face[i] * normalf[3 * i + 1]
               + Dzz * wz_face[i] * normalf[3 * i + 2];
    if (namef[i] == 0) {
      dissip_w[cellidf[2 * i]] += q;
      dissip_w[cellidf[2 * i + 1]] -= q;
    } else {
      dissip_w[cellidf[2 * i]] += q;
    }
  }
}

/* manapy/solvers/advecdiff/fvm_utils.py:317-340 */
double or_time_step(const double *u, const double *v, const double *w, double cfl,
                    const double *normal, const double *volume, const int32_t *faceid, int wf,
                    int nc, double Dxx, double Dyy, double Dzz) {
  double dt = 1e6;
  for (int i = 0; i < nc; i++) {
    double lam = 0.;
    const int32_t *r = ROW(faceid, wf, i);
    for (int j = 0; j < CNT(faceid, wf, i); j++) {
      const double *n = normal + 3 * r[j];
      double lam_convect = fabs(u[i] * n[0] + v[i] * n[1] + w[i] * n[2]);
      lam += lam_convect;
      double mes = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      double lam_diff = Dxx * (mes * mes) + Dyy * (mes * mes) + Dzz * (mes * mes);
      lam += lam_diff / volume[i];
    }
    if (lam != 0) dt = dmin(dt, cfl * volume[i] / lam);
  }
  return dt;
}

/* manapy/solvers/advecdiff/fvm_utils.py:342-346 */
void or_update_new_value(double *ne_c, const double *rez, const double *dissip, const double *src,
                         double dtime, const double *vol, int nc) {
  for (int i = 0; i < nc; i++) ne_c[i] += dtime * ((rez[i] + dissip[i]) / vol[i] + src[i]);
}

/* ------------------------------------------------------------------ shallow water */

/* manapy/solvers/shallowater/fvm_utils.py:3-14 (no coriolis, no wind) */
void or_update_sw(double *h, double *hu, double *hv, double *hc, double *Z, const double *rh,
                  const double *rhu, const double *rhv, const double *rhc, const double *rZ,
                  const double *sh, const double *shu, const double *shv, const double *shc,
                  const double *sZ, const double *dissip_hc, const double *corio_hu,
                  const double *corio_hv, double wind_hu, double wind_hv, double dtime,
                  const double *vol, int nc) {
  for (int i = 0; i < nc; i++) {
    h[i] += dtime * (rh[i] + sh[i]) / vol[i];
    hu[i] += dtime * ((rhu[i] + shu[i]) / vol[i] + corio_hu[i] + wind_hu);
    hv[i] += dtime * ((rhv[i] + shv[i]) / vol[i] + corio_hv[i] + wind_hv);
    hc[i] += dtime * (rhc[i] + shc[i] - dissip_hc[i]) / vol[i];
    Z[i] += dtime * (rZ[i] + sZ[i]) / vol[i];
  }
}

/* manapy/solvers/shallowater/fvm_utils.py:16-42 */
double or_time_step_sw(const double *h, const double *hu, const double *hv, double cfl,
                       const double *normal, const double *mesure, const double *volume,
                       const int32_t *faceid, int wf, int nc, double grav, double Dxx, double Dyy) {
  double dt = 1e6;
  for (int i = 0; i < nc; i++) {
    double velson = sqrt(grav * h[i]);
    double lam = 0.;
    const int32_t *r = ROW(faceid, wf, i);
    for (int j = 0; j < CNT(faceid, wf, i); j++) {
      int f = r[j];
      const double *n = normal + 3 * f;
      double u_n = fabs(hu[i] / h[i] * n[0] + hv[i] / h[i] * n[1]);
      double lam_convect = u_n / mesure[f] + velson;
      lam += lam_convect * mesure[f];
      double mes = sqrt(n[0] * n[0] + n[1] * n[1]);
      double lam_diff = Dxx * (mes * mes) + Dyy * (mes * mes);
      lam += lam_diff / volume[i];
    }
    dt = dmin(dt, cfl * volume[i] / lam);
  }
  return dt;
}

/* manapy/solvers/shallowater/fvm_utils.py:152-342 with As = 0 (so d = 0 and
 * beta = 0); terms multiplied by those zeros are kept so the rounding sequence
 * matches the reference. */
void or_srnh_scheme(double hu_l, double hu_r, double hv_l, double hv_r, double h_l, double h_r,
                    double hc_l, double hc_r, double Z_l, double Z_r, const double *normal,
                    double mesure, double grav, double *flux) {
  const double As = 0., p = 0.4, xi = 1 / (1 - p);
  double ninv0 = -1 * normal[1], ninv1 = normal[0];
  double sl = sqrt(h_l), sr = sqrt(h_r);
  double u_h = (hu_l / h_l * sl + hu_r / h_r * sr) / (sl + sr);
  double v_h = (hv_l / h_l * sl + hv_r / h_r * sr) / (sl + sr);
  double c_h = (hc_l / h_l * sl + hc_r / h_r * sr) / (sl + sr);
  double un_h = u_h * normal[0] + v_h * normal[1];
  un_h = un_h / mesure;
  double vn_h = u_h * ninv0 + v_h * ninv1;
  vn_h = vn_h / mesure;
  double hroe = (h_l + h_r) / 2, uroe = un_h, vroe = vn_h, croe = c_h;
  double uleft = hu_l * normal[0] + hv_l * normal[1];
  uleft = uleft / mesure;
  double vleft = hu_l * ninv0 + hv_l * ninv1;
  vleft = vleft / mesure;
  double uright = hu_r * normal[0] + hv_r * normal[1];
  uright = uright / mesure;
  double vright = hu_r * ninv0 + hv_r * ninv1;
  vright = vright / mesure;
  double w_lrh = (h_l + h_r) / 2, w_lrhu = (uleft + uright) / 2, w_lrhv = (vleft + vright) / 2;
  double w_lrhc = (hc_l + hc_r) / 2, w_lrz = (Z_l + Z_r) / 2;
  double w_dif[5] = {h_r - h_l, uright - uleft, vright - vleft, hc_r - hc_l, Z_r - Z_l};
  double d = As * xi * (3 * (uroe * uroe) + (vroe * vroe));
  double sound = sqrt(grav * hroe);
  double Q = -((uroe * uroe) + 3 * grav * (hroe + d)) / 9;
  double R = uroe * (9 * grav * (2 * hroe - d) - 2 * (uroe * uroe)) / 54;
  double theta = acos(R / (sqrt(-(Q * Q * Q))));
  double sq = 2 * sqrt(-Q);
  double lambda1 = sq * cos(theta / 3) + (2. / 3) * uroe;
  double lambda2 = sq * cos((theta + 2 * M_PI) / 3) + (2. / 3) * uroe;
  double lambda3 = sq * cos((theta + 4 * M_PI) / 3) + (2. / 3) * uroe;
  double lambda4 = uroe, lambda5 = uroe;
  double alpha1 = lambda1 - uroe, alpha2 = lambda2 - uroe, alpha3 = lambda3 - uroe;
  double beta = 2 * As * xi * vroe / hroe;
  double s2 = sound * sound, u2 = uroe * uroe;
  double gamma1 = s2 - u2 + lambda2 * lambda3 - beta * alpha2 * alpha3 * vroe;
  double gamma2 = s2 - u2 + lambda1 * lambda3 - beta * alpha1 * alpha3 * vroe;
  double gamma3 = s2 - u2 + lambda1 * lambda2 - beta * alpha1 * alpha2 * vroe;
  double sigma1 = -alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 + (alpha1 * alpha1);
  double sigma2 = alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 - (alpha2 * alpha2);
  double sigma3 = alpha1 * alpha2 - alpha2 * alpha3 - alpha1 * alpha3 + (alpha3 * alpha3);
  const double epsilon = 1e-10;
  double sign1 = fabs(lambda1) < epsilon ? 0. : lambda1 / fabs(lambda1);
  double sign2 = fabs(lambda2) < epsilon ? 0. : lambda2 / fabs(lambda2);
  double sign3 = fabs(lambda3) < epsilon ? 0. : lambda3 / fabs(lambda3);
  double sign4 = fabs(lambda4) < epsilon ? 0. : lambda4 / fabs(lambda4);
  double sign5 = fabs(lambda5) < epsilon ? 0. : lambda5 / fabs(lambda5);
  double a1 = (alpha1 * alpha1) / s2 - 1, a2 = (alpha2 * alpha2) / s2 - 1, a3 = (alpha3 * alpha3) / s2 - 1;
  double g1 = gamma1 / sigma1, g2 = gamma2 / sigma2, g3 = gamma3 / sigma3;
  double rmat[5][5];
  rmat[0][0] = sign1 * g1 - sign2 * g2 + sign3 * g3 + sign5 * (beta * vroe);
  rmat[1][0] = lambda1 * sign1 * g1 - lambda2 * sign2 * g2 + lambda3 * sign3 * g3 + sign5 * (beta * uroe * vroe);
  rmat[2][0] = vroe * sign1 * g1 - vroe * sign2 * g2 + vroe * sign3 * g3 - vroe * sign5 * (1 - beta * vroe);
  rmat[3][0] = croe * sign1 * g1 - croe * sign2 * g2 + croe * sign3 * g3 - croe * sign4 + croe * sign5 * beta * vroe;
  rmat[4][0] = a1 * sign1 * g1 - a2 * sign2 * g2 + a3 * sign3 * g3 - sign5 * (beta * vroe);
  rmat[0][1] = -sign1 * (alpha2 + alpha3) / sigma1 + sign2 * (alpha1 + alpha3) / sigma2 - sign3 * (alpha1 + alpha2) / sigma3;
  rmat[1][1] = -lambda1 * sign1 * (alpha2 + alpha3) / sigma1 + lambda2 * sign2 * (alpha1 + alpha3) / sigma2
               - lambda3 * sign3 * (alpha1 + alpha2) / sigma3;
  rmat[2][1] = -vroe * sign1 * (alpha2 + alpha3) / sigma1 + vroe * sign2 * (alpha1 + alpha3) / sigma2
               - vroe * sign3 * (alpha1 + alpha2) / sigma3;
  rmat[3][1] = -croe * sign1 * (alpha2 + alpha3) / sigma1 + croe * sign2 * (alpha1 + alpha3) / sigma2
               - croe * sign3 * (alpha1 + alpha2) / sigma3;
  rmat[4][1] = -a1 * sign1 * (alpha2 + alpha3) / sigma1 + a2 * sign2 * (alpha1 + alpha3) / sigma2
               - a3 * sign3 * (alpha1 + alpha2) / sigma3;
  rmat[0][2] = sign1 * beta * alpha2 * alpha3 / sigma1 - sign2 * beta * alpha1 * alpha3 / sigma2
               + sign3 * beta * alpha1 * alpha2 / sigma3 - sign5 * beta;
  rmat[1][2] = lambda1 * sign1 * beta * alpha2 * alpha3 / sigma1 - lambda2 * sign2 * beta * alpha1 * alpha3 / sigma2
               + lambda3 * sign3 * beta * alpha1 * alpha2 / sigma3 - sign5 * beta * uroe;
  rmat[2][2] = vroe * sign1 * beta * alpha2 * alpha3 / sigma1 - vroe * sign2 * beta * alpha1 * alpha3 / sigma2
               + vroe * sign3 * beta * alpha1 * alpha2 / sigma3 + sign5 * (1 - beta * vroe);
  rmat[3][2] = croe * sign1 * beta * alpha2 * alpha3 / sigma1 - croe * sign2 * beta * alpha1 * alpha3 / sigma2
               + croe * sign3 * beta * alpha1 * alpha2 / sigma3 - croe * sign5 * beta;
  rmat[4][2] = a1 * sign1 * beta * alpha2 * alpha3 / sigma1 - a2 * sign2 * beta * alpha1 * alpha3 / sigma2
               + a3 * sign3 * beta * alpha1 * alpha2 / sigma3 + sign5 * beta;
  rmat[0][3] = 0.; rmat[1][3] = 0.; rmat[2][3] = 0.; rmat[3][3] = sign4; rmat[4][3] = 0.;
  rmat[0][4] = sign1 * s2 / sigma1 - sign2 * s2 / sigma2 + sign3 * s2 / sigma3;
  rmat[1][4] = lambda1 * sign1 * s2 / sigma1 - lambda2 * sign2 * s2 / sigma2 + lambda3 * sign3 * s2 / sigma3;
  rmat[2][4] = vroe * sign1 * s2 / sigma1 - vroe * sign2 * s2 / sigma2 + vroe * sign3 * s2 / sigma3;
  rmat[3][4] = croe * sign1 * s2 / sigma1 - croe * sign2 * s2 / sigma2 + croe * sign3 * s2 / sigma3;
  rmat[4][4] = a1 * sign1 * s2 / sigma1 - a2 * sign2 * s2 / sigma2 + a3 * sign3 * s2 / sigma3;
  double nw[5];
  for (int r = 0; r < 5; r++) {
    double s = 0.;
    for (int c = 0; c < 5; c++) s += rmat[r][c] * w_dif[c];
    nw[r] = s;
  }
  w_lrh = w_lrh - nw[0] / 2;
  w_lrhu = w_lrhu - nw[1] / 2;
  w_lrhv = w_lrhv - nw[2] / 2;
  w_lrhc = w_lrhc - nw[3] / 2;
  w_lrz = w_lrz - nw[4] / 2;
  (void)w_lrz;
  double unew = w_lrhu * normal[0] + w_lrhv * -1 * normal[1];
  unew = unew / mesure;
  double vnew = w_lrhu * -1 * ninv0 + w_lrhv * ninv1;
  vnew = vnew / mesure;
  w_lrhu = unew;
  w_lrhv = vnew;
  double q_s = normal[0] * unew + normal[1] * vnew;
  flux[0] = q_s;
  flux[1] = q_s * w_lrhu / w_lrh + 0.5 * grav * w_lrh * w_lrh * normal[0];
  flux[2] = q_s * w_lrhv / w_lrh + 0.5 * grav * w_lrh * w_lrh * normal[1];
  flux[3] = q_s * w_lrhc / w_lrh;
  double w3 = w_lrh * w_lrh * w_lrh;
  flux[4] = As * xi * normal[0] * unew * ((unew * unew) + (vnew * vnew)) / w3
            + As * xi * normal[1] * vnew * ((unew * unew) + (vnew * vnew)) / w3;
}

/* manapy/solvers/shallowater/fvm_utils.py:344-496: inner faces scatter to
 * both cells, boundary faces to the left cell.  Reconstruction of h and hc
 * uses hc's limiter (manapy/solvers/shallowater/system.py:172-174). */
void or_explicitscheme_convective_sw(double *rez_h, double *rez_hu, double *rez_hv, double *rez_hc,
                                     double *rez_Z, const double *h_c, const double *hu_c,
                                     const double *hv_c, const double *hc_c, const double *Z_c,
                                     const double *h_g, const double *hu_g, const double *hv_g,
                                     const double *hc_g, const double *Z_g, const double *h_x,
                                     const double *h_y, const double *hc_x, const double *hc_y,
                                     const double *psi, const double *centerc,
                                     const double *centerf, const int32_t *cellidf,
                                     const double *mesuref, const double *normalf,
                                     const int32_t *innerfaces, int ni,
                                     const int32_t *boundaryfaces, int nb, int nc, double grav,
                                     int order) {
  for (int i = 0; i < nc; i++) { rez_h[i] = 0.; rez_hu[i] = 0.; rez_hv[i] = 0.; rez_hc[i] = 0.; rez_Z[i] = 0.; }
  double flux[5];
  for (int k = 0; k < ni; k++) {
    int i = innerfaces[k];
    int l = cellidf[2 * i], r = cellidf[2 * i + 1];
    double rl0 = centerf[3 * i] - centerc[3 * l], rr0 = centerf[3 * i] - centerc[3 * r];
    double rl1 = centerf[3 * i + 1] - centerc[3 * l + 1], rr1 = centerf[3 * i + 1] - centerc[3 * r + 1];
    double h_l = h_c[l] + (order - 1) * psi[l] * (h_x[l] * rl0 + h_y[l] * rl1);
    double h_r = h_c[r] + (order - 1) * psi[r] * (h_x[r] * rr0 + h_y[r] * rr1);
    double hc_l = hc_c[l] + (order - 1) * psi[l] * (hc_x[l] * rl0 + hc_y[l] * rl1);
    double hc_r = hc_c[r] + (order - 1) * psi[r] * (hc_x[r] * rr0 + hc_y[r] * rr1);
    or_srnh_scheme(hu_c[l], hu_c[r], hv_c[l], hv_c[r], h_l, h_r, hc_l, hc_r, Z_c[l], Z_c[r],
                   normalf + 3 * i, mesuref[i], grav, flux);
    rez_h[l] -= flux[0]; rez_hu[l] -= flux[1]; rez_hv[l] -= flux[2]; rez_hc[l] -= flux[3]; rez_Z[l] -= flux[4];
    rez_h[r] += flux[0]; rez_hu[r] += flux[1]; rez_hv[r] += flux[2]; rez_hc[r] += flux[3]; rez_Z[r] += flux[4];
  }
  for (int k = 0; k < nb; k++) {
    int i = boundaryfaces[k];
    int l = cellidf[2 * i];
    double rl0 = centerf[3 * i] - centerc[3 * l], rl1 = centerf[3 * i + 1] - centerc[3 * l + 1];
    double h_l = h_c[l] + (order - 1) * psi[l] * (h_x[l] * rl0 + h_y[l] * rl1);
    double hc_l = hc_c[l] + (order - 1) * psi[l] * (hc_x[l] * rl0 + hc_y[l] * rl1);
    or_srnh_scheme(hu_c[l], hu_g[i], hv_c[l], hv_g[i], h_l, h_g[i], hc_l, hc_g[i], Z_c[l], Z_g[i],
                   normalf + 3 * i, mesuref[i], grav, flux);
    rez_h[l] -= flux[0]; rez_hu[l] -= flux[1]; rez_hv[l] -= flux[2]; rez_hc[l] -= flux[3]; rez_Z[l] -= flux[4];
  }
}

/* manapy/solvers/shallowater/fvm_utils.py:44-148 (triangles).  nf is the
 * per-cell outward normal table [nc][3][3]. */
void or_term_source_srnh_sw(double *src_h, double *src_hu, double *src_hv, double *src_hc,
                            double *src_Z, const double *h_c, const double *Z_c,
                            const double *h_g, const double *Z_g, const int32_t *nodeidc, int wn,
                            const int32_t *faceidc, int wf, const int32_t *cellidc, int wcf,
                            const double *centerc, const double *nf, const int32_t *namef,
                            const double *vertexn, int nc, double grav) {
  for (int i = 0; i < nc; i++) {
    double G0 = centerc[3 * i], G1 = centerc[3 * i + 1];
    double c_1 = 0., c_2 = 0.;
    double ss[3][3], mata[3], matb[3], zv[3], hi_p[3], zi_p[3];
    double h_1p = 0., z_1p = 0.;
    for (int j = 0; j < 3; j++) {
      int f = ROW(faceidc, wf, i)[j];
      for (int c = 0; c < 3; c++) ss[j][c] = nf[(int64_t)i * 9 + j * 3 + c];
      double h_p1, z_p1;
      h_1p = h_c[i];
      z_1p = Z_c[i];
      if (namef[f] == 0) {
        /* cellfid is compacted (boundary faces skipped), so slot j may hold the
         * -1 padding; Numba wraps a negative index to the last element. */
        int nb = ROW(cellidc, wcf, i)[j];
        if (nb < 0) nb += nc;
        h_p1 = h_c[nb];
        z_p1 = Z_c[nb];
      } else {
        h_p1 = h_g[f];
        z_p1 = Z_g[f];
      }
      zv[j] = z_p1;
      mata[j] = h_p1 * ss[j][0];
      matb[j] = h_p1 * ss[j][1];
      double hm = 0.5 * (h_1p + h_p1);
      c_1 = c_1 + (hm * 0.5 * (h_1p + h_p1)) * ss[j][0];
      c_2 = c_2 + (hm * 0.5 * (h_1p + h_p1)) * ss[j][1];
      hi_p[j] = h_1p;
      zi_p[j] = z_1p;
    }
    double c_3 = 3.0 * h_1p;
    double delta = (mata[1] * matb[2] - mata[2] * matb[1]) - (mata[0] * matb[2] - matb[0] * mata[2])
                   + (mata[0] * matb[1] - matb[0] * mata[1]);
    double deltax = c_3 * (mata[1] * matb[2] - mata[2] * matb[1]) - (c_1 * matb[2] - c_2 * mata[2])
                    + (c_1 * matb[1] - c_2 * mata[1]);
    double deltay = (c_1 * matb[2] - c_2 * mata[2]) - c_3 * (mata[0] * matb[2] - matb[0] * mata[2])
                    + (mata[0] * c_2 - matb[0] * c_1);
    double deltaz = (mata[1] * c_2 - matb[1] * c_1) - (mata[0] * c_2 - matb[0] * c_1)
                    + c_3 * (mata[0] * matb[1] - matb[0] * mata[1]);
    double h_1 = deltax / delta, h_2 = deltay / delta, h_3 = deltaz / delta;
    double z_1 = zi_p[0] + hi_p[0] - h_1;
    double z_2 = zi_p[1] + hi_p[1] - h_2;
    double z_3 = zi_p[2] + hi_p[2] - h_3;
    int nb1 = ROW(nodeidc, wn, i)[1];
    double b0 = vertexn[4 * nb1], b1 = vertexn[4 * nb1 + 1];
    double ns0[3] = {(G1 - b1), -(G0 - b0), 0.};
    double ns1[3], ns2[3];
    for (int c = 0; c < 3; c++) { ns1[c] = ns0[c] - ss[1][c]; ns2[c] = ns0[c] + ss[0][c]; }
    double s_1[2], s_2[2], s_3[2];
    for (int c = 0; c < 2; c++) {
      s_1[c] = 0.5 * h_1 * (zv[0] * ss[0][c] + z_2 * ns0[c] + z_3 * (-1) * ns2[c]);
      s_2[c] = 0.5 * h_2 * (zv[1] * ss[1][c] + z_1 * (-1) * ns0[c] + z_3 * ns1[c]);
      s_3[c] = 0.5 * h_3 * (zv[2] * ss[2][c] + z_1 * ns2[c] + z_2 * (-1) * ns1[c]);
    }
    src_h[i] = 0;
    src_hu[i] = -grav * (s_1[0] + s_2[0] + s_3[0]);
    src_hv[i] = -grav * (s_1[1] + s_2[1] + s_3[1]);
    src_hc[i] = 0.;
    src_Z[i] = 0.;
  }
}

/* ---- Euler, 2D, first-order Rusanov (manapy/solvers/euler/fvm_utils2d.py) ---- */

static double pymax3(double a, double b, double c) {
  /* Python's max(a, b, c): the first of the largest */
  double m = a;
  if (b > m) m = b;
  if (c > m) m = c;
  return m;
}

/* fvm_utils2d.py:1248-1292 compute_flux_euler_2d_rusanov (qr reads rhovl, as manapy does) */
static void euler_rusanov(double rhol, double Pl, double rhoul, double rhovl, double rhoEl, double rhor, double Pr,
                          double rhour, double rhovr, double rhoEr, const double *normal, double mesure,
                          double gamma, double *F) {
  double ql = (rhoul * normal[0] + rhovl * normal[1]);
  double qr = (rhour * normal[0] + rhovl * normal[1]);
  double cl = sqrt(gamma * Pl / rhol);
  double cr = sqrt(gamma * Pr / rhor);
  double fl_rho = (rhoul * normal[0] + rhovl * normal[1]);
  double fl_rhou = ((rhoul * rhoul / rhol + Pl) * normal[0] + (rhoul * rhovl / rhol) * normal[1]);
  double fl_rhov = ((rhovl * rhoul / rhol) * normal[0] + (rhovl * rhovl / rhol + Pl) * normal[1]);
  double fl_rhoE = (rhoul / rhol * (rhoEl + Pl) * normal[0] + rhovl / rhol * (rhoEl + Pl) * normal[1]);
  double fr_rho = (rhour * normal[0] + rhovr * normal[1]);
  double fr_rhou = ((rhour * rhour / rhor + Pr) * normal[0] + (rhour * rhovr / rhor) * normal[1]);
  double fr_rhov = ((rhovr * rhour / rhor) * normal[0] + (rhovr * rhovr / rhor + Pr) * normal[1]);
  double fr_rhoE = (rhour / rhor * (rhoEr + Pr) * normal[0] + rhovr / rhor * (rhoEr + Pr) * normal[1]);
  double Ll = pymax3(fabs((ql) / rhol - cl), fabs((ql) / rhol), fabs((ql) / rhol + cl));
  double Lr = pymax3(fabs((qr) / rhor - cr), fabs((qr) / rhor), fabs((qr) / rhor + cr));
  double S = Ll > Lr ? Ll : Lr;
  F[0] = (0.5 * (fl_rho + fr_rho) - 0.5 * S * (rhor - rhol)) * mesure;
  F[1] = (0.5 * (fl_rhou + fr_rhou) - 0.5 * S * (rhour - rhoul)) * mesure;
  F[2] = (0.5 * (fl_rhov + fr_rhov) - 0.5 * S * (rhovr - rhovl)) * mesure;
  F[3] = (0.5 * (fl_rhoE + fr_rhoE) - 0.5 * S * (rhoEr - rhoEl)) * mesure;
}

/* fvm_utils2d.py:1490-1611 explicitscheme_euler_2d_rusanov, face loop in face-id order
 * (single rank: every face not named 0 reads the ghost arrays).
 * q, g: rho, P, rhou, rhov, rhoE (cells / faces); rez: rho, rhou, rhov, rhoE */
void or_euler_rusanov_2d(double *const rez[4], const double *const q[5], const double *const g[5],
                         const int32_t *cellidf, const double *normalf, const double *mesuref,
                         const int32_t *namef, int nf, int nc, double gamma) {
  for (int c = 0; c < 4; c++)
    for (int i = 0; i < nc; i++) rez[c][i] = 0.;
  for (int i = 0; i < nf; i++) {
    double norm[2] = {normalf[3 * i] / mesuref[i], normalf[3 * i + 1] / mesuref[i]};
    double mesu = mesuref[i];
    int l = cellidf[2 * i], r = cellidf[2 * i + 1];
    double F[4];
    if (namef[i] == 0) {
      euler_rusanov(q[0][l], q[1][l], q[2][l], q[3][l], q[4][l], q[0][r], q[1][r], q[2][r], q[3][r], q[4][r], norm,
                    mesu, gamma, F);
      for (int c = 0; c < 4; c++) {
        rez[c][l] -= F[c];
        rez[c][r] += F[c];
      }
    } else {
      euler_rusanov(q[0][l], q[1][l], q[2][l], q[3][l], q[4][l], g[0][i], g[1][i], g[2][i], g[3][i], g[4][i], norm,
                    mesu, gamma, F);
      for (int c = 0; c < 4; c++) rez[c][l] -= F[c];
    }
  }
}

/* fvm_utils2d.py:1083-1102 time_step_euler_2d (faces in the cell's own order) */
void or_time_step_euler_2d(const double *rho, const double *P, const double *rhou, const double *rhov, double cfl,
                           const double *normalf, const double *mesuref, const double *volume,
                           const int32_t *faceid, int wf, int nc, double gamma, double *dt_c) {
  for (int i = 0; i < nc; i++) {
    double lam = 0.;
    double velson = sqrt(gamma * fabs(P[i] / rho[i]));
    for (int j = 0; j < 3; j++) {
      int f = ROW(faceid, wf, i)[j];
      double n0 = normalf[3 * f], n1 = normalf[3 * f + 1];
      double u_n = fabs((rhou[i] * n0 + rhov[i] * n1) / rho[i]) / sqrt(n0 * n0 + n1 * n1);
      double lam_convect = u_n + velson;
      lam += lam_convect * mesuref[f];
    }
    dt_c[i] = cfl * volume[i] / lam;
  }
}

/* fvm_utils2d.py:1687-1696 update_euler_2d_fvc; q = rho, P, rhou, rhov, rhoE */
void or_update_euler_2d(double *const q[5], const double *const rez[4], double gamma, double dtime,
                        const double *vol, int nc) {
  for (int i = 0; i < nc; i++) {
    q[0][i] += dtime * ((rez[0][i]) / vol[i]);
    q[2][i] += dtime * ((rez[1][i]) / vol[i]);
    q[3][i] += dtime * ((rez[2][i]) / vol[i]);
    q[4][i] += dtime * ((rez[3][i]) / vol[i]);
  }
  for (int i = 0; i < nc; i++)
    q[1][i] = (gamma - 1) * (q[4][i] - 0.5 * (q[2][i] * q[2][i] + q[3][i] * q[3][i]) / q[0][i]);
}
