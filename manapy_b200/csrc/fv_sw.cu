// Shallow-water kernels: manapy's SRNH scheme on triangles, FP64.
//
// Reference loops (manapy source tree):
//   srnh_scheme                   manapy/solvers/shallowater/fvm_utils.py:152-342
//   explicitscheme_convective_SW  manapy/solvers/shallowater/fvm_utils.py:344-496
//   term_source_srnh_SW           manapy/solvers/shallowater/fvm_utils.py:44-148
//   time_step_SW                  manapy/solvers/shallowater/fvm_utils.py:16-42
//   update_SW                     manapy/solvers/shallowater/fvm_utils.py:3-14
//
// The face flux costs two transcendentals, four square roots and ~30 divisions,
// so each face flux is computed once (face kernel, one thread per face) and the
// five residuals are gathered per cell in manapy's order (inner faces by
// ascending id, then boundary faces by ascending id).
#include "fv_common.cuh"
#include "fv_compact.cuh"

namespace mb {

// SRNH flux with As = 0 (so d = 0 and beta = 0).  Terms multiplied by those
// zeros are kept, as in manapy, so that NaN/Inf propagate the same way.
__device__ __forceinline__ void srnh(double hu_l, double hu_r, double hv_l, double hv_r, double h_l, double h_r,
                                     double hc_l, double hc_r, double Z_l, double Z_r, double n0, double n1,
                                     double mesure, double grav, double flux[5]) {
  const double As = 0., p = 0.4, xi = 1 / (1 - p);
  const double ninv0 = -1 * n1, ninv1 = n0;
  const double sl = sqrt(h_l), sr = sqrt(h_r);
  const double u_h = (hu_l / h_l * sl + hu_r / h_r * sr) / (sl + sr);
  const double v_h = (hv_l / h_l * sl + hv_r / h_r * sr) / (sl + sr);
  const double c_h = (hc_l / h_l * sl + hc_r / h_r * sr) / (sl + sr);
  const double un_h = (u_h * n0 + v_h * n1) / mesure;
  const double vn_h = (u_h * ninv0 + v_h * ninv1) / mesure;
  const double hroe = (h_l + h_r) / 2, uroe = un_h, vroe = vn_h, croe = c_h;
  const double uleft = (hu_l * n0 + hv_l * n1) / mesure;
  const double vleft = (hu_l * ninv0 + hv_l * ninv1) / mesure;
  const double uright = (hu_r * n0 + hv_r * n1) / mesure;
  const double vright = (hu_r * ninv0 + hv_r * ninv1) / mesure;
  double w_lrh = (h_l + h_r) / 2, w_lrhu = (uleft + uright) / 2, w_lrhv = (vleft + vright) / 2;
  double w_lrhc = (hc_l + hc_r) / 2;
  const double wd0 = h_r - h_l, wd1 = uright - uleft, wd2 = vright - vleft, wd3 = hc_r - hc_l, wd4 = Z_r - Z_l;
  const double u2 = uroe * uroe;
  const double d = As * xi * (3 * u2 + (vroe * vroe));
  const double sound = sqrt(grav * hroe);
  const double Q = -(u2 + 3 * grav * (hroe + d)) / 9;
  const double R = uroe * (9 * grav * (2 * hroe - d) - 2 * u2) / 54;
  const double theta = acos(R / (sqrt(-(Q * Q * Q))));
  const double sq = 2 * sqrt(-Q);
  const double lambda1 = sq * cos(theta / 3) + (2. / 3) * uroe;
  const double lambda2 = sq * cos((theta + 2 * 3.141592653589793) / 3) + (2. / 3) * uroe;
  const double lambda3 = sq * cos((theta + 4 * 3.141592653589793) / 3) + (2. / 3) * uroe;
  const double lambda4 = uroe, lambda5 = uroe;
  const double alpha1 = lambda1 - uroe, alpha2 = lambda2 - uroe, alpha3 = lambda3 - uroe;
  const double beta = 2 * As * xi * vroe / hroe;
  const double s2 = sound * sound;
  const double gamma1 = s2 - u2 + lambda2 * lambda3 - beta * alpha2 * alpha3 * vroe;
  const double gamma2 = s2 - u2 + lambda1 * lambda3 - beta * alpha1 * alpha3 * vroe;
  const double gamma3 = s2 - u2 + lambda1 * lambda2 - beta * alpha1 * alpha2 * vroe;
  const double sigma1 = -alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 + (alpha1 * alpha1);
  const double sigma2 = alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 - (alpha2 * alpha2);
  const double sigma3 = alpha1 * alpha2 - alpha2 * alpha3 - alpha1 * alpha3 + (alpha3 * alpha3);
  const double eps = 1e-10;
  const double sign1 = fabs(lambda1) < eps ? 0. : lambda1 / fabs(lambda1);
  const double sign2 = fabs(lambda2) < eps ? 0. : lambda2 / fabs(lambda2);
  const double sign3 = fabs(lambda3) < eps ? 0. : lambda3 / fabs(lambda3);
  const double sign4 = fabs(lambda4) < eps ? 0. : lambda4 / fabs(lambda4);
  const double sign5 = fabs(lambda5) < eps ? 0. : lambda5 / fabs(lambda5);
  const double a1 = (alpha1 * alpha1) / s2 - 1, a2 = (alpha2 * alpha2) / s2 - 1, a3 = (alpha3 * alpha3) / s2 - 1;
  const double g1 = gamma1 / sigma1, g2 = gamma2 / sigma2, g3 = gamma3 / sigma3;
  // column 1
  const double r00 = sign1 * g1 - sign2 * g2 + sign3 * g3 + sign5 * (beta * vroe);
  const double r10 = lambda1 * sign1 * g1 - lambda2 * sign2 * g2 + lambda3 * sign3 * g3 + sign5 * (beta * uroe * vroe);
  const double r20 = vroe * sign1 * g1 - vroe * sign2 * g2 + vroe * sign3 * g3 - vroe * sign5 * (1 - beta * vroe);
  const double r30 = croe * sign1 * g1 - croe * sign2 * g2 + croe * sign3 * g3 - croe * sign4 + croe * sign5 * beta * vroe;
  const double r40 = a1 * sign1 * g1 - a2 * sign2 * g2 + a3 * sign3 * g3 - sign5 * (beta * vroe);
  // column 2
  const double t1 = (alpha2 + alpha3), t2 = (alpha1 + alpha3), t3 = (alpha1 + alpha2);
  const double r01 = -sign1 * t1 / sigma1 + sign2 * t2 / sigma2 - sign3 * t3 / sigma3;
  const double r11 = -lambda1 * sign1 * t1 / sigma1 + lambda2 * sign2 * t2 / sigma2 - lambda3 * sign3 * t3 / sigma3;
  const double r21 = -vroe * sign1 * t1 / sigma1 + vroe * sign2 * t2 / sigma2 - vroe * sign3 * t3 / sigma3;
  const double r31 = -croe * sign1 * t1 / sigma1 + croe * sign2 * t2 / sigma2 - croe * sign3 * t3 / sigma3;
  const double r41 = -a1 * sign1 * t1 / sigma1 + a2 * sign2 * t2 / sigma2 - a3 * sign3 * t3 / sigma3;
  // column 3
  const double r02 = sign1 * beta * alpha2 * alpha3 / sigma1 - sign2 * beta * alpha1 * alpha3 / sigma2 +
                     sign3 * beta * alpha1 * alpha2 / sigma3 - sign5 * beta;
  const double r12 = lambda1 * sign1 * beta * alpha2 * alpha3 / sigma1 - lambda2 * sign2 * beta * alpha1 * alpha3 / sigma2 +
                     lambda3 * sign3 * beta * alpha1 * alpha2 / sigma3 - sign5 * beta * uroe;
  const double r22 = vroe * sign1 * beta * alpha2 * alpha3 / sigma1 - vroe * sign2 * beta * alpha1 * alpha3 / sigma2 +
                     vroe * sign3 * beta * alpha1 * alpha2 / sigma3 + sign5 * (1 - beta * vroe);
  const double r32 = croe * sign1 * beta * alpha2 * alpha3 / sigma1 - croe * sign2 * beta * alpha1 * alpha3 / sigma2 +
                     croe * sign3 * beta * alpha1 * alpha2 / sigma3 - croe * sign5 * beta;
  const double r42 = a1 * sign1 * beta * alpha2 * alpha3 / sigma1 - a2 * sign2 * beta * alpha1 * alpha3 / sigma2 +
                     a3 * sign3 * beta * alpha1 * alpha2 / sigma3 + sign5 * beta;
  // column 4: only rmat[3][3] = sign4 is non-zero
  // column 5
  const double r04 = sign1 * s2 / sigma1 - sign2 * s2 / sigma2 + sign3 * s2 / sigma3;
  const double r14 = lambda1 * sign1 * s2 / sigma1 - lambda2 * sign2 * s2 / sigma2 + lambda3 * sign3 * s2 / sigma3;
  const double r24 = vroe * sign1 * s2 / sigma1 - vroe * sign2 * s2 / sigma2 + vroe * sign3 * s2 / sigma3;
  const double r34 = croe * sign1 * s2 / sigma1 - croe * sign2 * s2 / sigma2 + croe * sign3 * s2 / sigma3;
  const double r44 = a1 * sign1 * s2 / sigma1 - a2 * sign2 * s2 / sigma2 + a3 * sign3 * s2 / sigma3;
  // rows . w_dif, summed left to right from 0 as manapy's sum() does
  const double hnew = 0. + r00 * wd0 + r01 * wd1 + r02 * wd2 + 0. * wd3 + r04 * wd4;
  const double unew0 = 0. + r10 * wd0 + r11 * wd1 + r12 * wd2 + 0. * wd3 + r14 * wd4;
  const double vnew0 = 0. + r20 * wd0 + r21 * wd1 + r22 * wd2 + 0. * wd3 + r24 * wd4;
  const double cnew = 0. + r30 * wd0 + r31 * wd1 + r32 * wd2 + sign4 * wd3 + r34 * wd4;
  (void)r40; (void)r41; (void)r42; (void)r44;
  w_lrh = w_lrh - hnew / 2;
  w_lrhu = w_lrhu - unew0 / 2;
  w_lrhv = w_lrhv - vnew0 / 2;
  w_lrhc = w_lrhc - cnew / 2;
  double unew = (w_lrhu * n0 + w_lrhv * -1 * n1) / mesure;
  double vnew = (w_lrhu * -1 * ninv0 + w_lrhv * ninv1) / mesure;
  const double q_s = n0 * unew + n1 * vnew;
  flux[0] = q_s;
  flux[1] = q_s * unew / w_lrh + 0.5 * grav * w_lrh * w_lrh * n0;
  flux[2] = q_s * vnew / w_lrh + 0.5 * grav * w_lrh * w_lrh * n1;
  flux[3] = q_s * w_lrhc / w_lrh;
  const double w3 = w_lrh * w_lrh * w_lrh;
  const double uv = (unew * unew) + (vnew * vnew);
  flux[4] = As * xi * n0 * unew * uv / w3 + As * xi * n1 * vnew * uv / w3;
}

// SRNH flux specialised to manapy's constant As = 0 (d = 0, beta = 0): every
// term multiplied by those zeros is dropped and flux[4] is identically zero.
// For finite inputs this changes no rounding: dropped terms are signed zeros
// added to sums, and sign_k * x / sigma equals sign_k * (x / sigma) exactly
// because sign_k is +-1 or 0.  FAST additionally takes the eigenvalues of
// manapy's cubic in closed form ({0, u+c, u-c}, ordered as the trigonometric
// formula orders them) and replaces divisions by a shared denominator with
// one reciprocal: results then differ from manapy by rounding only.
template <bool FAST>
__device__ __forceinline__ void srnh0(double hu_l, double hu_r, double hv_l, double hv_r, double h_l, double h_r,
                                      double hc_l, double hc_r, double Z_l, double Z_r, double n0, double n1,
                                      double mesure, double grav, double flux[4]) {
  const double ninv0 = -1 * n1, ninv1 = n0;
  const double sl = sqrt(h_l), sr = sqrt(h_r);
  double u_h, v_h, c_h, un_h, vn_h, uleft, vleft, uright, vright;
  if (FAST) {
    const double il = 1 / h_l, ir = 1 / h_r, is = 1 / (sl + sr), im = 1 / mesure;
    u_h = (hu_l * il * sl + hu_r * ir * sr) * is;
    v_h = (hv_l * il * sl + hv_r * ir * sr) * is;
    c_h = (hc_l * il * sl + hc_r * ir * sr) * is;
    un_h = (u_h * n0 + v_h * n1) * im;
    vn_h = (u_h * ninv0 + v_h * ninv1) * im;
    uleft = (hu_l * n0 + hv_l * n1) * im;
    vleft = (hu_l * ninv0 + hv_l * ninv1) * im;
    uright = (hu_r * n0 + hv_r * n1) * im;
    vright = (hu_r * ninv0 + hv_r * ninv1) * im;
  } else {
    u_h = (hu_l / h_l * sl + hu_r / h_r * sr) / (sl + sr);
    v_h = (hv_l / h_l * sl + hv_r / h_r * sr) / (sl + sr);
    c_h = (hc_l / h_l * sl + hc_r / h_r * sr) / (sl + sr);
    un_h = (u_h * n0 + v_h * n1) / mesure;
    vn_h = (u_h * ninv0 + v_h * ninv1) / mesure;
    uleft = (hu_l * n0 + hv_l * n1) / mesure;
    vleft = (hu_l * ninv0 + hv_l * ninv1) / mesure;
    uright = (hu_r * n0 + hv_r * n1) / mesure;
    vright = (hu_r * ninv0 + hv_r * ninv1) / mesure;
  }
  const double hroe = (h_l + h_r) / 2, uroe = un_h, vroe = vn_h, croe = c_h;
  double w_lrh = (h_l + h_r) / 2, w_lrhu = (uleft + uright) / 2, w_lrhv = (vleft + vright) / 2;
  double w_lrhc = (hc_l + hc_r) / 2;
  const double wd0 = h_r - h_l, wd1 = uright - uleft, wd2 = vright - vleft, wd3 = hc_r - hc_l, wd4 = Z_r - Z_l;
  const double u2 = uroe * uroe;
  const double sound = sqrt(grav * hroe);
  double lambda1, lambda2, lambda3;
  if (FAST) {
    // roots of lambda (lambda^2 - 2 u lambda + u^2 - c^2): 0, u + c, u - c; the
    // trigonometric formula returns the largest, the smallest, then the middle one
    const double a = uroe + sound, b = uroe - sound;  // a > b
    const double hi = fmax(a, 0.0), lo = fmin(b, 0.0);
    lambda1 = hi;
    lambda2 = lo;
    lambda3 = (a < 0.0) ? a : ((b > 0.0) ? b : 0.0);
  } else {
    const double Q = -(u2 + 3 * grav * hroe) / 9;
    const double R = uroe * (9 * grav * (2 * hroe) - 2 * u2) / 54;
    const double theta = acos(R / (sqrt(-(Q * Q * Q))));
    const double sq = 2 * sqrt(-Q);
    lambda1 = sq * cos(theta / 3) + (2. / 3) * uroe;
    lambda2 = sq * cos((theta + 2 * 3.141592653589793) / 3) + (2. / 3) * uroe;
    lambda3 = sq * cos((theta + 4 * 3.141592653589793) / 3) + (2. / 3) * uroe;
  }
  const double alpha1 = lambda1 - uroe, alpha2 = lambda2 - uroe, alpha3 = lambda3 - uroe;
  const double s2 = sound * sound;
  const double gamma1 = s2 - u2 + lambda2 * lambda3;
  const double gamma2 = s2 - u2 + lambda1 * lambda3;
  const double gamma3 = s2 - u2 + lambda1 * lambda2;
  const double sigma1 = -alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 + (alpha1 * alpha1);
  const double sigma2 = alpha1 * alpha2 + alpha2 * alpha3 - alpha1 * alpha3 - (alpha2 * alpha2);
  const double sigma3 = alpha1 * alpha2 - alpha2 * alpha3 - alpha1 * alpha3 + (alpha3 * alpha3);
  const double eps = 1e-10;
  // lambda / |lambda| is exactly +-1
  const double sign1 = fabs(lambda1) < eps ? 0. : copysign(1.0, lambda1);
  const double sign2 = fabs(lambda2) < eps ? 0. : copysign(1.0, lambda2);
  const double sign3 = fabs(lambda3) < eps ? 0. : copysign(1.0, lambda3);
  const double sign4 = fabs(uroe) < eps ? 0. : copysign(1.0, uroe);
  const double sign5 = sign4;
  const double t1 = (alpha2 + alpha3), t2 = (alpha1 + alpha3), t3 = (alpha1 + alpha2);
  // |lambda_k| sign_k = lambda_k sign_k exactly
  const double l1 = lambda1 * sign1, l2 = lambda2 * sign2, l3 = lambda3 * sign3;
  double g1, g2, g3, q1, q2, q3, lq1, lq2, lq3, vq1, vq2, vq3, cq1, cq2, cq3;
  double e1, e2, e3, le1, le2, le3, ve1, ve2, ve3, ce1, ce2, ce3;
  if (FAST) {
    const double i1 = 1 / sigma1, i2 = 1 / sigma2, i3 = 1 / sigma3;
    g1 = gamma1 * i1; g2 = gamma2 * i2; g3 = gamma3 * i3;
    q1 = t1 * i1; q2 = t2 * i2; q3 = t3 * i3;
    lq1 = l1 * q1; lq2 = l2 * q2; lq3 = l3 * q3;
    vq1 = vroe * q1; vq2 = vroe * q2; vq3 = vroe * q3;
    cq1 = croe * q1; cq2 = croe * q2; cq3 = croe * q3;
    e1 = s2 * i1; e2 = s2 * i2; e3 = s2 * i3;
    le1 = l1 * e1; le2 = l2 * e2; le3 = l3 * e3;
    ve1 = vroe * e1; ve2 = vroe * e2; ve3 = vroe * e3;
    ce1 = croe * e1; ce2 = croe * e2; ce3 = croe * e3;
  } else {
    g1 = gamma1 / sigma1; g2 = gamma2 / sigma2; g3 = gamma3 / sigma3;
    q1 = t1 / sigma1; q2 = t2 / sigma2; q3 = t3 / sigma3;
    lq1 = (l1 * t1) / sigma1; lq2 = (l2 * t2) / sigma2; lq3 = (l3 * t3) / sigma3;
    vq1 = (vroe * t1) / sigma1; vq2 = (vroe * t2) / sigma2; vq3 = (vroe * t3) / sigma3;
    cq1 = (croe * t1) / sigma1; cq2 = (croe * t2) / sigma2; cq3 = (croe * t3) / sigma3;
    e1 = s2 / sigma1; e2 = s2 / sigma2; e3 = s2 / sigma3;
    le1 = (l1 * s2) / sigma1; le2 = (l2 * s2) / sigma2; le3 = (l3 * s2) / sigma3;
    ve1 = (vroe * s2) / sigma1; ve2 = (vroe * s2) / sigma2; ve3 = (vroe * s2) / sigma3;
    ce1 = (croe * s2) / sigma1; ce2 = (croe * s2) / sigma2; ce3 = (croe * s2) / sigma3;
  }
  // rows 0-3 of manapy's rmat (row 4 only feeds the bed flux, identically zero)
  const double r00 = sign1 * g1 - sign2 * g2 + sign3 * g3;
  const double r10 = l1 * g1 - l2 * g2 + l3 * g3;
  const double r20 = vroe * sign1 * g1 - vroe * sign2 * g2 + vroe * sign3 * g3 - vroe * sign5;
  const double r30 = croe * sign1 * g1 - croe * sign2 * g2 + croe * sign3 * g3 - croe * sign4;
  const double r01 = -sign1 * q1 + sign2 * q2 - sign3 * q3;
  const double r11 = -sign1 * lq1 * sign1 + sign2 * lq2 * sign2 - sign3 * lq3 * sign3;
  const double r21 = -sign1 * vq1 + sign2 * vq2 - sign3 * vq3;
  const double r31 = -sign1 * cq1 + sign2 * cq2 - sign3 * cq3;
  const double r04 = sign1 * e1 - sign2 * e2 + sign3 * e3;
  const double r14 = le1 - le2 + le3;
  const double r24 = sign1 * ve1 - sign2 * ve2 + sign3 * ve3;
  const double r34 = sign1 * ce1 - sign2 * ce2 + sign3 * ce3;
  const double hnew = r00 * wd0 + r01 * wd1 + r04 * wd4;
  const double unew0 = r10 * wd0 + r11 * wd1 + r14 * wd4;
  const double vnew0 = r20 * wd0 + r21 * wd1 + sign5 * wd2 + r24 * wd4;
  const double cnew = r30 * wd0 + r31 * wd1 + sign4 * wd3 + r34 * wd4;
  w_lrh = w_lrh - hnew / 2;
  w_lrhu = w_lrhu - unew0 / 2;
  w_lrhv = w_lrhv - vnew0 / 2;
  w_lrhc = w_lrhc - cnew / 2;
  double unew, vnew;
  if (FAST) {
    const double im = 1 / mesure;
    unew = (w_lrhu * n0 + w_lrhv * -1 * n1) * im;
    vnew = (w_lrhu * -1 * ninv0 + w_lrhv * ninv1) * im;
  } else {
    unew = (w_lrhu * n0 + w_lrhv * -1 * n1) / mesure;
    vnew = (w_lrhu * -1 * ninv0 + w_lrhv * ninv1) / mesure;
  }
  const double q_s = n0 * unew + n1 * vnew;
  const double gh = 0.5 * grav * w_lrh * w_lrh;
  flux[0] = q_s;
  if (FAST) {
    const double iw = 1 / w_lrh;
    flux[1] = q_s * unew * iw + gh * n0;
    flux[2] = q_s * vnew * iw + gh * n1;
    flux[3] = q_s * w_lrhc * iw;
  } else {
    flux[1] = q_s * unew / w_lrh + gh * n0;
    flux[2] = q_s * vnew / w_lrh + gh * n1;
    flux[3] = q_s * w_lrhc / w_lrh;
  }
}

struct SWState {
  const double *q[5];  // h, hu, hv, hc, Z (cells)
  const double *g[5];  // ghosts (faces); null -> neumann copy of the interior cell
  const double *gr[4]; // h_x, h_y, hc_x, hc_y (order 2)
  const double *psi;   // hc's limiter (order 2)
  int walls;           // boundary faces of the fused step: MB_WALLS_NEUMANN or MB_WALLS_REFLECT
};

// Momentum of a reflective-wall ghost: the interior momentum with its normal
// component reversed, q - 2 (q.n) n / |n|^2 (no counterpart in manapy).
__device__ __forceinline__ void wall_mirror(double hu, double hv, double n0, double n1, double &gu, double &gv) {
  const double k = 2 * (hu * n0 + hv * n1) / (n0 * n0 + n1 * n1);
  gu = hu - k * n0;
  gv = hv - k * n1;
}

__device__ __forceinline__ double sw_ghost(const SWState &s, int k, int f, int c0) {
  return s.g[k] ? ld(s.g[k] + f) : ld(s.q[k] + c0);
}

template <bool ORDER2>
__global__ void __launch_bounds__(kBlock) k_sw_face_flux(mb_mesh m, SWState s, double grav, double *ff) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nbfaces; f += gridDim.x * blockDim.x) {
    const int l = ld(m.face_cellid + 2 * f), r = ld(m.face_cellid + 2 * f + 1);
    const double *N = m.face_normal + 3 * f;
    const double n0 = ld(N), n1 = ld(N + 1), mes = ld(m.face_mesure + f);
    double h_l = ld(s.q[0] + l), hc_l = ld(s.q[3] + l);
    double h_r, hu_r, hv_r, hc_r, Z_r;
    const double *fc = m.face_center + 3 * f, *cc = m.cell_center;
    if (ORDER2) {
      const double rl0 = ld(fc) - ld(cc + 3 * l), rl1 = ld(fc + 1) - ld(cc + 3 * l + 1);
      const double pl = ld(s.psi + l);
      h_l = h_l + pl * (ld(s.gr[0] + l) * rl0 + ld(s.gr[1] + l) * rl1);
      hc_l = hc_l + pl * (ld(s.gr[2] + l) * rl0 + ld(s.gr[3] + l) * rl1);
    }
    if (r >= 0) {
      h_r = ld(s.q[0] + r); hu_r = ld(s.q[1] + r); hv_r = ld(s.q[2] + r); hc_r = ld(s.q[3] + r);
      Z_r = ld(s.q[4] + r);
      if (ORDER2) {
        const double rr0 = ld(fc) - ld(cc + 3 * r), rr1 = ld(fc + 1) - ld(cc + 3 * r + 1);
        const double pr = ld(s.psi + r);
        h_r = h_r + pr * (ld(s.gr[0] + r) * rr0 + ld(s.gr[1] + r) * rr1);
        hc_r = hc_r + pr * (ld(s.gr[2] + r) * rr0 + ld(s.gr[3] + r) * rr1);
      }
    } else {
      h_r = sw_ghost(s, 0, f, l); hu_r = sw_ghost(s, 1, f, l); hv_r = sw_ghost(s, 2, f, l);
      hc_r = sw_ghost(s, 3, f, l); Z_r = sw_ghost(s, 4, f, l);
    }
    double fl[5];
    srnh(ld(s.q[1] + l), hu_r, ld(s.q[2] + l), hv_r, h_l, h_r, hc_l, hc_r, ld(s.q[4] + l), Z_r, n0, n1, mes, grav, fl);
#pragma unroll
    for (int k = 0; k < 5; ++k) ff[(long long)5 * f + k] = fl[k];
  }
}

__device__ __forceinline__ int order_slot_sw(uint8_t code, int k) { return (code >> (2 * k)) & 3; }

// Residuals of cell i gathered in manapy's order.
__device__ __forceinline__ void sw_gather(const mb_mesh &m, const double *__restrict__ ff, int i, double rez[5]) {
  int fs[3];
  bool own[3], bnd[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int f = ld(m.cell_faces + 4 * i + j);
    fs[j] = f;
    own[j] = ld(m.face_cellid + 2 * f) == i;
    bnd[j] = ld(m.face_cellid + 2 * f + 1) < 0;
  }
  const uint8_t code = ld(m.cell_order + i);
#pragma unroll
  for (int k = 0; k < 5; ++k) rez[k] = 0.;
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int s = order_slot_sw(code, k);
      if (bnd[s] != (pass == 1)) continue;
      const double *F = ff + (long long)5 * fs[s];
#pragma unroll
      for (int c = 0; c < 5; ++c) rez[c] = own[s] ? rez[c] - ld(F + c) : rez[c] + ld(F + c);
    }
  }
}

// Well-balanced bathymetry source of triangle i -> (src_hu, src_hv).
template <class GH, class GZ>
__device__ __forceinline__ void sw_source(const mb_mesh &m, const double *__restrict__ h,
                                          const double *__restrict__ Z, GH hg, GZ zg, double grav, int i,
                                          double &shu, double &shv) {
  const double G0 = ld(m.cell_center + 3 * i), G1 = ld(m.cell_center + 3 * i + 1);
  double c_1 = 0., c_2 = 0.;
  double ss[3][3], mata[3], matb[3], zv[3];
  const double h_1p = ld(h + i), z_1p = ld(Z + i);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int f = ld(m.cell_faces + 4 * i + j);
#pragma unroll
    for (int c = 0; c < 3; ++c) ss[j][c] = ld(m.cell_nf + 9 * i + 3 * j + c);
    double h_p1, z_p1;
    if (ld(m.face_name + f) == 0) {
      // cells.cellfid is compacted, so slot j may hold the -1 padding; manapy's
      // Numba indexing wraps it to the last cell.
      int nb = ld(m.cell_cellfid + 4 * i + j);
      if (nb < 0) nb += m.nbcells;
      h_p1 = ld(h + nb);
      z_p1 = ld(Z + nb);
    } else {
      h_p1 = hg(f);
      z_p1 = zg(f);
    }
    zv[j] = z_p1;
    mata[j] = h_p1 * ss[j][0];
    matb[j] = h_p1 * ss[j][1];
    const double hm = 0.5 * (h_1p + h_p1);
    c_1 = c_1 + (hm * 0.5 * (h_1p + h_p1)) * ss[j][0];
    c_2 = c_2 + (hm * 0.5 * (h_1p + h_p1)) * ss[j][1];
  }
  const double c_3 = 3.0 * h_1p;
  const double delta = (mata[1] * matb[2] - mata[2] * matb[1]) - (mata[0] * matb[2] - matb[0] * mata[2]) +
                       (mata[0] * matb[1] - matb[0] * mata[1]);
  const double deltax = c_3 * (mata[1] * matb[2] - mata[2] * matb[1]) - (c_1 * matb[2] - c_2 * mata[2]) +
                        (c_1 * matb[1] - c_2 * mata[1]);
  const double deltay = (c_1 * matb[2] - c_2 * mata[2]) - c_3 * (mata[0] * matb[2] - matb[0] * mata[2]) +
                        (mata[0] * c_2 - matb[0] * c_1);
  const double deltaz = (mata[1] * c_2 - matb[1] * c_1) - (mata[0] * c_2 - matb[0] * c_1) +
                        c_3 * (mata[0] * matb[1] - matb[0] * mata[1]);
  const double h_1 = deltax / delta, h_2 = deltay / delta, h_3 = deltaz / delta;
  const double z_1 = z_1p + h_1p - h_1, z_2 = z_1p + h_1p - h_2, z_3 = z_1p + h_1p - h_3;
  const double b0 = ld(m.cell_vertex1 + 2 * i), b1 = ld(m.cell_vertex1 + 2 * i + 1);
  const double ns0[2] = {(G1 - b1), -(G0 - b0)};
  double ns1[2], ns2[2], s1[2], s2[2], s3[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) { ns1[c] = ns0[c] - ss[1][c]; ns2[c] = ns0[c] + ss[0][c]; }
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    s1[c] = 0.5 * h_1 * (zv[0] * ss[0][c] + z_2 * ns0[c] + z_3 * (-1) * ns2[c]);
    s2[c] = 0.5 * h_2 * (zv[1] * ss[1][c] + z_1 * (-1) * ns0[c] + z_3 * ns1[c]);
    s3[c] = 0.5 * h_3 * (zv[2] * ss[2][c] + z_1 * ns2[c] + z_2 * (-1) * ns1[c]);
  }
  shu = -grav * (s1[0] + s2[0] + s3[0]);
  shv = -grav * (s1[1] + s2[1] + s3[1]);
}

struct FaceArr {
  const double *g;
  __device__ __forceinline__ double operator()(int f) const { return ld(g + f); }
};
struct FaceCopy {  // neumann ghost: the interior cell's value
  const double *q;
  const int32_t *fcell;
  __device__ __forceinline__ double operator()(int f) const { return ld(q + ld(fcell + 2 * f)); }
};

__global__ void __launch_bounds__(kBlock) k_time_step_sw(mb_mesh m, const double *h, const double *hu,
                                                         const double *hv, double cfl, double grav, double Dxx,
                                                         double Dyy, double *dt) {
  double best = 1e300;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    const double hi = ld(h + i), hui = ld(hu + i), hvi = ld(hv + i), vol = ld(m.cell_volume + i);
    const double velson = sqrt(grav * hi);
    double lam = 0.;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int f = ld(m.cell_faces + 4 * i + j);
      const double *N = m.face_normal + 3 * f;
      const double n0 = ld(N), n1 = ld(N + 1), mf = ld(m.face_mesure + f);
      const double u_n = fabs(hui / hi * n0 + hvi / hi * n1);
      lam += (u_n / mf + velson) * mf;
      const double mes = sqrt(n0 * n0 + n1 * n1);
      lam += (Dxx * (mes * mes) + Dyy * (mes * mes)) / vol;
    }
    best = pmin(best, cfl * vol / lam);
  }
  best = block_min(best);
  if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(dt, best);
}

__global__ void __launch_bounds__(kBlock) k_sw_gather_rez(mb_mesh m, const double *ff, double *r0, double *r1,
                                                          double *r2, double *r3, double *r4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double rez[5];
    sw_gather(m, ff, i, rez);
    r0[i] = rez[0]; r1[i] = rez[1]; r2[i] = rez[2]; r3[i] = rez[3]; r4[i] = rez[4];
  }
}

__global__ void __launch_bounds__(kBlock) k_sw_source(mb_mesh m, const double *h, const double *Z,
                                                      const double *hg, const double *zg, double grav,
                                                      double *shu, double *shv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double a, b;
    sw_source(m, h, Z, FaceArr{hg}, FaceArr{zg}, grav, i, a, b);
    shu[i] = a;
    shv[i] = b;
  }
}

struct SWQ {
  double *q[5];
};
struct SWR {
  const double *r[5];
};

__global__ void __launch_bounds__(kBlock) k_update_sw(int n, SWQ q, SWR r, const double *shu, const double *shv,
                                                      const double *dt_dev, const double *vol) {
  const double dt = *dt_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = ld(vol + i);
    q.q[0][i] += dt * (ld(r.r[0] + i) + 0.) / v;
    q.q[1][i] += dt * ((ld(r.r[1] + i) + ld(shu + i)) / v + 0. + 0.);
    q.q[2][i] += dt * ((ld(r.r[2] + i) + ld(shv + i)) / v + 0. + 0.);
    q.q[3][i] += dt * (ld(r.r[3] + i) + 0. - 0.) / v;
    q.q[4][i] += dt * (ld(r.r[4] + i) + 0.) / v;
  }
}

// Fused gather + source + update of one step (neumann ghosts), q_in -> q_out.
__global__ void __launch_bounds__(kBlock) k_sw_cell_update(mb_mesh m, SWState s, SWQ out, const double *ff,
                                                           const double *dt_dev, double grav) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  double rez[5];
  sw_gather(m, ff, i, rez);
  double shu, shv;
  sw_source(m, s.q[0], s.q[4], FaceCopy{s.q[0], m.face_cellid}, FaceCopy{s.q[4], m.face_cellid}, grav, i, shu, shv);
  const double dt = *dt_dev, v = ld(m.cell_volume + i);
  out.q[0][i] = ld(s.q[0] + i) + dt * (rez[0] + 0.) / v;
  out.q[1][i] = ld(s.q[1] + i) + dt * ((rez[1] + shu) / v + 0. + 0.);
  out.q[2][i] = ld(s.q[2] + i) + dt * ((rez[2] + shv) / v + 0. + 0.);
  out.q[3][i] = ld(s.q[3] + i) + dt * (rez[3] + 0. - 0.) / v;
  out.q[4][i] = ld(s.q[4] + i) + dt * (rez[4] + 0.) / v;
}

// ---------------------------------------------------------------- fused step (Neumann ghosts)
//
// Launch 1 (one thread per face): SRNH flux, 4 components per face (the bed
// flux is identically zero).  Launch 2 (one thread per cell): residuals
// gathered in manapy's order, bathymetry source from normals recomputed from
// the vertex coordinates, forward-Euler update, and the CFL dt of the *next*
// step from the updated state (manapy's time_step_SW on that state), reduced
// into dt_next.

#ifndef MB_SW_FAST
#define MB_SW_FAST 1
#endif

__device__ __forceinline__ int4 ldi4(const int32_t *p) { return __ldg(reinterpret_cast<const int4 *>(p)); }
__device__ __forceinline__ double2 ldd2s(const double *p) { return __ldg(reinterpret_cast<const double2 *>(p)); }
__device__ __forceinline__ int compi(const int4 v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : v.z); }

#ifndef MB_SW_FLUX_MIN_BLOCKS
#define MB_SW_FLUX_MIN_BLOCKS 3
#endif
#ifndef MB_SW_FLUX_BLOCK
#define MB_SW_FLUX_BLOCK kBlock
#endif
#ifndef MB_SW_CELL_MIN_BLOCKS
#define MB_SW_CELL_MIN_BLOCKS 4
#endif

// SRNH flux of face f of the compact-layout step, written as one 32-byte record.
template <bool ORDER2, bool FAST>
__device__ __forceinline__ void sw2_flux_face(const mb_mesh &m, const SWState &s, double grav, double *ff, int f) {
  const int l = ld(m.face_cellid + 2 * f), r = ld(m.face_cellid + 2 * f + 1);
  const double n0 = ld(m.face_normal + 3 * f), n1 = ld(m.face_normal + 3 * f + 1), mes = ld(m.face_mesure + f);
  double h_l = ld(s.q[0] + l), hc_l = ld(s.q[3] + l);
  const int rr = r >= 0 ? r : l;  // Neumann ghost: the interior cell's state
  double h_r = ld(s.q[0] + rr), hc_r = ld(s.q[3] + rr);
  if (ORDER2) {
    const double *fc = m.face_center + 3 * f, *cc = m.cell_center;
    const double rl0 = ld(fc) - ld(cc + 3 * l), rl1 = ld(fc + 1) - ld(cc + 3 * l + 1);
    const double pl = ld(s.psi + l);
    h_l = h_l + pl * (ld(s.gr[0] + l) * rl0 + ld(s.gr[1] + l) * rl1);
    hc_l = hc_l + pl * (ld(s.gr[2] + l) * rl0 + ld(s.gr[3] + l) * rl1);
    if (r >= 0) {
      const double rr0 = ld(fc) - ld(cc + 3 * r), rr1 = ld(fc + 1) - ld(cc + 3 * r + 1);
      const double pr = ld(s.psi + r);
      h_r = h_r + pr * (ld(s.gr[0] + r) * rr0 + ld(s.gr[1] + r) * rr1);
      hc_r = hc_r + pr * (ld(s.gr[2] + r) * rr0 + ld(s.gr[3] + r) * rr1);
    }
  }
  const double hu_l = ld(s.q[1] + l), hv_l = ld(s.q[2] + l);
  double hu_r, hv_r;
  if (r < 0 && s.walls == MB_WALLS_REFLECT) {
    wall_mirror(hu_l, hv_l, n0, n1, hu_r, hv_r);
  } else {
    hu_r = ld(s.q[1] + rr);
    hv_r = ld(s.q[2] + rr);
  }
  double fl[4];
  srnh0<FAST>(hu_l, hu_r, hv_l, hv_r, h_l, h_r, hc_l, hc_r, ld(s.q[4] + l), ld(s.q[4] + rr), n0, n1, mes, grav, fl);
#if MB_V4_IO
  st4d_plain(ff + 4 * (long long)f, fl[0], fl[1], fl[2], fl[3]);
#else
  reinterpret_cast<double2 *>(ff)[2 * f] = make_double2(fl[0], fl[1]);
  reinterpret_cast<double2 *>(ff)[2 * f + 1] = make_double2(fl[2], fl[3]);
#endif
}

template <bool ORDER2, bool FAST>
__global__ void __launch_bounds__(MB_SW_FLUX_BLOCK, MB_SW_FLUX_MIN_BLOCKS) k_sw2_flux(mb_mesh m, SWState s, double grav, double *ff,
                                                     double *dt_next) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f == 0 && dt_next) *dt_next = 1e6;
  if (f >= m.nbfaces) return;
  sw2_flux_face<ORDER2, FAST>(m, s, grav, ff, f);
}

// CFL dt candidate of a cell (manapy/solvers/shallowater/fvm_utils.py:16-42, without
// diffusion) from its state and its three face normals, written with explicit
// round-to-nearest operations: no multiply-add is contracted, so every kernel that calls
// it (the fused step's next dt, mb_sw_dt) gives the same bits.
__device__ __forceinline__ double sw_dt_candidate(double h, double hu, double hv, const double n0[3],
                                                  const double n1[3], double vol, double cfl, double grav) {
  const double velson = __dsqrt_rn(__dmul_rn(grav, h));
  const double u = __ddiv_rn(hu, h), v = __ddiv_rn(hv, h);
  double lam = 0.;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double mes = __dsqrt_rn(__dadd_rn(__dmul_rn(n0[j], n0[j]), __dmul_rn(n1[j], n1[j])));  // faces.mesure
    const double u_n = fabs(__dadd_rn(__dmul_rn(u, n0[j]), __dmul_rn(v, n1[j])));
    lam = __dadd_rn(lam, __dmul_rn(__dadd_rn(__ddiv_rn(u_n, mes), velson), mes));
  }
  return __ddiv_rn(__dmul_rn(cfl, vol), lam);
}

// the three stored face normals of cell i (exact), from the compact 2D tables
__device__ __forceinline__ void sw_cell_normals(const mb_mesh &m, int i, double n0[3], double n1[3]) {
  const int4 vt = __ldg(reinterpret_cast<const int4 *>(m.cell_vtx + 4 * i));
  const uint32_t fl = ld(m.cell_flags + i);
  const double2 P0 = __ldg(reinterpret_cast<const double2 *>(m.node_coord + 2 * vt.x));
  const double2 P1 = __ldg(reinterpret_cast<const double2 *>(m.node_coord + 2 * vt.y));
  const double2 P2 = __ldg(reinterpret_cast<const double2 *>(m.node_coord + 2 * vt.z));
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const bool rev = (fl >> (3 + j)) & 1u;
    const double2 Pj = j == 0 ? P0 : (j == 1 ? P1 : P2), Pk = j == 0 ? P1 : (j == 1 ? P2 : P0);
    const double2 Xa = rev ? Pk : Pj, Xb = rev ? Pj : Pk;
    double x = Xa.y - Xb.y, y = Xb.x - Xa.x;
    if ((fl >> (6 + j)) & 1u) { x = -1 * x; y = -1 * y; }
    n0[j] = x;
    n1[j] = y;
  }
}

__global__ void __launch_bounds__(kBlock) k_sw_dt(mb_mesh m, const double *h, const double *hu, const double *hv,
                                                  double cfl, double grav, double *dt) {
  double best = 1e300;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double n0[3], n1[3];
    sw_cell_normals(m, i, n0, n1);
    best = pmin(best, sw_dt_candidate(ld(h + i), ld(hu + i), ld(hv + i), n0, n1, ld(m.cell_volume + i), cfl, grav));
  }
  best = block_min(best);
  if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(dt, best);
}

// flags of the compact 2D layout (cell_flags): bit j own, 3+j node order, 6+j normal
// flipped, 9+j the cell's outward normal table (cells.nf) holds minus the face normal
__device__ __forceinline__ double sw2_cell_body(const mb_mesh &m, const SWState &s, const SWQ &out, const double *ff,
                                                const double *dt_cur, bool want_dt, double cfl, double grav,
                                                int i);

__global__ void __launch_bounds__(kBlock, MB_SW_CELL_MIN_BLOCKS) k_sw2_cell(mb_mesh m, SWState s, SWQ out, const double *ff,
                                                     const double *dt_cur, double *dt_next, double cfl,
                                                     double grav, int c0, int c1) {
  const int i = c0 + blockIdx.x * blockDim.x + threadIdx.x;   // cells [c0, c1)
  // every thread of the block reaches the dt reduction below (it synchronises the block)
  double best = 1e300;
  if (i < c1) best = sw2_cell_body(m, s, out, ff, dt_cur, dt_next != nullptr, cfl, grav, i);
  if (dt_next) {
    best = block_min(best);
    if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(dt_next, best);
  }
}

// One cell of k_sw2_cell; returns the cell's next-step dt candidate (1e300 if not wanted).
__device__ __forceinline__ double sw2_cell_body(const mb_mesh &m, const SWState &s, const SWQ &out, const double *ff,
                                                const double *dt_cur, bool want_dt, double cfl, double grav,
                                                int i) {
  const int4 vt = ldi4(m.cell_vtx + 4 * i);
  const int4 nb = ldi4(m.cell_nbr + 4 * i);
  const int4 cf = ldi4(m.cell_faces + 4 * i);
  const int4 fid = ldi4(m.cell_cellfid + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const uint8_t code = ld(m.cell_order + i);
  const double2 P0 = ldd2s(m.node_coord + 2 * vt.x), P1 = ldd2s(m.node_coord + 2 * vt.y),
                P2 = ldd2s(m.node_coord + 2 * vt.z);
  const double2 G = ldd2s(m.cell_xy + 2 * i);
  const double h_i = ld(s.q[0] + i), hu_i = ld(s.q[1] + i), hv_i = ld(s.q[2] + i), hc_i = ld(s.q[3] + i);
  const double Z_i = ld(s.q[4] + i);
  const double vol = ld(m.cell_volume + i);
  // face fluxes and normals of the three local faces
  double F[3][4], n0[3], n1[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int f = compi(cf, j);
#if MB_V4_IO
    ld4d(ff + 4 * (long long)f, F[j][0], F[j][1], F[j][2], F[j][3]);
#else
    const double2 a = ldd2s(ff + 4 * f), b = ldd2s(ff + 4 * f + 2);
    F[j][0] = a.x; F[j][1] = a.y; F[j][2] = b.x; F[j][3] = b.y;
#endif
    const bool rev = (fl >> (3 + j)) & 1u;
    const double2 Pj = j == 0 ? P0 : (j == 1 ? P1 : P2), Pk = j == 0 ? P1 : (j == 1 ? P2 : P0);
    const double2 Xa = rev ? Pk : Pj, Xb = rev ? Pj : Pk;
    double x = Xa.y - Xb.y, y = Xb.x - Xa.x;          // stored face normal, exact
    if ((fl >> (6 + j)) & 1u) { x = -1 * x; y = -1 * y; }
    n0[j] = x;
    n1[j] = y;
  }
  // residuals: inner faces by ascending manapy face id, then boundary faces
  double rez[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int sl = (code >> (2 * k)) & 3;
      const int o = compi(nb, sl);
      if ((o < 0) != (pass == 1)) continue;
      const bool own = (fl >> sl) & 1u;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double v = sl == 0 ? F[0][c] : (sl == 1 ? F[1][c] : F[2][c]);
        rez[c] = own ? rez[c] - v : rez[c] + v;
      }
    }
  }
  // bathymetry source (manapy/solvers/shallowater/fvm_utils.py:72-148)
  double c_1 = 0., c_2 = 0., ss0[3], ss1[3], mata[3], matb[3], zv[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const bool neg = (fl >> (9 + j)) & 1u;
    ss0[j] = neg ? -1.0 * n0[j] : n0[j];
    ss1[j] = neg ? -1.0 * n1[j] : n1[j];
    double h_p1, z_p1;
    if (compi(nb, j) >= 0) {
      // cells.cellfid slot j (compacted; its padding already maps to manapy's wrapped last cell)
      const int c = compi(fid, j);
      h_p1 = ld(s.q[0] + c);
      z_p1 = ld(s.q[4] + c);
    } else {
      h_p1 = h_i;  // Neumann ghost
      z_p1 = Z_i;
    }
    zv[j] = z_p1;
    mata[j] = h_p1 * ss0[j];
    matb[j] = h_p1 * ss1[j];
    const double hm = 0.5 * (h_i + h_p1);
    c_1 = c_1 + (hm * 0.5 * (h_i + h_p1)) * ss0[j];
    c_2 = c_2 + (hm * 0.5 * (h_i + h_p1)) * ss1[j];
  }
  const double c_3 = 3.0 * h_i;
  const double delta = (mata[1] * matb[2] - mata[2] * matb[1]) - (mata[0] * matb[2] - matb[0] * mata[2]) +
                       (mata[0] * matb[1] - matb[0] * mata[1]);
  const double deltax = c_3 * (mata[1] * matb[2] - mata[2] * matb[1]) - (c_1 * matb[2] - c_2 * mata[2]) +
                        (c_1 * matb[1] - c_2 * mata[1]);
  const double deltay = (c_1 * matb[2] - c_2 * mata[2]) - c_3 * (mata[0] * matb[2] - matb[0] * mata[2]) +
                        (mata[0] * c_2 - matb[0] * c_1);
  const double deltaz = (mata[1] * c_2 - matb[1] * c_1) - (mata[0] * c_2 - matb[0] * c_1) +
                        c_3 * (mata[0] * matb[1] - matb[0] * mata[1]);
  const double h_1 = deltax / delta, h_2 = deltay / delta, h_3 = deltaz / delta;
  const double z_1 = Z_i + h_i - h_1, z_2 = Z_i + h_i - h_2, z_3 = Z_i + h_i - h_3;
  const double ns0x = (G.y - P1.y), ns0y = -(G.x - P1.x);
  const double ns1x = ns0x - ss0[1], ns1y = ns0y - ss1[1];
  const double ns2x = ns0x + ss0[0], ns2y = ns0y + ss1[0];
  const double s1x = 0.5 * h_1 * (zv[0] * ss0[0] + z_2 * ns0x + z_3 * (-1) * ns2x);
  const double s1y = 0.5 * h_1 * (zv[0] * ss1[0] + z_2 * ns0y + z_3 * (-1) * ns2y);
  const double s2x = 0.5 * h_2 * (zv[1] * ss0[1] + z_1 * (-1) * ns0x + z_3 * ns1x);
  const double s2y = 0.5 * h_2 * (zv[1] * ss1[1] + z_1 * (-1) * ns0y + z_3 * ns1y);
  const double s3x = 0.5 * h_3 * (zv[2] * ss0[2] + z_1 * ns2x + z_2 * (-1) * ns1x);
  const double s3y = 0.5 * h_3 * (zv[2] * ss1[2] + z_1 * ns2y + z_2 * (-1) * ns1y);
  const double shu = -grav * (s1x + s2x + s3x);
  const double shv = -grav * (s1y + s2y + s3y);
  // update (manapy/solvers/shallowater/fvm_utils.py:3-14, no Coriolis/wind/diffusion)
  const double dt = *dt_cur;
  const double h_n = h_i + dt * (rez[0] + 0.) / vol;
  const double hu_n = hu_i + dt * ((rez[1] + shu) / vol + 0. + 0.);
  const double hv_n = hv_i + dt * ((rez[2] + shv) / vol + 0. + 0.);
  const double hc_n = hc_i + dt * (rez[3] + 0. - 0.) / vol;
  out.q[0][i] = h_n;
  out.q[1][i] = hu_n;
  out.q[2][i] = hv_n;
  out.q[3][i] = hc_n;
  if (out.q[4] != s.q[4]) out.q[4][i] = Z_i;  // the bed does not move
  // next step's dt from the updated state (manapy/solvers/shallowater/fvm_utils.py:16-42)
  if (!want_dt) return 1e300;
  return sw_dt_candidate(h_n, hu_n, hv_n, n0, n1, vol, cfl, grav);
}

__global__ void __launch_bounds__(kBlock) k_srnh_batch(int n, const double *st, const double *nrm,
                                                       const double *mes, double grav, double *flux) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double *s = st + 10 * (long long)k;
    double fl[5];
    srnh(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], s[8], s[9], nrm[3 * k], nrm[3 * k + 1], mes[k], grav, fl);
    for (int c = 0; c < 5; ++c) flux[5 * (long long)k + c] = fl[c];
  }
}

__global__ void k_fill_sw(double *p, double v) { *p = v; }

inline int grid_for_sw(long long n) {
  int g = ceil_div(n, kBlock);
  const int cap = 148 * 16;
  return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace mb

using namespace mb;

#define ST(s) reinterpret_cast<cudaStream_t>(s)

static bool sw_mesh_ok(const mb_mesh *m) {
  return m && m->dim == 2 && m->nlf == 3 && m->nbcells > 0 && m->nbfaces > 0;
}

// declared in fv_advdiff.cu
namespace mb {
int sw_gradients(const mb_mesh &m, const double *h, const double *hc, double *hx, double *hy, double *cx,
                 double *cy, double *psi, cudaStream_t st);
}

namespace mb {

// ---------------------------------------------------------------- batches of meshes, FP64
//
// The FP64 twin of mb_sw_batch_step_f32c: block b of a launch belongs to item
// map[b] and runs the single-mesh block body (first order, Neumann walls) on
// that item's tables; the batch clock picks each item's ping-pong state and dt.

__global__ void __launch_bounds__(MB_SW_FLUX_BLOCK, MB_SW_FLUX_MIN_BLOCKS)
    k_sw2_batch_flux(const mb_sw_item_f64 *__restrict__ items, const int32_t *__restrict__ map,
                     const int32_t *__restrict__ clock) {
  const mb_sw_item_f64 &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;
  const int par = (t - it.start_step) & 1;
  const int f = ((int)blockIdx.x - it.f_begin) * blockDim.x + threadIdx.x;
  if (f == 0) it.dt[par ^ 1] = 1e6;
  if (f >= it.m.nbfaces) return;
  SWState s{};
  for (int k = 0; k < 5; ++k) s.q[k] = it.q[par][k];
  sw2_flux_face<false, MB_SW_FAST>(it.m, s, it.grav, it.face_flux, f);
}

#ifndef MB_SW_BATCH_CELL_MIN_BLOCKS
#define MB_SW_BATCH_CELL_MIN_BLOCKS MB_SW_CELL_MIN_BLOCKS
#endif
__global__ void __launch_bounds__(kBlock, MB_SW_BATCH_CELL_MIN_BLOCKS)
    k_sw2_batch_cell(const mb_sw_item_f64 *__restrict__ items, const int32_t *__restrict__ map,
                     const int32_t *__restrict__ clock) {
  const mb_sw_item_f64 &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;  // uniform over the block
  const int par = (t - it.start_step) & 1;
  SWState s{};
  SWQ out;
  for (int k = 0; k < 5; ++k) {
    s.q[k] = it.q[par][k];
    out.q[k] = it.q[par ^ 1][k];
  }
  const int i = ((int)blockIdx.x - it.c_begin) * blockDim.x + threadIdx.x;
  double best = 1e300;
  if (i < it.m.nbcells) best = sw2_cell_body(it.m, s, out, it.face_flux, it.dt + par, true, it.cfl, it.grav, i);
  best = block_min(best);
  if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(it.dt + (par ^ 1), best);
}

__global__ void k_sw_batch_tick(int32_t *clock) { *clock += 1; }

}  // namespace mb

extern "C" {

int mb_srnh_flux(int32_t n, const double *states, const double *normals, const double *mesure, double grav,
                 double *flux, void *stream) {
  MB_NVTX();
  if (n < 0 || (n > 0 && (!states || !normals || !mesure || !flux))) return MB_EINVAL;
  if (n == 0) return MB_OK;
  k_srnh_batch<<<grid_for_sw(n), kBlock, 0, ST(stream)>>>(n, states, normals, mesure, grav, flux);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_time_step_sw(const mb_mesh *m, const double *h, const double *hu, const double *hv, double cfl,
                    double grav, double Dxx, double Dyy, double *dt_dev, void *stream) {
  MB_NVTX();
  if (!sw_mesh_ok(m) || !h || !hu || !hv || !dt_dev) return MB_EINVAL;
  k_fill_sw<<<1, 1, 0, ST(stream)>>>(dt_dev, 1e6);
  k_time_step_sw<<<grid_for_sw(m->nbcells), kBlock, 0, ST(stream)>>>(*m, h, hu, hv, cfl, grav, Dxx, Dyy, dt_dev);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_explicitscheme_convective_sw(const mb_mesh *m, double *const rez[5], const double *const q[5],
                                    const double *const g[5], const double *const grads[4], const double *psi,
                                    double grav, int32_t order, double *face_flux, void *stream) {
  MB_NVTX();
  if (!sw_mesh_ok(m) || !rez || !q || !g || !face_flux || (order != 1 && order != 2)) return MB_EINVAL;
  SWState s{};
  for (int k = 0; k < 5; ++k) {
    if (!rez[k] || !q[k] || !g[k]) return MB_EINVAL;
    s.q[k] = q[k];
    s.g[k] = g[k];
  }
  if (order == 2) {
    if (!grads || !psi) return MB_EINVAL;
    for (int k = 0; k < 4; ++k) {
      if (!grads[k]) return MB_EINVAL;
      s.gr[k] = grads[k];
    }
    s.psi = psi;
    k_sw_face_flux<true><<<grid_for_sw(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, s, grav, face_flux);
  } else {
    k_sw_face_flux<false><<<grid_for_sw(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, s, grav, face_flux);
  }
  k_sw_gather_rez<<<grid_for_sw(m->nbcells), kBlock, 0, ST(stream)>>>(*m, face_flux, rez[0], rez[1], rez[2],
                                                                       rez[3], rez[4]);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_term_source_srnh_sw(const mb_mesh *m, const double *h, const double *Z, const double *h_ghost,
                           const double *Z_ghost, double grav, double *src_hu, double *src_hv, void *stream) {
  MB_NVTX();
  if (!sw_mesh_ok(m) || !h || !Z || !h_ghost || !Z_ghost || !src_hu || !src_hv || !m->cell_cellfid ||
      !m->cell_nf || !m->cell_vertex1)
    return MB_EINVAL;
  k_sw_source<<<grid_for_sw(m->nbcells), kBlock, 0, ST(stream)>>>(*m, h, Z, h_ghost, Z_ghost, grav, src_hu, src_hv);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_update_sw(const mb_mesh *m, double *const q[5], const double *const rez[5], const double *src_hu,
                 const double *src_hv, const double *dt_dev, void *stream) {
  MB_NVTX();
  if (!sw_mesh_ok(m) || !q || !rez || !src_hu || !src_hv || !dt_dev) return MB_EINVAL;
  SWQ qq;
  SWR rr;
  for (int k = 0; k < 5; ++k) {
    if (!q[k] || !rez[k]) return MB_EINVAL;
    qq.q[k] = q[k];
    rr.r[k] = rez[k];
  }
  k_update_sw<<<grid_for_sw(m->nbcells), kBlock, 0, ST(stream)>>>(m->nbcells, qq, rr, src_hu, src_hv, dt_dev,
                                                                   m->cell_volume);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_sw_step(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl, double grav,
               int32_t order, double *scratch, double *face_flux, const double *dt_cur, double *dt_next,
               void *stream) {
  MB_NVTX();
  return mb_sw_step_ex(m, q_in, q_out, cfl, grav, order, MB_WALLS_NEUMANN, scratch, face_flux, dt_cur, dt_next,
                       stream);
}

// part < 0: the whole step; part 0: the face fluxes and the cells [0, nfirst); part 1: the
// cells [nfirst, nbcells), reading the face fluxes part 0 left in face_flux
static int sw_step(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl, double grav,
                   int32_t order, int32_t walls, double *scratch, double *face_flux, const double *dt_cur,
                   double *dt_next, int part, int nfirst, void *stream) {
  if (!sw_mesh_ok(m) || !q_in || !q_out || !face_flux || !dt_cur || (order != 1 && order != 2)) return MB_EINVAL;
  if (part >= 0 && (nfirst < 0 || nfirst > m->nbcells)) return MB_EINVAL;
  if (walls != MB_WALLS_NEUMANN && walls != MB_WALLS_REFLECT) return MB_EINVAL;
  if (!m->cell_cellfid || !m->cell_vtx || !m->cell_nbr || !m->cell_flags || !m->node_coord || !m->cell_xy)
    return MB_EINVAL;
  SWState s{};
  SWQ out;
  for (int k = 0; k < 5; ++k) {
    if (!q_in[k] || !q_out[k] || (k < 4 && q_in[k] == q_out[k])) return MB_EINVAL;
    s.q[k] = q_in[k];
    s.g[k] = nullptr;  // neumann ghosts
    out.q[k] = q_out[k];
  }
  s.walls = walls;
  if (dt_next == dt_cur) return MB_EINVAL;
#if MB_V4_IO
  if ((reinterpret_cast<uintptr_t>(face_flux) & 31) != 0) return MB_EINVAL;   // 256-bit flux records
#endif
  cudaStream_t st = ST(stream);
  const int fb = ceil_div(m->nbfaces, MB_SW_FLUX_BLOCK);
  const int c0 = part == 1 ? nfirst : 0, c1 = part == 0 ? nfirst : m->nbcells;
  if (part == 1) {
    if (c1 > c0)
      k_sw2_cell<<<ceil_div(c1 - c0, kBlock), kBlock, 0, st>>>(*m, s, out, face_flux, dt_cur, dt_next, cfl, grav, c0,
                                                                c1);
    return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
  }
  if (order == 2) {
    if (!scratch) return MB_EINVAL;
    const long long n = m->nbcells;
    double *hx = scratch, *hy = scratch + n, *cx = scratch + 2 * n, *cy = scratch + 3 * n, *psi = scratch + 4 * n;
    const int rc = sw_gradients(*m, q_in[0], q_in[3], hx, hy, cx, cy, psi, st);
    if (rc != MB_OK) return rc;
    s.gr[0] = hx; s.gr[1] = hy; s.gr[2] = cx; s.gr[3] = cy;
    s.psi = psi;
    k_sw2_flux<true, MB_SW_FAST><<<fb, MB_SW_FLUX_BLOCK, 0, st>>>(*m, s, grav, face_flux, dt_next);
  } else {
    k_sw2_flux<false, MB_SW_FAST><<<fb, MB_SW_FLUX_BLOCK, 0, st>>>(*m, s, grav, face_flux, dt_next);
  }
  if (c1 > c0)
    k_sw2_cell<<<ceil_div(c1 - c0, kBlock), kBlock, 0, st>>>(*m, s, out, face_flux, dt_cur, dt_next, cfl, grav, c0, c1);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_sw_step_ex(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl, double grav,
                  int32_t order, int32_t walls, double *scratch, double *face_flux, const double *dt_cur,
                  double *dt_next, void *stream) {
  MB_NVTX();
  return sw_step(m, q_in, q_out, cfl, grav, order, walls, scratch, face_flux, dt_cur, dt_next, -1, 0, stream);
}

int mb_sw_step_split(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl,
                     double grav, int32_t order, int32_t walls, double *scratch, double *face_flux,
                     const double *dt_cur, double *dt_next, int32_t part, int32_t nfirst, void *stream) {
  MB_NVTX();
  if (part != 0 && part != 1) return MB_EINVAL;
  return sw_step(m, q_in, q_out, cfl, grav, order, walls, scratch, face_flux, dt_cur, dt_next, part, nfirst, stream);
}

int mb_sw_dt(const mb_mesh *m, const double *h, const double *hu, const double *hv, double cfl, double grav,
             double *dt_dev, void *stream) {
  MB_NVTX();
  if (!sw_mesh_ok(m) || !h || !hu || !hv || !dt_dev || !m->cell_vtx || !m->cell_flags || !m->node_coord)
    return MB_EINVAL;
  k_fill_sw<<<1, 1, 0, ST(stream)>>>(dt_dev, 1e6);
  k_sw_dt<<<grid_for_sw(m->nbcells), kBlock, 0, ST(stream)>>>(*m, h, hu, hv, cfl, grav, dt_dev);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_sw_batch_step(const mb_sw_item_f64 *items, const int32_t *face_map, int32_t face_blocks,
                     const int32_t *cell_map, int32_t cell_blocks, int32_t *clock, void *stream) {
  MB_NVTX();
  if (!items || !face_map || !cell_map || !clock || face_blocks <= 0 || cell_blocks <= 0) return MB_EINVAL;
  cudaStream_t st = ST(stream);
  k_sw2_batch_flux<<<face_blocks, MB_SW_FLUX_BLOCK, 0, st>>>(items, face_map, clock);
  k_sw2_batch_cell<<<cell_blocks, kBlock, 0, st>>>(items, cell_map, clock);
  k_sw_batch_tick<<<1, 1, 0, st>>>(clock);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

}  // extern "C"
