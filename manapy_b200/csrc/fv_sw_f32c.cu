// FP32-compensated shallow-water step (first order, Neumann ghosts).
//
// Same two launches as mb_sw_step (manapy/solvers/shallowater/system.py:186-281):
// one thread per face evaluates the SRNH flux with As = 0
// (manapy/solvers/shallowater/fvm_utils.py:152-342), one thread per cell gathers
// the residuals in manapy's order, adds the bathymetry source
// (fvm_utils.py:44-148), updates the state (fvm_utils.py:3-14) and evaluates
// the next step's CFL dt (fvm_utils.py:16-42).  Precision split:
//   FP32  state (h, hu, hv, hc, Z), SRNH flux arithmetic and face fluxes,
//         residuals (compensated sums);
//   FP64  coordinates, normals and areas (rounded once to FP32 for the flux),
//         the bathymetry source (its 3x3 Cramer solve cancels), dt.
#include "fv_compact.cuh"

namespace mb {

namespace {

struct CompSumF {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float t = s + x;
    c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s + c; }
};

// SRNH flux with As = 0 in FP32: closed-form eigenvalues {0, u + c, u - c} in the
// order manapy's trigonometric formula returns them (largest, smallest, middle).
__device__ __forceinline__ void srnh_f32(float hu_l, float hu_r, float hv_l, float hv_r, float h_l, float h_r,
                                         float hc_l, float hc_r, float Z_l, float Z_r, float n0, float n1, float im,
                                         float grav, float flux[4]) {
  const float ninv0 = -n1, ninv1 = n0;
  const float sl = sqrtf(h_l), sr = sqrtf(h_r);
  const float il = 1.f / h_l, ir = 1.f / h_r, is = 1.f / (sl + sr);
  const float u_h = (hu_l * il * sl + hu_r * ir * sr) * is;
  const float v_h = (hv_l * il * sl + hv_r * ir * sr) * is;
  const float c_h = (hc_l * il * sl + hc_r * ir * sr) * is;
  const float uroe = (u_h * n0 + v_h * n1) * im;
  const float vroe = (u_h * ninv0 + v_h * ninv1) * im;
  const float uleft = (hu_l * n0 + hv_l * n1) * im, vleft = (hu_l * ninv0 + hv_l * ninv1) * im;
  const float uright = (hu_r * n0 + hv_r * n1) * im, vright = (hu_r * ninv0 + hv_r * ninv1) * im;
  const float hroe = 0.5f * (h_l + h_r), croe = c_h;
  float w_lrh = hroe, w_lrhu = 0.5f * (uleft + uright), w_lrhv = 0.5f * (vleft + vright);
  float w_lrhc = 0.5f * (hc_l + hc_r);
  const float wd0 = h_r - h_l, wd1 = uright - uleft, wd2 = vright - vleft, wd3 = hc_r - hc_l, wd4 = Z_r - Z_l;
  const float u2 = uroe * uroe;
  const float sound = sqrtf(grav * hroe);
  const float a = uroe + sound, b = uroe - sound;
  const float lambda1 = fmaxf(a, 0.f), lambda2 = fminf(b, 0.f);
  const float lambda3 = (a < 0.f) ? a : ((b > 0.f) ? b : 0.f);
  const float alpha1 = lambda1 - uroe, alpha2 = lambda2 - uroe, alpha3 = lambda3 - uroe;
  const float s2 = sound * sound;
  const float gamma1 = s2 - u2 + lambda2 * lambda3;
  const float gamma2 = s2 - u2 + lambda1 * lambda3;
  const float gamma3 = s2 - u2 + lambda1 * lambda2;
  // sigma_k = prod_{j != k} (alpha_k - alpha_j) up to sign, factored (no cancellation)
  const float sigma1 = (alpha1 - alpha2) * (alpha1 - alpha3);
  const float sigma2 = -(alpha2 - alpha1) * (alpha2 - alpha3);
  const float sigma3 = (alpha3 - alpha1) * (alpha3 - alpha2);
  const float eps = 1e-10f;
  const float sign1 = fabsf(lambda1) < eps ? 0.f : copysignf(1.f, lambda1);
  const float sign2 = fabsf(lambda2) < eps ? 0.f : copysignf(1.f, lambda2);
  const float sign3 = fabsf(lambda3) < eps ? 0.f : copysignf(1.f, lambda3);
  const float sign4 = fabsf(uroe) < eps ? 0.f : copysignf(1.f, uroe);
  const float sign5 = sign4;
  const float t1 = alpha2 + alpha3, t2 = alpha1 + alpha3, t3 = alpha1 + alpha2;
  const float l1 = lambda1 * sign1, l2 = lambda2 * sign2, l3 = lambda3 * sign3;
  const float i1 = 1.f / sigma1, i2 = 1.f / sigma2, i3 = 1.f / sigma3;
  const float g1 = gamma1 * i1, g2 = gamma2 * i2, g3 = gamma3 * i3;
  const float q1 = t1 * i1, q2 = t2 * i2, q3 = t3 * i3;
  const float e1 = s2 * i1, e2 = s2 * i2, e3 = s2 * i3;
  const float r00 = sign1 * g1 - sign2 * g2 + sign3 * g3;
  const float r10 = l1 * g1 - l2 * g2 + l3 * g3;
  const float r20 = vroe * (r00 - sign5);
  const float r30 = croe * (r00 - sign4);
  const float r01 = -sign1 * q1 + sign2 * q2 - sign3 * q3;
  const float r11 = -l1 * q1 + l2 * q2 - l3 * q3;
  const float r21 = vroe * r01, r31 = croe * r01;
  const float r04 = sign1 * e1 - sign2 * e2 + sign3 * e3;
  const float r14 = l1 * e1 - l2 * e2 + l3 * e3;
  const float r24 = vroe * r04, r34 = croe * r04;
  const float hnew = r00 * wd0 + r01 * wd1 + r04 * wd4;
  const float unew0 = r10 * wd0 + r11 * wd1 + r14 * wd4;
  const float vnew0 = r20 * wd0 + r21 * wd1 + sign5 * wd2 + r24 * wd4;
  const float cnew = r30 * wd0 + r31 * wd1 + sign4 * wd3 + r34 * wd4;
  w_lrh -= 0.5f * hnew;
  w_lrhu -= 0.5f * unew0;
  w_lrhv -= 0.5f * vnew0;
  w_lrhc -= 0.5f * cnew;
  const float unew = (w_lrhu * n0 - w_lrhv * n1) * im;
  const float vnew = (-w_lrhu * ninv0 + w_lrhv * ninv1) * im;
  const float q_s = n0 * unew + n1 * vnew;
  const float gh = 0.5f * grav * w_lrh * w_lrh;
  const float iw = 1.f / w_lrh;
  flux[0] = q_s;
  flux[1] = q_s * unew * iw + gh * n0;
  flux[2] = q_s * vnew * iw + gh * n1;
  flux[3] = q_s * w_lrhc * iw;
}

struct SWStateF {
  const float *q[5];   // h, hu, hv, hc, Z
  const float *lo[4];  // rounding errors of h, hu, hv, hc (all NULL: plain FP32 state)
  int walls;           // MB_WALLS_NEUMANN or MB_WALLS_REFLECT
};
struct SWOutF {
  float *q[5];
  float *lo[4];
};

// (q, lo) + inc -> (q', lo') with q' + lo' = q + (inc + lo) exactly (Knuth's two-sum)
__device__ __forceinline__ float sw_store(float q, float inc, const float *lo_in, float *lo_out, float *q_out, int i) {
  if (!lo_in) {
    q_out[i] = q + inc;
    return q_out[i];
  }
  const float a = inc + lo_in[i];
  const float s = q + a;
  const float bv = s - q;
  lo_out[i] = (q - (s - bv)) + (a - bv);
  q_out[i] = s;
  return s;
}

__device__ __forceinline__ void sw2c_face(const mb_mesh &m, const SWStateF &s, float grav, float *ff, double *dt_next,
                                          int f) {
  if (f == 0 && dt_next) *dt_next = 1e6;
  if (f >= m.nbfaces) return;
  const int l = ld(m.face_cellid + 2 * f), r = ld(m.face_cellid + 2 * f + 1);
  const int rr = r >= 0 ? r : l;  // Neumann ghost: the interior cell's state
  const float4 nm = __ldg(reinterpret_cast<const float4 *>(m.face_nm_f32) + f);  // n0, n1, 1/mesure
  const float hu_l = ld(s.q[1] + l), hv_l = ld(s.q[2] + l);
  float hu_r, hv_r;
  if (r < 0 && s.walls == MB_WALLS_REFLECT) {
    // reflective wall: normal momentum reversed, q - 2 (q.n) n / |n|^2 with 1/|n| = nm.z
    const float k = 2.f * (hu_l * nm.x + hv_l * nm.y) * (nm.z * nm.z);
    hu_r = hu_l - k * nm.x;
    hv_r = hv_l - k * nm.y;
  } else {
    hu_r = ld(s.q[1] + rr);
    hv_r = ld(s.q[2] + rr);
  }
  float fl[4];
  srnh_f32(hu_l, hu_r, hv_l, hv_r, ld(s.q[0] + l), ld(s.q[0] + rr), ld(s.q[3] + l), ld(s.q[3] + rr),
           ld(s.q[4] + l), ld(s.q[4] + rr), nm.x, nm.y, nm.z, grav, fl);
  reinterpret_cast<float4 *>(ff)[f] = make_float4(fl[0], fl[1], fl[2], fl[3]);
}

__global__ void __launch_bounds__(kBlock) k_sw2c_flux(mb_mesh m, SWStateF s, float grav, float *ff, double *dt_next) {
  sw2c_face(m, s, grav, ff, dt_next, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void k_sw_clock_tick(int32_t *clock) { *clock += 1; }

__device__ __forceinline__ double sw2c_cell_body(const mb_mesh &m, const SWStateF &s, const SWOutF &out,
                                                 const float *ff, double dt, bool want_dt, double cfl, double grav,
                                                 int i) {
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const int4 cf = ld4(m.cell_faces + 4 * i);
  const int4 fid = ld4(m.cell_cellfid + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const uint8_t code = ld(m.cell_order + i);
  const double2 P0 = ldd2(m.node_coord + 2 * vt.x), P1 = ldd2(m.node_coord + 2 * vt.y),
                P2 = ldd2(m.node_coord + 2 * vt.z);
  const double2 G = ldd2(m.cell_xy + 2 * i);
  const float h_i = ld(s.q[0] + i), hu_i = ld(s.q[1] + i), hv_i = ld(s.q[2] + i), hc_i = ld(s.q[3] + i);
  const float Z_i = ld(s.q[4] + i);
  const double vol = ld(m.cell_volume + i);
  float4 F[3];
  double n0[3], n1[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    F[j] = __ldg(reinterpret_cast<const float4 *>(ff) + comp(cf, j));
    const bool rev = f2_rev(fl, j);
    const double2 Pj = j == 0 ? P0 : (j == 1 ? P1 : P2), Pk = j == 0 ? P1 : (j == 1 ? P2 : P0);
    const double2 Xa = rev ? Pk : Pj, Xb = rev ? Pj : Pk;
    double x = Xa.y - Xb.y, y = Xb.x - Xa.x;
    if (f2_flip(fl, j)) { x = -1 * x; y = -1 * y; }
    n0[j] = x;
    n1[j] = y;
  }
  CompSumF rez[4];
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int sl = order_slot(code, k);
      const int o = comp(nb, sl);
      if ((o < 0) != (pass == 1)) continue;
      const float sg = f2_own(fl, sl) ? -1.f : 1.f;
      const float4 v = pick3(F[0], F[1], F[2], sl);
      rez[0].add(sg * v.x);
      rez[1].add(sg * v.y);
      rez[2].add(sg * v.z);
      rez[3].add(sg * v.w);
    }
  }
  // bathymetry source in FP64 (its Cramer solve cancels)
  const double hi = h_i, Zi = Z_i;
  double c_1 = 0., c_2 = 0., ss0[3], ss1[3], mata[3], matb[3], zv[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const bool neg = (fl >> (9 + j)) & 1u;
    ss0[j] = neg ? -1.0 * n0[j] : n0[j];
    ss1[j] = neg ? -1.0 * n1[j] : n1[j];
    double h_p1, z_p1;
    if (comp(nb, j) >= 0) {
      const int c = comp(fid, j);
      h_p1 = ld(s.q[0] + c);
      z_p1 = ld(s.q[4] + c);
    } else {
      h_p1 = hi;
      z_p1 = Zi;
    }
    zv[j] = z_p1;
    mata[j] = h_p1 * ss0[j];
    matb[j] = h_p1 * ss1[j];
    const double hm = 0.5 * (hi + h_p1);
    c_1 = c_1 + (hm * 0.5 * (hi + h_p1)) * ss0[j];
    c_2 = c_2 + (hm * 0.5 * (hi + h_p1)) * ss1[j];
  }
  const double c_3 = 3.0 * hi;
  const double delta = (mata[1] * matb[2] - mata[2] * matb[1]) - (mata[0] * matb[2] - matb[0] * mata[2]) +
                       (mata[0] * matb[1] - matb[0] * mata[1]);
  const double deltax = c_3 * (mata[1] * matb[2] - mata[2] * matb[1]) - (c_1 * matb[2] - c_2 * mata[2]) +
                        (c_1 * matb[1] - c_2 * mata[1]);
  const double deltay = (c_1 * matb[2] - c_2 * mata[2]) - c_3 * (mata[0] * matb[2] - matb[0] * mata[2]) +
                        (mata[0] * c_2 - matb[0] * c_1);
  const double deltaz = (mata[1] * c_2 - matb[1] * c_1) - (mata[0] * c_2 - matb[0] * c_1) +
                        c_3 * (mata[0] * matb[1] - matb[0] * mata[1]);
  const double rdelta = 1. / delta;
  const double h_1 = deltax * rdelta, h_2 = deltay * rdelta, h_3 = deltaz * rdelta;
  const double z_1 = Zi + hi - h_1, z_2 = Zi + hi - h_2, z_3 = Zi + hi - h_3;
  const double ns0x = (G.y - P1.y), ns0y = -(G.x - P1.x);
  const double ns1x = ns0x - ss0[1], ns1y = ns0y - ss1[1];
  const double ns2x = ns0x + ss0[0], ns2y = ns0y + ss1[0];
  const double s1x = 0.5 * h_1 * (zv[0] * ss0[0] + z_2 * ns0x - z_3 * ns2x);
  const double s1y = 0.5 * h_1 * (zv[0] * ss1[0] + z_2 * ns0y - z_3 * ns2y);
  const double s2x = 0.5 * h_2 * (zv[1] * ss0[1] - z_1 * ns0x + z_3 * ns1x);
  const double s2y = 0.5 * h_2 * (zv[1] * ss1[1] - z_1 * ns0y + z_3 * ns1y);
  const double s3x = 0.5 * h_3 * (zv[2] * ss0[2] + z_1 * ns2x - z_2 * ns1x);
  const double s3y = 0.5 * h_3 * (zv[2] * ss1[2] + z_1 * ns2y - z_2 * ns1y);
  const float shu = (float)(-grav * (s1x + s2x + s3x));
  const float shv = (float)(-grav * (s1y + s2y + s3y));
  const float k = (float)(dt / vol);
  const float h_n = sw_store(h_i, k * rez[0].value(), s.lo[0], out.lo[0], out.q[0], i);
  const float hu_n = sw_store(hu_i, k * (rez[1].value() + shu), s.lo[1], out.lo[1], out.q[1], i);
  const float hv_n = sw_store(hv_i, k * (rez[2].value() + shv), s.lo[2], out.lo[2], out.q[2], i);
  sw_store(hc_i, k * rez[3].value(), s.lo[3], out.lo[3], out.q[3], i);
  if (out.q[4] != s.q[4]) out.q[4][i] = Z_i;
  if (!want_dt) return 1e300;
  const double hn = h_n, un = hu_n / hn, vn = hv_n / hn;
  const double velson = sqrt(grav * hn);
  double lam = 0.;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double mes = sqrt(__dadd_rn(__dmul_rn(n0[j], n0[j]), __dmul_rn(n1[j], n1[j])));
    lam += (fabs(un * n0[j] + vn * n1[j]) / mes + velson) * mes;
  }
  return cfl * vol / lam;
}

#ifndef MB_SW2C_CELL_MIN_BLOCKS
#define MB_SW2C_CELL_MIN_BLOCKS 4
#endif
#ifndef MB_SW2C_BATCH_CELL_MIN_BLOCKS
#define MB_SW2C_BATCH_CELL_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(kBlock, MB_SW2C_CELL_MIN_BLOCKS) k_sw2c_cell(mb_mesh m, SWStateF s, SWOutF out, const float *ff,
                                                      const double *dt_cur, double *dt_next, double cfl,
                                                      double grav) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // every thread of the block reaches the dt reduction below (it synchronises the block)
  double best = 1e300;
  if (i < m.nbcells) best = sw2c_cell_body(m, s, out, ff, *dt_cur, dt_next != nullptr, cfl, grav, i);
  if (dt_next) {
    best = block_min(best);
    if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(dt_next, best);
  }
}

// batches: block b of a launch belongs to item map[b]; see mb_sw_item
__global__ void __launch_bounds__(kBlock) k_sw2c_batch_flux(const mb_sw_item *__restrict__ items,
                                                            const int32_t *__restrict__ map,
                                                            const int32_t *__restrict__ clock) {
  const mb_sw_item &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;
  const int par = (t - it.start_step) & 1;
  SWStateF s{{it.q[par][0], it.q[par][1], it.q[par][2], it.q[par][3], it.Z}, {}};
  sw2c_face(it.m, s, (float)it.grav, it.face_flux, it.dt + (par ^ 1),
            ((int)blockIdx.x - it.f_begin) * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(kBlock, MB_SW2C_BATCH_CELL_MIN_BLOCKS) k_sw2c_batch_cell(const mb_sw_item *__restrict__ items,
                                                            const int32_t *__restrict__ map,
                                                            const int32_t *__restrict__ clock) {
  const mb_sw_item &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;  // uniform over the block
  const int par = (t - it.start_step) & 1;
  SWStateF s{{it.q[par][0], it.q[par][1], it.q[par][2], it.q[par][3], it.Z},
             {it.lo[par][0], it.lo[par][1], it.lo[par][2], it.lo[par][3]}};
  SWOutF out{{it.q[par ^ 1][0], it.q[par ^ 1][1], it.q[par ^ 1][2], it.q[par ^ 1][3], const_cast<float *>(it.Z)},
             {it.lo[par ^ 1][0], it.lo[par ^ 1][1], it.lo[par ^ 1][2], it.lo[par ^ 1][3]}};
  const int i = ((int)blockIdx.x - it.c_begin) * blockDim.x + threadIdx.x;
  double best = 1e300;
  if (i < it.m.nbcells) best = sw2c_cell_body(it.m, s, out, it.face_flux, it.dt[par], true, it.cfl, it.grav, i);
  best = block_min(best);
  if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(it.dt + (par ^ 1), best);
}

}  // namespace

}  // namespace mb

using namespace mb;

extern "C" int mb_sw_step_f32c(const mb_mesh *m, const float *const q_in[5], float *const q_out[5],
                               const float *const lo_in[4], float *const lo_out[4], double cfl, double grav,
                               int32_t order, float *face_flux, const double *dt_cur, double *dt_next, void *stream) {
  MB_NVTX();
  return mb_sw_step_f32c_ex(m, q_in, q_out, lo_in, lo_out, cfl, grav, order, MB_WALLS_NEUMANN, face_flux, dt_cur,
                            dt_next, stream);
}

extern "C" int mb_sw_step_f32c_ex(const mb_mesh *m, const float *const q_in[5], float *const q_out[5],
                                  const float *const lo_in[4], float *const lo_out[4], double cfl, double grav,
                                  int32_t order, int32_t walls, float *face_flux, const double *dt_cur,
                                  double *dt_next, void *stream) {
  MB_NVTX();
  if (!m || m->dim != 2 || m->nlf != 3 || m->nbcells <= 0 || m->nbfaces <= 0) return MB_EINVAL;
  if (walls != MB_WALLS_NEUMANN && walls != MB_WALLS_REFLECT) return MB_EINVAL;
  if (!q_in || !q_out || !face_flux || !dt_cur || dt_next == dt_cur || order != 1) return MB_EINVAL;
  if (!m->cell_cellfid || !m->cell_vtx || !m->cell_nbr || !m->cell_flags || !m->node_coord || !m->cell_xy ||
      !m->cell_faces || !m->face_nm_f32)
    return MB_EINVAL;
  SWStateF s{};
  SWOutF out{};
  for (int k = 0; k < 5; ++k) {
    if (!q_in[k] || !q_out[k] || (k < 4 && q_in[k] == q_out[k])) return MB_EINVAL;
    s.q[k] = q_in[k];
    out.q[k] = q_out[k];
  }
  s.walls = walls;
  if ((lo_in == nullptr) != (lo_out == nullptr)) return MB_EINVAL;
  if (lo_in) {
    for (int k = 0; k < 4; ++k) {
      if (!lo_in[k] || !lo_out[k] || lo_in[k] == lo_out[k]) return MB_EINVAL;
      s.lo[k] = lo_in[k];
      out.lo[k] = lo_out[k];
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  k_sw2c_flux<<<ceil_div(m->nbfaces, kBlock), kBlock, 0, st>>>(*m, s, (float)grav, face_flux, dt_next);
  k_sw2c_cell<<<ceil_div(m->nbcells, kBlock), kBlock, 0, st>>>(*m, s, out, face_flux, dt_cur, dt_next, cfl, grav);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

extern "C" int mb_sw_batch_step_f32c(const mb_sw_item *items, const int32_t *face_map, int32_t face_blocks,
                                     const int32_t *cell_map, int32_t cell_blocks, int32_t *clock, void *stream) {
  MB_NVTX();
  if (!items || !face_map || !cell_map || !clock || face_blocks <= 0 || cell_blocks <= 0) return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  k_sw2c_batch_flux<<<face_blocks, kBlock, 0, st>>>(items, face_map, clock);
  k_sw2c_batch_cell<<<cell_blocks, kBlock, 0, st>>>(items, cell_map, clock);
  k_sw_clock_tick<<<1, 1, 0, st>>>(clock);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}
