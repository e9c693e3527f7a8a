// Advection-diffusion kernels: manapy's explicit scheme on triangles (DIM 2)
// and tetrahedra (DIM 3), FP64.
//
// Reference loops (manapy source tree):
//   cell gradient       manapy/ast/functions2d.py:5-104, functions3d.py:4-120
//   Barth limiter       manapy/ast/functions2d.py:280-325, functions3d.py:364-408
//   centre -> vertex    manapy/ast/functions2d.py:199-276, functions3d.py:251-362
//   face gradient       manapy/ast/functions2d.py:108-196, functions3d.py:122-248
//   upwind flux         manapy/solvers/advecdiff/fvm_utils.py:43-314
//   diamond diffusion   manapy/solvers/advecdiff/fvm_utils.py:5-26
//   time step           manapy/solvers/advecdiff/fvm_utils.py:317-340
//   update              manapy/solvers/advecdiff/fvm_utils.py:342-346
#include "fv_compact.cuh"

namespace mb {

// ---------------------------------------------------------------- per-cell pieces

// Unweighted least-squares gradient over the vertex neighbours, then the
// stencil's boundary ghosts, in manapy's order.
template <int DIM, class G>
__device__ __forceinline__ void lsq_gradient(const mb_mesh &m, const double *__restrict__ w, G ghost,
                                             int i, double &gx, double &gy, double &gz) {
  const double *cc = m.cell_center;
  const double cx = ld(cc + 3 * i), cy = ld(cc + 3 * i + 1);
  const double cz = DIM == 3 ? ld(cc + 3 * i + 2) : 0.0;
  const double wi = ld(w + i);
  double ixx = 0., iyy = 0., izz = 0., ixy = 0., ixz = 0., iyz = 0.;
  double jx = 0., jy = 0., jz = 0.;
  const int b = ld(m.cellnid_ptr + i), e = ld(m.cellnid_ptr + i + 1);
  for (int k = b; k < e; ++k) {
    const int c = ld(m.cellnid_idx + k);
    const double dx = ld(cc + 3 * c) - cx, dy = ld(cc + 3 * c + 1) - cy;
    const double dw = ld(w + c) - wi;
    ixx += dx * dx; iyy += dy * dy; ixy += (dx * dy);
    jx += (dx * dw); jy += (dy * dw);
    if (DIM == 3) {
      const double dz = ld(cc + 3 * c + 2) - cz;
      izz += dz * dz; ixz += (dx * dz); iyz += (dy * dz);
      jz += (dz * dw);
    }
  }
  const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
  const double *gc = m.face_ghostcenter;
  for (int k = gb; k < ge; ++k) {
    const int f = ld(m.ghostnid_idx + k);
    const double dx = ld(gc + 3 * f) - cx, dy = ld(gc + 3 * f + 1) - cy;
    const double dw = ghost(f) - wi;
    ixx += dx * dx; iyy += dy * dy; ixy += (dx * dy);
    jx += (dx * dw); jy += (dy * dw);
    if (DIM == 3) {
      const double dz = ld(gc + 3 * f + 2) - cz;
      izz += dz * dz; ixz += (dx * dz); iyz += (dy * dz);
      jz += (dz * dw);
    }
  }
  if (DIM == 2) {
    const double dia = ixx * iyy - ixy * ixy;
    gx = (iyy * jx - ixy * jy) / dia;
    gy = (ixx * jy - ixy * jx) / dia;
    gz = 0.;
  } else {
    const double dia = ixx * iyy * izz + 2. * ixy * ixz * iyz - ixx * (iyz * iyz) - iyy * (ixz * ixz)
                       - izz * (ixy * ixy);
    gx = ((iyy * izz - iyz * iyz) * jx + (ixz * iyz - ixy * izz) * jy + (ixy * iyz - ixz * iyy) * jz) / dia;
    gy = ((ixz * iyz - ixy * izz) * jx + (ixx * izz - ixz * ixz) * jy + (ixy * ixz - iyz * ixx) * jz) / dia;
    gz = ((ixy * iyz - ixz * iyy) * jx + (ixy * ixz - iyz * ixx) * jy + (ixx * iyy - ixy * ixy) * jz) / dia;
  }
}

// Barth-Jespersen limiter of cell i.
template <int DIM, class G>
__device__ __forceinline__ double barth(const mb_mesh &m, const double *__restrict__ w, G ghost,
                                        int i, double gx, double gy, double gz) {
  const int nlf = DIM == 2 ? 3 : 4;
  const double wi = ld(w + i);
  double wmax = wi, wmin = wi;
  int fs[4];
#pragma unroll
  for (int j = 0; j < nlf; ++j) {
    const int f = ld(m.cell_faces + 4 * i + j);
    fs[j] = f;
    const int nm = ld(m.face_name + f);
    const double a = ld(w + ld(m.face_cellid + 2 * f));
    const double b = (nm == 0 || nm > 10) ? ld(w + ld(m.face_cellid + 2 * f + 1)) : ghost(f);
    wmax = pmax(pmax(wmax, a), b);
    wmin = pmin(pmin(wmin, a), b);
  }
  const double eps = DIM == 2 ? 1e-8 : 1e-10;
  const double *cc = m.cell_center, *fc = m.face_center;
  const double cx = ld(cc + 3 * i), cy = ld(cc + 3 * i + 1);
  const double cz = DIM == 3 ? ld(cc + 3 * i + 2) : 0.0;
  double psi = 1.;
#pragma unroll
  for (int j = 0; j < nlf; ++j) {
    const int f = fs[j];
    const double r1 = ld(fc + 3 * f) - cx, r2 = ld(fc + 3 * f + 1) - cy;
    double delta = gx * r1 + gy * r2;
    if (DIM == 3) delta = gx * r1 + gy * r2 + gz * (ld(fc + 3 * f + 2) - cz);
    double psi_ij = 1.;
    if (!(fabs(delta) < eps)) {
      if (delta > 0.) psi_ij = pmin(1., (wmax - wi) / delta);
      if (delta < 0.) psi_ij = pmin(1., (wmin - wi) / delta);
    }
    psi = pmin(psi, psi_ij);
  }
  return psi;
}

// Centre -> vertex value of node n: cells, then ghosts, precomputed weights.
template <class G>
__device__ __forceinline__ double node_value(const mb_mesh &m, const double *__restrict__ w, G ghost, int n) {
  double acc = 0.;
  const int b = ld(m.n2c_ptr + n), e = ld(m.n2c_ptr + n + 1);
  for (int k = b; k < e; ++k) acc += ld(m.n2c_alpha + k) * ld(w + ld(m.n2c_idx + k));
  const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
  for (int k = gb; k < ge; ++k) acc += ld(m.n2g_alpha + k) * ghost(ld(m.n2g_idx + k));
  return acc;
}

// Diamond-cell face gradient of face f; vr = value on the right (cell or ghost).
template <int DIM>
__device__ __forceinline__ void face_gradient(const mb_mesh &m, const double *__restrict__ wn, int f,
                                              double vl, double vr, double &gx, double &gy, double &gz) {
  const int *nd = m.face_nodeid + 4 * f;
  if (DIM == 2) {
    const double vi1 = ld(wn + ld(nd)), vi2 = ld(wn + ld(nd + 1));
    const double *F = m.face_f + 8 * f;
    const double inv = 1 / (2 * ld(m.face_air + f));
    const double s1 = vi1 + vl, s2 = vl + vi2, s3 = vi2 + vr, s4 = vr + vi1;
    gx = inv * (s1 * ld(F + 1) + s2 * ld(F + 3) + s3 * ld(F + 5) + s4 * ld(F + 7));
    gy = -1 / (2 * ld(m.face_air + f)) * (s1 * ld(F + 0) + s2 * ld(F + 2) + s3 * ld(F + 4) + s4 * ld(F + 6));
    gz = 0.;
  } else {
    const double VA = ld(wn + ld(nd)), VB = ld(wn + ld(nd + 1)), VC = ld(wn + ld(nd + 2));
    const double VD = VC;  // tetrahedra: the fourth face node is the third
    const double *F = m.face_f + 6 * f;
    const double *N = m.face_normal + 3 * f;
    const double a = ld(m.face_air + f);
    const double dAC = VA - VC, dBD = VB - VD, dRL = vr - vl;
    gx = (ld(F + 0) * dAC + ld(F + 3) * dBD + ld(N + 0) * dRL) / a;
    gy = (ld(F + 1) * dAC + ld(F + 4) * dBD + ld(N + 1) * dRL) / a;
    gz = (ld(F + 2) * dAC + ld(F + 5) * dBD + ld(N + 2) * dRL) / a;
  }
}

// Linear reconstruction at face f from cell c (order 2), 2D uses x, y only.
template <int DIM>
__device__ __forceinline__ double reconstruct(const mb_mesh &m, const double *__restrict__ w,
                                              const double *__restrict__ gx, const double *__restrict__ gy,
                                              const double *__restrict__ gz, const double *__restrict__ psi,
                                              int c, int f) {
  const double *cc = m.cell_center + 3 * c, *fc = m.face_center + 3 * f;
  double d = ld(gx + c) * (ld(fc) - ld(cc)) + ld(gy + c) * (ld(fc + 1) - ld(cc + 1));
  if (DIM == 3)
    d = ld(gx + c) * (ld(fc) - ld(cc)) + ld(gy + c) * (ld(fc + 1) - ld(cc + 1)) + ld(gz + c) * (ld(fc + 2) - ld(cc + 2));
  return ld(w + c) + ld(psi + c) * d;
}

// ---------------------------------------------------------------- kernels: reference entry points

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_cell_gradient(mb_mesh m, const double *w, const double *ghost,
                                                          double *gx, double *gy, double *gz) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double x, y, z;
    lsq_gradient<DIM>(m, w, GhostArray{ghost}, i, x, y, z);
    gx[i] = x; gy[i] = y; gz[i] = z;
  }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_barth(mb_mesh m, const double *w, const double *ghost,
                                                  const double *gx, const double *gy, const double *gz,
                                                  double *psi) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x)
    psi[i] = barth<DIM>(m, w, GhostArray{ghost}, i, ld(gx + i), ld(gy + i), DIM == 3 ? ld(gz + i) : 0.0);
}

__global__ void __launch_bounds__(kBlock) k_centertovertex(mb_mesh m, const double *w, const double *ghost,
                                                           double *wn) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.nbnodes; n += gridDim.x * blockDim.x)
    wn[n] = node_value(m, w, GhostArray{ghost}, n);
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_face_gradient(mb_mesh m, const uint8_t *on, const double *w,
                                                          const double *ghost, const double *wn,
                                                          double *gfx, double *gfy, double *gfz) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nbfaces; f += gridDim.x * blockDim.x) {
    if (!on[f]) continue;
    const int c0 = ld(m.face_cellid + 2 * f), c1 = ld(m.face_cellid + 2 * f + 1);
    const double vl = ld(w + c0), vr = c1 >= 0 ? ld(w + c1) : ld(ghost + f);
    double x, y, z;
    face_gradient<DIM>(m, wn, f, vl, vr, x, y, z);
    gfx[f] = x; gfy[f] = y;
    if (DIM == 3) gfz[f] = z;
  }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_convective(mb_mesh m, double *rez, const double *w,
                                                       const double *ghost, const double *uf,
                                                       const double *vf, const double *wf,
                                                       const double *gx, const double *gy,
                                                       const double *gz, const double *psi, int order) {
  const int nlf = DIM == 2 ? 3 : 4;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double cv[4];
    bool bnd[4];
#pragma unroll
    for (int j = 0; j < nlf; ++j) {
      const int f = ld(m.cell_faces + 4 * i + j);
      const int c0 = ld(m.face_cellid + 2 * f), c1 = ld(m.face_cellid + 2 * f + 1);
      const double *N = m.face_normal + 3 * f;
      const double s = ld(uf + f) * ld(N) + ld(vf + f) * ld(N + 1) + ld(wf + f) * ld(N + 2);
      double sol;
      if (s >= 0) sol = order == 2 ? reconstruct<DIM>(m, w, gx, gy, gz, psi, c0, f) : ld(w + c0);
      else if (c1 < 0) sol = ld(ghost + f);
      else sol = order == 2 ? reconstruct<DIM>(m, w, gx, gy, gz, psi, c1, f) : ld(w + c1);
      const double F = s * sol;
      cv[j] = (i == c0) ? -F : F;
      bnd[j] = c1 < 0;
    }
    const uint8_t code = ld(m.cell_order + i);
    double acc = 0.;
#pragma unroll
    for (int k = 0; k < nlf; ++k) {
      const int s = order_slot(code, k);
      if (!bnd[s]) acc += cv[s];
    }
#pragma unroll
    for (int k = 0; k < nlf; ++k) {
      const int s = order_slot(code, k);
      if (bnd[s]) acc += cv[s];
    }
    rez[i] = acc;
  }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock) k_dissipative(mb_mesh m, const double *gfx, const double *gfy,
                                                        const double *gfz, double *dis, double Dxx,
                                                        double Dyy, double Dzz) {
  const int nlf = DIM == 2 ? 3 : 4;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double q[4];
#pragma unroll
    for (int j = 0; j < nlf; ++j) {
      const int f = ld(m.cell_faces + 4 * i + j);
      const double *N = m.face_normal + 3 * f;
      const double v = Dxx * ld(gfx + f) * ld(N) + Dyy * ld(gfy + f) * ld(N + 1) + Dzz * ld(gfz + f) * ld(N + 2);
      const int c0 = ld(m.face_cellid + 2 * f);
      q[j] = (i == c0) ? v : -v;
    }
    const uint8_t code = ld(m.cell_order + i);
    double acc = 0.;
#pragma unroll
    for (int k = 0; k < nlf; ++k) acc += q[order_slot(code, k)];
    dis[i] = acc;
  }
}

__global__ void __launch_bounds__(kBlock) k_facetocell(mb_mesh m, const double *uf, double *uc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double acc = 0.;
    for (int j = 0; j < m.nlf; ++j) acc += ld(uf + ld(m.cell_faces + 4 * i + j));
    uc[i] = acc / m.nlf;
  }
}

__global__ void __launch_bounds__(kBlock) k_ghost(mb_mesh m, mb_bc bc, const double *w, double *ghost) {
  const GhostRule g = make_rule(m, bc, w);
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nbfaces; f += gridDim.x * blockDim.x)
    if (bc.kind[f] != MB_G_NONE) ghost[f] = g(f);
}

__global__ void k_fill(double *p, double v) { *p = v; }

__global__ void __launch_bounds__(kBlock) k_time_step(mb_mesh m, const double *u, const double *v,
                                                      const double *w, double cfl, double Dxx, double Dyy,
                                                      double Dzz, double *dt) {
  double best = 1e300;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    const double vol = ld(m.cell_volume + i);
    const double ui = ld(u + i), vi = ld(v + i), wi = ld(w + i);
    double lam = 0.;
    for (int j = 0; j < m.nlf; ++j) {
      const double *N = m.face_normal + 3 * ld(m.cell_faces + 4 * i + j);
      const double n0 = ld(N), n1 = ld(N + 1), n2 = ld(N + 2);
      lam += fabs(ui * n0 + vi * n1 + wi * n2);
      const double mes = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
      const double lam_diff = Dxx * (mes * mes) + Dyy * (mes * mes) + Dzz * (mes * mes);
      lam += lam_diff / vol;
    }
    if (lam != 0) best = pmin(best, cfl * vol / lam);
  }
  best = block_min(best);
  if (threadIdx.x == 0 && best < 1e300) atomic_min_pos(dt, best);
}

__global__ void __launch_bounds__(kBlock) k_update(int n, double *wc, const double *rez, const double *dis,
                                                   const double *src, const double *dt_dev,
                                                   const double *vol) {
  const double dt = *dt_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    wc[i] += dt * ((ld(rez + i) + ld(dis + i)) / ld(vol + i) + ld(src + i));
}

__global__ void __launch_bounds__(kBlock) k_cell_face_sign(mb_mesh m, const double *uf, const double *vf,
                                                           const double *wf, double *s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    for (int j = 0; j < 4; ++j) {
      double v = 0.;
      if (j < m.nlf) {
        const int f = ld(m.cell_faces + 4 * i + j);
        const double *N = m.face_normal + 3 * f;
        v = ld(uf + f) * ld(N) + ld(vf + f) * ld(N + 1) + ld(wf + f) * ld(N + 2);
      }
      s[4 * i + j] = v;
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_face_sign(mb_mesh m, const double *uf, const double *vf,
                                                      const double *wf, double *s) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nbfaces; f += gridDim.x * blockDim.x) {
    const double *N = m.face_normal + 3 * f;
    s[f] = ld(uf + f) * ld(N) + ld(vf + f) * ld(N + 1) + ld(wf + f) * ld(N + 2);
  }
}

// ---------------------------------------------------------------- kernels: fused step

// Phase 1: blocks [0, ncb) do cell gradients + limiter, blocks [ncb, ...) do node values.
template <int DIM, bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock) k_step_phase1(mb_mesh m, mb_bc bc, const double *w, double *gx,
                                                        double *gy, double *gz, double *psi, double *wn,
                                                        int ncb) {
  const GhostRule ghost = make_rule(m, bc, w);
  if (ORDER2 && (int)blockIdx.x < ncb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nbcells) return;
    double x, y, z;
    lsq_gradient<DIM>(m, w, ghost, i, x, y, z);
    gx[i] = x; gy[i] = y;
    if (DIM == 3) gz[i] = z;
    psi[i] = barth<DIM>(m, w, ghost, i, x, y, z);
    return;
  }
  if (DIFF) {
    const int n = (blockIdx.x - (ORDER2 ? ncb : 0)) * blockDim.x + threadIdx.x;
    if (n >= m.nbnodes) return;
    wn[n] = node_value(m, w, ghost, n);
  }
}

// Phase 2: per cell, upwind + diamond fluxes over its faces and the update.
template <int DIM, bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock) k_step_phase2(mb_mesh m, mb_bc bc, mb_advdiff_params p,
                                                        const double *w, double *w_out, const double *sign,
                                                        const double *src, const double *dt_dev,
                                                        const double *gx, const double *gy, const double *gz,
                                                        const double *psi, const double *wn) {
  const int nlf = DIM == 2 ? 3 : 4;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const GhostRule ghost = make_rule(m, bc, w);
  const double wi = ld(w + i);
  double cv[4], q[4];
  bool bnd[4];
#pragma unroll
  for (int j = 0; j < nlf; ++j) {
    const int f = ld(m.cell_faces + 4 * i + j);
    const int c0 = ld(m.face_cellid + 2 * f), c1 = ld(m.face_cellid + 2 * f + 1);
    const bool own = (i == c0);
    const int other = own ? c1 : c0;
    const bool b = c1 < 0;
    const double vo = b ? ghost(f) : ld(w + other);  // unreconstructed value across the face
    // upwind flux of face f in manapy's orientation (left = c0)
    const double s = ld(sign + 4 * i + j);
    double sol;
    if (s >= 0) {
      // left state
      if (ORDER2) sol = reconstruct<DIM>(m, w, gx, gy, gz, psi, c0, f);
      else sol = own ? wi : vo;
    } else {
      if (b) sol = vo;
      else if (ORDER2) sol = reconstruct<DIM>(m, w, gx, gy, gz, psi, c1, f);
      else sol = own ? vo : wi;
    }
    const double F = s * sol;
    cv[j] = own ? -F : F;
    bnd[j] = b;
    if (DIFF) {
      double v = 0.;
      if (ld(bc.face_grad_on + f)) {
        const double vl = own ? wi : vo;
        const double vr = own ? vo : wi;
        double fx, fy, fz;
        face_gradient<DIM>(m, wn, f, vl, vr, fx, fy, fz);
        const double *N = m.face_normal + 3 * f;
        v = p.Dxx * fx * ld(N) + p.Dyy * fy * ld(N + 1) + p.Dzz * fz * ld(N + 2);
      }
      q[j] = own ? v : -v;
    }
  }
  const uint8_t code = ld(m.cell_order + i);
  double rez = 0.;
#pragma unroll
  for (int k = 0; k < nlf; ++k) {
    const int s = order_slot(code, k);
    if (!bnd[s]) rez += cv[s];
  }
#pragma unroll
  for (int k = 0; k < nlf; ++k) {
    const int s = order_slot(code, k);
    if (bnd[s]) rez += cv[s];
  }
  double dis = 0.;
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < nlf; ++k) dis += q[order_slot(code, k)];
  }
  const double dt = *dt_dev;
  const double sc = src ? ld(src + i) : 0.0;
  w_out[i] = wi + dt * ((rez + dis) / ld(m.cell_volume + i) + sc);
}

// ---------------------------------------------------------------- fused step, compact 2D layout
//
// Per cell: its three vertices (manapy's local order), the neighbour across
// each local face (or -1-f for boundary face f), three orientation bits per
// face and the upwind sign u.n of each face.  Face normals, centres, diamond
// vectors and areas are recomputed from the vertex coordinates with manapy's
// expressions: the subtractions are exact, so normals and face centres are the
// same numbers manapy stores.
//
// Neighbour lists (LSQ stencil, node -> cells) are stored SELL-32: for each
// group of 32 consecutive rows (one warp), entry k of every row sits in one
// 128-byte segment, so a warp reads its k-th neighbours with one coalesced
// load; rows are padded with -1 to the group's longest row.  Entries keep
// manapy's order.
//
// Phase 1 writes a packed record {w, gx, gy, psi} per cell, so phase 2 fetches
// everything it needs from a neighbour with two 16-byte loads.


#ifndef MB_P1_MIN_BLOCKS
#define MB_P1_MIN_BLOCKS 6
#endif
#ifndef MB_F2_LSQ_BATCH
#define MB_F2_LSQ_BATCH 4
#endif
#ifndef MB_P1_BLOCK
#define MB_P1_BLOCK kBlock
#endif

// block `bid` of phase 1: blocks [0, ncb) gradient + limiter records, the rest node values
// ROWS: the least-squares neighbours are read from rows {x, y, w, 0} of the step's input
// (one 256-bit load each) instead of the centre table and the state (two loads)
template <bool ORDER2, bool DIFF, bool ROWS = false>
__device__ __forceinline__ void f2_phase1(const mb_mesh &m, const mb_bc &bc, const double *__restrict__ w,
                                          double *__restrict__ rec, double *__restrict__ wn, int ncb, int bid,
                                          const double *__restrict__ rows = nullptr) {
  const GhostRule ghost = make_rule(m, bc, w);
  const int lane = threadIdx.x & 31;
  if (ORDER2 && bid < ncb) {
    const int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.nbcells) return;
    double2 c;
    double wi;
    if (ROWS) {
      double pad;
      ld4d(rows + 4 * (long long)i, c.x, c.y, wi, pad);
    } else {
      c = ldd2(m.cell_xy + 2 * i);
      wi = ld(w + i);
    }
    // least-squares gradient: vertex neighbours (SELL-32), then stencil ghosts
    // every row of the warp runs to the group length (a uniform trip count keeps
    // several gathers in flight); a padding entry points at the cell itself,
    // whose terms are exact zeros
    double ixx = 0., iyy = 0., ixy = 0., jx = 0., jy = 0.;
    const int sb = ld(m.lsq_sell_ptr + (i >> 5)), se = ld(m.lsq_sell_ptr + (i >> 5) + 1);
    const int L = (se - sb) >> 5;
    const int32_t *ix = m.lsq_sell_idx + sb + lane;
    const uint64_t pst = l2_stream();
    int k = 0;
    // batches of MB_F2_LSQ_BATCH: the index loads, then twice as many gathers in flight,
    // then the terms accumulated in manapy's order
    for (; k + MB_F2_LSQ_BATCH <= L; k += MB_F2_LSQ_BATCH) {
      int cc[MB_F2_LSQ_BATCH];
#pragma unroll
      for (int u = 0; u < MB_F2_LSQ_BATCH; ++u) cc[u] = ld1_stream(ix + 32 * (k + u), pst);
      double2 pc[MB_F2_LSQ_BATCH];
      double wc[MB_F2_LSQ_BATCH];
#pragma unroll
      for (int u = 0; u < MB_F2_LSQ_BATCH; ++u) {
        if (cc[u] < 0) {            // padding: the cell itself, no gather issued
          pc[u] = c;
          wc[u] = wi;
        } else if (ROWS) {
          double pad;
          ld4d(rows + 4 * (long long)cc[u], pc[u].x, pc[u].y, wc[u], pad);
        } else {
          pc[u] = ldd2(m.cell_xy + 2 * cc[u]);
          wc[u] = ld(w + cc[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < MB_F2_LSQ_BATCH; ++u) {
        const double dx = pc[u].x - c.x, dy = pc[u].y - c.y, dw = wc[u] - wi;
        ixx += dx * dx; iyy += dy * dy; ixy += (dx * dy);
        jx += (dx * dw); jy += (dy * dw);
      }
    }
    for (; k < L; ++k) {
      const int cc = ld1_stream(ix + 32 * k, pst);
      double2 pc;
      double wcc;
      if (cc < 0) {
        pc = c;
        wcc = wi;
      } else if (ROWS) {
        double pad;
        ld4d(rows + 4 * (long long)cc, pc.x, pc.y, wcc, pad);
      } else {
        pc = ldd2(m.cell_xy + 2 * cc);
        wcc = ld(w + cc);
      }
      const double dx = pc.x - c.x, dy = pc.y - c.y, dw = wcc - wi;
      ixx += dx * dx; iyy += dy * dy; ixy += (dx * dy);
      jx += (dx * dw); jy += (dy * dw);
    }
    const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
    for (int k = gb; k < ge; ++k) {
      const int f = ld(m.ghostnid_idx + k);
      const double dx = ld(m.face_ghostcenter + 3 * f) - c.x, dy = ld(m.face_ghostcenter + 3 * f + 1) - c.y;
      const double dw = ghost(f) - wi;
      ixx += dx * dx; iyy += dy * dy; ixy += (dx * dy);
      jx += (dx * dw); jy += (dy * dw);
    }
    const double dia = ixx * iyy - ixy * ixy;
    const double x = (iyy * jx - ixy * jy) / dia;
    const double y = (ixx * jy - ixy * jx) / dia;
    // Barth limiter over the three faces
    const int4 vt = ld4(m.cell_vtx + 4 * i);
    const int4 nb = ld4(m.cell_nbr + 4 * i);
    const double2 P0 = ldd2(m.node_coord + 2 * vt.x), P1 = ldd2(m.node_coord + 2 * vt.y),
                  P2 = ldd2(m.node_coord + 2 * vt.z);
    double wmax = wi, wmin = wi;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int o = comp(nb, j);
      const double b = o < 0 ? ghost(-1 - o) : ld(w + o);
      wmax = pmax(wmax, b);
      wmin = pmin(wmin, b);
    }
    double ps = 1.;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double2 a = j == 0 ? P0 : (j == 1 ? P1 : P2), b = j == 0 ? P1 : (j == 1 ? P2 : P0);
      const double r1 = 0.5 * (a.x + b.x) - c.x, r2 = 0.5 * (a.y + b.y) - c.y;
      const double delta = x * r1 + y * r2;
      double psi_ij = 1.;
      if (!(fabs(delta) < 1e-8)) {
        if (delta > 0.) psi_ij = pmin(1., (wmax - wi) / delta);
        if (delta < 0.) psi_ij = pmin(1., (wmin - wi) / delta);
      }
      ps = pmin(ps, psi_ij);
    }
    const uint64_t keep = l2_keep();
#if MB_V4_IO
    st4_keep(rec + 4 * i, wi, x, y, ps, keep);
#else
    st2_keep(rec + 4 * i, wi, x, keep);
    st2_keep(rec + 4 * i + 2, y, ps, keep);
#endif
    return;
  }
  if (DIFF) {
    const int n = (bid - (ORDER2 ? ncb : 0)) * blockDim.x + threadIdx.x;
    if (n >= m.nbnodes) return;
    double acc = 0.;
    const int sb = ld(m.n2c_sell_ptr + (n >> 5)), se = ld(m.n2c_sell_ptr + (n >> 5) + 1);
    const uint64_t pst = l2_stream();
#pragma unroll 4
    for (int k = sb + lane; k < se; k += 32) {
      // padding repeats the row's first cell with weight 0: an exact zero term
      const int cc = ld1_stream(m.n2c_sell_idx + k, pst);
      acc += ldd_stream(m.n2c_sell_alpha + k, pst) * ld(w + cc);
    }
    const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
    for (int k = gb; k < ge; ++k) acc += ld(m.n2g_alpha + k) * ghost(ld(m.n2g_idx + k));
    st1_keep(wn + n, acc, l2_keep());
  }
}

// Launch shapes of the fused phases: variant v of a kernel runs blocks of kP*B[v] threads
// with launch bounds for kP*M[v] resident blocks per SM.  Variant 0 is the measured default;
// the others are selected per mesh (mb_mesh.variant, picked by the autotuner) for second
// order with diffusion.
constexpr int kP1B[4] = {MB_P1_BLOCK, 128, 256, 512};
constexpr int kP1M[4] = {MB_P1_MIN_BLOCKS, 12, 4, 3};

template <bool ORDER2, bool DIFF, bool ROWS, int VAR>
__global__ void __launch_bounds__(kP1B[VAR], kP1M[VAR]) k_f2_phase1(mb_mesh m, mb_bc bc, const double *__restrict__ w,
                                                      double *__restrict__ rec, double *__restrict__ wn, int ncb,
                                                      const double *__restrict__ rows) {
  f2_phase1<ORDER2, DIFF, ROWS>(m, bc, w, rec, wn, ncb, blockIdx.x, rows);
}

#ifndef MB_P2_MIN_BLOCKS
#define MB_P2_MIN_BLOCKS 7
#endif
#ifndef MB_P2_BLOCK
#define MB_P2_BLOCK 128
#endif

// block `bid` of phase 2: fluxes and update of its cells
// WROWS: also write the rows {x, y, w_out, 0} of the result (the next step's ROWS input)
template <bool ORDER2, bool DIFF, bool WROWS = false>
__device__ __forceinline__ void f2_phase2(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p,
                                          const double *__restrict__ w, double *__restrict__ w_out,
                                          const double *__restrict__ sign, const double *__restrict__ src,
                                          const double *__restrict__ dt_dev, const double *__restrict__ rec,
                                          const double *__restrict__ wn, int bid,
                                          double *__restrict__ rows_out = nullptr, int c0 = 0, int c1 = -1) {
  // cells [c0, c1) (c1 < 0: to the last cell)
  const int i = c0 + bid * blockDim.x + threadIdx.x;
  if (i >= (c1 < 0 ? m.nbcells : c1)) return;
  const GhostRule ghost = make_rule(m, bc, w);
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const double2 P0 = ldd2(m.node_coord + 2 * vt.x), P1 = ldd2(m.node_coord + 2 * vt.y),
                P2 = ldd2(m.node_coord + 2 * vt.z);
  const double2 ci = ldd2(m.cell_xy + 2 * i);
  const uint64_t pst = l2_stream();
#if MB_V4_IO
  double2 s01;
  double s2, s_pad;
  ld4d_stream(sign + 4 * i, s01.x, s01.y, s2, s_pad, pst);
#else
  const double2 s01 = ldd2_stream(sign + 4 * i, pst);
  const double s2 = ldd_stream(sign + 4 * i + 2, pst);
#endif
  double wi, gxi = 0., gyi = 0., psii = 0.;
  if (ORDER2) {
    ld4d(rec + 4 * i, wi, gxi, gyi, psii);
  } else {
    wi = ld(w + i);
  }
  double cv[3], q[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int o = comp(nb, j);
    const bool b = o < 0;
    const int f = -1 - o;
    const bool own = f2_own(fl, j);
    const bool rev = f2_rev(fl, j);
    const double2 Pj = j == 0 ? P0 : (j == 1 ? P1 : P2), Pk = j == 0 ? P1 : (j == 1 ? P2 : P0);
    const double2 Xa = rev ? Pk : Pj;   // faces.nodeid[f][0]
    const double2 Xb = rev ? Pj : Pk;   // faces.nodeid[f][1]
    const double fcx = 0.5 * (Xa.x + Xb.x), fcy = 0.5 * (Xa.y + Xb.y);
    double vo, gxo = 0., gyo = 0., pso = 0.;
    double2 co;
    if (b) {
      vo = ghost(f);
      co = make_double2(ld(m.face_ghostcenter + 3 * f), ld(m.face_ghostcenter + 3 * f + 1));
    } else {
      if (ORDER2) {
        ld4d(rec + 4 * o, vo, gxo, gyo, pso);
      } else {
        vo = ld(w + o);
      }
      co = ldd2(m.cell_xy + 2 * o);
    }
    // upwind flux of the face in manapy's orientation (left = faces.cellid[f][0])
    const double s = j == 0 ? s01.x : (j == 1 ? s01.y : s2);
    const bool take_me = (s >= 0) == own;
    double sol;
    if (take_me) {
      sol = ORDER2 ? wi + psii * (gxi * (fcx - ci.x) + gyi * (fcy - ci.y)) : wi;
    } else if (b) {
      sol = vo;  // boundary ghost, never reconstructed
    } else {
      sol = ORDER2 ? vo + pso * (gxo * (fcx - co.x) + gyo * (fcy - co.y)) : vo;
    }
    const double F = s * sol;
    cv[j] = own ? -F : F;
    if (DIFF) {
      double v = 0.;
      if (!b || ld(bc.face_grad_on + f)) {
        const double2 v1 = own ? ci : co, v2 = own ? co : ci;   // centres of cellid[f][0], [1]
        const double vl = own ? wi : vo, vr = own ? vo : wi;
        const double air = 0.5 * ((Xb.x - Xa.x) * (v2.y - v1.y) + (v1.x - v2.x) * (Xb.y - Xa.y));
        const int ia = rev ? comp(vt, (j + 1) % 3) : comp(vt, j);
        const int ib = rev ? comp(vt, j) : comp(vt, (j + 1) % 3);
        const double vi1 = ld(wn + ia), vi2 = ld(wn + ib);
        // manapy's diamond gradient (manapy/ast/functions2d.py:108-196, face_gradient_2d) sums
        // (V_i1 + V_L) f_1 + (V_L + V_i2) f_2 + (V_i2 + V_R) f_3 + (V_R + V_i1) f_4 with
        // f_1 = v1 - Xa, f_2 = Xb - v1, f_3 = v2 - Xb, f_4 = Xa - v2; grouped by value, the
        // same sum is (V_i1 - V_i2) (v1 - v2) + (V_L - V_R) (Xb - Xa) (equal up to rounding)
        const double dab = vi1 - vi2, dlr = vl - vr;
        const double sx = dab * (v1.x - v2.x) + dlr * (Xb.x - Xa.x);
        const double sy = dab * (v1.y - v2.y) + dlr * (Xb.y - Xa.y);
        // -1 / (2 air) is exactly -(1 / (2 air)): one division serves both components
        const double rda = 1 / (2 * air);
        const double fgx = rda * sy;
        const double fgy = -rda * sx;
        double n0 = Xa.y - Xb.y, n1 = Xb.x - Xa.x;
        if (f2_flip(fl, j)) { n0 = -1 * n0; n1 = -1 * n1; }
        v = p.Dxx * fgx * n0 + p.Dyy * fgy * n1;
      }
      q[j] = own ? v : -v;
    }
  }
  // manapy's accumulation order, with register selects instead of indexed arrays
  const uint8_t code = ld(m.cell_order + i);
  double rez = 0.;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int sl = order_slot(code, k);
    if (pick3(nb.x, nb.y, nb.z, sl) >= 0) rez += pick3(cv[0], cv[1], cv[2], sl);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int sl = order_slot(code, k);
    if (pick3(nb.x, nb.y, nb.z, sl) < 0) rez += pick3(cv[0], cv[1], cv[2], sl);
  }
  double dis = 0.;
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 3; ++k) dis += pick3(q[0], q[1], q[2], order_slot(code, k));
  }
  const double dt = *dt_dev;
  const double sc = src ? ld(src + i) : 0.0;
  const double wnew = wi + dt * ((rez + dis) / ld(m.cell_volume + i) + sc);
  w_out[i] = wnew;
  if (WROWS) st4d_plain(rows_out + 4 * (long long)i, ci.x, ci.y, wnew, 0.0);
}

constexpr int kP2B[4] = {MB_P2_BLOCK, 256, 64, 128};
constexpr int kP2M[4] = {MB_P2_MIN_BLOCKS, 3, 14, 8};

template <bool ORDER2, bool DIFF, bool WROWS, int VAR>
__global__ void __launch_bounds__(kP2B[VAR], kP2M[VAR]) k_f2_phase2(mb_mesh m, mb_bc bc, mb_advdiff_params p,
                                                         const double *__restrict__ w, double *__restrict__ w_out,
                                                         const double *__restrict__ sign,
                                                         const double *__restrict__ src,
                                                         const double *__restrict__ dt_dev,
                                                         const double *__restrict__ rec,
                                                         const double *__restrict__ wn,
                                                         double *__restrict__ rows_out, int c0, int c1) {
  f2_phase2<ORDER2, DIFF, WROWS>(m, bc, p, w, w_out, sign, src, dt_dev, rec, wn, blockIdx.x, rows_out, c0, c1);
}

// ---------------------------------------------------------------- batches of triangle meshes, FP64
//
// Block b of a launch belongs to item map[b] (blocks never straddle two meshes) and runs
// the single-mesh block body above on that item's tables, so each item computes exactly
// what mb_advdiff_step computes for it alone.  The batch clock selects each item's
// ping-pong state and skips items outside their [start_step, end_step) window.

#ifndef MB_P2_BATCH_MIN_BLOCKS
#define MB_P2_BATCH_MIN_BLOCKS 4
#endif
#ifndef MB_P1_BATCH_MIN_BLOCKS
#define MB_P1_BATCH_MIN_BLOCKS MB_P1_MIN_BLOCKS
#endif

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock, MB_P1_BATCH_MIN_BLOCKS)
    k_f2_batch_phase1(const mb_advdiff_item_f64 *__restrict__ items, const int32_t *__restrict__ map,
                      const int32_t *__restrict__ clock) {
  const mb_advdiff_item_f64 &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;
  f2_phase1<ORDER2, DIFF>(it.m, it.bc, it.w[(t - it.start_step) & 1], it.cell_scratch, it.node_scratch,
                          it.p1_cell_blocks, (int)blockIdx.x - it.p1_begin);
}

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock, MB_P2_BATCH_MIN_BLOCKS)
    k_f2_batch_phase2(const mb_advdiff_item_f64 *__restrict__ items, const int32_t *__restrict__ map,
                      const int32_t *__restrict__ clock) {
  const mb_advdiff_item_f64 &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (t < it.start_step || t >= it.end_step) return;
  const int par = (t - it.start_step) & 1;
  f2_phase2<ORDER2, DIFF>(it.m, it.bc, it.p, it.w[par], it.w[par ^ 1], it.sign_cf, it.src, it.dt_dev,
                          it.cell_scratch, it.node_scratch, (int)blockIdx.x - it.p2_begin);
}

__global__ void k_batch_tick(int32_t *clock) { *clock += 1; }

// ---------------------------------------------------------------- fused step, compact 3D layout
//
// Tetrahedra.  Local face j of a cell is (v0,v1,v2), (v2,v3,v0), (v0,v1,v3),
// (v3,v1,v2) (manapy/ddm/ddm_utils3d.py:785-791).  cell_flags holds six bits per
// face at bit 6j: bit 0 the cell is faces.cellid[f][0]; bits 1-3 the permutation
// taking the local face's vertices to manapy's descending node order (which fixes
// the face centre and the stored normal); bit 4 manapy's orientation swap of the
// last two nodes (the order of the diamond vectors); bit 5 the stored normal is
// minus 0.5 (v_d1 - v_d0) x (v_d2 - v_d0).  Node coordinates and cell centres
// are stored [n][4].  Cell scratch [8][nbcells]: the phase-1 records {w, psi gx,
// psi gy, psi gz} ([n][4], the limiter folded into the gradient), then the pack
// pass's rows {x, y, z, w} ([n][4]) from which the least-squares stencil reads
// each neighbour's centre and value with one 256-bit load.


#ifndef MB_P1_3D_MIN_BLOCKS
#define MB_P1_3D_MIN_BLOCKS 4
#endif
#ifndef MB_F3_LSQ_BATCH
#define MB_F3_LSQ_BATCH 4
#endif

// Pack pass: rows of every cell with its centre and value in one 32-byte row ({x, y, w, 0}
// for triangles, {x, y, z, w} for tetrahedra), so that the least-squares stencil gathers
// one row per neighbour.
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_pack_rows(mb_mesh m, const double *__restrict__ w, double *__restrict__ rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  if (DIM == 2) {
    const double2 c = ldd2(m.cell_xy + 2 * i);
    st4_keep(rows + 4 * (long long)i, c.x, c.y, ld(w + i), 0.0, l2_keep());
  } else {
    double x, y, z, pad;
    ld4d_stream(m.cell_xy + 4 * (long long)i, x, y, z, pad, l2_stream());
    st4_keep(rows + 4 * (long long)i, x, y, z, ld(w + i), l2_keep());
  }
}

// one row {x, y, z, w} (written by the previous launch, read-only in phase 1)
__device__ __forceinline__ void ld_row(const double *p, double &x, double &y, double &z, double &w) {
  ld4d(p, x, y, z, w);
}

constexpr int kQ1B[4] = {kBlock, 128, 256, 128};
constexpr int kQ1M[4] = {MB_P1_3D_MIN_BLOCKS, 8, 3, 6};

template <bool ORDER2, bool DIFF, int VAR, bool PRE = false>
__global__ void __launch_bounds__(kQ1B[VAR], kQ1M[VAR]) k_f3_phase1(mb_mesh m, mb_bc bc, const double *__restrict__ w,
                                                                        double *__restrict__ rec,
                                                                        const double *__restrict__ rows,
                                                                        double *__restrict__ wn, int ncb) {
  const GhostRule ghost = make_rule(m, bc, w);
  const int lane = threadIdx.x & 31;
  if (ORDER2 && (int)blockIdx.x < ncb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nbcells) return;
    D3 c;
    double wi;
    ld_row(rows + 4 * (long long)i, c.x, c.y, c.z, wi);
    double ixx = 0., iyy = 0., izz = 0., ixy = 0., ixz = 0., iyz = 0., jx = 0., jy = 0., jz = 0.;
    const int sb = ld(m.lsq_sell_ptr + (i >> 5)), se = ld(m.lsq_sell_ptr + (i >> 5) + 1);
    const int L = (se - sb) >> 5;
    const int32_t *ix = m.lsq_sell_idx + sb + lane;
    const uint64_t pst = l2_stream();
    int k = 0;
    // batches of MB_F3_LSQ_BATCH neighbours: the next batch's indices are loaded before this
    // batch's row gathers are issued, the terms are accumulated in stencil order
    constexpr int B = MB_F3_LSQ_BATCH;
    int nx[B];
#pragma unroll
    for (int u = 0; u < B; ++u) nx[u] = u < L ? ld1_stream(ix + 32 * u, pst) : -1;
    // PRE: the moment matrix comes from m.cell_lsq; only the right-hand side is summed here
    auto acc = [&](const D3 &pc, double wc) {
      const double dx = pc.x - c.x, dy = pc.y - c.y, dz = pc.z - c.z, dw = wc - wi;
      if (!PRE) {
        ixx += dx * dx; iyy += dy * dy; izz += dz * dz;
        ixy += (dx * dy); ixz += (dx * dz); iyz += (dy * dz);
      }
      jx += (dx * dw); jy += (dy * dw); jz += (dz * dw);
    };
    for (; k + B <= L; k += B) {
      int cc[B];
#pragma unroll
      for (int u = 0; u < B; ++u) {
        cc[u] = nx[u];
        nx[u] = k + B + u < L ? ld1_stream(ix + 32 * (k + B + u), pst) : -1;
      }
      D3 pc[B];
      double wc[B];
#pragma unroll
      for (int u = 0; u < B; ++u) {
        if (cc[u] < 0) {            // padding: the cell itself, no gather issued, exact zero terms
          pc[u] = c;
          wc[u] = wi;
        } else {
          ld_row(rows + 4 * (long long)cc[u], pc[u].x, pc[u].y, pc[u].z, wc[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < B; ++u) acc(pc[u], wc[u]);
    }
    // the last L - k < B entries, whose indices are in nx
#pragma unroll
    for (int u = 0; u < B - 1; ++u) {
      if (k + u < L) {
        D3 pc = c;
        double wcc = wi;
        if (nx[u] >= 0) ld_row(rows + 4 * (long long)nx[u], pc.x, pc.y, pc.z, wcc);
        acc(pc, wcc);
      }
    }
    const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
    for (int k = gb; k < ge; ++k) {
      const int f = ld(m.ghostnid_idx + k);
      const double *gc = m.face_ghostcenter + 3 * f;
      acc(d3(ld(gc), ld(gc + 1), ld(gc + 2)), ghost(f));
    }
    double gx, gy, gz;
    if (PRE) {
      double a, b, cc, d, e, ff, dia, pad;
      ld4d(m.cell_lsq + 12 * (long long)i, a, b, cc, d);
      ld4d(m.cell_lsq + 12 * (long long)i + 4, e, ff, dia, pad);
      gx = (a * jx + b * jy + cc * jz) / dia;
      gy = (b * jx + d * jy + e * jz) / dia;
      gz = (cc * jx + e * jy + ff * jz) / dia;
    } else {
      const double dia = ixx * iyy * izz + 2. * ixy * ixz * iyz - ixx * (iyz * iyz) - iyy * (ixz * ixz) - izz * (ixy * ixy);
      gx = ((iyy * izz - iyz * iyz) * jx + (ixz * iyz - ixy * izz) * jy + (ixy * iyz - ixz * iyy) * jz) / dia;
      gy = ((ixz * iyz - ixy * izz) * jx + (ixx * izz - ixz * ixz) * jy + (ixy * ixz - iyz * ixx) * jz) / dia;
      gz = ((ixy * iyz - ixz * iyy) * jx + (ixy * ixz - iyz * ixx) * jy + (ixx * iyy - ixy * ixy) * jz) / dia;
    }
    // Barth limiter over the four faces
    const int4 vt = ld4(m.cell_vtx + 4 * i);
    const int4 nb = ld4(m.cell_nbr + 4 * i);
    const uint32_t fl = ld(m.cell_flags + i);
    const D3 P[4] = {ld3(m.node_coord + 4 * vt.x), ld3(m.node_coord + 4 * vt.y), ld3(m.node_coord + 4 * vt.z),
                     ld3(m.node_coord + 4 * vt.w)};
    double wmax = wi, wmin = wi;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int o = comp(nb, j);
      const double b = o < 0 ? ghost(-1 - o) : ld(w + o);
      wmax = pmax(wmax, b);
      wmin = pmin(wmin, b);
    }
    double ps = 1.;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int d0, d1, d2;
      face_desc(fl, j, d0, d1, d2);
      const D3 fc = (1. / 3) * tet_face_sum(P, j, d2);
      const double delta = gx * (fc.x - c.x) + gy * (fc.y - c.y) + gz * (fc.z - c.z);
      double psi_ij = 1.;
      if (!(fabs(delta) < 1e-10)) {
        if (delta > 0.) psi_ij = pmin(1., (wmax - wi) / delta);
        if (delta < 0.) psi_ij = pmin(1., (wmin - wi) / delta);
      }
      ps = pmin(ps, psi_ij);
    }
    st4_keep(rec + 4 * (long long)i, wi, ps * gx, ps * gy, ps * gz, l2_keep());
    return;
  }
  if (DIFF) {
    const int n = (blockIdx.x - (ORDER2 ? ncb : 0)) * blockDim.x + threadIdx.x;
    if (n >= m.nbnodes) return;
    double acc = 0.;
    const int sb = ld(m.n2c_sell_ptr + (n >> 5)), se = ld(m.n2c_sell_ptr + (n >> 5) + 1);
    for (int k = sb + lane; k < se; k += 32) acc += ld(m.n2c_sell_alpha + k) * ld(w + ld(m.n2c_sell_idx + k));
    const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
    for (int k = gb; k < ge; ++k) acc += ld(m.n2g_alpha + k) * ghost(ld(m.n2g_idx + k));
    wn[n] = acc;
  }
}

// cell_lsq of a tetrahedral mesh: the moment matrix of each cell's stencil summed in the
// order of k_f3_phase1 (SELL slots, then stencil ghosts), as cofactors and determinant with
// the expressions k_f3_phase1 uses when it forms the matrix itself
__global__ void __launch_bounds__(kBlock) k_lsq_matrix3(mb_mesh m, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const int lane = threadIdx.x & 31;
  const D3 c = ld3(m.cell_xy + 4 * (long long)i);
  double ixx = 0., iyy = 0., izz = 0., ixy = 0., ixz = 0., iyz = 0.;
  auto acc = [&](const D3 &pc) {
    const double dx = pc.x - c.x, dy = pc.y - c.y, dz = pc.z - c.z;
    ixx += dx * dx; iyy += dy * dy; izz += dz * dz;
    ixy += (dx * dy); ixz += (dx * dz); iyz += (dy * dz);
  };
  // D = sum over the cell stencil (ghosts excluded) of the centre offsets
  double sx = 0., sy = 0., sz = 0.;
  const int sb = ld(m.lsq_sell_ptr + (i >> 5)), se = ld(m.lsq_sell_ptr + (i >> 5) + 1);
  for (int k = 0; k < (se - sb) >> 5; ++k) {
    const int cc = ld(m.lsq_sell_idx + sb + lane + 32 * k);
    const D3 pc = cc < 0 ? c : ld3(m.cell_xy + 4 * (long long)cc);
    acc(pc);
    sx += pc.x - c.x; sy += pc.y - c.y; sz += pc.z - c.z;
  }
  const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
  for (int k = gb; k < ge; ++k) {
    const double *gc = m.face_ghostcenter + 3 * ld(m.ghostnid_idx + k);
    acc(d3(ld(gc), ld(gc + 1), ld(gc + 2)));
  }
  const double dia = ixx * iyy * izz + 2. * ixy * ixz * iyz - ixx * (iyz * iyz) - iyy * (ixz * ixz) - izz * (ixy * ixy);
  double *o = out + 12 * (long long)i;
  st4d_plain(o, iyy * izz - iyz * iyz, ixz * iyz - ixy * izz, ixy * iyz - ixz * iyy, ixx * izz - ixz * ixz);
  st4d_plain(o + 4, ixy * ixz - iyz * ixx, ixx * iyy - ixy * ixy, dia, 0.0);
  st4d_plain(o + 8, sx, sy, sz, 0.0);
}

// ---------------------------------------------------------------- tetrahedra: LSQ sums by inclusion-exclusion
//
// The stencil of tetrahedron i (manapy's cells.cellnid: the cells that share a vertex with i,
// i excluded) is the union of its four vertices' cell lists.  Two of the lists meet in the
// cells of an edge, three in the cells of a face (i and its face neighbour), four in i alone,
// so by inclusion-exclusion, for any f,
//   sum_stencil f = sum_4 vertices F_v - sum_6 edges F_e + sum_face neighbours f(o),
// f(i) appearing 4 - 6 + 4 - 1 - 1 = 0 times.  With sums kept relative to an origin x of each
// vertex or edge, F = P + (x - c_i) Q, P = sum_j (c_j - x) w_j, Q = sum_j w_j, and the
// right-hand side of manapy's gradient (manapy/ast/functions3d.py:4-120) is
//   sum_stencil (c_j - c_i)(w_j - w_i) = sum_stencil (c_j - c_i) w_j - w_i D_i
// with D_i = sum_stencil (c_j - c_i) (cell_lsq), then the stencil ghosts as before.  It
// equals the direct sum up to rounding; a cell gathers 4 vertex and 6 edge records and its
// face neighbours instead of about 60 neighbours, and each cell's row is read by its 4
// vertices' and 6 edges' sums.

// vertex blocks [0, nnb): the vertex's sums and (DIFF) its centre->vertex value; edge blocks:
// the edge's sums.  Records {P, Q} (32 bytes).
template <bool DIFF>
__global__ void __launch_bounds__(kBlock) k_f3_sums(mb_mesh m, mb_bc bc, const double *__restrict__ w,
                                                    const double *__restrict__ rows, double *__restrict__ nrec,
                                                    double *__restrict__ erec, double *__restrict__ wn, int nnb) {
  const int lane = threadIdx.x & 31;
  const uint64_t pst = l2_stream();
  double px = 0., py = 0., pz = 0., q = 0.;
  if ((int)blockIdx.x < nnb) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nbnodes) return;
    const D3 X = ld3(m.node_coord + 4 * (long long)n);
    const int sb = ld(m.n2c_sum_ptr + (n >> 5)), se = ld(m.n2c_sum_ptr + (n >> 5) + 1);
    double acc = 0.;
    for (int k = sb + lane; k < se; k += 32) {
      const int cc = ld1_stream(m.n2c_sum_idx + k, pst);
      if (cc < 0) continue;       // empty slot
      double x, y, z, wc;
      ld_row(rows + 4 * (long long)cc, x, y, z, wc);
      if (DIFF) acc += ldd_stream(m.n2c_sum_alpha + k, pst) * wc;
      px += (x - X.x) * wc; py += (y - X.y) * wc; pz += (z - X.z) * wc;
      q += wc;
    }
    if (DIFF) {
      const GhostRule ghost = make_rule(m, bc, w);
      const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
      for (int k = gb; k < ge; ++k) acc += ld(m.n2g_alpha + k) * ghost(ld(m.n2g_idx + k));
      wn[n] = acc;
    }
    st4_keep(nrec + 4 * (long long)n, px, py, pz, q, l2_keep());
    return;
  }
  const int e = (blockIdx.x - nnb) * blockDim.x + threadIdx.x;
  if (e >= m.nbedges) return;
  const D3 X = ld3(m.node_coord + 4 * (long long)ld(m.edge_origin + e));
  const int sb = ld(m.edge_sell_ptr + (e >> 5)), se = ld(m.edge_sell_ptr + (e >> 5) + 1);
  for (int k = sb + lane; k < se; k += 32) {
    const int cc = ld1_stream(m.edge_sell_idx + k, pst);
    if (cc < 0) continue;
    double x, y, z, wc;
    ld_row(rows + 4 * (long long)cc, x, y, z, wc);
    px += (x - X.x) * wc; py += (y - X.y) * wc; pz += (z - X.z) * wc;
    q += wc;
  }
  st4_keep(erec + 4 * (long long)e, px, py, pz, q, l2_keep());
}

// cell pass: the gradient from the vertex, edge and face-neighbour sums, the Barth limiter;
// the same record as k_f3_phase1
template <int VAR>
__global__ void __launch_bounds__(kQ1B[VAR], kQ1M[VAR]) k_f3_grad(mb_mesh m, mb_bc bc, const double *__restrict__ w,
                                                                    double *__restrict__ rec,
                                                                    const double *__restrict__ rows,
                                                                    const double *__restrict__ nrec,
                                                                    const double *__restrict__ erec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const GhostRule ghost = make_rule(m, bc, w);
  D3 c;
  double wi;
  ld_row(rows + 4 * (long long)i, c.x, c.y, c.z, wi);
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const int4 ea = ld4(m.cell_edges + 8 * (long long)i), eb = ld4(m.cell_edges + 8 * (long long)i + 4);
  const D3 P[4] = {ld3(m.node_coord + 4 * vt.x), ld3(m.node_coord + 4 * vt.y), ld3(m.node_coord + 4 * vt.z),
                   ld3(m.node_coord + 4 * vt.w)};
  double sx = 0., sy = 0., sz = 0.;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double px, py, pz, q;
    ld4d(nrec + 4 * (long long)comp(vt, v), px, py, pz, q);
    const D3 d = P[v] - c;
    sx += px + d.x * q; sy += py + d.y * q; sz += pz + d.z * q;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    // local vertex pairs (0,1), (0,2), (0,3), (1,2), (1,3), (2,3); origin: the vertex of smaller index
    const int a = k < 3 ? 0 : (k < 5 ? 1 : 2), b = k < 3 ? k + 1 : (k < 5 ? k - 1 : 3);
    const int e = k == 0 ? ea.x : (k == 1 ? ea.y : (k == 2 ? ea.z : (k == 3 ? ea.w : (k == 4 ? eb.x : eb.y))));
    double px, py, pz, q;
    ld4d(erec + 4 * (long long)e, px, py, pz, q);
    const D3 d = (comp(vt, a) < comp(vt, b) ? P[a] : P[b]) - c;
    sx -= px + d.x * q; sy -= py + d.y * q; sz -= pz + d.z * q;
  }
  double wmax = wi, wmin = wi;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int o = comp(nb, j);
    double b;
    if (o >= 0) {
      double x, y, z;
      ld_row(rows + 4 * (long long)o, x, y, z, b);
      sx += (x - c.x) * b; sy += (y - c.y) * b; sz += (z - c.z) * b;
    } else {
      b = ghost(-1 - o);
    }
    wmax = pmax(wmax, b);
    wmin = pmin(wmin, b);
  }
  double a0, a1, a2, a3, a4, a5, dia, pad, Dx, Dy, Dz;
  ld4d(m.cell_lsq + 12 * (long long)i, a0, a1, a2, a3);
  ld4d(m.cell_lsq + 12 * (long long)i + 4, a4, a5, dia, pad);
  ld4d(m.cell_lsq + 12 * (long long)i + 8, Dx, Dy, Dz, pad);
  double jx = sx - wi * Dx, jy = sy - wi * Dy, jz = sz - wi * Dz;
  const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
  for (int k = gb; k < ge; ++k) {
    const int f = ld(m.ghostnid_idx + k);
    const double *gc = m.face_ghostcenter + 3 * f;
    const double dw = ghost(f) - wi;
    jx += (ld(gc) - c.x) * dw; jy += (ld(gc + 1) - c.y) * dw; jz += (ld(gc + 2) - c.z) * dw;
  }
  const double gx = (a0 * jx + a1 * jy + a2 * jz) / dia;
  const double gy = (a1 * jx + a3 * jy + a4 * jz) / dia;
  const double gz = (a2 * jx + a4 * jy + a5 * jz) / dia;
  // Barth limiter over the four faces (as k_f3_phase1)
  const uint32_t fl = ld(m.cell_flags + i);
  double ps = 1.;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int d0, d1, d2;
    face_desc(fl, j, d0, d1, d2);
    const D3 fc = (1. / 3) * tet_face_sum(P, j, d2);
    const double delta = gx * (fc.x - c.x) + gy * (fc.y - c.y) + gz * (fc.z - c.z);
    double psi_ij = 1.;
    if (!(fabs(delta) < 1e-10)) {
      if (delta > 0.) psi_ij = pmin(1., (wmax - wi) / delta);
      if (delta < 0.) psi_ij = pmin(1., (wmin - wi) / delta);
    }
    ps = pmin(ps, psi_ij);
  }
  st4_keep(rec + 4 * (long long)i, wi, ps * gx, ps * gy, ps * gz, l2_keep());
}

// manapy's dissipative flux of one tetrahedron face, D (grad w . N) with the diamond
// gradient of manapy/ast/functions3d.py:122-248 (face_gradient_3d, its f_1 / f_2 vectors from
// manapy/ddm/ddm_utils3d.py) and manapy/solvers/advecdiff/fvm_utils.py:5-26: the same
// quantity with the algebra folded, so that no vector of the gradient is formed.
// f_1 = (s1 x s2 + s2 x s3) / 2 with s1 = v2 - Q2, s2 = Q3 - Q2, s3 = v1 - Q2 equals
// (Q3 - Q2) x (v1 - v2) / 2, likewise f_2 = (Q1 - Q3) x (v1 - v2) / 2, and
// (a x e) . d = a . (e x d); so with DN = (Dxx N_x, Dyy N_y, Dzz N_z), t = (v1 - v2) x DN:
//   D grad . N = [(V_A - V_C) (Q3 - Q2).t / 2 + (V_B - V_C) (Q1 - Q3).t / 2
//                 + (V_R - V_L) N.DN] / (N . (v2 - v1))
// (V_D = V_C on triangular faces).  Equal to manapy's expression up to rounding.
__device__ __forceinline__ double diamond3(const mb_advdiff_params &p, const D3 &N, const D3 &Q1, const D3 &Q2,
                                           const D3 &Q3, const D3 &v1, const D3 &v2, double VA, double VB,
                                           double VC, double VL, double VR) {
  const D3 DN = d3(p.Dxx * N.x, p.Dyy * N.y, p.Dzz * N.z);
  const D3 t = cross(v1 - v2, DN);
  const double f1d = 0.5 * dot(Q3 - Q2, t), f2d = 0.5 * dot(Q1 - Q3, t);
  return ((VA - VC) * f1d + (VB - VC) * f2d + (VR - VL) * dot(N, DN)) / dot(N, v2 - v1);
}

#ifndef MB_P2_3D_MIN_BLOCKS
#define MB_P2_3D_MIN_BLOCKS 2
#endif
#ifndef MB_P2_3D_BLOCK
#define MB_P2_3D_BLOCK kBlock
#endif

constexpr int kQ2B[4] = {MB_P2_3D_BLOCK, 128, 128, 128};
constexpr int kQ2M[4] = {MB_P2_3D_MIN_BLOCKS, 4, 5, 6};

template <bool ORDER2, bool DIFF, bool WROWS, int VAR>
__global__ void __launch_bounds__(kQ2B[VAR], kQ2M[VAR]) k_f3_phase2(mb_mesh m, mb_bc bc, mb_advdiff_params p,
                                                         const double *__restrict__ w, double *__restrict__ w_out,
                                                         const double *__restrict__ sign,
                                                         const double *__restrict__ src,
                                                         const double *__restrict__ dt_dev,
                                                         const double *__restrict__ rec,
                                                         const double *__restrict__ wn,
                                                         double *__restrict__ rows_out, int c0, int c1) {
  const int i = c0 + blockIdx.x * blockDim.x + threadIdx.x;   // cells [c0, c1)
  if (i >= c1) return;
  const GhostRule ghost = make_rule(m, bc, w);
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const D3 ci = ld3(m.cell_xy + 4 * i);
  const double2 sa = ldd2(sign + 4 * i), sb = ldd2(sign + 4 * i + 2);
  // order 2: the record {w, psi gx, psi gy, psi gz} of phase 1
  double wi, gxi = 0., gyi = 0., gzi = 0.;
  if (ORDER2) {
    ld4d(rec + 4 * (long long)i, wi, gxi, gyi, gzi);
  } else {
    wi = ld(w + i);
  }
  double cv[4], q[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int o = comp(nb, j);
    const bool b = o < 0;
    const int f = -1 - o;
    const bool own = (fl >> (6 * j)) & 1u;
    int d0, d1, d2;
    face_desc(fl, j, d0, d1, d2);
    // the face's vertices gathered by index (L1 hits after the first face) instead of
    // selected among four held in registers
    const int g0 = comp(vt, d0), g1 = comp(vt, d1), g2 = comp(vt, d2);
    const D3 V0 = ld3(m.node_coord + 4 * g0), V1 = ld3(m.node_coord + 4 * g1), V2 = ld3(m.node_coord + 4 * g2);
    const D3 fc = (1. / 3) * ((V0 + V1) + V2);
    double vo, gxo = 0., gyo = 0., gzo = 0.;
    D3 co;
    if (b) {
      vo = ghost(f);
      co = d3(ld(m.face_ghostcenter + 3 * f), ld(m.face_ghostcenter + 3 * f + 1), ld(m.face_ghostcenter + 3 * f + 2));
    } else {
      if (ORDER2) {
        ld4d(rec + 4 * (long long)o, vo, gxo, gyo, gzo);
      } else {
        vo = ld(w + o);
      }
      co = ld3(m.cell_xy + 4 * o);
    }
    const double s = pick4v(sa.x, sa.y, sb.x, sb.y, j);
    const bool take_me = (s >= 0) == own;
    double sol;
    if (take_me) {
      sol = ORDER2 ? wi + (gxi * (fc.x - ci.x) + gyi * (fc.y - ci.y) + gzi * (fc.z - ci.z)) : wi;
    } else if (b) {
      sol = vo;
    } else {
      sol = ORDER2 ? vo + (gxo * (fc.x - co.x) + gyo * (fc.y - co.y) + gzo * (fc.z - co.z)) : vo;
    }
    const double F = s * sol;
    cv[j] = own ? -F : F;
    if (DIFF) {
      double v = 0.;
      if (!b || ld(bc.face_grad_on + f)) {
        const D3 Nd = 0.5 * cross(V1 - V0, V2 - V0);
        const D3 N = ((fl >> (6 * j + 5)) & 1u) ? (-1.0) * Nd : Nd;
        const bool swp = (fl >> (6 * j + 4)) & 1u;
        // faces.nodeid order: (d0, d1, d2), or (d0, d2, d1) when swapped
        const D3 Q2 = swp ? V2 : V1, Q3 = swp ? V1 : V2;
        const D3 v1 = own ? ci : co, v2 = own ? co : ci;
        const int gi2 = swp ? g2 : g1, gi3 = swp ? g1 : g2;
        const double VL = own ? wi : vo, VR = own ? vo : wi;
        v = diamond3(p, N, V0, Q2, Q3, v1, v2, ld(wn + g0), ld(wn + gi2), ld(wn + gi3), VL, VR);
      }
      q[j] = own ? v : -v;
    }
  }
  const uint8_t code = ld(m.cell_order + i);
  double rez = 0.;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int sl = order_slot(code, k);
    if (pick4v(nb.x, nb.y, nb.z, nb.w, sl) >= 0) rez += pick4v(cv[0], cv[1], cv[2], cv[3], sl);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int sl = order_slot(code, k);
    if (pick4v(nb.x, nb.y, nb.z, nb.w, sl) < 0) rez += pick4v(cv[0], cv[1], cv[2], cv[3], sl);
  }
  double dis = 0.;
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 4; ++k) dis += pick4v(q[0], q[1], q[2], q[3], order_slot(code, k));
  }
  const double dt = *dt_dev;
  const double sc = src ? ld(src + i) : 0.0;
  const double wnew = wi + dt * ((rez + dis) / ld(m.cell_volume + i) + sc);
  w_out[i] = wnew;
  if (WROWS) st4d_plain(rows_out + 4 * (long long)i, ci.x, ci.y, ci.z, wnew);
}

// ---------------------------------------------------------------- shallow-water order-2 pre-pass

// Neumann ghost: the interior cell's value (the default boundary of a manapy Variable).
struct NeumannCopy {
  const double *w;
  const int32_t *fcell;
  __device__ __forceinline__ double operator()(int f) const { return ld(w + ld(fcell + 2 * f)); }
};

// h and hc LSQ gradients and hc's Barth limiter (manapy/solvers/shallowater/system.py:164-166).
__global__ void __launch_bounds__(kBlock) k_sw_grad(mb_mesh m, const double *h, const double *hc, double *hx,
                                                    double *hy, double *cx, double *cy, double *psi) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    double x, y, z;
    lsq_gradient<2>(m, h, NeumannCopy{h, m.face_cellid}, i, x, y, z);
    hx[i] = x; hy[i] = y;
    lsq_gradient<2>(m, hc, NeumannCopy{hc, m.face_cellid}, i, x, y, z);
    cx[i] = x; cy[i] = y;
    psi[i] = barth<2>(m, hc, NeumannCopy{hc, m.face_cellid}, i, x, y, 0.0);
  }
}

// ---------------------------------------------------------------- launch helpers

inline int grid_for(long long n) {
  int g = ceil_div(n, kBlock);
  const int cap = 148 * 16;
  return g < 1 ? 1 : (g > cap ? cap : g);
}

inline int check_launch() { return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA; }

inline bool compact_tables(const mb_mesh &m) {
  return m.cell_vtx && m.cell_nbr && m.cell_flags && m.node_coord && m.cell_xy && m.lsq_sell_ptr &&
         m.lsq_sell_idx && m.n2c_sell_ptr && m.n2c_sell_idx && m.n2c_sell_alpha;
}

// launches of the fused phases in launch-shape variant v (variants beyond 0 exist for
// second order with diffusion only)
template <bool O2, bool DF, bool ROWS, int V>
inline void f2_p1_run(const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, double *wn,
                      const double *rows, cudaStream_t st) {
  const int ncb = O2 ? ceil_div(m.nbcells, kP1B[V]) : 0, nnb = DF ? ceil_div(m.nbnodes, kP1B[V]) : 0;
  k_f2_phase1<O2, DF, ROWS, V><<<ncb + nnb, kP1B[V], 0, st>>>(m, bc, w, cs, wn, ncb, rows);
}
template <bool O2, bool DF, bool ROWS>
inline void f2_p1_pick(int v, const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, double *wn,
                       const double *rows, cudaStream_t st) {
  if constexpr (O2 && DF) {
    if (v == 1) return f2_p1_run<O2, DF, ROWS, 1>(m, bc, w, cs, wn, rows, st);
    if (v == 2) return f2_p1_run<O2, DF, ROWS, 2>(m, bc, w, cs, wn, rows, st);
    if (v == 3) return f2_p1_run<O2, DF, ROWS, 3>(m, bc, w, cs, wn, rows, st);
  }
  f2_p1_run<O2, DF, ROWS, 0>(m, bc, w, cs, wn, rows, st);
}
template <bool O2, bool DF, bool WROWS, int V>
inline void f2_p2_run(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const double *w_in,
                      double *w_out, const double *sign, const double *src, const double *dt, const double *cs,
                      const double *wn, double *rows_out, int c0, int c1, cudaStream_t st) {
  if (c1 <= c0) return;
  k_f2_phase2<O2, DF, WROWS, V><<<ceil_div(c1 - c0, kP2B[V]), kP2B[V], 0, st>>>(m, bc, p, w_in, w_out, sign, src, dt,
                                                                                 cs, wn, rows_out, c0, c1);
}
template <bool O2, bool DF, bool WROWS>
inline void f2_p2_pick(int v, const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const double *w_in,
                       double *w_out, const double *sign, const double *src, const double *dt, const double *cs,
                       const double *wn, double *rows_out, int c0, int c1, cudaStream_t st) {
  if constexpr (O2 && DF) {
    if (v == 1) return f2_p2_run<O2, DF, WROWS, 1>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
    if (v == 2) return f2_p2_run<O2, DF, WROWS, 2>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
    if (v == 3) return f2_p2_run<O2, DF, WROWS, 3>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
  }
  f2_p2_run<O2, DF, WROWS, 0>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
}
template <bool O2, bool DF, int V>
inline void f3_p1_run(const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, const double *rows, double *wn,
                      cudaStream_t st) {
  const int B = kQ1B[V];
  const int ncb = O2 ? ceil_div(m.nbcells, B) : 0, nnb = DF ? ceil_div(m.nbnodes, B) : 0;
  if (O2 && m.cell_lsq)
    k_f3_phase1<O2, DF, V, true><<<ncb + nnb, B, 0, st>>>(m, bc, w, cs, rows, wn, ncb);
  else
    k_f3_phase1<O2, DF, V, false><<<ncb + nnb, B, 0, st>>>(m, bc, w, cs, rows, wn, ncb);
}
// the first phase by inclusion-exclusion: vertex and edge sums (and node values), then the
// cells; records of the sums after the cell records and rows in the cell scratch
inline bool f3_sums_tables(const mb_mesh &m) {
  return m.cell_edges && m.edge_origin && m.edge_sell_ptr && m.edge_sell_idx && m.nbedges > 0 && m.cell_lsq &&
         m.n2c_sum_ptr && m.n2c_sum_idx && m.n2c_sum_alpha;
}
template <bool DF, int V>
inline void f3_sums_run(const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, const double *rows,
                        double *wn, cudaStream_t st) {
  double *nrec = cs + 8 * (long long)m.nbcells, *erec = nrec + 4 * (long long)m.nbnodes;
  const int nnb = ceil_div(m.nbnodes, kBlock), neb = ceil_div(m.nbedges, kBlock);
  k_f3_sums<DF><<<nnb + neb, kBlock, 0, st>>>(m, bc, w, rows, nrec, erec, wn, nnb);
  k_f3_grad<V><<<ceil_div(m.nbcells, kQ1B[V]), kQ1B[V], 0, st>>>(m, bc, w, cs, rows, nrec, erec);
}
template <bool DF>
inline void f3_sums_pick(int v, const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, const double *rows,
                         double *wn, cudaStream_t st) {
  if (v == 1) return f3_sums_run<DF, 1>(m, bc, w, cs, rows, wn, st);
  if (v == 2) return f3_sums_run<DF, 2>(m, bc, w, cs, rows, wn, st);
  if (v == 3) return f3_sums_run<DF, 3>(m, bc, w, cs, rows, wn, st);
  f3_sums_run<DF, 0>(m, bc, w, cs, rows, wn, st);
}
template <bool O2, bool DF>
inline void f3_p1_pick(int v, const mb_mesh &m, const mb_bc &bc, const double *w, double *cs, const double *rows,
                       double *wn, cudaStream_t st) {
  if constexpr (O2 && DF) {
    if (v == 1) return f3_p1_run<O2, DF, 1>(m, bc, w, cs, rows, wn, st);
    if (v == 2) return f3_p1_run<O2, DF, 2>(m, bc, w, cs, rows, wn, st);
    if (v == 3) return f3_p1_run<O2, DF, 3>(m, bc, w, cs, rows, wn, st);
  }
  f3_p1_run<O2, DF, 0>(m, bc, w, cs, rows, wn, st);
}
template <bool O2, bool DF, bool WROWS, int V>
inline void f3_p2_run(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const double *w_in,
                      double *w_out, const double *sign, const double *src, const double *dt, const double *cs,
                      const double *wn, double *rows_out, int c0, int c1, cudaStream_t st) {
  if (c1 <= c0) return;
  k_f3_phase2<O2, DF, WROWS, V><<<ceil_div(c1 - c0, kQ2B[V]), kQ2B[V], 0, st>>>(m, bc, p, w_in, w_out, sign, src, dt,
                                                                                 cs, wn, rows_out, c0, c1);
}
template <bool O2, bool DF, bool WROWS>
inline void f3_p2_pick(int v, const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const double *w_in,
                       double *w_out, const double *sign, const double *src, const double *dt, const double *cs,
                       const double *wn, double *rows_out, int c0, int c1, cudaStream_t st) {
  if constexpr (O2 && DF) {
    if (v == 1) return f3_p2_run<O2, DF, WROWS, 1>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
    if (v == 2) return f3_p2_run<O2, DF, WROWS, 2>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
    if (v == 3) return f3_p2_run<O2, DF, WROWS, 3>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
  }
  f3_p2_run<O2, DF, WROWS, 0>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
}

// cell scratch: [4][nbcells] planes gx, gy, gz, psi (face-table path), [nbcells][4]
// records {w, gx, gy, psi} (compact 2D path) or [nbcells][4] records {w, psi gx, psi gy,
// psi gz} then [nbcells][4] rows {x, y, z, w} (compact 3D path); node scratch: [nbnodes]
// part < 0: the whole step; part 0: phase 1 and phase 2 of cells [0, nfirst); part 1: phase 2
// of cells [nfirst, nbcells), reading what part 0 left in the scratch (compact tables only)
template <int DIM, bool O2, bool DF>
int launch_step(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const double *w_in,
                double *w_out, const double *sign, const double *src, const double *dt, double *cs,
                double *wn, cudaStream_t st, const double *rows_in = nullptr, double *rows_out = nullptr,
                int part = -1, int nfirst = 0) {
  if (part >= 0 && (!compact_tables(m) || nfirst < 0 || nfirst > m.nbcells)) return MB_EINVAL;
  const int c0 = part == 1 ? nfirst : 0, c1 = part == 0 ? nfirst : m.nbcells;
  const bool p1 = part != 1;
  const int ncb = O2 ? ceil_div(m.nbcells, kBlock) : 0;
  const int nnb = DF ? ceil_div(m.nbnodes, kBlock) : 0;
  if (compact_tables(m)) {
#if MB_LD256
    // 256-bit loads of [n][4] rows: the phase-1 records (2D) and the centre and vertex
    // tables (3D) must start on 32-byte boundaries
    auto a32 = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 31) == 0; };
    if ((O2 && !a32(cs)) || (DIM == 3 && (!a32(m.cell_xy) || !a32(m.node_coord) || !a32(m.cell_lsq)))) return MB_EINVAL;
    if ((rows_in && !a32(rows_in)) || (rows_out && !a32(rows_out))) return MB_EINVAL;
#endif
#if MB_V4_IO
    if (DIM == 2 && (reinterpret_cast<uintptr_t>(sign) & 31) != 0) return MB_EINVAL;
#endif
    // launch-shape variants (second order with diffusion only): bits 0-1 phase 1, bits 2-3 phase 2
    const int v1 = (O2 && DF) ? (m.variant & 3) : 0, v2 = (O2 && DF) ? ((m.variant >> 2) & 3) : 0;
    if (DIM == 2) {
      if ((O2 || DF) && p1) {
        if (rows_in) f2_p1_pick<O2, DF, true>(v1, m, bc, w_in, cs, wn, rows_in, st);
        else f2_p1_pick<O2, DF, false>(v1, m, bc, w_in, cs, wn, nullptr, st);
      }
      if (rows_out) f2_p2_pick<O2, DF, true>(v2, m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
      else f2_p2_pick<O2, DF, false>(v2, m, bc, p, w_in, w_out, sign, src, dt, cs, wn, nullptr, c0, c1, st);
    } else {
      // cell scratch: records [0, 4 nbcells), then (without rows_in) the pack pass's rows
      const double *rows = rows_in;
      if (O2 && !rows && p1) {
        double *pk = cs + 4 * (long long)m.nbcells;
        k_pack_rows<3><<<ceil_div(m.nbcells, kBlock), kBlock, 0, st>>>(m, w_in, pk);
        rows = pk;
      }
      if (O2 && p1 && f3_sums_tables(m)) {
        f3_sums_pick<DF>((m.variant & 3), m, bc, w_in, cs, rows, wn, st);
      } else if ((O2 || DF) && p1) {
        f3_p1_pick<O2, DF>(v1, m, bc, w_in, cs, rows, wn, st);
      }
      if (rows_out) f3_p2_pick<O2, DF, true>(v2, m, bc, p, w_in, w_out, sign, src, dt, cs, wn, rows_out, c0, c1, st);
      else f3_p2_pick<O2, DF, false>(v2, m, bc, p, w_in, w_out, sign, src, dt, cs, wn, nullptr, c0, c1, st);
    }
    return check_launch();
  }
  const long long n = m.nbcells;
  double *gx = cs, *gy = cs + n, *gz = cs + 2 * n, *psi = cs + 3 * n;
  if (ncb + nnb > 0)
    k_step_phase1<DIM, O2, DF><<<ncb + nnb, kBlock, 0, st>>>(m, bc, w_in, gx, gy, gz, psi, wn, ncb);
  k_step_phase2<DIM, O2, DF><<<ceil_div(m.nbcells, kBlock), kBlock, 0, st>>>(m, bc, p, w_in, w_out, sign, src,
                                                                             dt, gx, gy, gz, psi, wn);
  return check_launch();
}

int sw_gradients(const mb_mesh &m, const double *h, const double *hc, double *hx, double *hy, double *cx,
                 double *cy, double *psi, cudaStream_t st) {
  k_sw_grad<<<grid_for(m.nbcells), kBlock, 0, st>>>(m, h, hc, hx, hy, cx, cy, psi);
  return check_launch();
}

}  // namespace mb

using namespace mb;

static bool mesh_ok(const mb_mesh *m) {
  return m && (m->dim == 2 || m->dim == 3) && m->nbcells > 0 && m->nbfaces > 0 && m->nbnodes > 0 &&
         m->nlf == (m->dim == 2 ? 3 : 4);
}

#define ST(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

int mb_facetocell(const mb_mesh *m, const double *u_face, double *u_cell, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !u_face || !u_cell) return MB_EINVAL;
  k_facetocell<<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, u_face, u_cell);
  return check_launch();
}

int mb_ghost_value(const mb_mesh *m, const mb_bc *bc, const double *w_c, double *w_ghost, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !w_c || !w_ghost) return MB_EINVAL;
  k_ghost<<<grid_for(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, *bc, w_c, w_ghost);
  return check_launch();
}

int mb_cell_gradient(const mb_mesh *m, const double *w_c, const double *w_ghost, double *w_x, double *w_y,
                     double *w_z, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !w_c || !w_ghost || !w_x || !w_y || !w_z) return MB_EINVAL;
  if (m->dim == 2)
    k_cell_gradient<2><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, w_c, w_ghost, w_x, w_y, w_z);
  else
    k_cell_gradient<3><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, w_c, w_ghost, w_x, w_y, w_z);
  return check_launch();
}

int mb_barthlimiter(const mb_mesh *m, const double *w_c, const double *w_ghost, const double *w_x,
                    const double *w_y, const double *w_z, double *psi, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !w_c || !w_ghost || !w_x || !w_y || !w_z || !psi) return MB_EINVAL;
  if (m->dim == 2)
    k_barth<2><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, w_c, w_ghost, w_x, w_y, w_z, psi);
  else
    k_barth<3><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, w_c, w_ghost, w_x, w_y, w_z, psi);
  return check_launch();
}

int mb_centertovertex(const mb_mesh *m, const double *w_c, const double *w_ghost, double *w_node,
                      void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !w_c || !w_ghost || !w_node) return MB_EINVAL;
  k_centertovertex<<<grid_for(m->nbnodes), kBlock, 0, ST(stream)>>>(*m, w_c, w_ghost, w_node);
  return check_launch();
}

int mb_face_gradient(const mb_mesh *m, const mb_bc *bc, const double *w_c, const double *w_ghost,
                     const double *w_node, double *wx_face, double *wy_face, double *wz_face, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !bc->face_grad_on || !w_c || !w_ghost || !w_node || !wx_face || !wy_face ||
      (m->dim == 3 && !wz_face))
    return MB_EINVAL;
  if (m->dim == 2)
    k_face_gradient<2><<<grid_for(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, bc->face_grad_on, w_c, w_ghost,
                                                                         w_node, wx_face, wy_face, wz_face);
  else
    k_face_gradient<3><<<grid_for(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, bc->face_grad_on, w_c, w_ghost,
                                                                         w_node, wx_face, wy_face, wz_face);
  return check_launch();
}

int mb_explicitscheme_convective(const mb_mesh *m, double *rez_w, const double *w_c, const double *w_ghost,
                                 const double *u_face, const double *v_face, const double *w_face,
                                 const double *w_x, const double *w_y, const double *w_z, const double *psi,
                                 int32_t order, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !rez_w || !w_c || !w_ghost || !u_face || !v_face || !w_face || (order != 1 && order != 2))
    return MB_EINVAL;
  if (order == 2 && (!w_x || !w_y || !w_z || !psi)) return MB_EINVAL;
  if (m->dim == 2)
    k_convective<2><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, rez_w, w_c, w_ghost, u_face, v_face,
                                                                      w_face, w_x, w_y, w_z, psi, order);
  else
    k_convective<3><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, rez_w, w_c, w_ghost, u_face, v_face,
                                                                      w_face, w_x, w_y, w_z, psi, order);
  return check_launch();
}

int mb_explicitscheme_dissipative(const mb_mesh *m, const double *wx_face, const double *wy_face,
                                  const double *wz_face, double *dissip_w, double Dxx, double Dyy, double Dzz,
                                  void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !wx_face || !wy_face || !wz_face || !dissip_w) return MB_EINVAL;
  if (m->dim == 2)
    k_dissipative<2><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, wx_face, wy_face, wz_face, dissip_w,
                                                                       Dxx, Dyy, Dzz);
  else
    k_dissipative<3><<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, wx_face, wy_face, wz_face, dissip_w,
                                                                       Dxx, Dyy, Dzz);
  return check_launch();
}

int mb_time_step(const mb_mesh *m, const double *u, const double *v, const double *w, double cfl, double Dxx,
                 double Dyy, double Dzz, double *dt_dev, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !u || !v || !w || !dt_dev) return MB_EINVAL;
  k_fill<<<1, 1, 0, ST(stream)>>>(dt_dev, 1e6);
  k_time_step<<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, u, v, w, cfl, Dxx, Dyy, Dzz, dt_dev);
  return check_launch();
}

int mb_update_new_value(const mb_mesh *m, double *ne_c, const double *rez, const double *dissip,
                        const double *src, const double *dt_dev, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !ne_c || !rez || !dissip || !src || !dt_dev) return MB_EINVAL;
  k_update<<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(m->nbcells, ne_c, rez, dissip, src, dt_dev,
                                                            m->cell_volume);
  return check_launch();
}

int mb_face_sign(const mb_mesh *m, const double *u_face, const double *v_face, const double *w_face,
                 double *sign_face, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !u_face || !v_face || !w_face || !sign_face) return MB_EINVAL;
  k_face_sign<<<grid_for(m->nbfaces), kBlock, 0, ST(stream)>>>(*m, u_face, v_face, w_face, sign_face);
  return check_launch();
}

int mb_cell_face_sign(const mb_mesh *m, const double *u_face, const double *v_face, const double *w_face,
                      double *sign_cf, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !u_face || !v_face || !w_face || !sign_cf) return MB_EINVAL;
  k_cell_face_sign<<<grid_for(m->nbcells), kBlock, 0, ST(stream)>>>(*m, u_face, v_face, w_face, sign_cf);
  return check_launch();
}

int mb_advdiff_step(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p, const double *w_in,
                    double *w_out, const double *sign_cf, const double *src, const double *dt_dev,
                    double *cell_scratch, double *node_scratch, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !p || !w_in || !w_out || w_in == w_out || !sign_cf || !dt_dev) return MB_EINVAL;
  if (p->order != 1 && p->order != 2) return MB_EINVAL;
  const bool o2 = p->order == 2, df = p->diffusion != 0;
  if (o2 && !cell_scratch) return MB_EINVAL;
  if (df && (!node_scratch || !bc->face_grad_on)) return MB_EINVAL;
  if (!bc->kind || !bc->value) return MB_EINVAL;
  cudaStream_t st = ST(stream);
#define MB_STEP(D, O, F) \
  return launch_step<D, O, F>(*m, *bc, *p, w_in, w_out, sign_cf, src, dt_dev, cell_scratch, node_scratch, st)
  if (m->dim == 2) {
    if (o2) { if (df) MB_STEP(2, true, true); else MB_STEP(2, true, false); }
    else { if (df) MB_STEP(2, false, true); else MB_STEP(2, false, false); }
  } else {
    if (o2) { if (df) MB_STEP(3, true, true); else MB_STEP(3, true, false); }
    else { if (df) MB_STEP(3, false, true); else MB_STEP(3, false, false); }
  }
#undef MB_STEP
}

int mb_advdiff_step_split(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p, const double *w_in,
                          double *w_out, const double *sign_cf, const double *src, const double *dt_dev,
                          double *cell_scratch, double *node_scratch, int32_t part, int32_t nfirst, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !p || !w_in || !w_out || w_in == w_out || !sign_cf || !dt_dev) return MB_EINVAL;
  if ((part != 0 && part != 1) || !compact_tables(*m) || nfirst < 0 || nfirst > m->nbcells) return MB_EINVAL;
  if (p->order != 1 && p->order != 2) return MB_EINVAL;
  const bool o2 = p->order == 2, df = p->diffusion != 0;
  if (o2 && !cell_scratch) return MB_EINVAL;
  if (df && (!node_scratch || !bc->face_grad_on)) return MB_EINVAL;
  if (!bc->kind || !bc->value) return MB_EINVAL;
  cudaStream_t st = ST(stream);
#define MB_STEP(D, O, F)                                                                                     \
  return launch_step<D, O, F>(*m, *bc, *p, w_in, w_out, sign_cf, src, dt_dev, cell_scratch, node_scratch, st, \
                              nullptr, nullptr, part, nfirst)
  if (m->dim == 2) {
    if (o2) { if (df) MB_STEP(2, true, true); else MB_STEP(2, true, false); }
    else { if (df) MB_STEP(2, false, true); else MB_STEP(2, false, false); }
  } else {
    if (o2) { if (df) MB_STEP(3, true, true); else MB_STEP(3, true, false); }
    else { if (df) MB_STEP(3, false, true); else MB_STEP(3, false, false); }
  }
#undef MB_STEP
}

int mb_lsq_matrix(const mb_mesh *m, double *out, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || m->dim != 3 || !out || !compact_tables(*m) || !m->ghostnid_ptr || !m->ghostnid_idx ||
      !m->face_ghostcenter || (reinterpret_cast<uintptr_t>(out) & 31) != 0)
    return MB_EINVAL;
  k_lsq_matrix3<<<ceil_div(m->nbcells, kBlock), kBlock, 0, ST(stream)>>>(*m, out);
  return check_launch();
}

int mb_pack_rows(const mb_mesh *m, const double *w, double *rows, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !w || !rows || !m->cell_xy || (reinterpret_cast<uintptr_t>(rows) & 31) != 0) return MB_EINVAL;
  if (m->dim == 2)
    k_pack_rows<2><<<ceil_div(m->nbcells, kBlock), kBlock, 0, ST(stream)>>>(*m, w, rows);
  else
    k_pack_rows<3><<<ceil_div(m->nbcells, kBlock), kBlock, 0, ST(stream)>>>(*m, w, rows);
  return check_launch();
}

int mb_advdiff_step_rows(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p, const double *w_in,
                         double *w_out, const double *rows_in, double *rows_out, const double *sign_cf,
                         const double *src, const double *dt_dev, double *cell_scratch, double *node_scratch,
                         void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !p || !w_in || !w_out || w_in == w_out || !sign_cf || !dt_dev) return MB_EINVAL;
  if (!rows_in || !rows_out || rows_in == rows_out || !compact_tables(*m)) return MB_EINVAL;
  if (p->order != 1 && p->order != 2) return MB_EINVAL;
  const bool o2 = p->order == 2, df = p->diffusion != 0;
  if (o2 && !cell_scratch) return MB_EINVAL;
  if (df && (!node_scratch || !bc->face_grad_on)) return MB_EINVAL;
  if (!bc->kind || !bc->value) return MB_EINVAL;
  cudaStream_t st = ST(stream);
#define MB_STEP(D, O, F)                                                                                     \
  return launch_step<D, O, F>(*m, *bc, *p, w_in, w_out, sign_cf, src, dt_dev, cell_scratch, node_scratch, st, \
                              rows_in, rows_out)
  if (m->dim == 2) {
    if (o2) { if (df) MB_STEP(2, true, true); else MB_STEP(2, true, false); }
    else { if (df) MB_STEP(2, false, true); else MB_STEP(2, false, false); }
  } else {
    if (o2) { if (df) MB_STEP(3, true, true); else MB_STEP(3, true, false); }
    else { if (df) MB_STEP(3, false, true); else MB_STEP(3, false, false); }
  }
#undef MB_STEP
}

int mb_advdiff_batch_step(const mb_advdiff_item_f64 *items, const int32_t *p1_map, int32_t p1_blocks,
                          const int32_t *p2_map, int32_t p2_blocks, int32_t order, int32_t diffusion,
                          int32_t *clock, void *stream) {
  MB_NVTX();
  if (!items || !p2_map || !clock || p2_blocks <= 0 || p1_blocks < 0 || (order != 1 && order != 2)) return MB_EINVAL;
  const bool o2 = order == 2, df = diffusion != 0;
  if ((o2 || df) && (!p1_map || p1_blocks <= 0)) return MB_EINVAL;
  cudaStream_t st = ST(stream);
#define MB_BATCH(O, F)                                                                              \
  do {                                                                                              \
    if (O || F) k_f2_batch_phase1<O, F><<<p1_blocks, kBlock, 0, st>>>(items, p1_map, clock);        \
    k_f2_batch_phase2<O, F><<<p2_blocks, kBlock, 0, st>>>(items, p2_map, clock);                    \
  } while (0)
  if (o2 && df) MB_BATCH(true, true);
  else if (o2) MB_BATCH(true, false);
  else if (df) MB_BATCH(false, true);
  else MB_BATCH(false, false);
#undef MB_BATCH
  k_batch_tick<<<1, 1, 0, st>>>(clock);
  return check_launch();
}

}  // extern "C"

// ---------------------------------------------------------------- no-allocation variant
//
// mb_advdiff_step needs 4*nbcells (3D: 8*nbcells) + nbnodes doubles of scratch that the caller
// allocates.  Some callers cannot allocate device memory at all: a plugin that
// lives inside a host application owning every device allocation through its
// own pool, a service that reserves its whole device-memory budget up front,
// or a loop that must not call cudaMalloc because that call can synchronise the
// device.  For them the scratch below is a fixed array in the library's own
// device image, reserved on every GPU that loads the library until the process
// exits.
#include <mutex>

namespace {

static __device__ __align__(256) double g_noalloc_scratch[MB_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_base[kMaxDevices] = {};

}  // namespace

extern "C" int mb_advdiff_step_noalloc(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                                       const double *w_in, double *w_out, const double *sign_cf,
                                       const double *src, const double *dt_dev, void *stream) {
  MB_NVTX();
  if (!mesh_ok(m) || !bc || !p) return MB_EINVAL;
  // cell scratch 4*nbcells (2D) or 8*nbcells (3D), then the node scratch
  const long long cell_need = (m->dim == 2 ? 4LL : 8LL) * m->nbcells;
  const long long need = cell_need + m->nbnodes;
  if (need > (long long)MB_NOALLOC_SCRATCH_DOUBLES) return MB_ETOOBIG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MB_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return MB_EINVAL;
  double *base = nullptr;
  {
    // first call on this device: look up where the array lives on it (host code
    // cannot use the symbol itself as a device address)
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
      void *ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return MB_ECUDA;
      g_noalloc_base[dev] = static_cast<double *>(ptr);
    }
    base = g_noalloc_base[dev];
  }
  // Every slice is written by the first launch of the step before the second
  // launch reads it, so nothing has to be cleared between calls.  The scratch holds the
  // step without the edge sums (their records need more), so their tables are left out.
  mb_mesh mm = *m;
  mm.cell_edges = nullptr;
  return mb_advdiff_step(&mm, bc, p, w_in, w_out, sign_cf, src, dt_dev, base, base + cell_need, stream);
}
