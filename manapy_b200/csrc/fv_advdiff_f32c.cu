// FP32-compensated advection-diffusion step on the compact cell-centred tables.
//
// Same scheme and the same per-cell gathers as the FP64 fused step
// (manapy/solvers/advecdiff/system.py:156-172: ghost values, LSQ gradient +
// Barth limiter, centre->vertex values, upwind and diamond fluxes, forward
// Euler), with the precision split:
//   FP32  cell state, phase-1 records {w, grad, psi}, node values, u.n,
//         centre->vertex weights, every flux and the per-cell residual, whose
//         face terms are summed with Neumaier's compensated summation;
//   FP64  vertex and centre coordinates, every geometric quantity derived from
//         them (face centres, normals, diamond vectors and areas, LSQ moment
//         matrices, 1/volume) until it is multiplied by a state value, and dt.
// Geometric coefficients are formed in FP64 and rounded once to FP32, so the
// FP32 arithmetic only ever sees state x coefficient products.
//
// Difference form.  A cell's face terms nearly cancel (sum of u.n over a cell is the
// velocity divergence, the diamond coefficients of a face sum to zero), so at fine
// resolution the residual is a small difference of large terms.  The kernels
// evaluate every face term on state *differences* from the cell's own value,
//   sum_j s_j w_j          = sum_j s_j (w_j - w_i) + w_i sum_j s_j,
//   sum_k c_k t_k          = sum_k a_k (v_k - w_i) + w_i sum_k a_k,
// with sum_j s_j (the cell's signed u.n sum) and sum_k a_k formed in FP64, so FP32
// rounding stays relative to the residual instead of to the state.
#include "fv_compact.cuh"

namespace mb {

// Ghost value of boundary face f for an FP32 state (the rules of GhostRule).
struct GhostRuleF {
  const int8_t *kind;
  const double *value;
  const double *dist;
  const int32_t *face_cellid;
  const float *w;
  __device__ __forceinline__ float operator()(int f) const {
    const int k = kind[f];
    if (k == MB_G_DIRICHLET) return (float)ld(value + f);
    const float wc = ld(w + ld(face_cellid + 2 * f));
    if (k == MB_G_NEUMANN) return wc;
    if (k == MB_G_NONSLIP) return -1.f * wc;
    if (k == MB_G_NEUMANN_NH) return (float)((double)wc + ld(value + f) * ld(dist + f));
    if (k == MB_G_CELL_AT_FACE) return ld(w + (long long)ld(value + f));
    return 0.f;
  }
};

__device__ __forceinline__ GhostRuleF make_rule_f(const mb_mesh &m, const mb_bc &bc, const float *w) {
  return GhostRuleF{bc.kind, bc.value, m.face_dist, m.face_cellid, w};
}

__device__ __forceinline__ float fminp(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float fmaxp(float a, float b) { return b > a ? b : a; }

// Neumaier's compensated sum (the error of every addition is carried in c).
struct CompSum {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float t = s + x;
    c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s + c; }
};

__device__ __forceinline__ float4 ldf4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4_keep(float *a, float4 v, uint64_t pol) {
#if MB_L2_HINTS
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w), "l"(pol)
               : "memory");
#else
  *reinterpret_cast<float4 *>(a) = v;
#endif
}
__device__ __forceinline__ void st1f_keep(float *a, float x, uint64_t pol) {
#if MB_L2_HINTS
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(x), "l"(pol) : "memory");
#else
  *a = x;
#endif
}
__device__ __forceinline__ float ldf_stream(const float *a, uint64_t pol) {
#if MB_L2_HINTS
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return v;
#else
  return __ldg(a);
#endif
}

// State update with its rounding error carried: (w, lo) + inc -> (w', lo') with
// w' + lo' = w + (inc + lo) exactly (Knuth's two-sum), so the FP32 state w loses no
// increment to rounding from step to step; without lo (NULL) a plain FP32 add.
__device__ __forceinline__ void store_state(float wi, float inc, const float *__restrict__ lo_in,
                                            float *__restrict__ w_out, float *__restrict__ lo_out, int i) {
  if (lo_in) {
    const float a = inc + lo_in[i];
    const float s = wi + a;
    const float bv = s - wi;
    lo_out[i] = (wi - (s - bv)) + (a - bv);
    w_out[i] = s;
  } else {
    w_out[i] = wi + inc;
  }
}

// centre->vertex value of node n (phase 1, node blocks): FP32 weights, FP32 sum
__device__ __forceinline__ void node_value_f32(const mb_mesh &m, const GhostRuleF &ghost, const float *__restrict__ w,
                                               float *__restrict__ wn, int n, int lane) {
  if (n >= m.nbnodes) return;
  float acc = 0.f;
  const int sb = ld(m.n2c_sell_ptr + (n >> 5)), se = ld(m.n2c_sell_ptr + (n >> 5) + 1);
  const uint64_t pst = l2_stream();
#pragma unroll 4
  for (int k = sb + lane; k < se; k += 32) {
    const int cc = ld1_stream(m.n2c_sell_idx + k, pst);
    acc = fmaf(ldf_stream(m.n2c_sell_alpha_f32 + k, pst), ld(w + cc), acc);
  }
  const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
  for (int k = gb; k < ge; ++k) acc = fmaf((float)ld(m.n2g_alpha + k), ghost(ld(m.n2g_idx + k)), acc);
  st1f_keep(wn + n, acc, l2_keep());
}

// ---------------------------------------------------------------- triangles

#ifndef MB_P1C_MIN_BLOCKS
#define MB_P1C_MIN_BLOCKS 6
#endif
#ifndef MB_P2C_BLOCK
#define MB_P2C_BLOCK 128   // threads per block of the single-mesh phase 2 (batches: kBlock)
#endif
#ifndef MB_P2C_BATCH_MIN_BLOCKS
#define MB_P2C_BATCH_MIN_BLOCKS 5
#endif
#ifndef MB_P2C_MIN_BLOCKS
#define MB_P2C_MIN_BLOCKS 7
#endif

// phase 1 of block `bid` of one mesh: blocks [0, ncb) gradient + limiter records,
// the rest centre->vertex node values
template <bool ORDER2, bool DIFF>
__device__ __forceinline__ void f2c_phase1(const mb_mesh &m, const mb_bc &bc, const float *__restrict__ w,
                                           float *__restrict__ rec, float *__restrict__ wn, int ncb, int bid) {
  const GhostRuleF ghost = make_rule_f(m, bc, w);
  const int lane = threadIdx.x & 31;
  if (ORDER2 && bid < ncb) {
    const int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.nbcells) return;
    const double2 c = ldd2(m.cell_xy + 2 * i);
    const float wi = ld(w + i);
    // LSQ: moment matrix in FP64 (geometry), right-hand side in FP32
    double ixx = 0., iyy = 0., ixy = 0.;
    float jx = 0.f, jy = 0.f;
    const int sb = ld(m.lsq_sell_ptr + (i >> 5)), se = ld(m.lsq_sell_ptr + (i >> 5) + 1);
    const int L = (se - sb) >> 5;
    const int32_t *ix = m.lsq_sell_idx + sb + lane;
    const uint64_t pst = l2_stream();
    int k = 0;
    for (; k + 4 <= L; k += 4) {
      int cc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { cc[u] = ld1_stream(ix + 32 * (k + u), pst); cc[u] = cc[u] < 0 ? i : cc[u]; }
      double2 pc[4];
      float wc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { pc[u] = ldd2(m.cell_xy + 2 * cc[u]); wc[u] = ld(w + cc[u]); }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double dx = pc[u].x - c.x, dy = pc[u].y - c.y;
        const float dw = wc[u] - wi;
        ixx += dx * dx; iyy += dy * dy; ixy += dx * dy;
        jx = fmaf((float)dx, dw, jx); jy = fmaf((float)dy, dw, jy);
      }
    }
    for (; k < L; ++k) {
      int cc = ld1_stream(ix + 32 * k, pst);
      cc = cc < 0 ? i : cc;
      const double2 pc = ldd2(m.cell_xy + 2 * cc);
      const double dx = pc.x - c.x, dy = pc.y - c.y;
      const float dw = ld(w + cc) - wi;
      ixx += dx * dx; iyy += dy * dy; ixy += dx * dy;
      jx = fmaf((float)dx, dw, jx); jy = fmaf((float)dy, dw, jy);
    }
    const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
    for (int k = gb; k < ge; ++k) {
      const int f = ld(m.ghostnid_idx + k);
      const double dx = ld(m.face_ghostcenter + 3 * f) - c.x, dy = ld(m.face_ghostcenter + 3 * f + 1) - c.y;
      const float dw = ghost(f) - wi;
      ixx += dx * dx; iyy += dy * dy; ixy += dx * dy;
      jx = fmaf((float)dx, dw, jx); jy = fmaf((float)dy, dw, jy);
    }
    const double rdia = 1. / (ixx * iyy - ixy * ixy);
    const float a = (float)(iyy * rdia), b = (float)(ixy * rdia), e = (float)(ixx * rdia);
    const float x = a * jx - b * jy;
    const float y = e * jy - b * jx;
    // Barth limiter over the three faces
    const int4 vt = ld4(m.cell_vtx + 4 * i);
    const int4 nb = ld4(m.cell_nbr + 4 * i);
    const double2 P0 = ldd2(m.node_coord + 2 * vt.x), P1 = ldd2(m.node_coord + 2 * vt.y),
                  P2 = ldd2(m.node_coord + 2 * vt.z);
    float wmax = wi, wmin = wi;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int o = comp(nb, j);
      const float bv = o < 0 ? ghost(-1 - o) : ld(w + o);
      wmax = fmaxp(wmax, bv);
      wmin = fminp(wmin, bv);
    }
    float ps = 1.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double2 pa = j == 0 ? P0 : (j == 1 ? P1 : P2), pb = j == 0 ? P1 : (j == 1 ? P2 : P0);
      const float r1 = (float)(0.5 * (pa.x + pb.x) - c.x), r2 = (float)(0.5 * (pa.y + pb.y) - c.y);
      const float delta = x * r1 + y * r2;
      float psi_ij = 1.f;
      if (!(fabsf(delta) < 1e-8f)) {
        if (delta > 0.f) psi_ij = fminp(1.f, (wmax - wi) / delta);
        if (delta < 0.f) psi_ij = fminp(1.f, (wmin - wi) / delta);
      }
      ps = fminp(ps, psi_ij);
    }
    st4_keep(rec + 4 * (long long)i, make_float4(wi, x, y, ps), l2_keep());
    return;
  }
  if (DIFF) node_value_f32(m, ghost, w, wn, (bid - (ORDER2 ? ncb : 0)) * blockDim.x + threadIdx.x, lane);
}

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock, MB_P1C_MIN_BLOCKS)
    k_f2c_phase1(mb_mesh m, mb_bc bc, const float *__restrict__ w, float *__restrict__ rec, float *__restrict__ wn,
                 int ncb) {
  f2c_phase1<ORDER2, DIFF>(m, bc, w, rec, wn, ncb, blockIdx.x);
}

// phase 2 of block `bid` of one mesh: fluxes and update of its cells
template <bool ORDER2, bool DIFF>
__device__ __forceinline__ void f2c_phase2(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p,
                                           const float *__restrict__ w, float *__restrict__ w_out,
                                           const float *__restrict__ sign, const float *__restrict__ src,
                                           const double *__restrict__ dt_dev, const float *__restrict__ rec,
                                           const float *__restrict__ wn, const float *__restrict__ lo_in,
                                           float *__restrict__ lo_out, int bid) {
  const int i = bid * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const GhostRuleF ghost = make_rule_f(m, bc, w);
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const double2 P0 = ldd2(m.node_coord + 2 * vt.x), P1 = ldd2(m.node_coord + 2 * vt.y),
                P2 = ldd2(m.node_coord + 2 * vt.z);
  const double2 ci = ldd2(m.cell_xy + 2 * i);
  const float4 s4 = ldf4(sign + 4 * (long long)i);
  float wi, gxi = 0.f, gyi = 0.f, psii = 0.f;
  if (ORDER2) {
    const float4 r = ldf4(rec + 4 * (long long)i);
    wi = r.x; gxi = r.y; gyi = r.z; psii = r.w;
  } else {
    wi = ld(w + i);
  }
  float cv[3], q[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int o = comp(nb, j);
    const bool b = o < 0;
    const int f = -1 - o;
    const bool own = f2_own(fl, j);
    const bool rev = f2_rev(fl, j);
    const double2 Pj = j == 0 ? P0 : (j == 1 ? P1 : P2), Pk = j == 0 ? P1 : (j == 1 ? P2 : P0);
    const double2 Xa = rev ? Pk : Pj;
    const double2 Xb = rev ? Pj : Pk;
    const double fcx = 0.5 * (Xa.x + Xb.x), fcy = 0.5 * (Xa.y + Xb.y);
    float vo, gxo = 0.f, gyo = 0.f, pso = 0.f;
    double2 co;
    if (b) {
      vo = ghost(f);
      co = make_double2(ld(m.face_ghostcenter + 3 * f), ld(m.face_ghostcenter + 3 * f + 1));
    } else {
      if (ORDER2) {
        const float4 r = ldf4(rec + 4 * (long long)o);
        vo = r.x; gxo = r.y; gyo = r.z; pso = r.w;
      } else {
        vo = ld(w + o);
      }
      co = ldd2(m.cell_xy + 2 * o);
    }
    const float s = j == 0 ? s4.x : (j == 1 ? s4.y : s4.z);
    const bool take_me = (s >= 0.f) == own;
    // upwind value minus w_i
    float dsol;
    if (take_me) {
      dsol = ORDER2 ? psii * (gxi * (float)(fcx - ci.x) + gyi * (float)(fcy - ci.y)) : 0.f;
    } else if (b) {
      dsol = vo - wi;
    } else {
      dsol = ORDER2 ? (vo - wi) + pso * (gxo * (float)(fcx - co.x) + gyo * (float)(fcy - co.y)) : vo - wi;
    }
    const float F = s * dsol;
    cv[j] = own ? -F : F;
    if (DIFF) {
      float v = 0.f;
      if (!b || ld(bc.face_grad_on + f)) {
        const double2 v1 = own ? ci : co, v2 = own ? co : ci;
        const double air = 0.5 * ((Xb.x - Xa.x) * (v2.y - v1.y) + (v1.x - v2.x) * (Xb.y - Xa.y));
        double n0 = Xa.y - Xb.y, n1 = Xb.x - Xa.x;
        if (f2_flip(fl, j)) { n0 = -1 * n0; n1 = -1 * n1; }
        // Dxx n0 gx + Dyy n1 gy with manapy's diamond gradient, whose sum over f_1..f_4 of
        // (vi1 + vl) f_1 + (vl + vi2) f_2 + (vi2 + vr) f_3 + (vr + vi1) f_4 is, grouped by
        // value, (vi1 - vi2)(v1 - v2) + (vl - vr)(Xb - Xa): coefficients in FP64, the
        // differences of values in FP32
        const double r2a = 1. / (2 * air);
        const double gxk = p.Dxx * n0 * r2a, gyk = p.Dyy * n1 * r2a;
        const double a1 = gxk * (v1.y - v2.y) - gyk * (v1.x - v2.x);
        const double al = gxk * (Xb.y - Xa.y) - gyk * (Xb.x - Xa.x);
        const float ao = (float)(own ? -al : al);  // coefficient of (other side - this cell)
        const int ia = rev ? comp(vt, (j + 1) % 3) : comp(vt, j);
        const int ib = rev ? comp(vt, j) : comp(vt, (j + 1) % 3);
        const float vi1 = ld(wn + ia), vi2 = ld(wn + ib);
        v = (float)a1 * (vi1 - vi2) + ao * (vo - wi);
      }
      q[j] = own ? v : -v;
    }
  }
  // manapy's order: inner faces, boundary faces, then the diffusive terms
  const uint8_t code = ld(m.cell_order + i);
  CompSum res;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int sl = order_slot(code, k);
    if (pick3(nb.x, nb.y, nb.z, sl) >= 0) res.add(pick3(cv[0], cv[1], cv[2], sl));
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int sl = order_slot(code, k);
    if (pick3(nb.x, nb.y, nb.z, sl) < 0) res.add(pick3(cv[0], cv[1], cv[2], sl));
  }
  res.add(wi * s4.w);  // w_i times the cell's signed u.n sum
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 3; ++k) res.add(pick3(q[0], q[1], q[2], order_slot(code, k)));
  }
  const double dt = *dt_dev;
  float inc = (float)(dt / ld(m.cell_volume + i)) * res.value();
  if (src) inc = fmaf((float)dt, ld(src + i), inc);
  store_state(wi, inc, lo_in, w_out, lo_out, i);
}

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(MB_P2C_BLOCK, MB_P2C_MIN_BLOCKS)
    k_f2c_phase2(mb_mesh m, mb_bc bc, mb_advdiff_params p, const float *__restrict__ w, float *__restrict__ w_out,
                 const float *__restrict__ sign, const float *__restrict__ src, const double *__restrict__ dt_dev,
                 const float *__restrict__ rec, const float *__restrict__ wn, const float *__restrict__ lo_in,
                 float *__restrict__ lo_out) {
  f2c_phase2<ORDER2, DIFF>(m, bc, p, w, w_out, sign, src, dt_dev, rec, wn, lo_in, lo_out, blockIdx.x);
}

// ---------------------------------------------------------------- batches of triangle meshes
//
// Many independent meshes advance in the same two launches: block b of a launch
// belongs to item map[b] (blocks never straddle two meshes), which runs the
// single-mesh block body on its own tables.  A device step counter (the batch
// clock) selects each item's ping-pong buffer and skips items outside their
// [start_step, end_step) window, so a captured graph of the step stays valid
// while items come and go between replays.

__device__ __forceinline__ bool item_active(int t, int start, int end) { return t >= start && t < end; }

#ifndef MB_P1C_BATCH_MIN_BLOCKS
#define MB_P1C_BATCH_MIN_BLOCKS 8
#endif
template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock, MB_P1C_BATCH_MIN_BLOCKS)
    k_f2c_batch_phase1(const mb_advdiff_item *__restrict__ items, const int32_t *__restrict__ map,
                       const int32_t *__restrict__ clock) {
  const mb_advdiff_item &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (!item_active(t, it.start_step, it.end_step)) return;
  const float *w = it.w[(t - it.start_step) & 1];
  f2c_phase1<ORDER2, DIFF>(it.m, it.bc, w, it.cell_scratch, it.node_scratch, it.p1_cell_blocks,
                           (int)blockIdx.x - it.p1_begin);
}

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(kBlock, MB_P2C_BATCH_MIN_BLOCKS)
    k_f2c_batch_phase2(const mb_advdiff_item *__restrict__ items, const int32_t *__restrict__ map,
                       const int32_t *__restrict__ clock) {
  const mb_advdiff_item &it = items[map[blockIdx.x]];
  const int t = *clock;
  if (!item_active(t, it.start_step, it.end_step)) return;
  const int par = (t - it.start_step) & 1;
  f2c_phase2<ORDER2, DIFF>(it.m, it.bc, it.p, it.w[par], it.w[par ^ 1], it.sign_cf, it.src, it.dt_dev,
                           it.cell_scratch, it.node_scratch, it.lo[par], it.lo[par ^ 1],
                           (int)blockIdx.x - it.p2_begin);
}

__global__ void k_clock_tick(int32_t *clock) { *clock += 1; }

// ---------------------------------------------------------------- tetrahedra

#ifndef MB_P1C_3D_MIN_BLOCKS
#define MB_P1C_3D_MIN_BLOCKS 3
#endif

// record layout: float4 {w, gx, gy, gz} at rec[4i], psi at rec[4 nbcells + i]
// PRE: the moment matrix's cofactors and determinant come from m.cell_lsq ([nbcells][12],
// mb_lsq_matrix) and only the right-hand side is summed over the stencil
template <bool ORDER2, bool DIFF, bool PRE = false>
__global__ void __launch_bounds__(kBlock, MB_P1C_3D_MIN_BLOCKS)
    k_f3c_phase1(mb_mesh m, mb_bc bc, const float *__restrict__ w, float *__restrict__ rec, float *__restrict__ wn,
                 int ncb) {
  const GhostRuleF ghost = make_rule_f(m, bc, w);
  const int lane = threadIdx.x & 31;
  if (ORDER2 && (int)blockIdx.x < ncb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nbcells) return;
    const D3 c = ld3(m.cell_xy + 4 * i);
    const float wi = ld(w + i);
    double ixx = 0., iyy = 0., izz = 0., ixy = 0., ixz = 0., iyz = 0.;
    float jx = 0.f, jy = 0.f, jz = 0.f;
    const int sb = ld(m.lsq_sell_ptr + (i >> 5)), se = ld(m.lsq_sell_ptr + (i >> 5) + 1);
    const int L = (se - sb) >> 5;
    const int32_t *ix = m.lsq_sell_idx + sb + lane;
    auto acc = [&](const D3 &pc, float dw) {
      const double dx = pc.x - c.x, dy = pc.y - c.y, dz = pc.z - c.z;
      if (!PRE) {
        ixx += dx * dx; iyy += dy * dy; izz += dz * dz;
        ixy += dx * dy; ixz += dx * dz; iyz += dy * dz;
      }
      jx = fmaf((float)dx, dw, jx); jy = fmaf((float)dy, dw, jy); jz = fmaf((float)dz, dw, jz);
    };
    // batches of four neighbours: their indices, then their centres and values in flight
    // together, then the terms in stencil order (padding: the cell itself, exact zeros)
    int k = 0;
    for (; k + 4 <= L; k += 4) {
      int cc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { cc[u] = ld(ix + 32 * (k + u)); cc[u] = cc[u] < 0 ? i : cc[u]; }
      D3 pc[4];
      float wc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { pc[u] = ld3(m.cell_xy + 4 * cc[u]); wc[u] = ld(w + cc[u]); }
#pragma unroll
      for (int u = 0; u < 4; ++u) acc(pc[u], wc[u] - wi);
    }
    for (; k < L; ++k) {
      int cc = ld(ix + 32 * k);
      cc = cc < 0 ? i : cc;
      acc(ld3(m.cell_xy + 4 * cc), ld(w + cc) - wi);
    }
    const int gb = ld(m.ghostnid_ptr + i), ge = ld(m.ghostnid_ptr + i + 1);
    for (int k = gb; k < ge; ++k) {
      const int f = ld(m.ghostnid_idx + k);
      const double *gc = m.face_ghostcenter + 3 * f;
      acc(d3(ld(gc), ld(gc + 1), ld(gc + 2)), ghost(f) - wi);
    }
    // inverse moment matrix (symmetric cofactors / determinant), rounded once
    double c11, c12, c13, c22, c23, c33, dia;
    if (PRE) {
      double pad;
      ld4d(m.cell_lsq + 12 * (long long)i, c11, c12, c13, c22);
      ld4d(m.cell_lsq + 12 * (long long)i + 4, c23, c33, dia, pad);
    } else {
      dia = ixx * iyy * izz + 2. * ixy * ixz * iyz - ixx * (iyz * iyz) - iyy * (ixz * ixz) - izz * (ixy * ixy);
      c11 = iyy * izz - iyz * iyz; c12 = ixz * iyz - ixy * izz; c13 = ixy * iyz - ixz * iyy;
      c22 = ixx * izz - ixz * ixz; c23 = ixy * ixz - iyz * ixx; c33 = ixx * iyy - ixy * ixy;
    }
    const double rdia = 1. / dia;
    const float a11 = (float)(c11 * rdia), a12 = (float)(c12 * rdia), a13 = (float)(c13 * rdia);
    const float a22 = (float)(c22 * rdia), a23 = (float)(c23 * rdia), a33 = (float)(c33 * rdia);
    const float gx = a11 * jx + a12 * jy + a13 * jz;
    const float gy = a12 * jx + a22 * jy + a23 * jz;
    const float gz = a13 * jx + a23 * jy + a33 * jz;
    const int4 vt = ld4(m.cell_vtx + 4 * i);
    const int4 nb = ld4(m.cell_nbr + 4 * i);
    const uint32_t fl = ld(m.cell_flags + i);
    const D3 P[4] = {ld3(m.node_coord + 4 * vt.x), ld3(m.node_coord + 4 * vt.y), ld3(m.node_coord + 4 * vt.z),
                     ld3(m.node_coord + 4 * vt.w)};
    float wmax = wi, wmin = wi;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int o = comp(nb, j);
      const float bv = o < 0 ? ghost(-1 - o) : ld(w + o);
      wmax = fmaxp(wmax, bv);
      wmin = fminp(wmin, bv);
    }
    float ps = 1.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int d0, d1, d2;
      face_desc(fl, j, d0, d1, d2);
      const D3 fc = (1. / 3) * tet_face_sum(P, j, d2);
      const float delta = gx * (float)(fc.x - c.x) + gy * (float)(fc.y - c.y) + gz * (float)(fc.z - c.z);
      float psi_ij = 1.f;
      if (!(fabsf(delta) < 1e-10f)) {
        if (delta > 0.f) psi_ij = fminp(1.f, (wmax - wi) / delta);
        if (delta < 0.f) psi_ij = fminp(1.f, (wmin - wi) / delta);
      }
      ps = fminp(ps, psi_ij);
    }
    const uint64_t keep = l2_keep();
    st4_keep(rec + 4 * (long long)i, make_float4(wi, gx, gy, gz), keep);
    st1f_keep(rec + 4 * (long long)m.nbcells + i, ps, keep);
    return;
  }
  if (DIFF) node_value_f32(m, ghost, w, wn, (blockIdx.x - (ORDER2 ? ncb : 0)) * blockDim.x + threadIdx.x, lane);
}

// 128 x 7: 72 registers, 28 warps per SM (at 1.57M tetrahedra: 256 x 2, 90 registers, 13 %
// slower; 128 x 6 and 256 x 3, 80 registers, 2-3 % slower; 64 x 12 2 % slower)
#ifndef MB_P2C_3D_BLOCK
#define MB_P2C_3D_BLOCK 128
#endif
#ifndef MB_P2C_3D_MIN_BLOCKS
#define MB_P2C_3D_MIN_BLOCKS 7
#endif

template <bool ORDER2, bool DIFF>
__global__ void __launch_bounds__(MB_P2C_3D_BLOCK, MB_P2C_3D_MIN_BLOCKS)
    k_f3c_phase2(mb_mesh m, mb_bc bc, mb_advdiff_params p, const float *__restrict__ w, float *__restrict__ w_out,
                 const float *__restrict__ sign, const float *__restrict__ src, const double *__restrict__ dt_dev,
                 const float *__restrict__ rec, const float *__restrict__ wn, const float *__restrict__ lo_in,
                 float *__restrict__ lo_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const GhostRuleF ghost = make_rule_f(m, bc, w);
  const int4 vt = ld4(m.cell_vtx + 4 * i);
  const int4 nb = ld4(m.cell_nbr + 4 * i);
  const uint32_t fl = ld(m.cell_flags + i);
  const D3 ci = ld3(m.cell_xy + 4 * i);
  const float4 s4 = ldf4(sign + 4 * (long long)i);
  const long long nc = m.nbcells;
  float wi, gxi = 0.f, gyi = 0.f, gzi = 0.f, psii = 0.f;
  if (ORDER2) {
    const float4 r = ldf4(rec + 4 * (long long)i);
    wi = r.x; gxi = r.y; gyi = r.z; gzi = r.w;
    psii = ld(rec + 4 * nc + i);
  } else {
    wi = ld(w + i);
  }
  float cv[4], q[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int o = comp(nb, j);
    const bool b = o < 0;
    const int f = -1 - o;
    const bool own = (fl >> (6 * j)) & 1u;
    int d0, d1, d2;
    face_desc(fl, j, d0, d1, d2);
    // the face's vertices gathered by index instead of selected among four in registers
    const int g0 = comp(vt, d0), g1 = comp(vt, d1), g2 = comp(vt, d2);
    const D3 V0 = ld3(m.node_coord + 4 * g0), V1 = ld3(m.node_coord + 4 * g1), V2 = ld3(m.node_coord + 4 * g2);
    const D3 fc = (1. / 3) * ((V0 + V1) + V2);
    float vo, gxo = 0.f, gyo = 0.f, gzo = 0.f, pso = 0.f;
    D3 co;
    if (b) {
      vo = ghost(f);
      co = d3(ld(m.face_ghostcenter + 3 * f), ld(m.face_ghostcenter + 3 * f + 1), ld(m.face_ghostcenter + 3 * f + 2));
    } else {
      if (ORDER2) {
        const float4 r = ldf4(rec + 4 * (long long)o);
        vo = r.x; gxo = r.y; gyo = r.z; gzo = r.w;
        pso = ld(rec + 4 * nc + o);
      } else {
        vo = ld(w + o);
      }
      co = ld3(m.cell_xy + 4 * o);
    }
    const float s = pick4v(s4.x, s4.y, s4.z, s4.w, j);
    const bool take_me = (s >= 0.f) == own;
    float dsol;  // upwind value minus w_i
    if (take_me) {
      dsol = ORDER2 ? psii * (gxi * (float)(fc.x - ci.x) + gyi * (float)(fc.y - ci.y) + gzi * (float)(fc.z - ci.z))
                    : 0.f;
    } else if (b) {
      dsol = vo - wi;
    } else {
      dsol = ORDER2 ? (vo - wi) + pso * (gxo * (float)(fc.x - co.x) + gyo * (float)(fc.y - co.y) +
                                         gzo * (float)(fc.z - co.z))
                    : vo - wi;
    }
    const float F = s * dsol;
    cv[j] = own ? -F : F;
    if (DIFF) {
      float v = 0.f;
      if (!b || ld(bc.face_grad_on + f)) {
        const D3 Nd = 0.5 * cross(V1 - V0, V2 - V0);
        const D3 N = ((fl >> (6 * j + 5)) & 1u) ? (-1.0) * Nd : Nd;
        const bool swp = (fl >> (6 * j + 4)) & 1u;
        const D3 Q1 = V0, Q2 = swp ? V2 : V1, Q3 = swp ? V1 : V2;   // faces.nodeid order
        const int gi2 = swp ? g2 : g1, gi3 = swp ? g1 : g2;
        const D3 v1 = own ? ci : co, v2 = own ? co : ci;
        const double rair = 1. / dot(N, v2 - v1);
        // sum_d D_d g_d N_d = ca (V_A - V_C) + cb (V_B - V_D) + cr (V_R - V_L), with manapy's
        // f_1 = (Q3 - Q2) x (v1 - v2) / 2, f_2 = (Q1 - Q3) x (v1 - v2) / 2 folded into triple
        // products with t = (v1 - v2) x DN
        const D3 DN = d3(p.Dxx * N.x, p.Dyy * N.y, p.Dzz * N.z);
        const D3 t = cross(v1 - v2, DN);
        const float ca = (float)(0.5 * dot(Q3 - Q2, t) * rair), cb = (float)(0.5 * dot(Q1 - Q3, t) * rair),
                    cr = (float)(dot(DN, N) * rair);
        const float VA = ld(wn + g0), VB = ld(wn + gi2), VC = ld(wn + gi3);
        const float VL = own ? wi : vo, VR = own ? vo : wi;
        v = ca * (VA - VC) + cb * (VB - VC) + cr * (VR - VL);  // already differences
      }
      q[j] = own ? v : -v;
    }
  }
  const uint8_t code = ld(m.cell_order + i);
  CompSum res;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int sl = order_slot(code, k);
    if (pick4v(nb.x, nb.y, nb.z, nb.w, sl) >= 0) res.add(pick4v(cv[0], cv[1], cv[2], cv[3], sl));
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int sl = order_slot(code, k);
    if (pick4v(nb.x, nb.y, nb.z, nb.w, sl) < 0) res.add(pick4v(cv[0], cv[1], cv[2], cv[3], sl));
  }
  res.add(wi * ld(sign + 4 * nc + i));  // w_i times the cell's signed u.n sum
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 4; ++k) res.add(pick4v(q[0], q[1], q[2], q[3], order_slot(code, k)));
  }
  const double dt = *dt_dev;
  float inc = (float)(dt / ld(m.cell_volume + i)) * res.value();
  if (src) inc = fmaf((float)dt, ld(src + i), inc);
  store_state(wi, inc, lo_in, w_out, lo_out, i);
}

// ---- tetrahedra, the first phase by inclusion-exclusion (the FP64 step's k_f3_sums /
// k_f3_grad over the FP32 state; manapy/ast/functions3d.py:4-120 cell_gradient_3d and
// :364-408 barthlimiter_3d): each cell's least-squares right-hand side from the FP64
// sums of its 4 vertices and 6 edges and its face neighbours, instead of gathering its ~60
// stencil neighbours.  The sums are FP64 over the FP32 values: a cell's right-hand side is
// the difference of sums of undifferenced values, which FP32 sums would lose to
// cancellation.  Scratch after the 5 nbcells floats of records (rounded up to 8 floats):
// [nbnodes][4] vertex sums, then [nbedges][4] edge sums, doubles {P, Q}.

#ifndef MB_P1C_3D_SUMS_MIN_BLOCKS
#define MB_P1C_3D_SUMS_MIN_BLOCKS 4
#endif

inline bool f3c_sums_tables(const mb_mesh &m) {
  return m.cell_edges && m.edge_origin && m.edge_sell_ptr && m.edge_sell_idx && m.nbedges > 0 && m.cell_lsq &&
         m.n2c_sum_ptr && m.n2c_sum_idx && m.n2c_sum_alpha;
}
inline long long f3c_rec_floats(const mb_mesh &m) { return (5LL * m.nbcells + 7) & ~7LL; }

// vertex blocks [0, nnb): the vertex's sums and (DIFF) its centre->vertex value, FP64 weights
// rounded once; edge blocks: the edge's sums
template <bool DIFF>
__global__ void __launch_bounds__(kBlock) k_f3c_sums(mb_mesh m, mb_bc bc, const float *__restrict__ w,
                                                     double *__restrict__ nrec, double *__restrict__ erec,
                                                     float *__restrict__ wn, int nnb) {
  const int lane = threadIdx.x & 31;
  const uint64_t pst = l2_stream();
  double px = 0., py = 0., pz = 0., q = 0.;
  int sb, se;
  const int32_t *idx;
  D3 X;
  const bool vertex = (int)blockIdx.x < nnb;
  const int n = (vertex ? blockIdx.x : blockIdx.x - nnb) * blockDim.x + threadIdx.x;
  if (vertex) {
    if (n >= m.nbnodes) return;
    X = ld3(m.node_coord + 4 * (long long)n);
    sb = ld(m.n2c_sum_ptr + (n >> 5)); se = ld(m.n2c_sum_ptr + (n >> 5) + 1);
    idx = m.n2c_sum_idx;
  } else {
    if (n >= m.nbedges) return;
    X = ld3(m.node_coord + 4 * (long long)ld(m.edge_origin + n));
    sb = ld(m.edge_sell_ptr + (n >> 5)); se = ld(m.edge_sell_ptr + (n >> 5) + 1);
    idx = m.edge_sell_idx;
  }
  double acc = 0.;
  for (int k = sb + lane; k < se; k += 32) {
    const int cc = ld1_stream(idx + k, pst);
    if (cc < 0) continue;  // empty slot
    const D3 x = ld3(m.cell_xy + 4 * (long long)cc);
    const double wc = ld(w + cc);
    if (DIFF && vertex) acc += ldd_stream(m.n2c_sum_alpha + k, pst) * wc;
    px += (x.x - X.x) * wc; py += (x.y - X.y) * wc; pz += (x.z - X.z) * wc;
    q += wc;
  }
  if (vertex) {
    if (DIFF) {
      const GhostRuleF ghost = make_rule_f(m, bc, w);
      const int gb = ld(m.n2g_ptr + n), ge = ld(m.n2g_ptr + n + 1);
      for (int k = gb; k < ge; ++k) acc += ld(m.n2g_alpha + k) * (double)ghost(ld(m.n2g_idx + k));
      st1f_keep(wn + n, (float)acc, l2_keep());
    }
    st4_keep(nrec + 4 * (long long)n, px, py, pz, q, l2_keep());
  } else {
    st4_keep(erec + 4 * (long long)n, px, py, pz, q, l2_keep());
  }
}

// cell pass: the gradient from the vertex, edge and face-neighbour sums (FP64, rounded once),
// the Barth limiter in FP32 as k_f3c_phase1; the same records as k_f3c_phase1
__global__ void __launch_bounds__(kBlock, MB_P1C_3D_SUMS_MIN_BLOCKS)
    k_f3c_grad(mb_mesh m, mb_bc bc, const float *__restrict__ w, float *__restrict__ rec,
               const double *__restrict__ nrec, const double *__restrict__ erec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const GhostRuleF ghost = make_rule_f(m, bc, w);
  const D3 c = ld3(m.cell_xy + 4 * (long long)i);
  const float wf = ld(w + i);
  const double wi = wf;
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
  float wmax = wf, wmin = wf;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int o = comp(nb, j);
    float bv;
    if (o >= 0) {
      const D3 x = ld3(m.cell_xy + 4 * (long long)o);
      bv = ld(w + o);
      const double b = bv;
      sx += (x.x - c.x) * b; sy += (x.y - c.y) * b; sz += (x.z - c.z) * b;
    } else {
      bv = ghost(-1 - o);
    }
    wmax = fmaxp(wmax, bv);
    wmin = fminp(wmin, bv);
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
    const double dw = (double)ghost(f) - wi;
    jx += (ld(gc) - c.x) * dw; jy += (ld(gc + 1) - c.y) * dw; jz += (ld(gc + 2) - c.z) * dw;
  }
  const double rdia = 1. / dia;
  const float gx = (float)((a0 * jx + a1 * jy + a2 * jz) * rdia);
  const float gy = (float)((a1 * jx + a3 * jy + a4 * jz) * rdia);
  const float gz = (float)((a2 * jx + a4 * jy + a5 * jz) * rdia);
  const uint32_t fl = ld(m.cell_flags + i);
  float ps = 1.f;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int d0, d1, d2;
    face_desc(fl, j, d0, d1, d2);
    const D3 fc = (1. / 3) * tet_face_sum(P, j, d2);
    const float delta = gx * (float)(fc.x - c.x) + gy * (float)(fc.y - c.y) + gz * (float)(fc.z - c.z);
    float psi_ij = 1.f;
    if (!(fabsf(delta) < 1e-10f)) {
      if (delta > 0.f) psi_ij = fminp(1.f, (wmax - wf) / delta);
      if (delta < 0.f) psi_ij = fminp(1.f, (wmin - wf) / delta);
    }
    ps = fminp(ps, psi_ij);
  }
  const uint64_t keep = l2_keep();
  st4_keep(rec + 4 * (long long)i, make_float4(wf, gx, gy, gz), keep);
  st1f_keep(rec + 4 * (long long)m.nbcells + i, ps, keep);
}

// FP32 u.n per cell face and, in FP64 then rounded, the cell's signed sum of them
// (minus for the faces the cell owns, which the residual subtracts)
__global__ void __launch_bounds__(kBlock) k_sign_f32c(mb_mesh m, const double *__restrict__ s64,
                                                      float *__restrict__ s32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  const uint32_t fl = ld(m.cell_flags + i);
  double div = 0.;
  for (int j = 0; j < m.nlf; ++j) {
    const double s = ld(s64 + 4 * (long long)i + j);
    const bool own = m.dim == 2 ? f2_own(fl, j) : ((fl >> (6 * j)) & 1u);
    div += own ? -s : s;
    s32[4 * (long long)i + j] = (float)s;
  }
  if (m.dim == 2)
    s32[4 * (long long)i + 3] = (float)div;
  else
    s32[4 * (long long)m.nbcells + i] = (float)div;
}

template <bool O2, bool DF>
int launch_step_f32c(const mb_mesh &m, const mb_bc &bc, const mb_advdiff_params &p, const float *w_in, float *w_out,
                     const float *sign, const float *src, const double *dt, float *cs, float *wn, const float *lo_in,
                     float *lo_out, cudaStream_t st) {
  const int ncb = O2 ? ceil_div(m.nbcells, kBlock) : 0;
  const int nnb = DF ? ceil_div(m.nbnodes, kBlock) : 0;
  if (m.dim == 2) {
    if (ncb + nnb > 0) k_f2c_phase1<O2, DF><<<ncb + nnb, kBlock, 0, st>>>(m, bc, w_in, cs, wn, ncb);
    k_f2c_phase2<O2, DF><<<ceil_div(m.nbcells, MB_P2C_BLOCK), MB_P2C_BLOCK, 0, st>>>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn,
                                                                           lo_in, lo_out);
  } else {
    if (O2 && f3c_sums_tables(m)) {
      // the sums path: records, then the vertex and edge sums (32-byte aligned doubles)
      if ((reinterpret_cast<uintptr_t>(cs) & 31) != 0 || (reinterpret_cast<uintptr_t>(m.cell_lsq) & 31) != 0)
        return MB_EINVAL;
      double *nrec = reinterpret_cast<double *>(cs + f3c_rec_floats(m)), *erec = nrec + 4 * (long long)m.nbnodes;
      const int nvb = ceil_div(m.nbnodes, kBlock), neb = ceil_div(m.nbedges, kBlock);
      k_f3c_sums<DF><<<nvb + neb, kBlock, 0, st>>>(m, bc, w_in, nrec, erec, wn, nvb);
      k_f3c_grad<<<ceil_div(m.nbcells, kBlock), kBlock, 0, st>>>(m, bc, w_in, cs, nrec, erec);
    } else if (ncb + nnb > 0) {
      if (O2 && m.cell_lsq)
        k_f3c_phase1<O2, DF, true><<<ncb + nnb, kBlock, 0, st>>>(m, bc, w_in, cs, wn, ncb);
      else
        k_f3c_phase1<O2, DF, false><<<ncb + nnb, kBlock, 0, st>>>(m, bc, w_in, cs, wn, ncb);
    }
    k_f3c_phase2<O2, DF><<<ceil_div(m.nbcells, MB_P2C_3D_BLOCK), MB_P2C_3D_BLOCK, 0, st>>>(m, bc, p, w_in, w_out, sign, src, dt, cs, wn,
                                                                           lo_in, lo_out);
  }
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

}  // namespace mb

using namespace mb;

extern "C" int mb_advdiff_step_f32c(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                                    const float *w_in, float *w_out, const float *lo_in, float *lo_out,
                                    const float *sign_cf, const float *src, const double *dt_dev, float *cell_scratch,
                                    float *node_scratch, void *stream) {
  MB_NVTX();
  if (!m || !bc || !p || !w_in || !w_out || !sign_cf || !dt_dev || w_in == w_out) return MB_EINVAL;
  if (m->dim != 2 && m->dim != 3) return MB_EINVAL;
  if ((lo_in == nullptr) != (lo_out == nullptr) || (lo_in && lo_in == lo_out)) return MB_EINVAL;
  if (!(m->cell_vtx && m->cell_nbr && m->cell_flags && m->node_coord && m->cell_xy && m->lsq_sell_ptr &&
        m->lsq_sell_idx && m->n2c_sell_ptr && m->n2c_sell_idx && m->n2c_sell_alpha_f32))
    return MB_EINVAL;
  const bool o2 = p->order == 2, df = p->diffusion != 0;
  if (p->order != 1 && !o2) return MB_EINVAL;
  if ((o2 && !cell_scratch) || (df && !node_scratch) || (df && !bc->face_grad_on)) return MB_EINVAL;
#if MB_LD256
  // 256-bit loads of the [n][4] centre and vertex rows of a tetrahedral mesh
  if (m->dim == 3 && (((reinterpret_cast<uintptr_t>(m->cell_xy) | reinterpret_cast<uintptr_t>(m->node_coord)) & 31) != 0))
    return MB_EINVAL;
#endif
  cudaStream_t st = (cudaStream_t)stream;
#define MB_F32C(O, D) \
  return launch_step_f32c<O, D>(*m, *bc, *p, w_in, w_out, sign_cf, src, dt_dev, cell_scratch, node_scratch, lo_in, \
                                lo_out, st)
  if (o2 && df) MB_F32C(true, true);
  if (o2) MB_F32C(true, false);
  if (df) MB_F32C(false, true);
  MB_F32C(false, false);
#undef MB_F32C
}

extern "C" int mb_advdiff_batch_step_f32c(const mb_advdiff_item *items, const int32_t *p1_map, int32_t p1_blocks,
                                          const int32_t *p2_map, int32_t p2_blocks, int32_t order,
                                          int32_t diffusion, int32_t *clock, void *stream) {
  MB_NVTX();
  if (!items || !p2_map || !clock || p2_blocks <= 0 || p1_blocks < 0 || (order != 1 && order != 2)) return MB_EINVAL;
  const bool o2 = order == 2, df = diffusion != 0;
  if ((o2 || df) && (!p1_map || p1_blocks <= 0)) return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (o2 && df) {
    k_f2c_batch_phase1<true, true><<<p1_blocks, kBlock, 0, st>>>(items, p1_map, clock);
    k_f2c_batch_phase2<true, true><<<p2_blocks, kBlock, 0, st>>>(items, p2_map, clock);
  } else if (o2) {
    k_f2c_batch_phase1<true, false><<<p1_blocks, kBlock, 0, st>>>(items, p1_map, clock);
    k_f2c_batch_phase2<true, false><<<p2_blocks, kBlock, 0, st>>>(items, p2_map, clock);
  } else if (df) {
    k_f2c_batch_phase1<false, true><<<p1_blocks, kBlock, 0, st>>>(items, p1_map, clock);
    k_f2c_batch_phase2<false, true><<<p2_blocks, kBlock, 0, st>>>(items, p2_map, clock);
  } else {
    k_f2c_batch_phase2<false, false><<<p2_blocks, kBlock, 0, st>>>(items, p2_map, clock);
  }
  k_clock_tick<<<1, 1, 0, st>>>(clock);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

extern "C" int mb_cell_face_sign_f32c(const mb_mesh *m, const double *sign_cf, float *sign_f32, void *stream) {
  MB_NVTX();
  if (!m || !sign_cf || !sign_f32 || !m->cell_flags || (m->dim != 2 && m->dim != 3)) return MB_EINVAL;
  k_sign_f32c<<<ceil_div(m->nbcells, kBlock), kBlock, 0, (cudaStream_t)stream>>>(*m, sign_cf, sign_f32);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}
