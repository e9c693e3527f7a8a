// Euler equations, 2D, first-order Rusanov scheme (manapy/solvers/euler/fvm_utils2d.py).
//
// manapy ships these as kernels without a solver class; each entry point below
// replaces one of them and keeps its argument meaning:
//   Rusanov face flux         compute_flux_euler_2d_rusanov     fvm_utils2d.py:1248-1292
//   residuals                 explicitscheme_euler_2d_rusanov   fvm_utils2d.py:1490-1611
//   per-cell CFL time step    time_step_euler_2d                fvm_utils2d.py:1083-1102
//   update + pressure         update_euler_2d_fvc               fvm_utils2d.py:1687-1696
//   Neumann ghosts            ghost_value_Neumann               fvm_utils2d.py:592-648
// plus a fused step (face fluxes, then update + next dt: two launches per step) for meshes
// whose boundary faces all carry manapy's Neumann rule.
//
// The residual kernels gather per cell: each face flux is evaluated by both of its cells
// from the same (left, right) states, and a cell adds its faces in ascending face id, the
// order of manapy's face loop.  This file is compiled without multiply-add contraction, so
// every operation rounds as manapy's code does and the results are bit-identical to it.
// manapy's flux reads the left cell's rhov in the right normal momentum
// (qr = rhour n0 + rhovl n1); reproduced.
#include "fv_common.cuh"
#include "fv_compact.cuh"

namespace mb {

struct EulerQ {
  const double *rho, *P, *rhou, *rhov, *rhoE;
};

struct EulerW {
  double *rho, *P, *rhou, *rhov, *rhoE;
};

__device__ __forceinline__ double dmax3(double a, double b, double c) {
  // Python's max(a, b, c): the first of the largest
  double m = a;
  if (b > m) m = b;
  if (c > m) m = c;
  return m;
}

__device__ __forceinline__ void rusanov(double rhol, double Pl, double rhoul, double rhovl, double rhoEl, double rhor,
                                        double Pr, double rhour, double rhovr, double rhoEr, double n0, double n1,
                                        double mesure, double gamma, double F[4]) {
  const double ql = (rhoul * n0 + rhovl * n1);
  const double qr = (rhour * n0 + rhovl * n1);
  const double cl = sqrt(gamma * Pl / rhol);
  const double cr = sqrt(gamma * Pr / rhor);
  const double fl_rho = (rhoul * n0 + rhovl * n1);
  const double fl_rhou = ((rhoul * rhoul / rhol + Pl) * n0 + (rhoul * rhovl / rhol) * n1);
  const double fl_rhov = ((rhovl * rhoul / rhol) * n0 + (rhovl * rhovl / rhol + Pl) * n1);
  const double fl_rhoE = (rhoul / rhol * (rhoEl + Pl) * n0 + rhovl / rhol * (rhoEl + Pl) * n1);
  const double fr_rho = (rhour * n0 + rhovr * n1);
  const double fr_rhou = ((rhour * rhour / rhor + Pr) * n0 + (rhour * rhovr / rhor) * n1);
  const double fr_rhov = ((rhovr * rhour / rhor) * n0 + (rhovr * rhovr / rhor + Pr) * n1);
  const double fr_rhoE = (rhour / rhor * (rhoEr + Pr) * n0 + rhovr / rhor * (rhoEr + Pr) * n1);
  const double Ll = dmax3(fabs(ql / rhol - cl), fabs(ql / rhol), fabs(ql / rhol + cl));
  const double Lr = dmax3(fabs(qr / rhor - cr), fabs(qr / rhor), fabs(qr / rhor + cr));
  const double S = Ll > Lr ? Ll : Lr;
  F[0] = (0.5 * (fl_rho + fr_rho) - 0.5 * S * (rhor - rhol)) * mesure;
  F[1] = (0.5 * (fl_rhou + fr_rhou) - 0.5 * S * (rhour - rhoul)) * mesure;
  F[2] = (0.5 * (fl_rhov + fr_rhov) - 0.5 * S * (rhovr - rhovl)) * mesure;
  F[3] = (0.5 * (fl_rhoE + fr_rhoE) - 0.5 * S * (rhoEr - rhoEl)) * mesure;
}

// the three faces of cell i in its own order (cells.faceid): ids, raw normals, measures
__device__ __forceinline__ void cell_face_geom(const mb_mesh &m, int i, int f[3], double n0[3], double n1[3],
                                               double mes[3]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    f[j] = ld(m.cell_faces + 4 * i + j);
    n0[j] = ld(m.face_normal + 3 * f[j]);
    n1[j] = ld(m.face_normal + 3 * f[j] + 1);
    mes[j] = ld(m.face_mesure + f[j]);
  }
}

// time_step_euler_2d's per-cell dt, faces in the cell's own order
__device__ __forceinline__ double euler_cell_dt(double rho, double P, double rhou, double rhov, const double n0[3],
                                                const double n1[3], const double mes[3], double vol, double cfl,
                                                double gamma) {
  const double velson = sqrt(gamma * fabs(P / rho));
  double lam = 0.;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double u_n = fabs((rhou * n0[j] + rhov * n1[j]) / rho) / sqrt(n0[j] * n0[j] + n1[j] * n1[j]);
    lam += (u_n + velson) * mes[j];
  }
  return cfl * vol / lam;
}

__global__ void __launch_bounds__(kBlock) k_euler_rusanov(mb_mesh m, EulerQ q, EulerQ g, double *r0, double *r1,
                                                          double *r2, double *r3, double gamma) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    const uint8_t code = ld(m.cell_order + i);
    double rez[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int f = ld(m.cell_faces + 4 * i + order_slot(code, k));
      const int c0 = ld(m.face_cellid + 2 * f);
      const double mes = ld(m.face_mesure + f);
      const double n0 = ld(m.face_normal + 3 * f) / mes, n1 = ld(m.face_normal + 3 * f + 1) / mes;
      double rr, Pr, rur, rvr, rEr;
      if (ld(m.face_name + f) == 0) {
        const int c1 = ld(m.face_cellid + 2 * f + 1);
        rr = ld(q.rho + c1); Pr = ld(q.P + c1); rur = ld(q.rhou + c1); rvr = ld(q.rhov + c1); rEr = ld(q.rhoE + c1);
      } else {
        rr = ld(g.rho + f); Pr = ld(g.P + f); rur = ld(g.rhou + f); rvr = ld(g.rhov + f); rEr = ld(g.rhoE + f);
      }
      double F[4];
      rusanov(ld(q.rho + c0), ld(q.P + c0), ld(q.rhou + c0), ld(q.rhov + c0), ld(q.rhoE + c0), rr, Pr, rur, rvr, rEr,
              n0, n1, mes, gamma, F);
      const bool left = c0 == i;
#pragma unroll
      for (int c = 0; c < 4; ++c) rez[c] = left ? rez[c] - F[c] : rez[c] + F[c];
    }
    r0[i] = rez[0]; r1[i] = rez[1]; r2[i] = rez[2]; r3[i] = rez[3];
  }
}

__global__ void __launch_bounds__(kBlock) k_time_step_euler(mb_mesh m, EulerQ q, double cfl, double gamma,
                                                            double *dt_c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nbcells; i += gridDim.x * blockDim.x) {
    int f[3];
    double n0[3], n1[3], mes[3];
    cell_face_geom(m, i, f, n0, n1, mes);
    dt_c[i] = euler_cell_dt(ld(q.rho + i), ld(q.P + i), ld(q.rhou + i), ld(q.rhov + i), n0, n1, mes,
                            ld(m.cell_volume + i), cfl, gamma);
  }
}

__global__ void __launch_bounds__(kBlock) k_update_euler(int n, EulerW q, const double *r0, const double *r1,
                                                         const double *r2, const double *r3, double gamma,
                                                         double dt, const double *vol) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = ld(vol + i);
    const double rho = q.rho[i] + dt * (ld(r0 + i) / v);
    const double rhou = q.rhou[i] + dt * (ld(r1 + i) / v);
    const double rhov = q.rhov[i] + dt * (ld(r2 + i) / v);
    const double rhoE = q.rhoE[i] + dt * (ld(r3 + i) / v);
    q.rho[i] = rho; q.rhou[i] = rhou; q.rhov[i] = rhov; q.rhoE[i] = rhoE;
    q.P[i] = (gamma - 1) * (rhoE - 0.5 * (rhou * rhou + rhov * rhov) / rho);
  }
}

__global__ void __launch_bounds__(kBlock) k_ghost_euler_neumann(mb_mesh m, EulerQ q, EulerW g, double *ug,
                                                                double *vg) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nbfaces; f += gridDim.x * blockDim.x) {
    const int nm = ld(m.face_name + f);
    if (nm < 1 || nm > 4) continue;
    const int c = ld(m.face_cellid + 2 * f);
    const double rho = ld(q.rho + c), rhou = ld(q.rhou + c), rhov = ld(q.rhov + c);
    g.rho[f] = rho; g.rhou[f] = rhou; g.rhov[f] = rhov; g.rhoE[f] = ld(q.rhoE + c); g.P[f] = ld(q.P + c);
    ug[f] = rhou / rho;
    vg[f] = rhov / rho;
  }
}

// ---- fused step: face fluxes, then update + the next step's dt in one pass over the cells ----
//
// Two launches per step.  k_euler_face evaluates every face flux once (faces in device
// order, Neumann ghost = the cell's own state on boundary faces) into face_flux (four
// doubles per face).  k_euler_cell adds its three fluxes in ascending face id with manapy's
// signs, updates the state and min-reduces the dt of the new state.  Evaluating each flux
// once instead of from both cells halves the FP64 division work that bounds the
// single-pass form, at the price of 32 bytes per face written and read back.
//
// Both kernels read two static tables built once per mesh (mb_euler_tables_2d): a 32-byte
// record per face {n0, n1, mesure, (c0, c1)} -- one 256-bit load where four arrays would
// take five loads -- and a byte per cell whose bit j says the cell is the left cell
// (faces.cellid[f][0]) of its local face j.  Flux records are read and written as one
// 256-bit access each.
//
// dt ring of three device slots: the step of time index t reads slot t%3 (the dt of its
// input state, complete since the previous step), min-reduces the dt of its output state
// into slot (t+1)%3, and resets slot (t+2)%3 for the step after.

constexpr double kNoDt = 1e300;

#ifndef MB_EULER_MIN_BLOCKS
#define MB_EULER_MIN_BLOCKS 4
#endif

// the two cells of a face in the fourth double of its record (bit pattern only; never used
// in arithmetic); c1 = -1 on boundary faces
__device__ __forceinline__ double pack_cells(int c0, int c1) {
  return __longlong_as_double((long long)(((unsigned long long)(unsigned)c1 << 32) | (unsigned)c0));
}
__device__ __forceinline__ void unpack_cells(double v, int &c0, int &c1) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  c0 = (int)(unsigned)(u & 0xffffffffull);
  c1 = (int)(unsigned)(u >> 32);
}

__device__ __forceinline__ void st4d(double *p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

__global__ void __launch_bounds__(kBlock) k_euler_face_rec(mb_mesh m, double *rec) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nbfaces) return;
  const int c0 = ld(m.face_cellid + 2 * f);
  const int c1 = ld(m.face_name + f) == 0 ? ld(m.face_cellid + 2 * f + 1) : -1;
  st4d(rec + 4 * (long long)f, ld(m.face_normal + 3 * f), ld(m.face_normal + 3 * f + 1), ld(m.face_mesure + f),
       pack_cells(c0, c1));
}

__global__ void __launch_bounds__(kBlock) k_euler_cell_left(mb_mesh m, uint8_t *left) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nbcells) return;
  unsigned bits = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) bits |= (ld(m.face_cellid + 2 * ld(m.cell_faces + 4 * i + j)) == i ? 1u : 0u) << j;
  left[i] = (uint8_t)bits;
}

__global__ void __launch_bounds__(kBlock) k_euler_face(int nf, EulerQ q, double gamma, const double *rec,
                                                       double *ff) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double r0, r1, mes, cb;
  ld4d(rec + 4 * (long long)f, r0, r1, mes, cb);
  int c0, c1;
  unpack_cells(cb, c0, c1);
  const double nx = r0 / mes, ny = r1 / mes;
  const double rl = ld(q.rho + c0), Pl = ld(q.P + c0), ul = ld(q.rhou + c0), vl = ld(q.rhov + c0),
               El = ld(q.rhoE + c0);
  double F[4];
  if (c1 >= 0) {
    rusanov(rl, Pl, ul, vl, El, ld(q.rho + c1), ld(q.P + c1), ld(q.rhou + c1), ld(q.rhov + c1), ld(q.rhoE + c1), nx,
            ny, mes, gamma, F);
  } else {
    rusanov(rl, Pl, ul, vl, El, rl, Pl, ul, vl, El, nx, ny, mes, gamma, F);
  }
  st4d(ff + 4 * (long long)f, F[0], F[1], F[2], F[3]);
}

__global__ void __launch_bounds__(kBlock, MB_EULER_MIN_BLOCKS) k_euler_cell(mb_mesh m, EulerQ q, EulerW out,
                                                                            const double *rec,
                                                                            const uint8_t *cell_left,
                                                                            const double *ff, double cfl,
                                                                            double gamma, double *ring, int a, int b,
                                                                            int c, double *time) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = ld(ring + a);
  double dtc = kNoDt;
  if (i < m.nbcells) {
    const int4 fc = ld4(m.cell_faces + 4 * i);
    const int f[3] = {fc.x, fc.y, fc.z};
    double n0[3], n1[3], mes[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double unused;
      ld4d(rec + 4 * (long long)f[j], n0[j], n1[j], mes[j], unused);
    }
    const uint8_t code = ld(m.cell_order + i);
    const unsigned lb = ld(cell_left + i);
    double rez[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int s = order_slot(code, k);
      const int fk = pick3(f[0], f[1], f[2], s);
      const bool left = (lb >> s) & 1u;
      double F[4];
      ld4d(ff + 4 * (long long)fk, F[0], F[1], F[2], F[3]);
#pragma unroll
      for (int e = 0; e < 4; ++e) rez[e] = left ? rez[e] - F[e] : rez[e] + F[e];
    }
    const double v = ld(m.cell_volume + i);
    const double r1 = ld(q.rho + i) + dt * (rez[0] / v);
    const double u1 = ld(q.rhou + i) + dt * (rez[1] / v);
    const double w1 = ld(q.rhov + i) + dt * (rez[2] / v);
    const double E1 = ld(q.rhoE + i) + dt * (rez[3] / v);
    const double P1 = (gamma - 1) * (E1 - 0.5 * (u1 * u1 + w1 * w1) / r1);
    out.rho[i] = r1; out.P[i] = P1; out.rhou[i] = u1; out.rhov[i] = w1; out.rhoE[i] = E1;
    dtc = euler_cell_dt(r1, P1, u1, w1, n0, n1, mes, v, cfl, gamma);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ring[c] = kNoDt;
    if (time) *time += dt;
  }
  const double best = block_min(dtc);
  if (threadIdx.x == 0 && best < kNoDt) atomic_min_pos(ring + b, best);
}

__global__ void k_euler_ring_reset(double *ring) {
  if (threadIdx.x < 3) ring[threadIdx.x] = kNoDt;
}

__global__ void __launch_bounds__(kBlock) k_euler_dt(mb_mesh m, EulerQ q, double cfl, double gamma, double *slot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = kNoDt;
  if (i < m.nbcells) {
    int f[3];
    double n0[3], n1[3], mes[3];
    cell_face_geom(m, i, f, n0, n1, mes);
    dtc = euler_cell_dt(ld(q.rho + i), ld(q.P + i), ld(q.rhou + i), ld(q.rhov + i), n0, n1, mes,
                        ld(m.cell_volume + i), cfl, gamma);
  }
  const double best = block_min(dtc);
  if (threadIdx.x == 0 && best < kNoDt) atomic_min_pos(slot, best);
}

inline int grid_e(long long n) {
  const long long g = (n + kBlock - 1) / kBlock;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace mb

using namespace mb;

static bool euler_mesh_ok(const mb_mesh *m) {
  return m && m->dim == 2 && m->nlf == 3 && m->nbcells > 0 && m->cell_faces && m->face_cellid && m->face_name &&
         m->face_normal && m->face_mesure && m->cell_order && m->cell_volume;
}

static bool q_ok(const double *const q[5]) {
  if (!q) return false;
  for (int k = 0; k < 5; ++k)
    if (!q[k]) return false;
  return true;
}

extern "C" {

int mb_euler_rusanov_2d(const mb_mesh *m, const double *const q[5], const double *const g[5], double *const rez[4],
                        double gamma, void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !q_ok(q) || !q_ok(g) || !rez) return MB_EINVAL;
  for (int k = 0; k < 4; ++k)
    if (!rez[k]) return MB_EINVAL;
  EulerQ qq{q[0], q[1], q[2], q[3], q[4]}, gg{g[0], g[1], g[2], g[3], g[4]};
  k_euler_rusanov<<<grid_e(m->nbcells), kBlock, 0, (cudaStream_t)stream>>>(*m, qq, gg, rez[0], rez[1], rez[2],
                                                                            rez[3], gamma);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_time_step_euler_2d(const mb_mesh *m, const double *const q[5], double cfl, double gamma, double *dt_c,
                          void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !q_ok(q) || !dt_c) return MB_EINVAL;
  EulerQ qq{q[0], q[1], q[2], q[3], q[4]};
  k_time_step_euler<<<grid_e(m->nbcells), kBlock, 0, (cudaStream_t)stream>>>(*m, qq, cfl, gamma, dt_c);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_update_euler_2d(const mb_mesh *m, double *const q[5], const double *const rez[4], double gamma, double dt,
                       void *stream) {
  MB_NVTX();
  if (!m || !m->cell_volume || m->nbcells <= 0 || !q || !rez) return MB_EINVAL;
  for (int k = 0; k < 5; ++k)
    if (!q[k] || (k < 4 && !rez[k])) return MB_EINVAL;
  EulerW qq{q[0], q[1], q[2], q[3], q[4]};
  k_update_euler<<<grid_e(m->nbcells), kBlock, 0, (cudaStream_t)stream>>>(m->nbcells, qq, rez[0], rez[1], rez[2],
                                                                           rez[3], gamma, dt, m->cell_volume);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_ghost_euler_neumann_2d(const mb_mesh *m, const double *const q[5], double *const g[5], double *ug, double *vg,
                              void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !q_ok(q) || !g || !ug || !vg || m->nbfaces <= 0) return MB_EINVAL;
  for (int k = 0; k < 5; ++k)
    if (!g[k]) return MB_EINVAL;
  EulerQ qq{q[0], q[1], q[2], q[3], q[4]};
  EulerW gg{g[0], g[1], g[2], g[3], g[4]};
  k_ghost_euler_neumann<<<grid_e(m->nbfaces), kBlock, 0, (cudaStream_t)stream>>>(*m, qq, gg, ug, vg);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_euler_dt_2d(const mb_mesh *m, const double *const q[5], double cfl, double gamma, double *ring, int t,
                   void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !q_ok(q) || !ring || t < 0) return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  EulerQ qq{q[0], q[1], q[2], q[3], q[4]};
  k_euler_ring_reset<<<1, 32, 0, st>>>(ring);
  k_euler_dt<<<(m->nbcells + kBlock - 1) / kBlock, kBlock, 0, st>>>(*m, qq, cfl, gamma, ring + t % 3);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

static bool a32(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 31) == 0; }

int mb_euler_tables_2d(const mb_mesh *m, double *face_rec, uint8_t *cell_left, void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !face_rec || !cell_left || m->nbfaces <= 0 || !a32(face_rec)) return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  k_euler_face_rec<<<(m->nbfaces + kBlock - 1) / kBlock, kBlock, 0, st>>>(*m, face_rec);
  k_euler_cell_left<<<(m->nbcells + kBlock - 1) / kBlock, kBlock, 0, st>>>(*m, cell_left);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

int mb_euler_step_2d(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl,
                     double gamma, const double *face_rec, const uint8_t *cell_left, double *face_flux, double *ring,
                     int t, double *time, void *stream) {
  MB_NVTX();
  if (!euler_mesh_ok(m) || !q_ok(q_in) || !q_out || !ring || !face_flux || !face_rec || !cell_left || t < 0 ||
      m->nbfaces <= 0)
    return MB_EINVAL;
  if (!a32(face_flux) || !a32(face_rec)) return MB_EINVAL;
  for (int k = 0; k < 5; ++k)
    if (!q_out[k] || q_out[k] == q_in[k]) return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  EulerQ qq{q_in[0], q_in[1], q_in[2], q_in[3], q_in[4]};
  EulerW oo{q_out[0], q_out[1], q_out[2], q_out[3], q_out[4]};
  k_euler_face<<<(m->nbfaces + kBlock - 1) / kBlock, kBlock, 0, st>>>(m->nbfaces, qq, gamma, face_rec, face_flux);
  k_euler_cell<<<(m->nbcells + kBlock - 1) / kBlock, kBlock, 0, st>>>(*m, qq, oo, face_rec, cell_left, face_flux,
                                                                      cfl, gamma, ring, t % 3, (t + 1) % 3,
                                                                      (t + 2) % 3, time);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

}  // extern "C"
