/*
 * manapy_b200 -- C ABI of the B200 (sm_100a) explicit finite-volume step.
 *
 * Every entry point takes device pointers, plain sizes and a CUDA stream
 * (cudaStream_t passed as void*), returns 0 on success or a negative MB_E*
 * code, and never allocates device memory.  Field arrays are indexed in the
 * numbering of the mb_mesh they are passed with: either manapy's own (the
 * numbering of manapy/ddm/domain.py:294-334) or any relabelling of cells, faces
 * and nodes the caller applied consistently to every table (the Python layer
 * uses a Morton-curve relabelling for locality; per-cell lists keep manapy's
 * order, so accumulation order is unchanged).  Vectors are [n][3].
 *
 * A mesh is described once by mb_mesh (device tables built on the host from
 * manapy's Domain arrays); the per-variable ghost rules by mb_bc.  The
 * kernels reproduce manapy's per-cell accumulation order: a cell gathers its
 * faces instead of faces scattering into cells, so there are no atomics and
 * the results do not depend on scheduling.
 *
 * Each function below names the manapy function it replaces (file:line in
 * the manapy source tree).
 */
#ifndef MANAPY_B200_H
#define MANAPY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MB_OK 0
#define MB_EINVAL (-1)   /* bad argument (null pointer, bad size, bad dim) */
#define MB_ECUDA (-2)    /* a CUDA launch or call failed */
#define MB_ETOOBIG (-3)  /* the mesh needs more scratch than mb_advdiff_step_noalloc holds */
#define MB_ENONFINITE (-4) /* mb_check_state: a NaN or infinite value */
#define MB_ENEGATIVE (-5)  /* mb_check_state: a negative value where none is allowed (water depth) */

/* Ghost rule of a boundary face (manapy/boundary/bc_utils.py:45-68). */
#define MB_G_NONE 0
#define MB_G_DIRICHLET 1     /* ghost = value[f] */
#define MB_G_NEUMANN 2       /* ghost = w[c0] */
#define MB_G_NONSLIP 3       /* ghost = -w[c0] */
#define MB_G_NEUMANN_NH 4    /* ghost = w[c0] + value[f] * dist[f] */
#define MB_G_CELL_AT_FACE 5  /* ghost = w[(int)value[f]]: manapy reads its cell array at the
                                face's own index; value[f] holds that cell index */

typedef struct mb_mesh {
  int32_t dim;       /* 2 (triangles) or 3 (tetrahedra) */
  int32_t nbcells;
  int32_t nbfaces;
  int32_t nbnodes;
  int32_t nlf;       /* faces per cell: 3 or 4 */
  int32_t variant;   /* launch shapes of the fused advection-diffusion phases (second order with
                        diffusion): bits 0-1 first phase, bits 2-3 second; 0 = the defaults */
  /* cells */
  const double *cell_center;    /* [nbcells][3] */
  const double *cell_volume;    /* [nbcells] */
  const int32_t *cell_faces;    /* [nbcells][4], manapy's local face order (cells.faceid) */
  const uint8_t *cell_order;    /* [nbcells], 2 bits per slot: slot visited k-th in ascending face id */
  const int32_t *cellnid_ptr;   /* [nbcells+1] CSR of vertex neighbours (cells.cellnid) */
  const int32_t *cellnid_idx;
  const int32_t *ghostnid_ptr;  /* [nbcells+1] CSR of stencil boundary faces (cells.ghostnid) */
  const int32_t *ghostnid_idx;
  /* faces */
  const int32_t *face_cellid;   /* [nbfaces][2], second = -1 on boundary faces (faces.cellid) */
  const int32_t *face_nodeid;   /* [nbfaces][4] (faces.nodeid without the count column) */
  const int32_t *face_name;     /* [nbfaces] (faces.name) */
  const double *face_normal;    /* [nbfaces][3] */
  const double *face_center;    /* [nbfaces][3] */
  const double *face_mesure;    /* [nbfaces] */
  const double *face_ghostcenter; /* [nbfaces][3] ghost cell centre (faces.ghostcenter) */
  const double *face_air;       /* [nbfaces] diamond measure (faces.airDiamond) */
  const double *face_f;         /* 2D: [nbfaces][4][2] = f_1..f_4; 3D: [nbfaces][2][3] = f_1, f_2 */
  const double *face_dist;      /* [nbfaces] (faces.dist_ortho) */
  /* nodes */
  const int32_t *n2c_ptr;       /* [nbnodes+1] CSR node -> cells (nodes.cellid) */
  const int32_t *n2c_idx;
  const double *n2c_alpha;      /* centre->vertex weight of each node->cell incidence */
  const int32_t *n2g_ptr;       /* [nbnodes+1] CSR node -> boundary faces (nodes.ghostid) */
  const int32_t *n2g_idx;
  const double *n2g_alpha;
  /* SW bathymetry source (2D): cells.cellfid [nbcells][4], cells.nf [nbcells][3][3],
   * vertex of local node 1 of each cell [nbcells][2] */
  const int32_t *cell_cellfid;
  const double *cell_nf;
  const double *cell_vertex1;
  /* compact cell-centred tables read by the fused step (2D; NULL selects the
   * face tables above):
   *   cell_vtx   [nbcells][4] vertices in manapy's local order (cells.nodeid);
   *   cell_nbr   [nbcells][4] cell across local face j (faces (v_j, v_j+1)), or
   *              -1-f for boundary face f;
   *   cell_flags [nbcells] bit j: the cell is faces.cellid[f][0]; bit 3+j:
   *              faces.nodeid[f][0] is v_j+1 (else v_j); bit 6+j: the stored
   *              normal is -(y_a - y_b, x_b - x_a), a = faces.nodeid[f][0]; bit 9+j:
 *              cells.nf (outward normal) of face j is minus the face normal;
   *   node_coord [nbnodes][2] vertex coordinates; cell_xy [nbcells][2] centres.
   * 3D (tetrahedra): cell_nbr / cell_vtx as above with local faces (v0,v1,v2),
   * (v2,v3,v0), (v0,v1,v3), (v3,v1,v2); cell_flags has 6 bits per face j at bit 6j:
   * own, 3-bit permutation to manapy's descending face-node order, orientation
   * swap, normal flip; node_coord and cell_xy are [n][4] (x, y, z, unused). */
  const int32_t *cell_vtx;
  const int32_t *cell_nbr;
  const uint32_t *cell_flags;
  const double *node_coord;
  const double *cell_xy;
  /* the same neighbour lists as cellnid_* and n2c_*, stored SELL-32: rows are taken
   * in groups of 32 (one warp); group g occupies idx[ptr[g] .. ptr[g+1]) as
   * [len_g][32] (entry k of row 32g+l at ptr[g] + 32k + l).  An lsq row holds each of
   * its neighbours once, in any slots, and -1 in the others (the kernels sum a row's
   * terms in slot order); n2c rows are padded at their end with their first cell and
   * weight 0 */
  const int32_t *lsq_sell_ptr;
  const int32_t *lsq_sell_idx;
  const int32_t *n2c_sell_ptr;
  const int32_t *n2c_sell_idx;
  const double *n2c_sell_alpha;
  /* n2c_sell_alpha rounded to FP32 (read by the FP32-compensated step only) */
  const float *n2c_sell_alpha_f32;
  /* [nbfaces][4] = {n_x, n_y, 1/mesure, 0} rounded to FP32 (FP32-compensated shallow water, 2D) */
  const float *face_nm_f32;
  /* tetrahedra, optional: [nbcells][12] the least-squares moment matrix of each cell's
   * stencil (the lsq_sell neighbours, then its stencil ghosts) as {c_xx, c_xy, c_xz, c_yy,
   * c_yz, c_zz, det, 0}, cofactors and determinant, followed by {D_x, D_y, D_z, 0}, the sum
   * of the lsq_sell neighbours' centre offsets (read by the edge-sum step), 32-byte aligned
   * (mb_lsq_matrix).  The
   * matrix depends on the geometry only; when given, the second-order fused 3D step reads
   * it instead of forming it every step.  Must come from the lsq_sell table of this
   * struct.  Triangles: NULL (their step forms the matrix; reading it measured slower). */
  const double *cell_lsq;
  /* tetrahedra, optional: the edges of the mesh, with which the second-order step forms each
   * cell's least-squares right-hand side from node, edge and face-neighbour sums instead of
   * gathering its whole stencil (needs cell_lsq; see mb_advdiff_step):
   *   cell_edges [nbcells][8] the edge of local vertex pair (0,1), (0,2), (0,3), (1,2), (1,3),
   *              (2,3), then -1, -1;
   *   edge_origin [nbedges] the edge's vertex with the smaller index (the origin of its sums);
   *   edge_sell_ptr / edge_sell_idx: the cells of each edge, SELL-32 as lsq_sell (-1 in
   *              empty slots). */
  const int32_t *cell_edges;
  const int32_t *edge_origin;
  const int32_t *edge_sell_ptr;
  const int32_t *edge_sell_idx;
  int32_t nbedges;
  int32_t pad_;
  /* with the edge tables: the vertex -> cells lists (as n2c_*) in the slot-shared SELL-32
   * layout of lsq_sell, with their centre->vertex weights (-1 and weight 0 in empty slots) */
  const int32_t *n2c_sum_ptr;
  const int32_t *n2c_sum_idx;
  const double *n2c_sum_alpha;
} mb_mesh;

typedef struct mb_bc {
  const int8_t *kind;   /* [nbfaces] MB_G_* */
  const double *value;  /* [nbfaces] dirichlet value / neumannNH gradient */
  /* faces whose diamond gradient manapy computes: inner, dirichlet and
   * neumann-list faces (manapy/ast/core.py:480-490); 1 = computed */
  const uint8_t *face_grad_on;
} mb_bc;

/* ---- reference kernels, one entry point each ---------------------------------- */

/* manapy/ast/ast_utils.py:8-18 facetocell */
int mb_facetocell(const mb_mesh *m, const double *u_face, double *u_cell, void *stream);

/* manapy/boundary/bc_utils.py:45-68 ghost_value_* for every boundary face (Variable.update_ghost_value,
 * manapy/ast/core.py:492-497) */
int mb_ghost_value(const mb_mesh *m, const mb_bc *bc, const double *w_c, double *w_ghost, void *stream);

/* manapy/ast/functions2d.py:5-104 cell_gradient_2d, manapy/ast/functions3d.py:4-120 cell_gradient_3d */
int mb_cell_gradient(const mb_mesh *m, const double *w_c, const double *w_ghost, double *w_x,
                     double *w_y, double *w_z, void *stream);

/* manapy/ast/functions2d.py:280-325 barthlimiter_2d, manapy/ast/functions3d.py:364-408 barthlimiter_3d */
int mb_barthlimiter(const mb_mesh *m, const double *w_c, const double *w_ghost, const double *w_x,
                    const double *w_y, const double *w_z, double *psi, void *stream);

/* manapy/ast/functions2d.py:199-276 centertovertex_2d, manapy/ast/functions3d.py:251-362 */
int mb_centertovertex(const mb_mesh *m, const double *w_c, const double *w_ghost, double *w_node,
                      void *stream);

/* manapy/ast/functions2d.py:108-196 face_gradient_2d, manapy/ast/functions3d.py:122-248 */
int mb_face_gradient(const mb_mesh *m, const mb_bc *bc, const double *w_c, const double *w_ghost,
                     const double *w_node, double *wx_face, double *wy_face, double *wz_face,
                     void *stream);

/* manapy/solvers/advecdiff/fvm_utils.py:43-176 explicitscheme_convective_2d, :180-314 _3d */
int mb_explicitscheme_convective(const mb_mesh *m, double *rez_w, const double *w_c,
                                 const double *w_ghost, const double *u_face, const double *v_face,
                                 const double *w_face, const double *w_x, const double *w_y,
                                 const double *w_z, const double *psi, int32_t order, void *stream);

/* manapy/solvers/advecdiff/fvm_utils.py:5-26 explicitscheme_dissipative */
int mb_explicitscheme_dissipative(const mb_mesh *m, const double *wx_face, const double *wy_face,
                                  const double *wz_face, double *dissip_w, double Dxx, double Dyy,
                                  double Dzz, void *stream);

/* manapy/solvers/advecdiff/fvm_utils.py:317-340 time_step; the min lands in *dt_dev (device) */
int mb_time_step(const mb_mesh *m, const double *u, const double *v, const double *w, double cfl,
                 double Dxx, double Dyy, double Dzz, double *dt_dev, void *stream);

/* manapy/solvers/advecdiff/fvm_utils.py:342-346 update_new_value; dt read from *dt_dev */
int mb_update_new_value(const mb_mesh *m, double *ne_c, const double *rez, const double *dissip,
                        const double *src, const double *dt_dev, void *stream);

/* ---- shallow water ------------------------------------------------------------------- */

/* manapy/solvers/shallowater/fvm_utils.py:152-342 srnh_scheme for n independent states:
 * states [n][10] = hu_l hu_r hv_l hv_r h_l h_r hc_l hc_r Z_l Z_r, normals [n][3], mesure [n]
 * -> flux [n][5] */
int mb_srnh_flux(int32_t n, const double *states, const double *normals, const double *mesure,
                 double grav, double *flux, void *stream);

/* manapy/solvers/shallowater/fvm_utils.py:16-42 time_step_SW -> *dt_dev */
int mb_time_step_sw(const mb_mesh *m, const double *h, const double *hu, const double *hv,
                    double cfl, double grav, double Dxx, double Dyy, double *dt_dev, void *stream);

/* manapy/solvers/shallowater/fvm_utils.py:344-496 explicitscheme_convective_SW.
 * q = {h, hu, hv, hc, Z} cell states, g = their ghosts; grads = {h_x, h_y, hc_x, hc_y}, psi = hc's
 * limiter (manapy/solvers/shallowater/system.py:168-178).  face_flux is scratch [nbfaces][5]. */
int mb_explicitscheme_convective_sw(const mb_mesh *m, double *const rez[5], const double *const q[5],
                                    const double *const g[5], const double *const grads[4],
                                    const double *psi, double grav, int32_t order,
                                    double *face_flux, void *stream);

/* manapy/solvers/shallowater/fvm_utils.py:44-148 term_source_srnh_SW -> src_hu, src_hv
 * (src_h, src_hc, src_Z are zero in the reference and are not written) */
int mb_term_source_srnh_sw(const mb_mesh *m, const double *h, const double *Z, const double *h_ghost,
                           const double *Z_ghost, double grav, double *src_hu, double *src_hv,
                           void *stream);

/* manapy/solvers/shallowater/fvm_utils.py:3-14 update_SW (no coriolis, no wind) */
int mb_update_sw(const mb_mesh *m, double *const q[5], const double *const rez[5],
                 const double *src_hu, const double *src_hv, const double *dt_dev, void *stream);

/* ---- Euler equations, 2D, first-order Rusanov (manapy/solvers/euler/fvm_utils2d.py) ----
 * q: cell arrays rho, P, rhou, rhov, rhoE; g: the same on the faces (ghost values).
 * Results are bit-identical to manapy's kernels (no multiply-add contraction). */

/* fvm_utils2d.py:1490-1611 explicitscheme_euler_2d_rusanov (flux :1248-1292) -> rez rho, rhou,
 * rhov, rhoE (each face flux evaluated by both of its cells; cells add faces by ascending id).
 * Every face not named 0 reads its right state from g, halo faces (name 10) included: on a
 * shard the caller places the neighbour rank's values there. */
int mb_euler_rusanov_2d(const mb_mesh *m, const double *const q[5], const double *const g[5],
                        double *const rez[4], double gamma, void *stream);

/* fvm_utils2d.py:1083-1102 time_step_euler_2d: the CFL dt of every cell into dt_c
 * (reads q[0..3]; q[4] must be non-null) */
int mb_time_step_euler_2d(const mb_mesh *m, const double *const q[5], double cfl, double gamma,
                          double *dt_c, void *stream);

/* fvm_utils2d.py:1687-1696 update_euler_2d_fvc: conserved variables += dt rez / V, then P */
int mb_update_euler_2d(const mb_mesh *m, double *const q[5], const double *const rez[4], double gamma,
                       double dt, void *stream);

/* fvm_utils2d.py:592-648 ghost_value_Neumann: faces named 1-4 copy their cell's state
 * into g (rho, P, rhou, rhov, rhoE) and set ug = rhou / rho, vg = rhov / rho */
int mb_ghost_euler_neumann_2d(const mb_mesh *m, const double *const q[5], double *const g[5], double *ug,
                              double *vg, void *stream);

/* Fused Euler step (manapy ships the kernels above without a driver):
 * ghost_value_Neumann + explicitscheme_euler_2d_rusanov + update_euler_2d_fvc with
 * dt = min(time_step_euler_2d), bit-identical to that sequence, in two launches (every face
 * flux once into face_flux, then update + next dt per cell).  Every boundary face must carry
 * the Neumann rule (names 1-4); no halo faces.
 * mb_euler_tables_2d fills, once per mesh, face_rec (4 * nbfaces doubles, 32-byte aligned:
 * normal x, y, mesure and the two cells of each face) and cell_left (nbcells bytes: bit j set
 * when the cell is the left cell of its local face j).
 * face_flux: device scratch of 4 * nbfaces doubles, 32-byte aligned.
 * ring: 3 device doubles.  mb_euler_dt_2d resets the ring and puts the dt of q into slot t%3;
 * mb_euler_step_2d at time index t reads slot t%3, writes q_out (buffers distinct from q_in),
 * min-reduces the dt of q_out into slot (t+1)%3 and resets slot (t+2)%3, so consecutive calls
 * with t, t+1, ... need no host synchronisation.  time (nullable, device): += the dt used. */
int mb_euler_dt_2d(const mb_mesh *m, const double *const q[5], double cfl, double gamma, double *ring, int t,
                   void *stream);
int mb_euler_tables_2d(const mb_mesh *m, double *face_rec, uint8_t *cell_left, void *stream);
int mb_euler_step_2d(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl,
                     double gamma, const double *face_rec, const uint8_t *cell_left, double *face_flux,
                     double *ring, int t, double *time, void *stream);

/* ---- fused steps ---------------------------------------------------------------------- */

typedef struct mb_advdiff_params {
  int32_t order;       /* 1 or 2 */
  int32_t diffusion;   /* 0: Dxx = Dyy = Dzz = 0 (manapy skips the diffusive flux) */
  double Dxx, Dyy, Dzz;
} mb_advdiff_params;

/* One advection-diffusion step, the work of AdvectionDiffusionSolver.compute_fluxes +
 * compute_new_val (manapy/solvers/advecdiff/system.py:156-172) in two launches:
 *   1. cell gradients + Barth limiter (order 2) and centre->vertex values (diffusion);
 *   2. per cell: upwind fluxes, diamond diffusion, forward-Euler update;
 * tetrahedra at order 2 add a pack pass before 1 (rows {centre, value} of every cell).
 * w_in is read, w_out written (distinct buffers).  sign_cf[4*i+j] = u.n of the j-th
 * local face of cell i in manapy's face orientation (mb_cell_face_sign); src may be
 * NULL (zero source).  Scratch: cell_scratch [4*nbcells] in 2D, [8*nbcells] in 3D
 * (order 2; [8*nbcells + 4*(nbnodes + nbedges)] when m carries the edge tables),
 * node_scratch [nbnodes] (diffusion); NULL where not needed. */
int mb_advdiff_step(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                    const double *w_in, double *w_out, const double *sign_cf, const double *src,
                    const double *dt_dev, double *cell_scratch, double *node_scratch, void *stream);

/* Rows {centre, value} of a state, [nbcells][4] doubles, 32-byte aligned: {x, y, w, 0} for
 * triangles, {x, y, z, w} for tetrahedra (no counterpart in manapy). */
int mb_pack_rows(const mb_mesh *m, const double *w, double *rows, void *stream);

/* mb_advdiff_step in two parts, so that the values of cells [0, nfirst) are final before the
 * rest are computed (a sharded run numbers the cells its peers read first and sends them
 * while part 1 runs): part 0 runs the first phase over every cell and node and the second
 * phase over cells [0, nfirst); part 1 the second phase over cells [nfirst, nbcells),
 * reading the first phase's results that part 0 left in cell_scratch / node_scratch (both
 * parts with the same arguments, part 1 after part 0 on the same stream or ordered after
 * it).  Together they compute exactly what mb_advdiff_step computes.  Compact tables only.
 * Replaces the same step as mb_advdiff_step (manapy/solvers/advecdiff/system.py:156-172);
 * the split has no counterpart in manapy, whose halo exchange follows the whole step. */
int mb_advdiff_step_split(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p, const double *w_in,
                          double *w_out, const double *sign_cf, const double *src, const double *dt_dev,
                          double *cell_scratch, double *node_scratch, int32_t part, int32_t nfirst, void *stream);

/* The cell_lsq table of a tetrahedral mesh with compact tables ([nbcells][12] doubles,
 * 32-byte aligned; layout at mb_mesh.cell_lsq): the moment matrix sum over the stencil of
 * d d^T, d = centre offset, of
 * manapy/ast/functions3d.py:4-120 (cell_gradient_3d), as cofactors and determinant, summed in
 * the order the fused step sums its right-hand side.  Once per mesh.  MB_EINVAL for
 * triangles. */
int mb_lsq_matrix(const mb_mesh *m, double *out, void *stream);

/* mb_advdiff_step for a run of consecutive steps (no counterpart in manapy): rows_in holds
 * the rows of w_in (mb_pack_rows, or the previous step's rows_out), from which the first
 * launch reads each least-squares neighbour's centre and value with one 256-bit load; the
 * second launch also writes the rows of w_out into rows_out.  Same results as
 * mb_advdiff_step, same scratch (3D: the first 4*nbcells doubles of cell_scratch are used);
 * compact tables required; rows_in != rows_out. */
int mb_advdiff_step_rows(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                         const double *w_in, double *w_out, const double *rows_in, double *rows_out,
                         const double *sign_cf, const double *src, const double *dt_dev,
                         double *cell_scratch, double *node_scratch, void *stream);

/* The u.n table of the FP32-compensated step from mb_cell_face_sign's FP64 table: per
 * cell the FP32 u.n of each local face and the cell's signed sum of them (sum over its
 * faces of -u.n where the cell is faces.cellid[f][0], +u.n elsewhere), formed in FP64:
 * 2D [nbcells][4] = {s0, s1, s2, sum}; 3D [nbcells][4] then [nbcells] sums (5*nbcells). */
int mb_cell_face_sign_f32c(const mb_mesh *m, const double *sign_cf, float *sign_f32, void *stream);

/* FP32-compensated twin of mb_advdiff_step (no counterpart in manapy, whose single
 * precision mode is FP32 throughout, manapy/backends/cpu/backend.py:46-49): the same
 * two launches with FP32 state (w_in, w_out), FP32 u.n (sign_cf from mb_cell_face_sign_f32c), FP32
 * source (src, may be NULL), FP32 phase-1 records and node values, FP32 fluxes summed
 * per cell with compensated (Neumaier) summation on differences from the cell's own
 * value; coordinates, every geometric coefficient and dt stay FP64.  Scratch:
 * cell_scratch [4*nbcells] floats in 2D, [5*nbcells] in 3D (order 2), node_scratch
 * [nbnodes] floats (diffusion).  Tetrahedra whose struct carries the edge tables (order 2)
 * form the least-squares sums by inclusion-exclusion as mb_advdiff_step does, in FP64 over
 * the FP32 state: cell_scratch then holds 5*nbcells floats rounded up to a multiple of 8,
 * followed by the vertex and edge sums, 8*(nbnodes + nbedges) floats, and must be
 * 32-byte aligned.  Needs the
 * compact tables of mb_mesh, n2c_sell_alpha_f32 included.
 * Compensated state: lo_in / lo_out (FP32 [nbcells], both or neither) carry the rounding
 * error of the state, w + lo; the update is w_out + lo_out = w_in + (increment + lo_in)
 * exactly, so the FP32 state loses nothing to rounding from step to step (fluxes still see
 * the FP32 w).  NULL: plain FP32 state. */
int mb_advdiff_step_f32c(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                         const float *w_in, float *w_out, const float *lo_in, float *lo_out,
                         const float *sign_cf, const float *src, const double *dt_dev,
                         float *cell_scratch, float *node_scratch, void *stream);

/* sign_cf[4*i+j] = u_face[f] n_x + v_face[f] n_y + w_face[f] n_z for the j-th local face f
 * of cell i (zero for unused slots): the upwind selector of
 * manapy/solvers/advecdiff/fvm_utils.py:53-64 laid out per cell for mb_advdiff_step */
int mb_cell_face_sign(const mb_mesh *m, const double *u_face, const double *v_face,
                      const double *w_face, double *sign_cf, void *stream);

/* sign_face[f] = u_face[f] n_x + v_face[f] n_y + w_face[f] n_z, the upwind selector of
 * manapy/solvers/advecdiff/fvm_utils.py:53-64 */
int mb_face_sign(const mb_mesh *m, const double *u_face, const double *v_face,
                 const double *w_face, double *sign_face, void *stream);

/* One shallow-water step (ShallowWaterSolver.compute_fluxes + compute_new_val,
 * manapy/solvers/shallowater/system.py:248-281,237-242) with Neumann ghosts on every
 * boundary face (manapy's default), in two launches: [order 2: h, hc gradients and hc
 * limiter] face fluxes, then per cell the residual gather, bathymetry source and update.
 * The update uses *dt_cur (from mb_time_step_sw, or the previous step's dt_next); the
 * second launch also evaluates time_step_SW on the updated state into *dt_next (the next
 * step's dt), unless dt_next is NULL.  q_in / q_out: 5 cell arrays each (h, hu, hv, hc, Z);
 * q_out[k] != q_in[k] except Z (the bed does not change and may be shared).  Scratch:
 * face_flux [nbfaces][4], scratch [5][nbcells] (order 2 only, else NULL).  Needs the
 * compact 2D tables of mb_mesh. */
int mb_sw_step(const mb_mesh *m, const double *const q_in[5], double *const q_out[5],
               double cfl, double grav, int32_t order, double *scratch, double *face_flux,
               const double *dt_cur, double *dt_next, void *stream);

/* Boundary treatment of the shallow-water steps' boundary faces. */
#define MB_WALLS_NEUMANN 0  /* ghost = the interior cell's state (manapy's default, and what its
                               `slip` condition degrades to, manapy/boundary/bc.py:59-76) */
#define MB_WALLS_REFLECT 1  /* reflective wall: ghost h, hc, Z copied, momentum mirrored,
                               q - 2 (q.n) n / |n|^2; no counterpart in manapy (its `slip` ghost
                               function is commented out, manapy/boundary/bc.py:68-72): the mass
                               flux through a wall vanishes up to rounding */

/* The CFL dt of a shallow-water state with the fused step's formula (the next-step dt
 * that mb_sw_step writes into dt_next, manapy/solvers/shallowater/fvm_utils.py:16-42
 * without diffusion): *dt_dev = min over cells.  Needs the compact 2D tables. */
int mb_sw_dt(const mb_mesh *m, const double *h, const double *hu, const double *hv, double cfl, double grav,
             double *dt_dev, void *stream);

/* mb_sw_step with a choice of wall treatment (walls: MB_WALLS_*); mb_sw_step is this with
 * MB_WALLS_NEUMANN. */
int mb_sw_step_ex(const mb_mesh *m, const double *const q_in[5], double *const q_out[5],
                  double cfl, double grav, int32_t order, int32_t walls, double *scratch,
                  double *face_flux, const double *dt_cur, double *dt_next, void *stream);

/* mb_sw_step_ex in two parts, so that the values of cells [0, nfirst) are final before the
 * rest are computed (a sharded run numbers the cells its peers read first and sends them
 * while part 1 runs): part 0 computes every face flux (and, for order 2, the gradients) and
 * updates cells [0, nfirst); part 1 updates cells [nfirst, nbcells) from the face fluxes that
 * part 0 left in face_flux (both parts with the same arguments, part 1 after part 0 on the
 * same stream or ordered after it).  Together they compute exactly what mb_sw_step_ex
 * computes, dt_next included.  Replaces the same step (manapy/solvers/shallowater/
 * system.py:186-281); the split has no counterpart in manapy. */
int mb_sw_step_split(const mb_mesh *m, const double *const q_in[5], double *const q_out[5], double cfl,
                     double grav, int32_t order, int32_t walls, double *scratch, double *face_flux,
                     const double *dt_cur, double *dt_next, int32_t part, int32_t nfirst, void *stream);

/* FP32-compensated twin of mb_sw_step (no counterpart in manapy), first order, Neumann
 * ghosts: FP32 state (q_in, q_out: h, hu, hv, hc, Z), FP32 SRNH flux arithmetic and face
 * fluxes (face_flux [nbfaces][4] floats), residuals summed per cell with compensated
 * (Neumaier) summation; normals come from face_nm_f32; the bathymetry source, dt_cur and
 * dt_next (time_step_SW of the updated state) are FP64.  lo_in / lo_out (4 FP32 arrays each
 * for h, hu, hv, hc, or both NULL) carry the rounding error of the state: q_out + lo_out =
 * q_in + (increment + lo_in) exactly. */
int mb_sw_step_f32c(const mb_mesh *m, const float *const q_in[5], float *const q_out[5],
                    const float *const lo_in[4], float *const lo_out[4], double cfl, double grav,
                    int32_t order, float *face_flux, const double *dt_cur, double *dt_next, void *stream);

/* mb_sw_step_f32c with a choice of wall treatment (walls: MB_WALLS_*). */
int mb_sw_step_f32c_ex(const mb_mesh *m, const float *const q_in[5], float *const q_out[5],
                       const float *const lo_in[4], float *const lo_out[4], double cfl, double grav,
                       int32_t order, int32_t walls, float *face_flux, const double *dt_cur,
                       double *dt_next, void *stream);

/* ---- batches of independent triangle meshes (serving) ----------------------------------
 *
 * No counterpart in manapy (one mesh per process).  Many meshes advance in the same
 * launches: the caller lays out one item per mesh in device memory and, per launch, a
 * map from block to item (each item owns a contiguous block range, so no block spans two
 * meshes).  A device step counter (*clock, incremented by the last launch of every step)
 * selects each item's ping-pong buffer -- the input of global step t is w[(t - start_step)
 * & 1] -- and items outside [start_step, end_step) do nothing, so one captured CUDA graph
 * of a step serves while items are admitted and retired between replays (the caller
 * rewrites items and maps only between steps). */
typedef struct mb_advdiff_item {
  mb_mesh m;                /* the mesh's tables (compact 2D tables required) */
  mb_bc bc;
  mb_advdiff_params p;
  float *w[2];              /* ping-pong FP32 state */
  float *lo[2];             /* ping-pong rounding errors of the state (NULL: none) */
  const float *sign_cf;     /* [4*nbcells] from mb_cell_face_sign_f32c */
  const float *src;         /* NULL: no source */
  const double *dt_dev;     /* the item's dt */
  float *cell_scratch;      /* [4*nbcells] (order 2) */
  float *node_scratch;      /* [nbnodes] (diffusion) */
  int32_t start_step;       /* first global step the item runs */
  int32_t end_step;         /* first global step it does not run */
  int32_t p1_begin;         /* first block of the item in the phase-1 launch */
  int32_t p1_cell_blocks;   /* its phase-1 blocks [p1_begin, p1_begin + this) do cells, the rest nodes */
  int32_t p2_begin;         /* first block of the item in the phase-2 launch */
  int32_t pad_;
} mb_advdiff_item;

/* One FP32-compensated advection-diffusion step of every active item (the step of
 * mb_advdiff_step_f32c per mesh), order and diffusion common to the batch; then *clock += 1.
 * p1_map [p1_blocks], p2_map [p2_blocks]: item of each block (p1 unused when order 1 without
 * diffusion). */
int mb_advdiff_batch_step_f32c(const mb_advdiff_item *items, const int32_t *p1_map, int32_t p1_blocks,
                               const int32_t *p2_map, int32_t p2_blocks, int32_t order, int32_t diffusion,
                               int32_t *clock, void *stream);

/* A shallow-water mesh of a batch (first order, Neumann ghosts, FP32-compensated). */
typedef struct mb_sw_item {
  mb_mesh m;                /* compact 2D tables and face_nm_f32 required */
  float *q[2][4];           /* ping-pong FP32 h, hu, hv, hc; step t reads q[(t - start_step) & 1] */
  float *lo[2][4];          /* their rounding errors (all NULL: plain FP32 state) */
  const float *Z;           /* bed, FP32 */
  float *face_flux;         /* [nbfaces][4] scratch */
  double *dt;               /* [2]: step t uses dt[(t - start_step) & 1] and writes the next step's dt
                               into the other slot; dt[0] must hold the first step's dt */
  double cfl, grav;
  int32_t start_step, end_step;
  int32_t f_begin;          /* first block of the item in the face launch */
  int32_t c_begin;          /* first block of the item in the cell launch */
} mb_sw_item;

/* One FP32-compensated shallow-water step (mb_sw_step_f32c per mesh) of every active item;
 * then *clock += 1.  face_map [face_blocks], cell_map [cell_blocks]: item of each block. */
int mb_sw_batch_step_f32c(const mb_sw_item *items, const int32_t *face_map, int32_t face_blocks,
                          const int32_t *cell_map, int32_t cell_blocks, int32_t *clock, void *stream);

/* FP64 batches: the same block -> item maps, clock and [start_step, end_step) windows as
 * the FP32-compensated batches above, running the plain FP64 steps (mb_advdiff_step and
 * mb_sw_step per mesh, bit-identical to them).  No counterpart in manapy.  Block maps use
 * 256-cell (and 256-face) blocks. */
typedef struct mb_advdiff_item_f64 {
  mb_mesh m;                /* compact 2D tables required */
  mb_bc bc;
  mb_advdiff_params p;
  double *w[2];             /* ping-pong FP64 state; step t reads w[(t - start_step) & 1] */
  const double *sign_cf;    /* [4*nbcells] from mb_cell_face_sign, 32-byte aligned */
  const double *src;        /* NULL: no source */
  const double *dt_dev;     /* the item's dt */
  double *cell_scratch;     /* [4*nbcells] records (order 2), 32-byte aligned */
  double *node_scratch;     /* [nbnodes] (diffusion) */
  int32_t start_step, end_step;
  int32_t p1_begin;         /* first block of the item in the phase-1 launch */
  int32_t p1_cell_blocks;   /* its phase-1 blocks [p1_begin, p1_begin + this) do cells, the rest nodes */
  int32_t p2_begin;         /* first block of the item in the phase-2 launch */
  int32_t pad_;
} mb_advdiff_item_f64;

int mb_advdiff_batch_step(const mb_advdiff_item_f64 *items, const int32_t *p1_map, int32_t p1_blocks,
                          const int32_t *p2_map, int32_t p2_blocks, int32_t order, int32_t diffusion,
                          int32_t *clock, void *stream);

typedef struct mb_sw_item_f64 {
  mb_mesh m;                /* compact 2D tables required */
  double *q[2][5];          /* ping-pong h, hu, hv, hc, Z (the Z slots may be one array) */
  double *face_flux;        /* [nbfaces][4] scratch, 32-byte aligned */
  double *dt;               /* [2]: step t uses dt[(t - start_step) & 1], writes the next one into
                               the other slot; dt[0] must hold the first step's dt */
  double cfl, grav;
  int32_t start_step, end_step;
  int32_t f_begin;          /* first block of the item in the face launch */
  int32_t c_begin;          /* first block of the item in the cell launch */
} mb_sw_item_f64;

/* One first-order FP64 shallow-water step (Neumann walls) of every active item; then
 * *clock += 1. */
int mb_sw_batch_step(const mb_sw_item_f64 *items, const int32_t *face_map, int32_t face_blocks,
                     const int32_t *cell_map, int32_t cell_blocks, int32_t *clock, void *stream);

/* ---- halo exchange of a mesh sharded over ranks ---------------------------------------
 *
 * manapy exchanges halo values with MPI neighbourhood all-to-alls of per-rank send lists
 * (manapy/comms/communication.py:93-145).  With every peer's list concatenated into one
 * index list idx[n] (device, int64 cell indices, each at most once), mb_halo_pack writes
 * buf[k*nfields + j] = fields[j][idx[k]] for the nfields fields (a host array of device
 * pointers), and mb_halo_unpack writes fields[j][idx[k]] = buf[k*nfields + j]: one launch
 * for all peers and fields on each side of the point-to-point transfers, each peer's
 * entries one contiguous message. */
#define MB_HALO_MAX_FIELDS 8
int mb_halo_pack(double *const *fields, int32_t nfields, const int64_t *idx, int64_t n, double *buf,
                 void *stream);
int mb_halo_unpack(double *const *fields, int32_t nfields, const int64_t *idx, int64_t n, const double *buf,
                   void *stream);

/* Same step as mb_advdiff_step, for callers that cannot allocate device memory.
 *
 * No counterpart in the reference: manapy allocates its work arrays with numpy.
 * This variant is for code that may not call cudaMalloc at all -- a plugin whose
 * host application owns every device allocation through its own pool, a service
 * that reserves its device-memory budget up front, or a loop where a cudaMalloc
 * (which can synchronise the device) is not acceptable.  Its scratch
 * (4*nbcells + nbnodes doubles in 2D, 8*nbcells + nbnodes in 3D) lives in a fixed
 * array inside the library,
 * MB_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB), which every GPU that loads the
 * library keeps reserved until the process exits; larger meshes get MB_ETOOBIG.
 * The first call on each device looks up that array's device address, so make
 * it before any stream capture.  The address is kept for the life of the
 * process: after cudaDeviceReset on a device the library's module is loaded
 * again and the kept address is stale, so a process that resets a device must
 * not call this entry point on that device afterwards.  All calls share the one array: calls that may
 * overlap on the GPU (different streams, or host threads) race with each other
 * and must be serialised by the caller.  Nothing in the array needs clearing
 * between calls.  Arguments as for mb_advdiff_step, without the scratch. */
#define MB_NOALLOC_SCRATCH_DOUBLES (2 * 1024 * 1024)
int mb_advdiff_step_noalloc(const mb_mesh *m, const mb_bc *bc, const mb_advdiff_params *p,
                            const double *w_in, double *w_out, const double *sign_cf,
                            const double *src, const double *dt_dev, void *stream);

/* State check (no counterpart in manapy, where NaNs propagate silently): scans n FP64 values
 * (f64 != NULL) or FP32 values (f32 != NULL) for NaN / infinity and, with nonneg != 0, for
 * negative values; ORs bit 0 (non-finite) and bit 1 (negative) into *flags (device int,
 * zeroed by the caller).  The host reads flags after the stream: MB_ENONFINITE /
 * MB_ENEGATIVE. */
int mb_check_state(const double *f64, const float *f32, int64_t n, int32_t nonneg, int32_t *flags, void *stream);

/* Debug check of a mesh's index tables (no counterpart in manapy, whose Numba kernels do
 * not check their indices either): every entry of every index table the struct holds is
 * compared with the range the kernels gather with it, and every CSR / SELL-32 offset table
 * with being non-decreasing from 0 (SELL group offsets: multiples of 32), one launch per
 * table, reading nothing outside the tables.  *first (device) receives UINT64_MAX, or the
 * first bad entry as table << 40 | offsets << 39 | position, the smallest such key.
 * Tables, in this order (dense tables: position = row * stride + column; CSR / SELL:
 * position in the index array, or with bit 39 the position in the offsets):
 *   0 cell_faces [0, nbfaces)   1 cellnid [0, nbcells)   2 ghostnid [0, nbfaces)
 *   3 face_cellid[.][0] [0, nbcells)   4 face_cellid[.][1] [-1, nbcells) (position counted
 *   from face_cellid + 1)   5 face_nodeid [0, nbnodes)   6 n2c [0, nbcells)   7 n2g [0, nbfaces)
 *   8 cell_cellfid [0, nbcells)   9 cell_vtx [0, nbnodes)   10 cell_nbr [-nbfaces, nbcells)
 *   11 lsq_sell [-1, nbcells)   12 n2c_sell [0, nbcells)   and, when cell_edges is set,
 *   13 cell_edges [0, nbedges)   14 edge_origin [0, nbnodes)   15 edge_sell [-1, nbcells)
 *   16 n2c_sum [-1, nbcells)
 * A CSR or SELL table's last offset is taken as the length of its index array. */
int mb_check_tables(const mb_mesh *m, uint64_t *first, void *stream);

/* Library build information (architecture string), for diagnostics. */
const char *mb_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* MANAPY_B200_H */
