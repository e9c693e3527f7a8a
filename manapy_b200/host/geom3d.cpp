// Native host builder of the manapy Domain arrays of a 3D tetrahedral mesh (manapy
// numbering): the same numbers as geometry.build(elements, vertex, 3), operation for
// operation, so its output is bit-identical to it.
//
//   cell centres / volumes             manapy/ddm/ddm_utils3d.py:686-764
//   node -> cells, vertex neighbours   ddm_utils3d.py (cellnid)
//   faces (unique descending node triples, numbered in ascending order), cell -> face,
//   face -> cells, face neighbours     manapy/ddm/domain.py:313-315
//   face names, normals, areas, node order re-oriented with the normal
//                                      ddm_utils3d.py:530-683, :362-377
//   ghost centres, node -> ghosts      ddm_utils3d.py:87-157
//   centre -> vertex weights           ddm_utils3d.py:813-981
//   diamond vectors, areas             ddm_utils3d.py:459-527
//
// The device tables are then derived from these arrays by the Python DeviceMesh.
// Compiled with -ffp-contract=off: every operation rounds as written.
// C ABI: mbh_geometry3d() returns a handle read with mbh_count / mbh_info / mbh_data.
#include "common.hpp"

namespace {

using namespace mbh;

struct V3 {
  double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 scale(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }

Result *geometry3d(const i32 *el, i64 nc, const double *vx, i64 nn) {
  auto *res = new Result();
  for (i64 c = 0; c < nc; ++c)
    if (el[5 * c + 4] != 4) {
      res->error = "3D meshes must be all tetrahedra";
      return res;
    }
  auto P = [&](i64 n) { return V3{vx[4 * n], vx[4 * n + 1], vx[4 * n + 2]}; };
  auto node = [&](i64 c, int j) { return (i64)el[5 * c + j]; };

  // ---- cell centre and volume
  std::vector<double> cc(3 * nc), vol(nc);
  for (i64 c = 0; c < nc; ++c) {
    const V3 p0 = P(node(c, 0)), p1 = P(node(c, 1)), p2 = P(node(c, 2)), p3 = P(node(c, 3));
    V3 s{0.0 + p0.x, 0.0 + p0.y, 0.0 + p0.z};
    s = add(s, p1);
    s = add(s, p2);
    s = add(s, p3);
    cc[3 * c] = s.x / 4;
    cc[3 * c + 1] = s.y / 4;
    cc[3 * c + 2] = s.z / 4;
    const V3 u = sub(p1, p0), v = sub(p2, p0), w = sub(p3, p0);
    vol[c] = std::fabs(dot(u, cross(v, w))) / 6.0;
  }
  auto C = [&](i64 c) { return V3{cc[3 * c], cc[3 * c + 1], cc[3 * c + 2]}; };

  // ---- node -> cells (ascending cell), cell -> vertex neighbours
  std::vector<i64> flat_nodes(4 * nc), flat_cells(4 * nc), c2n_ptr(nc + 1);
  for (i64 c = 0; c < nc; ++c)
    for (int j = 0; j < 4; ++j) {
      flat_nodes[4 * c + j] = node(c, j);
      flat_cells[4 * c + j] = c;
    }
  for (i64 c = 0; c <= nc; ++c) c2n_ptr[c] = 4 * c;
  std::vector<i64> n2c_ptr, n2c_idx;
  group_csr(flat_nodes, flat_cells, nn, n2c_ptr, n2c_idx);
  std::vector<i64> cnid_ptr, cnid_idx;
  ragged_union(nc, c2n_ptr, flat_nodes, n2c_ptr, n2c_idx, true, cnid_ptr, cnid_idx);

  // ---- faces: descending node triples, numbered by ascending key
  static const int LOC[4][3] = {{0, 1, 2}, {2, 3, 0}, {0, 1, 3}, {3, 1, 2}};
  const i64 ne = 4 * nc;
  std::vector<i64> pa(ne), pb(ne), pc(ne);
  for (i64 c = 0; c < nc; ++c)
    for (int j = 0; j < 4; ++j) {
      i64 t[3] = {node(c, LOC[j][0]), node(c, LOC[j][1]), node(c, LOC[j][2])};
      std::sort(t, t + 3);
      pa[4 * c + j] = t[2];
      pb[4 * c + j] = t[1];
      pc[4 * c + j] = t[0];
    }
  // stable order of the keys (a, b, c): counting-sort passes by c, b, then a
  std::vector<i64> ord(ne);
  {
    std::vector<i64> tmp(ne), cnt(nn + 1);
    auto pass = [&](const std::vector<i64> &digit, const std::vector<i64> &in, std::vector<i64> &out) {
      std::fill(cnt.begin(), cnt.end(), 0);
      for (i64 e : in) cnt[digit[e] + 1]++;
      for (i64 d = 0; d < nn; ++d) cnt[d + 1] += cnt[d];
      for (i64 e : in) out[cnt[digit[e]]++] = e;
    };
    std::vector<i64> id(ne);
    std::iota(id.begin(), id.end(), 0);
    pass(pc, id, tmp);
    pass(pb, tmp, id);
    pass(pa, id, ord);
  }
  std::vector<i64> inv(ne), fa, fb, fc, f0, f1;
  for (i64 e = 0; e < ne; ++e) {
    const i64 o = ord[e];
    const bool same = e > 0 && pa[o] == pa[ord[e - 1]] && pb[o] == pb[ord[e - 1]] && pc[o] == pc[ord[e - 1]];
    if (!same) {
      fa.push_back(pa[o]);
      fb.push_back(pb[o]);
      fc.push_back(pc[o]);
      f0.push_back(o / 4);
      f1.push_back(-1);
    } else {
      if (f1.back() != -1) {
        res->error = "non-manifold mesh: a face is shared by more than two cells";
        return res;
      }
      f1.back() = o / 4;
    }
    inv[o] = (i64)fa.size() - 1;
  }
  const i64 nf = (i64)fa.size();
  // face neighbours, compacted (boundary faces skipped)
  std::vector<i32> cellfid(5 * nc, -1), faceid(5 * nc);
  for (i64 c = 0; c < nc; ++c) {
    int k = 0;
    for (int j = 0; j < 4; ++j) {
      const i64 f = inv[4 * c + j];
      faceid[5 * c + j] = (i32)f;
      if (f1[f] == -1) continue;
      cellfid[5 * c + k++] = (i32)(f0[f] == c ? f1[f] : f0[f]);
    }
    faceid[5 * c + 4] = 4;
    cellfid[5 * c + 4] = k;
  }

  // ---- names (from the descending node order), normals, areas, centres
  std::vector<i32> namen(nn);
  for (i64 n = 0; n < nn; ++n) namen[n] = (i32)vx[4 * n + 3];
  std::vector<i32> name(nf, 0);
  std::vector<double> nrm(3 * nf), mes(nf), fcen(3 * nf);
  std::vector<i64> fn0(nf), fn1(nf), fn2(nf);  // node order re-oriented with the normal
  for (i64 f = 0; f < nf; ++f) {
    const i64 v[3] = {fa[f], fb[f], fc[f]};
    if (f1[f] == -1) {
      const i32 t[3] = {namen[v[0]], namen[v[1]], namen[v[2]]};
      i32 r = 100;
      for (i32 tag : {44, 33, 66, 55, 4, 3, 6, 5}) {
        bool m = false;
        for (int j = 0; j < 3; ++j) {
          bool mj = t[j] == tag;
          for (int jj = 0; jj < 3; ++jj)
            if (jj != j) mj = mj && t[jj] != 0;
          m = m || mj;
        }
        if (m) r = tag;
      }
      if (t[0] == t[1] && t[0] == t[2]) r = t[0];
      name[f] = r;
      if (r >= 100 || r == 0) {
        res->error = "mesh has boundary faces that match no boundary side (manapy names them 100/200 and "
                     "leaves them out of every face list)";
        return res;
      }
    }
    const V3 V0 = P(v[0]), V1 = P(v[1]), V2 = P(v[2]);
    const V3 cen = scale(1.0 / 3, add(add(V0, V1), V2));
    const V3 cr = cross(sub(V1, V0), sub(V2, V0));
    const V3 nm = scale(0.5, cr);
    mes[f] = std::sqrt(nm.x * nm.x + nm.y * nm.y + nm.z * nm.z);
    const V3 sn = sub(C(f0[f]), cen);
    const bool flip = dot(sn, nm) > 0;
    const V3 n = flip ? scale(-1, nm) : nm;
    const bool swap = dot(cr, n) < 0;
    fn0[f] = v[0];
    fn1[f] = swap ? v[2] : v[1];
    fn2[f] = swap ? v[1] : v[2];
    nrm[3 * f] = n.x; nrm[3 * f + 1] = n.y; nrm[3 * f + 2] = n.z;
    fcen[3 * f] = cen.x; fcen[3 * f + 1] = cen.y; fcen[3 * f + 2] = cen.z;
  }
  auto N = [&](i64 f) { return V3{nrm[3 * f], nrm[3 * f + 1], nrm[3 * f + 2]}; };

  // ---- face lists (manapy numbering)
  std::vector<i64> lists[7], bfaces;
  for (i64 f = 0; f < nf; ++f) {
    if (name[f] >= 0 && name[f] <= 6) lists[name[f]].push_back(f);
    if (name[f] >= 1 && name[f] <= 6) bfaces.push_back(f);
  }

  // ---- ghost centres
  std::vector<double> gc(4 * nf, -1.0);
  for (i64 f : bfaces) {
    const V3 nf_ = {nrm[3 * f] / mes[f], nrm[3 * f + 1] / mes[f], nrm[3 * f + 2] / mes[f]};
    const V3 v1 = C(f0[f]);
    const V3 u = sub(V3{fcen[3 * f], fcen[3 * f + 1], fcen[3 * f + 2]}, v1);
    const double gamma = dot(u, nf_);
    const V3 kk = add(v1, scale(gamma, nf_));
    gc[4 * f] = 2 * kk.x + (-1 * v1.x);
    gc[4 * f + 1] = 2 * kk.y + (-1 * v1.y);
    gc[4 * f + 2] = 2 * kk.z + (-1 * v1.z);
    gc[4 * f + 3] = gamma;
  }
  // node -> boundary faces (nodes in the re-oriented order), cell -> stencil ghosts
  std::vector<i64> gkey, gval;
  for (i64 f : bfaces) {
    for (i64 nd : {fn0[f], fn1[f], fn2[f]}) {
      gkey.push_back(nd);
      gval.push_back(f);
    }
  }
  std::vector<i64> n2g_ptr, n2g_idx;
  group_csr(gkey, gval, nn, n2g_ptr, n2g_idx);
  std::vector<i64> gnid_ptr, gnid_idx;
  ragged_union(nc, c2n_ptr, flat_nodes, n2g_ptr, n2g_idx, false, gnid_ptr, gnid_idx);

  // ---- centre -> vertex weights: cells, then ghosts, summed in that order
  std::vector<double> Rx(nn), Ry(nn), Rz(nn), lx(nn), ly(nn), lz(nn);
  std::vector<i32> number(nn);
  for (i64 n = 0; n < nn; ++n) {
    const V3 X = P(n);
    double Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0, sx = 0, sy = 0, sz = 0;
    auto acc = [&](V3 p) {
      const V3 r = sub(p, X);
      Ixx += r.x * r.x; Iyy += r.y * r.y; Izz += r.z * r.z;
      Ixy += r.x * r.y; Ixz += r.x * r.z; Iyz += r.y * r.z;
      sx += r.x; sy += r.y; sz += r.z;
    };
    for (i64 a = n2c_ptr[n]; a < n2c_ptr[n + 1]; ++a) acc(C(n2c_idx[a]));
    for (i64 a = n2g_ptr[n]; a < n2g_ptr[n + 1]; ++a) {
      const i64 g = n2g_idx[a];
      acc(V3{gc[4 * g], gc[4 * g + 1], gc[4 * g + 2]});
    }
    const double D = Ixx * Iyy * Izz + 2 * Ixy * Ixz * Iyz - Ixx * Iyz * Iyz - Iyy * Ixz * Ixz - Izz * Ixy * Ixy;
    lx[n] = ((Iyz * Iyz - Iyy * Izz) * sx + (Ixy * Izz - Ixz * Iyz) * sy + (Ixz * Iyy - Ixy * Iyz) * sz) / D;
    ly[n] = ((Ixy * Izz - Ixz * Iyz) * sx + (Ixz * Ixz - Ixx * Izz) * sy + (Iyz * Ixx - Ixz * Ixy) * sz) / D;
    lz[n] = ((Ixz * Iyy - Ixy * Iyz) * sx + (Iyz * Ixx - Ixz * Ixy) * sy + (Ixy * Ixy - Ixx * Iyy) * sz) / D;
    Rx[n] = sx; Ry[n] = sy; Rz[n] = sz;
    number[n] = (i32)((n2c_ptr[n + 1] - n2c_ptr[n]) + (n2g_ptr[n + 1] - n2g_ptr[n]));
  }

  // ---- diamond vectors and coefficients
  std::vector<double> F1(3 * nf), F2(3 * nf), air(nf), p1(nf), p2(nf), p3(nf), zero3(3 * nf, 0.0), zero(nf, 0.0);
  for (i64 f = 0; f < nf; ++f) {
    const bool inner = name[f] == 0;
    const V3 v1 = C(f0[f]);
    const V3 v2 = inner ? C(f1[f]) : V3{gc[4 * f], gc[4 * f + 1], gc[4 * f + 2]};
    const V3 A1 = P(fn0[f]), A2 = P(fn1[f]), A3 = P(fn2[f]), A4 = A3;
    const V3 s1 = sub(v2, A2), s2 = sub(A4, A2), s3 = sub(v1, A2);
    const V3 g1 = add(scale(0.5, cross(s1, s2)), scale(0.5, cross(s2, s3)));
    const V3 s4 = sub(v2, A3), s5 = sub(A1, A3), s6 = sub(v1, A3);
    const V3 g2 = add(scale(0.5, cross(s4, s5)), scale(0.5, cross(s5, s6)));
    const V3 n = N(f);
    air[f] = dot(n, sub(v2, v1));
    p1[f] = dot(g1, n) / air[f];
    p2[f] = dot(g2, n) / air[f];
    p3[f] = dot(n, n) / air[f];
    F1[3 * f] = g1.x; F1[3 * f + 1] = g1.y; F1[3 * f + 2] = g1.z;
    F2[3 * f] = g2.x; F2[3 * f + 1] = g2.y; F2[3 * f + 2] = g2.z;
  }

  // ---- output
  auto to32 = [](const std::vector<i64> &v) { return std::vector<i32>(v.begin(), v.end()); };
  std::vector<i32> nodeid(el, el + 5 * nc), fcid(2 * nf), fnid(4 * nf);
  for (i64 f = 0; f < nf; ++f) {
    fcid[2 * f] = (i32)f0[f]; fcid[2 * f + 1] = (i32)f1[f];
    fnid[4 * f] = (i32)fn0[f]; fnid[4 * f + 1] = (i32)fn1[f]; fnid[4 * f + 2] = (i32)fn2[f]; fnid[4 * f + 3] = 3;
  }
  res->add("A.cells_nodeid", 'i', {nc, 5}, nodeid);
  res->add("A.nodes_vertex", 'd', {nn, 4}, std::vector<double>(vx, vx + 4 * nn));
  res->add("A.cells_center", 'd', {nc, 3}, cc);
  res->add("A.cells_volume", 'd', {nc}, vol);
  res->add("A.n2c_ptr", 'l', {nn + 1}, n2c_ptr);
  res->add("A.n2c_idx", 'i', {(i64)n2c_idx.size()}, to32(n2c_idx));
  res->add("A.cellnid_ptr", 'l', {nc + 1}, cnid_ptr);
  res->add("A.cellnid_idx", 'i', {(i64)cnid_idx.size()}, to32(cnid_idx));
  res->add("A.faces_cellid", 'i', {nf, 2}, fcid);
  res->add("A.cells_faceid", 'i', {nc, 5}, faceid);
  res->add("A.cells_cellfid", 'i', {nc, 5}, cellfid);
  res->add("A.faces_nodeid", 'i', {nf, 4}, fnid);
  res->add("A.faces_name", 'i', {nf}, name);
  res->add("A.faces_normal", 'd', {nf, 3}, nrm);
  res->add("A.faces_mesure", 'd', {nf}, mes);
  res->add("A.faces_center", 'd', {nf, 3}, fcen);
  res->add("A.nodes_name", 'i', {nn}, namen);
  static const char *LN[7] = {"A.innerfaces", "A.infaces", "A.outfaces", "A.upperfaces", "A.bottomfaces",
                              "A.frontfaces", "A.backfaces"};
  for (int t = 0; t < 7; ++t) res->add(LN[t], 'i', {(i64)lists[t].size()}, to32(lists[t]));
  res->add("A.boundaryfaces", 'i', {(i64)bfaces.size()}, to32(bfaces));
  const std::vector<i32> none;
  res->add("A.halofaces", 'i', {0}, none);
  res->add("A.periodicboundaryfaces", 'i', {0}, none);
  res->add("A.unmatched_boundary_faces", 'i', {0}, none);
  res->add("A.faces_ghostcenter", 'd', {nf, 4}, gc);
  res->add("A.n2g_ptr", 'l', {nn + 1}, n2g_ptr);
  res->add("A.n2g_idx", 'i', {(i64)n2g_idx.size()}, to32(n2g_idx));
  res->add("A.ghostnid_ptr", 'l', {nc + 1}, gnid_ptr);
  res->add("A.ghostnid_idx", 'i', {(i64)gnid_idx.size()}, to32(gnid_idx));
  res->add("A.nodes_R_x", 'd', {nn}, Rx);
  res->add("A.nodes_R_y", 'd', {nn}, Ry);
  res->add("A.nodes_R_z", 'd', {nn}, Rz);
  res->add("A.nodes_lambda_x", 'd', {nn}, lx);
  res->add("A.nodes_lambda_y", 'd', {nn}, ly);
  res->add("A.nodes_lambda_z", 'd', {nn}, lz);
  res->add("A.nodes_number", 'i', {nn}, number);
  res->add("A.faces_param1", 'd', {nf}, p1);
  res->add("A.faces_param2", 'd', {nf}, p2);
  res->add("A.faces_param3", 'd', {nf}, p3);
  res->add("A.faces_f_1", 'd', {nf, 3}, F1);
  res->add("A.faces_f_2", 'd', {nf, 3}, F2);
  res->add("A.faces_f_3", 'd', {nf, 3}, zero3);
  res->add("A.faces_f_4", 'd', {nf, 3}, zero3);
  res->add("A.faces_airDiamond", 'd', {nf}, air);
  res->add("A.faces_dist_ortho", 'd', {nf}, zero);
  return res;
}

}  // namespace

extern "C" void *mbh_geometry3d(const int32_t *elements, int64_t nbcells, const double *vertex, int64_t nbnodes) {
  if (!elements || !vertex || nbcells <= 0 || nbnodes <= 0) return nullptr;
  return geometry3d(elements, nbcells, vertex, nbnodes);
}
