// Native host builder of the device tables of a 2D triangle mesh.
//
// One pass from (elements, vertex) -- the layout of manapy's per-rank mesh files
// (manapy/ddm/pure_ddm.py:21-33) -- to every table the CUDA kernels read, in
// the locality numbering, without building manapy's Domain arrays first.  It
// computes the same numbers as the vectorised Python path (geometry.build +
// DeviceMesh), operation for operation, so its output is bit-identical to it:
//
//   cell centres / volumes           manapy/ddm/ddm_utils2d.py:433-452
//   node -> cells, vertex neighbours ddm_utils2d.py:55-97
//   faces (unique descending node pairs, numbered in ascending order), cell -> face,
//   face -> cells, face neighbours   manapy/ddm/domain.py:313-315, ddm_utils2d.py:12-53
//   face names, normals, areas       ddm_utils2d.py:507-551
//   outward normals per cell         ddm_utils2d.py:99-120
//   ghost centres, node -> ghosts    ddm_utils2d.py:163-197, 122-161
//   centre -> vertex weights         ddm_utils2d.py:608-705, manapy/ast/functions2d.py:219
//   diamond vectors, areas           ddm_utils2d.py:553-605
//   orthogonal distances             ddm_utils2d.py:716-744
//
// then the Morton / face / node renumbering and the compact, SELL-32 and FP32
// tables.  Compiled with -ffp-contract=off: every operation rounds as written.
//
// C ABI: mbh_build2d() returns a handle holding named tables (dtype, shape, bytes);
// mbh_count / mbh_info / mbh_data read them; mbh_free releases the handle.
#include "common.hpp"

namespace {

using namespace mbh;

Result *build2d(const i32 *el, i64 nc, const double *vx, i64 nn, bool reorder, bool full, bool shared) {
  auto *res = new Result();
  for (i64 c = 0; c < nc; ++c)
    if (el[4 * c + 3] != 3) {
      res->error = "2D meshes must be all triangles";
      return res;
    }
  auto X = [&](i64 n) { return vx[4 * n]; };
  auto Y = [&](i64 n) { return vx[4 * n + 1]; };
  auto Zv = [&](i64 n) { return vx[4 * n + 2]; };
  auto node = [&](i64 c, int j) { return (i64)el[4 * c + j]; };

  // ---- cell centre and volume
  std::vector<double> cx(nc), cy(nc), vol(nc);
  parallel_for(nc, [&](i64 c) {
    const double x1 = X(node(c, 0)), x2 = X(node(c, 1)), x3 = X(node(c, 2));
    const double y1 = Y(node(c, 0)), y2 = Y(node(c, 1)), y3 = Y(node(c, 2));
    cx[c] = 1.0 / 3 * (x1 + x2 + x3);
    cy[c] = 1.0 / 3 * (y1 + y2 + y3);
    vol[c] = 0.5 * std::fabs((x1 - x2) * (y1 - y3) - (x1 - x3) * (y1 - y2));
  });
  // ---- node -> cells, cell -> vertex neighbours
  std::vector<i64> flat_nodes(3 * nc), flat_cells(3 * nc), c2n_ptr(nc + 1);
  for (i64 c = 0; c < nc; ++c)
    for (int j = 0; j < 3; ++j) {
      flat_nodes[3 * c + j] = node(c, j);
      flat_cells[3 * c + j] = c;
    }
  for (i64 c = 0; c <= nc; ++c) c2n_ptr[c] = 3 * c;
  std::vector<i64> n2c_ptr, n2c_idx;
  group_csr(flat_nodes, flat_cells, nn, n2c_ptr, n2c_idx);
  std::vector<i64> cnid_ptr, cnid_idx;
  ragged_union(nc, c2n_ptr, flat_nodes, n2c_ptr, n2c_idx, true, cnid_ptr, cnid_idx);

  // ---- faces: descending node pairs, numbered by ascending key
  static const int LOC[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  std::vector<i64> key(3 * nc), pa(3 * nc), pb(3 * nc);
  parallel_for(nc, [&](i64 c) {
    for (int j = 0; j < 3; ++j) {
      i64 a = node(c, LOC[j][0]), b = node(c, LOC[j][1]);
      if (a < b) std::swap(a, b);
      pa[3 * c + j] = a;
      pb[3 * c + j] = b;
      key[3 * c + j] = a * nn + b;
    }
  });
  // stable order of the keys (a, b): two counting-sort passes, by b then by a
  std::vector<i64> ord;
  {
    std::vector<i64> tmp;
    stable_by_digit(pb, nullptr, 3 * nc, nn, tmp);
    stable_by_digit(pa, &tmp, 3 * nc, nn, ord);
  }
  std::vector<i64> inv(3 * nc);
  std::vector<i64> fa, fb;  // face nodes (descending)
  std::vector<i64> f0, f1;  // face -> cells
  for (size_t e = 0; e < ord.size(); ++e) {
    const i64 o = ord[e];
    if (e == 0 || key[o] != key[ord[e - 1]]) {
      fa.push_back(pa[o]);
      fb.push_back(pb[o]);
      f0.push_back(o / 3);
      f1.push_back(-1);
    } else {
      if (f1.back() != -1) {
        res->error = "non-manifold mesh: a face is shared by more than two cells";
        return res;
      }
      f1.back() = o / 3;
    }
    inv[o] = (i64)fa.size() - 1;
  }
  const i64 nf = (i64)fa.size();
  // face neighbours, compacted (boundary faces skipped)
  std::vector<i64> cellfid(3 * nc, -1);
  parallel_for(nc, [&](i64 c) {
    int k = 0;
    for (int j = 0; j < 3; ++j) {
      const i64 f = inv[3 * c + j];
      if (f1[f] == -1) continue;
      cellfid[3 * c + k++] = f0[f] == c ? f1[f] : f0[f];
    }
  });
  // ---- names, normals, areas, centres
  std::vector<i32> namen(nn);
  for (i64 n = 0; n < nn; ++n) namen[n] = (i32)vx[4 * n + 3];
  std::vector<i32> name(nf, 0);
  std::vector<double> nx(nf), ny(nf), nz(nf), mes(nf), fcx(nf), fcy(nf), fcz(nf);
  parallel_for(nf, [&](i64 f) {
    if (f1[f] == -1) {
      const i32 a = namen[fa[f]], b = namen[fb[f]];
      i32 r = 100;
      for (i32 tag : {44, 33, 4, 3})
        if ((a == tag && b != 0) || (a != 0 && b == tag)) r = tag;
      if (a == b) r = a;
      name[f] = r;
    }
    const double n0 = Y(fa[f]) - Y(fb[f]), n1 = X(fb[f]) - X(fa[f]);
    fcx[f] = 0.5 * (X(fa[f]) + X(fb[f]));
    fcy[f] = 0.5 * (Y(fa[f]) + Y(fb[f]));
    fcz[f] = 0.5 * (Zv(fa[f]) + Zv(fb[f]));
    const double sx = cx[f0[f]] - fcx[f], sy = cy[f0[f]] - fcy[f];
    const bool flip = (sx * n0 + sy * n1) > 0;
    nx[f] = flip ? -1 * n0 : n0;
    ny[f] = flip ? -1 * n1 : n1;
    nz[f] = flip ? -1 * 0.0 : 0.0;
    mes[f] = std::sqrt(nx[f] * nx[f] + ny[f] * ny[f]);
  });
  for (i64 f = 0; f < nf; ++f)
    if (f1[f] == -1 && (name[f] >= 100 || name[f] == 0)) {
      res->error = "mesh has boundary faces that match no boundary side (manapy names them 100/200 and "
                   "leaves them out of every face list)";
      return res;
    }
  // outward normal of each local face (cells.nf)
  uvec<double> cnf(9 * nc);
  parallel_for(nc, [&](i64 c) {
    for (int j = 0; j < 3; ++j) {
      const i64 f = inv[3 * c + j];
      const double s = (cx[c] - fcx[f]) * nx[f] + (cy[c] - fcy[f]) * ny[f] + (0.0 - fcz[f]) * nz[f];
      const bool keep = s < 0;
      cnf[9 * c + 3 * j + 0] = keep ? nx[f] : -1.0 * nx[f];
      cnf[9 * c + 3 * j + 1] = keep ? ny[f] : -1.0 * ny[f];
      cnf[9 * c + 3 * j + 2] = keep ? nz[f] : -1.0 * nz[f];
    }
  });
  // ---- face lists (manapy numbering)
  std::vector<i64> lists[5];
  std::vector<i64> bfaces;
  for (i64 f = 0; f < nf; ++f) {
    if (name[f] >= 0 && name[f] <= 4) lists[name[f]].push_back(f);
    if (name[f] >= 1 && name[f] <= 4) bfaces.push_back(f);
  }
  // ---- ghost centres
  std::vector<double> gc(3 * nf, -1.0);
  parallel_for((i64)bfaces.size(), [&](i64 i) {
    const i64 f = bfaces[i];
    const double x1x = X(fb[f]), x1y = Y(fb[f]), x2x = X(fa[f]), x2y = Y(fa[f]);
    const double v1x = cx[f0[f]], v1y = cy[f0[f]];
    const double gamma = ((v1x - x2x) * (x1x - x2x) + (v1y - x2y) * (x1y - x2y)) /
                         ((x1x - x2x) * (x1x - x2x) + (x1y - x2y) * (x1y - x2y));
    const double kk0 = gamma * x1x + (1 - gamma) * x2x, kk1 = gamma * x1y + (1 - gamma) * x2y;
    gc[3 * f] = 2 * kk0 + (-1 * v1x);
    gc[3 * f + 1] = 2 * kk1 + (-1 * v1y);
    gc[3 * f + 2] = gamma;
  });
  // node -> boundary faces (ascending face), cell -> stencil ghosts
  std::vector<i64> gkey, gval;
  for (i64 f : bfaces) {
    gkey.push_back(fa[f]);
    gval.push_back(f);
    gkey.push_back(fb[f]);
    gval.push_back(f);
  }
  std::vector<i64> n2g_ptr, n2g_idx;
  group_csr(gkey, gval, nn, n2g_ptr, n2g_idx);
  std::vector<i64> gnid_ptr, gnid_idx;
  ragged_union(nc, c2n_ptr, flat_nodes, n2g_ptr, n2g_idx, false, gnid_ptr, gnid_idx);
  // ---- centre -> vertex weights
  std::vector<double> lx(nn), ly(nn), Rx(nn), Ry(nn);
  std::vector<i64> number(nn);
  parallel_for(nn, [&](i64 n) {
    double xx = 0, yy = 0, xy = 0, sx = 0, sy = 0;
    auto acc = [&](double px, double py) {
      const double rx = px - X(n), ry = py - Y(n);
      xx += rx * rx;
      yy += ry * ry;
      xy += rx * ry;
      sx += rx;
      sy += ry;
    };
    for (i64 a = n2c_ptr[n]; a < n2c_ptr[n + 1]; ++a) acc(cx[n2c_idx[a]], cy[n2c_idx[a]]);
    for (i64 a = n2g_ptr[n]; a < n2g_ptr[n + 1]; ++a) acc(gc[3 * n2g_idx[a]], gc[3 * n2g_idx[a] + 1]);
    const double D = xx * yy - xy * xy;
    lx[n] = (xy * sy - yy * sx) / D;
    ly[n] = (xy * sx - xx * sy) / D;
    Rx[n] = sx;
    Ry[n] = sy;
    number[n] = (n2c_ptr[n + 1] - n2c_ptr[n]) + (n2g_ptr[n + 1] - n2g_ptr[n]);
  });
  auto alpha = [&](i64 n, double px, double py) {
    const double den = (double)number[n] + lx[n] * Rx[n] + ly[n] * Ry[n];
    const double xd = px - X(n), yd = py - Y(n);
    return (1. + lx[n] * xd + ly[n] * yd) / den;
  };
  // ---- diamond vectors and areas, orthogonal distances
  uvec<double> ff(8 * nf), air(nf), dist(nf);
  auto proj = [&](i64 K, i64 f) {
    const double vx_ = cx[K] - fcx[f], vy_ = cy[K] - fcy[f];
    const double s = vx_ * nx[f] + vy_ * ny[f];
    const double px = cx[K] - s * nx[f], py = cy[K] - s * ny[f];
    const double z0 = cx[K] - px, z1 = cy[K] - py;
    return std::sqrt(z0 * z0 + z1 * z1);
  };
  parallel_for(nf, [&](i64 f) {
    const bool inner = name[f] == 0;
    const double v1x = cx[f0[f]], v1y = cy[f0[f]];
    const double v2x = inner ? cx[f1[f]] : gc[3 * f], v2y = inner ? cy[f1[f]] : gc[3 * f + 1];
    const double ax = X(fa[f]), ay = Y(fa[f]), bx = X(fb[f]), by = Y(fb[f]);
    double *F = &ff[8 * f];
    F[0] = v1x - ax; F[1] = v1y - ay;
    F[2] = bx - v1x; F[3] = by - v1y;
    F[4] = v2x - bx; F[5] = v2y - by;
    F[6] = ax - v2x; F[7] = ay - v2y;
    air[f] = 0.5 * ((bx - ax) * (v2y - v1y) + (v1x - v2x) * (by - ay));
    if (inner)
      dist[f] = proj(f0[f], f) + proj(f1[f], f);
    else if (name[f] >= 1 && name[f] <= 4)
      dist[f] = 2 * proj(f0[f], f);
    else
      dist[f] = 0.0;
  });

  // ---- locality numbering
  std::vector<i64> cperm(nc), fperm(nf), nperm(nn);
  if (reorder) {
    double lo0 = cx[0], lo1 = cy[0], hi0 = cx[0], hi1 = cy[0];
    for (i64 c = 1; c < nc; ++c) {
      lo0 = std::min(lo0, cx[c]); hi0 = std::max(hi0, cx[c]);
      lo1 = std::min(lo1, cy[c]); hi1 = std::max(hi1, cy[c]);
    }
    const double sp0 = std::max(hi0 - lo0, 1e-300), sp1 = std::max(hi1 - lo1, 1e-300);
    const double scale = (double)((1 << 20) - 1);
    std::vector<uint64_t> mk(nc);
    parallel_for(nc, [&](i64 c) {
      const i64 q0 = (i64)std::floor((cx[c] - lo0) / sp0 * scale), q1 = (i64)std::floor((cy[c] - lo1) / sp1 * scale);
      mk[c] = part1by1((uint64_t)q0) | (part1by1((uint64_t)q1) << 1);
    });
    cperm = radix_argsort(mk);
  } else {
    std::iota(cperm.begin(), cperm.end(), 0);
  }
  std::vector<i64> cinv(nc);
  for (i64 k = 0; k < nc; ++k) cinv[cperm[k]] = k;
  if (reorder) {
    std::vector<i64> lo(nf), hi(nf);
    parallel_for(nf, [&](i64 f) {
      const i64 a = cinv[f0[f]], b = f1[f] >= 0 ? cinv[f1[f]] : a;
      lo[f] = std::min(a, b);
      hi[f] = std::max(a, b);
    });
    // stable order of (lo, hi): by hi, then stably by lo
    std::vector<i64> byhi;
    stable_by_digit(hi, nullptr, nf, nc, byhi);
    stable_by_digit(lo, &byhi, nf, nc, fperm);
    // nodes by their first cell (nodes in no cell last)
    std::vector<i64> first(nn, nc);
    parallel_for(nn, [&](i64 n) {
      for (i64 a = n2c_ptr[n]; a < n2c_ptr[n + 1]; ++a) first[n] = std::min(first[n], cinv[n2c_idx[a]]);
    });
    nperm = counting_argsort(first, nc + 1);
  } else {
    std::iota(fperm.begin(), fperm.end(), 0);
    std::iota(nperm.begin(), nperm.end(), 0);
  }
  std::vector<i64> finv(nf), ninv(nn);
  for (i64 k = 0; k < nf; ++k) finv[fperm[k]] = k;
  for (i64 k = 0; k < nn; ++k) ninv[nperm[k]] = k;

  auto relabel = [](const std::vector<i64> &ptr, const std::vector<i64> &idx, const std::vector<i64> &rows,
                    const std::vector<i64> &vinv, std::vector<i64> &optr, std::vector<i64> &oidx,
                    std::vector<i64> *src) { relabel_csr(ptr, idx, rows, vinv, optr, oidx, src); };
  auto to32 = [](const std::vector<i64> &v) {
    uvec<i32> o(v.size());
    parallel_for((i64)v.size(), [&](i64 i) { o[i] = (i32)v[i]; });
    return o;
  };

  // ---- device tables
  {
    uvec<double> t(3 * nc);
    parallel_for(nc, [&](i64 k) { t[3 * k] = cx[cperm[k]]; t[3 * k + 1] = cy[cperm[k]]; t[3 * k + 2] = 0.0; });
    res->add("cell_center", 'd', {nc, 3}, std::move(t));
    uvec<double> v(nc);
    parallel_for(nc, [&](i64 k) { v[k] = vol[cperm[k]]; });
    res->add("cell_volume", 'd', {nc}, std::move(v));
  }
  {
    uvec<i32> cf(4 * nc);
    uvec<uint8_t> code(nc);
    parallel_for(nc, [&](i64 k) {
      const i64 c = cperm[k];
      i64 fo[3];
      for (int j = 0; j < 3; ++j) { fo[j] = inv[3 * c + j]; cf[4 * k + j] = (i32)finv[fo[j]]; }
      cf[4 * k + 3] = -1;
      int o[3] = {0, 1, 2};  // stable order of the three face ids
      if (fo[o[1]] < fo[o[0]]) std::swap(o[0], o[1]);
      if (fo[o[2]] < fo[o[1]]) std::swap(o[1], o[2]);
      if (fo[o[1]] < fo[o[0]]) std::swap(o[0], o[1]);
      code[k] = (uint8_t)(o[0] | (o[1] << 2) | (o[2] << 4));
    });
    res->add("cell_faces", 'i', {nc, 4}, std::move(cf));
    res->add("cell_order", 'b', {nc}, std::move(code));
  }
  {
    std::vector<i64> p, ix;
    relabel(cnid_ptr, cnid_idx, cperm, cinv, p, ix, nullptr);
    res->add("cellnid_ptr", 'i', {nc + 1}, to32(p));
    res->add("cellnid_idx", 'i', {(i64)ix.size()}, to32(ix));
    std::vector<i32> gp, gi;
    std::vector<double> gv;
    if (shared)
      sell32_aligned(p, ix, 0, gp, gi);  // the slot-shared layout
    else
      sell32(p, ix, nullptr, false, gp, gi, gv);  // manapy's order, -1 after each row
    res->add("lsq_sell_ptr", 'i', {(i64)gp.size()}, std::move(gp));
    res->add("lsq_sell_idx", 'i', {(i64)gi.size()}, std::move(gi));
    relabel(gnid_ptr, gnid_idx, cperm, finv, p, ix, nullptr);
    res->add("ghostnid_ptr", 'i', {nc + 1}, to32(p));
    res->add("ghostnid_idx", 'i', {(i64)ix.size()}, to32(ix));
  }
  {
    uvec<i32> cid(2 * nf), fn(4 * nf), nm(nf);
    uvec<double> nrm(3 * nf), fc(3 * nf), ms(nf), g(3 * nf), a(nf), F(8 * nf), d(nf);
    uvec<float> nm32(4 * nf);
    parallel_for(nf, [&](i64 k) {
      const i64 f = fperm[k];
      cid[2 * k] = (i32)cinv[f0[f]];
      cid[2 * k + 1] = f1[f] >= 0 ? (i32)cinv[f1[f]] : -1;
      fn[4 * k] = (i32)ninv[fa[f]];
      fn[4 * k + 1] = (i32)ninv[fb[f]];
      fn[4 * k + 2] = -1;
      fn[4 * k + 3] = -1;
      nm[k] = name[f];
      nrm[3 * k] = nx[f]; nrm[3 * k + 1] = ny[f]; nrm[3 * k + 2] = nz[f];
      fc[3 * k] = fcx[f]; fc[3 * k + 1] = fcy[f]; fc[3 * k + 2] = fcz[f];
      ms[k] = mes[f];
      nm32[4 * k] = (float)nx[f];
      nm32[4 * k + 1] = (float)ny[f];
      nm32[4 * k + 2] = (float)(1.0 / mes[f]);
      nm32[4 * k + 3] = 0.f;
      for (int c = 0; c < 3; ++c) g[3 * k + c] = gc[3 * f + c];
      a[k] = air[f];
      for (int c = 0; c < 8; ++c) F[8 * k + c] = ff[8 * f + c];
      d[k] = dist[f];
    });
    res->add("face_cellid", 'i', {nf, 2}, std::move(cid));
    res->add("face_nodeid", 'i', {nf, 4}, std::move(fn));
    res->add("face_name", 'i', {nf}, std::move(nm));
    res->add("face_normal", 'd', {nf, 3}, std::move(nrm));
    res->add("face_center", 'd', {nf, 3}, std::move(fc));
    res->add("face_mesure", 'd', {nf}, std::move(ms));
    res->add("face_nm_f32", 'f', {nf, 4}, std::move(nm32));
    res->add("face_ghostcenter", 'd', {nf, 3}, std::move(g));
    res->add("face_air", 'd', {nf}, std::move(a));
    res->add("face_f", 'd', {nf, 8}, std::move(F));
    res->add("face_dist", 'd', {nf}, std::move(d));
  }
  {
    std::vector<i64> p, ix, src;
    relabel(n2c_ptr, n2c_idx, nperm, cinv, p, ix, &src);
    uvec<double> al(ix.size());
    parallel_for(nn, [&](i64 r) {  // row r of the new table is node nperm[r]
      const i64 n = nperm[r];
      for (i64 e = p[r]; e < p[r + 1]; ++e) {
        const i64 c = n2c_idx[src[e]];
        al[e] = alpha(n, cx[c], cy[c]);
      }
    });
    res->add("n2c_ptr", 'i', {nn + 1}, to32(p));
    res->add("n2c_idx", 'i', {(i64)ix.size()}, to32(ix));
    std::vector<double> alv(al.begin(), al.end());
    res->add("n2c_alpha", 'd', {(i64)al.size()}, std::move(al));
    std::vector<i32> gp, gi;
    std::vector<double> gv;
    sell32(p, ix, &alv, true, gp, gi, gv);
    uvec<float> gv32(gv.size());
    parallel_for((i64)gv.size(), [&](i64 i) { gv32[i] = (float)gv[i]; });
    res->add("n2c_sell_ptr", 'i', {(i64)gp.size()}, std::move(gp));
    res->add("n2c_sell_idx", 'i', {(i64)gi.size()}, std::move(gi));
    res->add("n2c_sell_alpha", 'd', {(i64)gv.size()}, std::move(gv));
    res->add("n2c_sell_alpha_f32", 'f', {(i64)gv32.size()}, std::move(gv32));
    relabel(n2g_ptr, n2g_idx, nperm, finv, p, ix, &src);
    uvec<double> ag(ix.size());
    parallel_for(nn, [&](i64 r) {
      const i64 n = nperm[r];
      for (i64 e = p[r]; e < p[r + 1]; ++e) {
        const i64 f = n2g_idx[src[e]];
        ag[e] = alpha(n, gc[3 * f], gc[3 * f + 1]);
      }
    });
    res->add("n2g_ptr", 'i', {nn + 1}, to32(p));
    res->add("n2g_idx", 'i', {(i64)ix.size()}, to32(ix));
    res->add("n2g_alpha", 'd', {(i64)ag.size()}, std::move(ag));
  }
  {
    uvec<i32> cf(4 * nc), vtx(4 * nc), nbr(4 * nc);
    uvec<uint32_t> flags(nc);
    uvec<double> nf_(9 * nc), v1(2 * nc), xy(2 * nc), ncoord(2 * nn);
    parallel_for(nc, [&](i64 k) {
      const i64 c = cperm[k];
      cf[4 * k + 3] = -1;
      vtx[4 * k + 3] = 0;
      nbr[4 * k + 3] = -1;
      for (int j = 0; j < 3; ++j) {
        const i64 o = cellfid[3 * c + j];
        cf[4 * k + j] = (i32)(o >= 0 ? cinv[o] : cinv[nc - 1]);
      }
      for (int q = 0; q < 9; ++q) nf_[9 * k + q] = cnf[9 * c + q];
      v1[2 * k] = X(node(c, 1));
      v1[2 * k + 1] = Y(node(c, 1));
      xy[2 * k] = cx[c];
      xy[2 * k + 1] = cy[c];
      uint32_t fl = 0;
      for (int j = 0; j < 3; ++j) {
        vtx[4 * k + j] = (i32)ninv[node(c, j)];
        const i64 f = inv[3 * c + j];
        const bool own = f0[f] == c;
        const i64 other = own ? f1[f] : f0[f];
        nbr[4 * k + j] = f1[f] < 0 ? (i32)(-1 - finv[f]) : (i32)cinv[other];
        const i64 vj = node(c, j), vn = node(c, (j + 1) % 3);
        const bool rev = fa[f] == vn;
        const i64 a = rev ? vn : vj, b = rev ? vj : vn;
        const double n0 = Y(a) - Y(b), n1 = X(b) - X(a);
        const bool flip = nx[f] != n0 || ny[f] != n1;
        const bool nfneg = cnf[9 * c + 3 * j] != nx[f] || cnf[9 * c + 3 * j + 1] != ny[f];
        fl |= ((uint32_t)own << j) | ((uint32_t)rev << (3 + j)) | ((uint32_t)flip << (6 + j)) |
              ((uint32_t)nfneg << (9 + j));
      }
      flags[k] = fl;
    });
    parallel_for(nn, [&](i64 r) { ncoord[2 * r] = X(nperm[r]); ncoord[2 * r + 1] = Y(nperm[r]); });
    res->add("cell_cellfid", 'i', {nc, 4}, std::move(cf));
    res->add("cell_nf", 'd', {nc, 3, 3}, std::move(nf_));
    res->add("cell_vertex1", 'd', {nc, 2}, std::move(v1));
    res->add("cell_vtx", 'i', {nc, 4}, std::move(vtx));
    res->add("cell_nbr", 'i', {nc, 4}, std::move(nbr));
    res->add("cell_flags", 'i', {nc}, std::move(flags));
    res->add("node_coord", 'd', {nn, 2}, std::move(ncoord));
    res->add("cell_xy", 'd', {nc, 2}, std::move(xy));
  }
  // permutations and the manapy-numbered arrays the boundary set-up reads
  res->add("perm_cell", 'l', {nc}, cperm);
  res->add("perm_face", 'l', {nf}, fperm);
  res->add("perm_node", 'l', {nn}, nperm);
  res->add("inv_cell", 'l', {nc}, cinv);
  res->add("inv_face", 'l', {nf}, finv);
  res->add("inv_node", 'l', {nn}, ninv);
  {
    uvec<double> fc(3 * nf), cc(3 * nc);
    parallel_for(nf, [&](i64 f) { fc[3 * f] = fcx[f]; fc[3 * f + 1] = fcy[f]; fc[3 * f + 2] = fcz[f]; });
    parallel_for(nc, [&](i64 c) { cc[3 * c] = cx[c]; cc[3 * c + 1] = cy[c]; cc[3 * c + 2] = 0.0; });
    res->add("A.faces_center", 'd', {nf, 3}, std::move(fc));
    res->add("A.cells_center", 'd', {nc, 3}, std::move(cc));
    static const char *LN[5] = {"A.innerfaces", "A.infaces", "A.outfaces", "A.upperfaces", "A.bottomfaces"};
    for (int t = 0; t < 5; ++t) res->add(LN[t], 'i', {(i64)lists[t].size()}, to32(lists[t]));
  }
  if (full) {
    // every array of geometry.build (manapy's Domain arrays, manapy numbering)
    std::vector<i32> nodeid(4 * nc), faceid(4 * nc), cfid(4 * nc);
    for (i64 c = 0; c < nc; ++c) {
      int k = 0;
      for (int j = 0; j < 4; ++j) nodeid[4 * c + j] = el[4 * c + j];
      for (int j = 0; j < 3; ++j) {
        faceid[4 * c + j] = (i32)inv[3 * c + j];
        cfid[4 * c + j] = (i32)cellfid[3 * c + j];
        if (cellfid[3 * c + j] != -1) ++k;
      }
      faceid[4 * c + 3] = 3;
      cfid[4 * c + 3] = k;
    }
    res->add("A.cells_nodeid", 'i', {nc, 4}, nodeid);
    res->add("A.cells_faceid", 'i', {nc, 4}, faceid);
    res->add("A.cells_cellfid", 'i', {nc, 4}, cfid);
    res->add("A.cells_volume", 'd', {nc}, vol);
    res->add("A.cells_nf", 'd', {nc, 3, 3}, cnf);
    res->add("A.n2c_ptr", 'l', {nn + 1}, n2c_ptr);
    res->add("A.n2c_idx", 'i', {(i64)n2c_idx.size()}, to32(n2c_idx));
    res->add("A.n2g_ptr", 'l', {nn + 1}, n2g_ptr);
    res->add("A.n2g_idx", 'i', {(i64)n2g_idx.size()}, to32(n2g_idx));
    res->add("A.cellnid_ptr", 'l', {nc + 1}, cnid_ptr);
    res->add("A.cellnid_idx", 'i', {(i64)cnid_idx.size()}, to32(cnid_idx));
    res->add("A.ghostnid_ptr", 'l', {nc + 1}, gnid_ptr);
    res->add("A.ghostnid_idx", 'i', {(i64)gnid_idx.size()}, to32(gnid_idx));
    std::vector<i32> fnid(3 * nf), fcid(2 * nf);
    std::vector<double> nrm(3 * nf), fdn[4], par[4];
    for (int k = 0; k < 4; ++k) {
      fdn[k].resize(2 * nf);
      par[k].resize(nf);
    }
    for (i64 f = 0; f < nf; ++f) {
      fnid[3 * f] = (i32)fa[f]; fnid[3 * f + 1] = (i32)fb[f]; fnid[3 * f + 2] = 2;
      fcid[2 * f] = (i32)f0[f]; fcid[2 * f + 1] = (i32)f1[f];
      nrm[3 * f] = nx[f]; nrm[3 * f + 1] = ny[f]; nrm[3 * f + 2] = nz[f];
      const double *F = &ff[8 * f];
      for (int k = 0; k < 4; ++k) { fdn[k][2 * f] = F[2 * k]; fdn[k][2 * f + 1] = F[2 * k + 1]; }
      // diamond coefficients (ddm_utils2d.py:602-605): pairs (f1, f2), (f2, f3), (f3, f4), (f4, f1)
      const double inv2a = 1.0 / (2.0 * air[f]);
      for (int k = 0; k < 4; ++k) {
        const int a = k, b = (k + 1) % 4;
        par[k][f] = inv2a * ((F[2 * a + 1] + F[2 * b + 1]) * nx[f] - (F[2 * a] + F[2 * b]) * ny[f]);
      }
    }
    res->add("A.faces_nodeid", 'i', {nf, 3}, fnid);
    res->add("A.faces_cellid", 'i', {nf, 2}, fcid);
    res->add("A.faces_name", 'i', {nf}, name);
    res->add("A.faces_normal", 'd', {nf, 3}, nrm);
    res->add("A.faces_mesure", 'd', {nf}, mes);
    res->add("A.faces_ghostcenter", 'd', {nf, 3}, gc);
    res->add("A.faces_airDiamond", 'd', {nf}, air);
    static const char *FN[4] = {"A.faces_f_1", "A.faces_f_2", "A.faces_f_3", "A.faces_f_4"};
    static const char *PN[4] = {"A.faces_param1", "A.faces_param2", "A.faces_param3", "A.faces_param4"};
    for (int k = 0; k < 4; ++k) {
      res->add(FN[k], 'd', {nf, 2}, fdn[k]);
      res->add(PN[k], 'd', {nf}, par[k]);
    }
    res->add("A.faces_dist_ortho", 'd', {nf}, dist);
    std::vector<double> vtx(vx, vx + 4 * nn), zero(nn, 0.0);
    res->add("A.nodes_vertex", 'd', {nn, 4}, vtx);
    res->add("A.nodes_name", 'i', {nn}, namen);
    res->add("A.nodes_R_x", 'd', {nn}, Rx);
    res->add("A.nodes_R_y", 'd', {nn}, Ry);
    res->add("A.nodes_R_z", 'd', {nn}, zero);
    res->add("A.nodes_lambda_x", 'd', {nn}, lx);
    res->add("A.nodes_lambda_y", 'd', {nn}, ly);
    res->add("A.nodes_lambda_z", 'd', {nn}, zero);
    res->add("A.nodes_number", 'i', {nn}, to32(number));
    res->add("A.boundaryfaces", 'i', {(i64)bfaces.size()}, to32(bfaces));
    const std::vector<i32> none;
    res->add("A.halofaces", 'i', {0}, none);
    res->add("A.periodicboundaryfaces", 'i', {0}, none);
    res->add("A.unmatched_boundary_faces", 'i', {0}, none);
  }
  return res;
}

}  // namespace

extern "C" {

// full != 0 also returns every array of geometry.build as "A.<name>" (manapy numbering);
// shared != 0 writes the least-squares stencil (lsq_sell_*) in the slot-shared SELL-32
// layout of sell32_aligned, else in manapy's neighbour order
void *mbh_build2d(const int32_t *elements, int64_t nbcells, const double *vertex, int64_t nbnodes, int32_t reorder,
                  int32_t full, int32_t shared) {
  if (!elements || !vertex || nbcells <= 0 || nbnodes <= 0) return nullptr;
  return build2d(elements, nbcells, vertex, nbnodes, reorder != 0, full != 0, shared != 0);
}

// the slot-shared SELL-32 (sell32_aligned) of a CSR table: tables "gptr" and "idx"
void *mbh_sell_aligned(const int64_t *ptr, int64_t n, const int32_t *idx, int32_t slack) {
  if (!ptr || n < 0 || slack < 0) return nullptr;
  auto *res = new Result();
  std::vector<i64> p(ptr, ptr + n + 1), ix(ptr[n]);
  for (i64 e = 0; e < ptr[n]; ++e) ix[e] = idx[e];
  std::vector<i64> len(n);
  i64 total = 0;
  for (i64 g = 0; g < (n + 31) / 32; ++g) {
    i64 m = 0;
    for (i64 r = 32 * g; r < std::min(n, 32 * g + 32); ++r) m = std::max(m, p[r + 1] - p[r]);
    total += 32 * (m + (m ? slack : 0));
  }
  if (total >= ((i64)1 << 31)) {
    res->error = "neighbour table too large for 32-bit offsets";
    return res;
  }
  std::vector<i32> gp, gi;
  sell32_aligned(p, ix, slack, gp, gi);
  res->add("gptr", 'i', {(i64)gp.size()}, gp);
  res->add("idx", 'i', {(i64)gi.size()}, gi);
  return res;
}

const char *mbh_error(void *h) { return h ? static_cast<Result *>(h)->error.c_str() : "null handle"; }

int32_t mbh_count(void *h) { return h ? (int32_t) static_cast<Result *>(h)->tables.size() : 0; }

// name, dtype code and up to 3 dimensions of table k; returns its number of dimensions
int32_t mbh_info(void *h, int32_t k, const char **name, char *dtype, int64_t shape[3]) {
  const Table &t = static_cast<Result *>(h)->tables[k];
  *name = t.name.c_str();
  *dtype = t.dtype;
  for (size_t d = 0; d < 3; ++d) shape[d] = d < t.shape.size() ? t.shape[d] : 0;
  return (int32_t)t.shape.size();
}

const void *mbh_data(void *h, int32_t k) { return static_cast<Result *>(h)->tables[k].data; }

void mbh_free(void *h) { delete static_cast<Result *>(h); }

}  // extern "C"
