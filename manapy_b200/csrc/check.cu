// State checks: non-finite and negative values (the error statuses a caller raises on).
#include "fv_common.cuh"

namespace mb {

template <class T>
__global__ void __launch_bounds__(kBlock) k_check(const T *__restrict__ v, long long n, int nonneg, int32_t *flags) {
  int f = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T x = v[i];
    if (!isfinite(x)) f |= 1;
    if (nonneg && x < T(0)) f |= 2;
  }
  f = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

}  // namespace mb

extern "C" int mb_check_state(const double *f64, const float *f32, int64_t n, int32_t nonneg, int32_t *flags,
                              void *stream) {
  MB_NVTX();
  if (!flags || n < 0 || (f64 == nullptr) == (f32 == nullptr)) return MB_EINVAL;
  if (n == 0) return MB_OK;
  long long blocks = (n + mb::kBlock - 1) / mb::kBlock;
  const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
  cudaStream_t st = (cudaStream_t)stream;
  if (f64)
    mb::k_check<<<grid, mb::kBlock, 0, st>>>(f64, (long long)n, nonneg, flags);
  else
    mb::k_check<<<grid, mb::kBlock, 0, st>>>(f32, (long long)n, nonneg, flags);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

// ---------------------------------------------------------------- index tables of a mesh
//
// One launch per table present in the mb_mesh: every entry of an index table is checked
// against the range a kernel may gather with it, and every offset table against being
// non-decreasing from 0 (multiples of 32 for the SELL-32 group offsets).  The first bad
// entry, smallest (table, position), is recorded in *first as table << 40 | offsets-flag
// << 39 | position.  A CSR or SELL table's last offset is taken as the length of its index
// array (the check cannot see allocation sizes).

namespace mb {

struct TableCheck {
  const int32_t *a;    // dense table, or the index array of a CSR / SELL table
  const int32_t *ptr;  // CSR row offsets or SELL group offsets; null for a dense table
  long long rows;      // dense rows, CSR rows or SELL groups
  int cols, used;      // dense: row stride and the leading columns that are checked
  int lo, hi;          // accepted values [lo, hi)
  int sell;            // offsets are SELL-32 group offsets
};

__global__ void __launch_bounds__(kBlock) k_check_table(TableCheck t, int id, unsigned long long *first) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long step = (long long)gridDim.x * blockDim.x;
  const unsigned long long key = (unsigned long long)id << 40;
  if (!t.ptr) {
    for (long long e = tid; e < t.rows * t.used; e += step) {
      const long long pos = (e / t.used) * t.cols + e % t.used;
      const int v = t.a[pos];
      if (v < t.lo || v >= t.hi) atomicMin(first, key | (unsigned long long)pos);
    }
    return;
  }
  for (long long r = tid; r <= t.rows; r += step) {
    const int p = t.ptr[r];
    if ((r == 0 && p != 0) || (r > 0 && p < t.ptr[r - 1]) || (t.sell && (p & 31)))
      atomicMin(first, key | (1ull << 39) | (unsigned long long)r);
  }
  const long long n = t.ptr[t.rows];
  if (n < 0) return;
  for (long long e = tid; e < n; e += step) {
    const int v = t.a[e];
    if (v < t.lo || v >= t.hi) atomicMin(first, key | (unsigned long long)e);
  }
}

inline void check_one(const TableCheck &t, int id, unsigned long long *first, cudaStream_t st) {
  if (!t.a || t.rows <= 0) return;
  k_check_table<<<148 * 4, kBlock, 0, st>>>(t, id, first);
}

}  // namespace mb

extern "C" int mb_check_tables(const mb_mesh *m, uint64_t *first, void *stream) {
  MB_NVTX();
  using mb::TableCheck;
  if (!m || !first || (m->dim != 2 && m->dim != 3) || m->nbcells <= 0 || m->nbfaces <= 0 || m->nbnodes <= 0)
    return MB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long *f = reinterpret_cast<unsigned long long *>(first);
  if (cudaMemsetAsync(f, 0xff, sizeof(unsigned long long), st) != cudaSuccess) return MB_ECUDA;
  const int nc = m->nbcells, nf = m->nbfaces, nn = m->nbnodes, nlf = m->dim == 2 ? 3 : 4;
  const long long ncg = (nc + 31) / 32, nng = (nn + 31) / 32;
  // ids: the order of the tables in mb_check_table_names (manapy_b200/_lib.py: CHECK_TABLES)
  mb::check_one(TableCheck{m->cell_faces, nullptr, nc, 4, nlf, 0, nf, 0}, 0, f, st);
  mb::check_one(TableCheck{m->cellnid_idx, m->cellnid_ptr, nc, 0, 0, 0, nc, 0}, 1, f, st);
  mb::check_one(TableCheck{m->ghostnid_idx, m->ghostnid_ptr, nc, 0, 0, 0, nf, 0}, 2, f, st);
  mb::check_one(TableCheck{m->face_cellid, nullptr, nf, 2, 1, 0, nc, 0}, 3, f, st);
  mb::check_one(TableCheck{m->face_cellid ? m->face_cellid + 1 : nullptr, nullptr, nf, 2, 1, -1, nc, 0}, 4, f, st);
  mb::check_one(TableCheck{m->face_nodeid, nullptr, nf, 4, m->dim, 0, nn, 0}, 5, f, st);
  mb::check_one(TableCheck{m->n2c_idx, m->n2c_ptr, nn, 0, 0, 0, nc, 0}, 6, f, st);
  mb::check_one(TableCheck{m->n2g_idx, m->n2g_ptr, nn, 0, 0, 0, nf, 0}, 7, f, st);
  mb::check_one(TableCheck{m->cell_cellfid, nullptr, nc, 4, 3, 0, nc, 0}, 8, f, st);
  mb::check_one(TableCheck{m->cell_vtx, nullptr, nc, 4, nlf, 0, nn, 0}, 9, f, st);
  mb::check_one(TableCheck{m->cell_nbr, nullptr, nc, 4, nlf, -nf, nc, 0}, 10, f, st);
  mb::check_one(TableCheck{m->lsq_sell_idx, m->lsq_sell_ptr, ncg, 0, 0, -1, nc, 1}, 11, f, st);
  mb::check_one(TableCheck{m->n2c_sell_idx, m->n2c_sell_ptr, nng, 0, 0, 0, nc, 1}, 12, f, st);
  if (m->cell_edges && m->nbedges > 0) {
    const int ne = m->nbedges;
    mb::check_one(TableCheck{m->cell_edges, nullptr, nc, 8, 6, 0, ne, 0}, 13, f, st);
    mb::check_one(TableCheck{m->edge_origin, nullptr, ne, 1, 1, 0, nn, 0}, 14, f, st);
    mb::check_one(TableCheck{m->edge_sell_idx, m->edge_sell_ptr, (ne + 31) / 32, 0, 0, -1, nc, 1}, 15, f, st);
    mb::check_one(TableCheck{m->n2c_sum_idx, m->n2c_sum_ptr, nng, 0, 0, -1, nc, 1}, 16, f, st);
  }
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}
