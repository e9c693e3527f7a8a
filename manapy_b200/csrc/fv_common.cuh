// Shared device helpers of the explicit finite-volume kernels (sm_100a).
//
// All kernels are gathers: a thread owns one cell (or node, or face) and reads
// its neighbours; nothing is scattered, so there are no atomics except the
// dt min-reduction, whose result does not depend on order.  Sums that manapy
// accumulates into a cell are accumulated here in manapy's order, so results
// match manapy's serial loops to rounding.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "manapy_b200.h"

namespace mb {

// A named NVTX range over a C-ABI entry point: profilers show each call around the
// kernels it launches (header-only NVTX v3; without a tool attached a push/pop is a
// few nanoseconds of host time).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
#define MB_NVTX() ::mb::NvtxRange mb_nvtx_range_(__func__)

constexpr int kBlock = 256;

__host__ __device__ inline int ceil_div(long long a, int b) { return (int)((a + b - 1) / b); }

// Python's two-argument min/max: the first argument wins ties and NaN
// comparisons, as in manapy's min(...)/max(...).
__device__ __forceinline__ double pmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double pmax(double a, double b) { return b > a ? b : a; }

// Slot of a cell's local face visited k-th in manapy's accumulation order (2 bits per k).
__device__ __forceinline__ int order_slot(uint8_t code, int k) { return (code >> (2 * k)) & 3; }

// Read-only loads through the non-coherent path.
template <class T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// Ghost value of boundary face f from the live cell array (manapy/boundary/bc_utils.py:45-68).
struct GhostRule {
  const int8_t *kind;
  const double *value;
  const double *dist;
  const int32_t *face_cellid;
  const double *w;
  __device__ __forceinline__ double operator()(int f) const {
    const int k = kind[f];
    if (k == MB_G_DIRICHLET) return ld(value + f);
    const double wc = ld(w + ld(face_cellid + 2 * f));
    if (k == MB_G_NEUMANN) return wc;
    if (k == MB_G_NONSLIP) return -1 * wc;
    if (k == MB_G_NEUMANN_NH) return wc + ld(value + f) * ld(dist + f);
    if (k == MB_G_CELL_AT_FACE) return ld(w + (long long)ld(value + f));
    return 0.0;
  }
};

// Ghost value read from an explicit ghost array (the w_ghost argument of manapy's kernels).
struct GhostArray {
  const double *g;
  __device__ __forceinline__ double operator()(int f) const { return ld(g + f); }
};

__device__ __forceinline__ GhostRule make_rule(const mb_mesh &m, const mb_bc &bc, const double *w) {
  return GhostRule{bc.kind, bc.value, m.face_dist, m.face_cellid, w};
}

// dt min-reduction: positive doubles order like their bit patterns, so an
// unsigned 64-bit atomicMin is an exact, order-independent min.
__device__ __forceinline__ void atomic_min_pos(double *addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double block_min(double v) {
  __shared__ double red[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v = pmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 1e300;
    for (int o = 16; o > 0; o >>= 1) v = pmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

}  // namespace mb
