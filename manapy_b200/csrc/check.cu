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
