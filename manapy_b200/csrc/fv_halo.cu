// Halo exchange of a sharded mesh: packing of the owned values peers hold as halo,
// and unpacking of the received values into the halo cells.
//
// manapy exchanges its halo with MPI neighbourhood all-to-alls of per-rank send
// lists (manapy/comms/communication.py:93-145, called from manapy/ast/core.py:415-478).
// Here every peer's send list is concatenated into one index list, so one launch
// packs every field for every peer into one contiguous buffer [entry][field] (each
// peer's entries form one contiguous slice, the message of its point-to-point send),
// and one launch scatters the received buffer back.  Entries are independent (each
// index appears once per list), so the kernels are plain gathers with coalesced stores
// and scatters with coalesced loads.
#include "fv_common.cuh"

namespace mb {
namespace {

struct HaloFields {
  double *f[MB_HALO_MAX_FIELDS];
  int32_t count;
};

__global__ void __launch_bounds__(kBlock) k_halo_pack(HaloFields fs, const int64_t *__restrict__ idx, int64_t n,
                                                      double *__restrict__ buf) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = ld(idx + k);
    for (int j = 0; j < fs.count; ++j) buf[k * fs.count + j] = ld(fs.f[j] + c);
  }
}

__global__ void __launch_bounds__(kBlock) k_halo_unpack(HaloFields fs, const int64_t *__restrict__ idx, int64_t n,
                                                        const double *__restrict__ buf) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = ld(idx + k);
    for (int j = 0; j < fs.count; ++j) fs.f[j][c] = ld(buf + k * fs.count + j);
  }
}

int halo_fields(double *const *fields, int32_t nfields, HaloFields &fs) {
  if (!fields || nfields <= 0 || nfields > MB_HALO_MAX_FIELDS) return MB_EINVAL;
  fs.count = nfields;
  for (int j = 0; j < nfields; ++j) {
    if (!fields[j]) return MB_EINVAL;
    fs.f[j] = fields[j];
  }
  return MB_OK;
}

int grid_of(int64_t n) {
  const int64_t g = (n + kBlock - 1) / kBlock;
  return (int)(g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : g));
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_halo_pack(double *const *fields, int32_t nfields, const int64_t *idx, int64_t n, double *buf,
                            void *stream) {
  MB_NVTX();
  HaloFields fs{};
  const int rc = halo_fields(fields, nfields, fs);
  if (rc != MB_OK || n < 0 || (n > 0 && (!idx || !buf))) return rc != MB_OK ? rc : MB_EINVAL;
  if (n == 0) return MB_OK;
  k_halo_pack<<<grid_of(n), kBlock, 0, (cudaStream_t)stream>>>(fs, idx, n, buf);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}

extern "C" int mb_halo_unpack(double *const *fields, int32_t nfields, const int64_t *idx, int64_t n,
                              const double *buf, void *stream) {
  MB_NVTX();
  HaloFields fs{};
  const int rc = halo_fields(fields, nfields, fs);
  if (rc != MB_OK || n < 0 || (n > 0 && (!idx || !buf))) return rc != MB_OK ? rc : MB_EINVAL;
  if (n == 0) return MB_OK;
  k_halo_unpack<<<grid_of(n), kBlock, 0, (cudaStream_t)stream>>>(fs, idx, n, buf);
  return cudaGetLastError() == cudaSuccess ? MB_OK : MB_ECUDA;
}
