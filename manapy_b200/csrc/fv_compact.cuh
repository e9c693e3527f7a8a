// Helpers of the compact cell-centred step kernels (FP64 and FP32-compensated).
//
// Compact layout: per cell its vertices (manapy's local order), the neighbour
// across each local face (or -1-f for boundary face f) and orientation bits per
// face; face geometry is recomputed from the vertex coordinates.
#pragma once

#include "fv_common.cuh"

namespace mb {

__device__ __forceinline__ int4 ld4(const int32_t *p) { return __ldg(reinterpret_cast<const int4 *>(p)); }
__device__ __forceinline__ double2 ldd2(const double *p) { return __ldg(reinterpret_cast<const double2 *>(p)); }
__device__ __forceinline__ int comp(const int4 v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }
template <class T>
__device__ __forceinline__ T pick3(T a, T b, T c, int k) { return k == 0 ? a : (k == 1 ? b : c); }

// L2 eviction-priority hints (per instruction; no device state is changed).
// Phase 1 writes its outputs with evict_last so they are still in L2 when
// phase 2 reads them; tables read once per step are loaded with evict_first.
#ifndef MB_L2_HINTS
#define MB_L2_HINTS 1
#endif
// streamed loads: optionally without an L1 allocation (the gathers own L1), and as
// non-volatile asm so the compiler may schedule them freely (they read read-only data)
#ifndef MB_STREAM_L1NA
#define MB_STREAM_L1NA 0
#endif
#ifndef MB_STREAM_VOLATILE
#define MB_STREAM_VOLATILE 1
#endif
#if MB_STREAM_L1NA
#define MB_LDNC "ld.global.nc.L1::no_allocate.L2::cache_hint"
#else
#define MB_LDNC "ld.global.nc.L2::cache_hint"
#endif
#if MB_STREAM_VOLATILE
#define MB_ASM_LD asm volatile
#else
#define MB_ASM_LD asm
#endif
__device__ __forceinline__ uint64_t l2_keep() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_stream() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st2_keep(double *a, double x, double y, uint64_t pol) {
#if MB_L2_HINTS
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(x), "d"(y), "l"(pol) : "memory");
#else
  *reinterpret_cast<double2 *>(a) = make_double2(x, y);
#endif
}
__device__ __forceinline__ void st1_keep(double *a, double x, uint64_t pol) {
#if MB_L2_HINTS
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(x), "l"(pol) : "memory");
#else
  *a = x;
#endif
}
__device__ __forceinline__ int ld1_stream(const int32_t *a, uint64_t pol) {
#if MB_L2_HINTS
  int v;
  MB_ASM_LD(MB_LDNC ".s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
#else
  return __ldg(a);
#endif
}
__device__ __forceinline__ double2 ldd2_stream(const double *a, uint64_t pol) {
#if MB_L2_HINTS
  double2 v;
  MB_ASM_LD(MB_LDNC ".v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
#else
  return __ldg(reinterpret_cast<const double2 *>(a));
#endif
}
__device__ __forceinline__ double ldd_stream(const double *a, uint64_t pol) {
#if MB_L2_HINTS
  double v;
  MB_ASM_LD(MB_LDNC ".f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
#else
  return __ldg(a);
#endif
}

// flags of the compact 2D layout
__device__ __forceinline__ bool f2_own(uint32_t fl, int j) { return (fl >> j) & 1u; }
__device__ __forceinline__ bool f2_rev(uint32_t fl, int j) { return (fl >> (3 + j)) & 1u; }
__device__ __forceinline__ bool f2_flip(uint32_t fl, int j) { return (fl >> (6 + j)) & 1u; }

// ---------------------------------------------------------------- tetrahedra

// Local faces of a tetrahedron, (v0,v1,v2), (v2,v3,v0), (v0,v1,v3), (v3,v1,v2)
// (manapy/ddm/ddm_utils3d.py:785-791), and the six permutations of three items
// (0,1,2), (0,2,1), (1,0,2), (1,2,0), (2,0,1), (2,1,0): two bits per entry,
// entry e at bits 2e, row-major.
constexpr uint32_t kTetFacePacked = 0x9f43a4u;
constexpr uint64_t kPerm3Packed = 0x192261624ull;
__device__ __forceinline__ int tet_face(int j, int k) { return (kTetFacePacked >> (2 * (3 * j + k))) & 3; }
__device__ __forceinline__ int perm3(int code, int k) { return (int)((kPerm3Packed >> (2 * (3 * code + k))) & 3); }

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return d3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// 32-byte rows ([n][4] doubles, 32-byte aligned) in one 256-bit load (sm_100), or as two
// 16-byte loads
#ifndef MB_LD256
#define MB_LD256 1
#endif
__device__ __forceinline__ void ld4d(const double *p, double &a, double &b, double &c, double &d) {
#if MB_LD256
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
#else
  const double2 u = __ldg(reinterpret_cast<const double2 *>(p)), v = __ldg(reinterpret_cast<const double2 *>(p + 2));
  a = u.x; b = u.y; c = v.x; d = v.y;
#endif
}
// one 256-bit access per 32-byte record where a kernel writes or streams whole rows
#ifndef MB_V4_IO
#define MB_V4_IO 1
#endif
__device__ __forceinline__ void st4_keep(double *a, double x, double y, double z, double w, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f64 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a), "d"(x), "d"(y), "d"(z), "d"(w),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st4d_plain(double *a, double x, double y, double z, double w) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(a), "d"(x), "d"(y), "d"(z), "d"(w) : "memory");
}
__device__ __forceinline__ void ld4d_stream(const double *p, double &a, double &b, double &c, double &d,
                                            uint64_t pol) {
  MB_ASM_LD(MB_LDNC ".v4.f64 {%0, %1, %2, %3}, [%4], %5;" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p), "l"(pol));
}
__device__ __forceinline__ D3 ld3(const double *p) {  // [n][4] rows
  double a, b, c, d;
  ld4d(p, a, b, c, d);
  return d3(a, b, c);
}
__device__ __forceinline__ D3 pick4(const D3 *P, int k) { return k == 0 ? P[0] : (k == 1 ? P[1] : (k == 2 ? P[2] : P[3])); }
template <class T>
__device__ __forceinline__ T pick4v(T a, T b, T c, T d, int k) { return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d)); }

// (V_d0 + V_d1) + V_d2 for local face j, d = face_desc's descending order: the pair added
// first is the face's two vertices other than d2 (an addition of two commutes exactly), so
// the sum is one of three candidates chosen by d2, with no 4-way selects of coordinates
// (j a compile-time constant after unrolling)
__device__ __forceinline__ D3 tet_face_sum(const D3 *P, int j, int d2) {
  const int a = tet_face(j, 0), b = tet_face(j, 1), c = tet_face(j, 2);
  const D3 x = P[a], y = P[b], z = P[c];
  if (d2 == a) return (y + z) + x;
  if (d2 == b) return (x + z) + y;
  return (x + y) + z;
}

// manapy's descending-order vertices of local face j: (d0, d1, d2), as local vertex indices
__device__ __forceinline__ void face_desc(uint32_t fl, int j, int &d0, int &d1, int &d2) {
  const int code = (fl >> (6 * j + 1)) & 7u;
  d0 = tet_face(j, perm3(code, 0));
  d1 = tet_face(j, perm3(code, 1));
  d2 = tet_face(j, perm3(code, 2));
}

}  // namespace mb
