// Row access for the 2-D warp strip-march kernels (forward step and its
// adjoint): a lane owns VEC adjacent columns of a row; whole 16-byte chunks
// are moved with one vector load or store when all VEC columns are in the
// grid and the row offset is 16-byte aligned (the host checks the pitch and
// the array addresses before it selects VEC > 1).
#pragma once

#include <stdint.h>

#include <type_traits>

namespace dn {

constexpr unsigned STRIP_FULL_MASK = 0xffffffffu;

// VEC adjacent values of one row, from column jv
template <typename T, int VEC>
struct Vec {
  T v[VEC];
  __device__ __forceinline__ T& operator[](int q) { return v[q]; }
  __device__ __forceinline__ const T& operator[](int q) const { return v[q]; }
};

template <typename T>
__device__ __forceinline__ T ld(const T* a, long long o, bool ok) {
  return ok ? __ldg(a + o) : T(0);
}

// Columns jv .. jv+VEC-1 at offset o; columns at or past W (and all of them
// when !ok) read as 0.  NC: the array is not written during the launch
// (read through the non-coherent path); otherwise plain loads.
template <typename T, int VEC, bool NC = true>
__device__ __forceinline__ Vec<T, VEC> ldv(const T* a, long long o, bool ok, bool full, int jv,
                                           int W) {
  Vec<T, VEC> r;
  constexpr int PER = 16 / static_cast<int>(sizeof(T));  // elements per 16 bytes
  if constexpr (VEC >= PER && VEC % PER == 0) {
    if (ok && full) {
#pragma unroll
      for (int c = 0; c < VEC / PER; ++c) {
        if constexpr (std::is_same<T, float>::value) {
          const float4* s = reinterpret_cast<const float4*>(a + o) + c;
          const float4 x = NC ? __ldg(s) : *s;
          r[4 * c + 0] = x.x, r[4 * c + 1] = x.y, r[4 * c + 2] = x.z, r[4 * c + 3] = x.w;
        } else {
          const double2* s = reinterpret_cast<const double2*>(a + o) + c;
          const double2 x = NC ? __ldg(s) : *s;
          r[2 * c + 0] = x.x, r[2 * c + 1] = x.y;
        }
      }
      return r;
    }
  }
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    const bool in = ok && jv + q < W;
    r[q] = in ? (NC ? __ldg(a + o + q) : a[o + q]) : T(0);
  }
  return r;
}

// Store the columns of v that are in the grid (whole 16-byte chunks when all are).
template <typename T, int VEC>
__device__ __forceinline__ void stv(T* a, long long o, const Vec<T, VEC>& v, bool full, int jv,
                                    int W) {
  constexpr int PER = 16 / static_cast<int>(sizeof(T));
  if constexpr (VEC >= PER && VEC % PER == 0) {
    if (full) {
#pragma unroll
      for (int c = 0; c < VEC / PER; ++c) {
        if constexpr (std::is_same<T, float>::value)
          reinterpret_cast<float4*>(a + o)[c] =
              make_float4(v[4 * c + 0], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        else
          reinterpret_cast<double2*>(a + o)[c] = make_double2(v[2 * c + 0], v[2 * c + 1]);
      }
      return;
    }
  }
#pragma unroll
  for (int q = 0; q < VEC; ++q)
    if (jv + q < W) a[o + q] = v[q];
}

inline bool aligned16(const void* a) { return (reinterpret_cast<uintptr_t>(a) & 15) == 0; }

}  // namespace dn
