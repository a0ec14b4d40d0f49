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

// Load paths: LD_NC for arrays no thread writes during the launch
// (non-coherent read-only path), LD_CG for arrays other CTAs of the same
// launch write (L2 only, never a stale L1 line), LD_PLAIN otherwise.
enum { LD_NC = 0, LD_CG = 1, LD_PLAIN = 2 };

template <int LDP, typename P>
__device__ __forceinline__ P load_as(const P* s) {
  if constexpr (LDP == LD_NC)
    return __ldg(s);
  else if constexpr (LDP == LD_CG)
    return __ldcg(s);
  else
    return *s;
}

template <typename T, int LDP = LD_NC>
__device__ __forceinline__ T ld(const T* a, long long o, bool ok) {
  return ok ? load_as<LDP>(a + o) : T(0);
}

// Columns jv .. jv+VEC-1 at offset o; columns at or past W (and all of them
// when !ok) read as 0.
template <typename T, int VEC, int LDP = LD_NC>
__device__ __forceinline__ Vec<T, VEC> ldv(const T* a, long long o, bool ok, bool full, int jv,
                                           int W) {
  Vec<T, VEC> r;
  constexpr int PER = 16 / static_cast<int>(sizeof(T));  // elements per 16 bytes
  if constexpr (VEC >= PER && VEC % PER == 0) {
    if (ok && full) {
#pragma unroll
      for (int c = 0; c < VEC / PER; ++c) {
        if constexpr (std::is_same<T, float>::value) {
          const float4 x = load_as<LDP>(reinterpret_cast<const float4*>(a + o) + c);
          r[4 * c + 0] = x.x, r[4 * c + 1] = x.y, r[4 * c + 2] = x.z, r[4 * c + 3] = x.w;
        } else {
          const double2 x = load_as<LDP>(reinterpret_cast<const double2*>(a + o) + c);
          r[2 * c + 0] = x.x, r[2 * c + 1] = x.y;
        }
      }
      return r;
    }
  }
#pragma unroll
  for (int q = 0; q < VEC; ++q) r[q] = ld<T, LDP>(a, o + q, ok && jv + q < W);
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
