// Shared device/host helpers for the dn_fdtd kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dn_fdtd.h"

namespace dn {

// ---------------------------------------------------------------------------
// host-side error bookkeeping
// ---------------------------------------------------------------------------
void set_last_cuda_error(int e);
int last_cuda_error();

#define DN_CUDA_CHECK(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) {                                  \
      ::dn::set_last_cuda_error(static_cast<int>(_e));        \
      return DN_ECUDA;                                        \
    }                                                         \
  } while (0)

// ---------------------------------------------------------------------------
// kernel-side views of the ABI structs (passed by value as kernel params)
// ---------------------------------------------------------------------------
struct BoxDev {
  int lo[3];
  int hi[3];
  __host__ __device__ bool contains(int i, int j, int k) const {
    return i >= lo[0] && i < hi[0] && j >= lo[1] && j < hi[1] && k >= lo[2] && k < hi[2];
  }
  __host__ __device__ long long ny() const { return hi[1] - lo[1]; }
  __host__ __device__ long long nx() const { return hi[2] - lo[2]; }
  __host__ __device__ long long cells() const {
    return (long long)(hi[0] - lo[0]) * ny() * nx();
  }
  // row-major (z, y, x) offset of (i, j, k) inside the box
  __host__ __device__ long long offset(int i, int j, int k) const {
    return ((long long)(i - lo[0]) * ny() + (j - lo[1])) * nx() + (k - lo[2]);
  }
  // does the box intersect plane i?
  __host__ __device__ bool has_plane(int i) const { return i >= lo[0] && i < hi[0]; }
};

struct MonDev {
  int comp;
  int nf;
  long long ncell;
  BoxDev box;
  const double* phase;
  double* acc;
};

template <typename T>
struct SrcDev {
  int comp;  // DN_NONE disables
  BoxDev box;
  const T* wave;
};

template <typename T>
struct ProbeDev {
  int comp;  // DN_NONE disables
  int pos[3];
  T* out;
};

template <typename T>
struct StepParams {
  int D, H, W;
  long long py, pz;
  const T* in[6];
  T* out[6];
  const T* ce;
  const double* b[3];
  const double* c[3];
  T dt;
  T inv_dl;
  SrcDev<T> src;
  int n_mon;
  MonDev mon[DN_MAX_MONITORS];
  ProbeDev<T> probe;
  int t;  // absolute step index of this launch
  int* status;
};

// Does plane i hold a source, monitor or probe cell?  (Unrolled over the
// fixed monitor capacity so the parameter array is never indexed at run time,
// which would move it to local memory.)
template <typename T>
__device__ __forceinline__ bool any_special(const StepParams<T>& p, int i) {
  bool any = p.src.comp >= 0 && p.src.box.has_plane(i);
  any |= p.probe.comp >= 0 && p.probe.pos[0] == i;
#pragma unroll
  for (int m = 0; m < DN_MAX_MONITORS; ++m) any |= m < p.n_mon && p.mon[m].box.has_plane(i);
  return any;
}

// ---------------------------------------------------------------------------
// mbarrier / TMA PTX wrappers (sm_90+; used here on sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// One bounded probe of the barrier's phase; returns true when phase `parity`
// has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// One probe that may suspend the thread for up to `hint_ns` nanoseconds
// (woken early when the phase completes); returns true when phase `parity`
// has completed.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity,
                                                    uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `max_probes` probes (each probe may suspend
// the thread for a hardware-chosen time) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint32_t max_probes) {
  for (uint32_t n = 0; n < max_probes; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 3-D tiled TMA load global -> shared, completion counted on `bar`.
// Coordinates are element indices (x innermost); x * sizeof(T) must be a
// multiple of 16 bytes.  No multicast.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int x,
                                            int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// hint: bring the cache line holding `a` into L2 (no register is written)
__device__ __forceinline__ void prefetch_l2(const void* a) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

// record the first error code into a device status word
__device__ __forceinline__ void report_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

}  // namespace dn
