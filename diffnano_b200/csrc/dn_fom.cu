// Figure-of-merit reduction: sum over a monitor DFT of |F|^2, in FP64.
//
// The reference has no monitors and no FOM (its tests build losses with
// torch ops on the final field).  The running DFTs that the step kernels
// accumulate are FP64; this kernel reduces them without leaving FP64:
// grid-stride partial sums, warp-shuffle trees inside each block, one
// partial per block in caller-provided scratch, and the last block to finish
// (an atomic ticket, also in the scratch) adds the partials in block order,
// so the result is deterministic.  The ticket is reset by that block for the
// next call.
#include "dn_common.cuh"

namespace dn {
namespace {

constexpr int FOM_THREADS = 256;
constexpr int FOM_MAX_BLOCKS = 1024;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum(double v) {
  __shared__ double s_w[FOM_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) s_w[warp] = v;
  __syncthreads();
  v = threadIdx.x < FOM_THREADS / 32 ? s_w[threadIdx.x] : 0.0;
  if (warp == 0) v = warp_sum(v);
  return v;  // valid in thread 0
}

// scratch layout: [0] ticket (unsigned int, padded to 16 bytes), then one
// double per block
__global__ void __launch_bounds__(FOM_THREADS)
    k_fom_abs2(const double2* __restrict__ f, long long n, double* out, unsigned char* scratch) {
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
  double* partial = reinterpret_cast<double*>(scratch + 16);
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)FOM_THREADS + threadIdx.x; i < n;
       i += (long long)gridDim.x * FOM_THREADS) {
    const double2 z = f[i];
    v = fma(z.x, z.x, fma(z.y, z.y, v));
  }
  v = block_sum(v);
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = v;
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += FOM_THREADS)
    t += reinterpret_cast<volatile double*>(partial)[b];
  t = block_sum(t);
  if (threadIdx.x == 0) {
    *out = t;
    *ticket = 0u;
  }
}

int blocks_for(long long n) {
  long long b = (n + FOM_THREADS - 1) / FOM_THREADS;
  if (b < 1) b = 1;
  if (b > FOM_MAX_BLOCKS) b = FOM_MAX_BLOCKS;
  return (int)b;
}

}  // namespace
}  // namespace dn

extern "C" int64_t dn_fom_abs2_scratch_bytes(int64_t n_complex) {
  return 16 + 8 * (int64_t)dn::blocks_for(n_complex);
}

extern "C" int32_t dn_fom_abs2(const double* dft, int64_t n_complex, double* out, void* scratch,
                               int64_t scratch_bytes, void* stream) {
  if (!out || !scratch || n_complex < 0 || (n_complex > 0 && !dft)) return DN_EINVAL;
  if ((reinterpret_cast<uintptr_t>(dft) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 15))
    return DN_EINVAL;
  if (scratch_bytes < dn_fom_abs2_scratch_bytes(n_complex)) return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the ticket must start at zero; the kernel leaves it at zero afterwards
  DN_CUDA_CHECK(cudaMemsetAsync(scratch, 0, 16, s));
  dn::k_fom_abs2<<<dn::blocks_for(n_complex), dn::FOM_THREADS, 0, s>>>(
      reinterpret_cast<const double2*>(dft), n_complex, out,
      static_cast<unsigned char*>(scratch));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}
