// Non-finite watchdog: one read of a solve's outputs, DN_ENONFINITE on a NaN/Inf.
//
// The reference returns NaN fields and gradients without a word (its TE
// update grows exponentially and overflows FP32 within a few hundred steps,
// diffnano/solvers/fdtd2d.py:269-303).  A NaN or an infinity is sticky under
// the leapfrog update (every stored value is b*f + c*curl of earlier values),
// so a scan of a solve's final state, its monitor DFTs and its gradient
// catches a blow-up anywhere in the run.  The solvers call this once per
// solve or reverse sweep, just before they read their status word; it costs
// one read of those arrays (for the six fields of a 3-D grid, about half the
// traffic of one time step) and nothing inside the time loop.
//
// Layout: one CTA row of blocks per span (blockIdx.y), blocks stride over the
// span's rows, threads over the columns (consecutive threads, consecutive
// elements: coalesced).  A block that saw a bad value records the code once.
#include "dn_common.cuh"

namespace dn {
namespace {

struct SpanDev {
  const void* ptr;
  long long rows, cols, pitch;
  int dtype;
};

struct SpanSet {
  SpanDev s[DN_MAX_SPANS];
};

constexpr int NT_W = 256;

template <typename T>
__device__ __forceinline__ bool scan(const SpanDev& sp) {
  const T* base = static_cast<const T*>(sp.ptr);
  bool bad = false;
  for (long long r = blockIdx.x; r < sp.rows; r += gridDim.x) {
    const T* row = base + r * sp.pitch;
    for (long long c = threadIdx.x; c < sp.cols; c += NT_W) bad |= !isfinite(__ldg(row + c));
  }
  return bad;
}

__global__ void __launch_bounds__(NT_W) k_check_finite(SpanSet set, int* status) {
  const SpanDev& sp = set.s[blockIdx.y];
  const bool bad = sp.dtype == DN_F32 ? scan<float>(sp) : scan<double>(sp);
  if (__syncthreads_or(bad) && threadIdx.x == 0) report_status(status, DN_ENONFINITE);
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_check_finite(const dn_span* spans, int32_t n_spans, int32_t* status,
                                   void* stream) {
  if (!spans || !status || n_spans < 1 || n_spans > DN_MAX_SPANS) return DN_EINVAL;
  dn::SpanSet set{};
  long long max_rows = 1;
  for (int n = 0; n < n_spans; ++n) {
    const dn_span& s = spans[n];
    if (!s.ptr || (s.dtype != DN_F32 && s.dtype != DN_F64) || s.rows < 1 || s.cols < 1 ||
        s.pitch < s.cols)
      return DN_EINVAL;
    set.s[n] = {s.ptr, s.rows, s.cols, s.pitch, s.dtype};
    max_rows = s.rows > max_rows ? s.rows : max_rows;
  }
  // enough blocks per span to keep every SM busy on the largest one
  int dev = 0, nsm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long long want = (long long)nsm * 8;
  const unsigned gx = static_cast<unsigned>(max_rows < want ? max_rows : want);
  dn::k_check_finite<<<dim3(gx, static_cast<unsigned>(n_spans)), dn::NT_W, 0,
                       static_cast<cudaStream_t>(stream)>>>(set, status);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}
