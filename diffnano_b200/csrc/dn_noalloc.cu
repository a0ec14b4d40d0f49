// dn_fdtd2d_run_noalloc: the 2-D step run without any device allocation.
//
// dn_fdtd2d_run ping-pongs between two caller-provided field sets, so a
// caller must own a second set of device buffers.  Some callers cannot
// allocate device memory at the point where they step the solver: a plugin
// embedded in a host application that owns the whole device-memory budget
// (for example through a caching allocator that has already reserved the
// GPU), or a time-critical loop whose policy forbids new allocations.  This
// variant takes one field set (read and updated in place) and uses a
// file-scope device array as the other half of the ping-pong pair.
//
// The array is DN_NOALLOC_MAX_BYTES (6 MiB) on every GPU that loads the
// library and lives until the process exits.  It holds the polarisation's
// three fields of the grid, each padded as the caller's (H x pitch_y
// elements), so H * pitch_y * element size * 3 must fit; larger grids are
// rejected with DN_ENOMEM before any work is queued.
//
// Contract:
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it per
//    device.  Make that first call before any stream capture on the device.
//    The cached address belongs to that device's context: after
//    cudaDeviceReset on the device it is stale, so this entry point must not
//    be used on that device again in the same process.
//  * Every call on a device shares the same array and it keeps the previous
//    call's contents.  Nothing in it has to start at zero: each step writes
//    every in-domain cell of the set it targets before the next step reads
//    it, and padding columns are never read.
//  * Calls whose GPU work overlaps (different streams without ordering, or
//    different host threads) race on the array; serialise them.
//  * When the step count is odd the result is left in the array by the
//    ping-pong and is copied back into the caller's set (device-to-device
//    copies on the same stream), so the result is always in `f`.
//  * No cudaMalloc, cudaFree or allocating library call is made.
#include <mutex>

#include "dn_host.cuh"

extern "C" int32_t dn_fdtd2d_run(const dn_grid* g, void* const fa[6], void* const fb[6],
                                 const void* ce, const dn_cpml* cpml, const dn_source* src,
                                 const dn_monitor* mons, int32_t n_mon, const dn_probe* probe,
                                 const dn_curl_record* rec, int32_t t0, int32_t nsteps,
                                 int32_t* status, void* stream, int32_t* final_in_b);

namespace dn {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[DN_NOALLOC_MAX_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mutex;
void* g_addr[MAX_DEVICES] = {};

// device address of the scratch array for the current device (looked up once
// per device, with that device current); nullptr on failure
int scratch_address(void** out) {
  int dev = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) return DN_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
      set_last_cuda_error(static_cast<int>(e));
      return DN_ECUDA;
    }
    g_addr[dev] = ptr;
  }
  *out = g_addr[dev];
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd2d_run_noalloc(const dn_grid* g, void* const f[6], const void* ce,
                                         const dn_cpml* cpml, const dn_source* src,
                                         const dn_monitor* mons, int32_t n_mon,
                                         const dn_probe* probe, int32_t t0, int32_t nsteps,
                                         int32_t* status, void* stream) {
  if (!g || !f) return DN_EINVAL;
  if (g->dtype != DN_F32 && g->dtype != DN_F64) return DN_EINVAL;
  if (g->D != 1 || g->H < 1 || g->pitch_y < g->W || (g->pol != DN_TM && g->pol != DN_TE))
    return DN_EINVAL;
  const size_t es = g->dtype == DN_F32 ? 4 : 8;
  // bound the pitch before multiplying, so that H * pitch_y * es cannot wrap
  if ((uint64_t)g->pitch_y > (uint64_t)DN_NOALLOC_MAX_BYTES / (3 * es * (size_t)g->H))
    return DN_ENOMEM;
  // one field of the scratch set, rounded up to keep 256-byte alignment
  const size_t field_bytes = ((size_t)g->H * (size_t)g->pitch_y * es + 255) / 256 * 256;
  if (3 * field_bytes > (size_t)DN_NOALLOC_MAX_BYTES) return DN_ENOMEM;

  void* base = nullptr;
  int rc = dn::scratch_address(&base);
  if (rc != DN_OK) return rc;
  const int comps[3] = {g->pol == DN_TM ? DN_EZ : DN_HZ, g->pol == DN_TM ? DN_HX : DN_EX,
                        g->pol == DN_TM ? DN_HY : DN_EY};
  void* fb[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  for (int n = 0; n < 3; ++n) {
    if (!f[comps[n]]) return DN_EINVAL;
    fb[comps[n]] = static_cast<unsigned char*>(base) + n * field_bytes;
  }
  int32_t in_b = 0;
  rc = dn_fdtd2d_run(g, f, fb, ce, cpml, src, mons, n_mon, probe, nullptr, t0, nsteps, status,
                     stream, &in_b);
  if (rc != DN_OK) return rc;
  if (in_b) {  // odd step count: bring the result back into the caller's set
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t pitch = (size_t)g->pitch_y * es;
    for (int n = 0; n < 3; ++n)
      DN_CUDA_CHECK(cudaMemcpy2DAsync(f[comps[n]], pitch, fb[comps[n]], pitch, (size_t)g->W * es,
                                      (size_t)g->H, cudaMemcpyDeviceToDevice, s));
  }
  return DN_OK;
}
