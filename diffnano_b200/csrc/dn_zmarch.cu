// Host helpers of the 3-D z-marching kernels: TMA tensor-map encoding (via
// the driver entry point, no libcuda link) and the work split.
#include <cstdlib>
#include <mutex>

#include "dn_zmarch.cuh"

namespace dn {
namespace zm {

EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

static int encode(CUtensorMap* m, const void* base, int elem_bytes, int rank,
                  const cuuint64_t* dims, const cuuint64_t* strides, const cuuint32_t* box) {
  EncodeTiledFn fn = get_encode();
  if (!fn) return DN_ECUDA;
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(m, elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                           : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                        rank, const_cast<void*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_cuda_error(static_cast<int>(r));
    return DN_ECUDA;
  }
  return DN_OK;
}

int encode_ring(CUtensorMap* m, const void* base, const dn_grid* g, int elem_bytes, int bx,
                int by) {
  const cuuint64_t dims[3] = {(cuuint64_t)g->W, (cuuint64_t)g->H, (cuuint64_t)g->D};
  const cuuint64_t strides[2] = {(cuuint64_t)g->pitch_y * elem_bytes,
                                 (cuuint64_t)g->pitch_z * elem_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  return encode(m, base, elem_bytes, 3, dims, strides, box);
}

int encode_tile4(CUtensorMap* m, const void* base, const dn_grid* g, int elem_bytes, int nslots,
                 long long slot_stride) {
  const cuuint64_t dims[4] = {(cuuint64_t)g->W, (cuuint64_t)g->H, (cuuint64_t)g->D,
                              (cuuint64_t)nslots};
  const cuuint64_t strides[3] = {(cuuint64_t)g->pitch_y * elem_bytes,
                                 (cuuint64_t)g->pitch_z * elem_bytes,
                                 (cuuint64_t)slot_stride * elem_bytes};
  const cuuint32_t box[4] = {TX, TY, 1, 1};
  return encode(m, base, elem_bytes, 4, dims, strides, box);
}

Plan make_plan(const dn_grid* g, long long capacity, long long* nctas, int tx, int ty) {
  Plan plan;
  plan.tx = tx;
  plan.ty = ty;
  plan.ntx = (g->W + tx - 1) / tx;
  const int nty = (g->H + ty - 1) / ty;
  plan.ntiles = plan.ntx * nty;
  // as many z ranges per tile as keep every CTA resident at once, each at
  // least MIN_CHUNK planes long
  long long nsplit = capacity / plan.ntiles;
  if (nsplit > g->D / MIN_CHUNK) nsplit = g->D / MIN_CHUNK;
  if (nsplit < 1) nsplit = 1;
  plan.nsplit = (int)nsplit;
  *nctas = (long long)plan.ntiles * nsplit;
  return plan;
}

#ifndef DN_FWD3D_LANE_COLUMNS
#define DN_FWD3D_LANE_COLUMNS 2
#endif
bool two_column_fp32() {
  static const bool on = [] {
    const char* v = std::getenv("DN_FDTD3D_LANE_COLUMNS");
    if (v && v[0] == '1' && v[1] == '\0') return false;
    if (v && v[0] == '2' && v[1] == '\0') return true;
    return DN_FWD3D_LANE_COLUMNS == 2;
  }();
  return on;
}

bool tma_ok(const dn_grid* g, int elem_bytes, const void* const* ptrs, int n) {
  if ((g->pitch_y * (int64_t)elem_bytes) % 16 || (g->pitch_z * (int64_t)elem_bytes) % 16)
    return false;
  for (int i = 0; i < n; ++i)
    if (!ptrs[i] || (reinterpret_cast<uintptr_t>(ptrs[i]) & 15)) return false;
  return true;
}

}  // namespace zm
}  // namespace dn
