// Shared machinery of the 3-D z-marching kernels (forward step and adjoint
// step): tile geometry, the TMA tensor maps, the work split, the staged
// shared-memory ring with its producer warp, and bounded mbarrier waits.
//
// A CTA owns a TY (y) x TX (x) tile over a range of z planes (Geo: 16 x 32
// with one column per lane, 16 x 64 with two).  Per plane it stages NRING
// arrays as (TX+8) x (TY+2) boxes (x from k0-4, y from j0-1: the tile plus a
// one-cell ring, x start 16-byte aligned for TMA) and NTILE arrays as TX x TY
// tile boxes, through a ring of S stages drained by eight consumer warps (two
// rows each) and filled either by a producer warp (producer_run) or, in
// eight-warp CTAs, by the consumer warp that releases a stage last
// (issue_job).
#pragma once

#include <cuda.h>

#include "dn_host.cuh"

namespace dn {
namespace zm {

// Tile geometry: TX_ columns (one warp: 32 lanes x TX_/32 columns) by TY_
// rows (TY_/2 consumer warps, two rows each, plus one producer warp); ring
// boxes are BX x BY = (TX_+8) x (TY_+2): x from k0-4 (16-byte aligned) to
// k0+TX_+3, y from j0-1 to j0+TY_.
template <int TX_, int TY_>
struct Geo {
  static constexpr int TX = TX_;
  static constexpr int TY = TY_;
  static constexpr int NCW = TY_ / 2;
  static constexpr int NT = (NCW + 1) * 32;
  static constexpr int BX = TX_ + 8;
  static constexpr int BY = TY_ + 2;
};
using Geo32 = Geo<32, 16>;  // one column per lane (FP64 forward, the adjoint)
using Geo64 = Geo<64, 16>;  // two columns per lane (FP32 forward)

constexpr int TX = Geo32::TX;        // tile x (one warp)
constexpr int TY = Geo32::TY;        // tile y
constexpr int NCW = Geo32::NCW;      // consumer warps, two rows each
constexpr int NT = Geo32::NT;        // + one producer warp
constexpr int BX = Geo32::BX;        // ring box x: k0-4 .. k0+TX+3
constexpr int BY = Geo32::BY;        // ring box y: j0-1 .. j0+TY
constexpr int MIN_CHUNK = 8;         // min planes per CTA range
constexpr uint32_t WAIT_PROBES = 1u << 16;  // bound on mbarrier probes per wait
constexpr uint32_t SLEEP_NS = 20000;        // suspend-time hint per probe (~1.3 s bound)
constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int MAX_MAPS = 10;

// Shared-memory layout of one kernel configuration.
template <typename T, int NRING, int NTILE, int S_, typename G_ = Geo32>
struct Layout {
  using G = G_;
  static constexpr int S = S_;
  static constexpr int RING_BYTES = G::BX * G::BY * (int)sizeof(T);
  static constexpr int TILE_BYTES = G::TX * G::TY * (int)sizeof(T);
  static constexpr int RING_ARR = (RING_BYTES + 127) / 128 * 128;
  static constexpr int TILE_ARR = (TILE_BYTES + 127) / 128 * 128;
  static constexpr int STAGE_BYTES = NRING * RING_ARR + NTILE * TILE_ARR;
  static constexpr int TX_BYTES = NRING * RING_BYTES + NTILE * TILE_BYTES;
  static constexpr int TAB_ELEMS = 2 * (G::TY + 2) + 2 * (G::TX + 2);
  static constexpr int TAB_BYTES = TAB_ELEMS * (int)sizeof(T);
  static constexpr int BAR_OFF = ((S * STAGE_BYTES + TAB_BYTES + 15) / 16) * 16;
  // bytes of dynamic shared memory (stages, profile tables, barriers, flags,
  // and 128 bytes of slack for aligning the carve)
  static constexpr size_t BYTES =
      (size_t)BAR_OFF + 2 * S * sizeof(uint64_t) + (4 + S) * sizeof(int) + 128;
};

struct alignas(64) TmapSet {
  CUtensorMap m[MAX_MAPS];
};

// Work split: CTA b owns tile (b % ntiles) for z in [split*D/nsplit,
// (split+1)*D/nsplit), split = b / ntiles.  Consecutive CTAs are neighbouring
// tiles over the same z range, so CTAs that run together march through z in
// lockstep and the halo rows/columns one CTA fetches are L2 hits for its
// neighbours.
struct Plan {
  int ntx;     // tiles along x
  int ntiles;  // tiles per plane
  int nsplit;  // z ranges per tile
  int tx, ty;  // tile size (columns, rows)
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait on an mbarrier phase that also gives up when another warp has
// flagged an abort
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t n = 0; n < WAIT_PROBES; ++n) {
    if (mbar_try_wait_sleep(bar, parity, SLEEP_NS)) return true;
    if ((n & 15u) == 15u && *abort) return false;
  }
  return false;
}

// 4-D tiled TMA load (x, y, z, w); same alignment rule as the 3-D one.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, uint64_t* bar, int x,
                                            int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// Pointers into the carved dynamic shared memory of one CTA.
template <typename T, typename L>
struct Smem {
  unsigned char* stages;
  T* sbJ;  // b_y of rows j0-1 .. j0+TY
  T* sgJ;  // 1 + c_y of the same rows
  T* sbK;  // b_x of columns k0-1 .. k0+TX (the geometry's TX)
  T* sgK;  // 1 + c_x of the same columns
  uint64_t* full;
  uint64_t* empty;
  int* flags;         // [0] job count, [1] abort flag, [2] jobs issued
  unsigned* release;  // per stage: warp releases so far (refill by the last one)

  __device__ explicit Smem(unsigned char* raw) {
    // TMA destinations must be 128-byte aligned: align the carve explicitly
    unsigned char* s = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(raw) + 127) & ~static_cast<uintptr_t>(127));
    stages = s;
    sbJ = reinterpret_cast<T*>(s + L::S * L::STAGE_BYTES);
    sgJ = sbJ + (L::G::TY + 2);
    sbK = sgJ + (L::G::TY + 2);
    sgK = sbK + (L::G::TX + 2);
    full = reinterpret_cast<uint64_t*>(s + L::BAR_OFF);
    empty = full + L::S;
    flags = reinterpret_cast<int*>(empty + L::S);
    release = reinterpret_cast<unsigned*>(flags + 4);
  }
  // ring array a of job q's stage
  __device__ const T* arr(int q, int a) const {
    return reinterpret_cast<const T*>(stages + (q % L::S) * L::STAGE_BYTES + a * L::RING_ARR);
  }
  // tile array t (after the nring ring arrays) of job q's stage
  __device__ const T* tile_arr(int q, int nring, int t) const {
    return reinterpret_cast<const T*>(stages + (q % L::S) * L::STAGE_BYTES +
                                      nring * L::RING_ARR + t * L::TILE_ARR);
  }
};

// Per-CTA geometry derived from the plan.  The CTA stages the planes
// zs .. zs + njobs - 1 in this order: the warm-up plane z0-1 (when z0 > 0),
// z0 .. z1-1, and plane z1 (when z1 < D), read only as the "next" plane.
struct Range {
  int tile, z0, z1, k0, j0, zs, njobs;
  __device__ Range(const Plan& plan, int D) {
    tile = blockIdx.x % plan.ntiles;
    const int split = blockIdx.x / plan.ntiles;
    z0 = (int)((long long)split * D / plan.nsplit);
    z1 = (int)((long long)(split + 1) * D / plan.nsplit);
    k0 = (tile % plan.ntx) * plan.tx;
    j0 = (tile / plan.ntx) * plan.ty;
    zs = z0 > 0 ? z0 - 1 : z0;
    njobs = (z1 - zs) + (z1 < D ? 1 : 0);
  }
};

// Thread 0 initialises the barriers and the job count; all threads fill the
// CPML profile tables of the tile.  Ends with the kernel's only CTA-wide
// barrier.  Returns the job count (0 when a previous launch recorded an
// error, which turns this launch into a no-op).
template <typename T, typename L>
__device__ int pipe_setup(const Smem<T, L>& sm, const Range& R, int D, int H, int W,
                          const double* const b[3], const double* const c[3],
                          const int* status) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    const bool skip = status != nullptr && *reinterpret_cast<const volatile int*>(status) != 0;
    sm.flags[0] = skip ? 0 : R.njobs;
    sm.flags[1] = 0;
    sm.flags[2] = 0;
    for (int s = 0; s < L::S; ++s) sm.release[s] = 0;
    for (int s = 0; s < L::S; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], L::G::NCW);
    }
    fence_barrier_init();
  }
  for (int e = tid; e < L::G::TY + 2; e += blockDim.x) {
    const int j = R.j0 - 1 + e;
    const bool ok = j >= 0 && j < H;
    sm.sbJ[e] = ok ? static_cast<T>(b[1][j]) : T(1);
    sm.sgJ[e] = ok ? static_cast<T>(1.0 + c[1][j]) : T(1);
  }
  for (int e = tid; e < L::G::TX + 2; e += blockDim.x) {
    const int kx = R.k0 - 1 + e;
    const bool ok = kx >= 0 && kx < W;
    sm.sbK[e] = ok ? static_cast<T>(b[2][kx]) : T(1);
    sm.sgK[e] = ok ? static_cast<T>(1.0 + c[2][kx]) : T(1);
  }
  __syncthreads();
  return sm.flags[0];
}

// Issue job q's loads into stage q % S: NRING ring boxes and NTILE tile boxes
// (4-D tile maps, slot coordinate `tile_slot(z)`), completion counted on the
// stage's "full" barrier.  The stage must have been released by every
// consumer warp.
template <typename T, typename L, int NRING, int NTILE, typename SlotFn>
__device__ __forceinline__ void issue_job(const Smem<T, L>& sm, const TmapSet& tm,
                                          const Range& R, int q, SlotFn tile_slot) {
  const int z = R.zs + q;
  uint64_t* bar = &sm.full[q % L::S];
  unsigned char* dst = sm.stages + (q % L::S) * L::STAGE_BYTES;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(bar, L::TX_BYTES);
#pragma unroll
  for (int a = 0; a < NRING; ++a)
    tma_load_3d(dst + a * L::RING_ARR, &tm.m[a], bar, R.k0 - 4, R.j0 - 1, z);
#pragma unroll
  for (int a = 0; a < NTILE; ++a)
    tma_load_4d(dst + NRING * L::RING_ARR + a * L::TILE_ARR, &tm.m[NRING + a], bar, R.k0, R.j0,
                z, tile_slot(z));
}

// Wait (bounded) until the copies of the last S issued jobs have landed, so
// that none is in flight when the CTA gives its shared memory back (error
// paths; jobs before those were consumed before their stage was reused).
template <typename T, typename L>
__device__ __forceinline__ void drain_jobs(const Smem<T, L>& sm, int issued) {
  for (int q = max(0, issued - L::S); q < issued; ++q)
    (void)mbar_wait_bounded(&sm.full[q % L::S], (q / L::S) & 1, WAIT_PROBES);
}

// Producer (lane 0 of the last warp): stream job q's NRING ring boxes and
// NTILE tile boxes into stage q % S once the consumers released the stage's
// previous job; tile maps are 4-D (x, y, z, slot) with the slot coordinate
// `tile_slot(z)`.  Stays until the consumers released the last stages so no
// copy is still in flight when the shared memory is given back.
template <typename T, typename L, int NRING, int NTILE, typename SlotFn>
__device__ void producer_run(const Smem<T, L>& sm, const TmapSet& tm, const Range& R, int nj,
                             int* status, SlotFn tile_slot) {
  volatile int* abort = sm.flags + 1;
  bool ok = true;
  int issued = 0;
  for (int q = 0; q < nj && ok; ++q) {
    if (q >= L::S) ok = wait_phase(&sm.empty[q % L::S], ((q / L::S) - 1) & 1, abort);
    if (!ok) break;
    issue_job<T, L, NRING, NTILE>(sm, tm, R, q, tile_slot);
    issued = q + 1;
  }
  for (int q = max(0, nj - L::S); q < nj && ok; ++q)
    ok = wait_phase(&sm.empty[q % L::S], (q / L::S) & 1, abort);
  if (!ok) {
    report_status(status, DN_ETIMEOUT);
    *abort = 1;
    drain_jobs(sm, issued);
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode();

// ring (bx x by x 1; default 40 x 18) map over a (D, H, W) field with the
// grid's pitches
int encode_ring(CUtensorMap* m, const void* base, const dn_grid* g, int elem_bytes, int bx = BX,
                int by = BY);
// tile (32 x 16 x 1 x 1) map over `nslots` fields of the grid's shape,
// `slot_stride` elements apart
int encode_tile4(CUtensorMap* m, const void* base, const dn_grid* g, int elem_bytes, int nslots,
                 long long slot_stride);
// work split for `capacity` resident CTAs over tx x ty tiles
Plan make_plan(const dn_grid* g, long long capacity, long long* nctas, int tx = TX, int ty = TY);
// Does the FP32 forward step (and the adjoint's replay) run the two-column
// kernel?  DN_FWD3D_LANE_COLUMNS at build time (default 2), or the
// environment variable DN_FDTD3D_LANE_COLUMNS = "1" or "2" (read once per
// process), e.g. to compare the one- and two-column kernels.
bool two_column_fp32();
// TMA constraints: 16-byte aligned bases and byte strides
bool tma_ok(const dn_grid* g, int elem_bytes, const void* const* ptrs, int n);

}  // namespace zm
}  // namespace dn
