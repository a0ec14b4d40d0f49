// BF16 tensor-core GEMM for sm_100a: tcgen05.mma with FP32 accumulators in
// tensor memory (TMEM), operands staged by TMA, fused epilogue.
//
//   C[z] (M x N) = sum_s A_s[z] (M x K_s) * B_s[z] (N x K_s)^T, then
//   scale / bias / addend / GELU or GELU-gradient, stored through a
//   two-digit index map (so one GEMM can write a transposed or re-blocked
//   layout that the next GEMM reads directly).
//
// Persistent CTAs (one per SM, 320 threads) walk the tile list: per batch,
// groups of 16 m tiles, n tiles inside a group, m fastest (neighbouring CTAs
// share A rows and B columns in L2):
//   warp 0, lane 0  TMA producer.  Per 64-wide k block it loads the 128 x 64
//                   A tile and the BN x 64 B tile into one ring stage
//                   (128-byte swizzle; a K-major operand is one box, an
//                   MN-major operand one 64 x 64 box per 64 rows);
//   warp 1, lane 0  MMA issuer.  Four tcgen05.mma.cta_group::1.kind::f16
//                   (M = 128, N = BN, K = 16) per stage from shared-memory
//                   descriptors; tcgen05.commit frees the stage, and after the
//                   last k block signals the accumulator buffer (two TMEM
//                   buffers of BN columns, so the epilogue of one tile runs
//                   under the MMAs of the next);
//   warps 2..9      epilogue.  Warp w reads TMEM lanes 32*(w%4) .. +31 (its
//                   rows) of one half of the tile's columns ((w-2)/4) with
//                   tcgen05.ld.32x32b.x32, applies the epilogue and stores 32
//                   consecutive columns per thread.  Two warps per lane
//                   quadrant: the operator's transform GEMMs (K ~ 1 000, a
//                   GELU per element) are bound by epilogue instructions.
// Pair mode (two-CTA clusters, tcgen05 cta_group::2): the tile is 256 x BN;
// each CTA of the pair loads its own 128 rows of A and half (BN / 2 rows) of
// B, both loads completing on the leading CTA's ring barrier, and the leading
// CTA's MMA thread issues M = 256 MMAs that read both CTAs' shared memory and
// write 128 accumulator rows into each CTA's tensor memory.  Per SM that is
// 32 KB of operands per 64-wide k block instead of 48 KB, so 6 ring stages
// fit.  Stage and accumulator releases are two plain commits (one per CTA's
// barrier); the epilogue warps of both CTAs release an accumulator buffer on
// the leading CTA's barrier.  No multicast anywhere.
// Descriptor encodings follow the PTX ISA's tcgen05 shared-memory matrix
// descriptor (start >> 4, leading byte offset >> 4, stride byte offset >> 4,
// version 1, swizzle mode 2 = 128 B) and instruction descriptor (F32
// accumulator, BF16 A and B, per-operand major-ness, N >> 3, M >> 4).  Every
// wait is bounded by the global timer; a wait that gives up raises an abort
// flag that every role polls, reports DN_ETIMEOUT, lets copies and MMAs in
// flight finish (again bounded) and frees TMEM before the CTA exits.
#include <atomic>
#include <cuda.h>
#include <cuda_bf16.h>

#include "dn_common.cuh"
#include "dn_fno.h"
#include "dn_zmarch.cuh"

namespace dn {
namespace gm {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int NEPI = 8;  // epilogue warps: two per tensor-memory lane quadrant
constexpr int NT = 64 + 32 * NEPI;
constexpr int ATOM = 64;                   // MN extent of one 128-byte swizzle atom
constexpr int ATOM_BYTES = ATOM * BK * 2;  // 8 KB
constexpr int RING_BYTES = 192 * 1024;
constexpr int RING_BYTES_PAIR = 192 * 1024;
constexpr unsigned long long WAIT_NS = 4000000000ull;  // 4 s per wait
constexpr uint32_t SLEEP_NS = 20000;

template <int BN, bool PAIR>
struct Cfg {
  static constexpr int TILE_M = PAIR ? 2 * BM : BM;  // rows of one tile
  static constexpr int B_ROWS = PAIR ? BN / 2 : BN;  // B rows this CTA loads
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = B_ROWS * BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  // 8, 6, 4 stages for BN 64, 128, 256; 6 in pair mode at BN 256
  static constexpr int S = (PAIR ? RING_BYTES_PAIR : RING_BYTES) / STAGE;
  static constexpr int TMEM_COLS = 2 * BN;  // two accumulator buffers
  static constexpr int TEMPTY_ARRIVALS = PAIR ? 2 * NEPI : NEPI;  // one per epilogue warp
  static constexpr size_t SMEM = (size_t)S * STAGE + 1024 + 256;
  static_assert(SMEM <= 232448, "dynamic shared memory above the per-CTA limit");
  static_assert(B_ROWS % ATOM == 0, "B tile in whole swizzle atoms");
};

struct OpDev {
  int mn;       // MN-major
  int fold;     // 0 = no fold
  int batched;  // z coordinate = GEMM batch (else 0)
};

struct Params {
  long long M, N;
  int n_seg;
  int kb[2];
  OpDev a[2], b[2];
  int tiles_m, tiles_n;
  long long n_tiles;
  char* out;
  int out_bf16, accumulate;
  long long sb, R0, r0, r1, C0, c0, c1;
  float alpha;
  int act;
  const float* bias;
  const float* row_scale;
  const float* row_bias;
  const float* col_scale;
  const float* batch_scale;
  const char* addend;
  int addend_bf16;
  const char* aux;
  int aux_bf16;
  char* pre;
  int pre_bf16;
  int vec;
  int vec32;  // 32-byte aligned chunk rows: 256-bit stores
  int csub;   // column radix dividing 32 (else 0): per-element column offsets
  int* status;
};

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded spin (no suspend) for the producer / MMA hand-offs, where the
// wake-up latency of a suspended wait shows in the throughput
__device__ __forceinline__ bool gwait_spin(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const unsigned long long t0 = gtimer();
  for (uint32_t n = 0;; ++n) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((n & 255) == 255) {
      if (*abort) return false;
      if (gtimer() - t0 > WAIT_NS) return false;
    }
  }
}

// bounded wait; false when it gave up or another role aborted
__device__ __forceinline__ bool gwait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const unsigned long long t0 = gtimer();
  while (true) {
    if (mbar_try_wait_sleep(bar, parity, SLEEP_NS)) return true;
    if (*abort) return false;
    if (gtimer() - t0 > WAIT_NS) return false;
  }
}

// ---- cluster (CTA pair) helpers ---------------------------------------------
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// shared::cluster address of the same shared-memory offset in CTA `rank`
__device__ __forceinline__ uint32_t map_rank(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(caddr)
               : "memory");
}
__device__ __forceinline__ void st_cluster_u32(uint32_t caddr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(caddr), "r"(v) : "memory");
}
// every thread of both CTAs (no convergence requirement)
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// raise the abort flag of this CTA and (pair mode, peer_abort != 0) of the
// other CTA of the pair, and report the timeout
__device__ __forceinline__ void fail(volatile int* abort, int* status, uint32_t peer_abort = 0) {
  *abort = 1;
  if (peer_abort) st_cluster_u32(peer_abort, 1u);
  report_status(status, DN_ETIMEOUT);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_4d_g(void* dst, const CUtensorMap* m, uint64_t* bar,
                                              int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// pair-mode TMA loads: the data lands in this CTA's shared memory, the
// completion is counted on the barrier at cluster address `bar` (the leading
// CTA's).  No multicast.
__device__ __forceinline__ void tma_load_3d_pair(void* dst, const CUtensorMap* m, uint32_t bar,
                                                 int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void tma_load_4d_pair(void* dst, const CUtensorMap* m, uint32_t bar,
                                                 int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(bar), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// one operand tile (`rows_tile` rows from r0, k block from k0) into `dst`;
// pair mode: completion on the barrier at cluster address `cbar`
template <bool PAIR>
__device__ __forceinline__ void load_operand(unsigned char* dst, const CUtensorMap* m,
                                             const OpDev& o, uint64_t* bar, uint32_t cbar,
                                             int r0, int k0, int bz, int rows_tile) {
  const int z = o.batched ? bz : 0;
  if (!o.mn) {
    if constexpr (PAIR)
      tma_load_3d_pair(dst, m, cbar, k0, r0, z);
    else
      tma_load_3d(dst, m, bar, k0, r0, z);
  } else {
    for (int j = 0; j < rows_tile / ATOM; ++j) {
      const int r = r0 + j * ATOM;
      const int x = o.fold ? r % o.fold : r;
      const int f = o.fold ? r / o.fold : 0;
      if constexpr (PAIR)
        tma_load_4d_pair(dst + j * ATOM_BYTES, m, cbar, x, k0, f, z);
      else
        tma_load_4d_g(dst + j * ATOM_BYTES, m, bar, x, k0, f, z);
    }
  }
}

// K-major 128-byte-swizzled tile: 128-byte rows, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
         (2ull << 61);
}
// MN-major 128-byte-swizzled tile: 64-element atoms ATOM_BYTES apart
// (leading byte offset), 8-row k groups 1024 B apart (stride byte offset)
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(ATOM_BYTES >> 4) << 16) |
         (64ull << 32) | (1ull << 46) | (2ull << 61);
}

template <int BN, int TILE_M>
__device__ __forceinline__ uint32_t idesc(int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

// GELU in its tanh form (Hendrycks & Gimpel 2016):
//   gelu(v) = v/2 (1 + tanh(u)),  u = sqrt(2/pi) (v + 0.044715 v^3)
//   gelu'(v) = (1 + t)/2 + v/2 (1 - t^2) sqrt(2/pi) (1 + 3 * 0.044715 v^2),  t = tanh(u)
// with the hardware tanh (tanh.approx.f32, ~2^-11 relative error, far below
// the BF16 rounding of the activations).  The transform GEMMs of the
// operator are bound by epilogue instructions; this form costs a few FMAs
// and one special-function op per element.
constexpr float GELU_K0 = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float GELU_K1 = 0.044715f;
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float v) {
  const float t = tanh_hw(GELU_K0 * fmaf(GELU_K1 * v * v, v, v));
  return 0.5f * fmaf(v, t, v);
}
__device__ __forceinline__ float gelu_grad_f(float v) {
  const float v2 = v * v;
  const float t = tanh_hw(GELU_K0 * fmaf(GELU_K1 * v2, v, v));
  const float du = GELU_K0 * fmaf(3.0f * GELU_K1, v2, 1.0f);
  return 0.5f * fmaf(v * fmaf(-t, t, 1.0f), du, 1.0f + t);
}

__device__ __forceinline__ float bf2f(unsigned short h) {
  return __uint_as_float(static_cast<uint32_t>(h) << 16);
}
__device__ __forceinline__ unsigned short f2bf(float v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// 32 values starting at element offset `off` (column stride `cs`; `vec`:
// contiguous and 16-byte aligned), `nv` of them valid
__device__ __forceinline__ void load32(const char* base, int bf16, long long off, long long cs,
                                       bool vec, int nv, float* v) {
  if (vec) {
    if (bf16) {
      const uint4* p = reinterpret_cast<const uint4*>(base + off * 2);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 u = p[q];
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          v[q * 8 + 2 * e] = __uint_as_float(w[e] << 16);
          v[q * 8 + 2 * e + 1] = __uint_as_float(w[e] & 0xFFFF0000u);
        }
      }
    } else {
      const float4* p = reinterpret_cast<const float4*>(base + off * 4);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 u = p[q];
        v[4 * q] = u.x;
        v[4 * q + 1] = u.y;
        v[4 * q + 2] = u.z;
        v[4 * q + 3] = u.w;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      float x = 0.0f;
      if (j < nv) {
        const long long o = off + j * cs;
        x = bf16 ? bf2f(reinterpret_cast<const unsigned short*>(base)[o])
                 : reinterpret_cast<const float*>(base)[o];
      }
      v[j] = x;
    }
  }
}

__device__ __forceinline__ void st256(void* p, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                      uint32_t e, uint32_t f, uint32_t g, uint32_t h) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(a), "r"(b),
               "r"(c), "r"(d), "r"(e), "r"(f), "r"(g), "r"(h)
               : "memory");
}

// 32 values from element offset `off` with 256-bit stores, so that every
// lane writes whole 32-byte sectors (the lanes of a warp write 32 different
// rows); the chunk start is 32-byte aligned
__device__ __forceinline__ void store32_v8(char* base, int bf16, long long off, const float* v) {
  if (bf16) {
    char* p = base + off * 2;
    uint32_t w[16];
#pragma unroll
    for (int e = 0; e < 16; ++e)
      w[e] = static_cast<uint32_t>(f2bf(v[2 * e])) |
             (static_cast<uint32_t>(f2bf(v[2 * e + 1])) << 16);
    st256(p, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7]);
    st256(p + 32, w[8], w[9], w[10], w[11], w[12], w[13], w[14], w[15]);
  } else {
    char* p = base + off * 4;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      st256(p + 32 * q, __float_as_uint(v[8 * q]), __float_as_uint(v[8 * q + 1]),
            __float_as_uint(v[8 * q + 2]), __float_as_uint(v[8 * q + 3]),
            __float_as_uint(v[8 * q + 4]), __float_as_uint(v[8 * q + 5]),
            __float_as_uint(v[8 * q + 6]), __float_as_uint(v[8 * q + 7]));
  }
}

__device__ __forceinline__ void store32(char* base, int bf16, long long off, long long cs,
                                        bool vec, int nv, const float* v) {
  if (vec) {
    if (bf16) {
      uint4* p = reinterpret_cast<uint4*>(base + off * 2);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e)
          w[e] = static_cast<uint32_t>(f2bf(v[q * 8 + 2 * e])) |
                 (static_cast<uint32_t>(f2bf(v[q * 8 + 2 * e + 1])) << 16);
        p[q] = make_uint4(w[0], w[1], w[2], w[3]);
      }
    } else {
      float4* p = reinterpret_cast<float4*>(base + off * 4);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        p[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < nv) {
        const long long o = off + j * cs;
        if (bf16)
          reinterpret_cast<unsigned short*>(base)[o] = f2bf(v[j]);
        else
          reinterpret_cast<float*>(base)[o] = v[j];
      }
    }
  }
}

__device__ __forceinline__ void tile_coords(long long t, const Params& p, int& mt, int& nt,
                                            int& bz) {
  const long long per_batch = (long long)p.tiles_m * p.tiles_n;
  bz = (int)(t / per_batch);
  long long r = t % per_batch;
  const int G = 16;
  const long long gsize = (long long)G * p.tiles_n;
  const int g = (int)(r / gsize);
  const int m0 = g * G;
  const int gm = p.tiles_m - m0 < G ? p.tiles_m - m0 : G;
  r -= (long long)g * gsize;
  mt = m0 + (int)(r % gm);
  nt = (int)(r / gm);
}

template <int BN, bool PAIR>
__global__ void __launch_bounds__(NT, 1)
    k_gemm(const __grid_constant__ CUtensorMap ta0, const __grid_constant__ CUtensorMap tb0,
           const __grid_constant__ CUtensorMap ta1, const __grid_constant__ CUtensorMap tb1,
           const Params p) {
  using C = Cfg<BN, PAIR>;
  constexpr int S = C::S;
  extern __shared__ __align__(1024) unsigned char g_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(g_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + S * C::STAGE);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // pair mode: rank 0 of the cluster leads (issues the MMAs, owns the ring
  // and accumulator-release barriers that both CTAs signal)
  const uint32_t rank = PAIR ? cluster_rank() : 0u;
  const long long unit0 = PAIR ? (long long)cluster_id() : (long long)blockIdx.x;
  const long long n_units = PAIR ? (long long)cluster_count() : (long long)gridDim.x;
  const uint32_t peer_abort = PAIR ? map_rank((const void*)abort, rank ^ 1u) : 0u;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], C::TEMPTY_ARRIVALS);
    }
    mbar_init(drain, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    if constexpr (PAIR) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"((uint32_t)C::TMEM_COLS)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"((uint32_t)C::TMEM_COLS)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if constexpr (PAIR) cluster_barrier();  // both CTAs' barriers initialised
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int kb_total = p.kb[0] + (p.n_seg > 1 ? p.kb[1] : 0);

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer (both CTAs in pair mode) -----------------------------
      long long g = 0;
      for (long long t = unit0; t < p.n_tiles && !*abort; t += n_units) {
        int mt, nt, bz;
        tile_coords(t, p, mt, nt, bz);
        bool ok = true;
        for (int kb = 0; kb < kb_total; ++kb, ++g) {
          const int s = (int)(g % S);
          if (g >= S && !gwait_spin(&empty[s], (uint32_t)(((g / S) - 1) & 1), abort)) {
            fail(abort, p.status, peer_abort);
            ok = false;
            break;
          }
          const int seg = kb < p.kb[0] ? 0 : 1;
          const int k0 = (seg == 0 ? kb : kb - p.kb[0]) * BK;
          unsigned char* st = ring + s * C::STAGE;
          uint32_t cbar = 0;
          if constexpr (PAIR) {
            // the leading CTA's barrier counts both CTAs' bytes
            cbar = map_rank(&full[s], 0u);
            if (rank == 0) mbar_arrive_expect_tx(&full[s], 2 * C::STAGE);
          } else {
            mbar_arrive_expect_tx(&full[s], C::STAGE);
          }
          const int ar0 = mt * C::TILE_M + (int)rank * BM;
          const int br0 = nt * BN + (int)rank * C::B_ROWS;
          load_operand<PAIR>(st, seg == 0 ? &ta0 : &ta1, p.a[seg], &full[s], cbar, ar0, k0, bz,
                             BM);
          load_operand<PAIR>(st + C::A_BYTES, seg == 0 ? &tb0 : &tb1, p.b[seg], &full[s], cbar,
                             br0, k0, bz, C::B_ROWS);
        }
        if (!ok) break;
      }
      if (*abort && rank == 0) {
        // let the copies already issued land before the CTA goes away
        for (long long q = (g > S ? g - S : 0); q < g; ++q) {
          const int s = (int)(q % S);
          const unsigned long long t0 = gtimer();
          while (!mbar_try_wait_sleep(&full[s], (uint32_t)((q / S) & 1), SLEEP_NS) &&
                 gtimer() - t0 < WAIT_NS) {
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---- MMA issuer (the leading CTA only in pair mode) ---------------------
      const uint32_t id0 = idesc<BN, C::TILE_M>(p.a[0].mn, p.b[0].mn);
      const uint32_t id1 = idesc<BN, C::TILE_M>(p.a[1].mn, p.b[1].mn);
      long long g = 0;
      int it = 0;
      for (long long t = unit0; t < p.n_tiles && !*abort; t += n_units, ++it) {
        const int buf = it & 1;
        if (it >= 2 && !gwait_spin(&tempty[buf], (uint32_t)(((it >> 1) - 1) & 1), abort)) {
          fail(abort, p.status, peer_abort);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_addr = tmem + (uint32_t)(buf * BN);
        bool ok = true;
        for (int kb = 0; kb < kb_total; ++kb, ++g) {
          const int s = (int)(g % S);
          if (!gwait_spin(&full[s], (uint32_t)((g / S) & 1), abort)) {
            fail(abort, p.status, peer_abort);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int seg = kb < p.kb[0] ? 0 : 1;
          const uint32_t id = seg == 0 ? id0 : id1;
          const int amn = p.a[seg].mn, bmn = p.b[seg].mn;
          const uint32_t sa = smem_u32(ring + s * C::STAGE);
          const uint32_t sbb = sa + C::A_BYTES;
#pragma unroll
          for (int k16 = 0; k16 < BK / 16; ++k16) {
            const uint64_t da = amn ? desc_mnmajor(sa + k16 * 2048) : desc_kmajor(sa + k16 * 32);
            const uint64_t db =
                bmn ? desc_mnmajor(sbb + k16 * 2048) : desc_kmajor(sbb + k16 * 32);
            const uint32_t accum = (kb > 0 || k16 > 0) ? 1u : 0u;
            if constexpr (PAIR) {
              asm volatile(
                  "{\n\t.reg .pred p;\n\t"
                  "setp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc_addr),
                  "l"(da), "l"(db), "r"(id), "r"(accum)
                  : "memory");
            } else {
              asm volatile(
                  "{\n\t.reg .pred p;\n\t"
                  "setp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc_addr),
                  "l"(da), "l"(db), "r"(id), "r"(accum)
                  : "memory");
            }
          }
          if constexpr (PAIR) {
            asm volatile(
                "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&empty[s]))
                : "memory");
            asm volatile(
                "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    map_rank(&empty[s], 1u))
                : "memory");
          } else {
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&empty[s]))
                : "memory");
          }
        }
        if (!ok) break;
        if constexpr (PAIR) {
          asm volatile(
              "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  smem_u32(&tfull[buf]))
              : "memory");
          asm volatile(
              "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  map_rank(&tfull[buf], 1u))
              : "memory");
        } else {
          asm volatile(
              "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  smem_u32(&tfull[buf]))
              : "memory");
        }
      }
      // every MMA issued by this thread completes before TMEM is freed
      if constexpr (PAIR) {
        asm volatile(
            "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(drain))
            : "memory");
      } else {
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(drain))
            : "memory");
      }
      const unsigned long long t0 = gtimer();
      while (!mbar_try_wait_sleep(drain, 0, SLEEP_NS) && gtimer() - t0 < WAIT_NS) {
      }
    }
  } else {
    // ---- epilogue: warps 2..9 ----------------------------------------------
    const int quad = warp & 3;  // TMEM lanes 32*quad .. 32*quad+31
    const int c_beg = ((warp - 2) >> 2) * (BN / 2);  // this warp's half of the columns
    int it = 0;
    for (long long t = unit0; t < p.n_tiles; t += n_units, ++it) {
      const int buf = it & 1;
      const bool ready = gwait(&tfull[buf], (uint32_t)((it >> 1) & 1), abort);
      if (!__all_sync(0xffffffffu, ready)) {
        if (lane == 0) fail(abort, p.status, peer_abort);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int mt, nt, bz;
      tile_coords(t, p, mt, nt, bz);
      const long long row = (long long)mt * C::TILE_M + (long long)rank * BM + quad * 32 + lane;
      const bool row_ok = row < p.M;
      float scale = p.alpha;
      if (row_ok && p.row_scale) scale *= p.row_scale[row];
      const float rbias = (row_ok && p.row_bias) ? p.row_bias[row] : 0.0f;
      if (p.batch_scale) scale *= p.batch_scale[bz];
      const long long roff = (long long)bz * p.sb + (row % p.R0) * p.r0 + (row / p.R0) * p.r1;
#pragma unroll 1
      for (int c = c_beg; c < c_beg + BN / 2; c += 32) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * BN + c);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
            "%26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
              "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
              "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const long long col = (long long)nt * BN + c;
        if (row_ok && col < p.N) {
          const int nv = (int)(p.N - col < 32 ? p.N - col : 32);
          const bool vec = p.vec && nv == 32;
          const long long off = roff + (col % p.C0) * p.c0 + (col / p.C0) * p.c1;
          float v[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]) * scale;
          if (p.col_scale) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (j < nv) v[j] *= p.col_scale[col + j];
          }
          if (p.row_bias) {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] += rbias;
          }
          if (p.bias) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (j < nv) v[j] += p.bias[col + j];
          }
          float w[32];
          if (p.addend) {
            load32(p.addend, p.addend_bf16, off, p.c0, vec, nv, w);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] += w[j];
          }
          if (p.act == DN_ACT_GELU) {
            if (p.pre) {
              if (vec && p.vec32)
                store32_v8(p.pre, p.pre_bf16, off, v);
              else
                store32(p.pre, p.pre_bf16, off, p.c0, vec, nv, v);
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = gelu_f(v[j]);
          } else if (p.act == DN_ACT_GELU_GRAD) {
            load32(p.aux, p.aux_bf16, off, p.c0, vec, nv, w);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] *= gelu_grad_f(w[j]);
          }
          if (p.accumulate) {
            load32(p.out, 0, off, p.c0, vec, nv, w);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] += w[j];
          }
          if (p.csub) {
            // column radix dividing 32: a chunk holds 32 / csub whole radix
            // groups; plain stores only (checked on the host)
            const long long ob = roff + (col / p.csub) * p.c1;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              if (j >= nv) continue;
              const long long o = ob + (j % p.csub) * p.c0 + (j / p.csub) * p.c1;
              if (p.out_bf16)
                reinterpret_cast<unsigned short*>(p.out)[o] = f2bf(v[j]);
              else
                reinterpret_cast<float*>(p.out)[o] = v[j];
            }
          } else if (vec && p.vec32) {
            store32_v8(p.out, p.out_bf16, off, v);
          } else {
            store32(p.out, p.out_bf16, off, p.c0, vec, nv, v);
          }
        }
        __syncwarp();  // reconverge before the next warp-wide tcgen05.ld
      }
      // release the accumulator buffer: one arrival per warp, on the leading
      // CTA's barrier in pair mode
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        if constexpr (PAIR)
          mbar_arrive_cluster(map_rank(&tempty[buf], 0u));
        else
          mbar_arrive(&tempty[buf]);
      }
    }
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // pair mode: neither CTA leaves (or frees its tensor memory) while the
  // other may still signal its barriers or the MMAs read its shared memory
  if constexpr (PAIR) cluster_barrier();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if constexpr (PAIR) {
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"((uint32_t)C::TMEM_COLS)
                   : "memory");
    } else {
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"((uint32_t)C::TMEM_COLS)
                   : "memory");
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int check_operand(const dn_gemm_operand& o) {
  if (!o.ptr || !aligned16(o.ptr) || o.rows < 1 || o.k < 1 || o.ld < 1) return DN_EINVAL;
  if (o.ld % 8 || o.batch_stride % 8 || o.batch_stride < 0) return DN_EINVAL;
  if (o.mn_major != 0 && o.mn_major != 1) return DN_EINVAL;
  if (o.mn_major) {
    if (o.fold < 0 || o.fold % 64) return DN_EINVAL;
    if (o.fold && (o.fold_stride < 1 || o.fold_stride % 8)) return DN_EINVAL;
  } else if (o.fold) {
    return DN_EINVAL;
  }
  if (o.rows > 0x7fffffffLL || o.k > 0x7fffffffLL) return DN_EUNSUPPORTED;
  return DN_OK;
}

int encode_operand(CUtensorMap* m, const dn_gemm_operand& o, int batch, int rows_tile) {
  zm::EncodeTiledFn fn = zm::get_encode();
  if (!fn) return DN_ECUDA;
  const long long nb = o.batch_stride > 0 ? batch : 1;
  const cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r;
  if (!o.mn_major) {
    const long long zs = o.batch_stride > 0 ? o.batch_stride : o.ld * o.rows;
    const cuuint64_t dims[3] = {(cuuint64_t)o.k, (cuuint64_t)o.rows, (cuuint64_t)nb};
    const cuuint64_t strides[2] = {(cuuint64_t)o.ld * 2, (cuuint64_t)zs * 2};
    const cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)rows_tile, 1};
    r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(o.ptr), dims, strides, box,
           es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const long long inner = o.fold ? o.fold : o.rows;
    const long long nf = o.fold ? (o.rows + o.fold - 1) / o.fold : 1;
    const long long fs = o.fold ? o.fold_stride : o.ld * o.k;
    const long long zs = o.batch_stride > 0 ? o.batch_stride : fs * nf;
    const cuuint64_t dims[4] = {(cuuint64_t)inner, (cuuint64_t)o.k, (cuuint64_t)nf,
                                (cuuint64_t)nb};
    const cuuint64_t strides[3] = {(cuuint64_t)o.ld * 2, (cuuint64_t)fs * 2, (cuuint64_t)zs * 2};
    const cuuint32_t box[4] = {(cuuint32_t)ATOM, (cuuint32_t)BK, 1, 1};
    r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(o.ptr), dims, strides, box,
           es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS) {
    set_last_cuda_error(static_cast<int>(r));
    return DN_ECUDA;
  }
  return DN_OK;
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
  return n > 0 ? n : 148;
}

// co-resident two-CTA clusters of the pair kernel (0 when none fit)
template <int BN>
int pair_clusters() {
  // filled once; an atomic so that concurrent host threads may both fill it
  // (same value, and the shared-memory attribute they set is idempotent)
  static std::atomic<int> cached{-1};
  const int c = cached.load(std::memory_order_acquire);
  if (c >= 0) return c;
  using C = Cfg<BN, true>;
  auto kern = k_gemm<BN, true>;
  int n = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM) ==
      cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (unsigned)sm_count(), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = C::SMEM;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) n = 0;
  }
  (void)cudaGetLastError();
  cached.store(n, std::memory_order_release);
  return n;
}

template <int BN, bool PAIR>
int launch(const dn_gemm& g, Params p, int* status, cudaStream_t s) {
  using C = Cfg<BN, PAIR>;
  CUtensorMap m[4];
  int rc;
  for (int seg = 0; seg < 2; ++seg) {
    const int src = seg < g.n_seg ? seg : 0;  // unused segment: a valid copy of segment 0
    if ((rc = encode_operand(&m[2 * seg], g.a[src], g.batch, BM)) != DN_OK) return rc;
    if ((rc = encode_operand(&m[2 * seg + 1], g.b[src], g.batch, C::B_ROWS)) != DN_OK) return rc;
  }
  p.tiles_m = (int)((g.M + C::TILE_M - 1) / C::TILE_M);
  p.tiles_n = (int)((g.N + BN - 1) / BN);
  p.n_tiles = (long long)p.tiles_m * p.tiles_n * g.batch;
  p.status = status;
  auto kern = k_gemm<BN, PAIR>;
  DN_CUDA_CHECK(
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  if constexpr (!PAIR) {
    long long ctas = g.max_ctas > 0 ? g.max_ctas : sm_count();
    if (ctas > p.n_tiles) ctas = p.n_tiles;
    kern<<<(unsigned)ctas, NT, C::SMEM, s>>>(m[0], m[1], m[2], m[3], p);
  } else {
    long long pairs = pair_clusters<BN>();
    if (g.max_ctas > 0 && g.max_ctas / 2 < pairs) pairs = g.max_ctas / 2;
    if (pairs > p.n_tiles) pairs = p.n_tiles;
    if (pairs < 1) return DN_EUNSUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * pairs), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = C::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DN_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m[0], m[1], m[2], m[3], p));
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

bool dtype_ok(int32_t d) { return d == DN_F32 || d == DN_BF16; }
int esize(int32_t d) { return d == DN_BF16 ? 2 : 4; }

// `bytes`-wide vector access to a 32-column chunk is valid for this pointer
bool vec_ok(const dn_gemm& g, const void* ptr, int es, int bytes = 16) {
  if (!ptr) return true;
  if (reinterpret_cast<uintptr_t>(ptr) % bytes) return false;
  const long long q = bytes / es;
  const long long strides[4] = {g.c_batch_stride, g.c_row_stride0, g.c_row_stride1,
                                g.c_col_stride1};
  for (long long st : strides)
    if (st % q) return false;
  return true;
}

}  // namespace gm
}  // namespace dn

extern "C" int32_t dn_gemm_run(const dn_gemm* g, int32_t* status, void* stream) {
  using namespace dn::gm;
  if (!g || g->M < 1 || g->N < 1 || g->batch < 1 || g->n_seg < 1 || g->n_seg > 2 || !g->out)
    return DN_EINVAL;
  if (g->M > 0x7fffffffLL || g->N > 0x7fffffffLL || g->batch > 0x7fffffff / 2)
    return DN_EUNSUPPORTED;
  Params p{};
  for (int s = 0; s < g->n_seg; ++s) {
    int rc;
    if ((rc = check_operand(g->a[s])) != DN_OK || (rc = check_operand(g->b[s])) != DN_OK)
      return rc;
    if (g->a[s].k != g->b[s].k) return DN_EINVAL;
    p.kb[s] = (int)((g->a[s].k + BK - 1) / BK);
    p.a[s] = OpDev{g->a[s].mn_major, g->a[s].fold, g->a[s].batch_stride > 0 ? 1 : 0};
    p.b[s] = OpDev{g->b[s].mn_major, g->b[s].fold, g->b[s].batch_stride > 0 ? 1 : 0};
  }
  if (g->n_seg == 1) {
    p.kb[1] = 0;
    p.a[1] = p.a[0];
    p.b[1] = p.b[0];
  }
  if (!dtype_ok(g->out_dtype) || (g->accumulate && g->out_dtype != DN_F32)) return DN_EINVAL;
  if (g->act < DN_ACT_NONE || g->act > DN_ACT_GELU_GRAD) return DN_EINVAL;
  if (g->act == DN_ACT_GELU_GRAD && (!g->aux || !dtype_ok(g->aux_dtype))) return DN_EINVAL;
  if (g->pre && (g->act != DN_ACT_GELU || !dtype_ok(g->pre_dtype))) return DN_EINVAL;
  if (g->addend && !dtype_ok(g->addend_dtype)) return DN_EINVAL;
  if (g->c_row_radix < 0 || g->c_col_radix < 0) return DN_EINVAL;
  // a column radix is a multiple of 32, or a divisor of 32 for plain stores
  const bool small_radix = g->c_col_radix > 0 && g->c_col_radix < 32;
  if (small_radix && (32 % g->c_col_radix || g->addend || g->aux || g->pre || g->accumulate))
    return DN_EINVAL;
  if (!small_radix && (g->c_col_radix % 32)) return DN_EINVAL;
  if (g->block_n != 0 && g->block_n != 64 && g->block_n != 128 && g->block_n != 256)
    return DN_EINVAL;
  if (g->pair < 0 || g->pair > 2 || (g->pair == 2 && g->block_n != 0 && g->block_n != 256))
    return DN_EINVAL;

  p.M = g->M;
  p.N = g->N;
  p.n_seg = g->n_seg;
  p.out = static_cast<char*>(g->out);
  p.out_bf16 = g->out_dtype == DN_BF16;
  p.accumulate = g->accumulate != 0;
  p.sb = g->c_batch_stride;
  p.R0 = g->c_row_radix > 0 ? g->c_row_radix : (1LL << 62);
  p.r0 = g->c_row_stride0;
  p.r1 = g->c_row_stride1;
  p.C0 = g->c_col_radix >= 32 ? g->c_col_radix : (1LL << 62);
  p.csub = small_radix ? (int)g->c_col_radix : 0;
  p.c0 = g->c_col_stride0;
  p.c1 = g->c_col_stride1;
  p.alpha = g->alpha;
  p.act = g->act;
  p.bias = g->bias;
  p.row_scale = g->row_scale;
  p.col_scale = g->col_scale;
  p.row_bias = g->row_bias;
  p.batch_scale = g->batch_scale;
  p.addend = static_cast<const char*>(g->addend);
  p.addend_bf16 = g->addend_dtype == DN_BF16;
  p.aux = static_cast<const char*>(g->aux);
  p.aux_bf16 = g->aux_dtype == DN_BF16;
  p.pre = static_cast<char*>(g->pre);
  p.pre_bf16 = g->pre_dtype == DN_BF16;
  p.vec = g->c_col_stride0 == 1 && vec_ok(*g, g->out, esize(g->out_dtype)) &&
          vec_ok(*g, g->addend, esize(g->addend_dtype)) &&
          vec_ok(*g, g->aux, esize(g->aux_dtype)) && vec_ok(*g, g->pre, esize(g->pre_dtype));
  // a chunk starts at a multiple of 32 columns (and of the column radix), so
  // 32-byte aligned bases and strides keep every chunk start 32-byte aligned
  p.vec32 = p.vec && vec_ok(*g, g->out, esize(g->out_dtype), 32) &&
            vec_ok(*g, g->pre, esize(g->pre_dtype), 32);

  int bn = g->block_n;
  if (bn == 0) {
    const long long n64 = (g->N + 63) / 64 * 64;
    const long long tiles_m = (g->M + BM - 1) / BM;
    const long long sms = sm_count();
    bn = 64;
    for (int cand : {256, 128}) {
      if (cand > n64) continue;
      if (tiles_m * ((g->N + cand - 1) / cand) * g->batch >= sms) {
        bn = cand;
        break;
      }
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // two-CTA 256 x 256 tiles only when asked for: on B200 they measured
  // 2-5 % slower than one-CTA tiles at 4096^3 / 8192^3 and on the operator's
  // transform GEMMs (the one-CTA kernel is not operand-bandwidth bound)
  if (g->pair == 2) {
    if (pair_clusters<256>() < 1) return DN_EUNSUPPORTED;
    return launch<256, true>(*g, p, status, s);
  }
  if (bn == 64) return launch<64, false>(*g, p, status, s);
  if (bn == 128) return launch<128, false>(*g, p, status, s);
  return launch<256, false>(*g, p, status, s);
}
