// 3-D Yee step for sm_100a: all six components updated in one pass.
//
// Replaces the loop body of DiffNano's FDTDSolver3D._run_steps
// (diffnano/solvers/fdtd3d.py:490-502): _time_step (:378-465) -- H from the
// old E, then E from the new H, each with the CPML damping b and the curl
// scale (1+c) -- followed by the soft-source add.  Axes: i = z (D), j = y
// (H), k = x (W, contiguous).  Forward differences are 0 on the last index,
// backward differences 0 on the first.  Two coefficient mappings:
//   DN_AXES_REFERENCE  the reference's own broadcasting (cubic grids only):
//                      every profile is indexed by j or k, none by i;
//   DN_AXES_PHYSICAL   each profile indexed along its own axis.
//
// Design (memory bound, 52 B per cell-step in FP32: 7 arrays read, 6 written):
//  * a CTA owns a 16 (y) x 32 (x) column of cells over a range of planes and
//    marches along z; consecutive CTAs are neighbouring tiles over the same
//    z range, so CTAs that run together stay in lockstep and the halo rows /
//    columns one CTA fetches are L2 hits for its neighbours;
//  * a producer warp streams each plane's inputs (Ex, Ey, Ez, Hx, Hy, Hz,
//    dt/eps) with 3-D TMA boxes (x from k0-4 so the start is 16-byte aligned,
//    y from j0-1) into a ring of shared-memory stages guarded by "full"
//    (transaction-count) and "empty" (consumer-release) mbarriers, several
//    planes ahead of the consumers;
//  * eight consumer warps each own two rows of the tile and never synchronise
//    with each other: a warp recomputes the new H of the row above its pair
//    (instead of exchanging it), takes the x-1 neighbour by warp shuffle (two
//    lanes compute the k0-1 halo column), keeps new Hx, Hy of the plane below
//    in registers (the z sliding window), updates E, applies the source, DFT
//    monitors and probe in registers, and stores all six results to the other
//    ping-pong buffer (neighbouring CTAs still read the old one).
#include <cuda.h>

#include <mutex>

#include "dn_host.cuh"

namespace dn {
namespace {

constexpr int TX = 32;                // tile x (one warp)
constexpr int TY = 16;                // tile y
constexpr int NCW = TY / 2;           // consumer warps, two rows each
constexpr int NT3 = (NCW + 1) * 32;   // + one producer warp
constexpr int BX = TX + 8;            // box x: k0-4 .. k0+TX+3
constexpr int BY = TY + 2;            // box y: j0-1 .. j0+TY
constexpr int NARR = 7;               // Ex Ey Ez Hx Hy Hz ce
constexpr int A_CE = 6;
constexpr int MIN_CHUNK = 8;          // min planes per CTA range
constexpr uint32_t WAIT_PROBES = 1u << 16;  // bound on mbarrier probes per wait
constexpr uint32_t SLEEP_NS = 20000;        // suspend-time hint per probe (~1.3 s bound)

template <typename T>
struct Cfg {
  static constexpr int S = sizeof(T) == 4 ? 5 : 3;  // ring stages
  static constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
  static constexpr int BOX_BYTES = BX * BY * (int)sizeof(T);
  static constexpr int ARR_BYTES = (BOX_BYTES + 127) / 128 * 128;
  static constexpr int STAGE_BYTES = NARR * ARR_BYTES;
  static constexpr int TX_BYTES = NARR * BOX_BYTES;
  static constexpr int TAB_BYTES = (2 * (TY + 2) + 2 * (TX + 2)) * (int)sizeof(T);
};

struct alignas(64) TmapSet {
  CUtensorMap m[NARR];
};

// Work split: CTA b owns tile (b % ntiles) for z in [split*D/nsplit,
// (split+1)*D/nsplit), split = b / ntiles.
struct Plan {
  int ntx;     // tiles along x
  int ntiles;  // tiles per plane
  int nsplit;  // z ranges per tile
  int maxj;    // job-list capacity
};

constexpr unsigned FULL_MASK = 0xffffffffu;

// bounded wait on an mbarrier phase that also gives up when another warp has
// flagged an abort
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t n = 0; n < WAIT_PROBES; ++n) {
    if (mbar_try_wait_sleep(bar, parity, SLEEP_NS)) return true;
    if ((n & 15u) == 15u && *abort) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// source / DFT monitors / probe on one cell's six new values (kept in
// registers: components are selected, never indexed)
template <typename T>
__device__ __forceinline__ T pick(int c, T ex, T ey, T ez, T hx, T hy, T hz) {
  return c == DN_EX ? ex : c == DN_EY ? ey : c == DN_EZ ? ez : c == DN_HX ? hx : c == DN_HY ? hy : hz;
}

template <typename T>
__device__ __forceinline__ void special_cell(const StepParams<T>& p, int i, int j, int k, T& ex,
                                             T& ey, T& ez, T& hx, T& hy, T& hz) {
  if (p.src.comp >= 0 && p.src.box.contains(i, j, k)) {
    const T w = p.src.wave[p.t];
    const int c = p.src.comp;
    ex += c == DN_EX ? w : T(0);
    ey += c == DN_EY ? w : T(0);
    ez += c == DN_EZ ? w : T(0);
    hx += c == DN_HX ? w : T(0);
    hy += c == DN_HY ? w : T(0);
    hz += c == DN_HZ ? w : T(0);
  }
#pragma unroll
  for (int m = 0; m < DN_MAX_MONITORS; ++m) {
    if (m >= p.n_mon) break;
    const MonDev& M = p.mon[m];
    if (!M.box.contains(i, j, k)) continue;
    const double x = static_cast<double>(pick(M.comp, ex, ey, ez, hx, hy, hz));
    const long long cell = M.box.offset(i, j, k);
    const double* ph = M.phase + (long long)p.t * M.nf * 2;
    for (int f = 0; f < M.nf; ++f) {
      double* a = M.acc + ((long long)f * M.ncell + cell) * 2;
      a[0] = fma(x, ph[2 * f + 0], a[0]);
      a[1] = fma(x, ph[2 * f + 1], a[1]);
    }
  }
  if (p.probe.comp >= 0 && i == p.probe.pos[0] && j == p.probe.pos[1] && k == p.probe.pos[2])
    p.probe.out[p.t] = pick(p.probe.comp, ex, ey, ez, hx, hy, hz);
}

template <typename T, int AXES>
__global__ void __launch_bounds__(NT3, Cfg<T>::MINB)
    k_fdtd3d(const StepParams<T> p, const __grid_constant__ TmapSet tm, const Plan plan) {
  using C = Cfg<T>;
  constexpr int S = C::S;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must be 128-byte aligned: align the carve explicitly
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  unsigned char* stages = smem;
  T* sbJ = reinterpret_cast<T*>(smem + S * C::STAGE_BYTES);
  T* sgJ = sbJ + (TY + 2);
  T* sbK = sgJ + (TY + 2);
  T* sgK = sbK + (TX + 2);
  uint64_t* full = reinterpret_cast<uint64_t*>(
      smem + ((S * C::STAGE_BYTES + C::TAB_BYTES + 15) / 16) * 16);
  uint64_t* empty = full + S;
  int* s_flags = reinterpret_cast<int*>(empty + S);  // [0] job count, [1] abort flag
  int2* jobs = reinterpret_cast<int2*>(s_flags + 2);
  volatile int* s_abort = s_flags + 1;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int D = p.D, H = p.H, W = p.W;
  const long long py = p.py, pz = p.pz;
  const T dt = p.dt, idl = p.inv_dl;
  const int tile = blockIdx.x % plan.ntiles;
  const int split = blockIdx.x / plan.ntiles;
  const int z0 = (int)((long long)split * D / plan.nsplit);
  const int z1 = (int)((long long)(split + 1) * D / plan.nsplit);
  const int tyi = tile / plan.ntx, txi = tile % plan.ntx;
  const int k0 = txi * TX, j0 = tyi * TY;

  if (tid == 0) {
    // jobs = planes whose inputs this CTA loads, in consumption order: the
    // warm-up plane z0-1 (new Hx, Hy below the range), z0..z1-1, and plane z1
    // (E only, for the forward z-differences of plane z1-1)
    int nj = 0;
    if (z0 > 0) jobs[nj++] = make_int2(tile, z0 - 1);
    for (int z = z0; z < z1; ++z) jobs[nj++] = make_int2(tile, z);
    if (z1 < D) jobs[nj++] = make_int2(tile, z1);
    // a previous launch that recorded an error turns this one into a no-op
    const bool skip = p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0;
    s_flags[0] = skip ? 0 : nj;
    s_flags[1] = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    fence_barrier_init();
  }
  for (int e = tid; e < TY + 2; e += NT3) {
    const int j = j0 - 1 + e;
    const bool ok = j >= 0 && j < H;
    sbJ[e] = ok ? static_cast<T>(p.b[1][j]) : T(1);
    sgJ[e] = ok ? static_cast<T>(1.0 + p.c[1][j]) : T(1);
  }
  for (int e = tid; e < TX + 2; e += NT3) {
    const int kx = k0 - 1 + e;
    const bool ok = kx >= 0 && kx < W;
    sbK[e] = ok ? static_cast<T>(p.b[2][kx]) : T(1);
    sgK[e] = ok ? static_cast<T>(1.0 + p.c[2][kx]) : T(1);
  }
  __syncthreads();  // the only CTA-wide barrier
  const int nj = s_flags[0];
  if (nj == 0) return;

  auto stage_arr = [&](int q, int a) -> const T* {
    return reinterpret_cast<const T*>(stages + (q % S) * C::STAGE_BYTES + a * C::ARR_BYTES);
  };
  constexpr int AE = C::ARR_BYTES / (int)sizeof(T);  // elements between staged arrays

  // ======================= producer warp ====================================
  if (warp == NCW) {
    if (lane == 0) {
      bool ok = true;
      int issued = 0;
      for (int q = 0; q < nj && ok; ++q) {
        if (q >= S) ok = wait_phase(&empty[q % S], ((q / S) - 1) & 1, s_abort);
        if (!ok) break;
        const int2 jb = jobs[q];
        uint64_t* bar = &full[q % S];
        unsigned char* dst = stages + (q % S) * C::STAGE_BYTES;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, C::TX_BYTES);
        for (int a = 0; a < NARR; ++a)
          tma_load_3d(dst + a * C::ARR_BYTES, &tm.m[a], bar, k0 - 4, j0 - 1, jb.y);
        issued = q + 1;
      }
      // stay until the consumers released the last stages, so no copy can
      // still be in flight when the CTA's shared memory is given back
      for (int q = max(0, nj - S); q < nj && ok; ++q)
        ok = wait_phase(&empty[q % S], (q / S) & 1, s_abort);
      if (!ok) {
        report_status(p.status, DN_ETIMEOUT);
        *s_abort = 1;
        for (int q = max(0, issued - S); q < issued; ++q)
          (void)mbar_wait_bounded(&full[q % S], (q / S) & 1, WAIT_PROBES);
      }
    }
    return;
  }

  // ======================= consumer warps ===================================
  const int w = warp;
  const int ja = j0 + 2 * w;  // rows ja, ja+1 are owned; row ja-1 is recomputed
  const int k = k0 + lane;
  const bool kin = k < W;
  const T dti = dt * idl;
  // Per-lane coefficients with the boundary rules folded in: a forward
  // difference on the last index and a backward difference on the first one
  // get a zero coefficient.  The neighbour read there is a zero-filled TMA
  // element or an in-range finite value, so 0 * value == 0 exactly.
  const T bK = sbK[lane + 1], gK = sgK[lane + 1];
  const T bKh = sbK[0], gKh = sgK[0];
  const T kf = (k < W - 1) ? T(1) : T(0);
  const T kb = (k > 0) ? T(1) : T(0);
  const T cKf = kf * dti * gK;  // dt (1+c_k)/dl on a forward x difference
  const T cKb = kb * gK * idl;  // (1+c_k)/dl on a backward x difference
  T bJ[3], gJ[3], cJf[3], cJb[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int j = ja + r - 1;
    bJ[r] = sbJ[2 * w + r];
    gJ[r] = sgJ[2 * w + r];
    cJf[r] = (j < H - 1) ? dti * gJ[r] : T(0);  // dt (1+c_j)/dl, forward y
    cJb[r] = (j > 0) ? gJ[r] * idl : T(0);       // (1+c_j)/dl, backward y
  }
  T prevHx[2] = {T(0), T(0)}, prevHy[2] = {T(0), T(0)};
  int q = 0;

  auto wait_full = [&](int qa) -> bool {
    const bool r = wait_phase(&full[qa % S], (qa / S) & 1, s_abort);
    __syncwarp();
    return r;
  };
  auto release = [&](int qa) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[qa % S]);
  };
  auto fail = [&]() {
    if (lane == 0) {
      report_status(p.status, DN_ETIMEOUT);
      *s_abort = 1;
    }
  };
  // coefficients of the z (i) roles: per lane for the reference mapping,
  // per plane for the physical one
  auto i_roles = [&](int i, T& hx_c2, T& hy_b, T& hy_c1, T& e_ci, T& bI) {
    if (AXES == DN_AXES_REFERENCE) {
      hx_c2 = dti * gK;
      hy_b = bK;
      hy_c1 = dti * gK;
      e_ci = gK * idl;
      bI = T(1);
    } else {
      bI = static_cast<T>(__ldg(p.b[0] + i));
      const T gI = static_cast<T>(1.0 + __ldg(p.c[0] + i));
      hx_c2 = dti * gI;
      hy_b = bI;
      hy_c1 = dti * gI;
      e_ci = gI * idl;
    }
  };

  // ---- warm-up: new Hx, Hy of plane z0-1 for the owned rows ----------------
  if (z0 > 0) {
    if (!(wait_full(q) && wait_full(q + 1))) {
      fail();
      return;
    }
    T hx_c2, hy_b, hy_c1, e_ci, bI;
    i_roles(z0 - 1, hx_c2, hy_b, hy_c1, e_ci, bI);
    const T* cEx = stage_arr(q, DN_EX);
    const T* cEy = stage_arr(q, DN_EY);
    const T* cEz = stage_arr(q, DN_EZ);
    const T* cHx = stage_arr(q, DN_HX);
    const T* cHy = stage_arr(q, DN_HY);
    const T* nEx = stage_arr(q + 1, DN_EX);
    const T* nEy = stage_arr(q + 1, DN_EY);
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int e = (2 * w + r) * BX + lane + 4;
      const T hy_c2 = AXES == DN_AXES_REFERENCE ? kf * dti * gJ[r] : cKf;
      const T ez = cEz[e];
      prevHx[r - 1] = bJ[r] * cHx[e] - cJf[r] * (cEz[e + BX] - ez) + hx_c2 * (nEy[e] - cEy[e]);
      prevHy[r - 1] = hy_b * cHy[e] - hy_c1 * (nEx[e] - cEx[e]) + hy_c2 * (cEz[e + 1] - ez);
    }
    release(q);
    ++q;
  }

  // ---- march -----------------------------------------------------------------
  for (int i = z0; i < z1; ++i) {
    const bool has_next = (i + 1 < D);
    // plane i was already waited for as "next" unless it is the very first
    if ((i == 0 && !wait_full(q)) || (has_next && !wait_full(q + 1))) {
      fail();
      return;
    }
    T hx_c2, hy_b, hy_c1, e_ci, bI;
    i_roles(i, hx_c2, hy_b, hy_c1, e_ci, bI);
    // this lane's element of row ja-1 in the stage of plane i and of plane i+1
    // (on the last plane the forward z difference is 0: "next" = current);
    // every other access is a compile-time offset from these two pointers
    const T* cur = stage_arr(q, 0) + 2 * w * BX + lane + 4;
    const T* nxt = has_next ? stage_arr(q + 1, 0) + 2 * w * BX + lane + 4 : cur;
    const T* cEx = cur + DN_EX * AE;
    const T* cEy = cur + DN_EY * AE;
    const T* cEz = cur + DN_EZ * AE;
    const T* cHx = cur + DN_HX * AE;
    const T* cHy = cur + DN_HY * AE;
    const T* cHz = cur + DN_HZ * AE;
    const T* cCe = cur + A_CE * AE;
    const T* nEx = nxt + DN_EX * AE;
    const T* nEy = nxt + DN_EY * AE;

    // ---- new H of rows ja-1 (Hx, Hz), ja, ja+1 (all three) at column k ----
    T Hx[3], Hy[3], Hz[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int e = r * BX;
      const T ey = cEy[e], ex = cEx[e], ez = cEz[e];
      Hx[r] = bJ[r] * cHx[e] - cJf[r] * (cEz[e + BX] - ez) + hx_c2 * (nEy[e] - ey);
      Hz[r] = bK * cHz[e] - cKf * (cEy[e + 1] - ey) + cJf[r] * (cEx[e + BX] - ex);
      if (r > 0) {
        const T hy_c2 = AXES == DN_AXES_REFERENCE ? kf * dti * gJ[r] : cKf;
        Hy[r] = hy_b * cHy[e] - hy_c1 * (nEx[e] - ex) + hy_c2 * (cEz[e + 1] - ez);
      } else {
        Hy[r] = T(0);
      }
    }

    // ---- k0-1 halo column of rows ja, ja+1 (lanes 0 and 1) ----------------
    T haloHy = T(0), haloHz = T(0);
    if (lane < 2 && k0 > 0) {
      // lane 0 takes row ja, lane 1 row ja+1 (selected, not indexed, so the
      // coefficient arrays stay in registers)
      const T gJr = lane == 0 ? gJ[1] : gJ[2];
      const T cJfr = lane == 0 ? cJf[1] : cJf[2];
      const int e = (1 + lane) * BX - 1 - lane;  // column k0-1 (pointers sit at k0+lane)
      const T ex = cEx[e], ey = cEy[e], ez = cEz[e];
      const T b = AXES == DN_AXES_REFERENCE ? bKh : bI;
      const T c1 = AXES == DN_AXES_REFERENCE ? dti * gKh : hy_c1;
      const T c2 = AXES == DN_AXES_REFERENCE ? dti * gJr : dti * gKh;
      haloHy = b * cHy[e] - c1 * (nEx[e] - ex) + c2 * (cEz[e + 1] - ez);
      haloHz = bKh * cHz[e] - dti * gKh * (cEy[e + 1] - ey) + cJfr * (cEx[e + BX] - ex);
    }
    const T hHy0 = __shfl_sync(FULL_MASK, haloHy, 0), hHy1 = __shfl_sync(FULL_MASK, haloHy, 1);
    const T hHz0 = __shfl_sync(FULL_MASK, haloHz, 0), hHz1 = __shfl_sync(FULL_MASK, haloHz, 1);

    if (i == 0) {  // the backward z difference is 0 on the first plane
      prevHx[0] = Hx[1];
      prevHx[1] = Hx[2];
      prevHy[0] = Hy[1];
      prevHy[1] = Hy[2];
    }

    // ---- new E of rows ja, ja+1, source, monitors, stores -----------------
    const bool special = any_special(p, i);
    const long long o_plane = i * pz + (long long)ja * py + k;
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int j = ja + r - 1;
      T hyL = __shfl_up_sync(FULL_MASK, Hy[r], 1);
      T hzL = __shfl_up_sync(FULL_MASK, Hz[r], 1);
      if (lane == 0) {
        hyL = r == 1 ? hHy0 : hHy1;
        hzL = r == 1 ? hHz0 : hHz1;
      }
      if (j < H && kin) {
        const int e = r * BX;
        const T ce = cCe[e];
        const T ex_b = AXES == DN_AXES_REFERENCE ? bJ[r] * bK : bJ[r] * bI;
        const T ey_b = AXES == DN_AXES_REFERENCE ? bK * bJ[r] : bI * bK;
        const T ey_c2 = AXES == DN_AXES_REFERENCE ? kb * gJ[r] * idl : cKb;
        T ex = ex_b * cEx[e] + ce * (cJb[r] * (Hz[r] - Hz[r - 1]) - e_ci * (Hy[r] - prevHy[r - 1]));
        T ey = ey_b * cEy[e] + ce * (e_ci * (Hx[r] - prevHx[r - 1]) - ey_c2 * (Hz[r] - hzL));
        T ez = bK * bJ[r] * cEz[e] + ce * (cKb * (Hy[r] - hyL) - cJb[r] * (Hx[r] - Hx[r - 1]));
        T hx = Hx[r], hy = Hy[r], hz = Hz[r];
        if (special) special_cell(p, i, j, k, ex, ey, ez, hx, hy, hz);
        const long long o = o_plane + (r - 1) * py;
        p.out[DN_EX][o] = ex;
        p.out[DN_EY][o] = ey;
        p.out[DN_EZ][o] = ez;
        p.out[DN_HX][o] = hx;
        p.out[DN_HY][o] = hy;
        p.out[DN_HZ][o] = hz;
      }
      prevHx[r - 1] = Hx[r];
      prevHy[r - 1] = Hy[r];
    }
    release(q);
    ++q;
  }
  if (z1 < D) release(q);  // the E-only job of plane z1 was read as "next"
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

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

template <typename T>
int encode(CUtensorMap* m, const void* base, const dn_grid* g) {
  EncodeTiledFn fn = get_encode();
  if (!fn) return DN_ECUDA;
  const cuuint64_t dims[3] = {(cuuint64_t)g->W, (cuuint64_t)g->H, (cuuint64_t)g->D};
  const cuuint64_t strides[2] = {(cuuint64_t)g->pitch_y * sizeof(T),
                                 (cuuint64_t)g->pitch_z * sizeof(T)};
  const cuuint32_t box[3] = {BX, BY, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r =
      fn(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
         3, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_cuda_error(static_cast<int>(r));
    return DN_ECUDA;
  }
  return DN_OK;
}

template <typename T, int AXES>
int launch_all(const StepParams<T>& base, const TmapSet& ta, const TmapSet& tb, void* const fa[6],
               void* const fb[6], int t0, int nsteps, const Plan& plan, int nctas, size_t smem,
               cudaStream_t s) {
  auto kern = k_fdtd3d<T, AXES>;
  DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  StepParams<T> p = base;
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    set_io(&p, even ? fa : fb, even ? fb : fa);
    p.t = t0 + n;
    kern<<<nctas, NT3, smem, s>>>(p, even ? ta : tb, plan);
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

template <typename T>
int run3d(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
          const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons, int32_t n_mon,
          const dn_probe* probe, int32_t t0, int32_t nsteps, int32_t* status, void* stream, int32_t* final_in_b) {
  using C = Cfg<T>;
  StepParams<T> p;
  int rc = build_params<T>(true, g, fa, fb, ce, cpml, src, mons, n_mon, probe, status, &p);
  if (rc != DN_OK) return rc;
  if (t0 < 0 || nsteps < 0 || !final_in_b) return DN_EINVAL;
  // TMA constraints: 16-byte aligned bases and byte strides
  if ((g->pitch_y * (int64_t)sizeof(T)) % 16 || (g->pitch_z * (int64_t)sizeof(T)) % 16)
    return DN_EINVAL;
  for (int c = 0; c < 6; ++c)
    if ((reinterpret_cast<uintptr_t>(fa[c]) | reinterpret_cast<uintptr_t>(fb[c])) & 15)
      return DN_EINVAL;
  if (reinterpret_cast<uintptr_t>(ce) & 15) return DN_EINVAL;

  TmapSet ta, tb;
  for (int c = 0; c < 6; ++c) {
    if ((rc = encode<T>(&ta.m[c], fa[c], g)) != DN_OK) return rc;
    if ((rc = encode<T>(&tb.m[c], fb[c], g)) != DN_OK) return rc;
  }
  if ((rc = encode<T>(&ta.m[A_CE], ce, g)) != DN_OK) return rc;
  tb.m[A_CE] = ta.m[A_CE];

  Plan plan;
  plan.ntx = (g->W + TX - 1) / TX;
  const int nty = (g->H + TY - 1) / TY;
  plan.ntiles = plan.ntx * nty;

  int dev = 0, nsm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  // first guess of the shared-memory need, for the occupancy query
  const size_t fixed = ((size_t)(C::S * C::STAGE_BYTES + C::TAB_BYTES + 15) / 16) * 16 +
                       2 * C::S * sizeof(uint64_t) + 2 * sizeof(int) + 128;
  // as many z ranges per tile as keep every CTA resident at once, each at
  // least MIN_CHUNK planes long
  const long long capacity = (long long)nsm * C::MINB;
  long long nsplit = capacity / plan.ntiles;
  if (nsplit > g->D / MIN_CHUNK) nsplit = g->D / MIN_CHUNK;
  if (nsplit < 1) nsplit = 1;
  plan.nsplit = (int)nsplit;
  const long long nctas = (long long)plan.ntiles * nsplit;
  if (nctas > 0x7fffffffLL) return DN_EUNSUPPORTED;
  plan.maxj = (g->D + nsplit - 1) / nsplit + 2;
  const size_t smem = fixed + (size_t)plan.maxj * sizeof(int2);
  if (smem > 227 * 1024) return DN_EUNSUPPORTED;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g->axes == DN_AXES_REFERENCE)
    rc = launch_all<T, DN_AXES_REFERENCE>(p, ta, tb, fa, fb, t0, nsteps, plan, (int)nctas, smem, s);
  else
    rc = launch_all<T, DN_AXES_PHYSICAL>(p, ta, tb, fa, fb, t0, nsteps, plan, (int)nctas, smem, s);
  if (rc != DN_OK) return rc;
  *final_in_b = nsteps % 2;
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd3d_run(const dn_grid* g, void* const fa[6], void* const fb[6],
                                 const void* ce, const dn_cpml* cpml, const dn_source* src,
                                 const dn_monitor* mons, int32_t n_mon,
                                 const dn_probe* probe, int32_t t0, int32_t nsteps,
                                 int32_t* status, void* stream, int32_t* final_in_b) {
  if (!g) return DN_EINVAL;
  if (g->dtype == DN_F32)
    return dn::run3d<float>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, t0, nsteps, status, stream,
                            final_in_b);
  if (g->dtype == DN_F64)
    return dn::run3d<double>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, t0, nsteps, status, stream,
                             final_in_b);
  return DN_EINVAL;
}
