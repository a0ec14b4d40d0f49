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
// Design (memory bound, 52 B per cell-step in FP32: 7 arrays read, 6 written),
// on the z-march pipeline of dn_zmarch.cuh:
//  * a producer warp streams each plane's Ex, Ey, Ez, Hx, Hy, Hz and dt/eps
//    into a ring of shared-memory stages with 3-D TMA boxes;
//  * eight consumer warps each own two rows of the 16 x 32 tile and never
//    synchronise with each other: a warp recomputes the new H of the row
//    above its pair (instead of exchanging it), takes the x-1 neighbour by
//    warp shuffle (two lanes compute the k0-1 halo column), keeps new Hx, Hy
//    of the plane below in registers (the z sliding window), updates E,
//    applies the source, DFT monitors and probe in registers, and stores all
//    six results to the other ping-pong buffer (neighbouring CTAs still read
//    the old one);
//  * optionally (adjoint replay) the curl term of each E update is recorded.
// FP32 runs k_fdtd3d_v2 by default: the same march with two columns per lane
// on 16 x 64 tiles (float2 shared-memory reads and global stores, ~30 % fewer
// instructions per cell) in eight-warp CTAs whose stage loads are issued by
// the warp that releases a stage last (two CTAs per SM at 128 registers);
// FP64 and the one-column switch run k_fdtd3d.
#include "dn_zmarch.cuh"

namespace dn {
namespace {

using namespace zm;

constexpr int NRING_F = 7;  // Ex Ey Ez Hx Hy Hz ce
constexpr int A_CE = 6;

// resident CTAs per SM the work split plans for (a build-time override exists for
// measurements of the split; the default is the occupancy the kernel is built for)
#ifndef DN_FWD3D_PLAN_PER_SM
#define DN_FWD3D_PLAN_PER_SM(minb) (minb)
#endif

// ring depth in planes (FP32: two CTAs per SM must fit 228 KB of shared memory)
#ifndef DN_FWD3D_STAGES_F32
#define DN_FWD3D_STAGES_F32 4
#endif

template <typename T>
struct FwdCfg {
  static constexpr int S = sizeof(T) == 4 ? DN_FWD3D_STAGES_F32 : 3;
  static constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
  using L = Layout<T, NRING_F, 0, S>;
};

// curl record for the adjoint replay: curl[c][slot * stride + cell] holds the
// bracket term of the E_c update of step t0 + slot
template <typename T>
struct CurlRec {
  T* curl[3];
  long long stride;
  int t0;
};

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

template <typename T, int AXES, bool REC>
__global__ void __launch_bounds__(NT, FwdCfg<T>::MINB)
    k_fdtd3d(const StepParams<T> p, const __grid_constant__ TmapSet tm, const Plan plan,
             const CurlRec<T> rec) {
  using L = typename FwdCfg<T>::L;
  constexpr int S = L::S;
  constexpr int AE = L::RING_ARR / (int)sizeof(T);  // elements between staged arrays
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const Smem<T, L> sm(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = p.D, H = p.H, W = p.W;
  const long long py = p.py, pz = p.pz;
  const T dt = p.dt, idl = p.inv_dl;
  const Range R(plan, D);
  const int z0 = R.z0, z1 = R.z1, k0 = R.k0, j0 = R.j0;

  const int nj = pipe_setup(sm, R, D, H, W, p.b, p.c, p.status);
  if (nj == 0) return;

  if (warp == NCW) {  // producer warp
    if (lane == 0)
      producer_run<T, L, NRING_F, 0>(sm, tm, R, nj, p.status, [](int) { return 0; });
    return;
  }

  // ======================= consumer warps ===================================
  volatile int* s_abort = sm.flags + 1;
  const int w = warp;
  const int ja = j0 + 2 * w;  // rows ja, ja+1 are owned; row ja-1 is recomputed
  const int k = k0 + lane;
  const bool kin = k < W;
  const T dti = dt * idl;
  // Per-lane coefficients with the boundary rules folded in: a forward
  // difference on the last index and a backward difference on the first one
  // get a zero coefficient.  The neighbour read there is a zero-filled TMA
  // element or an in-range finite value, so 0 * value == 0 exactly.
  const T bK = sm.sbK[lane + 1], gK = sm.sgK[lane + 1];
  const T bKh = sm.sbK[0], gKh = sm.sgK[0];
  const T kf = (k < W - 1) ? T(1) : T(0);
  const T kb = (k > 0) ? T(1) : T(0);
  const T cKf = kf * dti * gK;  // dt (1+c_k)/dl on a forward x difference
  const T cKb = kb * gK * idl;  // (1+c_k)/dl on a backward x difference
  T bJ[3], gJ[3], cJf[3], cJb[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int j = ja + r - 1;
    bJ[r] = sm.sbJ[2 * w + r];
    gJ[r] = sm.sgJ[2 * w + r];
    cJf[r] = (j < H - 1) ? dti * gJ[r] : T(0);  // dt (1+c_j)/dl, forward y
    cJb[r] = (j > 0) ? gJ[r] * idl : T(0);       // (1+c_j)/dl, backward y
  }
  T prevHx[2] = {T(0), T(0)}, prevHy[2] = {T(0), T(0)};
  int q = 0;

  auto wait_full = [&](int qa) -> bool {
    const bool r = wait_phase(&sm.full[qa % S], (qa / S) & 1, s_abort);
    __syncwarp();
    return r;
  };
  auto release = [&](int qa) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[qa % S]);
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
    const T* cur = sm.arr(q, 0) + 2 * w * BX + lane + 4;
    const T* nxt = sm.arr(q + 1, 0) + 2 * w * BX + lane + 4;
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int e = r * BX;
      const T hy_c2 = AXES == DN_AXES_REFERENCE ? kf * dti * gJ[r] : cKf;
      const T ez = cur[DN_EZ * AE + e];
      prevHx[r - 1] = bJ[r] * cur[DN_HX * AE + e] - cJf[r] * (cur[DN_EZ * AE + e + BX] - ez) +
                      hx_c2 * (nxt[DN_EY * AE + e] - cur[DN_EY * AE + e]);
      prevHy[r - 1] = hy_b * cur[DN_HY * AE + e] -
                      hy_c1 * (nxt[DN_EX * AE + e] - cur[DN_EX * AE + e]) +
                      hy_c2 * (cur[DN_EZ * AE + e + 1] - ez);
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
    // this lane's element of row ja-1 in the stage of plane i and of plane
    // i+1 (on the last plane the forward z difference is 0: "next" = current);
    // every other access is a compile-time offset from these two pointers
    const T* cur = sm.arr(q, 0) + 2 * w * BX + lane + 4;
    const T* nxt = has_next ? sm.arr(q + 1, 0) + 2 * w * BX + lane + 4 : cur;
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
        const T curl_x = cJb[r] * (Hz[r] - Hz[r - 1]) - e_ci * (Hy[r] - prevHy[r - 1]);
        const T curl_y = e_ci * (Hx[r] - prevHx[r - 1]) - ey_c2 * (Hz[r] - hzL);
        const T curl_z = cKb * (Hy[r] - hyL) - cJb[r] * (Hx[r] - Hx[r - 1]);
        T ex = ex_b * cEx[e] + ce * curl_x;
        T ey = ey_b * cEy[e] + ce * curl_y;
        T ez = bK * bJ[r] * cEz[e] + ce * curl_z;
        T hx = Hx[r], hy = Hy[r], hz = Hz[r];
        if (special) special_cell(p, i, j, k, ex, ey, ez, hx, hy, hz);
        const long long o = o_plane + (r - 1) * py;
        p.out[DN_EX][o] = ex;
        p.out[DN_EY][o] = ey;
        p.out[DN_EZ][o] = ez;
        p.out[DN_HX][o] = hx;
        p.out[DN_HY][o] = hy;
        p.out[DN_HZ][o] = hz;
        if (REC) {
          const long long oc = (long long)(p.t - rec.t0) * rec.stride + o;
          rec.curl[0][oc] = curl_x;
          rec.curl[1][oc] = curl_y;
          rec.curl[2][oc] = curl_z;
        }
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
// FP32, two columns per lane.  The same march on 16 x 64 tiles: lane l owns
// columns k0+2l and k0+2l+1 of its two rows, reads the staged arrays as
// float2 (one shared-memory instruction for both columns), takes the x+1
// neighbour of its second column with a scalar read and the x-1 neighbour of
// its first column from lane l-1 by shuffle (lanes 0 and 1 recompute the
// k0-1 halo column as above), and writes float2 to global memory.  Per cell
// that halves the shared-memory reads, the global store instructions and the
// halo-column and per-plane overhead; the arithmetic of every column is the
// one-column kernel's, expression for expression.
// ---------------------------------------------------------------------------
constexpr int S_V2 = 3;  // ring depth: two 109 KB CTAs per SM (maximum carveout)
using LV2 = Layout<float, NRING_F, 0, S_V2, Geo64>;

__device__ __forceinline__ float2 ld2(const float* a) {
  return *reinterpret_cast<const float2*>(a);
}
__device__ __forceinline__ float sel(const float2 v, int c) { return c == 0 ? v.x : v.y; }

// store one or both columns (the second one only when it is inside the grid)
__device__ __forceinline__ void st2(float* base, long long o, float a, float b, bool both) {
  if (both)
    *reinterpret_cast<float2*>(base + o) = make_float2(a, b);
  else
    base[o] = a;
}

// eight warps x up to 128 registers: two CTAs per SM (each SM sub-partition
// holds four warps of 128 x 32 registers)
template <int AXES, bool REC>
__global__ void __launch_bounds__(Geo64::NCW * 32, 2)
    k_fdtd3d_v2(const StepParams<float> p, const __grid_constant__ TmapSet tm, const Plan plan,
                const CurlRec<float> rec) {
  using T = float;
  using L = LV2;
  using G = Geo64;
  constexpr int S = L::S;
  constexpr int AE = L::RING_ARR / (int)sizeof(T);
  constexpr int RB = G::BX;  // row stride of a staged box
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const Smem<T, L> sm(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = p.D, H = p.H, W = p.W;
  const long long py = p.py, pz = p.pz;
  const T dt = p.dt, idl = p.inv_dl;
  const Range R(plan, D);
  const int z0 = R.z0, z1 = R.z1, k0 = R.k0, j0 = R.j0;

  const int nj = pipe_setup(sm, R, D, H, W, p.b, p.c, p.status);
  if (nj == 0) return;

  // No separate producer warp (eight warps per CTA keep two CTAs per SM within
  // the register file): lane 0 of warp 0 issues the first S jobs, and the
  // warp that releases job q last issues job q + S into its stage at once.
  auto slot0 = [](int) { return 0; };
  if (warp == 0 && lane == 0) {
    const int n0 = min(S, nj);
    for (int qa = 0; qa < n0; ++qa) issue_job<T, L, NRING_F, 0>(sm, tm, R, qa, slot0);
    atomicMax(&sm.flags[2], n0);
  }

  // ======================= consumer warps ===================================
  volatile int* s_abort = sm.flags + 1;
  const int w = warp;
  const int ja = j0 + 2 * w;      // rows ja, ja+1 are owned; row ja-1 is recomputed
  const int kA = k0 + 2 * lane;   // columns kA (c = 0) and kA+1 (c = 1)
  const bool inA = kA < W, inB = kA + 1 < W;
  const T dti = dt * idl;
  // per-column coefficients, boundary rules folded in (see k_fdtd3d)
  T bK[2], gK[2], kf[2], kb[2], cKf[2], cKb[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int k = kA + c;
    bK[c] = sm.sbK[2 * lane + 1 + c];
    gK[c] = sm.sgK[2 * lane + 1 + c];
    kf[c] = (k < W - 1) ? T(1) : T(0);
    kb[c] = (k > 0) ? T(1) : T(0);
    cKf[c] = kf[c] * dti * gK[c];
    cKb[c] = kb[c] * gK[c] * idl;
  }
  const T bKh = sm.sbK[0], gKh = sm.sgK[0];
  T bJ[3], gJ[3], cJf[3], cJb[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int j = ja + r - 1;
    bJ[r] = sm.sbJ[2 * w + r];
    gJ[r] = sm.sgJ[2 * w + r];
    cJf[r] = (j < H - 1) ? dti * gJ[r] : T(0);
    cJb[r] = (j > 0) ? gJ[r] * idl : T(0);
  }
  T prevHx[2][2] = {{T(0), T(0)}, {T(0), T(0)}};  // [owned row][column]
  T prevHy[2][2] = {{T(0), T(0)}, {T(0), T(0)}};
  int q = 0;

  auto wait_full = [&](int qa) -> bool {
    const bool r = wait_phase(&sm.full[qa % S], (qa / S) & 1, s_abort);
    __syncwarp();
    return r;
  };
  // release job qa: the warp's reads of its stage are ordered before its
  // count; the warp whose count completes the stage's (qa / S + 1)-th use
  // refills it with job qa + S (counts only grow, so no reset races)
  auto release = [&](int qa) {
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      const unsigned prev = atomicAdd(&sm.release[qa % S], 1u);
      if (prev == (unsigned)(G::NCW * (qa / S + 1) - 1) && qa + S < nj) {
        __threadfence_block();
        issue_job<T, L, NRING_F, 0>(sm, tm, R, qa + S, slot0);
        atomicMax(&sm.flags[2], qa + S + 1);
      }
    }
  };
  // on an error every warp waits (bounded) for the copies still in flight
  auto fail = [&]() {
    if (lane == 0) {
      report_status(p.status, DN_ETIMEOUT);
      *s_abort = 1;
      drain_jobs(sm, *reinterpret_cast<volatile int*>(&sm.flags[2]));
    }
  };
  // z (i) roles per column: per lane for the reference mapping, per plane for
  // the physical one
  auto i_roles = [&](int i, T hx_c2[2], T hy_b[2], T hy_c1[2], T e_ci[2], T& bI) {
    if (AXES == DN_AXES_REFERENCE) {
      bI = T(1);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        hx_c2[c] = dti * gK[c];
        hy_b[c] = bK[c];
        hy_c1[c] = dti * gK[c];
        e_ci[c] = gK[c] * idl;
      }
    } else {
      bI = static_cast<T>(__ldg(p.b[0] + i));
      const T gI = static_cast<T>(1.0 + __ldg(p.c[0] + i));
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        hx_c2[c] = dti * gI;
        hy_b[c] = bI;
        hy_c1[c] = dti * gI;
        e_ci[c] = gI * idl;
      }
    }
  };

  // ---- warm-up: new Hx, Hy of plane z0-1 for the owned rows ----------------
  if (z0 > 0) {
    if (!(wait_full(q) && wait_full(q + 1))) {
      fail();
      return;
    }
    T hx_c2[2], hy_b[2], hy_c1[2], e_ci[2], bI;
    i_roles(z0 - 1, hx_c2, hy_b, hy_c1, e_ci, bI);
    const T* cur = sm.arr(q, 0) + 2 * w * RB + 2 * lane + 4;
    const T* nxt = sm.arr(q + 1, 0) + 2 * w * RB + 2 * lane + 4;
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int e = r * RB;
      const float2 ez = ld2(cur + DN_EZ * AE + e), ezj = ld2(cur + DN_EZ * AE + e + RB);
      const float2 ey = ld2(cur + DN_EY * AE + e), ney = ld2(nxt + DN_EY * AE + e);
      const float2 ex = ld2(cur + DN_EX * AE + e), nex = ld2(nxt + DN_EX * AE + e);
      const float2 hx = ld2(cur + DN_HX * AE + e), hy = ld2(cur + DN_HY * AE + e);
      const T ezk2 = cur[DN_EZ * AE + e + 2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const T hy_c2 = AXES == DN_AXES_REFERENCE ? kf[c] * dti * gJ[r] : cKf[c];
        const T ezk = c == 0 ? ez.y : ezk2;
        prevHx[r - 1][c] = bJ[r] * sel(hx, c) - cJf[r] * (sel(ezj, c) - sel(ez, c)) +
                           hx_c2[c] * (sel(ney, c) - sel(ey, c));
        prevHy[r - 1][c] = hy_b[c] * sel(hy, c) - hy_c1[c] * (sel(nex, c) - sel(ex, c)) +
                           hy_c2 * (ezk - sel(ez, c));
      }
    }
    release(q);
    ++q;
  }

  // ---- march -----------------------------------------------------------------
  for (int i = z0; i < z1; ++i) {
    const bool has_next = (i + 1 < D);
    if ((i == 0 && !wait_full(q)) || (has_next && !wait_full(q + 1))) {
      fail();
      return;
    }
    T hx_c2[2], hy_b[2], hy_c1[2], e_ci[2], bI;
    i_roles(i, hx_c2, hy_b, hy_c1, e_ci, bI);
    const T* cur = sm.arr(q, 0) + 2 * w * RB + 2 * lane + 4;
    const T* nxt = has_next ? sm.arr(q + 1, 0) + 2 * w * RB + 2 * lane + 4 : cur;
    const T* cEx = cur + DN_EX * AE;
    const T* cEy = cur + DN_EY * AE;
    const T* cEz = cur + DN_EZ * AE;
    const T* cHx = cur + DN_HX * AE;
    const T* cHy = cur + DN_HY * AE;
    const T* cHz = cur + DN_HZ * AE;
    const T* cCe = cur + A_CE * AE;
    const T* nEx = nxt + DN_EX * AE;
    const T* nEy = nxt + DN_EY * AE;

    // ---- new H of rows ja-1 (Hx, Hz), ja, ja+1 (all three), both columns --
    T Hx[3][2], Hy[3][2], Hz[3][2];
    float2 Ex[3], Ey[3], Ez[3];  // E of rows ja-1 .. ja+1 (reused by the E update)
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int e = r * RB;
      Ex[r] = ld2(cEx + e);
      Ey[r] = ld2(cEy + e);
      Ez[r] = ld2(cEz + e);
      const float2 ezj = ld2(cEz + e + RB), exj = ld2(cEx + e + RB);
      const float2 hx = ld2(cHx + e), hz = ld2(cHz + e), ney = ld2(nEy + e);
      const T eyk2 = cEy[e + 2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const T ex = sel(Ex[r], c), ey = sel(Ey[r], c), ez = sel(Ez[r], c);
        const T eyk = c == 0 ? Ey[r].y : eyk2;
        Hx[r][c] = bJ[r] * sel(hx, c) - cJf[r] * (sel(ezj, c) - ez) +
                   hx_c2[c] * (sel(ney, c) - ey);
        Hz[r][c] = bK[c] * sel(hz, c) - cKf[c] * (eyk - ey) + cJf[r] * (sel(exj, c) - ex);
      }
      if (r > 0) {
        const float2 hy = ld2(cHy + e), nex = ld2(nEx + e);
        const T ezk2 = cEz[e + 2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const T ex = sel(Ex[r], c), ez = sel(Ez[r], c);
          const T ezk = c == 0 ? Ez[r].y : ezk2;
          const T hy_c2 = AXES == DN_AXES_REFERENCE ? kf[c] * dti * gJ[r] : cKf[c];
          Hy[r][c] = hy_b[c] * sel(hy, c) - hy_c1[c] * (sel(nex, c) - ex) + hy_c2 * (ezk - ez);
        }
      } else {
        Hy[r][0] = Hy[r][1] = T(0);
      }
    }

    // ---- k0-1 halo column of rows ja, ja+1 (lanes 0 and 1) ----------------
    T haloHy = T(0), haloHz = T(0);
    if (lane < 2 && k0 > 0) {
      const T gJr = lane == 0 ? gJ[1] : gJ[2];
      const T cJfr = lane == 0 ? cJf[1] : cJf[2];
      const int e = (1 + lane) * RB - 1 - 2 * lane;  // column k0-1 (pointers sit at k0+2*lane)
      const T ex = cEx[e], ey = cEy[e], ez = cEz[e];
      const T b = AXES == DN_AXES_REFERENCE ? bKh : bI;
      const T c1 = AXES == DN_AXES_REFERENCE ? dti * gKh : hy_c1[0];
      const T c2 = AXES == DN_AXES_REFERENCE ? dti * gJr : dti * gKh;
      haloHy = b * cHy[e] - c1 * (nEx[e] - ex) + c2 * (cEz[e + 1] - ez);
      haloHz = bKh * cHz[e] - dti * gKh * (cEy[e + 1] - ey) + cJfr * (cEx[e + RB] - ex);
    }
    const T hHy0 = __shfl_sync(FULL_MASK, haloHy, 0), hHy1 = __shfl_sync(FULL_MASK, haloHy, 1);
    const T hHz0 = __shfl_sync(FULL_MASK, haloHz, 0), hHz1 = __shfl_sync(FULL_MASK, haloHz, 1);

    if (i == 0) {  // the backward z difference is 0 on the first plane
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        prevHx[0][c] = Hx[1][c];
        prevHx[1][c] = Hx[2][c];
        prevHy[0][c] = Hy[1][c];
        prevHy[1][c] = Hy[2][c];
      }
    }

    // ---- new E of rows ja, ja+1, source, monitors, stores -----------------
    const bool special = any_special(p, i);
    const long long o_plane = i * pz + (long long)ja * py + kA;
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int j = ja + r - 1;
      // x-1 neighbours: column kA-1 is lane l-1's second column (the halo on
      // lane 0), column kA is this lane's first
      T hyL[2], hzL[2];
      hyL[0] = __shfl_up_sync(FULL_MASK, Hy[r][1], 1);
      hzL[0] = __shfl_up_sync(FULL_MASK, Hz[r][1], 1);
      if (lane == 0) {
        hyL[0] = r == 1 ? hHy0 : hHy1;
        hzL[0] = r == 1 ? hHz0 : hHz1;
      }
      hyL[1] = Hy[r][0];
      hzL[1] = Hz[r][0];
      if (j < H && inA) {
        const int e = r * RB;
        const float2 ce2 = ld2(cCe + e);
        T nE[3][2], nH[3][2], crl[3][2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const T ce = sel(ce2, c);
          const T ex_b = AXES == DN_AXES_REFERENCE ? bJ[r] * bK[c] : bJ[r] * bI;
          const T ey_b = AXES == DN_AXES_REFERENCE ? bK[c] * bJ[r] : bI * bK[c];
          const T ey_c2 = AXES == DN_AXES_REFERENCE ? kb[c] * gJ[r] * idl : cKb[c];
          const T curl_x =
              cJb[r] * (Hz[r][c] - Hz[r - 1][c]) - e_ci[c] * (Hy[r][c] - prevHy[r - 1][c]);
          const T curl_y =
              e_ci[c] * (Hx[r][c] - prevHx[r - 1][c]) - ey_c2 * (Hz[r][c] - hzL[c]);
          const T curl_z = cKb[c] * (Hy[r][c] - hyL[c]) - cJb[r] * (Hx[r][c] - Hx[r - 1][c]);
          T ex = ex_b * sel(Ex[r], c) + ce * curl_x;
          T ey = ey_b * sel(Ey[r], c) + ce * curl_y;
          T ez = bK[c] * bJ[r] * sel(Ez[r], c) + ce * curl_z;
          T hx = Hx[r][c], hy = Hy[r][c], hz = Hz[r][c];
          if (special) special_cell(p, i, j, kA + c, ex, ey, ez, hx, hy, hz);
          nE[0][c] = ex;
          nE[1][c] = ey;
          nE[2][c] = ez;
          nH[0][c] = hx;
          nH[1][c] = hy;
          nH[2][c] = hz;
          crl[0][c] = curl_x;
          crl[1][c] = curl_y;
          crl[2][c] = curl_z;
        }
        const long long o = o_plane + (r - 1) * py;
        st2(p.out[DN_EX], o, nE[0][0], nE[0][1], inB);
        st2(p.out[DN_EY], o, nE[1][0], nE[1][1], inB);
        st2(p.out[DN_EZ], o, nE[2][0], nE[2][1], inB);
        st2(p.out[DN_HX], o, nH[0][0], nH[0][1], inB);
        st2(p.out[DN_HY], o, nH[1][0], nH[1][1], inB);
        st2(p.out[DN_HZ], o, nH[2][0], nH[2][1], inB);
        if (REC) {
          const long long oc = (long long)(p.t - rec.t0) * rec.stride + o;
          st2(rec.curl[0], oc, crl[0][0], crl[0][1], inB);
          st2(rec.curl[1], oc, crl[1][0], crl[1][1], inB);
          st2(rec.curl[2], oc, crl[2][0], crl[2][1], inB);
        }
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        prevHx[r - 1][c] = Hx[r][c];
        prevHy[r - 1][c] = Hy[r][c];
      }
    }
    release(q);
    ++q;
  }
  if (z1 < D) release(q);  // the E-only job of plane z1 was read as "next"
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <typename T, int AXES, bool REC, bool TWO_COL>
int launch_all(const StepParams<T>& base, const TmapSet& ta, const TmapSet& tb, void* const fa[6],
               void* const fb[6], int t0, int nsteps, const Plan& plan, int nctas, size_t smem,
               const CurlRec<T>& rec, cudaStream_t s) {
  void (*kern)(const StepParams<T>, const TmapSet, const Plan, const CurlRec<T>);
  int nt = NT;
  if constexpr (TWO_COL) {
    kern = k_fdtd3d_v2<AXES, REC>;
    nt = Geo64::NCW * 32;  // eight warps, no separate producer warp
    DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
  } else {
    kern = k_fdtd3d<T, AXES, REC>;
  }
  DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  StepParams<T> p = base;
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    set_io(&p, even ? fa : fb, even ? fb : fa);
    p.t = t0 + n;
    kern<<<nctas, nt, smem, s>>>(p, even ? ta : tb, plan, rec);
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

template <typename T, bool TWO_COL>
int dispatch(const dn_grid* g, bool record, const StepParams<T>& p, const TmapSet& ta,
             const TmapSet& tb, void* const fa[6], void* const fb[6], int t0, int nsteps,
             const Plan& plan, int n, size_t smem, const CurlRec<T>& rec, cudaStream_t s) {
  if (g->axes == DN_AXES_REFERENCE)
    return record ? launch_all<T, DN_AXES_REFERENCE, true, TWO_COL>(p, ta, tb, fa, fb, t0, nsteps,
                                                                    plan, n, smem, rec, s)
                  : launch_all<T, DN_AXES_REFERENCE, false, TWO_COL>(p, ta, tb, fa, fb, t0,
                                                                     nsteps, plan, n, smem, rec, s);
  return record ? launch_all<T, DN_AXES_PHYSICAL, true, TWO_COL>(p, ta, tb, fa, fb, t0, nsteps,
                                                                 plan, n, smem, rec, s)
                : launch_all<T, DN_AXES_PHYSICAL, false, TWO_COL>(p, ta, tb, fa, fb, t0, nsteps,
                                                                  plan, n, smem, rec, s);
}


template <typename T>
int run3d(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
          const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons, int32_t n_mon,
          const dn_probe* probe, const dn_curl_record* crec, int32_t t0, int32_t nsteps,
          int32_t* status, void* stream, int32_t* final_in_b) {
  using L = typename FwdCfg<T>::L;
  StepParams<T> p;
  int rc = build_params<T>(true, g, fa, fb, ce, cpml, src, mons, n_mon, probe, status, &p);
  if (rc != DN_OK) return rc;
  if (t0 < 0 || nsteps < 0 || !final_in_b) return DN_EINVAL;
  if (!steps_ok(src, mons, n_mon, probe, t0, (int64_t)t0 + nsteps)) return DN_EINVAL;
  const void* ptrs[13];
  for (int c = 0; c < 6; ++c) {
    ptrs[c] = fa[c];
    ptrs[6 + c] = fb[c];
  }
  ptrs[12] = ce;
  if (!tma_ok(g, sizeof(T), ptrs, 13)) return DN_EINVAL;

  CurlRec<T> rec{};
  const bool record = crec != nullptr;
  if (record) {
    for (int c = 0; c < 3; ++c) {
      if (!crec->curl[c]) return DN_EINVAL;
      rec.curl[c] = static_cast<T*>(crec->curl[c]);
    }
    if (crec->step_stride < g->pitch_z * (int64_t)g->D || crec->t0 < 0 || t0 < crec->t0 ||
        t0 + nsteps > crec->t0 + crec->nslots)
      return DN_EINVAL;
    rec.stride = crec->step_stride;
    rec.t0 = crec->t0;
  }

  // FP32: two columns per lane (float2 stores need 8-byte aligned curl-record
  // arrays and an even record stride; otherwise the one-column kernel runs)
  bool rec_pairs = !record || rec.stride % 2 == 0;
  for (int c = 0; c < 3 && record; ++c)
    rec_pairs = rec_pairs && (reinterpret_cast<uintptr_t>(rec.curl[c]) & 7) == 0;
  const bool two_col = sizeof(T) == 4 && two_column_fp32() && rec_pairs;
  const int bx = two_col ? Geo64::BX : BX, by = two_col ? Geo64::BY : BY;
  TmapSet ta, tb;
  for (int c = 0; c < 6; ++c) {
    if ((rc = encode_ring(&ta.m[c], fa[c], g, sizeof(T), bx, by)) != DN_OK) return rc;
    if ((rc = encode_ring(&tb.m[c], fb[c], g, sizeof(T), bx, by)) != DN_OK) return rc;
  }
  if ((rc = encode_ring(&ta.m[A_CE], ce, g, sizeof(T), bx, by)) != DN_OK) return rc;
  tb.m[A_CE] = ta.m[A_CE];

  int dev = 0, nsm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  long long nctas = 0;
  const Plan plan =
      two_col ? make_plan(g, (long long)nsm * 2, &nctas, Geo64::TX, Geo64::TY)
              : make_plan(g, (long long)nsm * DN_FWD3D_PLAN_PER_SM(FwdCfg<T>::MINB), &nctas);
  if (nctas > 0x7fffffffLL) return DN_EUNSUPPORTED;
  const size_t smem = two_col ? LV2::BYTES : L::BYTES;
  if (smem > 227 * 1024) return DN_EUNSUPPORTED;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = (int)nctas;
  if constexpr (sizeof(T) == 4) {
    rc = two_col
             ? dispatch<T, true>(g, record, p, ta, tb, fa, fb, t0, nsteps, plan, n, smem, rec, s)
             : dispatch<T, false>(g, record, p, ta, tb, fa, fb, t0, nsteps, plan, n, smem, rec, s);
  } else {
    rc = dispatch<T, false>(g, record, p, ta, tb, fa, fb, t0, nsteps, plan, n, smem, rec, s);
  }
  if (rc != DN_OK) return rc;
  *final_in_b = nsteps % 2;
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd3d_run(const dn_grid* g, void* const fa[6], void* const fb[6],
                                 const void* ce, const dn_cpml* cpml, const dn_source* src,
                                 const dn_monitor* mons, int32_t n_mon, const dn_probe* probe,
                                 const dn_curl_record* rec, int32_t t0, int32_t nsteps,
                                 int32_t* status, void* stream, int32_t* final_in_b) {
  if (!g) return DN_EINVAL;
  if (g->dtype == DN_F32)
    return dn::run3d<float>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, rec, t0, nsteps, status,
                            stream, final_in_b);
  if (g->dtype == DN_F64)
    return dn::run3d<double>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, rec, t0, nsteps,
                             status, stream, final_in_b);
  return DN_EINVAL;
}
