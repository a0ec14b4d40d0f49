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
//  * a CTA owns a 16 (y) x 32 (x) column of cells and marches along z over a
//    contiguous range of planes; the ranges of all CTAs tile the
//    (tile, plane) space evenly, so the persistent grid is balanced;
//  * each plane's inputs (Ex, Ey, Ez, Hx, Hy, Hz, dt/eps) arrive by 3-D TMA
//    boxes (x from k0-4 so the start is 16-byte aligned, y from j0-1) into a
//    ring of shared-memory stages tracked by mbarriers, several planes ahead;
//  * new H of the plane is computed for the tile plus the one-cell low halo
//    (recomputed, not exchanged) into shared memory; new Hx, Hy of the plane
//    below stay in registers (the z sliding window);
//  * E of the plane is updated from those, the source and the running DFT
//    monitors are applied in registers, and all six results are stored to the
//    other ping-pong buffer (neighbouring CTAs still read the old one).
#include <cuda.h>

#include <mutex>

#include "dn_host.cuh"

namespace dn {
namespace {

constexpr int TX = 32;           // tile x (one warp)
constexpr int TY = 16;           // tile y
constexpr int NT3 = 256;         // 8 warps
constexpr int RW = TY / 8;       // rows per thread
constexpr int BX = TX + 8;       // box x: k0-4 .. k0+TX+3
constexpr int BY = TY + 2;       // box y: j0-1 .. j0+TY
constexpr int NARR = 7;          // Ex Ey Ez Hx Hy Hz ce
constexpr int A_CE = 6;
constexpr int MIN_CHUNK = 8;     // min planes per CTA range
constexpr uint32_t WAIT_PROBES = 1u << 20;  // ~1 s of probing at most

template <typename T>
struct Cfg {
  static constexpr int S = sizeof(T) == 4 ? 4 : 3;  // stages
  static constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
  static constexpr int BOX_BYTES = BX * BY * (int)sizeof(T);
  static constexpr int ARR_BYTES = (BOX_BYTES + 127) / 128 * 128;
  static constexpr int STAGE_BYTES = NARR * ARR_BYTES;
  static constexpr int TX_BYTES = NARR * BOX_BYTES;
  static constexpr int SH_BYTES = 3 * (TY + 1) * (TX + 1) * (int)sizeof(T);
  static constexpr int TAB_BYTES = (2 * (TY + 2) + 2 * (TX + 2)) * (int)sizeof(T);
};

struct alignas(64) TmapSet {
  CUtensorMap m[NARR];
};

// Work split: CTA b owns tile (b % ntiles) for z in [split*D/nsplit,
// (split+1)*D/nsplit), split = b / ntiles.  Consecutive CTAs are neighbouring
// tiles at the same z range, so CTAs that run together march through z in
// lockstep and the halo rows/columns one CTA fetches are L2 hits for its
// neighbours.
struct Plan {
  int ntx;     // tiles along x
  int ntiles;  // tiles per plane
  int nsplit;  // z ranges per tile
  int maxj;    // job-list capacity
};

__device__ __forceinline__ long long fidx(const long long pz, const long long py, int i, int j,
                                          int k) {
  return i * pz + j * py + k;
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
  T* sHx = reinterpret_cast<T*>(smem + S * C::STAGE_BYTES);
  T* sHy = sHx + (TY + 1) * (TX + 1);
  T* sHz = sHy + (TY + 1) * (TX + 1);
  T* sbJ = sHz + (TY + 1) * (TX + 1);
  T* sgJ = sbJ + (TY + 2);
  T* sbK = sgJ + (TY + 2);
  T* sgK = sbK + (TX + 2);
  uint64_t* full = reinterpret_cast<uint64_t*>(
      smem + ((S * C::STAGE_BYTES + C::SH_BYTES + C::TAB_BYTES + 15) / 16) * 16);
  int* s_flags = reinterpret_cast<int*>(full + S);  // [0] job count, [1] failure flag
  int2* jobs = reinterpret_cast<int2*>(s_flags + 2);
  int& s_nj = s_flags[0];
  int& s_fail = s_flags[1];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int D = p.D, H = p.H, W = p.W;
  const long long py = p.py, pz = p.pz;
  const T dt = p.dt, idl = p.inv_dl;
  const int tile = blockIdx.x % plan.ntiles;
  const int split = blockIdx.x / plan.ntiles;
  const int zA = (int)((long long)split * D / plan.nsplit);
  const int zB = (int)((long long)(split + 1) * D / plan.nsplit);

  if (tid == 0) {
    // jobs = planes whose inputs this CTA loads, in consumption order: the
    // warm-up plane zA-1 (new Hx, Hy below the range), zA..zB-1, and plane zB
    // (E only, for the forward differences of plane zB-1)
    int nj = 0;
    if (zA > 0) jobs[nj++] = make_int2(tile, zA - 1);
    for (int z = zA; z < zB; ++z) jobs[nj++] = make_int2(tile, z);
    if (zB < D) jobs[nj++] = make_int2(tile, zB);
    // a previous launch that recorded an error turns this one into a no-op
    const bool skip = p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0;
    s_nj = skip ? 0 : nj;
    s_fail = 0;
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int nj = s_nj;

  auto stage_arr = [&](int q, int a) -> const T* {
    return reinterpret_cast<const T*>(stages + (q % S) * C::STAGE_BYTES + a * C::ARR_BYTES);
  };
  auto issue = [&](int q) {
    const int2 jb = jobs[q];
    const int tyi = jb.x / plan.ntx, txi = jb.x % plan.ntx;
    const int k0 = txi * TX, j0 = tyi * TY;
    uint64_t* bar = &full[q % S];
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, C::TX_BYTES);
    unsigned char* dst = stages + (q % S) * C::STAGE_BYTES;
    for (int a = 0; a < NARR; ++a)
      tma_load_3d(dst + a * C::ARR_BYTES, &tm.m[a], bar, k0 - 4, j0 - 1, jb.y);
  };

  int issued = 0, rel = 0, q = 0;
  if (tid == 0)
    for (; issued < min(nj, S); ++issued) issue(issued);

  // wait for jobs q (and q+1); every thread waits so every thread acquires
  // the TMA writes; any timeout makes the whole CTA leave together.
  auto wait_jobs = [&](int qa, bool two) -> bool {
    bool ok = mbar_wait_bounded(&full[qa % S], (qa / S) & 1, WAIT_PROBES);
    if (two && ok) ok = mbar_wait_bounded(&full[(qa + 1) % S], ((qa + 1) / S) & 1, WAIT_PROBES);
    if (!ok) s_fail = 1;
    __syncthreads();
    if (s_fail) return false;
    if (tid == 0)
      for (; issued < nj && issued < rel + S; ++issued) issue(issued);
    return true;
  };

  bool failed = false;
  do {
    if (nj == 0) break;
    const int t = tile, z0 = zA, z1 = zB;
    const int tyi = t / plan.ntx, txi = t % plan.ntx;
    const int k0 = txi * TX, j0 = tyi * TY;
    const int kk = lane, k = k0 + kk;

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
    // (tables become visible at the next barrier inside wait_jobs)

    T prevHx[RW], prevHy[RW];
#pragma unroll
    for (int r = 0; r < RW; ++r) prevHx[r] = prevHy[r] = T(0);

    // ---- warm-up: new Hx, Hy of plane z0-1 for the owned cells -----------
    if (z0 > 0) {
      if (!wait_jobs(q, true)) {
        failed = true;
        break;
      }
      const int i = z0 - 1;
      T bI = T(1), gI = T(1);
      if (AXES == DN_AXES_PHYSICAL) {
        bI = static_cast<T>(__ldg(p.b[0] + i));
        gI = static_cast<T>(1.0 + __ldg(p.c[0] + i));
      }
      const T* cEx = stage_arr(q, DN_EX);
      const T* cEy = stage_arr(q, DN_EY);
      const T* cEz = stage_arr(q, DN_EZ);
      const T* cHx = stage_arr(q, DN_HX);
      const T* cHy = stage_arr(q, DN_HY);
      const T* nEx = stage_arr(q + 1, DN_EX);
      const T* nEy = stage_arr(q + 1, DN_EY);
#pragma unroll
      for (int r = 0; r < RW; ++r) {
        const int jj = warp + 8 * r, j = j0 + jj;
        if (j >= H || k >= W) continue;
        const int e = (jj + 1) * BX + kk + 4;
        const T bj = sbJ[jj + 1], gj = sgJ[jj + 1], bk = sbK[kk + 1], gk = sgK[kk + 1];
        const T dEz_j = (j < H - 1) ? cEz[e + BX] - cEz[e] : T(0);
        const T dEy_i = nEy[e] - cEy[e];
        const T dEx_i = nEx[e] - cEx[e];
        const T dEz_k = (k < W - 1) ? cEz[e + 1] - cEz[e] : T(0);
        const T hx_g2 = AXES == DN_AXES_REFERENCE ? gk : gI;
        const T hy_b = AXES == DN_AXES_REFERENCE ? bk : bI;
        const T hy_g1 = AXES == DN_AXES_REFERENCE ? gk : gI;
        const T hy_g2 = AXES == DN_AXES_REFERENCE ? gj : gk;
        prevHx[r] = bj * cHx[e] - dt * (gj * (dEz_j * idl) - hx_g2 * (dEy_i * idl));
        prevHy[r] = hy_b * cHy[e] - dt * (hy_g1 * (dEx_i * idl) - hy_g2 * (dEz_k * idl));
      }
      ++rel;
      ++q;
    }

    // ---- march -----------------------------------------------------------
    for (int i = z0; i < z1; ++i) {
      const bool has_next = (i + 1 < D);
      if (!wait_jobs(q, has_next)) {
        failed = true;
        break;
      }
      T bI = T(1), gI = T(1);
      if (AXES == DN_AXES_PHYSICAL) {
        bI = static_cast<T>(__ldg(p.b[0] + i));
        gI = static_cast<T>(1.0 + __ldg(p.c[0] + i));
      }
      const T* cEx = stage_arr(q, DN_EX);
      const T* cEy = stage_arr(q, DN_EY);
      const T* cEz = stage_arr(q, DN_EZ);
      const T* cHx = stage_arr(q, DN_HX);
      const T* cHy = stage_arr(q, DN_HY);
      const T* cHz = stage_arr(q, DN_HZ);
      const T* cCe = stage_arr(q, A_CE);
      const T* nEx = stage_arr(q + 1, DN_EX);
      const T* nEy = stage_arr(q + 1, DN_EY);

      // new H at one cell; `e` is its stage offset, (jt, kt) its table index
      auto h_update = [&](int e, int j, int kx, int jt, int kt, bool want_hx, bool want_hy,
                          bool want_hz, T& hx, T& hy, T& hz) {
        const T bj = sbJ[jt], gj = sgJ[jt], bk = sbK[kt], gk = sgK[kt];
        if (want_hx) {
          const T dEz_j = (j < H - 1) ? cEz[e + BX] - cEz[e] : T(0);
          const T dEy_i = has_next ? nEy[e] - cEy[e] : T(0);
          const T g2 = AXES == DN_AXES_REFERENCE ? gk : gI;
          hx = bj * cHx[e] - dt * (gj * (dEz_j * idl) - g2 * (dEy_i * idl));
        }
        if (want_hy) {
          const T dEx_i = has_next ? nEx[e] - cEx[e] : T(0);
          const T dEz_k = (kx < W - 1) ? cEz[e + 1] - cEz[e] : T(0);
          const T b = AXES == DN_AXES_REFERENCE ? bk : bI;
          const T g1 = AXES == DN_AXES_REFERENCE ? gk : gI;
          const T g2 = AXES == DN_AXES_REFERENCE ? gj : gk;
          hy = b * cHy[e] - dt * (g1 * (dEx_i * idl) - g2 * (dEz_k * idl));
        }
        if (want_hz) {
          const T dEy_k = (kx < W - 1) ? cEy[e + 1] - cEy[e] : T(0);
          const T dEx_j = (j < H - 1) ? cEx[e + BX] - cEx[e] : T(0);
          hz = bk * cHz[e] - dt * (gk * (dEy_k * idl) - gj * (dEx_j * idl));
        }
      };

      // ---- step A: new H of plane i (tile + low halo) -> shared -----------
      T ownHx[RW], ownHy[RW], ownHz[RW];
#pragma unroll
      for (int r = 0; r < RW; ++r) {
        const int jj = warp + 8 * r, j = j0 + jj;
        ownHx[r] = ownHy[r] = ownHz[r] = T(0);
        if (j < H && k < W)
          h_update((jj + 1) * BX + kk + 4, j, k, jj + 1, kk + 1, true, true, true, ownHx[r],
                   ownHy[r], ownHz[r]);
        const int s = (jj + 1) * (TX + 1) + kk + 1;
        sHx[s] = ownHx[r];
        sHy[s] = ownHy[r];
        sHz[s] = ownHz[r];
      }
      if (warp == 0) {  // row halo j0-1: Hx, Hz
        T hx = T(0), hy = T(0), hz = T(0);
        if (j0 > 0 && k < W) h_update(kk + 4, j0 - 1, k, 0, kk + 1, true, false, true, hx, hy, hz);
        sHx[kk + 1] = hx;
        sHz[kk + 1] = hz;
      } else if (warp == 1 && lane < TY) {  // column halo k0-1: Hy, Hz
        const int jj = lane, j = j0 + jj;
        T hx = T(0), hy = T(0), hz = T(0);
        if (k0 > 0 && j < H)
          h_update((jj + 1) * BX + 3, j, k0 - 1, jj + 1, 0, false, true, true, hx, hy, hz);
        sHy[(jj + 1) * (TX + 1)] = hy;
        sHz[(jj + 1) * (TX + 1)] = hz;
      }
      __syncthreads();

      // ---- step B: new E of plane i, source, monitors, stores ------------
      const bool special = any_special(p, i);
#pragma unroll
      for (int r = 0; r < RW; ++r) {
        const int jj = warp + 8 * r, j = j0 + jj;
        if (j < H && k < W) {
          const int e = (jj + 1) * BX + kk + 4;
          const int s = (jj + 1) * (TX + 1) + kk + 1;
          const T bj = sbJ[jj + 1], gj = sgJ[jj + 1], bk = sbK[kk + 1], gk = sgK[kk + 1];
          const T ce = cCe[e];
          const T hx = sHx[s], hy = sHy[s], hz = sHz[s];
          const T dHz_j = (j > 0) ? hz - sHz[s - (TX + 1)] : T(0);
          const T dHy_i = (i > 0) ? hy - prevHy[r] : T(0);
          const T dHx_i = (i > 0) ? hx - prevHx[r] : T(0);
          const T dHz_k = (k > 0) ? hz - sHz[s - 1] : T(0);
          const T dHy_k = (k > 0) ? hy - sHy[s - 1] : T(0);
          const T dHx_j = (j > 0) ? hx - sHx[s - (TX + 1)] : T(0);
          T v[6];
          if (AXES == DN_AXES_REFERENCE) {
            v[DN_EX] = bj * bk * cEx[e] + ce * (gj * (dHz_j * idl) - gk * (dHy_i * idl));
            v[DN_EY] = bk * bj * cEy[e] + ce * (gk * (dHx_i * idl) - gj * (dHz_k * idl));
          } else {
            v[DN_EX] = bj * bI * cEx[e] + ce * (gj * (dHz_j * idl) - gI * (dHy_i * idl));
            v[DN_EY] = bI * bk * cEy[e] + ce * (gI * (dHx_i * idl) - gk * (dHz_k * idl));
          }
          v[DN_EZ] = bk * bj * cEz[e] + ce * (gk * (dHy_k * idl) - gj * (dHx_j * idl));
          v[DN_HX] = hx;
          v[DN_HY] = hy;
          v[DN_HZ] = hz;
          if (special) {
            inject_source(p, i, j, k, v);
            accumulate_monitors(p, i, j, k, v);
            record_probe(p, i, j, k, v);
          }
          const long long o = fidx(pz, py, i, j, k);
#pragma unroll
          for (int a = 0; a < 6; ++a) p.out[a][o] = v[a];
        }
        prevHx[r] = ownHx[r];
        prevHy[r] = ownHy[r];
      }
      ++rel;
      ++q;
    }
    if (failed) break;
    if (z1 < D) {  // the E-only job of plane z1 was consumed as "next"
      ++rel;
      ++q;
    }
  } while (false);

  if (failed) {
    if (tid == 0) {
      report_status(p.status, DN_ETIMEOUT);
      // let copies still in flight land before the CTA's shared memory goes
      for (int qq = q; qq < issued; ++qq)
        (void)mbar_wait_bounded(&full[qq % S], (qq / S) & 1, WAIT_PROBES);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host side
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
  const size_t fixed = ((size_t)(C::S * C::STAGE_BYTES + C::SH_BYTES + C::TAB_BYTES + 15) / 16) *
                           16 +
                       C::S * sizeof(uint64_t) + 2 * sizeof(int) + 128;
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
