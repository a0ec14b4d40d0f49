// 2-D TMz / TE Yee step for sm_100a: H and E updated in one pass.
//
// Replaces the loop body of DiffNano's FDTDSolver2D._run_steps
// (diffnano/solvers/fdtd2d.py:330-357): _time_step_tm (:233-267) or
// _time_step_te (:269-303) followed by the soft-source add.  Update equations
// (c = 1, cell size dl, row index i on the H axis with profile (b_y, c_y),
// column index j on the W axis with profile (b_x, c_x); forward differences
// are 0 on the last index, backward differences 0 on the first):
//
//   TM  Hx <- b_y[i] Hx - dt (1+c_y[i]) dEz/dj
//       Hy <- b_x[j] Hy + dt (1+c_x[j]) dEz/di
//       Ez <- b_x[j] b_y[i] Ez + (dt/eps) [(1+c_x[j]) dHy/di - (1+c_y[i]) dHx/dj]
//   TE  Ex <- b_x[j] Ex + (dt/eps) (1+c_x[j]) dHz/dj
//       Ey <- b_y[i] Ey - (dt/eps) (1+c_y[i]) dHz/di
//       Hz <- b_x[j] b_y[i] Hz + dt [(1+c_x[j]) dEy/di - (1+c_y[i]) dEx/dj]
//
// Work layout: a warp owns a strip of 32*VEC columns, VEC adjacent columns
// per lane (16-byte loads and stores: VEC = 4 in FP32, 2 in FP64, when the
// rows and arrays are 16-byte aligned; VEC = 1 otherwise), and R consecutive
// rows, which it marches down.  The row neighbours of a cell are carried in
// registers from one row to the next; column neighbours are in the lane's
// own registers or, across a lane boundary, come from the adjacent lane by
// shuffle; the two values a strip needs from outside its columns (TM: Hx at
// column j0-1 and Ez at j0+32*VEC; TE: Hz at j0-1 and Ex at j0+32*VEC) are
// loaded or recomputed by the edge lane with the owner's own arithmetic.
// The intermediate field of the row just above (TM: Hy) or below (TE: Ey,
// Ex) the warp's rows is recomputed the same way, so warps never exchange
// data: no shared memory, no barrier.  A step reads each array once and
// writes each once (28 B per cell in FP32); ping-pong buffers keep other
// warps from seeing this step's writes.  R is chosen by the host so that the
// grid fits one wave of resident CTAs (3 per SM), with a floor that keeps the
// recomputed rows a small share of a warp's loads.
#include <algorithm>
#include <atomic>

#include "dn_host.cuh"
#include "dn_strip.cuh"

namespace dn {
namespace {

constexpr int NT2 = 256;  // threads per CTA: 8 warps stacked along the rows
constexpr int WARPS2 = NT2 / 32;
constexpr unsigned FULL = STRIP_FULL_MASK;

// curl record for the adjoint replay (see dn_curl_record)
template <typename T>
struct CurlRec2 {
  T* curl[3];
  long long stride;
  int t0;
};

// Does row i hold a source, monitor or probe cell?  (A superset test per
// row; the per-cell tests in the helpers decide.  Unrolled over the fixed
// monitor capacity so the parameter array is never indexed at run time.)
template <typename T>
__device__ __forceinline__ bool row_special(const StepParams<T>& p, int i) {
  bool any = p.src.comp >= 0 && i >= p.src.box.lo[1] && i < p.src.box.hi[1];
  any |= p.probe.comp >= 0 && p.probe.pos[1] == i;
#pragma unroll
  for (int m = 0; m < DN_MAX_MONITORS; ++m)
    any |= m < p.n_mon && i >= p.mon[m].box.lo[1] && i < p.mon[m].box.hi[1];
  return any;
}

// Component c of the lane's cell q.  A 2-D cell carries three components
// (TM: Ez, Hx, Hy; TE: Hz, Ex, Ey) held as three named values, never as an
// array indexed by a run-time component id, which would move it to a
// per-thread stack frame.
template <int F, int A, int B, typename T, int VEC>
__device__ __forceinline__ T pick(int c, const Vec<T, VEC>& f, const Vec<T, VEC>& a,
                                  const Vec<T, VEC>& b, int q) {
  return c == F ? f[q] : c == A ? a[q] : c == B ? b[q] : T(0);
}

// Row i holds a source, monitor or probe cell: add the soft source to the
// values about to be stored, accumulate the monitors' running DFTs of those
// values and record the probe.  The monitor accumulators of one frequency are
// all loaded before any is stored, so a lane waits for one memory round trip
// per frequency, not one per cell and frequency.
template <typename T, int POL, int VEC>
__device__ __forceinline__ void special_row(const StepParams<T>& p, int i, int jv,
                                            Vec<T, VEC>& f, Vec<T, VEC>& a, Vec<T, VEC>& b) {
  constexpr int F = (POL == DN_TM) ? DN_EZ : DN_HZ;
  constexpr int A = (POL == DN_TM) ? DN_HX : DN_EX;
  constexpr int B = (POL == DN_TM) ? DN_HY : DN_EY;
  const int W = p.W;
  if (p.src.comp >= 0 && i >= p.src.box.lo[1] && i < p.src.box.hi[1]) {
    const int c = p.src.comp;
    const T w = p.src.wave[p.t];
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      if (jv + q >= W || !p.src.box.contains(0, i, jv + q)) continue;
      if (c == F)
        f[q] += w;
      else if (c == A)
        a[q] += w;
      else if (c == B)
        b[q] += w;
    }
  }
#pragma unroll
  for (int m = 0; m < DN_MAX_MONITORS; ++m) {
    if (m >= p.n_mon) break;
    const MonDev& M = p.mon[m];
    bool in[VEC], any = false;
    long long cell[VEC];
    double x[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      in[q] = jv + q < W && M.box.contains(0, i, jv + q);
      cell[q] = in[q] ? M.box.offset(0, i, jv + q) : 0;
      x[q] = static_cast<double>(pick<F, A, B>(M.comp, f, a, b, q));
      any |= in[q];
    }
    if (!any) continue;
    const double* ph = M.phase + (long long)p.t * M.nf * 2;
    for (int fr = 0; fr < M.nf; ++fr) {
      const double c = ph[2 * fr + 0], s = ph[2 * fr + 1];
      double* base = M.acc + (long long)fr * M.ncell * 2;
      double re[VEC], im[VEC];
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        re[q] = in[q] ? base[cell[q] * 2 + 0] : 0.0;
        im[q] = in[q] ? base[cell[q] * 2 + 1] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        if (!in[q]) continue;
        base[cell[q] * 2 + 0] = fma(x[q], c, re[q]);
        base[cell[q] * 2 + 1] = fma(x[q], s, im[q]);
      }
    }
  }
  if (p.probe.comp >= 0 && p.probe.pos[0] == 0 && p.probe.pos[1] == i) {
#pragma unroll
    for (int q = 0; q < VEC; ++q)
      if (jv + q == p.probe.pos[2] && jv + q < W)
        p.probe.out[p.t] = pick<F, A, B>(p.probe.comp, f, a, b, q);
  }
}

// Store row i's new values for the lane's columns: f = Ez (TM) / Hz (TE),
// a = Hx / Ex, b = Hy / Ey; rows with a source, monitor or probe go through
// special_row first.
template <typename T, int POL, int VEC>
__device__ __forceinline__ void store_row(const StepParams<T>& p, bool special, int i, int jv,
                                          long long o, bool full, Vec<T, VEC> f, Vec<T, VEC> a,
                                          Vec<T, VEC> b) {
  constexpr int F = (POL == DN_TM) ? DN_EZ : DN_HZ;
  constexpr int A = (POL == DN_TM) ? DN_HX : DN_EX;
  constexpr int B = (POL == DN_TM) ? DN_HY : DN_EY;
  const int W = p.W;
  if (special) special_row<T, POL, VEC>(p, i, jv, f, a, b);
  stv(p.out[F], o, f, full, jv, W);
  stv(p.out[A], o, a, full, jv, W);
  stv(p.out[B], o, b, full, jv, W);
}

// Column profile of the lane's columns (1 outside the grid).
template <typename T, int VEC>
__device__ __forceinline__ void column_profile(const StepParams<T>& p, int jv, Vec<T, VEC>& bx,
                                               Vec<T, VEC>& gx) {
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    const int j = jv + q;
    bx[q] = j < p.W ? static_cast<T>(p.b[2][j]) : T(1);
    gx[q] = j < p.W ? static_cast<T>(1.0 + p.c[2][j]) : T(1);
  }
}

// TM: rows [ia, ib) of the strip of columns from j0.
template <typename T, int VEC, bool REC>
__device__ __forceinline__ void march_tm(const StepParams<T>& p, const CurlRec2<T>& rec, int j0,
                                         int ia, int ib) {
  using V = Vec<T, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = p.dt, idl = p.inv_dl;
  const T* Ez = p.in[DN_EZ];
  const T* Hx = p.in[DN_HX];
  const T* Hy = p.in[DN_HY];
  V bx, gx;
  column_profile(p, jv, bx, gx);
  const bool edge_l = lane == 0 && j0 > 0;         // recomputes Hx at column j0-1
  const bool edge_r = lane == 31 && jv + VEC < W;  // loads Ez at column j0+32*VEC

  long long o = (long long)ia * py + jv;
  V ez_c = ldv<T, VEC>(Ez, o, any, full, jv, W);
  // Hy of row ia-1, recomputed with its owner's arithmetic
  V hy_up;
#pragma unroll
  for (int q = 0; q < VEC; ++q) hy_up[q] = T(0);
  if (ia > 0) {
    const V ez_u = ldv<T, VEC>(Ez, o - py, any, full, jv, W);
    const V hy_o = ldv<T, VEC>(Hy, o - py, any, full, jv, W);
#pragma unroll
    for (int q = 0; q < VEC; ++q) hy_up[q] = bx[q] * hy_o[q] + dt * gx[q] * ((ez_c[q] - ez_u[q]) * idl);
  }
  for (int i = ia; i < ib; ++i, o += py) {
    const V ez_n = ldv<T, VEC>(Ez, o + py, any && i + 1 < H, full, jv, W);
    const V hx_o = ldv<T, VEC>(Hx, o, any, full, jv, W);
    const V hy_o = ldv<T, VEC>(Hy, o, any, full, jv, W);
    const V c_e = ldv<T, VEC>(p.ce, o, any, full, jv, W);
    const T ez_r31 = ld(Ez, o + VEC, edge_r);
    const T ez_l0 = ld(Ez, o - 1, edge_l);
    const T hx_l0 = ld(Hx, o - 1, edge_l);
    const T by = static_cast<T>(p.b[1][i]);
    const T gy = static_cast<T>(1.0 + p.c[1][i]);

    T ez_rl = __shfl_down_sync(FULL, ez_c[0], 1);
    if (lane == 31) ez_rl = ez_r31;
    V hx, hy;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T ez_r = (q < VEC - 1) ? ez_c[q < VEC - 1 ? q + 1 : q] : ez_rl;
      const T dj = (j < W - 1) ? ez_r - ez_c[q] : T(0);
      const T di = (i < H - 1) ? ez_n[q] - ez_c[q] : T(0);
      hx[q] = by * hx_o[q] - dt * gy * (dj * idl);
      hy[q] = bx[q] * hy_o[q] + dt * gx[q] * (di * idl);
    }
    T hx_ll = __shfl_up_sync(FULL, hx[VEC - 1], 1);
    if (lane == 0) hx_ll = edge_l ? by * hx_l0 - dt * gy * ((ez_c[0] - ez_l0) * idl) : T(0);
    V ez, cz;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T hx_l = (q > 0) ? hx[q > 0 ? q - 1 : 0] : hx_ll;
      const T dHy = (i > 0) ? hy[q] - hy_up[q] : T(0);
      const T dHx = (j > 0) ? hx[q] - hx_l : T(0);
      cz[q] = gx[q] * (dHy * idl) - gy * (dHx * idl);
      ez[q] = (bx[q] * by) * ez_c[q] + c_e[q] * cz[q];
    }
    const bool sp = row_special(p, i);
    if (any) {
      if (REC) stv(rec.curl[2], (long long)(p.t - rec.t0) * rec.stride + o, cz, full, jv, W);
      store_row<T, DN_TM, VEC>(p, sp, i, jv, o, full, ez, hx, hy);
    }
    hy_up = hy;
    ez_c = ez_n;
  }
}

// TE: rows [ia, ib) of the strip of columns from j0.  E of row i+1 is
// computed in iteration i (Hz of row i needs Ey of row i+1) and carried to
// iteration i+1.
template <typename T, int VEC, bool REC>
__device__ __forceinline__ void march_te(const StepParams<T>& p, const CurlRec2<T>& rec, int j0,
                                         int ia, int ib) {
  using V = Vec<T, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = p.dt, idl = p.inv_dl;
  const T* Hz = p.in[DN_HZ];
  const T* Ex = p.in[DN_EX];
  const T* Ey = p.in[DN_EY];
  V bx, gx;
  column_profile(p, jv, bx, gx);
  const bool edge_l = lane == 0 && j0 > 0;         // loads Hz at column j0-1
  const bool edge_r = lane == 31 && jv + VEC < W;  // recomputes Ex at column j0+32*VEC
  const T bx_r = edge_r ? static_cast<T>(p.b[2][jv + VEC]) : T(1);
  const T gx_r = edge_r ? static_cast<T>(1.0 + p.c[2][jv + VEC]) : T(1);

  // new Ex, Ey of row r (offset oo) from old Hz of rows r (hz) and r-1
  // (hz_u), with the curl terms the adjoint replays; all 32 lanes call it
  auto e_row = [&](int r, long long oo, const V& hz, const V& hz_u, V& ex, V& ey, V& cx, V& cy) {
    const V ex_o = ldv<T, VEC>(Ex, oo, any, full, jv, W);
    const V ey_o = ldv<T, VEC>(Ey, oo, any, full, jv, W);
    const V c_e = ldv<T, VEC>(p.ce, oo, any, full, jv, W);
    const T hz_l0 = ld(Hz, oo - 1, edge_l);
    const T by = static_cast<T>(p.b[1][r]);
    const T gy = static_cast<T>(1.0 + p.c[1][r]);
    T hz_ll = __shfl_up_sync(FULL, hz[VEC - 1], 1);
    if (lane == 0) hz_ll = hz_l0;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T hz_l = (q > 0) ? hz[q > 0 ? q - 1 : 0] : hz_ll;
      const T dj = (j > 0) ? hz[q] - hz_l : T(0);
      const T di = (r > 0) ? hz[q] - hz_u[q] : T(0);
      cx[q] = gx[q] * (dj * idl);
      cy[q] = -(gy * (di * idl));
      ex[q] = bx[q] * ex_o[q] + c_e[q] * cx[q];
      ey[q] = by * ey_o[q] + c_e[q] * cy[q];
    }
  };

  long long o = (long long)ia * py + jv;
  V hz_c = ldv<T, VEC>(Hz, o, any, full, jv, W);
  const V hz_u = ldv<T, VEC>(Hz, o - py, any && ia > 0, full, jv, W);
  V ex_c, ey_c, cx_c, cy_c;
  e_row(ia, o, hz_c, hz_u, ex_c, ey_c, cx_c, cy_c);
  for (int i = ia; i < ib; ++i, o += py) {
    const bool nxt = i + 1 < H;
    const V hz_n = ldv<T, VEC>(Hz, o + py, any && nxt, full, jv, W);
    const T ex_o31 = ld(Ex, o + VEC, edge_r);
    const T ce31 = ld(p.ce, o + VEC, edge_r);
    const T hz31 = ld(Hz, o + VEC, edge_r);
    const T by = static_cast<T>(p.b[1][i]);
    const T gy = static_cast<T>(1.0 + p.c[1][i]);
    V ex_n, ey_n, cx_n, cy_n;
#pragma unroll
    for (int q = 0; q < VEC; ++q) ex_n[q] = ey_n[q] = cx_n[q] = cy_n[q] = T(0);
    if (nxt) e_row(i + 1, o + py, hz_n, hz_c, ex_n, ey_n, cx_n, cy_n);

    T ex_rl = __shfl_down_sync(FULL, ex_c[0], 1);
    if (lane == 31)
      ex_rl = edge_r ? bx_r * ex_o31 + ce31 * (gx_r * ((hz31 - hz_c[VEC - 1]) * idl)) : T(0);
    V hz;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T ex_r = (q < VEC - 1) ? ex_c[q < VEC - 1 ? q + 1 : q] : ex_rl;
      const T dEy = (i < H - 1) ? ey_n[q] - ey_c[q] : T(0);
      const T dEx = (j < W - 1) ? ex_r - ex_c[q] : T(0);
      hz[q] = (bx[q] * by) * hz_c[q] + dt * (gx[q] * (dEy * idl) - gy * (dEx * idl));
    }
    const bool sp = row_special(p, i);
    if (any) {
      if (REC) {
        const long long oc = (long long)(p.t - rec.t0) * rec.stride + o;
        stv(rec.curl[0], oc, cx_c, full, jv, W);
        stv(rec.curl[1], oc, cy_c, full, jv, W);
      }
      store_row<T, DN_TE, VEC>(p, sp, i, jv, o, full, hz, ex_c, ey_c);
    }
    hz_c = hz_n;
    ex_c = ex_n;
    ey_c = ey_n;
    cx_c = cx_n;
    cy_c = cy_n;
  }
}

template <typename T, int POL, bool REC, int VEC>
__global__ void __launch_bounds__(NT2, 3) k_fdtd2d_step(const StepParams<T> p, const CurlRec2<T> rec,
                                                     int R) {
  // a previous launch that recorded an error turns this one into a no-op
  if (p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0) return;
  const int warp = threadIdx.x >> 5;
  const int j0 = blockIdx.x * 32 * VEC;
  const long long ia = ((long long)blockIdx.y * WARPS2 + warp) * R;
  if (ia >= p.H) return;  // whole warp: the shuffles below see all 32 lanes
  const int ib = static_cast<int>(std::min<long long>(ia + R, p.H));
  if (POL == DN_TM)
    march_tm<T, VEC, REC>(p, rec, j0, static_cast<int>(ia), ib);
  else
    march_te<T, VEC, REC>(p, rec, j0, static_cast<int>(ia), ib);
}

// Rows per warp: the smallest R for which the grid of CTAs fits one wave of
// resident CTAs, so that no SM runs a second, partial wave; at least 4 (a
// warp recomputes about three rows of loads above or below its own, so short
// marches spend a large share on them) unless that leaves fewer than 8 warps
// per SM, then at least 2.
template <typename T, int POL, bool REC, int VEC>
int rows_per_warp(int H, int strips, int* R) {
  // per kernel instance, identical on every B200; atomics so that concurrent
  // host threads may fill them (the SM count is published before the
  // per-SM count that readers test)
  static std::atomic<int> per_sm{0}, nsm{0};
  if (per_sm.load(std::memory_order_acquire) == 0) {
    int dev = 0, n = 0, b = 0;
    DN_CUDA_CHECK(cudaGetDevice(&dev));
    DN_CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    DN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &b, k_fdtd2d_step<T, POL, REC, VEC>, NT2, 0));
    nsm.store(n, std::memory_order_relaxed);
    per_sm.store(std::max(b, 1), std::memory_order_release);
  }
  const int q = per_sm.load(std::memory_order_acquire);
  const long long slots = (long long)nsm.load(std::memory_order_relaxed) * q;
  const long long row_ctas = std::max<long long>(1, slots / strips);
  const long long r = (H + WARPS2 * row_ctas - 1) / (WARPS2 * row_ctas);
  const long long warps4 = (long long)strips * ((H + 3) / 4);
  const long long r_min = warps4 >= 8LL * nsm.load(std::memory_order_relaxed) ? 4 : 2;
  *R = static_cast<int>(std::max<long long>(r_min, r));
  return DN_OK;
}

template <typename T, int POL, bool REC, int VEC>
int launch_steps(StepParams<T>& p, const CurlRec2<T>& rec, void* const fa[6], void* const fb[6],
                 int32_t t0, int32_t nsteps, cudaStream_t s) {
  const int strips = (p.W + 32 * VEC - 1) / (32 * VEC);
  int R = 2;
  const int rc = rows_per_warp<T, POL, REC, VEC>(p.H, strips, &R);
  if (rc != DN_OK) return rc;
  const long long rows_per_cta = (long long)WARPS2 * R;
  const dim3 grid(strips, static_cast<unsigned>((p.H + rows_per_cta - 1) / rows_per_cta));
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    set_io(&p, even ? fa : fb, even ? fb : fa);
    p.t = t0 + n;
    k_fdtd2d_step<T, POL, REC, VEC><<<grid, NT2, 0, s>>>(p, rec, R);
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

// 16-byte row access needs the pitch, every array the polarisation uses and
// (when recording) the curl slots and their step stride on 16-byte boundaries.
template <typename T>
bool vector_rows_ok(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
                    const CurlRec2<T>* rec) {
  if ((g->pitch_y * (int64_t)sizeof(T)) % 16 != 0 || !aligned16(ce)) return false;
  const int comps[2][3] = {{DN_EZ, DN_HX, DN_HY}, {DN_HZ, DN_EX, DN_EY}};
  for (int c : comps[g->pol == DN_TM ? 0 : 1])
    if (!aligned16(fa[c]) || !aligned16(fb[c])) return false;
  if (rec) {
    if ((rec->stride * (long long)sizeof(T)) % 16 != 0) return false;
    const int slots[2][2] = {{2, 2}, {0, 1}};
    for (int c : slots[g->pol == DN_TM ? 0 : 1])
      if (!aligned16(rec->curl[c])) return false;
  }
  return true;
}

template <typename T, int POL, bool REC>
int launch_pol(const dn_grid* g, StepParams<T>& p, const CurlRec2<T>& rec, void* const fa[6],
               void* const fb[6], const void* ce, int32_t t0, int32_t nsteps, cudaStream_t s) {
  constexpr int VEC = 16 / static_cast<int>(sizeof(T));
  if (vector_rows_ok<T>(g, fa, fb, ce, REC ? &rec : nullptr))
    return launch_steps<T, POL, REC, VEC>(p, rec, fa, fb, t0, nsteps, s);
  return launch_steps<T, POL, REC, 1>(p, rec, fa, fb, t0, nsteps, s);
}

template <typename T>
int run2d(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
          const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons, int32_t n_mon,
          const dn_probe* probe, const dn_curl_record* crec, int32_t t0, int32_t nsteps,
          int32_t* status, void* stream, int32_t* final_in_b) {
  StepParams<T> p;
  int rc = build_params<T>(false, g, fa, fb, ce, cpml, src, mons, n_mon, probe, status, &p);
  if (rc != DN_OK) return rc;
  if (t0 < 0 || nsteps < 0 || !final_in_b) return DN_EINVAL;
  if (!steps_ok(src, mons, n_mon, probe, t0, (int64_t)t0 + nsteps)) return DN_EINVAL;
  CurlRec2<T> rec{};
  const bool record = crec != nullptr;
  if (record) {
    const bool tm = g->pol == DN_TM;
    if ((tm && !crec->curl[2]) || (!tm && (!crec->curl[0] || !crec->curl[1]))) return DN_EINVAL;
    if (crec->step_stride < (int64_t)g->H * g->pitch_y || crec->t0 < 0 || t0 < crec->t0 ||
        t0 + nsteps > crec->t0 + crec->nslots)
      return DN_EINVAL;
    for (int c = 0; c < 3; ++c) rec.curl[c] = static_cast<T*>(crec->curl[c]);
    rec.stride = crec->step_stride;
    rec.t0 = crec->t0;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (nsteps > 0) {
    if (g->pol == DN_TM)
      rc = record ? launch_pol<T, DN_TM, true>(g, p, rec, fa, fb, ce, t0, nsteps, s)
                  : launch_pol<T, DN_TM, false>(g, p, rec, fa, fb, ce, t0, nsteps, s);
    else
      rc = record ? launch_pol<T, DN_TE, true>(g, p, rec, fa, fb, ce, t0, nsteps, s)
                  : launch_pol<T, DN_TE, false>(g, p, rec, fa, fb, ce, t0, nsteps, s);
    if (rc != DN_OK) return rc;
  }
  *final_in_b = nsteps % 2;
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd2d_run(const dn_grid* g, void* const fa[6], void* const fb[6],
                                 const void* ce, const dn_cpml* cpml, const dn_source* src,
                                 const dn_monitor* mons, int32_t n_mon,
                                 const dn_probe* probe, const dn_curl_record* rec, int32_t t0,
                                 int32_t nsteps, int32_t* status, void* stream,
                                 int32_t* final_in_b) {
  if (!g) return DN_EINVAL;
  if (g->dtype == DN_F32)
    return dn::run2d<float>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, rec, t0, nsteps, status, stream,
                            final_in_b);
  if (g->dtype == DN_F64)
    return dn::run2d<double>(g, fa, fb, ce, cpml, src, mons, n_mon, probe, rec, t0, nsteps, status, stream,
                             final_in_b);
  return DN_EINVAL;
}
