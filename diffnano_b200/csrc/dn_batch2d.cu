// Batched 2-D FDTD: many independent TMz / TE grids in one persistent launch.
//
// The reference runs one FDTDSolver2D object per grid, one Python step loop
// each (diffnano/solvers/fdtd2d.py:309-357).  A design study (robust
// erosion/dilation variants, wavelength sweeps) has many small-to-medium
// grids of different sizes and step counts; launching each step of each grid
// separately is launch-latency bound.  Here one cooperative kernel advances
// all of them:
//
//   for each global step n:                       (forward kernel)
//     every tile of every instance with n < n_steps is stepped
//     (instances are sorted by step count, so the active tiles are a prefix
//     of the tile list and are dealt round-robin to the CTAs);
//     grid barrier (bounded spin, DN_ETIMEOUT)
//
// and the backward kernel walks the checkpoint segments from the last:
// replay of the segment from its checkpoint with the curl record on, then the
// segment's reverse steps (the same transpose as dn_adjoint2d.cu), with the
// monitor-DFT gradient added to the adjoint field as it is loaded.  Field
// loads bypass L1 (other SMs wrote them during the previous step).
//
// Tile: `TI` rows x 32*VEC columns (VEC = 4 in FP32, 2 in FP64), 256 threads:
// each warp marches TI/8 rows of its 32 lanes x VEC columns with 16-byte
// loads and stores, no shared memory (the strip march of dn_fdtd2d.cu /
// dn_adjoint2d.cu: same equations, same boundary rules).
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "dn_host.cuh"
#include "dn_strip.cuh"

// L2 prefetch of the FP64 gradient two rows ahead in the reverse march (1) or
// none (0)
#ifndef DN_BATCH2D_PREFETCH
#define DN_BATCH2D_PREFETCH 1
#endif

namespace dn {
namespace {

// tile columns: 32 lanes x VEC values (16 bytes per lane and array)
inline int tile_cols(int dtype) { return dtype == DN_F32 ? 128 : 64; }
constexpr int NTB = 256;
constexpr unsigned long long BAR_SPIN_LIMIT = 1ull << 24;  // x 64 ns ~ 1 s

struct TableHeader {
  int n_inst;
  int total_tiles;
  int max_steps;
  int K;
  int nseg;
  int tile_rows;
  int pad[2];
  unsigned int bar[4];  // arrive count, generation, abort, unused
};

// table layout (all offsets 16-byte aligned):
//   TableHeader | int tile_prefix[n+1] | int steps[n] (descending) |
//   int2 tile_map[total_tiles] | dn_batch2d_inst inst[n] (sorted)
struct TableView {
  TableHeader* h;
  const int* tile_prefix;
  const int* steps;
  const int2* tile_map;
  const dn_batch2d_inst* inst;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) / 16 * 16; }

__host__ __device__ inline void table_offsets(int n, int total_tiles, size_t* o_prefix,
                                              size_t* o_steps, size_t* o_map, size_t* o_inst,
                                              size_t* o_end) {
  *o_prefix = align16(sizeof(TableHeader));
  *o_steps = align16(*o_prefix + sizeof(int) * (n + 1));
  *o_map = align16(*o_steps + sizeof(int) * n);
  *o_inst = align16(*o_map + sizeof(int2) * (size_t)total_tiles);
  *o_end = align16(*o_inst + sizeof(dn_batch2d_inst) * n);
}

__device__ TableView view(unsigned char* base) {
  TableView v;
  v.h = reinterpret_cast<TableHeader*>(base);
  size_t op, os, om, oi, oe;
  table_offsets(v.h->n_inst, v.h->total_tiles, &op, &os, &om, &oi, &oe);
  v.tile_prefix = reinterpret_cast<const int*>(base + op);
  v.steps = reinterpret_cast<const int*>(base + os);
  v.tile_map = reinterpret_cast<const int2*>(base + om);
  v.inst = reinterpret_cast<const dn_batch2d_inst*>(base + oi);
  return v;
}

// tiles of the instances that still have a step at global step n
__device__ int active_tiles(const TableView& v, int n) {
  int lo = 0, hi = v.h->n_inst;  // first instance with steps <= n
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (v.steps[mid] > n) lo = mid + 1; else hi = mid;
  }
  return v.tile_prefix[lo];
}

// grid barrier over `expected` arrivals (all CTAs of the launch): arrive count
// + generation word, at most `spin_limit` probes 64 ns apart; returns false
// (and raises the abort word) on expiry or when another CTA aborted
__device__ bool grid_sync_n(unsigned int* bar, unsigned int& gen, int* status,
                            unsigned int expected, unsigned long long spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    const unsigned int g = gen;
    if (atomicAdd(&bar[0], 1u) == expected - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicExch(&bar[1], g + 1u);
    } else {
      unsigned long long spins = 0;
      while (*reinterpret_cast<volatile unsigned int*>(&bar[1]) == g) {
        if (*reinterpret_cast<volatile unsigned int*>(&bar[2])) {
          ok = 0;
          break;
        }
        __nanosleep(64);
        if (++spins > spin_limit) {
          ok = 0;
          atomicExch(&bar[2], 1u);
          report_status(status, DN_ETIMEOUT);
          break;
        }
      }
    }
    gen = g + 1u;
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ bool grid_sync(unsigned int* bar, unsigned int& gen, int* status) {
  return grid_sync_n(bar, gen, status, gridDim.x, BAR_SPIN_LIMIT);
}

// The barrier alone, `rounds` times, for dn_batch2d_barrier_selftest: with
// `missing` > 0 arrivals that never come, every CTA's wait runs out.
__global__ void k_barrier_selftest(unsigned int* bar, int* status, unsigned int missing,
                                   unsigned long long spin_limit, int rounds) {
  unsigned int gen = 0;
  for (int r = 0; r < rounds; ++r)
    if (!grid_sync_n(bar, gen, status, gridDim.x + missing, spin_limit)) return;
}

__device__ __forceinline__ bool in_box(const dn_box& b, int i, int j) {
  return i >= b.lo[1] && i < b.hi[1] && j >= b.lo[2] && j < b.hi[2];
}

__device__ __forceinline__ long long box_cell(const dn_box& b, int i, int j) {
  return (long long)(i - b.lo[1]) * (b.hi[2] - b.lo[2]) + (j - b.lo[2]);
}

template <typename T>
struct Sets {
  T* p[3];
};

// ---------------------------------------------------------------------------
// forward step of one warp's strip: rows [ia, ib) of the columns j0 ..
// j0+32*VEC-1 (the single-grid step's march, dn_fdtd2d.cu: row neighbours in
// registers, column neighbours by shuffle, the edge lanes load or recompute
// the value outside the strip, the warp recomputes the intermediate row above
// (TM) or below (TE) its own).  Fields go through L2 only (other CTAs wrote
// them the step before); zero_in: the input is the all-zero state.
// ---------------------------------------------------------------------------
template <typename T, int POL, int VEC, bool RECORD, bool MONITORS>
__device__ void fwd_strip(const dn_batch2d_inst& I, int j0, int ia, int ib, int n,
                          const Sets<T> in, bool zero_in, const Sets<T> out, const Sets<T> ckpt,
                          bool save, const Sets<T> curl) {
  using V = Vec<T, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = I.H, W = I.W;
  const long long py = I.pitch;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = static_cast<T>(I.dt), idl = static_cast<T>(1.0 / I.dl);
  const T* ce = static_cast<const T*>(I.ce);
  const T* F = in.p[0];
  const T* A = in.p[1];
  const T* B = in.p[2];
  V bx, gx;
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    const int j = jv + q;
    bx[q] = j < W ? static_cast<T>(I.b[1][j]) : T(1);
    gx[q] = j < W ? static_cast<T>(1.0 + I.c[1][j]) : T(1);
  }
  const bool edge_l = lane == 0 && j0 > 0;
  const bool edge_r = lane == 31 && jv + VEC < W;
  auto ldf = [&](const T* a, long long o, bool ok) {
    return ldv<T, VEC, LD_CG>(a, o, ok && !zero_in, full, jv, W);
  };
  auto ldf1 = [&](const T* a, long long o, bool ok) {
    return dn::ld<T, LD_CG>(a, o, ok && !zero_in);
  };
  auto ldce = [&](long long o) { return ldv<T, VEC, LD_NC>(ce, o, any, full, jv, W); };

  // source, monitor, stores, checkpoint and curl record of row i
  auto finish = [&](int i, long long o, V& v, const V& a, const V& b, const V& c0, const V& c1) {
    if (!any) return;
    if (I.src_comp >= 0 && i >= I.src_box.lo[1] && i < I.src_box.hi[1]) {
      const T w = static_cast<const T*>(I.wave)[n];
#pragma unroll
      for (int q = 0; q < VEC; ++q)
        if (jv + q < W && in_box(I.src_box, i, jv + q)) v[q] += w;
    }
    if (MONITORS && I.mon_comp >= 0 && i >= I.mon_box.lo[1] && i < I.mon_box.hi[1]) {
      // all accumulators of a frequency are loaded before any is stored
      const long long ncell = (long long)(I.mon_box.hi[1] - I.mon_box.lo[1]) *
                              (I.mon_box.hi[2] - I.mon_box.lo[2]);
      bool inq[VEC];
      long long cell[VEC];
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        inq[q] = jv + q < W && in_box(I.mon_box, i, jv + q);
        cell[q] = inq[q] ? box_cell(I.mon_box, i, jv + q) : 0;
      }
      const double* ph = I.phase + (long long)n * I.n_freq * 2;
      for (int f = 0; f < I.n_freq; ++f) {
        const double cr = ph[2 * f], ci = ph[2 * f + 1];
        double* base = I.acc + (long long)f * ncell * 2;
        double re[VEC], im[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
          re[q] = inq[q] ? __ldcg(base + cell[q] * 2) : 0.0;
          im[q] = inq[q] ? __ldcg(base + cell[q] * 2 + 1) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
          if (!inq[q]) continue;
          const double x = static_cast<double>(v[q]);
          base[cell[q] * 2] = fma(x, cr, re[q]);
          base[cell[q] * 2 + 1] = fma(x, ci, im[q]);
        }
      }
    }
    stv(out.p[0], o, v, full, jv, W);
    stv(out.p[1], o, a, full, jv, W);
    stv(out.p[2], o, b, full, jv, W);
    if (save) {
      stv(ckpt.p[0], o, v, full, jv, W);
      stv(ckpt.p[1], o, a, full, jv, W);
      stv(ckpt.p[2], o, b, full, jv, W);
    }
    if (RECORD) {
      stv(curl.p[0], o, c0, full, jv, W);
      if (POL == DN_TE) stv(curl.p[1], o, c1, full, jv, W);
    }
  };

  long long o = (long long)ia * py + jv;
  if (POL == DN_TM) {
    V f_c = ldf(F, o, any);
    V b_up;  // Hy of row ia-1, recomputed with its owner's arithmetic
#pragma unroll
    for (int q = 0; q < VEC; ++q) b_up[q] = T(0);
    if (ia > 0) {
      const V f_u = ldf(F, o - py, any);
      const V b_o = ldf(B, o - py, any);
#pragma unroll
      for (int q = 0; q < VEC; ++q) b_up[q] = bx[q] * b_o[q] + dt * gx[q] * ((f_c[q] - f_u[q]) * idl);
    }
    for (int i = ia; i < ib; ++i, o += py) {
      const V f_n = ldf(F, o + py, any && i + 1 < H);
      const V a_o = ldf(A, o, any);
      const V b_o = ldf(B, o, any);
      const V c_e = ldce(o);
      const T f_r31 = ldf1(F, o + VEC, edge_r);
      const T f_l0 = ldf1(F, o - 1, edge_l);
      const T a_l0 = ldf1(A, o - 1, edge_l);
      const T by = static_cast<T>(I.b[0][i]);
      const T gy = static_cast<T>(1.0 + I.c[0][i]);
      T f_rl = __shfl_down_sync(STRIP_FULL_MASK, f_c[0], 1);
      if (lane == 31) f_rl = f_r31;
      V a, b;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T f_r = (q < VEC - 1) ? f_c[q < VEC - 1 ? q + 1 : q] : f_rl;
        const T dj = (j < W - 1) ? f_r - f_c[q] : T(0);
        const T di = (i < H - 1) ? f_n[q] - f_c[q] : T(0);
        a[q] = by * a_o[q] - dt * gy * (dj * idl);
        b[q] = bx[q] * b_o[q] + dt * gx[q] * (di * idl);
      }
      T a_ll = __shfl_up_sync(STRIP_FULL_MASK, a[VEC - 1], 1);
      if (lane == 0) a_ll = edge_l ? by * a_l0 - dt * gy * ((f_c[0] - f_l0) * idl) : T(0);
      V v, cz;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T a_l = (q > 0) ? a[q > 0 ? q - 1 : 0] : a_ll;
        const T dHy = (i > 0) ? b[q] - b_up[q] : T(0);
        const T dHx = (j > 0) ? a[q] - a_l : T(0);
        cz[q] = gx[q] * (dHy * idl) - gy * (dHx * idl);
        v[q] = (bx[q] * by) * f_c[q] + c_e[q] * cz[q];
      }
      finish(i, o, v, a, b, cz, cz);
      b_up = b;
      f_c = f_n;
    }
  } else {
    const T bx_r = edge_r ? static_cast<T>(I.b[1][jv + VEC]) : T(1);
    const T gx_r = edge_r ? static_cast<T>(1.0 + I.c[1][jv + VEC]) : T(1);
    // new Ex, Ey of row r from old Hz of rows r (f) and r-1 (f_u), with the
    // curl terms; all 32 lanes call it
    auto e_row = [&](int r, long long oo, const V& f, const V& f_u, V& a, V& b, V& cx, V& cy) {
      const V a_o = ldf(A, oo, any);
      const V b_o = ldf(B, oo, any);
      const V c_e = ldce(oo);
      const T f_l0 = ldf1(F, oo - 1, edge_l);
      const T by = static_cast<T>(I.b[0][r]);
      const T gy = static_cast<T>(1.0 + I.c[0][r]);
      T f_ll = __shfl_up_sync(STRIP_FULL_MASK, f[VEC - 1], 1);
      if (lane == 0) f_ll = f_l0;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T f_l = (q > 0) ? f[q > 0 ? q - 1 : 0] : f_ll;
        const T dj = (j > 0) ? f[q] - f_l : T(0);
        const T di = (r > 0) ? f[q] - f_u[q] : T(0);
        cx[q] = gx[q] * (dj * idl);
        cy[q] = -(gy * (di * idl));
        a[q] = bx[q] * a_o[q] + c_e[q] * cx[q];
        b[q] = by * b_o[q] + c_e[q] * cy[q];
      }
    };
    V f_c = ldf(F, o, any);
    const V f_u = ldf(F, o - py, any && ia > 0);
    V a_c, b_c, cx_c, cy_c;
    e_row(ia, o, f_c, f_u, a_c, b_c, cx_c, cy_c);
    for (int i = ia; i < ib; ++i, o += py) {
      const bool nxt = i + 1 < H;
      const V f_n = ldf(F, o + py, any && nxt);
      const T a_o31 = ldf1(A, o + VEC, edge_r);
      const T ce31 = dn::ld<T, LD_NC>(ce, o + VEC, edge_r);
      const T f31 = ldf1(F, o + VEC, edge_r);
      const T by = static_cast<T>(I.b[0][i]);
      const T gy = static_cast<T>(1.0 + I.c[0][i]);
      V a_n, b_n, cx_n, cy_n;
#pragma unroll
      for (int q = 0; q < VEC; ++q) a_n[q] = b_n[q] = cx_n[q] = cy_n[q] = T(0);
      if (nxt) e_row(i + 1, o + py, f_n, f_c, a_n, b_n, cx_n, cy_n);
      T a_rl = __shfl_down_sync(STRIP_FULL_MASK, a_c[0], 1);
      if (lane == 31)
        a_rl = edge_r ? bx_r * a_o31 + ce31 * (gx_r * ((f31 - f_c[VEC - 1]) * idl)) : T(0);
      V v;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T a_r = (q < VEC - 1) ? a_c[q < VEC - 1 ? q + 1 : q] : a_rl;
        const T dEy = (i < H - 1) ? b_n[q] - b_c[q] : T(0);
        const T dEx = (j < W - 1) ? a_r - a_c[q] : T(0);
        v[q] = (bx[q] * by) * f_c[q] + dt * (gx[q] * (dEy * idl) - gy * (dEx * idl));
      }
      finish(i, o, v, a_c, b_c, cx_c, cy_c);
      f_c = f_n;
      a_c = a_n;
      b_c = b_n;
      cx_c = cx_n;
      cy_c = cy_n;
    }
  }
}

// monitor-DFT gradient added to the adjoint field at (i, j) for step n
template <typename T>
__device__ __forceinline__ T mon_inject(const dn_batch2d_inst& I, int i, int j, int n) {
  if (!I.gmon || I.mon_comp < 0 || !in_box(I.mon_box, i, j)) return T(0);
  const long long cell = box_cell(I.mon_box, i, j);
  const long long ncell =
      (long long)(I.mon_box.hi[1] - I.mon_box.lo[1]) * (I.mon_box.hi[2] - I.mon_box.lo[2]);
  const double* ph = I.phase + (long long)n * I.n_freq * 2;
  double g = 0.0;
  for (int f = 0; f < I.n_freq; ++f) {
    const double* a = I.gmon + ((long long)f * ncell + cell) * 2;
    g = fma(a[0], ph[2 * f], fma(a[1], ph[2 * f + 1], g));
  }
  return static_cast<T>(g);
}

// ---------------------------------------------------------------------------
// reverse step of one warp's strip (transpose of fwd_strip; the single-grid
// reverse march of dn_adjoint2d.cu).  Every load of lambda_F (TM: Ez, TE: Hz)
// has the monitor-DFT gradient of step n added.  Adjoint fields and curl
// records go through L2 only; the FP64 gradient is read the same way.
// ---------------------------------------------------------------------------
template <typename T, int POL, int VEC>
__device__ void adj_strip(const dn_batch2d_inst& I, int j0, int ia, int ib, int n,
                          const Sets<T> lin, const Sets<T> lout, const Sets<T> curl) {
  using V = Vec<T, VEC>;
  using D = Vec<double, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = I.H, W = I.W;
  const long long py = I.pitch;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = static_cast<T>(I.dt), idl = static_cast<T>(1.0 / I.dl);
  const T* ce = static_cast<const T*>(I.ce);
  const T* L0 = lin.p[0];
  const T* L1 = lin.p[1];
  const T* L2 = lin.p[2];
  const bool inject = I.gmon != nullptr && I.mon_comp >= 0;
  auto ldl = [&](const T* a, long long o, bool ok) { return ldv<T, VEC, LD_CG>(a, o, ok, full, jv, W); };
  auto ldl1 = [&](const T* a, long long o, bool ok) { return dn::ld<T, LD_CG>(a, o, ok); };
  auto ldce = [&](long long o) { return ldv<T, VEC, LD_NC>(ce, o, any, full, jv, W); };
  // lambda_F of row r with the monitor gradient of step n added
  auto ldl0 = [&](int r, long long o, bool ok) {
    V l = ldl(L0, o, ok);
    if (inject && ok && r >= I.mon_box.lo[1] && r < I.mon_box.hi[1]) {
#pragma unroll
      for (int q = 0; q < VEC; ++q)
        if (jv + q < W) l[q] += mon_inject<T>(I, r, jv + q, n);
    }
    return l;
  };
  auto ldl0_1 = [&](int r, int j, long long o, bool ok) {
    T l = ldl1(L0, o, ok);
    if (ok) l += mon_inject<T>(I, r, j, n);
    return l;
  };
  auto add_grad = [&](long long o, const V& x0, const V& c0, const V& x1, const V& c1, bool two) {
    D g = ldv<double, VEC, LD_CG>(I.grad, o, any, full, jv, W);
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      if (two)
        g[q] += static_cast<double>(x0[q]) * static_cast<double>(c0[q]) +
                static_cast<double>(x1[q]) * static_cast<double>(c1[q]);
      else
        g[q] += static_cast<double>(x0[q]) * static_cast<double>(c0[q]);
    }
    stv(I.grad, o, g, full, jv, W);
  };

  long long o = (long long)ia * py + jv;
  if (POL == DN_TM) {
    V bx, gx;  // gx = (1 + c_x) / dl
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      bx[q] = j < W ? static_cast<T>(I.b[1][j]) : T(1);
      gx[q] = (j < W ? static_cast<T>(1.0 + I.c[1][j]) : T(1)) * idl;
    }
    const bool edge_l = lane == 0 && j0 > 0;         // recomputes vx at column j0-1
    const bool edge_r = lane == 31 && jv + VEC < W;  // loads u at column j0+32*VEC
    V l_c = ldl0(ia, o, any);
    V u_c;
    {
      const V c_e = ldce(o);
#pragma unroll
      for (int q = 0; q < VEC; ++q) u_c[q] = c_e[q] * l_c[q];
    }
    V vy_up;  // vy of row ia-1 (row ia-1 < H-1)
#pragma unroll
    for (int q = 0; q < VEC; ++q) vy_up[q] = T(0);
    if (ia > 0) {
      const V l_u = ldl0(ia - 1, o - py, any);
      const V c_u = ldce(o - py);
      const V l2_u = ldl(L2, o - py, any);
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const T uu = c_u[q] * l_u[q];
        const T lh = l2_u[q] + gx[q] * ((ia - 1 > 0 ? uu : T(0)) - u_c[q]);
        vy_up[q] = dt * gx[q] * lh;
      }
    }
    for (int i = ia; i < ib; ++i, o += py) {
      const bool nxt = i + 1 < H;
#if DN_BATCH2D_PREFETCH
      // the FP64 gradient row two ahead into L2 (its read-modify-write comes
      // at the end of a row and would otherwise wait for DRAM)
      if (any && i + 2 < ib) prefetch_l2(I.grad + o + 2 * py);
#endif
      const V l_n = ldl0(i + 1, o + py, any && nxt);
      const V c_n = ldv<T, VEC, LD_NC>(ce, o + py, any && nxt, full, jv, W);
      const V l1 = ldl(L1, o, any);
      const V l2 = ldl(L2, o, any);
      const V crl = ldl(curl.p[0], o, any);
      const T c_r31 = dn::ld<T, LD_NC>(ce, o + VEC, edge_r);
      const T l_r31 = ldl0_1(i, jv + VEC, o + VEC, edge_r);
      const T c_l0 = dn::ld<T, LD_NC>(ce, o - 1, edge_l);
      const T l_l0 = ldl0_1(i, j0 - 1, o - 1, edge_l);
      const T l1_l0 = ldl1(L1, o - 1, edge_l);
      const T by = static_cast<T>(I.b[0][i]);
      const T gy = static_cast<T>(1.0 + I.c[0][i]) * idl;
      V u_n;
#pragma unroll
      for (int q = 0; q < VEC; ++q) u_n[q] = c_n[q] * l_n[q];
      T u_rl = __shfl_down_sync(STRIP_FULL_MASK, u_c[0], 1);
      if (lane == 31) u_rl = c_r31 * l_r31;
      V a, b, vx, vy;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T u_r = (q < VEC - 1) ? u_c[q < VEC - 1 ? q + 1 : q] : u_rl;
        a[q] = l1[q] - gy * ((j > 0 ? u_c[q] : T(0)) - u_r);
        b[q] = l2[q] + gx[q] * ((i > 0 ? u_c[q] : T(0)) - u_n[q]);
        vx[q] = (j < W - 1) ? dt * gy * a[q] : T(0);
        vy[q] = (i < H - 1) ? dt * gx[q] * b[q] : T(0);
      }
      T vx_ll = __shfl_up_sync(STRIP_FULL_MASK, vx[VEC - 1], 1);
      if (lane == 0) {
        T v = T(0);
        if (edge_l) {  // column j0-1 < W-1
          const T ul = c_l0 * l_l0;
          const T lh = l1_l0 - gy * ((j0 - 1 > 0 ? ul : T(0)) - u_c[0]);
          v = dt * gy * lh;
        }
        vx_ll = v;
      }
      V o0, o1, o2;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const T vx_l = (q > 0) ? vx[q > 0 ? q - 1 : 0] : vx_ll;
        o0[q] = bx[q] * by * l_c[q] + (vx[q] - vx_l) - (vy[q] - vy_up[q]);
        o1[q] = by * a[q];
        o2[q] = bx[q] * b[q];
      }
      if (any) {
        add_grad(o, l_c, crl, l_c, crl, false);
        stv(lout.p[0], o, o0, full, jv, W);
        stv(lout.p[1], o, o1, full, jv, W);
        stv(lout.p[2], o, o2, full, jv, W);
      }
      vy_up = vy;
      u_c = u_n;
      l_c = l_n;
    }
  } else {
    V bx, gxr, cx;  // gxr = 1 + c_x, cx = dt (1 + c_x) / dl
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      bx[q] = j < W ? static_cast<T>(I.b[1][j]) : T(1);
      gxr[q] = j < W ? static_cast<T>(1.0 + I.c[1][j]) : T(1);
      cx[q] = dt * gxr[q] * idl;
    }
    const bool edge_l = lane == 0 && j0 > 0;         // loads lambda_Hz at column j0-1
    const bool edge_r = lane == 31 && jv + VEC < W;  // recomputes ux at column j0+32*VEC
    const T gxr_r = edge_r ? static_cast<T>(1.0 + I.c[1][jv + VEC]) : T(1);
    // E-adjoint half of row r from lambda_Hz of rows r (lh) and r-1 (lh_u);
    // the row's gradient when `own`; all 32 lanes call it
    auto e_row = [&](int r, long long oo, const V& lh, const V& lh_u, bool own, V& a, V& b, V& ux,
                     V& uy) {
      const V l1 = ldl(L1, oo, any);
      const V l2 = ldl(L2, oo, any);
      const V c_e = ldce(oo);
      const T lh_l0 = ldl0_1(r, j0 - 1, oo - 1, edge_l);
      const T gyr = static_cast<T>(1.0 + I.c[0][r]);
      const T cy = dt * gyr * idl;
      T lh_ll = __shfl_up_sync(STRIP_FULL_MASK, lh[VEC - 1], 1);
      if (lane == 0) lh_ll = lh_l0;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const int j = jv + q;
        const T lh_l = (q > 0) ? lh[q > 0 ? q - 1 : 0] : lh_ll;
        const T wj = (j < W - 1) ? cy * lh[q] : T(0);
        const T wjm = (j > 0) ? cy * lh_l : T(0);
        const T wi = (r < H - 1) ? cx[q] * lh[q] : T(0);
        const T wim = (r > 0) ? cx[q] * lh_u[q] : T(0);
        a[q] = l1[q] + wj - wjm;
        b[q] = l2[q] - wi + wim;
        ux[q] = (j > 0) ? c_e[q] * gxr[q] * idl * a[q] : T(0);
        uy[q] = (r > 0) ? c_e[q] * gyr * idl * b[q] : T(0);
      }
      if (own && any) {
        const V c0 = ldl(curl.p[0], oo, any);
        const V c1 = ldl(curl.p[1], oo, any);
        add_grad(oo, a, c0, b, c1, true);
      }
    };
    V lh_c = ldl0(ia, o, any);
    const V lh_u = ldl0(ia - 1, o - py, any && ia > 0);
    V a_c, b_c, ux_c, uy_c;
    e_row(ia, o, lh_c, lh_u, true, a_c, b_c, ux_c, uy_c);
    for (int i = ia; i < ib; ++i, o += py) {
      const bool nxt = i + 1 < H;
#if DN_BATCH2D_PREFETCH
      if (any && i + 2 < ib) prefetch_l2(I.grad + o + 2 * py);  // as in the TM march
#endif
      const V lh_n = ldl0(i + 1, o + py, any && nxt);
      const T l1_31 = ldl1(L1, o + VEC, edge_r);
      const T c31 = dn::ld<T, LD_NC>(ce, o + VEC, edge_r);
      const T lh31 = ldl0_1(i, jv + VEC, o + VEC, edge_r);
      const T by = static_cast<T>(I.b[0][i]);
      const T cy = dt * static_cast<T>(1.0 + I.c[0][i]) * idl;
      V a_n, b_n, ux_n, uy_n;
#pragma unroll
      for (int q = 0; q < VEC; ++q) a_n[q] = b_n[q] = ux_n[q] = uy_n[q] = T(0);
      if (nxt) e_row(i + 1, o + py, lh_n, lh_c, i + 1 < ib, a_n, b_n, ux_n, uy_n);
      T ux_rl = __shfl_down_sync(STRIP_FULL_MASK, ux_c[0], 1);
      if (lane == 31) {
        T v = T(0);
        if (edge_r) {  // column jh = j0+32*VEC > 0
          const T wj = (jv + VEC < W - 1) ? cy * lh31 : T(0);
          const T wjm = cy * lh_c[VEC - 1];
          const T lex = l1_31 + wj - wjm;
          v = c31 * gxr_r * idl * lex;
        }
        ux_rl = v;
      }
      V o0, o1, o2;
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        const T ux_r = (q < VEC - 1) ? ux_c[q < VEC - 1 ? q + 1 : q] : ux_rl;
        o0[q] = bx[q] * by * lh_c[q] + (ux_c[q] - ux_r) - (uy_c[q] - uy_n[q]);
        o1[q] = bx[q] * a_c[q];
        o2[q] = by * b_c[q];
      }
      if (any) {
        stv(lout.p[0], o, o0, full, jv, W);
        stv(lout.p[1], o, o1, full, jv, W);
        stv(lout.p[2], o, o2, full, jv, W);
      }
      lh_c = lh_n;
      a_c = a_n;
      b_c = b_n;
      ux_c = ux_n;
      uy_c = uy_n;
    }
  }
}

template <typename T>
__device__ __forceinline__ Sets<T> field_set(void* const f[3]) {
  return Sets<T>{{static_cast<T*>(f[0]), static_cast<T*>(f[1]), static_cast<T*>(f[2])}};
}

template <typename T>
__device__ __forceinline__ Sets<T> slot_set(void* base, long long slot, long long field_elems,
                                            int nfields) {
  Sets<T> s{{nullptr, nullptr, nullptr}};
  T* b = static_cast<T*>(base) + slot * nfields * field_elems;
  for (int c = 0; c < nfields; ++c) s.p[c] = b + c * field_elems;
  return s;
}

// Warp `threadIdx.x / 32`'s share of tile q of instance I: the tile is TI
// rows x 32*VEC columns, each of the CTA's 8 warps marches TI/8 of its rows.
struct StripTask {
  int j0, ia, ib;
};

template <int VEC, int TI>
__device__ __forceinline__ StripTask strip_of(const dn_batch2d_inst& I, int q) {
  const int ntx = (I.W + 32 * VEC - 1) / (32 * VEC);
  const int ty = q / ntx, tx = q % ntx;
  constexpr int R = TI / (NTB / 32);
  StripTask st;
  st.j0 = tx * 32 * VEC;
  st.ia = ty * TI + (threadIdx.x >> 5) * R;
  st.ib = min(st.ia + R, I.H);
  return st;
}

template <typename T, int POL, int TI>
__global__ void __launch_bounds__(NTB, 2) k_batch2d_fwd(unsigned char* table, int* status) {
  constexpr int VEC = 16 / static_cast<int>(sizeof(T));
  const TableView v = view(table);
  __shared__ unsigned int s_gen;
  if (threadIdx.x == 0) s_gen = *reinterpret_cast<volatile unsigned int*>(&v.h->bar[1]);
  __syncthreads();
  unsigned int gen = s_gen;
  const int K = v.h->K;
  for (int n = 0; n < v.h->max_steps; ++n) {
    const int nt = active_tiles(v, n);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
      const int2 m = v.tile_map[t];
      const dn_batch2d_inst& I = v.inst[m.x];
      const StripTask st = strip_of<VEC, TI>(I, m.y);
      if (st.ia >= I.H) continue;  // whole warp: the shuffles see all 32 lanes
      const Sets<T> in = field_set<T>(I.f[n & 1]);
      const Sets<T> out = field_set<T>(I.f[(n + 1) & 1]);
      Sets<T> ck{{nullptr, nullptr, nullptr}};
      const bool save = I.ckpt != nullptr && K > 0 && (n + 1) % K == 0 && (n + 1) < I.n_steps;
      if (save) ck = slot_set<T>(I.ckpt, (n + 1) / K - 1, (long long)I.H * I.pitch, 3);
      fwd_strip<T, POL, VEC, false, true>(I, st.j0, st.ia, st.ib, n, in, false, out, ck, save,
                                          ck);
    }
    if (!grid_sync(v.h->bar, gen, status)) return;
  }
}

template <typename T, int POL, int TI>
__global__ void __launch_bounds__(NTB, 2) k_batch2d_bwd(unsigned char* table, int* status) {
  constexpr int VEC = 16 / static_cast<int>(sizeof(T));
  const TableView v = view(table);
  __shared__ unsigned int s_gen;
  if (threadIdx.x == 0) s_gen = *reinterpret_cast<volatile unsigned int*>(&v.h->bar[1]);
  __syncthreads();
  unsigned int gen = s_gen;
  const int K = v.h->K;
  constexpr int NCURL = POL == DN_TM ? 1 : 2;
  for (int g = v.h->nseg - 1; g >= 0; --g) {
    const int ta = g * K, tb = min(v.h->max_steps, ta + K);
    // replay steps ta..tb-1 from the checkpoint at ta, curls recorded
    for (int n = ta; n < tb; ++n) {
      const int nt = active_tiles(v, n);
      for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 m = v.tile_map[t];
        const dn_batch2d_inst& I = v.inst[m.x];
        const StripTask st = strip_of<VEC, TI>(I, m.y);
        if (st.ia >= I.H) continue;
        const long long fe = (long long)I.H * I.pitch;
        const bool zero_in = n == ta && g == 0;
        const Sets<T> in = n == ta ? (g == 0 ? field_set<T>(I.f[0]) : slot_set<T>(I.ckpt, g - 1, fe, 3))
                                   : field_set<T>(I.f[n & 1]);
        const Sets<T> out = field_set<T>(I.f[(n + 1) & 1]);
        const Sets<T> cr = slot_set<T>(I.curl, n - ta, fe, NCURL);
        fwd_strip<T, POL, VEC, true, false>(I, st.j0, st.ia, st.ib, n, in, zero_in, out, out,
                                            false, cr);
      }
      if (!grid_sync(v.h->bar, gen, status)) return;
    }
    // reverse steps tb-1 .. ta
    for (int n = tb - 1; n >= ta; --n) {
      const int nt = active_tiles(v, n);
      for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 m = v.tile_map[t];
        const dn_batch2d_inst& I = v.inst[m.x];
        const StripTask st = strip_of<VEC, TI>(I, m.y);
        if (st.ia >= I.H) continue;
        const long long fe = (long long)I.H * I.pitch;
        const Sets<T> lin = field_set<T>(I.lam[(n + 1) & 1]);
        const Sets<T> lout = field_set<T>(I.lam[n & 1]);
        const Sets<T> cr = slot_set<T>(I.curl, n - ta, fe, NCURL);
        adj_strip<T, POL, VEC>(I, st.j0, st.ia, st.ib, n, lin, lout, cr);
      }
      if (!grid_sync(v.h->bar, gen, status)) return;
    }
  }
}

// ---------------------------------------------------------------------------
// forward-only solve with every grid held in one thread-block cluster
// ---------------------------------------------------------------------------
// Cluster c (CL CTAs) solves instance c of the table.  CTA r of the cluster
// owns rows [r*rows, r*rows + rows) of the grid (rows = ceil(H/CL)) and keeps
// the three fields and dt/eps of its band in shared memory for the whole run;
// the one neighbouring row each half-step needs is read from the next or
// previous CTA's shared memory (distributed shared memory), and two cluster
// barriers per step order the half-steps.  Every CTA of a cluster runs the same
// instance's step count, so the barrier sequence is identical on all of them.
// The arithmetic is fwd_strip's, expression for expression.
namespace cg = cooperative_groups;

template <typename T>
struct Band {
  T* f;   // injected field (Ez / Hz)   rows x W
  T* a;   // Hx / Ex
  T* b;   // Hy / Ey
  T* ce;  // dt / eps
  T* bx;  // W
  T* gx;  // W
  T* by;  // rows
  T* gy;  // rows
};

__host__ __device__ inline long long band_elems(long long rows, long long W) {
  return 4 * rows * W + 2 * W + 2 * rows;
}

template <typename T>
__device__ __forceinline__ Band<T> band_layout(unsigned char* smem, int rows, int W) {
  Band<T> s;
  T* p = reinterpret_cast<T*>(smem);
  const long long n = (long long)rows * W;
  s.f = p;
  s.a = p + n;
  s.b = p + 2 * n;
  s.ce = p + 3 * n;
  s.bx = p + 4 * n;
  s.gx = s.bx + W;
  s.by = s.gx + W;
  s.gy = s.by + rows;
  return s;
}

template <typename T, int POL, int CL>
__global__ void __launch_bounds__(512, 1) k_batch2d_cluster(unsigned char* table) {
  extern __shared__ __align__(16) unsigned char c_smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const TableView v = view(table);
  // the instance's fields in registers: the monitor stores below go to global
  // memory and would otherwise force re-reads of the descriptor
  const dn_batch2d_inst* Ip = v.inst + blockIdx.x / CL;
  const int H = Ip->H, W = Ip->W, T_steps = Ip->n_steps;
  const long long py = Ip->pitch;
  const T dt = static_cast<T>(Ip->dt), idl = static_cast<T>(1.0 / Ip->dl);
  const bool src = Ip->src_comp >= 0, mon = Ip->mon_comp >= 0;
  const dn_box sb = Ip->src_box, mb = Ip->mon_box;
  const int nfq = Ip->n_freq;
  const double* __restrict__ phase = Ip->phase;
  double* __restrict__ accb = Ip->acc;
  const T* __restrict__ wave = static_cast<const T*>(Ip->wave);
  const double* pb0 = Ip->b[0];
  const double* pb1 = Ip->b[1];
  const double* pc0 = Ip->c[0];
  const double* pc1 = Ip->c[1];
  const T* __restrict__ ceg = static_cast<const T*>(Ip->ce);
  T* const* outp = reinterpret_cast<T* const*>(Ip->f[T_steps & 1]);
  T* const o0 = outp[0];
  T* const o1 = outp[1];
  T* const o2 = outp[2];
  const int rows = (H + CL - 1) / CL;
  const int r0 = rank * rows;
  const int nr = max(0, min(rows, H - r0));
  Band<T> s = band_layout<T>(c_smem, rows, W);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  // this band's monitor accumulators (FP64, in shared memory for the whole run)
  const int mw = mb.hi[2] - mb.lo[2];
  const int mr0 = mon ? max(mb.lo[1], r0) : 0;
  const int mr1 = mon ? min(mb.hi[1], r0 + nr) : 0;
  const int mrows = max(0, mr1 - mr0);
  const long long ncell = mon ? (long long)(mb.hi[1] - mb.lo[1]) * mw : 0;
  double* macc = reinterpret_cast<double*>(
      c_smem + ((band_elems(rows, W) * sizeof(T) + 15) / 16) * 16);
  const long long mcells = (long long)mrows * mw;
  for (long long q = threadIdx.x; q < mcells * nfq; q += blockDim.x) {
    const long long fq = q / mcells, c = q % mcells;
    const long long cell = (long long)(mr0 - mb.lo[1]) * mw + c;
    macc[2 * q] = accb[(fq * ncell + cell) * 2];
    macc[2 * q + 1] = accb[(fq * ncell + cell) * 2 + 1];
  }

  for (int j = threadIdx.x; j < W; j += blockDim.x) {
    s.bx[j] = static_cast<T>(pb1[j]);
    s.gx[j] = static_cast<T>(1.0 + pc1[j]);
  }
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    s.by[r] = static_cast<T>(pb0[r0 + r]);
    s.gy[r] = static_cast<T>(1.0 + pc0[r0 + r]);
  }
  for (int r = warp; r < nr; r += nw)
    for (int j = lane; j < W; j += 32) {
      const long long o = (long long)r * W + j;
      s.f[o] = T(0);
      s.a[o] = T(0);
      s.b[o] = T(0);
      s.ce[o] = ceg[(long long)(r0 + r) * py + j];
    }
  cl.sync();  // every band initialised before any neighbour reads it

  // neighbour bands (distributed shared memory); unused when out of range
  const int up = rank + 1 < CL ? rank + 1 : rank, dn_ = rank > 0 ? rank - 1 : rank;
  const Band<T> nxt = band_layout<T>(cl.map_shared_rank(c_smem, up), rows, W);
  const Band<T> prv = band_layout<T>(cl.map_shared_rank(c_smem, dn_), rows, W);

  for (int n = 0; n < T_steps; ++n) {
    // half-step 1: H (TM) / E (TE) from the injected field
    for (int r = warp; r < nr; r += nw) {
      const int i = r0 + r;
      const T byr = s.by[r], gyr = s.gy[r];
      const bool last = i == H - 1, first = i == 0;
      const T* below = (r + 1 < nr) ? s.f + (long long)(r + 1) * W : nxt.f;
      const T* above = (r > 0) ? s.f + (long long)(r - 1) * W : prv.f + (long long)(rows - 1) * W;
      for (int j = lane; j < W; j += 32) {
        const long long o = (long long)r * W + j;
        if (POL == DN_TM) {
          const T ez = s.f[o];
          const T dj = (j < W - 1) ? s.f[o + 1] - ez : T(0);
          const T di = !last ? below[j] - ez : T(0);
          s.a[o] = byr * s.a[o] - dt * gyr * (dj * idl);
          s.b[o] = s.bx[j] * s.b[o] + dt * s.gx[j] * (di * idl);
        } else {
          const T hz = s.f[o];
          const T dj = (j > 0) ? hz - s.f[o - 1] : T(0);
          const T di = !first ? hz - above[j] : T(0);
          const T cx = s.gx[j] * (dj * idl);
          const T cy = -(gyr * (di * idl));
          const T c = s.ce[o];
          s.a[o] = s.bx[j] * s.a[o] + c * cx;
          s.b[o] = byr * s.b[o] + c * cy;
        }
      }
    }
    cl.sync();
    // half-step 2: the injected field from the new pair, source, monitors
    const T wv = src ? wave[n] : T(0);
    const double* ph = mon ? phase + (long long)n * nfq * 2 : nullptr;
    for (int r = warp; r < nr; r += nw) {
      const int i = r0 + r;
      const T byr = s.by[r], gyr = s.gy[r];
      const bool last = i == H - 1, first = i == 0;
      const T* bup = (r > 0) ? s.b + (long long)(r - 1) * W : prv.b + (long long)(rows - 1) * W;
      const T* bdn = (r + 1 < nr) ? s.b + (long long)(r + 1) * W : nxt.b;
      const bool src_row = src && i >= sb.lo[1] && i < sb.hi[1];
      const bool mon_row = mon && i >= mb.lo[1] && i < mb.hi[1];
      for (int j = lane; j < W; j += 32) {
        const long long o = (long long)r * W + j;
        const T fo = s.f[o];
        const T bb = s.bx[j] * byr;
        T v0;
        if (POL == DN_TM) {
          const T dHy = !first ? s.b[o] - bup[j] : T(0);
          const T dHx = (j > 0) ? s.a[o] - s.a[o - 1] : T(0);
          const T cz = s.gx[j] * (dHy * idl) - gyr * (dHx * idl);
          v0 = bb * fo + s.ce[o] * cz;
        } else {
          const T dEy = !last ? bdn[j] - s.b[o] : T(0);
          const T dEx = (j < W - 1) ? s.a[o + 1] - s.a[o] : T(0);
          v0 = bb * fo + dt * (s.gx[j] * (dEy * idl) - gyr * (dEx * idl));
        }
        if (src_row && j >= sb.lo[2] && j < sb.hi[2]) v0 += wv;
        if (mon_row && j >= mb.lo[2] && j < mb.hi[2]) {
          const long long c = (long long)(i - mr0) * mw + (j - mb.lo[2]);
          const double x = static_cast<double>(v0);
          for (int fq = 0; fq < nfq; ++fq) {
            double* acc = macc + (fq * mcells + c) * 2;
            acc[0] = fma(x, ph[2 * fq], acc[0]);
            acc[1] = fma(x, ph[2 * fq + 1], acc[1]);
          }
        }
        s.f[o] = v0;
      }
    }
    cl.sync();
  }
  // final state into the set a step-by-step run would end in; monitor sums out
  for (int r = warp; r < nr; r += nw)
    for (int j = lane; j < W; j += 32) {
      const long long o = (long long)r * W + j, g = (long long)(r0 + r) * py + j;
      o0[g] = s.f[o];
      o1[g] = s.a[o];
      o2[g] = s.b[o];
    }
  for (long long q = threadIdx.x; q < mcells * nfq; q += blockDim.x) {
    const long long fq = q / mcells, c = q % mcells;
    const long long cell = (long long)(mr0 - mb.lo[1]) * mw + c;
    accb[(fq * ncell + cell) * 2] = macc[2 * q];
    accb[(fq * ncell + cell) * 2 + 1] = macc[2 * q + 1];
  }
}

// ---------------------------------------------------------------------------
// Double-buffered cluster solve: every field has two band buffers; step n
// reads buffer n & 1 and writes the other.  The one row of the other
// half-step's field that comes from a neighbouring band (TM: Hy of the row
// above the band; TE: Ey of the row below it) is recomputed here from the
// neighbour's unchanged input buffers with the neighbour's own arithmetic, so
// the two half-steps need only a CTA barrier between them and each step one
// cluster barrier (the in-place kernel above needs two).  Twice the field
// shared memory: used when the grid fits, else the in-place kernel.
// ---------------------------------------------------------------------------
template <typename T>
struct BandDB {
  // buffer k of the fields at fld + (3k + {0, 1, 2}) * n: the injected field
  // (Ez / Hz), Hx / Ex, Hy / Ey, rows x W each (pointer arithmetic, not an
  // array indexed by the step parity, keeps the view in registers)
  T* fld;
  long long n;
  __device__ __forceinline__ T* f(int k) const { return fld + (3 * k) * n; }
  __device__ __forceinline__ T* a(int k) const { return fld + (3 * k + 1) * n; }
  __device__ __forceinline__ T* b(int k) const { return fld + (3 * k + 2) * n; }
  T* ce;    // dt / eps
  T* bx;    // W
  T* gx;    // W
  T* by;    // rows
  T* gy;    // rows
  T* halo;  // W: the neighbour-row value of the second half-step
};

__host__ __device__ inline long long band_elems_db(long long rows, long long W) {
  return 7 * rows * W + 3 * W + 2 * rows;
}

template <typename T>
__device__ __forceinline__ BandDB<T> band_layout_db(unsigned char* smem, int rows, int W) {
  BandDB<T> s;
  T* p = reinterpret_cast<T*>(smem);
  const long long n = (long long)rows * W;
  s.fld = p;
  s.n = n;
  s.ce = p + 6 * n;
  s.bx = p + 7 * n;
  s.gx = s.bx + W;
  s.by = s.gx + W;
  s.gy = s.by + rows;
  s.halo = s.gy + rows;
  return s;
}

template <typename T, int POL, int CL>
__global__ void __launch_bounds__(512, 1) k_batch2d_cluster_db(unsigned char* table) {
  extern __shared__ __align__(16) unsigned char c_smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const TableView v = view(table);
  const dn_batch2d_inst* Ip = v.inst + blockIdx.x / CL;
  const int H = Ip->H, W = Ip->W, T_steps = Ip->n_steps;
  const long long py = Ip->pitch;
  const T dt = static_cast<T>(Ip->dt), idl = static_cast<T>(1.0 / Ip->dl);
  const bool src = Ip->src_comp >= 0, mon = Ip->mon_comp >= 0;
  const dn_box sb = Ip->src_box, mb = Ip->mon_box;
  const int nfq = Ip->n_freq;
  const double* __restrict__ phase = Ip->phase;
  double* __restrict__ accb = Ip->acc;
  const T* __restrict__ wave = static_cast<const T*>(Ip->wave);
  const double* pb0 = Ip->b[0];
  const double* pb1 = Ip->b[1];
  const double* pc0 = Ip->c[0];
  const double* pc1 = Ip->c[1];
  const T* __restrict__ ceg = static_cast<const T*>(Ip->ce);
  T* const* outp = reinterpret_cast<T* const*>(Ip->f[T_steps & 1]);
  T* const o0 = outp[0];
  T* const o1 = outp[1];
  T* const o2 = outp[2];
  const int rows = (H + CL - 1) / CL;
  const int r0 = rank * rows;
  const int nr = max(0, min(rows, H - r0));
  BandDB<T> s = band_layout_db<T>(c_smem, rows, W);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int mw = mb.hi[2] - mb.lo[2];
  const int mr0 = mon ? max(mb.lo[1], r0) : 0;
  const int mr1 = mon ? min(mb.hi[1], r0 + nr) : 0;
  const int mrows = max(0, mr1 - mr0);
  const long long ncell = mon ? (long long)(mb.hi[1] - mb.lo[1]) * mw : 0;
  double* macc = reinterpret_cast<double*>(
      c_smem + ((band_elems_db(rows, W) * sizeof(T) + 15) / 16) * 16);
  const long long mcells = (long long)mrows * mw;
  for (long long q = threadIdx.x; q < mcells * nfq; q += blockDim.x) {
    const long long fq = q / mcells, c = q % mcells;
    const long long cell = (long long)(mr0 - mb.lo[1]) * mw + c;
    macc[2 * q] = accb[(fq * ncell + cell) * 2];
    macc[2 * q + 1] = accb[(fq * ncell + cell) * 2 + 1];
  }
  for (int j = threadIdx.x; j < W; j += blockDim.x) {
    s.bx[j] = static_cast<T>(pb1[j]);
    s.gx[j] = static_cast<T>(1.0 + pc1[j]);
  }
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    s.by[r] = static_cast<T>(pb0[r0 + r]);
    s.gy[r] = static_cast<T>(1.0 + pc0[r0 + r]);
  }
  for (int r = warp; r < nr; r += nw)
    for (int j = lane; j < W; j += 32) {
      const long long o = (long long)r * W + j;
      s.f(0)[o] = T(0);
      s.a(0)[o] = T(0);
      s.b(0)[o] = T(0);
      s.ce[o] = ceg[(long long)(r0 + r) * py + j];
    }
  cl.sync();  // every band initialised before any neighbour reads it

  const int up = rank + 1 < CL ? rank + 1 : rank, dn_ = rank > 0 ? rank - 1 : rank;
  const BandDB<T> nxt = band_layout_db<T>(cl.map_shared_rank(c_smem, up), rows, W);
  const BandDB<T> prv = band_layout_db<T>(cl.map_shared_rank(c_smem, dn_), rows, W);
  // the neighbour row of the second half-step exists (TM: a band above; TE: a
  // band below that holds rows)
  const bool halo_tm = r0 > 0 && nr > 0;
  const bool halo_te = nr > 0 && r0 + nr < H;

  for (int n = 0; n < T_steps; ++n) {
    const int p = n & 1, q = p ^ 1;
    const T* fp = s.f(p);
    const T* ap = s.a(p);
    const T* bp = s.b(p);
    T* aq = s.a(q);
    T* bq = s.b(q);
    // the neighbour row is spread over all threads, one column each (more
    // columns than threads: the rest after the own rows); the remote loads of
    // the first column are issued here and used after the own rows
    const bool hal = POL == DN_TM ? halo_tm : halo_te;
    const int hj = threadIdx.x;
    const long long hrow = POL == DN_TM ? (long long)(rows - 1) * W : 0;  // neighbour's row
    const long long orow = POL == DN_TM ? 0 : (long long)(nr - 1) * W;   // own boundary row
    const T* hf = POL == DN_TM ? prv.f(p) : nxt.f(p);
    const T* hb = POL == DN_TM ? prv.b(p) : nxt.b(p);
    T pf = T(0), pb = T(0), pc = T(0);
    if (hal && hj < W) {
      pf = hf[hrow + hj];
      pb = hb[hrow + hj];
      if (POL == DN_TE) pc = nxt.ce[hj];
    }
    // half-step 1: H (TM) / E (TE) from the injected field of buffer p
    for (int r = warp; r < nr; r += nw) {
      const int i = r0 + r;
      const T byr = s.by[r], gyr = s.gy[r];
      const bool last = i == H - 1, first = i == 0;
      const T* below = (r + 1 < nr) ? fp + (long long)(r + 1) * W : nxt.f(p);
      const T* above = (r > 0) ? fp + (long long)(r - 1) * W : prv.f(p) + (long long)(rows - 1) * W;
#pragma unroll 4
      for (int j = lane; j < W; j += 32) {
        const long long o = (long long)r * W + j;
        if (POL == DN_TM) {
          const T ez = fp[o];
          const T dj = (j < W - 1) ? fp[o + 1] - ez : T(0);
          const T di = !last ? below[j] - ez : T(0);
          aq[o] = byr * ap[o] - dt * gyr * (dj * idl);
          bq[o] = s.bx[j] * bp[o] + dt * s.gx[j] * (di * idl);
        } else {
          const T hz = fp[o];
          const T dj = (j > 0) ? hz - fp[o - 1] : T(0);
          const T di = !first ? hz - above[j] : T(0);
          const T cx = s.gx[j] * (dj * idl);
          const T cy = -(gyr * (di * idl));
          const T c = s.ce[o];
          aq[o] = s.bx[j] * ap[o] + c * cx;
          bq[o] = byr * bp[o] + c * cy;
        }
      }
    }
    // the neighbour row, with the neighbour's own arithmetic
    if (hal) {
      const T nby = POL == DN_TE ? nxt.by[0] : T(0), ngy = POL == DN_TE ? nxt.gy[0] : T(0);
      for (int j = hj; j < W; j += blockDim.x) {
        T vf = pf, vb = pb, vc = pc;
        if (j != hj) {
          vf = hf[hrow + j];
          vb = hb[hrow + j];
          if (POL == DN_TE) vc = nxt.ce[j];
        }
        if (POL == DN_TM) {
          // Hy of row r0-1 (the band above's last row; r0-1 < H-1)
          const T di = fp[orow + j] - vf;
          s.halo[j] = s.bx[j] * vb + dt * s.gx[j] * (di * idl);
        } else {
          // Ey of row r0+nr (the band below's first row; r0+nr > 0)
          const T di = vf - fp[orow + j];
          const T cy = -(ngy * (di * idl));
          s.halo[j] = nby * vb + vc * cy;
        }
      }
    }
    __syncthreads();
    // half-step 2: the injected field from the new pair, source, monitors
    const T wv = src ? wave[n] : T(0);
    const double* ph = mon ? phase + (long long)n * nfq * 2 : nullptr;
    T* fq = s.f(q);
    for (int r = warp; r < nr; r += nw) {
      const int i = r0 + r;
      const T byr = s.by[r], gyr = s.gy[r];
      const bool last = i == H - 1, first = i == 0;
      const T* bup = (r > 0) ? bq + (long long)(r - 1) * W : s.halo;
      const T* bdn = (r + 1 < nr) ? bq + (long long)(r + 1) * W : s.halo;
      const bool src_row = src && i >= sb.lo[1] && i < sb.hi[1];
      const bool mon_row = mon && i >= mb.lo[1] && i < mb.hi[1];
#pragma unroll 4
      for (int j = lane; j < W; j += 32) {
        const long long o = (long long)r * W + j;
        const T fo = fp[o];
        const T bb = s.bx[j] * byr;
        T v0;
        if (POL == DN_TM) {
          const T dHy = !first ? bq[o] - bup[j] : T(0);
          const T dHx = (j > 0) ? aq[o] - aq[o - 1] : T(0);
          const T cz = s.gx[j] * (dHy * idl) - gyr * (dHx * idl);
          v0 = bb * fo + s.ce[o] * cz;
        } else {
          const T dEy = !last ? bdn[j] - bq[o] : T(0);
          const T dEx = (j < W - 1) ? aq[o + 1] - aq[o] : T(0);
          v0 = bb * fo + dt * (s.gx[j] * (dEy * idl) - gyr * (dEx * idl));
        }
        if (src_row && j >= sb.lo[2] && j < sb.hi[2]) v0 += wv;
        if (mon_row && j >= mb.lo[2] && j < mb.hi[2]) {
          const long long c = (long long)(i - mr0) * mw + (j - mb.lo[2]);
          const double x = static_cast<double>(v0);
          for (int f = 0; f < nfq; ++f) {
            double* acc = macc + (f * mcells + c) * 2;
            acc[0] = fma(x, ph[2 * f], acc[0]);
            acc[1] = fma(x, ph[2 * f + 1], acc[1]);
          }
        }
        fq[o] = v0;
      }
    }
    cl.sync();  // buffer q complete everywhere before step n+1 reads it
  }
  const int fin = T_steps & 1;  // the buffer the last step wrote
  for (int r = warp; r < nr; r += nw)
    for (int j = lane; j < W; j += 32) {
      const long long o = (long long)r * W + j, g = (long long)(r0 + r) * py + j;
      o0[g] = s.f(fin)[o];
      o1[g] = s.a(fin)[o];
      o2[g] = s.b(fin)[o];
    }
  for (long long q = threadIdx.x; q < mcells * nfq; q += blockDim.x) {
    const long long fq = q / mcells, c = q % mcells;
    const long long cell = (long long)(mr0 - mb.lo[1]) * mw + c;
    accb[(fq * ncell + cell) * 2] = macc[2 * q];
    accb[(fq * ncell + cell) * 2 + 1] = macc[2 * q + 1];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int validate(const dn_batch2d* cfg, const dn_batch2d_inst* insts) {
  if (!cfg || !insts || cfg->n_inst < 1) return DN_EINVAL;
  if (cfg->pol != DN_TM && cfg->pol != DN_TE) return DN_EINVAL;
  if (cfg->dtype != DN_F32 && cfg->dtype != DN_F64) return DN_EINVAL;
  if (cfg->K < 1) return DN_EINVAL;
  if (cfg->tile_rows != 8 && cfg->tile_rows != 16 && cfg->tile_rows != 32) return DN_EINVAL;
  const int first = cfg->pol == DN_TM ? DN_EZ : DN_HZ;
  for (int b = 0; b < cfg->n_inst; ++b) {
    const dn_batch2d_inst& I = insts[b];
    if (I.H < 1 || I.W < 1 || I.pitch < I.W || I.n_steps < 1) return DN_EINVAL;
    if (!(I.dt > 0.0) || !(I.dl > 0.0) || !I.ce || !I.b[0] || !I.b[1] || !I.c[0] || !I.c[1])
      return DN_EINVAL;
    for (int s = 0; s < 2; ++s)
      for (int c = 0; c < 3; ++c)
        if (!I.f[s][c]) return DN_EINVAL;
    // rows move in 16-byte chunks: 16-byte rows (fields and the FP64
    // gradient) and 16-byte aligned arrays
    const int64_t esz = cfg->dtype == DN_F32 ? 4 : 8;
    if ((I.pitch * esz) % 16 != 0 || (I.pitch * 8) % 16 != 0 || !aligned16(I.ce)) return DN_EINVAL;
    for (int s = 0; s < 2; ++s)
      for (int c = 0; c < 3; ++c)
        if (!aligned16(I.f[s][c]) || (I.lam[s][c] && !aligned16(I.lam[s][c]))) return DN_EINVAL;
    if ((I.ckpt && !aligned16(I.ckpt)) || (I.curl && !aligned16(I.curl)) ||
        (I.grad && !aligned16(I.grad)))
      return DN_EINVAL;
    if (I.src_comp != DN_NONE) {
      if (I.src_comp != first || !I.wave || !box_ok(I.src_box, 1, I.H, I.W)) return DN_EINVAL;
    }
    if (I.mon_comp != DN_NONE) {
      if (I.mon_comp != first || !box_ok(I.mon_box, 1, I.H, I.W) || I.n_freq < 1 ||
          I.n_freq > DN_MAX_FREQS || !I.phase || !I.acc)
        return DN_EINVAL;
    }
  }
  return DN_OK;
}

int total_tiles_of(const dn_batch2d* cfg, const dn_batch2d_inst* insts) {
  long long t = 0;
  for (int b = 0; b < cfg->n_inst; ++b)
    t += (long long)((insts[b].W + tile_cols(cfg->dtype) - 1) / tile_cols(cfg->dtype)) *
         ((insts[b].H + cfg->tile_rows - 1) / cfg->tile_rows);
  return t > 0x7fffffffLL ? -1 : (int)t;
}

template <typename T, int POL, int TI>
int launch(bool fwd, void* table, int* status, cudaStream_t s, int max_tiles) {
  auto kern = fwd ? k_batch2d_fwd<T, POL, TI> : k_batch2d_bwd<T, POL, TI>;
  int dev = 0, nsm = 0, per_sm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  DN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NTB, 0));
  if (per_sm < 1) return DN_EUNSUPPORTED;
  int grid = nsm * per_sm;
  if (grid > max_tiles) grid = max_tiles;
  // the barrier words start from zero arrivals and no abort
  DN_CUDA_CHECK(cudaMemsetAsync(static_cast<unsigned char*>(table) + offsetof(TableHeader, bar),
                                0, sizeof(unsigned int) * 4, s));
  void* args[] = {&table, &status};
  DN_CUDA_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kern), dim3(grid), dim3(NTB),
                                            args, 0, s));
  return DN_OK;
}

template <typename T, int POL>
int dispatch_rows(bool fwd, int rows, void* table, int* status, cudaStream_t s, int max_tiles) {
  if (rows == 8) return launch<T, POL, 8>(fwd, table, status, s, max_tiles);
  if (rows == 16) return launch<T, POL, 16>(fwd, table, status, s, max_tiles);
  return launch<T, POL, 32>(fwd, table, status, s, max_tiles);
}

int run(bool fwd, const dn_batch2d* cfg, void* dev_table, int32_t* status, void* stream,
        int max_tiles) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool tm = cfg->pol == DN_TM;
  if (cfg->dtype == DN_F32)
    return tm ? dispatch_rows<float, DN_TM>(fwd, cfg->tile_rows, dev_table, status, s, max_tiles)
              : dispatch_rows<float, DN_TE>(fwd, cfg->tile_rows, dev_table, status, s, max_tiles);
  return tm ? dispatch_rows<double, DN_TM>(fwd, cfg->tile_rows, dev_table, status, s, max_tiles)
            : dispatch_rows<double, DN_TE>(fwd, cfg->tile_rows, dev_table, status, s, max_tiles);
}

constexpr long long CLUSTER_SMEM_MAX = 227 * 1024;

// bytes of shared memory per CTA for a cluster of cl CTAs (db: the
// double-buffered kernel), -1 if too large
long long cluster_bytes(const dn_batch2d* cfg, const dn_batch2d_inst* insts, int cl, bool db) {
  const long long es = cfg->dtype == DN_F32 ? 4 : 8;
  long long need = 0;
  for (int b = 0; b < cfg->n_inst; ++b) {
    const dn_batch2d_inst& I = insts[b];
    const long long rows = (I.H + cl - 1) / cl;
    const long long elems = db ? band_elems_db(rows, I.W) : band_elems(rows, I.W);
    long long bytes = (elems * es + 15) / 16 * 16;
    if (I.mon_comp != DN_NONE) {  // the band's share of the monitor box, FP64 complex
      const long long bh = I.mon_box.hi[1] - I.mon_box.lo[1];
      const long long bw = I.mon_box.hi[2] - I.mon_box.lo[2];
      bytes += std::min(rows, bh) * bw * I.n_freq * 16;
    }
    need = std::max(need, bytes);
  }
  return need <= CLUSTER_SMEM_MAX ? need : -1;
}

template <typename T, int POL, int CL, bool DB>
int launch_cluster(void* table, int n_inst, long long smem, cudaStream_t s) {
  auto kern = DB ? k_batch2d_cluster_db<T, POL, CL> : k_batch2d_cluster<T, POL, CL>;
  DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (CL > 8)
    DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3((unsigned)(n_inst * CL));
  lc.blockDim = dim3(512);
  lc.dynamicSmemBytes = (size_t)smem;
  lc.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  int clusters = 0;
  DN_CUDA_CHECK(cudaOccupancyMaxActiveClusters(&clusters, kern, &lc));
  if (clusters < 1) return DN_EUNSUPPORTED;
  DN_CUDA_CHECK(cudaLaunchKernelEx(&lc, kern, static_cast<unsigned char*>(table)));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

template <typename T, int POL>
int dispatch_cluster(int cl, bool db, void* table, int n_inst, long long smem, cudaStream_t s) {
  if (db)
    return cl == 8 ? launch_cluster<T, POL, 8, true>(table, n_inst, smem, s)
                   : launch_cluster<T, POL, 16, true>(table, n_inst, smem, s);
  return cl == 8 ? launch_cluster<T, POL, 8, false>(table, n_inst, smem, s)
                 : launch_cluster<T, POL, 16, false>(table, n_inst, smem, s);
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_batch2d_cluster_size(const dn_batch2d* cfg, const dn_batch2d_inst* insts,
                                           int64_t* smem_bytes) {
  if (dn::validate(cfg, insts) != DN_OK || !smem_bytes) return -1;
  // 16 CTAs per grid (half the band of 8 each, twice the SMs per grid) is the
  // faster size on B200; the double-buffered kernel (one cluster barrier per
  // step) where its twice-as-large bands fit, else the in-place one
  for (int cl : {16, 8})
    for (bool db : {true, false}) {
      const long long b = dn::cluster_bytes(cfg, insts, cl, db);
      if (b > 0) {
        *smem_bytes = b;
        return cl | (db ? DN_CLUSTER_DOUBLE_BUFFERED : 0);
      }
    }
  return 0;
}

extern "C" int32_t dn_batch2d_forward_cluster(const dn_batch2d* cfg, void* dev_table,
                                              int32_t cluster, int64_t smem_bytes,
                                              void* stream) {
  if (!cfg || !dev_table || (reinterpret_cast<uintptr_t>(dev_table) & 15)) return DN_EINVAL;
  if (cfg->pol != DN_TM && cfg->pol != DN_TE) return DN_EINVAL;
  if (cfg->dtype != DN_F32 && cfg->dtype != DN_F64) return DN_EINVAL;
  const bool db = (cluster & DN_CLUSTER_DOUBLE_BUFFERED) != 0;
  const int csize = cluster & ~DN_CLUSTER_DOUBLE_BUFFERED;
  if ((csize != 8 && csize != 16) || smem_bytes < 1 || smem_bytes > dn::CLUSTER_SMEM_MAX ||
      cfg->n_inst < 1 || (long long)cfg->n_inst * csize > 0x7fffffffLL)
    return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool tm = cfg->pol == DN_TM;
  const int n = cfg->n_inst;
  if (cfg->dtype == DN_F32)
    return tm ? dn::dispatch_cluster<float, DN_TM>(csize, db, dev_table, n, smem_bytes, s)
              : dn::dispatch_cluster<float, DN_TE>(csize, db, dev_table, n, smem_bytes, s);
  return tm ? dn::dispatch_cluster<double, DN_TM>(csize, db, dev_table, n, smem_bytes, s)
            : dn::dispatch_cluster<double, DN_TE>(csize, db, dev_table, n, smem_bytes, s);
}

extern "C" int64_t dn_batch2d_table_bytes(const dn_batch2d* cfg, const dn_batch2d_inst* insts) {
  if (dn::validate(cfg, insts) != DN_OK) return -1;
  const int tt = dn::total_tiles_of(cfg, insts);
  if (tt < 0) return -1;
  size_t op, os, om, oi, oe;
  dn::table_offsets(cfg->n_inst, tt, &op, &os, &om, &oi, &oe);
  return (int64_t)oe;
}

extern "C" int32_t dn_batch2d_pack(const dn_batch2d* cfg, const dn_batch2d_inst* insts,
                                   void* host_table, int64_t bytes) {
  int rc = dn::validate(cfg, insts);
  if (rc != DN_OK) return rc;
  if (!host_table || bytes < dn_batch2d_table_bytes(cfg, insts)) return DN_EINVAL;
  const int n = cfg->n_inst;
  const int tt = dn::total_tiles_of(cfg, insts);
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return insts[a].n_steps > insts[b].n_steps; });
  unsigned char* base = static_cast<unsigned char*>(host_table);
  std::memset(base, 0, (size_t)bytes);
  size_t op, os, om, oi, oe;
  dn::table_offsets(n, tt, &op, &os, &om, &oi, &oe);
  dn::TableHeader* h = reinterpret_cast<dn::TableHeader*>(base);
  h->n_inst = n;
  h->total_tiles = tt;
  h->K = cfg->K;
  h->tile_rows = cfg->tile_rows;
  int* prefix = reinterpret_cast<int*>(base + op);
  int* steps = reinterpret_cast<int*>(base + os);
  int2* map = reinterpret_cast<int2*>(base + om);
  dn_batch2d_inst* inst = reinterpret_cast<dn_batch2d_inst*>(base + oi);
  int t = 0, max_steps = 0;
  for (int k = 0; k < n; ++k) {
    const dn_batch2d_inst& I = insts[order[k]];
    inst[k] = I;
    steps[k] = I.n_steps;
    prefix[k] = t;
    const int tc = dn::tile_cols(cfg->dtype);
    const int ntiles = ((I.W + tc - 1) / tc) * ((I.H + cfg->tile_rows - 1) / cfg->tile_rows);
    for (int q = 0; q < ntiles; ++q) map[t++] = make_int2(k, q);
    max_steps = std::max(max_steps, I.n_steps);
  }
  prefix[n] = t;
  h->max_steps = max_steps;
  h->nseg = (max_steps + cfg->K - 1) / cfg->K;
  return DN_OK;
}

extern "C" int32_t dn_batch2d_forward(const dn_batch2d* cfg, void* dev_table, int32_t* status,
                                      void* stream) {
  if (!cfg || !dev_table || (reinterpret_cast<uintptr_t>(dev_table) & 15)) return DN_EINVAL;
  if (cfg->tile_rows != 8 && cfg->tile_rows != 16 && cfg->tile_rows != 32) return DN_EINVAL;
  if (cfg->pol != DN_TM && cfg->pol != DN_TE) return DN_EINVAL;
  if (cfg->dtype != DN_F32 && cfg->dtype != DN_F64) return DN_EINVAL;
  return dn::run(true, cfg, dev_table, status, stream, cfg->max_ctas > 0 ? cfg->max_ctas : 1 << 30);
}

extern "C" int32_t dn_batch2d_backward(const dn_batch2d* cfg, void* dev_table, int32_t* status,
                                       void* stream) {
  if (!cfg || !dev_table || (reinterpret_cast<uintptr_t>(dev_table) & 15)) return DN_EINVAL;
  if (cfg->tile_rows != 8 && cfg->tile_rows != 16 && cfg->tile_rows != 32) return DN_EINVAL;
  if (cfg->pol != DN_TM && cfg->pol != DN_TE) return DN_EINVAL;
  if (cfg->dtype != DN_F32 && cfg->dtype != DN_F64) return DN_EINVAL;
  return dn::run(false, cfg, dev_table, status, stream, cfg->max_ctas > 0 ? cfg->max_ctas : 1 << 30);
}

extern "C" int32_t dn_batch2d_barrier_selftest(int32_t n_ctas, int32_t missing, int64_t spin_limit,
                                               int32_t rounds, void* dev_bar, int32_t* status,
                                               void* stream) {
  if (n_ctas < 1 || missing < 0 || missing > 1024 || rounds < 1 || spin_limit < 1 ||
      spin_limit > static_cast<int64_t>(dn::BAR_SPIN_LIMIT) || !dev_bar || !status ||
      (reinterpret_cast<uintptr_t>(dev_bar) & 15))
    return DN_EINVAL;
  int dev = 0, nsm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (n_ctas > nsm) return DN_EINVAL;  // one 32-thread CTA per SM at most: all resident at once
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DN_CUDA_CHECK(cudaMemsetAsync(dev_bar, 0, 4 * sizeof(unsigned int), s));
  dn::k_barrier_selftest<<<n_ctas, 32, 0, s>>>(static_cast<unsigned int*>(dev_bar), status,
                                               static_cast<unsigned int>(missing),
                                               static_cast<unsigned long long>(spin_limit), rounds);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}
