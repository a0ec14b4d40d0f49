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
// One CTA owns a 16 x 32 tile.  The field differenced first (Ez for TM, Hz
// for TE) is staged in shared memory with a one-cell ring; the tile's two
// intermediate fields are computed for the tile plus the one-cell halo that
// the second update needs (recomputed, never exchanged), so a step reads
// each array once and writes each once (28 B per cell in FP32).  Ping-pong
// buffers keep neighbouring CTAs from seeing this step's writes.
#include "dn_host.cuh"

namespace dn {
namespace {

constexpr int TJ2 = 32;  // tile columns (x, contiguous)
constexpr int TI2 = 16;  // tile rows (y)
constexpr int NT2 = 256;
constexpr int R2 = TI2 / (NT2 / 32);  // rows per thread

// curl record for the adjoint replay (see dn_curl_record)
template <typename T>
struct CurlRec2 {
  T* curl[3];
  long long stride;
  int t0;
};

template <typename T, int POL, bool REC>
__global__ void __launch_bounds__(NT2, 8) k_fdtd2d_step(const StepParams<T> p, const CurlRec2<T> rec) {
  __shared__ T s_f[TI2 + 2][TJ2 + 2];
  __shared__ T s_a[TI2 + 1][TJ2 + 1];
  __shared__ T s_b[TI2 + 1][TJ2 + 1];
  __shared__ T s_bx[TJ2 + 2], s_gx[TJ2 + 2];
  __shared__ T s_by[TI2 + 2], s_gy[TI2 + 2];
  __shared__ int s_skip;
  // a previous launch that recorded an error turns this one into a no-op
  if (threadIdx.x == 0)
    s_skip = p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0;
  __syncthreads();
  if (s_skip) return;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = blockIdx.y * TI2, j0 = blockIdx.x * TJ2;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  constexpr int F = (POL == DN_TM) ? DN_EZ : DN_HZ;
  const T dt = p.dt, idl = p.inv_dl;

  // profile tables: entry t <-> position origin - 1 + t
  for (int t = threadIdx.x; t < TJ2 + 2; t += NT2) {
    const int j = j0 - 1 + t;
    const bool ok = j >= 0 && j < W;
    s_bx[t] = ok ? static_cast<T>(p.b[2][j]) : T(1);
    s_gx[t] = ok ? static_cast<T>(1.0 + p.c[2][j]) : T(1);
  }
  for (int t = threadIdx.x; t < TI2 + 2; t += NT2) {
    const int i = i0 - 1 + t;
    const bool ok = i >= 0 && i < H;
    s_by[t] = ok ? static_cast<T>(p.b[1][i]) : T(1);
    s_gy[t] = ok ? static_cast<T>(1.0 + p.c[1][i]) : T(1);
  }
  for (int t = threadIdx.x; t < (TI2 + 2) * (TJ2 + 2); t += NT2) {
    const int r = t / (TJ2 + 2), c = t % (TJ2 + 2);
    const int i = i0 - 1 + r, j = j0 - 1 + c;
    s_f[r][c] = (i >= 0 && i < H && j >= 0 && j < W) ? p.in[F][i * py + j] : T(0);
  }
  __syncthreads();

  const int jj = lane;
  const int j = j0 + jj;
  T a_own[R2], b_own[R2];  // TM: Hx, Hy   TE: Ex, Ey  (new values of owned cells)

  if (POL == DN_TM) {
    // ---- H from old Ez: owned cells ------------------------------------
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const int ii = warp + 8 * r, i = i0 + ii;
      a_own[r] = b_own[r] = T(0);
      if (i < H && j < W) {
        const long long o = i * py + j;
        const T ez = s_f[ii + 1][jj + 1];
        const T dj = (j < W - 1) ? s_f[ii + 1][jj + 2] - ez : T(0);
        const T di = (i < H - 1) ? s_f[ii + 2][jj + 1] - ez : T(0);
        a_own[r] = s_by[ii + 1] * p.in[DN_HX][o] - dt * s_gy[ii + 1] * (dj * idl);
        b_own[r] = s_bx[jj + 1] * p.in[DN_HY][o] + dt * s_gx[jj + 1] * (di * idl);
      }
      s_a[ii][jj + 1] = a_own[r];
      s_b[ii + 1][jj] = b_own[r];
    }
    // ---- halos: Hx at column j0-1, Hy at row i0-1 ------------------------
    if (warp == 0 && lane < TI2) {
      const int ii = lane, i = i0 + ii, jh = j0 - 1;
      T v = T(0);
      if (jh >= 0 && i < H) {
        const T dj = s_f[ii + 1][1] - s_f[ii + 1][0];
        v = s_by[ii + 1] * p.in[DN_HX][i * py + jh] - dt * s_gy[ii + 1] * (dj * idl);
      }
      s_a[ii][0] = v;
    } else if (warp == 1) {
      const int ih = i0 - 1;
      T v = T(0);
      if (ih >= 0 && j < W) {
        const T di = s_f[1][jj + 1] - s_f[0][jj + 1];
        v = s_bx[jj + 1] * p.in[DN_HY][ih * py + j] + dt * s_gx[jj + 1] * (di * idl);
      }
      s_b[0][jj] = v;
    }
  } else {
    // ---- E from old Hz: owned cells ------------------------------------
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const int ii = warp + 8 * r, i = i0 + ii;
      a_own[r] = b_own[r] = T(0);
      if (i < H && j < W) {
        const long long o = i * py + j;
        const T ce = p.ce[o];
        const T hz = s_f[ii + 1][jj + 1];
        const T dj = (j > 0) ? hz - s_f[ii + 1][jj] : T(0);
        const T di = (i > 0) ? hz - s_f[ii][jj + 1] : T(0);
        const T curl_x = s_gx[jj + 1] * (dj * idl);
        const T curl_y = -(s_gy[ii + 1] * (di * idl));
        a_own[r] = s_bx[jj + 1] * p.in[DN_EX][o] + ce * curl_x;
        b_own[r] = s_by[ii + 1] * p.in[DN_EY][o] + ce * curl_y;
        if (REC) {
          const long long oc = (long long)(p.t - rec.t0) * rec.stride + o;
          rec.curl[0][oc] = curl_x;
          rec.curl[1][oc] = curl_y;
        }
      }
      s_a[ii][jj] = a_own[r];
      s_b[ii][jj] = b_own[r];
    }
    // ---- halos: Ex at column j0+TJ, Ey at row i0+TI ----------------------
    if (warp == 0 && lane < TI2) {
      const int ii = lane, i = i0 + ii, jh = j0 + TJ2;
      T v = T(0);
      if (jh < W && i < H) {
        const long long o = i * py + jh;
        const T dj = s_f[ii + 1][TJ2 + 1] - s_f[ii + 1][TJ2];
        v = s_bx[TJ2 + 1] * p.in[DN_EX][o] + p.ce[o] * s_gx[TJ2 + 1] * (dj * idl);
      }
      s_a[ii][TJ2] = v;
    } else if (warp == 1) {
      const int ih = i0 + TI2;
      T v = T(0);
      if (ih < H && j < W) {
        const long long o = ih * py + j;
        const T di = s_f[TI2 + 1][jj + 1] - s_f[TI2][jj + 1];
        v = s_by[TI2 + 1] * p.in[DN_EY][o] - p.ce[o] * s_gy[TI2 + 1] * (di * idl);
      }
      s_b[TI2][jj] = v;
    }
  }
  __syncthreads();

  // ---- second update, source, monitors, stores ----------------------------
#pragma unroll
  for (int r = 0; r < R2; ++r) {
    const int ii = warp + 8 * r, i = i0 + ii;
    if (i >= H || j >= W) continue;
    const long long o = i * py + j;
    T v[6];
    const T fo = s_f[ii + 1][jj + 1];
    const T bb = s_bx[jj + 1] * s_by[ii + 1];
    if (POL == DN_TM) {
      const T dHy = (i > 0) ? s_b[ii + 1][jj] - s_b[ii][jj] : T(0);
      const T dHx = (j > 0) ? s_a[ii][jj + 1] - s_a[ii][jj] : T(0);
      const T curl_z = s_gx[jj + 1] * (dHy * idl) - s_gy[ii + 1] * (dHx * idl);
      v[DN_EZ] = bb * fo + p.ce[o] * curl_z;
      if (REC) rec.curl[2][(long long)(p.t - rec.t0) * rec.stride + o] = curl_z;
      v[DN_HX] = a_own[r];
      v[DN_HY] = b_own[r];
      v[DN_HZ] = v[DN_EX] = v[DN_EY] = T(0);
    } else {
      const T dEy = (i < H - 1) ? s_b[ii + 1][jj] - s_b[ii][jj] : T(0);
      const T dEx = (j < W - 1) ? s_a[ii][jj + 1] - s_a[ii][jj] : T(0);
      v[DN_HZ] = bb * fo + dt * (s_gx[jj + 1] * (dEy * idl) - s_gy[ii + 1] * (dEx * idl));
      v[DN_EX] = a_own[r];
      v[DN_EY] = b_own[r];
      v[DN_EZ] = v[DN_HX] = v[DN_HY] = T(0);
    }
    inject_source(p, 0, i, j, v);
    if (p.n_mon) accumulate_monitors(p, 0, i, j, v);
    record_probe(p, 0, i, j, v);
    if (POL == DN_TM) {
      p.out[DN_EZ][o] = v[DN_EZ];
      p.out[DN_HX][o] = v[DN_HX];
      p.out[DN_HY][o] = v[DN_HY];
    } else {
      p.out[DN_HZ][o] = v[DN_HZ];
      p.out[DN_EX][o] = v[DN_EX];
      p.out[DN_EY][o] = v[DN_EY];
    }
  }
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
  const dim3 grid((g->W + TJ2 - 1) / TJ2, (g->H + TI2 - 1) / TI2);
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    set_io(&p, even ? fa : fb, even ? fb : fa);
    p.t = t0 + n;
    if (g->pol == DN_TM) {
      if (record)
        k_fdtd2d_step<T, DN_TM, true><<<grid, NT2, 0, s>>>(p, rec);
      else
        k_fdtd2d_step<T, DN_TM, false><<<grid, NT2, 0, s>>>(p, rec);
    } else {
      if (record)
        k_fdtd2d_step<T, DN_TE, true><<<grid, NT2, 0, s>>>(p, rec);
      else
        k_fdtd2d_step<T, DN_TE, false><<<grid, NT2, 0, s>>>(p, rec);
    }
  }
  DN_CUDA_CHECK(cudaGetLastError());
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
