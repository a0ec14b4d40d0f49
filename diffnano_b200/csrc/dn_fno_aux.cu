// Memory-bound helper kernels of the Fourier-neural-operator surrogate (the
// contractions themselves run on the tcgen05 GEMM in dn_gemm.cu):
//   * input features from a permittivity map, and their gradient back to eps
//   * the readout that collapses the field's row axis with learned per-row,
//     per-channel weights, and its backward pass
//   * deterministic column sums (bias gradients, reductions of per-sample
//     weight-gradient partials)
//   * mean-squared-error loss with its BF16 gradient
//   * Adam on an FP32 master copy with a BF16 mirror
//   * packing of the complex per-mode weights into the real 2x2 block form the
//     mixing GEMM reads, and the matching gradient unpacking
// Activations are channel-first (sample, channel, row, column) unless stated.
#include <cuda_bf16.h>

#include "dn_common.cuh"
#include "dn_fno.h"

namespace dn {
namespace fa {

__device__ __forceinline__ float bf2f(unsigned short h) {
  return __uint_as_float(static_cast<uint32_t>(h) << 16);
}
__device__ __forceinline__ unsigned short f2bf(float v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

constexpr int FEAT = 8;  // features per pixel: eps (normalised), x, y, 5 zeros

__global__ void k_features(const float* __restrict__ eps, long long n_img, int H, int W,
                           float lo, float inv_span, unsigned short* __restrict__ feat) {
  const long long n = n_img * H * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const int h = (int)((i / W) % H);
    const float f0 = (eps[i] - lo) * inv_span;
    const float fx = W > 1 ? (float)w / (float)(W - 1) : 0.0f;
    const float fy = H > 1 ? (float)h / (float)(H - 1) : 0.0f;
    uint4 u;
    u.x = (uint32_t)f2bf(f0) | ((uint32_t)f2bf(fx) << 16);
    u.y = (uint32_t)f2bf(fy);
    u.z = 0u;
    u.w = 0u;
    reinterpret_cast<uint4*>(feat)[i] = u;
  }
}

__global__ void k_features_bwd(const float* __restrict__ dfeat, long long n, float inv_span,
                               float* __restrict__ deps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    deps[i] = dfeat[i * FEAT] * inv_span;
}

// x0[b, c, p] = bf16(sum_k P[c, k] * feat[b, p, k] + bias[c]) (the lifting
// layer; K = FEAT = 8).  One thread per 8 consecutive pixels of one sample:
// the 8 feature rows are read once (128 bytes), then every channel's 8
// outputs go out as one 16-byte store, so a warp writes 512 contiguous bytes
// per channel.  The BF16 products are exact in FP32 and are summed in FP32,
// as the tensor-core path does.  `vec`: n_pix is a multiple of 8.
template <bool VEC>
__global__ void k_lift(const unsigned short* __restrict__ feat,
                       const unsigned short* __restrict__ P, const float* __restrict__ bias,
                       long long nb, long long n_pix, int C, unsigned short* __restrict__ x0) {
  extern __shared__ float s_lift[];  // P as FP32 (C x FEAT), then bias (C)
  for (int e = threadIdx.x; e < C * FEAT; e += blockDim.x) s_lift[e] = bf2f(P[e]);
  for (int e = threadIdx.x; e < C; e += blockDim.x) s_lift[C * FEAT + e] = bias[e];
  __syncthreads();
  const long long groups = (n_pix + 7) / 8;
  const long long n = nb * groups;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / groups;
    const long long p0 = (i % groups) * 8;
    const int np = (int)(n_pix - p0 < 8 ? n_pix - p0 : 8);
    float f[8][FEAT];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      uint4 u = make_uint4(0u, 0u, 0u, 0u);
      if (q < np) u = reinterpret_cast<const uint4*>(feat)[b * n_pix + p0 + q];
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        f[q][2 * e] = __uint_as_float(w[e] << 16);
        f[q][2 * e + 1] = __uint_as_float(w[e] & 0xFFFF0000u);
      }
    }
    unsigned short* out = x0 + b * (long long)C * n_pix + p0;
    for (int c = 0; c < C; ++c) {
      const float* pc = s_lift + c * FEAT;
      const float bc = s_lift[C * FEAT + c];
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < FEAT; ++k) acc = fmaf(pc[k], f[q][k], acc);
        v[q] = acc + bc;
      }
      unsigned short* o = out + (long long)c * n_pix;
      if (VEC) {
        uint4 u;
        u.x = (uint32_t)f2bf(v[0]) | ((uint32_t)f2bf(v[1]) << 16);
        u.y = (uint32_t)f2bf(v[2]) | ((uint32_t)f2bf(v[3]) << 16);
        u.z = (uint32_t)f2bf(v[4]) | ((uint32_t)f2bf(v[5]) << 16);
        u.w = (uint32_t)f2bf(v[6]) | ((uint32_t)f2bf(v[7]) << 16);
        *reinterpret_cast<uint4*>(o) = u;
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < np) o[q] = f2bf(v[q]);
      }
    }
  }
}

// out[b, w, c] = sum_h r[h, c] * x[b, c, h, w]; one thread per (b, c, w)
// (x channel-first, out channel-last)
__global__ void k_readout(const unsigned short* __restrict__ x, const float* __restrict__ r,
                          long long nb, int H, int W, int C, unsigned short* __restrict__ out) {
  const long long n = nb * C * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const int c = (int)((i / W) % C);
    const long long b = i / ((long long)W * C);
    const unsigned short* xp = x + (b * C + c) * (long long)H * W + w;
    float s = 0.0f;
    for (int h = 0; h < H; ++h) s = fmaf(r[h * C + c], bf2f(xp[(long long)h * W]), s);
    out[(b * W + w) * C + c] = f2bf(s);
  }
}

// the same with four consecutive columns w per thread (W % 4 == 0, x 8-byte
// aligned): 8-byte loads, a warp reads 256 contiguous bytes per row h
__global__ void k_readout4(const unsigned short* __restrict__ x, const float* __restrict__ r,
                           long long nb, int H, int W, int C, unsigned short* __restrict__ out) {
  const int W4 = W / 4;
  const long long n = nb * C * W4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w0 = (int)(i % W4) * 4;
    const int c = (int)((i / W4) % C);
    const long long b = i / ((long long)W4 * C);
    const unsigned short* xp = x + (b * C + c) * (long long)H * W + w0;
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
#pragma unroll 4
    for (int h = 0; h < H; ++h) {
      const uint2 u = *reinterpret_cast<const uint2*>(xp + (long long)h * W);
      const float rv = r[h * C + c];
      s0 = fmaf(rv, __uint_as_float(u.x << 16), s0);
      s1 = fmaf(rv, __uint_as_float(u.x & 0xFFFF0000u), s1);
      s2 = fmaf(rv, __uint_as_float(u.y << 16), s2);
      s3 = fmaf(rv, __uint_as_float(u.y & 0xFFFF0000u), s3);
    }
    unsigned short* o = out + (b * W + w0) * C + c;
    o[0] = f2bf(s0);
    o[C] = f2bf(s1);
    o[2 * C] = f2bf(s2);
    o[3 * C] = f2bf(s3);
  }
}

// readout backward, one block per (b, c): dR[b, :, c] staged in shared memory,
//   dx[b, c, h, w] = r[h, c] * dR[b, w, c]                       (dx != NULL)
//   dr_part[b, h, c] = sum_w dR[b, w, c] * x[b, c, h, w]         (dr_part != NULL)
// warps over rows h, lanes over w (x and dx rows are contiguous)
__global__ void k_readout_bwd(const unsigned short* __restrict__ x, const float* __restrict__ r,
                              const unsigned short* __restrict__ dR, int nb, int H, int W, int C,
                              unsigned short* __restrict__ dx, float* __restrict__ dr_part) {
  extern __shared__ float s_dr[];  // W
  const int c = blockIdx.x % C;
  const long long b = blockIdx.x / C;
  for (int w = threadIdx.x; w < W; w += blockDim.x) s_dr[w] = bf2f(dR[(b * W + w) * C + c]);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long base = (b * C + c) * (long long)H * W;
  for (int h = warp; h < H; h += nw) {
    const float rv = r[h * C + c];
    const unsigned short* xr = x + base + (long long)h * W;
    float acc = 0.0f;
    for (int w = lane; w < W; w += 32) {
      const float d = s_dr[w];
      if (dr_part) acc = fmaf(d, bf2f(xr[w]), acc);
      if (dx) dx[base + (long long)h * W + w] = f2bf(rv * d);
    }
    if (dr_part) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) dr_part[(b * H + h) * C + c] = acc;
    }
  }
}

// blockdiag(W, W) and blockdiag(W^T, W^T) (2C x 2C, BF16) and [b, b]
__global__ void k_pack_pointwise(const float* __restrict__ Wm, const float* __restrict__ bias,
                                 int C, unsigned short* __restrict__ blk,
                                 unsigned short* __restrict__ blkT, float* __restrict__ bias2) {
  const int n = 4 * C * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = i / (2 * C), q = i % (2 * C);
    const bool diag = (r < C) == (q < C);
    const int rr = r % C, qq = q % C;
    blk[i] = f2bf(diag ? Wm[rr * C + qq] : 0.0f);
    blkT[i] = f2bf(diag ? Wm[qq * C + rr] : 0.0f);
    if (i < 2 * C) bias2[i] = bias[i % C];
  }
}

// channel sums, pass 1: block (c, q) sums samples q, q + 256, ... of channel c
__global__ void k_channel_part(const unsigned short* __restrict__ x, long long nb, int C,
                               long long npix, float* __restrict__ part) {
  __shared__ float s_w[8];
  const int c = blockIdx.x, q = blockIdx.y;
  float s = 0.0f;
  for (long long b = q; b < nb; b += gridDim.y) {
    const uint4* row = reinterpret_cast<const uint4*>(x + (b * C + c) * npix);
    for (long long i = threadIdx.x; i < npix / 8; i += blockDim.x) {
      const uint4 u = row[i];
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        s += __uint_as_float(w[e] << 16) + __uint_as_float(w[e] & 0xFFFF0000u);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < 8; ++w) t += s_w[w];
    part[q * C + c] = t;
  }
}

// mode-major <-> row-major spectra:
//   modes (m, b, r, c): ((m * nb + b) * 2 + r) * C + c
//   rows  (b, c, r, m): ((b * C + c) * 2 + r) * nm + m
// tiled 32 x 32 transpose of the (m, c) plane of every (b, r)
__global__ void k_modes_rows(const unsigned short* __restrict__ src, unsigned short* __restrict__ dst,
                             int nm, long long nb, int C, int to_rows) {
  __shared__ unsigned short tile[32][33];
  const long long br = blockIdx.z;
  const long long b = br >> 1;
  const int r = (int)(br & 1);
  const int m0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  if (to_rows) {
    for (int k = ty; k < 32; k += 8) {  // read rows m, columns c
      const int m = m0 + k, c = c0 + tx;
      if (m < nm && c < C) tile[k][tx] = src[((m * nb + b) * 2 + r) * C + c];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {  // write rows c, columns m
      const int c = c0 + k, m = m0 + tx;
      if (m < nm && c < C) dst[((b * C + c) * 2 + r) * nm + m] = tile[tx][k];
    }
  } else {
    for (int k = ty; k < 32; k += 8) {  // read rows c, columns m
      const int c = c0 + k, m = m0 + tx;
      if (m < nm && c < C) tile[k][tx] = src[((b * C + c) * 2 + r) * nm + m];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {  // write rows m, columns c
      const int m = m0 + k, c = c0 + tx;
      if (m < nm && c < C) dst[((m * nb + b) * 2 + r) * C + c] = tile[tx][k];
    }
  }
}

// The same permutation on 64 x 64 tiles with two elements (4 bytes) per lane
// on both sides, so a warp moves 128 contiguous bytes per instruction (the
// 32 x 32 kernel above moves 64).  nm and C even, pointers 4-byte aligned.
// Shared tile rows of 66 elements: the 4-byte stores of the read side are
// aligned and conflict-free; the 2-byte loads of the write side conflict at
// most 2-way.
__global__ void k_modes_rows64(const unsigned short* __restrict__ src,
                               unsigned short* __restrict__ dst, int nm, long long nb, int C,
                               int to_rows) {
  __shared__ __align__(16) unsigned short tile[64][66];
  const long long br = blockIdx.z;
  const long long b = br >> 1;
  const int r = (int)(br & 1);
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  // tile rows are the source's rows (m when to_rows, else c; grid x), tile
  // columns the other index (grid y)
  const int a0 = blockIdx.x * 64;  // source row index base
  const int e0 = blockIdx.y * 64;  // source column index base
  const int na = to_rows ? nm : C, ne = to_rows ? C : nm;
  for (int k = ty; k < 64; k += 8) {
    const int a = a0 + k, e = e0 + 2 * tx;
    uint32_t u = 0u;
    if (a < na && e < ne) {
      const long long off = to_rows ? ((a * nb + b) * 2 + r) * (long long)C + e
                                    : ((b * C + a) * 2 + r) * (long long)nm + e;
      u = *reinterpret_cast<const uint32_t*>(src + off);
    }
    *reinterpret_cast<uint32_t*>(&tile[k][2 * tx]) = u;
  }
  __syncthreads();
  for (int k = ty; k < 64; k += 8) {
    const int e = e0 + k, a = a0 + 2 * tx;  // destination row e, columns a, a+1
    if (e < ne && a < na) {
      const uint32_t u = (uint32_t)tile[2 * tx][k] | ((uint32_t)tile[2 * tx + 1][k] << 16);
      const long long off = to_rows ? ((b * C + e) * 2 + r) * (long long)nm + a
                                    : ((e * nb + b) * 2 + r) * (long long)C + a;
      *reinterpret_cast<uint32_t*>(dst + off) = u;
    }
  }
}

// column sums, pass 1: block (bx, by) sums rows [by*rpb, (by+1)*rpb) of
// columns bx*256 + threadIdx.x into part[by, col]
__global__ void k_colsum_part(const void* __restrict__ in, int bf16, long long rows,
                              long long cols, long long ld, long long rpb,
                              float* __restrict__ part) {
  const long long col = blockIdx.x * 256LL + threadIdx.x;
  if (col >= cols) return;
  const long long r0 = blockIdx.y * rpb;
  const long long r1 = r0 + rpb < rows ? r0 + rpb : rows;
  float s = 0.0f;
  if (bf16) {
    const unsigned short* p = static_cast<const unsigned short*>(in);
    for (long long r = r0; r < r1; ++r) s += bf2f(p[r * ld + col]);
  } else {
    const float* p = static_cast<const float*>(in);
    for (long long r = r0; r < r1; ++r) s += p[r * ld + col];
  }
  part[blockIdx.y * cols + col] = s;
}

// pass 2: out[col] (+)= sum over the parts, in order
// pass 2: block (32 x 8) per 32 columns; warp w sums partial rows w, w+8,
// w+16, ... of its lane's column, then the 8 warp sums are added in warp
// order (fixed partition and order: deterministic)
__global__ void k_colsum_final(const float* __restrict__ part, long long nparts, long long cols,
                               float* __restrict__ out, int accumulate) {
  __shared__ float s_w[8][33];
  const long long col = blockIdx.x * 32LL + threadIdx.x;
  const int w = threadIdx.y;
  float s = 0.0f;
  if (col < cols)
    for (long long q = w; q < nparts; q += 8) s += part[q * cols + col];
  s_w[w][threadIdx.x] = s;
  __syncthreads();
  if (w == 0 && col < cols) {
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += s_w[k][threadIdx.x];
    out[col] = accumulate ? out[col] + t : t;
  }
}

// MSE over the first `used` of `ld` columns; grad = scale * 2 (pred - target)
// as BF16 (padding columns zero); per-block partial losses in double
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ target,
                      long long rows, int ld, int used, float gscale,
                      unsigned short* __restrict__ grad, double* __restrict__ part) {
  __shared__ double s_w[8];
  double acc = 0.0;
  const long long n = rows * ld;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const int c = (int)(i % ld);
    float g = 0.0f;
    if (c < used) {
      const float d = pred[i] - target[i];
      acc += (double)d * (double)d;
      g = 2.0f * d * gscale;
    }
    grad[i] = f2bf(g);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += s_w[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2,
                       float eps, float bc1, float bc2, float wd,
                       unsigned short* __restrict__ mirror) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / bc1, vh = vi / bc2;
    const float pi = p[i] - lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
    p[i] = pi;
    if (mirror) mirror[i] = f2bf(pi);
  }
}

// blk[m, (ro, o), (ri, i)] for ro, ri in {0, 1} (real, imaginary):
//   [[wre, -wim], [wim, wre]] so that [yre; yim] = blk [zre; zim]
// one thread per two consecutive inputs i of one (m, o): reads the two complex
// weights once and writes the four 2x2-block entries of both as BF16 pairs
// (ci even; the odd-ci kernel below writes element by element)
__global__ void k_pack_modes2(const float* __restrict__ wre, const float* __restrict__ wim,
                              long long nm, int co, int ci, unsigned int* __restrict__ blk2) {
  const int hc = ci / 2;
  const long long n = nm * co * hc;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i2 = (int)(idx % hc);
    const long long mo = idx / hc;  // m * co + o
    const int o = (int)(mo % co);
    const long long m = mo / co;
    const long long w = mo * ci + 2 * i2;
    const float re0 = wre[w], re1 = wre[w + 1], im0 = wim[w], im1 = wim[w + 1];
    const uint32_t pre = (uint32_t)f2bf(re0) | ((uint32_t)f2bf(re1) << 16);
    const uint32_t pim = (uint32_t)f2bf(im0) | ((uint32_t)f2bf(im1) << 16);
    const uint32_t nim = (uint32_t)f2bf(-im0) | ((uint32_t)f2bf(-im1) << 16);
    // rows o (real out) and co + o (imaginary out) of mode m, in pairs of columns
    const long long top = ((m * 2 * co + o) * 2 * ci) / 2;
    const long long bot = ((m * 2 * co + co + o) * 2 * ci) / 2;
    blk2[top + i2] = pre;       // [wre, ...
    blk2[top + hc + i2] = nim;  //  ..., -wim]
    blk2[bot + i2] = pim;       // [wim, ...
    blk2[bot + hc + i2] = pre;  //  ..., wre]
  }
}

__global__ void k_pack_modes(const float* __restrict__ wre, const float* __restrict__ wim,
                             long long nm, int co, int ci, unsigned short* __restrict__ blk) {
  const long long n = nm * 2 * co * 2 * ci;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int col = (int)(idx % (2 * ci));
    const int row = (int)((idx / (2 * ci)) % (2 * co));
    const long long m = idx / ((long long)4 * co * ci);
    const int ri = col / ci, i = col % ci, ro = row / co, o = row % co;
    const long long w = (m * co + o) * ci + i;
    float val;
    if (ro == ri)
      val = wre[w];
    else
      val = ro == 0 ? -wim[w] : wim[w];
    blk[idx] = f2bf(val);
  }
}

__global__ void k_unpack_mode_grads(const float* __restrict__ dblk, long long nm, int co, int ci,
                                    float* __restrict__ dwre, float* __restrict__ dwim) {
  const long long n = nm * co * ci;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % ci);
    const int o = (int)((idx / ci) % co);
    const long long m = idx / ((long long)co * ci);
    const float* b = dblk + m * 4LL * co * ci;
    const long long ld = 2LL * ci;
    dwre[idx] = b[o * ld + i] + b[(co + o) * ld + ci + i];
    dwim[idx] = b[(co + o) * ld + i] - b[o * ld + ci + i];
  }
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, long long n,
                              unsigned short* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = f2bf(in[i]);
}

unsigned grid_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  const long long cap = 148LL * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace fa
}  // namespace dn

using namespace dn::fa;

extern "C" int32_t dn_fno_features(const float* eps, int64_t n_img, int32_t H, int32_t W,
                                   float eps_lo, float eps_hi, void* feat, void* stream) {
  if (!eps || !feat || n_img < 1 || H < 1 || W < 1 || !(eps_hi > eps_lo) || !al16(feat))
    return DN_EINVAL;
  const long long n = n_img * (long long)H * W;
  k_features<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      eps, n_img, H, W, eps_lo, 1.0f / (eps_hi - eps_lo), static_cast<unsigned short*>(feat));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_features_bwd(const float* dfeat, int64_t n_pix, float eps_lo,
                                       float eps_hi, float* deps, void* stream) {
  if (!dfeat || !deps || n_pix < 1 || !(eps_hi > eps_lo)) return DN_EINVAL;
  k_features_bwd<<<grid_for(n_pix), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dfeat, n_pix, 1.0f / (eps_hi - eps_lo), deps);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_lift(const void* feat, const void* P, const float* bias, int64_t nb,
                               int64_t n_pix, int32_t C, void* x0, void* stream) {
  if (!feat || !P || !bias || !x0 || nb < 1 || n_pix < 1 || C < 1 || C > 1024 || !al16(feat) ||
      !al16(x0))
    return DN_EINVAL;
  const long long n = nb * ((n_pix + 7) / 8);
  const size_t smem = (size_t)C * (FEAT + 1) * sizeof(float);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* fp = static_cast<const unsigned short*>(feat);
  const auto* pp = static_cast<const unsigned short*>(P);
  auto* xp = static_cast<unsigned short*>(x0);
  if (n_pix % 8 == 0)
    k_lift<true><<<grid_for(n), 256, smem, s>>>(fp, pp, bias, nb, n_pix, C, xp);
  else
    k_lift<false><<<grid_for(n), 256, smem, s>>>(fp, pp, bias, nb, n_pix, C, xp);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_readout(const void* x, const float* r, int64_t nb, int32_t H,
                                  int32_t W, int32_t C, void* out, void* stream) {
  if (!x || !r || !out || nb < 1 || H < 1 || W < 1 || C < 1) return DN_EINVAL;
  if (W % 4 == 0 && (reinterpret_cast<uintptr_t>(x) & 7) == 0) {
    k_readout4<<<grid_for(nb * C * (W / 4)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const unsigned short*>(x), r, nb, H, W, C, static_cast<unsigned short*>(out));
    DN_CUDA_CHECK(cudaGetLastError());
    return DN_OK;
  }
  k_readout<<<grid_for(nb * C * W), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const unsigned short*>(x), r, nb, H, W, C, static_cast<unsigned short*>(out));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_readout_bwd(const void* x, const float* r, const void* dR, int64_t nb,
                                      int32_t H, int32_t W, int32_t C, void* dx, float* dr_part,
                                      void* stream) {
  if (!x || !r || !dR || nb < 1 || H < 1 || W < 1 || C < 1 || (!dx && !dr_part))
    return DN_EINVAL;
  if (nb * C > 0x7fffffffLL || W > 12 * 1024) return DN_EUNSUPPORTED;
  k_readout_bwd<<<(unsigned)(nb * C), 256, W * sizeof(float),
                  static_cast<cudaStream_t>(stream)>>>(
      static_cast<const unsigned short*>(x), r, static_cast<const unsigned short*>(dR), (int)nb, H,
      W, C, static_cast<unsigned short*>(dx), dr_part);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int64_t dn_colsum_scratch_elems(int64_t rows, int64_t cols) {
  if (rows < 1 || cols < 1) return 0;
  const long long parts = rows < 512 ? rows : 512;
  return parts * cols;
}

extern "C" int32_t dn_colsum(const void* in, int32_t dtype, int64_t rows, int64_t cols, int64_t ld,
                             float* out, int32_t accumulate, float* scratch, int64_t scratch_elems,
                             void* stream) {
  if (!in || !out || !scratch || rows < 1 || cols < 1 || ld < cols) return DN_EINVAL;
  if (dtype != DN_F32 && dtype != DN_BF16) return DN_EINVAL;
  const long long parts = rows < 512 ? rows : 512;
  if (scratch_elems < parts * cols) return DN_EINVAL;
  const long long rpb = (rows + parts - 1) / parts;
  const long long nparts = (rows + rpb - 1) / rpb;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 g1((unsigned)((cols + 255) / 256), (unsigned)nparts);
  k_colsum_part<<<g1, 256, 0, s>>>(in, dtype == DN_BF16, rows, cols, ld, rpb, scratch);
  DN_CUDA_CHECK(cudaGetLastError());
  k_colsum_final<<<(unsigned)((cols + 31) / 32), dim3(32, 8), 0, s>>>(scratch, nparts, cols, out,
                                                                        accumulate);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_mse(const float* pred, const float* target, int64_t rows, int32_t ld,
                          int32_t used, float grad_scale, void* grad, double* loss_part,
                          int32_t n_part, void* stream) {
  if (!pred || !target || !grad || !loss_part || rows < 1 || ld < 1 || used < 1 || used > ld ||
      n_part < 1)
    return DN_EINVAL;
  k_mse<<<n_part, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      pred, target, rows, ld, used, grad_scale, static_cast<unsigned short*>(grad), loss_part);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr,
                           float beta1, float beta2, float eps, int32_t step, float weight_decay,
                           void* mirror_bf16, void* stream) {
  if (!p || !g || !m || !v || n < 1 || step < 1) return DN_EINVAL;
  const float bc1 = 1.0f - powf(beta1, (float)step);
  const float bc2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, n, lr, beta1, beta2, eps, bc1, bc2, weight_decay,
      static_cast<unsigned short*>(mirror_bf16));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_pack_modes(const float* wre, const float* wim, int64_t n_modes,
                                     int32_t c_out, int32_t c_in, void* blk, void* stream) {
  if (!wre || !wim || !blk || n_modes < 1 || c_out < 1 || c_in < 1) return DN_EINVAL;
  if (c_in % 2 == 0 && (reinterpret_cast<uintptr_t>(blk) & 3) == 0) {
    k_pack_modes2<<<grid_for(n_modes * (long long)c_out * (c_in / 2)), 256, 0,
                    static_cast<cudaStream_t>(stream)>>>(wre, wim, n_modes, c_out, c_in,
                                                         static_cast<unsigned int*>(blk));
    DN_CUDA_CHECK(cudaGetLastError());
    return DN_OK;
  }
  k_pack_modes<<<grid_for(n_modes * 4LL * c_out * c_in), 256, 0,
                 static_cast<cudaStream_t>(stream)>>>(wre, wim, n_modes, c_out, c_in,
                                                      static_cast<unsigned short*>(blk));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_unpack_mode_grads(const float* dblk, int64_t n_modes, int32_t c_out,
                                            int32_t c_in, float* dwre, float* dwim,
                                            void* stream) {
  if (!dblk || !dwre || !dwim || n_modes < 1 || c_out < 1 || c_in < 1) return DN_EINVAL;
  k_unpack_mode_grads<<<grid_for(n_modes * (long long)c_out * c_in), 256, 0,
                        static_cast<cudaStream_t>(stream)>>>(dblk, n_modes, c_out, c_in, dwre,
                                                             dwim);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_f32_to_bf16(const float* in, int64_t n, void* out, void* stream) {
  if (!in || !out || n < 1) return DN_EINVAL;
  k_f32_to_bf16<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      in, n, static_cast<unsigned short*>(out));
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_modes_rows(const void* src, void* dst, int32_t n_modes, int64_t nb,
                                     int32_t C, int32_t to_rows, void* stream) {
  if (!src || !dst || src == dst || n_modes < 1 || nb < 1 || C < 1) return DN_EINVAL;
  if (nb * 2 > 65535) return DN_EUNSUPPORTED;
  if (n_modes % 2 == 0 && C % 2 == 0 && (reinterpret_cast<uintptr_t>(src) & 3) == 0 &&
      (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
    // grid x covers the source rows, y the source columns
    const int na = to_rows ? n_modes : C, ne = to_rows ? C : n_modes;
    const dim3 g64((unsigned)((na + 63) / 64), (unsigned)((ne + 63) / 64), (unsigned)(nb * 2));
    k_modes_rows64<<<g64, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const unsigned short*>(src), static_cast<unsigned short*>(dst), n_modes, nb,
        C, to_rows != 0);
    DN_CUDA_CHECK(cudaGetLastError());
    return DN_OK;
  }
  const dim3 grid((unsigned)((n_modes + 31) / 32), (unsigned)((C + 31) / 32), (unsigned)(nb * 2));
  k_modes_rows<<<grid, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const unsigned short*>(src), static_cast<unsigned short*>(dst), n_modes, nb, C,
      to_rows != 0);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_channel_sums(const void* x, int64_t nb, int32_t C, int64_t n_pix,
                                       float* out, float* scratch, void* stream) {
  if (!x || !out || !scratch || nb < 1 || C < 1 || n_pix < 8 || n_pix % 8 || !al16(x))
    return DN_EINVAL;
  if (C > 65535) return DN_EUNSUPPORTED;
  const int parts = nb < 256 ? (int)nb : 256;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_channel_part<<<dim3((unsigned)C, (unsigned)parts), 256, 0, s>>>(
      static_cast<const unsigned short*>(x), nb, C, n_pix, scratch);
  DN_CUDA_CHECK(cudaGetLastError());
  k_colsum_final<<<(unsigned)((C + 31) / 32), dim3(32, 8), 0, s>>>(scratch, parts, C, out, 0);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_fno_pack_pointwise(const float* Wm, const float* bias, int32_t C, void* blk,
                                         void* blkT, float* bias2, void* stream) {
  if (!Wm || !bias || !blk || !blkT || !bias2 || C < 1) return DN_EINVAL;
  k_pack_pointwise<<<grid_for(4LL * C * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      Wm, bias, C, static_cast<unsigned short*>(blk), static_cast<unsigned short*>(blkT), bias2);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}
