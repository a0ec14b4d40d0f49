// Design-layer kernels: density -> permittivity for the inverse-design loop.
//
//   rho (n_layers, H, W) --Gaussian filter in each layer--> rho_f
//   rho_f --projection--> p in (0, 1) --> eps = lo + (hi - lo) * p
//
// The filter is separable (a pass along x, then one along y) with the taps of
// the reference's smooth_filter (kernel 2r+1 rounded up to odd, sigma = r/2,
// normalised, zero padding).  Projections: the reference's sigmoid
// Heaviside, and the tanh projection
//   p = (tanh(beta eta) + tanh(beta (x - eta))) / (tanh(beta eta) + tanh(beta (1 - eta))).
// The backward pass maps d eps to d rho: the projection's derivative, then the
// same separable filter (its kernel is symmetric and zero padded, so the
// filter is its own transpose).  Erosion / dilation are 3x3 min / max pools
// per layer (cells outside the layer ignored) whose backward pass is a gather:
// every input adds the output gradients of the windows that selected it, in a
// fixed order, so results are deterministic.
#include "dn_common.cuh"
#include "dn_design.h"

namespace dn {
namespace ds {

constexpr int MAX_TAPS = 63;

struct Taps {
  float t[MAX_TAPS];
  int n;
};

__global__ void k_filter_axis(const float* __restrict__ in, float* __restrict__ out, long long nl,
                              int H, int W, int axis_x, const Taps taps) {
  const long long n = nl * H * W;
  const int c = taps.n / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const int h = (int)((i / W) % H);
    const long long base = i - (axis_x ? w : (long long)h * W);
    const int pos = axis_x ? w : h;
    const int len = axis_x ? W : H;
    const long long stride = axis_x ? 1 : W;
    float s = 0.0f;
    for (int t = 0; t < taps.n; ++t) {
      const int q = pos + t - c;
      if (q >= 0 && q < len) s = fmaf(taps.t[t], in[base + q * stride], s);
    }
    out[i] = s;
  }
}

__device__ __forceinline__ float project(float x, int kind, float beta, float eta, float den,
                                         float off) {
  if (kind == DN_PROJ_NONE) return x;
  if (kind == DN_PROJ_SIGMOID) return 1.0f / (1.0f + expf(-beta * (x - eta)));
  return (off + tanhf(beta * (x - eta))) / den;
}

__device__ __forceinline__ float project_grad(float x, int kind, float beta, float eta,
                                              float den) {
  if (kind == DN_PROJ_NONE) return 1.0f;
  if (kind == DN_PROJ_SIGMOID) {
    const float s = 1.0f / (1.0f + expf(-beta * (x - eta)));
    return beta * s * (1.0f - s);
  }
  const float t = tanhf(beta * (x - eta));
  return beta * (1.0f - t * t) / den;
}

__global__ void k_project(const float* __restrict__ xf, long long n, int kind, float beta,
                          float eta, float den, float off, float lo, float span,
                          float* __restrict__ eps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    eps[i] = lo + span * project(xf[i], kind, beta, eta, den, off);
}

__global__ void k_project_bwd(const float* __restrict__ xf, const float* __restrict__ deps,
                              long long n, int kind, float beta, float eta, float den,
                              float span, float* __restrict__ dxf) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dxf[i] = deps[i] * span * project_grad(xf[i], kind, beta, eta, den);
}

// 3x3 pool per layer; arg = flat index of the selected input (first extremum
// in row-major window order, as max_pool2d keeps the first maximum)
__global__ void k_morph3(const float* __restrict__ x, long long nl, int H, int W, int dilate,
                         float* __restrict__ y, int* __restrict__ arg) {
  const long long n = nl * H * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i % W);
    const int h = (int)((i / W) % H);
    const long long layer = i - (long long)h * W - w;
    float best = 0.0f;
    long long bi = -1;
    for (int dh = -1; dh <= 1; ++dh) {
      const int hh = h + dh;
      if (hh < 0 || hh >= H) continue;
      for (int dw = -1; dw <= 1; ++dw) {
        const int ww = w + dw;
        if (ww < 0 || ww >= W) continue;
        const long long j = layer + (long long)hh * W + ww;
        const float v = x[j];
        const bool better = dilate ? v > best : v < best;
        if (bi < 0 || better) {
          best = v;
          bi = j;
        }
      }
    }
    y[i] = best;
    arg[i] = (int)(bi - layer);  // index inside the layer
  }
}

// dx[j] = sum of dy[i] over the windows i around j that selected j
__global__ void k_morph3_bwd(const float* __restrict__ dy, const int* __restrict__ arg,
                             long long nl, int H, int W, float* __restrict__ dx) {
  const long long n = nl * H * W;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(j % W);
    const int h = (int)((j / W) % H);
    const long long layer = j - (long long)h * W - w;
    const int jin = h * W + w;
    float s = 0.0f;
    for (int dh = -1; dh <= 1; ++dh) {
      const int hh = h + dh;
      if (hh < 0 || hh >= H) continue;
      for (int dw = -1; dw <= 1; ++dw) {
        const int ww = w + dw;
        if (ww < 0 || ww >= W) continue;
        const long long i = layer + (long long)hh * W + ww;
        if (arg[i] == jin) s += dy[i];
      }
    }
    dx[j] = s;
  }
}

unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

// the reference smooth_filter's 1-D taps for `radius`
int make_taps(float radius, Taps* t) {
  if (!(radius >= 0.0f)) return DN_EINVAL;
  int k = (int)(2.0f * radius + 1.0f);
  if (k % 2 == 0) k += 1;
  if (k > MAX_TAPS) return DN_EUNSUPPORTED;
  const double sigma = radius / 2.0;
  double sum = 0.0, v[MAX_TAPS];
  for (int i = 0; i < k; ++i) {
    const double x = i - k / 2;
    v[i] = exp(-(x * x) / (2.0 * sigma * sigma + 1e-12));
    sum += v[i];
  }
  for (int i = 0; i < k; ++i) t->t[i] = (float)(v[i] / sum);
  t->n = k;
  return DN_OK;
}

int check(const dn_density* d) {
  if (!d || d->n_layers < 1 || d->H < 1 || d->W < 1) return DN_EINVAL;
  if (d->kind != DN_PROJ_SIGMOID && d->kind != DN_PROJ_TANH && d->kind != DN_PROJ_NONE)
    return DN_EINVAL;
  if (!(d->beta > 0.0f) || !(d->eps_hi >= d->eps_lo)) return DN_EINVAL;
  if (d->kind == DN_PROJ_TANH && !(d->eta > 0.0f && d->eta < 1.0f)) return DN_EINVAL;
  return DN_OK;
}

void proj_consts(const dn_density* d, float* den, float* off) {
  *off = tanhf(d->beta * d->eta);
  *den = *off + tanhf(d->beta * (1.0f - d->eta));
}

// two filter passes in -> (work) -> out; radius 0 copies
int filter(const dn_density* d, const float* in, float* work, float* out, cudaStream_t s) {
  Taps t;
  int rc = make_taps(d->radius, &t);
  if (rc != DN_OK) return rc;
  const long long n = (long long)d->n_layers * d->H * d->W;
  k_filter_axis<<<grid_for(n), 256, 0, s>>>(in, work, d->n_layers, d->H, d->W, 1, t);
  DN_CUDA_CHECK(cudaGetLastError());
  k_filter_axis<<<grid_for(n), 256, 0, s>>>(work, out, d->n_layers, d->H, d->W, 0, t);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

}  // namespace ds
}  // namespace dn

using namespace dn::ds;

extern "C" int32_t dn_density_forward(const dn_density* d, const float* rho, float* work,
                                      float* filtered, float* eps, void* stream) {
  int rc = check(d);
  if (rc != DN_OK) return rc;
  if (!rho || !work || !filtered || !eps) return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if ((rc = filter(d, rho, work, filtered, s)) != DN_OK) return rc;
  float den, off;
  proj_consts(d, &den, &off);
  const long long n = (long long)d->n_layers * d->H * d->W;
  k_project<<<grid_for(n), 256, 0, s>>>(filtered, n, d->kind, d->beta, d->eta, den, off,
                                        d->eps_lo, d->eps_hi - d->eps_lo, eps);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_density_backward(const dn_density* d, const float* filtered,
                                       const float* deps, float* work, float* drho,
                                       void* stream) {
  int rc = check(d);
  if (rc != DN_OK) return rc;
  if (!filtered || !deps || !work || !drho) return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float den, off;
  proj_consts(d, &den, &off);
  const long long n = (long long)d->n_layers * d->H * d->W;
  // d rho_f = d eps * (hi - lo) * p'(rho_f) into drho, then the two filter
  // passes (x and y commute) through `work` back into drho
  k_project_bwd<<<grid_for(n), 256, 0, s>>>(filtered, deps, n, d->kind, d->beta, d->eta, den,
                                            d->eps_hi - d->eps_lo, drho);
  DN_CUDA_CHECK(cudaGetLastError());
  if ((rc = filter(d, drho, work, drho, s)) != DN_OK) return rc;
  return DN_OK;
}

extern "C" int32_t dn_morph3(const float* x, int32_t n_layers, int32_t H, int32_t W,
                             int32_t dilate, float* y, int32_t* arg, void* stream) {
  if (!x || !y || !arg || n_layers < 1 || H < 1 || W < 1) return DN_EINVAL;
  if ((long long)H * W > 0x7fffffffLL) return DN_EUNSUPPORTED;
  const long long n = (long long)n_layers * H * W;
  k_morph3<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, n_layers, H, W,
                                                                       dilate != 0, y, arg);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

extern "C" int32_t dn_morph3_backward(const float* dy, const int32_t* arg, int32_t n_layers,
                                      int32_t H, int32_t W, float* dx, void* stream) {
  if (!dy || !arg || !dx || n_layers < 1 || H < 1 || W < 1) return DN_EINVAL;
  const long long n = (long long)n_layers * H * W;
  k_morph3_bwd<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(dy, arg, n_layers, H,
                                                                           W, dx);
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}
