/*
 * dn_fno.h -- C ABI of the surrogate kernels in libdn_fdtd.so: a BF16
 * tensor-core GEMM (sm_100a tcgen05, FP32 accumulation in tensor memory) with
 * a fused epilogue, the building block of the Fourier-neural-operator
 * surrogate's training and inference passes.
 *
 * Same conventions as dn_fdtd.h: raw device pointers, element counts and
 * strides, int status codes (DN_OK ...), asynchronous on the given stream.
 *
 * Reference interfaces replaced (DiffNano, paths relative to its checkout):
 * the reference's surrogate is a small CNN trained with torch ops
 * (diffnano/solvers/surrogate.py:78-285, NeuralSurrogate); it has no Fourier neural
 * operator and no GEMM of its own.  dn_gemm_run is the one compute entry the
 * surrogate's Python layer calls for every contraction of the operator
 * (lifting, truncated 2-D DFT and its inverse, per-mode complex channel
 * mixing, 1x1 channel mixing, readout) and their gradients.
 */
#ifndef DN_FNO_H
#define DN_FNO_H

#include <stdint.h>

#include "dn_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DN_BF16 2 /* element type code next to DN_F32 / DN_F64 */

#define DN_ACT_NONE 0
#define DN_ACT_GELU 1      /* y = gelu(v) (tanh form); `pre` (optional) receives v */
#define DN_ACT_GELU_GRAD 2 /* y = v * gelu'(aux), aux = the pre-activation       */

/* One BF16 operand of C = A * B^T.  Element (r, k), r the row index (M for A,
 * N for B) and k the contraction index, of GEMM batch z is at
 *   K-major  (mn_major = 0): ptr + z*batch_stride + r*ld + k
 *   MN-major (mn_major = 1): ptr + z*batch_stride + (r / fold)*fold_stride
 *                                + k*ld + r % fold       (fold = 0: no fold)
 * Rows r >= rows and k >= k extent read as zero.  ptr is 16-byte aligned;
 * ld, fold_stride and batch_stride are multiples of 8 elements; fold is a
 * multiple of 64; batch_stride = 0 shares the operand across batches. */
typedef struct dn_gemm_operand {
  const void* ptr;
  int32_t mn_major;
  int32_t fold;
  int64_t rows;
  int64_t k;
  int64_t ld;
  int64_t fold_stride;
  int64_t batch_stride;
} dn_gemm_operand;

/* C[z] (M x N) = sum over segments s of A_s[z] * B_s[z]^T  (K_s = a[s].k =
 * b[s].k), then the epilogue, per element (z, r, c):
 *   v = alpha * acc * row_scale[r] * col_scale[c] * batch_scale[z] + bias[c]
 *       + row_bias[r] + addend[z,r,c]
 *   y = v | gelu(v) | v * gelu'(aux[z,r,c])          (act)
 *   out[z,r,c] = y   (or += y when accumulate, FP32 output only)
 * with every optional pointer NULL to skip it.  out, addend, aux and pre
 * share one index map:
 *   off(z, r, c) = z*c_batch_stride + (r % c_row_radix)*c_row_stride0
 *                + (r / c_row_radix)*c_row_stride1
 *                + (c % c_col_radix)*c_col_stride0 + (c / c_col_radix)*c_col_stride1
 * (radix 0 = no split).  c_col_radix, when set, is a multiple of 32, or a
 * divisor of 32 (2 .. 16) for plain stores (no addend, aux, pre, accumulate). */
typedef struct dn_gemm {
  int64_t M;
  int64_t N;
  int32_t batch;
  int32_t n_seg; /* 1 or 2 */
  dn_gemm_operand a[2];
  dn_gemm_operand b[2];
  void* out;
  int32_t out_dtype; /* DN_F32 or DN_BF16 */
  int32_t accumulate;
  int64_t c_batch_stride;
  int64_t c_row_radix;
  int64_t c_row_stride0;
  int64_t c_row_stride1;
  int64_t c_col_radix;
  int64_t c_col_stride0;
  int64_t c_col_stride1;
  float alpha;
  int32_t act;
  const float* bias;
  const float* row_scale;
  const float* batch_scale;
  const void* addend;
  int32_t addend_dtype;
  int32_t aux_dtype;
  const void* aux;
  void* pre;
  int32_t pre_dtype;
  int32_t block_n;  /* 0 = choose; else 64, 128 or 256 */
  int32_t max_ctas; /* 0 = one per SM */
  const float* col_scale;
  const float* row_bias;
  int32_t pair; /* 0 or 1 = one-CTA tiles; 2 = two-CTA 256 x 256 tiles */
} dn_gemm;

/* Persistent warp-specialised kernel: a TMA producer warp (128-byte swizzled
 * 128x64 / block_n x64 tiles), one thread issuing tcgen05.mma (M = 128, K =
 * 16 each) into double-buffered tensor-memory accumulators, eight epilogue
 * warps.  Pair mode (pair = 2) runs two-CTA clusters on 256 x 256 tiles
 * (tcgen05 cta_group::2, M = 256; each CTA loads half the operand bytes).
 * Bounded waits; a wait that gives up stores DN_ETIMEOUT in *status (status
 * may be NULL). */
int32_t dn_gemm_run(const dn_gemm* g, int32_t* status, void* stream);

/* ---- memory-bound helpers of the operator's passes ----------------------
 * BF16 activations are channel-first (sample, channel, row, column). */

/* feat[i, 0..7] = ((eps - lo) / (hi - lo), column / (W-1), row / (H-1), 0 x 5)
 * as BF16 for every pixel of n_img (H, W) FP32 maps; feat 16-byte aligned.
 * Replaces the reference network's input reshaping
 * (diffnano/solvers/surrogate.py:62-72, _SurrogateNet.forward). */
int32_t dn_fno_features(const float* eps, int64_t n_img, int32_t H, int32_t W, float eps_lo,
                        float eps_hi, void* feat, void* stream);
/* deps[i] = dfeat[i, 0] / (hi - lo): dfeat FP32 (n_pix, 8) */
int32_t dn_fno_features_bwd(const float* dfeat, int64_t n_pix, float eps_lo, float eps_hi,
                            float* deps, void* stream);

/* The lifting layer: x0[b, c, p] = sum_k P[c, k] * feat[b, p, k] + bias[c]
 * (feat (nb, n_pix, 8) and P (C, 8) BF16, bias FP32, x0 (nb, C, n_pix) BF16;
 * FP32 sums of the exact BF16 products, as the tensor-core GEMM forms them).
 * A memory-bound kernel in place of a K = 8 GEMM.  feat, x0 16-byte aligned;
 * C <= 1024.  Replaces the input layer of the reference network
 * (diffnano/solvers/surrogate.py:62-72, _SurrogateNet.forward). */
int32_t dn_fno_lift(const void* feat, const void* P, const float* bias, int64_t nb,
                    int64_t n_pix, int32_t C, void* x0, void* stream);

/* out[b, w, c] = sum_h r[h, c] * x[b, c, h, w]   (x, out BF16; r FP32 (H, C)) */
int32_t dn_fno_readout(const void* x, const float* r, int64_t nb, int32_t H, int32_t W,
                       int32_t C, void* out, void* stream);
/* dx[b, c, h, w] = r[h, c] * dR[b, w, c] (BF16; NULL skips) and
 * dr_part[b, h, c] = sum_w dR[b, w, c] * x[b, c, h, w] (FP32; NULL skips) */
int32_t dn_fno_readout_bwd(const void* x, const float* r, const void* dR, int64_t nb, int32_t H,
                           int32_t W, int32_t C, void* dx, float* dr_part, void* stream);

/* out[c] (+)= sum_r in[r * ld + c], deterministic (fixed partition and order).
 * in FP32 or BF16 (dtype); scratch: dn_colsum_scratch_elems(rows, cols) floats. */
int64_t dn_colsum_scratch_elems(int64_t rows, int64_t cols);
int32_t dn_colsum(const void* in, int32_t dtype, int64_t rows, int64_t cols, int64_t ld,
                  float* out, int32_t accumulate, float* scratch, int64_t scratch_elems,
                  void* stream);

/* Squared error over the first `used` of `ld` columns of (rows, ld) FP32
 * prediction and target: grad = grad_scale * 2 * (pred - target) as BF16
 * (zero in the padding columns); loss_part[n_part] receives per-block sums of
 * squares in FP64 (the caller adds them and divides).  Replaces the
 * reference's mse_loss training criterion (diffnano/solvers/surrogate.py:193). */
int32_t dn_mse(const float* pred, const float* target, int64_t rows, int32_t ld, int32_t used,
               float grad_scale, void* grad, double* loss_part, int32_t n_part, void* stream);

/* One Adam step (bias-corrected, decoupled weight decay) over n FP32
 * parameters; writes the BF16 mirror when mirror_bf16 is not NULL.  Replaces
 * torch.optim.Adam in the reference's surrogate training
 * (diffnano/solvers/surrogate.py:128, 195-197). */
int32_t dn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1,
                float beta2, float eps, int32_t step, float weight_decay, void* mirror_bf16,
                void* stream);

/* Complex per-mode weights w = wre + i*wim, (n_modes, c_out, c_in) FP32, to
 * the real block matrix blk (n_modes, 2*c_out, 2*c_in) BF16 =
 * [[wre, -wim], [wim, wre]]; and the gradient of that map. */
int32_t dn_fno_pack_modes(const float* wre, const float* wim, int64_t n_modes, int32_t c_out,
                          int32_t c_in, void* blk, void* stream);
int32_t dn_fno_unpack_mode_grads(const float* dblk, int64_t n_modes, int32_t c_out, int32_t c_in,
                                 float* dwre, float* dwim, void* stream);

/* Kept Fourier modes between the per-mode layout the mixing GEMM reads and
 * writes, (n_modes, nb, 2, C), and the per-channel layout of the transform
 * GEMMs, (nb, C, 2, n_modes) (2 = real, imaginary); to_rows != 0 converts the
 * first to the second.  BF16, src != dst. */
int32_t dn_fno_modes_rows(const void* src, void* dst, int32_t n_modes, int64_t nb, int32_t C,
                          int32_t to_rows, void* stream);

/* out[c] = sum over samples b and pixels p of x[b, c, p] (BF16, channel-first
 * (nb, C, n_pix)), FP32, deterministic; scratch: 256 * C floats. */
int32_t dn_fno_channel_sums(const void* x, int64_t nb, int32_t C, int64_t n_pix, float* out,
                            float* scratch, void* stream);

/* The 1x1 channel mix of two samples at once: blk = blockdiag(W, W), blkT =
 * blockdiag(W^T, W^T) ((2C, 2C) BF16) and bias2 = [bias, bias] (FP32), from
 * W (C, C) and bias (C) FP32. */
int32_t dn_fno_pack_pointwise(const float* W, const float* bias, int32_t C, void* blk, void* blkT,
                              float* bias2, void* stream);

/* out[i] = bf16(in[i]) */
int32_t dn_f32_to_bf16(const float* in, int64_t n, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DN_FNO_H */
