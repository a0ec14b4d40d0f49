/*
 * dn_design.h -- C ABI of the design-layer kernels in libdn_fdtd.so: the map
 * from a density field to the permittivity the FDTD solvers take, and its
 * gradient, for the inverse-design loop.
 *
 * Same conventions as dn_fdtd.h: raw device pointers (FP32), element counts,
 * int status codes, asynchronous on the given stream.  A density field is
 * (n_layers, H, W), W fastest; filters and pools act inside each layer.
 *
 * Reference interfaces replaced (DiffNano, paths relative to its checkout):
 *   dn_density_forward / _backward <- smooth_filter + heaviside_projection
 *       (diffnano/design/projection.py:15-85) applied to a density and mapped
 *       to eps = lo + (hi - lo) * projected; the tanh projection is an
 *       addition (the reference projects with a sigmoid only)
 *   dn_morph3 / _backward <- erosion / dilation as -max_pool2d(-x, 3, 1, 1) /
 *       max_pool2d(x, 3, 1, 1)
 *       (diffnano/design/constraints_shared/primitives.py:56-60)
 */
#ifndef DN_DESIGN_H
#define DN_DESIGN_H

#include <stdint.h>

#include "dn_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DN_PROJ_SIGMOID 0 /* p = sigmoid(beta (x - eta))                          */
#define DN_PROJ_TANH 1    /* p = (tanh(b e) + tanh(b (x - e))) / (tanh(b e) + tanh(b (1 - e))) */
#define DN_PROJ_NONE 2    /* p = x (filter only)                                   */

typedef struct dn_density {
  int32_t n_layers;
  int32_t H;
  int32_t W;
  int32_t kind;  /* DN_PROJ_SIGMOID, DN_PROJ_TANH or DN_PROJ_NONE */
  float radius;  /* Gaussian filter radius in cells (kernel 2r+1 made odd, sigma r/2; 0: none) */
  float beta;
  float eta;
  float eps_lo;
  float eps_hi;
} dn_density;

/* filtered = filter(rho); eps = lo + (hi - lo) * project(filtered).  work,
 * filtered and eps each hold n_layers*H*W floats; keep `filtered` for the
 * backward pass. */
int32_t dn_density_forward(const dn_density* d, const float* rho, float* work, float* filtered,
                           float* eps, void* stream);
/* drho = filter(d eps * (hi - lo) * project'(filtered)); work as above. */
int32_t dn_density_backward(const dn_density* d, const float* filtered, const float* deps,
                            float* work, float* drho, void* stream);

/* y = 3x3 max (dilate != 0) or min pool of x in each layer, cells outside the
 * layer ignored; arg receives the in-layer index of the selected cell (the
 * first extremum in row-major window order). */
int32_t dn_morph3(const float* x, int32_t n_layers, int32_t H, int32_t W, int32_t dilate,
                  float* y, int32_t* arg, void* stream);
/* dx = the gradient of dn_morph3 for dy, from its arg (deterministic gather). */
int32_t dn_morph3_backward(const float* dy, const int32_t* arg, int32_t n_layers, int32_t H,
                           int32_t W, float* dx, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DN_DESIGN_H */
