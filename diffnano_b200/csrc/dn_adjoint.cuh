// Parameters and helpers shared by the 2-D and 3-D adjoint (reverse-step)
// kernels.
#pragma once

#include "dn_host.cuh"

namespace dn {

// adjoint-step parameters (shared with the 3-D adjoint)
template <typename T>
struct AdjParams {
  int D, H, W;
  long long py, pz;
  const T* in[6];
  T* out[6];
  const T* ce;
  const double* b[3];
  const double* c[3];
  T dt, inv_dl;
  const T* curl[3];
  long long curl_stride;
  int curl_t0;
  double* grad;
  int t;
  int* status;
};

template <typename T>
int build_adj_params(bool is3d, const dn_grid* g, void* const la[6], void* const lb[6],
                     const void* ce, const dn_cpml* cpml, const dn_curl_record* curl,
                     double* grad, int t_end, int nsteps, int* status, AdjParams<T>* p);

// Inject every monitor's DFT gradient into the adjoint field of step p.t:
// lambda[comp][cell] += sum_f g[f][cell] . phase[t][f] (one small launch per
// monitor, before the reverse step).
template <typename T>
int inject_monitors(const AdjParams<T>& p, const dn_monitor* mons, int n_mon, bool is3d, int pol,
                    cudaStream_t s);

}  // namespace dn
