// Library-wide C-ABI helpers: status strings, version, last CUDA error.
#include "dn_common.cuh"

namespace dn {
namespace {
thread_local int g_last_cuda_error = 0;
}
void set_last_cuda_error(int e) { g_last_cuda_error = e; }
int last_cuda_error() { return g_last_cuda_error; }
}  // namespace dn

extern "C" const char* dn_strerror(int32_t status) {
  switch (status) {
    case DN_OK: return "ok";
    case DN_EINVAL: return "invalid argument";
    case DN_ENOMEM: return "fixed-size resource limit exceeded";
    case DN_ECUDA: return "CUDA call failed";
    case DN_ETIMEOUT: return "bounded device-side wait timed out";
    case DN_ENONFINITE: return "non-finite value detected";
    case DN_EUNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

extern "C" int32_t dn_version(void) { return 1; }

extern "C" int32_t dn_last_cuda_error(void) { return dn::last_cuda_error(); }
