// Library-wide C-ABI helpers: status strings, version, last CUDA error.
#include "dn_common.cuh"
#include "dn_fno.h"
#include "dn_design.h"

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

#include <cstring>

extern "C" int64_t dn_struct_size(const char* name) {
  if (!name) return -1;
  struct Entry {
    const char* n;
    int64_t s;
  };
  static const Entry table[] = {
      {"dn_box", sizeof(dn_box)},         {"dn_grid", sizeof(dn_grid)},
      {"dn_cpml", sizeof(dn_cpml)},       {"dn_source", sizeof(dn_source)},
      {"dn_monitor", sizeof(dn_monitor)}, {"dn_probe", sizeof(dn_probe)},
      {"dn_curl_record", sizeof(dn_curl_record)},
      {"dn_batch2d_inst", sizeof(dn_batch2d_inst)},
      {"dn_batch2d", sizeof(dn_batch2d)},
      {"dn_gemm_operand", sizeof(dn_gemm_operand)},
      {"dn_gemm", sizeof(dn_gemm)},
      {"dn_density", sizeof(dn_density)},
      {"dn_span", sizeof(dn_span)},
  };
  for (const Entry& e : table)
    if (std::strcmp(e.n, name) == 0) return e.s;
  return -1;
}

extern "C" int32_t dn_last_cuda_error(void) { return dn::last_cuda_error(); }
