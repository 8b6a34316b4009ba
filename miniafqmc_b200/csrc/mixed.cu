// Mixed-precision stages (tensor cores).  Placeholder until the tcgen05 kernels land:
// creating a mixed handle reports the form as unavailable.
#include "afq_mixed.h"

namespace afq {

struct MixedState {
  int dummy;
};

cudaError_t mixed_create(const MixedInit*, MixedState** out, std::string* msg, cudaStream_t) {
  *out = nullptr;
  if (msg) *msg = "mixed-precision form not built";
  return cudaSuccess;
}
void mixed_destroy(MixedState* m) { delete m; }
cudaError_t mixed_vbias(MixedState*, const z_t*, z_t*, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t mixed_vhs(MixedState*, const z_t*, z_t*, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t mixed_propagate(MixedState*, z_t*, const z_t*, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t mixed_energy_chol(MixedState*, const z_t*, z_t*, z_t*, int, cudaStream_t) {
  return cudaErrorNotSupported;
}
int mixed_launches(const MixedState*, int) { return 0; }

}  // namespace afq
