// ffa_pending.cu -- entry points whose kernels are not built yet; each
// returns FFA_ERR_UNSUPPORTED without touching device memory.
#include "ffa_internal.cuh"

namespace ffa {
cudaError_t launch_boris_f32c(const PushK &, cudaStream_t) { return cudaErrorNotSupported; }
}  // namespace ffa

extern "C" {
int ffa_fp32c_split(ffa_state_soa *, int64_t, void *) { return FFA_ERR_UNSUPPORTED; }
int ffa_fp32c_merge(ffa_state_soa *, int64_t, void *) { return FFA_ERR_UNSUPPORTED; }
}
