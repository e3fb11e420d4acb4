// ffa_pending.cu -- entry points whose kernels are not built yet; each
// returns FFA_ERR_UNSUPPORTED without touching device memory.
#include "ffa_internal.cuh"

namespace ffa {
cudaError_t launch_boris_f32c(const PushK &, cudaStream_t) { return cudaErrorNotSupported; }
}  // namespace ffa

extern "C" {
int ffa_fp32c_split(ffa_state_soa *, int64_t, void *) { return FFA_ERR_UNSUPPORTED; }
int ffa_fp32c_merge(ffa_state_soa *, int64_t, void *) { return FFA_ERR_UNSUPPORTED; }
int ffa_sc_plan_create(const ffa_sc_desc *, void *, ffa_sc_plan **out)
{
    if (out) *out = nullptr;
    return FFA_ERR_UNSUPPORTED;
}
int ffa_sc_plan_destroy(ffa_sc_plan *) { return FFA_OK; }
int ffa_sc_step(ffa_sc_plan *, ffa_state_soa *, int64_t, int32_t, int32_t, void *, int64_t *, ffa_sc_diag *)
{
    return FFA_ERR_UNSUPPORTED;
}
int ffa_sc_buffers(const ffa_sc_plan *, const float **, const float **, const float **, const float **,
                   const int32_t **, const int64_t **)
{
    return FFA_ERR_UNSUPPORTED;
}
}
