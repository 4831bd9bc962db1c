// Spherical-harmonic FMM (placeholder until the FMM kernels land).
#include "mms_internal.cuh"

struct FmmPlan {
    int dummy;
};

int fmm_plan_create(mms_ctx *ctx)
{
    (void)ctx;
    mms_set_error("FMM solver not built yet");
    return MMS_ERR_ARG;
}
void fmm_plan_destroy(mms_ctx *ctx) { (void)ctx; }
int launch_potential_fmm(mms_ctx *ctx, const float *rho, float *phi)
{
    (void)ctx; (void)rho; (void)phi;
    mms_set_error("FMM solver not built yet");
    return MMS_ERR_ARG;
}
size_t fmm_plan_bytes(const mms_ctx *ctx) { (void)ctx; return 0; }
