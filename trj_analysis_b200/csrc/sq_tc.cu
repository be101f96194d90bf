// sq_tc.cu -- tensor-core (tcgen05) split-BF16 S(Q) path.  Placeholder until the kernel lands.
#include "sq_plan.cuh"

int trj_sq_tc_prepare(trj_sq_plan* plan) { (void)plan; return TRJ_ERR_UNSUPPORTED; }
void trj_sq_tc_release(trj_sq_plan* plan) { (void)plan; }
int trj_sq_tc_run(trj_sq_plan* plan, const float box[3], cudaStream_t s) {
    (void)box; (void)s;
    return trj_fail(plan->ctx, TRJ_ERR_UNSUPPORTED, "tensor-core S(Q) not built");
}
