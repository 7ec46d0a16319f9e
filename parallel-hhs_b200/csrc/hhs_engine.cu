// hhs_engine.cu -- device-resident HOLD schedule (placeholder until the persistent
// engine lands; the host-driven schedule is used while engine_workspace_bytes is 0).
#include "hhs_ctx.h"

size_t engine_workspace_bytes(int, int) { return 0; }
hhs_status engine_init(hhs_ctx*, void*) { return HHS_OK; }
hhs_status engine_hold_step(hhs_ctx*, const SoA&, int, double, bool, hhs_precision,
                            cudaStream_t) {
    return HHS_ERR_INVALID_ARG;
}
