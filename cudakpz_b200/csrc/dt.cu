// dt.cu -- double-tiling random-sequential dynamics (placeholder until the DT kernel lands).
#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"

namespace kpzb {
kpzb_status dt_init(DtState* s, int, int, int)
{
    s->ready = false;
    return fail(KPZB_EUNSUPPORTED, "DT dynamics not built yet");
}
void dt_free(DtState* s) { s->ready = false; }
kpzb_status dt_enqueue(DtState*, uint32_t*, int, int, uint64_t, int, double, double, uint64_t,
                       uint32_t, cudaStream_t)
{
    return fail(KPZB_EUNSUPPORTED, "DT dynamics not built yet");
}
}  // namespace kpzb
