// batch.cu -- batched replicas (placeholder until the batched kernel lands).
#include "kpzb_api_internal.h"

using namespace kpzb;
struct kpzb_batch {
    int n;
};
extern "C" {
kpzb_status kpzb_batch_create(kpzb_batch** b, int, const int*, const double*, const double*,
                              const uint64_t*, const uint32_t*, int)
{
    if (b) *b = nullptr;
    return fail(KPZB_EUNSUPPORTED, "batch not built yet");
}
kpzb_status kpzb_batch_destroy(kpzb_batch*) { return KPZB_OK; }
kpzb_status kpzb_batch_init_homogeneous(kpzb_batch*) { return fail(KPZB_EUNSUPPORTED, "batch"); }
kpzb_status kpzb_batch_mcs(kpzb_batch*, int) { return fail(KPZB_EUNSUPPORTED, "batch"); }
kpzb_status kpzb_batch_push(kpzb_batch*, int, const uint32_t*) { return fail(KPZB_EUNSUPPORTED, "batch"); }
kpzb_status kpzb_batch_pop(kpzb_batch*, int, uint32_t*) { return fail(KPZB_EUNSUPPORTED, "batch"); }
kpzb_status kpzb_batch_roughness(kpzb_batch*, double*) { return fail(KPZB_EUNSUPPORTED, "batch"); }
}
