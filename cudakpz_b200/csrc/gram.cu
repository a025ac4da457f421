// gram.cu -- exact height autocorrelator (placeholder until the Gram kernels land).
#include "kpzb_api_internal.h"

using namespace kpzb;
struct kpzb_gram {
    int n;
};
extern "C" {
kpzb_status kpzb_gram_create(kpzb_gram** g, int, int, int, int)
{
    if (g) *g = nullptr;
    return fail(KPZB_EUNSUPPORTED, "gram not built yet");
}
kpzb_status kpzb_gram_destroy(kpzb_gram*) { return KPZB_OK; }
kpzb_status kpzb_gram_add_device(kpzb_gram*, const uint32_t*) { return fail(KPZB_EUNSUPPORTED, "gram"); }
kpzb_status kpzb_gram_add_host(kpzb_gram*, const uint32_t*) { return fail(KPZB_EUNSUPPORTED, "gram"); }
kpzb_status kpzb_gram_compute(kpzb_gram*, int, int64_t*, int64_t*) { return fail(KPZB_EUNSUPPORTED, "gram"); }
int kpzb_gram_count(const kpzb_gram*) { return 0; }
}
