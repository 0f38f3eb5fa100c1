// fvb_batch.cpp -- batched form (placeholder until the batch scheduler lands).
#include "fvb_host.h"

using namespace fvb;

static fvb_status nb() { return fail(FVB_ERR_INVALID, "batched form not available in this build"); }

extern "C" {
fvb_status fvb_batch_create(const fvb_batch_config *, fvb_batch **out) { if (out) *out = nullptr; return nb(); }
void fvb_batch_destroy(fvb_batch *) {}
size_t fvb_batch_instance_bytes(const fvb_batch *, int) { return 0; }
fvb_status fvb_batch_add(fvb_batch *, const fvb_instance_desc *, int *) { return nb(); }
fvb_status fvb_batch_run(fvb_batch *, int) { return nb(); }
fvb_status fvb_batch_poll(fvb_batch *, int *, int, int *) { return nb(); }
fvb_status fvb_batch_get_state(fvb_batch *, int, void *, int, int, int) { return nb(); }
fvb_status fvb_batch_instance_stats(fvb_batch *, int, fvb_stats *) { return nb(); }
fvb_status fvb_batch_remove(fvb_batch *, int) { return nb(); }
int fvb_batch_active(const fvb_batch *) { return 0; }
size_t fvb_batch_bytes_in_use(const fvb_batch *) { return 0; }
fvb_status fvb_serve_run(const fvb_serve_config *, const fvb_request *, int, fvb_request_result *, double *) { return nb(); }
}
