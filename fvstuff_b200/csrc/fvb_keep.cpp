// fvb_keep.cpp -- KEEP flux family (keep_fv_euler_2d.cu) behind fvb_solver.
#include "fvb_host.h"

namespace fvb {

static fvb_status not_yet() { return fail(FVB_ERR_INVALID, "the KEEP flux family is not available in this build"); }
fvb_status keep_create(const fvb_config *, fvb_solver **) { return not_yet(); }
void keep_destroy(fvb_solver *) {}
fvb_status keep_init_case(fvb_solver *, const fvb_case *) { return not_yet(); }
fvb_status keep_set_state(fvb_solver *, const void *, int, int, int, int) { return not_yet(); }
fvb_status keep_get_state(fvb_solver *, void *, int, int, int, int) { return not_yet(); }
fvb_status keep_step(fvb_solver *, int, double) { return not_yet(); }
fvb_status keep_sync(fvb_solver *, fvb_stats *) { return not_yet(); }
fvb_status keep_stats_sums(fvb_solver *, fvb_stats *) { return not_yet(); }

}  // namespace fvb
