// heat.cu -- implicit heat step (titerate, heat3mg.c:287-788).
#include "heat_markers.cuh"

namespace i3g {
int heat_alloc(i3g_ctx *) { return 0; }
void heat_free(i3g_ctx *) {}
int heat_solve(i3g_ctx *c, double *) { return set_error(c, I3G_E_UNSUPPORTED, "heat solve not built yet"); }
int heat_get_solution(i3g_ctx *c, void *, int64_t) { return set_error(c, I3G_E_UNSUPPORTED, "heat solve not built yet"); }
int heat_time_kernel(i3g_ctx *c, int, double *, double *) { return set_error(c, I3G_E_UNSUPPORTED, "heat solve not built yet"); }
}  // namespace i3g
