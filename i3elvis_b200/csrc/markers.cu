// markers.cu -- marker advection (movemark, mark3mg.c:2-397) and marker->node averaging
// (ronurecalc, mark3mg.c:404-1015).
#include "heat_markers.cuh"

namespace i3g {
int markers_alloc(i3g_ctx *) { return 0; }
void markers_free(i3g_ctx *) {}
int markers_upload(i3g_ctx *, const i3g_model *) { return 0; }
int markers_download(i3g_ctx *, i3g_model *) { return 0; }
int markers_move(i3g_ctx *c, double) { return set_error(c, I3G_E_UNSUPPORTED, "markers not built yet"); }
int markers_to_nodes(i3g_ctx *c, double) { return set_error(c, I3G_E_UNSUPPORTED, "markers not built yet"); }
int markers_time_kernel(i3g_ctx *c, int, int, double *, double *) { return set_error(c, I3G_E_UNSUPPORTED, "markers not built yet"); }
}  // namespace i3g
