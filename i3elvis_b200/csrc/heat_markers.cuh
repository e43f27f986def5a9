// heat_markers.cuh -- heat solve (heat3mg.c) and marker kernels (mark3mg.c) of the library.
#pragma once
#include "i3g_internal.cuh"

namespace i3g {
int heat_alloc(i3g_ctx *c);
void heat_free(i3g_ctx *c);
int heat_solve(i3g_ctx *c, double *timestep);
int heat_get_solution(i3g_ctx *c, void *dst, int64_t nbytes);
int heat_time_kernel(i3g_ctx *c, int reps, double *ms, double *bytes);

int markers_alloc(i3g_ctx *c);
void markers_free(i3g_ctx *c);
// async: copies on the context's copy stream; marker operations wait for them on the device
int markers_upload(i3g_ctx *c, const i3g_model *m, bool async = false);
int markers_download(i3g_ctx *c, i3g_model *m);
int markers_move(i3g_ctx *c, double timestep);
int markers_to_nodes(i3g_ctx *c, double timestep);
int markers_time_kernel(i3g_ctx *c, int kind, int reps, double *ms, double *bytes);
// marker temperature update after the heat solve (heat3mg.c:592-782)
int markers_heat_update(i3g_ctx *c, double timestep, const float *tk0, const float *tk1, const float *tk2);
}  // namespace i3g
