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

// initial markers (in3mg.c:131-797): placement, jitter, rock bodies, temperature
struct BodyDev {
    int rock, shape;        // shape 0: box with bilinear faces, 1: ellipsoid shell, 2: cylinder along y
    double k[6][4];         // box faces left, right, up, down, front, back: a0 + a1 u + a2 v + a3 u v
    double c[3], s[3];      // ellipsoid / cylinder: centre and axis scales (relative coordinates)
    double r0, r1;          // accepted radius range
    float ex, e;            // markex and marke of the body's markers
};
struct InitDev {
    int mx, my, mz;                 // markers per cell along x, y, z
    double st[3];                   // cell spacing of the placement grid (size / (n - 1))
    float jit[3];                   // jitter amplitude (m) along x, y, z
    int nonstab;                    // jitter resolution (0: none)
    unsigned long long seed;
    int background;                 // rock type outside every body
    double ttop, tbot;              // marker temperature linear in y between these
    int nbodies;
    const BodyDev *bodies;          // device array
};
int markers_init(i3g_ctx *c, const InitDev &d);
}  // namespace i3g
