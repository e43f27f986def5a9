// vtr.cu -- ParaView rectilinear-grid output of the nodal fields, straight from device memory.
//
// The reference writes VTK XML RectilinearGrid files with raw appended binary data every 50th
// output file (i3vis_output_paraview.c:700-792, called at i3mg.c:159): Float64 grid-line
// coordinates, then viscosity, temperature, density, vy, vx, vz (Float32) and pressure
// (Float64), each array preceded by its byte count as a 4-byte int.  VTK orders points x
// fastest, the model y fastest (node = z*nx*ny + x*ny + y), so every field is transposed per
// z plane; the reference does that on the host (ivis_2_pv_permute_nodal_array_F32,
// i3vis_output_paraview.c:326-347).  Here a tiled shared-memory transpose reorders each field
// on the GPU, and the copy of field k to page-locked memory and its fwrite overlap the
// transpose of field k + 1.
#include <cstdio>
#include <cstring>
#include "i3g_internal.cuh"

namespace i3g {

// dst[(z*ny + y)*nx + x] = src[(z*nx + x)*ny + y]: a 32 x 32 tile per block, coalesced reads
// along y and writes along x; the tile's extra column avoids shared-memory bank conflicts
template <typename T>
__global__ void __launch_bounds__(256) k_vtk_order(const T *__restrict__ src, T *__restrict__ dst, int nx, int ny)
{
    __shared__ T tile[32][33];
    const long plane = (long)nx * ny * blockIdx.z;
    const int y0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int x = x0 + r, y = y0 + threadIdx.x;
        if (x < nx && y < ny) tile[r][threadIdx.x] = src[plane + (long)x * ny + y];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int y = y0 + r, x = x0 + threadIdx.x;
        if (x < nx && y < ny) dst[plane + (long)y * nx + x] = tile[threadIdx.x][r];
    }
}

}  // namespace i3g

using namespace i3g;

namespace {

struct VtrField {
    const char *name;
    const void *dev;
    int size;   // 4: Float32, 8: Float64
};

// the byte offsets of the appended data are 4-byte ints in this format
bool offset_ok(long off) { return off >= 0 && off < 0x7fffffffL; }

}  // namespace

extern "C" int i3g_write_vtr(i3g_ctx *c, const char *path)
{
    if (!c || !path) return I3G_E_ARG;
    const long nx = c->m.xnumx, ny = c->m.ynumy, nz = c->m.znumz, N = nx * ny * nz;
    const VtrField fields[7] = {{"viscosity", c->lev[0].nu, 4}, {"temperature", c->tk, 4}, {"density", c->ro, 4},
                                {"vy", c->vy, 4},               {"vx", c->vx, 4},          {"vz", c->vz, 4},
                                {"pressure", c->pr, 8}};
    long off = 0, offs[10];
    const long nc[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) { offs[a] = off; off += 4 + nc[a] * 8; }
    for (int f = 0; f < 7; f++) { offs[3 + f] = off; off += 4 + N * fields[f].size; }
    if (!offset_ok(off)) return set_error(c, I3G_E_ARG, "VTR appended data of %ld bytes exceeds the format's 4-byte offsets", off);
    FILE *fl = fopen(path, "wb");
    if (!fl) return set_error(c, I3G_E_ARG, "cannot create %s", path);
    // the staging buffers live for this call only; freed on every path
    void *dbuf = nullptr, *hbuf[2] = {nullptr, nullptr};
    cudaEvent_t ready[2] = {nullptr, nullptr};
    int rc = 0;
    auto fail = [&](int code, const char *msg) {
        if (!rc) rc = set_error(c, code, "%s (%s)", msg, path);
        return rc;
    };
    if (cudaMalloc(&dbuf, 2 * N * 8) != cudaSuccess || cudaMallocHost(&hbuf[0], N * 8) != cudaSuccess ||
        cudaMallocHost(&hbuf[1], N * 8) != cudaSuccess || cudaEventCreateWithFlags(&ready[0], cudaEventDisableTiming) ||
        cudaEventCreateWithFlags(&ready[1], cudaEventDisableTiming)) {
        cudaGetLastError();
        fail(I3G_E_NOMEM, "VTR staging buffers");
    }
    if (!rc) {
        fprintf(fl, "<VTKFile type=\"RectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
        fprintf(fl, "  <RectilinearGrid WholeExtent=\"0 %ld 0 %ld 0 %ld\">\n", nx - 1, ny - 1, nz - 1);
        fprintf(fl, "    <Piece Extent=\"0 %ld 0 %ld 0 %ld\">\n", nx - 1, ny - 1, nz - 1);
        fprintf(fl, "      <Coordinates>\n");
        const char *cn[3] = {"xcoor", "ycoor", "zcoor"};
        for (int a = 0; a < 3; a++)
            fprintf(fl, "        <DataArray Name=\"%s\" type=\"Float64\" NumberOfComponents=\"1\" format=\"appended\" offset=\"%ld\">\n"
                        "        </DataArray>\n", cn[a], offs[a]);
        fprintf(fl, "      </Coordinates>\n      <PointData>\n");
        for (int f = 0; f < 7; f++)
            fprintf(fl, "        <DataArray Name=\"%s\" type=\"%s\" NumberOfComponents=\"1\" format=\"appended\" offset=\"%ld\">\n"
                        "        </DataArray>\n", fields[f].name, fields[f].size == 8 ? "Float64" : "Float32", offs[3 + f]);
        fprintf(fl, "      </PointData>\n    </Piece>\n  </RectilinearGrid>\n  <AppendedData encoding=\"raw\">\n_");
        const double *g[3] = {c->hgx, c->hgy, c->hgz};
        for (int a = 0; a < 3 && !rc; a++) {
            const int len = (int)(nc[a] * 8);
            if (fwrite(&len, 4, 1, fl) != 1 || fwrite(g[a], 8, nc[a], fl) != (size_t)nc[a]) fail(I3G_E_ARG, "VTR write failed");
        }
    }
    // field f: transpose into device slot f % 2, copy to host slot f % 2, write when its event is done
    const dim3 blk(32, 8), grd((unsigned)((ny + 31) / 32), (unsigned)((nx + 31) / 32), (unsigned)nz);
    auto enqueue = [&](int f) {
        void *d = (char *)dbuf + (size_t)(f % 2) * N * 8;
        if (fields[f].size == 8)
            k_vtk_order<double><<<grd, blk, 0, c->st>>>((const double *)fields[f].dev, (double *)d, (int)nx, (int)ny);
        else
            k_vtk_order<float><<<grd, blk, 0, c->st>>>((const float *)fields[f].dev, (float *)d, (int)nx, (int)ny);
        c->launches++;
        cudaMemcpyAsync(hbuf[f % 2], d, (size_t)N * fields[f].size, cudaMemcpyDeviceToHost, c->st);
        cudaEventRecord(ready[f % 2], c->st);
    };
    if (!rc) enqueue(0);
    for (int f = 0; f < 7 && !rc; f++) {
        if (f + 1 < 7) enqueue(f + 1);   // the next field's transpose and copy overlap this write
        if (cudaEventSynchronize(ready[f % 2]) != cudaSuccess) {
            fail(I3G_E_CUDA, "VTR transpose or copy failed");
            break;
        }
        const int len = (int)(N * fields[f].size);
        if (fwrite(&len, 4, 1, fl) != 1 || fwrite(hbuf[f % 2], fields[f].size, N, fl) != (size_t)N) fail(I3G_E_ARG, "VTR write failed");
        // slot f % 2 is free again only after its data are written: the field after next uses it
    }
    if (!rc) fprintf(fl, "\n  </AppendedData>\n</VTKFile>\n");
    if (fclose(fl) && !rc) fail(I3G_E_ARG, "VTR close failed");
    cudaStreamSynchronize(c->st);
    cudaFree(dbuf);
    cudaFreeHost(hbuf[0]);
    cudaFreeHost(hbuf[1]);
    if (ready[0]) cudaEventDestroy(ready[0]);
    if (ready[1]) cudaEventDestroy(ready[1]);
    cudaError_t e = cudaGetLastError();
    if (!rc && e != cudaSuccess) rc = cuda_fail(c, e, "i3g_write_vtr", __FILE__, __LINE__);
    return rc;
}
