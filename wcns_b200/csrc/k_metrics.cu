// k_metrics.cu -- one-time grid metrics on the device.
//
// Restates GRID_DERIVATIVE_gcl (WCNSE5.f90:1478-1728, gcl=1) called from
// grid_derivative_nb (PreProcess.f90:1639-1660): sixth-order coordinate
// derivatives (VALUE_HALF_NODE then FLUX_DXYZ along each index line), then
// the Visbal-Gaitonde conservative form (differences of the products
// x_xi*y, ... along the lines) and the Jacobian vol.  kct=ett=ctt=0.
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

// sixth-order derivative along direction d at point (i,j,k) of a field
// `a` (interior values only are read)
__device__ double line_derivative(const DevBlock &B, const double *a, int i, int j, int k, int d) {
    const int n = dimof(B, d);
    const int l = d == 0 ? i : (d == 1 ? j : k);
    const long long st = dstride(B, d);
    const long long l0 = gidx(B, i, j, k) - (long long)l * st;
    auto Q = [&](int x) { return a[l0 + (long long)x * st]; };
    auto H = [&](int h) { return value_half_node_at(Q, n, h); };
    return flux_dxyz_at(H, n, l);
}

// pass 1: coordinate derivatives; products stored in the metric fields,
// dx/dkc, dx/det, dx/dct in work[0..2]
__global__ void k_metrics_pass1(DevFields F, const DevBlock *__restrict__ blocks, const double *x, const double *y,
                                const double *z, double *work, long long wstride) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % B.ni) + 1, j = (int)((q / B.ni) % B.nj) + 1, k = (int)(q / ((long long)B.ni * B.nj)) + 1;
        long long id = gidx(B, i, j, k);
        double D[9];
        const double *c3[3] = {x, y, z};
        for (int c = 0; c < 3; c++)
            for (int d = 0; d < 3; d++) D[3 * c + d] = line_derivative(B, c3[c], i, j, k, d);
        double xm = x[id], ym = y[id], zm = z[id];
        work[0 * wstride + id] = D[0];
        work[1 * wstride + id] = D[1];
        work[2 * wstride + id] = D[2];
        F.f[F_KCX][id] = D[0] * ym;
        F.f[F_KCY][id] = D[1] * ym;
        F.f[F_KCZ][id] = D[2] * ym;
        F.f[F_ETX][id] = D[3] * zm;
        F.f[F_ETY][id] = D[4] * zm;
        F.f[F_ETZ][id] = D[5] * zm;
        F.f[F_CTX][id] = D[6] * xm;
        F.f[F_CTY][id] = D[7] * xm;
        F.f[F_CTZ][id] = D[8] * xm;
    }
}

// pass 2: conservative metrics into work[3..12]
__global__ void k_metrics_pass2(DevFields F, const DevBlock *__restrict__ blocks, double *work, long long wstride) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % B.ni) + 1, j = (int)((q / B.ni) % B.nj) + 1, k = (int)(q / ((long long)B.ni * B.nj)) + 1;
        long long id = gidx(B, i, j, k);
        const int src[3][6] = {{F_CTY, F_CTZ, F_KCY, F_KCZ, F_ETY, F_ETZ},
                               {F_CTX, F_CTZ, F_KCX, F_KCZ, F_ETX, F_ETZ},
                               {F_CTX, F_CTY, F_KCX, F_KCY, F_ETX, F_ETY}};
        double D[18];
        for (int d = 0; d < 3; d++)
            for (int m = 0; m < 6; m++) D[6 * d + m] = line_derivative(B, F.f[src[d][m]], i, j, k, d);
        double kcx = D[17] - D[11], kcy = D[13] - D[7], kcz = D[15] - D[9];
        double etx = D[5] - D[16], ety = D[1] - D[12], etz = D[3] - D[14];
        double ctx = D[10] - D[4], cty = D[6] - D[0], ctz = D[8] - D[2];
        double vol = work[0 * wstride + id] * kcx + work[1 * wstride + id] * etx + work[2 * wstride + id] * ctx;
        double out[10] = {kcx, kcy, kcz, etx, ety, etz, ctx, cty, ctz, vol};
        for (int c = 0; c < 10; c++) work[(3 + c) * wstride + id] = out[c];
    }
}

__global__ void k_metrics_store(DevFields F, const DevBlock *__restrict__ blocks, const double *work, long long wstride) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % B.ni) + 1, j = (int)((q / B.ni) % B.nj) + 1, k = (int)(q / ((long long)B.ni * B.nj)) + 1;
        long long id = gidx(B, i, j, k);
        for (int c = 0; c < 10; c++) F.f[F_KCX + c][id] = work[(3 + c) * wstride + id];
    }
}

// xyz_dev: x, y, z fields (ghosted layout); work: 13 * wstride doubles
void launch_metrics(const LaunchCtx &c, double *const *xyz_dev, double *work) {
    long long maxp = 0, wstride = 0;
    for (int b = 0; b < c.nblocks; b++) {
        maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
        long long end = c.hblocks[b].off + (long long)c.hblocks[b].gx * c.hblocks[b].gy * c.hblocks[b].gz;
        wstride = end > wstride ? end : wstride;
    }
    dim3 grid((unsigned)((maxp + 127) / 128), c.nblocks);
    k_metrics_pass1<<<grid, 128, 0, c.stream>>>(*c.F, c.blocks, xyz_dev[0], xyz_dev[1], xyz_dev[2], work, wstride);
    k_metrics_pass2<<<grid, 128, 0, c.stream>>>(*c.F, c.blocks, work, wstride);
    k_metrics_store<<<grid, 128, 0, c.stream>>>(*c.F, c.blocks, work, wstride);
}

}  // namespace wcns
