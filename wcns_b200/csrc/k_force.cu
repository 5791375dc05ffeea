// k_force.cu -- wall forces and moments: force (PostProcess.f90:1415-1480)
// -> force_dif (1505-1678) with getnxyz_mml (Sub1.f90:750-780), getgeo,
// getuvwtder (383-480), getduvwdxyz, stress (181-270) and getforce
// (PostProcess.f90:1680-1824) with lenth/halen/aver3 (Sub1.f90:858-889).
//
// Three kernels: every wall point's surface force (pressure, plus the
// viscous stress for laminar runs); every wall quad's force and moment from
// its four triangles; and the sums, one thread per component walking the
// quads in the reference's loop order (blocks, regions, then i, j, k), so
// the totals are the reference's sequential sums.
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

__device__ __forceinline__ double wf_lenth(double x1, double y1, double z1, double x2, double y2, double z2) {
    double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    return sqrt(dx * dx + dy * dy + dz * dz);
}
__device__ __forceinline__ double wf_halen(double a, double b, double c) {
    double p = 0.5 * (a + b + c);
    double s = p * (p - a) * (p - b) * (p - c);
    return s < 0 ? 0.0 : sqrt(s);  // the reference warns and uses 0 for a degenerate triangle
}
__device__ __forceinline__ double wf_aver3(double a, double b, double c) { return (a + b + c) / 3.0; }

__global__ void k_wall_points(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                              const DevWall *__restrict__ walls, double *__restrict__ pf) {
    const DevWall Wr = walls[blockIdx.y];
    const DevBlock B = blocks[Wr.blk];
    const int e0 = Wr.e[0], e1 = Wr.e[1], npts = Wr.e[0] * Wr.e[1] * Wr.e[2];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npts; t += gridDim.x * blockDim.x) {
        const int i = Wr.s_st[0] + t % e0, j = Wr.s_st[1] + (t / e0) % e1, k = Wr.s_st[2] + t / (e0 * e1);
        const long long id = gidx(B, i, j, k);
        // getnxyz_mml
        double nx = 0.0, ny = 0.0, nz = 0.0;
        if (Wr.s_lr3d[0]) { nx = nx + F.f[F_KCX][id]; ny = ny + F.f[F_KCY][id]; nz = nz + F.f[F_KCZ][id]; }
        if (Wr.s_lr3d[1]) { nx = nx + F.f[F_ETX][id]; ny = ny + F.f[F_ETY][id]; nz = nz + F.f[F_ETZ][id]; }
        if (Wr.s_lr3d[2]) { nx = nx + F.f[F_CTX][id]; ny = ny + F.f[F_CTY][id]; nz = nz + F.f[F_CTZ][id]; }
        const double s1 = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
        nx = nx / s1;
        ny = ny / s1;
        nz = nz / s1;
        double pn = 2.0 * (F.f[F_P][id] - B.poo);
        const double slr = (double)Wr.s_lr;
        double fx = slr * nx * pn, fy = slr * ny * pn, fz = slr * nz * pn;
        if (P.nvis == 1) {
            const int c[3] = {i, j, k}, dims[3] = {B.ni, B.nj, B.nk};
            double der[3][4];  // [direction][u, v, w, t]
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const long long st = dstride(B, d);
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const double *f = F.f[m == 3 ? F_T : F_U + m];
                    if (c[d] == 1) der[d][m] = -(1.5 * f[id] + -2.0 * f[id + st] + 0.5 * f[id + 2 * st]);
                    else if (c[d] == dims[d]) der[d][m] = 1.5 * f[id] + -2.0 * f[id - st] + 0.5 * f[id - 2 * st];
                    else der[d][m] = 0.5 * (f[id + st] - f[id - st]);
                }
            }
            const double kx = F.f[F_KCX][id], ky = F.f[F_KCY][id], kz = F.f[F_KCZ][id];
            const double ex = F.f[F_ETX][id], ey = F.f[F_ETY][id], ez = F.f[F_ETZ][id];
            const double cx = F.f[F_CTX][id], cy = F.f[F_CTY][id], cz = F.f[F_CTZ][id];
            const double vj = F.f[F_VOL][id];
            const double dudx = (kx * der[0][0] + ex * der[1][0] + cx * der[2][0]) / vj;
            const double dudy = (ky * der[0][0] + ey * der[1][0] + cy * der[2][0]) / vj;
            const double dudz = (kz * der[0][0] + ez * der[1][0] + cz * der[2][0]) / vj;
            const double dvdx = (kx * der[0][1] + ex * der[1][1] + cx * der[2][1]) / vj;
            const double dvdy = (ky * der[0][1] + ey * der[1][1] + cy * der[2][1]) / vj;
            const double dvdz = (kz * der[0][1] + ez * der[1][1] + cz * der[2][1]) / vj;
            const double dwdx = (kx * der[0][2] + ex * der[1][2] + cx * der[2][2]) / vj;
            const double dwdy = (ky * der[0][2] + ey * der[1][2] + cy * der[2][2]) / vj;
            const double dwdz = (kz * der[0][2] + ez * der[1][2] + cz * der[2][2]) / vj;
            const double c23 = 0.66666666667;  // stress (Sub1.f90:181-198)
            const double vis = F.f[F_VISL][id];
            const double txx = vis * c23 * (2.0 * dudx - dvdy - dwdz);
            const double tyy = vis * c23 * (2.0 * dvdy - dwdz - dudx);
            const double tzz = vis * c23 * (2.0 * dwdz - dudx - dvdy);
            const double txy = vis * (dudy + dvdx), txz = vis * (dudz + dwdx), tyz = vis * (dvdz + dwdy);
            pn = 2.0 * slr;
            fx = fx - pn * (nx * txx + ny * txy + nz * txz) * P.re;
            fy = fy - pn * (nx * txy + ny * tyy + nz * tyz) * P.re;
            fz = fz - pn * (nx * txz + ny * tyz + nz * tzz) * P.re;
        }
        double *o = pf + 3 * (Wr.pt_off + t);
        o[0] = fx;
        o[1] = fy;
        o[2] = fz;
    }
}

__global__ void k_wall_quads(const DevWall *__restrict__ walls, const double *__restrict__ pf,
                             const double *__restrict__ wxyz, double xref, double yref, double zref,
                             double *__restrict__ quad) {
    const DevWall Wr = walls[blockIdx.y];
    const int id_ = 1 - abs(Wr.s_lr3d[0]), jd = 1 - abs(Wr.s_lr3d[1]), kd = 1 - abs(Wr.s_lr3d[2]);
    const int n0 = Wr.e[0] - id_, n1 = Wr.e[1] - jd, n2 = Wr.e[2] - kd;
    const int nq = n0 * n1 * n2;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += gridDim.x * blockDim.x) {
        // quads in the reference's loop order: i outermost, k innermost
        const int a = t / (n1 * n2), b = (t / n2) % n1, c = t % n2;
        int q[4][3] = {{a, b, c}, {a, b, c}, {a, b, c}, {a, b, c}};
        if (id_ == 0) { q[1][1] += 1; q[2][1] += 1; q[2][2] += 1; q[3][2] += 1; }
        if (jd == 0) { q[1][0] += 1; q[2][0] += 1; q[2][2] += 1; q[3][2] += 1; }
        if (kd == 0) { q[1][0] += 1; q[2][0] += 1; q[2][1] += 1; q[3][1] += 1; }
        double px[4], py[4], pz[4], xx[4], yy[4], zz[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const long long g = Wr.pt_off + q[v][0] + (long long)Wr.e[0] * (q[v][1] + (long long)Wr.e[1] * q[v][2]);
            px[v] = pf[3 * g];
            py[v] = pf[3 * g + 1];
            pz[v] = pf[3 * g + 2];
            xx[v] = wxyz[3 * g];
            yy[v] = wxyz[3 * g + 1];
            zz[v] = wxyz[3 * g + 2];
        }
        const double px5 = 0.25 * (px[0] + px[1] + px[2] + px[3]);
        const double py5 = 0.25 * (py[0] + py[1] + py[2] + py[3]);
        const double pz5 = 0.25 * (pz[0] + pz[1] + pz[2] + pz[3]);
        const double x5 = 0.25 * (xx[0] + xx[1] + xx[2] + xx[3]);
        const double y5 = 0.25 * (yy[0] + yy[1] + yy[2] + yy[3]);
        const double z5 = 0.25 * (zz[0] + zz[1] + zz[2] + zz[3]);
        double r[4], rc[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int w = (v + 1) & 3;
            r[v] = wf_lenth(xx[v], yy[v], zz[v], xx[w], yy[w], zz[w]);  // r12, r23, r34, r41
            rc[v] = wf_lenth(xx[v], yy[v], zz[v], x5, y5, z5);          // r15, r25, r35, r45
        }
        double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int w = (v + 1) & 3;
            const double s = wf_halen(r[v], rc[v], rc[w]);
            const double pxc = wf_aver3(px[v], px[w], px5), pyc = wf_aver3(py[v], py[w], py5), pzc = wf_aver3(pz[v], pz[w], pz5);
            const double xc = wf_aver3(xx[v], xx[w], x5), yc = wf_aver3(yy[v], yy[w], y5), zc = wf_aver3(zz[v], zz[w], z5);
            const double ddfx = pxc * s, ddfy = pyc * s, ddfz = pzc * s;
            const double ddmx = (yc - yref) * ddfz - (zc - zref) * ddfy;
            const double ddmy = (zc - zref) * ddfx - (xc - xref) * ddfz;
            const double ddmz = (xc - xref) * ddfy - (yc - yref) * ddfx;
            d[0] = d[0] + ddfx;
            d[1] = d[1] + ddfy;
            d[2] = d[2] + ddfz;
            d[3] = d[3] + ddmx;
            d[4] = d[4] + ddmy;
            d[5] = d[5] + ddmz;
        }
        double *o = quad + 6 * (Wr.quad_off + t);
#pragma unroll
        for (int m = 0; m < 6; m++) o[m] = d[m];
    }
}

// sums over the quads q0..q1-1 (the walls of a range of blocks are a
// contiguous range of quads)
__global__ void k_wall_sum(const double *__restrict__ quad, long long q0, long long q1, double *out) {
    const int m = threadIdx.x;
    if (m >= 6) return;
    double s = 0.0;
    for (long long q = q0; q < q1; q++) s = s + quad[6 * q + m];
    out[m] = s;
}

void launch_forces(const LaunchCtx &c, double xref, double yref, double zref, long long q0, long long q1) {
    if (c.nwall == 0) return;
    k_wall_points<<<dim3(16, c.nwall), 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, c.walls, c.wall_pf);
    k_wall_quads<<<dim3(16, c.nwall), 256, 0, c.stream>>>(c.walls, c.wall_pf, c.wall_xyz, xref, yref, zref, c.wall_quad);
    k_wall_sum<<<1, 32, 0, c.stream>>>(c.wall_quad, q0, q1, c.wall_out);
}

}  // namespace wcns
