// k_sweep_plane.cu -- GS_PR_Single (LHS.f90:1559-1613) as one launch per
// hyperplane i+j+k = p and sweep: lusgs_l (381-478), lusgs_u (480-577),
// gs_pr_l (1777-1866), gs_pr_u (1956-2046), all blocks of the context in each
// launch.
//
// A point needs its neighbours one plane below (forward) or above (backward)
// from the same sweep and, in the Gauss-Seidel sweeps, those on the other
// side from the previous sweep; walking the planes in order with one launch
// each therefore reproduces the reference's in-place lexicographic sweep on
// the field layout itself, with the reference's per-point arithmetic (the
// neighbour terms mxdq_std, 756-828, evaluated from the neighbours' prim,
// metrics and spectral radii).  The launch boundary is the only
// synchronisation, so the shape has no limit on block size; it is the path
// for blocks whose (j,k) columns do not fit the clustered sweep kernel's
// shared memory, and the per-launch baseline that kernel is measured against.
#include <algorithm>

#include "wcns_launch.h"

namespace wcns {

namespace {

// mxdq_std with gettmhmgm_ns (GasModel.f90:411-426), nt = 0
__device__ __forceinline__ void mxdq_std_dev(double gama, const double *prim, double nx, double ny, double nz,
                                             const double *dq, double rad, double npn, double *f) {
    const double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    const double nt = 0.0;
    const double hint = gama / (gama - 1.0) * pm / rm;
    const double c2 = gama * pm / rm;
    const double cm = sqrt(c2);
    const double v2 = um * um + vm * vm + wm * wm;
    const double hm = hint + 0.5 * v2;
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    if (!(cgm >= SML_SSS)) cgm = SML_SSS;
    double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    l1 = 0.5 * (l1 + npn * rad);
    l4 = 0.5 * (l4 + npn * rad);
    l5 = 0.5 * (l5 + npn * rad);
    const double x1 = (2.0 * l1 - l4 - l5) / (2.0 * c2);
    const double x2 = (l4 - l5) / (2.0 * cm);
    const double cgm1 = 1.0 / cgm;
    nx = nx * cgm1;
    ny = ny * cgm1;
    nz = nz * cgm1;
    ct = (ct - nt) * cgm1;
    const double ae = gama - 1.0;
    const double af = 0.5 * ae * v2;
    const double dc = ct * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
    const double dh = af * dq[0] - ae * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
    const double c2dc = c2 * dc;
    f[0] = l1 * dq[0] - dh * x1 - dc * x2;
    f[1] = l1 * dq[1] + (nx * c2dc - um * dh) * x1 + (nx * dh - um * dc) * x2;
    f[2] = l1 * dq[2] + (ny * c2dc - vm * dh) * x1 + (ny * dh - vm * dc) * x2;
    f[3] = l1 * dq[3] + (nz * c2dc - wm * dh) * x1 + (nz * dh - wm * dc) * x2;
    f[4] = l1 * dq[4] + (ct * c2dc - hm * dh) * x1 + (ct * dh - hm * dc) * x2;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The term of the neighbour one point along direction d on side `side`
// (-1 lower with npn = +1, +1 upper with npn = -1): its prim, its metrics of
// direction d with the index clamped into the block (getrkec_mml), the
// spectral radius of direction d at the clamped neighbour index
// (getrarbrc, method 1), applied to the neighbour's dq `dqn`.
__device__ __forceinline__ void nbr_term(const DevParams &P, const DevFields &F, const DevBlock &B, int i, int j, int k,
                                         int d, int side, const double *dqn, double *f) {
    int c[3] = {i, j, k};
    c[d] += side;
    const long long nid = gidx(B, c[0], c[1], c[2]);
    double prim[5];
#pragma unroll
    for (int m = 0; m < 5; m++) prim[m] = F.f[F_R + m][nid];
    const int dims[3] = {B.ni, B.nj, B.nk};
    int g[3] = {clampi(c[0], 1, B.ni), clampi(c[1], 1, B.nj), clampi(c[2], 1, B.nk)};
    const long long gid = gidx(B, g[0], g[1], g[2]);
    const double nx = F.f[F_KCX + 3 * d][gid], ny = F.f[F_KCX + 3 * d + 1][gid], nz = F.f[F_KCX + 3 * d + 2][gid];
    int r[3] = {i, j, k};
    r[d] = clampi(r[d] + side, 1, dims[d]);
    const double rad = F.f[F_SRA + d][gidx(B, r[0], r[1], r[2])];
    mxdq_std_dev(P.gama, prim, nx, ny, nz, dqn, rad, side < 0 ? 1.0 : -1.0, f);
}

__device__ __forceinline__ void load_dq(const DevFields &F, long long id, double *v) {
#pragma unroll
    for (int m = 0; m < 5; m++) v[m] = F.f[F_DQ1 + m][id];
}

// getcoed (LHS.f90:602-645), wmig = beta = 1, no dual time stepping
__device__ __forceinline__ double coed_at(const DevParams &P, const DevFields &F, long long id) {
    double rad_ns = F.f[F_SRA][id] + F.f[F_SRB][id] + F.f[F_SRC][id];
    if (P.nvis >= 1) rad_ns = rad_ns + F.f[F_SRVA][id] + F.f[F_SRVB][id] + F.f[F_SRVC][id];
    const double ct = 1.0 / F.f[F_DTDT][id];
    return 1.0 / (ct + 1.0 * 1.0 * rad_ns);
}

}  // namespace

// MODE 0 lusgs_l, 1 lusgs_u, 2 gs_pr_l, 3 gs_pr_u; one thread per (j,k)
// column of each block, the point of the column in plane p
template <int MODE>
__global__ void __launch_bounds__(256) k_sweep_plane(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int p) {
    const DevBlock B = blocks[blockIdx.y];
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= B.nj * B.nk) return;
    const int j = col % B.nj + 1, k = col / B.nj + 1, i = p - j - k;
    if (i < 1 || i > B.ni) return;
    const long long id = gidx(B, i, j, k);
    const long long sx = 1, sy = B.gx, sz = (long long)B.gx * B.gy;
    const double coed = coed_at(P, F, id);
    double rhs0[5], dqa[5], dqb[5], dqc[5], ta[5], tb[5], tc[5];
    if (MODE == 0 || MODE == 1) {
        const int s = MODE == 0 ? -1 : 1;
        load_dq(F, id + s * sx, dqa);
        load_dq(F, id + s * sy, dqb);
        load_dq(F, id + s * sz, dqc);
        nbr_term(P, F, B, i, j, k, 0, s, dqa, ta);
        nbr_term(P, F, B, i, j, k, 1, s, dqb, tb);
        nbr_term(P, F, B, i, j, k, 2, s, dqc, tc);
#pragma unroll
        for (int m = 0; m < 5; m++) rhs0[m] = 1.0 * (ta[m] + tb[m] + tc[m]);
        if (P.nvis > 0) {
            const double rva = F.f[F_SRVA][id + s * sx], rvb = F.f[F_SRVB][id + s * sy], rvc = F.f[F_SRVC][id + s * sz];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                const double v = 0.5 * (rva * dqa[m] + rvb * dqb[m] + rvc * dqc[m]);
                rhs0[m] = MODE == 0 ? rhs0[m] + v : rhs0[m] - v;
            }
        }
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double d0 = F.f[F_DQ1 + m][id];
            F.f[F_DQ1 + m][id] = MODE == 0 ? (-d0 + rhs0[m]) * coed : d0 - rhs0[m] * coed;
        }
    } else {
        double lo[3][5], up[3][5];
        const long long st[3] = {sx, sy, sz};
        const int c[3] = {i, j, k}, n[3] = {B.ni, B.nj, B.nk};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (c[d] == 1) {
#pragma unroll
                for (int m = 0; m < 5; m++) dqa[m] = 0.0;
            } else {
                load_dq(F, id - st[d], dqa);
            }
            nbr_term(P, F, B, i, j, k, d, -1, dqa, lo[d]);
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (c[d] == n[d]) {
#pragma unroll
                for (int m = 0; m < 5; m++) dqa[m] = 0.0;
            } else {
                load_dq(F, id + st[d], dqa);
            }
            nbr_term(P, F, B, i, j, k, d, 1, dqa, up[d]);
        }
#pragma unroll
        for (int m = 0; m < 5; m++) {
            rhs0[m] = 1.0 * (lo[0][m] + lo[1][m] + lo[2][m] - up[0][m] - up[1][m] - up[2][m]);
            F.f[F_DQ1 + m][id] = (rhs0[m] - F.f[F_RHS1 + m][id]) * coed;
        }
    }
}

// store_rhs_nb (LHS.f90:1592-1613): the right-hand side the Gauss-Seidel
// sweeps start from
__global__ void k_store_rhs(DevFields F, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_point(B, q, i, j, k);
        const long long id = gidx(B, i, j, k);
#pragma unroll
        for (int m = 0; m < 5; m++) F.f[F_RHS1 + m][id] = F.f[F_DQ1 + m][id];
    }
}

// the four sweeps plane by plane; returns the number of launches
int launch_sweeps_by_plane(const LaunchCtx &c) {
    int maxcols = 0, pmax = 0;
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) {
        const DevBlock &B = c.hblocks[b];
        maxcols = std::max(maxcols, B.nj * B.nk);
        pmax = std::max(pmax, B.ni + B.nj + B.nk);
        maxp = std::max(maxp, B.npts);
    }
    int n = 0;
    k_store_rhs<<<dim3((unsigned)std::min<long long>((maxp + 255) / 256, 4096), c.nblocks), 256, 0, c.stream>>>(*c.F,
                                                                                                                 c.blocks);
    n++;
    const dim3 grid((unsigned)((maxcols + 255) / 256), c.nblocks);
    for (int p = 3; p <= pmax; p++, n++) k_sweep_plane<0><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p);
    prof_mark(c, "sweep_lusgs_l");
    for (int p = pmax; p >= 3; p--, n++) k_sweep_plane<1><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p);
    prof_mark(c, "sweep_lusgs_u");
    for (int p = 3; p <= pmax; p++, n++) k_sweep_plane<2><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p);
    prof_mark(c, "sweep_gs_pr_l");
    for (int p = pmax; p >= 3; p--, n++) k_sweep_plane<3><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p);
    prof_mark(c, "sweep_gs_pr_u");
    return n;
}

}  // namespace wcns
