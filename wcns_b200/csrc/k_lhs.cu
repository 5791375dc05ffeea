// k_lhs.cu -- implicit update: l_h_s_tgh (LHS.f90:1-34) -> GS_PR_Single
// (LHS.f90:1559-1587): lusgs_l (381-478), lusgs_u (480-577), gs_pr_l
// (1777-1866), gs_pr_u (1956-2046), each point update using getcoed
// (602-645), getrarbrc (647-678), getrkec_mml (Sub1.f90:676-717) and
// mxdq_std (LHS.f90:756-828); set_nonconnect_boundary_dq_0 (CIC.f90:2-17)
// before and after.
//
// The reference sweeps each block lexicographically.  A point only reads
// lower neighbours (already updated in this sweep) and upper neighbours (not
// yet updated), so processing the hyperplanes i+j+k = p in order reproduces
// the sequential result exactly.  One CTA owns one block; its threads own
// (j,k) columns and march the planes with a barrier per plane (blocks are
// independent: the reference's LU-SGS is block-Jacobi).
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

__global__ void k_zero_faces(DevFields F, const long long *__restrict__ pts, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        long long id = pts[e];
#pragma unroll
        for (int m = 0; m < 5; m++) F.f[F_DQ1 + m][id] = 0.0;
    }
}

// A+-(neighbour) * dq(neighbour) along direction d; side -1 lower (npn=+1),
// side +1 upper (npn=-1).  `c` is the point's coordinate along d.
__device__ __forceinline__ void nbr_term(const DevParams &P, const DevFields &F, const DevBlock &B, long long id, int d,
                                         int c, int side, const double *dqn, double *f) {
    const long long st = dstride(B, d);
    const long long nid = side < 0 ? id - st : id + st;
    double prim[5];
#pragma unroll
    for (int m = 0; m < 5; m++) prim[m] = __ldg(F.f[F_R + m] + nid);
    const int n = dimof(B, d);
    // metrics at the neighbour with 0 -> 1 and n+1 -> n (getrkec_mml), the
    // spectral radius at the neighbour clamped to 1..n (getrarbrc)
    long long mid = nid;
    if (c + side < 1) mid = id;
    if (c + side > n) mid = id;
    double gx = __ldg(F.f[F_KCX + 3 * d] + mid), gy = __ldg(F.f[F_KCX + 3 * d + 1] + mid),
           gz = __ldg(F.f[F_KCX + 3 * d + 2] + mid);
    double rad = __ldg(F.f[F_SRA + d] + mid);
    mxdq_std(P, prim, gx, gy, gz, dqn, f, rad, side < 0 ? 1 : -1);
}

template <int MODE>  // 0 lusgs_l, 1 lusgs_u, 2 gs_pr_l, 3 gs_pr_u
__global__ void __launch_bounds__(1024) k_sweep(DevParams P, DevFields F, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.x];
    const int ni = B.ni, nj = B.nj, nk = B.nk;
    const int ncol = nj * nk;
    const bool forward = (MODE == 0 || MODE == 2);
    const int pfirst = forward ? 3 : ni + nj + nk, plast = forward ? ni + nj + nk : 3, pstep = forward ? 1 : -1;
    const long long sj = B.gx, sk = (long long)B.gx * B.gy;
    for (int p = pfirst;; p += pstep) {
        for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
            const int j = col % nj + 1, k = col / nj + 1, i = p - j - k;
            if (i < 1 || i > ni) continue;
            const long long id = gidx(B, i, j, k);
            const double coed = F.f[F_COED][id];
            const int cc[3] = {i, j, k};
            const long long sts[3] = {1, sj, sk};
            double r0[5];
            if (MODE == 0 || MODE == 1) {
                double dn[3][5], term[3][5];
                const int side = MODE == 0 ? -1 : 1;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    long long nid = side < 0 ? id - sts[d] : id + sts[d];
#pragma unroll
                    for (int m = 0; m < 5; m++) dn[d][m] = F.f[F_DQ1 + m][nid];
                    nbr_term(P, F, B, id, d, cc[d], side, dn[d], term[d]);
                }
#pragma unroll
                for (int m = 0; m < 5; m++) r0[m] = 1.0 * (term[0][m] + term[1][m] + term[2][m]);
                if (P.nvis > 0) {
                    double rva = F.f[F_SRVA][side < 0 ? id - 1 : id + 1];
                    double rvb = F.f[F_SRVB][side < 0 ? id - sj : id + sj];
                    double rvc = F.f[F_SRVC][side < 0 ? id - sk : id + sk];
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        double v = 0.5 * (rva * dn[0][m] + rvb * dn[1][m] + rvc * dn[2][m]);
                        r0[m] = MODE == 0 ? r0[m] + v : r0[m] - v;
                    }
                }
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    double *dq = F.f[F_DQ1 + m];
                    double own = dq[id];
                    if (MODE == 0) {
                        F.f[F_RHS1 + m][id] = own;  // store_rhs_nb
                        dq[id] = (-own + r0[m]) * coed;
                    } else {
                        dq[id] = own - r0[m] * coed;
                    }
                }
            } else {
                double lo[3][5], hi[3][5];
                const int dims[3] = {ni, nj, nk};
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    double dn[5];
#pragma unroll
                    for (int m = 0; m < 5; m++) dn[m] = cc[d] == 1 ? 0.0 : F.f[F_DQ1 + m][id - sts[d]];
                    nbr_term(P, F, B, id, d, cc[d], -1, dn, lo[d]);
#pragma unroll
                    for (int m = 0; m < 5; m++) dn[m] = cc[d] == dims[d] ? 0.0 : F.f[F_DQ1 + m][id + sts[d]];
                    nbr_term(P, F, B, id, d, cc[d], 1, dn, hi[d]);
                }
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    r0[m] = 1.0 * (lo[0][m] + lo[1][m] + lo[2][m] - hi[0][m] - hi[1][m] - hi[2][m]);
                    F.f[F_DQ1 + m][id] = (r0[m] - F.f[F_RHS1 + m][id]) * coed;
                }
            }
        }
        __syncthreads();
        if (p == plast) break;
    }
}

void launch_lhs(const LaunchCtx &c) {
    int zg = (int)((c.nzero + 255) / 256);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
    k_sweep<0><<<c.nblocks, 1024, 0, c.stream>>>(*c.P, *c.F, c.blocks);
    k_sweep<1><<<c.nblocks, 1024, 0, c.stream>>>(*c.P, *c.F, c.blocks);
    k_sweep<2><<<c.nblocks, 1024, 0, c.stream>>>(*c.P, *c.F, c.blocks);
    k_sweep<3><<<c.nblocks, 1024, 0, c.stream>>>(*c.P, *c.F, c.blocks);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
}

}  // namespace wcns
