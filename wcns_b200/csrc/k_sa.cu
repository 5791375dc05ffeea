// k_sa.cu -- Spalart-Allmaras turbulence model: turbulence(nb) ->
// differential_model_turbulence (turblence.f90:15-103) with nlamtur=1,
// nameturb='SA', ncmpcor<=9, ndes=0, ntrans=0, nwtmax=0 and method=1
// (finite differences), for all blocks at once.
//
// Per step:
//   k_sa_point<SA_DMU>    derivatives of qke at points 1..n (dfidxyz_center)
//   k_sa_point<SA_RHS>    per interior point: SA source, diffusion, spectral
//                         radius and first-order upwind convection, in the
//                         reference's order of accumulation into dqke/spec
//   k_sa_lusgs            scalar LU-SGS, forward and backward hyperplane
//                         wavefronts, one CTA per block
//   k_sa_point<SA_UPDATE> qke update, vist, kmaxlim clamp
// Set-up: k_sa_wall_dist (calc_wall_dists_parallel) and k_sa_init (init_SA).
#include "wcns_launch.h"

namespace wcns {

namespace {

constexpr double SA_CB1 = 0.1355, SA_CB2 = 0.622, SA_EPS = 1.0e-20;  // turblence.f90:2508-2513
constexpr double SA_CGA = 2. / 3.0;
constexpr double SA_CW2 = 0.3;
constexpr double SA_MUOO = 1.0e-1;    // inflow_turbulence, turblence.f90:3174
constexpr double SA_MINLIM = 1.0e-20; // update_turbulence, turblence.f90:589

enum SaPhase { SA_DMU = 0, SA_RHS = 1, SA_UPDATE = 2 };

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// dfidxyz_center, turblence.f90:753-849 (finite-difference branch)
__device__ __forceinline__ void center_deriv(const DevFields &F, const DevBlock &B, const double *fi, long long id,
                                             double *d) {
    const long long sj = B.gx, sk = (long long)B.gx * B.gy;
    double dkc = fi[id + 1] - fi[id - 1];
    double det = fi[id + sj] - fi[id - sj];
    double dct = fi[id + sk] - fi[id - sk];
    double ddx = dkc * F.f[F_KCX][id] + det * F.f[F_ETX][id] + dct * F.f[F_CTX][id];
    double ddy = dkc * F.f[F_KCY][id] + det * F.f[F_ETY][id] + dct * F.f[F_CTY][id];
    double ddz = dkc * F.f[F_KCZ][id] + det * F.f[F_ETZ][id] + dct * F.f[F_CTZ][id];
    double vol2 = 0.5 / F.f[F_VOL][id];
    d[0] = ddx * vol2;
    d[1] = ddy * vol2;
    d[2] = ddz * vol2;
}

// viscosity_equivalent_SA_r, turblence.f90:2785-2808
__device__ __forceinline__ double viseq_at(const DevFields &F, const SaFields &S, long long id) {
    return 1.5 * (F.f[F_VISL][id] / F.f[F_R][id] + S.qke[id]);
}

// flux_turbulence, turblence.f90:437-459, of the state at id
__device__ __forceinline__ double conv_flux(const DevFields &F, const SaFields &S, long long id, double nx, double ny,
                                            double nz, double npn) {
    double l1 = nx * F.f[F_U][id] + ny * F.f[F_V][id] + nz * F.f[F_W][id];
    l1 = 0.5 * (l1 + npn * sqrt(l1 * l1));
    return l1 * S.qke[id] * F.f[F_R][id];
}

__device__ void sa_rhs_point(const DevFields &F, const SaFields &S, const SaParams &P, const DevBlock &B, long long id) {
    const long long st[3] = {1, B.gx, (long long)B.gx * B.gy};
    // cal_rhs_source_SA, turblence.f90:2567-2686
    double du[3], dv[3], dw[3];
    center_deriv(F, B, F.f[F_U], id, du);
    center_deriv(F, B, F.f[F_V], id, dv);
    center_deriv(F, B, F.f[F_W], id, dw);
    const double ro = F.f[F_R][id], volume = F.f[F_VOL][id], vsl = F.f[F_VISL][id], vtbar = S.qke[id];
    const double romu = ro * vtbar;
    const double ds = S.dist[id];
    const double dn = ds > P.re ? ds : P.re;
    const double dn2 = dn * dn;
    const double reki2dn2 = P.reynolds * P.ki2 * dn2;
    const double kafan = romu / vsl;
    const double kf3 = pow(kafan, 3.0);
    const double fv1 = kf3 / (kf3 + P.cv13);
    const double fv2 = 1.0 - kafan / (1.0 + kafan * fv1);
    const double a = du[1] - dv[0], b = dv[2] - dw[1], c = dw[0] - du[2];
    const double omg = sqrt(a * a + b * b + c * c);
    double sbar = omg + vtbar / reki2dn2 * fv2;
    sbar = sbar > SA_EPS ? sbar : SA_EPS;
    double rbar = vtbar / (sbar * reki2dn2);
    rbar = rbar < 10.0 ? rbar : 10.0;
    const double rbar5 = pow(rbar, 5.0);
    const double gbar = rbar + SA_CW2 * rbar * (rbar5 - 1.0);
    const double gbar6 = pow(gbar, 6.0);
    const double fw = gbar * pow((1.0 + P.cw36) / (gbar6 + P.cw36), P.onesix);
    const double ft2 = 0.0;
    const double cpmu = SA_CB1 * (1.0 - ft2) * sbar;
    const double cdmu = (P.cw1 * fw - SA_CB1 * ft2 / P.ki2) * vtbar / dn2 / P.reynolds;
    const double sp = cpmu * vtbar, sd = cdmu * vtbar;
    const double dmx = S.dmu[0][id], dmy = S.dmu[1][id], dmz = S.dmu[2][id];
    const double dbar = SA_CB2 / SA_CGA * (dmx * dmx + dmy * dmy + dmz * dmz) * P.re;
    double dq = 0.0 - ro * (sp - sd + dbar) * volume;
    const double sm = cpmu - 2.0 * cdmu;
    double spec = 0.0 - (sm < 0.0 ? sm : 0.0) * volume;
    // cal_rhs_viscous_turbulence_dif_r, turblence.f90:1022-1185: half-point
    // fluxes on both sides of the point, directions i, j, k
    const double rre = P.re * ro;
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        const double *mx = F.f[F_KCX + 3 * d], *my = F.f[F_KCY + 3 * d], *mz = F.f[F_KCZ + 3 * d];
        double fvl[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const long long im = id + (h ? st[d] : 0), in = im - st[d];
            double nx = 0.5 * (mx[im] + mx[in]);
            double ny = 0.5 * (my[im] + my[in]);
            double nz = 0.5 * (mz[im] + mz[in]);
            double dmudx = S.dmu[0][im] + S.dmu[0][in];
            double dmudy = S.dmu[1][im] + S.dmu[1][in];
            double dmudz = S.dmu[2][im] + S.dmu[2][in];
            double vis = viseq_at(F, S, im) + viseq_at(F, S, in);
            fvl[h] = (dmudx * nx + dmudy * ny + dmudz * nz) * vis * 0.25;
        }
        dq = dq - rre * (fvl[1] - fvl[0]);
    }
    // cal_spec_turbulence_r, turblence.f90:218-259
    {
        const double u = F.f[F_U][id], v = F.f[F_V][id], w = F.f[F_W][id];
        const double kx = F.f[F_KCX][id], ky = F.f[F_KCY][id], kz = F.f[F_KCZ][id];
        const double ex = F.f[F_ETX][id], ey = F.f[F_ETY][id], ez = F.f[F_ETZ][id];
        const double cx = F.f[F_CTX][id], cy = F.f[F_CTY][id], cz = F.f[F_CTZ][id];
        double unx = u * kx + v * ky + w * kz;
        double uny = u * ex + v * ey + w * ez;
        double unz = u * cx + v * cy + w * cz;
        spec = spec + fabs(unx) + fabs(uny) + fabs(unz) + 1.0 / (F.f[F_DTDT][id] * P.timedt_turb);
        double nx = kx * kx + ky * ky + kz * kz;
        double ny = ex * ex + ey * ey + ez * ez;
        double nz = cx * cx + cy * cy + cz * cz;
        double vis = viseq_at(F, S, id) / volume;
        spec = spec + P.re * 2.0 * vis * (nx + ny + nz);
    }
    // cal_rhs_inviscous_turbulence / NND_turbulence, turblence.f90:291-435.
    // xk = xb = 0 (never assigned in the reference), so the minmod slopes
    // are zeros and the half-point states are the neighbouring points'
    // values exactly: fc(l) = f+(q(l-1)) + f-(q(l)).
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        const double *mx = F.f[F_KCX + 3 * d], *my = F.f[F_KCY + 3 * d], *mz = F.f[F_KCZ + 3 * d];
        double fc[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const long long i1 = id + (h ? st[d] : 0), i0 = i1 - st[d];
            double nx = 0.50 * (mx[i0] + mx[i1]);
            double ny = 0.50 * (my[i0] + my[i1]);
            double nz = 0.50 * (mz[i0] + mz[i1]);
            double fl = conv_flux(F, S, i0, nx, ny, nz, 1.0);
            double fr = conv_flux(F, S, i1, nx, ny, nz, -1.0);
            fc[h] = fl + fr;
        }
        dq = dq + (fc[1] - fc[0]);
    }
    S.dqke[id] = dq;
    S.spec[id] = spec;
}

// cal_vist_SA (turblence.f90:2735-2760) at one point
__device__ __forceinline__ double vist_of(double r, double qke, double visl, double cv13) {
    double romu = r * qke;
    double kafan = romu / visl;
    double kf3 = pow(kafan, 3.0);
    double fv1 = kf3 / (kf3 + cv13);
    return romu * fv1;
}

// One kernel for the point-wise phases.  lo: first index of the range in
// every direction (1 for SA_DMU, 2 for SA_RHS, 0 for SA_UPDATE); the range
// ends at n - (lo == 2 ? 1 : 0).  The right-hand side runs four CTAs per SM
// (64 registers, a little spill): 0.74 -> 0.58 ms per channel step against
// two CTAs of 109 registers; the other phases keep their own register counts.
template <int PHASE>
__global__ void __launch_bounds__(256, PHASE == SA_RHS ? 4 : 0) k_sa_point(DevFields F, SaFields S, SaParams P, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    const int lo = PHASE == SA_DMU ? 1 : PHASE == SA_RHS ? 2 : 0;
    const int hi_off = PHASE == SA_RHS ? 1 : 0;
    const int mi = B.ni - hi_off - lo + 1, mj = B.nj - hi_off - lo + 1, mk = B.nk - hi_off - lo + 1;
    if (mi <= 0 || mj <= 0 || mk <= 0) return;
    const long long np = (long long)mi * mj * mk;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        {
            const long long r = q / mi;
            i = (int)(q - r * mi) + lo;
            j = (int)(r % mj) + lo;
            k = (int)(r / mj) + lo;
        }
        const long long id = gidx(B, i, j, k);
        if (PHASE == SA_DMU) {
            double d[3];
            center_deriv(F, B, S.qke, id, d);
            S.dmu[0][id] = d[0];
            S.dmu[1][id] = d[1];
            S.dmu[2][id] = d[2];
        } else if (PHASE == SA_RHS) {
            sa_rhs_point(F, S, P, B, id);
        } else {
            const bool in1 = i >= 1 && j >= 1 && k >= 1;
            const bool in2 = i >= 2 && j >= 2 && k >= 2 && i <= B.ni - 1 && j <= B.nj - 1 && k <= B.nk - 1;
            double vt = S.vist[id];
            if (in1) {
                double qk = S.qke[id];
                const double r = F.f[F_R][id];
                if (in2) {  // update_turbulence, turblence.f90:606-615
                    double qn = qk + S.dqke[id] / r, lim = SA_MINLIM * SA_MUOO;
                    qk = dmax(qn, lim);
                    S.qke[id] = qk;
                }
                vt = vist_of(r, qk, F.f[F_VISL][id], P.cv13);
            }
            if (P.kmaxlim > 1.0e-15) vt = dmin(vt, P.kmaxlim * F.f[F_VISL][id]);  // max_control_turbulence
            S.vist[id] = vt;
        }
    }
}

// lusgs_turbulence, turblence.f90:477-558.  The lexicographic forward sweep
// reads the already updated lower neighbours (i-1, j-1, k-1) and the
// backward sweep the upper ones, so every hyperplane i+j+k = p can be
// updated at once after the previous one; one CTA per block walks the
// planes with a barrier in between (dqke stays in global memory, which the
// barrier makes visible to the whole CTA).
__device__ __forceinline__ double mxdq(const DevFields &F, long long nid, long long mid, int d, double dq, double npn) {
    // mxdq_std_turbulence (turblence.f90:560-583) with the neighbour's
    // velocity and the metrics of getrkec_mml at the neighbour (mid: the
    // neighbour with indices 0 and n+1 clamped to the block)
    double l1 = F.f[F_KCX + 3 * d][mid] * F.f[F_U][nid] + F.f[F_KCY + 3 * d][mid] * F.f[F_V][nid] +
                F.f[F_KCZ + 3 * d][mid] * F.f[F_W][nid];
    l1 = 0.5 * (l1 + npn * fabs(l1));
    return l1 * dq;
}

__global__ void __launch_bounds__(1024) k_sa_lusgs(DevFields F, SaFields S, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.x];
    const int ni = B.ni, nj = B.nj, nk = B.nk;
    if (ni < 3 || nj < 3 || nk < 3) return;
    const int wj = nj - 2, ncol = (nj - 2) * (nk - 2);
    const long long st[3] = {1, B.gx, (long long)B.gx * B.gy};
    const int n3[3] = {ni, nj, nk};
    double *dqke = S.dqke;
    for (int pass = 0; pass < 2; pass++) {
        const int np = (ni - 1) + (nj - 1) + (nk - 1) - 6 + 1;  // planes 6 .. (ni-1)+(nj-1)+(nk-1)
        for (int pp = 0; pp < np; pp++) {
            const int p = pass == 0 ? 6 + pp : (ni - 1) + (nj - 1) + (nk - 1) - pp;
            for (int t = threadIdx.x; t < ncol; t += blockDim.x) {
                const int j = 2 + t % wj, k = 2 + t / wj, i = p - j - k;
                if (i < 2 || i > ni - 1) continue;
                const long long id = gidx(B, i, j, k);
                const int c[3] = {i, j, k};
                double tt[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const long long nid = pass == 0 ? id - st[d] : id + st[d];
                    const int cn = pass == 0 ? c[d] - 1 : c[d] + 1;
                    // getrkec_mml clamps 0 -> 1 and n+1 -> n; neighbours of
                    // interior points stay within 1..n, so mid == nid
                    const long long mid = (cn == 0) ? nid + st[d] : (cn == n3[d] + 1) ? nid - st[d] : nid;
                    tt[d] = mxdq(F, nid, mid, d, dqke[nid], pass == 0 ? 1.0 : -1.0);
                }
                const double rhs0 = tt[0] + tt[1] + tt[2];
                if (pass == 0) dqke[id] = (rhs0 - dqke[id]) / S.spec[id];
                else dqke[id] = dqke[id] - rhs0 / S.spec[id];
            }
            __syncthreads();
        }
    }
}

// calc_wall_dists_parallel, parallel.f90:4313-4470: the squared distance to
// the nearest wall point (exact minimum, so the order of the wall list does
// not matter), then sqrt + small, at points 1..n.
constexpr int WD_TILE = 512;
// The wall points a block measures to are those of its own set of blocks
// joined through interfaces (wall_range[2b] .. wall_range[2b+1]): one case,
// also when independent cases share a context.
__global__ void __launch_bounds__(256) k_sa_wall_dist(SaFields S, const double *__restrict__ xyz, long long total,
                                                      const double *__restrict__ wall, const int *__restrict__ wall_range,
                                                      const DevBlock *__restrict__ blocks) {
    __shared__ double sw[3 * WD_TILE];
    const DevBlock B = blocks[blockIdx.y];
    const int wbeg = wall_range[2 * blockIdx.y], nwall = wall_range[2 * blockIdx.y + 1];
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = q < B.npts;
    long long id = 0;
    double xc = 0.0, yc = 0.0, zc = 0.0, dmn = 1.0e30;
    if (act) {
        int i, j, k;
        decode_point(B, q, i, j, k);
        id = gidx(B, i, j, k);
        xc = xyz[id];
        yc = xyz[total + id];
        zc = xyz[2 * total + id];
    }
    for (int w0 = wbeg; w0 < nwall; w0 += WD_TILE) {
        const int nt = nwall - w0 < WD_TILE ? nwall - w0 : WD_TILE;
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * nt; e += blockDim.x) sw[e] = wall[3 * (long long)w0 + e];
        __syncthreads();
        if (act)
            for (int w = 0; w < nt; w++) {
                double dx = xc - sw[3 * w], dy = yc - sw[3 * w + 1], dz = zc - sw[3 * w + 2];
                double dist = dx * dx + dy * dy + dz * dz;
                dmn = dist < dmn ? dist : dmn;
            }
    }
    if (act) S.dist[id] = sqrt(dmn) + SMALL;
}

// init_SA, turblence.f90:2701-2733: qke = muoo, vist = vt over -1..n+1
__global__ void k_sa_init(SaFields S, double vt, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    const int mi = B.ni + 3, mj = B.nj + 3, mk = B.nk + 3;
    const long long np = (long long)mi * mj * mk;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / mi;
        const int i = (int)(q - r * mi) - 1, j = (int)(r % mj) - 1, k = (int)(r / mj) - 1;
        const long long id = gidx(B, i, j, k);
        S.qke[id] = SA_MUOO;
        S.vist[id] = vt;
    }
}

long long max_points(const LaunchCtx &c, int extra) {
    long long m = 0;
    for (int b = 0; b < c.nblocks; b++) {
        const DevBlock &B = c.hblocks[b];
        long long n = (long long)(B.ni + extra) * (B.nj + extra) * (B.nk + extra);
        m = n > m ? n : m;
    }
    return m;
}

unsigned grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

}  // namespace

void launch_sa_setup(const LaunchCtx &c, const double *xyz, const double *wall, const int *wall_range, double vt) {
    k_sa_init<<<dim3(grid_for(max_points(c, 3)), c.nblocks), 256, 0, c.stream>>>(*c.SA, vt, c.blocks);
    k_sa_wall_dist<<<dim3((unsigned)((max_points(c, 0) + 255) / 256), c.nblocks), 256, 0, c.stream>>>(
        *c.SA, xyz, c.total, wall, wall_range, c.blocks);
}

int launch_turbulence(const LaunchCtx &c) {
    k_sa_point<SA_DMU><<<dim3(grid_for(max_points(c, 0)), c.nblocks), 256, 0, c.stream>>>(*c.F, *c.SA, *c.SAP, c.blocks);
    k_sa_point<SA_RHS><<<dim3(grid_for(max_points(c, 0)), c.nblocks), 256, 0, c.stream>>>(*c.F, *c.SA, *c.SAP, c.blocks);
    prof_mark(c, "sa_rhs");
    // large blocks: the scalar sweeps on the wide chunks of the mean-flow sweeps
    const int nl = (c.wide && c.wide->A.sa) ? launch_sa_lusgs_wide(c) : 1;
    if (nl == 1) k_sa_lusgs<<<c.nblocks, 1024, 0, c.stream>>>(*c.F, *c.SA, c.blocks);
    prof_mark(c, "sa_lusgs");
    k_sa_point<SA_UPDATE><<<dim3(grid_for(max_points(c, 1)), c.nblocks), 256, 0, c.stream>>>(*c.F, *c.SA, *c.SAP, c.blocks);
    prof_mark(c, "sa_update");
    return 3 + nl;
}

}  // namespace wcns
