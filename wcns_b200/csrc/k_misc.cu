// k_misc.cu -- pointwise phases of the WCNS step:
//   initial_q_dq_c_t (sub_tgh.f90:1-32): temperature (get_c_t_only
//     RHS.f90:307-409) and dq = 0 (set_dq_to_0 PreProcess.f90:1189-1205).
//     Sound speed, Sutherland viscosity and the conservative variables are
//     recomputed where they are used, from the same expressions.
//   timestep_tgh (sub_tgh.f90:1270-1348): spectinv (Convect.f90:1338-1461),
//     spectvisl (LHS.f90:243-343), localdt0 (LHS.f90:1343-1377) and the
//     LU-SGS diagonal getcoed (LHS.f90:602-645).
//   update_limited (Sub2.f90:603-794).
//   residual_curve (PostProcess.f90:1195-1347).
//   communicate_dq_npp / communicate_pv_npp (parallel.f90:3020-3326).
#include <cooperative_groups.h>

#include <algorithm>

#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace cg = cooperative_groups;

namespace wcns {

__device__ __forceinline__ void decode(const DevBlock &B, long long p, int &i, int &j, int &k) { decode_point(B, p, i, j, k); }

// ---------------------------------------------------------------------------
// initial_q_dq_c_t (sub_tgh.f90:1-32) at one interior point: dq = 0 and, for
// the viscous path, T and the Sutherland viscosity (plus T on the three
// ghost layers of the faces the point sits on)
__device__ __forceinline__ void init_point(const DevParams &P, DevFields &F, const DevBlock &B, int i, int j, int k,
                                           long long id) {
    const double gama = P.gama, moo2 = B.moo2;
    double *r = F.f[F_R], *p = F.f[F_P], *t = F.f[F_T];
#pragma unroll
    for (int m = 0; m < 5; m++) F.f[F_DQ1 + m][id] = 0.0;
    if (P.nvis != 1) return;
    t[id] = moo2 * (gama * p[id] / r[id]);
    F.f[F_VISL][id] = sutherland(P, t[id]);  // compute_visl_ns (GasModel.f90:219-235)
    // ghost layers of the face this point sits on
    int dims[3] = {B.ni, B.nj, B.nk};
    int c[3] = {i, j, k};
    for (int d = 0; d < 3; d++) {
        long long st = dstride(B, d);
        for (int s = 0; s < 2; s++) {
            if (c[d] != (s ? dims[d] : 1)) continue;
            long long sg = s ? st : -st;
            long long i1 = id + sg, i2 = id + 2 * sg, i3 = id + 3 * sg;
            double a2 = gama * p[i1] / r[i1];
            t[i1] = moo2 * a2;
            a2 = gama * p[i2] / r[i2];
            t[i2] = moo2 * a2;
            if (d != 0) a2 = gama * p[i3] / fabs(r[i3]);  // i faces reuse a2 (RHS.f90:351-353)
            t[i3] = moo2 * a2;
        }
    }
}

// timestep_tgh (sub_tgh.f90:1270-1348) at one interior point: spectral radii,
// dtdt and the LU-SGS diagonal coefficient; point-local, reading the point's
// own T
__device__ __forceinline__ void timestep_point(const DevParams &P, DevFields &F, long long id) {
    double rm = F.f[F_R][id], um = F.f[F_U][id], vm = F.f[F_V][id], wm = F.f[F_W][id], pm = F.f[F_P][id];
    double cm = sqrt(P.gama * pm / rm);
    double kx = F.f[F_KCX][id], ky = F.f[F_KCY][id], kz = F.f[F_KCZ][id], kt = 0.0;
    double ex = F.f[F_ETX][id], ey = F.f[F_ETY][id], ez = F.f[F_ETZ][id], et = 0.0;
    double cx = F.f[F_CTX][id], cy = F.f[F_CTY][id], cz = F.f[F_CTZ][id], ct = 0.0;
    double cita = kx * um + ky * vm + kz * wm + kt;
    double citb = ex * um + ey * vm + ez * wm + et;
    double citc = cx * um + cy * vm + cz * wm + ct;
    double cgma = sqrt(kx * kx + ky * ky + kz * kz);
    double cgmb = sqrt(ex * ex + ey * ey + ez * ez);
    double cgmc = sqrt(cx * cx + cy * cy + cz * cz);
    double ra = fabs(cita) + cm * cgma, rb = fabs(citb) + cm * cgmb, rc = fabs(citc) + cm * cgmc;
    double sva = 0.0, svb = 0.0, svc = 0.0;
    if (P.nvis == 1 && P.csrv > 0.0) {
        double rm_vol = rm * F.f[F_VOL][id];
        double ri = kx * kx + ky * ky + kz * kz;
        double rj = ex * ex + ey * ey + ez * ez;
        double rk = cx * cx + cy * cy + cz * cz;
        double vis = sutherland(P, F.f[F_T][id]);
        if (F.f[F_VIST]) vis = vis + F.f[F_VIST][id];  // spectvist, LHS.f90:141-241
        double coef = 2.0 * vis / (P.reynolds * rm_vol + SMALL);
        double coef1 = P.csrv * coef;
        sva = coef1 * ri;
        svb = coef1 * rj;
        svc = coef1 * rk;
    }
    F.f[F_SRA][id] = ra;
    F.f[F_SRB][id] = rb;
    F.f[F_SRC][id] = rc;
    F.f[F_SRVA][id] = sva;
    F.f[F_SRVB][id] = svb;
    F.f[F_SRVC][id] = svc;
    double rv = sva + svb + svc;
    double rabc = ra + rb + rc + rv;
    double dt;
    if (P.timedt_rate > SMALL) {
        double a = P.cfl / rabc, b = P.timedt_rate / F.f[F_VOL][id];
        dt = a < b ? a : b;
    } else {
        dt = P.cfl / rabc;
    }
    F.f[F_DTDT][id] = dt;
    double rad_ns = ra + rb + rc;
    if (P.nvis == 1) rad_ns = rad_ns + sva + svb + svc;
    double ctt = 1.0 / dt;
    F.f[F_COED][id] = 1.0 / (ctt + 1.0 * 1.0 * rad_ns);
}

template <bool INIT, bool TIMESTEP>
__global__ void k_init_timestep(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int nblocks) {
    const int bi = blockIdx.y;
    const DevBlock B = blocks[bi];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(B, q, i, j, k);
        long long id = gidx(B, i, j, k);
        if (INIT) init_point(P, F, B, i, j, k, id);
        if (TIMESTEP) timestep_point(P, F, id);
    }
}

template <bool INIT, bool TIMESTEP>
static void launch_init_timestep_t(const LaunchCtx &c) {
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
    dim3 grid((unsigned)((maxp + 255) / 256), c.nblocks);
    k_init_timestep<INIT, TIMESTEP><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, c.nblocks);
}

void launch_init(const LaunchCtx &c) { launch_init_timestep_t<true, false>(c); }
void launch_timestep(const LaunchCtx &c) { launch_init_timestep_t<false, true>(c); }
// both at once, as the step runs them back to back: every value the time
// step reads at a point is the point's own, written just before
void launch_init_timestep(const LaunchCtx &c) { launch_init_timestep_t<true, true>(c); }

// ---------------------------------------------------------------------------
// update_limited: pass A (parallel) + ordered fix-up of non-physical points
__global__ void k_update(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int *bad_count,
                         long long *bad_list) {
    const int bi = blockIdx.y;
    const DevBlock B = blocks[bi];
    const double gama = P.gama, gamam1 = gama - 1.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(B, q, i, j, k);
        long long id = gidx(B, i, j, k);
        double r0 = F.f[F_R][id], u0 = F.f[F_U][id], v0 = F.f[F_V][id], w0 = F.f[F_W][id], p0 = F.f[F_P][id];
        // prim_to_q (Sub1.f90:106-131) as get_q_only stored it
        double qq[5];
        qq[0] = r0;
        qq[1] = r0 * u0;
        qq[2] = r0 * v0;
        qq[3] = r0 * w0;
        qq[4] = p0 / (gama - 1.0) + 0.5 * r0 * (u0 * u0 + v0 * v0 + w0 * w0);
        double dq[5], qt[5];
#pragma unroll
        for (int m = 0; m < 5; m++) { dq[m] = F.f[F_DQ1 + m][id]; qt[m] = qq[m] + dq[m]; }
        double rm = qt[0], rm1 = 1.0 / rm;
        double um = qt[1] * rm1, vm = qt[2] * rm1, wm = qt[3] * rm1, em = qt[4];
        double pm = gamam1 * (em - 0.5 * rm * (um * um + vm * vm + wm * wm));
        double pd = fabs((pm - p0) / p0) + -0.3;
        double mx = 0.0 > pd ? 0.0 : pd;
        double Falpha = 1. / (1. + 2. * mx);
#pragma unroll
        for (int m = 0; m < 5; m++) qt[m] = qq[m] + dq[m] * Falpha;
        rm = qt[0];
        rm1 = 1.0 / rm;
        um = qt[1] * rm1;
        vm = qt[2] * rm1;
        wm = qt[3] * rm1;
        em = qt[4];
        pm = gamam1 * (em - 0.5 * rm * (um * um + vm * vm + wm * wm));
        F.f[F_OLD1][id] = r0;
        F.f[F_OLD2][id] = u0;
        F.f[F_OLD3][id] = v0;
        F.f[F_OLD4][id] = w0;
        F.f[F_OLD5][id] = p0;
        if (pm <= PMIN_LIMIT || rm <= RMIN_LIMIT || pm >= PMAX_LIMIT || rm >= RMAX_LIMIT) {
            int slot = atomicAdd(&bad_count[bi], 1);
            if (slot < BAD_CAP) bad_list[(long long)bi * BAD_CAP + slot] = id;
        }
        F.f[F_R][id] = rm;
        F.f[F_U][id] = um;
        F.f[F_V][id] = vm;
        F.f[F_W][id] = wm;
        F.f[F_P][id] = pm;
    }
}

// Bad points are handled in the reference's loop order: lower neighbours
// already hold updated values, upper interior neighbours still the old ones.
__global__ void k_update_fix(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int *bad_count,
                             long long *bad_list, int *err) {
    const int bi = blockIdx.x;
    if (threadIdx.x != 0) return;
    const DevBlock B = blocks[bi];
    int n = bad_count[bi];
    if (n == 0) return;
    long long lim = (long long)B.ni * B.nj * B.nk / 64;
    if (n > lim || n >= 500 || n > BAD_CAP) {
        atomicAdd(&err[ERR_UPDATE_BLOCKS], 1);
        bad_count[bi] = 0;
        return;
    }
    long long *lst = bad_list + (long long)bi * BAD_CAP;
    for (int a = 1; a < n; a++) {
        long long v = lst[a];
        int b = a - 1;
        while (b >= 0 && lst[b] > v) { lst[b + 1] = lst[b]; b--; }
        lst[b + 1] = v;
    }
    const long long sx = 1, sy = B.gx, sz = (long long)B.gx * B.gy;
    for (int e = 0; e < n; e++) {
        long long id = lst[e];
        long long rel = id - B.off;
        int i = (int)(rel % B.gx) - 2, j = (int)((rel / B.gx) % B.gy) - 2, k = (int)(rel / sz) - 2;
        const long long nb[6] = {id - sx, id - sy, id - sz, id + sz, id + sy, id + sx};
        const bool upper_int[6] = {false, false, false, k + 1 <= B.nk, j + 1 <= B.nj, i + 1 <= B.ni};
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int q = 0; q < 6; q++) {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                double v = upper_int[q] ? F.f[F_OLD1 + m][nb[q]] : F.f[F_R + m][nb[q]];
                acc[m] = acc[m] + v;
            }
        }
        double rnp = 6.0;
#pragma unroll
        for (int m = 0; m < 5; m++) F.f[F_R + m][id] = acc[m] / rnp;
    }
    bad_count[bi] = 0;
    (void)P;
}

void launch_update(const LaunchCtx &c) {
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
    dim3 grid((unsigned)((maxp + 255) / 256), c.nblocks);
    k_update<<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, c.bad_count, c.bad_list);
    k_update_fix<<<c.nblocks, 32, 0, c.stream>>>(*c.P, *c.F, c.blocks, c.bad_count, c.bad_list, c.err);
}

// ---------------------------------------------------------------------------
// residual_curve: per block sum and max of (|dq|/(dtdt*vol))^2 over 2..n-1
__global__ void k_residual_partial(DevFields F, const DevBlock *__restrict__ blocks, double *partial, int ctas) {
    const int bi = blockIdx.y;
    const DevBlock B = blocks[bi];
    int mi = B.ni - 2, mj = B.nj - 2, mk = B.nk - 2;
    long long np = (mi > 0 && mj > 0 && mk > 0) ? (long long)mi * mj * mk : 0;
    double s = 0.0, mx = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (q < 0x7fffffffLL) {  // 32-bit divisions where they suffice
            const int qq = (int)q, r = qq / mi;
            i = qq - r * mi + 2;
            j = r % mj + 2;
            k = r / mj + 2;
        } else {
            i = (int)(q % mi) + 2;
            j = (int)((q / mi) % mj) + 2;
            k = (int)(q / ((long long)mi * mj)) + 2;
        }
        long long id = gidx(B, i, j, k);
        double dtime1 = 1.0 / (F.f[F_DTDT][id] * F.f[F_VOL][id]);
#pragma unroll
        for (int m = 0; m < 5; m++) {
            double d = fabs(F.f[F_DQ1 + m][id]) * dtime1;
            s = s + d * d;
            mx = d > mx ? d : mx;
        }
    }
    __shared__ double ss[256], sm[256];
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
            sm[threadIdx.x] = sm[threadIdx.x + w] > sm[threadIdx.x] ? sm[threadIdx.x + w] : sm[threadIdx.x];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * ((long long)bi * ctas + blockIdx.x)] = ss[0];
        partial[2 * ((long long)bi * ctas + blockIdx.x) + 1] = sm[0];
    }
}

__global__ void k_residual_final(const DevBlock *__restrict__ blocks, int nblocks, const double *partial, int ctas,
                                 double *out, double *rms_slot) {
    // all partials are fetched in parallel into shared memory first; one
    // thread then sums them in the fixed order (block by block, CTA by CTA)
    extern __shared__ double sp[];
    const int n2 = 2 * nblocks * ctas;
    for (int e = threadIdx.x; e < n2; e += blockDim.x) sp[e] = partial[e];
    __syncthreads();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double total = 0.0;
    long long np = 0;
    for (int b = 0; b < nblocks; b++) {
        double s = 0.0, mx = 0.0;
        for (int c = 0; c < ctas; c++) {
            s = s + sp[2 * (b * ctas + c)];
            double m = sp[2 * (b * ctas + c) + 1];
            mx = m > mx ? m : mx;
        }
        total = total + s;
        long long npb = (long long)(blocks[b].ni - 2) * (blocks[b].nj - 2) * (blocks[b].nk - 2) * 5;
        out[b] = s / (double)npb;
        out[nblocks + b] = mx;
        np += npb;
    }
    double rms = sqrt(total / (double)np);
    out[2 * nblocks] = rms;
    if (rms_slot) *rms_slot = rms;
}

// dq -= c1, dq -= c2 (viscous) or dq += c1, dq += c2 (inviscid) over the
// interior points, after direction 0 updated dq in place: the same sequence
// of operations as three directions applied one after the other
__global__ void k_combine_dq(DevFields F, const DevBlock *__restrict__ blocks, const double *__restrict__ c1,
                             const double *__restrict__ c2, long long stride, int sub) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(B, q, i, j, k);
        const long long id = gidx(B, i, j, k);
#pragma unroll
        for (int m = 0; m < 5; m++) {
            double v = F.f[F_DQ1 + m][id];
            if (c1) v = sub ? v - c1[m * stride + id] : v + c1[m * stride + id];
            if (c2) v = sub ? v - c2[m * stride + id] : v + c2[m * stride + id];
            F.f[F_DQ1 + m][id] = v;
        }
    }
}

// The three directions of one residual kind.  The FP64 inviscid kernels
// fill the device on their own, so they run one after the other, each adding
// into dq in place (3.52 -> 3.39 ms per channel step against the concurrent
// form).  The viscous and the mixed-precision kernels gain from running
// directions 1 and 2 beside direction 0 on the side streams (3.30 against
// 3.62 ms serial for the FP64 viscous); their fluxes go to the contribution
// buffers, which k_combine_dq adds in the reference's direction order.
void launch_rhs_dirs(const LaunchCtx &c, bool vis) {
    if (!vis && !c.mixed) {
        for (int d = 0; d < 3; d++) launch_rhs_invis(c, d, c.stream, nullptr);
        return;
    }
    const DirTable *T = c.mixed ? (vis ? c.vis_mx : c.inv_mx) : (vis ? c.vis : c.inv);
    double *out[3] = {nullptr, c.contrib, c.contrib + 5 * c.total};
    const bool has[3] = {T[0].ngroups > 0, T[1].ngroups > 0, T[2].ngroups > 0};
    cudaEventRecord(c.ev_fork, c.stream);
    for (int d = 1; d <= 2; d++) {
        cudaStreamWaitEvent(c.side[d - 1], c.ev_fork, 0);
        if (vis) launch_rhs_vis(c, d, c.side[d - 1], out[d]);
        else launch_rhs_invis(c, d, c.side[d - 1], out[d]);
        cudaEventRecord(c.ev_join[d - 1], c.side[d - 1]);
    }
    if (vis) launch_rhs_vis(c, 0, c.stream, nullptr);
    else launch_rhs_invis(c, 0, c.stream, nullptr);
    cudaStreamWaitEvent(c.stream, c.ev_join[0], 0);
    cudaStreamWaitEvent(c.stream, c.ev_join[1], 0);
    if (has[1] || has[2]) {
        long long maxp = 0;
        for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
        dim3 grid((unsigned)((maxp + 255) / 256), c.nblocks);
        k_combine_dq<<<grid, 256, 0, c.stream>>>(*c.F, c.blocks, has[1] ? out[1] : nullptr, has[2] ? out[2] : nullptr,
                                                 c.total, vis ? 1 : 0);
    }
}

int setup_residual(int nblocks, int ctas) {
    const size_t bytes = sizeof(double) * 2 * (size_t)nblocks * ctas;
    if (bytes > 200 * 1024) return -1;
    if (bytes > 48 * 1024) cudaFuncSetAttribute(k_residual_final, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return 0;
}

// interior points of one field between the ghosted layout and a contiguous
// staging buffer (block b at stage[first[b] + p], p = (i-1) + ni*((j-1) + nj*(k-1)),
// the flow-file order): TO_DEV scatters the staged values into the field,
// otherwise the field is gathered into the buffer
template <bool TO_DEV>
__global__ void k_interior_stage(const DevBlock *__restrict__ blocks, const long long *__restrict__ first,
                                 double *field, double *stage) {
    const DevBlock B = blocks[blockIdx.y];
    double *sb = stage + first[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(B, q, i, j, k);
        const long long id = gidx(B, i, j, k);
        if (TO_DEV) field[id] = sb[q];
        else sb[q] = field[id];
    }
}

void launch_interior_stage(const LaunchCtx &c, bool to_device, const long long *first, double *field, double *stage) {
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
    const dim3 grid((unsigned)std::min<long long>((maxp + 255) / 256, 2048), c.nblocks);
    if (to_device) k_interior_stage<true><<<grid, 256, 0, c.stream>>>(c.blocks, first, field, stage);
    else k_interior_stage<false><<<grid, 256, 0, c.stream>>>(c.blocks, first, field, stage);
}

void launch_residual(const LaunchCtx &c, double *rms_slot) {
    dim3 grid(c.res_ctas_per_block, c.nblocks);
    k_residual_partial<<<grid, 256, 0, c.stream>>>(*c.F, c.blocks, c.res_partial, c.res_ctas_per_block);
    k_residual_final<<<1, 256, sizeof(double) * 2 * c.nblocks * c.res_ctas_per_block, c.stream>>>(
        c.blocks, c.nblocks, c.res_partial, c.res_ctas_per_block, c.res_out, rms_slot);
}

// ---------------------------------------------------------------------------
// interface averaging
__global__ void k_snapshot(DevFields F, const long long *__restrict__ pts, int n, double *snap, int which) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        long long id = pts[s];
        if (which == 0) {
            double vol = F.f[F_VOL][id];
#pragma unroll
            for (int m = 0; m < 5; m++) snap[(long long)m * n + s] = F.f[F_DQ1 + m][id] / vol;
        } else {
#pragma unroll
            for (int m = 0; m < 6; m++) snap[(long long)m * n + s] = F.f[F_R + m][id];
        }
    }
}

// boundary_match_dq_2pm / boundary_match_pv_2pm: one cluster per block walks
// the block's groups of independent pairs in order, with a cluster barrier
// between groups (an edge point can belong to two regions; the host puts a
// pair after every earlier pair it depends on).  Then, as
// boundary_match_dq_3pp / boundary_match_pv_3pp, the block's points shared
// by more than two blocks take the mean over all copies (snapshot values,
// member order); those means only read the snapshot and overwrite whatever
// the pairs left at the point.
__global__ void k_match(DevFields F, const PairEntry *__restrict__ pairs, const int *__restrict__ blk_reg_first,
                        const int *__restrict__ reg_pair_first, const int *__restrict__ comp_first,
                        const int *__restrict__ comp_n, const int *__restrict__ mem_slot,
                        const int *__restrict__ mem_comp, const long long *__restrict__ mem_idx,
                        const int *__restrict__ blk_mem_first, const double *__restrict__ snap, int nsnap, int which) {
    cg::cluster_group cluster = cg::this_cluster();
    const int bi = blockIdx.x / BC_CLUSTER;
    const int t0 = (int)cluster.block_rank() * blockDim.x + threadIdx.x, tstride = BC_CLUSTER * blockDim.x;
    for (int r = blk_reg_first[bi]; r < blk_reg_first[bi + 1]; r++) {
        for (int e = reg_pair_first[r] + t0; e < reg_pair_first[r + 1]; e += tstride) {
            PairEntry pe = pairs[e];
            if (which == 0) {
                double vs = F.f[F_VOL][pe.own];
                if (pe.same) {
                    double vol_p = vs / F.f[F_VOL][pe.partner];
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        double *dq = F.f[F_DQ1 + m];
                        dq[pe.own] = 0.5 * (dq[pe.partner] * vol_p + dq[pe.own]);
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        double *dq = F.f[F_DQ1 + m];
                        dq[pe.own] = 0.5 * (snap[(long long)m * nsnap + pe.partner_slot] * vs + dq[pe.own]);
                    }
                }
            } else {
#pragma unroll
                for (int m = 0; m < 6; m++) {
                    double *x = F.f[F_R + m];
                    double tv = pe.same ? x[pe.partner] : snap[(long long)m * nsnap + pe.partner_slot];
                    x[pe.own] = 0.5 * (tv + x[pe.own]);
                }
            }
        }
        cluster.sync();
    }
    const int nf = which == 0 ? 5 : 6;
    const int e0 = blk_mem_first[bi], ne = blk_mem_first[bi + 1] - e0;
    for (int t = t0; t < nf * ne; t += tstride) {
        const int m = t / ne, e = e0 + (t - m * ne);
        const int cc = mem_comp[e];
        const int f0 = comp_first[cc], np = comp_n[cc];
        const long long id = mem_idx[e];
        const double *sm = snap + (long long)m * nsnap;
        double s = 0.0;
        for (int q = 0; q < np; q++) {
            double v = sm[mem_slot[f0 + q]];
            if (which == 1) v = v / 1.0;
            s = s + v;
        }
        s = s / (np * 1.0);
        if (which == 0) F.f[F_DQ1 + m][id] = s * F.f[F_VOL][id];
        else F.f[F_R + m][id] = s * 1.0;
    }
}

void launch_communicate(const LaunchCtx &c, int which) {
    if (c.nsnap == 0) return;
    k_snapshot<<<(c.nsnap + 255) / 256, 256, 0, c.stream>>>(*c.F, c.snap_pts, c.nsnap, c.snap, which);
    launch_block_clusters(k_match, c.nblocks, 256, c.stream, *c.F, (const PairEntry *)c.pairs,
                          (const int *)c.blk_reg_first, (const int *)c.reg_pair_first, (const int *)c.comp_first,
                          (const int *)c.comp_n, (const int *)c.mem_slot, (const int *)c.mem_comp,
                          (const long long *)c.mem_idx, (const int *)c.blk_mem_first, (const double *)c.snap, c.nsnap,
                          which);
}

}  // namespace wcns
