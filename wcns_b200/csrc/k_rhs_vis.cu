// k_rhs_vis.cu -- laminar viscous residual.
//
// Restates r_h_s_vis (RHS.f90:2-30) -> WCNSE5_VIS_virtual
// (sub_tgh.f90:1511-1810):
//   * node derivatives of (u,v,w,T) along each index direction
//     (UVWT_DER_4th_virtual sub_tgh.f90:1909-2029 with
//     DUVWT_NODE_LINE_virtual 2217-2272) -> 12 fields, one kernel;
//   * per line and half node: VALUE_line_half_virtual (2335-2387),
//     VALUE_HALF_NODE_IJK (newvis.f90:421-554), half-node derivatives
//     (DUVWT_half_line_virtual 2277-2330), metric/volume/viscosity
//     interpolation (VALUE_HALF_NODE WCNSE5.f90:799-852), Cartesian
//     gradients (DUVWT_DXYZ WCNSE5.f90:854-890), stress and heat flux
//     (FLUX_VIS_LINE_new newvis.f90:283-349);
//   * per point: FLUX_DXYZ and dq -= re*dFv.
// The boundary flag of a line is the reference's uvwt(4,-2) test: -1 when the
// third ghost density is negative, otherwise the ghost temperature.
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

// ---------------------------------------------------------------------------
// node derivatives: one thread per interior point
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 4) k_node_deriv(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int nblocks) {
    int bi = blockIdx.y;
    if (bi >= nblocks) return;
    const DevBlock B = blocks[bi];
    long long np = B.npts;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_point(B, p, i, j, k);
        long long id = gidx(B, i, j, k);
        for (int d = 0; d < 3; d++) {
            int n = dimof(B, d);
            int l = d == 0 ? i : (d == 1 ? j : k);
            long long st = dstride(B, d);
            long long l0 = id - (long long)l * st;  // index of position 0 on the line
            double rl = __ldg(F.f[F_R] + l0 - 2 * st), rr = __ldg(F.f[F_R] + l0 + (long long)(n + 3) * st);
            bool fl = rl < 0.0 ? true : (__ldg(F.f[F_T] + l0 - 2 * st) < 0.0);
            bool fr = rr < 0.0 ? true : (__ldg(F.f[F_T] + l0 + (long long)(n + 3) * st) < 0.0);
            for (int m = 0; m < 4; m++) {
                const double *u = F.f[m == 3 ? F_T : F_U + m] + l0;
                auto U = [&](int x) { return __ldg(u + (long long)x * st); };
                double du;
                if (n <= NIJK2ND) {
                    du = 0.5 * (U(l + 1) - U(l - 1));
                } else if (fl && l == 1) {
                    du = (-11. * U(1) + 18. * U(2) - 9. * U(3) + 2. * U(4)) / 6.0;
                } else if (fl && l == 2) {
                    du = (-3.0 * U(1) + -10.0 * U(2) + 18.0 * U(3) + -6.0 * U(4) + 1.0 * U(5)) / 12.0;
                } else if (fr && l == n) {
                    du = -(-11. * U(n) + 18. * U(n - 1) - 9.0 * U(n - 2) + 2. * U(n - 3)) / 6.0;
                } else if (fr && l == n - 1) {
                    du = -(-3.0 * U(n) + -10.0 * U(n - 1) + 18.0 * U(n - 2) + -6.0 * U(n - 3) + 1.0 * U(n - 4)) / 12.0;
                } else {
                    du = (8.0 * (U(l + 1) - U(l - 1)) + -1.0 * (U(l + 2) - U(l - 2))) / 12.0;
                }
                F.f[F_DUV0 + m + 4 * d][id] = du;
            }
        }
    }
}

void launch_node_derivatives(const LaunchCtx &c) {
    if (c.mixed) return launch_node_derivatives_mx(c);
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
    int gx = (int)((maxp + 255) / 256);
    dim3 grid(gx, c.nblocks);
    k_node_deriv<<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, c.nblocks);
}

// ---------------------------------------------------------------------------
// viscous line flux
// ---------------------------------------------------------------------------
struct VisLine {
    long long l0;  // field index of position 0 on the line
    long long st;
    int n;
    bool fl, fr;
};

// Shared-memory staging of one line: VIS_NF values per point l = -1 .. n+2
// (slot l+1): u, v, w, T; the 8 node derivatives along the two other
// directions; the 9 metrics in the order kcx,etx,ctx,kcy,ety,cty,kcz,etz,ctz;
// vol; the two Sutherland viscosities.  Then the line's viscous flux, 5 x (n+1).
constexpr int VIS_NF = 24;
constexpr int VIS_MAX_LINES = 32;  // lines per CTA (short k-lines are grouped many to a CTA)
// 384 threads: the half-node fluxes of two 129-point lines (260) in one pass;
// two CTAs per SM at 80 registers
constexpr int VIS_THREADS = 320;
enum : int { VS_U = 0, VS_DN = 4, VS_MET = 12, VS_VOL = 21, VS_V1 = 22, VS_V2 = 23 };

__host__ __device__ inline int vis_line_stride(int n) {
    // doubles per line, padded to 2 mod 16 so that the lines of a group fall
    // on different banks when consecutive threads walk consecutive lines
    int raw = VIS_NF * (n + 4) + 5 * (n + 1);
    return (raw + 13) / 16 * 16 + 2;
}

// out == nullptr: dq -= re*dFv in place; otherwise re*dFv is stored in
// out[m*stride + point] for an ordered combine (k_combine_dq).  Two CTAs of
// 320 threads per SM, 96 registers with almost no spill: 3.30 ms per channel
// step for the three directions, against 3.40 at 384 threads and 80
// registers, 4.07 at three CTAs of 256 and 5.30 at one CTA of 512.
template <int dir>
__global__ void __launch_bounds__(VIS_THREADS, 2) k_rhs_vis(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                    const LineGroup *__restrict__ groups, int hmax, double *out,
                                                    long long stride) {
    extern __shared__ double smem[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir);
    const int H = n + 1, W = n + 4;
    const int NL = G.nl;
    const int LS = vis_line_stride(n);
    __shared__ VisLine lines[VIS_MAX_LINES];
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    if (threadIdx.x < NL) {
        int c[3];
        c[a1] = G.a0 + threadIdx.x;
        c[a2] = G.b;
        c[dir] = 0;
        VisLine L;
        L.l0 = gidx(B, c[0], c[1], c[2]);
        L.st = dstride(B, dir);
        L.n = n;
        double rl = F.f[F_R][L.l0 - 2 * L.st], rr = F.f[F_R][L.l0 + (long long)(n + 3) * L.st];
        L.fl = rl < 0.0 ? true : (F.f[F_T][L.l0 - 2 * L.st] < 0.0);
        L.fr = rr < 0.0 ? true : (F.f[F_T][L.l0 + (long long)(n + 3) * L.st] < 0.0);
        lines[threadIdx.x] = L;
    }
    __syncthreads();
    const bool posmajor = (dir == 0);
    const FastDiv dNL = fast_div_init(NL), dW = fast_div_init(W);
    // ---- stage the line inputs: one thread per (line, point), all VIS_NF
    // loads of the point issued back to back (coalesced along the line for
    // i-lines, across the group's neighbouring lines otherwise)
    {
        const int g0 = dir == 0 ? 1 : 0, g1 = dir == 2 ? 1 : 2;  // the two other directions
        for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
            const int qq = posmajor ? fdiv(e, dW) : fdiv(e, dNL);
            const int ln = posmajor ? qq : e - qq * NL;
            const int p = posmajor ? e - qq * W : qq;
            const VisLine &L = lines[ln];
            const int l = p - 1;
            const long long gi = L.l0 + (long long)l * L.st;
            const bool inner = l >= 1 && l <= n;
            double v[VIS_NF];
#pragma unroll
            for (int m = 0; m < 4; m++) v[VS_U + m] = __ldg(F.f[m == 3 ? F_T : F_U + m] + gi);
#pragma unroll
            for (int m = 0; m < 4; m++) {
                v[VS_DN + m] = inner ? __ldg(F.f[F_DUV0 + m + 4 * g0] + gi) : 0.0;
                v[VS_DN + 4 + m] = inner ? __ldg(F.f[F_DUV0 + m + 4 * g1] + gi) : 0.0;
            }
#pragma unroll
            for (int c = 0; c < 9; c++)  // kcx,etx,ctx,kcy,... = F_KCX + 3*(c%3) + c/3
                v[VS_MET + c] = inner ? __ldg(F.f[F_KCX + 3 * (c % 3) + c / 3] + gi) : 0.0;
            v[VS_VOL] = inner ? __ldg(F.f[F_VOL] + gi) : 0.0;
            // viscosity at the point, as the reference's visl/vist arrays:
            // mu + vist and mu*cp_prl + vist*cp_prt (vist = 0 when laminar)
            const double mu = inner ? sutherland(P, v[VS_U + 3]) : 0.0;
            const double vt = (inner && F.f[F_VIST]) ? __ldg(F.f[F_VIST] + gi) : 0.0;
            v[VS_V1] = inner ? mu + vt : 0.0;
            v[VS_V2] = inner ? mu * B.cp_prl + vt * B.cp_prt : 0.0;
            double *S = smem + (size_t)ln * LS + p;
#pragma unroll
            for (int f = 0; f < VIS_NF; f++) S[f * W] = v[f];
        }
    }
    __syncthreads();
    // ---- per half node: viscous flux fv (line-fastest in every direction, so
    // that the lanes of a warp share a position and its control path)
    for (int idx = threadIdx.x; idx < NL * H; idx += blockDim.x) {
        const int h = fdiv(idx, dNL);
        const int ln = idx - h * NL;
        const VisLine &L = lines[ln];
        const double *S = smem + (size_t)ln * LS;
        auto at = [&](int f, int x) { return S[f * W + x + 1]; };
        // (u,v,w,T) at the half node: VALUE_line_half_virtual
        double uh[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            auto Q = [&](int x) { return at(VS_U + m, x); };
            double v;
            if (n <= NIJK2ND) v = 0.5 * (Q(h) + Q(h + 1));
            else if (L.fl && h == 0) v = (35.0 * Q(1) + -35.0 * Q(2) + 21.0 * Q(3) + -5.0 * Q(4)) / 16.0;
            else if (L.fl && h == 1) v = (5.0 * Q(1) + 15.0 * Q(2) + -5.0 * Q(3) + 1.0 * Q(4)) / 16.0;
            else if (L.fr && h == n) v = (35.0 * Q(n) + -35.0 * Q(n - 1) + 21.0 * Q(n - 2) + -5.0 * Q(n - 3)) / 16.0;
            else if (L.fr && h == n - 1) v = (5.0 * Q(n) + 15.0 * Q(n - 1) + -5.0 * Q(n - 2) + 1.0 * Q(n - 3)) / 16.0;
            else v = (9.0 * (Q(h) + Q(h + 1)) + -1.0 * (Q(h + 2) + Q(h - 1))) / 16.0;
            uh[m] = v;
        }
        // derivatives at the half node: own direction from DUVWT_half_line_virtual,
        // the two others interpolated from node derivatives
        double dh[12];
#pragma unroll
        for (int g = 0; g < 3; g++) {
#pragma unroll
            for (int m = 0; m < 4; m++) {
                double v;
                if (g == dir) {
                    auto Q = [&](int x) { return at(VS_U + m, x); };
                    if (n <= NIJK2ND) v = Q(h + 1) - Q(h);
                    else if (L.fl && h == 0) v = (-71.0 * Q(1) + 141.0 * Q(2) + -93.0 * Q(3) + 23.0 * Q(4)) / 24.0;
                    else if (L.fl && h == 1) v = (-22.0 * Q(1) + 17.0 * Q(2) + 9.0 * Q(3) + -5.0 * Q(4) + 1.0 * Q(5)) / 24.0;
                    else if (L.fr && h == n) v = -(-71.0 * Q(n) + 141.0 * Q(n - 1) + -93.0 * Q(n - 2) + 23.0 * Q(n - 3)) / 24.0;
                    else if (L.fr && h == n - 1) v = -(-22.0 * Q(n) + 17.0 * Q(n - 1) + 9.0 * Q(n - 2) + -5.0 * Q(n - 3) + 1.0 * Q(n - 4)) / 24.0;
                    else v = (27.0 * (Q(h + 1) - Q(h)) + -1.0 * (Q(h + 2) - Q(h - 1))) / 24.0;
                } else {
                    const int slot = VS_DN + 4 * (g < dir ? g : g - 1) + m;
                    auto D = [&](int x) { return at(slot, x); };
                    v = value_half_node_ijk_at(D, n, h);
                }
                dh[m + 4 * g] = v;
            }
        }
        // metrics (kcx,etx,ctx,kcy,ety,cty,kcz,etz,ctz), volume, viscosities
        double kh[9];
#pragma unroll
        for (int c = 0; c < 9; c++) {
            auto Q = [&](int x) { return at(VS_MET + c, x); };
            kh[c] = value_half_node_at(Q, n, h);
        }
        double volh, v1h, v2h;
        {
            auto Q = [&](int x) { return at(VS_VOL, x); };
            auto V1 = [&](int x) { return at(VS_V1, x); };
            auto V2 = [&](int x) { return at(VS_V2, x); };
            volh = value_half_node_at(Q, n, h);
            v1h = value_half_node_at(V1, n, h);
            v2h = value_half_node_at(V2, n, h);
        }
        // DUVWT_DXYZ
        double dx[12];
#pragma unroll
        for (int m = 1; m <= 3; m++) {
            int m1 = m + m + m - 2, m2 = m1 + 1, m3 = m2 + 1;
            dx[m - 1] = (kh[m1 - 1] * dh[0] + kh[m2 - 1] * dh[4] + kh[m3 - 1] * dh[8]) / volh;
            dx[m + 2] = (kh[m1 - 1] * dh[1] + kh[m2 - 1] * dh[5] + kh[m3 - 1] * dh[9]) / volh;
            dx[m + 5] = (kh[m1 - 1] * dh[2] + kh[m2 - 1] * dh[6] + kh[m3 - 1] * dh[10]) / volh;
            dx[m + 8] = (kh[m1 - 1] * dh[3] + kh[m2 - 1] * dh[7] + kh[m3 - 1] * dh[11]) / volh;
        }
        // FLUX_VIS_LINE_new
        double vs = v1h;
        double vscc = vs * P.cc23;
        double dudx = dx[0], dudy = dx[1], dudz = dx[2];
        double dvdx = dx[3], dvdy = dx[4], dvdz = dx[5];
        double dwdx = dx[6], dwdy = dx[7], dwdz = dx[8];
        double t1 = vscc * (2.0 * dudx - dvdy - dwdz);
        double t5 = vscc * (2.0 * dvdy - dwdz - dudx);
        double t9 = vscc * (2.0 * dwdz - dudx - dvdy);
        double t2 = vs * (dudy + dvdx);
        double t3 = vs * (dudz + dwdx);
        double t6 = vs * (dvdz + dwdy);
        double kcp = v2h;
        const double nx = dir == 0 ? kh[0] : dir == 1 ? kh[1] : kh[2];
        const double ny = dir == 0 ? kh[3] : dir == 1 ? kh[4] : kh[5];
        const double nz = dir == 0 ? kh[6] : dir == 1 ? kh[7] : kh[8];
        double f1 = t1 * nx + t2 * ny + t3 * nz;
        double f2 = t2 * nx + t5 * ny + t6 * nz;
        double f3 = t3 * nx + t6 * ny + t9 * nz;
        double f4 = uh[0] * f1 + uh[1] * f2 + uh[2] * f3 + kcp * (dx[9] * nx + dx[10] * ny + dx[11] * nz);
        double *fv = smem + (size_t)ln * LS + (size_t)VIS_NF * W;
        fv[0 * H + h] = 0.0;
        fv[1 * H + h] = f1;
        fv[2 * H + h] = f2;
        fv[3 * H + h] = f3;
        fv[4 * H + h] = f4;
    }
    __syncthreads();
    // ---- per point: FLUX_DXYZ and dq -= re*dfv
    for (int idx = threadIdx.x; idx < NL * n; idx += blockDim.x) {
        const int l0 = fdiv(idx, dNL);
        const int ln = idx - l0 * NL;
        const int l = 1 + l0;
        const VisLine &L = lines[ln];
        const double *fv = smem + (size_t)ln * LS + (size_t)VIS_NF * W;
        long long gi = L.l0 + (long long)l * L.st;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            auto fa = [&](int hh) { return fv[m * H + hh]; };
            double dfv = flux_dxyz_at(fa, n, l);
            if (out) {
                out[m * stride + gi] = P.re * dfv;
            } else {
                double *dq = F.f[F_DQ1 + m];
                dq[gi] = dq[gi] - P.re * dfv;
            }
        }
    }
    (void)hmax;
}

size_t rhs_vis_line_bytes(int n) { return (size_t)vis_line_stride(n) * 8; }
int rhs_vis_max_lines() { return VIS_MAX_LINES; }
int rhs_vis_threads() { return VIS_THREADS; }

void launch_rhs_vis(const LaunchCtx &c, int dir, cudaStream_t st, double *out) {
    if (c.mixed) return launch_rhs_vis_mx(c, dir, st, out);
    const DirTable &T = c.vis[dir];
    if (T.ngroups == 0) return;
    const long long stride = c.total;
    if (dir == 0) k_rhs_vis<0><<<T.ngroups, VIS_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, T.hmax, out, stride);
    else if (dir == 1) k_rhs_vis<1><<<T.ngroups, VIS_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, T.hmax, out, stride);
    else k_rhs_vis<2><<<T.ngroups, VIS_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, T.hmax, out, stride);
}

void setup_rhs_vis_attrs(size_t max_smem) {
    cudaFuncSetAttribute(k_rhs_vis<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    cudaFuncSetAttribute(k_rhs_vis<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    cudaFuncSetAttribute(k_rhs_vis<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
}

}  // namespace wcns
