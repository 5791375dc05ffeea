// k_rhs_inv.cu -- inviscid residual along one index direction.
//
// Restates r_h_s_invis (RHS.f90:35-72) -> invcode -> inviscd3d
// (Convect.f90:2-56, 58-649) with the WCNS-E-5 line scheme WCNS_E_5
// (WCNSE5.f90:2-206, nscheme=4), WCNS_E_5_41 (WCNSE5.f90:2087-2759,
// nscheme=41) or WCNS_E_5_42 (WCNSE5.f90:2766-3438, nscheme=42, the 41
// sections with second-order end states), Steger-Warming (flux.f90:2-77),
// Van Leer (flux.f90:395-501) or Roe (flux.f90:116-244) fluxes, and
// FLUX_DXYZ (WCNSE5.f90:209-254).  dq += dF.
//
// One CTA owns a group of NL lines of one block.  The reference's
// sequential line loop is split into three parallel phases:
//   A  per point i: smoothness indicators and nonlinear weights, giving the
//      left state at half node i and the right state at half node i-1;
//   B  per half node: boundary closures, positivity fallback, numerical flux;
//      plus the 26 independent fluxes of the nscheme=41/42 boundary sections;
//   C  per point: sixth-order flux difference (or the boundary-section
//      difference where the reference overrides it) accumulated into dq.
// Each value is produced with the reference's exact operation sequence.
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

struct InvLine {
    const double *sq;  // shared-memory copy of the prim line: sq[m*(n+6) + l+2], l = -2..n+3
    const double *sk;  // shared-memory copy of the metrics (kx,ky,kz) of the line: sk[c*n + l-1], l = 1..n
    long long stride;
    long long dqbase;  // field index of point l=0 on the line (point l at dqbase + l*stride)
    int n, ist, ied;
};

__device__ __forceinline__ double qv(const InvLine &L, int m, int l) { return L.sq[m * (L.n + 6) + l + 2]; }

constexpr int INV_MAX_LINES = 32;  // lines per CTA (short lines are grouped many to a CTA)

// doubles of shared memory per line: prim 5 x (n+6), metrics 3 x n, qwl, qwr,
// f (5 x (n+1) each) and the 26 boundary-section fluxes; padded to 2 mod 16
// so that the lines of a group fall on different banks
__host__ __device__ inline int inv_line_stride(int n) {
    int raw = 5 * (n + 6) + 3 * n + 15 * (n + 1) + 130;
    return (raw + 13) / 16 * 16 + 2;
}

// qwl/qwr after phase B (main value from smem or the 4-style closure)
__device__ __forceinline__ double qwl_postB(const InvLine &L, const double *sqwl, int m, int h) {
    int n = L.n;
    if (L.ist > 1) {
        if (h == 0) return (35.0 * qv(L, m, 1) - 35.0 * qv(L, m, 2) + 21.0 * qv(L, m, 3) - 5.0 * qv(L, m, 4)) / 16.0;
        if (h == 1) return (5.0 * qv(L, m, 1) + 15.0 * qv(L, m, 2) - 5.0 * qv(L, m, 3) + qv(L, m, 4)) / 16.0;
        if (h == 2) return (-qv(L, m, 1) + 9.0 * qv(L, m, 2) + 9.0 * qv(L, m, 3) - qv(L, m, 4)) / 16.0;
    }
    if (L.ied < n) {
        if (h == n) return (35.0 * qv(L, m, n) - 35.0 * qv(L, m, n - 1) + 21.0 * qv(L, m, n - 2) - 5.0 * qv(L, m, n - 3)) / 16.0;
        if (h == n - 1) return (5.0 * qv(L, m, n) + 15.0 * qv(L, m, n - 1) - 5.0 * qv(L, m, n - 2) + qv(L, m, n - 3)) / 16.0;
    }
    return sqwl[m * (n + 1) + h];
}
__device__ __forceinline__ double qwr_postB(const InvLine &L, const double *sqwr, int m, int h) {
    int n = L.n;
    if (L.ist > 1) {
        if (h == 0) return (35.0 * qv(L, m, 1) - 35.0 * qv(L, m, 2) + 21.0 * qv(L, m, 3) - 5.0 * qv(L, m, 4)) / 16.0;
        if (h == 1) return (5.0 * qv(L, m, 1) + 15.0 * qv(L, m, 2) - 5.0 * qv(L, m, 3) + qv(L, m, 4)) / 16.0;
    }
    if (L.ied < n) {
        if (h == n) return (35.0 * qv(L, m, n) - 35.0 * qv(L, m, n - 1) + 21.0 * qv(L, m, n - 2) - 5.0 * qv(L, m, n - 3)) / 16.0;
        if (h == n - 1) return (5.0 * qv(L, m, n) + 15.0 * qv(L, m, n - 1) - 5.0 * qv(L, m, n - 2) + qv(L, m, n - 3)) / 16.0;
        if (h == n - 2) return (-qv(L, m, n) + 9.0 * qv(L, m, n - 1) + 9.0 * qv(L, m, n - 2) - qv(L, m, n - 3)) / 16.0;
    }
    return sqwr[m * (n + 1) + h];
}

// Left boundary-section states (WCNSE5.f90:2284-2459); nscheme=42 has
// second-order states at the first four half nodes (WCNSE5.f90:2967-2986)
__device__ __forceinline__ double s1_state(const InvLine &L, int m, int h, bool s42) {
    if (s42) switch (h) {
        case 0: return (677.0 * qv(L, m, 1) - 421.0 * qv(L, m, 2) + 99.0 * qv(L, m, 3) + 13.0 * qv(L, m, 4)) / 368.0;
        case 1: return (5.0 * qv(L, m, 1) + 15.0 * qv(L, m, 2) - 5.0 * qv(L, m, 3) + qv(L, m, 4)) / 16.0;
        case 2: return (-qv(L, m, 1) + 9.0 * qv(L, m, 2) + 9.0 * qv(L, m, 3) - qv(L, m, 4)) / 16.0;
        default: return (qv(L, m, 1) - 5.0 * qv(L, m, 2) + 15.0 * qv(L, m, 3) + 5.0 * qv(L, m, 4)) / 16.0;
        }
    switch (h) {
    case 0: return (3.0 * qv(L, m, 1) - 1.0 * qv(L, m, 2) - 0. * qv(L, m, 3)) / 2.0;
    case 1: return (19.0 * qv(L, m, 1) + 25.0 * qv(L, m, 2) - 2. * qv(L, m, 3)) / 42.0;
    case 2: return (4.0 * qv(L, m, 1) + 3.0 * qv(L, m, 2) + 9.0 * qv(L, m, 3) + 2. * qv(L, m, 4)) / 18.0;
    default: return (-2.0 * qv(L, m, 1) + 3.0 * qv(L, m, 2) + 3.0 * qv(L, m, 3) + 2. * qv(L, m, 4)) / 6.0;
    }
}
__device__ __forceinline__ double s2_left(const InvLine &L, int m, int h) {
    switch (h) {
    case 1: return (3.0 * qv(L, m, 1) + 6.0 * qv(L, m, 2) - qv(L, m, 3)) / 8.0;
    case 2: return (-30.0 * qv(L, m, 1) + 145.0 * qv(L, m, 2) + 29.0 * qv(L, m, 3) - 8.0 * qv(L, m, 4)) / 136.0;
    case 3: return (-qv(L, m, 2) + 6.0 * qv(L, m, 3) + 3.0 * qv(L, m, 4)) / 8.0;
    case 4: return (qv(L, m, 2) + 2.0 * qv(L, m, 3) + 5.0 * qv(L, m, 4)) / 8.0;
    default: return (qv(L, m, 2) + qv(L, m, 3) + 6.0 * qv(L, m, 4)) / 8.0;
    }
}
__device__ __forceinline__ double s2_right(const InvLine &L, int m, int h) {
    if (h == 2) return (2.0 * qv(L, m, 1) + 49.0 * qv(L, m, 2) + 125.0 * qv(L, m, 3) - 40.0 * qv(L, m, 4)) / 136.0;
    return s2_left(L, m, h);
}
__device__ __forceinline__ double s3_left(const InvLine &L, int m, int h) {
    if (h == 2) return (-29.0 * qv(L, m, 1) + 170.0 * qv(L, m, 2) + 63.0 * qv(L, m, 3) + 12.0 * qv(L, m, 4)) / 216.0;
    return s2_left(L, m, h);
}
// Right boundary-section states (WCNSE5.f90:2524-2705); h counts down from
// n; nscheme=42 as on the left (WCNSE5.f90:3207-3226)
__device__ __forceinline__ double s4_state(const InvLine &L, int m, int h, bool s42) {
    int n = L.n;
    int o = n - h;
    if (s42) switch (o) {
        case 0: return (677.0 * qv(L, m, n) - 421.0 * qv(L, m, n - 1) + 99.0 * qv(L, m, n - 2) + 13.0 * qv(L, m, n - 3)) / 368.0;
        case 1: return (5.0 * qv(L, m, n) + 15.0 * qv(L, m, n - 1) - 5.0 * qv(L, m, n - 2) + qv(L, m, n - 3)) / 16.0;
        case 2: return (-qv(L, m, n) + 9.0 * qv(L, m, n - 1) + 9.0 * qv(L, m, n - 2) - qv(L, m, n - 3)) / 16.0;
        default: return (qv(L, m, n) - 5.0 * qv(L, m, n - 1) + 15.0 * qv(L, m, n - 2) + 5.0 * qv(L, m, n - 3)) / 16.0;
        }
    switch (o) {
    case 0: return (3.0 * qv(L, m, n) - 1.0 * qv(L, m, n - 1) - 0. * qv(L, m, n - 2)) / 2.0;
    case 1: return (19.0 * qv(L, m, n) + 25.0 * qv(L, m, n - 1) - 2. * qv(L, m, n - 2)) / 42.0;
    case 2: return (4.0 * qv(L, m, n) + 3.0 * qv(L, m, n - 1) + 9.0 * qv(L, m, n - 2) + 2. * qv(L, m, n - 3)) / 18.0;
    default: return (-2.0 * qv(L, m, n) + 3.0 * qv(L, m, n - 1) + 3.0 * qv(L, m, n - 2) + 2. * qv(L, m, n - 3)) / 6.0;
    }
}
__device__ __forceinline__ double s5_right(const InvLine &L, int m, int h) {
    int n = L.n;
    switch (n - h) {
    case 1: return (3.0 * qv(L, m, n) + 6.0 * qv(L, m, n - 1) - qv(L, m, n - 2)) / 8.0;
    case 2: return (-30.0 * qv(L, m, n) + 145.0 * qv(L, m, n - 1) + 29.0 * qv(L, m, n - 2) - 8.0 * qv(L, m, n - 3)) / 136.0;
    case 3: return (-qv(L, m, n - 1) + 6.0 * qv(L, m, n - 2) + 3.0 * qv(L, m, n - 3)) / 8.0;
    case 4: return (qv(L, m, n - 1) + 2.0 * qv(L, m, n - 2) + 5.0 * qv(L, m, n - 3)) / 8.0;
    default: return (qv(L, m, n - 1) + qv(L, m, n - 2) + 6.0 * qv(L, m, n - 3)) / 8.0;
    }
}
__device__ __forceinline__ double s5_left(const InvLine &L, int m, int h) {
    int n = L.n;
    if (n - h == 2) return (2.0 * qv(L, m, n) + 49.0 * qv(L, m, n - 1) + 125.0 * qv(L, m, n - 2) - 40.0 * qv(L, m, n - 3)) / 136.0;
    return s5_right(L, m, h);
}
__device__ __forceinline__ double s6_right(const InvLine &L, int m, int h) {
    int n = L.n;
    if (n - h == 2) return (-29.0 * qv(L, m, n) + 170.0 * qv(L, m, n - 1) + 63.0 * qv(L, m, n - 2) + 12.0 * qv(L, m, n - 3)) / 216.0;
    return s5_right(L, m, h);
}
// qwl(h) at the moment the right sections save u_l_old: the left sections'
// final values where they ran (h<=5), otherwise the phase-B value.
__device__ __forceinline__ double qwl_preright(const InvLine &L, const double *sqwl, int nscheme, int m, int h) {
    if ((nscheme == 41 || nscheme == 42) && L.ist > 1 && h <= 5) {
        if (h == 0) return s1_state(L, m, 0, nscheme == 42);
        if (h == 2) return s3_left(L, m, 2);
        return s2_left(L, m, h);
    }
    return qwl_postB(L, sqwl, m, h);
}

// out == nullptr: dq += dF in place; otherwise dF is stored in
// out[m*stride + point] for an ordered combine (k_combine_dq).  Four CTAs
// per SM (64 registers, with some spill; at most 54 KB of staged lines):
// 3.52 ms per channel step for the three directions against 3.62 at three
// CTAs of 80 registers.  (The viscous kernel at four 256-thread CTAs of 64
// registers spills 0.5 KB per thread and runs 4.1 ms against 3.4.)
template <int dir>
__global__ void __launch_bounds__(256, 4) k_rhs_invis(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                   const LineGroup *__restrict__ groups, int *err, double *out,
                                                   long long stride) {
    extern __shared__ double smem[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir);
    const int H = n + 1, W = n + 6;
    const int NL = G.nl;
    const int LS = inv_line_stride(n);
    // per line: prim, metrics, then qwl, qwr, f (5 x H each) and 26 section fluxes
    const size_t work0 = (size_t)5 * W + (size_t)3 * n;
    __shared__ InvLine lines[INV_MAX_LINES];
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    if (threadIdx.x < NL) {
        int c[3];
        c[a1] = G.a0 + threadIdx.x;
        c[a2] = G.b;
        c[dir] = -2;
        long long base = gidx(B, c[0], c[1], c[2]);
        InvLine L;
        L.sq = smem + (size_t)threadIdx.x * LS;
        L.sk = L.sq + (size_t)5 * W;
        L.stride = dstride(B, dir);
        L.dqbase = base + 2 * L.stride;
        L.n = n;
        L.ist = __ldg(F.f[F_R] + base) < SMALL ? 2 : 0;
        L.ied = __ldg(F.f[F_R] + base + (long long)(n + 5) * L.stride) < SMALL ? n - 2 : n;
        lines[threadIdx.x] = L;
    }
    __syncthreads();
    constexpr bool posmajor = (dir == 0);
    const FastDiv dNL = fast_div_init(NL), d5NL = fast_div_init(5 * NL), dW = fast_div_init(W);
    // ---- stage the prim line (l = -2..n+3) and the metrics of this
    // direction (l = 1..n): one thread per (line, point), coalesced along the
    // line for i-lines and across the group's neighbouring lines otherwise
    for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
        const int qq = posmajor ? fdiv(e, dW) : fdiv(e, dNL);
        const int ln = posmajor ? qq : e - qq * NL;
        const int p = posmajor ? e - qq * W : qq;
        const InvLine &L = lines[ln];
        const long long gi = L.dqbase + (long long)(p - 2) * L.stride;
        double v[8];
#pragma unroll
        for (int m = 0; m < 5; m++) v[m] = __ldg(F.f[F_R + m] + gi);
        const bool inner = p >= 3 && p <= n + 2;
#pragma unroll
        for (int c = 0; c < 3; c++) v[5 + c] = inner ? __ldg(F.f[F_KCX + 3 * dir + c] + gi) : 0.0;
        double *sq = smem + (size_t)ln * LS;
#pragma unroll
        for (int m = 0; m < 5; m++) sq[m * W + p] = v[m];
        if (inner) {
#pragma unroll
            for (int c = 0; c < 3; c++) sq[5 * W + c * n + p - 3] = v[5 + c];
        }
    }
    __syncthreads();
    const double CL[3] = {1.0 / 16.0, 10.0 / 16.0, 5.0 / 16.0};
    const double CR[3] = {5.0 / 16.0, 10.0 / 16.0, 1.0 / 16.0};
    const double EPS = 1.0e-6;

    // Phases A, B and C walk the items line-fastest in every direction: the lanes
    // of a warp take the same position on neighbouring lines and follow one
    // control path, and items without work (boundary sections of a line that
    // has none) gather into whole warps that skip them.
    // ---- phase A: weights per (line, variable, point i in [ist, ied+1])
    {
        const int NP = n + 2;
        const int nitems = NL * 5 * NP;
        for (int idx = threadIdx.x; idx < nitems; idx += blockDim.x) {
            const int q1 = fdiv(idx, dNL), i = fdiv(idx, d5NL);
            const int ln = idx - q1 * NL, m = q1 - 5 * i;
            const InvLine &L = lines[ln];
            if (i < L.ist || i > L.ied + 1) continue;
            double *ql_ = smem + (size_t)ln * LS + work0;
            double *qr_ = ql_ + (size_t)5 * H;
            double qm2 = qv(L, m, i - 2), qm1 = qv(L, m, i - 1), q0 = qv(L, m, i), qp1 = qv(L, m, i + 1), qp2 = qv(L, m, i + 2);
            double g[3], sdv[3], bl[3], br[3];
            g[0] = 0.5 * (qm2 - 4.0 * qm1 + 3.0 * q0);
            g[1] = 0.5 * (qp1 - qm1);
            g[2] = 0.5 * (-3.0 * q0 + 4.0 * qp1 - qp2);
            sdv[0] = qm2 - 2.0 * qm1 + q0;
            sdv[1] = qm1 - 2.0 * q0 + qp1;
            sdv[2] = q0 - 2.0 * qp1 + qp2;
#pragma unroll
            for (int kk = 0; kk < 3; kk++) {
                double IS = g[kk] * g[kk] + sdv[kk] * sdv[kk];
                double tt = EPS + IS;
                double EIS2 = tt * tt;
                bl[kk] = CL[kk] / EIS2;
                br[kk] = CR[kk] / EIS2;
            }
            if (i <= L.ied) {
                double IS = bl[0] + bl[1] + bl[2];
                double w0 = bl[0] / IS, w1 = bl[1] / IS, w2 = bl[2] / IS;
                ql_[m * H + i] = q0 + 0.125 * (w0 * (sdv[0] + 4.0 * g[0]) + w1 * (sdv[1] + 4.0 * g[1]) + w2 * (sdv[2] + 4.0 * g[2]));
            }
            if (i - 1 >= L.ist) {
                double IS = br[0] + br[1] + br[2];
                double w0 = br[0] / IS, w1 = br[1] / IS, w2 = br[2] / IS;
                qr_[m * H + i - 1] = q0 + 0.125 * (w0 * (sdv[0] - 4.0 * g[0]) + w1 * (sdv[1] - 4.0 * g[1]) + w2 * (sdv[2] - 4.0 * g[2]));
            }
        }
    }
    __syncthreads();
    // ---- phase B: fluxes at half nodes, and the nscheme=41/42 boundary-section fluxes
    {
        const int NT = H + 26;
        int nbad = 0;
        for (int idx = threadIdx.x; idx < NL * NT; idx += blockDim.x) {
            const int t = fdiv(idx, dNL);
            const int ln = idx - t * NL;
            const InvLine &L = lines[ln];
            const double *ql_ = smem + (size_t)ln * LS + work0;
            const double *qr_ = ql_ + (size_t)5 * H;
            double ql[5], qr[5], fl[5];
            int h, mode = 0;  // 0 main, 1..6 sections
            if (t < H) {
                h = t;
                for (int m = 0; m < 5; m++) { ql[m] = qwl_postB(L, ql_, m, h); qr[m] = qwr_postB(L, qr_, m, h); }
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) { int ii = h > 1 ? h : 1; for (int m = 0; m < 5; m++) ql[m] = qv(L, m, ii); }
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) { int ii = h + 1 < n ? h + 1 : n; for (int m = 0; m < 5; m++) qr[m] = qv(L, m, ii); }
            } else {
                if (P.nscheme != 41 && P.nscheme != 42) continue;
                int sidx = t - H;  // 0..25
                if (sidx < 13) {
                    if (L.ist <= 1) continue;
                    if (sidx < 4) { mode = 1; h = sidx; }
                    else if (sidx < 9) { mode = 2; h = sidx - 4 + 1; }
                    else { mode = 3; h = sidx - 9 + 1; }
                } else {
                    if (L.ied >= n) continue;
                    int r = sidx - 13;
                    if (r < 4) { mode = 4; h = n - r; }
                    else if (r < 9) { mode = 5; h = n - 1 - (r - 4); }
                    else { mode = 6; h = n - 1 - (r - 9); }
                }
                for (int m = 0; m < 5; m++) {
                    switch (mode) {
                    case 1: ql[m] = qr[m] = s1_state(L, m, h, P.nscheme == 42); break;
                    case 2: ql[m] = s2_left(L, m, h); qr[m] = s2_right(L, m, h); break;
                    case 3: ql[m] = s3_left(L, m, h); qr[m] = qwr_postB(L, qr_, m, h); break;
                    case 4: ql[m] = qr[m] = s4_state(L, m, h, P.nscheme == 42); break;
                    case 5: ql[m] = s5_left(L, m, h); qr[m] = s5_right(L, m, h); break;
                    default: ql[m] = qwl_preright(L, ql_, P.nscheme, m, h); qr[m] = s6_right(L, m, h); break;
                    }
                }
                bool badl = ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT;
                bool badr = qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT;
                int ia = h > 1 ? h : 1, ib = h + 1 < n ? h + 1 : n;
                for (int m = 0; m < 5; m++) {
                    if (mode == 1) {
                        if (badl) ql[m] = (qv(L, m, ia) + qv(L, m, h + 1)) / 2.;
                        if (badr) qr[m] = (qv(L, m, ia) + qv(L, m, h + 1)) / 2.;
                    } else if (mode == 4) {
                        if (badl) ql[m] = (qv(L, m, 1) + qv(L, m, h)) / 2.0;
                        if (badr) qr[m] = (qv(L, m, 1) + qv(L, m, h)) / 2.0;
                    } else {
                        if (badl) ql[m] = qv(L, m, ia);
                        if (badr) qr[m] = qv(L, m, ib);
                    }
                }
            }
            // half-node metrics: VALUE_HALF_NODE of (kx,ky,kz) along the line
            auto ax = [&](int l) { return L.sk[l - 1]; };
            auto ay = [&](int l) { return L.sk[n + l - 1]; };
            auto az = [&](int l) { return L.sk[2 * n + l - 1]; };
            double kx = value_half_node_at(ax, n, h), ky = value_half_node_at(ay, n, h), kz = value_half_node_at(az, n, h);
            const double kt = 0.0;  // kct=0, so every half-node value of kt is +0
            nbad += flux_type(P, ql, qr, kx, ky, kz, kt, fl);
            if (mode == 0) {
                double *f_ = smem + (size_t)ln * LS + work0 + (size_t)10 * H;
                for (int m = 0; m < 5; m++) f_[m * H + h] = fl[m];
            } else {
                double *sc = smem + (size_t)ln * LS + work0 + (size_t)15 * H + (size_t)(t - H) * 5;
                for (int m = 0; m < 5; m++) sc[m] = fl[m];
            }
        }
        if (nbad) atomicAdd(&err[ERR_ROE], nbad);
    }
    __syncthreads();
    // ---- phase C: flux difference and accumulation into dq, per (line, point, variable)
    {
        const int nitems = NL * n * 5;
        for (int idx = threadIdx.x; idx < nitems; idx += blockDim.x) {
            const int q1 = fdiv(idx, dNL), l0 = fdiv(idx, d5NL);
            const int ln = idx - q1 * NL, m = q1 - 5 * l0, l = 1 + l0;
            const InvLine &L = lines[ln];
            const double *f_ = smem + (size_t)ln * LS + work0 + (size_t)10 * H;
            const double *sc = smem + (size_t)ln * LS + work0 + (size_t)15 * H;
            const bool sections = P.nscheme == 41 || P.nscheme == 42;
            bool right = sections && L.ied < n && l >= n - 2;
            bool left = sections && L.ist > 1 && l <= 3;
            long long gi = L.dqbase + (long long)l * L.stride;
            double df;
            if (right) {
                const double *s4 = sc + 13 * 5, *s5 = sc + 17 * 5, *s6 = sc + 22 * 5;
                // section fluxes f(ni-h): s4[k] holds f(k), s5[k] and s6[k] hold f(k+1)
                if (l == n) df = -(-23.0 * s4[0 * 5 + m] + 21.0 * s4[1 * 5 + m] + 3.0 * s4[2 * 5 + m] - 1.0 * s4[3 * 5 + m]) / 24.0;
                else if (l == n - 1) df = -(-22.0 * s5[0 * 5 + m] + 17.0 * s5[1 * 5 + m] + 9.0 * s5[2 * 5 + m] - 5.0 * s5[3 * 5 + m] + s5[4 * 5 + m]) / 24.0;
                else df = -(s6[0 * 5 + m] - 27.0 * s6[1 * 5 + m] + 27.0 * s6[2 * 5 + m] - s6[3 * 5 + m]) / 24.0;
            } else if (left) {
                const double *s1 = sc, *s2 = sc + 4 * 5, *s3 = sc + 9 * 5;
                if (l == 1) df = (-23.0 * s1[0 * 5 + m] + 21.0 * s1[1 * 5 + m] + 3.0 * s1[2 * 5 + m] - 1.0 * s1[3 * 5 + m]) / 24.0;
                else if (l == 2) df = (-22.0 * s2[0 * 5 + m] + 17.0 * s2[1 * 5 + m] + 9.0 * s2[2 * 5 + m] - 5.0 * s2[3 * 5 + m] + s2[4 * 5 + m]) / 24.0;
                else df = (s3[0 * 5 + m] - 27.0 * s3[1 * 5 + m] + 27.0 * s3[2 * 5 + m] - s3[3 * 5 + m]) / 24.0;
            } else {
                auto fa = [&](int hh) { return f_[m * H + hh]; };
                df = flux_dxyz_at(fa, n, l);
            }
            if (out) {
                out[m * stride + gi] = df;
            } else {
                double *dq = F.f[F_DQ1 + m];
                dq[gi] = dq[gi] + df;
            }
        }
    }
}

void launch_rhs_invis(const LaunchCtx &c, int dir, cudaStream_t st, double *out) {
    if (c.mixed) return launch_rhs_invis_mx(c, dir, st, out);
    const DirTable &T = c.inv[dir];
    if (T.ngroups == 0) return;
    const long long stride = c.total;
    if (dir == 0) k_rhs_invis<0><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, stride);
    else if (dir == 1) k_rhs_invis<1><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, stride);
    else k_rhs_invis<2><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, stride);
}

void setup_rhs_invis_attrs(size_t max_smem) {
    cudaFuncSetAttribute(k_rhs_invis<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    cudaFuncSetAttribute(k_rhs_invis<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    cudaFuncSetAttribute(k_rhs_invis<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
}

size_t rhs_invis_line_bytes(int n) { return (size_t)inv_line_stride(n) * 8; }
int rhs_invis_max_lines() { return INV_MAX_LINES; }

}  // namespace wcns
