// wcns_dev.cuh -- device data model and arithmetic shared by all WCNS kernels.
//
// Every per-point field lives in the reference's ghosted index space
// (-2:n+3 in each direction, i fastest) so that index arithmetic is the same
// for prim (which has real ghosts) and interior-only fields.  All blocks of a
// field are concatenated in one allocation; DevBlock::off is the block base.
//
// Arithmetic restates the reference operation by operation.  The library is
// compiled with -fmad=false so that no multiply-add is fused: with IEEE
// division and square root (the CUDA defaults for double) each expression
// then rounds exactly as gfortran -O2 does on x86-64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace wcns {

constexpr double SMALL = 1.0e-38;     // Globalvar.f90:215
constexpr double SML_SSS = 1.0e-30;   // Globalvar.f90:218
constexpr double PMIN_LIMIT = 1.0e-8; // Globalvar.f90:223
constexpr double PMAX_LIMIT = 1.0e+3;
constexpr double RMIN_LIMIT = 1.0e-8;
constexpr double RMAX_LIMIT = 1.0e+3;
constexpr double TMIN_LIMIT = 1.0e-8;
constexpr int NIJK2D = 4;   // Main.f90:20
constexpr int NIJK2ND = 4;  // Main.f90:21

enum Field : int {
    F_R = 0, F_U, F_V, F_W, F_P, F_T,
    F_DQ1, F_DQ2, F_DQ3, F_DQ4, F_DQ5,
    F_DTDT, F_SRA, F_SRB, F_SRC, F_SRVA, F_SRVB, F_SRVC,
    F_KCX, F_KCY, F_KCZ, F_ETX, F_ETY, F_ETZ, F_CTX, F_CTY, F_CTZ, F_VOL,
    F_C, F_VISL, F_Q1, F_Q2, F_Q3, F_Q4, F_Q5,
    F_NPUBLIC,
    // internal work arrays
    F_RHS1 = F_NPUBLIC, F_RHS2, F_RHS3, F_RHS4, F_RHS5,
    F_COED,
    F_OLD1, F_OLD2, F_OLD3, F_OLD4, F_OLD5,
    F_DUV0,  // 12 node derivatives of (u,v,w,T): F_DUV0 .. F_DUV0+11
    F_NPOOL = F_DUV0 + 12,  // fields of the pool
    // the SA model's eddy viscosity (its own allocation; null while the
    // model is not set up, which the kernels read as vist = 0)
    F_VIST = F_NPOOL,
    F_NALL
};

struct DevParams {
    double gama, g1;  // g1 = gama/(gama-1)
    double moo, moo2, moocp;
    double reynolds, re, visc;
    double cp_prl, cp_prt, cc23;
    double cfl, timedt_rate, efix, csrv;
    double roo, uoo, voo, woo, poo, coo;
    double twall_nd;
    int nvis, nscheme, nflux, adiabatic;
};

struct DevBlock {
    int ni, nj, nk;
    int gx, gy, gz;
    long long off;   // base offset of this block in every field
    long long npts;  // ni*nj*nk
    long long pmoff; // base offset in the plane-major sweep arrays
    // the free stream's Mach-dependent constants of init_inflow
    // (PreProcess.f90:968-1113) for this block: the context's by default,
    // a case's own when independent cases of different Mach numbers share
    // one context (wcns_set_block_freestream)
    double moo2, moocp, poo, coo, cp_prl, cp_prt;
};

// Plane-major layout for the LU-SGS sweeps.  Cell (i,j,k) of a block lives
// in plane p = i+j+k at column slot c(j,k); the cells of one hyperplane are
// contiguous.  Columns are grouped in j-chunks, one chunk per CTA of the
// block's sweep cluster: chunk q covers j-1 in [q*nj/C, (q+1)*nj/C) for all
// k, and slot = j0(q)*nk + (k-1)*width(q) + (j-1-j0(q)).
__host__ __device__ inline int chunk_j0(int q, int nj, int C) { return q * nj / C; }  // q <= C <= 16: no overflow
__host__ __device__ inline int chunk_of(int jj, int nj, int C) {  // jj = j-1
    int q = (int)(((long long)jj * C) / nj);
    if (q > C - 1) q = C - 1;
    while (q > 0 && chunk_j0(q, nj, C) > jj) q--;
    while (q < C - 1 && chunk_j0(q + 1, nj, C) <= jj) q++;
    return q;
}
__host__ __device__ inline int col_slot(int j, int k, int nj, int nk, int C) {
    int jj = j - 1, q = chunk_of(jj, nj, C);
    int j0 = chunk_j0(q, nj, C), w = chunk_j0(q + 1, nj, C) - j0;
    return j0 * nk + (k - 1) * w + (jj - j0);
}

// static per-cell record of the sweeps (written once per step by k_lhs_prep)
enum StatRec : int {
    SR_COED = 0, SR_RHS = 1,              // coed, rhs(5)
    SR_JS = 6,                            // um, vm, wm, c2, hm, af
    SR_JD = 12,                           // per direction d: ct, nx, ny, nz at SR_JD + 4d
    SR_JP = 24,                           // npn=+1 (lower neighbour): l1, x1, x2 at SR_JP + 3d
    SR_JM = 33,                           // npn=-1 (upper neighbour): l1, x1, x2 at SR_JM + 3d
    SR_SRV = 42,                          // srva, srvb, srvc
    SR_N = 46                             // record length (16-byte multiple)
};
constexpr int DYN_N = 16;                 // dynamic per-cell record: dq of lusgs_l, or old-side terms 5*d + m

struct PmFields {
    double *dq[5];   // SoA dq in plane-major order (result of gs_pr_u, the last sweep)
    long long dq_stride;  // dq[m] = dq[0] + m * dq_stride
    double *stat;    // [cell][SR_N]
    double *dyn;     // [cell][DYN_N] dq of lusgs_l, read by lusgs_u
    double *gs[2];   // [cell][DYN_N] old-side terms along i, j, k: written by lusgs_u for gs_pr_l (gs[0])
                     // and by gs_pr_l for gs_pr_u (gs[1]); zero where the neighbour is outside the block
    int csize;       // CTAs per block cluster (defines the column slots)
};

__host__ __device__ inline long long pmidx(const DevBlock &b, int p, int slot) {
    return b.pmoff + (long long)(p - 3) * ((long long)b.nj * b.nk) + slot;
}

struct DevFields {
    double *f[F_NALL];
};

__host__ __device__ inline long long gidx(const DevBlock &b, int i, int j, int k) {
    return b.off + (long long)(i + 2) + (long long)b.gx * ((long long)(j + 2) + (long long)b.gy * (long long)(k + 2));
}

// Division by a divisor that is the same for the whole kernel: one high
// multiply instead of a division sequence.  Exact for 0 <= n, d and
// n * d < 2^32 (m = ceil(2^32 / d); the error n * (m - 2^32/d) / 2^32 < n / 2^32
// stays below 1/d).
struct FastDiv {
    unsigned d, m;
};
__host__ __device__ inline FastDiv fast_div_init(int d) {
    FastDiv f;
    f.d = (unsigned)d;
    f.m = d <= 1 ? 0u : 0xFFFFFFFFu / (unsigned)d + 1u;
    return f;
}
__device__ __forceinline__ int fdiv(int n, FastDiv f) { return f.d <= 1 ? n : (int)__umulhi((unsigned)n, f.m); }

// interior point index p = (i-1) + ni*((j-1) + nj*(k-1)) -> (i, j, k); 32-bit
// divisions whenever p fits (every realistic block)
__device__ __forceinline__ void decode_point(const DevBlock &B, long long p, int &i, int &j, int &k) {
    if (p < 0x7fffffffLL) {
        const int q = (int)p, r = q / B.ni;
        i = q - r * B.ni + 1;
        j = r % B.nj + 1;
        k = r / B.nj + 1;
    } else {
        i = (int)(p % B.ni) + 1;
        j = (int)((p / B.ni) % B.nj) + 1;
        k = (int)(p / ((long long)B.ni * B.nj)) + 1;
    }
}

__host__ __device__ inline int dimof(const DevBlock &b, int d) { return d == 0 ? b.ni : (d == 1 ? b.nj : b.nk); }

// stride (in elements) along direction d
__host__ __device__ inline long long dstride(const DevBlock &b, int d) {
    return d == 0 ? 1LL : (d == 1 ? (long long)b.gx : (long long)b.gx * b.gy);
}

// ---------------------------------------------------------------------------
// Line operators evaluated at one position.  `Acc` maps a 1-based point index
// to a value.
// ---------------------------------------------------------------------------

// VALUE_HALF_NODE (WCNSE5.f90:799-852) at half node h in 0..n
template <class Acc>
__device__ __forceinline__ double value_half_node_at(const Acc &q, int n, int h) {
    if (n <= NIJK2ND) {
        if (h == 0) {
            int i2 = n < 2 ? n : 2, i3 = n < 3 ? n : 3;
            return (15.0 * q(1) - 10.0 * q(i2) + 3.0 * q(i3)) / 8.0;
        }
        if (h == n) {
            int j1 = n - 1 > 1 ? n - 1 : 1, j2 = n - 2 > 1 ? n - 2 : 1;
            return (15.0 * q(n) - 10.0 * q(j1) + 3.0 * q(j2)) / 8.0;
        }
        return 0.5 * (q(h) + q(h + 1));
    }
    if (h == 0) return (35.0 * q(1) - 35.0 * q(2) + 21.0 * q(3) - 5.0 * q(4)) / 16.0;
    if (h == n) return (35.0 * q(n) - 35.0 * q(n - 1) + 21.0 * q(n - 2) - 5.0 * q(n - 3)) / 16.0;
    if (h == 1) return (5.0 * q(1) + 15.0 * q(2) + -5.0 * q(3) + 1.0 * q(4)) / 16.0;
    if (h == n - 1) return (5.0 * q(n) + 15.0 * q(n - 1) + -5.0 * q(n - 2) + 1.0 * q(n - 3)) / 16.0;
    return (9.0 * (q(h) + q(h + 1)) + -1.0 * (q(h + 2) + q(h - 1))) / 16.0;
}

// VALUE_HALF_NODE_IJK (newvis.f90:421-554) for one component at half node h
template <class Acc>
__device__ __forceinline__ double value_half_node_ijk_at(const Acc &q, int n, int h) {
    if (n <= NIJK2ND) {
        if (h == 0) return 1.5 * q(1) - 0.5 * q(n < 2 ? n : 2);
        if (h == n) return 1.5 * q(n) - 0.5 * q(n - 1 > 1 ? n - 1 : 1);
        return 0.5 * (q(h) + q(h + 1));
    }
    if (h == 0) return (35.0 * q(1) - 35.0 * q(2) + 21.0 * q(3) - 5.0 * q(4)) / 16.0;
    if (h == n) return (35.0 * q(n) - 35.0 * q(n - 1) + 21.0 * q(n - 2) - 5.0 * q(n - 3)) / 16.0;
    if (h == 1) return (5.0 * q(1) + 15.0 * q(2) + -5.0 * q(3) + 1.0 * q(4)) / 16.0;
    if (h == n - 1) return (5.0 * q(n) + 15.0 * q(n - 1) + -5.0 * q(n - 2) + 1.0 * q(n - 3)) / 16.0;
    return (9.0 * (q(h) + q(h + 1)) + -1.0 * (q(h + 2) + q(h - 1))) / 16.0;
}

// FLUX_DXYZ (WCNSE5.f90:209-254) at point l in 1..n; f(h) for h in 0..n
template <class Acc>
__device__ __forceinline__ double flux_dxyz_at(const Acc &f, int n, int l) {
    if (n <= NIJK2ND) return f(l) - f(l - 1);
    if (l == 1) return (-23.0 * f(0) + 21.0 * f(1) + 3.0 * f(2) - f(3)) / 24.0;
    if (l == n) return -(-23.0 * f(n) + 21.0 * f(n - 1) + 3.0 * f(n - 2) - f(n - 3)) / 24.0;
    if (l == 2) return (f(0) - 27.0 * f(1) + 27.0 * f(2) - f(3)) / 24.0;
    if (l == n - 1) return -(f(n) - 27.0 * f(n - 1) + 27.0 * f(n - 2) - f(n - 3)) / 24.0;
    return (2250.0 * (f(l) - f(l - 1)) - 125.0 * (f(l + 1) - f(l - 2)) + 9.0 * (f(l + 2) - f(l - 3))) / 1920.0;
}

// ---------------------------------------------------------------------------
// Numerical fluxes
// ---------------------------------------------------------------------------

// flux_SW_pn (flux.f90:17-77); gethmgm_ns (GasModel.f90:385-399)
__device__ __forceinline__ void flux_sw_pn(const DevParams &P, const double *prim, double nx, double ny, double nz,
                                           double nt, double *f, int npn) {
    const double gama = P.gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double u2 = 0.5 * (um * um + vm * vm + wm * wm);
    double hint = P.g1 * pm / rm;
    double eint = hint - pm / rm;
    double em = eint + u2;
    double cm = sqrt(gama * pm / rm);
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    cgm = fmax(cgm, SML_SSS);
    double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    double eps = P.efix * P.efix * cgm * cgm;
    double dn = (double)npn;
    l1 = 0.5 * (l1 + dn * sqrt(l1 * l1 + eps));
    l4 = 0.5 * (l4 + dn * sqrt(l4 * l4 + eps));
    l5 = 0.5 * (l5 + dn * sqrt(l5 * l5 + eps));
    double cgm1 = 1.0 / cgm;
    double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
    double cta = (ct - nt) * cgm1;
    double c2r = cm * cm / gama;
    double x1 = c2r * (2.0 * l1 - l4 - l5) / (2.0 * cm * cm);
    double x2 = c2r * (l4 - l5) / (2.0 * cm);
    double hm = em + pm / rm;
    f[0] = (l1 - x1) * rm;
    f[1] = (l1 * um - x1 * um + nxa * x2) * rm;
    f[2] = (l1 * vm - x1 * vm + nya * x2) * rm;
    f[3] = (l1 * wm - x1 * wm + nza * x2) * rm;
    f[4] = (l1 * em - x1 * hm + cta * x2) * rm;
}

// flux_vanleer_pn (flux.f90:410-501), gethmgm -> gethmgm_ns
// (GasModel.f90:376-399).  Returns 1 when c^2 < 0 (the reference stops).
// (b +- 1)**2 is a product, as gfortran evaluates an integer exponent 2.
__device__ __forceinline__ int flux_vl_pn(const DevParams &P, const double *prim, double nx, double ny, double nz,
                                          double nt, double *f, int npn) {
    const double gama = P.gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double u2 = 0.5 * (um * um + vm * vm + wm * wm);
    double hint = P.g1 * pm / rm;
    double hm = hint + u2;
    double c2 = gama * pm / rm;
    const int bad = c2 < 0.0 ? 1 : 0;
    double cm = sqrt(c2);
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz) + SML_SSS;
    double cgm1 = 1.0 / cgm;
    double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
    double cta = ct * cgm1;
    double bmvl = cta / cm;
#pragma unroll
    for (int m = 0; m < 5; m++) f[m] = 0.0;
    if (fabs(bmvl) < 1.0) {
        double ctcm, b;
        if (npn == 1) {
            ctcm = (-cta + 2.0 * cm) / gama;
            b = (bmvl + 1.0) * (bmvl + 1.0);
            f[0] = 0.25 * cgm * rm * cm * b;
        } else {
            ctcm = (-cta - 2.0 * cm) / gama;
            b = (bmvl - 1.0) * (bmvl - 1.0);
            f[0] = -(0.25 * cgm * rm * cm * b);
        }
        f[1] = f[0] * (um + nxa * ctcm);
        f[2] = f[0] * (vm + nya * ctcm);
        f[3] = f[0] * (wm + nza * ctcm);
        f[4] = f[0] * hm;
    } else if (npn == 1 ? bmvl >= 1.0 : bmvl <= -1.0) {
        double rmct = rm * cta;
        f[0] = cgm * rmct;
        f[1] = cgm * (rmct * um + pm * nxa);
        f[2] = cgm * (rmct * vm + pm * nya);
        f[3] = cgm * (rmct * wm + pm * nza);
        f[4] = cgm * rmct * hm;
    }
    return bad;
}

// flux (Convect.f90:1245-1272) with getem (GasModel.f90:358-374)
__device__ __forceinline__ void phys_flux(double gama, const double *prim, double nx, double ny, double nz, double nt,
                                          double *f) {
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double em = pm / (gama - 1.0) + 0.5 * rm * (um * um + vm * vm + wm * wm);
    double cit = nx * um + ny * vm + nz * wm + nt;
    f[0] = rm * cit;
    f[1] = f[0] * um + nx * pm;
    f[2] = f[0] * vm + ny * pm;
    f[3] = f[0] * wm + nz * pm;
    f[4] = (em + pm) * cit - pm * nt;
}

// flux_Roe (flux.f90:116-244).  Returns 1 when c^2 <= 0.
__device__ __forceinline__ int flux_roe(const DevParams &P, const double *qlin, const double *qrin, double nx,
                                        double ny, double nz, double nt, double *f) {
    const double gama = P.gama;
    double ql[5], qr[5], fl[5], fr[5], dq[5];
#pragma unroll
    for (int m = 0; m < 5; m++) { ql[m] = qlin[m]; qr[m] = qrin[m]; }
    phys_flux(gama, ql, nx, ny, nz, nt, fl);
    phys_flux(gama, qr, nx, ny, nz, nt, fr);
#pragma unroll
    for (int m = 0; m < 5; m++) dq[m] = qr[m] - ql[m];
    double gama1 = gama - 1.0;
    double gama2 = gama / gama1;
    ql[4] = gama2 * ql[4] / ql[0] + 0.5 * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
    qr[4] = gama2 * qr[4] / qr[0] + 0.5 * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    double qroe0 = sqrt(ql[0] * qr[0]);
    double rrl = sqrt(qr[0] / ql[0]);
    double rrl_1 = rrl + 1.0;
    double um = (ql[1] + qr[1] * rrl) / rrl_1;
    double vm = (ql[2] + qr[2] * rrl) / rrl_1;
    double wm = (ql[3] + qr[3] * rrl) / rrl_1;
    double hm = (ql[4] + qr[4] * rrl) / rrl_1;
    double rm = qroe0;
    double c2 = (hm - 0.5 * (um * um + vm * vm + wm * wm)) * gama1;
    int bad = c2 <= 0.0 ? 1 : 0;
    double c = sqrt(c2);
    double cta = um * nx + vm * ny + wm * nz + nt;
    double cgm = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
    double cgm1 = 1.0 / cgm;
    nx = nx * cgm1;
    ny = ny * cgm1;
    nz = nz * cgm1;
    double ccgm = c * cgm;
    double l1 = fabs(cta - ccgm), l4 = fabs(cta), l5 = fabs(cta + ccgm);
    double l12 = l1 * l1, l42 = l4 * l4, l52 = l5 * l5;
    double deti = P.efix * cgm;
    double det2 = deti * deti;
    l1 = sqrt(l12 + det2);
    l4 = sqrt(l42 + det2);
    l5 = sqrt(l52 + det2);
    double dcta = dq[1] * nx + dq[2] * ny + dq[3] * nz;
    double cta1 = cta * cgm1;
    double rodcta = qroe0 * dcta;
    double dp_c2 = dq[4] / c2;
    double rodctac = rodcta / c;
    double a1 = l4 * (dq[0] - dp_c2);
    double a2 = l5 * (dp_c2 + rodctac) * 0.5;
    double a3 = l1 * (dp_c2 - rodctac) * 0.5;
    double a4 = a1 + a2 + a3;
    double a5 = c * (a2 - a3);
    double a6 = l4 * (rm * dq[1] - nx * rodcta);
    double a7 = l4 * (rm * dq[2] - ny * rodcta);
    double a8 = l4 * (rm * dq[3] - nz * rodcta);
    double df0 = a4;
    double df1 = um * a4 + nx * a5 + a6;
    double df2 = vm * a4 + ny * a5 + a7;
    double df3 = wm * a4 + nz * a5 + a8;
    double df4 = hm * a4 + cta1 * a5 + um * a6 + vm * a7 + wm * a8 - c2 * a1 / gama1;
    f[0] = 0.5 * (fr[0] + fl[0] - df0);
    f[1] = 0.5 * (fr[1] + fl[1] - df1);
    f[2] = 0.5 * (fr[2] + fl[2] - df2);
    f[3] = 0.5 * (fr[3] + fl[3] - df3);
    f[4] = 0.5 * (fr[4] + fl[4] - df4);
    return bad;
}

// the flux routine chosen by nflux (Convect.f90:12-46): 1 Steger-Warming,
// 2 Van Leer, 3 Roe.  Returns the number of c^2 failures.
__device__ __forceinline__ int flux_type(const DevParams &P, const double *ql, const double *qr, double nx, double ny,
                                         double nz, double nt, double *f) {
    if (P.nflux == 2) {
        double fl[5], fr[5];
        int bad = flux_vl_pn(P, ql, nx, ny, nz, nt, fl, 1);
        bad += flux_vl_pn(P, qr, nx, ny, nz, nt, fr, -1);
#pragma unroll
        for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
        return bad;
    }
    if (P.nflux == 1) {
        double fl[5], fr[5];
        flux_sw_pn(P, ql, nx, ny, nz, nt, fl, 1);
        flux_sw_pn(P, qr, nx, ny, nz, nt, fr, -1);
#pragma unroll
        for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
        return 0;
    }
    return flux_roe(P, ql, qr, nx, ny, nz, nt, f);
}

// mxdq_std (LHS.f90:756-828) with gettmhmgm_ns (GasModel.f90:411-426)
__device__ __forceinline__ void mxdq_std(const DevParams &P, const double *prim, double gx, double gy, double gz,
                                         const double *dq, double *f, double rad, int npn) {
    const double gama = P.gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double hint = P.g1 * pm / rm;
    double c2 = gama * pm / rm;
    double cm = sqrt(c2);
    double v2 = um * um + vm * vm + wm * wm;
    double hm = hint + 0.5 * v2;
    double nx = gx, ny = gy, nz = gz, nt = 0.0;
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
    double dn = (double)npn;
    double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    l1 = 0.5 * (l1 + dn * rad);
    l4 = 0.5 * (l4 + dn * rad);
    l5 = 0.5 * (l5 + dn * rad);
    double x1 = (2.0 * l1 - l4 - l5) / (2.0 * c2);
    double x2 = (l4 - l5) / (2.0 * cm);
    double cgm1 = 1.0 / cgm;
    nx = nx * cgm1;
    ny = ny * cgm1;
    nz = nz * cgm1;
    ct = (ct - nt) * cgm1;
    double ae = gama - 1.0;
    double af = 0.5 * ae * v2;
    double dc = ct * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3];
    double dh = af * dq[0] - ae * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4]);
    double c2dc = c2 * dc;
    f[0] = l1 * dq[0] - dh * x1 - dc * x2;
    f[1] = l1 * dq[1] + (nx * c2dc - um * dh) * x1 + (nx * dh - um * dc) * x2;
    f[2] = l1 * dq[2] + (ny * c2dc - vm * dh) * x1 + (ny * dh - vm * dc) * x2;
    f[3] = l1 * dq[3] + (nz * c2dc - wm * dh) * x1 + (nz * dh - wm * dc) * x2;
    f[4] = l1 * dq[4] + (ct * c2dc - hm * dh) * x1 + (ct * dh - hm * dc) * x2;
}

// Sutherland viscosity, compute_visl_ns (GasModel.f90:219-235)
__device__ __forceinline__ double sutherland(const DevParams &P, double tm) {
    return tm * sqrt(tm) * (1.0 + P.visc) / (tm + P.visc);
}

// error counters
enum ErrSlot : int { ERR_ROE = 0, ERR_UPDATE_BLOCKS = 1, ERR_BADLIST_OVERFLOW = 2, ERR_TIMEOUT = 3, ERR_NSLOTS = 4 };

}  // namespace wcns
