// k_rhs_mixed.cu -- the residual in mixed precision.
//
// The same residual as k_rhs_inv.cu / k_rhs_vis.cu (r_h_s_invis and
// r_h_s_vis, RHS.f90:2-72, with WCNS-E-5 and its 41/42 boundary sections,
// the Steger-Warming / Van Leer / Roe fluxes and the viscous line flux), with
// the precision split:
//   FP32  the staged prim line, the interpolation stencils, the nonlinear
//         weights' numerators, the numerical fluxes, the node and half-node
//         derivatives of (u,v,w,T), the stress and heat flux, and the flux
//         differences;
//   FP64  the grid metrics and volume (read as stored; their half-node
//         values are interpolated in FP64 and rounded once), the smoothness
//         indicators' denominators (eps + IS)^2 and the normalisation of the
//         weights, and the accumulation of every direction's difference into
//         dq; the time step, the LU-SGS sweeps and the update are unchanged.
// The arithmetic is free to differ from the reference's operation order (the
// file is compiled with multiply-add contraction); its error against the FP64
// path is what the mixed-precision tests measure.
#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

namespace {

// ---------------------------------------------------------------------------
// FP32 numerical fluxes (kct = 0: no grid velocity term)
// ---------------------------------------------------------------------------

// flux_SW_pn (flux.f90:17-77)
__device__ __forceinline__ void sw_pn_f(float gama, float g1, float efix, const float *q, float nx, float ny, float nz,
                                        float dn, float *f) {
    const float rm = q[0], um = q[1], vm = q[2], wm = q[3], pm = q[4];
    const float rinv = 1.0f / rm;
    const float u2 = 0.5f * (um * um + vm * vm + wm * wm);
    const float hint = g1 * pm * rinv;
    const float em = hint - pm * rinv + u2;
    const float c2 = gama * pm * rinv;
    const float cm = sqrtf(c2);
    const float ct = nx * um + ny * vm + nz * wm;
    const float cgm = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1.0e-30f);
    float l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    const float eps = efix * efix * cgm * cgm;
    l1 = 0.5f * (l1 + dn * sqrtf(l1 * l1 + eps));
    l4 = 0.5f * (l4 + dn * sqrtf(l4 * l4 + eps));
    l5 = 0.5f * (l5 + dn * sqrtf(l5 * l5 + eps));
    const float cgm1 = 1.0f / cgm;
    const float x1 = (2.0f * l1 - l4 - l5) / (2.0f * gama);
    const float x2 = cm * (l4 - l5) / (2.0f * gama);
    const float hm = em + pm * rinv;
    f[0] = (l1 - x1) * rm;
    f[1] = ((l1 - x1) * um + nx * cgm1 * x2) * rm;
    f[2] = ((l1 - x1) * vm + ny * cgm1 * x2) * rm;
    f[3] = ((l1 - x1) * wm + nz * cgm1 * x2) * rm;
    f[4] = (l1 * em - x1 * hm + ct * cgm1 * x2) * rm;
}

// flux_vanleer_pn (flux.f90:410-501); returns 1 when c^2 < 0
__device__ __forceinline__ int vl_pn_f(float gama, float g1, const float *q, float nx, float ny, float nz, int npn,
                                       float *f) {
    const float rm = q[0], um = q[1], vm = q[2], wm = q[3], pm = q[4];
    const float hm = g1 * pm / rm + 0.5f * (um * um + vm * vm + wm * wm);
    const float c2 = gama * pm / rm;
    const int bad = c2 < 0.0f ? 1 : 0;
    const float cm = sqrtf(c2);
    const float cgm = sqrtf(nx * nx + ny * ny + nz * nz) + 1.0e-30f;
    const float cgm1 = 1.0f / cgm;
    const float nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
    const float cta = (nx * um + ny * vm + nz * wm) * cgm1;
    const float bm = cta / cm;
#pragma unroll
    for (int m = 0; m < 5; m++) f[m] = 0.0f;
    if (fabsf(bm) < 1.0f) {
        const float ctcm = npn == 1 ? (-cta + 2.0f * cm) / gama : (-cta - 2.0f * cm) / gama;
        const float b = npn == 1 ? (bm + 1.0f) * (bm + 1.0f) : (bm - 1.0f) * (bm - 1.0f);
        f[0] = (npn == 1 ? 0.25f : -0.25f) * cgm * rm * cm * b;
        f[1] = f[0] * (um + nxa * ctcm);
        f[2] = f[0] * (vm + nya * ctcm);
        f[3] = f[0] * (wm + nza * ctcm);
        f[4] = f[0] * hm;
    } else if (npn == 1 ? bm >= 1.0f : bm <= -1.0f) {
        const float rmct = rm * cta;
        f[0] = cgm * rmct;
        f[1] = cgm * (rmct * um + pm * nxa);
        f[2] = cgm * (rmct * vm + pm * nya);
        f[3] = cgm * (rmct * wm + pm * nza);
        f[4] = cgm * rmct * hm;
    }
    return bad;
}

// flux (Convect.f90:1245-1272)
__device__ __forceinline__ void phys_flux_f(float gama, const float *q, float nx, float ny, float nz, float *f) {
    const float em = q[4] / (gama - 1.0f) + 0.5f * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float cit = nx * q[1] + ny * q[2] + nz * q[3];
    f[0] = q[0] * cit;
    f[1] = f[0] * q[1] + nx * q[4];
    f[2] = f[0] * q[2] + ny * q[4];
    f[3] = f[0] * q[3] + nz * q[4];
    f[4] = (em + q[4]) * cit;
}

// flux_Roe (flux.f90:116-244); returns 1 when c^2 <= 0
__device__ __forceinline__ int roe_f(float gama, float efix, const float *qlin, const float *qrin, float nx, float ny,
                                     float nz, float *f) {
    float fl[5], fr[5], dq[5];
    phys_flux_f(gama, qlin, nx, ny, nz, fl);
    phys_flux_f(gama, qrin, nx, ny, nz, fr);
#pragma unroll
    for (int m = 0; m < 5; m++) dq[m] = qrin[m] - qlin[m];
    const float gama1 = gama - 1.0f, gama2 = gama / gama1;
    const float hl = gama2 * qlin[4] / qlin[0] + 0.5f * (qlin[1] * qlin[1] + qlin[2] * qlin[2] + qlin[3] * qlin[3]);
    const float hr = gama2 * qrin[4] / qrin[0] + 0.5f * (qrin[1] * qrin[1] + qrin[2] * qrin[2] + qrin[3] * qrin[3]);
    const float qroe0 = sqrtf(qlin[0] * qrin[0]);
    const float rrl = sqrtf(qrin[0] / qlin[0]);
    const float w1 = 1.0f / (rrl + 1.0f);
    const float um = (qlin[1] + qrin[1] * rrl) * w1;
    const float vm = (qlin[2] + qrin[2] * rrl) * w1;
    const float wm = (qlin[3] + qrin[3] * rrl) * w1;
    const float hm = (hl + hr * rrl) * w1;
    const float c2 = (hm - 0.5f * (um * um + vm * vm + wm * wm)) * gama1;
    const int bad = c2 <= 0.0f ? 1 : 0;
    const float c = sqrtf(c2);
    const float cta = um * nx + vm * ny + wm * nz;
    const float cgm = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1.0e-30f);
    const float cgm1 = 1.0f / cgm;
    const float ux = nx * cgm1, uy = ny * cgm1, uz = nz * cgm1;
    const float ccgm = c * cgm;
    const float det2 = efix * cgm * efix * cgm;
    const float l1 = sqrtf((cta - ccgm) * (cta - ccgm) + det2);
    const float l4 = sqrtf(cta * cta + det2);
    const float l5 = sqrtf((cta + ccgm) * (cta + ccgm) + det2);
    const float rodcta = qroe0 * (dq[1] * ux + dq[2] * uy + dq[3] * uz);
    const float dp_c2 = dq[4] / c2;
    const float rodctac = rodcta / c;
    const float a1 = l4 * (dq[0] - dp_c2);
    const float a2 = l5 * (dp_c2 + rodctac) * 0.5f;
    const float a3 = l1 * (dp_c2 - rodctac) * 0.5f;
    const float a4 = a1 + a2 + a3;
    const float a5 = c * (a2 - a3);
    const float a6 = l4 * (qroe0 * dq[1] - ux * rodcta);
    const float a7 = l4 * (qroe0 * dq[2] - uy * rodcta);
    const float a8 = l4 * (qroe0 * dq[3] - uz * rodcta);
    f[0] = 0.5f * (fr[0] + fl[0] - a4);
    f[1] = 0.5f * (fr[1] + fl[1] - (um * a4 + ux * a5 + a6));
    f[2] = 0.5f * (fr[2] + fl[2] - (vm * a4 + uy * a5 + a7));
    f[3] = 0.5f * (fr[3] + fl[3] - (wm * a4 + uz * a5 + a8));
    f[4] = 0.5f * (fr[4] + fl[4] - (hm * a4 + cta * cgm1 * a5 + um * a6 + vm * a7 + wm * a8 - c2 * a1 / gama1));
    return bad;
}

__device__ __forceinline__ int flux_f(const DevParams &P, const float *ql, const float *qr, float nx, float ny,
                                      float nz, float *f) {
    const float gama = (float)P.gama, g1 = (float)P.g1;
    if (P.nflux == 3) return roe_f(gama, (float)P.efix, ql, qr, nx, ny, nz, f);
    float fl[5], fr[5];
    int bad = 0;
    if (P.nflux == 2) {
        bad = vl_pn_f(gama, g1, ql, nx, ny, nz, 1, fl);
        bad += vl_pn_f(gama, g1, qr, nx, ny, nz, -1, fr);
    } else {
        sw_pn_f(gama, g1, (float)P.efix, ql, nx, ny, nz, 1.0f, fl);
        sw_pn_f(gama, g1, (float)P.efix, qr, nx, ny, nz, -1.0f, fr);
    }
#pragma unroll
    for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
    return bad;
}

// ---------------------------------------------------------------------------
// inviscid line
// ---------------------------------------------------------------------------

// One-sided states of the boundary closures and the nscheme=41/42 boundary
// sections (WCNSE5.f90:2284-2459, 2524-2705, 2967-2986, 3207-3226): each
// state is (c0 q(1) + c1 q(2) + c2 q(3) + c3 q(4)) / den over the first four
// points of the line, or mirrored, over q(n), q(n-1), q(n-2), q(n-3).
enum SecRow : int {
    SEC_S1 = 0,      // section 1, h = 0..3 (rows 0..3); nscheme=42: rows 4..7
    SEC_S1_42 = 4,
    SEC_S2L = 8,     // section 2 left states, h = 1..5 (rows 8..12)
    SEC_S2R_2 = 13,  // section 2 right state at h = 2 (the others are the left ones)
    SEC_S3L_2 = 14,  // section 3 left state at h = 2
    SEC_C0 = 15,     // closure at the end half node (35,-35,21,-5)/16
    SEC_N = 16
};
__constant__ float c_sec[SEC_N][5] = {
    {3.f, -1.f, 0.f, 0.f, 2.f}, {19.f, 25.f, -2.f, 0.f, 42.f}, {4.f, 3.f, 9.f, 2.f, 18.f}, {-2.f, 3.f, 3.f, 2.f, 6.f},
    {677.f, -421.f, 99.f, 13.f, 368.f}, {5.f, 15.f, -5.f, 1.f, 16.f}, {-1.f, 9.f, 9.f, -1.f, 16.f}, {1.f, -5.f, 15.f, 5.f, 16.f},
    {3.f, 6.f, -1.f, 0.f, 8.f}, {-30.f, 145.f, 29.f, -8.f, 136.f}, {0.f, -1.f, 6.f, 3.f, 8.f}, {0.f, 1.f, 2.f, 5.f, 8.f},
    {0.f, 1.f, 1.f, 6.f, 8.f}, {2.f, 49.f, 125.f, -40.f, 136.f}, {-29.f, 170.f, 63.f, 12.f, 216.f}, {35.f, -35.f, 21.f, -5.f, 16.f}};

struct MxLine {
    const float *sq;  // prim minus the block's free stream, sq[m*(n+6) + l+2] for l = -2..n+3
    double *sk;       // metrics of the line direction, sk[c*n + l-1] for l = 1..n, until the
                      // half-node metrics are formed; then their difference at point l
    double *kh;       // half-node metrics, kh[c*(n+1) + h]
    long long stride, dqbase;
    int n, ist, ied;
};

__device__ __forceinline__ float mqv(const MxLine &L, int m, int l) { return L.sq[m * (L.n + 6) + l + 2]; }

// row r applied at the left end (right = false) or mirrored at the right end
__device__ __forceinline__ float sec_state(const MxLine &L, int m, int r, bool right) {
    const float *c = c_sec[r];
    const int n = L.n;
    const float a = right ? mqv(L, m, n) : mqv(L, m, 1), b = right ? mqv(L, m, n - 1) : mqv(L, m, 2);
    const float d = right ? mqv(L, m, n - 2) : mqv(L, m, 3), e = right ? mqv(L, m, n - 3) : mqv(L, m, 4);
    return (c[0] * a + c[1] * b + c[2] * d + c[3] * e) / c[4];
}

// qwl / qwr after the interpolation, with the end closures of a line that
// touches a physical boundary (ist > 1 or ied < n)
__device__ __forceinline__ float mx_qwl(const MxLine &L, const float *ql_, int m, int h) {
    const int n = L.n;
    if (L.ist > 1 && h <= 2) return sec_state(L, m, h == 0 ? SEC_C0 : (h == 1 ? SEC_S1_42 + 1 : SEC_S1_42 + 2), false);
    if (L.ied < n && h >= n - 1) return sec_state(L, m, h == n ? SEC_C0 : SEC_S1_42 + 1, true);
    return ql_[m * (n + 1) + h];
}
__device__ __forceinline__ float mx_qwr(const MxLine &L, const float *qr_, int m, int h) {
    const int n = L.n;
    if (L.ist > 1 && h <= 1) return sec_state(L, m, h == 0 ? SEC_C0 : SEC_S1_42 + 1, false);
    if (L.ied < n && h >= n - 2)
        return sec_state(L, m, h == n ? SEC_C0 : (h == n - 1 ? SEC_S1_42 + 1 : SEC_S1_42 + 2), true);
    return qr_[m * (n + 1) + h];
}
// left-section rows: section 1 at h = 0..3, section 2 (left/right) and 3 (left) at h = 1..5
__device__ __forceinline__ int row_s1(int o, bool s42) { return (s42 ? SEC_S1_42 : SEC_S1) + o; }
__device__ __forceinline__ int row_s2l(int o) { return SEC_S2L + o - 1; }
__device__ __forceinline__ int row_s2r(int o) { return o == 2 ? SEC_S2R_2 : SEC_S2L + o - 1; }
__device__ __forceinline__ int row_s3l(int o) { return o == 2 ? SEC_S3L_2 : SEC_S2L + o - 1; }

// FLUX_DXYZ (WCNSE5.f90:209-254) in FP32, f(h) for h in 0..n
template <class Acc>
__device__ __forceinline__ float mx_flux_dxyz(const Acc &f, int n, int l) {
    if (n <= NIJK2ND) return f(l) - f(l - 1);
    if (l == 1) return (-23.0f * f(0) + 21.0f * f(1) + 3.0f * f(2) - f(3)) / 24.0f;
    if (l == n) return -(-23.0f * f(n) + 21.0f * f(n - 1) + 3.0f * f(n - 2) - f(n - 3)) / 24.0f;
    if (l == 2) return (f(0) - 27.0f * f(1) + 27.0f * f(2) - f(3)) / 24.0f;
    if (l == n - 1) return -(f(n) - 27.0f * f(n - 1) + 27.0f * f(n - 2) - f(n - 3)) / 24.0f;
    return (2250.0f * (f(l) - f(l - 1)) - 125.0f * (f(l + 1) - f(l - 2)) + 9.0f * (f(l + 2) - f(l - 3))) / 1920.0f;
}

constexpr int MXI_MAX_LINES = 32;
// floats per line: prim 5 x (n+6), qwl, qwr, f 5 x (n+1) each, 26 x 5 section
// fluxes; odd, so that the lines of a group fall on different banks
__host__ __device__ inline int mxi_line_floats(int n) { return (5 * (n + 6) + 15 * (n + 1) + 130) | 1; }
// doubles per line: the metrics (later their half-node differences) 3 x n
// and the half-node metrics 3 x (n+1), odd for the same reason
__host__ __device__ inline int mxi_line_doubles(int n) { return (3 * n + 3 * (n + 1)) | 1; }

// The difference operator of the flux difference at point l: FLUX_DXYZ, or
// the boundary-section differences of nscheme=41/42 (WCNSE5.f90:2460-2523,
// 2706-2759) on values at the sections' half nodes.
template <class Acc>
__device__ __forceinline__ double mx_point_diff(const Acc &k, int n, int l, bool left, bool right) {
    if (right) {
        if (l == n) return -(-23.0 * k(n) + 21.0 * k(n - 1) + 3.0 * k(n - 2) - k(n - 3)) / 24.0;
        if (l == n - 1) return -(-22.0 * k(n - 1) + 17.0 * k(n - 2) + 9.0 * k(n - 3) - 5.0 * k(n - 4) + k(n - 5)) / 24.0;
        return -(k(n - 1) - 27.0 * k(n - 2) + 27.0 * k(n - 3) - k(n - 4)) / 24.0;
    }
    if (left) {
        if (l == 1) return (-23.0 * k(0) + 21.0 * k(1) + 3.0 * k(2) - k(3)) / 24.0;
        if (l == 2) return (-22.0 * k(1) + 17.0 * k(2) + 9.0 * k(3) - 5.0 * k(4) + k(5)) / 24.0;
        return (k(1) - 27.0 * k(2) + 27.0 * k(3) - k(4)) / 24.0;
    }
    return flux_dxyz_at(k, n, l);
}

// Physical flux (Convect.f90:1245-1272) at R + d minus the one at R, for a
// small deviation d of prim from the reference state R: every O(1) product
// of R alone is left out, so the FP32 result carries the rounding of the
// deviation's size only.  Ur = k.u(R), base0 = rho(R) Ur, Gr = rho H at R.
__device__ __forceinline__ void dev_phys(const float *R, float Ur, float base0, float Gr, float g1, const float *d,
                                         float nx, float ny, float nz, float *o) {
    const float Up = nx * d[1] + ny * d[2] + nz * d[3];
    const float U = Ur + Up;
    const float d0 = R[0] * Up + d[0] * U;
    const float u = R[1] + d[1], v = R[2] + d[2], w = R[3] + d[3];
    o[0] = d0;
    o[1] = base0 * d[1] + d0 * u + nx * d[4];
    o[2] = base0 * d[2] + d0 * v + ny * d[4];
    o[3] = base0 * d[3] + d0 * w + nz * d[4];
    const float Gp = g1 * d[4] + 0.5f * (d[0] * (u * u + v * v + w * w) +
                                         R[0] * (d[1] * (R[1] + u) + d[2] * (R[2] + v) + d[3] * (R[3] + w)));
    o[4] = Up * Gr + U * Gp;
}

// flux_Roe (flux.f90:116-244) minus the free-stream flux at the same
// metrics: the central part in deviation form, the dissipation |A|(qr - ql)
// from the Roe average of the full states; a, b the left and right states'
// deviations from R.  Returns 1 when c^2 <= 0.
__device__ __forceinline__ int roe_dev(float gama, float g1, float efix, const float *R, const float *a, const float *b,
                                       float nx, float ny, float nz, float *f) {
    const float Ur = nx * R[1] + ny * R[2] + nz * R[3];
    const float base0 = R[0] * Ur;
    const float Gr = g1 * R[4] + 0.5f * R[0] * (R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
    float da[5], db[5], ql[5], qr[5], dq[5];
    dev_phys(R, Ur, base0, Gr, g1, a, nx, ny, nz, da);
    dev_phys(R, Ur, base0, Gr, g1, b, nx, ny, nz, db);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        ql[m] = R[m] + a[m];
        qr[m] = R[m] + b[m];
        dq[m] = b[m] - a[m];
    }
    const float gama1 = gama - 1.0f;
    const float hl = g1 * ql[4] / ql[0] + 0.5f * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
    const float hr = g1 * qr[4] / qr[0] + 0.5f * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    const float qroe0 = sqrtf(ql[0] * qr[0]);
    const float rrl = sqrtf(qr[0] / ql[0]);
    const float w1 = 1.0f / (rrl + 1.0f);
    const float um = (ql[1] + qr[1] * rrl) * w1;
    const float vm = (ql[2] + qr[2] * rrl) * w1;
    const float wm = (ql[3] + qr[3] * rrl) * w1;
    const float hm = (hl + hr * rrl) * w1;
    const float c2 = (hm - 0.5f * (um * um + vm * vm + wm * wm)) * gama1;
    const int bad = c2 <= 0.0f ? 1 : 0;
    const float c = sqrtf(c2);
    const float cta = um * nx + vm * ny + wm * nz;
    const float cgm = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1.0e-30f);
    const float cgm1 = 1.0f / cgm;
    const float ux = nx * cgm1, uy = ny * cgm1, uz = nz * cgm1;
    const float ccgm = c * cgm;
    const float det2 = efix * cgm * efix * cgm;
    const float l1 = sqrtf((cta - ccgm) * (cta - ccgm) + det2);
    const float l4 = sqrtf(cta * cta + det2);
    const float l5 = sqrtf((cta + ccgm) * (cta + ccgm) + det2);
    const float rodcta = qroe0 * (dq[1] * ux + dq[2] * uy + dq[3] * uz);
    const float dp_c2 = dq[4] / c2;
    const float rodctac = rodcta / c;
    const float a1 = l4 * (dq[0] - dp_c2);
    const float a2 = l5 * (dp_c2 + rodctac) * 0.5f;
    const float a3 = l1 * (dp_c2 - rodctac) * 0.5f;
    const float a4 = a1 + a2 + a3;
    const float a5 = c * (a2 - a3);
    const float a6 = l4 * (qroe0 * dq[1] - ux * rodcta);
    const float a7 = l4 * (qroe0 * dq[2] - uy * rodcta);
    const float a8 = l4 * (qroe0 * dq[3] - uz * rodcta);
    f[0] = 0.5f * (da[0] + db[0] - a4);
    f[1] = 0.5f * (da[1] + db[1] - (um * a4 + ux * a5 + a6));
    f[2] = 0.5f * (da[2] + db[2] - (vm * a4 + uy * a5 + a7));
    f[3] = 0.5f * (da[3] + db[3] - (wm * a4 + uz * a5 + a8));
    f[4] = 0.5f * (da[4] + db[4] - (hm * a4 + cta * cgm1 * a5 + um * a6 + vm * a7 + wm * a8 - c2 * a1 / gama1));
    return bad;
}

}  // namespace

// The inviscid residual along one direction in mixed precision, in
// deviation form: with R the block's free stream (roo, uoo, voo, woo, poo),
// every flux is F(R, k_h) + F', where the first part is linear in the
// half-node metrics k_h and is differenced in FP64 as
// sum_d F_d(R) * D[k_h,d] (D the point's difference operator), and F', the
// flux minus F(R, k_h), is formed and differenced in FP32.  The staged prim
// are q - R, which the (consistent) interpolation stencils carry unchanged.
template <int dir>
__global__ void __launch_bounds__(256, 3) k_rhs_invis_mx(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                      const LineGroup *__restrict__ groups, int *err, double *out,
                                                      long long stride) {
    extern __shared__ double smem_d[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir);
    const int H = n + 1, W = n + 6;
    const int NL = G.nl;
    const int LF = mxi_line_floats(n), LD = mxi_line_doubles(n);
    double *sdbase = smem_d;                              // NL x LD doubles
    float *sfbase = (float *)(smem_d + (size_t)NL * LD);  // NL x LF floats
    __shared__ MxLine lines[MXI_MAX_LINES];
    __shared__ double FR[15];  // Cartesian fluxes at R: x, y, z, five components each
    const double Rd[5] = {P.roo, P.uoo, P.voo, P.woo, B.poo};
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    if (threadIdx.x < NL) {
        int c[3];
        c[a1] = G.a0 + threadIdx.x;
        c[a2] = G.b;
        c[dir] = -2;
        const long long base = gidx(B, c[0], c[1], c[2]);
        MxLine L;
        L.sq = sfbase + (size_t)threadIdx.x * LF;
        L.sk = sdbase + (size_t)threadIdx.x * LD;
        L.kh = L.sk + 3 * n;
        L.stride = dstride(B, dir);
        L.dqbase = base + 2 * L.stride;
        L.n = n;
        L.ist = __ldg(F.f[F_R] + base) < SMALL ? 2 : 0;
        L.ied = __ldg(F.f[F_R] + base + (long long)(n + 5) * L.stride) < SMALL ? n - 2 : n;
        lines[threadIdx.x] = L;
    } else if (threadIdx.x == 32) {
        const double rho = Rd[0], u = Rd[1], v = Rd[2], w = Rd[3], p = Rd[4];
        const double G = P.g1 * p + 0.5 * rho * (u * u + v * v + w * w);
        const double vel[3] = {u, v, w};
        for (int d = 0; d < 3; d++) {
            FR[5 * d] = rho * vel[d];
            FR[5 * d + 1] = rho * vel[d] * u + (d == 0 ? p : 0.0);
            FR[5 * d + 2] = rho * vel[d] * v + (d == 1 ? p : 0.0);
            FR[5 * d + 3] = rho * vel[d] * w + (d == 2 ? p : 0.0);
            FR[5 * d + 4] = vel[d] * G;
        }
    }
    __syncthreads();
    constexpr bool posmajor = (dir == 0);
    const FastDiv dNL = fast_div_init(NL), d5NL = fast_div_init(5 * NL), dW = fast_div_init(W);
    // ---- stage prim - R (rounded to FP32) and the metrics (FP64)
    for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
        const int qq = posmajor ? fdiv(e, dW) : fdiv(e, dNL);
        const int ln = posmajor ? qq : e - qq * NL;
        const int p = posmajor ? e - qq * W : qq;
        const MxLine &L = lines[ln];
        const long long gi = L.dqbase + (long long)(p - 2) * L.stride;
        double v[8];
#pragma unroll
        for (int m = 0; m < 5; m++) v[m] = __ldg(F.f[F_R + m] + gi);
        const bool inner = p >= 3 && p <= n + 2;
#pragma unroll
        for (int c = 0; c < 3; c++) v[5 + c] = inner ? __ldg(F.f[F_KCX + 3 * dir + c] + gi) : 0.0;
        float *sq = sfbase + (size_t)ln * LF;
#pragma unroll
        for (int m = 0; m < 5; m++) sq[m * W + p] = (float)(v[m] - Rd[m]);
        if (inner) {
#pragma unroll
            for (int c = 0; c < 3; c++) L.sk[c * n + p - 3] = v[5 + c];
        }
    }
    __syncthreads();
    const size_t work0 = (size_t)5 * W;
    // ---- interpolation per (line, variable, point i in [ist, ied+1]); the
    // half-node metrics per (line, half node)
    {
        const int NP = n + 2;
        for (int idx = threadIdx.x; idx < NL * 5 * NP; idx += blockDim.x) {
            const int q1 = fdiv(idx, dNL), i = fdiv(idx, d5NL);
            const int ln = idx - q1 * NL, m = q1 - 5 * i;
            const MxLine &L = lines[ln];
            if (i < L.ist || i > L.ied + 1) continue;
            float *ql_ = sfbase + (size_t)ln * LF + work0;
            float *qr_ = ql_ + (size_t)5 * H;
            const float qm2 = mqv(L, m, i - 2), qm1 = mqv(L, m, i - 1), q0 = mqv(L, m, i), qp1 = mqv(L, m, i + 1),
                        qp2 = mqv(L, m, i + 2);
            const float g0 = 0.5f * (qm2 - 4.0f * qm1 + 3.0f * q0), g1 = 0.5f * (qp1 - qm1),
                        g2 = 0.5f * (-3.0f * q0 + 4.0f * qp1 - qp2);
            const float s0 = qm2 - 2.0f * qm1 + q0, s1 = qm1 - 2.0f * q0 + qp1, s2 = q0 - 2.0f * qp1 + qp2;
            // denominators (eps + IS)^2 in FP64; the weights c_k/a_k normalised
            // as c_k prod_{j!=k} a_j / sum_l c_l prod_{j!=l} a_j (one division)
            const double t0 = 1.0e-6 + (double)(g0 * g0 + s0 * s0), t1 = 1.0e-6 + (double)(g1 * g1 + s1 * s1),
                         t2 = 1.0e-6 + (double)(g2 * g2 + s2 * s2);
            const double a0 = t0 * t0, a1 = t1 * t1, a2 = t2 * t2;
            const double p0 = a1 * a2, p1 = a0 * a2, p2 = a0 * a1;
            if (i <= L.ied) {  // left state at half node i: weights 1, 10, 5 (/16)
                const double inv = 1.0 / (p0 + 10.0 * p1 + 5.0 * p2);
                const float w0 = (float)(p0 * inv), w1 = (float)(10.0 * p1 * inv), w2 = (float)(5.0 * p2 * inv);
                ql_[m * H + i] = q0 + 0.125f * (w0 * (s0 + 4.0f * g0) + w1 * (s1 + 4.0f * g1) + w2 * (s2 + 4.0f * g2));
            }
            if (i - 1 >= L.ist) {  // right state at half node i-1: weights 5, 10, 1 (/16)
                const double inv = 1.0 / (5.0 * p0 + 10.0 * p1 + p2);
                const float w0 = (float)(5.0 * p0 * inv), w1 = (float)(10.0 * p1 * inv), w2 = (float)(p2 * inv);
                qr_[m * H + i - 1] = q0 + 0.125f * (w0 * (s0 - 4.0f * g0) + w1 * (s1 - 4.0f * g1) + w2 * (s2 - 4.0f * g2));
            }
        }
        for (int idx = threadIdx.x; idx < NL * H; idx += blockDim.x) {  // VALUE_HALF_NODE of the metrics
            const int h = fdiv(idx, dNL), ln = idx - h * NL;
            const MxLine &L = lines[ln];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                auto a = [&](int l) { return L.sk[c * n + l - 1]; };
                L.kh[c * H + h] = value_half_node_at(a, n, h);
            }
        }
    }
    __syncthreads();
    // ---- deviation fluxes at the half nodes and the boundary-section
    // fluxes; the difference of the half-node metrics at every point
    const bool sections = P.nscheme == 41 || P.nscheme == 42;
    {
        const bool s42 = P.nscheme == 42;
        const float Rf[5] = {(float)Rd[0], (float)Rd[1], (float)Rd[2], (float)Rd[3], (float)Rd[4]};
        const float gama = (float)P.gama, g1f = (float)P.g1, efix = (float)P.efix;
        int nbad = 0;
        for (int idx = threadIdx.x; idx < NL * (H + 26); idx += blockDim.x) {
            const int t = fdiv(idx, dNL);
            const int ln = idx - t * NL;
            const MxLine &L = lines[ln];
            const float *ql_ = sfbase + (size_t)ln * LF + work0;
            const float *qr_ = ql_ + (size_t)5 * H;
            float ql[5], qr[5], fl[5];
            int h, mode = 0;
            if (t < H) {
                h = t;
#pragma unroll
                for (int m = 0; m < 5; m++) { ql[m] = mx_qwl(L, ql_, m, h); qr[m] = mx_qwr(L, qr_, m, h); }
                if (Rf[0] + ql[0] <= (float)RMIN_LIMIT || Rf[4] + ql[4] <= (float)PMIN_LIMIT) {
                    const int ii = h > 1 ? h : 1;
#pragma unroll
                    for (int m = 0; m < 5; m++) ql[m] = mqv(L, m, ii);
                }
                if (Rf[0] + qr[0] <= (float)RMIN_LIMIT || Rf[4] + qr[4] <= (float)PMIN_LIMIT) {
                    const int ii = h + 1 < n ? h + 1 : n;
#pragma unroll
                    for (int m = 0; m < 5; m++) qr[m] = mqv(L, m, ii);
                }
            } else {
                if (!sections) continue;
                const int sidx = t - H;
                if (sidx < 13) {
                    if (L.ist <= 1) continue;
                    if (sidx < 4) { mode = 1; h = sidx; }
                    else if (sidx < 9) { mode = 2; h = sidx - 3; }
                    else { mode = 3; h = sidx - 8; }
                } else {
                    if (L.ied >= n) continue;
                    const int r = sidx - 13;
                    if (r < 4) { mode = 4; h = n - r; }
                    else if (r < 9) { mode = 5; h = n - 1 - (r - 4); }
                    else { mode = 6; h = n - 1 - (r - 9); }
                }
                const int o = mode <= 3 ? h : n - h;  // distance from the line end
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    switch (mode) {
                    case 1: ql[m] = qr[m] = sec_state(L, m, row_s1(o, s42), false); break;
                    case 2: ql[m] = sec_state(L, m, row_s2l(o), false); qr[m] = sec_state(L, m, row_s2r(o), false); break;
                    case 3: ql[m] = sec_state(L, m, row_s3l(o), false); qr[m] = mx_qwr(L, qr_, m, h); break;
                    case 4: ql[m] = qr[m] = sec_state(L, m, row_s1(o, s42), true); break;
                    case 5: ql[m] = sec_state(L, m, row_s2r(o), true); qr[m] = sec_state(L, m, row_s2l(o), true); break;
                    default:
                        // the left value as the right sections saw it: the left
                        // sections' result where they ran (h <= 5)
                        ql[m] = (L.ist > 1 && h <= 5)
                                    ? sec_state(L, m, h == 0 ? row_s1(0, s42) : row_s3l(h), false)
                                    : mx_qwl(L, ql_, m, h);
                        qr[m] = sec_state(L, m, row_s3l(o), true);
                        break;
                    }
                }
                const bool badl = Rf[0] + ql[0] <= (float)RMIN_LIMIT || Rf[4] + ql[4] <= (float)PMIN_LIMIT;
                const bool badr = Rf[0] + qr[0] <= (float)RMIN_LIMIT || Rf[4] + qr[4] <= (float)PMIN_LIMIT;
                const int ia = h > 1 ? h : 1, ib = h + 1 < n ? h + 1 : n;
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    if (mode == 1) {
                        if (badl) ql[m] = 0.5f * (mqv(L, m, ia) + mqv(L, m, h + 1));
                        if (badr) qr[m] = 0.5f * (mqv(L, m, ia) + mqv(L, m, h + 1));
                    } else if (mode == 4) {
                        if (badl) ql[m] = 0.5f * (mqv(L, m, 1) + mqv(L, m, h));
                        if (badr) qr[m] = 0.5f * (mqv(L, m, 1) + mqv(L, m, h));
                    } else {
                        if (badl) ql[m] = mqv(L, m, ia);
                        if (badr) qr[m] = mqv(L, m, ib);
                    }
                }
            }
            const double kxd = L.kh[h], kyd = L.kh[H + h], kzd = L.kh[2 * H + h];
            const float kx = (float)kxd, ky = (float)kyd, kz = (float)kzd;
            if (P.nflux == 3) {
                nbad += roe_dev(gama, g1f, efix, Rf, ql, qr, kx, ky, kz, fl);
            } else {
                // Steger-Warming / Van Leer: the full FP32 flux less F(R, k_h)
                float a[5], b[5];
#pragma unroll
                for (int m = 0; m < 5; m++) { a[m] = Rf[m] + ql[m]; b[m] = Rf[m] + qr[m]; }
                nbad += flux_f(P, a, b, kx, ky, kz, fl);
#pragma unroll
                for (int m = 0; m < 5; m++) fl[m] -= (float)(kxd * FR[m] + kyd * FR[5 + m] + kzd * FR[10 + m]);
            }
            float *dst = mode == 0 ? sfbase + (size_t)ln * LF + work0 + (size_t)10 * H + h
                                   : sfbase + (size_t)ln * LF + work0 + (size_t)15 * H + (size_t)(t - H) * 5;
            const int dm = mode == 0 ? H : 1;
#pragma unroll
            for (int m = 0; m < 5; m++) dst[m * dm] = fl[m];
        }
        if (nbad) atomicAdd(&err[ERR_ROE], nbad);
        for (int idx = threadIdx.x; idx < NL * n; idx += blockDim.x) {  // D[k_h] at every point
            const int l0 = fdiv(idx, dNL), ln = idx - l0 * NL, l = l0 + 1;
            const MxLine &L = lines[ln];
            const bool right = sections && L.ied < n && l >= n - 2;
            const bool left = !right && sections && L.ist > 1 && l <= 3;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                auto k = [&](int hh) { return L.kh[c * H + hh]; };
                L.sk[c * n + l0] = mx_point_diff(k, n, l, left, right);
            }
        }
    }
    __syncthreads();
    // ---- flux difference per (line, point, variable): the deviation part in
    // FP32, the free-stream part and the accumulation into dq in FP64
    for (int idx = threadIdx.x; idx < NL * n * 5; idx += blockDim.x) {
        const int q1 = fdiv(idx, dNL), l0 = fdiv(idx, d5NL);
        const int ln = idx - q1 * NL, m = q1 - 5 * l0, l = 1 + l0;
        const MxLine &L = lines[ln];
        const float *f_ = sfbase + (size_t)ln * LF + work0 + (size_t)10 * H;
        const float *sc = sfbase + (size_t)ln * LF + work0 + (size_t)15 * H;
        const bool right = sections && L.ied < n && l >= n - 2;
        const bool left = !right && sections && L.ist > 1 && l <= 3;
        float df;
        if (right) {
            const float *s4 = sc + 13 * 5, *s5 = sc + 17 * 5, *s6 = sc + 22 * 5;
            if (l == n) df = -(-23.0f * s4[m] + 21.0f * s4[5 + m] + 3.0f * s4[10 + m] - s4[15 + m]) / 24.0f;
            else if (l == n - 1) df = -(-22.0f * s5[m] + 17.0f * s5[5 + m] + 9.0f * s5[10 + m] - 5.0f * s5[15 + m] + s5[20 + m]) / 24.0f;
            else df = -(s6[m] - 27.0f * s6[5 + m] + 27.0f * s6[10 + m] - s6[15 + m]) / 24.0f;
        } else if (left) {
            const float *s1 = sc, *s2 = sc + 4 * 5, *s3 = sc + 9 * 5;
            if (l == 1) df = (-23.0f * s1[m] + 21.0f * s1[5 + m] + 3.0f * s1[10 + m] - s1[15 + m]) / 24.0f;
            else if (l == 2) df = (-22.0f * s2[m] + 17.0f * s2[5 + m] + 9.0f * s2[10 + m] - 5.0f * s2[15 + m] + s2[20 + m]) / 24.0f;
            else df = (s3[m] - 27.0f * s3[5 + m] + 27.0f * s3[10 + m] - s3[15 + m]) / 24.0f;
        } else {
            auto fa = [&](int hh) { return f_[m * H + hh]; };
            df = mx_flux_dxyz(fa, n, l);
        }
        const double dfr = FR[m] * L.sk[l0] + FR[5 + m] * L.sk[n + l0] + FR[10 + m] * L.sk[2 * n + l0];
        const double v = dfr + (double)df;
        const long long gi = L.dqbase + (long long)l * L.stride;
        if (out) out[m * stride + gi] = v;
        else F.f[F_DQ1 + m][gi] += v;
    }
}
// ---------------------------------------------------------------------------
// viscous: node derivatives of (u,v,w,T) in FP32, stored as FP32
// (UVWT_DER_4th_virtual sub_tgh.f90:1909-2029, DUVWT_NODE_LINE_virtual
// 2217-2272); duv[(m + 4d) * total + point]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 4) k_node_deriv_mx(DevFields F, const DevBlock *__restrict__ blocks, int nblocks,
                                                        float *__restrict__ duv, long long total) {
    const int bi = blockIdx.y;
    if (bi >= nblocks) return;
    const DevBlock B = blocks[bi];
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < B.npts; p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_point(B, p, i, j, k);
        const long long id = gidx(B, i, j, k);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const int n = dimof(B, d);
            const int l = d == 0 ? i : (d == 1 ? j : k);
            const long long st = dstride(B, d);
            const long long l0 = id - (long long)l * st;
            const bool fl = __ldg(F.f[F_R] + l0 - 2 * st) < 0.0 || __ldg(F.f[F_T] + l0 - 2 * st) < 0.0;
            const bool fr = __ldg(F.f[F_R] + l0 + (long long)(n + 3) * st) < 0.0 ||
                            __ldg(F.f[F_T] + l0 + (long long)(n + 3) * st) < 0.0;
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const double *u = F.f[m == 3 ? F_T : F_U + m] + l0;
                auto U = [&](int x) { return (float)__ldg(u + (long long)x * st); };
                float du;
                if (n <= NIJK2ND) du = 0.5f * (U(l + 1) - U(l - 1));
                else if (fl && l == 1) du = (-11.f * U(1) + 18.f * U(2) - 9.f * U(3) + 2.f * U(4)) / 6.0f;
                else if (fl && l == 2) du = (-3.f * U(1) - 10.f * U(2) + 18.f * U(3) - 6.f * U(4) + U(5)) / 12.0f;
                else if (fr && l == n) du = -(-11.f * U(n) + 18.f * U(n - 1) - 9.f * U(n - 2) + 2.f * U(n - 3)) / 6.0f;
                else if (fr && l == n - 1)
                    du = -(-3.f * U(n) - 10.f * U(n - 1) + 18.f * U(n - 2) - 6.f * U(n - 3) + U(n - 4)) / 12.0f;
                else du = (8.f * (U(l + 1) - U(l - 1)) - (U(l + 2) - U(l - 2))) / 12.0f;
                duv[(long long)(m + 4 * d) * total + id] = du;
            }
        }
    }
}

namespace {
// staged line of the viscous kernel: FP32 u, v, w, T, the 8 node derivatives
// along the other two directions and the two viscosities; FP64 metrics
// (kcx,etx,ctx,kcy,ety,cty,kcz,etz,ctz) and volume; per point l = -1..n+2
constexpr int MXV_NF = 14, MXV_ND = 10;
enum : int { MV_U = 0, MV_DN = 4, MV_V1 = 12, MV_V2 = 13 };
constexpr int MXV_MAX_LINES = 32;
constexpr int MXV_THREADS = 384;
__host__ __device__ inline int mxv_line_floats(int n) { return (MXV_NF * (n + 4) + 4 * (n + 1)) | 1; }
__host__ __device__ inline int mxv_line_doubles(int n) { return (MXV_ND * (n + 4)) | 1; }

struct MxvLine {
    long long l0, st;
    int n;
    bool fl, fr;
};
}  // namespace

template <int dir>
__global__ void __launch_bounds__(MXV_THREADS, 2) k_rhs_vis_mx(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                           const LineGroup *__restrict__ groups,
                                                           const float *__restrict__ duv, long long total, double *out,
                                                           long long stride) {
    extern __shared__ double smem_d[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir);
    const int H = n + 1, W = n + 4;
    const int NL = G.nl;
    const int LF = mxv_line_floats(n), LD = mxv_line_doubles(n);
    double *sdbase = smem_d;
    float *sfbase = (float *)(smem_d + (size_t)NL * LD);
    __shared__ MxvLine lines[MXV_MAX_LINES];
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    if (threadIdx.x < NL) {
        int c[3];
        c[a1] = G.a0 + threadIdx.x;
        c[a2] = G.b;
        c[dir] = 0;
        MxvLine L;
        L.l0 = gidx(B, c[0], c[1], c[2]);
        L.st = dstride(B, dir);
        L.n = n;
        L.fl = F.f[F_R][L.l0 - 2 * L.st] < 0.0 || F.f[F_T][L.l0 - 2 * L.st] < 0.0;
        L.fr = F.f[F_R][L.l0 + (long long)(n + 3) * L.st] < 0.0 || F.f[F_T][L.l0 + (long long)(n + 3) * L.st] < 0.0;
        lines[threadIdx.x] = L;
    }
    __syncthreads();
    const bool posmajor = (dir == 0);
    const FastDiv dNL = fast_div_init(NL), dW = fast_div_init(W);
    {
        const int g0 = dir == 0 ? 1 : 0, g1 = dir == 2 ? 1 : 2;
        for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
            const int qq = posmajor ? fdiv(e, dW) : fdiv(e, dNL);
            const int ln = posmajor ? qq : e - qq * NL;
            const int p = posmajor ? e - qq * W : qq;
            const MxvLine &L = lines[ln];
            const int l = p - 1;
            const long long gi = L.l0 + (long long)l * L.st;
            const bool inner = l >= 1 && l <= n;
            float v[MXV_NF];
            double dv[MXV_ND];
            double tm = 0.0;
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const double x = __ldg(F.f[m == 3 ? F_T : F_U + m] + gi);
                v[MV_U + m] = (float)x;
                if (m == 3) tm = x;
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                v[MV_DN + m] = inner ? __ldg(duv + (long long)(m + 4 * g0) * total + gi) : 0.0f;
                v[MV_DN + 4 + m] = inner ? __ldg(duv + (long long)(m + 4 * g1) * total + gi) : 0.0f;
            }
#pragma unroll
            for (int c = 0; c < 9; c++) dv[c] = inner ? __ldg(F.f[F_KCX + 3 * (c % 3) + c / 3] + gi) : 0.0;
            dv[9] = inner ? __ldg(F.f[F_VOL] + gi) : 0.0;
            const float tf = (float)tm, visc = (float)P.visc;
            const float mu = inner ? tf * sqrtf(tf) * (1.0f + visc) / (tf + visc) : 0.0f;
            const float vt = (inner && F.f[F_VIST]) ? (float)__ldg(F.f[F_VIST] + gi) : 0.0f;
            v[MV_V1] = inner ? mu + vt : 0.0f;
            v[MV_V2] = inner ? mu * (float)B.cp_prl + vt * (float)B.cp_prt : 0.0f;
            float *S = sfbase + (size_t)ln * LF + p;
#pragma unroll
            for (int f = 0; f < MXV_NF; f++) S[f * W] = v[f];
            double *D = sdbase + (size_t)ln * LD + p;
#pragma unroll
            for (int f = 0; f < MXV_ND; f++) D[f * W] = dv[f];
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < NL * H; idx += blockDim.x) {
        const int h = fdiv(idx, dNL);
        const int ln = idx - h * NL;
        const MxvLine &L = lines[ln];
        const float *S = sfbase + (size_t)ln * LF;
        const double *D = sdbase + (size_t)ln * LD;
        auto at = [&](int f, int x) { return S[f * W + x + 1]; };
        // (u,v,w,T) at the half node (VALUE_line_half_virtual)
        float uh[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            auto Q = [&](int x) { return at(MV_U + m, x); };
            float v;
            if (n <= NIJK2ND) v = 0.5f * (Q(h) + Q(h + 1));
            else if (L.fl && h == 0) v = (35.f * Q(1) - 35.f * Q(2) + 21.f * Q(3) - 5.f * Q(4)) / 16.f;
            else if (L.fl && h == 1) v = (5.f * Q(1) + 15.f * Q(2) - 5.f * Q(3) + Q(4)) / 16.f;
            else if (L.fr && h == n) v = (35.f * Q(n) - 35.f * Q(n - 1) + 21.f * Q(n - 2) - 5.f * Q(n - 3)) / 16.f;
            else if (L.fr && h == n - 1) v = (5.f * Q(n) + 15.f * Q(n - 1) - 5.f * Q(n - 2) + Q(n - 3)) / 16.f;
            else v = (9.f * (Q(h) + Q(h + 1)) - (Q(h + 2) + Q(h - 1))) / 16.f;
            uh[m] = v;
        }
        // derivatives at the half node: own direction from the line
        // (DUVWT_half_line_virtual), the others interpolated from the node
        // derivatives (VALUE_HALF_NODE_IJK)
        float dh[12];
#pragma unroll
        for (int g = 0; g < 3; g++) {
#pragma unroll
            for (int m = 0; m < 4; m++) {
                float v;
                if (g == dir) {
                    auto Q = [&](int x) { return at(MV_U + m, x); };
                    if (n <= NIJK2ND) v = Q(h + 1) - Q(h);
                    else if (L.fl && h == 0) v = (-71.f * Q(1) + 141.f * Q(2) - 93.f * Q(3) + 23.f * Q(4)) / 24.f;
                    else if (L.fl && h == 1) v = (-22.f * Q(1) + 17.f * Q(2) + 9.f * Q(3) - 5.f * Q(4) + Q(5)) / 24.f;
                    else if (L.fr && h == n) v = -(-71.f * Q(n) + 141.f * Q(n - 1) - 93.f * Q(n - 2) + 23.f * Q(n - 3)) / 24.f;
                    else if (L.fr && h == n - 1)
                        v = -(-22.f * Q(n) + 17.f * Q(n - 1) + 9.f * Q(n - 2) - 5.f * Q(n - 3) + Q(n - 4)) / 24.f;
                    else v = (27.f * (Q(h + 1) - Q(h)) - (Q(h + 2) - Q(h - 1))) / 24.f;
                } else {
                    const int slot = MV_DN + 4 * (g < dir ? g : g - 1) + m;
                    auto Dn = [&](int x) { return at(slot, x); };
                    if (n <= NIJK2ND) {
                        if (h == 0) v = 1.5f * Dn(1) - 0.5f * Dn(n < 2 ? n : 2);
                        else if (h == n) v = 1.5f * Dn(n) - 0.5f * Dn(n - 1 > 1 ? n - 1 : 1);
                        else v = 0.5f * (Dn(h) + Dn(h + 1));
                    } else if (h == 0) v = (35.f * Dn(1) - 35.f * Dn(2) + 21.f * Dn(3) - 5.f * Dn(4)) / 16.f;
                    else if (h == n) v = (35.f * Dn(n) - 35.f * Dn(n - 1) + 21.f * Dn(n - 2) - 5.f * Dn(n - 3)) / 16.f;
                    else if (h == 1) v = (5.f * Dn(1) + 15.f * Dn(2) - 5.f * Dn(3) + Dn(4)) / 16.f;
                    else if (h == n - 1) v = (5.f * Dn(n) + 15.f * Dn(n - 1) - 5.f * Dn(n - 2) + Dn(n - 3)) / 16.f;
                    else v = (9.f * (Dn(h) + Dn(h + 1)) - (Dn(h + 2) + Dn(h - 1))) / 16.f;
                }
                dh[m + 4 * g] = v;
            }
        }
        // metrics and volume at the half node in FP64, rounded once
        float kh[9];
#pragma unroll
        for (int c = 0; c < 9; c++) {
            auto Q = [&](int x) { return D[c * W + x + 1]; };
            kh[c] = (float)value_half_node_at(Q, n, h);
        }
        auto Qv = [&](int x) { return D[9 * W + x + 1]; };
        const float rvol = (float)(1.0 / value_half_node_at(Qv, n, h));
        auto half_f = [&](int f) {
            auto Q = [&](int x) { return at(f, x); };
            if (n <= NIJK2ND) {
                if (h == 0) return (15.f * Q(1) - 10.f * Q(n < 2 ? n : 2) + 3.f * Q(n < 3 ? n : 3)) / 8.f;
                if (h == n) return (15.f * Q(n) - 10.f * Q(n - 1 > 1 ? n - 1 : 1) + 3.f * Q(n - 2 > 1 ? n - 2 : 1)) / 8.f;
                return 0.5f * (Q(h) + Q(h + 1));
            }
            if (h == 0) return (35.f * Q(1) - 35.f * Q(2) + 21.f * Q(3) - 5.f * Q(4)) / 16.f;
            if (h == n) return (35.f * Q(n) - 35.f * Q(n - 1) + 21.f * Q(n - 2) - 5.f * Q(n - 3)) / 16.f;
            if (h == 1) return (5.f * Q(1) + 15.f * Q(2) - 5.f * Q(3) + Q(4)) / 16.f;
            if (h == n - 1) return (5.f * Q(n) + 15.f * Q(n - 1) - 5.f * Q(n - 2) + Q(n - 3)) / 16.f;
            return (9.f * (Q(h) + Q(h + 1)) - (Q(h + 2) + Q(h - 1))) / 16.f;
        };
        const float vs = half_f(MV_V1), kcp = half_f(MV_V2);
        // Cartesian gradients (DUVWT_DXYZ)
        float dx[12];
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const float k1 = kh[3 * m], k2 = kh[3 * m + 1], k3 = kh[3 * m + 2];
#pragma unroll
            for (int v = 0; v < 4; v++) dx[m + 3 * v] = (k1 * dh[v] + k2 * dh[4 + v] + k3 * dh[8 + v]) * rvol;
        }
        // stress and heat flux (FLUX_VIS_LINE_new)
        const float vscc = vs * (float)P.cc23;
        const float t1 = vscc * (2.f * dx[0] - dx[4] - dx[8]);
        const float t5 = vscc * (2.f * dx[4] - dx[8] - dx[0]);
        const float t9 = vscc * (2.f * dx[8] - dx[0] - dx[4]);
        const float t2 = vs * (dx[1] + dx[3]);
        const float t3 = vs * (dx[2] + dx[6]);
        const float t6 = vs * (dx[5] + dx[7]);
        const float nx = kh[dir], ny = kh[3 + dir], nz = kh[6 + dir];
        const float f1 = t1 * nx + t2 * ny + t3 * nz;
        const float f2 = t2 * nx + t5 * ny + t6 * nz;
        const float f3 = t3 * nx + t6 * ny + t9 * nz;
        const float f4 = uh[0] * f1 + uh[1] * f2 + uh[2] * f3 + kcp * (dx[9] * nx + dx[10] * ny + dx[11] * nz);
        float *fv = sfbase + (size_t)ln * LF + (size_t)MXV_NF * W;
        fv[0 * H + h] = f1;
        fv[1 * H + h] = f2;
        fv[2 * H + h] = f3;
        fv[3 * H + h] = f4;
    }
    __syncthreads();
    // ---- per point: FLUX_DXYZ and dq -= re*dfv, accumulated in FP64
    // (the continuity component of the viscous flux is zero)
    for (int idx = threadIdx.x; idx < NL * n; idx += blockDim.x) {
        const int l0 = fdiv(idx, dNL);
        const int ln = idx - l0 * NL;
        const int l = 1 + l0;
        const MxvLine &L = lines[ln];
        const float *fv = sfbase + (size_t)ln * LF + (size_t)MXV_NF * W;
        const long long gi = L.l0 + (long long)l * L.st;
        if (out) out[gi] = 0.0;
#pragma unroll
        for (int m = 1; m < 5; m++) {
            auto fa = [&](int hh) { return fv[(m - 1) * H + hh]; };
            const double dfv = (double)mx_flux_dxyz(fa, n, l);
            if (out) out[m * stride + gi] = P.re * dfv;
            else F.f[F_DQ1 + m][gi] -= P.re * dfv;
        }
    }
}

// ---------------------------------------------------------------------------
// launches
// ---------------------------------------------------------------------------
size_t rhs_invis_mx_line_bytes(int n) { return (size_t)mxi_line_floats(n) * 4 + (size_t)mxi_line_doubles(n) * 8; }
size_t rhs_vis_mx_line_bytes(int n) { return (size_t)mxv_line_floats(n) * 4 + (size_t)mxv_line_doubles(n) * 8; }
int rhs_invis_mx_max_lines() { return MXI_MAX_LINES; }
int rhs_vis_mx_max_lines() { return MXV_MAX_LINES; }

void setup_rhs_mx_attrs(size_t inv_smem, size_t vis_smem) {
    cudaFuncSetAttribute(k_rhs_invis_mx<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem);
    cudaFuncSetAttribute(k_rhs_invis_mx<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem);
    cudaFuncSetAttribute(k_rhs_invis_mx<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem);
    cudaFuncSetAttribute(k_rhs_vis_mx<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vis_smem);
    cudaFuncSetAttribute(k_rhs_vis_mx<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vis_smem);
    cudaFuncSetAttribute(k_rhs_vis_mx<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vis_smem);
}

void launch_rhs_invis_mx(const LaunchCtx &c, int dir, cudaStream_t st, double *out) {
    const DirTable &T = c.inv_mx[dir];
    if (T.ngroups == 0) return;
    if (dir == 0) k_rhs_invis_mx<0><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, c.total);
    else if (dir == 1) k_rhs_invis_mx<1><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, c.total);
    else k_rhs_invis_mx<2><<<T.ngroups, 256, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.err, out, c.total);
}

void launch_rhs_vis_mx(const LaunchCtx &c, int dir, cudaStream_t st, double *out) {
    const DirTable &T = c.vis_mx[dir];
    if (T.ngroups == 0) return;
    if (dir == 0) k_rhs_vis_mx<0><<<T.ngroups, MXV_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.duv32, c.total, out, c.total);
    else if (dir == 1) k_rhs_vis_mx<1><<<T.ngroups, MXV_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.duv32, c.total, out, c.total);
    else k_rhs_vis_mx<2><<<T.ngroups, MXV_THREADS, T.smem, st>>>(*c.P, *c.F, c.blocks, T.groups, c.duv32, c.total, out, c.total);
}

void launch_node_derivatives_mx(const LaunchCtx &c) {
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = c.hblocks[b].npts > maxp ? c.hblocks[b].npts : maxp;
    k_node_deriv_mx<<<dim3((unsigned)((maxp + 255) / 256), c.nblocks), 256, 0, c.stream>>>(*c.F, c.blocks, c.nblocks,
                                                                                          c.duv32, c.total);
}

}  // namespace wcns
