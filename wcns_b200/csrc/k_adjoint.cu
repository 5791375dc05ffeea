// k_adjoint.cu -- tangent and adjoint of the inviscid residual, and of the
// LU-SGS operator, for the discrete adjoint.
//
// Residual (r_h_s_invis, RHS.f90:35-72, with WCNS-E-5 nscheme=4,
// WCNSE5.f90:2-206, the Steger-Warming (flux.f90:2-77) or Roe
// (flux.f90:116-244) flux and FLUX_DXYZ, WCNSE5.f90:209-254), as a function
// of the ghosted prim field q (ghosts included: they are inputs):
//   tangent  rdot = (dr/dq) v     k_rhs_invis_jvp: forward mode, one dual
//                                 component through the whole line;
//   adjoint  qbar = (dr/dq)^T l   k_rhs_invis_vjp: per line the forward
//                                 states are recomputed, then the flux
//                                 difference is transposed, the flux's
//                                 Jacobian (dual numbers over the ten left
//                                 and right state components) is applied
//                                 transposed, and the WCNS interpolation is
//                                 transposed with its nonlinear weights
//                                 recomputed (dual numbers over the five
//                                 stencil points), not stored.
// Interface ghosts are copies of partner points (k_ghost_copy), so their
// adjoint is added to the partner point (k_ghost_copy_adj); the ghosts of
// physical boundaries are held fixed (their adjoint is returned separately).
//
// LU-SGS (lusgs_l / lusgs_u, LHS.f90:381-577, neighbour terms mxdq_std
// 756-828, inviscid): the linear operator P b = -(I + C U)^-1 (I - C L)^-1 C b
// of one lower and one upper sweep (C = coed, L / U the lower / upper
// neighbour terms), and its transpose P^T y = -C (I - L^T C)^-1 (I + U^T C)^-1 y.
// The neighbour term of point p in L^T and U^T is the split Jacobian
// evaluated at p itself, A^T y = l1 y + a (x1 c2 N.y - x2 V.y) + b (x2 N.y - x1 V.y)
// for A = l1 I + x1 (c2 N a^T - V b^T) + x2 (N b^T - V a^T) (the rank-two form
// of mxdq_std), so each transposed sweep is again a wavefront over planes.
#include <algorithm>

#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace wcns {

namespace {

// ---------------------------------------------------------------------------
// forward-mode dual numbers (FP64 value, N tangents)
// ---------------------------------------------------------------------------
template <int N>
struct Dual {
    double v;
    double d[N];
};
template <int N>
__device__ __forceinline__ Dual<N> dconst(double v) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = 0.0;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a) {
    Dual<N> r; r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, double b) { Dual<N> r = a; r.v = a.v + b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator+(double b, const Dual<N> &a) { return a + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, double b) { Dual<N> r = a; r.v = a.v - b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator-(double b, const Dual<N> &a) { return -(a - b); }
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, double b) {
    Dual<N> r; r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double b, const Dual<N> &a) { return a * b; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, double b) {
    Dual<N> r; r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] / b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N> &b) { return dconst<N>(a) / b; }
template <int N> __device__ __forceinline__ Dual<N> dsqrt(const Dual<N> &a) {
    Dual<N> r; r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * h;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dabs(const Dual<N> &a) { return a.v < 0.0 ? -a : a; }

// ---------------------------------------------------------------------------
// WCNS-E-5 half-node states (WCNSE5.f90:2-206): the left state at half node
// i and the right state at half node i-1 from q(i-2..i+2), weights recomputed
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void wcns_states(const T &qm2, const T &qm1, const T &q0, const T &qp1, const T &qp2, T &ql,
                                            T &qr) {
    const double CL[3] = {1.0 / 16.0, 10.0 / 16.0, 5.0 / 16.0};
    const double CR[3] = {5.0 / 16.0, 10.0 / 16.0, 1.0 / 16.0};
    T g[3], s[3], bl[3], br[3];
    g[0] = 0.5 * (qm2 - 4.0 * qm1 + 3.0 * q0);
    g[1] = 0.5 * (qp1 - qm1);
    g[2] = 0.5 * (-3.0 * q0 + 4.0 * qp1 - qp2);
    s[0] = qm2 - 2.0 * qm1 + q0;
    s[1] = qm1 - 2.0 * q0 + qp1;
    s[2] = q0 - 2.0 * qp1 + qp2;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const T tt = 1.0e-6 + (g[k] * g[k] + s[k] * s[k]);
        const T e2 = tt * tt;
        bl[k] = CL[k] / e2;
        br[k] = CR[k] / e2;
    }
    const T sl = bl[0] + bl[1] + bl[2], sr = br[0] + br[1] + br[2];
    ql = q0 + 0.125 * ((bl[0] / sl) * (s[0] + 4.0 * g[0]) + (bl[1] / sl) * (s[1] + 4.0 * g[1]) +
                       (bl[2] / sl) * (s[2] + 4.0 * g[2]));
    qr = q0 + 0.125 * ((br[0] / sr) * (s[0] - 4.0 * g[0]) + (br[1] / sr) * (s[1] - 4.0 * g[1]) +
                       (br[2] / sr) * (s[2] - 4.0 * g[2]));
}

// the end closures of a line at a physical boundary (ist > 1 / ied < n):
// the state at half node h is sum_j c[j] q(l_j) over four points; returns
// the number of terms (0: h is not a closure half node for this side)
__device__ __forceinline__ int closure(int n, int ist, int ied, bool left_state, int h, double *c, int *l) {
    const double C0[4] = {35.0 / 16.0, -35.0 / 16.0, 21.0 / 16.0, -5.0 / 16.0};
    const double C1[4] = {5.0 / 16.0, 15.0 / 16.0, -5.0 / 16.0, 1.0 / 16.0};
    const double C2[4] = {-1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0};
    const double *r = nullptr;
    bool right_end = false;
    if (ist > 1 && (h == 0 || h == 1 || (left_state && h == 2))) r = h == 0 ? C0 : (h == 1 ? C1 : C2);
    else if (ied < n && (h == n || h == n - 1 || (!left_state && h == n - 2))) {
        r = h == n ? C0 : (h == n - 1 ? C1 : C2);
        right_end = true;
    }
    if (!r) return 0;
    for (int j = 0; j < 4; j++) {
        c[j] = r[j];
        l[j] = right_end ? n - j : 1 + j;
    }
    return 4;
}

// ---------------------------------------------------------------------------
// fluxes (kct = 0) for T = double or a dual number
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void sw_pn_t(const DevParams &P, const T *q, double nx, double ny, double nz, int npn, T *f) {
    const double gama = P.gama;
    const T rm = q[0], um = q[1], vm = q[2], wm = q[3], pm = q[4];
    const T u2 = 0.5 * (um * um + vm * vm + wm * wm);
    const T hint = P.g1 * pm / rm;
    const T eint = hint - pm / rm;
    const T em = eint + u2;
    const T cm = dsqrt(gama * pm / rm);
    const T ct = nx * um + ny * vm + nz * wm;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    cgm = fmax(cgm, SML_SSS);
    T l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    const double eps = P.efix * P.efix * cgm * cgm;
    const double dn = (double)npn;
    l1 = 0.5 * (l1 + dn * dsqrt(l1 * l1 + eps));
    l4 = 0.5 * (l4 + dn * dsqrt(l4 * l4 + eps));
    l5 = 0.5 * (l5 + dn * dsqrt(l5 * l5 + eps));
    const double cgm1 = 1.0 / cgm;
    const double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
    const T cta = ct * cgm1;
    const T c2r = cm * cm / gama;
    const T x1 = c2r * (2.0 * l1 - l4 - l5) / (2.0 * cm * cm);
    const T x2 = c2r * (l4 - l5) / (2.0 * cm);
    const T hm = em + pm / rm;
    f[0] = (l1 - x1) * rm;
    f[1] = (l1 * um - x1 * um + nxa * x2) * rm;
    f[2] = (l1 * vm - x1 * vm + nya * x2) * rm;
    f[3] = (l1 * wm - x1 * wm + nza * x2) * rm;
    f[4] = (l1 * em - x1 * hm + cta * x2) * rm;
}

template <class T>
__device__ __forceinline__ void phys_t(double gama, const T *q, double nx, double ny, double nz, T *f) {
    const T em = q[4] / (gama - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const T cit = nx * q[1] + ny * q[2] + nz * q[3];
    f[0] = q[0] * cit;
    f[1] = f[0] * q[1] + nx * q[4];
    f[2] = f[0] * q[2] + ny * q[4];
    f[3] = f[0] * q[3] + nz * q[4];
    f[4] = (em + q[4]) * cit;
}

template <class T>
__device__ __forceinline__ void roe_t(const DevParams &P, const T *qlin, const T *qrin, double nx, double ny, double nz,
                                     T *f) {
    const double gama = P.gama;
    T ql[5], qr[5], fl[5], fr[5], dq[5];
#pragma unroll
    for (int m = 0; m < 5; m++) { ql[m] = qlin[m]; qr[m] = qrin[m]; }
    phys_t(gama, ql, nx, ny, nz, fl);
    phys_t(gama, qr, nx, ny, nz, fr);
#pragma unroll
    for (int m = 0; m < 5; m++) dq[m] = qr[m] - ql[m];
    const double gama1 = gama - 1.0, gama2 = gama / gama1;
    ql[4] = gama2 * ql[4] / ql[0] + 0.5 * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
    qr[4] = gama2 * qr[4] / qr[0] + 0.5 * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    const T qroe0 = dsqrt(ql[0] * qr[0]);
    const T rrl = dsqrt(qr[0] / ql[0]);
    const T rrl_1 = rrl + 1.0;
    const T um = (ql[1] + qr[1] * rrl) / rrl_1, vm = (ql[2] + qr[2] * rrl) / rrl_1, wm = (ql[3] + qr[3] * rrl) / rrl_1;
    const T hm = (ql[4] + qr[4] * rrl) / rrl_1;
    const T c2 = (hm - 0.5 * (um * um + vm * vm + wm * wm)) * gama1;
    const T c = dsqrt(c2);
    const T cta = um * nx + vm * ny + wm * nz;
    const double cgm = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
    const double cgm1 = 1.0 / cgm;
    const double ux = nx * cgm1, uy = ny * cgm1, uz = nz * cgm1;
    const T ccgm = c * cgm;
    const T a_l1 = dabs(cta - ccgm), a_l4 = dabs(cta), a_l5 = dabs(cta + ccgm);
    const double deti = P.efix * cgm;
    const double det2 = deti * deti;
    const T l1 = dsqrt(a_l1 * a_l1 + det2), l4 = dsqrt(a_l4 * a_l4 + det2), l5 = dsqrt(a_l5 * a_l5 + det2);
    const T dcta = dq[1] * ux + dq[2] * uy + dq[3] * uz;
    const T cta1 = cta * cgm1;
    const T rodcta = qroe0 * dcta;
    const T dp_c2 = dq[4] / c2;
    const T rodctac = rodcta / c;
    const T a1 = l4 * (dq[0] - dp_c2);
    const T a2 = l5 * (dp_c2 + rodctac) * 0.5;
    const T a3 = l1 * (dp_c2 - rodctac) * 0.5;
    const T a4 = a1 + a2 + a3;
    const T a5 = c * (a2 - a3);
    const T a6 = l4 * (qroe0 * dq[1] - ux * rodcta);
    const T a7 = l4 * (qroe0 * dq[2] - uy * rodcta);
    const T a8 = l4 * (qroe0 * dq[3] - uz * rodcta);
    f[0] = 0.5 * (fr[0] + fl[0] - a4);
    f[1] = 0.5 * (fr[1] + fl[1] - (um * a4 + ux * a5 + a6));
    f[2] = 0.5 * (fr[2] + fl[2] - (vm * a4 + uy * a5 + a7));
    f[3] = 0.5 * (fr[3] + fl[3] - (wm * a4 + uz * a5 + a8));
    f[4] = 0.5 * (fr[4] + fl[4] - (hm * a4 + cta1 * a5 + um * a6 + vm * a7 + wm * a8 - c2 * a1 / gama1));
}

template <class T>
__device__ __forceinline__ void flux_t(const DevParams &P, const T *ql, const T *qr, double nx, double ny, double nz,
                                      T *f) {
    if (P.nflux == 1) {
        T fl[5], fr[5];
        sw_pn_t(P, ql, nx, ny, nz, 1, fl);
        sw_pn_t(P, qr, nx, ny, nz, -1, fr);
#pragma unroll
        for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
    } else {
        roe_t(P, ql, qr, nx, ny, nz, f);
    }
}

// doubles of shared memory per line of the tangent / adjoint kernels:
// prim and a second 5 x (n+6) array (the tangent, or the adjoint
// accumulators), the line's lambda 5 x n, the metrics 3 x n, the half-node
// tangent fluxes 5 x (n+1); odd, so that the lines of a group fall on
// different banks
__host__ __device__ inline int adj_line_stride(int n) { return (10 * (n + 6) + 8 * n + 15 * (n + 1)) | 1; }

struct AdjLine {
    double *q, *x, *lam, *sk, *fd;  // x: tangent (jvp) or accumulated adjoint (vjp)
    double *sb;  // (vjp) adjoint of the WCNS left (m*(n+1)+h) and right ((5+m)*(n+1)+h) states
    long long stride, base;          // base: field index of position l = 0
    int n, ist, ied;
};

__device__ __forceinline__ void adj_line_init(AdjLine &L, double *smem, int ln, int LS, const DevFields &F,
                                              const DevBlock &B, const LineGroup &G, int dir) {
    const int n = dimof(B, dir), W = n + 6;
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    int c[3];
    c[a1] = G.a0 + ln;
    c[a2] = G.b;
    c[dir] = 0;
    L.base = gidx(B, c[0], c[1], c[2]);
    L.stride = dstride(B, dir);
    L.n = n;
    double *S = smem + (size_t)ln * LS;
    L.q = S;
    L.x = S + 5 * W;
    L.lam = S + 10 * W;
    L.sk = L.lam + 5 * n;
    L.fd = L.sk + 3 * n;
    L.sb = L.fd + 5 * (n + 1);
    L.ist = F.f[F_R][L.base - 2 * L.stride] < SMALL ? 2 : 0;
    L.ied = F.f[F_R][L.base + (long long)(n + 3) * L.stride] < SMALL ? n - 2 : n;
}

// value at point l (-2..n+3) of variable m
__device__ __forceinline__ double &aq(const AdjLine &L, double *a, int m, int l) { return a[m * (L.n + 6) + l + 2]; }

// The state of variable m at half node h (left = true: left state), as the
// residual forms it: closure, else WCNS-E-5 at point h (left) or h+1 (right).
template <class T, class Get>
__device__ __forceinline__ T half_state(const AdjLine &L, bool left, int h, const Get &get) {
    double c[4];
    int l[4];
    if (closure(L.n, L.ist, L.ied, left, h, c, l)) return c[0] * get(l[0]) + c[1] * get(l[1]) + c[2] * get(l[2]) + c[3] * get(l[3]);
    const int i = left ? h : h + 1;
    T ql, qr;
    wcns_states<T>(get(i - 2), get(i - 1), get(i), get(i + 1), get(i + 2), ql, qr);
    return left ? ql : qr;
}

}  // namespace

// tangent: out[m*stride + point] += d r_dir / dq . v  for every interior point
// of the lines of this direction (v: five ghosted fields, stride apart)
template <int dir>
__global__ void __launch_bounds__(256) k_rhs_invis_jvp(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                    const LineGroup *__restrict__ groups, const double *__restrict__ v,
                                                    double *out, long long stride) {
    extern __shared__ double smem[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir), W = n + 6, H = n + 1, NL = G.nl, LS = adj_line_stride(n);
    __shared__ AdjLine lines[INV_LINES_DEFAULT];
    if (threadIdx.x < NL) adj_line_init(lines[threadIdx.x], smem, threadIdx.x, LS, F, B, G, dir);
    __syncthreads();
    for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
        const int ln = e / W, p = e - ln * W;
        const AdjLine &L = lines[ln];
        const long long gi = L.base + (long long)(p - 2) * L.stride;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            aq(L, L.q, m, p - 2) = F.f[F_R + m][gi];
            aq(L, L.x, m, p - 2) = v[m * stride + gi];
        }
        if (p >= 3 && p <= n + 2)
#pragma unroll
            for (int c = 0; c < 3; c++) L.sk[c * n + p - 3] = F.f[F_KCX + 3 * dir + c][gi];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NL * H; e += blockDim.x) {
        const int ln = e / H, h = e - ln * H;
        const AdjLine &L = lines[ln];
        Dual<1> ql[5], qr[5], f[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            auto get = [&](int l) { Dual<1> d; d.v = aq(L, L.q, m, l); d.d[0] = aq(L, L.x, m, l); return d; };
            ql[m] = half_state<Dual<1>>(L, true, h, get);
            qr[m] = half_state<Dual<1>>(L, false, h, get);
        }
        if (ql[0].v <= RMIN_LIMIT || ql[4].v <= PMIN_LIMIT) {
            const int ii = h > 1 ? h : 1;
#pragma unroll
            for (int m = 0; m < 5; m++) { ql[m].v = aq(L, L.q, m, ii); ql[m].d[0] = aq(L, L.x, m, ii); }
        }
        if (qr[0].v <= RMIN_LIMIT || qr[4].v <= PMIN_LIMIT) {
            const int ii = h + 1 < n ? h + 1 : n;
#pragma unroll
            for (int m = 0; m < 5; m++) { qr[m].v = aq(L, L.q, m, ii); qr[m].d[0] = aq(L, L.x, m, ii); }
        }
        auto ax = [&](int l) { return L.sk[l - 1]; };
        auto ay = [&](int l) { return L.sk[n + l - 1]; };
        auto az = [&](int l) { return L.sk[2 * n + l - 1]; };
        flux_t(P, ql, qr, value_half_node_at(ax, n, h), value_half_node_at(ay, n, h), value_half_node_at(az, n, h), f);
#pragma unroll
        for (int m = 0; m < 5; m++) L.fd[m * H + h] = f[m].d[0];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NL * n * 5; e += blockDim.x) {
        const int ln = e / (5 * n), r = e - ln * 5 * n, m = r / n, l = r - m * n + 1;
        const AdjLine &L = lines[ln];
        auto fa = [&](int hh) { return L.fd[m * H + hh]; };
        out[m * stride + L.base + (long long)l * L.stride] += flux_dxyz_at(fa, n, l);
    }
}


namespace {
// coefficient of f(h) in the flux difference at point l (FLUX_DXYZ applied
// to the indicator of half node h)
__device__ __forceinline__ double dxyz_coef(int n, int l, int h) {
    auto ind = [&](int hh) { return hh == h ? 1.0 : 0.0; };
    return flux_dxyz_at(ind, n, l);
}

// routes the adjoint `sbar` of one half-node state of variable m: through
// the closure's constant coefficients into the line's point adjoints, or
// into the line's state adjoints for the WCNS phase; returns nothing to do
// when it is zero
__device__ __forceinline__ void route_state(const AdjLine &L, bool left, int h, int m, double sbar) {
    double c[4];
    int l[4];
    const int H = L.n + 1;
    double &slot = L.sb[(left ? m : 5 + m) * H + h];
    if (closure(L.n, L.ist, L.ied, left, h, c, l)) {
        slot = 0.0;
        if (sbar != 0.0)
            for (int j = 0; j < 4; j++) atomicAdd(&aq(L, L.x, m, l[j]), c[j] * sbar);
        return;
    }
    slot = sbar;
}
}  // namespace

// adjoint: out[m*stride + point] += (d r_dir / dq)^T lam at every point of
// the lines of this direction, ghosts included (lam: five fields, interior
// values used)
template <int dir>
__global__ void __launch_bounds__(256) k_rhs_invis_vjp(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                    const LineGroup *__restrict__ groups, const double *__restrict__ lam,
                                                    double *out, long long stride) {
    extern __shared__ double smem[];
    const LineGroup G = groups[blockIdx.x];
    const DevBlock B = blocks[G.blk];
    const int n = dimof(B, dir), W = n + 6, H = n + 1, NL = G.nl, LS = adj_line_stride(n);
    __shared__ AdjLine lines[INV_LINES_DEFAULT];
    if (threadIdx.x < NL) adj_line_init(lines[threadIdx.x], smem, threadIdx.x, LS, F, B, G, dir);
    __syncthreads();
    for (int e = threadIdx.x; e < NL * W; e += blockDim.x) {
        const int ln = e / W, p = e - ln * W;
        const AdjLine &L = lines[ln];
        const long long gi = L.base + (long long)(p - 2) * L.stride;
        const bool inner = p >= 3 && p <= n + 2;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            aq(L, L.q, m, p - 2) = F.f[F_R + m][gi];
            aq(L, L.x, m, p - 2) = 0.0;
            if (inner) L.lam[m * n + p - 3] = lam[m * stride + gi];
        }
        if (inner)
#pragma unroll
            for (int c = 0; c < 3; c++) L.sk[c * n + p - 3] = F.f[F_KCX + 3 * dir + c][gi];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NL * H; e += blockDim.x) {
        const int ln = e / H, h = e - ln * H;
        const AdjLine &L = lines[ln];
        // f_bar(h) = sum over the points whose difference reads f(h)
        double fb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        const int l0 = h - 2 > 1 ? h - 2 : 1, l1 = h + 3 < n ? h + 3 : n;
        for (int l = l0; l <= l1; l++) {
            const double cf = dxyz_coef(n, l, h);
            if (cf != 0.0)
#pragma unroll
                for (int m = 0; m < 5; m++) fb[m] += cf * L.lam[m * n + l - 1];
        }
        // the states as the residual forms them, then the flux's Jacobian,
        // one side's five components at a time (left, then right)
        double vl[5], vr[5];
        bool fall_l, fall_r;
        {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                auto get = [&](int l) { return aq(L, L.q, m, l); };
                vl[m] = half_state<double>(L, true, h, get);
                vr[m] = half_state<double>(L, false, h, get);
            }
            fall_l = vl[0] <= RMIN_LIMIT || vl[4] <= PMIN_LIMIT;
            fall_r = vr[0] <= RMIN_LIMIT || vr[4] <= PMIN_LIMIT;
            const int il = h > 1 ? h : 1, ir = h + 1 < n ? h + 1 : n;
#pragma unroll
            for (int m = 0; m < 5; m++) {
                if (fall_l) vl[m] = aq(L, L.q, m, il);
                if (fall_r) vr[m] = aq(L, L.q, m, ir);
            }
        }
        auto ax = [&](int l) { return L.sk[l - 1]; };
        auto ay = [&](int l) { return L.sk[n + l - 1]; };
        auto az = [&](int l) { return L.sk[2 * n + l - 1]; };
        const double kx = value_half_node_at(ax, n, h), ky = value_half_node_at(ay, n, h), kz = value_half_node_at(az, n, h);
        double qlb[5], qrb[5];
#pragma unroll 1
        for (int side = 0; side < 2; side++) {
            Dual<5> ql[5], qr[5], f[5];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                ql[m] = dconst<5>(vl[m]);
                qr[m] = dconst<5>(vr[m]);
                if (side == 0) ql[m].d[m] = 1.0;
                else qr[m].d[m] = 1.0;
            }
            flux_t(P, ql, qr, kx, ky, kz, f);
            double *dst = side == 0 ? qlb : qrb;
#pragma unroll
            for (int j = 0; j < 5; j++) {
                double a = 0.0;
#pragma unroll
                for (int m = 0; m < 5; m++) a += fb[m] * f[m].d[j];
                dst[j] = a;
            }
        }
        const int il = h > 1 ? h : 1, ir = h + 1 < n ? h + 1 : n;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            if (fall_l) {
                atomicAdd(&aq(L, L.x, m, il), qlb[m]);
                L.sb[m * H + h] = 0.0;
            } else {
                route_state(L, true, h, m, qlb[m]);
            }
            if (fall_r) {
                atomicAdd(&aq(L, L.x, m, ir), qrb[m]);
                L.sb[(5 + m) * H + h] = 0.0;
            } else {
                route_state(L, false, h, m, qrb[m]);
            }
        }
    }
    __syncthreads();
    // WCNS-E-5 transposed, per (line, variable, point i): the left state at
    // half node i and the right state at half node i-1 come from the same
    // stencil q(i-2..i+2); one evaluation with five dual tangents recomputes
    // the weights and gives both states' derivatives
    for (int e = threadIdx.x; e < NL * 5 * (n + 2); e += blockDim.x) {
        const int ln = e / (5 * (n + 2)), r = e - ln * 5 * (n + 2), m = r / (n + 2), i = r - m * (n + 2);
        const AdjLine &L = lines[ln];
        const double a = i <= n ? L.sb[m * H + i] : 0.0;
        const double b = i >= 1 ? L.sb[(5 + m) * H + i - 1] : 0.0;
        if (a == 0.0 && b == 0.0) continue;
        Dual<5> sv[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            sv[k] = dconst<5>(aq(L, L.q, m, i - 2 + k));
            sv[k].d[k] = 1.0;
        }
        Dual<5> ql, qr;
        wcns_states<Dual<5>>(sv[0], sv[1], sv[2], sv[3], sv[4], ql, qr);
#pragma unroll
        for (int k = 0; k < 5; k++) atomicAdd(&aq(L, L.x, m, i - 2 + k), ql.d[k] * a + qr.d[k] * b);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NL * W * 5; e += blockDim.x) {
        const int ln = e / (5 * W), r = e - ln * 5 * W, m = r / W, p = r - m * W;
        const AdjLine &L = lines[ln];
        const double a = aq(L, L.x, m, p - 2);
        if (a != 0.0) out[m * stride + L.base + (long long)(p - 2) * L.stride] += a;
    }
}


// ---------------------------------------------------------------------------
// the LU-SGS operator and its transpose
// ---------------------------------------------------------------------------
namespace {

// the rank-two form of mxdq_std (LHS.f90:756-828) at point id, direction d:
// A = l1 I + x1 (c2 N a^T - V b^T) + x2 (N b^T - V a^T)
struct Split {
    double l1, x1, x2, c2, a[5], b[5], N[5], V[5];
};

__device__ __forceinline__ Split split_at(const DevParams &P, const DevFields &F, long long id, int d, int npn) {
    Split S;
    const double gama = P.gama;
    const double rm = F.f[F_R][id], um = F.f[F_U][id], vm = F.f[F_V][id], wm = F.f[F_W][id], pm = F.f[F_P][id];
    const double hint = P.g1 * pm / rm, c2 = gama * pm / rm, cm = sqrt(c2);
    const double v2 = um * um + vm * vm + wm * wm, hm = hint + 0.5 * v2;
    double nx = F.f[F_KCX + 3 * d][id], ny = F.f[F_KCX + 3 * d + 1][id], nz = F.f[F_KCX + 3 * d + 2][id];
    double ct = nx * um + ny * vm + nz * wm;
    const double cgm = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
    const double rad = F.f[F_SRA + d][id], dn = (double)npn;
    const double l1 = 0.5 * (ct + dn * rad), l4 = 0.5 * (ct + cm * cgm + dn * rad), l5 = 0.5 * (ct - cm * cgm + dn * rad);
    S.l1 = l1;
    S.c2 = c2;
    S.x1 = (2.0 * l1 - l4 - l5) / (2.0 * c2);
    S.x2 = (l4 - l5) / (2.0 * cm);
    const double cgm1 = 1.0 / cgm;
    nx *= cgm1;
    ny *= cgm1;
    nz *= cgm1;
    ct *= cgm1;
    const double ae = gama - 1.0, af = 0.5 * ae * v2;
    const double a[5] = {ct, -nx, -ny, -nz, 0.0}, b[5] = {af, -ae * um, -ae * vm, -ae * wm, ae};
    const double N[5] = {0.0, nx, ny, nz, ct}, V[5] = {1.0, um, vm, wm, hm};
#pragma unroll
    for (int m = 0; m < 5; m++) { S.a[m] = a[m]; S.b[m] = b[m]; S.N[m] = N[m]; S.V[m] = V[m]; }
    return S;
}
__device__ __forceinline__ void split_apply(const Split &S, const double *y, double *f, bool transpose) {
    double p = 0.0, q = 0.0;  // A: a.y, b.y; A^T: N.y, V.y
#pragma unroll
    for (int m = 0; m < 5; m++) {
        p += (transpose ? S.N[m] : S.a[m]) * y[m];
        q += (transpose ? S.V[m] : S.b[m]) * y[m];
    }
    if (!transpose) {  // f = l1 y + N (x1 c2 a.y + x2 b.y) - V (x1 b.y + x2 a.y)
        const double cn = S.x1 * S.c2 * p + S.x2 * q, cv = S.x1 * q + S.x2 * p;
#pragma unroll
        for (int m = 0; m < 5; m++) f[m] = S.l1 * y[m] + S.N[m] * cn - S.V[m] * cv;
    } else {  // f = l1 y + a (x1 c2 N.y - x2 V.y) + b (x2 N.y - x1 V.y)
        const double ca = S.x1 * S.c2 * p - S.x2 * q, cb = S.x2 * p - S.x1 * q;
#pragma unroll
        for (int m = 0; m < 5; m++) f[m] = S.l1 * y[m] + S.a[m] * ca + S.b[m] * cb;
    }
}
__device__ __forceinline__ double coed_inv(const DevFields &F, long long id) {  // getcoed, inviscid
    return 1.0 / (1.0 / F.f[F_DTDT][id] + (F.f[F_SRA][id] + F.f[F_SRB][id] + F.f[F_SRC][id]));
}
}  // namespace

// one plane p = i+j+k of a sweep of the operator, every block:
// MODE 0 forward lower, 1 forward upper, 2 transposed upper (ascending),
// 3 transposed lower (descending); x and b five arrays `stride` apart
template <int MODE>
__global__ void __launch_bounds__(256) k_adj_lu(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, int p,
                                             double *x, const double *__restrict__ b, long long stride) {
    const DevBlock B = blocks[blockIdx.y];
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= B.nj * B.nk) return;
    const int j = col % B.nj + 1, k = col / B.nj + 1, i = p - j - k;
    if (i < 1 || i > B.ni) return;
    const long long id = gidx(B, i, j, k);
    const int c[3] = {i, j, k}, n[3] = {B.ni, B.nj, B.nk};
    const long long st[3] = {1, B.gx, (long long)B.gx * B.gy};
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, y[5], f[5];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const bool lower = MODE == 0 || MODE == 2;  // the neighbour below along d
        if (lower ? c[d] < 2 : c[d] > n[d] - 1) continue;
        const long long nid = lower ? id - st[d] : id + st[d];
        Split S;
        if (MODE == 0) S = split_at(P, F, nid, d, 1);        // A+_d at the neighbour
        else if (MODE == 1) S = split_at(P, F, nid, d, -1);  // A-_d at the neighbour
        else if (MODE == 2) S = split_at(P, F, id, d, -1);   // A-_d(p)^T
        else S = split_at(P, F, id, d, 1);                   // A+_d(p)^T
        const double w = MODE >= 2 ? coed_inv(F, nid) : 1.0;
#pragma unroll
        for (int m = 0; m < 5; m++) y[m] = w * x[m * stride + nid];
        split_apply(S, y, f, MODE >= 2);
#pragma unroll
        for (int m = 0; m < 5; m++) acc[m] += f[m];
    }
    const double ce = coed_inv(F, id);
#pragma unroll
    for (int m = 0; m < 5; m++) {
        double &xp = x[m * stride + id];
        if (MODE == 0) xp = (-b[m * stride + id] + acc[m]) * ce;
        else if (MODE == 1) xp = xp - acc[m] * ce;
        else if (MODE == 2) xp = b[m * stride + id] - acc[m];
        else xp = xp + acc[m];
    }
}

// pointwise over the interior: x = -coed x (the last factor of P^T), or
// x = (d prim / d Q)^T x + g (conserved adjoint of a prim-space adjoint)
template <int MODE>
__global__ void k_adj_point(DevParams P, DevFields F, const DevBlock *__restrict__ blocks, double *x,
                            const double *__restrict__ g, long long stride) {
    const DevBlock B = blocks[blockIdx.y];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_point(B, q, i, j, k);
        const long long id = gidx(B, i, j, k);
        double v[5];
#pragma unroll
        for (int m = 0; m < 5; m++) v[m] = x[m * stride + id];
        if (MODE == 0) {
            const double ce = coed_inv(F, id);
#pragma unroll
            for (int m = 0; m < 5; m++) x[m * stride + id] = -ce * v[m];
        } else {
            const double r = F.f[F_R][id], u = F.f[F_U][id], vv = F.f[F_V][id], w = F.f[F_W][id], g1 = P.gama - 1.0;
            const double ri = 1.0 / r;
            double o[5];
            o[0] = v[0] - (u * v[1] + vv * v[2] + w * v[3]) * ri + 0.5 * g1 * (u * u + vv * vv + w * w) * v[4];
            o[1] = v[1] * ri - g1 * u * v[4];
            o[2] = v[2] * ri - g1 * vv * v[4];
            o[3] = v[3] * ri - g1 * w * v[4];
            o[4] = g1 * v[4];
#pragma unroll
            for (int m = 0; m < 5; m++) x[m * stride + id] = o[m] + (g ? g[m * stride + id] : 0.0);
        }
    }
}

// interface ghosts are copies (ghost <- partner point): their adjoint moves
// to the partner point
__global__ void k_ghost_copy_adj(const GhostCopy *__restrict__ gc, long long n, double *x, long long stride) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const GhostCopy g = gc[e];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double a = x[m * stride + g.dst];
            if (a != 0.0) {
                atomicAdd(&x[m * stride + g.src], a);
                x[m * stride + g.dst] = 0.0;
            }
        }
    }
}


// x = 0 at the points of physical faces (whose dq the step zeroes before
// and after the sweeps, set_nonconnect_boundary_dq_0)
__global__ void k_adj_zero_pts(const long long *__restrict__ pts, long long n, double *x, long long stride) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int m = 0; m < 5; m++) x[m * stride + pts[e]] = 0.0;
}

void launch_adj_zero_faces(const LaunchCtx &c, double *x) {
    if (c.nzero > 0)
        k_adj_zero_pts<<<(unsigned)std::min<long long>((c.nzero + 255) / 256, 4096), 256, 0, c.stream>>>(c.zero_pts, c.nzero,
                                                                                                        x, c.total);
}

// y += x over the interior (a = 1), or the squared 2-norm of x over the
// interior into *out
template <int MODE>
__global__ void k_adj_reduce(const DevBlock *__restrict__ blocks, double *y, const double *__restrict__ x,
                             long long stride, double *out) {
    const DevBlock B = blocks[blockIdx.y];
    double s = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < B.npts; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_point(B, q, i, j, k);
        const long long id = gidx(B, i, j, k);
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double v = x[m * stride + id];
            if (MODE == 0) y[m * stride + id] += v;
            else s += v * v;
        }
    }
    if (MODE == 1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(out, s);
    }
}

// ---------------------------------------------------------------------------
// launches
// ---------------------------------------------------------------------------
static size_t adj_smem(const LaunchCtx &c, int dir) {
    int nmax = 0;
    for (int b = 0; b < c.nblocks; b++) nmax = std::max(nmax, dimof(c.hblocks[b], dir));
    return (size_t)c.inv[dir].nl_max * adj_line_stride(nmax) * sizeof(double);
}

void launch_rhs_invis_jvp(const LaunchCtx &c, const double *v, double *out) {
    for (int d = 0; d < 3; d++) {
        const DirTable &T = c.inv[d];
        if (!T.ngroups) continue;
        const size_t sm = adj_smem(c, d);
        if (d == 0) {
            cudaFuncSetAttribute(k_rhs_invis_jvp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_jvp<0><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, v, out, c.total);
        } else if (d == 1) {
            cudaFuncSetAttribute(k_rhs_invis_jvp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_jvp<1><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, v, out, c.total);
        } else {
            cudaFuncSetAttribute(k_rhs_invis_jvp<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_jvp<2><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, v, out, c.total);
        }
    }
}

void launch_rhs_invis_vjp(const LaunchCtx &c, const double *lam, double *out, bool fold) {
    for (int d = 0; d < 3; d++) {
        const DirTable &T = c.inv[d];
        if (!T.ngroups) continue;
        const size_t sm = adj_smem(c, d);
        if (d == 0) {
            cudaFuncSetAttribute(k_rhs_invis_vjp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_vjp<0><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, lam, out, c.total);
        } else if (d == 1) {
            cudaFuncSetAttribute(k_rhs_invis_vjp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_vjp<1><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, lam, out, c.total);
        } else {
            cudaFuncSetAttribute(k_rhs_invis_vjp<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_rhs_invis_vjp<2><<<T.ngroups, 256, sm, c.stream>>>(*c.P, *c.F, c.blocks, T.groups, lam, out, c.total);
        }
    }
    if (fold && c.nghost > 0)
        k_ghost_copy_adj<<<(unsigned)std::min<long long>((c.nghost + 255) / 256, 4096), 256, 0, c.stream>>>(c.ghost, c.nghost,
                                                                                                          out, c.total);
}

void launch_lusgs_operator(const LaunchCtx &c, double *x, const double *b, bool transpose) {
    int maxcols = 0, pmax = 0;
    long long maxp = 0;
    for (int q = 0; q < c.nblocks; q++) {
        const DevBlock &B = c.hblocks[q];
        maxcols = std::max(maxcols, B.nj * B.nk);
        pmax = std::max(pmax, B.ni + B.nj + B.nk);
        maxp = std::max(maxp, B.npts);
    }
    const dim3 grid((unsigned)((maxcols + 255) / 256), c.nblocks);
    if (!transpose) {
        for (int p = 3; p <= pmax; p++) k_adj_lu<0><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p, x, b, c.total);
        for (int p = pmax; p >= 3; p--) k_adj_lu<1><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p, x, b, c.total);
    } else {
        for (int p = 3; p <= pmax; p++) k_adj_lu<2><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p, x, b, c.total);
        for (int p = pmax; p >= 3; p--) k_adj_lu<3><<<grid, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, p, x, b, c.total);
        const dim3 pg((unsigned)std::min<long long>((maxp + 255) / 256, 4096), c.nblocks);
        k_adj_point<0><<<pg, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, x, nullptr, c.total);
    }
}

// x = (d prim / d Q)^T x + g over the interior
void launch_adj_to_conserved(const LaunchCtx &c, double *x, const double *g) {
    long long maxp = 0;
    for (int q = 0; q < c.nblocks; q++) maxp = std::max(maxp, c.hblocks[q].npts);
    const dim3 pg((unsigned)std::min<long long>((maxp + 255) / 256, 4096), c.nblocks);
    k_adj_point<1><<<pg, 256, 0, c.stream>>>(*c.P, *c.F, c.blocks, x, g, c.total);
}

// y += x (interior), or *out += |x|^2 (interior; out: device)
void launch_adj_axpy(const LaunchCtx &c, double *y, const double *x) {
    long long maxp = 0;
    for (int q = 0; q < c.nblocks; q++) maxp = std::max(maxp, c.hblocks[q].npts);
    const dim3 pg((unsigned)std::min<long long>((maxp + 255) / 256, 4096), c.nblocks);
    k_adj_reduce<0><<<pg, 256, 0, c.stream>>>(c.blocks, y, x, c.total, nullptr);
}
void launch_adj_norm2(const LaunchCtx &c, const double *x, double *out) {
    long long maxp = 0;
    for (int q = 0; q < c.nblocks; q++) maxp = std::max(maxp, c.hblocks[q].npts);
    const dim3 pg((unsigned)std::min<long long>((maxp + 255) / 256, 4096), c.nblocks);
    k_adj_reduce<1><<<pg, 256, 0, c.stream>>>(c.blocks, nullptr, x, c.total, out);
}

}  // namespace wcns
