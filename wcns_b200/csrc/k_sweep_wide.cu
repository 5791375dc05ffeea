// k_sweep_wide.cu -- GS_PR_Single (LHS.f90:1559-1613) for blocks too large
// for the clustered sweep kernel: lusgs_l (381-478), lusgs_u (480-577),
// gs_pr_l (1777-1866), gs_pr_u (1956-2046), one cooperative launch per
// sweep over all blocks of the context.
//
// Work split.  Each block's (j,k) columns are cut into chunks of whole
// j-rows (all k); one CTA owns a chunk, one thread a column, and the CTA
// walks the block's hyperplanes p = i+j+k in sweep order, the thread
// meeting its column's cell of each plane.  A cell's lower (forward) or
// upper (backward) neighbours are on the previous plane, so a cell can be
// computed once the contributions A*dq of those neighbours are known.  After
// computing its new dq a cell pushes the three contributions to its
// successors (the terms mxdq_std, 756-828, with the cell's own coefficients,
// exactly what the successor would evaluate from the cell's dq):
//   along i -- the same thread's next plane: kept in registers;
//   along k -- another thread of the CTA: shared memory, double-buffered
//              by plane parity, so one CTA barrier per plane suffices;
//   along j -- the next thread of the chunk, or, at the chunk's edge, the
//              neighbouring chunk's CTA: a ring of planes in global memory
//              with produced/consumed plane counters (release/acquire at
//              GPU scope, bounded waits).
// Every CTA of the launch is resident at once (cooperative launch), so the
// counters only wait on running CTAs; the ring's slack of planes hides the
// latency of the hop between SMs.
//
// Inputs are re-laid plane-major by k_wide_prep (once per step): for every
// cell the dq-independent split-Jacobian coefficients of both signs (from
// its prim, nine metrics and inviscid spectral radii), coed (getcoed,
// 602-645), the viscous radii, and rhs = dq (store_rhs_nb, 1592-1613); the
// cells of one chunk and plane are contiguous in every array, so a warp's
// loads are coalesced.  A thread issues its cell's loads at the top of the
// plane, before the plane barrier, off the dependency chain.  (Neither an L2
// prefetch of the next planes by one thread, nor per-thread prefetches, nor
// staging the words in shared memory with cp.async, one plane ahead or not,
// made the sweeps faster on the SA channel: all of them were slower.)
// lusgs_l stores its dq for lusgs_u; lusgs_u stores the
// terms it received from its upper neighbours -- evaluated with their final
// dq they are the old-side terms of gs_pr_l (der, dfr, dgr); gs_pr_l stores
// the sum of the terms it received from its lower neighbours, the old side of
// gs_pr_u ((del + dfl) + dgl, added first there).  gs_pr_u writes the result
// to the field layout.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "wcns_launch.h"

namespace wcns {

namespace {

// words per slot of the coefficient array: the direction-independent part of
// the split Jacobian (um, vm, wm, hm, c2, af), per direction the normalised
// metric and contravariant velocity (nx, ny, nz, ct), per direction and sign
// (npn = +1 forward, -1 backward) l1, x1, x2, then coed and the three
// viscous radii
enum : int { WS_SH = 0, WS_D = 6, WS_P = 18, WS_MN = 27, WS_COED = 36, WS_SRV = 37, WS_N = 40 };
static_assert(WS_N == WIDE_COEF_WORDS, "coefficient words per slot");
constexpr int WIDE_RING = 8;
constexpr int WIDE_PREFETCH = 3;  // planes prefetched into L2 ahead of the one being swept (SA sweep)
constexpr int PREP_DS = 4;        // planes per column that neighbouring lanes of a prep kernel take

// The chunk's slots t = (k-1)*w + jj (j = j0+jj+1) that hold a cell of plane
// p, i.e. 1 <= p-j-k <= ni: the first and last of them (the range between
// may include slots outside the block).  False when there is none.
__host__ __device__ __forceinline__ bool active_slots(int p, int j0, int w, int ni, int nk, int &lo, int &hi) {
    const int klo = max(1, p - ni - j0 - w), khi = min(nk, p - 2 - j0);
    if (klo > khi) return false;
    lo = (klo - 1) * w + max(0, p - ni - klo - j0 - 1);
    hi = (khi - 1) * w + min(w - 1, p - khi - j0 - 2);
    return lo <= hi;
}

struct Jsc {  // split-Jacobian coefficients of a cell along one direction (one sign)
    double nx, ny, nz, ct, l1, x1, x2;
};
struct Jsh {  // direction-independent part
    double um, vm, wm, hm, c2, af;
};

// the dq-dependent part of mxdq_std
__device__ __forceinline__ void jac_apply_w(double gama, const Jsh &H, const Jsc &J, const double *dq, double *f) {
    const double ae = gama - 1.0;
    const double dc = J.ct * dq[0] - J.nx * dq[1] - J.ny * dq[2] - J.nz * dq[3];
    const double dh = H.af * dq[0] - ae * (H.um * dq[1] + H.vm * dq[2] + H.wm * dq[3] - dq[4]);
    const double c2dc = H.c2 * dc;
    f[0] = J.l1 * dq[0] - dh * J.x1 - dc * J.x2;
    f[1] = J.l1 * dq[1] + (J.nx * c2dc - H.um * dh) * J.x1 + (J.nx * dh - H.um * dc) * J.x2;
    f[2] = J.l1 * dq[2] + (J.ny * c2dc - H.vm * dh) * J.x1 + (J.ny * dh - H.vm * dc) * J.x2;
    f[3] = J.l1 * dq[3] + (J.nz * c2dc - H.wm * dh) * J.x1 + (J.nz * dh - H.wm * dc) * J.x2;
    f[4] = J.l1 * dq[4] + (J.ct * c2dc - H.hm * dh) * J.x1 + (J.ct * dh - H.hm * dc) * J.x2;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned *p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// publishes every write that the CTA made before its last __syncthreads():
// the barrier orders the other threads' writes before this thread's fence,
// and fence.acq_rel.gpu followed by a relaxed store is a release pattern at
// GPU scope, cumulative over what the barrier ordered before it (a
// fence.sc.gpu, __threadfence(), costs about a microsecond more per plane)
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;\n" ::: "memory"); }
// waits until *p >= want; gives up after `limit` clock cycles.  `seen` is the
// largest count this thread has acquired from *p so far: a count it has
// already seen needs no new load (the acquire that saw it orders every
// later read of the entries it covers)
__device__ __forceinline__ bool wait_count(const unsigned *p, unsigned want, long long limit, unsigned &seen) {
    if (seen >= want) return true;
    const long long t0 = clock64();
    unsigned v;
    while ((v = ld_acquire(p)) < want)
        if (clock64() - t0 > limit) return false;
    seen = v;
    return true;
}
// bring [ptr, ptr + n doubles) into L2 (the range is widened to 16-byte
// boundaries; every array is padded so that the widening stays inside it)
__device__ __forceinline__ void prefetch_l2(const double *ptr, int n) {
    const unsigned long long a = (unsigned long long)ptr & ~15ull;
    const unsigned long long e = ((unsigned long long)(ptr + n) + 15ull) & ~15ull;
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

}  // namespace

// plane-major coefficients of every cell, evaluated once per step for all
// four sweeps: the dq-independent part of mxdq_std for the cell acting as a
// neighbour (getrkec_mml and getrarbrc return the cell's own metrics and
// spectral radius for interior cells) for both signs, coed (getcoed,
// 602-645), the viscous radii, and rhs = dq (set_nonconnect_boundary_dq_0
// has run, so rhs holds the zeros of the physical faces); one thread per
// slot, four CTAs of 256 threads per SM (64 registers: 0.95 ms per channel
// step, against 1.02 at two CTAs per SM and 1.18 at 108 registers)
__global__ void __launch_bounds__(256, 4) k_wide_prep(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                  const WideChunk *__restrict__ chunks, WideArrays A) {
    const WideChunk C = chunks[blockIdx.y];
    const DevBlock B = blocks[C.blk];
    const int ncolc = C.w * B.nk, np = B.ni + B.nj + B.nk - 2;
    const long long n = (long long)((np + PREP_DS - 1) / PREP_DS * PREP_DS) * ncolc;
    const double gama = P.gama;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        // PREP_DS consecutive planes of one column per group of lanes: their
        // cells are consecutive in i, so a group's gathers from the field
        // layout share sectors, while a plane's stores stay runs of columns
        const long long sb = e / ((long long)PREP_DS * ncolc);
        const int r = (int)(e - sb * PREP_DS * ncolc), t = r / PREP_DS;
        const int s = (int)sb * PREP_DS + (r - t * PREP_DS);
        if (s >= np) continue;
        const int p = s + 3, j = C.j0 + t % C.w + 1, k = t / C.w + 1, i = p - j - k;
        if (i < 1 || i > B.ni) continue;
        const long long id = gidx(B, i, j, k);
        const long long pm = C.pmoff + (long long)s * (B.nj * B.nk) + (long long)C.j0 * B.nk + t;
        double *o = A.stat + pm;
        const size_t N = (size_t)A.n;
        // the dq-independent part of mxdq_std (gettmhmgm_ns GasModel.f90:411-426,
        // nt = 0) from the prim, the nine metrics and the three inviscid
        // radii, each value stored as soon as it is known so that few are
        // live at a time
        const double rm = F.f[F_R][id], um = F.f[F_U][id], vm = F.f[F_V][id], wm = F.f[F_W][id], pres = F.f[F_P][id];
        const double nt = 0.0;
        const double hint = gama / (gama - 1.0) * pres / rm;
        const double c2 = gama * pres / rm;
        const double cm = sqrt(c2);
        const double v2 = um * um + vm * vm + wm * wm;
        const double ae = gama - 1.0;
        o[(WS_SH + 0) * N] = um;
        o[(WS_SH + 1) * N] = vm;
        o[(WS_SH + 2) * N] = wm;
        o[(WS_SH + 3) * N] = hint + 0.5 * v2;
        o[(WS_SH + 4) * N] = c2;
        o[(WS_SH + 5) * N] = 0.5 * ae * v2;
#pragma unroll 1
        for (int d = 0; d < 3; d++) {
            const double nx = F.f[F_KCX + 3 * d][id], ny = F.f[F_KCX + 3 * d + 1][id], nz = F.f[F_KCX + 3 * d + 2][id];
            const double rad = F.f[F_SRA + d][id];
            const double ct = nx * um + ny * vm + nz * wm + nt;
            double cgm = sqrt(nx * nx + ny * ny + nz * nz);
            if (!(cgm >= SML_SSS)) cgm = SML_SSS;
            const double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
#pragma unroll
            for (int sg = 0; sg < 2; sg++) {
                const double npn = sg == 0 ? 1.0 : -1.0;
                const double a1 = 0.5 * (l1 + npn * rad), a4 = 0.5 * (l4 + npn * rad), a5 = 0.5 * (l5 + npn * rad);
                const int w0 = sg == 0 ? WS_P : WS_MN;
                o[(w0 + 3 * d + 0) * N] = a1;
                o[(w0 + 3 * d + 1) * N] = (2.0 * a1 - a4 - a5) / (2.0 * c2);
                o[(w0 + 3 * d + 2) * N] = (a4 - a5) / (2.0 * cm);
            }
            const double cgm1 = 1.0 / cgm;
            o[(WS_D + 4 * d + 0) * N] = nx * cgm1;
            o[(WS_D + 4 * d + 1) * N] = ny * cgm1;
            o[(WS_D + 4 * d + 2) * N] = nz * cgm1;
            o[(WS_D + 4 * d + 3) * N] = (ct - nt) * cgm1;
        }
        // getcoed (LHS.f90:602-645), wmig = beta = 1, no dual time stepping
        double rad_ns = F.f[F_SRA][id] + F.f[F_SRB][id] + F.f[F_SRC][id];
        if (P.nvis >= 1) rad_ns = rad_ns + F.f[F_SRVA][id] + F.f[F_SRVB][id] + F.f[F_SRVC][id];
        const double ct = 1.0 / F.f[F_DTDT][id];
        o[WS_COED * N] = 1.0 / (ct + 1.0 * 1.0 * rad_ns);
#pragma unroll
        for (int m = 0; m < 3; m++) o[(WS_SRV + m) * N] = F.f[F_SRVA + m][id];
#pragma unroll
        for (int m = 0; m < 5; m++) A.rhs[(size_t)m * N + pm] = F.f[F_DQ1 + m][id];
    }
}

// MODE 0 lusgs_l, 1 lusgs_u, 2 gs_pr_l, 3 gs_pr_u
template <int MODE>
__global__ void __maxnreg__(WIDE_MAX_REGS) k_sweep_wide(DevParams P, DevFields F,
                                                                    const DevBlock *__restrict__ blocks,
                                                                    const WideChunk *__restrict__ chunks, WideArrays A,
                                                                    int *err) {
    constexpr bool FWD = MODE == 0 || MODE == 2;
    constexpr bool LU = MODE <= 1;
    constexpr int NC = LU ? 10 : 5;  // pushed values: A*dq (5) and, in lusgs, srv*dq (5)
    const WideChunk C = chunks[blockIdx.x];
    const DevBlock B = blocks[C.blk];
    const int t = threadIdx.x, ncolc = C.w * B.nk, ncol = B.nj * B.nk;
    const bool own = t < ncolc;
    const int jj = own ? t % C.w : 0;
    const int j = C.j0 + jj + 1, k = own ? t / C.w + 1 : 1;
    const int np = B.ni + B.nj + B.nk - 2;
    const bool vis = LU && P.nvis > 0;
    // ring roles: forward sweeps take j-contributions from the previous chunk
    // and give to the next one, backward sweeps the other way round
    const int rin = FWD ? C.bnd_lo : C.bnd_hi, rout = FWD ? C.bnd_hi : C.bnd_lo;
    // j-predecessor in this chunk (t -/+ 1), in the neighbouring chunk (ring), or none
    const bool jedge_in = FWD ? jj == 0 : jj == C.w - 1;
    const bool jedge_out = FWD ? jj == C.w - 1 : jj == 0;
    const bool hasj = FWD ? j > 1 : j < B.nj;
    const bool hask = FWD ? k > 1 : k < B.nk;
    extern __shared__ double smem[];
    // inbox[parity][dir 0 = j, 1 = k][column][NC], written by the producing column at its own index
    const size_t half = (size_t)2 * ncolc * NC;
    double *const ring_in = rin >= 0 ? A.ring + (size_t)rin * WIDE_RING * A.nkmax * 10 : nullptr;
    double *const ring_out = rout >= 0 ? A.ring + (size_t)rout * WIDE_RING * A.nkmax * 10 : nullptr;
    unsigned *const prod_in = rin >= 0 ? A.flags + 2 * rin : nullptr, *const cons_in = prod_in ? prod_in + 1 : nullptr;
    unsigned *const prod_out = rout >= 0 ? A.flags + 2 * rout : nullptr, *const cons_out = prod_out ? prod_out + 1 : nullptr;
    bool timed_out = false;
    auto limit = [&]() { return timed_out ? (1LL << 21) : (1LL << 31); };  // ~1 s for the first wait, then ~1 ms
    const double gama = P.gama;
    double ibuf[NC];  // contribution along i from this column's previous cell
#pragma unroll
    for (int m = 0; m < NC; m++) ibuf[m] = 0.0;
    const int pfirst = FWD ? 3 : B.ni + B.nj + B.nk;
    const int pstep = FWD ? 1 : -1;
    unsigned seen_prod = 0, seen_cons = 0;
    for (int s = 0; s < np; s++) {
        const int p = pfirst + s * pstep;
        const int i = p - j - k;
        const bool act = own && i >= 1 && i <= B.ni;
        const bool hasi = FWD ? i > 1 : i < B.ni;
        const long long pm = C.pmoff + (long long)(p - 3) * ncol + (long long)C.j0 * B.nk + t;
        // coefficients of this plane's cell, independent of the new values
        Jsh H;
        Jsc J[3];
        double base[5], coed = 0.0, rv[3] = {0.0, 0.0, 0.0};
        if (act) {
            const double *cf = A.stat + pm;
            const size_t N = (size_t)A.n;
            const int sg = FWD ? WS_P : WS_MN;
            H.um = cf[(WS_SH + 0) * N];
            H.vm = cf[(WS_SH + 1) * N];
            H.wm = cf[(WS_SH + 2) * N];
            H.hm = cf[(WS_SH + 3) * N];
            H.c2 = cf[(WS_SH + 4) * N];
            H.af = cf[(WS_SH + 5) * N];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                J[d].nx = cf[(WS_D + 4 * d + 0) * N];
                J[d].ny = cf[(WS_D + 4 * d + 1) * N];
                J[d].nz = cf[(WS_D + 4 * d + 2) * N];
                J[d].ct = cf[(WS_D + 4 * d + 3) * N];
                J[d].l1 = cf[(sg + 3 * d + 0) * N];
                J[d].x1 = cf[(sg + 3 * d + 1) * N];
                J[d].x2 = cf[(sg + 3 * d + 2) * N];
            }
            coed = cf[WS_COED * N];
            if (LU) {
#pragma unroll
                for (int d = 0; d < 3; d++) rv[d] = cf[(WS_SRV + d) * N];
            }
            const double *bsrc = MODE == 1 ? A.dql : A.rhs;
#pragma unroll
            for (int m = 0; m < 5; m++) base[m] = bsrc[(size_t)m * A.n + pm];
        }
        if (t == 0) {
            if (ring_in && s > 0 && !wait_count(prod_in, (unsigned)s, limit(), seen_prod)) timed_out = true;
            if (ring_out && s >= WIDE_RING && !wait_count(cons_out, (unsigned)(s - WIDE_RING + 1), limit(), seen_cons))
                timed_out = true;
        }
        __syncthreads();  // the previous plane's inbox and ring entries are complete
        // the counters move at every second plane: half the fences on thread
        // 0's path, and a consumer that sees two planes per acquire, for one
        // more plane of lag per chunk boundary (3.76 -> 3.56 ms for the four
        // sweeps of the SA channel; every third plane is no better)
        if (t == 0 && (ring_out || ring_in) && (s & 1) == 0) {
            fence_acq_rel_gpu();
            if (ring_out && s > 0) st_relaxed(prod_out, (unsigned)s);      // planes 0..s-1 published
            if (ring_in && s > 1) st_relaxed(cons_in, (unsigned)(s - 1));  // planes 0..s-2 read
        }
        if (!act) continue;
        const double *rd = smem + (size_t)((s + 1) & 1) * half;
        double *wr = smem + (size_t)(s & 1) * half;
        // contributions of the three neighbours on the previous plane (zero
        // outside the block: the reference's ghost dq is zero)
        double cj[NC], ck[NC];
        if (hasj) {
            if (jedge_in) {
                const double *r = ring_in + ((size_t)((s - 1) % WIDE_RING) * A.nkmax + (k - 1)) * 10;
#pragma unroll
                for (int m = 0; m < NC; m++) cj[m] = __ldcg(r + m);
            } else {
                const double *r = rd + (size_t)(FWD ? t - 1 : t + 1) * NC;
#pragma unroll
                for (int m = 0; m < NC; m++) cj[m] = r[m];
            }
        } else {
#pragma unroll
            for (int m = 0; m < NC; m++) cj[m] = 0.0;
        }
        if (hask) {
            const double *r = rd + (size_t)ncolc * NC + (size_t)(FWD ? t - C.w : t + C.w) * NC;
#pragma unroll
            for (int m = 0; m < NC; m++) ck[m] = r[m];
        } else {
#pragma unroll
            for (int m = 0; m < NC; m++) ck[m] = 0.0;
        }
        if (!hasi) {
#pragma unroll
            for (int m = 0; m < NC; m++) ibuf[m] = 0.0;
        }
        double nw[5];
        if (LU) {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                double r0 = 1.0 * (ibuf[m] + cj[m] + ck[m]);
                if (vis) {
                    const double v = 0.5 * (ibuf[5 + m] + cj[5 + m] + ck[5 + m]);
                    r0 = MODE == 0 ? r0 + v : r0 - v;
                }
                nw[m] = MODE == 0 ? (-base[m] + r0) * coed : base[m] - r0 * coed;
            }
            if (MODE == 0) {
#pragma unroll
                for (int m = 0; m < 5; m++) A.dql[(size_t)m * A.n + pm] = nw[m];
            } else {
                // der, dfr, dgr of gs_pr_l: the upper neighbours' terms with their final dq
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    A.gs1[(size_t)m * A.n + pm] = ibuf[m];
                    A.gs1[(size_t)(5 + m) * A.n + pm] = cj[m];
                    A.gs1[(size_t)(10 + m) * A.n + pm] = ck[m];
                }
            }
        } else if (MODE == 2) {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                const double der = A.gs1[(size_t)m * A.n + pm], dfr = A.gs1[(size_t)(5 + m) * A.n + pm],
                             dgr = A.gs1[(size_t)(10 + m) * A.n + pm];
                const double lo = ibuf[m] + cj[m] + ck[m];
                A.gs2[(size_t)m * A.n + pm] = lo;  // (del + dfl) + dgl for gs_pr_u
                const double r0 = 1.0 * (lo - der - dfr - dgr);
                nw[m] = (r0 - base[m]) * coed;
            }
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                const double lo = A.gs2[(size_t)m * A.n + pm];
                const double r0 = 1.0 * (lo - ibuf[m] - cj[m] - ck[m]);
                nw[m] = (r0 - base[m]) * coed;
            }
            const long long id = gidx(B, i, j, k);
#pragma unroll
            for (int m = 0; m < 5; m++) F.f[F_DQ1 + m][id] = nw[m];
        }
        // the three contributions for the successors on the next plane
        {
            double o[3][NC];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                jac_apply_w(gama, H, J[d], nw, o[d]);
                if (LU) {
#pragma unroll
                    for (int m = 0; m < 5; m++) o[d][5 + m] = rv[d] * nw[m];
                }
            }
#pragma unroll
            for (int m = 0; m < NC; m++) ibuf[m] = o[0][m];
            double *wj = wr + (size_t)t * NC, *wk = wr + (size_t)ncolc * NC + (size_t)t * NC;
#pragma unroll
            for (int m = 0; m < NC; m++) {
                wj[m] = o[1][m];
                wk[m] = o[2][m];
            }
            if (jedge_out && ring_out) {
                double *r = ring_out + ((size_t)(s % WIDE_RING) * A.nkmax + (k - 1)) * 10;
#pragma unroll
                for (int m = 0; m < NC; m++) __stcg(r + m, o[1][m]);
            }
        }
    }
    __syncthreads();
    if (t == 0) {
        fence_acq_rel_gpu();
        if (ring_out) st_relaxed(prod_out, (unsigned)np);
        if (ring_in) st_relaxed(cons_in, (unsigned)np);
        if (timed_out) atomicAdd(&err[ERR_TIMEOUT], 1);
    }
}

size_t wide_smem_bytes(int ncolc, int nc) { return (size_t)2 * 2 * ncolc * nc * sizeof(double); }

// Chunking: columns per CTA near (all columns) / (CTAs the device holds at
// once), whole j-rows per chunk, at most WIDE_MAX_THREADS columns.
// Returns -1 when the blocks cannot be swept this way.
int setup_sweep_wide(LaunchCtx &c, WideSweep &W) {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long cols = 0;
    int nkmax = 0;
    for (int b = 0; b < c.nblocks; b++) {
        cols += (long long)c.hblocks[b].nj * c.hblocks[b].nk;
        nkmax = std::max(nkmax, c.hblocks[b].nk);
    }
    if (nkmax > WIDE_MAX_THREADS) return -1;
    int min_cols = 128;
    if (const char *e = getenv("WCNS_WIDE_MIN_COLS")) min_cols = std::max(1, atoi(e));  // tests: narrow chunks
    // columns per chunk: start from an even share of the SMs and widen the
    // chunks until every CTA of the launch fits on the device at once
    for (long long target = std::max<long long>(1, (cols + nsm - 1) / nsm);; target = target + target / 25 + 1) {
        std::vector<WideChunk> ch;
        std::vector<long long> pmoff(c.nblocks);
        long long n = 0;
        int nbnd = 0, maxcols = 0;
        for (int b = 0; b < c.nblocks; b++) {
            const DevBlock &B = c.hblocks[b];
            int w = (int)std::max<long long>(1, std::min<long long>(target / B.nk, WIDE_MAX_THREADS / B.nk));
            // at least min_cols columns per chunk: every chunk edge adds a hop between SMs per plane
            w = std::max(w, std::min((min_cols + B.nk - 1) / B.nk, WIDE_MAX_THREADS / B.nk));
            w = std::max(1, std::min(w, B.nj));
            const int G = (B.nj + w - 1) / w;
            pmoff[b] = n;
            n += (long long)(B.ni + B.nj + B.nk - 2) * B.nj * B.nk;
            n = (n + 1) / 2 * 2;
            for (int q = 0; q < G; q++) {
                WideChunk C{};
                C.blk = b;
                C.j0 = q * B.nj / G;
                C.w = (q + 1) * B.nj / G - C.j0;
                C.pmoff = pmoff[b];
                C.bnd_lo = q > 0 ? nbnd + q - 1 : -1;
                C.bnd_hi = q < G - 1 ? nbnd + q : -1;
                ch.push_back(C);
                maxcols = std::max(maxcols, C.w * B.nk);
            }
            nbnd += G - 1;
        }
        const int threads = (maxcols + 31) / 32 * 32;
        const size_t smem = wide_smem_bytes(maxcols, 10);
        const bool verbose = getenv("WCNS_VERBOSE") != nullptr;
        if (threads > WIDE_MAX_THREADS || smem > 227 * 1024) {
            if (verbose) fprintf(stderr, "wide sweeps: %d threads, %zu bytes of shared memory per CTA do not fit\n", threads, smem);
            return -1;
        }
        int per_sm = 0;
        cudaFuncSetAttribute(k_sweep_wide<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_sweep_wide<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_sweep_wide<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_sweep_wide<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_wide<0>, threads, smem);
        if (oe != cudaSuccess) {
            if (verbose) fprintf(stderr, "wide sweeps: occupancy query failed: %s\n", cudaGetErrorString(oe));
            cudaGetLastError();
            return -1;
        }
        if (verbose)
            fprintf(stderr, "wide sweeps: %zu chunks, %d threads, %zu bytes of shared memory, %d CTAs per SM on %d SMs\n",
                    ch.size(), threads, smem, per_sm, nsm);
        if ((long long)per_sm * nsm < (long long)ch.size()) {
            if (threads >= WIDE_MAX_THREADS) return -1;
            continue;
        }
        W.nchunks = (int)ch.size();
        W.threads = threads;
        W.smem_lu = smem;
        W.smem_gs = wide_smem_bytes(maxcols, 5);
        W.hchunks = ch;
        W.A.n = n;
        W.A.nkmax = nkmax;
        W.A.nbnd = nbnd;
        return 0;
    }
}

// every CTA resident at once: a cooperative launch (capturable in the step graph)
template <int MODE>
static void launch_wide_t(const LaunchCtx &c) {
    const WideSweep &W = *c.wide;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(W.nchunks, 1, 1);
    cfg.blockDim = dim3(W.threads, 1, 1);
    cfg.dynamicSmemBytes = MODE <= 1 ? W.smem_lu : W.smem_gs;
    cfg.stream = c.stream;
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_sweep_wide<MODE>, *c.P, *c.F, (const DevBlock *)c.blocks, (const WideChunk *)W.chunks, W.A,
                       c.err);
}

int launch_sweeps_wide(const LaunchCtx &c) {
    const WideSweep &W = *c.wide;
    int maxslots = 0;
    for (const WideChunk &C : W.hchunks) {
        const DevBlock &B = c.hblocks[C.blk];
        maxslots = std::max(maxslots, (B.ni + B.nj + B.nk - 2) * C.w * B.nk);
    }
    k_wide_prep<<<dim3((unsigned)std::min(4096, (maxslots + 255) / 256), W.nchunks), 256, 0, c.stream>>>(
        *c.P, *c.F, c.blocks, W.chunks, W.A);
    prof_mark(c, "lhs_prep");
    int n = 1;
    const size_t fbytes = sizeof(unsigned) * 2 * (size_t)std::max(1, W.A.nbnd);
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_wide_t<0>(c);
    prof_mark(c, "sweep_lusgs_l");
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_wide_t<1>(c);
    prof_mark(c, "sweep_lusgs_u");
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_wide_t<2>(c);
    prof_mark(c, "sweep_gs_pr_l");
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_wide_t<3>(c);
    prof_mark(c, "sweep_gs_pr_u");
    return n + 4;
}


// ---------------------------------------------------------------------------
// lusgs_turbulence (turblence.f90:477-558) on the same chunks: the SA model's
// scalar forward and backward sweeps over the points 2..n-1 of every
// direction.  A point's term for a successor is mxdq_std_turbulence
// (560-583) of the point itself: 0.5*(l + npn*|l|)*dqke with l the
// contravariant velocity along the direction, so the prep keeps l for the
// three directions, spec and the right-hand side per slot.

// sa words per slot: l along i, j, k; spec; dqke (right-hand side); the forward result
enum : int { WSA_L = 0, WSA_SPEC = 3, WSA_RHS = 4, WSA_FWD = 5, WSA_N = 6 };

__global__ void __launch_bounds__(256) k_sa_wide_prep(DevFields F, SaFields S, const DevBlock *__restrict__ blocks,
                                                     const WideChunk *__restrict__ chunks, WideArrays A) {
    const WideChunk C = chunks[blockIdx.y];
    const DevBlock B = blocks[C.blk];
    const int ncolc = C.w * B.nk, np = B.ni + B.nj + B.nk - 2;
    const long long n = (long long)((np + PREP_DS - 1) / PREP_DS * PREP_DS) * ncolc;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        // PREP_DS consecutive planes of one column per group of lanes: their
        // cells are consecutive in i, so a group's gathers from the field
        // layout share sectors, while a plane's stores stay runs of columns
        const long long sb = e / ((long long)PREP_DS * ncolc);
        const int r = (int)(e - sb * PREP_DS * ncolc), t = r / PREP_DS;
        const int s = (int)sb * PREP_DS + (r - t * PREP_DS);
        if (s >= np) continue;
        const int p = s + 3, j = C.j0 + t % C.w + 1, k = t / C.w + 1, i = p - j - k;
        if (i < 2 || i > B.ni - 1 || j < 2 || j > B.nj - 1 || k < 2 || k > B.nk - 1) continue;
        const long long id = gidx(B, i, j, k);
        const long long pm = C.pmoff + (long long)s * (B.nj * B.nk) + (long long)C.j0 * B.nk + t;
        const double u = F.f[F_U][id], v = F.f[F_V][id], w = F.f[F_W][id];
#pragma unroll
        for (int d = 0; d < 3; d++)
            A.sa[(size_t)(WSA_L + d) * A.n + pm] =
                F.f[F_KCX + 3 * d][id] * u + F.f[F_KCX + 3 * d + 1][id] * v + F.f[F_KCX + 3 * d + 2][id] * w;
        A.sa[(size_t)WSA_SPEC * A.n + pm] = S.spec[id];
        A.sa[(size_t)WSA_RHS * A.n + pm] = S.dqke[id];
    }
}

template <bool FWD>
__global__ void __launch_bounds__(WIDE_MAX_THREADS, 1) k_sa_sweep_wide(SaFields S, const DevBlock *__restrict__ blocks,
                                                                       const WideChunk *__restrict__ chunks,
                                                                       WideArrays A, int *err) {
    const double npn = FWD ? 1.0 : -1.0;
    const WideChunk C = chunks[blockIdx.x];
    const DevBlock B = blocks[C.blk];
    const int t = threadIdx.x, ncolc = C.w * B.nk, ncol = B.nj * B.nk;
    const bool own = t < ncolc;
    // the thread that waits on and publishes the ring counters: an idle lane
    // when the CTA has one, so that no column's cell waits behind it (this
    // scalar sweep gains 11 % on the SA channel; the mean-flow sweeps, whose
    // idle lanes share a warp with busy ones, do not, and keep thread 0)
    const int tc = ncolc < (int)blockDim.x ? (int)blockDim.x - 1 : 0;
    const int jj = own ? t % C.w : 0;
    const int j = C.j0 + jj + 1, k = own ? t / C.w + 1 : 1;
    const bool colin = own && j >= 2 && j <= B.nj - 1 && k >= 2 && k <= B.nk - 1;
    const int np = B.ni + B.nj + B.nk - 2;
    const int rin = FWD ? C.bnd_lo : C.bnd_hi, rout = FWD ? C.bnd_hi : C.bnd_lo;
    const bool jedge_in = FWD ? jj == 0 : jj == C.w - 1;
    const bool jedge_out = FWD ? jj == C.w - 1 : jj == 0;
    // a predecessor outside 2..n-1 contributes zero (its dqke is zero)
    const bool hasj = FWD ? j > 2 : j < B.nj - 1;
    const bool hask = FWD ? k > 2 : k < B.nk - 1;
    __shared__ double inbox[2][2][WIDE_MAX_THREADS];
    double *const ring_in = rin >= 0 ? A.ring + (size_t)rin * WIDE_RING * A.nkmax * 10 : nullptr;
    double *const ring_out = rout >= 0 ? A.ring + (size_t)rout * WIDE_RING * A.nkmax * 10 : nullptr;
    unsigned *const prod_in = rin >= 0 ? A.flags + 2 * rin : nullptr, *const cons_in = prod_in ? prod_in + 1 : nullptr;
    unsigned *const prod_out = rout >= 0 ? A.flags + 2 * rout : nullptr, *const cons_out = prod_out ? prod_out + 1 : nullptr;
    bool timed_out = false;
    auto limit = [&]() { return timed_out ? (1LL << 21) : (1LL << 31); };
    double ibuf = 0.0;
    const int pfirst = FWD ? 3 : B.ni + B.nj + B.nk, pstep = FWD ? 1 : -1;
    const int pwarp = blockDim.x > 32 ? 32 : 0;
    const int plane_lane = t - pwarp;
    auto prefetch_plane = [&](int s) {  // one word array per lane of the prefetch warp
        if (s >= np || plane_lane < 0 || plane_lane >= WSA_N) return;
        const int p = pfirst + s * pstep;
        int lo, hi;
        if (!active_slots(p, C.j0, C.w, B.ni, B.nk, lo, hi)) return;
        const long long pm0 = C.pmoff + (long long)(p - 3) * ncol + (long long)C.j0 * B.nk + lo;
        prefetch_l2(A.sa + (size_t)plane_lane * A.n + pm0, hi - lo + 1);
    };
    for (int a = 0; a < WIDE_PREFETCH; a++) prefetch_plane(a);
    unsigned seen_prod = 0, seen_cons = 0;
    for (int s = 0; s < np; s++) {
        const int p = pfirst + s * pstep;
        const int i = p - j - k;
        const bool act = colin && i >= 2 && i <= B.ni - 1;
        const bool hasi = FWD ? i > 2 : i < B.ni - 1;
        const long long pm = C.pmoff + (long long)(p - 3) * ncol + (long long)C.j0 * B.nk + t;
        double l[3] = {0.0, 0.0, 0.0}, spec = 1.0, base = 0.0;
        if (act) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double ct = A.sa[(size_t)(WSA_L + d) * A.n + pm];
                l[d] = 0.5 * (ct + npn * fabs(ct));
            }
            spec = A.sa[(size_t)WSA_SPEC * A.n + pm];
            base = A.sa[(size_t)(FWD ? WSA_RHS : WSA_FWD) * A.n + pm];
        }
        prefetch_plane(s + WIDE_PREFETCH);
        if (t == tc) {
            if (ring_in && s > 0 && !wait_count(prod_in, (unsigned)s, limit(), seen_prod)) timed_out = true;
            if (ring_out && s >= WIDE_RING && !wait_count(cons_out, (unsigned)(s - WIDE_RING + 1), limit(), seen_cons))
                timed_out = true;
        }
        __syncthreads();
        if (t == tc && (ring_out || ring_in) && (s & 1) == 0) {  // every second plane, as in the mean-flow sweeps
            fence_acq_rel_gpu();
            if (ring_out && s > 0) st_relaxed(prod_out, (unsigned)s);
            if (ring_in && s > 1) st_relaxed(cons_in, (unsigned)(s - 1));
        }
        if (!act) continue;
        const int rp = (s + 1) & 1, wp = s & 1;
        const double ti = hasi ? ibuf : 0.0;
        double tj = 0.0, tk = 0.0;
        if (hasj) {
            if (jedge_in) tj = __ldcg(ring_in + ((size_t)((s - 1) % WIDE_RING) * A.nkmax + (k - 1)) * 10);
            else tj = inbox[rp][0][FWD ? t - 1 : t + 1];
        }
        if (hask) tk = inbox[rp][1][FWD ? t - C.w : t + C.w];
        const double rhs0 = ti + tj + tk;
        const double nw = FWD ? (rhs0 - base) / spec : base - rhs0 / spec;
        if (FWD) A.sa[(size_t)WSA_FWD * A.n + pm] = nw;
        else S.dqke[gidx(B, i, j, k)] = nw;
        ibuf = l[0] * nw;
        inbox[wp][0][t] = l[1] * nw;
        inbox[wp][1][t] = l[2] * nw;
        if (jedge_out && ring_out) __stcg(ring_out + ((size_t)(s % WIDE_RING) * A.nkmax + (k - 1)) * 10, l[1] * nw);
    }
    __syncthreads();
    if (t == tc) {
        fence_acq_rel_gpu();
        if (ring_out) st_relaxed(prod_out, (unsigned)np);
        if (ring_in) st_relaxed(cons_in, (unsigned)np);
        if (timed_out) atomicAdd(&err[ERR_TIMEOUT], 1);
    }
}

template <bool FWD>
static void launch_sa_wide_t(const LaunchCtx &c) {
    const WideSweep &W = *c.wide;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(W.nchunks, 1, 1);
    cfg.blockDim = dim3(W.threads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.stream;
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_sa_sweep_wide<FWD>, *c.SA, (const DevBlock *)c.blocks, (const WideChunk *)W.chunks, W.A,
                       c.err);
}

// the SA model's scalar LU-SGS on the wide chunks; returns the number of launches
int launch_sa_lusgs_wide(const LaunchCtx &c) {
    const WideSweep &W = *c.wide;
    int maxslots = 0;
    for (const WideChunk &C : W.hchunks) {
        const DevBlock &B = c.hblocks[C.blk];
        maxslots = std::max(maxslots, (B.ni + B.nj + B.nk - 2) * C.w * B.nk);
    }
    k_sa_wide_prep<<<dim3((unsigned)std::min(4096, (maxslots + 255) / 256), W.nchunks), 256, 0, c.stream>>>(
        *c.F, *c.SA, c.blocks, W.chunks, W.A);
    const size_t fbytes = sizeof(unsigned) * 2 * (size_t)std::max(1, W.A.nbnd);
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_sa_wide_t<true>(c);
    cudaMemsetAsync(W.A.flags, 0, fbytes, c.stream);
    launch_sa_wide_t<false>(c);
    return 3;
}

}  // namespace wcns
