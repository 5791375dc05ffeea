// k_lhs.cu -- implicit update: l_h_s_tgh (LHS.f90:1-34) -> GS_PR_Single
// (LHS.f90:1559-1587): lusgs_l (381-478), lusgs_u (480-577), gs_pr_l
// (1777-1866), gs_pr_u (1956-2046), each point update using getcoed
// (602-645), getrarbrc (647-678), getrkec_mml (Sub1.f90:676-717) and
// mxdq_std (LHS.f90:756-828); set_nonconnect_boundary_dq_0 (CIC.f90:2-17)
// before and after.
//
// The reference sweeps each block lexicographically.  A point reads only
// lower neighbours (already updated in the sweep) and upper neighbours (not
// yet updated), so walking the hyperplanes i+j+k = p in order reproduces the
// sequential result exactly.
//
// Work split:
//   k_lhs_prep   (all cells in parallel) evaluates everything that does not
//                depend on dq -- the coefficients of mxdq_std for the cell
//                acting as a neighbour (both signs, three directions), coed,
//                the viscous radii -- and rhs = dq (store_rhs_nb), as one
//                packed 368-byte record per cell in plane-major order.
//   k_gs_old     (all cells in parallel) the Gauss-Seidel terms of the side
//                that holds the previous sweep's values.
//   k_sweep      one thread-block cluster per grid block (the reference's
//                LU-SGS is block-Jacobi, so blocks are independent).  CTA q
//                of the cluster owns a j-chunk of the block's (j,k) columns,
//                a thread owns one column and meets its cell once per plane.
//                The records of a CTA's cells of one plane are contiguous, so
//                one bulk copy (three planes ahead, mbarrier completion)
//                stages them.  After computing its new dq a cell pushes its
//                contributions A*dq to the next plane: the own (i) column
//                keeps it in registers, the j and k successors receive it in
//                their CTA's shared-memory inbox (a distributed-shared-memory
//                store when the successor is in another CTA).  One cluster
//                barrier per plane orders producers and consumers.
#include <algorithm>
#include <cooperative_groups.h>

#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace cg = cooperative_groups;

namespace wcns {

__global__ void k_zero_faces(DevFields F, const long long *__restrict__ pts, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        long long id = pts[e];
#pragma unroll
        for (int m = 0; m < 5; m++) F.f[F_DQ1 + m][id] = 0.0;
    }
}

// mxdq_std (LHS.f90:756-828) split into dq-independent coefficients
// (k_lhs_prep) and the linear map applied to dq (jac_apply); operations and
// their order are those of the reference routine.
struct Jac {
    double l1, x1, x2, ct, nx, ny, nz, af, um, vm, wm, c2, hm;
};

__device__ __forceinline__ void jac_apply(const DevParams &P, const Jac &J, const double *dq, double *f) {
    const double ae = P.gama - 1.0;
    double dc = J.ct * dq[0] - J.nx * dq[1] - J.ny * dq[2] - J.nz * dq[3];
    double dh = J.af * dq[0] - ae * (J.um * dq[1] + J.vm * dq[2] + J.wm * dq[3] - dq[4]);
    double c2dc = J.c2 * dc;
    f[0] = J.l1 * dq[0] - dh * J.x1 - dc * J.x2;
    f[1] = J.l1 * dq[1] + (J.nx * c2dc - J.um * dh) * J.x1 + (J.nx * dh - J.um * dc) * J.x2;
    f[2] = J.l1 * dq[2] + (J.ny * c2dc - J.vm * dh) * J.x1 + (J.ny * dh - J.vm * dc) * J.x2;
    f[3] = J.l1 * dq[3] + (J.nz * c2dc - J.wm * dh) * J.x1 + (J.nz * dh - J.wm * dc) * J.x2;
    f[4] = J.l1 * dq[4] + (J.ct * c2dc - J.hm * dh) * J.x1 + (J.ct * dh - J.hm * dc) * J.x2;
}

// split Jacobian of a record acting as neighbour along d, sign s (0: npn=+1, 1: npn=-1)
__device__ __forceinline__ Jac rec_jac(const double *R, int d, int s) {
    Jac J;
    J.um = R[SR_JS + 0];
    J.vm = R[SR_JS + 1];
    J.wm = R[SR_JS + 2];
    J.c2 = R[SR_JS + 3];
    J.hm = R[SR_JS + 4];
    J.af = R[SR_JS + 5];
    J.ct = R[SR_JD + 4 * d + 0];
    J.nx = R[SR_JD + 4 * d + 1];
    J.ny = R[SR_JD + 4 * d + 2];
    J.nz = R[SR_JD + 4 * d + 3];
    const int b = (s == 0 ? SR_JP : SR_JM) + 3 * d;
    J.l1 = R[b + 0];
    J.x1 = R[b + 1];
    J.x2 = R[b + 2];
    return J;
}

__host__ __device__ inline long long pm_size(const DevBlock &B) { return (long long)(B.ni + B.nj + B.nk - 2) * B.nj * B.nk; }

// plane-major index q (relative to the block) -> cell (i,j,k); false when
// the slot lies outside the block.  Inverts col_slot: the chunk is the last
// one whose first slot is <= the slot (never an empty chunk).
__device__ __forceinline__ bool pm_cell(const DevBlock &B, int C, long long q, int &i, int &j, int &k) {
    const int ncol = B.nj * B.nk;
    const int p = (int)(q / ncol) + 3;
    const int slot = (int)(q % ncol);
    int lo = 0, hi = C - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (chunk_j0(mid, B.nj, C) * B.nk <= slot) lo = mid;
        else hi = mid - 1;
    }
    const int j0 = chunk_j0(lo, B.nj, C), w = chunk_j0(lo + 1, B.nj, C) - j0;
    const int lc = slot - j0 * B.nk;
    k = lc / w + 1;
    j = j0 + lc % w + 1;
    i = p - j - k;
    return i >= 1 && i <= B.ni;
}

// ---------------------------------------------------------------------------
// prep: for interior neighbours getrkec_mml/getrarbrc return the neighbour's
// own metrics and spectral radius, so the coefficients depend on the
// neighbour cell only and are evaluated once per cell.
__global__ void k_lhs_prep(DevParams P, DevFields F, PmFields M, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    const double gama = P.gama;
    const long long nq = pm_size(B);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!pm_cell(B, M.csize, q, i, j, k)) continue;
        const long long id = gidx(B, i, j, k);
        const long long pm = B.pmoff + q;
        double *R = M.stat + pm * SR_N;
        double rm = F.f[F_R][id], um = F.f[F_U][id], vm = F.f[F_V][id], wm = F.f[F_W][id], pmr = F.f[F_P][id];
        double hint = P.g1 * pmr / rm;
        double c2 = gama * pmr / rm;
        double cm = sqrt(c2);
        double v2 = um * um + vm * vm + wm * wm;
        double hm = hint + 0.5 * v2;
        double ae = gama - 1.0;
        R[SR_COED] = F.f[F_COED][id];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double v = F.f[F_DQ1 + m][id];
            R[SR_RHS + m] = v;  // store_rhs_nb (LHS.f90:1592-1613)
            M.dq[m][pm] = v;
        }
        R[SR_JS + 0] = um;
        R[SR_JS + 1] = vm;
        R[SR_JS + 2] = wm;
        R[SR_JS + 3] = c2;
        R[SR_JS + 4] = hm;
        R[SR_JS + 5] = 0.5 * ae * v2;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double nx = F.f[F_KCX + 3 * d][id], ny = F.f[F_KCX + 3 * d + 1][id], nz = F.f[F_KCX + 3 * d + 2][id], nt = 0.0;
            double rad = F.f[F_SRA + d][id];
            double ct = nx * um + ny * vm + nz * wm + nt;
            double cgm = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
            double cgm1 = 1.0 / cgm;
            R[SR_JD + 4 * d + 0] = (ct - nt) * cgm1;
            R[SR_JD + 4 * d + 1] = nx * cgm1;
            R[SR_JD + 4 * d + 2] = ny * cgm1;
            R[SR_JD + 4 * d + 3] = nz * cgm1;
#pragma unroll
            for (int sg = 0; sg < 2; sg++) {
                double dn = sg == 0 ? 1.0 : -1.0;
                double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
                l1 = 0.5 * (l1 + dn * rad);
                l4 = 0.5 * (l4 + dn * rad);
                l5 = 0.5 * (l5 + dn * rad);
                const int b = (sg == 0 ? SR_JP : SR_JM) + 3 * d;
                R[b + 0] = l1;
                R[b + 1] = (2.0 * l1 - l4 - l5) / (2.0 * c2);
                R[b + 2] = (l4 - l5) / (2.0 * cm);
            }
        }
        R[SR_SRV + 0] = F.f[F_SRVA][id];
        R[SR_SRV + 1] = F.f[F_SRVB][id];
        R[SR_SRV + 2] = F.f[F_SRVC][id];
        R[SR_N - 1] = 0.0;
    }
}

// Gauss-Seidel side holding the previous sweep's values, for all cells:
// MODE 2 (gs_pr_l) needs the three upper terms der, dfr, dgr separately;
// MODE 3 (gs_pr_u) needs the lower prefix (del + dfl) + dgl.  A neighbour
// outside the block has dq = 0 and contributes nothing.
template <int MODE>
__global__ void k_gs_old(DevParams P, PmFields M, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    const int C = M.csize;
    const long long nq = pm_size(B);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!pm_cell(B, C, q, i, j, k)) continue;
        const int p = i + j + k;
        const int cc[3] = {i, j, k}, dims[3] = {B.ni, B.nj, B.nk};
        constexpr int e = MODE == 2 ? 1 : -1;
        double term[3][5];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const bool inside = MODE == 2 ? cc[d] < dims[d] : cc[d] > 1;
            if (!inside) {
#pragma unroll
                for (int m = 0; m < 5; m++) term[d][m] = 0.0;
                continue;
            }
            const int jn = d == 1 ? j + e : j, kn = d == 2 ? k + e : k;
            const long long npm = pmidx(B, p + e, col_slot(jn, kn, B.nj, B.nk, C));
            double dn[5];
#pragma unroll
            for (int m = 0; m < 5; m++) dn[m] = M.dq[m][npm];
            Jac J = rec_jac(M.stat + npm * SR_N, d, MODE == 2 ? 1 : 0);
            jac_apply(P, J, dn, term[d]);
        }
        double *D = M.dyn + (B.pmoff + q) * DYN_N;
        if (MODE == 2) {
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int m = 0; m < 5; m++) D[5 * d + m] = term[d][m];
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) D[m] = term[0][m] + term[1][m] + term[2][m];
        }
    }
}

__global__ void k_pm_to_std(DevFields F, PmFields M, const DevBlock *__restrict__ blocks) {
    const DevBlock B = blocks[blockIdx.y];
    const long long nq = pm_size(B);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!pm_cell(B, M.csize, q, i, j, k)) continue;
        const long long id = gidx(B, i, j, k), pm = B.pmoff + q;
#pragma unroll
        for (int m = 0; m < 5; m++) F.f[F_DQ1 + m][id] = M.dq[m][pm];
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory"); }

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Waits for the phase with the given parity to complete; gives up after
// `limit` clock cycles and returns false.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, long long limit) {
    const long long t0 = clock64();
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred pp;\n\tmbarrier.try_wait.parity.shared::cta.b64 pp, [%1], %2;\n\tselp.u32 %0, 1, 0, pp;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}
// bulk copy global -> own shared memory, completion counted on `bar`
// (addresses 16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

constexpr int SWEEP_STAGES = 4;  // ring of staged planes: the current one and three ahead

// shared memory of one CTA with `cpc` column slots: [stages][cpc][SR_N]
// static records, [stages][cpc][DYN_N] dynamic records, the inbox
// [2 plane parity][2 dir (j,k)][cpc][10 = A*dq, srv*dq], then the mbarriers
__host__ __device__ inline size_t sweep_smem_bytes(int cpc) {
    return (size_t)SWEEP_STAGES * cpc * (SR_N + DYN_N) * 8 + (size_t)2 * 2 * cpc * 10 * 8 + SWEEP_STAGES * 8;
}

template <int MODE>  // 0 lusgs_l, 1 lusgs_u, 2 gs_pr_l, 3 gs_pr_u
__global__ void __launch_bounds__(256) k_sweep(DevParams P, PmFields M, const DevBlock *__restrict__ blocks, int *err) {
    constexpr bool lu = MODE <= 1;
    constexpr bool with_dyn = MODE != 0;  // lusgs_u: dq of lusgs_l; gs_pr_l/u: old-side terms
    constexpr bool forward = (MODE == 0 || MODE == 2);
    constexpr int step = forward ? 1 : -1;
    const int C = M.csize;
    cg::cluster_group cluster = cg::this_cluster();
    const int q = (int)cluster.block_rank();
    const DevBlock B = blocks[blockIdx.x / C];
    const int ni = B.ni, nj = B.nj, nk = B.nk;
    const int j0 = chunk_j0(q, nj, C), w = chunk_j0(q + 1, nj, C) - j0;
    const int ncell = w * nk;               // columns of this CTA
    const int cpc = (nj + C - 1) / C * nk;  // column slots per CTA (>= ncell)
    extern __shared__ __align__(16) double smem[];
    double *sstat = smem;
    double *sdyn = sstat + (size_t)SWEEP_STAGES * cpc * SR_N;
    double *inbox = sdyn + (size_t)SWEEP_STAGES * cpc * DYN_N;
    unsigned long long *bars = (unsigned long long *)(inbox + (size_t)2 * 2 * cpc * 10);
    const size_t inbox_half = (size_t)2 * cpc * 10;
    const int t = threadIdx.x;
    const bool own = t < ncell;
    const int k = own ? t / w + 1 : 1;
    const int j = own ? j0 + t % w + 1 : 1;
    const int pfirst = forward ? 3 : ni + nj + nk, plast = forward ? ni + nj + nk : 3;
    // successors of this column along j and k (one step on) receive its contributions
    const int jn = j + step, kn = k + step;
    const bool outj = own && jn >= 1 && jn <= nj, outk = own && kn >= 1 && kn <= nk;
    double *dstj = nullptr, *dstk = nullptr;
    if (outj) {
        const int qj = chunk_of(jn - 1, nj, C), j0j = chunk_j0(qj, nj, C), wj = chunk_j0(qj + 1, nj, C) - j0j;
        double *base = qj == q ? inbox : cluster.map_shared_rank(inbox, qj);
        dstj = base + (size_t)((k - 1) * wj + (jn - 1 - j0j)) * 10;
    }
    if (outk) dstk = inbox + (size_t)cpc * 10 + (size_t)((kn - 1) * w + (j - 1 - j0)) * 10;
    // predecessors along j and k exist inside the block (at the block faces
    // the reference multiplies a zero dq: ghost value or the explicit zero of
    // gs_pr_l/u, so those terms are zero)
    const bool hasj = own && (forward ? j > 1 : j < nj), hask = own && (forward ? k > 1 : k < nk);
    const bool vis = lu && P.nvis > 0;

    if (t == 0) {
        for (int s = 0; s < SWEEP_STAGES; s++) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const unsigned stat_bytes = (unsigned)(ncell * SR_N * 8), dyn_bytes = with_dyn ? (unsigned)(ncell * DYN_N * 8) : 0u;
    auto issue = [&](int p) {  // thread 0: stage plane p
        if (ncell == 0 || (forward ? p > plast : p < plast)) return;
        const int s = ((p - pfirst) * step) % SWEEP_STAGES;
        const long long pm0 = pmidx(B, p, j0 * nk);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive_expect_tx(&bars[s], stat_bytes + dyn_bytes);
        bulk_g2s(sstat + (size_t)s * cpc * SR_N, M.stat + pm0 * SR_N, stat_bytes, &bars[s]);
        if (with_dyn) bulk_g2s(sdyn + (size_t)s * cpc * DYN_N, M.dyn + pm0 * DYN_N, dyn_bytes, &bars[s]);
    };
    if (t == 0)
        for (int a = 0; a < SWEEP_STAGES - 1; a++) issue(pfirst + a * step);
    // Barrier phases: the arrive after a plane's inbox stores releases them
    // to the consumers, which wait before reading.  Global stores of dq come
    // after the arrive (no other CTA reads them in this launch).
    cluster_arrive();

    bool timed_out = false;
    double cin[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, vin[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // own-column incoming
    for (int p = pfirst;; p += step) {
        const int i = p - j - k;
        const bool act = own && i >= 1 && i <= ni;
        const int pi = (p - pfirst) * step;
        const int s = pi % SWEEP_STAGES;
        // about a second for the first wait that runs out, then half a millisecond
        if (ncell > 0 && !mbar_wait(&bars[s], (unsigned)((pi / SWEEP_STAGES) & 1), timed_out ? (1LL << 20) : (1LL << 31)))
            timed_out = true;
        cluster_wait();
        // every thread of this CTA is done with plane p-1: refill its stage
        if (t == 0) issue(p + (SWEEP_STAGES - 1) * step);
        double nw[5];
        if (act) {
            const double *R = sstat + ((size_t)s * cpc + t) * SR_N;
            const double *D = sdyn + ((size_t)s * cpc + t) * DYN_N;
            const double *ib = inbox + (size_t)((p - step) & 1) * inbox_half + (size_t)t * 10;
            const double *inj = ib, *ink = ib + (size_t)cpc * 10;
            const double coed = R[SR_COED];
#pragma unroll
            for (int m = 0; m < 5; m++) {
                const double cj = hasj ? inj[m] : 0.0, ck = hask ? ink[m] : 0.0;
                if (MODE == 0 || MODE == 1) {
                    const double base = MODE == 0 ? R[SR_RHS + m] : D[m];
                    double r0 = 1.0 * (cin[m] + cj + ck);
                    if (vis) {
                        const double vj = hasj ? inj[5 + m] : 0.0, vk = hask ? ink[5 + m] : 0.0;
                        const double v = 0.5 * (vin[m] + vj + vk);
                        r0 = MODE == 0 ? r0 + v : r0 - v;
                    }
                    nw[m] = MODE == 0 ? (-base + r0) * coed : base - r0 * coed;
                } else if (MODE == 2) {
                    const double r0 = 1.0 * (cin[m] + cj + ck - D[m] - D[5 + m] - D[10 + m]);
                    nw[m] = (r0 - R[SR_RHS + m]) * coed;
                } else {
                    const double r0 = 1.0 * (D[m] - cin[m] - cj - ck);
                    nw[m] = (r0 - R[SR_RHS + m]) * coed;
                }
            }
            // this cell's contributions to its successors on the next plane
            const size_t wb = (size_t)(p & 1) * inbox_half;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const Jac J = rec_jac(R, d, forward ? 0 : 1);
                double o[5];
                jac_apply(P, J, nw, o);
                const double rv = vis ? R[SR_SRV + d] : 0.0;
                if (d == 0) {
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        cin[m] = o[m];
                        vin[m] = rv * nw[m];
                    }
                } else if ((d == 1 && outj) || (d == 2 && outk)) {
                    double *dst = (d == 1 ? dstj : dstk) + wb;
#pragma unroll
                    for (int m = 0; m < 5; m++) {
                        dst[m] = o[m];
                        dst[5 + m] = rv * nw[m];
                    }
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < 5; m++) {
                cin[m] = 0.0;
                vin[m] = 0.0;
            }
        }
        cluster_arrive();
        if (act) {
            const long long pm = pmidx(B, p, j0 * nk + t);
#pragma unroll
            for (int m = 0; m < 5; m++) M.dq[m][pm] = nw[m];
            if (MODE == 0) {
                double *Dg = M.dyn + pm * DYN_N;  // lusgs_u starts from it
#pragma unroll
                for (int m = 0; m < 5; m++) Dg[m] = nw[m];
            }
        }
        if (p == plast) break;
    }
    // the final wait keeps every CTA alive until the others' remote inbox
    // stores into it are done; every issued copy has been waited for above
    cluster_wait();
    if (timed_out && t == 0) atomicAdd(&err[ERR_TIMEOUT], 1);
}

template <int MODE>
static void launch_sweep(const LaunchCtx &c) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(c.nblocks * c.sweep_cluster, 1, 1);
    cfg.blockDim = dim3(c.sweep_threads, 1, 1);
    cfg.dynamicSmemBytes = sweep_smem_bytes(c.sweep_cpc);
    cfg.stream = c.stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c.sweep_cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_sweep<MODE>, *c.P, *c.PM, (const DevBlock *)c.blocks, c.err);
}

template <int MODE>
static void sweep_attrs(int smem, bool nonportable) {
    cudaFuncSetAttribute(k_sweep<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (nonportable) cudaFuncSetAttribute(k_sweep<MODE>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

// Chooses the cluster size (CTAs per block): the largest power of two <=
// `cluster` that the hardware can co-schedule with at most 256 column slots
// and 200 KB of shared memory per CTA.  Returns -1 when nothing fits.
int setup_sweep(LaunchCtx &c, int cluster) {
    int maxnj = 0, maxnk = 0;
    for (int b = 0; b < c.nblocks; b++) {
        maxnj = std::max(maxnj, c.hblocks[b].nj);
        maxnk = std::max(maxnk, c.hblocks[b].nk);
    }
    for (int cl = std::max(1, std::min(16, cluster)); cl >= 1; cl /= 2) {
        const int cpc = (maxnj + cl - 1) / cl * maxnk;
        const size_t sm = sweep_smem_bytes(cpc);
        if (cpc > 256 || sm > 200 * 1024) continue;
        const int threads = std::max(32, (cpc + 31) / 32 * 32);
        sweep_attrs<0>((int)sm, cl > 8);
        sweep_attrs<1>((int)sm, cl > 8);
        sweep_attrs<2>((int)sm, cl > 8);
        sweep_attrs<3>((int)sm, cl > 8);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim = dim3(c.nblocks * cl, 1, 1);
        cfg.blockDim = dim3(threads, 1, 1);
        cfg.dynamicSmemBytes = sm;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, k_sweep<2>, &cfg);
        if (e == cudaSuccess && nclusters >= 1) {
            c.sweep_cluster = cl;
            c.sweep_cpc = cpc;
            c.sweep_threads = threads;
            return 0;
        }
        cudaGetLastError();
    }
    return -1;
}

void launch_lhs(const LaunchCtx &c) {
    const int zg = (int)((c.nzero + 255) / 256);
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = std::max(maxp, pm_size(c.hblocks[b]));
    const dim3 pg((unsigned)((maxp + 255) / 256), c.nblocks);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
    k_lhs_prep<<<pg, 256, 0, c.stream>>>(*c.P, *c.F, *c.PM, c.blocks);
    launch_sweep<0>(c);
    launch_sweep<1>(c);
    k_gs_old<2><<<pg, 256, 0, c.stream>>>(*c.P, *c.PM, c.blocks);
    launch_sweep<2>(c);
    k_gs_old<3><<<pg, 256, 0, c.stream>>>(*c.P, *c.PM, c.blocks);
    launch_sweep<3>(c);
    k_pm_to_std<<<pg, 256, 0, c.stream>>>(*c.F, *c.PM, c.blocks);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
}

}  // namespace wcns
