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
//   k_sweep      one thread-block cluster per grid block (the reference's
//                LU-SGS is block-Jacobi, so blocks are independent).  CTA q
//                of the cluster owns a j-chunk of the block's (j,k) columns;
//                a column's lanes meet its cell once per plane.  The records
//                of a CTA's cells of one plane are contiguous, so one bulk
//                copy (issued planes ahead, mbarrier completion) stages them.
//                After computing its new dq a cell pushes its contributions
//                A*dq to its three successors on the next plane through
//                shared-memory inboxes; the j successor of a chunk's edge
//                column lives in the neighbouring CTA and is fed through a
//                ring of planes in that CTA's shared memory.  lusgs_u and
//                gs_pr_l also store these contributions in the successors'
//                records: evaluated with the sweep's final dq, they are the
//                Gauss-Seidel terms of the old side that the next sweep
//                (gs_pr_l, gs_pr_u) reads.
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
    int p, slot;
    if (q < 0x7fffffffLL) {  // 32-bit division where it suffices
        p = (int)q / ncol + 3;
        slot = (int)q % ncol;
    } else {
        p = (int)(q / ncol) + 3;
        slot = (int)(q % ncol);
    }
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
// The records of a CTA's PREP_THREADS consecutive slots are contiguous in
// memory: each thread builds its record in shared memory, then the CTA
// writes the rows of the slots inside the block with coalesced stores.
// Slots outside the block (about 40% of a plane-major array) keep the zero
// records they were allocated with: nothing ever writes them.
constexpr int PREP_THREADS = 128;
constexpr int PREP_LD = SR_N + 1;  // odd stride: conflict-free record rows

__global__ void __launch_bounds__(PREP_THREADS) k_lhs_prep(DevParams P, DevFields F, PmFields M,
                                                           const DevBlock *__restrict__ blocks) {
    __shared__ double srec[PREP_THREADS * PREP_LD];
    __shared__ unsigned char srow[PREP_THREADS];  // slot inside the block
    const DevBlock B = blocks[blockIdx.y];
    const double gama = P.gama;
    const long long nq = pm_size(B);
    for (long long q0 = (long long)blockIdx.x * PREP_THREADS; q0 < nq; q0 += (long long)gridDim.x * PREP_THREADS) {
        const long long q = q0 + threadIdx.x;
        double *R = srec + threadIdx.x * PREP_LD;
        int i, j, k;
        const bool valid = q < nq && pm_cell(B, M.csize, q, i, j, k);
        srow[threadIdx.x] = valid ? 1 : 0;
        if (valid) {
            const long long id = gidx(B, i, j, k);
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
        __syncthreads();
        const long long nvalid = nq - q0 < PREP_THREADS ? nq - q0 : PREP_THREADS;
        double *dst = M.stat + (B.pmoff + q0) * SR_N;
        for (int e = threadIdx.x; e < nvalid * SR_N; e += PREP_THREADS) {
            const int r = e / SR_N;
            if (srow[r]) dst[e] = srec[r * PREP_LD + e - r * SR_N];
        }
        __syncthreads();
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

constexpr int SWEEP_STAGES = 3;  // ring of staged planes: the current one and two ahead
constexpr int JRING = 6;         // ring of planes in flight between neighbouring CTAs
constexpr int SWEEP_COARSE_MAX_THREADS = 384;
constexpr int SWEEP_FINE_MAX_THREADS = 768;

// shared memory of one CTA with `cpc` column slots:
//   [SWEEP_STAGES][cpc][SR_N]  static records of a plane
//   [SWEEP_STAGES][cpc][DYN_N] dynamic records of a plane
//   [2 plane parity][3 dir (i,j,k)][cpc][10]  inbox from this CTA's own cells
//   [JRING][cpc][10]           inbox from the neighbouring CTA (j direction)
//   mbarriers: SWEEP_STAGES (bulk copies), JRING full, JRING empty
__host__ __device__ inline size_t sweep_smem_bytes(int cpc) {
    return (size_t)SWEEP_STAGES * cpc * (SR_N + DYN_N) * 8 + (size_t)2 * 3 * cpc * 10 * 8 + (size_t)JRING * cpc * 10 * 8 +
           (size_t)(SWEEP_STAGES + 2 * JRING) * 8;
}

__device__ __forceinline__ unsigned remote_u32(const void *local, int rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}
// arrive on an mbarrier of another CTA of the cluster without a release
// fence (the caller orders what must come before it)
__device__ __forceinline__ void mbar_arrive_remote_relaxed(unsigned cluster_addr) {
    asm volatile("mbarrier.arrive.relaxed.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}
// stores into another CTA's shared memory, counted as transaction bytes on
// that CTA's mbarrier
__device__ __forceinline__ void st_async_v2(unsigned cluster_addr, double a, double b, unsigned cluster_mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];\n" ::"r"(cluster_addr),
                 "d"(a), "d"(b), "r"(cluster_mbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_f64(unsigned cluster_addr, double a, unsigned cluster_mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];\n" ::"r"(cluster_addr), "d"(a),
                 "r"(cluster_mbar)
                 : "memory");
}

// One sweep, one cluster per block, CTA q owning j-chunk q (every chunk at
// least one column wide).  The work of a cell -- its new dq and the three
// contributions A*dq for its successors one plane on -- is spread over the
// lanes of its column:
//   FINE   16 lanes per column; lane (d, m), d = lane/5, m = lane%5 for
//          lanes 0..14, evaluates component m of the new dq, receives the
//          other four from its direction group by warp shuffles, and
//          evaluates row m of the split Jacobian product along d.
//   coarse three threads per column (d-major), each evaluating all of dq
//          and the product along its d (blocks whose chunks are too wide
//          for FINE).
// The arithmetic of every value is that of mxdq_std in either layout.  One
// extra control warp does all mbarrier work, so the compute threads meet
// nothing but one __syncthreads per plane.
//
// Dependencies between CTAs run one way only: in a forward sweep CTA q needs
// the last column of chunk q-1 from the previous plane, in a backward sweep
// the first column of chunk q+1.  They travel point to point through a ring
// of JRING planes in the consumer's shared memory: the producer's boundary
// threads write 10 values per cell and plane with st.async, whose bytes
// complete the consumer's `full` mbarrier for that slot (armed by the
// consumer's control thread with the plane's byte count); once the slot has
// been read the consumer's control thread re-arms it and arrives on the
// producer's `empty` mbarrier.  Boundary producers write every plane, inside
// the block or not, so the byte count per plane is fixed.  No release fence
// is on the per-plane path, and a CTA may run ahead of its downstream
// neighbour, so the cross-CTA latency is paid once per chunk rather than
// once per plane.
//
// Per plane pi the control thread, before the CTA's __syncthreads, waits for
// the bulk copy of plane pi+1, the ring slot holding plane pi-1 (upstream),
// and the free ring slot for plane pi (downstream); after it, it refills the
// stage of plane pi with plane pi+SWEEP_STAGES (the compute threads have
// loaded their coefficients into registers before the barrier) and releases
// the ring slot read during plane pi-1.
template <int MODE, bool FINE>  // MODE 0 lusgs_l, 1 lusgs_u, 2 gs_pr_l, 3 gs_pr_u
__global__ void __launch_bounds__(FINE ? SWEEP_FINE_MAX_THREADS : SWEEP_COARSE_MAX_THREADS)
    k_sweep(DevParams P, PmFields M, const DevBlock *__restrict__ blocks, int *err) {
    constexpr bool lu = MODE <= 1;
    constexpr bool with_dyn = MODE != 0;  // lusgs_u: dq of lusgs_l; gs_pr_l/u: old-side terms
    constexpr bool forward = (MODE == 0 || MODE == 2);
    constexpr int step = forward ? 1 : -1;
    constexpr int NC = FINE ? 1 : 5;  // dq components evaluated per thread
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
    double *jring = inbox + (size_t)2 * 3 * cpc * 10;
    unsigned long long *bars = (unsigned long long *)(jring + (size_t)JRING * cpc * 10);
    unsigned long long *full = bars + SWEEP_STAGES, *empty = full + JRING;
    const size_t inbox_half = (size_t)3 * cpc * 10, inbox_dir = (size_t)cpc * 10;
    const int t = threadIdx.x;
    const bool ctl = t == (int)blockDim.x - 32;  // control thread: lane 0 of the last warp
    const bool own = FINE ? (t < 16 * ncell && (t & 15) < 15) : t < 3 * ncell;
    const int d = !own ? 0 : FINE ? (t & 15) / 5 : t / ncell;  // direction of this thread's contribution
    const int m0 = FINE && own ? (t & 15) % 5 : 0;             // first dq component of this thread
    const int c = !own ? 0 : FINE ? t >> 4 : t % ncell;        // column within the CTA
    const int jj = c % w;                                      // column within the chunk
    const int k = c / w + 1;
    const int j = j0 + jj + 1;
    const int pfirst = forward ? 3 : ni + nj + nk;
    const int nplanes = ni + nj + nk - 2;
    // neighbouring CTAs: upstream feeds this CTA, downstream is fed by it
    const int qu = q - step, qd = q + step;
    const bool has_up = qu >= 0 && qu < C, has_down = qd >= 0 && qd < C;
    const bool bconsumer = own && has_up && jj == (forward ? 0 : w - 1);
    const bool bproducer = own && d == 1 && has_down && jj == (forward ? w - 1 : 0);
    const unsigned ring_bytes = (unsigned)nk * 80u;  // one plane of the boundary column
    // predecessors along j and k inside the block (at the block faces the
    // reference multiplies a zero dq: ghost value or the explicit zero of
    // gs_pr_l/u, so those terms are zero); along i see `hasi` below
    const bool hasj = own && (forward ? j > 1 : j < nj), hask = own && (forward ? k > 1 : k < nk);
    // destination of this thread's contribution inside the CTA
    double *dst = nullptr;
    if (own) {
        if (d == 0) dst = inbox + (size_t)c * 10;
        else if (d == 1 && !bproducer && (forward ? j < nj : j > 1)) dst = inbox + inbox_dir + (size_t)(c + step) * 10;
        else if (d == 2 && (forward ? k < nk : k > 1)) dst = inbox + 2 * inbox_dir + (size_t)(c + step * w) * 10;
    }
    const double *srci = inbox + (size_t)c * 10 + m0;
    const double *srcj = (bconsumer ? jring + (size_t)(k - 1) * 10 : inbox + inbox_dir + (size_t)c * 10) + m0;
    const double *srck = inbox + 2 * inbox_dir + (size_t)c * 10 + m0;
    const bool vis = lu && P.nvis > 0;

    if (ctl) {
        for (int s = 0; s < SWEEP_STAGES; s++) mbar_init(&bars[s], 1);
        for (int s = 0; s < JRING; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        if (has_up)
            for (int s = 0; s < JRING; s++) mbar_arrive_expect_tx(&full[s], ring_bytes);
    }
    // every CTA's barriers are initialised and armed before anyone writes remotely
    cluster_arrive();
    cluster_wait();
    unsigned ring_remote = 0, full_remote = 0, empty_remote = 0;
    if (bproducer) {
        ring_remote = remote_u32(jring + (size_t)(k - 1) * 10, qd);
        full_remote = remote_u32(full, qd);
    }
    if (ctl && has_up) empty_remote = remote_u32(empty, qu);

    const unsigned stat_bytes = (unsigned)(ncell * SR_N * 8), dyn_bytes = with_dyn ? (unsigned)(ncell * DYN_N * 8) : 0u;
    // lusgs_u reads the dq of lusgs_l, gs_pr_l / gs_pr_u the old-side terms that
    // lusgs_u / gs_pr_l left behind
    const double *dyn_src = MODE == 1 ? M.dyn : MODE == 2 ? M.gs[0] : M.gs[1];
    auto issue = [&](int pi) {  // control thread: stage plane index pi
        if (pi >= nplanes) return;
        const int s = pi % SWEEP_STAGES;
        const long long pm0 = pmidx(B, pfirst + pi * step, j0 * nk);
        mbar_arrive_expect_tx(&bars[s], stat_bytes + dyn_bytes);
        bulk_g2s(sstat + (size_t)s * cpc * SR_N, M.stat + pm0 * SR_N, stat_bytes, &bars[s]);
        if (with_dyn) bulk_g2s(sdyn + (size_t)s * cpc * DYN_N, dyn_src + pm0 * DYN_N, dyn_bytes, &bars[s]);
    };
    bool timed_out = false;
    auto limit = [&]() { return timed_out ? (1LL << 20) : (1LL << 31); };  // ~1 s for the first, then ~0.5 ms
    if (ctl) {
        for (int a = 0; a < SWEEP_STAGES; a++) issue(a);
        if (!mbar_wait(&bars[0], 0u, limit())) timed_out = true;
    }
    __syncthreads();

    // lusgs_u and gs_pr_l: this thread's product along d, evaluated with the
    // cell's final dq of this sweep, is the old-side term of the successor
    // along d in the next sweep (what gs_pr_l / gs_pr_u would recompute from
    // the stored dq); it goes to the successor's record, column slot gs_slot
    // (plane p + step, column slot gs_slot: gs_rec + (p + step - 3) * one plane)
    double *gs_rec = nullptr;
    if ((MODE == 1 || MODE == 2) && own) {
        int gs_slot = -1;
        if (d == 0) gs_slot = j0 * nk + c;
        else if (d == 1 ? (forward ? j < nj : j > 1) : (forward ? k < nk : k > 1))
            gs_slot = col_slot(d == 1 ? j + step : j, d == 2 ? k + step : k, nj, nk, C);
        if (gs_slot >= 0) gs_rec = M.gs[MODE == 2 ? 1 : 0] + (B.pmoff + gs_slot) * DYN_N + 5 * d + m0;
    }
    const long long gs_plane = (long long)nj * nk * DYN_N;
    const double ae = P.gama - 1.0;
    for (int pi = 0; pi < nplanes; pi++) {
        const int p = pfirst + pi * step;
        const int i = p - j - k;
        const bool act = own && i >= 1 && i <= ni;
        const bool hasi = forward ? i > 1 : i < ni;
        const int s = pi % SWEEP_STAGES;
        // the cell's coefficients (independent of this sweep's new values)
        double coed = 0.0, base[NC], old0[NC], old1[NC], old2[NC], rv = 0.0, nn = 0.0, uu = 0.0;
        Jac J;
        if (act) {
            const double *R = sstat + ((size_t)s * cpc + c) * SR_N;
            const double *D = sdyn + ((size_t)s * cpc + c) * DYN_N + m0;
            coed = R[SR_COED];
#pragma unroll
            for (int m = 0; m < NC; m++) {
                base[m] = MODE == 1 ? D[m] : R[SR_RHS + m0 + m];
                // gs_pr_u: (del + dfl) + dgl of the lower neighbours, gs_pr_l: the three upper terms
                old0[m] = MODE == 3 ? D[m] + D[5 + m] + D[10 + m] : MODE == 2 ? D[m] : 0.0;
                old1[m] = MODE == 2 ? D[5 + m] : 0.0;
                old2[m] = MODE == 2 ? D[10 + m] : 0.0;
            }
            J = rec_jac(R, d, forward ? 0 : 1);
            if (vis) rv = R[SR_SRV + d];
            if (FINE && m0 > 0) {  // row m0 of the product: (nx, um), (ny, vm), (nz, wm) or (ct, hm)
                nn = R[SR_JD + 4 * d + (m0 & 3)];
                uu = R[SR_JS + (m0 == 4 ? 4 : m0 - 1)];
            }
        }
        if (ctl) {
            if (pi + 1 < nplanes &&
                !mbar_wait(&bars[(pi + 1) % SWEEP_STAGES], (unsigned)(((pi + 1) / SWEEP_STAGES) & 1), limit()))
                timed_out = true;
            // upstream plane pi-1 in ring slot (pi-1) % JRING
            if (has_up && pi > 0 && !mbar_wait(&full[(pi - 1) % JRING], (unsigned)(((pi - 1) / JRING) & 1), limit()))
                timed_out = true;
            // downstream ring slot pi % JRING free (its plane pi - JRING read)
            if (has_down && pi < nplanes - 1 &&
                !mbar_wait(&empty[pi % JRING], (unsigned)(((pi / JRING) & 1) ^ 1), limit()))
                timed_out = true;
        }
        __syncthreads();  // own inbox of plane pi-1 complete; coefficients of plane pi in registers
        if (ctl) {
            issue(pi + SWEEP_STAGES);
            if (has_up && pi >= 2) {
                const int sr = (pi - 2) % JRING;
                mbar_arrive_expect_tx(&full[sr], ring_bytes);
                mbar_arrive_remote_relaxed(empty_remote + (unsigned)(sr * 8));
            }
        }
        const size_t rd = (size_t)((pi + 1) & 1) * inbox_half, wr = (size_t)(pi & 1) * inbox_half;
        // new dq, components m0 .. m0+NC-1
        double nw[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (act) {
            const double *inj = srcj + (bconsumer ? (size_t)((pi - 1) % JRING) * cpc * 10 : rd);
#pragma unroll
            for (int m = 0; m < NC; m++) {
                const double ci = hasi ? srci[rd + m] : 0.0, cj = hasj ? inj[m] : 0.0, ck = hask ? srck[rd + m] : 0.0;
                if (MODE == 0 || MODE == 1) {
                    double r0 = 1.0 * (ci + cj + ck);
                    if (vis) {
                        const double vi = hasi ? srci[rd + 5 + m] : 0.0, vj = hasj ? inj[5 + m] : 0.0,
                                     vk = hask ? srck[rd + 5 + m] : 0.0;
                        const double v = 0.5 * (vi + vj + vk);
                        r0 = MODE == 0 ? r0 + v : r0 - v;
                    }
                    nw[m] = MODE == 0 ? (-base[m] + r0) * coed : base[m] - r0 * coed;
                } else if (MODE == 2) {
                    const double r0 = 1.0 * (ci + cj + ck - old0[m] - old1[m] - old2[m]);
                    nw[m] = (r0 - base[m]) * coed;
                } else {
                    const double r0 = 1.0 * (old0[m] - ci - cj - ck);
                    nw[m] = (r0 - base[m]) * coed;
                }
            }
        }
        const double own_nw = nw[0];  // FINE: component m0
        if constexpr (FINE) {
            // gather the five components from the direction group (all lanes take part)
            const int g = (t & ~15) + 5 * d;
#pragma unroll
            for (int m = 0; m < 5; m++) nw[m] = __shfl_sync(0xffffffffu, own_nw, (g + m) & 31);
        }
        // contribution along d for the successor (rows m0 .. m0+NC-1 of mxdq_std)
        double o[2 * NC];
        if (act) {
            if constexpr (FINE) {
                const double dc = J.ct * nw[0] - J.nx * nw[1] - J.ny * nw[2] - J.nz * nw[3];
                const double dh = J.af * nw[0] - ae * (J.um * nw[1] + J.vm * nw[2] + J.wm * nw[3] - nw[4]);
                const double c2dc = J.c2 * dc;
                o[0] = m0 == 0 ? J.l1 * nw[0] - dh * J.x1 - dc * J.x2
                               : J.l1 * own_nw + (nn * c2dc - uu * dh) * J.x1 + (nn * dh - uu * dc) * J.x2;
                o[1] = rv * own_nw;
            } else {
                double f[5];
                jac_apply(P, J, nw, f);
#pragma unroll
                for (int m = 0; m < 5; m++) {
                    o[m] = f[m];
                    o[5 + m] = rv * nw[m];
                }
            }
            if (dst) {
#pragma unroll
                for (int m = 0; m < NC; m++) {
                    dst[wr + m0 + m] = o[m];
                    dst[wr + 5 + m0 + m] = o[NC + m];
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < 2 * NC; m++) o[m] = 0.0;  // a boundary producer still sends the plane
        }
        if (bproducer && pi < nplanes - 1) {
            const int so = pi % JRING;
            const unsigned a = ring_remote + (unsigned)(so * cpc * 80), mb = full_remote + (unsigned)(so * 8);
            if constexpr (FINE) {
                st_async_f64(a + 8u * m0, o[0], mb);
                st_async_f64(a + 8u * (5 + m0), o[1], mb);
            } else {
#pragma unroll
                for (int m = 0; m < 10; m += 2) st_async_v2(a + 8u * m, o[m], o[m + 1], mb);
            }
        }
        if ((MODE == 1 || MODE == 2) && act && gs_rec && (d != 0 || (forward ? i < ni : i > 1))) {
            double *G = gs_rec + (long long)(p + step - 3) * gs_plane;
#pragma unroll
            for (int m = 0; m < NC; m++) G[m] = o[m];
        }
        if (act && d == 0) {
            const long long pm = pmidx(B, p, j0 * nk + c);
            if (MODE == 3)  // the result of the four sweeps
#pragma unroll
                for (int m = 0; m < NC; m++) M.dq[0][(m0 + m) * M.dq_stride + pm] = FINE ? own_nw : nw[m];
            if (MODE == 0) {
                double *Dg = M.dyn + pm * DYN_N + m0;  // lusgs_u starts from it
#pragma unroll
                for (int m = 0; m < NC; m++) Dg[m] = FINE ? own_nw : nw[m];
            }
        }
    }
    // Every issued bulk copy has been waited for above.  Keep every CTA
    // alive until the others' remote stores and arrivals into it are done:
    // every ring write has been waited for by its consumer, and the
    // consumer's arrivals on the producer's `empty` barriers precede the
    // final barrier.
    cluster_arrive();
    cluster_wait();
    if (timed_out) atomicAdd(&err[ERR_TIMEOUT], 1);
}

// One thread initialises an mbarrier that nothing arrives at and waits for
// its first phase with the sweep's bounded wait; the wait gives up after
// `limit` cycles and the timeout is reported in the error slot the sweeps
// use.  No copy or remote store is in flight, so giving up is safe.
__global__ void k_wait_probe(int *err, long long limit) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    if (!mbar_wait(&bar, 0u, limit)) atomicAdd(&err[ERR_TIMEOUT], 1);
}

void launch_wait_probe(const LaunchCtx &c, long long limit) { k_wait_probe<<<1, 32, 0, c.stream>>>(c.err, limit); }

template <int MODE, bool FINE>
static void launch_sweep_t(const LaunchCtx &c) {
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
    cudaLaunchKernelEx(&cfg, k_sweep<MODE, FINE>, *c.P, *c.PM, (const DevBlock *)c.blocks, c.err);
}
template <int MODE>
static void launch_sweep(const LaunchCtx &c) {
    if (c.sweep_fine) launch_sweep_t<MODE, true>(c);
    else launch_sweep_t<MODE, false>(c);
}

template <bool FINE>
static void sweep_attrs(int smem, bool nonportable) {
    auto set = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (nonportable) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    };
    set(k_sweep<0, FINE>);
    set(k_sweep<1, FINE>);
    set(k_sweep<2, FINE>);
    set(k_sweep<3, FINE>);
}

// Chooses the sweep shape: the lane layout (FINE when `fine` and the chunk
// fits, else coarse) and the cluster size (CTAs per block), the largest size
// <= `cluster` and <= the smallest nj (every j-chunk non-empty) that the
// hardware can co-schedule within the layout's thread limit and 200 KB of
// shared memory per CTA.  Returns -1 when nothing fits.
template <bool FINE>
static bool try_sweep_shape(LaunchCtx &c, int cl, int cpc) {
    const size_t sm = sweep_smem_bytes(cpc);
    const int lanes = FINE ? 16 : 3, maxt = FINE ? SWEEP_FINE_MAX_THREADS : SWEEP_COARSE_MAX_THREADS;
    const int threads = (lanes * cpc + 31) / 32 * 32 + 32;  // compute warps + the control warp
    if (threads > maxt || sm > 200 * 1024) return false;
    sweep_attrs<FINE>((int)sm, cl > 8);
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
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, k_sweep<2, FINE>, &cfg);
    if (e != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return false;
    }
    c.sweep_cluster = cl;
    c.sweep_cpc = cpc;
    c.sweep_threads = threads;
    c.sweep_fine = FINE ? 1 : 0;
    return true;
}

int setup_sweep(LaunchCtx &c, int cluster, int fine) {
    int maxnj = 0, maxnk = 0, minnj = 1 << 30;
    for (int b = 0; b < c.nblocks; b++) {
        maxnj = std::max(maxnj, c.hblocks[b].nj);
        maxnk = std::max(maxnk, c.hblocks[b].nk);
        minnj = std::min(minnj, c.hblocks[b].nj);
    }
    const int top = std::max(1, std::min(std::min(16, minnj), cluster));
    if (fine)
        for (int cl = top; cl >= 1; cl--)
            if (try_sweep_shape<true>(c, cl, (maxnj + cl - 1) / cl * maxnk)) return 0;
    for (int cl = top; cl >= 1; cl--)
        if (try_sweep_shape<false>(c, cl, (maxnj + cl - 1) / cl * maxnk)) return 0;
    return -1;
}

// Exactly the shape (cl CTAs per block cluster, sixteen lanes per column
// when fine, else three); -1 when the blocks cannot be swept with it, with
// the shape in use left as it was.
int setup_sweep_exact(LaunchCtx &c, int cl, int fine) {
    int maxnj = 0, maxnk = 0, minnj = 1 << 30;
    for (int b = 0; b < c.nblocks; b++) {
        maxnj = std::max(maxnj, c.hblocks[b].nj);
        maxnk = std::max(maxnk, c.hblocks[b].nk);
        minnj = std::min(minnj, c.hblocks[b].nj);
    }
    if (cl < 1 || cl > 16 || cl > minnj) return -1;
    const int cpc = (maxnj + cl - 1) / cl * maxnk;
    const int old_cl = c.sweep_cluster, old_cpc = c.sweep_cpc, old_fine = c.sweep_fine;
    if (fine ? try_sweep_shape<true>(c, cl, cpc) : try_sweep_shape<false>(c, cl, cpc)) return 0;
    // a refused shape may have changed the kernels' shared-memory attributes
    if (old_fine) try_sweep_shape<true>(c, old_cl, old_cpc);
    else try_sweep_shape<false>(c, old_cl, old_cpc);
    return -1;
}

int launch_lhs(const LaunchCtx &c) {
    const int zg = (int)((c.nzero + 255) / 256);
    if (c.wide) {
        if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
        int n = launch_sweeps_wide(c);
        if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
        prof_mark(c, "lhs_store");
        return n + (c.nzero > 0 ? 2 : 0);
    }
    if (c.sweep_plane) {
        // set_nonconnect_boundary_dq_0, the sweeps plane by plane, again the faces
        if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
        prof_mark(c, "lhs_prep");
        int n = launch_sweeps_by_plane(c);
        if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
        prof_mark(c, "lhs_store");
        return n + (c.nzero > 0 ? 2 : 0);
    }
    long long maxp = 0;
    for (int b = 0; b < c.nblocks; b++) maxp = std::max(maxp, pm_size(c.hblocks[b]));
    const dim3 pg((unsigned)((maxp + 255) / 256), c.nblocks);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
    const dim3 pg128((unsigned)((maxp + PREP_THREADS - 1) / PREP_THREADS), c.nblocks);
    k_lhs_prep<<<pg128, PREP_THREADS, 0, c.stream>>>(*c.P, *c.F, *c.PM, c.blocks);
    prof_mark(c, "lhs_prep");
    launch_sweep<0>(c);
    prof_mark(c, "sweep_lusgs_l");
    launch_sweep<1>(c);
    prof_mark(c, "sweep_lusgs_u");
    launch_sweep<2>(c);
    prof_mark(c, "sweep_gs_pr_l");
    launch_sweep<3>(c);
    prof_mark(c, "sweep_gs_pr_u");
    k_pm_to_std<<<pg, 256, 0, c.stream>>>(*c.F, *c.PM, c.blocks);
    if (c.nzero > 0) k_zero_faces<<<zg, 256, 0, c.stream>>>(*c.F, c.zero_pts, c.nzero);
    prof_mark(c, "lhs_store");
    return 6 + (c.nzero > 0 ? 2 : 0);  // prep, four sweeps, plane-major dq to the fields
}

}  // namespace wcns
