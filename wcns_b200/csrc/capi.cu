// capi.cu -- C ABI and host-side set-up of the WCNS B200 path.
//
// Host work done once per context (the reference's pre-processing):
//   * BC regions: analyze_bc / analyze_bc_connect (parallel.f90:1123-1300)
//     give the face ranges, outward directions and interface image maps;
//     set_bc_index (PreProcess.f90:2543-2572) orders regions -1,4,5,6,2,3.
//   * multi-point interface sets: connect_pre_parallel and comp_list_insert
//     (parallel.f90:177-393, 4202-4311), build_nppos_list_ex (2939-3018).
//   * device tables: interface ghost-copy list, physical regions per block,
//     dq-zero list, interface point snapshot list, averaging pairs, line
//     groups for the residual kernels.
// Semantics are those of the reference run with one block per MPI rank:
// exchanges between different blocks use start-of-exchange snapshots; a
// block connected to itself uses the in-place same-rank path.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/wcns_b200.h"
#include "wcns_dev.cuh"
#include "wcns_launch.h"

using namespace wcns;

static thread_local std::string g_err;
static void set_err(const std::string &s) { g_err = s; }
extern "C" const char *wcns_last_error(void) { return g_err.c_str(); }
namespace wcns {
void set_last_error(const std::string &msg) { g_err = msg; }  // for entry points in other files
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            set_err(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);      \
            return WCNS_ERR_CUDA;                                                              \
        }                                                                                      \
    } while (0)

namespace {

struct HReg {
    int bctype = 0;
    int raw_s_st[3], raw_s_ed[3], raw_t_st[3], raw_t_ed[3];
    int nbt = 0, ibcwin = 0;
    int s_st[3], s_ed[3], s_nd = 0, s_lr = 0, s_lr3d[3];
    int t_st[3], t_ed[3], t_nd = 0, t_lr = 0, t_lr3d[3];
    std::vector<int> img[3];
    int iused = 0;
    int box(int i, int j, int k) const {
        int nx = s_ed[0] - s_st[0] + 1, ny = s_ed[1] - s_st[1] + 1;
        return (i - s_st[0]) + nx * ((j - s_st[1]) + ny * (k - s_st[2]));
    }
};

struct HBlock {
    DevBlock d;
    std::vector<HReg> regs;
    std::vector<int> bcindex;
};

template <class T>
T *dev_upload(const std::vector<T> &v) {
    if (v.empty()) return nullptr;
    T *p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * v.size()) != cudaSuccess) return nullptr;
    cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return p;
}

}  // namespace

struct WcnsContext {
    WcnsParams prm{};
    DevParams P{};
    DevFields F{};
    std::vector<HBlock> blk;  // 0-based
    long long total = 0;      // ghosted points over all blocks
    long long total_pm = 0;   // plane-major sweep points over all blocks
    double *pool = nullptr;
    double *pm_pool = nullptr;
    PmFields PM{};
    cudaStream_t stream = nullptr;
    LaunchCtx L;
    std::vector<void *> owned;  // device allocations to free
    int *d_err = nullptr;
    double *d_hist = nullptr;
    int hist_cap = 0;
    cudaGraphExec_t graph = nullptr;
    int nmulti = 0;
    // Spalart-Allmaras model (wcns_sa_setup)
    double *sa_pool = nullptr;
    SaFields SA{};
    SaParams SAP{};
    int launches = 0;
    std::unique_ptr<WideSweep> wide;
    std::vector<DevWall> hwalls;  // host copy of the wall table (block order)
    double *adj_pool = nullptr;   // the adjoint slots (WCNS_ADJ_*), five fields each, on first use
    // staging of wcns_set_interior / wcns_get_interior: the interior points of
    // up to stage_fields fields, contiguous per block and field; stage_first:
    // per (field slot, block) the first element, device
    double *stage = nullptr;
    long long *stage_first = nullptr;
    int stage_fields = 0;
    ~WcnsContext() {
        if (graph) cudaGraphExecDestroy(graph);
        for (int q = 0; q < 2; q++) {
            if (L.side[q]) cudaStreamDestroy(L.side[q]);
            if (L.ev_join[q]) cudaEventDestroy(L.ev_join[q]);
        }
        if (L.ev_fork) cudaEventDestroy(L.ev_fork);
        for (void *p : owned) cudaFree(p);
        if (pool) cudaFree(pool);
        if (pm_pool) cudaFree(pm_pool);
        if (sa_pool) cudaFree(sa_pool);
        if (adj_pool) cudaFree(adj_pool);
        if (stage) cudaFree(stage);
        if (stage_first) cudaFree(stage_first);
        if (stream) cudaStreamDestroy(stream);
    }
    template <class T>
    T *up(const std::vector<T> &v) {
        T *p = dev_upload(v);
        if (p) owned.push_back(p);
        return p;
    }
    long long gi(int nb1, int i, int j, int k) const { return gidx(blk[nb1 - 1].d, i, j, k); }
};

// ---------------------------------------------------------------------------
// analyze_bc + analyze_bc_connect (parallel.f90:1123-1300)
static int analyze(WcnsContext *c) {
    const int nbk = (int)c->blk.size();
    for (int b = 0; b < nbk; b++) {
        HBlock &B = c->blk[b];
        int dims[3] = {B.d.ni, B.d.nj, B.d.nk};
        for (HReg &R : B.regs) {
            for (int m = 0; m < 3; m++) {
                int a = std::abs(R.raw_s_st[m]), e = std::abs(R.raw_s_ed[m]);
                R.s_st[m] = std::min(a, e);
                R.s_ed[m] = std::max(a, e);
                R.s_lr3d[m] = 0;
                if (R.raw_s_st[m] == R.raw_s_ed[m]) {
                    R.s_nd = m + 1;
                    R.s_lr = R.raw_s_st[m] == 1 ? -1 : 1;
                    R.s_lr3d[m] = R.s_lr;
                }
                if (R.s_st[m] < 1 || R.s_ed[m] > dims[m]) {
                    set_err("BC region outside its block (block " + std::to_string(b + 1) + ")");
                    return WCNS_ERR_ARGUMENT;
                }
            }
            if (R.s_nd == 0) { set_err("BC region is not a face"); return WCNS_ERR_ARGUMENT; }
            if (R.bctype < 0) {
                if (R.nbt < 1 || R.nbt > nbk) { set_err("interface target block out of range"); return WCNS_ERR_ARGUMENT; }
                int std_[3][3] = {{0}};
                for (int m = 0; m < 3; m++) {
                    R.t_lr3d[m] = 0;
                    if (R.raw_t_st[m] == R.raw_t_ed[m]) {
                        R.t_nd = m + 1;
                        R.t_lr = R.raw_t_st[m] == 1 ? -1 : 1;
                        R.t_lr3d[m] = R.t_lr;
                    }
                }
                if (R.t_nd == 0) { set_err("interface target is not a face"); return WCNS_ERR_ARGUMENT; }
                bool done = false;
                for (int m = 1; m <= 3 && !done; m++)
                    for (int n = 1; n <= 3 && !done; n++) {
                        if (m == R.s_nd || n == R.t_nd) continue;
                        int js1 = R.raw_s_st[m - 1];
                        if (std::abs(js1) < std::abs(R.raw_s_ed[m - 1])) js1 = R.raw_s_ed[m - 1];
                        int js2 = R.raw_t_st[n - 1];
                        if (std::abs(js2) < std::abs(R.raw_t_ed[n - 1])) js2 = R.raw_t_ed[n - 1];
                        if ((long long)js1 * js2 > 0) {
                            std_[n - 1][m - 1] = 1;
                            std_[R.t_nd - 1][R.s_nd - 1] = 1;
                            std_[6 - n - R.t_nd - 1][6 - m - R.s_nd - 1] = 1;
                            done = true;
                        }
                    }
                int s_st[3], s_ed[3], t_st[3], s_sign[3], t_sign[3], st_sign[3];
                for (int m = 0; m < 3; m++) {
                    s_st[m] = std::abs(R.raw_s_st[m]);
                    s_ed[m] = std::abs(R.raw_s_ed[m]);
                    t_st[m] = std::abs(R.raw_t_st[m]);
                    int t_ed = std::abs(R.raw_t_ed[m]);
                    s_sign[m] = (m + 1 != R.s_nd && s_st[m] > s_ed[m]) ? -1 : 1;
                    t_sign[m] = (m + 1 != R.t_nd && t_st[m] > t_ed) ? -1 : 1;
                    R.t_st[m] = std::min(t_st[m], t_ed);
                    R.t_ed[m] = std::max(t_st[m], t_ed);
                }
                for (int m = 0; m < 3; m++) {
                    int co = 0;
                    for (int n = 0; n < 3; n++)
                        if (std_[n][m]) co = n + 1;
                    if (!co) { set_err("interface orientation could not be resolved"); return WCNS_ERR_ARGUMENT; }
                    st_sign[m] = t_sign[co - 1] * s_sign[m];
                }
                int nbox = (R.s_ed[0] - R.s_st[0] + 1) * (R.s_ed[1] - R.s_st[1] + 1) * (R.s_ed[2] - R.s_st[2] + 1);
                for (int q = 0; q < 3; q++) R.img[q].assign(nbox, 0);
                for (int i = s_st[0];; i += s_sign[0]) {
                    int id_ = (i - s_st[0]) * st_sign[0];
                    for (int j = s_st[1];; j += s_sign[1]) {
                        int jd = (j - s_st[1]) * st_sign[1];
                        for (int k = s_st[2];; k += s_sign[2]) {
                            int kd = (k - s_st[2]) * st_sign[2];
                            int bx = R.box(i, j, k);
                            for (int q = 0; q < 3; q++) R.img[q][bx] = t_st[q] + std_[q][0] * id_ + std_[q][1] * jd + std_[q][2] * kd;
                            if (k == s_ed[2]) break;
                        }
                        if (j == s_ed[1]) break;
                    }
                    if (i == s_ed[0]) break;
                }
                const HBlock &T = c->blk[R.nbt - 1];
                int tdims[3] = {T.d.ni, T.d.nj, T.d.nk};
                for (int bx = 0; bx < nbox; bx++)
                    for (int q = 0; q < 3; q++) {
                        int v = R.img[q][bx];
                        int lo = q + 1 == R.t_nd ? (R.t_lr < 0 ? 1 : tdims[q]) : 1;
                        if (v < lo || v > tdims[q] || (q + 1 == R.t_nd && v != lo)) {
                            set_err("interface image outside the target face");
                            return WCNS_ERR_ARGUMENT;
                        }
                    }
                if (dims[R.s_nd - 1] < 4 || tdims[R.t_nd - 1] < 4) {
                    set_err("interface needs at least 4 points normal to the face");
                    return WCNS_ERR_ARGUMENT;
                }
            } else if (R.bctype < 2 || R.bctype > 6) {
                set_err("unsupported BC type " + std::to_string(R.bctype) + " (supported: -1,2,3,4,5,6)");
                return WCNS_ERR_UNSUPPORTED;
            }
        }
        static const int order[6] = {-1, 4, 5, 6, 2, 3};
        B.bcindex.clear();
        for (int l = 0; l < 6; l++)
            for (int r = 0; r < (int)B.regs.size(); r++) {
                int t = B.regs[r].bctype < 0 ? -1 : B.regs[r].bctype;
                if (t == order[l]) B.bcindex.push_back(r);
            }
    }
    return 0;
}

// ---------------------------------------------------------------------------
static void free_owned(WcnsContext *c, void *p) {
    if (!p) return;
    c->owned.erase(std::remove(c->owned.begin(), c->owned.end(), p), c->owned.end());
    cudaFree(p);
}

// The wide cooperative sweeps' chunks and arrays (and the SA model's when it
// is set up); L.wide points to them.  -1: the blocks cannot be swept wide;
// a CUDA error code when an allocation fails.
static int wide_alloc(WcnsContext *c) {
    LaunchCtx &L = c->L;
    if (c->wide) {
        L.wide = c->wide.get();
        return 0;
    }
    auto W = std::make_unique<WideSweep>();
    if (setup_sweep_wide(L, *W) != 0) return -1;
    WideArrays &A = W->A;
    const size_t words = (size_t)(WIDE_COEF_WORDS + 5 + 5 + 15 + 5) * A.n + 8;
    CK(cudaMalloc(&A.stat, sizeof(double) * words));
    c->owned.push_back(A.stat);
    A.rhs = A.stat + (size_t)WIDE_COEF_WORDS * A.n;
    A.dql = A.rhs + (size_t)5 * A.n;
    A.gs1 = A.dql + (size_t)5 * A.n;
    A.gs2 = A.gs1 + (size_t)15 * A.n;
    CK(cudaMalloc(&A.ring, sizeof(double) * (size_t)std::max(1, A.nbnd) * 8 * A.nkmax * 10));
    c->owned.push_back(A.ring);
    CK(cudaMalloc(&A.flags, sizeof(unsigned) * 2 * (size_t)std::max(1, A.nbnd)));
    c->owned.push_back(A.flags);
    if (c->sa_pool) {  // the model's scalar sweeps run on the wide chunks too
        CK(cudaMalloc(&A.sa, sizeof(double) * (6 * (size_t)A.n + 8)));
        c->owned.push_back(A.sa);
    }
    W->chunks = c->up(W->hchunks);
    c->wide = std::move(W);
    L.wide = c->wide.get();
    return 0;
}

static void wide_free(WcnsContext *c) {
    if (!c->wide) return;
    WideSweep &W = *c->wide;
    free_owned(c, W.A.stat);
    free_owned(c, W.A.ring);
    free_owned(c, W.A.flags);
    free_owned(c, W.A.sa);
    free_owned(c, W.chunks);
    c->wide.reset();
    c->L.wide = nullptr;
}

// Line groups of the residual kernels for every direction (passes 2 and 3:
// the mixed-precision kernels): at most inv_cap / vis_cap lines of a block
// per CTA, fewer where the staged lines would pass 72 KB of shared memory.
static int build_line_tables(WcnsContext *c, int inv_cap, int vis_cap) {
    LaunchCtx &L = c->L;
    const int nbk = (int)c->blk.size();
    size_t inv_smem = 0, vis_smem = 0, inv_mx_smem = 0, vis_mx_smem = 0;
    for (int dir = 0; dir < 3; dir++) {
        for (int pass = 0; pass < 4; pass++) {  // 0 inviscid, 1 viscous, 2 and 3 the same in mixed precision
            std::vector<LineGroup> g;
            int nl_max = 0, hmax = 0;
            size_t sm_dir = 0;
            for (int b = 0; b < nbk; b++) {
                const DevBlock &D = c->blk[b].d;
                int n = dimof(D, dir);
                if ((pass == 0 || pass == 2) && n <= NIJK2D) continue;
                int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
                int na = dimof(D, a1), nb2 = dimof(D, a2);
                size_t per_line = pass == 0 ? rhs_invis_line_bytes(n) : pass == 1 ? rhs_vis_line_bytes(n)
                                : pass == 2 ? rhs_invis_mx_line_bytes(n) : rhs_vis_mx_line_bytes(n);
                // staged lines per CTA: at most 54 KB for the FP64 inviscid kernel (four
                // 256-thread CTAs of 64 registers per SM), 108 KB for the FP64 viscous
                // kernel (two 320-thread CTAs of 96 registers), 72 KB for the
                // mixed-precision kernels
                int NL = pass == 0 ? std::max(1, std::min({std::min(inv_cap, rhs_invis_max_lines()), 3072 / (5 * (n + 2)),
                                                           (int)((54 * 1024) / per_line)}))
                       : pass == 1 ? std::max(1, std::min({std::min(vis_cap, rhs_vis_max_lines()), 512 / (n + 1), (int)((108 * 1024) / per_line)}))
                       : pass == 2 ? std::max(1, std::min({std::min(inv_cap, rhs_invis_mx_max_lines()), 3072 / (5 * (n + 2)),
                                                           (int)((72 * 1024) / per_line)}))
                                   : std::max(1, std::min({std::min(vis_cap, rhs_vis_mx_max_lines()), 512 / (n + 1), (int)((72 * 1024) / per_line)}));
                if (pass == 1) {
                    // the FP64 viscous kernel's heavy phase has one item per (line, half
                    // node): of NL/2..NL lines take the count whose items fill the last
                    // pass of the CTA's threads best, so that few threads idle at the
                    // barrier after it (3.29 -> 3.11 ms per channel step with the larger
                    // staging limit)
                    const int thr = rhs_vis_threads();
                    int best = NL;
                    double best_fill = 0.0;
                    for (int q = NL; q >= std::max(1, (NL + 1) / 2); q--) {
                        const int items = q * (n + 1), rounds = (items + thr - 1) / thr;
                        const double fill = (double)items / ((double)rounds * thr);
                        if (fill > best_fill + 1e-9) {
                            best_fill = fill;
                            best = q;
                        }
                    }
                    NL = best;
                }
                for (int bb = 1; bb <= nb2; bb++)
                    for (int a = 1; a <= na; a += NL) {
                        LineGroup lg{b, a, bb, std::min(NL, na - a + 1)};
                        g.push_back(lg);
                        nl_max = std::max(nl_max, lg.nl);
                        sm_dir = std::max(sm_dir, per_line * lg.nl);
                    }
                hmax = std::max(hmax, n + 1);
            }
            DirTable &T = pass == 0 ? L.inv[dir] : pass == 1 ? L.vis[dir] : pass == 2 ? L.inv_mx[dir] : L.vis_mx[dir];
            T.ngroups = (int)g.size();
            T.nl_max = nl_max;
            T.hmax = hmax;
            T.smem = sm_dir;
            if (T.groups) {  // a rebuild (wcns_set_shape): the old table goes
                c->owned.erase(std::remove(c->owned.begin(), c->owned.end(), (void *)T.groups), c->owned.end());
                cudaFree(T.groups);
            }
            T.groups = c->up(g);
            size_t sm = sm_dir;
            size_t &acc = pass == 0 ? inv_smem : pass == 1 ? vis_smem : pass == 2 ? inv_mx_smem : vis_mx_smem;
            acc = std::max(acc, sm);
        }
    }
    if (inv_smem > 227 * 1024 || vis_smem > 227 * 1024) { set_err("line too long for shared memory"); return WCNS_ERR_ARGUMENT; }
    setup_rhs_invis_attrs(std::max<size_t>(inv_smem, 48 * 1024));
    setup_rhs_vis_attrs(std::max<size_t>(vis_smem, 48 * 1024));
    if (inv_mx_smem > 227 * 1024 || vis_mx_smem > 227 * 1024) { set_err("line too long for shared memory"); return WCNS_ERR_ARGUMENT; }
    setup_rhs_mx_attrs(std::max<size_t>(inv_mx_smem, 48 * 1024), std::max<size_t>(vis_mx_smem, 48 * 1024));
    L.inv_cap = inv_cap;
    L.vis_cap = vis_cap;
    return 0;
}

static int build_tables(WcnsContext *c) {
    const int nbk = (int)c->blk.size();
    LaunchCtx &L = c->L;
    // interface ghost copies
    std::vector<GhostCopy> ghost;
    for (int b = 0; b < nbk; b++)
        for (const HReg &R : c->blk[b].regs) {
            if (R.bctype >= 0) continue;
            for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                    for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                        int bx = R.box(i, j, k);
                        for (int l = 1; l <= 3; l++) {
                            GhostCopy g;
                            g.dst = c->gi(b + 1, i + l * R.s_lr3d[0], j + l * R.s_lr3d[1], k + l * R.s_lr3d[2]);
                            g.src = c->gi(R.nbt, R.img[0][bx] - l * R.t_lr3d[0], R.img[1][bx] - l * R.t_lr3d[1],
                                          R.img[2][bx] - l * R.t_lr3d[2]);
                            ghost.push_back(g);
                        }
                    }
        }
    L.nghost = (long long)ghost.size();
    L.ghost = c->up(ghost);
    // physical regions in bcindex order, dq-zero points
    std::vector<DevRegion> regs;
    std::vector<int> first(nbk + 1, 0);
    std::vector<long long> zero, sa_src;
    for (int b = 0; b < nbk; b++) {
        first[b] = (int)regs.size();
        for (int r : c->blk[b].bcindex) {
            const HReg &R = c->blk[b].regs[r];
            DevRegion d{};
            d.blk = b;
            d.bctype = R.bctype < 0 ? -1 : R.bctype;
            for (int m = 0; m < 3; m++) { d.s_st[m] = R.s_st[m]; d.s_ed[m] = R.s_ed[m]; d.s_lr3d[m] = R.s_lr3d[m]; }
            d.s_nd = R.s_nd;
            d.s_lr = R.s_lr;
            if (R.bctype < 0) {
                // the SA interface rule reads the partner's first interior
                // point behind the image point (parallel.f90:2763-2766)
                d.same = R.nbt == b + 1 ? 1 : 0;
                d.sa_first = (long long)sa_src.size();
                for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                    for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                        for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                            int bx = R.box(i, j, k);
                            sa_src.push_back(c->gi(R.nbt, R.img[0][bx] - R.t_lr3d[0], R.img[1][bx] - R.t_lr3d[1],
                                                   R.img[2][bx] - R.t_lr3d[2]));
                        }
            }
            regs.push_back(d);
        }
        for (const HReg &R : c->blk[b].regs) {
            if (R.bctype <= 0) continue;
            for (int i = R.s_st[0]; i <= R.s_ed[0]; i++)
                for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                    for (int k = R.s_st[2]; k <= R.s_ed[2]; k++) zero.push_back(c->gi(b + 1, i, j, k));
        }
    }
    first[nbk] = (int)regs.size();
    L.regions = c->up(regs);
    L.reg_first = c->up(first);
    L.nsa_if = (long long)sa_src.size();
    L.sa_if_src = c->up(sa_src);
    if (L.nsa_if) {
        CK(cudaMalloc(&L.sa_if_snap, sizeof(double) * 2 * (size_t)L.nsa_if));
        c->owned.push_back(L.sa_if_snap);
    }
    L.nzero = (long long)zero.size();
    L.zero_pts = c->up(zero);
    // interface averaging: snapshot slots, pairs per region (region order)
    std::unordered_map<long long, int> slot;
    std::vector<long long> snap_pts;
    auto slot_of = [&](long long id) {
        auto it = slot.find(id);
        if (it != slot.end()) return it->second;
        int s = (int)snap_pts.size();
        slot[id] = s;
        snap_pts.push_back(id);
        return s;
    };
    // The reference averages a block's interface points sequentially, region
    // by region (boundary_match_dq_2pm / boundary_match_pv_2pm).  Each pair
    // goes to the earliest group (level) after every earlier pair that wrote
    // its point, wrote the in-block partner it reads, or read its point as a
    // partner; the pairs of one level are then independent, and running the
    // levels in order gives the sequential result.
    std::vector<PairEntry> pairs;
    std::vector<int> reg_pair_first, blk_reg_first(nbk + 1, 0);
    for (int b = 0; b < nbk; b++) {
        blk_reg_first[b] = (int)reg_pair_first.size();
        std::vector<PairEntry> seq;  // the block's pairs in reference order
        for (const HReg &R : c->blk[b].regs) {
            if (R.bctype >= 0) continue;
            for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                    for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                        int bx = R.box(i, j, k);
                        PairEntry e;
                        e.own = c->gi(b + 1, i, j, k);
                        e.partner = c->gi(R.nbt, R.img[0][bx], R.img[1][bx], R.img[2][bx]);
                        slot_of(e.own);
                        e.partner_slot = slot_of(e.partner);
                        e.same = (R.nbt == b + 1) ? 1 : 0;
                        seq.push_back(e);
                    }
        }
        std::unordered_map<long long, int> last_write, last_read;
        std::vector<int> level(seq.size());
        int nlev = 0;
        for (size_t a = 0; a < seq.size(); a++) {
            const PairEntry &e = seq[a];
            int lv = 0;
            auto after = [&](const std::unordered_map<long long, int> &mp, long long id) {
                auto it = mp.find(id);
                if (it != mp.end()) lv = std::max(lv, it->second + 1);
            };
            after(last_write, e.own);
            after(last_read, e.own);
            if (e.same) after(last_write, e.partner);
            level[a] = lv;
            last_write[e.own] = lv;
            if (e.same) {
                auto it = last_read.find(e.partner);
                last_read[e.partner] = it == last_read.end() ? lv : std::max(it->second, lv);
            }
            nlev = std::max(nlev, lv + 1);
        }
        for (int lv = 0; lv < nlev; lv++) {
            reg_pair_first.push_back((int)pairs.size());
            for (size_t a = 0; a < seq.size(); a++)
                if (level[a] == lv) pairs.push_back(seq[a]);
        }
    }
    blk_reg_first[nbk] = (int)reg_pair_first.size();
    reg_pair_first.push_back((int)pairs.size());
    L.nsnap = (int)snap_pts.size();
    L.snap_pts = c->up(snap_pts);
    L.pairs = c->up(pairs);
    L.reg_pair_first = c->up(reg_pair_first);
    L.blk_reg_first = c->up(blk_reg_first);
    if (L.nsnap) {
        CK(cudaMalloc(&L.snap, sizeof(double) * 6 * L.nsnap));
        c->owned.push_back(L.snap);
    }
    // multi-point sets: connect_pre_parallel + comp_list_insert
    for (auto &B : c->blk)
        for (auto &R : B.regs) R.iused = 0;
    for (int b = 0; b < nbk; b++)
        for (auto &R : c->blk[b].regs) {
            if (R.bctype < 0 && R.iused == 0) {
                R.iused = 1;
                HBlock &T = c->blk[R.nbt - 1];
                if (R.ibcwin >= 1 && R.ibcwin <= (int)T.regs.size()) T.regs[R.ibcwin - 1].iused = -1;
            }
        }
    std::vector<std::vector<long long>> comps;  // members as field indices, list order
    for (int b = 0; b < nbk; b++)
        for (auto &R : c->blk[b].regs) {
            if (R.bctype >= 0 || R.iused != 1) continue;
            static const int mcyc[5] = {1, 2, 3, 1, 2};
            int d2 = mcyc[R.s_nd] - 1, d3 = mcyc[R.s_nd + 1] - 1;
            for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                    for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                        int cc[3] = {i, j, k};
                        bool inner = cc[d2] >= R.s_st[d2] + 1 && cc[d2] <= R.s_ed[d2] - 1 && cc[d3] >= R.s_st[d3] + 1 &&
                                     cc[d3] <= R.s_ed[d3] - 1;
                        if (inner) continue;
                        int bx = R.box(i, j, k);
                        long long a = c->gi(b + 1, i, j, k);
                        long long t = c->gi(R.nbt, R.img[0][bx], R.img[1][bx], R.img[2][bx]);
                        bool ok = false;
                        for (auto &cl : comps) {
                            bool ea = std::find(cl.begin(), cl.end(), a) != cl.end();
                            bool et = std::find(cl.begin(), cl.end(), t) != cl.end();
                            if (ea || et) {
                                if (!ea) cl.push_back(a);
                                if (!et) cl.push_back(t);
                                ok = true;
                                break;
                            }
                        }
                        if (!ok) comps.push_back({a, t});
                    }
        }
    std::vector<int> comp_first, comp_n, mem_slot, mem_comp;
    std::vector<long long> mem_idx;
    for (auto &cl : comps) {
        if (cl.size() <= 2) continue;
        int cid = (int)comp_first.size();
        comp_first.push_back((int)mem_idx.size());
        comp_n.push_back((int)cl.size());
        for (long long id : cl) {
            mem_idx.push_back(id);
            mem_slot.push_back(slot_of(id));
            mem_comp.push_back(cid);
        }
    }
    if ((int)snap_pts.size() != L.nsnap) { set_err("internal: snapshot list grew"); return WCNS_ERR_ARGUMENT; }
    c->nmulti = (int)comp_first.size();
    L.ncomp = (int)comp_first.size();
    L.nmem = (int)mem_idx.size();
    L.comp_first = c->up(comp_first);
    L.comp_n = c->up(comp_n);
    L.mem_slot = c->up(mem_slot);
    // the members' writes grouped by the block that owns the point (the
    // block's cluster writes them after its two-block pairs)
    {
        std::vector<int> wr_comp, blk_wr_first(nbk + 1, 0);
        std::vector<long long> wr_idx;
        for (int b = 0; b < nbk; b++) {
            blk_wr_first[b] = (int)wr_idx.size();
            const long long lo = c->blk[b].d.off, hi = lo + (long long)c->blk[b].d.gx * c->blk[b].d.gy * c->blk[b].d.gz;
            for (size_t e = 0; e < mem_idx.size(); e++)
                if (mem_idx[e] >= lo && mem_idx[e] < hi) {
                    wr_comp.push_back(mem_comp[e]);
                    wr_idx.push_back(mem_idx[e]);
                }
        }
        blk_wr_first[nbk] = (int)wr_idx.size();
        if (wr_idx.size() != mem_idx.size()) { set_err("internal: a multi-block point outside every block"); return WCNS_ERR_ARGUMENT; }
        L.mem_comp = c->up(wr_comp);
        L.mem_idx = c->up(wr_idx);
        L.blk_mem_first = c->up(blk_wr_first);
    }
    if (int rc = build_line_tables(c, INV_LINES_DEFAULT, VIS_LINES_DEFAULT)) return rc;
    // LU-SGS sweep shape; WCNS_SWEEP_CLUSTER (CTAs per block) and WCNS_SWEEP_FINE (0: three
    // threads per column) override it for tuning
    {
        int cl = 16, fine = 1;
        if (const char *e = getenv("WCNS_SWEEP_CLUSTER")) cl = atoi(e);
        if (const char *e = getenv("WCNS_SWEEP_FINE")) fine = atoi(e);
        // blocks whose columns do not fit the clustered kernel run the wide
        // cooperative sweeps, or, when those do not fit either, sweep plane by plane
        const bool want_plane = c->prm.flags & WCNS_FLAG_SWEEP_BY_PLANE, want_wide = c->prm.flags & WCNS_FLAG_SWEEP_WIDE;
        const bool clustered = !want_plane && !want_wide && setup_sweep(L, cl, fine) == 0;
        if (!clustered && !want_plane)
            if (int rc = wide_alloc(c); rc > 0) return rc;
        L.sweep_plane = !clustered && !L.wide ? 1 : 0;
    }
    // residual partials, update bad lists
    L.res_ctas_per_block = 32;
    if (setup_residual(nbk, L.res_ctas_per_block)) { set_err("too many blocks for the residual reduction (at most 400)"); return WCNS_ERR_ARGUMENT; }
    CK(cudaMalloc(&L.res_partial, sizeof(double) * 2 * 32 * nbk));
    c->owned.push_back(L.res_partial);
    CK(cudaMalloc(&L.res_out, sizeof(double) * (2 * nbk + 1)));
    c->owned.push_back(L.res_out);
    CK(cudaMalloc(&L.bad_count, sizeof(int) * nbk));
    c->owned.push_back(L.bad_count);
    CK(cudaMemset(L.bad_count, 0, sizeof(int) * nbk));
    CK(cudaMalloc(&L.bad_list, sizeof(long long) * BAD_CAP * nbk));
    c->owned.push_back(L.bad_list);
    return 0;
}

static int check_errors(WcnsContext *c) {
    int h[ERR_NSLOTS];
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(h, c->d_err, sizeof h, cudaMemcpyDeviceToHost));
    CK(cudaMemset(c->d_err, 0, sizeof h));
    if (h[ERR_ROE]) {
        set_err(std::string(c->P.nflux == 2 ? "flux_vanleer: c^2 < 0" : "flux_Roe: c^2 <= 0") + " at " +
                std::to_string(h[ERR_ROE]) + " half-node states");
        return WCNS_ERR_ROE;
    }
    if (h[ERR_UPDATE_BLOCKS]) { set_err("update_limited: too many non-physical points"); return WCNS_ERR_UPDATE; }
    if (h[ERR_TIMEOUT]) { set_err("LU-SGS sweep: a bounded wait for a plane's coefficients ran out"); return WCNS_ERR_CUDA; }
    return 0;
}

// The Mach-dependent free-stream constants of init_inflow (PreProcess.f90:
// 968-1113) and read_perfect_gasmodel (GasModel.f90:184-217) for one block,
// evaluated as the context does for its common Mach number.
static void set_block_freestream(DevBlock &d, const DevParams &P, double moo) {
    d.moo2 = moo * moo;
    d.moocp = moo * moo * P.gama;
    d.poo = 1.0 / (P.gama * moo * moo);
    d.coo = sqrt(P.gama * d.poo / P.roo);
    const double cp = 1.0 / ((P.gama - 1.0) * moo * moo);
    d.cp_prl = cp / 0.72;
    d.cp_prt = cp / 0.90;
}

// ---------------------------------------------------------------------------
extern "C" int wcns_create(const WcnsParams *prm, int nblocks, const int *dims, const double *const *xyz, int nregions,
                           const int *regions, WcnsContext **out) {
    if (!prm || nblocks < 1 || !dims || !xyz || !out || (nregions > 0 && !regions)) {
        set_err("wcns_create: invalid argument");
        return WCNS_ERR_ARGUMENT;
    }
    if (prm->nscheme != 4 && prm->nscheme != 41 && prm->nscheme != 42) { set_err("nscheme must be 4, 41 or 42"); return WCNS_ERR_UNSUPPORTED; }
    if (prm->nflux < 1 || prm->nflux > 3) { set_err("nflux must be 1 (Steger-Warming), 2 (Van Leer) or 3 (Roe)"); return WCNS_ERR_UNSUPPORTED; }
    if (prm->nvis != 0 && prm->nvis != 1) { set_err("nvis must be 0 or 1"); return WCNS_ERR_ARGUMENT; }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_err("no CUDA device"); return WCNS_ERR_CUDA; }
    WcnsContext *c = new WcnsContext();
    c->prm = *prm;
    // derived constants (init_inflow PreProcess.f90:968-1113; read_perfect_gasmodel GasModel.f90:184-217)
    const double PAI = 3.14159265;
    DevParams &P = c->P;
    P.gama = 1.40;
    P.g1 = P.gama / (P.gama - 1.0);
    P.moo = prm->moo;
    P.moo2 = prm->moo * prm->moo;
    P.moocp = prm->moo * prm->moo * P.gama;
    P.reynolds = (prm->reynolds / 1.0) * 1.0;
    P.re = 1.0 / P.reynolds;
    P.visc = 110.4 / prm->tref;
    double cp = 1.0 / ((P.gama - 1.0) * prm->moo * prm->moo);
    P.cp_prl = cp / 0.72;
    P.cp_prt = cp / 0.90;
    P.cc23 = 2.0 / 3.0;
    P.cfl = prm->cfl;
    P.timedt_rate = prm->timedt_rate;
    P.efix = prm->efix;
    P.csrv = prm->csrv;
    double attack = prm->attack * PAI / 180.0, sideslip = prm->sideslip * PAI / 180.0;
    P.uoo = cos(attack) * cos(sideslip);
    P.voo = sin(attack) * cos(sideslip);
    P.woo = sin(sideslip);
    P.roo = 1.0;
    P.poo = 1.0 / (P.gama * prm->moo * prm->moo);
    P.coo = sqrt(P.gama * P.poo / P.roo);
    P.twall_nd = prm->twall / prm->tref;
    P.nvis = prm->nvis;
    P.nscheme = prm->nscheme;
    P.nflux = prm->nflux;
    P.adiabatic = prm->twall > 0.0 ? 0 : 1;
    // blocks
    c->blk.resize(nblocks);
    long long off = 0;
    for (int b = 0; b < nblocks; b++) {
        DevBlock &d = c->blk[b].d;
        d.ni = dims[3 * b];
        d.nj = dims[3 * b + 1];
        d.nk = dims[3 * b + 2];
        if (d.ni < 2 || d.nj < 2 || d.nk < 2) { delete c; set_err("block dimensions must be >= 2"); return WCNS_ERR_ARGUMENT; }
        d.gx = d.ni + 6;
        d.gy = d.nj + 6;
        d.gz = d.nk + 6;
        d.off = off;
        d.npts = (long long)d.ni * d.nj * d.nk;
        d.pmoff = c->total_pm;
        set_block_freestream(d, P, prm->moo);
        c->total_pm += (long long)(d.ni + d.nj + d.nk - 2) * d.nj * d.nk;
        c->total_pm = (c->total_pm + 31) / 32 * 32;
        off += (long long)d.gx * d.gy * d.gz;
        off = (off + 31) / 32 * 32;
    }
    c->total = off;
    for (int r = 0; r < nregions; r++) {
        const int *rr = regions + 16 * r;
        if (rr[0] < 1 || rr[0] > nblocks) { delete c; set_err("BC region block number out of range"); return WCNS_ERR_ARGUMENT; }
        HReg R;
        for (int m = 0; m < 3; m++) {
            R.raw_s_st[m] = rr[1 + 2 * m];
            R.raw_s_ed[m] = rr[2 + 2 * m];
            R.raw_t_st[m] = rr[8 + 2 * m];
            R.raw_t_ed[m] = rr[9 + 2 * m];
        }
        R.bctype = rr[7];
        R.nbt = rr[14];
        R.ibcwin = rr[15];
        c->blk[rr[0] - 1].regs.push_back(R);
    }
    int rc = analyze(c);
    if (rc) { delete c; return rc; }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        set_err("cudaStreamCreate failed");
        return WCNS_ERR_CUDA;
    }
    // field pool
    size_t bytes = sizeof(double) * (size_t)F_NPOOL * (size_t)c->total;
    if (cudaMalloc(&c->pool, bytes) != cudaSuccess) { delete c; set_err("device allocation of the field pool failed"); return WCNS_ERR_CUDA; }
    cudaMemset(c->pool, 0, bytes);
    for (int f = 0; f < F_NPOOL; f++) c->F.f[f] = c->pool + (size_t)f * c->total;
    c->F.f[F_VIST] = nullptr;
    std::vector<DevBlock> hb(nblocks);
    for (int b = 0; b < nblocks; b++) hb[b] = c->blk[b].d;
    LaunchCtx &L = c->L;
    L.stream = c->stream;
    L.total = c->total;
    for (int q = 0; q < 2; q++) {
        if (cudaStreamCreateWithFlags(&L.side[q], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.ev_join[q], cudaEventDisableTiming) != cudaSuccess) {
            delete c;
            set_err("stream/event creation failed");
            return WCNS_ERR_CUDA;
        }
    }
    if (cudaEventCreateWithFlags(&L.ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&L.contrib, sizeof(double) * 10 * (size_t)c->total) != cudaSuccess) {
        delete c;
        set_err("allocation of the residual contribution buffers failed");
        return WCNS_ERR_CUDA;
    }
    c->owned.push_back(L.contrib);
    L.P = &c->P;
    L.F = &c->F;
    L.PM = &c->PM;
    L.nblocks = nblocks;
    L.blocks = c->up(hb);
    {
        auto *hbl = new DevBlock[nblocks];
        for (int b = 0; b < nblocks; b++) hbl[b] = hb[b];
        L.hblocks = hbl;
    }
    rc = build_tables(c);
    if (rc) { delete c; return rc; }
    if (!L.sweep_plane && !L.wide) {
        // sweep arrays, plane-major: dq (5 planes of values), the static records
        // (SR_N per cell) and three dynamic records (DYN_N per cell); the memset
        // leaves zero the records that no kernel ever writes
        size_t pmbytes = sizeof(double) * (size_t)(5 + SR_N + 3 * DYN_N) * (size_t)c->total_pm;
        if (cudaMalloc(&c->pm_pool, pmbytes) != cudaSuccess) { delete c; set_err("device allocation of the sweep arrays failed"); return WCNS_ERR_CUDA; }
        cudaMemset(c->pm_pool, 0, pmbytes);
        for (int m = 0; m < 5; m++) c->PM.dq[m] = c->pm_pool + (size_t)m * c->total_pm;
        c->PM.dq_stride = c->total_pm;
        c->PM.stat = c->pm_pool + (size_t)5 * c->total_pm;
        c->PM.dyn = c->PM.stat + (size_t)SR_N * c->total_pm;
        c->PM.gs[0] = c->PM.dyn + (size_t)DYN_N * c->total_pm;
        c->PM.gs[1] = c->PM.gs[0] + (size_t)DYN_N * c->total_pm;
    }
    c->PM.csize = L.sweep_cluster;
    CK(cudaMalloc(&c->d_err, sizeof(int) * ERR_NSLOTS));
    c->owned.push_back(c->d_err);
    CK(cudaMemset(c->d_err, 0, sizeof(int) * ERR_NSLOTS));
    L.err = c->d_err;
    // grid metrics on the device
    double *xyzd = nullptr, *work = nullptr;
    CK(cudaMalloc(&xyzd, sizeof(double) * 3 * (size_t)c->total));
    CK(cudaMalloc(&work, sizeof(double) * 13 * (size_t)c->total));
    cudaMemset(xyzd, 0, sizeof(double) * 3 * (size_t)c->total);
    std::vector<double> tmp;
    for (int b = 0; b < nblocks; b++) {
        const DevBlock &d = hb[b];
        tmp.assign((size_t)d.gx * d.gy * d.gz, 0.0);
        for (int q = 0; q < 3; q++) {
            const double *src = xyz[3 * b + q];
            if (!src) { set_err("missing coordinates"); cudaFree(xyzd); cudaFree(work); delete c; return WCNS_ERR_ARGUMENT; }
            for (int k = 1; k <= d.nk; k++)
                for (int j = 1; j <= d.nj; j++)
                    for (int i = 1; i <= d.ni; i++)
                        tmp[gidx(d, i, j, k) - d.off] = src[(i - 1) + (size_t)d.ni * ((j - 1) + (size_t)d.nj * (k - 1))];
            if (cudaMemcpy(xyzd + (size_t)q * c->total + d.off, tmp.data(), sizeof(double) * tmp.size(),
                           cudaMemcpyHostToDevice) != cudaSuccess) {
                set_err("wcns_create: copy of the coordinates to the device failed");
                cudaFree(xyzd);
                cudaFree(work);
                delete c;
                return WCNS_ERR_CUDA;
            }
        }
    }
    double *xyzp[3] = {xyzd, xyzd + c->total, xyzd + 2 * c->total};
    launch_metrics(L, xyzp, work);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(xyzd);
    cudaFree(work);
    if (e != cudaSuccess) { set_err(std::string("metrics: ") + cudaGetErrorString(e)); delete c; return WCNS_ERR_CUDA; }
    // wall regions for the force integration, in block and region order
    {
        std::vector<DevWall> walls;
        std::vector<double> wxyz;
        long long npt = 0, nq = 0;
        for (int b = 0; b < nblocks; b++)
            for (const HReg &R : c->blk[b].regs) {
                if (!(R.bctype == 2 || R.bctype / 10 == 2)) continue;
                DevWall W{};
                W.blk = b;
                int nqr = 1;
                for (int m = 0; m < 3; m++) {
                    W.s_st[m] = R.s_st[m];
                    W.e[m] = R.s_ed[m] - R.s_st[m] + 1;
                    W.s_lr3d[m] = R.s_lr3d[m];
                    nqr *= W.e[m] - (1 - std::abs(R.s_lr3d[m]));
                }
                W.s_lr = R.s_lr;
                W.pt_off = npt;
                W.quad_off = nq;
                W.nquad = nqr;
                const int ni = c->blk[b].d.ni, nj = c->blk[b].d.nj;
                for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                    for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                        for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                            size_t g = (size_t)(i - 1) + (size_t)ni * ((size_t)(j - 1) + (size_t)nj * (k - 1));
                            for (int q = 0; q < 3; q++) wxyz.push_back(xyz[3 * b + q][g]);
                        }
                npt += (long long)W.e[0] * W.e[1] * W.e[2];
                nq += nqr;
                walls.push_back(W);
            }
        L.nwall = (int)walls.size();
        L.nwall_quads = nq;
        c->hwalls = walls;
        if (L.nwall) {
            L.walls = c->up(walls);
            L.wall_xyz = c->up(wxyz);
            CK(cudaMalloc(&L.wall_pf, sizeof(double) * 3 * (size_t)npt));
            c->owned.push_back(L.wall_pf);
            CK(cudaMalloc(&L.wall_quad, sizeof(double) * 6 * (size_t)std::max(nq, 1LL)));
            c->owned.push_back(L.wall_quad);
            CK(cudaMalloc(&L.wall_out, sizeof(double) * 6));
            c->owned.push_back(L.wall_out);
        }
    }
    *out = c;
    return 0;
}

extern "C" void wcns_destroy(WcnsContext *c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    delete[] c->L.hblocks;
    delete c;
}

static int block_range(WcnsContext *c, int nb, const DevBlock **d) {
    if (!c || nb < 1 || nb > (int)c->blk.size()) { set_err("block number out of range"); return WCNS_ERR_ARGUMENT; }
    *d = &c->blk[nb - 1].d;
    return 0;
}

extern "C" int wcns_set_prim(WcnsContext *c, int nb, const double *r, const double *u, const double *v, const double *w,
                             const double *p, const double *t) {
    const DevBlock *d;
    if (int rc = block_range(c, nb, &d)) return rc;
    const double *src[6] = {r, u, v, w, p, t};
    size_t n = (size_t)d->gx * d->gy * d->gz;
    for (int f = 0; f < 6; f++) {
        if (!src[f]) { set_err("wcns_set_prim: null array"); return WCNS_ERR_ARGUMENT; }
        CK(cudaMemcpyAsync(c->F.f[F_R + f] + d->off, src[f], sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// device base of a public field: the path's fields, and the SA model's
// qke, vist and wall distance once wcns_sa_setup has run
static double *field_base(WcnsContext *c, int field) {
    if (field >= 0 && field <= WCNS_F_VOL) return c->F.f[field];
    if (!c->sa_pool) return nullptr;
    if (field == WCNS_F_QKE) return c->SA.qke;
    if (field == WCNS_F_VIST) return c->SA.vist;
    if (field == WCNS_F_DIST) return c->SA.dist;
    return nullptr;
}

extern "C" int wcns_get_field(WcnsContext *c, int field, int nb, double *out) {
    const DevBlock *d;
    if (int rc = block_range(c, nb, &d)) return rc;
    double *base = field_base(c, field);
    if (!base || !out) { set_err("wcns_get_field: unsupported field"); return WCNS_ERR_UNSUPPORTED; }
    size_t n = (size_t)d->gx * d->gy * d->gz;
    CK(cudaMemcpyAsync(out, base + d->off, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// Device address of block nb's ghosted slice of a public field and its
// element count; the caller synchronises with the context's stream
// (wcns_sync) before reading or writing through it.
extern "C" int wcns_field_device_ptr(WcnsContext *c, int field, int nb, void **ptr, long long *count) {
    const DevBlock *d;
    if (int rc = block_range(c, nb, &d)) return rc;
    double *base = field_base(c, field);
    if (!base || !ptr || !count) { set_err("wcns_field_device_ptr: unsupported field or null output"); return WCNS_ERR_UNSUPPORTED; }
    *ptr = base + d->off;
    *count = (long long)d->gx * d->gy * d->gz;
    return 0;
}

extern "C" int wcns_get_prim(WcnsContext *c, int nb, double *r, double *u, double *v, double *w, double *p, double *t) {
    const DevBlock *d;
    if (int rc = block_range(c, nb, &d)) return rc;
    double *dst[6] = {r, u, v, w, p, t};
    for (int f = 0; f < 5; f++)
        if (!dst[f]) { set_err("wcns_get_prim: null array"); return WCNS_ERR_ARGUMENT; }
    size_t n = (size_t)d->gx * d->gy * d->gz;
    for (int f = 0; f < 6; f++)
        if (dst[f]) CK(cudaMemcpyAsync(dst[f], c->F.f[F_R + f] + d->off, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// All blocks at once: the copies of every block go into the stream and the
// call synchronises once (the per-block loop of the reference's set-up and
// flow-file write).  prim: 6 pointers per block, r u v w p t.
extern "C" int wcns_set_prim_all(WcnsContext *c, const double *const *prim) {
    if (!c || !prim) { set_err("wcns_set_prim_all: null argument"); return WCNS_ERR_ARGUMENT; }
    const int nbk = (int)c->blk.size();
    for (int e = 0; e < 6 * nbk; e++)
        if (!prim[e]) { set_err("wcns_set_prim_all: null array"); return WCNS_ERR_ARGUMENT; }
    // the copies are spread over the context's three streams so that their
    // set-up overlaps, after the work already queued on the context's stream;
    // the call returns once all have landed
    CK(cudaEventRecord(c->L.ev_fork, c->stream));
    cudaStream_t st[3] = {c->stream, c->L.side[0], c->L.side[1]};
    for (int q = 1; q < 3; q++) CK(cudaStreamWaitEvent(st[q], c->L.ev_fork, 0));
    int e = 0;
    for (int b = 0; b < nbk; b++) {
        const DevBlock &d = c->blk[b].d;
        const size_t n = (size_t)d.gx * d.gy * d.gz;
        for (int f = 0; f < 6; f++, e++)
            CK(cudaMemcpyAsync(c->F.f[F_R + f] + d.off, prim[6 * b + f], sizeof(double) * n, cudaMemcpyHostToDevice,
                               st[e % 3]));
    }
    for (int q = 0; q < 3; q++) CK(cudaStreamSynchronize(st[q]));
    return 0;
}

// prim: 6 pointers per block, r u v w p t; a null t skips T of that block.
extern "C" int wcns_get_prim_all(WcnsContext *c, double *const *prim) {
    if (!c || !prim) { set_err("wcns_get_prim_all: null argument"); return WCNS_ERR_ARGUMENT; }
    const int nbk = (int)c->blk.size();
    for (int b = 0; b < nbk; b++)
        for (int f = 0; f < 5; f++)
            if (!prim[6 * b + f]) { set_err("wcns_get_prim_all: null array"); return WCNS_ERR_ARGUMENT; }
    // the state is final once the work queued on the context's stream is
    // done; the copies then spread over the three streams as above
    CK(cudaEventRecord(c->L.ev_fork, c->stream));
    cudaStream_t st[3] = {c->stream, c->L.side[0], c->L.side[1]};
    for (int q = 1; q < 3; q++) CK(cudaStreamWaitEvent(st[q], c->L.ev_fork, 0));
    int e = 0;
    for (int b = 0; b < nbk; b++) {
        const DevBlock &d = c->blk[b].d;
        const size_t n = (size_t)d.gx * d.gy * d.gz;
        for (int f = 0; f < 6; f++)
            if (prim[6 * b + f]) {
                CK(cudaMemcpyAsync(prim[6 * b + f], c->F.f[F_R + f] + d.off, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   st[e % 3]));
                e++;
            }
    }
    for (int q = 0; q < 3; q++) CK(cudaStreamSynchronize(st[q]));
    return 0;
}

// The interior state of every block in the flow-file layout
// (write_flow_file_parallel, parallel.f90:4073-4145: i = 1..ni fastest,
// then j, then k, no ghost layers): one strided copy per field and block.
// flow: 6 pointers per block, r u v w p t; a null t skips T of that block.
extern "C" int wcns_get_flow(WcnsContext *c, double *const *flow) {
    if (!c || !flow) { set_err("wcns_get_flow: null argument"); return WCNS_ERR_ARGUMENT; }
    const int nbk = (int)c->blk.size();
    for (int b = 0; b < nbk; b++)
        for (int f = 0; f < 5; f++)
            if (!flow[6 * b + f]) { set_err("wcns_get_flow: null array"); return WCNS_ERR_ARGUMENT; }
    CK(cudaEventRecord(c->L.ev_fork, c->stream));
    cudaStream_t st[3] = {c->stream, c->L.side[0], c->L.side[1]};
    for (int q = 1; q < 3; q++) CK(cudaStreamWaitEvent(st[q], c->L.ev_fork, 0));
    int e = 0;
    for (int b = 0; b < nbk; b++) {
        const DevBlock &d = c->blk[b].d;
        for (int f = 0; f < 6; f++) {
            if (!flow[6 * b + f]) continue;
            cudaMemcpy3DParms cp = {};
            // the ghosted box (-2:n+3) starts 3 points before the interior in each direction
            cp.srcPtr = make_cudaPitchedPtr(c->F.f[F_R + f] + d.off, sizeof(double) * d.gx, d.gx, d.gy);
            cp.srcPos = make_cudaPos(sizeof(double) * 3, 3, 3);
            cp.dstPtr = make_cudaPitchedPtr(flow[6 * b + f], sizeof(double) * d.ni, d.ni, d.nj);
            cp.dstPos = make_cudaPos(0, 0, 0);
            cp.extent = make_cudaExtent(sizeof(double) * d.ni, d.nj, d.nk);
            cp.kind = cudaMemcpyDeviceToHost;
            CK(cudaMemcpy3DAsync(&cp, st[e % 3]));
            e++;
        }
    }
    for (int q = 0; q < 3; q++) CK(cudaStreamSynchronize(st[q]));
    return 0;
}

// Interior points of any public fields of every block, in the flow-file
// layout (i = 1..ni fastest, then j, then k, no ghost layers), both ways:
// ptrs[nfields * b + q] is field fields[q] of block b+1; a null pointer skips
// that array.  One strided copy per array, spread over the context's three
// streams, one synchronisation.  Writing leaves every ghost point as it was:
// boundary_all refills the ghost layers the path reads.
// The interior points of named fields between host arrays (one per block and
// field, flow-file order) and the field pool: every (block, field) array is
// one contiguous copy into (or out of) a staging buffer of the context, and
// one kernel per field scatters (gathers) between the buffer and the
// ghosted layout, so the copies run at full link bandwidth instead of one
// DMA row of ni points at a time.
static int interior_copy(WcnsContext *c, int nfields, const int *fields, double *const *ptrs, bool to_device) {
    const char *fn = to_device ? "wcns_set_interior" : "wcns_get_interior";
    if (!c || nfields < 1 || !fields || !ptrs) { set_err(std::string(fn) + ": invalid argument"); return WCNS_ERR_ARGUMENT; }
    for (int q = 0; q < nfields; q++)
        if (!field_base(c, fields[q])) { set_err(std::string(fn) + ": unsupported field " + std::to_string(fields[q])); return WCNS_ERR_UNSUPPORTED; }
    const int nbk = (int)c->blk.size();
    if (nfields > c->stage_fields) {  // (re)size the staging buffer and its offset table
        long long pts = 0;
        for (int b = 0; b < nbk; b++) pts += c->blk[b].d.npts;
        std::vector<long long> first((size_t)nfields * nbk);
        for (int q = 0; q < nfields; q++) {
            long long o = (long long)q * pts;
            for (int b = 0; b < nbk; b++) {
                first[(size_t)q * nbk + b] = o;
                o += c->blk[b].d.npts;
            }
        }
        if (c->stage) cudaFree(c->stage);
        if (c->stage_first) cudaFree(c->stage_first);
        c->stage = nullptr;
        c->stage_first = nullptr;
        c->stage_fields = 0;
        CK(cudaMalloc(&c->stage, sizeof(double) * (size_t)nfields * pts));
        CK(cudaMalloc(&c->stage_first, sizeof(long long) * first.size()));
        CK(cudaMemcpy(c->stage_first, first.data(), sizeof(long long) * first.size(), cudaMemcpyHostToDevice));
        c->stage_fields = nfields;
    }
    long long pts = 0;
    for (int b = 0; b < nbk; b++) pts += c->blk[b].d.npts;
    for (int q = 0; q < nfields; q++) {
        double *field = field_base(c, fields[q]);
        double *stage = c->stage + (size_t)q * pts;
        // a block without a host array keeps its values: gather them first,
        // so that the scatter writes them back unchanged
        bool anynull = false;
        for (int b = 0; b < nbk; b++) anynull = anynull || !ptrs[(size_t)nfields * b + q];
        if (!to_device || anynull) launch_interior_stage(c->L, false, c->stage_first + (size_t)q * nbk, field, c->stage);
        long long o = 0;
        for (int b = 0; b < nbk; b++) {
            const size_t n = (size_t)c->blk[b].d.npts;
            double *host = ptrs[(size_t)nfields * b + q];
            if (host)
                CK(cudaMemcpyAsync(to_device ? (void *)(stage + o) : (void *)host, to_device ? (const void *)host : (const void *)(stage + o),
                                   sizeof(double) * n, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, c->stream));
            o += (long long)n;
        }
        if (to_device) launch_interior_stage(c->L, true, c->stage_first + (size_t)q * nbk, field, c->stage);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_set_interior(WcnsContext *c, int nfields, const int *fields, const double *const *ptrs) {
    return interior_copy(c, nfields, fields, const_cast<double *const *>(ptrs), true);
}

extern "C" int wcns_get_interior(WcnsContext *c, int nfields, const int *fields, double *const *ptrs) {
    return interior_copy(c, nfields, fields, ptrs, false);
}

extern "C" int wcns_set_field(WcnsContext *c, int field, int nb, const double *in) {
    const DevBlock *d;
    if (int rc = block_range(c, nb, &d)) return rc;
    double *base = field_base(c, field);
    if (!base || !in) { set_err("wcns_set_field: unsupported field"); return WCNS_ERR_UNSUPPORTED; }
    size_t n = (size_t)d->gx * d->gy * d->gz;
    CK(cudaMemcpyAsync(base + d->off, in, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// Spalart-Allmaras model set-up: the model's arrays, the wall distance of
// calc_wall_dists_parallel (parallel.f90:4313-4470; wall points: every point
// of the bctype 2, 20 and 21 regions) and init_SA (turblence.f90:2701-2733).
extern "C" int wcns_sa_setup(WcnsContext *c, const double *const *xyz, double timedt_turb, double kmaxlim) {
    if (!c || !xyz) { set_err("wcns_sa_setup: null argument"); return WCNS_ERR_ARGUMENT; }
    const int nbk = (int)c->blk.size();
    for (int q = 0; q < 3 * nbk; q++)
        if (!xyz[q]) { set_err("wcns_sa_setup: missing coordinates"); return WCNS_ERR_ARGUMENT; }
    if (c->P.nvis != 1) { set_err("wcns_sa_setup: the SA model needs the viscous path (nvis 1)"); return WCNS_ERR_UNSUPPORTED; }
    if (!(timedt_turb > 0.0)) { set_err("wcns_sa_setup: timedt_turb must be positive"); return WCNS_ERR_ARGUMENT; }
    if (!c->sa_pool) {
        CK(cudaMalloc(&c->sa_pool, sizeof(double) * SA_NFIELDS * (size_t)c->total));
        CK(cudaMemset(c->sa_pool, 0, sizeof(double) * SA_NFIELDS * (size_t)c->total));
        double *f[SA_NFIELDS];
        for (int q = 0; q < SA_NFIELDS; q++) f[q] = c->sa_pool + (size_t)q * c->total;
        c->SA = SaFields{f[0], f[1], f[2], f[3], f[4], {f[5], f[6], f[7]}};
    }
    // constants as cal_rhs_source_SA evaluates its parameter statements
    const double cb1 = 0.1355, cb2 = 0.622, cv1 = 7.1, cga = 2. / 3.0, ki = 0.419, cw3 = 2.0;
    SaParams &S = c->SAP;
    S.reynolds = c->P.reynolds;
    S.re = c->P.re;
    S.ki2 = ki * ki;
    S.cv13 = pow(cv1, 3.0);
    S.cw36 = pow(cw3, 6.0);
    S.onesix = 1.0 / 6.0;
    S.cw1 = cb1 / ki / ki + (1.0 + cb2) / cga;
    S.timedt_turb = timedt_turb;
    S.kmaxlim = kmaxlim;
    c->L.SA = &c->SA;
    c->L.SAP = &c->SAP;
    if (c->L.wide && !c->L.wide->A.sa) {
        // the model's scalar sweeps run on the wide chunks too
        WideArrays &A = c->L.wide->A;
        CK(cudaMalloc(&A.sa, sizeof(double) * (6 * (size_t)A.n + 8)));
        c->owned.push_back(A.sa);
    }
    // the mean-flow kernels now read vist (spectvist, the viscous
    // coefficients); a step graph captured before holds the old arguments
    c->F.f[F_VIST] = c->SA.vist;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    c->launches = 0;
    // coordinates in the pool's layout and the wall point list, grouped by
    // the sets of blocks joined through interfaces (one case each): a block
    // measures its distance to its own set's walls, as
    // calc_wall_dists_parallel does for the one case it runs
    std::vector<int> comp(nbk);
    for (int b = 0; b < nbk; b++) comp[b] = b;
    auto root = [&](int b) {
        while (comp[b] != b) b = comp[b] = comp[comp[b]];
        return b;
    };
    for (int b = 0; b < nbk; b++)
        for (const HReg &R : c->blk[b].regs)
            if (R.bctype < 0) comp[root(b)] = root(R.nbt - 1);
    std::vector<double> wall, tmp;
    std::vector<int> wrange(2 * nbk, 0);
    double *xyzd = nullptr, *walld = nullptr;
    CK(cudaMalloc(&xyzd, sizeof(double) * 3 * (size_t)c->total));
    for (int b = 0; b < nbk; b++) {
        const DevBlock &d = c->blk[b].d;
        tmp.assign((size_t)d.gx * d.gy * d.gz, 0.0);
        for (int q = 0; q < 3; q++) {
            const double *src = xyz[3 * b + q];
            for (int k = 1; k <= d.nk; k++)
                for (int j = 1; j <= d.nj; j++)
                    for (int i = 1; i <= d.ni; i++)
                        tmp[gidx(d, i, j, k) - d.off] = src[(i - 1) + (size_t)d.ni * ((j - 1) + (size_t)d.nj * (k - 1))];
            cudaError_t e = cudaMemcpy(xyzd + (size_t)q * c->total + d.off, tmp.data(), sizeof(double) * tmp.size(),
                                       cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { cudaFree(xyzd); set_err(std::string("wcns_sa_setup: ") + cudaGetErrorString(e)); return WCNS_ERR_CUDA; }
        }
    }
    for (int r = 0; r < nbk; r++) {
        if (root(r) != r) continue;
        const int w0 = (int)(wall.size() / 3);
        for (int b = 0; b < nbk; b++) {
            if (root(b) != r) continue;
            const DevBlock &d = c->blk[b].d;
            for (const HReg &R : c->blk[b].regs) {
                if (!(R.bctype == 2 || R.bctype == 20 || R.bctype == 21)) continue;
                for (int k = R.s_st[2]; k <= R.s_ed[2]; k++)
                    for (int j = R.s_st[1]; j <= R.s_ed[1]; j++)
                        for (int i = R.s_st[0]; i <= R.s_ed[0]; i++) {
                            size_t g = (size_t)(i - 1) + (size_t)d.ni * ((size_t)(j - 1) + (size_t)d.nj * (k - 1));
                            for (int q = 0; q < 3; q++) wall.push_back(xyz[3 * b + q][g]);
                        }
            }
        }
        if (wall.size() / 3 > 0x7fffffff) { cudaFree(xyzd); set_err("wcns_sa_setup: too many wall points"); return WCNS_ERR_ARGUMENT; }
        const int w1 = (int)(wall.size() / 3);
        for (int b = 0; b < nbk; b++)
            if (root(b) == r) { wrange[2 * b] = w0; wrange[2 * b + 1] = w1; }
    }
    int *wranged = nullptr;
    {
        cudaError_t e = cudaMalloc(&wranged, sizeof(int) * wrange.size());
        if (e == cudaSuccess) e = cudaMemcpy(wranged, wrange.data(), sizeof(int) * wrange.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !wall.empty()) e = cudaMalloc(&walld, sizeof(double) * wall.size());
        if (e == cudaSuccess && !wall.empty()) e = cudaMemcpy(walld, wall.data(), sizeof(double) * wall.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(xyzd); cudaFree(walld); cudaFree(wranged);
            set_err(std::string("wcns_sa_setup: ") + cudaGetErrorString(e));
            return WCNS_ERR_CUDA;
        }
    }
    // init_SA: vt = muoo * fv1(muoo)
    const double muoo = 1.0e-1, kf3 = pow(muoo, 3.0), vt = muoo * (kf3 / (kf3 + S.cv13));
    launch_sa_setup(c->L, xyzd, walld, wranged, vt);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(xyzd);
    cudaFree(wranged);
    if (walld) cudaFree(walld);
    if (e != cudaSuccess) { set_err(std::string("wcns_sa_setup: ") + cudaGetErrorString(e)); return WCNS_ERR_CUDA; }
    return 0;
}

#define PHASE(name, body)                                              \
    extern "C" int name(WcnsContext *c) {                              \
        if (!c) { set_err(#name ": null context"); return WCNS_ERR_ARGUMENT; } \
        body;                                                          \
        CK(cudaGetLastError());                                        \
        return check_errors(c);                                        \
    }

PHASE(wcns_boundary_all, launch_boundary(c->L))
PHASE(wcns_initial_q_dq_c_t, launch_init(c->L))
PHASE(wcns_timestep, launch_timestep(c->L))
PHASE(wcns_rhs_vis, if (c->P.nvis == 1) {
    if (c->sa_pool) launch_turbulence(c->L);  // turbulence(nb), RHS.f90:22
    launch_node_derivatives(c->L);
    launch_rhs_dirs(c->L, true);
})
// the viscous residual without the model step (a driver that advances the
// SA model itself with wcns_turbulence, e.g. a sharded run)
PHASE(wcns_rhs_vis_flux, if (c->P.nvis == 1) {
    launch_node_derivatives(c->L);
    launch_rhs_dirs(c->L, true);
})
PHASE(wcns_communicate_dq, launch_communicate(c->L, 0))
PHASE(wcns_turbulence, {
    if (!c->sa_pool) { set_err("wcns_turbulence: wcns_sa_setup was not called"); return WCNS_ERR_ARGUMENT; }
    launch_turbulence(c->L);
})
PHASE(wcns_rhs_invis, launch_rhs_dirs(c->L, false))
PHASE(wcns_lhs, {
    launch_lhs(c->L);
    launch_update(c->L);
})
PHASE(wcns_communicate_pv, launch_communicate(c->L, 1))

extern "C" int wcns_residual(WcnsContext *c, double *res, double *resmax, double *rms) {
    if (!c) { set_err("null context"); return WCNS_ERR_ARGUMENT; }
    launch_residual(c->L, nullptr);
    CK(cudaGetLastError());
    int nb = (int)c->blk.size();
    std::vector<double> h(2 * nb + 1);
    CK(cudaMemcpyAsync(h.data(), c->L.res_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (res) std::copy(h.begin(), h.begin() + nb, res);
    if (resmax) std::copy(h.begin() + nb, h.begin() + 2 * nb, resmax);
    if (rms) *rms = h[2 * nb];
    return 0;
}

// A block's free stream at its own Mach number, for contexts holding
// independent cases of different Mach numbers (every other parameter is the
// context's); the kernels read the block table on the device at run time, so
// a captured step graph needs no rebuild.
extern "C" int wcns_set_block_freestream(WcnsContext *c, int nb, double moo) {
    if (!c || nb < 1 || nb > (int)c->blk.size() || !(moo > 0.0)) {
        set_err("wcns_set_block_freestream: invalid argument");
        return WCNS_ERR_ARGUMENT;
    }
    DevBlock &d = c->blk[nb - 1].d;
    set_block_freestream(d, c->P, moo);
    const_cast<DevBlock *>(c->L.hblocks)[nb - 1] = d;
    CK(cudaMemcpyAsync(c->L.blocks + (nb - 1), &d, sizeof(DevBlock), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// force (PostProcess.f90:1415-1480): integrate over the wall quads of blocks
// nb0..nb1, then normalise on the host as the reference does after its
// MPI_REDUCE
static int forces_range(WcnsContext *c, int nb0, int nb1, const double *ref, double *out) {
    if (!c || !ref || !out || nb0 < 1 || nb1 < nb0 || nb1 > (int)c->blk.size()) {
        set_err("wcns_forces: invalid argument");
        return WCNS_ERR_ARGUMENT;
    }
    double cf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    long long q0 = -1, q1 = 0;
    for (const DevWall &W : c->hwalls)
        if (W.blk >= nb0 - 1 && W.blk <= nb1 - 1) {
            if (q0 < 0) q0 = W.quad_off;
            q1 = W.quad_off + W.nquad;
        }
    if (c->L.nwall && q0 >= 0) {
        launch_forces(c->L, ref[2], ref[3], ref[4], q0, q1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(cf, c->L.wall_out, sizeof cf, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    const double sref = ref[0], lfref = ref[1], whole = ref[5];
    const double scf = 1.0 / sref, vcm = 1.0 / (sref * lfref);
    for (int m = 0; m < 3; m++) out[m] = (2 - whole) * cf[m] * scf;
    for (int m = 3; m < 6; m++) out[m] = (2 - whole) * cf[m] * vcm;
    const double PAI = 3.14159265;
    const double attack = c->prm.attack * PAI / 180.0, sideslip = c->prm.sideslip * PAI / 180.0;
    const double sina = sin(attack), cosa = cos(attack), sinb = sin(sideslip), cosb = cos(sideslip);
    out[6] = out[1] * cosa - out[0] * sina;
    out[7] = cosb * (out[1] * sina + out[0] * cosa) + sinb * out[2];
    out[8] = copysign(1.0, out[1]) * out[5] / (fabs(out[1]) + SMALL);
    return 0;
}

extern "C" int wcns_forces(WcnsContext *c, const double *ref, double *out) {
    if (!c) { set_err("wcns_forces: invalid argument"); return WCNS_ERR_ARGUMENT; }
    return forces_range(c, 1, (int)c->blk.size(), ref, out);
}

extern "C" int wcns_forces_blocks(WcnsContext *c, int nb0, int nb1, const double *ref, double *out) {
    return forces_range(c, nb0, nb1, ref, out);
}

// one complete step (Main.f90:85-109) on the context stream
static int enqueue_step(WcnsContext *c, double *rms_slot) {
    LaunchCtx &L = c->L;
    int n = 0;
    launch_boundary(L); n += 2;
    prof_mark(L, "boundary_all");
    launch_init_timestep(L); n += 1;
    prof_mark(L, "initial_q_dq_c_t+timestep");
    if (c->P.nvis == 1) {
        if (c->sa_pool) n += launch_turbulence(L);
        launch_node_derivatives(L); n += 1;
        launch_rhs_dirs(L, true);
        for (int d = 0; d < 3; d++) n += L.vis[d].ngroups ? 1 : 0;
        n += (L.vis[1].ngroups || L.vis[2].ngroups) ? 1 : 0;
        prof_mark(L, "rhs_vis");
        launch_communicate(L, 0); n += L.nsnap ? 2 : 0;
        prof_mark(L, "communicate_dq");
    }
    launch_rhs_dirs(L, false);
    for (int d = 0; d < 3; d++) n += L.inv[d].ngroups ? 1 : 0;
    n += (L.mixed && (L.inv[1].ngroups || L.inv[2].ngroups)) ? 1 : 0;  // k_combine_dq (the FP64 directions add in place)
    prof_mark(L, "rhs_invis");
    launch_communicate(L, 0); n += L.nsnap ? 2 : 0;
    prof_mark(L, "communicate_dq");
    n += launch_lhs(L);
    launch_update(L); n += 2;
    prof_mark(L, "update");
    launch_communicate(L, 1); n += L.nsnap ? 2 : 0;
    prof_mark(L, "communicate_pv");
    launch_residual(L, rms_slot); n += 2;
    prof_mark(L, "residual");
    c->launches = n;
    CK(cudaGetLastError());
    return 0;
}

// One whole step enqueued phase by phase (not from the graph) with an event
// after each phase; ms[q] is the device time of phase q, names[q] its name
// (static strings), *nphases their count (at most cap).  The step advances
// the state like wcns_step(c, 1, NULL).
extern "C" int wcns_profile_step(WcnsContext *c, int cap, double *ms, const char **names, int *nphases) {
    if (!c || cap < 1 || !ms || !names || !nphases) { set_err("wcns_profile_step: invalid argument"); return WCNS_ERR_ARGUMENT; }
    std::vector<cudaEvent_t> ev(cap + 1, nullptr);
    std::vector<const char *> nm(cap, nullptr);
    int rc = 0;
    for (auto &e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) { set_err("wcns_profile_step: event creation failed"); rc = WCNS_ERR_CUDA; }
    if (!rc) {
        ProfMarks pm;
        pm.cap = cap;
        pm.ev = ev.data() + 1;
        pm.name = nm.data();
        cudaEventRecord(ev[0], c->stream);
        c->L.prof = &pm;
        rc = enqueue_step(c, nullptr);
        c->L.prof = nullptr;
        if (!rc) rc = check_errors(c);
        if (!rc) {
            for (int q = 0; q < pm.n; q++) {
                float t = 0.0f;
                cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
                ms[q] = t;
                names[q] = nm[q];
            }
            *nphases = pm.n;
        }
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

static int build_graph(WcnsContext *c) {
    if (c->graph) return 0;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(c, nullptr);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) { set_err(std::string("graph capture: ") + cudaGetErrorString(e)); return WCNS_ERR_CUDA; }
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_err(std::string("graph instantiate: ") + cudaGetErrorString(e)); return WCNS_ERR_CUDA; }
    return 0;
}

extern "C" int wcns_step_async(WcnsContext *c, int nsteps) {
    if (!c || nsteps < 0) { set_err("wcns_step_async: invalid argument"); return WCNS_ERR_ARGUMENT; }
    if (int rc = build_graph(c)) return rc;
    for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c->graph, c->stream));
    return 0;
}

extern "C" int wcns_sync(WcnsContext *c) {
    if (!c) return WCNS_ERR_ARGUMENT;
    return check_errors(c);
}

// The error slots are read after every step, so that a multi-step call
// stops after the first step at which the reference would stop
// (update_limited's bad-point limit, Sub2.f90:781-785; the Roe c^2 check,
// flux.f90:179-182): the state is that after the failing step, later steps
// are not run and their rms_history entries are left untouched.
extern "C" int wcns_step(WcnsContext *c, int nsteps, double *rms_history) {
    if (!c || nsteps < 0) { set_err("wcns_step: invalid argument"); return WCNS_ERR_ARGUMENT; }
    if (int rc = build_graph(c)) return rc;
    int nb = (int)c->blk.size();
    for (int s = 0; s < nsteps; s++) {
        CK(cudaGraphLaunch(c->graph, c->stream));
        if (rms_history) CK(cudaMemcpyAsync(rms_history + s, c->L.res_out + 2 * nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (int rc = check_errors(c)) {
            g_err += " (step " + std::to_string(s + 1) + " of " + std::to_string(nsteps) + " of this call)";
            return rc;
        }
    }
    return 0;
}

// The LU-SGS sweep's bounded wait on an mbarrier that nothing completes,
// with a limit of limit_cycles clock cycles: returns what a step returns
// after a sweep timed out (WCNS_ERR_CUDA and its message), with no other
// work in flight, and leaves the context usable.
extern "C" int wcns_selftest_timeout(WcnsContext *c, long long limit_cycles) {
    if (!c || limit_cycles < 0 || limit_cycles > (1LL << 32)) {
        set_err("wcns_selftest_timeout: invalid argument (0 <= limit_cycles <= 2^32)");
        return WCNS_ERR_ARGUMENT;
    }
    launch_wait_probe(c->L, limit_cycles);
    CK(cudaGetLastError());
    return check_errors(c);
}

extern "C" void *wcns_stream(WcnsContext *c) { return c ? (void *)c->stream : nullptr; }
extern "C" int wcns_launches_per_step(WcnsContext *c) {
    if (!c) return 0;
    if (!c->launches) {
        // count by enqueueing into a throw-away capture
        build_graph(c);
    }
    return c->launches;
}
extern "C" int wcns_n_multipoints(WcnsContext *c) { return c ? c->nmulti : 0; }
// 64: the residual in FP64 with the reference's operation order (default);
// 32: the mixed-precision residual of k_rhs_mixed.cu.  The rest of the step
// is FP64 either way.
extern "C" int wcns_set_precision(WcnsContext *c, int bits) {
    if (!c) { set_err("wcns_set_precision: null context"); return WCNS_ERR_ARGUMENT; }
    if (bits != 64 && bits != 32) { set_err("wcns_set_precision: bits must be 64 or 32"); return WCNS_ERR_ARGUMENT; }
    const int mixed = bits == 32 ? 1 : 0;
    if (mixed != c->L.mixed) {
        CK(cudaStreamSynchronize(c->stream));
        c->L.mixed = mixed;
        c->L.duv32 = (float *)c->F.f[F_DUV0];  // the FP64 node derivatives are unused meanwhile
        if (c->graph) {  // the captured step holds the other kernels
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
    }
    return 0;
}

extern "C" int wcns_get_precision(WcnsContext *c) {
    if (!c) return -1;
    return c->L.mixed ? 32 : 64;
}

// ---------------------------------------------------------------------------
// Launch shapes and their autotuner.  shape[0]: CTAs per block cluster of the
// clustered LU-SGS sweeps (0 when the sweeps run wide or by plane);
// shape[1]: 1 sixteen lanes per column, 0 three; shape[2], shape[3]: lines
// per CTA of the inviscid / viscous residual kernels at most.  No shape
// changes a result: every point's arithmetic is the same in each.

static bool clustered_sweeps(const WcnsContext *c) { return !c->L.wide && !c->L.sweep_plane; }

static void drop_graph(WcnsContext *c) {
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
}

// name of the context's device (for keying tuned shapes), NUL-terminated in buf[len]
extern "C" int wcns_device_name(WcnsContext *c, char *buf, int len) {
    if (!c || !buf || len < 1) { set_err("wcns_device_name: invalid argument"); return WCNS_ERR_ARGUMENT; }
    int dev = 0;
    cudaDeviceProp prop;
    CK(cudaGetDevice(&dev));
    CK(cudaGetDeviceProperties(&prop, dev));
    snprintf(buf, (size_t)len, "%s sm_%d%d %d SMs", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    return 0;
}

extern "C" int wcns_get_shape(WcnsContext *c, int *shape) {
    if (!c || !shape) { set_err("wcns_get_shape: invalid argument"); return WCNS_ERR_ARGUMENT; }
    shape[0] = clustered_sweeps(c) ? c->L.sweep_cluster : 0;
    shape[1] = clustered_sweeps(c) ? c->L.sweep_fine : 0;
    shape[2] = c->L.inv_cap;
    shape[3] = c->L.vis_cap;
    return 0;
}

// a context whose blocks fit the clustered sweeps (its plane-major arrays
// exist) can also sweep wide, and switch between the two
static bool can_cluster(const WcnsContext *c) { return c->pm_pool != nullptr; }

static int apply_shape(WcnsContext *c, const int *shape) {
    LaunchCtx &L = c->L;
    if (can_cluster(c) && !L.sweep_plane) {
        if (shape[0] == 0) {  // wide sweeps
            if (!L.wide) {
                const int rc = wide_alloc(c);
                if (rc) {
                    if (rc < 0) set_err("wcns_set_shape: the blocks cannot be swept wide");
                    return rc < 0 ? WCNS_ERR_ARGUMENT : rc;
                }
            }
        } else if (L.wide || shape[0] != L.sweep_cluster || shape[1] != L.sweep_fine) {
            if (setup_sweep_exact(L, shape[0], shape[1])) {
                set_err("wcns_set_shape: the blocks cannot be swept with " + std::to_string(shape[0]) +
                        " CTAs per cluster in that lane mode");
                return WCNS_ERR_ARGUMENT;
            }
            c->PM.csize = L.sweep_cluster;
            wide_free(c);
        }
    }
    if (shape[2] != L.inv_cap || shape[3] != L.vis_cap)
        if (int rc = build_line_tables(c, shape[2], shape[3])) return rc;
    drop_graph(c);
    return 0;
}

extern "C" int wcns_set_shape(WcnsContext *c, const int *shape) {
    if (!c || !shape) { set_err("wcns_set_shape: invalid argument"); return WCNS_ERR_ARGUMENT; }
    if (shape[2] < 1 || shape[2] > INV_LINES_DEFAULT || shape[3] < 1 || shape[3] > VIS_LINES_DEFAULT) {
        set_err("wcns_set_shape: lines per CTA must be in 1..32");
        return WCNS_ERR_ARGUMENT;
    }
    if (shape[0] < 0 || shape[1] < 0 || shape[1] > 1) {
        set_err("wcns_set_shape: shape[0] >= 0 (0: wide sweeps) and shape[1] in 0..1");
        return WCNS_ERR_ARGUMENT;
    }
    if (!can_cluster(c) && shape[0] != 0) {
        set_err("wcns_set_shape: these blocks only sweep wide or by plane (shape[0] = 0)");
        return WCNS_ERR_ARGUMENT;
    }
    CK(cudaStreamSynchronize(c->stream));
    return apply_shape(c, shape);
}

// Device ms of `reps` runs of `body` on the context stream, dq restored from
// `saved` before each (outside the timed interval).
template <class Body>
static double time_reps(WcnsContext *c, int reps, const double *saved, Body body) {
    double *dq = c->F.f[F_DQ1];
    const size_t bytes = sizeof(double) * 5 * (size_t)c->total;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double total = 0.0;
    for (int r = 0; r <= reps; r++) {  // the first run is a warm-up
        cudaMemcpyAsync(dq, saved, bytes, cudaMemcpyDeviceToDevice, c->stream);
        cudaEventRecord(e0, c->stream);
        body();
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0) total += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return total / reps;
}

// Times every candidate shape on the context's current state with the
// phases it shapes (the LU-SGS phase for the sweep shape, the inviscid and
// viscous residual for the line caps), keeps the fastest, and returns it in
// shape[4]; ms[3] (may be NULL) receives the best device ms of the three
// phases.  The state (prim, SA fields) is not changed; dq is restored.
extern "C" int wcns_autotune(WcnsContext *c, int reps, int *shape, double *ms) {
    if (!c || !shape || reps < 1) { set_err("wcns_autotune: invalid argument"); return WCNS_ERR_ARGUMENT; }
    LaunchCtx &L = c->L;
    CK(cudaStreamSynchronize(c->stream));
    double *saved = nullptr;
    const size_t bytes = sizeof(double) * 5 * (size_t)c->total;
    CK(cudaMalloc(&saved, bytes));
    CK(cudaMemcpy(saved, c->F.f[F_DQ1], bytes, cudaMemcpyDeviceToDevice));
    int best[4];
    wcns_get_shape(c, best);
    double best_ms[3] = {0.0, 0.0, 0.0};
    // the LU-SGS sweep form and shape: every cluster shape, and the wide sweeps
    if (can_cluster(c) && !L.sweep_plane) {
        double tbest = 1e300;
        const bool was_wide = L.wide != nullptr;
        L.wide = nullptr;
        const int cls[5] = {1, 2, 4, 8, 16};
        for (int fine = 1; fine >= 0; fine--)
            for (int q = 0; q < 5; q++) {
                int cand[4] = {cls[q], fine, best[2], best[3]};
                if (setup_sweep_exact(L, cand[0], cand[1])) continue;
                c->PM.csize = L.sweep_cluster;
                const double t = time_reps(c, reps, saved, [&] { launch_lhs(L); });
                if (t < tbest) { tbest = t; best[0] = cand[0]; best[1] = cand[1]; }
            }
        if (was_wide) L.wide = c->wide.get();
        const int wr = wide_alloc(c);
        if (wr > 0) { cudaFree(saved); return wr; }
        if (wr == 0) {
            const double t = time_reps(c, reps, saved, [&] { launch_lhs(L); });
            if (t < tbest) { tbest = t; best[0] = 0; best[1] = 0; }
        }
        if (best[0] > 0) {
            setup_sweep_exact(L, best[0], best[1]);
            c->PM.csize = L.sweep_cluster;
            wide_free(c);
        }
        best_ms[0] = tbest;
    }
    // lines per CTA of the residual kernels
    const int caps[4] = {4, 8, 16, 32};
    for (int vis = 0; vis <= (c->P.nvis == 1 ? 1 : 0); vis++) {
        if (vis) launch_node_derivatives(L);
        double tbest = 1e300;
        int kbest = vis ? best[3] : best[2];
        for (int q = 0; q < 4; q++) {
            const int ic = vis ? best[2] : caps[q], vc = vis ? caps[q] : best[3];
            if (build_line_tables(c, ic, vc)) continue;
            const double t = time_reps(c, reps, saved, [&] { launch_rhs_dirs(L, vis == 1); });
            if (t < tbest) { tbest = t; kbest = caps[q]; }
        }
        best[vis ? 3 : 2] = kbest;
        best_ms[vis ? 2 : 1] = tbest;
        build_line_tables(c, best[2], best[3]);
    }
    cudaMemcpy(c->F.f[F_DQ1], saved, bytes, cudaMemcpyDeviceToDevice);
    cudaFree(saved);
    drop_graph(c);
    CK(cudaGetLastError());
    for (int q = 0; q < 4; q++) shape[q] = best[q];
    if (ms)
        for (int q = 0; q < 3; q++) ms[q] = best_ms[q];
    return check_errors(c);
}

extern "C" int wcns_sweep_mode(WcnsContext *c) {
    if (!c) return -1;
    return c->L.wide ? 2 : c->L.sweep_plane ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Tangent / adjoint of the inviscid residual and the LU-SGS operator pair
// (k_adjoint.cu), on five-field slots of the context (WCNS_ADJ_*).

static int adj_ready(WcnsContext *c, const char *who) {
    if (c->P.nvis != 0 || c->P.nscheme != 4 || (c->P.nflux != 1 && c->P.nflux != 3)) {
        set_err(std::string(who) + ": the adjoint covers the inviscid residual with nscheme 4 and the Steger-Warming or Roe flux");
        return WCNS_ERR_UNSUPPORTED;
    }
    if (!c->adj_pool) {
        const size_t bytes = sizeof(double) * 5 * (size_t)WCNS_ADJ_NSLOTS * (size_t)c->total;
        CK(cudaMalloc(&c->adj_pool, bytes));
        CK(cudaMemset(c->adj_pool, 0, bytes));
    }
    return 0;
}
static double *adj_slot(WcnsContext *c, int s) { return c->adj_pool + (size_t)s * 5 * (size_t)c->total; }

static int adj_copy(WcnsContext *c, int slot, int nb, double *const *ptrs, bool to_device, const char *who) {
    if (int rc = adj_ready(c, who)) return rc;
    if (slot < 0 || slot >= WCNS_ADJ_NSLOTS || !ptrs) { set_err(std::string(who) + ": invalid argument"); return WCNS_ERR_ARGUMENT; }
    const DevBlock *d = nullptr;
    if (int rc = block_range(c, nb, &d)) return rc;
    const size_t n = (size_t)d->gx * d->gy * d->gz;
    for (int m = 0; m < 5; m++) {
        if (!ptrs[m]) { set_err(std::string(who) + ": null array"); return WCNS_ERR_ARGUMENT; }
        double *dev = adj_slot(c, slot) + (size_t)m * c->total + d->off;
        CK(cudaMemcpyAsync(to_device ? (void *)dev : (void *)ptrs[m], to_device ? (const void *)ptrs[m] : (const void *)dev,
                           sizeof(double) * n, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_adj_set(WcnsContext *c, int slot, int nb, const double *const *five) {
    if (!c) { set_err("wcns_adj_set: null context"); return WCNS_ERR_ARGUMENT; }
    return adj_copy(c, slot, nb, (double *const *)five, true, "wcns_adj_set");
}
extern "C" int wcns_adj_get(WcnsContext *c, int slot, int nb, double *const *five) {
    if (!c) { set_err("wcns_adj_get: null context"); return WCNS_ERR_ARGUMENT; }
    return adj_copy(c, slot, nb, five, false, "wcns_adj_get");
}
extern "C" int wcns_adj_zero(WcnsContext *c, int slot) {
    if (!c) { set_err("wcns_adj_zero: null context"); return WCNS_ERR_ARGUMENT; }
    if (int rc = adj_ready(c, "wcns_adj_zero")) return rc;
    if (slot < 0 || slot >= WCNS_ADJ_NSLOTS) { set_err("wcns_adj_zero: invalid slot"); return WCNS_ERR_ARGUMENT; }
    CK(cudaMemsetAsync(adj_slot(c, slot), 0, sizeof(double) * 5 * (size_t)c->total, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_rhs_invis_tangent(WcnsContext *c) {
    if (!c) { set_err("wcns_rhs_invis_tangent: null context"); return WCNS_ERR_ARGUMENT; }
    if (int rc = adj_ready(c, "wcns_rhs_invis_tangent")) return rc;
    CK(cudaMemsetAsync(adj_slot(c, WCNS_ADJ_RDOT), 0, sizeof(double) * 5 * (size_t)c->total, c->stream));
    launch_rhs_invis_jvp(c->L, adj_slot(c, WCNS_ADJ_V), adj_slot(c, WCNS_ADJ_RDOT));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_rhs_invis_adjoint(WcnsContext *c, int fold) {
    if (!c) { set_err("wcns_rhs_invis_adjoint: null context"); return WCNS_ERR_ARGUMENT; }
    if (int rc = adj_ready(c, "wcns_rhs_invis_adjoint")) return rc;
    CK(cudaMemsetAsync(adj_slot(c, WCNS_ADJ_QBAR), 0, sizeof(double) * 5 * (size_t)c->total, c->stream));
    launch_rhs_invis_vjp(c->L, adj_slot(c, WCNS_ADJ_LAM), adj_slot(c, WCNS_ADJ_QBAR), fold != 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_lusgs_operator(WcnsContext *c, int transpose) {
    if (!c) { set_err("wcns_lusgs_operator: null context"); return WCNS_ERR_ARGUMENT; }
    if (int rc = adj_ready(c, "wcns_lusgs_operator")) return rc;
    launch_lusgs_operator(c->L, adj_slot(c, WCNS_ADJ_X), adj_slot(c, WCNS_ADJ_B), transpose != 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int wcns_adjoint_iterate(WcnsContext *c, int iters, double *hist) {
    if (!c || iters < 1) { set_err("wcns_adjoint_iterate: invalid argument"); return WCNS_ERR_ARGUMENT; }
    if (int rc = adj_ready(c, "wcns_adjoint_iterate")) return rc;
    LaunchCtx &L = c->L;
    // the linearisation point's ghosts, time step and spectral radii
    launch_boundary(L);
    launch_init_timestep(L);
    double *t = adj_slot(c, WCNS_ADJ_W), *psi = adj_slot(c, WCNS_ADJ_PSI), *x = adj_slot(c, WCNS_ADJ_X);
    double *nrm = nullptr;
    CK(cudaMalloc(&nrm, sizeof(double)));
    const size_t bytes = sizeof(double) * 5 * (size_t)c->total;
    int rc = 0;
    for (int it = 0; it < iters && !rc; it++) {
        cudaMemsetAsync(t, 0, bytes, c->stream);
        launch_rhs_invis_vjp(L, psi, t, true);                        // (dr/dq)^T psi
        launch_adj_to_conserved(L, t, adj_slot(c, WCNS_ADJ_G));       // r_Q^T psi + g
        launch_adj_zero_faces(L, t);                                  // the step's operator is Z P Z
        cudaMemsetAsync(nrm, 0, sizeof(double), c->stream);
        launch_adj_norm2(L, t, nrm);
        launch_lusgs_operator(L, x, t, true);                         // Z P^T Z (r_Q^T psi + g)
        launch_adj_zero_faces(L, x);
        launch_adj_axpy(L, psi, x);
        double h = 0.0;
        if (cudaMemcpyAsync(&h, nrm, sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess) {
            set_err(std::string("wcns_adjoint_iterate: ") + cudaGetErrorString(cudaGetLastError()));
            rc = WCNS_ERR_CUDA;
        }
        if (hist) hist[it] = sqrt(h);
    }
    cudaFree(nrm);
    if (rc) return rc;
    CK(cudaGetLastError());
    return check_errors(c);
}
