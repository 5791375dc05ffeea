// wcns_launch.h -- host-side launch context shared by the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "wcns_dev.cuh"

namespace wcns {

// A group of up to 8 lines of one block along direction `dir`: lines are
// indexed by (a, b) = the two other indices, a running fastest in memory for
// dir != 0 (so that a group reads coalesced rows) and along j for dir == 0.
struct LineGroup {
    int blk, a0, b, nl;
};

struct DirTable {
    LineGroup *groups = nullptr;  // device
    int ngroups = 0, nl_max = 0, hmax = 0;
    size_t smem = 0;              // dynamic shared memory of the launch (max over groups)
};

// One boundary region as the device sees it (bcindex order within a block).
// Interface regions (bctype -1) are in the list too: the BC walk applies the
// SA model's qke/vist copies there when the model is set up, and skips them
// otherwise.  sa_first: the region's first entry in the interface source
// list (LaunchCtx::sa_if_src); same: 1 for a block connected to itself.
struct DevRegion {
    int blk, bctype;
    int s_st[3], s_ed[3];
    int s_nd, s_lr, s_lr3d[3];
    int same;
    long long sa_first;
};

// interface ghost copy: ghost (dst) <- partner interior (src)
struct GhostCopy {
    long long dst, src;
};

// interface averaging entry: own face point <- partner face point
struct PairEntry {
    long long own, partner;  // field indices
    int partner_slot;        // index of the partner point in the snapshot list
    int same;                // 1 for a block connected to itself
};

// a wall region for the force integration (bctype 2), in the reference's
// block and region order
struct DevWall {
    int blk;
    int s_st[3], e[3], s_lr3d[3], s_lr;
    long long pt_off;    // first point in the wall point arrays
    long long quad_off;  // first quad in the quad array
    long long nquad;     // quads of the region
};

// Spalart-Allmaras model arrays (one field each, the pool's layout): qke,
// vist, the wall distance, and the model's dqke, spec and qke derivatives
struct SaFields {
    double *qke, *vist, *dist, *dqke, *spec, *dmu[3];
};
constexpr int SA_NFIELDS = 8;

// SA constants as the reference evaluates them (cal_rhs_source_SA,
// turblence.f90:2508-2513), computed on the host, and the $step/$turbulence
// values timedt_turb and kmaxlim
struct SaParams {
    double reynolds, re, ki2, cv13, cw36, onesix, cw1, timedt_turb, kmaxlim;
};

// Phase marks for wcns_profile_step: an event recorded on the context stream
// after each phase of a step enqueued outside the graph (null: no marks).
struct ProfMarks {
    int n = 0, cap = 0;
    cudaEvent_t *ev = nullptr;
    const char **name = nullptr;
};

// Wide sweeps (k_sweep_wide.cu): a chunk of whole j-rows of one block per
// CTA, plane-major arrays, rings of planes between neighbouring chunks.
constexpr int WIDE_MAX_THREADS = 512;
// 16 warps x 32 x 128 registers fill one SM's register file, four warps of
// 4,096 registers per sub-partition
constexpr int WIDE_MAX_REGS = 128;
constexpr int WIDE_COEF_WORDS = 40;  // coefficient words per slot (k_sweep_wide.cu)
struct WideChunk {
    int blk, j0, w;         // block (0-based), first j-row (0-based) and width of the chunk
    int bnd_lo, bnd_hi;     // ring between this chunk and the previous / next one (-1: none)
    long long pmoff;        // the block's first slot in the plane-major arrays
};
struct WideArrays {
    long long n = 0;        // slots per word array
    double *stat = nullptr; // WIDE_COEF_WORDS per slot: split-Jacobian coefficients, coed, srv
    double *rhs = nullptr;  // 5
    double *dql = nullptr;  // 5: lusgs_l's dq, the start of lusgs_u
    double *gs1 = nullptr;  // 15: lusgs_u -> gs_pr_l, terms of the upper neighbours
    double *gs2 = nullptr;  // 5: gs_pr_l -> gs_pr_u, summed terms of the lower neighbours
    double *sa = nullptr;   // 6: the SA model's scalar sweeps (after wcns_sa_setup)
    double *ring = nullptr; // [boundary][ring slot][nkmax][10]
    unsigned *flags = nullptr;  // [boundary][produced, consumed] plane counts
    int nbnd = 0, nkmax = 0;
};
struct WideSweep {
    WideChunk *chunks = nullptr;  // device
    std::vector<WideChunk> hchunks;
    int nchunks = 0, threads = 0;
    size_t smem_lu = 0, smem_gs = 0;
    WideArrays A;
};

struct LaunchCtx {
    ProfMarks *prof = nullptr;
    cudaStream_t stream = 0;
    long long total = 0;               // points of the field pool (stride of a field)
    // the three directions of a residual run concurrently: directions 1 and 2
    // on side streams into contribution buffers, combined in order afterwards
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    double *contrib = nullptr;         // 2 directions x 5 components x total
    const DevParams *P = nullptr;  // host copy, passed by value
    const DevFields *F = nullptr;
    DevBlock *blocks = nullptr;    // device
    const DevBlock *hblocks = nullptr;
    int nblocks = 0;
    int *err = nullptr;            // device error slots
    DirTable inv[3], vis[3];
    // mixed precision (wcns_set_precision(ctx, 32)): the residual kernels of
    // k_rhs_mixed.cu with their own line groups, and FP32 node derivatives
    // of (u,v,w,T) in the storage of the FP64 ones (12 x total floats)
    int mixed = 0;
    // lines per CTA of the inviscid / viscous residual kernels at most (the
    // tunable pencil tile, wcns_set_shape / wcns_autotune)
    int inv_cap = 32, vis_cap = 32;
    DirTable inv_mx[3], vis_mx[3];
    float *duv32 = nullptr;
    // boundary conditions
    GhostCopy *ghost = nullptr;
    long long nghost = 0;
    DevRegion *regions = nullptr;  // all regions, grouped per block in bcindex order (-1 first)
    int *reg_first = nullptr;      // per block: first region index (nblocks+1 entries), device
    int max_regions_per_block = 0;
    // SA interface rule: per interface face point (region order, i fastest)
    // the partner's point whose qke/vist go to the first ghost, and a
    // start-of-pass snapshot of those two values (2 per point)
    long long *sa_if_src = nullptr;
    double *sa_if_snap = nullptr;
    long long nsa_if = 0;
    // dq-zero list (points on physical faces)
    long long *zero_pts = nullptr;
    long long nzero = 0;
    // interface averaging
    long long *snap_pts = nullptr;  // field index of every interface face point
    int nsnap = 0;
    double *snap = nullptr;         // 6 * nsnap
    PairEntry *pairs = nullptr;     // grouped per block, region order
    int *pair_first = nullptr;      // per block (nblocks+1), device
    int *reg_pair_first = nullptr;  // per block, boundaries of its groups of independent pairs (flattened), device
    int *blk_reg_first = nullptr;   // per block, index of its first group in reg_pair_first, device
    int max_pair_regions = 0;
    int ncomp = 0, nmem = 0;
    int *comp_first = nullptr, *comp_n = nullptr, *mem_slot = nullptr;
    int *mem_comp = nullptr;        // members' writes grouped by block: component of the point
    long long *mem_idx = nullptr;   // ... and the point (field index)
    int *blk_mem_first = nullptr;   // per block (nblocks+1), first of its writes
    // residual
    double *res_partial = nullptr;  // per CTA partial sums
    int res_ctas_per_block = 0;
    double *res_out = nullptr;      // per block: res, resmax; then rms
    // LU-SGS sweeps: CTAs per block cluster, columns per CTA, threads per CTA
    int sweep_cluster = 1, sweep_cpc = 1, sweep_threads = 32, sweep_fine = 0;
    // 1: the sweeps run as one launch per hyperplane on the field layout
    // (blocks too large for the clustered kernel, or asked for)
    int sweep_plane = 0;
    // non-null: the sweeps run as wide cooperative sweeps (blocks too large
    // for the clustered kernel)
    WideSweep *wide = nullptr;
    const PmFields *PM = nullptr;  // plane-major sweep arrays
    // wall forces
    DevWall *walls = nullptr;
    int nwall = 0;
    long long nwall_quads = 0;
    double *wall_pf = nullptr, *wall_xyz = nullptr, *wall_quad = nullptr, *wall_out = nullptr;
    // update bad-point lists
    int *bad_count = nullptr;       // per block
    long long *bad_list = nullptr;  // per block, capacity BAD_CAP
    // Spalart-Allmaras model (after wcns_sa_setup)
    const SaFields *SA = nullptr;
    const SaParams *SAP = nullptr;
};

constexpr int BAD_CAP = 512;

inline void prof_mark(const LaunchCtx &c, const char *name) {
    if (!c.prof || c.prof->n >= c.prof->cap) return;
    cudaEventRecord(c.prof->ev[c.prof->n], c.stream);
    c.prof->name[c.prof->n++] = name;
}

// CTAs per block for the kernels that walk a block's BC or interface
// regions in order (one cluster per block, cluster barrier between regions)
constexpr int BC_CLUSTER = 8;

template <class... KArgs, class... Args>
inline void launch_block_clusters(void (*kern)(KArgs...), int nblocks, int threads, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(nblocks * BC_CLUSTER, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = BC_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

void launch_rhs_invis(const LaunchCtx &c, int dir, cudaStream_t st, double *out);
void setup_rhs_invis_attrs(size_t max_smem);
size_t rhs_invis_line_bytes(int n);  // shared memory of one line in k_rhs_invis
int rhs_invis_max_lines();           // lines per CTA in k_rhs_invis
void launch_node_derivatives(const LaunchCtx &c);
void launch_rhs_vis(const LaunchCtx &c, int dir, cudaStream_t st, double *out);
// all three directions of the viscous (vis = true) or inviscid residual
void launch_rhs_dirs(const LaunchCtx &c, bool vis);
void setup_rhs_vis_attrs(size_t max_smem);
size_t rhs_vis_line_bytes(int n);  // shared memory of one line in k_rhs_vis
int rhs_vis_max_lines();           // lines per CTA in k_rhs_vis
int rhs_vis_threads();            // threads per CTA in k_rhs_vis
// mixed-precision residual (k_rhs_mixed.cu)
void launch_rhs_invis_mx(const LaunchCtx &c, int dir, cudaStream_t st, double *out);
void launch_rhs_vis_mx(const LaunchCtx &c, int dir, cudaStream_t st, double *out);
void launch_node_derivatives_mx(const LaunchCtx &c);
void setup_rhs_mx_attrs(size_t inv_smem, size_t vis_smem);
size_t rhs_invis_mx_line_bytes(int n);
size_t rhs_vis_mx_line_bytes(int n);
int rhs_invis_mx_max_lines();
int rhs_vis_mx_max_lines();
// tangent and adjoint of the inviscid residual, the LU-SGS operator pair
// (k_adjoint.cu); x, v, lam, out, b, g: five arrays LaunchCtx::total apart
void launch_rhs_invis_jvp(const LaunchCtx &c, const double *v, double *out);
void launch_rhs_invis_vjp(const LaunchCtx &c, const double *lam, double *out, bool fold);
void launch_lusgs_operator(const LaunchCtx &c, double *x, const double *b, bool transpose);
void launch_adj_to_conserved(const LaunchCtx &c, double *x, const double *g);
void launch_adj_axpy(const LaunchCtx &c, double *y, const double *x);
void launch_adj_norm2(const LaunchCtx &c, const double *x, double *out);
void launch_adj_zero_faces(const LaunchCtx &c, double *x);
void launch_boundary(const LaunchCtx &c);
void launch_init(const LaunchCtx &c);
void launch_timestep(const LaunchCtx &c);
void launch_init_timestep(const LaunchCtx &c);
void launch_communicate(const LaunchCtx &c, int which /*0 dq, 1 pv*/);
int launch_lhs(const LaunchCtx &c);  // returns the number of launches
int launch_sweeps_by_plane(const LaunchCtx &c);
int setup_sweep_wide(LaunchCtx &c, WideSweep &W);  // -1: the blocks cannot be swept this way
int launch_sweeps_wide(const LaunchCtx &c);
int launch_sa_lusgs_wide(const LaunchCtx &c);  // needs wide->A.sa
int setup_sweep(LaunchCtx &c, int cluster, int fine);
int setup_sweep_exact(LaunchCtx &c, int cluster, int fine);  // -1: not valid for the blocks
constexpr int INV_LINES_DEFAULT = 32, VIS_LINES_DEFAULT = 32;
// the sweeps' bounded wait on an mbarrier nothing completes (self-test)
void launch_wait_probe(const LaunchCtx &c, long long limit);
void launch_update(const LaunchCtx &c);
void launch_forces(const LaunchCtx &c, double xref, double yref, double zref, long long q0, long long q1);
void launch_residual(const LaunchCtx &c, double *rms_slot);
// interior points of one field <-> a contiguous staging buffer (block b from first[b], device)
void launch_interior_stage(const LaunchCtx &c, bool to_device, const long long *first, double *field, double *stage);
int setup_residual(int nblocks, int ctas);  // -1 when the block count is too large
void launch_metrics(const LaunchCtx &c, double *const *xyz_dev, double *work);
// SA model: set-up (init_SA and the wall distance; xyz: 3 fields of the
// pool's layout, wall: 3 doubles per wall point) and one model step
// wall_range: per block the [begin, end) of its set's wall points (device)
void launch_sa_setup(const LaunchCtx &c, const double *xyz, const double *wall, const int *wall_range, double vt);
int launch_turbulence(const LaunchCtx &c);  // returns the number of launches

}  // namespace wcns
