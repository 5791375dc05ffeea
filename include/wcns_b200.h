/*
 * wcns_b200.h -- C ABI of the B200 (sm_100a) implementation of WCNS's
 * per-step residual (RHS) and implicit LU-SGS update (LHS) on multi-block
 * structured grids.
 *
 * The reference exposes this path as argument-less Fortran subroutines that
 * act on module globals and are called from its time loop (Main.f90:79-127).
 * Each entry point below replaces one of those calls; a Fortran driver binds
 * them with iso_c_binding.  All functions return 0 on
 * success and a nonzero WcnsStatus otherwise; wcns_last_error() gives the
 * message.  No exception crosses this boundary.  One host thread drives one
 * context; all device work of a context is ordered on the context's stream.
 *
 * Array conventions (host side): per block and per variable one double array
 * in the reference's ghosted index space (-2:n+3 in every direction), i
 * fastest, i.e. (ni+6)*(nj+6)*(nk+6) values; coordinates are interior only,
 * ni*nj*nk values, i fastest.  Block numbers are 1-based as in the reference.
 */
#ifndef WCNS_B200_H
#define WCNS_B200_H
#ifdef __cplusplus
extern "C" {
#endif

/* The param.dat namelist values the path reads ($inflow, $step, $flowtype,
 * $technic; read_parameter, PreProcess.f90:80-159).  Supported: nvis 0 or 1
 * (viscous; laminar, or turbulent once wcns_sa_setup has run), nscheme 4, 41
 * or 42, nflux 1 (Steger-Warming), 2 (Van Leer) or 3 (Roe); anything else is
 * rejected with WCNS_ERR_UNSUPPORTED. */
typedef struct WcnsParams {
    double moo, attack, sideslip, reynolds, tref, twall;
    double cfl, timedt_rate, efix, csrv;
    int nvis, nscheme, nflux, flags; /* flags: WCNS_FLAG_* bits, 0 for the defaults */
} WcnsParams;

/* Run the LU-SGS sweeps as one launch per hyperplane i+j+k on the field
 * layout.  The context does this by itself when a block has more (j,k)
 * columns than the clustered sweep kernel holds; the flag asks for it on
 * any case (same results). */
#define WCNS_FLAG_SWEEP_BY_PLANE 1
/* Run the LU-SGS sweeps as wide cooperative sweeps: chunks of whole j-rows
 * of a block per CTA, all CTAs resident, neighbouring chunks coupled through
 * rings of planes in device memory.  The context picks this by itself for
 * blocks too large for the clustered sweep kernel; the flag asks for it on
 * any case that fits (same results). */
#define WCNS_FLAG_SWEEP_WIDE 2

typedef struct WcnsContext WcnsContext;

typedef enum WcnsStatus {
    WCNS_OK = 0,
    WCNS_ERR_ARGUMENT = 1,   /* invalid input (replaces the reference's stop) */
    WCNS_ERR_ROE = 2,        /* Roe flux c^2 <= 0 (flux.f90:179-182), Van Leer c^2 < 0 (flux.f90:432-436) */
    WCNS_ERR_UPDATE = 3,     /* too many non-physical points (Sub2.f90:781-785) */
    WCNS_ERR_CUDA = 4,
    WCNS_ERR_UNSUPPORTED = 5 /* BC type or field not handled (BC.f90:203-205) */
} WcnsStatus;

/* Field identifiers for wcns_get_field / wcns_set_field. */
enum {
    WCNS_F_R = 0, WCNS_F_U, WCNS_F_V, WCNS_F_W, WCNS_F_P, WCNS_F_T,
    WCNS_F_DQ1, WCNS_F_DQ2, WCNS_F_DQ3, WCNS_F_DQ4, WCNS_F_DQ5,
    WCNS_F_DTDT, WCNS_F_SRA, WCNS_F_SRB, WCNS_F_SRC, WCNS_F_SRVA, WCNS_F_SRVB, WCNS_F_SRVC,
    WCNS_F_KCX, WCNS_F_KCY, WCNS_F_KCZ, WCNS_F_ETX, WCNS_F_ETY, WCNS_F_ETZ,
    WCNS_F_CTX, WCNS_F_CTY, WCNS_F_CTZ, WCNS_F_VOL,
    /* the Spalart-Allmaras model's fields, present after wcns_sa_setup:
     * qke (the model variable), vist (eddy viscosity), the wall distance */
    WCNS_F_QKE, WCNS_F_VIST, WCNS_F_DIST
};

/* Pre-processing.  Replaces read_bc_parallel + analyze_bc + set_bc_index
 * (parallel.f90:852-1300, PreProcess.f90:2543-2572), build_nppos_list_ex
 * (parallel.f90:2939-3018) and set_grid_derivative / GRID_DERIVATIVE_gcl
 * (WCNSE5.f90:1478-1728).  dims: 3 ints per block; xyz: 3 pointers per block
 * (x,y,z); regions: 16 ints per BC region, the integers of the 1976-format BC
 * file: nb, s_st1,s_ed1,s_st2,s_ed2,s_st3,s_ed3, bctype,
 * t_st1,t_ed1,t_st2,t_ed2,t_st3,t_ed3, nbt, ibcwin. */
int wcns_create(const WcnsParams *prm, int nblocks, const int *dims, const double *const *xyz, int nregions,
                const int *regions, WcnsContext **out);
void wcns_destroy(WcnsContext *ctx);
const char *wcns_last_error(void);

/* State transfer (init_nstart0/1, flow-file read/write PostProcess.f90:1387-1396) */
int wcns_set_prim(WcnsContext *ctx, int nb, const double *r, const double *u, const double *v, const double *w,
                  const double *p, const double *t);
int wcns_get_field(WcnsContext *ctx, int field, int nb, double *out);
/* The device address of block nb's slice of a field (the ghosted layout of
 * wcns_get_field) and its number of doubles, for exchanges that stay on the
 * device (peer copies, NCCL).  Work on the context's stream must be finished
 * (wcns_sync) before the slice is read or written another way, and that
 * access finished before the context's next call. */
int wcns_field_device_ptr(WcnsContext *ctx, int field, int nb, void **ptr, long long *count);
/* The primitive state of block nb (r, u, v, w, p, t; t may be NULL) in the
 * ghosted layout of wcns_set_prim, with one synchronisation for the block:
 * what the flow-file write reads per block (write_flow_file_parallel,
 * parallel.f90:4073-4145). */
int wcns_get_prim(WcnsContext *ctx, int nb, double *r, double *u, double *v, double *w, double *p, double *t);
/* All blocks of the context at once, one synchronisation per call: the
 * per-block loops of the set-up (init_nstart0/1 with recast_field,
 * Sub2.f90:367-405) and of the flow-file write (parallel.f90:4073-4145).
 * prim holds 6 pointers per block in block order: r, u, v, w, p, t (for
 * wcns_get_prim_all a null t skips T of that block). */
int wcns_set_prim_all(WcnsContext *ctx, const double *const *prim);
int wcns_get_prim_all(WcnsContext *ctx, double *const *prim);
/* The interior primitive state of every block in the flow-file layout of
 * write_flow_file_parallel (parallel.f90:4073-4145): per block six arrays
 * of ni*nj*nk doubles (r, u, v, w, p, t; i fastest, no ghost layers), a null
 * t skipping T of that block.  One synchronisation. */
int wcns_get_flow(WcnsContext *ctx, double *const *flow);
int wcns_set_field(WcnsContext *ctx, int field, int nb, const double *in);
/* Interior points of any of the fields above for every block, in the
 * flow-file layout (ni*nj*nk doubles per array, i fastest, no ghost
 * layers), with one synchronisation: ptrs holds nfields pointers per block
 * in block order (ptrs[nfields*(nb-1) + q] is field fields[q] of block nb); a
 * NULL pointer skips that array.  wcns_set_interior leaves every ghost point
 * as it was on the device (the next wcns_boundary_all refills the ghost
 * layers the path reads): the restart read of a flow file (init_nstart1,
 * Sub2.f90:367-405) without its ghost frame. */
int wcns_set_interior(WcnsContext *ctx, int nfields, const int *fields, const double *const *ptrs);
int wcns_get_interior(WcnsContext *ctx, int nfields, const int *fields, double *const *ptrs);

/* Per-step drop-ins, in the reference's call order (Main.f90:85-109). */
int wcns_boundary_all(WcnsContext *ctx);        /* exchange_bc + boundary_all (Main.f90:85-87) */
int wcns_initial_q_dq_c_t(WcnsContext *ctx);    /* initial_q_dq_c_t (sub_tgh.f90:1-32) */
int wcns_timestep(WcnsContext *ctx);            /* timestep_tgh (sub_tgh.f90:1270-1348) */
/* wcns_rhs_vis without the SA model step: the node derivatives and the
 * viscous flux only.  For a driver that advances the model itself
 * (wcns_turbulence) between other work in the same step, e.g. a block-
 * sharded run that refreshes its copies of other ranks' qke and vist. */
int wcns_rhs_vis_flux(WcnsContext *ctx);
int wcns_rhs_vis(WcnsContext *ctx);             /* r_h_s_vis (RHS.f90:2-30); with the SA model
                                                   set up it first runs the model step, see below */
int wcns_communicate_dq(WcnsContext *ctx);      /* communicate_dq_npp (parallel.f90:3020-3058) */
int wcns_rhs_invis(WcnsContext *ctx);           /* r_h_s_invis (RHS.f90:35-72) */
int wcns_lhs(WcnsContext *ctx);                 /* l_h_s_tgh (LHS.f90:1-34) */
int wcns_communicate_pv(WcnsContext *ctx);      /* communicate_pv_npp (parallel.f90:3166-3215) */
int wcns_residual(WcnsContext *ctx, double *res_per_block, double *resmax_per_block, double *rms);
                                                /* residual_curve (PostProcess.f90:1195-1347) */

/* Spalart-Allmaras turbulence model: turbulence(nb) -> differential_model_
 * turbulence (turblence.f90:15-103), called per block at the start of
 * r_h_s_vis (RHS.f90:22), for nlamtur=1, nameturb='SA', ncmpcor<=9, ndes=0,
 * ntrans=0, nwtmax=0.
 * wcns_sa_setup: allocates the model's arrays, computes the wall distance
 * (calc_wall_dists_parallel, parallel.f90:4313-4470) from xyz (as for
 * wcns_create), sets qke and vist to their free-stream values over the
 * points -1..n+1 (init_SA, turblence.f90:2701-2733) and keeps timedt_turb
 * ($step) and kmaxlim ($turbulence; <= 1e-15 for no clamp).  Needs nvis 1.
 * Once the model is set up:
 *   - wcns_rhs_vis runs the model step first, as r_h_s_vis calls
 *     turbulence(nb) (RHS.f90:22), and the viscous flux then uses visl+vist
 *     and visl*cp/prl + vist*cp/prt; wcns_timestep adds the eddy viscosity to
 *     the viscous spectral radii (spectvist, LHS.f90:141-241).  A driver that
 *     calls wcns_rhs_vis must not also call wcns_turbulence in the same step,
 *     or the model advances twice.
 *   - wcns_boundary_all also applies the model's one-layer qke/vist boundary
 *     rules inside each BC routine (interface copies and face means,
 *     parallel.f90:2775-2792 and Sub2.f90:262-278; far field
 *     BC_farfield_turbulence_tgh, sub_tgh.f90:713-787; inflow, outflow,
 *     wall and symmetry, BC.f90:269,416,627-640,686-721,1280,1301).
 *   - wcns_step includes all of this.
 * wcns_turbulence: one model step on every block on its own (source,
 * diffusion, spectral radius, convection, scalar LU-SGS, update of qke at
 * the interior points 2..n-1, vist at 1..n, kmaxlim clamp at 0..n), reading
 * the current prim, visl and dtdt: for drivers that sequence the model
 * themselves. */
int wcns_sa_setup(WcnsContext *ctx, const double *const *xyz, double timedt_turb, double kmaxlim);
int wcns_turbulence(WcnsContext *ctx);

/* Wall force and moment coefficients: force (PostProcess.f90:1415-1480) with
 * force_dif / getforce (1505-1824), over all bctype-2 regions.
 * ref = {sref, lfref, xref, yref, zref, nwholefield} (param.dat $force);
 * out = {cfx, cfy, cfz, cmx, cmy, cmz, cl, cd, xcp}. */
int wcns_forces(WcnsContext *ctx, const double *ref, double *out);
/* The same over the wall regions of blocks nb0..nb1 only: the forces of one
 * case when independent cases share a context. */
int wcns_forces_blocks(WcnsContext *ctx, int nb0, int nb1, const double *ref, double *out);

/* Several independent cases in one context: their blocks and BC records are
 * concatenated for wcns_create (block numbers renumbered, no interface
 * between cases), the parameters of wcns_create are common to all of them,
 * and a case at another Mach number sets it on each of its blocks here: the
 * free-stream pressure, speed of sound and the Mach-dependent constants of
 * init_inflow (PreProcess.f90:968-1113) used by the BCs, T, the heat-flux
 * coefficients and the wall forces.  The SA model's wall distance is measured
 * within each set of blocks joined through interfaces, i.e. within a case.
 * A batch of small cases then runs as one launch per kernel.  No counterpart
 * in the reference, which runs one case per job. */
int wcns_set_block_freestream(WcnsContext *ctx, int nb, double moo);

/* The whole step of Main.f90:85-109 repeated nsteps times, replayed from a
 * CUDA graph.  rms_history (may be NULL) receives the residual RMS of every
 * step.  The device error slots are read after every step: at the first step
 * where the reference would stop (too many non-physical points in
 * update_limited, Sub2.f90:781-785; Roe c^2 <= 0) the call returns the
 * error, with the step number in the message, the state is that after the
 * failing step and no later step runs. */
int wcns_step(WcnsContext *ctx, int nsteps, double *rms_history);

/* Asynchronous form for timing: enqueue nsteps graph replays on the
 * context's stream without waiting; wcns_sync waits and checks errors (an
 * error is then reported after all nsteps have run). */
int wcns_step_async(WcnsContext *ctx, int nsteps);
int wcns_sync(WcnsContext *ctx);
/* The context's CUDA stream (cudaStream_t) for event timing. */
void *wcns_stream(WcnsContext *ctx);
/* Number of kernel launches one step issues. */
int wcns_launches_per_step(WcnsContext *ctx);
/* One whole step (it advances the state like wcns_step(ctx, 1, NULL)),
 * enqueued phase by phase instead of from the graph, with a CUDA event after
 * each phase: ms[q] receives the device time of phase q and names[q] its
 * name (a static string: boundary_all, the SA model's parts, rhs_vis,
 * rhs_invis, the four LU-SGS sweeps, ...), *nphases the count (at most cap).
 * For profiling; the graph replay of wcns_step is what production runs. */
int wcns_profile_step(WcnsContext *ctx, int cap, double *ms, const char **names, int *nphases);
/* Number of points shared by more than two blocks (multi-point sets). */
int wcns_n_multipoints(WcnsContext *ctx);
/* How the context runs the LU-SGS sweeps: 0 clustered kernel (one thread-
 * block cluster per block), 1 one launch per hyperplane, 2 wide cooperative
 * sweeps (see WCNS_FLAG_SWEEP_BY_PLANE and WCNS_FLAG_SWEEP_WIDE). */
int wcns_sweep_mode(WcnsContext *ctx);
/* Arithmetic of the residual (r_h_s_vis and r_h_s_invis): 64 (default) the
 * FP64 restatement of the reference's operation order; 32 mixed precision,
 * with FP32 interpolation, fluxes, viscous derivatives and stresses while
 * the metrics, the smoothness indicators' denominators and the accumulation
 * into dq stay FP64.  The time step, the SA model, the LU-SGS sweeps and the
 * update are FP64 in both.  A precision change drops the captured step graph
 * (it is captured again at the next wcns_step).  Returns WCNS_ERR_ARGUMENT
 * for any other value. */
int wcns_set_precision(WcnsContext *ctx, int bits);
/* 64 or 32, as set by wcns_set_precision. */
int wcns_get_precision(WcnsContext *ctx);
/* Launch shapes: shape[0] CTAs per block cluster of the clustered LU-SGS
 * sweeps (0 when the context sweeps wide or by plane), shape[1] 1 for
 * sixteen lanes per (j,k) column, 0 for three, shape[2] / shape[3] lines per
 * CTA of the inviscid / viscous residual kernels at most (1..32).  No shape
 * changes a result.  wcns_set_shape returns WCNS_ERR_ARGUMENT for a shape the
 * blocks cannot run (the shape in use stays); it drops the captured step
 * graph. */
int wcns_get_shape(WcnsContext *ctx, int *shape);
/* The context device's name, compute capability and SM count (for keying
 * cached shapes), NUL-terminated in buf[len]. */
int wcns_device_name(WcnsContext *ctx, char *buf, int len);
int wcns_set_shape(WcnsContext *ctx, const int *shape);
/* Autotuner: times every candidate shape (clusters of 1, 2, 4, 8, 16 CTAs in
 * both lane modes; 4, 8, 16, 32 lines per CTA for each residual kernel) on
 * the context's current state, reps timed runs each after one warm-up, with
 * the phase each shapes (the LU-SGS phase; the inviscid and the viscous
 * residual), keeps the fastest and returns it in shape[4]; ms[3] (may be
 * NULL) receives the best device ms of those three phases.  The state is
 * not changed (dq is restored).  Takes a few hundred phase runs. */
int wcns_autotune(WcnsContext *ctx, int reps, int *shape, double *ms);

/* Tangent and adjoint of the inviscid residual and of the LU-SGS operator
 * (inviscid contexts with nscheme 4 and the Steger-Warming or Roe flux;
 * other contexts return WCNS_ERR_UNSUPPORTED).  The operands live in slots
 * of the context, five fields each in the ghosted layout of wcns_set_prim
 * (allocated on first use): */
#define WCNS_ADJ_V 0     /* tangent input: a prim-space direction (ghosts included) */
#define WCNS_ADJ_RDOT 1  /* tangent output: (dr/dq) v at the interior points */
#define WCNS_ADJ_LAM 2   /* adjoint input: lambda at the interior points */
#define WCNS_ADJ_QBAR 3  /* adjoint output: (dr/dq)^T lambda in prim space, ghosts included */
#define WCNS_ADJ_B 4     /* LU-SGS operator input */
#define WCNS_ADJ_X 5     /* LU-SGS operator output */
#define WCNS_ADJ_G 6     /* adjoint iteration: dJ/dQ, the objective's gradient in conserved variables */
#define WCNS_ADJ_PSI 7   /* adjoint iteration: the adjoint state (conserved variables) */
#define WCNS_ADJ_W 8     /* work */
#define WCNS_ADJ_NSLOTS 9
/* r is the inviscid residual of wcns_rhs_invis (dq of r_h_s_invis,
 * RHS.f90:35-72) as a function of the ghosted prim q, linearised at the
 * context's current state (run wcns_boundary_all first, and
 * wcns_initial_q_dq_c_t and wcns_timestep before the LU-SGS operator). */
int wcns_adj_set(WcnsContext *ctx, int slot, int nb, const double *const *five);
int wcns_adj_get(WcnsContext *ctx, int slot, int nb, double *const *five);
int wcns_adj_zero(WcnsContext *ctx, int slot);
/* forward: RDOT = (dr/dq) V */
int wcns_rhs_invis_tangent(WcnsContext *ctx);
/* backward: QBAR = (dr/dq)^T LAM (WCNS-E-5 transposed with its nonlinear
 * weights recomputed, the flux Jacobian applied transposed).  fold != 0:
 * interface ghosts are copies of partner points (exchange_bc), so their
 * adjoint is moved to the partner point; the ghosts of physical boundaries
 * keep their share either way (they are inputs held fixed). */
int wcns_rhs_invis_adjoint(WcnsContext *ctx, int fold);
/* X = P B (transpose 0) or X = P^T B (transpose 1), P the operator of one
 * lower and one upper LU-SGS sweep (lusgs_l, lusgs_u, LHS.f90:381-577):
 * P b = -(I + C U)^-1 (I - C L)^-1 C b over the interior points. */
int wcns_lusgs_operator(WcnsContext *ctx, int transpose);
/* iters steps of the adjoint fixed point psi <- psi + Z P^T Z (r_Q^T psi + g)
 * (r_Q: the residual's Jacobian in conserved variables; Z zeroes the points
 * of physical faces, whose dq the step zeroes before and after the sweeps),
 * whose fixed point solves Z (r_Q^T psi + g) = 0 with psi = 0 on those
 * faces; hist[iters] (may be NULL) receives the 2-norm of
 * Z (r_Q^T psi + g) before each step.  Sets the ghosts, time step and spectral
 * radii of the current state first; the state itself is not changed. */
int wcns_adjoint_iterate(WcnsContext *ctx, int iters, double *hist);
/* Failure-path self-test: runs the LU-SGS sweep's bounded wait (every wait
 * of the sweep kernels gives up after a clock-cycle limit instead of hanging)
 * on an mbarrier that nothing completes, with a limit of limit_cycles
 * (0..2^32), and returns what a step returns after a sweep wait ran out:
 * WCNS_ERR_CUDA with the message.  Nothing else is in flight; the context
 * stays usable. */
int wcns_selftest_timeout(WcnsContext *ctx, long long limit_cycles);

/* Residual norms of wcns_residual computed from caller-owned device arrays
 * without allocating any device memory.  No counterpart in the reference:
 * it exists for callers that may not call cudaMalloc/cudaFree when they need
 * the residual (a host code whose own pool allocator owns all GPU memory, a
 * call made from inside another library's callback, a fully committed memory
 * budget).
 *   fields: 7*nblocks device pointers, per block dq1..dq5, dtdt, vol, each in
 *           the ghosted layout above; dims: 3*nblocks (ni, nj, nk >= 3);
 *   res_per_block, resmax_per_block (nblocks each) and rms: host memory, any
 *           may be NULL; stream: a cudaStream_t, NULL for the default stream.
 * The partial sums live in one fixed device array of the library (about
 * 150 KB, held by every GPU that loads the library until the process exits),
 * which limits nblocks to WCNS_NOALLOC_MAX_BLOCKS; larger counts are
 * rejected with WCNS_ERR_ARGUMENT.  The first call on a device looks up that
 * array's device address and keeps it per device ordinal, which assumes one
 * CUDA context per device in the process (the runtime's primary context).
 * Every call synchronises its stream and copies the results to the host, so
 * it must not be called while its stream (or the legacy default stream) is
 * being captured into a CUDA graph.  Every call on a device shares the
 * array: calls that overlap on the GPU (other host threads, other streams)
 * race and must be serialised by the caller.  The call returns after the
 * results are on the host. */
#define WCNS_NOALLOC_MAX_BLOCKS 256
int wcns_residual_noalloc(int nblocks, const int *dims, const double *const *fields, double *res_per_block,
                          double *resmax_per_block, double *rms, void *stream);

#ifdef __cplusplus
}
#endif
#endif
