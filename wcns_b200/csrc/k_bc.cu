// k_bc.cu -- on-device boundary conditions and interface halos.
//
// boundary_all (sub_tgh.f90:123-186) -> boundary_sequence (BC.f90:169-210)
// processes, per block, interfaces first and then the physical regions in the
// order -1,4,5,6,2,3 (set_bc_index, PreProcess.f90:2543-2572).
//   * interfaces: boundary_n1_vir3 (Sub2.f90:206-322) /
//     boundary_n1_vir3_other (parallel.f90:2723-2846) copy three ghost
//     layers from the partner's interior.  The copy list is precomputed on the
//     host; every ghost point is written once and only interior points are
//     read, so one gather kernel does all blocks at once.
//   * physical regions: far field (BC.f90:460-607), supersonic inflow
//     (609-665), supersonic outflow (667-749), viscous wall (1244-1409),
//     inviscid wall (1412-1486), symmetry (227-457), with dif_average
//     (1972-2008).  Regions of one block can share edge points, so one
//     cluster per block walks its regions in order with a cluster barrier
//     between regions.
#include <cooperative_groups.h>

#include "wcns_dev.cuh"
#include "wcns_launch.h"

namespace cg = cooperative_groups;

namespace wcns {

constexpr double SA_MUOO_BC = 1.0e-1;  // muoo, the model's free-stream value (inflow_turbulence, turblence.f90:3174)

// With the SA model set up (qke != null) the same launch also takes the
// start-of-pass snapshot of qke and vist at the interface rule's source
// points (the exchange buffer qpvpack, parallel.f90:2775-2792), before the
// BC walk writes any face point.
__global__ void k_ghost_copy(DevFields F, const GhostCopy *__restrict__ list, long long n, const double *__restrict__ qke,
                             const long long *__restrict__ sa_src, double *__restrict__ sa_snap, long long nsa) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        GhostCopy g = list[e];
#pragma unroll
        for (int f = 0; f < 5; f++) F.f[F_R + f][g.dst] = F.f[F_R + f][g.src];
    }
    if (qke)
        for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nsa; e += stride) {
            const long long s = sa_src[e];
            sa_snap[2 * e] = qke[s];
            sa_snap[2 * e + 1] = F.f[F_VIST][s];
        }
}

__device__ __forceinline__ void set5(DevFields &F, long long id, double r, double u, double v, double w, double p) {
    F.f[F_R][id] = r;
    F.f[F_U][id] = u;
    F.f[F_V][id] = v;
    F.f[F_W][id] = w;
    F.f[F_P][id] = p;
}

// getnxyz_mml (Sub1.f90:750-780)
__device__ __forceinline__ void getnxyz(const DevFields &F, long long id, int is, int js, int ks, double &nx, double &ny,
                                        double &nz) {
    double x = 0.0, y = 0.0, z = 0.0;
    if (is) { x = x + F.f[F_KCX][id]; y = y + F.f[F_KCY][id]; z = z + F.f[F_KCZ][id]; }
    if (js) { x = x + F.f[F_ETX][id]; y = y + F.f[F_ETY][id]; z = z + F.f[F_ETZ][id]; }
    if (ks) { x = x + F.f[F_CTX][id]; y = y + F.f[F_CTY][id]; z = z + F.f[F_CTZ][id]; }
    double s1 = fmax(sqrt(x * x + y * y + z * z), SML_SSS);
    nx = x / s1;
    ny = y / s1;
    nz = z / s1;
}

// One cluster of BC_CLUSTER CTAs per block: the points of a region are
// spread over the whole cluster, and a cluster barrier (release/acquire at
// cluster scope, covering the global-memory writes) separates regions.
// With the SA model set up (qke != null), each BC routine also applies the
// model's one-layer qke rules where the reference calls them inside it (F:
// face point, G = F + s_lr3d the first ghost, T = F - s_lr3d):
//   interface  G <- partner (snapshot, or in place for a self-connection),
//              F <- (G + T)/2, for vist too (parallel.f90:2775-2792,
//              Sub2.f90:262-278)
//   far field  F, G <- muoo where the boundary state flows in, else T
//              (BC_farfield_turbulence_tgh, sub_tgh.f90:713-787; BC.f90:570)
//   inflow     F, G <- muoo (BC.f90:627-640)
//   outflow    F, G <- T (BC.f90:686-721)
//   wall       G <- -T, F <- (T + G)/2 (BC_wall_turbulence, BC.f90:1280,
//              BC_face_dif_turbulence 1301, turblence.f90:2238-2300)
//   symmetry   G <- T (clamped to the block in 2-D), F <- (T + G)/2
//              (BC_symmetry_turbulence BC.f90:269,416; dif_average 2002)
// Interface regions come first in a block's list (set_bc_index), so a point
// that two regions share keeps the later region's value, as in the
// reference's sequence.
__global__ void __launch_bounds__(512) k_bc_physical(DevParams P, DevFields F, const DevBlock *__restrict__ blocks,
                                                     const DevRegion *__restrict__ regions,
                                                     const int *__restrict__ reg_first, double *__restrict__ qke,
                                                     const long long *__restrict__ sa_src,
                                                     const double *__restrict__ sa_snap) {
    cg::cluster_group cluster = cg::this_cluster();
    const int bi = blockIdx.x / BC_CLUSTER;
    const int t0 = (int)cluster.block_rank() * blockDim.x + threadIdx.x, tstride = BC_CLUSTER * blockDim.x;
    const DevBlock B = blocks[bi];
    const int r0 = reg_first[bi], r1 = reg_first[bi + 1];
    double *vist = F.f[F_VIST];
    for (int r = r0; r < r1; r++) {
        const DevRegion R = regions[r];
        if (R.bctype < 0 && !qke) continue;  // uniform over the cluster: no barrier is skipped by a part of it
        const int *L = R.s_lr3d;
        const int e0 = R.s_ed[0] - R.s_st[0] + 1, e1 = R.s_ed[1] - R.s_st[1] + 1, e2 = R.s_ed[2] - R.s_st[2] + 1;
        const int npts = e0 * e1 * e2;
        const long long sL = (long long)L[0] + (long long)L[1] * B.gx + (long long)L[2] * B.gx * B.gy;
        // region-wide constant for symmetry: unit normal at the centre point
        double snx = 0.0, sny = 0.0, snz = 0.0;
        bool sym2d = false;
        if (R.bctype == 3) {
            int dims[3] = {B.ni, B.nj, B.nk};
            sym2d = dims[R.s_nd - 1] <= NIJK2D;
            if (!sym2d) {
                int ci = (R.s_st[0] + R.s_ed[0]) / 2, cj = (R.s_st[1] + R.s_ed[1]) / 2, ck = (R.s_st[2] + R.s_ed[2]) / 2;
                double nx1, ny1, nz1;
                getnxyz(F, gidx(B, ci, cj, ck), L[0], L[1], L[2], nx1, ny1, nz1);
                double sss1 = sqrt(nx1 * nx1 + ny1 * ny1 + nz1 * nz1);
                snx = nx1 / sss1;
                sny = ny1 / sss1;
                snz = nz1 / sss1;
            }
        }
        for (int t = t0; t < npts; t += tstride) {
            int i = R.s_st[0] + t % e0;
            int j = R.s_st[1] + (t / e0) % e1;
            int k = R.s_st[2] + t / (e0 * e1);
            const long long f = gidx(B, i, j, k);
            double *rr = F.f[F_R], *uu = F.f[F_U], *vv = F.f[F_V], *ww = F.f[F_W], *pp = F.f[F_P];
            switch (R.bctype) {
            case 4: {  // far field, Riemann invariants
                const double gama = P.gama;
                double nx, ny, nz;
                getnxyz(F, f, L[0], L[1], L[2], nx, ny, nz);
                long long tI = f - sL;
                double rin = rr[tI], uin = uu[tI], vin = vv[tI], win = ww[tI], pin = pp[tI];
                double s_in = pin / pow(rin, gama);
                double s_oo = B.poo / pow(P.roo, gama);
                double cin = sqrt(gama * pin / rin);
                double cg = fmax(sqrt(nx * nx + ny * ny + nz * nz), SML_SSS);
                double cgm1 = (double)R.s_lr / cg;
                double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
                double vnoo = nxa * P.uoo + nya * P.voo + nza * P.woo;
                double vnin = nxa * uin + nya * vin + nza * win;
                double mach = sqrt(uin * uin + vin * vin + win * win) / cin;
                double rb, ub, vb, wb, pb;
                if (mach < 1.0) {
                    double rp = vnin + 2.0 * cin / (gama - 1.0);
                    double rn = vnoo - 2.0 * B.coo / (gama - 1.0);
                    double vnb = 0.5 * (rp + rn);
                    double ab = 0.25 * (gama - 1.0) * (rp - rn);
                    double sb, uref, vref, wref, vnref;
                    if (vnb > 0.0) { sb = s_in; uref = uin; vref = vin; wref = win; vnref = vnin; }
                    else { sb = s_oo; uref = P.uoo; vref = P.voo; wref = P.woo; vnref = vnoo; }
                    rb = pow(ab * ab / gama / sb, 1.0 / (gama - 1.0));
                    ub = uref + nxa * (vnb - vnref);
                    vb = vref + nya * (vnb - vnref);
                    wb = wref + nza * (vnb - vnref);
                    pb = sb * pow(rb, gama);
                } else if (vnin > 0.0) {
                    rb = rin; ub = uin; vb = vin; wb = win; pb = pin;
                } else {
                    rb = P.roo; ub = P.uoo; vb = P.voo; wb = P.woo; pb = B.poo;
                }
                set5(F, f, rb, ub, vb, wb, pb);
                if (qke) {
                    // contravariant velocity of the boundary state with the
                    // face point's metrics of the face direction
                    const int m0 = F_KCX + 3 * (R.s_nd - 1);
                    double ut = (double)L[R.s_nd - 1] * (F.f[m0][f] * ub + F.f[m0 + 1][f] * vb + F.f[m0 + 2][f] * wb);
                    double qt = qke[tI];
                    qke[f] = ut < 0.0 ? SA_MUOO_BC : qt;
                    qke[f + sL] = ut < 0.0 ? SA_MUOO_BC : qt;
                }
                set5(F, f + sL, rb, ub, vb, wb, pb);
                set5(F, f + 2 * sL, rb, ub, vb, wb, pb);
                set5(F, f + 3 * sL, -rb, ub, vb, wb, pb);
                break;
            }
            case 5: {  // supersonic inflow
                for (int n = 0; n <= 3; n++) set5(F, f + n * sL, P.roo, P.uoo, P.voo, P.woo, B.poo);
                if (qke) qke[f] = qke[f + sL] = SA_MUOO_BC;
                break;
            }
            case 6: {  // supersonic outflow
                long long tI = f - sL;
                double rm = rr[tI], um = uu[tI], vm = vv[tI], wm = ww[tI], pm = pp[tI];
                for (int n = 0; n <= 3; n++) set5(F, f + n * sL, rm, um, vm, wm, pm);
                if (qke) {
                    double qt = qke[tI];
                    qke[f] = qt;
                    qke[f + sL] = qt;
                }
                break;
            }
            case 2: {
                if (P.nvis == 1) {  // viscous wall
                    long long t1 = f - sL, t2 = f - 2 * sL, t3 = f - 3 * sL;
                    set5(F, f + sL, rr[t1], -uu[t1], -vv[t1], -ww[t1], pp[t1]);
                    if (qke) {
                        qke[f + sL] = -qke[t1];
                        qke[f] = 0.5 * (qke[t1] + qke[f + sL]);
                    }
                    double pres = (4.0 * pp[t1] - pp[t2]) / 3.0;
                    double tres;
                    if (P.adiabatic) {
                        const double *tt = F.f[F_T];
                        tres = (4.0 * tt[t1] - tt[t2]) / 3.0;
                        if (pres < PMIN_LIMIT) pres = pp[t1];
                        if (tres < TMIN_LIMIT) tres = tt[t1];
                    } else {
                        if (pres < PMIN_LIMIT) pres = pp[t1];
                        tres = P.twall_nd;
                    }
                    double dres = B.moocp * pres / tres;
                    set5(F, f, dres, 0.0, 0.0, 0.0, pres);
                    set5(F, f + 2 * sL, rr[t2], -uu[t2], -vv[t2], -ww[t2], pp[t2]);
                    set5(F, f + 3 * sL, -rr[t3], -uu[t3], -vv[t3], -ww[t3], pp[t3]);
                } else {  // inviscid wall + dif_average
                    double nx, ny, nz;
                    getnxyz(F, f, L[0], L[1], L[2], nx, ny, nz);
                    for (int l = 1; l <= 3; l++) {
                        long long s = f + l * sL, tI = f - l * sL;
                        double s1 = 2.0 * (uu[tI] * nx + vv[tI] * ny + ww[tI] * nz);
                        double rv = l == 3 ? -rr[tI] : rr[tI];
                        set5(F, s, rv, uu[tI] - s1 * nx, vv[tI] - s1 * ny, ww[tI] - s1 * nz, pp[tI]);
                    }
                    long long s = f + sL, tI = f - sL;
                    set5(F, f, 0.5 * (rr[s] + rr[tI]), 0.5 * (uu[s] + uu[tI]), 0.5 * (vv[s] + vv[tI]), 0.5 * (ww[s] + ww[tI]),
                         0.5 * (pp[s] + pp[tI]));
                    if (qke) qke[f] = 0.5 * (qke[tI] + qke[s]);
                }
                break;
            }
            case 3: {  // symmetry + dif_average
                if (sym2d) {
                    int it = i - L[0], jt = j - L[1], kt = k - L[2];
                    it = it < 1 ? 1 : (it > B.ni ? B.ni : it);
                    jt = jt < 1 ? 1 : (jt > B.nj ? B.nj : jt);
                    kt = kt < 1 ? 1 : (kt > B.nk ? B.nk : kt);
                    long long tI = gidx(B, it, jt, kt);
                    if (qke) qke[f + sL] = qke[tI];
                    double rm = rr[tI], um = uu[tI], vm = vv[tI], wm = -ww[tI], pm = pp[tI];
                    set5(F, f + sL, rm, um, vm, wm, pm);
                    set5(F, f + 2 * sL, rm, um, vm, 0.0, pm);
                    set5(F, f + 3 * sL, rm, um, vm, 0.0, pm);
                } else {
                    for (int l = 1; l <= 3; l++) {
                        long long s = f + l * sL, tI = f - l * sL;
                        double s1 = 2.0 * (snx * uu[tI] + sny * vv[tI] + snz * ww[tI]);
                        set5(F, s, rr[tI], uu[tI] - s1 * snx, vv[tI] - s1 * sny, ww[tI] - s1 * snz, pp[tI]);
                        if (l == 1 && qke) qke[s] = qke[tI];
                    }
                }
                long long s = f + sL, tI = f - sL;
                set5(F, f, 0.5 * (rr[s] + rr[tI]), 0.5 * (uu[s] + uu[tI]), 0.5 * (vv[s] + vv[tI]), 0.5 * (ww[s] + ww[tI]),
                     0.5 * (pp[s] + pp[tI]));
                if (qke) qke[f] = 0.5 * (qke[tI] + qke[s]);
                break;
            }
            case -1: {  // interface: the SA model's qke/vist copy and face mean
                const long long e = R.sa_first + t, g = f + sL, tI = f - sL;
                double pv, pq;
                if (R.same) { pq = qke[sa_src[e]]; pv = vist[sa_src[e]]; }
                else { pq = sa_snap[2 * e]; pv = sa_snap[2 * e + 1]; }
                vist[g] = pv;
                vist[f] = (vist[g] + vist[tI]) * 0.5;
                qke[g] = pq;
                qke[f] = (qke[g] + qke[tI]) * 0.5;
                break;
            }
            default: break;
            }
        }
        cluster.sync();
    }
}

void launch_boundary(const LaunchCtx &c) {
    if (c.nghost > 0) {
        int grid = (int)((c.nghost + 255) / 256);
        if (grid > 148 * 16) grid = 148 * 16;
        k_ghost_copy<<<grid, 256, 0, c.stream>>>(*c.F, c.ghost, c.nghost, c.SA ? c.SA->qke : nullptr, c.sa_if_src,
                                                 c.sa_if_snap, c.nsa_if);
    }
    double *qke = c.SA ? c.SA->qke : nullptr;
    launch_block_clusters(k_bc_physical, c.nblocks, 512, c.stream, *c.P, *c.F, (const DevBlock *)c.blocks,
                          (const DevRegion *)c.regions, (const int *)c.reg_first, qke, (const long long *)c.sa_if_src,
                          (const double *)c.sa_if_snap);
}

}  // namespace wcns
