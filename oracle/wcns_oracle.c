/*
 * wcns_oracle.c -- CPU FP64 restatement of WCNS's per-step residual (RHS) and
 * implicit LU-SGS update (LHS) on multi-block structured grids.
 *
 * TEST INFRASTRUCTURE: this is the oracle the CUDA path is checked against.
 * It is never part of the product.  Parity is unpinned against the reference
 * binary (the Fortran/MPI reference cannot be built in this image and ships no
 * golden data); see wcns_oracle.h for how it is pinned instead.
 *
 * Every routine restates one reference routine with the same floating-point
 * operation order (left-to-right association as gfortran evaluates it without
 * -ffast-math; this file must be compiled with -ffp-contract=off).  Citations
 * are file:line within the reference's src/ directory.
 *
 * Storage: every per-block field uses the reference's ghosted index space
 * (-2:n+3 in each direction), i fastest, as one contiguous double array.
 */
#include "wcns_oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Globalvar.f90:215-229, Main.f90:20-21 */
#define SMALL 1.0e-38
#define SML_SSS 1.0e-30
#define PMIN_LIMIT 1.0e-8
#define PMAX_LIMIT 1.0e+3
#define RMIN_LIMIT 1.0e-8
#define RMAX_LIMIT 1.0e+3
#define TMIN_LIMIT 1.0e-8
#define NIJK2D 4
#define NIJK2ND 4
#define PAI 3.14159265

enum {
    F_R = 0, F_U, F_V, F_W, F_P, F_T,
    F_DQ1, F_DQ2, F_DQ3, F_DQ4, F_DQ5,
    F_DTDT, F_SRA, F_SRB, F_SRC, F_SRVA, F_SRVB, F_SRVC,
    F_KCX, F_KCY, F_KCZ, F_ETX, F_ETY, F_ETZ, F_CTX, F_CTY, F_CTZ, F_VOL,
    F_C, F_VISL, F_Q1, F_Q2, F_Q3, F_Q4, F_Q5, F_NFIELDS
};

static char g_err[512];
const char *orc_last_error(void) { return g_err; }
static void set_err(const char *m) { snprintf(g_err, sizeof g_err, "%s", m); }

typedef struct {
    int bctype, s_st[3], s_ed[3], s_nd, s_lr, s_lr3d[3];
    int nbt, ibcwin, t_st[3], t_ed[3], t_nd, t_lr, t_lr3d[3];
    int raw_s_st[3], raw_s_ed[3], raw_t_st[3], raw_t_ed[3];
    int *image, *jmage, *kmage;
    int iused;
} Reg;

typedef struct {
    int ni, nj, nk, gx, gy, gz;
    size_t ng;
    double *fld[F_NFIELDS];
    double *rhs[5];
    double *vist;
    /* Spalart-Allmaras model (allocated by orc_sa_setup): qke, the wall
     * distance and the model's work arrays */
    double *qke, *dist, *dqke, *spec, *viseq, *dmu[3];
    double *sa_snap; /* qke and vist at the start of the BC pass (2 x ng) */
    int nreg;
    Reg *reg;
    int *bcindex;
    double *xyz[3]; /* grid coordinates, ni*nj*nk each, i fastest (wall forces) */
} Blk;

typedef struct {
    OrcParams prm;
    double gama, prl, prt, roo, uoo, voo, woo, poo, coo, visc, reynolds;
    int nb;
    Blk *b; /* 1-based */
    /* multi-point connection sets (parallel.f90:2939-3018, 4202-4311) */
    int ncomp, nmem;
    int *comp_first, *comp_n;
    int *mem_nb, *mem_i, *mem_j, *mem_k;
    double **snap; /* per block snapshot buffer, 6 fields x ng */
    int sa;        /* 1 after orc_sa_setup */
    int sa_bc;     /* 1: boundary_all also applies the model's qke/vist rules */
    double timedt_turb, kmaxlim;
} Orc;

#define IX(B, i, j, k) ((size_t)((i) + 2) + (size_t)(B)->gx * ((size_t)((j) + 2) + (size_t)(B)->gy * (size_t)((k) + 2)))
#define R(B) ((B)->fld[F_R])
#define U(B) ((B)->fld[F_U])
#define V(B) ((B)->fld[F_V])
#define W(B) ((B)->fld[F_W])
#define P(B) ((B)->fld[F_P])
#define T(B) ((B)->fld[F_T])
#define DQ(B, m) ((B)->fld[F_DQ1 + (m)])

static int reg_box_index(const Reg *rg, int i, int j, int k) {
    int nx = rg->s_ed[0] - rg->s_st[0] + 1, ny = rg->s_ed[1] - rg->s_st[1] + 1;
    return (i - rg->s_st[0]) + nx * ((j - rg->s_st[1]) + ny * (k - rg->s_st[2]));
}

/* ------------------------------------------------------------------ */
/* Line operators                                                      */
/* ------------------------------------------------------------------ */

/* VALUE_HALF_NODE, WCNSE5.f90:799-852.  q[m + n*(i-1)], i=1..ni ->
 * qh[m + n*i], i=0..ni */
static void value_half_node(int n, int ni, const double *q, double *qh) {
#define Q(m, i) q[(m) + n * ((i) - 1)]
#define QH(m, i) qh[(m) + n * (i)]
    if (ni <= NIJK2ND) {
        for (int i = 1; i <= ni - 1; i++)
            for (int m = 0; m < n; m++) QH(m, i) = 0.5 * (Q(m, i) + Q(m, i + 1));
        for (int m = 0; m < n; m++) {
            int i2 = ni < 2 ? ni : 2, i3 = ni < 3 ? ni : 3;
            int j1 = ni - 1 > 1 ? ni - 1 : 1, j2 = ni - 2 > 1 ? ni - 2 : 1;
            QH(m, 0) = (15.0 * Q(m, 1) - 10.0 * Q(m, i2) + 3.0 * Q(m, i3)) / 8.0;
            QH(m, ni) = (15.0 * Q(m, ni) - 10.0 * Q(m, j1) + 3.0 * Q(m, j2)) / 8.0;
        }
    } else {
        for (int i = 2; i <= ni - 2; i++)
            for (int m = 0; m < n; m++)
                QH(m, i) = (9.0 * (Q(m, i) + Q(m, i + 1)) + -1.0 * (Q(m, i + 2) + Q(m, i - 1))) / 16.0;
        for (int m = 0; m < n; m++) {
            QH(m, 1) = (5.0 * Q(m, 1) + 15.0 * Q(m, 2) + -5.0 * Q(m, 3) + 1.0 * Q(m, 4)) / 16.0;
            QH(m, ni - 1) = (5.0 * Q(m, ni) + 15.0 * Q(m, ni - 1) + -5.0 * Q(m, ni - 2) + 1.0 * Q(m, ni - 3)) / 16.0;
            QH(m, 0) = (35.0 * Q(m, 1) - 35.0 * Q(m, 2) + 21.0 * Q(m, 3) - 5.0 * Q(m, 4)) / 16.0;
            QH(m, ni) = (35.0 * Q(m, ni) - 35.0 * Q(m, ni - 1) + 21.0 * Q(m, ni - 2) - 5.0 * Q(m, ni - 3)) / 16.0;
        }
    }
#undef Q
#undef QH
}

/* FLUX_DXYZ, WCNSE5.f90:209-254.  f[m + nl*i], i=0..ni -> df[m + nl*(i-1)] */
static void flux_dxyz(int nl, int ni, const double *f, double *df) {
#define FF(m, i) f[(m) + nl * (i)]
#define DF(m, i) df[(m) + nl * ((i) - 1)]
    if (ni <= NIJK2ND) {
        for (int i = 1; i <= ni; i++)
            for (int m = 0; m < nl; m++) DF(m, i) = FF(m, i) - FF(m, i - 1);
    } else {
        for (int i = 3; i <= ni - 2; i++)
            for (int m = 0; m < nl; m++)
                DF(m, i) = (2250.0 * (FF(m, i) - FF(m, i - 1)) - 125.0 * (FF(m, i + 1) - FF(m, i - 2)) +
                            9.0 * (FF(m, i + 2) - FF(m, i - 3))) / 1920.0;
        for (int m = 0; m < nl; m++) {
            DF(m, 2) = (FF(m, 0) - 27.0 * FF(m, 1) + 27.0 * FF(m, 2) - FF(m, 3)) / 24.0;
            DF(m, ni - 1) = -(FF(m, ni) - 27.0 * FF(m, ni - 1) + 27.0 * FF(m, ni - 2) - FF(m, ni - 3)) / 24.0;
            DF(m, 1) = (-23.0 * FF(m, 0) + 21.0 * FF(m, 1) + 3.0 * FF(m, 2) - FF(m, 3)) / 24.0;
            DF(m, ni) = -(-23.0 * FF(m, ni) + 21.0 * FF(m, ni - 1) + 3.0 * FF(m, ni - 2) - FF(m, ni - 3)) / 24.0;
        }
    }
#undef FF
#undef DF
}

/* ------------------------------------------------------------------ */
/* Numerical fluxes                                                    */
/* ------------------------------------------------------------------ */

/* flux_SW_pn, flux.f90:17-77 (gethmgm_ns GasModel.f90:385-399) */
static void flux_sw_pn(const Orc *o, const double *prim, double nx, double ny, double nz, double nt,
                       double *f, double efix, int npn) {
    double gama = o->gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double u2 = 0.5 * (um * um + vm * vm + wm * wm);
    double hint = gama / (gama - 1.0) * pm / rm;
    double eint = hint - pm / rm;
    double em = eint + u2;
    double hm;
    double cm = sqrt(gama * pm / rm);
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    if (!(cgm >= SML_SSS)) cgm = SML_SSS;
    double l1 = ct, l4 = ct + cm * cgm, l5 = ct - cm * cgm;
    double eps = efix * efix * cgm * cgm;
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
    hm = em + pm / rm;
    f[0] = (l1 - x1) * rm;
    f[1] = (l1 * um - x1 * um + nxa * x2) * rm;
    f[2] = (l1 * vm - x1 * vm + nya * x2) * rm;
    f[3] = (l1 * wm - x1 * wm + nza * x2) * rm;
    f[4] = (l1 * em - x1 * hm + cta * x2) * rm;
}

/* flux_SW, flux.f90:2-15 */
static void flux_sw(const Orc *o, const double *ql, const double *qr, double nx, double ny, double nz,
                    double nt, double *f, double efix) {
    double fl[5], fr[5];
    flux_sw_pn(o, ql, nx, ny, nz, nt, fl, efix, 1);
    flux_sw_pn(o, qr, nx, ny, nz, nt, fr, efix, -1);
    for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
}

/* flux_vanleer_pn, flux.f90:410-501 (gethmgm -> gethmgm_ns,
 * GasModel.f90:376-399): Van Leer's split flux of one state.  Returns
 * nonzero when c^2 < 0 (the reference stops there).  (b +- 1)**2 is
 * evaluated as a product, as gfortran does for an integer exponent 2. */
static int flux_vl_pn(const Orc *o, const double *prim, double nx, double ny, double nz, double nt, double *f,
                      int npn) {
    double gama = o->gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double u2 = 0.5 * (um * um + vm * vm + wm * wm);
    double hint = gama / (gama - 1.0) * pm / rm;
    double hm = hint + u2;
    double c2 = gama * pm / rm;
    int bad = c2 < 0.0;
    double cm = sqrt(c2);
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz) + SML_SSS;
    double cgm1 = 1.0 / cgm;
    double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
    double cta = ct * cgm1;
    double bmvl = cta / cm;
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

/* flux_vanleer, flux.f90:395-408 */
static int flux_vanleer(const Orc *o, const double *ql, const double *qr, double nx, double ny, double nz, double nt,
                        double *f) {
    double fl[5], fr[5];
    int bad = flux_vl_pn(o, ql, nx, ny, nz, nt, fl, 1);
    bad += flux_vl_pn(o, qr, nx, ny, nz, nt, fr, -1);
    for (int m = 0; m < 5; m++) f[m] = fl[m] + fr[m];
    return bad;
}

/* flux, Convect.f90:1245-1272 with getem GasModel.f90:358-374 */
static void phys_flux(double gama, const double *prim, double nx, double ny, double nz, double nt, double *f) {
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double em = pm / (gama - 1.0) + 0.5 * rm * (um * um + vm * vm + wm * wm);
    double cit = nx * um + ny * vm + nz * wm + nt;
    f[0] = rm * cit;
    f[1] = f[0] * um + nx * pm;
    f[2] = f[0] * vm + ny * pm;
    f[3] = f[0] * wm + nz * pm;
    f[4] = (em + pm) * cit - pm * nt;
}

/* flux_Roe, flux.f90:116-244.  Returns nonzero when c^2 <= 0 (the reference
 * stops there). */
static int flux_roe(const Orc *o, const double *qlin, const double *qrin, double nx, double ny, double nz,
                    double nt, double *f, double efix) {
    double gama = o->gama;
    double ql[5], qr[5], fl[5], fr[5], dq[5], qroe[5], df[5];
    memcpy(ql, qlin, sizeof ql);
    memcpy(qr, qrin, sizeof qr);
    phys_flux(gama, ql, nx, ny, nz, nt, fl);
    phys_flux(gama, qr, nx, ny, nz, nt, fr);
    for (int m = 0; m < 5; m++) dq[m] = qr[m] - ql[m];
    double gama1 = gama - 1.0;
    double gama2 = gama / gama1;
    ql[4] = gama2 * ql[4] / ql[0] + 0.5 * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
    qr[4] = gama2 * qr[4] / qr[0] + 0.5 * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    qroe[0] = sqrt(ql[0] * qr[0]);
    double rrl = sqrt(qr[0] / ql[0]);
    double rrl_1 = rrl + 1.0;
    for (int m = 1; m < 5; m++) qroe[m] = (ql[m] + qr[m] * rrl) / rrl_1;
    double rm = qroe[0], um = qroe[1], vm = qroe[2], wm = qroe[3], hm = qroe[4];
    double c2 = (hm - 0.5 * (um * um + vm * vm + wm * wm)) * gama1;
    int bad = 0;
    if (c2 <= 0.0) bad = 1;
    double c = sqrt(c2);
    double cta = um * nx + vm * ny + wm * nz + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    if (!(cgm >= SML_SSS)) cgm = SML_SSS;
    double cgm1 = 1.0 / cgm;
    nx = nx * cgm1;
    ny = ny * cgm1;
    nz = nz * cgm1;
    double ccgm = c * cgm;
    double l1 = fabs(cta - ccgm), l4 = fabs(cta), l5 = fabs(cta + ccgm);
    double l12 = l1 * l1, l42 = l4 * l4, l52 = l5 * l5;
    double deti = efix * cgm;
    double det2 = deti * deti;
    l1 = sqrt(l12 + det2);
    l4 = sqrt(l42 + det2);
    l5 = sqrt(l52 + det2);
    double dcta = dq[1] * nx + dq[2] * ny + dq[3] * nz;
    double cta1 = cta * cgm1;
    double rodcta = qroe[0] * dcta;
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
    df[0] = a4;
    df[1] = um * a4 + nx * a5 + a6;
    df[2] = vm * a4 + ny * a5 + a7;
    df[3] = wm * a4 + nz * a5 + a8;
    df[4] = hm * a4 + cta1 * a5 + um * a6 + vm * a7 + wm * a8 - c2 * a1 / gama1;
    for (int m = 0; m < 5; m++) f[m] = 0.5 * (fr[m] + fl[m] - df[m]);
    return bad;
}

/* the flux routine chosen by nflux (Convect.f90:12-46): 1 Steger-Warming,
 * 2 Van Leer, 3 Roe */
static int flux_type(const Orc *o, const double *ql, const double *qr, const double *nx4, double *f) {
    if (o->prm.nflux == 1) {
        flux_sw(o, ql, qr, nx4[0], nx4[1], nx4[2], nx4[3], f, o->prm.efix);
        return 0;
    }
    if (o->prm.nflux == 2) return flux_vanleer(o, ql, qr, nx4[0], nx4[1], nx4[2], nx4[3], f);
    return flux_roe(o, ql, qr, nx4[0], nx4[1], nx4[2], nx4[3], f, o->prm.efix);
}

/* ------------------------------------------------------------------ */
/* WCNS-E-5 line scheme: WCNS_E_5 (WCNSE5.f90:2-206, nscheme=4),       */
/* WCNS_E_5_41 (WCNSE5.f90:2087-2759, nscheme=41) and WCNS_E_5_42       */
/* (WCNSE5.f90:2766-3438, nscheme=42: the same boundary sections with   */
/* second-order states at the first four half nodes of each end,        */
/* WCNSE5.f90:2967-2986 and 3207-3226).                                 */
/* q: prim line, q[m*L + (i+2)], i=-2..n+3, L=n+6.                      */
/* nx: half-node metrics nx[c + 4*i], i=0..n.                           */
/* df: df[m + 5*(i-1)], i=1..n.  Returns count of Roe c^2<=0 events.    */
/* ------------------------------------------------------------------ */
static int wcns_line(const Orc *o, int ni, const double *q, const double *nx, double *df) {
    const double CL[3] = {1.0 / 16.0, 10.0 / 16.0, 5.0 / 16.0};
    const double CR[3] = {5.0 / 16.0, 10.0 / 16.0, 1.0 / 16.0};
    const double EPS = 1.0e-6;
    int L = ni + 6;
#define QL(m, i) q[(m) * L + (i) + 2]
    int nn = ni + 3; /* index range -1..ni+1 for g,s,wl,wr -> offset 1 */
    double *g = malloc(sizeof(double) * 5 * 3 * nn), *s = malloc(sizeof(double) * 5 * 3 * nn);
    double *wl = malloc(sizeof(double) * 5 * 3 * nn), *wr = malloc(sizeof(double) * 5 * 3 * nn);
    double *qwl = malloc(sizeof(double) * 5 * (ni + 1)), *qwr = malloc(sizeof(double) * 5 * (ni + 1));
    double *f = malloc(sizeof(double) * 5 * (ni + 1));
#define G3(a, m, n_, i) a[((m) * 3 + (n_)) * nn + (i) + 1]
#define QWL(m, i) qwl[(m) + 5 * (i)]
#define QWR(m, i) qwr[(m) + 5 * (i)]
#define FL(m, i) f[(m) + 5 * (i)]
#define DFL(m, i) df[(m) + 5 * ((i) - 1)]
    int nbad = 0;
    int ist = (QL(0, -2) < SMALL) ? 2 : 0;
    int ied = (QL(0, ni + 3) < SMALL) ? ni - 2 : ni;
    double bl[3], br[3], ql[5], qr[5], flr[5];

    for (int m = 0; m < 5; m++) {
        int i = ist - 1;
        G3(s, m, 1, i) = QL(m, i - 1) - 2.0 * QL(m, i) + QL(m, i + 1);
        G3(s, m, 2, i) = QL(m, i) - 2.0 * QL(m, i + 1) + QL(m, i + 2);
        for (i = ist; i <= ied + 1; i++) {
            G3(g, m, 0, i) = 0.5 * (QL(m, i - 2) - 4.0 * QL(m, i - 1) + 3.0 * QL(m, i));
            G3(g, m, 1, i) = 0.5 * (QL(m, i + 1) - QL(m, i - 1));
            G3(g, m, 2, i) = 0.5 * (-3.0 * QL(m, i) + 4.0 * QL(m, i + 1) - QL(m, i + 2));
            G3(s, m, 0, i) = G3(s, m, 1, i - 1);
            G3(s, m, 1, i) = G3(s, m, 2, i - 1);
            G3(s, m, 2, i) = QL(m, i) - 2.0 * QL(m, i + 1) + QL(m, i + 2);
            for (int n = 0; n < 3; n++) {
                double IS = G3(g, m, n, i) * G3(g, m, n, i) + G3(s, m, n, i) * G3(s, m, n, i);
                double t = EPS + IS;
                double EIS2 = t * t;
                bl[n] = CL[n] / EIS2;
                br[n] = CR[n] / EIS2;
            }
            double IS = bl[0] + bl[1] + bl[2];
            for (int n = 0; n < 3; n++) G3(wl, m, n, i) = bl[n] / IS;
            IS = br[0] + br[1] + br[2];
            for (int n = 0; n < 3; n++) G3(wr, m, n, i) = br[n] / IS;
        }
    }
    for (int i = ist; i <= ied; i++) {
        int i1 = i + 1;
        for (int m = 0; m < 5; m++) {
            QWL(m, i) = QL(m, i) + 0.125 * (G3(wl, m, 0, i) * (G3(s, m, 0, i) + 4.0 * G3(g, m, 0, i)) +
                                             G3(wl, m, 1, i) * (G3(s, m, 1, i) + 4.0 * G3(g, m, 1, i)) +
                                             G3(wl, m, 2, i) * (G3(s, m, 2, i) + 4.0 * G3(g, m, 2, i)));
            QWR(m, i) = QL(m, i1) + 0.125 * (G3(wr, m, 0, i1) * (G3(s, m, 0, i1) - 4.0 * G3(g, m, 0, i1)) +
                                              G3(wr, m, 1, i1) * (G3(s, m, 1, i1) - 4.0 * G3(g, m, 1, i1)) +
                                              G3(wr, m, 2, i1) * (G3(s, m, 2, i1) - 4.0 * G3(g, m, 2, i1)));
        }
    }
    if (ist > 1) {
        for (int m = 0; m < 5; m++) {
            QWL(m, 0) = (35.0 * QL(m, 1) - 35.0 * QL(m, 2) + 21.0 * QL(m, 3) - 5.0 * QL(m, 4)) / 16.0;
            QWL(m, 1) = (5.0 * QL(m, 1) + 15.0 * QL(m, 2) - 5.0 * QL(m, 3) + QL(m, 4)) / 16.0;
            QWL(m, 2) = (-QL(m, 1) + 9.0 * QL(m, 2) + 9.0 * QL(m, 3) - QL(m, 4)) / 16.0;
            QWR(m, 0) = QWL(m, 0);
            QWR(m, 1) = QWL(m, 1);
        }
    }
    if (ied < ni) {
        for (int m = 0; m < 5; m++) {
            QWR(m, ni) = (35.0 * QL(m, ni) - 35.0 * QL(m, ni - 1) + 21.0 * QL(m, ni - 2) - 5.0 * QL(m, ni - 3)) / 16.0;
            QWR(m, ni - 1) = (5.0 * QL(m, ni) + 15.0 * QL(m, ni - 1) - 5.0 * QL(m, ni - 2) + QL(m, ni - 3)) / 16.0;
            QWR(m, ni - 2) = (-QL(m, ni) + 9.0 * QL(m, ni - 1) + 9.0 * QL(m, ni - 2) - QL(m, ni - 3)) / 16.0;
            QWL(m, ni) = QWR(m, ni);
            QWL(m, ni - 1) = QWR(m, ni - 1);
        }
    }
    for (int i = 0; i <= ni; i++) {
        for (int m = 0; m < 5; m++) {
            ql[m] = QWL(m, i);
            qr[m] = QWR(m, i);
        }
        if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) {
            int ii = i > 1 ? i : 1;
            for (int m = 0; m < 5; m++) ql[m] = QL(m, ii);
        }
        if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) {
            int ii = i + 1 < ni ? i + 1 : ni;
            for (int m = 0; m < 5; m++) qr[m] = QL(m, ii);
        }
        nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
        for (int m = 0; m < 5; m++) FL(m, i) = flr[m];
    }
    flux_dxyz(5, ni, f, df);

    if (o->prm.nscheme == 41 || o->prm.nscheme == 42) {
        const int s42 = o->prm.nscheme == 42;
        double u_l_old[5][9], u_r_old[5][9];
        if (ist > 1) {
            for (int i = 1; i <= 4; i++)
                for (int m = 0; m < 5; m++) {
                    u_l_old[m][i] = QWL(m, i);
                    u_r_old[m][i] = QWR(m, i);
                }
            /* (1) boundary point 1 */
            for (int m = 0; m < 5; m++) {
                if (s42) {
                    QWL(m, 0) = (677.0 * QL(m, 1) - 421.0 * QL(m, 2) + 99.0 * QL(m, 3) + 13.0 * QL(m, 4)) / 368.0;
                    QWL(m, 1) = (5.0 * QL(m, 1) + 15.0 * QL(m, 2) - 5.0 * QL(m, 3) + QL(m, 4)) / 16.0;
                    QWL(m, 2) = (-QL(m, 1) + 9.0 * QL(m, 2) + 9.0 * QL(m, 3) - QL(m, 4)) / 16.0;
                    QWL(m, 3) = (QL(m, 1) - 5.0 * QL(m, 2) + 15.0 * QL(m, 3) + 5.0 * QL(m, 4)) / 16.0;
                } else {
                    QWL(m, 0) = (3.0 * QL(m, 1) - 1.0 * QL(m, 2) - 0. * QL(m, 3)) / 2.0;
                    QWL(m, 1) = (19.0 * QL(m, 1) + 25.0 * QL(m, 2) - 2. * QL(m, 3)) / 42.0;
                    QWL(m, 2) = (4.0 * QL(m, 1) + 3.0 * QL(m, 2) + 9.0 * QL(m, 3) + 2. * QL(m, 4)) / 18.0;
                    QWL(m, 3) = (-2.0 * QL(m, 1) + 3.0 * QL(m, 2) + 3.0 * QL(m, 3) + 2. * QL(m, 4)) / 6.0;
                }
                QWR(m, 0) = QWL(m, 0);
                QWR(m, 1) = QWL(m, 1);
                QWR(m, 2) = QWL(m, 2);
                QWR(m, 3) = QWL(m, 3);
            }
            for (int i = 0; i <= 3; i++) {
                for (int m = 0; m < 5; m++) {
                    ql[m] = QWL(m, i);
                    qr[m] = QWR(m, i);
                }
                int ia = i > 1 ? i : 1;
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT)
                    for (int m = 0; m < 5; m++) ql[m] = (QL(m, ia) + QL(m, i + 1)) / 2.;
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT)
                    for (int m = 0; m < 5; m++) qr[m] = (QL(m, ia) + QL(m, i + 1)) / 2.;
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, i) = flr[m];
            }
            for (int m = 0; m < 5; m++)
                DFL(m, 1) = (-23.0 * FL(m, 0) + 21.0 * FL(m, 1) + 3.0 * FL(m, 2) - 1.0 * FL(m, 3)) / 24.0;
            /* (2) boundary point 2 */
            for (int m = 0; m < 5; m++) {
                QWL(m, 1) = (3.0 * QL(m, 1) + 6.0 * QL(m, 2) - QL(m, 3)) / 8.0;
                QWR(m, 1) = QWL(m, 1);
                QWL(m, 2) = (-30.0 * QL(m, 1) + 145.0 * QL(m, 2) + 29.0 * QL(m, 3) - 8.0 * QL(m, 4)) / 136.0;
                QWR(m, 2) = (2.0 * QL(m, 1) + 49.0 * QL(m, 2) + 125.0 * QL(m, 3) - 40.0 * QL(m, 4)) / 136.0;
                QWL(m, 3) = (-QL(m, 2) + 6.0 * QL(m, 3) + 3.0 * QL(m, 4)) / 8.0;
                QWR(m, 3) = QWL(m, 3);
                QWL(m, 4) = (QL(m, 2) + 2.0 * QL(m, 3) + 5.0 * QL(m, 4)) / 8.0;
                QWR(m, 4) = QWL(m, 4);
                QWL(m, 5) = (QL(m, 2) + QL(m, 3) + 6.0 * QL(m, 4)) / 8.0;
                QWR(m, 5) = QWL(m, 5);
            }
            for (int i = 1; i <= 5; i++) {
                for (int m = 0; m < 5; m++) {
                    ql[m] = QWL(m, i);
                    qr[m] = QWR(m, i);
                }
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) {
                    int ia = i > 1 ? i : 1;
                    for (int m = 0; m < 5; m++) ql[m] = QL(m, ia);
                }
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) {
                    int ib = i + 1 < ni ? i + 1 : ni;
                    for (int m = 0; m < 5; m++) qr[m] = QL(m, ib);
                }
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, i) = flr[m];
            }
            for (int m = 0; m < 5; m++)
                DFL(m, 2) = (-22.0 * FL(m, 1) + 17.0 * FL(m, 2) + 9.0 * FL(m, 3) - 5.0 * FL(m, 4) + FL(m, 5)) / 24.0;
            /* (3) boundary point 3 */
            for (int m = 0; m < 5; m++) {
                QWR(m, 1) = u_r_old[m][1];
                QWL(m, 2) = (-29.0 * QL(m, 1) + 170.0 * QL(m, 2) + 63.0 * QL(m, 3) + 12.0 * QL(m, 4)) / 216.0;
                QWR(m, 2) = u_r_old[m][2];
                QWR(m, 3) = u_r_old[m][3];
                QWR(m, 4) = u_r_old[m][4];
            }
            for (int i = 1; i <= 4; i++) {
                for (int m = 0; m < 5; m++) {
                    ql[m] = QWL(m, i);
                    qr[m] = QWR(m, i);
                }
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) {
                    int ia = i > 1 ? i : 1;
                    for (int m = 0; m < 5; m++) ql[m] = QL(m, ia);
                }
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) {
                    int ib = i + 1 < ni ? i + 1 : ni;
                    for (int m = 0; m < 5; m++) qr[m] = QL(m, ib);
                }
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, i) = flr[m];
            }
            for (int m = 0; m < 5; m++) DFL(m, 3) = (FL(m, 1) - 27.0 * FL(m, 2) + 27.0 * FL(m, 3) - FL(m, 4)) / 24.0;
        }
        if (ied < ni) {
            for (int i = 1; i <= 4; i++) {
                int i1 = ni - i;
                for (int m = 0; m < 5; m++) {
                    u_l_old[m][9 - i] = QWL(m, i1);
                    u_r_old[m][9 - i] = QWR(m, i1);
                }
            }
            /* (4) boundary point N */
            for (int m = 0; m < 5; m++) {
                if (s42) {
                    QWR(m, ni) = (677.0 * QL(m, ni) - 421.0 * QL(m, ni - 1) + 99.0 * QL(m, ni - 2) + 13.0 * QL(m, ni - 3)) / 368.0;
                    QWR(m, ni - 1) = (5.0 * QL(m, ni) + 15.0 * QL(m, ni - 1) - 5.0 * QL(m, ni - 2) + QL(m, ni - 3)) / 16.0;
                    QWR(m, ni - 2) = (-QL(m, ni) + 9.0 * QL(m, ni - 1) + 9.0 * QL(m, ni - 2) - QL(m, ni - 3)) / 16.0;
                    QWR(m, ni - 3) = (QL(m, ni) - 5.0 * QL(m, ni - 1) + 15.0 * QL(m, ni - 2) + 5.0 * QL(m, ni - 3)) / 16.0;
                } else {
                    QWR(m, ni) = (3.0 * QL(m, ni) - 1.0 * QL(m, ni - 1) - 0. * QL(m, ni - 2)) / 2.0;
                    QWR(m, ni - 1) = (19.0 * QL(m, ni) + 25.0 * QL(m, ni - 1) - 2. * QL(m, ni - 2)) / 42.0;
                    QWR(m, ni - 2) = (4.0 * QL(m, ni) + 3.0 * QL(m, ni - 1) + 9.0 * QL(m, ni - 2) + 2. * QL(m, ni - 3)) / 18.0;
                    QWR(m, ni - 3) = (-2.0 * QL(m, ni) + 3.0 * QL(m, ni - 1) + 3.0 * QL(m, ni - 2) + 2. * QL(m, ni - 3)) / 6.0;
                }
                QWL(m, ni) = QWR(m, ni);
                QWL(m, ni - 1) = QWR(m, ni - 1);
                QWL(m, ni - 2) = QWR(m, ni - 2);
                QWL(m, ni - 3) = QWR(m, ni - 3);
            }
            for (int i = ni; i >= ni - 3; i--) {
                for (int m = 0; m < 5; m++) {
                    ql[m] = QWL(m, i);
                    qr[m] = QWR(m, i);
                }
                /* min(i+1,1) is 1 for every i>=0: the reference falls back on point 1 */
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT)
                    for (int m = 0; m < 5; m++) ql[m] = (QL(m, 1) + QL(m, i)) / 2.0;
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT)
                    for (int m = 0; m < 5; m++) qr[m] = (QL(m, 1) + QL(m, i)) / 2.0;
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, ni - i) = flr[m];
            }
            for (int m = 0; m < 5; m++)
                DFL(m, ni) = -(-23.0 * FL(m, 0) + 21.0 * FL(m, 1) + 3.0 * FL(m, 2) - 1.0 * FL(m, 3)) / 24.0;
            /* (5) boundary point N-1 */
            for (int m = 0; m < 5; m++) {
                QWR(m, ni - 1) = (3.0 * QL(m, ni) + 6.0 * QL(m, ni - 1) - QL(m, ni - 2)) / 8.0;
                QWL(m, ni - 1) = QWR(m, ni - 1);
                QWR(m, ni - 2) = (-30.0 * QL(m, ni) + 145.0 * QL(m, ni - 1) + 29.0 * QL(m, ni - 2) - 8.0 * QL(m, ni - 3)) / 136.0;
                QWL(m, ni - 2) = (2.0 * QL(m, ni) + 49.0 * QL(m, ni - 1) + 125.0 * QL(m, ni - 2) - 40.0 * QL(m, ni - 3)) / 136.0;
                QWR(m, ni - 3) = (-QL(m, ni - 1) + 6.0 * QL(m, ni - 2) + 3.0 * QL(m, ni - 3)) / 8.0;
                QWL(m, ni - 3) = QWR(m, ni - 3);
                QWR(m, ni - 4) = (QL(m, ni - 1) + 2.0 * QL(m, ni - 2) + 5.0 * QL(m, ni - 3)) / 8.0;
                QWL(m, ni - 4) = QWR(m, ni - 4);
                QWR(m, ni - 5) = (QL(m, ni - 1) + QL(m, ni - 2) + 6.0 * QL(m, ni - 3)) / 8.0;
                QWL(m, ni - 5) = QWR(m, ni - 5);
            }
            for (int i = ni - 1; i >= ni - 5; i--) {
                for (int m = 0; m < 5; m++) {
                    ql[m] = QWL(m, i);
                    qr[m] = QWR(m, i);
                }
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) {
                    int ia = i > 1 ? i : 1;
                    for (int m = 0; m < 5; m++) ql[m] = QL(m, ia);
                }
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) {
                    int ib = i + 1 < ni ? i + 1 : ni;
                    for (int m = 0; m < 5; m++) qr[m] = QL(m, ib);
                }
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, ni - i) = flr[m];
            }
            for (int m = 0; m < 5; m++)
                DFL(m, ni - 1) = -(-22.0 * FL(m, 1) + 17.0 * FL(m, 2) + 9.0 * FL(m, 3) - 5.0 * FL(m, 4) + FL(m, 5)) / 24.0;
            /* (6) boundary point N-2 */
            for (int m = 0; m < 5; m++) {
                QWL(m, ni - 1) = u_l_old[m][8];
                QWR(m, ni - 2) = (-29.0 * QL(m, ni) + 170.0 * QL(m, ni - 1) + 63.0 * QL(m, ni - 2) + 12.0 * QL(m, ni - 3)) / 216.0;
                QWL(m, ni - 2) = u_l_old[m][7];
                QWL(m, ni - 3) = u_l_old[m][6];
                QWL(m, ni - 4) = u_l_old[m][5];
            }
            for (int i = ni - 1; i >= ni - 4; i--) {
                for (int m = 0; m < 5; m++) {
                    qr[m] = QWR(m, i);
                    ql[m] = QWL(m, i);
                }
                if (ql[0] <= RMIN_LIMIT || ql[4] <= PMIN_LIMIT) {
                    int ia = i > 1 ? i : 1;
                    for (int m = 0; m < 5; m++) ql[m] = QL(m, ia);
                }
                if (qr[0] <= RMIN_LIMIT || qr[4] <= PMIN_LIMIT) {
                    int ib = i + 1 < ni ? i + 1 : ni;
                    for (int m = 0; m < 5; m++) qr[m] = QL(m, ib);
                }
                nbad += flux_type(o, ql, qr, &nx[4 * i], flr);
                for (int m = 0; m < 5; m++) FL(m, ni - i) = flr[m];
            }
            for (int m = 0; m < 5; m++)
                DFL(m, ni - 2) = -(FL(m, 1) - 27.0 * FL(m, 2) + 27.0 * FL(m, 3) - FL(m, 4)) / 24.0;
        }
    }
    free(g); free(s); free(wl); free(wr); free(qwl); free(qwr); free(f);
    return nbad;
#undef QL
#undef G3
#undef QWL
#undef QWR
#undef FL
#undef DFL
}

/* ------------------------------------------------------------------ */
/* Block-level helpers                                                 */
/* ------------------------------------------------------------------ */

static const double *metric_dir(const Blk *b, int d, int c) {
    /* d: 0=kc,1=et,2=ct ; c: 0=x,1=y,2=z */
    return b->fld[F_KCX + 3 * d + c];
}

/* getrkec_mml, Sub1.f90:676-717: metrics of direction d at (i,j,k), with
 * indices 0 and n+1 clamped to the block. */
static void getrkec(const Blk *b, int i, int j, int k, int d, double *g4) {
    if (i == 0) i = 1;
    if (i == b->ni + 1) i = b->ni;
    if (j == 0) j = 1;
    if (j == b->nj + 1) j = b->nj;
    if (k == 0) k = 1;
    if (k == b->nk + 1) k = b->nk;
    size_t id = IX(b, i, j, k);
    g4[0] = metric_dir(b, d, 0)[id];
    g4[1] = metric_dir(b, d, 1)[id];
    g4[2] = metric_dir(b, d, 2)[id];
    g4[3] = 0.0; /* kct=ett=ctt=0, PreProcess.f90:1639-1660 */
}

/* getnxyz_mml, Sub1.f90:750-780 */
static void getnxyz(const Blk *b, double *nx, double *ny, double *nz, int i, int j, int k, int is, int js, int ks) {
    size_t id = IX(b, i, j, k);
    double x = 0, y = 0, z = 0;
    for (int n = 1; n <= abs(is); n++) { x = x + b->fld[F_KCX][id]; y = y + b->fld[F_KCY][id]; z = z + b->fld[F_KCZ][id]; }
    for (int n = 1; n <= abs(js); n++) { x = x + b->fld[F_ETX][id]; y = y + b->fld[F_ETY][id]; z = z + b->fld[F_ETZ][id]; }
    for (int n = 1; n <= abs(ks); n++) { x = x + b->fld[F_CTX][id]; y = y + b->fld[F_CTY][id]; z = z + b->fld[F_CTZ][id]; }
    double s1 = sqrt(x * x + y * y + z * z);
    if (!(s1 >= SML_SSS)) s1 = SML_SSS;
    *nx = x / s1;
    *ny = y / s1;
    *nz = z / s1;
}

/* ------------------------------------------------------------------ */
/* Metrics: GRID_DERIVATIVE_gcl, WCNSE5.f90:1478-1728 (gcl=1)          */
/* ------------------------------------------------------------------ */
static void grid_derivative(Blk *b, const double *x, const double *y, const double *z) {
    int ni = b->ni, nj = b->nj, nk = b->nk;
    size_t np = (size_t)ni * nj * nk;
    int nmax = ni > nj ? ni : nj;
    if (nk > nmax) nmax = nk;
    double *d = calloc(18 * np, sizeof(double));
    double *xk = calloc(3 * np, sizeof(double));
    double *tem = malloc(sizeof(double) * 6 * (nmax + 2)), *temh = malloc(sizeof(double) * 6 * (nmax + 2));
    double *dt = malloc(sizeof(double) * 6 * (nmax + 2));
#define PI(i, j, k) ((size_t)((i) - 1) + (size_t)ni * ((size_t)((j) - 1) + (size_t)nj * (size_t)((k) - 1)))
#define DD(c, i, j, k) d[(size_t)(c) * np + PI(i, j, k)]
    /* coordinate derivatives along each direction */
    for (int dir = 0; dir < 3; dir++) {
        int n = dir == 0 ? ni : (dir == 1 ? nj : nk);
        int na = dir == 0 ? nj : ni, nb2 = dir == 2 ? nj : nk;
        for (int b2 = 1; b2 <= nb2; b2++)
            for (int a = 1; a <= na; a++) {
                for (int l = 1; l <= n; l++) {
                    int i = dir == 0 ? l : a, j = dir == 1 ? l : (dir == 0 ? a : b2), k = dir == 2 ? l : b2;
                    if (dir == 0) { j = a; k = b2; }
                    if (dir == 1) { i = a; k = b2; }
                    if (dir == 2) { i = a; j = b2; }
                    size_t id = PI(i, j, k);
                    tem[0 + 3 * (l - 1)] = x[id];
                    tem[1 + 3 * (l - 1)] = y[id];
                    tem[2 + 3 * (l - 1)] = z[id];
                }
                value_half_node(3, n, tem, temh);
                flux_dxyz(3, n, temh, tem);
                for (int l = 1; l <= n; l++) {
                    int i, j, k;
                    if (dir == 0) { i = l; j = a; k = b2; }
                    else if (dir == 1) { i = a; j = l; k = b2; }
                    else { i = a; j = b2; k = l; }
                    DD(dir + 0, i, j, k) = tem[0 + 3 * (l - 1)];
                    DD(dir + 3, i, j, k) = tem[1 + 3 * (l - 1)];
                    DD(dir + 6, i, j, k) = tem[2 + 3 * (l - 1)];
                }
            }
    }
    double *kcx = b->fld[F_KCX], *kcy = b->fld[F_KCY], *kcz = b->fld[F_KCZ];
    double *etx = b->fld[F_ETX], *ety = b->fld[F_ETY], *etz = b->fld[F_ETZ];
    double *ctx = b->fld[F_CTX], *cty = b->fld[F_CTY], *ctz = b->fld[F_CTZ];
    double *vol = b->fld[F_VOL];
    /* (the non-conservative metrics WCNSE5.f90:1567-1587 are overwritten by
     * the GCL branch below; only xkcetct = dx/dkc, dx/det, dx/dct survives) */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                size_t g = IX(b, i, j, k), id = PI(i, j, k);
                xk[0 * np + id] = DD(0, i, j, k);
                xk[1 * np + id] = DD(1, i, j, k);
                xk[2 * np + id] = DD(2, i, j, k);
                double xm = x[id], ym = y[id], zm = z[id];
                kcx[g] = DD(0, i, j, k) * ym;
                kcy[g] = DD(1, i, j, k) * ym;
                kcz[g] = DD(2, i, j, k) * ym;
                etx[g] = DD(3, i, j, k) * zm;
                ety[g] = DD(4, i, j, k) * zm;
                etz[g] = DD(5, i, j, k) * zm;
                ctx[g] = DD(6, i, j, k) * xm;
                cty[g] = DD(7, i, j, k) * xm;
                ctz[g] = DD(8, i, j, k) * xm;
            }
    /* Visbal conservative metrics: three directional difference passes */
    for (int dir = 0; dir < 3; dir++) {
        int n = dir == 0 ? ni : (dir == 1 ? nj : nk);
        int na = dir == 0 ? nj : ni, nb2 = dir == 2 ? nj : nk;
        for (int b2 = 1; b2 <= nb2; b2++)
            for (int a = 1; a <= na; a++) {
                for (int l = 1; l <= n; l++) {
                    int i, j, k;
                    if (dir == 0) { i = l; j = a; k = b2; }
                    else if (dir == 1) { i = a; j = l; k = b2; }
                    else { i = a; j = b2; k = l; }
                    size_t g = IX(b, i, j, k);
                    double *t6 = &tem[6 * (l - 1)];
                    if (dir == 0) { t6[0] = cty[g]; t6[1] = ctz[g]; t6[2] = kcy[g]; t6[3] = kcz[g]; t6[4] = ety[g]; t6[5] = etz[g]; }
                    else if (dir == 1) { t6[0] = ctx[g]; t6[1] = ctz[g]; t6[2] = kcx[g]; t6[3] = kcz[g]; t6[4] = etx[g]; t6[5] = etz[g]; }
                    else { t6[0] = ctx[g]; t6[1] = cty[g]; t6[2] = kcx[g]; t6[3] = kcy[g]; t6[4] = etx[g]; t6[5] = ety[g]; }
                }
                value_half_node(6, n, tem, temh);
                flux_dxyz(6, n, temh, dt);
                for (int l = 1; l <= n; l++) {
                    int i, j, k;
                    if (dir == 0) { i = l; j = a; k = b2; }
                    else if (dir == 1) { i = a; j = l; k = b2; }
                    else { i = a; j = b2; k = l; }
                    for (int m = 0; m < 6; m++) DD(6 * dir + m, i, j, k) = dt[m + 6 * (l - 1)];
                }
            }
    }
    for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++)
            for (int k = 1; k <= nk; k++) {
                size_t g = IX(b, i, j, k), id = PI(i, j, k);
                /* 1-based component c of the reference is DD(c-1) here */
                kcx[g] = DD(17, i, j, k) - DD(11, i, j, k);
                kcy[g] = DD(13, i, j, k) - DD(7, i, j, k);
                kcz[g] = DD(15, i, j, k) - DD(9, i, j, k);
                etx[g] = DD(5, i, j, k) - DD(16, i, j, k);
                ety[g] = DD(1, i, j, k) - DD(12, i, j, k);
                etz[g] = DD(3, i, j, k) - DD(14, i, j, k);
                ctx[g] = DD(10, i, j, k) - DD(4, i, j, k);
                cty[g] = DD(6, i, j, k) - DD(0, i, j, k);
                ctz[g] = DD(8, i, j, k) - DD(2, i, j, k);
                vol[g] = xk[0 * np + id] * kcx[g] + xk[1 * np + id] * etx[g] + xk[2 * np + id] * ctx[g];
            }
#undef PI
#undef DD
    free(d); free(xk); free(tem); free(temh); free(dt);
}

/* ------------------------------------------------------------------ */
/* BC preprocessing: analyze_bc / analyze_bc_connect (parallel.f90:1123-1300),
 * set_bc_index (PreProcess.f90:2543-2572)                              */
/* ------------------------------------------------------------------ */
static int analyze_regions(Orc *o) {
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int nr = 0; nr < b->nreg; nr++) {
            Reg *rg = &b->reg[nr];
            int s_nd = 0, s_lr = 0;
            for (int m = 0; m < 3; m++) {
                int a = abs(rg->raw_s_st[m]), c = abs(rg->raw_s_ed[m]);
                rg->s_st[m] = a < c ? a : c;
                rg->s_ed[m] = a > c ? a : c;
                rg->s_lr3d[m] = 0;
                if (rg->raw_s_st[m] == rg->raw_s_ed[m]) {
                    s_nd = m + 1;
                    if (rg->raw_s_st[m] == 1) { s_lr = -1; rg->s_lr3d[m] = -1; }
                    else { s_lr = 1; rg->s_lr3d[m] = 1; }
                }
            }
            rg->s_nd = s_nd;
            rg->s_lr = s_lr;
            if (rg->bctype < 0) {
                int t_nd = 0, t_lr = 0, std[3][3] = {{0}};
                int s_st[3], s_ed[3], t_st[3], t_ed[3], s_sign[3], t_sign[3], st_sign[3];
                for (int m = 0; m < 3; m++) {
                    rg->t_lr3d[m] = 0;
                    if (rg->raw_t_st[m] == rg->raw_t_ed[m]) {
                        t_nd = m + 1;
                        if (rg->raw_t_st[m] == 1) { t_lr = -1; rg->t_lr3d[m] = -1; }
                        else { t_lr = 1; rg->t_lr3d[m] = 1; }
                    }
                }
                rg->t_nd = t_nd;
                rg->t_lr = t_lr;
                for (int m = 1; m <= 3; m++) {
                    int done = 0;
                    for (int n = 1; n <= 3; n++) {
                        if (m != s_nd && n != t_nd) {
                            int js1 = rg->raw_s_st[m - 1];
                            if (abs(js1) < abs(rg->raw_s_ed[m - 1])) js1 = rg->raw_s_ed[m - 1];
                            int js2 = rg->raw_t_st[n - 1];
                            if (abs(js2) < abs(rg->raw_t_ed[n - 1])) js2 = rg->raw_t_ed[n - 1];
                            if ((long)js1 * js2 > 0) {
                                std[n - 1][m - 1] = 1;
                                std[t_nd - 1][s_nd - 1] = 1;
                                std[6 - n - t_nd - 1][6 - m - s_nd - 1] = 1;
                                done = 1;
                                break;
                            }
                        }
                    }
                    if (done) break;
                }
                for (int m = 0; m < 3; m++) {
                    s_sign[m] = 1;
                    s_st[m] = abs(rg->raw_s_st[m]);
                    s_ed[m] = abs(rg->raw_s_ed[m]);
                    if (m + 1 != s_nd && s_st[m] > s_ed[m]) s_sign[m] = -1;
                    t_sign[m] = 1;
                    t_st[m] = abs(rg->raw_t_st[m]);
                    t_ed[m] = abs(rg->raw_t_ed[m]);
                    if (m + 1 != t_nd && t_st[m] > t_ed[m]) t_sign[m] = -1;
                }
                for (int m = 0; m < 3; m++) {
                    int co = 0;
                    for (int n = 0; n < 3; n++)
                        if (std[n][m] == 1) co = n + 1;
                    if (co == 0) { set_err("interface direction mapping failed"); return -1; }
                    st_sign[m] = t_sign[co - 1] * s_sign[m];
                }
                int nbox = (rg->s_ed[0] - rg->s_st[0] + 1) * (rg->s_ed[1] - rg->s_st[1] + 1) * (rg->s_ed[2] - rg->s_st[2] + 1);
                rg->image = malloc(sizeof(int) * nbox);
                rg->jmage = malloc(sizeof(int) * nbox);
                rg->kmage = malloc(sizeof(int) * nbox);
                for (int i = s_st[0];; i += s_sign[0]) {
                    int idelt = (i - s_st[0]) * st_sign[0];
                    for (int j = s_st[1];; j += s_sign[1]) {
                        int jdelt = (j - s_st[1]) * st_sign[1];
                        for (int k = s_st[2];; k += s_sign[2]) {
                            int kdelt = (k - s_st[2]) * st_sign[2];
                            int bi = reg_box_index(rg, i, j, k);
                            rg->image[bi] = t_st[0] + std[0][0] * idelt + std[0][1] * jdelt + std[0][2] * kdelt;
                            rg->jmage[bi] = t_st[1] + std[1][0] * idelt + std[1][1] * jdelt + std[1][2] * kdelt;
                            rg->kmage[bi] = t_st[2] + std[2][0] * idelt + std[2][1] * jdelt + std[2][2] * kdelt;
                            if (k == s_ed[2]) break;
                        }
                        if (j == s_ed[1]) break;
                    }
                    if (i == s_ed[0]) break;
                }
                for (int m = 0; m < 3; m++) {
                    int a = abs(rg->raw_t_st[m]), c = abs(rg->raw_t_ed[m]);
                    rg->t_st[m] = a < c ? a : c;
                    rg->t_ed[m] = a > c ? a : c;
                }
                if (rg->nbt < 1 || rg->nbt > o->nb) { set_err("interface target block out of range"); return -1; }
            }
        }
        /* set_bc_index */
        static const int order[6] = {-1, 4, 5, 6, 2, 3};
        b->bcindex = malloc(sizeof(int) * b->nreg);
        int cnt = 0;
        for (int l = 0; l < 6; l++)
            for (int nr = 0; nr < b->nreg; nr++)
                if (b->reg[nr].bctype == order[l]) b->bcindex[cnt++] = nr;
        if (cnt != b->nreg) { set_err("unsupported BC type (only -1,2,3,4,5,6)"); return -1; }
    }
    return 0;
}

/* connect_pre_parallel + comp_list_insert + build_nppos_list_ex
 * (parallel.f90:177-393, 2939-3018, 4202-4311) */
typedef struct { int nbijk[4]; } Pt;
typedef struct { Pt *p; int n, cap; } PtList;
static void ptl_push(PtList *l, const int *v) {
    if (l->n == l->cap) { l->cap = l->cap ? 2 * l->cap : 4; l->p = realloc(l->p, sizeof(Pt) * l->cap); }
    memcpy(l->p[l->n].nbijk, v, 4 * sizeof(int));
    l->n++;
}
static int ptl_has(const PtList *l, const int *v) {
    for (int i = 0; i < l->n; i++)
        if (!memcmp(l->p[i].nbijk, v, 4 * sizeof(int))) return 1;
    return 0;
}
static void build_multipoints(Orc *o) {
    for (int nb = 1; nb <= o->nb; nb++)
        for (int nr = 0; nr < o->b[nb].nreg; nr++) o->b[nb].reg[nr].iused = 0;
    for (int nb = 1; nb <= o->nb; nb++)
        for (int nr = 0; nr < o->b[nb].nreg; nr++) {
            Reg *rg = &o->b[nb].reg[nr];
            if (rg->bctype < 0 && rg->iused == 0) {
                rg->iused = 1;
                int nrt = rg->ibcwin;
                if (nrt >= 1 && nrt <= o->b[rg->nbt].nreg) o->b[rg->nbt].reg[nrt - 1].iused = -1;
            }
        }
    PtList *comps = NULL;
    int ncomps = 0;
    for (int nb = 1; nb <= o->nb; nb++)
        for (int nr = 0; nr < o->b[nb].nreg; nr++) {
            Reg *rg = &o->b[nb].reg[nr];
            if (rg->bctype >= 0 || rg->iused != 1) continue;
            int idir = rg->s_nd;
            static const int mcyc[5] = {1, 2, 3, 1, 2};
            int d2 = mcyc[idir] - 1, d3 = mcyc[idir + 1] - 1;
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                        int c[3] = {i, j, k};
                        int inner = c[d2] >= rg->s_st[d2] + 1 && c[d2] <= rg->s_ed[d2] - 1 &&
                                    c[d3] >= rg->s_st[d3] + 1 && c[d3] <= rg->s_ed[d3] - 1;
                        if (inner) continue;
                        int bi = reg_box_index(rg, i, j, k);
                        int a[4] = {nb, i, j, k};
                        int t[4] = {rg->nbt, rg->image[bi], rg->jmage[bi], rg->kmage[bi]};
                        int ok = 0;
                        for (int cidx = 0; cidx < ncomps && !ok; cidx++) {
                            PtList *cl = &comps[cidx];
                            int e = ptl_has(cl, a), et = ptl_has(cl, t);
                            if (e || et) {
                                if (!e) ptl_push(cl, a);
                                if (!et) ptl_push(cl, t);
                                ok = 1;
                            }
                        }
                        if (!ok) {
                            comps = realloc(comps, sizeof(PtList) * (ncomps + 1));
                            memset(&comps[ncomps], 0, sizeof(PtList));
                            ptl_push(&comps[ncomps], a);
                            ptl_push(&comps[ncomps], t);
                            ncomps++;
                        }
                    }
        }
    int nc = 0, nm = 0;
    for (int c = 0; c < ncomps; c++)
        if (comps[c].n > 2) { nc++; nm += comps[c].n; }
    o->ncomp = nc;
    o->nmem = nm;
    o->comp_first = malloc(sizeof(int) * (nc + 1));
    o->comp_n = malloc(sizeof(int) * (nc + 1));
    o->mem_nb = malloc(sizeof(int) * (nm + 1));
    o->mem_i = malloc(sizeof(int) * (nm + 1));
    o->mem_j = malloc(sizeof(int) * (nm + 1));
    o->mem_k = malloc(sizeof(int) * (nm + 1));
    int ci = 0, mi = 0;
    for (int c = 0; c < ncomps; c++) {
        if (comps[c].n > 2) {
            o->comp_first[ci] = mi;
            o->comp_n[ci] = comps[c].n;
            for (int q = 0; q < comps[c].n; q++) {
                o->mem_nb[mi] = comps[c].p[q].nbijk[0];
                o->mem_i[mi] = comps[c].p[q].nbijk[1];
                o->mem_j[mi] = comps[c].p[q].nbijk[2];
                o->mem_k[mi] = comps[c].p[q].nbijk[3];
                mi++;
            }
            ci++;
        }
        free(comps[c].p);
    }
    free(comps);
}

int orc_n_multipoints(void *h) { return ((Orc *)h)->ncomp; }

/* ------------------------------------------------------------------ */
/* Creation                                                            */
/* ------------------------------------------------------------------ */
void *orc_create(const OrcParams *prm, int nblocks, const int *dims, const double *const *xyz, int nregions,
                 const int *regions) {
    Orc *o = calloc(1, sizeof(Orc));
    o->prm = *prm;
    /* read_perfect_gasmodel GasModel.f90:184-217 */
    o->gama = 1.40;
    o->prl = 0.72;
    o->prt = 0.90;
    /* init_inflow PreProcess.f90:968-1113 with lfref=lref=1, height<0 */
    double attack = prm->attack * PAI / 180.0, sideslip = prm->sideslip * PAI / 180.0;
    o->uoo = cos(attack) * cos(sideslip);
    o->voo = sin(attack) * cos(sideslip);
    o->woo = sin(sideslip);
    o->roo = 1.0;
    o->reynolds = (prm->reynolds / 1.0) * 1.0;
    o->poo = 1.0 / (o->gama * prm->moo * prm->moo);
    o->coo = sqrt(o->gama * o->poo / o->roo);
    o->visc = 110.4 / prm->tref;
    o->nb = nblocks;
    o->b = calloc(nblocks + 1, sizeof(Blk));
    o->snap = calloc(nblocks + 1, sizeof(double *));
    for (int nb = 1; nb <= nblocks; nb++) {
        Blk *b = &o->b[nb];
        b->ni = dims[3 * (nb - 1)];
        b->nj = dims[3 * (nb - 1) + 1];
        b->nk = dims[3 * (nb - 1) + 2];
        b->gx = b->ni + 6;
        b->gy = b->nj + 6;
        b->gz = b->nk + 6;
        b->ng = (size_t)b->gx * b->gy * b->gz;
        for (int f = 0; f < F_NFIELDS; f++) b->fld[f] = calloc(b->ng, sizeof(double));
        for (int m = 0; m < 5; m++) b->rhs[m] = calloc(b->ng, sizeof(double));
        b->vist = calloc(b->ng, sizeof(double));
        o->snap[nb] = calloc(6 * b->ng, sizeof(double));
    }
    for (int r = 0; r < nregions; r++) {
        const int *rr = &regions[16 * r];
        int nb = rr[0];
        if (nb < 1 || nb > nblocks) { set_err("region block out of range"); orc_destroy(o); return NULL; }
        o->b[nb].nreg++;
    }
    for (int nb = 1; nb <= nblocks; nb++) {
        o->b[nb].reg = calloc(o->b[nb].nreg > 0 ? o->b[nb].nreg : 1, sizeof(Reg));
        o->b[nb].nreg = 0;
    }
    for (int r = 0; r < nregions; r++) {
        const int *rr = &regions[16 * r];
        Blk *b = &o->b[rr[0]];
        Reg *rg = &b->reg[b->nreg++];
        rg->raw_s_st[0] = rr[1]; rg->raw_s_ed[0] = rr[2];
        rg->raw_s_st[1] = rr[3]; rg->raw_s_ed[1] = rr[4];
        rg->raw_s_st[2] = rr[5]; rg->raw_s_ed[2] = rr[6];
        rg->bctype = rr[7];
        rg->raw_t_st[0] = rr[8]; rg->raw_t_ed[0] = rr[9];
        rg->raw_t_st[1] = rr[10]; rg->raw_t_ed[1] = rr[11];
        rg->raw_t_st[2] = rr[12]; rg->raw_t_ed[2] = rr[13];
        rg->nbt = rr[14];
        rg->ibcwin = rr[15];
    }
    if (analyze_regions(o)) { orc_destroy(o); return NULL; }
    build_multipoints(o);
    for (int nb = 1; nb <= nblocks; nb++) grid_derivative(&o->b[nb], xyz[3 * (nb - 1)], xyz[3 * (nb - 1) + 1], xyz[3 * (nb - 1) + 2]);
    for (int nb = 1; nb <= nblocks; nb++) {
        Blk *b = &o->b[nb];
        size_t np = (size_t)b->ni * b->nj * b->nk;
        for (int c = 0; c < 3; c++) {
            b->xyz[c] = malloc(np * sizeof(double));
            memcpy(b->xyz[c], xyz[3 * (nb - 1) + c], np * sizeof(double));
        }
    }
    return o;
}

void orc_destroy(void *h) {
    Orc *o = h;
    if (!o) return;
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int f = 0; f < F_NFIELDS; f++) free(b->fld[f]);
        for (int m = 0; m < 5; m++) free(b->rhs[m]);
        free(b->vist);
        free(b->qke); free(b->dist); free(b->dqke); free(b->spec); free(b->viseq); free(b->sa_snap);
        for (int c = 0; c < 3; c++) free(b->dmu[c]);
        for (int c = 0; c < 3; c++) free(b->xyz[c]);
        for (int nr = 0; nr < b->nreg; nr++) { free(b->reg[nr].image); free(b->reg[nr].jmage); free(b->reg[nr].kmage); }
        free(b->reg);
        free(b->bcindex);
        free(o->snap[nb]);
    }
    free(o->b); free(o->snap);
    free(o->comp_first); free(o->comp_n); free(o->mem_nb); free(o->mem_i); free(o->mem_j); free(o->mem_k);
    free(o);
}

int orc_set_prim(void *h, int nb, const double *r, const double *u, const double *v, const double *w,
                 const double *p, const double *t) {
    Orc *o = h;
    if (nb < 1 || nb > o->nb) return -1;
    Blk *b = &o->b[nb];
    memcpy(b->fld[F_R], r, b->ng * 8);
    memcpy(b->fld[F_U], u, b->ng * 8);
    memcpy(b->fld[F_V], v, b->ng * 8);
    memcpy(b->fld[F_W], w, b->ng * 8);
    memcpy(b->fld[F_P], p, b->ng * 8);
    memcpy(b->fld[F_T], t, b->ng * 8);
    return 0;
}
/* field numbers past the path's 28 fields: the SA model's qke, vist and wall
 * distance (present after orc_sa_setup), then c, visl, q1..q5 */
enum { F_X_QKE = 28, F_X_VIST = 29, F_X_DIST = 30, F_X_C = 31 };
static double *field_ptr(const Orc *o, Blk *b, int field) {
    if (field >= 0 && field <= F_VOL) return b->fld[field];
    if (field >= F_X_C && field < F_X_C + (F_NFIELDS - F_C)) return b->fld[F_C + (field - F_X_C)];
    if (!o->sa) return NULL;
    if (field == F_X_QKE) return b->qke;
    if (field == F_X_VIST) return b->vist;
    if (field == F_X_DIST) return b->dist;
    return NULL;
}
int orc_get_field(void *h, int field, int nb, double *out) {
    Orc *o = h;
    if (nb < 1 || nb > o->nb) return -1;
    double *f = field_ptr(o, &o->b[nb], field);
    if (!f) return -1;
    memcpy(out, f, o->b[nb].ng * 8);
    return 0;
}
int orc_set_field(void *h, int field, int nb, const double *in) {
    Orc *o = h;
    if (nb < 1 || nb > o->nb) return -1;
    double *f = field_ptr(o, &o->b[nb], field);
    if (!f) return -1;
    memcpy(f, in, o->b[nb].ng * 8);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Boundary conditions: boundary_all -> boundary_sequence               */
/* (sub_tgh.f90:123-186, BC.f90:169-210)                                */
/* ------------------------------------------------------------------ */
#define SET5(B, id, a, bb, c, d, e) do { R(B)[id] = (a); U(B)[id] = (bb); V(B)[id] = (c); W(B)[id] = (d); P(B)[id] = (e); } while (0)

#define SA_MUOO_BC 1.0e-1 /* muoo, inflow_turbulence turblence.f90:3174 */

/* The SA model's one-layer boundary rules for qke and vist, applied when
 * o->sa_bc is set, point by point where the reference calls them inside each
 * BC routine.  F: face point, G: first ghost, T: interior neighbour. */
#define SA_BC(o) ((o)->sa && (o)->sa_bc)
/* BC_face_dif_turbulence, turblence.f90:2255-2267: face <- (T + G) / 2 */
static void sa_face_dif(Blk *b, size_t f, size_t g, size_t t) { b->qke[f] = 0.5 * (b->qke[t] + b->qke[g]); }

/* boundary_n1_vir3 (Sub2.f90:206-322) / boundary_n1_vir3_other
 * (parallel.f90:2723-2846): ghost layers from the partner's interior. */
static void bc_vir3(Orc *o, int nb, Reg *rg) {
    Blk *b = &o->b[nb];
    Blk *bt = &o->b[rg->nbt];
    int same = (rg->nbt == nb);
    const double *sr, *su, *sv, *sw, *sp;
    if (same) { sr = R(bt); su = U(bt); sv = V(bt); sw = W(bt); sp = P(bt); }
    else {
        double *s = o->snap[rg->nbt];
        sr = s; su = s + bt->ng; sv = s + 2 * bt->ng; sw = s + 3 * bt->ng; sp = s + 4 * bt->ng;
    }
    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) {
                int bi = reg_box_index(rg, i, j, k);
                int it = rg->image[bi], jt = rg->jmage[bi], kt = rg->kmage[bi];
                int is = i, js = j, ks = k;
                if (SA_BC(o) && (!same || o->prm.nvis == 1)) {
                    /* parallel.f90:2775-2792 (Sub2.f90:262-278 in place, only
                     * with nvis = 1 there, Sub2.f90:224-228): the
                     * first ghost takes the partner's vist and qke, the face
                     * point the mean of that ghost and its interior neighbour */
                    size_t g = IX(b, i + rg->s_lr3d[0], j + rg->s_lr3d[1], k + rg->s_lr3d[2]);
                    size_t f = IX(b, i, j, k), t = IX(b, i - rg->s_lr3d[0], j - rg->s_lr3d[1], k - rg->s_lr3d[2]);
                    size_t ps = IX(bt, it - rg->t_lr3d[0], jt - rg->t_lr3d[1], kt - rg->t_lr3d[2]);
                    const double *pq = same ? bt->qke : o->b[rg->nbt].sa_snap;
                    const double *pv = same ? bt->vist : o->b[rg->nbt].sa_snap + bt->ng;
                    b->vist[g] = pv[ps];
                    b->vist[f] = (b->vist[g] + b->vist[t]) * 0.5;
                    b->qke[g] = pq[ps];
                    b->qke[f] = (b->qke[g] + b->qke[t]) * 0.5;
                }
                for (int l = 1; l <= 3; l++) {
                    is += rg->s_lr3d[0]; js += rg->s_lr3d[1]; ks += rg->s_lr3d[2];
                    it -= rg->t_lr3d[0]; jt -= rg->t_lr3d[1]; kt -= rg->t_lr3d[2];
                    size_t d = IX(b, is, js, ks), s = IX(bt, it, jt, kt);
                    double rr = sr[s];
                    if (l == 3) rr = sr[s] * (double)(1 - 2 * 0); /* cic1 = 0 */
                    SET5(b, d, rr, su[s], sv[s], sw[s], sp[s]);
                }
            }
}

/* dif_average, BC.f90:1972-2008 */
static void bc_dif_average(const Orc *o, Blk *b, Reg *rg) {
    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) {
                size_t f = IX(b, i, j, k);
                size_t s = IX(b, i + rg->s_lr3d[0], j + rg->s_lr3d[1], k + rg->s_lr3d[2]);
                size_t t = IX(b, i - rg->s_lr3d[0], j - rg->s_lr3d[1], k - rg->s_lr3d[2]);
                R(b)[f] = 0.5 * (R(b)[s] + R(b)[t]);
                U(b)[f] = 0.5 * (U(b)[s] + U(b)[t]);
                V(b)[f] = 0.5 * (V(b)[s] + V(b)[t]);
                W(b)[f] = 0.5 * (W(b)[s] + W(b)[t]);
                P(b)[f] = 0.5 * (P(b)[s] + P(b)[t]);
                if (SA_BC(o)) sa_face_dif(b, f, s, t);
            }
}

/* boundary_3 (symmetry), BC.f90:227-457 */
static void bc_symmetry(Orc *o, Blk *b, Reg *rg) {
    int dims[3] = {b->ni, b->nj, b->nk};
    const int *L = rg->s_lr3d;
    if (dims[rg->s_nd - 1] <= NIJK2D) {
        for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
            for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                    int is = i + L[0], js = j + L[1], ks = k + L[2];
                    int it = i - L[0], jt = j - L[1], kt = k - L[2];
                    it = it < 1 ? 1 : (it > b->ni ? b->ni : it);
                    jt = jt < 1 ? 1 : (jt > b->nj ? b->nj : jt);
                    kt = kt < 1 ? 1 : (kt > b->nk ? b->nk : kt);
                    size_t t = IX(b, it, jt, kt);
                    if (SA_BC(o)) b->qke[IX(b, is, js, ks)] = b->qke[t]; /* BC_symmetry_turbulence, BC.f90:269 */
                    double rm = R(b)[t], um = U(b)[t], vm = V(b)[t], wm = -W(b)[t], pm = P(b)[t];
                    SET5(b, IX(b, is, js, ks), rm, um, vm, wm, pm);
                    is += L[0]; js += L[1]; ks += L[2];
                    wm = 0.0;
                    SET5(b, IX(b, is, js, ks), rm, um, vm, wm, pm);
                    is += L[0]; js += L[1]; ks += L[2];
                    wm = 0.0;
                    SET5(b, IX(b, is, js, ks), rm, um, vm, wm, pm);
                }
        bc_dif_average(o, b, rg);
        return;
    }
    int ci = (rg->s_st[0] + rg->s_ed[0]) / 2, cj = (rg->s_st[1] + rg->s_ed[1]) / 2, ck = (rg->s_st[2] + rg->s_ed[2]) / 2;
    double nx1, ny1, nz1;
    getnxyz(b, &nx1, &ny1, &nz1, ci, cj, ck, L[0], L[1], L[2]);
    double sss1 = sqrt(nx1 * nx1 + ny1 * ny1 + nz1 * nz1);
    double nx = nx1 / sss1, ny = ny1 / sss1, nz = nz1 / sss1;
    for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                int is = i + L[0], js = j + L[1], ks = k + L[2];
                int it = i - L[0], jt = j - L[1], kt = k - L[2];
                for (int l = 1; l <= 3; l++) {
                    if (l > 1) { is += L[0]; js += L[1]; ks += L[2]; it -= L[0]; jt -= L[1]; kt -= L[2]; }
                    size_t t = IX(b, it, jt, kt), s = IX(b, is, js, ks);
                    double s1 = 2.0 * (nx * U(b)[t] + ny * V(b)[t] + nz * W(b)[t]);
                    SET5(b, s, R(b)[t], U(b)[t] - s1 * nx, V(b)[t] - s1 * ny, W(b)[t] - s1 * nz, P(b)[t]);
                    if (l == 1 && SA_BC(o)) b->qke[s] = b->qke[t]; /* BC_symmetry_turbulence, BC.f90:416 */
                }
            }
    bc_dif_average(o, b, rg);
}

/* boundary_4 (far field, Riemann invariants), BC.f90:460-607 */
static void bc_farfield(Orc *o, Blk *b, Reg *rg) {
    const int *L = rg->s_lr3d;
    double gama = o->gama;
    int lr = rg->s_lr;
    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) {
                int it = i - L[0], jt = j - L[1], kt = k - L[2];
                double nx, ny, nz;
                getnxyz(b, &nx, &ny, &nz, i, j, k, L[0], L[1], L[2]);
                size_t t = IX(b, it, jt, kt);
                double rin = R(b)[t], uin = U(b)[t], vin = V(b)[t], win = W(b)[t], pin = P(b)[t];
                double s_in = pin / pow(rin, gama);
                double s_oo = o->poo / pow(o->roo, gama);
                double cin = sqrt(gama * pin / rin);
                double cg = sqrt(nx * nx + ny * ny + nz * nz);
                if (!(cg >= SML_SSS)) cg = SML_SSS;
                double cgm1 = lr / cg;
                double nxa = nx * cgm1, nya = ny * cgm1, nza = nz * cgm1;
                double vnoo = nxa * o->uoo + nya * o->voo + nza * o->woo;
                double vnin = nxa * uin + nya * vin + nza * win;
                double mach = sqrt(uin * uin + vin * vin + win * win) / cin;
                double rb, ub, vb, wb, pb;
                if (mach < 1.0) {
                    double rp = vnin + 2.0 * cin / (gama - 1.0);
                    double rn = vnoo - 2.0 * o->coo / (gama - 1.0);
                    double vnb = 0.5 * (rp + rn);
                    double ab = 0.25 * (gama - 1.0) * (rp - rn);
                    double sb, uref, vref, wref, vnref;
                    if (vnb > 0.0) { sb = s_in; uref = uin; vref = vin; wref = win; vnref = vnin; }
                    else { sb = s_oo; uref = o->uoo; vref = o->voo; wref = o->woo; vnref = vnoo; }
                    rb = pow(ab * ab / gama / sb, 1.0 / (gama - 1.0));
                    ub = uref + nxa * (vnb - vnref);
                    vb = vref + nya * (vnb - vnref);
                    wb = wref + nza * (vnb - vnref);
                    pb = sb * pow(rb, gama);
                } else {
                    if (vnin > 0.0) { rb = rin; ub = uin; vb = vin; wb = win; pb = pin; }
                    else { rb = o->roo; ub = o->uoo; vb = o->voo; wb = o->woo; pb = o->poo; }
                }
                SET5(b, IX(b, i, j, k), rb, ub, vb, wb, pb);
                if (SA_BC(o)) {
                    /* BC_farfield_turbulence_tgh, sub_tgh.f90:713-787: the
                     * sign of the contravariant velocity of the boundary state
                     * with the face point's metrics picks muoo (inflow) or the
                     * interior value, for the face point and the first ghost */
                    size_t f = IX(b, i, j, k);
                    const double *mx = metric_dir(b, rg->s_nd - 1, 0), *my = metric_dir(b, rg->s_nd - 1, 1),
                                 *mz = metric_dir(b, rg->s_nd - 1, 2);
                    double tem_lr = (double)L[rg->s_nd - 1];
                    double ut = tem_lr * (mx[f] * U(b)[f] + my[f] * V(b)[f] + mz[f] * W(b)[f]);
                    double qv = ut < 0.0 ? SA_MUOO_BC : b->qke[t];
                    b->qke[f] = qv;
                    b->qke[IX(b, i + L[0], j + L[1], k + L[2])] = ut < 0.0 ? SA_MUOO_BC : b->qke[t];
                }
                SET5(b, IX(b, i + L[0], j + L[1], k + L[2]), rb, ub, vb, wb, pb);
                SET5(b, IX(b, i + 2 * L[0], j + 2 * L[1], k + 2 * L[2]), rb, ub, vb, wb, pb);
                SET5(b, IX(b, i + 3 * L[0], j + 3 * L[1], k + 3 * L[2]), -rb, ub, vb, wb, pb);
            }
}

/* boundary_5 (supersonic inflow), BC.f90:609-665 */
static void bc_inflow(Orc *o, Blk *b, Reg *rg) {
    const int *L = rg->s_lr3d;
    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
                for (int n = 0; n <= 3; n++) {
                    SET5(b, IX(b, i + n * L[0], j + n * L[1], k + n * L[2]), o->roo, o->uoo, o->voo, o->woo, o->poo);
                    /* BC_farfield_turbulence, BC.f90:638: face and first ghost */
                    if (n <= 1 && SA_BC(o)) b->qke[IX(b, i + n * L[0], j + n * L[1], k + n * L[2])] = SA_MUOO_BC;
                }
}

/* boundary_6 (supersonic outflow), BC.f90:667-749 */
static void bc_outflow(const Orc *o, Blk *b, Reg *rg) {
    const int *L = rg->s_lr3d;
    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
        for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) {
                size_t t = IX(b, i - L[0], j - L[1], k - L[2]);
                double rm = R(b)[t], um = U(b)[t], vm = V(b)[t], wm = W(b)[t], pm = P(b)[t];
                for (int n = 0; n <= 3; n++) {
                    SET5(b, IX(b, i + n * L[0], j + n * L[1], k + n * L[2]), rm, um, vm, wm, pm);
                    /* BC_outflow_turbulence, BC.f90:721: face and first ghost */
                    if (n <= 1 && SA_BC(o)) b->qke[IX(b, i + n * L[0], j + n * L[1], k + n * L[2])] = b->qke[t];
                }
            }
}

/* viscid_wall (BC.f90:1244-1409) and inviscid_wall (BC.f90:1412-1486) */
static void bc_wall(Orc *o, Blk *b, Reg *rg) {
    const int *L = rg->s_lr3d;
    if (o->prm.nvis == 1) {
        double moocp = o->prm.moo * o->prm.moo * o->gama;
        for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
            for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                    size_t g1 = IX(b, i + L[0], j + L[1], k + L[2]);
                    size_t t1 = IX(b, i - L[0], j - L[1], k - L[2]);
                    size_t t2 = IX(b, i - 2 * L[0], j - 2 * L[1], k - 2 * L[2]);
                    size_t t3 = IX(b, i - 3 * L[0], j - 3 * L[1], k - 3 * L[2]);
                    SET5(b, g1, R(b)[t1], -U(b)[t1], -V(b)[t1], -W(b)[t1], P(b)[t1]);
                    if (SA_BC(o)) b->qke[g1] = -b->qke[t1]; /* BC_wall_turbulence, BC.f90:1280 */
                    double pres = (4.0 * P(b)[t1] - P(b)[t2]) / 3.0;
                    double tres, dres;
                    if (o->prm.twall > 0.0) {
                        if (pres < PMIN_LIMIT) pres = P(b)[t1];
                        tres = o->prm.twall / o->prm.tref;
                    } else {
                        tres = (4.0 * T(b)[t1] - T(b)[t2]) / 3.0;
                        if (pres < PMIN_LIMIT) pres = P(b)[t1];
                        if (tres < TMIN_LIMIT) tres = T(b)[t1];
                    }
                    dres = moocp * pres / tres;
                    SET5(b, IX(b, i, j, k), dres, 0.0, 0.0, 0.0, pres);
                    if (SA_BC(o)) sa_face_dif(b, IX(b, i, j, k), g1, t1); /* BC.f90:1301 */
                    size_t g2 = IX(b, i + 2 * L[0], j + 2 * L[1], k + 2 * L[2]);
                    size_t g3 = IX(b, i + 3 * L[0], j + 3 * L[1], k + 3 * L[2]);
                    SET5(b, g2, R(b)[t2], -U(b)[t2], -V(b)[t2], -W(b)[t2], P(b)[t2]);
                    SET5(b, g3, -R(b)[t3], -U(b)[t3], -V(b)[t3], -W(b)[t3], P(b)[t3]);
                }
    } else {
        for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
            for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                    double nx, ny, nz;
                    getnxyz(b, &nx, &ny, &nz, i, j, k, L[0], L[1], L[2]);
                    for (int l = 1; l <= 3; l++) {
                        size_t s = IX(b, i + l * L[0], j + l * L[1], k + l * L[2]);
                        size_t t = IX(b, i - l * L[0], j - l * L[1], k - l * L[2]);
                        double s1 = 2.0 * (U(b)[t] * nx + V(b)[t] * ny + W(b)[t] * nz);
                        double rr = l == 3 ? -R(b)[t] : R(b)[t];
                        SET5(b, s, rr, U(b)[t] - s1 * nx, V(b)[t] - s1 * ny, W(b)[t] - s1 * nz, P(b)[t]);
                    }
                }
        bc_dif_average(o, b, rg);
    }
}

int orc_boundary_all(void *h) {
    Orc *o = h;
    /* exchange_bc: start-of-step snapshot of every block (parallel.f90:1559-1674) */
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int f = 0; f < 5; f++) memcpy(o->snap[nb] + f * b->ng, b->fld[F_R + f], b->ng * 8);
        if (SA_BC(o)) {
            memcpy(b->sa_snap, b->qke, b->ng * 8);
            memcpy(b->sa_snap + b->ng, b->vist, b->ng * 8);
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int l = 0; l < b->nreg; l++) {
            Reg *rg = &b->reg[b->bcindex[l]];
            switch (rg->bctype) {
            case 2: bc_wall(o, b, rg); break;
            case 3: bc_symmetry(o, b, rg); break;
            case 4: bc_farfield(o, b, rg); break;
            case 5: bc_inflow(o, b, rg); break;
            case 6: bc_outflow(o, b, rg); break;
            default: bc_vir3(o, nb, rg); break;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* initial_q_dq_c_t, sub_tgh.f90:1-32                                   */
/* ------------------------------------------------------------------ */
static void get_c_t_only(Orc *o, Blk *b, int with_t) {
    /* RHS.f90:307-409 (with_t) and RHS.f90:171-237 */
    double gama = o->gama, moo2 = o->prm.moo * o->prm.moo;
    int ni = b->ni, nj = b->nj, nk = b->nk;
    double *c = b->fld[F_C], *t = T(b), *r = R(b), *p = P(b);
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                size_t id = IX(b, i, j, k);
                double a2 = gama * p[id] / r[id];
                c[id] = sqrt(a2);
                if (with_t) t[id] = moo2 * a2;
            }
    if (!with_t) {
        for (int k = 1; k <= nk; k++)
            for (int j = 1; j <= nj; j++)
                for (int s = 0; s < 2; s++) { size_t id = IX(b, s ? ni + 1 : 0, j, k); c[id] = sqrt(gama * p[id] / r[id]); }
        for (int k = 1; k <= nk; k++)
            for (int i = 1; i <= ni; i++)
                for (int s = 0; s < 2; s++) { size_t id = IX(b, i, s ? nj + 1 : 0, k); c[id] = sqrt(gama * p[id] / r[id]); }
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++)
                for (int s = 0; s < 2; s++) { size_t id = IX(b, i, j, s ? nk + 1 : 0); c[id] = sqrt(gama * p[id] / r[id]); }
        return;
    }
    /* i faces: the third layer reuses a2 of the second layer (RHS.f90:351-353) */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int s = 0; s < 2; s++) {
                int n1 = s ? ni + 1 : 0, n2 = s ? ni + 2 : -1, n3 = s ? ni + 3 : -2;
                size_t i1 = IX(b, n1, j, k), i2 = IX(b, n2, j, k), i3 = IX(b, n3, j, k);
                double a2 = gama * p[i1] / r[i1];
                c[i1] = sqrt(a2);
                t[i1] = moo2 * a2;
                a2 = gama * p[i2] / r[i2];
                t[i2] = moo2 * a2;
                t[i3] = moo2 * a2;
            }
    for (int k = 1; k <= nk; k++)
        for (int i = 1; i <= ni; i++)
            for (int s = 0; s < 2; s++) {
                int n1 = s ? nj + 1 : 0, n2 = s ? nj + 2 : -1, n3 = s ? nj + 3 : -2;
                size_t i1 = IX(b, i, n1, k), i2 = IX(b, i, n2, k), i3 = IX(b, i, n3, k);
                double a2 = gama * p[i1] / r[i1];
                c[i1] = sqrt(a2);
                t[i1] = moo2 * a2;
                a2 = gama * p[i2] / r[i2];
                t[i2] = moo2 * a2;
                a2 = gama * p[i3] / fabs(r[i3]);
                t[i3] = moo2 * a2;
            }
    for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++)
            for (int s = 0; s < 2; s++) {
                int n1 = s ? nk + 1 : 0, n2 = s ? nk + 2 : -1, n3 = s ? nk + 3 : -2;
                size_t i1 = IX(b, i, j, n1), i2 = IX(b, i, j, n2), i3 = IX(b, i, j, n3);
                double a2 = gama * p[i1] / r[i1];
                c[i1] = sqrt(a2);
                t[i1] = moo2 * a2;
                a2 = gama * p[i2] / r[i2];
                t[i2] = moo2 * a2;
                a2 = gama * p[i3] / fabs(r[i3]);
                t[i3] = moo2 * a2;
            }
}

int orc_initial_q_dq_c_t(void *h) {
    Orc *o = h;
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        double gama = o->gama;
        if (o->prm.nvis == 1) {
            get_c_t_only(o, b, 1);
            /* compute_visl_ns GasModel.f90:219-235 */
            for (int k = 1; k <= b->nk; k++)
                for (int j = 1; j <= b->nj; j++)
                    for (int i = 1; i <= b->ni; i++) {
                        size_t id = IX(b, i, j, k);
                        double tm = T(b)[id];
                        b->fld[F_VISL][id] = tm * sqrt(tm) * (1.0 + o->visc) / (tm + o->visc);
                    }
        } else {
            get_c_t_only(o, b, 0);
        }
        /* get_q_only RHS.f90:75-166 (interior; prim_to_q Sub1.f90:106-131) */
        for (int k = 1; k <= b->nk; k++)
            for (int j = 1; j <= b->nj; j++)
                for (int i = 1; i <= b->ni; i++) {
                    size_t id = IX(b, i, j, k);
                    double rm = R(b)[id], um = U(b)[id], vm = V(b)[id], wm = W(b)[id], pm = P(b)[id];
                    double em = pm / (gama - 1.0) + 0.5 * rm * (um * um + vm * vm + wm * wm);
                    b->fld[F_Q1][id] = rm;
                    b->fld[F_Q2][id] = rm * um;
                    b->fld[F_Q3][id] = rm * vm;
                    b->fld[F_Q4][id] = rm * wm;
                    b->fld[F_Q5][id] = em;
                }
        /* set_dq_to_0 PreProcess.f90:1189-1205 */
        for (int m = 0; m < 5; m++) memset(DQ(b, m), 0, b->ng * 8);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* timestep_tgh (sub_tgh.f90:1270-1348): spectinv (Convect.f90:1338-1461),
 * spectvisl (LHS.f90:243-343), localdt0 (LHS.f90:1343-1377)            */
/* ------------------------------------------------------------------ */
static void spect_point(Orc *o, Blk *b, int i, int j, int k, int ii, int jj, int kk) {
    size_t id = IX(b, i, j, k), ic = IX(b, ii, jj, kk);
    double um = U(b)[id], vm = V(b)[id], wm = W(b)[id], cm = b->fld[F_C][id];
    double kx = b->fld[F_KCX][ic], ky = b->fld[F_KCY][ic], kz = b->fld[F_KCZ][ic], kt = 0.0;
    double ex = b->fld[F_ETX][ic], ey = b->fld[F_ETY][ic], ez = b->fld[F_ETZ][ic], et = 0.0;
    double cx = b->fld[F_CTX][ic], cy = b->fld[F_CTY][ic], cz = b->fld[F_CTZ][ic], ct = 0.0;
    double cita = kx * um + ky * vm + kz * wm + kt;
    double citb = ex * um + ey * vm + ez * wm + et;
    double citc = cx * um + cy * vm + cz * wm + ct;
    double cgma = sqrt(kx * kx + ky * ky + kz * kz);
    double cgmb = sqrt(ex * ex + ey * ey + ez * ez);
    double cgmc = sqrt(cx * cx + cy * cy + cz * cz);
    b->fld[F_SRA][id] = fabs(cita) + cm * cgma;
    b->fld[F_SRB][id] = fabs(citb) + cm * cgmb;
    b->fld[F_SRC][id] = fabs(citc) + cm * cgmc;
    if (o->prm.nvis == 1) {
        if (o->prm.csrv > 0.0) {
            double rm_vol = R(b)[id] * b->fld[F_VOL][ic];
            double ri = kx * kx + ky * ky + kz * kz;
            double rj = ex * ex + ey * ey + ez * ez;
            double rk = cx * cx + cy * cy + cz * cz;
            double vis = b->fld[F_VISL][ic];
            if (o->sa) vis = vis + b->vist[ic]; /* spectvist, LHS.f90:141-241 */
            double coef = 2.0 * vis / (o->reynolds * rm_vol + SMALL);
            double coef1 = o->prm.csrv * coef;
            b->fld[F_SRVA][id] = coef1 * ri;
            b->fld[F_SRVB][id] = coef1 * rj;
            b->fld[F_SRVC][id] = coef1 * rk;
        }
    } else {
        b->fld[F_SRVA][id] = 0.0;
        b->fld[F_SRVB][id] = 0.0;
        b->fld[F_SRVC][id] = 0.0;
    }
}

int orc_timestep(void *h) {
    Orc *o = h;
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        int ni = b->ni, nj = b->nj, nk = b->nk;
        for (int k = 1; k <= nk; k++)
            for (int j = 1; j <= nj; j++)
                for (int i = 1; i <= ni; i++) spect_point(o, b, i, j, k, i, j, k);
        for (int k = 1; k <= nk; k++)
            for (int j = 1; j <= nj; j++)
                for (int s = 0; s < 2; s++) { int i = s ? ni + 1 : 0; spect_point(o, b, i, j, k, i < 1 ? 1 : (i > ni ? ni : i), j, k); }
        for (int k = 1; k <= nk; k++)
            for (int i = 1; i <= ni; i++)
                for (int s = 0; s < 2; s++) { int j = s ? nj + 1 : 0; spect_point(o, b, i, j, k, i, j < 1 ? 1 : (j > nj ? nj : j), k); }
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++)
                for (int s = 0; s < 2; s++) { int k = s ? nk + 1 : 0; spect_point(o, b, i, j, k, i, j, k < 1 ? 1 : (k > nk ? nk : k)); }
        for (int k = 1; k <= nk; k++)
            for (int j = 1; j <= nj; j++)
                for (int i = 1; i <= ni; i++) {
                    size_t id = IX(b, i, j, k);
                    double ra = b->fld[F_SRA][id], rb = b->fld[F_SRB][id], rc = b->fld[F_SRC][id];
                    double rv = b->fld[F_SRVA][id] + b->fld[F_SRVB][id] + b->fld[F_SRVC][id];
                    double rabc = ra + rb + rc + rv;
                    double dt;
                    if (o->prm.timedt_rate > SMALL) {
                        double a = o->prm.cfl / rabc, c = o->prm.timedt_rate / b->fld[F_VOL][id];
                        dt = a < c ? a : c;
                    } else dt = o->prm.cfl / rabc;
                    b->fld[F_DTDT][id] = dt;
                }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Inviscid RHS: r_h_s_invis (RHS.f90:35-72) -> invcode -> inviscd3d    */
/* (Convect.f90:2-56, 58-649)                                           */
/* ------------------------------------------------------------------ */
static int rhs_invis_block(Orc *o, Blk *b) {
    int dims[3] = {b->ni, b->nj, b->nk};
    int nbad = 0;
    for (int dir = 0; dir < 3; dir++) {
        int n = dims[dir];
        if (n <= NIJK2D) continue;
        int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2; /* the two other directions */
        int na = dims[a1], nb2 = dims[a2];
        const double *mx = metric_dir(b, dir, 0), *my = metric_dir(b, dir, 1), *mz = metric_dir(b, dir, 2);
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : nbad)
        for (int bb = 1; bb <= nb2; bb++)
            for (int aa = 1; aa <= na; aa++) {
                int L = n + 6;
                double *q = malloc(sizeof(double) * 5 * L);
                double *tr = malloc(sizeof(double) * 4 * (n + 1));
                double *nx = malloc(sizeof(double) * 4 * (n + 1));
                double *df = malloc(sizeof(double) * 5 * n);
                int c[3];
                c[a1] = aa;
                c[a2] = bb;
                for (int l = -2; l <= n + 3; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    q[0 * L + l + 2] = R(b)[id];
                    q[1 * L + l + 2] = U(b)[id];
                    q[2 * L + l + 2] = V(b)[id];
                    q[3 * L + l + 2] = W(b)[id];
                    q[4 * L + l + 2] = P(b)[id];
                }
                for (int l = 1; l <= n; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    tr[0 + 4 * (l - 1)] = mx[id];
                    tr[1 + 4 * (l - 1)] = my[id];
                    tr[2 + 4 * (l - 1)] = mz[id];
                    tr[3 + 4 * (l - 1)] = 0.0;
                }
                value_half_node(4, n, tr, nx);
                nbad += wcns_line(o, n, q, nx, df);
                for (int l = 1; l <= n; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    for (int m = 0; m < 5; m++) DQ(b, m)[id] = DQ(b, m)[id] + df[m + 5 * (l - 1)];
                }
                free(q); free(tr); free(nx); free(df);
            }
    }
    return nbad;
}

int orc_rhs_invis(void *h) {
    Orc *o = h;
    int nbad = 0;
    for (int nb = 1; nb <= o->nb; nb++) nbad += rhs_invis_block(o, &o->b[nb]);
    if (nbad) { set_err("flux_Roe: c^2 <= 0"); return 2; }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Viscous RHS: WCNSE5_VIS_virtual (sub_tgh.f90:1511-1810)             */
/* ------------------------------------------------------------------ */

/* DUVWT_NODE_LINE_virtual, sub_tgh.f90:2217-2272; u[m + 4*(i+2)] */
static void duvwt_node_line(int ni, const double *u, double *du, int fl, int fr) {
#define UU(m, i) u[(m) + 4 * ((i) + 2)]
#define DU(m, i) du[(m) + 4 * ((i) - 1)]
    if (ni <= NIJK2ND) {
        for (int i = 1; i <= ni; i++)
            for (int m = 0; m < 4; m++) DU(m, i) = 0.5 * (UU(m, i + 1) - UU(m, i - 1));
        return;
    }
    int st = 1, ed = ni;
    if (fl) {
        st = 3;
        for (int m = 0; m < 4; m++) {
            DU(m, 1) = (-11. * UU(m, 1) + 18. * UU(m, 2) - 9. * UU(m, 3) + 2. * UU(m, 4)) / 6.0;
            DU(m, 2) = (-3.0 * UU(m, 1) + -10.0 * UU(m, 2) + 18.0 * UU(m, 3) + -6.0 * UU(m, 4) + 1.0 * UU(m, 5)) / 12.0;
        }
    }
    if (fr) {
        ed = ni - 2;
        for (int m = 0; m < 4; m++) {
            DU(m, ni) = -(-11. * UU(m, ni) + 18. * UU(m, ni - 1) - 9.0 * UU(m, ni - 2) + 2. * UU(m, ni - 3)) / 6.0;
            DU(m, ni - 1) = -(-3.0 * UU(m, ni) + -10.0 * UU(m, ni - 1) + 18.0 * UU(m, ni - 2) + -6.0 * UU(m, ni - 3) +
                              1.0 * UU(m, ni - 4)) / 12.0;
        }
    }
    for (int i = st; i <= ed; i++)
        for (int m = 0; m < 4; m++)
            DU(m, i) = (8.0 * (UU(m, i + 1) - UU(m, i - 1)) + -1.0 * (UU(m, i + 2) - UU(m, i - 2))) / 12.0;
#undef DU
}

/* DUVWT_half_line_virtual, sub_tgh.f90:2277-2330; dh[m + 4*i], i=0..ni */
static void duvwt_half_line(int ni, const double *u, double *dh, int fl, int fr) {
#define DH(m, i) dh[(m) + 4 * (i)]
    if (ni <= NIJK2ND) {
        for (int m = 0; m < 4; m++)
            for (int i = 0; i <= ni; i++) DH(m, i) = UU(m, i + 1) - UU(m, i);
        return;
    }
    int st = 0, ed = ni;
    if (fl) {
        st = 2;
        for (int m = 0; m < 4; m++) {
            DH(m, 0) = (-71.0 * UU(m, 1) + 141.0 * UU(m, 2) + -93.0 * UU(m, 3) + 23.0 * UU(m, 4)) / 24.0;
            DH(m, 1) = (-22.0 * UU(m, 1) + 17.0 * UU(m, 2) + 9.0 * UU(m, 3) + -5.0 * UU(m, 4) + 1.0 * UU(m, 5)) / 24.0;
        }
    }
    if (fr) {
        ed = ni - 2;
        for (int m = 0; m < 4; m++) {
            DH(m, ni) = -(-71.0 * UU(m, ni) + 141.0 * UU(m, ni - 1) + -93.0 * UU(m, ni - 2) + 23.0 * UU(m, ni - 3)) / 24.0;
            DH(m, ni - 1) = -(-22.0 * UU(m, ni) + 17.0 * UU(m, ni - 1) + 9.0 * UU(m, ni - 2) + -5.0 * UU(m, ni - 3) +
                              1.0 * UU(m, ni - 4)) / 24.0;
        }
    }
    for (int i = st; i <= ed; i++)
        for (int m = 0; m < 4; m++)
            DH(m, i) = (27.0 * (UU(m, i + 1) - UU(m, i)) + -1.0 * (UU(m, i + 2) - UU(m, i - 1))) / 24.0;
#undef DH
}

/* VALUE_line_half_virtual, sub_tgh.f90:2335-2387 */
static void value_line_half(int ni, const double *u, double *qh, int fl, int fr) {
#define QH(m, i) qh[(m) + 4 * (i)]
    if (ni <= NIJK2ND) {
        for (int i = 0; i <= ni; i++)
            for (int m = 0; m < 4; m++) QH(m, i) = 0.5 * (UU(m, i) + UU(m, i + 1));
        return;
    }
    int st = 0, ed = ni;
    if (fl) {
        st = 2;
        for (int m = 0; m < 4; m++) {
            QH(m, 0) = (35.0 * UU(m, 1) + -35.0 * UU(m, 2) + 21.0 * UU(m, 3) + -5.0 * UU(m, 4)) / 16.0;
            QH(m, 1) = (5.0 * UU(m, 1) + 15.0 * UU(m, 2) + -5.0 * UU(m, 3) + 1.0 * UU(m, 4)) / 16.0;
        }
    }
    if (fr) {
        ed = ni - 2;
        for (int m = 0; m < 4; m++) {
            QH(m, ni) = (35.0 * UU(m, ni) + -35.0 * UU(m, ni - 1) + 21.0 * UU(m, ni - 2) + -5.0 * UU(m, ni - 3)) / 16.0;
            QH(m, ni - 1) = (5.0 * UU(m, ni) + 15.0 * UU(m, ni - 1) + -5.0 * UU(m, ni - 2) + 1.0 * UU(m, ni - 3)) / 16.0;
        }
    }
    for (int i = st; i <= ed; i++)
        for (int m = 0; m < 4; m++) QH(m, i) = (9.0 * (UU(m, i) + UU(m, i + 1)) + -1.0 * (UU(m, i + 2) + UU(m, i - 1))) / 16.0;
#undef QH
#undef UU
}

/* VALUE_HALF_NODE_IJK (newvis.f90:421-554) for the 4-component group
 * starting at m0 of a 12-component line: dl[m + 12*(i-1)] -> dh[m + 12*i] */
static void value_half_node_group(int ni, const double *dl, double *dh, int m0) {
#define QL(m, i) dl[(m) + 12 * ((i) - 1)]
#define QH(m, i) dh[(m) + 12 * (i)]
    if (ni <= NIJK2ND) {
        for (int i = 1; i <= ni - 1; i++)
            for (int m = m0; m < m0 + 4; m++) QH(m, i) = 0.5 * (QL(m, i) + QL(m, i + 1));
        for (int m = m0; m < m0 + 4; m++) {
            int i2 = ni < 2 ? ni : 2, j1 = ni - 1 > 1 ? ni - 1 : 1;
            QH(m, 0) = 1.5 * QL(m, 1) - 0.5 * QL(m, i2);
            QH(m, ni) = 1.5 * QL(m, ni) - 0.5 * QL(m, j1);
        }
        return;
    }
    for (int i = 2; i <= ni - 2; i++)
        for (int m = m0; m < m0 + 4; m++) QH(m, i) = (9.0 * (QL(m, i) + QL(m, i + 1)) + -1.0 * (QL(m, i + 2) + QL(m, i - 1))) / 16.0;
    for (int m = m0; m < m0 + 4; m++) {
        QH(m, 1) = (5.0 * QL(m, 1) + 15.0 * QL(m, 2) + -5.0 * QL(m, 3) + 1.0 * QL(m, 4)) / 16.0;
        QH(m, ni - 1) = (5.0 * QL(m, ni) + 15.0 * QL(m, ni - 1) + -5.0 * QL(m, ni - 2) + 1.0 * QL(m, ni - 3)) / 16.0;
        QH(m, 0) = (35.0 * QL(m, 1) - 35.0 * QL(m, 2) + 21.0 * QL(m, 3) - 5.0 * QL(m, 4)) / 16.0;
        QH(m, ni) = (35.0 * QL(m, ni) - 35.0 * QL(m, ni - 1) + 21.0 * QL(m, ni - 2) - 5.0 * QL(m, ni - 3)) / 16.0;
    }
#undef QL
#undef QH
}

/* UVWT_DER_4th_virtual (sub_tgh.f90:1909-2029): node derivatives of
 * (u,v,w,T) along each index direction -> duv[(m + 4*dir) + 12*pid] */
static void node_derivatives(Blk *b, double *duv) {
    int dims[3] = {b->ni, b->nj, b->nk};
    for (int dir = 0; dir < 3; dir++) {
        int n = dims[dir];
        int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
#pragma omp parallel for collapse(2) schedule(static)
        for (int bb = 1; bb <= dims[a2]; bb++)
            for (int aa = 1; aa <= dims[a1]; aa++) {
                double *u = malloc(sizeof(double) * 4 * (n + 6));
                double *du = malloc(sizeof(double) * 4 * n);
                int c[3];
                c[a1] = aa;
                c[a2] = bb;
                c[dir] = -2;
                int rl = R(b)[IX(b, c[0], c[1], c[2])] < 0.0;
                c[dir] = n + 3;
                int rr = R(b)[IX(b, c[0], c[1], c[2])] < 0.0;
                for (int l = -2; l <= n + 3; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    u[0 + 4 * (l + 2)] = U(b)[id];
                    u[1 + 4 * (l + 2)] = V(b)[id];
                    u[2 + 4 * (l + 2)] = W(b)[id];
                    u[3 + 4 * (l + 2)] = T(b)[id];
                }
                /* uvwt(4,-2)/uvwt(4,n+3) carry the boundary flag (-1 when the
                 * third ghost density is negative) */
                if (rl) u[3] = -1.0;
                if (rr) u[3 + 4 * (n + 5)] = -1.0;
                int fl = u[3] < 0.0, fr = u[3 + 4 * (n + 5)] < 0.0;
                duvwt_node_line(n, u, du, fl, fr);
                for (int l = 1; l <= n; l++) {
                    c[dir] = l;
                    size_t pid = (size_t)(c[0] - 1) + (size_t)b->ni * ((size_t)(c[1] - 1) + (size_t)b->nj * (size_t)(c[2] - 1));
                    for (int m = 0; m < 4; m++) duv[(m + 4 * dir) + 12 * pid] = du[m + 4 * (l - 1)];
                }
                free(u); free(du);
            }
    }
}

static void rhs_vis_block(Orc *o, Blk *b) {
    int dims[3] = {b->ni, b->nj, b->nk};
    size_t np = (size_t)b->ni * b->nj * b->nk;
    double *duv = malloc(sizeof(double) * 12 * np);
    node_derivatives(b, duv);
    double re = 1.0 / o->reynolds;
    double cp = 1.0 / ((o->gama - 1.0) * o->prm.moo * o->prm.moo);
    double cp_prl = cp / o->prl, cp_prt = cp / o->prt;
    const double CC = 2.0 / 3.0;
    for (int dir = 0; dir < 3; dir++) {
        int n = dims[dir];
        int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
#pragma omp parallel for collapse(2) schedule(static)
        for (int bb = 1; bb <= dims[a2]; bb++)
            for (int aa = 1; aa <= dims[a1]; aa++) {
                double *u = malloc(sizeof(double) * 4 * (n + 6));
                double *uh = malloc(sizeof(double) * 4 * (n + 1));
                double *dl = malloc(sizeof(double) * 12 * n), *dh = malloc(sizeof(double) * 12 * (n + 1));
                double *kl = malloc(sizeof(double) * 9 * n), *kh = malloc(sizeof(double) * 9 * (n + 1));
                double *s3 = malloc(sizeof(double) * 3 * n), *s3h = malloc(sizeof(double) * 3 * (n + 1));
                double *vol = malloc(sizeof(double) * n), *volh = malloc(sizeof(double) * (n + 1));
                double *v1 = malloc(sizeof(double) * n), *v1h = malloc(sizeof(double) * (n + 1));
                double *v2 = malloc(sizeof(double) * n), *v2h = malloc(sizeof(double) * (n + 1));
                double *dmid = malloc(sizeof(double) * 4 * (n + 1));
                double *dx = malloc(sizeof(double) * 12 * (n + 1));
                double *fv = malloc(sizeof(double) * 5 * (n + 1)), *dfv = malloc(sizeof(double) * 5 * n);
                int c[3];
                c[a1] = aa;
                c[a2] = bb;
                for (int l = 1; l <= n; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    size_t pid = (size_t)(c[0] - 1) + (size_t)b->ni * ((size_t)(c[1] - 1) + (size_t)b->nj * (size_t)(c[2] - 1));
                    double vl = b->fld[F_VISL][id];
                    v1[l - 1] = vl;
                    v2[l - 1] = vl * cp_prl;
                    v1[l - 1] = v1[l - 1] + b->vist[id];
                    v2[l - 1] = v2[l - 1] + b->vist[id] * cp_prt;
                    double *k9 = &kl[9 * (l - 1)];
                    k9[0] = b->fld[F_KCX][id]; k9[1] = b->fld[F_ETX][id]; k9[2] = b->fld[F_CTX][id];
                    k9[3] = b->fld[F_KCY][id]; k9[4] = b->fld[F_ETY][id]; k9[5] = b->fld[F_CTY][id];
                    k9[6] = b->fld[F_KCZ][id]; k9[7] = b->fld[F_ETZ][id]; k9[8] = b->fld[F_CTZ][id];
                    vol[l - 1] = b->fld[F_VOL][id];
                    for (int m = 0; m < 12; m++) dl[m + 12 * (l - 1)] = duv[m + 12 * pid];
                }
                for (int l = -2; l <= n + 3; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    u[0 + 4 * (l + 2)] = U(b)[id];
                    u[1 + 4 * (l + 2)] = V(b)[id];
                    u[2 + 4 * (l + 2)] = W(b)[id];
                    u[3 + 4 * (l + 2)] = T(b)[id];
                }
                c[dir] = -2;
                int rl = R(b)[IX(b, c[0], c[1], c[2])] < 0.0;
                c[dir] = n + 3;
                int rr = R(b)[IX(b, c[0], c[1], c[2])] < 0.0;
                if (rl) u[3 + 4 * 0] = -1.0;
                if (rr) u[3 + 4 * (n + 5)] = -1.0;
                int fl = u[3] < 0.0, fr = u[3 + 4 * (n + 5)] < 0.0;
                value_line_half(n, u, uh, fl, fr);
                for (int g = 0; g < 3; g++)
                    if (g != dir) value_half_node_group(n, dl, dh, 4 * g);
                value_half_node(9, n, kl, kh);
                value_half_node(1, n, vol, volh);
                value_half_node(1, n, v1, v1h);
                value_half_node(1, n, v2, v2h);
                /* UVWT_DER_4th_half_virtual (sub_tgh.f90:2032-2155) */
                duvwt_half_line(n, u, dmid, fl, fr);
                for (int l = 0; l <= n; l++)
                    for (int m = 0; m < 4; m++) dh[4 * dir + m + 12 * l] = dmid[m + 4 * l];
                /* DUVWT_DXYZ, WCNSE5.f90:854-890 */
                for (int l = 0; l <= n; l++) {
                    const double *dd = &dh[12 * l], *kk = &kh[9 * l];
                    double vv = volh[l];
                    for (int m = 1; m <= 3; m++) {
                        int m1 = m + m + m - 2, m2 = m1 + 1, m3 = m2 + 1;
                        dx[(m - 1) + 12 * l] = (kk[m1 - 1] * dd[0] + kk[m2 - 1] * dd[4] + kk[m3 - 1] * dd[8]) / vv;
                        dx[(m + 2) + 12 * l] = (kk[m1 - 1] * dd[1] + kk[m2 - 1] * dd[5] + kk[m3 - 1] * dd[9]) / vv;
                        dx[(m + 5) + 12 * l] = (kk[m1 - 1] * dd[2] + kk[m2 - 1] * dd[6] + kk[m3 - 1] * dd[10]) / vv;
                        dx[(m + 8) + 12 * l] = (kk[m1 - 1] * dd[3] + kk[m2 - 1] * dd[7] + kk[m3 - 1] * dd[11]) / vv;
                    }
                }
                /* FLUX_VIS_LINE_new, newvis.f90:283-349 */
                for (int l = 0; l <= n; l++) {
                    const double *d = &dx[12 * l];
                    double vs = v1h[l];
                    double vscc = vs * CC;
                    double dudx = d[0], dudy = d[1], dudz = d[2];
                    double dvdx = d[3], dvdy = d[4], dvdz = d[5];
                    double dwdx = d[6], dwdy = d[7], dwdz = d[8];
                    double t1 = vscc * (2.0 * dudx - dvdy - dwdz);
                    double t5 = vscc * (2.0 * dvdy - dwdz - dudx);
                    double t9 = vscc * (2.0 * dwdz - dudx - dvdy);
                    double t2 = vs * (dudy + dvdx);
                    double t3 = vs * (dudz + dwdx);
                    double t6 = vs * (dvdz + dwdy);
                    double t4 = t2, t7 = t3, t8 = t6;
                    double kcp = v2h[l];
                    double nx = kh[9 * l + dir], ny = kh[9 * l + dir + 3], nz = kh[9 * l + dir + 6];
                    double *ff = &fv[5 * l];
                    ff[0] = 0.0;
                    ff[1] = t1 * nx + t2 * ny + t3 * nz;
                    ff[2] = t4 * nx + t5 * ny + t6 * nz;
                    ff[3] = t7 * nx + t8 * ny + t9 * nz;
                    ff[4] = uh[0 + 4 * l] * ff[1] + uh[1 + 4 * l] * ff[2] + uh[2 + 4 * l] * ff[3] +
                            kcp * (d[9] * nx + d[10] * ny + d[11] * nz);
                }
                flux_dxyz(5, n, fv, dfv);
                for (int l = 1; l <= n; l++) {
                    c[dir] = l;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    for (int m = 0; m < 5; m++) DQ(b, m)[id] = DQ(b, m)[id] - re * dfv[m + 5 * (l - 1)];
                }
                free(u); free(uh); free(dl); free(dh); free(kl); free(kh); free(s3); free(s3h);
                free(vol); free(volh); free(v1); free(v1h); free(v2); free(v2h); free(dmid); free(dx); free(fv); free(dfv);
            }
    }
    free(duv);
}

static void sa_block(const Orc *o, Blk *b);
int orc_rhs_vis(void *h) {
    Orc *o = h;
    if (o->prm.nvis != 1) return 0;
    /* turbulence(nb) at the start of r_h_s_vis (RHS.f90:22); a block's model
     * step reads only that block, so all blocks can go first */
    if (o->sa) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int nb = 1; nb <= o->nb; nb++) sa_block(o, &o->b[nb]);
    }
    for (int nb = 1; nb <= o->nb; nb++) rhs_vis_block(o, &o->b[nb]);
    return 0;
}

/* the viscous residual without the model step (a sharded run advances the
 * model first and refreshes its proxies' qke and vist in between) */
int orc_rhs_vis_flux(void *h) {
    Orc *o = h;
    if (o->prm.nvis != 1) return 0;
    for (int nb = 1; nb <= o->nb; nb++) rhs_vis_block(o, &o->b[nb]);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Interface averaging: communicate_dq_npp (parallel.f90:3020-3164) and */
/* communicate_pv_npp (parallel.f90:3166-3326), one block per rank      */
/* ------------------------------------------------------------------ */
int orc_communicate_dq(void *h) {
    Orc *o = h;
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int m = 0; m < 5; m++) memcpy(o->snap[nb] + m * b->ng, DQ(b, m), b->ng * 8);
    }
    /* boundary_match_dq_2pm */
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int nr = 0; nr < b->nreg; nr++) {
            Reg *rg = &b->reg[nr];
            if (rg->bctype >= 0) continue;
            Blk *bt = &o->b[rg->nbt];
            int same = rg->nbt == nb;
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                        int bi = reg_box_index(rg, i, j, k);
                        size_t s = IX(b, i, j, k), t = IX(bt, rg->image[bi], rg->jmage[bi], rg->kmage[bi]);
                        if (same) {
                            double vol_p = b->fld[F_VOL][s] / bt->fld[F_VOL][t];
                            for (int m = 0; m < 5; m++) DQ(b, m)[s] = 0.5 * (DQ(bt, m)[t] * vol_p + DQ(b, m)[s]);
                        } else {
                            double vol_p = b->fld[F_VOL][s];
                            for (int m = 0; m < 5; m++) {
                                double pk = o->snap[rg->nbt][m * bt->ng + t] / bt->fld[F_VOL][t];
                                DQ(b, m)[s] = 0.5 * (pk * vol_p + DQ(b, m)[s]);
                            }
                        }
                    }
        }
    }
    /* boundary_match_dq_3pp */
    for (int c = 0; c < o->ncomp; c++) {
        double dqq[5] = {0, 0, 0, 0, 0};
        int f0 = o->comp_first[c], np = o->comp_n[c];
        for (int q = 0; q < np; q++) {
            Blk *b = &o->b[o->mem_nb[f0 + q]];
            size_t id = IX(b, o->mem_i[f0 + q], o->mem_j[f0 + q], o->mem_k[f0 + q]);
            for (int m = 0; m < 5; m++) dqq[m] = dqq[m] + o->snap[o->mem_nb[f0 + q]][m * b->ng + id] / b->fld[F_VOL][id];
        }
        for (int m = 0; m < 5; m++) dqq[m] = dqq[m] / (np * 1.0);
        for (int q = 0; q < np; q++) {
            Blk *b = &o->b[o->mem_nb[f0 + q]];
            size_t id = IX(b, o->mem_i[f0 + q], o->mem_j[f0 + q], o->mem_k[f0 + q]);
            for (int m = 0; m < 5; m++) DQ(b, m)[id] = dqq[m] * b->fld[F_VOL][id];
        }
    }
    return 0;
}

int orc_communicate_pv(void *h) {
    Orc *o = h;
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int f = 0; f < 6; f++) memcpy(o->snap[nb] + f * b->ng, b->fld[F_R + f], b->ng * 8);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int nr = 0; nr < b->nreg; nr++) {
            Reg *rg = &b->reg[nr];
            if (rg->bctype >= 0) continue;
            Blk *bt = &o->b[rg->nbt];
            int same = rg->nbt == nb;
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                        int bi = reg_box_index(rg, i, j, k);
                        size_t s = IX(b, i, j, k), t = IX(bt, rg->image[bi], rg->jmage[bi], rg->kmage[bi]);
                        for (int f = 0; f < 6; f++) {
                            double tv = same ? bt->fld[F_R + f][t] : o->snap[rg->nbt][f * bt->ng + t];
                            b->fld[F_R + f][s] = 0.5 * (tv + b->fld[F_R + f][s]);
                        }
                    }
        }
    }
    for (int c = 0; c < o->ncomp; c++) {
        double dqq[6] = {0, 0, 0, 0, 0, 0};
        int f0 = o->comp_first[c], np = o->comp_n[c];
        for (int q = 0; q < np; q++) {
            Blk *b = &o->b[o->mem_nb[f0 + q]];
            size_t id = IX(b, o->mem_i[f0 + q], o->mem_j[f0 + q], o->mem_k[f0 + q]);
            for (int f = 0; f < 6; f++) dqq[f] = dqq[f] + o->snap[o->mem_nb[f0 + q]][f * b->ng + id] / 1.0;
        }
        for (int f = 0; f < 6; f++) dqq[f] = dqq[f] / (np * 1.0);
        for (int q = 0; q < np; q++) {
            Blk *b = &o->b[o->mem_nb[f0 + q]];
            size_t id = IX(b, o->mem_i[f0 + q], o->mem_j[f0 + q], o->mem_k[f0 + q]);
            for (int f = 0; f < 6; f++) b->fld[F_R + f][id] = dqq[f] * 1.0;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* LHS: l_h_s_tgh (LHS.f90:1-34) -> GS_PR_Single (LHS.f90:1559-1587)    */
/* ------------------------------------------------------------------ */
static void zero_physical_faces(Blk *b) {
    /* set_nonconnect_boundary_dq_0, CIC.f90:2-17, 482-506 */
    for (int nr = 0; nr < b->nreg; nr++) {
        Reg *rg = &b->reg[nr];
        if (rg->bctype <= 0) continue;
        for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
            for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) {
                    size_t id = IX(b, i, j, k);
                    for (int m = 0; m < 5; m++) DQ(b, m)[id] = 0.0;
                }
    }
}

/* mxdq_std, LHS.f90:756-828 (gettmhmgm_ns GasModel.f90:411-426) */
static void mxdq_std(const Orc *o, const double *prim, const double *g4, const double *dq, double *f, double rad, int npn) {
    double gama = o->gama;
    double rm = prim[0], um = prim[1], vm = prim[2], wm = prim[3], pm = prim[4];
    double hint = gama / (gama - 1.0) * pm / rm;
    double c2 = gama * pm / rm;
    double cm = sqrt(c2);
    double v2 = um * um + vm * vm + wm * wm;
    double hm = hint + 0.5 * v2;
    double nx = g4[0], ny = g4[1], nz = g4[2], nt = g4[3];
    double ct = nx * um + ny * vm + nz * wm + nt;
    double cgm = sqrt(nx * nx + ny * ny + nz * nz);
    if (!(cgm >= SML_SSS)) cgm = SML_SSS;
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

static void getprim(const Blk *b, int i, int j, int k, double *p) {
    size_t id = IX(b, i, j, k);
    p[0] = R(b)[id]; p[1] = U(b)[id]; p[2] = V(b)[id]; p[3] = W(b)[id]; p[4] = P(b)[id];
}

static double coed_of(const Orc *o, const Blk *b, size_t id) {
    /* getcoed, LHS.f90:602-645 with wmig=beta=1, ndualtst=0 */
    double rad_ns = b->fld[F_SRA][id] + b->fld[F_SRB][id] + b->fld[F_SRC][id];
    for (int m = 1; m <= o->prm.nvis; m++) rad_ns = rad_ns + b->fld[F_SRVA][id] + b->fld[F_SRVB][id] + b->fld[F_SRVC][id];
    double ct = 1.0 / b->fld[F_DTDT][id];
    return 1.0 / (ct + 1.0 * 1.0 * rad_ns);
}

static double clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* neighbour contribution A+/- (nbr) * dq(nbr) along direction d */
static void nbr_term(const Orc *o, const Blk *b, int i, int j, int k, int d, int side, const double *dqn, double *f) {
    /* side = -1: lower neighbour with npn=+1; side=+1: upper neighbour with npn=-1 */
    int c[3] = {i, j, k};
    c[d] += side;
    double prim[5], g4[4];
    getprim(b, c[0], c[1], c[2], prim);
    getrkec(b, c[0], c[1], c[2], d, g4);
    /* getrarbrc LHS.f90:647-678 (method=1 clamps to 1..n) */
    int cc[3] = {i, j, k};
    int dims[3] = {b->ni, b->nj, b->nk};
    cc[d] = (int)clampi(cc[d] + side, 1, dims[d]);
    const double *sr = b->fld[F_SRA + d];
    double rad = sr[IX(b, cc[0], cc[1], cc[2])];
    mxdq_std(o, prim, g4, dqn, f, rad, side < 0 ? 1 : -1);
}

static void load_dq(const Blk *b, int i, int j, int k, double *v) {
    size_t id = IX(b, i, j, k);
    for (int m = 0; m < 5; m++) v[m] = DQ(b, m)[id];
}

static void lhs_block(Orc *o, Blk *b) {
    int ni = b->ni, nj = b->nj, nk = b->nk;
    zero_physical_faces(b);
    /* store_rhs_nb LHS.f90:1592-1613 */
    for (int m = 0; m < 5; m++) memcpy(b->rhs[m], DQ(b, m), b->ng * 8);
    double dqi[5], dqj[5], dqk[5], de[5], df[5], dg[5], rhs0[5];
    /* lusgs_l LHS.f90:381-478 */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                size_t id = IX(b, i, j, k);
                double coed = coed_of(o, b, id);
                load_dq(b, i - 1, j, k, dqi);
                load_dq(b, i, j - 1, k, dqj);
                load_dq(b, i, j, k - 1, dqk);
                nbr_term(o, b, i, j, k, 0, -1, dqi, de);
                nbr_term(o, b, i, j, k, 1, -1, dqj, df);
                nbr_term(o, b, i, j, k, 2, -1, dqk, dg);
                for (int m = 0; m < 5; m++) rhs0[m] = 1.0 * (de[m] + df[m] + dg[m]);
                if (o->prm.nvis > 0) {
                    double rva = b->fld[F_SRVA][IX(b, i - 1, j, k)];
                    double rvb = b->fld[F_SRVB][IX(b, i, j - 1, k)];
                    double rvc = b->fld[F_SRVC][IX(b, i, j, k - 1)];
                    for (int m = 0; m < 5; m++) rhs0[m] = rhs0[m] + 0.5 * (rva * dqi[m] + rvb * dqj[m] + rvc * dqk[m]);
                }
                for (int m = 0; m < 5; m++) DQ(b, m)[id] = (-DQ(b, m)[id] + rhs0[m]) * coed;
            }
    /* lusgs_u LHS.f90:480-577 */
    for (int k = nk; k >= 1; k--)
        for (int j = nj; j >= 1; j--)
            for (int i = ni; i >= 1; i--) {
                size_t id = IX(b, i, j, k);
                double coed = coed_of(o, b, id);
                load_dq(b, i + 1, j, k, dqi);
                load_dq(b, i, j + 1, k, dqj);
                load_dq(b, i, j, k + 1, dqk);
                nbr_term(o, b, i, j, k, 0, 1, dqi, de);
                nbr_term(o, b, i, j, k, 1, 1, dqj, df);
                nbr_term(o, b, i, j, k, 2, 1, dqk, dg);
                for (int m = 0; m < 5; m++) rhs0[m] = 1.0 * (de[m] + df[m] + dg[m]);
                if (o->prm.nvis > 0) {
                    double rva = b->fld[F_SRVA][IX(b, i + 1, j, k)];
                    double rvb = b->fld[F_SRVB][IX(b, i, j + 1, k)];
                    double rvc = b->fld[F_SRVC][IX(b, i, j, k + 1)];
                    for (int m = 0; m < 5; m++) rhs0[m] = rhs0[m] - 0.5 * (rva * dqi[m] + rvb * dqj[m] + rvc * dqk[m]);
                }
                for (int m = 0; m < 5; m++) DQ(b, m)[id] = DQ(b, m)[id] - rhs0[m] * coed;
            }
    /* gs_pr_l (LHS.f90:1777-1866) and gs_pr_u (LHS.f90:1956-2046) */
    for (int pass = 0; pass < 2; pass++) {
        for (int kk = 1; kk <= nk; kk++)
            for (int jj = 1; jj <= nj; jj++)
                for (int ii = 1; ii <= ni; ii++) {
                    int i = pass ? ni + 1 - ii : ii, j = pass ? nj + 1 - jj : jj, k = pass ? nk + 1 - kk : kk;
                    size_t id = IX(b, i, j, k);
                    double coed = coed_of(o, b, id);
                    double del[5], dfl[5], dgl[5], der[5], dfr[5], dgr[5];
                    load_dq(b, i - 1, j, k, dqi);
                    load_dq(b, i, j - 1, k, dqj);
                    load_dq(b, i, j, k - 1, dqk);
                    if (i == 1) memset(dqi, 0, sizeof dqi);
                    if (j == 1) memset(dqj, 0, sizeof dqj);
                    if (k == 1) memset(dqk, 0, sizeof dqk);
                    nbr_term(o, b, i, j, k, 0, -1, dqi, del);
                    nbr_term(o, b, i, j, k, 1, -1, dqj, dfl);
                    nbr_term(o, b, i, j, k, 2, -1, dqk, dgl);
                    load_dq(b, i + 1, j, k, dqi);
                    load_dq(b, i, j + 1, k, dqj);
                    load_dq(b, i, j, k + 1, dqk);
                    if (i == ni) memset(dqi, 0, sizeof dqi);
                    if (j == nj) memset(dqj, 0, sizeof dqj);
                    if (k == nk) memset(dqk, 0, sizeof dqk);
                    nbr_term(o, b, i, j, k, 0, 1, dqi, der);
                    nbr_term(o, b, i, j, k, 1, 1, dqj, dfr);
                    nbr_term(o, b, i, j, k, 2, 1, dqk, dgr);
                    for (int m = 0; m < 5; m++) rhs0[m] = 1.0 * (del[m] + dfl[m] + dgl[m] - der[m] - dfr[m] - dgr[m]);
                    for (int m = 0; m < 5; m++) DQ(b, m)[id] = (rhs0[m] - b->rhs[m][id]) * coed;
                }
    }
    zero_physical_faces(b);
}

/* update_limited, Sub2.f90:603-794.  Returns the bad-point count. */
static int update_block(Orc *o, Blk *b) {
    double gama = o->gama, gamam1 = gama - 1.0;
    int n_count = 0;
    for (int k = 1; k <= b->nk; k++)
        for (int j = 1; j <= b->nj; j++)
            for (int i = 1; i <= b->ni; i++) {
                size_t id = IX(b, i, j, k);
                double qt[5];
                for (int m = 0; m < 5; m++) qt[m] = b->fld[F_Q1 + m][id] + DQ(b, m)[id];
                double rm = qt[0], rm1 = 1.0 / rm;
                double um = qt[1] * rm1, vm = qt[2] * rm1, wm = qt[3] * rm1, em = qt[4];
                double pm = gamam1 * (em - 0.5 * rm * (um * um + vm * vm + wm * wm));
                double pd = fabs((pm - P(b)[id]) / P(b)[id]) + -0.3;
                double mx = 0.0 > pd ? 0.0 : pd;
                double Falpha = 1. / (1. + 2. * mx);
                for (int m = 0; m < 5; m++) {
                    qt[m] = b->fld[F_Q1 + m][id] + DQ(b, m)[id] * Falpha;
                    b->fld[F_Q1 + m][id] = qt[m];
                }
                rm = qt[0];
                rm1 = 1.0 / rm;
                um = qt[1] * rm1; vm = qt[2] * rm1; wm = qt[3] * rm1; em = qt[4];
                pm = gamam1 * (em - 0.5 * rm * (um * um + vm * vm + wm * wm));
                if (pm <= PMIN_LIMIT || rm <= RMIN_LIMIT || pm >= PMAX_LIMIT || rm >= RMAX_LIMIT) {
                    n_count++;
                    rm = 0.0; um = 0.0; vm = 0.0; wm = 0.0; pm = 0.0;
                    int np = 0;
                    for (int ii = -1; ii <= 1; ii++)
                        for (int jj = -1; jj <= 1; jj++)
                            for (int kk = -1; kk <= 1; kk++)
                                if (abs(ii) + abs(jj) + abs(kk) == 1) {
                                    np++;
                                    size_t n = IX(b, i + ii, j + jj, k + kk);
                                    rm = rm + R(b)[n]; um = um + U(b)[n]; vm = vm + V(b)[n]; wm = wm + W(b)[n]; pm = pm + P(b)[n];
                                }
                    double rnp = (double)np;
                    rm = rm / rnp; um = um / rnp; vm = vm / rnp; wm = wm / rnp; pm = pm / rnp;
                    em = pm / (gama - 1.0) + 0.5 * rm * (um * um + vm * vm + wm * wm);
                    b->fld[F_Q1][id] = rm;
                    b->fld[F_Q2][id] = rm * um;
                    b->fld[F_Q3][id] = rm * vm;
                    b->fld[F_Q4][id] = rm * wm;
                    b->fld[F_Q5][id] = em;
                }
                R(b)[id] = rm; U(b)[id] = um; V(b)[id] = vm; W(b)[id] = wm; P(b)[id] = pm;
            }
    return n_count;
}

int orc_lhs(void *h) {
    Orc *o = h;
    int fail = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : fail)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        lhs_block(o, b);
        int n = update_block(o, b);
        if (n > b->ni * b->nj * b->nk / 64 || n >= 500) fail |= 1;
    }
    if (fail) { set_err("update_limited: too many non-physical points"); return 3; }
    return 0;
}

/* residual_curve, PostProcess.f90:1195-1347 (ndualtst=0) */
int orc_residual(void *h, double *res_per_block, double *resmax_per_block, double *rms) {
    Orc *o = h;
    double dres_add = 0.0;
    long np = 0;
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        double res = 0.0, resmax = 0.0;
        for (int k = 2; k <= b->nk - 1; k++)
            for (int j = 2; j <= b->nj - 1; j++)
                for (int i = 2; i <= b->ni - 1; i++) {
                    size_t id = IX(b, i, j, k);
                    double dtime1 = 1.0 / (b->fld[F_DTDT][id] * b->fld[F_VOL][id]);
                    for (int m = 0; m < 5; m++) {
                        double dq0 = fabs(DQ(b, m)[id]);
                        double dresm = dq0 * dtime1;
                        if (dresm > resmax) resmax = dresm;
                        res = res + dresm * dresm;
                    }
                }
        dres_add = dres_add + res;
        long npb = (long)(b->ni - 2) * (b->nj - 2) * (b->nk - 2) * 5;
        if (res_per_block) res_per_block[nb - 1] = res / npb;
        if (resmax_per_block) resmax_per_block[nb - 1] = resmax;
        np += npb;
    }
    if (rms) *rms = sqrt(dres_add / np);
    return 0;
}

int orc_step(void *h, int nsteps, double *rms_history) {
    Orc *o = h;
#ifdef _OPENMP
    if (o->prm.nthreads > 0) omp_set_num_threads(o->prm.nthreads);
#endif
    for (int s = 0; s < nsteps; s++) {
        int rc;
        orc_boundary_all(o);
        orc_initial_q_dq_c_t(o);
        orc_timestep(o);
        if (o->prm.nvis == 1) {
            orc_rhs_vis(o);
            orc_communicate_dq(o);
        }
        if ((rc = orc_rhs_invis(o))) return rc;
        orc_communicate_dq(o);
        if ((rc = orc_lhs(o))) return rc;
        orc_communicate_pv(o);
        double rms = 0;
        orc_residual(o, NULL, NULL, &rms);
        if (rms_history) rms_history[s] = rms;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Line-operator hooks for the known-answer tests                      */
/* ------------------------------------------------------------------ */

/* ------------------------------------------------------------------ */
/* Wall forces: force (PostProcess.f90:1415-1480), force_dif (1505-1678), */
/* getforce (1680-1824), getuvwtder (Sub1.f90:383-480), getgeo,          */
/* getduvwdxyz, stress (Sub1.f90:181-270), aver3/halen/lenth (858-889).  */
/* ------------------------------------------------------------------ */
static double lenth(double x1, double y1, double z1, double x2, double y2, double z2) {
    double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    return sqrt(dx * dx + dy * dy + dz * dz);
}
static double halen(double a, double b, double c) {
    double p = 0.5 * (a + b + c);
    double s = p * (p - a) * (p - b) * (p - c);
    if (s < 0) return 0.0;
    return sqrt(s);
}
static double aver3(double a, double b, double c) { return (a + b + c) / 3.0; }

static void getforce(const double *px, const double *py, const double *pz, const double *xx, const double *yy,
                     const double *zz, const double *ref, double *d) {
    double px5 = 0.25 * (px[0] + px[1] + px[2] + px[3]);
    double py5 = 0.25 * (py[0] + py[1] + py[2] + py[3]);
    double pz5 = 0.25 * (pz[0] + pz[1] + pz[2] + pz[3]);
    double x5 = 0.25 * (xx[0] + xx[1] + xx[2] + xx[3]);
    double y5 = 0.25 * (yy[0] + yy[1] + yy[2] + yy[3]);
    double z5 = 0.25 * (zz[0] + zz[1] + zz[2] + zz[3]);
    double r12 = lenth(xx[0], yy[0], zz[0], xx[1], yy[1], zz[1]);
    double r23 = lenth(xx[1], yy[1], zz[1], xx[2], yy[2], zz[2]);
    double r34 = lenth(xx[2], yy[2], zz[2], xx[3], yy[3], zz[3]);
    double r41 = lenth(xx[3], yy[3], zz[3], xx[0], yy[0], zz[0]);
    double r15 = lenth(xx[0], yy[0], zz[0], x5, y5, z5);
    double r25 = lenth(xx[1], yy[1], zz[1], x5, y5, z5);
    double r35 = lenth(xx[2], yy[2], zz[2], x5, y5, z5);
    double r45 = lenth(xx[3], yy[3], zz[3], x5, y5, z5);
    double s[4] = {halen(r12, r15, r25), halen(r23, r25, r35), halen(r34, r35, r45), halen(r41, r45, r15)};
    double xref = ref[2], yref = ref[3], zref = ref[4];
    for (int c = 0; c < 6; c++) d[c] = 0.0;
    for (int t = 0; t < 4; t++) {
        int a = t, bq = (t + 1) % 4;
        double pxc = aver3(px[a], px[bq], px5), pyc = aver3(py[a], py[bq], py5), pzc = aver3(pz[a], pz[bq], pz5);
        double xc = aver3(xx[a], xx[bq], x5), yc = aver3(yy[a], yy[bq], y5), zc = aver3(zz[a], zz[bq], z5);
        double ddfx = pxc * s[t], ddfy = pyc * s[t], ddfz = pzc * s[t];
        double ddmx = (yc - yref) * ddfz - (zc - zref) * ddfy;
        double ddmy = (zc - zref) * ddfx - (xc - xref) * ddfz;
        double ddmz = (xc - xref) * ddfy - (yc - yref) * ddfx;
        d[0] = d[0] + ddfx; d[1] = d[1] + ddfy; d[2] = d[2] + ddfz;
        d[3] = d[3] + ddmx; d[4] = d[4] + ddmy; d[5] = d[5] + ddmz;
    }
}

/* surface force per unit-normalised wall point: pressure and, for viscous
 * runs, the stress tensor from 2nd-order node derivatives */
static void wall_point_force(const Orc *o, const Blk *b, const Reg *rg, int i, int j, int k, double *pf) {
    double nx, ny, nz;
    getnxyz(b, &nx, &ny, &nz, i, j, k, rg->s_lr3d[0], rg->s_lr3d[1], rg->s_lr3d[2]);
    size_t id = IX(b, i, j, k);
    double pn = 2.0 * (P(b)[id] - o->poo);
    double slr = (double)rg->s_lr;
    pf[0] = slr * nx * pn;
    pf[1] = slr * ny * pn;
    pf[2] = slr * nz * pn;
    if (o->prm.nvis != 1) return;
    const double *fu[4] = {U(b), V(b), W(b), T(b)};
    int c[3] = {i, j, k}, dims[3] = {b->ni, b->nj, b->nk};
    double der[3][4]; /* [direction][u,v,w,t] */
    for (int d = 0; d < 3; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        for (int m = 0; m < 4; m++) {
            const double *f = fu[m];
            if (c[d] == 1) {
                double f1 = f[id], f2 = f[IX(b, i + e[0], j + e[1], k + e[2])], f3 = f[IX(b, i + 2 * e[0], j + 2 * e[1], k + 2 * e[2])];
                der[d][m] = -(1.5 * f1 + -2.0 * f2 + 0.5 * f3);
            } else if (c[d] == dims[d]) {
                double f1 = f[id], f2 = f[IX(b, i - e[0], j - e[1], k - e[2])], f3 = f[IX(b, i - 2 * e[0], j - 2 * e[1], k - 2 * e[2])];
                der[d][m] = 1.5 * f1 + -2.0 * f2 + 0.5 * f3;
            } else {
                double fp = f[IX(b, i + e[0], j + e[1], k + e[2])], fm = f[IX(b, i - e[0], j - e[1], k - e[2])];
                der[d][m] = 0.5 * (fp - fm);
            }
        }
    }
    double kx = b->fld[F_KCX][id], ky = b->fld[F_KCY][id], kz = b->fld[F_KCZ][id];
    double ex = b->fld[F_ETX][id], ey = b->fld[F_ETY][id], ez = b->fld[F_ETZ][id];
    double cx = b->fld[F_CTX][id], cy = b->fld[F_CTY][id], cz = b->fld[F_CTZ][id];
    double vj = b->fld[F_VOL][id];
    double dudx = (kx * der[0][0] + ex * der[1][0] + cx * der[2][0]) / vj;
    double dudy = (ky * der[0][0] + ey * der[1][0] + cy * der[2][0]) / vj;
    double dudz = (kz * der[0][0] + ez * der[1][0] + cz * der[2][0]) / vj;
    double dvdx = (kx * der[0][1] + ex * der[1][1] + cx * der[2][1]) / vj;
    double dvdy = (ky * der[0][1] + ey * der[1][1] + cy * der[2][1]) / vj;
    double dvdz = (kz * der[0][1] + ez * der[1][1] + cz * der[2][1]) / vj;
    double dwdx = (kx * der[0][2] + ex * der[1][2] + cx * der[2][2]) / vj;
    double dwdy = (ky * der[0][2] + ey * der[1][2] + cy * der[2][2]) / vj;
    double dwdz = (kz * der[0][2] + ez * der[1][2] + cz * der[2][2]) / vj;
    const double c23 = 0.66666666667;
    double vis = b->fld[F_VISL][id];
    double txx = vis * c23 * (2.0 * dudx - dvdy - dwdz);
    double tyy = vis * c23 * (2.0 * dvdy - dwdz - dudx);
    double tzz = vis * c23 * (2.0 * dwdz - dudx - dvdy);
    double txy = vis * (dudy + dvdx);
    double txz = vis * (dudz + dwdx);
    double tyz = vis * (dvdz + dwdy);
    double tyx = txy, tzx = txz, tzy = tyz;
    double re = 1.0 / o->reynolds;
    pn = 2.0 * slr;
    pf[0] = pf[0] - pn * (nx * txx + ny * tyx + nz * tzx) * re;
    pf[1] = pf[1] - pn * (nx * txy + ny * tyy + nz * tzy) * re;
    pf[2] = pf[2] - pn * (nx * txz + ny * tyz + nz * tzz) * re;
}

int orc_forces(void *h, const double *ref, double *out) {
    Orc *o = h;
    double cf[6] = {0, 0, 0, 0, 0, 0};
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int nr = 0; nr < b->nreg; nr++) {
            Reg *rg = &b->reg[nr];
            if (!(rg->bctype == 2 || rg->bctype / 10 == 2)) continue;
            int id_ = 1 - abs(rg->s_lr3d[0]), jd = 1 - abs(rg->s_lr3d[1]), kd = 1 - abs(rg->s_lr3d[2]);
            int e0 = rg->s_ed[0] - rg->s_st[0] + 1, e1 = rg->s_ed[1] - rg->s_st[1] + 1, e2 = rg->s_ed[2] - rg->s_st[2] + 1;
            double *pf = malloc(sizeof(double) * 3 * (size_t)e0 * e1 * e2);
#define PF(i, j, k) (pf + 3 * (size_t)(((i) - rg->s_st[0]) + e0 * (((j) - rg->s_st[1]) + e1 * ((k) - rg->s_st[2]))))
            for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                    for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++) wall_point_force(o, b, rg, i, j, k, PF(i, j, k));
            for (int i = rg->s_st[0]; i <= rg->s_ed[0] - id_; i++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1] - jd; j++)
                    for (int k = rg->s_st[2]; k <= rg->s_ed[2] - kd; k++) {
                        int q[4][3] = {{i, j, k}, {0}, {0}, {0}};
                        if (id_ == 0) { q[1][0] = i; q[1][1] = j + 1; q[1][2] = k; q[2][0] = i; q[2][1] = j + 1; q[2][2] = k + 1; q[3][0] = i; q[3][1] = j; q[3][2] = k + 1; }
                        if (jd == 0) { q[1][0] = i + 1; q[1][1] = j; q[1][2] = k; q[2][0] = i + 1; q[2][1] = j; q[2][2] = k + 1; q[3][0] = i; q[3][1] = j; q[3][2] = k + 1; }
                        if (kd == 0) { q[1][0] = i + 1; q[1][1] = j; q[1][2] = k; q[2][0] = i + 1; q[2][1] = j + 1; q[2][2] = k; q[3][0] = i; q[3][1] = j + 1; q[3][2] = k; }
                        double px[4], py[4], pz[4], xx[4], yy[4], zz[4], d[6];
                        for (int v = 0; v < 4; v++) {
                            const double *f = PF(q[v][0], q[v][1], q[v][2]);
                            px[v] = f[0]; py[v] = f[1]; pz[v] = f[2];
                            size_t g = (size_t)(q[v][0] - 1) + (size_t)b->ni * ((size_t)(q[v][1] - 1) + (size_t)b->nj * (q[v][2] - 1));
                            xx[v] = b->xyz[0][g]; yy[v] = b->xyz[1][g]; zz[v] = b->xyz[2][g];
                        }
                        getforce(px, py, pz, xx, yy, zz, ref, d);
                        for (int cc = 0; cc < 6; cc++) cf[cc] = cf[cc] + d[cc];
                    }
#undef PF
            free(pf);
        }
    }
    double sref = ref[0], lfref = ref[1], whole = ref[5];
    double scf = 1.0 / sref, vcm = 1.0 / (sref * lfref);
    for (int cc = 0; cc < 3; cc++) out[cc] = (2 - whole) * cf[cc] * scf;
    for (int cc = 3; cc < 6; cc++) out[cc] = (2 - whole) * cf[cc] * vcm;
    double attack = o->prm.attack * PAI / 180.0, sideslip = o->prm.sideslip * PAI / 180.0;
    double sina = sin(attack), cosa = cos(attack), sinb = sin(sideslip), cosb = cos(sideslip);
    out[6] = out[1] * cosa - out[0] * sina;
    out[7] = cosb * (out[1] * sina + out[0] * cosa) + sinb * out[2];
    out[8] = copysign(1.0, out[1]) * out[5] / (fabs(out[1]) + 1.0e-38);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Spalart-Allmaras model: turbulence -> differential_model_turbulence */
/* (turblence.f90:15-103) with nlamtur=1, nameturb='SA', ncmpcor<=9,   */
/* ndes=0, ntrans=0, nwtmax=0 and method=1 (finite differences).       */
/* ------------------------------------------------------------------ */
/* model constants, cal_rhs_source_SA turblence.f90:2508-2513 */
#define SA_CB1 0.1355
#define SA_CB2 0.622
#define SA_CV1 7.1
#define SA_EPS 1.0e-20
#define SA_CGA (2. / 3.0)
#define SA_KI 0.419
#define SA_CW2 0.3
#define SA_CW3 2.0
#define SA_MUOO 1.0e-1 /* inflow_turbulence, turblence.f90:3174 */
#define SA_MINLIM 1.0e-20 /* update_turbulence, turblence.f90:589 */

/* calc_wall_dists_parallel, parallel.f90:4313-4470: squared distance to the
 * nearest point of any bctype 2, 20 or 21 region (all blocks), then
 * sqrt + small, over the block's points 1..n */
static void sa_wall_distance(Orc *o) {
    size_t nw = 0;
    for (int nb = 1; nb <= o->nb; nb++)
        for (int r = 0; r < o->b[nb].nreg; r++) {
            const Reg *rg = &o->b[nb].reg[r];
            if (rg->bctype == 2 || rg->bctype == 20 || rg->bctype == 21)
                nw += (size_t)(rg->s_ed[0] - rg->s_st[0] + 1) * (rg->s_ed[1] - rg->s_st[1] + 1) * (rg->s_ed[2] - rg->s_st[2] + 1);
        }
    double *wp = malloc((nw ? nw : 1) * 3 * sizeof(double));
    size_t m = 0;
    for (int nb = 1; nb <= o->nb; nb++) {
        const Blk *b = &o->b[nb];
        for (int r = 0; r < b->nreg; r++) {
            const Reg *rg = &b->reg[r];
            if (!(rg->bctype == 2 || rg->bctype == 20 || rg->bctype == 21)) continue;
            for (int k = rg->s_st[2]; k <= rg->s_ed[2]; k++)
                for (int j = rg->s_st[1]; j <= rg->s_ed[1]; j++)
                    for (int i = rg->s_st[0]; i <= rg->s_ed[0]; i++) {
                        size_t g = (size_t)(i - 1) + (size_t)b->ni * ((size_t)(j - 1) + (size_t)b->nj * (k - 1));
                        for (int c = 0; c < 3; c++) wp[3 * m + c] = b->xyz[c][g];
                        m++;
                    }
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        for (int k = 1; k <= b->nk; k++)
            for (int j = 1; j <= b->nj; j++)
                for (int i = 1; i <= b->ni; i++) {
                    size_t g = (size_t)(i - 1) + (size_t)b->ni * ((size_t)(j - 1) + (size_t)b->nj * (k - 1));
                    double xc = b->xyz[0][g], yc = b->xyz[1][g], zc = b->xyz[2][g];
                    double d = 1.0e30;
                    for (size_t w = 0; w < nw; w++) {
                        double dx = xc - wp[3 * w], dy = yc - wp[3 * w + 1], dz = zc - wp[3 * w + 2];
                        double dist = dx * dx + dy * dy + dz * dz;
                        d = dist < d ? dist : d;
                    }
                    b->dist[IX(b, i, j, k)] = sqrt(d) + SMALL;
                }
    }
    free(wp);
}

/* init_SA, turblence.f90:2701-2733: qke = muoo, vist = muoo*fv1(muoo) over
 * -1..n+1 */
static void sa_init(Blk *b, double cv13) {
    double kafan = SA_MUOO;
    double kf3 = pow(kafan, 3.0);
    double fv1 = kf3 / (kf3 + cv13);
    double vt = SA_MUOO * fv1;
    for (int k = -1; k <= b->nk + 1; k++)
        for (int j = -1; j <= b->nj + 1; j++)
            for (int i = -1; i <= b->ni + 1; i++) {
                b->qke[IX(b, i, j, k)] = SA_MUOO;
                b->vist[IX(b, i, j, k)] = vt;
            }
}

int orc_sa_setup(void *h, double timedt_turb, double kmaxlim) { return orc_sa_setup_ex(h, timedt_turb, kmaxlim, 1); }

int orc_sa_setup_ex(void *h, double timedt_turb, double kmaxlim, int with_distance) {
    Orc *o = h;
    const double cv13 = pow(SA_CV1, 3.0);
    for (int nb = 1; nb <= o->nb; nb++) {
        Blk *b = &o->b[nb];
        if (!b->qke) {
            b->qke = calloc(b->ng, sizeof(double));
            b->dist = calloc(b->ng, sizeof(double));
            b->dqke = calloc(b->ng, sizeof(double));
            b->spec = calloc(b->ng, sizeof(double));
            b->viseq = calloc(b->ng, sizeof(double));
            b->sa_snap = calloc(2 * b->ng, sizeof(double));
            for (int c = 0; c < 3; c++) b->dmu[c] = calloc(b->ng, sizeof(double));
        }
        sa_init(b, cv13);
    }
    o->timedt_turb = timedt_turb;
    o->kmaxlim = kmaxlim;
    if (!o->sa) o->sa_bc = 1; /* the reference always applies the model's BC rules (nlamtur >= 0) */
    o->sa = 1;
    if (with_distance) sa_wall_distance(o);
    return 0;
}

/* dfidxyz_center, turblence.f90:753-849 (finite-difference branch) at one
 * point: central differences along i, j, k mapped to x, y, z */
static void sa_center_deriv(const Blk *b, const double *fi, int i, int j, int k, double *d) {
    size_t id = IX(b, i, j, k);
    double dkc = fi[IX(b, i + 1, j, k)] - fi[IX(b, i - 1, j, k)];
    double det = fi[IX(b, i, j + 1, k)] - fi[IX(b, i, j - 1, k)];
    double dct = fi[IX(b, i, j, k + 1)] - fi[IX(b, i, j, k - 1)];
    double *const *f = b->fld;
    double ddx = dkc * f[F_KCX][id] + det * f[F_ETX][id] + dct * f[F_CTX][id];
    double ddy = dkc * f[F_KCY][id] + det * f[F_ETY][id] + dct * f[F_CTY][id];
    double ddz = dkc * f[F_KCZ][id] + det * f[F_ETZ][id] + dct * f[F_CTZ][id];
    double vol2 = 0.5 / f[F_VOL][id];
    d[0] = ddx * vol2;
    d[1] = ddy * vol2;
    d[2] = ddz * vol2;
}

/* minmod, Convect.f90:1281-1286 */
static double minmod(double x, double y) {
    return 0.5 * (copysign(1.0, x) + copysign(1.0, y)) * fmin(fabs(x), fabs(y));
}

/* flux_turbulence, turblence.f90:437-459 */
static double sa_flux(const double *prim, double nx, double ny, double nz, int npn) {
    double l1 = nx * prim[1] + ny * prim[2] + nz * prim[3];
    l1 = 0.5 * (l1 + (double)npn * sqrt(l1 * l1));
    return l1 * prim[4] * prim[0];
}

/* mxdq_std_turbulence, turblence.f90:560-583 */
static double sa_mxdq(const double *prim, const double *g, double dq, int npn) {
    double l1 = g[0] * prim[1] + g[1] * prim[2] + g[2] * prim[3];
    l1 = 0.5 * (l1 + (double)npn * fabs(l1));
    return l1 * dq;
}

static void sa_block(const Orc *o, Blk *b) {
    const int ni = b->ni, nj = b->nj, nk = b->nk;
    const int n3[3] = {ni, nj, nk};
    const double reynolds = o->reynolds, re = 1.0 / reynolds;
    const double cv13 = pow(SA_CV1, 3.0), ki2 = SA_KI * SA_KI, cw36 = pow(SA_CW3, 6.0), onesix = 1.0 / 6.0;
    const double cw1 = SA_CB1 / SA_KI / SA_KI + (1.0 + SA_CB2) / SA_CGA;
    const double ft2 = 0.0;
    double *const *f = b->fld;
    /* set_dq_to_zero_turbulence, turblence.f90:270-289 */
    memset(b->dqke, 0, b->ng * sizeof(double));
    memset(b->spec, 0, b->ng * sizeof(double));
    /* cal_rhs_source_SA, turblence.f90:2506-2699: derivatives of qke over 1..n
     * (those of u, v, w are taken where they are used) */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                double d[3];
                sa_center_deriv(b, b->qke, i, j, k, d);
                for (int c = 0; c < 3; c++) b->dmu[c][IX(b, i, j, k)] = d[c];
            }
    for (int k = 2; k <= nk - 1; k++)
        for (int j = 2; j <= nj - 1; j++)
            for (int i = 2; i <= ni - 1; i++) {
                size_t id = IX(b, i, j, k);
                double du[3], dv[3], dw[3];
                sa_center_deriv(b, f[F_U], i, j, k, du);
                sa_center_deriv(b, f[F_V], i, j, k, dv);
                sa_center_deriv(b, f[F_W], i, j, k, dw);
                double ro = R(b)[id], volume = f[F_VOL][id], vsl = f[F_VISL][id], vtbar = b->qke[id];
                double romu = ro * vtbar;
                double dn = b->dist[id] > re ? b->dist[id] : re;
                double dn2 = dn * dn;
                double reki2dn2 = reynolds * ki2 * dn2;
                double kafan = romu / vsl;
                double kf3 = pow(kafan, 3.0);
                double fv1 = kf3 / (kf3 + cv13);
                double fv2 = 1.0 - kafan / (1.0 + kafan * fv1);
                double a = du[1] - dv[0], bb = dv[2] - dw[1], c = dw[0] - du[2];
                double omg = sqrt(a * a + bb * bb + c * c);
                double sbar = omg + vtbar / reki2dn2 * fv2;
                sbar = sbar > SA_EPS ? sbar : SA_EPS;
                double rbar = vtbar / (sbar * reki2dn2);
                rbar = rbar < 10.0 ? rbar : 10.0;
                double rbar5 = pow(rbar, 5.0);
                double gbar = rbar + SA_CW2 * rbar * (rbar5 - 1.0);
                double gbar6 = pow(gbar, 6.0);
                double fw = gbar * pow((1.0 + cw36) / (gbar6 + cw36), onesix);
                double cpmu = SA_CB1 * (1.0 - ft2) * sbar;
                double cdmu = (cw1 * fw - SA_CB1 * ft2 / ki2) * vtbar / dn2 / reynolds;
                double sp = cpmu * vtbar, sd = cdmu * vtbar;
                double dmx = b->dmu[0][id], dmy = b->dmu[1][id], dmz = b->dmu[2][id];
                double dbar = SA_CB2 / SA_CGA * (dmx * dmx + dmy * dmy + dmz * dmz) * re;
                b->dqke[id] = b->dqke[id] - ro * (sp - sd + dbar) * volume;
                double sm = cpmu - 2.0 * cdmu;
                b->spec[id] = b->spec[id] - (sm < 0.0 ? sm : 0.0) * volume;
            }
    /* viscosity_equivalent_SA_r, turblence.f90:2785-2808, over 1..n */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                size_t id = IX(b, i, j, k);
                b->viseq[id] = 1.5 * (f[F_VISL][id] / R(b)[id] + b->qke[id]);
            }
    /* cal_rhs_viscous_turbulence_dif_r, turblence.f90:1022-1185: per
     * direction the half-point fluxes 2..n, differenced into 2..n-1 */
    for (int d = 0; d < 3; d++) {
        const double *mx = metric_dir(b, d, 0), *my = metric_dir(b, d, 1), *mz = metric_dir(b, d, 2);
        for (int k = 2; k <= nk - 1; k++)
            for (int j = 2; j <= nj - 1; j++)
                for (int i = 2; i <= ni - 1; i++) {
                    int c[3] = {i, j, k};
                    double fvl[2];
                    for (int h = 0; h < 2; h++) {
                        int cm[3] = {i, j, k}, cn[3] = {i, j, k};
                        cm[d] = c[d] + h;      /* half point l = c[d] + h between l-1 and l */
                        cn[d] = c[d] + h - 1;
                        size_t im = IX(b, cm[0], cm[1], cm[2]), in = IX(b, cn[0], cn[1], cn[2]);
                        double nx = 0.5 * (mx[im] + mx[in]);
                        double ny = 0.5 * (my[im] + my[in]);
                        double nz = 0.5 * (mz[im] + mz[in]);
                        double dmudx = b->dmu[0][im] + b->dmu[0][in];
                        double dmudy = b->dmu[1][im] + b->dmu[1][in];
                        double dmudz = b->dmu[2][im] + b->dmu[2][in];
                        double vis = b->viseq[im] + b->viseq[in];
                        fvl[h] = (dmudx * nx + dmudy * ny + dmudz * nz) * vis * 0.25;
                    }
                    size_t id = IX(b, i, j, k);
                    b->dqke[id] = b->dqke[id] - re * R(b)[id] * (fvl[1] - fvl[0]);
                }
    }
    /* cal_spec_turbulence_r, turblence.f90:218-259 */
    const double re2 = re * 2.0;
    for (int k = 2; k <= nk - 1; k++)
        for (int j = 2; j <= nj - 1; j++)
            for (int i = 2; i <= ni - 1; i++) {
                size_t id = IX(b, i, j, k);
                double u = U(b)[id], v = V(b)[id], w = W(b)[id];
                double unx = u * f[F_KCX][id] + v * f[F_KCY][id] + w * f[F_KCZ][id];
                double uny = u * f[F_ETX][id] + v * f[F_ETY][id] + w * f[F_ETZ][id];
                double unz = u * f[F_CTX][id] + v * f[F_CTY][id] + w * f[F_CTZ][id];
                b->spec[id] = b->spec[id] + fabs(unx) + fabs(uny) + fabs(unz) + 1.0 / (f[F_DTDT][id] * o->timedt_turb);
                double nx = f[F_KCX][id] * f[F_KCX][id] + f[F_KCY][id] * f[F_KCY][id] + f[F_KCZ][id] * f[F_KCZ][id];
                double ny = f[F_ETX][id] * f[F_ETX][id] + f[F_ETY][id] * f[F_ETY][id] + f[F_ETZ][id] * f[F_ETZ][id];
                double nz = f[F_CTX][id] * f[F_CTX][id] + f[F_CTY][id] * f[F_CTY][id] + f[F_CTZ][id] * f[F_CTZ][id];
                double vis = b->viseq[id] / f[F_VOL][id];
                b->spec[id] = b->spec[id] + re2 * vis * (nx + ny + nz);
            }
    /* cal_rhs_inviscous_turbulence + NND_turbulence, turblence.f90:291-435,
     * xk = xb = 0 (never assigned in the reference) */
    const double xk = 0.0, xb = 0.0, c1 = 0.25 * (1.0 + xk), c2 = 0.25 * (1.0 - xk);
    for (int d = 0; d < 3; d++) {
        const int n = n3[d];
        const double *mx = metric_dir(b, d, 0), *my = metric_dir(b, d, 1), *mz = metric_dir(b, d, 2);
        const int la = d == 0 ? 1 : 0, lb = d == 2 ? 1 : 2;  /* the two other directions */
        for (int bq = 2; bq <= n3[lb] - 1; bq++)
            for (int aq = 2; aq <= n3[la] - 1; aq++) {
                double *ql = malloc((size_t)(n + 3) * 5 * sizeof(double));   /* l = -1..n+1 */
                double *dqv = malloc((size_t)(n + 3) * 5 * sizeof(double));
                double *qcl = malloc((size_t)(n + 3) * 5 * sizeof(double));
                double *qcr = malloc((size_t)(n + 3) * 5 * sizeof(double));
                double *fc = malloc((size_t)(n + 3) * sizeof(double));
#define QL(m, l) ql[5 * ((l) + 1) + (m)]
#define DQV(m, l) dqv[5 * ((l) + 1) + (m)]
#define QCL(m, l) qcl[5 * ((l) + 1) + (m)]
#define QCR(m, l) qcr[5 * ((l) + 1) + (m)]
                for (int l = 0; l <= n + 1; l++) {
                    int c[3];
                    c[d] = l; c[la] = aq; c[lb] = bq;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    QL(0, l) = R(b)[id]; QL(1, l) = U(b)[id]; QL(2, l) = V(b)[id]; QL(3, l) = W(b)[id];
                    QL(4, l) = b->qke[id];
                }
                for (int l = 1; l <= n + 1; l++)
                    for (int m = 0; m < 5; m++) DQV(m, l) = QL(m, l) - QL(m, l - 1);
                for (int l = 1; l <= n; l++)
                    for (int m = 0; m < 5; m++) {
                        QCL(m, l) = minmod(xb * DQV(m, l + 1), DQV(m, l));
                        QCR(m, l) = minmod(DQV(m, l + 1), xb * DQV(m, l));
                    }
                for (int l = 2; l <= n; l++) {
                    int c0[3], c1i[3];
                    c0[d] = l - 1; c0[la] = aq; c0[lb] = bq;
                    c1i[d] = l; c1i[la] = aq; c1i[lb] = bq;
                    size_t i0 = IX(b, c0[0], c0[1], c0[2]), i1 = IX(b, c1i[0], c1i[1], c1i[2]);
                    double nx = 0.50 * (mx[i0] + mx[i1]);
                    double ny = 0.50 * (my[i0] + my[i1]);
                    double nz = 0.50 * (mz[i0] + mz[i1]);
                    double dql[5], dqr[5];
                    for (int m = 0; m < 5; m++) {
                        dql[m] = QL(m, l - 1) + c1 * QCR(m, l - 1) + c2 * QCL(m, l - 1);
                        dqr[m] = QL(m, l) - c1 * QCL(m, l) - c2 * QCR(m, l);
                    }
                    double fl = sa_flux(dql, nx, ny, nz, 1);
                    double fr = sa_flux(dqr, nx, ny, nz, -1);
                    fc[l] = fl + fr;
                }
                for (int l = 2; l <= n - 1; l++) {
                    int c[3];
                    c[d] = l; c[la] = aq; c[lb] = bq;
                    size_t id = IX(b, c[0], c[1], c[2]);
                    b->dqke[id] = b->dqke[id] + (fc[l + 1] - fc[l]);
                }
#undef QL
#undef DQV
#undef QCL
#undef QCR
                free(ql); free(dqv); free(qcl); free(qcr); free(fc);
            }
    }
    /* lusgs_turbulence, turblence.f90:477-558 */
    for (int k = 2; k <= nk - 1; k++)
        for (int j = 2; j <= nj - 1; j++)
            for (int i = 2; i <= ni - 1; i++) {
                double rhs0 = 0.0, t[3];
                for (int d = 0; d < 3; d++) {
                    int c[3] = {i, j, k};
                    c[d] -= 1;
                    double prim[5], g[4];
                    getprim(b, c[0], c[1], c[2], prim);
                    getrkec(b, c[0], c[1], c[2], d, g);
                    t[d] = sa_mxdq(prim, g, b->dqke[IX(b, c[0], c[1], c[2])], 1);
                }
                rhs0 = t[0] + t[1] + t[2];
                size_t id = IX(b, i, j, k);
                b->dqke[id] = (rhs0 - b->dqke[id]) / b->spec[id];
            }
    for (int k = nk - 1; k >= 2; k--)
        for (int j = nj - 1; j >= 2; j--)
            for (int i = ni - 1; i >= 2; i--) {
                double rhs0, t[3];
                for (int d = 0; d < 3; d++) {
                    int c[3] = {i, j, k};
                    c[d] += 1;
                    double prim[5], g[4];
                    getprim(b, c[0], c[1], c[2], prim);
                    getrkec(b, c[0], c[1], c[2], d, g);
                    t[d] = sa_mxdq(prim, g, b->dqke[IX(b, c[0], c[1], c[2])], -1);
                }
                rhs0 = t[0] + t[1] + t[2];
                size_t id = IX(b, i, j, k);
                b->dqke[id] = b->dqke[id] - rhs0 / b->spec[id];
            }
    /* update_turbulence, turblence.f90:585-623 */
    for (int k = 2; k <= nk - 1; k++)
        for (int j = 2; j <= nj - 1; j++)
            for (int i = 2; i <= ni - 1; i++) {
                size_t id = IX(b, i, j, k);
                double qn = b->qke[id] + b->dqke[id] / R(b)[id], lim = SA_MINLIM * SA_MUOO;
                b->qke[id] = qn > lim ? qn : lim;
            }
    /* cal_vist_SA, turblence.f90:2735-2760, over 1..n */
    for (int k = 1; k <= nk; k++)
        for (int j = 1; j <= nj; j++)
            for (int i = 1; i <= ni; i++) {
                size_t id = IX(b, i, j, k);
                double romu = R(b)[id] * b->qke[id];
                double kafan = romu / f[F_VISL][id];
                double kf3 = pow(kafan, 3.0);
                double fv1 = kf3 / (kf3 + cv13);
                b->vist[id] = romu * fv1;
            }
    /* max_control_turbulence, turblence.f90:625-660, over 0..n (layer 0 of
     * visl is never computed: compute_visl_ns covers 1..n) */
    if (o->kmaxlim > 1.0e-15)
        for (int k = 0; k <= nk; k++)
            for (int j = 0; j <= nj; j++)
                for (int i = 0; i <= ni; i++) {
                    size_t id = IX(b, i, j, k);
                    double lim = o->kmaxlim * f[F_VISL][id];
                    b->vist[id] = b->vist[id] < lim ? b->vist[id] : lim;
                }
}

/* on/off switch of the model's qke/vist BC rules (on from orc_sa_setup);
 * the known-answer test turns them off to see that they are the only change */
int orc_sa_boundary_rules(void *h, int on) {
    ((Orc *)h)->sa_bc = on ? 1 : 0;
    return 0;
}

/* turbulence(nb) for every block (RHS.f90:22 inside r_h_s_vis) */
int orc_turbulence(void *h) {
    Orc *o = h;
    if (!o->sa) { set_err("orc_turbulence: orc_sa_setup was not called"); return 1; }
#pragma omp parallel for schedule(dynamic, 1)
    for (int nb = 1; nb <= o->nb; nb++) sa_block(o, &o->b[nb]);
    return 0;
}

void orc_value_half_node(int n, int ni, const double *q, double *qh) { value_half_node(n, ni, q, qh); }
void orc_flux_dxyz(int nl, int ni, const double *f, double *df) { flux_dxyz(nl, ni, f, df); }
void orc_fluxes(const OrcParams *prm, int nflux, const double *ql, const double *qr, const double *nx4, double *f) {
    Orc o;
    memset(&o, 0, sizeof o);
    o.prm = *prm;
    o.prm.nflux = nflux;
    o.gama = 1.4;
    if (nflux == 0) phys_flux(1.4, ql, nx4[0], nx4[1], nx4[2], nx4[3], f);
    else flux_type(&o, ql, qr, nx4, f);
}
int orc_wcns_line(const OrcParams *prm, int ni, const double *q, const double *nx, double *df) {
    Orc o;
    memset(&o, 0, sizeof o);
    o.prm = *prm;
    o.gama = 1.4;
    return wcns_line(&o, ni, q, nx, df);
}
