/*
 * chan_oracle.c -- CPU restatement of the compressible-channel time-step hot
 * path of theparvezahmad/compChan3Dmpi, used ONLY as test infrastructure.
 *
 *   This file is the checker, never the product.  Only tests/, the smoke()
 *   entry point and bench.py's CPU-baseline / reference legs may load it.
 *   The GPU library (compchan3dmpi_b200/csrc) never links or calls it.
 *
 * What it restates (reference paths are relative to the reference project):
 *   - mesh            v1.9/codes/comdata.f90:70-110        (orc_setup_mesh)
 *   - wall FD coeffs  v1.10/codes/main_v1.9.f90:59-83      (orc_coeffs)
 *   - initSolV        v1.10/codes/main_v1.9.f90:284-313    (orc_upload)
 *   - one RK stage    v1.10/codes/main_v1.9.f90:329-720    (orc_stage)
 *   - blow-up check   v1.10/codes/main_v1.9.f90:729-740    (orc_check)
 *   - wall shear      v1.10/codes/main_v1.9.f90:930-987    (orc_tau_wall)
 *   - plane moments   v1.10/codes/main_v1.9.f90:995-1025   (orc_avg_spatial)
 *   - step driver     v1.10/codes/main_v1.9.f90:320-327, 726-1072
 *
 * Semantics are those of v1.10/codes/main_v1.9.f90 (v1.9 plus the 2-deep
 * ghost layer of `var`) run on ONE MPI rank with periodic x and y:
 *   * arrays carry the reference's index ranges 0..nP+1 in every direction;
 *   * every halo exchange is the reference's single-rank sendrecv with itself,
 *     restricted to the same sub-ranges the MPI datatypes cover (x halos only
 *     for interior j,k; y halos only for interior i,k; z is never exchanged),
 *     so corner ghosts keep whatever the input deck held, exactly as in the
 *     reference;
 *   * arithmetic follows the Fortran source's operator order (left to right,
 *     no reassociation); build with -ffp-contract=off so no FMA is formed.
 *
 * Additions with no reference counterpart (documented per function):
 *   SSP-RK3 stage table, per-wall wall temperature, Prandtl number as a
 *   parameter, "no forcing" switch.  The default parameters reproduce the
 *   reference exactly.
 *
 * Parity pinning: the coefficient block is pinned by the reference's own
 * known-answer output (v1.8_validation/codes/nohupDebug.out:23-26).  No
 * reference field data exists in the project and the Fortran sources cannot
 * be compiled on this image (no Fortran compiler), so field parity of this
 * restatement is otherwise unpinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* parameter vector layout shared with oracle/oracle.py */
enum {
    P_RE = 0, P_MAC, P_DT, P_PR, P_GAMA, P_PEX, P_PEY, P_PEZ,
    P_LX, P_LY, P_TWB, P_TWT, P_ISTAT, P_RK, P_FORCING, P_NPARAM
};

typedef struct {
    int n1, n2, n3;              /* nP(1), nP(2), nP(3) */
    int NI, NJ, NK;              /* n+2 (index range 0..n+1) */
    size_t NP;                   /* NI*NJ*NK */
    double Re, invRe, Mac, dt, PexVal, PeyVal, PezVal, ggM, gama, invPr;
    double Twb, Twt;
    int istat, rk, forcing;
    double dx, dy, dXi, invdx, invdy, invdXi;
    double *x3, *jac, *invJac;   /* 1-based, length n3+1 */
    double dz1, dzN;
    double f1d2c0, f1d2c1, f1d2c2, b1d2c0, b1d2c1, b1d2c2;
    double f2d1c0, f2d1c1, f2d1c2, b2d1c0, b2d1c1, b2d1c2;
    double *solV;                /* [lev 0..1][var 0..4][NP]  lev0=current, lev1=RK base */
    double *var;                 /* [7][NP] rho,u,v,w,E,T,p */
    double *mu, *kt;             /* [NP] */
    double *fD, *gD, *hD;        /* [5][NP] */
    double *F1, *G1, *H1;        /* [5][NP] inviscid F(:,1),G(:,1),H(:,1) */
    double tauL, tauU;
    double *stat1, *stat2, *corr;/* [7][n3], [7][n3], [9][n3] (k fastest, 0-based k) */
    long nstep;
    double time;
    double tstage;       /* time seen by the wall BC during a stage (the step's new time) */
    int blown, blown_ijk[3];
    /* wall-BC variants (see orc_set_wall_bc) */
    int wvel[2], wtherm[2];
    double wTw[2], wdTdz[2], wg[2], wwave[2][4];
    unsigned char *wmask[2];
    double *wuv[2], *wx1[2];
    /* buoyancy body force (orc_set_buoyancy); ri = 0: off */
    double ri, tref;
    /* 1: the v1.9 binary's single-rank reads of var beyond its bounds (orc_set_v19_alias) */
    int v19alias;
} orc_t;

#define ID(o, i, j, k) ((((size_t)(k)) * (o)->NJ + (size_t)(j)) * (o)->NI + (size_t)(i))
#define SOLV(o, lev, m, i, j, k) (o)->solV[((size_t)(lev) * 5 + (size_t)((m) - 1)) * (o)->NP + ID(o, i, j, k)]
#define VAR(o, m, i, j, k) (o)->var[(size_t)((m) - 1) * (o)->NP + ID(o, i, j, k)]
#define MU(o, i, j, k) (o)->mu[ID(o, i, j, k)]
#define KT(o, i, j, k) (o)->kt[ID(o, i, j, k)]
#define FD(o, m, i, j, k) (o)->fD[(size_t)((m) - 1) * (o)->NP + ID(o, i, j, k)]
#define GD(o, m, i, j, k) (o)->gD[(size_t)((m) - 1) * (o)->NP + ID(o, i, j, k)]
#define HD(o, m, i, j, k) (o)->hD[(size_t)((m) - 1) * (o)->NP + ID(o, i, j, k)]
#define FF(o, a, m, i, j, k) (o)->a[(size_t)((m) - 1) * (o)->NP + ID(o, i, j, k)]

/* var(i,j,k,m) as the 4th-order central fluxes read it.  main19fix
 * (v1.10/codes/main_v1.9.f90:44) declares var(0:nP+1,...) and fills the
 * periodic ghosts; v1.9 (v1.9/codes/main_v1.9.f90:38) declares
 * var(nP1,nP2,nP3,7) without ghosts, yet the central branch reads var(i+-2,...)
 * and var(...,j+-2,...) (main_v1.9.f90:348-351, 386-389).  On one rank those
 * reads land, through the column-major layout, on the neighbouring column or
 * plane of the same variable: var(nP1+1,j,k) is var(1,j+1,k), var(0,j,k) is
 * var(nP1,j-1,k), var(i,nP2+1,k) is var(i,1,k+1) and var(i,0,k) is
 * var(i,nP2,k-1).  For interior points (2 <= i <= nP1-1, 2 <= j <= nP2-1,
 * 2 <= k <= nP3-1) every such read stays inside the array. */
static inline double var_c(const orc_t *o, int m, int i, int j, int k)
{
    if (o->v19alias) {
        if (i == o->n1 + 1) { i = 1; j++; }
        else if (i == 0) { i = o->n1; j--; }
        if (j == o->n2 + 1) { j = 1; k++; }
        else if (j == 0) { j = o->n2; k--; }
    }
    return VAR(o, m, i, j, k);
}

static const double haf = 0.5, two = 2.0, zer = 0.0, one = 1.0;
static const double two3rd = 2.0 / 3.0, one12th = 1.0 / 12.0;

/* ------------------------------------------------------------------ mesh */
/* v1.9/codes/comdata.f90:70-110 (cosine wall-normal map).  x1,x2 are only
 * needed for diagnostics; dx/dy come from the caller's periodic lengths. */
void orc_setup_mesh_cosine(int n3, double *x3, double *jac, double *invJac)
{
    const double Pi = 4.0 * atan(1.0);
    double *Xi = (double *)malloc(sizeof(double) * (size_t)(n3 + 1));
    double dXi;
    int k;
    Xi[1] = 0.0;
    dXi = 2.0 / (double)(n3 - 1);
    for (k = 1; k <= n3 - 1; k++) Xi[k + 1] = Xi[k] + dXi;
    for (k = 1; k <= n3; k++) {
        x3[k] = 1.0 - cos(0.50 * Xi[k] * Pi);
        jac[k] = 0.50 * Pi * sin(0.50 * Xi[k] * Pi);
    }
    invJac[1] = 0.0; /* never set by the reference (invJac(2:nP3) only) */
    for (k = 2; k <= n3; k++) invJac[k] = 1.0 / jac[k];
    free(Xi);
}

/* v1.10/codes/main_v1.9.f90:59-83 -- one-sided wall coefficients.
 * out[0..11] = f1d2c0..2, f2d1c0..2, b1d2c0..2, b2d1c0..2 ; out[12..13] = dz1, dzN
 * x3 is 1-based (x3[1..n3]). */
void orc_coeffs(int n3, const double *x3, double *out)
{
    double dz1, dzN, alpha, t;
    dz1 = x3[2] - x3[1];
    alpha = (x3[3] - x3[2]) / dz1;
    t = dz1 * alpha * (alpha + one);
    out[0] = (one - (alpha + one) * (alpha + one)) / t;
    out[1] = ((alpha + one) * (alpha + one)) / t;
    out[2] = -one / t;
    t = haf * (dz1 * dz1) * alpha * (alpha + one);
    out[3] = alpha / t;
    out[4] = -(alpha + one) / t;
    out[5] = one / t;
    dzN = x3[n3] - x3[n3 - 1];
    alpha = (x3[n3 - 1] - x3[n3 - 2]) / dzN;
    t = dzN * alpha * (alpha + one);
    out[6] = ((alpha + one) * (alpha + one) - one) / t;
    out[7] = -((alpha + one) * (alpha + one)) / t;
    out[8] = one / t;
    t = haf * (dzN * dzN) * alpha * (alpha + one);
    out[9] = alpha / t;
    out[10] = -(alpha + one) / t;
    out[11] = one / t;
    out[12] = dz1;
    out[13] = dzN;
}

/* ------------------------------------------------------------ lifecycle */
static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n, s);
    return p;
}

void orc_free(orc_t *o)
{
    if (!o) return;
    free(o->x3); free(o->jac); free(o->invJac);
    free(o->solV); free(o->var); free(o->mu); free(o->kt);
    free(o->fD); free(o->gD); free(o->hD);
    free(o->F1); free(o->G1); free(o->H1);
    free(o->stat1); free(o->stat2); free(o->corr);
    for (int w = 0; w < 2; w++) { free(o->wmask[w]); free(o->wuv[w]); free(o->wx1[w]); }
    free(o);
}

/* nP[3]; prm[P_NPARAM]; x3,jac,invJac are 0-based arrays of length n3
 * (x3[0] is the reference's x3(1)). */
orc_t *orc_create(const int *nP, const double *prm, const double *x3,
                  const double *jac, const double *invJac)
{
    orc_t *o = (orc_t *)xcalloc(1, sizeof(orc_t));
    double c[14];
    int k;
    if (!o) return NULL;
    o->n1 = nP[0]; o->n2 = nP[1]; o->n3 = nP[2];
    if (o->n1 < 6 || o->n2 < 6 || o->n3 < 6) { free(o); return NULL; }
    o->NI = o->n1 + 2; o->NJ = o->n2 + 2; o->NK = o->n3 + 2;
    o->NP = (size_t)o->NI * o->NJ * o->NK;
    o->Re = prm[P_RE]; o->Mac = prm[P_MAC]; o->dt = prm[P_DT];
    o->gama = prm[P_GAMA];
    o->invPr = 1.0 / prm[P_PR];           /* comdata.f90:12 invPr=1/0.71 */
    o->PexVal = prm[P_PEX]; o->PeyVal = prm[P_PEY]; o->PezVal = prm[P_PEZ];
    o->Twb = prm[P_TWB]; o->Twt = prm[P_TWT];
    o->wTw[0] = o->Twb; o->wTw[1] = o->Twt;
    o->istat = (int)prm[P_ISTAT]; o->rk = (int)prm[P_RK]; o->forcing = (int)prm[P_FORCING];
    o->invRe = 1.0 / o->Re;               /* comdata.f90:59 */
    o->ggM = o->gama * (o->gama - 1) * (o->Mac * o->Mac); /* comdata.f90:60 */
    o->dx = prm[P_LX] / (double)(o->n1 - 1); /* comdata.f90:85-87 */
    o->dy = prm[P_LY] / (double)(o->n2 - 1);
    o->dXi = 2.0 / (double)(o->n3 - 1);
    o->invdx = 1.0 / o->dx; o->invdy = 1.0 / o->dy; o->invdXi = 1.0 / o->dXi;
    o->x3 = (double *)xcalloc((size_t)o->n3 + 1, sizeof(double));
    o->jac = (double *)xcalloc((size_t)o->n3 + 1, sizeof(double));
    o->invJac = (double *)xcalloc((size_t)o->n3 + 1, sizeof(double));
    for (k = 1; k <= o->n3; k++) {
        o->x3[k] = x3[k - 1]; o->jac[k] = jac[k - 1]; o->invJac[k] = invJac[k - 1];
    }
    orc_coeffs(o->n3, o->x3, c);
    o->f1d2c0 = c[0]; o->f1d2c1 = c[1]; o->f1d2c2 = c[2];
    o->f2d1c0 = c[3]; o->f2d1c1 = c[4]; o->f2d1c2 = c[5];
    o->b1d2c0 = c[6]; o->b1d2c1 = c[7]; o->b1d2c2 = c[8];
    o->b2d1c0 = c[9]; o->b2d1c1 = c[10]; o->b2d1c2 = c[11];
    o->dz1 = c[12]; o->dzN = c[13];
    o->solV = (double *)xcalloc(2 * 5 * o->NP, sizeof(double));
    o->var = (double *)xcalloc(7 * o->NP, sizeof(double));
    o->mu = (double *)xcalloc(o->NP, sizeof(double));
    o->kt = (double *)xcalloc(o->NP, sizeof(double));
    o->fD = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->gD = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->hD = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->F1 = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->G1 = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->H1 = (double *)xcalloc(5 * o->NP, sizeof(double));
    o->stat1 = (double *)xcalloc((size_t)7 * o->n3, sizeof(double));
    o->stat2 = (double *)xcalloc((size_t)7 * o->n3, sizeof(double));
    o->corr = (double *)xcalloc((size_t)9 * o->n3, sizeof(double));
    if (!o->solV || !o->var || !o->mu || !o->kt || !o->fD || !o->gD || !o->hD ||
        !o->F1 || !o->G1 || !o->H1 || !o->stat1 || !o->stat2 || !o->corr ||
        !o->x3 || !o->jac || !o->invJac) {
        orc_free(o);
        return NULL;
    }
    return o;
}

/* ------------------------------------------------------- halo exchanges */
/* Single-rank periodic sendrecv of main19fix:297-313 / 589-619 for `nv`
 * consecutive variables of array `a` (stride NP), 2 planes deep.  x covers
 * interior j,k only; y covers interior i,k only (the MPI datatypes'
 * sub-ranges); z is never exchanged (walls). */
static void share2P(orc_t *o, double *a, int nv)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    int m, i, j, k;
    for (m = 0; m < nv; m++) {
        double *b = a + (size_t)m * o->NP;
        for (k = 2; k <= n3 - 1; k++)
            for (j = 2; j <= n2 - 1; j++) {
                b[ID(o, 0, j, k)] = b[ID(o, n1 - 2, j, k)];
                b[ID(o, 1, j, k)] = b[ID(o, n1 - 1, j, k)];
                b[ID(o, n1, j, k)] = b[ID(o, 2, j, k)];
                b[ID(o, n1 + 1, j, k)] = b[ID(o, 3, j, k)];
            }
        for (k = 2; k <= n3 - 1; k++)
            for (i = 2; i <= n1 - 1; i++) {
                b[ID(o, i, 0, k)] = b[ID(o, i, n2 - 2, k)];
                b[ID(o, i, 1, k)] = b[ID(o, i, n2 - 1, k)];
                b[ID(o, i, n2, k)] = b[ID(o, i, 2, k)];
                b[ID(o, i, n2 + 1, k)] = b[ID(o, i, 3, k)];
            }
    }
}

/* 1-plane exchanges of fD along x and gD along y (main19fix:543-550);
 * hD along z is a no-op on one rank. */
static void share_flux(orc_t *o)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    int m, i, j, k;
    for (m = 1; m <= 5; m++) {
        for (k = 2; k <= n3 - 1; k++)
            for (j = 2; j <= n2 - 1; j++) {
                FD(o, m, 1, j, k) = FD(o, m, n1 - 1, j, k);
                FD(o, m, n1, j, k) = FD(o, m, 2, j, k);
            }
        for (k = 2; k <= n3 - 1; k++)
            for (i = 2; i <= n1 - 1; i++) {
                GD(o, m, i, 1, k) = GD(o, m, i, n2 - 1, k);
                GD(o, m, i, n2, k) = GD(o, m, i, 2, k);
            }
    }
}

/* --------------------------------------------------------------- upload */
/* Input deck -> state.  `v` is the reference's var(1:nP1,1:nP2,1:nP3,1:7) in
 * Fortran (column-major) order.  main19fix:233-313. */
void orc_upload(orc_t *o, const double *v, long nstep, double time)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    int i, j, k, m;
    memset(o->var, 0, sizeof(double) * 7 * o->NP);
    memset(o->solV, 0, sizeof(double) * 10 * o->NP);
    for (m = 1; m <= 7; m++)
        for (k = 1; k <= n3; k++)
            for (j = 1; j <= n2; j++)
                for (i = 1; i <= n1; i++)
                    VAR(o, m, i, j, k) = v[(((size_t)(m - 1) * n3 + (k - 1)) * n2 + (j - 1)) * n1 + (i - 1)];
    /* initSolV, main19fix:284-294 */
    for (k = 1; k <= n3; k++)
        for (j = 1; j <= n2; j++)
            for (i = 1; i <= n1; i++) {
                SOLV(o, 0, 1, i, j, k) = VAR(o, 1, i, j, k);
                for (m = 2; m <= 5; m++) SOLV(o, 0, m, i, j, k) = VAR(o, 1, i, j, k) * VAR(o, m, i, j, k);
                MU(o, i, j, k) = pow(VAR(o, 6, i, j, k), 0.7);
                KT(o, i, j, k) = pow(VAR(o, 6, i, j, k), 0.7);
            }
    share2P(o, o->solV, 5);
    share2P(o, o->var, 7);
    o->nstep = nstep;
    o->time = time;
    o->tstage = time + o->dt;
    o->tauL = 0.0; o->tauU = 0.0;       /* never set before the first stats step */
    memset(o->stat1, 0, sizeof(double) * 7 * n3);
    o->blown = 0;
}

/* Forcing state (the lagged wall shear and plane-mean density) */
/* on = 1: the canonical v1.9 binary's aliased var reads (var_c above);
 * on = 0 (default): main19fix's true periodic ghosts */
void orc_set_v19_alias(orc_t *o, int on) { o->v19alias = on ? 1 : 0; }

void orc_set_buoyancy(orc_t *o, double ri, double tref)
{
    o->ri = ri;
    o->tref = tref;
}

void orc_set_forcing(orc_t *o, double tauL, double tauU, const double *rhobar)
{
    int k;
    o->tauL = tauL; o->tauU = tauU;
    for (k = 0; k < o->n3; k++) o->stat1[k] = rhobar[k];
}

/* ----------------------------------------------------------- one stage */
/* QUICK face-upwinded flux along one direction: the four sign branches of
 * main19fix:335-361 (x), :373-399 (y), :415-442 (z).  q(o) is the conservative
 * variable at offset o along the direction; scale multiplies the bracket
 * exactly as the reference does ( (...)*invdx/8.0d0 -> (b*s1)/8 ). */
static inline double quick(double tmpR1, double tmpR2, double qm2, double qm1,
                           double q0, double qp1, double qp2)
{
    double r = 0.0;
    if (tmpR1 >= 0.0 && tmpR2 >= 0.0)
        r = tmpR1 * (6.0 * q0 + 3.0 * qp1 - 1.0 * qm1) - tmpR2 * (6.0 * qm1 + 3.0 * q0 - 1.0 * qm2);
    if (tmpR1 < 0.0 && tmpR2 < 0.0)
        r = tmpR1 * (6.0 * qp1 + 3.0 * q0 - 1.0 * qp2) - tmpR2 * (6.0 * q0 + 3.0 * qm1 - 1.0 * qp1);
    if (tmpR1 < 0.0 && tmpR2 >= 0.0)
        r = tmpR1 * (6.0 * qp1 + 3.0 * q0 - 1.0 * qp2) - tmpR2 * (6.0 * qm1 + 3.0 * q0 - 1.0 * qm2);
    if (tmpR1 >= 0.0 && tmpR2 < 0.0)
        r = tmpR1 * (6.0 * q0 + 3.0 * qp1 - 1.0 * qm1) - tmpR2 * (6.0 * q0 + 3.0 * qm1 - 1.0 * qp1);
    return r;
}

/* RK stage coefficients Q <- a*Qbase + b*Q + c*dt*R.
 * rk==2 : the reference's midpoint scheme (maxiter=2, main19fix:575-582).
 * rk==3 : SSP-RK3 (Shu-Osher form); no reference counterpart. */
static void rk_coef(int rk, int iter, double *a, double *b, double *c)
{
    if (rk == 3) {
        if (iter == 1) { *a = 0.0; *b = 1.0; *c = 1.0; }
        else if (iter == 2) { *a = 0.75; *b = 0.25; *c = 0.25; }
        else { *a = 1.0 / 3.0; *b = 2.0 / 3.0; *c = 2.0 / 3.0; }
    } else {
        if (iter == 1) { *a = 0.0; *b = 1.0; *c = 0.5; }
        else { *a = 1.0; *b = 0.0; *c = 1.0; }
    }
}

void orc_stage(orc_t *o, int iter)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    const double Re = o->Re, invRe = o->invRe, dx = o->dx, dy = o->dy, dXi = o->dXi;
    const double invdx = o->invdx, invdy = o->invdy, invdXi = o->invdXi;
    const double ggM = o->ggM, gama = o->gama, invPr = o->invPr, Mac = o->Mac;
    int k;

    /* ---- inviscid F(:,1), G(:,1), H(:,1): main19fix:329-454 */
#pragma omp parallel for schedule(static)
    for (k = 2; k <= n3 - 1; k++) {
        int i, j, m;
        double Pe, tmpR1, tmpR2;
        for (j = 2; j <= n2 - 1; j++)
            for (i = 2; i <= n1 - 1; i++) {
                Pe = Re * fabs(SOLV(o, 0, 2, i, j, k)) * dx / MU(o, i, j, k);
                if (Pe > o->PexVal) {
                    tmpR1 = (VAR(o, 2, i, j, k) + VAR(o, 2, i + 1, j, k)) * haf;
                    tmpR2 = (VAR(o, 2, i, j, k) + VAR(o, 2, i - 1, j, k)) * haf;
                    for (m = 1; m <= 5; m++)
                        FF(o, F1, m, i, j, k) = quick(tmpR1, tmpR2,
                            SOLV(o, 0, m, i - 2, j, k), SOLV(o, 0, m, i - 1, j, k), SOLV(o, 0, m, i, j, k),
                            SOLV(o, 0, m, i + 1, j, k), SOLV(o, 0, m, i + 2, j, k)) * invdx / 8.0;
                } else {
                    for (m = 1; m <= 5; m++)
                        FF(o, F1, m, i, j, k) =
                            (-(var_c(o, 2, i + 2, j, k) * SOLV(o, 0, m, i + 2, j, k))
                             + 8.0 * VAR(o, 2, i + 1, j, k) * SOLV(o, 0, m, i + 1, j, k)
                             - 8.0 * VAR(o, 2, i - 1, j, k) * SOLV(o, 0, m, i - 1, j, k)
                             + var_c(o, 2, i - 2, j, k) * SOLV(o, 0, m, i - 2, j, k)) * invdx * one12th;
                }
                Pe = Re * fabs(SOLV(o, 0, 3, i, j, k)) * dy / MU(o, i, j, k);
                if (Pe > o->PeyVal) {
                    tmpR1 = (VAR(o, 3, i, j, k) + VAR(o, 3, i, j + 1, k)) * haf;
                    tmpR2 = (VAR(o, 3, i, j, k) + VAR(o, 3, i, j - 1, k)) * haf;
                    for (m = 1; m <= 5; m++)
                        FF(o, G1, m, i, j, k) = quick(tmpR1, tmpR2,
                            SOLV(o, 0, m, i, j - 2, k), SOLV(o, 0, m, i, j - 1, k), SOLV(o, 0, m, i, j, k),
                            SOLV(o, 0, m, i, j + 1, k), SOLV(o, 0, m, i, j + 2, k)) * invdy / 8.0;
                } else {
                    for (m = 1; m <= 5; m++)
                        FF(o, G1, m, i, j, k) =
                            (-(var_c(o, 3, i, j + 2, k) * SOLV(o, 0, m, i, j + 2, k))
                             + 8.0 * VAR(o, 3, i, j + 1, k) * SOLV(o, 0, m, i, j + 1, k)
                             - 8.0 * VAR(o, 3, i, j - 1, k) * SOLV(o, 0, m, i, j - 1, k)
                             + var_c(o, 3, i, j - 2, k) * SOLV(o, 0, m, i, j - 2, k)) * invdy * one12th;
                }
                Pe = Re * fabs(SOLV(o, 0, 4, i, j, k)) * dXi * o->jac[k] / MU(o, i, j, k);
                if (k < 3 || k > n3 - 2) {
                    for (m = 1; m <= 5; m++)
                        FF(o, H1, m, i, j, k) =
                            (VAR(o, 4, i, j, k + 1) * SOLV(o, 0, m, i, j, k + 1)
                             - VAR(o, 4, i, j, k - 1) * SOLV(o, 0, m, i, j, k - 1)) * invdXi * o->invJac[k] * haf;
                } else if (Pe > o->PezVal) {
                    tmpR1 = (VAR(o, 4, i, j, k) + VAR(o, 4, i, j, k + 1)) * haf;
                    tmpR2 = (VAR(o, 4, i, j, k) + VAR(o, 4, i, j, k - 1)) * haf;
                    for (m = 1; m <= 5; m++)
                        FF(o, H1, m, i, j, k) = quick(tmpR1, tmpR2,
                            SOLV(o, 0, m, i, j, k - 2), SOLV(o, 0, m, i, j, k - 1), SOLV(o, 0, m, i, j, k),
                            SOLV(o, 0, m, i, j, k + 1), SOLV(o, 0, m, i, j, k + 2)) * invdXi * o->invJac[k] / 8.0;
                } else {
                    for (m = 1; m <= 5; m++)
                        FF(o, H1, m, i, j, k) =
                            (-(VAR(o, 4, i, j, k + 2) * SOLV(o, 0, m, i, j, k + 2))
                             + 8.0 * VAR(o, 4, i, j, k + 1) * SOLV(o, 0, m, i, j, k + 1)
                             - 8.0 * VAR(o, 4, i, j, k - 1) * SOLV(o, 0, m, i, j, k - 1)
                             + VAR(o, 4, i, j, k - 2) * SOLV(o, 0, m, i, j, k - 2)) * invdXi * o->invJac[k] * one12th;
                }
            }
    }

    /* ---- viscous / pressure flux vectors fD,gD,hD: main19fix:457-538 */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3; k++) {
        int i, j;
        double Ut, Vt, Wt, dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz;
        double dTdx, dTdy, dTdz, divg, muT, ktT, PressT, dissF, dissG, dissH;
        for (j = 2; j <= n2 - 1; j++)
            for (i = 2; i <= n1 - 1; i++) {
                Ut = VAR(o, 2, i, j, k);
                Vt = VAR(o, 3, i, j, k);
                Wt = VAR(o, 4, i, j, k);
                dudx = (VAR(o, 2, i + 1, j, k) - VAR(o, 2, i - 1, j, k)) * haf * invdx;
                dudy = (VAR(o, 2, i, j + 1, k) - VAR(o, 2, i, j - 1, k)) * haf * invdy;
                dvdx = (VAR(o, 3, i + 1, j, k) - VAR(o, 3, i - 1, j, k)) * haf * invdx;
                dvdy = (VAR(o, 3, i, j + 1, k) - VAR(o, 3, i, j - 1, k)) * haf * invdy;
                dwdx = (VAR(o, 4, i + 1, j, k) - VAR(o, 4, i - 1, j, k)) * haf * invdx;
                dwdy = (VAR(o, 4, i, j + 1, k) - VAR(o, 4, i, j - 1, k)) * haf * invdy;
                dTdx = (VAR(o, 6, i + 1, j, k) - VAR(o, 6, i - 1, j, k)) * haf * invdx;
                dTdy = (VAR(o, 6, i, j + 1, k) - VAR(o, 6, i, j - 1, k)) * haf * invdy;
                if (k == 1) {
                    dudz = (VAR(o, 2, i, j, 2) - VAR(o, 2, i, j, 1)) / o->dz1;
                    dvdz = (VAR(o, 3, i, j, 2) - VAR(o, 3, i, j, 1)) / o->dz1;
                    dwdz = (VAR(o, 4, i, j, 2) - VAR(o, 4, i, j, 1)) / o->dz1;
                    dTdz = (VAR(o, 6, i, j, 2) - VAR(o, 6, i, j, 1)) / o->dz1;
                } else if (k == n3) {
                    dudz = (VAR(o, 2, i, j, n3) - VAR(o, 2, i, j, n3 - 1)) / o->dzN;
                    dvdz = (VAR(o, 3, i, j, n3) - VAR(o, 3, i, j, n3 - 1)) / o->dzN;
                    dwdz = (VAR(o, 4, i, j, n3) - VAR(o, 4, i, j, n3 - 1)) / o->dzN;
                    dTdz = (VAR(o, 6, i, j, n3) - VAR(o, 6, i, j, n3 - 1)) / o->dzN;
                } else {
                    dudz = (VAR(o, 2, i, j, k + 1) - VAR(o, 2, i, j, k - 1)) * haf * invdXi * o->invJac[k];
                    dvdz = (VAR(o, 3, i, j, k + 1) - VAR(o, 3, i, j, k - 1)) * haf * invdXi * o->invJac[k];
                    dwdz = (VAR(o, 4, i, j, k + 1) - VAR(o, 4, i, j, k - 1)) * haf * invdXi * o->invJac[k];
                    dTdz = (VAR(o, 6, i, j, k + 1) - VAR(o, 6, i, j, k - 1)) * haf * invdXi * o->invJac[k];
                }
                divg = dudx + dvdy + dwdz;
                muT = MU(o, i, j, k);
                ktT = KT(o, i, j, k);
                PressT = VAR(o, 7, i, j, k);
                dissF = ggM * invRe * (two3rd * muT * Ut * divg - two * muT * Ut * dudx
                                       - muT * Vt * (dvdx + dudy) - muT * Wt * (dwdx + dudz));
                dissG = ggM * invRe * (-(muT * Ut * (dvdx + dudy)) + two3rd * muT * Vt * divg
                                       - two * muT * Vt * dvdy - muT * Wt * (dwdy + dvdz));
                dissH = ggM * invRe * (-(muT * Ut * (dwdx + dudz)) - muT * Vt * (dwdy + dvdz)
                                       + two3rd * muT * Wt * divg - two * muT * Wt * dwdz);
                FD(o, 1, i, j, k) = zer;
                FD(o, 2, i, j, k) = PressT + two3rd * muT * invRe * divg - two * muT * invRe * dudx;
                FD(o, 3, i, j, k) = -(muT * invRe * (dvdx + dudy));
                FD(o, 4, i, j, k) = -(muT * invRe * (dwdx + dudz));
                FD(o, 5, i, j, k) = -(gama * ktT * invRe * invPr * dTdx) + ggM * Ut * PressT + dissF;
                GD(o, 1, i, j, k) = zer;
                GD(o, 2, i, j, k) = -(muT * invRe * (dvdx + dudy));
                GD(o, 3, i, j, k) = PressT + two3rd * muT * invRe * divg - two * muT * invRe * dvdy;
                GD(o, 4, i, j, k) = -(muT * invRe * (dwdy + dvdz));
                GD(o, 5, i, j, k) = -(gama * ktT * invRe * invPr * dTdy) + ggM * Vt * PressT + dissG;
                HD(o, 1, i, j, k) = zer;
                HD(o, 2, i, j, k) = -(muT * invRe * (dwdx + dudz));
                HD(o, 3, i, j, k) = -(muT * invRe * (dwdy + dvdz));
                HD(o, 4, i, j, k) = PressT + two3rd * muT * invRe * divg - two * muT * invRe * dwdz;
                HD(o, 5, i, j, k) = -(gama * ktT * invRe * invPr * dTdz) + ggM * Wt * PressT + dissH;
            }
    }
    share_flux(o);

    /* ---- F(:,2),G(:,2),H(:,2), source, R, RK update: main19fix:553-586 */
    {
        double a, b, c, cdt;
        const double fcoef = haf * (o->tauL - o->tauU);
        const int force = (o->forcing == 0);
        rk_coef(o->rk, iter, &a, &b, &c);
        cdt = c * o->dt;   /* haf*dt for the reference's first stage */
#pragma omp parallel for schedule(static)
        for (k = 2; k <= n3 - 1; k++) {
            int i, j, m;
            double F2, G2, H2, src[6], R;
            for (j = 2; j <= n2 - 1; j++)
                for (i = 2; i <= n1 - 1; i++) {
                    src[1] = zer;
                    src[2] = force ? fcoef * o->stat1[k - 1] : zer;
                    src[3] = zer; src[4] = zer;
                    src[5] = force ? ggM * VAR(o, 2, i, j, k) * haf * (o->tauL - o->tauU) * o->stat1[k - 1] : zer;
                    if (o->ri != zer) {
                        /* buoyancy ri*rho*(T - tref) on rho*w (w wall-normal, gravity along -x3)
                         * and its work ggM*w*(that) on rho*E; no reference counterpart */
                        const double bq = o->ri * (VAR(o, 1, i, j, k) * (VAR(o, 6, i, j, k) - o->tref));
                        src[4] = bq;
                        src[5] = src[5] + (ggM * VAR(o, 4, i, j, k)) * bq;
                    }
                    for (m = 1; m <= 5; m++) {
                        F2 = (FD(o, m, i + 1, j, k) - FD(o, m, i - 1, j, k)) * haf * invdx;
                        G2 = (GD(o, m, i, j + 1, k) - GD(o, m, i, j - 1, k)) * haf * invdy;
                        H2 = (HD(o, m, i, j, k + 1) - HD(o, m, i, j, k - 1)) * haf * invdXi * o->invJac[k];
                        R = src[m] - (FF(o, F1, m, i, j, k) + F2 + FF(o, G1, m, i, j, k) + G2
                                      + FF(o, H1, m, i, j, k) + H2);
                        if (iter == 1) {
                            SOLV(o, 1, m, i, j, k) = SOLV(o, 0, m, i, j, k);
                            SOLV(o, 0, m, i, j, k) = SOLV(o, 0, m, i, j, k) + cdt * R;
                        } else if (a == 1.0 && b == 0.0) {
                            SOLV(o, 0, m, i, j, k) = SOLV(o, 1, m, i, j, k) + cdt * R;
                        } else {
                            SOLV(o, 0, m, i, j, k) = a * SOLV(o, 1, m, i, j, k) + b * SOLV(o, 0, m, i, j, k) + cdt * R;
                        }
                    }
                }
        }
    }
    share2P(o, o->solV, 5);

    /* ---- primitives: main19fix:600-609 */
#pragma omp parallel for schedule(static)
    for (k = 2; k <= n3 - 1; k++) {
        int i, j, m;
        for (j = 2; j <= n2 - 1; j++)
            for (i = 2; i <= n1 - 1; i++) {
                double u2, v2, w2;
                VAR(o, 1, i, j, k) = SOLV(o, 0, 1, i, j, k);
                for (m = 2; m <= 5; m++) VAR(o, m, i, j, k) = SOLV(o, 0, m, i, j, k) / SOLV(o, 0, 1, i, j, k);
                u2 = VAR(o, 2, i, j, k) * VAR(o, 2, i, j, k);
                v2 = VAR(o, 3, i, j, k) * VAR(o, 3, i, j, k);
                w2 = VAR(o, 4, i, j, k) * VAR(o, 4, i, j, k);
                VAR(o, 6, i, j, k) = VAR(o, 5, i, j, k) - ggM * haf * (u2 + v2 + w2);
                VAR(o, 7, i, j, k) = VAR(o, 1, i, j, k) * VAR(o, 6, i, j, k) / (gama * (Mac * Mac));
            }
    }
    share2P(o, o->var, 7);

    /* ---- wall boundary conditions: main19fix:623-641, with the wall-BC
     * variants of v1.9_strat (st1-st4: T_w, fixed dT/dz), v1.9_groov and
     * v1.9_groov_strat (slip stripes), v1.9_STWNV (s1-s6: travelling wave v_w)
     * and v1.9_RD (rd1-rd3: prescribed disc velocity), lines ~605-640 there. */
    {
        int i, j;
        for (j = 1; j <= n2; j++)
            for (i = 1; i <= n1; i++) {
                int kw;
                for (kw = 0; kw < 2; kw++) {
                    const int kk = kw == 0 ? 1 : n3, k2 = kw == 0 ? 2 : n3 - 1, k3 = kw == 0 ? 3 : n3 - 2;
                    const double c0 = kw == 0 ? o->f1d2c0 : o->b1d2c0, c1 = kw == 0 ? o->f1d2c1 : o->b1d2c1;
                    const double c2 = kw == 0 ? o->f1d2c2 : o->b1d2c2;
                    const size_t pi = (size_t)(j - 1) * n1 + (i - 1);
                    double s;
                    VAR(o, 2, i, j, kk) = 0.0; VAR(o, 3, i, j, kk) = 0.0; VAR(o, 4, i, j, kk) = 0.0;
                    if (o->wvel[kw] == 1 && o->wmask[kw][pi]) {
                        VAR(o, 2, i, j, kk) = (o->wg[kw] - c1 * VAR(o, 2, i, j, k2) - c2 * VAR(o, 2, i, j, k3)) / c0;
                        VAR(o, 3, i, j, kk) = (o->wg[kw] - c1 * VAR(o, 3, i, j, k2) - c2 * VAR(o, 3, i, j, k3)) / c0;
                    } else if (o->wvel[kw] == 2) {
                        VAR(o, 2, i, j, kk) = o->wuv[kw][pi];
                        VAR(o, 3, i, j, kk) = o->wuv[kw][(size_t)n1 * n2 + pi];
                    } else if (o->wvel[kw] == 3) {
                        VAR(o, 3, i, j, kk) = o->wwave[kw][0] *
                            sin(o->wwave[kw][1] * o->wx1[kw][i - 1] + o->wwave[kw][2] * o->tstage + ((j & 1) ? o->wwave[kw][3] : 0.0));
                    }
                    if (o->wtherm[kw] == 1)
                        VAR(o, 6, i, j, kk) = (o->wdTdz[kw] - c1 * VAR(o, 6, i, j, k2) - c2 * VAR(o, 6, i, j, k3)) / c0;
                    else
                        VAR(o, 6, i, j, kk) = o->wTw[kw];
                    s = VAR(o, 2, i, j, kk) * VAR(o, 2, i, j, kk) + VAR(o, 3, i, j, kk) * VAR(o, 3, i, j, kk)
                        + VAR(o, 4, i, j, kk) * VAR(o, 4, i, j, kk);
                    VAR(o, 5, i, j, kk) = VAR(o, 6, i, j, kk) + ggM * haf * s;
                    VAR(o, 1, i, j, kk) = gama * (Mac * Mac) * VAR(o, 7, i, j, kk) / VAR(o, 6, i, j, kk);
                }
            }
    }
    /* mu over bn-1:en+1 = 1..nP in x,y and all k: main19fix:643 */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3; k++) {
        int i, j;
        for (j = 1; j <= n2; j++)
            for (i = 1; i <= n1; i++) MU(o, i, j, k) = pow(VAR(o, 6, i, j, k), 0.7);
    }
    /* ---- wall pressure BC: main19fix:645-719 */
    {
        int i, j;
        const double c0 = o->f1d2c0, c1 = o->f1d2c1, c2 = o->f1d2c2;
        const double e0 = o->f2d1c0, e1 = o->f2d1c1, e2 = o->f2d1c2;
        const double b0 = o->b1d2c0, b1 = o->b1d2c1, b2 = o->b1d2c2;
        const double g0 = o->b2d1c0, g1 = o->b2d1c1, g2 = o->b2d1c2;
        for (j = 2; j <= n2 - 1; j++)
            for (i = 2; i <= n1 - 1; i++) {
                double dudxdz, dvdydz, d2wdz2, drhow2dz, lhs;
                const int N = n3;
                /* bottom */
                dudxdz = ((c0 * MU(o, i + 1, j, 1) * VAR(o, 2, i + 1, j, 1)
                           + c1 * MU(o, i + 1, j, 2) * VAR(o, 2, i + 1, j, 2)
                           + c2 * MU(o, i + 1, j, 3) * VAR(o, 2, i + 1, j, 3))
                          - (c0 * MU(o, i - 1, j, 1) * VAR(o, 2, i - 1, j, 1)
                             + c1 * MU(o, i - 1, j, 2) * VAR(o, 2, i - 1, j, 2)
                             + c2 * MU(o, i - 1, j, 3) * VAR(o, 2, i - 1, j, 3))) * haf * invdx;
                dvdydz = ((c0 * MU(o, i, j + 1, 1) * VAR(o, 3, i, j + 1, 1)
                           + c1 * MU(o, i, j + 1, 2) * VAR(o, 3, i, j + 1, 2)
                           + c2 * MU(o, i, j + 1, 3) * VAR(o, 3, i, j + 1, 3))
                          - (c0 * MU(o, i, j - 1, 1) * VAR(o, 3, i, j - 1, 1)
                             + c1 * MU(o, i, j - 1, 2) * VAR(o, 3, i, j - 1, 2)
                             + c2 * MU(o, i, j - 1, 3) * VAR(o, 3, i, j - 1, 3))) * haf * invdy;
                d2wdz2 = e0 * MU(o, i, j, 1) * VAR(o, 4, i, j, 1)
                         + e1 * MU(o, i, j, 2) * VAR(o, 4, i, j, 2)
                         + e2 * MU(o, i, j, 3) * VAR(o, 4, i, j, 3);
                drhow2dz = c0 * VAR(o, 1, i, j, 1) * (VAR(o, 4, i, j, 1) * VAR(o, 4, i, j, 1))
                           + c1 * VAR(o, 1, i, j, 2) * (VAR(o, 4, i, j, 2) * VAR(o, 4, i, j, 2))
                           + c2 * VAR(o, 1, i, j, 3) * (VAR(o, 4, i, j, 3) * VAR(o, 4, i, j, 3));
                lhs = invRe * (-dudxdz - dvdydz + two3rd * (dudxdz + dvdydz - two * d2wdz2)) + drhow2dz;
                VAR(o, 7, i, j, 1) = -(lhs + c1 * VAR(o, 7, i, j, 2) + c2 * VAR(o, 7, i, j, 3)) / c0;
                /* top */
                dudxdz = ((b0 * MU(o, i + 1, j, N) * VAR(o, 2, i + 1, j, N)
                           + b1 * MU(o, i + 1, j, N - 1) * VAR(o, 2, i + 1, j, N - 1)
                           + b2 * MU(o, i + 1, j, N - 2) * VAR(o, 2, i + 1, j, N - 2))
                          - (b0 * MU(o, i - 1, j, N) * VAR(o, 2, i - 1, j, N)
                             + b1 * MU(o, i - 1, j, N - 1) * VAR(o, 2, i - 1, j, N - 1)
                             + b2 * MU(o, i - 1, j, N - 2) * VAR(o, 2, i - 1, j, N - 2))) * haf * invdx;
                dvdydz = ((b0 * MU(o, i, j + 1, N) * VAR(o, 3, i, j + 1, N)
                           + b1 * MU(o, i, j + 1, N - 1) * VAR(o, 3, i, j + 1, N - 1)
                           + b2 * MU(o, i, j + 1, N - 2) * VAR(o, 3, i, j + 1, N - 2))
                          - (b0 * MU(o, i, j - 1, N) * VAR(o, 3, i, j - 1, N)
                             + b1 * MU(o, i, j - 1, N - 1) * VAR(o, 3, i, j - 1, N - 1)
                             + b2 * MU(o, i, j - 1, N - 2) * VAR(o, 3, i, j - 1, N - 2))) * haf * invdy;
                d2wdz2 = g0 * MU(o, i, j, N) * VAR(o, 4, i, j, N)
                         + g1 * MU(o, i, j, N - 1) * VAR(o, 4, i, j, N - 1)
                         + g2 * MU(o, i, j, N - 2) * VAR(o, 4, i, j, N - 2);
                drhow2dz = b0 * VAR(o, 1, i, j, N) * (VAR(o, 4, i, j, N) * VAR(o, 4, i, j, N))
                           + b1 * VAR(o, 1, i, j, N - 1) * (VAR(o, 4, i, j, N - 1) * VAR(o, 4, i, j, N - 1))
                           + b2 * VAR(o, 1, i, j, N - 2) * (VAR(o, 4, i, j, N - 2) * VAR(o, 4, i, j, N - 2));
                lhs = invRe * (-dudxdz - dvdydz + two3rd * (dudxdz + dvdydz - two * d2wdz2)) + drhow2dz;
                VAR(o, 7, i, j, N) = -(lhs + b1 * VAR(o, 7, i, j, N - 1) + b2 * VAR(o, 7, i, j, N - 2)) / b0;
            }
    }
    /* kt over all points: main19fix:720 */
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3; k++) {
        int i, j;
        for (j = 1; j <= n2; j++)
            for (i = 1; i <= n1; i++) KT(o, i, j, k) = pow(VAR(o, 6, i, j, k), 0.7);
    }
}

/* ------------------------------------------------------ per-step tail */
/* main19fix:729-740: returns 1 and records the first (i,j,k) if rho<0 or T<0 */
int orc_check(orc_t *o)
{
    int i, j, k;
    for (k = 1; k <= o->n3; k++)
        for (j = 1; j <= o->n2; j++)
            for (i = 1; i <= o->n1; i++)
                if (VAR(o, 1, i, j, k) < 0.0 || VAR(o, 6, i, j, k) < 0.0) {
                    if (!o->blown) {
                        o->blown_ijk[0] = i; o->blown_ijk[1] = j; o->blown_ijk[2] = k;
                    }
                    o->blown = 1;
                }
    return o->blown;
}

/* main19fix:930-977 (one rank: Reduce+Bcast are identities) */
void orc_tau_wall(orc_t *o)
{
    const int n1 = o->n1, n2 = o->n2, N = o->n3;
    int i, j;
    double t, dwdx, dudz;
    t = 0.0;
    for (j = 2; j <= n2 - 1; j++)
        for (i = 2; i <= n1 - 1; i++) {
            dwdx = MU(o, i, j, 1) * (VAR(o, 4, i + 1, j, 1) - VAR(o, 4, i - 1, j, 1)) * haf * o->invdx;
            dudz = MU(o, i, j, 1) * (o->f1d2c0 * VAR(o, 2, i, j, 1) + o->f1d2c1 * VAR(o, 2, i, j, 2)
                                     + o->f1d2c2 * VAR(o, 2, i, j, 3));
            t = t + (dwdx + dudz) * o->invRe;
        }
    o->tauL = t / (double)((n1 - 2) * (n2 - 2));
    t = 0.0;
    for (j = 2; j <= n2 - 1; j++)
        for (i = 2; i <= n1 - 1; i++) {
            dwdx = MU(o, i, j, N) * (VAR(o, 4, i + 1, j, N) - VAR(o, 4, i - 1, j, N)) * haf * o->invdx;
            dudz = MU(o, i, j, N) * (o->b1d2c0 * VAR(o, 2, i, j, N) + o->b1d2c1 * VAR(o, 2, i, j, N - 1)
                                     + o->b1d2c2 * VAR(o, 2, i, j, N - 2));
            t = t + (dwdx + dudz) * o->invRe;
        }
    o->tauU = t / (double)((n1 - 2) * (n2 - 2));
}

/* main19fix:995-1025: plane moments over i=1..nP1, j=1..nP2 (duplicate
 * points included), summed in column-major order then divided by nXY. */
void orc_avg_spatial(orc_t *o)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    const double nXY = (double)(n1 * n2);
    int k;
    static const int cp[9][2] = {{1, 4}, {1, 6}, {2, 3}, {2, 4}, {3, 4}, {3, 6}, {6, 4}, {7, 4}, {7, 6}};
#pragma omp parallel for schedule(static)
    for (k = 1; k <= n3; k++) {
        int i, j, p, c;
        for (p = 1; p <= 7; p++) {
            double s1 = 0.0, s2 = 0.0;
            for (j = 1; j <= n2; j++)
                for (i = 1; i <= n1; i++) {
                    double x = VAR(o, p, i, j, k);
                    s1 = s1 + x;
                    s2 = s2 + x * x;
                }
            o->stat1[(size_t)(p - 1) * n3 + (k - 1)] = s1 / nXY;
            o->stat2[(size_t)(p - 1) * n3 + (k - 1)] = s2 / nXY;
        }
        for (c = 0; c < 9; c++) {
            double s = 0.0;
            for (j = 1; j <= n2; j++)
                for (i = 1; i <= n1; i++)
                    s = s + VAR(o, cp[c][0], i, j, k) * VAR(o, cp[c][1], i, j, k);
            o->corr[(size_t)c * n3 + (k - 1)] = s / nXY;
        }
    }
}

/* One full time step: main19fix:320-327 (counter, time), the stage loop,
 * then the tail in the reference's order (check, tau, stats).  Returns the
 * blow-up flag. */
int orc_step(orc_t *o, int nsteps)
{
    int s, iter, nstage = (o->rk == 3) ? 3 : 2;
    for (s = 0; s < nsteps; s++) {
        o->nstep = o->nstep + 1;
        o->time = o->time + o->dt;
        o->tstage = o->time;
        for (iter = 1; iter <= nstage; iter++) orc_stage(o, iter);
        o->tstage = o->time + o->dt;   /* a stage run alone belongs to the next step */
        if (orc_check(o)) return 1;
        if (o->istat > 0 && o->nstep % o->istat == 0) {
            orc_tau_wall(o);
            orc_avg_spatial(o);
        }
    }
    return 0;
}

/* Wall-BC variant of wall w (0 bottom, 1 top).  vel: 0 no-slip, 1 slip mask
 * (c0*u1+c1*u2+c2*u3 = g), 2 prescribed uv field, 3 travelling wave
 * v = A sin(k x1 + om t + ph*(j odd)); therm: 0 isothermal Tw, 1 fixed dT/dz.
 * mask/uv are nP1*nP2 (i fastest), uv holds u then v; x1 has nP1 values. */
void orc_set_wall_bc(orc_t *o, int w, int vel, int therm, double Tw, double dTdz, double g, const double *wave,
                     const unsigned char *mask, const double *uv, const double *x1)
{
    const size_t n12 = (size_t)o->n1 * o->n2;
    o->wvel[w] = vel; o->wtherm[w] = therm; o->wTw[w] = Tw; o->wdTdz[w] = dTdz; o->wg[w] = g;
    for (int m = 0; m < 4; m++) o->wwave[w][m] = wave ? wave[m] : 0.0;
    if (!o->wmask[w]) {
        o->wmask[w] = (unsigned char *)calloc(n12, 1);
        o->wuv[w] = (double *)calloc(2 * n12, sizeof(double));
        o->wx1[w] = (double *)calloc((size_t)o->n1, sizeof(double));
    }
    if (mask) memcpy(o->wmask[w], mask, n12);
    if (uv) memcpy(o->wuv[w], uv, 2 * n12 * sizeof(double));
    if (x1) memcpy(o->wx1[w], x1, sizeof(double) * (size_t)o->n1);
    else { o->wx1[w][0] = 0.0; for (int i = 1; i < o->n1; i++) o->wx1[w][i] = o->wx1[w][i - 1] + o->dx; }
    if (w == 0) o->Twb = Tw; else o->Twt = Tw;
}

/* ------------------------------------------------------------ accessors */
/* var(1:nP1,1:nP2,1:nP3,1:7) in Fortran order */
void orc_download(const orc_t *o, double *v)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    int i, j, k, m;
    for (m = 1; m <= 7; m++)
        for (k = 1; k <= n3; k++)
            for (j = 1; j <= n2; j++)
                for (i = 1; i <= n1; i++)
                    v[(((size_t)(m - 1) * n3 + (k - 1)) * n2 + (j - 1)) * n1 + (i - 1)] = VAR(o, m, i, j, k);
}

/* conservative state solV(1:nP1,1:nP2,1:nP3,1:5, lev) in Fortran order */
void orc_download_solv(const orc_t *o, int lev, double *q)
{
    const int n1 = o->n1, n2 = o->n2, n3 = o->n3;
    int i, j, k, m;
    for (m = 1; m <= 5; m++)
        for (k = 1; k <= n3; k++)
            for (j = 1; j <= n2; j++)
                for (i = 1; i <= n1; i++)
                    q[(((size_t)(m - 1) * n3 + (k - 1)) * n2 + (j - 1)) * n1 + (i - 1)] = SOLV(o, lev, m, i, j, k);
}

/* tau2[2] = tauL, tauU ; stat1/stat2 [7*n3], corr [9*n3] (k fastest) */
void orc_get_stats(const orc_t *o, double *tau2, double *stat1, double *stat2, double *corr)
{
    tau2[0] = o->tauL; tau2[1] = o->tauU;
    if (stat1) memcpy(stat1, o->stat1, sizeof(double) * 7 * (size_t)o->n3);
    if (stat2) memcpy(stat2, o->stat2, sizeof(double) * 7 * (size_t)o->n3);
    if (corr) memcpy(corr, o->corr, sizeof(double) * 9 * (size_t)o->n3);
}

long orc_nstep(const orc_t *o) { return o->nstep; }
double orc_time(const orc_t *o) { return o->time; }
int orc_blown(const orc_t *o, int *ijk)
{
    if (ijk) { ijk[0] = o->blown_ijk[0]; ijk[1] = o->blown_ijk[1]; ijk[2] = o->blown_ijk[2]; }
    return o->blown;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---- diagnostics series of a field var(1:nP1,1:nP2,1:nP3,1:7) (i fastest):
 * main_v1.9.f90:799-906 on one rank (bs=1, es=nP, bn(1)=2, en(1)=nP1-1).
 * out = [KE, rho_b[np], U_b[np], rhoU_b[np]]; x3q are the x3 the reference
 * holds, x2end its x2(nP2), dy = Ly/(nP2-1). */
#define FV(m, i, j, k) var[(size_t)((m) - 1) * N + (((size_t)(k) - 1) * n2 + ((size_t)(j) - 1)) * n1 + ((size_t)(i) - 1)]
void orc_diagnostics(const double *var, const int *nP, const int *planes, int np, const double *x3q, double dy,
                     double x2end, double *out)
{
    const int n1 = nP[0], n2 = nP[1], n3 = nP[2];
    const size_t N = (size_t)n1 * n2 * n3;
    const double quar = 0.25, two = 2.0;
    double tmpR1 = 0.0, Ayz;
    int i, j, k, p, q;
    (void)two;
    /* KE: main19:801-817 */
    for (k = 1; k <= n3; k++)
        for (j = 1; j <= n2; j++)
            for (i = 1; i <= n1; i++) {
                const double u = FV(2, i, j, k), v = FV(3, i, j, k), w = FV(4, i, j, k);
                tmpR1 = tmpR1 + ((u * u + v * v) + w * w);
            }
    out[0] = tmpR1 / ((double)n1 * (double)n2 * (double)n3);
    /* bulk rho, U, rho*U: main19:821-906 */
    Ayz = x3q[n3 - 1] * x2end;
    for (q = 0; q < 3; q++)
        for (p = 0; p < np; p++) {
            const int ip = planes[p];
            tmpR1 = 0.0;
            if (ip > 2 && ip < n1 - 1) {
                for (k = 1; k <= n3 - 1; k++)
                    for (j = 1; j <= n2 - 1; j++) {
                        const double dAyz = dy * (x3q[k] - x3q[k - 1]);
                        double a, b, c, d;
                        if (q == 0) {
                            a = FV(1, ip, j, k); b = FV(1, ip, j + 1, k); c = FV(1, ip, j, k + 1); d = FV(1, ip, j + 1, k + 1);
                        } else if (q == 1) {
                            a = FV(2, ip, j, k); b = FV(2, ip, j + 1, k); c = FV(2, ip, j, k + 1); d = FV(2, ip, j + 1, k + 1);
                        } else {
                            a = FV(1, ip, j, k) * FV(2, ip, j, k);
                            b = FV(1, ip, j + 1, k) * FV(2, ip, j + 1, k);
                            c = FV(1, ip, j, k + 1) * FV(2, ip, j, k + 1);
                            d = FV(1, ip, j + 1, k + 1) * FV(2, ip, j + 1, k + 1);
                        }
                        tmpR1 = tmpR1 + quar * (((a + b) + c) + d) * dAyz;
                    }
            }
            out[1 + q * np + p] = tmpR1 / Ayz;
        }
}
#undef FV

/* ---- Q-criterion: v1.9_strat/v1.9_st1/codes/qInvariant.f90:26-81.
 * u,v,w,Q are nP1*nP2*nP3 (i fastest); box faces get 0. */
void orc_qcrit(const int *nP, const double *u, const double *v, const double *w, const double *x, const double *y,
               const double *z, double *Q)
{
    const int n1 = nP[0], n2 = nP[1], n3 = nP[2];
    const double haf = 0.5;
    const double *Ut[3] = {u, v, w};
    int i, j, k;
    memset(Q, 0, sizeof(double) * (size_t)n1 * n2 * n3);
    for (k = 2; k <= n3 - 1; k++)
        for (j = 2; j <= n2 - 1; j++)
            for (i = 2; i <= n1 - 1; i++) {
                const size_t c0 = (((size_t)k - 1) * n2 + (j - 1)) * n1 + (i - 1);
                const size_t si = 1, sj = (size_t)n1, sk = (size_t)n1 * n2;
                double dx[3][2], Jt[3][3], S[3][3], R[3][3], As1, As2, P;
                int jc, a, b;
                dx[0][0] = x[i] - x[i - 1]; dx[1][0] = y[j] - y[j - 1]; dx[2][0] = z[k] - z[k - 1];
                dx[0][1] = x[i - 1] - x[i - 2]; dx[1][1] = y[j - 1] - y[j - 2]; dx[2][1] = z[k - 1] - z[k - 2];
                for (jc = 0; jc < 3; jc++) {
                    const double *U = Ut[jc];
                    Jt[jc][0] = ((dx[0][1] / dx[0][0]) * (U[c0 + si] - U[c0]) + (dx[0][0] / dx[0][1]) * (U[c0] - U[c0 - si]))
                                / (dx[0][0] + dx[0][1]);
                    Jt[jc][1] = ((dx[1][1] / dx[1][0]) * (U[c0 + sj] - U[c0]) + (dx[1][0] / dx[1][1]) * (U[c0] - U[c0 - sj]))
                                / (dx[1][0] + dx[1][1]);
                    Jt[jc][2] = ((dx[2][1] / dx[2][0]) * (U[c0 + sk] - U[c0]) + (dx[2][0] / dx[2][1]) * (U[c0] - U[c0 - sk]))
                                / (dx[2][0] + dx[2][1]);
                }
                S[0][0] = Jt[0][0]; S[0][1] = haf * (Jt[0][1] + Jt[1][0]); S[0][2] = haf * (Jt[0][2] + Jt[2][0]);
                S[1][0] = haf * (Jt[1][0] + Jt[0][1]); S[1][1] = Jt[1][1]; S[1][2] = haf * (Jt[2][1] + Jt[1][2]);
                S[2][0] = haf * (Jt[2][0] + Jt[0][2]); S[2][1] = haf * (Jt[2][1] + Jt[1][2]); S[2][2] = Jt[2][2];
                R[0][0] = 0.0; R[0][1] = haf * (Jt[0][1] - Jt[1][0]); R[0][2] = haf * (Jt[0][2] - Jt[2][0]);
                R[1][0] = haf * (Jt[1][0] - Jt[0][1]); R[1][1] = 0.0; R[1][2] = haf * (Jt[1][2] - Jt[2][1]);
                R[2][0] = haf * (Jt[2][0] - Jt[0][2]); R[2][1] = haf * (Jt[2][1] - Jt[1][2]); R[2][2] = 0.0;
                /* sum(S**2.0), sum(-R**2.0) in array-element (column-major) order */
                As1 = 0.0; As2 = 0.0;
                for (b = 0; b < 3; b++)
                    for (a = 0; a < 3; a++) {
                        As1 = As1 + S[a][b] * S[a][b];
                        As2 = As2 + (-(R[a][b] * R[a][b]));
                    }
                P = -((S[0][0] + S[1][1]) + S[2][2]);
                Q[c0] = haf * ((P * P - As1) - As2);
            }
}
