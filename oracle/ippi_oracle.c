/*
 * ippi_oracle.c -- FP64 CPU restatement of the IPPI-LBM D2Q9 step.
 * TEST INFRASTRUCTURE ONLY (the checker); see ippi_oracle.h for the map of
 * reference functions restated here.  Storage mirrors the reference's
 * LatMesh: local column i = x + 1 with one halo column on each side
 * (i = 0 and i = nx + 1), rows j = y.  Arithmetic follows the reference's
 * expression order so that, compiled without FMA contraction, the flat-plate
 * step reproduces the reference build bit for bit.
 */
#include "ippi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* D2Q9 velocity order of the reference: NodeAndLattice.cpp:3-13, mesh.cpp:3-13 */
static const int E[9][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1},
                            {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
/* weight[] of NodeAndLattice.cpp:14 */
static const double W[9] = {4. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 9.,
                            1. / 36., 1. / 36., 1. / 36., 1. / 36.};
static const int OPP[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

enum { COLL_BGK = 0, COLL_MRT = 1, COLL_RR = 2 };
enum { BC_REF = 0, BC_CHANNEL = 1 };

typedef struct {
    double x, y, ubx, uby, ds;
    double vref_x, vref_y, fx, fy;
    int body;
} marker;

typedef struct {
    int nin;
    float* w;
} band_net;

struct orc {
    orc_params p;
    int NX, NY;                 /* NX = nx + 2 (halo columns), NY = ny */
    double* fnew;               /* [9][NX*NY] */
    double* fcol;
    double *rho, *ux, *uy, *tau, *fxn, *fyn;
    double *avg_u, *avg_v, *avg_rho;
    unsigned char* nnflag;
    char* style;
    band_net nets[8];
    int nmark, nbody;
    marker* mk;
    double* body_force;         /* [2*nbody] */
    double mass;
    double mrt_tm[9][9], mrt_tminv[9][9];
    double mlp[1313 + 25];      /* learned tau network (les_model 2) */
    double* tau_field;          /* les_model 3: tau per node, [ny][nx] global */
    int mlp_loaded;
    unsigned char* solid;       /* [NX*NY] solid nodes, or NULL */
    double* wall_dist;          /* les_model 6: [ny][nx] global */
};

#define ID(s, i, j) ((size_t)(i) * (size_t)(s)->NY + (size_t)(j))
#define FN(s, k, i, j) ((s)->fnew[(size_t)(k) * (size_t)(s)->NX * (s)->NY + ID(s, i, j)])
#define FC(s, k, i, j) ((s)->fcol[(size_t)(k) * (size_t)(s)->NX * (s)->NY + ID(s, i, j)])

/* ---------------------------------------------------------------------- */
/* per-node building blocks                                                */
/* ---------------------------------------------------------------------- */

/* Lattice::Compute_feq, NodeAndLattice.cpp:124-149 (same expression order). */
static void compute_feq(double rho, double ux, double uy, double* feq)
{
    double w0 = rho * (4.0 / 9.0);
    double w1 = rho / 9.0;
    double w2 = rho / 36.0;
    double uu = 1 - 1.5 * (ux * ux + uy * uy);
    feq[0] = w0 * (uu);
    feq[1] = w1 * (uu + 3.0 * (ux) + 4.5 * (ux) * (ux));
    feq[2] = w1 * (uu + 3.0 * (uy) + 4.5 * (uy) * (uy));
    feq[3] = w1 * (uu - 3.0 * (ux) + 4.5 * (ux) * (ux));
    feq[4] = w1 * (uu - 3.0 * (uy) + 4.5 * (uy) * (uy));
    feq[5] = w2 * (uu + 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    feq[6] = w2 * (uu - 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
    feq[7] = w2 * (uu - 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    feq[8] = w2 * (uu + 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
}

/* Lattice::InitialLatticeFeq, NodeAndLattice.cpp:104-119: note rho*4.0/9.0. */
static void initial_feq(double rho, double ux, double uy, double* f)
{
    double w0 = rho * 4.0 / 9.0;
    double w1 = rho / 9.0;
    double w2 = rho / 36.0;
    double uu = 1 - 1.5 * (ux * ux + uy * uy);
    f[0] = w0 * (uu);
    f[1] = w1 * (uu + 3.0 * (ux) + 4.5 * (ux) * (ux));
    f[2] = w1 * (uu + 3.0 * (uy) + 4.5 * (uy) * (uy));
    f[3] = w1 * (uu - 3.0 * (ux) + 4.5 * (ux) * (ux));
    f[4] = w1 * (uu - 3.0 * (uy) + 4.5 * (uy) * (uy));
    f[5] = w2 * (uu + 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    f[6] = w2 * (uu - 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
    f[7] = w2 * (uu - 3.0 * (ux + uy) + 4.5 * (ux + uy) * (ux + uy));
    f[8] = w2 * (uu + 3.0 * (ux - uy) + 4.5 * (ux - uy) * (ux - uy));
}

/* Lattice::CalMacro, NodeAndLattice.cpp:196-227. */
static void cal_macro(const double* f, double* rho, double* ux, double* uy)
{
    double trho = 0.0, tx = 0.0, ty = 0.0;
    for (int k = 0; k < 9; k++) {
        trho += f[k];
        tx += f[k] * E[k][0];
        ty += f[k] * E[k][1];
    }
    if (trho < 1.e-6) {
        tx = 0.0;
        ty = 0.0;
    } else {
        tx /= trho;
        ty /= trho;
    }
    *rho = trho;
    *ux = tx;
    *uy = ty;
}

/* Mesh::CaculateLESTau, active SmagorinskyByHybrid block mesh.cpp:877-910.
 * tau0 is startTau (not the node's own tau, mesh.cpp:882). */
double orc_les_tau(const double* fnew, double rho, double ux, double uy,
                   double tau0, double cs)
{
    double rhoTemp = 1.0;
    rhoTemp *= rho;
    double feq[9];
    compute_feq(rho, ux, uy, feq);
    double Tau = tau0;
    double Sxx = 0.0, Sxy = 0.0, Syx = 0.0, Syy = 0.0;
    for (int k = 0; k < 9; k++) {
        Sxx += E[k][0] * E[k][0] * (fnew[k] - feq[k]);
        Sxy += E[k][0] * E[k][1] * (fnew[k] - feq[k]);
        Syy += E[k][1] * E[k][1] * (fnew[k] - feq[k]);
    }
    Syx = Sxy;
    Sxx *= -3.0 / (2 * rhoTemp * Tau);
    Sxy *= -3.0 / (2 * rhoTemp * Tau);
    Syx *= -3.0 / (2 * rhoTemp * Tau);
    Syy *= -3.0 / (2 * rhoTemp * Tau);
    double S2 = Sxx * Sxx + Sxy * Sxy + Syx * Syx + Syy * Syy;
    double Q = sqrt(2.0 * S2);
    double g1 = tau0 * tau0 + 18.0 * cs * cs * Q / (rhoTemp);
    return (sqrt(g1) + tau0) / 2.0;
}

/* Mesh::GetDuxDx / GetDuyDx (mesh.cpp:1659-1724, 1795-1864) and GetDuxDy /
 * GetDuyDy (1725-1794, 1865-1934) on one rank: forward differences of the
 * current u (comp 0) or v (comp 1) along x (dir 0) or y (dir 1); 0 towards a
 * solid node, in the last column (imax = NX - 1) and from the second-to-last
 * row up (jmax >= Ny - 1). */
static double grad_u(const orc* s, int i, int j, int comp, int dir)
{
    const double* u = comp ? s->uy : s->ux;
    if (dir == 0) {
        int imax = i + 1;
        if ((s->solid && s->solid[ID(s, imax, j)]) || imax == s->NX - 1) return 0.0;
        return (u[ID(s, imax, j)] - u[ID(s, i, j)]) / 1.0;
    }
    int jmax = j + 1;
    if (jmax >= s->NY - 1 || (s->solid && s->solid[ID(s, i, jmax)])) return 0.0;
    return (u[ID(s, i, jmax)] - u[ID(s, i, j)]) / 1.0;
}

/* sum_k e_a e_b (fnew - feq) */
static void pi_noneq(const double* fnew, double rho, double ux, double uy, double* qxx, double* qxy,
                     double* qyy)
{
    double feq[9];
    compute_feq(rho, ux, uy, feq);
    *qxx = *qxy = *qyy = 0.0;
    for (int k = 0; k < 9; k++) {
        *qxx += E[k][0] * E[k][0] * (fnew[k] - feq[k]);
        *qxy += E[k][0] * E[k][1] * (fnew[k] - feq[k]);
        *qyy += E[k][1] * E[k][1] * (fnew[k] - feq[k]);
    }
}

/* The alternative closures of Mesh::CaculateLESTau for node (i, j):
 * 4 WALE (mesh.cpp:934-967), 5 coherent structure (1034-1071 with
 * ComputeDynamicCs, 2113-2146), 6 wall-damped Cs (968-1000). */
static double ext_tau(const orc* s, int i, int j, const double* fnew, double rho, double ux, double uy)
{
    double startTau = s->p.tau0, delta = 1.0;
    if (s->p.les_model == 4) {
        double Cw = 0.45;
        double gxx = grad_u(s, i, j, 0, 0), gxy = grad_u(s, i, j, 0, 1);
        double gyx = grad_u(s, i, j, 1, 0), gyy = grad_u(s, i, j, 1, 1);
        double Sxx = 0.5 * (gxx + gxx), Sxy = 0.5 * (gxy + gyx), Syx = Sxy, Syy = 0.5 * (gyy + gyy);
        double SS = Sxx * Sxx + Sxy * Sxy + Syx * Syx + Syy * Syy;
        double gxx2 = gxx * gxx + gxy * gyx, gxy2 = gxx * gxy + gxy * gyy;
        double gyx2 = gyx * gxx + gyy * gyx, gyy2 = gyx * gxy + gyy * gyy;
        double grr2 = gxx * gxx + gxy * gyx + gyx * gxy + gyy * gyy;
        double Gxx = 0.5 * (gxx2 + gxx2) - grr2 / 3.0, Gxy = 0.5 * (gxy2 + gyx2);
        double Gyx = 0.5 * (gyx2 + gxy2), Gyy = 0.5 * (gyy2 + gyy2) - grr2 / 3.0;
        double GG = Gxx * Gxx + Gxy * Gxy + Gyx * Gyx + Gyy * Gyy;
        double vt = Cw * Cw * delta * delta * pow(GG, 1.5) / (pow(SS, 2.5) + pow(GG, 1.25) + 1e-12);
        return startTau + 3 * vt;
    }
    double Qxx, Qxy, Qyy;
    pi_noneq(fnew, rho, ux, uy, &Qxx, &Qxy, &Qyy);
    double Qyx = Qxy;
    if (s->p.les_model == 5) {
        double gxx = grad_u(s, i, j, 0, 0), gxy = grad_u(s, i, j, 0, 1);
        double gyx = grad_u(s, i, j, 1, 0), gyy = grad_u(s, i, j, 1, 1);
        double Sxx = 0.5 * (gxx + gxx), Sxy = 0.5 * (gxy + gyx), Syx = Sxy, Syy = 0.5 * (gyy + gyy);
        double SS = Sxx * Sxx + Sxy * Sxy + Syx * Syx + Syy * Syy;
        double Wxy = 0.5 * (gxy - gyx);
        double WW = 2 * Wxy * Wxy;
        double Q = 0.5 * (WW - SS), Ev = 0.5 * (WW + SS);
        double Ccsm;
        if (Ev == 0) {
            Ccsm = 0.016;
        } else {
            double Fcs = fabs(Q / Ev);
            Ccsm = (1 / 11.0) * pow(Fcs, 1.5) * (1 - Fcs);
        }
        double S2 = Qxx * Qxx + Qxy * Qxy + Qyx * Qyx + Qyy * Qyy;
        double vt = Ccsm * delta * delta * sqrt(2 * S2);
        return startTau + 3 * vt;
    }
    double d = s->wall_dist[(size_t)j * s->p.nx + (i - 1)];
    double SC = 3.0 / (1 + pow(1.71828, 6.0 - 1.0 * d));
    double Q = sqrt(2 * (Qxx * Qxx + Qxy * Qxy + Qyx * Qyx + Qyy * Qyy));
    double tauT = (sqrt(startTau * startTau + 18.0 * delta * SC * SC * Q / rho) - startTau) / 2.0;
    return startTau + tauT;
}

int orc_set_wall_distance(orc* s, const double* d)
{
    size_t n = (size_t)s->p.nx * s->p.ny;
    if (!s->wall_dist) s->wall_dist = (double*)malloc(n * sizeof(double));
    memcpy(s->wall_dist, d, n * sizeof(double));
    return 0;
}

/* Learned relaxation time (no reference code).  Features from the node's
 * post-stream state: rho, |u|, the direction Pi/|Pi| of
 * Pi = sum_k e e (fnew - feq) (|Pi| = sqrt(Pxx^2 + 2 Pxy^2 + Pyy^2)) and
 * |S| = sqrt(2 S:S) with S = -3/(2 rho tau0) Pi, as in orc_les_tau.  Outside
 * the training range of any feature the Smagorinsky tau is used. */
double orc_learned_tau(const double* fnew, double rho, double ux, double uy,
                       double tau0, double cs, const double* p)
{
    const double* W1 = p;
    const double* b1 = p + 192;
    const double* W2 = p + 224;
    const double* b2 = p + 1248;
    const double* w3 = p + 1280;
    const double b3 = p[1312];
    const double* st = p + 1313;
    double feq[9];
    compute_feq(rho, ux, uy, feq);
    double pxx = 0.0, pxy = 0.0, pyy = 0.0;
    for (int k = 0; k < 9; k++) {
        pxx += E[k][0] * E[k][0] * (fnew[k] - feq[k]);
        pxy += E[k][0] * E[k][1] * (fnew[k] - feq[k]);
        pyy += E[k][1] * E[k][1] * (fnew[k] - feq[k]);
    }
    double c = -1.5 / (rho * tau0);
    double sxx = pxx * c, sxy = pxy * c, syy = pyy * c;
    double pn = sqrt(pxx * pxx + 2.0 * pxy * pxy + pyy * pyy);
    double inv = pn > 0 ? 1.0 / pn : 0.0;
    double x[6] = {rho, sqrt(ux * ux + uy * uy), pxx * inv, pxy * inv, pyy * inv,
                   sqrt(2.0 * (sxx * sxx + 2.0 * sxy * sxy + syy * syy))};
    for (int i = 0; i < 6; i++) {
        if (!(x[i] >= st[12 + i] && x[i] <= st[18 + i])) return orc_les_tau(fnew, rho, ux, uy, tau0, cs);
        x[i] = (x[i] - st[i]) / st[6 + i];
    }
    double h1[32];
    for (int j = 0; j < 32; j++) {
        double a = b1[j];
        for (int i = 0; i < 6; i++) a += W1[j * 6 + i] * x[i];
        h1[j] = tanh(a);
    }
    double z = b3;
    for (int j = 0; j < 32; j++) {
        double a = b2[j];
        for (int i = 0; i < 32; i++) a += W2[j * 32 + i] * h1[i];
        z += w3[j] * tanh(a);
    }
    double sp = (z > 0 ? z : 0.0) + log1p(exp(-fabs(z)));
    return tau0 + st[24] * sp;
}

int orc_set_tau_field(orc* s, const double* tau)
{
    size_t n = (size_t)s->p.nx * s->p.ny;
    if (!s->tau_field) s->tau_field = (double*)malloc(n * sizeof(double));
    memcpy(s->tau_field, tau, n * sizeof(double));
    return 0;
}

int orc_load_tau_mlp(orc* s, const float* w, size_t n, const float* stats, size_t nstats)
{
    if (!s || !w || !stats || n != 1313 || nstats != 25) return -1;
    for (size_t i = 0; i < n; i++) s->mlp[i] = w[i];
    for (size_t i = 0; i < nstats; i++) s->mlp[1313 + i] = stats[i];
    s->mlp_loaded = 1;
    return 0;
}

/* D2Q9 MRT transformation matrix in the reference velocity order, built from
 * its moment definitions (1, e, eps, jx, qx, jy, qy, pxx, pxy); the inverse
 * is M^T diag(1/|row|^2), written as integer multiples of 1/36 as the
 * reference's tminv table is (NodeAndLattice.cpp:18-29). */
static void build_mrt(double tm[9][9], double tminv[9][9])
{
    static const int mult[9] = {4, 1, 1, 6, 3, 6, 3, 9, 9}; /* 36/|row|^2 */
    const double a1 = 1.0 / 36.0;
    for (int k = 0; k < 9; k++) {
        int cx = E[k][0], cy = E[k][1];
        int c2 = cx * cx + cy * cy;
        int row[9];
        row[0] = 1;
        row[1] = -4 + 3 * c2;
        row[2] = (8 - 21 * c2 + 9 * c2 * c2) / 2;
        row[3] = cx;
        row[4] = (-5 + 3 * c2) * cx;
        row[5] = cy;
        row[6] = (-5 + 3 * c2) * cy;
        row[7] = cx * cx - cy * cy;
        row[8] = cx * cy;
        for (int i = 0; i < 9; i++) {
            tm[i][k] = (double)row[i];
            tminv[k][i] = (double)(row[i] * mult[i]) * a1;
        }
    }
}

static double g_tm[9][9], g_tminv[9][9];
static int g_mrt_ready = 0;

/* The MRT matrices, built once before any threaded loop reads them. */
static void mrt_tables(void)
{
    if (!g_mrt_ready) {
        build_mrt(g_tm, g_tminv);
        g_mrt_ready = 1;
    }
}

static void collide_bgk(const double* fnew, const double* feq, double tau, double* fcol)
{
    /* Lattice::ComputeBGKCollision, NodeAndLattice.cpp:150-161 */
    for (int k = 0; k < 9; k++)
        fcol[k] = (1.0 - 1.0 / tau) * fnew[k] + feq[k] / tau;
}

static void collide_mrt(const double* fnew, double rho, double ux, double uy,
                        double tau, double* fcol)
{
    /* Lattice::ComputeMRTCollision, NodeAndLattice.cpp:290-360 */
    if (!g_mrt_ready) {
        build_mrt(g_tm, g_tminv);
        g_mrt_ready = 1;
    }
    double sm[9] = {0, 1.2, 1.1, 0, 1.2, 0, 1.2, 1. / tau, 1. / tau};
    double stmiv[9][9], fmom[9], fmeq[9];
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < 9; j++) stmiv[i][j] = g_tminv[i][j] * sm[j];
    double t1 = ux * ux + uy * uy;
    double t2 = ux * ux - uy * uy;
    fmeq[0] = rho;
    fmeq[1] = rho * (-2.0 + 3.0 * t1);
    fmeq[2] = rho * (1.0 - 3.0 * t1);
    fmeq[3] = rho * ux;
    fmeq[4] = -rho * ux;
    fmeq[5] = rho * uy;
    fmeq[6] = -rho * uy;
    fmeq[7] = rho * t2;
    fmeq[8] = rho * ux * uy;
    for (int k = 0; k < 9; k++) {
        double suma = 0.0;
        for (int l = 0; l < 9; l++) suma += g_tm[k][l] * fnew[l];
        fmom[k] = suma;
    }
    for (int k = 0; k < 9; k++) {
        double sumb = 0.;
        for (int l = 0; l < 9; l++) sumb += stmiv[k][l] * (fmom[l] - fmeq[l]);
        fcol[k] = fnew[k] - sumb;
    }
}

static void collide_rr(const double* fnew, const double* feq, double tau, double* fcol)
{
    /* Lattice::ComputeRRCollision, NodeAndLattice.cpp:228-288 */
    double mftxx = 0, mfttempxx = 0, mftxy = 0, mfttempxy = 0;
    double mftyx = 0, mfttempyx = 0, mftyy = 0, mfttempyy = 0;
    for (int k = 0; k < 9; k++) {
        mftxx += fnew[k] * E[k][0] * E[k][0];
        mfttempxx += feq[k] * E[k][0] * E[k][0];
        mftxy += fnew[k] * E[k][0] * E[k][1];
        mfttempxy += feq[k] * E[k][0] * E[k][1];
        mftyx += fnew[k] * E[k][1] * E[k][0];
        mfttempyx += feq[k] * E[k][1] * E[k][0];
        mftyy += fnew[k] * E[k][1] * E[k][1];
        mfttempyy += feq[k] * E[k][1] * E[k][1];
    }
    double XX = mftxx - mfttempxx, XY = mftxy - mfttempxy;
    double YX = mftyx - mfttempyx, YY = mftyy - mfttempyy;
    for (int k = 0; k < 9; k++) {
        double Q0 = E[k][0] * E[k][0] - 1. / 3;
        double Q1 = E[k][0] * E[k][1];
        double Q2 = E[k][1] * E[k][0];
        double Q3 = E[k][1] * E[k][1] - 1. / 3;
        double fone = 4.5 * W[k] * (Q0 * XX + Q1 * XY + Q2 * YX + Q3 * YY);
        fcol[k] = feq[k] + (1.0 - 1.0 / tau) * fone;
    }
}

void orc_collide_node(int collision, const double* fnew, double rho, double ux,
                      double uy, double tau, double* fcol)
{
    double feq[9];
    compute_feq(rho, ux, uy, feq);
    if (collision == COLL_MRT)
        collide_mrt(fnew, rho, ux, uy, tau, fcol);
    else if (collision == COLL_RR)
        collide_rr(fnew, feq, tau, fcol);
    else
        collide_bgk(fnew, feq, tau, fcol);
}

/* Lattice::Compute_Disforce, NodeAndLattice.cpp:162-195 (tau0 = TauAtBeginning). */
static void guo_force(double ux, double uy, double Fx, double Fy, double tau0, double* lf)
{
    double omega = 1.0 - 0.5 * (1.0 / tau0);
    for (int k = 0; k < 9; k++) {
        double eu = (E[k][0] * ux + E[k][1] * uy);
        double fx = W[k] * omega * (3.0 * (E[k][0] - ux) + 9.0 * eu * E[k][0]) * Fx;
        double fy = W[k] * omega * (3.0 * (E[k][1] - uy) + 9.0 * eu * E[k][1]) * Fy;
        lf[k] = fx + fy;
    }
}

/* Forcing term of the IB force (Fx, Fy) for the collision operator in use
 * (no reference code: the reference's IB path is not active).  Each form
 * adds exactly F to a forced node's momentum in one collision, the
 * equilibrium being taken at the corrected velocity u = u* + F / (2 rho):
 *   BGK  Lattice::Compute_Disforce (Guo, omega from tau0), as the reference
 *   MRT  the Guo source G in moment space, M^-1 (I - S/2) M G: conserved
 *        moments take it whole, the others (1 - s_m / 2), s_7 = s_8 = 1/tau
 *   RR   first-order part of G halved (the shifted equilibrium carries the
 *        other half), second-order part (1 - 1/(2 tau)) */
static void force_term(int coll, double ux, double uy, double Fx, double Fy, double tau0,
                       double tau, double* lf)
{
    if (coll == COLL_BGK) {
        guo_force(ux, uy, Fx, Fy, tau0, lf);
        return;
    }
    double g[9];
    for (int k = 0; k < 9; k++) {
        double eu = E[k][0] * ux + E[k][1] * uy;
        double eF = E[k][0] * Fx + E[k][1] * Fy;
        double uF = ux * Fx + uy * Fy;
        if (coll == COLL_RR)
            lf[k] = W[k] * (0.5 * 3.0 * eF + (1.0 - 0.5 / tau) * (9.0 * eu * eF - 3.0 * uF));
        g[k] = W[k] * (3.0 * eF - 3.0 * uF + 9.0 * eu * eF);
    }
    if (coll == COLL_RR) return;
    if (!g_mrt_ready) {
        build_mrt(g_tm, g_tminv);
        g_mrt_ready = 1;
    }
    double sm[9] = {0, 1.2, 1.1, 0, 1.2, 0, 1.2, 1. / tau, 1. / tau};
    double a[9];
    for (int m = 0; m < 9; m++) {
        double gm = 0.0, norm = 0.0;
        for (int k = 0; k < 9; k++) {
            gm += g_tm[m][k] * g[k];
            norm += g_tm[m][k] * g_tm[m][k];
        }
        a[m] = (1.0 - 0.5 * sm[m]) * gm / norm;
    }
    for (int k = 0; k < 9; k++) {
        double v = 0.0;
        for (int m = 0; m < 9; m++) v += g_tm[m][k] * a[m];
        lf[k] = v;
    }
}

void orc_force_node(int collision, double ux, double uy, double fx, double fy, double tau0,
                    double tau, double* lf)
{
    force_term(collision, ux, uy, fx, fy, tau0, tau, lf);
}

/* Mesh::DiracDelta, mesh.cpp:1354-1385 */
double orc_peskin_phi(double x)
{
    if (fabs(x) < 1) {
        double R = 1.0 + 4.0 * fabs(x) - 4 * (x * x);
        return (1.0 / 8.0) * (3.0 - 2.0 * fabs(x) + sqrt(R));
    } else if (fabs(x) < 2) {
        double R = -7.0 + 12.0 * fabs(x) - 4 * (x * x);
        return (1.0 / 8.0) * (5.0 - 2.0 * fabs(x) - sqrt(R));
    }
    return 0;
}

/* Marker stencil of Mesh::InterpolateVel / SpreadForce (mesh.cpp:566-585 for
 * the 4x4 Peskin kernel, 618-638 for the 2x2 bilinear kernel), in global
 * coordinates: XInt = (int)x, node position = its integer index.  A node's
 * contribution is (value * wa) * wb: the Peskin kernel multiplies by the
 * product phi(dx)phi(dy) (wb = 1), the bilinear one by WeightX then WeightY,
 * the order of mesh.cpp:580 and 633. */
static int marker_stencil2(int delta_kernel, double mx, double my, int* xs, int* ys,
                           double* wa, double* wb)
{
    int XInt = (int)(mx), YInt = (int)(my);
    int n = 0;
    if (delta_kernel == 1) {
        for (int X = XInt - 1; X <= XInt + 2; X++)
            for (int Y = YInt - 1; Y <= YInt + 2; Y++) {
                double DistX = mx - X, DistY = my - Y;
                xs[n] = X;
                ys[n] = Y;
                wa[n] = orc_peskin_phi(DistX) * orc_peskin_phi(DistY);
                wb[n] = 1.0;
                n++;
            }
    } else {
        for (int X = XInt; X <= XInt + 1; X++)
            for (int Y = YInt; Y <= YInt + 1; Y++) {
                double DistX = mx - X, DistY = my - Y;
                xs[n] = X;
                ys[n] = Y;
                wa[n] = 1 - fabs(DistX);
                wb[n] = 1 - fabs(DistY);
                n++;
            }
    }
    return n;
}

int orc_marker_stencil(int delta_kernel, double mx, double my, int* xs, int* ys, double* ws)
{
    double wa[16], wb[16];
    int n = marker_stencil2(delta_kernel, mx, my, xs, ys, wa, wb);
    for (int q = 0; q < n; q++) ws[q] = wa[q] * wb[q];
    return n;
}

/* Boundary net forward pass: Linear(nin,128)+ReLU, 6 x (Linear(128,128)+ReLU),
 * Linear(128,1), float32 -- the TorchScript Net of NNmodel/AutoT0x.pt
 * (dropout is inactive, the archives were saved in eval mode).  Weights are
 * the TorchScript parameters in order, each Linear as weight[out][in], bias[out]. */
float orc_band_forward(const float* w, int nin, const float* in)
{
    float a[128], b[128];
    const float* p = w;
    for (int o = 0; o < 128; o++) {
        float acc = 0.f;
        for (int i = 0; i < nin; i++) acc += p[o * nin + i] * in[i];
        acc += p[128 * nin + o];
        a[o] = acc > 0.f ? acc : 0.f;
    }
    p += 128 * nin + 128;
    for (int layer = 0; layer < 6; layer++) {
        for (int o = 0; o < 128; o++) {
            float acc = 0.f;
            for (int i = 0; i < 128; i++) acc += p[o * 128 + i] * a[i];
            acc += p[128 * 128 + o];
            b[o] = acc > 0.f ? acc : 0.f;
        }
        memcpy(a, b, sizeof a);
        p += 128 * 128 + 128;
    }
    float acc = 0.f;
    for (int i = 0; i < 128; i++) acc += p[i] * a[i];
    acc += p[128];
    return acc;
}

/* ---------------------------------------------------------------------- */
/* mesh-level state                                                        */
/* ---------------------------------------------------------------------- */

/* Mesh::JudgeStyle (mesh.cpp:1398-1425) for one rank; plate_x0 replaces the
 * hard-coded 400 of mesh.cpp:1413.  The channel scene marks its inlet 'i',
 * outlet 'o', wall rows 'w'. */
static void judge_style(orc* s)
{
    int NX = s->NX, Ny = s->NY;
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < Ny; j++) {
            char st = 'f';
            if (s->p.bc_set == BC_REF) {
                double posx = (i == 0) ? -1 : (i == NX - 1 ? (double)(NX - 2) : (double)(i - 1));
                if (i == 1)
                    st = 'i';
                else if (i == NX - 2)
                    st = 'o';
                else if (j == 0)
                    st = (posx < s->p.plate_x0) ? 'm' : 'd';
                else if (j == Ny - 1)
                    st = 'u';
            } else {
                if (i == 1)
                    st = 'i';
                else if (i == NX - 2)
                    st = 'o';
                else if (j == 0 || j == Ny - 1)
                    st = 'w';
            }
            s->style[ID(s, i, j)] = st;
        }
    if (!s->solid) return;
    /* solid 's' and fluid nodes with a link into a solid 'b' (the styles
     * Mesh::OutputCd, mesh.cpp:1472-1478, sums over) */
    for (int i = 2; i < NX - 2; i++)
        for (int j = 1; j < Ny - 1; j++) {
            if (s->solid[ID(s, i, j)]) {
                s->style[ID(s, i, j)] = 's';
                continue;
            }
            for (int k = 1; k < 9; k++)
                if (s->solid[ID(s, i + E[k][0], j + E[k][1])]) s->style[ID(s, i, j)] = 'b';
        }
}

orc* orc_create(const orc_params* p)
{
    if (p->nx < 4 || p->ny < 4) return NULL;
    if (p->delta_kernel != 0 && p->delta_kernel != 1) return NULL;
    orc* s = (orc*)calloc(1, sizeof(orc));
    s->p = *p;
    if (s->p.mdf_iters < 1) s->p.mdf_iters = 1;
    if (s->p.rho0 == 0) s->p.rho0 = 1.0;
    s->NX = p->nx + 2;
    s->NY = p->ny;
    size_t n = (size_t)s->NX * s->NY;
    s->fnew = (double*)calloc(9 * n, sizeof(double));
    s->fcol = (double*)calloc(9 * n, sizeof(double));
    s->rho = (double*)calloc(n, sizeof(double));
    s->ux = (double*)calloc(n, sizeof(double));
    s->uy = (double*)calloc(n, sizeof(double));
    s->tau = (double*)calloc(n, sizeof(double));
    s->fxn = (double*)calloc(n, sizeof(double));
    s->fyn = (double*)calloc(n, sizeof(double));
    s->avg_u = (double*)calloc(n, sizeof(double));
    s->avg_v = (double*)calloc(n, sizeof(double));
    s->avg_rho = (double*)calloc(n, sizeof(double));
    s->nnflag = (unsigned char*)calloc(n, 1);
    s->style = (char*)calloc(n, 1);
    judge_style(s);
    orc_init_macros(s, NULL, NULL, NULL);
    return s;
}

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_destroy(orc* s)
{
    if (!s) return;
    free(s->fnew); free(s->fcol); free(s->rho); free(s->ux); free(s->uy);
    free(s->tau); free(s->fxn); free(s->fyn); free(s->avg_u); free(s->avg_v);
    free(s->avg_rho); free(s->nnflag); free(s->style); free(s->mk);
    free(s->body_force);
    free(s->tau_field);
    free(s->solid);
    free(s->wall_dist);
    for (int t = 0; t < 8; t++) free(s->nets[t].w);
    free(s);
}

/* Mesh::InitialLatMesh (mesh.cpp:88-166) + the rho=1 reset of JudgeStyle;
 * halo columns take rho=1, u=0 as the reference's do. */
void orc_init_macros(orc* s, const double* rho, const double* ux, const double* uy)
{
    int nx = s->p.nx;
    for (int i = 0; i < s->NX; i++)
        for (int j = 0; j < s->NY; j++) {
            size_t id = ID(s, i, j);
            int x = i - 1;
            double r = 1.0, vx = 0.0, vy = 0.0;
            if (x >= 0 && x < nx) {
                size_t g = (size_t)j * nx + x;
                if (rho) r = rho[g];
                if (ux) vx = ux[g];
                if (uy) vy = uy[g];
            }
            s->rho[id] = r;
            s->ux[id] = vx;
            s->uy[id] = vy;
            s->tau[id] = s->p.tau0;
            s->nnflag[id] = 0;
            s->fxn[id] = s->fyn[id] = 0;
            s->avg_u[id] = s->avg_v[id] = s->avg_rho[id] = 0;
            double f[9];
            initial_feq(r, vx, vy, f);
            for (int k = 0; k < 9; k++) {
                FN(s, k, i, j) = f[k];
                FC(s, k, i, j) = f[k];
            }
        }
}

int orc_load_band_net(orc* s, int type, const float* w, size_t n)
{
    if (type < 0 || type > 7) return -1;
    int nin = (type % 2 == 0) ? 9 : 15;
    size_t need = (size_t)128 * nin + 128 + 6 * (128 * 128 + 128) + 128 + 1;
    if (n != need) return -1;
    free(s->nets[type].w);
    s->nets[type].w = (float*)malloc(n * sizeof(float));
    memcpy(s->nets[type].w, w, n * sizeof(float));
    s->nets[type].nin = nin;
    return 0;
}

int orc_set_markers(orc* s, int n, const double* xy, const double* ub,
                    const int* body, const double* ds)
{
    int xs[16], ys[16];
    double ws[16];
    for (int m = 0; m < n; m++) {
        double mx = xy[2 * m], my = xy[2 * m + 1];
        if (!(mx >= 0 && mx < s->p.nx && my >= 0 && my < s->p.ny)) return -1;
        int c = orc_marker_stencil(s->p.delta_kernel, mx, my, xs, ys, ws);
        for (int q = 0; q < c; q++)
            if (xs[q] < 3 || xs[q] > s->p.nx - 4 || ys[q] < 3 || ys[q] > s->p.ny - 4) return -1;
    }
    free(s->mk);
    free(s->body_force);
    s->mk = (marker*)calloc(n > 0 ? n : 1, sizeof(marker));
    s->nmark = n;
    s->nbody = 0;
    for (int m = 0; m < n; m++) {
        marker* k = &s->mk[m];
        k->x = xy[2 * m];
        k->y = xy[2 * m + 1];
        k->ubx = ub ? ub[2 * m] : 0.0;
        k->uby = ub ? ub[2 * m + 1] : 0.0;
        k->ds = ds ? ds[m] : 1.0;
        k->body = body ? body[m] : 0;
        if (k->body + 1 > s->nbody) s->nbody = k->body + 1;
    }
    s->body_force = (double*)calloc(2 * (s->nbody > 0 ? s->nbody : 1), sizeof(double));
    return 0;
}

int orc_num_bodies(orc* s) { return s->nbody; }

/* ---------------------------------------------------------------------- */
/* step phases                                                             */
/* ---------------------------------------------------------------------- */

/* Mesh::NNmodel_TypeXX: neighbour lists of mesh.cpp:2788-2804 (03),
 * 2854-2870 (07), 2915-2924 (00), 2974-2983 (02), 3032-3041 (04),
 * 3088-3097 (06), 3149-3165 (01), 3216-3232 (05); call order of
 * mesh.cpp:364-379: 00 01 02 04 05 06 03 07. */
static void nn_eval(orc* s, int type, int i, int j, const int nb[][2], int nnb)
{
    float in[15];
    for (int q = 0; q < nnb; q++) {
        size_t id = ID(s, nb[q][0], nb[q][1]);
        in[3 * q + 0] = (float)s->ux[id];
        in[3 * q + 1] = (float)s->uy[id];
        in[3 * q + 2] = (float)s->rho[id];
    }
    double NN_Tau = (double)orc_band_forward(s->nets[type].w, s->nets[type].nin, in);
    size_t id = ID(s, i, j);
    if (NN_Tau >= 0.501) {
        s->tau[id] = NN_Tau;
        s->nnflag[id] = 1;
    } else {
        s->nnflag[id] = 0;
    }
}

static void nn_band(orc* s)
{
    int NX = s->NX, Ny = s->NY;
    static const int order[8] = {0, 1, 2, 4, 5, 6, 3, 7};
    for (int oi = 0; oi < 8; oi++) {
        int t = order[oi];
        if (!s->nets[t].w) continue;
        int nb[5][2];
        switch (t) {
        case 0: {
            int a[3][2] = {{1, 1}, {2, 1}, {2, 0}};
            memcpy(nb, a, sizeof a);
            nn_eval(s, t, 1, 0, (const int(*)[2])nb, 3);
        } break;
        case 2: {
            int j = Ny - 1;
            int a[3][2] = {{1, j - 1}, {2, j - 1}, {2, j}};
            memcpy(nb, a, sizeof a);
            nn_eval(s, t, 1, j, (const int(*)[2])nb, 3);
        } break;
        case 4: {
            int i = NX - 2, j = Ny - 1;
            int a[3][2] = {{i - 1, j}, {i - 1, j - 1}, {i, j - 1}};
            memcpy(nb, a, sizeof a);
            nn_eval(s, t, i, j, (const int(*)[2])nb, 3);
        } break;
        case 6: {
            int i = NX - 2;
            int a[3][2] = {{i, 1}, {i - 1, 1}, {i - 1, 0}};
            memcpy(nb, a, sizeof a);
            nn_eval(s, t, i, 0, (const int(*)[2])nb, 3);
        } break;
        case 1:
            for (int j = 1; j < Ny - 1; j++) {
                int i = 1;
                int a[5][2] = {{i, j + 1}, {i + 1, j + 1}, {i + 1, j}, {i + 1, j - 1}, {i, j - 1}};
                nn_eval(s, t, i, j, (const int(*)[2])a, 5);
            }
            break;
        case 5:
            for (int j = 1; j < Ny - 1; j++) {
                int i = NX - 2;
                int a[5][2] = {{i, j + 1}, {i - 1, j + 1}, {i - 1, j}, {i - 1, j - 1}, {i, j - 1}};
                nn_eval(s, t, i, j, (const int(*)[2])a, 5);
            }
            break;
        case 3:
            for (int i = 1; i < NX - 1; i++) {
                int j = Ny - 2;
                int a[5][2] = {{i + 1, j}, {i + 1, j - 1}, {i, j - 1}, {i - 1, j - 1}, {i - 1, j}};
                nn_eval(s, t, i, j, (const int(*)[2])a, 5);
            }
            break;
        case 7:
            for (int i = 1; i < NX - 1; i++) {
                int j = 1;
                int a[5][2] = {{i - 1, j}, {i - 1, j + 1}, {i, j + 1}, {i + 1, j + 1}, {i + 1, j}};
                nn_eval(s, t, i, j, (const int(*)[2])a, 5);
            }
            break;
        }
    }
}

/* IB sub-step: InterpolateVel -> CalParticleForce -> SpreadForce ->
 * UpdateVelocity (mesh.cpp:552-655, 514-551, 656-832, 1244-1281), with
 * mdf_iters > 1 repeating it on the corrected velocity (multi-direct forcing)
 * and accumulating the marker and node forces. */
static void ib_substep(orc* s)
{
    if (s->nmark == 0) return;
    size_t n = (size_t)s->NX * s->NY;
    memset(s->fxn, 0, n * sizeof(double));
    memset(s->fyn, 0, n * sizeof(double));
    for (int m = 0; m < s->nmark; m++) s->mk[m].fx = s->mk[m].fy = 0;
    double* dfx = (double*)calloc(n, sizeof(double));
    double* dfy = (double*)calloc(n, sizeof(double));
    double* mfx = (double*)calloc(s->nmark, sizeof(double));
    double* mfy = (double*)calloc(s->nmark, sizeof(double));
    int xs[16], ys[16];
    double wa[16], wb[16];
    for (int it = 0; it < s->p.mdf_iters; it++) {
        for (int m = 0; m < s->nmark; m++) {
            marker* k = &s->mk[m];
            int c = marker_stencil2(s->p.delta_kernel, k->x, k->y, xs, ys, wa, wb);
            double vx = 0, vy = 0;
            for (int q = 0; q < c; q++) {
                size_t id = ID(s, xs[q] + 1, ys[q]);
                vx += (s->ux[id] * wa[q] * wb[q]);
                vy += (s->uy[id] * wa[q] * wb[q]);
            }
            k->vref_x = vx;
            k->vref_y = vy;
            mfx[m] = 2 * (k->ubx - k->vref_x);
            mfy[m] = 2 * (k->uby - k->vref_y);
            k->fx += mfx[m];
            k->fy += mfy[m];
        }
        memset(dfx, 0, n * sizeof(double));
        memset(dfy, 0, n * sizeof(double));
        for (int m = 0; m < s->nmark; m++) {
            marker* k = &s->mk[m];
            int c = marker_stencil2(s->p.delta_kernel, k->x, k->y, xs, ys, wa, wb);
            for (int q = 0; q < c; q++) {
                size_t id = ID(s, xs[q] + 1, ys[q]);
                dfx[id] += (mfx[m] * wa[q] * wb[q]);
                dfy[id] += (mfy[m] * wa[q] * wb[q]);
            }
        }
        /* UpdateVelocity for one rank: local i = 2 .. NX-2 (mesh.cpp:1250-1256) */
#pragma omp parallel for schedule(static)
        for (int i = 2; i < s->NX - 1; i++)
            for (int j = 0; j < s->NY; j++) {
                size_t id = ID(s, i, j);
                if (dfx[id] == 0.0 && dfy[id] == 0.0) continue;
                s->ux[id] = s->ux[id] + 0.5 * 1 * dfx[id] / s->rho[id];
                s->uy[id] = s->uy[id] + 0.5 * 1 * dfy[id] / s->rho[id];
                s->fxn[id] += dfx[id];
                s->fyn[id] += dfy[id];
            }
    }
    for (int b = 0; b < s->nbody; b++) s->body_force[2 * b] = s->body_force[2 * b + 1] = 0;
    for (int m = 0; m < s->nmark; m++) {
        marker* k = &s->mk[m];
        s->body_force[2 * k->body] -= k->fx * k->ds;
        s->body_force[2 * k->body + 1] -= k->fy * k->ds;
    }
    free(dfx); free(dfy); free(mfx); free(mfy);
}

/* Collision loop of OneLBMStep (mesh.cpp:386-402 SRT, 413-423 RR, 426-437 MRT);
 * returns -3 if ErrorCatch fired. */
static int collide_all(orc* s)
{
    int err = 0;
    int coll = s->p.collision;
    mrt_tables();
    /* every node's collision reads only its own state (and, for the gradient
     * closures, neighbour velocities nothing here writes): the columns run in
     * parallel with the same arithmetic per node */
#pragma omp parallel for schedule(static) reduction(min : err)
    for (int i = 1; i < s->NX - 1; ++i)
        for (int j = 0; j < s->NY; ++j) {
            size_t id = ID(s, i, j);
            double r = s->rho[id];
            if (coll != COLL_RR && (r > 10 || r < 0)) err = -3;
            if (r != r) err = -3;
            double fn[9], fc[9];
            for (int k = 0; k < 9; k++) fn[k] = FN(s, k, i, j);
            int use_les = s->p.les_model == 1 && !(coll == COLL_BGK && s->nnflag[id]);
            if (s->solid && s->solid[id])
                s->tau[id] = s->p.tau0;
            else if (s->p.les_model >= 4)
                s->tau[id] = ext_tau(s, i, j, fn, r, s->ux[id], s->uy[id]);
            else if (s->p.les_model == 3 && !(coll == COLL_BGK && s->nnflag[id]))
                s->tau[id] = s->tau_field[(size_t)j * s->p.nx + (i - 1)];
            else if (s->p.les_model == 2)
                s->tau[id] = orc_learned_tau(fn, r, s->ux[id], s->uy[id], s->p.tau0, s->p.cs, s->mlp);
            else if (use_les)
                s->tau[id] = orc_les_tau(fn, r, s->ux[id], s->uy[id], s->p.tau0, s->p.cs);
            else if (!(coll == COLL_BGK && s->nnflag[id]))
                s->tau[id] = s->p.tau0;
            orc_collide_node(coll, fn, r, s->ux[id], s->uy[id], s->tau[id], fc);
            if (s->nmark > 0) {
                double lf[9];
                force_term(coll, s->ux[id], s->uy[id], s->fxn[id], s->fyn[id], s->p.tau0, s->tau[id], lf);
                for (int k = 0; k < 9; k++) fc[k] += lf[k];
            }
            for (int k = 0; k < 9; k++) FC(s, k, i, j) = fc[k];
        }
    return err;
}

/* Single-rank halo exchange of mesh.cpp:440-499 (periodic ring). */
static void halo_exchange(orc* s)
{
    int NX = s->NX;
    for (int j = 0; j < s->NY; j++) {
        for (int k = 0; k < 9; k++) {
            FC(s, k, 0, j) = FC(s, k, NX - 2, j);
            FC(s, k, NX - 1, j) = FC(s, k, 1, j);
        }
        size_t L = ID(s, 0, j), R = ID(s, NX - 1, j);
        size_t a = ID(s, NX - 2, j), b = ID(s, 1, j);
        s->ux[L] = s->ux[a]; s->uy[L] = s->uy[a]; s->rho[L] = s->rho[a];
        s->ux[R] = s->ux[b]; s->uy[R] = s->uy[b]; s->rho[R] = s->rho[b];
    }
}

/* Mesh::Streaming (mesh.cpp:192-226). */
static void streaming_ref(orc* s)
{
#pragma omp parallel for schedule(static)
    for (int i = 1; i < s->NX - 1; i++)
        for (int j = 1; j < s->NY - 1; j++) {
            if (s->style[ID(s, i, j)] != 'f') continue;
            double f[9];
            for (int k = 0; k < 9; k++) {
                f[k] = FC(s, k, i - E[k][0], j - E[k][1]);
                FN(s, k, i, j) = f[k];
            }
            size_t id = ID(s, i, j);
            cal_macro(f, &s->rho[id], &s->ux[id], &s->uy[id]);
        }
}

static void nee_node(orc* s, int i, int j, int ni, int nj)
{
    /* fnew(i,j) = feq(i,j) + fnew(ni,nj) - feq(ni,nj), mesh.cpp:245-249 etc. */
    double fa[9], fb[9];
    size_t a = ID(s, i, j), b = ID(s, ni, nj);
    compute_feq(s->rho[a], s->ux[a], s->uy[a], fa);
    compute_feq(s->rho[b], s->ux[b], s->uy[b], fb);
    for (int k = 0; k < 9; k++) FN(s, k, i, j) = fa[k] + FN(s, k, ni, nj) - fb[k];
}

/* Mesh::BoundaryCondition (mesh.cpp:228-356), one rank; u_in replaces the
 * hard-coded inlet velocity 0.1 of mesh.cpp:244. */
static void boundary_ref(orc* s)
{
    int Nx = s->NX, Ny = s->NY;
    for (int j = 1; j < Ny - 1; j++) {
        size_t id = ID(s, 1, j);
        s->rho[id] = 1.0;
        s->ux[id] = s->p.u_in;
        s->uy[id] = 0.0;
        nee_node(s, 1, j, 2, j);
    }
    for (int j = 1; j < Ny - 1; j++) {
        size_t id = ID(s, Nx - 2, j), nb = ID(s, Nx - 3, j);
        s->rho[id] = 1.0;
        s->ux[id] = s->ux[nb];
        s->uy[id] = s->uy[nb];
        nee_node(s, Nx - 2, j, Nx - 3, j);
    }
    for (int i = 1; i < Nx - 1; i++) {
        size_t id = ID(s, i, Ny - 1), nb = ID(s, i, Ny - 2);
        s->rho[id] = 1.0;
        s->ux[id] = s->ux[nb];
        s->uy[id] = s->uy[nb];
        nee_node(s, i, Ny - 1, i, Ny - 2);
    }
    for (int i = 1; i < Nx - 1; i++) {
        int j = 0;
        size_t id = ID(s, i, j);
        if (s->style[id] == 'm') {
            double f[9];
            f[0] = FC(s, 0, i, j);
            f[1] = FC(s, 1, i - 1, j);
            f[2] = FC(s, 4, i, j + 1);
            f[3] = FC(s, 3, i + 1, j);
            f[4] = FC(s, 4, i, j + 1);
            f[5] = FC(s, 8, i - 1, j + 1);
            f[6] = FC(s, 7, i + 1, j + 1);
            f[7] = FC(s, 7, i + 1, j + 1);
            f[8] = FC(s, 8, i - 1, j + 1);
            for (int k = 0; k < 9; k++) FN(s, k, i, j) = f[k];
            cal_macro(f, &s->rho[id], &s->ux[id], &s->uy[id]);
        }
        if (s->style[id] == 'd') {
            s->rho[id] = s->rho[ID(s, i, j + 1)];
            s->ux[id] = 0.0;
            s->uy[id] = 0.0;
            nee_node(s, i, j, i, j + 1);
        }
    }
}

/* Channel scene (no reference code for it): pull streaming with halfway
 * bounce-back on the y walls and a parabolic Zou-He velocity inlet at x = 0
 * (regularised);
 * those nodes then take their moments (CalMacro).  The outlet x = nx-1 is the
 * reference's outlet (mesh.cpp:273-286): rho = rho0, u copied from x = nx-2,
 * populations by non-equilibrium extrapolation from x = nx-2. */
static double inlet_profile(const orc* s, int y)
{
    double H = (double)s->p.ny;
    double yy = (double)y + 0.5;
    return 4.0 * s->p.u_in * yy * (H - yy) / (H * H);
}

static void streaming_channel(orc* s)
{
    int nx = s->p.nx, ny = s->p.ny;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx - 1; x++)
        for (int y = 0; y < ny; y++) {
            int i = x + 1;
            double f[9];
            if (s->solid && s->solid[ID(s, i, y)]) {
                /* a solid node: not updated, reads as fluid at rest */
                size_t id = ID(s, i, y);
                for (int k = 0; k < 9; k++) FN(s, k, i, y) = W[k] * s->p.rho0;
                s->rho[id] = s->p.rho0;
                s->ux[id] = s->uy[id] = 0.0;
                continue;
            }
            for (int k = 0; k < 9; k++) {
                int sx = x - E[k][0], sy = y - E[k][1];
                if (sy < 0 || sy >= ny)
                    f[k] = FC(s, OPP[k], i, y);
                else if (sx < 0)
                    f[k] = 0.0; /* replaced by Zou-He below */
                else if (s->solid && s->solid[ID(s, sx + 1, sy)])
                    f[k] = FC(s, OPP[k], i, y); /* halfway bounce-back on the solid */
                else
                    f[k] = FC(s, k, sx + 1, sy);
            }
            if (x == 0) {
                /* Zou-He density and unknowns, then the regularised
                 * reconstruction (Latt & Chopard 2008): equilibrium at
                 * (rho, u_in, 0) plus the second-order projection of the
                 * non-equilibrium part.  Plain Zou-He with BGK diverges at
                 * tau = 0.53 in a 400 x 100 channel; this form does not. */
                double ux = inlet_profile(s, y);
                double rho = (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7])) / (1.0 - ux);
                f[1] = f[3] + (2.0 / 3.0) * rho * ux;
                f[5] = f[7] - 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * rho * ux;
                f[8] = f[6] + 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * rho * ux;
                double fe[9], pxx = 0.0, pxy = 0.0, pyy = 0.0;
                compute_feq(rho, ux, 0.0, fe);
                for (int k = 0; k < 9; k++) {
                    pxx += E[k][0] * E[k][0] * (f[k] - fe[k]);
                    pxy += E[k][0] * E[k][1] * (f[k] - fe[k]);
                    pyy += E[k][1] * E[k][1] * (f[k] - fe[k]);
                }
                for (int k = 0; k < 9; k++) {
                    double qxx = E[k][0] * E[k][0] - 1.0 / 3.0, qyy = E[k][1] * E[k][1] - 1.0 / 3.0;
                    double qxy = E[k][0] * E[k][1];
                    f[k] = fe[k] + 4.5 * W[k] * (qxx * pxx + 2.0 * qxy * pxy + qyy * pyy);
                }
            }
            size_t id = ID(s, i, y);
            for (int k = 0; k < 9; k++) FN(s, k, i, y) = f[k];
            cal_macro(f, &s->rho[id], &s->ux[id], &s->uy[id]);
        }
    for (int y = 0; y < ny; y++) {
        size_t id = ID(s, nx, y), nb = ID(s, nx - 1, y);
        s->rho[id] = s->p.rho0;
        s->ux[id] = s->ux[nb];
        s->uy[id] = s->uy[nb];
        nee_node(s, nx, y, nx - 1, y);
    }
}

/* Mesh::ComputeAvgVelocity (mesh.cpp:1954-1974). */
static void average(orc* s, int t)
{
    if (t < s->p.avg_start) return;
    double a = (double)(t - s->p.avg_start), b = (double)(t - s->p.avg_start + 1);
    size_t n = (size_t)s->NX * s->NY;
#pragma omp parallel for schedule(static)
    for (size_t id = 0; id < n; id++) {
        if (s->solid && s->solid[id]) continue;
        s->avg_u[id] = (s->avg_u[id] * a + s->ux[id]) / b;
        s->avg_v[id] = (s->avg_v[id] * a + s->uy[id]) / b;
        s->avg_rho[id] = (s->avg_rho[id] * a + s->rho[id]) / b;
    }
}

static void update_mass(orc* s)
{
    double m = 0.0;
    for (int y = 0; y < s->p.ny; y++)
        for (int x = 0; x < s->p.nx; x++) m += s->rho[ID(s, x + 1, y)];
    s->mass = m;
}

int orc_step(orc* s, int nsteps, int t0)
{
    int status = 0;
    if (s->p.les_model == 2 && !s->mlp_loaded) return -1;
    if (s->p.les_model == 3 && !s->tau_field) return -1;
    if (s->p.les_model == 6 && !s->wall_dist) return -1;
    for (int t = t0; t < t0 + nsteps; t++) {
        ib_substep(s);
        if (s->p.collision == COLL_BGK) nn_band(s);
        int e = collide_all(s);
        if (e) status = e;
        halo_exchange(s);
        if (s->p.bc_set == BC_REF) {
            streaming_ref(s);
            boundary_ref(s);
        } else {
            streaming_channel(s);
        }
        average(s, t);
    }
    update_mass(s);
    return status;
}

/* Relaxation time of the next collision, for every node: the net's tau where
 * its flag would be set, else Smagorinsky (or tau0).  Pure: runs the NN band
 * and the LES on a copy of tau/nnflag and the current (t) state. */
static void next_tau(orc* s, double* tau_out, unsigned char* flag_out)
{
    size_t n = (size_t)s->NX * s->NY;
    double* tsave = (double*)malloc(n * sizeof(double));
    unsigned char* fsave = (unsigned char*)malloc(n);
    memcpy(tsave, s->tau, n * sizeof(double));
    memcpy(fsave, s->nnflag, n);
    /* the IB correction changes u of forced nodes before the collision */
    double* uxs = (double*)malloc(n * sizeof(double));
    double* uys = (double*)malloc(n * sizeof(double));
    double* fxs = (double*)malloc(n * sizeof(double));
    double* fys = (double*)malloc(n * sizeof(double));
    memcpy(uxs, s->ux, n * sizeof(double));
    memcpy(uys, s->uy, n * sizeof(double));
    memcpy(fxs, s->fxn, n * sizeof(double));
    memcpy(fys, s->fyn, n * sizeof(double));
    double* bfs = (double*)malloc(2 * (s->nbody + 1) * sizeof(double));
    if (s->nbody) memcpy(bfs, s->body_force, 2 * s->nbody * sizeof(double));
    ib_substep(s);
    if (s->p.collision == COLL_BGK) nn_band(s);
    for (int i = 1; i < s->NX - 1; i++)
        for (int j = 0; j < s->NY; j++) {
            size_t id = ID(s, i, j);
            double fn[9];
            for (int k = 0; k < 9; k++) fn[k] = FN(s, k, i, j);
            double t;
            int nnf = (s->p.collision == COLL_BGK) && s->nnflag[id];
            if (s->solid && s->solid[id])
                t = s->p.tau0; /* a solid node reads as fluid at rest */
            else if (nnf)
                t = s->tau[id];
            else if (s->p.les_model >= 4)
                t = ext_tau(s, i, j, fn, s->rho[id], s->ux[id], s->uy[id]);
            else if (s->p.les_model == 3)
                t = s->tau_field[(size_t)j * s->p.nx + (i - 1)];
            else if (s->p.les_model == 2)
                t = orc_learned_tau(fn, s->rho[id], s->ux[id], s->uy[id], s->p.tau0, s->p.cs, s->mlp);
            else if (s->p.les_model == 1)
                t = orc_les_tau(fn, s->rho[id], s->ux[id], s->uy[id], s->p.tau0, s->p.cs);
            else
                t = s->p.tau0;
            size_t g = (size_t)j * s->p.nx + (i - 1);
            if (tau_out) tau_out[g] = t;
            if (flag_out) flag_out[g] = (unsigned char)nnf;
        }
    memcpy(s->tau, tsave, n * sizeof(double));
    memcpy(s->nnflag, fsave, n);
    memcpy(s->ux, uxs, n * sizeof(double));
    memcpy(s->uy, uys, n * sizeof(double));
    memcpy(s->fxn, fxs, n * sizeof(double));
    memcpy(s->fyn, fys, n * sizeof(double));
    if (s->nbody) memcpy(s->body_force, bfs, 2 * s->nbody * sizeof(double));
    free(tsave); free(fsave); free(uxs); free(uys); free(fxs); free(fys); free(bfs);
}

void orc_get(orc* s, int field, double* out)
{
    int nx = s->p.nx, ny = s->p.ny;
    size_t plane = (size_t)nx * ny;
    if (field == ORC_TAU || field == ORC_NNFLAG) {
        if (field == ORC_TAU) {
            next_tau(s, out, NULL);
        } else {
            unsigned char* fl = (unsigned char*)malloc(plane);
            next_tau(s, NULL, fl);
            for (size_t g = 0; g < plane; g++) out[g] = fl[g];
            free(fl);
        }
        return;
    }
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            size_t id = ID(s, x + 1, y), g = (size_t)y * nx + x;
            switch (field) {
            case ORC_F:
                for (int k = 0; k < 9; k++) out[k * plane + g] = FN(s, k, x + 1, y);
                break;
            case ORC_RHO: out[g] = s->rho[id]; break;
            case ORC_UX: out[g] = s->ux[id]; break;
            case ORC_UY: out[g] = s->uy[id]; break;
            case ORC_AVG_U: out[g] = s->avg_u[id]; break;
            case ORC_AVG_V: out[g] = s->avg_v[id]; break;
            case ORC_AVG_RHO: out[g] = s->avg_rho[id]; break;
            case ORC_FLAGS: out[g] = (double)(unsigned char)s->style[id]; break;
            default: out[g] = 0; break;
            }
        }
}

/* Body forces of an IB sub-step evaluated on the current velocity field
 * (the forces the next collision will apply); the state is left untouched. */
int orc_forces(orc* s, double* force_xy, double* mass)
{
    if (force_xy && s->nmark > 0) {
        size_t n = (size_t)s->NX * s->NY;
        double* sv[4] = {s->ux, s->uy, s->fxn, s->fyn};
        double* cp[4];
        for (int q = 0; q < 4; q++) {
            cp[q] = (double*)malloc(n * sizeof(double));
            memcpy(cp[q], sv[q], n * sizeof(double));
        }
        ib_substep(s);
        for (int b = 0; b < 2 * s->nbody; b++) force_xy[b] = s->body_force[b];
        for (int q = 0; q < 4; q++) {
            memcpy(sv[q], cp[q], n * sizeof(double));
            free(cp[q]);
        }
    }
    if (mass) {
        update_mass(s);
        *mass = s->mass;
    }
    return s->nbody;
}

void orc_ib_probe(orc* s, double* vref, double* mforce, double* nforce)
{
    ib_substep(s);
    for (int m = 0; m < s->nmark; m++) {
        if (vref) { vref[2 * m] = s->mk[m].vref_x; vref[2 * m + 1] = s->mk[m].vref_y; }
        if (mforce) { mforce[2 * m] = s->mk[m].fx; mforce[2 * m + 1] = s->mk[m].fy; }
    }
    if (nforce) {
        size_t plane = (size_t)s->p.nx * s->p.ny;
        for (int y = 0; y < s->p.ny; y++)
            for (int x = 0; x < s->p.nx; x++) {
                size_t id = ID(s, x + 1, y), g = (size_t)y * s->p.nx + x;
                nforce[g] = s->fxn[id];
                nforce[plane + g] = s->fyn[id];
            }
    }
}

/* ---------------------------------------------------------------------- */
/* Implicit tau inference: Mesh::FindAndWriteTau (mesh.cpp:2625-2715).    */
/* ---------------------------------------------------------------------- */
/* For a node (x, y) and target moments (R, U, V): for m = m_lo .. m_hi,
 * dtau = m * step, relax each upstream neighbour (x - e_k, y - e_k) with
 * BGK at tau + dtau -- fcol_k = (1 - 1/(tau + dtau)) fnew_k + feq_k/(tau +
 * dtau) -- and stream it into (x, y); the candidate's error is
 * |sum f - R| + |sum f e_x - U| + |sum f e_y - V| (momentum against the
 * target velocity, as mesh.cpp:2675-2681 does).  The first minimum wins
 * (strict <).  f [9][ny][nx] are the post-stream populations, m3 [3][ny][nx]
 * their rho, ux, uy (feq is Compute_feq of those), tau [ny][nx]. */
void orc_tau_scan_state(const double* f, const double* m3, const double* tau, int nx, int ny,
                        int n, const int* xy, const double* target, int m_lo, int m_hi,
                        double step, double* best_dtau, double* best_err)
{
    size_t nn = (size_t)nx * ny;
    for (int q = 0; q < n; q++) {
        int x = xy[2 * q], y = xy[2 * q + 1];
        double fn[9], fe[9], tn[9];
        for (int k = 0; k < 9; k++) {
            /* the neighbour whose population k streams into (x, y) */
            size_t g = (size_t)(y - E[k][1]) * nx + (x - E[k][0]);
            double feq[9];
            compute_feq(m3[g], m3[nn + g], m3[2 * nn + g], feq);
            fn[k] = f[k * nn + g];
            fe[k] = feq[k];
            tn[k] = tau[g];
        }
        double R = target[3 * q], U = target[3 * q + 1], V = target[3 * q + 2];
        double bestDeltaTau = 1e10, bestABS = 1e10;
        for (int mm = m_lo; mm <= m_hi; mm++) {
            double deltaTau = (double)mm * step;
            double trho = 0, tu = 0, tv = 0;
            for (int k = 0; k < 9; k++) {
                double c = (1.0 - 1.0 / (tn[k] + deltaTau)) * fn[k] + fe[k] / (tn[k] + deltaTau);
                trho += c;
                tu += c * E[k][0];
                tv += c * E[k][1];
            }
            double TargetAbs = fabs(trho - R) + fabs(tu - U) + fabs(tv - V);
            if (TargetAbs < bestABS) {
                bestABS = TargetAbs;
                bestDeltaTau = deltaTau;
            }
        }
        best_dtau[q] = bestDeltaTau;
        best_err[q] = bestABS;
    }
}

int orc_set_solid(orc* s, const unsigned char* solid)
{
    free(s->solid);
    s->solid = NULL;
    if (solid) {
        int nx = s->p.nx, ny = s->p.ny;
        s->solid = (unsigned char*)calloc((size_t)s->NX * s->NY, 1);
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                if (!solid[(size_t)y * nx + x]) continue;
                if (s->p.bc_set != BC_CHANNEL || x < 3 || x > nx - 4 || y < 3 || y > ny - 4) {
                    free(s->solid);
                    s->solid = NULL;
                    judge_style(s);
                    return -1;
                }
                s->solid[ID(s, x + 1, y)] = 1;
            }
    }
    judge_style(s);
    return 0;
}

/* Mesh::OutputCd (mesh.cpp:1461-1488): sum over 'b' nodes, i then j, and
 * every k whose neighbour is 's' of e_k (fnew_opp(k) + fcol_k); fcol is the
 * collision whose streaming produced the current fnew. */
void orc_solid_force(orc* s, double* force_xy)
{
    double fx = 0.0, fy = 0.0;
    for (int i = 1; i < s->NX - 1; i++)
        for (int j = 1; j < s->NY - 1; j++) {
            if (s->style[ID(s, i, j)] != 'b') continue;
            for (int k = 0; k < 9; k++) {
                int ip = i + E[k][0], jp = j + E[k][1];
                if (s->style[ID(s, ip, jp)] == 's') {
                    fx += E[k][0] * (FN(s, OPP[k], i, j) + FC(s, k, i, j));
                    fy += E[k][1] * (FN(s, OPP[k], i, j) + FC(s, k, i, j));
                }
            }
        }
    force_xy[0] = fx;
    force_xy[1] = fy;
}
