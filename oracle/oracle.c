/*
 * oracle.c -- FP64 CPU restatement of the reference NNP hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  The product never calls this.
 *
 * Each routine follows the cited reference function operation by operation
 * (same association of + and *, same loop order) so that, compiled without
 * FMA contraction, it reproduces the reference compiled the same way.
 * Parity: pinned against the reference's own sources through tests/golden/.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* math/const.hpp:8-15 */
#define ORC_ZERO 1e-12
#define ORC_PI 3.141592653589793
#define ORC_RADPI 1.772453850905516
#define ORC_RAD2 1.414213562373095
#define ORC_LOG2 0.693147180559945

/* ------------------------------------------------------------------------ */
/* special functions                                                          */
/* ------------------------------------------------------------------------ */

/* Pade exp2 of the reference (math/special.cpp:235-274): 2^floor(x+.5) by
 * setting the IEEE exponent, times a (2,3) Pade of 2^f on [-.5,.5). */
static double orc_exp2(double x)
{
    static const double q[2] = {2.33184211722314911771e2, 4.36821166879210612817e3};
    static const double p[3] = {2.30933477057345225087e-2, 2.02020656693165307700e1,
                                1.51390680115615096133e3};
    union { double f; uint64_t u; struct { int32_t i0, i1; } s; } ep;
    const double ipart = floor(x + 0.5);
    const double fpart = x - ipart;
    ep.s.i0 = 0;
    ep.s.i1 = (((int)ipart) + 1023) << 20;
    x = fpart * fpart;
    double px = p[0];
    px = px * x + p[1];
    double qx = x + q[0];
    px = px * x + p[2];
    qx = qx * x + q[1];
    px = px * fpart;
    x = 1.0 + 2.0 * (px / (qx - px));
    return ep.f * x;
}

#define ORC_LOG2OFE 1.4426950408889634074
/* math/special.cpp:276-284 */
double orc_fmexp(double x)
{
    if (x < -1022.0 / ORC_LOG2OFE) return 0;
    if (x > 1023.0 / ORC_LOG2OFE) return INFINITY;
    return orc_exp2(ORC_LOG2OFE * x);
}

/* Taylor series of cos/sin about pi/2 (math/special.cpp:21-41) */
double orc_coscut(double x)
{
    x -= 0.5 * ORC_PI;
    const double x2 = x * x;
    return x * (-1.0 + x2 * (1.0 / 6.0 + x2 * (-1.0 / 120.0 + x2 * (1.0 / 5040.0 + x2 * (-1.0 / 362880.0 +
           x2 * (1.0 / 39916800.0 + x2 * (-1.0 / 6227020800.0 + x2 * 1.0 / 1307674368000.0)))))));
}

double orc_sincut(double x)
{
    x -= 0.5 * ORC_PI;
    const double x2 = x * x;
    return 1.0 + x2 * (-1.0 / 2.0 + x2 * (1.0 / 24.0 + x2 * (-1.0 / 720.0 + x2 * (1.0 / 40320.0 +
           x2 * (-1.0 / 3628800.0 + x2 * (1.0 / 479001600.0 + x2 * (-1.0 / 87178291200.0 +
           x2 * 1.0 / 20922789888000.0)))))));
}

/* math/special.cpp:139-148 */
static double orc_powint(double x, const int n)
{
    double yy, ww;
    if (n == 0) return 1.0;
    if (x == 0.0) return 0.0;
    int nn = (n > 0) ? n : -n;
    ww = x;
    for (yy = 1.0; nn != 0; nn >>= 1, ww *= ww)
        if (nn & 1) yy *= ww;
    return (n > 0) ? yy : 1.0 / yy;
}

/* ------------------------------------------------------------------------ */
/* cutoff (nnp/cutoff.cpp:50-114); rci = 1/rc and pirci = PI/rc as in the    */
/* constructor (cutoff.cpp:55-56)                                            */
/* ------------------------------------------------------------------------ */

double orc_cutf(int cut, double rc, double dr)
{
    const double rci = 1.0 / rc, pirci = ORC_PI / rc;
    switch (cut) {
    case ORC_CUT_STEP: return (dr < rc) ? 1.0 : 0.0;
    case ORC_CUT_COS: return (dr < rc) ? 0.5 * (orc_coscut(dr * pirci) + 1.0) : 0.0;
    case ORC_CUT_TANH: { const double f = (dr > rc) ? 0.0 : tanh(1.0 - dr * rci); return f * f * f; }
    case ORC_CUT_POLY3:
        if (dr < rc) { dr *= rci; return (2.0 * dr - 3.0) * dr * dr + 1.0; }
        return 0;
    default: return NAN;
    }
}

double orc_cutg(int cut, double rc, double dr)
{
    const double rci = 1.0 / rc, pirci = ORC_PI / rc;
    switch (cut) {
    case ORC_CUT_STEP: return 0.0;
    case ORC_CUT_COS: return (dr < rc) ? -0.5 * pirci * orc_sincut(dr * pirci) : 0.0;
    case ORC_CUT_TANH:
        if (dr < rc) { const double f = tanh(1.0 - dr * rci); return -3.0 * f * f * (1.0 - f * f) * rci; }
        return 0;
    case ORC_CUT_POLY3:
        if (dr < rc) { dr *= rci; return 6.0 * dr * (dr - 1.0) * rci; }
        return 0;
    default: return NAN;
    }
}

/* ------------------------------------------------------------------------ */
/* radial basis (nnp/basis_radial.cpp)                                        */
/* ------------------------------------------------------------------------ */

/* BasisR::symm (basis_radial.cpp:263-309) */
static void orc_basisR_symm(const orc_pot *p, int b, double dr, double *out)
{
    const int n = p->r_n[b];
    const double *rs = p->r_rs + p->r_off[b], *eta = p->r_eta + p->r_off[b];
    const double cutf = orc_cutf(p->r_cut[b], p->r_rc[b], dr);
    for (int i = 0; i < n; ++i) {
        switch (p->r_form[b]) {
        case ORC_R_GAUSSIAN: { const double arg = eta[i] * (dr - rs[i]); out[i] = orc_fmexp(-arg * arg) * cutf; } break;
        case ORC_R_SECH: { const double e = orc_fmexp(-eta[i] * (dr - rs[i])); out[i] = 2.0 * e / (1.0 + e * e) * cutf; } break;
        case ORC_R_LOGISTIC: { const double e = orc_fmexp(-2.0 * eta[i] * (dr - rs[i])); out[i] = 4.0 * e / ((1.0 + e) * (1.0 + e)) * cutf; } break;
        case ORC_R_TANH: out[i] = 0.5 * (tanh(-eta[i] * (dr - rs[i])) + 1.0) * cutf; break;
        case ORC_R_LOGCOSH: out[i] = 0.5 * log1p(orc_fmexp(-2.0 * eta[i] * (dr - rs[i]))) * cutf; break;
        case ORC_R_LOGCOSH2: {
            const double arg = -eta[i] * (dr - rs[i]);
            const double fexp = orc_fmexp(2.0 * ORC_RAD2 * arg);
            out[i] = (arg == 0.0) ? 0.5 * cutf / ORC_RAD2 : arg * fexp / (fexp - 1.0) * cutf;
        } break;
        default: out[i] = NAN;
        }
    }
}

/* BasisR::symmd (basis_radial.cpp:213-257): dG_i/dr per function */
static void orc_basisR_symmd(const orc_pot *p, int b, double dr, double *out)
{
    const int n = p->r_n[b];
    const double *rs = p->r_rs + p->r_off[b], *eta = p->r_eta + p->r_off[b];
    const double cutf = orc_cutf(p->r_cut[b], p->r_rc[b], dr);
    const double cutg = orc_cutg(p->r_cut[b], p->r_rc[b], dr);
    for (int i = 0; i < n; ++i) {
        switch (p->r_form[b]) {
        case ORC_R_GAUSSIAN: { const double arg = eta[i] * (dr - rs[i]); out[i] = orc_fmexp(-arg * arg) * (-2.0 * eta[i] * arg * cutf + cutg); } break;
        case ORC_R_SECH: {
            const double e = orc_fmexp(-eta[i] * (dr - rs[i])), e2 = e * e, den = 1.0 / (1.0 + e2);
            out[i] = 2.0 * e * den * (-1.0 * eta[i] * (1.0 - e2) * den * cutf + cutg);
        } break;
        case ORC_R_LOGISTIC: {
            const double e2 = orc_fmexp(-2.0 * eta[i] * (dr - rs[i])), den = 1.0 / (1.0 + e2);
            const double th = (1.0 - e2) * den, s2 = 4.0 * e2 * den * den;
            out[i] = s2 * (-2.0 * eta[i] * th * cutf + cutg);
        } break;
        case ORC_R_TANH: { const double th = tanh(-eta[i] * (dr - rs[i])); out[i] = 0.5 * (-eta[i] * (1.0 - th * th) * cutf + (1.0 + th) * cutg); } break;
        case ORC_R_LOGCOSH: { const double e = orc_fmexp(-2.0 * eta[i] * (dr - rs[i])); out[i] = -eta[i] * e / (1.0 + e) * cutf + 0.5 * log1p(e) * cutg; } break;
        case ORC_R_LOGCOSH2: {
            const double arg = -eta[i] * (dr - rs[i]);
            const double fexp = orc_fmexp(2.0 * ORC_RAD2 * arg), den = 1.0 / (fexp - 1.0);
            out[i] = (arg == 0.0) ? 0.5 * (-eta[i] * cutg + cutf / ORC_RAD2)
                                  : fexp * (eta[i] * (1.0 + 2.0 * ORC_RAD2 * arg - fexp) * den * cutf + arg * cutg) * den;
        } break;
        default: out[i] = NAN;
        }
    }
}

/* BasisR::force (basis_radial.cpp:316-376): returns -sum_i dEdG_i dG_i/dr */
static double orc_basisR_force(const orc_pot *p, int b, double dr, const double *dEdG)
{
    const int n = p->r_n[b];
    const double *rs = p->r_rs + p->r_off[b], *eta = p->r_eta + p->r_off[b];
    const double cutf = orc_cutf(p->r_cut[b], p->r_rc[b], dr);
    const double cutg = orc_cutg(p->r_cut[b], p->r_rc[b], dr);
    double amp = 0;
    for (int i = 0; i < n; ++i) {
        switch (p->r_form[b]) {
        case ORC_R_GAUSSIAN: { const double arg = eta[i] * (dr - rs[i]); amp -= dEdG[i] * orc_fmexp(-arg * arg) * (-2.0 * eta[i] * arg * cutf + cutg); } break;
        case ORC_R_SECH: {
            const double e = orc_fmexp(-eta[i] * (dr - rs[i])), e2 = e * e, den = 1.0 / (1.0 + e2);
            amp -= dEdG[i] * 2.0 * e * den * (-eta[i] * (1.0 - e2) * den * cutf + cutg);
        } break;
        case ORC_R_LOGISTIC: {
            const double e2 = orc_fmexp(-2.0 * eta[i] * (dr - rs[i])), den = 1.0 / (1.0 + e2);
            const double th = (1.0 - e2) * den, s2 = 4.0 * e2 * den * den;
            amp -= dEdG[i] * s2 * (-2.0 * eta[i] * th * cutf + cutg);
        } break;
        case ORC_R_TANH: { const double th = tanh(-eta[i] * (dr - rs[i])); amp -= dEdG[i] * 0.5 * (-eta[i] * (1.0 - th * th) * cutf + (1.0 + th) * cutg); } break;
        case ORC_R_LOGCOSH: { const double e = orc_fmexp(-2.0 * eta[i] * (dr - rs[i])); amp -= dEdG[i] * (-eta[i] * e / (1.0 + e) * cutf + 0.5 * log1p(e) * cutg); } break;
        case ORC_R_LOGCOSH2: {
            const double arg = -eta[i] * (dr - rs[i]);
            const double fexp = orc_fmexp(2.0 * ORC_RAD2 * arg), den = 1.0 / (fexp - 1.0);
            const double val = (arg == 0.0) ? 0.5 * (-eta[i] * cutg + cutf / ORC_RAD2)
                                            : fexp * (eta[i] * (1.0 + 2.0 * ORC_RAD2 * arg - fexp) * den * cutf + arg * cutg) * den;
            amp -= dEdG[i] * val;
        } break;
        default: amp = NAN;
        }
    }
    return amp;
}

/* ------------------------------------------------------------------------ */
/* angular basis (nnp/basis_angular.cpp)                                      */
/* ------------------------------------------------------------------------ */

#define ORC_MAX_A 256
typedef struct {
    int n, ng;
    double ieta2[ORC_MAX_A], lambdaf[ORC_MAX_A], ietar2[ORC_MAX_A];
    int rflag[ORC_MAX_A];
} orc_agroups;

/* BasisA::init (basis_angular.cpp:178-205): adjacent functions whose eta
 * differ by < 1e-6 share one radial damping factor. */
static void orc_basisA_init(const orc_pot *p, int b, orc_agroups *g)
{
    const int n = p->a_n[b];
    const double *eta = p->a_eta + p->a_off[b];
    const int32_t *lam = p->a_lambda + p->a_off[b];
    double etar[ORC_MAX_A];
    g->n = n; g->ng = 0;
    for (int i = 0; i < n; ++i) {
        g->ieta2[i] = 1.0 / (eta[i] * eta[i]);
        g->lambdaf[i] = 0.5 * lam[i];
    }
    if (n > 0) {
        int flag = 0;
        g->rflag[0] = flag;
        etar[0] = eta[0];
        for (int i = 1; i < n; ++i) {
            if (fabs(eta[i] - eta[i - 1]) < 1.0e-6) g->rflag[i] = flag;
            else { g->rflag[i] = ++flag; etar[flag] = eta[i]; }
        }
        flag++;
        g->ng = flag;
        for (int i = 0; i < flag; ++i) g->ietar2[i] = 1.0 / (etar[i] * etar[i]);
    }
}

/* BasisA::symm (basis_angular.cpp:371-420) */
static void orc_basisA_symm(const orc_pot *p, int b, const orc_agroups *g, double rij, double rik,
                            double cs, double *out)
{
    const int n = g->n;
    const double *zeta = p->a_zeta + p->a_off[b];
    const int cut = p->a_cut[b];
    const double rc = p->a_rc[b];
    const double cprod = orc_cutf(cut, rc, rij) * orc_cutf(cut, rc, rik);
    const double r2s = rij * rij + rik * rik;
    double fd[ORC_MAX_A];
    switch (p->a_form[b]) {
    case ORC_A_GAUSS:
        for (int j = 0; j < g->ng; ++j) fd[j] = cprod * orc_fmexp(-g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) out[i] = pow(fabs(0.5 + g->lambdaf[i] * cs), zeta[i]) * fd[g->rflag[i]];
        break;
    case ORC_A_GAUSS2:
        for (int j = 0; j < g->ng; ++j) fd[j] = orc_fmexp(-0.5 * ORC_PI * g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i)
            out[i] = cprod * pow(fabs(0.5 + g->lambdaf[i] * cs), zeta[i]) * 2.0 * fd[g->rflag[i]] / (1.0 + fd[g->rflag[i]]);
        break;
    case ORC_A_SECH:
        for (int j = 0; j < g->ng; ++j) fd[j] = orc_fmexp(-0.5 * ORC_PI * g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) {
            const double fexp = fd[g->rflag[i]];
            out[i] = cprod * pow(fabs(0.5 + g->lambdaf[i] * cs), zeta[i]) * 2.0 * fexp / (1.0 + fexp * fexp);
        }
        break;
    case ORC_A_STUDENT3: case ORC_A_STUDENT4: case ORC_A_STUDENT5: {
        const int pw = 4 + (p->a_form[b] - ORC_A_STUDENT3);
        for (int j = 0; j < g->ng; ++j) fd[j] = cprod * orc_powint(1.0 / sqrt(1.0 + g->ietar2[j] * r2s), pw);
        for (int i = 0; i < n; ++i) out[i] = pow(fabs(0.5 + g->lambdaf[i] * cs), zeta[i]) * fd[g->rflag[i]];
    } break;
    default:
        for (int i = 0; i < n; ++i) out[i] = NAN;
    }
}

/* BasisA::force (basis_angular.cpp:430-563): phi and eta[2] */
static void orc_basisA_force(const orc_pot *p, int b, const orc_agroups *g, double rij, double rik,
                             double cs, double *phi, double *eta, const double *dEdG)
{
    const int n = g->n;
    const double *zeta = p->a_zeta + p->a_off[b];
    const int cut = p->a_cut[b];
    const double rc = p->a_rc[b];
    const double c[2] = {orc_cutf(cut, rc, rij), orc_cutf(cut, rc, rik)};
    const double gg[2] = {orc_cutg(cut, rc, rij), orc_cutg(cut, rc, rik)};
    double fd[ORC_MAX_A];
    *phi = 0; eta[0] = 0; eta[1] = 0;
    const double r2s = rij * rij + rik * rik;
    switch (p->a_form[b]) {
    case ORC_A_GAUSS: {
        const double dij = 2.0 * rij * c[0], dik = 2.0 * rik * c[1];
        for (int j = 0; j < g->ng; ++j) fd[j] = orc_fmexp(-g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) {
            const double cw = fabs(0.5 + g->lambdaf[i] * cs);
            const double gangle = dEdG[i] * pow(cw, zeta[i] - 1.0) * fd[g->rflag[i]];
            const double fangle = cw * gangle;
            *phi -= zeta[i] * g->lambdaf[i] * gangle;
            eta[0] -= fangle * (-dij * g->ieta2[i] + gg[0]);
            eta[1] -= fangle * (-dik * g->ieta2[i] + gg[1]);
        }
    } break;
    case ORC_A_GAUSS2: {
        const double dij = ORC_PI * rij * c[0], dik = ORC_PI * rik * c[1];
        for (int j = 0; j < g->ng; ++j) fd[j] = orc_fmexp(-0.5 * ORC_PI * g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) {
            const double fexp = fd[g->rflag[i]];
            const double den = 1.0 / (1.0 + fexp);
            const double cw = fabs(0.5 + g->lambdaf[i] * cs);
            const double gangle = dEdG[i] * pow(cw, zeta[i] - 1.0) * 2.0 * fexp * den;
            const double fangle = cw * gangle;
            *phi -= zeta[i] * g->lambdaf[i] * gangle;
            eta[0] -= fangle * (-dij * g->ieta2[i] * den + gg[0]);
            eta[1] -= fangle * (-dik * g->ieta2[i] * den + gg[1]);
        }
    } break;
    case ORC_A_SECH: {
        const double dij = ORC_PI * rij * c[0], dik = ORC_PI * rik * c[1];
        for (int j = 0; j < g->ng; ++j) fd[j] = orc_fmexp(-0.5 * ORC_PI * g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) {
            const double fexp = fd[g->rflag[i]];
            const double fexp2 = fexp * fexp;
            const double den = 1.0 / (1.0 + fexp2);
            const double ftanh = (1.0 - fexp2) * den;
            const double fsech = 2.0 * fexp * den;
            const double cw = fabs(0.5 + g->lambdaf[i] * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * dEdG[i] * fsech;
            const double fangle = cw * gangle;
            *phi -= zeta[i] * g->lambdaf[i] * gangle;
            eta[0] -= fangle * (-dij * g->ieta2[i] * ftanh + gg[0]);
            eta[1] -= fangle * (-dik * g->ieta2[i] * ftanh + gg[1]);
        }
    } break;
    case ORC_A_STUDENT3: case ORC_A_STUDENT4: case ORC_A_STUDENT5: {
        const int pw = 4 + (p->a_form[b] - ORC_A_STUDENT3);
        const double dij = pw * rij * c[0], dik = pw * rik * c[1];
        for (int j = 0; j < g->ng; ++j) fd[j] = 1.0 / sqrt(1.0 + g->ietar2[j] * r2s);
        for (int i = 0; i < n; ++i) {
            const double den = fd[g->rflag[i]];
            const double cw = fabs(0.5 + g->lambdaf[i] * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * dEdG[i] * orc_powint(den, pw);
            const double fangle = cw * gangle;
            *phi -= zeta[i] * g->lambdaf[i] * gangle;
            eta[0] -= fangle * (-dij * g->ieta2[i] * den * den + gg[0]);
            eta[1] -= fangle * (-dik * g->ieta2[i] * den * den + gg[1]);
        }
    } break;
    default:
        *phi = NAN;
    }
    *phi *= c[0] * c[1];
    eta[0] *= c[1];
    eta[1] *= c[0];
}

/* BasisA::symmd (basis_angular.cpp:259-364), per function: dG/dcos, dG/drij,
 * dG/drik.  Used only by the force-loss gradient (no reference counterpart). */
static void orc_basisA_symmd(const orc_pot *p, int b, double rij, double rik, double cs,
                             double *dphi, double *drj, double *drk)
{
    const int n = p->a_n[b];
    const double *etaa = p->a_eta + p->a_off[b], *zeta = p->a_zeta + p->a_off[b];
    const int32_t *lam = p->a_lambda + p->a_off[b];
    const int cut = p->a_cut[b];
    const double rc = p->a_rc[b];
    const double c[2] = {orc_cutf(cut, rc, rij), orc_cutf(cut, rc, rik)};
    const double g[2] = {orc_cutg(cut, rc, rij), orc_cutg(cut, rc, rik)};
    const double r2s = rij * rij + rik * rik;
    const double dij = 2.0 * rij * c[0], dik = 2.0 * rik * c[1];
    for (int i = 0; i < n; ++i) {
        const double lambdaf = 0.5 * lam[i];
        const double ieta2 = 1.0 / (etaa[i] * etaa[i]);
        double fphi = 0, fe0 = 0, fe1 = 0;
        switch (p->a_form[b]) {
        case ORC_A_GAUSS: {
            const double cw = fabs(0.5 + lambdaf * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * orc_fmexp(-ieta2 * r2s);
            const double fangle = cw * gangle;
            fphi = zeta[i] * lambdaf * gangle;
            fe0 = fangle * (-dij * ieta2 + g[0]);
            fe1 = fangle * (-dik * ieta2 + g[1]);
        } break;
        case ORC_A_GAUSS2: {
            const double fexp = orc_fmexp(-0.5 * ORC_PI * ieta2 * r2s), den = 1.0 / (1.0 + fexp);
            const double cw = fabs(0.5 + lambdaf * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * 2.0 * fexp * den;
            const double fangle = cw * gangle;
            fphi = zeta[i] * lambdaf * gangle;
            fe0 = fangle * (-dij * ieta2 * 0.5 * ORC_PI * den + g[0]);
            fe1 = fangle * (-dik * ieta2 * 0.5 * ORC_PI * den + g[1]);
        } break;
        case ORC_A_SECH: {
            const double fexp = orc_fmexp(-0.5 * ORC_PI * ieta2 * r2s), fexp2 = fexp * fexp;
            const double den = 1.0 / (1.0 + fexp2), ftanh = (1.0 - fexp2) * den, fsech = 2.0 * fexp * den;
            const double cw = fabs(0.5 + lambdaf * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * fsech;
            const double fangle = cw * gangle;
            fphi = zeta[i] * lambdaf * gangle;
            fe0 = fangle * (-dij * 0.5 * ORC_PI * ieta2 * ftanh + g[0]);
            fe1 = fangle * (-dik * 0.5 * ORC_PI * ieta2 * ftanh + g[1]);
        } break;
        case ORC_A_STUDENT3: case ORC_A_STUDENT4: case ORC_A_STUDENT5: {
            const int pw = 4 + (p->a_form[b] - ORC_A_STUDENT3);
            const double den = 1.0 / sqrt(1.0 + ieta2 * r2s);
            const double cw = fabs(0.5 + lambdaf * cs);
            const double gangle = pow(cw, zeta[i] - 1.0) * orc_powint(den, pw);
            const double fangle = cw * gangle;
            fphi = zeta[i] * lambdaf * gangle;
            fe0 = fangle * (-dij * ieta2 * pw / 2.0 * den * den + g[0]);
            fe1 = fangle * (-dik * ieta2 * pw / 2.0 * den * den + g[1]);
        } break;
        default: fphi = NAN;
        }
        dphi[i] = fphi * c[0] * c[1];
        drj[i] = fe0 * c[1];
        drk[i] = fe1 * c[0];
    }
}

/* ------------------------------------------------------------------------ */
/* atomic networks (ml/nn.cpp)                                                */
/* ------------------------------------------------------------------------ */

#define ORC_MAX_NODES 1024

typedef struct {
    int nlayer, nin, neuron;
    const int32_t *nodes;   /* nodes[0]=nin, nodes[1..nlayer] */
    double c;
    const double *inpw, *inpb, *outw, *outb;
    const double *b[ORC_MAX_LAYERS];
    const double *w[ORC_MAX_LAYERS];   /* column-major nodes[l+1] x nodes[l] */
} orc_net;

static void orc_net_view(const orc_pot *p, int II, orc_net *nn)
{
    nn->nlayer = p->nn_nlayer[II];
    nn->nodes = p->nn_nodes + II * ORC_MAX_LAYERS;
    nn->nin = nn->nodes[0];
    nn->neuron = p->nn_neuron[II];
    nn->c = p->nn_c[II];
    const double *q = p->nn_par + p->nn_off[II];
    const int nout = nn->nodes[nn->nlayer];
    nn->inpw = q; q += nn->nin;
    nn->inpb = q; q += nn->nin;
    nn->outw = q; q += nout;
    nn->outb = q; q += nout;
    for (int l = 0; l < nn->nlayer; ++l) { nn->b[l] = q; q += nn->nodes[l + 1]; }
    for (int l = 0; l < nn->nlayer; ++l) { nn->w[l] = q; q += (int64_t)nn->nodes[l + 1] * nn->nodes[l]; }
}

int orc_nparams(const orc_pot *p, int II)
{
    orc_net nn;
    orc_net_view(p, II, &nn);
    int s = 0;
    for (int l = 0; l < nn.nlayer; ++l) s += nn.nodes[l + 1] + nn.nodes[l + 1] * nn.nodes[l];
    return s;
}

/* AFFPBP (ml/nn.cpp:148-848): a = f(z), d = f'(z); d2 = f''(z) from AFFPBP2
 * for the activations the training path supports (else NAN). */
static void orc_act(int neuron, double c, double z, double *a, double *d, double *d2)
{
    double dd2 = NAN;
    switch (neuron) {
    case ORC_NEU_LINEAR: *a = z; *d = 1.0; dd2 = 0.0; break;
    case ORC_NEU_SIGMOID:
        if (z >= 0) { const double e = exp(-c * z), fr = 1.0 / (1.0 + e); *a = fr; *d = c * e * fr * fr; dd2 = -c * c * e * (1.0 - e) * fr * fr * fr; }
        else { const double e = exp(c * z), fr = 1.0 / (1.0 + e); *a = e * fr; *d = c * e * fr * fr; dd2 = -c * c * e * (e - 1.0) * fr * fr * fr; }
        break;
    case ORC_NEU_TANH: { const double t = tanh(c * z); *a = t; *d = c * (1.0 - t * t); dd2 = c * c * (-2.0 * t * (1.0 - t * t)); } break;
    case ORC_NEU_ISRU: { const double zz = c * z, isr = 1.0 / sqrt(1.0 + zz * zz); *a = zz * isr; *d = c * isr * isr * isr; } break;
    case ORC_NEU_ARCTAN: { const double zz = c * z * ORC_PI / 2.0; *a = (2.0 / ORC_PI) * atan(zz); *d = c / (1.0 + zz * zz); } break;
    case ORC_NEU_RELU: if (z > 0.0) { *a = z; *d = 1.0; } else { *a = 0.0; *d = 0.0; } break;
    case ORC_NEU_ELU: if (z >= 0.0) { *a = z; *d = 1.0; } else { const double e = exp(c * z); *a = e - 1.0; *d = c * e; } break;
    case ORC_NEU_TANHRE:
        if (z >= 0) { *a = z; *d = 1.0; }
        else { const double e = exp(2.0 * c * z); *a = (e - 1.0) / (e + 1.0); *d = c * (1.0 - (*a) * (*a)); }
        break;
    case ORC_NEU_SQRE:
        if (z >= 0) { *a = z; *d = 1.0; }
        else { const double den = 1.0 / sqrt(1.0 + z * z); *a = z * den; *d = den * den * den; }
        break;
    case ORC_NEU_SWISH: {
        const double zz = c * z;
        if (zz > 0.0) { const double e = exp(-zz), den = 1.0 / (1.0 + e); *a = z * den; *d = (1.0 + e * (1.0 + zz)) * den * den; }
        else { const double e = exp(zz), den = 1.0 / (1.0 + e); *a = z * e * den; *d = e * (1.0 + zz + e) * den * den; }
    } break;
    case ORC_NEU_GELU: {
        const double zz = 0.5 * ORC_RADPI * c * z, ep1 = (1.0 + erf(zz));
        *a = 0.5 * z * ep1; *d = 0.5 * (ep1 + c * z * exp(-zz * zz));
    } break;
    case ORC_NEU_MISH: {
        const double zz = c * z;
        if (zz > 0.0) {
            const double e = exp(-zz), e2 = e * e, den = 1.0 / ((1.0 + e) * (1.0 + e) + e2);
            *a = z * (1.0 - 2.0 * e2 * den); *d = 1.0 - 2.0 * e2 * den * (1.0 - 2.0 * zz * (1.0 + e) * den);
        } else {
            const double e = exp(zz), den = 1.0 / (e * (e + 2.0) + 2.0);
            *a = z * e * (e + 2.0) * den; *d = 1.0 + 2.0 * den * (-1.0 + 2.0 * zz * (1.0 - (e + 2.0) * den));
        }
    } break;
    case ORC_NEU_PFLU: {
        const double zz = c * z, z2 = zz * zz, fs = 1.0 / sqrt(z2 + 1.0);
        *a = 0.5 * z * (1.0 + zz * fs); *d = 0.5 * (zz * (z2 + 2.0) * fs * fs * fs + 1.0);
    } break;
    case ORC_NEU_LOGISH: {
        const double l2i = 1.0 / ORC_LOG2, e = exp(-z), lf = log(1.0 + 1.0 / (1.0 + e));
        *a = l2i * z * lf; *d = l2i * (lf + z * e / ((1.0 + e) * (2.0 + e)));
    } break;
    case ORC_NEU_SOFTPLUS: {
        const double ci = 1.0 / c;
        if (z > 0.0) { const double e = exp(-c * z); *a = z + ci * (log1p(e) - ORC_LOG2); *d = 1.0 / (e + 1.0); }
        else { const double e = exp(c * z); *a = ci * (log1p(e) - ORC_LOG2); *d = e / (e + 1.0); }
    } break;
    case ORC_NEU_SQPLUS: {
        const double ci = 1.0 / c, zz = c * z, fs = sqrt(1.0 + zz * zz);
        *a = 0.5 * ci * (zz - 1.0 + fs); *d = 0.5 * (zz / fs + 1.0);
    } break;
    case ORC_NEU_ATISH: {
        const double zz = 1 * 0.5 * ORC_PI * z;
        *a = z * 0.5 * (1.0 + 2.0 / ORC_PI * atan(zz)); *d = 0.5 * (1.0 + z / (1.0 + zz * zz)) + 1.0 / ORC_PI * atan(zz);
    } break;
    case ORC_NEU_IERF: {
        const double fexp = exp(-z * z);
        const double zs = (double)((0.0 < z) - (z < 0.0));
        const double t = 1.0 / (1.0 + 0.3275911 * z * zs);
        const double ferf = zs * (1.0 - t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429)))) * fexp);
        *a = 0.5 * (z * ferf + (fexp + z * ORC_RADPI - 1.0) / ORC_RADPI); *d = 0.5 * (ferf + 1.0);
    } break;
    case ORC_NEU_TEST: {
        const double zz = c * z, z2 = zz * zz, z4 = z2 * z2, den = 1.0 / sqrt(sqrt(z4 + 1.0));
        *a = 0.5 * z * (1.0 + zz * den); *d = 0.5 * (zz * den * (1.0 + 1.0 / (z4 + 1.0)) + 1.0);
    } break;
    default: *a = NAN; *d = NAN;
    }
    if (d2) *d2 = dd2;
}

typedef struct {
    double ins[ORC_MAX_NODES];
    double z[ORC_MAX_LAYERS][ORC_MAX_NODES];
    double a[ORC_MAX_LAYERS][ORC_MAX_NODES];
    double d[ORC_MAX_LAYERS][ORC_MAX_NODES];
    double d2[ORC_MAX_LAYERS][ORC_MAX_NODES];
    double out;
} orc_work;

/* ANN::fpbp (ml/nn.cpp:1402-1420); the last layer is linear (nn.cpp:1349-1352).
 * z_l = b_l, then z_l += W_l x column by column (the Eigen-subset GEMV order). */
static double orc_net_fpbp(const orc_net *nn, const double *inp, orc_work *w)
{
    for (int m = 0; m < nn->nin; ++m) w->ins[m] = nn->inpw[m] * (inp[m] + nn->inpb[m]);
    const double *x = w->ins;
    for (int l = 0; l < nn->nlayer; ++l) {
        const int no = nn->nodes[l + 1], ni = nn->nodes[l];
        double *z = w->z[l];
        for (int n = 0; n < no; ++n) z[n] = nn->b[l][n];
        for (int m = 0; m < ni; ++m) {
            const double xm = x[m];
            const double *col = nn->w[l] + (int64_t)m * no;
            for (int n = 0; n < no; ++n) z[n] += col[n] * xm;
        }
        const int neuron = (l == nn->nlayer - 1) ? ORC_NEU_LINEAR : nn->neuron;
        for (int n = 0; n < no; ++n) orc_act(neuron, nn->c, z[n], &w->a[l][n], &w->d[l][n], &w->d2[l][n]);
        x = w->a[l];
    }
    const int L = nn->nlayer - 1;
    w->out = nn->outb[0] + w->a[L][0] * nn->outw[0];
    return w->out;
}

/* DODZ::grad (ml/nn.cpp:1836-1859) for output 0: dodz_L = outw*d_L, then
 * dodz_{l-1} = (dodz_l W_l) diag(d_{l-1}), dodi = (dodz_0 W_0) diag(inpw). */
static void orc_net_dodi(const orc_net *nn, const orc_work *w, double *dodi)
{
    double g[ORC_MAX_NODES], t[ORC_MAX_NODES];
    const int L = nn->nlayer - 1;
    g[0] = nn->outw[0] * w->d[L][0];
    int ng = nn->nodes[L + 1];
    for (int l = L; l >= 0; --l) {
        const int no = nn->nodes[l + 1], ni = nn->nodes[l];
        for (int m = 0; m < ni; ++m) {
            double s = 0;
            const double *col = nn->w[l] + (int64_t)m * no;
            for (int n = 0; n < no; ++n) s += g[n] * col[n];
            t[m] = s;
        }
        if (l > 0) for (int m = 0; m < ni; ++m) g[m] = t[m] * w->d[l - 1][m];
        else for (int m = 0; m < ni; ++m) dodi[m] = t[m] * nn->inpw[m];
        ng = ni;
    }
    (void)ng;
}

/* Cost::grad (ml/nn.cpp:1747-1805) with dc/do = dcdo; accumulates s*grad into acc */
static void orc_net_costgrad(const orc_net *nn, const orc_work *w, double dcdo, double *grad)
{
    double dcdz[ORC_MAX_LAYERS][ORC_MAX_NODES];
    const int L = nn->nlayer - 1;
    dcdz[L][0] = dcdo;
    dcdz[L][0] *= nn->outw[0] * w->d[L][0];
    for (int l = L; l > 0; --l) {
        const int no = nn->nodes[l + 1], ni = nn->nodes[l];
        for (int m = 0; m < ni; ++m) {
            double s = 0;
            const double *col = nn->w[l] + (int64_t)m * no;
            for (int n = 0; n < no; ++n) s += col[n] * dcdz[l][n];
            dcdz[l - 1][m] = s;
        }
        for (int m = 0; m < ni; ++m) dcdz[l - 1][m] *= w->d[l - 1][m];
    }
    int count = 0;
    for (int l = 0; l <= L; ++l)
        for (int n = 0; n < nn->nodes[l + 1]; ++n) grad[count++] = dcdz[l][n];
    for (int l = 0; l <= L; ++l) {
        const double *x = (l == 0) ? w->ins : w->a[l - 1];
        for (int m = 0; m < nn->nodes[l]; ++m)
            for (int n = 0; n < nn->nodes[l + 1]; ++n) grad[count++] = dcdz[l][n] * x[m];
    }
}

double orc_ann_fpbp(const orc_pot *p, int II, const double *inp, double *dodi)
{
    orc_net nn;
    orc_net_view(p, II, &nn);
    orc_work *w = (orc_work *)malloc(sizeof(orc_work));
    const double out = orc_net_fpbp(&nn, inp, w);
    if (dodi) orc_net_dodi(&nn, w, dodi);
    free(w);
    return out;
}

double orc_cost_grad(const orc_pot *p, int II, const double *inp, double *grad)
{
    orc_net nn;
    orc_net_view(p, II, &nn);
    orc_work *w = (orc_work *)malloc(sizeof(orc_work));
    const double out = orc_net_fpbp(&nn, inp, w);
    orc_net_costgrad(&nn, w, 1.0, grad);
    free(w);
    return out;
}

/* ------------------------------------------------------------------------ */
/* neighbour list (struc/neighbor.cpp:46-87)                                  */
/* ------------------------------------------------------------------------ */

/* R*v for R with columns = lattice vectors (cell[3*n+d] = R(d,n)) */
static void orc_Rv(const double *cell, const double *v, double *out)
{
    for (int d = 0; d < 3; ++d) out[d] = cell[d] * v[0] + cell[3 + d] * v[1] + cell[6 + d] * v[2];
}

typedef struct {
    int natoms, cap;
    int32_t *cnt, *idx;
    double *img;
} orc_nl;

static int orc_nlist_build(double rc, int natoms, const double *pos, const double *cell, int pbc, orc_nl *nl)
{
    static const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double *R = pbc ? cell : zero9;
    const double rc2 = rc * rc;
    int cellf[3] = {0, 0, 0};
    double rn = 0;
    for (int k = 0; k < 9; ++k) rn += R[k] * R[k];
    if (sqrt(rn) > ORC_ZERO)
        for (int n = 0; n < 3; ++n) {
            const double *a = R + 3 * n;
            cellf[n] = (int)ceil(3.0 * rc / sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
        }
    int overflow = 0;
    for (int n = 0; n < natoms; ++n) {
        int c = 0;
        for (int m = 0; m < natoms; ++m) {
            double dr[3];
            for (int d = 0; d < 3; ++d) dr[d] = pos[3 * n + d] - pos[3 * m + d];
            for (int i = -cellf[0]; i <= cellf[0]; ++i)
                for (int j = -cellf[1]; j <= cellf[1]; ++j)
                    for (int k = -cellf[2]; k <= cellf[2]; ++k) {
                        const double iv[3] = {1.0 * i, 1.0 * j, 1.0 * k};
                        double t[3];
                        orc_Rv(R, iv, t);
                        const double x = dr[0] - t[0], y = dr[1] - t[1], z = dr[2] - t[2];
                        const double ds2 = x * x + y * y + z * z;
                        if (m != n || ds2 > ORC_ZERO) {
                            if (ds2 < rc2) {
                                if (c < nl->cap) {
                                    nl->idx[(int64_t)n * nl->cap + c] = m;
                                    double *im = nl->img + ((int64_t)n * nl->cap + c) * 3;
                                    im[0] = iv[0]; im[1] = iv[1]; im[2] = iv[2];
                                } else overflow = 1;
                                ++c;
                            }
                        }
                    }
        }
        nl->cnt[n] = c;
    }
    return overflow ? -1 : 0;
}

int orc_nlist(double rc, int natoms, const double *pos, const double *cell, int pbc,
              int cap, int32_t *counts, int32_t *idx, double *img)
{
    orc_nl nl = {natoms, cap, counts, idx, img};
    return orc_nlist_build(rc, natoms, pos, cell, pbc, &nl);
}

/* rIJ = posn(i) - (posn(j) + R*img) as in nnp.cpp:363 */
static double orc_rij(const double *pos, const double *R, int i, int j, const double *img, double *r)
{
    double t[3];
    orc_Rv(R, img, t);
    for (int d = 0; d < 3; ++d) r[d] = pos[3 * i + d] - (pos[3 * j + d] + t[d]);
    return sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

static int orc_tt(int i, int j) { return (i > j) ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

static int orc_alloc_nl(const orc_pot *p, int natoms, const double *pos, const double *cell, int pbc, orc_nl *nl)
{
    nl->natoms = natoms;
    nl->cap = 64;
    for (;;) {
        nl->cnt = (int32_t *)malloc(sizeof(int32_t) * (natoms > 0 ? natoms : 1));
        nl->idx = (int32_t *)malloc(sizeof(int32_t) * (int64_t)(natoms > 0 ? natoms : 1) * nl->cap);
        nl->img = (double *)malloc(sizeof(double) * 3 * (int64_t)(natoms > 0 ? natoms : 1) * nl->cap);
        if (orc_nlist_build(p->rc, natoms, pos, cell, pbc, nl) == 0) return 0;
        int mx = 0;
        for (int i = 0; i < natoms; ++i) if (nl->cnt[i] > mx) mx = nl->cnt[i];
        free(nl->cnt); free(nl->idx); free(nl->img);
        nl->cap = mx + 1;
    }
}

static void orc_free_nl(orc_nl *nl) { free(nl->cnt); free(nl->idx); free(nl->img); }

/* NNP::compute_symm (nnp.cpp:350-392) over a prebuilt list */
static void orc_symm_nl(const orc_pot *p, int natoms, const double *pos, const int32_t *type,
                        const double *R, const orc_nl *nl, int gstride, double *symm)
{
    const int T = p->ntypes, TT = T * (T + 1) / 2;
    double buf[ORC_MAX_A];
    orc_agroups *grp = (orc_agroups *)malloc(sizeof(orc_agroups) * T * TT);
    for (int b = 0; b < T * TT; ++b) orc_basisA_init(p, b, &grp[b]);
    for (int i = 0; i < natoms; ++i) {
        double *G = symm + (int64_t)i * gstride;
        const int II = type[i];
        for (int g = 0; g < p->n_input[II]; ++g) G[g] = 0;
        const int n = nl->cnt[i];
        const int32_t *ix = nl->idx + (int64_t)i * nl->cap;
        const double *im = nl->img + (int64_t)i * nl->cap * 3;
        for (int j = 0; j < n; ++j) {
            const int jj = ix[j], JJ = type[jj];
            double rIJ[3];
            const double drIJ = orc_rij(pos, R, i, jj, im + 3 * j, rIJ);
            const int br = II * T + JJ;
            orc_basisR_symm(p, br, drIJ, buf);
            const int oR = p->offset_r[br];
            for (int nr = 0; nr < p->r_n[br]; ++nr) G[oR + nr] += buf[nr];
            for (int k = j + 1; k < n; ++k) {
                const int kk = ix[k], KK = type[kk];
                double rIK[3];
                const double drIK = orc_rij(pos, R, i, kk, im + 3 * k, rIK);
                const double cosIJK = (rIJ[0] * rIK[0] + rIJ[1] * rIK[1] + rIJ[2] * rIK[2]) / (drIJ * drIK);
                const int ba = II * TT + orc_tt(JJ, KK);
                orc_basisA_symm(p, ba, &grp[ba], drIJ, drIK, cosIJK, buf);
                const int oA = p->n_input_r[II] + p->offset_a[ba];
                for (int na = 0; na < p->a_n[ba]; ++na) G[oA + na] += buf[na];
            }
        }
    }
    free(grp);
}

int orc_compute_symm(const orc_pot *p, int natoms, const double *pos, const int32_t *type,
                     const double *cell, int pbc, int gstride, double *symm)
{
    static const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    orc_nl nl;
    orc_alloc_nl(p, natoms, pos, cell, pbc, &nl);
    orc_symm_nl(p, natoms, pos, type, pbc ? cell : zero9, &nl, gstride, symm);
    orc_free_nl(&nl);
    return 0;
}

/* NNP::compute_energy (nnp.cpp:329-338) with NNH::energy (nnh.cpp:207-210) */
double orc_compute_energy(const orc_pot *p, int natoms, const int32_t *type, int gstride, const double *symm)
{
    double pe = 0;
    for (int i = 0; i < natoms; ++i) {
        const int II = type[i];
        pe += orc_ann_fpbp(p, II, symm + (int64_t)i * gstride, NULL) + p->energy[II];
    }
    return pe;
}

/* NNP::compute_force (nnp.cpp:412-476) over a prebuilt list */
static double orc_force_nl(const orc_pot *p, int natoms, const double *pos, const int32_t *type,
                           const double *R, const orc_nl *nl, int gstride, const double *symm,
                           double *force, double *dedg_out)
{
    const int T = p->ntypes, TT = T * (T + 1) / 2;
    orc_agroups *grp = (orc_agroups *)malloc(sizeof(orc_agroups) * T * TT);
    for (int b = 0; b < T * TT; ++b) orc_basisA_init(p, b, &grp[b]);
    orc_work *w = (orc_work *)malloc(sizeof(orc_work));
    double dEdG[ORC_MAX_NODES];
    double pe = 0;
    for (int i = 0; i < 3 * natoms; ++i) force[i] = 0;
    for (int i = 0; i < natoms; ++i) {
        const int II = type[i];
        orc_net nn;
        orc_net_view(p, II, &nn);
        pe += orc_net_fpbp(&nn, symm + (int64_t)i * gstride, w);
        orc_net_dodi(&nn, w, dEdG);
        if (dedg_out) for (int g = 0; g < nn.nin; ++g) dedg_out[(int64_t)i * gstride + g] = dEdG[g];
        const int n = nl->cnt[i];
        const int32_t *ix = nl->idx + (int64_t)i * nl->cap;
        const double *im = nl->img + (int64_t)i * nl->cap * 3;
        double *Fi = force + 3 * i;
        for (int j = 0; j < n; ++j) {
            const int jj = ix[j], JJ = type[jj];
            double rIJ[3];
            const double drIJ = orc_rij(pos, R, i, jj, im + 3 * j, rIJ);
            const double dIJi = 1.0 / drIJ;
            const int br = II * T + JJ;
            const double amp = orc_basisR_force(p, br, drIJ, dEdG + p->offset_r[br]) * dIJi;
            double *Fj = force + 3 * jj;
            for (int d = 0; d < 3; ++d) Fi[d] += amp * rIJ[d];
            for (int d = 0; d < 3; ++d) Fj[d] -= amp * rIJ[d];
            for (int k = j + 1; k < n; ++k) {
                const int kk = ix[k], KK = type[kk];
                double rIK[3];
                const double drIK = orc_rij(pos, R, i, kk, im + 3 * k, rIK);
                const double dIKi = 1.0 / drIK;
                const int ba = II * TT + orc_tt(JJ, KK);
                const int oA = p->n_input_r[II] + p->offset_a[ba];
                double phi = 0, eta[2] = {0, 0};
                const double cs = (rIJ[0] * rIK[0] + rIJ[1] * rIK[1] + rIJ[2] * rIK[2]) * dIJi * dIKi;
                orc_basisA_force(p, ba, &grp[ba], drIJ, drIK, cs, &phi, eta, dEdG + oA);
                double *Fk = force + 3 * kk;
                const double s1 = phi * (dIKi - cs * dIJi) + eta[0];
                for (int d = 0; d < 3; ++d) Fi[d] += s1 * rIJ[d] * dIJi;
                const double s2 = phi * (dIJi - cs * dIKi) + eta[1];
                for (int d = 0; d < 3; ++d) Fi[d] += s2 * rIK[d] * dIKi;
                const double s3 = -phi * cs * dIJi + eta[0];
                for (int d = 0; d < 3; ++d) Fj[d] -= s3 * rIJ[d] * dIJi + phi * dIJi * rIK[d] * dIKi;
                const double s4 = -phi * cs * dIKi + eta[1];
                for (int d = 0; d < 3; ++d) Fk[d] -= s4 * rIK[d] * dIKi + phi * dIKi * rIJ[d] * dIJi;
            }
        }
    }
    free(w);
    free(grp);
    return pe;
}

double orc_compute_force(const orc_pot *p, int natoms, const double *pos, const int32_t *type,
                         const double *cell, int pbc, int gstride, const double *symm,
                         double *force, double *dedg)
{
    static const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    orc_nl nl;
    orc_alloc_nl(p, natoms, pos, cell, pbc, &nl);
    const double e = orc_force_nl(p, natoms, pos, type, pbc ? cell : zero9, &nl, gstride, symm, force, dedg);
    orc_free_nl(&nl);
    return e;
}

double orc_compute(const orc_pot *p, int natoms, const double *pos, const int32_t *type,
                   const double *cell, int pbc, int gstride, double *symm, double *force)
{
    static const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double *R = pbc ? cell : zero9;
    orc_nl nl;
    orc_alloc_nl(p, natoms, pos, cell, pbc, &nl);
    orc_symm_nl(p, natoms, pos, type, R, &nl, gstride, symm);
    const double e = orc_force_nl(p, natoms, pos, type, R, &nl, gstride, symm, force, NULL);
    orc_free_nl(&nl);
    return e;
}

/* ------------------------------------------------------------------------ */
/* training                                                                   */
/* ------------------------------------------------------------------------ */

/* nnptefr.cpp:614-620 */
static double orc_norm(int mode, double n)
{
    switch (mode) {
    case 0: return 1.0;
    case 1: return 1.0 / n;
    case 2: return 1.0 / sqrt(n);
    case 3: return 1.0 / cbrt(n);
    case 4: return 1.0 / (log(n) + 1.0);
    default: return NAN;
    }
}

/* Loss of one structure's scaled energy error dU and its derivative
 * dloss/ddU (*dl), NNPTEFR::error_cost_o1 (nnptefr.cpp:1340-1376). */
static double orc_loss(int kind, double delta, double dU, double *dl)
{
    switch (kind) {
    case 2:
        *dl = (dU > 0) - (dU < 0);
        return fabs(dU);
    case 3: {
        const double arg = dU / delta, sq = sqrt(1.0 + arg * arg);
        *dl = dU / sq;
        return delta * delta * (sq - 1.0);
    }
    case 4: {
        const double arg = dU / delta, sq = sqrt(1.0 + arg * arg), lg = log(arg + sq);
        *dl = lg * delta;
        return delta * delta * (1.0 - sq + arg * lg);
    }
    case 1:
        *dl = dU;
        return 0.5 * dU * dU;
    default:
        *dl = NAN;
        return NAN;
    }
}

static int orc_param_offsets(const orc_pot *p, int *off)
{
    int tot = 0;
    for (int t = 0; t < p->ntypes; ++t) { off[t] = tot; tot += orc_nparams(p, t); }
    return tot;
}

/* NNPTEFR::error_cost_o1 (nnptefr.cpp:1292-1380), then the batch average of
 * nnptefr.cpp:996-1000. */
double orc_energy_loss_grad(const orc_pot *p, int nstruct, const int64_t *atom_off,
                            const int32_t *type, int gstride, const double *symm,
                            const double *e_ref, int norm_mode, int loss_kind, double delta,
                            double *grad)
{
    int off[64];
    const int np = orc_param_offsets(p, off);
    double *gs = (double *)calloc(np, sizeof(double));
    double *ga = (double *)malloc(sizeof(double) * np);
    orc_work *w = (orc_work *)malloc(sizeof(orc_work));
    double err = 0;
    for (int k = 0; k < np; ++k) grad[k] = 0;
    for (int s = 0; s < nstruct; ++s) {
        for (int k = 0; k < np; ++k) gs[k] = 0;
        double pe = 0;
        for (int64_t n = atom_off[s]; n < atom_off[s + 1]; ++n) {
            const int t = type[n];
            orc_net nn;
            orc_net_view(p, t, &nn);
            pe += orc_net_fpbp(&nn, symm + n * gstride, w);
            orc_net_costgrad(&nn, w, 1.0, ga);
            const int npt = orc_nparams(p, t);
            for (int k = 0; k < npt; ++k) gs[off[t] + k] += ga[k];
        }
        const double nat = (double)(atom_off[s + 1] - atom_off[s]);
        const double nrm = orc_norm(norm_mode, nat);
        const double dE = pe - e_ref[s];
        const double dU = dE * nrm;
        double dl;
        err += orc_loss(loss_kind, delta, dU, &dl);
        const double gfac = nrm * dl;
        for (int k = 0; k < np; ++k) grad[k] += gs[k] * gfac;
    }
    const double bi = 1.0 / nstruct;
    for (int k = 0; k < np; ++k) grad[k] *= bi;
    free(w); free(ga); free(gs);
    return err * bi;
}

/* Weight gradient of s = dN/dG(G) . cdir (forward-over-reverse through one
 * network); accumulates scale * ds/dtheta into grad (reference packing). */
static void orc_net_jvp_grad(const orc_net *nn, const orc_work *w, const double *cdir, double scale, double *grad)
{
    static double zt[ORC_MAX_LAYERS][ORC_MAX_NODES], at[ORC_MAX_LAYERS][ORC_MAX_NODES];
    double inst[ORC_MAX_NODES];
    const int L = nn->nlayer - 1;
    for (int m = 0; m < nn->nin; ++m) inst[m] = nn->inpw[m] * cdir[m];
    /* tangent forward */
    for (int l = 0; l <= L; ++l) {
        const int no = nn->nodes[l + 1], ni = nn->nodes[l];
        const double *xt = (l == 0) ? inst : at[l - 1];
        for (int n = 0; n < no; ++n) zt[l][n] = 0;
        for (int m = 0; m < ni; ++m) {
            const double *col = nn->w[l] + (int64_t)m * no;
            for (int n = 0; n < no; ++n) zt[l][n] += col[n] * xt[m];
        }
        for (int n = 0; n < no; ++n) at[l][n] = w->d[l][n] * zt[l][n];
    }
    /* reverse: adjoints of primal (ab) and tangent (abt) activations */
    double ab[ORC_MAX_NODES], abt[ORC_MAX_NODES], zb[ORC_MAX_NODES], zbt[ORC_MAX_NODES];
    double nab[ORC_MAX_NODES], nabt[ORC_MAX_NODES];
    const int nout = nn->nodes[L + 1];
    for (int n = 0; n < nout; ++n) { ab[n] = 0; abt[n] = (n == 0) ? nn->outw[0] : 0; }
    int boff[ORC_MAX_LAYERS], woff[ORC_MAX_LAYERS], cnt = 0;
    for (int l = 0; l <= L; ++l) { boff[l] = cnt; cnt += nn->nodes[l + 1]; }
    for (int l = 0; l <= L; ++l) { woff[l] = cnt; cnt += nn->nodes[l + 1] * nn->nodes[l]; }
    for (int l = L; l >= 0; --l) {
        const int no = nn->nodes[l + 1], ni = nn->nodes[l];
        for (int n = 0; n < no; ++n) {
            zbt[n] = abt[n] * w->d[l][n];
            zb[n] = ab[n] * w->d[l][n] + abt[n] * w->d2[l][n] * zt[l][n];
        }
        const double *x = (l == 0) ? w->ins : w->a[l - 1];
        const double *xt = (l == 0) ? inst : at[l - 1];
        for (int n = 0; n < no; ++n) grad[boff[l] + n] += scale * zb[n];
        for (int m = 0; m < ni; ++m)
            for (int n = 0; n < no; ++n)
                grad[woff[l] + m * no + n] += scale * (zb[n] * x[m] + zbt[n] * xt[m]);
        if (l > 0) {
            for (int m = 0; m < ni; ++m) {
                const double *col = nn->w[l] + (int64_t)m * no;
                double s = 0, st = 0;
                for (int n = 0; n < no; ++n) { s += col[n] * zb[n]; st += col[n] * zbt[n]; }
                nab[m] = s; nabt[m] = st;
            }
            for (int m = 0; m < ni; ++m) { ab[m] = nab[m]; abt[m] = nabt[m]; }
        }
    }
}

double orc_ef_loss_grad(const orc_pot *p, int nstruct, const int64_t *atom_off,
                        const double *pos, const int32_t *type, const double *cell, int pbc,
                        const double *e_ref, const double *f_ref, double w_f, int norm_mode,
                        int loss_kind, double delta, double *grad, double *eout, double *fout)
{
    static const double zero9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int T = p->ntypes, TT = T * (T + 1) / 2;
    int off[64];
    const int np = orc_param_offsets(p, off);
    int gstride = 0;
    for (int t = 0; t < T; ++t) if (p->n_input[t] > gstride) gstride = p->n_input[t];
    double *ga = (double *)malloc(sizeof(double) * (np + 1));
    orc_work *w = (orc_work *)malloc(sizeof(orc_work));
    double bufr[ORC_MAX_A], dphi[ORC_MAX_A], drj[ORC_MAX_A], drk[ORC_MAX_A];
    const double bi = 1.0 / nstruct;
    double loss = 0;
    if (grad) for (int k = 0; k < np; ++k) grad[k] = 0;
    for (int s = 0; s < nstruct; ++s) {
        const int64_t a0 = atom_off[s];
        const int nat = (int)(atom_off[s + 1] - a0);
        const double *ps = pos + 3 * a0;
        const int32_t *ts = type + a0;
        const double *R = pbc ? cell + 9 * s : zero9;
        orc_nl nl;
        orc_alloc_nl(p, nat, ps, pbc ? cell + 9 * s : zero9, pbc, &nl);
        double *G = (double *)calloc((size_t)nat * gstride + 1, sizeof(double));
        double *F = (double *)calloc((size_t)nat * 3 + 1, sizeof(double));
        double *C = (double *)calloc((size_t)nat * gstride + 1, sizeof(double));
        double *V = (double *)calloc((size_t)nat * 3 + 1, sizeof(double));
        orc_symm_nl(p, nat, ps, ts, R, &nl, gstride, G);
        const double E = orc_force_nl(p, nat, ps, ts, R, &nl, gstride, G, F, NULL);
        if (eout) eout[s] = E;
        if (fout) for (int k = 0; k < 3 * nat; ++k) fout[3 * a0 + k] = F[k];
        const double nrm = orc_norm(norm_mode, (double)nat);
        const double dU = (E - e_ref[s]) * nrm;
        double lf = 0;
        const double fs = w_f / (3.0 * nat);
        for (int k = 0; k < 3 * nat; ++k) {
            const double df = F[k] - f_ref[3 * a0 + k];
            lf += df * df;
            V[k] = fs * df * bi;
        }
        double dl;
        loss += bi * (orc_loss(loss_kind, delta, dU, &dl) + 0.5 * fs * lf);
        if (grad) {
            /* c_a = sum_i dG_a/dx_i . v_i over every pair and triplet */
            for (int i = 0; i < nat; ++i) {
                const int II = ts[i];
                double *Ca = C + (int64_t)i * gstride;
                const int n = nl.cnt[i];
                const int32_t *ix = nl.idx + (int64_t)i * nl.cap;
                const double *im = nl.img + (int64_t)i * nl.cap * 3;
                for (int j = 0; j < n; ++j) {
                    const int jj = ix[j], JJ = ts[jj];
                    double rIJ[3];
                    const double drIJ = orc_rij(ps, R, i, jj, im + 3 * j, rIJ);
                    double uj[3], vj[3];
                    for (int d = 0; d < 3; ++d) { uj[d] = rIJ[d] / drIJ; vj[d] = V[3 * i + d] - V[3 * jj + d]; }
                    const int br = II * T + JJ;
                    orc_basisR_symmd(p, br, drIJ, bufr);
                    const double pj = uj[0] * vj[0] + uj[1] * vj[1] + uj[2] * vj[2];
                    for (int q = 0; q < p->r_n[br]; ++q) Ca[p->offset_r[br] + q] += bufr[q] * pj;
                    for (int k = j + 1; k < n; ++k) {
                        const int kk = ix[k], KK = ts[kk];
                        double rIK[3];
                        const double drIK = orc_rij(ps, R, i, kk, im + 3 * k, rIK);
                        double uk[3], vk[3];
                        for (int d = 0; d < 3; ++d) { uk[d] = rIK[d] / drIK; vk[d] = V[3 * i + d] - V[3 * kk + d]; }
                        const double cs = uj[0] * uk[0] + uj[1] * uk[1] + uj[2] * uk[2];
                        const int ba = II * TT + orc_tt(JJ, KK);
                        orc_basisA_symmd(p, ba, drIJ, drIK, cs, dphi, drj, drk);
                        /* dcos/dd_j = (u_k - cos u_j)/r_j, dcos/dd_k = (u_j - cos u_k)/r_k */
                        double cj = 0, ck = 0, rj = 0, rk = 0;
                        for (int d = 0; d < 3; ++d) {
                            cj += (uk[d] - cs * uj[d]) / drIJ * vj[d];
                            ck += (uj[d] - cs * uk[d]) / drIK * vk[d];
                            rj += uj[d] * vj[d];
                            rk += uk[d] * vk[d];
                        }
                        const int oA = p->n_input_r[II] + p->offset_a[ba];
                        for (int q = 0; q < p->a_n[ba]; ++q)
                            Ca[oA + q] += dphi[q] * (cj + ck) + drj[q] * rj + drk[q] * rk;
                    }
                }
            }
            /* gradient: energy term g_s dE/dtheta, force term -d(dE/dG . c)/dtheta */
            const double gfac = nrm * dl * bi;
            for (int i = 0; i < nat; ++i) {
                const int t = ts[i];
                orc_net nn;
                orc_net_view(p, t, &nn);
                orc_net_fpbp(&nn, G + (int64_t)i * gstride, w);
                orc_net_costgrad(&nn, w, 1.0, ga);
                const int npt = orc_nparams(p, t);
                for (int k = 0; k < npt; ++k) grad[off[t] + k] += gfac * ga[k];
                orc_net_jvp_grad(&nn, w, C + (int64_t)i * gstride, -1.0, grad + off[t]);
            }
        }
        free(G); free(F); free(C); free(V);
        orc_free_nl(&nl);
    }
    free(w); free(ga);
    return loss;
}
