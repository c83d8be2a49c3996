/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * MOS1 (Shichman-Hodges), restated from models/mos1.va with hand-written
 * derivatives (the reference differentiates by VerA's forward AD):
 *   :150-271  parameter defaulting, temperature and geometry (mos1temp.c)
 *   :272-304  limiting: fetlim on the controlling gate leg, limvds, pnjlim
 *             on one bulk junction (mos1load.c:361-384), MODEINITJCT seeds
 *   :306-345  bulk junctions, mode swap, drain current
 *   :347-350  junction depletion charges
 *   :351-441  Meyer gate capacitance: only its overlap part (CGSO, CGDO,
 *             CGBO) is supported; with TOX given the bias-dependent halves
 *             and their $prev averaging are not built, so such a circuit's
 *             transient is refused (orc_mos1_supported); its DC runs, TOX
 *             entering only through the KP default (:159-192).
 *
 * Frame: the model runs on type-frame voltages v = type * V (PMOS negated).
 * Limited images, three per instance: vgs, vds, vbs in the type frame.
 * A limited instance is evaluated at its images and every current and
 * charge is linearised back to x: f += sum_k df/dv_k * (v_k(x) - v_k,lim).
 */
#include "orc_internal.h"

#include <math.h>
#include <string.h>

#define KB 1.38064852e-23
#define QE 1.6021766208e-19

enum {
    MD_TYPE, MD_VT, MD_VBIT, MD_GAMMA, MD_PHIT, MD_BETA, MD_LAMBDA, MD_ISATS, MD_ISATD,
    MD_VCRITS, MD_VCRITD, MD_GDRAIN, MD_GSOURCE, MD_CZBD, MD_CZBS, MD_CZBDSW, MD_CZBSSW,
    MD_PBT, MD_MJ, MD_MJSW, MD_FC, MD_F2D, MD_F3D, MD_F4D, MD_F2S, MD_F3S, MD_F4S,
    MD_CGS, MD_CGD, MD_CGB, MD_GMIN, MD_HASQ, MD_NDER
};

int orc_mos1_supported(const double *p) { return !(p[ORC_M_TOX] > 0.0); }

void mos1_derive(const double *p, double *d) {
    memset(d, 0, sizeof(double) * ORC_NDER);
    const double type = p[ORC_M_TYPE];
    const double tnomk = p[ORC_M_TNOM] + 273.15;
    const double vtnom = tnomk * (KB / QE);
    const double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    const double phix = p[ORC_M_PHI];
    const double gammax = p[ORC_M_GAMMA];
    const double vtox = p[ORC_M_VTO] + p[ORC_M_DELVTO];
    /* KP: the card's, else u0 * Cox' with TOX given, else 2e-5 (mos1.va:159-192) */
    const double coxp = p[ORC_M_TOX] > 0.0 ? 3.9 * 8.854214871e-12 / p[ORC_M_TOX] : 0.0;
    const double kpx = !isnan(p[ORC_M_KP]) ? p[ORC_M_KP] : coxp > 0.0 ? p[ORC_M_U0] * coxp * 1.0e-4 : 2.0e-5;
    const double tk = p[ORC_M_TEMP];
    const double vt = tk * (KB / QE);
    const double fact1 = tnomk / 300.15;
    const double fact2 = tk / 300.15;
    const double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    const double arg1 = -egfet1 / (2.0 * KB * tnomk) + 1.1150877 / (2.0 * KB * 300.15);
    const double argt = -egfet / (2.0 * KB * tk) + 1.1150877 / (2.0 * KB * 300.15);
    const double pbfact1 = -2.0 * vtnom * (1.5 * esl_log(fact1) + QE * arg1);
    const double pbfact = -2.0 * vt * (1.5 * esl_log(fact2) + QE * argt);
    const double ratio4 = (tk / tnomk) * sqrt(tk / tnomk);
    const double kpt = kpx / ratio4;
    const double phio = (phix - pbfact1) / fact1;
    const double phit = fact2 * phio + pbfact;
    const double vbit = vtox - type * (gammax * sqrt(phix)) + 0.5 * (egfet1 - egfet) + type * 0.5 * (phit - phix);
    const double ist = p[ORC_M_IS] * esl_exp(-egfet / vt + egfet1 / vtnom);
    const double pb = p[ORC_M_PB], mj = p[ORC_M_MJ], mjsw = p[ORC_M_MJSW];
    const double pbo = (pb - pbfact1) / fact1;
    const double pbt = fact2 * pbo + pbfact;
    const double gmaold = (pb - pbo) / pbo;
    const double gmanew = (pbt - pbo) / pbo;
    const double cfb = (1.0 + mj * (4.0e-4 * (tk - 300.15) - gmanew)) /
                       (1.0 + mj * (4.0e-4 * (tnomk - 300.15) - gmaold));
    const double cfsw = (1.0 + mjsw * (4.0e-4 * (tk - 300.15) - gmanew)) /
                        (1.0 + mjsw * (4.0e-4 * (tnomk - 300.15) - gmaold));
    const double m = p[ORC_M_M], w = p[ORC_M_W];
    double leff = p[ORC_M_L] - 2.0 * p[ORC_M_LD];
    if (leff < 1.0e-10) leff = 1.0e-10;
    const double beta = kpt * m * w / leff;
    const double isatd = ist * m, isats = ist * m;
    const double cj = p[ORC_M_CJ], cjsw = p[ORC_M_CJSW];
    const double czbd = p[ORC_M_CBD] > 0.0 ? p[ORC_M_CBD] * cfb * m : cj * cfb * p[ORC_M_AD] * m;
    const double czbs = p[ORC_M_CBS] > 0.0 ? p[ORC_M_CBS] * cfb * m : cj * cfb * p[ORC_M_AS] * m;
    const double czbdsw = cjsw * cfsw * p[ORC_M_PD] * m;
    const double czbssw = cjsw * cfsw * p[ORC_M_PS] * m;
    const double fc = p[ORC_M_FC];
    const double depcap = fc * pbt;
    const double argf = 1.0 - fc;
    const double sargb = esl_pow(argf, -mj);
    const double sargs = esl_pow(argf, -mjsw);
    const double f2d = czbd * (1.0 - fc * (1.0 + mj)) * sargb / argf + czbdsw * (1.0 - fc * (1.0 + mjsw)) * sargs / argf;
    const double f3d = czbd * mj * sargb / (argf * pbt) + czbdsw * mjsw * sargs / (argf * pbt);
    const double f4d = czbd * pbt * (1.0 - argf * sargb) / (1.0 - mj) + czbdsw * pbt * (1.0 - argf * sargs) / (1.0 - mjsw) -
                       0.5 * f3d * depcap * depcap - depcap * f2d;
    const double f2s = czbs * (1.0 - fc * (1.0 + mj)) * sargb / argf + czbssw * (1.0 - fc * (1.0 + mjsw)) * sargs / argf;
    const double f3s = czbs * mj * sargb / (argf * pbt) + czbssw * mjsw * sargs / (argf * pbt);
    const double f4s = czbs * pbt * (1.0 - argf * sargb) / (1.0 - mj) + czbssw * pbt * (1.0 - argf * sargs) / (1.0 - mjsw) -
                       0.5 * f3s * depcap * depcap - depcap * f2s;
    d[MD_TYPE] = type;
    d[MD_VT] = vt;
    d[MD_VBIT] = vbit;
    d[MD_GAMMA] = gammax;
    d[MD_PHIT] = phit;
    d[MD_BETA] = beta;
    d[MD_LAMBDA] = p[ORC_M_LAMBDA];
    d[MD_ISATS] = isats;
    d[MD_ISATD] = isatd;
    d[MD_VCRITS] = vt * esl_log(vt / (1.4142135623730951 * isats));
    d[MD_VCRITD] = vt * esl_log(vt / (1.4142135623730951 * isatd));
    d[MD_GDRAIN] = p[ORC_M_RD] > 0.0 ? m / p[ORC_M_RD] : 0.0;
    d[MD_GSOURCE] = p[ORC_M_RS] > 0.0 ? m / p[ORC_M_RS] : 0.0;
    d[MD_CZBD] = czbd;
    d[MD_CZBS] = czbs;
    d[MD_CZBDSW] = czbdsw;
    d[MD_CZBSSW] = czbssw;
    d[MD_PBT] = pbt;
    d[MD_MJ] = mj;
    d[MD_MJSW] = mjsw;
    d[MD_FC] = fc;
    d[MD_F2D] = f2d; d[MD_F3D] = f3d; d[MD_F4D] = f4d;
    d[MD_F2S] = f2s; d[MD_F3S] = f3s; d[MD_F4S] = f4s;
    d[MD_CGS] = p[ORC_M_CGSO] * w * m;
    d[MD_CGD] = p[ORC_M_CGDO] * w * m;
    d[MD_CGB] = p[ORC_M_CGBO] * leff * m;
    d[MD_GMIN] = p[ORC_M_GMIN];
    d[MD_HASQ] = (czbd != 0.0 || czbs != 0.0 || czbdsw != 0.0 || czbssw != 0.0 || d[MD_CGS] != 0.0 ||
                  d[MD_CGD] != 0.0 || d[MD_CGB] != 0.0) ? 1.0 : 0.0;
}

int mos1_has_charge(const double *der) { return der[MD_HASQ] != 0.0; }

/* jcur (mos1.va:118-129) and its slope. */
static void jcur(double v, double isat, double vtx, double gm, double *i, double *g) {
    if (v > -3.0 * vtx) {
        double u = fmin(v / vtx, 80.0);
        double e = esl_exp(u);
        *i = isat * (e * (1.0 + (v / vtx - u)) - 1.0) + gm * v;
        *g = isat * e / vtx + gm;
    } else {
        *i = gm * v - isat;
        *g = gm;
    }
}

/* sbody (mos1.va:131-141); ds = d sbody / d vbx as ngspice takes it,
 * -1 / (2 sarg) on both branches (mos1.va:316-323). */
static double sbody(double vbx, double phit, double *ds) {
    double s;
    if (vbx <= 0.0) s = sqrt(phit - vbx);
    else s = fmax(sqrt(phit) - vbx / (2.0 * sqrt(phit)), 0.0);
    if (ds) *ds = s > 0.0 ? -1.0 / (2.0 * s) : 0.0;
    return s;
}

/* jchg (mos1.va:143-163) and its capacitance. */
static void jchg(double v, double cz, double czsw, double pbx, double mjx, double mjswx, double fcx,
                 double f2, double f3, double f4, double *q, double *c) {
    if (cz == 0.0 && czsw == 0.0) {
        *q = 0.0;
        *c = 0.0;
    } else if (v < fcx * pbx) {
        double a = 1.0 - v / pbx;
        *q = pbx * (cz * (1.0 - esl_pow(a, 1.0 - mjx)) / (1.0 - mjx) + czsw * (1.0 - esl_pow(a, 1.0 - mjswx)) / (1.0 - mjswx));
        *c = cz * esl_pow(a, -mjx) + czsw * esl_pow(a, -mjswx);
    } else {
        *q = f4 + v * (f2 + 0.5 * f3 * v);
        *c = f2 + f3 * v;
    }
}

void mos1_eval(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *lim, const double *st, const sim_t *sim, devout_t *o) {
    (void)prm;
    (void)st;
    memset(o, 0, sizeof(*o));
    const double type = der[MD_TYPE], vt = der[MD_VT];
    const double xd = x[nd[0]], xg = x[nd[1]], xs = x[nd[2]], xb = x[nd[3]], xdi = x[nd[4]], xsi = x[nd[5]];
    /* raw type-frame voltages, then the evaluation point */
    const double vgs_r = type * (xg - xsi), vds_r = type * (xdi - xsi), vbs_r = type * (xb - xsi);
    const double vgs = lim ? lim[0] : vgs_r, vds = lim ? lim[1] : vds_r, vbs = lim ? lim[2] : vbs_r;
    const double vbd = vbs - vds, vgd = vgs - vds;
    double ibs, gbs, ibd, gbd;
    jcur(vbs, der[MD_ISATS], vt, der[MD_GMIN], &ibs, &gbs);
    jcur(vbd, der[MD_ISATD], vt, der[MD_GMIN], &ibd, &gbd);

    /* mode swap and drain current (mos1.va:306-345) */
    const double mode = vds >= 0.0 ? 1.0 : -1.0;
    const double vbx = mode > 0 ? vbs : vbd;
    const double vgsx = mode > 0 ? vgs : vgd;
    const double vdsx = mode * vds;
    double ds;
    const double sarg = sbody(vbx, der[MD_PHIT], &ds);
    const double von = der[MD_VBIT] * type + der[MD_GAMMA] * sarg;
    const double vgst = vgsx - von;
    const double beta = der[MD_BETA], lambda = der[MD_LAMBDA];
    const double bp = beta * (1.0 + lambda * vdsx);
    double id = 0.0, gm = 0.0, gds = 0.0;
    if (vgst <= 0.0) {
        id = 0.0;
    } else if (vgst <= vdsx) {
        id = 0.5 * bp * vgst * vgst;
        gm = bp * vgst;
        gds = 0.5 * beta * lambda * vgst * vgst;
    } else {
        id = bp * vdsx * (vgst - 0.5 * vdsx);
        gm = bp * vdsx;
        gds = beta * lambda * vdsx * (vgst - 0.5 * vdsx) + bp * (vgst - vdsx);
    }
    const double gmbs = gm * (-der[MD_GAMMA] * ds);
    /* ich = mode * id and its type-frame partials in (vgs, vds, vbs) */
    double ich, gmg, gdd, gbb;
    if (mode > 0) {
        ich = id;
        gmg = gm;
        gdd = gds;
        gbb = gmbs;
    } else {
        ich = -id;
        gmg = -gm;
        gbb = -gmbs;
        gdd = gm + gds + gmbs;
    }
    const double cgs_ = vgs_r - vgs, cds = vds_r - vds, cbs = vbs_r - vbs;
    const double cbd = (vbs_r - vds_r) - vbd;
    if (lim) {
        if (cgs_ != 0.0 || cds != 0.0 || cbs != 0.0) ich = ich + (gmg * cgs_ + gdd * cds + gbb * cbs);
        if (cbs != 0.0) ibs = ibs + gbs * cbs;
        if (cbd != 0.0) ibd = ibd + gbd * cbd;
    }
    const double ids = type * ich, tbs = type * ibs, tbd = type * ibd;
    const double gdr = der[MD_GDRAIN], gsr = der[MD_GSOURCE];
    const double idr = gdr * (xd - xdi), isr = gsr * (xs - xsi);
    /* residuals: 0 d, 1 g, 2 s, 3 b, 4 di, 5 si */
    o->f[0] = idr;
    o->f[2] = isr;
    o->f[3] = tbd + tbs;
    o->f[4] = (ids - tbd) - idr;
    o->f[5] = ((-ids) - tbs) - isr;
    const double gsum = gmg + gdd + gbb;
    o->J[0][0] = gdr; o->J[0][4] = -gdr;
    o->J[2][2] = gsr; o->J[2][5] = -gsr;
    o->J[3][3] = gbd + gbs; o->J[3][4] = -gbd; o->J[3][5] = -gbs;
    o->J[4][0] = -gdr; o->J[4][1] = gmg; o->J[4][3] = gbb - gbd; o->J[4][4] = (gdd + gbd) + gdr; o->J[4][5] = -gsum;
    o->J[5][1] = -gmg; o->J[5][2] = -gsr; o->J[5][3] = (-gbb) - gbs; o->J[5][4] = -gdd; o->J[5][5] = (gsum + gbs) + gsr;

    if (sim->kind == 1 && der[MD_HASQ] != 0.0) {
        double qbd, cbdc, qbs, cbsc;
        jchg(vbd, der[MD_CZBD], der[MD_CZBDSW], der[MD_PBT], der[MD_MJ], der[MD_MJSW], der[MD_FC],
             der[MD_F2D], der[MD_F3D], der[MD_F4D], &qbd, &cbdc);
        jchg(vbs, der[MD_CZBS], der[MD_CZBSSW], der[MD_PBT], der[MD_MJ], der[MD_MJSW], der[MD_FC],
             der[MD_F2S], der[MD_F3S], der[MD_F4S], &qbs, &cbsc);
        if (lim) {
            if (cbd != 0.0) qbd = qbd + cbdc * cbd;
            if (cbs != 0.0) qbs = qbs + cbsc * cbs;
        }
        const double cgs = der[MD_CGS], cgd = der[MD_CGD], cgb = der[MD_CGB];
        const double qgs = cgs * (xg - xsi), qgd = cgd * (xg - xdi), qgb = cgb * (xg - xb);
        const double tqbd = type * qbd, tqbs = type * qbs;
        o->q[1] = (qgs + qgd) + qgb;
        o->q[3] = (tqbd + tqbs) - qgb;
        o->q[4] = (-tqbd) - qgd;
        o->q[5] = (-tqbs) - qgs;
        o->C[1][1] = (cgs + cgd) + cgb; o->C[1][3] = -cgb; o->C[1][4] = -cgd; o->C[1][5] = -cgs;
        o->C[3][1] = -cgb; o->C[3][3] = (cbdc + cbsc) + cgb; o->C[3][4] = -cbdc; o->C[3][5] = -cbsc;
        o->C[4][1] = -cgd; o->C[4][3] = -cbdc; o->C[4][4] = cbdc + cgd;
        o->C[5][1] = -cgs; o->C[5][3] = -cbsc; o->C[5][5] = cbsc + cgs;
    }
}

/* The limiting ladder of mos1load.c:361-384 in the type frame, against
 * the previous images (or x_old before the first pass). Returns pnjlim's
 * limited flag; fetlim and limvds clamp without vetoing convergence, as in
 * ngspice. Images within 16 ulps of the raw value snap to it, so a derived
 * leg's rounding never runs the correction (src/device/eval.zig:979-993). */
int mos1_limit(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *x_old, const double *lim_old, double *lim_new) {
    (void)prm;
    const double type = der[MD_TYPE], vt = der[MD_VT];
    const double xg = x[nd[1]], xb = x[nd[3]], xdi = x[nd[4]], xsi = x[nd[5]];
    const double vgs_n = type * (xg - xsi), vds_n = type * (xdi - xsi), vbs_n = type * (xb - xsi);
    const double vgd_n = type * (xg - xdi), vbd_n = type * (xb - xdi);
    double vgs_o, vds_o, vbs_o;
    if (lim_old) {
        vgs_o = lim_old[0];
        vds_o = lim_old[1];
        vbs_o = lim_old[2];
    } else {
        vgs_o = type * (x_old[nd[1]] - x_old[nd[5]]);
        vds_o = type * (x_old[nd[4]] - x_old[nd[5]]);
        vbs_o = type * (x_old[nd[3]] - x_old[nd[5]]);
    }
    const double vgd_o = vgs_o - vds_o, vbd_o = vbs_o - vds_o;
    const double vbx = vds_o >= 0.0 ? vbs_o : vbd_o;
    const double von = der[MD_VBIT] * type + der[MD_GAMMA] * sbody(vbx, der[MD_PHIT], NULL);
    double vgs, vds, vbs;
    if (vds_o >= 0.0) {
        vgs = fetlim(vgs_n, vgs_o, von);
        vds = vgs - vgd_n;
        vds = limvds(vds, vds_o);
    } else {
        double vgd = fetlim(vgd_n, vgd_o, von);
        vds = vgs_n - vgd;
        vds = -limvds(-vds, -vds_o);
        vgs = vgd + vds;
    }
    int l = 0;
    if (vds >= 0.0) {
        vbs = pnjlim(vbs_n, vbs_o, vt, der[MD_VCRITS], &l);
    } else {
        double vbd = pnjlim(vbd_n, vbd_o, vt, der[MD_VCRITD], &l);
        vbs = vbd + vds;
    }
    const double scale = fmax(fmax(fabs(xg), fabs(xb)), fmax(fabs(xdi), fabs(xsi)));
    const double tol = 16.0 * 2.220446049250313e-16 * scale;
    if (fabs(vgs - vgs_n) <= tol) vgs = vgs_n;
    if (fabs(vds - vds_n) <= tol) vds = vds_n;
    if (fabs(vbs - vbs_n) <= tol) vbs = vbs_n;
    lim_new[0] = vgs;
    lim_new[1] = vds;
    lim_new[2] = vbs;
    return l;
}

/* Meyer (overlap) gate charges, the sites mos1trun.c truncates: qgs, qgd,
 * qgb, each kept when its capacitance is nonzero. */
int mos1_qtape(const uint32_t *nd, const double *der, const double *x, double *out) {
    int k = 0;
    const double xg = x[nd[1]];
    if (der[MD_CGS] != 0.0) out[k++] = der[MD_CGS] * (xg - x[nd[5]]);
    if (der[MD_CGD] != 0.0) out[k++] = der[MD_CGD] * (xg - x[nd[4]]);
    if (der[MD_CGB] != 0.0) out[k++] = der[MD_CGB] * (xg - x[nd[3]]);
    return k;
}

/* MODEINITJCT (mos1load.c:397-407): vgs = type * tVto, vds = 0, vbs = -1. */
int mos1_seed(const uint32_t *nd, const double *prm, const double *der, const double *x, double *lim) {
    (void)nd; (void)prm; (void)x;
    lim[0] = der[MD_TYPE] * der[MD_VBIT] + der[MD_GAMMA] * sqrt(der[MD_PHIT]);
    lim[1] = 0.0;
    lim[2] = -1.0;
    return 1;
}
