/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * BSIM3v3.3 DC core, restated from models/bsim3.va:
 *   :186-376  bias-independent prep (b3temp.c): temperature, geometry,
 *             parameter defaulting by $param_given, junction sizing,
 *             series resistance
 *   :378-397  limiting: mos1's ladder (fetlim on the controlling gate leg,
 *             limvds, pnjlim on one bulk junction) with the zero-bias
 *             threshold type*vth0i as fetlim's threshold and pnjlim at the
 *             300.15 K thermal voltage; MODEINITJCT seeds vgs =
 *             type*vth0i + 0.1, vds = 0.1, vbs = 0
 *   :399-611  bulk junctions (jcur, :166-184), mode swap, the channel
 *             current chain of b3ld.c and the substrate current
 *   :613-624  contributions
 * The model has no charges (capMod is not built), as in the reference.
 *
 * Derivatives: the reference differentiates the value chain by VerA's
 * forward AD. Here every bias-dependent quantity is a dual number carrying
 * its partials in the type-frame (vgs, vds, vbs) images; the junction
 * currents take their closed-form slopes. A limited instance is evaluated
 * at its images and linearised back to x: f += df/dv . (v(x) - v_lim).
 * Parameter slots: ORC_B3_* (NaN = not given).
 */
#include "orc_internal.h"

#include <math.h>
#include <string.h>

enum {
    BD_TYPE, BD_MOBMOD, BD_VT, BD_TRATIO1, BD_VTH0I, BD_ISATS, BD_ISATD, BD_NVTMJ, BD_VJSM,
    BD_ISEVJSM, BD_VJDM, BD_ISEVJDM, BD_IJTH, BD_GMIN, BD_VBSC, BD_PHI, BD_SQRTPHI, BD_PHIS3,
    BD_XDEP0, BD_FACTOR1, BD_DVT2, BD_DVT2W, BD_DVT1, BD_DVT1W, BD_DVT0, BD_DVT0W, BD_LEFF,
    BD_WEFF, BD_VBI, BD_NLX, BD_K1X, BD_K1OX, BD_K2OX, BD_KT1, BD_KT1L, BD_KT2, BD_TOX, BD_W0,
    BD_K3, BD_K3B, BD_ETA0, BD_ETAB, BD_THETA0VB0, BD_NFACTOR, BD_CDSC, BD_CDSCB, BD_CDSCD,
    BD_CIT, BD_COX, BD_VFBI, BD_NGATE, BD_VOFF, BD_CDEP0, BD_DWG, BD_DWB, BD_RDS0, BD_PRWG,
    BD_PRWB, BD_XJ, BD_A0, BD_B0, BD_B1, BD_AGS, BD_KETA, BD_UA, BD_UB, BD_UC, BD_U0TEMP,
    BD_VSATTEMP, BD_A1, BD_A2, BD_DELTA, BD_PCLM, BD_LITL, BD_THETAROUT, BD_PDIBLCB, BD_PVAG,
    BD_PSCBE1, BD_PSCBE2, BD_ALPHA0, BD_ALPHA1, BD_BETA0, BD_M, BD_GDRAIN, BD_GSOURCE, BD_VT0,
    BD_VCRIT, BD_NDER
};

_Static_assert(BD_NDER <= ORC_NDER, "BSIM3 derived values exceed the per-instance block");
_Static_assert(ORC_B3_NP == 109, "BSIM3 parameter slots");

#define GIVEN(k) (!isnan(p[k]))

void bsim3_derive(const double *p, double *d) {
    memset(d, 0, sizeof(double) * ORC_NDER);
    const double type = p[ORC_B3_TYPE];
    const double tox = p[ORC_B3_TOX];
    /* temperature scaling (bsim3.va:188-212) */
    const double tnomk = p[ORC_B3_TNOM] + 273.15;
    const double tk = p[ORC_B3_TEMP];
    const double tratio = tk / tnomk;
    const double vtnom = 8.617087e-5 * tnomk;
    const double vt = 8.617087e-5 * tk;
    const double eg0 = 1.16 - 7.02e-4 * tnomk * tnomk / (tnomk + 1108.0);
    const double eg = 1.16 - 7.02e-4 * tk * tk / (tk + 1108.0);
    const double ni = 1.45e10 * (tnomk / 300.15) * sqrt(tnomk / 300.15) * esl_exp(21.5565981 - eg0 / (2.0 * vtnom));
    const double cox = 3.453133e-11 / tox;
    const double factor1 = sqrt(1.03594e-10 / 3.453133e-11 * tox);
    const double vt0 = 1.38064852e-23 * 300.15 / 1.6021766208e-19;
    const double vcrit = vt0 * esl_log(vt0 / (1.4142135623730951 * 1.0e-14));
    double jst, jswt;
    if (tk != tnomk) {
        const double jtmp = esl_exp((eg0 / vtnom - eg / vt + p[ORC_B3_XTI] * esl_log(tratio)) / p[ORC_B3_NJ]);
        jst = p[ORC_B3_JS] * jtmp;
        jswt = p[ORC_B3_JSW] * jtmp;
    } else {
        jst = p[ORC_B3_JS];
        jswt = p[ORC_B3_JSW];
    }
    if (jst < 0.0) jst = 0.0;
    if (jswt < 0.0) jswt = 0.0;

    /* geometry (:214-229) */
    const double l = p[ORC_B3_L], w = p[ORC_B3_W];
    double t0 = esl_pow(l, p[ORC_B3_LLN]);
    double t1 = esl_pow(w, p[ORC_B3_LWN]);
    const double dl = p[ORC_B3_LINT] + p[ORC_B3_LL] / t0 + p[ORC_B3_LW] / t1 + p[ORC_B3_LWL] / (t0 * t1);
    double t2 = esl_pow(l, p[ORC_B3_WLN]);
    double t3 = esl_pow(w, p[ORC_B3_WWN]);
    const double dwx = p[ORC_B3_WINT] + p[ORC_B3_WL] / t2 + p[ORC_B3_WW] / t3 + p[ORC_B3_WWL] / (t2 * t3);
    double leff = l + p[ORC_B3_XL] - 2.0 * dl;
    double weff = w + p[ORC_B3_XW] - 2.0 * dwx;
    if (leff < 1.0e-9) leff = 1.0e-9;
    if (weff < 1.0e-9) weff = 1.0e-9;

    /* mobility and velocity temperature (:231-247) */
    const double uax = p[ORC_B3_UA] + p[ORC_B3_UA1] * (tratio - 1.0);
    const double ubx = p[ORC_B3_UB] + p[ORC_B3_UB1] * (tratio - 1.0);
    const int mobmod = (int)p[ORC_B3_MOBMOD];
    double ucx, uc1x, u0x;
    if (GIVEN(ORC_B3_UC)) ucx = p[ORC_B3_UC];
    else if (mobmod == 3) ucx = -0.0465;
    else ucx = -0.0465e-9;
    if (GIVEN(ORC_B3_UC1)) uc1x = p[ORC_B3_UC1];
    else if (mobmod == 3) uc1x = -0.056;
    else uc1x = -0.056e-9;
    ucx = ucx + uc1x * (tratio - 1.0);
    if (GIVEN(ORC_B3_U0)) u0x = p[ORC_B3_U0];
    else if (type > 0.0) u0x = 0.067;
    else u0x = 0.025;
    if (u0x > 1.0) u0x = u0x / 1.0e4;
    const double u0temp = u0x * esl_pow(tratio, p[ORC_B3_UTE]) * p[ORC_B3_MULU0];
    const double vsattemp = p[ORC_B3_VSAT] - p[ORC_B3_AT] * (tratio - 1.0);
    const double rds0 = (p[ORC_B3_RDSW] + p[ORC_B3_PRT] * (tratio - 1.0)) / esl_pow(weff * 1.0e6, p[ORC_B3_WR]);

    /* doping-derived quantities (:249-268) */
    double npeakx;
    if (GIVEN(ORC_B3_NCH)) {
        npeakx = p[ORC_B3_NCH];
        if (npeakx > 1.0e20) npeakx = npeakx * 1.0e-6;
    } else if (GIVEN(ORC_B3_GAMMA1)) {
        t0 = p[ORC_B3_GAMMA1] * cox;
        npeakx = 3.021e22 * t0 * t0;
    } else {
        npeakx = 1.7e17;
    }
    double ngatex = p[ORC_B3_NGATE];
    if (ngatex > 1.000001e24) ngatex = ngatex * 1.0e-6;
    const double phi = 2.0 * vtnom * esl_log(npeakx / ni);
    const double sqrtphi = sqrt(phi);
    const double phis3 = sqrtphi * phi;
    const double xdep0 = sqrt(2.0 * 1.03594e-10 / (1.60219e-19 * npeakx * 1.0e6)) * sqrtphi;
    const double litl = sqrt(3.0 * p[ORC_B3_XJ] * tox);
    const double vbi = vtnom * esl_log(1.0e20 * npeakx / (ni * ni));
    const double cdep0 = sqrt(1.60219e-19 * 1.03594e-10 * npeakx * 1.0e6 / 2.0 / phi);

    /* k1/k2 ladder (:270-290) */
    double vbmx = p[ORC_B3_VBM], k1x, k2x;
    if (GIVEN(ORC_B3_K1) || GIVEN(ORC_B3_K2)) {
        k1x = GIVEN(ORC_B3_K1) ? p[ORC_B3_K1] : 0.53;
        k2x = GIVEN(ORC_B3_K2) ? p[ORC_B3_K2] : -0.0186;
    } else {
        const double xt = p[ORC_B3_XT];
        double vbxx = GIVEN(ORC_B3_VBX) ? p[ORC_B3_VBX] : phi - 7.7348e-4 * npeakx * xt * xt;
        if (vbxx > 0.0) vbxx = -vbxx;
        if (vbmx > 0.0) vbmx = -vbmx;
        const double g1 = GIVEN(ORC_B3_GAMMA1) ? p[ORC_B3_GAMMA1] : 5.753e-12 * sqrt(npeakx) / cox;
        const double g2 = GIVEN(ORC_B3_GAMMA2) ? p[ORC_B3_GAMMA2] : 5.753e-12 * sqrt(p[ORC_B3_NSUB]) / cox;
        t0 = g1 - g2;
        t1 = sqrt(phi - vbxx) - sqrtphi;
        t2 = sqrt(phi * (phi - vbmx)) - phi;
        k2x = t0 * t1 / (2.0 * t2 + vbmx);
        k1x = g2 - 2.0 * k2x * sqrt(phi - vbmx);
    }
    double vbsc;
    if (k2x < 0.0) {
        t0 = 0.5 * k1x / k2x;
        vbsc = 0.9 * (phi - t0 * t0);
        if (vbsc > -3.0) vbsc = -3.0;
        else if (vbsc < -30.0) vbsc = -30.0;
    } else {
        vbsc = -30.0;
    }
    if (vbsc > vbmx) vbsc = vbmx;

    /* vfb / vth0 mutual defaults (:300-309) */
    double vfbx, vth0x;
    if (GIVEN(ORC_B3_VFB)) vfbx = p[ORC_B3_VFB];
    else if (GIVEN(ORC_B3_VTH0)) vfbx = type * p[ORC_B3_VTH0] - phi - k1x * sqrtphi;
    else vfbx = -1.0;
    if (GIVEN(ORC_B3_VTH0)) vth0x = p[ORC_B3_VTH0];
    else vth0x = type * (vfbx + phi + k1x * sqrtphi);
    const double vth0i = vth0x + p[ORC_B3_DELVTO];
    const double vfbi = vfbx + type * p[ORC_B3_DELVTO];
    const double toxmx = GIVEN(ORC_B3_TOXM) ? p[ORC_B3_TOXM] : tox;
    const double k1ox = k1x * tox / toxmx;
    const double k2ox = k2x * tox / toxmx;

    const double dsubx = GIVEN(ORC_B3_DSUB) ? p[ORC_B3_DSUB] : p[ORC_B3_DROUT];
    const double lt0 = factor1 * sqrt(xdep0);
    t0 = esl_exp(-0.5 * dsubx * leff / lt0);
    const double theta0vb0 = t0 + 2.0 * t0 * t0;
    t0 = esl_exp(-0.5 * p[ORC_B3_DROUT] * leff / lt0);
    const double thetarout = p[ORC_B3_PDIBLC1] * (t0 + 2.0 * t0 * t0) + p[ORC_B3_PDIBLC2];

    /* junction sizing (:323-338) */
    const double nvtmj = vt * p[ORC_B3_NJ];
    const double as = p[ORC_B3_AS], ps = p[ORC_B3_PS], ad = p[ORC_B3_AD], pd = p[ORC_B3_PD];
    const double ijth = p[ORC_B3_IJTH];
    const double isats = (as <= 0.0 && ps <= 0.0) ? 1.0e-14 : as * jst + ps * jswt;
    const double isatd = (ad <= 0.0 && pd <= 0.0) ? 1.0e-14 : ad * jst + pd * jswt;
    double vjsm = 0.0, isevjsm = 0.0, vjdm = 0.0, isevjdm = 0.0;
    if (isats > 0.0 && ijth > 0.0) {
        vjsm = nvtmj * esl_log(ijth / isats + 1.0);
        isevjsm = isats * esl_exp(vjsm / nvtmj);
    }
    if (isatd > 0.0 && ijth > 0.0) {
        vjdm = nvtmj * esl_log(ijth / isatd + 1.0);
        isevjdm = isatd * esl_exp(vjdm / nvtmj);
    }

    /* series resistance (:340-346) */
    const double m = p[ORC_B3_M], rsh = p[ORC_B3_RSH];
    const double gdrain = (rsh > 0.0 && p[ORC_B3_NRD] > 0.0) ? m / (rsh * p[ORC_B3_NRD]) : 0.0;
    const double gsource = (rsh > 0.0 && p[ORC_B3_NRS] > 0.0) ? m / (rsh * p[ORC_B3_NRS]) : 0.0;

    d[BD_TYPE] = type;
    d[BD_MOBMOD] = (double)mobmod;
    d[BD_VT] = vt;
    d[BD_TRATIO1] = tk / tnomk - 1.0;
    d[BD_VTH0I] = vth0i;
    d[BD_ISATS] = isats;
    d[BD_ISATD] = isatd;
    d[BD_NVTMJ] = nvtmj;
    d[BD_VJSM] = vjsm;
    d[BD_ISEVJSM] = isevjsm;
    d[BD_VJDM] = vjdm;
    d[BD_ISEVJDM] = isevjdm;
    d[BD_IJTH] = ijth;
    d[BD_GMIN] = p[ORC_B3_GMIN];
    d[BD_VBSC] = vbsc;
    d[BD_PHI] = phi;
    d[BD_SQRTPHI] = sqrtphi;
    d[BD_PHIS3] = phis3;
    d[BD_XDEP0] = xdep0;
    d[BD_FACTOR1] = factor1;
    d[BD_DVT2] = p[ORC_B3_DVT2];
    d[BD_DVT2W] = p[ORC_B3_DVT2W];
    d[BD_DVT1] = p[ORC_B3_DVT1];
    d[BD_DVT1W] = p[ORC_B3_DVT1W];
    d[BD_DVT0] = p[ORC_B3_DVT0];
    d[BD_DVT0W] = p[ORC_B3_DVT0W];
    d[BD_LEFF] = leff;
    d[BD_WEFF] = weff;
    d[BD_VBI] = vbi;
    d[BD_NLX] = p[ORC_B3_NLX];
    d[BD_K1X] = k1x;
    d[BD_K1OX] = k1ox;
    d[BD_K2OX] = k2ox;
    d[BD_KT1] = p[ORC_B3_KT1];
    d[BD_KT1L] = p[ORC_B3_KT1L];
    d[BD_KT2] = p[ORC_B3_KT2];
    d[BD_TOX] = tox;
    d[BD_W0] = p[ORC_B3_W0];
    d[BD_K3] = p[ORC_B3_K3];
    d[BD_K3B] = p[ORC_B3_K3B];
    d[BD_ETA0] = p[ORC_B3_ETA0];
    d[BD_ETAB] = p[ORC_B3_ETAB];
    d[BD_THETA0VB0] = theta0vb0;
    d[BD_NFACTOR] = p[ORC_B3_NFACTOR];
    d[BD_CDSC] = p[ORC_B3_CDSC];
    d[BD_CDSCB] = p[ORC_B3_CDSCB];
    d[BD_CDSCD] = p[ORC_B3_CDSCD];
    d[BD_CIT] = p[ORC_B3_CIT];
    d[BD_COX] = cox;
    d[BD_VFBI] = vfbi;
    d[BD_NGATE] = ngatex;
    d[BD_VOFF] = p[ORC_B3_VOFF];
    d[BD_CDEP0] = cdep0;
    d[BD_DWG] = p[ORC_B3_DWG];
    d[BD_DWB] = p[ORC_B3_DWB];
    d[BD_RDS0] = rds0;
    d[BD_PRWG] = p[ORC_B3_PRWG];
    d[BD_PRWB] = p[ORC_B3_PRWB];
    d[BD_XJ] = p[ORC_B3_XJ];
    d[BD_A0] = p[ORC_B3_A0];
    d[BD_B0] = p[ORC_B3_B0];
    d[BD_B1] = p[ORC_B3_B1];
    d[BD_AGS] = p[ORC_B3_AGS];
    d[BD_KETA] = p[ORC_B3_KETA];
    d[BD_UA] = uax;
    d[BD_UB] = ubx;
    d[BD_UC] = ucx;
    d[BD_U0TEMP] = u0temp;
    d[BD_VSATTEMP] = vsattemp;
    d[BD_A1] = p[ORC_B3_A1];
    d[BD_A2] = p[ORC_B3_A2];
    d[BD_DELTA] = p[ORC_B3_DELTA];
    d[BD_PCLM] = p[ORC_B3_PCLM];
    d[BD_LITL] = litl;
    d[BD_THETAROUT] = thetarout;
    d[BD_PDIBLCB] = p[ORC_B3_PDIBLCB];
    d[BD_PVAG] = p[ORC_B3_PVAG];
    d[BD_PSCBE1] = p[ORC_B3_PSCBE1];
    d[BD_PSCBE2] = p[ORC_B3_PSCBE2];
    d[BD_ALPHA0] = p[ORC_B3_ALPHA0];
    d[BD_ALPHA1] = p[ORC_B3_ALPHA1];
    d[BD_BETA0] = p[ORC_B3_BETA0];
    d[BD_M] = m;
    d[BD_GDRAIN] = gdrain;
    d[BD_GSOURCE] = gsource;
    d[BD_VT0] = vt0;
    d[BD_VCRIT] = vcrit;
}

/* ------------------------------------------------------------------ */
/* dual numbers: a value and its partials in the (vgs, vds, vbs) images */

typedef struct {
    double v, g, d, b;
} dual;

static dual dk(double c) {
    dual r = {c, 0.0, 0.0, 0.0};
    return r;
}
static dual dadd(dual a, dual b) {
    dual r = {a.v + b.v, a.g + b.g, a.d + b.d, a.b + b.b};
    return r;
}
static dual dsub(dual a, dual b) {
    dual r = {a.v - b.v, a.g - b.g, a.d - b.d, a.b - b.b};
    return r;
}
static dual dneg(dual a) {
    dual r = {-a.v, -a.g, -a.d, -a.b};
    return r;
}
static dual dmul(dual a, dual b) {
    dual r = {a.v * b.v, a.g * b.v + a.v * b.g, a.d * b.v + a.v * b.d, a.b * b.v + a.v * b.b};
    return r;
}
/* a * c, c a constant */
static dual dscl(dual a, double c) {
    dual r = {a.v * c, a.g * c, a.d * c, a.b * c};
    return r;
}
static dual ddiv(dual a, dual b) {
    const double q = a.v / b.v;
    dual r = {q, (a.g - q * b.g) / b.v, (a.d - q * b.d) / b.v, (a.b - q * b.b) / b.v};
    return r;
}
/* a / c, c a constant */
static dual ddivk(dual a, double c) {
    dual r = {a.v / c, a.g / c, a.d / c, a.b / c};
    return r;
}
/* c / b, c a constant */
static dual dkdiv(double c, dual b) {
    const double q = c / b.v;
    const double s = -q / b.v;
    dual r = {q, s * b.g, s * b.d, s * b.b};
    return r;
}
static dual dsqrt(dual a) {
    const double s = sqrt(a.v);
    const double h = 0.5 / s;
    dual r = {s, a.g * h, a.d * h, a.b * h};
    return r;
}
static dual dexp(dual a) {
    const double e = esl_exp(a.v);
    dual r = {e, a.g * e, a.d * e, a.b * e};
    return r;
}
static dual dlog(dual a) {
    dual r = {esl_log(a.v), a.g / a.v, a.d / a.v, a.b / a.v};
    return r;
}
/* a + c and c - a, c a constant */
static dual daddk(dual a, double c) {
    dual r = {a.v + c, a.g, a.d, a.b};
    return r;
}
static dual dksub(double c, dual a) {
    dual r = {c - a.v, -a.g, -a.d, -a.b};
    return r;
}

/* jcur (bsim3.va:166-184) and its slope. */
static void b3_jcur(double v, double isat, double nvt, double vjm, double isevjm, double ijth, double gmin,
                    double *i, double *g) {
    if (isat <= 0.0) {
        *i = gmin * v;
        *g = gmin;
    } else if (ijth > 0.0 && v >= vjm) {
        *i = isevjm - isat + (isevjm / nvt) * (v - vjm) + gmin * v;
        *g = isevjm / nvt + gmin;
    } else {
        const double u = fmin(v / nvt, 80.0);
        const double e = esl_exp(u);
        *i = isat * (e * (1.0 + (v / nvt - u)) - 1.0) + gmin * v;
        *g = isat * e / nvt + gmin;
    }
}

/* The channel current id and substrate current isubst in the swapped frame
 * (bsim3.va:420-611), from the swapped duals vgsx, vdsx, vbsx. */
static void b3_channel(const double *q, dual vgsx, dual vdsx, dual vbsx, dual *id_out, dual *isub_out) {
    const double vt = q[BD_VT], phi = q[BD_PHI], sqrtphi = q[BD_SQRTPHI], vbsc = q[BD_VBSC];
    const double leff = q[BD_LEFF], weff = q[BD_WEFF], tox = q[BD_TOX], cox = q[BD_COX];
    const double type = q[BD_TYPE];
    dual t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, tmp1, tmp2, tmp3, tmp4;

    /* Vbseff, Phis, Xdep */
    t0 = daddk(daddk(vbsx, -vbsc), -0.001);
    t1 = dsqrt(dsub(dmul(t0, t0), dk(0.004 * vbsc)));
    dual vbseff = daddk(dscl(dadd(t0, t1), 0.5), vbsc);
    if (vbseff.v < vbsx.v) vbseff = vbsx;
    dual phis, sqrtphis;
    if (vbseff.v > 0.0) {
        t0 = dkdiv(phi, daddk(vbseff, phi));
        phis = dscl(t0, phi);
        sqrtphis = dkdiv(q[BD_PHIS3], daddk(dscl(vbseff, 0.5), phi));
    } else {
        phis = dksub(phi, vbseff);
        sqrtphis = dsqrt(phis);
    }
    dual xdep = ddivk(dscl(sqrtphis, q[BD_XDEP0]), sqrtphi);

    /* Vth */
    t3 = dsqrt(xdep);
    t0 = dscl(vbseff, q[BD_DVT2]);
    if (t0.v >= -0.5) t1 = daddk(t0, 1.0);
    else t1 = ddiv(daddk(dscl(t0, 3.0), 1.0), daddk(dscl(t0, 8.0), 3.0));
    dual lt1 = dmul(dscl(t3, q[BD_FACTOR1]), t1);
    t0 = dscl(vbseff, q[BD_DVT2W]);
    if (t0.v >= -0.5) t1 = daddk(t0, 1.0);
    else t1 = ddiv(daddk(dscl(t0, 3.0), 1.0), daddk(dscl(t0, 8.0), 3.0));
    dual ltw = dmul(dscl(t3, q[BD_FACTOR1]), t1);

    t0 = dkdiv(-0.5 * q[BD_DVT1] * leff, lt1);
    if (t0.v > -34.0) t1 = dexp(t0);
    else t1 = dk(1.713908431e-15);
    dual theta0 = dmul(t1, daddk(dscl(t1, 2.0), 1.0));
    dual deltvth = dscl(dscl(theta0, q[BD_DVT0]), q[BD_VBI] - phi);

    t0 = dkdiv(-0.5 * q[BD_DVT1W] * weff * leff, ltw);
    if (t0.v > -34.0) t1 = dexp(t0);
    else t1 = dk(1.713908431e-15);
    dual dvthw = dscl(dmul(dscl(t1, q[BD_DVT0W]), daddk(dscl(t1, 2.0), 1.0)), q[BD_VBI] - phi);

    const double tempratio = q[BD_TRATIO1];
    const double nlxt = sqrt(1.0 + q[BD_NLX] / leff);
    t5 = daddk(dscl(daddk(dscl(vbseff, q[BD_KT2]), q[BD_KT1] + q[BD_KT1L] / leff), tempratio),
               q[BD_K1OX] * (nlxt - 1.0) * sqrtphi);
    const double tmp2k = tox * phi / (weff + q[BD_W0]);

    t3 = daddk(dscl(vbseff, q[BD_ETAB]), q[BD_ETA0]);
    if (t3.v < 1.0e-4) t3 = ddiv(dksub(2.0e-4, t3), dksub(3.0, dscl(t3, 2.0e4)));
    dual diblsft = dmul(dscl(t3, q[BD_THETA0VB0]), vdsx);

    dual vth = dk(type * q[BD_VTH0I] - q[BD_K1X] * sqrtphi);
    vth = dadd(vth, dscl(sqrtphis, q[BD_K1OX]));
    vth = dsub(vth, dscl(vbseff, q[BD_K2OX]));
    vth = dsub(vth, deltvth);
    vth = dsub(vth, dvthw);
    vth = dadd(vth, dscl(daddk(dscl(vbseff, q[BD_K3B]), q[BD_K3]), tmp2k));
    vth = dadd(vth, t5);
    vth = dsub(vth, diblsft);

    /* n, the subthreshold swing */
    tmp2 = dkdiv(q[BD_NFACTOR] * 1.03594e-10, xdep);
    tmp3 = dadd(daddk(dscl(vbseff, q[BD_CDSCB]), q[BD_CDSC]), dscl(vdsx, q[BD_CDSCD]));
    tmp4 = ddivk(daddk(dadd(tmp2, dmul(tmp3, theta0)), q[BD_CIT]), cox);
    dual n;
    if (tmp4.v >= -0.5) n = daddk(tmp4, 1.0);
    else n = ddiv(daddk(dscl(tmp4, 3.0), 1.0), daddk(dscl(tmp4, 8.0), 3.0));

    /* poly gate depletion, Vgsteff */
    const double vfbphi = q[BD_VFBI] + phi;
    const double ngatex = q[BD_NGATE];
    dual vgs_eff;
    if (ngatex > 1.0e18 && ngatex < 1.0e25 && vgsx.v > vfbphi) {
        const double k = 1.0e6 * 1.60219e-19 * 1.03594e-10 * ngatex / (cox * cox);
        t4 = dsqrt(daddk(ddivk(dscl(daddk(vgsx, -vfbphi), 2.0), k), 1.0));
        t2 = dscl(daddk(t4, -1.0), k);
        t3 = ddivk(dscl(dmul(t2, t2), 0.5), k);
        t7 = daddk(dksub(1.12, t3), -0.05);
        t6 = dsqrt(daddk(dmul(t7, t7), 0.224));
        vgs_eff = dsub(vgsx, dksub(1.12, dscl(dadd(t7, t6), 0.5)));
    } else {
        vgs_eff = vgsx;
    }
    dual vgst = dsub(vgs_eff, vth);

    t10 = dscl(n, 2.0 * vt);
    t11 = ddiv(vgst, t10);
    t9 = ddiv(dksub(2.0 * q[BD_VOFF], vgst), t10);
    dual vgsteff;
    if (t11.v > 34.0) {
        vgsteff = vgst;
    } else if (t9.v > 34.0) {
        t0 = ddiv(daddk(vgst, -q[BD_VOFF]), dscl(n, vt));
        vgsteff = dscl(dexp(t0), vt * q[BD_CDEP0] / cox);
    } else {
        dual expvgst = dexp(t11);
        t1 = dmul(t10, dlog(daddk(expvgst, 1.0)));
        t2 = daddk(dmul(ddivk(dscl(t10, cox), vt * q[BD_CDEP0]), dexp(t9)), 1.0);
        vgsteff = ddiv(t1, t2);
    }

    /* Weff', Rds, Abulk */
    t9 = daddk(sqrtphis, -sqrtphi);
    dual weffp = dksub(weff, dscl(dadd(dscl(vgsteff, q[BD_DWG]), dscl(t9, q[BD_DWB])), 2.0));
    if (weffp.v < 2.0e-8) weffp = ddiv(dscl(dksub(4.0e-8, weffp), 2.0e-8), dksub(6.0e-8, dscl(weffp, 2.0)));
    t0 = dadd(dscl(vgsteff, q[BD_PRWG]), dscl(t9, q[BD_PRWB]));
    dual rds;
    if (t0.v >= -0.9) rds = dscl(daddk(t0, 1.0), q[BD_RDS0]);
    else rds = ddiv(dscl(daddk(t0, 0.8), q[BD_RDS0]), daddk(dscl(t0, 20.0), 17.0));

    t1 = dkdiv(0.5 * q[BD_K1OX], sqrtphis);
    t9 = dsqrt(dscl(xdep, q[BD_XJ]));
    tmp1 = daddk(dscl(t9, 2.0), leff);
    t5 = dkdiv(leff, tmp1);
    tmp2 = dscl(t5, q[BD_A0]);
    const double tmp4k = q[BD_B0] / (weff + q[BD_B1]);
    t2 = daddk(tmp2, tmp4k);
    t6 = dmul(t5, t5);
    t7 = dmul(t5, t6);
    dual abulk0 = daddk(dmul(t1, t2), 1.0);
    t8 = dscl(t7, q[BD_AGS] * q[BD_A0]);
    dual abulk = dsub(abulk0, dmul(dmul(t1, t8), vgsteff));
    if (abulk0.v < 0.1) abulk0 = ddiv(dksub(0.2, abulk0), dksub(3.0, dscl(abulk0, 20.0)));
    if (abulk.v < 0.1) abulk = ddiv(dksub(0.2, abulk), dksub(3.0, dscl(abulk, 20.0)));
    t2 = dscl(vbseff, q[BD_KETA]);
    if (t2.v >= -0.9) t0 = dkdiv(1.0, daddk(t2, 1.0));
    else t0 = ddiv(daddk(dscl(t2, 20.0), 17.0), daddk(t2, 0.8));
    abulk = dmul(abulk, t0);
    abulk0 = dmul(abulk0, t0);

    /* mobility */
    const int mobmod = (int)q[BD_MOBMOD];
    if (mobmod == 1) {
        t0 = dadd(dadd(vgsteff, vth), vth);
        t2 = daddk(dscl(vbseff, q[BD_UC]), q[BD_UA]);
        t3 = ddivk(t0, tox);
        t5 = dmul(t3, dadd(t2, dscl(t3, q[BD_UB])));
    } else if (mobmod == 2) {
        t5 = dmul(ddivk(vgsteff, tox),
                  dadd(daddk(dscl(vbseff, q[BD_UC]), q[BD_UA]), ddivk(dscl(vgsteff, q[BD_UB]), tox)));
    } else {
        t0 = dadd(dadd(vgsteff, vth), vth);
        t2 = daddk(dscl(vbseff, q[BD_UC]), 1.0);
        t3 = ddivk(t0, tox);
        t4 = dmul(t3, daddk(dscl(t3, q[BD_UB]), q[BD_UA]));
        t5 = dmul(t4, t2);
    }
    dual denomi;
    if (t5.v >= -0.8) denomi = daddk(t5, 1.0);
    else denomi = ddiv(daddk(t5, 0.6), daddk(dscl(t5, 10.0), 7.0));
    dual ueff = dkdiv(q[BD_U0TEMP], denomi);

    /* Esat, Lambda, Vdsat */
    const double vsattemp = q[BD_VSATTEMP];
    dual wvcox = dscl(dscl(weffp, vsattemp), cox);
    dual wvcoxrds = dmul(wvcox, rds);
    dual esat = dkdiv(2.0 * vsattemp, ueff);
    dual esatl = dscl(esat, leff);
    const double a1 = q[BD_A1], a2 = q[BD_A2];
    dual lambda;
    if (a1 == 0.0) {
        lambda = dk(a2);
    } else if (a1 > 0.0) {
        const double c0 = 1.0 - a2;
        t1 = daddk(dksub(c0, dscl(vgsteff, a1)), -0.0001);
        t2 = dsqrt(daddk(dmul(t1, t1), 0.0004 * c0));
        lambda = dksub(a2 + c0, dscl(dadd(t1, t2), 0.5));
    } else {
        t1 = daddk(daddk(dscl(vgsteff, a1), a2), -0.0001);
        t2 = dsqrt(daddk(dmul(t1, t1), 0.0004 * a2));
        lambda = dscl(dadd(t1, t2), 0.5);
    }
    dual vgst2vtm = daddk(vgsteff, 2.0 * vt);
    dual vdsat;
    if (rds.v == 0.0 && lambda.v == 1.0) {
        vdsat = ddiv(dmul(esatl, vgst2vtm), dadd(dmul(abulk, esatl), vgst2vtm));
    } else {
        t9 = dmul(abulk, wvcoxrds);
        t7 = dmul(vgst2vtm, t9);
        t6 = dmul(vgst2vtm, wvcoxrds);
        t0 = dscl(dmul(abulk, dadd(daddk(t9, -1.0), dkdiv(1.0, lambda))), 2.0);
        t1 = dadd(dadd(dmul(vgst2vtm, daddk(dkdiv(2.0, lambda), -1.0)), dmul(abulk, esatl)), dscl(t7, 3.0));
        t2 = dmul(vgst2vtm, dadd(esatl, dscl(t6, 2.0)));
        t3 = dsqrt(dsub(dmul(t1, t1), dmul(dscl(t0, 2.0), t2)));
        vdsat = ddiv(dsub(t1, t3), t0);
    }

    /* Vdseff */
    const double delta = q[BD_DELTA];
    t1 = daddk(dsub(vdsat, vdsx), -delta);
    t2 = dsqrt(dadd(dmul(t1, t1), dscl(vdsat, 4.0 * delta)));
    dual vdseff = dsub(vdsat, dscl(dadd(t1, t2), 0.5));
    if (vdsx.v == 0.0) vdseff = dk(0.0);

    /* VAsat (from Vdsat and the unclamped Vdseff) */
    tmp4 = dksub(1.0, ddiv(dscl(dmul(abulk, vdsat), 0.5), vgst2vtm));
    t9 = dmul(wvcoxrds, vgsteff);
    t0 = dadd(dadd(esatl, vdsat), dmul(dscl(t9, 2.0), tmp4));
    t9 = dmul(wvcoxrds, abulk);
    t1 = dadd(daddk(dkdiv(2.0, lambda), -1.0), t9);
    dual vasat = ddiv(t0, t1);
    if (vdseff.v > vdsx.v) vdseff = vdsx;
    dual diffvds = dsub(vdsx, vdseff);

    /* VACLM, VADIBL, VA, VASCBE */
    const double pclm = q[BD_PCLM], litl = q[BD_LITL];
    dual vaclm;
    if (pclm > 0.0 && diffvds.v > 1.0e-10) {
        t0 = dkdiv(1.0, dscl(dscl(abulk, pclm), litl));
        t2 = ddiv(vgsteff, esatl);
        t1 = dscl(dadd(abulk, t2), leff);
        vaclm = dmul(dmul(t0, t1), diffvds);
    } else {
        vaclm = dk(5.834617425e14);
    }
    const double thetarout = q[BD_THETAROUT];
    dual vadibl;
    if (thetarout > 0.0) {
        t8 = dmul(abulk, vdsat);
        t0 = dmul(vgst2vtm, t8);
        t1 = dadd(vgst2vtm, t8);
        vadibl = ddivk(dsub(vgst2vtm, ddiv(t0, t1)), thetarout);
        t7 = dscl(vbseff, q[BD_PDIBLCB]);
        if (t7.v >= -0.9) vadibl = ddiv(vadibl, daddk(t7, 1.0));
        else vadibl = ddiv(dmul(vadibl, daddk(dscl(t7, 20.0), 17.0)), daddk(t7, 0.8));
    } else {
        vadibl = dk(5.834617425e14);
    }
    t8 = dkdiv(q[BD_PVAG], esatl);
    t9 = dmul(t8, vgsteff);
    if (t9.v > -0.9) t0 = daddk(t9, 1.0);
    else t0 = ddiv(daddk(t9, 0.8), daddk(dscl(t9, 20.0), 17.0));
    t1 = ddiv(dmul(vaclm, vadibl), dadd(vaclm, vadibl));
    dual va = dadd(vasat, dmul(t0, t1));
    const double pscbe1 = q[BD_PSCBE1], pscbe2 = q[BD_PSCBE2];
    dual vascbe;
    if (pscbe2 > 0.0) {
        if (diffvds.v > pscbe1 * litl / 34.0)
            vascbe = ddivk(dscl(dexp(dkdiv(pscbe1 * litl, diffvds)), leff), pscbe2);
        else
            vascbe = dk(5.834617425e14 * leff / pscbe2);
    } else {
        vascbe = dk(5.834617425e14);
    }

    /* Ids chain */
    dual betax = ddivk(dmul(dscl(ueff, cox), weffp), leff);
    dual fgche1 = dmul(vgsteff, dksub(1.0, ddiv(dscl(dmul(abulk, vdseff), 0.5), vgst2vtm)));
    dual fgche2 = daddk(ddiv(vdseff, esatl), 1.0);
    dual gche = ddiv(dmul(betax, fgche1), fgche2);
    dual idl = ddiv(dmul(gche, vdseff), daddk(dmul(gche, rds), 1.0));
    dual idsa = dmul(idl, daddk(ddiv(diffvds, va), 1.0));
    *id_out = dmul(idsa, daddk(ddiv(diffvds, vascbe), 1.0));

    /* substrate (impact ionisation) current */
    const double tmp1k = q[BD_ALPHA0] + q[BD_ALPHA1] * leff;
    const double beta0 = q[BD_BETA0];
    if (tmp1k <= 0.0 || beta0 <= 0.0) {
        *isub_out = dk(0.0);
    } else {
        const double t2k = tmp1k / leff;
        if (diffvds.v > beta0 / 34.0)
            t1 = dmul(dscl(diffvds, t2k), dexp(dkdiv(-beta0, diffvds)));
        else
            t1 = dscl(diffvds, t2k * 1.713908431e-15);
        *isub_out = dmul(t1, idsa);
    }
}

void bsim3_eval(const uint32_t *nd, const double *der, const double *x, const double *lim, double gmin,
                devout_t *o) {
    memset(o, 0, sizeof(*o));
    const double *q = der;
    const double type = q[BD_TYPE], m = q[BD_M];
    const double xd = x[nd[0]], xg = x[nd[1]], xs = x[nd[2]], xb = x[nd[3]], xdi = x[nd[4]], xsi = x[nd[5]];
    const double vgs_r = type * (xg - xsi), vds_r = type * (xdi - xsi), vbs_r = type * (xb - xsi);
    const double vgs_v = lim ? lim[0] : vgs_r, vds_v = lim ? lim[1] : vds_r, vbs_v = lim ? lim[2] : vbs_r;
    const dual vgs = {vgs_v, 1.0, 0.0, 0.0};
    const dual vds = {vds_v, 0.0, 1.0, 0.0};
    const dual vbs = {vbs_v, 0.0, 0.0, 1.0};
    const dual vgd = dsub(vgs, vds), vbd = dsub(vbs, vds);

    /* gminx = $simparam("gmin", 1e-12) (bsim3.va:353): the stepping rung's
     * gmin while it runs, else the card's */
    if (!(gmin >= 0.0)) gmin = q[BD_GMIN];
    double ibs, gbs, ibd, gbd;
    b3_jcur(vbs.v, q[BD_ISATS], q[BD_NVTMJ], q[BD_VJSM], q[BD_ISEVJSM], q[BD_IJTH], gmin, &ibs, &gbs);
    b3_jcur(vbd.v, q[BD_ISATD], q[BD_NVTMJ], q[BD_VJDM], q[BD_ISEVJDM], q[BD_IJTH], gmin, &ibd, &gbd);

    const int fwd = vds.v >= 0.0;
    const dual vdsx = fwd ? vds : dneg(vds);
    const dual vgsx = fwd ? vgs : vgd;
    const dual vbsx = fwd ? vbs : vbd;
    dual id, isub;
    b3_channel(q, vgsx, vdsx, vbsx, &id, &isub);
    /* channel current di -> si and substrate current, times m */
    const dual ich = dscl(fwd ? id : dneg(id), m);
    const dual isb = dscl(isub, m);
    ibs = m * ibs;
    gbs = m * gbs;
    ibd = m * ibd;
    gbd = m * gbd;

    double ichv = ich.v, isbv = isb.v;
    if (lim) {
        const double cgs = vgs_r - vgs.v, cds = vds_r - vds.v, cbs = vbs_r - vbs.v;
        const double cbd = (vbs_r - vds_r) - vbd.v;
        if (cgs != 0.0 || cds != 0.0 || cbs != 0.0) {
            ichv = ichv + (ich.g * cgs + ich.d * cds + ich.b * cbs);
            isbv = isbv + (isb.g * cgs + isb.d * cds + isb.b * cbs);
        }
        if (cbs != 0.0) ibs = ibs + gbs * cbs;
        if (cbd != 0.0) ibd = ibd + gbd * cbd;
    }
    const double ids = type * ichv, tsub = type * isbv, tbs = type * ibs, tbd = type * ibd;
    const double gdr = q[BD_GDRAIN], gsr = q[BD_GSOURCE];
    const double idr = gdr * (xd - xdi), isr = gsr * (xs - xsi);
    const double csum = (ich.g + ich.d) + ich.b, ssum = (isb.g + isb.d) + isb.b;
    /* residuals: 0 d, 1 g, 2 s, 3 b, 4 di, 5 si; the substrate current
     * leaves the channel end that is the drain in the swapped frame */
    o->f[0] = idr;
    o->f[2] = isr;
    o->f[3] = (tbd + tbs) - tsub;
    o->f[4] = (ids - tbd) - idr;
    o->f[5] = ((-ids) - tbs) - isr;
    if (fwd) o->f[4] = o->f[4] + tsub;
    else o->f[5] = o->f[5] + tsub;
    o->J[0][0] = gdr; o->J[0][4] = -gdr;
    o->J[2][2] = gsr; o->J[2][5] = -gsr;
    o->J[3][1] = -isb.g;
    o->J[3][3] = (gbd + gbs) - isb.b;
    o->J[3][4] = (-gbd) - isb.d;
    o->J[3][5] = ssum - gbs;
    o->J[4][0] = -gdr;
    o->J[4][1] = ich.g;
    o->J[4][3] = ich.b - gbd;
    o->J[4][4] = (ich.d + gbd) + gdr;
    o->J[4][5] = -csum;
    o->J[5][1] = -ich.g;
    o->J[5][2] = -gsr;
    o->J[5][3] = (-ich.b) - gbs;
    o->J[5][4] = -ich.d;
    o->J[5][5] = (csum + gbs) + gsr;
    const int r = fwd ? 4 : 5;
    o->J[r][1] = o->J[r][1] + isb.g;
    o->J[r][3] = o->J[r][3] + isb.b;
    o->J[r][4] = o->J[r][4] + isb.d;
    o->J[r][5] = o->J[r][5] - ssum;
}

/* The limiting ladder (bsim3.va:378-397): mos1's, with fetlim's threshold
 * the zero-bias type*vth0i and pnjlim at the 300.15 K vt0 and its vcrit.
 * Images within 16 ulps of the raw value snap to it. */
int bsim3_limit(const uint32_t *nd, const double *der, const double *x, const double *x_old,
                const double *lim_old, double *lim_new) {
    const double type = der[BD_TYPE];
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
    const double von = type * der[BD_VTH0I];
    double vgs, vds, vbs;
    if (vds_o >= 0.0) {
        vgs = fetlim(vgs_n, vgs_o, von);
        vds = vgs - vgd_n;
        vds = limvds(vds, vds_o);
    } else {
        const double vgd = fetlim(vgd_n, vgd_o, von);
        vds = vgs_n - vgd;
        vds = -limvds(-vds, -vds_o);
        vgs = vgd + vds;
    }
    int l = 0;
    if (vds >= 0.0) {
        vbs = pnjlim(vbs_n, vbs_o, der[BD_VT0], der[BD_VCRIT], &l);
    } else {
        const double vbd = pnjlim(vbd_n, vbd_o, der[BD_VT0], der[BD_VCRIT], &l);
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

/* MODEINITJCT (bsim3.va:378-397, b3ld.c:202-214). */
int bsim3_seed(const double *der, double *lim) {
    lim[0] = der[BD_TYPE] * der[BD_VTH0I] + 0.1;
    lim[1] = 0.1;
    lim[2] = 0.0;
    return 1;
}
