/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * Device models restated from the reference's Verilog-A sources with
 * hand-written derivatives (the reference differentiates by VerA's forward
 * AD, which is not vendored):
 *   models/resistor.va:42-54, capacitor.va:64, vsource.va:131-333,
 *   isource.va (vsource with I() contributions), diode.va:115-371
 * Limiters: ngspice DEVpnjlim / DEVfetlim / DEVlimvds as the reference
 * documents them (dev/solvers/newton-raphson-convergence.md:42-75).
 * The limiting correction follows src/device/eval.zig:820-877: a limited
 * device is evaluated at its limited junction voltage and its residual is
 * linearised back to x, f += g * (v - v_lim).
 *
 * Stamp order (shared with the CUDA library, which writes the same cells
 * in the same order): per instance, rows in local-unknown order, the
 * residual first, then the Jacobian entries of that row by local column.
 */
#include "orc_internal.h"

#include <math.h>
#include <string.h>

#define KB 1.38064852e-23
#define QE 1.6021766208e-19

int orc_nodes_per(uint32_t type) {
    static const int t[ORC_NTYPES] = {2, 2, 3, 2, 3, 6, 6};
    return type < ORC_NTYPES ? t[type] : 0;
}

int orc_params_per(uint32_t type) {
    static const int t[ORC_NTYPES] = {1, 1, ORC_SRC_NP, ORC_SRC_NP, ORC_D_NP, ORC_M_NP, ORC_B3_NP};
    return type < ORC_NTYPES ? t[type] : 0;
}

int dev_nstate(uint32_t type) { (void)type; return 0; }

static void add_ent(layout_t *l, int ru, int cu) {
    l->jac[l->nj].ru = (uint8_t)ru;
    l->jac[l->nj].cu = (uint8_t)cu;
    l->nj++;
}

static void add_qent(layout_t *l, int ru, int cu) {
    l->qjac[l->nq].ru = (uint8_t)ru;
    l->qjac[l->nq].cu = (uint8_t)cu;
    l->nq++;
}

/* Entries must be listed row-major with columns ascending. */
void dev_layout(uint32_t type, const double *prm, layout_t *l) {
    memset(l, 0, sizeof(*l));
    l->nu = orc_nodes_per(type);
    switch (type) {
    case ORC_R:
        l->res_row[0] = l->res_row[1] = 1;
        add_ent(l, 0, 0); add_ent(l, 0, 1); add_ent(l, 1, 0); add_ent(l, 1, 1);
        break;
    case ORC_C:
        l->q_row[0] = l->q_row[1] = 1;
        add_qent(l, 0, 0); add_qent(l, 0, 1); add_qent(l, 1, 0); add_qent(l, 1, 1);
        break;
    case ORC_V: /* p n br */
        l->res_row[0] = l->res_row[1] = l->res_row[2] = 1;
        add_ent(l, 0, 2); add_ent(l, 1, 2); add_ent(l, 2, 0); add_ent(l, 2, 1);
        break;
    case ORC_I:
        l->res_row[0] = l->res_row[1] = 1;
        break;
    case ORC_D: { /* a c ai */
        int rs = prm[ORC_D_RS] > 0;
        l->nlim = 1;
        if (rs) {
            l->res_row[0] = 1;
            add_ent(l, 0, 0); add_ent(l, 0, 2);
        }
        l->res_row[1] = l->res_row[2] = 1;
        add_ent(l, 1, 1); add_ent(l, 1, 2);
        if (rs) add_ent(l, 2, 0);
        add_ent(l, 2, 1); add_ent(l, 2, 2);
        if (prm[ORC_D_CJO] > 0 || prm[ORC_D_TT] > 0) {
            l->q_row[1] = l->q_row[2] = 1;
            add_qent(l, 1, 1); add_qent(l, 1, 2); add_qent(l, 2, 1); add_qent(l, 2, 2);
        }
        break;
    }
    case ORC_M: { /* d g s b di si */
        double der[ORC_NDER];
        mos1_derive(prm, der);
        int rd = prm[ORC_M_RD] > 0, rs = prm[ORC_M_RS] > 0;
        l->nlim = 3;
        if (rd) {
            l->res_row[0] = 1;
            add_ent(l, 0, 0); add_ent(l, 0, 4);
        }
        if (rs) {
            l->res_row[2] = 1;
            add_ent(l, 2, 2); add_ent(l, 2, 5);
        }
        l->res_row[3] = l->res_row[4] = l->res_row[5] = 1;
        add_ent(l, 3, 3); add_ent(l, 3, 4); add_ent(l, 3, 5);
        if (rd) add_ent(l, 4, 0);
        add_ent(l, 4, 1); add_ent(l, 4, 3); add_ent(l, 4, 4); add_ent(l, 4, 5);
        add_ent(l, 5, 1);
        if (rs) add_ent(l, 5, 2);
        add_ent(l, 5, 3); add_ent(l, 5, 4); add_ent(l, 5, 5);
        if (mos1_has_charge(der)) {
            l->q_row[1] = l->q_row[3] = l->q_row[4] = l->q_row[5] = 1;
            add_qent(l, 1, 1); add_qent(l, 1, 3); add_qent(l, 1, 4); add_qent(l, 1, 5);
            add_qent(l, 3, 1); add_qent(l, 3, 3); add_qent(l, 3, 4); add_qent(l, 3, 5);
            add_qent(l, 4, 1); add_qent(l, 4, 3); add_qent(l, 4, 4);
            add_qent(l, 5, 1); add_qent(l, 5, 3); add_qent(l, 5, 5);
        }
        break;
    }
    case ORC_B3: { /* d g s b di si (models/bsim3.va:613-624); no charges */
        const double rsh = prm[ORC_B3_RSH];
        int rd = rsh > 0 && prm[ORC_B3_NRD] > 0, rs = rsh > 0 && prm[ORC_B3_NRS] > 0;
        l->nlim = 3;
        if (rd) {
            l->res_row[0] = 1;
            add_ent(l, 0, 0); add_ent(l, 0, 4);
        }
        if (rs) {
            l->res_row[2] = 1;
            add_ent(l, 2, 2); add_ent(l, 2, 5);
        }
        l->res_row[3] = l->res_row[4] = l->res_row[5] = 1;
        add_ent(l, 3, 1); add_ent(l, 3, 3); add_ent(l, 3, 4); add_ent(l, 3, 5);
        if (rd) add_ent(l, 4, 0);
        add_ent(l, 4, 1); add_ent(l, 4, 3); add_ent(l, 4, 4); add_ent(l, 4, 5);
        add_ent(l, 5, 1);
        if (rs) add_ent(l, 5, 2);
        add_ent(l, 5, 3); add_ent(l, 5, 4); add_ent(l, 5, 5);
        break;
    }
    default:
        break;
    }
}

int dev_pattern(uint32_t type, const uint32_t *nd, const double *prm, uint32_t *rows, uint32_t *cols) {
    layout_t l;
    dev_layout(type, prm, &l);
    int ne = 0;
    for (int e = 0; e < l.nj; e++) {
        rows[ne] = nd[l.jac[e].ru];
        cols[ne] = nd[l.jac[e].cu];
        ne++;
    }
    for (int e = 0; e < l.nq; e++) {
        rows[ne] = nd[l.qjac[e].ru];
        cols[ne] = nd[l.qjac[e].cu];
        ne++;
    }
    return ne;
}

/* ------------------------------------------------------------------ */
/* limiters (ngspice devsup.c as documented by the reference)         */

double pnjlim(double vnew, double vold, double vt, double vcrit, int *lim) {
    if (vnew > vcrit && fabs(vnew - vold) > vt + vt) {
        if (vold > 0) {
            double arg = (vnew - vold) / vt;
            if (arg > 0) vnew = vold + vt * (2 + esl_log(arg - 2));
            else vnew = vold - vt * (2 + esl_log(2 - arg));
        } else {
            vnew = vt * esl_log(vnew / vt);
        }
        *lim = 1;
    } else if (vnew < 0) {
        double arg = vold > 0 ? -1 * vold - 1 : 2 * vold - 1;
        if (vnew < arg) {
            vnew = arg;
            *lim = 1;
        } else {
            *lim = 0;
        }
    } else {
        *lim = 0;
    }
    return vnew;
}

double fetlim(double vnew, double vold, double vto) {
    double vtsthi = fabs(2 * (vold - vto)) + 2;
    double vtstlo = fabs(vold - vto) + 1;
    double vtox = vto + 3.5;
    double delv = vnew - vold;
    if (vold >= vto) {
        if (vold >= vtox) {
            if (delv <= 0) {
                if (vnew >= vtox) {
                    if (-delv > vtstlo) vnew = vold - vtstlo;
                } else {
                    vnew = fmax(vnew, vto + 2);
                }
            } else if (delv >= vtsthi) {
                vnew = vold + vtsthi;
            }
        } else if (delv <= 0) {
            vnew = fmax(vnew, vto - 0.5);
        } else {
            vnew = fmin(vnew, vto + 4);
        }
    } else if (delv <= 0) {
        if (-delv > vtsthi) vnew = vold - vtsthi;
    } else {
        double vtemp = vto + 0.5;
        if (vnew <= vtemp) {
            if (delv > vtstlo) vnew = vold + vtstlo;
        } else {
            vnew = vtemp;
        }
    }
    return vnew;
}

double limvds(double vnew, double vold) {
    if (vold >= 3.5) {
        if (vnew > vold) vnew = fmin(vnew, 3 * vold + 2);
        else if (vnew < 3.5) vnew = fmax(vnew, 2);
    } else if (vnew > vold) {
        vnew = fmin(vnew, 4);
    } else {
        vnew = fmax(vnew, -0.5);
    }
    return vnew;
}

/* ------------------------------------------------------------------ */
/* diode.va: bias-independent temperature map (TLEV 0, TLEVC 0)        */

enum {
    DD_VTE, DD_IS, DD_VCRIT, DD_RS, DD_GMIN, DD_BV, DD_XBV, DD_VTEBRK, DD_CJO,
    DD_VJ, DD_MT, DD_FC, DD_TT, DD_NDER
};

static void diode_derive(const double *p, double *d) {
    double tk = p[ORC_D_TEMP];
    double tnomk = p[ORC_D_TNOM] + 273.15;
    double ratio = tk / tnomk;
    double vt = KB / QE * tk;
    double vtnom = KB / QE * tnomk;
    double n = p[ORC_D_N];
    double vte = n * vt;
    double ae = p[ORC_D_AREA];
    double egp = p[ORC_D_EG];
    double vtebrk = n * vt;
    double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    double mt = p[ORC_D_M];
    double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
    double arg1 = -egfet1 / (2.0 * KB * tnomk) + 1.1150877 / (2.0 * KB * 300.15);
    double argt = -egfet / (2.0 * KB * tk) + 1.1150877 / (2.0 * KB * 300.15);
    double pbfact1 = -2.0 * vtnom * (1.5 * esl_log(fact1) + QE * arg1);
    double pbfact = -2.0 * vt * (1.5 * esl_log(fact2) + QE * argt);
    double vj = p[ORC_D_VJ];
    double pbo = (vj - pbfact1) / fact1;
    double gmaold = (vj - pbo) / pbo;
    double vj_t = pbfact + fact2 * pbo;
    double gmanew = (vj_t - pbo) / pbo;
    double cjo_t = p[ORC_D_CJO] * (1.0 + mt * (400e-6 * (tk - 300.15) - gmanew)) /
                   (1.0 + mt * (400e-6 * (tnomk - 300.15) - gmaold));
    cjo_t = cjo_t * ae;
    double is_t = p[ORC_D_IS] * ae * esl_exp((ratio - 1.0) * egp / vte + (p[ORC_D_XTI] / n) * esl_log(ratio));
    double bv_t = p[ORC_D_BV];
    double ibvx = p[ORC_D_IBV];
    double xbv = bv_t;
    if (p[ORC_D_BV] > 0.0 && ibvx >= is_t * bv_t / vt) {
        xbv = bv_t - vtebrk * esl_log(1.0 + ibvx / is_t);
        xbv = bv_t - vtebrk * esl_log(ibvx / is_t + 1.0 - xbv / vt);
    }
    double rs_t = p[ORC_D_RS] / ae;
    if (rs_t < 1.0e-9) rs_t = 1.0e-9;
    d[DD_VTE] = vte;
    d[DD_IS] = is_t;
    d[DD_VCRIT] = vte * esl_log(vte / (1.4142135623730951 * is_t));
    d[DD_RS] = rs_t;
    d[DD_GMIN] = p[ORC_D_GMIN];
    d[DD_BV] = p[ORC_D_BV];
    d[DD_XBV] = xbv;
    d[DD_VTEBRK] = vtebrk;
    d[DD_CJO] = cjo_t;
    d[DD_VJ] = vj_t;
    d[DD_MT] = mt;
    d[DD_FC] = p[ORC_D_FC];
    d[DD_TT] = p[ORC_D_TT];
}

/* Junction current and conductance at vd (diode.va:261-318, no ISR/IKF). */
static void diode_iv(const double *d, double vd, double *i, double *g) {
    double vte = d[DD_VTE], is = d[DD_IS];
    double id, gd;
    if (vd >= -3.0 * vte) {
        double u = vd / vte;
        double ulim = u < 80.0 ? u : 80.0;
        double e = esl_exp(ulim);
        id = is * ((e * (1.0 + (u - ulim))) - 1.0);
        gd = is * e / vte;
    } else {
        double a = 3.0 * vte / (vd * 2.718281828459045);
        double a3 = esl_pow(a, 3.0);
        id = -is * (1.0 + a3);
        gd = 3.0 * is * a3 / vd;
    }
    if (d[DD_BV] > 0.0 && vd < -3.0 * vte && vd < -d[DD_XBV]) {
        double wb = -(d[DD_XBV] + vd) / d[DD_VTEBRK];
        double wlim = wb < 80.0 ? wb : 80.0;
        double e = esl_exp(wlim);
        id = -is * e * (1.0 + (wb - wlim));
        gd = is * e / d[DD_VTEBRK];
    }
    *i = id + d[DD_GMIN] * vd;
    *g = gd + d[DD_GMIN];
}

/* Junction charge and capacitance at vd (diode.va:338-363, no sidewall). */
static void diode_qc(const double *d, double vd, double itot, double gtot, double *q, double *c) {
    double qj = 0.0, cj = 0.0;
    if (d[DD_CJO] > 0.0) {
        double vj = d[DD_VJ], mt = d[DD_MT], fc = d[DD_FC], cjo = d[DD_CJO];
        double vfc = fc * vj;
        if (vd < vfc) {
            double b = 1.0 - vd / vj;
            qj = cjo * vj * (1.0 - esl_pow(b, 1.0 - mt)) / (1.0 - mt);
            cj = cjo * esl_pow(b, -mt);
        } else {
            double f1 = vj * (1.0 - esl_pow(1.0 - fc, 1.0 - mt)) / (1.0 - mt);
            double f2 = esl_pow(1.0 - fc, 1.0 + mt);
            double f3 = 1.0 - fc * (1.0 + mt);
            qj = cjo * (f1 + (1.0 / f2) * (f3 * (vd - vfc) + (mt / (2.0 * vj)) * (vd * vd - vfc * vfc)));
            cj = cjo * ((1.0 / f2) * (f3 + (mt / vj) * vd));
        }
    }
    if (d[DD_TT] > 0.0) {
        qj = qj + d[DD_TT] * itot;
        cj = cj + d[DD_TT] * gtot;
    }
    *q = qj;
    *c = cj;
}

void dev_derive(uint32_t type, const double *prm, double *der) {
    memset(der, 0, sizeof(double) * ORC_NDER);
    if (type == ORC_D) diode_derive(prm, der);
    if (type == ORC_M) mos1_derive(prm, der);
    if (type == ORC_B3) bsim3_derive(prm, der);
}

/* PULSE waveform (vsource.va:211-222). */
static double pulse(const double *p, double t) {
    double v1 = p[2], v2 = p[3], td = p[4];
    double tr = p[5] > 1.0e-12 ? p[5] : 1.0e-12;
    double tf = p[6] > 1.0e-12 ? p[6] : 1.0e-12;
    double pw = (p[7] > 0.0 ? p[7] : 0.0) + (-p[7] > 0.0 ? -p[7] : 0.0) * 1.0e30;
    double per = p[8];
    double per_min = tr + pw + tf + 1.0e-12;
    if (per < per_min) per = per_min;
    double t_rel = t - td;
    double t_mod = t_rel + (p[9] / 360.0) * per;
    t_mod = t_mod - floor(t_mod / per) * per;
    if (t_mod < 0.0) t_mod = 0.0;
    if (t_rel < 0.0) return v1;
    if (t_mod < tr) return v1 + (v2 - v1) * (t_mod / tr);
    if (t_mod < tr + pw) return v2;
    if (t_mod < tr + pw + tf) return v2 - (v2 - v1) * ((t_mod - (tr + pw)) / tf);
    return v1;
}

#define ORC_PI 3.141592653589793
#define ORC_TWO_PI 6.283185307179586

/* SIN (vsource.va:224-236): before TD the wave's own t = 0 value; the
 * damping applies after TD, its exponent clamped at 80. */
static double sine(const double *p, double t) {
    double vo = p[2], va = p[3], freq = p[4], td = p[5], theta = p[6], phase = p[7];
    double t_sin = t - td;
    if (t_sin < 0.0) return vo + va * esl_sin(phase * ORC_PI / 180.0);
    return vo + va * esl_sin(ORC_TWO_PI * freq * t_sin + phase * ORC_PI / 180.0) * esl_exp(fmin(-theta * t_sin, 80.0));
}

/* EXP (vsource.va:238-246): two one-sided exponentials on V1. */
static double expo(const double *p, double t) {
    double v1 = p[2], v2 = p[3], td1 = p[4], tau1 = p[5], td2 = p[6], tau2 = p[7];
    double t_e1 = t - td1, t_e2 = t - td2;
    double out = v1;
    if (t_e1 > 0.0) out = out + (v2 - v1) * (1.0 - esl_exp(fmin(-t_e1 / fmax(tau1, 1.0e-15), 80.0)));
    if (t_e2 > 0.0) out = out + (v1 - v2) * (1.0 - esl_exp(fmin(-t_e2 / fmax(tau2, 1.0e-15), 80.0)));
    return out;
}

/* PWL (vsource.va:248-290): the repeat wraps [r, t_last]; bisection for the
 * segment holding t. */
static double pwl(const double *p, double t) {
    const int len = (int)p[2];
    if (len <= 0) return p[0];
    const double repeat = p[3], td = p[4];
    const double *tt = p + ORC_SRC_PWL_T, *vv = p + ORC_SRC_PWL_V;
    double t_e = t - td;
    const double t_first = tt[0], v_first = vv[0], t_last = tt[len - 1], v_last = vv[len - 1];
    if (repeat >= 0.0 && len > 1 && t_e > t_last && t_last > repeat) {
        double span = t_last - repeat;
        if (span > 0.0) {
            double excess = t_e - repeat;
            t_e = repeat + (excess - floor(excess / span) * span);
        }
    }
    if (t_e < 0.0 || t_e <= t_first) return v_first;
    if (t_e >= t_last) return v_last;
    int klo = 0, khi = len - 1;
    while (khi - klo > 1) {
        int k = (klo + khi) / 2;
        if (tt[k] > t_e) khi = k;
        else klo = k;
    }
    const double tp = tt[klo], vp = vv[klo], tk = tt[khi], vk = vv[khi];
    return vp + (vk - vp) * (t_e - tp) / fmax(tk - tp, 1.0e-15);
}

/* The source's value (vsource.va:198-290): static analyses at `dc`, the
 * transient and its own operating point at the wave; times the source-
 * stepping factor. */
double source_value(const double *p, const sim_t *sim) {
    double out = p[0];
    if (sim->kind != 0) {
        if (p[1] == 1.0) out = pulse(p, sim->t);
        else if (p[1] == 2.0) out = sine(p, sim->t);
        else if (p[1] == 3.0) out = expo(p, sim->t);
        else if (p[1] == 4.0) out = pwl(p, sim->t);
    }
    return out * sim->src_scale;
}

void dev_eval(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, const double *lim, const double *st, const sim_t *sim,
              devout_t *o) {
    memset(o, 0, sizeof(*o));
    switch (type) {
    case ORC_R: {
        double g = 1.0 / prm[0];
        double i = (x[nd[0]] - x[nd[1]]) / prm[0];
        o->f[0] = i;
        o->f[1] = -i;
        o->J[0][0] = g; o->J[0][1] = -g; o->J[1][0] = -g; o->J[1][1] = g;
        break;
    }
    case ORC_C: {
        double c = prm[0];
        double qv = c * (x[nd[0]] - x[nd[1]]);
        o->q[0] = qv;
        o->q[1] = -qv;
        o->C[0][0] = c; o->C[0][1] = -c; o->C[1][0] = -c; o->C[1][1] = c;
        break;
    }
    case ORC_V: {
        double v = source_value(prm, sim);
        o->f[0] = x[nd[2]];
        o->f[1] = -x[nd[2]];
        o->f[2] = x[nd[0]] - x[nd[1]] - v;
        o->J[0][2] = 1.0; o->J[1][2] = -1.0; o->J[2][0] = 1.0; o->J[2][1] = -1.0;
        break;
    }
    case ORC_I: {
        double v = source_value(prm, sim);
        o->f[0] = v;
        o->f[1] = -v;
        break;
    }
    case ORC_D: {
        double vraw = x[nd[2]] - x[nd[1]];
        double ve = lim ? lim[0] : vraw;
        double i, g, qj, cj;
        diode_iv(der, ve, &i, &g);
        double ires = i;
        if (lim) {
            double corr = vraw - ve;
            if (corr != 0.0) ires = ires + g * corr;
        }
        double grs = 1.0 / der[DD_RS];
        double irs = (x[nd[0]] - x[nd[2]]) / der[DD_RS];
        int rs = prm[ORC_D_RS] > 0;
        if (rs) {
            o->f[0] = irs;
            o->J[0][0] = grs;
            o->J[0][2] = -grs;
        }
        o->f[1] = -ires;
        o->J[1][1] = g;
        o->J[1][2] = -g;
        o->f[2] = rs ? ires - irs : ires;
        if (rs) o->J[2][0] = -grs;
        o->J[2][1] = -g;
        o->J[2][2] = rs ? g + grs : g;
        if (prm[ORC_D_CJO] > 0 || prm[ORC_D_TT] > 0) {
            diode_qc(der, ve, i, g, &qj, &cj);
            if (lim) {
                double corr = vraw - ve;
                if (corr != 0.0) qj = qj + cj * corr;
            }
            o->q[1] = -qj;
            o->q[2] = qj;
            o->C[1][1] = cj; o->C[1][2] = -cj; o->C[2][1] = -cj; o->C[2][2] = cj;
        }
        break;
    }
    case ORC_M:
        mos1_eval(nd, prm, der, x, lim, st, sim, o);
        break;
    case ORC_B3:
        bsim3_eval(nd, der, x, lim, sim->gmin, o);
        break;
    default:
        break;
    }
}

int dev_qtape(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, double *out) {
    if (type == ORC_C) {
        out[0] = prm[0] * (x[nd[0]] - x[nd[1]]);
        return 1;
    }
    if (type == ORC_D && (prm[ORC_D_CJO] > 0 || prm[ORC_D_TT] > 0)) {
        double i, g, qj, cj;
        double vd = x[nd[2]] - x[nd[1]];
        diode_iv(der, vd, &i, &g);
        diode_qc(der, vd, i, g, &qj, &cj);
        out[0] = qj;
        return 1;
    }
    if (type == ORC_M) return mos1_qtape(nd, der, x, out);
    return 0;
}

int dev_limit(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, const double *x_old, const double *lim_old, double *lim_new) {
    if (type == ORC_D) {
        double vnew = x[nd[2]] - x[nd[1]];
        double vold = lim_old ? lim_old[0] : x_old[nd[2]] - x_old[nd[1]];
        int l = 0;
        lim_new[0] = pnjlim(vnew, vold, der[DD_VTE], der[DD_VCRIT], &l);
        return l;
    }
    if (type == ORC_M) return mos1_limit(nd, prm, der, x, x_old, lim_old, lim_new);
    if (type == ORC_B3) return bsim3_limit(nd, der, x, x_old, lim_old, lim_new);
    return 0;
}

int dev_seed(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
             const double *x, double *lim) {
    (void)nd;
    (void)prm;
    (void)x;
    if (type == ORC_D) {
        /* ngspice MODEINITJCT: vd = tVcrit (dioload.c), the reference's
         * `D.seed` image. */
        lim[0] = der[DD_VCRIT];
        return 1;
    }
    if (type == ORC_M) return mos1_seed(nd, prm, der, x, lim);
    if (type == ORC_B3) return bsim3_seed(der, lim);
    return 0;
}

int orc_dev_stamp(uint32_t type, const double *prm, const double *xloc, double *f, double *J) {
    if (type >= ORC_NTYPES) return 1;
    uint32_t nd[ORC_MAX_U];
    for (uint32_t k = 0; k < ORC_MAX_U; k++) nd[k] = k;
    double der[ORC_NDER];
    dev_derive(type, prm, der);
    sim_t sim;
    memset(&sim, 0, sizeof(sim));
    sim.src_scale = 1.0;
    sim.gmin = -1.0;
    sim.iteration = 1;
    devout_t o;
    dev_eval(type, nd, prm, der, xloc, NULL, NULL, &sim, &o);
    for (int r = 0; r < ORC_MAX_U; r++) {
        f[r] = o.f[r];
        for (int c = 0; c < ORC_MAX_U; c++) J[r * ORC_MAX_U + c] = o.J[r][c];
    }
    return 0;
}

/* The model code's exp, log and pow (esl_math.h's, or the C library's in
 * the libm build) for the accuracy tests: which 0 exp(x), 1 log(x),
 * 2 pow(x, y); n values from x (and y) into out. */
void orc_math(int which, uint32_t n, const double *x, const double *y, double *out) {
    for (uint32_t i = 0; i < n; i++)
        out[i] = which == 0 ? esl_exp(x[i]) : which == 1 ? esl_log(x[i]) : esl_pow(x[i], y[i]);
}
