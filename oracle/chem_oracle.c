/* CPU oracle: constant-pressure chemistry RHS and analytic Jacobian.
 * TEST INFRASTRUCTURE ONLY -- see chem_oracle.h.
 *
 * Restates the pyJac C kernels of the reference, table-driven:
 *   eval_conc          src/Mechanism/CPU/chem_utils.c:4-97
 *   eval_rxn_rates     src/Mechanism/CPU/rxn_rates.c:2-3862
 *   get_rxn_pres_mod   src/Mechanism/CPU/rxn_rates_pres_mod.c:5-366
 *   eval_spec_rates    src/Mechanism/CPU/spec_rates.c:4-2830
 *   eval_cp / eval_h   src/Mechanism/CPU/chem_utils.c:194,1160
 *   dydt               src/Mechanism/CPU/dydt.c:7-133
 *   eval_jacob         src/Mechanism/CPU/jacob.c:3-372 (exact derivative of dydt)
 * and, for mechanisms the reference integrates only through Cantera
 * (src/Integrators/CanteraIntegrator.cpp), the rate forms pyJac's tables do
 * not cover: pressure-dependent Arrhenius (PLOG) reactions and fractional
 * product coefficients of irreversible reactions, with Cantera's published
 * PLOG definition (ln k linear in ln P between the bracketing levels, clamped
 * to the end levels; a level's k is the sum of its Arrhenius terms).
 * The Jacobian is derived here from the RHS (chain rule through the
 * concentrations and the closure species), not from pyJac's expression
 * layout; it agrees with pyJac's to round-off.
 */
#include "chem_oracle.h"
#include "bdf_oracle.h"

#include <math.h>
#include <string.h>
#include <stdlib.h>

#include "../hpc_ode_b200/csrc/mech/gri30_mech.h"
#include "../hpc_ode_b200/csrc/mech/h2o2_mech.h"
#include "../hpc_ode_b200/csrc/mech/nDodecane_Reitz_mech.h"
#include "../hpc_ode_b200/csrc/mech/h2_li_2004_mech.h"
#include "../hpc_ode_b200/csrc/mech/ESTiMatE-Mech_04042022_mech.h"

#define RU 8314.4621
#define PATM 101325.0
#define MAXNSP 256
#define MAXP_ORACLE 8   /* participants per side (the generated MAXP is at most this) */

typedef struct {
    int nsp, nrxn, maxp;
    const double *mw, *tmid, *lo, *hi;
    const int *type, *rev;
    const double *A, *logA, *b, *EaR, *A0, *logA0, *b0, *EaR0, *troe;
    const int *troeT2, *reac_sp, *reac_nu, *prod_sp;
    const double *prod_nu;   /* fractional only in irreversible reactions */
    const int *tb_off, *tb_sp;
    const double *tb_alpha;
    const int *plog_off, *plog_term_off;
    const double *plog_lnP, *plog_A, *plog_logA, *plog_b, *plog_EaR;
} mech_t;

#define MECH_INIT(tag, PFX) { PFX##_NSP, PFX##_NRXN, PFX##_MAXP, \
    tag##_mw, tag##_tmid, tag##_nasa_lo, tag##_nasa_hi, tag##_rxn_type, tag##_rxn_rev, \
    tag##_rxn_A, tag##_rxn_logA, tag##_rxn_b, tag##_rxn_EaR, tag##_rxn_A0, tag##_rxn_logA0, \
    tag##_rxn_b0, tag##_rxn_EaR0, tag##_rxn_troe, tag##_rxn_troe_T2, tag##_rxn_reac_sp, \
    tag##_rxn_reac_nu, tag##_rxn_prod_sp, tag##_rxn_prod_nu, tag##_rxn_tb_off, tag##_tb_sp, \
    tag##_tb_alpha, tag##_plog_off, tag##_plog_term_off, tag##_plog_lnP, tag##_plog_A, \
    tag##_plog_logA, tag##_plog_b, tag##_plog_EaR }

#define NMECH 5
#if MECH_GRI30_MAXP > MAXP_ORACLE || MECH_ESTIMATE_MECH_04042022_MAXP > MAXP_ORACLE || \
    MECH_NDODECANE_REITZ_MAXP > MAXP_ORACLE
#error "participant lists longer than the oracle's scratch"
#endif
static const mech_t MECHS[NMECH] = { MECH_INIT(gri30, MECH_GRI30), MECH_INIT(h2o2, MECH_H2O2),
                                     MECH_INIT(ndodecane_reitz, MECH_NDODECANE_REITZ),
                                     MECH_INIT(h2_li_2004, MECH_H2_LI_2004),
                                     MECH_INIT(estimate_mech_04042022, MECH_ESTIMATE_MECH_04042022) };

int oracle_mech_id(const char* name) {
    if (!name) return -1;
    if (!strncmp(name, "gri30", 5)) return ORACLE_MECH_GRI30;
    if (!strncmp(name, "h2o2", 4)) return ORACLE_MECH_H2O2;
    if (!strncmp(name, "nDodecane_Reitz", 15)) return ORACLE_MECH_NDODECANE;
    if (!strncmp(name, "h2_li_2004", 10)) return ORACLE_MECH_H2LI;
    if (!strncmp(name, "ESTiMatE-Mech_04042022", 22)) return ORACLE_MECH_ESTIMATE;
    return -1;
}

int oracle_mech_nsp(int mech) {
    if (mech < 0 || mech >= NMECH) return -1;
    return MECHS[mech].nsp;
}

/* ---------------------------------------------------------------- thermo */
static const double* nasa(const mech_t* M, int k, double T) {
    return (T <= M->tmid[k]) ? &M->lo[7 * k] : &M->hi[7 * k];
}
/* cp/R, h/RT, s/R - h/RT (= -g/RT), d(cp/R)/dT */
static double cp_R(const double* a, double T) {
    return a[0] + T * (a[1] + T * (a[2] + T * (a[3] + a[4] * T)));
}
static double h_RT(const double* a, double T) {
    return a[0] + T * (a[1] / 2.0 + T * (a[2] / 3.0 + T * (a[3] / 4.0 + a[4] / 5.0 * T))) + a[5] / T;
}
static double mg_RT(const double* a, double T, double logT) {
    return a[0] * (logT - 1.0) + T * (a[1] / 2.0 + T * (a[2] / 6.0 + T * (a[3] / 12.0 + a[4] / 20.0 * T)))
           - a[5] / T + a[6];
}
static double dcp_R(const double* a, double T) {
    return a[1] + T * (2.0 * a[2] + T * (3.0 * a[3] + 4.0 * a[4] * T));
}

/* ------------------------------------------------------- per-reaction core */
typedef struct {
    double kf, kr;        /* rate coefficients (kr = 0 if irreversible) */
    double Rf, Rr;        /* kf * prod C^nu', kr * prod C^nu'' */
    double phi;           /* pressure modification (1 for elementary) */
    double thd;           /* third-body concentration */
    double dphi_dthd;     /* d phi / d thd at fixed T */
    double dphi_dT;       /* d phi / d T at fixed thd */
    double dlnkf_dT, dlnkr_dT;
    double dlnk_dlnP;     /* PLOG: d ln k / d ln P at fixed T (0 otherwise) */
    int ordf, ordr;
} rxn_eval_t;

static double arrh(double A, double logA, double b, double EaR, double logT, double T) {
    if (b == 0.0 && EaR == 0.0) return A;
    return exp(logA + b * logT - EaR / T);
}

/* k of PLOG level l (sum of its Arrhenius terms) and d ln k / dT. */
static double plog_level(const mech_t* M, int l, double T, double logT, double* dlnk_dT) {
    double k = 0.0, dk = 0.0;
    for (int t = M->plog_term_off[l]; t < M->plog_term_off[l + 1]; ++t) {
        double kt = arrh(M->plog_A[t], M->plog_logA[t], M->plog_b[t], M->plog_EaR[t], logT, T);
        k += kt;
        dk += kt * (M->plog_b[t] + M->plog_EaR[t] / T) / T;
    }
    *dlnk_dT = dk / k;
    return k;
}

/* PLOG rate of reaction r at (T, P): ln k linear in ln P between the levels
 * that bracket P, the end level's k outside their range. */
static double plog_rate(const mech_t* M, int r, double T, double logT, double lnP, double* dlnk_dT,
                        double* dlnk_dlnP) {
    const int l0 = M->plog_off[r], l1 = M->plog_off[r + 1] - 1;
    int lo = l0, hi = l0;
    double w = 0.0;
    if (lnP >= M->plog_lnP[l1]) {
        lo = hi = l1;
    } else if (lnP > M->plog_lnP[l0]) {
        while (M->plog_lnP[lo + 1] < lnP) ++lo;
        hi = lo + 1;
        w = (lnP - M->plog_lnP[lo]) / (M->plog_lnP[hi] - M->plog_lnP[lo]);
    }
    double d0, d1;
    const double k0 = plog_level(M, lo, T, logT, &d0);
    const double k1 = plog_level(M, hi, T, logT, &d1);
    *dlnk_dT = (1.0 - w) * d0 + w * d1;
    *dlnk_dlnP = hi != lo ? (log(k1) - log(k0)) / (M->plog_lnP[hi] - M->plog_lnP[lo]) : 0.0;
    return exp((1.0 - w) * log(k0) + w * log(k1));
}

static void eval_reaction(const mech_t* M, int r, double T, double logT, double m,
                          const double* C, const double* mgRT, int want_deriv, rxn_eval_t* o) {
    const int P = M->maxp;
    double dlnkf_dT = (M->b[r] + M->EaR[r] / T) / T, dlnk_dlnP = 0.0;
    double kf = M->type[r] == 4 ? plog_rate(M, r, T, logT, log(m * RU * T), &dlnkf_dT, &dlnk_dlnP)
                                : arrh(M->A[r], M->logA[r], M->b[r], M->EaR[r], logT, T);
    o->dlnk_dlnP = dlnk_dlnP;
    double Rf = 1.0, Rr = 1.0;
    int ordf = 0, ordr = 0, dnu = 0;
    double sum_g = 0.0;
    for (int i = 0; i < P; ++i) {
        int s = M->reac_sp[r * P + i];
        if (s < 0) break;
        int nu = M->reac_nu[r * P + i];
        for (int q = 0; q < nu; ++q) Rf *= C[s];
        ordf += nu; dnu -= nu; sum_g -= nu * mgRT[s];
    }
    for (int i = 0; M->rev[r] && i < P; ++i) {   /* products enter the reverse rate only */
        int s = M->prod_sp[r * P + i];
        if (s < 0) break;
        int nu = (int)M->prod_nu[r * P + i];
        for (int q = 0; q < nu; ++q) Rr *= C[s];
        ordr += nu; dnu += nu; sum_g += nu * mgRT[s];
    }
    o->ordf = ordf; o->ordr = ordr;
    o->kf = kf;
    o->dlnkf_dT = dlnkf_dT;
    if (M->rev[r]) {
        /* Kc = exp(sum nu (s/R - h/RT)) * (Patm / (R T))^dnu */
        double Kc = exp(sum_g - dnu * logT) * pow(PATM / RU, (double)dnu);
        o->kr = kf / Kc;
        o->dlnkr_dT = o->dlnkf_dT;   /* corrected below once dH is known */
    } else {
        o->kr = 0.0;
        o->dlnkr_dT = 0.0;
    }
    o->Rf = kf * Rf;
    o->Rr = o->kr * Rr;
    o->phi = 1.0; o->thd = 0.0; o->dphi_dthd = 0.0; o->dphi_dT = 0.0;
    int type = M->type[r];
    if (type == 0 || type == 4) return;
    double thd = m;
    for (int t = M->tb_off[r]; t < M->tb_off[r + 1]; ++t) thd += M->tb_alpha[t] * C[M->tb_sp[t]];
    o->thd = thd;
    if (type == 1) { o->phi = thd; o->dphi_dthd = 1.0; return; }
    /* falloff: kf above is k_inf */
    double k0 = arrh(M->A0[r], M->logA0[r], M->b0[r], M->EaR0[r], logT, T);
    double Pr = k0 * thd / kf;
    double F = 1.0, dlog10F_dx = 0.0, dlog10F_dT = 0.0;
    if (type == 3) {
        const double* tr = &M->troe[4 * r];
        double a = tr[0], T3 = tr[1], T1 = tr[2], T2 = tr[3];
        double e3 = exp(-T / T3), e1 = exp(-T / T1);
        double Fcent = (1.0 - a) * e3 + a * e1;
        double dFcent = -(1.0 - a) / T3 * e3 - a / T1 * e1;
        if (M->troeT2[r]) { double e2 = exp(-T2 / T); Fcent += e2; dFcent += T2 / (T * T) * e2; }
        int fc_clamped = !(Fcent > 1.0e-300);
        double Fc = log10(fmax(Fcent, 1.0e-300));
        int pr_clamped = !(Pr > 1.0e-300);
        double x = log10(fmax(Pr, 1.0e-300));
        double A = x - 0.67 * Fc - 0.4;
        double B = 0.806 - 1.1762 * Fc - 0.14 * x;
        double u = A / B;
        double den = 1.0 + u * u;
        double lF = Fc / den;
        F = pow(10.0, lF);
        if (want_deriv) {
            double du_dx = (B + 0.14 * A) / (B * B);
            double du_dFc = (-0.67 * B + 1.1762 * A) / (B * B);
            dlog10F_dx = pr_clamped ? 0.0 : -Fc * 2.0 * u * du_dx / (den * den);
            double dl_dFc = 1.0 / den - Fc * 2.0 * u * du_dFc / (den * den);
            double dFc_dT = fc_clamped ? 0.0 : dFcent / (Fcent * log(10.0));
            dlog10F_dT = dl_dFc * dFc_dT;
        }
    }
    double blend = Pr / (1.0 + Pr);
    o->phi = F * blend;
    if (want_deriv) {
        /* d phi / d Pr = F/(1+Pr)^2 + blend * dF/dPr,  dF/dPr = F/Pr * dlog10F/dx */
        double dphi_dPr = F / ((1.0 + Pr) * (1.0 + Pr)) + F / (1.0 + Pr) * dlog10F_dx;
        o->dphi_dthd = dphi_dPr * (k0 / kf);
        double dlnPr_dT = (M->b0[r] + M->EaR0[r] / T) / T - (M->b[r] + M->EaR[r] / T) / T;
        o->dphi_dT = dphi_dPr * Pr * dlnPr_dT + blend * F * log(10.0) * dlog10F_dT;
    }
}

/* Forward rate coefficient of every reaction at (T, P) (for falloff
 * reactions the high-pressure limit); kf[nrxn]. */
void oracle_kf(int mech, double pres, double T, double* kf) {
    const mech_t* M = &MECHS[mech];
    static const double zero[MAXNSP];
    double C[MAXNSP];
    for (int k = 0; k < M->nsp; ++k) C[k] = 1.0;
    for (int r = 0; r < M->nrxn; ++r) {
        rxn_eval_t e;
        eval_reaction(M, r, T, log(T), pres / (RU * T), C, zero, 0, &e);
        kf[r] = e.kf;
    }
}

/* ------------------------------------------------------------------ RHS */
typedef struct {
    double T, logT, m, yN, mw_avg, rho, cp_avg;
    double Y[MAXNSP], C[MAXNSP], mgRT[MAXNSP], hRT[MAXNSP], cp[MAXNSP], h[MAXNSP];
    double omega[MAXNSP];
} state_t;

/* Cell state.  Constant pressure (conv = 0): pres is P.  Constant volume
 * (conv = 1): pres is the cell's fixed density rho, and the pressure follows
 * from the state, P = rho R T / W (so m = rho / W). */
static void eval_state(const mech_t* M, double pres, int conv, const double* y, state_t* s) {
    const int n = M->nsp;
    s->T = y[0];
    s->logT = log(s->T);
    double sumY = 0.0;
    for (int k = 0; k < n - 1; ++k) { s->Y[k] = y[k + 1]; sumY += y[k + 1]; }
    s->yN = 1.0 - sumY;
    s->Y[n - 1] = s->yN;
    double inv = 0.0;
    for (int k = 0; k < n; ++k) inv += s->Y[k] * (1.0 / M->mw[k]);
    s->mw_avg = 1.0 / inv;
    s->rho = conv ? pres : pres * s->mw_avg / (RU * s->T);
    for (int k = 0; k < n; ++k) s->C[k] = s->rho * s->Y[k] * (1.0 / M->mw[k]);
    s->m = conv ? pres / s->mw_avg : pres / (RU * s->T);
    s->cp_avg = 0.0;
    for (int k = 0; k < n; ++k) {
        const double* a = nasa(M, k, s->T);
        s->mgRT[k] = mg_RT(a, s->T, s->logT);
        s->hRT[k] = h_RT(a, s->T);
        s->cp[k] = RU / M->mw[k] * cp_R(a, s->T);
        s->h[k] = RU / M->mw[k] * s->T * s->hRT[k];
        s->cp_avg += s->cp[k] * s->Y[k];
    }
}

static void add_stoich(const mech_t* M, int r, double q, double* acc) {
    const int P = M->maxp;
    for (int i = 0; i < P; ++i) {
        int s = M->reac_sp[r * P + i];
        if (s < 0) break;
        acc[s] -= M->reac_nu[r * P + i] * q;
    }
    for (int i = 0; i < P; ++i) {
        int s = M->prod_sp[r * P + i];
        if (s < 0) break;
        acc[s] += M->prod_nu[r * P + i] * q;
    }
}

/* dT/dt = -sum_k e_k W_k omega_k / (rho c), e = h, c = cp at constant
 * pressure; e = u = h - R T / W_k, c = cv = cp - R / W at constant volume
 * (closed adiabatic reactor: enthalpy, resp. internal energy, conserved). */
static void rhs_from_state(const mech_t* M, state_t* s, int conv, double* dy, double* scale) {
    const int n = M->nsp;
    double absacc[MAXNSP];
    memset(s->omega, 0, sizeof(double) * n);
    memset(absacc, 0, sizeof(absacc));
    for (int r = 0; r < M->nrxn; ++r) {
        rxn_eval_t e;
        eval_reaction(M, r, s->T, s->logT, s->m, s->C, s->mgRT, 0, &e);
        double q = (e.Rf - e.Rr) * e.phi;
        add_stoich(M, r, q, s->omega);
        if (scale) {
            double qa = (fabs(e.Rf) + fabs(e.Rr)) * fabs(e.phi);
            const int P = M->maxp;
            for (int i = 0; i < P; ++i) { int sp = M->reac_sp[r * P + i]; if (sp < 0) break; absacc[sp] += M->reac_nu[r * P + i] * qa; }
            for (int i = 0; i < P; ++i) { int sp = M->prod_sp[r * P + i]; if (sp < 0) break; absacc[sp] += M->prod_nu[r * P + i] * qa; }
        }
    }
    double Q = 0.0, Qa = 0.0;
    for (int k = 0; k < n; ++k) {
        const double e = conv ? s->h[k] - RU * s->T / M->mw[k] : s->h[k];
        Q += s->omega[k] * e * M->mw[k];
        Qa += absacc[k] * fabs(e) * M->mw[k];
    }
    const double c = conv ? s->cp_avg - RU / s->mw_avg : s->cp_avg;
    dy[0] = (-1.0 / (s->rho * c)) * Q;
    for (int k = 0; k < n - 1; ++k) dy[k + 1] = s->omega[k] * (M->mw[k] / s->rho);
    if (scale) {
        scale[0] = Qa / (s->rho * c);
        for (int k = 0; k < n - 1; ++k) scale[k + 1] = absacc[k] * (M->mw[k] / s->rho);
    }
}

void oracle_dydt(int mech, double pres, const double* y, double* dy) {
    const mech_t* M = &MECHS[mech];
    state_t s;
    eval_state(M, pres, 0, y, &s);
    rhs_from_state(M, &s, 0, dy, NULL);
}

void oracle_dydt_conv(int mech, double rho, const double* y, double* dy) {
    const mech_t* M = &MECHS[mech];
    state_t s;
    eval_state(M, rho, 1, y, &s);
    rhs_from_state(M, &s, 1, dy, NULL);
}

double oracle_density(int mech, double pres, const double* y) {
    const mech_t* M = &MECHS[mech];
    state_t s;
    eval_state(M, pres, 0, y, &s);
    return s.rho;
}

void oracle_dydt_scale(int mech, double pres, const double* y, double* scale) {
    const mech_t* M = &MECHS[mech];
    state_t s;
    double dy[MAXNSP];
    eval_state(M, pres, 0, y, &s);
    rhs_from_state(M, &s, 0, dy, scale);
}

void oracle_dydt_scale_conv(int mech, double rho, const double* y, double* scale) {
    const mech_t* M = &MECHS[mech];
    state_t s;
    double dy[MAXNSP];
    eval_state(M, rho, 1, y, &s);
    rhs_from_state(M, &s, 1, dy, scale);
}

/* -------------------------------------------------------------- Jacobian */

/* Stoichiometric coefficient of entry e of the reactant (side 0) or product
 * (side 1) list. */
static double stoich(const mech_t* M, int side, int e) {
    return side ? M->prod_nu[e] : (double)M->reac_nu[e];
}

/* Exact Jacobian of rhs_from_state.  Constant pressure: C_k = rho(Y, T) Y_k / W_k
 * with rho = P W / (R T) and m = P / (R T).  Constant volume: rho fixed,
 * m = sum_k C_k, P = m R T, so C and m do not depend on T, the third-body
 * concentration and the PLOG pressure depend on every C_i (g_k below), and the
 * energy equation uses u and cv. */
static void jacob_impl(int mech, double pres, int conv, const double* y, double* jac) {
    const mech_t* M = &MECHS[mech];
    const int n = M->nsp, P = M->maxp;
    state_t s;
    eval_state(M, pres, conv, y, &s);
    const double T = s.T;
    /* Jc[k][i] = d omega_k / d C_i (dense, closure column/row included) */
    double* Jc = (double*)calloc((size_t)n * n, sizeof(double));
    double domega_dT[MAXNSP], sk[MAXNSP];
    memset(s.omega, 0, sizeof(double) * n);
    memset(domega_dT, 0, sizeof(domega_dT));
    memset(sk, 0, sizeof(sk));
    for (int r = 0; r < M->nrxn; ++r) {
        rxn_eval_t e;
        eval_reaction(M, r, T, s.logT, s.m, s.C, s.mgRT, 1, &e);
        double R = e.Rf - e.Rr;
        double q = R * e.phi;
        /* d ln kr / dT = d ln kf / dT - d ln Kc / dT,
           d ln Kc / dT = (sum nu h/RT - dnu) / T */
        double dH = 0.0, dnu = 0.0;
        for (int i = 0; i < P; ++i) { int sp = M->reac_sp[r * P + i]; if (sp < 0) break; dH -= M->reac_nu[r * P + i] * s.hRT[sp]; dnu -= M->reac_nu[r * P + i]; }
        for (int i = 0; i < P; ++i) { int sp = M->prod_sp[r * P + i]; if (sp < 0) break; dH += M->prod_nu[r * P + i] * s.hRT[sp]; dnu += M->prod_nu[r * P + i]; }
        double dlnkr = M->rev[r] ? e.dlnkf_dT - (dH - dnu) / T : 0.0;
        double dR_dT = e.Rf * e.dlnkf_dT - e.Rr * dlnkr;   /* at fixed C */
        double Sr = e.phi * (e.ordf * e.Rf - e.ordr * e.Rr);
        double thd_term = R * e.dphi_dthd;                  /* dq/dthd */
        double dq_dT, s_r;
        if (!conv) {
            dq_dT = e.phi * dR_dT + R * e.dphi_dT - (Sr + thd_term * e.thd) / T;
            s_r = Sr + thd_term * (e.thd - s.m);            /* sum_i dq/dC_i C_i */
        } else {
            /* C fixed in T; P = m R T moves PLOG rates with T and with m */
            dq_dT = e.phi * dR_dT + R * e.dphi_dT + q * e.dlnk_dlnP / T;
            s_r = thd_term + q * e.dlnk_dlnP / s.m;         /* dq/dm, m = sum_i C_i */
        }
        /* dq/dC_j for mass-action participants */
        double dqdC[2 * MAXP_ORACLE];
        int jsp[2 * MAXP_ORACLE], nj = 0;
        for (int side = 0; side < 1 + M->rev[r]; ++side) {   /* products: reverse rate only */
            const int* sp_t = side ? M->prod_sp : M->reac_sp;
            double kcoef = side ? -e.kr : e.kf;
            for (int i = 0; i < P; ++i) {
                int sp = sp_t[r * P + i];
                if (sp < 0) break;
                double d = kcoef * stoich(M, side, r * P + i);
                for (int i2 = 0; i2 < P; ++i2) {
                    int sp2 = sp_t[r * P + i2];
                    if (sp2 < 0) break;
                    int nu2 = (int)stoich(M, side, r * P + i2) - (i2 == i ? 1 : 0);
                    for (int qq = 0; qq < nu2; ++qq) d *= s.C[sp2];
                }
                jsp[nj] = sp; dqdC[nj] = d * e.phi; ++nj;
            }
        }
        /* scatter into rows of species with nonzero net stoichiometry */
        for (int side = 0; side < 2; ++side) {
            const int* sp_t = side ? M->prod_sp : M->reac_sp;
            double sg = side ? 1.0 : -1.0;
            for (int i = 0; i < P; ++i) {
                int k = sp_t[r * P + i];
                if (k < 0) break;
                double nu = sg * stoich(M, side, r * P + i);
                s.omega[k] += nu * q;
                domega_dT[k] += nu * dq_dT;
                sk[k] += nu * s_r;
                for (int a = 0; a < nj; ++a) Jc[k * n + jsp[a]] += nu * dqdC[a];
                if (thd_term != 0.0 || M->type[r] != 0)
                    for (int t = M->tb_off[r]; t < M->tb_off[r + 1]; ++t)
                        Jc[k * n + M->tb_sp[t]] += nu * thd_term * M->tb_alpha[t];
            }
        }
    }
    const int N = n - 1;   /* closure species index */
    double f[MAXNSP], dfdT[MAXNSP], e[MAXNSP], c[MAXNSP];
    /* energy per mass and heat capacity of each species: h, cp (constant
       pressure) or u = h - R T / W_k, cv = cp - R / W_k (constant volume) */
    for (int k = 0; k < n; ++k) {
        e[k] = conv ? s.h[k] - RU * T / M->mw[k] : s.h[k];
        c[k] = conv ? s.cp[k] - RU / M->mw[k] : s.cp[k];
    }
    const double c_avg = conv ? s.cp_avg - RU / s.mw_avg : s.cp_avg;
    /* species rows (including the closure row k = N) */
    double Q = 0.0;
    for (int k = 0; k < n; ++k) {
        f[k] = s.omega[k] * M->mw[k] / s.rho;
        Q += e[k] * f[k];
        dfdT[k] = (M->mw[k] / s.rho) * (domega_dT[k] + (conv ? 0.0 : s.omega[k] / T));
    }
    double fT = -Q / c_avg;
    double* JY = (double*)calloc((size_t)n * n, sizeof(double));   /* JY[k*n + j], j < N */
    const double WN = M->mw[N];
    for (int k = 0; k < n; ++k) {
        /* d/dY_j beyond the direct dC_j: rho(W) at constant pressure, m(C) at constant volume */
        const double X = conv ? sk[k] : (s.mw_avg / s.rho) * (s.omega[k] - sk[k]);
        for (int j = 0; j < N; ++j) {
            double dj = 1.0 / M->mw[j] - 1.0 / WN;
            JY[k * n + j] = M->mw[k] * (Jc[k * n + j] / M->mw[j] - Jc[k * n + N] / WN + dj * X);
        }
    }
    /* assemble column-major output */
    for (int j = 0; j < N; ++j) {
        double acc = 0.0;
        for (int k = 0; k < n; ++k) acc += e[k] * JY[k * n + j];
        jac[0 + n * (j + 1)] = -(acc + fT * (c[j] - c[N])) / c_avg;
        for (int k = 0; k < N; ++k) jac[(k + 1) + n * (j + 1)] = JY[k * n + j];
    }
    double accT = 0.0, dcp = 0.0;
    for (int k = 0; k < n; ++k) {
        accT += c[k] * f[k] + e[k] * dfdT[k];
        dcp += s.Y[k] * RU / M->mw[k] * dcp_R(nasa(M, k, T), T);
    }
    jac[0] = -(accT + fT * dcp) / c_avg;
    for (int k = 0; k < N; ++k) jac[k + 1] = dfdT[k];
    free(Jc);
    free(JY);
}

void oracle_jacob(int mech, double pres, const double* y, double* jac) { jacob_impl(mech, pres, 0, y, jac); }
void oracle_jacob_conv(int mech, double rho, const double* y, double* jac) { jacob_impl(mech, rho, 1, y, jac); }

void oracle_gri30_dydt(double t, double pres, const double* y, double* dy) { (void)t; oracle_dydt(ORACLE_MECH_GRI30, pres, y, dy); }
void oracle_gri30_jacob(double t, double pres, const double* y, double* jac) { (void)t; oracle_jacob(ORACLE_MECH_GRI30, pres, y, jac); }
void oracle_h2o2_dydt(double t, double pres, const double* y, double* dy) { (void)t; oracle_dydt(ORACLE_MECH_H2O2, pres, y, dy); }
void oracle_h2o2_jacob(double t, double pres, const double* y, double* jac) { (void)t; oracle_jacob(ORACLE_MECH_H2O2, pres, y, jac); }
void oracle_ndodecane_dydt(double t, double pres, const double* y, double* dy) { (void)t; oracle_dydt(ORACLE_MECH_NDODECANE, pres, y, dy); }
void oracle_ndodecane_jacob(double t, double pres, const double* y, double* jac) { (void)t; oracle_jacob(ORACLE_MECH_NDODECANE, pres, y, jac); }
void oracle_h2li_dydt(double t, double pres, const double* y, double* dy) { (void)t; oracle_dydt(ORACLE_MECH_H2LI, pres, y, dy); }
void oracle_h2li_jacob(double t, double pres, const double* y, double* jac) { (void)t; oracle_jacob(ORACLE_MECH_H2LI, pres, y, jac); }
void oracle_estimate_dydt(double t, double pres, const double* y, double* dy) { (void)t; oracle_dydt(ORACLE_MECH_ESTIMATE, pres, y, dy); }
void oracle_estimate_jacob(double t, double pres, const double* y, double* jac) { (void)t; oracle_jacob(ORACLE_MECH_ESTIMATE, pres, y, jac); }

/* Constant-volume forms with pyJac's signature (the pres argument carries the
 * cell's density), for the BDF driver. */
#define CONV_FNS(tag, ID)                                                                              \
    static void tag##_dydt_conv(double t, double rho, const double* y, double* dy) {                   \
        (void)t; oracle_dydt_conv(ID, rho, y, dy);                                                       \
    }                                                                                                    \
    static void tag##_jacob_conv(double t, double rho, const double* y, double* jac) {                 \
        (void)t; oracle_jacob_conv(ID, rho, y, jac);                                                     \
    }
CONV_FNS(gri30, ORACLE_MECH_GRI30)
CONV_FNS(h2o2, ORACLE_MECH_H2O2)
CONV_FNS(ndodecane, ORACLE_MECH_NDODECANE)
CONV_FNS(h2li, ORACLE_MECH_H2LI)
CONV_FNS(estimate, ORACLE_MECH_ESTIMATE)

void oracle_mech_fns(int mech, int conv, oracle_rhs_fn* f, oracle_jac_fn* J) {
    static const oracle_rhs_fn F[2][NMECH] = {
        {oracle_gri30_dydt, oracle_h2o2_dydt, oracle_ndodecane_dydt, oracle_h2li_dydt, oracle_estimate_dydt},
        {gri30_dydt_conv, h2o2_dydt_conv, ndodecane_dydt_conv, h2li_dydt_conv, estimate_dydt_conv}};
    static const oracle_jac_fn G[2][NMECH] = {
        {oracle_gri30_jacob, oracle_h2o2_jacob, oracle_ndodecane_jacob, oracle_h2li_jacob, oracle_estimate_jacob},
        {gri30_jacob_conv, h2o2_jacob_conv, ndodecane_jacob_conv, h2li_jacob_conv, estimate_jacob_conv}};
    *f = F[conv ? 1 : 0][mech];
    *J = G[conv ? 1 : 0][mech];
}
