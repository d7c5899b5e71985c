/* CPU oracle: CVODE-semantics BDF -- TEST INFRASTRUCTURE ONLY (see bdf_oracle.h).
 *
 * Restated from CVODE's published algorithm (Hindmarsh et al. 2005; CVODE
 * user guide, "Mathematical considerations"), with CVODE's documented
 * defaults: maxord 5; Nordsieck history zn[0..q]; fixed-leading-coefficient
 * BDF coefficients l[] and error constants tq[1..5]; modified Newton on
 * M = I - gamma*J with at most 3 iterations, crate/CRDOWN=0.3 convergence
 * test against tq[4] = 0.1/tq[2] and RDIV=2 divergence test; linear-solver
 * setup when gamma changed by more than 30 %, every 20 steps (msbp) or after a
 * failure; Jacobian re-evaluation every 51 steps (msbj), after a convergence
 * failure, or when a failed iteration with a stale J had |gamma/gammap-1| <
 * 0.2; solution scaling 2/(1+gamrat); error test dsm = ||acor||*tq[2] <= 1,
 * eta = 1/((6 dsm)^(1/L) + 1e-6) bounded by [0.1, 0.2] after repeated
 * failures, order drop after 3 failures, fail at 7; convergence failures
 * eta = 0.25, fail at 10; step/order selection with biases 6/6/10, growth
 * cap 1e4 on the first step then 10, no change for eta < 1.5; initial step
 * from CVODE's h0 heuristic; CV_NORMAL output by interpolation of zn at tout.
 *
 * The reference calls CVode once per cell from t=0 to tout=dt
 * (CVodeIntegrator.cpp:143) after CVodeSStolerances (:122) and
 * CVodeSetMaxNumSteps(10000) (:137).
 */
#include "bdf_oracle.h"
#include "chem_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define QMAX 5
#define LMAX (QMAX + 1)
#define UROUND DBL_EPSILON

/* CVODE defaults */
#define ETAMX1 10000.0
#define ETAMX2 10.0
#define ETAMX3 10.0
#define ETAMXF 0.2
#define ETAMIN 0.1
#define ETACF 0.25
#define ADDON 1.0e-6
#define BIAS1 6.0
#define BIAS2 6.0
#define BIAS3 10.0
#define THRESH 1.5
#define SMALL_NST 10
#define MXNCF 10
#define MXNEF 7
#define MXNEF1 3
#define SMALL_NEF 2
#define LONG_WAIT 10
#define NLS_MAXCOR 3
#define CRDOWN 0.3
#define RDIV 2.0
#define DGMAX_LSETUP 0.3
#define MSBP 20
#define DGMAX_JBAD 0.2
#define MSBJ 51
#define NLSCOEF 0.1
#define HLB_FACTOR 100.0
#define HUB_FACTOR 0.1
#define H_BIAS 0.5
#define MAX_HIN_ITERS 4

enum { FIRST_CALL, PREV_CONV_FAIL, PREV_ERR_FAIL };
enum { CV_NO_FAILURES, CV_FAIL_BAD_J, CV_FAIL_OTHER };
enum { DO_ERROR_TEST = 2, PREDICT_AGAIN = 3, TRY_AGAIN = 5 };
#define CONV_RECVR 901

typedef struct {
    int n;
    oracle_rhs_fn f;
    oracle_jac_fn jacf;
    double pres, rtol, atol;
    int max_steps, qmax;
    /* Nordsieck history and work vectors */
    double* zn[LMAX + 1];
    double *ewt, *acor, *tempv, *ftemp, *y, *delta;
    double *J, *M;           /* saved Jacobian and LU factors, column-major */
    int* piv;
    double tq[6], l[LMAX + 1], tau[LMAX + 2];
    double tn, h, hprime, hscale, eta, etamax, hu, saved_tq5;
    double gamma, gammap, gamrat, rl1, crate, acnrm;
    double etaq, etaqm1, etaqp1;
    int q, qprime, qwait, L, indx_acor;
    long nst, nstlp, nstlj;
    int jcur, convfail;
    oracle_bdf_stats st;
} bdf_mem;

/* ------------------------------------------------------------ vector ops */
static double wrms(int n, const double* x, const double* w) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) { double t = x[i] * w[i]; s += t * t; }
    return sqrt(s / n);
}
static void set_ewt(bdf_mem* m, const double* y) {
    for (int i = 0; i < m->n; ++i) m->ewt[i] = 1.0 / (m->rtol * fabs(y[i]) + m->atol);
}
static void rhs(bdf_mem* m, double t, const double* y, double* out) {
    m->f(t, m->pres, y, out);
    m->st.nfe++;
}

/* -------------------------------------------------------- dense LU (n x n) */
/* Column-major LU with partial pivoting (first index of max |a_ik|),
 * multipliers by reciprocal of the pivot. Returns 0 or k+1 on a zero pivot. */
static int lu_factor(int n, double* a, int* p) {
    for (int k = 0; k < n; ++k) {
        double* ck = a + (size_t)k * n;
        int l = k;
        for (int i = k + 1; i < n; ++i) if (fabs(ck[i]) > fabs(ck[l])) l = i;
        p[k] = l;
        if (ck[l] == 0.0) return k + 1;
        if (l != k) for (int j = 0; j < n; ++j) { double t = a[l + (size_t)j * n]; a[l + (size_t)j * n] = a[k + (size_t)j * n]; a[k + (size_t)j * n] = t; }
        double mult = 1.0 / ck[k];
        for (int i = k + 1; i < n; ++i) ck[i] *= mult;
        for (int j = k + 1; j < n; ++j) {
            double* cj = a + (size_t)j * n;
            double akj = cj[k];
            if (akj != 0.0) for (int i = k + 1; i < n; ++i) cj[i] -= akj * ck[i];
        }
    }
    return 0;
}
static void lu_solve(int n, const double* a, const int* p, double* b) {
    for (int k = 0; k < n; ++k) { int pk = p[k]; if (pk != k) { double t = b[k]; b[k] = b[pk]; b[pk] = t; } }
    for (int k = 0; k < n - 1; ++k) { double bk = b[k]; const double* ck = a + (size_t)k * n; for (int i = k + 1; i < n; ++i) b[i] -= ck[i] * bk; }
    for (int k = n - 1; k > 0; --k) { const double* ck = a + (size_t)k * n; b[k] /= ck[k]; double bk = b[k]; for (int i = 0; i < k; ++i) b[i] -= ck[i] * bk; }
    b[0] /= a[0];
}

/* ------------------------------------------------------ Nordsieck helpers */
static void rescale(bdf_mem* m) {
    double factor = m->eta;
    for (int j = 1; j <= m->q; ++j) {
        for (int i = 0; i < m->n; ++i) m->zn[j][i] *= factor;
        factor *= m->eta;
    }
    m->h = m->hscale * m->eta;
    m->hscale = m->h;
}
static void predict(bdf_mem* m) {
    m->tn += m->h;
    for (int k = 1; k <= m->q; ++k)
        for (int j = m->q; j >= k; --j)
            for (int i = 0; i < m->n; ++i) m->zn[j - 1][i] += m->zn[j][i];
}
static void restore(bdf_mem* m, double saved_t) {
    m->tn = saved_t;
    for (int k = 1; k <= m->q; ++k)
        for (int j = m->q; j >= k; --j)
            for (int i = 0; i < m->n; ++i) m->zn[j - 1][i] -= m->zn[j][i];
}
static void increase_bdf(bdf_mem* m) {
    for (int j = 0; j <= QMAX; ++j) m->l[j] = 0.0;
    m->l[2] = 1.0;
    double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = m->hscale;
    if (m->q > 1) {
        for (int j = 1; j < m->q; ++j) {
            hsum += m->tau[j + 1];
            double xi = hsum / m->hscale;
            prod *= xi;
            alpha0 -= 1.0 / (j + 1);
            alpha1 += 1.0 / xi;
            for (int i = j + 2; i >= 2; --i) m->l[i] = m->l[i] * xiold + m->l[i - 1];
            xiold = xi;
        }
    }
    double A1 = (-alpha0 - alpha1) / prod;
    int L = m->L;   /* q + 1 at the old order: the new column */
    for (int i = 0; i < m->n; ++i) m->zn[L][i] = A1 * m->zn[m->indx_acor][i];
    for (int j = 2; j <= m->q; ++j)
        for (int i = 0; i < m->n; ++i) m->zn[j][i] += m->l[j] * m->zn[L][i];
}
static void decrease_bdf(bdf_mem* m) {
    for (int j = 0; j <= QMAX; ++j) m->l[j] = 0.0;
    m->l[2] = 1.0;
    double hsum = 0.0;
    for (int j = 1; j <= m->q - 2; ++j) {
        hsum += m->tau[j];
        double xi = hsum / m->hscale;
        for (int i = j + 2; i >= 2; --i) m->l[i] = m->l[i] * xi + m->l[i - 1];
    }
    for (int j = 2; j < m->q; ++j)
        for (int i = 0; i < m->n; ++i) m->zn[j][i] += -m->l[j] * m->zn[m->q][i];
}
static void adjust_order(bdf_mem* m, int deltaq) {
    if (m->q == 2 && deltaq != 1) return;   /* CVODE: no change below order 2 adjustment */
    if (deltaq == 1) increase_bdf(m);
    else if (deltaq == -1) decrease_bdf(m);
}
static void adjust_params(bdf_mem* m) {
    if (m->qprime != m->q) {
        adjust_order(m, m->qprime - m->q);
        m->q = m->qprime;
        m->L = m->q + 1;
        m->qwait = m->L;
    }
    rescale(m);
}

/* --------------------------------------------------- method coefficients */
static void set_tq_bdf(bdf_mem* m, double hsum, double alpha0, double alpha0_hat,
                       double xi_inv, double xistar_inv) {
    int q = m->q;
    double A1 = 1.0 - alpha0_hat + alpha0;
    double A2 = 1.0 + q * A1;
    m->tq[2] = fabs(A1 / (alpha0 * A2));
    m->tq[5] = fabs(A2 * xistar_inv / (m->l[q] * xi_inv));
    if (m->qwait == 1) {
        if (q > 1) {
            double C = xistar_inv / m->l[q];
            double A3 = alpha0 + 1.0 / q;
            double A4 = alpha0_hat + xi_inv;
            double Cpinv = (1.0 - A4 + A3) / A3;
            m->tq[1] = fabs(C * Cpinv);
        } else {
            m->tq[1] = 1.0;
        }
        hsum += m->tau[q];
        xi_inv = m->h / hsum;
        double A5 = alpha0 - 1.0 / (q + 1);
        double A6 = alpha0_hat - xi_inv;
        double Cppinv = (1.0 - A6 + A5) / A2;
        m->tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    m->tq[4] = NLSCOEF / m->tq[2];
}
static void set_bdf(bdf_mem* m) {
    int q = m->q;
    m->l[0] = m->l[1] = 1.0;
    double xi_inv = 1.0, xistar_inv = 1.0;
    for (int j = 2; j <= q; ++j) m->l[j] = 0.0;
    double alpha0 = -1.0, alpha0_hat = -1.0, hsum = m->h;
    if (q > 1) {
        for (int j = 2; j < q; ++j) {
            hsum += m->tau[j - 1];
            xi_inv = m->h / hsum;
            alpha0 -= 1.0 / j;
            for (int i = j; i >= 1; --i) m->l[i] += m->l[i - 1] * xi_inv;
        }
        alpha0 -= 1.0 / q;
        xistar_inv = -m->l[1] - alpha0;
        hsum += m->tau[q - 1];
        xi_inv = m->h / hsum;
        alpha0_hat = -m->l[1] - xi_inv;
        for (int i = q; i >= 1; --i) m->l[i] += m->l[i - 1] * xistar_inv;
    }
    set_tq_bdf(m, hsum, alpha0, alpha0_hat, xi_inv, xistar_inv);
}
static void set_coeffs(bdf_mem* m) {
    set_bdf(m);
    m->rl1 = 1.0 / m->l[1];
    m->gamma = m->h * m->rl1;
    if (m->nst == 0) m->gammap = m->gamma;
    m->gamrat = (m->nst > 0) ? m->gamma / m->gammap : 1.0;
}

/* ------------------------------------------------------- Newton iteration */
/* residual: y = zn0 + ycor; ftemp = f(y); res = rl1*zn1 + ycor - gamma*ftemp */
static void nls_residual(bdf_mem* m, const double* ycor, double* res) {
    int n = m->n;
    for (int i = 0; i < n; ++i) m->y[i] = m->zn[0][i] + ycor[i];
    rhs(m, m->tn, m->y, m->ftemp);
    for (int i = 0; i < n; ++i) res[i] = m->rl1 * m->zn[1][i] + ycor[i];
    for (int i = 0; i < n; ++i) res[i] = -m->gamma * m->ftemp[i] + res[i];
}
/* linear-solver setup (J reuse decision, M = I - gamma J, LU) */
static int ls_setup(bdf_mem* m, int convfail) {
    int n = m->n;
    double dgamma = fabs(m->gamma / m->gammap - 1.0);
    int jbad = (m->nst == 0) || (m->nst >= m->nstlj + MSBJ) ||
               ((convfail == CV_FAIL_BAD_J) && (dgamma < DGMAX_JBAD)) ||
               (convfail == CV_FAIL_OTHER);
    if (!jbad) {
        m->jcur = 0;
    } else {
        m->st.nje++;
        m->nstlj = m->nst;
        m->jcur = 1;
        memset(m->J, 0, sizeof(double) * (size_t)n * n);
        m->jacf(m->tn, m->pres, m->y, m->J);
    }
    for (size_t i = 0; i < (size_t)n * n; ++i) m->M[i] = -m->gamma * m->J[i];
    for (int i = 0; i < n; ++i) m->M[i + (size_t)i * n] += 1.0;
    return lu_factor(n, m->M, m->piv) ? 1 : 0;
}
static int nls_lsetup(bdf_mem* m, int jbad) {
    if (jbad) m->convfail = CV_FAIL_BAD_J;
    int ret = ls_setup(m, m->convfail);
    m->st.nsetups++;
    m->gamrat = 1.0;
    m->gammap = m->gamma;
    m->crate = 1.0;
    m->nstlp = m->nst;
    return ret ? CONV_RECVR : 0;
}
static void ls_solve(bdf_mem* m, double* b) {
    lu_solve(m->n, m->M, m->piv, b);
    if (m->gamrat != 1.0) {
        double s = 2.0 / (1.0 + m->gamrat);
        for (int i = 0; i < m->n; ++i) b[i] *= s;
    }
}
/* returns 0 converged, CONV_RECVR, or a negative error */
static int nls_solve(bdf_mem* m, int call_setup) {
    int n = m->n;
    double* ycor = m->acor;
    double* delta = m->delta;
    int jbad = 0, ret = 0;
    for (;;) {
        nls_residual(m, ycor, delta);
        if (call_setup) {
            ret = nls_lsetup(m, jbad);
            if (ret) break;
        }
        double delp = 0.0;
        int m_it = 0;
        for (;;) {
            m->st.nni++;
            for (int i = 0; i < n; ++i) delta[i] = -delta[i];
            ls_solve(m, delta);
            for (int i = 0; i < n; ++i) ycor[i] += delta[i];
            /* convergence test */
            double del = wrms(n, delta, m->ewt);
            if (m_it > 0) m->crate = fmax(CRDOWN * m->crate, del / delp);
            double dcon = del * fmin(1.0, m->crate) / m->tq[4];
            if (dcon <= 1.0) {
                m->acnrm = (m_it == 0) ? del : wrms(n, ycor, m->ewt);
                m->jcur = 0;
                return 0;
            }
            if (m_it >= 1 && del > RDIV * delp) { ret = CONV_RECVR; break; }
            delp = del;
            m_it++;
            if (m_it >= NLS_MAXCOR) { ret = CONV_RECVR; break; }
            nls_residual(m, ycor, delta);
        }
        if (ret == CONV_RECVR && !m->jcur) {
            call_setup = 1;
            jbad = 1;
            for (int i = 0; i < n; ++i) ycor[i] = 0.0;
            continue;
        }
        break;
    }
    return ret;
}
static int nls(bdf_mem* m, int nflag) {
    m->convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? CV_NO_FAILURES : CV_FAIL_OTHER;
    int call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (m->nst == 0) ||
                     (m->nst >= m->nstlp + MSBP) || (fabs(m->gamrat - 1.0) > DGMAX_LSETUP);
    for (int i = 0; i < m->n; ++i) m->acor[i] = 0.0;
    int ret = nls_solve(m, call_setup);
    for (int i = 0; i < m->n; ++i) m->y[i] = m->zn[0][i] + m->acor[i];
    return ret;
}

static int handle_nflag(bdf_mem* m, int* nflag, double saved_t, int* ncf) {
    if (*nflag == 0) return DO_ERROR_TEST;
    m->st.ncfn++;
    restore(m, saved_t);
    (*ncf)++;
    m->etamax = 1.0;
    if (*ncf == MXNCF) return ORACLE_CV_CONV_FAILURE;
    m->eta = ETACF;
    *nflag = PREV_CONV_FAIL;
    rescale(m);
    return PREDICT_AGAIN;
}

static int do_error_test(bdf_mem* m, int* nflag, double saved_t, int* nef, double* dsm_out) {
    double dsm = m->acnrm * m->tq[2];
    *dsm_out = dsm;
    if (dsm <= 1.0) return 0;
    (*nef)++;
    m->st.netf++;
    *nflag = PREV_ERR_FAIL;
    restore(m, saved_t);
    if (*nef == MXNEF) return ORACLE_CV_ERR_FAILURE;
    m->etamax = 1.0;
    if (*nef <= MXNEF1) {
        m->eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / m->L) + ADDON);
        m->eta = fmax(ETAMIN, m->eta);
        if (*nef >= SMALL_NEF) m->eta = fmin(m->eta, ETAMXF);
        rescale(m);
        return TRY_AGAIN;
    }
    if (m->q > 1) {
        m->eta = ETAMIN;
        adjust_order(m, -1);
        m->L = m->q;
        m->q--;
        m->qwait = m->L;
        rescale(m);
        return TRY_AGAIN;
    }
    m->eta = ETAMIN;
    m->h *= m->eta;
    m->hscale = m->h;
    m->qwait = LONG_WAIT;
    rhs(m, m->tn, m->zn[0], m->tempv);
    for (int i = 0; i < m->n; ++i) m->zn[1][i] = m->h * m->tempv[i];
    return TRY_AGAIN;
}

static void complete_step(bdf_mem* m) {
    m->nst++;
    m->hu = m->h;
    for (int i = m->q; i >= 2; --i) m->tau[i] = m->tau[i - 1];
    if (m->q == 1 && m->nst > 1) m->tau[2] = m->tau[1];
    m->tau[1] = m->h;
    for (int j = 0; j <= m->q; ++j)
        for (int i = 0; i < m->n; ++i) m->zn[j][i] += m->l[j] * m->acor[i];
    m->qwait--;
    if (m->qwait == 1 && m->q != m->qmax) {
        memcpy(m->zn[m->qmax], m->acor, sizeof(double) * m->n);
        m->saved_tq5 = m->tq[5];
        m->indx_acor = m->qmax;
    }
}

static void set_eta(bdf_mem* m) {
    if (m->eta < THRESH) {
        m->eta = 1.0;
        m->hprime = m->h;
    } else {
        m->eta = fmin(m->eta, m->etamax);
        m->hprime = m->h * m->eta;
    }
}
static double compute_etaqm1(bdf_mem* m) {
    double e = 0.0;
    if (m->q > 1) {
        double ddn = wrms(m->n, m->zn[m->q], m->ewt) * m->tq[1];
        e = 1.0 / (pow(BIAS1 * ddn, 1.0 / m->q) + ADDON);
    }
    return e;
}
static double compute_etaqp1(bdf_mem* m) {
    double e = 0.0;
    if (m->q != m->qmax) {
        if (m->saved_tq5 == 0.0) return 0.0;
        double cquot = (m->tq[5] / m->saved_tq5) * pow(m->h / m->tau[2], (double)m->L);
        for (int i = 0; i < m->n; ++i) m->tempv[i] = m->acor[i] - cquot * m->zn[m->qmax][i];
        double dup = wrms(m->n, m->tempv, m->ewt) * m->tq[3];
        e = 1.0 / (pow(BIAS3 * dup, 1.0 / (m->L + 1)) + ADDON);
    }
    return e;
}
static void choose_eta(bdf_mem* m) {
    double etam = fmax(m->etaqm1, fmax(m->etaq, m->etaqp1));
    if (etam < THRESH) {
        m->eta = 1.0;
        m->qprime = m->q;
        return;
    }
    if (etam == m->etaqm1) {
        m->eta = m->etaqm1;
        m->qprime = m->q - 1;
    } else if (etam == m->etaq) {
        m->eta = m->etaq;
        m->qprime = m->q;
    } else {
        m->eta = m->etaqp1;
        m->qprime = m->q + 1;
        memcpy(m->zn[m->qmax], m->acor, sizeof(double) * m->n);
    }
}
static void prepare_next_step(bdf_mem* m, double dsm) {
    if (m->etamax == 1.0) {
        if (m->qwait < 2) m->qwait = 2;
        m->qprime = m->q;
        m->hprime = m->h;
        m->eta = 1.0;
        return;
    }
    m->etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / m->L) + ADDON);
    if (m->qwait != 0) {
        m->eta = m->etaq;
        m->qprime = m->q;
        set_eta(m);
        return;
    }
    m->qwait = 2;
    m->etaqm1 = compute_etaqm1(m);
    m->etaqp1 = compute_etaqp1(m);
    choose_eta(m);
    set_eta(m);
}

static int step(bdf_mem* m) {
    double saved_t = m->tn;
    int ncf = 0, nef = 0, nflag = FIRST_CALL;
    double dsm = 0.0;
    if (m->nst > 0 && m->hprime != m->h) adjust_params(m);
    for (;;) {
        predict(m);
        set_coeffs(m);
        nflag = nls(m, nflag);
        int kflag = handle_nflag(m, &nflag, saved_t, &ncf);
        if (kflag == PREDICT_AGAIN) continue;
        if (kflag != DO_ERROR_TEST) return kflag;
        int eflag = do_error_test(m, &nflag, saved_t, &nef, &dsm);
        if (eflag == TRY_AGAIN) continue;
        if (eflag != 0) return eflag;
        break;
    }
    complete_step(m);
    prepare_next_step(m, dsm);
    m->etamax = (m->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
    for (int i = 0; i < m->n; ++i) m->acor[i] *= m->tq[2];
    return 0;
}

/* ------------------------------------------------------------ initial h */
static double upper_bound_h0(bdf_mem* m, double tdist) {
    double hub_inv = 0.0;
    for (int i = 0; i < m->n; ++i) {
        double den = HUB_FACTOR * fabs(m->zn[0][i]) + 1.0 / m->ewt[i];
        double r = fabs(m->zn[1][i]) / den;
        if (r > hub_inv) hub_inv = r;
    }
    double hub = HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    return hub;
}
static double ydd_norm(bdf_mem* m, double hg) {
    for (int i = 0; i < m->n; ++i) m->y[i] = hg * m->zn[1][i] + m->zn[0][i];
    rhs(m, m->tn + hg, m->y, m->tempv);
    for (int i = 0; i < m->n; ++i) m->tempv[i] = (m->tempv[i] - m->zn[1][i]) * (1.0 / hg);
    return wrms(m->n, m->tempv, m->ewt);
}
static int hin(bdf_mem* m, double tout, double* h0_out) {
    double tdiff = tout - m->tn;
    if (tdiff == 0.0) return ORACLE_CV_TOO_CLOSE;
    int sign = (tdiff > 0.0) ? 1 : -1;
    double tdist = fabs(tdiff);
    double tround = UROUND * fmax(fabs(m->tn), fabs(tout));
    if (tdist < 2.0 * tround) return ORACLE_CV_TOO_CLOSE;
    double hlb = HLB_FACTOR * tround;
    double hub = upper_bound_h0(m, tdist);
    double hg = sqrt(hlb * hub);
    if (hub < hlb) { *h0_out = sign * hg; return 0; }
    double hnew = hg;
    for (int count1 = 1; count1 <= MAX_HIN_ITERS; ++count1) {
        double yddnrm = ydd_norm(m, hg * sign);
        hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
        if (count1 == MAX_HIN_ITERS) break;
        double hrat = hnew / hg;
        if (hrat > 0.5 && hrat < 2.0) break;
        if (count1 > 1 && hrat > 2.0) { hnew = hg; break; }
        hg = hnew;
    }
    double h0 = H_BIAS * hnew;
    if (h0 < hlb) h0 = hlb;
    if (h0 > hub) h0 = hub;
    *h0_out = sign * h0;
    return 0;
}

/* CVodeGetDky(t, 0): y(t) = sum_j s^j zn[j], s = (t - tn)/h */
static void get_dky(bdf_mem* m, double t, double* out) {
    double s = (t - m->tn) / m->h;
    for (int i = 0; i < m->n; ++i) out[i] = m->zn[m->q][i];
    for (int j = m->q - 1; j >= 0; --j)
        for (int i = 0; i < m->n; ++i) out[i] = m->zn[j][i] + s * out[i];
}

int oracle_bdf_solve(oracle_rhs_fn f, oracle_jac_fn J, int n, double pres, double* y,
                     double t0, double tout, const oracle_bdf_opts* opts,
                     oracle_bdf_stats* stats) {
    bdf_mem mm;
    bdf_mem* m = &mm;
    memset(m, 0, sizeof(*m));
    m->n = n; m->f = f; m->jacf = J; m->pres = pres;
    m->rtol = opts->rtol; m->atol = opts->atol;
    m->max_steps = opts->max_steps > 0 ? opts->max_steps : 500;
    m->qmax = (opts->max_order >= 1 && opts->max_order <= QMAX) ? opts->max_order : QMAX;
    size_t nv = (size_t)(LMAX + 7) * n + 2 * (size_t)n * n;
    double* buf = (double*)calloc(nv, sizeof(double));
    int* piv = (int*)calloc((size_t)n, sizeof(int));
    double* p = buf;
    for (int j = 0; j <= LMAX; ++j) { m->zn[j] = p; p += n; }
    m->ewt = p; p += n; m->acor = p; p += n; m->tempv = p; p += n; m->ftemp = p; p += n;
    m->y = p; p += n; m->delta = p; p += n;
    m->J = p; p += (size_t)n * n; m->M = p; p += (size_t)n * n;
    m->piv = piv;

    memcpy(m->zn[0], y, sizeof(double) * n);
    m->tn = t0;
    m->q = 1; m->L = 2; m->qwait = m->L; m->qprime = 1;
    m->etamax = ETAMX1;
    m->indx_acor = m->qmax;
    m->crate = 1.0;
    set_ewt(m, m->zn[0]);
    rhs(m, t0, m->zn[0], m->zn[1]);
    int status = 0;
    double h0 = 0.0;
    status = hin(m, tout, &h0);
    if (status == 0) {
        m->h = h0;
        m->hscale = h0; m->hprime = h0;
        for (int i = 0; i < n; ++i) m->zn[1][i] *= h0;
        long nstloc = 0;
        for (;;) {
            if (m->nst > 0) set_ewt(m, m->zn[0]);
            if (nstloc >= m->max_steps) { status = ORACLE_CV_TOO_MUCH_WORK; break; }
            double tolsf = UROUND * wrms(n, m->zn[0], m->ewt);
            if (tolsf > 1.0) { status = ORACLE_CV_TOO_MUCH_ACC; break; }
            int kflag = step(m);
            if (kflag != 0) { status = kflag; break; }
            nstloc++;
            if ((m->tn - tout) * m->h >= 0.0) {
                get_dky(m, tout, y);
                break;
            }
        }
        if (status != 0) memcpy(y, m->zn[0], sizeof(double) * n);
    }
    m->st.status = status;
    m->st.nst = (int)m->nst;
    m->st.qlast = m->q;
    m->st.hlast = m->h;
    if (stats) *stats = m->st;
    free(buf);
    free(piv);
    return status;
}

long oracle_bdf_batch(oracle_rhs_fn f, oracle_jac_fn J, int n, long ncells, const double* pres,
                      double pres_scalar, double* y, double t0, double tout,
                      const oracle_bdf_opts* opts, oracle_bdf_stats* stats, int nthreads) {
    long nfail = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(+ : nfail)
#endif
    for (long c = 0; c < ncells; ++c) {
        oracle_bdf_stats st;
        double P = pres ? pres[c] : pres_scalar;
        int s = oracle_bdf_solve(f, J, n, P, y + (size_t)c * n, t0, tout, opts, &st);
        if (stats) stats[c] = st;
        if (s != 0) nfail++;
    }
    (void)nthreads;
    return nfail;
}

long oracle_bdf_batch_mech(int mech, long ncells, const double* pres, double pres_scalar,
                           double* y, double t0, double tout, const oracle_bdf_opts* opts,
                           oracle_bdf_stats* stats, int nthreads) {
    oracle_rhs_fn f;
    oracle_jac_fn J;
    oracle_mech_fns(mech, 0, &f, &J);
    return oracle_bdf_batch(f, J, oracle_mech_nsp(mech), ncells, pres, pres_scalar, y, t0, tout,
                            opts, stats, nthreads);
}

long oracle_bdf_batch_mech_conv(int mech, long ncells, const double* pres, double pres_scalar,
                                double* y, double t0, double tout, const oracle_bdf_opts* opts,
                                oracle_bdf_stats* stats, int nthreads) {
    oracle_rhs_fn f;
    oracle_jac_fn J;
    oracle_mech_fns(mech, 1, &f, &J);
    const int n = oracle_mech_nsp(mech);
    double* rho = (double*)malloc((size_t)(ncells > 0 ? ncells : 1) * sizeof(double));
    if (!rho) return ncells;
    for (long c = 0; c < ncells; ++c)
        rho[c] = oracle_density(mech, pres ? pres[c] : pres_scalar, y + (size_t)c * n);
    const long nfail = oracle_bdf_batch(f, J, n, ncells, rho, 0.0, y, t0, tout, opts, stats, nthreads);
    free(rho);
    return nfail;
}
