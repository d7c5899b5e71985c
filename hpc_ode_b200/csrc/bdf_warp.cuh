// Warp-per-cell CVODE-semantics BDF.
//
// The per-cell algorithm of the reference's serial integrator
// (src/Integrators/CVodeIntegrator.cpp:98-155: CVODE BDF, dense direct linear
// solver, analytic Jacobian, CVodeSetMaxNumSteps(10000), CV_NORMAL to tout),
// run entirely on the device: one warp per cell, no host round trip per step.
// The reference's GPU path instead runs one CVODE instance over the whole
// batch with a shared step size and a global WRMS norm
// (src/Integrators/CVodeIntegratorGPU.cpp:59-108); this keeps the serial
// semantics (own h, q and error test per cell).
//
// Algorithm and constants follow CVODE's published description (Hindmarsh et
// al., ACM TOMS 31(3), 2005; CVODE user guide): Nordsieck history zn[0..q],
// fixed-leading-coefficient BDF coefficients, modified Newton on
// M = I - gamma*J (3 iterations max, CRDOWN 0.3, RDIV 2, tq[4] = 0.1/tq[2]),
// linear-solver setup on a 30 % gamma change / 20 steps / failure, Jacobian
// reuse (51 steps, bad-J rule 0.2), error test, eta/order selection with
// biases 6/6/10, growth caps 1e4 then 10, CVODE's initial-step heuristic,
// interpolation at tout.  The CPU oracle (oracle/bdf_oracle.c) is the same
// algorithm in scalar C; the GPU kernel is checked against it.
//
// Storage: the Nordsieck history and the method arrays (l, tq, tau) live in
// the warp's shared memory (compact rolled loops, few registers); the work
// vectors (ewt, acor, y, ftemp, ...) are lane registers (element i = lane +
// 32 s, internal order Y_0..Y_{N-2}, T).  Scalars are computed identically by
// all 32 lanes from identical warp-reduced values, so control flow is uniform
// across the warp; shared arrays are written by every lane with the same value.
// Every loop is bounded (max_steps, 10 convergence failures, 7 error-test
// failures, 3 Newton iterations), so a cell cannot spin.
#pragma once

#include "chem_warp.cuh"
#include "linalg_warp.cuh"

namespace b200 {

namespace cv {
constexpr int QMAX = 5;
constexpr double ETAMX1 = 10000.0, ETAMX2 = 10.0, ETAMX3 = 10.0, ETAMXF = 0.2, ETAMIN = 0.1,
                 ETACF = 0.25, ADDON = 1.0e-6, BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0,
                 THRESH = 1.5, CRDOWN = 0.3, RDIV = 2.0, DGMAX_LSETUP = 0.3, DGMAX_JBAD = 0.2,
                 NLSCOEF = 0.1, HLB_FACTOR = 100.0, HUB_FACTOR = 0.1, H_BIAS = 0.5,
                 UROUND = 2.220446049250313e-16;
constexpr int SMALL_NST = 10, MXNCF = 10, MXNEF = 7, MXNEF1 = 3, SMALL_NEF = 2, LONG_WAIT = 10,
              NLS_MAXCOR = 3, MSBP = 20, MSBJ = 51, MAX_HIN_ITERS = 4;
enum { FIRST_CALL = 0, PREV_CONV_FAIL = 1, PREV_ERR_FAIL = 2 };
enum { NO_FAILURES = 0, FAIL_BAD_J = 1, FAIL_OTHER = 2 };
enum { DO_ERROR_TEST = 2, PREDICT_AGAIN = 3, TRY_AGAIN = 5, CONV_RECVR = 901 };
enum { CV_SUCCESS = 0, CV_TOO_MUCH_WORK = -1, CV_TOO_MUCH_ACC = -2, CV_ERR_FAILURE = -3,
       CV_CONV_FAILURE = -4, CV_TOO_CLOSE = -27 };
}  // namespace cv

// Phases of the per-phase cycle profile.
enum { PH_RHS = 0, PH_JAC = 1, PH_LU = 2, PH_SOLVE = 3, PH_TOTAL = 4 };

// Per-warp shared memory.
template <class MT, class LinT>
struct WarpSmem {
    ChemSmem<MT> chem;
    double zn[cv::QMAX + 1][32 * MT::NS];   // Nordsieck history zn[j][i]
    double l[8], tq[8], tau[8];             // method coefficients (l[0..q], tq[1..5], tau[1..q+1])
    LinT A[MT::N * MT::LDA];                // Jacobian, then the LU factors of M = I - gamma J
    LinT dinv[MT::N];
    int perm[MT::N];
    long long prof[8];                      // per-phase clock64 totals when profiling
};

// Per-warp global scratch: saved Jacobian (CVODE keeps it to form new M
// without re-evaluating J) and the Jacobian's rate-derivative scratch.
template <class MT, class LinT>
struct WarpGlobal {
    LinT savedJ[MT::N * MT::N];
    JacScratch<MT> js;
};

struct CellCounters {
    int nst, nfe, nje, nsetups, nni, ncfn, netf;
};

template <class MT, class LinT>
struct WarpBdf {
    static constexpr int N = MT::N, NS = MT::NS;
    // problem
    double P, rtol, atol;
    int max_steps, qmax, refine, lane;
    WarpSmem<MT, LinT>* sm;
    WarpGlobal<MT, LinT>* wg;
    // work vectors (lane elements)
    double ewt[NS], acor[NS], tempv[NS], ftemp[NS], y[NS], delta[NS];
    // method scalars (identical on all lanes)
    double tn, h, hprime, hscale, eta, etamax, hu, saved_tq5;
    double gamma, gammap, gamrat, rl1, crate, acnrm, etaq, etaqm1, etaqp1;
    int q, qprime, qwait, L, indx_acor, jcur, convfail;
    int nst, nstlp, nstlj, nstloc;
    int lu_dirty;   // an LU was computed since the last save (step form)
    int profiling;  // accumulate per-phase clock64 into sm->prof
    CellCounters cnt;

    __device__ __forceinline__ WarpBdf(WarpSmem<MT, LinT>* sm_, WarpGlobal<MT, LinT>* wg_, int lane_)
        : lane(lane_), sm(sm_), wg(wg_) {}

    __device__ __forceinline__ bool valid(int s) const { return lane + 32 * s < N; }
    __device__ __forceinline__ double* zn(int j) const { return sm->zn[j] + lane; }

    __device__ __forceinline__ double wrms(const double (&x)[NS]) const {
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) { const double t = x[s] * ewt[s]; acc += t * t; }
        return sqrt(warp_sum(acc) / N);
    }
    __device__ __forceinline__ double wrms_zn(int j) const {
        const double* z = zn(j);
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) { const double t = z[32 * s] * ewt[s]; acc += t * t; }
        return sqrt(warp_sum(acc) / N);
    }
    __device__ __forceinline__ void set_ewt_zn0() {
        const double* z = zn(0);
#pragma unroll
        for (int s = 0; s < NS; ++s) ewt[s] = valid(s) ? 1.0 / (rtol * fabs(z[32 * s]) + atol) : 0.0;
    }
    __device__ __forceinline__ long long tick() const { return profiling ? clock64() : 0; }
    __device__ __forceinline__ void tock(int ph, long long t0) {
        if (profiling && lane == 0) sm->prof[ph] += clock64() - t0;
    }
    __device__ __forceinline__ void rhs(const double (&yy)[NS], double (&out)[NS]) {
        const long long t0 = tick();
        Vec<NS> a;
#pragma unroll
        for (int s = 0; s < NS; ++s) a.v[s] = yy[s];
        const Vec<NS> r = warp_rhs<MT>(P, a, &sm->chem, lane);
#pragma unroll
        for (int s = 0; s < NS; ++s) out[s] = r.v[s];
        cnt.nfe++;
        tock(PH_RHS, t0);
    }
    __device__ __forceinline__ void rhs_zn0(double (&out)[NS]) {
        double a[NS];
        const double* z = zn(0);
#pragma unroll
        for (int s = 0; s < NS; ++s) a[s] = z[32 * s];
        rhs(a, out);
    }
    __device__ __forceinline__ void lu_solve(double (&b)[NS]) {
        const long long t0 = tick();
        Vec<NS> a;
#pragma unroll
        for (int s = 0; s < NS; ++s) a.v[s] = b[s];
        const Vec<NS> r = warp_lu_solve<MT, LinT>(sm->A, sm->perm, sm->dinv, a, lane);
#pragma unroll
        for (int s = 0; s < NS; ++s) b[s] = r.v[s];
        tock(PH_SOLVE, t0);
    }

    // ----------------------------------------------------------- Nordsieck
    __device__ __forceinline__ void rescale() {
        double factor = eta;
#pragma unroll 1
        for (int j = 1; j <= q; ++j) {
            double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] *= factor;
            factor *= eta;
        }
        h = hscale * eta;
        hscale = h;
    }
    __device__ __forceinline__ void predict() {
        tn += h;
#pragma unroll 1
        for (int k = 1; k <= q; ++k)
#pragma unroll 1
            for (int j = q; j >= k; --j) {
                double* a = zn(j - 1);
                const double* b = zn(j);
#pragma unroll
                for (int s = 0; s < NS; ++s) a[32 * s] += b[32 * s];
            }
    }
    __device__ __forceinline__ void restore(double saved_t) {
        tn = saved_t;
#pragma unroll 1
        for (int k = 1; k <= q; ++k)
#pragma unroll 1
            for (int j = q; j >= k; --j) {
                double* a = zn(j - 1);
                const double* b = zn(j);
#pragma unroll
                for (int s = 0; s < NS; ++s) a[32 * s] -= b[32 * s];
            }
    }
    __device__ __forceinline__ void increase_bdf() {
        double* l = sm->l;
        const double* tau = sm->tau;
        for (int j = 0; j <= cv::QMAX; ++j) l[j] = 0.0;
        l[2] = 1.0;
        double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = hscale;
        for (int j = 1; j < q; ++j) {
            hsum += tau[j + 1];
            const double xi = hsum / hscale;
            prod *= xi;
            alpha0 -= 1.0 / (j + 1);
            alpha1 += 1.0 / xi;
            for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xiold + l[i - 1];
            xiold = xi;
        }
        const double A1 = (-alpha0 - alpha1) / prod;
        const double* acs = zn(indx_acor);
        double* zl = zn(L);
        double col[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) { col[s] = A1 * acs[32 * s]; zl[32 * s] = col[s]; }
        for (int j = 2; j <= q; ++j) {
            double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] += l[j] * col[s];
        }
    }
    __device__ __forceinline__ void decrease_bdf() {
        double* l = sm->l;
        const double* tau = sm->tau;
        for (int j = 0; j <= cv::QMAX; ++j) l[j] = 0.0;
        l[2] = 1.0;
        double hsum = 0.0;
        for (int j = 1; j <= q - 2; ++j) {
            hsum += tau[j];
            const double xi = hsum / hscale;
            for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xi + l[i - 1];
        }
        const double* zq = zn(q);
        for (int j = 2; j < q; ++j) {
            double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] += -l[j] * zq[32 * s];
        }
    }
    __device__ __forceinline__ void adjust_order(int dq) {
        if (q == 2 && dq != 1) return;
        if (dq == 1) increase_bdf();
        else if (dq == -1) decrease_bdf();
    }
    __device__ __forceinline__ void adjust_params() {
        if (qprime != q) {
            adjust_order(qprime - q);
            q = qprime;
            L = q + 1;
            qwait = L;
        }
        rescale();
    }

    // --------------------------------------------------------- coefficients
    __device__ __forceinline__ void set_coeffs() {
        double* l = sm->l;
        double* tq = sm->tq;
        const double* tau = sm->tau;
        l[0] = l[1] = 1.0;
        double xi_inv = 1.0, xistar_inv = 1.0;
        for (int j = 2; j <= cv::QMAX; ++j) l[j] = 0.0;
        double alpha0 = -1.0, alpha0_hat = -1.0, hsum = h;
        if (q > 1) {
            for (int j = 2; j < q; ++j) {
                hsum += tau[j - 1];
                xi_inv = h / hsum;
                alpha0 -= 1.0 / j;
                for (int i = j; i >= 1; --i) l[i] += l[i - 1] * xi_inv;
            }
            alpha0 -= 1.0 / q;
            xistar_inv = -l[1] - alpha0;
            hsum += tau[q - 1];
            xi_inv = h / hsum;
            alpha0_hat = -l[1] - xi_inv;
            for (int i = q; i >= 1; --i) l[i] += l[i - 1] * xistar_inv;
        }
        // error constants (CVODE's cvSetTqBDF)
        const double A1 = 1.0 - alpha0_hat + alpha0;
        const double A2 = 1.0 + q * A1;
        tq[2] = fabs(A1 / (alpha0 * A2));
        tq[5] = fabs(A2 * xistar_inv / (l[q] * xi_inv));
        if (qwait == 1) {
            if (q > 1) {
                const double C = xistar_inv / l[q];
                const double A3 = alpha0 + 1.0 / q;
                const double A4 = alpha0_hat + xi_inv;
                const double Cpinv = (1.0 - A4 + A3) / A3;
                tq[1] = fabs(C * Cpinv);
            } else {
                tq[1] = 1.0;
            }
            hsum += tau[q];
            xi_inv = h / hsum;
            const double A5 = alpha0 - 1.0 / (q + 1);
            const double A6 = alpha0_hat - xi_inv;
            const double Cppinv = (1.0 - A6 + A5) / A2;
            tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
        }
        tq[4] = cv::NLSCOEF / tq[2];
        rl1 = 1.0 / l[1];
        gamma = h * rl1;
        if (nst == 0) gammap = gamma;
        gamrat = (nst > 0) ? gamma / gammap : 1.0;
    }

    // -------------------------------------------------------------- Newton
    // residual: y = zn0 + ycor; ftemp = f(y); res = rl1*zn1 + ycor - gamma*ftemp
    __device__ __forceinline__ void nls_residual(const double (&ycor)[NS], double (&res)[NS]) {
        const double* z0 = zn(0);
#pragma unroll
        for (int s = 0; s < NS; ++s) y[s] = z0[32 * s] + ycor[s];
        rhs(y, ftemp);
        const double* z1 = zn(1);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            res[s] = rl1 * z1[32 * s] + ycor[s];
            res[s] = -gamma * ftemp[s] + res[s];
        }
    }
    // J reuse decision, M = I - gamma J, LU.  Returns nonzero if singular.
    __device__ __forceinline__ int ls_setup(int cf) {
        constexpr int LDA = MT::LDA;
        const double dgamma = fabs(gamma / gammap - 1.0);
        const bool jbad = (nst == 0) || (nst >= nstlj + cv::MSBJ) ||
                          ((cf == cv::FAIL_BAD_J) && (dgamma < cv::DGMAX_JBAD)) || (cf == cv::FAIL_OTHER);
        LinT* A = sm->A;
        LinT* J = wg->savedJ;
        if (!jbad) {
            jcur = 0;
            for (int i = 0; i < N; ++i)
                for (int j = lane; j < N; j += 32) A[i * LDA + j] = J[i * N + j];
        } else {
            cnt.nje++;
            nstlj = nst;
            jcur = 1;
            const long long tj = tick();
            Vec<NS> yy;
#pragma unroll
            for (int s = 0; s < NS; ++s) yy.v[s] = y[s];
            warp_jac<MT, LinT>(P, yy, A, &sm->chem, &wg->js, lane);
            tock(PH_JAC, tj);
            for (int i = 0; i < N; ++i)
                for (int j = lane; j < N; j += 32) J[i * N + j] = A[i * LDA + j];
        }
        __syncwarp();
        const LinT mg = (LinT)(-gamma);
        for (int i = 0; i < N; ++i)
            for (int j = lane; j < N; j += 32) {
                LinT v = mg * A[i * LDA + j];
                if (i == j) v += LinT(1);
                A[i * LDA + j] = v;
            }
        __syncwarp();
        lu_dirty = 1;
        const long long tl = tick();
        const int r = warp_lu<MT, LinT>(A, sm->perm, sm->dinv, lane);
        tock(PH_LU, tl);
        return r;
    }
    __device__ __forceinline__ int nls_lsetup(int jbad) {
        if (jbad) convfail = cv::FAIL_BAD_J;
        const int ret = ls_setup(convfail);
        cnt.nsetups++;
        gamrat = 1.0;
        gammap = gamma;
        crate = 1.0;
        nstlp = nst;
        return ret ? cv::CONV_RECVR : 0;
    }
    // r = b - (I - gammap J) x in FP64, J from the saved Jacobian.
    __device__ __forceinline__ void refine_residual(const double (&b)[NS], const double (&x)[NS],
                                                 double (&r)[NS]) {
#pragma unroll
        for (int s = 0; s < NS; ++s) r[s] = b[s] - x[s];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int i = lane + 32 * s;
            double acc = 0.0;
#pragma unroll 1
            for (int j = 0; j < N; ++j) {
                const double xj = __shfl_sync(kFull, x[j >> 5 < NS ? j >> 5 : 0], j & 31);
                if (i < N) acc += (double)wg->savedJ[i * N + j] * xj;
            }
            if (i < N) r[s] += gammap * acc;
        }
    }
    __device__ __forceinline__ void ls_solve(double (&b)[NS]) {
        if (refine && sizeof(LinT) < sizeof(double)) {
            double b0[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) b0[s] = b[s];
            lu_solve(b);
            double r[NS];
            refine_residual(b0, b, r);
            lu_solve(r);
#pragma unroll
            for (int s = 0; s < NS; ++s) b[s] += r[s];
        } else {
            lu_solve(b);
        }
        if (gamrat != 1.0) {
            const double sc = 2.0 / (1.0 + gamrat);
#pragma unroll
            for (int s = 0; s < NS; ++s) b[s] *= sc;
        }
    }
    __device__ __forceinline__ int nls_solve(int call_setup) {
        int jbad = 0, ret = 0;
#pragma unroll 1
        for (int attempt = 0; attempt < 4; ++attempt) {
            nls_residual(acor, delta);
            if (call_setup) {
                ret = nls_lsetup(jbad);
                if (ret) break;
            }
            double delp = 0.0;
            ret = 0;
#pragma unroll 1
            for (int m = 0;; ++m) {
                cnt.nni++;
#pragma unroll
                for (int s = 0; s < NS; ++s) delta[s] = -delta[s];
                ls_solve(delta);
#pragma unroll
                for (int s = 0; s < NS; ++s) acor[s] += delta[s];
                const double del = wrms(delta);
                if (m > 0) crate = fmax(cv::CRDOWN * crate, del / delp);
                const double dcon = del * fmin(1.0, crate) / sm->tq[4];
                if (dcon <= 1.0) {
                    acnrm = (m == 0) ? del : wrms(acor);
                    jcur = 0;
                    return 0;
                }
                if (m >= 1 && del > cv::RDIV * delp) { ret = cv::CONV_RECVR; break; }
                delp = del;
                if (m + 1 >= cv::NLS_MAXCOR) { ret = cv::CONV_RECVR; break; }
                nls_residual(acor, delta);
            }
            if (ret == cv::CONV_RECVR && !jcur) {
                call_setup = 1;
                jbad = 1;
#pragma unroll
                for (int s = 0; s < NS; ++s) acor[s] = 0.0;
                continue;
            }
            break;
        }
        return ret;
    }
    __device__ __forceinline__ int nls(int nflag) {
        convfail = ((nflag == cv::FIRST_CALL) || (nflag == cv::PREV_ERR_FAIL)) ? cv::NO_FAILURES : cv::FAIL_OTHER;
        const int call_setup = (nflag == cv::PREV_CONV_FAIL) || (nflag == cv::PREV_ERR_FAIL) || (nst == 0) ||
                               (nst >= nstlp + cv::MSBP) || (fabs(gamrat - 1.0) > cv::DGMAX_LSETUP);
#pragma unroll
        for (int s = 0; s < NS; ++s) acor[s] = 0.0;
        return nls_solve(call_setup);
    }
    __device__ __forceinline__ int handle_nflag(int& nflag, double saved_t, int& ncf) {
        if (nflag == 0) return cv::DO_ERROR_TEST;
        cnt.ncfn++;
        restore(saved_t);
        ncf++;
        etamax = 1.0;
        if (ncf == cv::MXNCF) return cv::CV_CONV_FAILURE;
        eta = cv::ETACF;
        nflag = cv::PREV_CONV_FAIL;
        rescale();
        return cv::PREDICT_AGAIN;
    }
    __device__ __forceinline__ int do_error_test(int& nflag, double saved_t, int& nef, double& dsm) {
        dsm = acnrm * sm->tq[2];
        if (dsm <= 1.0) return 0;
        nef++;
        cnt.netf++;
        nflag = cv::PREV_ERR_FAIL;
        restore(saved_t);
        if (nef == cv::MXNEF) return cv::CV_ERR_FAILURE;
        etamax = 1.0;
        if (nef <= cv::MXNEF1) {
            eta = 1.0 / (pow(cv::BIAS2 * dsm, 1.0 / L) + cv::ADDON);
            eta = fmax(cv::ETAMIN, eta);
            if (nef >= cv::SMALL_NEF) eta = fmin(eta, cv::ETAMXF);
            rescale();
            return cv::TRY_AGAIN;
        }
        if (q > 1) {
            eta = cv::ETAMIN;
            adjust_order(-1);
            L = q;
            q--;
            qwait = L;
            rescale();
            return cv::TRY_AGAIN;
        }
        eta = cv::ETAMIN;
        h *= eta;
        hscale = h;
        qwait = cv::LONG_WAIT;
        rhs_zn0(tempv);
        double* z1 = zn(1);
#pragma unroll
        for (int s = 0; s < NS; ++s) z1[32 * s] = h * tempv[s];
        return cv::TRY_AGAIN;
    }
    __device__ __forceinline__ void complete_step() {
        double* tau = sm->tau;
        const double* l = sm->l;
        nst++;
        hu = h;
        for (int i = q; i >= 2; --i) tau[i] = tau[i - 1];
        if (q == 1 && nst > 1) tau[2] = tau[1];
        tau[1] = h;
#pragma unroll 1
        for (int j = 0; j <= q; ++j) {
            double* z = zn(j);
            const double lj = l[j];
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] += lj * acor[s];
        }
        qwait--;
        if (qwait == 1 && q != qmax) {
            double* zm = zn(qmax);
#pragma unroll
            for (int s = 0; s < NS; ++s) zm[32 * s] = acor[s];
            saved_tq5 = sm->tq[5];
            indx_acor = qmax;
        }
    }
    __device__ __forceinline__ void set_eta() {
        if (eta < cv::THRESH) {
            eta = 1.0;
            hprime = h;
        } else {
            eta = fmin(eta, etamax);
            hprime = h * eta;
        }
    }
    __device__ __forceinline__ void prepare_next_step(double dsm) {
        if (etamax == 1.0) {
            if (qwait < 2) qwait = 2;
            qprime = q;
            hprime = h;
            eta = 1.0;
            return;
        }
        etaq = 1.0 / (pow(cv::BIAS2 * dsm, 1.0 / L) + cv::ADDON);
        if (qwait != 0) {
            eta = etaq;
            qprime = q;
            set_eta();
            return;
        }
        qwait = 2;
        // eta at order q-1
        etaqm1 = 0.0;
        if (q > 1) {
            const double ddn = wrms_zn(q) * sm->tq[1];
            etaqm1 = 1.0 / (pow(cv::BIAS1 * ddn, 1.0 / q) + cv::ADDON);
        }
        // eta at order q+1
        etaqp1 = 0.0;
        if (q != qmax && saved_tq5 != 0.0) {
            const double cquot = (sm->tq[5] / saved_tq5) * pow(h / sm->tau[2], (double)L);
            const double* zm = zn(qmax);
#pragma unroll
            for (int s = 0; s < NS; ++s) tempv[s] = acor[s] - cquot * zm[32 * s];
            const double dup = wrms(tempv) * sm->tq[3];
            etaqp1 = 1.0 / (pow(cv::BIAS3 * dup, 1.0 / (L + 1)) + cv::ADDON);
        }
        // choose
        const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
        if (etam < cv::THRESH) {
            eta = 1.0;
            qprime = q;
        } else if (etam == etaqm1) {
            eta = etaqm1;
            qprime = q - 1;
        } else if (etam == etaq) {
            eta = etaq;
            qprime = q;
        } else {
            eta = etaqp1;
            qprime = q + 1;
            double* zm = zn(qmax);
#pragma unroll
            for (int s = 0; s < NS; ++s) zm[32 * s] = acor[s];
        }
        set_eta();
    }
    // One internal step.  Returns 0 or a negative CVODE code.
    __device__ __forceinline__ int step() {
        const double saved_t = tn;
        int ncf = 0, nef = 0, nflag = cv::FIRST_CALL;
        double dsm = 0.0;
        if (nst > 0 && hprime != h) adjust_params();
#pragma unroll 1
        for (int guard = 0; guard < 64; ++guard) {
            predict();
            set_coeffs();
            nflag = nls(nflag);
            const int kflag = handle_nflag(nflag, saved_t, ncf);
            if (kflag == cv::PREDICT_AGAIN) continue;
            if (kflag != cv::DO_ERROR_TEST) return kflag;
            const int eflag = do_error_test(nflag, saved_t, nef, dsm);
            if (eflag == cv::TRY_AGAIN) continue;
            if (eflag != 0) return eflag;
            complete_step();
            prepare_next_step(dsm);
            etamax = (nst <= cv::SMALL_NST) ? cv::ETAMX2 : cv::ETAMX3;
            const double t2 = sm->tq[2];
#pragma unroll
            for (int s = 0; s < NS; ++s) acor[s] *= t2;
            return 0;
        }
        return cv::CV_CONV_FAILURE;   // unreachable: ncf < 10 and nef < 7 bound the attempts
    }

    // ------------------------------------------------------------ initial h
    __device__ __forceinline__ int hin(double tout, double& h0) {
        const double tdiff = tout - tn;
        if (tdiff == 0.0) return cv::CV_TOO_CLOSE;
        const int sign = (tdiff > 0.0) ? 1 : -1;
        const double tdist = fabs(tdiff);
        const double tround = cv::UROUND * fmax(fabs(tn), fabs(tout));
        if (tdist < 2.0 * tround) return cv::CV_TOO_CLOSE;
        const double hlb = cv::HLB_FACTOR * tround;
        // upper bound from |y0| / |y0'| (CVODE's cvUpperBoundH0)
        const double* z0 = zn(0);
        const double* z1 = zn(1);
        double r = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s)
            if (valid(s)) {
                const double den = cv::HUB_FACTOR * fabs(z0[32 * s]) + 1.0 / ewt[s];
                r = fmax(r, fabs(z1[32 * s]) / den);
            }
        const double hub_inv = warp_max(r);
        double hub = cv::HUB_FACTOR * tdist;
        if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
        double hg = sqrt(hlb * hub);
        if (hub < hlb) { h0 = sign * hg; return 0; }
        double hnew = hg;
#pragma unroll 1
        for (int count1 = 1; count1 <= cv::MAX_HIN_ITERS; ++count1) {
            // ||y''|| estimate from one RHS evaluation (cvYddNorm)
            const double hgs = hg * sign;
#pragma unroll
            for (int s = 0; s < NS; ++s) y[s] = hgs * z1[32 * s] + z0[32 * s];
            rhs(y, tempv);
            const double ih = 1.0 / hgs;
#pragma unroll
            for (int s = 0; s < NS; ++s) tempv[s] = (tempv[s] - z1[32 * s]) * ih;
            const double yddnrm = wrms(tempv);
            hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
            if (count1 == cv::MAX_HIN_ITERS) break;
            const double hrat = hnew / hg;
            if (hrat > 0.5 && hrat < 2.0) break;
            if (count1 > 1 && hrat > 2.0) { hnew = hg; break; }
            hg = hnew;
        }
        double hh = cv::H_BIAS * hnew;
        if (hh < hlb) hh = hlb;
        if (hh > hub) hh = hub;
        h0 = sign * hh;
        return 0;
    }

    // ---------------------------------------------------------------- driver
    // Set up y0 at t0 toward tout: ewt, f(y0), initial step (CVode's first-call
    // path).  Returns 0 or a CVODE code.
    __device__ __forceinline__ int begin(const double (&y0)[NS], double t0, double tout) {
        cnt = CellCounters{0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j <= cv::QMAX; ++j) {
            double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] = (j == 0 && valid(s)) ? y0[s] : 0.0;
        }
        for (int j = 0; j < 8; ++j) sm->l[j] = sm->tq[j] = sm->tau[j] = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) acor[s] = tempv[s] = ftemp[s] = y[s] = delta[s] = 0.0;
        tn = t0;
        q = 1; L = 2; qwait = L; qprime = 1;
        etamax = cv::ETAMX1;
        indx_acor = qmax;
        crate = 1.0;
        h = hprime = hscale = eta = hu = saved_tq5 = 0.0;
        gamma = gammap = gamrat = rl1 = acnrm = etaq = etaqm1 = etaqp1 = 0.0;
        jcur = 0; convfail = 0; nst = nstlp = nstlj = 0; nstloc = 0;
        set_ewt_zn0();
        double f0[NS];
        rhs_zn0(f0);
        double* z1 = zn(1);
#pragma unroll
        for (int s = 0; s < NS; ++s) z1[32 * s] = valid(s) ? f0[s] : 0.0;
        double h0 = 0.0;
        const int status = hin(tout, h0);
        if (status == 0) {
            h = h0;
            hscale = h0;
            hprime = h0;
#pragma unroll
            for (int s = 0; s < NS; ++s) z1[32 * s] *= h0;
        }
        return status;
    }
    // Take up to max_new internal steps toward tout.  Sets done when tout is
    // reached or a step failed; returns 0 or a negative CVODE code.
    __device__ __forceinline__ int advance(double tout, int max_new, bool& done) {
        done = false;
#pragma unroll 1
        for (int k = 0; k < max_new; ++k) {
            if (nst > 0) set_ewt_zn0();
            if (nstloc >= max_steps) { done = true; return cv::CV_TOO_MUCH_WORK; }
            const double tolsf = cv::UROUND * wrms_zn(0);
            if (tolsf > 1.0) { done = true; return cv::CV_TOO_MUCH_ACC; }
            const int kflag = step();
            if (kflag != 0) { done = true; return kflag; }
            nstloc++;
            if ((tn - tout) * h >= 0.0) { done = true; return 0; }
        }
        return 0;
    }
    // Output: y(tout) by interpolation on success (CVodeGetDky), else the last
    // accepted state.
    __device__ __forceinline__ void finish(int status, double tout, double (&yout)[NS]) {
        if (status == 0) {
            const double s_ = (tout - tn) / h;
            const double* zq = zn(q);
#pragma unroll
            for (int s = 0; s < NS; ++s) yout[s] = zq[32 * s];
#pragma unroll 1
            for (int j = q - 1; j >= 0; --j) {
                const double* z = zn(j);
#pragma unroll
                for (int s = 0; s < NS; ++s) yout[s] = z[32 * s] + s_ * yout[s];
            }
        } else {
            const double* z0 = zn(0);
#pragma unroll
            for (int s = 0; s < NS; ++s) yout[s] = z0[32 * s];
        }
        cnt.nst = nst;
    }

    // ------------------------------------------- state in HBM (step form)
    // Per-cell record of the one-launch-per-step form: method scalars and
    // arrays, the Nordsieck history and the Newton-matrix factors (the saved
    // Jacobian lives in the cell's WarpGlobal).
    struct Scalars {
        double l[8], tq[8], tau[8];
        double tn, h, hprime, hscale, eta, etamax, hu, saved_tq5, gamma, gammap, gamrat, rl1,
            crate, acnrm, etaq, etaqm1, etaqp1, P;
        int q, qprime, qwait, L, indx_acor, jcur, convfail, nst, nstlp, nstlj, nstloc;
        int status, phase, cnt[7];
    };
    static constexpr size_t kScalarBytes = (sizeof(Scalars) + 255) & ~size_t(255);
    static constexpr size_t kZnBytes = ((cv::QMAX + 1) * N * sizeof(double) + 255) & ~size_t(255);
    static constexpr size_t kLuBytes =
        ((N * MT::LDA + N) * sizeof(LinT) + N * sizeof(int) + 255) & ~size_t(255);
    static constexpr size_t kRecordBytes = kScalarBytes + kZnBytes + kLuBytes;

    __device__ __forceinline__ void save(unsigned char* rec, int status, int phase, bool lu_dirty_) const {
        Scalars* S = reinterpret_cast<Scalars*>(rec);
        if (lane < 8) { S->l[lane] = sm->l[lane]; S->tq[lane] = sm->tq[lane]; S->tau[lane] = sm->tau[lane]; }
        if (lane == 0) {
            S->tn = tn; S->h = h; S->hprime = hprime; S->hscale = hscale; S->eta = eta;
            S->etamax = etamax; S->hu = hu; S->saved_tq5 = saved_tq5; S->gamma = gamma;
            S->gammap = gammap; S->gamrat = gamrat; S->rl1 = rl1; S->crate = crate; S->acnrm = acnrm;
            S->etaq = etaq; S->etaqm1 = etaqm1; S->etaqp1 = etaqp1; S->P = P;
            S->q = q; S->qprime = qprime; S->qwait = qwait; S->L = L; S->indx_acor = indx_acor;
            S->jcur = jcur; S->convfail = convfail; S->nst = nst; S->nstlp = nstlp; S->nstlj = nstlj;
            S->nstloc = nstloc; S->status = status; S->phase = phase;
            S->cnt[0] = cnt.nst; S->cnt[1] = cnt.nfe; S->cnt[2] = cnt.nje; S->cnt[3] = cnt.nsetups;
            S->cnt[4] = cnt.nni; S->cnt[5] = cnt.ncfn; S->cnt[6] = cnt.netf;
        }
        double* Z = reinterpret_cast<double*>(rec + kScalarBytes);
        for (int j = 0; j <= cv::QMAX; ++j) {
            const double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s)
                if (valid(s)) Z[j * N + lane + 32 * s] = z[32 * s];
        }
        if (lu_dirty_) {
            LinT* Ag = reinterpret_cast<LinT*>(rec + kScalarBytes + kZnBytes);
            for (int e = lane; e < N * MT::LDA; e += 32) Ag[e] = sm->A[e];
            for (int e = lane; e < N; e += 32) Ag[N * MT::LDA + e] = sm->dinv[e];
            int* pg = reinterpret_cast<int*>(Ag + N * MT::LDA + N);
            for (int e = lane; e < N; e += 32) pg[e] = sm->perm[e];
        }
    }
    __device__ __forceinline__ void load(const unsigned char* rec, int& status, int& phase) {
        const Scalars* S = reinterpret_cast<const Scalars*>(rec);
        if (lane < 8) { sm->l[lane] = S->l[lane]; sm->tq[lane] = S->tq[lane]; sm->tau[lane] = S->tau[lane]; }
        tn = S->tn; h = S->h; hprime = S->hprime; hscale = S->hscale; eta = S->eta;
        etamax = S->etamax; hu = S->hu; saved_tq5 = S->saved_tq5; gamma = S->gamma;
        gammap = S->gammap; gamrat = S->gamrat; rl1 = S->rl1; crate = S->crate; acnrm = S->acnrm;
        etaq = S->etaq; etaqm1 = S->etaqm1; etaqp1 = S->etaqp1; P = S->P;
        q = S->q; qprime = S->qprime; qwait = S->qwait; L = S->L; indx_acor = S->indx_acor;
        jcur = S->jcur; convfail = S->convfail; nst = S->nst; nstlp = S->nstlp; nstlj = S->nstlj;
        nstloc = S->nstloc; status = S->status; phase = S->phase;
        cnt.nst = S->cnt[0]; cnt.nfe = S->cnt[1]; cnt.nje = S->cnt[2]; cnt.nsetups = S->cnt[3];
        cnt.nni = S->cnt[4]; cnt.ncfn = S->cnt[5]; cnt.netf = S->cnt[6];
        const double* Z = reinterpret_cast<const double*>(rec + kScalarBytes);
        for (int j = 0; j <= cv::QMAX; ++j) {
            double* z = zn(j);
#pragma unroll
            for (int s = 0; s < NS; ++s) z[32 * s] = valid(s) ? Z[j * N + lane + 32 * s] : 0.0;
        }
        const LinT* Ag = reinterpret_cast<const LinT*>(rec + kScalarBytes + kZnBytes);
        for (int e = lane; e < N * MT::LDA; e += 32) sm->A[e] = Ag[e];
        for (int e = lane; e < N; e += 32) sm->dinv[e] = Ag[N * MT::LDA + e];
        const int* pg = reinterpret_cast<const int*>(Ag + N * MT::LDA + N);
        for (int e = lane; e < N; e += 32) sm->perm[e] = pg[e];
#pragma unroll
        for (int s = 0; s < NS; ++s) acor[s] = tempv[s] = ftemp[s] = y[s] = delta[s] = 0.0;
        __syncwarp();
    }
};

}  // namespace b200
