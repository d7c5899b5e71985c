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
// Layout for a small instruction footprint: the method state (scalars, l, tq,
// tau, counters) and the Nordsieck history live in the warp's shared memory;
// every lane computes the same scalar values and writes them (identical
// values, so the shared words are consistent).  Work vectors (ewt, acor, y,
// ftemp, delta) are lane registers (element i = lane + G s; internal order
// Y_0..Y_{N-2}, T).  Only the Newton loop is inlined; step-size/order
// selection, coefficient updates, the linear-solver setup, the initial step and
// the HBM record I/O are single out-of-line copies addressed by a shared-memory
// offset, so the kernel's hot code stays inside the instruction cache.
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
       CV_CONV_FAILURE = -4, CV_ILL_INPUT = -22, CV_TOO_CLOSE = -27 };
}  // namespace cv

// Phases of the per-phase cycle profile.
enum { PH_RHS = 0, PH_JAC = 1, PH_LU = 2, PH_SOLVE = 3, PH_TOTAL = 4 };
enum { C_NST = 0, C_NFE, C_NJE, C_NSETUPS, C_NNI, C_NCFN, C_NETF };

// Method state of one cell (CVODE's cv_mem scalars), in shared memory.
struct BdfState {
    double l[8], tq[8], tau[8];
    double tn, h, hprime, hscale, eta, etamax, hu, saved_tq5;
    double gamma, gammap, gamrat, rl1, crate, acnrm, etaq, etaqm1, etaqp1;
    double P, rtol, atol;
    int q, qprime, qwait, L, indx_acor, jcur, convfail;
    int nst, nstlp, nstlj, nstloc, max_steps, qmax, refine, lu_dirty, profiling;
    int cnt[7];
    long long* prof;     // per-phase clock64 totals when profiling (the warp's WarpGlobal::prof)
};

// Per-warp shared memory.
template <class MT, class LinT>
struct WarpSmem {
    ChemSmem<MT> chem;
    double zn[cv::QMAX + 1][MT::G * MT::NS];   // Nordsieck history zn[j][i]
    BdfState st;
    LinT A[MT::N * MT::LDA];                // Jacobian, then the LU factors of M = I - gamma J
                                            // (diagonal: 1 / U_kk)
    unsigned char perm[MT::N];              // row permutation of the factors
};

// Per-warp global scratch: saved Jacobian (CVODE keeps it to form new M
// without re-evaluating J) and the Jacobian's rate-derivative scratch.
template <class MT, class LinT>
struct WarpGlobal {
    // the saved Jacobian N x N; while a new Jacobian is evaluated (before it
    // is saved here) the same space holds its per-slot derivative pieces
    // [kJacPieces][NSLOT], so it is sized for the larger of the two
    static constexpr int kSaved = (MT::N * MT::N > kJacPieces * MT::NSLOT) ? MT::N * MT::N : kJacPieces * MT::NSLOT;
    LinT savedJ[kSaved];
    JacScratch<MT> js;
    long long prof[8];   // per-phase clock64 totals when profiling
};

template <class MT, class LinT>
__device__ __forceinline__ WarpSmem<MT, LinT>* wsm(unsigned off) {
    return smem_at<WarpSmem<MT, LinT>>(off);
}

template <int G>
__device__ __forceinline__ bool valid_el(int lane, int s, int N) { return lane + G * s < N; }

// sqrt(sum over the cell's lanes of acc / n): the tail of every WRMS norm, out of line.
template <int G>
__device__ __noinline__ double wrms_reduce(double acc, int n) { return sqrt(group_sum<G>(acc) / n); }

template <int NS, int G>
__device__ __forceinline__ double wrms_v(const double (&x)[NS], const double (&w)[NS], int N) {
    double acc = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) { const double t = x[s] * w[s]; acc += t * t; }
    return wrms_reduce<G>(acc, N);
}

template <class MT, class LinT>
__device__ __forceinline__ double wrms_zn(const WarpSmem<MT, LinT>* w, int j, const double (&ewt)[MT::NS], int lane) {
    double acc = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) { const double t = w->zn[j][lane + MT::G * s] * ewt[s]; acc += t * t; }
    return wrms_reduce<MT::G>(acc, MT::N);
}

__device__ __forceinline__ long long ph_tick(const BdfState& S) { return S.profiling ? clock64() : 0; }
__device__ __forceinline__ void ph_tock(BdfState& S, int ph, long long t0, int lane) {
    if (S.profiling && lane == 0) S.prof[ph] += clock64() - t0;
}

// f(y) for the warp's cell (counted as one RHS evaluation).
template <class MT, class LinT>
__device__ __forceinline__ void bdf_rhs(unsigned off, const double (&y)[MT::NS], double (&out)[MT::NS], int lane) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    const long long t0 = ph_tick(w->st);
    Vec<MT::NS> a;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) a.v[s] = y[s];
    const Vec<MT::NS> r = warp_rhs<MT>(w->st.P, a, smem_off(&w->chem), lane);
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) out[s] = r.v[s];
    w->st.cnt[C_NFE]++;
    ph_tock(w->st, PH_RHS, t0, lane);
}

// ---------------------------------------------------------------- Nordsieck
template <class MT, class LinT>
__device__ __forceinline__ void bdf_rescale(unsigned off, int lane) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    const double eta = S.eta;
    double factor = eta;
    const int q = S.q;
#pragma unroll 1
    for (int j = 1; j <= q; ++j) {
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) w->zn[j][lane + MT::G * s] *= factor;
        factor *= eta;
    }
    S.h = S.hscale * eta;
    S.hscale = S.h;
}

// zn <- Pascal-triangle prediction (sign = +1) or its inverse (sign = -1).
template <class MT, class LinT>
__device__ __forceinline__ void bdf_pascal(unsigned off, int lane, bool forward) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    const int q = w->st.q;
#pragma unroll 1
    for (int k = 1; k <= q; ++k)
#pragma unroll 1
        for (int j = q; j >= k; --j)
#pragma unroll
            for (int s = 0; s < MT::NS; ++s) {
                const int i = lane + MT::G * s;
                w->zn[j - 1][i] = forward ? w->zn[j - 1][i] + w->zn[j][i] : w->zn[j - 1][i] - w->zn[j][i];
            }
}

// Order change by +-1 of the Nordsieck array (CVODE's cvIncreaseBDF /
// cvDecreaseBDF).  Out of line: order changes are rare.
template <class MT, class LinT>
__device__ __noinline__ void bdf_adjust_order(unsigned off, int dq, int lane) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    const int q = S.q;
    if (q == 2 && dq != 1) return;
    double* l = S.l;
    #pragma unroll 1
    for (int j = 0; j <= cv::QMAX; ++j) l[j] = 0.0;
    l[2] = 1.0;
    if (dq == 1) {
        double alpha1 = 1.0, prod = 1.0, xiold = 1.0, alpha0 = -1.0, hsum = S.hscale;
        #pragma unroll 1
        for (int j = 1; j < q; ++j) {
            hsum += S.tau[j + 1];
            const double xi = ode_div(hsum, S.hscale);
            prod *= xi;
            alpha0 -= ode_div(1.0, (double)(j + 1));
            alpha1 += ode_div(1.0, xi);
            #pragma unroll 1
            for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xiold + l[i - 1];
            xiold = xi;
        }
        const double A1 = ode_div(-alpha0 - alpha1, prod);
        const int L = S.L, ia = S.indx_acor;
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) {
            const int i = lane + MT::G * s;
            const double col = A1 * w->zn[ia][i];
            w->zn[L][i] = col;
            #pragma unroll 1
            for (int j = 2; j <= q; ++j) w->zn[j][i] += l[j] * col;
        }
    } else if (dq == -1) {
        double hsum = 0.0;
        #pragma unroll 1
        for (int j = 1; j <= q - 2; ++j) {
            hsum += S.tau[j];
            const double xi = ode_div(hsum, S.hscale);
            #pragma unroll 1
            for (int i = j + 2; i >= 2; --i) l[i] = l[i] * xi + l[i - 1];
        }
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) {
            const int i = lane + MT::G * s;
            const double zq = w->zn[q][i];
            #pragma unroll 1
            for (int j = 2; j < q; ++j) w->zn[j][i] += -l[j] * zq;
        }
    }
}

// BDF coefficients l[0..q], error constants tq[1..5], gamma (CVODE's cvSet,
// cvSetBDF, cvSetTqBDF).
template <class MT, class LinT>
__device__ __noinline__ void bdf_set_coeffs(unsigned off) {
    BdfState& S = wsm<MT, LinT>(off)->st;
    double* l = S.l;
    double* tq = S.tq;
    const double* tau = S.tau;
    const int q = S.q;
    const double h = S.h;
    l[0] = l[1] = 1.0;
    double xi_inv = 1.0, xistar_inv = 1.0;
    #pragma unroll 1
    for (int j = 2; j <= cv::QMAX; ++j) l[j] = 0.0;
    double alpha0 = -1.0, alpha0_hat = -1.0, hsum = h;
    if (q > 1) {
        #pragma unroll 1
        for (int j = 2; j < q; ++j) {
            hsum += tau[j - 1];
            xi_inv = ode_div(h, hsum);
            alpha0 -= ode_div(1.0, (double)j);
            #pragma unroll 1
            for (int i = j; i >= 1; --i) l[i] += l[i - 1] * xi_inv;
        }
        alpha0 -= ode_div(1.0, (double)q);
        xistar_inv = -l[1] - alpha0;
        hsum += tau[q - 1];
        xi_inv = ode_div(h, hsum);
        alpha0_hat = -l[1] - xi_inv;
        #pragma unroll 1
        for (int i = q; i >= 1; --i) l[i] += l[i - 1] * xistar_inv;
    }
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    tq[2] = fabs(ode_div(A1, alpha0 * A2));
    tq[5] = fabs(ode_div(A2 * xistar_inv, l[q] * xi_inv));
    if (S.qwait == 1) {
        if (q > 1) {
            const double C = ode_div(xistar_inv, l[q]);
            const double A3 = alpha0 + ode_div(1.0, (double)q);
            const double A4 = alpha0_hat + xi_inv;
            const double Cpinv = ode_div(1.0 - A4 + A3, A3);
            tq[1] = fabs(C * Cpinv);
        } else {
            tq[1] = 1.0;
        }
        hsum += tau[q];
        xi_inv = ode_div(h, hsum);
        const double A5 = alpha0 - ode_div(1.0, (double)(q + 1));
        const double A6 = alpha0_hat - xi_inv;
        const double Cppinv = ode_div(1.0 - A6 + A5, A2);
        tq[3] = fabs(ode_div(Cppinv, xi_inv * (q + 2) * A5));
    }
    tq[4] = ode_div(cv::NLSCOEF, tq[2]);
    S.rl1 = ode_div(1.0, l[1]);
    S.gamma = h * S.rl1;
    if (S.nst == 0) S.gammap = S.gamma;
    S.gamrat = (S.nst > 0) ? ode_div(S.gamma, S.gammap) : 1.0;
}

// Linear-solver setup (CVODE's cvNlsLSetup + cvLsSetup): Jacobian reuse
// decision, M = I - gamma J, LU.  Returns nonzero if M is singular.
template <class MT, class LinT>
__device__ __noinline__ int bdf_ls_setup(unsigned off, const Vec<MT::NS> yv, WarpGlobal<MT, LinT>* wg, int jbad_in,
                                         int lane) {
    constexpr int N = MT::N, LDA = MT::LDA;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    if (jbad_in) S.convfail = cv::FAIL_BAD_J;
    const int cf = S.convfail;
    const double dgamma = fabs(ode_div(S.gamma, S.gammap) - 1.0);
    const bool jbad = (S.nst == 0) || (S.nst >= S.nstlj + cv::MSBJ) ||
                      ((cf == cv::FAIL_BAD_J) && (dgamma < cv::DGMAX_JBAD)) || (cf == cv::FAIL_OTHER);
    LinT* A = w->A;
    LinT* J = wg->savedJ;
    // M = I - gamma J, fused with the copy from (or to) the saved Jacobian in
    // global memory (mostly L2 resident): rows go in batches whose loads are all
    // issued before any store, so their latencies overlap instead of adding up
    // element by element.  Lane j owns columns j, j + G, ...: every element is
    // read and written by the same lane.
    constexpr int kB = (MT::NS <= 2) ? 8 : ((16 / MT::NS) > 1 ? 16 / MT::NS : 1);
    const LinT mg = (LinT)(-S.gamma);
    const bool from_saved = !jbad;
    if (from_saved) {
        S.jcur = 0;
    } else {
        S.cnt[C_NJE]++;
        S.nstlj = S.nst;
        S.jcur = 1;
        const long long tj = ph_tick(S);
        warp_jac<MT, LinT>(S.P, yv, smem_off(A), smem_off(&w->chem), &wg->js, wg->savedJ, lane);
        ph_tock(S, PH_JAC, tj, lane);
    }
#pragma unroll 1
    for (int i0 = 0; i0 < N; i0 += kB) {
        LinT v[kB][MT::NS];
#pragma unroll
        for (int r = 0; r < kB; ++r)
#pragma unroll
            for (int s = 0; s < MT::NS; ++s) {
                const int i = i0 + r, j = lane + MT::G * s;
                v[r][s] = (i < N && j < N) ? (from_saved ? J[i * N + j] : A[i * LDA + j]) : LinT(0);
            }
#pragma unroll
        for (int r = 0; r < kB; ++r)
#pragma unroll
            for (int s = 0; s < MT::NS; ++s) {
                const int i = i0 + r, j = lane + MT::G * s;
                if (i < N && j < N) {
                    if (!from_saved) J[i * N + j] = v[r][s];
                    LinT x = mg * v[r][s];
                    if (i == j) x += LinT(1);
                    A[i * LDA + j] = x;
                }
            }
    }
    __syncwarp(gmask<MT::G>());
    S.lu_dirty = 1;
    const long long tl = ph_tick(S);
    const int r = warp_lu<MT, LinT>(smem_off(A), smem_off(w->perm), lane);
    ph_tock(S, PH_LU, tl, lane);
    S.cnt[C_NSETUPS]++;
    S.gamrat = 1.0;
    S.gammap = S.gamma;
    S.crate = 1.0;
    S.nstlp = S.nst;
    return r;
}

// Newton correction solve: M delta = b, then CVODE's 2/(1+gamrat) scaling;
// optional FP64 refinement sweep against the saved Jacobian.
template <class MT, class LinT>
__device__ __forceinline__ void bdf_solve(unsigned off, double (&b)[MT::NS], const WarpGlobal<MT, LinT>* wg,
                                          int lane) {
    constexpr int N = MT::N, NS = MT::NS;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    const long long t0 = ph_tick(S);
    Vec<NS> a;
#pragma unroll
    for (int s = 0; s < NS; ++s) a.v[s] = b[s];
    Vec<NS> x = warp_lu_solve<MT, LinT>(smem_off(w->A), smem_off(w->perm), a, lane);
    if (S.refine && sizeof(LinT) < sizeof(double)) {
        // r = b - (I - gammap J) x in FP64; x += M^{-1} r
        Vec<NS> r;
#pragma unroll
        for (int s = 0; s < NS; ++s) r.v[s] = a.v[s] - x.v[s];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int i = lane + MT::G * s;
            double acc = 0.0;
#pragma unroll 1
            for (int j = 0; j < N; ++j) {
                const double xj = group_shfl<MT::G>(pick<NS>(x.v, j / MT::G), j % MT::G);
                if (i < N) acc += (double)wg->savedJ[i * N + j] * xj;
            }
            if (i < N) r.v[s] += S.gammap * acc;
        }
        const Vec<NS> d = warp_lu_solve<MT, LinT>(smem_off(w->A), smem_off(w->perm), r, lane);
#pragma unroll
        for (int s = 0; s < NS; ++s) x.v[s] += d.v[s];
    }
    const double gamrat = S.gamrat;
    const double sc = (gamrat != 1.0) ? ode_div(2.0, 1.0 + gamrat) : 1.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) b[s] = (gamrat != 1.0) ? x.v[s] * sc : x.v[s];
    ph_tock(S, PH_SOLVE, t0, lane);
}

// Step-size / order selection after an accepted step (CVODE's
// cvPrepareNextStep, cvComputeEtaqm1/qp1, cvChooseEta, cvSetEta).
template <class MT, class LinT>
__device__ __noinline__ void bdf_prepare_next_step(unsigned off, double dsm, const Vec<MT::NS> acv,
                                                   const Vec<MT::NS> ewv, int lane) {
    constexpr int NS = MT::NS;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    const int q = S.q, L = S.L;
    if (S.etamax == 1.0) {
        if (S.qwait < 2) S.qwait = 2;
        S.qprime = q;
        S.hprime = S.h;
        S.eta = 1.0;
        return;
    }
    S.etaq = ode_div(1.0, ode_pow(cv::BIAS2 * dsm, ode_div(1.0, (double)L)) + cv::ADDON);
    double eta;
    int qprime = q;
    if (S.qwait != 0) {
        eta = S.etaq;
    } else {
        S.qwait = 2;
        double etaqm1 = 0.0, etaqp1 = 0.0;
        if (q > 1) {
            const double ddn = wrms_zn<MT, LinT>(w, q, ewv.v, lane) * S.tq[1];
            etaqm1 = ode_div(1.0, ode_pow(cv::BIAS1 * ddn, ode_div(1.0, (double)q)) + cv::ADDON);
        }
        if (q != S.qmax && S.saved_tq5 != 0.0) {
            const double cquot = ode_div(S.tq[5], S.saved_tq5) * ode_pow(ode_div(S.h, S.tau[2]), (double)L);
            double tmp[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) tmp[s] = acv.v[s] - cquot * w->zn[S.qmax][lane + MT::G * s];
            const double dup = wrms_v<NS, MT::G>(tmp, ewv.v, MT::N) * S.tq[3];
            etaqp1 = ode_div(1.0, ode_pow(cv::BIAS3 * dup, ode_div(1.0, (double)(L + 1))) + cv::ADDON);
        }
        S.etaqm1 = etaqm1;
        S.etaqp1 = etaqp1;
        const double etaq = S.etaq;
        const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
        if (etam < cv::THRESH) {
            eta = 1.0;
        } else if (etam == etaqm1) {
            eta = etaqm1;
            qprime = q - 1;
        } else if (etam == etaq) {
            eta = etaq;
        } else {
            eta = etaqp1;
            qprime = q + 1;
#pragma unroll
            for (int s = 0; s < NS; ++s) w->zn[S.qmax][lane + MT::G * s] = acv.v[s];
        }
    }
    S.qprime = qprime;
    // cvSetEta
    if (eta < cv::THRESH) {
        eta = 1.0;
        S.hprime = S.h;
    } else {
        eta = fmin(eta, S.etamax);
        S.hprime = S.h * eta;
    }
    S.eta = eta;
}

// Failed error test: counters, restore and the new step (CVODE's
// cvDoErrorTest failure branch).  Returns TRY_AGAIN or CV_ERR_FAILURE.
template <class MT, class LinT>
__device__ __noinline__ int bdf_error_fail(unsigned off, double dsm, double saved_t, int nef, int lane) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    S.cnt[C_NETF]++;
    S.tn = saved_t;
    bdf_pascal<MT, LinT>(off, lane, false);
    if (nef == cv::MXNEF) return cv::CV_ERR_FAILURE;
    S.etamax = 1.0;
    if (nef <= cv::MXNEF1) {
        double eta = ode_div(1.0, ode_pow(cv::BIAS2 * dsm, ode_div(1.0, (double)S.L)) + cv::ADDON);
        eta = fmax(cv::ETAMIN, eta);
        if (nef >= cv::SMALL_NEF) eta = fmin(eta, cv::ETAMXF);
        S.eta = eta;
        bdf_rescale<MT, LinT>(off, lane);
        return cv::TRY_AGAIN;
    }
    if (S.q > 1) {
        S.eta = cv::ETAMIN;
        bdf_adjust_order<MT, LinT>(off, -1, lane);
        S.L = S.q;
        S.q--;
        S.qwait = S.L;
        bdf_rescale<MT, LinT>(off, lane);
        return cv::TRY_AGAIN;
    }
    S.eta = cv::ETAMIN;
    S.h *= S.eta;
    S.hscale = S.h;
    S.qwait = cv::LONG_WAIT;
    double z0[MT::NS], f[MT::NS];
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) z0[s] = w->zn[0][lane + MT::G * s];
    bdf_rhs<MT, LinT>(off, z0, f, lane);
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) w->zn[1][lane + MT::G * s] = S.h * f[s];
    return cv::TRY_AGAIN;
}

// Initial state and step (CVode's first call: ewt, f(y0), cvHin).  Returns 0 or
// a CVODE code.  Out of line: once per cell.
template <class MT, class LinT>
__device__ __noinline__ int bdf_begin(unsigned off, const Vec<MT::NS> y0, double t0, double tout, int lane) {
    constexpr int NS = MT::NS, N = MT::N;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
#pragma unroll 1
    for (int j = 0; j <= cv::QMAX; ++j)
#pragma unroll
        for (int s = 0; s < NS; ++s) w->zn[j][lane + MT::G * s] = (j == 0 && valid_el<MT::G>(lane, s, N)) ? y0.v[s] : 0.0;
    #pragma unroll 1
    for (int j = 0; j < 8; ++j) S.l[j] = S.tq[j] = S.tau[j] = 0.0;
    #pragma unroll 1
    for (int j = 0; j < 7; ++j) S.cnt[j] = 0;
    S.tn = t0;
    S.q = 1; S.L = 2; S.qwait = 2; S.qprime = 1;
    S.etamax = cv::ETAMX1;
    S.indx_acor = S.qmax;
    S.crate = 1.0;
    S.h = S.hprime = S.hscale = S.eta = S.hu = S.saved_tq5 = 0.0;
    S.gamma = S.gammap = S.gamrat = S.rl1 = S.acnrm = S.etaq = S.etaqm1 = S.etaqp1 = 0.0;
    S.jcur = 0; S.convfail = 0; S.nst = S.nstlp = S.nstlj = 0; S.nstloc = 0;
    double ewt[NS], z0[NS], z1[NS], y[NS], tmp[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        z0[s] = valid_el<MT::G>(lane, s, N) ? y0.v[s] : 0.0;
        ewt[s] = valid_el<MT::G>(lane, s, N) ? ode_div(1.0, S.rtol * fabs(z0[s]) + S.atol) : 0.0;
    }
    bdf_rhs<MT, LinT>(off, z0, z1, lane);
#pragma unroll
    for (int s = 0; s < NS; ++s) if (!valid_el<MT::G>(lane, s, N)) z1[s] = 0.0;
    // ---- cvHin
    const double tdiff = tout - t0;
    if (tdiff == 0.0) return cv::CV_TOO_CLOSE;
    const int sign = (tdiff > 0.0) ? 1 : -1;
    const double tdist = fabs(tdiff);
    const double tround = cv::UROUND * fmax(fabs(t0), fabs(tout));
    if (tdist < 2.0 * tround) return cv::CV_TOO_CLOSE;
    const double hlb = cv::HLB_FACTOR * tround;
    double r = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if (valid_el<MT::G>(lane, s, N)) {
            const double den = cv::HUB_FACTOR * fabs(z0[s]) + ode_div(1.0, ewt[s]);
            r = fmax(r, ode_div(fabs(z1[s]), den));
        }
    const double hub_inv = group_max<MT::G>(r);
    double hub = cv::HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = ode_div(1.0, hub_inv);
    double hg = sqrt(hlb * hub);
    double h0;
    if (hub < hlb) {
        h0 = sign * hg;
    } else {
        double hnew = hg;
        #pragma unroll 1
        for (int count1 = 1; count1 <= cv::MAX_HIN_ITERS; ++count1) {
            const double hgs = hg * sign;
#pragma unroll
            for (int s = 0; s < NS; ++s) y[s] = hgs * z1[s] + z0[s];
            bdf_rhs<MT, LinT>(off, y, tmp, lane);
            const double ih = ode_div(1.0, hgs);
#pragma unroll
            for (int s = 0; s < NS; ++s) tmp[s] = (tmp[s] - z1[s]) * ih;
            const double yddnrm = wrms_v<NS, MT::G>(tmp, ewt, N);
            hnew = (yddnrm * hub * hub > 2.0) ? sqrt(ode_div(2.0, yddnrm)) : sqrt(hg * hub);
            if (count1 == cv::MAX_HIN_ITERS) break;
            const double hrat = ode_div(hnew, hg);
            if (hrat > 0.5 && hrat < 2.0) break;
            if (count1 > 1 && hrat > 2.0) { hnew = hg; break; }
            hg = hnew;
        }
        double hh = cv::H_BIAS * hnew;
        if (hh < hlb) hh = hlb;
        if (hh > hub) hh = hub;
        h0 = sign * hh;
    }
    S.h = h0;
    S.hscale = h0;
    S.hprime = h0;
#pragma unroll
    for (int s = 0; s < NS; ++s) w->zn[1][lane + MT::G * s] = z1[s] * h0;
    return 0;
}

// Output: y(tout) by interpolation on success (CVodeGetDky), else the last
// accepted state.
template <class MT, class LinT>
__device__ __noinline__ Vec<MT::NS> bdf_finish(unsigned off, int status, double tout, int lane) {
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    Vec<MT::NS> out;
    if (status == 0) {
        const double s_ = ode_div(tout - S.tn, S.h);
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) out.v[s] = w->zn[S.q][lane + MT::G * s];
        #pragma unroll 1
        for (int j = S.q - 1; j >= 0; --j)
#pragma unroll
            for (int s = 0; s < MT::NS; ++s) out.v[s] = w->zn[j][lane + MT::G * s] + s_ * out.v[s];
    } else {
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) out.v[s] = w->zn[0][lane + MT::G * s];
    }
    S.cnt[C_NST] = S.nst;
    return out;
}

// Take up to max_new internal steps toward tout (CVode's main loop with
// cvStep inlined).  Sets done when tout is reached or a step failed; returns 0
// or a negative CVODE code.
template <class MT, class LinT>
__device__ __forceinline__ int bdf_advance(unsigned off, WarpGlobal<MT, LinT>* wg, double tout, int max_new,
                                           bool& done, int lane) {
    constexpr int NS = MT::NS, N = MT::N;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    BdfState& S = w->st;
    double ewt[NS], acor[NS], y[NS], ftemp[NS], delta[NS];
    done = false;
#pragma unroll 1
    for (int k = 0; k < max_new; ++k) {
        // ---- CVode loop: error weights, work limit, accuracy check
#pragma unroll
        for (int s = 0; s < NS; ++s)
            ewt[s] = valid_el<MT::G>(lane, s, N) ? ode_div(1.0, S.rtol * fabs(w->zn[0][lane + MT::G * s]) + S.atol) : 0.0;
        if (S.nstloc >= S.max_steps) { done = true; return cv::CV_TOO_MUCH_WORK; }
        if (cv::UROUND * wrms_zn<MT, LinT>(w, 0, ewt, lane) > 1.0) { done = true; return cv::CV_TOO_MUCH_ACC; }
        // ---- cvStep
        const double saved_t = S.tn;
        int ncf = 0, nef = 0, nflag = cv::FIRST_CALL;
        double dsm = 0.0;
        int kflag = 0;
        if (S.nst > 0 && S.hprime != S.h) {
            if (S.qprime != S.q) {
                bdf_adjust_order<MT, LinT>(off, S.qprime - S.q, lane);
                S.q = S.qprime;
                S.L = S.q + 1;
                S.qwait = S.L;
            }
            bdf_rescale<MT, LinT>(off, lane);
        }
#pragma unroll 1
        for (int guard = 0; guard < 64; ++guard) {
            S.tn += S.h;
            bdf_pascal<MT, LinT>(off, lane, true);
            bdf_set_coeffs<MT, LinT>(off);
            // ---- cvNls: modified Newton
            S.convfail = ((nflag == cv::FIRST_CALL) || (nflag == cv::PREV_ERR_FAIL)) ? cv::NO_FAILURES : cv::FAIL_OTHER;
            int call_setup = (nflag == cv::PREV_CONV_FAIL) || (nflag == cv::PREV_ERR_FAIL) || (S.nst == 0) ||
                             (S.nst >= S.nstlp + cv::MSBP) || (fabs(S.gamrat - 1.0) > cv::DGMAX_LSETUP);
#pragma unroll
            for (int s = 0; s < NS; ++s) acor[s] = 0.0;
            int jbad = 0, ret = 0;
#pragma unroll 1
            for (int attempt = 0; attempt < 4; ++attempt) {
                // residual at ycor = acor
#pragma unroll
                for (int s = 0; s < NS; ++s) y[s] = w->zn[0][lane + MT::G * s] + acor[s];
                bdf_rhs<MT, LinT>(off, y, ftemp, lane);
#pragma unroll
                for (int s = 0; s < NS; ++s) delta[s] = -S.gamma * ftemp[s] + (S.rl1 * w->zn[1][lane + MT::G * s] + acor[s]);
                if (call_setup) {
                    Vec<NS> yv;
#pragma unroll
                    for (int s = 0; s < NS; ++s) yv.v[s] = y[s];
                    ret = bdf_ls_setup<MT, LinT>(off, yv, wg, jbad, lane) ? cv::CONV_RECVR : 0;
                    if (ret) break;
                }
                double delp = 0.0;
                ret = 0;
                bool converged = false;
#pragma unroll 1
                for (int m = 0;; ++m) {
                    S.cnt[C_NNI]++;
#pragma unroll
                    for (int s = 0; s < NS; ++s) delta[s] = -delta[s];
                    bdf_solve<MT, LinT>(off, delta, wg, lane);
#pragma unroll
                    for (int s = 0; s < NS; ++s) acor[s] += delta[s];
                    const double del = wrms_v<NS, MT::G>(delta, ewt, N);
                    if (m > 0) S.crate = fmax(cv::CRDOWN * S.crate, ode_div(del, delp));
                    const double dcon = ode_div(del * fmin(1.0, S.crate), S.tq[4]);
                    if (dcon <= 1.0) {
                        S.acnrm = (m == 0) ? del : wrms_v<NS, MT::G>(acor, ewt, N);
                        S.jcur = 0;
                        converged = true;
                        break;
                    }
                    if (m >= 1 && del > cv::RDIV * delp) { ret = cv::CONV_RECVR; break; }
                    delp = del;
                    if (m + 1 >= cv::NLS_MAXCOR) { ret = cv::CONV_RECVR; break; }
#pragma unroll
                    for (int s = 0; s < NS; ++s) y[s] = w->zn[0][lane + MT::G * s] + acor[s];
                    bdf_rhs<MT, LinT>(off, y, ftemp, lane);
#pragma unroll
                    for (int s = 0; s < NS; ++s) delta[s] = -S.gamma * ftemp[s] + (S.rl1 * w->zn[1][lane + MT::G * s] + acor[s]);
                }
                if (converged) { ret = 0; break; }
                if (ret == cv::CONV_RECVR && !S.jcur) {
                    call_setup = 1;
                    jbad = 1;
#pragma unroll
                    for (int s = 0; s < NS; ++s) acor[s] = 0.0;
                    continue;
                }
                break;
            }
            nflag = ret;
            // ---- cvHandleNFlag
            if (nflag != 0) {
                S.cnt[C_NCFN]++;
                S.tn = saved_t;
                bdf_pascal<MT, LinT>(off, lane, false);
                ncf++;
                S.etamax = 1.0;
                if (ncf == cv::MXNCF) { kflag = cv::CV_CONV_FAILURE; break; }
                S.eta = cv::ETACF;
                nflag = cv::PREV_CONV_FAIL;
                bdf_rescale<MT, LinT>(off, lane);
                continue;
            }
            // ---- cvDoErrorTest
            dsm = S.acnrm * S.tq[2];
            if (dsm > 1.0) {
                nef++;
                nflag = cv::PREV_ERR_FAIL;
                const int ef = bdf_error_fail<MT, LinT>(off, dsm, saved_t, nef, lane);
                if (ef == cv::TRY_AGAIN) continue;
                kflag = ef;
                break;
            }
            // ---- cvCompleteStep
            S.nst++;
            S.hu = S.h;
            {
                const int q = S.q;
                #pragma unroll 1
                for (int i = q; i >= 2; --i) S.tau[i] = S.tau[i - 1];
                if (q == 1 && S.nst > 1) S.tau[2] = S.tau[1];
                S.tau[1] = S.h;
#pragma unroll 1
                for (int j = 0; j <= q; ++j) {
                    const double lj = S.l[j];
#pragma unroll
                    for (int s = 0; s < NS; ++s) w->zn[j][lane + MT::G * s] += lj * acor[s];
                }
                S.qwait--;
                if (S.qwait == 1 && q != S.qmax) {
#pragma unroll
                    for (int s = 0; s < NS; ++s) w->zn[S.qmax][lane + MT::G * s] = acor[s];
                    S.saved_tq5 = S.tq[5];
                    S.indx_acor = S.qmax;
                }
            }
            {
                Vec<NS> av, ev;
#pragma unroll
                for (int s = 0; s < NS; ++s) { av.v[s] = acor[s]; ev.v[s] = ewt[s]; }
                bdf_prepare_next_step<MT, LinT>(off, dsm, av, ev, lane);
            }
            S.etamax = (S.nst <= cv::SMALL_NST) ? cv::ETAMX2 : cv::ETAMX3;
            kflag = 0;
            break;
        }
        if (kflag != 0) { done = true; return kflag; }
        S.nstloc++;
        if ((S.tn - tout) * S.h >= 0.0) { done = true; return 0; }
    }
    return 0;
}

// ------------------------------------------------- state in HBM (step form)
// Per-cell record of the one-launch-per-step form: the method state, the
// Nordsieck history and the Newton-matrix factors (the saved Jacobian lives in
// the cell's WarpGlobal).
template <class MT, class LinT>
struct StepRecord {
    static constexpr int N = MT::N;
    static constexpr size_t kStateBytes = (sizeof(BdfState) + 255) & ~size_t(255);
    static constexpr size_t kZnBytes = ((cv::QMAX + 1) * N * sizeof(double) + 255) & ~size_t(255);
    static constexpr size_t kLuBytes = (N * MT::LDA * sizeof(LinT) + N * sizeof(int) + 255) & ~size_t(255);
    static constexpr size_t kBytes = kStateBytes + 8 + kZnBytes + kLuBytes;   // + phase word
    static constexpr size_t kPhaseOff = kStateBytes;
};

template <class MT, class LinT>
__device__ __noinline__ void bdf_save(unsigned off, unsigned char* rec, int phase, int lane) {
    using R = StepRecord<MT, LinT>;
    constexpr int N = MT::N;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    const int* src = reinterpret_cast<const int*>(&w->st);
    int* dst = reinterpret_cast<int*>(rec);
#pragma unroll 1
    for (int e = lane; e < (int)(sizeof(BdfState) / 4); e += MT::G) dst[e] = src[e];
    if (lane == 0) *reinterpret_cast<int*>(rec + R::kPhaseOff) = phase;
    double* Z = reinterpret_cast<double*>(rec + R::kStateBytes + 8);
    #pragma unroll 1
    for (int j = 0; j <= cv::QMAX; ++j)
#pragma unroll
        for (int s = 0; s < MT::NS; ++s)
            if (valid_el<MT::G>(lane, s, N)) Z[j * N + lane + MT::G * s] = w->zn[j][lane + MT::G * s];
    if (w->st.lu_dirty) {
        LinT* Ag = reinterpret_cast<LinT*>(rec + R::kStateBytes + 8 + R::kZnBytes);
#pragma unroll 1
        for (int e = lane; e < N * MT::LDA; e += MT::G) Ag[e] = w->A[e];
        int* pg = reinterpret_cast<int*>(Ag + N * MT::LDA);
        #pragma unroll 1
        for (int e = lane; e < N; e += MT::G) pg[e] = w->perm[e];
    }
    __syncwarp(gmask<MT::G>());
}

template <class MT, class LinT>
__device__ __noinline__ void bdf_load(unsigned off, const unsigned char* rec, int lane) {
    using R = StepRecord<MT, LinT>;
    constexpr int N = MT::N;
    WarpSmem<MT, LinT>* w = wsm<MT, LinT>(off);
    const int* src = reinterpret_cast<const int*>(rec);
    int* dst = reinterpret_cast<int*>(&w->st);
#pragma unroll 1
    for (int e = lane; e < (int)(sizeof(BdfState) / 4); e += MT::G) dst[e] = src[e];
    const double* Z = reinterpret_cast<const double*>(rec + R::kStateBytes + 8);
    #pragma unroll 1
    for (int j = 0; j <= cv::QMAX; ++j)
#pragma unroll
        for (int s = 0; s < MT::NS; ++s)
            w->zn[j][lane + MT::G * s] = valid_el<MT::G>(lane, s, N) ? Z[j * N + lane + MT::G * s] : 0.0;
    const LinT* Ag = reinterpret_cast<const LinT*>(rec + R::kStateBytes + 8 + R::kZnBytes);
#pragma unroll 1
    for (int e = lane; e < N * MT::LDA; e += MT::G) w->A[e] = Ag[e];
    const int* pg = reinterpret_cast<const int*>(Ag + N * MT::LDA);
    #pragma unroll 1
    for (int e = lane; e < N; e += MT::G) w->perm[e] = (unsigned char)pg[e];
    __syncwarp(gmask<MT::G>());
}

}  // namespace b200
