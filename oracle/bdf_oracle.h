/* CPU oracle: CVODE-semantics variable-order BDF -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs to
 * check results; never linked by the product.
 *
 * Stands in for the reference's serial CVODE integrator
 * (src/Integrators/CVodeIntegrator.cpp:98-155: CVodeCreate(CV_BDF),
 * CVodeSStolerances, SUNDenseMatrix + SUNLinSol_Dense, CVodeSetJacFn,
 * CVodeSetMaxNumSteps(10000), CVode(..., tout, CV_NORMAL)).  SUNDIALS (pinned
 * at v6.3.0 by the reference's CMakeLists.txt:46) is an un-vendored submodule,
 * so the algorithm is restated from CVODE's published description
 * (Hindmarsh et al., ACM TOMS 31(3) 2005, and the CVODE user guide), with
 * CVODE's default heuristics.  Parity of the BDF with SUNDIALS itself is
 * therefore unpinned; the solution is cross-checked against scipy's VODE and
 * Radau at tight tolerance.
 *
 * The RHS / Jacobian callbacks have pyJac's signatures
 * (src/Mechanism/CPU/dydt.h:6, jacob.h:8), so the compiled reference kernels
 * can be passed in directly, as CVodeSerialDriver.cpp:19-36 does.
 */
#ifndef HPC_ODE_ORACLE_BDF_H
#define HPC_ODE_ORACLE_BDF_H

#ifdef __cplusplus
extern "C" {
#endif

typedef void (*oracle_rhs_fn)(double t, double pres, const double* y, double* dy);
typedef void (*oracle_jac_fn)(double t, double pres, const double* y, double* jac);

typedef struct {
    double rtol;
    double atol;
    int max_steps;     /* CVodeSetMaxNumSteps; reference uses 10000 */
    int max_order;     /* 1..5, CVODE default 5 */
} oracle_bdf_opts;

/* Per-cell counters, named after CVODE's CVodeGet* outputs. */
typedef struct {
    int status;        /* 0 = CV_SUCCESS, else a CVODE return code (negative) */
    int nst;           /* steps taken */
    int nfe;           /* RHS evaluations */
    int nje;           /* Jacobian evaluations */
    int nsetups;       /* linear-solver setups (= LU factorizations) */
    int nni;           /* Newton iterations (= linear solves) */
    int ncfn;          /* nonlinear convergence failures */
    int netf;          /* error-test failures */
    int qlast;
    double hlast;
} oracle_bdf_stats;

/* CVODE return codes used as per-cell status. */
enum {
    ORACLE_CV_SUCCESS = 0,
    ORACLE_CV_TOO_MUCH_WORK = -1,
    ORACLE_CV_TOO_MUCH_ACC = -2,
    ORACLE_CV_ERR_FAILURE = -3,
    ORACLE_CV_CONV_FAILURE = -4,
    ORACLE_CV_TOO_CLOSE = -27
};

/* Integrate one system of size n from t0 to tout (CV_NORMAL).  y is in/out.
 * On failure y holds the last accepted state, as CVode returns zn[0]. */
int oracle_bdf_solve(oracle_rhs_fn f, oracle_jac_fn J, int n, double pres, double* y,
                     double t0, double tout, const oracle_bdf_opts* opts,
                     oracle_bdf_stats* stats);

/* Batch driver: y is cell-major [ncells][n].  pres is per cell (or NULL to use
 * pres_scalar).  nthreads > 1 runs an OpenMP parallel-for with dynamic
 * schedule, chunk 1, over cells (the reference's CVodeIntegratorOMP.cpp:21
 * under OpenMPRuntime's "dynamic,1").  stats may be NULL.  Returns the number
 * of cells whose status is not CV_SUCCESS. */
long oracle_bdf_batch(oracle_rhs_fn f, oracle_jac_fn J, int n, long ncells, const double* pres,
                      double pres_scalar, double* y, double t0, double tout,
                      const oracle_bdf_opts* opts, oracle_bdf_stats* stats, int nthreads);

/* Same, with the chemistry selected by mechanism id (chem_oracle.h). */
long oracle_bdf_batch_mech(int mech, long ncells, const double* pres, double pres_scalar,
                           double* y, double t0, double tout, const oracle_bdf_opts* opts,
                           oracle_bdf_stats* stats, int nthreads);

/* Constant-volume form: pres (or pres_scalar) is each cell's initial
 * pressure; the cell's density follows from its initial state and stays fixed. */
long oracle_bdf_batch_mech_conv(int mech, long ncells, const double* pres, double pres_scalar,
                                double* y, double t0, double tout, const oracle_bdf_opts* opts,
                                oracle_bdf_stats* stats, int nthreads);

/* The chemistry callbacks of a mechanism id (conv = 1: constant volume, the
 * pres argument carrying the density). */
void oracle_mech_fns(int mech, int conv, oracle_rhs_fn* f, oracle_jac_fn* J);

#ifdef __cplusplus
}
#endif
#endif
