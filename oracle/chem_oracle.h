/* CPU oracle for the chemistry source terms -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
 * this code, to check results.  The product path (hpc_ode_b200/csrc) never
 * links it.
 *
 * It restates, table-driven, what the reference's pyJac C kernels compute:
 *   dydt(t, pres, y, dy)        src/Mechanism/CPU/dydt.c:7-133
 *   eval_jacob(t, pres, y, jac) src/Mechanism/CPU/jacob.c:3-372
 * with the same argument meaning: y = [T, Y_0 .. Y_{n-2}] (length n = number
 * of species), dy the same length, jac column-major n x n with
 * jac[i + n*j] = d f_i / d y_j.  The last species closes the mass balance.
 *
 * Parity: pinned against the compiled reference pyJac kernels for GRI-Mech 3.0
 * through committed golden vectors (tests/golden/gri30_chem_golden.npz).
 */
#ifndef HPC_ODE_ORACLE_CHEM_H
#define HPC_ODE_ORACLE_CHEM_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mechanism ids. */
enum { ORACLE_MECH_GRI30 = 0, ORACLE_MECH_H2O2 = 1, ORACLE_MECH_NDODECANE = 2, ORACLE_MECH_H2LI = 3,
       ORACLE_MECH_ESTIMATE = 4 };

int oracle_mech_id(const char* name);      /* "gri30"/"gri30.yaml"/"h2o2"... ; -1 if unknown */
int oracle_mech_nsp(int mech);             /* number of species == state length */

/* pyJac-signature entry points (one per mechanism). */
void oracle_gri30_dydt(double t, double pres, const double* y, double* dy);
void oracle_gri30_jacob(double t, double pres, const double* y, double* jac);
void oracle_h2o2_dydt(double t, double pres, const double* y, double* dy);
void oracle_h2o2_jacob(double t, double pres, const double* y, double* jac);
void oracle_ndodecane_dydt(double t, double pres, const double* y, double* dy);
void oracle_ndodecane_jacob(double t, double pres, const double* y, double* jac);
void oracle_h2li_dydt(double t, double pres, const double* y, double* dy);
void oracle_h2li_jacob(double t, double pres, const double* y, double* jac);
void oracle_estimate_dydt(double t, double pres, const double* y, double* dy);
void oracle_estimate_jacob(double t, double pres, const double* y, double* jac);

/* Generic forms. */
void oracle_dydt(int mech, double pres, const double* y, double* dy);
void oracle_jacob(int mech, double pres, const double* y, double* jac);

/* Constant-volume forms: rho is the cell's fixed density, the pressure
 * follows from the state (P = rho R T / W); the energy equation conserves
 * internal energy instead of enthalpy.  The reference's pyJac CONV branch
 * (src/Mechanism/CPU/dydt.c:135-265, eval_conc_rho in chem_utils.c:99-137;
 * it does not compile as shipped) states the same formulation. */
void oracle_dydt_conv(int mech, double rho, const double* y, double* dy);
void oracle_jacob_conv(int mech, double rho, const double* y, double* jac);
void oracle_dydt_scale_conv(int mech, double rho, const double* y, double* scale);
/* Density of the state y at pressure pres. */
double oracle_density(int mech, double pres, const double* y);

/* Forward rate coefficient of every reaction at (T, P), kf[nrxn] (falloff:
 * the high-pressure limit; PLOG: interpolated in ln P). */
void oracle_kf(int mech, double pres, double T, double* kf);

/* Magnitude companion of dydt: |dy|-scale built from |forward| + |reverse|
 * contributions, used by tests to form cancellation-aware tolerances. */
void oracle_dydt_scale(int mech, double pres, const double* y, double* scale);

#ifdef __cplusplus
}
#endif
#endif
