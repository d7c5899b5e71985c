// Warp-per-cell chemistry: constant-pressure RHS and analytic Jacobian.
//
// One group of G lanes evaluates one cell (G = 32, a whole warp, except for the
// smallest mechanisms; see MechT).  The lanes split the work three ways:
//   * species phase   -- lane l owns species l, l+G, ... (thermo, concentrations);
//   * reaction phase  -- lane l evaluates reaction slot G*g + l of group g
//                        (kf, Kc, third-body / falloff modifiers, rates of progress);
//   * gather phase    -- production rates summed from the rates of progress with
//                        a balanced, coalesced (species, reaction) list dealt to
//                        32 lists (lane l sums lists l, l+G, ...) in a fixed order;
//                        partial sums are combined per species in a fixed order
//                        (no atomics, so results do not depend on scheduling).
// Per-cell intermediates (concentrations, -g/RT, rates) live in shared memory,
// never in HBM (the reference's GPU path keeps ~31.8 KB of them per cell in global
// memory: src/Mechanism/GPU/gpu_memory.cu:3-37).
//
// Reference math (pyJac C, src/Mechanism/CPU): eval_conc chem_utils.c:4-97,
// eval_rxn_rates rxn_rates.c:2-3862, get_rxn_pres_mod rxn_rates_pres_mod.c:5-366,
// eval_spec_rates spec_rates.c:4, dydt dydt.c:7-133, eval_jacob jacob.c:3-372.
//
// Internal element order of a state vector: element i < N-1 is Y_i, element N-1
// is T (so that a lane's species slot and state slot coincide); the reference's
// order is [T, Y_0 .. Y_{N-2}].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mech_dev.h"

namespace b200 {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kRU = 8314.4621;

// Compile-time shape of one generated mechanism: species count, reaction
// count, descriptor index, the denominator of its stoichiometric coefficients
// (1, or 2 / 4 with fractional product coefficients), its gather units and
// whether it has PLOG reactions (the PLOG branch is compiled only then: the
// reaction code is on the instruction-fetch-bound hot path), and the reactor
// formulation: constant pressure, or constant volume (CONV_ = 1; the kernels'
// pressure slot then carries the cell's fixed density).  Both are compile-time
// so a kernel holds no code of the other case.  G_ is the number of lanes that
// integrate one cell; the device code takes every shuffle, vote and sync over
// the cell's aligned group of G lanes.  All compiled kernels use G = 32 (a warp
// per cell): 2 or 4 cells per warp for the 9-10-species H2 mechanisms ran
// slower than one (the cells' step logic diverges, and the extra registers
// cost resident warps), so those instances are not built.
template <int N_, int NR_, int ID_, int NU_DEN_, int NUNITS_, int NPLOG_, int CONV_ = 0, int G_ = 32>
struct MechT {
    static_assert(G_ == 32 || G_ == 16 || G_ == 8, "lanes per cell: 32, 16 or 8");
    static constexpr int ID = ID_;                            // index into c_mech
    static constexpr int N = N_;                              // state length == species count
    static constexpr int G = G_;                              // lanes per cell (32 / G cells per warp)
    static constexpr int NS = (N_ + G_ - 1) / G_;             // elements per lane
    static constexpr int NSLOT = ((NR_ + 32) / 32) * 32;      // reaction slots (>= 1 padding slot)
    static constexpr int NG = NSLOT / G_;                     // reaction groups (G slots each)
    static constexpr int LDA = (N_ % 2 == 0) ? N_ + 1 : N_;   // odd stride: conflict-free rows/cols
    static constexpr int NU_DEN = NU_DEN_;                    // gather words hold nu * NU_DEN
    static constexpr int NUNITMAX = NUNITS_;                  // gather units (checked at creation)
    static constexpr bool PLOG = NPLOG_ > 0;
    static constexpr bool CONV = CONV_ != 0;
};

// Mechanism descriptors (one per compiled mechanism), set once per device.
constexpr int kNumMech = 5;
__constant__ DevMech c_mech[kNumMech];

template <class MT>
__device__ __forceinline__ const DevMech& mech() { return c_mech[MT::ID]; }

// A lane's slice of a state vector (element i = lane + G*s, lane within the
// cell's group of MT::G lanes), passed by value
// so the heavy phases can be single-copy (non-inlined) functions without
// forcing the caller's state into local memory.
template <int NS>
struct Vec {
    double v[NS];
};

// Element s of a lane's register slice (s not known at compile time): a select
// chain over the NS registers instead of a local-memory index.
template <int NS, class T>
__device__ __forceinline__ T pick(const T (&x)[NS], int s) {
    T r = x[0];
#pragma unroll
    for (int q = 1; q < NS; ++q) r = (s == q) ? x[q] : r;
    return r;
}
template <int NS, class T>
__device__ __forceinline__ void place(T (&x)[NS], int s, T v) {
#pragma unroll
    for (int q = 0; q < NS; ++q) if (s == q) x[q] = v;
}

// The kernels' dynamic shared memory.  Out-of-line phases receive byte offsets
// into it (not pointers) and rebuild typed pointers here, so every access
// compiles to a shared-memory instruction instead of a generic one.
__device__ __forceinline__ unsigned char* dyn_smem() {
    extern __shared__ __align__(16) unsigned char b200_dyn_smem[];
    return b200_dyn_smem;
}
__device__ __forceinline__ unsigned smem_off(const void* p) {
    return (unsigned)((const unsigned char*)p - dyn_smem());
}
template <class T>
__device__ __forceinline__ T* smem_at(unsigned off) {
    return reinterpret_cast<T*>(dyn_smem() + off);
}

// Mask of the aligned group of G lanes this thread belongs to.
template <int G>
__device__ __forceinline__ unsigned gmask() {
    if constexpr (G == 32) return kFull;
    else return ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
}

// Sum / max over the thread's group of G lanes (every lane gets the result).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
    const unsigned m = gmask<G>();
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o, G);
    return v;
}
template <int G>
__device__ __forceinline__ double group_max(double v) {
    const unsigned m = gmask<G>();
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(m, v, o, G));
    return v;
}
// Value of lane `src` (0..G-1) of the thread's group.
template <int G, class T>
__device__ __forceinline__ T group_shfl(T v, int src) {
    return __shfl_sync(gmask<G>(), v, src, G);
}
__device__ __forceinline__ double warp_sum(double v) { return group_sum<32>(v); }
__device__ __forceinline__ double warp_max(double v) { return group_max<32>(v); }

// Per-warp shared scratch of the chemistry.
template <class MT>
struct ChemSmem {
    double C[MT::N + 1];          // concentrations [kmol/m^3]; C[N] = 1 (padding factor)
    double G[MT::N + 1];          // s/R - h/RT; G[N] = 0
    double q[MT::NSLOT];          // rates of progress (Jacobian: reused for per-species work)
    double part[MT::NUNITMAX];    // gather partial sums
};

// Per-warp global scratch of the Jacobian (L1/L2 resident; the Jacobian is rare).
template <class MT>
struct JacScratch {
    double dqdT[MT::NSLOT];       // d q / d T at fixed mass fractions
    double sr[MT::NSLOT];         // sum_i (d q / d C_i) C_i
    double H[MT::N + 1];          // h/RT of every species (H[N] = 0)
};

// NASA-7 polynomials of species k at T: cp/R, h/RT, s/R - h/RT, d(cp/R)/dT.
// Coefficients from the species-innermost copy (nasa_sk), so the lanes of a
// warp, which hold consecutive species, read consecutive words.
__device__ __forceinline__ void nasa7(const DevMech& M, int k, double T, double logT, double invT,
                                      double& cpR, double& hRT, double& mgRT, double& dcpR) {
    const int nsp = M.nsp;
    const double* a = M.nasa_sk + ((T <= __ldg(M.tmid + k)) ? 0 : 7) * nsp + k;
    const double a0 = __ldg(a), a1 = __ldg(a + nsp), a2 = __ldg(a + 2 * nsp), a3 = __ldg(a + 3 * nsp),
                 a4 = __ldg(a + 4 * nsp), a5 = __ldg(a + 5 * nsp), a6 = __ldg(a + 6 * nsp);
    cpR = a0 + T * (a1 + T * (a2 + T * (a3 + a4 * T)));
    hRT = a0 + T * (a1 * 0.5 + T * (a2 * (1.0 / 3.0) + T * (a3 * 0.25 + a4 * 0.2 * T))) + a5 * invT;
    mgRT = a0 * (logT - 1.0) + T * (a1 * 0.5 + T * (a2 * (1.0 / 6.0) + T * (a3 * (1.0 / 12.0) + a4 * 0.05 * T)))
           - a5 * invT + a6;
    dcpR = a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T));
}

// Common cell quantities of one RHS / Jacobian evaluation.
struct CellThermo {
    double T, logT, invT, m, rho, mw_avg, yN, mC;   // mC = m - sum_k C_k
};

// Out-of-line FP64 transcendentals: one copy of each library routine in the
// kernel image instead of one per call site.  The integration kernel is bound
// by instruction fetch (its hot code is larger than the SM's instruction
// cache), so every call site that is not a full inline expansion helps.
__device__ __noinline__ double ode_exp(double x) { return exp(x); }
// Two independent exponentials in one call, so that their dependency chains
// overlap (same function, same results as two ode_exp calls).  Taken by the
// mechanisms of kPairedExpMinN unknowns up; the smaller ones' kernels are bound
// by instruction fetch and registers, where the second copy of exp costs more
// than the overlap saves.
struct Exp2 {
    double a, b;
};
__device__ __noinline__ Exp2 ode_exp2(double x, double y) { return Exp2{exp(x), exp(y)}; }
constexpr int kPairedExpMinN = 64;
__device__ __noinline__ double ode_log10(double x) { return log10(x); }
__device__ __noinline__ double ode_log(double x) { return log(x); }
__device__ __noinline__ double ode_exp10(double x) { return exp10(x); }
__device__ __noinline__ double ode_pow(double x, double y) { return pow(x, y); }
// IEEE division out of line: an inline FP64 division is ~40 instructions, so
// the scalar step-control code calls this single copy instead.
__device__ __noinline__ double ode_div(double a, double b) { return a / b; }

// Species phase: concentrations and Gibbs terms into shared memory; with a
// non-null H (the Jacobian), h/RT of every species into H as well.
template <class MT>
__device__ __forceinline__ CellThermo species_phase(const DevMech& M, double P, const double (&y)[MT::NS],
                                                    ChemSmem<MT>* sm, int lane, double (&Yk)[MT::NS],
                                                    double (&cpR)[MT::NS], double (&hRT)[MT::NS],
                                                    double (&dcpR)[MT::NS], double* H = nullptr) {
    constexpr int N = MT::N, G = MT::G;
    CellThermo c;
    c.T = group_shfl<G>(y[(N - 1) / G], (N - 1) % G);
    double sy = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        if (i < N - 1) sy += y[s];
    }
    c.yN = 1.0 - group_sum<G>(sy);
    double sw = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        Yk[s] = (i < N - 1) ? y[s] : ((i == N - 1) ? c.yN : 0.0);
        if (i < N) sw += Yk[s] * __ldg(M.inv_mw + i);
    }
    c.mw_avg = ode_div(1.0, group_sum<G>(sw));
    c.logT = log(c.T);
    c.invT = ode_div(1.0, c.T);
    if constexpr (!MT::CONV) {
        c.rho = ode_div(P * c.mw_avg, kRU * c.T);
        c.m = ode_div(P, kRU * c.T);
    } else {
        // constant volume: P is the cell's fixed density, the pressure follows
        // from the state (P = rho R T / W)
        c.rho = P;
        c.m = ode_div(P, c.mw_avg);
    }
    double csum = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        if (i < N) {
            double g;
            nasa7(M, i, c.T, c.logT, c.invT, cpR[s], hRT[s], g, dcpR[s]);
            const double Ci = c.rho * Yk[s] * __ldg(M.inv_mw + i);
            csum += Ci;
            sm->C[i] = Ci;
            sm->G[i] = g;
            if (H) H[i] = hRT[s];
        } else {
            cpR[s] = hRT[s] = dcpR[s] = 0.0;
        }
    }
    c.mC = c.m - group_sum<G>(csum);
    if (lane == 0) {
        sm->C[N] = 1.0;
        sm->G[N] = 0.0;
        if (H) H[N] = 0.0;
    }
    if (H) __threadfence_block();   // H is global: order it for the other lanes
    __syncwarp(gmask<G>());
    return c;
}


// Rates of one reaction slot.  With Deriv, also the pieces of its derivative.
struct RxnOut {
    double q;            // (Rf - Rr) * phi
    double kf, kr;       // rate coefficients
    double Rf, Rr;       // kf prod C', kr prod C''
    double phi, thd, dphi_dthd, dphi_dT, dlnkf_dT;
};

// Falloff blending of one reaction (Lindemann or Troe): sets phi and, with
// Deriv, its derivatives.  Out of line: one reaction group of the mechanism
// uses it, and keeping it out of the reaction loop keeps that loop small.
struct FallOut {
    double phi, dphi_dthd, dphi_dT;
};

template <class MT>
__device__ __noinline__ FallOut falloff(int s, int fl, double T, double logT, double invT,
                                        double kf, double thd, int Deriv) {
    const DevMech& M = mech<MT>();
    const int type = fl & kFlagTypeMask;
    struct { double T, logT, invT; } c = {T, logT, invT};
    FallOut o;
    o.dphi_dthd = 0.0;
    o.dphi_dT = 0.0;
    const double b = __ldg(M.b + s), EaR = __ldg(M.EaR + s);
    const double b0 = __ldg(M.b0 + s), EaR0 = __ldg(M.EaR0 + s);
    const double k0 = (fl & kFlagConstK0) ? __ldg(M.A0const + s)
                                          : ode_exp(__ldg(M.logA0 + s) + b0 * c.logT - EaR0 * c.invT);
    const double Pr = ode_div(k0 * thd, kf);
    double F = 1.0, dl_dx = 0.0, dl_dT = 0.0;
    if (type == 3) {
        const double a = __ldg(M.troe_a + s), iT3 = __ldg(M.troe_iT3 + s), iT1 = __ldg(M.troe_iT1 + s);
        double e3, e1;
        if constexpr (MT::N >= kPairedExpMinN) {
            const Exp2 e31 = ode_exp2(-c.T * iT3, -c.T * iT1);
            e3 = e31.a;
            e1 = e31.b;
        } else {
            e3 = ode_exp(-c.T * iT3);
            e1 = ode_exp(-c.T * iT1);
        }
        double Fcent = (1.0 - a) * e3 + a * e1;
        double dFcent = 0.0;
        if (Deriv) dFcent = -(1.0 - a) * iT3 * e3 - a * iT1 * e1;
        if (fl & kFlagT2) {
            const double T2 = __ldg(M.troe_T2 + s);
            const double e2 = ode_exp(-T2 * c.invT);
            Fcent += e2;
            if (Deriv) dFcent += T2 * c.invT * c.invT * e2;
        }
        const double Fc = ode_log10(fmax(Fcent, 1.0e-300));
        const double x = ode_log10(fmax(Pr, 1.0e-300));
        const double A = x - 0.67 * Fc - 0.4;
        const double B = 0.806 - 1.1762 * Fc - 0.14 * x;
        const double u = ode_div(A, B);
        const double den = 1.0 + u * u;
        F = ode_exp10(ode_div(Fc, den));
        if (Deriv) {
            const double du_dx = ode_div(B + 0.14 * A, B * B);
            const double du_dFc = ode_div(-0.67 * B + 1.1762 * A, B * B);
            dl_dx = (Pr > 1.0e-300) ? ode_div(-Fc * 2.0 * u * du_dx, den * den) : 0.0;
            const double dl_dFc = ode_div(1.0, den) - ode_div(Fc * 2.0 * u * du_dFc, den * den);
            const double dFc_dT = (Fcent > 1.0e-300) ? ode_div(dFcent, Fcent * 2.302585092994046) : 0.0;
            dl_dT = dl_dFc * dFc_dT;
        }
    }
    const double blend = ode_div(Pr, 1.0 + Pr);
    o.phi = F * blend;
    if (Deriv) {
        const double dphi_dPr = ode_div(F, (1.0 + Pr) * (1.0 + Pr)) + ode_div(F, 1.0 + Pr) * dl_dx;
        o.dphi_dthd = dphi_dPr * ode_div(k0, kf);
        const double dlnPr_dT = (b0 + EaR0 * c.invT) * c.invT - (b + EaR * c.invT) * c.invT;
        o.dphi_dT = dphi_dPr * Pr * dlnPr_dT + blend * F * 2.302585092994046 * dl_dT;
    }
    return o;
}

// Pressure-dependent Arrhenius (PLOG) rate of slot s: ln k linear in ln P
// between the two tabulated pressures that bracket the cell's P, the end
// level's k outside the table (Cantera's PLOG definition, which the
// reference's Cantera integrator evaluates for these reactions); a level's k
// is the sum of its Arrhenius terms.  Returns ln k and d ln k / dT.
struct PlogOut {
    double lnk, dlnk_dT, dlnk_dlnP;   // d ln k / d ln P: 0 outside the table
};

template <class MT>
__device__ __noinline__ PlogOut plog_rate(int s, double T, double logT, double invT, double lnP) {
    const DevMech& M = mech<MT>();
    const int l0 = __ldg(M.plog_lev0 + s), l1 = l0 + __ldg(M.plog_nlev + s) - 1;
    int lo = l0, hi = l0;
    double w = 0.0;
    if (lnP >= __ldg(M.plog_lnP + l1)) {
        lo = hi = l1;
    } else if (lnP > __ldg(M.plog_lnP + l0)) {
        while (lo + 1 < l1 && __ldg(M.plog_lnP + lo + 1) < lnP) ++lo;
        hi = lo + 1;
        const double p0 = __ldg(M.plog_lnP + lo);
        w = ode_div(lnP - p0, __ldg(M.plog_lnP + hi) - p0);
    }
    double lk[2], dl[2];
#pragma unroll 1
    for (int e = 0; e < 2; ++e) {
        const int l = e ? hi : lo;
        double k = 0.0, dk = 0.0;
        const int t1 = __ldg(M.plog_toff + l + 1);
#pragma unroll 1
        for (int t = __ldg(M.plog_toff + l); t < t1; ++t) {
            const double b = __ldg(M.plog_b + t), EaR = __ldg(M.plog_EaR + t);
            const double kt = (b == 0.0 && EaR == 0.0) ? __ldg(M.plog_A + t)
                                                       : ode_exp(__ldg(M.plog_logA + t) + b * logT - EaR * invT);
            k += kt;
            dk += kt * (b + EaR * invT) * invT;
        }
        lk[e] = ode_log(k);
        dl[e] = ode_div(dk, k);
    }
    const double slope = (hi != lo) ? ode_div(lk[1] - lk[0], __ldg(M.plog_lnP + hi) - __ldg(M.plog_lnP + lo)) : 0.0;
    return PlogOut{(1.0 - w) * lk[0] + w * lk[1], (1.0 - w) * dl[0] + w * dl[1], slope};
}

// Cell quantities the reaction phase needs (passed by value to the
// out-of-line slot evaluation).
struct RxnCtx {
    double T, logT, invT, m, mC;
};

// Rates of reaction slot s; with deriv, also the pieces of its derivative.
// Out of line and shared by the RHS and the Jacobian: one copy of the reaction
// code in the instruction cache (a separate q-only copy for the RHS measured
// slower: the kernel is bound by instruction fetch).  C_off / G_off:
// shared-memory byte offsets of the concentrations and -g/RT (index N holds the
// padding entries).
template <class MT>
__device__ __noinline__ RxnOut rxn_slot(int s, const RxnCtx c, unsigned C_off, unsigned G_off, int deriv) {
    const DevMech& M = mech<MT>();
    const double* C = smem_at<double>(C_off);
    const double* G = smem_at<double>(G_off);
    RxnOut o;
    o.q = 0.0; o.kf = 0.0; o.kr = 0.0; o.Rf = 0.0; o.Rr = 0.0; o.phi = 1.0; o.thd = 0.0;
    o.dphi_dthd = 0.0; o.dphi_dT = 0.0; o.dlnkf_dT = 0.0;
    const uint2 fw = __ldg(M.fac + s);   // factor species, flags, dnu in one word
    const int fl = (fw.y >> 16) & 511;
    if (!(fl & kFlagActive)) return o;
    static_assert(MT::N < 256, "packed reaction words hold species as bytes");
    const int r0 = fw.x & 255, r1 = (fw.x >> 8) & 255, r2 = (fw.x >> 16) & 255;
    const double2 bE = __ldg(M.bEa + s), lP = __ldg(M.lAP + s);
    const double b = bE.x, EaR = bE.y;
    double lkf = lP.x + b * c.logT - EaR * c.invT;
    if (deriv) o.dlnkf_dT = (b + EaR * c.invT) * c.invT;
    if constexpr (MT::PLOG) {
        if (fl & kFlagPlog) {   // P = m R T
            const PlogOut pl = plog_rate<MT>(s, c.T, c.logT, c.invT, ode_log(c.m * kRU * c.T));
            lkf = pl.lnk;
            o.dlnkf_dT = pl.dlnk_dT;
        }
    }
    const bool constk = fl & kFlagConstK;
    double kf;
    if (fl & kFlagRev) {
        const int p0 = fw.x >> 24, p1 = fw.y & 255, p2 = (fw.y >> 8) & 255;
        const int dnu = (int)(fw.y >> 25) - kFacDnuBias;
        const double sg = (G[p0] + G[p1] + G[p2]) - (G[r0] + G[r1] + G[r2]);
        const double lnKc = sg - dnu * c.logT + lP.y;
        double kr;
        if constexpr (MT::N >= kPairedExpMinN) {   // kf's and kr's exponentials in one call
            const Exp2 e = ode_exp2(lkf, constk ? -lnKc : lkf - lnKc);
            kf = constk ? __ldg(M.Aconst + s) : e.a;
            kr = constk ? __ldg(M.Aconst + s) * e.b : e.b;
        } else {
            kf = constk ? __ldg(M.Aconst + s) : ode_exp(lkf);
            kr = constk ? __ldg(M.Aconst + s) * ode_exp(-lnKc) : ode_exp(lkf - lnKc);
        }
        o.kr = kr;
        o.Rr = kr * ((C[p0] * C[p1]) * C[p2]);
    } else {
        kf = constk ? __ldg(M.Aconst + s) : ode_exp(lkf);
    }
    o.kf = kf;
    o.Rf = kf * ((C[r0] * C[r1]) * C[r2]);
    const int type = fl & kFlagTypeMask;
    if (type != 0) {
        double thd;
        if (fl & kFlagCatalyst) {
            thd = c.mC + C[__ldg(M.cat_sp + s)];   // m - sum_{k != s} C_k
        } else {
            thd = c.m;
            const int off = __ldg(M.tb_off + s), len = __ldg(M.tb_len + s);
#pragma unroll 1
            for (int t = 0; t < len; ++t) thd += __ldg(M.tb_alpha + off + t) * C[__ldg(M.tb_sp + off + t)];
        }
        o.thd = thd;
        if (type == 1) {
            o.phi = thd;
            o.dphi_dthd = 1.0;
        } else {
            const FallOut f = falloff<MT>(s, fl, c.T, c.logT, c.invT, kf, thd, deriv);
            o.phi = f.phi;
            o.dphi_dthd = f.dphi_dthd;
            o.dphi_dT = f.dphi_dT;
        }
    }
    o.q = (o.Rf - o.Rr) * o.phi;
    return o;
}

__device__ __forceinline__ RxnCtx rxn_ctx(const CellThermo& c) { return RxnCtx{c.T, c.logT, c.invT, c.m, c.mC}; }

// ---- One cell on a CTA's four warps (mechanisms of kWideN+ unknowns).
// Their Newton matrix fills an SM's shared memory, so one cell runs per SM and
// a single warp would leave three of the SM's four schedulers idle.  Warp 0
// runs the integration; warps 1-3 ("helpers") take a share of its two widest
// loops -- the reaction groups of the RHS and the trailing update of the
// blocked LU -- when warp 0 posts them.  Each share writes disjoint outputs
// with the same operations a single warp would use, so results do not depend
// on whether helpers serve.  The hand-off goes through a shared-memory control
// block with bounded polling waits (no hardware barrier a warp could miss).
//
// Recovery when a wait runs out:
//   * warp 0's wait for a command's completion (join) runs out: warp 0 keeps
//     waiting, bounded again (drain), for the late shares.  If they arrive, the
//     command's outputs are complete and the cell goes on unchanged; the helpers
//     are released (kCmdExit) and warp 0 works alone for the rest of the launch.
//   * the drain runs out too: a late helper might still write into warp 0's
//     shared memory at any time, so the CTA is poisoned: the current cell and
//     every later cell the CTA claims fail with CV_ERR_FAILURE, later cells
//     without being integrated (their state is left as given).
//   * a helper's wait for the next command runs out (warp 0 silent for ~10 s):
//     the helper leaves; warp 0's next join and drain then run out (poisoned).
constexpr int kWideN = 192;
constexpr int kHelperWarps = 3;
enum { kCmdRhs = 1, kCmdLu = 2, kCmdExit = 3 };
// Default limits in SM clock cycles: a helper waits for the next command at
// most ~10 s (warp 0 works alone between commands: Jacobian, step control);
// warp 0 waits for a command's completion ~2 s, then ~2 s more for late shares
// (a share takes microseconds).
constexpr long long kHelperIdleCycles = 20000000000LL;
constexpr long long kJoinCycles = 4000000000LL;
constexpr long long kDrainCycles = 4000000000LL;

struct HelperCtl {
    unsigned seq;      // commands posted
    unsigned done;     // helper completions (kHelperWarps per command)
    unsigned posted;   // warp 0's count of commands posted
    int cmd;
    int nhelpers;      // kHelperWarps while the helpers serve, else 0
    int err;           // a bounded wait ran out (join or helper idle)
    int poisoned;      // a drain ran out: late helper writes possible, fail every cell
    int exit_posted;   // kCmdExit posted (helpers released)
    int k0, kend;      // kCmdLu: the LU panel
    unsigned A_off, C_off, G_off, q_off;
    long long join_cycles, drain_cycles, idle_cycles;   // wait limits of this launch
    RxnCtx rc;         // kCmdRhs: the cell's reaction context
};
// One per CTA, in the kernels of the mechanisms that use it.
__shared__ HelperCtl g_helper_ctl;

__device__ __forceinline__ unsigned ld_volatile(const unsigned* p) { return *(const volatile unsigned*)p; }

// Warp 0: post a command whose arguments it has written (every lane's earlier
// shared-memory writes are made visible to the helpers first).
__device__ __forceinline__ void helpers_post(HelperCtl* h, int cmd, int lane) {
    __threadfence_block();
    __syncwarp();
    if (lane == 0) {
        h->cmd = cmd;
        h->posted += 1;
        __threadfence_block();
        atomicAdd(&h->seq, 1u);
    }
    __syncwarp();
}

// Warp 0: wait, at most `limit` cycles, until the helpers have reported
// `expected` completions.  Every lane returns the same answer.
__device__ __forceinline__ bool helpers_wait_done(HelperCtl* h, unsigned expected, long long limit) {
    const long long t0 = clock64();
    bool ok = true;
    while (ld_volatile(&h->done) < expected) {
        if (clock64() - t0 > limit) { ok = false; break; }
    }
    __threadfence_block();
    return __all_sync(kFull, ok);
}

// Warp 0: wait until the helpers have finished every posted command.  If the
// join runs out, the drain waits for the late shares: when they arrive the
// outputs are complete and the helpers are released (warp 0 alone from here
// on); when the drain runs out too the CTA is poisoned (see above).  Either
// way nhelpers becomes 0 and err is set.
__device__ __noinline__ void helpers_join(HelperCtl* h, int lane) {
    const unsigned expected = kHelperWarps * h->posted;
    if (helpers_wait_done(h, expected, h->join_cycles)) return;
    const bool drained = helpers_wait_done(h, expected, h->drain_cycles);
    if (lane == 0) {
        h->err = 1;
        h->nhelpers = 0;
        if (!drained) h->poisoned = 1;
    }
    __syncwarp();
    // release the helpers (a late one leaves once it has finished its share)
    helpers_post(h, kCmdExit, lane);
    if (lane == 0) h->exit_posted = 1;
    __syncwarp();
}

// Rates of progress of the reaction groups g = g0, g0 + dg, ... into the
// shared rate array at byte offset q_off.
template <class MT>
__device__ __forceinline__ void rhs_groups(const RxnCtx rc, unsigned C_off, unsigned G_off, unsigned q_off, int g0,
                                           int dg, int lane) {
    static_assert(MT::G == 32, "helper warps serve one cell per warp");
    double* q = smem_at<double>(q_off);
#pragma unroll 1
    for (int g = g0; g < MT::NG; g += dg) {
        const int s = 32 * g + lane;
        q[s] = rxn_slot<MT>(s, rc, C_off, G_off, 0).q;
    }
}

// The RHS's reaction groups on warp 0, with the CTA's helper warps taking every
// (kHelperWarps + 1)-th group from their own index when they serve it.
template <class MT>
__device__ __forceinline__ void rhs_groups_forked(const RxnCtx rc, unsigned C_off, unsigned G_off, unsigned q_off,
                                                  int lane) {
    HelperCtl* h = &g_helper_ctl;
    if (h->nhelpers != kHelperWarps) {
        rhs_groups<MT>(rc, C_off, G_off, q_off, 0, 1, lane);
        return;
    }
    if (lane == 0) {
        h->rc = rc;
        h->C_off = C_off;
        h->G_off = G_off;
        h->q_off = q_off;
    }
    helpers_post(h, kCmdRhs, lane);
    rhs_groups<MT>(rc, C_off, G_off, q_off, 0, kHelperWarps + 1, lane);
    // after a drained join every share is complete; a poisoned CTA fails the cell
    helpers_join(h, lane);
}

// Balanced gather: out[s] = sum over species (lane + G s)'s (slot, nu) pairs of
// nu * src[slot]; src is the shared-memory array at byte offset src_off, or,
// with kGlobal, the global array gsrc.  Unit partial sums go through the
// chemistry scratch's part[].  Out of line: the RHS and the Jacobian share it.
template <class MT, bool kGlobal>
__device__ __noinline__ Vec<MT::NS> gather(const double* gsrc, unsigned src_off, unsigned chem_off, int lane) {
    constexpr int G = MT::G, LISTS = 32 / G;   // the tables deal the units to 32 lists
    const DevMech& M = mech<MT>();
    const double* src = kGlobal ? gsrc : smem_at<double>(src_off);
    ChemSmem<MT>* sm = smem_at<ChemSmem<MT>>(chem_off);
    double acc[LISTS];
#pragma unroll
    for (int r = 0; r < LISTS; ++r) acc[r] = 0.0;
    const int gmax = M.gmax;
    const int* gw = M.gword + lane;
#pragma unroll 2
    for (int e = 0; e < gmax; ++e) {
#pragma unroll
        for (int r = 0; r < LISTS; ++r) {   // lane's lists: lane, lane + G, ...
            const int w = __ldg(gw + 32 * e + G * r);
            double nu = (double)(((w >> 11) & 31) - 16);
            if constexpr (MT::NU_DEN != 1) nu *= 1.0 / MT::NU_DEN;   // exact: a power of two
            acc[r] += nu * src[w & 2047];
            const bool last = (w >> 16) & 1;
            if (last) sm->part[w >> 17] = acc[r];
            acc[r] = last ? 0.0 : acc[r];
        }
    }
    __syncwarp(gmask<G>());
    Vec<MT::NS> out;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        double v = 0.0;
        if (i < MT::N) {
            const int u0 = __ldg(M.unit_off + i), u1 = __ldg(M.unit_off + i + 1);
            for (int u = u0; u < u1; ++u) v += sm->part[u];
        }
        out.v[s] = v;
    }
    __syncwarp(gmask<G>());
    return out;
}

// f = dy/dt for the warp's cell.  y, f: lane elements in internal order.
template <class MT>
__device__ __noinline__ Vec<MT::NS> warp_rhs(double P, const Vec<MT::NS> yv, unsigned chem_off, int lane) {
    constexpr int N = MT::N, G = MT::G;
    const DevMech& M = mech<MT>();
    ChemSmem<MT>* sm = smem_at<ChemSmem<MT>>(chem_off);
    double y[MT::NS];
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) y[s] = yv.v[s];
    double Yk[MT::NS], cpR[MT::NS], hRT[MT::NS], dcpR[MT::NS];
    const CellThermo c = species_phase<MT>(M, P, y, sm, lane, Yk, cpR, hRT, dcpR);
    const RxnCtx rc = rxn_ctx(c);
    const unsigned C_off = smem_off(sm->C), G_off = smem_off(sm->G);
    if constexpr (MT::N >= kWideN) {
        rhs_groups_forked<MT>(rc, C_off, G_off, smem_off(sm->q), lane);
    } else {
#pragma unroll 1
        for (int g = 0; g < MT::NG; ++g) {
            const int s = G * g + lane;
            sm->q[s] = rxn_slot<MT>(s, rc, C_off, G_off, 0).q;
        }
    }
    __syncwarp(gmask<G>());
    double om[MT::NS];
    {
        const Vec<MT::NS> g = gather<MT, false>(nullptr, smem_off(sm->q), chem_off, lane);
#pragma unroll
        for (int s = 0; s < MT::NS; ++s) om[s] = g.v[s];
    }
    // energy equation: enthalpy and cp at constant pressure; internal energy
    // u = h - R T / W_k and cv = cp - R / W_k at constant volume
    double qsum = 0.0, cpsum = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        if (i < N) {
            if constexpr (!MT::CONV) {
                qsum += om[s] * hRT[s];
                cpsum += cpR[s] * Yk[s] * __ldg(M.inv_mw + i);
            } else {
                qsum += om[s] * (hRT[s] - 1.0);
                cpsum += (cpR[s] - 1.0) * Yk[s] * __ldg(M.inv_mw + i);
            }
        }
    }
    const double Q = kRU * c.T * group_sum<G>(qsum);      // sum_k w_k e_k W_k   [W/m^3]
    const double cp_avg = kRU * group_sum<G>(cpsum);       // cp or cv [J/kg/K]
    const double dTdt = ode_div(-Q, c.rho * cp_avg);
    const double inv_rho = ode_div(1.0, c.rho);
    Vec<MT::NS> fv;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + G * s;
        if (i < N - 1) fv.v[s] = om[s] * (__ldg(M.mw + i) * inv_rho);
        else if (i == N - 1) fv.v[s] = dTdt;
        else fv.v[s] = 0.0;
    }
    __syncwarp(gmask<G>());   // shared scratch is reused by the next evaluation
    return fv;
}

// Analytic Jacobian J = d f / d y (internal order) into A (row-major, lda MT::LDA),
// in precision LinT.  Chain rule through concentrations and the closure species:
//   dC_i/dY_j = rho/W_i (delta_ij - delta_{i,N-1}) - C_i Wbar (1/W_j - 1/W_{N-1})
// at constant pressure (rho = P Wbar / (R T)); at constant volume (MT::CONV, rho
// fixed) the second term is absent, C does not depend on T, and the total
// concentration m = sum_i C_i (third bodies, PLOG pressure) adds
// dw/dm (1/W_j - 1/W_{N-1}) rho to every column.
// Each reaction slot's derivative pieces (d q / d C of its reactant and product
// factors and its third-body term) go to dpiece (global scratch: the space the
// Jacobian is saved into afterwards); the species-space block is then summed
// from them by the Jacobian gather, each output element by one lane.
template <class MT, class LinT>
__device__ __noinline__ void warp_jac(double P, const Vec<MT::NS> yv, unsigned A_off, unsigned chem_off,
                                      JacScratch<MT>* js, LinT* dpiece, int lane) {
    constexpr int N = MT::N, LDA = MT::LDA, NS = MT::NS, G = MT::G;
    static_assert(3 * N <= MT::NSLOT, "the per-species work [3][N] reuses the rate buffer q[NSLOT]");
    const unsigned gm = gmask<G>();
    const DevMech& M = mech<MT>();
    LinT* A = smem_at<LinT>(A_off);
    ChemSmem<MT>* sm = smem_at<ChemSmem<MT>>(chem_off);
    double y[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) y[s] = yv.v[s];
    double Yk[NS], cpR[NS], hRT[NS], dcpR[NS];
#pragma unroll 2
    for (int e = lane; e < N * LDA; e += G) A[e] = LinT(0);
    const CellThermo c = species_phase<MT>(M, P, y, sm, lane, Yk, cpR, hRT, dcpR, js->H);
    constexpr bool conv = MT::CONV;   // constant volume (see species_phase)
    constexpr int ns = MT::NSLOT;
    const RxnCtx rc = rxn_ctx(c);
    const unsigned C_off = smem_off(sm->C), G_off = smem_off(sm->G);
#pragma unroll 1
    for (int g = 0; g < MT::NG; ++g) {
        const int s = G * g + lane;
        const RxnOut o = rxn_slot<MT>(s, rc, C_off, G_off, 1);
        const int fl = __ldg(M.flags + s);
        double dqdT = 0.0, sr = 0.0, thd_term = 0.0;
        double dRf[3] = {0.0, 0.0, 0.0}, dRr[3] = {0.0, 0.0, 0.0};
        int rf[3], pf[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            rf[a] = __ldg(M.rf + a * ns + s);
            pf[a] = __ldg(M.pf + a * ns + s);
        }
        if (fl & kFlagActive) {
            // d ln kr / dT = d ln kf / dT - (sum nu h/RT - dnu) / T
            double dlnkr = 0.0;
            if (fl & kFlagRev) {
                double dH = 0.0;
#pragma unroll
                for (int e = 0; e < kJRow; ++e) {
                    const int k = __ldg(M.jrow + e * ns + s);
                    if (k >= 0) dH += __ldg(M.jnu + e * ns + s) * js->H[k];
                }
                dlnkr = o.dlnkf_dT - (dH - (double)__ldg(M.dnu + s)) * c.invT;
            }
            const double R = o.Rf - o.Rr;
            const double dR_dT = o.Rf * o.dlnkf_dT - o.Rr * dlnkr;
            int ordf = 0, ordr = 0;
#pragma unroll
            for (int a = 0; a < 3; ++a) { ordf += (rf[a] < N); ordr += (pf[a] < N); }
            const double Sr = o.phi * (ordf * o.Rf - ordr * o.Rr);
            thd_term = R * o.dphi_dthd;
            if constexpr (!conv) {
                // C = rho Y / W with rho = P W / (R T): C and m fall as 1/T
                dqdT = o.phi * dR_dT + R * o.dphi_dT - (Sr + thd_term * o.thd) * c.invT;
                sr = Sr + thd_term * (o.thd - c.m);          // sum_i dq/dC_i C_i
            } else {
                // C fixed in T; m = sum_i C_i, and P = m R T moves PLOG rates
                // with T and with every C_i: sr = dq/dm
                dqdT = o.phi * dR_dT + R * o.dphi_dT;
                sr = thd_term;
                if constexpr (MT::PLOG) {
                    if (fl & kFlagPlog) {
                        const PlogOut pl = plog_rate<MT>(s, c.T, c.logT, c.invT, ode_log(c.m * kRU * c.T));
                        dqdT += o.q * pl.dlnk_dlnP * c.invT;
                        sr += ode_div(o.q * pl.dlnk_dlnP, c.m);
                    }
                }
            }
            const double* C = sm->C;
            dRf[0] = o.phi * o.kf * (C[rf[1]] * C[rf[2]]);
            dRf[1] = o.phi * o.kf * (C[rf[0]] * C[rf[2]]);
            dRf[2] = o.phi * o.kf * (C[rf[0]] * C[rf[1]]);
            dRr[0] = o.phi * o.kr * (C[pf[1]] * C[pf[2]]);
            dRr[1] = o.phi * o.kr * (C[pf[0]] * C[pf[2]]);
            dRr[2] = o.phi * o.kr * (C[pf[0]] * C[pf[1]]);
        }
        sm->q[s] = o.q;
        js->dqdT[s] = dqdT;
        js->sr[s] = sr;
        // the slot's derivative pieces (every slot, inactive ones as 0, so the
        // gather's padding entries read finite values)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            dpiece[a * ns + s] = (LinT)dRf[a];
            dpiece[(3 + a) * ns + s] = (LinT)dRr[a];
        }
        dpiece[6 * ns + s] = (LinT)thd_term;
    }
    __syncwarp(gm);
    // species-space block d omega_k / d C_j = sum_r nu_kr d q_r / d C_j by the
    // Jacobian gather (mech_dev.h): every output element is summed by one lane
    // in a fixed order and stored once -- no atomics, no conflicts between
    // lanes that share a row or column (a third-body reaction reaches a whole
    // row; most reactions share H, O or OH), results independent of scheduling
    {
        constexpr int LISTS = 32 / G;
        const int jgmax = M.jgmax;
        double acc[LISTS];
#pragma unroll
        for (int r = 0; r < LISTS; ++r) acc[r] = 0.0;
#pragma unroll 2
        for (int e = 0; e < jgmax; ++e) {
#pragma unroll
            for (int r = 0; r < LISTS; ++r) {
                const int x = 32 * e + lane + G * r;
                const int w = __ldg(M.jword + x);
                const double cf = __ldg(M.jcoef + x);
                acc[r] += cf * (double)dpiece[((w >> 11) & 7) * ns + (w & 2047)];
                const bool last = (w >> 14) & 1;
                if (last) A[w >> 15] = (LinT)acc[r];
                acc[r] = last ? 0.0 : acc[r];
            }
        }
    }
    __syncwarp(gm);
    // per-species totals (fixed-order gathers)
    const Vec<NS> wv = gather<MT, false>(nullptr, smem_off(sm->q), chem_off, lane);
    const Vec<NS> dwv = gather<MT, true>(js->dqdT, 0u, chem_off, lane);
    const Vec<NS> skv = gather<MT, true>(js->sr, 0u, chem_off, lane);
    const double (&w)[NS] = wv.v;
    const double (&dw)[NS] = dwv.v;
    const double (&sk)[NS] = skv.v;
    double* spw = sm->q;   // per-species work reuses the rate buffer: [3][N]
    const double inv_rho = ode_div(1.0, c.rho);
    const double iWN = __ldg(M.inv_mw + N - 1);
    const double RT = kRU * c.T;
    double dfdT[NS];
    double qsum = 0.0, cpsum = 0.0, Ssum2 = 0.0, Ssum3 = 0.0, accTT = 0.0, dcpsum = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int i = lane + G * s;
        dfdT[s] = 0.0;
        if (i < N) {
            const double Wi = __ldg(M.mw + i), iWi = __ldg(M.inv_mw + i);
            const double Wr = Wi * inv_rho;
            const double fk = w[s] * Wr;
            // constant pressure: energy h, heat capacity cp, f = w W / rho(T, Y);
            // constant volume: u = h - R T / W_k, cv = cp - R / W_k, rho fixed,
            // and sk holds dw/dm (m = sum_i C_i) instead of sum_i dw/dC_i C_i
            dfdT[s] = conv ? Wr * dw[s] : Wr * (dw[s] + w[s] * c.invT);
            const double hW = conv ? RT * (hRT[s] - 1.0) : RT * hRT[s];                // e_k W_k  [J/kmol]
            const double hk = hW * iWi;                                                 // J/kg
            const double cpk = conv ? kRU * (cpR[s] - 1.0) * iWi : kRU * cpR[s] * iWi;  // J/kg/K
            const double X = conv ? sk[s] : (c.mw_avg * inv_rho) * (w[s] - sk[s]);
            spw[0 * N + i] = hW;
            spw[1 * N + i] = cpk;
            spw[2 * N + i] = X;
            qsum += hk * fk;
            cpsum += cpk * Yk[s];
            Ssum2 += hW * (double)A[i * LDA + (N - 1)];
            Ssum3 += hW * X;
            accTT += cpk * fk + hk * dfdT[s];
            dcpsum += Yk[s] * kRU * dcpR[s] * iWi;
        }
    }
    const double inv_cp = ode_div(1.0, group_sum<G>(cpsum));
    const double fT = -group_sum<G>(qsum) * inv_cp;
    const double S2 = group_sum<G>(Ssum2);
    const double S3 = group_sum<G>(Ssum3);
    const double JTT = -(group_sum<G>(accTT) + fT * group_sum<G>(dcpsum)) * inv_cp;
    __syncwarp(gm);
    // T row (state row N-1): lane owns columns j < N-1
    double trow[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int j = lane + G * s;
        trow[s] = 0.0;
        if (j < N - 1) {
            double S1 = 0.0;
#pragma unroll 4
            for (int k = 0; k < N; ++k) S1 += spw[k] * (double)A[k * LDA + j];
            const double iWj = __ldg(M.inv_mw + j);
            trow[s] = -(S1 * iWj - S2 * iWN + (iWj - iWN) * S3 + fT * (spw[N + j] - spw[N + N - 1])) * inv_cp;
        }
    }
    __syncwarp(gm);
    // species rows k < N-1 (lane owns rows), then the T column; each row goes
    // in batches of 8 columns whose loads are issued before their stores
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int k = lane + G * s;
        if (k < N - 1) {
            LinT* row = A + k * LDA;
            const double Wk = __ldg(M.mw + k);
            const double cN = (double)row[N - 1] * iWN;
            const double X = spw[2 * N + k];
            constexpr int kB = 8;
#pragma unroll 1
            for (int j0 = 0; j0 < N - 1; j0 += kB) {
                LinT a[kB];
                double iw[kB];
#pragma unroll
                for (int r = 0; r < kB; ++r) {
                    const int j = j0 + r < N - 1 ? j0 + r : N - 2;
                    a[r] = row[j];
                    iw[r] = __ldg(M.inv_mw + j);
                }
#pragma unroll
                for (int r = 0; r < kB; ++r)
                    if (j0 + r < N - 1) row[j0 + r] = (LinT)(Wk * ((double)a[r] * iw[r] - cN + X * (iw[r] - iWN)));
            }
            row[N - 1] = (LinT)dfdT[s];
        }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int j = lane + G * s;
        if (j < N - 1) A[(N - 1) * LDA + j] = (LinT)trow[s];
    }
    if (lane == 0) A[(N - 1) * LDA + (N - 1)] = (LinT)JTT;
    __syncwarp(gm);
}

}  // namespace b200
