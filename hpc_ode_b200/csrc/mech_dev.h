// Device-side mechanism description and its host packing.
//
// The generated tables (csrc/mech/<name>_mech.h, written by
// hpc_ode_b200/mechanism.py with the pyJac conventions of the reference's
// src/Mechanism/CPU kernels) are repacked on the host into the layout the warp
// kernels read:
//   * species arrays (molecular weights, NASA-7 coefficients), index k;
//   * reaction "slots": reactions sorted by kind (elementary, third-body,
//     catalyst third-body, Lindemann, Troe, pressure-dependent Arrhenius) and
//     padded to groups of 32 so that
//     the 32 lanes of a warp evaluate 32 reactions of one kind with the same
//     instruction stream.  Every field is a separate array indexed by slot,
//     so one group's load is one coalesced 32-wide access;
//   * a species-major gather list (slot, net stoichiometry) so that each lane
//     sums the production rate of its own species in a fixed order (no
//     atomics: results do not depend on scheduling).
#pragma once

#include <stdint.h>
#if !defined(__CUDACC__) && !defined(__VECTOR_TYPES_H__)
// host-only builds without the CUDA headers (the CPU packing checks): the two
// vector types DevMech's pointers name
struct uint2 {
    unsigned int x, y;
};
struct alignas(16) double2 {
    double x, y;
};
#endif

#include <algorithm>
#include <map>
#include <cmath>
#include <string>
#include <vector>

namespace b200 {

constexpr int kFlagTypeMask = 3;     // 0 elementary, 1 third-body, 2 Lindemann, 3 Troe
constexpr int kFlagRev = 1 << 2;     // reversible
constexpr int kFlagConstK = 1 << 3;  // kf = A (b = 0, Ea = 0)
constexpr int kFlagActive = 1 << 4;  // real reaction (0 for padding slots)
constexpr int kFlagT2 = 1 << 5;      // Troe with T2 term
constexpr int kFlagConstK0 = 1 << 6; // k0 = A0
constexpr int kFlagCatalyst = 1 << 7;  // third body is one species s: [M] = m - sum(C) + C_s
constexpr int kFlagPlog = 1 << 8;    // pressure-dependent Arrhenius (type 0): kf from the PLOG tables

// Packed reaction word (uint2 per slot, read by the RHS's reaction loop in one
// load): x = rf0 | rf1 << 8 | rf2 << 16 | pf0 << 24, y = pf1 | pf2 << 8 |
// flags << 16 (9 bits) | (dnu + 64) << 25; factor species are < 256 (the
// padding factor is N), dnu in [-64, 63].  The RHS reads (b, EaR) and
// (logA, lnPfac) as two double2 loads.
constexpr int kFacDnuBias = 64;

// Species with nonzero net stoichiometry per reaction (rows of jrow / jnu).
constexpr int kJRow = 8;

// Balanced species gather: the (species, reaction) pairs are cut into units of
// at most kGatherUnit entries, and units are dealt to the 32 lanes so each lane
// sums about the same number of entries.  Entry word (int32):
//   bits 0-10  reaction slot            bits 11-15 net stoichiometry x nu_den + 16
//   bit  16    last entry of its unit   bits 17-31 unit index
// (nu_den = 1, or 2 / 4 for mechanisms with fractional product coefficients).
constexpr int kGatherUnit = 24;

// Jacobian gather (the species-space block of the analytic Jacobian,
// d omega_k / d C_j = sum over reactions r of nu_kr d q_r / d C_j): one list
// entry per (output element (k, j), reaction slot, derivative piece), the
// entries of each output element contiguous and in a fixed order, output
// elements dealt longest-first to the 32 lists.  Entry word (int32):
//   bits 0-10  reaction slot     bits 11-13 derivative piece (0-2: d(forward
//   rate)/d(reactant factor a), 3-5: d(reverse rate)/d(product factor a), 6: the
//   third-body term)     bit 14  last entry of its output element
//   bits 15-31 output element k * LDA + j
// with a double coefficient per entry (nu_kr, -nu_kr, nu_kr * alpha_j or
// -nu_kr for a catalyst's "all other species").
constexpr int kJacPieces = 7;

// Pointers into one device allocation (all arrays contiguous).
struct DevMech {
    int nsp, nrxn, nslot, ntb, nent;
    const double* mw;       // [nsp]
    const double* inv_mw;   // [nsp]
    const double* tmid;     // [nsp]
    const double* nasa;     // [nsp][14]: low range a0..a6, high range a0..a6
    const double* nasa_sk;  // [14][nsp]: the same, species innermost (lane-coalesced)
    // reaction slots [nslot]
    const double* logA;
    const double* b;
    const double* EaR;
    const double* Aconst;
    const double* lnPfac;   // dnu * ln(Patm / R)
    const double* logA0;
    const double* b0;
    const double* EaR0;
    const double* A0const;
    const double* troe_a;
    const double* troe_iT3;
    const double* troe_iT1;
    const double* troe_T2;
    const uint2* fac;       // [nslot] packed factor species, flags, dnu (see kFacDnuBias)
    const double2* bEa;     // [nslot] (b, EaR)
    const double2* lAP;     // [nslot] (logA, lnPfac)
    const int* flags;
    const int* rf;          // [3][nslot] reactant factor species (nsp = dummy: C = 1, G = 0)
    const int* pf;          // [3][nslot] product factor species
    const int* dnu;         // [nslot]
    const int* tb_off;      // [nslot]
    const int* tb_len;      // [nslot]
    const int* tb_sp;       // [ntb]
    const double* tb_alpha; // [ntb]
    const int* jrow;        // [kJRow][nslot] species with nonzero net stoichiometry (-1 = none)
    const double* jnu;      // [kJRow][nslot] their net stoichiometric coefficient
    const int* sp_off;      // [nsp + 1]
    const int* sp_slot;     // [nent]
    const int* sp_nu;       // [nent] net stoichiometry x nu_den
    const int* cat_sp;      // [nslot] catalyst species (or -1)
    int gmax;               // entries per lane in the balanced gather
    int nunit;              // gather units
    const int* gword;       // [gmax][32] entry words, lane innermost (coalesced)
    const int* unit_off;    // [nsp + 1] units of each species (contiguous, in order)
    // PLOG slots: levels plog_lev0[s] .. plog_lev0[s] + plog_nlev[s] - 1 (ln P
    // ascending); level l's Arrhenius terms plog_toff[l] .. plog_toff[l + 1] - 1
    const int* plog_lev0;   // [nslot]
    const int* plog_nlev;   // [nslot]
    const double* plog_lnP; // [nlev]
    const int* plog_toff;   // [nlev + 1]
    const double* plog_A;   // [nterm]
    const double* plog_logA;
    const double* plog_b;
    const double* plog_EaR;
    const int* inert;       // [nsp] 1: no reaction changes species k (its rows of J are zero)
    int jgmax;              // entries per list of the Jacobian gather
    const int* jword;       // [jgmax][32] Jacobian gather words, list innermost
    const double* jcoef;    // [jgmax][32] their coefficients
};

// Host image of DevMech: one byte buffer plus offsets, copied to the device once.
struct HostMech {
    std::string name;
    int nsp = 0, nrxn = 0, nslot = 0, ntb = 0, nent = 0;
    std::vector<std::string> species;
    std::vector<double> mw;
    std::vector<int> slot_rxn;   // slot -> original reaction index (-1 = padding)
    std::vector<unsigned char> blob;
    // byte offsets of each array inside blob
    size_t o_mw, o_inv_mw, o_tmid, o_nasa, o_logA, o_b, o_EaR, o_Aconst, o_lnPfac, o_logA0, o_b0,
        o_EaR0, o_A0const, o_troe_a, o_troe_iT3, o_troe_iT1, o_troe_T2, o_flags, o_rf, o_pf,
        o_dnu, o_tb_off, o_tb_len, o_tb_sp, o_tb_alpha, o_jrow, o_jnu, o_sp_off, o_sp_slot,
        o_sp_nu, o_cat_sp, o_gword, o_unit_off, o_plog_lev0, o_plog_nlev, o_plog_lnP, o_plog_toff,
        o_plog_A, o_plog_logA, o_plog_b, o_plog_EaR, o_inert, o_jword, o_jcoef, o_fac, o_bEa, o_lAP,
        o_nasa_sk;
    int gmax = 0, nunit = 0, jgmax = 0, njent = 0;
    std::vector<int> jword;      // Jacobian gather (see kJacPieces), also kept for host checks
    std::vector<double> jcoef;

    DevMech bind(const unsigned char* base) const {
        DevMech d;
        d.nsp = nsp; d.nrxn = nrxn; d.nslot = nslot; d.ntb = ntb; d.nent = nent;
        d.mw = (const double*)(base + o_mw);
        d.inv_mw = (const double*)(base + o_inv_mw);
        d.tmid = (const double*)(base + o_tmid);
        d.nasa = (const double*)(base + o_nasa);
        d.nasa_sk = (const double*)(base + o_nasa_sk);
        d.logA = (const double*)(base + o_logA);
        d.b = (const double*)(base + o_b);
        d.EaR = (const double*)(base + o_EaR);
        d.Aconst = (const double*)(base + o_Aconst);
        d.lnPfac = (const double*)(base + o_lnPfac);
        d.logA0 = (const double*)(base + o_logA0);
        d.b0 = (const double*)(base + o_b0);
        d.EaR0 = (const double*)(base + o_EaR0);
        d.A0const = (const double*)(base + o_A0const);
        d.troe_a = (const double*)(base + o_troe_a);
        d.troe_iT3 = (const double*)(base + o_troe_iT3);
        d.troe_iT1 = (const double*)(base + o_troe_iT1);
        d.troe_T2 = (const double*)(base + o_troe_T2);
        d.fac = (const uint2*)(base + o_fac);
        d.bEa = (const double2*)(base + o_bEa);
        d.lAP = (const double2*)(base + o_lAP);
        d.flags = (const int*)(base + o_flags);
        d.rf = (const int*)(base + o_rf);
        d.pf = (const int*)(base + o_pf);
        d.dnu = (const int*)(base + o_dnu);
        d.tb_off = (const int*)(base + o_tb_off);
        d.tb_len = (const int*)(base + o_tb_len);
        d.tb_sp = (const int*)(base + o_tb_sp);
        d.tb_alpha = (const double*)(base + o_tb_alpha);
        d.jrow = (const int*)(base + o_jrow);
        d.jnu = (const double*)(base + o_jnu);
        d.sp_off = (const int*)(base + o_sp_off);
        d.sp_slot = (const int*)(base + o_sp_slot);
        d.sp_nu = (const int*)(base + o_sp_nu);
        d.cat_sp = (const int*)(base + o_cat_sp);
        d.gmax = gmax;
        d.nunit = nunit;
        d.gword = (const int*)(base + o_gword);
        d.unit_off = (const int*)(base + o_unit_off);
        d.plog_lev0 = (const int*)(base + o_plog_lev0);
        d.plog_nlev = (const int*)(base + o_plog_nlev);
        d.plog_lnP = (const double*)(base + o_plog_lnP);
        d.plog_toff = (const int*)(base + o_plog_toff);
        d.plog_A = (const double*)(base + o_plog_A);
        d.plog_logA = (const double*)(base + o_plog_logA);
        d.plog_b = (const double*)(base + o_plog_b);
        d.plog_EaR = (const double*)(base + o_plog_EaR);
        d.inert = (const int*)(base + o_inert);
        d.jgmax = jgmax;
        d.jword = (const int*)(base + o_jword);
        d.jcoef = (const double*)(base + o_jcoef);
        return d;
    }
};

// Raw generated tables of one mechanism (pointers to the static arrays).
struct GenTables {
    const char* name;
    int nsp, nrxn, maxp, ntb, nu_den, nplog_lev, nplog_term;
    const char* const* species_names;
    const double *mw, *tmid, *nasa_lo, *nasa_hi;
    const int *type, *rev;
    const double *A, *logA, *b, *EaR, *A0, *logA0, *b0, *EaR0, *troe;
    const int *troeT2, *reac_sp, *reac_nu, *prod_sp;
    const double* prod_nu;   // fractional only in irreversible reactions (multiples of 1 / nu_den)
    const int *tb_off, *tb_sp;
    const double* tb_alpha;
    const int* plog_off;     // [nrxn + 1] level range of each reaction
    const double* plog_lnP;
    const int* plog_term_off;
    const double *plog_A, *plog_logA, *plog_b, *plog_EaR;
};

// Build the packed image.  Returns an empty name on failure (message in err).
inline HostMech pack_mechanism(const GenTables& g, std::string* err) {
    HostMech h;
    const int n = g.nsp, nr = g.nrxn, P = g.maxp;
    h.name = g.name;
    h.nsp = n;
    h.nrxn = nr;
    for (int k = 0; k < n; ++k) h.species.push_back(g.species_names[k]);
    h.mw.assign(g.mw, g.mw + n);
    // ---- reaction order: group by kind so a warp group shares one code path
    auto kind = [&](int r) {
        int t = g.type[r];
        int tbl = g.tb_off[r + 1] - g.tb_off[r];
        if (t == 0) return g.rev[r] ? 1 : 0;
        if (t == 1) return tbl > 16 ? 3 : 2;
        return 2 + t;   // 4 Lindemann, 5 Troe, 6 PLOG
    };
    const int den = g.nu_den;
    auto scaled = [&](double nu, int* out) {   // nu * nu_den as an exact integer
        const double x = nu * den;
        *out = (int)std::lround(x);
        return std::fabs(x - *out) < 1e-9;
    };
    std::vector<int> order(nr);
    for (int r = 0; r < nr; ++r) order[r] = r;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return kind(a) < kind(b); });
    const int ns = ((nr + 32) / 32) * 32;   // at least one padding slot (q == 0)
    h.nslot = ns;
    h.slot_rxn.assign(ns, -1);
    for (int s = 0; s < nr; ++s) h.slot_rxn[s] = order[s];

    std::vector<double> logA(ns, 0), b(ns, 0), EaR(ns, 0), Ac(ns, 0), lnPfac(ns, 0), logA0(ns, 0),
        b0(ns, 0), EaR0(ns, 0), A0c(ns, 0), ta(ns, 0), tiT3(ns, 0), tiT1(ns, 0), tT2(ns, 0);
    std::vector<int> flags(ns, 0), rf(3 * ns, n), pf(3 * ns, n), dnu(ns, 0), tboff(ns, 0),
        tblen(ns, 0), jrow(kJRow * ns, -1), catsp(ns, -1), plev0(ns, 0), pnlev(ns, 0);
    std::vector<double> jnu(kJRow * ns, 0.0);
    std::vector<int> jnu_scaled(kJRow * ns, 0);
    std::vector<int> tbsp;
    std::vector<double> tbal;
    const double lnPR = std::log(101325.0 / 8314.4621);
    for (int s = 0; s < ns; ++s) {
        int r = h.slot_rxn[s];
        if (r < 0) continue;
        const bool plog = g.type[r] == 4;
        int fl = (plog ? 0 : g.type[r]) | kFlagActive;
        if (g.rev[r]) fl |= kFlagRev;
        if (plog) {
            fl |= kFlagPlog;
            plev0[s] = g.plog_off[r];
            pnlev[s] = g.plog_off[r + 1] - g.plog_off[r];
            if (pnlev[s] < 1) { *err = "PLOG reaction without pressure levels"; return HostMech(); }
        } else if (g.b[r] == 0.0 && g.EaR[r] == 0.0) {
            fl |= kFlagConstK;
        }
        if (g.b0[r] == 0.0 && g.EaR0[r] == 0.0) fl |= kFlagConstK0;
        if (g.troeT2[r]) fl |= kFlagT2;
        flags[s] = fl;
        logA[s] = g.logA[r]; b[s] = g.b[r]; EaR[s] = g.EaR[r]; Ac[s] = g.A[r];
        logA0[s] = g.logA0[r]; b0[s] = g.b0[r]; EaR0[s] = g.EaR0[r]; A0c[s] = g.A0[r];
        if (g.type[r] == 3) {   // (type 4, PLOG, carries no falloff data)
            ta[s] = g.troe[4 * r + 0];
            tiT3[s] = 1.0 / g.troe[4 * r + 1];
            tiT1[s] = 1.0 / g.troe[4 * r + 2];
            tT2[s] = g.troe[4 * r + 3];
        }
        int nf = 0, npf = 0, d = 0;
        for (int i = 0; i < P; ++i) {
            int sp = g.reac_sp[r * P + i];
            if (sp < 0) break;
            for (int q = 0; q < g.reac_nu[r * P + i]; ++q) {
                if (nf >= 3) { *err = "more than 3 reactant molecules"; return HostMech(); }
                rf[nf * ns + s] = sp; ++nf;
            }
            d -= g.reac_nu[r * P + i];
        }
        for (int i = 0; i < P; ++i) {
            int sp = g.prod_sp[r * P + i];
            if (sp < 0) break;
            // product factors only enter the reverse rate
            if (!g.rev[r]) continue;
            const double nu = g.prod_nu[r * P + i];
            if (nu != (double)(int)nu) { *err = "fractional product coefficient in a reversible reaction"; return HostMech(); }
            for (int q = 0; q < (int)nu; ++q) {
                if (npf >= 3) { *err = "more than 3 product molecules in a reversible reaction"; return HostMech(); }
                pf[npf * ns + s] = sp; ++npf;
            }
            d += (int)nu;
        }
        dnu[s] = g.rev[r] ? d : 0;   // enters Kc only
        lnPfac[s] = d * lnPR;
        tboff[s] = (int)tbsp.size();
        // a third-body list of all species but one with alpha = -1 is pyJac's
        // "single collider" form: keep it as a catalyst species instead
        const int tl = g.tb_off[r + 1] - g.tb_off[r];
        bool catalyst = (g.type[r] == 1 && tl == n - 1);
        if (catalyst) {
            std::vector<int> seen(n, 0);
            for (int t = g.tb_off[r]; t < g.tb_off[r + 1]; ++t) {
                if (g.tb_alpha[t] != -1.0) catalyst = false;
                seen[g.tb_sp[t]] = 1;
            }
            int miss = -1;
            for (int k = 0; k < n; ++k) if (!seen[k]) miss = k;
            if (catalyst && miss >= 0) {
                catsp[s] = miss;
                flags[s] |= kFlagCatalyst;
            } else {
                catalyst = false;
            }
        }
        if (!catalyst) {
            for (int t = g.tb_off[r]; t < g.tb_off[r + 1]; ++t) {
                tbsp.push_back(g.tb_sp[t]);
                tbal.push_back(g.tb_alpha[t]);
            }
        }
        tblen[s] = (int)tbsp.size() - tboff[s];
        // net stoichiometry rows
        std::vector<std::pair<int, double>> net;
        auto add = [&](int sp, double nu) {
            for (auto& e : net) if (e.first == sp) { e.second += nu; return; }
            net.push_back({sp, nu});
        };
        for (int i = 0; i < P; ++i) { int sp = g.reac_sp[r * P + i]; if (sp < 0) break; add(sp, -(double)g.reac_nu[r * P + i]); }
        for (int i = 0; i < P; ++i) { int sp = g.prod_sp[r * P + i]; if (sp < 0) break; add(sp, g.prod_nu[r * P + i]); }
        int nrow = 0;
        for (auto& e : net) {
            if (e.second == 0.0) continue;
            if (nrow >= kJRow) { *err = "more than 8 species in one reaction"; return HostMech(); }
            int sc = 0;
            if (!scaled(e.second, &sc) || sc < -16 || sc > 15) {
                *err = "net stoichiometric coefficient not encodable (multiple of 1/nu_den in [-16, 15] / nu_den)";
                return HostMech();
            }
            jrow[nrow * ns + s] = e.first;
            jnu[nrow * ns + s] = e.second;
            jnu_scaled[nrow * ns + s] = sc;
            ++nrow;
        }
    }
    if (tbsp.empty()) { tbsp.push_back(0); tbal.push_back(0.0); }
    h.ntb = (int)tbsp.size();
    // ---- species gather list in original reaction order
    std::vector<int> rxn_slot(nr);
    for (int s = 0; s < ns; ++s) if (h.slot_rxn[s] >= 0) rxn_slot[h.slot_rxn[s]] = s;
    std::vector<int> spoff(n + 1, 0), spslot, spnu;
    for (int k = 0; k < n; ++k) {
        spoff[k] = (int)spslot.size();
        for (int r = 0; r < nr; ++r) {
            int s = rxn_slot[r];
            for (int e = 0; e < kJRow; ++e)
                if (jrow[e * ns + s] == k) { spslot.push_back(s); spnu.push_back(jnu_scaled[e * ns + s]); }
        }
    }
    spoff[n] = (int)spslot.size();
    // balanced gather: cut each species' list into units, deal units to lanes
    struct Unit { int sp, e0, e1; };
    std::vector<Unit> units;
    std::vector<int> unitoff(n + 1, 0);
    for (int k = 0; k < n; ++k) {
        unitoff[k] = (int)units.size();
        for (int e = spoff[k]; e < spoff[k + 1]; e += kGatherUnit)
            units.push_back({k, e, std::min(e + kGatherUnit, spoff[k + 1])});
    }
    unitoff[n] = (int)units.size();
    std::vector<std::vector<int>> lane_units(32);
    std::vector<int> load(32, 0);
    std::vector<int> uorder(units.size());
    for (size_t u = 0; u < units.size(); ++u) uorder[u] = (int)u;
    std::stable_sort(uorder.begin(), uorder.end(), [&](int a, int b) {
        return (units[a].e1 - units[a].e0) > (units[b].e1 - units[b].e0);
    });
    for (int u : uorder) {   // longest-first onto the least-loaded lane
        int best = 0;
        for (int l = 1; l < 32; ++l) if (load[l] < load[best]) best = l;
        lane_units[best].push_back(u);
        load[best] += units[u].e1 - units[u].e0;
    }
    int gmax = 1;
    for (int l = 0; l < 32; ++l) gmax = std::max(gmax, load[l]);
    const int pad_slot = ns - 1 >= nr ? ns - 1 : -1;   // an inactive slot (q == 0)
    std::vector<int> gword((size_t)gmax * 32, 0);
    for (int l = 0; l < 32; ++l) {
        int e = 0;
        for (int u : lane_units[l]) {
            for (int x = units[u].e0; x < units[u].e1; ++x, ++e) {
                const int last = (x == units[u].e1 - 1) ? 1 : 0;
                gword[(size_t)e * 32 + l] = spslot[x] | ((spnu[x] + 16) << 11) | (last << 16) | (u << 17);
            }
        }
        for (; e < gmax; ++e) gword[(size_t)e * 32 + l] = (pad_slot >= 0 ? pad_slot : 0) | (16 << 11);
    }
    if (pad_slot < 0) { *err = "no padding slot for the gather (reaction count multiple of 32)"; return HostMech(); }
    if (ns > 2048 || (int)units.size() >= (1 << 15)) { *err = "mechanism too large for the gather encoding"; return HostMech(); }
    h.gmax = gmax;
    h.nunit = (int)units.size();
    // ---- Jacobian gather: entries per output element (k, j) in slot order
    {
        const int lda = (n % 2 == 0) ? n + 1 : n;
        struct JEnt { int slot, piece; double coef; };
        std::map<int, std::vector<JEnt>> outs;   // output element -> entries
        for (int s = 0; s < ns; ++s) {
            if (h.slot_rxn[s] < 0) continue;
            for (int e = 0; e < kJRow; ++e) {
                const int k = jrow[e * ns + s];
                if (k < 0) break;
                const double nu = jnu[e * ns + s];
                for (int a = 0; a < 3; ++a) {
                    if (rf[a * ns + s] < n) outs[k * lda + rf[a * ns + s]].push_back({s, a, nu});
                    if (pf[a * ns + s] < n) outs[k * lda + pf[a * ns + s]].push_back({s, 3 + a, -nu});
                }
                if (flags[s] & kFlagCatalyst) {
                    for (int j = 0; j < n; ++j)
                        if (j != catsp[s]) outs[k * lda + j].push_back({s, 6, -nu});
                } else if ((flags[s] & kFlagTypeMask) != 0) {
                    for (int t = tboff[s]; t < tboff[s] + tblen[s]; ++t)
                        outs[k * lda + tbsp[t]].push_back({s, 6, nu * tbal[t]});
                }
            }
        }
        std::vector<std::pair<int, const std::vector<JEnt>*>> ol;
        for (auto& kv : outs) ol.push_back({kv.first, &kv.second});
        std::vector<int> oord(ol.size());
        for (size_t i = 0; i < ol.size(); ++i) oord[i] = (int)i;
        std::stable_sort(oord.begin(), oord.end(), [&](int a, int b2) { return ol[a].second->size() > ol[b2].second->size(); });
        std::vector<std::vector<int>> lane_outs(32);
        std::vector<int> jload(32, 0);
        for (int o : oord) {   // longest-first onto the least-loaded list
            int best = 0;
            for (int l = 1; l < 32; ++l) if (jload[l] < jload[best]) best = l;
            lane_outs[best].push_back(o);
            jload[best] += (int)ol[o].second->size();
        }
        int jgmax = 1;
        for (int l = 0; l < 32; ++l) jgmax = std::max(jgmax, jload[l]);
        if ((long long)(n - 1) * lda + n - 1 >= (1LL << 17)) { *err = "mechanism too large for the Jacobian gather"; return HostMech(); }
        h.jword.assign((size_t)jgmax * 32, (ns - 1) | (6 << 11));   // padding: inactive slot, coefficient 0
        h.jcoef.assign((size_t)jgmax * 32, 0.0);
        int nj = 0;
        for (int l = 0; l < 32; ++l) {
            int e = 0;
            for (int o : lane_outs[l]) {
                const auto& v = *ol[o].second;
                for (size_t x = 0; x < v.size(); ++x, ++e) {
                    const int last = (x + 1 == v.size()) ? 1 : 0;
                    h.jword[(size_t)e * 32 + l] = v[x].slot | (v[x].piece << 11) | (last << 14) | (ol[o].first << 15);
                    h.jcoef[(size_t)e * 32 + l] = v[x].coef;
                    ++nj;
                }
            }
        }
        h.jgmax = jgmax;
        h.njent = nj;
    }
    if (spslot.empty()) { spslot.push_back(0); spnu.push_back(0); }
    h.nent = (int)spslot.size();
    // ---- species arrays
    std::vector<double> inv_mw(n), tmid(g.tmid, g.tmid + n), nasa(14 * n);
    for (int k = 0; k < n; ++k) {
        inv_mw[k] = 1.0 / g.mw[k];
        for (int i = 0; i < 7; ++i) {
            nasa[14 * k + i] = g.nasa_lo[7 * k + i];
            nasa[14 * k + 7 + i] = g.nasa_hi[7 * k + i];
        }
    }
    // ---- serialize
    auto put = [&](const void* src, size_t bytes) {
        size_t off = (h.blob.size() + 255) & ~size_t(255);
        h.blob.resize(off + bytes);
        std::copy((const unsigned char*)src, (const unsigned char*)src + bytes, h.blob.begin() + off);
        return off;
    };
#define PUTV(v) put((v).data(), (v).size() * sizeof((v)[0]))
    h.o_mw = put(g.mw, n * sizeof(double));
    h.o_inv_mw = PUTV(inv_mw);
    h.o_tmid = PUTV(tmid);
    h.o_nasa = PUTV(nasa);
    h.o_logA = PUTV(logA); h.o_b = PUTV(b); h.o_EaR = PUTV(EaR); h.o_Aconst = PUTV(Ac);
    h.o_lnPfac = PUTV(lnPfac); h.o_logA0 = PUTV(logA0); h.o_b0 = PUTV(b0); h.o_EaR0 = PUTV(EaR0);
    h.o_A0const = PUTV(A0c); h.o_troe_a = PUTV(ta); h.o_troe_iT3 = PUTV(tiT3);
    h.o_troe_iT1 = PUTV(tiT1); h.o_troe_T2 = PUTV(tT2); h.o_flags = PUTV(flags);
    h.o_rf = PUTV(rf); h.o_pf = PUTV(pf); h.o_dnu = PUTV(dnu); h.o_tb_off = PUTV(tboff);
    h.o_tb_len = PUTV(tblen); h.o_tb_sp = PUTV(tbsp); h.o_tb_alpha = PUTV(tbal);
    h.o_jrow = PUTV(jrow); h.o_jnu = PUTV(jnu); h.o_sp_off = PUTV(spoff);
    h.o_sp_slot = PUTV(spslot); h.o_sp_nu = PUTV(spnu);
    h.o_cat_sp = PUTV(catsp); h.o_gword = PUTV(gword); h.o_unit_off = PUTV(unitoff);
    h.o_plog_lev0 = PUTV(plev0); h.o_plog_nlev = PUTV(pnlev);
    h.o_plog_lnP = put(g.plog_lnP, g.nplog_lev * sizeof(double));
    h.o_plog_toff = put(g.plog_term_off, (g.nplog_lev + 1) * sizeof(int));
    h.o_plog_A = put(g.plog_A, g.nplog_term * sizeof(double));
    h.o_plog_logA = put(g.plog_logA, g.nplog_term * sizeof(double));
    h.o_plog_b = put(g.plog_b, g.nplog_term * sizeof(double));
    h.o_plog_EaR = put(g.plog_EaR, g.nplog_term * sizeof(double));
    std::vector<int> inert(n);
    for (int k = 0; k < n; ++k) inert[k] = spoff[k + 1] == spoff[k];
    h.o_inert = PUTV(inert);
    h.o_jword = PUTV(h.jword);
    h.o_jcoef = PUTV(h.jcoef);
    // the RHS's packed per-slot words
    std::vector<unsigned> fac(2 * ns);
    std::vector<double> bEa(2 * ns), lAP(2 * ns);
    for (int s = 0; s < ns; ++s) {
        for (int a = 0; a < 3; ++a)
            if (rf[a * ns + s] < 0 || rf[a * ns + s] > 255 || pf[a * ns + s] < 0 || pf[a * ns + s] > 255) {
                *err = "mechanism too large for the packed reaction words (256 species)";
                return HostMech();
            }
        if (flags[s] < 0 || flags[s] > 511 || dnu[s] < -kFacDnuBias || dnu[s] >= kFacDnuBias) {
            *err = "reaction flags or dnu out of the packed word's range";
            return HostMech();
        }
        fac[2 * s] = (unsigned)rf[s] | ((unsigned)rf[ns + s] << 8) | ((unsigned)rf[2 * ns + s] << 16) |
                     ((unsigned)pf[s] << 24);
        fac[2 * s + 1] = (unsigned)pf[ns + s] | ((unsigned)pf[2 * ns + s] << 8) | ((unsigned)flags[s] << 16) |
                         ((unsigned)(dnu[s] + kFacDnuBias) << 25);
        bEa[2 * s] = b[s];
        bEa[2 * s + 1] = EaR[s];
        lAP[2 * s] = logA[s];
        lAP[2 * s + 1] = lnPfac[s];
    }
    std::vector<double> nasa_sk(14 * n);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < 14; ++i) nasa_sk[(size_t)i * n + k] = nasa[14 * k + i];
    h.o_nasa_sk = PUTV(nasa_sk);
    h.o_fac = PUTV(fac);
    h.o_bEa = PUTV(bEa);
    h.o_lAP = PUTV(lAP);
#undef PUTV
    h.blob.resize((h.blob.size() + 255) & ~size_t(255));
    return h;
}

}  // namespace b200
