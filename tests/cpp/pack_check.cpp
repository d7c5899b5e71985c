// CPU check of the device-table packing (hpc_ode_b200/csrc/mech_dev.h) for every
// compiled mechanism: the packer accepts it, its gather-unit count equals the
// generated NUNITS the kernels size their shared scratch by, and the balanced
// gather words reproduce, per (species, reaction), the net stoichiometric
// coefficient computed directly from the generated reactant/product lists
// (fractional coefficients included); PLOG slots and inert species agree with
// the tables.  Prints one "ok <mechanism> ..." line per mechanism, exits 1 on
// the first mismatch.
#include <cmath>
#include <cstdio>
#include <map>
#include <tuple>
#include <string>
#include <utility>
#include <vector>

#include "../../hpc_ode_b200/csrc/mech_dev.h"
#include "../../hpc_ode_b200/csrc/mech/ESTiMatE-Mech_04042022_mech.h"
#include "../../hpc_ode_b200/csrc/mech/gri30_mech.h"
#include "../../hpc_ode_b200/csrc/mech/h2_li_2004_mech.h"
#include "../../hpc_ode_b200/csrc/mech/h2o2_mech.h"
#include "../../hpc_ode_b200/csrc/mech/nDodecane_Reitz_mech.h"

using b200::GenTables;
using b200::HostMech;

#define TABLES(tag, PFX)                                                                             \
    GenTables{#tag, PFX##_NSP, PFX##_NRXN, PFX##_MAXP, PFX##_NTB, PFX##_NU_DEN, PFX##_NPLOGLEV,       \
              PFX##_NPLOGTERM, tag##_species_names, tag##_mw, tag##_tmid, tag##_nasa_lo,              \
              tag##_nasa_hi, tag##_rxn_type, tag##_rxn_rev, tag##_rxn_A, tag##_rxn_logA, tag##_rxn_b, \
              tag##_rxn_EaR, tag##_rxn_A0, tag##_rxn_logA0, tag##_rxn_b0, tag##_rxn_EaR0,            \
              tag##_rxn_troe, tag##_rxn_troe_T2, tag##_rxn_reac_sp, tag##_rxn_reac_nu,               \
              tag##_rxn_prod_sp, tag##_rxn_prod_nu, tag##_rxn_tb_off, tag##_tb_sp, tag##_tb_alpha,   \
              tag##_plog_off, tag##_plog_lnP, tag##_plog_term_off, tag##_plog_A, tag##_plog_logA,    \
              tag##_plog_b, tag##_plog_EaR}

template <class T>
const T* at(const HostMech& h, size_t off) {
    return reinterpret_cast<const T*>(h.blob.data() + off);
}

static int check(const GenTables& g, int nunits_generated, int nplog_generated) {
    std::string err;
    const HostMech h = b200::pack_mechanism(g, &err);
    if (h.nsp == 0) { std::printf("FAIL %s: pack: %s\n", g.name, err.c_str()); return 1; }
    const int ns = h.nslot, n = g.nsp, P = g.maxp;
    if (ns != ((g.nrxn + 32) / 32) * 32 || ns > 2048) { std::printf("FAIL %s: nslot %d\n", g.name, ns); return 1; }
    if (h.nunit != nunits_generated) {
        std::printf("FAIL %s: %d gather units, generated NUNITS %d\n", g.name, h.nunit, nunits_generated);
        return 1;
    }
    // net stoichiometry per (species, reaction) from the generated lists
    std::map<std::pair<int, int>, double> want;
    for (int r = 0; r < g.nrxn; ++r) {
        for (int i = 0; i < P && g.reac_sp[r * P + i] >= 0; ++i)
            want[{g.reac_sp[r * P + i], r}] -= g.reac_nu[r * P + i];
        for (int i = 0; i < P && g.prod_sp[r * P + i] >= 0; ++i)
            want[{g.prod_sp[r * P + i], r}] += g.prod_nu[r * P + i];
    }
    for (auto it = want.begin(); it != want.end();) it = (it->second == 0.0) ? want.erase(it) : std::next(it);
    // the same from the gather words: units -> species, word -> (slot, nu * den)
    const int* gword = at<int>(h, h.o_gword);
    const int* unit_off = at<int>(h, h.o_unit_off);
    std::vector<int> unit_sp(h.nunit, -1);
    for (int k = 0; k < n; ++k)
        for (int u = unit_off[k]; u < unit_off[k + 1]; ++u) unit_sp[u] = k;
    std::map<std::pair<int, int>, double> got;
    const int pad_slot = ns - 1;
    for (int e = 0; e < h.gmax; ++e) {
        for (int l = 0; l < 32; ++l) {
            const int w = gword[e * 32 + l];
            const int slot = w & 2047, nu = ((w >> 11) & 31) - 16, unit = w >> 17;
            if (nu == 0) {   // padding entry
                if (slot != pad_slot) { std::printf("FAIL %s: padding word at slot %d\n", g.name, slot); return 1; }
                continue;
            }
            const int r = h.slot_rxn[slot];
            if (r < 0 || unit >= h.nunit) { std::printf("FAIL %s: word slot %d unit %d\n", g.name, slot, unit); return 1; }
            got[{unit_sp[unit], r}] += (double)nu / g.nu_den;
        }
    }
    if (got.size() != want.size()) {
        std::printf("FAIL %s: %zu gather entries, %zu nonzero coefficients\n", g.name, got.size(), want.size());
        return 1;
    }
    for (const auto& kv : want) {
        auto it = got.find(kv.first);
        if (it == got.end() || std::fabs(it->second - kv.second) > 1e-12) {
            std::printf("FAIL %s: species %d reaction %d: %g vs %g\n", g.name, kv.first.first, kv.first.second,
                        it == got.end() ? 0.0 : it->second, kv.second);
            return 1;
        }
    }
    // PLOG slots and inert species
    const int* flags = at<int>(h, h.o_flags);
    int nplog = 0;
    for (int s = 0; s < ns; ++s) nplog += (flags[s] & b200::kFlagPlog) != 0;
    if (nplog != nplog_generated) { std::printf("FAIL %s: %d PLOG slots\n", g.name, nplog); return 1; }
    const int* inert = at<int>(h, h.o_inert);
    int ninert = 0;
    for (int k = 0; k < n; ++k) {
        bool reacts = false;
        for (const auto& kv : want) reacts = reacts || kv.first.first == k;
        if (inert[k] != (reacts ? 0 : 1)) { std::printf("FAIL %s: inert flag of species %d\n", g.name, k); return 1; }
        ninert += inert[k];
    }
    // every table-derived index the kernels use, against the array it indexes
    // (the device code does not check them): reaction factor species index the
    // concentrations / Gibbs terms C[0..N] (N = the padding factor 1 / 0),
    // Jacobian scatter rows and third-body species index rows/columns 0..N-1,
    // third-body lists stay inside tb_sp, catalysts are species, gather words
    // address slots 0..nslot-1 and units 0..NUNITS-1, each species' units are a
    // contiguous in-range run, PLOG slots' levels and terms stay in their tables;
    // and the Jacobian's per-species work ([3][N] doubles) fits the rate buffer
    // (nslot doubles) it reuses.
    auto bad = [&](const char* what, int s, int v) {
        std::printf("FAIL %s: %s (slot %d, value %d)\n", g.name, what, s, v);
        return 1;
    };
    const int* rf = at<int>(h, h.o_rf);
    const int* pf = at<int>(h, h.o_pf);
    const int* dnu = at<int>(h, h.o_dnu);
    const double* bb = at<double>(h, h.o_b);
    const double* EaR = at<double>(h, h.o_EaR);
    const double* logA = at<double>(h, h.o_logA);
    const double* lnPfac = at<double>(h, h.o_lnPfac);
    const unsigned* fac = at<unsigned>(h, h.o_fac);
    // the species-innermost NASA-7 copy holds the same coefficients
    const double* nasa = at<double>(h, h.o_nasa);
    const double* nasa_sk = at<double>(h, h.o_nasa_sk);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < 14; ++i)
            if (nasa_sk[(size_t)i * n + k] != nasa[14 * k + i]) return bad("NASA-7 species-innermost copy", k, i);
    const double* bEa = at<double>(h, h.o_bEa);
    const double* lAP = at<double>(h, h.o_lAP);
    const int* tb_off = at<int>(h, h.o_tb_off);
    const int* tb_len = at<int>(h, h.o_tb_len);
    const int* tb_sp = at<int>(h, h.o_tb_sp);
    const int* cat_sp = at<int>(h, h.o_cat_sp);
    const int* jrow = at<int>(h, h.o_jrow);
    const int* plev0 = at<int>(h, h.o_plog_lev0);
    const int* pnlev = at<int>(h, h.o_plog_nlev);
    const int* ptoff = at<int>(h, h.o_plog_toff);
    for (int s = 0; s < ns; ++s) {
        for (int a = 0; a < 3; ++a) {
            if (rf[a * ns + s] < 0 || rf[a * ns + s] > n) return bad("reactant factor species", s, rf[a * ns + s]);
            if (pf[a * ns + s] < 0 || pf[a * ns + s] > n) return bad("product factor species", s, pf[a * ns + s]);
        }
        if (tb_off[s] < 0 || tb_len[s] < 0 || tb_off[s] + tb_len[s] > h.ntb) return bad("third-body list", s, tb_off[s]);
        for (int t = 0; t < tb_len[s]; ++t)
            if (tb_sp[tb_off[s] + t] < 0 || tb_sp[tb_off[s] + t] >= n) return bad("third-body species", s, tb_sp[tb_off[s] + t]);
        if ((flags[s] & b200::kFlagCatalyst) && (cat_sp[s] < 0 || cat_sp[s] >= n)) return bad("catalyst", s, cat_sp[s]);
        for (int e = 0; e < b200::kJRow; ++e) {
            const int k = jrow[e * ns + s];
            if (k < -1 || k >= n) return bad("Jacobian row", s, k);
        }
        if (flags[s] & b200::kFlagPlog) {
            if (plev0[s] < 0 || pnlev[s] < 1 || plev0[s] + pnlev[s] > g.nplog_lev) return bad("PLOG levels", s, plev0[s]);
            for (int l = plev0[s]; l < plev0[s] + pnlev[s]; ++l)
                if (ptoff[l] < 0 || ptoff[l + 1] < ptoff[l] || ptoff[l + 1] > g.nplog_term) return bad("PLOG terms", s, l);
        }
        // the RHS's packed words decode (as the kernel decodes them) to the same
        // factor species, flags, dnu, Arrhenius terms and pressure factor
        const unsigned fx = fac[2 * s], fy = fac[2 * s + 1];
        const int dec_rf[3] = {(int)(fx & 255), (int)((fx >> 8) & 255), (int)((fx >> 16) & 255)};
        const int dec_pf[3] = {(int)(fx >> 24), (int)(fy & 255), (int)((fy >> 8) & 255)};
        for (int a = 0; a < 3; ++a) {
            if (dec_rf[a] != rf[a * ns + s]) return bad("packed reactant factor", s, dec_rf[a]);
            if (dec_pf[a] != pf[a * ns + s]) return bad("packed product factor", s, dec_pf[a]);
        }
        if ((int)((fy >> 16) & 511) != flags[s]) return bad("packed flags", s, (int)((fy >> 16) & 511));
        if ((int)(fy >> 25) - b200::kFacDnuBias != dnu[s]) return bad("packed dnu", s, (int)(fy >> 25));
        if (bEa[2 * s] != bb[s] || bEa[2 * s + 1] != EaR[s] || lAP[2 * s] != logA[s] || lAP[2 * s + 1] != lnPfac[s])
            return bad("packed Arrhenius / pressure factor", s, 0);
    }
    for (int e = 0; e < h.gmax; ++e)
        for (int l = 0; l < 32; ++l) {
            const int w = gword[e * 32 + l];
            if ((w & 2047) >= ns) return bad("gather slot", e, w & 2047);
            if ((w >> 17) >= nunits_generated) return bad("gather unit", e, w >> 17);
        }
    for (int k = 0; k < n; ++k)
        if (unit_off[k] < 0 || unit_off[k + 1] < unit_off[k] || unit_off[k + 1] > h.nunit) return bad("species units", k, unit_off[k]);
    if (3 * n > ns) return bad("Jacobian per-species work [3][N] exceeds the rate buffer", ns, 3 * n);
    // the Jacobian gather: its (output element, slot, piece) -> coefficient map
    // equals the scatter the tables describe -- for each net-stoichiometry row k
    // of each slot: +nu at (k, reactant factor a) piece a, -nu at (k, product
    // factor a) piece 3 + a, and at (k, j) piece 6: nu * alpha_j for the
    // third-body species j, or -nu for every j but the catalyst; every output
    // element is written exactly once, by its last entry
    {
        const int lda = (n % 2 == 0) ? n + 1 : n;
        std::map<std::tuple<int, int, int>, double> jwant, jgot;
        const double* jnu = at<double>(h, h.o_jnu);
        const double* tb_al = at<double>(h, h.o_tb_alpha);
        for (int s = 0; s < ns; ++s) {
            if (h.slot_rxn[s] < 0) continue;
            for (int e = 0; e < b200::kJRow; ++e) {
                const int k = jrow[e * ns + s];
                if (k < 0) break;
                const double nu = jnu[e * ns + s];
                for (int a = 0; a < 3; ++a) {
                    if (rf[a * ns + s] < n) jwant[{k * lda + rf[a * ns + s], s, a}] += nu;
                    if (pf[a * ns + s] < n) jwant[{k * lda + pf[a * ns + s], s, 3 + a}] += -nu;
                }
                if (flags[s] & b200::kFlagCatalyst) {
                    for (int j = 0; j < n; ++j) if (j != cat_sp[s]) jwant[{k * lda + j, s, 6}] += -nu;
                } else if (flags[s] & b200::kFlagTypeMask) {
                    for (int t = tb_off[s]; t < tb_off[s] + tb_len[s]; ++t) jwant[{k * lda + tb_sp[t], s, 6}] += nu * tb_al[t];
                }
            }
        }
        const int* jw = at<int>(h, h.o_jword);
        const double* jc = at<double>(h, h.o_jcoef);
        std::map<int, int> written;
        for (int l = 0; l < 32; ++l) {
            int cur = -1;
            for (int e = 0; e < h.jgmax; ++e) {
                const int w = jw[e * 32 + l];
                const int slot = w & 2047, piece = (w >> 11) & 7, last = (w >> 14) & 1, out = w >> 15;
                if (slot >= ns || piece >= b200::kJacPieces) return bad("Jacobian gather word", e, w);
                if (jc[e * 32 + l] == 0.0 && !last && h.slot_rxn[slot] < 0) continue;   // padding
                if (out >= n * lda || out % lda >= n) return bad("Jacobian gather output", e, out);
                if (cur >= 0 && out != cur) return bad("Jacobian gather unit not contiguous", e, out);
                cur = out;
                jgot[{out, slot, piece}] += jc[e * 32 + l];
                if (last) { written[out] += 1; cur = -1; }
            }
            if (cur >= 0) return bad("Jacobian gather unit without a last entry", l, cur);
        }
        if (jgot.size() != jwant.size()) return bad("Jacobian gather entry count", (int)jgot.size(), (int)jwant.size());
        for (const auto& kv : jwant) {
            auto it = jgot.find(kv.first);
            if (it == jgot.end() || std::fabs(it->second - kv.second) > 1e-12 * (1.0 + std::fabs(kv.second)))
                return bad("Jacobian gather coefficient", std::get<1>(kv.first), std::get<0>(kv.first));
        }
        for (const auto& kv : written) if (kv.second != 1) return bad("Jacobian output written twice", kv.first, kv.second);
    }
    std::printf("ok %s nslot %d nunit %d gmax %d plog %d inert %d nu_den %d jac entries %d jgmax %d (indices in range)\n",
                g.name, ns, h.nunit, h.gmax, nplog, ninert, g.nu_den, h.njent, h.jgmax);
    return 0;
}

int main() {
    int bad = 0;
    bad |= check(TABLES(gri30, MECH_GRI30), MECH_GRI30_NUNITS, MECH_GRI30_NPLOG);
    bad |= check(TABLES(h2o2, MECH_H2O2), MECH_H2O2_NUNITS, MECH_H2O2_NPLOG);
    bad |= check(TABLES(ndodecane_reitz, MECH_NDODECANE_REITZ), MECH_NDODECANE_REITZ_NUNITS,
                 MECH_NDODECANE_REITZ_NPLOG);
    bad |= check(TABLES(h2_li_2004, MECH_H2_LI_2004), MECH_H2_LI_2004_NUNITS, MECH_H2_LI_2004_NPLOG);
    bad |= check(TABLES(estimate_mech_04042022, MECH_ESTIMATE_MECH_04042022), MECH_ESTIMATE_MECH_04042022_NUNITS,
                 MECH_ESTIMATE_MECH_04042022_NPLOG);
    return bad;
}
