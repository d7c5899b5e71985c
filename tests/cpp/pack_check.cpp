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
    std::printf("ok %s nslot %d nunit %d gmax %d plog %d inert %d nu_den %d\n", g.name, ns, h.nunit, h.gmax, nplog,
                ninert, g.nu_den);
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
