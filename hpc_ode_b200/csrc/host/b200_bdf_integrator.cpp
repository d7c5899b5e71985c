// B200BDFIntegrator (b200ode_integrator.hpp): the reference's Integrator on
// the C ABI of b200ode.h.  The mesh's cell-major rows (temperature[i],
// species[i][k]) are packed into structure-of-arrays staging (T[i],
// Y[k * n + i]) for one b200ode_integrate call and unpacked afterwards, which is
// what CVodeIntegratorGPU::setGPUArrayInitialConditions / saveGPUArrayResults
// do for its device arrays (src/Integrators/CVodeIntegratorGPU.cpp:128-161).
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200ode_integrator.hpp"

B200BDFIntegrator::B200BDFIntegrator() {
    b200ode_default_options(&opts_);
    std::memset(&stats_, 0, sizeof(stats_));
}

B200BDFIntegrator::~B200BDFIntegrator() {
    if (handle_) b200ode_destroy(handle_);
    handle_ = nullptr;
}

void B200BDFIntegrator::setOptions(const b200ode_options& opts) { opts_ = opts; }

namespace {

// One solver option from the integrator config.  With the reference's headers
// the app passes config["integrator"]["omp"] as ompConfig, so the options sit
// under integrator.omp.b200.<key> in its YAML; the restated interface keeps
// them as "b200.<key>" entries of the ompConfig map.
bool cfg_get(const IntegratorConfig& c, const char* key, std::string* out) {
#ifdef B200ODE_WITH_REFERENCE_HEADERS
    const YAML::Node n = c.ompConfig["b200"];
    if (!n || !n[key]) return false;
    *out = n[key].as<std::string>();
    return true;
#else
    auto it = c.ompConfig.find(std::string("b200.") + key);
    if (it == c.ompConfig.end()) return false;
    *out = it->second;
    return true;
#endif
}

int cfg_int(const std::string& key, const std::string& v) {
    try {
        size_t pos = 0;
        const int x = std::stoi(v, &pos);
        if (pos == v.size()) return x;
    } catch (...) {
    }
    throw std::runtime_error("b200." + key + ": not an integer: '" + v + "'");
}

// Applies the b200 options of the config: precision (fp64 | mixed), refine (0 | 1),
// max_steps, max_order, form (persistent | step), graph (0 | 1), warps_per_block,
// blocks_per_sm, device, enthalpy (keep | update), formulation (conp | conv:
// constant volume, the config's pressure then being each cell's initial
// pressure).  Unknown values throw
// std::runtime_error.
void apply_config(const IntegratorConfig& c, b200ode_options* o, bool* update_enthalpy) {
    std::string v;
    if (cfg_get(c, "enthalpy", &v)) {
        if (v == "keep") *update_enthalpy = false;
        else if (v == "update") *update_enthalpy = true;
        else throw std::runtime_error("b200.enthalpy must be keep or update, not '" + v + "'");
    }
    if (cfg_get(c, "precision", &v)) {
        if (v == "fp64") o->precision = B200ODE_FP64;
        else if (v == "mixed") o->precision = B200ODE_MIXED;
        else throw std::runtime_error("b200.precision must be fp64 or mixed, not '" + v + "'");
    }
    if (cfg_get(c, "formulation", &v)) {
        if (v == "conp") o->formulation = B200ODE_CONP;
        else if (v == "conv") o->formulation = B200ODE_CONV;
        else throw std::runtime_error("b200.formulation must be conp or conv, not '" + v + "'");
    }
    if (cfg_get(c, "form", &v)) {
        if (v == "persistent") o->persistent = 1;
        else if (v == "step") o->persistent = 0;
        else throw std::runtime_error("b200.form must be persistent or step, not '" + v + "'");
    }
    if (cfg_get(c, "refine", &v)) o->refine = cfg_int("refine", v);
    if (cfg_get(c, "max_steps", &v)) o->max_steps = cfg_int("max_steps", v);
    if (cfg_get(c, "max_order", &v)) o->max_order = cfg_int("max_order", v);
    if (cfg_get(c, "graph", &v)) o->use_graph = cfg_int("graph", v);
    if (cfg_get(c, "warps_per_block", &v)) o->warps_per_block = cfg_int("warps_per_block", v);
    if (cfg_get(c, "blocks_per_sm", &v)) o->blocks_per_sm = cfg_int("blocks_per_sm", v);
    if (cfg_get(c, "device", &v)) o->device = cfg_int("device", v);
}

}  // namespace

void B200BDFIntegrator::init(std::shared_ptr<Context> c, IntegratorConfig config) {
    Integrator::init(std::move(c), config);
    // mechanism check before any device work (CVodeIntegrator.cpp:41-48)
    const int nsp = b200ode_mechanism_species(mechanism.c_str());
    if (nsp < 0 || systemSize != nsp) {
        std::stringstream ss;
        ss << "mechanism size of: " << mechanism << " (" << nsp << ") differs from the mesh size: " << systemSize;
        logger->error(ss.str());
        throw std::runtime_error(ss.str());
    }
    if (handle_) b200ode_destroy(handle_);
    handle_ = nullptr;
    b200ode_options o = opts_;
    try {
        apply_config(config, &o, &update_enthalpy_);
    } catch (const std::exception& e) {
        logger->error(e.what());
        throw;
    }
    o.reltol = reltol;
    o.abstol = abstol;
    const b200ode_status rc = b200ode_create(mechanism.c_str(), &o, &handle_);
    if (rc != B200ODE_OK) {
        const std::string msg = std::string("B200BDFIntegrator: ") + b200ode_last_error();
        logger->error(msg);
        throw std::runtime_error(msg);
    }
    logger->info("B200BDFIntegrator initialized");
}

void B200BDFIntegrator::integrate(double t0, double t) {
    Integrator::integrate(t0, t);
    if (!handle_) throw std::runtime_error("B200BDFIntegrator: integrate() before init()");
    const int n = mesh->totalSize();
    const int nsp = systemSize;
    T_.resize(n);
    Y_.resize((size_t)n * nsp);
    status_.assign(n, 0);
    const double* Tm = mesh->getTemperaturePointer();
    for (int i = 0; i < n; ++i) {
        T_[i] = Tm[i];
        const double* y = mesh->getSpeciesPointer(i);
        for (int k = 0; k < nsp; ++k) Y_[(size_t)k * n + i] = y[k];
    }
    std::memset(&stats_, 0, sizeof(stats_));
    const b200ode_status rc =
        b200ode_integrate(handle_, n, nullptr, pressure, T_.data(), Y_.data(), t0, t, status_.data(), &stats_);
    if (rc != B200ODE_OK) {
        const std::string msg = std::string("B200BDFIntegrator: ") + b200ode_last_error();
        logger->error(msg);
        throw std::runtime_error(msg);
    }
    double* Tw = mesh->getTemperaturePointer();
    for (int i = 0; i < n; ++i) {
        Tw[i] = T_[i];
        double* y = mesh->getSpeciesPointer(i);
        for (int k = 0; k < nsp; ++k) y[k] = Y_[(size_t)k * n + i];
    }
    if (update_enthalpy_ && mesh->hasEnthalpy()) {
        // ENTHA of the integrated state (the reference's CVODE integrators keep the old value)
        std::vector<double> hm(n);
        const b200ode_status rh = b200ode_eval_enthalpy(handle_, n, T_.data(), Y_.data(), hm.data());
        if (rh != B200ODE_OK) {
            const std::string msg = std::string("B200BDFIntegrator: ") + b200ode_last_error();
            logger->error(msg);
            throw std::runtime_error(msg);
        }
        double* H = mesh->getEnthalpyPointer();
        for (int i = 0; i < n; ++i) H[i] = hm[i];
    }
    if (stats_.n_failed) {
        std::stringstream ss;
        ss << stats_.n_failed << " of " << n << " cells did not reach t (CVODE status kept per cell)";
        logger->error(ss.str());
    }
}

void B200BDFIntegrator::clean() {
    if (handle_) b200ode_destroy(handle_);
    handle_ = nullptr;
    T_.clear();
    Y_.clear();
    Integrator::clean();
}
