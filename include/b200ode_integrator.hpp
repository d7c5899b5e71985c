// B200BDFIntegrator: the reference's Integrator (Integrator.hpp:22-40) on the
// B200 batched BDF of b200ode.h.  Factory type string: "BDFIntegratorB200".
//
// Drop-in behaviour, as CVodeIntegrator / CVodeIntegratorGPU
// (src/Integrators/CVodeIntegrator.cpp:34-96, CVodeIntegratorGPU.cpp:30-161):
//   init      base-class bookkeeping and logging, then the mechanism check: an
//             unknown mechanism or a species count that differs from the mesh's
//             is logged and thrown as std::runtime_error;
//   integrate every cell of the mesh from t0 to t with the cell state
//             [T, Y_0 .. Y_{nsp-2}], reltol/abstol from the config, 10000 steps at
//             most, the config's pressure; on return the mesh holds the new T
//             and Y with Y_{nsp-1} = 1 - sum(Y_0 .. Y_{nsp-2}); ENTHA is not
//             touched (as in the CVODE integrators) unless the config says
//             b200.enthalpy: update, which writes the enthalpy of the new state;
//   clean     releases the device handle.
// Differences: per-cell failures do not throw; the count is logged and the
// per-cell CVODE status is kept (cellStatus()).  CUDA and allocation errors
// throw std::runtime_error (the reference's GPU driver calls exit()).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#ifdef B200ODE_WITH_REFERENCE_HEADERS
#include "ODEIntegrator/Integrators/Integrator.hpp"
#else
#include "b200ode_host_interface.hpp"
#endif
#include "b200ode.h"

class B200BDFIntegrator : public Integrator {
public:
    B200BDFIntegrator();
    ~B200BDFIntegrator();

    void init(std::shared_ptr<Context> ctx, IntegratorConfig config) override;
    void integrate(double t0, double t) override;
    void clean() override;

    // Solver options (precision, launch shape, ...) used by the next init();
    // tolerances still come from the IntegratorConfig.
    void setOptions(const b200ode_options& opts);
    // CVODE return code of every cell after the last integrate().
    const std::vector<int32_t>& cellStatus() const { return status_; }
    // Counters and device timings of the last integrate().
    const b200ode_stats& lastStats() const { return stats_; }

private:
    b200ode_handle* handle_ = nullptr;
    b200ode_options opts_;
    std::vector<double> T_, Y_;   // SoA staging: T[n], Y[k * n + i]
    std::vector<int32_t> status_;
    b200ode_stats stats_;
    bool update_enthalpy_ = false;   // config b200.enthalpy: update
};
