// Implementation of the restated host interface (b200ode_host_interface.hpp):
// Mesh bookkeeping, the base Integrator's logging, the integrator factory.
// Behaviour follows src/Mesh/Mesh.cpp, src/Integrators/Integrator.cpp:8-39 and
// ODEIntegratorFactory::createIntegrator (ODEIntegratorFactory.hpp:55-69).
#include <iostream>
#include <sstream>

#include "b200ode_integrator.hpp"

std::vector<double>& Mesh::getEnthalpyVector() {
    if (!hasEnthalpy()) throw std::runtime_error("Mesh does not have enthalpy");
    return enthalpy_;
}

std::vector<Coords>& Mesh::getCoordinatesVector() {
    if (!hasCoordinates()) throw std::runtime_error("Mesh does not have coordinates");
    return coords_;
}

double* Mesh::getEnthalpyPointer() {
    if (!hasEnthalpy()) throw std::runtime_error("Mesh does not have enthalpy");
    return enthalpy_.data();
}

void Mesh::addPoint(const Point& p) {
    if (totalSize() == 0 && p.isReady()) {
        enthalpyFlag_ = p.hasEnthalpy();
        coordFlag_ = p.hasCoordinates();
        nsp_ = p.numSpecies();
    }
    const bool compatible = p.isReady() && p.numSpecies() == nsp_ && p.hasEnthalpy() == enthalpyFlag_ &&
                            p.hasCoordinates() == coordFlag_;
    if (!compatible) throw std::runtime_error("Trying to add an incompatible Point to Mesh");
    temperature_.push_back(p.getTemperature());
    species_.push_back(p.getSpecies());
    if (enthalpyFlag_) enthalpy_.push_back(p.getEnthalpy());
    if (coordFlag_) coords_.push_back(p.getCoordinates());
}

void Mesh::clear() {
    temperature_.clear();
    enthalpy_.clear();
    species_.clear();
    coords_.clear();
    nsp_ = 0;
    enthalpyFlag_ = coordFlag_ = false;
}

void ConsoleLogger::log(const std::string& line) { std::cerr << line << std::endl; }

void Integrator::init(std::shared_ptr<Context> c, IntegratorConfig config) {
    ctx = std::move(c);
    logger = ctx->getLogger();
    mesh = ctx->getMesh();
    totalSize = mesh->totalSize();
    systemSize = mesh->numSpecies();
    mechanism = config.mechanism;
    reltol = config.reltol;
    abstol = config.abstol;
    pressure = config.pressure;
    ompConfig = config.ompConfig;
    logger->info("Initializing integrator...");
    std::stringstream ss;
    ss << "{ mechanism: " << mechanism << ", reltol: " << reltol << ", abstol: " << abstol
       << ", pressure: " << pressure << " }";
    logger->info(ss.str());
}

void Integrator::integrate(double t0, double t) {
    std::stringstream ss;
    ss << "Integrating interval of: " << t - t0 << " seconds";
    logger->info(ss.str());
}

void Integrator::clean() { logger->info("Integrator clean completed"); }

std::unique_ptr<Integrator> createIntegrator(const std::string& integratorType) {
    if (integratorType == "BDFIntegratorB200") return std::make_unique<B200BDFIntegrator>();
    throw std::runtime_error("Integrator type is not valid");
}
