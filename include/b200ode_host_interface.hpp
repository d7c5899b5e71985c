// The host-side interface the reference's integrators implement, restated so the
// B200 integrator builds and is tested without the reference tree (which needs
// yaml-cpp, SUNDIALS and Cantera).  Names, signatures and observable behaviour
// follow the reference:
//   IntegratorConfig, Integrator      include/ODEIntegrator/Integrators/Integrator.hpp:13-40,
//                                     src/Integrators/Integrator.cpp:8-39
//   Mesh (AoS cells: T[i], species row i)  include/ODEIntegrator/Mesh/Mesh.hpp:8-47
//   Point / Coords                    include/ODEIntegrator/Mesh/Point.hpp
//   Context (mesh + logger)           include/ODEIntegrator/Context/Context.hpp:14-64
//   BaseLogger::info / error          include/ODEIntegrator/Logger/BaseLogger.hpp
//   createIntegrator(type) string switch  include/ODEIntegrator/ODEIntegratorFactory.hpp:55-69
// Differences, all outside the integrator's contract: ompConfig is a plain
// key/value map instead of a YAML::Node; the logger writes synchronously; only
// the integrator types built here are known to the factory; Integrator has a
// virtual destructor.  Built with -DB200ODE_WITH_REFERENCE_HEADERS,
// b200ode_integrator.hpp includes the reference's own headers instead of this
// file.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

struct Coords {
    double x, y, z;
};

// One cell: temperature, optional enthalpy/coordinates, nsp mass fractions.
class Point {
public:
    explicit Point(int nsp) : nsp_(nsp) {}
    Point& setTemperature(double T) { temperature_ = T; hasT_ = true; return *this; }
    Point& setEnthalpy(double h) { enthalpy_ = h; hasH_ = true; return *this; }
    Point& setSpecies(std::vector<double> y) { species_ = std::move(y); return *this; }
    Point& setCoordinates(Coords c) { coords_ = c; hasC_ = true; return *this; }
    bool hasTemperature() const { return hasT_; }
    bool hasEnthalpy() const { return hasH_; }
    bool hasSpecies() const { return (int)species_.size() == nsp_; }
    bool hasCoordinates() const { return hasC_; }
    bool isReady() const { return hasTemperature() && hasSpecies(); }
    double getTemperature() const { return temperature_; }
    double getEnthalpy() const { return enthalpy_; }
    std::vector<double> getSpecies() const { return species_; }
    Coords getCoordinates() const { return coords_; }
    int numSpecies() const { return nsp_; }

private:
    int nsp_;
    double temperature_ = 0.0, enthalpy_ = 0.0;
    std::vector<double> species_;
    Coords coords_{0.0, 0.0, 0.0};
    bool hasT_ = false, hasH_ = false, hasC_ = false;
};

// Cells in the reference's layout: temperature[i], speciesMatrix[i][k].
class Mesh {
public:
    Mesh() = default;
    Mesh(const Mesh&) = delete;
    Mesh& operator=(const Mesh&) = delete;

    std::vector<double>& getTemperatureVector() { return temperature_; }
    std::vector<double>& getEnthalpyVector();
    std::vector<double>& getSpeciesVector(int index) { return species_.at(index); }
    std::vector<std::vector<double>>& getSpeciesMatrix() { return species_; }
    std::vector<Coords>& getCoordinatesVector();
    double* getTemperaturePointer() { return temperature_.data(); }
    double* getEnthalpyPointer();
    double* getSpeciesPointer(int index) { return species_.at(index).data(); }

    // Throws std::runtime_error for a point incompatible with the cells already held.
    void addPoint(const Point& p);
    int totalSize() const { return (int)temperature_.size(); }
    int numSpecies() const { return nsp_; }
    bool hasEnthalpy() const { return enthalpyFlag_; }
    bool hasCoordinates() const { return coordFlag_; }
    void clear();

private:
    std::vector<double> temperature_, enthalpy_;
    std::vector<std::vector<double>> species_;
    std::vector<Coords> coords_;
    int nsp_ = 0;
    bool enthalpyFlag_ = false, coordFlag_ = false;
};

enum class LogLevel { DEBUG, INFO };

class BaseLogger {
public:
    explicit BaseLogger(LogLevel level = LogLevel::INFO) : level_(level) {}
    virtual ~BaseLogger() = default;
    void info(const std::string& msg) { log("INFO:  " + msg); }
    void debug(const std::string& msg) { if (level_ == LogLevel::DEBUG) log("DEBUG: " + msg); }
    void error(const std::string& msg) { log("ERROR: " + msg); }

protected:
    virtual void log(const std::string& line) = 0;
    LogLevel level_;
};

// Writes log lines to stderr.
class ConsoleLogger : public BaseLogger {
public:
    explicit ConsoleLogger(LogLevel level = LogLevel::INFO) : BaseLogger(level) {}

protected:
    void log(const std::string& line) override;
};

// Keeps log lines in memory (tests, embedding).
class MemoryLogger : public BaseLogger {
public:
    explicit MemoryLogger(LogLevel level = LogLevel::INFO) : BaseLogger(level) {}
    const std::vector<std::string>& lines() const { return lines_; }

protected:
    void log(const std::string& line) override { lines_.push_back(line); }

private:
    std::vector<std::string> lines_;
};

class Context {
public:
    Context() : logger_(std::make_shared<ConsoleLogger>()), mesh_(std::make_shared<Mesh>()) {}
    explicit Context(std::shared_ptr<Mesh> mesh) : logger_(std::make_shared<ConsoleLogger>()), mesh_(std::move(mesh)) {}
    Context(std::shared_ptr<BaseLogger> logger, std::shared_ptr<Mesh> mesh)
        : logger_(std::move(logger)), mesh_(std::move(mesh)) {}
    void setLogger(std::shared_ptr<BaseLogger> l) { logger_ = std::move(l); }
    void setMesh(std::shared_ptr<Mesh> m) { mesh_ = std::move(m); }
    std::shared_ptr<BaseLogger> getLogger() const { return logger_; }
    std::shared_ptr<Mesh> getMesh() const { return mesh_; }

private:
    std::shared_ptr<BaseLogger> logger_;
    std::shared_ptr<Mesh> mesh_;
};

struct IntegratorConfig {
    std::string mechanism;
    double reltol;
    double abstol;
    double pressure;
    std::map<std::string, std::string> ompConfig;
};

// Abstract integrator: init fills the protected fields from the context and
// config and logs them; integrate(t0, t) advances every cell of the mesh by
// t - t0; clean releases what init acquired.
class Integrator {
public:
    virtual ~Integrator() = default;
    virtual void init(std::shared_ptr<Context> ctx, IntegratorConfig config);
    virtual void integrate(double t0, double t);
    virtual void clean();

protected:
    int totalSize = 0;
    int systemSize = 0;
    std::shared_ptr<Mesh> mesh;
    std::shared_ptr<BaseLogger> logger;
    std::shared_ptr<Context> ctx;
    std::string mechanism;
    double reltol = 0.0;
    double abstol = 0.0;
    double pressure = 0.0;
    std::map<std::string, std::string> ompConfig;
};

// The factory's integrator switch: "BDFIntegratorB200" -> B200BDFIntegrator;
// any other type throws std::runtime_error("Integrator type is not valid").
std::unique_ptr<Integrator> createIntegrator(const std::string& integratorType);
