// Test driver for B200BDFIntegrator through the restated reference interface:
// builds a Mesh from a binary file, creates the integrator through the factory
// string, runs init / integrate(0, dt) / clean as the reference's application
// does (app/main.cpp), and writes the mesh back.
//
//   integrator_driver <type> <mechanism> <in.bin> <out.bin> [b200.key=value ...]
// in.bin:  int32 n, int32 nsp, double dt, double pressure, double T[n], double Y[n][nsp]
// out.bin: the same layout after integration, then int32 status[n], then
//          double enthalpy[n] (every point is created with enthalpy 0)
// Exit 0 on success; on an exception prints "EXCEPTION: <what>" and exits 3.
#include <cstdint>
#include <cstdio>
#include <exception>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "b200ode_integrator.hpp"

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <type> <mechanism> <in.bin> <out.bin> [b200.key=value ...]\n", argv[0]);
        return 2;
    }
    try {
        std::ifstream in(argv[3], std::ios::binary);
        int32_t n = 0, nsp = 0;
        double dt = 0.0, P = 0.0;
        in.read(reinterpret_cast<char*>(&n), 4).read(reinterpret_cast<char*>(&nsp), 4);
        in.read(reinterpret_cast<char*>(&dt), 8).read(reinterpret_cast<char*>(&P), 8);
        std::vector<double> T(n), Y((size_t)n * nsp);
        in.read(reinterpret_cast<char*>(T.data()), 8 * (std::streamsize)n);
        in.read(reinterpret_cast<char*>(Y.data()), 8 * (std::streamsize)Y.size());
        if (!in) throw std::runtime_error("short input file");

        auto mesh = std::make_shared<Mesh>();
        for (int i = 0; i < n; ++i)
            mesh->addPoint(Point(nsp).setTemperature(T[i]).setEnthalpy(0.0).setSpecies(
                std::vector<double>(Y.begin() + (size_t)i * nsp, Y.begin() + (size_t)(i + 1) * nsp)));
        auto logger = std::make_shared<MemoryLogger>();
        auto ctx = std::make_shared<Context>(logger, mesh);
        std::unique_ptr<Integrator> integrator = createIntegrator(argv[1]);
        IntegratorConfig config{argv[2], 1.0e-6, 1.0e-10, P, {}};
        for (int a = 5; a < argc; ++a) {   // config options, as the app's YAML would give them
            const std::string kv = argv[a];
            const size_t eq = kv.find('=');
            if (eq == std::string::npos) throw std::runtime_error("option without '=': " + kv);
            config.ompConfig[kv.substr(0, eq)] = kv.substr(eq + 1);
        }
        integrator->init(ctx, config);
        integrator->integrate(0.0, dt);
        auto* b200 = dynamic_cast<B200BDFIntegrator*>(integrator.get());
        std::vector<int32_t> status = b200 ? b200->cellStatus() : std::vector<int32_t>(n, 0);
        integrator->clean();
        for (const auto& line : logger->lines()) std::cout << line << "\n";

        std::ofstream out(argv[4], std::ios::binary);
        out.write(reinterpret_cast<const char*>(&n), 4).write(reinterpret_cast<const char*>(&nsp), 4);
        out.write(reinterpret_cast<const char*>(&dt), 8).write(reinterpret_cast<const char*>(&P), 8);
        out.write(reinterpret_cast<const char*>(mesh->getTemperaturePointer()), 8 * (std::streamsize)n);
        for (int i = 0; i < n; ++i)
            out.write(reinterpret_cast<const char*>(mesh->getSpeciesPointer(i)), 8 * (std::streamsize)nsp);
        out.write(reinterpret_cast<const char*>(status.data()), 4 * (std::streamsize)n);
        out.write(reinterpret_cast<const char*>(mesh->getEnthalpyPointer()), 8 * (std::streamsize)n);
        return out ? 0 : 4;
    } catch (const std::exception& e) {
        std::cout << "EXCEPTION: " << e.what() << std::endl;
        return 3;
    }
}
