// Drop-in check: the reference's own objects drive the GPU path through its residual seam.
//
// A fv::Simulation is set up as the reference's tests do; its TimeScheme (SSP-RK3, SSP-RK2, MUSCL-Hancock, ...) then
// steps one copy of the state with the reference's Simulation::residual and another with fvg::GpuResidual (the C ABI of
// libfenice_gpu.so, include/fenice_gpu.hpp) passed as the `ResidualFn`. The adapter `to_fvg` below is the whole binding
// a maintainer adds to the reference: SimParams -> fvg_config. The two states and every step's (dt, s_max) must agree bit
// for bit. Built by oracle/ref/Makefile (target dropin_check, it needs the reference's sources and a built
// libfenice_gpu.so); run on a GPU host by tests/test_gpu_dropin.py.
//   dropin_check <case: vortex | tgv | riemann> <steps>
#include "fv/Params.hpp"
#include "fv/Schemes.hpp"
#include "fv/Simulation.hpp"
#include "fv/TestCases.hpp"
#include "fv/TimeScheme.hpp"

#include "fenice_gpu.hpp"

#include <cstdio>
#include <vector>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>

namespace fs = std::filesystem;

static int bc_code(const std::string& s) {
    const fv::BCType t = fv::parse_bc(s);
    return static_cast<int>(t);   // fvg's BC enumeration is the reference's BCType order
}

// The binding: the reference's typed parameters -> the C ABI's configuration.
static fvg_config to_fvg(const fv::SimParams& p) {
    fvg_config c{};
    c.nx = p.nx;
    c.ny = p.ny;
    c.nz = p.nz;
    c.Lx = p.Lx;
    c.Ly = p.Ly;
    c.Lz = p.Lz;
    std::string eos = p.eos_type;
    for (auto& ch : eos) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    c.eos_type = eos == "ideal gas" ? FVG_EOS_IDEAL : FVG_EOS_STIFFENED;
    c.gamma = p.gamma;
    c.p_inf = p.p_inf;
    const std::string* bcs[6] = {&p.bc_xmin, &p.bc_xmax, &p.bc_ymin, &p.bc_ymax, &p.bc_zmin, &p.bc_zmax};
    for (int s = 0; s < 6; ++s) c.bc[s] = bc_code(*bcs[s]);
    c.u_in = p.u_in;
    c.v_in = p.v_in;
    c.rho_in = p.rho_in;
    c.p_out = p.p_out;
    c.riemann = fv::parse_riemann(p.riemann_solver) == fv::RiemannType::LowMachHLLC ? FVG_RIEMANN_LOWMACH : FVG_RIEMANN_HLLC;
    c.shock_blend = p.shock_blend;
    c.reconstruction = p.reconstruction == "muscl" ? FVG_RECON_MUSCL
                       : p.reconstruction == "weno3" ? FVG_RECON_WENO3
                       : p.reconstruction == "weno5" ? FVG_RECON_WENO5 : FVG_RECON_NONE;
    c.limiter = static_cast<int>(fv::parse_limiter(p.muscl_limiter));
    c.weno_epsilon = p.weno_epsilon;
    c.boundary_order = p.boundary_order;
    c.time_scheme = static_cast<int>(fv::parse_time_scheme(p.time_scheme));
    c.cfl = p.cfl;
    c.dt_max = p.dt_max;
    c.use_viscous = p.use_viscous ? 1 : 0;
    c.mu = p.mu;
    c.pr = p.pr;
    c.precision = FVG_PREC_FP64;
    c.device = 0;
    c.use_ibm = p.use_ibm ? 1 : 0;
    std::string shape = p.ibm_shape;
    for (auto& ch : shape) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    c.ibm_shape = shape == "sphere" ? 1 : 0;
    c.ibm_radius = p.ibm_radius;
    c.ibm_cx = p.ibm_cx;
    c.ibm_cy = p.ibm_cy;
    c.ibm_cz = p.ibm_cz;
    c.ibm_curvature = p.ibm_curvature ? 1 : 0;
    c.use_bodyforce = p.use_bodyforce ? 1 : 0;
    c.gx = p.gx;
    c.gy = p.gy;
    c.gz = p.gz;
    c.nrbc_sigma = p.nrbc_sigma;
    c.nrbc_beta = p.nrbc_beta;
    c.positivity_fallback = p.positivity_fallback ? 1 : 0;
    // case-file expressions: the source terms, boundary values given as expressions of t, and every numeric parameter
    // bound by name (the strings live in `keep` until fvg_create has compiled them)
    static std::vector<std::string> keep;
    static std::vector<const char*> names;
    static std::vector<double> values;
    keep.clear();
    keep.reserve(64 + p.source.values().size());
    static const char* const skeys[5] = {"source_rho", "source_mx", "source_my", "source_E", "source_mz"};
    for (int q = 0; q < 5; ++q) c.source[q] = keep.emplace_back(p.source.str(skeys[q], "0")).c_str();
    static const char* const bkeys[4] = {"u_in", "v_in", "rho_in", "p_out"};
    for (int k = 0; k < 4; ++k) {
        const std::string raw = p.source.str(bkeys[k], k >= 2 ? "1.0" : "0.0");
        char* end = nullptr;
        std::strtod(raw.c_str(), &end);
        if (!(end && end != raw.c_str() && *end == '\0')) c.boundary_expr[k] = keep.emplace_back(raw).c_str();
    }
    names.clear();
    values.clear();
    for (const auto& [k, v] : p.source.values()) {
        char* end = nullptr;
        const double d = std::strtod(v.c_str(), &end);
        while (end && (*end == ' ' || *end == '\t')) ++end;
        if (!v.empty() && end && *end == '\0') {
            names.push_back(keep.emplace_back(k).c_str());
            values.push_back(d);
        }
    }
    c.param_names = names.data();
    c.param_values = values.data();
    c.nparams = (int)names.size();
    return c;
}

int main(int argc, char** argv) {
    if (fvg_abi_version() != FVG_ABI_VERSION) {   // fvg_config's layout must be the one this file was compiled with
        std::fprintf(stderr, "libfenice_gpu.so has ABI %d, this check was built for %d: rebuild it (make -C oracle/ref dropin)\n",
                     fvg_abi_version(), FVG_ABI_VERSION);
        return 2;
    }
    const std::string which = argc > 1 ? argv[1] : "vortex";
    const int nsteps = argc > 2 ? std::atoi(argv[2]) : 10;
    char tmpl[] = "/tmp/fenice_dropin_XXXXXX";
    if (!mkdtemp(tmpl)) return 2;
    const fs::path dir = tmpl;
    std::ofstream(dir / "case.toml") << "[case]\nname = \"dropin\"\n[initial]\n"
                                     << (which == "cylinder" ? "state = { rho = 1.4, u = 2.0, v = 0.0, p = 1.0 }\n"
                                         : which == "vortex" ? "profile = \"isentropic_vortex\"\n"
                                         : which == "tgv"  ? "profile = \"taylor_green_3d\"\n"
                                                           : "state = { rho = 1.0, u = 0.1, v = -0.2, p = 1.0 }\n[[initial.region]]\nshape = \"box\"\n"
                                                             "min = [0.0, 0.0]\nmax = [0.5, 0.5]\nstate = { rho = 0.5, u = 0.3, v = 0.1, p = 0.4 }\n");
    fv::Params P = fv::baseline_defaults();
    P.merge(fv::get_test_case((dir / "case.toml").string()).defaults);
    P.set("test_case", (dir / "case.toml").string());
    P.set("output_root", (dir / "out").string());
    if (which == "vortex") {
        for (auto kv : {std::pair<const char*, const char*>{"nx", "128"}, {"ny", "128"}, {"Lx", "10"}, {"Ly", "10"}, {"reconstruction", "muscl"},
                        {"muscl_limiter", "Van Leer"}, {"time_scheme", "MUSCL-Hancock"}, {"bc_xmin", "periodic"}, {"bc_xmax", "periodic"},
                        {"bc_ymin", "periodic"}, {"bc_ymax", "periodic"}})
            P.set(kv.first, kv.second);
    } else if (which == "cylinder") {
        for (auto kv : {std::pair<const char*, const char*>{"nx", "160"}, {"ny", "240"}, {"Lx", "8"}, {"Ly", "12"}, {"reconstruction", "muscl"},
                        {"muscl_limiter", "MC"}, {"time_scheme", "MUSCL-Hancock"}, {"bc_xmin", "vel_inlet"}, {"bc_xmax", "transmissive"},
                        {"bc_ymin", "transmissive"}, {"bc_ymax", "transmissive"}, {"u_in", "2.0"}, {"rho_in", "1.4"}, {"p_out", "1.0"},
                        {"use_ibm", "true"}, {"ibm_shape", "Cylinder"}, {"ibm_radius", "0.5"}, {"ibm_cx", "3.0"}, {"ibm_cy", "6.0"}})
            P.set(kv.first, kv.second);
    } else if (which == "tgv") {
        for (auto kv : {std::pair<const char*, const char*>{"nx", "32"}, {"ny", "32"}, {"nz", "32"}, {"Lx", "6.283185307179586"},
                        {"Ly", "6.283185307179586"}, {"Lz", "6.283185307179586"}, {"reconstruction", "weno5"}, {"riemann_solver", "HLLC (Low-Mach Thornber)"},
                        {"time_scheme", "SSP Runge-Kutta 3"}, {"use_viscous", "true"}, {"mu", "6.25e-4"}, {"pr", "0.71"}, {"bc_xmin", "periodic"},
                        {"bc_xmax", "periodic"}, {"bc_ymin", "periodic"}, {"bc_ymax", "periodic"}})
            P.set(kv.first, kv.second);
    } else if (which == "sources") {   // unsteady sources and boundary values of t (arithmetic: the same bits on the device)
        for (auto kv : {std::pair<const char*, const char*>{"nx", "64"}, {"ny", "48"}, {"Lx", "2"}, {"Ly", "1"}, {"reconstruction", "muscl"},
                        {"muscl_limiter", "MC"}, {"time_scheme", "MUSCL-Hancock"}, {"bc_xmin", "vel_inlet"}, {"bc_xmax", "outlet"},
                        {"bc_ymin", "periodic"}, {"bc_ymax", "periodic"}, {"u_in", "0.3 + 0.5*t"}, {"v_in", "0.05*t"}, {"p_out", "1 - 0.1*t"},
                        {"source_rho", "0.01*(x - 0.5)*(y - 0.25)*(1 + t)"}, {"source_mx", "0.02*x*x - 0.01*t"}, {"source_my", "-0.03*y*t"},
                        {"source_E", "0.05*(x + y)*(1 - 2*t) + gamma*0.001"}})
            P.set(kv.first, kv.second);
    } else if (which == "sources_rk3") {   // steady sources with transcendental functions (evaluated once on the host)
        for (auto kv : {std::pair<const char*, const char*>{"nx", "48"}, {"ny", "48"}, {"reconstruction", "weno5"}, {"time_scheme", "SSP Runge-Kutta 3"},
                        {"bc_xmin", "periodic"}, {"bc_xmax", "periodic"}, {"bc_ymin", "periodic"}, {"bc_ymax", "periodic"},
                        {"source_rho", "0.1*sin(2*pi*x)*cos(2*pi*y)"}, {"source_mx", "0.05*exp(-x)"}, {"source_my", "0.02*log(1 + y)"},
                        {"source_E", "0.2*tanh(x - y)"}})
            P.set(kv.first, kv.second);
    } else {
        for (auto kv : {std::pair<const char*, const char*>{"nx", "96"}, {"ny", "96"}, {"reconstruction", "weno5"}, {"time_scheme", "SSP Runge-Kutta 3"},
                        {"cfl", "0.4"}, {"bc_xmin", "transmissive"}, {"bc_xmax", "transmissive"}, {"bc_ymin", "transmissive"},
                        {"bc_ymax", "transmissive"}})
            P.set(kv.first, kv.second);
    }
    fv::Simulation ref, host;
    ref.setup(fv::SimParams::from(P), false);
    ref.initialize_field();
    host.setup(fv::SimParams::from(P), false);   // its TimeScheme drives the GPU residual
    host.initialize_field();

    fvg::GpuRun run(to_fvg(host.p));
    fvg::GpuResidual<fv::Field> gpu(run);
    const fv::ResidualFn gpu_res = [&](const fv::Field& U, fv::Field& R) {
        gpu.predictor_half_dt = host.scheme->predictor_half_dt;
        gpu.stage_time = host.scheme->stage_time;
        return gpu(U, R);
    };
    const fv::ResidualFn ref_res = [&](const fv::Field& U, fv::Field& R) { return ref.residual(U, R); };
    double t_ref = 0.0, t_gpu = 0.0;
    int bad = 0;
    for (int k = 0; k < nsteps; ++k) {
        const fv::StepResult a = ref.scheme->step(ref.U, ref_res, ref.dt_length, t_ref, 1e30, 0.0);
        const fv::StepResult b = host.scheme->step(host.U, gpu_res, host.dt_length, t_gpu, 1e30, 0.0);
        t_ref += a.dt;
        t_gpu += b.dt;
        if (std::memcmp(&a.dt, &b.dt, sizeof(double)) || std::memcmp(&a.s_max, &b.s_max, sizeof(double))) ++bad;
    }
    const bool same = std::memcmp(ref.U.data(), host.U.data(), ref.U.size() * sizeof(fv::State)) == 0;
    std::printf("dropin %s: %d steps, t = %.17g, dt/s_max mismatches %d, state %s\n", which.c_str(), nsteps, t_gpu, bad,
                same ? "bit-identical" : "DIFFERS");
    std::error_code ec;
    fs::remove_all(dir, ec);
    return (same && bad == 0) ? 0 : 1;
}
