// extern "C" harness over the compiled reference solver (test infrastructure, built into oracle/_ref/ by
// oracle/ref/Makefile). It drives the reference's own objects exactly as its unit tests and its time loop do:
//   * a run is fv::Simulation::setup of SimParams::from(baseline_defaults + case + overrides)
//     (cpp/tests/test_common.hpp:83-90), then initialize_field (cpp/src/Simulation.cpp:609-627);
//   * one residual is Simulation::residual with the scheme's stage_time / predictor_half_dt set
//     (cpp/src/Simulation.cpp:1351-1354, cpp/include/fv/TimeScheme.hpp:88-92);
//   * one step is the body of the serial time loop: scheme->step, check_progress, the solid reset of the
//     immersed body, t += dt (cpp/src/SimulationRun.cpp:441-464).
// Nothing here changes the reference's arithmetic; it only moves arrays across the C ABI.
#include "fv/CellAdvance.hpp"
#include "fv/CellFlux.hpp"
#include "fv/CellMesh.hpp"
#include "fv/Params.hpp"
#include "fv/Physics.hpp"
#include "fv/Simulation.hpp"
#include "fv/TestCases.hpp"
#include "fv/TimeScheme.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>

namespace fs = std::filesystem;

namespace {

thread_local std::string g_error;

struct RefRun {
    fv::Simulation sim;
    fs::path dir;
    int steps = 0;
};

// The cell engine of the adaptive mesh on a run's objects, as the reference's level-0 tests build it
// (cpp/tests/test_amr_octree_advance.cpp:17-49, cpp/tests/test_amr_mesh.cpp:484-530): the CellMesh of the run's base mesh
// with its periodic axes, a CellFluxEngine on the run's EOS, Riemann solver, reconstruction and boundaries, and a
// CellAdvance with a time scheme of the run's type. The run must outlive it.
struct RefCells {
    std::unique_ptr<fv::CellMesh> mesh;
    std::unique_ptr<fv::CellFluxEngine> eng;
    std::unique_ptr<fv::TimeScheme> ts;
    std::unique_ptr<fv::CellAdvance> adv;
};

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r");
    return s.substr(a, b - a + 1);
}

// The case file the run is set up from: only its initial condition matters, every parameter comes as an override.
std::string case_text(const std::string& profile, const std::string& state) {
    std::ostringstream o;
    o << "[case]\nname = \"oracle run\"\ndescription = \"oracle harness\"\n\n[initial]\n";
    if (!profile.empty()) {
        o << "profile = \"" << profile << "\"\n";
    } else {
        double v[5] = {1.0, 0.0, 0.0, 1.0, 0.0};
        std::stringstream ss(state);
        std::string item;
        for (int q = 0; q < 5 && std::getline(ss, item, ','); ++q) v[q] = std::stod(item);
        char buf[256];
        std::snprintf(buf, sizeof buf, "state = { rho = %.17g, u = %.17g, v = %.17g, p = %.17g, w = %.17g }\n", v[0], v[1], v[2], v[3], v[4]);
        o << buf;
    }
    return o.str();
}

}   // namespace

extern "C" {

const char* ref_error() { return g_error.c_str(); }

// kv: "key=value" lines. Keys of the reference's parameter table, plus initial_profile (isentropic_vortex,
// taylor_green_3d, taylor_green) or initial_state ("rho,u,v,p[,w]", a uniform field), or case (a test case name of
// the reference or a case folder / case.toml: its defaults and its own initial condition, as `fenice --case`).
void* ref_create(const char* kv) {
    try {
        auto* r = new RefRun();
        char tmpl[] = "/tmp/fenice_ref_XXXXXX";
        if (!mkdtemp(tmpl)) throw std::runtime_error("mkdtemp failed");
        r->dir = tmpl;
        std::string profile, state = "1,0,0,1,0", case_name;
        fv::Params p = fv::baseline_defaults();
        std::stringstream ss(kv ? kv : "");
        std::string line;
        std::vector<std::pair<std::string, std::string>> over;
        while (std::getline(ss, line)) {
            line = trim(line);
            if (line.empty()) continue;
            const size_t eq = line.find('=');
            if (eq == std::string::npos) throw std::invalid_argument("bad override line: " + line);
            const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
            if (k == "initial_profile")
                profile = v;
            else if (k == "initial_state")
                state = v;
            else if (k == "case")
                case_name = v;
            else
                over.emplace_back(k, v);
        }
        std::string cf = case_name;
        if (cf.empty()) {
            cf = (r->dir / "case.toml").string();
            std::ofstream f(cf);
            f << case_text(profile, state);
        }
        const fv::TestCase& tc = fv::get_test_case(cf);
        p.merge(tc.defaults);
        p.set("test_case", cf);
        p.set("output_root", (r->dir / "out").string());
        p.set("save_interval", "1000000000");
        for (const auto& e : over) p.set(e.first, e.second);
        r->sim.setup(fv::SimParams::from(p), false);
        r->sim.initialize_field();
        return r;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void ref_destroy(void* h) {
    auto* r = static_cast<RefRun*>(h);
    if (!r) return;
    std::error_code ec;
    fs::remove_all(r->dir, ec);
    delete r;
}

int ref_dims(void* h, int* nx, int* ny, int* nz) {
    auto* r = static_cast<RefRun*>(h);
    *nx = r->sim.mesh.nx;
    *ny = r->sim.mesh.ny;
    *nz = r->sim.mesh.nz;
    return 0;
}

double ref_time(void* h) { return static_cast<RefRun*>(h)->sim.t; }
double ref_dt_length(void* h) { return static_cast<RefRun*>(h)->sim.dt_length; }
double ref_lagged_speed(void* h) { return static_cast<RefRun*>(h)->sim.scheme->lagged_speed(); }

int ref_get_state(void* h, double* U) {
    auto* r = static_cast<RefRun*>(h);
    std::memcpy(U, r->sim.U.data(), r->sim.U.size() * sizeof(fv::State));
    return 0;
}

// Replace the state; with `force` the immersed body's ghost cells are forced as initialize_field does for a fresh start.
int ref_set_state(void* h, const double* U, int force) {
    auto* r = static_cast<RefRun*>(h);
    std::memcpy(r->sim.U.data(), U, r->sim.U.size() * sizeof(fv::State));
    if (force && r->sim.p.use_ibm && r->sim.ibm) r->sim.ibm->apply_forcing(r->sim.U, r->sim.fluid);
    return 0;
}

void ref_set_time(void* h, double t) { static_cast<RefRun*>(h)->sim.t = t; }

// One residual of the state U (AoS, 5 per cell) at stage_time, with the MUSCL-Hancock predictor of half a step
// `predictor_half_dt` (0: none). R gets the residual, *smax the wave speed the residual returns.
int ref_residual(void* h, const double* U, double* R, double stage_time, double predictor_half_dt, double* smax) {
    auto* r = static_cast<RefRun*>(h);
    try {
        fv::Field Uin(r->sim.U.size()), Rout;
        std::memcpy(Uin.data(), U, Uin.size() * sizeof(fv::State));
        r->sim.scheme->stage_time = stage_time;
        r->sim.scheme->predictor_half_dt = predictor_half_dt;
        const double s = r->sim.residual(Uin, Rout);
        r->sim.scheme->predictor_half_dt = 0.0;
        std::memcpy(R, Rout.data(), Rout.size() * sizeof(fv::State));
        *smax = s;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// `n` steps of the serial time loop toward t_end (fewer if t reaches t_end); per step the dt and wave speed are
// written to dts / smaxs when those are not null. Returns the number of steps taken, or -1 on an error.
int ref_steps(void* h, int n, double t_end, double* dts, double* smaxs) {
    auto* r = static_cast<RefRun*>(h);
    try {
        fv::Simulation& s = r->sim;
        const fv::ResidualFn res = [&s](const fv::Field& Uin, fv::Field& R) { return s.residual(Uin, R); };
        int k = 0;
        for (; k < n && s.t < t_end; ++k) {
            const fv::StepResult st = s.scheme->step(s.U, res, s.dt_length, s.t, t_end, s.p.dt_max);
            if (!(std::isfinite(st.s_max) && std::isfinite(st.dt) && s.t + st.dt > s.t))
                throw std::runtime_error("the solution diverged");
            if (s.p.use_ibm) s.ibm->apply_solid_reset(s.U, s.fluid);
            s.t += st.dt;
            s.scheme->stage_time = s.t;
            if (dts) dts[k] = st.dt;
            if (smaxs) smaxs[k] = st.s_max;
            ++r->steps;
        }
        return k;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The IBM solid mask (1 = solid cell) into `mask` (one byte per cell); returns the number of solid cells, or -1 without a body.
int ref_solid_mask(void* h, char* mask) {
    auto* r = static_cast<RefRun*>(h);
    if (!r->sim.p.use_ibm || !r->sim.ibm) return -1;
    const std::vector<char>& m = r->sim.ibm->mask();
    int n = 0;
    for (size_t c = 0; c < m.size(); ++c) {
        mask[c] = m[c];
        n += m[c] != 0;
    }
    return n;
}

// The immersed body's loads {Fx, Fy, Mz} of the current state, as the monitor takes them (Simulation::ibm_loads on a
// residual of U with the predictor off); returns -1 without a body or on an error.
int ref_ibm_loads(void* h, double* loads) {
    auto* r = static_cast<RefRun*>(h);
    if (!r->sim.p.use_ibm || !r->sim.ibm) return -1;
    try {
        fv::Field R;
        r->sim.scheme->stage_time = r->sim.t;
        r->sim.scheme->predictor_half_dt = 0.0;
        r->sim.residual(r->sim.U, R);
        const std::array<double, 3> f = r->sim.ibm_loads(r->sim.mesh, *r->sim.ibm, r->sim.U, R);
        loads[0] = f[0];
        loads[1] = f[1];
        loads[2] = f[2];
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The monitor's volume averages {mass, kinetic energy, total energy} of the current state (Simulation::volume_averages
// over every cell, as the serial time loop's monitor row takes them).
int ref_volume_averages(void* h, double* out) {
    auto* r = static_cast<RefRun*>(h);
    const std::array<double, 3> v = r->sim.volume_averages(r->sim.U, static_cast<long long>(r->sim.U.size()));
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
    return 0;
}

// ---- the level-0 cell engine (see RefCells)

void* ref_cells_create(void* h, int max_level) {
    try {
        auto* r = static_cast<RefRun*>(h);
        const fv::Simulation& sim = r->sim;
        const fv::Mesh& u = sim.mesh;
        auto per = [&](int a) { return sim.boundaries.type(static_cast<fv::Face>(2 * a)) == fv::BCType::Periodic; };
        auto* c = new RefCells();
        if (u.nz > 1)
            c->mesh = std::make_unique<fv::CellMesh>(fv::CellMesh::make_3d(u.Lx, u.Ly, u.Lz, u.nx, u.ny, u.nz, max_level, per(0), per(1), per(2), u.x0, u.y0, u.z0));
        else
            c->mesh = std::make_unique<fv::CellMesh>(u.Lx, u.Ly, u.nx, u.ny, max_level, per(0), per(1), u.x0, u.y0);
        c->mesh->U.assign(static_cast<size_t>(c->mesh->num_leaves()), fv::State{});
        c->eng = std::make_unique<fv::CellFluxEngine>(sim.fluid, sim.riemann, sim.muscl.get(), sim.boundaries);
        if (sim.ns || sim.body_force) {   // the viscous terms and the body force, as the reference's tests set them (physics_of,
                                          // cpp/tests/test_amr_common.hpp:424-438)
            fv::CellPhysics ph;
            ph.ns = sim.ns.get();
            ph.body = sim.body_force.get();
            c->eng->set_physics(ph);
        }
        c->eng->build(*c->mesh);
        c->ts = fv::make_time_scheme(fv::parse_time_scheme(sim.p.time_scheme), sim.p.cfl);
        c->adv = std::make_unique<fv::CellAdvance>(*c->mesh, *c->eng, *c->ts);
        return c;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void ref_cells_destroy(void* hc) { delete static_cast<RefCells*>(hc); }

int ref_cells_count(void* hc, int* nleaf, int* nface) {
    auto* c = static_cast<RefCells*>(hc);
    *nleaf = c->mesh->num_leaves();
    *nface = static_cast<int>(c->mesh->faces.size());
    return 0;
}

int ref_cells_leaves(void* hc, int* level, int* ci, int* cj, int* ck) {
    const fv::CellMesh& m = *static_cast<RefCells*>(hc)->mesh;
    for (int l = 0; l < m.num_leaves(); ++l) {
        level[l] = m.level[l];
        ci[l] = m.ci[l];
        cj[l] = m.cj[l];
        ck[l] = m.ck[l];
    }
    return 0;
}

int ref_cells_set_state(void* hc, const double* U) {
    fv::CellMesh& m = *static_cast<RefCells*>(hc)->mesh;
    for (int l = 0; l < m.num_leaves(); ++l)
        for (int q = 0; q < 5; ++q) m.U[l][q] = U[5 * l + q];
    return 0;
}

int ref_cells_get_state(void* hc, double* U) {
    const fv::CellMesh& m = *static_cast<RefCells*>(hc)->mesh;
    for (int l = 0; l < m.num_leaves(); ++l)
        for (int q = 0; q < 5; ++q) U[5 * l + q] = m.U[l][q];
    return 0;
}

// CellFluxEngine::residual of the state held
int ref_cells_residual(void* hc, double* R, double* smax) {
    try {
        auto* c = static_cast<RefCells*>(hc);
        fv::Field Rf;
        *smax = c->eng->residual(*c->mesh, c->mesh->U, Rf);
        for (size_t l = 0; l < Rf.size(); ++l)
            for (int q = 0; q < 5; ++q) R[5 * l + q] = Rf[l][q];
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// CellAdvance::step(dt, t) of the state held, n times from t0 (step k at t0 + k dt); smax: the speed of each step
int ref_cells_steps(void* hc, double dt, double t0, int n, double* smax) {
    try {
        auto* c = static_cast<RefCells*>(hc);
        for (int k = 0; k < n; ++k) smax[k] = c->adv->step(dt, t0 + k * dt);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

}   // extern "C"
