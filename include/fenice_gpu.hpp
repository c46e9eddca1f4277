// fenice_gpu.hpp: header-only C++17 adapter over the C ABI (fenice_gpu.h), for C++ callers of the reference's interface.
//
//   fvg::GpuRun run(cfg);                       // fvg_create; throws like the reference (invalid_argument / runtime_error)
//   fvg::GpuResidual<Field> res(run);           // a drop-in for `ResidualFn` (cpp/include/fv/TimeScheme.hpp:14):
//   double s = res(U, R);                       //   R = residual(U), returns the wave speed (Simulation::residual)
//   fvg::StepResult r = run.step(U, t_end);     // TimeScheme::step + check_progress + t += dt, state kept on the device
//
// `Field` is any contiguous container of 5-double states in the reference's order [rho, rho u, rho v, rho E, rho w]
// (e.g. the reference's std::vector<std::array<double, 5>>).
#pragma once

#include <limits>
#include <stdexcept>
#include <string>

#include "fenice_gpu.h"

namespace fvg {

struct StepResult {
    double dt = 0.0;
    double s_max = 0.0;
};

inline void check(int rc, const char* what, const char* msg) {
    if (rc == FVG_OK) return;
    const std::string m = std::string(what) + ": " + (msg ? msg : "");
    if (rc == FVG_ERR_CONFIG || rc == FVG_ERR_ARGUMENT || rc == FVG_ERR_STATE) throw std::invalid_argument(m);
    throw std::runtime_error(m);
}

class GpuRun {
public:
    explicit GpuRun(const fvg_config& cfg) {
        const int rc = fvg_create(&cfg, &h_);
        check(rc, "fvg_create", fvg_create_error());
        ncells_ = static_cast<size_t>(cfg.nx) * cfg.ny * cfg.nz;
    }
    ~GpuRun() { fvg_destroy(h_); }
    GpuRun(const GpuRun&) = delete;
    GpuRun& operator=(const GpuRun&) = delete;

    fvg_run* handle() const { return h_; }
    size_t ncells() const { return ncells_; }

    template <class Field> void upload(const Field& U) {
        if (U.size() != ncells_) throw std::invalid_argument("state size is not the mesh's");
        check(fvg_upload_state(h_, U.data()->data(), U.size()), "upload", fvg_last_error(h_));
    }
    template <class Field> void download(Field& U) const {
        U.resize(ncells_);
        check(fvg_download_state(h_, U.data()->data(), U.size()), "download", fvg_last_error(h_));
    }
    // R = residual of the run's state (predictor_half_dt > 0: with the MUSCL-Hancock predictor); returns the wave speed
    template <class Field> double residual(Field& R, double predictor_half_dt = 0.0) {
        R.resize(ncells_);
        double s = 0.0;
        check(fvg_residual(h_, predictor_half_dt, R.data()->data(), R.size(), &s), "residual", fvg_last_error(h_));
        return s;
    }
    // one step of the time loop on the device state toward t_end
    StepResult step(double t_end) {
        StepResult r;
        check(fvg_step(h_, t_end, &r.dt, &r.s_max), "step", fvg_last_error(h_));
        return r;
    }
    // the same on a host state, updated in place (fvg_step_host: the bits of upload + step + download, the copies
    // overlapped with the first and last stages where the run allows it; pin U's memory for the overlap)
    template <class Field> StepResult step(Field& U, double t_end) {
        StepResult r;
        double* p = U.data()->data();
        check(fvg_step_host(h_, p, p, U.size(), t_end, &r.dt, &r.s_max), "step", fvg_last_error(h_));
        return r;
    }
    int run_until(double t_end, int max_steps = 0) {
        int n = 0;
        check(fvg_run_until(h_, t_end, max_steps, &n), "run_until", fvg_last_error(h_));
        return n;
    }
    double time() const {
        double t = 0.0;
        check(fvg_get_time(h_, &t), "time", fvg_last_error(h_));
        return t;
    }
    void set_time(double t) { check(fvg_set_time(h_, t), "time", fvg_last_error(h_)); }
    // the time the next residual evaluates time-dependent sources and boundary values at (NaN: the run's time)
    void set_stage_time(double t) { check(fvg_set_stage_time(h_, t), "stage time", fvg_last_error(h_)); }

private:
    fvg_run* h_ = nullptr;
    size_t ncells_ = 0;
};

// The residual seam of the reference (`ResidualFn`): usable wherever a `std::function<double(const Field&, Field&)>` is,
// e.g. as the `res` argument of the reference's TimeScheme::step. `predictor_half_dt` and `stage_time` are read at each
// call, so a caller sets them from its scheme's predictor_half_dt and stage_time before the call (stage_time NaN: the
// run's time).
template <class Field> class GpuResidual {
public:
    explicit GpuResidual(GpuRun& run) : run_(run) {}
    double operator()(const Field& U, Field& R) {
        run_.upload(U);
        run_.set_stage_time(stage_time);
        return run_.residual(R, predictor_half_dt);
    }
    double predictor_half_dt = 0.0;
    double stage_time = std::numeric_limits<double>::quiet_NaN();

private:
    GpuRun& run_;
};

}   // namespace fvg
