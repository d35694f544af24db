// Drop-in replacement for the reference's kmc_solver.hpp: BarrierGenerator,
// KmcSimulation2D and KmcSimulation3D with the reference's constructors and
// run_simulation / elastic_run signatures, running on the GPU through
// libmgkmc_b200 (include/mgkmc_b200.h).  A caller such as the reference's
// main.cpp, compiled with this directory ahead of the reference's on its
// include path and linked with -lmgkmc_b200, builds unchanged and writes the
// same logs.
//
// The simulation state lives on the device; the public field members
// (eps_field, sig_field, eps_plastic, soft_prop) are host copies refreshed
// after run_simulation and elastic_run (with fast patching, sig_field is the
// kept, stencil-updated stress, as in the reference).  Errors throw
// std::runtime_error.
#pragma once
#include <Eigen/Dense>

#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../mgkmc_b200.h"
#include "linear_elastic_solver.hpp"

std::string get_current_timestamp();  // kmc_solver.hpp:22 (defined by the caller, as in the reference)

// kmc_solver.hpp:24-33: the barrier distribution and its parameters
struct BarrierGenerator {
    std::string type;
    double mean = 2.0;
    double std_val = 0.6;
    double min_cutoff = 0.1;
    double max_cutoff = -1.0;
    double loc = 1.0;
    double scale = 0.5;
    double epsilon = 0.1;
    double ratio = 0.8;
};

namespace mgk_shim {

inline int barrier_code(const std::string& t) {
    if (t == "gaussian" || t.empty()) return 0;
    if (t == "rayleigh") return 1;
    if (t == "modified_rayleigh") return 2;
    if (t == "modified_rayleigh_with_exponential") return 3;
    throw std::runtime_error("unknown barrier type: " + t);
}

inline void check(mgk_status s, const char* what) {
    if (s != MGK_OK && s != MGK_TERMINATED)  // the reference's instability stop returns normally
        throw std::runtime_error(std::string(what) + ": " + mgk_last_error());
}

// The common part of KmcSimulation2D / 3D: parameters, handle, run.
template <int D>
class KmcBase {
public:
    using Mat = Eigen::Matrix<double, D, D>;
    int nx, ny, nz, M;
    std::vector<Mat> eps_field, sig_field, eps_plastic;
    std::vector<Eigen::Vector2d> soft_prop;

    KmcBase(const KmcBase&) = delete;
    KmcBase& operator=(const KmcBase&) = delete;
    ~KmcBase() {
        if (h_) mgk_kmc_destroy(h_);
    }

    // kmc_solver.hpp:721-729 (checkpointing is not implemented by the
    // reference either; track_cascades only adds a reference log detail)
    void run_simulation(int n_global_steps, double step_size, std::pair<int, int> component,
                        const std::map<std::pair<int, int>, double>& stress_targets, double mixed_tol = 1e-4,
                        int mixed_max_iter = 50, std::string /*checkpoint_interval*/ = "none",
                        std::string /*checkpoint_path*/ = "checkpoint", std::string vtk_interval = "none",
                        bool vtk_elastic_only = true, bool /*track_cascades*/ = false, bool enable_console_log = true,
                        std::string summary_filename = "summary_log.txt", bool enable_summary_log = true,
                        bool enable_global_log = true, double max_kmc_steps_pct = 0.3) {
        mgk_run_params r{};
        r.n_global_steps = n_global_steps;
        r.step_size = step_size;
        r.comp_i = component.first;
        r.comp_j = component.second;
        r.n_targets = 0;
        for (const auto& t : stress_targets) {  // std::map iterates sorted by (i, j)
            if (r.n_targets == 9) break;
            r.target_i[r.n_targets] = t.first.first;
            r.target_j[r.n_targets] = t.first.second;
            r.target_v[r.n_targets] = t.second;
            ++r.n_targets;
        }
        r.mixed_tol = mixed_tol;
        r.mixed_max_iter = mixed_max_iter;
        r.max_kmc_steps_pct = max_kmc_steps_pct;
        r.max_events = 0;
        r.output_dir = output_dir_.c_str();
        r.summary_filename = summary_filename.c_str();
        r.enable_summary_log = enable_summary_log;
        r.enable_global_log = enable_global_log;
        r.enable_console = enable_console_log;
        r.vtk_interval = vtk_interval.c_str();
        r.vtk_elastic_only = vtk_elastic_only;
        r.max_cascade_batches = 0;
        check(mgk_kmc_run(h_, &r, nullptr, 0, nullptr), "run_simulation");
        sync_fields();
    }

    // kmc_solver.hpp:334-339 / :1333-1338
    void elastic_run() {
        check(mgk_kmc_elastic_run(h_), "elastic_run");
        sync_fields();
    }

    // host copies of the device fields
    void sync_fields() {
        const size_t N = (size_t)nx * ny * nz;
        std::vector<double> buf(N * D * D);
        auto tensors = [&](int id, std::vector<Mat>& out) {
            check(mgk_kmc_get_field(h_, id, buf.data(), nullptr), "get_field");
            out.resize(N);
            for (size_t v = 0; v < N; ++v)
                for (int i = 0; i < D; ++i)
                    for (int j = 0; j < D; ++j) out[v](i, j) = buf[v * D * D + i * D + j];
        };
        tensors(0, eps_field);
        tensors(1, sig_field);
        tensors(2, eps_plastic);
        std::vector<double> sp(2 * N);
        check(mgk_kmc_get_field(h_, 3, sp.data(), nullptr), "get_field");
        soft_prop.resize(N);
        for (size_t v = 0; v < N; ++v) {
            soft_prop[v](0) = sp[2 * v];
            soft_prop[v](1) = sp[2 * v + 1];
        }
    }

    mgk_kmc* handle() const { return h_; }

protected:
    KmcBase() = default;
    void create(int nx_, int ny_, int nz_, int M_, double gamma0, const std::vector<double>& E,
                const std::vector<double>& nu, double pixel, const BarrierGenerator& bg, const std::string& scheme,
                double cap, double jp, double jt, double neigh, double q_act, const std::string& out_dir, double T,
                double rate, double thr, double nu0, bool plane_stress, bool fp, int fp_r, int fp_sync,
                const std::string& instab, bool scale_vol, bool redraw_d, bool redraw_b, bool b3d, int seed) {
        nx = nx_, ny = ny_, nz = nz_, M = M_;
        output_dir_ = out_dir;
        mgk_kmc_params p{};
        p.dim = D;
        p.nx = nx_, p.ny = ny_, p.nz = nz_, p.M = M_;
        p.plane_stress = plane_stress ? 1 : 0;
        p.seed = seed;
        p.gamma0 = gamma0;
        p.pixel = pixel;
        p.barrier_type = barrier_code(bg.type);
        p.bar_mean = bg.mean, p.bar_std = bg.std_val, p.bar_min_cutoff = bg.min_cutoff, p.bar_max_cutoff = bg.max_cutoff;
        p.bar_loc = bg.loc, p.bar_scale = bg.scale, p.bar_epsilon = bg.epsilon, p.bar_ratio = bg.ratio;
        p.directional = scheme == "directional" ? 1 : 0;
        p.softening_cap = cap, p.jp = jp, p.jt = jt, p.neighbor_fraction = neigh, p.q_act_temp = q_act;
        p.temperature = T, p.strain_rate = rate, p.stability_threshold = thr, p.nu0 = nu0;
        p.instability_kmc = instab == "kmc" ? 1 : 0;
        p.scale_rate_by_volume = scale_vol, p.redraw_directions = redraw_d, p.redraw_barriers = redraw_b;
        p.use_3d_barriers = b3d;
        p.fast_patching = fp, p.patch_radius = fp_r, p.sync_interval = fp_sync;
        p.ls_tol = 1e-6;   // elastic_run's tolerance and iteration cap (kmc_solver.hpp:337)
        p.ls_max_iter = 200;
        check(mgk_kmc_create(&h_, &p, E.data(), nu.data()), "KmcSimulation");
        sync_fields();
    }

    mgk_kmc* h_ = nullptr;
    std::string output_dir_;
};

}  // namespace mgk_shim

// kmc_solver.hpp:165-182: the same 27 arguments and defaults
class KmcSimulation2D : public mgk_shim::KmcBase<2> {
public:
    KmcSimulation2D(int nx_, int ny_, int M_, double gamma0_, const std::vector<double>& E_field_,
                    const std::vector<double>& nu_field_, double pixel_ = 1.0,
                    const BarrierGenerator& barrier_gen_ = BarrierGenerator(),
                    std::string softening_scheme_ = "isotropic", double softening_cap_ = 2.0, double jp_ = 10.0,
                    double jt_ = 30.0, double neighbor_softening_fraction_ = 0.0, double q_act_temp_ = 0.37,
                    std::string output_dir_ = "output", double temperature_ = 0.0, double strain_rate_ = 1.0,
                    double stability_threshold_ = 0.0, double nu0_ = 1e13, std::string plane_mode_ = "plane_strain",
                    bool fast_patching_enabled_ = false, int patch_radius_ = 5, int sync_interval_ = 100,
                    std::string instability_mode_ = "cascade", std::string /*cascade_timing_*/ = "none",
                    bool scale_rate_by_volume_ = true, bool redraw_directions_ = true, bool redraw_barriers_ = true,
                    int seed_ = 42) {
        create(nx_, ny_, 1, M_, gamma0_, E_field_, nu_field_, pixel_, barrier_gen_, softening_scheme_, softening_cap_,
               jp_, jt_, neighbor_softening_fraction_, q_act_temp_, output_dir_, temperature_, strain_rate_,
               stability_threshold_, nu0_, plane_mode_ == "plane_stress", fast_patching_enabled_, patch_radius_,
               sync_interval_, instability_mode_, scale_rate_by_volume_, redraw_directions_, redraw_barriers_, false,
               seed_);
    }
};

// kmc_solver.hpp:1142-1158: the same 28 arguments and defaults
class KmcSimulation3D : public mgk_shim::KmcBase<3> {
public:
    KmcSimulation3D(int nx_, int ny_, int nz_, int M_, double gamma0_, const std::vector<double>& E_field_,
                    const std::vector<double>& nu_field_, double pixel_ = 1.0,
                    const BarrierGenerator& barrier_gen_ = BarrierGenerator(),
                    std::string softening_scheme_ = "isotropic", double softening_cap_ = 2.0, double jp_ = 10.0,
                    double jt_ = 30.0, double neighbor_softening_fraction_ = 0.0, double q_act_temp_ = 0.37,
                    std::string output_dir_ = "output", double temperature_ = 0.0, double strain_rate_ = 1.0,
                    double stability_threshold_ = 0.0, double nu0_ = 1e13, bool fast_patching_enabled_ = false,
                    int patch_radius_ = 5, int sync_interval_ = 100, std::string instability_mode_ = "cascade",
                    std::string /*cascade_timing_*/ = "none", bool scale_rate_by_volume_ = true,
                    bool redraw_directions_ = true, bool redraw_barriers_ = true, bool use_3d_barriers_ = false,
                    int seed_ = 42) {
        create(nx_, ny_, nz_, M_, gamma0_, E_field_, nu_field_, pixel_, barrier_gen_, softening_scheme_, softening_cap_,
               jp_, jt_, neighbor_softening_fraction_, q_act_temp_, output_dir_, temperature_, strain_rate_,
               stability_threshold_, nu0_, false, fast_patching_enabled_, patch_radius_, sync_interval_,
               instability_mode_, scale_rate_by_volume_, redraw_directions_, redraw_barriers_, use_3d_barriers_, seed_);
    }
};
