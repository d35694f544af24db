// ref_driver: test-infrastructure harness around the UNMODIFIED mgkmc_cpp headers.
//
// Built by oracle/Makefile from the reference sources where they lie (the
// reference headers are included, never copied).  It is the checker for the
// CUDA path and the timed CPU reference arm; nothing in the product links it.
//
// Commands (all arrays are .npy float64, C order):
//   ls2d DIR   spectral_solver_2d (linear_elastic_solver.hpp:146-309) on
//              DIR/{E,nu}.npy, optional DIR/eps0.npy (N x 4, row-major 2x2:
//              xx,xy,yx,yy) warm start and DIR/epsp.npy; parameters in
//              DIR/params.txt "nx ny plane_mode pixel max_iter tol e00 e01 e10 e11".
//              Gamma is built as KmcSimulation2D::init_gamma does
//              (kmc_solver.hpp:259-274).  Writes DIR/out_{eps,sig,macro}.npy.
//   ls3d DIR   spectral_solver_3d (linear_elastic_solver.hpp:431-593); params
//              "nx ny nz pixel max_iter tol e00 e01 e02 e10 ... e22"; 3x3 row-major.
//   kmc_run CFG OUT NSTEPS
//              builds KmcSimulation2D/3D from a YAML file with the key surface of
//              main.cpp:40-377 and calls the reference's own run_simulation
//              (kmc_solver.hpp:721 / :1735) for NSTEPS elastic steps, then dumps
//              the final state and OUT/timing.txt (wall seconds, KMC events).
//   kmc_trace CFG OUT NSTEPS MAXEV
//              same construction, then drives the reference object's public
//              methods (update_barriers, find_unstable_indices, run_cascade,
//              apply_flip_soa_*, elastic_run) through the control flow of
//              run_simulation, recording one row per event in OUT/trace.npy.
//              Stops after NSTEPS elastic steps or MAXEV thermal events.
//   kmc_init CFG OUT  construct only, dump the initial state (Q0, catalog, ...).
//   draws SEED N OUT  dump N uniform/normal draws of std::mt19937 + libstdc++
//              distributions (pins the RNG restatement of the oracle).
#include <Eigen/Dense>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

std::string get_current_timestamp() {
    std::time_t t = std::time(nullptr);
    char buf[64];
    std::strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S", std::localtime(&t));
    return buf;
}

#include "yaml_parser.hpp"
#include "material_generator.hpp"
#include "kmc_solver.hpp"

// ---------------------------------------------------------------- npy io
static void write_npy(const std::string& path, const std::vector<double>& v, std::vector<size_t> shape) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    std::string shp = "(";
    for (size_t i = 0; i < shape.size(); ++i) shp += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    shp += ")";
    std::string hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': " + shp + ", }";
    size_t total = 10 + hdr.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    hdr += std::string(pad, ' ') + "\n";
    const char magic[] = "\x93NUMPY";
    f.write(magic, 6);
    char ver[2] = {1, 0};
    f.write(ver, 2);
    uint16_t hl = (uint16_t)hdr.size();
    f.write((const char*)&hl, 2);
    f.write(hdr.data(), hdr.size());
    f.write((const char*)v.data(), v.size() * sizeof(double));
}

static std::vector<double> read_npy(const std::string& path) {
    std::vector<size_t> shape;
    return read_npy_double(path, shape);
}

static bool file_exists(const std::string& p) { std::ifstream f(p); return (bool)f; }

template <int D>
static std::vector<double> flat_mats(const std::vector<Eigen::Matrix<double, D, D>>& m) {
    std::vector<double> out(m.size() * D * D);
    for (size_t i = 0; i < m.size(); ++i)
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) out[i * D * D + r * D + c] = m[i](r, c);
    return out;
}

template <int D>
static std::vector<Eigen::Matrix<double, D, D>> unflat_mats(const std::vector<double>& v) {
    size_t n = v.size() / (D * D);
    std::vector<Eigen::Matrix<double, D, D>> m(n);
    for (size_t i = 0; i < n; ++i)
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) m[i](r, c) = v[i * D * D + r * D + c];
    return m;
}

template <int D>
static std::vector<double> flat_mat(const Eigen::Matrix<double, D, D>& m) {
    std::vector<double> out(D * D);
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) out[r * D + c] = m(r, c);
    return out;
}

// ---------------------------------------------------------------- LS commands
static int cmd_ls2d(const std::string& dir) {
    std::ifstream pf(dir + "/params.txt");
    int nx, ny, max_iter; std::string plane_mode; double pixel, tol; Eigen::Matrix2d ebar;
    pf >> nx >> ny >> plane_mode >> pixel >> max_iter >> tol >> ebar(0, 0) >> ebar(0, 1) >> ebar(1, 0) >> ebar(1, 1);
    if (!pf) { std::cerr << "bad params.txt\n"; return 2; }
    std::vector<double> E = read_npy(dir + "/E.npy"), nu = read_npy(dir + "/nu.npy");
    int N = nx * ny;
    double Es = 0, ns = 0;
    for (int i = 0; i < N; ++i) { Es += E[i]; ns += nu[i]; }
    auto [lam0, mu0] = compute_lame_2d(Es / N, ns / N, plane_mode);
    std::vector<double> kx(N), ky(N);
    std::vector<double> fx = fftfreq(nx, pixel), fy = fftfreq(ny, pixel);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) { kx[x * ny + y] = 2.0 * M_PI * fx[x]; ky[x * ny + y] = 2.0 * M_PI * fy[y]; }
    std::vector<GreenTensor> G = green_operator_2d(nx, ny, kx, ky, lam0, mu0);
    std::vector<Eigen::Matrix2d> eps, sig, epsp;
    if (file_exists(dir + "/eps0.npy")) eps = unflat_mats<2>(read_npy(dir + "/eps0.npy"));
    if (file_exists(dir + "/epsp.npy")) epsp = unflat_mats<2>(read_npy(dir + "/epsp.npy"));
    Eigen::Matrix2d em, sm;
    auto t0 = std::chrono::steady_clock::now();
    spectral_solver_2d(nx, ny, E, nu, ebar, plane_mode, G, eps, sig, em, sm, max_iter, tol, false, epsp);
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    write_npy(dir + "/out_eps.npy", flat_mats<2>(eps), {(size_t)N, 4});
    write_npy(dir + "/out_sig.npy", flat_mats<2>(sig), {(size_t)N, 4});
    std::vector<double> mac = flat_mat<2>(em);
    std::vector<double> s2 = flat_mat<2>(sm);
    mac.insert(mac.end(), s2.begin(), s2.end());
    mac.push_back(dt);
    write_npy(dir + "/out_macro.npy", mac, {mac.size()});
    return 0;
}

static int cmd_ls3d(const std::string& dir) {
    std::ifstream pf(dir + "/params.txt");
    int nx, ny, nz, max_iter; double pixel, tol; Eigen::Matrix3d ebar;
    pf >> nx >> ny >> nz >> pixel >> max_iter >> tol;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) pf >> ebar(r, c);
    if (!pf) { std::cerr << "bad params.txt\n"; return 2; }
    std::vector<double> E = read_npy(dir + "/E.npy"), nu = read_npy(dir + "/nu.npy");
    int N = nx * ny * nz;
    double Es = 0, ns = 0;
    for (int i = 0; i < N; ++i) { Es += E[i]; ns += nu[i]; }
    auto [lam0, mu0] = compute_lame_3d(Es / N, ns / N);
    std::vector<double> kx(N), ky(N), kz(N);
    std::vector<double> fx = fftfreq(nx, pixel), fy = fftfreq(ny, pixel), fz = fftfreq(nz, pixel);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int i = x * ny * nz + y * nz + z;
                kx[i] = 2.0 * M_PI * fx[x]; ky[i] = 2.0 * M_PI * fy[y]; kz[i] = 2.0 * M_PI * fz[z];
            }
    std::vector<GreenTensor3D> G = green_operator_3d(nx, ny, nz, kx, ky, kz, lam0, mu0);
    std::vector<Eigen::Matrix3d> eps, sig, epsp;
    if (file_exists(dir + "/eps0.npy")) eps = unflat_mats<3>(read_npy(dir + "/eps0.npy"));
    if (file_exists(dir + "/epsp.npy")) epsp = unflat_mats<3>(read_npy(dir + "/epsp.npy"));
    Eigen::Matrix3d em, sm;
    auto t0 = std::chrono::steady_clock::now();
    spectral_solver_3d(nx, ny, nz, E, nu, ebar, G, eps, sig, em, sm, max_iter, tol, false, epsp);
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    write_npy(dir + "/out_eps.npy", flat_mats<3>(eps), {(size_t)N, 9});
    write_npy(dir + "/out_sig.npy", flat_mats<3>(sig), {(size_t)N, 9});
    std::vector<double> mac = flat_mat<3>(em);
    std::vector<double> s2 = flat_mat<3>(sm);
    mac.insert(mac.end(), s2.begin(), s2.end());
    mac.push_back(dt);
    write_npy(dir + "/out_macro.npy", mac, {mac.size()});
    return 0;
}

// ---------------------------------------------------------------- KMC construction
struct RunCfg {
    bool is3d = false;
    int nx = 32, ny = 32, nz = 1, M = 20, seed = 42;
    std::string plane_mode = "plane_strain";
    double pixel = 1.0, gamma0 = 0.14;
    std::vector<double> E, nu;
    BarrierGenerator bg;
    std::string soft_scheme = "isotropic";
    double soft_cap = 2.0, jp = 10.0, jt = 30.0, neigh = 0.0, q_act = 0.37;
    bool redraw_b = true, redraw_d = true, use3db = false, fp = false, scale_vol = true;
    double stab = 0.0, nu0 = 1e13, rate = 1.0, temp = 0.0;
    int fp_r = 5, fp_s = 100;
    std::string instab = "cascade", ctim = "none";
    double eps_target = 0.05, step_size = 1e-4, mixed_tol = 1e6, max_pct = 0.3;
    std::pair<int, int> comp{0, 0};
    std::map<std::pair<int, int>, double> targets;
};

static std::pair<int, int> comp_of(const std::string& s, bool is3d, bool& ok) {
    static const std::map<std::string, std::pair<int, int>> m2 = {{"xx", {0, 0}}, {"yy", {1, 1}}, {"xy", {0, 1}}, {"yx", {1, 0}}};
    static const std::map<std::string, std::pair<int, int>> m3 = {{"xx", {0, 0}}, {"yy", {1, 1}}, {"zz", {2, 2}}, {"xy", {0, 1}}, {"yx", {1, 0}},
                                                                  {"xz", {0, 2}}, {"zx", {2, 0}}, {"yz", {1, 2}}, {"zy", {2, 1}}};
    const auto& m = is3d ? m3 : m2;
    auto it = m.find(s);
    ok = it != m.end();
    return ok ? it->second : std::pair<int, int>{0, 0};
}

// Parameter mapping of main.cpp:40-377 (constant or .npy modulus fields).
static RunCfg load_cfg(const std::string& path) {
    YAMLConfig c;
    if (!c.load(path)) throw std::runtime_error("cannot load " + path);
    RunCfg r;
    std::string dim = c.getString("system.dimensionality", "2d");
    for (auto& ch : dim) ch = (char)tolower(ch);
    r.is3d = dim == "3d";
    r.plane_mode = c.getString("system.plane_mode", "plane_strain");
    r.nx = c.getInt("system.nx", 32); r.ny = c.getInt("system.ny", 32);
    r.nz = r.is3d ? c.getInt("system.nz", 32) : 1;
    r.pixel = c.getDouble("system.pixel", 1.0);
    int N = r.nx * r.ny * r.nz;
    std::string em = c.getString("material.E.mode", "constant");
    if (em == "file") {
        r.E = read_npy(c.getString("material.E.parameters.path", ""));
        double s = 0; for (double v : r.E) s += v;
        if (s / r.E.size() < 1e6) for (double& v : r.E) v *= 1e9;
    } else {
        double e = c.getDouble("material.E.value", 70.0);
        if (e < 1e6) e *= 1e9;
        r.E.assign(N, e);
    }
    std::string nm = c.getString("material.nu.mode", "constant");
    if (nm == "file") r.nu = read_npy(c.getString("material.nu.parameters.path", ""));
    else r.nu.assign(N, c.getDouble("material.nu.value", 0.3));
    if ((int)r.E.size() != N || (int)r.nu.size() != N) throw std::runtime_error("field size mismatch");
    r.eps_target = c.getDouble("loading.eps_target", 0.05);
    r.step_size = c.getDouble("loading.step_size", 1e-4);
    r.mixed_tol = c.getDouble("boundary_conditions.mixed_tol", 1.0) * 1e6;
    r.bg.type = c.getString("barriers.type", "gaussian");
    r.bg.mean = c.getDouble("barriers.kwargs.mean", 2.0);
    r.bg.std_val = c.getDouble("barriers.kwargs.std", 0.6);
    r.bg.min_cutoff = c.getDouble("barriers.kwargs.min_cutoff", 0.1);
    r.bg.max_cutoff = c.getDouble("barriers.kwargs.max_cutoff", -1.0);
    r.bg.loc = c.getDouble("barriers.kwargs.loc", 1.0);
    r.bg.scale = c.getDouble("barriers.kwargs.scale", 0.5);
    r.bg.epsilon = c.getDouble("barriers.kwargs.epsilon", 0.1);
    r.bg.ratio = c.getDouble("barriers.kwargs.ratio", 0.8);
    bool soft = c.getBool("physics.enable_softening", true);
    r.soft_scheme = c.getString("physics.softening_scheme", "isotropic");
    r.soft_cap = soft ? c.getDouble("physics.softening_cap", 2.0) : 0.0;
    r.jp = soft ? c.getDouble("physics.jp", 10.0) : 0.0;
    r.jt = soft ? c.getDouble("physics.jt", 30.0) : 0.0;
    r.neigh = soft ? c.getDouble("physics.neighbor_softening_fraction", 0.0) : 0.0;
    r.q_act = c.getDouble("physics.q_act_temp", 0.37);
    r.redraw_b = c.getBool("physics.redraw_barriers", true);
    r.redraw_d = c.getBool("physics.redraw_directions", true);
    r.stab = c.getDouble("physics.stability_threshold", 0.0);
    r.instab = c.getString("dynamics.instability_mode", "cascade");
    r.ctim = c.getString("dynamics.cascade_timing", "none");
    r.scale_vol = c.getBool("dynamics.scale_rate_by_volume", true);
    r.nu0 = c.getDouble("dynamics.nu0", 1e13);
    r.rate = c.getDouble("dynamics.physical_strain_rate", 1.0);
    r.temp = c.getDouble("dynamics.temperature", 0.0);
    r.fp = c.getBool("dynamics.fast_patching.enabled", false);
    r.fp_r = c.getInt("dynamics.fast_patching.patch_radius", 5);
    r.fp_s = c.getInt("dynamics.fast_patching.sync_interval", 100);
    r.M = c.getInt("system.M", 20);
    r.gamma0 = c.getDouble("system.gamma0", 0.14);
    r.seed = c.getInt("seed", 42);
    r.use3db = c.getBool("system.3d_barriers", false);
    r.max_pct = c.getDouble("detection.max_kmc_steps_pct", 0.3);
    bool ok;
    r.comp = comp_of(c.getString("boundary_conditions.driving_component", "xx"), r.is3d, ok);
    for (auto& kv : c.getDict("boundary_conditions.mixed_targets")) {
        auto ij = comp_of(kv.first, r.is3d, ok);
        if (!ok) continue;
        double v = kv.second;
        if (v < 1e6) v *= 1e9;
        r.targets[ij] = v;
    }
    return r;
}

template <class Sim>
static void dump_state(Sim& s, const std::string& out) {
    size_t N = s.E_field.size();
    int D = (int)s.eps_field[0].Rows;
    write_npy(out + "/eps.npy", flat_mats(s.eps_field), {N, (size_t)(D * D)});
    write_npy(out + "/sig.npy", flat_mats(s.sig_field), {N, (size_t)(D * D)});
    write_npy(out + "/epsp.npy", flat_mats(s.eps_plastic), {N, (size_t)(D * D)});
    write_npy(out + "/catalog.npy", flat_mats(s.catalog), {s.catalog.size(), (size_t)(D * D)});
    write_npy(out + "/prev_dir.npy", flat_mats(s.prev_strain_dir), {N, (size_t)(D * D)});
    write_npy(out + "/Q0.npy", s.Q0, {s.Q0.size()});
    write_npy(out + "/Q.npy", s.Q, {s.Q.size()});
    std::vector<double> sp(2 * N);
    for (size_t i = 0; i < N; ++i) { sp[2 * i] = s.soft_prop[i](0); sp[2 * i + 1] = s.soft_prop[i](1); }
    write_npy(out + "/soft.npy", sp, {N, 2});
    write_npy(out + "/last_t.npy", s.last_event_time, {N});
    std::vector<double> mac = flat_mat(s.eps_macro), s2 = flat_mat(s.sig_macro);
    mac.insert(mac.end(), s2.begin(), s2.end());
    mac.push_back(s.time);
    write_npy(out + "/macro.npy", mac, {mac.size()});
}

static KmcSimulation2D* make2d(const RunCfg& r, const std::string& out) {
    return new KmcSimulation2D(r.nx, r.ny, r.M, r.gamma0, r.E, r.nu, r.pixel, r.bg, r.soft_scheme, r.soft_cap, r.jp, r.jt, r.neigh,
                               r.q_act, out, r.temp, r.rate, r.stab, r.nu0, r.plane_mode, r.fp, r.fp_r, r.fp_s, r.instab, r.ctim,
                               r.scale_vol, r.redraw_d, r.redraw_b, r.seed);
}
static KmcSimulation3D* make3d(const RunCfg& r, const std::string& out) {
    return new KmcSimulation3D(r.nx, r.ny, r.nz, r.M, r.gamma0, r.E, r.nu, r.pixel, r.bg, r.soft_scheme, r.soft_cap, r.jp, r.jt,
                               r.neigh, r.q_act, out, r.temp, r.rate, r.stab, r.nu0, r.fp, r.fp_r, r.fp_s, r.instab, r.ctim,
                               r.scale_vol, r.redraw_d, r.redraw_b, r.use3db, r.seed);
}

template <class Sim>
static int run_ref(Sim* s, const RunCfg& r, const std::string& out, int nsteps) {
    auto t0 = std::chrono::steady_clock::now();
    s->run_simulation(nsteps, r.step_size, r.comp, r.targets, r.mixed_tol, 50, "none", "checkpoint", "none", true, false, false,
                      "summary_log.txt", true, false, r.max_pct);
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    dump_state(*s, out);
    std::ofstream tf(out + "/timing.txt");
    tf.precision(17);
    tf << dt << "\n";
    return 0;
}

// Control flow of run_simulation (kmc_solver.hpp:721-1037 / :1735-2062), fast
// patching off, with one trace row per event:
//  [kind, a, b, total_rate, t_wait, time, eps_macro(DxD), sig_macro(DxD)]
//  kind 0 = thermal flip (a = flat mode index, b = is_instab)
//  kind 1 = cascade (a = batches, b = flips)
//  kind 2 = interval end without event (a = u1 draw consumed)
//  kind 3 = elastic step done (a = mixed-BC solves, b = elastic step count)
template <class Sim, int D>
static int trace_ref(Sim* s, const RunCfg& r, const std::string& out, int nsteps, long maxev, double* elapsed) {
    std::vector<double> rows;
    auto push = [&](double kind, double a, double b, double R, double tw) {
        rows.push_back(kind); rows.push_back(a); rows.push_back(b); rows.push_back(R); rows.push_back(tw); rows.push_back(s->time);
        for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) rows.push_back(s->eps_macro(i, j));
        for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) rows.push_back(s->sig_macro(i, j));
    };
    auto t0 = std::chrono::steady_clock::now();
    s->elastic_run();
    auto t_loop = std::chrono::steady_clock::now();
    Eigen::Matrix<double, D, D> unit = Eigen::Matrix<double, D, D>::Zero();
    unit(r.comp.first, r.comp.second) = 1.0;
    double dt_step = std::abs(r.step_size) / s->strain_rate, remaining = 0.0;
    std::uniform_real_distribution<double> U(0.0, 1.0);
    long nev = 0;
    int done = 0, seq_instab = 0;
    int max_seq = (int)(r.max_pct * (double)s->E_field.size());
    bool stop = false;
    while (done < nsteps && !stop) {
        remaining += dt_step;
        while (remaining > 0.0) {
            s->update_barriers();
            if (s->instability_mode == "cascade" && !s->find_unstable_indices().empty()) {
                auto cs = s->run_cascade(0, r.comp);
                if (cs.second > 0) push(1, cs.first, cs.second, 0, 0);
                continue;
            }
            double vol = s->scale_rate_by_volume ? s->volume : 1.0;
            double beta = s->temperature > 0.0 ? 1.0 / (8.617e-5 * s->temperature) : std::numeric_limits<double>::infinity();
            std::vector<double> rates; std::vector<int> idx; double R = 0.0;
            for (int i = 0; i < (int)s->Q.size(); ++i) {
                double q = s->Q[i];
                if (s->instability_mode == "kmc" || q > 0.0) {
                    double rr = q <= 0.0 ? vol * s->nu0 : vol * s->nu0 * std::exp(-q * beta);
                    rates.push_back(rr); R += rr; idx.push_back(i);
                }
            }
            if (R > 0.0) {
                double u1 = U(s->rng);
                double tw = -std::log(u1) / R;
                if (tw < remaining) {
                    s->time += tw;
                    s->eps_macro += unit * (s->strain_rate * tw);
                    remaining -= tw;
                    double target = U(s->rng) * R, cur = 0.0;
                    int sel = (int)rates.size() - 1;
                    for (size_t i = 0; i < rates.size(); ++i) { cur += rates[i]; if (cur >= target) { sel = (int)i; break; } }
                    int f = idx[sel], m = f % s->M, vox = f / s->M;
                    bool instab = s->Q[f] <= s->stability_threshold;
                    auto C = s->catalog[f];
                    if constexpr (D == 2) s->apply_flip_soa_2d(vox / s->ny, vox % s->ny, m);
                    else s->apply_flip_soa_3d(vox / (s->ny * s->nz), (vox / s->nz) % s->ny, vox % s->nz, m);
                    s->prev_strain_dir[vox] = C;
                    // redraw, kmc_solver.hpp:839-864 / :1854-1875
                    std::normal_distribution<double> sn(0.0, 1.0);
                    auto redraw_one = [&](int mi) {
                        if constexpr (D == 2) {
                            double gxx = 0.5 * s->gamma0 * sn(s->rng), gxy = 0.5 * s->gamma0 * sn(s->rng);
                            s->catalog[mi](0, 0) = gxx; s->catalog[mi](1, 1) = -gxx; s->catalog[mi](0, 1) = gxy; s->catalog[mi](1, 0) = gxy;
                        }
                    };
                    if constexpr (D == 2) {
                        if (s->redraw_directions || s->redraw_barriers) {
                            for (int mm = 0; mm < s->M; ++mm) {
                                int ci = vox * s->M + mm;
                                if (s->redraw_directions) redraw_one(ci);
                                if (s->redraw_barriers) s->Q0[ci] = s->barrier_gen.generate(s->rng);
                            }
                        } else { redraw_one(f); s->Q0[f] = s->barrier_gen.generate(s->rng); }
                    } else {
                        // the 3D redraw goes through the class's private mode generators;
                        // reproduce their draw order with the same distributions.
                        auto mode = [&]() {
                            Eigen::Matrix3d G = Eigen::Matrix3d::Zero();
                            if (!s->use_3d_barriers) {
                                std::normal_distribution<double> g(0.0, 1.0);
                                double gxx = 0.5 * s->gamma0 * g(s->rng), gxy = 0.5 * s->gamma0 * g(s->rng);
                                G(0, 0) = gxx; G(1, 1) = -gxx; G(0, 1) = gxy; G(1, 0) = gxy;
                                return G;
                            }
                            std::normal_distribution<double> g(0.0, 1.0);
                            Eigen::Matrix3d Mx;
                            for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Mx(i, j) = g(s->rng);
                            Eigen::Matrix3d Ms = 0.5 * (Mx + Mx.transpose());
                            G = Ms - (1.0 / 3.0) * Ms.trace() * Eigen::Matrix3d::Identity();
                            double nrm = G.norm();
                            if (nrm < 1e-12) return Eigen::Matrix3d(Eigen::Matrix3d::Zero());
                            G = G * (1.0 / (std::sqrt(2.0) * nrm));
                            std::uniform_real_distribution<double> ud(1e-15, 1.0);
                            double u = ud(s->rng);
                            return Eigen::Matrix3d(G * (s->gamma0 * std::sqrt(-2.0 * std::log(u))));
                        };
                        if (s->redraw_directions || s->redraw_barriers) {
                            for (int mm = 0; mm < s->M; ++mm) {
                                int ci = vox * s->M + mm;
                                if (s->redraw_directions) s->catalog[ci] = mode();
                                if (s->redraw_barriers) s->Q0[ci] = s->barrier_gen.generate(s->rng);
                            }
                        } else { s->catalog[f] = mode(); s->Q0[f] = s->barrier_gen.generate(s->rng); }
                    }
                    s->elastic_run();
                    seq_instab = instab ? seq_instab + 1 : 0;
                    push(0, f, instab ? 1 : 0, R, tw);
                    if (++nev >= maxev || seq_instab > max_seq) { stop = true; break; }
                    continue;
                } else {
                    push(2, u1, 0, R, tw);
                }
            }
            s->eps_macro += unit * (s->strain_rate * remaining);
            s->time += remaining;
            remaining = 0.0;
        }
        if (stop) break;
        double Es = 0, ns = 0;
        for (double v : s->E_field) Es += v;
        for (double v : s->nu_field) ns += v;
        double Ea = Es / s->E_field.size(), na = ns / s->nu_field.size();
        int solves = 0;
        for (int it = 0; it < 50; ++it) {
            s->elastic_run(); ++solves;
            Eigen::Matrix<double, D, D> err = Eigen::Matrix<double, D, D>::Zero();
            double emax = 0.0;
            for (auto& t : r.targets) { double e = t.second - s->sig_macro(t.first.first, t.first.second); err(t.first.first, t.first.second) = e; emax = std::max(emax, std::abs(e)); }
            if (emax < r.mixed_tol) break;
            double tr = err.trace();
            Eigen::Matrix<double, D, D> de = (err - na * tr * Eigen::Matrix<double, D, D>::Identity()) / Ea;
            for (auto& t : r.targets) s->eps_macro(t.first.first, t.first.second) += de(t.first.first, t.first.second);
        }
        ++done;
        push(3, solves, done, 0, 0);
    }
    *elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    size_t w = 6 + 2 * D * D;
    write_npy(out + "/trace.npy", rows, {rows.size() / w, w});
    dump_state(*s, out);
    std::ofstream tf(out + "/timing.txt");
    tf.precision(17);
    tf << *elapsed << " " << nev << " " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count() << "\n";
    return 0;
}

static int cmd_draws(int seed, int n, const std::string& out) {
    std::mt19937 g(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::normal_distribution<double> Nn(0.0, 1.0);
    std::vector<double> v;
    for (int i = 0; i < n; ++i) { v.push_back(U(g)); v.push_back(Nn(g)); v.push_back(Nn(g)); v.push_back((double)g()); }
    write_npy(out, v, {(size_t)n, 4});
    return 0;
}

// generate_correlated_field_cpp (material_generator.hpp:130-258), as main.cpp's
// "generated" material mode calls it: the field of NX x NY x NZ voxels.
static int cmd_grf(char** a, const std::string& out) {
    const int nx = atoi(a[0]), ny = atoi(a[1]), nz = atoi(a[2]), is3d = atoi(a[3]);
    const double mean = atof(a[4]), sd = atof(a[5]), corr = atof(a[6]);
    const int has_min = atoi(a[7]);
    const double cmin = atof(a[8]);
    const int has_max = atoi(a[9]);
    const double cmax = atof(a[10]);
    const int seed = atoi(a[11]);
    std::vector<double> f = generate_correlated_field_cpp(nx, ny, nz, is3d != 0, mean, sd, corr, has_min != 0, cmin,
                                                          has_max != 0, cmax, seed);
    write_npy(out, f, {f.size()});
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) { std::cerr << "usage: ref_driver ls2d|ls3d DIR | kmc_run CFG OUT NSTEPS | kmc_trace CFG OUT NSTEPS MAXEV | kmc_init CFG OUT | draws SEED N OUT | grf NX NY NZ IS3D MEAN STD CORR HASMIN MIN HASMAX MAX SEED OUT\n"; return 2; }
    std::string cmd = argv[1];
    try {
        if (cmd == "ls2d") return cmd_ls2d(argv[2]);
        if (cmd == "ls3d") return cmd_ls3d(argv[2]);
        if (cmd == "draws" && argc >= 5) return cmd_draws(atoi(argv[2]), atoi(argv[3]), argv[4]);
        if (cmd == "grf" && argc >= 15) return cmd_grf(argv + 2, argv[14]);
        if ((cmd == "kmc_run" || cmd == "kmc_trace" || cmd == "kmc_init") && argc >= 4) {
            RunCfg r = load_cfg(argv[2]);
            std::string out = argv[3];
            std::cout.setstate(std::ios::failbit);  // silence constructor banners
            int nsteps = argc >= 5 ? atoi(argv[4]) : 1;
            long maxev = argc >= 6 ? atol(argv[5]) : (1L << 62);
            double el = 0;
            if (r.is3d) {
                KmcSimulation3D* s = make3d(r, out);
                if (cmd == "kmc_init") { dump_state(*s, out); return 0; }
                return cmd == "kmc_run" ? run_ref(s, r, out, nsteps) : trace_ref<KmcSimulation3D, 3>(s, r, out, nsteps, maxev, &el);
            } else {
                KmcSimulation2D* s = make2d(r, out);
                if (cmd == "kmc_init") { dump_state(*s, out); return 0; }
                return cmd == "kmc_run" ? run_ref(s, r, out, nsteps) : trace_ref<KmcSimulation2D, 2>(s, r, out, nsteps, maxev, &el);
            }
        }
    } catch (const std::exception& e) {
        std::cerr << "ref_driver error: " << e.what() << "\n";
        return 1;
    }
    std::cerr << "bad command\n";
    return 2;
}
