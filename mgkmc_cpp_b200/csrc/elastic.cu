// The reference's linear-elastic simulation (simulation_type "linear_elastic",
// main.cpp:418-869): proportional loading of the macroscopic target in
// n_steps + 1 steps (s = 0 .. n_steps, target * s / n_steps), each step an
// outer mixed-control loop of at most max_iter_macro warm-started LS solves
// (spectral_solver_2d/3d with tol 1e-6, 200 iterations) that corrects the
// stress-controlled components of the applied strain by
// d_eps = (err - nu_avg * tr(err) * I) / E_avg until every stress error is
// below the tolerance; then the summary / global log rows and the VTU
// schedule of the reference.  The LS solves run on the GPU (LsSolver); the
// loop is host logic over one device-resident field.
#include <chrono>
#include <cmath>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "elastic.cuh"
#include "ls.cuh"
#include "vtu.h"

namespace mgk {

namespace {

std::string now_stamp() {
    std::time_t t = std::time(nullptr);
    char buf[64];
    std::strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S", std::localtime(&t));
    return buf;
}

const char* kComp[3][3] = {{"xx", "xy", "xz"}, {"yx", "yy", "yz"}, {"zx", "zy", "zz"}};

}  // namespace

mgk_status elastic_run(const mgk_le_params& p, const double* E, const double* nu, double* macro_out, int* ls_iters_out,
                       std::string* err) {
    const int D = p.dim;
    const int dims[3] = {p.nx, p.ny, D == 3 ? p.nz : 1};
    const long N = (long)dims[0] * dims[1] * dims[2];
    const int n_steps = (int)std::lround(p.eps_target / p.step_size);
    if (n_steps < 1) {
        *err = "eps_target / step_size rounds to zero steps";
        return MGK_BAD_ARG;
    }
    double E_avg = 0.0, nu_avg = 0.0;
    for (long i = 0; i < N; ++i) E_avg += E[i];
    E_avg /= (double)N;
    for (long i = 0; i < N; ++i) nu_avg += nu[i];
    nu_avg /= (double)N;

    // targets: the driving strain, the other components strain-controlled to
    // zero, the mixed targets stress-controlled (values in Pa)
    double target[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool strain_ctl[9];
    for (int k = 0; k < 9; ++k) strain_ctl[k] = true;
    target[p.drive_i * D + p.drive_j] = p.eps_target;
    for (int t = 0; t < p.n_targets; ++t) {
        const int k = p.target_i[t] * D + p.target_j[t];
        target[k] = p.target_v[t];
        strain_ctl[k] = false;
    }
    const std::string drv = kComp[p.drive_i][p.drive_j];
    const std::string dir = p.output_dir ? p.output_dir : "";
    const bool summary = p.enable_summary_log && !dir.empty();
    const bool global = p.enable_global_log && !dir.empty();
    std::ofstream slog, glog;
    if (summary) {
        slog.open(dir + "/" + (p.summary_filename ? p.summary_filename : "summary_log.txt"));
        slog << std::left << std::setw(20) << "Timestamp" << " " << std::setw(12) << "Elapsed(s)" << " " << std::setw(8)
             << "Step" << " " << std::setw(14) << ("Eps_" + drv) << " " << std::setw(16) << ("Sig_" + drv + "(GPa)") << "\n";
        slog << std::string(75, '-') << "\n";
    }
    // global log columns: the independent components xx, yy, (zz), xy, (xz, yz)
    std::vector<int> cols;
    if (D == 2) cols = {0, 3, 1};
    else cols = {0, 4, 8, 1, 2, 5};
    if (global) {
        glog.open(dir + "/global_log.txt");
        glog << std::left << std::setw(12) << "GlobalStep" << " ";
        for (int k : cols) glog << std::setw(14) << ("Eps_" + std::string(kComp[k / D][k % D])) << " ";
        for (size_t c = 0; c < cols.size(); ++c) {
            const int k = cols[c];
            glog << std::setw(16) << ("Sig_" + std::string(kComp[k / D][k % D]) + "(GPa)") << (c + 1 < cols.size() ? " " : "\n");
        }
        glog << std::string(D == 2 ? 110 : 195, '-') << "\n";
    }
    std::string vtk = p.vtk_interval ? p.vtk_interval : "none";
    for (auto& ch : vtk) ch = (char)std::tolower((unsigned char)ch);
    int vtk_every = -1;
    if (vtk != "none" && vtk != "last" && vtk != "current") {
        try {
            vtk_every = std::stoi(vtk);
        } catch (...) {
            vtk_every = -1;
        }
    }
    const std::string vtk_path = dir + "/step";

    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        *err = "stream creation failed";
        return MGK_CUDA_ERROR;
    }
    mgk_status status = MGK_OK;
    try {
        LsSolver ls(D, dims, p.plane_stress != 0, p.pixel, E, nu, st);
        std::vector<double> h_eps, h_sig;
        double ebar[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        bool filled = false;
        long long iters_total = 0;
        const auto t0 = std::chrono::high_resolution_clock::now();
        for (int s = 0; s <= n_steps; ++s) {
            double tgt[9];
            for (int k = 0; k < D * D; ++k) tgt[k] = target[k] * ((double)s / n_steps);
            double em[9] = {0}, sm[9] = {0};
            for (int it = 0; it < p.max_iter_macro; ++it) {
                for (int k = 0; k < D * D; ++k)
                    if (strain_ctl[k]) ebar[k] = tgt[k];
                cudaError_t ce = ls.solve(ebar, filled, nullptr, p.max_iter_ls, p.tol_ls);
                if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
                if (ce != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(ce));
                if (ls.device_error()) {
                    *err = "device wait timed out in the LS solve";
                    status = MGK_DEVICE_TIMEOUT;
                    throw std::runtime_error(*err);
                }
                filled = true;
                int iters = 0;
                ls.macro(em, sm, &iters);
                iters_total += iters;
                double serr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, emax = 0.0;
                bool stress_ctl = false;
                for (int k = 0; k < D * D; ++k)
                    if (!strain_ctl[k]) {
                        serr[k] = tgt[k] - sm[k];
                        emax = std::max(emax, std::fabs(serr[k]));
                        stress_ctl = true;
                    }
                if (!stress_ctl || emax < p.mixed_tol) break;
                double tr = 0.0;
                for (int a = 0; a < D; ++a) tr += serr[a * D + a];
                for (int k = 0; k < D * D; ++k)
                    if (!strain_ctl[k]) ebar[k] += (serr[k] - nu_avg * tr * ((k % (D + 1)) == 0 ? 1.0 : 0.0)) / E_avg;
            }
            if (macro_out)
                for (int k = 0; k < D * D; ++k) {
                    macro_out[(long)s * 2 * D * D + k] = em[k];
                    macro_out[(long)s * 2 * D * D + D * D + k] = sm[k];
                }
            const double eps_drv = em[p.drive_i * D + p.drive_j], sig_drv = sm[p.drive_i * D + p.drive_j];
            if (p.enable_console)
                std::cout << "step " << s << "/" << n_steps << ": " << "eps_" << drv << "=" << std::fixed << std::setprecision(4)
                          << eps_drv << ", " << "sig_" << drv << "=" << std::setprecision(2) << (sig_drv / 1e6) << " MPa"
                          << std::endl;
            const double elapsed = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
            if (summary)
                slog << std::left << std::setw(20) << now_stamp() << " " << std::setw(12) << std::fixed << std::setprecision(3)
                     << elapsed << " " << std::setw(8) << s << " " << std::setw(14) << std::setprecision(6) << eps_drv << " "
                     << std::setw(16) << (sig_drv / 1e9) << "\n";
            if (global) {
                glog << std::left << std::setw(12) << s << " " << std::fixed << std::setprecision(6);
                for (int k : cols) glog << std::setw(14) << em[k] << " ";
                for (size_t c = 0; c < cols.size(); ++c)
                    glog << std::setw(16) << (sm[cols[c]] / 1e9) << (c + 1 < cols.size() ? " " : "\n");
            }
            std::string vt_name;
            if (vtk != "none" && !dir.empty()) {
                if (vtk == "current") {
                    vt_name = vtk_path + ".vtu";
                } else if (vtk_every > 0 && s % vtk_every == 0) {
                    std::ostringstream os;
                    os << vtk_path << "_" << std::setfill('0') << std::setw(6) << s << ".vtu";
                    vt_name = os.str();
                }
                if (s == n_steps && (vtk == "last" || (vtk_every > 0 && n_steps % vtk_every != 0)))
                    vt_name = vtk_path + "_final.vtu";
            }
            if (!vt_name.empty()) {
                h_eps.resize((size_t)N * D * D);
                h_sig.resize((size_t)N * D * D);
                cudaError_t ce = ls.download_eps(h_eps.data());
                if (ce == cudaSuccess) ce = ls.download_sig(nullptr, h_sig.data());
                if (ce != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(ce));
                write_vtu_fields(vt_name, D, dims[0], dims[1], dims[2], h_eps.data(), h_sig.data(), E, nu, p.pixel, nullptr,
                                 nullptr);
            }
        }
        if (ls_iters_out) *ls_iters_out = (int)std::min<long long>(iters_total, 2147483647LL);
    } catch (const std::invalid_argument& e) {
        *err = e.what();
        status = MGK_BAD_SHAPE;
    } catch (const std::exception& e) {
        if (status == MGK_OK) {
            *err = e.what();
            status = std::strstr(e.what(), "out of memory") ? MGK_OOM : MGK_CUDA_ERROR;
        }
    }
    cudaStreamDestroy(st);
    return status;
}

}  // namespace mgk
