// Drop-in replacement for the reference's linear_elastic_solver.hpp: the same
// free functions and types, with the LS solve running on the GPU through
// libmgkmc_b200 (include/mgkmc_b200.h).  A caller compiled with this directory
// ahead of the reference's on its include path (and linked with
// -lmgkmc_b200) builds unchanged.
//
// Differences a caller can see:
//  * green_operator_2d/3d return an empty table: the GPU evaluates the
//    closed-form Green operator on the fly, so the N x 16 (N x 81) table the
//    reference precomputes is never built; spectral_solver_* ignore Gamma.
//  * errors throw std::runtime_error (the reference has none to report).
#pragma once
#include <Eigen/Dense>

#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../mgkmc_b200.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

// linear_elastic_solver.hpp:19 / :312 (the same types, so callers' declarations compile)
using GreenTensor = std::array<std::array<std::array<std::array<double, 2>, 2>, 2>, 2>;
using GreenTensor3D = std::array<std::array<std::array<std::array<double, 3>, 3>, 3>, 3>;

// linear_elastic_solver.hpp:22-33: sample frequencies of a length-n DFT with spacing d
inline std::vector<double> fftfreq(int n, double d) {
    std::vector<double> f(n);
    const int npos = (n - 1) / 2 + 1;  // 0 .. ceil(n/2) - 1 non-negative, the rest negative
    for (int i = 0; i < n; ++i) f[i] = (double)(i < npos ? i : i - n) / (d * n);
    return f;
}

// linear_elastic_solver.hpp:36-45 / :315-319: Lame constants of (E, nu)
inline std::pair<double, double> compute_lame_2d(double E, double nu, const std::string& plane_mode) {
    const double mu = E / (2.0 * (1.0 + nu));
    const double lam = plane_mode == "plane_stress" ? E * nu / (1.0 - nu * nu) : E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    return {lam, mu};
}

inline std::pair<double, double> compute_lame_3d(double E, double nu) {
    return {E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))};
}

// linear_elastic_solver.hpp:70-119 / :344-396: not tabulated (see the header comment)
inline std::vector<GreenTensor> green_operator_2d(int, int, const std::vector<double>&, const std::vector<double>&,
                                                  double, double) {
    return {};
}

inline std::vector<GreenTensor3D> green_operator_3d(int, int, int, const std::vector<double>&,
                                                    const std::vector<double>&, const std::vector<double>&, double,
                                                    double) {
    return {};
}

namespace mgk_shim {

// One GPU solver per thread, rebuilt when the grid or the moduli change
// (a caller's loop of solves on one material reuses it).
struct LsCache {
    mgk_ls* h = nullptr;
    int dim = 0, nx = 0, ny = 0, nz = 0, ps = 0;
    std::vector<double> E, nu;
    ~LsCache() {
        if (h) mgk_ls_destroy(h);
    }
    mgk_ls* get(int d, int x, int y, int z, int plane_stress, const std::vector<double>& E_, const std::vector<double>& nu_) {
        if (h && d == dim && x == nx && y == ny && z == nz && plane_stress == ps && E_ == E && nu_ == nu) return h;
        if (h) mgk_ls_destroy(h);
        h = nullptr;
        if (mgk_ls_create(&h, d, x, y, z, plane_stress, 1.0, E_.data(), nu_.data()) != MGK_OK)
            throw std::runtime_error(std::string("mgk_ls_create: ") + mgk_last_error());
        dim = d, nx = x, ny = y, nz = z, ps = plane_stress, E = E_, nu = nu_;
        return h;
    }
};

inline LsCache& cache() {
    thread_local LsCache c;
    return c;
}

template <int D, typename Mat>
void solve(int nx, int ny, int nz, int plane_stress, const std::vector<double>& E, const std::vector<double>& nu,
           const Mat& eps_bar, std::vector<Mat>& eps, std::vector<Mat>& sig_out, Mat& eps_macro, Mat& sig_macro,
           int max_iter, double tol, const std::vector<Mat>& eps_plastic) {
    const size_t N = (size_t)nx * ny * nz;
    if (E.size() != N || nu.size() != N) throw std::runtime_error("spectral_solver: E / nu size differs from the grid");
    mgk_ls* h = cache().get(D, nx, ny, nz, plane_stress, E, nu);
    // row-major D x D per voxel (Eigen stores column-major: copy element-wise)
    std::vector<double> e(N * D * D), s(N * D * D), ep;
    const bool warm = eps.size() == N;  // linear_elastic_solver.hpp:181-194
    if (warm)
        for (size_t v = 0; v < N; ++v)
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) e[v * D * D + i * D + j] = eps[v](i, j);
    if (eps_plastic.size() == N) {
        ep.resize(N * D * D);
        for (size_t v = 0; v < N; ++v)
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) ep[v * D * D + i * D + j] = eps_plastic[v](i, j);
    }
    double eb[9], mac[18];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) eb[i * D + j] = eps_bar(i, j);
    int iters = 0;
    const mgk_status st = mgk_ls_solve(h, eb, ep.empty() ? nullptr : ep.data(), e.data(), warm ? 1 : 0, s.data(), mac,
                                       max_iter, tol, &iters);
    if (st != MGK_OK && st != MGK_LS_NOT_CONVERGED)  // the reference stops silently at max_iter
        throw std::runtime_error(std::string("mgk_ls_solve: ") + mgk_last_error());
    eps.resize(N);
    sig_out.resize(N);
    for (size_t v = 0; v < N; ++v)
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j) {
                eps[v](i, j) = e[v * D * D + i * D + j];
                sig_out[v](i, j) = s[v * D * D + i * D + j];
            }
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            eps_macro(i, j) = mac[i * D + j];
            sig_macro(i, j) = mac[D * D + i * D + j];
        }
}

}  // namespace mgk_shim

// linear_elastic_solver.hpp:146-160: the same signature; Gamma and verbose are not used
inline void spectral_solver_2d(int nx, int ny, const std::vector<double>& E_field, const std::vector<double>& nu_field,
                               const Eigen::Matrix2d& eps_bar, const std::string& plane_mode,
                               const std::vector<GreenTensor>& /*Gamma*/, std::vector<Eigen::Matrix2d>& eps,
                               std::vector<Eigen::Matrix2d>& sig_out, Eigen::Matrix2d& eps_macro,
                               Eigen::Matrix2d& sig_macro, int max_iter = 200, double tol = 1e-6, bool /*verbose*/ = false,
                               const std::vector<Eigen::Matrix2d>& eps_plastic = {}) {
    mgk_shim::solve<2>(nx, ny, 1, plane_mode == "plane_stress" ? 1 : 0, E_field, nu_field, eps_bar, eps, sig_out, eps_macro,
                       sig_macro, max_iter, tol, eps_plastic);
}

// linear_elastic_solver.hpp:431-444
inline void spectral_solver_3d(int nx, int ny, int nz, const std::vector<double>& E_field,
                               const std::vector<double>& nu_field, const Eigen::Matrix3d& eps_bar,
                               const std::vector<GreenTensor3D>& /*Gamma*/, std::vector<Eigen::Matrix3d>& eps,
                               std::vector<Eigen::Matrix3d>& sig_out, Eigen::Matrix3d& eps_macro,
                               Eigen::Matrix3d& sig_macro, int max_iter = 200, double tol = 1e-6, bool /*verbose*/ = false,
                               const std::vector<Eigen::Matrix3d>& eps_plastic = {}) {
    mgk_shim::solve<3>(nx, ny, nz, 0, E_field, nu_field, eps_bar, eps, sig_out, eps_macro, sig_macro, max_iter, tol,
                       eps_plastic);
}
