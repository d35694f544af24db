// Lippmann-Schwinger solver kernels and host driver (see ls.cuh for the design).
//
// Reference semantics kept (linear_elastic_solver.hpp:146-309 / :431-593):
//  * warm start shifts the field mean to eps_bar (:181-191), cold start fills it;
//  * one iteration: sigma = C:(eps - eps_p); tau = sigma - C0:eps; eps_new =
//    eps_bar - IFFT(Gamma0 : FFT(tau)); diff = |eps_new - eps| / (|eps| + 1e-20)
//    (Frobenius norms over all voxels, full tensors); stop when diff < tol;
//  * lam0, mu0 from the voxel means of E and nu (:162-178); Gamma0 closed form
//    with A = 1/(4 mu0), B = (lam0+mu0)/(mu0 (lam0+2 mu0)), Gamma(0) = 0 (:70-119).
// Differences in arithmetic only:
//  * the reference transforms every component with complex FFTs and keeps the
//    real part of the inverse; on even-length axes its Gamma is not Hermitian on
//    the Nyquist planes, so the kept real part equals the inverse transform of
//    the Hermitian average 0.5*(Gamma(q) + Gamma(q with the Nyquist components
//    negated)) : tau_hat.  This solver applies exactly that average on Nyquist
//    bins and uses real-to-complex transforms;
//  * the mean of the fluctuation field is zero by construction (Gamma(0) = 0),
//    so the reference's mean subtraction (:263-271) only removes rounding noise
//    and is not repeated here;
//  * the symmetric part of eps is stored; the antisymmetric part is uniform
//    (it only ever comes from eps_bar) and is carried as three scalars.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/mgkmc_b200.h"
#include "ls.cuh"
#include "ls_device.cuh"

namespace mgk {

namespace {

using namespace lsdev;

template <int D, typename T>
__global__ void __launch_bounds__(256, 2) ls_kernel(const __grid_constant__ LsArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const GridBar gb{a.bar, gridDim.x, a.err, a.wait_ns ? a.wait_ns : kBarrierTimeoutNs};
    ls_solve_group<D, T>(a, blockIdx.x, gridDim.x, gb, smem_raw);
}

// full row-major DxD tensors from the symmetric storage (+ uniform antisymmetric part)
template <int D>
__global__ void full_tensor_kernel(const double* __restrict__ s, const double* __restrict__ epsp, const double* __restrict__ lam,
                                   const double* __restrict__ mu, double w0, double w1, double w2, int N, int want_sig,
                                   double* __restrict__ out) {
    constexpr int S = D == 2 ? 3 : 6;
    const double w[3] = {w0, w1, w2};
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < N; v += (long)gridDim.x * blockDim.x) {
        double e[S], ep[S];
#pragma unroll
        for (int c = 0; c < S; ++c) {
            e[c] = s[(long)c * N + v];
            ep[c] = epsp ? epsp[(long)c * N + v] : 0.0;
        }
        double* o = out + v * D * D;
        if (!want_sig) {
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    const double ww = (i == j) ? 0.0 : w[(D == 2) ? 0 : (i + j - 1)];
                    o[i * D + j] = e[sym_idx(D, i, j)] + (i < j ? ww : -ww);
                }
        } else {
            double tr = 0.0;
#pragma unroll
            for (int c = 0; c < D; ++c) tr += e[c] - ep[c];
            const double m2 = 2.0 * mu[v], l = lam[v];
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    const int c = sym_idx(D, i, j);
                    if (i == j) {
                        o[i * D + j] = m2 * (e[c] - ep[c]) + l * tr;
                    } else {
                        const double ww = w[(D == 2) ? 0 : (i + j - 1)];
                        o[i * D + j] = m2 * (e[c] + (i < j ? ww : -ww) - ep[c]);
                    }
                }
        }
    }
}

template <int D>
__global__ void split_tensor_kernel(const double* __restrict__ full, int N, double* __restrict__ s) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < N; v += (long)gridDim.x * blockDim.x) {
        const double* f = full + v * D * D;
        for (int i = 0; i < D; ++i)
            for (int j = i; j < D; ++j) s[(long)sym_idx(D, i, j) * N + v] = (i == j) ? f[i * D + i] : 0.5 * (f[i * D + j] + f[j * D + i]);
    }
}

}  // namespace

// ---------------------------------------------------------------- host side
// shared-memory line length of a length-n transform (pad_len in fft.cuh)
static size_t padded_len(int n) { return (size_t)n + (size_t)(n >> 3) + 1; }

bool plan_radices(int n, FftAxis* ax) {
    std::memset(ax, 0, sizeof(*ax));
    ax->n = n;
    int m = n, k = 0;
    while (m % 8 == 0 && m >= 64 && k < kMaxStages) { ax->radix[k++] = 8; m /= 8; }
    while (m % 4 == 0 && k < kMaxStages) { ax->radix[k++] = 4; m /= 4; }
    static const int primes[] = {2, 3, 5, 7};
    for (int p : primes)
        while (m % p == 0 && k < kMaxStages) { ax->radix[k++] = p; m /= p; }
    if (m != 1) return false;
    ax->nst = k;
    ax->lw = warp_lines(*ax);
    return true;
}

bool plan_axis(int n, FftAxis* ax, std::vector<void*>* owned) {
    if (!plan_radices(n, ax)) return false;
    std::vector<double> t64(2 * (size_t)n);
    std::vector<float> t32(2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)i / (long double)n;
        t64[2 * i] = (double)cosl(ang);
        t64[2 * i + 1] = (double)sinl(ang);
        t32[2 * i] = (float)cosl(ang);
        t32[2 * i + 1] = (float)sinl(ang);
    }
    void *d64 = nullptr, *d32 = nullptr;
    if (cudaMalloc(&d64, sizeof(double) * 2 * n) != cudaSuccess) return false;
    if (cudaMalloc(&d32, sizeof(float) * 2 * n) != cudaSuccess) return false;
    cudaMemcpy(d64, t64.data(), sizeof(double) * 2 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d32, t32.data(), sizeof(float) * 2 * n, cudaMemcpyHostToDevice);
    owned->push_back(d64);
    owned->push_back(d32);
    ax->tw64 = reinterpret_cast<const cplx<double>*>(d64);
    ax->tw32 = reinterpret_cast<const cplx<float>*>(d32);
    return true;
}

int plan_items(const LsArgs& a) {
    const int row_items = (a.nrows + a.rpb - 1) / a.rpb;
    const int no = a.D == 2 ? 1 : std::min(a.dims[0], a.dims[1]);
    const int col_items = no * ((a.nh + a.tk - 1) / a.tk);
    return std::max(row_items, col_items);
}

size_t plan_passes(LsArgs& a, int ncta, size_t smem_cap, LsPlan plan) {
    const int D = a.D, S = a.S;
    ncta = std::max(ncta, 1);
    int rpb = plan.rpb, tk = plan.tk;
    const int path = plan.path < 0 ? (D == 2 ? 1 : 0) : plan.path;
    for (int ax = 0; ax < D; ++ax) {
        a.ax[ax].lw = 0;
        if (path == 0) a.ax[ax].lw = warp_lines(a.ax[ax]);
    }
    a.nhs = (a.nh + 3) / 4 * 4;
    const size_t elem = sizeof(cplx<double>);  // the FP32 kernel uses half of it
    auto al = [](size_t b) { return (b + 127) / 128 * 128; };
    const bool two = true;  // both transform paths run between two line buffers
    size_t maxn = a.nr;
    size_t colp = 0;
    for (int ax = 0; ax < D - 1; ++ax) {
        colp = std::max(colp, padded_len(a.dims[ax]));
        maxn = std::max(maxn, (size_t)a.dims[ax]);
    }
    const size_t tw_b = al(maxn * elem);
    auto row_b = [&](int r) { return (size_t)((r * S + 1) / 2) * padded_len(a.nr) * elem; };
    auto col_b = [&](int t) { return (size_t)S * t * colp * elem; };
    auto total = [&](size_t line) { return (two ? 2 : 1) * al(line) + tw_b + kLsScratchBytes; };
    if (total(std::max(row_b(1), col_b(1))) > smem_cap) return 0;
    // largest chunk / tile that fits
    int rpb_max = 1;
    while (rpb_max < a.nrows && total(std::max(row_b(rpb_max + 1), col_b(1))) <= smem_cap) ++rpb_max;
    int tk_max = 1;
    while (tk_max < a.nh && total(std::max(row_b(1), col_b(tk_max + 1))) <= smem_cap) ++tk_max;
    // default: every CTA gets one chunk (row pass) and one tile (strided
    // passes) when the grid allows it; tiles of at least two columns on
    // larger grids, so that a tile row is a whole 32-byte sector
    const int no = D == 2 ? 1 : std::min(a.dims[0], a.dims[1]);
    if (rpb <= 0) rpb = std::max((a.nrows + ncta - 1) / ncta, D == 2 ? 2 : 1);
    if (tk <= 0) {
        const int tiles = std::max(1, (ncta + no - 1) / no);  // tiles wanted per outer index
        tk = (a.nh + tiles - 1) / tiles;
        if ((long)a.N >= (1L << 18)) tk = std::max(tk, 2);
    }
    a.rpb = std::max(1, std::min(rpb, rpb_max));
    a.tk = std::max(1, std::min(tk, tk_max));
    const size_t line = al(std::max(row_b(a.rpb), col_b(a.tk)));
    a.smem_half = (int)line;
    a.tw_off = (int)((two ? 2 : 1) * line);
    a.scr_off = a.tw_off + (int)tw_b;
    return (size_t)a.scr_off + kLsScratchBytes;
}

static void lame(double E, double nu, int D, bool ps, double* lam, double* mu) {
    // compute_lame_2d / compute_lame_3d (linear_elastic_solver.hpp:36-45, :315-319)
    *mu = E / (2.0 * (1.0 + nu));
    if (D == 2 && ps) *lam = E * nu / (1.0 - nu * nu);
    else *lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

#define MGK_CK(x)                                                        \
    do {                                                                 \
        cudaError_t e_ = (x);                                            \
        if (e_ != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e_)); \
    } while (0)

LsSolver::LsSolver(int D, const int* dims, bool plane_stress, double pixel, const double* E, const double* nu, cudaStream_t stream)
    : D_(D), S_(n_sym(D)), plane_stress_(plane_stress), pixel_(pixel), stream_(stream) {
    if (D != 2 && D != 3) throw std::invalid_argument("dimension must be 2 or 3");
    dims_[0] = dims[0];
    dims_[1] = dims[1];
    dims_[2] = D == 3 ? dims[2] : 1;
    for (int i = 0; i < D; ++i)
        if (dims_[i] < 1) throw std::invalid_argument("grid sizes must be positive");
    long N = (long)dims_[0] * dims_[1] * dims_[2];
    if (N > (1L << 30)) throw std::invalid_argument("grid too large");
    N_ = (int)N;
    // reference medium from voxel means (serial sums as linear_elastic_solver.hpp:164-169)
    double Es = 0.0, ns = 0.0;
    for (long i = 0; i < N; ++i) {
        Es += E[i];
        ns += nu[i];
    }
    lame(Es / N, ns / N, D, plane_stress, &lam0_, &mu0_);
    std::vector<double> lam(N), mu(N);
    sum_two_mu_ = 0.0;
    for (long i = 0; i < N; ++i) {
        lame(E[i], nu[i], D, plane_stress, &lam[i], &mu[i]);
        sum_two_mu_ += 2.0 * mu[i];
    }
    const int nr = dims_[D - 1];
    const int nh = nr / 2 + 1;
    const int nrows = (int)(N / nr);
    LsArgs& a = args_;
    a.D = D;
    a.S = S_;
    for (int i = 0; i < 3; ++i) a.dims[i] = dims_[i];
    a.N = N_;
    a.nr = nr;
    a.nh = nh;
    a.nrows = nrows;
    a.inv_n = 1.0 / (double)N;
    a.lam0 = lam0_;
    a.mu0 = mu0_;
    a.inv2mu0 = 1.0 / (2.0 * mu0_);
    a.bcoef = (lam0_ + mu0_) / (mu0_ * (lam0_ + 2.0 * mu0_));
    a.pixel = pixel;
    for (int i = 0; i < D; ++i)
        if (!plan_axis(dims_[i], &a.ax[i], &tw_bufs_)) throw std::invalid_argument("unsupported FFT length (prime factor > 7)");
    // decomposition: two CTAs per SM (the kernel's register bound), each with
    // up to half an SM's shared memory; passes tiled over every CTA
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm_, cudaDevAttrMultiProcessorCount, dev);
    if (plan_passes(a, kLsCtasPerSm * nsm_, kLsSmemCap) == 0)
        throw std::invalid_argument("grid axis too long for the shared-memory FFT");
    auto kfn = (D == 2) ? (const void*)ls_kernel<2, double> : (const void*)ls_kernel<3, double>;
    auto kfn32 = (D == 2) ? (const void*)ls_kernel<2, float> : (const void*)ls_kernel<3, float>;
    MGK_CK(ensure_dyn_smem(kfn, kLsSmemCap));
    MGK_CK(ensure_dyn_smem(kfn32, kLsSmemCap));
    // buffers (the partial sums sized for the largest grid any plan launches)
    bytes_ = 0;
    auto alloc = [&](void** p, size_t b) {
        MGK_CK(cudaMalloc(p, b));
        bytes_ += b;
    };
    alloc((void**)&d_eps_s_, sizeof(double) * S_ * N);
    alloc((void**)&d_lam_, sizeof(double) * N);
    alloc((void**)&d_mu_, sizeof(double) * N);
    alloc(&d_spec_, sizeof(cplx<double>) * S_ * (size_t)nrows * a.nhs);
    alloc((void**)&d_partials_, sizeof(double) * kMaxPartials * (kLsCtasPerSm * nsm_ + 1));
    alloc((void**)&d_res_, sizeof(LsResult));
    alloc((void**)&d_res32_, sizeof(LsResult));
    MGK_CK(cudaEventCreate(&ev0_));
    MGK_CK(cudaEventCreate(&ev1_));
    alloc((void**)&d_bar_, sizeof(unsigned) * 4);
    MGK_CK(cudaMemcpy(d_lam_, lam.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    MGK_CK(cudaMemcpy(d_mu_, mu.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    MGK_CK(cudaMemset(d_eps_s_, 0, sizeof(double) * S_ * N));
    MGK_CK(cudaMemset(d_bar_, 0, sizeof(unsigned) * 4));
    MGK_CK(cudaMemset(d_res_, 0, sizeof(LsResult)));
    MGK_CK(cudaMemset(d_res32_, 0, sizeof(LsResult)));
    a.eps_s = d_eps_s_;
    a.lam = d_lam_;
    a.mu = d_mu_;
    a.spec = d_spec_;
    a.partials = d_partials_;
    a.result = d_res_;
    a.bar = d_bar_;
    a.err = d_bar_ + 2;
    set_plan(autotune_enabled() ? tune(kLsCtasPerSm * nsm_, kLsSmemCap) : LsPlan());
}

bool LsSolver::autotune_enabled() {
    const char* e = std::getenv("MGK_LS_AUTOTUNE");
    return !(e && e[0] == '0');
}

void LsSolver::set_plan(const LsPlan& p) {
    LsArgs& a = args_;
    smem_ = plan_passes(a, kLsCtasPerSm * nsm_, kLsSmemCap, p);
    if (smem_ == 0) throw std::invalid_argument("grid axis too long for the shared-memory FFT");
    auto kfn = (D_ == 2) ? (const void*)ls_kernel<2, double> : (const void*)ls_kernel<3, double>;
    auto kfn32 = (D_ == 2) ? (const void*)ls_kernel<2, float> : (const void*)ls_kernel<3, float>;
    // the FP64 kernel and its FP32 twin (FP32-refined solves) share one grid:
    // the smaller of their co-resident block counts
    int per_sm = 0, per_sm32 = 0;
    MGK_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads_, smem_));
    MGK_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, kfn32, threads_, smem_));
    per_sm = std::min(per_sm, per_sm32);
    if (per_sm < 1) throw std::runtime_error("LS kernel does not fit on an SM");
    grid_ = std::max(1, std::min(plan_items(a), per_sm * nsm_));
    a.red = d_partials_ + (size_t)kMaxPartials * grid_;
    plan_ = LsPlan{a.rpb, a.tk, p.path < 0 ? (D_ == 2 ? 1 : 0) : p.path};
}

LsPlan LsSolver::tune(int ncta, size_t smem_cap) {
    static std::mutex mu;
    static std::map<std::string, LsPlan> cache;
    char key[160];
    int dev = 0;
    cudaGetDevice(&dev);
    snprintf(key, sizeof(key), "%d:%d:%dx%dx%d:%d:%zu:%d", dev, D_, dims_[0], dims_[1], dims_[2], ncta, smem_cap,
             (int)plane_stress_);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const int D = D_, S = S_;
    auto kfn = (D == 2) ? (const void*)ls_kernel<2, double> : (const void*)ls_kernel<3, double>;
    auto kfn32 = (D == 2) ? (const void*)ls_kernel<2, float> : (const void*)ls_kernel<3, float>;
    // candidates: both FFT paths, row chunks of 1x, 2x, 4x the one-per-CTA
    // size, column tiles of 1x and 2x the default width
    LsArgs base = args_;
    plan_passes(base, ncta, smem_cap, LsPlan{0, 0, 0});
    const int r0 = std::max(1, (base.nrows + ncta - 1) / ncta), t0 = base.tk;
    std::vector<LsPlan> cands;
    for (int path = 0; path < 2; ++path)
        for (int rm : {1, 2, 4})
            for (int tm : {1, 2}) {
                LsArgs t = args_;
                if (plan_passes(t, ncta, smem_cap, LsPlan{r0 * rm, t0 * tm, path}) == 0) continue;
                LsPlan c{t.rpb, t.tk, path};
                bool dup = false;
                for (const LsPlan& q : cands) dup |= q.rpb == c.rpb && q.tk == c.tk && q.path == c.path;
                if (!dup) cands.push_back(c);
            }
    // scratch state: the solver's own fields stay untouched
    double *eps = nullptr, *part = nullptr;
    LsResult* res = nullptr;
    unsigned* bar = nullptr;
    LsPlan best = LsPlan();
    float best_ms = 1e30f;
    if (cudaMalloc(&eps, sizeof(double) * S * N_) == cudaSuccess &&
        cudaMalloc(&part, sizeof(double) * kMaxPartials * (ncta + 1)) == cudaSuccess &&
        cudaMalloc(&res, sizeof(LsResult)) == cudaSuccess && cudaMalloc(&bar, sizeof(unsigned) * 4) == cudaSuccess) {
        for (const LsPlan& c : cands) {
            LsArgs t = args_;
            const size_t sm = plan_passes(t, ncta, smem_cap, c);
            int per_sm = 0, per_sm32 = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads_, sm) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, kfn32, threads_, sm) != cudaSuccess)
                continue;
            const int grid = std::min({plan_items(t), std::min(per_sm, per_sm32) * nsm_, ncta});
            if (grid < 1) continue;
            t.eps_s = eps;
            t.epsp_s = nullptr;
            t.partials = part;
            t.red = part + (size_t)kMaxPartials * grid;
            t.result = res;
            t.bar = bar;
            t.err = bar + 2;
            t.warm = 0;
            t.max_iter = 3;
            t.tol = 0.0;
            t.norm_extra = t.norm_extra_first = t.diff_extra_first = 0.0;
            for (int k = 0; k < 6; ++k) t.ebar_s[k] = k == 0 ? 1e-3 : (k < D ? -3e-4 : 0.0);
            void* prm[] = {&t};
            float ms = 1e30f;
            bool ok = true;
            for (int rep = 0; rep < 2 && ok; ++rep) {
                ok = cudaMemsetAsync(bar, 0, sizeof(unsigned) * 4, stream_) == cudaSuccess;
                ok = ok && cudaEventRecord(ev0_, stream_) == cudaSuccess;
                ok = ok && cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(threads_), prm, sm, stream_) == cudaSuccess;
                ok = ok && cudaEventRecord(ev1_, stream_) == cudaSuccess;
                ok = ok && cudaStreamSynchronize(stream_) == cudaSuccess;
                float m = 0.f;
                if (ok && rep == 1 && cudaEventElapsedTime(&m, ev0_, ev1_) == cudaSuccess) ms = m;
            }
            unsigned err = 0;
            if (ok) cudaMemcpy(&err, bar + 2, sizeof(unsigned), cudaMemcpyDeviceToHost);
            if (!ok || err) {
                cudaGetLastError();
                continue;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    }
    cudaFree(eps);
    cudaFree(part);
    cudaFree(res);
    cudaFree(bar);
    cudaGetLastError();
    cache[key] = best;
    return best;
}

LsSolver::~LsSolver() {
    cudaFree(d_eps_s_);
    cudaFree(d_lam_);
    cudaFree(d_mu_);
    cudaFree(d_spec_);
    cudaFree(d_partials_);
    cudaFree(d_res_);
    cudaFree(d_res32_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    cudaFree(d_bar_);
    for (void* p : tw_bufs_) cudaFree(p);
}

cudaError_t LsSolver::solve(const double* ebar, bool warm, const double* epsp_s, int max_iter, double tol) {
    LsArgs a = args_;
    const int D = D_;
    double wbar[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i)
        for (int j = i; j < D; ++j) {
            const int c = sym_idx(D, i, j);
            a.ebar_s[c] = (i == j) ? ebar[i * D + i] : 0.5 * (ebar[i * D + j] + ebar[j * D + i]);
            if (i != j) wbar[(D == 2) ? 0 : (i + j - 1)] = 0.5 * (ebar[i * D + j] - ebar[j * D + i]);
        }
    const int noff = D == 2 ? 1 : 3;
    double sw2 = 0.0, sdev = 0.0;
    for (int k = 0; k < noff; ++k) {
        sw2 += wbar[k] * wbar[k];
        sdev += asym_dev2_[k];
    }
    a.norm_extra = 2.0 * (double)N_ * sw2;
    if (warm) {
        a.norm_extra_first = 2.0 * (sdev + (double)N_ * sw2);
        a.diff_extra_first = 2.0 * sdev;
    } else {
        a.norm_extra_first = a.norm_extra;
        a.diff_extra_first = 0.0;
    }
    for (int k = 0; k < 3; ++k) {
        w_[k] = wbar[k];
        asym_dev2_[k] = 0.0;
    }
    a.warm = warm ? 1 : 0;
    a.max_iter = max_iter;
    a.tol = tol;
    a.epsp_s = epsp_s;
    h_res32_ = LsResult{};
    cudaEventRecord(ev0_, stream_);
    if (precision_ == 1 && max_iter > 1) {
        // FP32 phase: same passes on an FP32 spectrum (twiddles, Green
        // operator and FFT arithmetic in FP32), its own result record
        LsArgs a32 = a;
        a32.tol = std::max(tol, kFp32Tol);
        a32.max_iter = max_iter - 1;
        a32.result = d_res32_;
        void* p32[] = {&a32};
        auto k32 = (D == 2) ? (const void*)ls_kernel<2, float> : (const void*)ls_kernel<3, float>;
        cudaError_t e = cudaLaunchCooperativeKernel(k32, dim3(grid_), dim3(threads_), p32, smem_, stream_);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(&h_res32_, d_res32_, sizeof(LsResult), cudaMemcpyDeviceToHost, stream_);
        if (e != cudaSuccess) return e;
        // FP64 refinement from that field: a warm start whose mean is already
        // eps_bar, every iteration FP64, to the requested tolerance
        a.warm = 1;
        a.norm_extra_first = a.norm_extra;
        a.diff_extra_first = 0.0;
        a.max_iter = max_iter;  // each phase has the caller's cap; the reported count is their sum
    }
    void* params[] = {&a};
    auto kfn = (D == 2) ? (const void*)ls_kernel<2, double> : (const void*)ls_kernel<3, double>;
    cudaError_t e = cudaLaunchCooperativeKernel(kfn, dim3(grid_), dim3(threads_), params, smem_, stream_);
    if (e != cudaSuccess) return e;
    cudaEventRecord(ev1_, stream_);
    return cudaMemcpyAsync(&h_res_, d_res_, sizeof(LsResult), cudaMemcpyDeviceToHost, stream_);
}

double LsSolver::last_solve_ms() const {
    float ms = 0.f;
    return cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess ? (double)ms : -1.0;
}

void LsSolver::macro(double* em, double* sm, int* iters) const {
    const int D = D_;
    const double invN = 1.0 / (double)N_;
    const double mean2mu = sum_two_mu_ * invN;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            const int c = sym_idx(D, i, j);
            const double w = (i == j) ? 0.0 : w_[(D == 2) ? 0 : (i + j - 1)];
            const double sgn = (i < j) ? 1.0 : -1.0;
            em[i * D + j] = h_res_.sum_s[c] * invN + sgn * w;
            sm[i * D + j] = h_res_.sum_sig[c] * invN + sgn * w * mean2mu;
        }
    if (iters) *iters = h_res_.iters + h_res32_.iters;
}

unsigned LsSolver::device_error() const {
    unsigned e = 0;
    cudaMemcpy(&e, d_bar_ + 2, sizeof(unsigned), cudaMemcpyDeviceToHost);
    return e;
}

// on the solver's own (non-blocking) stream, so that the next launch on it
// sees the cleared words
void LsSolver::clear_error() {
    cudaMemsetAsync(d_bar_, 0, sizeof(unsigned) * 4, stream_);
    cudaStreamSynchronize(stream_);
}

cudaError_t LsSolver::download_eps(double* host) const {
    double* tmp = nullptr;
    size_t b = sizeof(double) * (size_t)N_ * D_ * D_;
    cudaError_t e = cudaMalloc(&tmp, b);
    if (e != cudaSuccess) return e;
    if (D_ == 2) full_tensor_kernel<2><<<256, 256, 0, stream_>>>(d_eps_s_, nullptr, d_lam_, d_mu_, w_[0], w_[1], w_[2], N_, 0, tmp);
    else full_tensor_kernel<3><<<256, 256, 0, stream_>>>(d_eps_s_, nullptr, d_lam_, d_mu_, w_[0], w_[1], w_[2], N_, 0, tmp);
    e = cudaMemcpyAsync(host, tmp, b, cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
    cudaFree(tmp);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t LsSolver::download_sig(const double* epsp_s, double* host) const {
    double* tmp = nullptr;
    size_t b = sizeof(double) * (size_t)N_ * D_ * D_;
    cudaError_t e = cudaMalloc(&tmp, b);
    if (e != cudaSuccess) return e;
    if (D_ == 2) full_tensor_kernel<2><<<256, 256, 0, stream_>>>(d_eps_s_, epsp_s, d_lam_, d_mu_, w_[0], w_[1], w_[2], N_, 1, tmp);
    else full_tensor_kernel<3><<<256, 256, 0, stream_>>>(d_eps_s_, epsp_s, d_lam_, d_mu_, w_[0], w_[1], w_[2], N_, 1, tmp);
    e = cudaMemcpyAsync(host, tmp, b, cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
    cudaFree(tmp);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t LsSolver::upload_eps(const double* host) {
    const int D = D_;
    // antisymmetric part: mean and spread per off-diagonal pair
    double mean[3] = {0, 0, 0}, dev[3] = {0, 0, 0};
    const int noff = D == 2 ? 1 : 3;
    const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
    for (int k = 0; k < noff; ++k) {
        const int i = pi[k], j = pj[k];
        double s = 0.0;
        for (int v = 0; v < N_; ++v) s += 0.5 * (host[(size_t)v * D * D + i * D + j] - host[(size_t)v * D * D + j * D + i]);
        mean[k] = s / N_;
        double d2 = 0.0;
        for (int v = 0; v < N_; ++v) {
            const double a = 0.5 * (host[(size_t)v * D * D + i * D + j] - host[(size_t)v * D * D + j * D + i]) - mean[k];
            d2 += a * a;
        }
        dev[k] = d2;
    }
    for (int k = 0; k < 3; ++k) {
        w_[k] = mean[k];
        asym_dev2_[k] = dev[k];
    }
    double* tmp = nullptr;
    size_t b = sizeof(double) * (size_t)N_ * D * D;
    cudaError_t e = cudaMalloc(&tmp, b);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(tmp, host, b, cudaMemcpyHostToDevice, stream_);
    if (D == 2) split_tensor_kernel<2><<<256, 256, 0, stream_>>>(tmp, N_, d_eps_s_);
    else split_tensor_kernel<3><<<256, 256, 0, stream_>>>(tmp, N_, d_eps_s_);
    cudaStreamSynchronize(stream_);
    cudaFree(tmp);
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace mgk

// ---------------------------------------------------------------------------
// Solve without allocating: mgk_ls_solve_noalloc (declared in mgkmc_b200.h).
//
// For callers that must not allocate device memory themselves or through this
// library: host applications that reserve the whole GPU for their own memory
// pool (a further cudaMalloc fails or fragments it), and loops that cannot
// afford cudaMalloc/cudaFree, which synchronise the device.  They hand in
// device buffers for the inputs and outputs; every intermediate (strain
// components, moduli, spectrum, twiddles, reduction partials, barrier words)
// lives in one static device array of MGK_NOALLOC_SCRATCH_BYTES that the
// library holds on every GPU it is loaded on, until the process exits.
namespace mgk {
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[MGK_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on the current device.  In host code the
// symbol g_noalloc_scratch only names a host-side stand-in, so it is never
// passed to a kernel; the address comes from cudaGetSymbolAddress with the
// device current.  It is looked up on every call (cheap once the module is
// loaded) rather than cached, so that a context re-created after
// cudaDeviceReset gets its own, valid address.
cudaError_t noalloc_scratch(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

// One CTA: sums of E, nu, mu and of the antisymmetric parts of eps (fixed order).
template <int D>
__global__ void noalloc_prep_kernel(const double* __restrict__ E, const double* __restrict__ nu, const double* __restrict__ eps,
                                    int N, int warm, double* __restrict__ out) {
    constexpr int NO = D == 2 ? 1 : 3;
    double v[3 + 2 * NO];
#pragma unroll
    for (int k = 0; k < 3 + 2 * NO; ++k) v[k] = 0.0;
    const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        v[0] += E[i];
        v[1] += nu[i];
        v[2] += E[i] / (2.0 * (1.0 + nu[i]));
        if (warm)
#pragma unroll
            for (int k = 0; k < NO; ++k) {
                const double a = 0.5 * (eps[(long)i * D * D + pi[k] * D + pj[k]] - eps[(long)i * D * D + pj[k] * D + pi[k]]);
                v[3 + k] += a;
                v[3 + NO + k] += a * a;
            }
    }
    __shared__ double scratch[(3 + 2 * NO) * 32];
    block_sum<3 + 2 * NO>(v, scratch);
    if (threadIdx.x == 0)
        for (int k = 0; k < 3 + 2 * NO; ++k) out[k] = v[k];
}

__global__ void noalloc_moduli_kernel(const double* __restrict__ E, const double* __restrict__ nu, int N, int D, int ps,
                                      double* __restrict__ lam, double* __restrict__ mu) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        mu[i] = E[i] / (2.0 * (1.0 + nu[i]));
        lam[i] = (D == 2 && ps) ? E[i] * nu[i] / (1.0 - nu[i] * nu[i]) : E[i] * nu[i] / ((1.0 + nu[i]) * (1.0 - 2.0 * nu[i]));
    }
}

__global__ void noalloc_twiddle_kernel(int n, cplx<double>* tw64, cplx<float>* tw32) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)k / (double)n, &s, &c);
        tw64[k] = {c, s};
        tw32[k] = {(float)c, (float)s};
    }
}

}  // namespace
}  // namespace mgk

namespace {
thread_local std::string g_noalloc_err;
mgk_status noalloc_fail(mgk_status s, const std::string& m) {
    g_noalloc_err = m;
    return s;
}
}  // namespace

const char* mgk_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

mgk_status mgk_ls_solve_noalloc(int dim, int nx, int ny, int nz, int plane_stress, double pixel, const double* E_dev,
                                const double* nu_dev, const double* eps_bar, const double* eps_plastic_dev, double* eps_dev,
                                int warm, double* sig_dev, double* macro_out, int max_iter, double tol, int* iters_out,
                                void* stream) {
    using namespace mgk;
    if (!E_dev || !nu_dev || !eps_bar || !eps_dev) return noalloc_fail(MGK_BAD_ARG, "null argument");
    if (dim != 2 && dim != 3) return noalloc_fail(MGK_BAD_SHAPE, "dim must be 2 or 3");
    if (nx < 1 || ny < 1 || (dim == 3 && nz < 1)) return noalloc_fail(MGK_BAD_SHAPE, "grid sizes must be positive");
    if (max_iter < 0) return noalloc_fail(MGK_BAD_ARG, "max_iter < 0");
    const int D = dim, S = n_sym(D), DD = D * D;
    const int dims[3] = {nx, ny, D == 3 ? nz : 1};
    const long N = (long)dims[0] * dims[1] * dims[2];
    const int nr = dims[D - 1], nh = nr / 2 + 1;
    const long nrows = N / nr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    LsArgs a{};
    a.D = D;
    a.S = S;
    for (int i = 0; i < 3; ++i) a.dims[i] = dims[i];
    a.nr = nr;
    a.nh = nh;
    for (int i = 0; i < D; ++i)
        if (!plan_radices(dims[i], &a.ax[i])) return noalloc_fail(MGK_BAD_SHAPE, "unsupported FFT length (prime factor > 7)");
    a.N = (int)N;
    a.nrows = (int)nrows;
    // decomposition: the same rules as LsSolver
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = plan_passes(a, kLsCtasPerSm * nsm, kLsSmemCap);
    if (smem == 0) return noalloc_fail(MGK_BAD_SHAPE, "grid axis too long for the shared-memory FFT");
    auto kfn = (D == 2) ? (const void*)ls_kernel<2, double> : (const void*)ls_kernel<3, double>;
    if (ensure_dyn_smem(kfn, kLsSmemCap) != cudaSuccess)
        return noalloc_fail(MGK_CUDA_ERROR, "cannot configure the LS kernel");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, 256, smem) != cudaSuccess || per_sm < 1)
        return noalloc_fail(MGK_CUDA_ERROR, "LS kernel does not fit on an SM");
    const int grid = std::max(1, std::min(plan_items(a), per_sm * nsm));
    const size_t elem = sizeof(cplx<double>);
    // carve the static scratch array
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = (off + bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_bar = take(4 * sizeof(unsigned)), o_res = take(sizeof(LsResult)), o_sum = take(16 * sizeof(double));
    const size_t o_part = take(sizeof(double) * kMaxPartials * (grid + 1));
    size_t o_tw64[3] = {0, 0, 0}, o_tw32[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i) {
        o_tw64[i] = take(sizeof(cplx<double>) * dims[i]);
        o_tw32[i] = take(sizeof(cplx<float>) * dims[i]);
    }
    const size_t o_lam = take(sizeof(double) * N), o_mu = take(sizeof(double) * N), o_eps = take(sizeof(double) * S * N);
    const size_t o_epsp = eps_plastic_dev ? take(sizeof(double) * S * N) : 0;
    const size_t o_spec = take(elem * S * (size_t)nrows * a.nhs);
    if (off > (size_t)MGK_NOALLOC_SCRATCH_BYTES) {
        char msg[160];
        snprintf(msg, sizeof(msg), "grid needs %zu scratch bytes, above the %u-byte static limit", off,
                 (unsigned)MGK_NOALLOC_SCRATCH_BYTES);
        return noalloc_fail(MGK_BAD_SHAPE, msg);
    }
    unsigned char* base = nullptr;
    cudaError_t e = noalloc_scratch(&base);
    if (e != cudaSuccess) return noalloc_fail(MGK_CUDA_ERROR, std::string("scratch lookup: ") + cudaGetErrorString(e));
    double* sums = reinterpret_cast<double*>(base + o_sum);
    double* lam = reinterpret_cast<double*>(base + o_lam);
    double* mu = reinterpret_cast<double*>(base + o_mu);
    double* eps_s = reinterpret_cast<double*>(base + o_eps);
    double* epsp_s = eps_plastic_dev ? reinterpret_cast<double*>(base + o_epsp) : nullptr;
    // sums for the reference medium and the antisymmetric part of the warm start
    if (D == 2) noalloc_prep_kernel<2><<<1, 1024, 0, st>>>(E_dev, nu_dev, eps_dev, (int)N, warm, sums);
    else noalloc_prep_kernel<3><<<1, 1024, 0, st>>>(E_dev, nu_dev, eps_dev, (int)N, warm, sums);
    double hs[9] = {0};
    e = cudaMemcpyAsync(hs, sums, sizeof(double) * 9, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    double lam0, mu0;
    lame(hs[0] / N, hs[1] / N, D, plane_stress != 0, &lam0, &mu0);
    const double sum_two_mu = 2.0 * hs[2];
    a.N = (int)N;
    a.nrows = (int)nrows;
    a.inv_n = 1.0 / (double)N;
    a.lam0 = lam0;
    a.mu0 = mu0;
    a.inv2mu0 = 1.0 / (2.0 * mu0);
    a.bcoef = (lam0 + mu0) / (mu0 * (lam0 + 2.0 * mu0));
    a.pixel = pixel;
    const int noff = D == 2 ? 1 : 3;
    double wbar[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i)
        for (int j = i; j < D; ++j) {
            const int c = sym_idx(D, i, j);
            a.ebar_s[c] = (i == j) ? eps_bar[i * D + i] : 0.5 * (eps_bar[i * D + j] + eps_bar[j * D + i]);
            if (i != j) wbar[(D == 2) ? 0 : (i + j - 1)] = 0.5 * (eps_bar[i * D + j] - eps_bar[j * D + i]);
        }
    double sw2 = 0.0, sdev = 0.0;
    for (int k = 0; k < noff; ++k) {
        sw2 += wbar[k] * wbar[k];
        if (warm) {
            const double m = hs[3 + k] / N;
            sdev += std::max(0.0, hs[3 + noff + k] - N * m * m);
        }
    }
    a.norm_extra = 2.0 * (double)N * sw2;
    a.norm_extra_first = warm ? 2.0 * (sdev + (double)N * sw2) : a.norm_extra;
    a.diff_extra_first = warm ? 2.0 * sdev : 0.0;
    a.warm = warm ? 1 : 0;
    a.max_iter = max_iter;
    a.tol = tol;
    // device set-up of the intermediates, all inside the scratch array
    noalloc_moduli_kernel<<<256, 256, 0, st>>>(E_dev, nu_dev, (int)N, D, plane_stress != 0, lam, mu);
    for (int i = 0; i < D; ++i) {
        auto* t64 = reinterpret_cast<cplx<double>*>(base + o_tw64[i]);
        auto* t32 = reinterpret_cast<cplx<float>*>(base + o_tw32[i]);
        noalloc_twiddle_kernel<<<(dims[i] + 255) / 256, 256, 0, st>>>(dims[i], t64, t32);
        a.ax[i].tw64 = t64;
        a.ax[i].tw32 = t32;
    }
    if (warm) {
        if (D == 2) split_tensor_kernel<2><<<256, 256, 0, st>>>(eps_dev, (int)N, eps_s);
        else split_tensor_kernel<3><<<256, 256, 0, st>>>(eps_dev, (int)N, eps_s);
    }
    if (epsp_s) {
        if (D == 2) split_tensor_kernel<2><<<256, 256, 0, st>>>(eps_plastic_dev, (int)N, epsp_s);
        else split_tensor_kernel<3><<<256, 256, 0, st>>>(eps_plastic_dev, (int)N, epsp_s);
    }
    // barrier words and the error word must start at zero on every call
    e = cudaMemsetAsync(base + o_bar, 0, 4 * sizeof(unsigned), st);
    if (e != cudaSuccess) return noalloc_fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    a.eps_s = eps_s;
    a.epsp_s = epsp_s;
    a.lam = lam;
    a.mu = mu;
    a.spec = base + o_spec;
    a.partials = reinterpret_cast<double*>(base + o_part);
    a.red = a.partials + (size_t)kMaxPartials * grid;
    a.result = reinterpret_cast<LsResult*>(base + o_res);
    a.bar = reinterpret_cast<unsigned*>(base + o_bar);
    a.err = a.bar + 2;
    void* params[] = {&a};
    e = cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(256), params, smem, st);
    if (e != cudaSuccess) return noalloc_fail(MGK_CUDA_ERROR, std::string("LS launch: ") + cudaGetErrorString(e));
    if (D == 2) full_tensor_kernel<2><<<256, 256, 0, st>>>(eps_s, nullptr, lam, mu, wbar[0], wbar[1], wbar[2], (int)N, 0, eps_dev);
    else full_tensor_kernel<3><<<256, 256, 0, st>>>(eps_s, nullptr, lam, mu, wbar[0], wbar[1], wbar[2], (int)N, 0, eps_dev);
    if (sig_dev) {
        if (D == 2) full_tensor_kernel<2><<<256, 256, 0, st>>>(eps_s, epsp_s, lam, mu, wbar[0], wbar[1], wbar[2], (int)N, 1, sig_dev);
        else full_tensor_kernel<3><<<256, 256, 0, st>>>(eps_s, epsp_s, lam, mu, wbar[0], wbar[1], wbar[2], (int)N, 1, sig_dev);
    }
    LsResult res{};
    unsigned err_word = 0;
    e = cudaMemcpyAsync(&res, a.result, sizeof(LsResult), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err_word, a.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    if (err_word) return noalloc_fail(MGK_DEVICE_TIMEOUT, "device wait timed out in the LS solver");
    if (macro_out) {
        const double invN = 1.0 / (double)N, mean2mu = sum_two_mu * invN;
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j) {
                const int c = sym_idx(D, i, j);
                const double w = (i == j) ? 0.0 : wbar[(D == 2) ? 0 : (i + j - 1)];
                const double sgn = (i < j) ? 1.0 : -1.0;
                macro_out[i * D + j] = res.sum_s[c] * invN + sgn * w;
                macro_out[DD + i * D + j] = res.sum_sig[c] * invN + sgn * w * mean2mu;
            }
    }
    if (iters_out) *iters_out = res.iters;
    if (res.iters >= max_iter && max_iter > 0 && !(res.diff < tol)) return MGK_LS_NOT_CONVERGED;
    return MGK_OK;
}
