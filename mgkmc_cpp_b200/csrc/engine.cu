// KmcEngine implementation: construction (kmc_solver.hpp:165-257 / :1142-1232),
// elastic_run (:334-339), run_simulation (:721-1037 / :1735-2062) and
// run_cascade (:464-564 / :1473-1590) over device-resident fields.
//
// Per thermal event the host does one stream synchronisation: the device has
// already swept every mode (Q, rates, double-double total, unstable count);
// the host draws u1 (and, if the event happens, u2 and the redraw values) from
// the reference's RNG objects, uploads them with the target u2 * total, and
// enqueues select+flip, the warm-started LS solve and the next sweep in one go.
#include <chrono>
#include <cmath>
#include <sstream>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <limits>
#include <stdexcept>
#include <sys/stat.h>

#include "engine.cuh"
#include "vtu.h"

namespace mgk {

double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static std::string timestamp() {
    std::time_t t = std::time(nullptr);
    char buf[64];
    std::strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S", std::localtime(&t));
    return buf;
}

static double uniform(std::mt19937& g, double a, double b) {
    std::uniform_real_distribution<double> d(a, b);
    return d(g);
}

static double mod_rayleigh(const BarrierGen& b, std::mt19937& rng) {
    double lo = std::max(0.0, b.mean - 6.0 * b.std_val);
    double hi = b.mean + 6.0 * b.std_val;
    double xm = (b.mean + std::sqrt(b.mean * b.mean + 4.0 * b.std_val * b.std_val)) / 2.0;
    double cm = xm * std::exp(-((xm - b.mean) * (xm - b.mean)) / (2.0 * b.std_val * b.std_val));
    std::uniform_real_distribution<double> dx(lo, hi), du(0.0, cm);
    for (;;) {
        double x = dx(rng);
        double u = du(rng);
        double pdf = x * std::exp(-((x - b.mean) * (x - b.mean)) / (2.0 * b.std_val * b.std_val));
        if (u < pdf) return x;
    }
}

double BarrierGen::generate(std::mt19937& rng) const {
    double v = 0.0;
    if (type == 0) {
        std::normal_distribution<double> d(mean, std_val);
        v = d(rng);
    } else if (type == 1) {
        double u = uniform(rng, 0.0, 1.0);
        v = loc + scale * std::sqrt(-2.0 * std::log(1.0 - u));
    } else if (type == 2) {
        v = mod_rayleigh(*this, rng);
    } else if (type == 3) {
        double umix = uniform(rng, 0.0, 1.0);
        if (umix < ratio) v = -epsilon * std::log(1.0 - uniform(rng, 0.0, 1.0));
        else v = mod_rayleigh(*this, rng);
    }
    if (min_cutoff >= 0.0 && v < min_cutoff) v = min_cutoff;
    if (max_cutoff >= 0.0 && v > max_cutoff) v = max_cutoff;
    return v;
}

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

static const double kB = 8.617e-5;

KmcEngine::KmcEngine(const mgk_kmc_params& p, const double* E, const double* nu) : p_(p), rng_((unsigned)p.seed) {
    if (p.dim != 2 && p.dim != 3) throw std::invalid_argument("dim must be 2 or 3");
    if (p.nx < 1 || p.ny < 1 || (p.dim == 3 && p.nz < 1) || p.M < 1) throw std::invalid_argument("bad grid or M");
    if (p.fast_patching && (p.patch_radius < 0 || p.sync_interval < 1))
        throw std::invalid_argument("fast patching needs patch_radius >= 0 and sync_interval >= 1");
    if (p.catalog_type < 0 || p.catalog_type > 2) throw std::invalid_argument("catalog_type must be 0, 1 or 2");
    if (p.catalog_type == 2 && p.dim != 3) throw std::invalid_argument("the fibonacci catalog needs a 3D system");
    if (p.catalog_type == 2 && p.fast_patching)
        throw std::domain_error("fast patching needs a stored catalog (not the fibonacci catalog)");
    D_ = p.dim;
    S_ = D_ == 2 ? 3 : 6;
    C_ = (D_ == 3 && (p.use_3d_barriers || p.catalog_type == 2)) ? 6 : 2;
    M_ = p.M;
    const long N = (long)p.nx * p.ny * (D_ == 3 ? p.nz : 1);
    if (N * (long)M_ > 0x7fffffffL) throw std::invalid_argument("N*M exceeds 2^31");
    N_ = (int)N;
    NM_ = N * M_;
    E_.assign(E, E + N);
    nu_.assign(nu, nu + N);
    {
        double Es = 0.0, ns = 0.0;
        for (double v : E_) Es += v;
        for (double v : nu_) ns += v;
        E_avg_ = Es / E_.size();
        nu_avg_ = ns / nu_.size();
    }
    CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    int dims[3] = {p.nx, p.ny, D_ == 3 ? p.nz : 1};
    ls_.reset(new LsSolver(D_, dims, p.plane_stress != 0, p.pixel, E, nu, st_));
    if (p.ls_precision < 0 || p.ls_precision > 1) throw std::invalid_argument("ls_precision must be 0 or 1");
    ls_->set_precision(p.ls_precision);
    bar_.type = p.barrier_type;
    bar_.mean = p.bar_mean;
    bar_.std_val = p.bar_std;
    bar_.min_cutoff = p.bar_min_cutoff;
    bar_.max_cutoff = p.bar_max_cutoff;
    bar_.loc = p.bar_loc;
    bar_.scale = p.bar_scale;
    bar_.epsilon = p.bar_epsilon;
    bar_.ratio = p.bar_ratio;
    // physics constants (kmc_solver.hpp:182, 206-214, 784-786)
    phys_.volume = p.pixel * p.pixel * p.pixel;
    phys_.vnu = (p.scale_rate_by_volume ? phys_.volume : 1.0) * p.nu0;
    phys_.beta = p.temperature > 0.0 ? 1.0 / (kB * p.temperature) : std::numeric_limits<double>::infinity();
    phys_.tau = p.temperature > 0.0 ? 1.0 / (p.nu0 * std::exp(-p.q_act_temp / (kB * p.temperature)))
                                    : std::numeric_limits<double>::infinity();
    phys_.softening_cap = p.softening_cap;
    phys_.jp = p.jp;
    phys_.jt = p.jt;
    phys_.neigh = p.neighbor_fraction;
    phys_.threshold = p.stability_threshold;
    phys_.directional = p.directional;
    phys_.kmc_mode = p.instability_kmc;
    phys_.nx = p.nx;
    phys_.ny = p.ny;
    phys_.nz = D_ == 3 ? p.nz : 1;
    // redraw modes of a flip (kmc_solver.hpp:839-864; the catalog and
    // per-voxel barrier extensions: fixed catalogs are never redrawn, a
    // per-voxel barrier is one value for all M modes)
    {
        const bool all = p.redraw_directions || p.redraw_barriers;
        if (p.catalog_type == 0 && !p.barrier_per_voxel) {
            rd_dir_ = all ? (p.redraw_directions ? RD_ALL : RD_NONE) : RD_FLIPPED;
            rd_bar_ = all ? (p.redraw_barriers ? RD_ALL : RD_NONE) : RD_FLIPPED;
        } else {
            rd_dir_ = p.catalog_type != 0 ? RD_NONE : (p.redraw_directions ? RD_ALL : (all ? RD_NONE : RD_FLIPPED));
            if (p.barrier_per_voxel) rd_bar_ = (p.redraw_barriers || !all) ? RD_VOXEL : RD_NONE;
            else rd_bar_ = all ? (p.redraw_barriers ? RD_ALL : RD_NONE) : RD_FLIPPED;
        }
        nrec_ = (rd_dir_ == RD_ALL || rd_bar_ == RD_ALL) ? M_ : 1;
    }
    // initial barriers and catalog, voxel-major / mode-minor (kmc_solver.hpp:222-240 / :1200-1215);
    // a per-voxel barrier is drawn before the voxel's modes
    std::vector<double> Q0(NM_), cat(p.catalog_type == 2 ? 0 : NM_ * C_);
    std::normal_distribution<double> sn(0.0, 1.0);  // 2D: one object for the whole fill
    for (long v = 0; v < N; ++v) {
        const double qv = p.barrier_per_voxel ? bar_.generate(rng_) : 0.0;
        for (int m = 0; m < M_; ++m) {
            const long i = v * M_ + m;
            Q0[i] = p.barrier_per_voxel ? qv : bar_.generate(rng_);
            if (p.catalog_type == 0) {
                draw_mode(sn, &cat[i * C_]);
            } else if (p.catalog_type == 1) {
                // slip along (cos t, sin t) on the plane of normal (-sin t, cos t),
                // t = m pi / M: (gamma0/2) [[-sin 2t, cos 2t], [cos 2t, sin 2t]]
                const double a = 2.0 * M_PI * (double)m / (double)M_;
                cat[i * C_] = -0.5 * p.gamma0 * std::sin(a);
                cat[i * C_ + 1] = 0.5 * p.gamma0 * std::cos(a);
            }
        }
    }
    // device state
    auto alloc = [&](void** ptr, size_t b) { CK(cudaMalloc(ptr, b)); };
    dev_.D = D_;
    dev_.S = S_;
    dev_.C = C_;
    dev_.M = M_;
    dev_.N = N_;
    dev_.NM = NM_;
    alloc((void**)&dev_.Q0, sizeof(double) * NM_);
    alloc((void**)&dev_.Q, sizeof(double) * NM_);
    dev_.cat = nullptr;
    dev_.normals = nullptr;
    dev_.gamma0 = p.gamma0;
    if (p.catalog_type == 2) {
        // Fibonacci lattice on the upper hemisphere: z = 1 - (m + 1/2) / M,
        // azimuth m pi (3 - sqrt 5)
        std::vector<double> nv(3 * (size_t)M_);
        const double ga = M_PI * (3.0 - std::sqrt(5.0));
        for (int m = 0; m < M_; ++m) {
            const double z = 1.0 - ((double)m + 0.5) / (double)M_;
            const double r = std::sqrt(1.0 - z * z);
            const double ph = (double)m * ga;
            nv[3 * m] = r * std::cos(ph);
            nv[3 * m + 1] = r * std::sin(ph);
            nv[3 * m + 2] = z;
        }
        alloc((void**)&d_normals_, sizeof(double) * 3 * M_);
        CK(cudaMemcpy(d_normals_, nv.data(), sizeof(double) * 3 * M_, cudaMemcpyHostToDevice));
        dev_.normals = d_normals_;
    } else {
        alloc((void**)&dev_.cat, sizeof(double) * NM_ * C_);
    }
    alloc((void**)&dev_.epsp_s, sizeof(double) * S_ * N);
    alloc((void**)&dev_.soft, sizeof(double) * 2 * N);
    alloc((void**)&dev_.last_t, sizeof(double) * N);
    alloc((void**)&dev_.prev, sizeof(double) * C_ * N);
    dev_.eps_s = ls_->eps_s();
    dev_.lam = ls_->lam();
    dev_.mu = ls_->mu();
    CK(cudaMemcpy(dev_.Q0, Q0.data(), sizeof(double) * NM_, cudaMemcpyHostToDevice));
    if (dev_.cat) CK(cudaMemcpy(dev_.cat, cat.data(), sizeof(double) * NM_ * C_, cudaMemcpyHostToDevice));
    CK(cudaMemset(dev_.Q, 0, sizeof(double) * NM_));
    CK(cudaMemset(dev_.epsp_s, 0, sizeof(double) * S_ * N));
    CK(cudaMemset(dev_.soft, 0, sizeof(double) * 2 * N));
    CK(cudaMemset(dev_.prev, 0, sizeof(double) * C_ * N));
    std::vector<double> lt(N, -std::numeric_limits<double>::infinity());
    CK(cudaMemcpy(dev_.last_t, lt.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    nblk_ = kmc_sweep_blocks(NM_, items_);
    alloc((void**)&d_blk_, sizeof(dd) * nblk_);
    alloc((void**)&d_blk_unst_, sizeof(int) * nblk_);
    alloc((void**)&d_blk_last_, sizeof(int) * nblk_);
    alloc((void**)&d_status_, sizeof(KmcStatus));
    CK(cudaMemset(d_status_, 0, sizeof(KmcStatus)));
    CK(cudaMallocHost((void**)&h_status_, sizeof(KmcStatus)));
    CK(cudaMallocHost((void**)&h_lsres_, sizeof(LsResult)));
    CK(cudaMallocHost((void**)&h_lserr_, sizeof(unsigned)));
    *h_lserr_ = 0;
    std::memset(h_status_, 0, sizeof(KmcStatus));
    upload_cap_ = 1 + (size_t)M_ * (C_ + 1);
    alloc((void**)&d_upload_, sizeof(double) * upload_cap_);
    CK(cudaMallocHost((void**)&h_upload_, sizeof(double) * upload_cap_));
    int npow2 = 1;
    while (npow2 < N_) npow2 <<= 1;
    alloc((void**)&d_ckeys_, sizeof(double) * N);
    alloc((void**)&d_cmodes_, sizeof(int) * N);
    alloc((void**)&d_ckeys2_, sizeof(double) * npow2);
    alloc((void**)&d_cmodes2_, sizeof(int) * npow2);
    if (p.fast_patching) {
        fp_ = true;
        fp_R_ = p.patch_radius;
        fp_sync_ = p.sync_interval;
        alloc((void**)&dev_.sig_s, sizeof(double) * S_ * N);
        alloc((void**)&dev_.flipcat, sizeof(double) * C_ * N);
        alloc((void**)&d_unit_, sizeof(double) * S_);
        CK(cudaMemset(dev_.sig_s, 0, sizeof(double) * S_ * N));
        aux_.reset(new LsSolver(D_, dims, p.plane_stress != 0, p.pixel, E, nu, st_));
        precompute_patches();
    }
}

// precompute_patch_kernels (kmc_solver.hpp:276-332 / :1256-1331): the stress
// of a unit deviatoric eigenstrain at the centre voxel, for every basis,
// cropped to (2R+1)^D around it, plus the mean the crop misses.
void KmcEngine::precompute_patches() {
    const int D = D_, S = S_, R = fp_R_;
    const int nx = p_.nx, ny = p_.ny, nz = D == 3 ? p_.nz : 1;
    const int nb = D == 2 ? 2 : 5, side = 2 * R + 1, side_z = (D == 3 && nz > 1) ? side : 1;
    const long P = (long)side * side * side_z;
    const long N = N_;
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const long centre = ((long)cx * ny + cy) * nz + cz;
    // bases in symmetric components (2D: xx, yy, xy; 3D: xx, yy, zz, xy, xz, yz)
    static const double b2[2][3] = {{1, -1, 0}, {0, 0, 1}};
    static const double b3[5][6] = {{1, -1, 0, 0, 0, 0}, {0, 1, -1, 0, 0, 0}, {0, 0, 0, 1, 0, 0}, {0, 0, 0, 0, 1, 0},
                                    {0, 0, 0, 0, 0, 1}};
    static const int sym2[4] = {0, 2, 2, 1};
    static const int sym3[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
    std::vector<double> K((size_t)nb * P * S), miss((size_t)nb * S), sig((size_t)N * D * D);
    double* d_ep = nullptr;
    CK(cudaMalloc((void**)&d_ep, sizeof(double) * S * N));
    const double zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nb; ++b) {
        CK(cudaMemsetAsync(d_ep, 0, sizeof(double) * S * N, st_));
        for (int c = 0; c < S; ++c) {
            const double v = D == 2 ? b2[b][c] : b3[b][c];
            CK(cudaMemcpyAsync(d_ep + (long)c * N + centre, &v, sizeof(double), cudaMemcpyHostToDevice, st_));
            CK(cudaStreamSynchronize(st_));
        }
        CK(aux_->solve(zero, false, d_ep, 200, 1e-6));
        CK(cudaStreamSynchronize(st_));
        if (aux_->device_error()) throw std::runtime_error("device wait timed out in the LS solver");
        CK(aux_->download_sig(d_ep, sig.data()));
        double sum_crop[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int dx = -R; dx <= R; ++dx)
            for (int dy = -R; dy <= R; ++dy)
                for (int dz = (side_z > 1 ? -R : 0); dz <= (side_z > 1 ? R : 0); ++dz) {
                    const long sx = ((cx + dx) % nx + nx) % nx, sy = ((cy + dy) % ny + ny) % ny,
                               sz = ((cz + dz) % nz + nz) % nz;
                    const double* val = &sig[(size_t)((sx * ny + sy) * nz + sz) * D * D];
                    const long crop = ((long)(dx + R) * side + (dy + R)) * side_z + (side_z > 1 ? dz + R : 0);
                    for (int k = 0; k < D * D; ++k) {
                        const int c = D == 2 ? sym2[k] : sym3[k];
                        if (k / D <= k % D) K[((size_t)b * P + crop) * S + c] = val[k];
                        sum_crop[k] += val[k];
                    }
                }
        double sum_sig[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (long i = 0; i < N; ++i)
            for (int k = 0; k < D * D; ++k) sum_sig[k] += sig[(size_t)i * D * D + k];
        for (int k = 0; k < D * D; ++k) {
            if (k / D > k % D) continue;
            const double mean = sum_sig[k] / (double)N;
            miss[(size_t)b * S + (D == 2 ? sym2[k] : sym3[k])] = mean - sum_crop[k] / (double)N;
        }
    }
    cudaFree(d_ep);
    CK(cudaMalloc((void**)&d_patchK_, sizeof(double) * K.size()));
    CK(cudaMalloc((void**)&d_patchMiss_, sizeof(double) * miss.size()));
    CK(cudaMemcpy(d_patchK_, K.data(), sizeof(double) * K.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_patchMiss_, miss.data(), sizeof(double) * miss.size(), cudaMemcpyHostToDevice));
}

// After the flips of d_modes[0..nflips) (their pre-redraw catalog entries in
// dev_.flipcat): on the first thermal flip the macroscopic stress of a unit
// driving strain (sigma_macro_unit, one side solve); then the predictor
// (pred = strain_rate * t_wait, 0 for none) and the stencils.  Cascade flips
// (thermal false) add stencils only.
mgk_status KmcEngine::patch_after_flips(const int* d_modes, int nflips, double pred, bool thermal, int comp_i,
                                        int comp_j) {
    if (thermal && !unit_init_) {
        double eb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, em[9], sm[9];
        eb[comp_i * D_ + comp_j] = 1.0;
        CK(aux_->solve(eb, false, nullptr, 200, 1e-6));
        LsResult r;
        CK(cudaMemcpyAsync(&r, aux_->device_result(), sizeof(LsResult), cudaMemcpyDeviceToHost, st_));
        CK(cudaStreamSynchronize(st_));
        if (aux_->device_error()) {
            last_error = "device wait timed out in the LS solver";
            return MGK_DEVICE_TIMEOUT;
        }
        const_cast<LsResult&>(aux_->host_result()) = r;
        int it = 0;
        aux_->macro(em, sm, &it);
        double u[6];
        if (D_ == 2) {
            u[0] = sm[0], u[1] = sm[3], u[2] = sm[1];
        } else {
            u[0] = sm[0], u[1] = sm[4], u[2] = sm[8], u[3] = sm[1], u[4] = sm[2], u[5] = sm[5];
        }
        CK(cudaMemcpy(d_unit_, u, sizeof(double) * S_, cudaMemcpyHostToDevice));
        unit_init_ = true;
    }
    stats_.launches += 1;
    CK(kmc_patch(dev_, phys_, d_modes, nflips, d_patchK_, d_patchMiss_, fp_R_, d_unit_, unit_init_ ? pred : 0.0, st_));
    return MGK_OK;
}

KmcEngine::~KmcEngine() {
    if (st_) cudaStreamSynchronize(st_);
    if (f_summary_) fclose(f_summary_);
    if (f_global_) fclose(f_global_);
    cudaFree(dev_.Q0);
    cudaFree(dev_.Q);
    cudaFree(dev_.cat);
    cudaFree(d_normals_);
    cudaFree(dev_.epsp_s);
    cudaFree(dev_.soft);
    cudaFree(dev_.last_t);
    cudaFree(dev_.prev);
    cudaFree(d_blk_);
    cudaFree(d_blk_unst_);
    cudaFree(d_blk_last_);
    cudaFree(d_status_);
    cudaFree(d_upload_);
    cudaFree(d_ckeys_);
    cudaFree(d_cmodes_);
    cudaFree(d_ckeys2_);
    cudaFree(d_cmodes2_);
    cudaFree(dev_.sig_s);
    cudaFree(dev_.flipcat);
    cudaFree(d_unit_);
    cudaFree(d_patchK_);
    cudaFree(d_patchMiss_);
    cudaFreeHost(h_status_);
    cudaFreeHost(h_upload_);
    cudaFreeHost(h_lsres_);
    cudaFreeHost(h_lserr_);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    ls_.reset();
    if (st_) cudaStreamDestroy(st_);
}

// Mode generators: the 2D catalog draw (kmc_solver.hpp:231-238, 845-850),
// stz_mode_glass (:1042-1052, a fresh normal object per call) and
// stz_mode_glass_3d (:1054-1074).  `sn` is the caller's persistent object (2D).
void KmcEngine::draw_mode(std::normal_distribution<double>& sn, double* out) {
    const double g0 = p_.gamma0;
    if (D_ == 2) {
        double gxx = 0.5 * g0 * sn(rng_);
        double gxy = 0.5 * g0 * sn(rng_);
        out[0] = gxx;
        out[1] = gxy;
        return;
    }
    if (!p_.use_3d_barriers) {
        std::normal_distribution<double> g(0.0, 1.0);
        double gxx = 0.5 * g0 * g(rng_);
        double gxy = 0.5 * g0 * g(rng_);
        out[0] = gxx;
        out[1] = gxy;
        return;
    }
    std::normal_distribution<double> g(0.0, 1.0);
    double Mx[3][3], G[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Mx[i][j] = g(rng_);
    double Ms[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Ms[i][j] = 0.5 * (Mx[i][j] + Mx[j][i]);
    double tr = (Ms[0][0] + Ms[1][1]) + Ms[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i][j] = Ms[i][j] - (1.0 / 3.0) * tr * (i == j ? 1.0 : 0.0);
    double sq = 0.0;  // Frobenius norm, storage (column-major) order
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) sq += G[i][j] * G[i][j];
    double nrm = std::sqrt(sq);
    if (nrm < 1e-12) {
        for (int k = 0; k < 6; ++k) out[k] = 0.0;
        return;
    }
    double f = 1.0 / (std::sqrt(2.0) * nrm);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i][j] = G[i][j] * f;
    double u = uniform(rng_, 1e-15, 1.0);
    double mag = g0 * std::sqrt(-2.0 * std::log(u));
    out[0] = G[0][0] * mag;
    out[1] = G[1][1] * mag;
    out[2] = G[2][2] * mag;
    out[3] = G[0][1] * mag;
    out[4] = G[0][2] * mag;
    out[5] = G[1][2] * mag;
}

// One flip's redraw values (kmc_solver.hpp:839-864 / :1854-1875), in draw
// order, as nrec_ records of C + 1 values for the rd_dir_ / rd_bar_ modes.
void KmcEngine::gen_flip_draws(double* out) {
    std::normal_distribution<double> sn(0.0, 1.0);
    if (p_.catalog_type != 0 || p_.barrier_per_voxel) {
        // extensions: the per-voxel barrier first, then the modes' draws
        if (rd_bar_ == RD_VOXEL) out[C_] = bar_.generate(rng_);
        if (rd_dir_ == RD_ALL)
            for (int mm = 0; mm < M_; ++mm) draw_mode(sn, out + (size_t)mm * (C_ + 1));
        else if (rd_dir_ == RD_FLIPPED)
            draw_mode(sn, out);
        if (rd_bar_ == RD_ALL)
            for (int mm = 0; mm < M_; ++mm) out[(size_t)mm * (C_ + 1) + C_] = bar_.generate(rng_);
        else if (rd_bar_ == RD_FLIPPED)
            out[C_] = bar_.generate(rng_);
        return;
    }
    if (p_.redraw_directions || p_.redraw_barriers) {
        for (int mm = 0; mm < M_; ++mm) {
            double* r = out + (size_t)mm * (C_ + 1);
            if (p_.redraw_directions) draw_mode(sn, r);
            if (p_.redraw_barriers) r[C_] = bar_.generate(rng_);
        }
    } else {
        draw_mode(sn, out);
        out[C_] = bar_.generate(rng_);
    }
}

void KmcEngine::set_profiling(bool on) {
    if (on && !ev_[0])
        for (auto& e : ev_) cudaEventCreate(&e);
    profiling_ = on;
    prof_ = EngineProfile();
}

// event pairs: 0 LS solve, 1 sweep, 2 select+flip, 3 whole run
void KmcEngine::prof_begin(int pair) {
    if (profiling_) cudaEventRecord(ev_[2 * pair], st_);
}
void KmcEngine::prof_end(int pair) {
    if (!profiling_) return;
    cudaEventRecord(ev_[2 * pair + 1], st_);
    if (pair == 0) ls_ev_pending_ = true;
    if (pair == 1) sw_ev_pending_ = true;
    if (pair == 2) sel_ev_pending_ = true;
}
// after a stream sync: fold the recorded intervals into the profile
void KmcEngine::prof_collect() {
    if (!profiling_) return;
    float ms = 0.f;
    if (ls_ev_pending_ && cudaEventElapsedTime(&ms, ev_[0], ev_[1]) == cudaSuccess) {
        prof_.ls_ms += ms;
        prof_.ls_n++;
        prof_.ls_iters += h_lsres_->iters;
    }
    if (sw_ev_pending_ && cudaEventElapsedTime(&ms, ev_[2], ev_[3]) == cudaSuccess) {
        prof_.sweep_ms += ms;
        prof_.sweep_n++;
    }
    if (sel_ev_pending_ && cudaEventElapsedTime(&ms, ev_[4], ev_[5]) == cudaSuccess) {
        prof_.select_ms += ms;
        prof_.select_n++;
    }
    ls_ev_pending_ = sw_ev_pending_ = sel_ev_pending_ = false;
}

cudaError_t KmcEngine::enqueue_elastic() {
    prof_begin(0);
    stats_.launches += 1;
    cudaError_t e = ls_->solve(eps_macro_, true, dev_.epsp_s, p_.ls_max_iter, p_.ls_tol);
    prof_end(0);
    if (e == cudaSuccess && fp_) {
        stats_.launches += 1;
        e = kmc_stress(dev_, st_);  // the kept stress restarts from the solve
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_lsres_, ls_->device_result(), sizeof(LsResult), cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_lserr_, ls_->device_error_ptr(), sizeof(unsigned), cudaMemcpyDeviceToHost, st_);
    ls_pending_ = true;
    return e;
}

mgk_status KmcEngine::finish_elastic() {
    if (!ls_pending_) return MGK_OK;
    ls_pending_ = false;
    const_cast<LsResult&>(ls_->host_result()) = *h_lsres_;
    double em[9], sm[9];
    int it = 0;
    ls_->macro(em, sm, &it);
    std::memcpy(eps_macro_, em, sizeof(double) * D_ * D_);
    std::memcpy(sig_macro_, sm, sizeof(double) * D_ * D_);
    stats_.ls_solves++;
    stats_.ls_iters += it;
    return MGK_OK;
}

cudaError_t KmcEngine::enqueue_sweep() {
    prof_begin(1);
    stats_.launches += 1;
    cudaError_t e = kmc_sweep(dev_, phys_, time_, d_blk_, d_blk_unst_, d_blk_last_, nblk_, items_, d_status_, st_);
    prof_end(1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_status_, d_status_, sizeof(KmcStatus), cudaMemcpyDeviceToHost, st_);
    return e;
}

mgk_status KmcEngine::sync_status() {
    cudaError_t e = cudaStreamSynchronize(st_);
    stats_.syncs++;
    if (e != cudaSuccess) {
        last_error = cudaGetErrorString(e);
        return MGK_CUDA_ERROR;
    }
    if (h_status_->err) {
        last_error = "device selection error";
        return MGK_CUDA_ERROR;
    }
    if (ls_pending_ && *h_lserr_) {
        last_error = "device wait timed out in the LS solver";
        return MGK_DEVICE_TIMEOUT;
    }
    prof_collect();
    return finish_elastic();
}

mgk_status KmcEngine::elastic_run() {
    cudaError_t e = enqueue_elastic();
    if (e != cudaSuccess) {
        last_error = cudaGetErrorString(e);
        return MGK_CUDA_ERROR;
    }
    e = cudaStreamSynchronize(st_);
    if (e != cudaSuccess) {
        last_error = cudaGetErrorString(e);
        return MGK_CUDA_ERROR;
    }
    prof_collect();
    if (*h_lserr_) {
        last_error = "device wait timed out in the LS solver";
        return MGK_DEVICE_TIMEOUT;
    }
    return finish_elastic();
}

// run_cascade (kmc_solver.hpp:464-564): entered with a fresh sweep in
// h_status_ that found unstable modes.
mgk_status KmcEngine::run_cascade(int* steps, int* flips, long long cap) {
    int total = 0, local = 0;
    const long long limit = cap > 0 ? cap : (long long)N_;
    const size_t rec = (size_t)nrec_ * (C_ + 1);
    while (true) {
        if (h_status_->n_unstable == 0) break;
        int zero = 0;
        CK(cudaMemcpyAsync(&d_status_->n_collect, &zero, sizeof(int), cudaMemcpyHostToDevice, st_));
        CK(kmc_cascade_collect(dev_, phys_, d_ckeys_, d_cmodes_, d_status_, st_));
        stats_.launches += 1;
        CK(cudaMemcpyAsync(&h_status_->n_collect, &d_status_->n_collect, sizeof(int), cudaMemcpyDeviceToHost, st_));
        CK(cudaStreamSynchronize(st_));
        stats_.syncs++;
        const int n = h_status_->n_collect;
        if (n <= 0) break;
        // draws of the n flips in flip order (one normal object per flip)
        const size_t need = (size_t)n * rec;
        if (need > upload_cap_) {
            CK(cudaStreamSynchronize(st_));
            cudaFree(d_upload_);
            cudaFreeHost(h_upload_);
            upload_cap_ = need + 1;
            CK(cudaMalloc((void**)&d_upload_, sizeof(double) * upload_cap_));
            CK(cudaMallocHost((void**)&h_upload_, sizeof(double) * upload_cap_));
        }
        for (int f = 0; f < n; ++f) gen_flip_draws(h_upload_ + (size_t)f * rec);
        CK(cudaMemcpyAsync(d_upload_, h_upload_, sizeof(double) * need, cudaMemcpyHostToDevice, st_));
        CK(kmc_cascade_flip(dev_, phys_, d_ckeys_, d_cmodes_, n, d_ckeys2_, d_cmodes2_, time_, d_upload_, rd_dir_,
                            rd_bar_, d_status_, st_));
        {
            int np2 = 1, lg = 0;
            while (np2 < n) np2 <<= 1;
            while ((1 << lg) < np2) ++lg;
            stats_.launches += 1 + (np2 <= 8192 ? 1 : 1 + lg * (lg + 1) / 2);
        }
        if (fp_) {  // stencils per flip, in flip order; the LS solve after the cascade (kmc_solver.hpp:525-560)
            int np2 = 1;
            while (np2 < n) np2 <<= 1;
            mgk_status ps = patch_after_flips(np2 <= 8192 ? d_cmodes_ : d_cmodes2_, n, 0.0, false, 0, 0);
            if (ps != MGK_OK) return ps;
        } else {
            CK(enqueue_elastic());
        }
        total += n;
        ++local;
        CK(enqueue_sweep());
        mgk_status s = sync_status();
        if (s != MGK_OK) return s;
        if (local > limit) break;
    }
    if (fp_ && total > 0) {
        CK(enqueue_elastic());
        CK(enqueue_sweep());
        mgk_status s = sync_status();
        if (s != MGK_OK) return s;
    }
    *steps = local;
    *flips = total;
    stats_.cascades++;
    stats_.cascade_flips += total;
    return MGK_OK;
}

void KmcEngine::log_line(int global_step, int elastic_steps_done, int total_kmc, const char* type, int csteps, int cflips) {
    // do_logging (kmc_solver.hpp:606-719 / :1632-1733), same formats
    if (!f_summary_ && !f_global_ && !console_) return;
    const int D = D_;
    double elapsed = wall_seconds() - t_start_;
    double ev = eps_macro_[comp_i_ * D + comp_j_], sv = sig_macro_[comp_i_ * D + comp_j_];
    char buf[256];
    std::string now = timestamp();
    snprintf(buf, sizeof(buf), "%-22s %-12.2f %-8d %-15s %-12.6f %-15.3f %-8d %-8d %-8d %-15.6e\n", now.c_str(), elapsed,
             global_step, type, ev, sv / 1e9, total_kmc, csteps, cflips, time_);
    if (f_summary_) fputs(buf, f_summary_);
    if (console_) fputs(buf, stdout);
    if (f_global_) {
        char g[1024];
        if (D == 2) {
            double sig_zz = 0.0;
            if (!p_.plane_stress) {
                sig_zz = nu_avg_ * (sig_macro_[0] + sig_macro_[3]);
            }
            snprintf(g, sizeof(g),
                     "%-10d %-12d %-10d %-15.6f %-15.6f %-15.6f %-15.6f %-15.6f %-15.6f %-15.3f %-15.3f %-15.3f %-15.3f %-15.3f "
                     "%-15.3f %-14d %-17d %-15.6e\n",
                     global_step, elastic_steps_done, total_kmc, eps_macro_[0], eps_macro_[3], 0.0, eps_macro_[1], 0.0, 0.0,
                     sig_macro_[0] / 1e9, sig_macro_[3] / 1e9, sig_zz / 1e9, sig_macro_[1] / 1e9, 0.0, 0.0, csteps, cflips, time_);
        } else {
            snprintf(g, sizeof(g),
                     "%-10d %-12d %-10d %-15.6f %-15.6f %-15.6f %-15.6f %-15.6f %-15.6f %-15.3f %-15.3f %-15.3f %-15.3f %-15.3f "
                     "%-15.3f %-14d %-17d %-15.6e\n",
                     global_step, elastic_steps_done, total_kmc, eps_macro_[0], eps_macro_[4], eps_macro_[8], eps_macro_[1],
                     eps_macro_[2], eps_macro_[5], sig_macro_[0] / 1e9, sig_macro_[4] / 1e9, sig_macro_[8] / 1e9,
                     sig_macro_[1] / 1e9, sig_macro_[2] / 1e9, sig_macro_[5] / 1e9, csteps, cflips, time_);
        }
        fputs(g, f_global_);
    }
}

void KmcEngine::export_vtu(const std::string& name) {
    const int D = D_;
    const size_t N = N_;
    std::vector<double> eps(N * D * D), sig(N * D * D), epsp(N * D * D), soft(2 * N);
    long long cnt;
    get_field(0, eps.data(), &cnt);
    get_field(1, sig.data(), &cnt);
    get_field(2, epsp.data(), &cnt);
    get_field(3, soft.data(), &cnt);
    write_vtu_fields(name, D, p_.nx, p_.ny, D == 3 ? p_.nz : 1, eps.data(), sig.data(), E_.data(), nu_.data(), p_.pixel,
                     epsp.data(), soft.data());
}

void KmcEngine::maybe_vtk(int global_step, int elastic_steps_done, const char* type, bool init) {
    if (outdir_.empty() || vtk_interval_ == "none") return;
    std::string name;
    if (init) {
        if (vtk_interval_ == "last") return;
        if (vtk_interval_ == "current") name = outdir_ + "/step.vtu";
        else {
            char b[64];
            snprintf(b, sizeof(b), "/vtk_step_%06d.vtu", 0);
            name = outdir_ + b;
        }
    } else if (vtk_interval_ == "current") {
        name = outdir_ + "/step.vtu";
    } else {
        int interval = 0;
        try {
            interval = std::stoi(vtk_interval_);
        } catch (...) {
            return;
        }
        if (interval <= 0) return;
        bool ok = vtk_elastic_only_ ? (std::strcmp(type, "ELASTIC") == 0 && elastic_steps_done % interval == 0)
                                    : (global_step % interval == 0);
        if (!ok) return;
        char b[64];
        snprintf(b, sizeof(b), "/vtk_step_%06d.vtu", global_step);
        name = outdir_ + b;
    }
    export_vtu(name);
}

void KmcEngine::sync_host_rng() {
    if (batch_mt_.empty()) return;
    // std::mt19937's text form: the 624 state words, then the index
    std::ostringstream os;
    for (int i = 0; i < 624; ++i) os << batch_mt_[i] << " ";
    os << batch_mt_[624];
    std::istringstream is(os.str());
    is >> rng_;
    batch_mt_.clear();
}

mgk_status KmcEngine::run(const mgk_run_params& rp, double* trace, long long cap, long long* rows_out) {
    sync_host_rng();
    const int D = D_, DD = D * D;
    long long rows = 0;
    auto push = [&](double kind, double a, double b, double R, double tw) {
        if (trace && rows < cap) {
            double* r = trace + rows * (6 + 2 * DD);
            r[0] = kind;
            r[1] = a;
            r[2] = b;
            r[3] = R;
            r[4] = tw;
            r[5] = time_;
            for (int c = 0; c < DD; ++c) {
                r[6 + c] = eps_macro_[c];
                r[6 + DD + c] = sig_macro_[c];
            }
        }
        ++rows;
    };
    comp_i_ = rp.comp_i;
    comp_j_ = rp.comp_j;
    console_ = rp.enable_console != 0;
    vtk_interval_ = rp.vtk_interval ? rp.vtk_interval : "none";
    vtk_elastic_only_ = rp.vtk_elastic_only != 0;
    outdir_.clear();
    if (rp.output_dir && rp.output_dir[0]) {
        outdir_ = rp.output_dir;
        mkdir(outdir_.c_str(), 0755);
        const std::string header =
            "Timestamp              Elapsed(s)   Step     Type            Eps_xx       Sig_xx(GPa)     KMC      Cascade  Flips    SimTime(s)\n";
        if (rp.enable_summary_log) {
            f_summary_ = fopen((outdir_ + "/" + (rp.summary_filename ? rp.summary_filename : "summary_log.txt")).c_str(), "w");
            if (f_summary_) {
                fputs(header.c_str(), f_summary_);
                fputs((std::string(header.size() - 1, '-') + "\n").c_str(), f_summary_);
            }
        }
        if (rp.enable_global_log) {
            f_global_ = fopen((outdir_ + "/global_log.txt").c_str(), "w");
            if (f_global_)
                fprintf(f_global_, "%-10s %-12s %-10s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-15s %-14s %-17s SimTime(s)\n",
                        "GlobalStep", "ElasticStep", "KMCStep", "Eps_xx", "Eps_yy", "Eps_zz", "Eps_xy", "Eps_xz", "Eps_yz",
                        "Sig_xx(GPa)", "Sig_yy(GPa)", "Sig_zz(GPa)", "Sig_xy(GPa)", "Sig_xz(GPa)", "Sig_yz(GPa)", "CascadeSteps",
                        "TotalCascadeFlips");
        }
    }
    t_start_ = wall_seconds();
    auto close_logs = [&]() {
        if (f_summary_) fclose(f_summary_);
        if (f_global_) fclose(f_global_);
        f_summary_ = f_global_ = nullptr;
    };
    int elastic_done = 0, total_kmc = 0, step = 1, seq_instab = 0;
    const long long events_at_start = stats_.thermal_events;
    const int max_seq = (int)(rp.max_kmc_steps_pct * (double)N_);
    mgk_status s;
    try {
        if (profiling_) cudaEventRecord(ev_[6], st_);
        CK(enqueue_elastic());
        CK(enqueue_sweep());
        s = sync_status();
        if (s != MGK_OK) return s;
        if (console_) {
            fputs("Timestamp              Elapsed(s)   Step     Type            Eps_xx       Sig_xx(GPa)     KMC      Cascade  Flips    SimTime(s)\n", stdout);
            fputs("-----------------------------------------------------------------------------------------------------------------------------\n", stdout);
        }
        maybe_vtk(0, 0, "INIT", true);
        const int ci = rp.comp_i * D + rp.comp_j;
        const double dt_step = std::fabs(rp.step_size) / p_.strain_rate;
        double remaining = 0.0;
        std::uniform_real_distribution<double> U(0.0, 1.0);
        bool stop = false;
        while (elastic_done < rp.n_global_steps && !stop) {
            remaining += dt_step;
            while (remaining > 0.0) {
                // h_status_ holds the sweep of the current state (update_barriers)
                if (!p_.instability_kmc && h_status_->n_unstable > 0) {
                    int cs = 0, cf = 0;
                    s = run_cascade(&cs, &cf, rp.max_cascade_batches);
                    if (s != MGK_OK) {
                        close_logs();
                        return s;
                    }
                    if (cf > 0) {
                        log_line(step, elastic_done, total_kmc, "CASCADE", cs, cf);
                        maybe_vtk(step, elastic_done, "CASCADE", false);
                        push(1, cs, cf, 0, 0);
                        step++;
                    }
                    continue;
                }
                const double R = h_status_->total_hi + h_status_->total_lo;
                const double t_ev = wall_seconds();
                if (R > 0.0) {
                    const double u1 = U(rng_);
                    const double tw = -std::log(u1) / R;
                    if (tw < remaining) {
                        time_ += tw;
                        eps_macro_[ci] += 1.0 * (p_.strain_rate * tw);
                        remaining -= tw;
                        h_upload_[0] = U(rng_) * R;
                        gen_flip_draws(h_upload_ + 1);
                        const size_t nup = 1 + (size_t)nrec_ * (C_ + 1);
                        CK(cudaMemcpyAsync(d_upload_, h_upload_, sizeof(double) * nup, cudaMemcpyHostToDevice, st_));
                        prof_begin(2);
                        stats_.launches += 1;
                        CK(kmc_select_flip(dev_, phys_, d_blk_, d_blk_last_, nblk_, items_, d_upload_, time_, d_upload_ + 1,
                                           rd_dir_, rd_bar_, d_status_, st_));
                        prof_end(2);
                        if (fp_) {  // kmc_solver.hpp:866-915: predictor, stencil, LS only every sync_interval flips
                            s = patch_after_flips(&d_status_->selected, 1, tw > 0.0 ? p_.strain_rate * tw : 0.0, true,
                                                  rp.comp_i, rp.comp_j);
                            if (s != MGK_OK) {
                                close_logs();
                                return s;
                            }
                            if (++flips_since_sync_ >= fp_sync_) {
                                CK(enqueue_elastic());
                                flips_since_sync_ = 0;
                            }
                        } else {
                            CK(enqueue_elastic());
                        }
                        CK(enqueue_sweep());
                        s = sync_status();
                        if (s != MGK_OK) {
                            close_logs();
                            return s;
                        }
                        stats_.thermal_events++;
                        if (profiling_) prof_.event_us.push_back((wall_seconds() - t_ev) * 1e6);
                        if (h_status_->margin < stats_.min_margin) stats_.min_margin = h_status_->margin;
                        const bool instab = h_status_->is_instab != 0;
                        seq_instab = instab ? seq_instab + 1 : 0;
                        if (seq_instab > max_seq) {
                            if (console_)
                                printf("\n[TERMINATE] KMC instability sequence limit reached! %d steps.\n", seq_instab);
                            push(0, h_status_->selected, 1, R, tw);
                            close_logs();
                            if (rows_out) *rows_out = rows;
                            return MGK_TERMINATED;
                        }
                        log_line(step, elastic_done, total_kmc, instab ? "KMC_INSTAB" : "KMC", 0, 1);
                        maybe_vtk(step, elastic_done, instab ? "KMC_INSTAB" : "KMC", false);
                        push(0, h_status_->selected, instab ? 1 : 0, R, tw);
                        total_kmc++;
                        step++;
                        if (rp.max_events > 0 && stats_.thermal_events - events_at_start >= rp.max_events) {
                            stop = true;
                            break;
                        }
                        continue;
                    }
                    push(2, u1, 0, R, tw);
                }
                eps_macro_[ci] += 1.0 * (p_.strain_rate * remaining);
                time_ += remaining;
                remaining = 0.0;
            }
            if (stop) break;
            // mixed boundary conditions (kmc_solver.hpp:955-987)
            const double Ea = E_avg_, na = nu_avg_;
            int solves = 0;
            for (int it = 0; it < rp.mixed_max_iter; ++it) {
                s = elastic_run();
                if (s != MGK_OK) {
                    close_logs();
                    return s;
                }
                ++solves;
                double err[9] = {0}, emax = 0.0;
                for (int t = 0; t < rp.n_targets; ++t) {
                    const int k = rp.target_i[t] * D + rp.target_j[t];
                    const double e = rp.target_v[t] - sig_macro_[k];
                    err[k] = e;
                    emax = std::max(emax, std::fabs(e));
                }
                if (emax < rp.mixed_tol) break;
                double tr = 0.0;
                for (int a = 0; a < D; ++a) tr += err[a * D + a];
                for (int t = 0; t < rp.n_targets; ++t) {
                    const int a = rp.target_i[t], b = rp.target_j[t], k = a * D + b;
                    eps_macro_[k] += (err[k] - na * tr * (a == b ? 1.0 : 0.0)) / Ea;
                }
            }
            elastic_done++;
            stats_.elastic_steps++;
            log_line(step, elastic_done, total_kmc, "ELASTIC", 0, 0);
            maybe_vtk(step, elastic_done, "ELASTIC", false);
            push(3, solves, elastic_done, 0, 0);
            step++;
            // the state changed (eps_macro, LS): fresh sweep for the next interval
            CK(enqueue_sweep());
            s = sync_status();
            if (s != MGK_OK) {
                close_logs();
                return s;
            }
        }
        // final VTK (kmc_solver.hpp:998-1016)
        if (!outdir_.empty() && vtk_interval_ != "none") {
            bool fin = vtk_interval_ == "last";
            if (!fin) {
                try {
                    int interval = std::stoi(vtk_interval_);
                    fin = interval > 0 && (step - 1) % interval != 0;
                } catch (...) {
                }
            }
            if (fin) {
                char b[64];
                snprintf(b, sizeof(b), "/vtk_step_%06d_final.vtu", step - 1);
                export_vtu(outdir_ + b);
            }
        }
        double dur = wall_seconds() - t_start_;
        int h = (int)(dur / 3600.0), m = (int)((dur - h * 3600.0) / 60.0);
        double sec = dur - h * 3600.0 - m * 60.0;
        char fin[256];
        snprintf(fin, sizeof(fin), "\nSimulation Finish Time: %s\nTotal Duration: %.2f seconds (%dh %02dm %02ds)\n",
                 timestamp().c_str(), dur, h, m, (int)sec);
        if (f_summary_) fputs(fin, f_summary_);
        if (console_) fputs(fin, stdout);
    } catch (const std::exception& ex) {
        last_error = ex.what();
        close_logs();
        return MGK_CUDA_ERROR;
    }
    if (profiling_) {
        float ms = 0.f;
        cudaEventRecord(ev_[7], st_);
        cudaEventSynchronize(ev_[7]);
        if (cudaEventElapsedTime(&ms, ev_[6], ev_[7]) == cudaSuccess) prof_.run_ms += ms;
    }
    close_logs();
    if (rows_out) *rows_out = rows;
    return MGK_OK;
}

mgk_status KmcEngine::get_field(int field, double* dst, long long* count) {
    const int D = D_, DD = D * D;
    const long N = N_;
    long long n = 0;
    switch (field) {
        case 0: case 1: case 2: case 8: n = N * DD; break;
        case 3: n = 2 * N; break;
        case 4: case 9: case 10: n = N; break;
        case 5: case 6: n = NM_; break;
        case 7: n = dev_.cat ? NM_ * DD : 0; break;  // stress-dependent modes: no stored catalog
        default: last_error = "unknown field"; return MGK_BAD_ARG;
    }
    if (count) *count = n;
    if (!dst) return MGK_OK;
    cudaStreamSynchronize(st_);
    auto sym_to_full = [&](const std::vector<double>& s, int ncomp_is_cat, long cnt, double* out) {
        // s: per-item C (catalog) or S (sym) values, item-major for catalog, comp-major for fields
        (void)ncomp_is_cat;
        (void)cnt;
        (void)s;
        (void)out;
    };
    (void)sym_to_full;
    auto cat_full = [&](const double* c, double* o) {
        for (int k = 0; k < DD; ++k) o[k] = 0.0;
        if (C_ == 2) {
            o[0] = c[0];
            o[D + 1] = -c[0];
            o[1] = c[1];
            o[D] = c[1];
        } else {
            o[0] = c[0]; o[4] = c[1]; o[8] = c[2];
            o[1] = o[3] = c[3];
            o[2] = o[6] = c[4];
            o[5] = o[7] = c[5];
        }
    };
    try {
        if (field == 0) {
            CK(ls_->download_eps(dst));
        } else if (field == 1 && fp_) {
            // the kept (patched) stress field: its symmetric part, plus the
            // antisymmetric part of the last LS solve's stress (2 mu w, from
            // an applied strain with unequal off-diagonal halves)
            CK(ls_->download_sig(dev_.epsp_s, dst));
            std::vector<double> s((size_t)S_ * N);
            CK(cudaMemcpy(s.data(), dev_.sig_s, sizeof(double) * S_ * N, cudaMemcpyDeviceToHost));
            static const int m2[4] = {0, 2, 2, 1};
            static const int m3[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
            for (long v = 0; v < N; ++v) {
                double* o = dst + v * DD;
                double a[9];
                for (int i = 0; i < D; ++i)
                    for (int j = 0; j < D; ++j) a[i * D + j] = 0.5 * (o[i * D + j] - o[j * D + i]);
                for (int k = 0; k < DD; ++k) o[k] = s[(size_t)(D == 2 ? m2[k] : m3[k]) * N + v] + a[k];
            }
        } else if (field == 1) {
            CK(ls_->download_sig(dev_.epsp_s, dst));
        } else if (field == 2) {
            std::vector<double> s((size_t)S_ * N);
            CK(cudaMemcpy(s.data(), dev_.epsp_s, sizeof(double) * S_ * N, cudaMemcpyDeviceToHost));
            static const int map2[4] = {0, 2, 2, 1};
            static const int map3[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
            for (long v = 0; v < N; ++v)
                for (int k = 0; k < DD; ++k) dst[v * DD + k] = s[(size_t)(D == 2 ? map2[k] : map3[k]) * N + v];
        } else if (field == 3) {
            CK(cudaMemcpy(dst, dev_.soft, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost));
        } else if (field == 4) {
            CK(cudaMemcpy(dst, dev_.last_t, sizeof(double) * N, cudaMemcpyDeviceToHost));
        } else if (field == 5) {
            CK(cudaMemcpy(dst, dev_.Q, sizeof(double) * NM_, cudaMemcpyDeviceToHost));
        } else if (field == 6) {
            CK(cudaMemcpy(dst, dev_.Q0, sizeof(double) * NM_, cudaMemcpyDeviceToHost));
        } else if (field == 7) {
            if (!dev_.cat) return MGK_OK;
            std::vector<double> c((size_t)NM_ * C_);
            CK(cudaMemcpy(c.data(), dev_.cat, sizeof(double) * NM_ * C_, cudaMemcpyDeviceToHost));
            for (long i = 0; i < NM_; ++i) cat_full(&c[(size_t)i * C_], dst + i * DD);
        } else if (field == 8) {
            std::vector<double> c((size_t)N * C_);
            CK(cudaMemcpy(c.data(), dev_.prev, sizeof(double) * N * C_, cudaMemcpyDeviceToHost));
            for (long v = 0; v < N; ++v) cat_full(&c[(size_t)v * C_], dst + v * DD);
        } else if (field == 9) {
            std::memcpy(dst, E_.data(), sizeof(double) * N);
        } else if (field == 10) {
            std::memcpy(dst, nu_.data(), sizeof(double) * N);
        }
    } catch (const std::exception& ex) {
        last_error = ex.what();
        return MGK_CUDA_ERROR;
    }
    return MGK_OK;
}

void KmcEngine::get_macro(double* out, int n) const {
    const int DD = D_ * D_;
    std::vector<double> v;
    for (int c = 0; c < DD; ++c) v.push_back(eps_macro_[c]);
    for (int c = 0; c < DD; ++c) v.push_back(sig_macro_[c]);
    v.push_back(time_);
    v.push_back((double)stats_.thermal_events);
    v.push_back((double)stats_.cascades);
    v.push_back((double)stats_.ls_solves);
    v.push_back((double)stats_.ls_iters);
    v.push_back((double)stats_.elastic_steps);
    v.push_back(stats_.min_margin);
    v.push_back((double)stats_.syncs);
    v.push_back((double)stats_.launches);
    for (int i = 0; i < n && i < (int)v.size(); ++i) out[i] = v[i];
}

}  // namespace mgk
