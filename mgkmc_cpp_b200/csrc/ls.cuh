// Lippmann-Schwinger (Moulinec-Suquet basic scheme) solver on the GPU.
//
// Replaces spectral_solver_2d / spectral_solver_3d of linear_elastic_solver.hpp
// (:146-309, :431-593) and the stored Green tensor of green_operator_2d/3d
// (:70-119, :344-396).  Design (B200):
//  * state in HBM, structure-of-arrays FP64: the symmetric part of the strain
//    (3 components in 2D, 6 in 3D) plus, per solve, the constant antisymmetric
//    part of the macroscopic strain (the reference keeps full 2x2 / 3x3
//    tensors; their antisymmetric part is always uniform, see ls.cu);
//  * one persistent cooperative kernel per solve: all iterations, the
//    convergence test and the macro averages run on the device, separated by
//    bounded grid barriers; no host round trip per iteration;
//  * real-to-complex transforms along the contiguous axis by packing two real
//    component lines into one complex FFT; strided passes along the other axes
//    on tiles staged through shared memory; the Green operator is applied in
//    closed form per k-point inside the last strided pass (no 16/81-double
//    tensor per voxel is stored or streamed).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "fft.cuh"

namespace mgk {

constexpr int kMaxPartials = 16;
// Launch shape of the one-solve kernel: 256-thread CTAs, two per SM (its
// register bound), each with at most this much dynamic shared memory (two
// such CTAs and their static shared memory fit an SM's 228 KB).
constexpr int kLsCtasPerSm = 2;
constexpr size_t kLsSmemCap = 104 * 1024;
// Reduction scratch of a solve in its dynamic shared memory: block sums (14
// values x 32 warps), the 256 group sums of the partials' gather, the sums
// and the warm-start shift.  (As static arrays every template instance of
// the solve held its own copy: 23 KB of the batched kernel's shared memory.)
constexpr size_t kLsScratchBytes = sizeof(double) * (14 * 32 + 256 + 16 + 8);
// relative-change target of the FP32 phase of an FP32-refined solve: above
// the FP32 rounding floor of the iteration (~1e-7 relative)
constexpr double kFp32Tol = 1e-6;

struct LsResult {
    int iters;
    int pad;
    double diff;
    double sum_s[6];
    double sum_sig[6];
};

struct LsArgs {
    int D, S;
    int dims[3];
    int N, nr, nh, nrows;  // voxels, contiguous-axis length, its half spectrum, rows = N / nr
    int nhs;               // spectrum row stride (nh rounded up to 4: 32-byte aligned rows)
    int rpb;               // rows per row-pass chunk
    int tk;                // columns per strided-pass tile
    int max_iter;
    int warm;
    double tol;
    double inv_n;          // 1 / N
    double norm_extra;     // 2 N sum_offdiag w^2: antisymmetric part of |eps|^2 (uniform field)
    double norm_extra_first;  // same for the first iteration (warm start of a non-uniform field)
    double diff_extra_first;  // antisymmetric part of |eps_new - eps|^2 in the first iteration
    int smem_half;         // byte offset of the second line buffer
    int tw_off;            // byte offset of the shared-memory twiddle table
    int scr_off;           // byte offset of the reduction scratch (kLsScratchBytes)
    double ebar_s[6];      // symmetric part of the prescribed mean strain
    double lam0, mu0, inv2mu0, bcoef;
    double pixel;
    // device arrays
    double* eps_s;         // S x N
    const double* epsp_s;  // S x N or null
    const double* lam;     // N
    const double* mu;      // N
    void* spec;            // S x nrows x nhs complex (T)
    double* partials;      // gridDim.x x kMaxPartials
    double* red;           // kMaxPartials: the reduced partials (written by the last CTA of a barrier)
    LsResult* result;
    unsigned* bar;
    unsigned* err;
    unsigned long long wait_ns;  // limit of one barrier wait (0: kBarrierTimeoutNs)
    int test_absent;       // fault injection: k > 0 makes CTA k-1 leave before its first barrier
    int pad1;
    FftAxis ax[3];         // per axis (x, y, z)
};

// A pass plan: rows per row chunk, columns per strided tile, and the FFT
// path (0 warp-owned lines where the axis allows it, 1 CTA-wide lines);
// 0 / -1 fields ask for the defaults.
struct LsPlan {
    int rpb = 0, tk = 0, path = -1;
};

class BatchEngine;

class LsSolver {
    friend class BatchEngine;

public:
    // dims: {nx, ny} (D=2) or {nx, ny, nz}; E, nu host arrays of N values.
    LsSolver(int D, const int* dims, bool plane_stress, double pixel, const double* E, const double* nu, cudaStream_t stream);
    ~LsSolver();
    LsSolver(const LsSolver&) = delete;
    LsSolver& operator=(const LsSolver&) = delete;

    // Enqueue one solve on the stream.  ebar: full DxD row-major.  warm: keep the
    // current field and shift its mean to ebar (else fill with ebar).  epsp_s:
    // device S x N plastic strain or null.  Returns a cudaError_t.
    cudaError_t solve(const double* ebar, bool warm, const double* epsp_s, int max_iter, double tol);
    // Precision of the iterations: 0 FP64 (the reference's), 1 FP32 spectrum
    // and FFTs with an FP64 refinement: FP32 iterations (real-space fields,
    // polarisation, norms and sums stay FP64) until the relative change is
    // below max(tol, kFp32Tol), then FP64 iterations from that field to tol.
    void set_precision(int p) { precision_ = p; }
    // Limit of every device-side barrier wait of this solver's launches
    // (0: the 120 s default); a wait that runs out ends the launch with the
    // error word set (MGK_DEVICE_TIMEOUT on the C ABI).
    void set_wait_limit_ns(unsigned long long ns) { args_.wait_ns = ns; }
    // Fault injection for tests: cta >= 0 makes that CTA of the next solves
    // leave before its first barrier; -1 turns it off.
    void set_test_absent_cta(int cta) { args_.test_absent = cta >= 0 ? cta + 1 : 0; }
    int precision() const { return precision_; }
    // device time of the last solve's launches (CUDA events on the solver's
    // stream), after the stream has synchronised
    double last_solve_ms() const;

    // After the stream has synchronised: mean strain / stress (full DxD
    // row-major) of the last solve and its iteration count.
    void macro(double* eps_macro, double* sig_macro, int* iters) const;
    const LsResult& host_result() const { return h_res_; }
    LsResult* device_result() const { return d_res_; }
    unsigned device_error() const;  // syncs
    const unsigned* device_error_ptr() const { return d_bar_ + 2; }
    void clear_error();

    // Full-tensor fields (row-major DxD per voxel) to host; syncs.
    cudaError_t download_eps(double* host) const;
    cudaError_t download_sig(const double* epsp_s, double* host) const;
    cudaError_t upload_eps(const double* host);  // full tensors; sets the antisymmetric part

    int D() const { return D_; }
    int S() const { return S_; }
    int N() const { return N_; }
    double* eps_s() { return d_eps_s_; }
    const double* lam() const { return d_lam_; }
    const double* mu() const { return d_mu_; }
    double asym(int k) const { return w_[k]; }
    cudaStream_t stream() const { return stream_; }
    int grid() const { return grid_; }
    // Pass plan of the solver's launches, and the measured choice of one for
    // `ncta` CTAs within smem_cap bytes of shared memory: every candidate
    // (both FFT paths, row chunks of 1x/2x/4x the one-chunk-per-CTA size,
    // column tiles of 1x/2x the default width) runs three LS iterations of the
    // one-solve kernel on this solver's grid and moduli, on scratch copies of
    // the state, and the fastest wins.  Choices are cached per device, grid
    // shape and CTA count for the life of the process, so that solvers of
    // one shape run one plan (and round alike).  MGK_LS_AUTOTUNE=0 in the
    // environment turns the measurement off (the planner's defaults then).
    const LsPlan& plan() const { return plan_; }
    LsPlan tune(int ncta, size_t smem_cap);
    static bool autotune_enabled();
    size_t device_bytes() const { return bytes_; }

private:
    int D_, S_, N_;
    int dims_[3];
    bool plane_stress_;
    double pixel_;
    double lam0_, mu0_, sum_two_mu_;
    double w_[3] = {0, 0, 0};  // antisymmetric half-differences (xy, xz, yz): mean over voxels
    double asym_dev2_[3] = {0, 0, 0};  // sum over voxels of (a_v - w)^2 (non-uniform uploads)
    cudaStream_t stream_;
    double *d_eps_s_ = nullptr, *d_lam_ = nullptr, *d_mu_ = nullptr, *d_partials_ = nullptr;
    void* d_spec_ = nullptr;
    LsResult* d_res_ = nullptr;
    LsResult h_res_{};
    LsResult* d_res32_ = nullptr;  // result of the FP32 phase (precision 1)
    LsResult h_res32_{};
    int precision_ = 0;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    unsigned* d_bar_ = nullptr;  // {arrivals, generation, err}
    std::vector<void*> tw_bufs_;
    LsArgs args_{};
    void set_plan(const LsPlan& p);
    LsPlan plan_;
    int nsm_ = 148;
    int grid_ = 1, threads_ = 256;
    size_t smem_ = 0, bytes_ = 0;
};

// Plans the radix sequence of a length-n transform (radix-8 while n >= 64,
// radix-4, then 2, 3, 5, 7).  Returns false for lengths with other prime factors.
bool plan_axis(int n, FftAxis* ax, std::vector<void*>* owned);
// The radices alone (no twiddle tables); false for unsupported lengths.
bool plan_radices(int n, FftAxis* ax);

// Pass tiling of one solve run by ncta CTAs whose dynamic shared memory may
// not exceed smem_cap bytes: rows per row chunk (rpb) and columns per strided
// tile (tk) spread the work over the CTAs (defaults: one chunk and one tile
// per CTA, at least two rows a chunk in 2D; given values are clamped to what
// fits), the FFT path of every axis (default: CTA-wide lines in 2D,
// warp-owned lines in 3D, the faster of the two on B200 at these sizes), and
// the shared-memory layout (two line buffers and the twiddle table).  Needs
// a.D, a.S, a.dims, a.N, a.nr, a.nh, a.nrows and the axes' radices.  Returns
// the dynamic shared-memory bytes of a launch, 0 when nothing fits.
size_t plan_passes(LsArgs& a, int ncta, size_t smem_cap, LsPlan plan = LsPlan());
// Work items of a plan: the larger of the row chunks and the column tiles
// (a CTA beyond it idles in every pass).
int plan_items(const LsArgs& a);

}  // namespace mgk
