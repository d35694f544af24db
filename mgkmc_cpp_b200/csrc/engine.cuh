// KmcEngine: the KmcSimulation2D / KmcSimulation3D object of kmc_solver.hpp,
// with its fields resident on the GPU.  Host side keeps what the reference's
// control flow needs: the RNG (std::mt19937 and libstdc++ distributions, the
// same objects in the same order as the reference, so every draw is identical),
// the clock, the macroscopic tensors and the logs.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/mgkmc_b200.h"
#include "kmc_kernels.cuh"
#include "ls.cuh"

namespace mgk {

// BarrierGenerator::generate (kmc_solver.hpp:35-95), same algorithm and draws.
struct BarrierGen {
    int type = 0;
    double mean = 2.0, std_val = 0.6, min_cutoff = 0.1, max_cutoff = -1.0, loc = 1.0, scale = 0.5, epsilon = 0.1, ratio = 0.8;
    double generate(std::mt19937& rng) const;
};

struct EngineStats {
    long long thermal_events = 0, cascades = 0, cascade_flips = 0, ls_solves = 0, ls_iters = 0, elastic_steps = 0;
    long long syncs = 0, launches = 0;
    double min_margin = 1.0;
};

// Optional per-kernel timing with CUDA events on the engine's stream
// (profiling mode): LS solves, sweeps, select+flip, plus per-event latency.
struct EngineProfile {
    double ls_ms = 0, sweep_ms = 0, select_ms = 0, run_ms = 0;
    long long ls_n = 0, ls_iters = 0, sweep_n = 0, select_n = 0;
    std::vector<double> event_us;  // host wall time per thermal event
};

class BatchEngine;

class KmcEngine {
    friend class BatchEngine;

public:
    KmcEngine(const mgk_kmc_params& p, const double* E, const double* nu);
    ~KmcEngine();

    mgk_status run(const mgk_run_params& rp, double* trace, long long cap, long long* rows);
    mgk_status elastic_run();  // solve and wait
    mgk_status get_field(int field, double* dst, long long* count);
    void get_macro(double* out, int n) const;

    const EngineStats& stats() const { return stats_; }
    void set_profiling(bool on);
    const EngineProfile& profile() const { return prof_; }
    int D() const { return D_; }
    long long N() const { return N_; }
    long long NM() const { return NM_; }
    std::string last_error;
    // interval state of the batched (device-resident) runs, kept with the
    // simulation so that it may move from one batch launch to the next
    bool batch_started = false;
    double batch_remaining = 0.0;

private:
    // enqueue an LS solve with eps_bar = eps_macro (no sync)
    cudaError_t enqueue_elastic();
    // read the LS result after a sync and update eps_macro / sig_macro
    mgk_status finish_elastic();
    cudaError_t enqueue_sweep();
    mgk_status sync_status();  // waits for the stream, copies status + LS result
    void gen_flip_draws(double* out);
    void draw_mode(std::normal_distribution<double>& sn, double* out);
    mgk_status run_cascade(int* steps, int* flips, long long cap);
    void log_line(int global_step, int elastic_steps_done, int total_kmc, const char* type, int csteps, int cflips);
    void maybe_vtk(int global_step, int elastic_steps_done, const char* type, bool init);
    void export_vtu(const std::string& name);
    // fast patching (kmc_solver.hpp:276-332 / :1256-1331, 866-913 / :1877-1939)
    void precompute_patches();
    mgk_status patch_after_flips(const int* d_modes, int nflips, double pred, bool thermal, int comp_i, int comp_j);

    mgk_kmc_params p_;
    int D_, S_, C_, M_, N_;
    int rd_dir_ = 0, rd_bar_ = 0, nrec_ = 1;  // RD_* redraw modes of a flip, records per flip
    double* d_normals_ = nullptr;             // catalog_type 2: M plane normals
    long NM_;
    cudaStream_t st_ = nullptr;
    std::unique_ptr<LsSolver> ls_;
    KmcDevState dev_{};
    KmcPhys phys_{};
    BarrierGen bar_;
    std::mt19937 rng_;
    // While batched runs own the generator, its state stays in their layout
    // (624 state words, the index, a pad word) and rng_ is brought up to date
    // from it only when the plain form draws again: a serving loop runs many
    // short batched runs back to back.  Empty: rng_ is current.
    std::vector<unsigned> batch_mt_;
    void sync_host_rng();
    std::vector<double> E_, nu_;
    double E_avg_ = 0.0, nu_avg_ = 0.0;  // means of E_ and nu_ (left-to-right sums), for the mixed-BC update
    double eps_macro_[9] = {0}, sig_macro_[9] = {0};
    double time_ = 0.0;
    // device scratch
    dd* d_blk_ = nullptr;
    int *d_blk_unst_ = nullptr, *d_blk_last_ = nullptr;
    int nblk_ = 0, items_ = 8;
    KmcStatus* d_status_ = nullptr;
    KmcStatus* h_status_ = nullptr;  // pinned
    double* d_upload_ = nullptr;     // target + draws
    double* h_upload_ = nullptr;     // pinned
    size_t upload_cap_ = 0;
    double *d_ckeys_ = nullptr, *d_ckeys2_ = nullptr;
    int *d_cmodes_ = nullptr, *d_cmodes2_ = nullptr;
    LsResult* h_lsres_ = nullptr;    // pinned copy of the last LS result
    bool fp_ = false;                 // fast patching
    int fp_R_ = 5, fp_sync_ = 100, flips_since_sync_ = 0;
    bool unit_init_ = false;          // sigma_macro_unit computed
    std::unique_ptr<LsSolver> aux_;   // the reference's side solves (patch kernels, unit macro stress)
    double *d_patchK_ = nullptr, *d_patchMiss_ = nullptr, *d_unit_ = nullptr;
    bool ls_pending_ = false;
    EngineStats stats_;
    // profiling
    bool profiling_ = false;
    EngineProfile prof_;
    cudaEvent_t ev_[8] = {};
    void prof_begin(int pair);
    void prof_end(int pair);
    void prof_collect();
    bool ls_ev_pending_ = false, sw_ev_pending_ = false, sel_ev_pending_ = false;
    unsigned* h_lserr_ = nullptr;  // pinned copy of the LS error word
    // logging
    FILE* f_summary_ = nullptr;
    FILE* f_global_ = nullptr;
    bool console_ = false;
    std::string outdir_, vtk_interval_;
    bool vtk_elastic_only_ = true;
    int comp_i_ = 0, comp_j_ = 0;
    double t_start_ = 0.0;
};

double wall_seconds();

}  // namespace mgk
