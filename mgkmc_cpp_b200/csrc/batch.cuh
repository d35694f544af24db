// BatchEngine: replicas of KmcEngine advanced together by one persistent
// cooperative kernel with no host round trip per event (see batch.cu).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "engine.cuh"

namespace mgk {

struct BatchRep;
constexpr int kSelLog = 1 << 16;  // selected-mode log entries kept per replica and run

struct BatchStats {
    long long events = 0, cascades = 0, cascade_flips = 0, ls_solves = 0, ls_iters = 0, elastic_steps = 0, fallbacks = 0;
    double min_margin = 1.0;
    int terminated = 0;  // 1: instability sequence limit, 2: time limit
    int ncta = 0;
    double phase_ms[6] = {0, 0, 0, 0, 0, 0};  // group time in sweep, decide, event solve, cascade flips, cascade solve, interval end
    std::vector<int> sel;  // flat mode index of each thermal event, in order
};

class BatchEngine {
public:
    BatchEngine(int n, const mgk_kmc_params* params, const double* const* E, const double* const* nu);
    ~BatchEngine();
    // Advance every replica by up to max_events thermal events (or until its
    // n_global_steps elastic steps are done); rp holds one entry per replica.
    mgk_status run(const mgk_run_params* rp, long long max_events, double* elapsed_ms);
    int size() const { return (int)eng_.size(); }
    KmcEngine* replica(int r) { return eng_[r].get(); }
    const BatchStats& stats(int r) const { return last_[r]; }
    int total_ctas() const { return total_ctas_; }
    void set_time_limit(double seconds) { time_limit_s_ = seconds; }
    std::string last_error;

private:
    std::vector<std::unique_ptr<KmcEngine>> eng_;
    std::vector<int> ncta_;
    std::vector<void*> owned_;
    std::vector<BatchRep> reps_host_;
    std::vector<int> first_run_;
    std::vector<double> remaining_;
    std::vector<BatchStats> last_;
    BatchRep* alloc_reps_ = nullptr;
    int2* map_ = nullptr;
    size_t smem_ = 0;
    int total_ctas_ = 0;
    double time_limit_s_ = 60.0;
    cudaStream_t st_ = nullptr;
};

}  // namespace mgk
