// BatchEngine: replicas of KmcEngine advanced together by one persistent
// cooperative kernel with no host round trip per event (see batch.cu).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "engine.cuh"

namespace mgk {

struct BatchRep;
struct RepState;
constexpr int kSelLog = 1 << 16;  // selected-mode log entries kept per replica and run

struct BatchStats {
    long long events = 0, cascades = 0, cascade_flips = 0, ls_solves = 0, ls_iters = 0, elastic_steps = 0, fallbacks = 0;
    double min_margin = 1.0;
    int terminated = 0;  // 1: instability sequence limit, 2: time limit
    int ncta = 0;
    long long sweeps = 0;  // sweeps of every (voxel, mode) done by the run
    long long h2d_bytes = 0, d2h_bytes = 0;  // host<->device bytes the run call copied for this replica
    double phase_ms[6] = {0, 0, 0, 0, 0, 0};  // group time in sweep, decide, event solve, cascade flips, cascade solve, interval end
    std::vector<int> sel;  // flat mode index of each thermal event, in order
    std::vector<double> event_us;  // device time from the previous event (or the run's first decision) to each event
};

// How a batch spreads its CTAs over the replicas (read when a batch is
// built): 0 throughput -- each CTA to the replica whose modelled event rate
// it raises most (small, latency-bound grids gain most); 1 balanced -- each
// CTA to the replica whose modelled rate is furthest below its rate on the
// whole GPU, so that every replica advances at a similar fraction of its
// single-replica speed (a shorter makespan for mixed sizes).
void set_batch_plan_objective(int objective);
int batch_plan_objective();

class BatchEngine {
public:
    BatchEngine(int n, const mgk_kmc_params* params, const double* const* E, const double* const* nu);
    // A batch over existing simulations (not owned; they must outlive the
    // batch).  Runs advance them in place; a simulation may belong to several
    // batches over its life, but to one running batch at a time.
    explicit BatchEngine(const std::vector<KmcEngine*>& sims);
    ~BatchEngine();
    // Advance every replica by up to max_events thermal events (or until its
    // n_global_steps elastic steps are done); rp holds one entry per replica.
    mgk_status run(const mgk_run_params* rp, long long max_events, double* elapsed_ms);
    int size() const { return (int)eng_.size(); }
    KmcEngine* replica(int r) { return eng_[r]; }
    const BatchStats& stats(int r) const { return last_[r]; }
    int total_ctas() const { return total_ctas_; }
    void set_time_limit(double seconds) { time_limit_s_ = seconds; }
    std::string last_error;

private:
    void init();  // device scratch and CTA plan for eng_
    std::vector<KmcEngine*> eng_;
    std::vector<std::unique_ptr<KmcEngine>> owned_eng_;
    std::vector<int> ncta_;
    char* arena_ = nullptr;       // every replica's device scratch (one allocation)
    RepState* d_state_ = nullptr;  // per replica: control block, generator, barrier words (in the arena)
    RepState* h_state_ = nullptr;  // pinned host copy of d_state_
    char* h_logs_ = nullptr;       // pinned staging of the run's event-time and selection logs
    size_t h_logs_cap_ = 0;
    std::vector<BatchRep> reps_host_;
    std::vector<long long> h2d_;
    std::vector<BatchStats> last_;
    BatchRep* alloc_reps_ = nullptr;
    int2* map_ = nullptr;
    unsigned* d_past_ = nullptr;  // {replicas past the time limit or finished, replicas} (in the arena)
    size_t smem_ = 0;
    int total_ctas_ = 0;
    double time_limit_s_ = 60.0;
    cudaStream_t st_ = nullptr;
};

}  // namespace mgk
