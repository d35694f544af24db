// extern "C" entry points of libmgkmc_b200.so (declared in include/mgkmc_b200.h).
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mgkmc_b200.h"
#include "batch.cuh"
#include "elastic.cuh"
#include "fieldgen.cuh"
#include "engine.cuh"
#include "ls.cuh"

namespace {
thread_local std::string g_err;

mgk_status fail(mgk_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

mgk_status from_exception(const std::exception& e) {
    g_err = e.what();
    if (dynamic_cast<const std::bad_alloc*>(&e)) return MGK_OOM;
    if (dynamic_cast<const std::domain_error*>(&e)) return MGK_UNSUPPORTED;
    if (dynamic_cast<const std::invalid_argument*>(&e)) return MGK_BAD_SHAPE;
    if (std::strstr(e.what(), "out of memory")) return MGK_OOM;
    return MGK_CUDA_ERROR;
}
}  // namespace

struct mgk_ls {
    cudaStream_t st = nullptr;
    mgk::LsSolver* solver = nullptr;
    int D = 2, N = 0;
    double* d_epsp = nullptr;  // S x N
};

struct mgk_kmc {
    mgk::KmcEngine* eng = nullptr;
};

struct mgk_batch {
    mgk::BatchEngine* b = nullptr;
};

extern "C" {

const char* mgk_last_error(void) { return g_err.c_str(); }
int mgk_version(void) { return 100; }
int mgk_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

mgk_status mgk_ls_create(mgk_ls** out, int dim, int nx, int ny, int nz, int plane_stress, double pixel, const double* E,
                         const double* nu) {
    if (!out || !E || !nu) return fail(MGK_BAD_ARG, "null argument");
    *out = nullptr;
    if (dim != 2 && dim != 3) return fail(MGK_BAD_SHAPE, "dim must be 2 or 3");
    if (nx < 1 || ny < 1 || (dim == 3 && nz < 1)) return fail(MGK_BAD_SHAPE, "grid sizes must be positive");
    mgk_ls* h = new (std::nothrow) mgk_ls;
    if (!h) return fail(MGK_OOM, "host allocation failed");
    try {
        if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) throw std::runtime_error("no CUDA device");
        int dims[3] = {nx, ny, dim == 3 ? nz : 1};
        h->solver = new mgk::LsSolver(dim, dims, plane_stress != 0, pixel, E, nu, h->st);
        h->D = dim;
        h->N = h->solver->N();
    } catch (const std::exception& e) {
        mgk_status s = from_exception(e);
        delete h->solver;
        if (h->st) cudaStreamDestroy(h->st);
        delete h;
        return s;
    }
    *out = h;
    return MGK_OK;
}

mgk_status mgk_ls_set_precision(mgk_ls* h, int precision) {
    if (!h || precision < 0 || precision > 1) return fail(MGK_BAD_ARG, "precision must be 0 (FP64) or 1 (FP32-refined)");
    h->solver->set_precision(precision);
    return MGK_OK;
}

mgk_status mgk_ls_set_wait_limit(mgk_ls* h, double seconds) {
    if (!h || !(seconds >= 0.0) || seconds > 1e6) return fail(MGK_BAD_ARG, "wait limit must be in [0, 1e6] seconds");
    h->solver->set_wait_limit_ns((unsigned long long)(seconds * 1e9));
    return MGK_OK;
}

mgk_status mgk_ls_inject_absent_cta(mgk_ls* h, int cta) {
    if (!h || cta < -1) return fail(MGK_BAD_ARG, "cta must be -1 (off) or a CTA index");
    if (cta >= h->solver->grid()) return fail(MGK_BAD_ARG, "cta beyond the solver's grid");
    h->solver->set_test_absent_cta(cta);
    return MGK_OK;
}

mgk_status mgk_ls_plan(mgk_ls* h, int* out4) {
    if (!h || !out4) return fail(MGK_BAD_ARG, "null argument");
    const mgk::LsPlan& p = h->solver->plan();
    out4[0] = p.rpb;
    out4[1] = p.tk;
    out4[2] = p.path;
    out4[3] = h->solver->grid();
    return MGK_OK;
}

mgk_status mgk_ls_last_solve_ms(mgk_ls* h, double* ms) {
    if (!h || !ms) return fail(MGK_BAD_ARG, "null argument");
    *ms = h->solver->last_solve_ms();
    return MGK_OK;
}

mgk_status mgk_ls_solve(mgk_ls* h, const double* eps_bar, const double* eps_plastic, double* eps_inout, int warm,
                        double* sig_out, double* macro_out, int max_iter, double tol, int* iters_out) {
    if (!h || !eps_bar || !eps_inout) return fail(MGK_BAD_ARG, "null argument");
    if (max_iter < 0) return fail(MGK_BAD_ARG, "max_iter < 0");
    const int D = h->D, DD = D * D, S = D == 2 ? 3 : 6;
    const long N = h->N;
    try {
        if (warm) {
            cudaError_t e = h->solver->upload_eps(eps_inout);
            if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
        }
        const double* dep = nullptr;
        if (eps_plastic) {
            if (!h->d_epsp && cudaMalloc(&h->d_epsp, sizeof(double) * S * N) != cudaSuccess) throw std::bad_alloc();
            std::vector<double> s((size_t)S * N);
            for (long v = 0; v < N; ++v) {
                const double* f = eps_plastic + v * DD;
                if (D == 2) {
                    s[v] = f[0];
                    s[N + v] = f[3];
                    s[2 * N + v] = 0.5 * (f[1] + f[2]);
                } else {
                    s[v] = f[0];
                    s[N + v] = f[4];
                    s[2 * N + v] = f[8];
                    s[3 * N + v] = 0.5 * (f[1] + f[3]);
                    s[4 * N + v] = 0.5 * (f[2] + f[6]);
                    s[5 * N + v] = 0.5 * (f[5] + f[7]);
                }
            }
            cudaMemcpy(h->d_epsp, s.data(), sizeof(double) * S * N, cudaMemcpyHostToDevice);
            dep = h->d_epsp;
        }
        cudaError_t e = h->solver->solve(eps_bar, warm != 0, dep, max_iter, tol);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
        if (h->solver->device_error()) {
            h->solver->clear_error();
            return fail(MGK_DEVICE_TIMEOUT, "device wait timed out in the LS solver");
        }
        e = h->solver->download_eps(eps_inout);
        if (e == cudaSuccess && sig_out) e = h->solver->download_sig(dep, sig_out);
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
        int it = 0;
        double em[9], sm[9];
        h->solver->macro(em, sm, &it);
        if (macro_out) {
            std::memcpy(macro_out, em, sizeof(double) * DD);
            std::memcpy(macro_out + DD, sm, sizeof(double) * DD);
        }
        if (iters_out) *iters_out = it;
        if (it >= max_iter && max_iter > 0 && !(h->solver->host_result().diff < tol)) return MGK_LS_NOT_CONVERGED;
    } catch (const std::exception& e) {
        return from_exception(e);
    }
    return MGK_OK;
}

void mgk_ls_destroy(mgk_ls* h) {
    if (!h) return;
    delete h->solver;
    if (h->d_epsp) cudaFree(h->d_epsp);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

mgk_status mgk_kmc_create(mgk_kmc** out, const mgk_kmc_params* p, const double* E, const double* nu) {
    if (!out || !p || !E || !nu) return fail(MGK_BAD_ARG, "null argument");
    *out = nullptr;
    if (p->barrier_type < 0 || p->barrier_type > 3) return fail(MGK_BAD_ARG, "unknown barrier type");
    mgk_kmc* h = new (std::nothrow) mgk_kmc;
    if (!h) return fail(MGK_OOM, "host allocation failed");
    try {
        h->eng = new mgk::KmcEngine(*p, E, nu);
    } catch (const std::exception& e) {
        delete h;
        return from_exception(e);
    }
    *out = h;
    return MGK_OK;
}

mgk_status mgk_kmc_run(mgk_kmc* h, const mgk_run_params* rp, double* trace, long long trace_cap, long long* trace_rows) {
    if (!h || !rp) return fail(MGK_BAD_ARG, "null argument");
    if (rp->n_targets < 0 || rp->n_targets > 9) return fail(MGK_BAD_ARG, "n_targets out of range");
    const int D = h->eng->D();
    if (rp->comp_i < 0 || rp->comp_i >= D || rp->comp_j < 0 || rp->comp_j >= D) return fail(MGK_BAD_ARG, "bad driving component");
    for (int t = 0; t < rp->n_targets; ++t)
        if (rp->target_i[t] < 0 || rp->target_i[t] >= D || rp->target_j[t] < 0 || rp->target_j[t] >= D)
            return fail(MGK_BAD_ARG, "bad mixed target component");
    mgk_status s = h->eng->run(*rp, trace, trace_cap, trace_rows);
    if (s != MGK_OK && s != MGK_TERMINATED) g_err = h->eng->last_error;
    return s;
}

mgk_status mgk_kmc_elastic_run(mgk_kmc* h) {
    if (!h) return fail(MGK_BAD_ARG, "null argument");
    mgk_status s = h->eng->elastic_run();
    if (s != MGK_OK) g_err = h->eng->last_error;
    return s;
}

mgk_status mgk_kmc_get_field(mgk_kmc* h, int field, double* dst, long long* count) {
    if (!h) return fail(MGK_BAD_ARG, "null argument");
    mgk_status s = h->eng->get_field(field, dst, count);
    if (s != MGK_OK) g_err = h->eng->last_error;
    return s;
}

mgk_status mgk_kmc_get_macro(mgk_kmc* h, double* out, int n) {
    if (!h || !out) return fail(MGK_BAD_ARG, "null argument");
    h->eng->get_macro(out, n);
    return MGK_OK;
}

mgk_status mgk_kmc_set_profiling(mgk_kmc* h, int on) {
    if (!h) return fail(MGK_BAD_ARG, "null argument");
    h->eng->set_profiling(on != 0);
    return MGK_OK;
}

mgk_status mgk_kmc_get_profile(mgk_kmc* h, double* out, double* lat, long long lat_cap) {
    if (!h || !out) return fail(MGK_BAD_ARG, "null argument");
    const mgk::EngineProfile& p = h->eng->profile();
    double v[10] = {p.ls_ms, (double)p.ls_n, (double)p.ls_iters, p.sweep_ms, (double)p.sweep_n, p.select_ms,
                    (double)p.select_n, p.run_ms, (double)p.event_us.size(), 0.0};
    std::memcpy(out, v, sizeof(v));
    if (lat)
        for (long long i = 0; i < lat_cap && i < (long long)p.event_us.size(); ++i) lat[i] = p.event_us[i];
    return MGK_OK;
}

mgk_status mgk_correlated_field(int dim, int nx, int ny, int nz, double mean, double std_dev, double corr, int has_min,
                                double clip_min, int has_max, double clip_max, int seed, double* out) {
    if (!out) return fail(MGK_BAD_ARG, "null output");
    if (dim != 2 && dim != 3) return fail(MGK_BAD_ARG, "dim must be 2 or 3");
    if (nx < 1 || ny < 1 || (dim == 3 && nz < 1)) return fail(MGK_BAD_SHAPE, "bad grid");
    try {
        mgk::correlated_field(dim, nx, ny, nz, mean, std_dev, corr, has_min != 0, clip_min, has_max != 0, clip_max, seed,
                              out);
    } catch (const std::exception& e) {
        return from_exception(e);
    }
    return MGK_OK;
}

mgk_status mgk_le_run(const mgk_le_params* p, const double* E, const double* nu, double* macro_out, int* ls_iters_out) {
    if (!p || !E || !nu) return fail(MGK_BAD_ARG, "null argument");
    if (p->dim != 2 && p->dim != 3) return fail(MGK_BAD_ARG, "dim must be 2 or 3");
    if (p->nx < 1 || p->ny < 1 || (p->dim == 3 && p->nz < 1)) return fail(MGK_BAD_SHAPE, "bad grid");
    if (p->drive_i < 0 || p->drive_i >= p->dim || p->drive_j < 0 || p->drive_j >= p->dim)
        return fail(MGK_BAD_ARG, "bad driving component");
    if (p->n_targets < 0 || p->n_targets > 9) return fail(MGK_BAD_ARG, "n_targets out of range");
    for (int t = 0; t < p->n_targets; ++t)
        if (p->target_i[t] < 0 || p->target_i[t] >= p->dim || p->target_j[t] < 0 || p->target_j[t] >= p->dim)
            return fail(MGK_BAD_ARG, "bad mixed target component");
    if (p->max_iter_macro < 1 || p->max_iter_ls < 1) return fail(MGK_BAD_ARG, "iteration limits must be positive");
    std::string err;
    mgk_status s = mgk::elastic_run(*p, E, nu, macro_out, ls_iters_out, &err);
    if (s != MGK_OK) g_err = err;
    return s;
}

mgk_status mgk_batch_create(mgk_batch** out, int n, const mgk_kmc_params* params, const double* const* E,
                            const double* const* nu) {
    if (!out || !params || !E || !nu || n < 1) return fail(MGK_BAD_ARG, "null argument or empty batch");
    *out = nullptr;
    for (int r = 0; r < n; ++r) {
        if (!E[r] || !nu[r]) return fail(MGK_BAD_ARG, "null field");
        if (params[r].barrier_type < 0 || params[r].barrier_type > 3) return fail(MGK_BAD_ARG, "unknown barrier type");
    }
    mgk_batch* h = new (std::nothrow) mgk_batch;
    if (!h) return fail(MGK_OOM, "host allocation failed");
    try {
        h->b = new mgk::BatchEngine(n, params, E, nu);
    } catch (const std::exception& e) {
        delete h;
        return from_exception(e);
    }
    *out = h;
    return MGK_OK;
}

mgk_status mgk_batch_create_from(mgk_batch** out, int n, mgk_kmc* const* sims) {
    if (!out || !sims || n < 1) return fail(MGK_BAD_ARG, "null argument or empty batch");
    *out = nullptr;
    std::vector<mgk::KmcEngine*> v;
    for (int r = 0; r < n; ++r) {
        if (!sims[r] || !sims[r]->eng) return fail(MGK_BAD_ARG, "null simulation");
        for (mgk::KmcEngine* e : v)
            if (e == sims[r]->eng) return fail(MGK_BAD_ARG, "a simulation appears twice");
        v.push_back(sims[r]->eng);
    }
    mgk_batch* h = new (std::nothrow) mgk_batch;
    if (!h) return fail(MGK_OOM, "host allocation failed");
    try {
        h->b = new mgk::BatchEngine(v);
    } catch (const std::exception& e) {
        delete h;
        return from_exception(e);
    }
    *out = h;
    return MGK_OK;
}

mgk_status mgk_get_device(int* device) {
    if (!device) return fail(MGK_BAD_ARG, "null device pointer");
    cudaError_t e = cudaGetDevice(device);
    if (e != cudaSuccess) return fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    return MGK_OK;
}

mgk_status mgk_set_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return fail(MGK_BAD_ARG, "no such device");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    return MGK_OK;
}

mgk_status mgk_device_memory(unsigned long long* free_bytes, unsigned long long* total_bytes) {
    size_t f = 0, t = 0;
    cudaError_t e = cudaMemGetInfo(&f, &t);
    if (e != cudaSuccess) return fail(MGK_CUDA_ERROR, cudaGetErrorString(e));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return MGK_OK;
}

mgk_status mgk_batch_run(mgk_batch* h, const mgk_run_params* rp, long long max_events, double* elapsed_ms) {
    if (!h || !rp) return fail(MGK_BAD_ARG, "null argument");
    for (int r = 0; r < h->b->size(); ++r) {
        const int D = h->b->replica(r)->D();
        const mgk_run_params& p = rp[r];
        if (p.n_targets < 0 || p.n_targets > 9) return fail(MGK_BAD_ARG, "n_targets out of range");
        if (p.comp_i < 0 || p.comp_i >= D || p.comp_j < 0 || p.comp_j >= D) return fail(MGK_BAD_ARG, "bad driving component");
        for (int t = 0; t < p.n_targets; ++t)
            if (p.target_i[t] < 0 || p.target_i[t] >= D || p.target_j[t] < 0 || p.target_j[t] >= D)
                return fail(MGK_BAD_ARG, "bad mixed target component");
    }
    mgk_status s = h->b->run(rp, max_events, elapsed_ms);
    if (s != MGK_OK) g_err = h->b->last_error;
    return s;
}

mgk_status mgk_batch_stats(mgk_batch* h, int replica, double* out, int* sel, long long sel_cap, long long* sel_len) {
    if (!h || !out || replica < 0 || replica >= h->b->size()) return fail(MGK_BAD_ARG, "bad argument");
    const mgk::BatchStats& b = h->b->stats(replica);
    double v[19] = {(double)b.events, (double)b.cascades, (double)b.cascade_flips, (double)b.ls_solves, (double)b.ls_iters,
                    (double)b.elastic_steps, (double)b.fallbacks, b.min_margin, (double)b.terminated, (double)b.ncta,
                    b.phase_ms[0], b.phase_ms[1], b.phase_ms[2], b.phase_ms[3], b.phase_ms[4], b.phase_ms[5],
                    (double)b.sweeps, (double)b.h2d_bytes, (double)b.d2h_bytes};
    std::memcpy(out, v, sizeof(v));
    if (sel)
        for (long long i = 0; i < sel_cap && i < (long long)b.sel.size(); ++i) sel[i] = b.sel[i];
    if (sel_len) *sel_len = (long long)b.sel.size();
    return MGK_OK;
}

mgk_status mgk_batch_get_field(mgk_batch* h, int replica, int field, double* dst, long long* count) {
    if (!h || replica < 0 || replica >= h->b->size()) return fail(MGK_BAD_ARG, "bad argument");
    mgk::KmcEngine* e = h->b->replica(replica);
    mgk_status s = e->get_field(field, dst, count);
    if (s != MGK_OK) g_err = e->last_error;
    return s;
}

mgk_status mgk_batch_get_macro(mgk_batch* h, int replica, double* out, int n) {
    if (!h || !out || replica < 0 || replica >= h->b->size()) return fail(MGK_BAD_ARG, "bad argument");
    h->b->replica(replica)->get_macro(out, n);
    return MGK_OK;
}

mgk_status mgk_batch_event_times(mgk_batch* h, int replica, double* us, long long cap, long long* len) {
    if (!h || replica < 0 || replica >= h->b->size()) return fail(MGK_BAD_ARG, "bad argument");
    const mgk::BatchStats& b = h->b->stats(replica);
    if (us)
        for (long long i = 0; i < cap && i < (long long)b.event_us.size(); ++i) us[i] = b.event_us[i];
    if (len) *len = (long long)b.event_us.size();
    return MGK_OK;
}

mgk_status mgk_set_batch_plan(int objective) {
    if (objective < 0 || objective > 1) return fail(MGK_BAD_ARG, "batch plan: 0 throughput, 1 balanced");
    mgk::set_batch_plan_objective(objective);
    return MGK_OK;
}

mgk_status mgk_batch_set_time_limit(mgk_batch* h, double seconds) {
    if (!h || !(seconds > 0.0) || seconds > 3600.0) return fail(MGK_BAD_ARG, "time limit outside (0, 3600] s");
    h->b->set_time_limit(seconds);
    return MGK_OK;
}

void mgk_batch_destroy(mgk_batch* h) {
    if (!h) return;
    delete h->b;
    delete h;
}

void mgk_kmc_destroy(mgk_kmc* h) {
    if (!h) return;
    delete h->eng;
    delete h;
}

}  // extern "C"
