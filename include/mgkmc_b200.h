/*
 * mgkmc_b200.h -- C ABI of the B200 STZ-KMC / Lippmann-Schwinger library
 * (libmgkmc_b200.so).  Plain pointers and sizes only.
 *
 * The reference (mgkmc_cpp) is a header-only C++ program with no ABI; each
 * entry point below names the reference interface it replaces.  Tensors cross
 * the boundary as row-major D x D blocks per voxel (D = 2 or 3), voxels in the
 * reference's order (x slowest, then y, then z), exactly the element order of
 * the reference's std::vector<Eigen::Matrix{2,3}d> members read with (i, j).
 * Device memory is owned by the handles.  Calls are synchronous; a handle is
 * used by one host thread at a time (the reference objects are not re-entrant
 * either).
 */
#ifndef MGKMC_B200_H
#define MGKMC_B200_H

#if defined(__GNUC__)
#define MGK_API __attribute__((visibility("default")))
#else
#define MGK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MGK_OK = 0,
    MGK_LS_NOT_CONVERGED = 1, /* reached max_iter (the reference stops silently) */
    MGK_BAD_SHAPE = 2,        /* grid / field sizes inconsistent */
    MGK_OOM = 3,              /* device allocation failed */
    MGK_DEVICE_TIMEOUT = 4,   /* a bounded device wait gave up */
    MGK_CUDA_ERROR = 5,
    MGK_BAD_ARG = 6,
    MGK_UNSUPPORTED = 7,      /* option not built (e.g. fast patching in the batched form) */
    MGK_TERMINATED = 8,       /* KMC instability sequence limit (kmc_solver.hpp:925-929) */
    MGK_TIME_LIMIT = 9        /* a batched run reached its wall-time limit (mgk_batch_set_time_limit) */
} mgk_status;

/* Text of the last error on this thread. */
MGK_API const char* mgk_last_error(void);
MGK_API int mgk_version(void);
MGK_API int mgk_device_count(void);
/* Free and total memory of the current device, in bytes (admission control of
 * a request loop). */
MGK_API mgk_status mgk_device_memory(unsigned long long* free_bytes, unsigned long long* total_bytes);
/* The calling thread's current CUDA device (every handle's device state is
 * created there), and setting it: a host thread that builds simulations for
 * another thread's GPU first adopts that thread's device.  No counterpart in
 * the reference (single-GPU, single-threaded). */
MGK_API mgk_status mgk_get_device(int* device);
MGK_API mgk_status mgk_set_device(int device);

/* ---------------------------------------------------------------- LS solver
 * Replaces spectral_solver_2d (linear_elastic_solver.hpp:146-160) and
 * spectral_solver_3d (:431-444) together with the Green-operator setup that
 * callers do before them (green_operator_2d/3d, :70-119 / :344-396; the
 * operator is evaluated on the fly, so there is no Gamma argument).
 * mgk_ls_create: dim 2 or 3; nz ignored for dim 2; plane_stress selects
 * compute_lame_2d's plane-stress branch (dim 2 only); E, nu: N host values.
 * Axis lengths must factor into 2, 3, 5 and 7 (MGK_BAD_SHAPE otherwise). */
typedef struct mgk_ls mgk_ls;
MGK_API mgk_status mgk_ls_create(mgk_ls** out, int dim, int nx, int ny, int nz, int plane_stress, double pixel, const double* E,
                         const double* nu);
/* One solve.  eps_bar: D*D prescribed mean strain.  eps_plastic: N*D*D or NULL.
 * eps_inout: N*D*D; read as the warm start when warm != 0 (the reference's
 * eps.size() == N branch, :181-191), written with the solution.  sig_out:
 * N*D*D or NULL.  macro_out: 2*D*D (eps_macro then sig_macro) or NULL.
 * iters_out: iterations run or NULL.  Returns MGK_LS_NOT_CONVERGED when the
 * loop hit max_iter (fields are still written, like the reference). */
MGK_API mgk_status mgk_ls_solve(mgk_ls* h, const double* eps_bar, const double* eps_plastic, double* eps_inout, int warm,
                        double* sig_out, double* macro_out, int max_iter, double tol, int* iters_out);
/* Precision of later solves (no counterpart in the reference, which is FP64):
 * 0 FP64 (default); 1 FP32-refined -- FP32 spectrum, FFTs and Green operator
 * (real-space strain, polarisation, norms and macro sums stay FP64) until the
 * relative change is below max(tol, 1e-6), then FP64 iterations from that
 * field to tol; each phase is capped at max_iter and iters_out reports their
 * sum. */
MGK_API mgk_status mgk_ls_set_precision(mgk_ls* h, int precision);
/* Device time (ms, CUDA events on the solver's stream) of the last solve's
 * kernel launches, without its host copies. */
MGK_API mgk_status mgk_ls_last_solve_ms(mgk_ls* h, double* ms);
/* No counterpart in the reference.  The pass plan the handle's solves run
 * (chosen by timing candidates when the handle was created, unless the
 * environment sets MGK_LS_AUTOTUNE=0): out4 = {rows per row chunk, columns
 * per strided tile, FFT path (0 warp-owned lines, 1 CTA-wide lines), CTAs}. */
MGK_API mgk_status mgk_ls_plan(mgk_ls* h, int* out4);
/* No counterpart in the reference (which has no device waits).  Every
 * barrier wait inside the solver's persistent launch is bounded by device
 * time; this sets the bound (seconds; 0 restores the 120 s default).  A wait
 * that runs out makes every CTA of the launch return, and mgk_ls_solve then
 * returns MGK_DEVICE_TIMEOUT with the handle still usable. */
MGK_API mgk_status mgk_ls_set_wait_limit(mgk_ls* h, double seconds);
/* Fault injection for failure-detection tests, no counterpart in the
 * reference: cta >= 0 makes that CTA of the next solves leave before its first
 * barrier (as if it had died), so the others' bounded waits run out; -1 turns
 * it off.  The kernel never traps and never waits without a bound. */
MGK_API mgk_status mgk_ls_inject_absent_cta(mgk_ls* h, int cta);
MGK_API void mgk_ls_destroy(mgk_ls* h);

/* ---------------------------------------------------------------- LS solve without allocating
 * No counterpart in the reference.  One LS solve like mgk_ls_solve, for
 * callers that may not allocate device memory: a host application that has
 * reserved the GPU's memory for its own pool (another cudaMalloc would fail or
 * fragment it), or a loop that cannot pay for cudaMalloc/cudaFree, which
 * synchronise the whole device.  The caller passes DEVICE buffers:
 * E_dev, nu_dev (N values), eps_plastic_dev (N*D*D or NULL), eps_dev (N*D*D,
 * read as the warm start when warm != 0, written with the solution) and
 * sig_dev (N*D*D or NULL); eps_bar (D*D), macro_out (2*D*D or NULL) and
 * iters_out are host pointers; stream is a cudaStream_t (NULL: the legacy
 * default stream).  The call returns after the stream has finished the solve.
 * Nothing is allocated: every intermediate lives in one static device array of
 * MGK_NOALLOC_SCRATCH_BYTES (16 MiB), which every GPU that loads the library
 * holds until the process exits; grids whose intermediates exceed it are
 * refused with MGK_BAD_SHAPE.  The intermediates take about 88 bytes per voxel
 * in 2D and 170 in 3D with a plastic strain (64 and 112 without), so the limit
 * is about 190k voxels in 2D and 98k in 3D: 432x432 fits and 448x432 does not
 * (2D with a plastic strain); 45^3 fits and 48^3 does not (3D).  Every call
 * looks up the array's device address on the current device (the first one
 * may load the library's GPU code), so make the first call before any stream
 * capture.  All calls share the one array, which
 * keeps the previous call's contents (each call resets what must start at
 * zero): calls that overlap on the GPU, from several streams or threads, race
 * and must be serialised by the caller.  mgk_noalloc_last_error() describes
 * the last failure of this entry point on the calling thread. */
#define MGK_NOALLOC_SCRATCH_BYTES (16u << 20)
MGK_API mgk_status mgk_ls_solve_noalloc(int dim, int nx, int ny, int nz, int plane_stress, double pixel, const double* E_dev,
                                        const double* nu_dev, const double* eps_bar, const double* eps_plastic_dev,
                                        double* eps_dev, int warm, double* sig_dev, double* macro_out, int max_iter, double tol,
                                        int* iters_out, void* stream);
MGK_API const char* mgk_noalloc_last_error(void);

/* ---------------------------------------------------------------- KMC
 * Replaces the KmcSimulation2D constructor (kmc_solver.hpp:165-182) and the
 * KmcSimulation3D constructor (:1142-1158): the same parameters, in one struct. */
typedef struct {
    int dim, nx, ny, nz, M;
    int plane_stress;         /* 2D: plane_mode == "plane_stress" */
    int seed;
    double gamma0, pixel;
    /* BarrierGenerator (kmc_solver.hpp:24-33): type 0 gaussian, 1 rayleigh,
     * 2 modified_rayleigh, 3 modified_rayleigh_with_exponential */
    int barrier_type;
    double bar_mean, bar_std, bar_min_cutoff, bar_max_cutoff, bar_loc, bar_scale, bar_epsilon, bar_ratio;
    int directional;          /* softening_scheme == "directional" */
    double softening_cap, jp, jt, neighbor_fraction, q_act_temp;
    double temperature, strain_rate, stability_threshold, nu0;
    int instability_kmc;      /* instability_mode == "kmc" (else "cascade") */
    int scale_rate_by_volume, redraw_directions, redraw_barriers, use_3d_barriers;
    int fast_patching, patch_radius, sync_interval; /* kmc_solver.hpp:276-332, 866-913: stencil stress updates,
                                                        a full LS solve every sync_interval flips (plain form only) */
    double ls_tol;            /* elastic_run tolerance, reference 1e-6 (:337) */
    int ls_max_iter;          /* reference 200 */
    /* Extensions with no counterpart in the reference (0, 0: the reference's
     * behaviour).  catalog_type: 0 the reference's random modes; 1 M shears in
     * the x-y plane with slip directions evenly spaced in [0, pi) (magnitude
     * gamma0, never redrawn); 2 (3D only) M plane normals on a Fibonacci
     * lattice of the upper hemisphere, each sheared by gamma0 along its
     * largest resolved shear stress, recomputed from the local stress where it
     * is used (no per-mode catalog is stored).  barrier_per_voxel: one barrier
     * per voxel shared by its M modes (drawn before the voxel's modes; redrawn
     * as one value after a flip). */
    int catalog_type;
    int barrier_per_voxel;
    /* No counterpart in the reference: arithmetic of the LS re-solves
     * (elastic_run), 0 FP64 (the reference's), 1 FP32-refined (FP32 spectrum,
     * FFTs and Green operator to a relative change of max(ls_tol, 1e-6), then
     * FP64 iterations from that field to ls_tol), in both the plain and the
     * batched form. */
    int ls_precision;
} mgk_kmc_params;

/* run_simulation arguments (kmc_solver.hpp:721-729) plus a thermal-event cap. */
typedef struct {
    int n_global_steps;
    double step_size;
    int comp_i, comp_j;       /* driving component */
    int n_targets;            /* mixed stress targets (Pa), sorted by (i, j) */
    int target_i[9], target_j[9];
    double target_v[9];
    double mixed_tol;         /* Pa */
    int mixed_max_iter;
    double max_kmc_steps_pct;
    long long max_events;     /* stop after this many thermal events; <= 0: no cap */
    const char* output_dir;   /* NULL: no files */
    const char* summary_filename;
    int enable_summary_log, enable_global_log, enable_console;
    const char* vtk_interval; /* "none" | "last" | "current" | "<int>" */
    int vtk_elastic_only;
    long long max_cascade_batches; /* <= 0: the reference's limit, N batches (kmc_solver.hpp:467, 556) */
} mgk_run_params;

typedef struct mgk_kmc mgk_kmc;
MGK_API mgk_status mgk_kmc_create(mgk_kmc** out, const mgk_kmc_params* p, const double* E, const double* nu);
/* run_simulation.  trace (optional, trace_cap rows of 6 + 2*D*D doubles):
 * [kind, a, b, total_rate, t_wait, time, eps_macro(D*D), sig_macro(D*D)],
 * kind 0 thermal flip (a = flat mode index, b = is_instab), 1 cascade
 * (a = batches, b = flips), 2 interval end without event (a = u1),
 * 3 elastic step done (a = mixed-BC solves, b = elastic steps). */
MGK_API mgk_status mgk_kmc_run(mgk_kmc* h, const mgk_run_params* rp, double* trace, long long trace_cap, long long* trace_rows);
/* elastic_run (kmc_solver.hpp:334-339 / :1333-1338). */
MGK_API mgk_status mgk_kmc_elastic_run(mgk_kmc* h);
/* Public members of the reference object: 0 eps_field, 1 sig_field,
 * 2 eps_plastic (N*D*D), 3 soft_prop (N*2), 4 last_event_time (N), 5 Q,
 * 6 Q0 (N*M), 7 catalog (N*M*D*D), 8 prev_strain_dir (N*D*D), 9 E_field,
 * 10 nu_field (N).  Returns the element count in *count when dst is NULL. */
MGK_API mgk_status mgk_kmc_get_field(mgk_kmc* h, int field, double* dst, long long* count);
/* eps_macro (D*D), sig_macro (D*D), time, then counters: thermal events,
 * cascades, LS solves, LS iterations, elastic steps, selection margin min,
 * host synchronisations, kernel launches. */
MGK_API mgk_status mgk_kmc_get_macro(mgk_kmc* h, double* out, int n);
MGK_API void mgk_kmc_destroy(mgk_kmc* h);

/* ---------------------------------------------------------------- generated material fields
 * generate_correlated_field_cpp (material_generator.hpp:130-258, main.cpp's
 * "generated" material mode) on the GPU: N = nx*ny(*nz) values into out (host)
 * -- Box-Muller normals from std::mt19937(seed), an orthonormal FFT, the
 * Gaussian filter exp(-2 pi^2 corr^2 |f|^2), the inverse FFT, standardisation,
 * then mean + std * g clipped to [clip_min, clip_max] where enabled.  Axis
 * lengths must factor into 2, 3, 5 and 7 (MGK_BAD_SHAPE otherwise). */
MGK_API mgk_status mgk_correlated_field(int dim, int nx, int ny, int nz, double mean, double std_dev, double corr,
                                        int has_min, double clip_min, int has_max, double clip_max, int seed,
                                        double* out);

/* ---------------------------------------------------------------- linear-elastic simulation
 * Replaces main.cpp's simulation_type "linear_elastic" branch
 * (main.cpp:418-869): the macroscopic target (eps_target on the driving
 * component drive_i, drive_j; zero strain on the other components; the mixed
 * stress targets, in Pa, on their components) is applied proportionally in
 * n_steps = round(eps_target / step_size) steps, s = 0 .. n_steps; each step
 * runs up to max_iter_macro (the reference: 20) warm-started LS solves
 * (max_iter_ls 200, tol_ls 1e-6 there), correcting the stress-controlled
 * strain components by (err - nu_avg tr(err) I) / E_avg until every stress
 * error is below mixed_tol (Pa).  Writes the reference's summary and global
 * logs and VTU files into output_dir (NULL: no files).  macro_out (nullable)
 * gets (n_steps + 1) x 2 x D x D values: per step eps_macro then sig_macro,
 * row-major; ls_iters_out (nullable) the LS iterations of the whole run. */
typedef struct {
    int dim, nx, ny, nz, plane_stress;
    double pixel;
    double eps_target, step_size;
    int drive_i, drive_j;
    int n_targets;
    int target_i[9], target_j[9];
    double target_v[9];
    double mixed_tol;
    int max_iter_macro, max_iter_ls;
    double tol_ls;
    const char* output_dir;
    const char* summary_filename;
    int enable_summary_log, enable_global_log, enable_console;
    const char* vtk_interval; /* "none", "last", "current" or a step interval */
} mgk_le_params;
MGK_API mgk_status mgk_le_run(const mgk_le_params* p, const double* E, const double* nu, double* macro_out,
                              int* ls_iters_out);

/* ---------------------------------------------------------------- batched, device-resident KMC
 * No counterpart in the reference (single replica, single thread there).  n
 * independent simulations, each constructed exactly like mgk_kmc_create, run
 * together by one persistent GPU kernel: every replica's run_simulation
 * control flow (sweep, selection, flip, LS solve, cascades, mixed-BC loop)
 * executes on the device with no host round trip per event, each replica on
 * its own group of CTAs.  The random stream is the reference's: each replica's
 * std::mt19937 state continues on the device with the same distributions.
 * mgk_batch_run advances every replica by up to max_events thermal events
 * (<= 0: until its n_global_steps elastic steps are done); rp holds n entries
 * (log and VTU fields are ignored: device-resident runs write no files);
 * elapsed_ms gets the kernel's CUDA-event time.  mgk_batch_stats fills
 * out[0..18] = {events, cascades, cascade flips, LS solves, LS iterations,
 * elastic steps, selection fallbacks, smallest selection margin, terminated
 * (1 instability sequence limit, 2 time limit), CTAs of the replica, then the
 * replica's device time in ms spent in: sweeps, decisions (selection, flip,
 * redraw), event LS solves, cascade collection and flips, cascade LS solves,
 * interval ends (mixed-BC loop), then the number of sweeps and the bytes the
 * run call copied host-to-device and device-to-host for the replica} and
 * copies the flat mode index of each thermal event of the last run into sel
 * (up to sel_cap; *sel_len gets the count).  Time limit (default 60 s, set
 * with mgk_batch_set_time_limit): a replica whose run call has lasted longer
 * keeps working until every replica of the batch has (or has finished), then
 * every replica stops at its next decision -- the launch waits for its
 * slowest replica's decision in any case, so the others use that time -- and
 * the call returns MGK_TIME_LIMIT; the state stays consistent and a later
 * run continues from it. */
typedef struct mgk_batch mgk_batch;
MGK_API mgk_status mgk_batch_create(mgk_batch** out, int n, const mgk_kmc_params* params, const double* const* E,
                                    const double* const* nu);
/* A batch over n existing simulations (mgk_kmc_create), not owned: they
 * must outlive the batch, and mgk_kmc_get_field / get_macro read them after
 * a run.  A simulation may join different batches over its life (one running
 * batch at a time); its interval clock and random stream carry over, which is
 * how a request loop admits and retires jobs between launches. */
MGK_API mgk_status mgk_batch_create_from(mgk_batch** out, int n, mgk_kmc* const* sims);
/* rp[r].max_events > 0 sets replica r's own event budget for the call. */
MGK_API mgk_status mgk_batch_run(mgk_batch* h, const mgk_run_params* rp, long long max_events, double* elapsed_ms);
MGK_API mgk_status mgk_batch_stats(mgk_batch* h, int replica, double* out, int* sel, long long sel_cap, long long* sel_len);
MGK_API mgk_status mgk_batch_get_field(mgk_batch* h, int replica, int field, double* dst, long long* count);
MGK_API mgk_status mgk_batch_get_macro(mgk_batch* h, int replica, double* out, int n);
/* Per-step latency of the last run: for each logged thermal event of the
 * replica (up to 65536), the device time in microseconds since its previous
 * event (the first: since the run's first decision).  Copies up to cap values
 * into us; *len gets the count.  No counterpart in the reference. */
MGK_API mgk_status mgk_batch_event_times(mgk_batch* h, int replica, double* us, long long cap, long long* len);
MGK_API mgk_status mgk_batch_set_time_limit(mgk_batch* h, double seconds);
/* No counterpart in the reference.  How batches created from now on spread
 * their CTAs over the replicas: 0 (default) throughput -- each CTA goes to the
 * replica whose modelled event rate it raises most, so small latency-bound
 * grids get most; 1 balanced -- each CTA goes to the replica furthest below
 * the rate it would have on the whole GPU, so that mixed sizes advance at
 * similar fractions of their single-replica speed (shorter makespan). */
MGK_API mgk_status mgk_set_batch_plan(int objective);
MGK_API void mgk_batch_destroy(mgk_batch* h);

/* Measurement hooks (no counterpart in the reference, which only logs wall
 * time).  mgk_kmc_set_profiling(h, 1) clears the profile and records CUDA
 * events around every LS solve, sweep and selection on the engine's stream.
 * mgk_kmc_get_profile fills out[0..9] = {ls_ms, ls_launches, ls_iterations,
 * sweep_ms, sweeps, select_ms, selects, run_ms, events_timed, 0} and copies up
 * to lat_cap per-event host latencies (microseconds) into lat. */
MGK_API mgk_status mgk_kmc_set_profiling(mgk_kmc* h, int on);
MGK_API mgk_status mgk_kmc_get_profile(mgk_kmc* h, double* out, double* lat, long long lat_cap);

#ifdef __cplusplus
}
#endif
#endif /* MGKMC_B200_H */
