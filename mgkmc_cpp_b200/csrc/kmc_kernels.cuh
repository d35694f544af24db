// Device kernels of the STZ kinetic Monte Carlo step (see kmc_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace mgk {

// Per-voxel / per-mode state on the device.  Catalog modes are stored with
// C = 2 values (gxx, gxy: the deviatoric 2x2 mode [[gxx, gxy], [gxy, -gxx]],
// embedded in the xy block in 3D) or C = 6 symmetric components
// {xx, yy, zz, xy, xz, yz} (random 3D modes).
struct KmcDevState {
    int D, S, C, M, N;
    long NM;
    double* Q0;       // NM
    double* Q;        // NM (written by the sweep)
    double* cat;      // NM * C
    double* epsp_s;   // S * N
    double* soft;     // 2 * N: g_p, g_t
    double* last_t;   // N
    double* prev;     // N * C: catalog entry of the last flip per voxel
    const double* eps_s;  // S * N (owned by the LS solver)
    const double* lam;    // N
    const double* mu;     // N
    // fast patching only (else null): the stress field the sweep reads
    // (kept by stencil updates between LS solves) and, per flip of the last
    // select / cascade batch, the flipped mode's catalog entry before its redraw
    double* sig_s;        // S * N
    double* flipcat;      // N * C
    // stress-dependent catalog (catalog.type fibonacci; else null): M plane
    // normals (x, y, z); every mode is a shear of magnitude gamma0 along the
    // plane's largest resolved shear stress, computed where it is used; cat is
    // then null and prev / flipcat hold C = 6 symmetric components
    const double* normals;
    double gamma0;
};

// How a flip's redraw records (kmc_select_flip, kmc_cascade_flip) replace the
// voxel's modes.  Directions: none, all M modes from M records, or the
// flipped mode from record 0.  Barriers: none, all M from M records, the
// flipped mode from record 0, or one value (record 0) for all M modes (a
// barrier per voxel).  The reference's redraw (kmc_solver.hpp:839-864) is
// (ALL, ALL) with both flags set, (ALL, NONE) / (NONE, ALL) with one, and
// (FLIPPED, FLIPPED) with neither.
enum : int { RD_NONE = 0, RD_ALL = 1, RD_FLIPPED = 2, RD_VOXEL = 3 };

struct KmcPhys {
    double volume;        // pixel^3 (work term)
    double vnu;           // eff_volume * nu0
    double beta;          // 1 / (kB T), +inf at T = 0
    double tau;           // softening decay time, +inf at T = 0
    double softening_cap;
    double jp, jt, neigh;
    double threshold;     // stability threshold
    int directional;      // softening_scheme == "directional"
    int kmc_mode;         // instability_mode == "kmc" (rates for all modes)
    int nx, ny, nz;
};

struct KmcStatus {
    double total_hi, total_lo;  // sum of rates (double-double)
    int n_unstable;             // modes with Q < threshold
    int last_included;          // highest mode index with a rate entry, -1 if none
    int selected;               // last selected mode index
    int is_instab;              // Q[selected] <= threshold
    double margin;              // relative distance of the target to the nearest prefix boundary
    int n_collect;              // cascade: unstable voxels collected
    unsigned err;
    unsigned ticket;            // internal: last-block-done counter
    int pad;
};

// Enqueue helpers (all asynchronous on `st`).
cudaError_t kmc_sweep(const KmcDevState& s, const KmcPhys& p, double time, dd* blk, int* blk_unst, int* blk_last, int nblk,
                      int items, KmcStatus* status, cudaStream_t st);
int kmc_sweep_blocks(long NM, int items);
// Select the first mode whose rate prefix reaches `target` (from the host:
// u2 * total) and apply the flip at simulation time `time` with the redraw
// records in `draws` (M or 1 records of C + 1 values: catalog values then Q0;
// `redraw_dir`, `redraw_bar` are RD_* modes saying which parts replace what).
cudaError_t kmc_select_flip(const KmcDevState& s, const KmcPhys& p, const dd* blk, const int* blk_last, int nblk, int items,
                            const double* target_dev, double time, const double* draws, int redraw_dir, int redraw_bar,
                            KmcStatus* status, cudaStream_t st);
// Cascade: per-voxel most unstable mode -> list (Q, mode), count in status->n_collect.
cudaError_t kmc_cascade_collect(const KmcDevState& s, const KmcPhys& p, double* keys, int* modes, KmcStatus* status,
                                cudaStream_t st);
// Sort the collected list by (Q, mode) and apply the flips in that order with
// draw block k for the k-th flip.
cudaError_t kmc_cascade_flip(const KmcDevState& s, const KmcPhys& p, double* keys, int* modes, int n, double* tmp_keys,
                             int* tmp_modes, double time, const double* draws, int redraw_dir, int redraw_bar,
                             KmcStatus* status, cudaStream_t st);

// Fast patching (kmc_solver.hpp:276-332, 866-913, 525-546, 942-947):
// sig_s = stress of the current LS strain field (after every LS solve).
cudaError_t kmc_stress(const KmcDevState& s, cudaStream_t st);
// sig_s += unit * pred (when pred != 0), then for every flip f in order (flat
// mode modes[f], pre-redraw catalog flipcat[f]): the stencil of the stress
// kernels K (nb bases, side^D... entries of S values each) around the flipped
// voxel weighted by the mode's basis coefficients, then the missing mean.
cudaError_t kmc_patch(const KmcDevState& s, const KmcPhys& p, const int* modes, int nflips, const double* K,
                      const double* miss, int R, const double* unit, double pred, cudaStream_t st);

}  // namespace mgk
