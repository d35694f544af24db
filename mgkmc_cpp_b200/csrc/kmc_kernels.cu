// STZ kinetic Monte Carlo kernels.
//
// sweep       update_barriers + rate build (kmc_solver.hpp:341-410, 783-806 /
//             :1340-1411, 1796-1818): Q per mode, its rate, and per-block
//             double-double rate sums, unstable counts and last included mode;
//             the last block folds the block results into the status word.
// select_flip total/CDF selection (:808-838 / :1820-1852) and apply_flip_soa_*
//             with the catalog / barrier redraw (:423-462, 839-864 /
//             :1424-1471, 1854-1875).  Selection: first included mode whose
//             rate prefix reaches the target, with prefixes accumulated in
//             double-double (the reference adds left to right in FP64; the two
//             agree except when the target falls within ~n*2^-53 of a prefix
//             boundary, reported in status.margin).
// cascade     find_unstable_indices + sort + one flip per voxel (:412-421,
//             464-564 / :1413-1422, 1473-1590): the first entry per voxel of the
//             Q-sorted unstable list is that voxel's lowest-Q unstable mode, and
//             the flips run in the order of those Q values.
#include <algorithm>
#include "kmc_kernels.cuh"
#include "kmc_device.cuh"

namespace mgk {

namespace {

using namespace kmcdev;
constexpr int kSweepThreads = 256;

template <int D, int C>
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(KmcDevState s, KmcPhys p, double time, dd* blk, int* blk_unst,
                                                              int* blk_last, int items, KmcStatus* st) {
    __shared__ dd sd[32];
    __shared__ int si[32], sl[32];
    __shared__ int s_last_block;
    const long base = (long)blockIdx.x * blockDim.x * items;
    dd acc = {0.0, 0.0};
    int unst = 0, last = -1;
#pragma unroll 4
    for (int j = 0; j < items; ++j) {
        const long i = base + (long)j * blockDim.x + threadIdx.x;
        if (i < s.NM) {
            const int v = voxel_of(i, s.NM, s.M);
            const double q = mode_Q<D, C>(s, p, v, i, time);
            s.Q[i] = q;
            bool inc;
            const double r = rate_of(p, q, &inc);
            if (inc) {
                last = (int)i;
                acc = dd_add_d(acc, r);
            }
            if (q < p.threshold) ++unst;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    acc = warp_dd_sum(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unst += __shfl_down_sync(0xffffffffu, unst, o);
        last = max(last, __shfl_down_sync(0xffffffffu, last, o));
    }
    if (lane == 0) {
        sd[wid] = acc;
        si[wid] = unst;
        sl[wid] = last;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        dd a = lane < nw ? sd[lane] : dd{0.0, 0.0};
        int u = lane < nw ? si[lane] : 0;
        int l = lane < nw ? sl[lane] : -1;
        a = warp_dd_sum(a);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            u += __shfl_down_sync(0xffffffffu, u, o);
            l = max(l, __shfl_down_sync(0xffffffffu, l, o));
        }
        if (lane == 0) {
            blk[blockIdx.x] = a;
            blk_unst[blockIdx.x] = u;
            blk_last[blockIdx.x] = l;
            __threadfence();
            const unsigned t = atomicAdd(&st->ticket, 1u);
            s_last_block = (t == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!s_last_block) return;
    // last block: fold all block results in a fixed order
    dd tot = {0.0, 0.0};
    int nu = 0, lst = -1;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        dd x;
        x.hi = __ldcg(&blk[b].hi);
        x.lo = __ldcg(&blk[b].lo);
        tot = dd_add(tot, x);
        nu += __ldcg(&blk_unst[b]);
        lst = max(lst, __ldcg(&blk_last[b]));
    }
    tot = warp_dd_sum(tot);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nu += __shfl_down_sync(0xffffffffu, nu, o);
        lst = max(lst, __shfl_down_sync(0xffffffffu, lst, o));
    }
    __syncthreads();
    if (lane == 0) {
        sd[wid] = tot;
        si[wid] = nu;
        sl[wid] = lst;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dd a = {0.0, 0.0};
        int u = 0, l = -1;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a = dd_add(a, sd[w]);
            u += si[w];
            l = max(l, sl[w]);
        }
        st->total_hi = a.hi;
        st->total_lo = a.lo;
        st->n_unstable = u;
        st->last_included = l;
        st->ticket = 0;
    }
}

template <int D, int C>
__global__ void __launch_bounds__(512) select_flip_kernel(KmcDevState s, KmcPhys p, const dd* blk, const int* blk_last, int nblk,
                                                          int items, const double* target_dev, double time, const double* draws,
                                                          int redraw_dir, int redraw_bar, KmcStatus* st) {
    __shared__ dd sh[32];
    __shared__ int s_blk, s_sel;
    __shared__ dd s_before;
    __shared__ double s_margin;
    const double target = *target_dev;
    if (threadIdx.x == 0) {
        s_blk = 0x7fffffff;
        s_sel = 0x7fffffff;
    }
    __syncthreads();
    // 1. block containing the crossing
    const int seg = (nblk + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * seg, b1 = min(nblk, b0 + seg);
    dd mine = {0.0, 0.0};
    for (int b = b0; b < b1; ++b) mine = dd_add(mine, blk[b]);
    dd tot;
    dd run = block_excl_scan(mine, sh, &tot);
    int my_blk = -1;
    for (int b = b0; b < b1; ++b) {
        dd nx = dd_add(run, blk[b]);
        if (dd_ge(nx, target)) {
            my_blk = b;
            atomicMin(&s_blk, b);
            break;
        }
        run = nx;
    }
    __syncthreads();
    const int cb = s_blk;
    if (cb != 0x7fffffff) {
        // prefix before block cb: the exclusive prefix of the thread that found it
        if (my_blk == cb) s_before = run;
        __syncthreads();
        // 2. inside block cb: contiguous runs per thread, mode order
        const long m0 = (long)cb * kSweepThreads * items;
        const long m1 = min(s.NM, m0 + (long)kSweepThreads * items);
        const long len = m1 - m0;
        const long per = (len + blockDim.x - 1) / blockDim.x;
        const long r0 = m0 + threadIdx.x * per, r1 = min(m1, r0 + per);
        dd ms = {0.0, 0.0};
        for (long i = r0; i < r1; ++i) {
            bool inc;
            const double r = rate_of(p, s.Q[i], &inc);
            if (inc) ms = dd_add_d(ms, r);
        }
        dd ex = block_excl_scan(ms, sh, nullptr);
        dd pr = dd_add(s_before, ex);
        long cand = -1;
        double cmargin = 0.0;
        for (long i = r0; i < r1; ++i) {
            bool inc;
            const double r = rate_of(p, s.Q[i], &inc);
            if (!inc) continue;
            dd nx = dd_add_d(pr, r);
            if (dd_ge(nx, target)) {
                cand = i;
                const double below = target - (pr.hi + pr.lo), above = (nx.hi + nx.lo) - target;
                cmargin = fmin(below, above) / fmax(target, 1e-300);
                atomicMin(&s_sel, (int)i);
                break;
            }
            pr = nx;
        }
        __syncthreads();
        if (cand >= 0 && cand == s_sel) s_margin = cmargin;
        __syncthreads();
    }
    if (threadIdx.x == 0 && s_sel == 0x7fffffff) {
        int l = -1;
        if (cb != 0x7fffffff) {
            // the block sum said the crossing is in block cb but the in-block
            // prefix stopped short by rounding: it lies at the next included mode
            for (long i = min(s.NM, (long)(cb + 1) * kSweepThreads * items); i < s.NM; ++i) {
                bool inc;
                rate_of(p, s.Q[i], &inc);
                if (inc) {
                    l = (int)i;
                    break;
                }
            }
        }
        if (l < 0) {
            // no crossing at all (rounding at the very end of the list): the
            // reference keeps its default, the last rate entry (kmc_solver.hpp:819)
            for (int b = 0; b < nblk; ++b) l = max(l, blk_last[b]);
        }
        s_sel = l;
        s_margin = 0.0;
        if (l < 0) atomicOr(&st->err, MGK_DERR_SELECT);
    }
    __syncthreads();
    const int k = s_sel;
    if (k < 0) return;
    if (threadIdx.x == 0) {
        st->selected = k;
        st->is_instab = s.Q[k] <= p.threshold ? 1 : 0;
        st->margin = s_margin;
        apply_flip<D, C>(s, p, k, time, s.flipcat);
    }
    __syncthreads();
    redraw<C>(s, k, draws, redraw_dir, redraw_bar, threadIdx.x, blockDim.x);
}

template <int D, int C>
__global__ void cascade_collect_kernel(KmcDevState s, KmcPhys p, double* keys, int* modes, KmcStatus* st) {
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < s.N; v += (long)gridDim.x * blockDim.x) {
        double best = 0.0;
        int bm = -1;
        for (int m = 0; m < s.M; ++m) {
            const double q = s.Q[v * s.M + m];
            if (q < p.threshold && (bm < 0 || q < best)) {
                best = q;
                bm = m;
            }
        }
        if (bm >= 0) {
            const int slot = atomicAdd(&st->n_collect, 1);
            keys[slot] = best;
            modes[slot] = (int)(v * s.M + bm);
        }
    }
}

// bitonic sort of (key, mode) pairs, npow2 elements, in shared memory (one CTA)
__global__ void bitonic_smem_kernel(double* keys, int* modes, int n, int npow2) {
    extern __shared__ __align__(16) unsigned char sm[];
    double* k = reinterpret_cast<double*>(sm);
    int* m = reinterpret_cast<int*>(k + npow2);
    for (int i = threadIdx.x; i < npow2; i += blockDim.x) {
        k[i] = i < n ? keys[i] : INFINITY;
        m[i] = i < n ? modes[i] : 0x7fffffff;
    }
    __syncthreads();
    for (int size = 2; size <= npow2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < npow2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const bool sw = up ? key_less(k[j], m[j], k[i], m[i]) : key_less(k[i], m[i], k[j], m[j]);
                    if (sw) {
                        double tk = k[i]; k[i] = k[j]; k[j] = tk;
                        int tm = m[i]; m[i] = m[j]; m[j] = tm;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        keys[i] = k[i];
        modes[i] = m[i];
    }
}

__global__ void bitonic_global_step(double* k, int* m, int npow2, int size, int stride) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= npow2) return;
    const long j = i ^ stride;
    if (j <= i) return;
    const bool up = (i & size) == 0;
    const bool sw = up ? key_less(k[j], m[j], k[i], m[i]) : key_less(k[i], m[i], k[j], m[j]);
    if (sw) {
        double tk = k[i]; k[i] = k[j]; k[j] = tk;
        int tm = m[i]; m[i] = m[j]; m[j] = tm;
    }
}

__global__ void pad_kernel(const double* keys, const int* modes, int n, int npow2, double* k, int* m) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= npow2) return;
    k[i] = i < n ? keys[i] : INFINITY;
    m[i] = i < n ? modes[i] : 0x7fffffff;
}

// Apply the sorted flips; with neighbour softening the order matters and a
// single thread walks the list, else flips of distinct voxels run in parallel.
template <int D, int C>
__global__ void cascade_apply_kernel(KmcDevState s, KmcPhys p, const int* modes, int n, double time, const double* draws,
                                     int redraw_dir, int redraw_bar) {
    const int rec = (redraw_dir == RD_ALL || redraw_bar == RD_ALL) ? s.M : 1;
    if (p.neigh > 0.0) {
        if (blockIdx.x != 0) return;
        for (int f = 0; f < n; ++f) {
            const long k = modes[f];
            if (threadIdx.x == 0) apply_flip<D, C>(s, p, k, time, s.flipcat ? s.flipcat + (long)f * C : nullptr);
            __syncthreads();
            redraw<C>(s, k, draws + (long)f * rec * (C + 1), redraw_dir, redraw_bar, threadIdx.x, blockDim.x);
            __syncthreads();
        }
        return;
    }
    for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < n; f += (long)gridDim.x * blockDim.x) {
        const long k = modes[f];
        apply_flip<D, C>(s, p, k, time, s.flipcat ? s.flipcat + f * C : nullptr);
        redraw<C>(s, k, draws + f * rec * (C + 1), redraw_dir, redraw_bar, 0, 1);
    }
}

template <int D>
__global__ void stress_kernel(KmcDevState s) {
    constexpr int S = D == 2 ? 3 : 6;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < s.N; v += (long)gridDim.x * blockDim.x) {
        double sg[S];
        voxel_stress<D>(s, (int)v, sg);
#pragma unroll
        for (int c = 0; c < S; ++c) s.sig_s[(long)c * s.N + v] = sg[c];
    }
}

// Coefficients of a mode on the stress-kernel bases: 2D {xx = -yy, xy}
// (kmc_solver.hpp:884-885); 3D {diag(1,-1,0), diag(0,1,-1), xy, xz, yz} with
// c0 = C(0,0), c1 = -C(2,2), c2..c4 = C(0,1), C(0,2), C(1,2) (:1895-1899).
template <int D, int C>
MGK_DEV int basis_coef(const double* cat, double* coef) {
    constexpr int S = D == 2 ? 3 : 6;
    double cs[S];
    cat_sym<D, C>(cat, cs);
    if (D == 2) {
        coef[0] = cs[0];
        coef[1] = cs[2];
        return 2;
    }
    coef[0] = cs[0];
    coef[1] = -cs[2];
    coef[2] = cs[3];
    coef[3] = cs[4];
    coef[4] = cs[5];
    return 5;
}

// One thread per voxel: the voxel's own additions in the reference's order
// (predictor; per flip: every stencil offset that lands on the voxel, in
// dx, dy, dz loop order, then the missing mean), with explicit
// round-to-nearest operations so that no multiply-add is contracted.
template <int D, int C>
__global__ void patch_kernel(KmcDevState s, KmcPhys p, const int* modes, int nflips, const double* K, const double* miss,
                             int R, const double* unit, double pred) {
    constexpr int S = D == 2 ? 3 : 6;
    const int nx = p.nx, ny = p.ny, nz = D == 3 ? p.nz : 1;
    const int side = 2 * R + 1, side_z = (D == 3 && nz > 1) ? side : 1;
    const int P = side * side * side_z;
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < s.N; v += (long)gridDim.x * blockDim.x) {
        const int vx = (int)(v / ((long)ny * nz)), vy = (int)((v / nz) % ny), vz = (int)(v % nz);
        double val[S];
#pragma unroll
        for (int c = 0; c < S; ++c) val[c] = s.sig_s[(long)c * s.N + v];
        if (pred != 0.0)
#pragma unroll
            for (int c = 0; c < S; ++c) val[c] = __dadd_rn(val[c], __dmul_rn(unit[c], pred));
        for (int f = 0; f < nflips; ++f) {
            const long k = modes[f];
            const int u = (int)(k / s.M);
            const int x = u / (ny * nz), y = (u / nz) % ny, z = u % nz;
            double coef[5];
            const int nb = basis_coef<D, C>(s.flipcat + (long)f * C, coef);
            // offsets d in [-R, R] with (x + d) mod n == vx, ascending
            const int ddx = ((vx - x) % nx + nx) % nx, ddy = ((vy - y) % ny + ny) % ny, ddz = ((vz - z) % nz + nz) % nz;
            for (int dx = ddx - nx * ((ddx + R) / nx); dx <= R; dx += nx)
                for (int dy = ddy - ny * ((ddy + R) / ny); dy <= R; dy += ny) {
                    const int z0 = side_z > 1 ? ddz - nz * ((ddz + R) / nz) : 0, z1 = side_z > 1 ? R : 0;
                    for (int dz = z0; dz <= z1; dz += (side_z > 1 ? nz : 1)) {
                        const int crop = ((dx + R) * side + (dy + R)) * side_z + (side_z > 1 ? dz + R : 0);
#pragma unroll
                        for (int c = 0; c < S; ++c) {
                            double pv = __dmul_rn(coef[0], K[(long)crop * S + c]);
                            for (int b = 1; b < nb; ++b) pv = __dadd_rn(pv, __dmul_rn(coef[b], K[((long)b * P + crop) * S + c]));
                            val[c] = __dadd_rn(val[c], pv);
                        }
                    }
                }
#pragma unroll
            for (int c = 0; c < S; ++c) {
                double ms = __dmul_rn(coef[0], miss[c]);
                for (int b = 1; b < nb; ++b) ms = __dadd_rn(ms, __dmul_rn(coef[b], miss[b * S + c]));
                val[c] = __dadd_rn(val[c], ms);
            }
        }
#pragma unroll
        for (int c = 0; c < S; ++c) s.sig_s[(long)c * s.N + v] = val[c];
    }
}

}  // namespace

cudaError_t kmc_stress(const KmcDevState& s, cudaStream_t st) {
    const int grid = (int)std::min<long>((s.N + 255) / 256, 148 * 8);
    if (s.D == 2) stress_kernel<2><<<grid, 256, 0, st>>>(s);
    else stress_kernel<3><<<grid, 256, 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t kmc_patch(const KmcDevState& s, const KmcPhys& p, const int* modes, int nflips, const double* K,
                      const double* miss, int R, const double* unit, double pred, cudaStream_t st) {
    const int grid = (int)std::min<long>((s.N + 255) / 256, 148 * 8);
    if (s.D == 2) patch_kernel<2, 2><<<grid, 256, 0, st>>>(s, p, modes, nflips, K, miss, R, unit, pred);
    else if (s.C == 2) patch_kernel<3, 2><<<grid, 256, 0, st>>>(s, p, modes, nflips, K, miss, R, unit, pred);
    else patch_kernel<3, 6><<<grid, 256, 0, st>>>(s, p, modes, nflips, K, miss, R, unit, pred);
    return cudaGetLastError();
}

int kmc_sweep_blocks(long NM, int items) {
    const long per = (long)kSweepThreads * items;
    return (int)((NM + per - 1) / per);
}

#define MGK_DISPATCH(D, C, call)                         \
    do {                                                 \
        if ((D) == 2 && (C) == 2) { call(2, 2); }         \
        else if ((D) == 3 && (C) == 2) { call(3, 2); }    \
        else if ((D) == 3 && (C) == 6) { call(3, 6); }    \
        else return cudaErrorInvalidValue;               \
    } while (0)

cudaError_t kmc_sweep(const KmcDevState& s, const KmcPhys& p, double time, dd* blk, int* blk_unst, int* blk_last, int nblk,
                      int items, KmcStatus* status, cudaStream_t st) {
#define CALL(D_, C_) sweep_kernel<D_, C_><<<nblk, kSweepThreads, 0, st>>>(s, p, time, blk, blk_unst, blk_last, items, status)
    MGK_DISPATCH(s.D, s.C, CALL);
#undef CALL
    return cudaGetLastError();
}

cudaError_t kmc_select_flip(const KmcDevState& s, const KmcPhys& p, const dd* blk, const int* blk_last, int nblk, int items,
                            const double* target_dev, double time, const double* draws, int redraw_dir, int redraw_bar,
                            KmcStatus* status, cudaStream_t st) {
#define CALL(D_, C_)                                                                                                   \
    select_flip_kernel<D_, C_><<<1, 512, 0, st>>>(s, p, blk, blk_last, nblk, items, target_dev, time, draws, redraw_dir, \
                                                  redraw_bar, status)
    MGK_DISPATCH(s.D, s.C, CALL);
#undef CALL
    return cudaGetLastError();
}

cudaError_t kmc_cascade_collect(const KmcDevState& s, const KmcPhys& p, double* keys, int* modes, KmcStatus* status,
                                cudaStream_t st) {
    int nb = (s.N + 255) / 256;
    if (nb > 4096) nb = 4096;
#define CALL(D_, C_) cascade_collect_kernel<D_, C_><<<nb, 256, 0, st>>>(s, p, keys, modes, status)
    MGK_DISPATCH(s.D, s.C, CALL);
#undef CALL
    return cudaGetLastError();
}

cudaError_t kmc_cascade_flip(const KmcDevState& s, const KmcPhys& p, double* keys, int* modes, int n, double* tmp_keys,
                             int* tmp_modes, double time, const double* draws, int redraw_dir, int redraw_bar,
                             KmcStatus* status, cudaStream_t st) {
    (void)status;
    if (n <= 0) return cudaSuccess;
    int npow2 = 1;
    while (npow2 < n) npow2 <<= 1;
    const int* sorted_modes = modes;
    if (npow2 <= 8192) {
        const size_t smem = (size_t)npow2 * (sizeof(double) + sizeof(int));
        if (smem > 48 * 1024) {
            cudaError_t e = ensure_dyn_smem((const void*)bitonic_smem_kernel, smem);
            if (e != cudaSuccess) return e;
        }
        bitonic_smem_kernel<<<1, 1024, smem, st>>>(keys, modes, n, npow2);
    } else {
        const int nb = (npow2 + 255) / 256;
        pad_kernel<<<nb, 256, 0, st>>>(keys, modes, n, npow2, tmp_keys, tmp_modes);
        for (int size = 2; size <= npow2; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1)
                bitonic_global_step<<<nb, 256, 0, st>>>(tmp_keys, tmp_modes, npow2, size, stride);
        sorted_modes = tmp_modes;
    }
    int nb = (n + 127) / 128;
    if (p.neigh > 0.0) nb = 1;
#define CALL(D_, C_) \
    cascade_apply_kernel<D_, C_><<<nb, 128, 0, st>>>(s, p, sorted_modes, n, time, draws, redraw_dir, redraw_bar)
    MGK_DISPATCH(s.D, s.C, CALL);
#undef CALL
    return cudaGetLastError();
}

}  // namespace mgk
