// Device-resident, batched KMC: many replicas advance inside one persistent
// cooperative kernel, each replica on its own group of CTAs with its own
// bounded group barrier, and no host round trip per event.
//
// Per replica the kernel runs the control flow of run_simulation
// (kmc_solver.hpp:721-1037 / :1735-2062) on the device:
//   sweep (update_barriers + rates, every CTA of the group over its chunk of
//   modes) -> decision on the group's first CTA (total rate, u1 -> t_wait,
//   event / end of interval / cascade; u2 -> target; selection over the chunk
//   sums and then inside one chunk; flip with apply_flip_soa_* and the catalog
//   and barrier redraw) -> warm-started LS solve by the whole group ->
//   repeat; at the end of an interval the mixed-BC loop (:955-987); unstable
//   modes run the cascade batches (:464-564).
// Random numbers: the replica's std::mt19937 state after its host-side
// initial draws is handed to the device and continued by one thread with the
// reference's distributions (mt_device.cuh), so the draws follow the
// reference's stream; only device log/exp may differ from glibc by an ulp.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <cstring>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "batch.cuh"
#include "kmc_device.cuh"
#include "ls_device.cuh"
#include "mt_device.cuh"

namespace mgk {

enum : int { ACT_EVENT = 1, ACT_CASCADE = 2, ACT_END = 3, ACT_STOP = 4 };



struct BatchCtl {
    double time, remaining, dt_step, strain_rate;
    double eps_macro[9], sig_macro[9];
    double w[3];
    double sum_two_mu, Ea, na, mixed_tol, ls_tol;
    double tv[9];
    double min_margin;
    int tflat[9], tdiag[9];
    int n_targets, mixed_max_iter, ci, ls_max_iter;
    int n_global_steps, elastic_done;
    int seq_instab, max_seq;
    int need_initial_solve;
    int action, done, status;  // status: 0 ok, 1 instability limit reached, 2 time limit reached
    int cascade_active, cascade_batches, mixed_it, ccount;
    long long cascade_limit;
    long long max_events, events_done;
    long long events_total, cascades, cascade_flips, ls_solves, ls_iters, elastic_steps, fallbacks, sweeps;
    int sel_log_len, sel_log_cap;
    unsigned long long t_start_ns, limit_ns;  // device clock at the first decision; 0: unset
    int past_marked, pad_pm;                  // counted in the batch's past-the-limit word
    unsigned long long ph_ns[6];              // sweep, decide, event solve, cascade flips, cascade solve, interval end
};

// What a run call uploads and reads back for one replica, contiguous over the
// batch so that each direction is one copy for all replicas.
struct alignas(16) RepState {
    BatchCtl ctl;
    rng::Mt mt;
    unsigned bar[4];  // group barrier {arrivals, generation, error, spare}
};

struct BatchRep {
    KmcDevState s;
    KmcPhys p;
    LsArgs ls;
    rng::Barrier bg;
    double gamma0;
    int redraw_dir, redraw_bar, C, pad0;
    int ext, rd_dir, rd_bar, pad1;  // catalog / per-voxel barrier extensions and their RD_* redraw modes
    int ls_prec, pad2;              // LS re-solves: 0 FP64, 1 FP32-refined
    unsigned long long wait_ns;     // limit of one wait at the group's barriers
    int ncta;
    unsigned* bar;  // {arrivals, generation, error, spare}
    dd* chunk_sum;
    int* chunk_unst;
    int* chunk_last;
    dd* tile_sum;   // per chunk: rate sums of 32-mode tiles, tile_cap entries per chunk
    int tile_cap;
    double* ckeys;
    int* cmodes;
    int ccap;
    rng::Mt* mt;
    BatchCtl* ctl;
    int* sel_log;
    unsigned long long* ev_ns;  // device clock at the end of each logged thermal event
    unsigned* past;  // batch-wide: {replicas past the time limit or finished, replicas}
};

namespace {

using namespace kmcdev;

MGK_DEV int vld(const int* p) { return *(const volatile int*)p; }

// eps_macro / sig_macro of the last solve (as LsSolver::macro)
template <int D>
MGK_DEV void macro_from_result(const LsResult* r, BatchCtl* c, const double* w, int N) {
    const double invN = 1.0 / (double)N, mean2mu = c->sum_two_mu * invN;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            const int k = lsdev::sym_idx(D, i, j);
            const double ww = (i == j) ? 0.0 : w[(D == 2) ? 0 : (i + j - 1)];
            const double sgn = (i < j) ? 1.0 : -1.0;
            c->eps_macro[i * D + j] = r->sum_s[k] * invN + sgn * ww;
            c->sig_macro[i * D + j] = r->sum_sig[k] * invN + sgn * ww * mean2mu;
        }
}

// warm-started LS solve with eps_bar = eps_macro (elastic_run) by the group;
// one out-of-line copy per dimension (the passes inlined in it read their
// arguments from shared memory), shared by the replica kernels of that
// dimension
template <int D>
__device__ __noinline__ bool group_solve(BatchRep& R, int rank, const GridBar& gb, unsigned char* smem, LsArgs* sls) {
    BatchCtl* c = R.ctl;
    if (threadIdx.x == 0) {
        *sls = R.ls;
        double wbar[3] = {0, 0, 0};
        const double* eb = c->eps_macro;
        for (int i = 0; i < D; ++i)
            for (int j = i; j < D; ++j) {
                const int k = lsdev::sym_idx(D, i, j);
                sls->ebar_s[k] = (i == j) ? eb[i * D + i] : 0.5 * (eb[i * D + j] + eb[j * D + i]);
                if (i != j) wbar[(D == 2) ? 0 : (i + j - 1)] = 0.5 * (eb[i * D + j] - eb[j * D + i]);
            }
        double sw2 = 0.0;
        for (int k = 0; k < (D == 2 ? 1 : 3); ++k) sw2 += wbar[k] * wbar[k];
        sls->norm_extra = 2.0 * (double)sls->N * sw2;
        sls->norm_extra_first = sls->norm_extra;  // the field's antisymmetric part is uniform
        sls->diff_extra_first = 0.0;
        sls->warm = 1;
        sls->max_iter = c->ls_max_iter;
        sls->tol = c->ls_tol;
        sls->epsp_s = R.s.epsp_s;
        if (rank == 0)
            for (int k = 0; k < 3; ++k) c->w[k] = wbar[k];
    }
    __syncthreads();
    int it32 = 0;
    if (R.ls_prec == 1 && c->ls_max_iter > 1) {
        // FP32 phase (FP32 spectrum, FFTs and Green operator; real-space
        // fields, norms and sums in FP64) to a relative change of
        // max(tol, kFp32Tol), then the FP64 phase below from that field: a
        // warm start whose mean is already eps_bar (LsSolver::solve's scheme)
        __shared__ LsArgs s32;
        if (threadIdx.x == 0) {
            s32 = *sls;
            s32.tol = fmax(sls->tol, kFp32Tol);
            s32.max_iter = sls->max_iter - 1;
        }
        __syncthreads();
        if (!lsdev::ls_solve_group<D, float>(s32, rank, R.ncta, gb, smem)) return false;
        if (threadIdx.x == 0) {
            it32 = s32.result->iters;
            sls->norm_extra_first = sls->norm_extra;
            sls->diff_extra_first = 0.0;
        }
        __syncthreads();
    }
    if (!lsdev::ls_solve_group<D, double>(*sls, rank, R.ncta, gb, smem)) return false;
    if (rank == 0 && threadIdx.x == 0) {
        macro_from_result<D>(sls->result, c, c->w, R.s.N);
        c->ls_solves++;
        c->ls_iters += sls->result->iters + it32;
    }
    return true;
}

// Sweep of the group's rank-th chunk of modes: Q and rates of every mode
// (update_barriers + the rate block, kmc_solver.hpp:341-410, :783-803), with
// each warp handling 32-mode tiles: the tile's rate sum goes to tile_sum, the
// chunk's sum (double-double over tiles), unstable count and last included
// mode to the chunk arrays.  The chunk runs in pieces of whole tiles: the
// CTA first writes the voxel terms of the piece's voxels (stress, softening
// level, for the directional scheme the previous flip) to shared memory, then
// the modes read them there, so a mode loads only its barrier and catalog
// entry.  Warp w takes tiles w, w + nw, ... of the chunk in increasing order
// in every piece, so the sums are added in the same order whatever the pieces.
template <int D, int C>
MGK_DEV void sweep_chunk(BatchRep& R, int rank, double time, unsigned char* smem, size_t smem_bytes) {
    constexpr int S = D == 2 ? 3 : 6;
    __shared__ dd sd[32];
    __shared__ int si[32], sl[32];
    // the replica's state, physics and sweep scratch as locals (read once)
    const KmcDevState st = R.s;
    const KmcPhys ph = R.p;
    const int ncta = R.ncta;
    const long NM = st.NM;
    const int M = st.M;
    const long m0 = NM * rank / ncta, m1 = NM * (rank + 1) / ncta;
    const long ntile = (m1 - m0 + 31) >> 5;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    dd* const ts = R.tile_sum + (long)rank * R.tile_cap;
    // voxel record: sg[S], gb, then (directional) ps[S], npv
    const int rec = ph.directional ? 2 * S + 2 : S + 1;
    double* const vx = reinterpret_cast<double*>(smem);
    const long cap_vox = (long)(smem_bytes / (sizeof(double) * rec));
    // a run of 32 T modes touches at most 32 T / M + 2 voxels
    const long T = max(1L, ((cap_vox - 2) * M) / 32);
    dd acc = {0.0, 0.0};
    int unst = 0, last = -1;
    // four tiles per warp and pass: independent exp / reduction chains in
    // flight (two 256-thread CTAs per SM leave only 16 warps to hide latency)
    constexpr int U = 4;
    for (long T0 = 0; T0 < ntile; T0 += T) {
        const long T1 = min(ntile, T0 + T);
        const long mlo = m0 + (T0 << 5), mhi = min(m1, m0 + (T1 << 5));
        const int vlo = voxel_of(mlo, NM, M), vhi = voxel_of(mhi - 1, NM, M);
        for (int v = vlo + (int)threadIdx.x; v <= vhi; v += blockDim.x) {
            double* r = vx + (long)(v - vlo) * rec;
            sweep_stress<D>(st, v, r);
            r[S] = voxel_gb<D, C>(st, ph, v, time);
            if (ph.directional) r[2 * S + 1] = voxel_prev<D, C>(st, v, r + S + 1);
        }
        __syncthreads();
        const long tfirst = T0 + ((long)wid - T0 % nw + nw) % nw;
        for (long tb = tfirst; tb < T1; tb += (long)nw * U) {
            dd r[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const long t = tb + (long)k * nw;
                const long i = m0 + (t << 5) + lane;
                r[k] = dd{0.0, 0.0};
                if (t < T1 && i < m1) {
                    const int v = voxel_of(i, NM, M);
                    const double* vr = vx + (long)(v - vlo) * rec;
                    const double q = mode_Q_terms<D, C>(st, ph, v, i, vr, vr[S], vr + S + 1,
                                                        ph.directional ? vr[2 * S + 1] : 0.0, st.Q0[i]);
                    st.Q[i] = q;
                    bool inc;
                    r[k].hi = rate_of(ph, q, &inc);
                    if (inc) last = max(last, (int)i);
                    if (q < ph.threshold) ++unst;
                }
            }
            // a tile's 32 rates summed in FP64 by a fixed shuffle tree (within a
            // few ulp of the tile sum, far tighter than the reference's serial
            // sum over all modes); tiles accumulate in double-double
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int k = 0; k < U; ++k) r[k].hi += __shfl_down_sync(0xffffffffu, r[k].hi, o);
            if (lane == 0)
#pragma unroll
                for (int k = 0; k < U; ++k) {
                    const long t = tb + (long)k * nw;
                    if (t < T1) {
                        ts[t] = r[k];
                        acc = dd_add(acc, r[k]);
                    }
                }
        }
        __syncthreads();  // the next piece overwrites the voxel records
    }
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
    if (threadIdx.x == 0) {
        dd a = {0.0, 0.0};
        int u = 0, l = -1;
        for (int w = 0; w < nw; ++w) {
            a = dd_add(a, sd[w]);
            u += si[w];
            l = max(l, sl[w]);
        }
        R.chunk_sum[rank] = a;
        R.chunk_unst[rank] = u;
        R.chunk_last[rank] = l;
    }
    __syncthreads();
}

constexpr unsigned kAltBranch = 1u << 30;

template <int C>
MGK_DEV void redraw_seq(BatchRep& R, rng::Mt* g, long k) {
    const long v = k / R.s.M;
    if (R.ext) {
        // extensions (same order as the host-side draws of the plain form):
        // the per-voxel barrier first, then the modes' draws; fixed catalogs
        // draw no directions
        const int M = R.s.M;
        if (R.rd_bar == RD_VOXEL) {
            const double q = rng::barrier(R.bg, g);
            for (int mm = 0; mm < M; ++mm) R.s.Q0[v * M + mm] = q;
        }
        if (R.rd_dir == RD_ALL)
            for (int mm = 0; mm < M; ++mm) rng::mode<C>(g, R.gamma0, R.s.cat + (v * M + mm) * C);
        else if (R.rd_dir == RD_FLIPPED)
            rng::mode<C>(g, R.gamma0, R.s.cat + k * C);
        if (R.rd_bar == RD_ALL)
            for (int mm = 0; mm < M; ++mm) R.s.Q0[v * M + mm] = rng::barrier(R.bg, g);
        else if (R.rd_bar == RD_FLIPPED)
            R.s.Q0[k] = rng::barrier(R.bg, g);
        return;
    }
    if (R.redraw_dir || R.redraw_bar) {
        for (int mm = 0; mm < R.s.M; ++mm) {
            const long ci = v * R.s.M + mm;
            if (R.redraw_dir) rng::mode<C>(g, R.gamma0, R.s.cat + ci * C);
            if (R.redraw_bar) R.s.Q0[ci] = rng::barrier(R.bg, g);
        }
    } else {
        rng::mode<C>(g, R.gamma0, R.s.cat + k * C);
        R.s.Q0[k] = rng::barrier(R.bg, g);
    }
}

constexpr int kUnitsPerRound = 1024;  // modes redrawn per round of the parallel redraw
constexpr int kSlots = 8;             // draws of one mode at most (3D: 5 polar, 1 uniform; barrier: 2)
constexpr unsigned short kNoFit = 0xffff;
// dynamic shared memory used by redraw_par: two flag arrays, the jump table,
// the unit starts
constexpr size_t kRedrawSmem = 2 * rng::kRingWords + sizeof(unsigned short) * rng::kRingWords + sizeof(long long) * kUnitsPerRound;

// What one redrawn mode consumes, in the reference's order: the catalog
// mode (2D: one polar pair; 3D: five polar pairs and one uniform) and the
// barrier (gaussian: a polar pair; rayleigh: a uniform; modified rayleigh: a
// rejection loop of two uniforms per attempt; the mixture: a uniform, then a
// uniform or the rejection loop).
struct UnitShape {
    bool do_mode, do_bar;
    int C, btype;
    double ratio;
};

// Walk one mode's draws from word q over the acceptance flags; slot[] gets
// each draw's start (the mixture's exponential branch tagged with bit 30).
// Returns the word after the mode, or -1 when the window ends first.
MGK_DEV long long unit_walk(const rng::MtRing* ring, const unsigned char* flagP, const unsigned char* flagR,
                            const UnitShape& us, long long q, long long hi, int* slot) {
    int ns = 0;
    auto polar = [&](const unsigned char* fl) {
        while (q + 4 <= hi && !fl[q % rng::kRingWords]) q += 4;
        if (q + 4 > hi) return false;
        slot[ns++] = (int)(q % rng::kRingWords);
        q += 4;
        return true;
    };
    auto uniform = [&]() {
        if (q + 2 > hi) return false;
        slot[ns++] = (int)(q % rng::kRingWords);
        q += 2;
        return true;
    };
    if (us.do_mode) {
        for (int t = 0; t < (us.C == 2 ? 1 : 5); ++t)
            if (!polar(flagP)) return -1;
        if (us.C == 6 && !uniform()) return -1;
    }
    if (us.do_bar) {
        if (us.btype == 0) {
            if (!polar(flagP)) return -1;
        } else if (us.btype == 1) {
            if (!uniform()) return -1;
        } else if (us.btype == 2) {
            if (!polar(flagR)) return -1;
        } else {
            const long long qu = q;
            if (!uniform()) return -1;
            const double um = __dadd_rn(__dmul_rn(rng::ring_canonical(ring, qu), 1.0), 0.0);
            if (um < us.ratio) {
                if (!uniform()) return -1;
                slot[ns - 1] |= (int)kAltBranch;
            } else if (!polar(flagR)) {
                return -1;
            }
        }
    }
    return q;
}

// Redraw after the flips of modes[0..nflips) (in flip order), by the whole
// CTA, with the ring's stream: the same draws, in the same order, as
// redraw_seq applied flip by flip.  Per round: refill the ring; flag every
// attempt offset (polar acceptance, rejection acceptance) and tabulate, for
// every offset, where a mode starting there ends (all threads); chain the
// mode starts through that table (one thread, one lookup per mode); compute
// the modes' values (all threads).  g is scratch for the fallback (the
// sequential path from the program's starting state, taken if a 3D mode's
// deviatoric part vanishes -- the reference then skips one uniform -- or a
// mode needs more words than the ring holds).
template <int C>
MGK_DEV void redraw_par(BatchRep& R, rng::MtRing* ring, rng::Mt* g, const int* modes, int nflips, unsigned char* smem) {
    __shared__ long long s_unit;
    __shared__ int s_nu, s_fail;
    unsigned char* flagP = smem;
    unsigned char* flagR = smem + rng::kRingWords;
    unsigned short* jump = reinterpret_cast<unsigned short*>(smem + 2 * rng::kRingWords);
    long long* ustart = reinterpret_cast<long long*>(smem + 2 * rng::kRingWords + sizeof(unsigned short) * rng::kRingWords);
    const int M = R.s.M;
    const bool full = R.redraw_dir || R.redraw_bar;
    UnitShape us;
    us.do_mode = full ? R.redraw_dir != 0 : true;
    us.do_bar = full ? R.redraw_bar != 0 : true;
    us.C = C;
    us.btype = R.bg.type;
    us.ratio = R.bg.ratio;
    const int upf = full ? M : 1;
    const long long total = (long long)nflips * upf;
    const bool need_r = us.do_bar && (us.btype == 2 || us.btype == 3);
    const rng::RayleighK rk = need_r ? rng::rayleigh_k(R.bg) : rng::RayleighK{0, 0, 0, 0};
    rng::ring_store(ring, g);  // starting state, for the fallback
    if (R.ext) {
        // the extensions' redraws are short (a per-voxel barrier, or the
        // barriers of a fixed catalog): one thread walks them in order
        if (threadIdx.x == 0)
            for (int f = 0; f < nflips; ++f) redraw_seq<C>(R, g, modes[f]);
        __syncthreads();
        rng::ring_load(ring, g);
        return;
    }
    if (threadIdx.x == 0) {
        s_unit = 0;
        s_fail = 0;
    }
    __syncthreads();
    while (s_unit < total && !s_fail) {
        rng::ring_refill(ring);
        const long long p0 = ring->pos, hi = ring->hi;
        for (long long n = p0 + threadIdx.x; n + 4 <= hi; n += blockDim.x) {
            const int sl = (int)(n % rng::kRingWords);
            flagP[sl] = rng::polar_accepts(ring, n);
            if (need_r) {
                double x;
                flagR[sl] = rng::rayleigh_accepts(ring, n, R.bg, rk, &x);
            }
        }
        __syncthreads();
        // mode starts keep the parity of p0 (every draw takes an even number of words)
        for (long long n = p0 + 2 * threadIdx.x; n < hi; n += 2 * blockDim.x) {
            int sl[kSlots];
            const long long e = unit_walk(ring, flagP, flagR, us, n, hi, sl);
            jump[n % rng::kRingWords] = e < 0 ? kNoFit : (unsigned short)(e - n);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long o = p0, u = s_unit;
            int nu = 0;
            while (u < total && nu < kUnitsPerRound) {
                const unsigned short d = jump[o % rng::kRingWords];
                if (d == kNoFit) break;
                ustart[nu++] = o;
                o += d;
                ++u;
            }
            if (nu == 0) s_fail = 1;  // one mode needs more than the ring holds
            s_nu = nu;
            ring->pos = o;
        }
        __syncthreads();
        const int nu = s_nu;
        const long long ubase = s_unit;
        for (int j = threadIdx.x; j < nu; j += blockDim.x) {
            const long long u = ubase + j;
            const long f = (long)(u / upf);
            const long k = modes[f];
            const long ci = full ? (k / M) * M + (long)(u - (long long)f * upf) : k;
            int rr[kSlots];
            unit_walk(ring, flagP, flagR, us, ustart[j], hi, rr);
            int sl = 0;
            if (us.do_mode) {
                if (C == 2) {
                    double second;
                    const double first = rng::polar_at(ring, rr[sl++], &second);
                    const double h = __dmul_rn(0.5, R.gamma0);
                    R.s.cat[ci * C + 0] = __dmul_rn(h, rng::scale(first, 1.0, 0.0));
                    R.s.cat[ci * C + 1] = __dmul_rn(h, rng::scale(second, 1.0, 0.0));
                } else {
                    double m[10];
                    for (int t = 0; t < 5; ++t) {
                        double second;
                        m[2 * t] = rng::scale(rng::polar_at(ring, rr[sl++], &second), 1.0, 0.0);
                        m[2 * t + 1] = rng::scale(second, 1.0, 0.0);
                    }
                    double ms[9], G[9];
                    for (int i = 0; i < 3; ++i)
                        for (int jj = 0; jj < 3; ++jj) ms[i * 3 + jj] = __dmul_rn(0.5, __dadd_rn(m[i * 3 + jj], m[jj * 3 + i]));
                    const double tr = __dadd_rn(__dadd_rn(ms[0], ms[4]), ms[8]);
                    const double t3 = __dmul_rn(1.0 / 3.0, tr);
                    for (int i = 0; i < 3; ++i)
                        for (int jj = 0; jj < 3; ++jj) G[i * 3 + jj] = __dsub_rn(ms[i * 3 + jj], __dmul_rn(t3, i == jj ? 1.0 : 0.0));
                    double sq = 0.0;
                    for (int jj = 0; jj < 3; ++jj)
                        for (int i = 0; i < 3; ++i) sq = __dadd_rn(sq, __dmul_rn(G[i * 3 + jj], G[i * 3 + jj]));
                    const double nrm = __dsqrt_rn(sq);
                    if (nrm < 1e-12) {
                        atomicOr(&s_fail, 1);
                        ++sl;
                    } else {
                        const double fct = __ddiv_rn(1.0, __dmul_rn(1.4142135623730951, nrm));
                        for (int t = 0; t < 9; ++t) G[t] = __dmul_rn(G[t], fct);
                        const double uu = __dadd_rn(__dmul_rn(rng::ring_canonical(ring, rr[sl++]), __dsub_rn(1.0, 1e-15)), 1e-15);
                        const double mag = __dmul_rn(R.gamma0, __dsqrt_rn(__dmul_rn(-2.0, log(uu))));
                        double* out = R.s.cat + ci * C;
                        out[0] = __dmul_rn(G[0], mag);
                        out[1] = __dmul_rn(G[4], mag);
                        out[2] = __dmul_rn(G[8], mag);
                        out[3] = __dmul_rn(G[1], mag);
                        out[4] = __dmul_rn(G[2], mag);
                        out[5] = __dmul_rn(G[5], mag);
                    }
                }
            }
            if (us.do_bar) {
                const rng::Barrier& b = R.bg;
                double v = 0.0;
                if (us.btype == 0) {
                    double unused;
                    v = rng::scale(rng::polar_at(ring, rr[sl], &unused), b.std_val, b.mean);
                } else if (us.btype == 1) {
                    const double uu = __dadd_rn(__dmul_rn(rng::ring_canonical(ring, rr[sl]), 1.0), 0.0);
                    v = __dadd_rn(b.loc, __dmul_rn(b.scale, __dsqrt_rn(__dmul_rn(-2.0, log(__dsub_rn(1.0, uu))))));
                } else if (us.btype == 2) {
                    rng::rayleigh_accepts(ring, rr[sl], b, rk, &v);
                } else {
                    const int alt = rr[sl + 1];
                    if (alt & (int)kAltBranch) {
                        const double uu = __dadd_rn(__dmul_rn(rng::ring_canonical(ring, alt & ~(int)kAltBranch), 1.0), 0.0);
                        v = __dmul_rn(-b.epsilon, log(__dsub_rn(1.0, uu)));
                    } else {
                        rng::rayleigh_accepts(ring, alt, b, rk, &v);
                    }
                }
                if (b.min_cutoff >= 0.0 && v < b.min_cutoff) v = b.min_cutoff;
                if (b.max_cutoff >= 0.0 && v > b.max_cutoff) v = b.max_cutoff;
                R.s.Q0[ci] = v;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_unit += nu;
        __syncthreads();
    }
    if (s_fail) {
        if (threadIdx.x == 0)
            for (int f = 0; f < nflips; ++f) redraw_seq<C>(R, g, modes[f]);
        __syncthreads();
        rng::ring_load(ring, g);
    }
}

// First CTA of the group: decide the next action from the sweep; for an event
// also select the mode and flip it.  All threads of the CTA call it.
template <int D, int C>
MGK_DEV int decide(BatchRep& R, rng::MtRing* ring, rng::Mt* g, unsigned char* smem) {
    __shared__ int s_act, s_blk, s_sel, s_tile;
    __shared__ double s_target;
    __shared__ dd sh[32];
    __shared__ dd s_before, s_tile_before;
    __shared__ int s_flip;
    BatchCtl* c = R.ctl;
    if (ring->hi - ring->pos < 16) rng::ring_refill(ring);
    if (threadIdx.x == 0) {
        dd tot = {0.0, 0.0};
        int nun = 0;
        for (int b = 0; b < R.ncta; ++b) {
            tot = dd_add(tot, R.chunk_sum[b]);
            nun += R.chunk_unst[b];
        }
        int act = ACT_END;
        double target = 0.0;
        const unsigned long long now = global_ns();
        if (c->t_start_ns == 0) c->t_start_ns = now;
        // time limit of one run call (a sustained avalanche never ends an
        // event): a replica past it keeps working until every replica of the
        // batch is past it (or finished), then stops at its next decision --
        // the launch lasts until its slowest replica's decision anyway, and
        // the others stay busy meanwhile
        bool stop = false;
        if (now - c->t_start_ns > c->limit_ns) {
            if (!c->past_marked) {
                c->past_marked = 1;
                atomicAdd(R.past, 1u);
            }
            stop = *(volatile unsigned*)R.past >= R.past[1];
        }
        if (stop) {
            act = ACT_STOP;
            c->status = 2;
            c->done = 1;
        } else if (!R.p.kmc_mode && nun > 0) {
            act = ACT_CASCADE;
            c->ccount = 0;
        } else {
            if (c->cascade_active) {
                c->cascade_active = 0;
                c->cascades++;
            }
            const double Rv = tot.hi + tot.lo;
            if (Rv > 0.0) {
                const double u1 = rng::ring_uniform(ring, 0.0, 1.0);
                const double tw = __ddiv_rn(-log(u1), Rv);
                if (tw < c->remaining) {
                    c->time = __dadd_rn(c->time, tw);
                    c->eps_macro[c->ci] = __dadd_rn(c->eps_macro[c->ci], __dmul_rn(1.0, __dmul_rn(c->strain_rate, tw)));
                    c->remaining = __dsub_rn(c->remaining, tw);
                    target = __dmul_rn(rng::ring_uniform(ring, 0.0, 1.0), Rv);
                    act = ACT_EVENT;
                }
            }
            if (act == ACT_END) {
                c->eps_macro[c->ci] = __dadd_rn(c->eps_macro[c->ci], __dmul_rn(1.0, __dmul_rn(c->strain_rate, c->remaining)));
                c->time = __dadd_rn(c->time, c->remaining);
                c->remaining = 0.0;
            }
        }
        s_act = act;
        s_target = target;
        s_blk = 0x7fffffff;
        s_sel = 0x7fffffff;
        s_tile = 0x7fffffff;
        c->action = act;
    }
    __syncthreads();
    if (s_act != ACT_EVENT) return s_act;
    // selection (kmc_solver.hpp:817-838): the chunk holding the crossing of
    // the cumulative rate with the target, then its 32-mode tile, then the
    // mode, each by a fixed-order double-double prefix
    const double target = s_target;
    const int nc = R.ncta;
    {
        const int seg = (nc + blockDim.x - 1) / blockDim.x;
        const int b0 = threadIdx.x * seg, b1 = min(nc, b0 + seg);
        dd mine = {0.0, 0.0};
        for (int b = b0; b < b1; ++b) mine = dd_add(mine, R.chunk_sum[b]);
        dd run = block_excl_scan(mine, sh, nullptr);
        int my_blk = -1;
        for (int b = b0; b < b1; ++b) {
            const dd nx = dd_add(run, R.chunk_sum[b]);
            if (dd_ge(nx, target)) {
                my_blk = b;
                atomicMin(&s_blk, b);
                break;
            }
            run = nx;
        }
        __syncthreads();
        if (my_blk >= 0 && my_blk == s_blk) s_before = run;
    }
    __syncthreads();
    const int cb = s_blk;
    long m0 = 0, m1 = 0;
    if (cb != 0x7fffffff) {
        m0 = R.s.NM * cb / nc;
        m1 = R.s.NM * (cb + 1) / nc;
        const long ntile = (m1 - m0 + 31) >> 5;
        const dd* ts = R.tile_sum + (long)cb * R.tile_cap;
        const long seg = (ntile + blockDim.x - 1) / blockDim.x;
        const long t0 = threadIdx.x * seg, t1 = min(ntile, t0 + seg);
        dd mine = {0.0, 0.0};
        for (long t = t0; t < t1; ++t) mine = dd_add(mine, ts[t]);
        dd run = dd_add(s_before, block_excl_scan(mine, sh, nullptr));
        long my_tile = -1;
        for (long t = t0; t < t1; ++t) {
            const dd nx = dd_add(run, ts[t]);
            if (dd_ge(nx, target)) {
                my_tile = t;
                atomicMin(&s_tile, (int)t);
                break;
            }
            run = nx;
        }
        __syncthreads();
        if (my_tile >= 0 && my_tile == s_tile) s_tile_before = run;
    }
    __syncthreads();
    if (threadIdx.x < 32 && cb != 0x7fffffff && s_tile != 0x7fffffff) {
        const int lane = threadIdx.x;
        const long i = m0 + ((long)s_tile << 5) + lane;
        bool inc = false;
        double r = 0.0;
        if (i < m1) r = rate_of(R.p, R.s.Q[i], &inc);
        dd incl = {r, 0.0};
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const dd y = {__shfl_up_sync(0xffffffffu, incl.hi, o), __shfl_up_sync(0xffffffffu, incl.lo, o)};
            if (lane >= o) incl = dd_add(y, incl);
        }
        dd excl = {__shfl_up_sync(0xffffffffu, incl.hi, 1), __shfl_up_sync(0xffffffffu, incl.lo, 1)};
        if (lane == 0) excl = dd{0.0, 0.0};
        const dd before = s_tile_before;
        const dd nx = dd_add(before, incl);
        const dd pr = dd_add(before, excl);
        const unsigned hit = __ballot_sync(0xffffffffu, inc && dd_ge(nx, target));
        const unsigned incm = __ballot_sync(0xffffffffu, inc);
        if (lane == 0) {
            if (hit) {
                s_sel = (int)(m0 + ((long)s_tile << 5) + (__ffs(hit) - 1));
            } else if (incm) {  // the tile's sum and its scan differ in the last bits: its last mode
                s_sel = (int)(m0 + ((long)s_tile << 5) + (31 - __clz(incm)));
                c->fallbacks++;
            }
        }
        if (hit && lane == __ffs(hit) - 1) {
            const double below = target - (pr.hi + pr.lo), above = (nx.hi + nx.lo) - target;
            const double cmargin = fmin(below, above) / fmax(target, 1e-300);
            if (cmargin < c->min_margin) c->min_margin = cmargin;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long k = s_sel;
        if (k == 0x7fffffff) {
            k = -1;
            c->fallbacks++;
            for (int b = 0; b < nc; ++b) k = max(k, (long)R.chunk_last[b]);
        }
        s_flip = (int)k;
        if (k >= 0) {
            const bool instab = R.s.Q[k] <= R.p.threshold;
            apply_flip<D, C>(R.s, R.p, k, c->time, nullptr);
            c->seq_instab = instab ? c->seq_instab + 1 : 0;
            if (c->sel_log_len < c->sel_log_cap) R.sel_log[c->sel_log_len++] = (int)k;
        }
    }
    __syncthreads();
    if (s_flip >= 0) redraw_par<C>(R, ring, g, &s_flip, 1, smem);
    return ACT_EVENT;
}

// bitonic sort of (key, mode) in shared memory by one CTA (n <= cap)
MGK_DEV void cta_sort(double* keys, int* modes, int n, unsigned char* smem, size_t smem_bytes) {
    int npow2 = 1;
    while (npow2 < n) npow2 <<= 1;
    const bool in_smem = (size_t)npow2 * 12 <= smem_bytes;
    double* k = in_smem ? reinterpret_cast<double*>(smem) : keys;
    int* m = in_smem ? reinterpret_cast<int*>(smem + (size_t)npow2 * 8) : modes;
    if (in_smem) {
        for (int i = threadIdx.x; i < npow2; i += blockDim.x) {
            k[i] = i < n ? keys[i] : INFINITY;
            m[i] = i < n ? modes[i] : 0x7fffffff;
        }
    } else {
        for (int i = n + threadIdx.x; i < npow2; i += blockDim.x) {
            k[i] = INFINITY;
            m[i] = 0x7fffffff;
        }
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
                        const double tk = k[i];
                        k[i] = k[j];
                        k[j] = tk;
                        const int tm = m[i];
                        m[i] = m[j];
                        m[j] = tm;
                    }
                }
            }
            __syncthreads();
        }
    if (in_smem)
        for (int i = threadIdx.x; i < n; i += blockDim.x) modes[i] = m[i];
    __syncthreads();
}

// Sort of (keys, modes)[0..n) by key_less with every CTA of the group, for
// lists too long for one CTA's shared memory: a bitonic network over npow2
// entries (padded with +inf); strides whose pairs span more than one
// tile of `tile` entries run in global memory with a group barrier after
// each, the smaller strides of each merge size inside shared memory tile by
// tile.  keys and modes hold npow2 entries.  Returns false when a barrier
// wait gave up.
MGK_DEV bool group_sort(double* keys, int* modes, int n, int npow2, int tile, int rank, int ncta, const GridBar& gb,
                        unsigned char* smem) {
    const long gtid = (long)rank * blockDim.x + threadIdx.x, gthreads = (long)ncta * blockDim.x;
    for (long i = n + gtid; i < npow2; i += gthreads) {
        keys[i] = INFINITY;
        modes[i] = 0x7fffffff;
    }
    if (!grid_sync(gb)) return false;
    double* k = reinterpret_cast<double*>(smem);
    int* m = reinterpret_cast<int*>(smem + (size_t)tile * 8);
    for (int size = 2; size <= npow2; size <<= 1) {
        int stride = size >> 1;
        for (; 2 * stride > tile; stride >>= 1) {
            for (long i = gtid; i < npow2; i += gthreads) {
                const long j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const bool sw = up ? key_less(keys[j], modes[j], keys[i], modes[i])
                                       : key_less(keys[i], modes[i], keys[j], modes[j]);
                    if (sw) {
                        const double tk = keys[i];
                        keys[i] = keys[j];
                        keys[j] = tk;
                        const int tm = modes[i];
                        modes[i] = modes[j];
                        modes[j] = tm;
                    }
                }
            }
            if (!grid_sync(gb)) return false;
        }
        for (long t0 = (long)rank * tile; t0 < npow2; t0 += (long)ncta * tile) {
            for (int i = threadIdx.x; i < tile; i += blockDim.x) {
                k[i] = keys[t0 + i];
                m[i] = modes[t0 + i];
            }
            __syncthreads();
            for (int st = stride; st > 0; st >>= 1) {
                for (int i = threadIdx.x; i < tile; i += blockDim.x) {
                    const int j = i ^ st;
                    if (j > i) {
                        const bool up = ((t0 + i) & size) == 0;
                        const bool sw = up ? key_less(k[j], m[j], k[i], m[i]) : key_less(k[i], m[i], k[j], m[j]);
                        if (sw) {
                            const double tk = k[i];
                            k[i] = k[j];
                            k[j] = tk;
                            const int tm = m[i];
                            m[i] = m[j];
                            m[j] = tm;
                        }
                    }
                }
                __syncthreads();
            }
            for (int i = threadIdx.x; i < tile; i += blockDim.x) {
                keys[t0 + i] = k[i];
                modes[t0 + i] = m[i];
            }
            __syncthreads();
        }
        if (!grid_sync(gb)) return false;
    }
    return true;
}

template <int D, int C>
MGK_DEV void run_replica(BatchRep& R, int rank, unsigned char* smem, size_t smem_bytes) {
    __shared__ LsArgs s_ls;
    // the replica's generator (rank 0 only) lives at the end of the dynamic
    // shared memory, past everything the LS solve, sort and redraw use
    rng::Mt& s_mt = *reinterpret_cast<rng::Mt*>(smem + smem_bytes);
    rng::MtRing& s_ring = *reinterpret_cast<rng::MtRing*>(smem + smem_bytes + sizeof(rng::Mt));
    __shared__ int s_flag;
    BatchCtl* c = R.ctl;
    const GridBar gb{R.bar, (unsigned)R.ncta, R.bar + 2, R.wait_ns};
    if (rank == 0) {
        for (int i = threadIdx.x; i < 624; i += blockDim.x) s_mt.mt[i] = R.mt->mt[i];
        if (threadIdx.x == 0) s_mt.idx = R.mt->idx;
        __syncthreads();
        rng::ring_load(&s_ring, &s_mt);
    }
    bool ok = true;
    if (vld(&c->need_initial_solve)) {
        ok = group_solve<D>(R, rank, gb, smem, &s_ls);
        if (ok && rank == 0 && threadIdx.x == 0) {
            c->need_initial_solve = 0;
            c->remaining = __dadd_rn(c->remaining, c->dt_step);
        }
        ok = ok && grid_sync(gb);
    }
    const bool timer = rank == 0 && threadIdx.x == 0;
    unsigned long long tp = timer ? global_ns() : 0ull;
    auto phase = [&](int k) {
        if (timer) {
            const unsigned long long t = global_ns();
            c->ph_ns[k] += t - tp;
            tp = t;
        }
    };
    while (ok) {
        if (vld(&c->done)) break;
        sweep_chunk<D, C>(R, rank, c->time, smem, smem_bytes);
        if (!grid_sync(gb)) break;
        if (timer) c->sweeps++;
        phase(0);
        if (rank == 0) decide<D, C>(R, &s_ring, &s_mt, smem);
        if (!grid_sync(gb)) break;
        phase(1);
        const int act = vld(&c->action);
        if (act == ACT_STOP) break;
        if (act == ACT_EVENT) {
            if (!group_solve<D>(R, rank, gb, smem, &s_ls)) break;
            phase(2);
            if (rank == 0 && threadIdx.x == 0) {
                if (c->events_done < c->sel_log_cap) R.ev_ns[c->events_done] = global_ns();
                c->events_done++;
                c->events_total++;
                if (c->seq_instab > c->max_seq) {
                    c->status = 1;
                    c->done = 1;
                }
                if (c->events_done >= c->max_events) c->done = 1;
            }
        } else if (act == ACT_CASCADE) {
            // collect the lowest-Q unstable mode of every unstable voxel
            // (fields as locals: the stores below would otherwise reload them)
            const long v0 = (long)R.s.N * rank / R.ncta, v1 = (long)R.s.N * (rank + 1) / R.ncta;
            const double* const Qv = R.s.Q;
            const int Mv = R.s.M;
            const double thr = R.p.threshold;
            double* const ckeys = R.ckeys;
            int* const cmodes = R.cmodes;
            for (long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
                double best = 0.0;
                int bm = -1;
                for (int m = 0; m < Mv; ++m) {
                    const double q = Qv[v * Mv + m];
                    if (q < thr && (bm < 0 || q < best)) {
                        best = q;
                        bm = m;
                    }
                }
                if (bm >= 0) {
                    const int slot = atomicAdd(&c->ccount, 1);
                    ckeys[slot] = best;
                    cmodes[slot] = (int)(v * Mv + bm);
                }
            }
            if (!grid_sync(gb)) break;
            {
                // long lists: sorted by the whole group; short ones by rank 0 below
                const int n = vld(&c->ccount);
                int npow2 = 1;
                while (npow2 < n) npow2 <<= 1;
                if ((size_t)npow2 * 12 > smem_bytes) {
                    int tile = 1;
                    while ((size_t)tile * 2 * 12 <= smem_bytes && tile * 2 <= npow2) tile <<= 1;
                    if (!group_sort(R.ckeys, R.cmodes, n, npow2, tile, rank, R.ncta, gb, smem)) break;
                }
            }
            if (rank == 0) {
                const int n = vld(&c->ccount);
                int npow2 = 1;
                while (npow2 < n) npow2 <<= 1;
                if ((size_t)npow2 * 12 <= smem_bytes) cta_sort(R.ckeys, R.cmodes, n, smem, smem_bytes);
                if (threadIdx.x == 0) {
                    // state as locals: the flips store through pointers that
                    // could otherwise alias the replica record and the control
                    // block, and reload them at every flip
                    const KmcDevState st = R.s;
                    const KmcPhys ph = R.p;
                    const int* const cm = R.cmodes;
                    const double tnow = c->time;
                    for (int f = 0; f < n; ++f) apply_flip<D, C>(st, ph, cm[f], tnow, nullptr);
                }
                __syncthreads();
                // flips touch no other voxel's catalog or barriers, so all
                // redraws may follow all flips (same draws, same order)
                redraw_par<C>(R, &s_ring, &s_mt, R.cmodes, n, smem);
                if (threadIdx.x == 0) {
                    c->cascade_flips += n;
                    c->cascade_batches++;
                    c->cascade_active = 1;
                    if (c->cascade_batches > c->cascade_limit) {  // run_cascade's batch limit (:556)
                        c->cascades++;
                        c->cascade_batches = 0;
                    }
                }
            }
            if (!grid_sync(gb)) break;
            phase(3);
            if (!group_solve<D>(R, rank, gb, smem, &s_ls)) break;
            phase(4);
        } else {
            // end of interval: mixed-BC loop, then the next interval
            for (;;) {
                if (!group_solve<D>(R, rank, gb, smem, &s_ls)) {
                    ok = false;
                    break;
                }
                if (rank == 0 && threadIdx.x == 0) {
                    double err[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, emax = 0.0;
                    for (int t = 0; t < c->n_targets; ++t) {
                        const double e = c->tv[t] - c->sig_macro[c->tflat[t]];
                        err[c->tflat[t]] = e;
                        emax = fmax(emax, fabs(e));
                    }
                    int stop = emax < c->mixed_tol;
                    if (!stop) {
                        double tr = 0.0;
                        for (int a = 0; a < D; ++a) tr += err[a * D + a];
                        for (int t = 0; t < c->n_targets; ++t) {
                            const int k = c->tflat[t];
                            c->eps_macro[k] += (err[k] - c->na * tr * (c->tdiag[t] ? 1.0 : 0.0)) / c->Ea;
                        }
                        if (++c->mixed_it >= c->mixed_max_iter) stop = 1;
                    }
                    if (stop) {
                        c->mixed_it = 0;
                        c->elastic_done++;
                        c->elastic_steps++;
                        if (c->elastic_done >= c->n_global_steps) c->done = 1;
                        else c->remaining = __dadd_rn(c->remaining, c->dt_step);
                    }
                    s_flag = stop;
                    c->action = stop ? 0 : ACT_END;
                }
                if (!grid_sync(gb)) {
                    ok = false;
                    break;
                }
                if (vld(&c->action) == 0) break;
            }
            if (!ok) break;
            phase(5);
        }
        if (!grid_sync(gb)) break;
    }
    if (rank == 0 && threadIdx.x == 0 && !c->past_marked) {  // finished (or failed): no longer holds the others
        c->past_marked = 1;
        atomicAdd(R.past, 1u);
    }
    if (rank == 0) {
        __syncthreads();
        rng::ring_store(&s_ring, &s_mt);
        for (int i = threadIdx.x; i < 624; i += blockDim.x) R.mt->mt[i] = s_mt.mt[i];
        if (threadIdx.x == 0) R.mt->idx = s_mt.idx;
    }
}

__global__ void __launch_bounds__(256, 2) batch_kernel(BatchRep* reps, const int2* map, size_t smem_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int2 m = map[blockIdx.x];
    BatchRep& R = reps[m.x];
    if (R.s.D == 2) run_replica<2, 2>(R, m.y, smem, smem_bytes);
    else if (R.C == 2) run_replica<3, 2>(R, m.y, smem, smem_bytes);
    else run_replica<3, 6>(R, m.y, smem, smem_bytes);
}

}  // namespace

// ---------------------------------------------------------------- host side
#define BCK(x)                                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

static std::atomic<int> g_batch_plan{0};
void set_batch_plan_objective(int objective) { g_batch_plan = objective; }
int batch_plan_objective() { return g_batch_plan; }

BatchEngine::BatchEngine(int n, const mgk_kmc_params* params, const double* const* E, const double* const* nu) {
    if (n < 1) throw std::invalid_argument("empty batch");
    // replicas are built concurrently: each one's initial catalog and barrier
    // draws run on the host (the reference's std::mt19937 stream, sequential
    // within a replica), which dominates set-up for large grids
    owned_eng_.resize(n);
    {
        int dev0 = 0;
        cudaGetDevice(&dev0);
        std::vector<std::string> errs(n);
        std::atomic<int> next{0};
        auto work = [&]() {
            cudaSetDevice(dev0);
            for (int r = next++; r < n; r = next++) {
                try {
                    owned_eng_[r].reset(new KmcEngine(params[r], E[r], nu[r]));
                } catch (const std::exception& ex) {
                    errs[r] = ex.what();
                }
            }
        };
        const int nt = std::max(1, std::min(n, (int)std::max(1u, std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        for (int r = 0; r < n; ++r)
            if (!errs[r].empty()) throw std::runtime_error("replica " + std::to_string(r) + ": " + errs[r]);
    }
    for (auto& e : owned_eng_) eng_.push_back(e.get());
    init();
}

BatchEngine::BatchEngine(const std::vector<KmcEngine*>& sims) : eng_(sims) {
    if (eng_.empty()) throw std::invalid_argument("empty batch");
    for (KmcEngine* e : eng_)
        if (!e) throw std::invalid_argument("null simulation");
    init();
}

void BatchEngine::init() {
    const int n = (int)eng_.size();
    for (KmcEngine* e : eng_)
        if (e->fp_) throw std::domain_error("fast patching runs in the plain form (mgk_kmc_run) only");
    BCK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // two CTAs per SM: 128 registers a thread (the kernel spills ~2 kB a
    // thread at that bound, and still runs 12-37 % faster than one 254-register
    // CTA per SM, measured on B200); the dynamic shared memory of each holds
    // two LS FFT buffers (or the cascade sort / redraw scratch) and, past
    // them, the replica generator
    // shared memory of a replica's LS passes (line buffer + twiddle table);
    // the group tiling (plan_passes) fills it
    const size_t ls_budget = 72 * 1024;
    // CTAs per SM: two when the largest launch this plan can make fits twice
    int per_sm = 0;
    {
        const size_t smem_max = std::max({(size_t)4096 * 12, kRedrawSmem, ls_budget}) + sizeof(rng::Mt) +
                                sizeof(rng::MtRing);
        BCK(ensure_dyn_smem((const void*)batch_kernel, smem_max));
        BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, 256, smem_max));
        per_sm = std::min(per_sm, 2);
        if (per_sm < 1) throw std::runtime_error("batch kernel does not fit on an SM");
    }
    const int budget = per_sm * nsm;
    if (n > budget) throw std::invalid_argument("more replicas than co-resident CTAs");
    // CTA groups: every replica gets its floor (below), then each further CTA
    // goes to the replica whose event rate it raises most, by the model
    // t_event(c) = kSecPerWork * work / c + kSecPerEvent (work = modes swept +
    // 24 x LS voxels in 2D, 72 x in 3D; the constants are fitted to measured
    // 64^2 runs on one and nine CTAs).  This maximises the batch's total steps/s: small grids,
    // whose events are latency-bound, gain most from extra CTAs; the largest
    // grids still advance on the CTAs their share of the model gives them.
    constexpr double kSecPerWork = 12.7e-9, kSecPerEvent = 160e-6;
    std::vector<double> work(n);
    std::vector<int> lim(n);
    for (int r = 0; r < n; ++r) {
        // a 3D LS voxel costs ~3x a 2D one (6 components, 3 FFT axes; measured
        // 32^3 events against the 2D fit)
        work[r] = (double)eng_[r]->NM_ + (eng_[r]->D_ == 2 ? 24.0 : 72.0) * eng_[r]->N_;
        lim[r] = std::max(1, std::min(eng_[r]->ls_->grid_, 160));
    }
    auto rate = [&](int r, int c) { return 1.0 / (kSecPerWork * work[r] / c + kSecPerEvent); };
    // floor: enough CTAs that a replica's modelled event time stays under
    // kMaxEventSeconds (a large grid on one CTA would otherwise take seconds
    // per event, and a run or a serving slice waits for its last event)
    constexpr double kMaxEventSeconds = 0.25;
    ncta_.assign(n, 1);
    int used = 0;
    for (int r = 0; r < n; ++r) {
        const int need = (int)std::ceil(kSecPerWork * work[r] / (kMaxEventSeconds - kSecPerEvent));
        ncta_[r] = std::max(1, std::min(lim[r], need));
        used += ncta_[r];
    }
    while (used > budget) {  // the floors do not fit: take from the largest groups
        int big = 0;
        for (int r = 1; r < n; ++r)
            if (ncta_[r] > ncta_[big]) big = r;
        if (ncta_[big] <= 1) break;
        --ncta_[big];
        --used;
    }
    const bool balanced = batch_plan_objective() == 1;
    while (used < budget) {
        int best = -1;
        double key = 0.0;
        for (int r = 0; r < n; ++r) {
            if (ncta_[r] >= lim[r]) continue;
            if (balanced) {
                // the replica furthest behind the rate it would have on the
                // whole GPU (its modelled rate on `budget` CTAs) gets the CTA
                const double behind = rate(r, std::min(budget, lim[r])) / rate(r, ncta_[r]);
                if (behind > key) {
                    key = behind;
                    best = r;
                }
            } else {
                // throughput: the replica whose modelled event rate it raises most
                const double g = rate(r, ncta_[r] + 1) - rate(r, ncta_[r]);
                if (g > key) {
                    key = g;
                    best = r;
                }
            }
        }
        if (best < 0) break;
        ++ncta_[best];
        ++used;
    }
    total_ctas_ = used;
    std::vector<LsArgs> plans(n);
    smem_ = std::max((size_t)4096 * 12, kRedrawSmem);
    for (int r = 0; r < n; ++r) {
        // the LS pass plan for the replica's group, measured on the
        // replica's own grid at the group's CTA count (LsSolver::tune)
        plans[r] = eng_[r]->ls_->args_;
        // measured at the largest power of two <= the group's CTA count (a
        // serving loop re-plans its batch whenever jobs come and go: this
        // bounds the distinct measurements per grid shape to ~9)
        int tn = 1;
        while (tn * 2 <= ncta_[r]) tn *= 2;
        const LsPlan lp = LsSolver::autotune_enabled() ? eng_[r]->ls_->tune(tn, ls_budget) : LsPlan();
        const size_t need = plan_passes(plans[r], ncta_[r], ls_budget, lp);
        if (need == 0) throw std::invalid_argument("grid axis too long for the batched LS passes");
        smem_ = std::max(smem_, need);
    }
    smem_ = (smem_ + 15) & ~(size_t)15;
    const size_t smem_launch = smem_ + sizeof(rng::Mt) + sizeof(rng::MtRing);
    BCK(ensure_dyn_smem((const void*)batch_kernel, smem_launch));
    int fit = 0;
    BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, batch_kernel, 256, smem_launch));
    if (fit < per_sm) throw std::runtime_error("batch kernel does not fit its planned CTAs per SM");
    // device scratch of every replica in one allocation (a serving loop
    // re-plans its batch whenever jobs come and go: one cudaMalloc and one
    // cudaFree per batch instead of a dozen per replica), carved in two
    // passes: sizes first, then pointers into the arena
    std::vector<BatchRep> reps(n);
    std::vector<int2> map;
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < ncta_[r]; ++k) map.push_back(make_int2(r, k));
    char* base = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        size_t off = 0;
        auto take = [&](size_t bytes) -> void* {
            void* q = base ? base + off : nullptr;
            off += (bytes + 255) & ~(size_t)255;
            return q;
        };
        d_state_ = (RepState*)take(sizeof(RepState) * n);
        d_past_ = (unsigned*)take(2 * sizeof(unsigned));
        alloc_reps_ = (BatchRep*)take(sizeof(BatchRep) * n);
        map_ = (int2*)take(sizeof(int2) * map.size());
        for (int r = 0; r < n; ++r) {
            KmcEngine& e = *eng_[r];
            BatchRep& R = reps[r];
            R.ncta = ncta_[r];
            R.ctl = &d_state_[r].ctl;
            R.mt = &d_state_[r].mt;
            R.bar = d_state_[r].bar;
            R.past = d_past_;
            R.chunk_sum = (dd*)take(sizeof(dd) * R.ncta);
            R.chunk_unst = (int*)take(sizeof(int) * R.ncta);
            R.chunk_last = (int*)take(sizeof(int) * R.ncta);
            R.tile_cap = (int)((e.NM_ / R.ncta + 2 + 31) / 32);
            R.tile_sum = (dd*)take(sizeof(dd) * R.tile_cap * R.ncta);
            int npow2 = 1;
            while (npow2 < e.N_) npow2 <<= 1;
            R.ckeys = (double*)take(sizeof(double) * npow2);
            R.cmodes = (int*)take(sizeof(int) * npow2);
            R.ccap = npow2;
            R.sel_log = (int*)take(sizeof(int) * kSelLog);
            R.ev_ns = (unsigned long long*)take(sizeof(unsigned long long) * kSelLog);
            R.ls = plans[r];
            R.ls.partials = (double*)take(sizeof(double) * kMaxPartials * (R.ncta + 1));
            R.ls.red = R.ls.partials + (size_t)kMaxPartials * R.ncta;
            R.ls.result = (LsResult*)take(sizeof(LsResult));
            R.ls.bar = R.bar;
            R.ls.err = R.bar + 2;
        }
        if (pass == 0) {
            BCK(cudaMalloc((void**)&arena_, off));
            base = arena_;
        }
    }
    for (int r = 0; r < n; ++r) {
        KmcEngine& e = *eng_[r];
        BatchRep& R = reps[r];
        R.s = e.dev_;
        R.p = e.phys_;
        R.bg = rng::Barrier{e.bar_.type, e.bar_.mean, e.bar_.std_val, e.bar_.min_cutoff, e.bar_.max_cutoff, e.bar_.loc,
                            e.bar_.scale, e.bar_.epsilon, e.bar_.ratio};
        R.gamma0 = e.p_.gamma0;
        R.redraw_dir = e.p_.redraw_directions;
        R.redraw_bar = e.p_.redraw_barriers;
        R.ext = e.p_.catalog_type != 0 || e.p_.barrier_per_voxel;
        R.ls_prec = e.p_.ls_precision;
        R.rd_dir = e.rd_dir_;
        R.rd_bar = e.rd_bar_;
        R.C = e.C_;
        // the longest phase the group's other CTAs wait through is rank 0's
        // part of a cascade batch (flips one after another, then the redraw
        // of every mode): its limit grows with the grid, so an avalanche
        // through a large 3D grid (every voxel unstable, 100 modes each) is
        // not taken for a stalled group
        R.wait_ns = kBarrierTimeoutNs + 20000ull * (unsigned long long)e.N_ + 4000ull * (unsigned long long)e.NM_;
    }
    BCK(cudaMemset(d_state_, 0, sizeof(RepState) * n));
    BCK(cudaMemcpy(alloc_reps_, reps.data(), sizeof(BatchRep) * n, cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(map_, map.data(), sizeof(int2) * map.size(), cudaMemcpyHostToDevice));
    BCK(cudaMallocHost((void**)&h_state_, sizeof(RepState) * n));
    reps_host_ = reps;
    h2d_.assign(n, 0);
}

BatchEngine::~BatchEngine() {
    if (st_) cudaStreamSynchronize(st_);
    cudaFree(arena_);
    if (h_state_) cudaFreeHost(h_state_);
    if (h_logs_) cudaFreeHost(h_logs_);
    eng_.clear();
    owned_eng_.clear();
    if (st_) cudaStreamDestroy(st_);
}

static void mt_from_host(const std::mt19937& g, rng::Mt* out) {
    std::ostringstream os;
    os << g;
    std::istringstream is(os.str());
    unsigned long v;
    for (int i = 0; i < 624; ++i) {
        is >> v;
        out->mt[i] = (unsigned)v;
    }
    is >> v;
    out->idx = (int)v;
    out->pad = 0;
}

static_assert(sizeof(rng::Mt) == 626 * sizeof(unsigned), "generator state layout");

mgk_status BatchEngine::run(const mgk_run_params* rp, long long max_events, double* elapsed_ms) {
    const int n = (int)eng_.size();
    try {
        for (int r = 0; r < n; ++r) {
            KmcEngine& e = *eng_[r];
            const mgk_run_params& p = rp[r];
            const int D = e.D_;
            RepState& hs = h_state_[r];
            std::memset(&hs, 0, sizeof(RepState));
            BatchCtl& c = hs.ctl;
            c.time = e.time_;
            std::memcpy(c.eps_macro, e.eps_macro_, sizeof(c.eps_macro));
            std::memcpy(c.sig_macro, e.sig_macro_, sizeof(c.sig_macro));
            for (int k = 0; k < 3; ++k) c.w[k] = e.ls_->w_[k];
            c.remaining = e.batch_started ? e.batch_remaining : 0.0;
            c.dt_step = std::fabs(p.step_size) / e.p_.strain_rate;
            c.strain_rate = e.p_.strain_rate;
            c.sum_two_mu = e.ls_->sum_two_mu_;
            c.Ea = e.E_avg_;
            c.na = e.nu_avg_;
            c.mixed_tol = p.mixed_tol;
            c.mixed_max_iter = p.mixed_max_iter;
            c.ls_tol = e.p_.ls_tol;
            c.ls_max_iter = e.p_.ls_max_iter;
            c.n_targets = p.n_targets;
            for (int t = 0; t < p.n_targets; ++t) {
                c.tflat[t] = p.target_i[t] * D + p.target_j[t];
                c.tdiag[t] = p.target_i[t] == p.target_j[t];
                c.tv[t] = p.target_v[t];
            }
            c.ci = p.comp_i * D + p.comp_j;
            c.n_global_steps = p.n_global_steps;
            c.elastic_done = 0;
            c.max_seq = (int)(p.max_kmc_steps_pct * (double)e.N_);
            c.need_initial_solve = e.batch_started ? 0 : 1;
            // a replica's own budget (run params) wins over the call's
            c.max_events = p.max_events > 0 ? p.max_events : (max_events > 0 ? max_events : (1LL << 62));
            c.cascade_limit = p.max_cascade_batches > 0 ? p.max_cascade_batches : e.N_;
            c.min_margin = 1.0;
            c.sel_log_cap = kSelLog;
            c.t_start_ns = 0;
            c.limit_ns = (unsigned long long)(time_limit_s_ * 1e9);
            if (e.batch_mt_.size() == 626) std::memcpy(&hs.mt, e.batch_mt_.data(), sizeof(rng::Mt));
            else mt_from_host(e.rng_, &hs.mt);
            h2d_[r] = sizeof(RepState);
        }
        BCK(cudaMemcpyAsync(d_state_, h_state_, sizeof(RepState) * n, cudaMemcpyHostToDevice, st_));
        const unsigned past0[2] = {0u, (unsigned)n};
        BCK(cudaMemcpyAsync(d_past_, past0, sizeof(past0), cudaMemcpyHostToDevice, st_));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, st_);
        void* args[] = {&alloc_reps_, &map_, &smem_};
        const size_t smem_launch = smem_ + sizeof(rng::Mt) + sizeof(rng::MtRing);
        BCK(cudaLaunchCooperativeKernel((const void*)batch_kernel, dim3(total_ctas_), dim3(256), args, smem_launch, st_));
        cudaEventRecord(e1, st_);
        BCK(cudaMemcpyAsync(h_state_, d_state_, sizeof(RepState) * n, cudaMemcpyDeviceToHost, st_));
        BCK(cudaStreamSynchronize(st_));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (elapsed_ms) *elapsed_ms = ms;
        mgk_status st = MGK_OK;
        last_.assign(n, BatchStats{});
        // every replica's event-time and selection logs in one pinned
        // staging buffer, copied asynchronously, one synchronisation
        std::vector<size_t> log_off(n + 1, 0);
        for (int r = 0; r < n; ++r) {
            const BatchCtl& c = h_state_[r].ctl;
            const long long ne = std::min<long long>(c.events_done, kSelLog);
            log_off[r + 1] = log_off[r] + sizeof(unsigned long long) * ne + ((sizeof(int) * c.sel_log_len + 7) & ~(size_t)7);
        }
        if (log_off[n] > h_logs_cap_) {
            if (h_logs_) cudaFreeHost(h_logs_);
            h_logs_ = nullptr;
            h_logs_cap_ = 0;
            BCK(cudaMallocHost((void**)&h_logs_, 2 * log_off[n]));
            h_logs_cap_ = 2 * log_off[n];
        }
        for (int r = 0; r < n; ++r) {
            const BatchCtl& c = h_state_[r].ctl;
            const long long ne = std::min<long long>(c.events_done, kSelLog);
            char* dst = h_logs_ + log_off[r];
            if (ne)
                BCK(cudaMemcpyAsync(dst, reps_host_[r].ev_ns, sizeof(unsigned long long) * ne, cudaMemcpyDeviceToHost, st_));
            if (c.sel_log_len)
                BCK(cudaMemcpyAsync(dst + sizeof(unsigned long long) * ne, reps_host_[r].sel_log, sizeof(int) * c.sel_log_len,
                                    cudaMemcpyDeviceToHost, st_));
        }
        BCK(cudaStreamSynchronize(st_));
        for (int r = 0; r < n; ++r) {
            KmcEngine& e = *eng_[r];
            const BatchCtl& c = h_state_[r].ctl;
            const rng::Mt& mt = h_state_[r].mt;
            long long d2h = sizeof(RepState);
            if (h_state_[r].bar[2]) {
                last_error = "device wait timed out in the batched kernel";
                st = MGK_DEVICE_TIMEOUT;
            }
            // hand the state back to the replica's engine (host mirrors)
            e.time_ = c.time;
            std::memcpy(e.eps_macro_, c.eps_macro, sizeof(c.eps_macro));
            std::memcpy(e.sig_macro_, c.sig_macro, sizeof(c.sig_macro));
            for (int k = 0; k < 3; ++k) e.ls_->w_[k] = c.w[k], e.ls_->asym_dev2_[k] = 0.0;
            e.batch_mt_.resize(626);
            std::memcpy(e.batch_mt_.data(), &mt, sizeof(rng::Mt));
            e.batch_started = true;
            e.batch_remaining = c.remaining;
            BatchStats& b = last_[r];
            b.events = c.events_done;
            b.cascades = c.cascades + (c.cascade_active ? 1 : 0);
            b.cascade_flips = c.cascade_flips;
            b.ls_solves = c.ls_solves;
            b.ls_iters = c.ls_iters;
            b.elastic_steps = c.elastic_steps;
            b.fallbacks = c.fallbacks;
            b.min_margin = c.min_margin;
            b.terminated = c.status;
            if (c.status == 2 && st == MGK_OK) {
                last_error = "batched run stopped at its time limit";
                st = MGK_TIME_LIMIT;
            }
            b.ncta = ncta_[r];
            b.sweeps = c.sweeps;
            for (int k = 0; k < 6; ++k) b.phase_ms[k] = 1e-6 * (double)c.ph_ns[k];
            {
                const long long ne = std::min<long long>(c.events_done, kSelLog);
                const unsigned long long* t = reinterpret_cast<const unsigned long long*>(h_logs_ + log_off[r]);
                d2h += (long long)sizeof(unsigned long long) * ne;
                b.event_us.resize(ne);
                for (long long i = 0; i < ne; ++i) b.event_us[i] = 1e-3 * (double)(t[i] - (i ? t[i - 1] : c.t_start_ns));
                const int* sel = reinterpret_cast<const int*>(h_logs_ + log_off[r] + sizeof(unsigned long long) * ne);
                b.sel.assign(sel, sel + c.sel_log_len);
            }
            d2h += (long long)sizeof(int) * c.sel_log_len;
            b.h2d_bytes = h2d_[r];
            b.d2h_bytes = d2h;
            e.stats_.thermal_events += c.events_done;
            e.stats_.ls_solves += c.ls_solves;
            e.stats_.ls_iters += c.ls_iters;
        }
        return st;
    } catch (const std::exception& ex) {
        last_error = ex.what();
        return MGK_CUDA_ERROR;
    }
}

}  // namespace mgk
