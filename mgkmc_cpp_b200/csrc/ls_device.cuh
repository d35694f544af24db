// Device functions of the Lippmann-Schwinger solve, shared by the one-solve
// kernel (ls.cu) and the device-resident KMC kernel (batch.cu).  Every pass is
// parametrised by the CTA's rank in its group and the group size, so a group
// of CTAs can run the solve inside a larger launch.  See ls.cu for the
// reference semantics kept and the arithmetic differences.
#pragma once
#include "ls.cuh"

namespace mgk {
namespace lsdev {

__host__ __device__ inline int n_sym(int D) { return D == 2 ? 3 : 6; }

// symmetric component index of tensor entry (i, j): 2D {xx, yy, xy},
// 3D {xx, yy, zz, xy, xz, yz}
__host__ __device__ inline int sym_idx(int D, int i, int j) {
    if (i == j) return i;
    if (D == 2) return 2;
    int a = i < j ? i : j, b = i < j ? j : i;
    return (a == 0 && b == 1) ? 3 : (a == 0 ? 4 : 5);
}

MGK_DEV double kfreq(int i, int n, double pixel) {
    // 2*pi*fftfreq(n, pixel)[i], as init_gamma builds it (kmc_solver.hpp:259-274)
    const int lim = (n + 1) / 2;
    const double f = (i < lim) ? (double)i / (n * pixel) : (double)(i - n) / (n * pixel);
    return 2.0 * 3.14159265358979323846 * f;
}

// eps_hat = -Gamma0(q) : tau_hat for the symmetric components (in place).
template <int D, typename T>
MGK_DEV void green_q(const double* qd, cplx<T>* t, double inv2mu0, double bcoef) {
    constexpr int S = D == 2 ? 3 : 6;
    T q[D];
    T k2 = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        q[i] = (T)qd[i];
        k2 += q[i] * q[i];
    }
    if (k2 == T(0)) {
#pragma unroll
        for (int c = 0; c < S; ++c) t[c] = {T(0), T(0)};
        return;
    }
    cplx<T> v[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        cplx<T> acc = {T(0), T(0)};
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const cplx<T> tij = t[sym_idx(D, i, j)];
            acc.x += tij.x * q[j];
            acc.y += tij.y * q[j];
        }
        v[i] = acc;
    }
    cplx<T> qv = {T(0), T(0)};
#pragma unroll
    for (int i = 0; i < D; ++i) {
        qv.x += q[i] * v[i].x;
        qv.y += q[i] * v[i].y;
    }
    const T a = T(inv2mu0) / k2, b = T(bcoef) / (k2 * k2);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = i; j < D; ++j) {
            const int c = sym_idx(D, i, j);
            const T qq = b * q[i] * q[j];
            t[c].x = -(a * (q[j] * v[i].x + q[i] * v[j].x) - qq * qv.x);
            t[c].y = -(a * (q[j] * v[i].y + q[i] * v[j].y) - qq * qv.y);
        }
}

// Hermitian-averaged Green application (see the header comment): averages over
// the sign of every Nyquist component of q.
template <int D, typename T>
MGK_DEV void green_apply(const double* q, const bool* nyq, cplx<T>* t, double inv2mu0, double bcoef) {
    constexpr int S = D == 2 ? 3 : 6;
    bool any = false;
#pragma unroll
    for (int i = 0; i < D; ++i) any |= nyq[i];
    if (!any) {
        green_q<D, T>(q, t, inv2mu0, bcoef);
        return;
    }
    cplx<T> t0[S], t1[S];
    double q1[D];
#pragma unroll
    for (int c = 0; c < S; ++c) t0[c] = t1[c] = t[c];
#pragma unroll
    for (int i = 0; i < D; ++i) q1[i] = nyq[i] ? -q[i] : q[i];
    green_q<D, T>(q, t0, inv2mu0, bcoef);
    green_q<D, T>(q1, t1, inv2mu0, bcoef);
#pragma unroll
    for (int c = 0; c < S; ++c) t[c] = {T(0.5) * (t0[c].x + t1[c].x), T(0.5) * (t0[c].y + t1[c].y)};
}

MGK_DEV void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Shared-memory layout of a pass: the two line buffers at 0 and smem_half,
// the axis twiddle table at tw_off.
template <typename T>
struct PassSmem {
    cplx<T>* buf0;
    cplx<T>* buf1;
    cplx<T>* tw;
};
template <typename T>
MGK_DEV PassSmem<T> pass_smem(const LsArgs& a, unsigned char* smem) {
    return {reinterpret_cast<cplx<T>*>(smem), reinterpret_cast<cplx<T>*>(smem + a.smem_half),
            reinterpret_cast<cplx<T>*>(smem + a.tw_off)};
}

// Row pass along the contiguous axis.  MODE 0 (prologue): set the field (warm
// shift or fill), build tau, forward transform.  MODE 1 (iteration): inverse
// transform of the Green-filtered spectrum, strain update with norms and
// macro sums, then tau of the new field and its forward transform.  A chunk
// of rpb rows holds its S * rpb real lines packed two per complex line; the
// transforms are warp-owned (fft_any), so a chunk needs four CTA barriers.
template <int D, typename T, int MODE>
MGK_DEV void row_pass(const LsArgs& a, int cta, int ncta, unsigned char* smem, double* part, const double* shift) {
    constexpr int S = D == 2 ? 3 : 6;
    const int n = a.nr, nh = a.nh, N = a.N;
    cplx<T>* spec = reinterpret_cast<cplx<T>*>(a.spec);
    const long cs = (long)a.nrows * a.nhs;
    const int nchunks = (a.nrows + a.rpb - 1) / a.rpb;
    const FftAxis& ax = a.ax[D - 1];
    const int lsn = pad_len(n);
    const PassSmem<T> sm = pass_smem<T>(a, smem);
    load_twiddles<T>(ax, sm.tw);
    for (int ch = cta; ch < nchunks; ch += ncta) {
        const int row0 = ch * a.rpb;
        const int rows = min(a.rpb, a.nrows - row0);
        const int L = rows * S;        // real lines in this chunk
        const int P = (L + 1) >> 1;    // packed complex lines
        const long v0 = (long)row0 * n;
        cplx<T>* z = sm.buf0;
        cplx<T>* other = sm.buf1;
        if (MODE == 1) {
            // the update's operands go to L1 while the spectrum is loaded and
            // transformed (the chunk's rows are contiguous in every array)
            for (int o = threadIdx.x * 16; o < rows * n; o += blockDim.x * 16) {
#pragma unroll
                for (int c = 0; c < S; ++c) {
                    prefetch_l1(a.eps_s + (long)c * N + v0 + o);
                    if (a.epsp_s) prefetch_l1(a.epsp_s + (long)c * N + v0 + o);
                }
                prefetch_l1(a.lam + v0 + o);
                prefetch_l1(a.mu + v0 + o);
            }
            for (int idx = threadIdx.x; idx < P * n; idx += blockDim.x) {
                const int p = idx / n, k = idx - p * n;
                const bool hi = 2 * k > n;
                const int kk = hi ? n - k : k;
                const int la = 2 * p, lb = 2 * p + 1;
                cplx<T> A = spec[(la % S) * cs + (long)(row0 + la / S) * a.nhs + kk];
                cplx<T> B = {T(0), T(0)};
                if (lb < L) B = spec[(lb % S) * cs + (long)(row0 + lb / S) * a.nhs + kk];
                if (hi) {
                    A = cconj(A);
                    B = cconj(B);
                }
                z[p * lsn + pad_idx(k)] = {A.x - B.y, A.y + B.x};
            }
            __syncthreads();
            z = fft_any<T>(sm.buf0, sm.buf1, P, ax, sm.tw, +1);
            other = (z == sm.buf0) ? sm.buf1 : sm.buf0;
            __syncthreads();
        }
        for (int idx = threadIdx.x; idx < rows * n; idx += blockDim.x) {
            const int r = idx / n, y = idx - r * n;
            const long v = v0 + idx;
            double sn[S];
#pragma unroll
            for (int c = 0; c < S; ++c) {
                const double so = a.eps_s[(long)c * N + v];
                if (MODE == 1) {
                    const int l = r * S + c;
                    const cplx<T> zz = z[(l >> 1) * lsn + pad_idx(y)];
                    const double et = (double)((l & 1) ? zz.y : zz.x) * a.inv_n;
                    sn[c] = a.ebar_s[c] + et;
                    const double wc = c < D ? 1.0 : 2.0;
                    const double d = sn[c] - so;
                    part[0] += wc * d * d;
                    part[1] += wc * so * so;
                } else {
                    sn[c] = a.warm ? so + shift[c] : a.ebar_s[c];
                }
                a.eps_s[(long)c * N + v] = sn[c];
            }
            const double lam = a.lam[v], mu = a.mu[v];
            double e[S];
#pragma unroll
            for (int c = 0; c < S; ++c) e[c] = a.epsp_s ? sn[c] - a.epsp_s[(long)c * N + v] : sn[c];
            double tr = 0.0, tr0 = 0.0;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                tr += e[c];
                tr0 += sn[c];
            }
#pragma unroll
            for (int c = 0; c < S; ++c) {
                const double sig = 2.0 * mu * e[c] + (c < D ? lam * tr : 0.0);
                const double sig0 = 2.0 * a.mu0 * sn[c] + (c < D ? a.lam0 * tr0 : 0.0);
                part[2 + c] += sn[c];
                part[2 + S + c] += sig;
                const int l = r * S + c;
                cplx<T>* cell = &z[(l >> 1) * lsn + pad_idx(y)];
                if (l & 1) {
                    cell->y = (T)(sig - sig0);
                } else {
                    cell->x = (T)(sig - sig0);
                    if (l + 1 == L) cell->y = T(0);
                }
            }
        }
        __syncthreads();
        cplx<T>* Z = fft_any<T>(z, other, P, ax, sm.tw, -1);
        __syncthreads();
        for (int idx = threadIdx.x; idx < P * nh; idx += blockDim.x) {
            const int p = idx / nh, k = idx - p * nh;
            const cplx<T> zk = Z[p * lsn + pad_idx(k)];
            const cplx<T> zm = cconj(Z[p * lsn + pad_idx(k == 0 ? 0 : n - k)]);
            const int la = 2 * p, lb = 2 * p + 1;
            const cplx<T> A = {T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y + zm.y)};
            spec[(la % S) * cs + (long)(row0 + la / S) * a.nhs + k] = A;
            if (lb < L) {
                const cplx<T> B = {T(0.5) * (zk.y - zm.y), T(-0.5) * (zk.x - zm.x)};
                spec[(lb % S) * cs + (long)(row0 + lb / S) * a.nhs + k] = B;
            }
        }
        __syncthreads();
    }
}

// Strided pass along axis `axis` (not the contiguous one) over tiles of tk
// adjacent half-spectrum columns.  KIND 0: forward only; 1: inverse only;
// 2: forward, Green operator, inverse (the last non-contiguous axis, x).
template <int D, typename T, int KIND>
MGK_DEV void strided_pass(const LsArgs& a, int cta, int ncta, int axis, unsigned char* smem) {
    constexpr int S = D == 2 ? 3 : 6;
    const int nh = a.nh;
    const int n = a.dims[axis];
    cplx<T>* spec = reinterpret_cast<cplx<T>*>(a.spec);
    const long cs = (long)a.nrows * a.nhs;
    long st, os;
    int no;
    if (D == 2) {
        st = a.nhs; no = 1; os = 0;
    } else if (axis == 1) {
        st = a.nhs; no = a.dims[0]; os = (long)a.dims[1] * a.nhs;
    } else {
        st = (long)a.dims[1] * a.nhs; no = a.dims[1]; os = a.nhs;
    }
    const int tk = a.tk;
    const int ntk = (nh + tk - 1) / tk;
    const int items = no * ntk;
    const int nl = S * tk;
    const FftAxis& fx = a.ax[axis];
    const int lsn = pad_len(n);
    const PassSmem<T> sm = pass_smem<T>(a, smem);
    load_twiddles<T>(fx, sm.tw);
    for (int it = cta; it < items; it += ncta) {
        const int o = it / ntk;
        const int k0 = (it - o * ntk) * tk;
        const int tku = min(tk, nh - k0);
        const long base = o * os + k0;
        for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
            const int t = idx % tk;
            const int i = (idx / tk) % n;
            const int c = idx / (tk * n);
            sm.buf0[(c * tk + t) * lsn + pad_idx(i)] = (t < tku) ? spec[c * cs + base + t + i * st] : cplx<T>{T(0), T(0)};
        }
        __syncthreads();
        cplx<T>* Z = fft_any<T>(sm.buf0, sm.buf1, nl, fx, sm.tw, KIND == 1 ? +1 : -1);
        __syncthreads();
        if (KIND == 2) {
            for (int idx = threadIdx.x; idx < tku * n; idx += blockDim.x) {
                const int t = idx / n, kx = idx - t * n;
                double q[3];
                bool nyq[3];
                q[0] = kfreq(kx, a.dims[0], a.pixel);
                nyq[0] = (a.dims[0] % 2 == 0) && (2 * kx == a.dims[0]);
                if (D == 2) {
                    const int ky = k0 + t;
                    q[1] = kfreq(ky, a.dims[1], a.pixel);
                    nyq[1] = (a.dims[1] % 2 == 0) && (2 * ky == a.dims[1]);
                } else {
                    const int ky = o, kz = k0 + t;
                    q[1] = kfreq(ky, a.dims[1], a.pixel);
                    nyq[1] = (a.dims[1] % 2 == 0) && (2 * ky == a.dims[1]);
                    q[2] = kfreq(kz, a.dims[2], a.pixel);
                    nyq[2] = (a.dims[2] % 2 == 0) && (2 * kz == a.dims[2]);
                }
                cplx<T> tv[S];
#pragma unroll
                for (int c = 0; c < S; ++c) tv[c] = Z[(c * tk + t) * lsn + pad_idx(kx)];
                green_apply<D, T>(q, nyq, tv, a.inv2mu0, a.bcoef);
#pragma unroll
                for (int c = 0; c < S; ++c) Z[(c * tk + t) * lsn + pad_idx(kx)] = tv[c];
            }
            __syncthreads();
            cplx<T>* other = (Z == sm.buf0) ? sm.buf1 : sm.buf0;
            Z = fft_any<T>(Z, other, nl, fx, sm.tw, +1);
            __syncthreads();
        }
        for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
            const int t = idx % tk;
            const int i = (idx / tk) % n;
            const int c = idx / (tk * n);
            if (t < tku) spec[c * cs + base + t + i * st] = Z[(c * tk + t) * lsn + pad_idx(i)];
        }
        __syncthreads();
    }
}

template <int NP>
MGK_DEV void publish_partials(const LsArgs& a, int cta, double* part, double* red) {
    block_sum<NP>(part, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NP; ++k) a.partials[cta * kMaxPartials + k] = part[k];
}

// Every CTA reduces all partials in the same fixed order -> identical values:
// thread t sums value (t & 15) over CTAs (t >> 4), (t >> 4) + 16, ..., then
// the 16 group sums are added in group order.  256 threads per CTA.  (Reducing
// once, in the last CTA to reach the barrier, and reading the sums back was
// measured slower: one more L2 round trip on the critical path.)
template <int NP>
MGK_DEV void gather_partials(const LsArgs& a, int ncta, double* out /* shared, NP */, double* grp /* shared, 256 */) {
    const int k = threadIdx.x & 15, g = threadIdx.x >> 4;
    double s = 0.0;
    if (k < NP) {
#pragma unroll 4
        for (int b = g; b < ncta; b += 16) s += __ldcg(&a.partials[b * kMaxPartials + k]);
    }
    grp[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < NP) {
        double t = 0.0;
        for (int gg = 0; gg < 16; ++gg) t += grp[gg * 16 + threadIdx.x];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

// One LS solve by a group of ncta co-resident CTAs (rank cta), synchronised by
// the bounded barrier `gb`; smem_raw is the CTA's dynamic shared memory (the
// pass layout of pass_smem).  The result goes to a.result.  Returns false
// when a barrier wait gave up (the error word is set).
template <int D, typename T>
MGK_DEV bool ls_solve_group(const LsArgs& a, int cta, int ncta, const GridBar& gb, unsigned char* smem_raw) {
    constexpr int S = D == 2 ? 3 : 6;
    constexpr int NP = 2 + 2 * S;
    double* red = reinterpret_cast<double*>(smem_raw + a.scr_off);  // 14 x 32
    double* grp = red + 14 * 32;                                    // 256
    double* vals = grp + 256;                                       // 16
    double* s_shift = vals + 16;                                    // 8
    // fault injection (set from the host for tests): this CTA never arrives,
    // so the others' bounded waits run out and they return with the error set
    if (a.test_absent == cta + 1) return false;
    double shift[6] = {0, 0, 0, 0, 0, 0};
    if (a.warm) {
        double acc[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) acc[k] = 0.0;
        const int nchunks = (a.nrows + a.rpb - 1) / a.rpb;
        for (int ch = cta; ch < nchunks; ch += ncta) {
            const long v0 = (long)ch * a.rpb * a.nr;
            const long v1 = min((long)a.N, v0 + (long)a.rpb * a.nr);
            for (long v = v0 + threadIdx.x; v < v1; v += blockDim.x)
#pragma unroll
                for (int c = 0; c < S; ++c) acc[c] += a.eps_s[(long)c * a.N + v];
        }
        publish_partials<NP>(a, cta, acc, red);
        if (!grid_sync(gb)) return false;
        gather_partials<NP>(a, ncta, vals, grp);
        if (threadIdx.x < S) s_shift[threadIdx.x] = a.ebar_s[threadIdx.x] - vals[threadIdx.x] * a.inv_n;
        __syncthreads();
#pragma unroll
        for (int c = 0; c < S; ++c) shift[c] = s_shift[c];
        // the row pass below publishes new partials: every CTA must have read these first
        if (!grid_sync(gb)) return false;
    }
    double part[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) part[k] = 0.0;
    row_pass<D, T, 0>(a, cta, ncta, smem_raw, part, shift);
    publish_partials<NP>(a, cta, part, red);
    if (!grid_sync(gb)) return false;
        gather_partials<NP>(a, ncta, vals, grp);
    int it = 0;
    double diff = 0.0;
    while (it < a.max_iter) {
        if (D == 3) {
            strided_pass<D, T, 0>(a, cta, ncta, 1, smem_raw);
            if (!grid_sync(gb)) return false;
        }
        strided_pass<D, T, 2>(a, cta, ncta, 0, smem_raw);
        if (!grid_sync(gb)) return false;
        if (D == 3) {
            strided_pass<D, T, 1>(a, cta, ncta, 1, smem_raw);
            if (!grid_sync(gb)) return false;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) part[k] = 0.0;
        row_pass<D, T, 1>(a, cta, ncta, smem_raw, part, shift);
        publish_partials<NP>(a, cta, part, red);
        if (!grid_sync(gb)) return false;
        gather_partials<NP>(a, ncta, vals, grp);
        const double dx = it == 0 ? a.diff_extra_first : 0.0;
        const double nx = it == 0 ? a.norm_extra_first : a.norm_extra;
        ++it;
        diff = sqrt(vals[0] + dx) / (sqrt(vals[1] + nx) + 1e-20);
        if (diff < a.tol) break;
    }
    if (cta == 0 && threadIdx.x == 0) {
        a.result->iters = it;
        a.result->diff = diff;
        for (int c = 0; c < S; ++c) {
            a.result->sum_s[c] = vals[2 + c];
            a.result->sum_sig[c] = vals[2 + S + c];
        }
    }
    return true;
}

}  // namespace lsdev
}  // namespace mgk
