// Batched in-CTA FFTs for the Lippmann-Schwinger passes.
//
// Lines of length n sit in shared memory at a padded stride: element e of line
// l is at buf[l * pad_len(n) + pad_idx(e)], one spare slot after every 8
// elements, so the radix-strided 16-byte accesses of a stage spread over the
// banks.
// Each stage is a mixed-radix Stockham step (out-of-place between two shared
// buffers, natural-order output): stage s with radix R and Ns = product of the
// radices before it maps input element j + r*(n/R) through the twiddle
// w^(r*(j mod Ns)), w = exp(sign*2*pi*i/(Ns*R)), a radix-R DFT, and writes to
// (j/Ns)*Ns*R + (j mod Ns) + r*Ns.  Twiddles come from a per-length table
// tw[t] = exp(-2*pi*i*t/n) computed on the host in long double.
#pragma once
#include "common.cuh"

namespace mgk {

constexpr int kMaxStages = 24;

struct FftAxis {
    int n;
    int nst;
    int lw;  // lines a warp transforms together (warp-owned path, n <= kWarpFftMax)
    int pad;
    int radix[kMaxStages];
    const cplx<double>* tw64;  // length n
    const cplx<float>* tw32;   // length n
};

// Longest line the warp-owned transforms take; longer lines use the CTA-wide
// path (fft_lines).
constexpr int kWarpFftMax = 512;

// Lines of length n a warp transforms together: enough that every stage has
// at least 32 butterflies when n is small (1 for n >= 256); 0 when n is too
// long for the warp-owned path.
__host__ __device__ inline int warp_lines(const FftAxis& a) {
    if (a.n > kWarpFftMax) return 0;
    int lw = 1;
    while (lw * a.n < 256) lw *= 2;
    return lw;
}

template <typename T>
MGK_DEV const cplx<T>* tw_of(const FftAxis& a);
template <>
MGK_DEV const cplx<double>* tw_of<double>(const FftAxis& a) { return a.tw64; }
template <>
MGK_DEV const cplx<float>* tw_of<float>(const FftAxis& a) { return a.tw32; }

// multiply by sign*i: (x + iy) * (s*i) = -s*y + i*s*x
template <typename T>
MGK_DEV cplx<T> mul_si(cplx<T> a, int sign) {
    return sign < 0 ? cplx<T>{a.y, -a.x} : cplx<T>{-a.y, a.x};
}

template <typename T, int R>
MGK_DEV void small_dft(cplx<T>* v, int sign, const cplx<T>* tw, int n) {
    if constexpr (R == 2) {
        cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const T h = T(0.86602540378443864676372317075294);  // sqrt(3)/2
        cplx<T> t = cadd(v[1], v[2]);
        cplx<T> m = {v[0].x - T(0.5) * t.x, v[0].y - T(0.5) * t.y};
        cplx<T> d = mul_si(csub(v[1], v[2]), sign);
        d = cscale(d, h);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, d);
        v[2] = csub(m, d);
    } else if constexpr (R == 4) {
        cplx<T> t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        cplx<T> t2 = cadd(v[1], v[3]), t3 = mul_si(csub(v[1], v[3]), sign);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if constexpr (R == 8) {
        // two radix-4 layers with the internal 8-point twiddles
        const T r2 = T(0.70710678118654752440084436210485);
        cplx<T> a[4] = {v[0], v[2], v[4], v[6]}, b[4] = {v[1], v[3], v[5], v[7]};
        small_dft<T, 4>(a, sign, tw, n);
        small_dft<T, 4>(b, sign, tw, n);
        // b[k] *= exp(sign*2*pi*i*k/8)
        cplx<T> w1 = {r2, T(sign) * r2}, w3 = {-r2, T(sign) * r2};
        b[1] = cmul(b[1], w1);
        b[2] = mul_si(b[2], sign);
        b[3] = cmul(b[3], w3);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = cadd(a[k], b[k]);
            v[k + 4] = csub(a[k], b[k]);
        }
    } else {
        // direct DFT using the length-n table: exp(sign*2*pi*i*jk/R) = tw[(jk mod R) * n/R]^(sign)
        cplx<T> out[R];
        const int step = n / R;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            cplx<T> acc = v[0];
#pragma unroll
            for (int j = 1; j < R; ++j) {
                cplx<T> w = tw[((j * k) % R) * step];
                if (sign > 0) w = cconj(w);
                acc = cadd(acc, cmul(v[j], w));
            }
            out[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = out[k];
    }
}

MGK_DEV int pad_idx(int e) { return e + (e >> 3); }
MGK_DEV int pad_len(int n) { return n + (n >> 3) + 1; }

template <typename T, int R>
MGK_DEV void fft_stage(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, int nlines, int n, int Ns,
                       const cplx<T>* __restrict__ tw, int sign) {
    const int m = n / R;
    const int tstep = n / (Ns * R);
    const int total = nlines * m;
    const int ls = pad_len(n);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int l = idx / m, j = idx - l * m;
        const cplx<T>* src = in + l * ls;
        cplx<T>* dst = out + l * ls;
        const int k = j % Ns;
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[pad_idx(j + r * m)];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cplx<T> w = tw[r * k * tstep];
                if (sign > 0) w = cconj(w);
                v[r] = cmul(v[r], w);
            }
        }
        small_dft<T, R>(v, sign, tw, n);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[pad_idx(d + r * Ns)] = v[r];
    }
}

// Runs all stages of `ax` over `nlines` lines held in `a`; `b` is scratch of the
// same size.  Returns the buffer that holds the result.  Contains __syncthreads.
// tw_s: a shared-memory copy of the axis twiddle table (load_twiddles), or
// null to read the table from global memory.
template <typename T>
__device__ __noinline__ cplx<T>* fft_lines(cplx<T>* a, cplx<T>* b, int nlines, const FftAxis& ax, int sign,
                                           const cplx<T>* tw_s = nullptr) {
    const cplx<T>* tw = tw_s ? tw_s : tw_of<T>(ax);
    int Ns = 1;
    for (int s = 0; s < ax.nst; ++s) {
        const int R = ax.radix[s];
        switch (R) {
            case 2: fft_stage<T, 2>(a, b, nlines, ax.n, Ns, tw, sign); break;
            case 3: fft_stage<T, 3>(a, b, nlines, ax.n, Ns, tw, sign); break;
            case 4: fft_stage<T, 4>(a, b, nlines, ax.n, Ns, tw, sign); break;
            case 5: fft_stage<T, 5>(a, b, nlines, ax.n, Ns, tw, sign); break;
            case 7: fft_stage<T, 7>(a, b, nlines, ax.n, Ns, tw, sign); break;
            case 8: fft_stage<T, 8>(a, b, nlines, ax.n, Ns, tw, sign); break;
            default: break;  // host planner only emits the radices above
        }
        Ns *= R;
        cplx<T>* t = a;
        a = b;
        b = t;
        __syncthreads();
    }
    return a;
}

// ---------------------------------------------------------------- warp-owned transforms
// One Stockham stage (the arithmetic of fft_stage) of `cnt` lines of length
// n owned by one warp: lane after lane takes a butterfly, reads its R inputs
// from `in`, writes its R outputs to their autosorted positions in `out`, and
// the warp synchronises at the end.  tw is a shared-memory copy of the axis
// table.
template <typename T, int R>
MGK_DEV void warp_stage(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, int lsn, int cnt, int n, int Ns,
                        const cplx<T>* __restrict__ tw, int sign) {
    const int m = n / R;
    const int nb = cnt * m;
    const int tstep = n / (Ns * R);
    for (int b = threadIdx.x & 31; b < nb; b += 32) {
        const int l = b / m, j = b - l * m;
        const cplx<T>* src = in + l * lsn;
        cplx<T>* dst = out + l * lsn;
        const int k = j % Ns;
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[pad_idx(j + r * m)];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cplx<T> w = tw[r * k * tstep];
                if (sign > 0) w = cconj(w);
                v[r] = cmul(v[r], w);
            }
        }
        small_dft<T, R>(v, sign, tw, n);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[pad_idx(d + r * Ns)] = v[r];
    }
    __syncwarp();
}

// All stages of `nlines` lines (stride lsn) held in a, with b as the second
// buffer: each group of ax.lw lines is transformed by one warp, the warps of
// the CTA taking the groups in turn, so the stages need no CTA barrier.
// Returns the buffer holding the result (a after an even number of stages,
// else b, for every line).  The caller synchronises the CTA before other
// warps read the lines.  One out-of-line copy per type keeps the persistent
// kernels' code small.
template <typename T>
__device__ __noinline__ cplx<T>* fft_lines_warp(cplx<T>* a, cplx<T>* b, int nlines, int lsn, const FftAxis& ax,
                                                const cplx<T>* tw, int sign) {
    const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int lw = ax.lw;
    const int ngroups = (nlines + lw - 1) / lw;
    for (int g = wid; g < ngroups; g += nw) {
        const int l0 = g * lw;
        const int cnt = min(lw, nlines - l0);
        cplx<T>* x = a + l0 * lsn;
        cplx<T>* y = b + l0 * lsn;
        int Ns = 1;
        for (int s = 0; s < ax.nst; ++s) {
            const int R = ax.radix[s];
            switch (R) {
                case 2: warp_stage<T, 2>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                case 3: warp_stage<T, 3>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                case 4: warp_stage<T, 4>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                case 5: warp_stage<T, 5>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                case 7: warp_stage<T, 7>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                case 8: warp_stage<T, 8>(x, y, lsn, cnt, ax.n, Ns, tw, sign); break;
                default: break;
            }
            Ns *= R;
            cplx<T>* t = x;
            x = y;
            y = t;
        }
    }
    return (ax.nst & 1) ? b : a;
}

// Copies the axis twiddle table to shared memory (both transform paths read
// it there); the caller synchronises before use.
template <typename T>
MGK_DEV void load_twiddles(const FftAxis& ax, cplx<T>* tw_s) {
    const cplx<T>* tw = tw_of<T>(ax);
    for (int i = threadIdx.x; i < ax.n; i += blockDim.x) tw_s[i] = tw[i];
}

// Transform of `nlines` lines starting at a, with b as the second buffer:
// warp-owned when the axis allows it, else CTA-wide.  Returns the buffer
// holding the result.  The caller synchronises the CTA after it.
template <typename T>
MGK_DEV cplx<T>* fft_any(cplx<T>* a, cplx<T>* b, int nlines, const FftAxis& ax, const cplx<T>* tw_s, int sign) {
    if (ax.lw > 0) return fft_lines_warp<T>(a, b, nlines, pad_len(ax.n), ax, tw_s, sign);
    return fft_lines<T>(a, b, nlines, ax, sign, tw_s);
}

}  // namespace mgk
