// The reference's random stream on the device, for the device-resident KMC
// kernel: one thread per replica continues the replica's std::mt19937 state.
//
// Algorithms restated (not copied): MT19937 (Matsumoto & Nishimura 1998);
// libstdc++ generate_canonical<double,53> over a 32-bit engine (two engine
// calls, r0 + r1*2^32, divided by 2^64, clamped below 1);
// uniform_real_distribution (u*(b-a)+a); normal_distribution (Marsaglia polar
// method, the second value of a pair cached in the distribution object);
// BarrierGenerator::generate (kmc_solver.hpp:35-95); the catalog modes of
// kmc_solver.hpp:231-238, 1042-1074.  Every operation uses explicit
// round-to-nearest intrinsics so the device rounds as the host build
// (-ffp-contract=off) does; only log/exp can differ from glibc's by an ulp.
#pragma once
#include "common.cuh"

namespace mgk {
namespace rng {

struct Mt {
    unsigned mt[624];
    int idx;
    int pad;
};

MGK_DEV void twist(Mt* g) {
    for (int i = 0; i < 624; ++i) {
        const unsigned y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
        g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    g->idx = 0;
}

MGK_DEV unsigned next(Mt* g) {
    if (g->idx >= 624) twist(g);
    unsigned y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

MGK_DEV double canonical(Mt* g) {
    const double lo = (double)next(g);
    const double hi = (double)next(g);
    const double sum = __dadd_rn(lo, __dmul_rn(hi, 4294967296.0));
    double r = __dmul_rn(sum, 5.42101086242752217e-20);  // 2^-64, exact scaling
    if (r >= 1.0) r = 0.99999999999999988898;           // nextafter(1, 0)
    return r;
}

MGK_DEV double uniform(Mt* g, double a, double b) { return __dadd_rn(__dmul_rn(canonical(g), __dsub_rn(b, a)), a); }

// one polar pair: returns the first value (y * mult), *second = x * mult
MGK_DEV double polar_pair(Mt* g, double* second) {
    double x, y, r2;
    do {
        x = __dsub_rn(__dmul_rn(2.0, canonical(g)), 1.0);
        y = __dsub_rn(__dmul_rn(2.0, canonical(g)), 1.0);
        r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    } while (r2 > 1.0 || r2 == 0.0);
    const double mult = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
    *second = __dmul_rn(x, mult);
    return __dmul_rn(y, mult);
}

MGK_DEV double scale(double z, double sd, double mean) { return __dadd_rn(__dmul_rn(z, sd), mean); }

struct Barrier {
    int type;
    double mean, std_val, min_cutoff, max_cutoff, loc, scale, epsilon, ratio;
};

MGK_DEV double mod_rayleigh(const Barrier& b, Mt* g) {
    double lo = __dsub_rn(b.mean, __dmul_rn(6.0, b.std_val));
    if (lo < 0.0) lo = 0.0;
    const double hi = __dadd_rn(b.mean, __dmul_rn(6.0, b.std_val));
    const double ss = __dmul_rn(__dmul_rn(2.0, b.std_val), b.std_val);
    const double xm =
        __ddiv_rn(__dadd_rn(b.mean, __dsqrt_rn(__dadd_rn(__dmul_rn(b.mean, b.mean),
                                                         __dmul_rn(__dmul_rn(4.0, b.std_val), b.std_val)))), 2.0);
    const double dm = __dsub_rn(xm, b.mean);
    const double cm = __dmul_rn(xm, exp(__ddiv_rn(-__dmul_rn(dm, dm), ss)));
    for (;;) {
        const double x = uniform(g, lo, hi);
        const double u = uniform(g, 0.0, cm);
        const double d = __dsub_rn(x, b.mean);
        const double pdf = __dmul_rn(x, exp(__ddiv_rn(-__dmul_rn(d, d), ss)));
        if (u < pdf) return x;
    }
}

MGK_DEV double barrier(const Barrier& b, Mt* g) {
    double v = 0.0;
    if (b.type == 0) {
        double unused;
        v = scale(polar_pair(g, &unused), b.std_val, b.mean);
    } else if (b.type == 1) {
        const double u = uniform(g, 0.0, 1.0);
        v = __dadd_rn(b.loc, __dmul_rn(b.scale, __dsqrt_rn(__dmul_rn(-2.0, log(__dsub_rn(1.0, u))))));
    } else if (b.type == 2) {
        v = mod_rayleigh(b, g);
    } else if (b.type == 3) {
        const double um = uniform(g, 0.0, 1.0);
        if (um < b.ratio) v = __dmul_rn(-b.epsilon, log(__dsub_rn(1.0, uniform(g, 0.0, 1.0))));
        else v = mod_rayleigh(b, g);
    }
    if (b.min_cutoff >= 0.0 && v < b.min_cutoff) v = b.min_cutoff;
    if (b.max_cutoff >= 0.0 && v > b.max_cutoff) v = b.max_cutoff;
    return v;
}

// A catalog mode into out (C = 2: gxx, gxy; C = 6: xx, yy, zz, xy, xz, yz).
// 2D and stz_mode_glass consume one polar pair per mode (gxx from the first
// value, gxy from the cached second); stz_mode_glass_3d nine normals (five
// pairs, the last cached value dropped) and, unless the matrix vanishes, one
// uniform in [1e-15, 1).
template <int C>
MGK_DEV void mode(Mt* g, double gamma0, double* out) {
    if (C == 2) {
        double second;
        const double first = polar_pair(g, &second);
        const double h = __dmul_rn(0.5, gamma0);
        out[0] = __dmul_rn(h, scale(first, 1.0, 0.0));
        out[1] = __dmul_rn(h, scale(second, 1.0, 0.0));
        return;
    }
    double m[9];
    for (int k = 0; k < 9; k += 2) {
        double second;
        m[k] = scale(polar_pair(g, &second), 1.0, 0.0);
        if (k + 1 < 9) m[k + 1] = scale(second, 1.0, 0.0);
    }
    double ms[9], G[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) ms[i * 3 + j] = __dmul_rn(0.5, __dadd_rn(m[i * 3 + j], m[j * 3 + i]));
    const double tr = __dadd_rn(__dadd_rn(ms[0], ms[4]), ms[8]);
    const double t3 = __dmul_rn(1.0 / 3.0, tr);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i * 3 + j] = __dsub_rn(ms[i * 3 + j], __dmul_rn(t3, i == j ? 1.0 : 0.0));
    double sq = 0.0;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) sq = __dadd_rn(sq, __dmul_rn(G[i * 3 + j], G[i * 3 + j]));
    const double nrm = __dsqrt_rn(sq);
    if (nrm < 1e-12) {
        for (int k = 0; k < 6; ++k) out[k] = 0.0;
        return;
    }
    const double f = __ddiv_rn(1.0, __dmul_rn(1.4142135623730951, nrm));
    for (int k = 0; k < 9; ++k) G[k] = __dmul_rn(G[k], f);
    const double u = uniform(g, 1e-15, 1.0);
    const double mag = __dmul_rn(gamma0, __dsqrt_rn(__dmul_rn(-2.0, log(u))));
    out[0] = __dmul_rn(G[0], mag);
    out[1] = __dmul_rn(G[4], mag);
    out[2] = __dmul_rn(G[8], mag);
    out[3] = __dmul_rn(G[1], mag);
    out[4] = __dmul_rn(G[2], mag);
    out[5] = __dmul_rn(G[5], mag);
}

}  // namespace rng
}  // namespace mgk

namespace mgk {
namespace rng {

// ---------------------------------------------------------------------------
// The same stream, drawn by a whole CTA.  MT19937's output sequence obeys
// x[n] = x[n-227] ^ T(x[n-624], x[n-623]) on the untempered words, so a CTA
// extends it 227 words per parallel step into a ring in shared memory.  A
// redraw program (the polar-method normals, uniforms and rejection draws of
// the catalog and barrier redraws, in the reference's order) then needs, per
// draw, only "where does the next accepted attempt start": the acceptance of
// every attempt offset is computed in parallel, one thread walks the program
// over those flags, and the values are computed in parallel per mode.
constexpr int kRingGens = 8;
constexpr int kRingWords = 624 * kRingGens;

struct MtRing {
    unsigned x[kRingWords];  // x[n % kRingWords] for n in [lo, hi)
    long long lo, hi;        // hi and lo are multiples of 624
    long long pos;           // next word to consume
};

MGK_DEV unsigned temper(unsigned y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

MGK_DEV unsigned ring_word(const MtRing* r, long long n) { return temper(r->x[n % kRingWords]); }

MGK_DEV double ring_canonical(const MtRing* r, long long n) {
    const double lo = (double)ring_word(r, n);
    const double hi = (double)ring_word(r, n + 1);
    double v = __dmul_rn(__dadd_rn(lo, __dmul_rn(hi, 4294967296.0)), 5.42101086242752217e-20);
    if (v >= 1.0) v = 0.99999999999999988898;
    return v;
}

// all threads: ring <- generator state g (words of the current generation at
// positions 0..623, next word at g->idx)
MGK_DEV void ring_load(MtRing* r, const Mt* g) {
    for (int i = threadIdx.x; i < 624; i += blockDim.x) r->x[i] = g->mt[i];
    if (threadIdx.x == 0) {
        r->lo = 0;
        r->hi = 624;
        r->pos = g->idx;
    }
    __syncthreads();
}

// all threads: generator state of the ring's position
MGK_DEV void ring_store(const MtRing* r, Mt* g) {
    const long long pos = r->pos;
    const long long gs = pos == 0 ? 0 : ((pos - 1) / 624) * 624;  // generation holding word pos-1
    for (int i = threadIdx.x; i < 624; i += blockDim.x) g->mt[i] = r->x[(gs + i) % kRingWords];
    if (threadIdx.x == 0) g->idx = (int)(pos - gs);
    __syncthreads();
}

// all threads: drop words no longer needed and extend the ring as far as it
// holds (whole generations).
MGK_DEV void ring_refill(MtRing* r) {
    __shared__ long long s_lo, s_hi;
    if (threadIdx.x == 0) {
        const long long pos = r->pos;
        const long long gs = pos == 0 ? 0 : ((pos - 1) / 624) * 624;
        long long lo = r->lo;
        const long long keep = min(gs, r->hi - 624);
        if (keep > lo) lo = keep;
        r->lo = lo;
        s_lo = lo;
        s_hi = r->hi;
    }
    __syncthreads();
    const long long target = s_lo + kRingWords;
    for (long long n0 = s_hi; n0 < target; n0 += 227) {
        const long long n1 = min(n0 + 227, target);
        for (long long n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
            const unsigned a = r->x[(n - 624) % kRingWords], b = r->x[(n - 623) % kRingWords];
            const unsigned y = (a & 0x80000000u) | (b & 0x7fffffffu);
            r->x[n % kRingWords] = r->x[(n - 227) % kRingWords] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) r->hi = target;
    __syncthreads();
}

// one thread: a uniform in [a, b) from the ring (the caller made sure two
// words are available)
MGK_DEV double ring_uniform(MtRing* r, double a, double b) {
    const double c = ring_canonical(r, r->pos);
    r->pos += 2;
    return __dadd_rn(__dmul_rn(c, __dsub_rn(b, a)), a);
}

// the polar attempt starting at word n: accepted?  (x from words n, n+1;
// y from n+2, n+3)
MGK_DEV bool polar_accepts(const MtRing* r, long long n) {
    const double x = __dsub_rn(__dmul_rn(2.0, ring_canonical(r, n)), 1.0);
    const double y = __dsub_rn(__dmul_rn(2.0, ring_canonical(r, n + 2)), 1.0);
    const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    return !(r2 > 1.0 || r2 == 0.0);
}

// the normals of the accepted polar attempt at word n: returns the first
// (y * mult), *second = x * mult
MGK_DEV double polar_at(const MtRing* r, long long n, double* second) {
    const double x = __dsub_rn(__dmul_rn(2.0, ring_canonical(r, n)), 1.0);
    const double y = __dsub_rn(__dmul_rn(2.0, ring_canonical(r, n + 2)), 1.0);
    const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    const double mult = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
    *second = __dmul_rn(x, mult);
    return __dmul_rn(y, mult);
}

// constants of the modified-Rayleigh rejection sampler (mod_rayleigh above)
struct RayleighK {
    double lo, hi, ss, cm;
};

MGK_DEV RayleighK rayleigh_k(const Barrier& b) {
    RayleighK k;
    k.lo = __dsub_rn(b.mean, __dmul_rn(6.0, b.std_val));
    if (k.lo < 0.0) k.lo = 0.0;
    k.hi = __dadd_rn(b.mean, __dmul_rn(6.0, b.std_val));
    k.ss = __dmul_rn(__dmul_rn(2.0, b.std_val), b.std_val);
    const double xm = __ddiv_rn(
        __dadd_rn(b.mean, __dsqrt_rn(__dadd_rn(__dmul_rn(b.mean, b.mean), __dmul_rn(__dmul_rn(4.0, b.std_val), b.std_val)))),
        2.0);
    const double dm = __dsub_rn(xm, b.mean);
    k.cm = __dmul_rn(xm, exp(__ddiv_rn(-__dmul_rn(dm, dm), k.ss)));
    return k;
}

// the rejection attempt at word n (x from n, n+1; u from n+2, n+3): accepted?
// *x gets the candidate
MGK_DEV bool rayleigh_accepts(const MtRing* r, long long n, const Barrier& b, const RayleighK& k, double* xo) {
    const double x = __dadd_rn(__dmul_rn(ring_canonical(r, n), __dsub_rn(k.hi, k.lo)), k.lo);
    const double u = __dadd_rn(__dmul_rn(ring_canonical(r, n + 2), __dsub_rn(k.cm, 0.0)), 0.0);
    const double d = __dsub_rn(x, b.mean);
    const double pdf = __dmul_rn(x, exp(__ddiv_rn(-__dmul_rn(d, d), k.ss)));
    *xo = x;
    return u < pdf;
}

}  // namespace rng
}  // namespace mgk
