// Device functions of the KMC step shared by the per-event kernels
// (kmc_kernels.cu) and the device-resident batched kernel (batch.cu).
#pragma once
#include "kmc_kernels.cuh"

namespace mgk {
namespace kmcdev {

__host__ __device__ inline int sidx(int D, int i, int j) {
    if (i == j) return i;
    if (D == 2) return 2;
    int a = i < j ? i : j, b = i < j ? j : i;
    return (a == 0 && b == 1) ? 3 : (a == 0 ? 4 : 5);
}

// catalog entry -> symmetric components (S)
template <int D, int C>
MGK_DEV void cat_sym(const double* c, double* o) {
    constexpr int S = D == 2 ? 3 : 6;
#pragma unroll
    for (int k = 0; k < S; ++k) o[k] = 0.0;
    if (C == 2) {
        o[0] = c[0];
        o[1] = -c[0];
        o[sidx(D, 0, 1)] = c[1];
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) o[k] = c[k];
    }
}

// Stress of voxel v from the LS strain (stress_from_strain_2d/3d,
// linear_elastic_solver.hpp:48-67 / :322-341), symmetric components.
template <int D>
MGK_DEV void voxel_stress(const KmcDevState& s, int v, double* sg) {
    constexpr int S = D == 2 ? 3 : 6;
    const int N = s.N;
    double e[S];
#pragma unroll
    for (int c = 0; c < S; ++c) e[c] = s.eps_s[(long)c * N + v] - s.epsp_s[(long)c * N + v];
    double tr = 0.0;
#pragma unroll
    for (int c = 0; c < D; ++c) tr += e[c];
    const double m2 = 2.0 * s.mu[v], l = s.lam[v];
#pragma unroll
    for (int c = 0; c < S; ++c) sg[c] = m2 * e[c] + (c < D ? l * tr : 0.0);
}

// Voxel of flat mode index i (i < NM): a 32-bit division whenever the mode
// count fits in 32 bits (the same quotient), the 64-bit one otherwise.
MGK_DEV int voxel_of(long i, long NM, int M) {
    return NM <= 0xffffffffL ? (int)((unsigned)i / (unsigned)M) : (int)(i / M);
}

// Shear of magnitude gamma0 on the plane of normal n along the largest
// resolved shear traction tau = sigma n - (n . sigma n) n (where tau vanishes,
// along the projection of x -- or y when n is near x -- onto the plane);
// symmetric components of (gamma0 / 2)(s n + n s).  sg: symmetric stress
// {xx, yy, zz, xy, xz, yz}.  The catalog extension "fibonacci" (no
// counterpart in the reference).
MGK_DEV void fib_mode(const double* sg, const double* n, double gamma0, double* o) {
    const double sf[9] = {sg[0], sg[3], sg[4], sg[3], sg[1], sg[5], sg[4], sg[5], sg[2]};
    double t[3], tau[3], sv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) t[i] = sf[3 * i] * n[0] + sf[3 * i + 1] * n[1] + sf[3 * i + 2] * n[2];
    const double tn = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
    double tt = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        tau[i] = t[i] - tn * n[i];
        tt += tau[i] * tau[i];
    }
    if (tt > 0.0) {
        const double inv = 1.0 / sqrt(tt);
#pragma unroll
        for (int i = 0; i < 3; ++i) sv[i] = tau[i] * inv;
    } else {
        double e[3] = {0.0, 0.0, 0.0};
        e[fabs(n[0]) < 0.9 ? 0 : 1] = 1.0;
        const double d = e[0] * n[0] + e[1] * n[1] + e[2] * n[2];
        double q = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            sv[i] = e[i] - d * n[i];
            q += sv[i] * sv[i];
        }
        const double inv = 1.0 / sqrt(q);
#pragma unroll
        for (int i = 0; i < 3; ++i) sv[i] *= inv;
    }
    const double h = 0.5 * gamma0;
    o[0] = h * (sv[0] * n[0] + n[0] * sv[0]);
    o[1] = h * (sv[1] * n[1] + n[1] * sv[1]);
    o[2] = h * (sv[2] * n[2] + n[2] * sv[2]);
    o[3] = h * (sv[0] * n[1] + n[0] * sv[1]);
    o[4] = h * (sv[0] * n[2] + n[0] * sv[2]);
    o[5] = h * (sv[1] * n[2] + n[1] * sv[2]);
}

// Symmetric components of mode i (of voxel v, stress sg) now: the catalog
// entry, or the stress-dependent shear of the mode's plane.
template <int D, int C>
MGK_DEV void mode_eps(const KmcDevState& s, int v, long i, const double* sg, double* cs) {
    if (D == 3 && s.normals) {
        const int m = (int)(i - (long)v * s.M);
        fib_mode(sg, s.normals + 3 * m, s.gamma0, cs);
    } else {
        cat_sym<D, C>(s.cat + i * C, cs);
    }
}

// Stress of voxel v as the sweep reads it (the kept field with fast patching)
template <int D>
MGK_DEV void sweep_stress(const KmcDevState& s, int v, double* sg) {
    constexpr int S = D == 2 ? 3 : 6;
    if (s.sig_s) {
#pragma unroll
        for (int c = 0; c < S; ++c) sg[c] = s.sig_s[(long)c * s.N + v];
    } else {
        voxel_stress<D>(s, v, sg);
    }
}

// The voxel-only terms of update_barriers (kmc_solver.hpp:345-407 /
// :1344-1406): the softening level of voxel v now (decayed transient part plus
// the permanent part, capped) ...
template <int D, int C>
MGK_DEV double voxel_gb(const KmcDevState& s, const KmcPhys& p, int v, double time) {
    const double gt = s.soft[2 * v + 1];
    double gtc = 0.0;
    if (gt > 0.0) {
        const double tl = s.last_t[v];
        if (isinf(p.tau)) gtc = gt;
        else if (tl == -INFINITY) gtc = 0.0;
        else {
            double dt = time - tl;
            if (dt < 0.0) dt = 0.0;
            gtc = gt * exp(-dt / p.tau);
        }
    }
    double gb = s.soft[2 * v] + gtc;
    if (p.softening_cap > 0.0 && gb > p.softening_cap) gb = p.softening_cap;
    return gb;
}

// ... and, for the directional scheme, the symmetric components of the
// voxel's previous flip and their norm.
template <int D, int C>
MGK_DEV double voxel_prev(const KmcDevState& s, int v, double* ps) {
    constexpr int S = D == 2 ? 3 : 6;
    cat_sym<D, C>(s.prev + (long)v * C, ps);
    double np = 0.0;
#pragma unroll
    for (int c = 0; c < S; ++c) np += (c < D ? 1.0 : 2.0) * ps[c] * ps[c];
    return sqrt(np);
}

// Q of mode i at voxel v from the voxel terms (stress sg, softening gb, and
// for the directional scheme ps / npv) and the mode's barrier q0.
template <int D, int C>
MGK_DEV double mode_Q_terms(const KmcDevState& s, const KmcPhys& p, int v, long i, const double* sg, double gb,
                            const double* ps, double npv, double q0) {
    constexpr int S = D == 2 ? 3 : 6;
    double cs[S];
    mode_eps<D, C>(s, v, i, sg, cs);
    double mod = 1.0;
    if (p.directional) {
        double dp = 0.0, nm = 0.0;
#pragma unroll
        for (int c = 0; c < S; ++c) {
            const double wgt = c < D ? 1.0 : 2.0;
            dp += wgt * cs[c] * ps[c];
            nm += wgt * cs[c] * cs[c];
        }
        const double nmv = sqrt(nm);
        if (!(npv < 1e-12 || nmv < 1e-12)) {
            const double ct = dp / (nmv * npv);
            mod = (1.0 + ct) * (1.0 + ct) / 4.0;
        }
    }
    const double geff = mod * gb;
    double w = 0.0;
#pragma unroll
    for (int c = 0; c < S; ++c) w += (c < D ? 1.0 : 2.0) * sg[c] * cs[c];
    const double wv = 0.5 * p.volume * (w / 1e9) * 6.241509;
    // exp(-0) is exactly 1: skip the exponential for unsoftened voxels
    return (geff == 0.0 ? q0 : q0 * exp(-geff)) - wv;
}

// Q of mode i at voxel v (update_barriers, kmc_solver.hpp:345-407 / :1344-1406)
template <int D, int C>
MGK_DEV double mode_Q(const KmcDevState& s, const KmcPhys& p, int v, long i, double time) {
    constexpr int S = D == 2 ? 3 : 6;
    double sg[S];
    sweep_stress<D>(s, v, sg);
    const double gb = voxel_gb<D, C>(s, p, v, time);
    double ps[S];
    double npv = 0.0;
    if (p.directional) npv = voxel_prev<D, C>(s, v, ps);
    return mode_Q_terms<D, C>(s, p, v, i, sg, gb, ps, npv, s.Q0[i]);
}

MGK_DEV double rate_of(const KmcPhys& p, double q, bool* inc) {
    // kmc_solver.hpp:795-801
    *inc = p.kmc_mode || q > 0.0;
    if (!*inc) return 0.0;
    return q <= 0.0 ? p.vnu : p.vnu * exp(-q * p.beta);
}

MGK_DEV dd warp_dd_sum(dd a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a = dd_add(a, dd_shfl_down(a, o));
    return a;
}

MGK_DEV bool dd_ge(dd a, double t) { return a.hi > t || (a.hi == t && a.lo >= 0.0); }

// Exclusive scan of one dd value per thread across the block (fixed order).
// Returns this thread's exclusive prefix; `tot` gets the block total.
MGK_DEV dd block_excl_scan(dd x, dd* sh /* 32 */, dd* tot) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    dd inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        dd y = {__shfl_up_sync(0xffffffffu, inc.hi, o), __shfl_up_sync(0xffffffffu, inc.lo, o)};
        if (lane >= o) inc = dd_add(y, inc);
    }
    __syncthreads();
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        dd run = {0.0, 0.0};
        for (int w = 0; w < nw; ++w) {
            dd t = sh[w];
            sh[w] = run;
            run = dd_add(run, t);
        }
        sh[31] = run;  // nw <= 31 for 992 threads; the launcher uses <= 512 threads
    }
    __syncthreads();
    dd wex = sh[wid];
    if (tot) *tot = sh[31];
    dd excl = {__shfl_up_sync(0xffffffffu, inc.hi, 1), __shfl_up_sync(0xffffffffu, inc.lo, 1)};
    if (lane == 0) excl = {0.0, 0.0};
    dd r = dd_add(wex, excl);
    __syncthreads();
    return r;
}

template <int D, int C>
MGK_DEV void apply_flip(const KmcDevState& s, const KmcPhys& p, long k, double time, double* cat_out /*C*/) {
    // apply_flip_soa_2d / _3d (kmc_solver.hpp:423-462 / :1424-1471)
    constexpr int S = D == 2 ? 3 : 6;
    const int v = (int)(k / s.M);
    double c[6];
    if (D == 3 && s.normals) {  // stress-dependent mode: C = 6 symmetric components
        double sg[6];
        sweep_stress<D>(s, v, sg);
        mode_eps<D, C>(s, v, k, sg, c);
    } else {
#pragma unroll
        for (int j = 0; j < C; ++j) c[j] = s.cat[k * C + j];
    }
    double cs[S];
    cat_sym<D, C>(c, cs);
#pragma unroll
    for (int j = 0; j < S; ++j) s.epsp_s[(long)j * s.N + v] += cs[j];
    double ssq;
    if (D == 2) {
        const double e11 = cs[0], e22 = cs[1], e12 = cs[2];
        ssq = (e12 * e12) + (e22 * e22 + e11 * e11 + (e11 - e22) * (e11 - e22)) / 6.0;
    } else {
        const double e11 = cs[0], e22 = cs[1], e33 = cs[2], e12 = cs[3], e13 = cs[4], e23 = cs[5];
        ssq = (e12 * e12 + e23 * e23 + e13 * e13) +
              ((e22 - e33) * (e22 - e33) + (e33 - e11) * (e33 - e11) + (e11 - e22) * (e11 - e22)) / 6.0;
    }
    double gp = s.soft[2 * v] + p.jp * ssq;
    if (p.softening_cap > 0.0 && gp > p.softening_cap) gp = p.softening_cap;
    s.soft[2 * v] = gp;
    s.soft[2 * v + 1] = p.jt * ssq;
    s.last_t[v] = time;
    if (p.neigh > 0.0) {
        const int nz = D == 3 ? p.nz : 1;
        const int x = v / (p.ny * nz), y = (v / nz) % p.ny, z = v % nz;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz) {
                    if (dx == 0 && dy == 0 && dz == 0) continue;
                    const int nb = (((x + dx + p.nx) % p.nx) * p.ny + (y + dy + p.ny) % p.ny) * nz + (z + dz + nz) % nz;
                    double g = s.soft[2 * nb] + p.neigh * p.jp * ssq;
                    if (p.softening_cap > 0.0 && g > p.softening_cap) g = p.softening_cap;
                    s.soft[2 * nb] = g;
                    s.soft[2 * nb + 1] += p.neigh * p.jt * ssq;
                }
    }
#pragma unroll
    for (int j = 0; j < C; ++j) {
        s.prev[(long)v * C + j] = c[j];
        if (cat_out) cat_out[j] = c[j];
    }
}

template <int C>
MGK_DEV void redraw(const KmcDevState& s, long k, const double* draws, int redraw_dir, int redraw_bar, int tid, int nthr) {
    // kmc_solver.hpp:841-864 and the per-voxel barrier extension: the RD_*
    // modes of the two parts; draws hold M records of C + 1 values when either
    // part is RD_ALL, else one record.
    const long v = k / s.M;
    for (int mm = tid; mm < s.M; mm += nthr) {
        const long ci = v * s.M + mm;
        const double* d = draws + (long)mm * (C + 1);
        if (redraw_dir == RD_ALL)
            for (int j = 0; j < C; ++j) s.cat[ci * C + j] = d[j];
        if (redraw_bar == RD_ALL) s.Q0[ci] = d[C];
        if (redraw_bar == RD_VOXEL) s.Q0[ci] = draws[C];
    }
    if (tid == 0) {
        if (redraw_dir == RD_FLIPPED)
            for (int j = 0; j < C; ++j) s.cat[k * C + j] = draws[j];
        if (redraw_bar == RD_FLIPPED) s.Q0[k] = draws[C];
    }
}

MGK_DEV bool key_less(double ka, int ma, double kb, int mb) { return ka < kb || (ka == kb && ma < mb); }


}  // namespace kmcdev
}  // namespace mgk
