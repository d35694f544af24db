/*
 * mgk_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the mgkmc_cpp algorithm on the KMC + Lippmann-Schwinger
 * hot path.  It is the CPU checker for the CUDA path and the "port" CPU baseline;
 * the product never links or calls it.  Each function names the reference
 * file:line it follows.  The arithmetic is kept in the reference's order where
 * that order is observable (serial rate sums, CDF scan, draw order); the FFT is
 * an independent implementation, so fields agree with the reference to rounding.
 *
 * Third-party algorithms restated here (not copied):
 *   - MT19937 (Matsumoto & Nishimura 1998): init_genrand + genrand_int32, which
 *     std::mt19937(seed) implements.
 *   - libstdc++ generate_canonical<double,53> over a 32-bit engine: two engine
 *     calls, sum = r0 + r1*2^32 in double, divided by 2^64, clamped below 1.
 *   - libstdc++ normal_distribution: Marsaglia polar method with one cached value.
 * Pinned against the reference compiled here (oracle/_ref/ref_driver "draws",
 * "ls2d/ls3d", "kmc_trace") by tests/test_oracle_pins.py.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ RNG */
typedef struct { uint32_t mt[624]; int mti; } mt19937;

static void mt_seed(mt19937* g, uint32_t s) {
    g->mt[0] = s;
    for (int i = 1; i < 624; ++i) g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->mti = 624;
}

static uint32_t mt_next(mt19937* g) {
    if (g->mti >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->mti = 0;
    }
    uint32_t y = g->mt[g->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* generate_canonical<double,53>(mt19937) */
static double canonical(mt19937* g) {
    double sum = (double)mt_next(g);
    sum += (double)mt_next(g) * 4294967296.0;
    double r = sum / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

static double uniform_ab(mt19937* g, double a, double b) { return canonical(g) * (b - a) + a; }

typedef struct { double saved; int has; } normal_state;

/* normal_distribution<double>(mean, sd) call on a persistent object */
static double normal_draw(normal_state* st, mt19937* g, double mean, double sd) {
    double v;
    if (st->has) {
        st->has = 0;
        v = st->saved;
    } else {
        double x, y, r2;
        do {
            x = 2.0 * canonical(g) - 1.0;
            y = 2.0 * canonical(g) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        double mult = sqrt(-2 * log(r2) / r2);
        st->saved = x * mult;
        st->has = 1;
        v = y * mult;
    }
    return v * sd + mean;
}

/* BarrierGenerator::generate, kmc_solver.hpp:35-95 */
enum { BAR_GAUSSIAN = 0, BAR_RAYLEIGH = 1, BAR_MOD_RAYLEIGH = 2, BAR_MOD_RAYLEIGH_EXP = 3 };
typedef struct {
    int type;
    double mean, std_val, min_cutoff, max_cutoff, loc, scale, epsilon, ratio;
} barrier_params;

static double mod_rayleigh(const barrier_params* b, mt19937* g) {
    double lo = b->mean - 6.0 * b->std_val;
    if (lo < 0.0) lo = 0.0;
    double hi = b->mean + 6.0 * b->std_val;
    double xm = (b->mean + sqrt(b->mean * b->mean + 4.0 * b->std_val * b->std_val)) / 2.0;
    double cm = xm * exp(-((xm - b->mean) * (xm - b->mean)) / (2.0 * b->std_val * b->std_val));
    for (;;) {
        double x = uniform_ab(g, lo, hi);
        double u = uniform_ab(g, 0.0, cm);
        double pdf = x * exp(-((x - b->mean) * (x - b->mean)) / (2.0 * b->std_val * b->std_val));
        if (u < pdf) return x;
    }
}

double oracle_barrier_draw(const barrier_params* b, mt19937* g) {
    double v = 0.0;
    if (b->type == BAR_GAUSSIAN) {
        normal_state st = {0.0, 0};
        v = normal_draw(&st, g, b->mean, b->std_val);
    } else if (b->type == BAR_RAYLEIGH) {
        double u = uniform_ab(g, 0.0, 1.0);
        v = b->loc + b->scale * sqrt(-2.0 * log(1.0 - u));
    } else if (b->type == BAR_MOD_RAYLEIGH) {
        v = mod_rayleigh(b, g);
    } else if (b->type == BAR_MOD_RAYLEIGH_EXP) {
        double umix = uniform_ab(g, 0.0, 1.0);
        if (umix < b->ratio) v = -b->epsilon * log(1.0 - uniform_ab(g, 0.0, 1.0));
        else v = mod_rayleigh(b, g);
    }
    if (b->min_cutoff >= 0.0 && v < b->min_cutoff) v = b->min_cutoff;
    if (b->max_cutoff >= 0.0 && v > b->max_cutoff) v = b->max_cutoff;
    return v;
}

/* exported RNG probes (pinned against ref_driver "draws") */
void oracle_draws(int seed, int n, double* out) {
    mt19937 g; mt_seed(&g, (uint32_t)seed);
    normal_state st = {0.0, 0};
    for (int i = 0; i < n; ++i) {
        out[4 * i + 0] = uniform_ab(&g, 0.0, 1.0);
        out[4 * i + 1] = normal_draw(&st, &g, 0.0, 1.0);
        out[4 * i + 2] = normal_draw(&st, &g, 0.0, 1.0);
        out[4 * i + 3] = (double)mt_next(&g);
    }
}

/* ------------------------------------------------------------------ FFT */
/* In-place unnormalised complex DFT of length n on strided data.  Radix-2
 * iterative for powers of two, direct O(n^2) sums otherwise. sign=-1 forward. */
static void dft_line(double* re, double* im, int n, long stride, int sign, double* wr, double* wi, double* tr, double* ti) {
    if (n == 1) return;
    for (int k = 0; k < n; ++k) { tr[k] = re[k * stride]; ti[k] = im[k * stride]; }
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { double t = tr[i]; tr[i] = tr[j]; tr[j] = t; t = ti[i]; ti[i] = ti[j]; ti[j] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int step = n / len;
            for (int i = 0; i < n; i += len)
                for (int k = 0; k < len / 2; ++k) {
                    double c = wr[k * step], s = sign * wi[k * step];
                    double ur = tr[i + k], ui = ti[i + k];
                    double vr = tr[i + k + len / 2] * c - ti[i + k + len / 2] * s;
                    double vi = tr[i + k + len / 2] * s + ti[i + k + len / 2] * c;
                    tr[i + k] = ur + vr; ti[i + k] = ui + vi;
                    tr[i + k + len / 2] = ur - vr; ti[i + k + len / 2] = ui - vi;
                }
        }
        for (int k = 0; k < n; ++k) { re[k * stride] = tr[k]; im[k * stride] = ti[k]; }
    } else {
        for (int k = 0; k < n; ++k) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; ++j) {
                long p = ((long)j * k) % n;
                double c = wr[p], s = sign * wi[p];
                sr += tr[j] * c - ti[j] * s;
                si += tr[j] * s + ti[j] * c;
            }
            re[k * stride] = sr; im[k * stride] = si;
        }
    }
}

/* ortho-normalised C2C over the dims (pocketfft c2c, fct = 1/sqrt(N)), as used
 * by fft2d/ifft2d/fft3d/ifft3d, linear_elastic_solver.hpp:122-143, 399-428 */
static void fftnd(double* re, double* im, const int* dims, int nd, int sign) {
    long N = 1;
    for (int a = 0; a < nd; ++a) N *= dims[a];
    int nmax = 1;
    for (int a = 0; a < nd; ++a) if (dims[a] > nmax) nmax = dims[a];
    double* wr = malloc(sizeof(double) * nmax);
    double* wi = malloc(sizeof(double) * nmax);
    double* tr = malloc(sizeof(double) * nmax);
    double* ti = malloc(sizeof(double) * nmax);
    for (int a = 0; a < nd; ++a) {
        int n = dims[a];
        for (int k = 0; k < n; ++k) { wr[k] = cos(-2.0 * M_PI * k / n); wi[k] = sin(-2.0 * M_PI * k / n); }
        long stride = 1;
        for (int b = a + 1; b < nd; ++b) stride *= dims[b];
        long outer = N / (stride * n);
        for (long o = 0; o < outer; ++o)
            for (long in = 0; in < stride; ++in) {
                long base = o * stride * n + in;
                dft_line(re + base, im + base, n, stride, sign, wr, wi, tr, ti);
            }
    }
    double f = 1.0 / sqrt((double)N);
    for (long i = 0; i < N; ++i) { re[i] *= f; im[i] *= f; }
    free(wr); free(wi); free(tr); free(ti);
}

/* ------------------------------------------------------------------ LS */
/* fftfreq (linear_elastic_solver.hpp:22-33) times 2*pi, as in init_gamma */
static double kvec(int i, int n, double d) {
    int lim = (n + 1) / 2;
    double f = (i < lim) ? (double)i / (n * d) : (double)(i - n) / (n * d);
    return 2.0 * M_PI * f;
}

/* compute_lame_2d / compute_lame_3d, linear_elastic_solver.hpp:36-45, 315-319 */
static void lame(double E, double nu, int dim, int plane_stress, double* lam, double* mu) {
    *mu = E / (2.0 * (1.0 + nu));
    if (dim == 2 && plane_stress) *lam = E * nu / (1.0 - nu * nu);
    else *lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

/* Green operator entry Gamma_khij(q), linear_elastic_solver.hpp:98-115 / 374-391 */
static double gamma_entry(const double* q, int k, int h, int i, int j, double k2, double A, double B) {
    double t1 = 0.0;
    if (k == i) t1 += q[h] * q[j];
    if (h == i) t1 += q[k] * q[j];
    if (k == j) t1 += q[h] * q[i];
    if (h == j) t1 += q[k] * q[i];
    t1 = A * t1 / k2;
    double t2 = B * (q[k] * q[h] * q[i] * q[j]) / (k2 * k2);
    return t1 - t2;
}

/*
 * spectral_solver_2d / spectral_solver_3d (linear_elastic_solver.hpp:146-309,
 * 431-593).  Tensors are row-major D x D per voxel.  eps is in/out (warm start
 * when warm != 0, else filled with eps_bar).  epsp may be NULL.
 * Returns the number of iterations run; sig, macro_eps, macro_sig are outputs.
 */
int oracle_ls_solve(int dim, const int* dims, int plane_stress, double pixel, const double* E, const double* nu,
                    const double* eps_bar, double* eps, int warm, const double* epsp, int max_iter, double tol,
                    double* sig, double* macro_eps, double* macro_sig) {
    const int D = dim, DD = D * D;
    long N = 1;
    for (int a = 0; a < D; ++a) N *= dims[a];
    double Es = 0.0, ns = 0.0;
    for (long i = 0; i < N; ++i) { Es += E[i]; ns += nu[i]; }
    double lam0, mu0;
    lame(Es / N, ns / N, D, plane_stress, &lam0, &mu0);
    double* lamv = malloc(sizeof(double) * N);
    double* muv = malloc(sizeof(double) * N);
    for (long i = 0; i < N; ++i) lame(E[i], nu[i], D, plane_stress, &lamv[i], &muv[i]);
    if (warm) {
        double mean[9] = {0};
        for (long i = 0; i < N; ++i) for (int c = 0; c < DD; ++c) mean[c] += eps[i * DD + c];
        for (int c = 0; c < DD; ++c) mean[c] /= N;
        double diff[9];
        for (int c = 0; c < DD; ++c) diff[c] = eps_bar[c] - mean[c];
        for (long i = 0; i < N; ++i) for (int c = 0; c < DD; ++c) eps[i * DD + c] += diff[c];
    } else {
        for (long i = 0; i < N; ++i) for (int c = 0; c < DD; ++c) eps[i * DD + c] = eps_bar[c];
    }
    double* tre = malloc(sizeof(double) * N * DD);
    double* tim = malloc(sizeof(double) * N * DD);
    double* ore = malloc(sizeof(double) * N * DD);
    double* oim = malloc(sizeof(double) * N * DD);
    double A = 1.0 / (4.0 * mu0), B = (lam0 + mu0) / (mu0 * (lam0 + 2.0 * mu0));
    int it;
    for (it = 0; it < max_iter; ++it) {
        /* sigma = C:(eps - epsp); tau = sigma - C0:eps */
        for (long i = 0; i < N; ++i) {
            const double* e = eps + i * DD;
            double ee[9], tr = 0.0, tr0 = 0.0;
            for (int c = 0; c < DD; ++c) ee[c] = epsp ? e[c] - epsp[i * DD + c] : e[c];
            for (int a = 0; a < D; ++a) { tr += ee[a * D + a]; tr0 += e[a * D + a]; }
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) {
                    double s = 2.0 * muv[i] * ee[r * D + c] + lamv[i] * tr * (r == c ? 1.0 : 0.0);
                    double s0 = 2.0 * mu0 * e[r * D + c] + lam0 * tr0 * (r == c ? 1.0 : 0.0);
                    tre[(long)(r * D + c) * N + i] = s - s0;
                    tim[(long)(r * D + c) * N + i] = 0.0;
                }
        }
        for (int c = 0; c < DD; ++c) fftnd(tre + c * N, tim + c * N, dims, D, -1);
        /* eps_tilde_hat = -Gamma : tau_hat */
        for (long i = 0; i < N; ++i) {
            long rem = i;
            int idx[3] = {0, 0, 0};
            for (int a = D - 1; a >= 0; --a) { idx[a] = (int)(rem % dims[a]); rem /= dims[a]; }
            double q[3] = {0, 0, 0}, k2 = 0.0;
            int zero = 1;
            for (int a = 0; a < D; ++a) { q[a] = kvec(idx[a], dims[a], pixel); k2 += q[a] * q[a]; if (idx[a]) zero = 0; }
            for (int k = 0; k < D; ++k)
                for (int h = 0; h < D; ++h) {
                    double vr = 0.0, vi = 0.0;
                    if (!zero)
                        for (int r = 0; r < D; ++r)
                            for (int s = 0; s < D; ++s) {
                                double g = gamma_entry(q, k, h, r, s, k2, A, B);
                                vr += g * tre[(long)(r * D + s) * N + i];
                                vi += g * tim[(long)(r * D + s) * N + i];
                            }
                    ore[(long)(k * D + h) * N + i] = -vr;
                    oim[(long)(k * D + h) * N + i] = -vi;
                }
        }
        for (int c = 0; c < DD; ++c) fftnd(ore + c * N, oim + c * N, dims, D, +1);
        double mean[9];
        for (int c = 0; c < DD; ++c) {
            double s = 0.0;
            for (long i = 0; i < N; ++i) s += ore[(long)c * N + i];
            mean[c] = s / N;
        }
        double dsq = 0.0, nsq = 0.0;
        for (long i = 0; i < N; ++i) {
            for (int c = 0; c < DD; ++c) {
                double nv = eps_bar[c] + (ore[(long)c * N + i] - mean[c]);
                double d = nv - eps[i * DD + c];
                dsq += d * d;
                nsq += eps[i * DD + c] * eps[i * DD + c];
                tim[(long)c * N + i] = nv; /* stash */
            }
        }
        for (long i = 0; i < N; ++i) for (int c = 0; c < DD; ++c) eps[i * DD + c] = tim[(long)c * N + i];
        double diff = sqrt(dsq) / (sqrt(nsq) + 1e-20);
        if (diff < tol) { ++it; break; }
    }
    for (int c = 0; c < DD; ++c) { macro_eps[c] = 0.0; macro_sig[c] = 0.0; }
    for (long i = 0; i < N; ++i) {
        const double* e = eps + i * DD;
        double ee[9], tr = 0.0;
        for (int c = 0; c < DD; ++c) ee[c] = epsp ? e[c] - epsp[i * DD + c] : e[c];
        for (int a = 0; a < D; ++a) tr += ee[a * D + a];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double s = 2.0 * muv[i] * ee[r * D + c] + lamv[i] * tr * (r == c ? 1.0 : 0.0);
                if (sig) sig[i * DD + r * D + c] = s;
                macro_eps[r * D + c] += e[r * D + c];
                macro_sig[r * D + c] += s;
            }
    }
    for (int c = 0; c < DD; ++c) { macro_eps[c] /= N; macro_sig[c] /= N; }
    free(lamv); free(muv); free(tre); free(tim); free(ore); free(oim);
    return it;
}

/* ------------------------------------------------------------------ KMC */
typedef struct {
    int dim, nx, ny, nz, M, plane_stress, seed;
    double gamma0, pixel;
    barrier_params bar;
    int directional;               /* softening_scheme == "directional" */
    double softening_cap, jp, jt, neighbor_fraction, q_act_temp;
    double temperature, strain_rate, stability_threshold, nu0;
    int instability_kmc;           /* instability_mode == "kmc" (else cascade) */
    int scale_rate_by_volume, redraw_directions, redraw_barriers, use_3d_barriers;
    double step_size, mixed_tol, max_kmc_steps_pct;
    int comp_i, comp_j;
    int n_targets;
    int target_i[9], target_j[9];
    double target_v[9];
    /* catalog extensions (no counterpart in the reference): catalog_type 0
     * the reference's random modes, 1 M shears evenly spaced in [0, pi) in the
     * x-y plane, 2 (3D) M Fibonacci-lattice plane normals sheared along their
     * largest resolved shear stress; barrier_per_voxel: one barrier per voxel
     * shared by its M modes */
    int catalog_type, barrier_per_voxel;
} kmc_params;

typedef struct {
    kmc_params p;
    long N;
    int D, DD;
    double volume, tau, time;
    double *E, *nu, *eps, *sig, *epsp, *soft, *last_t, *Q, *Q0, *cat, *prev;
    double* normals;  /* catalog_type 2: M plane normals (x, y, z) */
    double eps_macro[9], sig_macro[9];
    mt19937 rng;
    int ls_iters_total, ls_solves;
} kmc_state;

/* stz_mode_glass / stz_mode_glass_3d (kmc_solver.hpp:1042-1074) and the 2D
 * catalog draw (kmc_solver.hpp:231-238); ns is the caller's normal object. */
static void draw_mode(kmc_state* s, normal_state* ns, double* out) {
    const int D = s->D;
    memset(out, 0, sizeof(double) * s->DD);
    if (D == 3 && s->p.use_3d_barriers) {
        normal_state g = {0.0, 0};
        double m[9], ms[9], G[9];
        for (int i = 0; i < 9; ++i) m[i] = normal_draw(&g, &s->rng, 0.0, 1.0);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) ms[i * 3 + j] = 0.5 * (m[i * 3 + j] + m[j * 3 + i]);
        double tr = (ms[0] + ms[4]) + ms[8];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) G[i * 3 + j] = ms[i * 3 + j] - (1.0 / 3.0) * tr * (i == j ? 1.0 : 0.0);
        /* Frobenius norm in Eigen's column-major storage order */
        double sq = 0.0;
        for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) sq += G[i * 3 + j] * G[i * 3 + j];
        double nrm = sqrt(sq);
        if (nrm < 1e-12) return;
        double f = 1.0 / (sqrt(2.0) * nrm);
        for (int i = 0; i < 9; ++i) G[i] = G[i] * f;
        double u = uniform_ab(&s->rng, 1e-15, 1.0);
        double mag = s->p.gamma0 * sqrt(-2.0 * log(u));
        for (int i = 0; i < 9; ++i) out[i] = G[i] * mag;
        return;
    }
    normal_state local = {0.0, 0};
    normal_state* g = (D == 3) ? &local : ns;  /* 3D: fresh object per mode */
    double gxx = 0.5 * s->p.gamma0 * normal_draw(g, &s->rng, 0.0, 1.0);
    double gxy = 0.5 * s->p.gamma0 * normal_draw(g, &s->rng, 0.0, 1.0);
    out[0] = gxx; out[D + 1] = -gxx; out[1] = gxy; out[D] = gxy;
}

/* Catalog extensions (no counterpart in the reference).
 * Even: shear m of M slips along s = (cos t, sin t, 0) on the plane of normal
 * n = (-sin t, cos t, 0), t = m pi / M; eigenstrain (gamma0 / 2)(s n + n s):
 * xx = -(gamma0/2) sin 2t, yy = +(gamma0/2) sin 2t, xy = (gamma0/2) cos 2t. */
static void even_mode(const kmc_state* s, int m, double* out) {
    const int D = s->D;
    const double h = 0.5 * s->p.gamma0;
    const double a = 2.0 * M_PI * (double)m / (double)s->p.M;
    const double sa = sin(a), ca = cos(a);
    memset(out, 0, sizeof(double) * s->DD);
    out[0] = -h * sa;
    out[D + 1] = h * sa;
    out[1] = h * ca;
    out[D] = h * ca;
}

/* Fibonacci lattice on the upper hemisphere: z = 1 - (m + 1/2) / M,
 * azimuth m * pi (3 - sqrt 5). */
static void fib_normals(int M, double* n) {
    const double ga = M_PI * (3.0 - sqrt(5.0));
    for (int m = 0; m < M; ++m) {
        const double z = 1.0 - ((double)m + 0.5) / (double)M;
        const double r = sqrt(1.0 - z * z);
        const double ph = (double)m * ga;
        n[3 * m] = r * cos(ph);
        n[3 * m + 1] = r * sin(ph);
        n[3 * m + 2] = z;
    }
}

/* Stress-dependent shear on the plane of normal n: slip along the resolved
 * shear traction tau = sigma n - (n . sigma n) n (where tau vanishes, along the
 * projection of x -- or y when n is near x -- onto the plane); eigenstrain
 * (gamma0 / 2)(s n + n s), so that sigma : eps0 = gamma0 |tau|. */
static void fib_mode(const double* sg, const double* n, double gamma0, double* out) {
    double t[3], tau[3], sv[3];
    for (int i = 0; i < 3; ++i) t[i] = sg[3 * i] * n[0] + sg[3 * i + 1] * n[1] + sg[3 * i + 2] * n[2];
    const double tn = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
    double tt = 0.0;
    for (int i = 0; i < 3; ++i) {
        tau[i] = t[i] - tn * n[i];
        tt += tau[i] * tau[i];
    }
    if (tt > 0.0) {
        const double inv = 1.0 / sqrt(tt);
        for (int i = 0; i < 3; ++i) sv[i] = tau[i] * inv;
    } else {
        double e[3] = {0.0, 0.0, 0.0};
        e[fabs(n[0]) < 0.9 ? 0 : 1] = 1.0;
        const double d = e[0] * n[0] + e[1] * n[1] + e[2] * n[2];
        double q = 0.0;
        for (int i = 0; i < 3; ++i) {
            sv[i] = e[i] - d * n[i];
            q += sv[i] * sv[i];
        }
        const double inv = 1.0 / sqrt(q);
        for (int i = 0; i < 3; ++i) sv[i] *= inv;
    }
    const double h = 0.5 * gamma0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = h * (sv[i] * n[j] + n[i] * sv[j]);
}

/* the eigenstrain of mode m of voxel v now (full D x D row-major) */
static void mode_of(const kmc_state* s, long v, int m, double* out) {
    if (s->p.catalog_type == 2) fib_mode(s->sig + v * 9, s->normals + 3 * m, s->p.gamma0, out);
    else memcpy(out, s->cat + (v * s->p.M + m) * s->DD, sizeof(double) * s->DD);
}

/* constructors, kmc_solver.hpp:165-257 / 1142-1232 */
void* oracle_kmc_create(const kmc_params* p, const double* E, const double* nu) {
    if (p->catalog_type == 2 && p->dim != 3) return NULL;  /* plane normals need 3D */
    kmc_state* s = calloc(1, sizeof(kmc_state));
    s->p = *p;
    s->D = p->dim; s->DD = p->dim * p->dim;
    s->N = (long)p->nx * p->ny * (p->dim == 3 ? p->nz : 1);
    long N = s->N, NM = N * p->M;
    s->volume = p->pixel * p->pixel * p->pixel;
    s->E = malloc(sizeof(double) * N); memcpy(s->E, E, sizeof(double) * N);
    s->nu = malloc(sizeof(double) * N); memcpy(s->nu, nu, sizeof(double) * N);
    s->eps = calloc(N * s->DD, sizeof(double));
    s->sig = calloc(N * s->DD, sizeof(double));
    s->epsp = calloc(N * s->DD, sizeof(double));
    s->soft = calloc(N * 2, sizeof(double));
    s->last_t = malloc(sizeof(double) * N);
    for (long i = 0; i < N; ++i) s->last_t[i] = -INFINITY;
    s->Q = calloc(NM, sizeof(double));
    s->Q0 = malloc(sizeof(double) * NM);
    s->cat = p->catalog_type == 2 ? NULL : calloc(NM * s->DD, sizeof(double));
    if (p->catalog_type == 2) {
        s->normals = malloc(sizeof(double) * 3 * p->M);
        fib_normals(p->M, s->normals);
    }
    s->prev = calloc(N * s->DD, sizeof(double));
    if (p->temperature > 0.0) s->tau = 1.0 / (p->nu0 * exp(-p->q_act_temp / (8.617e-5 * p->temperature)));
    else s->tau = INFINITY;
    mt_seed(&s->rng, (uint32_t)p->seed);
    normal_state ns = {0.0, 0};  /* 2D ctor: one normal object for the whole fill */
    for (long v = 0; v < N; ++v) {
        /* extension: one barrier per voxel, drawn before the voxel's modes */
        double qv = p->barrier_per_voxel ? oracle_barrier_draw(&p->bar, &s->rng) : 0.0;
        for (int m = 0; m < p->M; ++m) {
            long mi = v * p->M + m;
            s->Q0[mi] = p->barrier_per_voxel ? qv : oracle_barrier_draw(&p->bar, &s->rng);
            if (p->catalog_type == 0) draw_mode(s, &ns, s->cat + mi * s->DD);
            else if (p->catalog_type == 1) even_mode(s, m, s->cat + mi * s->DD);
        }
    }
    return s;
}

void oracle_kmc_destroy(void* h) {
    kmc_state* s = h;
    if (!s) return;
    free(s->E); free(s->nu); free(s->eps); free(s->sig); free(s->epsp); free(s->soft); free(s->last_t);
    free(s->Q); free(s->Q0); free(s->cat); free(s->prev); free(s->normals); free(s);
}

/* elastic_run, kmc_solver.hpp:334-339 / 1333-1338 */
static void elastic_run(kmc_state* s) {
    int dims[3] = {s->p.nx, s->p.ny, s->p.nz};
    double em[9], sm[9];
    int it = oracle_ls_solve(s->D, dims, s->p.plane_stress, s->p.pixel, s->E, s->nu, s->eps_macro, s->eps, 1, s->epsp, 200,
                             1e-6, s->sig, em, sm);
    memcpy(s->eps_macro, em, sizeof(double) * s->DD);
    memcpy(s->sig_macro, sm, sizeof(double) * s->DD);
    s->ls_iters_total += it;
    s->ls_solves += 1;
}

/* update_barriers, kmc_solver.hpp:341-410 / 1340-1411 */
static void update_barriers(kmc_state* s) {
    const int DD = s->DD, M = s->p.M;
    for (long v = 0; v < s->N; ++v) {
        double gt = s->soft[2 * v + 1], tl = s->last_t[v], gtc = 0.0;
        if (gt > 0.0) {
            if (isinf(s->tau)) gtc = gt;
            else if (tl == -INFINITY) gtc = 0.0;
            else { double dt = s->time - tl; if (dt < 0.0) dt = 0.0; gtc = gt * exp(-dt / s->tau); }
        }
        double gb = s->soft[2 * v] + gtc;
        if (s->p.softening_cap > 0.0 && gb > s->p.softening_cap) gb = s->p.softening_cap;
        const double* sg = s->sig + v * DD;
        const double* pv = s->prev + v * DD;
        for (int m = 0; m < M; ++m) {
            long mi = v * M + m;
            double cm[9];
            mode_of(s, v, m, cm);
            const double* c = cm;
            double mod = 1.0;
            if (s->p.directional) {
                double dp = 0.0, nm = 0.0, np = 0.0;
                for (int k = 0; k < DD; ++k) { dp += c[k] * pv[k]; nm += c[k] * c[k]; np += pv[k] * pv[k]; }
                double npv = sqrt(np), nmv = sqrt(nm);
                if (!(npv < 1e-12 || nmv < 1e-12)) { double ct = dp / (nmv * npv); mod = (1.0 + ct) * (1.0 + ct) / 4.0; }
            }
            double geff = mod * gb, w = 0.0;
            for (int k = 0; k < DD; ++k) w += sg[k] * c[k];
            double wv = 0.5 * s->volume * (w / 1e9) * 6.241509;
            s->Q[mi] = s->Q0[mi] * exp(-geff) - wv;
        }
    }
}

/* apply_flip_soa_2d / _3d, kmc_solver.hpp:423-462 / 1424-1471 */
static void apply_flip(kmc_state* s, long vox, int m) {
    const int D = s->D, DD = s->DD;
    double cm[9];
    mode_of(s, vox, m, cm);
    const double* c = cm;
    for (int k = 0; k < DD; ++k) s->epsp[vox * DD + k] += c[k];
    double ssq;
    if (D == 2) {
        double e11 = c[0], e22 = c[3], e12 = c[1];
        ssq = (e12 * e12) + (e22 * e22 + e11 * e11 + (e11 - e22) * (e11 - e22)) / 6.0;
    } else {
        double e11 = c[0], e22 = c[4], e33 = c[8], e12 = c[1], e13 = c[2], e23 = c[5];
        ssq = (e12 * e12 + e23 * e23 + e13 * e13) + ((e22 - e33) * (e22 - e33) + (e33 - e11) * (e33 - e11) + (e11 - e22) * (e11 - e22)) / 6.0;
    }
    double cap = s->p.softening_cap;
    double gp = s->soft[2 * vox] + s->p.jp * ssq;
    if (cap > 0.0 && gp > cap) gp = cap;
    s->soft[2 * vox] = gp;
    s->soft[2 * vox + 1] = s->p.jt * ssq;
    s->last_t[vox] = s->time;
    if (s->p.neighbor_fraction > 0.0) {
        int nx = s->p.nx, ny = s->p.ny, nz = D == 3 ? s->p.nz : 1;
        int x = (int)(vox / ((long)ny * nz)), y = (int)((vox / nz) % ny), z = (int)(vox % nz);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz) {
                    if (dx == 0 && dy == 0 && dz == 0) continue;
                    long nb = ((long)((x + dx + nx) % nx) * ny + (y + dy + ny) % ny) * nz + (z + dz + nz) % nz;
                    double g = s->soft[2 * nb] + s->p.neighbor_fraction * s->p.jp * ssq;
                    if (cap > 0.0 && g > cap) g = cap;
                    s->soft[2 * nb] = g;
                    s->soft[2 * nb + 1] += s->p.neighbor_fraction * s->p.jt * ssq;
                }
    }
}

/* redraw after a flip, kmc_solver.hpp:839-864 (thermal), 499-523 (cascade),
 * 1854-1875 / 1512-1533 (3D) */
static void redraw(kmc_state* s, long vox, long flat) {
    normal_state ns = {0.0, 0};
    const int M = s->p.M, DD = s->DD;
    if (s->p.catalog_type != 0 || s->p.barrier_per_voxel) {
        /* extensions: fixed catalogs are never redrawn; a per-voxel barrier is
         * one draw before the voxel's modes */
        const int rd = s->p.redraw_directions && s->p.catalog_type == 0;
        const int all = s->p.redraw_directions || s->p.redraw_barriers;
        if (s->p.barrier_per_voxel) {
            if (s->p.redraw_barriers || !all) {
                const double q = oracle_barrier_draw(&s->p.bar, &s->rng);
                for (int mm = 0; mm < M; ++mm) s->Q0[vox * M + mm] = q;
            }
            if (rd) for (int mm = 0; mm < M; ++mm) draw_mode(s, &ns, s->cat + (vox * M + mm) * DD);
            else if (!all && s->p.catalog_type == 0) draw_mode(s, &ns, s->cat + flat * DD);
        } else if (all) {
            if (s->p.redraw_barriers)
                for (int mm = 0; mm < M; ++mm) s->Q0[vox * M + mm] = oracle_barrier_draw(&s->p.bar, &s->rng);
        } else {
            s->Q0[flat] = oracle_barrier_draw(&s->p.bar, &s->rng);
        }
        return;
    }
    if (s->p.redraw_directions || s->p.redraw_barriers) {
        for (int mm = 0; mm < M; ++mm) {
            long ci = vox * M + mm;
            if (s->p.redraw_directions) draw_mode(s, &ns, s->cat + ci * DD);
            if (s->p.redraw_barriers) s->Q0[ci] = oracle_barrier_draw(&s->p.bar, &s->rng);
        }
    } else {
        draw_mode(s, &ns, s->cat + flat * DD);
        s->Q0[flat] = oracle_barrier_draw(&s->p.bar, &s->rng);
    }
}

static int cmp_q_idx(const void* a, const void* b) {
    const double* x = a; const double* y = b;
    if (x[0] < y[0]) return -1;
    if (x[0] > y[0]) return 1;
    return (x[1] < y[1]) ? -1 : (x[1] > y[1]);
}

/* run_cascade, kmc_solver.hpp:464-564 / 1473-1590 (fast patching off).
 * Ties in Q are broken by mode index (std::sort leaves them unspecified). */
static void run_cascade(kmc_state* s, int* steps, int* flips) {
    long NM = s->N * s->p.M;
    int total = 0, local = 0;
    double* lst = malloc(sizeof(double) * 2 * NM);
    unsigned char* seen = malloc(s->N);
    for (;;) {
        update_barriers(s);
        long nu = 0;
        for (long i = 0; i < NM; ++i) if (s->Q[i] < s->p.stability_threshold) { lst[2 * nu] = s->Q[i]; lst[2 * nu + 1] = (double)i; ++nu; }
        if (nu == 0) break;
        qsort(lst, nu, 2 * sizeof(double), cmp_q_idx);
        memset(seen, 0, s->N);
        int nb = 0;
        for (long k = 0; k < nu; ++k) {
            long mi = (long)lst[2 * k + 1];
            long vox = mi / s->p.M;
            int m = (int)(mi % s->p.M);
            if (seen[vox]) continue;
            seen[vox] = 1;
            ++nb;
            mode_of(s, vox, m, s->prev + vox * s->DD);
            apply_flip(s, vox, m);
            redraw(s, vox, mi);
        }
        elastic_run(s);
        total += nb;
        ++local;
        if (local > s->N) break;
    }
    free(lst); free(seen);
    *steps = local; *flips = total;
}

/*
 * run_simulation (kmc_solver.hpp:721-1037 / 1735-2062), fast patching off,
 * logging off.  Writes one trace row per event (same layout as the reference
 * harness): [kind, a, b, total_rate, t_wait, time, eps_macro(DD), sig_macro(DD)]
 * kind 0 thermal flip (a = flat mode, b = is_instab), 1 cascade (a = batches,
 * b = flips), 2 interval end without event (a = u1), 3 elastic step done
 * (a = mixed-BC solves, b = elastic steps done).  Returns rows written.
 */
long oracle_kmc_run(void* h, int nsteps, long maxev, double* trace, long trace_cap) {
    kmc_state* s = h;
    const int DD = s->DD;
    long rows = 0, nev = 0;
    int seq_instab = 0, max_seq = (int)(s->p.max_kmc_steps_pct * (double)s->N);
#define PUSH(kind, a, b, R, tw)                                                               \
    do {                                                                                      \
        if (rows < trace_cap) {                                                               \
            double* r_ = trace + rows * (6 + 2 * DD);                                         \
            r_[0] = kind; r_[1] = a; r_[2] = b; r_[3] = R; r_[4] = tw; r_[5] = s->time;         \
            for (int c_ = 0; c_ < DD; ++c_) { r_[6 + c_] = s->eps_macro[c_]; r_[6 + DD + c_] = s->sig_macro[c_]; } \
        }                                                                                     \
        ++rows;                                                                               \
    } while (0)
    elastic_run(s);
    int ci = s->p.comp_i * s->D + s->p.comp_j;
    double dt_step = fabs(s->p.step_size) / s->p.strain_rate, remaining = 0.0;
    long NM = s->N * s->p.M;
    double* rates = malloc(sizeof(double) * NM);
    long* idx = malloc(sizeof(long) * NM);
    int done = 0, stop = 0;
    while (done < nsteps && !stop) {
        remaining += dt_step;
        while (remaining > 0.0) {
            update_barriers(s);
            if (!s->p.instability_kmc) {
                long nu = 0;
                for (long i = 0; i < NM; ++i) if (s->Q[i] < s->p.stability_threshold) { ++nu; break; }
                if (nu) {
                    int cs, cf;
                    run_cascade(s, &cs, &cf);
                    if (cf > 0) PUSH(1, cs, cf, 0, 0);
                    continue;
                }
            }
            double vol = s->p.scale_rate_by_volume ? s->volume : 1.0;
            double beta = s->p.temperature > 0.0 ? 1.0 / (8.617e-5 * s->p.temperature) : INFINITY;
            long nr = 0;
            double R = 0.0;
            for (long i = 0; i < NM; ++i) {
                double q = s->Q[i];
                if (s->p.instability_kmc || q > 0.0) {
                    double r = q <= 0.0 ? vol * s->p.nu0 : vol * s->p.nu0 * exp(-q * beta);
                    rates[nr] = r; idx[nr] = i; ++nr; R += r;
                }
            }
            if (R > 0.0) {
                double u1 = uniform_ab(&s->rng, 0.0, 1.0);
                double tw = -log(u1) / R;
                if (tw < remaining) {
                    s->time += tw;
                    s->eps_macro[ci] += 1.0 * (s->p.strain_rate * tw);
                    remaining -= tw;
                    double target = uniform_ab(&s->rng, 0.0, 1.0) * R, cur = 0.0;
                    long sel = nr - 1;
                    for (long i = 0; i < nr; ++i) { cur += rates[i]; if (cur >= target) { sel = i; break; } }
                    long f = idx[sel], vox = f / s->p.M;
                    int m = (int)(f % s->p.M);
                    int instab = s->Q[f] <= s->p.stability_threshold;
                    mode_of(s, vox, m, s->prev + vox * DD);
                    apply_flip(s, vox, m);
                    redraw(s, vox, f);
                    elastic_run(s);
                    seq_instab = instab ? seq_instab + 1 : 0;
                    PUSH(0, (double)f, instab, R, tw);
                    if (++nev >= maxev || seq_instab > max_seq) { stop = 1; break; }
                    continue;
                } else {
                    PUSH(2, u1, 0, R, tw);
                }
            }
            s->eps_macro[ci] += 1.0 * (s->p.strain_rate * remaining);
            s->time += remaining;
            remaining = 0.0;
        }
        if (stop) break;
        double Es = 0.0, ns = 0.0;
        for (long i = 0; i < s->N; ++i) Es += s->E[i];
        for (long i = 0; i < s->N; ++i) ns += s->nu[i];
        double Ea = Es / s->N, na = ns / s->N;
        int solves = 0;
        for (int it = 0; it < 50; ++it) {
            elastic_run(s);
            ++solves;
            double err[9] = {0}, emax = 0.0;
            for (int t = 0; t < s->p.n_targets; ++t) {
                int k = s->p.target_i[t] * s->D + s->p.target_j[t];
                double e = s->p.target_v[t] - s->sig_macro[k];
                err[k] = e;
                if (fabs(e) > emax) emax = fabs(e);
            }
            if (emax < s->p.mixed_tol) break;
            double tr = 0.0;
            for (int a = 0; a < s->D; ++a) tr += err[a * s->D + a];
            for (int t = 0; t < s->p.n_targets; ++t) {
                int a = s->p.target_i[t], b = s->p.target_j[t], k = a * s->D + b;
                double d = (err[k] - na * tr * (a == b ? 1.0 : 0.0)) / Ea;
                s->eps_macro[k] += d;
            }
        }
        ++done;
        PUSH(3, solves, done, 0, 0);
    }
    free(rates); free(idx);
#undef PUSH
    return rows;
}

/* field accessors: 0 eps, 1 sig, 2 epsp, 3 soft, 4 last_t, 5 Q, 6 Q0, 7 catalog, 8 prev_dir */
long oracle_kmc_get(void* h, int field, double* out) {
    kmc_state* s = h;
    long NM = s->N * s->p.M;
    const double* src; long n;
    switch (field) {
        case 0: src = s->eps; n = s->N * s->DD; break;
        case 1: src = s->sig; n = s->N * s->DD; break;
        case 2: src = s->epsp; n = s->N * s->DD; break;
        case 3: src = s->soft; n = s->N * 2; break;
        case 4: src = s->last_t; n = s->N; break;
        case 5: src = s->Q; n = NM; break;
        case 6: src = s->Q0; n = NM; break;
        case 7: src = s->cat; n = src ? NM * s->DD : 0; break;  /* stress-dependent modes: none stored */
        case 8: src = s->prev; n = s->N * s->DD; break;
        default: return -1;
    }
    if (out) memcpy(out, src, sizeof(double) * n);
    return n;
}

void oracle_kmc_macro(void* h, double* out) {
    kmc_state* s = h;
    for (int c = 0; c < s->DD; ++c) { out[c] = s->eps_macro[c]; out[s->DD + c] = s->sig_macro[c]; }
    out[2 * s->DD] = s->time;
    out[2 * s->DD + 1] = s->ls_iters_total;
    out[2 * s->DD + 2] = s->ls_solves;
}

long oracle_sizeof_params(void) { return (long)sizeof(kmc_params); }
