// The reference's correlated random field (generate_correlated_field_cpp,
// material_generator.hpp:130-258: main.cpp's "generated" material mode) on
// the GPU: one standard normal per voxel by Box-Muller from std::mt19937(seed),
// an orthonormal forward FFT, the Gaussian filter exp(-2 pi^2 sigma^2 |f|^2),
// the orthonormal inverse FFT (real part), standardisation to mean 0 / std 1,
// then scale, shift and clipping.
//
// MT19937 words come from the recurrence x[n] = x[n-227] ^ T(x[n-624],
// x[n-623]) extended 227 at a time by one CTA (the seeded state leaves its
// first twist pending, so output k is temper(x[624 + k])).  Each voxel takes
// two words unless a u1 word is 0 (probability 2^-32 a voxel: the reference
// then draws again); that case is detected on the device and the normals are
// drawn on the host instead.  The FFTs are the shared-memory mixed-radix line
// transforms of the LS solver, applied along each axis.
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mgkmc_b200.h"
#include "fft.cuh"
#include "fieldgen.cuh"
#include "ls.cuh"

namespace mgk {
namespace {

__device__ __forceinline__ unsigned temper_word(unsigned y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// One CTA: outputs k = 0 .. nwords-1 of the stream whose state (x[0..623],
// twist pending) is `state`.
__global__ void mt_words_kernel(const unsigned* state, long nwords, unsigned* out) {
    __shared__ unsigned x[624];
    for (int i = threadIdx.x; i < 624; i += blockDim.x) x[i] = state[i];
    __syncthreads();
    // x[n] for n >= 624 lives at x[n % 624]; a chunk of 227 new words reads
    // only words written before the chunk
    for (long n0 = 624; n0 < 624 + nwords; n0 += 227) {
        const long n1 = min(n0 + 227, 624 + nwords);
        unsigned v = 0;
        const long n = n0 + threadIdx.x;
        if (n < n1) {
            const unsigned a = x[(n - 624) % 624], b = x[(n - 623) % 624];
            const unsigned y = (a & 0x80000000u) | (b & 0x7fffffffu);
            v = x[(n - 227) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        __syncthreads();
        if (n < n1) {
            x[n % 624] = v;
            out[n - 624] = temper_word(v);
        }
        __syncthreads();
    }
}

// material_generator.hpp:121-128 for voxel i from words 2i, 2i+1
__global__ void box_muller_kernel(const unsigned* w, long N, cplx<double>* z, int* redraw) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        const unsigned r1 = w[2 * i], r2 = w[2 * i + 1];
        if (r1 == 0u) atomicOr(redraw, 1);  // u1 = 0 <= 1e-15: the reference draws u1 again
        const double u1 = __ddiv_rn((double)r1, 4294967296.0), u2 = __ddiv_rn((double)r2, 4294967296.0);
        const double g = __dmul_rn(__dsqrt_rn(__dmul_rn(-2.0, log(u1))), cos(__dmul_rn(__dmul_rn(2.0, 3.14159265358979323846), u2)));
        z[i] = {g, 0.0};
    }
}

// Complex FFT along one axis of the (nx, ny, nz) row-major complex field:
// every CTA transforms `per` lines at a time in shared memory.
__global__ void fft_axis_kernel(cplx<double>* z, int nx, int ny, int nz, int axis, FftAxis ax, int per, int sign) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = ax.n, ls = pad_len(n);
    cplx<double>* b0 = reinterpret_cast<cplx<double>*>(smem);
    cplx<double>* b1 = b0 + (size_t)per * ls;
    const long nlines = (long)nx * ny * nz / n;
    // line l: its start and stride in the field
    auto line = [&](long l, long* base, long* stride) {
        if (axis == 2) {
            *base = l * nz;
            *stride = 1;
        } else if (axis == 1) {
            const long x = l / nz, zz = l % nz;
            *base = x * (long)ny * nz + zz;
            *stride = nz;
        } else {
            *base = l;  // l = y * nz + z
            *stride = (long)ny * nz;
        }
    };
    for (long l0 = (long)blockIdx.x * per; l0 < nlines; l0 += (long)gridDim.x * per) {
        const int cnt = (int)min((long)per, nlines - l0);
        for (int idx = threadIdx.x; idx < cnt * n; idx += blockDim.x) {
            const int li = idx / n, e = idx - li * n;
            long base, stride;
            line(l0 + li, &base, &stride);
            b0[li * ls + pad_idx(e)] = z[base + e * stride];
        }
        __syncthreads();
        cplx<double>* r = fft_lines<double>(b0, b1, cnt, ax, sign);
        for (int idx = threadIdx.x; idx < cnt * n; idx += blockDim.x) {
            const int li = idx / n, e = idx - li * n;
            long base, stride;
            line(l0 + li, &base, &stride);
            z[base + e * stride] = r[li * ls + pad_idx(e)];
        }
        __syncthreads();
    }
}

MGK_DEV double freq(int i, int n) {  // fftfreq(n) * 1: (i < ceil(n/2) ? i : i - n) / n
    return (double)(i < (n + 1) / 2 ? i : i - n) / (double)n;
}

// Gaussian filter and both orthonormal scalings (1/sqrt(N) twice = 1/N)
__global__ void filter_kernel(cplx<double>* z, int nx, int ny, int nz, int dim, double coeff) {
    const long N = (long)nx * ny * nz;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i / ((long)ny * nz)), y = (int)((i / nz) % ny), zz = (int)(i % nz);
        double f2 = freq(x, nx) * freq(x, nx) + freq(y, ny) * freq(y, ny);
        if (dim == 3) f2 += freq(zz, nz) * freq(zz, nz);
        const double m = exp(coeff * f2) / (double)N;
        z[i] = {z[i].x * m, z[i].y * m};
    }
}

// fixed-order sums: per-block partial sums (of the real parts, or of their
// squared deviations from `mean` when dev != 0), summed by one thread in block
// order afterwards
__global__ void partial_sum_kernel(const cplx<double>* z, long N, int dev, const double* mean, double* part) {
    __shared__ double sh[256];
    double s = 0.0;
    const double m = dev ? *mean : 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        const double v = z[i].x - m;
        s += dev ? v * v : z[i].x;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void finish_sum_kernel(const double* part, int n, long N, double* out) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += part[b];
    *out = s / (double)N;
}

__global__ void scale_kernel(const cplx<double>* z, long N, const double* mean, const double* var, double target_mean,
                             double target_std, int has_min, double cmin, int has_max, double cmax, double* out) {
    double sd = sqrt(*var);
    if (sd < 1e-15) sd = 1.0;
    const double m = *mean;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        double v = target_mean + target_std * ((z[i].x - m) / sd);
        if (has_min && v < cmin) v = cmin;
        if (has_max && v > cmax) v = cmax;
        out[i] = v;
    }
}

#define FCK(x)                                                                                   \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

// Host driver; throws on CUDA errors and unsupported lengths.
void correlated_field(int dim, int nx, int ny, int nz, double mean, double sd, double corr, bool has_min, double cmin,
                      bool has_max, double cmax, int seed, double* out_host) {
    if (dim == 2) nz = 1;
    const long N = (long)nx * ny * nz;
    std::vector<void*> owned;
    cudaStream_t st = nullptr;
    FCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    auto cleanup = [&]() {
        if (st) cudaStreamSynchronize(st);
        for (void* p : owned) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    };
    try {
        auto alloc = [&](size_t b) {
            void* p = nullptr;
            FCK(cudaMalloc(&p, b));
            owned.push_back(p);
            return p;
        };
        // the seeded generator's state (624 words; its first call twists)
        std::mt19937 g((unsigned)seed);
        std::ostringstream os;
        os << g;
        std::istringstream is(os.str());
        std::vector<unsigned> state(624);
        for (int i = 0; i < 624; ++i) {
            unsigned long v;
            is >> v;
            state[i] = (unsigned)v;
        }
        auto* d_state = (unsigned*)alloc(sizeof(unsigned) * 624);
        auto* d_words = (unsigned*)alloc(sizeof(unsigned) * 2 * N);
        auto* z = (cplx<double>*)alloc(sizeof(cplx<double>) * N);
        auto* d_flag = (int*)alloc(sizeof(int) * 4);
        auto* d_stats = (double*)alloc(sizeof(double) * 2);
        const int nb = (int)std::min<long>((N + 255) / 256, 1184);
        auto* d_part = (double*)alloc(sizeof(double) * nb);
        auto* d_out = (double*)alloc(sizeof(double) * N);
        FCK(cudaMemcpyAsync(d_state, state.data(), sizeof(unsigned) * 624, cudaMemcpyHostToDevice, st));
        FCK(cudaMemsetAsync(d_flag, 0, sizeof(int) * 4, st));
        mt_words_kernel<<<1, 256, 0, st>>>(d_state, 2 * N, d_words);
        box_muller_kernel<<<nb, 256, 0, st>>>(d_words, N, z, d_flag);
        int flag = 0;
        FCK(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        FCK(cudaStreamSynchronize(st));
        if (flag) {  // a u1 word was 0: draw the normals on the host, in order
            std::mt19937 h((unsigned)seed);
            std::vector<cplx<double>> zh(N);
            for (long i = 0; i < N; ++i) {
                double u1 = (h() - h.min()) / double(h.max() - h.min() + 1.0);
                const double u2 = (h() - h.min()) / double(h.max() - h.min() + 1.0);
                while (u1 <= 1e-15) u1 = (h() - h.min()) / double(h.max() - h.min() + 1.0);
                zh[i] = {std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2), 0.0};
            }
            FCK(cudaMemcpyAsync(z, zh.data(), sizeof(cplx<double>) * N, cudaMemcpyHostToDevice, st));
        }
        const int dims[3] = {nx, ny, nz};
        FftAxis ax[3];
        for (int a = 0; a < dim; ++a)
            if (!plan_axis(dims[a], &ax[a], &owned)) throw std::invalid_argument("field axis length has a prime factor > 7");
        auto pass = [&](int sign) {
            for (int a = 0; a < dim; ++a) {
                const int n = dims[a];
                const size_t line_b = (size_t)(n + (n >> 3) + 1) * sizeof(cplx<double>);
                int per = (int)std::max<size_t>(1, std::min<size_t>(64, (48 * 1024) / (2 * line_b)));
                const size_t smem = 2 * per * line_b;
                if (smem > 48 * 1024) FCK(ensure_dyn_smem((const void*)fft_axis_kernel, smem));
                const long nlines = N / n;
                const int grid = (int)std::min<long>((nlines + per - 1) / per, 1184);
                fft_axis_kernel<<<grid, 256, smem, st>>>(z, nx, ny, nz, a, ax[a], per, sign);
                FCK(cudaGetLastError());
            }
        };
        pass(-1);
        filter_kernel<<<nb, 256, 0, st>>>(z, nx, ny, nz, dim, -2.0 * M_PI * M_PI * corr * corr);
        pass(+1);
        partial_sum_kernel<<<nb, 256, 0, st>>>(z, N, 0, nullptr, d_part);
        finish_sum_kernel<<<1, 1, 0, st>>>(d_part, nb, N, d_stats);
        partial_sum_kernel<<<nb, 256, 0, st>>>(z, N, 1, d_stats, d_part);
        finish_sum_kernel<<<1, 1, 0, st>>>(d_part, nb, N, d_stats + 1);
        scale_kernel<<<nb, 256, 0, st>>>(z, N, d_stats, d_stats + 1, mean, sd, has_min, cmin, has_max, cmax, d_out);
        FCK(cudaGetLastError());
        FCK(cudaMemcpyAsync(out_host, d_out, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
        FCK(cudaStreamSynchronize(st));
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
}

}  // namespace mgk
