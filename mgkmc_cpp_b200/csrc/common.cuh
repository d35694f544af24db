// Shared device helpers for the mgkmc B200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#define MGK_DEV __device__ __forceinline__

// Raises a kernel's dynamic shared-memory limit to at least `bytes` and never
// lowers it.  The attribute belongs to the function (per device), not to the
// object that plans a launch: two solvers of different sizes share it, so
// setting it to one launch's own need would make the other's larger launch
// fail with cudaErrorInvalidValue.
inline cudaError_t ensure_dyn_smem(const void* fn, size_t bytes) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------- error words
// Device kernels never trap: a failed bounded wait or a bad size sets a bit in
// the handle's error word and the kernel returns; the host turns it into a status.
enum : unsigned {
    MGK_DERR_BARRIER_TIMEOUT = 1u,  // a grid barrier wait ran out of iterations
    MGK_DERR_SIZE = 2u,             // a launch got a size beyond its compiled limits
    MGK_DERR_NAN = 4u,              // non-finite value in a reduction
    MGK_DERR_SELECT = 8u,           // event selection found no candidate
};

// ---------------------------------------------------------------- complex
template <typename T>
struct cplx {
    T x, y;
};

template <typename T>
MGK_DEV cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
MGK_DEV cplx<T> cmulc(cplx<T> a, cplx<T> b) {  // a * conj(b)
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename T>
MGK_DEV cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
MGK_DEV cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
MGK_DEV cplx<T> cscale(cplx<T> a, T s) { return {a.x * s, a.y * s}; }
template <typename T>
MGK_DEV cplx<T> cconj(cplx<T> a) { return {a.x, -a.y}; }

// ---------------------------------------------------------------- double-double
// Error-free two-sum (Knuth) for accurate FP64 rate sums.
struct dd {
    double hi, lo;
};
MGK_DEV dd dd_add(dd a, dd b) {
    double s = __dadd_rn(a.hi, b.hi);
    double bb = __dsub_rn(s, a.hi);
    double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b.hi, bb));
    e = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
    double h = __dadd_rn(s, e);
    return {h, __dsub_rn(e, __dsub_rn(h, s))};
}
MGK_DEV dd dd_add_d(dd a, double b) { return dd_add(a, dd{b, 0.0}); }
MGK_DEV dd dd_shfl_down(dd a, int o) {
    return {__shfl_down_sync(0xffffffffu, a.hi, o), __shfl_down_sync(0xffffffffu, a.lo, o)};
}

// ---------------------------------------------------------------- grid barrier
MGK_DEV unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Default limit of one wait at a barrier, in device time.
// (long enough for the longest one-CTA phase a group waits on: the catalog
// and barrier redraw of a cascade of ~1e5 flips of 100 modes)
constexpr unsigned long long kBarrierTimeoutNs = 120ull * 1000000000ull;

// Sense-counting barrier for persistent kernels whose CTAs are co-resident
// (launched cooperatively).  Every wait is bounded: after limit_ns of device
// time (or as soon as another CTA has given up) the CTA records
// MGK_DERR_BARRIER_TIMEOUT and the barrier reports failure, so a kernel never
// spins forever.  `bar` points at two words: {arrivals, generation}.
struct GridBar {
    unsigned* bar;
    unsigned nblocks;
    unsigned* err;
    unsigned long long limit_ns;
};

MGK_DEV bool grid_sync(const GridBar& g) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = g.bar + 1;
        unsigned my_gen = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(g.bar, 1u);
        int ok = 1;
        if (arrived == g.nblocks - 1) {
            atomicExch(g.bar, 0u);
            __threadfence();
            atomicAdd(g.bar + 1, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned polls = 0;
            while (*gen == my_gen) {
                __nanosleep(32);
                if ((*(volatile unsigned*)g.err & MGK_DERR_BARRIER_TIMEOUT) ||
                    ((++polls & 255u) == 0 && global_ns() - t0 > g.limit_ns)) {
                    atomicOr(g.err, MGK_DERR_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ok && (*(volatile unsigned*)g.err & MGK_DERR_BARRIER_TIMEOUT)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------- reductions
template <typename T>
MGK_DEV T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread (deterministic order); result valid in
// thread 0.  `scratch` holds NV * 32 values.
template <int NV>
MGK_DEV void block_sum(double* v, double* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[k * 32 + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? scratch[k * 32 + lane] : 0.0;
            v[k] = warp_sum(x);
        }
    }
    __syncthreads();
}
