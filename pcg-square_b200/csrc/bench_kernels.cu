// Measurement helpers: the library's kernel-launch counter and an ARX
// throughput probe that bounds the ChaCha8-bound kernels from above.
//
// The probe runs the ChaCha8 double round (the same QR with PRMT/SHF
// rotations as chacha8.cuh) on two independent register-resident states per
// thread, with every SM fully occupied, and reports integer ops/s counting
// 12 ops per quarter round (4 add, 4 xor, 4 rotate).  It is the achievable
// peak for exactly the instruction mix of the DPF kernels.
#include "pcgb_internal.h"

#include <algorithm>

#include <atomic>

#include "chacha8.cuh"

namespace pcgb {
namespace {

std::atomic<unsigned long long> g_launches{0};

// Two independent ChaCha8 states per thread, every word seeded per thread,
// eight quarter-round pairs per iteration; every thread stores a digest of
// both states so no round can be pruned.
__global__ void __launch_bounds__(256) arx_probe_kernel(uint32_t seed, int iters, uint32_t* out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t x[16], y[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        x[i] = seed * (i + 1) ^ tid;
        y[i] = (seed + i) * 0x9e3779b9u + tid;
    }
    for (int it = 0; it < iters; ++it) {
        PCGB_QR(x[0], x[4], x[8], x[12])  PCGB_QR(y[0], y[4], y[8], y[12])
        PCGB_QR(x[1], x[5], x[9], x[13])  PCGB_QR(y[1], y[5], y[9], y[13])
        PCGB_QR(x[2], x[6], x[10], x[14]) PCGB_QR(y[2], y[6], y[10], y[14])
        PCGB_QR(x[3], x[7], x[11], x[15]) PCGB_QR(y[3], y[7], y[11], y[15])
        PCGB_QR(x[0], x[5], x[10], x[15]) PCGB_QR(y[0], y[5], y[10], y[15])
        PCGB_QR(x[1], x[6], x[11], x[12]) PCGB_QR(y[1], y[6], y[11], y[12])
        PCGB_QR(x[2], x[7], x[8], x[13])  PCGB_QR(y[2], y[7], y[8], y[13])
        PCGB_QR(x[3], x[4], x[9], x[14])  PCGB_QR(y[3], y[4], y[9], y[14])
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) r ^= x[i] + 3 * y[i];
    out[tid] = r;
}

// Probe variant for the pipe balance of the quarter round: the adds
// selected by M (bit 4q + k: add k of quarter round q of a double round)
// are issued as a multiply-add b * one + a with `one` read from constant
// memory, which the compiler cannot fold, so they go to the FMA pipe
// instead of the integer ALU.  Same values as the plain probe.
__constant__ uint32_t c_probe_one = 1;

__device__ __forceinline__ uint32_t add_on_fma(uint32_t a, uint32_t b, uint32_t one) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(b), "r"(one), "r"(a));
    return d;
}

template <uint32_t M, int Q>
__device__ __forceinline__ void qr_mix(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d,
                                       uint32_t one) {
    constexpr uint32_t m = (M >> (4 * Q)) & 0xF;
    a = (m & 1) ? add_on_fma(a, b, one) : a + b; d ^= a; d = rot16(d);
    c = (m & 2) ? add_on_fma(c, d, one) : c + d; b ^= c; b = rot12(b);
    a = (m & 4) ? add_on_fma(a, b, one) : a + b; d ^= a; d = rot8(d);
    c = (m & 8) ? add_on_fma(c, d, one) : c + d; b ^= c; b = rot7(b);
}

template <uint32_t M>
__device__ __forceinline__ void double_round_mix(uint32_t (&x)[16], uint32_t one) {
    qr_mix<M, 0>(x[0], x[4], x[8], x[12], one);
    qr_mix<M, 1>(x[1], x[5], x[9], x[13], one);
    qr_mix<M, 2>(x[2], x[6], x[10], x[14], one);
    qr_mix<M, 3>(x[3], x[7], x[11], x[15], one);
    qr_mix<M, 4>(x[0], x[5], x[10], x[15], one);
    qr_mix<M, 5>(x[1], x[6], x[11], x[12], one);
    qr_mix<M, 6>(x[2], x[7], x[8], x[13], one);
    qr_mix<M, 7>(x[3], x[4], x[9], x[14], one);
}

template <uint32_t M>
__global__ void __launch_bounds__(256) arx_probe_mix_kernel(uint32_t seed, int iters, uint32_t* out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t one = c_probe_one;
    uint32_t x[16], y[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        x[i] = seed * (i + 1) ^ tid;
        y[i] = (seed + i) * 0x9e3779b9u + tid;
    }
    for (int it = 0; it < iters; ++it) {
        double_round_mix<M>(x, one);
        double_round_mix<M>(y, one);
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) r ^= x[i] + 3 * y[i];
    out[tid] = r;
}

}  // namespace

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// G int-ops/s of each of `reps` launches of `iters` double-round iterations
// (after one short warm-up launch), in launch order.
void arx_probe_samples(int reps, int iters, double* gops) {
    cudaStream_t st = default_stream();
    const int sms = sm_count();
    const int blocks = sms * 8, threads = 256;
    uint32_t* sink =
        static_cast<uint32_t*>(pool_alloc(sizeof(uint32_t) * static_cast<size_t>(blocks) * threads, st));
    arx_probe_kernel<<<blocks, threads, 0, st>>>(1, 64, sink);  // warm-up
    PCGB_POST_LAUNCH();
    cudaEvent_t e0, e1;
    PCGB_CK(cudaEventCreate(&e0));
    PCGB_CK(cudaEventCreate(&e1));
    const double ops = static_cast<double>(blocks) * threads * iters * 2 /*states*/ * 8 * 12;
    for (int rep = 0; rep < reps; ++rep) {
        PCGB_CK(cudaEventRecord(e0, st));
        arx_probe_kernel<<<blocks, threads, 0, st>>>(2 + rep, iters, sink);
        PCGB_POST_LAUNCH();
        PCGB_CK(cudaEventRecord(e1, st));
        PCGB_CK(cudaEventSynchronize(e1));
        float t = 0;
        PCGB_CK(cudaEventElapsedTime(&t, e0, e1));
        gops[rep] = ops / (t * 1e-3) / 1e9;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PCGB_CK(cudaFreeAsync(sink, st));
}

// The pipe-balance variants of the probe (arx_probe_mix_kernel); returns
// false for a mask without an instance.
bool arx_probe_variant(uint32_t mask, int reps, int iters, double* gops) {
    cudaStream_t st = default_stream();
    const int blocks = sm_count() * 8, threads = 256;
    void (*kern)(uint32_t, int, uint32_t*) = nullptr;
    switch (mask) {
#define PCGB_MIX(M) \
    case M: kern = arx_probe_mix_kernel<M>; break;
        PCGB_MIX(0x00000000u) PCGB_MIX(0x10101010u) PCGB_MIX(0x11111111u)
        PCGB_MIX(0x22222222u) PCGB_MIX(0x33333333u) PCGB_MIX(0x55555555u)
        PCGB_MIX(0x15151515u) PCGB_MIX(0x77777777u) PCGB_MIX(0xFFFFFFFFu)
#undef PCGB_MIX
        default: return false;
    }
    uint32_t* sink =
        static_cast<uint32_t*>(pool_alloc(sizeof(uint32_t) * static_cast<size_t>(blocks) * threads, st));
    kern<<<blocks, threads, 0, st>>>(1, 64, sink);  // warm-up
    PCGB_POST_LAUNCH();
    cudaEvent_t e0, e1;
    PCGB_CK(cudaEventCreate(&e0));
    PCGB_CK(cudaEventCreate(&e1));
    const double ops = static_cast<double>(blocks) * threads * iters * 2 * 8 * 12;
    for (int rep = 0; rep < reps; ++rep) {
        PCGB_CK(cudaEventRecord(e0, st));
        kern<<<blocks, threads, 0, st>>>(2 + rep, iters, sink);
        PCGB_POST_LAUNCH();
        PCGB_CK(cudaEventRecord(e1, st));
        PCGB_CK(cudaEventSynchronize(e1));
        float t = 0;
        PCGB_CK(cudaEventElapsedTime(&t, e0, e1));
        gops[rep] = ops / (t * 1e-3) / 1e9;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PCGB_CK(cudaFreeAsync(sink, st));
    return true;
}

// Returns G int-ops/s of the fastest of three launches; *ms = its duration.
double arx_probe(float* ms_out) {
    constexpr int iters = 4096;
    double g[3];
    arx_probe_samples(3, iters, g);
    const double best = std::max(g[0], std::max(g[1], g[2]));
    if (ms_out) {
        const double ops = static_cast<double>(sm_count()) * 8 * 256 * iters * 2 * 8 * 12;
        *ms_out = static_cast<float>(ops / (best * 1e9) * 1e3);
    }
    return best;
}

}  // namespace pcgb
