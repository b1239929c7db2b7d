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
