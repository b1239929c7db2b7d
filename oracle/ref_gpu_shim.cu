// C entry points over the reference's own GPU kernels (GPU_baseline/common/
// dpf_gpu.cu, leaf_convert_cuda.cu, poly_mul_cuda.cu, aes_gpu.cu), compiled
// unmodified from the reference tree for sm_100a (see oracle/Makefile).
// TEST INFRASTRUCTURE: the GPU parity tests compare the library against these
// kernels, and oracle/plain_gpu_bench.py times them as the plain per-stage
// GPU path.  Never linked into the shipped library.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "common/aes_gpu.h"
#include "common/dpf_gpu.h"
#include "common/leaf_convert_cuda.h"
#include "common/poly_mul_cuda.h"

namespace {
thread_local std::string g_err;
template <class F>
int guard(F&& f) {
    try { f(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}
}  // namespace

extern "C" {

typedef void (*ref_exchange_fn)(const void* my, void* peer, size_t count, void* user);

const char* ref_last_error(void) { return g_err.c_str(); }

static pcg_cuda::DpfExchangeFn wrap(ref_exchange_fn ex, void* user) {
    return [ex, user](const pcg_cuda::DpfBlk* my, pcg_cuda::DpfBlk* peer, size_t n) {
        if (ex) ex(my, peer, n, user);
        else std::memset(peer, 0, n * sizeof(pcg_cuda::DpfBlk));
    };
}

int ref_dpf_batch_full_eval(int B, int n, int w, const void* roots, const void* dltsft,
                            const uint8_t* rks, int party, ref_exchange_fn ex, void* user,
                            void* out_leaves, int prg_chacha8) {
    return guard([&] {
        pcg_cuda::dpf_gpu_batch_full_eval(
            B, n, w, static_cast<const pcg_cuda::DpfBlk*>(roots),
            static_cast<const pcg_cuda::DpfBlk*>(dltsft), rks, party, wrap(ex, user),
            static_cast<pcg_cuda::DpfBlk*>(out_leaves),
            prg_chacha8 ? pcg_cuda::DpfGpuPrg::CHACHA8 : pcg_cuda::DpfGpuPrg::AES);
    });
}

int ref_dpf_batch_full_eval_device(int B, int n, int w, const void* roots, const void* dltsft,
                                   const uint8_t* rks, int party, ref_exchange_fn ex,
                                   void* user, int prg_chacha8, const void** d_leaves) {
    return guard([&] {
        *d_leaves = pcg_cuda::dpf_gpu_batch_full_eval_device(
            B, n, w, static_cast<const pcg_cuda::DpfBlk*>(roots),
            static_cast<const pcg_cuda::DpfBlk*>(dltsft), rks, party, wrap(ex, user),
            prg_chacha8 ? pcg_cuda::DpfGpuPrg::CHACHA8 : pcg_cuda::DpfGpuPrg::AES);
    });
}

int ref_dpf_out_sums(const void* d_leaves, int B, size_t D, uint64_t prime, uint64_t* sumC,
                     uint64_t* sumT) {
    return guard([&] {
        pcg_cuda::dpf_out_sums(static_cast<const pcg_cuda::DpfBlk*>(d_leaves), B, D, prime,
                               sumC, sumT);
    });
}

int ref_dpf_out_scatter_g(const void* d_leaves, int B, size_t D, int t, int party,
                          uint64_t prime, const uint64_t* CW, uint64_t* g, int N) {
    return guard([&] {
        pcg_cuda::dpf_out_scatter_g(static_cast<const pcg_cuda::DpfBlk*>(d_leaves), B, D, t,
                                    party, prime, CW, g, N);
    });
}

int ref_poly_mul_u64(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
                     uint64_t prime, double* device_ms) {
    return guard([&] {
        pcg_cuda::PolyMulStats st;
        pcg_cuda::poly_mul_u64(out, a, b, batch, N, prime, &st);
        if (device_ms) *device_ms = st.device_ms;
    });
}

int ref_aes128_ecb_encrypt_gpu(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count) {
    return guard([&] { pcg_cuda::aes128_ecb_encrypt_gpu(keys, in, out, count); });
}

void ref_aes128_expand_key_host(const uint8_t key[16], uint8_t rk[176]) {
    pcg_cuda::aes128_expand_key_host(key, rk);
}

// Device memory helpers for driving the device-resident entry points.
int ref_h2d(void* dst, const void* src, size_t bytes) {
    return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}
int ref_malloc(void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess ? 0 : -1; }
int ref_free(void* p) { return cudaFree(p) == cudaSuccess ? 0 : -1; }
int ref_sync(void) { return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1; }

}  // extern "C"
