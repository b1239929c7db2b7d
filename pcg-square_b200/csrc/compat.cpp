// C++ pcg_cuda:: wrappers with the reference's signatures (include/common/*.h)
// over the C ABI: std::function exchange callbacks are bridged through a
// trampoline, and failures are rethrown as std::runtime_error like the
// reference (GPU_baseline/common/dpf_gpu.cu:35-40, poly_mul_cuda.cu:426-436).
#include <exception>
#include <stdexcept>
#include <string>

#include "common/aes_gpu.h"
#include "common/dpf_gpu.h"
#include "common/leaf_convert_cuda.h"
#include "common/poly_mul_cuda.h"
#include "pcg_b200.h"

static_assert(sizeof(pcg_cuda::DpfBlk) == sizeof(pcgb_blk), "DpfBlk layout");

namespace pcg_cuda {
namespace {

void rethrow(int rc) {
    if (rc != PCGB_OK) throw std::runtime_error(pcgb_last_error());
}

struct Bridge {
    const DpfExchangeFn* fn;
    std::exception_ptr err;
};

int trampoline(const pcgb_blk* my, pcgb_blk* peer, size_t count, void* user) {
    auto* b = static_cast<Bridge*>(user);
    try {
        (*b->fn)(reinterpret_cast<const DpfBlk*>(my), reinterpret_cast<DpfBlk*>(peer), count);
        return 0;
    } catch (...) {
        b->err = std::current_exception();
        return 1;
    }
}

int prg_code(DpfGpuPrg p) { return p == DpfGpuPrg::CHACHA8 ? PCGB_PRG_CHACHA8 : PCGB_PRG_AES; }

bool supported(int variant, uint64_t prime, int N, std::string* reason) {
    char buf[256] = {0};
    const int r = pcgb_poly_mul_supported(variant, prime, N, buf, sizeof(buf));
    if (reason) *reason = buf;
    return r == 1;
}

void mul(int variant, uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
         uint64_t prime, PolyMulStats* stats) {
    double ms = 0;
    rethrow(pcgb_poly_mul_u64(variant, out, a, b, batch, N, prime, stats ? &ms : nullptr));
    if (stats) stats->device_ms = ms;
}

}  // namespace

void dpf_gpu_batch_full_eval(int B, int n, int w, const DpfBlk* roots, const DpfBlk* dltsft,
                             const uint8_t* round_keys, int party, const DpfExchangeFn& exchange,
                             DpfBlk* out_leaves, DpfGpuPrg prg) {
    Bridge br{&exchange, nullptr};
    const int rc = pcgb_dpf_batch_full_eval(
        B, n, w, reinterpret_cast<const pcgb_blk*>(roots), reinterpret_cast<const pcgb_blk*>(dltsft),
        round_keys, party, exchange ? trampoline : nullptr, &br,
        reinterpret_cast<pcgb_blk*>(out_leaves), prg_code(prg));
    if (br.err) std::rethrow_exception(br.err);
    rethrow(rc);
}

const DpfBlk* dpf_gpu_batch_full_eval_device(int B, int n, int w, const DpfBlk* roots,
                                             const DpfBlk* dltsft, const uint8_t* round_keys,
                                             int party, const DpfExchangeFn& exchange,
                                             DpfGpuPrg prg) {
    Bridge br{&exchange, nullptr};
    const pcgb_blk* d = nullptr;
    const int rc = pcgb_dpf_batch_full_eval_device(
        B, n, w, reinterpret_cast<const pcgb_blk*>(roots), reinterpret_cast<const pcgb_blk*>(dltsft),
        round_keys, party, exchange ? trampoline : nullptr, &br, prg_code(prg), &d);
    if (br.err) std::rethrow_exception(br.err);
    rethrow(rc);
    return reinterpret_cast<const DpfBlk*>(d);
}

void dpf_out_sums(const DpfBlk* d_leaves, int B, size_t D, uint64_t prime, uint64_t* sumC_host,
                  uint64_t* sumT_host) {
    rethrow(pcgb_dpf_out_sums(reinterpret_cast<const pcgb_blk*>(d_leaves), B, D, prime, sumC_host,
                              sumT_host));
}

void dpf_out_scatter_g(const DpfBlk* d_leaves, int B, size_t D, int t, int party, uint64_t prime,
                       const uint64_t* CW_host, uint64_t* g_out_host, int N) {
    rethrow(pcgb_dpf_out_scatter_g(reinterpret_cast<const pcgb_blk*>(d_leaves), B, D, t, party,
                                   prime, CW_host, g_out_host, N));
}

bool is_cuda_available() { return pcgb_is_cuda_available() == 1; }

std::string device_name() {
    char buf[256] = {0};
    return pcgb_device_name(buf, sizeof(buf)) == PCGB_OK ? std::string(buf) : "unavailable";
}

std::string runtime_version() {
    char buf[64] = {0};
    return pcgb_runtime_version(buf, sizeof(buf)) == PCGB_OK ? std::string(buf) : "unavailable";
}

bool poly_mul_supported(uint64_t prime, int N, std::string* reason) {
    return supported(PCGB_POLYMUL_V1, prime, N, reason);
}
void poly_mul_u64(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
                  uint64_t prime, PolyMulStats* stats) {
    mul(PCGB_POLYMUL_V1, out, a, b, batch, N, prime, stats);
}
bool poly_mul_gpuntt_supported(uint64_t prime, int N, std::string* reason) {
    return supported(PCGB_POLYMUL_MERGE, prime, N, reason);
}
void poly_mul_u64_gpuntt(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
                         uint64_t prime, PolyMulStats* stats) {
    mul(PCGB_POLYMUL_MERGE, out, a, b, batch, N, prime, stats);
}
bool poly_mul_gpuntt_4step_supported(uint64_t prime, int N, std::string* reason) {
    return supported(PCGB_POLYMUL_4STEP, prime, N, reason);
}
void poly_mul_u64_gpuntt_4step(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch,
                               int N, uint64_t prime, PolyMulStats* stats) {
    mul(PCGB_POLYMUL_4STEP, out, a, b, batch, N, prime, stats);
}
bool poly_mul_gpuntt_square_supported(uint64_t prime, int N, std::string* reason) {
    return supported(PCGB_POLYMUL_SQUARE, prime, N, reason);
}
void poly_mul_u64_gpuntt_square(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch,
                                int N, uint64_t prime, PolyMulStats* stats) {
    mul(PCGB_POLYMUL_SQUARE, out, a, b, batch, N, prime, stats);
}

void aes128_expand_key_host(const uint8_t key[16], uint8_t round_keys[176]) {
    rethrow(pcgb_aes128_expand_key(key, round_keys));
}

void aes128_ecb_encrypt_gpu(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count) {
    rethrow(pcgb_aes128_ecb_encrypt(keys, in, out, count));
}

}  // namespace pcg_cuda
