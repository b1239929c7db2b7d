// extern "C" entry points of include/pcg_b200.h: argument checks, error
// codes and the thread-local last-error message around the pcgb:: internals.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "pcg_b200.h"
#include "pcgb_internal.h"

namespace pcgb {

// Implemented in the .cu translation units.
const Blk* dpf_interactive_device(int B, int n, int w, const Blk* roots, const Blk* dltsft,
                                  const uint8_t* rks, int prg, pcgb_exchange_fn ex, void* user,
                                  Blk* host_out);
void dpf_interactive_convert_device(int B, int n, int w, const Blk* roots, const Blk* dltsft,
                                    const uint8_t* rks, int prg, pcgb_exchange_fn ex, void* user,
                                    uint64_t* d_conv, uint64_t* d_sumC, uint64_t* d_sumT,
                                    pcgb_exchange_device_fn dex = nullptr,
                                    void* dex_user = nullptr);
void dpf_out_sums_host(const Blk* d_leaves, int B, size_t D, uint64_t prime, uint64_t* sumC,
                       uint64_t* sumT);
void dpf_out_scatter_host(const Blk* d_leaves, int B, size_t D, int t, int party, uint64_t prime,
                          const uint64_t* CW, uint64_t* g_out, int N);
void dpf_out_scatter_device(const Blk* d_leaves, int B, size_t D, int t, int party,
                            const uint64_t* d_cw, uint64_t* d_g, int N, cudaStream_t st);
void aes_ecb_encrypt_device(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count);
void dpf_out_sums_noalloc(const Blk* d_leaves, int B, size_t D, uint64_t prime, uint64_t* d_sumC,
                          uint64_t* d_sumT, cudaStream_t st);
void dpf_out_convert_device(const Blk* d_leaves, int B, size_t D, uint64_t* d_conv,
                            uint64_t* d_sumC, uint64_t* d_sumT, cudaStream_t st);
void dpf_out_scatter_conv_device(const uint64_t* d_conv, int B, size_t D, int t, int party,
                                 const uint64_t* d_cw, uint64_t* d_g, int N, cudaStream_t st);
void out_beaver_open_device(int B, int party, const uint64_t* d_sumC, const uint64_t* d_sumT,
                            const uint64_t* d_beta, const uint64_t* d_r, const uint64_t* d_s,
                            uint64_t* d_de, cudaStream_t st);
void out_beaver_close_device(int B, int party, const uint64_t* d_de_my, const uint64_t* d_de_peer,
                             const uint64_t* d_r, const uint64_t* d_s, const uint64_t* d_rs,
                             uint64_t* d_cw, cudaStream_t st);
void expander_destroy(pcgb_expander* e);
void expand_device(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                   const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val, uint64_t* x,
                   uint64_t* z, cudaStream_t st);
void expand_host(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                 const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val, uint64_t* x,
                 uint64_t* z);
void expand_g_device(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                     const uint64_t* cw_out, uint64_t* d_g, cudaStream_t st);
void expander_info(const pcgb_expander* e, int* K, int* levels, int* nk, size_t* scratch);
void expander_set_profiling(pcgb_expander* e, int slots);
int expander_stage_times(pcgb_expander* e, float* ms, int max_exp);
void noise_host(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val);
void public_a_host(int N, int c, uint64_t a_seed, uint64_t* a);
void deal_keys_device(pcgb_expander* e, uint64_t seed, Blk* r0, Blk* r1, Blk* cws, uint64_t* cwo,
                      cudaStream_t st);
unsigned long long launch_count();
pcgb_server* server_create(int n_streams, size_t budget, int max_in_flight, uint64_t a_seed);
void server_prepare(pcgb_server* s, int N, int c, int t);
uint64_t server_submit(pcgb_server* s, const pcgb_request& r);
int server_wait(pcgb_server* s, uint64_t ticket, pcgb_result* out, int timeout_ms);
void server_run_trace(pcgb_server* s, const pcgb_request* reqs, int n, pcgb_result* out,
                      double timeout_s);
void server_destroy(pcgb_server* s, int timeout_ms);
void server_stats(pcgb_server* s, int* pending, int* in_flight, size_t* bytes, int* plans);
double arx_probe(float* ms_out);
void arx_probe_samples(int reps, int iters, double* gops);
bool arx_probe_variant(uint32_t mask, int reps, int iters, double* gops);

namespace {
thread_local std::string g_last_error;

int device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <class F>
int guarded(F&& f) {
    try {
        if (device_count() == 0) {
            g_last_error = "no CUDA device is available";
            return PCGB_ENODEV;
        }
        f();
        return PCGB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return PCGB_ENOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return PCGB_EINVAL;
    }
}

bool pow2(long long v) { return v > 0 && (v & (v - 1)) == 0; }

int ilog2i(long long v) {
    int l = 0;
    while ((1ll << l) < v) ++l;
    return l;
}

void copy_str(char* buf, size_t len, const std::string& s) {
    if (!buf || len == 0) return;
    std::snprintf(buf, len, "%s", s.c_str());
}

}  // namespace

void fail(int code, const std::string& msg) { throw Error(code, msg); }

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? PCGB_ENOMEM : PCGB_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

cudaStream_t default_stream() {
    static std::mutex mu;
    static cudaStream_t streams[64] = {nullptr};
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    if (!streams[dev]) check_cuda(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking),
                                  "cudaStreamCreate");
    return streams[dev];
}

cudaMemPool_t library_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {nullptr};
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        check_cuda(cudaMemPoolCreate(&pools[dev], &props), "cudaMemPoolCreate");
        // The default threshold (0) hands freed memory back at every
        // synchronisation, so each call would map its scratch again.
        uint64_t keep = UINT64_MAX;
        check_cuda(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep),
                   "cudaMemPoolSetAttribute");
    }
    return pools[dev];
}

void* pool_alloc(size_t bytes, cudaStream_t st) {
    void* p = nullptr;
    check_cuda(cudaMallocFromPoolAsync(&p, bytes, library_pool(), st), "cudaMallocFromPoolAsync");
    return p;
}

void upload_blocking(void* d_dst, const void* src, size_t bytes) {
    cudaStream_t st = default_stream();
    check_cuda(cudaMemcpyAsync(d_dst, src, bytes, cudaMemcpyHostToDevice, st), "upload");
    check_cuda(cudaStreamSynchronize(st), "upload sync");
}

int sm_count() {
    int dev = 0, n = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "sm count");
    return n;
}

// Supported-size rules of the reference's poly-mul entry points.
bool poly_mul_rules(int variant, uint64_t prime, int N, std::string* reason) {
    auto no = [&](const char* r) {
        if (reason) *reason = r;
        return false;
    };
    if (prime != kP) return no("CUDA backend only supports the project 62-bit prime");
    switch (variant) {
        case PCGB_POLYMUL_V1:
            if (!pow2(N) || N < 2 || N > 32768) return no("CUDA backend requires power-of-two N in [2,32768]");
            break;
        case PCGB_POLYMUL_MERGE:
            if (!pow2(N) || N < 2 || N > (1 << kMaxLogN)) return no("requires power-of-two N in [2, 2^24]");
            break;
        case PCGB_POLYMUL_4STEP:
            if (!pow2(N) || N < 4096 || N > (1 << kMaxLogN)) return no("4-step requires power-of-two N in [4096, 2^24]");
            break;
        case PCGB_POLYMUL_SQUARE:
            if (!pow2(N) || N < 256 || N > (1 << kMaxLogN)) return no("square requires logN in [8, 24]");
            break;
        default: return no("unknown poly-mul variant");
    }
    if ((prime - 1) % (2 * static_cast<uint64_t>(N)) != 0) return no("prime is not NTT-friendly for this N");
    if (device_count() == 0) return no("no CUDA device is available");
    if (reason) reason->clear();
    return true;
}

}  // namespace pcgb

using pcgb::Blk;
using pcgb::guarded;

extern "C" {

const char* pcgb_last_error(void) { return pcgb::g_last_error.c_str(); }
int pcgb_version(void) { return 100; }

int pcgb_is_cuda_available(void) { return pcgb::device_count() > 0 ? 1 : 0; }

int pcgb_device_name(char* buf, size_t len) {
    return guarded([&] {
        int dev = 0;
        PCGB_CK(cudaGetDevice(&dev));
        cudaDeviceProp prop;
        PCGB_CK(cudaGetDeviceProperties(&prop, dev));
        pcgb::copy_str(buf, len, prop.name);
    });
}

int pcgb_runtime_version(char* buf, size_t len) {
    int v = 0;
    if (cudaRuntimeGetVersion(&v) != cudaSuccess) {
        pcgb::copy_str(buf, len, "unavailable");
        return PCGB_ECUDA;
    }
    pcgb::copy_str(buf, len, std::to_string(v / 1000) + "." + std::to_string((v % 1000) / 10));
    return PCGB_OK;
}

int pcgb_set_device(int dev) { return guarded([&] { PCGB_CK(cudaSetDevice(dev)); }); }
int pcgb_get_device(int* dev) { return guarded([&] { PCGB_CK(cudaGetDevice(dev)); }); }
int pcgb_sm_count(int* n) { return guarded([&] { *n = pcgb::sm_count(); }); }

int pcgb_malloc(void** p, size_t bytes) { return guarded([&] { PCGB_CK(cudaMalloc(p, bytes)); }); }
int pcgb_free(void* p) { return guarded([&] { PCGB_CK(cudaFree(p)); }); }

int pcgb_memcpy_h2d(void* d, const void* s, size_t bytes, void* stream) {
    return guarded([&] {
        cudaStream_t st = pcgb::as_stream(stream);
        PCGB_CK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyHostToDevice, st));
        PCGB_CK(cudaStreamSynchronize(st));
    });
}
int pcgb_memcpy_d2h(void* d, const void* s, size_t bytes, void* stream) {
    return guarded([&] {
        cudaStream_t st = pcgb::as_stream(stream);
        PCGB_CK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToHost, st));
        PCGB_CK(cudaStreamSynchronize(st));
    });
}
int pcgb_memset(void* d, int v, size_t bytes, void* stream) {
    return guarded([&] { PCGB_CK(cudaMemsetAsync(d, v, bytes, pcgb::as_stream(stream))); });
}
int pcgb_stream_synchronize(void* stream) {
    return guarded([&] { PCGB_CK(cudaStreamSynchronize(pcgb::as_stream(stream))); });
}
int pcgb_trim_pool(void) {
    return guarded([&] {
        cudaStream_t st = pcgb::default_stream();
        PCGB_CK(cudaStreamSynchronize(st));
        PCGB_CK(cudaMemPoolTrimTo(pcgb::library_pool(), 0));
    });
}

int pcgb_device_synchronize(void) { return guarded([&] { PCGB_CK(cudaDeviceSynchronize()); }); }
void* pcgb_default_stream(void) {
    void* s = nullptr;
    guarded([&] { s = pcgb::default_stream(); });
    return s;
}

unsigned long long pcgb_launch_count(void) { return pcgb::launch_count(); }

int pcgb_arx_peak(double* gops, float* ms) {
    return guarded([&] {
        const double g = pcgb::arx_probe(ms);
        if (gops) *gops = g;
    });
}

int pcgb_arx_peak_samples(int reps, int iters, double* gops) {
    return guarded([&] {
        if (reps < 1 || iters < 1 || !gops)
            pcgb::fail(PCGB_EINVAL, "arx_peak_samples: reps and iters must be positive");
        pcgb::arx_probe_samples(reps, iters, gops);
    });
}

int pcgb_arx_peak_variant(uint32_t add_mask, int reps, int iters, double* gops) {
    return guarded([&] {
        if (reps < 1 || iters < 1 || !gops)
            pcgb::fail(PCGB_EINVAL, "arx_peak_variant: reps and iters must be positive");
        if (!pcgb::arx_probe_variant(add_mask, reps, iters, gops))
            pcgb::fail(PCGB_EINVAL, "arx_peak_variant: no probe instance for this add mask");
    });
}

int pcgb_event_create(void** ev) {
    return guarded([&] {
        cudaEvent_t e = nullptr;
        PCGB_CK(cudaEventCreate(&e));
        *ev = e;
    });
}
int pcgb_event_destroy(void* ev) {
    return guarded([&] { PCGB_CK(cudaEventDestroy(static_cast<cudaEvent_t>(ev))); });
}
int pcgb_event_record(void* ev, void* stream) {
    return guarded([&] {
        PCGB_CK(cudaEventRecord(static_cast<cudaEvent_t>(ev), pcgb::as_stream(stream)));
    });
}
int pcgb_event_elapsed(void* start, void* stop, float* ms) {
    return guarded([&] {
        PCGB_CK(cudaEventSynchronize(static_cast<cudaEvent_t>(stop)));
        PCGB_CK(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start),
                                     static_cast<cudaEvent_t>(stop)));
    });
}

// ---- DPF drop-ins -------------------------------------------------------
int pcgb_dpf_batch_full_eval(int B, int n, int w, const pcgb_blk* roots, const pcgb_blk* dltsft,
                             const uint8_t* round_keys, int party, pcgb_exchange_fn exchange,
                             void* user, pcgb_blk* out_leaves, int prg) {
    (void)party;
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        if (!out_leaves) pcgb::fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: null out_leaves");
        pcgb::dpf_interactive_device(B, n, w, reinterpret_cast<const Blk*>(roots),
                                     reinterpret_cast<const Blk*>(dltsft), round_keys, prg,
                                     exchange, user, reinterpret_cast<Blk*>(out_leaves));
    });
}

int pcgb_dpf_batch_full_eval_device(int B, int n, int w, const pcgb_blk* roots,
                                    const pcgb_blk* dltsft, const uint8_t* round_keys, int party,
                                    pcgb_exchange_fn exchange, void* user, int prg,
                                    const pcgb_blk** d_leaves) {
    (void)party;
    if (d_leaves) *d_leaves = nullptr;
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        const Blk* p = pcgb::dpf_interactive_device(B, n, w, reinterpret_cast<const Blk*>(roots),
                                                    reinterpret_cast<const Blk*>(dltsft),
                                                    round_keys, prg, exchange, user, nullptr);
        if (d_leaves) *d_leaves = reinterpret_cast<const pcgb_blk*>(p);
    });
}

size_t pcgb_gmw_position_add_gates(int off_bits) { return pcgb::gmw_position_add_gates(off_bits); }

int pcgb_gmw_position_add(int party, int B, int off_bits, const uint64_t* my_off,
                          const uint32_t* triple_a, const uint32_t* triple_b,
                          const uint32_t* triple_c, pcgb_exchange_fn exchange, void* user,
                          uint64_t* alpha_share) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::gmw_position_add(party, B, off_bits, my_off, triple_a, triple_b, triple_c, exchange,
                               user, alpha_share, pcgb::default_stream());
    });
}

size_t pcgb_gmw_dltsft_gates(int n, int w) { return pcgb::gmw_dltsft_gates(n, w); }

int pcgb_gmw_dltsft(int party, int B, int n, int w, const uint64_t* alpha_share,
                    pcgb_blk* delta_share, const uint32_t* triple_a, const uint32_t* triple_b,
                    const uint32_t* triple_c, pcgb_exchange_fn exchange, void* user,
                    pcgb_blk* dltsft) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::gmw_dltsft(party, B, n, w, alpha_share, reinterpret_cast<Blk*>(delta_share),
                         triple_a, triple_b, triple_c, exchange, user,
                         reinterpret_cast<Blk*>(dltsft), pcgb::default_stream());
    });
}

int pcgb_dpf_out_sums(const pcgb_blk* d_leaves, int B, size_t D, uint64_t prime,
                      uint64_t* sumC_host, uint64_t* sumT_host) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_sums_host(reinterpret_cast<const Blk*>(d_leaves), B, D, prime, sumC_host,
                                sumT_host);
    });
}

int pcgb_dpf_out_scatter_g_device(const pcgb_blk* d_leaves, int B, size_t D, int t, int party,
                                  const uint64_t* d_cw, uint64_t* d_g, int N, void* stream) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_scatter_device(reinterpret_cast<const Blk*>(d_leaves), B, D, t, party, d_cw,
                                     d_g, N, pcgb::as_stream(stream));
    });
}

int pcgb_dpf_out_scatter_g(const pcgb_blk* d_leaves, int B, size_t D, int t, int party,
                           uint64_t prime, const uint64_t* CW_host, uint64_t* g_out_host, int N) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_scatter_host(reinterpret_cast<const Blk*>(d_leaves), B, D, t, party, prime,
                                   CW_host, g_out_host, N);
    });
}

int pcgb_dpf_out_sums_noalloc(const pcgb_blk* d_leaves, int B, size_t D, uint64_t prime,
                              uint64_t* d_sumC, uint64_t* d_sumT, void* stream) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_sums_noalloc(reinterpret_cast<const Blk*>(d_leaves), B, D, prime, d_sumC,
                                   d_sumT, pcgb::as_stream(stream));
    });
}

int pcgb_dpf_batch_full_eval_convert_device(int B, int n, int w, const pcgb_blk* roots,
                                            const pcgb_blk* dltsft, const uint8_t* round_keys,
                                            int party, pcgb_exchange_fn exchange, void* user,
                                            int prg, uint64_t* d_conv, uint64_t* d_sumC,
                                            uint64_t* d_sumT) {
    (void)party;
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_interactive_convert_device(B, n, w, reinterpret_cast<const Blk*>(roots),
                                             reinterpret_cast<const Blk*>(dltsft), round_keys, prg,
                                             exchange, user, d_conv, d_sumC, d_sumT);
    });
}

int pcgb_dpf_batch_full_eval_convert_device_dx(int B, int n, int w, const pcgb_blk* roots,
                                               const pcgb_blk* dltsft, const uint8_t* round_keys,
                                               int party, pcgb_exchange_device_fn exchange,
                                               void* user, int prg, uint64_t* d_conv,
                                               uint64_t* d_sumC, uint64_t* d_sumT) {
    (void)party;
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        if (!exchange) pcgb::fail(PCGB_EINVAL, "device exchange callback required");
        pcgb::dpf_interactive_convert_device(B, n, w, reinterpret_cast<const Blk*>(roots),
                                             reinterpret_cast<const Blk*>(dltsft), round_keys, prg,
                                             nullptr, nullptr, d_conv, d_sumC, d_sumT, exchange,
                                             user);
    });
}

int pcgb_dpf_out_convert_device(const pcgb_blk* d_leaves, int B, size_t D, uint64_t* d_conv,
                                uint64_t* d_sumC, uint64_t* d_sumT, void* stream) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_convert_device(reinterpret_cast<const Blk*>(d_leaves), B, D, d_conv, d_sumC,
                                     d_sumT, pcgb::as_stream(stream));
    });
}

int pcgb_dpf_out_scatter_g_conv_device(const uint64_t* d_conv, int B, size_t D, int t, int party,
                                       const uint64_t* d_cw, uint64_t* d_g, int N, void* stream) {
    if (B <= 0) return PCGB_OK;
    return guarded([&] {
        pcgb::dpf_out_scatter_conv_device(d_conv, B, D, t, party, d_cw, d_g, N,
                                          pcgb::as_stream(stream));
    });
}

int pcgb_out_beaver_open_device(int B, int party, const uint64_t* d_sumC, const uint64_t* d_sumT,
                                const uint64_t* d_beta, const uint64_t* d_r, const uint64_t* d_s,
                                uint64_t* d_de, void* stream) {
    return guarded([&] {
        pcgb::out_beaver_open_device(B, party, d_sumC, d_sumT, d_beta, d_r, d_s, d_de,
                                     pcgb::as_stream(stream));
    });
}

int pcgb_out_beaver_close_device(int B, int party, const uint64_t* d_de_my,
                                 const uint64_t* d_de_peer, const uint64_t* d_r,
                                 const uint64_t* d_s, const uint64_t* d_rs, uint64_t* d_cw_share,
                                 void* stream) {
    return guarded([&] {
        pcgb::out_beaver_close_device(B, party, d_de_my, d_de_peer, d_r, d_s, d_rs, d_cw_share,
                                      pcgb::as_stream(stream));
    });
}

// ---- poly-mul drop-ins --------------------------------------------------
int pcgb_poly_mul_supported(int variant, uint64_t prime, int N, char* reason, size_t len) {
    std::string r;
    const bool ok = pcgb::poly_mul_rules(variant, prime, N, &r);
    pcgb::copy_str(reason, len, r);
    return ok ? 1 : 0;
}

int pcgb_poly_mul_u64(int variant, uint64_t* out, const uint64_t* a, const uint64_t* b, int batch,
                      int N, uint64_t prime, double* device_ms) {
    return guarded([&] {
        std::string why;
        if (!pcgb::poly_mul_rules(variant, prime, N, &why)) pcgb::fail(PCGB_EINVAL, why);
        if (batch <= 0) pcgb::fail(PCGB_EINVAL, "batch must be positive");
        const pcgb::NttPlan& pl = pcgb::ntt_plan(pcgb::ilog2i(N));
        cudaStream_t st = pcgb::default_stream();
        const size_t n = static_cast<size_t>(batch) * N;
        uint64_t* d = nullptr;
        d = static_cast<uint64_t*>(pcgb::pool_alloc(5 * n * sizeof(uint64_t), st));
        uint64_t *da = d, *db = d + n, *dc = d + 2 * n, *scratch = d + 3 * n;
        PCGB_CK(cudaMemcpyAsync(da, a, n * 8, cudaMemcpyHostToDevice, st));
        PCGB_CK(cudaMemcpyAsync(db, b, n * 8, cudaMemcpyHostToDevice, st));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (device_ms) {
            PCGB_CK(cudaEventCreate(&e0));
            PCGB_CK(cudaEventCreate(&e1));
            PCGB_CK(cudaEventRecord(e0, st));
        }
        pcgb::poly_mul_device(pl, dc, da, db, batch, scratch, st);
        if (device_ms) PCGB_CK(cudaEventRecord(e1, st));
        PCGB_CK(cudaMemcpyAsync(out, dc, n * 8, cudaMemcpyDeviceToHost, st));
        PCGB_CK(cudaFreeAsync(d, st));
        PCGB_CK(cudaStreamSynchronize(st));
        if (device_ms) {
            float ms = 0;
            PCGB_CK(cudaEventElapsedTime(&ms, e0, e1));
            *device_ms = ms;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
    });
}

// ---- AES ------------------------------------------------------------------
int pcgb_aes128_expand_key(const uint8_t key[16], uint8_t round_keys[176]) {
    try {
        pcgb::aes_expand_key_host(key, round_keys);
        return PCGB_OK;
    } catch (const std::exception& e) {
        pcgb::g_last_error = e.what();
        return PCGB_EINVAL;
    }
}

int pcgb_aes128_ecb_encrypt(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count) {
    if (count <= 0) return PCGB_OK;
    return guarded([&] { pcgb::aes_ecb_encrypt_device(keys, in, out, count); });
}

int pcgb_aes_tree_round_keys(const uint8_t master[16], int nk, uint8_t* round_keys) {
    if (nk < 1 || nk > 15) {
        pcgb::g_last_error = "nk must be in [1, 15]";
        return PCGB_EINVAL;
    }
    pcgb::aes_tree_round_keys_host(master, nk, round_keys);
    return PCGB_OK;
}

// ---- keyed DPF --------------------------------------------------------------
int pcgb_dpf_keyed_full_eval_multi(int groups, const int* K, const int* n, int w, int prg,
                                   const pcgb_blk* const* d_roots, const pcgb_blk* const* d_cws,
                                   const uint8_t* round_keys, pcgb_blk* const* d_leaves,
                                   void* stream) {
    if (groups <= 0) return PCGB_OK;
    return guarded([&] {
        if (prg != PCGB_PRG_AES && prg != PCGB_PRG_CHACHA8)
            pcgb::fail(PCGB_EINVAL, "keyed eval multi: unknown PRG");
        if (prg == PCGB_PRG_AES && !round_keys)
            pcgb::fail(PCGB_EINVAL, "keyed eval multi: AES needs round keys");
        if (w < 1 || w > 4) pcgb::fail(PCGB_EINVAL, "keyed eval multi: w must be in [1,4]");
        cudaStream_t st = pcgb::as_stream(stream);
        uint32_t* d_rk = nullptr;
        if (prg == PCGB_PRG_AES) d_rk = pcgb::aes_upload_round_keys(round_keys, (1 << w) - 1, st);
        try {
            pcgb::keyed_full_eval_multi(groups, K, n, w, prg,
                                        reinterpret_cast<const Blk* const*>(d_roots),
                                        reinterpret_cast<const Blk* const*>(d_cws), d_rk,
                                        reinterpret_cast<Blk* const*>(d_leaves), st);
        } catch (...) {
            if (d_rk) {
                cudaStreamSynchronize(st);
                cudaFree(d_rk);
            }
            throw;
        }
        if (d_rk) {   // a plain allocation: free once the launches that read it are done
            PCGB_CK(cudaStreamSynchronize(st));
            cudaFree(d_rk);
        }
    });
}

int pcgb_dpf_keyed_full_eval(int K, int n, int w, int prg, const pcgb_blk* d_roots,
                             const pcgb_blk* d_cws, const uint8_t* round_keys,
                             pcgb_blk* d_leaves, void* stream) {
    if (K <= 0) return PCGB_OK;
    return guarded([&] {
        if (w < 1 || w > 4 || n < 1 || n % w || n > 30) pcgb::fail(PCGB_EINVAL, "keyed eval: bad (n, w)");
        if (prg == PCGB_PRG_AES && !round_keys) pcgb::fail(PCGB_EINVAL, "keyed eval: AES needs round keys");
        cudaStream_t st = pcgb::as_stream(stream);
        const int levels = n / w, nk = (1 << w) - 1;
        uint32_t* d_rk = nullptr;
        if (prg == PCGB_PRG_AES) d_rk = pcgb::aes_upload_round_keys(round_keys, nk, st);
        const size_t sn = pcgb::keyed_tops_scratch_nodes(K, w, levels);
        Blk* scratch = nullptr;
        if (sn) scratch = static_cast<Blk*>(pcgb::pool_alloc(sn * sizeof(Blk), st));
        pcgb::keyed_expand_tops(K, n, w, prg, reinterpret_cast<const Blk*>(d_roots),
                                reinterpret_cast<const Blk*>(d_cws), d_rk, levels,
                                reinterpret_cast<Blk*>(d_leaves), scratch, st);
        if (scratch) PCGB_CK(cudaFreeAsync(scratch, st));
        if (d_rk) {
            PCGB_CK(cudaStreamSynchronize(st));
            cudaFree(d_rk);
        }
    });
}

// ---- batched NTT ------------------------------------------------------------
int pcgb_poly_mul_device(uint64_t* d_c, const uint64_t* d_a, const uint64_t* d_b, int batch, int N,
                         void* stream) {
    return guarded([&] {
        if (!pcgb::pow2(N) || N < 2 || N > (1 << pcgb::kMaxLogN)) pcgb::fail(PCGB_EINVAL, "N must be a power of two in [2, 2^24]");
        if (batch <= 0) pcgb::fail(PCGB_EINVAL, "batch must be positive");
        cudaStream_t st = pcgb::as_stream(stream);
        const pcgb::NttPlan& pl = pcgb::ntt_plan(pcgb::ilog2i(N));
        uint64_t* scratch = nullptr;
        const size_t n = static_cast<size_t>(batch) * N;
        scratch = static_cast<uint64_t*>(pcgb::pool_alloc(n * sizeof(uint64_t), st));
        pcgb::poly_mul_device(pl, d_c, d_a, d_b, batch, scratch, st);
        PCGB_CK(cudaFreeAsync(scratch, st));
    });
}

int pcgb_poly_mul_device_multi(int count, uint64_t* const* d_c, const uint64_t* const* d_a,
                               const uint64_t* const* d_b, const int* N, void* stream) {
    return guarded([&] {
        if (count < 0 || (count > 0 && (!d_c || !d_a || !d_b || !N)))
            pcgb::fail(PCGB_EINVAL, "multi poly-mul: bad arguments");
        cudaStream_t st = pcgb::as_stream(stream);
        std::vector<int> logN(count);
        bool mixed = count > 0;
        for (int i = 0; i < count; ++i) {
            if (!pcgb::pow2(N[i]) || N[i] < 2 || N[i] > (1 << pcgb::kMaxLogN))
                pcgb::fail(PCGB_EINVAL, "N must be a power of two in [2, 2^24]");
            logN[i] = pcgb::ilog2i(N[i]);
            mixed = mixed && pcgb::poly_mul_mixed_ok(logN[i]);
        }
        if (mixed) {
            // Lengths 2^16 .. 2^20 in any mix: one launch per pass for the batch.
            pcgb::poly_mul_device_mixed(count, d_c, d_a, d_b, logN.data(), st);
            return;
        }
        for (int i = 0; i < count; ++i) {
            const pcgb::NttPlan& pl = pcgb::ntt_plan(logN[i]);
            uint64_t* scratch = static_cast<uint64_t*>(
                pcgb::pool_alloc(static_cast<size_t>(N[i]) * sizeof(uint64_t), st));
            pcgb::poly_mul_device(pl, d_c[i], d_a[i], d_b[i], 1, scratch, st);
            PCGB_CK(cudaFreeAsync(scratch, st));
        }
    });
}

// ---- consumers: triples, relation checks -------------------------------------
int pcgb_triples_device(int N, int party, const uint64_t* d_x1, const uint64_t* d_z1,
                        const uint64_t* d_x2, const uint64_t* d_z2, uint64_t* d_a, uint64_t* d_b,
                        uint64_t* d_c, void* stream) {
    return guarded([&] {
        pcgb::triples_device(N, party, d_x1, d_z1, d_x2, d_z2, d_a, d_b, d_c,
                             pcgb::as_stream(stream));
    });
}

int pcgb_verify_ole_device(int N, const uint64_t* d_x0, const uint64_t* d_z0,
                           const uint64_t* d_x1, const uint64_t* d_z1,
                           unsigned long long* d_mismatches, void* stream) {
    return guarded([&] {
        pcgb::verify_ole_device(N, d_x0, d_z0, d_x1, d_z1, d_mismatches, pcgb::as_stream(stream));
    });
}

int pcgb_verify_triples_device(int N, const uint64_t* d_a0, const uint64_t* d_b0,
                               const uint64_t* d_c0, const uint64_t* d_a1,
                               const uint64_t* d_b1, const uint64_t* d_c1,
                               unsigned long long* d_mismatches, void* stream) {
    return guarded([&] {
        pcgb::verify_triples_device(N, d_a0, d_b0, d_c0, d_a1, d_b1, d_c1, d_mismatches,
                                    pcgb::as_stream(stream));
    });
}

// ---- expansion --------------------------------------------------------------
int pcgb_expander_create(pcgb_expander** e, int N, int c, int t, int w, int prg,
                         const uint64_t* public_a, const uint8_t* master_key) {
    if (e) *e = nullptr;
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander handle");
        *e = pcgb::expander_create(N, c, t, w, prg, public_a, master_key);
    });
}

int pcgb_expander_create_shard(pcgb_expander** e, int N, int c, int t, int w, int prg,
                               const uint64_t* public_a, const uint8_t* master_key, int rank,
                               int world) {
    if (e) *e = nullptr;
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander handle");
        *e = pcgb::expander_create(N, c, t, w, prg, public_a, master_key, rank, world);
    });
}

int pcgb_expander_create_public_a0(pcgb_expander** e, int N, int c, int t, int w, int prg,
                                   const uint64_t* public_a, const uint8_t* master_key) {
    if (e) *e = nullptr;
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander handle");
        *e = pcgb::expander_create(N, c, t, w, prg, public_a, master_key, 0, 1, 1);
    });
}

int pcgb_expander_shard(const pcgb_expander* e, int* rank, int* world, int* pairs_local,
                        int* pairs_total) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_shard(e, rank, world, pairs_local, pairs_total);
    });
}

int pcgb_reduce_mod_p(uint64_t* d, const uint64_t* s, size_t count, void* stream) {
    return guarded([&] {
        if (count && (!d || !s)) pcgb::fail(PCGB_EINVAL, "reduce_mod_p: null pointer");
        if (count) pcgb::reduce_mod_p(d, s, count, pcgb::as_stream(stream));
    });
}

int pcgb_add_mod_p_device(uint64_t* d, const uint64_t* u, const uint64_t* v, size_t count,
                          void* stream) {
    return guarded([&] {
        if (count && (!d || !u || !v)) pcgb::fail(PCGB_EINVAL, "add_mod_p: null pointer");
        if (count) pcgb::add_mod_p_device(d, u, v, count, pcgb::as_stream(stream));
    });
}

int pcgb_expander_destroy(pcgb_expander* e) {
    return guarded([&] { pcgb::expander_destroy(e); });
}

int pcgb_expander_info(const pcgb_expander* e, int* K, int* levels, int* nk, size_t* scratch) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_info(e, K, levels, nk, scratch);
    });
}

int pcgb_expand_device(pcgb_expander* e, int party, const pcgb_blk* d_roots, const pcgb_blk* d_cws,
                       const uint64_t* d_cw_out, const uint64_t* d_pos, const uint64_t* d_val,
                       uint64_t* d_x, uint64_t* d_z, void* stream) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expand_device(e, party, reinterpret_cast<const Blk*>(d_roots),
                            reinterpret_cast<const Blk*>(d_cws), d_cw_out, d_pos, d_val, d_x, d_z,
                            pcgb::as_stream(stream));
    });
}

int pcgb_expand_batch_device(int count, pcgb_expander* const* e, const int* party,
                             const pcgb_blk* const* d_roots, const pcgb_blk* const* d_cws,
                             const uint64_t* const* d_cw_out, const uint64_t* const* d_pos,
                             const uint64_t* const* d_val, uint64_t* const* d_x,
                             uint64_t* const* d_z, void* stream) {
    return guarded([&] {
        if (count < 0) pcgb::fail(PCGB_EINVAL, "expand batch: negative count");
        if (count == 0) return;
        if (!e || !party || !d_roots || !d_cws || !d_cw_out || !d_pos || !d_val || !d_x || !d_z)
            pcgb::fail(PCGB_EINVAL, "expand batch: null array");
        for (int i = 0; i < count; ++i)
            if (!e[i]) pcgb::fail(PCGB_EINVAL, "expand batch: null expander");
        cudaStream_t st = pcgb::as_stream(stream);
        std::vector<size_t> off(count + 1, 0);
        for (int i = 0; i < count; ++i)
            off[i + 1] = off[i] + ((pcgb::workspace_bytes(e[i]) + 255) & ~size_t{255});
        char* base = static_cast<char*>(pcgb::pool_alloc(off[count], st));
        std::vector<pcgb::Workspace> ws(count);
        for (int i = 0; i < count; ++i) ws[i] = pcgb::workspace_carve(e[i], base + off[i]);
        try {
            pcgb::expand_batch_ws(count, e, ws.data(), party,
                                  reinterpret_cast<const Blk* const*>(d_roots),
                                  reinterpret_cast<const Blk* const*>(d_cws), d_cw_out, d_pos,
                                  d_val, d_x, d_z, st);
        } catch (...) {
            cudaFreeAsync(base, st);
            throw;
        }
        PCGB_CK(cudaFreeAsync(base, st));
    });
}

int pcgb_expand_host_async(pcgb_expander* e, int party, const pcgb_blk* roots,
                           const pcgb_blk* cws, const uint64_t* cw_out, const uint64_t* pos,
                           const uint64_t* val, uint64_t* x, uint64_t* z) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expand_host_async(e, party, reinterpret_cast<const Blk*>(roots),
                                reinterpret_cast<const Blk*>(cws), cw_out, pos, val, x, z);
    });
}

int pcgb_expander_wait(pcgb_expander* e) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_wait(e);
    });
}

int pcgb_expand_host(pcgb_expander* e, int party, const pcgb_blk* roots, const pcgb_blk* cws,
                     const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val, uint64_t* x,
                     uint64_t* z) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expand_host(e, party, reinterpret_cast<const Blk*>(roots),
                          reinterpret_cast<const Blk*>(cws), cw_out, pos, val, x, z);
    });
}

int pcgb_expand_g_device(pcgb_expander* e, int party, const pcgb_blk* d_roots,
                         const pcgb_blk* d_cws, const uint64_t* d_cw_out, uint64_t* d_g,
                         void* stream) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        if (party != 0 && party != 1) pcgb::fail(PCGB_EINVAL, "party must be 0 or 1");
        pcgb::expand_g_device(e, party, reinterpret_cast<const Blk*>(d_roots),
                              reinterpret_cast<const Blk*>(d_cws), d_cw_out, d_g,
                              pcgb::as_stream(stream));
    });
}

int pcgb_expander_set_profiling(pcgb_expander* e, int slots) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_set_profiling(e, slots);
    });
}

int pcgb_expand_from_g_device(pcgb_expander* e, const uint64_t* d_g, const uint64_t* d_pos,
                              const uint64_t* d_val, uint64_t* d_x, uint64_t* d_z, void* stream) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expand_from_g_device(e, d_g, d_pos, d_val, d_x, d_z, pcgb::as_stream(stream));
    });
}

int pcgb_expander_set_graph(pcgb_expander* e, int enable) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_set_graph(e, enable != 0);
    });
}

int pcgb_expander_autotune(pcgb_expander* e, int* tpb_out) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        const int tpb = pcgb::expander_autotune(e);
        if (tpb_out) *tpb_out = tpb;
    });
}

int pcgb_expander_set_leaf_shape(pcgb_expander* e, int tpb, int leaves_per_thread) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_set_leaf_shape(e, tpb, leaves_per_thread);
    });
}

int pcgb_expander_leaf_shape(const pcgb_expander* e, int* tpb, int* leaves_per_thread) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::expander_leaf_shape(e, tpb, leaves_per_thread);
    });
}

int pcgb_expander_stage_times(pcgb_expander* e, float* ms, int max_expansions) {
    int r = 0;
    const int rc = guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        r = pcgb::expander_stage_times(e, ms, max_expansions);
    });
    return rc ? rc : r;
}

int pcgb_noise(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val) {
    if (N < 2 || t < 1 || N % t || c < 1 || !pos || !val) {
        pcgb::g_last_error = "noise: bad shape";
        return PCGB_EINVAL;
    }
    pcgb::noise_host(N, c, t, seed, party, pos, val);
    return PCGB_OK;
}

int pcgb_public_a(int N, int c, uint64_t a_seed, uint64_t* a) {
    if (N < 1 || c < 1 || (c > 1 && !a)) {
        pcgb::g_last_error = "public_a: bad shape";
        return PCGB_EINVAL;
    }
    pcgb::public_a_host(N, c, a_seed, a);
    return PCGB_OK;
}

int pcgb_deal_keys_device(pcgb_expander* e, uint64_t seed, pcgb_blk* d_roots0, pcgb_blk* d_roots1,
                          pcgb_blk* d_cws, uint64_t* d_cw_out, void* stream) {
    return guarded([&] {
        if (!e) pcgb::fail(PCGB_EINVAL, "null expander");
        pcgb::deal_keys_device(e, seed, reinterpret_cast<Blk*>(d_roots0),
                               reinterpret_cast<Blk*>(d_roots1), reinterpret_cast<Blk*>(d_cws),
                               d_cw_out, pcgb::as_stream(stream));
    });
}

// ---- serving ------------------------------------------------------------------
int pcgb_server_create(pcgb_server** s, int n_streams, size_t mem_budget, int max_in_flight,
                       uint64_t a_seed) {
    if (s) *s = nullptr;
    return guarded([&] {
        if (!s) pcgb::fail(PCGB_EINVAL, "null server handle");
        *s = pcgb::server_create(n_streams, mem_budget, max_in_flight, a_seed);
    });
}

int pcgb_server_prepare(pcgb_server* s, int N, int c, int t) {
    return guarded([&] {
        if (!s) pcgb::fail(PCGB_EINVAL, "null server");
        pcgb::server_prepare(s, N, c, t);
    });
}

int pcgb_server_submit(pcgb_server* s, const pcgb_request* r, uint64_t* ticket) {
    return guarded([&] {
        if (!s || !r || !ticket) pcgb::fail(PCGB_EINVAL, "null argument");
        *ticket = pcgb::server_submit(s, *r);
    });
}

int pcgb_server_wait(pcgb_server* s, uint64_t ticket, pcgb_result* out, int timeout_ms) {
    int rc = PCGB_OK;
    const int g = guarded([&] {
        if (!s) pcgb::fail(PCGB_EINVAL, "null server");
        rc = pcgb::server_wait(s, ticket, out, timeout_ms);
        if (rc == PCGB_ETIMEOUT) pcgb::fail(PCGB_ETIMEOUT, "server_wait: timed out");
    });
    return g;
}

int pcgb_server_run_trace(pcgb_server* s, const pcgb_request* reqs, int n, pcgb_result* out,
                          double timeout_s) {
    return guarded([&] {
        if (!s || (n > 0 && !reqs)) pcgb::fail(PCGB_EINVAL, "null argument");
        pcgb::server_run_trace(s, reqs, n, out, timeout_s);
    });
}

int pcgb_server_stats(pcgb_server* s, int* pending, int* in_flight, size_t* bytes_in_flight,
                      int* plans) {
    return guarded([&] {
        if (!s) pcgb::fail(PCGB_EINVAL, "null server");
        pcgb::server_stats(s, pending, in_flight, bytes_in_flight, plans);
    });
}

int pcgb_server_destroy(pcgb_server* s, int timeout_ms) {
    return guarded([&] {
        if (s) pcgb::server_destroy(s, timeout_ms);
    });
}

int pcgb_digest_device(const uint64_t* d_v, size_t n, uint64_t* d_out, void* stream) {
    return guarded([&] {
        if (!d_v || !d_out) pcgb::fail(PCGB_EINVAL, "null argument");
        pcgb::digest_device(d_v, n, d_out, pcgb::as_stream(stream));
    });
}

}  // extern "C"
