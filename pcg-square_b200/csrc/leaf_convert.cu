// Output-layer drop-ins: pcg_cuda::dpf_out_sums and dpf_out_scatter_g
// (GPU_baseline/common/leaf_convert_cuda.h:43-52).
//
//   C[b][d] = low64(ChaCha8OutHash(leaf)) mod p, tau[b][d] = lsb(leaf)
//   sumC[b] = sum_d C (mod p), sumT[b] = sum_d tau (plain integer)
//   y = C + tau*CW[b]; party 1 negates; pos = (b/t + b%t)*D/2 + d;
//   g[pos mod N] += (pos < N ? y : -y)              (mod p)
//
// dpf_out_sums reduces per-CTA partials in a fixed order.  dpf_out_scatter_g
// is written as a gather: one thread per output word of g visits the (at
// most 2t) instances whose shifted leaf ranges cover it, so every word is
// produced once without atomics (the reference resolves overlaps with a
// CAS-loop modular atomic, leaf_convert_cuda.cu:68-77,207-234).
//
// The drop-ins hash every leaf in both passes, as the reference does
// (leaf_convert_cuda.h:47-49 judges that cheaper than keeping B*D values).
// On B200 the hash is the bound (341 integer ops per 16-byte leaf) and HBM
// is not, so the convert/scatter-conv pair keeps each leaf's converted word
// C | tau << 63 (C < p < 2^62) from the sums pass, and the scatter reads 8
// bytes per leaf instead of hashing 16 again.
//
// The two-party expansion's output-layer Beaver multiplication
// (pcg_ole_impl.h:222-290) also runs here, on device-resident sums:
//   <A> = (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>
//   open d = <A> - r, e = <B> - s;  <CW> = d*s + e*r + rs (+ d*e, party 0).
#include "pcgb_internal.h"

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "chacha8.cuh"
#include "field.cuh"

namespace pcgb {
namespace {

constexpr int kTPB = 256;

__device__ __forceinline__ uint64_t leaf_C(const ulonglong2& v) {
    return reduce_p(out_hash_lo64(v.x, v.y));
}

constexpr uint64_t kTauBit = uint64_t{1} << 63;

// Sums are kept as 128-bit integers and reduced mod p once per output:
// hi*2^64 + lo with hi small and signed, and 2^64 = 3*2^27 - 4 (mod p).
constexpr uint64_t kTwo64ModP = 402653180ULL;
__device__ __forceinline__ uint64_t mod_p_128(unsigned __int128 a) {
    const int64_t hi = static_cast<int64_t>(static_cast<uint64_t>(a >> 64));
    const uint64_t mag = hi < 0 ? static_cast<uint64_t>(-hi) : static_cast<uint64_t>(hi);
    uint64_t t = reduce_p(mag * kTwo64ModP);   // |hi| < 2^35: no wrap
    if (hi < 0) t = neg_p(t);
    return add_p(reduce_p(static_cast<uint64_t>(a)), t);
}

// grid = (parts, B): partials[b*parts + part] (C lane), [B*parts + ...] (T lane).
// KEEP: also write conv[b*D + d] = C | tau << 63.
template <bool KEEP>
__global__ void __launch_bounds__(kTPB) out_sum_kernel(const ulonglong2* __restrict__ leaves,
                                                       size_t D, uint64_t* __restrict__ partials,
                                                       uint64_t* __restrict__ conv) {
    __shared__ uint64_t sc[kTPB / 32], stt[kTPB / 32];
    const int b = blockIdx.y, parts = gridDim.x;
    const ulonglong2* L = leaves + static_cast<size_t>(b) * D;
    uint64_t c = 0, t = 0;
    unsigned __int128 c128 = 0;   // without KEEP: raw hash words, reduced at the end
    for (size_t d = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; d < D;
         d += static_cast<size_t>(parts) * blockDim.x) {
        const ulonglong2 v = __ldg(L + d);
        t += v.x & 1;
        if (KEEP) {
            const uint64_t C = leaf_C(v);
            c = add_p(c, C);
            conv[static_cast<size_t>(b) * D + d] = C | (v.x << 63);
        } else {
            c128 += out_hash_lo64(v.x, v.y);
        }
    }
    if (!KEEP) c = mod_p_128(c128);
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        c = add_p(c, __shfl_xor_sync(0xffffffffu, c, off));
        t += __shfl_xor_sync(0xffffffffu, t, off);
    }
    if ((threadIdx.x & 31) == 0) { sc[threadIdx.x >> 5] = c; stt[threadIdx.x >> 5] = t; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t cc = 0, tt = 0;
        for (int w = 0; w < kTPB / 32; ++w) { cc = add_p(cc, sc[w]); tt += stt[w]; }
        const size_t slot = static_cast<size_t>(b) * parts + blockIdx.x;
        partials[slot] = cc;
        partials[static_cast<size_t>(gridDim.y) * parts + slot] = tt;
    }
}

// One thread per instance folds its partials in order.
__global__ void out_fold_kernel(const uint64_t* __restrict__ partials, int parts, int B,
                                uint64_t* __restrict__ sums) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t c = 0, t = 0;
    for (int i = 0; i < parts; ++i) {
        c = add_p(c, partials[static_cast<size_t>(b) * parts + i]);
        t += partials[static_cast<size_t>(B) * parts + static_cast<size_t>(b) * parts + i];
    }
    sums[b] = c;
    sums[B + b] = t;
}

// y = C + tau*CW of one leaf up to a multiple of p (below 2^65), from the
// leaf itself (the raw hash word stands for C) or from its converted word.
__device__ __forceinline__ unsigned __int128 leaf_y(const ulonglong2* leaves, size_t i,
                                                    uint64_t cw) {
    const ulonglong2 v = __ldg(leaves + i);
    return static_cast<unsigned __int128>(out_hash_lo64(v.x, v.y)) + ((v.x & 1) ? cw : 0);
}
__device__ __forceinline__ unsigned __int128 leaf_y(const uint64_t* conv, size_t i, uint64_t cw) {
    const uint64_t w = __ldg(conv + i);
    return static_cast<unsigned __int128>(w & ~kTauBit) + ((w & kTauBit) ? cw : 0);
}

// Gather scatter: thread per output word p < N.
template <class In>
__global__ void __launch_bounds__(kTPB, 4) out_gather_kernel(const In* __restrict__ leaves,
                                                          int B, size_t D, int t, int party,
                                                          const uint64_t* __restrict__ cws,
                                                          uint64_t* __restrict__ g, size_t N) {
    const size_t p = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const size_t bin = D >> 1;
    const int kk_max = (B - 1) / t;
    const long s_max = static_cast<long>(kk_max) + t - 1;
    unsigned __int128 acc = 0;   // two's complement; reduced mod p once, below
    for (int f = 0; f < 2; ++f) {
        const size_t P = p + (f ? N : 0);   // pre-fold position
        const long s_hi = static_cast<long>(P / bin);
        for (long s = s_hi; s >= s_hi - 1; --s) {
            if (s < 0 || s > s_max) continue;
            const size_t d = P - static_cast<size_t>(s) * bin;
            if (d >= D) continue;
            const int kk0 = static_cast<int>(s - (t - 1) > 0 ? s - (t - 1) : 0);
            const int kk1 = static_cast<int>(s < kk_max ? s : kk_max);
            for (int kk = kk0; kk <= kk1; ++kk) {
                const int b = kk * t + static_cast<int>(s - kk);
                if (b >= B) continue;
                const unsigned __int128 y =
                    leaf_y(leaves, static_cast<size_t>(b) * D + d, __ldg(cws + b));
                if ((party != 0) != (f != 0)) acc -= y;
                else acc += y;
            }
        }
    }
    g[p] = mod_p_128(acc);
}

__global__ void beaver_open_kernel(int B, int party, const uint64_t* __restrict__ sumC,
                                   const uint64_t* __restrict__ sumT,
                                   const uint64_t* __restrict__ beta,
                                   const uint64_t* __restrict__ r, const uint64_t* __restrict__ s,
                                   uint64_t* __restrict__ de) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t A = reduce_p(sumT[b]), Bs = reduce_p(sumC[b]);
    if (party) A = neg_p(A);
    else Bs = neg_p(Bs);
    Bs = add_p(Bs, reduce_p(beta[b]));
    de[b] = sub_p(A, reduce_p(r[b]));
    de[B + b] = sub_p(Bs, reduce_p(s[b]));
}

// a*b mod p for a, b < p: two Montgomery products, the second by R^2.
__device__ __forceinline__ uint64_t mul_p(uint64_t a, uint64_t b, uint64_t r2) {
    return mont_mul(mont_mul(a, b), r2);
}

__global__ void beaver_close_kernel(int B, int party, const uint64_t* __restrict__ de_my,
                                    const uint64_t* __restrict__ de_peer,
                                    const uint64_t* __restrict__ r, const uint64_t* __restrict__ s,
                                    const uint64_t* __restrict__ rs, uint64_t r2,
                                    uint64_t* __restrict__ cw) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const uint64_t d = add_p(reduce_p(de_my[b]), reduce_p(de_peer[b]));
    const uint64_t e = add_p(reduce_p(de_my[B + b]), reduce_p(de_peer[B + b]));
    uint64_t v = add_p(mul_p(d, reduce_p(s[b]), r2), mul_p(e, reduce_p(r[b]), r2));
    v = add_p(v, reduce_p(rs[b]));
    if (party == 0) v = add_p(v, mul_p(d, e, r2));
    cw[b] = v;
}

struct ConvPool {
    uint64_t* partials = nullptr;
    uint64_t* sums = nullptr;
    uint64_t* cws = nullptr;
    uint64_t* g = nullptr;
    size_t cap_part = 0, cap_b = 0, cap_cw = 0, cap_g = 0;
    std::mutex mu;
};

ConvPool& conv_pool() {
    static std::mutex mu;
    static ConvPool* pools[64] = {nullptr};
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) pools[dev] = new ConvPool();
    return *pools[dev];
}

void grow(uint64_t*& p, size_t& cap, size_t need) {
    if (need <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, need * sizeof(uint64_t)) != cudaSuccess) {
        cudaGetLastError();
        fail(PCGB_ENOMEM, "leaf convert: device allocation failed");
    }
    cap = need;
}

void check_common(const void* d_leaves, int B, size_t D, uint64_t prime) {
    if (prime != kP) fail(PCGB_EINVAL, "dpf_out: only the project prime is supported");
    if (!d_leaves) fail(PCGB_EINVAL, "dpf_out: null leaves");
    if (D < 2 || (D & (D - 1))) fail(PCGB_EINVAL, "dpf_out: D must be a power of two >= 2");
    (void)B;
}

}  // namespace

int out_sums_parts(size_t D) {
    size_t parts = (D + kTPB * 8 - 1) / (kTPB * 8);
    if (parts > 1024) parts = 1024;
    return static_cast<int>(parts < 1 ? 1 : parts);
}

void out_sums_launch(const Blk* d_leaves, int B, size_t D, uint64_t* partials, uint64_t* sums,
                     cudaStream_t st) {
    const int parts = out_sums_parts(D);
    out_sum_kernel<false><<<dim3(parts, B), kTPB, 0, st>>>(
        reinterpret_cast<const ulonglong2*>(d_leaves), D, partials, nullptr);
    PCGB_POST_LAUNCH();
    out_fold_kernel<<<(B + 127) / 128, 128, 0, st>>>(partials, parts, B, sums);
    PCGB_POST_LAUNCH();
}

void out_gather_launch(const Blk* d_leaves, int B, size_t D, int t, int party,
                       const uint64_t* d_cws, uint64_t* d_g, size_t N, cudaStream_t st) {
    out_gather_kernel<ulonglong2><<<static_cast<unsigned>((N + kTPB - 1) / kTPB), kTPB, 0, st>>>(
        reinterpret_cast<const ulonglong2*>(d_leaves), B, D, t, party, d_cws, d_g, N);
    PCGB_POST_LAUNCH();
}

void dpf_out_sums_host(const Blk* d_leaves, int B, size_t D, uint64_t prime, uint64_t* sumC,
                       uint64_t* sumT) {
    if (B <= 0) return;
    check_common(d_leaves, B, D, prime);
    ConvPool& pl = conv_pool();
    std::lock_guard<std::mutex> lk(pl.mu);
    cudaStream_t st = default_stream();
    grow(pl.partials, pl.cap_part, 2 * static_cast<size_t>(B) * out_sums_parts(D));
    grow(pl.sums, pl.cap_b, 2 * static_cast<size_t>(B));
    out_sums_launch(d_leaves, B, D, pl.partials, pl.sums, st);
    std::vector<uint64_t> both(2 * static_cast<size_t>(B));
    PCGB_CK(cudaMemcpyAsync(both.data(), pl.sums, both.size() * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
    for (int b = 0; b < B; ++b) {
        sumC[b] = both[b];
        sumT[b] = both[B + b];
    }
}

// ---- allocation-free sums ---------------------------------------------------
// Per-CTA partial sums of pcgb_dpf_out_sums_noalloc.  A file-scope device
// array: every device that loads the library holds these 1 MiB until the
// process exits, and all calls on a device share it.
constexpr size_t kNoAllocScratchWords = size_t{1} << 17;
static __device__ __align__(256) uint64_t g_noalloc_partials[kNoAllocScratchWords];

namespace {

// Splits the folded sums into the caller's two output arrays.
__global__ void out_fold_split_kernel(const uint64_t* __restrict__ partials, int parts, int B,
                                      uint64_t* __restrict__ sumC, uint64_t* __restrict__ sumT) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t c = 0, t = 0;
    for (int i = 0; i < parts; ++i) {
        c = add_p(c, partials[static_cast<size_t>(b) * parts + i]);
        t += partials[static_cast<size_t>(B) * parts + static_cast<size_t>(b) * parts + i];
    }
    sumC[b] = c;
    sumT[b] = t;
}

// Device address of the scratch array on the current device.  Host code
// only sees a host-side stand-in for g_noalloc_partials, so the address is
// looked up once per device with that device current.
uint64_t* noalloc_partials() {
    static std::mutex mu;
    static uint64_t* addr[64] = {nullptr};
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(PCGB_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        PCGB_CK(cudaGetSymbolAddress(&p, g_noalloc_partials));
        addr[dev] = static_cast<uint64_t*>(p);
    }
    return addr[dev];
}

}  // namespace

void dpf_out_sums_noalloc(const Blk* d_leaves, int B, size_t D, uint64_t prime, uint64_t* d_sumC,
                          uint64_t* d_sumT, cudaStream_t st) {
    if (B <= 0) return;
    check_common(d_leaves, B, D, prime);
    if (!d_sumC || !d_sumT) fail(PCGB_EINVAL, "dpf_out_sums_noalloc: null output array");
    const size_t max_b = kNoAllocScratchWords / 2;
    if (B > 65535 || static_cast<size_t>(B) > max_b)
        fail(PCGB_EINVAL, "dpf_out_sums_noalloc: B = " + std::to_string(B) +
                              " exceeds the limit of 65535 instances of the static scratch");
    // Fewer partials per instance when B is large, so they fit the array.
    const size_t fit = kNoAllocScratchWords / (2 * static_cast<size_t>(B));
    const int parts = static_cast<int>(std::min<size_t>(out_sums_parts(D), fit));
    uint64_t* partials = noalloc_partials();
    out_sum_kernel<false><<<dim3(parts, B), kTPB, 0, st>>>(
        reinterpret_cast<const ulonglong2*>(d_leaves), D, partials, nullptr);
    PCGB_POST_LAUNCH();
    out_fold_split_kernel<<<(B + 127) / 128, 128, 0, st>>>(partials, parts, B, d_sumC, d_sumT);
    PCGB_POST_LAUNCH();
}

void dpf_out_scatter_host(const Blk* d_leaves, int B, size_t D, int t, int party, uint64_t prime,
                          const uint64_t* CW, uint64_t* g_out, int N) {
    if (B <= 0) return;
    check_common(d_leaves, B, D, prime);
    if (t <= 0 || N <= 0) fail(PCGB_EINVAL, "dpf_out_scatter_g: t and N must be positive");
    const size_t bin = D >> 1;
    const size_t s_max = static_cast<size_t>((B - 1) / t) + t - 1;
    // Every pre-fold position must stay below 2N (the reference's fold
    // handles one wrap only).
    if ((s_max + 2) * bin > 2 * static_cast<size_t>(N))
        fail(PCGB_EINVAL, "dpf_out_scatter_g: N smaller than the instances' span (needs N >= t*D/2)");
    ConvPool& pl = conv_pool();
    std::lock_guard<std::mutex> lk(pl.mu);
    cudaStream_t st = default_stream();
    grow(pl.cws, pl.cap_cw, static_cast<size_t>(B));
    grow(pl.g, pl.cap_g, static_cast<size_t>(N));
    std::vector<uint64_t> cw(CW, CW + B);
    for (auto& v : cw) v %= kP;
    PCGB_CK(cudaMemcpyAsync(pl.cws, cw.data(), B * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    out_gather_launch(d_leaves, B, D, t, party, pl.cws, pl.g, static_cast<size_t>(N), st);
    PCGB_CK(cudaMemcpyAsync(g_out, pl.g, static_cast<size_t>(N) * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

// Device-pointer form: CWs already on the device (values in [0, p)), g
// written to the device (every position once, so it needs no clearing).
void dpf_out_scatter_device(const Blk* d_leaves, int B, size_t D, int t, int party,
                            const uint64_t* d_cw, uint64_t* d_g, int N, cudaStream_t st) {
    if (B <= 0) return;
    check_common(d_leaves, B, D, kP);
    if (!d_cw || !d_g) fail(PCGB_EINVAL, "dpf_out_scatter_g_device: null pointer");
    if (t <= 0 || N <= 0) fail(PCGB_EINVAL, "dpf_out_scatter_g_device: t and N must be positive");
    const size_t bin = D >> 1;
    const size_t s_max = static_cast<size_t>((B - 1) / t) + t - 1;
    if ((s_max + 2) * bin > 2 * static_cast<size_t>(N))
        fail(PCGB_EINVAL, "dpf_out_scatter_g_device: N smaller than the instances' span");
    out_gather_launch(d_leaves, B, D, t, party, d_cw, d_g, static_cast<size_t>(N), st);
}

void dpf_out_convert_device(const Blk* d_leaves, int B, size_t D, uint64_t* d_conv,
                            uint64_t* d_sumC, uint64_t* d_sumT, cudaStream_t st) {
    if (B <= 0) return;
    check_common(d_leaves, B, D, kP);
    if (!d_conv || !d_sumC || !d_sumT) fail(PCGB_EINVAL, "dpf_out_convert_device: null pointer");
    const int parts = out_sums_parts(D);
    uint64_t* partials =
        static_cast<uint64_t*>(pool_alloc(2 * static_cast<size_t>(B) * parts * sizeof(uint64_t), st));
    out_sum_kernel<true><<<dim3(parts, B), kTPB, 0, st>>>(
        reinterpret_cast<const ulonglong2*>(d_leaves), D, partials, d_conv);
    PCGB_POST_LAUNCH();
    out_fold_split_kernel<<<(B + 127) / 128, 128, 0, st>>>(partials, parts, B, d_sumC, d_sumT);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(partials, st));
}

void dpf_out_scatter_conv_device(const uint64_t* d_conv, int B, size_t D, int t, int party,
                                 const uint64_t* d_cw, uint64_t* d_g, int N, cudaStream_t st) {
    if (B <= 0) return;
    check_common(d_conv, B, D, kP);
    if (!d_cw || !d_g) fail(PCGB_EINVAL, "dpf_out_scatter_g_conv_device: null pointer");
    if (t <= 0 || N <= 0) fail(PCGB_EINVAL, "dpf_out_scatter_g_conv_device: t and N must be positive");
    const size_t bin = D >> 1;
    const size_t s_max = static_cast<size_t>((B - 1) / t) + t - 1;
    if ((s_max + 2) * bin > 2 * static_cast<size_t>(N))
        fail(PCGB_EINVAL, "dpf_out_scatter_g_conv_device: N smaller than the instances' span");
    out_gather_kernel<uint64_t><<<static_cast<unsigned>((N + kTPB - 1) / kTPB), kTPB, 0, st>>>(
        d_conv, B, D, t, party, d_cw, d_g, static_cast<size_t>(N));
    PCGB_POST_LAUNCH();
}

void out_beaver_open_device(int B, int party, const uint64_t* d_sumC, const uint64_t* d_sumT,
                            const uint64_t* d_beta, const uint64_t* d_r, const uint64_t* d_s,
                            uint64_t* d_de, cudaStream_t st) {
    if (B <= 0) return;
    if (party != 0 && party != 1) fail(PCGB_EINVAL, "out_beaver_open: party must be 0 or 1");
    if (!d_sumC || !d_sumT || !d_beta || !d_r || !d_s || !d_de)
        fail(PCGB_EINVAL, "out_beaver_open: null pointer");
    beaver_open_kernel<<<(B + 255) / 256, 256, 0, st>>>(B, party, d_sumC, d_sumT, d_beta, d_r, d_s,
                                                        d_de);
    PCGB_POST_LAUNCH();
}

void out_beaver_close_device(int B, int party, const uint64_t* d_de_my, const uint64_t* d_de_peer,
                             const uint64_t* d_r, const uint64_t* d_s, const uint64_t* d_rs,
                             uint64_t* d_cw, cudaStream_t st) {
    if (B <= 0) return;
    if (party != 0 && party != 1) fail(PCGB_EINVAL, "out_beaver_close: party must be 0 or 1");
    if (!d_de_my || !d_de_peer || !d_r || !d_s || !d_rs || !d_cw)
        fail(PCGB_EINVAL, "out_beaver_close: null pointer");
    beaver_close_kernel<<<(B + 255) / 256, 256, 0, st>>>(B, party, d_de_my, d_de_peer, d_r, d_s,
                                                         d_rs, r2_mod_p(), d_cw);
    PCGB_POST_LAUNCH();
}

}  // namespace pcgb
