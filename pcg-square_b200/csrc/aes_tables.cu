// AES-128 host side: S-box and T-tables generated from the FIPS-197
// definitions, the key schedule, the tree-PRG sub-key derivation of
// half_tree_dpf/tree_prg.h:45-57, and the ECB bring-up entry point that
// mirrors pcg_cuda::aes128_ecb_encrypt_gpu (GPU_baseline/common/aes_gpu.h:18).
#include "pcgb_internal.h"

#include <cstring>
#include <mutex>
#include <vector>

#include "aes128.cuh"

namespace pcgb {
namespace {

struct HostTables {
    uint8_t sbox[256];
    uint32_t te[1024];
    HostTables() {
        auto gmul = [](uint8_t a, uint8_t b) {
            uint8_t r = 0;
            while (b) {
                if (b & 1) r ^= a;
                a = static_cast<uint8_t>((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
                b >>= 1;
            }
            return r;
        };
        // Inverse in GF(2^8) by exponentiation: x^254.
        auto ginv = [&](uint8_t x) {
            uint8_t r = 1, b = x;
            for (int e = 254; e; e >>= 1) {
                if (e & 1) r = gmul(r, b);
                b = gmul(b, b);
            }
            return x ? r : static_cast<uint8_t>(0);
        };
        for (int x = 0; x < 256; ++x) {
            const uint8_t v = ginv(static_cast<uint8_t>(x));
            uint8_t s = v, r = v;
            for (int k = 0; k < 4; ++k) {
                r = static_cast<uint8_t>((r << 1) | (r >> 7));
                s ^= r;
            }
            sbox[x] = s ^ 0x63;
        }
        for (int x = 0; x < 256; ++x) {
            const uint8_t s = sbox[x], s2 = gmul(s, 2), s3 = gmul(s, 3);
            const uint32_t t0 = s2 | (static_cast<uint32_t>(s) << 8) |
                                (static_cast<uint32_t>(s) << 16) | (static_cast<uint32_t>(s3) << 24);
            for (int r = 0; r < 4; ++r)
                te[256 * r + x] = r ? ((t0 << (8 * r)) | (t0 >> (32 - 8 * r))) : t0;
        }
    }
};

const HostTables& host_tables() {
    static HostTables t;
    return t;
}

uint8_t xtime(uint8_t v) { return static_cast<uint8_t>((v << 1) ^ ((v & 0x80) ? 0x1b : 0)); }

// One thread per block, each block under its own 44-word key schedule.
__global__ void aes_ecb_kernel(const uint32_t* __restrict__ te_g, const uint32_t* __restrict__ rk,
                               const uint4* __restrict__ in, uint4* __restrict__ out, int count) {
    __shared__ uint32_t te[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) te[i] = te_g[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint4 v = in[i];
    aes128_encrypt_words(te, rk + 44 * static_cast<size_t>(i), v.x, v.y, v.z, v.w);
    out[i] = v;
}

}  // namespace

void aes_expand_key_host(const uint8_t key[16], uint8_t rk[176]) {
    const uint8_t* S = host_tables().sbox;
    std::memcpy(rk, key, 16);
    uint8_t rcon = 1;
    for (int i = 4; i < 44; ++i) {
        uint8_t w[4];
        std::memcpy(w, rk + 4 * (i - 1), 4);
        if ((i & 3) == 0) {  // RotWord, SubWord, Rcon
            const uint8_t w0 = w[0];
            w[0] = static_cast<uint8_t>(S[w[1]] ^ rcon);
            w[1] = S[w[2]];
            w[2] = S[w[3]];
            w[3] = S[w0];
            rcon = xtime(rcon);
        }
        for (int k = 0; k < 4; ++k) rk[4 * i + k] = rk[4 * (i - 4) + k] ^ w[k];
    }
}

void aes_encrypt_host(const uint8_t rk[176], const uint8_t in[16], uint8_t out[16]) {
    const uint32_t* te = host_tables().te;
    uint32_t w[4], k[44];
    std::memcpy(w, in, 16);
    std::memcpy(k, rk, 176);
    uint32_t s[4] = {w[0] ^ k[0], w[1] ^ k[1], w[2] ^ k[2], w[3] ^ k[3]};
    for (int r = 1; r < 10; ++r) {
        uint32_t t[4];
        for (int c = 0; c < 4; ++c)
            t[c] = te[s[c] & 0xff] ^ te[256 + ((s[(c + 1) & 3] >> 8) & 0xff)] ^
                   te[512 + ((s[(c + 2) & 3] >> 16) & 0xff)] ^ te[768 + (s[(c + 3) & 3] >> 24)] ^
                   k[4 * r + c];
        std::memcpy(s, t, 16);
    }
    const uint8_t* S = host_tables().sbox;
    uint32_t o[4];
    for (int c = 0; c < 4; ++c)
        o[c] = (S[s[c] & 0xff] | (S[(s[(c + 1) & 3] >> 8) & 0xff] << 8) |
                (S[(s[(c + 2) & 3] >> 16) & 0xff] << 16) |
                (static_cast<uint32_t>(S[s[(c + 3) & 3] >> 24]) << 24)) ^
               k[40 + c];
    std::memcpy(out, o, 16);
}

void aes_tree_round_keys_host(const uint8_t master[16], int nk, uint8_t* rks) {
    uint8_t mrk[176];
    aes_expand_key_host(master, mrk);
    for (int k = 0; k < nk; ++k) {
        uint8_t tweak[16] = {0}, c[16];
        const uint64_t kk = static_cast<uint64_t>(k);
        std::memcpy(tweak, &kk, 8);  // makeBlock(0, k): low 8 bytes = k
        aes_encrypt_host(mrk, tweak, c);
        for (int i = 0; i < 16; ++i) c[i] ^= tweak[i];
        aes_expand_key_host(c, rks + 176 * k);
    }
}

const uint32_t* aes_te_table_device() {
    static std::mutex mu;
    static uint32_t* per_dev[64] = {nullptr};
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (!per_dev[dev]) {
        uint32_t* d = nullptr;
        PCGB_CK(cudaMalloc(&d, sizeof(uint32_t) * 1024));
        upload_blocking(d, host_tables().te, sizeof(uint32_t) * 1024);
        per_dev[dev] = d;
    }
    return per_dev[dev];
}

uint32_t* aes_upload_round_keys(const uint8_t* rks_bytes, int nk, cudaStream_t st) {
    uint32_t* d = nullptr;
    PCGB_CK(cudaMalloc(&d, static_cast<size_t>(nk) * 176));
    PCGB_CK(cudaMemcpyAsync(d, rks_bytes, static_cast<size_t>(nk) * 176, cudaMemcpyHostToDevice,
                            st));
    return d;
}

void aes_ecb_encrypt_device(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count) {
    if (count <= 0) return;
    std::vector<uint8_t> rks(static_cast<size_t>(count) * 176);
    for (int i = 0; i < count; ++i) aes_expand_key_host(keys + 16 * i, rks.data() + 176 * i);
    cudaStream_t st = default_stream();
    uint8_t *d_rk = nullptr, *d_in = nullptr, *d_out = nullptr;
    const size_t bytes = static_cast<size_t>(count) * 16;
    d_rk = static_cast<uint8_t*>(pool_alloc(rks.size(), st));
    d_in = static_cast<uint8_t*>(pool_alloc(bytes, st));
    d_out = static_cast<uint8_t*>(pool_alloc(bytes, st));
    PCGB_CK(cudaMemcpyAsync(d_rk, rks.data(), rks.size(), cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_in, in, bytes, cudaMemcpyHostToDevice, st));
    aes_ecb_kernel<<<(count + 127) / 128, 128, 0, st>>>(
        aes_te_table_device(), reinterpret_cast<const uint32_t*>(d_rk),
        reinterpret_cast<const uint4*>(d_in), reinterpret_cast<uint4*>(d_out), count);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaFreeAsync(d_rk, st));
    PCGB_CK(cudaFreeAsync(d_in, st));
    PCGB_CK(cudaFreeAsync(d_out, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

}  // namespace pcgb
