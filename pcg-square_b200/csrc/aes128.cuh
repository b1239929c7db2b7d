// Device AES-128 encryption with four 256-word T-tables staged in shared
// memory (FIPS-197 rounds: SubBytes+ShiftRows+MixColumns folded into table
// lookups, AddRoundKey as word XORs).  The 16-byte state is four
// little-endian column words, so a DPF node {lo, hi} maps to words
// (lo, lo>>32, hi, hi>>32): the byte order the reference feeds its AES
// (GPU_baseline/common/aes_gpu.cuh:128-141).
//
// Te_r[x] holds column (2S, S, S, 3S)(x) rotated up by r bytes; the final
// round extracts S(x) as byte 1 of Te_0[x].
#ifndef PCGB_AES128_CUH_
#define PCGB_AES128_CUH_

#include <cstdint>

namespace pcgb {

// te: 1024 words in shared memory (Te0 | Te1 | Te2 | Te3); rk: 44 words.
__device__ __forceinline__ void aes128_encrypt_words(const uint32_t* __restrict__ te,
                                                     const uint32_t* __restrict__ rk,
                                                     uint32_t& w0, uint32_t& w1, uint32_t& w2,
                                                     uint32_t& w3) {
    uint32_t s0 = w0 ^ rk[0], s1 = w1 ^ rk[1], s2 = w2 ^ rk[2], s3 = w3 ^ rk[3];
    const uint32_t* te0 = te;
    const uint32_t* te1 = te + 256;
    const uint32_t* te2 = te + 512;
    const uint32_t* te3 = te + 768;
#pragma unroll
    for (int r = 1; r < 10; ++r) {
        const uint32_t t0 = te0[s0 & 0xff] ^ te1[(s1 >> 8) & 0xff] ^ te2[(s2 >> 16) & 0xff] ^
                            te3[s3 >> 24] ^ rk[4 * r + 0];
        const uint32_t t1 = te0[s1 & 0xff] ^ te1[(s2 >> 8) & 0xff] ^ te2[(s3 >> 16) & 0xff] ^
                            te3[s0 >> 24] ^ rk[4 * r + 1];
        const uint32_t t2 = te0[s2 & 0xff] ^ te1[(s3 >> 8) & 0xff] ^ te2[(s0 >> 16) & 0xff] ^
                            te3[s1 >> 24] ^ rk[4 * r + 2];
        const uint32_t t3 = te0[s3 & 0xff] ^ te1[(s0 >> 8) & 0xff] ^ te2[(s1 >> 16) & 0xff] ^
                            te3[s2 >> 24] ^ rk[4 * r + 3];
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
    // Final round: S-box bytes (byte 1 of Te0 entries), ShiftRows, AddRoundKey.
#define PCGB_SB(x) ((te0[(x)] >> 8) & 0xffu)
    w0 = (PCGB_SB(s0 & 0xff) | (PCGB_SB((s1 >> 8) & 0xff) << 8) |
          (PCGB_SB((s2 >> 16) & 0xff) << 16) | (PCGB_SB(s3 >> 24) << 24)) ^ rk[40];
    w1 = (PCGB_SB(s1 & 0xff) | (PCGB_SB((s2 >> 8) & 0xff) << 8) |
          (PCGB_SB((s3 >> 16) & 0xff) << 16) | (PCGB_SB(s0 >> 24) << 24)) ^ rk[41];
    w2 = (PCGB_SB(s2 & 0xff) | (PCGB_SB((s3 >> 8) & 0xff) << 8) |
          (PCGB_SB((s0 >> 16) & 0xff) << 16) | (PCGB_SB(s1 >> 24) << 24)) ^ rk[42];
    w3 = (PCGB_SB(s3 & 0xff) | (PCGB_SB((s0 >> 8) & 0xff) << 8) |
          (PCGB_SB((s1 >> 16) & 0xff) << 16) | (PCGB_SB(s2 >> 24) << 24)) ^ rk[43];
#undef PCGB_SB
}

// Bank-conflict-free form.  The state bytes index the tables at random, so
// the 32 lanes of a warp reading one 256-word table collide in several banks
// per lookup.  Here a single table Te0 is stored 32 times interleaved,
// te_rep[x * 32 + c] = Te0[x], and lane L reads copy L: every lookup of a
// warp hits 32 different banks.  Te1..Te3 are Te0 rotated left by 8, 16 and
// 24 bits, applied with byte permutes.
constexpr int kAesRepWords = 256 * 32;

__device__ __forceinline__ uint32_t rotl8_u32(uint32_t x) { return __byte_perm(x, 0, 0x2103); }
__device__ __forceinline__ uint32_t rotl16_u32(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t rotl24_u32(uint32_t x) { return __byte_perm(x, 0, 0x0321); }

// Fills te_rep (kAesRepWords words of shared memory) from Te0 (256 words in
// global memory); all threads of the CTA take part, no barrier inside.
__device__ __forceinline__ void aes_fill_rep(uint32_t* te_rep, const uint32_t* __restrict__ te0) {
    for (int i = threadIdx.x; i < kAesRepWords; i += blockDim.x) te_rep[i] = __ldg(te0 + (i >> 5));
}

__device__ __forceinline__ void aes128_encrypt_words_rep(const uint32_t* __restrict__ te_rep,
                                                         const uint32_t* __restrict__ rk,
                                                         uint32_t& w0, uint32_t& w1, uint32_t& w2,
                                                         uint32_t& w3) {
    const uint32_t* T = te_rep + (threadIdx.x & 31);
#define PCGB_TE(x) T[static_cast<uint32_t>(x) << 5]
    uint32_t s0 = w0 ^ rk[0], s1 = w1 ^ rk[1], s2 = w2 ^ rk[2], s3 = w3 ^ rk[3];
#pragma unroll
    for (int r = 1; r < 10; ++r) {
        const uint32_t t0 = PCGB_TE(s0 & 0xff) ^ rotl8_u32(PCGB_TE((s1 >> 8) & 0xff)) ^
                            rotl16_u32(PCGB_TE((s2 >> 16) & 0xff)) ^ rotl24_u32(PCGB_TE(s3 >> 24)) ^
                            rk[4 * r + 0];
        const uint32_t t1 = PCGB_TE(s1 & 0xff) ^ rotl8_u32(PCGB_TE((s2 >> 8) & 0xff)) ^
                            rotl16_u32(PCGB_TE((s3 >> 16) & 0xff)) ^ rotl24_u32(PCGB_TE(s0 >> 24)) ^
                            rk[4 * r + 1];
        const uint32_t t2 = PCGB_TE(s2 & 0xff) ^ rotl8_u32(PCGB_TE((s3 >> 8) & 0xff)) ^
                            rotl16_u32(PCGB_TE((s0 >> 16) & 0xff)) ^ rotl24_u32(PCGB_TE(s1 >> 24)) ^
                            rk[4 * r + 2];
        const uint32_t t3 = PCGB_TE(s3 & 0xff) ^ rotl8_u32(PCGB_TE((s0 >> 8) & 0xff)) ^
                            rotl16_u32(PCGB_TE((s1 >> 16) & 0xff)) ^ rotl24_u32(PCGB_TE(s2 >> 24)) ^
                            rk[4 * r + 3];
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
#define PCGB_SB(x) ((PCGB_TE(x) >> 8) & 0xffu)
    w0 = (PCGB_SB(s0 & 0xff) | (PCGB_SB((s1 >> 8) & 0xff) << 8) |
          (PCGB_SB((s2 >> 16) & 0xff) << 16) | (PCGB_SB(s3 >> 24) << 24)) ^ rk[40];
    w1 = (PCGB_SB(s1 & 0xff) | (PCGB_SB((s2 >> 8) & 0xff) << 8) |
          (PCGB_SB((s3 >> 16) & 0xff) << 16) | (PCGB_SB(s0 >> 24) << 24)) ^ rk[41];
    w2 = (PCGB_SB(s2 & 0xff) | (PCGB_SB((s3 >> 8) & 0xff) << 8) |
          (PCGB_SB((s0 >> 16) & 0xff) << 16) | (PCGB_SB(s1 >> 24) << 24)) ^ rk[42];
    w3 = (PCGB_SB(s3 & 0xff) | (PCGB_SB((s0 >> 8) & 0xff) << 8) |
          (PCGB_SB((s1 >> 16) & 0xff) << 16) | (PCGB_SB(s2 >> 24) << 24)) ^ rk[43];
#undef PCGB_SB
#undef PCGB_TE
}

__device__ __forceinline__ void aes_ccr_rep(const uint32_t* te_rep, const uint32_t* rk,
                                            uint64_t lo, uint64_t hi, uint64_t& olo,
                                            uint64_t& ohi) {
    uint32_t w0 = static_cast<uint32_t>(lo), w1 = static_cast<uint32_t>(lo >> 32);
    uint32_t w2 = static_cast<uint32_t>(hi), w3 = static_cast<uint32_t>(hi >> 32);
    aes128_encrypt_words_rep(te_rep, rk, w0, w1, w2, w3);
    olo = (w0 | (static_cast<uint64_t>(w1) << 32)) ^ lo;
    ohi = (w2 | (static_cast<uint64_t>(w3) << 32)) ^ hi;
}

// PRMT-addressed form, for kernels that keep one CTA per SM.  Te0 and Te1
// (= rotl8 Te0) are stored 32 times each, lane-interleaved, at a 256-byte
// stride per entry: entry x of table s for lane L is the word at byte
// region + 256x + 128s + 4L, the region 64 KB aligned in the shared window.
// A lookup's shared address is then one byte permute of the state word with
// the lane's base (byte 1 <- the state byte, the region's bits 16-31 and the
// lane/table offset in byte 0 kept), where the replicated form shifts,
// masks and scales the byte into an index.  Te2 and Te3 lookups share one rotation:
// rotl16(Te0[c]) ^ rotl24(Te0[d]) ^ rk = rotl16(Te0[c] ^ Te1[d] ^ rotl16(rk)).
// Every lookup of a warp hits 32 different banks, as in the replicated form.
constexpr uint32_t kAesPrmtRegionBytes = 65536;
// Dynamic shared memory a kernel requests to be sure of holding one aligned
// region wherever its dynamic shared memory starts.
constexpr uint32_t kAesPrmtSmemBytes = 2 * kAesPrmtRegionBytes;

// Shared address of the first 64 KB-aligned region inside `dsm` (which
// holds kAesPrmtSmemBytes): always inside it.
__device__ __forceinline__ uint32_t aes_prmt_region(const void* dsm) {
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(dsm));
    return (base + (kAesPrmtRegionBytes - 1)) & ~(kAesPrmtRegionBytes - 1);
}

// Fills the region from Te0 in global memory; all threads of the CTA take
// part, no barrier inside.
__device__ __forceinline__ void aes_prmt_fill(const void* dsm, const uint32_t* __restrict__ te0) {
    const uint32_t region = aes_prmt_region(dsm);
    uint32_t* R = reinterpret_cast<uint32_t*>(
        static_cast<char*>(const_cast<void*>(dsm)) +
        (region - static_cast<uint32_t>(__cvta_generic_to_shared(dsm))));
    for (uint32_t i = threadIdx.x; i < kAesPrmtRegionBytes / 4; i += blockDim.x) {
        const uint32_t v = __ldg(te0 + (i >> 6));
        R[i] = ((i >> 5) & 1) ? rotl8_u32(v) : v;
    }
}

// Per-lane base addresses of the two tables.
struct AesPrmt {
    uint32_t lb0, lb1;
    const uint32_t* rk;    // 44 words per sub-key, shared memory
    const uint32_t* rkr;   // the same words rotated by 16
};

__device__ __forceinline__ uint32_t lds_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ void aes128_encrypt_words_prmt(uint32_t lb0, uint32_t lb1,
                                                          const uint32_t* __restrict__ rk,
                                                          const uint32_t* __restrict__ rkr,
                                                          uint32_t& w0, uint32_t& w1,
                                                          uint32_t& w2, uint32_t& w3) {
#define PCGB_A0(s, k) lds_u32(__byte_perm((s), lb0, 0x7604 | ((k) << 4)))
#define PCGB_A1(s, k) lds_u32(__byte_perm((s), lb1, 0x7604 | ((k) << 4)))
    uint32_t s0 = w0 ^ rk[0], s1 = w1 ^ rk[1], s2 = w2 ^ rk[2], s3 = w3 ^ rk[3];
#pragma unroll
    for (int r = 1; r < 10; ++r) {
        const uint32_t t0 = PCGB_A0(s0, 0) ^ PCGB_A1(s1, 1) ^
                            rotl16_u32(PCGB_A0(s2, 2) ^ PCGB_A1(s3, 3) ^ rkr[4 * r + 0]);
        const uint32_t t1 = PCGB_A0(s1, 0) ^ PCGB_A1(s2, 1) ^
                            rotl16_u32(PCGB_A0(s3, 2) ^ PCGB_A1(s0, 3) ^ rkr[4 * r + 1]);
        const uint32_t t2 = PCGB_A0(s2, 0) ^ PCGB_A1(s3, 1) ^
                            rotl16_u32(PCGB_A0(s0, 2) ^ PCGB_A1(s1, 3) ^ rkr[4 * r + 2]);
        const uint32_t t3 = PCGB_A0(s3, 0) ^ PCGB_A1(s0, 1) ^
                            rotl16_u32(PCGB_A0(s1, 2) ^ PCGB_A1(s2, 3) ^ rkr[4 * r + 3]);
        s0 = t0; s1 = t1; s2 = t2; s3 = t3;
    }
    // Final round: S(x) is byte 1 of Te0[x]; four of them gathered into a word.
#define PCGB_FIN(a, b, c, d, k)                                                            \
    (__byte_perm(__byte_perm(PCGB_A0(a, 0), PCGB_A0(b, 1), 0x0051),                        \
                 __byte_perm(PCGB_A0(c, 2), PCGB_A0(d, 3), 0x0051), 0x5410) ^ rk[k])
    w0 = PCGB_FIN(s0, s1, s2, s3, 40);
    w1 = PCGB_FIN(s1, s2, s3, s0, 41);
    w2 = PCGB_FIN(s2, s3, s0, s1, 42);
    w3 = PCGB_FIN(s3, s0, s1, s2, 43);
#undef PCGB_FIN
#undef PCGB_A1
#undef PCGB_A0
}

__device__ __forceinline__ void aes_ccr_prmt(const AesPrmt& a, int k, uint64_t lo, uint64_t hi,
                                             uint64_t& olo, uint64_t& ohi) {
    uint32_t w0 = static_cast<uint32_t>(lo), w1 = static_cast<uint32_t>(lo >> 32);
    uint32_t w2 = static_cast<uint32_t>(hi), w3 = static_cast<uint32_t>(hi >> 32);
    aes128_encrypt_words_prmt(a.lb0, a.lb1, a.rk + 44 * k, a.rkr + 44 * k, w0, w1, w2, w3);
    olo = (w0 | (static_cast<uint64_t>(w1) << 32)) ^ lo;
    ohi = (w2 | (static_cast<uint64_t>(w3) << 32)) ^ hi;
}

// Round keys of up to 15 sub-keys in shared memory, plain and rotated by 16.
struct AesPrmtKeys {
    uint32_t rk[15 * 44], rkr[15 * 44];
};

// CTA set-up of the PRMT form: fills the table region of `dsm` (which holds
// kAesPrmtSmemBytes) and the NK sub-keys' round keys, then a barrier; every
// thread of the CTA must call it.
template <int NK>
__device__ __forceinline__ AesPrmt aes_prmt_setup(unsigned char* dsm, AesPrmtKeys& keys,
                                                  const uint32_t* __restrict__ te,
                                                  const uint32_t* __restrict__ rk) {
    aes_prmt_fill(dsm, te);
    for (int i = threadIdx.x; i < NK * 44; i += blockDim.x) {
        const uint32_t v = rk[i];
        keys.rk[i] = v;
        keys.rkr[i] = rotl16_u32(v);
    }
    __syncthreads();
    const uint32_t lb0 = aes_prmt_region(dsm) | ((threadIdx.x & 31u) * 4u);
    return AesPrmt{lb0, lb0 | 128u, keys.rk, keys.rkr};
}

// Correlation-robust hash H(x) = AES_k(x) ^ x on a node held as (lo, hi).
__device__ __forceinline__ void aes_ccr(const uint32_t* te, const uint32_t* rk, uint64_t lo,
                                        uint64_t hi, uint64_t& olo, uint64_t& ohi) {
    uint32_t w0 = static_cast<uint32_t>(lo), w1 = static_cast<uint32_t>(lo >> 32);
    uint32_t w2 = static_cast<uint32_t>(hi), w3 = static_cast<uint32_t>(hi >> 32);
    aes128_encrypt_words(te, rk, w0, w1, w2, w3);
    olo = (w0 | (static_cast<uint64_t>(w1) << 32)) ^ lo;
    ohi = (w2 | (static_cast<uint64_t>(w3) << 32)) ^ hi;
}

}  // namespace pcgb

#endif
