// Device ChaCha8 keystream block, register resident.
//
// State: words 0..3 the "expand 32-byte k" constants, 4..11 the 256-bit key
// (the DPF node in words 4..7, zeros in 8..11), 12..13 the block counter,
// 14..15 the nonce.  Four double rounds, then the feed-forward add.  Same
// keystream as the reference's ChaCha8PRG (CPU_baseline/chacha8.h:106-150)
// as used by ChaCha8TreePRG / ChaCha8OutHash (tree_prg.h:80-148).
//
// Rotations by 16 and 8 are byte permutes (PRMT), by 12 and 7 funnel shifts
// (SHF); callers read only the output words they need and the compiler
// drops the dead tail of the last round.
#ifndef PCGB_CHACHA8_CUH_
#define PCGB_CHACHA8_CUH_

#include <cstdint>

namespace pcgb {

__device__ __forceinline__ uint32_t rot16(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t rot8(uint32_t x) { return __byte_perm(x, 0, 0x2103); }
__device__ __forceinline__ uint32_t rot12(uint32_t x) { return __funnelshift_l(x, x, 12); }
__device__ __forceinline__ uint32_t rot7(uint32_t x) { return __funnelshift_l(x, x, 7); }

#define PCGB_QR(a, b, c, d)              \
    a += b; d ^= a; d = rot16(d);        \
    c += d; b ^= c; b = rot12(b);        \
    a += b; d ^= a; d = rot8(d);         \
    c += d; b ^= c; b = rot7(b);

// o[i] = keystream word i of the block with key (k0..k3, 0,0,0,0),
// counter (c0, 0) and nonce (n0, n1).
__device__ __forceinline__ void chacha8_block(uint32_t k0, uint32_t k1, uint32_t k2,
                                              uint32_t k3, uint32_t c0, uint32_t n0,
                                              uint32_t n1, uint32_t (&o)[16]) {
    const uint32_t s0 = 0x61707865u, s1 = 0x3320646eu, s2 = 0x79622d32u, s3 = 0x6b206574u;
    uint32_t x0 = s0, x1 = s1, x2 = s2, x3 = s3;
    uint32_t x4 = k0, x5 = k1, x6 = k2, x7 = k3;
    uint32_t x8 = 0, x9 = 0, x10 = 0, x11 = 0;
    uint32_t x12 = c0, x13 = 0, x14 = n0, x15 = n1;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        PCGB_QR(x0, x4, x8, x12)
        PCGB_QR(x1, x5, x9, x13)
        PCGB_QR(x2, x6, x10, x14)
        PCGB_QR(x3, x7, x11, x15)
        PCGB_QR(x0, x5, x10, x15)
        PCGB_QR(x1, x6, x11, x12)
        PCGB_QR(x2, x7, x8, x13)
        PCGB_QR(x3, x4, x9, x14)
    }
    o[0] = x0 + s0;   o[1] = x1 + s1;   o[2] = x2 + s2;   o[3] = x3 + s3;
    o[4] = x4 + k0;   o[5] = x5 + k1;   o[6] = x6 + k2;   o[7] = x7 + k3;
    o[8] = x8;        o[9] = x9;        o[10] = x10;      o[11] = x11;
    o[12] = x12 + c0; o[13] = x13;      o[14] = x14 + n0; o[15] = x15 + n1;
}

// Low 64 bits of the output-layer hash of a leaf (nonce "out_hash", ctr 0).
__device__ __forceinline__ uint64_t out_hash_lo64(uint64_t lo, uint64_t hi) {
    uint32_t o[16];
    chacha8_block(static_cast<uint32_t>(lo), static_cast<uint32_t>(lo >> 32),
                  static_cast<uint32_t>(hi), static_cast<uint32_t>(hi >> 32), 0,
                  0x68617368u /* lo32("out_hash") */, 0x6f75745fu, o);
    return o[0] | (static_cast<uint64_t>(o[1]) << 32);
}

// Tree hash chunk: H_k for k in [4*blk, 4*blk+4): words 4c..4c+3 of block blk.
__device__ __forceinline__ void tree_block(uint64_t lo, uint64_t hi, uint32_t blk,
                                           uint32_t (&o)[16]) {
    chacha8_block(static_cast<uint32_t>(lo), static_cast<uint32_t>(lo >> 32),
                  static_cast<uint32_t>(hi), static_cast<uint32_t>(hi >> 32), blk, 0, 0, o);
}

}  // namespace pcgb

#endif
