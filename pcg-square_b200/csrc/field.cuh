// Arithmetic mod p = 2^62 - 3*2^25 + 1 on 64-bit words (device + host).
//
// Values are kept canonical in [0, p).  Multiplication by a fixed constant
// uses Shoup's precomputed quotient (w' = floor(w*2^64/p)); a product of two
// variables uses Montgomery reduction with R = 2^64.
#ifndef PCGB_FIELD_CUH_
#define PCGB_FIELD_CUH_

#include <cstdint>

namespace pcgb {

constexpr uint64_t kPm = 4611686018326724609ULL;

constexpr uint64_t neg_inv_p() {
    uint64_t inv = 1;  // Newton iteration for p^-1 mod 2^64
    for (int i = 0; i < 7; ++i) inv *= 2 - kPm * inv;
    return ~inv + 1;
}
constexpr uint64_t kPNegInv = neg_inv_p();
static_assert(kPm * (~kPNegInv + 1) == 1, "bad inverse");

#if defined(__CUDACC__)
#define PCGB_HD __host__ __device__ __forceinline__
#else
#define PCGB_HD inline
#endif

PCGB_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) >> 64);
#endif
}

PCGB_HD uint64_t add_p(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= kPm ? s - kPm : s;
}
PCGB_HD uint64_t sub_p(uint64_t a, uint64_t b) { return a >= b ? a - b : a + kPm - b; }
PCGB_HD uint64_t neg_p(uint64_t a) { return a ? kPm - a : 0; }

// x mod p for any 64-bit x: p = 2^62 - d with d < 2^27, so subtracting
// (x >> 62) * p leaves a value below 2^62 + 4d < 2p.
PCGB_HD uint64_t reduce_p(uint64_t x) {
    x -= (x >> 62) * kPm;
    return x >= kPm ? x - kPm : x;
}

// Montgomery product a*b*2^-64 mod p for a, b < p.
PCGB_HD uint64_t mont_mul(uint64_t a, uint64_t b) {
    const uint64_t lo = a * b;
    const uint64_t hi = mulhi64(a, b);
    const uint64_t m = lo * kPNegInv;
    const uint64_t t = mulhi64(m, kPm);
    uint64_t r = hi + t + (lo != 0 ? 1 : 0);
    return r >= kPm ? r - kPm : r;
}

// a*w mod p with wq = floor(w*2^64/p); a any 64-bit value below 2^63.
PCGB_HD uint64_t shoup_mul(uint64_t a, uint64_t w, uint64_t wq) {
    const uint64_t q = mulhi64(a, wq);
    uint64_t r = a * w - q * kPm;
    return r >= kPm ? r - kPm : r;
}

inline uint64_t mul_p_host(uint64_t a, uint64_t b) {
    return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) % kPm);
}
inline uint64_t pow_p_host(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= kPm;
    while (e) {
        if (e & 1) r = mul_p_host(r, b);
        b = mul_p_host(b, b);
        e >>= 1;
    }
    return r;
}
inline uint64_t shoup_q_host(uint64_t w) {
    return static_cast<uint64_t>((static_cast<unsigned __int128>(w) << 64) / kPm);
}
// 2^64 mod p and 2^128 mod p.
inline uint64_t r_mod_p() { return static_cast<uint64_t>(((unsigned __int128)1 << 64) % kPm); }
inline uint64_t r2_mod_p() { return mul_p_host(r_mod_p(), r_mod_p()); }

}  // namespace pcgb

#endif
