// Where the four-step NTT (ntt.cu) leaves each evaluation.
//
// For N = n1 * n2 (n1 = 2^l1 rows, n2 = 2^l2 columns) the transform stores
// A(psi^(2(i1 + n1*i2) + 1)) at row brev_l1(i1), and within the row at the
// position the row pass gives output index i = brev_l2(i2): (i % 16) * (n2 /
// 16) + i / 16 when n2 >= 16, else i.  The natural slot order of the
// reference's CPU NTT (slot k = A(psi^(2k+1)), CPU_baseline/ntt.h:140-144)
// is k = i1 + n1*i2.
#ifndef PCGB_NTT_LAYOUT_CUH_
#define PCGB_NTT_LAYOUT_CUH_

#include <cstddef>
#include <cstdint>

namespace pcgb {

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int bits) {
    return bits ? __brev(x) >> (32 - bits) : 0;
}

// Index, in the transform's storage, of natural slot k.
__device__ __forceinline__ size_t ntt_slot_position(size_t k, int l1, int l2) {
    const uint32_t i1 = static_cast<uint32_t>(k & ((size_t{1} << l1) - 1));
    const uint32_t i2 = static_cast<uint32_t>(k >> l1);
    const size_t row = brev_bits(i1, l1);
    const uint32_t i = brev_bits(i2, l2);
    const size_t pos = l2 >= 4 ? static_cast<size_t>(i & 15) * (size_t{1} << (l2 - 4)) + (i >> 4) : i;
    return (row << l2) + pos;
}

}  // namespace pcgb

#endif
