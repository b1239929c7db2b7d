// Seeded synthetic PCG material: a counter-based generator so the host, the
// GPU dealer and the CPU oracle derive identical noise, keys and public
// polynomials from (seed, domain, index) without sharing state.
//   rnd(seed, dom, idx) = mix(mix(seed ^ dom*phi) + (idx+1)*c2)
// with mix the SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014).
#ifndef PCGB_SYNTH_H_
#define PCGB_SYNTH_H_

#include <cstdint>

#include "field.cuh"

namespace pcgb {

enum : uint64_t {
    kDomPos = 0x10, kDomVal = 0x20, kDomA = 0x30, kDomDelta = 0x40, kDomRoot = 0x50,
};

PCGB_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

PCGB_HD uint64_t synth_rnd(uint64_t seed, uint64_t dom, uint64_t idx) {
    return mix64(mix64(seed ^ (dom * 0x9e3779b97f4a7c15ULL)) + (idx + 1) * 0xd1b54a32d192ed03ULL);
}

// Regular noise of party `party`, polynomial i, block k: offset within the
// block of N/t and the nonzero value in [1, p-1].
PCGB_HD uint64_t synth_offset(uint64_t seed, int party, uint64_t idx, uint64_t bin) {
    return synth_rnd(seed, kDomPos + party, idx) % bin;
}
PCGB_HD uint64_t synth_value(uint64_t seed, int party, uint64_t idx) {
    return synth_rnd(seed, kDomVal + party, idx) % (kPm - 1) + 1;
}

}  // namespace pcgb

#endif
