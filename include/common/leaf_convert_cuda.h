// pcg_cuda:: output-layer entry points with the signatures of the
// reference's GPU_baseline/common/leaf_convert_cuda.h:33-54, served by
// libpcg_b200.
#ifndef PCGB_COMPAT_LEAF_CONVERT_CUDA_H_
#define PCGB_COMPAT_LEAF_CONVERT_CUDA_H_

#include <cstddef>
#include <cstdint>

#include "common/dpf_gpu.h"

namespace pcg_cuda {

// Output-layer hash nonce ("out_hash"); the tree PRG uses nonce 0.
constexpr uint64_t kOutHashDomain = 0x6f75745f68617368ULL;

// sumC_host[b] = sum_d low64(H'(leaf)) mod prime; sumT_host[b] = sum_d lsb(leaf).
void dpf_out_sums(const DpfBlk* d_leaves, int B, size_t D, uint64_t prime,
                  uint64_t* sumC_host, uint64_t* sumT_host);

// g_out_host (N residues) = folded sum of y = +-(C + tau*CW[b]) at
// (b/t + b%t)*D/2 + d.
void dpf_out_scatter_g(const DpfBlk* d_leaves, int B, size_t D, int t, int party, uint64_t prime,
                       const uint64_t* CW_host, uint64_t* g_out_host, int N);

}  // namespace pcg_cuda

#endif
