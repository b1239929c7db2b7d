// pcg_cuda:: DPF entry points with the signatures of the reference's
// GPU_baseline/common/dpf_gpu.h:17-77, served by libpcg_b200 (see
// include/pcg_b200.h).  Pointing the reference build's include path at this
// directory and linking libpcg_b200.so replaces GPU_baseline/common/dpf_gpu.cu.
#ifndef PCGB_COMPAT_DPF_GPU_H_
#define PCGB_COMPAT_DPF_GPU_H_

#include <cstddef>
#include <cstdint>
#include <functional>

namespace pcg_cuda {

// 128-bit node; lo = bytes 0..7, hi = bytes 8..15 (emp::block memory order).
struct alignas(16) DpfBlk {
    uint64_t lo;
    uint64_t hi;
};

// Per-level correction-word exchange: peer_cws[0..count) := peer's shares.
using DpfExchangeFn =
    std::function<void(const DpfBlk* my_cws, DpfBlk* peer_cws, size_t count)>;

enum class DpfGpuPrg { AES, CHACHA8 };

// B instances of domain 2^n, branching 2^w; roots[B]; dltsft[B][n/w][2^w-1];
// round_keys (AES only) (2^w-1)*176 bytes; out_leaves[B][2^n].  Throws
// std::runtime_error on failure.
void dpf_gpu_batch_full_eval(int B, int n, int w, const DpfBlk* roots, const DpfBlk* dltsft,
                             const uint8_t* round_keys, int party, const DpfExchangeFn& exchange,
                             DpfBlk* out_leaves, DpfGpuPrg prg = DpfGpuPrg::AES);

// Leaves stay on the device; the pointer aliases an internal pool and stays
// valid until the next dpf_gpu_* call.
const DpfBlk* dpf_gpu_batch_full_eval_device(int B, int n, int w, const DpfBlk* roots,
                                             const DpfBlk* dltsft, const uint8_t* round_keys,
                                             int party, const DpfExchangeFn& exchange,
                                             DpfGpuPrg prg = DpfGpuPrg::AES);

}  // namespace pcg_cuda

#endif
