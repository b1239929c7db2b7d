// pcg_cuda:: negacyclic poly-mul entry points with the signatures of the
// reference's GPU_baseline/common/poly_mul_cuda.h:7-33, plus the GPU-NTT
// merge / 4-step names that CPU_baseline/pcg_ole_2pc/pcg_ole.h:147,157,226-230
// calls but the reference tree never defines.  All are served by the same
// four-step sm_100a kernels of libpcg_b200.
#ifndef PCGB_COMPAT_POLY_MUL_CUDA_H_
#define PCGB_COMPAT_POLY_MUL_CUDA_H_

#include <cstdint>
#include <string>

namespace pcg_cuda {

struct PolyMulStats {
    double device_ms = 0.0;
};

bool is_cuda_available();
bool poly_mul_supported(uint64_t prime, int N, std::string* reason = nullptr);
std::string device_name();
std::string runtime_version();

void poly_mul_u64(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
                  uint64_t prime, PolyMulStats* stats = nullptr);

bool poly_mul_gpuntt_supported(uint64_t prime, int N, std::string* reason = nullptr);
void poly_mul_u64_gpuntt(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch, int N,
                         uint64_t prime, PolyMulStats* stats = nullptr);

bool poly_mul_gpuntt_4step_supported(uint64_t prime, int N, std::string* reason = nullptr);
void poly_mul_u64_gpuntt_4step(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch,
                               int N, uint64_t prime, PolyMulStats* stats = nullptr);

bool poly_mul_gpuntt_square_supported(uint64_t prime, int N, std::string* reason = nullptr);
void poly_mul_u64_gpuntt_square(uint64_t* out, const uint64_t* a, const uint64_t* b, int batch,
                                int N, uint64_t prime, PolyMulStats* stats = nullptr);

}  // namespace pcg_cuda

#endif
