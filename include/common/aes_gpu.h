// pcg_cuda:: AES-128 entry points with the signatures of the reference's
// GPU_baseline/common/aes_gpu.h:10-21, served by libpcg_b200.
#ifndef PCGB_COMPAT_AES_GPU_H_
#define PCGB_COMPAT_AES_GPU_H_

#include <cstdint>

namespace pcg_cuda {

// FIPS-197 AES-128 key schedule: 16-byte key -> 176 round-key bytes.
void aes128_expand_key_host(const uint8_t key[16], uint8_t round_keys[176]);

// ECB-encrypt `count` blocks on the GPU, each under its own 16-byte key.
void aes128_ecb_encrypt_gpu(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count);

}  // namespace pcg_cuda

#endif
