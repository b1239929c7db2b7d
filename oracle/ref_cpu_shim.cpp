// C entry points over the reference's own standalone CPU headers, compiled in
// place from the reference tree (see oracle/Makefile).  TEST INFRASTRUCTURE:
// used only to validate the oracle restatement (tests/) byte for byte.
//   chacha8.h : CPU_baseline/chacha8.h      (ChaCha8PRG)
//   ntt.h     : CPU_baseline/ntt.h          (NTT<P>::poly_mul, forward)
//   ntt_roots : GPU_baseline/common/ntt_roots.h (negacyclic_psi)
#include <cstdint>
#include <cstring>
#include <vector>

#include "chacha8.h"
#include "ntt.h"
#include "common/ntt_roots.h"

namespace {
constexpr uint64_t kP = 4611686018326724609ULL;
}

extern "C" {

// Keystream of ChaCha8PRG(key) with set_nonce(nonce) then set_counter(ctr).
void ref_chacha8_keystream(const uint8_t key[32], uint64_t nonce, uint64_t ctr,
                           uint8_t* out, size_t nblocks) {
    ChaCha8PRG prg(key);
    prg.set_nonce(nonce);
    prg.set_counter(ctr);
    prg.fill_blocks(out, nblocks);
}

void ref_ntt_poly_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, int batch, int N) {
    NTT<kP> ntt(N);
    std::vector<FFp<kP>> fa(N), fb(N), fc(N);
    for (int k = 0; k < batch; ++k) {
        for (int i = 0; i < N; ++i) {
            fa[i] = FFp<kP>(a[static_cast<size_t>(k) * N + i]);
            fb[i] = FFp<kP>(b[static_cast<size_t>(k) * N + i]);
        }
        ntt.poly_mul(fc.data(), fa.data(), fb.data());
        for (int i = 0; i < N; ++i) c[static_cast<size_t>(k) * N + i] = fc[i].val();
    }
}

// NTT<P>::forward of `batch` polys in place (inputs reduced by FFp's
// constructor): the slot order the reference's triple extraction uses.
void ref_ntt_forward(uint64_t* a, int batch, int N) {
    NTT<kP> ntt(N);
    std::vector<FFp<kP>> fa(N);
    for (int k = 0; k < batch; ++k) {
        for (int i = 0; i < N; ++i) fa[i] = FFp<kP>(a[static_cast<size_t>(k) * N + i]);
        ntt.forward(fa.data());
        for (int i = 0; i < N; ++i) a[static_cast<size_t>(k) * N + i] = fa[i].val();
    }
}

uint64_t ref_negacyclic_psi(int N) { return pcg_cuda::negacyclic_psi(kP, N); }

}  // extern "C"
