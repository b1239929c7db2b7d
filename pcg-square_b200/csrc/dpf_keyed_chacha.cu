// ChaCha8 instantiations of the keyed DPF kernels (dpf_keyed_impl.cuh);
// split by PRG so the two halves compile in parallel.
#include "dpf_keyed_impl.cuh"

namespace pcgb {

void keyed_tops_chacha(int K, int levels, int w, const Blk* roots, const Blk* cws,
                     const uint32_t* te, const uint32_t* rk, int to_level, Blk* out, Blk* scratch,
                     cudaStream_t st) {
    tops_for_prg<kPrgChaCha>(K, levels, w, roots, cws, te, rk, to_level, out, scratch, st);
}

void keyed_leaf_chacha(int w, int sl, const LeafLaunch& L) { leaf_for_prg<kPrgChaCha>(w, sl, L); }

void keyed_deal_chacha(int w, unsigned grid, size_t smem, uint64_t seed, int c, int t, int n,
                     uint64_t bin, Blk* roots0, Blk* roots1, Blk* cws, uint64_t* cw_out,
                     const uint32_t* te, const uint32_t* rk, uint64_t r2, cudaStream_t st) {
    deal_for_prg<kPrgChaCha>(w, grid, smem, seed, c, t, n, bin, roots0, roots1, cws, cw_out, te, rk,
                       r2, st);
}

void keyed_tops_multi_chacha(int w, const std::vector<TopsJob>& jobs, TopsJob* d_jobs,
                             unsigned long long total, cudaStream_t st) {
    tops_multi_for_prg<kPrgChaCha>(w, jobs, d_jobs, total, nullptr, nullptr, st);
}

void keyed_leaf_multi_chacha(int w, int sl, const LeafJob* d_jobs, int njobs, unsigned ctas, int tpb,
                          size_t smem, const uint32_t* te, const uint32_t* rk, cudaStream_t st) {
    leaf_multi_for_prg<kPrgChaCha>(w, sl, d_jobs, njobs, ctas, tpb, smem, te, rk, st);
}

void deal_multi_chacha_launch(int w, const DealJob* d_jobs, int njobs, unsigned ctas, uint64_t r2,
                              cudaStream_t st) {
    deal_multi_for_chacha(w, d_jobs, njobs, ctas, r2, st);
}

size_t keyed_aes_smem_bytes_chacha() { return sizeof(AesSmem); }

}  // namespace pcgb
