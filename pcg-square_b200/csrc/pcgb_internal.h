// Internal definitions shared by the library's translation units.
#ifndef PCGB_INTERNAL_H_
#define PCGB_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pcg_b200.h"

namespace pcgb {

// The project prime: p = 2^62 - 3*2^25 + 1 (p - 1 = 2^25 * (2^37 - 3)), so
// negacyclic transforms exist up to N = 2^24.
constexpr uint64_t kP = 4611686018326724609ULL;
// Output-layer hash nonce, "out_hash" in ASCII (the tree PRG uses nonce 0).
constexpr uint64_t kOutDomain = 0x6f75745f68617368ULL;
constexpr int kMaxLogN = 24;

struct alignas(16) Blk {
    uint64_t lo, hi;
};
static_assert(sizeof(Blk) == 16, "Blk must be 16 bytes");

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
#define PCGB_CK(call) ::pcgb::check_cuda((call), #call)

// Every kernel launch of the library is followed by PCGB_POST_LAUNCH(): it
// checks the launch and counts it (pcgb_launch_count).
void note_launch();
void note_launches(unsigned long long n);   // kernels replayed from a CUDA graph
#define PCGB_POST_LAUNCH()                                   \
    do {                                                     \
        ::pcgb::check_cuda(cudaGetLastError(), "kernel launch"); \
        ::pcgb::note_launch();                               \
    } while (0)

// Per-device default stream owned by the library (non-blocking).
cudaStream_t default_stream();
inline cudaStream_t as_stream(void* s) {
    return s ? static_cast<cudaStream_t>(s) : default_stream();
}

// Host-to-device copy that has landed when the call returns: a plain
// cudaMemcpy from pageable memory may return before its DMA completes, and
// work on the library's non-blocking streams is not ordered after it.
void upload_blocking(void* d_dst, const void* src, size_t bytes);
// Stream-ordered allocation from the library's own per-device pool, which
// keeps freed memory mapped for the next request (release with
// pcgb_trim_pool).  Free with cudaFreeAsync.
void* pool_alloc(size_t bytes, cudaStream_t st);
cudaMemPool_t library_pool();

// Number of SMs of the current device.
int sm_count();

// ---- keyed DPF (dpf_keyed.cu) ------------------------------------------
// Expand K keys from level 0 to level `to_level` (levels of w bits), writing
// m^to_level nodes per key to `out` ([k][node], natural order).  scratch
// must hold K * m^min(to_level, first_stage_levels) nodes (may be nullptr
// when to_level is small; see keyed_tops_scratch_nodes).
size_t keyed_tops_scratch_nodes(int K, int w, int to_level);

// One key group's part of a multi-group top-walk stage (expand_tops_multi_kernel).
struct TopsJob {
    const Blk* src;             // source nodes [K][m^src_lvl]
    Blk* dst;                   // written nodes [K][m^(src_lvl + nlev)]
    const Blk* cws;             // the group's CWs [K][levels][m-1]
    unsigned long long first;   // first global thread index of this job
    int K, src_lvl, nlev, levels;
};
// Top-level walk of `groups` key groups of different domains (same w and
// PRG), each to its own level to_level[g] into out[g]: one launch per stage
// for all groups.  scratch[g] holds keyed_tops_scratch_nodes(K[g], w,
// to_level[g]) nodes, or is null (scratch from the pool); scratch may be null.
void keyed_tops_multi(int groups, const int* K, const int* n, const int* to_level, int w, int prg,
                      const Blk* const* roots, const Blk* const* cws, const uint32_t* d_rk,
                      Blk* const* out, Blk* const* scratch, cudaStream_t st);
// Full-domain evaluation of `groups` key groups of different domains (same
// w and PRG): one launch per top-walk stage for all groups.
void keyed_full_eval_multi(int groups, const int* K, const int* n, int w, int prg,
                           const Blk* const* roots, const Blk* const* cws, const uint32_t* d_rk,
                           Blk* const* leaves, cudaStream_t st);
void keyed_tops_multi_chacha(int w, const std::vector<TopsJob>& jobs, TopsJob* d_jobs,
                             unsigned long long total, cudaStream_t st);
void keyed_tops_multi_aes(int w, const std::vector<TopsJob>& jobs, TopsJob* d_jobs,
                          unsigned long long total, const uint32_t* te, const uint32_t* rk,
                          cudaStream_t st);
void keyed_expand_tops(int K, int n, int w, int prg, const Blk* roots, const Blk* cws,
                       const uint32_t* d_aes_rk, int to_level, Blk* out, Blk* scratch,
                       cudaStream_t st);

// Contribution list of the gather form of the output-layer scatter: for
// every merged (i<=j) pair q and output bin r, the key halves that land in
// [r*bin, (r+1)*bin) of the folded g (see gather_plan in dpf_keyed.cu).
// Keyed top-level expansion runs in stages.  Each stage gives every node of
// its start level a thread that walks its subtree depth first down to the
// next boundary; the thread count grows at most 32-fold per stage (so the
// early, narrow stages do short walks) until K * m^l reaches this many
// subtrees, and the final stage walks from there to the target level.
// 2^19 threads keep every SM busy and the final walks shallow.
constexpr size_t kTopsStage2Threads = size_t{1} << 19;
// w = 1 ChaCha8 stages of up to this many levels walk a depth fixed at
// compile time (registers only); for w = 1 no stage is made deeper.
constexpr int kTopsFixedLevels = 8;
// Stage boundaries 0 = l_0 < l_1 < ... < l_s = to_level.
std::vector<int> tops_stages(int K, int w, int to_level);

struct GatherPlan {
    int N = 0, c = 0, t = 0, n = 0, w = 0, Q = 0;
    int sl = 0;          // levels expanded per thread in the leaf kernel
    int S = 0;           // leaves per thread = m^sl
    int hl = 0;          // frontier level = levels - sl
    int tpb = 0;         // leaf-kernel threads per CTA (0 = 256, halved to fit a bin)
    uint32_t* d_off = nullptr;      // [Q*t + 1]
    uint32_t* d_entries = nullptr;  // key_id << 2 | half << 1 | fold_negate
    uint16_t* d_qorder = nullptr;   // launch order of this shard's pairs (heavy first)
    uint16_t* d_qslot = nullptr;    // output slot of each launched pair
    std::vector<uint32_t> pair_ij;  // pair q -> block index i*c + j (i <= j)
    std::vector<int> shard_pairs;   // pairs of this shard, ascending; slot = index
    int rank = 0, world = 1;
    int Qs = 0;                     // pairs of this shard (Q when world = 1)
    int n_entries = 0;
};
// A shard (rank of world) owns a subset of the Q pairs, balanced by work
// (off-diagonal pairs weigh 2 blocks, diagonal 1), and writes and
// transforms only those, in slot order.  world = 1 owns all, slot = q.
void gather_plan_build(GatherPlan& gp, int N, int c, int t, int n, int w, int rank = 0,
                       int world = 1);
void gather_plan_free(GatherPlan& gp);

// Launch parameters of the fused leaf kernel (dpf_keyed_impl.cuh).
struct LeafLaunch {
    dim3 grid;
    int tpb = 0;
    size_t smem = 0;
    cudaStream_t st = nullptr;
    const Blk* F = nullptr;
    const Blk* cws = nullptr;
    const uint64_t* cw_out = nullptr;
    const uint32_t* off = nullptr;
    const uint32_t* entries = nullptr;
    const uint16_t* q_order = nullptr;
    const uint16_t* q_slot = nullptr;
    int t = 0, levels = 0, hl = 0;
    size_t bin = 0;
    int N = 0, party = 0;
    const uint32_t* te = nullptr;
    const uint32_t* rk = nullptr;
    uint64_t* gq = nullptr;
};

// One expansion's part of a multi-expansion leaf launch: its LeafLaunch
// fields plus its CTA range [first, first + gx*gy*gz) in the shared grid.
struct LeafJob {
    const Blk* F;
    const Blk* cws;
    const uint64_t* cw_out;
    const uint32_t* off;
    const uint32_t* entries;
    const uint16_t* q_order;
    const uint16_t* q_slot;
    uint64_t* gq;
    size_t bin;
    int t, levels, hl, N, party;
    unsigned gx, gy, first;
};

// One expansion's part of a multi-expansion dealer launch (ChaCha8).
struct DealJob {
    uint64_t seed;
    Blk* roots0;
    Blk* roots1;
    Blk* cws;
    uint64_t* cw_out;
    uint64_t bin;
    int c, t, n;
    unsigned first;   // first CTA (128 threads, one key each)
};
void deal_multi_chacha_launch(int w, const DealJob* d_jobs, int njobs, unsigned ctas, uint64_t r2,
                              cudaStream_t st);

// Per-PRG instantiations (dpf_keyed_chacha.cu / dpf_keyed_aes.cu).
#define PCGB_KEYED_DECL(NAME)                                                                   \
    void keyed_tops_##NAME(int K, int levels, int w, const Blk* roots, const Blk* cws,          \
                           const uint32_t* te, const uint32_t* rk, int to_level, Blk* out,     \
                           Blk* scratch, cudaStream_t st);                                     \
    void keyed_leaf_##NAME(int w, int sl, const LeafLaunch& L);                                 \
    void keyed_leaf_multi_##NAME(int w, int sl, const LeafJob* d_jobs, int njobs, unsigned ctas, \
                                 int tpb, size_t smem, const uint32_t* te, const uint32_t* rk,  \
                                 cudaStream_t st);                                              \
    void keyed_deal_##NAME(int w, unsigned grid, size_t smem, uint64_t seed, int c, int t,      \
                           int n, uint64_t bin, Blk* roots0, Blk* roots1, Blk* cws,            \
                           uint64_t* cw_out, const uint32_t* te, const uint32_t* rk,           \
                           uint64_t r2, cudaStream_t st);                                      \
    size_t keyed_aes_smem_bytes_##NAME();
PCGB_KEYED_DECL(chacha)
PCGB_KEYED_DECL(aes)
#undef PCGB_KEYED_DECL

// Fused leaf kernel: frontier F (level hl) -> leaves -> out-hash -> convert
// -> gather into the folded, pair-merged g' (Q buffers of N residues).
void keyed_leaf_gather(const GatherPlan& gp, int party, int prg, const Blk* F, const Blk* cws,
                       const uint64_t* cw_out, const uint32_t* d_aes_rk, uint64_t* gq,
                       cudaStream_t st);

// ---- expander internals (expand.cu) ----------------------------------------
struct Workspace {
    Blk* F = nullptr;
    Blk* tops = nullptr;
    uint64_t* g = nullptr;
};
// rank/world: this expander's shard of the pair blocks (see GatherPlan).
// public_a: a_1 .. a_{c-1} (a_0 = 1, the reference's convention), or with
// a0_public a_0 .. a_{c-1}; N coefficients each.
pcgb_expander* expander_create(int N, int c, int t, int w, int prg, const uint64_t* public_a,
                               const uint8_t* master_key, int rank = 0, int world = 1,
                               int a0_public = 0);
void expander_shard(const pcgb_expander* e, int* rank, int* world, int* q_local, int* q_total);
void expander_destroy(pcgb_expander* e);
void expander_info(const pcgb_expander* e, int* K, int* levels, int* nk, size_t* scratch);
int expander_autotune(pcgb_expander* e);  // leaf shape (leaves/thread, CTA size), cached per shape
// Pins the leaf shape to one of the autotuner's candidates.
void expander_set_leaf_shape(pcgb_expander* e, int tpb, int leaves_per_thread);
// Largest leaves-per-thread exponent of the fused leaf kernel for (n, w).
int leaf_sl_max(int n, int w);
void expander_leaf_shape(const pcgb_expander* e, int* tpb, int* leaves_per_thread);
void expand_host_async(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                       const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val,
                       uint64_t* x, uint64_t* z);
void expander_wait(pcgb_expander* e);
void expand_from_g_device(pcgb_expander* e, const uint64_t* g, const uint64_t* pos,
                          const uint64_t* val, uint64_t* x, uint64_t* z, cudaStream_t st);
void expander_set_graph(pcgb_expander* e, bool on);
size_t workspace_bytes(const pcgb_expander* e);
Workspace workspace_carve(const pcgb_expander* e, void* base);
void expand_device_ws(pcgb_expander* e, const Workspace& ws, int party, const Blk* roots,
                      const Blk* cws, const uint64_t* cw_out, const uint64_t* pos,
                      const uint64_t* val, uint64_t* x, uint64_t* z, cudaStream_t st);
// Several expansions of different shapes as one batch (ChaCha8, the same w
// and leaf shape for all; N in 2^14 .. 2^20): one launch per stage for the
// whole batch; each request's outputs equal expand_device_ws's.
void expand_batch_ws(int count, pcgb_expander* const* e, const Workspace* ws, const int* party,
                     const Blk* const* roots, const Blk* const* cws,
                     const uint64_t* const* cw_out, const uint64_t* const* pos,
                     const uint64_t* const* val, uint64_t* const* x, uint64_t* const* z,
                     cudaStream_t st);
void deal_noise_multi_device(int count, pcgb_expander* const* e, const uint64_t* seed,
                             const int* party, Blk* const* r0, Blk* const* r1, Blk* const* cws,
                             uint64_t* const* cwo, uint64_t* const* pos, uint64_t* const* val,
                             cudaStream_t st);
void digest_multi_device(int count, const uint64_t* const* v, const size_t* n, uint64_t* const* out,
                         cudaStream_t st);
void deal_keys_device(pcgb_expander* e, uint64_t seed, Blk* r0, Blk* r1, Blk* cws, uint64_t* cwo,
                      cudaStream_t st);
void noise_device(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val,
                  cudaStream_t st);
void public_a_host(int N, int c, uint64_t a_seed, uint64_t* a);
void digest_device(const uint64_t* d, size_t n, uint64_t* out, cudaStream_t st);

// ---- AES tree PRG (aes_tables.cu) ---------------------------------------
// Round keys as 44 little-endian words per sub-key, on the device.
uint32_t* aes_upload_round_keys(const uint8_t* rks_bytes, int nk, cudaStream_t st);
const uint32_t* aes_te_table_device();   // 4 x 256 words, resident
void aes_expand_key_host(const uint8_t key[16], uint8_t rk[176]);
void aes_encrypt_host(const uint8_t rk[176], const uint8_t in[16], uint8_t out[16]);
void aes_tree_round_keys_host(const uint8_t master[16], int nk, uint8_t* rks);

// ---- NTT (ntt.cu) --------------------------------------------------------
struct NttPlan;
const NttPlan& ntt_plan(int logN);   // resident per (device, logN)
// In-place forward transform of `batch` length-N polys into the internal
// evaluation layout (coefficients must be < p).
void ntt_forward(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st);
// dst = forward transform of src (batch polys, contiguous); reduce maps any
// uint64 input into [0, p) first, else inputs must be below 4p.
void ntt_forward_from(const NttPlan& pl, const uint64_t* src, uint64_t* dst, int batch,
                      bool reduce, cudaStream_t st);
void ntt_log_sizes(const NttPlan& pl, int* l1, int* l2);   // see ntt_layout.cuh
// c = a * b mod (X^N+1) for `batch` polys; c may alias a or b; inputs any
// uint64 (reduced mod p first).  scratch: batch*N words.
void poly_mul_device(const NttPlan& pl, uint64_t* c, const uint64_t* a, const uint64_t* b,
                     int batch, uint64_t* scratch, cudaStream_t st);
// c[i] = a[i] * b[i] mod (X^N_i + 1) for polynomials of different lengths
// N_i = 2^logN[i] in 2^16 .. 2^20, five launches for the whole batch; c[i]
// may alias a[i] or b[i]; inputs any uint64.
bool poly_mul_mixed_ok(int logN);
void poly_mul_device_mixed(int count, uint64_t* const* c, const uint64_t* const* a,
                           const uint64_t* const* b, const int* logN, cudaStream_t st);
// acc = INTT( sum_q img[q] (.) NTT(g[q]) ); g is consumed (transformed in
// place); img in Montgomery-scaled evaluation layout.
void ntt_mac_inverse(const NttPlan& pl, uint64_t* g, const uint64_t* img, int Q, uint64_t* acc,
                     cudaStream_t st);
// The same for `count` requests of different lengths N_i = 2^logN[i] in
// 2^14 .. 2^20 (Q[i] buffers each), three launches for all of them.
bool ntt_mac_multi_ok(int logN);
void ntt_mac_inverse_multi(int count, uint64_t* const* g, const uint64_t* const* img, const int* Q,
                           uint64_t* const* z, const int* logN, cudaStream_t st);
// Pointwise c[i] = a[i]*b[i]*R mod p over `count` words (R = 2^64): turns
// an evaluation vector into its Montgomery-scaled form when b = R^2 scaled.
void pointwise_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, size_t count, int mode,
                   cudaStream_t st);
void reduce_mod_p(uint64_t* d, const uint64_t* s, size_t count, cudaStream_t st);

// ---- triples and relation checks (triples.cu) ----------------------------
// d = (u + v) mod p for any 64-bit u, v.
void add_mod_p_device(uint64_t* d, const uint64_t* u, const uint64_t* v, size_t count,
                      cudaStream_t st);
void triples_device(int N, int party, const uint64_t* x1, const uint64_t* z1, const uint64_t* x2,
                    const uint64_t* z2, uint64_t* a, uint64_t* b, uint64_t* c, cudaStream_t st);
void verify_ole_device(int N, const uint64_t* x0, const uint64_t* z0, const uint64_t* x1,
                       const uint64_t* z1, unsigned long long* bad, cudaStream_t st);
void verify_triples_device(int N, const uint64_t* a0, const uint64_t* b0, const uint64_t* c0,
                           const uint64_t* a1, const uint64_t* b1, const uint64_t* c1,
                           unsigned long long* bad, cudaStream_t st);

// ---- boolean preprocessing, two-party GMW (gmw.cu) -------------------------
size_t gmw_position_add_gates(int off_bits);
size_t gmw_dltsft_gates(int n, int w);
void gmw_position_add(int party, int B, int off_bits, const uint64_t* my_off, const uint32_t* ta,
                      const uint32_t* tb, const uint32_t* tc, pcgb_exchange_fn ex, void* user,
                      uint64_t* alpha_share, cudaStream_t st);
void gmw_dltsft(int party, int B, int n, int w, const uint64_t* alpha_share, Blk* delta_share,
                const uint32_t* ta, const uint32_t* tb, const uint32_t* tc, pcgb_exchange_fn ex,
                void* user, Blk* dltsft, cudaStream_t st);

}  // namespace pcgb

#endif
