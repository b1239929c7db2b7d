/*
 * CPU oracle for the PCG-OLE expansion path (half-tree DPF full-domain
 * evaluation, output-layer convert, negacyclic NTT products).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links or calls
 * this code; only tests/, the smoke check and bench.py's CPU-baseline leg do.
 * Every function restates the reference algorithm it cites (paths are inside
 * the tkgong/pcg-square tree).  Parity is pinned by the reference's own known
 * answers: the FIPS-197 AES vector (GPU_baseline/test/aes_gpu.cpp:57-60), the
 * dpf_real_bench DPF+convert checksums (GPU_baseline/results_l40s/plateau.txt),
 * the NTT product checksums (results_l40s/ntt_naive.txt, ntt_4step.txt), and
 * byte-for-byte agreement with the reference's own chacha8.h / ntt.h compiled
 * from the reference sources (oracle/_ref).
 *
 * All entry points are plain C so Python tests can bind them with ctypes.
 */
#ifndef PCG_ORACLE_H_
#define PCG_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 128-bit node: lo = bytes 0..7, hi = bytes 8..15 (emp::block memory order;
 * GPU_baseline/common/dpf_gpu.h:19-26). */
typedef struct { uint64_t lo, hi; } orc_blk;

#define ORC_PRG_AES 0
#define ORC_PRG_CHACHA8 1

uint64_t orc_prime(void);

/* ---- primitives -------------------------------------------------------- */
/* One ChaCha8 block; key = 8 words, 64-bit counter, 64-bit nonce
 * (CPU_baseline/chacha8.h:22-40, :106-150). out = 16 little-endian words. */
void orc_chacha8_block(const uint32_t key[8], uint64_t counter, uint64_t nonce,
                       uint32_t out[16]);
/* out[j*nk+k] = H_k(parents[j]) (tree_prg.h:80-111). */
void orc_tree_hash_chacha8(orc_blk* out, const orc_blk* parents, size_t n, int nk);
/* low 64 bits of ChaCha8OutHash(leaf) (tree_prg.h:128-148). */
uint64_t orc_out_hash_lo64(orc_blk leaf);

void orc_aes128_expand_key(const uint8_t key[16], uint8_t rk[176]);
void orc_aes128_encrypt(const uint8_t rk[176], const uint8_t in[16], uint8_t out[16]);
/* nk sub-key schedules derived from master (tree_prg.h:45-57): rks = nk*176 B. */
void orc_aes_tree_round_keys(const uint8_t master[16], int nk, uint8_t* rks);
/* out[j*nk+k] = AES_{sub_k}(x) ^ x (mkey_prp.h:24-79). */
void orc_tree_hash_aes(orc_blk* out, const orc_blk* parents, size_t n, int nk,
                       const uint8_t* rks);

/* ---- half-tree DPF ----------------------------------------------------- */
/* Exchange callback: peer[0..count) := the other party's CW shares. */
typedef void (*orc_exchange_fn)(const orc_blk* my, orc_blk* peer, size_t count,
                                void* user);
/* Batched interactive full-domain evaluation, one party
 * (half_tree_dpf/dpf.cpp:485-578).  ex == NULL means the peer share is zero
 * (the stub exchange of GPU_baseline/dpf_real_bench.cu:274-283).
 * dltsft layout [b][level][k] (dpf_gpu.h:44-45); out_leaves [b][D]. */
int orc_dpf_batch_full_eval(int B, int n, int w, const orc_blk* roots,
                            const orc_blk* dltsft, const uint8_t* rks, int prg,
                            orc_exchange_fn ex, void* user, orc_blk* out_leaves);
/* Both parties in lockstep, exchange = memory swap.  cws_out (optional)
 * receives the reconstructed CW[b][level][0..nk). */
int orc_dpf_batch_full_eval_2p(int B, int n, int w, const orc_blk* roots0,
                               const orc_blk* roots1, const orc_blk* dlt0,
                               const orc_blk* dlt1, const uint8_t* rks, int prg,
                               orc_blk* leaves0, orc_blk* leaves1, orc_blk* cws_out);
/* Keyed full-domain evaluation with known CWs [k][level][nk]. */
int orc_dpf_keyed_full_eval(int K, int n, int w, const orc_blk* roots,
                            const orc_blk* cws, const uint8_t* rks, int prg,
                            orc_blk* out_leaves);
/* Single-point evaluation (dpf.cpp:302-327). */
orc_blk orc_dpf_eval(orc_blk root, const orc_blk* cws, int n, int w,
                     const uint8_t* rks, int prg, uint64_t j);
/* Dealer for one key: root1 = root0 ^ Delta; CWs per level so that the two
 * parties' trees differ by Delta exactly on the path to alpha (the Gen of
 * dpf.cpp:333-402 with both parties' shares known).  Also the output-layer CW
 * (pcg_ole_impl.h:324-329,397-407 with A, B evaluated at alpha) and the
 * interactive DltSft shares dlt1 = dlt0 ^ [digit==k]*Delta.
 * cws: levels*nk, dlt1: levels*nk (dlt0 given). */
int orc_dpf_deal(int n, int w, orc_blk root0, orc_blk delta, uint64_t alpha,
                 uint64_t beta, const uint8_t* rks, int prg, orc_blk* cws,
                 uint64_t* cw_out, const orc_blk* dlt0, orc_blk* dlt1);

/* ---- output layer (leaf_convert) --------------------------------------- */
/* sumC[b] = sum C mod P, sumT[b] = sum tau (leaf_convert_cuda.h:40-44). */
void orc_out_sums(const orc_blk* leaves, int B, size_t D, uint64_t* sumC,
                  uint64_t* sumT);
/* Folded g (N residues) for one block (leaf_convert_cuda.h:46-52). */
void orc_out_scatter_g(const orc_blk* leaves, int B, size_t D, int t, int party,
                       const uint64_t* CW, uint64_t* g, int N);

/* ---- NTT ---------------------------------------------------------------- */
/* c = a*b mod (X^N+1) over F_P, batch of polys (CPU_baseline/ntt.h:20-158);
 * inputs are reduced mod P first (FFp(uint64_t) constructor, ffp.h:23). */
void orc_poly_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, int batch, int N);
/* Schoolbook negacyclic product (pcg_ole.h:92-106), small N only. */
void orc_poly_mul_schoolbook(uint64_t* c, const uint64_t* a, const uint64_t* b, int N);
/* In-place negacyclic forward NTT of `batch` polys (inputs reduced mod P):
 * output k = A(psi^(2k+1)), the order of NTT<P>::forward (ntt.h:140-144). */
void orc_ntt_forward(uint64_t* a, int batch, int N);

/* ---- Beaver triples from two ring OLEs -----------------------------------
 * One party's N Z_p triple shares (CPU_baseline/pcg_ole_2pc/triple.h:45-110):
 * party 0 takes a = x1, b = x2, party 1 a = x2, b = x1; c = a*b + z1 + z2 in
 * R_p; a, b, c are then forward-NTT'd slot by slot. */
void orc_triples(int N, int party, const uint64_t* x1, const uint64_t* z1, const uint64_t* x2,
                 const uint64_t* z2, uint64_t* a, uint64_t* b, uint64_t* c);
uint64_t orc_mulmod(uint64_t a, uint64_t b);

/* ---- seeded synthetic material + expansion ----------------------------- */
/* Counter-based generator shared with the library's dealer (own definition,
 * since the reference draws from unseeded emp PRGs): with the SplitMix64
 * finaliser mix, rnd(seed, dom, idx) = mix(mix(seed ^ dom * phi) + (idx + 1)
 * * 0xd1b54a32d192ed03), phi = 0x9e3779b97f4a7c15. */
uint64_t orc_rnd(uint64_t seed, uint64_t dom, uint64_t idx);

typedef struct {
    int N, c, t, w, prg;     /* prg: ORC_PRG_* */
    int n, levels, nk, K;    /* derived */
} orc_shape;
int orc_shape_init(orc_shape* s, int N, int c, int t, int w, int prg);

/* Noise for party p: pos[c*t], val[c*t] (pcg_ole_impl.h:62-86). */
void orc_noise(const orc_shape* s, uint64_t seed, int party, uint64_t* pos, uint64_t* val);
/* Public a_1..a_{c-1} (c-1)*N coefficients uniform mod P. */
void orc_public_a(const orc_shape* s, uint64_t a_seed, uint64_t* a);
/* Keys for all K = c*c*t*t instances: roots0/roots1[K], cws[K*levels*nk],
 * cw_out[K].  Key id = (ii*c + jj)*t*t + kk*t + ll. */
int orc_deal_keys(const orc_shape* s, uint64_t seed, const uint8_t* rks,
                  orc_blk* roots0, orc_blk* roots1, orc_blk* cws, uint64_t* cw_out);
/* One party's expansion (pcg_ole_impl.h:213-312 device algebra,
 * :330-449 output layer, :453-484 step 4).  x, z: N each.
 * blocks_mask: run only the DPF blocks whose bit is set (bounded CPU samples);
 * pass ~0 for the full expansion.  threads: worker threads for the DPF part.
 * g_out (optional): c*c*N folded g per block. */
int orc_expand(const orc_shape* s, int party, const orc_blk* roots,
               const orc_blk* cws, const uint64_t* cw_out, const uint64_t* pos,
               const uint64_t* val, const uint64_t* a, const uint8_t* rks,
               uint64_t blocks_mask, int threads, uint64_t* x, uint64_t* z,
               uint64_t* g_out);

/* Step 4 of the expansion (pcg_ole_impl.h:455-483) for any public a_0 ..
 * a_{c-1} (a: c*N; the reference fixes a_0 = 1) and block outputs g (c*c*N,
 * block (i, j) at (i*c + j)*N): x = sum a_i e_i, z = sum_{i,j} a_i a_j g_ij. */
int orc_step4(int N, int c, int t, const uint64_t* pos, const uint64_t* val, const uint64_t* a,
              const uint64_t* g, uint64_t* x, uint64_t* z);

/* Bounded CPU sample of one party's expansion for the timed baseline:
 * output layer of n_blocks blocks x keys_per_block keys (keyed DPF + convert
 * + scatter, as orc_expand) and n_polymuls length-N products, the work split
 * over `threads` threads.  *t_dpf / *t_ntt: wall seconds of the two parts. */
int orc_bench_sample(const orc_shape* s, int party, const orc_blk* roots, const orc_blk* cws,
                     const uint64_t* cw_out, const uint64_t* a, int n_blocks,
                     int keys_per_block, int n_polymuls, int threads, double* t_dpf,
                     double* t_ntt);

/* One whole (i,j) block of one party's expansion on the host: all t^2 keys
 * of block blk (keyed DPF + convert + scatter into the block's g) and
 * n_polymuls length-N step-4 products, from one task queue on `threads`
 * threads.  *seconds: wall time. */
int orc_bench_block(const orc_shape* s, int party, const orc_blk* roots, const orc_blk* cws,
                    const uint64_t* cw_out, const uint64_t* a, int blk, int n_polymuls,
                    int threads, double* seconds);

/* mt19937_64 (reference fixtures use std::mt19937_64). */
void orc_mt64_fill(uint64_t seed, uint64_t* out, size_t n);

#ifdef __cplusplus
}
#endif
#endif
