/*
 * pcg_b200 — C ABI of the B200 (sm_100a) PCG-OLE expansion library.
 *
 * Two groups of entry points:
 *
 *  1. Drop-ins for the reference's pcg_cuda:: hooks (same argument meaning,
 *     host buffers in and out, same error cases).  Each names the reference
 *     declaration it replaces.  include/common/ declares the C++
 *     pcg_cuda:: wrappers with the reference's exact signatures on top of
 *     these, so CPU_baseline's PCG_ENABLE_CUDA code links unchanged.
 *
 *  2. Native device-resident entry points (keyed DPF, fused expansion,
 *     batched NTT, serving).  Pointers marked d_ are device pointers;
 *     `stream` is a cudaStream_t (NULL = the library's own stream on the
 *     current device).
 *
 * Every function returns 0 on success or a negative PCGB_E* code; the
 * message of the last failure on the calling thread is pcgb_last_error().
 * Nothing here falls back to the CPU: without a usable CUDA device the
 * calls fail with PCGB_ENODEV.
 */
#ifndef PCG_B200_H_
#define PCG_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCGB_OK 0
#define PCGB_EINVAL (-1)   /* bad argument / unsupported shape */
#define PCGB_ECUDA (-2)    /* CUDA runtime error */
#define PCGB_ENODEV (-3)   /* no CUDA device */
#define PCGB_ENOMEM (-4)   /* allocation failed / over the memory budget */
#define PCGB_ECALLBACK (-5) /* exchange callback reported failure */
#define PCGB_ETIMEOUT (-6) /* a bounded wait gave up */
#define PCGB_ESTATE (-7)   /* object in the wrong state (closed, cancelled) */

#define PCGB_PRG_AES 0
#define PCGB_PRG_CHACHA8 1

/* 128-bit DPF node: lo = bytes 0..7, hi = bytes 8..15 (the memory order of
 * emp::block; same layout as pcg_cuda::DpfBlk, GPU_baseline/common/dpf_gpu.h:23-26). */
typedef struct pcgb_blk {
    uint64_t lo, hi;
} pcgb_blk;

/* Per-level correction-word exchange: fill peer[0..count) with the other
 * party's shares of my[0..count).  Return 0, or nonzero to abort the call
 * (reported as PCGB_ECALLBACK).  Replaces the std::function DpfExchangeFn
 * (GPU_baseline/common/dpf_gpu.h:31-32). */
typedef int (*pcgb_exchange_fn)(const pcgb_blk* my, pcgb_blk* peer, size_t count, void* user);
/* The same exchange between device arrays (no reference counterpart): the
 * library has finished writing d_my when it calls; the callback fills
 * d_peer[0..count) on the same device (NCCL send/recv or peer copies over
 * NVLink) and returns once the data has landed. */
typedef int (*pcgb_exchange_device_fn)(const pcgb_blk* d_my, pcgb_blk* d_peer, size_t count,
                                       void* user);

const char* pcgb_last_error(void);
int pcgb_version(void); /* major*10000 + minor*100 + patch */

/* ---- device / runtime -------------------------------------------------- */
/* is_cuda_available / device_name / runtime_version
 * (GPU_baseline/common/poly_mul_cuda.h:13-16). */
int pcgb_is_cuda_available(void); /* 1 or 0 */
int pcgb_device_name(char* buf, size_t len);
int pcgb_runtime_version(char* buf, size_t len);
int pcgb_set_device(int dev);
int pcgb_get_device(int* dev);
int pcgb_sm_count(int* n);
int pcgb_malloc(void** d_ptr, size_t bytes);
int pcgb_free(void* d_ptr);
int pcgb_memcpy_h2d(void* d_dst, const void* src, size_t bytes, void* stream);
int pcgb_memcpy_d2h(void* dst, const void* d_src, size_t bytes, void* stream);
int pcgb_memset(void* d_dst, int value, size_t bytes, void* stream);
int pcgb_stream_synchronize(void* stream);
int pcgb_device_synchronize(void);
/* Scratch that the library allocates per call (drop-in poly-mul and DPF
 * helpers, server requests) comes from a stream-ordered pool of its own on
 * each device, which keeps freed memory mapped so the next call of the same
 * size maps nothing.  Returns that memory on the current device to the
 * driver. */
int pcgb_trim_pool(void);
void* pcgb_default_stream(void);
/* Kernel launches issued by the library since load (all devices). */
unsigned long long pcgb_launch_count(void);
/* Integer-ALU roofline probe: ChaCha8 quarter rounds on register-resident
 * states over every SM; *gops = G int-ops/s (12 ops per quarter round). */
int pcgb_arx_peak(double* gops, float* ms);
/* The same probe as `reps` launches of `iters` double-round iterations each
 * (4096 iterations take about 9 ms on B200); gops[r] = G int-ops/s of launch
 * r, so the caller can report the probe's spread. */
int pcgb_arx_peak_samples(int reps, int iters, double* gops);
/* Pipe-balance variants of the probe: the quarter-round adds selected by
 * add_mask (bit 4q + k = add k of quarter round q of a double round) are
 * issued as multiply-adds, moving them from the integer ALU to the FMA pipe.
 * Masks with an instance: 0, 0x10101010, 0x11111111, 0x22222222,
 * 0x33333333, 0x55555555, 0x15151515, 0x77777777, 0xFFFFFFFF. */
int pcgb_arx_peak_variant(uint32_t add_mask, int reps, int iters, double* gops);
/* CUDA events on the library's streams (device-side timing). */
int pcgb_event_create(void** ev);
int pcgb_event_destroy(void* ev);
int pcgb_event_record(void* ev, void* stream);
/* Waits for `stop`, then *ms = elapsed time start -> stop. */
int pcgb_event_elapsed(void* start, void* stop, float* ms);

/* ---- drop-ins: half-tree DPF (GPU_baseline/common/dpf_gpu.h:55-75) ------ */
/* dpf_gpu_batch_full_eval: B instances, domain 2^n, branching 2^w (w in
 * [1,4], w | n); roots[B]; dltsft[B][n/w][2^w-1]; round_keys: AES only,
 * (2^w-1)*176 bytes; party is accepted and unused (ordering lives inside
 * the exchange); out_leaves[B][2^n]. */
int pcgb_dpf_batch_full_eval(int B, int n, int w, const pcgb_blk* roots,
                             const pcgb_blk* dltsft, const uint8_t* round_keys, int party,
                             pcgb_exchange_fn exchange, void* user, pcgb_blk* out_leaves,
                             int prg);
/* dpf_gpu_batch_full_eval_device: leaves stay on the device; *d_leaves
 * aliases an internal pool, valid until the next pcgb_dpf_batch_* call on
 * this device (B <= 0 gives NULL). */
int pcgb_dpf_batch_full_eval_device(int B, int n, int w, const pcgb_blk* roots,
                                    const pcgb_blk* dltsft, const uint8_t* round_keys, int party,
                                    pcgb_exchange_fn exchange, void* user, int prg,
                                    const pcgb_blk** d_leaves);

/* ---- boolean preprocessing: two-party GMW ------------------------------
 * The circuits in front of the interactive DPF, evaluated on the device
 * for B instances at once: the Kogge-Stone position adder
 * (CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:118-159 over
 * CPU_baseline/bool_circuit/adder.h:22-63) and the DltSft circuit
 * (HalfTreeDPF::batch_F_DeltaShiftShare, CPU_baseline/half_tree_dpf/
 * dpf.cpp:171-283).  The reference's TripleGen (OT) is replaced by an
 * input: boolean AND triples, bit-sliced over instances -- gates rows of
 * W = ceil(B/32) uint32 words each (instance b = bit b%32 of word b/32),
 * XOR shares a, b, c with (a0^a1) & (b0^b1) = c0^c1 -- consumed one row per
 * AND gate.  Each AND depth costs one `exchange` call (party 0's message
 * first in the reference's NetIO order is the callback's concern); messages
 * are whole pcgb_blk, zero-padded.  The callback is required. */
/* AND gates of the position adder (0 if off_bits is outside [1,63]). */
size_t pcgb_gmw_position_add_gates(int off_bits);
/* alpha = off0 + off1 as XOR shares (off_bits + 1 bits, LSB first, the top
 * bit the carry): my_off[B] is this party's offsets (its private input),
 * alpha_share[B] receives its share. */
int pcgb_gmw_position_add(int party, int B, int off_bits, const uint64_t* my_off,
                          const uint32_t* triple_a, const uint32_t* triple_b,
                          const uint32_t* triple_c, pcgb_exchange_fn exchange, void* user,
                          uint64_t* alpha_share);
/* AND gates of the DltSft circuit for domain 2^n, branching 2^w (0 unless
 * 1 <= w <= 8, w | n, n <= 64). */
size_t pcgb_gmw_dltsft_gates(int n, int w);
/* dltsft[B][n/w][2^w-1] shares of [digit_i(alpha) == k] * Delta, digit 0
 * the top w bits of alpha; alpha_share[B] (n bits) and delta_share[B] are
 * XOR shares.  delta_share is updated in place to force lsb(Delta) = 1
 * (party 0 sets its bit 0, party 1 clears it), as the reference does. */
int pcgb_gmw_dltsft(int party, int B, int n, int w, const uint64_t* alpha_share,
                    pcgb_blk* delta_share, const uint32_t* triple_a, const uint32_t* triple_b,
                    const uint32_t* triple_c, pcgb_exchange_fn exchange, void* user,
                    pcgb_blk* dltsft);

/* ---- drop-ins: output layer (GPU_baseline/common/leaf_convert_cuda.h:43-52) */
int pcgb_dpf_out_sums(const pcgb_blk* d_leaves, int B, size_t D, uint64_t prime,
                      uint64_t* sumC_host, uint64_t* sumT_host);
int pcgb_dpf_out_scatter_g(const pcgb_blk* d_leaves, int B, size_t D, int t, int party,
                           uint64_t prime, const uint64_t* CW_host, uint64_t* g_out_host,
                           int N);
/* Device-pointer form of pcgb_dpf_out_scatter_g (no reference counterpart):
 * d_cw (B words in [0, p)) already on the device, folded g written to d_g
 * (N words, every one of them) on `stream`, no host synchronisation; the
 * prime is this library's p. */
int pcgb_dpf_out_scatter_g_device(const pcgb_blk* d_leaves, int B, size_t D, int t, int party,
                                  const uint64_t* d_cw, uint64_t* d_g, int N, void* stream);

/* Output layer hashing each leaf once (no reference counterpart; the pair
 * replaces dpf_out_sums + dpf_out_scatter_g, leaf_convert_cuda.h:43-52, for
 * callers that run both on the same leaves).  The sums pass also stores each
 * leaf's converted word C | tau << 63 in d_conv[B][D] (8 bytes per leaf),
 * and the scatter reads those words instead of hashing the leaves again.
 * Sums and g are as the drop-ins give them, bit for bit.  Device pointers,
 * ordered on `stream`. */
int pcgb_dpf_out_convert_device(const pcgb_blk* d_leaves, int B, size_t D, uint64_t* d_conv,
                                uint64_t* d_sumC, uint64_t* d_sumT, void* stream);
/* pcgb_dpf_batch_full_eval_device followed by pcgb_dpf_out_convert_device
 * in one call, with the last level fused into the sums pass: the leaves are
 * hashed as they are made and never stored (saves writing and re-reading
 * 16 bytes per leaf, and the leaf buffer).  Same arguments as the drop-in
 * plus the three device outputs of the convert pass, identical bit for bit;
 * complete when the call returns. */
int pcgb_dpf_batch_full_eval_convert_device(int B, int n, int w, const pcgb_blk* roots,
                                            const pcgb_blk* dltsft, const uint8_t* round_keys,
                                            int party, pcgb_exchange_fn exchange, void* user,
                                            int prg, uint64_t* d_conv, uint64_t* d_sumC,
                                            uint64_t* d_sumT);
/* Same, with the per-level CW shares exchanged device to device: no host
 * round trip per level, for parties on separate GPUs. */
int pcgb_dpf_batch_full_eval_convert_device_dx(int B, int n, int w, const pcgb_blk* roots,
                                               const pcgb_blk* dltsft, const uint8_t* round_keys,
                                               int party, pcgb_exchange_device_fn exchange,
                                               void* user, int prg, uint64_t* d_conv,
                                               uint64_t* d_sumC, uint64_t* d_sumT);
int pcgb_dpf_out_scatter_g_conv_device(const uint64_t* d_conv, int B, size_t D, int t, int party,
                                       const uint64_t* d_cw, uint64_t* d_g, int N, void* stream);

/* The output-layer Beaver multiplication of the two-party expansion
 * (CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:222-290) on device arrays of B
 * words.  Open: <A> = (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>;
 * d_de[0..B) = <A> - r, d_de[B..2B) = <B> - s (mod p), the message to send.
 * Close, with the peer's message: d = d0 + d1, e = e0 + e1, the CW share is
 * d*s + e*r + rs, plus d*e for party 0.  CW = the sum of the two shares
 * (pcgb_add_mod_p_device). */
int pcgb_out_beaver_open_device(int B, int party, const uint64_t* d_sumC, const uint64_t* d_sumT,
                                const uint64_t* d_beta, const uint64_t* d_r, const uint64_t* d_s,
                                uint64_t* d_de, void* stream);
int pcgb_out_beaver_close_device(int B, int party, const uint64_t* d_de_my,
                                 const uint64_t* d_de_peer, const uint64_t* d_r,
                                 const uint64_t* d_s, const uint64_t* d_rs, uint64_t* d_cw_share,
                                 void* stream);
/* d[i] = (u[i] + v[i]) mod p for any 64-bit u, v (d may alias either). */
int pcgb_add_mod_p_device(uint64_t* d, const uint64_t* u, const uint64_t* v, size_t count,
                          void* stream);

/* Allocation-free variant of pcgb_dpf_out_sums, with no counterpart in the
 * reference.  It is for callers that must not allocate device memory
 * themselves or through the library: code whose device memory is owned by a
 * framework's allocator or capped by a fixed budget, and latency-critical
 * loops where cudaMalloc's implicit device synchronisation is unacceptable.
 * The caller passes the leaves and two device output arrays of B words
 * (d_sumC, d_sumT, same values as sumC_host / sumT_host); the per-CTA
 * partial sums live in a 1 MiB static device array that every device
 * loading the library holds until the process exits, which limits B to at
 * most 65535 instances (larger B is rejected with PCGB_EINVAL).  The call
 * only enqueues work on `stream`: synchronise before reading the outputs.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  The address is kept for the life of the
 * process, like the library's other per-device state: after a
 * cudaDeviceReset it is stale, so do not call the library again on that
 * device in the same process.  All calls on a device share the array, so
 * calls that overlap on the GPU (unordered streams) race; each call
 * overwrites every partial it reads, so nothing needs clearing between
 * calls.  No cudaMalloc, cudaFree or allocating library routine is used. */
int pcgb_dpf_out_sums_noalloc(const pcgb_blk* d_leaves, int B, size_t D, uint64_t prime,
                              uint64_t* d_sumC, uint64_t* d_sumT, void* stream);

/* ---- drop-ins: negacyclic poly-mul (GPU_baseline/common/poly_mul_cuda.h:14-31,
 * plus the merge / 4-step names called from CPU_baseline/pcg_ole_2pc/pcg_ole.h:147,157,226-230).
 * variant selects the supported-size rules of each reference name; all run
 * the same four-step kernels. */
#define PCGB_POLYMUL_V1 0     /* poly_mul_u64: N in [2, 32768] */
#define PCGB_POLYMUL_MERGE 1  /* poly_mul_u64_gpuntt: N in [2, 2^24] */
#define PCGB_POLYMUL_4STEP 2  /* poly_mul_u64_gpuntt_4step: N in [4096, 2^24] */
#define PCGB_POLYMUL_SQUARE 3 /* poly_mul_u64_gpuntt_square: N in [256, 2^24] */
/* 1 if supported, 0 if not (reason filled), <0 on error. */
int pcgb_poly_mul_supported(int variant, uint64_t prime, int N, char* reason, size_t len);
int pcgb_poly_mul_u64(int variant, uint64_t* out, const uint64_t* a, const uint64_t* b,
                      int batch, int N, uint64_t prime, double* device_ms);

/* ---- drop-ins: AES-128 (GPU_baseline/common/aes_gpu.h:13-19) ------------ */
int pcgb_aes128_expand_key(const uint8_t key[16], uint8_t round_keys[176]);
int pcgb_aes128_ecb_encrypt(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count);
/* Tree-PRG sub-key schedules from a master key (half_tree_dpf/tree_prg.h:45-57;
 * half_tree_dpf/dpf.cpp:605-619): nk*176 bytes. */
int pcgb_aes_tree_round_keys(const uint8_t master[16], int nk, uint8_t* round_keys);

/* ---- native: keyed DPF ---------------------------------------------------
 * A keyed instance: root, CW[level][0..2^w-1) (the last child's CW is their
 * XOR), and for the output layer one field element cw_out.  Both parties
 * hold the same CWs; roots differ by Delta. */
/* Full-domain leaves of K keys: d_leaves[K][2^n]. */
int pcgb_dpf_keyed_full_eval(int K, int n, int w, int prg, const pcgb_blk* d_roots,
                             const pcgb_blk* d_cws, const uint8_t* round_keys,
                             pcgb_blk* d_leaves, void* stream);
/* Keyed full-domain evaluation of several key groups with different domains
 * in one batch (no reference counterpart): group g has K[g] keys of domain
 * 2^n[g]; all share w, the PRG and its round keys.  d_roots[g] (K[g]
 * blocks), d_cws[g] ([K[g]][n[g]/w][2^w-1]) and d_leaves[g] ([K[g]][2^n[g]])
 * are device arrays; K, n and the pointer arrays are host arrays.  One
 * launch per top-walk stage serves every group (a persistent grid over a
 * per-stage job table), so the batch takes as many launches as its deepest
 * group has stages; for ChaCha8 with w = 1, one launch per distinct walk
 * depth within a stage (each with the compile-time walk of that depth).
 * Leaves equal pcgb_dpf_keyed_full_eval's per group. */
int pcgb_dpf_keyed_full_eval_multi(int groups, const int* K, const int* n, int w, int prg,
                                   const pcgb_blk* const* d_roots, const pcgb_blk* const* d_cws,
                                   const uint8_t* round_keys, pcgb_blk* const* d_leaves,
                                   void* stream);


/* ---- native: batched NTT ----------------------------------------------- */
/* c[k] = a[k] * b[k] mod (X^N + 1) for k < batch (device, c may alias). */
int pcgb_poly_mul_device(uint64_t* d_c, const uint64_t* d_a, const uint64_t* d_b, int batch,
                         int N, void* stream);
/* Uneven batch: polys of different lengths in one call; d_a[i], d_b[i],
 * d_c[i] each of length N[i]; d_c[i] may alias d_a[i] or d_b[i].  When every
 * N[i] is in 2^16 .. 2^20 the whole batch runs as five launches (one per
 * pass, each CTA reading its polynomial and tile from a job table); other
 * lengths run one product at a time. */
int pcgb_poly_mul_device_multi(int count, uint64_t* const* d_c, const uint64_t* const* d_a,
                               const uint64_t* const* d_b, const int* N, void* stream);

/* ---- native: PCG-OLE expansion -------------------------------------------
 * An expander owns the resident per-shape state of one (N, c, t, w, prg)
 * shape: NTT plans, the a_i evaluation images and their pair products, the
 * gather plan and scratch.  public_a: (c-1)*N coefficients of a_1..a_{c-1}
 * (a_0 = 1).  master_key: AES tree-PRG master key (AES only, else NULL). */
typedef struct pcgb_expander pcgb_expander;
int pcgb_expander_create(pcgb_expander** e, int N, int c, int t, int w, int prg,
                         const uint64_t* public_a, const uint8_t* master_key);
int pcgb_expander_destroy(pcgb_expander* e);
/* Shape-derived sizes: K keys, levels, nk CWs per level. */
int pcgb_expander_info(const pcgb_expander* e, int* K, int* levels, int* nk, size_t* scratch_bytes);
/* An expander whose c public polynomials are all given, a_0 included
 * (public_a = a_0 .. a_{c-1}, N coefficients each), where the reference
 * fixes a_0 = 1 (pcg_ole_impl.h:455-483) and pcgb_expander_create takes
 * a_1 .. a_{c-1}.  x = sum a_i e_i and z = sum a_i a_j g_ij as before; the
 * cost is t extra products per x word.  No reference counterpart. */
int pcgb_expander_create_public_a0(pcgb_expander** e, int N, int c, int t, int w, int prg,
                                   const uint64_t* public_a, const uint8_t* master_key);
/* A shard of one expansion for multi-GPU runs (no reference counterpart):
 * the c(c+1)/2 pair blocks (i <= j) are split over `world` expanders,
 * balanced by work (off-diagonal pairs carry two blocks), and this one
 * (`rank`) evaluates, writes and transforms only its own, holding only their
 * a_i a_j images.  Its z is the partial INTT(sum over its pairs); the sum of
 * all shards' z mod p is the expansion's z (linearity), exact as a uint64
 * all-reduce for world <= 4 (4(p-1) < 2^64) followed by pcgb_reduce_mod_p.
 * Every shard's x is the full x.  rank 0 of world 1 is pcgb_expander_create. */
int pcgb_expander_create_shard(pcgb_expander** e, int N, int c, int t, int w, int prg,
                               const uint64_t* public_a, const uint8_t* master_key, int rank,
                               int world);
int pcgb_expander_shard(const pcgb_expander* e, int* rank, int* world, int* pairs_local,
                        int* pairs_total);
/* d[i] = s[i] mod p for any 64-bit words (d may equal s). */
int pcgb_reduce_mod_p(uint64_t* d, const uint64_t* s, size_t count, void* stream);
/* One party's expansion from device-resident inputs:
 *   d_roots[K], d_cws[K*levels*nk], d_cw_out[K], d_pos[c*t], d_val[c*t]
 *   -> d_x[N], d_z[N] (x = sum a_i e_i, z = sum_{i,j} a_i a_j g_ij). */
int pcgb_expand_device(pcgb_expander* e, int party, const pcgb_blk* d_roots,
                       const pcgb_blk* d_cws, const uint64_t* d_cw_out, const uint64_t* d_pos,
                       const uint64_t* d_val, uint64_t* d_x, uint64_t* d_z, void* stream);
/* Several expansions of different shapes as one batch (no reference
 * counterpart; the batching form of GPU_baseline/e2e_full_bench.cu's
 * expansion loop): request i runs expander e[i] for party[i] on the
 * device-resident inputs of pcgb_expand_device.  One launch per top-walk
 * stage and walk depth, one fused leaf launch, one x launch and three NTT
 * launches cover the whole batch.  The expanders must share w, the ChaCha8 PRG and the leaf
 * shape (leaves per thread; set with pcgb_expander_set_leaf_shape), be
 * unsharded, and have N in 2^14 .. 2^20; each request's x, z equal its
 * pcgb_expand_device outputs.  Each request's scratch comes from the
 * library's stream-ordered pool on `stream`. */
int pcgb_expand_batch_device(int count, pcgb_expander* const* e, const int* party,
                             const pcgb_blk* const* d_roots, const pcgb_blk* const* d_cws,
                             const uint64_t* const* d_cw_out, const uint64_t* const* d_pos,
                             const uint64_t* const* d_val, uint64_t* const* d_x,
                             uint64_t* const* d_z, void* stream);
/* Same with host buffers (copies in and out included). */
int pcgb_expand_host(pcgb_expander* e, int party, const pcgb_blk* roots, const pcgb_blk* cws,
                     const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val,
                     uint64_t* x, uint64_t* z);
/* pcgb_expand_host without waiting (no reference counterpart): the copies
 * and kernels are queued on one of two internal streams, alternating, with
 * the expansions themselves kept in order (they share the workspace), so one
 * expansion's host copies overlap the next one's kernels.  Host buffers must
 * stay valid until pcgb_expander_wait (pin them for real overlap).  Other
 * calls on the same expander first wait for pending asynchronous ones only
 * in pcgb_expand_host; call pcgb_expander_wait before pcgb_expand_device. */
int pcgb_expand_host_async(pcgb_expander* e, int party, const pcgb_blk* roots,
                           const pcgb_blk* cws, const uint64_t* cw_out, const uint64_t* pos,
                           const uint64_t* val, uint64_t* x, uint64_t* z);
int pcgb_expander_wait(pcgb_expander* e);
/* Only the DPF + output-layer stages: the folded, pair-merged g' buffers
 * (Q = c(c+1)/2 of N words, pair order (0,0),(0,1)..(0,c-1),(1,1),..),
 * g'_ij = g_ij + g_ji for i < j.  For parity checks and staged pipelines. */
/* Step 4 of the expansion (pcg_ole_impl.h:453-484) from output layers a
 * caller computed itself, e.g. through the interactive drop-ins in a real
 * two-party run: d_g holds the c*c folded blocks g_ij (N words each, block
 * i*c + j), d_pos/d_val this party's noise; writes x and z. */
int pcgb_expand_from_g_device(pcgb_expander* e, const uint64_t* d_g, const uint64_t* d_pos,
                              const uint64_t* d_val, uint64_t* d_x, uint64_t* d_z, void* stream);
int pcgb_expand_g_device(pcgb_expander* e, int party, const pcgb_blk* d_roots,
                         const pcgb_blk* d_cws, const uint64_t* d_cw_out, uint64_t* d_g,
                         void* stream);
/* Per-stage device timing without host synchronisation: with slots > 0 each
 * expansion records events into the next of `slots` slots (0 turns it off).
 * pcgb_expander_stage_times waits for the recorded expansions and writes
 * ms[4*i + s] for stage s of the i-th one ([0] tops, [1] leaf gather,
 * [2] x, [3] NTT products); returns how many expansions were recorded and
 * starts a new recording. */
int pcgb_expander_set_profiling(pcgb_expander* e, int slots);
int pcgb_expander_stage_times(pcgb_expander* e, float* ms, int max_expansions);
/* CUDA graph replay of pcgb_expand_device (no reference counterpart): with
 * enable != 0 the first expansion runs directly, the next is captured, and
 * repeated calls with the same pointers, party and stream replay the graph
 * with one launch; other pointers re-capture and update it.  The stream
 * must be capturable (not the legacy default stream).  Off by default. */
int pcgb_expander_set_graph(pcgb_expander* e, int enable);
/* Times the top-level walk plus the fused leaf kernel for each leaf shape
 * that fits the shape -- leaves per thread (the default and two smaller
 * powers of m; fewer leaves per thread means more threads and a deeper
 * frontier, which pays at small N) times CTA size -- on zero keys (their
 * work does not depend on key values), keeps the fastest for this expander
 * and caches it per device, shape and shard; *tpb_out gets the CTA size.
 * The workspace size (pcgb_expander_info) may change.  Synchronises the
 * library stream.  Server plans are tuned on creation. */
int pcgb_expander_autotune(pcgb_expander* e, int* tpb_out);
int pcgb_expander_leaf_shape(const pcgb_expander* e, int* tpb, int* leaves_per_thread);
/* Pins the leaf shape instead of tuning it (no reference counterpart): tpb
 * in {32, 64, 128, 256}, leaves_per_thread one of the autotuner's
 * candidates (2^(w*s) for the default s and up to two smaller), tpb x
 * leaves_per_thread <= N/t.  Drops a captured graph (the next call
 * re-captures); the workspace size may change. */
int pcgb_expander_set_leaf_shape(pcgb_expander* e, int tpb, int leaves_per_thread);

/* ---- native: consumers of the expansion -------------------------------- */
/* One party's N Beaver-triple slot shares from its two ring OLEs (x1, z1)
 * and (x2, z2) of length N (CPU_baseline/pcg_ole_2pc/triple.h:45-110):
 * party 0 uses a = x1, b = x2, party 1 a = x2, b = x1, c = a*b + z1 + z2 in
 * Z_p[X]/(X^N+1); d_a, d_b, d_c receive the forward NTTs in the reference's
 * slot order (slot k = evaluation at psi^(2k+1), CPU_baseline/ntt.h), so
 * (a0+a1)(b0+b1) = c0+c1 holds slot by slot.  Inputs any uint64. */
int pcgb_triples_device(int N, int party, const uint64_t* d_x1, const uint64_t* d_z1,
                        const uint64_t* d_x2, const uint64_t* d_z2, uint64_t* d_a, uint64_t* d_b,
                        uint64_t* d_c, void* stream);
/* *d_mismatches (device) = number of NTT slots where x0*x1 != z0+z1, i.e.
 * 0 iff the two parties' outputs satisfy the OLE relation in R_p
 * (CPU_baseline/test/pcg_ole_2pc.cpp:199-214).  No host synchronisation. */
int pcgb_verify_ole_device(int N, const uint64_t* d_x0, const uint64_t* d_z0,
                           const uint64_t* d_x1, const uint64_t* d_z1,
                           unsigned long long* d_mismatches, void* stream);
/* *d_mismatches (device) = number of slots k where (a0+a1)(b0+b1) != c0+c1. */
int pcgb_verify_triples_device(int N, const uint64_t* d_a0, const uint64_t* d_b0,
                               const uint64_t* d_c0, const uint64_t* d_a1,
                               const uint64_t* d_b1, const uint64_t* d_c1,
                               unsigned long long* d_mismatches, void* stream);

/* Seeded synthetic material: a counter-based generator of this library
 * (SplitMix64 finaliser over seed, domain and index; csrc/synth.h), since the
 * reference draws noise and public a_i from unseeded emp PRGs. */
int pcgb_noise(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val);
int pcgb_public_a(int N, int c, uint64_t a_seed, uint64_t* a);
/* Dealer on the GPU: keys for both parties of one expansion. */
int pcgb_deal_keys_device(pcgb_expander* e, uint64_t seed, pcgb_blk* d_roots0,
                          pcgb_blk* d_roots1, pcgb_blk* d_cws, uint64_t* d_cw_out,
                          void* stream);

/* ---- native: serving ------------------------------------------------------
 * Continuous batching of expansion requests of mixed (N, c, t) on one GPU:
 * requests wait in a FIFO and are admitted onto one of n_streams streams as
 * soon as a stream is free, fewer than max_in_flight requests are running and
 * the request's HBM footprint (keys, noise, outputs, expansion workspace)
 * fits mem_budget (0 = half of the free memory) next to what is in flight,
 * so their kernels overlap on the device.  Large requests (c^2 N > 2^20) run
 * one at a time.  When max_in_flight exceeds n_streams, up to 32 queued
 * small requests with N in 2^14 .. 2^20, of any shapes, are admitted
 * together onto one stream as one batch (pcgb_expand_batch_device: one
 * launch per stage for all of them).  Each request deals fresh keys and
 * noise on the GPU from its seed (w = 1, ChaCha8), expands one party against
 * the shape's resident plan (a_i images from a_seed), and reports order-
 * independent digests of x and z (pcgb_digest_device).  n_streams = 1 with
 * max_in_flight = 1 is one-request-at-a-time execution. */
typedef struct pcgb_server pcgb_server;
typedef struct pcgb_request {
    int N, c, t, party;
    uint64_t seed;
    double arrival_s; /* offset from the start of pcgb_server_run_trace */
} pcgb_request;
typedef struct pcgb_result {
    uint64_t digest_x, digest_z;
    double submit_s, start_s, done_s; /* seconds since the server started */
    int status;
    int reserved;
} pcgb_result;
int pcgb_server_create(pcgb_server** s, int n_streams, size_t mem_budget, int max_in_flight,
                       uint64_t a_seed);
/* Build (and keep resident) the plan of a shape before requests arrive. */
int pcgb_server_prepare(pcgb_server* s, int N, int c, int t);
int pcgb_server_submit(pcgb_server* s, const pcgb_request* r, uint64_t* ticket);
/* Wait for a ticket (timeout_ms < 0: no limit); PCGB_ETIMEOUT if not done. */
int pcgb_server_wait(pcgb_server* s, uint64_t ticket, pcgb_result* out, int timeout_ms);
/* Submit reqs[i] at arrival_s[i] after the call starts, then wait for all. */
int pcgb_server_run_trace(pcgb_server* s, const pcgb_request* reqs, int n, pcgb_result* out,
                          double timeout_s);
int pcgb_server_stats(pcgb_server* s, int* pending, int* in_flight, size_t* bytes_in_flight,
                      int* plans);
/* Cancels pending requests, waits up to timeout_ms for in-flight ones. */
int pcgb_server_destroy(pcgb_server* s, int timeout_ms);
/* d_out[0] = sum over i of mix64(d_v[i] ^ i*0x9e3779b97f4a7c15) mod 2^64. */
int pcgb_digest_device(const uint64_t* d_v, size_t n, uint64_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
