// One party's PCG-OLE expansion on the device (the algebra of
// CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:213-312 and :453-484):
//
//   g_ij   = output layer of the t^2 DPF keys of block (i, j), folded mod X^N+1
//   x      = sum_i a_i e_i                      (e_i the regular noise; a_0 = 1 as
//                                                the reference has it, or public)
//   z      = sum_{i,j} a_i a_j g_ij = INTT( sum_{i<=j} (a^_i a^_j) . NTT(g_ij + g_ji) )
//
// The expander keeps, per shape, the a_i coefficients (Montgomery form, for
// the sparse x product) and the c(c+1)/2 evaluation images a^_i a^_j
// (Montgomery-scaled) resident, so an expansion is four device stages:
// keyed tops -> fused leaf/convert/gather -> sparse x -> NTT multiply-
// accumulate + inverse.  Blocks (i,j) and (j,i) are merged while g is
// produced (a_i a_j = a_j a_i), so only c(c+1)/2 forward transforms run.
#include "pcgb_internal.h"

#include <array>
#include <map>
#include <mutex>
#include <tuple>

#include <algorithm>
#include <cstring>
#include <vector>

#include "field.cuh"
#include "synth.h"

namespace pcgb {

void deal_keys_launch(int N, int c, int t, int n, int w, int prg, uint64_t seed,
                      const uint32_t* d_rk, Blk* roots0, Blk* roots1, Blk* cws, uint64_t* cw_out,
                      cudaStream_t st);

namespace {

// x[p] = sum_{i>=i0,k} val_ik * a_i[p - pos_ik] with the negacyclic sign
// when p < pos_ik, plus sum_k [p == pos_0k] val_0k when a_0 = 1 (i0 = 1).
// aR holds a_i0 .. a_{c-1} times 2^64 mod p, so one Montgomery product
// gives a_i * val.
__device__ __forceinline__ void x_body(const uint64_t* __restrict__ pos,
                                       const uint64_t* __restrict__ val,
                                       const uint64_t* __restrict__ aR, int c, int t, int i0,
                                       size_t N, uint64_t* __restrict__ x, unsigned block,
                                       uint64_t* nz /* [c*t] positions then [c*t] values */) {
    const int ct = c * t;
    for (int i = threadIdx.x; i < ct; i += blockDim.x) {
        nz[i] = pos[i] % N;
        nz[ct + i] = reduce_p(val[i]);
    }
    __syncthreads();
    const size_t p = static_cast<size_t>(block) * blockDim.x + threadIdx.x;
    if (p >= N) return;
    uint64_t acc = 0;
    if (i0 == 1)
        for (int k = 0; k < t; ++k)
            if (nz[k] == p) acc = add_p(acc, nz[ct + k]);
    // The (i, k) terms as one flat run q = (i - i0) * t + k (t is a power of
    // two), eight gathers issued before their products so that eight loads
    // of the a_i rows are in flight per thread.
    const int nt = (c - i0) * t, lt = __ffs(t) - 1, q0 = i0 * t;
    const uint64_t* nv = nz + ct + q0;
    auto gather = [&](int q, bool& wrap) {
        const uint64_t ps = nz[q0 + q];
        wrap = p < ps;
        return __ldg(aR + static_cast<size_t>(q >> lt) * N + (wrap ? p + N - ps : p - ps));
    };
    int q = 0;
    for (; q + 8 <= nt; q += 8) {
        uint64_t v[8];
        bool w[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = gather(q + j, w[j]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t term = mont_mul(v[j], nv[q + j]);
            acc = w[j] ? sub_p(acc, term) : add_p(acc, term);
        }
    }
    for (; q < nt; ++q) {
        bool w;
        const uint64_t term = mont_mul(gather(q, w), nv[q]);
        acc = w ? sub_p(acc, term) : add_p(acc, term);
    }
    x[p] = acc;
}

__global__ void x_kernel(const uint64_t* __restrict__ pos, const uint64_t* __restrict__ val,
                         const uint64_t* __restrict__ aR, int c, int t, int i0, size_t N,
                         uint64_t* __restrict__ x) {
    extern __shared__ uint64_t nz[];
    x_body(pos, val, aR, c, t, i0, N, x, blockIdx.x, nz);
}

// x of several expansions in one launch: CTA b runs block b - first of the
// job whose CTA range holds b.
struct XJob {
    const uint64_t* pos;
    const uint64_t* val;
    const uint64_t* aR;
    uint64_t* x;
    size_t N;
    int c, t, i0;
    unsigned first;
};
__global__ void x_multi_kernel(const XJob* __restrict__ jobs, int njobs) {
    extern __shared__ uint64_t nz[];
    int k = 0;
    while (k + 1 < njobs && jobs[k + 1].first <= blockIdx.x) ++k;
    const XJob& J = jobs[k];
    x_body(J.pos, J.val, J.aR, J.c, J.t, J.i0, J.N, J.x, blockIdx.x - J.first, nz);
}

// Digests of several vectors in one launch: job k covers CTAs
// [k * per, (k + 1) * per); every output word must be zeroed first.
struct DigestJob {
    const uint64_t* v;
    size_t n;
    unsigned long long* out;
};
__global__ void digest_multi_kernel(const DigestJob* __restrict__ jobs, unsigned per) {
    __shared__ unsigned long long part[32];
    const DigestJob J = jobs[blockIdx.x / per];
    const unsigned b = blockIdx.x % per;
    unsigned long long acc = 0;
    for (size_t i = static_cast<size_t>(b) * blockDim.x + threadIdx.x; i < J.n;
         i += static_cast<size_t>(per) * blockDim.x)
        acc += mix64(J.v[i] ^ (i * 0x9e3779b97f4a7c15ULL));
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(J.out, s);
    }
}

// d[i] = mont(s[i], k): multiply by a constant given in Montgomery form.
// g'_q = g_ij (+ g_ji when i != j) mod p for the Q pairs i <= j, from the
// c*c per-block output-layer vectors g[(i*c + j)*N ..] (each in [0, p)).
__global__ void pair_merge_kernel(const uint64_t* __restrict__ g, int c, size_t N,
                                  uint64_t* __restrict__ gq) {
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (idx >= N) return;
    int i = 0, j = 0, k = q;
    while (k >= c - i) { k -= c - i; ++i; }
    j = i + k;
    uint64_t v = reduce_p(g[static_cast<size_t>(i * c + j) * N + idx]);
    if (i != j) v = add_p(v, reduce_p(g[static_cast<size_t>(j * c + i) * N + idx]));
    gq[static_cast<size_t>(q) * N + idx] = v;
}

__global__ void scale_kernel(uint64_t* d, const uint64_t* s, size_t n, uint64_t k) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) d[i] = mont_mul(reduce_p(s[i]), k);
}

// img = (A .* B) * R  given plain evaluations A, B (B == nullptr means 1).
__global__ void image_kernel(uint64_t* img, const uint64_t* A, const uint64_t* B, size_t n,
                             uint64_t r2, uint64_t r3) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!A) { img[i] = mont_mul(1, r2); return; }            // 1 * R (a_0 = 1 both sides)
    if (!B) { img[i] = mont_mul(A[i], r2); return; }         // A * R
    img[i] = mont_mul(mont_mul(A[i], B[i]), r3);             // A*B*R
}

__global__ void noise_kernel(uint64_t seed, int party, int ct, uint64_t bin, int t, uint64_t* pos,
                             uint64_t* val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ct) return;
    pos[i] = static_cast<uint64_t>(i % t) * bin + synth_offset(seed, party, i, bin);
    val[i] = synth_value(seed, party, i);
}

// Noise of several requests in one launch, one CTA each.
struct NoiseJob {
    uint64_t seed;
    uint64_t bin;
    uint64_t* pos;
    uint64_t* val;
    int party, ct, t;
};
__global__ void noise_multi_kernel(const NoiseJob* __restrict__ jobs) {
    const NoiseJob J = jobs[blockIdx.x];
    for (int i = threadIdx.x; i < J.ct; i += blockDim.x) {
        J.pos[i] = static_cast<uint64_t>(i % J.t) * J.bin + synth_offset(J.seed, J.party, i, J.bin);
        J.val[i] = synth_value(J.seed, J.party, i);
    }
}

// Order-independent 64-bit fingerprint of a word vector: sum (mod 2^64) of
// mix(v[i] ^ i*phi).  Used to compare outputs across runs without moving
// them to the host.
__global__ void digest_kernel(const uint64_t* __restrict__ v, size_t n, unsigned long long* out) {
    __shared__ unsigned long long part[32];
    unsigned long long acc = 0;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        acc += mix64(v[i] ^ (i * 0x9e3779b97f4a7c15ULL));
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(out, s);
    }
}

unsigned blocks_for(size_t n, int tpb) { return static_cast<unsigned>((n + tpb - 1) / tpb); }

int ilog2(uint64_t v) {
    int l = 0;
    while ((uint64_t{1} << l) < v) ++l;
    return l;
}

}  // namespace
}  // namespace pcgb

struct pcgb_expander {
    int dev = 0;
    int N = 0, c = 0, t = 0, w = 0, prg = 0, n = 0, levels = 0, nk = 0, K = 0, Q = 0;
    const pcgb::NttPlan* ntt = nullptr;
    pcgb::GatherPlan gp;
    uint64_t* d_img = nullptr;   // Q*N
    uint64_t* d_aR = nullptr;    // (c-i0)*N: a_i0 .. a_{c-1}, Montgomery form
    int i0 = 1;                  // 1: a_0 = 1 (the reference); 0: a_0 public
    pcgb::Blk* d_F = nullptr;
    pcgb::Blk* d_tops = nullptr;
    uint64_t* d_g = nullptr;     // Q*N
    uint32_t* d_rk = nullptr;    // AES sub-key schedules
    size_t scratch_bytes = 0;
    size_t own_ws_bytes = 0;     // size of d_F when allocated
    std::vector<cudaEvent_t> prof_ev;  // 5 per slot
    int prof_slots = 0, prof_used = 0;
    // CUDA graph of expand_device on the expander's own workspace.
    bool use_graph = false;
    bool graph_warm = false;
    cudaGraphExec_t graph_exec = nullptr;
    unsigned long long graph_kernels = 0;
    std::array<const void*, 7> graph_key{};
    int graph_party = -1;
    cudaStream_t graph_stream = nullptr;
    // host staging for pcgb_expand_host
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    void* d_in = nullptr;
    size_t d_in_bytes = 0;
    // pcgb_expand_host_async: two I/O slots, each with its own stream and
    // device buffers; the computes (which share the workspace) are chained
    // by `async_compute` so slot i's copies overlap slot i+1's kernels.
    struct AsyncSlot {
        cudaStream_t st = nullptr;
        void* d_io = nullptr;
        size_t bytes = 0;
    } aslot[2];
    int aturn = 0;
    cudaEvent_t async_compute = nullptr;
    bool async_pending = false;
};

namespace pcgb {

pcgb_expander* expander_create(int N, int c, int t, int w, int prg, const uint64_t* public_a,
                               const uint8_t* master_key, int rank, int world, int a0_public) {
    if (N < 4 || (N & (N - 1)) || N > (1 << kMaxLogN))
        fail(PCGB_EINVAL, "expander: N must be a power of two in [4, 2^24]");
    if (c < 1 || c > 8) fail(PCGB_EINVAL, "expander: c must be in [1, 8]");
    if (t < 1 || (t & (t - 1)) || N / t < 2) fail(PCGB_EINVAL, "expander: t must be a power of two <= N/2");
    if (prg != PCGB_PRG_AES && prg != PCGB_PRG_CHACHA8) fail(PCGB_EINVAL, "expander: unknown PRG");
    if (prg == PCGB_PRG_AES && !master_key) fail(PCGB_EINVAL, "expander: AES needs a master key");
    const int i0 = a0_public ? 0 : 1, na = c - i0;   // public polynomials given
    if (na > 0 && !public_a) fail(PCGB_EINVAL, "expander: public_a required");
    const int n = ilog2(2ull * (N / t));
    if (w < 1 || w > 4 || n % w) fail(PCGB_EINVAL, "expander: w must be in [1,4] and divide log2(2N/t)");
    auto* e = new pcgb_expander();
    try {
        PCGB_CK(cudaGetDevice(&e->dev));
        e->N = N; e->c = c; e->t = t; e->w = w; e->prg = prg; e->n = n;
        e->levels = n / w; e->nk = (1 << w) - 1; e->K = c * c * t * t; e->Q = c * (c + 1) / 2;
        e->i0 = i0;
        cudaStream_t st = default_stream();
        e->ntt = &ntt_plan(ilog2(N));
        gather_plan_build(e->gp, N, c, t, n, w, rank, world);
        const size_t NN = static_cast<size_t>(N);
        const int Qs = e->gp.Qs;
        PCGB_CK(cudaMalloc(&e->d_img, sizeof(uint64_t) * NN * std::max(Qs, 1)));
        if (na > 0) PCGB_CK(cudaMalloc(&e->d_aR, sizeof(uint64_t) * NN * na));
        // a_i coefficients (Montgomery form) and evaluations.
        std::vector<uint64_t*> ahat(c, nullptr);
        const uint64_t r2 = r2_mod_p(), r3 = mul_p_host(r2, r_mod_p());
        if (na > 0) {
            uint64_t* tmp = nullptr;
            PCGB_CK(cudaMalloc(&tmp, sizeof(uint64_t) * NN * na));
            upload_blocking(tmp, public_a, sizeof(uint64_t) * NN * na);
            reduce_mod_p(tmp, tmp, NN * na, st);
            scale_kernel<<<blocks_for(NN * na, 256), 256, 0, st>>>(e->d_aR, tmp, NN * na, r2);
            PCGB_POST_LAUNCH();
            ntt_forward(*e->ntt, tmp, na, st);
            for (int i = i0; i < c; ++i) ahat[i] = tmp + NN * (i - i0);
            // Images of this shard's pairs, in slot order (a null factor is a_0 = 1).
            for (int k = 0; k < Qs; ++k) {
                const int ij = static_cast<int>(e->gp.pair_ij[e->gp.shard_pairs[k]]);
                const uint64_t* A = ahat[ij / c];
                const uint64_t* B = ahat[ij % c];
                image_kernel<<<blocks_for(NN, 256), 256, 0, st>>>(
                    e->d_img + NN * k, A ? A : B, A ? B : nullptr, NN, r2, r3);
                PCGB_POST_LAUNCH();
            }
            PCGB_CK(cudaStreamSynchronize(st));
            cudaFree(tmp);
        } else if (Qs > 0) {
            image_kernel<<<blocks_for(NN, 256), 256, 0, st>>>(e->d_img, nullptr, nullptr, NN, r2, r3);
            PCGB_POST_LAUNCH();
        }
        if (prg == PCGB_PRG_AES) {
            std::vector<uint8_t> rks(static_cast<size_t>(e->nk) * 176);
            aes_tree_round_keys_host(master_key, e->nk, rks.data());
            e->d_rk = aes_upload_round_keys(rks.data(), e->nk, st);
        }
        e->scratch_bytes = workspace_bytes(e);  // allocated on first direct use
        PCGB_CK(cudaStreamSynchronize(st));
    } catch (...) {
        // release what was allocated, then rethrow
        gather_plan_free(e->gp);
        cudaFree(e->d_img); cudaFree(e->d_aR); cudaFree(e->d_F); cudaFree(e->d_rk);
        delete e;
        throw;
    }
    return e;
}

void expander_destroy(pcgb_expander* e) {
    if (!e) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(e->dev);
    cudaStreamSynchronize(default_stream());
    gather_plan_free(e->gp);
    cudaFree(e->d_img); cudaFree(e->d_aR); cudaFree(e->d_F); cudaFree(e->d_rk);
    cudaFree(e->d_in);
    if (e->h_stage) cudaFreeHost(e->h_stage);
    for (auto& a : e->aslot) {
        if (a.st) cudaStreamSynchronize(a.st);
        cudaFree(a.d_io);
        if (a.st) cudaStreamDestroy(a.st);
    }
    if (e->async_compute) cudaEventDestroy(e->async_compute);
    for (auto& ev : e->prof_ev) cudaEventDestroy(ev);
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    cudaSetDevice(cur);
    delete e;
}

// Scratch of one in-flight expansion: the frontier, the first-stage tops
// and the g' buffers.  An expander owns one; the server carves one per
// admitted request so expansions of the same shape can overlap.
size_t workspace_bytes(const pcgb_expander* e) {
    const size_t fnodes = static_cast<size_t>(e->K) << (e->w * e->gp.hl);
    const size_t tnodes = keyed_tops_scratch_nodes(e->K, e->w, e->gp.hl);
    return sizeof(Blk) * (fnodes + tnodes) +
           sizeof(uint64_t) * static_cast<size_t>(e->N) * std::max(e->gp.Qs, 1);
}

Workspace workspace_carve(const pcgb_expander* e, void* base) {
    const size_t fnodes = static_cast<size_t>(e->K) << (e->w * e->gp.hl);
    const size_t tnodes = keyed_tops_scratch_nodes(e->K, e->w, e->gp.hl);
    Workspace ws;
    ws.F = static_cast<Blk*>(base);
    ws.tops = tnodes ? ws.F + fnodes : nullptr;
    ws.g = reinterpret_cast<uint64_t*>(ws.F + fnodes + tnodes);
    return ws;
}

void expand_device_ws(pcgb_expander* e, const Workspace& ws, int party, const Blk* roots,
                      const Blk* cws, const uint64_t* cw_out, const uint64_t* pos,
                      const uint64_t* val, uint64_t* x, uint64_t* z, cudaStream_t st) {
    if (party != 0 && party != 1) fail(PCGB_EINVAL, "expand: party must be 0 or 1");
    if (!roots || !cws || !cw_out || !pos || !val || !x || !z) fail(PCGB_EINVAL, "expand: null pointer");
    const size_t NN = static_cast<size_t>(e->N);
    cudaEvent_t* ev = nullptr;
    if (e->prof_slots > 0 && e->prof_used < e->prof_slots) ev = &e->prof_ev[5 * e->prof_used++];
    if (ev) PCGB_CK(cudaEventRecord(ev[0], st));
    keyed_expand_tops(e->K, e->n, e->w, e->prg, roots, cws, e->d_rk, e->gp.hl, ws.F, ws.tops, st);
    if (ev) PCGB_CK(cudaEventRecord(ev[1], st));
    keyed_leaf_gather(e->gp, party, e->prg, ws.F, cws, cw_out, e->d_rk, ws.g, st);
    if (ev) PCGB_CK(cudaEventRecord(ev[2], st));
    const size_t sm = sizeof(uint64_t) * 2 * static_cast<size_t>(e->c) * e->t;
    x_kernel<<<blocks_for(NN, 256), 256, sm, st>>>(pos, val, e->d_aR, e->c, e->t, e->i0, NN, x);
    PCGB_POST_LAUNCH();
    if (ev) PCGB_CK(cudaEventRecord(ev[3], st));
    if (e->gp.Qs > 0) ntt_mac_inverse(*e->ntt, ws.g, e->d_img, e->gp.Qs, z, st);
    else PCGB_CK(cudaMemsetAsync(z, 0, sizeof(uint64_t) * NN, st));   // a shard with no pairs
    if (ev) PCGB_CK(cudaEventRecord(ev[4], st));
}

// Expansions of different shapes as one batch (ChaCha8, one w and one leaf
// depth sl for all): one launch per top-walk stage, one fused leaf launch,
// one x launch and three NTT launches for the whole batch, each CTA finding
// its expansion in a job table.  Outputs equal expand_device_ws's, request by
// request.  All job tables travel in one copy from pinned or pageable host
// memory on `st`.
void expand_batch_ws(int count, pcgb_expander* const* e, const Workspace* ws, const int* party,
                     const Blk* const* roots, const Blk* const* cws,
                     const uint64_t* const* cw_out, const uint64_t* const* pos,
                     const uint64_t* const* val, uint64_t* const* x, uint64_t* const* z,
                     cudaStream_t st) {
    if (count <= 0) return;
    const int w = e[0]->w, sl = e[0]->gp.sl, S = e[0]->gp.S;
    for (int i = 0; i < count; ++i) {
        const pcgb_expander* E = e[i];
        if (!E || !ws[i].F || !ws[i].g) fail(PCGB_EINVAL, "expand batch: null expander or workspace");
        if (E->prg != PCGB_PRG_CHACHA8) fail(PCGB_EINVAL, "expand batch: ChaCha8 expanders only");
        if (E->w != w || E->gp.sl != sl)
            fail(PCGB_EINVAL, "expand batch: every expander needs the same w and leaf shape");
        if (E->gp.world != 1) fail(PCGB_EINVAL, "expand batch: sharded expanders are not batched");
        if (!ntt_mac_multi_ok(ilog2(E->N))) fail(PCGB_EINVAL, "expand batch: N must be 2^14 .. 2^20");
        if (party[i] != 0 && party[i] != 1) fail(PCGB_EINVAL, "expand: party must be 0 or 1");
        if (!roots[i] || !cws[i] || !cw_out[i] || !pos[i] || !val[i] || !x[i] || !z[i])
            fail(PCGB_EINVAL, "expand: null pointer");
    }
    // Stage 1: the top-level walks, each to its expander's frontier level.
    {
        std::vector<int> K(count), n(count), hl(count);
        std::vector<const Blk*> r(count), c(count);
        std::vector<Blk*> out(count), scr(count);
        for (int i = 0; i < count; ++i) {
            K[i] = e[i]->K; n[i] = e[i]->n; hl[i] = e[i]->gp.hl;
            r[i] = roots[i];
            c[i] = cws[i]; out[i] = ws[i].F; scr[i] = ws[i].tops;
        }
        keyed_tops_multi(count, K.data(), n.data(), hl.data(), w, PCGB_PRG_CHACHA8, r.data(),
                         c.data(), nullptr, out.data(), scr.data(), st);
    }
    // Job tables of the leaf and x launches.
    int tpb = 256;
    for (int i = 0; i < count; ++i) {
        const size_t bin = static_cast<size_t>(e[i]->N) / e[i]->t;
        int tp = e[i]->gp.tpb > 0 ? e[i]->gp.tpb : 256;
        while (tp > 1 && static_cast<size_t>(tp) * S > bin) tp >>= 1;
        if (static_cast<size_t>(tp) * S > bin) fail(PCGB_EINVAL, "bin smaller than one tile");
        tpb = std::min(tpb, tp);
    }
    std::vector<LeafJob> leaf(count);
    std::vector<XJob> xj(count);
    unsigned leaf_ctas = 0, x_ctas = 0;
    size_t x_smem = 0;
    for (int i = 0; i < count; ++i) {
        const pcgb_expander* E = e[i];
        LeafJob& L = leaf[i];
        L.F = ws[i].F; L.cws = cws[i]; L.cw_out = cw_out[i];
        L.off = E->gp.d_off; L.entries = E->gp.d_entries;
        L.q_order = E->gp.d_qorder; L.q_slot = E->gp.d_qslot; L.gq = ws[i].g;
        L.bin = static_cast<size_t>(E->N) / E->t;
        L.t = E->t; L.levels = E->levels; L.hl = E->gp.hl; L.N = E->N; L.party = party[i];
        L.gx = static_cast<unsigned>(L.bin / (static_cast<size_t>(tpb) * S));
        L.gy = static_cast<unsigned>(E->t);
        L.first = leaf_ctas;
        leaf_ctas += L.gx * L.gy * static_cast<unsigned>(E->gp.Qs);
        XJob& X = xj[i];
        X.pos = pos[i]; X.val = val[i]; X.aR = E->d_aR; X.x = x[i];
        X.N = static_cast<size_t>(E->N); X.c = E->c; X.t = E->t; X.i0 = E->i0;
        X.first = x_ctas;
        x_ctas += blocks_for(X.N, 256);
        x_smem = std::max(x_smem, sizeof(uint64_t) * 2 * static_cast<size_t>(E->c) * E->t);
    }
    const size_t b_leaf = sizeof(LeafJob) * count;
    const size_t o_x = (b_leaf + 255) & ~size_t{255};
    const size_t total = o_x + sizeof(XJob) * count;
    std::vector<char> host(total);
    std::memcpy(host.data(), leaf.data(), b_leaf);
    std::memcpy(host.data() + o_x, xj.data(), sizeof(XJob) * count);
    char* tab = static_cast<char*>(pool_alloc(total, st));
    PCGB_CK(cudaMemcpyAsync(tab, host.data(), total, cudaMemcpyHostToDevice, st));
    // Stage 2: the fused leaf kernel over every expansion's tiles.
    const size_t leaf_smem = static_cast<size_t>(tpb) * (S + 1) * 2 * sizeof(uint64_t);
    keyed_leaf_multi_chacha(w, sl, reinterpret_cast<const LeafJob*>(tab), count, leaf_ctas, tpb,
                            leaf_smem, nullptr, nullptr, st);
    // Stage 3: the sparse x products.
    x_multi_kernel<<<x_ctas, 256, x_smem, st>>>(reinterpret_cast<const XJob*>(tab + o_x), count);
    PCGB_POST_LAUNCH();
    // Stage 4: NTT multiply-accumulate and inverse, all lengths at once.
    std::vector<uint64_t*> g(count), zz(count);
    std::vector<const uint64_t*> img(count);
    std::vector<int> Q(count), lg(count);
    for (int i = 0; i < count; ++i) {
        g[i] = ws[i].g; img[i] = e[i]->d_img; Q[i] = e[i]->gp.Qs; zz[i] = z[i];
        lg[i] = ilog2(e[i]->N);
    }
    ntt_mac_inverse_multi(count, g.data(), img.data(), Q.data(), zz.data(), lg.data(), st);
    PCGB_CK(cudaFreeAsync(tab, st));
}

// Keys and noise of several requests (ChaCha8 expanders of one w), one
// dealer launch and one noise launch for all: request i gets
// deal_keys_device(e[i], seed[i], ...) and noise_device(..., party[i], ...).
void deal_noise_multi_device(int count, pcgb_expander* const* e, const uint64_t* seed,
                             const int* party, Blk* const* r0, Blk* const* r1, Blk* const* cws,
                             uint64_t* const* cwo, uint64_t* const* pos, uint64_t* const* val,
                             cudaStream_t st) {
    if (count <= 0) return;
    const int w = e[0]->w;
    std::vector<DealJob> deal(count);
    std::vector<NoiseJob> noise(count);
    unsigned ctas = 0;
    for (int i = 0; i < count; ++i) {
        const pcgb_expander* E = e[i];
        if (E->prg != PCGB_PRG_CHACHA8 || E->w != w)
            fail(PCGB_EINVAL, "deal batch: ChaCha8 expanders of one w only");
        const uint64_t bin = static_cast<uint64_t>(E->N / E->t);
        deal[i] = DealJob{seed[i], r0[i], r1[i], cws[i], cwo[i], bin, E->c, E->t, E->n, ctas};
        ctas += static_cast<unsigned>((E->K + 127) / 128);
        noise[i] = NoiseJob{seed[i], bin, pos[i], val[i], party[i], E->c * E->t, E->t};
    }
    const size_t b_deal = sizeof(DealJob) * count;
    const size_t o_noise = (b_deal + 255) & ~size_t{255};
    const size_t total = o_noise + sizeof(NoiseJob) * count;
    std::vector<char> host(total);
    std::memcpy(host.data(), deal.data(), b_deal);
    std::memcpy(host.data() + o_noise, noise.data(), sizeof(NoiseJob) * count);
    char* tab = static_cast<char*>(pool_alloc(total, st));
    PCGB_CK(cudaMemcpyAsync(tab, host.data(), total, cudaMemcpyHostToDevice, st));
    deal_multi_chacha_launch(w, reinterpret_cast<const DealJob*>(tab), count, ctas, r2_mod_p(), st);
    noise_multi_kernel<<<count, 128, 0, st>>>(reinterpret_cast<const NoiseJob*>(tab + o_noise));
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(tab, st));
}

// out[i] (device words, zeroed here) = digest of v[i][0 .. n[i]), one launch.
void digest_multi_device(int count, const uint64_t* const* v, const size_t* n, uint64_t* const* out,
                         cudaStream_t st) {
    if (count <= 0) return;
    std::vector<DigestJob> jobs(count);
    size_t longest = 1;
    for (int i = 0; i < count; ++i) {
        jobs[i] = DigestJob{v[i], n[i], reinterpret_cast<unsigned long long*>(out[i])};
        longest = std::max(longest, n[i]);
    }
    const unsigned per = static_cast<unsigned>(std::min<size_t>((longest + 255) / 256, 256));
    DigestJob* d = static_cast<DigestJob*>(pool_alloc(sizeof(DigestJob) * count, st));
    PCGB_CK(cudaMemcpyAsync(d, jobs.data(), sizeof(DigestJob) * count, cudaMemcpyHostToDevice, st));
    for (int i = 0; i < count; ++i) PCGB_CK(cudaMemsetAsync(out[i], 0, sizeof(uint64_t), st));
    digest_multi_kernel<<<per * static_cast<unsigned>(count), 256, 0, st>>>(d, per);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(d, st));
}

// The expander's own workspace, allocated on first use (plans held by the
// server never need it: requests bring their own).
void ensure_own_workspace(pcgb_expander* e) {
    if (e->d_F && e->own_ws_bytes >= e->scratch_bytes) return;
    if (e->d_F) {
        // Regrow (the leaf shape changed): drain uses of the old one first;
        // a captured graph refers to it, so drop the graph too.
        PCGB_CK(cudaDeviceSynchronize());
        cudaFree(e->d_F);
        e->d_F = nullptr;
        if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
        e->graph_exec = nullptr;
        e->graph_warm = false;
    }
    PCGB_CK(cudaMalloc(&e->d_F, e->scratch_bytes));
    e->own_ws_bytes = e->scratch_bytes;
    const Workspace ws = workspace_carve(e, e->d_F);
    e->d_tops = ws.tops;
    e->d_g = ws.g;
}

// With graphs on, the first call runs directly (plans, tables and kernel
// attributes are set up lazily there), the second captures the launch
// sequence into a CUDA graph, and later calls with the same pointers, party
// and stream replay it with one cudaGraphLaunch.  New pointers re-capture
// and update the executable graph in place.  Profiling slots bypass graphs.
void expand_device(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                   const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val, uint64_t* x,
                   uint64_t* z, cudaStream_t st) {
    ensure_own_workspace(e);
    Workspace ws;
    ws.F = e->d_F;
    ws.tops = e->d_tops;
    ws.g = e->d_g;
    const bool profiling = e->prof_slots > 0 && e->prof_used < e->prof_slots;
    if (!e->use_graph || profiling || !e->graph_warm) {
        expand_device_ws(e, ws, party, roots, cws, cw_out, pos, val, x, z, st);
        e->graph_warm = true;
        return;
    }
    const std::array<const void*, 7> key{roots, cws, cw_out, pos, val, x, z};
    if (e->graph_exec && key == e->graph_key && party == e->graph_party && st == e->graph_stream) {
        PCGB_CK(cudaGraphLaunch(e->graph_exec, st));
        note_launches(e->graph_kernels);
        return;
    }
    cudaGraph_t graph = nullptr;
    PCGB_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
        expand_device_ws(e, ws, party, roots, cws, cw_out, pos, val, x, z, st);
    } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    PCGB_CK(cudaStreamEndCapture(st, &graph));
    size_t n_nodes = 0;
    PCGB_CK(cudaGraphGetNodes(graph, nullptr, &n_nodes));
    std::vector<cudaGraphNode_t> nodes(n_nodes);
    PCGB_CK(cudaGraphGetNodes(graph, nodes.data(), &n_nodes));
    unsigned long long kernels = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        PCGB_CK(cudaGraphNodeGetType(nd, &ty));
        if (ty == cudaGraphNodeTypeKernel) ++kernels;
    }
    if (e->graph_exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(e->graph_exec, graph, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(e->graph_exec);
            e->graph_exec = nullptr;
        }
    }
    if (!e->graph_exec) {
        const cudaError_t rc = cudaGraphInstantiate(&e->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        PCGB_CK(rc);
    } else {
        cudaGraphDestroy(graph);
    }
    e->graph_key = key;
    e->graph_party = party;
    e->graph_stream = st;
    e->graph_kernels = kernels;
    // The captured launches were counted once as they were recorded; this
    // launch is their one execution.
    PCGB_CK(cudaGraphLaunch(e->graph_exec, st));
}

void expander_set_graph(pcgb_expander* e, bool on) {
    if (!on && e->graph_exec) {
        PCGB_CK(cudaStreamSynchronize(e->graph_stream ? e->graph_stream : default_stream()));
        cudaGraphExecDestroy(e->graph_exec);
        e->graph_exec = nullptr;
    }
    e->use_graph = on;
}

// Leaf-kernel shape for this expander: leaves per thread (S = m^sl; fewer
// means more threads, shorter serial walks and a deeper frontier, which
// pays at small shapes) and CTA size.  Each candidate runs the top-level
// walk and the leaf kernel on zero keys (their work does not depend on key
// values); the fastest is kept and cached per device, shape and shard.
// Changing sl changes the frontier level, so the workspace size is
// recomputed (and an expander's own workspace regrown on next use).
namespace {
void set_leaf_sl(pcgb_expander* e, int sl) {
    e->gp.sl = sl;
    e->gp.S = 1 << (e->w * sl);
    e->gp.hl = e->levels - sl;
}
}  // namespace

int expander_autotune(pcgb_expander* e) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int, int>, std::pair<int, int>> cache;
    const auto key = std::make_tuple(e->dev, e->N, e->c, e->t, e->w, e->prg,
                                     e->gp.world * 64 + e->gp.rank);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            set_leaf_sl(e, it->second.first);
            e->gp.tpb = it->second.second;
            e->scratch_bytes = workspace_bytes(e);
            return e->gp.tpb;
        }
    }
    // Candidate leaves-per-thread exponents: the default and up to two
    // smaller, as long as the walk below the frontier keeps >= 1 level.
    const int sl0 = e->gp.sl;
    std::vector<int> sls;
    for (int sl = sl0; sl >= 1 && sl >= sl0 - 2; --sl) sls.push_back(sl);
    size_t ws_max = 0;
    for (int sl : sls) {
        set_leaf_sl(e, sl);
        ws_max = std::max(ws_max, workspace_bytes(e));
    }
    cudaStream_t st = default_stream();
    const size_t K = e->K;
    const size_t b_roots = K * sizeof(Blk), b_cws = K * e->levels * e->nk * sizeof(Blk);
    const size_t b_keys = (b_roots + b_cws + 8 * K + 255) & ~static_cast<size_t>(255);
    // A scratch workspace from the pool (server plans own none).
    char* d = static_cast<char*>(pool_alloc(b_keys + ws_max, st));
    PCGB_CK(cudaMemsetAsync(d, 0, b_roots + b_cws + 8 * K, st));
    const Blk* roots = reinterpret_cast<const Blk*>(d);
    const Blk* cws = reinterpret_cast<const Blk*>(d + b_roots);
    const uint64_t* cwo = reinterpret_cast<const uint64_t*>(d + b_roots + b_cws);
    const size_t bin = static_cast<size_t>(e->N) / e->t;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PCGB_CK(cudaEventCreate(&e0));
    PCGB_CK(cudaEventCreate(&e1));
    int best_sl = sl0, best_tpb = 0;
    float best_ms = 0;
    try {
        for (int sl : sls) {
            set_leaf_sl(e, sl);
            const Workspace ws = workspace_carve(e, d + b_keys);
            for (int tpb : {256, 128, 64, 32}) {
                if (static_cast<size_t>(tpb) * e->gp.S > bin) continue;
                e->gp.tpb = tpb;
                auto run = [&] {
                    keyed_expand_tops(e->K, e->n, e->w, e->prg, roots, cws, e->d_rk, e->gp.hl,
                                      ws.F, ws.tops, st);
                    keyed_leaf_gather(e->gp, 0, e->prg, ws.F, cws, cwo, e->d_rk, ws.g, st);
                };
                run();   // warm
                float ms = 0;
                for (int rep = 0; rep < 3; ++rep) {
                    PCGB_CK(cudaEventRecord(e0, st));
                    run();
                    PCGB_CK(cudaEventRecord(e1, st));
                    PCGB_CK(cudaEventSynchronize(e1));
                    float t = 0;
                    PCGB_CK(cudaEventElapsedTime(&t, e0, e1));
                    ms = rep == 0 ? t : std::min(ms, t);
                }
                if (best_tpb == 0 || ms < best_ms) { best_sl = sl; best_tpb = tpb; best_ms = ms; }
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFreeAsync(d, st);
        set_leaf_sl(e, sl0);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PCGB_CK(cudaFreeAsync(d, st));
    PCGB_CK(cudaStreamSynchronize(st));
    if (best_tpb == 0) best_tpb = 32;
    set_leaf_sl(e, best_sl);
    e->gp.tpb = best_tpb;
    e->scratch_bytes = workspace_bytes(e);
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {best_sl, best_tpb};
    return best_tpb;
}

void expander_set_leaf_shape(pcgb_expander* e, int tpb, int leaves_per_thread) {
    const int sl_max = leaf_sl_max(e->n, e->w);
    int sl = 0;
    for (int k = 1; k <= sl_max; ++k)
        if (leaves_per_thread == (1 << (e->w * k))) sl = k;
    const size_t bin = static_cast<size_t>(e->N) / e->t;
    if (sl == 0 || sl < sl_max - 2)
        fail(PCGB_EINVAL, "set_leaf_shape: leaves per thread must be m^s for one of the "
                          "autotuner's candidates s in [max(1, s_max - 2), s_max]");
    if (tpb != 32 && tpb != 64 && tpb != 128 && tpb != 256)
        fail(PCGB_EINVAL, "set_leaf_shape: CTA size must be 32, 64, 128 or 256");
    if (static_cast<size_t>(tpb) * leaves_per_thread > bin)
        fail(PCGB_EINVAL, "set_leaf_shape: CTA size x leaves per thread exceeds the bin N/t");
    const bool graph = e->use_graph;
    expander_set_graph(e, false);   // a captured graph replays the old shape
    set_leaf_sl(e, sl);
    e->gp.tpb = tpb;
    e->scratch_bytes = workspace_bytes(e);
    e->use_graph = graph;
}

void expander_leaf_shape(const pcgb_expander* e, int* tpb, int* leaves_per_thread) {
    if (tpb) *tpb = e->gp.tpb > 0 ? e->gp.tpb : 256;
    if (leaves_per_thread) *leaves_per_thread = e->gp.S;
}

void expander_wait(pcgb_expander* e) {
    for (auto& a : e->aslot)
        if (a.st) PCGB_CK(cudaStreamSynchronize(a.st));
    e->async_pending = false;
}

// One expansion from host inputs to host outputs without waiting for it.
// Host buffers must stay valid (and, for overlap, be pinned) until
// expander_wait.  Slot k's stream runs H2D -> (wait for the previous
// compute) -> kernels -> D2H, alternating k = 0, 1.
void expand_host_async(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                       const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val,
                       uint64_t* x, uint64_t* z) {
    if (!roots || !cws || !cw_out || !pos || !val || !x || !z)
        fail(PCGB_EINVAL, "expand_host_async: null pointer");
    const size_t K = e->K, ct = static_cast<size_t>(e->c) * e->t, NN = e->N;
    const size_t b_roots = K * sizeof(Blk), b_cws = K * e->levels * e->nk * sizeof(Blk);
    const size_t b_cwo = K * 8, b_noise = ct * 8, b_out = NN * 8;
    const size_t in_bytes = b_roots + b_cws + b_cwo + 2 * b_noise;
    const size_t dev_bytes = in_bytes + 2 * b_out;
    if (!e->async_compute) PCGB_CK(cudaEventCreateWithFlags(&e->async_compute, cudaEventDisableTiming));
    ensure_own_workspace(e);
    auto& a = e->aslot[e->aturn];
    e->aturn ^= 1;
    if (!a.st) PCGB_CK(cudaStreamCreateWithFlags(&a.st, cudaStreamNonBlocking));
    if (dev_bytes > a.bytes) {
        PCGB_CK(cudaStreamSynchronize(a.st));
        cudaFree(a.d_io);
        a.d_io = nullptr;
        PCGB_CK(cudaMalloc(&a.d_io, dev_bytes));
        a.bytes = dev_bytes;
    }
    char* d = static_cast<char*>(a.d_io);
    Blk* d_roots = reinterpret_cast<Blk*>(d);
    Blk* d_cws = reinterpret_cast<Blk*>(d + b_roots);
    uint64_t* d_cwo = reinterpret_cast<uint64_t*>(d + b_roots + b_cws);
    uint64_t* d_pos = reinterpret_cast<uint64_t*>(d + b_roots + b_cws + b_cwo);
    uint64_t* d_val = d_pos + ct;
    uint64_t* d_x = reinterpret_cast<uint64_t*>(d + in_bytes);
    uint64_t* d_z = d_x + NN;
    PCGB_CK(cudaMemcpyAsync(d_roots, roots, b_roots, cudaMemcpyHostToDevice, a.st));
    PCGB_CK(cudaMemcpyAsync(d_cws, cws, b_cws, cudaMemcpyHostToDevice, a.st));
    PCGB_CK(cudaMemcpyAsync(d_cwo, cw_out, b_cwo, cudaMemcpyHostToDevice, a.st));
    PCGB_CK(cudaMemcpyAsync(d_pos, pos, b_noise, cudaMemcpyHostToDevice, a.st));
    PCGB_CK(cudaMemcpyAsync(d_val, val, b_noise, cudaMemcpyHostToDevice, a.st));
    if (e->async_pending) PCGB_CK(cudaStreamWaitEvent(a.st, e->async_compute, 0));
    Workspace ws;
    ws.F = e->d_F;
    ws.tops = e->d_tops;
    ws.g = e->d_g;
    expand_device_ws(e, ws, party, d_roots, d_cws, d_cwo, d_pos, d_val, d_x, d_z, a.st);
    PCGB_CK(cudaEventRecord(e->async_compute, a.st));
    e->async_pending = true;
    PCGB_CK(cudaMemcpyAsync(x, d_x, b_out, cudaMemcpyDeviceToHost, a.st));
    PCGB_CK(cudaMemcpyAsync(z, d_z, b_out, cudaMemcpyDeviceToHost, a.st));
}

void expand_host(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                 const uint64_t* cw_out, const uint64_t* pos, const uint64_t* val, uint64_t* x,
                 uint64_t* z) {
    if (e->async_pending) expander_wait(e);
    cudaStream_t st = default_stream();
    const size_t K = e->K, ct = static_cast<size_t>(e->c) * e->t, NN = e->N;
    const size_t b_roots = K * sizeof(Blk), b_cws = K * e->levels * e->nk * sizeof(Blk);
    const size_t b_cwo = K * 8, b_noise = ct * 8, b_out = NN * 8;
    const size_t in_bytes = b_roots + b_cws + b_cwo + 2 * b_noise;
    const size_t dev_bytes = in_bytes + 2 * b_out;
    if (dev_bytes > e->d_in_bytes) {
        cudaFree(e->d_in);
        e->d_in = nullptr;
        PCGB_CK(cudaMalloc(&e->d_in, dev_bytes));
        e->d_in_bytes = dev_bytes;
    }
    char* d = static_cast<char*>(e->d_in);
    Blk* d_roots = reinterpret_cast<Blk*>(d);
    Blk* d_cws = reinterpret_cast<Blk*>(d + b_roots);
    uint64_t* d_cwo = reinterpret_cast<uint64_t*>(d + b_roots + b_cws);
    uint64_t* d_pos = reinterpret_cast<uint64_t*>(d + b_roots + b_cws + b_cwo);
    uint64_t* d_val = d_pos + ct;
    uint64_t* d_x = reinterpret_cast<uint64_t*>(d + in_bytes);
    uint64_t* d_z = d_x + NN;
    PCGB_CK(cudaMemcpyAsync(d_roots, roots, b_roots, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_cws, cws, b_cws, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_cwo, cw_out, b_cwo, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_pos, pos, b_noise, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_val, val, b_noise, cudaMemcpyHostToDevice, st));
    expand_device(e, party, d_roots, d_cws, d_cwo, d_pos, d_val, d_x, d_z, st);
    PCGB_CK(cudaMemcpyAsync(x, d_x, b_out, cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaMemcpyAsync(z, d_z, b_out, cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

// Step 4 from externally computed output layers (the interactive two-party
// path): g holds the c*c folded blocks g_ij (pcg_ole_impl.h:453-484 reads
// them the same way), pos/val this party's noise.
void expand_from_g_device(pcgb_expander* e, const uint64_t* g, const uint64_t* pos,
                          const uint64_t* val, uint64_t* x, uint64_t* z, cudaStream_t st) {
    if (!g || !pos || !val || !x || !z) fail(PCGB_EINVAL, "expand_from_g: null pointer");
    if (e->gp.world != 1) fail(PCGB_EINVAL, "expand_from_g: needs an unsharded expander");
    ensure_own_workspace(e);
    const size_t NN = static_cast<size_t>(e->N);
    pair_merge_kernel<<<dim3(blocks_for(NN, 256), e->Q), 256, 0, st>>>(g, e->c, NN, e->d_g);
    PCGB_POST_LAUNCH();
    const size_t sm = sizeof(uint64_t) * 2 * static_cast<size_t>(e->c) * e->t;
    x_kernel<<<blocks_for(NN, 256), 256, sm, st>>>(pos, val, e->d_aR, e->c, e->t, e->i0, NN, x);
    PCGB_POST_LAUNCH();
    ntt_mac_inverse(*e->ntt, e->d_g, e->d_img, e->Q, z, st);
}

void expand_g_device(pcgb_expander* e, int party, const Blk* roots, const Blk* cws,
                     const uint64_t* cw_out, uint64_t* d_g, cudaStream_t st) {
    if (!roots || !cws || !cw_out || !d_g) fail(PCGB_EINVAL, "expand_g: null pointer");
    ensure_own_workspace(e);
    keyed_expand_tops(e->K, e->n, e->w, e->prg, roots, cws, e->d_rk, e->gp.hl, e->d_F, e->d_tops, st);
    keyed_leaf_gather(e->gp, party, e->prg, e->d_F, cws, cw_out, e->d_rk, d_g, st);
}

// out (device, one word) = digest of d[0..n); accumulates, so zero it first.
void digest_device(const uint64_t* d, size_t n, uint64_t* out, cudaStream_t st) {
    PCGB_CK(cudaMemsetAsync(out, 0, sizeof(uint64_t), st));
    const unsigned grid = static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 1024));
    digest_kernel<<<grid, 256, 0, st>>>(d, n, reinterpret_cast<unsigned long long*>(out));
    PCGB_POST_LAUNCH();
}

void noise_device(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val,
                  cudaStream_t st) {
    const int ct = c * t;
    noise_kernel<<<(ct + 127) / 128, 128, 0, st>>>(seed, party, ct, static_cast<uint64_t>(N / t), t,
                                                    pos, val);
    PCGB_POST_LAUNCH();
}

void noise_host(int N, int c, int t, uint64_t seed, int party, uint64_t* pos, uint64_t* val) {
    const uint64_t bin = static_cast<uint64_t>(N / t);
    for (int i = 0; i < c * t; ++i) {
        pos[i] = static_cast<uint64_t>(i % t) * bin + synth_offset(seed, party, i, bin);
        val[i] = synth_value(seed, party, i);
    }
}

void public_a_host(int N, int c, uint64_t a_seed, uint64_t* a) {
    for (int i = 1; i < c; ++i)
        for (int j = 0; j < N; ++j)
            a[static_cast<size_t>(i - 1) * N + j] = synth_rnd(a_seed, kDomA + i, j) % kPm;
}

void deal_keys_device(pcgb_expander* e, uint64_t seed, Blk* r0, Blk* r1, Blk* cws, uint64_t* cwo,
                      cudaStream_t st) {
    deal_keys_launch(e->N, e->c, e->t, e->n, e->w, e->prg, seed, e->d_rk, r0, r1, cws, cwo, st);
}

}  // namespace pcgb

namespace pcgb {

void expander_shard(const pcgb_expander* e, int* rank, int* world, int* q_local, int* q_total) {
    if (rank) *rank = e->gp.rank;
    if (world) *world = e->gp.world;
    if (q_local) *q_local = e->gp.Qs;
    if (q_total) *q_total = e->Q;
}

void expander_info(const pcgb_expander* e, int* K, int* levels, int* nk, size_t* scratch) {
    if (K) *K = e->K;
    if (levels) *levels = e->levels;
    if (nk) *nk = e->nk;
    if (scratch) *scratch = e->scratch_bytes;
}

void expander_set_profiling(pcgb_expander* e, int slots) {
    if (slots < 0) fail(PCGB_EINVAL, "profiling slots must be >= 0");
    for (auto& ev : e->prof_ev) cudaEventDestroy(ev);
    e->prof_ev.assign(static_cast<size_t>(slots) * 5, nullptr);
    for (auto& ev : e->prof_ev) PCGB_CK(cudaEventCreate(&ev));
    e->prof_slots = slots;
    e->prof_used = 0;
}

int expander_stage_times(pcgb_expander* e, float* ms, int max_exp) {
    const int n = std::min(e->prof_used, max_exp);
    for (int i = 0; i < n; ++i) {
        cudaEvent_t* ev = &e->prof_ev[5 * i];
        PCGB_CK(cudaEventSynchronize(ev[4]));
        for (int s = 0; s < 4; ++s) PCGB_CK(cudaEventElapsedTime(&ms[4 * i + s], ev[s], ev[s + 1]));
    }
    const int used = e->prof_used;
    e->prof_used = 0;
    return std::min(used, max_exp);
}

}  // namespace pcgb
