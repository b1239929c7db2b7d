// Interactive half-tree DPF full-domain evaluation: the drop-in for
// pcg_cuda::dpf_gpu_batch_full_eval[_device] (GPU_baseline/common/dpf_gpu.h:55-75).
//
// Protocol per level i (half_tree_dpf/dpf.cpp:504-575): every party hashes
// its whole level-i frontier, XOR-reduces each hash column into its CW share
// (seeded with the DltSft share), exchanges the shares with the peer, and
// expands every node with CW = mine ^ peer.  The per-level global reduction
// is a real barrier, so the frontier is materialised level by level; what
// changes from the reference's hash/expand kernel pair (dpf_gpu.cu:212-330):
//   * one kernel per level: expand level i with its CW, write the children,
//     hash the children and XOR-reduce their columns for level i+1 (the
//     reference re-reads every node and hash in separate kernels);
//   * warp-shuffle reductions with one atomicXor per CTA and column;
//   * the per-level host round trip uses pinned buffers on the library's
//     stream (one synchronisation per level, before the callback).
// Leaves come out in the reference layout: instance b, leaf d at [b*D + d].
#include "pcgb_internal.h"

#include <algorithm>
#include <mutex>
#include <vector>

#include "aes128.cuh"
#include "chacha8.cuh"
#include "field.cuh"

namespace pcgb {

void aes_ecb_encrypt_device(const uint8_t* keys, const uint8_t* in, uint8_t* out, int count);

namespace {

constexpr int kTPB = 128;

// The compact four-table AES for the shallow levels: these kernels run one
// short pass per node, so staging a bank-conflict-free table would cost as
// much as the conflicts it removes.
struct AesSm {
    uint32_t te[1024];
    uint32_t rk[15 * 44];
};
// Levels with at least this many parents per instance hash with the
// PRMT-addressed table instead (expand_level_prmt_kernel).
constexpr size_t kRepMinParents = 4096;

// H_0..H_{nk-1} of one node.
template <int W, int PRG>
__device__ __forceinline__ void hash_node(const Blk& p, const AesSm* aes, Blk (&h)[(1 << W) - 1]) {
    constexpr int NK = (1 << W) - 1;
    if constexpr (PRG == PCGB_PRG_CHACHA8) {
#pragma unroll
        for (int b = 0; b < (NK + 3) / 4; ++b) {
            uint32_t o[16];
            tree_block(p.lo, p.hi, b, o);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int k = 4 * b + c;
                if (k < NK)
                    h[k] = Blk{o[4 * c] | (static_cast<uint64_t>(o[4 * c + 1]) << 32),
                               o[4 * c + 2] | (static_cast<uint64_t>(o[4 * c + 3]) << 32)};
            }
        }
    } else {
#pragma unroll 1
        for (int k = 0; k < NK; ++k) aes_ccr(aes->te, aes->rk + 44 * k, p.lo, p.hi, h[k].lo, h[k].hi);
    }
}

// XOR-reduce vals[0..NK) over the CTA and fold into dst[0..NK) atomically.
template <int NK>
__device__ __forceinline__ void cta_xor_reduce(Blk (&v)[NK], Blk* dst, Blk* red /* [32][NK] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        uint64_t lo = v[k].lo, hi = v[k].hi;
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            lo ^= __shfl_xor_sync(0xffffffffu, lo, off);
            hi ^= __shfl_xor_sync(0xffffffffu, hi, off);
        }
        if (lane == 0) red[warp * NK + k] = Blk{lo, hi};
    }
    __syncthreads();
    if (threadIdx.x < NK) {
        uint64_t lo = 0, hi = 0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 0; w < nw; ++w) {
            lo ^= red[w * NK + threadIdx.x].lo;
            hi ^= red[w * NK + threadIdx.x].hi;
        }
        atomicXor(reinterpret_cast<unsigned long long*>(&dst[threadIdx.x].lo), lo);
        atomicXor(reinterpret_cast<unsigned long long*>(&dst[threadIdx.x].hi), hi);
    }
}

template <int PRG>
__device__ __forceinline__ const AesSm* stage_aes(AesSm& s, const uint32_t* te, const uint32_t* rk,
                                                  int nk) {
    if constexpr (PRG == PCGB_PRG_AES) {
        for (int i = threadIdx.x; i < 1024; i += blockDim.x) s.te[i] = te[i];
        for (int i = threadIdx.x; i < nk * 44; i += blockDim.x) s.rk[i] = rk[i];
        __syncthreads();
    }
    return &s;
}

// Level 0: hash the B roots (frontier of size 1).  grid = (1, B).
template <int W, int PRG>
__global__ void __launch_bounds__(kTPB) hash_roots_kernel(const Blk* __restrict__ cur, size_t D,
                                                          Blk* __restrict__ H, size_t HS,
                                                          Blk* __restrict__ my,
                                                          const uint32_t* te, const uint32_t* rk) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    Blk* red = reinterpret_cast<Blk*>(smraw);
    AesSm& aes = *reinterpret_cast<AesSm*>(smraw + 32 * NK * sizeof(Blk));
    const AesSm* a = stage_aes<PRG>(aes, te, rk, NK);
    const int b = blockIdx.y;
    Blk h[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) h[k] = Blk{0, 0};
    if (threadIdx.x == 0) {
        hash_node<W, PRG>(cur[static_cast<size_t>(b) * D], a, h);
#pragma unroll
        for (int k = 0; k < NK; ++k) H[static_cast<size_t>(b) * HS + k] = h[k];
    }
    cta_xor_reduce<NK>(h, my + static_cast<size_t>(b) * NK, red);
}

// Expand level i (frontier size sz, hashes H) with CW = my ^ peer; write the
// children to nxt; when hash_next, hash the children into Hn and reduce
// their columns into my_next.  grid = (x, B); thread x*kTPB + t of an
// instance expands its parent x*kTPB + t.
template <int W, int PRG>
__global__ void __launch_bounds__(kTPB) expand_level_kernel(
    const Blk* __restrict__ cur, const Blk* __restrict__ H, const Blk* __restrict__ my,
    const Blk* __restrict__ peer, Blk* __restrict__ nxt, Blk* __restrict__ Hn,
    Blk* __restrict__ my_next, size_t sz, size_t D, size_t HS, int hash_next,
    const uint32_t* te, const uint32_t* rk) {
    constexpr int M = 1 << W, NK = M - 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    Blk* red = reinterpret_cast<Blk*>(smraw);
    AesSm& aes = *reinterpret_cast<AesSm*>(smraw + 32 * NK * sizeof(Blk));
    const AesSm* a = stage_aes<PRG>(aes, te, rk, NK);
    const int b = blockIdx.y;
    Blk cw[NK];
    Blk cwf{0, 0};
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const Blk m0 = my[static_cast<size_t>(b) * NK + k], p0 = peer[static_cast<size_t>(b) * NK + k];
        cw[k] = Blk{m0.lo ^ p0.lo, m0.hi ^ p0.hi};
        cwf.lo ^= cw[k].lo;
        cwf.hi ^= cw[k].hi;
    }
    Blk acc[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) acc[k] = Blk{0, 0};
    auto parent = [&](const size_t j) {
        const Blk p = cur[static_cast<size_t>(b) * D + j];
        const bool t = (p.lo & 1) != 0;
        Blk kids[M];
        uint64_t xl = 0, xh = 0;
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            const Blk h = H[static_cast<size_t>(b) * HS + j * NK + k];
            xl ^= h.lo;
            xh ^= h.hi;
            kids[k] = Blk{h.lo ^ (t ? cw[k].lo : 0), h.hi ^ (t ? cw[k].hi : 0)};
        }
        kids[NK] = Blk{xl ^ p.lo ^ (t ? cwf.lo : 0), xh ^ p.hi ^ (t ? cwf.hi : 0)};
        Blk* dst = nxt + static_cast<size_t>(b) * D + j * M;
#pragma unroll
        for (int k = 0; k < M; ++k) dst[k] = kids[k];
        if (hash_next) {
            auto hash_child = [&](int k) {
                Blk h[NK];
                hash_node<W, PRG>(kids[k], a, h);
                Blk* hd = Hn + static_cast<size_t>(b) * HS + (j * M + k) * NK;
#pragma unroll
                for (int kk = 0; kk < NK; ++kk) {
                    hd[kk] = h[kk];
                    acc[kk].lo ^= h[kk].lo;
                    acc[kk].hi ^= h[kk].hi;
                }
            };
            if constexpr (PRG == PCGB_PRG_CHACHA8 && W <= 2) {
                // All children's blocks in flight (one block each for
                // w <= 2): independent ARX chains keep the integer pipe busy
                // while the level's loads and stores are outstanding, and
                // the children stay in registers.
#pragma unroll
                for (int k = 0; k < M; ++k) hash_child(k);
            } else {
#pragma unroll 1
                for (int k = 0; k < M; ++k) hash_child(k);
            }
        }
    };
    const size_t j0 = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j0 < sz) parent(j0);
    if (hash_next) cta_xor_reduce<NK>(acc, my_next + static_cast<size_t>(b) * NK, red);
}

// AES levels of kRepMinParents or more parents per instance with the
// PRMT-addressed table (aes128.cuh): one 768-thread CTA per SM, filled
// once, walking (instance, chunk) tiles of kPrmtChunk parents; per tile the
// same work as expand_level_kernel, then the CTA's XOR reduction into the
// instance's my_next.
constexpr int kPrmtTPB = 768;   // no register spills (at most 80 a thread)
constexpr size_t kPrmtChunk = 4096;

template <int W>
__global__ void __launch_bounds__(kPrmtTPB) expand_level_prmt_kernel(
    const Blk* __restrict__ cur, const Blk* __restrict__ H, const Blk* __restrict__ my,
    const Blk* __restrict__ peer, Blk* __restrict__ nxt, Blk* __restrict__ Hn,
    Blk* __restrict__ my_next, size_t sz, size_t D, size_t HS, int hash_next, int B,
    const uint32_t* te, const uint32_t* rk) {
    constexpr int M = 1 << W, NK = M - 1;
    extern __shared__ __align__(16) unsigned char prmt_dsm[];
    __shared__ AesPrmtKeys keys;
    __shared__ Blk red[32 * NK];
    const AesPrmt A = aes_prmt_setup<NK>(prmt_dsm, keys, te, rk);
    const size_t chunks = (sz + kPrmtChunk - 1) / kPrmtChunk;
    const size_t tiles = static_cast<size_t>(B) * chunks;
    for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const size_t b = tile / chunks, x = tile % chunks;
        Blk cw[NK];
        Blk cwf{0, 0};
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            const Blk m0 = my[b * NK + k], p0 = peer[b * NK + k];
            cw[k] = Blk{m0.lo ^ p0.lo, m0.hi ^ p0.hi};
            cwf.lo ^= cw[k].lo;
            cwf.hi ^= cw[k].hi;
        }
        Blk acc[NK];
#pragma unroll
        for (int k = 0; k < NK; ++k) acc[k] = Blk{0, 0};
        const size_t j1 = (x + 1) * kPrmtChunk < sz ? (x + 1) * kPrmtChunk : sz;
        for (size_t j = x * kPrmtChunk + threadIdx.x; j < j1; j += blockDim.x) {
            const Blk p = cur[b * D + j];
            const bool t = (p.lo & 1) != 0;
            Blk kids[M];
            uint64_t xl = 0, xh = 0;
#pragma unroll
            for (int k = 0; k < NK; ++k) {
                const Blk h = H[b * HS + j * NK + k];
                xl ^= h.lo;
                xh ^= h.hi;
                kids[k] = Blk{h.lo ^ (t ? cw[k].lo : 0), h.hi ^ (t ? cw[k].hi : 0)};
            }
            kids[NK] = Blk{xl ^ p.lo ^ (t ? cwf.lo : 0), xh ^ p.hi ^ (t ? cwf.hi : 0)};
            Blk* dst = nxt + b * D + j * M;
#pragma unroll
            for (int k = 0; k < M; ++k) dst[k] = kids[k];
            if (hash_next) {
                if constexpr (W == 1) {
                    // Both children's hashes in flight at once.
                    Blk h0, h1;
                    aes_ccr_prmt(A, 0, kids[0].lo, kids[0].hi, h0.lo, h0.hi);
                    aes_ccr_prmt(A, 0, kids[1].lo, kids[1].hi, h1.lo, h1.hi);
                    Hn[b * HS + j * 2] = h0;
                    Hn[b * HS + j * 2 + 1] = h1;
                    acc[0].lo ^= h0.lo ^ h1.lo;
                    acc[0].hi ^= h0.hi ^ h1.hi;
                } else {
#pragma unroll 1
                    for (int k = 0; k < M; ++k) {
                        Blk* hd = Hn + b * HS + (j * M + k) * NK;
#pragma unroll 1
                        for (int q = 0; q < NK; ++q) {
                            Blk h;
                            aes_ccr_prmt(A, q, kids[k].lo, kids[k].hi, h.lo, h.hi);
                            hd[q] = h;
                            acc[q].lo ^= h.lo;
                            acc[q].hi ^= h.hi;
                        }
                    }
                }
            }
        }
        if (hash_next) cta_xor_reduce<NK>(acc, my_next + b * NK, red);
        __syncthreads();   // red is reused by the next tile
    }
}

// Last level fused with the output layer's first pass (the two-party
// expansion's form): expands level levels-1 with its CW like
// expand_level_kernel, but instead of storing the leaves it hashes each one
// (ChaCha8 out-hash, leaf_convert_cuda.cu's C and tau) into the converted
// word conv[b*D + d] = C | tau << 63 and reduces C (mod p) and tau over the
// CTA into partials[b*parts + x] and partials[(B + b)*parts + x].
// grid = (parts, B), parts = ceil(sz / kTPB).
template <int W>
__global__ void __launch_bounds__(kTPB) last_level_convert_kernel(
    const Blk* __restrict__ cur, const Blk* __restrict__ H, const Blk* __restrict__ my,
    const Blk* __restrict__ peer, size_t sz, size_t D, size_t HS, uint64_t* __restrict__ conv,
    uint64_t* __restrict__ partials) {
    constexpr int M = 1 << W, NK = M - 1;
    __shared__ uint64_t sc[kTPB / 32], st[kTPB / 32];
    const int b = blockIdx.y, parts = gridDim.x;
    const size_t j = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    Blk cw[NK];
    Blk cwf{0, 0};
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const Blk m0 = my[static_cast<size_t>(b) * NK + k], p0 = peer[static_cast<size_t>(b) * NK + k];
        cw[k] = Blk{m0.lo ^ p0.lo, m0.hi ^ p0.hi};
        cwf.lo ^= cw[k].lo;
        cwf.hi ^= cw[k].hi;
    }
    uint64_t csum = 0, tsum = 0;
    if (j < sz) {
        const Blk p = cur[static_cast<size_t>(b) * D + j];
        const bool t = (p.lo & 1) != 0;
        Blk kids[M];
        uint64_t xl = 0, xh = 0;
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            const Blk h = H[static_cast<size_t>(b) * HS + j * NK + k];
            xl ^= h.lo;
            xh ^= h.hi;
            kids[k] = Blk{h.lo ^ (t ? cw[k].lo : 0), h.hi ^ (t ? cw[k].hi : 0)};
        }
        kids[NK] = Blk{xl ^ p.lo ^ (t ? cwf.lo : 0), xh ^ p.hi ^ (t ? cwf.hi : 0)};
        uint64_t* dst = conv + static_cast<size_t>(b) * D + j * M;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const uint64_t C = reduce_p(out_hash_lo64(kids[k].lo, kids[k].hi));
            csum = add_p(csum, C);
            tsum += kids[k].lo & 1;
            dst[k] = C | (kids[k].lo << 63);
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        csum = add_p(csum, __shfl_xor_sync(0xffffffffu, csum, off));
        tsum += __shfl_xor_sync(0xffffffffu, tsum, off);
    }
    if ((threadIdx.x & 31) == 0) { sc[threadIdx.x >> 5] = csum; st[threadIdx.x >> 5] = tsum; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t cc = 0, tt = 0;
        for (int w = 0; w < kTPB / 32; ++w) { cc = add_p(cc, sc[w]); tt += st[w]; }
        const size_t slot = static_cast<size_t>(b) * parts + blockIdx.x;
        partials[slot] = cc;
        partials[static_cast<size_t>(gridDim.y) * parts + slot] = tt;
    }
}

// sumC[b], sumT[b] from the B x parts partials, in a fixed order.
__global__ void convert_fold_kernel(const uint64_t* __restrict__ partials, int parts, int B,
                                    uint64_t* __restrict__ sumC, uint64_t* __restrict__ sumT) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t c = 0, t = 0;
    for (int i = 0; i < parts; ++i) {
        c = add_p(c, partials[static_cast<size_t>(b) * parts + i]);
        t += partials[static_cast<size_t>(B) * parts + static_cast<size_t>(b) * parts + i];
    }
    sumC[b] = c;
    sumT[b] = t;
}

// Where the fused last level writes (see last_level_convert_kernel), and an
// optional device-side exchange that replaces the host round trip.
struct ConvOut {
    uint64_t* conv;
    uint64_t* partials;
    pcgb_exchange_device_fn dex = nullptr;
    void* dex_user = nullptr;
};

// my[b][k] = dlt[b][level][k].
__global__ void seed_kernel(Blk* my, const Blk* dlt, int B, int levels, int nk, int level) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * nk) return;
    const int b = i / nk, k = i % nk;
    my[i] = dlt[(static_cast<size_t>(b) * levels + level) * nk + k];
}

struct Pool {
    Blk *cur = nullptr, *nxt = nullptr, *H = nullptr, *Hn = nullptr, *dlt = nullptr;
    Blk *my = nullptr, *myn = nullptr, *peer = nullptr;
    uint32_t* rk = nullptr;
    Blk *h_my = nullptr, *h_peer = nullptr;   // pinned
    size_t cap_front = 0, cap_h = 0, cap_dlt = 0, cap_cw = 0;
    std::mutex mu;
};

Pool& pool_for_device() {
    static std::mutex mu;
    static Pool* pools[64] = {nullptr};
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) pools[dev] = new Pool();
    return *pools[dev];
}

template <class T>
void grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        fail(PCGB_ENOMEM, "dpf_gpu_batch_full_eval: device allocation failed");
    }
    cap = need;
}

template <int W, int PRG>
Blk* run_levels(Pool& pl, int B, int n, const Blk* roots, const Blk* dltsft,
                pcgb_exchange_fn ex, void* user, cudaStream_t st, const ConvOut* conv) {
    constexpr int M = 1 << W, NK = M - 1;
    const int levels = n / W;
    const size_t D = static_cast<size_t>(1) << n;
    const size_t HS = (D / M) * NK;
    const size_t ncw = static_cast<size_t>(B) * NK;
    const size_t smem = 32 * NK * sizeof(Blk) + (PRG == PCGB_PRG_AES ? sizeof(AesSm) : 0);
    const uint32_t* te = PRG == PCGB_PRG_AES ? aes_te_table_device() : nullptr;
    PCGB_CK(cudaMemcpy2DAsync(pl.cur, D * sizeof(Blk), roots, sizeof(Blk), sizeof(Blk),
                              static_cast<size_t>(B), cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(pl.dlt, dltsft, static_cast<size_t>(B) * levels * NK * sizeof(Blk),
                            cudaMemcpyHostToDevice, st));
    const unsigned sgrid = static_cast<unsigned>((ncw + 255) / 256);
    seed_kernel<<<sgrid, 256, 0, st>>>(pl.my, pl.dlt, B, levels, NK, 0);
    PCGB_POST_LAUNCH();
    hash_roots_kernel<W, PRG><<<dim3(1, B), kTPB, smem, st>>>(pl.cur, D, pl.H, HS, pl.my, te, pl.rk);
    PCGB_POST_LAUNCH();
    Blk *cur = pl.cur, *nxt = pl.nxt, *H = pl.H, *Hn = pl.Hn, *my = pl.my, *myn = pl.myn;
    for (int i = 0; i < levels; ++i) {
        if (conv && conv->dex) {
            // Shares stay on the device: the callback moves them (NCCL,
            // peer copies) after the level's reduction has finished.
            PCGB_CK(cudaStreamSynchronize(st));
            if (conv->dex(reinterpret_cast<const pcgb_blk*>(my), reinterpret_cast<pcgb_blk*>(pl.peer),
                          ncw, conv->dex_user) != 0)
                fail(PCGB_ECALLBACK, "dpf_gpu_batch_full_eval: device exchange callback failed");
        } else {
            PCGB_CK(cudaMemcpyAsync(pl.h_my, my, ncw * sizeof(Blk), cudaMemcpyDeviceToHost, st));
            PCGB_CK(cudaStreamSynchronize(st));
            if (ex) {
                if (ex(reinterpret_cast<const pcgb_blk*>(pl.h_my),
                       reinterpret_cast<pcgb_blk*>(pl.h_peer), ncw, user) != 0)
                    fail(PCGB_ECALLBACK, "dpf_gpu_batch_full_eval: exchange callback failed");
            } else {
                for (size_t k = 0; k < ncw; ++k) pl.h_peer[k] = Blk{0, 0};
            }
            PCGB_CK(cudaMemcpyAsync(pl.peer, pl.h_peer, ncw * sizeof(Blk), cudaMemcpyHostToDevice,
                                    st));
        }
        const int hash_next = (i + 1 < levels) ? 1 : 0;
        if (hash_next) {
            seed_kernel<<<sgrid, 256, 0, st>>>(myn, pl.dlt, B, levels, NK, i + 1);
            PCGB_POST_LAUNCH();
        }
        const size_t sz = static_cast<size_t>(1) << (W * i);
        if (!hash_next && conv) {
            // One parent per thread: the grid the fold's `parts` assumes.
            const dim3 cgrid(static_cast<unsigned>((sz + kTPB - 1) / kTPB), static_cast<unsigned>(B));
            last_level_convert_kernel<W><<<cgrid, kTPB, 0, st>>>(cur, H, my, pl.peer, sz, D, HS,
                                                                 conv->conv, conv->partials);
            PCGB_POST_LAUNCH();
            return nullptr;
        }
        // The last level only writes leaves (no hashing): the plain kernel.
        const bool rep = PRG == PCGB_PRG_AES && sz >= kRepMinParents && hash_next;
        const dim3 grid(static_cast<unsigned>((sz + kTPB - 1) / kTPB), static_cast<unsigned>(B));
        if constexpr (PRG == PCGB_PRG_AES) {
            if (rep) {
                PCGB_CK(cudaFuncSetAttribute(expand_level_prmt_kernel<W>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kAesPrmtSmemBytes)));
                const size_t tiles = static_cast<size_t>(B) * ((sz + kPrmtChunk - 1) / kPrmtChunk);
                const unsigned pgrid = static_cast<unsigned>(
                    std::min<size_t>(tiles, static_cast<size_t>(sm_count())));
                expand_level_prmt_kernel<W><<<pgrid, kPrmtTPB, kAesPrmtSmemBytes, st>>>(
                    cur, H, my, pl.peer, nxt, Hn, myn, sz, D, HS, hash_next, B, te, pl.rk);
            } else {
                expand_level_kernel<W, PRG><<<grid, kTPB, smem, st>>>(
                    cur, H, my, pl.peer, nxt, Hn, myn, sz, D, HS, hash_next, te, pl.rk);
            }
        } else {
            expand_level_kernel<W, PRG><<<grid, kTPB, smem, st>>>(
                cur, H, my, pl.peer, nxt, Hn, myn, sz, D, HS, hash_next, te, pl.rk);
        }
        PCGB_POST_LAUNCH();
        std::swap(cur, nxt);
        std::swap(H, Hn);
        std::swap(my, myn);
    }
    return cur;
}

void grow_pair(Blk*& a, Blk*& b, size_t& cap, size_t need) {
    if (need <= cap) return;
    size_t c1 = cap, c2 = cap;
    grow(a, c1, need);
    grow(b, c2, need);
    cap = need;
}

Blk* interactive_eval(int B, int n, int w, const Blk* roots, const Blk* dltsft, const uint8_t* rks,
                      int prg, pcgb_exchange_fn ex, void* user, cudaStream_t st, Pool& pl,
                      const ConvOut* conv = nullptr) {
    if (w < 1 || w > 4)
        fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: w must be in [1,4] (expand_kernel CW[16])");
    if (n < 1 || n % w != 0) fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: w must divide n");
    if (n > 30) fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: n must be at most 30");
    if (prg == PCGB_PRG_AES && rks == nullptr)
        fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: AES PRG requires round_keys");
    if (prg != PCGB_PRG_AES && prg != PCGB_PRG_CHACHA8)
        fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: unknown PRG");
    if (!roots || !dltsft) fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: null input");
    const int m = 1 << w, nk = m - 1, levels = n / w;
    const size_t D = static_cast<size_t>(1) << n;
    grow_pair(pl.cur, pl.nxt, pl.cap_front, static_cast<size_t>(B) * D);
    grow_pair(pl.H, pl.Hn, pl.cap_h, static_cast<size_t>(B) * (D / m) * nk);
    grow(pl.dlt, pl.cap_dlt, static_cast<size_t>(B) * levels * nk);
    const size_t ncw = static_cast<size_t>(B) * nk;
    if (ncw > pl.cap_cw) {
        size_t c1 = pl.cap_cw, c2 = pl.cap_cw, c3 = pl.cap_cw;
        grow(pl.my, c1, ncw);
        grow(pl.myn, c2, ncw);
        grow(pl.peer, c3, ncw);
        if (pl.h_my) cudaFreeHost(pl.h_my);
        if (pl.h_peer) cudaFreeHost(pl.h_peer);
        pl.h_my = pl.h_peer = nullptr;
        PCGB_CK(cudaMallocHost(&pl.h_my, ncw * sizeof(Blk)));
        PCGB_CK(cudaMallocHost(&pl.h_peer, ncw * sizeof(Blk)));
        pl.cap_cw = ncw;
    }
    if (!pl.rk) PCGB_CK(cudaMalloc(&pl.rk, 15 * 176));
    if (prg == PCGB_PRG_AES)
        PCGB_CK(cudaMemcpyAsync(pl.rk, rks, static_cast<size_t>(nk) * 176, cudaMemcpyHostToDevice,
                                st));
#define PCGB_RUN(W_)                                                                        \
    case W_:                                                                                \
        return prg == PCGB_PRG_AES                                                          \
                   ? run_levels<W_, PCGB_PRG_AES>(pl, B, n, roots, dltsft, ex, user, st, conv) \
                   : run_levels<W_, PCGB_PRG_CHACHA8>(pl, B, n, roots, dltsft, ex, user, st, conv);
    switch (w) {
        PCGB_RUN(1)
        PCGB_RUN(2)
        PCGB_RUN(3)
        PCGB_RUN(4)
    }
#undef PCGB_RUN
    return nullptr;
}

}  // namespace

// Runs the level loop under the per-device pool lock; the returned pointer
// aliases the pool (valid until the next call on this device).
const Blk* dpf_interactive_device(int B, int n, int w, const Blk* roots, const Blk* dltsft,
                                  const uint8_t* rks, int prg, pcgb_exchange_fn ex, void* user,
                                  Blk* host_out) {
    if (B <= 0) return nullptr;
    Pool& pl = pool_for_device();
    std::lock_guard<std::mutex> lk(pl.mu);
    cudaStream_t st = default_stream();
    Blk* leaves = interactive_eval(B, n, w, roots, dltsft, rks, prg, ex, user, st, pl);
    if (host_out)
        PCGB_CK(cudaMemcpyAsync(host_out, leaves, (static_cast<size_t>(B) << n) * sizeof(Blk),
                                cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
    return leaves;
}

// The interactive evaluation with its last level fused into the output
// layer's sums pass: no leaves are stored.  Outputs are complete on return.
void dpf_interactive_convert_device(int B, int n, int w, const Blk* roots, const Blk* dltsft,
                                    const uint8_t* rks, int prg, pcgb_exchange_fn ex, void* user,
                                    uint64_t* d_conv, uint64_t* d_sumC, uint64_t* d_sumT,
                                    pcgb_exchange_device_fn dex, void* dex_user) {
    if (B <= 0) return;
    if (!d_conv || !d_sumC || !d_sumT)
        fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval_convert: null output pointer");
    if (w < 1 || w > 4 || n < 1 || n % w != 0 || n > 30)
        fail(PCGB_EINVAL, "dpf_gpu_batch_full_eval: w must be in [1,4] and divide n <= 30");
    Pool& pl = pool_for_device();
    std::lock_guard<std::mutex> lk(pl.mu);
    cudaStream_t st = default_stream();
    const size_t last = static_cast<size_t>(1) << (n - w);   // parents at the last level
    const int parts = static_cast<int>((last + kTPB - 1) / kTPB);
    uint64_t* partials = static_cast<uint64_t*>(
        pool_alloc(2 * static_cast<size_t>(B) * parts * sizeof(uint64_t), st));
    const ConvOut conv{d_conv, partials, dex, dex_user};
    try {
        interactive_eval(B, n, w, roots, dltsft, rks, prg, ex, user, st, pl, &conv);
    } catch (...) {
        cudaFreeAsync(partials, st);
        throw;
    }
    convert_fold_kernel<<<(B + 127) / 128, 128, 0, st>>>(partials, parts, B, d_sumC, d_sumT);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(partials, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

}  // namespace pcgb
