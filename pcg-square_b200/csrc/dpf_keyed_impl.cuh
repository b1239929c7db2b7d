// Keyed half-tree DPF full-domain evaluation fused with the output layer.
//
// A key is (root, CW[level][0..nk), cw_out).  The per-level update is the
// half-tree rule of half_tree_dpf/dpf.cpp:553-574: children k < m-1 are
// H_k(parent) ^ t*CW[k]; child m-1 is (XOR_k H_k) ^ parent ^ t*CW[m-1] with
// CW[m-1] = XOR_k CW[k] and t = lsb(parent).  Because every CW is known,
// any subtree can be expanded independently: no per-level barrier.
//
// Two kernels:
//   expand_tops   root -> frontier at level hl (= levels - sl), one thread
//                 per source node, depth-first, nodes written in order.
//   leaf_gather   one thread per S = m^sl consecutive output positions of a
//                 folded, pair-merged g' buffer.  For every key half that
//                 lands on those positions (the gather plan) it loads one
//                 frontier node, expands sl levels in registers, hashes each
//                 leaf with the output-layer ChaCha8 (nonce "out_hash"),
//                 converts C = low64 mod p, y = C + tau*cw_out, applies the
//                 party / fold signs and accumulates mod p.  Each g' word is
//                 written once, coalesced, with no atomics: the result is
//                 bit-identical to the reference's CAS-atomic scatter
//                 (GPU_baseline/common/leaf_convert_cuda.cu:207-234), whose
//                 mod-p sum is order independent.
#ifndef PCGB_DPF_KEYED_IMPL_CUH_
#define PCGB_DPF_KEYED_IMPL_CUH_

#include "pcgb_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

#include "aes128.cuh"
#include "chacha8.cuh"
#include "field.cuh"
#include "synth.h"

namespace pcgb {
namespace {

constexpr int kPrgAes = PCGB_PRG_AES;
constexpr int kPrgChaCha = PCGB_PRG_CHACHA8;

// Per-thread DFS stack depth of the tops kernel: covers n <= 30 for any w.
template <int W>
__host__ __device__ constexpr int tops_max_depth() { return 30 / W + 1; }

struct AesSmem {
    uint32_t te_rep[kAesRepWords];   // Te0 replicated per lane (aes128.cuh)
    uint32_t rk[15 * 44];
};

__device__ __forceinline__ void load_aes_smem(AesSmem& s, const uint32_t* te, const uint32_t* rk,
                                              int nk) {
    aes_fill_rep(s.te_rep, te);
    for (int i = threadIdx.x; i < nk * 44; i += blockDim.x) s.rk[i] = rk[i];
    __syncthreads();
}

__device__ __forceinline__ Blk ldblk(const Blk* p) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
    return Blk{v.x, v.y};
}

__device__ __forceinline__ void stblk(Blk* p, const Blk& b) {
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(b.lo, b.hi);
}

// AES CCR hash H_k of one node, with the replicated table (AesSmem) or the
// PRMT-addressed one (AesPrmt).
__device__ __forceinline__ void aes_node(const AesSmem* a, int k, uint64_t lo, uint64_t hi,
                                         uint64_t& olo, uint64_t& ohi) {
    aes_ccr_rep(a->te_rep, a->rk + 44 * k, lo, hi, olo, ohi);
}
__device__ __forceinline__ void aes_node(const AesPrmt* a, int k, uint64_t lo, uint64_t hi,
                                         uint64_t& olo, uint64_t& ohi) {
    aes_ccr_prmt(*a, k, lo, hi, olo, ohi);
}

// m children of `p` under the level CWs cw[0..nk) (global, broadcast).
template <int W, int PRG, class A>
__device__ __forceinline__ void children(const Blk& p, const Blk* __restrict__ cw,
                                         const A* aes, Blk (&kids)[1 << W]) {
    constexpr int M = 1 << W, NK = M - 1;
    const bool t = (p.lo & 1) != 0;
    uint64_t hxl = 0, hxh = 0, cfl = 0, cfh = 0;
    if constexpr (PRG == kPrgChaCha) {
#pragma unroll
        for (int b = 0; b < (NK + 3) / 4; ++b) {
            uint32_t o[16];
            tree_block(p.lo, p.hi, b, o);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int k = 4 * b + c;
                if (k < NK) {
                    const uint64_t hl = o[4 * c] | (static_cast<uint64_t>(o[4 * c + 1]) << 32);
                    const uint64_t hh = o[4 * c + 2] | (static_cast<uint64_t>(o[4 * c + 3]) << 32);
                    const Blk cv = ldblk(cw + k);
                    cfl ^= cv.lo; cfh ^= cv.hi;
                    hxl ^= hl; hxh ^= hh;
                    kids[k] = Blk{hl ^ (t ? cv.lo : 0), hh ^ (t ? cv.hi : 0)};
                }
            }
        }
    } else {
#pragma unroll 1
        for (int k = 0; k < NK; ++k) {
            uint64_t hl, hh;
            aes_node(aes, k, p.lo, p.hi, hl, hh);
            const Blk cv = ldblk(cw + k);
            cfl ^= cv.lo; cfh ^= cv.hi;
            hxl ^= hl; hxh ^= hh;
            kids[k] = Blk{hl ^ (t ? cv.lo : 0), hh ^ (t ? cv.hi : 0)};
        }
    }
    kids[NK] = Blk{hxl ^ p.lo ^ (t ? cfl : 0), hxh ^ p.hi ^ (t ? cfh : 0)};
}

// Raw tree hashes H_0..H_{nk-1} of one node (no correction words).
template <int W, int PRG, class A>
__device__ __forceinline__ void hash_raw(const Blk& p, const A* aes, Blk (&h)[(1 << W) - 1]) {
    constexpr int NK = (1 << W) - 1;
    if constexpr (PRG == kPrgChaCha) {
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
        for (int k = 0; k < NK; ++k) aes_node(aes, k, p.lo, p.hi, h[k].lo, h[k].hi);
    }
}

// ---------------------------------------------------------------------------
// expand_tops: depth-first expansion of `nlev` levels below each source node.
// Thread `id` (< K * m^src_lvl) expands source node id: key id / m^src_lvl.
template <int W, int PRG, class A>
__device__ __forceinline__ void tops_walk(const Blk* __restrict__ src, size_t id, int src_lvl,
                                          int nlev, int levels, const Blk* __restrict__ cws,
                                          const A* aes, Blk* __restrict__ dst) {
    constexpr int M = 1 << W, NK = M - 1;
    constexpr int MAXD = tops_max_depth<W>();
    const size_t per_key_src = static_cast<size_t>(1) << (W * src_lvl);
    const size_t key = id / per_key_src;
    const size_t j = id % per_key_src;
    const Blk* kcw = cws + key * static_cast<size_t>(levels) * NK;
    const size_t fan = static_cast<size_t>(1) << (W * nlev);
    Blk* out = dst + key * (per_key_src * fan) + j * fan;
    const Blk root = ldblk(src + id);
    if (nlev == 0) { stblk(out, root); return; }

    // stack[d][k]: children at relative depth d+1; pos[d]: next child index.
    Blk stack[MAXD][M];
    int pos[MAXD];
    children<W, PRG>(root, kcw + static_cast<size_t>(src_lvl) * NK, aes, stack[0]);
    pos[0] = 0;
    int d = 0;
    size_t emitted = 0;
    while (d >= 0) {
        if (d == nlev - 1) {
#pragma unroll
            for (int k = 0; k < M; ++k) stblk(out + emitted + k, stack[d][k]);
            emitted += M;
            --d;
            if (d >= 0) ++pos[d];
            continue;
        }
        if (pos[d] == M) {
            --d;
            if (d >= 0) ++pos[d];
            continue;
        }
        Blk kids[M];
        children<W, PRG>(stack[d][pos[d]], kcw + static_cast<size_t>(src_lvl + d + 1) * NK, aes,
                         kids);
#pragma unroll
        for (int k = 0; k < M; ++k) stack[d + 1][k] = kids[k];
        ++d;
        pos[d] = 0;
    }
}

template <int W, int PRG>
__global__ void __launch_bounds__(128) expand_tops_kernel(
    const Blk* __restrict__ src, int K, int src_lvl, int nlev, int levels,
    const Blk* __restrict__ cws, const uint32_t* __restrict__ aes_te,
    const uint32_t* __restrict__ aes_rk, Blk* __restrict__ dst) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) uint64_t tops_dsm[];
    AesSmem& aes_s = *reinterpret_cast<AesSmem*>(tops_dsm);
    if constexpr (PRG == kPrgAes) load_aes_smem(aes_s, aes_te, aes_rk, NK);
    const size_t id = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= (static_cast<size_t>(K) << (W * src_lvl))) return;
    tops_walk<W, PRG>(src, id, src_lvl, nlev, levels, cws, &aes_s, dst);
}

// Binary (w = 1) ChaCha8 walk of a depth D fixed at compile time: the
// recursion keeps one pending right child per level in registers (its
// two-way loop is not unrolled, so the code grows linearly with D), where
// tops_walk's run-time depth keeps its stack in local memory.  LV is the
// level below the source node (its CWs are cw[LV]); u the output offset of
// the subtree.  Outputs in the same left-to-right order.
template <int D, int LV = 0>
struct TopsFixed1 {
    __device__ __forceinline__ static void run(const Blk& node, const Blk* __restrict__ cw,
                                               Blk* __restrict__ out, unsigned u) {
        Blk k2[2];
        children<1, kPrgChaCha>(node, cw + LV, static_cast<const AesSmem*>(nullptr), k2);
        if constexpr (D == 1) {
            stblk(out + u, k2[0]);
            stblk(out + u + 1, k2[1]);
        } else {
            Blk cur = k2[0];
            const Blk R = k2[1];
#pragma unroll 1
            for (unsigned i = 0; i < 2; ++i) {
                TopsFixed1<D - 1, LV + 1>::run(cur, cw, out, u + (i << (D - 1)));
                cur = R;
            }
        }
    }
};
constexpr int kTopsFixedMax = kTopsFixedLevels;
static_assert(kTopsFixedMax == 8, "one compile-time walk per depth 1 .. 8");

// expand_tops_kernel for ChaCha8, w = 1, nlev = D.
template <int D>
__global__ void __launch_bounds__(128) expand_tops_fixed_kernel(
    const Blk* __restrict__ src, int K, int src_lvl, int levels, const Blk* __restrict__ cws,
    Blk* __restrict__ dst) {
    const size_t id = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= (static_cast<size_t>(K) << src_lvl)) return;
    const size_t key = id >> src_lvl;
    TopsFixed1<D>::run(ldblk(src + id), cws + key * levels + src_lvl, dst + (id << D), 0);
}

// One stage of several key groups of different domains in one persistent
// launch: the grid strides over the concatenated source nodes of all jobs;
// job j owns global thread indices [first, first + K << (W * src_lvl)).
template <int W, int PRG>
__global__ void __launch_bounds__(128) expand_tops_multi_kernel(
    const TopsJob* __restrict__ jobs, int njobs, unsigned long long total,
    const uint32_t* __restrict__ aes_te, const uint32_t* __restrict__ aes_rk) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) uint64_t tops_dsm[];
    AesSmem& aes_s = *reinterpret_cast<AesSmem*>(tops_dsm);
    if constexpr (PRG == kPrgAes) load_aes_smem(aes_s, aes_te, aes_rk, NK);
    for (unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                                threadIdx.x;
         g < total; g += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].first <= g) ++j;
        const TopsJob J = jobs[j];
        tops_walk<W, PRG>(J.src, g - J.first, J.src_lvl, J.nlev, J.levels, J.cws, &aes_s, J.dst);
    }
}

// expand_tops_multi_kernel for ChaCha8, w = 1, every job D levels deep.
template <int D>
__global__ void __launch_bounds__(128) expand_tops_multi_depth_kernel(
    const TopsJob* __restrict__ jobs, int njobs, unsigned long long total) {
    for (unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                                threadIdx.x;
         g < total; g += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].first <= g) ++j;
        const TopsJob J = jobs[j];
        const size_t id = g - J.first;
        TopsFixed1<D>::run(ldblk(J.src + id), J.cws + (id >> J.src_lvl) * J.levels + J.src_lvl,
                           J.dst + (id << D), 0);
    }
}

// expand_tops_multi_kernel for ChaCha8, w = 1, jobs of different depths: a
// job of 1 .. kTopsFixedMax levels takes the compile-time-depth walk of its
// depth, a deeper one the run-time walk.
__global__ void __launch_bounds__(128) expand_tops_multi_fixed_kernel(
    const TopsJob* __restrict__ jobs, int njobs, unsigned long long total) {
    for (unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                                threadIdx.x;
         g < total; g += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].first <= g) ++j;
        const TopsJob J = jobs[j];
        const size_t id = g - J.first;
        const Blk* kcw = J.cws + (id >> J.src_lvl) * J.levels + J.src_lvl;
        switch (J.nlev) {
#define PCGB_TF(D)                                                          \
    case D:                                                                 \
        TopsFixed1<D>::run(ldblk(J.src + id), kcw, J.dst + (id << D), 0); \
        break;
            PCGB_TF(1) PCGB_TF(2) PCGB_TF(3) PCGB_TF(4)
            PCGB_TF(5) PCGB_TF(6) PCGB_TF(7) PCGB_TF(8)
#undef PCGB_TF
            default:
                tops_walk<1, kPrgChaCha>(J.src, id, J.src_lvl, J.nlev, J.levels, J.cws,
                                         static_cast<const AesSmem*>(nullptr), J.dst);
        }
    }
}

// AES top-level walks with the PRMT-addressed tables (aes128.cuh): the 64 KB
// table region takes most of an SM's shared memory, so these run one
// 1024-thread CTA per SM, each thread walking source nodes grid-stride (the
// table is filled once per CTA, not once per 128 threads).
constexpr int kAesPrmtThreads = 1024;

// TopsFixed1 for AES with the PRMT-addressed tables.
template <int D, int LV = 0>
struct TopsFixedAes {
    __device__ __forceinline__ static void run(const Blk& node, const Blk* __restrict__ cw,
                                               const AesPrmt* aes, Blk* __restrict__ out,
                                               unsigned u) {
        Blk k2[2];
        children<1, kPrgAes>(node, cw + LV, aes, k2);
        if constexpr (D == 1) {
            stblk(out + u, k2[0]);
            stblk(out + u + 1, k2[1]);
        } else {
            Blk cur = k2[0];
            const Blk R = k2[1];
#pragma unroll 1
            for (unsigned i = 0; i < 2; ++i) {
                TopsFixedAes<D - 1, LV + 1>::run(cur, cw, aes, out, u + (i << (D - 1)));
                cur = R;
            }
        }
    }
};

// expand_tops_prmt_kernel<1> with the walk depth D fixed at compile time.
template <int D>
__global__ void __launch_bounds__(kAesPrmtThreads) expand_tops_prmt_fixed_kernel(
    const Blk* __restrict__ src, int K, int src_lvl, int levels, const Blk* __restrict__ cws,
    const uint32_t* __restrict__ aes_te, const uint32_t* __restrict__ aes_rk,
    Blk* __restrict__ dst) {
    extern __shared__ __align__(16) unsigned char prmt_dsm[];
    __shared__ AesPrmtKeys keys;
    const AesPrmt A = aes_prmt_setup<1>(prmt_dsm, keys, aes_te, aes_rk);
    const size_t total = static_cast<size_t>(K) << src_lvl;
    for (size_t id = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; id < total;
         id += static_cast<size_t>(gridDim.x) * blockDim.x)
        TopsFixedAes<D>::run(ldblk(src + id), cws + (id >> src_lvl) * levels + src_lvl, &A,
                             dst + (id << D), 0);
}

template <int W>
__global__ void __launch_bounds__(kAesPrmtThreads) expand_tops_prmt_kernel(
    const Blk* __restrict__ src, int K, int src_lvl, int nlev, int levels,
    const Blk* __restrict__ cws, const uint32_t* __restrict__ aes_te,
    const uint32_t* __restrict__ aes_rk, Blk* __restrict__ dst) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) unsigned char prmt_dsm[];
    __shared__ AesPrmtKeys keys;
    const AesPrmt A = aes_prmt_setup<NK>(prmt_dsm, keys, aes_te, aes_rk);
    const size_t total = static_cast<size_t>(K) << (W * src_lvl);
    for (size_t id = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; id < total;
         id += static_cast<size_t>(gridDim.x) * blockDim.x)
        tops_walk<W, kPrgAes>(src, id, src_lvl, nlev, levels, cws, &A, dst);
}

template <int W>
__global__ void __launch_bounds__(kAesPrmtThreads) expand_tops_multi_prmt_kernel(
    const TopsJob* __restrict__ jobs, int njobs, unsigned long long total,
    const uint32_t* __restrict__ aes_te, const uint32_t* __restrict__ aes_rk) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) unsigned char prmt_dsm[];
    __shared__ AesPrmtKeys keys;
    const AesPrmt A = aes_prmt_setup<NK>(prmt_dsm, keys, aes_te, aes_rk);
    for (unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                                threadIdx.x;
         g < total; g += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].first <= g) ++j;
        const TopsJob J = jobs[j];
        tops_walk<W, kPrgAes>(J.src, g - J.first, J.src_lvl, J.nlev, J.levels, J.cws, &A, J.dst);
    }
}

// Work items of one full wave of PRMT CTAs (one per SM).
inline unsigned long long aes_prmt_wave() {
    return static_cast<unsigned long long>(sm_count()) * kAesPrmtThreads;
}

// Grid of a PRMT kernel over `threads` work items: at most one CTA per SM.
inline unsigned aes_prmt_grid(unsigned long long threads) {
    const unsigned long long need = (threads + kAesPrmtThreads - 1) / kAesPrmtThreads;
    const unsigned long long sms = static_cast<unsigned long long>(sm_count());
    return static_cast<unsigned>(need < sms ? (need ? need : 1) : sms);
}

// ---------------------------------------------------------------------------
// leaf_gather: see the file comment.

// Two output-layer hashes at once (independent states: twice the ILP).
__device__ __forceinline__ void out_hash_x2(const Blk& a, const Blk& b, uint64_t& ha,
                                            uint64_t& hb) {
    ha = out_hash_lo64(a.lo, a.hi);
    hb = out_hash_lo64(b.lo, b.hi);
}

// Output-layer accumulation with one reduction per output word.  Each
// position keeps a 128-bit two's-complement sum (lo, hi) of its leaves'
// y = h + tau*cwo, h the raw 64-bit out-hash word (so y < 2^65), added for
// one sign and subtracted for the other; it is reduced mod p once, at
// write-out.  Exact, since only the sum mod p is used, and far from
// overflow: a position receives at most 4t key halves.  Against reducing h,
// adding cwo mod p, negating and adding mod p for every leaf, this leaves a
// few integer adds per leaf on the ALU pipe the ChaCha8 rounds saturate.
struct LeafCtx {
    ulonglong2* acc;  // this thread's accumulator row: (lo, hi) per position
    uint64_t cwo;     // output-layer CW of the current key
    bool neg;         // party ^ fold; the same for every thread of the CTA
};

__device__ __forceinline__ void leaf_acc(const Blk& leaf, uint64_t h, int u, const LeafCtx& c) {
    const unsigned __int128 y =
        static_cast<unsigned __int128>(h) + ((leaf.lo & 1) ? c.cwo : uint64_t{0});
    const ulonglong2 a = c.acc[u];
    unsigned __int128 A = (static_cast<unsigned __int128>(a.y) << 64) | a.x;
    if (c.neg) A -= y;
    else A += y;
    c.acc[u] = make_ulonglong2(static_cast<uint64_t>(A), static_cast<uint64_t>(A >> 64));
}

// A 128-bit two's-complement accumulator mod p: hi*2^64 + lo with hi a
// small signed count, and 2^64 = 3*2^27 - 4 (mod p).
constexpr uint64_t kTwo64ModP = 402653180ULL;
__device__ __forceinline__ uint64_t acc_mod_p(const ulonglong2& a) {
    const int64_t hi = static_cast<int64_t>(a.y);
    const uint64_t mag = hi < 0 ? static_cast<uint64_t>(-hi) : static_cast<uint64_t>(hi);
    uint64_t t = reduce_p(mag * kTwo64ModP);   // |hi| <= 4t key halves: < 2^55
    if (hi < 0) t = neg_p(t);
    return add_p(reduce_p(a.x), t);
}

__device__ __forceinline__ void leaf_pair(const Blk& a, const Blk& b, int u, LeafCtx& c) {
    uint64_t ha, hb;
    out_hash_x2(a, b, ha, hb);
    leaf_acc(a, ha, u, c);
    leaf_acc(b, hb, u + 1, c);
}

// Binary (w = 1) subtree of SL levels below `node`, leaves u_base.. in order.
template <int SL, int PRG>
struct Dfs1 {
    __device__ __forceinline__ static void run(const Blk& node, const Blk* __restrict__ cw,
                                               const AesSmem* aes, int u, LeafCtx& c) {
        Blk k2[2];
        children<1, PRG>(node, cw, aes, k2);
        const Blk L = k2[0], R = k2[1];
#pragma unroll 1
        for (int i = 0; i < 2; ++i)
            Dfs1<SL - 1, PRG>::run(i ? R : L, cw + 1, aes, u + (i << (SL - 1)), c);
    }
};
template <int PRG>
struct Dfs1<1, PRG> {
    __device__ __forceinline__ static void run(const Blk& node, const Blk* __restrict__ cw,
                                               const AesSmem* aes, int u, LeafCtx& c) {
        Blk k2[2];
        children<1, PRG>(node, cw, aes, k2);
        leaf_pair(k2[0], k2[1], u, c);
    }
};

// m-ary subtree (w > 1).
template <int W, int SL, int PRG>
struct DfsM {
    __device__ __forceinline__ static void run(const Blk& node, const Blk* __restrict__ cw,
                                               const AesSmem* aes, int u, LeafCtx& c) {
        constexpr int M = 1 << W, NK = M - 1;
        Blk kids[M];
        children<W, PRG>(node, cw, aes, kids);
        if constexpr (SL == 1) {
#pragma unroll
            for (int k = 0; k < M; k += 2) leaf_pair(kids[k], kids[k + 1], u + k, c);
        } else {
#pragma unroll 1
            for (int k = 0; k < M; ++k)
                DfsM<W, SL - 1, PRG>::run(kids[k], cw + NK, aes, u + k * (1 << (W * (SL - 1))),
                                          c);
        }
    }
};

// One CTA's tile of the fused leaf kernel: output bin r of launched pair
// z, tile bx.  acc_s is the CTA's dynamic shared memory (blockDim.x rows of
// S + 1 128-bit accumulators).
template <int W, int SL, int PRG>
__device__ __forceinline__ void leaf_gather_tile(
    const Blk* __restrict__ F, const Blk* __restrict__ cws, const uint64_t* __restrict__ cw_out,
    const uint32_t* __restrict__ off, const uint32_t* __restrict__ entries,
    const uint16_t* __restrict__ q_order, const uint16_t* __restrict__ q_slot, int t, int levels,
    int hl, size_t bin, int N, int party, uint64_t* __restrict__ gq, unsigned bx, int r, int z,
    ulonglong2* acc_s, const AesSmem* aes_s) {
    constexpr int M = 1 << W, NK = M - 1;
    constexpr int S = 1 << (W * SL);
    constexpr int STRIDE = S + 1;  // padded accumulator rows: conflict-free
    const int q = q_order[z];
    const int slot = q_slot[z];
    const size_t tile = static_cast<size_t>(blockDim.x) * S;
    const size_t o = static_cast<size_t>(bx) * tile + static_cast<size_t>(threadIdx.x) * S;
    ulonglong2* acc = acc_s + threadIdx.x * STRIDE;
#pragma unroll
    for (int u = 0; u < S; ++u) acc[u] = make_ulonglong2(0, 0);

    const size_t per_key = static_cast<size_t>(1) << (W * hl);
    const uint32_t e0 = off[q * t + r], e1 = off[q * t + r + 1];
    LeafCtx c;
    c.acc = acc;
    for (uint32_t e = e0; e < e1; ++e) {
        const uint32_t ent = __ldg(entries + e);
        const size_t key = ent >> 2;
        const size_t half = (ent >> 1) & 1;
        c.neg = ((ent & 1) != 0) != (party != 0);
        c.cwo = __ldg(cw_out + key);
        const Blk node = ldblk(F + key * per_key + (half * bin + o) / S);
        const Blk* kcw = cws + (key * levels + hl) * NK;
        if constexpr (W == 1) Dfs1<SL, PRG>::run(node, kcw, aes_s, 0, c);
        else DfsM<W, SL, PRG>::run(node, kcw, aes_s, 0, c);
    }
    __syncthreads();
    // Coalesced write-out of the CTA's tile.
    uint64_t* dst = gq + static_cast<size_t>(slot) * N + static_cast<size_t>(r) * bin +
                    static_cast<size_t>(bx) * tile;
    for (size_t e = threadIdx.x; e < tile; e += blockDim.x)
        dst[e] = acc_mod_p(acc_s[(e / S) * STRIDE + (e % S)]);
}

template <int W, int SL, int PRG>
__global__ void __launch_bounds__(256) leaf_gather_kernel(
    const Blk* __restrict__ F, const Blk* __restrict__ cws, const uint64_t* __restrict__ cw_out,
    const uint32_t* __restrict__ off, const uint32_t* __restrict__ entries,
    const uint16_t* __restrict__ q_order, const uint16_t* __restrict__ q_slot, int t, int levels,
    int hl, size_t bin, int N,
    int party, const uint32_t* __restrict__ aes_te, const uint32_t* __restrict__ aes_rk,
    uint64_t* __restrict__ gq) {
    constexpr int NK = (1 << W) - 1, S = 1 << (W * SL);
    extern __shared__ __align__(16) ulonglong2 acc_s[];
    AesSmem& aes_s = *reinterpret_cast<AesSmem*>(acc_s + blockDim.x * (S + 1));
    if constexpr (PRG == kPrgAes) load_aes_smem(aes_s, aes_te, aes_rk, NK);
    leaf_gather_tile<W, SL, PRG>(F, cws, cw_out, off, entries, q_order, q_slot, t, levels, hl, bin,
                                 N, party, gq, blockIdx.x, blockIdx.y, blockIdx.z, acc_s, &aes_s);
}

// The fused leaf kernel over several expansions (one job each, same w, sl,
// PRG and CTA size): CTA b belongs to the job whose CTA range holds b, and
// runs that job's tile (bx, r, z) = its local index in x-fastest order.
template <int W, int SL, int PRG>
__global__ void __launch_bounds__(256) leaf_gather_multi_kernel(
    const LeafJob* __restrict__ jobs, int njobs, const uint32_t* __restrict__ aes_te,
    const uint32_t* __restrict__ aes_rk) {
    constexpr int NK = (1 << W) - 1, S = 1 << (W * SL);
    extern __shared__ __align__(16) ulonglong2 acc_s[];
    AesSmem& aes_s = *reinterpret_cast<AesSmem*>(acc_s + blockDim.x * (S + 1));
    if constexpr (PRG == kPrgAes) load_aes_smem(aes_s, aes_te, aes_rk, NK);
    int k = 0;
    while (k + 1 < njobs && jobs[k + 1].first <= blockIdx.x) ++k;
    const LeafJob& J = jobs[k];
    const unsigned local = blockIdx.x - J.first;
    const unsigned bx = local % J.gx, r = (local / J.gx) % J.gy, z = local / (J.gx * J.gy);
    leaf_gather_tile<W, SL, PRG>(J.F, J.cws, J.cw_out, J.off, J.entries, J.q_order, J.q_slot, J.t,
                                 J.levels, J.hl, J.bin, J.N, J.party, J.gq, bx,
                                 static_cast<int>(r), static_cast<int>(z), acc_s, &aes_s);
}

template <int W, int PRG>
void launch_tops(const Blk* src, int K, int src_lvl, int nlev, int levels, const Blk* cws,
                 const uint32_t* te, const uint32_t* rk, Blk* dst, cudaStream_t st) {
    if (nlev < 0 || nlev >= tops_max_depth<W>()) fail(PCGB_EINVAL, "keyed expansion deeper than the DFS stack");
    const size_t threads = static_cast<size_t>(K) << (W * src_lvl);
    if constexpr (PRG == kPrgAes) {
        // A stage with fewer threads than one wave of PRMT CTAs keeps the
        // replicated table in small CTAs, spread over every SM.
        if (threads >= aes_prmt_wave()) {
            if constexpr (W == 1) {
                if (nlev >= 1 && nlev <= kTopsFixedMax) {
                    switch (nlev) {
#define PCGB_TF(D)                                                                              \
    case D:                                                                                     \
        PCGB_CK(cudaFuncSetAttribute(expand_tops_prmt_fixed_kernel<D>,                          \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,               \
                                     static_cast<int>(kAesPrmtSmemBytes)));                     \
        expand_tops_prmt_fixed_kernel<D><<<aes_prmt_grid(threads), kAesPrmtThreads,             \
                                           kAesPrmtSmemBytes, st>>>(src, K, src_lvl, levels,    \
                                                                    cws, te, rk, dst);          \
        break;
                        PCGB_TF(1) PCGB_TF(2) PCGB_TF(3) PCGB_TF(4)
                        PCGB_TF(5) PCGB_TF(6) PCGB_TF(7) PCGB_TF(8)
#undef PCGB_TF
                        default: break;
                    }
                    PCGB_POST_LAUNCH();
                    return;
                }
            }
            PCGB_CK(cudaFuncSetAttribute(expand_tops_prmt_kernel<W>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kAesPrmtSmemBytes)));
            expand_tops_prmt_kernel<W><<<aes_prmt_grid(threads), kAesPrmtThreads,
                                         kAesPrmtSmemBytes, st>>>(src, K, src_lvl, nlev, levels,
                                                                  cws, te, rk, dst);
            PCGB_POST_LAUNCH();
            return;
        }
    }
    const int TPB = 128;
    const unsigned grid = static_cast<unsigned>((threads + TPB - 1) / TPB);
    if constexpr (PRG == kPrgChaCha && W == 1) {
        if (nlev >= 1 && nlev <= kTopsFixedMax) {
            switch (nlev) {
#define PCGB_TF(D)                                                                            \
    case D:                                                                                   \
        expand_tops_fixed_kernel<D><<<grid, TPB, 0, st>>>(src, K, src_lvl, levels, cws, dst); \
        break;
                PCGB_TF(1) PCGB_TF(2) PCGB_TF(3) PCGB_TF(4)
                PCGB_TF(5) PCGB_TF(6) PCGB_TF(7) PCGB_TF(8)
#undef PCGB_TF
                default: break;
            }
            PCGB_POST_LAUNCH();
            return;
        }
    }
    const size_t smem = PRG == kPrgAes ? sizeof(AesSmem) : 0;
    expand_tops_kernel<W, PRG><<<grid, TPB, smem, st>>>(src, K, src_lvl, nlev, levels, cws, te,
                                                        rk, dst);
    PCGB_POST_LAUNCH();
}

template <int W, int PRG>
void tops_dispatch(int K, int levels, const Blk* roots, const Blk* cws, const uint32_t* te,
                   const uint32_t* rk, int to_level, Blk* out, Blk* scratch, cudaStream_t st) {
    // Stages (tops_stages): intermediate levels alternate between the two
    // halves of the scratch, the last stage writes `out`.
    const std::vector<int> b = tops_stages(K, W, to_level);
    const size_t half = b.size() > 2 ? (static_cast<size_t>(K) << (W * b[b.size() - 2])) : 0;
    const Blk* src = roots;
    for (size_t k = 0; k + 1 < b.size(); ++k) {
        Blk* dst = (k + 2 == b.size()) ? out : scratch + (k % 2) * half;
        launch_tops<W, PRG>(src, K, b[k], b[k + 1] - b[k], levels, cws, te, rk, dst, st);
        src = dst;
    }
}

// Key `id` of an expansion's dealer (below): roots of both parties, the
// per-level CWs and the output CW.
template <int W, int PRG>
__device__ __forceinline__ void deal_one(int id, uint64_t seed, int c, int t, int n, uint64_t bin,
                                         Blk* roots0, Blk* roots1, Blk* cws, uint64_t* cw_out,
                                         const AesSmem* aes_s, uint64_t r2) {
    constexpr int M = 1 << W, NK = M - 1;
    const int blk = id / (t * t), rr = id % (t * t);
    const int ii = blk / c, jj = blk % c, kk = rr / t, ll = rr % t;
    const uint64_t alpha = synth_offset(seed, 0, static_cast<uint64_t>(ii) * t + kk, bin) +
                           synth_offset(seed, 1, static_cast<uint64_t>(jj) * t + ll, bin);
    const uint64_t v0 = synth_value(seed, 0, static_cast<uint64_t>(ii) * t + kk);
    const uint64_t v1 = synth_value(seed, 1, static_cast<uint64_t>(jj) * t + ll);
    const uint64_t beta = mont_mul(mont_mul(v0, v1), r2);
    const Blk delta{synth_rnd(seed, kDomDelta, id) | 1, synth_rnd(seed, kDomDelta + 1, id)};
    Blk p0{synth_rnd(seed, kDomRoot, id), synth_rnd(seed, kDomRoot + 1, id)};
    Blk p1{p0.lo ^ delta.lo, p0.hi ^ delta.hi};
    roots0[id] = p0;
    roots1[id] = p1;
    const int levels = n / W;
    Blk* kcw = cws + static_cast<size_t>(id) * levels * NK;
    for (int i = 0; i < levels; ++i) {
        const int digit = static_cast<int>((alpha >> (n - W * (i + 1))) & NK);
        Blk h0[NK], h1[NK];
        hash_raw<W, PRG>(p0, aes_s, h0);
        hash_raw<W, PRG>(p1, aes_s, h1);
        Blk cwf{0, 0}, cwd{0, 0};
        Blk x0{p0.lo, p0.hi}, x1{p1.lo, p1.hi};
        Blk n0{0, 0}, n1{0, 0};
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            Blk cw{h0[k].lo ^ h1[k].lo, h0[k].hi ^ h1[k].hi};
            if (digit == k) {
                cw.lo ^= delta.lo; cw.hi ^= delta.hi;
                cwd = cw; n0 = h0[k]; n1 = h1[k];
            }
            kcw[i * NK + k] = cw;
            cwf.lo ^= cw.lo; cwf.hi ^= cw.hi;
            x0.lo ^= h0[k].lo; x0.hi ^= h0[k].hi;
            x1.lo ^= h1[k].lo; x1.hi ^= h1[k].hi;
        }
        if (digit == NK) { cwd = cwf; n0 = x0; n1 = x1; }
        if (p0.lo & 1) { n0.lo ^= cwd.lo; n0.hi ^= cwd.hi; }
        if (p1.lo & 1) { n1.lo ^= cwd.lo; n1.hi ^= cwd.hi; }
        p0 = n0;
        p1 = n1;
    }
    const uint64_t C0 = reduce_p(out_hash_lo64(p0.lo, p0.hi));
    const uint64_t C1 = reduce_p(out_hash_lo64(p1.lo, p1.hi));
    const uint64_t Bv = add_p(sub_p(C1, C0), beta);
    const int A = static_cast<int>(p0.lo & 1) - static_cast<int>(p1.lo & 1);
    cw_out[id] = A == 1 ? Bv : (A == -1 ? neg_p(Bv) : 0);
}

template <int W, int PRG>
__global__ void deal_kernel(uint64_t seed, int c, int t, int n, uint64_t bin, Blk* roots0,
                            Blk* roots1, Blk* cws, uint64_t* cw_out, const uint32_t* aes_te,
                            const uint32_t* aes_rk, uint64_t r2) {
    constexpr int NK = (1 << W) - 1;
    extern __shared__ __align__(16) uint64_t deal_dsm[];
    AesSmem& aes_s = *reinterpret_cast<AesSmem*>(deal_dsm);
    if constexpr (PRG == kPrgAes) load_aes_smem(aes_s, aes_te, aes_rk, NK);
    const int K = c * c * t * t;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= K) return;
    deal_one<W, PRG>(id, seed, c, t, n, bin, roots0, roots1, cws, cw_out, &aes_s, r2);
}

// The dealer of several expansions (ChaCha8, one w) in one launch: CTA b
// deals keys of the job whose CTA range holds b.
template <int W>
__global__ void deal_multi_kernel(const DealJob* __restrict__ jobs, int njobs, uint64_t r2) {
    int k = 0;
    while (k + 1 < njobs && jobs[k + 1].first <= blockIdx.x) ++k;
    const DealJob& J = jobs[k];
    const int id = static_cast<int>((blockIdx.x - J.first) * blockDim.x + threadIdx.x);
    if (id >= J.c * J.c * J.t * J.t) return;
    deal_one<W, kPrgChaCha>(id, J.seed, J.c, J.t, J.n, J.bin, J.roots0, J.roots1, J.cws,
                            J.cw_out, nullptr, r2);
}


// ---- per-PRG host launchers (instantiated once per PRG in its own TU) -----
template <int PRG>
void tops_for_prg(int K, int levels, int w, const Blk* roots, const Blk* cws, const uint32_t* te,
                  const uint32_t* rk, int to_level, Blk* out, Blk* scratch, cudaStream_t st) {
    switch (w) {
        case 1: tops_dispatch<1, PRG>(K, levels, roots, cws, te, rk, to_level, out, scratch, st); break;
        case 2: tops_dispatch<2, PRG>(K, levels, roots, cws, te, rk, to_level, out, scratch, st); break;
        case 3: tops_dispatch<3, PRG>(K, levels, roots, cws, te, rk, to_level, out, scratch, st); break;
        case 4: tops_dispatch<4, PRG>(K, levels, roots, cws, te, rk, to_level, out, scratch, st); break;
        default: fail(PCGB_EINVAL, "w must be in [1,4]");
    }
}

template <int W, int PRG>
void tops_multi_launch(const std::vector<TopsJob>& jobs, TopsJob* d_jobs,
                       unsigned long long total, const uint32_t* te, const uint32_t* rk,
                       cudaStream_t st) {
    for (const TopsJob& J : jobs)
        if (J.nlev < 0 || J.nlev >= tops_max_depth<W>())
            fail(PCGB_EINVAL, "keyed expansion deeper than the DFS stack");
    const int TPB = 128;
    const unsigned long long cap = static_cast<unsigned long long>(sm_count()) * 8;  // persistent
    if constexpr (PRG == kPrgChaCha && W == 1) {
        // One launch per distinct depth in the stage, each with the
        // compile-time walk of that depth (its own register budget); the
        // jobs of a depth are contiguous in the table, their thread indices
        // counted from the first of them.
        std::vector<TopsJob> byd(jobs);
        std::stable_sort(byd.begin(), byd.end(),
                         [](const TopsJob& x, const TopsJob& y) { return x.nlev < y.nlev; });
        std::vector<size_t> seg{0};
        for (size_t i = 1; i < byd.size(); ++i)
            if (byd[i].nlev != byd[i - 1].nlev) seg.push_back(i);
        seg.push_back(byd.size());
        std::vector<unsigned long long> seg_total(seg.size() - 1, 0);
        for (size_t k = 0; k + 1 < seg.size(); ++k)
            for (size_t i = seg[k]; i < seg[k + 1]; ++i) {
                byd[i].first = seg_total[k];
                seg_total[k] += static_cast<unsigned long long>(byd[i].K) << byd[i].src_lvl;
            }
        PCGB_CK(cudaMemcpyAsync(d_jobs, byd.data(), byd.size() * sizeof(TopsJob),
                                cudaMemcpyHostToDevice, st));
        for (size_t k = 0; k + 1 < seg.size(); ++k) {
            const unsigned long long tot = seg_total[k];
            if (tot == 0) continue;
            const unsigned long long blocks = (tot + TPB - 1) / TPB;
            const unsigned grid = static_cast<unsigned>(blocks < cap ? blocks : cap);
            const TopsJob* dj = d_jobs + seg[k];
            const int nj = static_cast<int>(seg[k + 1] - seg[k]);
            switch (byd[seg[k]].nlev) {
#define PCGB_TF(D)                                                                         \
    case D: expand_tops_multi_depth_kernel<D><<<grid, TPB, 0, st>>>(dj, nj, tot); break;
                PCGB_TF(1) PCGB_TF(2) PCGB_TF(3) PCGB_TF(4)
                PCGB_TF(5) PCGB_TF(6) PCGB_TF(7) PCGB_TF(8)
#undef PCGB_TF
                default: expand_tops_multi_fixed_kernel<<<grid, TPB, 0, st>>>(dj, nj, tot);
            }
            PCGB_POST_LAUNCH();
        }
        return;
    }
    PCGB_CK(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(TopsJob),
                            cudaMemcpyHostToDevice, st));
    if constexpr (PRG == kPrgAes) {
        if (total >= aes_prmt_wave()) {   // as launch_tops
            PCGB_CK(cudaFuncSetAttribute(expand_tops_multi_prmt_kernel<W>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kAesPrmtSmemBytes)));
            expand_tops_multi_prmt_kernel<W><<<aes_prmt_grid(total), kAesPrmtThreads,
                                               kAesPrmtSmemBytes, st>>>(
                d_jobs, static_cast<int>(jobs.size()), total, te, rk);
            PCGB_POST_LAUNCH();
            return;
        }
    }
    const size_t smem = PRG == kPrgAes ? sizeof(AesSmem) : 0;
    const unsigned long long blocks = (total + TPB - 1) / TPB;
    const unsigned grid = static_cast<unsigned>(blocks < cap ? blocks : cap);
    expand_tops_multi_kernel<W, PRG><<<grid, TPB, smem, st>>>(d_jobs, static_cast<int>(jobs.size()),
                                                              total, te, rk);
    PCGB_POST_LAUNCH();
}

template <int PRG>
void tops_multi_for_prg(int w, const std::vector<TopsJob>& jobs, TopsJob* d_jobs,
                        unsigned long long total, const uint32_t* te, const uint32_t* rk,
                        cudaStream_t st) {
    switch (w) {
        case 1: tops_multi_launch<1, PRG>(jobs, d_jobs, total, te, rk, st); break;
        case 2: tops_multi_launch<2, PRG>(jobs, d_jobs, total, te, rk, st); break;
        case 3: tops_multi_launch<3, PRG>(jobs, d_jobs, total, te, rk, st); break;
        case 4: tops_multi_launch<4, PRG>(jobs, d_jobs, total, te, rk, st); break;
        default: fail(PCGB_EINVAL, "w must be in [1,4]");
    }
}

template <int W, int SL, int PRG>
void leaf_one(const LeafLaunch& L) {
    auto kern = leaf_gather_kernel<W, SL, PRG>;
    if (L.smem > 48 * 1024)
        PCGB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(L.smem)));
    kern<<<L.grid, L.tpb, L.smem, L.st>>>(L.F, L.cws, L.cw_out, L.off, L.entries, L.q_order,
                                         L.q_slot, L.t,
                                         L.levels, L.hl, L.bin, L.N, L.party, L.te, L.rk, L.gq);
    PCGB_POST_LAUNCH();
}

template <int W, int SL, int PRG>
void leaf_multi_one(const LeafJob* d_jobs, int njobs, unsigned ctas, int tpb, size_t smem,
                    const uint32_t* te, const uint32_t* rk, cudaStream_t st) {
    auto kern = leaf_gather_multi_kernel<W, SL, PRG>;
    if (smem > 48 * 1024)
        PCGB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    kern<<<ctas, tpb, smem, st>>>(d_jobs, njobs, te, rk);
    PCGB_POST_LAUNCH();
}

template <int PRG>
void leaf_multi_for_prg(int w, int sl, const LeafJob* d_jobs, int njobs, unsigned ctas, int tpb,
                        size_t smem, const uint32_t* te, const uint32_t* rk, cudaStream_t st) {
    switch (w * 8 + sl) {
#define PCGB_LM(W_, SL_)                                                              \
    case W_ * 8 + SL_:                                                                \
        leaf_multi_one<W_, SL_, PRG>(d_jobs, njobs, ctas, tpb, smem, te, rk, st); \
        break;
        PCGB_LM(1, 4) PCGB_LM(1, 3) PCGB_LM(1, 2) PCGB_LM(1, 1)
        PCGB_LM(2, 2) PCGB_LM(2, 1) PCGB_LM(3, 1) PCGB_LM(4, 1)
#undef PCGB_LM
        default: fail(PCGB_EINVAL, "unsupported (w, sl) for the leaf kernel");
    }
}

template <int PRG>
void leaf_for_prg(int w, int sl, const LeafLaunch& L) {
    switch (w * 8 + sl) {
        case 1 * 8 + 4: leaf_one<1, 4, PRG>(L); break;
        case 1 * 8 + 3: leaf_one<1, 3, PRG>(L); break;
        case 1 * 8 + 2: leaf_one<1, 2, PRG>(L); break;
        case 1 * 8 + 1: leaf_one<1, 1, PRG>(L); break;
        case 2 * 8 + 2: leaf_one<2, 2, PRG>(L); break;
        case 2 * 8 + 1: leaf_one<2, 1, PRG>(L); break;
        case 3 * 8 + 1: leaf_one<3, 1, PRG>(L); break;
        case 4 * 8 + 1: leaf_one<4, 1, PRG>(L); break;
        default: fail(PCGB_EINVAL, "unsupported (w, sl) for the leaf kernel");
    }
}

inline void deal_multi_for_chacha(int w, const DealJob* d_jobs, int njobs, unsigned ctas, uint64_t r2,
                           cudaStream_t st) {
    switch (w) {
        case 1: deal_multi_kernel<1><<<ctas, 128, 0, st>>>(d_jobs, njobs, r2); break;
        case 2: deal_multi_kernel<2><<<ctas, 128, 0, st>>>(d_jobs, njobs, r2); break;
        case 3: deal_multi_kernel<3><<<ctas, 128, 0, st>>>(d_jobs, njobs, r2); break;
        case 4: deal_multi_kernel<4><<<ctas, 128, 0, st>>>(d_jobs, njobs, r2); break;
        default: fail(PCGB_EINVAL, "w must be in [1,4]");
    }
    PCGB_POST_LAUNCH();
}

template <int PRG>
void deal_for_prg(int w, unsigned grid, size_t smem, uint64_t seed, int c, int t, int n,
                  uint64_t bin, Blk* roots0, Blk* roots1, Blk* cws, uint64_t* cw_out,
                  const uint32_t* te, const uint32_t* rk, uint64_t r2, cudaStream_t st) {
    switch (w) {
#define PCGB_DEAL(W_)                                                                          \
    case W_:                                                                                   \
        deal_kernel<W_, PRG><<<grid, 128, smem, st>>>(seed, c, t, n, bin, roots0, roots1, cws, \
                                                      cw_out, te, rk, r2);                     \
        break;
        PCGB_DEAL(1)
        PCGB_DEAL(2)
        PCGB_DEAL(3)
        PCGB_DEAL(4)
#undef PCGB_DEAL
        default: fail(PCGB_EINVAL, "w must be in [1,4]");
    }
    PCGB_POST_LAUNCH();
}

}  // namespace
}  // namespace pcgb

#endif
