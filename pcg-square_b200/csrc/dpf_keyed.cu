// Keyed DPF: host-side dispatch and the gather plan.  The kernels live in
// dpf_keyed_impl.cuh (instantiated per PRG by dpf_keyed_chacha.cu and
// dpf_keyed_aes.cu); see that header for the algorithm.
#include "pcgb_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

#include "field.cuh"

namespace pcgb {

std::vector<int> tops_stages(int K, int w, int to_level) {
    std::vector<int> b{0};
    int l = 0;
    while (l < to_level) {
        if ((static_cast<size_t>(K) << (w * l)) >= kTopsStage2Threads) {
            b.push_back(to_level);
            break;
        }
        int s = 1;
        while (l + s < to_level && (static_cast<size_t>(K) << (w * (l + s))) < kTopsStage2Threads &&
               (1 << (w * (s + 1))) <= 32)
            ++s;
        l += s;
        b.push_back(l);
    }
    if (w == 1) {
        // Split deeper stages into pieces of at most kTopsFixedLevels, the
        // last piece the full length: [7, 16) becomes [7, 8), [8, 16).
        std::vector<int> out{b[0]};
        for (size_t i = 1; i < b.size(); ++i) {
            std::vector<int> cuts;
            for (int e = b[i]; e - out.back() > kTopsFixedLevels; e -= kTopsFixedLevels)
                cuts.push_back(e - kTopsFixedLevels);
            out.insert(out.end(), cuts.rbegin(), cuts.rend());
            out.push_back(b[i]);
        }
        b = out;
    }
    return b;
}

// Two ping-pong halves, each holding the largest intermediate level.
size_t keyed_tops_scratch_nodes(int K, int w, int to_level) {
    const std::vector<int> b = tops_stages(K, w, to_level);
    if (b.size() <= 2) return 0;
    return 2 * (static_cast<size_t>(K) << (w * b[b.size() - 2]));
}

void keyed_expand_tops(int K, int n, int w, int prg, const Blk* roots, const Blk* cws,
                       const uint32_t* d_aes_rk, int to_level, Blk* out, Blk* scratch,
                       cudaStream_t st) {
    const int levels = n / w;
    if (prg == PCGB_PRG_AES)
        keyed_tops_aes(K, levels, w, roots, cws, aes_te_table_device(), d_aes_rk, to_level, out,
                       scratch, st);
    else
        keyed_tops_chacha(K, levels, w, roots, cws, nullptr, nullptr, to_level, out, scratch, st);
}

// Stage plan of a multi-group walk: every group walks its own geometric
// stages (tops_stages) down to its own target level with its own ping-pong
// scratch; launch s carries stage s of every group that has one, so the
// whole batch takes as many launches as its deepest plan has stages.
// scratch[g] (2 * keyed_tops_scratch_nodes-sized halves) may be null, in
// which case the scratch comes from the library's pool.
void keyed_tops_multi(int groups, const int* K, const int* n, const int* to_level, int w, int prg,
                      const Blk* const* roots, const Blk* const* cws, const uint32_t* d_rk,
                      Blk* const* out, Blk* const* scratch, cudaStream_t st) {
    if (groups <= 0) return;
    if (!K || !n || !to_level || !roots || !cws || !out)
        fail(PCGB_EINVAL, "keyed eval multi: null array");
    if (w < 1 || w > 4) fail(PCGB_EINVAL, "keyed eval multi: w must be in [1,4]");
    if (prg == PCGB_PRG_AES && !d_rk) fail(PCGB_EINVAL, "keyed eval multi: AES needs round keys");
    struct Plan {
        std::vector<int> b;
        size_t half = 0;
        Blk* base = nullptr;
        int levels = 0;
    };
    std::vector<Plan> plan(groups);
    size_t pool_nodes = 0;
    size_t stages = 0;
    for (int g = 0; g < groups; ++g) {
        if (K[g] < 0) fail(PCGB_EINVAL, "keyed eval multi: negative key count");
        if (K[g] == 0) continue;
        if (n[g] < 1 || n[g] > 30 || n[g] % w) fail(PCGB_EINVAL, "keyed eval multi: bad (n, w)");
        if (to_level[g] < 0 || to_level[g] > n[g] / w)
            fail(PCGB_EINVAL, "keyed eval multi: bad target level");
        if (!roots[g] || !cws[g] || !out[g]) fail(PCGB_EINVAL, "keyed eval multi: null group buffer");
        Plan& P = plan[g];
        P.levels = n[g] / w;
        P.b = tops_stages(K[g], w, to_level[g]);
        if (P.b.size() > 2) P.half = static_cast<size_t>(K[g]) << (w * P.b[P.b.size() - 2]);
        if (scratch && scratch[g]) P.base = scratch[g];
        else pool_nodes += 2 * P.half;
        stages = std::max(stages, P.b.size() - 1);
    }
    if (stages == 0) return;
    Blk* pool = pool_nodes ? static_cast<Blk*>(pool_alloc(pool_nodes * sizeof(Blk), st)) : nullptr;
    size_t o = 0;
    for (int g = 0; g < groups; ++g) {
        Plan& P = plan[g];
        if (K[g] == 0 || P.base || P.half == 0) continue;
        P.base = pool + o;
        o += 2 * P.half;
    }
    TopsJob* d_jobs = static_cast<TopsJob*>(pool_alloc(groups * sizeof(TopsJob), st));
    try {
        for (size_t s = 0; s < stages; ++s) {
            std::vector<TopsJob> jobs;
            unsigned long long total = 0;
            for (int g = 0; g < groups; ++g) {
                const Plan& P = plan[g];
                if (K[g] == 0 || s + 1 >= P.b.size()) continue;
                TopsJob J;
                J.src = s == 0 ? roots[g] : P.base + ((s - 1) % 2) * P.half;
                J.dst = (s + 2 == P.b.size()) ? out[g] : P.base + (s % 2) * P.half;
                J.cws = cws[g];
                J.first = total;
                J.K = K[g];
                J.src_lvl = P.b[s];
                J.nlev = P.b[s + 1] - P.b[s];
                J.levels = P.levels;
                total += static_cast<unsigned long long>(K[g]) << (w * P.b[s]);
                jobs.push_back(J);
            }
            if (prg == PCGB_PRG_AES)
                keyed_tops_multi_aes(w, jobs, d_jobs, total, aes_te_table_device(), d_rk, st);
            else
                keyed_tops_multi_chacha(w, jobs, d_jobs, total, st);
        }
    } catch (...) {
        if (pool) cudaFreeAsync(pool, st);
        cudaFreeAsync(d_jobs, st);
        throw;
    }
    if (pool) PCGB_CK(cudaFreeAsync(pool, st));
    PCGB_CK(cudaFreeAsync(d_jobs, st));
}

// Full-domain evaluation of key groups of different domains: the multi-group
// walk down to every group's last level.
void keyed_full_eval_multi(int groups, const int* K, const int* n, int w, int prg,
                           const Blk* const* roots, const Blk* const* cws, const uint32_t* d_rk,
                           Blk* const* leaves, cudaStream_t st) {
    if (groups <= 0) return;
    if (!n) fail(PCGB_EINVAL, "keyed eval multi: null array");
    std::vector<int> to(groups);
    for (int g = 0; g < groups; ++g) to[g] = (w >= 1 && w <= 4) ? n[g] / w : 0;
    keyed_tops_multi(groups, K, n, to.data(), w, prg, roots, cws, d_rk, leaves, nullptr, st);
}

// Gather plan: for pair q = (i <= j) and output bin r, the key halves of
// blocks (i,j) and (j,i) whose leaves land in [r*bin, (r+1)*bin) after the
// X^N = -1 fold.  Key (kk, ll) of a block covers pre-fold positions
// (kk+ll)*bin + [0, 2*bin) (pcg_ole_impl.h:435-444), so with s = kk+ll:
//   s = r     -> first half,  kept;   s = r-1   -> second half, kept;
//   s = r+t   -> first half,  negated; s = r+t-1 -> second half, negated.
int leaf_sl_max(int n, int w) {
    // Leaves per thread: 16 for w in {1,2,4}, 8 for w = 3; fewer when the
    // half domain is smaller.
    int sl = (w == 3) ? 1 : 4 / w;
    while (sl > 1 && w * sl > n - 1) --sl;
    if (w * sl > n - 1) fail(PCGB_EINVAL, "domain too small for the fused leaf kernel");
    return sl;
}

void gather_plan_build(GatherPlan& gp, int N, int c, int t, int n, int w, int rank, int world) {
    gather_plan_free(gp);
    if (world < 1 || rank < 0 || rank >= world) fail(PCGB_EINVAL, "expander: bad shard rank/world");
    gp.N = N; gp.c = c; gp.t = t; gp.n = n; gp.w = w;
    gp.rank = rank; gp.world = world;
    const int levels = n / w;
    const int sl = leaf_sl_max(n, w);
    gp.sl = sl;
    gp.S = 1 << (w * sl);
    gp.hl = levels - sl;
    std::vector<uint32_t> off, ent;
    std::vector<uint32_t> pair_ij;
    int Q = 0;
    off.push_back(0);
    const uint32_t tt = static_cast<uint32_t>(t) * t;
    for (int i = 0; i < c; ++i)
        for (int j = i; j < c; ++j) {
            pair_ij.push_back(static_cast<uint32_t>(i * c + j));
            for (int r = 0; r < t; ++r) {
                const int blocks[2] = {i * c + j, j * c + i};
                for (int bi = 0; bi < (i == j ? 1 : 2); ++bi) {
                    const uint32_t base = static_cast<uint32_t>(blocks[bi]) * tt;
                    const int svals[4] = {r, r - 1, r + t, r + t - 1};
                    const int halves[4] = {0, 1, 0, 1};
                    const int folds[4] = {0, 0, 1, 1};
                    for (int v = 0; v < 4; ++v) {
                        const int s = svals[v];
                        if (s < 0 || s > 2 * t - 2) continue;
                        for (int kk = 0; kk < t; ++kk) {
                            const int ll = s - kk;
                            if (ll < 0 || ll >= t) continue;
                            const uint32_t key = base + static_cast<uint32_t>(kk * t + ll);
                            ent.push_back(key << 2 | static_cast<uint32_t>(halves[v]) << 1 |
                                          static_cast<uint32_t>(folds[v]));
                        }
                    }
                }
                off.push_back(static_cast<uint32_t>(ent.size()));
            }
            ++Q;
        }
    gp.Q = Q;
    gp.n_entries = static_cast<int>(ent.size());
    // Heavy pairs (i != j carry two blocks) first so the tail is short.
    std::vector<int> heavy_first;
    for (int q = 0; q < Q; ++q) if ((pair_ij[q] / c) != (pair_ij[q] % c)) heavy_first.push_back(q);
    for (int q = 0; q < Q; ++q) if ((pair_ij[q] / c) == (pair_ij[q] % c)) heavy_first.push_back(q);
    // Shards: longest-first greedy by block count, ties to the lowest rank.
    std::vector<int> owner(Q, 0), load(world, 0);
    for (int q : heavy_first) {
        const int wgt = (pair_ij[q] / c) != (pair_ij[q] % c) ? 2 : 1;
        int best = 0;
        for (int r = 1; r < world; ++r) if (load[r] < load[best]) best = r;
        owner[q] = best;
        load[best] += wgt;
    }
    gp.shard_pairs.clear();
    for (int q = 0; q < Q; ++q) if (owner[q] == rank) gp.shard_pairs.push_back(q);
    gp.Qs = static_cast<int>(gp.shard_pairs.size());
    std::vector<uint16_t> order, slot;
    for (int q : heavy_first) {
        if (owner[q] != rank) continue;
        order.push_back(static_cast<uint16_t>(q));
        const auto it = std::find(gp.shard_pairs.begin(), gp.shard_pairs.end(), q);
        slot.push_back(static_cast<uint16_t>(it - gp.shard_pairs.begin()));
    }
    PCGB_CK(cudaMalloc(&gp.d_off, off.size() * sizeof(uint32_t)));
    PCGB_CK(cudaMalloc(&gp.d_entries, std::max<size_t>(ent.size(), 1) * sizeof(uint32_t)));
    PCGB_CK(cudaMalloc(&gp.d_qorder, std::max<size_t>(order.size(), 1) * sizeof(uint16_t)));
    PCGB_CK(cudaMalloc(&gp.d_qslot, std::max<size_t>(slot.size(), 1) * sizeof(uint16_t)));
    upload_blocking(gp.d_off, off.data(), off.size() * sizeof(uint32_t));
    if (!ent.empty())
        upload_blocking(gp.d_entries, ent.data(), ent.size() * sizeof(uint32_t));
    if (!order.empty()) {
        upload_blocking(gp.d_qorder, order.data(), order.size() * sizeof(uint16_t));
        upload_blocking(gp.d_qslot, slot.data(), slot.size() * sizeof(uint16_t));
    }
    gp.pair_ij = pair_ij;
}

void gather_plan_free(GatherPlan& gp) {
    if (gp.d_off) cudaFree(gp.d_off);
    if (gp.d_entries) cudaFree(gp.d_entries);
    if (gp.d_qorder) cudaFree(gp.d_qorder);
    if (gp.d_qslot) cudaFree(gp.d_qslot);
    gp.d_off = nullptr; gp.d_entries = nullptr; gp.d_qorder = nullptr; gp.d_qslot = nullptr;
}

void keyed_leaf_gather(const GatherPlan& gp, int party, int prg, const Blk* F, const Blk* cws,
                       const uint64_t* cw_out, const uint32_t* d_aes_rk, uint64_t* gq,
                       cudaStream_t st) {
    LeafLaunch L;
    L.levels = gp.n / gp.w;
    L.bin = static_cast<size_t>(gp.N) / gp.t;
    int tpb = gp.tpb > 0 ? gp.tpb : 256;
    while (tpb > 1 && static_cast<size_t>(tpb) * gp.S > L.bin) tpb >>= 1;
    if (static_cast<size_t>(tpb) * gp.S > L.bin) fail(PCGB_EINVAL, "bin smaller than one tile");
    L.tpb = tpb;
    if (gp.Qs == 0) return;   // a shard with no pairs
    L.grid = dim3(static_cast<unsigned>(L.bin / (static_cast<size_t>(tpb) * gp.S)),
                  static_cast<unsigned>(gp.t), static_cast<unsigned>(gp.Qs));
    L.smem = static_cast<size_t>(tpb) * (gp.S + 1) * 2 * sizeof(uint64_t) +
             (prg == PCGB_PRG_AES ? keyed_aes_smem_bytes_aes() : 0);
    L.st = st;
    L.F = F; L.cws = cws; L.cw_out = cw_out;
    L.off = gp.d_off; L.entries = gp.d_entries; L.q_order = gp.d_qorder; L.q_slot = gp.d_qslot;
    L.t = gp.t; L.hl = gp.hl; L.N = gp.N; L.party = party;
    L.rk = d_aes_rk; L.gq = gq;
    if (prg == PCGB_PRG_AES) {
        L.te = aes_te_table_device();
        keyed_leaf_aes(gp.w, gp.sl, L);
    } else {
        keyed_leaf_chacha(gp.w, gp.sl, L);
    }
}

void deal_keys_launch(int N, int c, int t, int n, int w, int prg, uint64_t seed,
                      const uint32_t* d_rk, Blk* roots0, Blk* roots1, Blk* cws, uint64_t* cw_out,
                      cudaStream_t st) {
    const int K = c * c * t * t;
    const uint64_t bin = static_cast<uint64_t>(N / t);
    const unsigned grid = static_cast<unsigned>((K + 127) / 128);
    if (prg == PCGB_PRG_AES)
        keyed_deal_aes(w, grid, keyed_aes_smem_bytes_aes(), seed, c, t, n, bin, roots0, roots1, cws,
                       cw_out, aes_te_table_device(), d_rk, r2_mod_p(), st);
    else
        keyed_deal_chacha(w, grid, 0, seed, c, t, n, bin, roots0, roots1, cws, cw_out, nullptr,
                          nullptr, r2_mod_p(), st);
}

}  // namespace pcgb
