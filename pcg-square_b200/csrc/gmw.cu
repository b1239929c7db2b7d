// Boolean preprocessing of the interactive DPF on the device: two-party GMW
// evaluation of the Kogge-Stone position adder (CPU_baseline/bool_circuit/
// adder.h:22-63, used by CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:118-159) and
// of the DltSft circuit [digit_i(alpha) == k] * Delta
// (CPU_baseline/half_tree_dpf/dpf.cpp:171-283).  AND triples are inputs: the
// OT layer that makes them stays outside the library.
//
// Bit-sliced layout.  One circuit is evaluated for B instances at once; a
// wire is a row of W = ceil(B/32) words, instance b being bit b % 32 of word
// b / 32, and every gate works on whole rows.  Shares are XOR shares.
//
// AND gate with a triple (a, b, c = a & b, each XOR-shared; the gate
// algebra of CPU_baseline/bool_circuit/circuit.cpp:326-368): each party
// opens d = x ^ a and e = y ^ b; with D = d0 ^ d1, E = e0 ^ e1 its output
// share is c ^ (D & b) ^ (E & a), and party 0 adds D & E.  NOT flips party
// 0's share; XOR is local.  All AND gates of one AND depth share one
// message exchange, so a circuit costs one exchange per AND level.
//
// Input sharing: each party's private input bits enter as the trivial
// sharing (its own bits, zero for the peer), which the first AND layer's
// triples mask; the reference's separate masking round is not needed.
#include <algorithm>

#include "pcgb_internal.h"

namespace pcgb {
namespace {

constexpr int kTpb = 256;
enum GateKind : int { kXor = 0, kNot = 1, kAnd = 2 };

struct Gate {
    int x, y, z, kind;
};

unsigned grid_for(size_t n) { return static_cast<unsigned>((n + kTpb - 1) / kTpb); }

// ---- kernels: one thread per (gate, word) ------------------------------
__global__ void local_kernel(uint32_t* __restrict__ wires, int W, const Gate* __restrict__ g,
                             size_t count, int party) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count * W) return;
    const Gate G = g[i / W];
    const size_t w = i % W;
    uint32_t v = wires[static_cast<size_t>(G.x) * W + w];
    if (G.kind == kXor)
        v ^= wires[static_cast<size_t>(G.y) * W + w];
    else if (party == 0)
        v = ~v;
    wires[static_cast<size_t>(G.z) * W + w] = v;
}

// de = [d rows | e rows], count rows each.
__global__ void and_open_kernel(const uint32_t* __restrict__ wires, int W,
                                const Gate* __restrict__ g, size_t count,
                                const uint32_t* __restrict__ ta, const uint32_t* __restrict__ tb,
                                uint32_t* __restrict__ de) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n = count * W;
    if (i >= n) return;
    const Gate G = g[i / W];
    const size_t w = i % W;
    de[i] = wires[static_cast<size_t>(G.x) * W + w] ^ ta[i];
    de[n + i] = wires[static_cast<size_t>(G.y) * W + w] ^ tb[i];
}

__global__ void and_close_kernel(int party, uint32_t* __restrict__ wires, int W,
                                 const Gate* __restrict__ g, size_t count,
                                 const uint32_t* __restrict__ de_my,
                                 const uint32_t* __restrict__ de_peer,
                                 const uint32_t* __restrict__ ta, const uint32_t* __restrict__ tb,
                                 const uint32_t* __restrict__ tc) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n = count * W;
    if (i >= n) return;
    const uint32_t D = de_my[i] ^ de_peer[i];
    const uint32_t E = de_my[n + i] ^ de_peer[n + i];
    uint32_t v = tc[i] ^ (D & tb[i]) ^ (E & ta[i]);
    if (party == 0) v ^= D & E;
    wires[static_cast<size_t>(g[i / W].z) * W + (i % W)] = v;
}

// rows[r] = wires[idx[r]].
__global__ void gather_rows_kernel(const uint32_t* __restrict__ wires, int W,
                                   const int* __restrict__ idx, size_t rows,
                                   uint32_t* __restrict__ out) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= rows * W) return;
    out[i] = wires[static_cast<size_t>(idx[i / W]) * W + (i % W)];
}

// vals[B] (bits 0..nbits-1) -> rows [nbits][W]; one warp per 32 instances,
// the 32 values read coalesced and transposed with ballots.
__global__ void bitslice_u64_kernel(const uint64_t* __restrict__ vals, int B, int nbits, int W,
                                    uint32_t* __restrict__ rows) {
    const int word = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32);
    const int lane = threadIdx.x & 31;
    if (word >= W) return;
    const int b = 32 * word + lane;
    const uint64_t v = b < B ? vals[b] : 0;
    for (int r = 0; r < nbits; ++r) {
        const uint32_t m = __ballot_sync(0xffffffffu, (v >> r) & 1u);
        if (lane == 0) rows[static_cast<size_t>(r) * W + word] = m;
    }
}

// 128-bit blocks -> rows [128][W]: row j = bit j (lo bits 0..63, hi 64..127).
__global__ void bitslice_blk_kernel(const Blk* __restrict__ blocks, int B, int W,
                                    uint32_t* __restrict__ rows) {
    const int word = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32);
    const int lane = threadIdx.x & 31;
    if (word >= W) return;
    const int b = 32 * word + lane;
    const Blk v = b < B ? blocks[b] : Blk{0, 0};
    for (int j = 0; j < 128; ++j) {
        const uint64_t h = j < 64 ? v.lo : v.hi;
        const uint32_t m = __ballot_sync(0xffffffffu, (h >> (j & 63)) & 1u);
        if (lane == 0) rows[static_cast<size_t>(j) * W + word] = m;
    }
}

// rows [nbits][W] -> vals[B].
__global__ void unbitslice_u64_kernel(const uint32_t* __restrict__ rows, int B, int nbits, int W,
                                      uint64_t* __restrict__ vals) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t v = 0;
    for (int r = 0; r < nbits; ++r)
        v |= static_cast<uint64_t>((rows[static_cast<size_t>(r) * W + b / 32] >> (b % 32)) & 1u) << r;
    vals[b] = v;
}

// rows [R*128][W] -> blocks [B][R]: block r of instance b from rows r*128+j.
__global__ void unbitslice_blk_kernel(const uint32_t* __restrict__ rows, int B, int R, int W,
                                      Blk* __restrict__ blocks) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<size_t>(B) * R) return;
    const int b = static_cast<int>(i / R), r = static_cast<int>(i % R);
    const uint32_t* base = rows + static_cast<size_t>(r) * 128 * W + b / 32;
    const int s = b % 32;
    uint64_t lo = 0, hi = 0;
    for (int j = 0; j < 64; ++j) {
        lo |= static_cast<uint64_t>((base[static_cast<size_t>(j) * W] >> s) & 1u) << j;
        hi |= static_cast<uint64_t>((base[static_cast<size_t>(64 + j) * W] >> s) & 1u) << j;
    }
    blocks[i] = Blk{lo, hi};
}

// ---- circuit description and schedule ---------------------------------
// A gate list in creation (topological) order.  depth = AND depth of a wire;
// sub = position of a local gate inside its depth's chain of local gates.
class BoolNet {
  public:
    int input() { return add_wire(0, 0); }
    int AND(int a, int b) { return add_gate(kAnd, a, b); }
    int XOR(int a, int b) { return add_gate(kXor, a, b); }
    int NOT(int a) { return add_gate(kNot, a, a); }
    void output(int w) { outs_.push_back(w); }

    int wires() const { return static_cast<int>(depth_.size()); }
    const std::vector<int>& outputs() const { return outs_; }
    size_t and_gates() const {
        size_t n = 0;
        for (const Gate& g : gates_) n += g.kind == kAnd;
        return n;
    }

    // Steps in evaluation order: for every AND depth d, the local gates of
    // depth d (by sub-level), then the AND gates of depth d + 1.
    struct Step {
        bool is_and;
        size_t off, count;
    };
    void schedule(std::vector<Gate>& table, std::vector<Step>& steps) const {
        int maxd = 0;
        for (int d : depth_) maxd = std::max(maxd, d);
        std::vector<std::vector<std::vector<Gate>>> local(maxd + 1);
        std::vector<std::vector<Gate>> ands(maxd + 2);
        for (const Gate& g : gates_) {
            const int d = depth_[g.z];
            if (g.kind == kAnd) {
                ands[d].push_back(g);
            } else {
                auto& lv = local[d];
                if (static_cast<int>(lv.size()) < sub_[g.z]) lv.resize(sub_[g.z]);
                lv[sub_[g.z] - 1].push_back(g);
            }
        }
        table.clear();
        steps.clear();
        auto emit = [&](const std::vector<Gate>& v, bool is_and) {
            if (v.empty()) return;
            steps.push_back({is_and, table.size(), v.size()});
            table.insert(table.end(), v.begin(), v.end());
        };
        for (int d = 0; d <= maxd; ++d) {
            for (const auto& lv : local[d]) emit(lv, false);
            if (d + 1 <= maxd) emit(ands[d + 1], true);
        }
    }

  private:
    int add_wire(int d, int s) {
        depth_.push_back(d);
        sub_.push_back(s);
        return wires() - 1;
    }
    int add_gate(int kind, int a, int b) {
        const int da = depth_[a], db = depth_[b];
        int d, s = 0;
        if (kind == kAnd) {
            d = std::max(da, db) + 1;
        } else {
            d = std::max(da, db);
            s = 1 + std::max(da == d ? sub_[a] : 0, db == d ? sub_[b] : 0);
        }
        const int z = add_wire(d, s);
        gates_.push_back({a, b, z, kind});
        return z;
    }

    std::vector<int> depth_, sub_, outs_;
    std::vector<Gate> gates_;
};

// Kogge-Stone adder of two off_bits-bit inputs (adder.h:22-63): inputs rows
// [0, m) = a (party 0's offset), [m, 2m) = b (party 1's); outputs the m + 1
// sum bits, LSB first, the last being the carry-out.
BoolNet kogge_stone_net(int m) {
    BoolNet net;
    std::vector<int> a(m), b(m), G(m), P(m), p0(m);
    for (int i = 0; i < m; ++i) a[i] = net.input();
    for (int i = 0; i < m; ++i) b[i] = net.input();
    for (int i = 0; i < m; ++i) {
        G[i] = net.AND(a[i], b[i]);
        P[i] = p0[i] = net.XOR(a[i], b[i]);
    }
    for (int d = 1; d < m; d <<= 1) {
        std::vector<int> Gn = G, Pn = P;
        for (int i = d; i < m; ++i) {
            Gn[i] = net.XOR(G[i], net.AND(P[i], G[i - d]));
            Pn[i] = net.AND(P[i], P[i - d]);
        }
        G.swap(Gn);
        P.swap(Pn);
    }
    net.output(p0[0]);
    for (int i = 1; i < m; ++i) net.output(net.XOR(p0[i], G[i - 1]));
    net.output(G[m - 1]);
    return net;
}

// DltSft circuit for one instance (dpf.cpp:214-238): inputs rows [0, n) =
// alpha bits, [n, n + 128) = Delta bits; output (i, k, j) for level i, branch
// k < 2^w - 1 and Delta bit j, in that order: the AND of the w literals
// alpha bit n - w(i+1) + c (negated where bit c of k is 0), then AND Delta_j.
BoolNet dltsft_net(int n, int w) {
    BoolNet net;
    const int levels = n / w, nk = (1 << w) - 1;
    std::vector<int> alpha(n), delta(128);
    for (int i = 0; i < n; ++i) alpha[i] = net.input();
    for (int j = 0; j < 128; ++j) delta[j] = net.input();
    for (int i = 0; i < levels; ++i) {
        for (int k = 0; k < nk; ++k) {
            std::vector<int> f(w);
            for (int c = 0; c < w; ++c) {
                const int a = alpha[n - w * (i + 1) + c];
                f[c] = ((k >> c) & 1) ? a : net.NOT(a);
            }
            while (f.size() > 1) {
                std::vector<int> next;
                for (size_t j = 0; j + 1 < f.size(); j += 2) next.push_back(net.AND(f[j], f[j + 1]));
                if (f.size() & 1) next.push_back(f.back());
                f.swap(next);
            }
            for (int j = 0; j < 128; ++j) net.output(net.AND(f[0], delta[j]));
        }
    }
    return net;
}

// ---- evaluation --------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st;
    DevBuf(size_t bytes, cudaStream_t s) : st(s) { p = bytes ? pool_alloc(bytes, s) : nullptr; }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, st);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// Evaluates `net` for B instances.  d_wires holds the input rows on entry
// (rows [0, inputs) filled by the caller) and every wire on return.
// Triples: and_gates rows of W words each, consumed in schedule order.
void evaluate(const BoolNet& net, int party, int B, uint32_t* d_wires, const uint32_t* ta,
              const uint32_t* tb, const uint32_t* tc, pcgb_exchange_fn ex, void* user,
              const char* who, cudaStream_t st) {
    const int W = (B + 31) / 32;
    std::vector<Gate> table;
    std::vector<BoolNet::Step> steps;
    net.schedule(table, steps);
    size_t max_and = 0;
    for (const auto& s : steps)
        if (s.is_and) max_and = std::max(max_and, s.count);
    const size_t ng = net.and_gates(), tri_words = ng * W;
    DevBuf d_table(table.size() * sizeof(Gate), st);
    DevBuf d_tri(3 * tri_words * sizeof(uint32_t), st);
    // Exchange messages: [d rows | e rows], padded to whole 16-byte blocks.
    const size_t max_words = 2 * max_and * W, max_blocks = (max_words + 3) / 4;
    DevBuf d_my(max_blocks * sizeof(Blk), st), d_peer(max_blocks * sizeof(Blk), st);
    std::vector<Blk> h_my(max_blocks), h_peer(max_blocks);
    if (!table.empty())
        PCGB_CK(cudaMemcpyAsync(d_table.p, table.data(), table.size() * sizeof(Gate),
                                cudaMemcpyHostToDevice, st));
    uint32_t* dt = d_tri.as<uint32_t>();
    if (tri_words) {
        PCGB_CK(cudaMemcpyAsync(dt, ta, tri_words * 4, cudaMemcpyHostToDevice, st));
        PCGB_CK(cudaMemcpyAsync(dt + tri_words, tb, tri_words * 4, cudaMemcpyHostToDevice, st));
        PCGB_CK(cudaMemcpyAsync(dt + 2 * tri_words, tc, tri_words * 4, cudaMemcpyHostToDevice, st));
    }
    const Gate* gt = d_table.as<Gate>();
    size_t tri_row = 0;
    for (const auto& s : steps) {
        const size_t words = s.count * W;
        if (!s.is_and) {
            local_kernel<<<grid_for(words), kTpb, 0, st>>>(d_wires, W, gt + s.off, s.count, party);
            PCGB_POST_LAUNCH();
            continue;
        }
        const uint32_t* a = dt + tri_row * W;
        const uint32_t* b = a + tri_words;
        const uint32_t* c = b + tri_words;
        uint32_t* my = d_my.as<uint32_t>();
        and_open_kernel<<<grid_for(words), kTpb, 0, st>>>(d_wires, W, gt + s.off, s.count, a, b, my);
        PCGB_POST_LAUNCH();
        const size_t blocks = (2 * words + 3) / 4;
        if (blocks * 4 > 2 * words) h_my[blocks - 1] = Blk{0, 0};   // zero the padding
        PCGB_CK(cudaMemcpyAsync(h_my.data(), my, 2 * words * 4, cudaMemcpyDeviceToHost, st));
        PCGB_CK(cudaStreamSynchronize(st));
        if (ex(reinterpret_cast<const pcgb_blk*>(h_my.data()),
               reinterpret_cast<pcgb_blk*>(h_peer.data()), blocks, user) != 0)
            fail(PCGB_ECALLBACK, std::string(who) + ": exchange callback failed");
        PCGB_CK(cudaMemcpyAsync(d_peer.p, h_peer.data(), 2 * words * 4, cudaMemcpyHostToDevice, st));
        and_close_kernel<<<grid_for(words), kTpb, 0, st>>>(party, d_wires, W, gt + s.off, s.count,
                                                           my, d_peer.as<uint32_t>(), a, b, c);
        PCGB_POST_LAUNCH();
        tri_row += s.count;
    }
    // h_peer is read by the last upload: keep it alive until the stream has it.
    PCGB_CK(cudaStreamSynchronize(st));
}

void gather_outputs(const BoolNet& net, int B, const uint32_t* d_wires, uint32_t* d_rows,
                    cudaStream_t st) {
    const int W = (B + 31) / 32;
    const auto& outs = net.outputs();
    DevBuf d_idx(outs.size() * sizeof(int), st);
    PCGB_CK(cudaMemcpyAsync(d_idx.p, outs.data(), outs.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
    gather_rows_kernel<<<grid_for(outs.size() * W), kTpb, 0, st>>>(d_wires, W, d_idx.as<int>(),
                                                                   outs.size(), d_rows);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaStreamSynchronize(st));   // d_idx's host source
}

void check_triples(const uint32_t* ta, const uint32_t* tb, const uint32_t* tc, size_t gates,
                   const char* who) {
    if (gates && (!ta || !tb || !tc)) fail(PCGB_EINVAL, std::string(who) + ": null triples");
}

}  // namespace

size_t gmw_position_add_gates(int off_bits) {
    if (off_bits < 1 || off_bits > 63) return 0;
    return kogge_stone_net(off_bits).and_gates();
}

size_t gmw_dltsft_gates(int n, int w) {
    if (w < 1 || w > 8 || n < 1 || n > 64 || n % w) return 0;
    return dltsft_net(n, w).and_gates();
}

void gmw_position_add(int party, int B, int off_bits, const uint64_t* my_off, const uint32_t* ta,
                      const uint32_t* tb, const uint32_t* tc, pcgb_exchange_fn ex, void* user,
                      uint64_t* alpha_share, cudaStream_t st) {
    const char* who = "gmw_position_add";
    if (party != 0 && party != 1) fail(PCGB_EINVAL, std::string(who) + ": party must be 0 or 1");
    if (off_bits < 1 || off_bits > 63) fail(PCGB_EINVAL, std::string(who) + ": off_bits must be in [1,63]");
    if (!my_off || !alpha_share) fail(PCGB_EINVAL, std::string(who) + ": null buffer");
    if (!ex) fail(PCGB_EINVAL, std::string(who) + ": an exchange callback is required");
    const BoolNet net = kogge_stone_net(off_bits);
    check_triples(ta, tb, tc, net.and_gates(), who);
    const int W = (B + 31) / 32, m = off_bits;
    DevBuf d_wires(static_cast<size_t>(net.wires()) * W * 4, st);
    DevBuf d_vals(static_cast<size_t>(B) * 8, st);
    DevBuf d_rows(static_cast<size_t>(m + 1) * W * 4, st);
    uint32_t* wires = d_wires.as<uint32_t>();
    // Trivial sharing: party 0's offset is input a (rows [0, m)), party 1's
    // is b (rows [m, 2m)); the other party's share of each is zero.
    PCGB_CK(cudaMemsetAsync(wires, 0, static_cast<size_t>(2 * m) * W * 4, st));
    PCGB_CK(cudaMemcpyAsync(d_vals.p, my_off, static_cast<size_t>(B) * 8, cudaMemcpyHostToDevice, st));
    bitslice_u64_kernel<<<grid_for(static_cast<size_t>(W) * 32), kTpb, 0, st>>>(
        d_vals.as<uint64_t>(), B, m, W, wires + static_cast<size_t>(party) * m * W);
    PCGB_POST_LAUNCH();
    evaluate(net, party, B, wires, ta, tb, tc, ex, user, who, st);
    gather_outputs(net, B, wires, d_rows.as<uint32_t>(), st);
    unbitslice_u64_kernel<<<grid_for(B), kTpb, 0, st>>>(d_rows.as<uint32_t>(), B, m + 1, W,
                                                        d_vals.as<uint64_t>());
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaMemcpyAsync(alpha_share, d_vals.p, static_cast<size_t>(B) * 8,
                            cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

void gmw_dltsft(int party, int B, int n, int w, const uint64_t* alpha_share, Blk* delta_share,
                const uint32_t* ta, const uint32_t* tb, const uint32_t* tc, pcgb_exchange_fn ex,
                void* user, Blk* dltsft, cudaStream_t st) {
    const char* who = "gmw_dltsft";
    if (party != 0 && party != 1) fail(PCGB_EINVAL, std::string(who) + ": party must be 0 or 1");
    if (w < 1 || w > 8 || n < 1 || n > 64 || n % w)
        fail(PCGB_EINVAL, std::string(who) + ": need 1 <= w <= 8, w | n, n <= 64");
    if (!alpha_share || !delta_share || !dltsft) fail(PCGB_EINVAL, std::string(who) + ": null buffer");
    if (!ex) fail(PCGB_EINVAL, std::string(who) + ": an exchange callback is required");
    // lsb(Delta) = 1: party 0 sets its share's bit 0, party 1 clears it
    // (dpf.cpp:182-190).
    for (int b = 0; b < B; ++b) delta_share[b].lo = party == 0 ? (delta_share[b].lo | 1u)
                                                               : (delta_share[b].lo & ~uint64_t{1});
    const BoolNet net = dltsft_net(n, w);
    check_triples(ta, tb, tc, net.and_gates(), who);
    const int W = (B + 31) / 32;
    const int R = (n / w) * ((1 << w) - 1);   // DltSft blocks per instance
    DevBuf d_wires(static_cast<size_t>(net.wires()) * W * 4, st);
    DevBuf d_alpha(static_cast<size_t>(B) * 8, st), d_delta(static_cast<size_t>(B) * 16, st);
    DevBuf d_rows(static_cast<size_t>(R) * 128 * W * 4, st);
    DevBuf d_out(static_cast<size_t>(B) * R * 16, st);
    uint32_t* wires = d_wires.as<uint32_t>();
    PCGB_CK(cudaMemcpyAsync(d_alpha.p, alpha_share, static_cast<size_t>(B) * 8, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(d_delta.p, delta_share, static_cast<size_t>(B) * 16, cudaMemcpyHostToDevice, st));
    bitslice_u64_kernel<<<grid_for(static_cast<size_t>(W) * 32), kTpb, 0, st>>>(
        d_alpha.as<uint64_t>(), B, n, W, wires);
    PCGB_POST_LAUNCH();
    bitslice_blk_kernel<<<grid_for(static_cast<size_t>(W) * 32), kTpb, 0, st>>>(
        d_delta.as<Blk>(), B, W, wires + static_cast<size_t>(n) * W);
    PCGB_POST_LAUNCH();
    evaluate(net, party, B, wires, ta, tb, tc, ex, user, who, st);
    gather_outputs(net, B, wires, d_rows.as<uint32_t>(), st);
    unbitslice_blk_kernel<<<grid_for(static_cast<size_t>(B) * R), kTpb, 0, st>>>(
        d_rows.as<uint32_t>(), B, R, W, d_out.as<Blk>());
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaMemcpyAsync(dltsft, d_out.p, static_cast<size_t>(B) * R * 16,
                            cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaStreamSynchronize(st));
}

}  // namespace pcgb
