// CPU oracle for the PCG-OLE expansion path.  TEST INFRASTRUCTURE ONLY: the
// shipped library never links or calls this file.  Each function restates the
// reference algorithm named in its comment (paths inside tkgong/pcg-square).
// See pcg_oracle.h for how parity is pinned.
#include "pcg_oracle.h"

#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr uint64_t P = 4611686018326724609ULL;  // 2^62 - 3*2^25 + 1

inline uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

// ChaCha8 block function: 16-word state = "expand 32-byte k" constants, eight
// key words, 64-bit block counter, 64-bit nonce; four double rounds (column
// round then diagonal round); each output word = final word + initial word.
// Restates CPU_baseline/chacha8.h:20-40 (state) and :106-150 (rounds).
void chacha8(const uint32_t in[16], uint32_t out[16]) {
    uint32_t x[16];
    std::memcpy(x, in, sizeof(x));
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);
        x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);
        x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);
        x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    };
    for (int r = 0; r < 4; ++r) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
}

void chacha8_state(uint32_t st[16], const uint32_t key[8], uint64_t ctr, uint64_t nonce) {
    st[0] = 0x61707865u; st[1] = 0x3320646eu; st[2] = 0x79622d32u; st[3] = 0x6b206574u;
    for (int i = 0; i < 8; ++i) st[4 + i] = key[i];
    st[12] = static_cast<uint32_t>(ctr); st[13] = static_cast<uint32_t>(ctr >> 32);
    st[14] = static_cast<uint32_t>(nonce); st[15] = static_cast<uint32_t>(nonce >> 32);
}

// The 128-bit node is the low half of the 256-bit ChaCha key (upper half 0):
// tree_prg.h:88-94 (memcpy of the block into key[0..15], rest zero).
void node_key(uint32_t key[8], orc_blk v) {
    key[0] = static_cast<uint32_t>(v.lo); key[1] = static_cast<uint32_t>(v.lo >> 32);
    key[2] = static_cast<uint32_t>(v.hi); key[3] = static_cast<uint32_t>(v.hi >> 32);
    key[4] = key[5] = key[6] = key[7] = 0;
}

inline orc_blk bxor(orc_blk a, orc_blk b) { return {a.lo ^ b.lo, a.hi ^ b.hi}; }
inline orc_blk band(bool c, orc_blk a) { return c ? a : orc_blk{0, 0}; }
inline bool lsb(orc_blk a) { return (a.lo & 1) != 0; }

// ---- AES-128 (FIPS-197), byte oriented -----------------------------------
// State bytes in memory order (column-major 4x4), like the emp block bytes
// the reference feeds its AES (GPU_baseline/common/aes_gpu.cuh:128-141).
struct AesTables {
    uint8_t sbox[256];
    AesTables() {
        // S-box from its definition: multiplicative inverse in GF(2^8) mod
        // x^8+x^4+x^3+x+1, then the affine map b ^ rotl(b,1..4) ^ 0x63.
        auto gmul = [](uint8_t a, uint8_t b) {
            uint8_t p = 0;
            for (int i = 0; i < 8; ++i) {
                if (b & 1) p ^= a;
                bool hi = a & 0x80;
                a <<= 1;
                if (hi) a ^= 0x1b;
                b >>= 1;
            }
            return p;
        };
        for (int x = 0; x < 256; ++x) {
            uint8_t inv = 0;
            if (x) for (int y = 1; y < 256; ++y) if (gmul(x, y) == 1) { inv = y; break; }
            uint8_t s = inv;
            uint8_t r = inv;
            for (int k = 0; k < 4; ++k) { r = static_cast<uint8_t>((r << 1) | (r >> 7)); s ^= r; }
            sbox[x] = s ^ 0x63;
        }
    }
};
const AesTables& aes_tables() { static AesTables t; return t; }

inline uint8_t xt(uint8_t v) { return static_cast<uint8_t>((v << 1) ^ ((v & 0x80) ? 0x1b : 0)); }

// ---- mod-P arithmetic ------------------------------------------------------
inline uint64_t addm(uint64_t a, uint64_t b) { uint64_t s = a + b; return s >= P ? s - P : s; }
inline uint64_t subm(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P - b; }
inline uint64_t mulm(uint64_t a, uint64_t b) {
    return static_cast<uint64_t>((static_cast<__uint128_t>(a) * b) % P);
}
uint64_t powm(uint64_t b, uint64_t e) {
    uint64_t r = 1; b %= P;
    while (e) { if (e & 1) r = mulm(r, b); b = mulm(b, b); e >>= 1; }
    return r;
}
// Shoup multiplication by a fixed w (companion wq = floor(w * 2^64 / P)).
inline uint64_t shoup(uint64_t a, uint64_t w, uint64_t wq) {
    uint64_t q = static_cast<uint64_t>((static_cast<__uint128_t>(a) * wq) >> 64);
    uint64_t r = a * w - q * P;
    return r >= P ? r - P : r;
}
inline uint64_t shoup_q(uint64_t w) {
    return static_cast<uint64_t>((static_cast<__uint128_t>(w) << 64) / P);
}

// Smallest primitive root of Z_P^*: factor P-1 by trial division and test
// g^((P-1)/q) != 1 for each prime factor q (CPU_baseline/ntt.h:199-222).
uint64_t primitive_root() {
    static uint64_t g = 0;
    if (g) return g;
    std::vector<uint64_t> f;
    uint64_t x = P - 1;
    for (uint64_t d = 2; d * d <= x; ++d) {
        if (x % d) continue;
        f.push_back(d);
        while (x % d == 0) x /= d;
    }
    if (x > 1) f.push_back(x);
    for (uint64_t c = 2;; ++c) {
        bool ok = true;
        for (uint64_t q : f) if (powm(c, (P - 1) / q) == 1) { ok = false; break; }
        if (ok) { g = c; return g; }
    }
}

// Negacyclic NTT tables for one N (CPU_baseline/ntt.h:98-135): psi a
// primitive 2N-th root (psi = g^((P-1)/2N)), omega = psi^2, twist tables
// psi^i and N^-1 * psi^-i, root tables omega^k and omega^-k for k < N/2.
struct NttPlan {
    int N = 0, logN = 0;
    std::vector<uint64_t> tw, twq, itw, itwq, rf, rfq, ri, riq;
    std::vector<uint32_t> brev;
    explicit NttPlan(int n) : N(n) {
        while ((1 << logN) < N) ++logN;
        uint64_t psi = powm(primitive_root(), (P - 1) / (2ull * N));
        uint64_t psi_inv = powm(psi, P - 2);
        uint64_t n_inv = powm(static_cast<uint64_t>(N), P - 2);
        uint64_t om = mulm(psi, psi), om_inv = mulm(psi_inv, psi_inv);
        tw.resize(N); itw.resize(N); twq.resize(N); itwq.resize(N);
        uint64_t a = 1, b = n_inv;
        for (int i = 0; i < N; ++i) {
            tw[i] = a; twq[i] = shoup_q(a); a = mulm(a, psi);
            itw[i] = b; itwq[i] = shoup_q(b); b = mulm(b, psi_inv);
        }
        int h = N / 2 > 0 ? N / 2 : 1;
        rf.resize(h); ri.resize(h); rfq.resize(h); riq.resize(h);
        a = 1; b = 1;
        for (int i = 0; i < h; ++i) {
            rf[i] = a; rfq[i] = shoup_q(a); a = mulm(a, om);
            ri[i] = b; riq[i] = shoup_q(b); b = mulm(b, om_inv);
        }
        brev.resize(N);
        for (int i = 0; i < N; ++i) {
            uint32_t r = 0;
            for (int k = 0; k < logN; ++k) r |= ((i >> k) & 1u) << (logN - 1 - k);
            brev[i] = r;
        }
    }
    // Bit-reverse permutation then radix-2 Cooley-Tukey stages with root
    // stride N/len (CPU_baseline/ntt.h:175-197).
    void core(uint64_t* a, const std::vector<uint64_t>& r, const std::vector<uint64_t>& rq) const {
        for (int i = 0; i < N; ++i) if (i < static_cast<int>(brev[i])) std::swap(a[i], a[brev[i]]);
        for (int len = 2; len <= N; len <<= 1) {
            int half = len >> 1, step = N / len;
            for (int i = 0; i < N; i += len)
                for (int j = 0; j < half; ++j) {
                    uint64_t u = a[i + j];
                    uint64_t v = shoup(a[i + j + half], r[j * step], rq[j * step]);
                    a[i + j] = addm(u, v);
                    a[i + j + half] = subm(u, v);
                }
        }
    }
    void forward(uint64_t* a) const {   // ntt.h:140-144
        for (int i = 0; i < N; ++i) a[i] = shoup(a[i], tw[i], twq[i]);
        core(a, rf, rfq);
    }
    void inverse(uint64_t* a) const {   // ntt.h:149-153
        core(a, ri, riq);
        for (int i = 0; i < N; ++i) a[i] = shoup(a[i], itw[i], itwq[i]);
    }
};

const NttPlan& plan_for(int N) {
    static std::mutex mu;
    static std::vector<NttPlan*> plans;
    std::lock_guard<std::mutex> g(mu);
    for (auto* p : plans) if (p->N == N) return *p;
    plans.push_back(new NttPlan(N));
    return *plans.back();
}

void poly_mul1(uint64_t* c, const uint64_t* a, const uint64_t* b, int N) {
    // ntt.h:156-163: forward both, pointwise, inverse.  Inputs are reduced
    // mod P as the FFp(uint64_t) constructor does (ffp.h:15,23).
    const NttPlan& pl = plan_for(N);
    std::vector<uint64_t> fa(N), fb(N);
    for (int i = 0; i < N; ++i) { fa[i] = a[i] % P; fb[i] = b[i] % P; }
    pl.forward(fa.data());
    pl.forward(fb.data());
    for (int i = 0; i < N; ++i) fa[i] = mulm(fa[i], fb[i]);
    pl.inverse(fa.data());
    std::memcpy(c, fa.data(), sizeof(uint64_t) * N);
}

// ---- tree PRG dispatch -----------------------------------------------------
void tree_hash(orc_blk* out, const orc_blk* parents, size_t n, int nk, const uint8_t* rks,
               int prg) {
    if (prg == ORC_PRG_CHACHA8) orc_tree_hash_chacha8(out, parents, n, nk);
    else orc_tree_hash_aes(out, parents, n, nk, rks);
}

// Expand one frontier level: children j*m+k (k<m-1) = H_k ^ t*CW[k]; child
// j*m+m-1 = (XOR_k H_k) ^ parent ^ t*CW[m-1]  (dpf.cpp:553-574).
void expand_level(const orc_blk* tree, size_t sz, const orc_blk* h, int m, const orc_blk* CW,
                  orc_blk* next) {
    const int nk = m - 1;
    for (size_t j = 0; j < sz; ++j) {
        const bool t = lsb(tree[j]);
        orc_blk hx{0, 0};
        for (int k = 0; k < nk; ++k) {
            hx = bxor(hx, h[j * nk + k]);
            next[j * m + k] = bxor(h[j * nk + k], band(t, CW[k]));
        }
        next[j * m + nk] = bxor(bxor(hx, tree[j]), band(t, CW[nk]));
    }
}

int check_shape(int n, int w) {
    if (w < 1 || w > 4 || n < 1 || n > 30 || n % w) return -1;
    return 0;
}

// Counter-based generator: SplitMix64 finaliser (Steele, Lea, Flood 2014)
// applied to a (seed, domain, index) mix.  Own definition, mirrored by the
// library's dealer.
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

enum : uint64_t {
    DOM_POS = 0x10, DOM_VAL = 0x20, DOM_A = 0x30, DOM_DELTA = 0x40, DOM_ROOT = 0x50,
};

}  // namespace

extern "C" {

uint64_t orc_prime(void) { return P; }

void orc_chacha8_block(const uint32_t key[8], uint64_t counter, uint64_t nonce,
                       uint32_t out[16]) {
    uint32_t st[16];
    chacha8_state(st, key, counter, nonce);
    chacha8(st, out);
}

// ChaCha8TreePRG::hash (tree_prg.h:86-104): keystream with key = parent || 0,
// nonce 0, counter 0,1,..; child k = 16-byte chunk k (block k/4, words
// 4*(k%4)..+3) assembled little-endian into (lo, hi).
void orc_tree_hash_chacha8(orc_blk* out, const orc_blk* parents, size_t n, int nk) {
    const int nblocks = (nk + 3) / 4;
    for (size_t j = 0; j < n; ++j) {
        uint32_t key[8], ks[16];
        node_key(key, parents[j]);
        for (int b = 0; b < nblocks; ++b) {
            orc_chacha8_block(key, static_cast<uint64_t>(b), 0, ks);
            for (int c = 0; c < 4; ++c) {
                const int k = b * 4 + c;
                if (k >= nk) break;
                out[j * nk + k].lo = ks[4 * c] | (static_cast<uint64_t>(ks[4 * c + 1]) << 32);
                out[j * nk + k].hi = ks[4 * c + 2] | (static_cast<uint64_t>(ks[4 * c + 3]) << 32);
            }
        }
    }
}

// ChaCha8OutHash::hash (tree_prg.h:134-147): same keying, nonce = "out_hash"
// (0x6f75745f68617368), counter 0; the convert uses bytes 0..7 of block 0.
uint64_t orc_out_hash_lo64(orc_blk leaf) {
    uint32_t key[8], ks[16];
    node_key(key, leaf);
    orc_chacha8_block(key, 0, 0x6f75745f68617368ULL, ks);
    return ks[0] | (static_cast<uint64_t>(ks[1]) << 32);
}

// FIPS-197 key expansion (AES-128: 44 words, RotWord/SubWord/Rcon every 4th).
void orc_aes128_expand_key(const uint8_t key[16], uint8_t rk[176]) {
    const uint8_t* S = aes_tables().sbox;
    std::memcpy(rk, key, 16);
    uint8_t rcon = 1;
    for (int i = 4; i < 44; ++i) {
        uint8_t t[4];
        std::memcpy(t, rk + 4 * (i - 1), 4);
        if (i % 4 == 0) {
            uint8_t t0 = t[0];
            t[0] = S[t[1]] ^ rcon; t[1] = S[t[2]]; t[2] = S[t[3]]; t[3] = S[t0];
            rcon = xt(rcon);
        }
        for (int k = 0; k < 4; ++k) rk[4 * i + k] = rk[4 * (i - 4) + k] ^ t[k];
    }
}

// FIPS-197 Cipher: AddRoundKey, 9 x (SubBytes, ShiftRows, MixColumns,
// AddRoundKey), final round without MixColumns.
void orc_aes128_encrypt(const uint8_t rk[176], const uint8_t in[16], uint8_t out[16]) {
    const uint8_t* S = aes_tables().sbox;
    uint8_t s[16];
    for (int i = 0; i < 16; ++i) s[i] = in[i] ^ rk[i];
    for (int r = 1; r <= 10; ++r) {
        uint8_t u[16];
        // SubBytes + ShiftRows: row j of column c comes from column (c+j)%4.
        for (int c = 0; c < 4; ++c)
            for (int j = 0; j < 4; ++j) u[4 * c + j] = S[s[4 * ((c + j) & 3) + j]];
        if (r < 10) {
            for (int c = 0; c < 4; ++c) {
                uint8_t* v = u + 4 * c;
                uint8_t a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
                uint8_t all = a0 ^ a1 ^ a2 ^ a3;
                v[0] = a0 ^ all ^ xt(a0 ^ a1);
                v[1] = a1 ^ all ^ xt(a1 ^ a2);
                v[2] = a2 ^ all ^ xt(a2 ^ a3);
                v[3] = a3 ^ all ^ xt(a3 ^ a0);
            }
        }
        for (int i = 0; i < 16; ++i) s[i] = u[i] ^ rk[16 * r + i];
    }
    std::memcpy(out, s, 16);
}

// AESTreePRG sub-keys (tree_prg.h:45-57): sub_k = AES_master(tweak) ^ tweak
// with tweak = makeBlock(0, k), i.e. bytes 0..7 = k little-endian, 8..15 = 0.
void orc_aes_tree_round_keys(const uint8_t master[16], int nk, uint8_t* rks) {
    uint8_t mrk[176];
    orc_aes128_expand_key(master, mrk);
    for (int k = 0; k < nk; ++k) {
        uint8_t tw[16] = {0}, c[16];
        uint64_t kk = static_cast<uint64_t>(k);
        std::memcpy(tw, &kk, 8);
        orc_aes128_encrypt(mrk, tw, c);
        for (int i = 0; i < 16; ++i) c[i] ^= tw[i];
        orc_aes128_expand_key(c, rks + 176 * k);
    }
}

// MKeyPRP::hash (mkey_prp.h:189-227): H_k(x) = AES_{sub_k}(x) ^ x.
void orc_tree_hash_aes(orc_blk* out, const orc_blk* parents, size_t n, int nk,
                       const uint8_t* rks) {
    for (size_t j = 0; j < n; ++j) {
        uint8_t in[16], c[16];
        std::memcpy(in, &parents[j].lo, 8);
        std::memcpy(in + 8, &parents[j].hi, 8);
        for (int k = 0; k < nk; ++k) {
            orc_aes128_encrypt(rks + 176 * k, in, c);
            orc_blk h;
            std::memcpy(&h.lo, c, 8);
            std::memcpy(&h.hi, c + 8, 8);
            out[j * nk + k] = bxor(h, parents[j]);
        }
    }
}

// HalfTreeDPF::batch_gen_full_eval (dpf.cpp:485-578), with the roots given
// directly (root = delta_share ^ W, as the GPU bridge precomputes at
// dpf.cpp:621-632) and the per-level network round abstracted as `ex`.
int orc_dpf_batch_full_eval(int B, int n, int w, const orc_blk* roots,
                            const orc_blk* dltsft, const uint8_t* rks, int prg,
                            orc_exchange_fn ex, void* user, orc_blk* out_leaves) {
    if (check_shape(n, w) || B <= 0) return -1;
    const int m = 1 << w, nk = m - 1, levels = n / w;
    const size_t D = static_cast<size_t>(1) << n;
    std::vector<orc_blk> cur(static_cast<size_t>(B) * D), nxt(static_cast<size_t>(B) * D);
    std::vector<orc_blk> h(D / m * nk);
    for (int b = 0; b < B; ++b) cur[static_cast<size_t>(b) * D] = roots[b];
    std::vector<orc_blk> my(static_cast<size_t>(B) * nk), peer(static_cast<size_t>(B) * nk);
    std::vector<std::vector<orc_blk>> hall(B);
    for (int i = 0; i < levels; ++i) {
        const size_t sz = static_cast<size_t>(1) << (w * i);
        for (int b = 0; b < B; ++b) {
            hall[b].resize(sz * nk);
            tree_hash(hall[b].data(), &cur[static_cast<size_t>(b) * D], sz, nk, rks, prg);
            for (int k = 0; k < nk; ++k) {
                orc_blk cw{0, 0};
                for (size_t j = 0; j < sz; ++j) cw = bxor(cw, hall[b][j * nk + k]);
                my[static_cast<size_t>(b) * nk + k] =
                    bxor(cw, dltsft[(static_cast<size_t>(b) * levels + i) * nk + k]);
            }
        }
        if (ex) ex(my.data(), peer.data(), my.size(), user);
        else std::fill(peer.begin(), peer.end(), orc_blk{0, 0});
        for (int b = 0; b < B; ++b) {
            orc_blk CW[16];
            CW[nk] = {0, 0};
            for (int k = 0; k < nk; ++k) {
                CW[k] = bxor(my[static_cast<size_t>(b) * nk + k], peer[static_cast<size_t>(b) * nk + k]);
                CW[nk] = bxor(CW[nk], CW[k]);
            }
            expand_level(&cur[static_cast<size_t>(b) * D], sz, hall[b].data(), m, CW,
                         &nxt[static_cast<size_t>(b) * D]);
        }
        std::swap(cur, nxt);
    }
    std::memcpy(out_leaves, cur.data(), sizeof(orc_blk) * cur.size());
    return 0;
}

struct SwapCtx {
    std::vector<orc_blk> other;
};

int orc_dpf_batch_full_eval_2p(int B, int n, int w, const orc_blk* roots0,
                               const orc_blk* roots1, const orc_blk* dlt0,
                               const orc_blk* dlt1, const uint8_t* rks, int prg,
                               orc_blk* leaves0, orc_blk* leaves1, orc_blk* cws_out) {
    if (check_shape(n, w) || B <= 0) return -1;
    const int m = 1 << w, nk = m - 1, levels = n / w;
    const size_t D = static_cast<size_t>(1) << n;
    const orc_blk* roots[2] = {roots0, roots1};
    const orc_blk* dlt[2] = {dlt0, dlt1};
    orc_blk* outs[2] = {leaves0, leaves1};
    std::vector<orc_blk> cur[2], nxt[2], my[2];
    std::vector<std::vector<orc_blk>> hall[2];
    for (int p = 0; p < 2; ++p) {
        cur[p].assign(static_cast<size_t>(B) * D, {0, 0});
        nxt[p].assign(static_cast<size_t>(B) * D, {0, 0});
        my[p].resize(static_cast<size_t>(B) * nk);
        hall[p].resize(B);
        for (int b = 0; b < B; ++b) cur[p][static_cast<size_t>(b) * D] = roots[p][b];
    }
    for (int i = 0; i < levels; ++i) {
        const size_t sz = static_cast<size_t>(1) << (w * i);
        for (int p = 0; p < 2; ++p)
            for (int b = 0; b < B; ++b) {
                hall[p][b].resize(sz * nk);
                tree_hash(hall[p][b].data(), &cur[p][static_cast<size_t>(b) * D], sz, nk, rks, prg);
                for (int k = 0; k < nk; ++k) {
                    orc_blk cw{0, 0};
                    for (size_t j = 0; j < sz; ++j) cw = bxor(cw, hall[p][b][j * nk + k]);
                    my[p][static_cast<size_t>(b) * nk + k] =
                        bxor(cw, dlt[p][(static_cast<size_t>(b) * levels + i) * nk + k]);
                }
            }
        for (int b = 0; b < B; ++b) {
            orc_blk CW[16];
            CW[nk] = {0, 0};
            for (int k = 0; k < nk; ++k) {
                CW[k] = bxor(my[0][static_cast<size_t>(b) * nk + k], my[1][static_cast<size_t>(b) * nk + k]);
                CW[nk] = bxor(CW[nk], CW[k]);
                if (cws_out) cws_out[(static_cast<size_t>(b) * levels + i) * nk + k] = CW[k];
            }
            for (int p = 0; p < 2; ++p)
                expand_level(&cur[p][static_cast<size_t>(b) * D], sz, hall[p][b].data(), m, CW,
                             &nxt[p][static_cast<size_t>(b) * D]);
        }
        for (int p = 0; p < 2; ++p) std::swap(cur[p], nxt[p]);
    }
    for (int p = 0; p < 2; ++p) std::memcpy(outs[p], cur[p].data(), sizeof(orc_blk) * cur[p].size());
    return 0;
}

// Level-by-level expansion of K independent keys with their CWs known: the
// same per-level update as dpf.cpp:553-574, with CW[m-1] = XOR of CW[0..nk)
// (dpf.cpp:380-382).
int orc_dpf_keyed_full_eval(int K, int n, int w, const orc_blk* roots,
                            const orc_blk* cws, const uint8_t* rks, int prg,
                            orc_blk* out_leaves) {
    if (check_shape(n, w) || K <= 0) return -1;
    const int m = 1 << w, nk = m - 1, levels = n / w;
    const size_t D = static_cast<size_t>(1) << n;
    std::vector<orc_blk> cur(D), nxt(D), h(D / m * nk);
    for (int k = 0; k < K; ++k) {
        cur[0] = roots[k];
        for (int i = 0; i < levels; ++i) {
            const size_t sz = static_cast<size_t>(1) << (w * i);
            tree_hash(h.data(), cur.data(), sz, nk, rks, prg);
            orc_blk CW[16];
            CW[nk] = {0, 0};
            for (int j = 0; j < nk; ++j) {
                CW[j] = cws[(static_cast<size_t>(k) * levels + i) * nk + j];
                CW[nk] = bxor(CW[nk], CW[j]);
            }
            expand_level(cur.data(), sz, h.data(), m, CW, nxt.data());
            std::swap(cur, nxt);
        }
        std::memcpy(out_leaves + static_cast<size_t>(k) * D, cur.data(), sizeof(orc_blk) * D);
    }
    return 0;
}

// HalfTreeDPF::eval (dpf.cpp:302-327): walk root->leaf along the base-m
// digits of j (most significant digit first).
orc_blk orc_dpf_eval(orc_blk root, const orc_blk* cws, int n, int w,
                     const uint8_t* rks, int prg, uint64_t j) {
    const int m = 1 << w, nk = m - 1, levels = n / w;
    orc_blk seed = root, h[16];
    for (int i = 0; i < levels; ++i) {
        const bool t = lsb(seed);
        const uint64_t digit = (j >> (n - w * (i + 1))) & static_cast<uint64_t>(nk);
        tree_hash(h, &seed, 1, nk, rks, prg);
        orc_blk hx{0, 0}, cwf{0, 0};
        for (int k = 0; k < nk; ++k) { hx = bxor(hx, h[k]); cwf = bxor(cwf, cws[i * nk + k]); }
        if (static_cast<int>(digit) < nk) seed = bxor(h[digit], band(t, cws[i * nk + digit]));
        else seed = bxor(bxor(hx, seed), band(t, cwf));
    }
    return seed;
}

int orc_dpf_deal(int n, int w, orc_blk root0, orc_blk delta, uint64_t alpha,
                 uint64_t beta, const uint8_t* rks, int prg, orc_blk* cws,
                 uint64_t* cw_out, const orc_blk* dlt0, orc_blk* dlt1) {
    if (check_shape(n, w) || !(delta.lo & 1) || (n < 64 && (alpha >> n))) return -1;
    const int m = 1 << w, nk = m - 1, levels = n / w;
    orc_blk p[2] = {root0, bxor(root0, delta)};
    for (int i = 0; i < levels; ++i) {
        const int digit = static_cast<int>((alpha >> (n - w * (i + 1))) & static_cast<uint64_t>(nk));
        orc_blk h[2][16], hx[2] = {{0, 0}, {0, 0}};
        for (int s = 0; s < 2; ++s) {
            tree_hash(h[s], &p[s], 1, nk, rks, prg);
            for (int k = 0; k < nk; ++k) hx[s] = bxor(hx[s], h[s][k]);
        }
        // Off-path nodes are equal in both trees, so the XOR over the whole
        // frontier of H_k (dpf.cpp:359-364) reduces to the on-path pair.
        orc_blk CW[16];
        CW[nk] = {0, 0};
        for (int k = 0; k < nk; ++k) {
            CW[k] = bxor(bxor(h[0][k], h[1][k]), band(digit == k, delta));
            CW[nk] = bxor(CW[nk], CW[k]);
            cws[i * nk + k] = CW[k];
            if (dlt1) dlt1[i * nk + k] = bxor(dlt0[i * nk + k], band(digit == k, delta));
        }
        for (int s = 0; s < 2; ++s) {
            const bool t = lsb(p[s]);
            if (digit < nk) p[s] = bxor(h[s][digit], band(t, CW[digit]));
            else p[s] = bxor(bxor(hx[s], p[s]), band(t, CW[nk]));
        }
        const orc_blk d = bxor(p[0], p[1]);
        if (d.lo != delta.lo || d.hi != delta.hi) return -2;
    }
    // Output-layer CW = A*B with A = tau0 - tau1 and B = C1 - C0 + beta at
    // alpha (pcg_ole_impl.h:358-364 shares, :397-407 Beaver product).
    const uint64_t C0 = orc_out_hash_lo64(p[0]) % P, C1 = orc_out_hash_lo64(p[1]) % P;
    const uint64_t A = subm(lsb(p[0]) ? 1 : 0, lsb(p[1]) ? 1 : 0);
    const uint64_t Bv = addm(subm(C1, C0), beta % P);
    *cw_out = mulm(A, Bv);
    return 0;
}

// dpf_out_sums semantics (leaf_convert_cuda.h:40-44; host loop
// pcg_ole_impl.h:347-357): C = low64(H'(leaf)) mod P, tau = lsb(leaf).
void orc_out_sums(const orc_blk* leaves, int B, size_t D, uint64_t* sumC, uint64_t* sumT) {
    for (int b = 0; b < B; ++b) {
        uint64_t c = 0, t = 0;
        for (size_t d = 0; d < D; ++d) {
            const orc_blk& l = leaves[static_cast<size_t>(b) * D + d];
            c = addm(c, orc_out_hash_lo64(l) % P);
            t += l.lo & 1;
        }
        sumC[b] = c;
        sumT[b] = t;
    }
}

// Output layer scatter (pcg_ole_impl.h:433-446) with the X^N = -1 fold of
// step 4 (pcg_ole_impl.h:474-478): y = C + tau*CW, party 1 negates,
// pos = (b/t + b%t)*D/2 + d, pos >= N lands negated at pos - N.
void orc_out_scatter_g(const orc_blk* leaves, int B, size_t D, int t, int party,
                       const uint64_t* CW, uint64_t* g, int N) {
    std::vector<uint64_t> g2(2 * static_cast<size_t>(N), 0);
    const size_t bin = D / 2;
    for (int b = 0; b < B; ++b) {
        const size_t base = static_cast<size_t>(b / t + b % t) * bin;
        for (size_t d = 0; d < D; ++d) {
            const orc_blk& l = leaves[static_cast<size_t>(b) * D + d];
            uint64_t y = orc_out_hash_lo64(l) % P;
            if (l.lo & 1) y = addm(y, CW[b] % P);
            if (party == 1) y = subm(0, y);
            const size_t pos = base + d;
            if (pos < 2 * static_cast<size_t>(N)) g2[pos] = addm(g2[pos], y);
        }
    }
    for (int d = 0; d < N; ++d) g[d] = subm(g2[d], g2[static_cast<size_t>(N) + d]);
}

uint64_t orc_mulmod(uint64_t a, uint64_t b) { return mulm(a % P, b % P); }

void orc_poly_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, int batch, int N) {
    for (int k = 0; k < batch; ++k)
        poly_mul1(c + static_cast<size_t>(k) * N, a + static_cast<size_t>(k) * N,
                  b + static_cast<size_t>(k) * N, N);
}

void orc_ntt_forward(uint64_t* a, int batch, int N) {
    const NttPlan& pl = plan_for(N);
    for (int k = 0; k < batch; ++k) {
        uint64_t* x = a + static_cast<size_t>(k) * N;
        for (int i = 0; i < N; ++i) x[i] %= P;
        pl.forward(x);
    }
}

// triple.h:72-107: ring triple shares, then NTT slot extraction.
void orc_triples(int N, int party, const uint64_t* x1, const uint64_t* z1, const uint64_t* x2,
                 const uint64_t* z2, uint64_t* a, uint64_t* b, uint64_t* c) {
    const uint64_t* as = party == 0 ? x1 : x2;
    const uint64_t* bs = party == 0 ? x2 : x1;
    for (int i = 0; i < N; ++i) { a[i] = as[i] % P; b[i] = bs[i] % P; }
    poly_mul1(c, a, b, N);                               // poly_mul_backend
    for (int i = 0; i < N; ++i) c[i] = addm(addm(c[i], z1[i] % P), z2[i] % P);   // poly_add
    const NttPlan& pl = plan_for(N);
    pl.forward(a);
    pl.forward(b);
    pl.forward(c);
}

// pcg_ole.h:92-106.
void orc_poly_mul_schoolbook(uint64_t* c, const uint64_t* a, const uint64_t* b, int N) {
    std::vector<uint64_t> r(N, 0);
    for (int i = 0; i < N; ++i) {
        const uint64_t ai = a[i] % P;
        if (!ai) continue;
        for (int j = 0; j < N; ++j) {
            const uint64_t v = mulm(ai, b[j] % P);
            const int k = i + j;
            if (k < N) r[k] = addm(r[k], v);
            else r[k - N] = subm(r[k - N], v);
        }
    }
    std::memcpy(c, r.data(), sizeof(uint64_t) * N);
}

uint64_t orc_rnd(uint64_t seed, uint64_t dom, uint64_t idx) {
    return mix64(mix64(seed ^ (dom * 0x9e3779b97f4a7c15ULL)) + (idx + 1) * 0xd1b54a32d192ed03ULL);
}

int orc_shape_init(orc_shape* s, int N, int c, int t, int w, int prg) {
    if (N < 4 || (N & (N - 1)) || c < 1 || c > 8 || t < 1 || (t & (t - 1)) || N % t ||
        N / t < 2)
        return -1;
    s->N = N; s->c = c; s->t = t; s->w = w; s->prg = prg;
    int n = 0;
    while ((1 << n) < 2 * (N / t)) ++n;  // D = 2N/t (pcg_ole_impl.h:54-56)
    if (check_shape(n, w)) return -1;
    s->n = n; s->levels = n / w; s->nk = (1 << w) - 1; s->K = c * c * t * t;
    return 0;
}

// Regular noise (pcg_ole_impl.h:68-77): one nonzero per block of N/t, at
// k*bin + (r % bin), value r % (P-1) + 1; r drawn from the seeded generator.
void orc_noise(const orc_shape* s, uint64_t seed, int party, uint64_t* pos, uint64_t* val) {
    const uint64_t bin = static_cast<uint64_t>(s->N / s->t);
    for (int i = 0; i < s->c; ++i)
        for (int k = 0; k < s->t; ++k) {
            const uint64_t idx = static_cast<uint64_t>(i) * s->t + k;
            pos[idx] = static_cast<uint64_t>(k) * bin + orc_rnd(seed, DOM_POS + party, idx) % bin;
            val[idx] = orc_rnd(seed, DOM_VAL + party, idx) % (P - 1) + 1;
        }
}

void orc_public_a(const orc_shape* s, uint64_t a_seed, uint64_t* a) {
    for (int i = 1; i < s->c; ++i)
        for (int j = 0; j < s->N; ++j)
            a[static_cast<size_t>(i - 1) * s->N + j] = orc_rnd(a_seed, DOM_A + i, j) % P;
}

// Dealer over all c*c blocks of t*t instances (pcg_ole_impl.h:114-199
// position/payload algebra): alpha = off0[ii][kk] + off1[jj][ll],
// beta = val0[ii][kk] * val1[jj][ll].
int orc_deal_keys(const orc_shape* s, uint64_t seed, const uint8_t* rks,
                  orc_blk* roots0, orc_blk* roots1, orc_blk* cws, uint64_t* cw_out) {
    const int c = s->c, t = s->t;
    const uint64_t bin = static_cast<uint64_t>(s->N / t);
    std::vector<uint64_t> pos[2], val[2];
    for (int p = 0; p < 2; ++p) {
        pos[p].resize(static_cast<size_t>(c) * t);
        val[p].resize(static_cast<size_t>(c) * t);
        orc_noise(s, seed, p, pos[p].data(), val[p].data());
    }
    const size_t per = static_cast<size_t>(s->levels) * s->nk;
    for (int ii = 0; ii < c; ++ii)
        for (int jj = 0; jj < c; ++jj)
            for (int kk = 0; kk < t; ++kk)
                for (int ll = 0; ll < t; ++ll) {
                    const uint64_t id = (static_cast<uint64_t>(ii) * c + jj) * t * t + kk * t + ll;
                    const uint64_t alpha = pos[0][ii * t + kk] % bin + pos[1][jj * t + ll] % bin;
                    const uint64_t beta = mulm(val[0][ii * t + kk], val[1][jj * t + ll]);
                    orc_blk delta{orc_rnd(seed, DOM_DELTA, id) | 1, orc_rnd(seed, DOM_DELTA + 1, id)};
                    orc_blk r0{orc_rnd(seed, DOM_ROOT, id), orc_rnd(seed, DOM_ROOT + 1, id)};
                    roots0[id] = r0;
                    roots1[id] = bxor(r0, delta);
                    int rc = orc_dpf_deal(s->n, s->w, r0, delta, alpha, beta, rks, s->prg,
                                          cws + id * per, cw_out + id, nullptr, nullptr);
                    if (rc) return rc;
                }
    return 0;
}

// Keyed DPF per block -> output layer into the 2N-long g (pcg_ole_impl.h:
// 330-449) -> fold and step 4 (pcg_ole_impl.h:453-484).
int orc_expand(const orc_shape* s, int party, const orc_blk* roots,
               const orc_blk* cws, const uint64_t* cw_out, const uint64_t* pos,
               const uint64_t* val, const uint64_t* a, const uint8_t* rks,
               uint64_t blocks_mask, int threads, uint64_t* x, uint64_t* z,
               uint64_t* g_out) {
    const int N = s->N, c = s->c, t = s->t, B = t * t;
    const size_t D = static_cast<size_t>(1) << s->n, bin = D / 2;
    const size_t per = static_cast<size_t>(s->levels) * s->nk;
    std::vector<std::vector<uint64_t>> g(c * c);
    std::mutex mu;
    int next_block = 0;
    auto worker = [&]() {
        std::vector<orc_blk> leaves(D);
        for (;;) {
            int blk;
            {
                std::lock_guard<std::mutex> lk(mu);
                while (next_block < c * c && !((blocks_mask >> next_block) & 1)) ++next_block;
                if (next_block >= c * c) return;
                blk = next_block++;
            }
            std::vector<uint64_t> g2(2 * static_cast<size_t>(N), 0);
            for (int b = 0; b < B; ++b) {
                const size_t id = static_cast<size_t>(blk) * B + b;
                orc_dpf_keyed_full_eval(1, s->n, s->w, roots + id, cws + id * per, rks, s->prg,
                                        leaves.data());
                const size_t base = static_cast<size_t>(b / t + b % t) * bin;
                for (size_t d = 0; d < D; ++d) {
                    uint64_t y = orc_out_hash_lo64(leaves[d]) % P;
                    if (leaves[d].lo & 1) y = addm(y, cw_out[id]);
                    if (party == 1) y = subm(0, y);
                    g2[base + d] = addm(g2[base + d], y);
                }
            }
            std::vector<uint64_t> gr(N);
            for (int d = 0; d < N; ++d) gr[d] = subm(g2[d], g2[static_cast<size_t>(N) + d]);
            std::lock_guard<std::mutex> lk(mu);
            g[blk] = std::move(gr);
        }
    };
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    for (int b = 0; b < c * c; ++b) if (g[b].empty()) g[b].assign(N, 0);
    if (g_out)
        for (int b = 0; b < c * c; ++b)
            std::memcpy(g_out + static_cast<size_t>(b) * N, g[b].data(), sizeof(uint64_t) * N);

    // Step 4 with the reference's a_0 = 1, a_i = public_a[i-1].
    std::vector<uint64_t> a_all(static_cast<size_t>(c) * N, 0), g_all(static_cast<size_t>(c) * c * N);
    a_all[0] = 1;
    if (c > 1) std::memcpy(a_all.data() + N, a, sizeof(uint64_t) * N * (c - 1));
    for (int b = 0; b < c * c; ++b)
        std::memcpy(g_all.data() + static_cast<size_t>(b) * N, g[b].data(), sizeof(uint64_t) * N);
    return orc_step4(N, c, t, pos, val, a_all.data(), g_all.data(), x, z);
}

// Step 4 (pcg_ole_impl.h:455-483) for any public a_0 .. a_{c-1}:
// x = sum a_i e_i; z = sum_{i,j} (a_i a_j) g_ij.
int orc_step4(int N, int c, int t, const uint64_t* pos, const uint64_t* val, const uint64_t* a,
              const uint64_t* g, uint64_t* x, uint64_t* z) {
    std::vector<std::vector<uint64_t>> av(c, std::vector<uint64_t>(N, 0));
    for (int i = 0; i < c; ++i)
        for (int d = 0; d < N; ++d) av[i][d] = a[static_cast<size_t>(i) * N + d] % P;
    std::vector<uint64_t> acc(N, 0), tmp(N), e(N), aa(N), gb(N);
    for (int i = 0; i < c; ++i) {
        std::fill(e.begin(), e.end(), 0);
        for (int k = 0; k < t; ++k) e[pos[i * t + k] % N] = val[i * t + k] % P;
        poly_mul1(tmp.data(), av[i].data(), e.data(), N);
        for (int d = 0; d < N; ++d) acc[d] = addm(acc[d], tmp[d]);
    }
    std::memcpy(x, acc.data(), sizeof(uint64_t) * N);
    std::fill(acc.begin(), acc.end(), 0);
    for (int i = 0; i < c; ++i)
        for (int j = 0; j < c; ++j) {
            for (int d = 0; d < N; ++d) gb[d] = g[static_cast<size_t>(i * c + j) * N + d] % P;
            poly_mul1(aa.data(), av[i].data(), av[j].data(), N);
            poly_mul1(tmp.data(), aa.data(), gb.data(), N);
            for (int d = 0; d < N; ++d) acc[d] = addm(acc[d], tmp[d]);
        }
    std::memcpy(z, acc.data(), sizeof(uint64_t) * N);
    return 0;
}

int orc_bench_sample(const orc_shape* s, int party, const orc_blk* roots, const orc_blk* cws,
                     const uint64_t* cw_out, const uint64_t* a, int n_blocks,
                     int keys_per_block, int n_polymuls, int threads, double* t_dpf,
                     double* t_ntt) {
    const int N = s->N, t = s->t, B = t * t;
    const size_t D = static_cast<size_t>(1) << s->n, bin = D / 2;
    const size_t per = static_cast<size_t>(s->levels) * s->nk;
    if (threads < 1) threads = 1;
    if (keys_per_block <= 0 || keys_per_block > B) keys_per_block = B;
    if (n_blocks > s->c * s->c) n_blocks = s->c * s->c;
    using clk = std::chrono::steady_clock;
    // Part 1: the keyed DPF + output layer of the sampled keys (the per-key
    // work of orc_expand), keys spread over the threads, one 2N-long g per
    // thread and block (pcg_ole_impl.h:330-446).
    auto t0 = clk::now();
    {
        std::vector<std::thread> pool;
        const int total = n_blocks * keys_per_block;
        for (int w = 0; w < threads; ++w)
            pool.emplace_back([&, w] {
                std::vector<orc_blk> leaves(D);
                std::vector<uint64_t> g2(2 * static_cast<size_t>(N), 0);
                for (int k = w; k < total; k += threads) {
                    const int blk = k / keys_per_block, b = k % keys_per_block;
                    const size_t id = static_cast<size_t>(blk) * B + b;
                    orc_dpf_keyed_full_eval(1, s->n, s->w, roots + id, cws + id * per, nullptr,
                                            s->prg, leaves.data());
                    const size_t base = static_cast<size_t>(b / t + b % t) * bin;
                    for (size_t d = 0; d < D; ++d) {
                        uint64_t y = orc_out_hash_lo64(leaves[d]) % P;
                        if (leaves[d].lo & 1) y = addm(y, cw_out[id]);
                        if (party == 1) y = subm(0, y);
                        g2[base + d] = addm(g2[base + d], y);
                    }
                }
            });
        for (auto& th : pool) th.join();
    }
    auto t1 = clk::now();
    // Part 2: step-4 products (pcg_ole_impl.h:460-483), one per task.
    {
        std::vector<std::thread> pool;
        for (int w = 0; w < threads; ++w)
            pool.emplace_back([&, w] {
                std::vector<uint64_t> c(N);
                for (int k = w; k < n_polymuls; k += threads) {
                    const uint64_t* x = a + static_cast<size_t>(k % (s->c > 1 ? s->c - 1 : 1)) * N;
                    poly_mul1(c.data(), x, x, N);
                }
            });
        for (auto& th : pool) th.join();
    }
    auto t2 = clk::now();
    *t_dpf = std::chrono::duration<double>(t1 - t0).count();
    *t_ntt = std::chrono::duration<double>(t2 - t1).count();
    return 0;
}

// One whole unit of the expansion on the host: every key of block `blk`
// (DPF, output hash, convert and the scatter into the block's g, the
// per-thread partial g's summed at the end) and `n_polymuls` step-4 products
// (pcg_ole_impl.h:460-483), all from one task queue on `threads` threads,
// the products (the longest tasks) first.  Returns the wall seconds.
int orc_bench_block(const orc_shape* s, int party, const orc_blk* roots, const orc_blk* cws,
                    const uint64_t* cw_out, const uint64_t* a, int blk, int n_polymuls,
                    int threads, double* seconds) {
    const int N = s->N, t = s->t, B = t * t;
    const size_t D = static_cast<size_t>(1) << s->n, bin = D / 2;
    const size_t per = static_cast<size_t>(s->levels) * s->nk;
    if (threads < 1) threads = 1;
    if (blk < 0 || blk >= s->c * s->c || n_polymuls < 0) return -1;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    std::vector<std::vector<uint64_t>> g2(threads);
    std::atomic<int> next{0};
    const int tasks = n_polymuls + B;
    std::vector<std::thread> pool;
    for (int w = 0; w < threads; ++w)
        pool.emplace_back([&, w] {
            std::vector<orc_blk> leaves;
            std::vector<uint64_t> c;
            for (int k = next++; k < tasks; k = next++) {
                if (k < n_polymuls) {
                    c.resize(N);
                    const uint64_t* x = a + static_cast<size_t>(k % (s->c > 1 ? s->c - 1 : 1)) * N;
                    poly_mul1(c.data(), x, x, N);
                    continue;
                }
                const int b = k - n_polymuls;
                const size_t id = static_cast<size_t>(blk) * B + b;
                leaves.resize(D);
                if (g2[w].empty()) g2[w].assign(2 * static_cast<size_t>(N), 0);
                orc_dpf_keyed_full_eval(1, s->n, s->w, roots + id, cws + id * per, nullptr, s->prg,
                                        leaves.data());
                const size_t base = static_cast<size_t>(b / t + b % t) * bin;
                for (size_t d = 0; d < D; ++d) {
                    uint64_t y = orc_out_hash_lo64(leaves[d]) % P;
                    if (leaves[d].lo & 1) y = addm(y, cw_out[id]);
                    if (party == 1) y = subm(0, y);
                    g2[w][base + d] = addm(g2[w][base + d], y);
                }
            }
        });
    for (auto& th : pool) th.join();
    // The block's g: the threads' partial sums added word by word.
    std::vector<uint64_t> g(2 * static_cast<size_t>(N), 0);
    for (const auto& part : g2)
        if (!part.empty())
            for (size_t i = 0; i < g.size(); ++i) g[i] = addm(g[i], part[i]);
    *seconds = std::chrono::duration<double>(clk::now() - t0).count();
    return g[0] == P ? -2 : 0;   // keeps the sum live; g[0] < P always
}

// mt19937_64 (Matsumoto & Nishimura 2000; the parameters of C++
// std::mt19937_64), used to regenerate the reference's fixture inputs.
void orc_mt64_fill(uint64_t seed, uint64_t* out, size_t n) {
    const int NN = 312, MM = 156;
    const uint64_t MATRIX_A = 0xB5026F5AA96619E9ULL, UM = 0xFFFFFFFF80000000ULL,
                   LM = 0x7FFFFFFFULL;
    uint64_t mt[312];
    mt[0] = seed;
    for (int i = 1; i < NN; ++i)
        mt[i] = 6364136223846793005ULL * (mt[i - 1] ^ (mt[i - 1] >> 62)) + static_cast<uint64_t>(i);
    int mti = NN;
    for (size_t o = 0; o < n; ++o) {
        if (mti >= NN) {
            for (int i = 0; i < NN; ++i) {
                uint64_t x = (mt[i] & UM) | (mt[(i + 1) % NN] & LM);
                uint64_t v = mt[(i + MM) % NN] ^ (x >> 1);
                if (x & 1) v ^= MATRIX_A;
                mt[i] = v;
            }
            mti = 0;
        }
        uint64_t x = mt[mti++];
        x ^= (x >> 29) & 0x5555555555555555ULL;
        x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
        x ^= (x << 37) & 0xFFF7EEE000000000ULL;
        x ^= x >> 43;
        out[o] = x;
    }
}

}  // extern "C"
