// Negacyclic NTT over F_p, four-step form, for N = 2^logN (1 <= logN <= 24).
//
// N = n1 * n2 with n1 = 2^floor(logN/2), n2 = 2^ceil(logN/2); coefficient j
// sits at row j / n2, column j % n2.  With psi a primitive 2N-th root:
//   column pass: negacyclic NTT of length n1 on every column (root
//                psi1 = psi^n2);
//   row pass:    multiply element (k, j2) by the twiddle
//                psi^(j2 * (2*i1 + 1 - n1)), i1 = brev(k), then a
//                negacyclic NTT of length n2 on every row (root psi2 =
//                psi^n1).  The row transform's first stage has a single
//                root w0; it is folded into the twiddles of the row's upper
//                half, so that stage only adds and subtracts, and each
//                element costs one Shoup product by a (value, quotient)
//                pair where a Montgomery twiddle product and half a
//                butterfly product stood.
// Element (k, k2) then holds A(psi^(2*(i1 + n1*i2) + 1)) with i1 = brev(k),
// i2 = brev(k2): the evaluations of a(x) mod x^N + 1.  The row pass stores
// its outputs in a fixed permuted order (below) that every operand of a
// pointwise product shares; the inverse runs the passes backwards with
// inverse roots and folds N^-1 into its twiddle.
//
// Each sub-transform is the merged-twist Cooley-Tukey (forward) /
// Gentleman-Sande (inverse) negacyclic NTT of Longa and Naehrig (CANS 2016,
// Algorithms 1-2) with Harvey's lazy butterflies (J. Symbolic Comput. 60,
// 2014): forward values live in [0, 4p), inverse values in [0, 2p), which
// 4p < 2^64 allows, and a Shoup product by a precomputed root costs one high
// and two low 64-bit multiplies.
//
// Register blocking.  A thread owns E = 16 elements of one sub-transform of
// length n = 2^L (all n when n < 16), so T = n / 16 threads share it.  The L
// stages run in phases of four (radix 16) entirely in registers; between
// phases the elements are exchanged through shared memory.  In phase P
// (first stage s0 = 4P, r = min(4, L - s0) stages) a unit is the 2^r
// elements g*2^(L-s0) + j + k*tl (tl = 2^(L-s0-r), k < 2^r) that the phase
// combines; thread t owns units t*U .. t*U+U-1 (U = 16 / 2^r), unit u = (g,
// j) with g = u / tl, j = u % tl.  Phase 0 owns elements t + T*k, the last
// phase the 16 consecutive elements 16t .. 16t+15, so global loads and stores
// coalesce in both the column pass (lanes run over adjacent columns) and the
// row pass (lanes run over t).  Row-pass outputs of element i are stored at
// (i % 16) * T + i / 16 -- the permuted evaluation order.  Shared memory holds
// element i at (i + i/16) * stride, which keeps every exchange free of bank
// conflicts for the strides used here.
//
// The twiddle of stage s and butterfly group i = g*2^q + sub (q = s - s0) is
// stored at 2^s + sub*2^s0 + g, so the lanes of a warp read the same or
// adjacent table entries in every phase.
//
// The passes are two HBM sweeps per transform; the pointwise product with a
// resident operand and the multiply-accumulate over several transforms are
// fused into the row pass, where the forward phases end in the same register
// layout the inverse phases start from.  Replaces the reference's radix-2
// per-stage v1 kernels (GPU_baseline/common/poly_mul_cuda.cu:137-200) and its
// 20-kernel four-step (poly_mul_gpuntt_square.cu:171-613).
#include "pcgb_internal.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

#include "field.cuh"

namespace pcgb {

struct NttPlan {
    int logN = 0, l1 = 0, l2 = 0;
    size_t N = 0;
    int n1 = 0, n2 = 0;
    ulonglong2* tw1 = nullptr;    // column roots (value, shoup), phase-permuted
    ulonglong2* tw1i = nullptr;
    ulonglong2* tw2 = nullptr;    // row roots
    ulonglong2* tw2i = nullptr;
    // [n1][n2] four-step twiddles as Shoup pairs, the row transform's first
    // (forward) / last (inverse) root folded into the upper half of each row
    ulonglong2* Wf = nullptr;     // forward twiddle
    ulonglong2* Wif = nullptr;    // inverse twiddle * N^-1
    ulonglong2* WiRf = nullptr;   // Wif * 2^64: for products of two plain transforms
    std::mutex mu;                // guards the lazy WiRf
};

namespace {

constexpr uint64_t k2P = 2 * kPm;

// ---- lazy field arithmetic ------------------------------------------------

__device__ __forceinline__ uint64_t csub(uint64_t a, uint64_t m) { return a >= m ? a - m : a; }

// a*w mod p in [0, 2p) for any 64-bit a; wq = floor(w * 2^64 / p).
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t a, uint64_t w, uint64_t wq) {
    const uint64_t q = __umul64hi(a, wq);
    return a * w - q * kPm;
}

// Montgomery product a*b*2^-64 in [0, 2p) for a < 4p, b < p.
__device__ __forceinline__ uint64_t mont_lazy(uint64_t a, uint64_t b) {
    const uint64_t lo = a * b;
    const uint64_t hi = __umul64hi(a, b);
    const uint64_t m = lo * kPNegInv;
    return hi + __umul64hi(m, kPm) + (lo != 0 ? 1 : 0);
}

// Forward butterfly: X, Y in [0, 4p) -> X + wY, X - wY in [0, 4p).
__device__ __forceinline__ void ct_bfly(uint64_t& X, uint64_t& Y, ulonglong2 w) {
    const uint64_t x = csub(X, k2P);
    const uint64_t t = shoup_lazy(Y, w.x, w.y);
    X = x + t;
    Y = x - t + k2P;
}

// Inverse butterfly: X, Y in [0, 2p) -> X + Y, (X - Y) w in [0, 2p).
__device__ __forceinline__ void gs_bfly(uint64_t& X, uint64_t& Y, ulonglong2 w) {
    const uint64_t s = csub(X + Y, k2P);
    Y = shoup_lazy(X - Y + k2P, w.x, w.y);
    X = s;
}

// Butterfly of a stage whose root has been folded into the per-element
// twiddles (the row pass's first forward stage and last inverse stage):
// X, Y in [0, 2p) -> X + Y, X - Y in [0, 4p).
__device__ __forceinline__ void add_sub_bfly(uint64_t& X, uint64_t& Y) {
    const uint64_t s = X + Y;
    Y = X - Y + k2P;
    X = s;
}

// Shoup product with a per-element twiddle pair (value, quotient).
__device__ __forceinline__ uint64_t shoup_tw(uint64_t a, const ulonglong2* __restrict__ w) {
    const ulonglong2 v = __ldg(w);
    return shoup_lazy(a, v.x, v.y);
}

// ---- phase geometry ----------------------------------------------------------

template <int L>
struct Geo {
    static constexpr int n = 1 << L;
    static constexpr int E = L >= 4 ? 16 : n;         // elements per thread
    static constexpr int T = n / E;                    // threads per transform
    static constexpr int NPH = (L + 3) / 4;            // phases (0 when n = 1)
    static constexpr int PAD = n + n / 16;             // padded smem length
    __host__ __device__ static constexpr int r(int p) { return L - 4 * p < 4 ? L - 4 * p : 4; }
};

__host__ __device__ constexpr int last_phase(int L) { return L == 0 ? 0 : (L + 3) / 4 - 1; }

// Element index (within the transform) of register e of thread t in phase P.
template <int L, int P>
__device__ __forceinline__ int eidx(int t, int e) {
    constexpr int s0 = 4 * P, r = Geo<L>::r(P), U = Geo<L>::E >> r, ltl = L - s0 - r;
    const int v = e >> r, k = e & ((1 << r) - 1);
    const int u = t * U + v;
    return ((u >> ltl) << (L - s0)) + (u & ((1 << ltl) - 1)) + (k << ltl);
}

// Position of element i in the permuted row-output order.
template <int L>
__device__ __forceinline__ int perm_pos(int i) {
    if constexpr (L >= 4) return (i & 15) * Geo<L>::T + (i >> 4);
    else return i;
}

// FOLD: stage 0 (a single root) has that root folded into the per-element
// twiddles the caller applies (before the forward phases, after the inverse
// ones), so it is a plain add/sub; its inputs are in [0, 2p).
template <int L, int P, bool INV, bool FOLD>
__device__ __forceinline__ void run_phase(uint64_t (&x)[Geo<L>::E], int t,
                                          const ulonglong2* __restrict__ tw) {
    constexpr int s0 = 4 * P, r = Geo<L>::r(P), U = Geo<L>::E >> r, ltl = L - s0 - r;
#pragma unroll
    for (int v = 0; v < U; ++v) {
        const int g = (t * U + v) >> ltl;
        const int o = v << r;
        if constexpr (!INV) {
#pragma unroll
            for (int q = 0; q < r; ++q) {
#pragma unroll
                for (int sub = 0; sub < (1 << q); ++sub) {
                    if (FOLD && s0 + q == 0) {
#pragma unroll
                        for (int kk = 0; kk < (1 << (r - 1)); ++kk)
                            add_sub_bfly(x[o + kk], x[o + kk + (1 << (r - 1))]);
                        continue;
                    }
                    const ulonglong2 w = __ldg(tw + (1 << (s0 + q)) + (sub << s0) + g);
#pragma unroll
                    for (int kk = 0; kk < (1 << (r - 1 - q)); ++kk) {
                        const int k = o + (sub << (r - q)) + kk;
                        ct_bfly(x[k], x[k + (1 << (r - 1 - q))], w);
                    }
                }
            }
        } else {
            // Gentleman-Sande: the same stages, last to first (an ascending
            // counter keeps the loop fully unrolled and x in registers).
#pragma unroll
            for (int qq = 0; qq < r; ++qq) {
                const int q = r - 1 - qq;
#pragma unroll
                for (int sub = 0; sub < (1 << q); ++sub) {
                    if (FOLD && s0 + q == 0) {
#pragma unroll
                        for (int kk = 0; kk < (1 << (r - 1)); ++kk)
                            add_sub_bfly(x[o + kk], x[o + kk + (1 << (r - 1))]);
                        continue;
                    }
                    const ulonglong2 w = __ldg(tw + (1 << (s0 + q)) + (sub << s0) + g);
#pragma unroll
                    for (int kk = 0; kk < (1 << (r - 1 - q)); ++kk) {
                        const int k = o + (sub << (r - q)) + kk;
                        gs_bfly(x[k], x[k + (1 << (r - 1 - q))], w);
                    }
                }
            }
        }
    }
}

// Element i of one transform in shared memory: base[(i + i/16) * S].
template <int S>
struct SmemLay {
    uint64_t* base;
    __device__ __forceinline__ uint64_t& at(int i) const { return base[(i + (i >> 4)) * S]; }
};

// Registers in phase A layout -> shared memory -> registers in phase B layout.
template <int L, int A, int B, class Lay>
__device__ __forceinline__ void exchange(uint64_t (&x)[Geo<L>::E], int t, const Lay& lay) {
#pragma unroll
    for (int e = 0; e < Geo<L>::E; ++e) lay.at(eidx<L, A>(t, e)) = x[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e < Geo<L>::E; ++e) x[e] = lay.at(eidx<L, B>(t, e));
    __syncthreads();
}

// All forward phases: registers start in phase 0 layout, end in the last.
template <int L, bool FOLD, int P = 0, class Lay>
__device__ __forceinline__ void forward_all(uint64_t (&x)[Geo<L>::E], int t,
                                            const ulonglong2* __restrict__ tw, const Lay& lay) {
    if constexpr (P < Geo<L>::NPH) {
        if constexpr (P > 0) exchange<L, P - 1, P>(x, t, lay);
        run_phase<L, P, false, FOLD>(x, t, tw);
        forward_all<L, FOLD, P + 1>(x, t, tw, lay);
    }
}

// All inverse phases: registers start in the last phase layout, end in phase 0.
template <int L, bool FOLD, int P = Geo<L>::NPH - 1, class Lay>
__device__ __forceinline__ void inverse_all(uint64_t (&x)[Geo<L>::E], int t,
                                            const ulonglong2* __restrict__ twi, const Lay& lay) {
    if constexpr (P >= 0) {
        if constexpr (P < Geo<L>::NPH - 1) exchange<L, P + 1, P>(x, t, lay);
        run_phase<L, P, true, FOLD>(x, t, twi);
        inverse_all<L, FOLD, P - 1>(x, t, twi, lay);
    }
}

// ---- kernels -----------------------------------------------------------------

// Columns per CTA of the column passes.  Adjacent columns ride on adjacent
// lanes: 128-byte row segments up to n1 = 512, then 64, 32 and 16 bytes so
// that the CTA stays at 512 threads.  The column kernels are register-capped
// for two CTAs per SM (a few spilled words at n1 >= 512), so one CTA's loads
// overlap the other's butterflies; measured faster than one uncapped CTA.  (n2 >= n1 = 2^L, so C never exceeds
// the row length.)
__host__ __device__ constexpr int col_C(int L) {
    return L <= 3 ? (1 << L) : (L <= 9 ? 16 : (L == 10 ? 8 : (L == 11 ? 4 : 2)));
}
template <int L>
__host__ __device__ constexpr int col_threads() { return Geo<L>::T * col_C(L); }
// Transforms per CTA of the row passes (n1 >= 2^(L-1) rows exist).
template <int L>
__host__ __device__ constexpr int row_V() {
    constexpr int half = L >= 1 ? (1 << L) / 2 : 1;
    return Geo<L>::T >= 64 ? 1 : (64 / Geo<L>::T < half ? 64 / Geo<L>::T : half);
}
template <int L>
__host__ __device__ constexpr int row_threads() { return Geo<L>::T * row_V<L>(); }

// ---- pass bodies ---------------------------------------------------------------
// Shared by the per-length kernels (one length, batch in gridDim.y) and the
// mixed-length kernels (a job table names each CTA's polynomial and tile).
// Pointers arrive already offset to the polynomial's first word.

// Column pass, forward, for columns [tile*C, tile*C + C).  src may equal
// dst (every CTA loads its columns before its first store).  REDUCE maps
// arbitrary 64-bit inputs into [0, p) first; otherwise inputs must be below
// 4p.  Outputs in [0, 4p), without the four-step twiddle: the row pass
// applies it together with its own first root.  L2 >= 0 fixes log2(n2) at
// compile time (element offsets become immediates); -1 takes l2.
template <int L, int C, bool REDUCE, int L2 = -1>
__device__ __forceinline__ void col_fwd_body(const uint64_t* src, uint64_t* dst, int l2,
                                             size_t tile, const ulonglong2* __restrict__ tw,
                                             uint64_t* sm) {
    constexpr int E = Geo<L>::E, LP = last_phase(L);
    const int t = threadIdx.x / C, c = threadIdx.x % C;
    const size_t n2 = size_t{1} << (L2 >= 0 ? L2 : l2);
    const size_t col = tile * C + c;
    uint64_t x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint64_t v = src[col + eidx<L, 0>(t, e) * n2];
        x[e] = REDUCE ? reduce_p(v) : v;
    }
    forward_all<L, false>(x, t, tw, SmemLay<C>{sm + c});
#pragma unroll
    for (int e = 0; e < E; ++e) dst[col + eidx<L, LP>(t, e) * n2] = x[e];
}

// Column pass, inverse, in place (output in natural coefficient order, in
// [0, p)).  L2 as in col_fwd_body.
template <int L, int C, int L2 = -1>
__device__ __forceinline__ void col_inv_body(uint64_t* d, int l2, size_t tile,
                                             const ulonglong2* __restrict__ twi, uint64_t* sm) {
    constexpr int E = Geo<L>::E, LP = last_phase(L);
    const int t = threadIdx.x / C, c = threadIdx.x % C;
    const size_t n2 = size_t{1} << (L2 >= 0 ? L2 : l2);
    const size_t col = tile * C + c;
    uint64_t x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = d[col + eidx<L, LP>(t, e) * n2];
    inverse_all<L, false>(x, t, twi, SmemLay<C>{sm + c});
#pragma unroll
    for (int e = 0; e < E; ++e) d[col + eidx<L, 0>(t, e) * n2] = csub(x[e], kPm);
}

// Row pass, forward, in place on rows [tile*V, tile*V + V) (each thread
// reads and writes the same set of positions): the four-step twiddle with
// the row transform's first root folded in (Wf, per element), then the row
// transform; outputs in [0, p) in the permuted order.
template <int L, int V>
__device__ __forceinline__ void row_fwd_body(uint64_t* d, size_t tile,
                                             const ulonglong2* __restrict__ tw,
                                             const ulonglong2* __restrict__ Wf, uint64_t* sm) {
    constexpr int E = Geo<L>::E, T = Geo<L>::T, LP = last_phase(L);
    const int t = threadIdx.x % T, v = threadIdx.x / T;
    const size_t base = (tile * V + v) * Geo<L>::n;
    uint64_t* row = d + base;
    uint64_t x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = eidx<L, 0>(t, e);
        x[e] = shoup_tw(row[i], Wf + base + i);
    }
    forward_all<L, true>(x, t, tw, SmemLay<1>{sm + v * Geo<L>::PAD});
#pragma unroll
    for (int e = 0; e < E; ++e)
        row[perm_pos<L>(eidx<L, LP>(t, e))] = csub(csub(x[e], k2P), kPm);
}

// Multiply-accumulate row pass on rows [tile*V, tile*V + V):
//   out row = Wi (.) INTT( sum_q NTT(g_q row) (.) img_q row ),
// g_q = g + q*N, img_q = img + q*N; img_q in the permuted evaluation order,
// Montgomery-scaled so that the Montgomery product gives the plain one.
// g rows come from the column pass (Wf, the forward twiddle, is applied
// here as in row_fwd_body); Wif is the inverse twiddle with the inverse
// row transform's last root folded in.  out is in [0, p) and may alias g
// (a CTA reads all its rows before its first store).  ONE (Q == 1, a plain
// product): the product stays in the transform's registers, with no
// separate accumulator live across the forward phases.
template <int L, int V, bool ONE>
__device__ __forceinline__ void row_mac_body(const uint64_t* g, const uint64_t* __restrict__ img,
                                             int Q, size_t N, size_t tile,
                                             const ulonglong2* __restrict__ tw,
                                             const ulonglong2* __restrict__ twi,
                                             const ulonglong2* __restrict__ Wf,
                                             const ulonglong2* __restrict__ Wif, uint64_t* out,
                                             uint64_t* sm) {
    constexpr int E = Geo<L>::E, T = Geo<L>::T, LP = last_phase(L);
    const int t = threadIdx.x % T, v = threadIdx.x / T;
    const size_t base = (tile * V + v) * Geo<L>::n;
    const SmemLay<1> lay{sm + v * Geo<L>::PAD};
    uint64_t acc[E];
    if constexpr (ONE) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const size_t i = base + eidx<L, 0>(t, e);
            acc[e] = shoup_tw(g[i], Wf + i);
        }
        forward_all<L, true>(acc, t, tw, lay);
#pragma unroll
        for (int e = 0; e < E; ++e)
            acc[e] = mont_lazy(acc[e], __ldg(img + base + perm_pos<L>(eidx<L, LP>(t, e))));
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) acc[e] = 0;
        for (int q = 0; q < Q; ++q) {
            const uint64_t* gr = g + q * N + base;
            const uint64_t* im = img + q * N + base;
            uint64_t x[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = eidx<L, 0>(t, e);
                x[e] = shoup_tw(gr[i], Wf + base + i);
            }
            forward_all<L, true>(x, t, tw, lay);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const uint64_t m = mont_lazy(x[e], __ldg(im + perm_pos<L>(eidx<L, LP>(t, e))));
                acc[e] = csub(acc[e] + m, k2P);
            }
        }
    }
    inverse_all<L, true>(acc, t, twi, lay);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const size_t i = base + eidx<L, 0>(t, e);
        out[i] = csub(shoup_tw(acc[e], Wif + i), kPm);
    }
}

// Pointwise product and inverse row pass on rows [tile*V, tile*V + V) of a
// transform already in the permuted evaluation order (row_fwd_body's
// output): out row = Wi (.) INTT( d row (.) img row ), in place, Wi given
// as WiRf (the inverse twiddle times 2^64, which cancels the Montgomery
// product's 2^-64, with the last root folded in).  Each thread loads the
// permuted positions of its last-phase registers, so the inverse starts
// where the fused forward would have ended.
template <int L, int V>
__device__ __forceinline__ void row_pmul_inv_body(uint64_t* d, const uint64_t* __restrict__ img,
                                                  size_t tile, const ulonglong2* __restrict__ twi,
                                                  const ulonglong2* __restrict__ WiRf,
                                                  uint64_t* sm) {
    constexpr int E = Geo<L>::E, T = Geo<L>::T, LP = last_phase(L);
    const int t = threadIdx.x % T, v = threadIdx.x / T;
    const size_t base = (tile * V + v) * Geo<L>::n;
    uint64_t x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const size_t i = base + perm_pos<L>(eidx<L, LP>(t, e));
        x[e] = mont_lazy(d[i], __ldg(img + i));
    }
    inverse_all<L, true>(x, t, twi, SmemLay<1>{sm + v * Geo<L>::PAD});
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const size_t i = base + eidx<L, 0>(t, e);
        d[i] = csub(shoup_tw(x[e], WiRf + i), kPm);
    }
}

// ---- per-length kernels: grid = (tiles, batch) ---------------------------------

// The column kernels fix the row length: l2 = L + DL (l2 - l1 is 0 or 1).
template <int L, bool REDUCE, int DL>
__global__ void __launch_bounds__(col_threads<L>(), 2) col_fwd_kernel(
    const uint64_t* src, uint64_t* dst, const ulonglong2* __restrict__ tw) {
    extern __shared__ uint64_t sm[];
    const size_t off = static_cast<size_t>(blockIdx.y) << (2 * L + DL);
    col_fwd_body<L, col_C(L), REDUCE, L + DL>(src + off, dst + off, L + DL, blockIdx.x, tw, sm);
}

template <int L, int DL>
__global__ void __launch_bounds__(col_threads<L>(), 2) col_inv_kernel(
    uint64_t* d, const ulonglong2* __restrict__ twi) {
    extern __shared__ uint64_t sm[];
    col_inv_body<L, col_C(L), L + DL>(d + (static_cast<size_t>(blockIdx.y) << (2 * L + DL)),
                                      L + DL, blockIdx.x, twi, sm);
}

template <int L>
__global__ void __launch_bounds__(row_threads<L>()) row_fwd_kernel(
    uint64_t* d, int l1, const ulonglong2* __restrict__ tw, const ulonglong2* __restrict__ Wf) {
    extern __shared__ uint64_t sm[];
    row_fwd_body<L, row_V<L>()>(d + (static_cast<size_t>(blockIdx.y) << (L + l1)), blockIdx.x,
                                tw, Wf, sm);
}

template <int L>
__global__ void __launch_bounds__(row_threads<L>()) row_pmul_inv_kernel(
    uint64_t* d, const uint64_t* __restrict__ img, int l1, const ulonglong2* __restrict__ twi,
    const ulonglong2* __restrict__ WiRf) {
    extern __shared__ uint64_t sm[];
    const size_t off = static_cast<size_t>(blockIdx.y) << (L + l1);
    row_pmul_inv_body<L, row_V<L>()>(d + off, img + off, blockIdx.x, twi, WiRf, sm);
}

// Instance b reads g and img at b*Q*N and writes out at b*N.
template <int L, bool ONE>
__global__ void __launch_bounds__(row_threads<L>()) row_mac_inv_kernel(
    const uint64_t* g, const uint64_t* __restrict__ img, int Q, int l1,
    const ulonglong2* __restrict__ tw, const ulonglong2* __restrict__ twi,
    const ulonglong2* __restrict__ Wf, const ulonglong2* __restrict__ Wif, uint64_t* out) {
    extern __shared__ uint64_t sm[];
    const size_t N = size_t{1} << (L + l1);
    const size_t b = blockIdx.y;
    row_mac_body<L, row_V<L>(), ONE>(g + b * Q * N, img + b * Q * N, Q, N, blockIdx.x, tw, twi,
                                     Wf, Wif, out + b * N, sm);
}

// ---- mixed-length kernels --------------------------------------------------------
// One launch per pass over a batch of products whose lengths range over
// 2^16 .. 2^20 (sub-lengths 2^8 .. 2^10 in both passes).  At these lengths
// every column CTA holds 512 threads x 16 elements (C = 32, 16, 8 columns)
// and every row CTA 64 threads (V = 4, 2, 1 rows), with the same shared
// memory, so one launch shape serves every length; each CTA reads its
// polynomial and tile from a job table and runs that length's body.

struct MixedPoly {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* c;
    uint64_t* A;                 // NTT(a), scratch
    const ulonglong2* tw1;
    const ulonglong2* tw1i;
    const ulonglong2* tw2;
    const ulonglong2* tw2i;
    const ulonglong2* Wf;
    const ulonglong2* WiRf;
    int l1, l2;
};
struct MixedCta {
    uint32_t poly, tile;
};
constexpr int kMixedColThreads = 512, kMixedRowThreads = 64;
constexpr int kMixedLmin = 8, kMixedLmax = 10;
template <int L>
__host__ __device__ constexpr int mixed_C() { return kMixedColThreads / Geo<L>::T; }
template <int L>
__host__ __device__ constexpr int mixed_V() { return kMixedRowThreads / Geo<L>::T; }
static_assert(mixed_V<8>() == row_V<8>() && mixed_V<9>() == row_V<9>() &&
              mixed_V<10>() == row_V<10>(), "row CTA shapes agree");
constexpr size_t kMixedColSmem = sizeof(uint64_t) * Geo<10>::PAD * mixed_C<10>();
constexpr size_t kMixedRowSmem = sizeof(uint64_t) * Geo<10>::PAD * mixed_V<10>();
static_assert(sizeof(uint64_t) * Geo<8>::PAD * mixed_C<8>() == kMixedColSmem &&
              sizeof(uint64_t) * Geo<9>::PAD * mixed_C<9>() == kMixedColSmem, "col smem");

#define PCGB_MIXED_SWITCH(LEN, CALL) \
    switch (LEN) {                    \
        case 8: CALL(8); break;       \
        case 9: CALL(9); break;       \
        case 10: CALL(10); break;     \
        default: break;               \
    }
// Column passes: (l1, l2) pairs, l2 = l1 or l1 + 1, both compile-time.
#define PCGB_MIXED_COL_SWITCH(P1, P2, CALL)           \
    switch (2 * (P1) + ((P2) - (P1))) {                \
        case 16: CALL(8, 8); break;                    \
        case 17: CALL(8, 9); break;                    \
        case 18: CALL(9, 9); break;                    \
        case 19: CALL(9, 10); break;                   \
        case 20: CALL(10, 10); break;                  \
        default: break;                                \
    }

// which = 0: column pass of a into A; which = 1: column pass of b into c.
__global__ void __launch_bounds__(kMixedColThreads, 2) mixed_col_fwd_kernel(
    const MixedPoly* __restrict__ polys, const MixedCta* __restrict__ ctas, int which) {
    extern __shared__ uint64_t sm[];
    const MixedCta j = ctas[blockIdx.x];
    const MixedPoly& p = polys[j.poly];
    const uint64_t* src = which ? p.b : p.a;
    uint64_t* dst = which ? p.c : p.A;
#define PCGB_CALL(LL, L2) \
    col_fwd_body<LL, mixed_C<LL>(), true, L2>(src, dst, L2, j.tile, p.tw1, sm)
    PCGB_MIXED_COL_SWITCH(p.l1, p.l2, PCGB_CALL)
#undef PCGB_CALL
}

__global__ void __launch_bounds__(kMixedRowThreads) mixed_row_fwd_kernel(
    const MixedPoly* __restrict__ polys, const MixedCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MixedCta j = ctas[blockIdx.x];
    const MixedPoly& p = polys[j.poly];
#define PCGB_CALL(LL) row_fwd_body<LL, mixed_V<LL>()>(p.A, j.tile, p.tw2, p.Wf, sm)
    PCGB_MIXED_SWITCH(p.l2, PCGB_CALL)
#undef PCGB_CALL
}

// c = Wi*R (.) INTT( NTT_rows(c) (.) A ), in place on c.
__global__ void __launch_bounds__(kMixedRowThreads) mixed_row_mac_kernel(
    const MixedPoly* __restrict__ polys, const MixedCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MixedCta j = ctas[blockIdx.x];
    const MixedPoly& p = polys[j.poly];
    const size_t N = size_t{1} << (p.l1 + p.l2);
#define PCGB_CALL(LL) \
    row_mac_body<LL, mixed_V<LL>(), true>(p.c, p.A, 1, N, j.tile, p.tw2, p.tw2i, p.Wf, p.WiRf, \
                                          p.c, sm)
    PCGB_MIXED_SWITCH(p.l2, PCGB_CALL)
#undef PCGB_CALL
}

__global__ void __launch_bounds__(kMixedColThreads, 2) mixed_col_inv_kernel(
    const MixedPoly* __restrict__ polys, const MixedCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MixedCta j = ctas[blockIdx.x];
    const MixedPoly& p = polys[j.poly];
#define PCGB_CALL(LL, L2) col_inv_body<LL, mixed_C<LL>(), L2>(p.c, L2, j.tile, p.tw1i, sm)
    PCGB_MIXED_COL_SWITCH(p.l1, p.l2, PCGB_CALL)
#undef PCGB_CALL
}
#undef PCGB_MIXED_SWITCH
#undef PCGB_MIXED_COL_SWITCH

// ---- multi-request multiply-accumulate ------------------------------------
// The step-4 transforms of several expansions of different lengths
// 2^14 .. 2^20 (sub-lengths 2^7 .. 2^10) in three launches: the column pass
// of every request's Q g' buffers, the Q-way multiply-accumulate row pass
// with its inverse, and the inverse column pass into each request's z.  The
// CTA shapes are the mixed kernels' (512 column threads, 64 row threads,
// the same shared memory at every sub-length down to 2^7).
struct MacReq {
    uint64_t* g;                 // Q*N words, column-transformed in place
    const uint64_t* img;         // Q*N, Montgomery-scaled evaluation images
    uint64_t* z;                 // N
    const ulonglong2* tw1;
    const ulonglong2* tw1i;
    const ulonglong2* tw2;
    const ulonglong2* tw2i;
    const ulonglong2* Wf;
    const ulonglong2* Wif;
    int Q, l1, l2;
};
struct MacCta {
    uint32_t req, q, tile;
};
constexpr int kMacLmin = 7;
static_assert(sizeof(uint64_t) * Geo<7>::PAD * mixed_C<7>() == kMixedColSmem &&
              sizeof(uint64_t) * Geo<7>::PAD * mixed_V<7>() == kMixedRowSmem,
              "sub-length 2^7 fits the mixed CTA shapes");

#define PCGB_MAC_SWITCH(LEN, CALL) \
    switch (LEN) {                  \
        case 7: CALL(7); break;     \
        case 8: CALL(8); break;     \
        case 9: CALL(9); break;     \
        case 10: CALL(10); break;   \
        default: break;             \
    }
#define PCGB_MAC_COL_SWITCH(P1, P2, CALL)             \
    switch (2 * (P1) + ((P2) - (P1))) {                \
        case 14: CALL(7, 7); break;                    \
        case 15: CALL(7, 8); break;                    \
        case 16: CALL(8, 8); break;                    \
        case 17: CALL(8, 9); break;                    \
        case 18: CALL(9, 9); break;                    \
        case 19: CALL(9, 10); break;                   \
        case 20: CALL(10, 10); break;                  \
        default: break;                                \
    }

__global__ void __launch_bounds__(kMixedColThreads, 2) mac_col_fwd_kernel(
    const MacReq* __restrict__ reqs, const MacCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MacCta j = ctas[blockIdx.x];
    const MacReq& r = reqs[j.req];
    uint64_t* d = r.g + (static_cast<size_t>(j.q) << (r.l1 + r.l2));
#define PCGB_CALL(LL, L2) col_fwd_body<LL, mixed_C<LL>(), false, L2>(d, d, L2, j.tile, r.tw1, sm)
    PCGB_MAC_COL_SWITCH(r.l1, r.l2, PCGB_CALL)
#undef PCGB_CALL
}

__global__ void __launch_bounds__(kMixedRowThreads) mac_row_kernel(
    const MacReq* __restrict__ reqs, const MacCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MacCta j = ctas[blockIdx.x];
    const MacReq& r = reqs[j.req];
    const size_t N = size_t{1} << (r.l1 + r.l2);
#define PCGB_CALL(LL) \
    row_mac_body<LL, mixed_V<LL>(), false>(r.g, r.img, r.Q, N, j.tile, r.tw2, r.tw2i, r.Wf, r.Wif, \
                                           r.z, sm)
    PCGB_MAC_SWITCH(r.l2, PCGB_CALL)
#undef PCGB_CALL
}

__global__ void __launch_bounds__(kMixedColThreads, 2) mac_col_inv_kernel(
    const MacReq* __restrict__ reqs, const MacCta* __restrict__ ctas) {
    extern __shared__ uint64_t sm[];
    const MacCta j = ctas[blockIdx.x];
    const MacReq& r = reqs[j.req];
#define PCGB_CALL(LL, L2) col_inv_body<LL, mixed_C<LL>(), L2>(r.z, L2, j.tile, r.tw1i, sm)
    PCGB_MAC_COL_SWITCH(r.l1, r.l2, PCGB_CALL)
#undef PCGB_CALL
}
#undef PCGB_MAC_SWITCH
#undef PCGB_MAC_COL_SWITCH

// Shoup pair (v, floor(v * 2^64 / p)) of v < p given in Montgomery form
// vR = v * 2^64 mod p: the quotient is (v * 2^64 - vR) / p, an exact
// division, so it equals vR * (-p^-1) mod 2^64.
__device__ __forceinline__ ulonglong2 shoup_pair_from_mont(uint64_t vR) {
    return make_ulonglong2(mont_mul(vR, 1), vR * kPNegInv);
}

// Twiddle tables, element k*n2 + j2 with e = j2*(2*brev(k)+1-n1) mod 2N:
//   Wf  = psi^e,          times w0 = psi2^(n2/2) for j2 >= n2/2,
//   Wif = psi^-e * N^-1,  times w0i = psi2^-(n2/2) for j2 >= n2/2,
// w0 / w0i being the single root of the row transform's first forward /
// last inverse stage (that stage then only adds and subtracts).
// powR[b] = psi^(2^b) * R mod p; w0R, w0iR are w0, w0i times R.
__global__ void twiddle_kernel(ulonglong2* Wf, ulonglong2* Wif, int l1, int l2,
                               const uint64_t* __restrict__ powR, uint64_t oneR, uint64_t ninvR,
                               uint64_t w0R, uint64_t w0iR) {
    const size_t N = static_cast<size_t>(1) << (l1 + l2);
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= N) return;
    const int n1 = 1 << l1;
    const uint32_t k = static_cast<uint32_t>(idx >> l2);
    const uint32_t j2 = static_cast<uint32_t>(idx & ((1u << l2) - 1));
    const uint32_t i1 = l1 ? (__brev(k) >> (32 - l1)) : 0;
    const int64_t twoN = static_cast<int64_t>(2 * N);
    int64_t e = (static_cast<int64_t>(j2) * (2 * static_cast<int64_t>(i1) + 1 - n1)) % twoN;
    if (e < 0) e += twoN;
    const int64_t ei = (twoN - e) % twoN;
    uint64_t a = oneR, b = oneR;
    for (int bit = 0; bit <= l1 + l2; ++bit) {
        if ((e >> bit) & 1) a = mont_mul(a, powR[bit]);
        if ((ei >> bit) & 1) b = mont_mul(b, powR[bit]);
    }
    b = mont_mul(b, ninvR);        // psi^-e * N^-1 * R
    if (j2 >= (1u << (l2 - 1))) {
        a = mont_mul(a, w0R);
        b = mont_mul(b, w0iR);
    }
    Wf[idx] = shoup_pair_from_mont(a);
    Wif[idx] = shoup_pair_from_mont(b);
}

// dst = src * 2^64 mod p, Shoup pairs; r2 = 2^128 mod p.
__global__ void scale_r_kernel(ulonglong2* dst, const ulonglong2* __restrict__ src, size_t n,
                               uint64_t r2) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t vR = mont_mul(src[i].x, r2);      // v * R: the new value
    dst[i] = shoup_pair_from_mont(mont_mul(vR, r2));  // from its Montgomery form
}

// Pointwise products, one word per thread.
//   mode 0: c = a*b*R^-1          (Montgomery product)
//   mode 1: c = a*b               (plain product; r2 = R^2 mod p)
__global__ void pointwise_kernel(uint64_t* c, const uint64_t* a, const uint64_t* b, size_t n,
                                 int mode, uint64_t r2) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t v = mont_mul(a[i], b[i]);
    if (mode == 1) v = mont_mul(v, r2);
    c[i] = v;
}

__global__ void reduce_kernel(uint64_t* d, const uint64_t* s, size_t n) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) d[i] = reduce_p(s[i]);
}

// ---- host side ---------------------------------------------------------------

uint32_t brev_host(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

// Smallest primitive root of F_p, as the reference's NTT picks it
// (CPU_baseline/ntt.h:200-222): p - 1 = 2^25 * 47189 * 2912521, and g is
// primitive iff g^((p-1)/q) != 1 for each prime q | p - 1.  (It is 3.)  The
// slot values of a transform, which triples expose, depend on this choice.
uint64_t primitive_root_host() {
    constexpr uint64_t kQ[3] = {2, 47189, 2912521};
    static_assert((kPm - 1) == (uint64_t{1} << 25) * 47189ULL * 2912521ULL, "p - 1 factors");
    for (uint64_t g = 2;; ++g) {
        bool ok = true;
        for (uint64_t q : kQ) ok = ok && pow_p_host(g, (kPm - 1) / q) != 1;
        if (ok) return g;
    }
}

// Roots of a length-2^logn negacyclic transform with psi_n a primitive
// 2n-th root: stage s, group i uses psi_n^brev_logn(2^s + i) (Longa-Naehrig
// table), stored at the phase-permuted slot 2^s + (i % 2^q) * 2^s0 + i / 2^q.
ulonglong2* upload_root_table(uint64_t psi_n, int logn) {
    const int n = 1 << logn;
    std::vector<uint64_t> pw(n);
    uint64_t a = 1;
    for (int k = 0; k < n; ++k) { pw[k] = a; a = mul_p_host(a, psi_n); }
    std::vector<ulonglong2> tab(n > 1 ? n : 2, make_ulonglong2(0, 0));
    for (int s = 0; s < logn; ++s) {
        const int s0 = 4 * (s / 4), q = s - s0;
        for (int i = 0; i < (1 << s); ++i) {
            const uint64_t v = pw[brev_host(static_cast<uint32_t>((1 << s) + i), logn)];
            const int slot = (1 << s) + ((i & ((1 << q) - 1)) << s0) + (i >> q);
            tab[slot] = make_ulonglong2(v, shoup_q_host(v));
        }
    }
    ulonglong2* d = nullptr;
    PCGB_CK(cudaMalloc(&d, sizeof(ulonglong2) * tab.size()));
    upload_blocking(d, tab.data(), sizeof(ulonglong2) * tab.size());
    return d;
}

NttPlan* build_plan(int logN) {
    auto* pl = new NttPlan();
    pl->logN = logN;
    pl->N = static_cast<size_t>(1) << logN;
    pl->l1 = logN / 2;
    pl->l2 = logN - pl->l1;
    pl->n1 = 1 << pl->l1;
    pl->n2 = 1 << pl->l2;
    const uint64_t g = primitive_root_host();
    const uint64_t psi = pow_p_host(g, (kPm - 1) / (2 * pl->N));
    const uint64_t psi_inv = pow_p_host(psi, kPm - 2);
    pl->tw1 = upload_root_table(pow_p_host(psi, pl->n2), pl->l1);
    pl->tw1i = upload_root_table(pow_p_host(psi_inv, pl->n2), pl->l1);
    pl->tw2 = upload_root_table(pow_p_host(psi, pl->n1), pl->l2);
    pl->tw2i = upload_root_table(pow_p_host(psi_inv, pl->n1), pl->l2);
    PCGB_CK(cudaMalloc(&pl->Wf, sizeof(ulonglong2) * pl->N));
    PCGB_CK(cudaMalloc(&pl->Wif, sizeof(ulonglong2) * pl->N));
    const uint64_t R = r_mod_p();
    std::vector<uint64_t> powR(logN + 2);
    uint64_t pb = psi;
    for (int b = 0; b < logN + 2; ++b) { powR[b] = mul_p_host(pb, R); pb = mul_p_host(pb, pb); }
    uint64_t* d_pow = nullptr;
    PCGB_CK(cudaMalloc(&d_pow, sizeof(uint64_t) * powR.size()));
    upload_blocking(d_pow, powR.data(), sizeof(uint64_t) * powR.size());
    const uint64_t ninvR = mul_p_host(pow_p_host(pl->N % kPm, kPm - 2), R);
    // The row transform's stage-0 root: psi2^brev(1) = psi2^(n2/2) = psi^(N/2).
    const uint64_t w0R = mul_p_host(pow_p_host(psi, pl->N / 2), R);
    const uint64_t w0iR = mul_p_host(pow_p_host(psi_inv, pl->N / 2), R);
    twiddle_kernel<<<static_cast<unsigned>((pl->N + 255) / 256), 256>>>(
        pl->Wf, pl->Wif, pl->l1, pl->l2, d_pow, R, ninvR, w0R, w0iR);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaDeviceSynchronize());
    cudaFree(d_pow);
    return pl;
}

template <int L>
constexpr size_t col_smem() { return Geo<L>::NPH > 1 ? sizeof(uint64_t) * Geo<L>::PAD * col_C(L) : 0; }
template <int L>
constexpr size_t row_smem() { return Geo<L>::NPH > 1 ? sizeof(uint64_t) * Geo<L>::PAD * row_V<L>() : 0; }

// Once per kernel and device: opt into dynamic shared memory above 48 KB and
// ask for the largest shared-memory carveout, so the CTAs that the register
// budget admits are not limited by a smaller L1/shared split.
struct OptinOnce {
    std::mutex mu;
    std::map<std::pair<const void*, int>, bool> done;
    template <class K>
    void operator()(K* kernel, size_t bytes) {
        if (bytes == 0) return;
        int dev = 0;
        PCGB_CK(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu);
        auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
        if (done[key]) return;
        const void* f = reinterpret_cast<const void*>(kernel);
        if (bytes > 48 * 1024)
            PCGB_CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bytes)));
        PCGB_CK(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
        done[key] = true;
    }
};
OptinOnce g_optin;

template <int L>
void col_fwd_l(const NttPlan& pl, const uint64_t* src, uint64_t* dst, int batch, bool reduce,
               cudaStream_t st) {
    constexpr size_t sm = col_smem<L>();
    const dim3 grid(pl.n2 / col_C(L), batch);
    auto go = [&](auto kernel) {
        g_optin(kernel, sm);
        kernel<<<grid, col_threads<L>(), sm, st>>>(src, dst, pl.tw1);
    };
    const bool odd = pl.l2 != L;
    if (reduce) odd ? go(col_fwd_kernel<L, true, 1>) : go(col_fwd_kernel<L, true, 0>);
    else odd ? go(col_fwd_kernel<L, false, 1>) : go(col_fwd_kernel<L, false, 0>);
    PCGB_POST_LAUNCH();
}

template <int L>
void col_inv_l(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    constexpr size_t sm = col_smem<L>();
    auto go = [&](auto kernel) {
        g_optin(kernel, sm);
        kernel<<<dim3(pl.n2 / col_C(L), batch), col_threads<L>(), sm, st>>>(d, pl.tw1i);
    };
    pl.l2 != L ? go(col_inv_kernel<L, 1>) : go(col_inv_kernel<L, 0>);
    PCGB_POST_LAUNCH();
}

template <int L>
void row_fwd_l(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    constexpr size_t sm = row_smem<L>();
    g_optin(row_fwd_kernel<L>, sm);
    row_fwd_kernel<L><<<dim3(pl.n1 / row_V<L>(), batch), row_threads<L>(), sm, st>>>(d, pl.l1,
                                                                                    pl.tw2, pl.Wf);
    PCGB_POST_LAUNCH();
}

template <int L>
void row_pmul_inv_l(const NttPlan& pl, uint64_t* d, const uint64_t* img, int batch,
                    const ulonglong2* WiRf, cudaStream_t st) {
    constexpr size_t sm = row_smem<L>();
    g_optin(row_pmul_inv_kernel<L>, sm);
    row_pmul_inv_kernel<L><<<dim3(pl.n1 / row_V<L>(), batch), row_threads<L>(), sm, st>>>(
        d, img, pl.l1, pl.tw2i, WiRf);
    PCGB_POST_LAUNCH();
}

template <int L>
void row_mac_l(const NttPlan& pl, const uint64_t* g, const uint64_t* img, int Q, int batch,
               const ulonglong2* Wif, uint64_t* out, cudaStream_t st) {
    constexpr size_t sm = row_smem<L>();
    const dim3 grid(pl.n1 / row_V<L>(), batch);
    if (Q == 1) {
        g_optin(row_mac_inv_kernel<L, true>, sm);
        row_mac_inv_kernel<L, true><<<grid, row_threads<L>(), sm, st>>>(g, img, Q, pl.l1, pl.tw2,
                                                                        pl.tw2i, pl.Wf, Wif, out);
    } else {
        g_optin(row_mac_inv_kernel<L, false>, sm);
        row_mac_inv_kernel<L, false><<<grid, row_threads<L>(), sm, st>>>(g, img, Q, pl.l1, pl.tw2,
                                                                         pl.tw2i, pl.Wf, Wif, out);
    }
    PCGB_POST_LAUNCH();
}

// Runtime sub-length -> template instance (2^0 .. 2^12).
template <class F>
void by_len(int L, F&& f) {
    switch (L) {
        case 0: f(std::integral_constant<int, 0>{}); break;
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 5: f(std::integral_constant<int, 5>{}); break;
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        case 11: f(std::integral_constant<int, 11>{}); break;
        case 12: f(std::integral_constant<int, 12>{}); break;
        default: fail(PCGB_EINVAL, "NTT sub-length out of range");
    }
}

void col_fwd(const NttPlan& pl, const uint64_t* src, uint64_t* dst, int batch, bool reduce,
             cudaStream_t st) {
    by_len(pl.l1, [&](auto L) { col_fwd_l<decltype(L)::value>(pl, src, dst, batch, reduce, st); });
}
void col_inv(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    by_len(pl.l1, [&](auto L) { col_inv_l<decltype(L)::value>(pl, d, batch, st); });
}
void row_fwd(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    by_len(pl.l2, [&](auto L) { row_fwd_l<decltype(L)::value>(pl, d, batch, st); });
}
void row_pmul_inv(const NttPlan& pl, uint64_t* d, const uint64_t* img, int batch,
                  const ulonglong2* WiRf, cudaStream_t st) {
    by_len(pl.l2,
           [&](auto L) { row_pmul_inv_l<decltype(L)::value>(pl, d, img, batch, WiRf, st); });
}
void row_mac(const NttPlan& pl, const uint64_t* g, const uint64_t* img, int Q, int batch,
             const ulonglong2* Wif, uint64_t* out, cudaStream_t st) {
    by_len(pl.l2,
           [&](auto L) { row_mac_l<decltype(L)::value>(pl, g, img, Q, batch, Wif, out, st); });
}

const ulonglong2* wi_times_r(NttPlan& pl, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(pl.mu);
    if (!pl.WiRf) {
        PCGB_CK(cudaMalloc(&pl.WiRf, sizeof(ulonglong2) * pl.N));
        scale_r_kernel<<<static_cast<unsigned>((pl.N + 255) / 256), 256, 0, st>>>(
            pl.WiRf, pl.Wif, pl.N, r2_mod_p());
        PCGB_POST_LAUNCH();
        PCGB_CK(cudaStreamSynchronize(st));
    }
    return pl.WiRf;
}

}  // namespace

const NttPlan& ntt_plan(int logN) {
    if (logN < 1 || logN > kMaxLogN) fail(PCGB_EINVAL, "NTT length must be 2^1 .. 2^24");
    static std::mutex mu;
    static std::map<std::pair<int, int>, std::unique_ptr<NttPlan>> cache;
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto& slot = cache[{dev, logN}];
    if (!slot) slot.reset(build_plan(logN));
    return *slot;
}

void ntt_forward_from(const NttPlan& pl, const uint64_t* src, uint64_t* dst, int batch,
                      bool reduce, cudaStream_t st) {
    col_fwd(pl, src, dst, batch, reduce, st);
    row_fwd(pl, dst, batch, st);
}

void ntt_log_sizes(const NttPlan& pl, int* l1, int* l2) {
    *l1 = pl.l1;
    *l2 = pl.l2;
}

void ntt_forward(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    col_fwd(pl, d, d, batch, false, st);
    row_fwd(pl, d, batch, st);
}

// Per device: a second stream and two events for the two-half schedule of
// poly_mul_device; the mutex keeps one call's fork, launches and join
// together when several host threads multiply on the same device.
struct HalfFork {
    std::mutex mu;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
HalfFork& half_fork() {
    static HalfFork f[64];
    int dev = 0;
    PCGB_CK(cudaGetDevice(&dev));
    return f[dev];
}

void poly_mul_device(const NttPlan& pl, uint64_t* c, const uint64_t* a, const uint64_t* b,
                     int batch, uint64_t* scratch, cudaStream_t st) {
    const ulonglong2* wir = wi_times_r(const_cast<NttPlan&>(pl), st);
    // A = NTT(a) in scratch; c = NTT(b); c = INTT(c (.) A): the forward row
    // pass of c and the pointwise product + inverse row pass are separate
    // launches (each needs about 70 registers a thread where the fused
    // pass needs 96, so more CTAs fit on an SM).
    // a is read before c is first written, so c may alias a or b.
    // A batch of two or more runs as two halves on two streams, pass by
    // pass: each pass kernel alone leaves the IMAD pipe a third idle (its
    // barriers and its tail), and the other half's CTAs fill those slots
    // (16 x 2^20: 0.882 -> 0.843 ms; four quarters gave 0.839).  Each half
    // reads and writes only its own products, so aliasing holds per half.
    if (batch >= 2) {
        HalfFork& f = half_fork();
        std::lock_guard<std::mutex> lk(f.mu);
        if (!f.side) {
            PCGB_CK(cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming));
            PCGB_CK(cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming));
            PCGB_CK(cudaStreamCreateWithFlags(&f.side, cudaStreamNonBlocking));
        }
        const int h0 = batch / 2, h1 = batch - h0;
        const size_t o = static_cast<size_t>(h0) * pl.N;
        PCGB_CK(cudaEventRecord(f.fork, st));
        PCGB_CK(cudaStreamWaitEvent(f.side, f.fork, 0));
        col_fwd(pl, a, scratch, h0, true, st);
        col_fwd(pl, a + o, scratch + o, h1, true, f.side);
        row_fwd(pl, scratch, h0, st);
        row_fwd(pl, scratch + o, h1, f.side);
        col_fwd(pl, b, c, h0, true, st);
        col_fwd(pl, b + o, c + o, h1, true, f.side);
        row_fwd(pl, c, h0, st);
        row_fwd(pl, c + o, h1, f.side);
        row_pmul_inv(pl, c, scratch, h0, wir, st);
        row_pmul_inv(pl, c + o, scratch + o, h1, wir, f.side);
        col_inv(pl, c, h0, st);
        col_inv(pl, c + o, h1, f.side);
        PCGB_CK(cudaEventRecord(f.join, f.side));
        PCGB_CK(cudaStreamWaitEvent(st, f.join, 0));
        return;
    }
    col_fwd(pl, a, scratch, batch, true, st);
    row_fwd(pl, scratch, batch, st);
    col_fwd(pl, b, c, batch, true, st);
    row_fwd(pl, c, batch, st);
    row_pmul_inv(pl, c, scratch, batch, wir, st);
    col_inv(pl, c, batch, st);
}

bool poly_mul_mixed_ok(int logN) { return logN >= 2 * kMixedLmin && logN <= 2 * kMixedLmax; }

void poly_mul_device_mixed(int count, uint64_t* const* c, const uint64_t* const* a,
                           const uint64_t* const* b, const int* logN, cudaStream_t st) {
    if (count <= 0) return;
    std::vector<int> order(count);
    size_t scratch_words = 0;
    for (int i = 0; i < count; ++i) {
        if (!poly_mul_mixed_ok(logN[i])) fail(PCGB_EINVAL, "mixed poly-mul: N must be 2^16 .. 2^20");
        order[i] = i;
        scratch_words += size_t{1} << logN[i];
    }
    // Longest products first, so the last CTAs of each pass are short ones.
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return logN[x] > logN[y]; });
    std::vector<MixedPoly> polys(count);
    std::vector<MixedCta> col, row;
    uint64_t* scratch = static_cast<uint64_t*>(pool_alloc(8 * scratch_words, st));
    size_t off = 0;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        NttPlan& pl = const_cast<NttPlan&>(ntt_plan(logN[i]));
        MixedPoly& m = polys[k];
        m.a = a[i]; m.b = b[i]; m.c = c[i]; m.A = scratch + off;
        m.tw1 = pl.tw1; m.tw1i = pl.tw1i; m.tw2 = pl.tw2; m.tw2i = pl.tw2i;
        m.Wf = pl.Wf; m.WiRf = wi_times_r(pl, st);
        m.l1 = pl.l1; m.l2 = pl.l2;
        off += pl.N;
        int C = 0, V = 0;
        by_len(pl.l1, [&](auto L) {
            if constexpr (decltype(L)::value >= kMixedLmin && decltype(L)::value <= kMixedLmax)
                C = mixed_C<decltype(L)::value>();
        });
        by_len(pl.l2, [&](auto L) {
            if constexpr (decltype(L)::value >= kMixedLmin && decltype(L)::value <= kMixedLmax)
                V = mixed_V<decltype(L)::value>();
        });
        for (uint32_t tl = 0; tl < static_cast<uint32_t>(pl.n2 / C); ++tl) col.push_back({uint32_t(k), tl});
        for (uint32_t tl = 0; tl < static_cast<uint32_t>(pl.n1 / V); ++tl) row.push_back({uint32_t(k), tl});
    }
    const size_t b_polys = sizeof(MixedPoly) * polys.size();
    const size_t b_col = sizeof(MixedCta) * col.size(), b_row = sizeof(MixedCta) * row.size();
    const size_t o_col = (b_polys + 255) & ~size_t{255};
    const size_t o_row = (o_col + b_col + 255) & ~size_t{255};
    char* tab = static_cast<char*>(pool_alloc(o_row + b_row, st));
    PCGB_CK(cudaMemcpyAsync(tab, polys.data(), b_polys, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(tab + o_col, col.data(), b_col, cudaMemcpyHostToDevice, st));
    PCGB_CK(cudaMemcpyAsync(tab + o_row, row.data(), b_row, cudaMemcpyHostToDevice, st));
    const MixedPoly* d_polys = reinterpret_cast<const MixedPoly*>(tab);
    const MixedCta* d_col = reinterpret_cast<const MixedCta*>(tab + o_col);
    const MixedCta* d_row = reinterpret_cast<const MixedCta*>(tab + o_row);
    const unsigned n_col = static_cast<unsigned>(col.size()), n_row = static_cast<unsigned>(row.size());
    g_optin(mixed_col_fwd_kernel, kMixedColSmem);
    g_optin(mixed_col_inv_kernel, kMixedColSmem);
    g_optin(mixed_row_fwd_kernel, kMixedRowSmem);
    g_optin(mixed_row_mac_kernel, kMixedRowSmem);
    mixed_col_fwd_kernel<<<n_col, kMixedColThreads, kMixedColSmem, st>>>(d_polys, d_col, 0);
    PCGB_POST_LAUNCH();
    mixed_row_fwd_kernel<<<n_row, kMixedRowThreads, kMixedRowSmem, st>>>(d_polys, d_row);
    PCGB_POST_LAUNCH();
    mixed_col_fwd_kernel<<<n_col, kMixedColThreads, kMixedColSmem, st>>>(d_polys, d_col, 1);
    PCGB_POST_LAUNCH();
    mixed_row_mac_kernel<<<n_row, kMixedRowThreads, kMixedRowSmem, st>>>(d_polys, d_row);
    PCGB_POST_LAUNCH();
    mixed_col_inv_kernel<<<n_col, kMixedColThreads, kMixedColSmem, st>>>(d_polys, d_col);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(tab, st));
    PCGB_CK(cudaFreeAsync(scratch, st));
}

void ntt_mac_inverse(const NttPlan& pl, uint64_t* g, const uint64_t* img, int Q, uint64_t* acc,
                     cudaStream_t st) {
    col_fwd(pl, g, g, Q, false, st);
    row_mac(pl, g, img, Q, 1, pl.Wif, acc, st);
    col_inv(pl, acc, 1, st);
}

bool ntt_mac_multi_ok(int logN) { return logN >= 2 * kMacLmin && logN <= 2 * kMixedLmax; }

void ntt_mac_inverse_multi(int count, uint64_t* const* g, const uint64_t* const* img, const int* Q,
                           uint64_t* const* z, const int* logN, cudaStream_t st) {
    if (count <= 0) return;
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) {
        if (!ntt_mac_multi_ok(logN[i])) fail(PCGB_EINVAL, "multi MAC: N must be 2^14 .. 2^20");
        if (Q[i] < 1 || !g[i] || !img[i] || !z[i]) fail(PCGB_EINVAL, "multi MAC: bad request");
        order[i] = i;
    }
    // Most work first, so the last CTAs of each pass are short ones.
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (static_cast<uint64_t>(Q[x]) << logN[x]) > (static_cast<uint64_t>(Q[y]) << logN[y]);
    });
    std::vector<MacReq> reqs(count);
    std::vector<MacCta> colf, row, coli;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        const NttPlan& pl = ntt_plan(logN[i]);
        MacReq& m = reqs[k];
        m.g = g[i]; m.img = img[i]; m.z = z[i];
        m.tw1 = pl.tw1; m.tw1i = pl.tw1i; m.tw2 = pl.tw2; m.tw2i = pl.tw2i;
        m.Wf = pl.Wf; m.Wif = pl.Wif;
        m.Q = Q[i]; m.l1 = pl.l1; m.l2 = pl.l2;
        int C = 0, V = 0;
        by_len(pl.l1, [&](auto L) {
            if constexpr (decltype(L)::value >= kMacLmin && decltype(L)::value <= kMixedLmax)
                C = mixed_C<decltype(L)::value>();
        });
        by_len(pl.l2, [&](auto L) {
            if constexpr (decltype(L)::value >= kMacLmin && decltype(L)::value <= kMixedLmax)
                V = mixed_V<decltype(L)::value>();
        });
        const uint32_t kk = static_cast<uint32_t>(k);
        for (uint32_t q = 0; q < static_cast<uint32_t>(m.Q); ++q)
            for (uint32_t tl = 0; tl < static_cast<uint32_t>(pl.n2 / C); ++tl) colf.push_back({kk, q, tl});
        for (uint32_t tl = 0; tl < static_cast<uint32_t>(pl.n1 / V); ++tl) row.push_back({kk, 0, tl});
        for (uint32_t tl = 0; tl < static_cast<uint32_t>(pl.n2 / C); ++tl) coli.push_back({kk, 0, tl});
    }
    const size_t b_req = sizeof(MacReq) * reqs.size();
    const size_t o_colf = (b_req + 255) & ~size_t{255};
    const size_t o_row = (o_colf + sizeof(MacCta) * colf.size() + 255) & ~size_t{255};
    const size_t o_coli = (o_row + sizeof(MacCta) * row.size() + 255) & ~size_t{255};
    const size_t total = o_coli + sizeof(MacCta) * coli.size();
    std::vector<char> host(total);
    std::memcpy(host.data(), reqs.data(), b_req);
    std::memcpy(host.data() + o_colf, colf.data(), sizeof(MacCta) * colf.size());
    std::memcpy(host.data() + o_row, row.data(), sizeof(MacCta) * row.size());
    std::memcpy(host.data() + o_coli, coli.data(), sizeof(MacCta) * coli.size());
    char* tab = static_cast<char*>(pool_alloc(total, st));
    PCGB_CK(cudaMemcpyAsync(tab, host.data(), total, cudaMemcpyHostToDevice, st));
    const MacReq* d_req = reinterpret_cast<const MacReq*>(tab);
    g_optin(mac_col_fwd_kernel, kMixedColSmem);
    g_optin(mac_row_kernel, kMixedRowSmem);
    g_optin(mac_col_inv_kernel, kMixedColSmem);
    mac_col_fwd_kernel<<<static_cast<unsigned>(colf.size()), kMixedColThreads, kMixedColSmem, st>>>(
        d_req, reinterpret_cast<const MacCta*>(tab + o_colf));
    PCGB_POST_LAUNCH();
    mac_row_kernel<<<static_cast<unsigned>(row.size()), kMixedRowThreads, kMixedRowSmem, st>>>(
        d_req, reinterpret_cast<const MacCta*>(tab + o_row));
    PCGB_POST_LAUNCH();
    mac_col_inv_kernel<<<static_cast<unsigned>(coli.size()), kMixedColThreads, kMixedColSmem, st>>>(
        d_req, reinterpret_cast<const MacCta*>(tab + o_coli));
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(tab, st));
}

void pointwise_mul(uint64_t* c, const uint64_t* a, const uint64_t* b, size_t count, int mode,
                   cudaStream_t st) {
    pointwise_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(c, a, b, count,
                                                                               mode, r2_mod_p());
    PCGB_POST_LAUNCH();
}

void reduce_mod_p(uint64_t* d, const uint64_t* s, size_t count, cudaStream_t st) {
    reduce_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(d, s, count);
    PCGB_POST_LAUNCH();
}

}  // namespace pcgb
