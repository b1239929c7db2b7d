// Negacyclic NTT over F_p, four-step form, for N = 2^logN (1 <= logN <= 24).
//
// N = n1 * n2 with n1 = 2^ceil(logN/2), n2 = 2^floor(logN/2); coefficient j
// sits at row j / n2, column j % n2.  With psi a primitive 2N-th root:
//   column pass: negacyclic NTT of length n1 on every column (root
//                psi1 = psi^n2), then multiply element (k, j2) by the
//                twiddle psi^(j2 * (2*i1 + 1 - n1)), i1 = brev(k);
//   row pass:    negacyclic NTT of length n2 on every row (root psi2 =
//                psi^n1).
// Element (k, k2) then holds A(psi^(2*(i1 + n1*i2) + 1)) with i1 = brev(k),
// i2 = brev(k2): the evaluations of a(x) mod x^N + 1, in a fixed permuted
// order that every operand of a pointwise product shares.  The inverse runs
// the passes backwards with inverse roots and folds N^-1 into its twiddle.
//
// Each sub-transform is the merged-twist Cooley-Tukey (forward) /
// Gentleman-Sande (inverse) negacyclic NTT of Longa and Naehrig (CANS 2016,
// Algorithms 1-2), done in shared memory with Shoup multiplications by
// precomputed roots.  The passes are two HBM sweeps per transform; the
// pointwise product with a resident operand is fused into the row pass, as is
// the multiply-accumulate over several transforms.  Replaces the reference's
// radix-2 per-stage v1 kernels (GPU_baseline/common/poly_mul_cuda.cu:137-200)
// and its 20-kernel four-step (poly_mul_gpuntt_square.cu:171-613).
#include "pcgb_internal.h"

#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "field.cuh"

namespace pcgb {

struct NttPlan {
    int logN = 0, l1 = 0, l2 = 0;
    size_t N = 0;
    int n1 = 0, n2 = 0;
    ulonglong2* psi1 = nullptr;   // (value, shoup) in bit-reversed order, n1
    ulonglong2* psi1i = nullptr;
    ulonglong2* psi2 = nullptr;   // n2
    ulonglong2* psi2i = nullptr;
    uint64_t* W = nullptr;        // [n1][n2] forward twiddle, Montgomery form
    uint64_t* Wi = nullptr;       // inverse twiddle * N^-1, Montgomery form
    int C = 1;                    // columns per CTA in the column passes
    int R = 1;                    // rows per CTA in the row passes
};

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ ulonglong2 ld2(const ulonglong2* p) { return __ldg(p); }

// Forward negacyclic NTT of `cnt` transforms of length n = 2^logn stored in
// shared memory at x + c*ld (c < cnt).  All threads of the CTA take part.
__device__ void smem_fwd(uint64_t* x, int cnt, int ld, int logn, const ulonglong2* __restrict__ psi) {
    const int half = 1 << (logn - 1);
    const int total = cnt * half;
    for (int s = 0; s < logn; ++s) {
        const int m = 1 << s;            // groups
        const int lt = logn - 1 - s;     // log2 of butterfly span t
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            const int c = b >> (logn - 1);
            const int bb = b & (half - 1);
            const int i = bb >> lt;
            const int j = bb & ((1 << lt) - 1);
            uint64_t* y = x + c * ld + (i << (lt + 1)) + j;
            const ulonglong2 S = ld2(psi + m + i);
            const uint64_t U = y[0];
            const uint64_t V = shoup_mul(y[1 << lt], S.x, S.y);
            y[0] = add_p(U, V);
            y[1 << lt] = sub_p(U, V);
        }
        __syncthreads();
    }
}

// Inverse (Gentleman-Sande), no 1/n scaling.
__device__ void smem_inv(uint64_t* x, int cnt, int ld, int logn, const ulonglong2* __restrict__ psii) {
    const int half = 1 << (logn - 1);
    const int total = cnt * half;
    for (int s = logn - 1; s >= 0; --s) {
        const int h = 1 << s;             // groups
        const int lt = logn - 1 - s;      // log2 t
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            const int c = b >> (logn - 1);
            const int bb = b & (half - 1);
            const int i = bb >> lt;
            const int j = bb & ((1 << lt) - 1);
            uint64_t* y = x + c * ld + (i << (lt + 1)) + j;
            const ulonglong2 S = ld2(psii + h + i);
            const uint64_t U = y[0], V = y[1 << lt];
            y[0] = add_p(U, V);
            y[1 << lt] = shoup_mul(sub_p(U, V), S.x, S.y);
        }
        __syncthreads();
    }
}

// Column pass, forward.  grid = (n2 / C, batch).  src may differ from dst;
// reduce_in maps arbitrary 64-bit inputs into [0, p) first.
__global__ void __launch_bounds__(kThreads) col_fwd_kernel(const uint64_t* __restrict__ src,
                                                           uint64_t* __restrict__ dst, int l1,
                                                           int l2, int C,
                                                           const ulonglong2* __restrict__ psi1,
                                                           const uint64_t* __restrict__ W,
                                                           int reduce_in) {
    extern __shared__ uint64_t sm[];
    const int n1 = 1 << l1, n2 = 1 << l2, ld = n1 + 1;
    const size_t N = static_cast<size_t>(n1) * n2;
    const uint64_t* s = src + blockIdx.y * N;
    uint64_t* d = dst + blockIdx.y * N;
    const int j0 = blockIdx.x * C;
    for (int e = threadIdx.x; e < n1 * C; e += blockDim.x) {
        const int k = e / C, c = e - k * C;
        uint64_t v = s[static_cast<size_t>(k) * n2 + j0 + c];
        sm[c * ld + k] = reduce_in ? reduce_p(v) : v;
    }
    __syncthreads();
    if (l1 > 0) smem_fwd(sm, C, ld, l1, psi1);
    for (int e = threadIdx.x; e < n1 * C; e += blockDim.x) {
        const int k = e / C, c = e - k * C;
        const size_t g = static_cast<size_t>(k) * n2 + j0 + c;
        d[g] = mont_mul(sm[c * ld + k], __ldg(W + g));
    }
}

// Column pass, inverse (output in natural coefficient order).
__global__ void __launch_bounds__(kThreads) col_inv_kernel(uint64_t* __restrict__ d_all, int l1,
                                                           int l2, int C,
                                                           const ulonglong2* __restrict__ psi1i) {
    extern __shared__ uint64_t sm[];
    const int n1 = 1 << l1, n2 = 1 << l2, ld = n1 + 1;
    const size_t N = static_cast<size_t>(n1) * n2;
    uint64_t* d = d_all + blockIdx.y * N;
    const int j0 = blockIdx.x * C;
    for (int e = threadIdx.x; e < n1 * C; e += blockDim.x) {
        const int k = e / C, c = e - k * C;
        sm[c * ld + k] = d[static_cast<size_t>(k) * n2 + j0 + c];
    }
    __syncthreads();
    if (l1 > 0) smem_inv(sm, C, ld, l1, psi1i);
    for (int e = threadIdx.x; e < n1 * C; e += blockDim.x) {
        const int k = e / C, c = e - k * C;
        d[static_cast<size_t>(k) * n2 + j0 + c] = sm[c * ld + k];
    }
}

// Row pass, forward.  grid = (n1 / R, batch).
__global__ void __launch_bounds__(kThreads) row_fwd_kernel(uint64_t* __restrict__ d_all, int l1,
                                                           int l2, int R,
                                                           const ulonglong2* __restrict__ psi2) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2;
    const size_t N = static_cast<size_t>(1) << (l1 + l2);
    uint64_t* d = d_all + blockIdx.y * N + static_cast<size_t>(blockIdx.x) * R * n2;
    for (int e = threadIdx.x; e < R * n2; e += blockDim.x) sm[e] = d[e];
    __syncthreads();
    if (l2 > 0) smem_fwd(sm, R, n2, l2, psi2);
    for (int e = threadIdx.x; e < R * n2; e += blockDim.x) d[e] = sm[e];
}

// Row pass, inverse, with the inverse twiddle (and N^-1) applied.
// If other != nullptr the rows are first forward-transformed and multiplied
// pointwise by `other` (a fully transformed operand): c = INTT(NTT(b) * a).
__global__ void __launch_bounds__(kThreads) row_inv_kernel(const uint64_t* __restrict__ src_all,
                                                           uint64_t* __restrict__ dst_all,
                                                           const uint64_t* __restrict__ other_all,
                                                           int l1, int l2, int R,
                                                           const ulonglong2* __restrict__ psi2,
                                                           const ulonglong2* __restrict__ psi2i,
                                                           const uint64_t* __restrict__ Wi,
                                                           uint64_t r2) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2;
    const size_t N = static_cast<size_t>(1) << (l1 + l2);
    const size_t base = blockIdx.y * N + static_cast<size_t>(blockIdx.x) * R * n2;
    const uint64_t* s = src_all + base;
    for (int e = threadIdx.x; e < R * n2; e += blockDim.x) sm[e] = s[e];
    __syncthreads();
    if (other_all) {
        if (l2 > 0) smem_fwd(sm, R, n2, l2, psi2);
        const uint64_t* o = other_all + base;
        for (int e = threadIdx.x; e < R * n2; e += blockDim.x)
            sm[e] = mont_mul(mont_mul(sm[e], __ldg(o + e)), r2);
        __syncthreads();
    }
    if (l2 > 0) smem_inv(sm, R, n2, l2, psi2i);
    uint64_t* d = dst_all + base;
    const uint64_t* w = Wi + static_cast<size_t>(blockIdx.x) * R * n2;
    for (int e = threadIdx.x; e < R * n2; e += blockDim.x) d[e] = mont_mul(sm[e], __ldg(w + e));
}

// Multiply-accumulate row pass: out row = INTT( sum_q NTTrow(g_q) * img_q ),
// img in Montgomery-scaled form (value * 2^64 mod p).  grid = (n1 / R).
__global__ void __launch_bounds__(kThreads) row_mac_inv_kernel(
    const uint64_t* __restrict__ g, const uint64_t* __restrict__ img, int Q, int l1, int l2,
    int R, const ulonglong2* __restrict__ psi2, const ulonglong2* __restrict__ psi2i,
    const uint64_t* __restrict__ Wi, uint64_t* __restrict__ out) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2;
    const int len = R * n2;
    uint64_t* acc = sm + len;
    const size_t N = static_cast<size_t>(1) << (l1 + l2);
    const size_t base = static_cast<size_t>(blockIdx.x) * len;
    for (int e = threadIdx.x; e < len; e += blockDim.x) acc[e] = 0;
    for (int q = 0; q < Q; ++q) {
        const uint64_t* s = g + q * N + base;
        for (int e = threadIdx.x; e < len; e += blockDim.x) sm[e] = s[e];
        __syncthreads();
        if (l2 > 0) smem_fwd(sm, R, n2, l2, psi2);
        const uint64_t* im = img + q * N + base;
        for (int e = threadIdx.x; e < len; e += blockDim.x)
            acc[e] = add_p(acc[e], mont_mul(sm[e], __ldg(im + e)));
        __syncthreads();
    }
    if (l2 > 0) smem_inv(acc, R, n2, l2, psi2i);
    const uint64_t* w = Wi + base;
    for (int e = threadIdx.x; e < len; e += blockDim.x)
        out[base + e] = mont_mul(acc[e], __ldg(w + e));
}

// Twiddle tables: W[k*n2 + j2] = psi^(j2*(2*brev(k)+1-n1)) (times R), and
// Wi = psi^-(...) * N^-1 (times R).  powR[b] = psi^(2^b) * R mod p.
__global__ void twiddle_kernel(uint64_t* W, uint64_t* Wi, int l1, int l2,
                               const uint64_t* __restrict__ powR, uint64_t oneR, uint64_t ninvR) {
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
    W[idx] = a;                    // psi^e * R
    Wi[idx] = mont_mul(b, ninvR);  // psi^-e * N^-1 * R
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

uint32_t brev_host(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

uint64_t primitive_root_host() {
    // p - 1 = 2^25 * (2^37 - 3); smallest g with g^((p-1)/q) != 1 for q in {2, 2^37-3}.
    const uint64_t q2 = (kPm - 1) >> 25;
    for (uint64_t g = 2;; ++g)
        if (pow_p_host(g, (kPm - 1) / 2) != 1 && pow_p_host(g, (kPm - 1) / q2) != 1) return g;
}

// Roots psi_n^brev(k) (Shoup pairs) for a length-n negacyclic transform.
ulonglong2* upload_psi_table(uint64_t psi_n, int logn) {
    const int n = 1 << logn;
    std::vector<uint64_t> pw(n);
    uint64_t a = 1;
    for (int k = 0; k < n; ++k) { pw[k] = a; a = mul_p_host(a, psi_n); }
    std::vector<ulonglong2> t(n);
    for (int k = 0; k < n; ++k) {
        const uint64_t v = pw[brev_host(static_cast<uint32_t>(k), logn)];
        t[k] = make_ulonglong2(v, shoup_q_host(v));
    }
    ulonglong2* d = nullptr;
    PCGB_CK(cudaMalloc(&d, sizeof(ulonglong2) * n));
    upload_blocking(d, t.data(), sizeof(ulonglong2) * n);
    return d;
}

NttPlan* build_plan(int logN) {
    auto* pl = new NttPlan();
    pl->logN = logN;
    pl->N = static_cast<size_t>(1) << logN;
    pl->l1 = (logN + 1) / 2;
    pl->l2 = logN / 2;
    pl->n1 = 1 << pl->l1;
    pl->n2 = 1 << pl->l2;
    const uint64_t g = primitive_root_host();
    const uint64_t psi = pow_p_host(g, (kPm - 1) / (2 * pl->N));
    const uint64_t psi_inv = pow_p_host(psi, kPm - 2);
    pl->psi1 = upload_psi_table(pow_p_host(psi, pl->n2), pl->l1);
    pl->psi1i = upload_psi_table(pow_p_host(psi_inv, pl->n2), pl->l1);
    pl->psi2 = upload_psi_table(pow_p_host(psi, pl->n1), pl->l2);
    pl->psi2i = upload_psi_table(pow_p_host(psi_inv, pl->n1), pl->l2);
    // Columns per CTA: 8 (64-byte row segments) unless the column is long.
    pl->C = std::min(pl->n2, std::max(1, std::min(8, 16384 / pl->n1)));
    pl->R = std::min(pl->n1, std::max(1, 4096 / pl->n2));
    PCGB_CK(cudaMalloc(&pl->W, sizeof(uint64_t) * pl->N));
    PCGB_CK(cudaMalloc(&pl->Wi, sizeof(uint64_t) * pl->N));
    const uint64_t R = r_mod_p();
    std::vector<uint64_t> powR(logN + 2);
    uint64_t pb = psi;
    for (int b = 0; b < logN + 2; ++b) { powR[b] = mul_p_host(pb, R); pb = mul_p_host(pb, pb); }
    uint64_t* d_pow = nullptr;
    PCGB_CK(cudaMalloc(&d_pow, sizeof(uint64_t) * powR.size()));
    upload_blocking(d_pow, powR.data(), sizeof(uint64_t) * powR.size());
    const uint64_t ninvR = mul_p_host(pow_p_host(pl->N % kPm, kPm - 2), R);
    twiddle_kernel<<<static_cast<unsigned>((pl->N + 255) / 256), 256>>>(pl->W, pl->Wi, pl->l1,
                                                                        pl->l2, d_pow, R, ninvR);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaDeviceSynchronize());
    cudaFree(d_pow);
    return pl;
}

size_t col_smem(const NttPlan& pl) { return sizeof(uint64_t) * static_cast<size_t>(pl.n1 + 1) * pl.C; }
size_t row_smem(const NttPlan& pl) { return sizeof(uint64_t) * static_cast<size_t>(pl.R) * pl.n2; }

void set_smem(const void* f, size_t bytes) {
    if (bytes > 48 * 1024)
        PCGB_CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(bytes)));
}

void col_fwd(const NttPlan& pl, const uint64_t* src, uint64_t* dst, int batch, bool reduce_in,
             cudaStream_t st) {
    const size_t sm = col_smem(pl);
    set_smem(reinterpret_cast<const void*>(col_fwd_kernel), sm);
    col_fwd_kernel<<<dim3(pl.n2 / pl.C, batch), kThreads, sm, st>>>(src, dst, pl.l1, pl.l2, pl.C,
                                                                    pl.psi1, pl.W, reduce_in);
    PCGB_POST_LAUNCH();
}

void col_inv(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    const size_t sm = col_smem(pl);
    set_smem(reinterpret_cast<const void*>(col_inv_kernel), sm);
    col_inv_kernel<<<dim3(pl.n2 / pl.C, batch), kThreads, sm, st>>>(d, pl.l1, pl.l2, pl.C,
                                                                    pl.psi1i);
    PCGB_POST_LAUNCH();
}

void row_fwd(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    const size_t sm = row_smem(pl);
    set_smem(reinterpret_cast<const void*>(row_fwd_kernel), sm);
    row_fwd_kernel<<<dim3(pl.n1 / pl.R, batch), kThreads, sm, st>>>(d, pl.l1, pl.l2, pl.R,
                                                                    pl.psi2);
    PCGB_POST_LAUNCH();
}

void row_inv(const NttPlan& pl, const uint64_t* src, uint64_t* dst, const uint64_t* other,
             int batch, cudaStream_t st) {
    const size_t sm = row_smem(pl);
    set_smem(reinterpret_cast<const void*>(row_inv_kernel), sm);
    row_inv_kernel<<<dim3(pl.n1 / pl.R, batch), kThreads, sm, st>>>(
        src, dst, other, pl.l1, pl.l2, pl.R, pl.psi2, pl.psi2i, pl.Wi, r2_mod_p());
    PCGB_POST_LAUNCH();
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

void ntt_forward(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    col_fwd(pl, d, d, batch, false, st);
    row_fwd(pl, d, batch, st);
}

void ntt_inverse(const NttPlan& pl, uint64_t* d, int batch, cudaStream_t st) {
    row_inv(pl, d, d, nullptr, batch, st);
    col_inv(pl, d, batch, st);
}

void poly_mul_device(const NttPlan& pl, uint64_t* c, const uint64_t* a, const uint64_t* b,
                     int batch, uint64_t* scratch, cudaStream_t st) {
    const size_t n = pl.N * static_cast<size_t>(batch);
    uint64_t* A = scratch;
    uint64_t* B = scratch + n;
    col_fwd(pl, a, A, batch, true, st);
    row_fwd(pl, A, batch, st);
    col_fwd(pl, b, B, batch, true, st);
    row_inv(pl, B, c, A, batch, st);  // c rows = INTT(NTT(B) * A) with the inverse twiddle
    col_inv(pl, c, batch, st);
}

void ntt_mac_inverse(const NttPlan& pl, uint64_t* g, const uint64_t* img, int Q, uint64_t* acc,
                     cudaStream_t st) {
    col_fwd(pl, g, g, Q, false, st);
    const size_t sm = 2 * row_smem(pl);
    set_smem(reinterpret_cast<const void*>(row_mac_inv_kernel), sm);
    row_mac_inv_kernel<<<pl.n1 / pl.R, kThreads, sm, st>>>(g, img, Q, pl.l1, pl.l2, pl.R, pl.psi2,
                                                           pl.psi2i, pl.Wi, acc);
    PCGB_POST_LAUNCH();
    col_inv(pl, acc, 1, st);
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
