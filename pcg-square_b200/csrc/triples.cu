// Consumers of the expansion on the device: Beaver-triple extraction from
// two ring OLEs, and the OLE / triple relations checked slot by slot.
//
// Triples (CPU_baseline/pcg_ole_2pc/triple.h:45-110): party 0 takes
// a = x1, b = x2, party 1 a = x2, b = x1, and c = a*b + z1 + z2 in R_p; the
// N slot triples are the forward NTTs of a, b, c.  The reference forms the
// ring product c (three transforms) and then transforms a, b and c again;
// by linearity the slots of c are NTT(a)(.)NTT(b) + NTT(z1 + z2), so here
// three forward transforms and one pointwise pass give all of a, b and c.
// Slots are written in the reference's order (slot k = A(psi^(2k+1)),
// CPU_baseline/ntt.h:140-144), so shares match its triple.h output exactly.
//
// Relations: the OLE relation z0 + z1 = x0*x1 (CPU_baseline/test/
// pcg_ole_2pc.cpp:199-214) holds iff it holds in every NTT slot, and a
// triple holds iff (a0+a1)(b0+b1) = c0+c1 in every slot; both checks count
// the slots that fail, on the device.
#include "pcgb_internal.h"

#include <algorithm>
#include <string>

#include "field.cuh"
#include "ntt_layout.cuh"

namespace pcgb {
namespace {

constexpr int kTpb = 256;

unsigned grid_for(size_t n) { return static_cast<unsigned>((n + kTpb - 1) / kTpb); }

// d = (u + v) mod p for any 64-bit inputs.
__global__ void add_reduce_kernel(uint64_t* d, const uint64_t* u, const uint64_t* v, size_t n) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) d[i] = add_p(reduce_p(u[i]), reduce_p(v[i]));
}

// Slot k of the outputs: a = A, b = B, c = A*B + S at the transform
// position of slot k (A, B, S transformed, values in [0, p)).
__global__ void triple_slots_kernel(const uint64_t* __restrict__ A, const uint64_t* __restrict__ B,
                                    const uint64_t* __restrict__ S, size_t n, int l1, int l2,
                                    uint64_t r2, uint64_t* a, uint64_t* b, uint64_t* c) {
    const size_t k = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t s = ntt_slot_position(k, l1, l2);
    const uint64_t x = __ldg(A + s), y = __ldg(B + s);
    a[k] = x;
    b[k] = y;
    c[k] = add_p(mont_mul(mont_mul(x, y), r2), __ldg(S + s));
}

// Counts slots where X0*X1 != Z (all transformed, in [0, p)).
__global__ void ole_check_kernel(const uint64_t* __restrict__ X0, const uint64_t* __restrict__ X1,
                                 const uint64_t* __restrict__ Z, size_t n, uint64_t r2,
                                 unsigned long long* bad) {
    unsigned long long mine = 0;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        mine += mont_mul(mont_mul(X0[i], X1[i]), r2) != Z[i];
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(bad, mine);
}

// Counts slots where (a0+a1)(b0+b1) != c0+c1 (slot values any 64-bit).
__global__ void triple_check_kernel(const uint64_t* __restrict__ a0, const uint64_t* __restrict__ b0,
                                    const uint64_t* __restrict__ c0, const uint64_t* __restrict__ a1,
                                    const uint64_t* __restrict__ b1, const uint64_t* __restrict__ c1,
                                    size_t n, uint64_t r2, unsigned long long* bad) {
    unsigned long long mine = 0;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint64_t a = add_p(reduce_p(a0[i]), reduce_p(a1[i]));
        const uint64_t b = add_p(reduce_p(b0[i]), reduce_p(b1[i]));
        const uint64_t c = add_p(reduce_p(c0[i]), reduce_p(c1[i]));
        mine += mont_mul(mont_mul(a, b), r2) != c;
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(bad, mine);
}

unsigned check_grid(size_t n) {
    return static_cast<unsigned>(std::min<size_t>(grid_for(n), static_cast<size_t>(sm_count()) * 8));
}

int log2_checked(int N, const char* what) {
    if (N < 2 || (N & (N - 1)) || N > (1 << kMaxLogN))
        fail(PCGB_EINVAL, std::string(what) + ": N must be a power of two in [2, 2^24]");
    int l = 0;
    while ((1 << l) < N) ++l;
    return l;
}

}  // namespace

void add_mod_p_device(uint64_t* d, const uint64_t* u, const uint64_t* v, size_t count,
                      cudaStream_t st) {
    add_reduce_kernel<<<grid_for(count), kTpb, 0, st>>>(d, u, v, count);
    PCGB_POST_LAUNCH();
}

void triples_device(int N, int party, const uint64_t* x1, const uint64_t* z1, const uint64_t* x2,
                    const uint64_t* z2, uint64_t* a, uint64_t* b, uint64_t* c, cudaStream_t st) {
    if (party != 0 && party != 1) fail(PCGB_EINVAL, "triples: party must be 0 or 1");
    if (!x1 || !z1 || !x2 || !z2 || !a || !b || !c) fail(PCGB_EINVAL, "triples: null pointer");
    const NttPlan& pl = ntt_plan(log2_checked(N, "triples"));
    int l1 = 0, l2 = 0;
    ntt_log_sizes(pl, &l1, &l2);
    const size_t n = static_cast<size_t>(N);
    uint64_t* T = static_cast<uint64_t*>(pool_alloc(3 * n * sizeof(uint64_t), st));  // A | B | S
    add_reduce_kernel<<<grid_for(n), kTpb, 0, st>>>(T + 2 * n, z1, z2, n);
    PCGB_POST_LAUNCH();
    ntt_forward_from(pl, party == 0 ? x1 : x2, T, 1, true, st);
    ntt_forward_from(pl, party == 0 ? x2 : x1, T + n, 1, true, st);
    ntt_forward_from(pl, T + 2 * n, T + 2 * n, 1, false, st);
    triple_slots_kernel<<<grid_for(n), kTpb, 0, st>>>(T, T + n, T + 2 * n, n, l1, l2, r2_mod_p(),
                                                      a, b, c);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(T, st));
}

void verify_ole_device(int N, const uint64_t* x0, const uint64_t* z0, const uint64_t* x1,
                       const uint64_t* z1, unsigned long long* bad, cudaStream_t st) {
    if (!x0 || !z0 || !x1 || !z1 || !bad) fail(PCGB_EINVAL, "verify_ole: null pointer");
    const NttPlan& pl = ntt_plan(log2_checked(N, "verify_ole"));
    const size_t n = static_cast<size_t>(N);
    uint64_t* T = static_cast<uint64_t*>(pool_alloc(3 * n * sizeof(uint64_t), st));  // X0 | X1 | Z
    PCGB_CK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st));
    add_reduce_kernel<<<grid_for(n), kTpb, 0, st>>>(T + 2 * n, z0, z1, n);
    PCGB_POST_LAUNCH();
    ntt_forward_from(pl, x0, T, 1, true, st);
    ntt_forward_from(pl, x1, T + n, 1, true, st);
    ntt_forward_from(pl, T + 2 * n, T + 2 * n, 1, false, st);
    ole_check_kernel<<<check_grid(n), kTpb, 0, st>>>(T, T + n, T + 2 * n, n, r2_mod_p(), bad);
    PCGB_POST_LAUNCH();
    PCGB_CK(cudaFreeAsync(T, st));
}

void verify_triples_device(int N, const uint64_t* a0, const uint64_t* b0, const uint64_t* c0,
                           const uint64_t* a1, const uint64_t* b1, const uint64_t* c1,
                           unsigned long long* bad, cudaStream_t st) {
    if (!a0 || !b0 || !c0 || !a1 || !b1 || !c1 || !bad) fail(PCGB_EINVAL, "verify_triples: null pointer");
    if (N < 1) fail(PCGB_EINVAL, "verify_triples: N must be positive");
    const size_t n = static_cast<size_t>(N);
    PCGB_CK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st));
    triple_check_kernel<<<check_grid(n), kTpb, 0, st>>>(a0, b0, c0, a1, b1, c1, n, r2_mod_p(), bad);
    PCGB_POST_LAUNCH();
}

}  // namespace pcgb
