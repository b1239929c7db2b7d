// Serving loop: continuous batching of PCG-OLE expansion requests on one GPU.
//
// A worker thread owns S slots, each with a low- and a high-priority CUDA
// stream.  Requests wait in arrival order; they are admitted as soon as a
// slot is free and their HBM footprint (keys, noise, outputs and the
// expansion workspace) fits the memory budget next to everything already in
// flight, so requests that arrive while others are on the GPU start
// immediately and their kernels overlap on the device.
//   * Large requests (c^2 * N > 2^20) run one at a time, each in its own
//     slot on a low-priority stream.
//   * Small ones pass queued large ones.  Up to `batch_max` pending small
//     requests of N in 2^14 .. 2^20, whatever their (N, c, t), are admitted
//     together into one slot and run as ONE batch (expand_batch_ws): one
//     launch per stage for all of them, on the slot's high-priority stream,
//     so the block scheduler starts their CTAs ahead of a large kernel's
//     pending ones.  Other small requests (N below 2^14) run alone there.
// Each admitted request deals fresh seeded keys and noise on its slot's
// stream and is expanded against its shape's resident plan (a_i images,
// gather plan, NTT tables); a device digest of x and z is copied back and a
// host callback (cudaLaunchHostFunc) stamps the completion time and wakes
// the worker.  Memory comes from the library's stream-ordered pool
// (allocated and freed on the slot's stream), so a finished request's
// memory is reused by the next one without a device synchronisation.
//
// The reference has no serving path; its one-request-at-a-time flow is
// GPU_baseline/e2e_full_bench.cu's serial arm.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "pcg_b200.h"
#include "pcgb_internal.h"

namespace pcgb {
namespace {

using clk = std::chrono::steady_clock;

// Requests with c^2 * N above this are "large".  At most one large request
// is in flight at a time (they run back to back, as one at a time would,
// instead of slowing each other down by sharing the GPU); small requests
// take any free slot ahead of queued large ones and run on their slot's
// high-priority stream, so the block scheduler starts their CTAs ahead of a
// large kernel's pending ones.  Small requests thus never wait behind a
// large one, and large ones lose only the SM time the small ones use.
constexpr uint64_t kSmallWork = uint64_t{1} << 20;

// Requests per batch at most (the pinned digest area holds this many per slot).
constexpr int kBatchCap = 32;
// Leaf shape of every plan that may run in a batch: one shape for all, so
// requests of any (N, c, t) share the fused leaf launch (the smallest bin of
// a batchable shape, N = 2^14 at t = 32, still holds one 64 x 8 tile).
constexpr int kBatchLeafThreads = 64, kBatchLeafLeaves = 8;

struct Req {
    uint64_t ticket = 0;
    pcgb_request r{};
    int state = 0;  // 0 pending, 1 running, 2 done, 3 failed
    int slot = -1;
    int index = 0;      // position within its slot's batch
    bool big = false;   // c^2 * N above kSmallWork
    bool batchable = false;
    size_t bytes = 0;
    double submit_s = 0, start_s = 0, done_s = 0;
    uint64_t dx = 0, dz = 0;
    int status = 0;
    std::string err;
};

struct CallbackCtx {
    pcgb_server* s;
    std::vector<Req*> rs;
};

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

}  // namespace
}  // namespace pcgb

struct pcgb_server {
    int dev = 0;
    int n_slots = 1;
    size_t budget = 0;
    int max_in_flight = 1;   // requests
    int batch_max = 1;       // small requests per batch
    uint64_t a_seed = 0;
    std::vector<cudaStream_t> streams;     // per slot, lowest priority
    std::vector<cudaStream_t> hi_streams;  // per slot, highest priority (small requests)
    std::vector<int> slot_busy;
    uint64_t* h_digest = nullptr;  // pinned, 2 words per request, kBatchCap requests per slot
    std::mutex plans_mu;
    std::map<std::tuple<int, int, int>, pcgb_expander*> plans;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<pcgb::Req*> pending;
    std::vector<pcgb::Req*> finished;  // filled by host callbacks
    std::unordered_map<uint64_t, std::unique_ptr<pcgb::Req>> reqs;
    size_t in_flight_bytes = 0;
    int in_flight = 0;          // requests
    int slots_in_use = 0;
    int big_in_flight = 0;
    uint64_t next_ticket = 1;
    bool stopping = false;
    std::thread worker;
    pcgb::clk::time_point t0;

    double now() const {
        return std::chrono::duration<double>(pcgb::clk::now() - t0).count();
    }
};

namespace pcgb {
namespace {

void validate(const pcgb_request& r) {
    if (r.N < 16 || (r.N & (r.N - 1)) || r.N > (1 << kMaxLogN))
        fail(PCGB_EINVAL, "request: N must be a power of two in [16, 2^24]");
    if (r.c < 1 || r.c > 8) fail(PCGB_EINVAL, "request: c must be in [1, 8]");
    if (r.t < 1 || (r.t & (r.t - 1)) || r.N / r.t < 4)
        fail(PCGB_EINVAL, "request: t must be a power of two with N/t >= 4");
    if (r.party != 0 && r.party != 1) fail(PCGB_EINVAL, "request: party must be 0 or 1");
}

// A request can join a batch: small, and a length the batched NTT handles.
bool batchable_shape(int N, int c) {
    int lg = 0;
    while ((1 << lg) < N) ++lg;
    return static_cast<uint64_t>(c) * c * static_cast<uint64_t>(N) <= kSmallWork &&
           ntt_mac_multi_ok(lg);
}

pcgb_expander* get_plan(pcgb_server* s, int N, int c, int t) {
    std::lock_guard<std::mutex> lk(s->plans_mu);
    auto key = std::make_tuple(N, c, t);
    auto it = s->plans.find(key);
    if (it != s->plans.end()) return it->second;
    std::vector<uint64_t> a(static_cast<size_t>(c > 1 ? c - 1 : 1) * N);
    public_a_host(N, c, s->a_seed, a.data());
    pcgb_expander* e = expander_create(N, c, t, 1, PCGB_PRG_CHACHA8, a.data(), nullptr);
    try {
        if (s->batch_max > 1 && batchable_shape(N, c))
            expander_set_leaf_shape(e, kBatchLeafThreads, kBatchLeafLeaves);
        else
            expander_autotune(e);
    } catch (...) {
        expander_destroy(e);
        throw;
    }
    s->plans[key] = e;
    return e;
}

// Footprint of one request: dealt keys of both parties, noise, outputs and
// the expansion workspace.
size_t footprint(pcgb_expander* e, const pcgb_request& r) {
    int K = 0, levels = 0, nk = 0;
    size_t ws = 0;
    expander_info(e, &K, &levels, &nk, &ws);
    const size_t ct = static_cast<size_t>(r.c) * r.t;
    return align256(2 * sizeof(Blk) * K) + align256(sizeof(Blk) * K * levels * nk) +
           align256(8 * static_cast<size_t>(K)) + align256(16 * ct) +
           align256(16 * static_cast<size_t>(r.N)) + align256(ws);
}

void CUDART_CB on_done(void* p) {
    auto* ctx = static_cast<CallbackCtx*>(p);
    pcgb_server* s = ctx->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const double t = s->now();
        for (Req* r : ctx->rs) {
            r->done_s = t;
            s->finished.push_back(r);
        }
    }
    s->cv_work.notify_one();
    delete ctx;
}

// One request's device buffers, carved from one pool block.
struct ReqMem {
    char* base = nullptr;
    Blk *roots = nullptr, *cws = nullptr;
    uint64_t *cwo = nullptr, *pos = nullptr, *val = nullptr, *x = nullptr, *z = nullptr;
    Workspace ws;
};

ReqMem carve_request(pcgb_expander* e, const Req* r, cudaStream_t st, bool deal) {
    int K = 0, levels = 0, nk = 0;
    size_t wsb = 0;
    expander_info(e, &K, &levels, &nk, &wsb);
    const size_t ct = static_cast<size_t>(r->r.c) * r->r.t, N = r->r.N;
    ReqMem m;
    m.base = static_cast<char*>(pool_alloc(r->bytes, st));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = m.base + off;
        off += align256(bytes);
        return p;
    };
    m.roots = reinterpret_cast<Blk*>(take(2 * sizeof(Blk) * K));
    m.cws = reinterpret_cast<Blk*>(take(sizeof(Blk) * K * levels * nk));
    m.cwo = reinterpret_cast<uint64_t*>(take(8 * static_cast<size_t>(K)));
    m.pos = reinterpret_cast<uint64_t*>(take(16 * ct));
    m.val = m.pos + ct;
    m.x = reinterpret_cast<uint64_t*>(take(16 * N));
    m.z = m.x + N;
    m.ws = workspace_carve(e, take(wsb));
    if (deal) {   // fresh keys (both parties' roots) and this party's noise
        deal_keys_device(e, r->r.seed, m.roots, m.roots + K, m.cws, m.cwo, st);
        noise_device(r->r.N, r->r.c, r->r.t, r->r.seed, r->r.party, m.pos, m.val, st);
    }
    return m;
}

// Enqueue admitted requests on their slot's stream (worker thread only): a
// batch of small requests as one batched expansion, or one request alone.
void launch(pcgb_server* s, const std::vector<Req*>& rs) {
    const int slot = rs[0]->slot;
    const bool batch = rs[0]->batchable && s->batch_max > 1;
    cudaStream_t st = rs[0]->big ? s->streams[slot] : s->hi_streams[slot];
    const int n = static_cast<int>(rs.size());
    std::vector<pcgb_expander*> es(n);
    std::vector<ReqMem> mem(n);
    for (int i = 0; i < n; ++i) {
        es[i] = get_plan(s, rs[i]->r.N, rs[i]->r.c, rs[i]->r.t);
        mem[i] = carve_request(es[i], rs[i], st, !batch);
    }
    if (batch) {
        // Keys and noise of the whole batch: one dealer and one noise launch.
        std::vector<uint64_t> seed(n);
        std::vector<int> pty(n);
        std::vector<Blk*> r0(n), r1(n), kc(n);
        std::vector<uint64_t*> co(n), ps(n), vl(n);
        for (int i = 0; i < n; ++i) {
            int K = 0, levels = 0, nk = 0;
            size_t wsb = 0;
            expander_info(es[i], &K, &levels, &nk, &wsb);
            seed[i] = rs[i]->r.seed;
            pty[i] = rs[i]->r.party;
            r0[i] = mem[i].roots; r1[i] = mem[i].roots + K; kc[i] = mem[i].cws;
            co[i] = mem[i].cwo; ps[i] = mem[i].pos; vl[i] = mem[i].val;
        }
        deal_noise_multi_device(n, es.data(), seed.data(), pty.data(), r0.data(), r1.data(),
                                kc.data(), co.data(), ps.data(), vl.data(), st);
        std::vector<Workspace> ws(n);
        std::vector<int> party(n);
        std::vector<const Blk*> roots(n), cws(n);
        std::vector<const uint64_t*> cwo(n), pos(n), val(n);
        std::vector<uint64_t*> x(n), z(n);
        for (int i = 0; i < n; ++i) {
            int K = 0, levels = 0, nk = 0;
            size_t wsb = 0;
            expander_info(es[i], &K, &levels, &nk, &wsb);
            ws[i] = mem[i].ws;
            party[i] = rs[i]->r.party;
            roots[i] = party[i] ? mem[i].roots + K : mem[i].roots;
            cws[i] = mem[i].cws; cwo[i] = mem[i].cwo;
            pos[i] = mem[i].pos; val[i] = mem[i].val;
            x[i] = mem[i].x; z[i] = mem[i].z;
        }
        expand_batch_ws(n, es.data(), ws.data(), party.data(), roots.data(), cws.data(),
                        cwo.data(), pos.data(), val.data(), x.data(), z.data(), st);
    } else {
        for (int i = 0; i < n; ++i) {
            int K = 0, levels = 0, nk = 0;
            size_t wsb = 0;
            expander_info(es[i], &K, &levels, &nk, &wsb);
            const ReqMem& m = mem[i];
            expand_device_ws(es[i], m.ws, rs[i]->r.party,
                             rs[i]->r.party ? m.roots + K : m.roots, m.cws, m.cwo, m.pos, m.val,
                             m.x, m.z, st);
        }
    }
    // Digests of every x and z in one launch, one copy back.
    uint64_t* dig = static_cast<uint64_t*>(pool_alloc(16 * static_cast<size_t>(n), st));
    std::vector<const uint64_t*> v(2 * n);
    std::vector<size_t> len(2 * n);
    std::vector<uint64_t*> out(2 * n);
    for (int i = 0; i < n; ++i) {
        v[2 * i] = mem[i].x; v[2 * i + 1] = mem[i].z;
        len[2 * i] = len[2 * i + 1] = static_cast<size_t>(rs[i]->r.N);
        out[2 * i] = dig + 2 * i; out[2 * i + 1] = dig + 2 * i + 1;
    }
    digest_multi_device(2 * n, v.data(), len.data(), out.data(), st);
    PCGB_CK(cudaMemcpyAsync(s->h_digest + 2 * static_cast<size_t>(slot) * kBatchCap, dig, 16 * n,
                            cudaMemcpyDeviceToHost, st));
    PCGB_CK(cudaFreeAsync(dig, st));
    for (int i = 0; i < n; ++i) PCGB_CK(cudaFreeAsync(mem[i].base, st));
    PCGB_CK(cudaLaunchHostFunc(st, on_done, new CallbackCtx{s, rs}));
}

// The request to admit next, or pending.end(): the first pending request in
// arrival order that may start now -- a large request is skipped while
// another large one is in flight, and the candidate's footprint must fit
// the budget next to what is in flight (one larger than the whole budget
// still runs alone).  The admission loop and the worker's wait use this same
// rule, so the wait never holds the lock while an admission is possible.
std::deque<Req*>::iterator next_admissible(pcgb_server* s) {
    if (s->in_flight >= s->max_in_flight || s->slots_in_use >= s->n_slots) return s->pending.end();
    for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
        Req* r = *it;
        if (r->big && s->big_in_flight > 0) continue;
        if (s->in_flight > 0 && s->in_flight_bytes + r->bytes > s->budget) return s->pending.end();
        return it;
    }
    return s->pending.end();
}

void release(pcgb_server* s, Req* r) {
    s->in_flight_bytes -= r->bytes;
    --s->in_flight;
    s->big_in_flight -= r->big ? 1 : 0;
    if (--s->slot_busy[r->slot] == 0) --s->slots_in_use;
}

void worker_loop(pcgb_server* s) {
    cudaSetDevice(s->dev);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // Completions: collect digests, release memory accounting and slots.
        for (Req* r : s->finished) {
            const size_t d = 2 * (static_cast<size_t>(r->slot) * kBatchCap + r->index);
            r->dx = s->h_digest[d];
            r->dz = s->h_digest[d + 1];
            r->state = 2;
            release(s, r);
        }
        if (!s->finished.empty()) {
            s->finished.clear();
            s->cv_done.notify_all();
        }
        if (s->stopping && s->in_flight == 0 && s->pending.empty()) break;
        // Admissions (next_admissible's rule); a batchable request takes
        // the next pending batchable ones along, up to batch_max, as long
        // as their footprints fit.
        for (auto it = next_admissible(s); it != s->pending.end(); it = next_admissible(s)) {
            int slot = -1;
            for (int i = 0; i < s->n_slots; ++i)
                if (!s->slot_busy[i]) { slot = i; break; }
            if (slot < 0) break;
            std::vector<Req*> unit{*it};
            s->pending.erase(it);
            size_t bytes = unit[0]->bytes;
            if (unit[0]->batchable && s->batch_max > 1) {
                const int cap = std::min({s->batch_max, kBatchCap, s->max_in_flight - s->in_flight});
                for (auto j = s->pending.begin();
                     j != s->pending.end() && static_cast<int>(unit.size()) < cap;) {
                    if ((*j)->batchable && s->in_flight_bytes + bytes + (*j)->bytes <= s->budget) {
                        bytes += (*j)->bytes;
                        unit.push_back(*j);
                        j = s->pending.erase(j);
                    } else {
                        ++j;
                    }
                }
            }
            const double t0 = s->now();
            for (size_t i = 0; i < unit.size(); ++i) {
                Req* r = unit[i];
                r->slot = slot;
                r->index = static_cast<int>(i);
                r->state = 1;
                r->start_s = t0;
                s->in_flight_bytes += r->bytes;
                ++s->in_flight;
                s->big_in_flight += r->big ? 1 : 0;
            }
            s->slot_busy[slot] = static_cast<int>(unit.size());
            ++s->slots_in_use;
            lk.unlock();
            bool ok = true;
            std::string msg;
            try {
                launch(s, unit);
            } catch (const std::exception& ex) {
                ok = false;
                msg = ex.what();
            }
            lk.lock();
            if (!ok) {
                for (Req* r : unit) {
                    r->state = 3;
                    r->status = PCGB_ECUDA;
                    r->err = msg;
                    release(s, r);
                }
                s->cv_done.notify_all();
            }
        }
        // Sleep until something can change: a completion, shutdown, or a
        // request that can actually be admitted now.
        s->cv_work.wait(lk, [s] {
            if (!s->finished.empty() || (s->stopping && s->in_flight == 0)) return true;
            return next_admissible(s) != s->pending.end();
        });
    }
}

}  // namespace

pcgb_server* server_create(int n_streams, size_t budget, int max_in_flight, uint64_t a_seed) {
    if (n_streams < 1 || n_streams > 64) fail(PCGB_EINVAL, "server: n_streams must be in [1, 64]");
    if (max_in_flight < 1) fail(PCGB_EINVAL, "server: max_in_flight must be >= 1");
    auto* s = new pcgb_server();
    PCGB_CK(cudaGetDevice(&s->dev));
    s->n_slots = n_streams;
    s->max_in_flight = max_in_flight;
    // Batching needs room for more requests than slots.
    s->batch_max = max_in_flight > n_streams ? kBatchCap : 1;
    s->a_seed = a_seed;
    if (budget == 0) {
        size_t free_b = 0, total_b = 0;
        PCGB_CK(cudaMemGetInfo(&free_b, &total_b));
        budget = free_b / 2;
    }
    s->budget = budget;
    s->streams.resize(n_streams);
    s->slot_busy.assign(n_streams, 0);
    int prio_low = 0, prio_high = 0;
    PCGB_CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    s->hi_streams.resize(n_streams);
    for (auto& st : s->streams)
        PCGB_CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_low));
    for (auto& st : s->hi_streams)
        PCGB_CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_high));
    PCGB_CK(cudaMallocHost(&s->h_digest, 16 * static_cast<size_t>(n_streams) * kBatchCap));
    s->t0 = clk::now();
    s->worker = std::thread(worker_loop, s);
    return s;
}

void server_prepare(pcgb_server* s, int N, int c, int t) {
    pcgb_request r{};
    r.N = N; r.c = c; r.t = t;
    validate(r);
    get_plan(s, N, c, t);
}

uint64_t server_submit(pcgb_server* s, const pcgb_request& r) {
    validate(r);
    pcgb_expander* e = get_plan(s, r.N, r.c, r.t);
    auto req = std::make_unique<Req>();
    req->r = r;
    req->big = static_cast<uint64_t>(r.c) * r.c * static_cast<uint64_t>(r.N) > kSmallWork;
    req->batchable = batchable_shape(r.N, r.c);
    req->bytes = footprint(e, r);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) fail(PCGB_ESTATE, "server: shutting down");
    req->ticket = s->next_ticket++;
    req->submit_s = s->now();
    Req* raw = req.get();
    s->reqs[raw->ticket] = std::move(req);
    s->pending.push_back(raw);
    s->cv_work.notify_one();
    return raw->ticket;
}

int server_wait(pcgb_server* s, uint64_t ticket, pcgb_result* out, int timeout_ms) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) fail(PCGB_EINVAL, "server: unknown ticket");
    Req* r = it->second.get();
    const auto pred = [r] { return r->state >= 2; };
    if (timeout_ms < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
        return PCGB_ETIMEOUT;
    if (out) {
        out->digest_x = r->dx;
        out->digest_z = r->dz;
        out->submit_s = r->submit_s;
        out->start_s = r->start_s;
        out->done_s = r->done_s;
        out->status = r->state == 2 ? PCGB_OK : r->status;
    }
    const int rc = r->state == 2 ? PCGB_OK : r->status;
    if (rc != PCGB_OK) fail(rc, "request failed: " + r->err);
    s->reqs.erase(it);
    return PCGB_OK;
}

void server_run_trace(pcgb_server* s, const pcgb_request* reqs, int n, pcgb_result* out,
                      double timeout_s) {
    std::vector<uint64_t> tickets(n);
    const auto start = clk::now();
    for (int i = 0; i < n; ++i) {
        const auto when = start + std::chrono::duration_cast<clk::duration>(
                                      std::chrono::duration<double>(reqs[i].arrival_s));
        std::this_thread::sleep_until(when);
        tickets[i] = server_submit(s, reqs[i]);
    }
    const auto deadline = start + std::chrono::duration_cast<clk::duration>(
                                      std::chrono::duration<double>(timeout_s));
    for (int i = 0; i < n; ++i) {
        const auto left = std::chrono::duration_cast<std::chrono::milliseconds>(deadline - clk::now());
        const int ms = static_cast<int>(std::max<long long>(0, left.count()));
        if (server_wait(s, tickets[i], out ? out + i : nullptr, ms) == PCGB_ETIMEOUT)
            fail(PCGB_ETIMEOUT, "server: trace did not finish within the timeout");
    }
}

void server_destroy(pcgb_server* s, int timeout_ms) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        for (Req* r : s->pending) {  // cancel what has not started
            r->state = 3;
            r->status = PCGB_ESTATE;
            r->err = "cancelled: server shut down";
        }
        s->pending.clear();
        s->cv_done.notify_all();
    }
    s->cv_work.notify_all();
    // The worker exits once in-flight work completed; bound the wait.
    const auto deadline = clk::now() + std::chrono::milliseconds(timeout_ms);
    bool drained = false;
    while (clk::now() < deadline) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->in_flight == 0) { drained = true; break; }
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
    s->cv_work.notify_all();
    if (!drained) {
        // Leave the object alive rather than free memory the GPU still uses.
        s->worker.detach();
        fail(PCGB_ETIMEOUT, "server: in-flight requests did not finish in time");
    }
    s->worker.join();
    for (auto& st : s->streams) cudaStreamSynchronize(st);
    for (auto& st : s->hi_streams) cudaStreamSynchronize(st);
    for (auto& kv : s->plans) expander_destroy(kv.second);
    for (auto& st : s->streams) cudaStreamDestroy(st);
    for (auto& st : s->hi_streams) cudaStreamDestroy(st);
    cudaFreeHost(s->h_digest);
    delete s;
}

void server_stats(pcgb_server* s, int* pending, int* in_flight, size_t* bytes, int* plans) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (pending) *pending = static_cast<int>(s->pending.size());
    if (in_flight) *in_flight = s->in_flight;
    if (bytes) *bytes = s->in_flight_bytes;
    std::lock_guard<std::mutex> lk2(s->plans_mu);
    if (plans) *plans = static_cast<int>(s->plans.size());
}

}  // namespace pcgb
