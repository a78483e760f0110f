// Batched products (pg_mul_batch) and library-owned device buffers (pg_buf_*).
//
// A batch is a list of independent products of any sizes, optionally with a second product
// added or subtracted in the transform domain (the binary-splitting form R = Qr*Rl + Pl*Rr,
// src/engine/binary_splitting.cpp:184-200 in the reference, which issues each of those
// products as its own Multiplier call). Jobs are bucketed by transform length; every bucket
// runs as one launch per pass over all of its jobs (operands located through a per-job
// table on the device), one pointwise step and one CRT + carry launch, so a bucket of
// thousands of small products costs a handful of launches instead of thousands.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pi_b200.h"
#include "ntt_engine.cuh"

struct pg_buf {
    uint64_t* d = nullptr;
    size_t cap = 0;
    size_t len = 0;
    int device = 0;
};

namespace pg {

const DeviceTables& ctx_tables(pg_ctx* c);
cudaStream_t ctx_stream(pg_ctx* c);
std::mutex& ctx_mutex(pg_ctx* c);
uint64_t* ctx_launches(pg_ctx* c);
void ctx_set_error(pg_ctx* c, const std::string& msg);
int ctx_device(pg_ctx* c);
struct BatchWork;
BatchWork* ctx_batch(pg_ctx* c);

// Residue arrays of the batch (growable), the per-job tables and the CRT sync words.
struct BatchWork {
    uint32_t* res[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t res_cap = 0;  // words per array
    uint32_t* sync = nullptr;
    uint64_t sync_cap = 0;
    uint32_t* errw = nullptr;
    SrcEntry* d_src = nullptr;
    uint64_t src_cap = 0;
    DstEntry* d_dst = nullptr;
    uint64_t dst_cap = 0;
    SrcEntry* h_src = nullptr;  // pinned staging
    DstEntry* h_dst = nullptr;
    uint64_t h_cap = 0;

    ~BatchWork() {
        for (auto* r : res)
            if (r) dev_free(r);
        if (sync) dev_free(sync);
        if (errw) dev_free(errw);
        if (d_src) dev_free(d_src);
        if (d_dst) dev_free(d_dst);
        if (h_src) pinned_free(h_src);
        if (h_dst) pinned_free(h_dst);
    }
};

BatchWork* batch_state_new() { return new (std::nothrow) BatchWork; }
void batch_state_delete(BatchWork* w) { delete w; }

namespace {

template <class T>
cudaError_t grow_dev(T** p, uint64_t& cap, uint64_t n) {
    if (n <= cap) return cudaSuccess;
    n = std::max(n, cap + cap / 2);
    if (*p) dev_free(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = pg::dev_malloc((void**)p, n * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
}

// out = A*B (+/-) C*D per element (Montgomery products; the 2^-32 factor is the one the CRT
// constants expect). Job j's arrays start at j * 3L; subtract when dtab[j].centred.
__global__ void batch_combine_kernel(uint32_t* A, const uint32_t* B, const uint32_t* C, const uint32_t* D,
                                     uint64_t L, uint64_t njobs, const DstEntry* dtab) {
    const uint64_t per_job = 3 * L / 4;  // uint4 groups per job
    const uint64_t total = per_job * njobs;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t job = i / per_job;
        const uint64_t off = (i - job * per_job) * 4;
        const int j = (int)(off / L);
        const uint32_t p = kPrime(j), pinv = inv_mod_2_32(p);
        const uint64_t g = job * 3 * L + off;
        const uint4 a = *reinterpret_cast<const uint4*>(A + g);
        const uint4 b = *reinterpret_cast<const uint4*>(B + g);
        const uint4 c = *reinterpret_cast<const uint4*>(C + g);
        const uint4 d = *reinterpret_cast<const uint4*>(D + g);
        const bool sub = dtab[job].centred != 0;
        auto f = [&](uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
            const uint32_t u = mul_mont(x, y, p, pinv), v = mul_mont(z, w, p, pinv);
            return sub ? sub_mod(u, v, p) : add_mod(u, v, p);
        };
        uint4 r;
        r.x = f(a.x, b.x, c.x, d.x);
        r.y = f(a.y, b.y, c.y, d.y);
        r.z = f(a.z, b.z, c.z, d.z);
        r.w = f(a.w, b.w, c.w, d.w);
        *reinterpret_cast<uint4*>(A + g) = r;
    }
}

enum class Kind { Mul, Sqr, Acc };

struct Item {
    size_t job;
    int logL;
    Kind kind;
    uint64_t nwords;  // output words
};

pg_status fail(pg_ctx* c, pg_status s, const std::string& msg) {
    ctx_set_error(c, msg);
    return s;
}

pg_status cuda_fail(pg_ctx* c, cudaError_t e, const char* where) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return fail(c, PG_ERR_OOM, std::string(where) + ": out of device memory");
    return fail(c, PG_ERR_DEVICE, std::string(where) + ": " + cudaGetErrorString(e));
}

bool misaligned(const void* p) { return ((uintptr_t)p & 15) != 0; }

std::string job_msg(size_t i, const char* what) { return "job " + std::to_string(i) + ": " + what; }

}  // namespace

// Residue words per batch array before a bucket is split into several chunks.
constexpr uint64_t kBatchChunkWords = 256ull << 20;

// A validated batch: items sorted by (transform length, kind), cut into chunks that run as one
// launch per pass each. prepare_batch sizes every buffer for all chunks and uploads the job tables;
// enqueue_batch then only enqueues kernels and memsets (no allocation, no host wait), so that it can
// run inside a stream capture (pg_graph_capture_level).
struct BatchPlan {
    struct Chunk {
        uint64_t k0, k1;  // items [k0, k1)
        int logL;
        Kind kind;
        uint64_t maxw;    // longest output in words
    };
    std::vector<Chunk> chunks;
    uint64_t n = 0;       // items
    std::vector<std::pair<uint64_t*, size_t>> zero;  // outputs of empty products (bytes)
};

static pg_status prepare_batch(pg_ctx* ctx, BatchWork* W, const pg_job* jobs, size_t njobs, BatchPlan& bp) {
    const size_t maxl = pg_mul_max_limbs();
    bp = BatchPlan{};

    // Validate, zero the outputs of empty products, bucket the rest.
    std::vector<Item> items;
    items.reserve(njobs);
    for (size_t i = 0; i < njobs; ++i) {
        const pg_job& J = jobs[i];
        const bool acc = J.acc != 0;
        if (J.acc < -1 || J.acc > 1) return fail(ctx, PG_ERR_BAD_ARG, job_msg(i, "acc must be -1, 0 or +1"));
        if (!J.out || (J.na && !J.a) || misaligned(J.a) || misaligned(J.b) || misaligned(J.out))
            return fail(ctx, PG_ERR_BAD_ARG, job_msg(i, "null or unaligned pointer"));
        const size_t nb = J.b ? J.nb : J.na;
        size_t nc = 0, nd = 0;
        if (acc) {
            if ((J.nc && !J.c) || misaligned(J.c) || misaligned(J.d))
                return fail(ctx, PG_ERR_BAD_ARG, job_msg(i, "null or unaligned pointer"));
            nc = J.nc;
            nd = J.d ? J.nd : J.nc;
        }
        if (J.na > maxl || nb > maxl - J.na || nc > maxl || nd > maxl - nc)
            return fail(ctx, PG_ERR_TOO_LARGE, job_msg(i, "product exceeds the transform range"));
        const size_t top = std::max(J.na + nb, nc + nd) + (J.acc > 0 ? 1 : 0);
        if (J.out_cap < top) return fail(ctx, PG_ERR_BAD_ARG, job_msg(i, "out_cap below the result length"));
        // A sum of two products needs |coefficient| < P/2: min(na,nb) + min(nc,nd) <= 2^24 limbs.
        if (acc && std::min(J.na, nb) + std::min(nc, nd) > ((size_t)1 << 24))
            return fail(ctx, PG_ERR_TOO_LARGE, job_msg(i, "accumulated products exceed the CRT bound"));
        const bool p1 = J.na && nb, p2 = acc && nc && nd;
        if (!p1 && !p2) {  // an empty product: its output is zeroed when the batch is enqueued
            bp.zero.push_back({J.out, top * 8});
            continue;
        }
        Item it;
        it.job = i;
        it.kind = acc ? Kind::Acc : (J.b ? Kind::Mul : Kind::Sqr);
        it.logL = std::max(p1 ? product_logL(J.na, nb) : kMinLogL, p2 ? product_logL(nc, nd) : kMinLogL);
        it.nwords = 2ull * top;
        items.push_back(it);
    }
    if (items.empty()) return PG_OK;
    bp.n = items.size();
    cudaStream_t st = ctx_stream(ctx);
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) {
        return x.logL != y.logL ? x.logL > y.logL : (int)x.kind < (int)y.kind;
    });

    // Per-job tables: sources grouped by operand slot ([slot][item], slots a, b, c, d) so that a
    // pass over one slot reads consecutive entries; one destination per item.
    const uint64_t n = items.size();
    // Reusing pinned staging: wait for the copies of an earlier batch on this stream.
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "stream");
    if (4 * n > W->h_cap) {
        if (W->h_src) pinned_free(W->h_src);
        if (W->h_dst) pinned_free(W->h_dst);
        W->h_src = nullptr;
        W->h_dst = nullptr;
        W->h_cap = 0;
        const uint64_t cap = std::max<uint64_t>(4 * n, 1024);
        e = pinned_malloc(&W->h_src, cap * sizeof(SrcEntry));
        if (e == cudaSuccess) e = pinned_malloc(&W->h_dst, cap * sizeof(DstEntry));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pinned tables");
        W->h_cap = cap;
    }
    for (uint64_t k = 0; k < n; ++k) {
        const pg_job& J = jobs[items[k].job];
        const uint64_t nb = J.b ? J.nb : J.na;
        // An empty operand still gets a valid address (it is never read: ncoef = 0).
        auto src = [&](const uint64_t* x, uint64_t nx) {
            SrcEntry s;
            s.words = reinterpret_cast<const uint32_t*>(x && nx ? x : J.out);
            s.ncoef = x ? 2 * nx : 0;
            return s;
        };
        W->h_src[0 * n + k] = src(J.a, J.na);
        W->h_src[1 * n + k] = src(J.b ? J.b : J.a, nb);
        W->h_src[2 * n + k] = src(J.acc ? J.c : nullptr, J.acc ? J.nc : 0);
        W->h_src[3 * n + k] = src(J.acc ? (J.d ? J.d : J.c) : nullptr, J.acc ? (J.d ? J.nd : J.nc) : 0);
        DstEntry d;
        d.out = reinterpret_cast<uint32_t*>(J.out);
        d.nwords = items[k].nwords;
        d.centred = J.acc < 0 ? 1u : 0u;
        d.pad = 0;
        W->h_dst[k] = d;
    }
    e = grow_dev(&W->d_src, W->src_cap, 4 * n);
    if (e == cudaSuccess) e = grow_dev(&W->d_dst, W->dst_cap, n);
    if (e == cudaSuccess && !W->errw) {
        e = pg::dev_malloc((void**)&W->errw, 4);
        if (e == cudaSuccess) e = cudaMemsetAsync(W->errw, 0, 4, st);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch tables");
    e = cudaMemcpyAsync(W->d_src, W->h_src, 4 * n * sizeof(SrcEntry), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(W->d_dst, W->h_dst, n * sizeof(DstEntry), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch table copy");

    // Chunks: consecutive items with the same (logL, kind), bounded by the array budget; every
    // buffer sized for the largest chunk before anything is enqueued.
    uint64_t res_need = 0, sync_need = 0;
    for (uint64_t k0 = 0; k0 < n;) {
        BatchPlan::Chunk ch;
        ch.k0 = k0;
        ch.logL = items[k0].logL;
        ch.kind = items[k0].kind;
        const uint64_t per = 3ull << ch.logL;
        const uint64_t fit = std::max<uint64_t>(1, kBatchChunkWords / per);
        uint64_t k1 = k0;
        ch.maxw = 0;
        while (k1 < n && k1 - k0 < fit && items[k1].logL == ch.logL && items[k1].kind == ch.kind) {
            ch.maxw = std::max(ch.maxw, items[k1].nwords);
            ++k1;
        }
        ch.k1 = k1;
        const uint64_t m = k1 - k0;
        const uint64_t bpj = (ch.maxw + kCrtThreads * kCrtWords - 1) / (kCrtThreads * kCrtWords);
        res_need = std::max(res_need, m * per);
        sync_need = std::max(sync_need, m + m * bpj);
        bp.chunks.push_back(ch);
        k0 = k1;
    }
    if (res_need > W->res_cap) {
        const uint64_t want = std::max(res_need, W->res_cap + W->res_cap / 2);
        for (auto*& r : W->res) {
            if (r) dev_free(r);
            r = nullptr;
        }
        W->res_cap = 0;
        for (auto*& r : W->res) {
            e = pg::dev_malloc((void**)&r, want * 4);
            if (e != cudaSuccess) {
                for (auto*& q : W->res) {
                    if (q) dev_free(q);
                    q = nullptr;
                }
                return cuda_fail(ctx, e, "batch residues");
            }
        }
        W->res_cap = want;
    }
    e = grow_dev(&W->sync, W->sync_cap, sync_need);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch sync words");
    return PG_OK;
}

static pg_status enqueue_batch(pg_ctx* ctx, BatchWork* W, const BatchPlan& bp, uint64_t* launches) {
    const DeviceTables& T = ctx_tables(ctx);
    cudaStream_t st = ctx_stream(ctx);
    const uint64_t n = bp.n;
    cudaError_t e = cudaSuccess;
    for (const auto& z : bp.zero)
        if ((e = cudaMemsetAsync(z.first, 0, z.second, st)) != cudaSuccess) return cuda_fail(ctx, e, "memset");
    if (n == 0) return PG_OK;
    e = cudaMemsetAsync(W->errw, 0, 4, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch error word");
    for (const BatchPlan::Chunk& ch : bp.chunks) {
        const uint64_t k0 = ch.k0;
        const int logL = ch.logL;
        const Kind kind = ch.kind;
        const uint64_t L = 1ull << logL;
        const uint64_t per = 3 * L;
        const uint64_t m = ch.k1 - ch.k0;
        const uint64_t maxw = ch.maxw;
        const Plan plan = T.plan(logL);
        const int last = plan.npass - 1;
        auto base = [&](uint32_t* data, int slot) {
            PassParams p{};
            p.data = data;
            p.out = data;
            p.L = L;
            p.logL = logL;
            p.job_stride = per;
            p.other_stride = per;
            p.njobs = (uint32_t)m;
            p.merge = 2;
            p.src = W->d_src + (uint64_t)slot * n + k0;
            p.error = W->errw;
            return p;
        };
        auto forward = [&](uint32_t* data, int slot, Fuse fuse_last, const uint32_t* other) -> cudaError_t {
            PassParams p = base(data, slot);
            p.other = other;
            for (int i = 0; i < plan.npass; ++i) {
                set_pass(p, plan, i);
                const Fuse f = (i == last) ? fuse_last : Fuse::None;
                cudaError_t r = launch_pass(plan, i, false, i == 0 ? Source::Limbs : Source::Residues, f, p, T.tw, st);
                if (r != cudaSuccess) return r;
                ++*launches;
            }
            return cudaSuccess;
        };
        auto inverse = [&](uint32_t* data, int from) -> cudaError_t {
            PassParams p = base(data, 0);
            for (int i = from; i >= 0; --i) {
                set_pass(p, plan, i);
                cudaError_t r = launch_pass(plan, i, true, Source::Residues, Fuse::None, p, T.tw, st);
                if (r != cudaSuccess) return r;
                ++*launches;
            }
            return cudaSuccess;
        };
        uint32_t* prod = W->res[0];
        if (kind == Kind::Sqr) {
            e = forward(W->res[0], 0, Fuse::SqrInverse, nullptr);
            if (e == cudaSuccess) e = inverse(W->res[0], last - 1);
        } else if (kind == Kind::Mul) {
            e = forward(W->res[0], 0, Fuse::None, nullptr);
            if (e == cudaSuccess) e = forward(W->res[1], 1, Fuse::MulInverse, W->res[0]);
            if (e == cudaSuccess) e = inverse(W->res[1], last - 1);
            prod = W->res[1];
        } else {
            for (int s = 0; s < 4 && e == cudaSuccess; ++s) e = forward(W->res[s], s, Fuse::None, nullptr);
            if (e == cudaSuccess) {
                const uint64_t groups = per / 4 * m;
                const unsigned blocks = (unsigned)std::min<uint64_t>((groups + 255) / 256, 148ull * 16);
                batch_combine_kernel<<<blocks, 256, 0, st>>>(W->res[0], W->res[1], W->res[2], W->res[3], L, m,
                                                             W->d_dst + k0);
                e = cudaGetLastError();
                ++*launches;
            }
            if (e == cudaSuccess) e = inverse(W->res[0], last);
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch passes");
        // CRT + carry over the chunk.
        const uint64_t bpj = (maxw + kCrtThreads * kCrtWords - 1) / (kCrtThreads * kCrtWords);
        e = cudaMemsetAsync(W->sync, 0, (m + m * bpj) * 4, st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch sync words");
        CrtParams c{};
        c.res = prod;
        c.res_stride = per;
        c.L = L;
        c.ticket = W->sync;
        c.status = W->sync + m;
        c.error = W->errw;
        c.blocks_per_job = bpj;
        c.k = make_crt_consts(logL);
        c.merge = 2;
        c.dtab = W->d_dst + k0;
        e = launch_crt(c, m * bpj, st, maxw);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch CRT");
        ++*launches;
    }
    return PG_OK;
}

// Wait for the enqueued batch, then read and clear the error word.
static pg_status finish_batch(pg_ctx* ctx, BatchWork* W) {
    cudaStream_t st = ctx_stream(ctx);
    uint32_t err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, W->errw, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch");
    if (err) {
        cudaMemsetAsync(W->errw, 0, 4, st);
        cudaStreamSynchronize(st);
        if (err == 1) return fail(ctx, PG_ERR_TIMEOUT, "carry look-back wait ran out of iterations");
        if (err & 4) return fail(ctx, PG_ERR_TIMEOUT, "tile load wait ran out of iterations");
        return fail(ctx, PG_ERR_BAD_ARG, "a job's result is negative (acc = -1 with a*b < c*d)");
    }
    return PG_OK;
}

static pg_status run_batch(pg_ctx* ctx, const pg_job* jobs, size_t njobs) {
    BatchWork* W = ctx_batch(ctx);
    if (!W) return fail(ctx, PG_ERR_OOM, "batch state");
    BatchPlan bp;
    pg_status s = prepare_batch(ctx, W, jobs, njobs, bp);
    if (s != PG_OK) return s;
    s = enqueue_batch(ctx, W, bp, ctx_launches(ctx));
    if (s != PG_OK || bp.n == 0) return s;
    return finish_batch(ctx, W);
}

}  // namespace pg

extern "C" {

pg_status pg_mul_batch(pg_ctx* ctx, const pg_job* jobs, size_t njobs) {
    if (!ctx || (njobs && !jobs)) return PG_ERR_BAD_ARG;
    if (njobs == 0) return PG_OK;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(pg::ctx_device(ctx));
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "cudaSetDevice");
    return pg::run_batch(ctx, jobs, njobs);
}

}  // extern "C"

// A captured level: its own buffers (so that later batches on the context, which may regrow the
// context's buffers, never move memory the graph points at) and the instantiated graph.
struct pg_graph {
    pg_ctx* ctx = nullptr;
    pg::BatchWork* W = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;  // kernels per replay
    uint64_t njobs = 0;     // products with work (empty products only zero their outputs)
};

extern "C" {

pg_status pg_graph_capture_level(pg_ctx* ctx, const pg_job* jobs, size_t njobs, pg_graph** out) {
    if (!ctx || !out || (njobs && !jobs)) return PG_ERR_BAD_ARG;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(pg::ctx_device(ctx));
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "cudaSetDevice");
    pg_graph* g = new (std::nothrow) pg_graph;
    if (!g) return PG_ERR_OOM;
    g->ctx = ctx;
    g->W = pg::batch_state_new();
    if (!g->W) {
        delete g;
        return PG_ERR_OOM;
    }
    auto drop = [&](pg_status s) {
        pg::batch_state_delete(g->W);
        delete g;
        return s;
    };
    // Validation, buffer sizing and the job tables' upload happen before the capture; the
    // capture records only kernels and memsets.
    pg::BatchPlan bp;
    pg_status s = pg::prepare_batch(ctx, g->W, jobs, njobs, bp);
    if (s != PG_OK) return drop(s);
    cudaStream_t st = pg::ctx_stream(ctx);
    e = cudaStreamSynchronize(st);  // the tables are in place before the graph is first replayed
    if (e != cudaSuccess) return drop(pg::cuda_fail(ctx, e, "stream"));
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return drop(pg::cuda_fail(ctx, e, "begin capture"));
    uint64_t counted = 0;
    s = pg::enqueue_batch(ctx, g->W, bp, &counted);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    if (s != PG_OK) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return drop(s);
    }
    if (e != cudaSuccess) return drop(pg::cuda_fail(ctx, e, "end capture"));
    e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g->exec = nullptr;
        return drop(pg::cuda_fail(ctx, e, "graph instantiate"));
    }
    g->launches = counted;
    g->njobs = bp.n;
    *out = g;
    return PG_OK;
}

pg_status pg_graph_launch(pg_graph* g) {
    if (!g || !g->exec) return PG_ERR_BAD_ARG;
    pg_ctx* ctx = g->ctx;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(pg::ctx_device(ctx));
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "cudaSetDevice");
    e = cudaGraphLaunch(g->exec, pg::ctx_stream(ctx));
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "graph launch");
    *pg::ctx_launches(ctx) += g->launches;
    if (g->njobs == 0) return cudaStreamSynchronize(pg::ctx_stream(ctx)) == cudaSuccess ? PG_OK : PG_ERR_DEVICE;
    return pg::finish_batch(ctx, g->W);
}

void pg_graph_destroy(pg_graph* g) {
    if (!g) return;
    {
        std::lock_guard<std::mutex> lock(pg::ctx_mutex(g->ctx));
        cudaSetDevice(pg::ctx_device(g->ctx));
        cudaStreamSynchronize(pg::ctx_stream(g->ctx));
        if (g->exec) cudaGraphExecDestroy(g->exec);
        pg::batch_state_delete(g->W);
    }
    delete g;
}

pg_status pg_buf_alloc(pg_ctx* ctx, size_t cap, pg_buf** out) {
    if (!ctx || !out) return PG_ERR_BAD_ARG;
    *out = nullptr;
    pg_buf* b = new (std::nothrow) pg_buf;
    if (!b) return PG_ERR_OOM;
    b->device = pg::ctx_device(ctx);
    b->cap = cap;
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess && cap) e = pg::dev_malloc((void**)&b->d, cap * 8);
    if (e == cudaSuccess && cap) e = cudaMemsetAsync(b->d, 0, cap * 8, pg::ctx_stream(ctx));
    if (e != cudaSuccess) {
        if (b->d) pg::dev_free(b->d);
        delete b;
        return pg::cuda_fail(ctx, e, "pg_buf_alloc");
    }
    *out = b;
    return PG_OK;
}

void pg_buf_free(pg_ctx* ctx, pg_buf* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (ctx) cudaStreamSynchronize(pg::ctx_stream(ctx));
    if (b->d) pg::dev_free(b->d);
    delete b;
}

pg_status pg_buf_upload(pg_ctx* ctx, pg_buf* b, const uint64_t* src, size_t n) {
    if (!ctx || !b || (n && !src)) return PG_ERR_BAD_ARG;
    if (n > b->cap) return pg::fail(ctx, PG_ERR_BAD_ARG, "pg_buf_upload: more limbs than the buffer holds");
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(b->device);
    cudaStream_t st = pg::ctx_stream(ctx);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(b->d, src, n * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && b->cap > n) e = cudaMemsetAsync(b->d + n, 0, (b->cap - n) * 8, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "pg_buf_upload");
    b->len = n;
    return PG_OK;
}

pg_status pg_buf_download(pg_ctx* ctx, const pg_buf* b, uint64_t* dst, size_t dst_cap, size_t* len) {
    if (!ctx || !b || !len || (b->len && !dst)) return PG_ERR_BAD_ARG;
    if (dst_cap < b->len) return pg::fail(ctx, PG_ERR_BAD_ARG, "pg_buf_download: destination too small");
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(b->device);
    cudaStream_t st = pg::ctx_stream(ctx);
    if (e == cudaSuccess && b->len) e = cudaMemcpyAsync(dst, b->d, b->len * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return pg::cuda_fail(ctx, e, "pg_buf_download");
    size_t n = b->len;
    while (n && dst[n - 1] == 0) --n;
    *len = n;
    return PG_OK;
}

uint64_t* pg_buf_device(pg_buf* b) { return b ? b->d : nullptr; }
size_t pg_buf_len(const pg_buf* b) { return b ? b->len : 0; }
size_t pg_buf_capacity(const pg_buf* b) { return b ? b->cap : 0; }

pg_status pg_buf_set_len(pg_buf* b, size_t n) {
    if (!b || n > b->cap) return PG_ERR_BAD_ARG;
    b->len = n;
    return PG_OK;
}

}  // extern "C"
