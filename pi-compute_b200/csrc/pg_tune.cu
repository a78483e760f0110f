// Autotuner of the pass split (pg_tune, pg_tune_save, pg_tune_load).
//
// For each transform length 2^logL the product can run as one contiguous pass (logL <= 14)
// or as 2 or 3 passes whose lengths multiply to 2^logL (plan_valid lists the constraints).
// pg_tune times every valid split on the device with a balanced product of that length,
// checks that it reproduces the built-in plan's product word for word, and keeps the fastest.
// The reference has no counterpart: its engines pick one radix-2 schedule per length
// (int_ntt.cu:57-104) or one cuFFT plan (ntt_engine.cu:76-107).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pi_b200.h"
#include "ntt_engine.cuh"

namespace pg {

DeviceTables& ctx_tables_mut(pg_ctx* c);
Workspace& ctx_workspace(pg_ctx* c);
cudaStream_t ctx_stream(pg_ctx* c);
std::mutex& ctx_mutex(pg_ctx* c);
void ctx_set_error(pg_ctx* c, const std::string& msg);
int ctx_device(pg_ctx* c);

namespace {

// Every valid split of 2^logL points.
std::vector<Plan> candidates(int logL) {
    std::vector<Plan> out;
    if (logL <= kMaxContigLog) {
        const int n[1] = {logL};
        Plan p = plan_from(logL, 1, n);
        if (plan_valid(p)) out.push_back(p);
    }
    for (int a = 5; a <= kMaxStridedLog; ++a) {
        const int n[2] = {a, logL - a};
        Plan p = plan_from(logL, 2, n);
        if (plan_valid(p)) out.push_back(p);
        for (int b = 5; b <= kMaxStridedLog; ++b) {
            const int m[3] = {a, b, logL - a - b};
            Plan q = plan_from(logL, 3, m);
            if (plan_valid(q)) out.push_back(q);
        }
    }
    return out;
}

// Pseudo-random limbs (splitmix64 of the index) with the top limb's high bit set.
__global__ void fill_kernel(uint64_t* x, uint64_t n, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        if (i == n - 1) z |= 1ull << 63;
        x[i] = z;
    }
}

// Counts words where x and y differ.
__global__ void diff_kernel(const uint64_t* x, const uint64_t* y, uint64_t n, unsigned long long* count) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (x[i] != y[i]) atomicAdd(count, 1ull);
}

pg_status fail(pg_ctx* c, pg_status s, const std::string& msg) {
    ctx_set_error(c, msg);
    return s;
}

void set_tuned(DeviceTables& T, const Plan& p, bool wide = false) {
    int8_t(&t)[kMaxLogL + 1][4] = wide ? T.tuned_wide : T.tuned;
    t[p.logL][0] = (int8_t)p.npass;
    for (int i = 0; i < 3; ++i) t[p.logL][1 + i] = (int8_t)(i < p.npass ? p.logN[i] : 0);
}

}  // namespace
}  // namespace pg

extern "C" {

pg_status pg_tune(pg_ctx* ctx, int lo, int hi, double* best_us) {
    using namespace pg;
    if (!ctx || lo < kMinLogL || hi > kMaxLogL || lo > hi) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(ctx_mutex(ctx));
    cudaError_t e = cudaSetDevice(ctx_device(ctx));
    if (e != cudaSuccess) return fail(ctx, PG_ERR_DEVICE, cudaGetErrorString(e));
    DeviceTables& T = ctx_tables_mut(ctx);
    Workspace& W = ctx_workspace(ctx);
    cudaStream_t st = ctx_stream(ctx);
    // balanced operands of 2^(hi-2) limbs: a product of n + n limbs has logL = log2(4n)
    const uint64_t nmax = 1ull << (hi - 2);
    uint64_t *a = nullptr, *b = nullptr, *ref = nullptr, *out = nullptr;
    unsigned long long* cnt = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    pg_status status = PG_OK;
    std::string msg;
    e = pg::dev_malloc(&a, nmax * 8);
    if (e == cudaSuccess) e = pg::dev_malloc(&b, nmax * 8);
    if (e == cudaSuccess) e = pg::dev_malloc(&ref, 2 * nmax * 8);
    if (e == cudaSuccess) e = pg::dev_malloc(&out, 2 * nmax * 8);
    if (e == cudaSuccess) e = pg::dev_malloc(&cnt, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    if (e == cudaSuccess) {
        fill_kernel<<<148 * 4, 256, 0, st>>>(a, nmax, 1);
        fill_kernel<<<148 * 4, 256, 0, st>>>(b, nmax, 2);
        e = cudaGetLastError();
    }
    // Each length is tuned in both configurations, on the same balanced product of n = 2^(logL-2)
    // limbs per operand: the 32-bit one's transform has 2^logL points, the wide one's 2^(logL-1).
    std::vector<double> best_narrow(hi - lo + 1, 1e30), best_wide(hi - lo + 1, 1e30);
    for (int logL = lo; logL <= hi && e == cudaSuccess && status == PG_OK; ++logL) {
        const uint64_t n = 1ull << (logL - 2);
        for (int cfg = 0; cfg < 2 && e == cudaSuccess && status == PG_OK; ++cfg) {
            const bool wide = cfg == 1;
            const int tl = wide ? logL - 1 : logL;  // transform length of this configuration
            if (wide && (!T.wide || tl < kMinLogL || tl > kWideMaxLogL)) continue;
            int8_t(&tab)[kMaxLogL + 1][4] = wide ? T.tuned_wide : T.tuned;
            int8_t saved[4];
            std::copy(tab[tl], tab[tl] + 4, saved);
            tab[tl][0] = 0;  // reference output: the built-in split
            e = enqueue_product_config(T, W, a, n, b, n, ref, st, wide);
            double best = 1e30;
            Plan best_plan = make_plan(tl);
            for (const Plan& p : candidates(tl)) {
                if (e != cudaSuccess) break;
                set_tuned(T, p, wide);
                e = enqueue_product_config(T, W, a, n, b, n, out, st, wide);  // warm-up and check
                if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
                if (e == cudaSuccess) {
                    diff_kernel<<<148 * 4, 256, 0, st>>>(ref, out, 2 * n, cnt);
                    e = cudaGetLastError();
                }
                unsigned long long bad = 0;
                if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, cnt, sizeof(bad), cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) break;
                if (bad) {
                    status = PG_ERR_INTERNAL;
                    msg = "pg_tune: split disagrees with the built-in plan at logL " + std::to_string(tl);
                    break;
                }
                const int reps = tl >= 24 ? 3 : (tl >= 18 ? 4 : 8);
                float ms = 0;
                e = cudaEventRecord(ev0, st);
                for (int r = 0; r < reps && e == cudaSuccess; ++r)
                    e = enqueue_product_config(T, W, a, n, b, n, out, st, wide);
                if (e == cudaSuccess) e = cudaEventRecord(ev1, st);
                if (e == cudaSuccess) e = cudaEventSynchronize(ev1);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
                if (e != cudaSuccess) break;
                const double us = 1e3 * ms / reps;
                if (std::getenv("PG_TUNE_VERBOSE"))
                    std::fprintf(stderr, "[pg_tune] %s logL %d split %d %d %d (%d passes): %.1f us\n",
                                 wide ? "wide" : "32-bit", tl, p.logN[0], p.npass > 1 ? p.logN[1] : 0,
                                 p.npass > 2 ? p.logN[2] : 0, p.npass, us);
                if (us < best) {
                    best = us;
                    best_plan = p;
                }
            }
            if (e == cudaSuccess && status == PG_OK) {
                set_tuned(T, best_plan, wide);
                (wide ? best_wide : best_narrow)[logL - lo] = best;
            } else {
                std::copy(saved, saved + 4, tab[tl]);
            }
        }
        if (best_us) best_us[logL - lo] = std::min(best_narrow[logL - lo], best_wide[logL - lo]);
    }
    // The crossover: products of at least 2^(logL-1) limbs run wide from the smallest tuned length
    // from which the wide configuration is faster at every longer tuned length.
    if (e == cudaSuccess && status == PG_OK && T.wide) {
        int from = -1;
        for (int logL = hi; logL >= lo; --logL) {
            if (best_wide[logL - lo] < best_narrow[logL - lo])
                from = logL;
            else
                break;
        }
        if (from >= 0) T.wide_min_limbs = 1ull << (from - 1);
        else if (hi >= kWideMaxLogL + 1) T.wide_min_limbs = 0;
    }
    // the device error word stays as it was: every product here was checked above
    cudaStreamSynchronize(st);
    if (a) dev_free(a);
    if (b) dev_free(b);
    if (ref) dev_free(ref);
    if (out) dev_free(out);
    if (cnt) dev_free(cnt);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, e == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_DEVICE,
                    std::string("pg_tune: ") + cudaGetErrorString(e));
    }
    if (status != PG_OK) return fail(ctx, status, msg);
    return PG_OK;
}

pg_status pg_tune_save(pg_ctx* ctx, const char* path) {
    using namespace pg;
    if (!ctx || !path) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(ctx_mutex(ctx));
    const DeviceTables& T = ctx_tables_mut(ctx);
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(ctx, PG_ERR_BAD_ARG, std::string("pg_tune_save: cannot open ") + path);
    std::fprintf(f, "# pi_b200 pass splits: logL npass logN0 logN1 logN2 [64: the wide configuration's]\n");
    for (int l = 0; l <= kMaxLogL; ++l)
        if (T.tuned[l][0] > 0)
            std::fprintf(f, "%d %d %d %d %d\n", l, T.tuned[l][0], T.tuned[l][1], T.tuned[l][2], T.tuned[l][3]);
    for (int l = 0; l <= kWideMaxLogL; ++l)
        if (T.tuned_wide[l][0] > 0)
            std::fprintf(f, "%d %d %d %d %d 64\n", l, T.tuned_wide[l][0], T.tuned_wide[l][1], T.tuned_wide[l][2],
                         T.tuned_wide[l][3]);
    if (T.wide_min_limbs != (1ull << 13))
        std::fprintf(f, "wide_min_limbs %llu\n", (unsigned long long)T.wide_min_limbs);
    const bool ok = std::fclose(f) == 0;
    return ok ? PG_OK : fail(ctx, PG_ERR_BAD_ARG, "pg_tune_save: write failed");
}

pg_status pg_tune_load(pg_ctx* ctx, const char* path) {
    using namespace pg;
    if (!ctx || !path) return PG_ERR_BAD_ARG;
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(ctx, PG_ERR_BAD_ARG, std::string("pg_tune_load: cannot open ") + path);
    std::vector<std::pair<Plan, bool>> plans;
    long long wmin = -1;
    char line[256];
    int lineno = 0;
    pg_status s = PG_OK;
    while (std::fgets(line, sizeof line, f)) {
        ++lineno;
        if (line[0] == '#' || line[0] == '\n') continue;
        unsigned long long v = 0;
        if (std::sscanf(line, "wide_min_limbs %llu", &v) == 1) {
            wmin = (long long)v;
            continue;
        }
        int l, np, n0, n1, n2, w = 32;
        const int got = std::sscanf(line, "%d %d %d %d %d %d", &l, &np, &n0, &n1, &n2, &w);
        const bool wide = got == 6 && w == 64;
        if ((got != 5 && !wide) || l < kMinLogL || l > (wide ? kWideMaxLogL : kMaxLogL) || np < 1 || np > 3) {
            s = fail(ctx, PG_ERR_BAD_ARG, "pg_tune_load: bad line " + std::to_string(lineno));
            break;
        }
        const int n[3] = {n0, n1, n2};
        Plan p = plan_from(l, np, n);
        if (!plan_valid(p)) {
            s = fail(ctx, PG_ERR_BAD_ARG, "pg_tune_load: invalid split on line " + std::to_string(lineno));
            break;
        }
        plans.push_back({p, wide});
    }
    std::fclose(f);
    if (s != PG_OK) return s;
    std::lock_guard<std::mutex> lock(ctx_mutex(ctx));
    DeviceTables& T = ctx_tables_mut(ctx);
    for (const auto& p : plans) set_tuned(T, p.first, p.second);
    if (wmin >= 0) T.wide_min_limbs = (uint64_t)wmin;
    return PG_OK;
}

}  // extern "C"
