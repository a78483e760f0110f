// C ABI of libpigpu.so (declarations and reference citations in include/pi_b200.h).
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pi_b200.h"
#include "ntt_engine.cuh"

namespace pg {
bool trace_on();
struct DeviceBS;
DeviceBS* bs_state_new();
void bs_state_delete(DeviceBS*);
struct BatchWork;
BatchWork* batch_state_new();
void batch_state_delete(BatchWork*);
struct FinishState;
FinishState* finish_state_new();
void finish_state_delete(FinishState*);
}  // namespace pg

struct pg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    pg::DeviceTables tables;
    pg::Workspace ws;
    std::string last_error;
    uint64_t launches = 0;
    pg::DeviceBS* bs = nullptr;  // binary-splitting buffers, kept for the next pg_bs call
    pg::BatchWork* batch = nullptr;  // pg_mul_batch buffers, kept for the next batch
    pg::FinishState* finish = nullptr;  // device finish pool, kept for the next pi computation
};

namespace {

pg_status fail(pg_ctx* c, pg_status s, const std::string& msg) {
    if (c) c->last_error = msg;
    return s;
}

pg_status cuda_fail(pg_ctx* c, cudaError_t e, const char* where) {
    cudaGetLastError();  // clear a sticky launch error so the context stays usable
    if (e == cudaErrorMemoryAllocation) return fail(c, PG_ERR_OOM, std::string(where) + ": out of device memory");
    return fail(c, PG_ERR_DEVICE, std::string(where) + ": " + cudaGetErrorString(e));
}

// memcpy split across host threads for large buffers (pinned staging of big operands).
void copy_parallel(void* dst, const void* src, size_t bytes) {
    constexpr size_t kChunk = 8u << 20;
    if (bytes < 2 * kChunk) {
        std::memcpy(dst, src, bytes);
        return;
    }
    unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    nt = (unsigned)std::min<size_t>(nt, bytes / kChunk);
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (unsigned i = 1; i < nt; ++i) {
        const size_t o = i * per;
        if (o >= bytes) break;
        th.emplace_back([=] { std::memcpy((char*)dst + o, (const char*)src + o, std::min(per, bytes - o)); });
    }
    std::memcpy(dst, src, std::min(per, bytes));
    for (auto& t : th) t.join();
}

size_t trimmed(const uint64_t* x, size_t n) {
    while (n > 0 && x[n - 1] == 0) --n;
    return n;
}

// Read and clear the device error word; map it to a status.
pg_status check_device_error(pg_ctx* c) {
    uint32_t err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, c->ws.sync, 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "pg_sync");
    if (err != 0) {
        cudaMemsetAsync(c->ws.sync, 0, 4, c->stream);
        cudaStreamSynchronize(c->stream);
        if (err == 1) return fail(c, PG_ERR_TIMEOUT, "carry look-back wait ran out of iterations");
        if (err & 4) return fail(c, PG_ERR_TIMEOUT, "tile load wait ran out of iterations");
        if (err & 8) return fail(c, PG_ERR_TIMEOUT, "sum look-back wait ran out of iterations");
        return fail(c, PG_ERR_INTERNAL, "carry out of the most significant word");
    }
    return PG_OK;
}

pg_status host_product(pg_ctx* c, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, bool square,
                       uint64_t* out, size_t out_cap, size_t* out_len) {
    if (!c || !out_len || (na && !a) || (!square && nb && !b)) return fail(c, PG_ERR_BAD_ARG, "null argument");
    if (square) nb = na, b = a;
    // Reject by buffer length before reading the operands (each length on its own: no wrap-around).
    if (na > pg_mul_max_limbs() || nb > pg_mul_max_limbs() - na) return fail(c, PG_ERR_TOO_LARGE, "product exceeds the transform range");
    na = trimmed(a, na);
    nb = trimmed(b, nb);
    if (na == 0 || nb == 0) {
        *out_len = 0;
        return PG_OK;
    }
    if (!out || out_cap < na + nb) return fail(c, PG_ERR_BAD_ARG, "output buffer smaller than na + nb limbs");
    std::lock_guard<std::mutex> lock(c->mu);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    e = c->ws.ensure_limbs(na + nb);
    if (e != cudaSuccess) return cuda_fail(c, e, "workspace");
    // Stage through pinned memory so the copies run at full PCIe/C2C speed and stay async.
    uint64_t* pin = c->ws.pinned;
    copy_parallel(pin, a, na * 8);
    e = cudaMemcpyAsync(c->ws.in_a, pin, na * 8, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && !square) {
        copy_parallel(pin + c->ws.limb_cap, b, nb * 8);
        e = cudaMemcpyAsync(c->ws.in_b, pin + c->ws.limb_cap, nb * 8, cudaMemcpyHostToDevice, c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "host to device copy");
    e = pg::enqueue_product(c->tables, c->ws, c->ws.in_a, na, square ? nullptr : c->ws.in_b, nb, c->ws.outl,
                            c->stream, &c->launches);
    if (e != cudaSuccess) return cuda_fail(c, e, "product launch");
    uint64_t* pout = pin + 2 * c->ws.limb_cap;
    e = cudaMemcpyAsync(pout, c->ws.outl, (na + nb) * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "device to host copy");
    pg_status s = check_device_error(c);
    if (s != PG_OK) return s;
    copy_parallel(out, pout, (na + nb) * 8);
    *out_len = trimmed(out, na + nb);
    return PG_OK;
}

}  // namespace

// Accessors used by the binary-splitting module (bs_device.cu).
namespace pg {
const DeviceTables& ctx_tables(pg_ctx* c) { return c->tables; }
DeviceTables& ctx_tables_mut(pg_ctx* c) { return c->tables; }
Workspace& ctx_workspace(pg_ctx* c) { return c->ws; }
cudaStream_t ctx_stream(pg_ctx* c) { return c->stream; }
std::mutex& ctx_mutex(pg_ctx* c) { return c->mu; }
uint64_t* ctx_launches(pg_ctx* c) { return &c->launches; }
void ctx_set_error(pg_ctx* c, const std::string& msg) { c->last_error = msg; }
int ctx_device(pg_ctx* c) { return c->device; }
DeviceBS* ctx_bs(pg_ctx* c) {
    if (!c->bs) c->bs = bs_state_new();
    return c->bs;
}
BatchWork* ctx_batch(pg_ctx* c) {
    if (!c->batch) c->batch = batch_state_new();
    return c->batch;
}
FinishState* ctx_finish(pg_ctx* c) {
    if (!c->finish) c->finish = finish_state_new();
    return c->finish;
}
}  // namespace pg

extern "C" {

int pg_version(void) { return (0 << 16) | (1 << 8) | 0; }

size_t pg_mul_max_limbs(void) { return (size_t)1 << (pg::kMaxLogL - 1); }

pg_status pg_create(int device, pg_ctx** out) {
    if (!out) return PG_ERR_BAD_ARG;
    *out = nullptr;
    int n = 0;
    const auto t_init = std::chrono::steady_clock::now();
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return PG_ERR_BAD_ARG;
    }
    pg_ctx* c = new (std::nothrow) pg_ctx;
    if (!c) return PG_ERR_OOM;
    c->device = device;
    const auto t0 = std::chrono::steady_clock::now();
    const double t_driver = std::chrono::duration<double, std::milli>(t0 - t_init).count();
    auto ms = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    const double t_ctx = ms(t0);
    if (e == cudaSuccess) e = c->tables.build(device);
    if (e == cudaSuccess) e = c->ws.ensure_sync(1);
    if (pg::trace_on())
        std::fprintf(stderr,
                     "[pg_create] device %d: driver and device count %.3f ms, context and stream %.3f ms, twiddle "
                     "tables %.3f ms\n",
                     device, t_driver, t_ctx, ms(t0) - t_ctx);
    if (e != cudaSuccess) {
        cudaGetLastError();
        pg_destroy(c);
        return e == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_DEVICE;
    }
    // Pass splits measured by pg_tune on this GPU model: PG_TUNE_FILE, else tune_b200.txt beside
    // the library (an empty PG_TUNE_FILE keeps the built-in splits). A missing file changes
    // nothing; an invalid one is reported in pg_last_error and ignored.
    {
        std::string path;
        if (const char* env = std::getenv("PG_TUNE_FILE")) {
            path = env;
        } else {
            Dl_info info;
            if (dladdr(reinterpret_cast<void*>(&pg_version), &info) && info.dli_fname) {
                std::string lib = info.dli_fname;
                const size_t slash = lib.rfind('/');
                path = (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/tune_b200.txt";
            }
        }
        if (!path.empty()) {
            if (FILE* f = std::fopen(path.c_str(), "r")) {
                std::fclose(f);
                if (pg_tune_load(c, path.c_str()) != PG_OK) c->last_error = "ignored " + path + ": " + c->last_error;
            }
        }
    }
    *out = c;
    return PG_OK;
}

void pg_destroy(pg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->bs) pg::bs_state_delete(c->bs);
    if (c->batch) pg::batch_state_delete(c->batch);
    if (c->finish) pg::finish_state_delete(c->finish);
    c->ws.release();
    c->tables.release();
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* pg_last_error(const pg_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

pg_status pg_mul(pg_ctx* c, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                 size_t out_cap, size_t* out_len) {
    return host_product(c, a, na, b, nb, false, out, out_cap, out_len);
}

pg_status pg_sqr(pg_ctx* c, const uint64_t* a, size_t na, uint64_t* out, size_t out_cap, size_t* out_len) {
    return host_product(c, a, na, nullptr, 0, true, out, out_cap, out_len);
}

pg_status pg_mul_device(pg_ctx* c, const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                        uint64_t* d_out) {
    if (!c || !d_out || (na && !d_a) || (nb && !d_b)) return fail(c, PG_ERR_BAD_ARG, "null argument");
    if (((uintptr_t)d_a | (uintptr_t)d_b | (uintptr_t)d_out) & 15)
        return fail(c, PG_ERR_BAD_ARG, "device pointers must be 16-byte aligned");
    if (na > pg_mul_max_limbs() || nb > pg_mul_max_limbs() - na)
        return fail(c, PG_ERR_TOO_LARGE, "product exceeds the transform range");
    std::lock_guard<std::mutex> lock(c->mu);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    if (na == 0 || nb == 0) {
        e = cudaMemsetAsync(d_out, 0, (na + nb) * 8, c->stream);
        return e == cudaSuccess ? PG_OK : cuda_fail(c, e, "memset");
    }
    e = pg::enqueue_product(c->tables, c->ws, d_a, na, d_b, nb, d_out, c->stream, &c->launches);
    return e == cudaSuccess ? PG_OK : cuda_fail(c, e, "product launch");
}

pg_status pg_sqr_device(pg_ctx* c, const uint64_t* d_a, size_t na, uint64_t* d_out) {
    if (!c || !d_out || (na && !d_a)) return fail(c, PG_ERR_BAD_ARG, "null argument");
    if (((uintptr_t)d_a | (uintptr_t)d_out) & 15) return fail(c, PG_ERR_BAD_ARG, "device pointers must be 16-byte aligned");
    if (na > pg_mul_max_limbs() / 2) return fail(c, PG_ERR_TOO_LARGE, "product exceeds the transform range");
    std::lock_guard<std::mutex> lock(c->mu);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    if (na == 0) return PG_OK;
    e = pg::enqueue_product(c->tables, c->ws, d_a, na, nullptr, na, d_out, c->stream, &c->launches);
    return e == cudaSuccess ? PG_OK : cuda_fail(c, e, "product launch");
}

pg_status pg_sync(pg_ctx* c) {
    if (!c) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    cudaSetDevice(c->device);
    return check_device_error(c);
}

void* pg_stream(pg_ctx* c) { return c ? (void*)c->stream : nullptr; }

uint64_t pg_launch_count(const pg_ctx* c) { return c ? c->launches : 0; }

}  // extern "C"
