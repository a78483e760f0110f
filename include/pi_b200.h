/*
 * pi_b200 -- exact big-integer multiplication on one NVIDIA B200 (sm_100a).
 *
 * C ABI of libpigpu.so, the drop-in boundary for the multiply hot path of
 * f97johan/pi-compute. The reference's boundary is the C++ strategy interface
 *
 *     class pi::Multiplier {                                   (src/arithmetic/multiplier.h:16-39)
 *       virtual void multiply(mpz_t result, const mpz_t a, const mpz_t b) = 0;    (:26)
 *       virtual void square(mpz_t result, const mpz_t a) { multiply(result,a,a); } (:36-38)
 *     };
 *
 * whose CUDA implementations are GpuNttMultiplier (src/arithmetic/gpu_ntt_multiplier.cpp:144-214)
 * and IntNttMultiplier (src/arithmetic/int_ntt_multiplier.cpp:115-163), each a GMP <-> device
 * bridge over an engine (src/gpu/ntt_engine.cu:109-158, src/gpu/int_ntt.cu:301-380).
 * This header replaces those engines' entry points with plain pointers and sizes: magnitudes
 * are little-endian arrays of 64-bit limbs, exactly the layout of mpz_limbs_read(); signs,
 * zero and mpz_t reallocation stay in the C++ adaptor (B200Multiplier, host/b200_multiplier.h).
 *
 * Errors are integer status codes (the reference throws std::runtime_error from CUDA_CHECK,
 * src/gpu/int_ntt.cu:20-26). There is no CPU fallback: a product outside the proven exact
 * range returns PG_ERR_TOO_LARGE instead of silently computing on the host (the reference's
 * IntNttMultiplier falls back to mpz_mul, src/arithmetic/int_ntt_multiplier.cpp:146-151).
 *
 * Thread safety: every call on one context is serialised by an internal lock (the reference
 * locks one mutex per GPU, src/arithmetic/gpu_ntt_multiplier.cpp:179-188).
 */
#ifndef PI_B200_H
#define PI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int pg_status;
#define PG_OK 0
#define PG_ERR_OOM 1          /* device allocation failed */
#define PG_ERR_TOO_LARGE 2    /* product outside the proven exact range of the transform */
#define PG_ERR_BAD_ARG 3      /* null pointer, output too small, bad device index */
#define PG_ERR_DEVICE 4       /* CUDA runtime error (message in pg_last_error) */
#define PG_ERR_TIMEOUT 5      /* a bounded device-side wait ran out (carry look-back) */
#define PG_ERR_INTERNAL 6     /* device consistency check failed (carry out of the top word) */
#define PG_ERR_IO 7           /* checkpoint file missing, unreadable, short, or not writable */

typedef struct pg_ctx pg_ctx;

/* Library version, (major << 16) | (minor << 8) | patch. */
int pg_version(void);

/* Create a context on CUDA device `device`: builds the twiddle tables and a stream.
 * Replaces the engine constructors (ntt_engine.cu NttEngine::NttEngine, int_ntt.cu
 * IntNttEngine::IntNttEngine, int_ntt.h:49). */
pg_status pg_create(int device, pg_ctx** out);
void pg_destroy(pg_ctx* ctx);

/* Message for the last non-OK status on this context ("" if none). */
const char* pg_last_error(const pg_ctx* ctx);

/* Largest na + nb (in 64-bit limbs) that pg_mul accepts: transforms of up to 2^26
 * points of 32-bit coefficients over three 31-bit primes. */
size_t pg_mul_max_limbs(void);

/* out = a * b for magnitudes in HOST memory (little-endian 64-bit limbs).
 * out must have room for na + nb limbs (out_cap >= na + nb); *out_len receives the
 * product's length without leading zero limbs (0 if either operand is empty).
 * out may alias a or b: both are read completely before out is written.
 * Replaces GpuNttMultiplier::multiply / IntNttMultiplier::multiply
 * (gpu_ntt_multiplier.cpp:144-210, int_ntt_multiplier.cpp:115-159). */
pg_status pg_mul(pg_ctx* ctx, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                 size_t out_cap, size_t* out_len);

/* out = a * a (two forward transforms fewer than pg_mul). Replaces the square()
 * overrides, which call multiply(a, a) (gpu_ntt_multiplier.cpp:212-214, int_ntt_multiplier.cpp:161-163). */
pg_status pg_sqr(pg_ctx* ctx, const uint64_t* a, size_t na, uint64_t* out, size_t out_cap, size_t* out_len);

/* Device-resident forms: d_a, d_b, d_out are device addresses (16-byte aligned) on the
 * context's device; d_out receives exactly na + nb limbs (leading zeros kept). The work is
 * queued on the context's stream and the call returns without waiting; pg_sync waits and
 * reports device-side errors. d_out must not overlap d_a or d_b.
 * Replaces the device part of IntNttEngine::multiply (int_ntt.cu:301-380), which round-trips
 * every operand through host memory. */
pg_status pg_mul_device(pg_ctx* ctx, const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                        uint64_t* d_out);
pg_status pg_sqr_device(pg_ctx* ctx, const uint64_t* d_a, size_t na, uint64_t* d_out);
pg_status pg_sync(pg_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own work after it. */
void* pg_stream(pg_ctx* ctx);

/* Number of kernels this context has launched so far (diagnostics and benchmarks; the
 * reference keeps per-multiplier call counters, gpu_ntt_multiplier.h:83-90). */
uint64_t pg_launch_count(const pg_ctx* ctx);

/* Level-batched, device-resident Chudnovsky binary splitting of the term range [a, b):
 * P(a,b), Q(a,b), R(a,b) as magnitudes in HOST buffers of `cap` limbs each (P may be NULL
 * when it is not needed, as for the root of a pi computation: then P is not computed at all,
 * nor the P of the rightmost node of any depth, and len[0] = sign[0] = 0), their lengths in
 * len[3] and signs in sign[3]. Same series, leaves and split point as the reference's BinarySplitting
 * (src/engine/binary_splitting.cpp:137-159, 161-293, 295-348), so the values are identical;
 * every depth of the tree runs as a few launches over all of its merges, with operands kept
 * in device memory from the leaves to the root. Replaces BinarySplitting::compute
 * (binary_splitting.cpp:605-644) with its per-merge Multiplier calls. */
pg_status pg_bs(pg_ctx* ctx, unsigned long a, unsigned long b, uint64_t* P, uint64_t* Q, uint64_t* R, size_t cap,
                size_t* len, int* sign);

/* ---- Library-owned device buffers (device-resident operands between calls). A buffer holds
 * `cap` limbs on the context's device and a length; upload sets the length and zero-fills
 * the rest, download copies `len` limbs and reports the length without leading zeros.
 * The reference keeps every operand in host mpz_t and copies it per call
 * (gpu_ntt_multiplier.cpp:74-142, int_ntt.cu:322-340); these handles let callers keep
 * operands in HBM across products instead. */
typedef struct pg_buf pg_buf;
pg_status pg_buf_alloc(pg_ctx* ctx, size_t cap, pg_buf** out);
void pg_buf_free(pg_ctx* ctx, pg_buf* buf);
pg_status pg_buf_upload(pg_ctx* ctx, pg_buf* buf, const uint64_t* src, size_t n);
pg_status pg_buf_download(pg_ctx* ctx, const pg_buf* buf, uint64_t* dst, size_t dst_cap, size_t* len);
uint64_t* pg_buf_device(pg_buf* buf);       /* device address (16-byte aligned) */
size_t pg_buf_len(const pg_buf* buf);
size_t pg_buf_capacity(const pg_buf* buf);
pg_status pg_buf_set_len(pg_buf* buf, size_t n);

/* ---- Batched products. Job i computes, on device-resident magnitudes (16-byte aligned),
 *     acc == 0:  out = a * b                     (b == NULL: a * a)
 *     acc == +1: out = a * b + c * d             (d == NULL: c * c)
 *     acc == -1: out = a * b - c * d             (the result must not be negative)
 * and writes exactly max(na + nb, nc + nd) (+1 when acc == +1) limbs to out (out_cap at
 * least that). The accumulating forms combine the two products in the transform domain, as
 * the binary-splitting merge R = Qr*Rl + Pl*Rr needs (binary_splitting.cpp:184-200, where the
 * reference issues two Multiplier calls and an mpz_add); their exactness bound asks
 * min(na, nb) + min(nc, nd) <= 2^24 (PG_ERR_TOO_LARGE otherwise).
 * Jobs are grouped by transform length and every group runs as one launch per pass over all of
 * its jobs. Outputs must not overlap each other or any operand. The call returns when every job
 * is complete; a negative acc == -1 result returns PG_ERR_BAD_ARG. Replaces the per-call
 * Multiplier::multiply sequence of a tree level (binary_splitting.cpp:183-238). */
typedef struct pg_job {
    const uint64_t* a;
    size_t na;
    const uint64_t* b;
    size_t nb;
    const uint64_t* c;
    size_t nc;
    const uint64_t* d;
    size_t nd;
    int acc;
    uint64_t* out;
    size_t out_cap;
} pg_job;
pg_status pg_mul_batch(pg_ctx* ctx, const pg_job* jobs, size_t njobs);

/* ---- A tree level as a CUDA graph. pg_graph_capture_level validates `jobs` like pg_mul_batch,
 * sizes buffers of its own for them, uploads their tables and captures the level's launches (one
 * per pass per transform-length group, the pointwise steps, one CRT + carry per group) into a CUDA
 * graph on the context's stream; nothing runs yet. pg_graph_launch replays it: the same products
 * over whatever the operand buffers hold at that moment, written to the same outputs, and returns
 * when they are complete (errors as pg_mul_batch). The pointers in `jobs` must stay valid while the
 * graph lives; the graph's buffers are its own, so products and batches on the same context may run
 * between replays. pg_graph_destroy waits for the context's stream and frees the graph.
 * The reference's level is a sequence of Multiplier calls issued from threads
 * (src/engine/binary_splitting.cpp:183-238); a caller that splits level by level captures each
 * level shape once and replays it with one launch call. */
typedef struct pg_graph pg_graph;
pg_status pg_graph_capture_level(pg_ctx* ctx, const pg_job* jobs, size_t njobs, pg_graph** out);
pg_status pg_graph_launch(pg_graph* g);
void pg_graph_destroy(pg_graph* g);

/* ---- Device-resident finish of a pi computation. Every operand stays in HBM; products run
 * on the transform above, additions, shifts and comparisons on carry-chain kernels.
 *
 * pg_recip_floor: z = floor(2^(2k) / r), k = bit length of r > 0 (Newton iteration at doubling
 *   precision with an exact final correction). The reference divides with mpf_div
 *   (src/arithmetic/newton_divider.cpp:13-25); this is its quotient core, exact to the last
 *   unit. z needs k/64 + 2 limbs.
 * pg_sqrt_scaled: out = floor(sqrt(a) * 2^s) for a >= 1 (Newton on the inverse
 *   square root, exact correction). Replaces mpf_sqrt (newton_divider.cpp:27-74).
 * pg_to_decimal: the ndigits decimal digits of x (x < 10^ndigits, leading zeros written) into
 *   out[0 .. ndigits), no terminator. Divide-and-conquer by 10^(2^j) batched per level on the
 *   device. Replaces BaseConverter / mpz_get_str (src/io/base_converter.cpp:48-147, 201-246).
 * pg_pi_finish: "3." followed by `digits` digits of pi (digits + 2 characters, no terminator)
 *   from the series root Q, R = Q(0, N), R(0, N) (host magnitudes, both positive).
 *   Replaces PiEngine::compute's final section (src/engine/pi_engine.cpp:432-491).
 * pg_pi: the whole computation on one device: level-batched binary splitting over the
 *   reference's term count, then pg_pi_finish's steps, all in HBM. out receives digits + 2
 *   characters; seconds (if not NULL, 4 entries) receives splitting, final formula,
 *   conversion and total wall time.
 * pg_pi, pg_pi_finish and pg_pi_checkpointed free no device buffer while they run (cudaFree
 *   waits for the whole device): the buffers they outgrow are freed by the next allocation or
 *   free the library makes after they return (at the latest by pg_destroy), or at once when an
 *   allocation fails for want of memory or when more than a quarter of the device's memory
 *   waits to be freed. */
pg_status pg_recip_floor(pg_ctx* ctx, const uint64_t* r, size_t nr, uint64_t* z, size_t zcap, size_t* zlen);
/* out = a * b mod (2^(32 L) - 1), L = 2^logL (6 <= logL <= 26), for na, nb <= L/2 limbs: one
 * L-point transform product (the product wraps around) and a fold of its top words. The result
 * lies in [0, 2^(32 L) - 1]; the modulus itself may stand for 0. The Newton steps of
 * pg_recip_floor / pg_sqrt_scaled take their residues this way when that halves the transform. */
pg_status pg_mul_wrap(pg_ctx* ctx, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, int logL, uint64_t* out,
                      size_t cap, size_t* len);
pg_status pg_sqrt_scaled(pg_ctx* ctx, uint64_t a, size_t s, uint64_t* out, size_t cap, size_t* len);
pg_status pg_to_decimal(pg_ctx* ctx, const uint64_t* x, size_t nx, size_t ndigits, char* out);
pg_status pg_pi_finish(pg_ctx* ctx, const uint64_t* q, size_t nq, const uint64_t* r, size_t nr, size_t digits,
                       char* out);
pg_status pg_pi(pg_ctx* ctx, size_t digits, char* out, double* seconds);

/* ---- Checkpoints, in the reference's file formats, so that files move between the two
 * programs in both directions:
 *   <dir>/bs_<a>_<b>.ckpt    P, Q, R of the splitting node [a, b): for each, int sign (-1, 0, 1),
 *                            size_t byte count, the bytes of |x| least significant first
 *                            (src/engine/binary_splitting.cpp:44-90: mpz_export order -1, size 1)
 *   <dir>/pi_int_<D>.ckpt    floor(pi 10^D): size_t byte count, then the bytes
 *                            (src/engine/pi_engine.cpp:263-284, 417-430)
 * int and size_t in the machine's own 4- and 8-byte little-endian form, as the reference writes.
 *
 * pg_ckpt_write_bs / pg_ckpt_read_bs, pg_ckpt_write_pi_int / pg_ckpt_read_pi_int: the formats on
 *   host limb arrays (no context, no device work). Reading with x == NULL (read_bs: all three
 *   NULL) only reports the capacities in limbs that the values need (and the signs); otherwise
 *   every non-NULL x[k] must hold `cap` limbs and receives the value, n[k] its length without
 *   leading zeros. PG_ERR_IO for a missing, short or unwritable file, PG_ERR_BAD_ARG for a
 *   capacity that is too small (n[k] then holds the capacity needed).
 * pg_bs_checkpointed: pg_bs resumed from and saved to `dir` like the reference's
 *   BinarySplitting::compute(a, b) with checkpointing on (binary_splitting.cpp:104-135, 295-302,
 *   350-360, 605-644): a node of the splitting tree whose file loads is taken from it; halves
 *   holding files below them are merged on the device; every other subtree is one level-batched
 *   device splitting; at the end bs_<a>_<b>.ckpt is written (unless it was loaded) and the
 *   files of its two children removed. P may be NULL. Results as pg_bs.
 * pg_pi_checkpointed: pg_pi with the reference's --checkpoint DIR behaviour: the root splitting
 *   as above, then pi_int_<digits>.ckpt loaded when present (no final formula) or written after
 *   the final formula, then the conversion. The directory is created when missing; files that
 *   cannot be written are skipped (the report says which were saved). */
typedef struct pg_ckpt_report {
    int root_loaded;           /* bs_0_<N>.ckpt (bs_<a>_<b>.ckpt) was read */
    int root_saved;            /* ... was written */
    int pi_int_loaded;         /* pi_int_<digits>.ckpt was read: no final formula */
    int pi_int_saved;          /* ... was written */
    size_t nodes_loaded;       /* splitting nodes read from files, the root included */
    size_t subtrees_computed;  /* level-batched device splittings of ranges with no file below */
    size_t merges;             /* device merges above loaded or computed nodes */
} pg_ckpt_report;

pg_status pg_ckpt_write_bs(const char* path, const uint64_t* const x[3], const size_t n[3], const int sign[3]);
pg_status pg_ckpt_read_bs(const char* path, uint64_t* const x[3], size_t cap, size_t n[3], int sign[3]);
pg_status pg_ckpt_write_pi_int(const char* path, const uint64_t* x, size_t n);
pg_status pg_ckpt_read_pi_int(const char* path, uint64_t* x, size_t cap, size_t* n);
pg_status pg_bs_checkpointed(pg_ctx* ctx, unsigned long a, unsigned long b, const char* dir, uint64_t* P, uint64_t* Q,
                             uint64_t* R, size_t cap, size_t* len, int* sign, pg_ckpt_report* report);
pg_status pg_pi_checkpointed(pg_ctx* ctx, size_t digits, const char* dir, char* out, double* seconds,
                             pg_ckpt_report* report);

/* ---- Autotuner of the transform's pass split. pg_tune times, for every transform length 2^l
 * with lo <= l <= hi (6 <= lo <= hi <= 26), each valid split into one to three passes on a
 * balanced product of that length, checks that it reproduces the built-in split's product
 * word for word, and makes the fastest the context's choice; best_us (if not NULL, hi-lo+1
 * entries) receives the winning times in microseconds. pg_tune_save writes the context's
 * choices as text ("logL npass logN0 logN1 logN2" per line), pg_tune_load reads such a file
 * (every split is validated). No counterpart in the reference, whose engines use one fixed
 * schedule per length (int_ntt.cu:57-104, ntt_engine.cu:76-107). */
pg_status pg_tune(pg_ctx* ctx, int lo, int hi, double* best_us);
pg_status pg_tune_save(pg_ctx* ctx, const char* path);
pg_status pg_tune_load(pg_ctx* ctx, const char* path);

/* d_out = d_a * d_b without allocating any device memory. This entry point has no
 * counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc, for example code running while another
 * framework owns the device allocator, or a plugin callback where allocating (and the device
 * synchronisation an allocation can imply) is not allowed. It needs no pg_ctx: the scratch
 * residues and the twiddle tables live in fixed-size device arrays inside libpigpu.so
 * (about 2.8 MB, held on every GPU that loads the library until the process exits).
 *
 * Limit: na + nb <= 16384 limbs; larger products return PG_ERR_TOO_LARGE without touching
 * any memory. Pointers are device addresses on the CURRENT device, 16-byte aligned; d_out
 * receives exactly na + nb limbs and must not overlap d_a or d_b (d_a == d_b is allowed).
 * `stream` is a cudaStream_t (NULL = the legacy default stream). Every call synchronises that
 * stream: it returns after the product is complete and reports device-side errors like pg_sync.
 *
 * The first call on a device sets that device up (looks up the arrays and fills the tables,
 * waiting for it); make it before any stream capture. All calls share the same arrays, so
 * calls whose GPU work overlaps (from several host threads or streams) race: serialise them. */
pg_status pg_mul_noalloc(const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb, uint64_t* d_out,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PI_B200_H */
