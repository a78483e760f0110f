// Checkpoint files on host limb arrays: pg_ckpt_write_bs / pg_ckpt_read_bs (the reference's
// save_bs_result / load_bs_result, src/engine/binary_splitting.cpp:48-90) and
// pg_ckpt_write_pi_int / pg_ckpt_read_pi_int (pi_engine.cpp:263-284, 417-430). Format in
// ckpt_io.h. No device work: these run on machines without a GPU.
#include <cstring>

#include "../../include/pi_b200.h"
#include "ckpt_io.h"

namespace {

using pg::ckpt::File;

size_t norm(const uint64_t* x, size_t n) {
    if (!x) return 0;
    while (n && x[n - 1] == 0) --n;
    return n;
}

// Reads one integer into x (cap limbs), or only its capacity when x is NULL.
pg_status read_one(File& f, bool with_sign, uint64_t* x, size_t cap, size_t& n, int& sign) {
    size_t count = 0;
    if (!pg::ckpt::get_header(f, with_sign, sign, count)) return PG_ERR_IO;
    const size_t need = (count + 7) / 8;
    if (!x) {
        n = need;
        sign = need ? (sign < 0 ? -1 : 1) : 0;
        return std::fseek(f.f, (long)count, SEEK_CUR) == 0 ? PG_OK : PG_ERR_IO;
    }
    if (need > cap) {  // step over the bytes so that the next value can still be sized
        n = need;
        return std::fseek(f.f, (long)count, SEEK_CUR) == 0 ? PG_ERR_BAD_ARG : PG_ERR_IO;
    }
    if (!pg::ckpt::get_limbs(f, x, count, n)) return PG_ERR_IO;
    sign = n ? (sign < 0 ? -1 : 1) : 0;
    return PG_OK;
}

}  // namespace

extern "C" {

pg_status pg_ckpt_write_bs(const char* path, const uint64_t* const x[3], const size_t n[3], const int sign[3]) {
    if (!path || !x || !n || !sign) return PG_ERR_BAD_ARG;
    for (int k = 0; k < 3; ++k)
        if (n[k] && !x[k]) return PG_ERR_BAD_ARG;
    File f(path, "wb");
    if (!f) return PG_ERR_IO;
    for (int k = 0; k < 3; ++k) {
        const size_t m = norm(x[k], n[k]);
        const int sg = m ? (sign[k] < 0 ? -1 : 1) : 0;
        if (!pg::ckpt::put_header(f, true, sg, pg::ckpt::byte_count(m, m ? x[k][m - 1] : 0)) ||
            !pg::ckpt::put_limbs(f, x[k], m))
            return PG_ERR_IO;
    }
    return f.close() ? PG_OK : PG_ERR_IO;
}

pg_status pg_ckpt_read_bs(const char* path, uint64_t* const x[3], size_t cap, size_t n[3], int sign[3]) {
    if (!path || !n || !sign) return PG_ERR_BAD_ARG;
    const bool query = !x || (!x[0] && !x[1] && !x[2]);
    File f(path, "rb");
    if (!f) return PG_ERR_IO;
    pg_status worst = PG_OK;
    for (int k = 0; k < 3; ++k) {
        uint64_t* dst = query ? nullptr : x[k];
        if (!query && !dst) {  // skip this value: read its header and step over its bytes
            size_t ignore = 0;
            int s2 = 0;
            const pg_status s = read_one(f, true, nullptr, 0, ignore, s2);
            if (s != PG_OK) return s;
            n[k] = 0;
            sign[k] = 0;
            continue;
        }
        const pg_status s = read_one(f, true, dst, cap, n[k], sign[k]);
        if (s == PG_ERR_IO) return s;
        if (s != PG_OK) worst = s;  // too small: keep going so every n[k] reports its capacity
    }
    return worst;
}

pg_status pg_ckpt_write_pi_int(const char* path, const uint64_t* x, size_t n) {
    if (!path || (n && !x)) return PG_ERR_BAD_ARG;
    File f(path, "wb");
    if (!f) return PG_ERR_IO;
    const size_t m = norm(x, n);
    if (!pg::ckpt::put_header(f, false, 0, pg::ckpt::byte_count(m, m ? x[m - 1] : 0)) || !pg::ckpt::put_limbs(f, x, m))
        return PG_ERR_IO;
    return f.close() ? PG_OK : PG_ERR_IO;
}

pg_status pg_ckpt_read_pi_int(const char* path, uint64_t* x, size_t cap, size_t* n) {
    if (!path || !n) return PG_ERR_BAD_ARG;
    File f(path, "rb");
    if (!f) return PG_ERR_IO;
    int sign = 1;
    return read_one(f, false, x, cap, *n, sign);
}

}  // extern "C"
