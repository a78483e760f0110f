// Checkpoint files in the reference's formats (host-side I/O; no CUDA in this header).
//
//   splitting node  <dir>/bs_<a>_<b>.ckpt   (src/engine/binary_splitting.cpp:44-90): for P, Q
//                   and R in turn an int sign (-1, 0 or +1), a size_t byte count and that many
//                   bytes of |x|, least significant byte first (mpz_export with order -1, size 1,
//                   endian -1, no nails: no leading zero bytes; zero is sign 0, count 0)
//   pi_int          <dir>/pi_int_<digits>.ckpt   (src/engine/pi_engine.cpp:263-284, 417-430):
//                   a size_t byte count and the bytes of floor(pi 10^digits), same byte order
//
// int and size_t are written in the machine's own representation (4 and 8 bytes, little-endian
// on x86-64), as the reference does with fwrite. On a little-endian machine the bytes of a
// little-endian 64-bit limb array ARE the mpz_export byte stream, so a magnitude of n limbs
// (top limb t != 0) is its first 8 (n - 1) + bytes(t) bytes.
#pragma once

#include <sys/stat.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace pg {
namespace ckpt {

static_assert(sizeof(int) == 4 && sizeof(size_t) == 8, "checkpoint header fields are 4-byte int, 8-byte size_t");

inline std::string bs_path(const std::string& dir, unsigned long a, unsigned long b) {
    return dir + "/bs_" + std::to_string(a) + "_" + std::to_string(b) + ".ckpt";
}

inline std::string pi_int_path(const std::string& dir, size_t digits) {
    return dir + "/pi_int_" + std::to_string(digits) + ".ckpt";
}

// Significant bytes of a limb whose value is nonzero (1 .. 8).
inline size_t limb_bytes(uint64_t t) { return t ? (size_t)8 - (size_t)(__builtin_clzll(t) / 8) : 0; }

// Byte count of a magnitude of n limbs whose top limb is `top` (n == 0: zero).
inline size_t byte_count(size_t n, uint64_t top) { return n ? 8 * (n - 1) + limb_bytes(top) : 0; }

// A FILE* closed on scope exit.
struct File {
    FILE* f = nullptr;
    File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
    File(const File&) = delete;
    File& operator=(const File&) = delete;
    explicit operator bool() const { return f != nullptr; }
    bool put(const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
    bool get(void* p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }
    // bytes from the current position to the end of the file
    uint64_t remaining() {
        struct stat sb;
        if (fstat(fileno(f), &sb) != 0) return 0;
        const long pos = std::ftell(f);
        return pos < 0 || (uint64_t)pos > (uint64_t)sb.st_size ? 0 : (uint64_t)sb.st_size - (uint64_t)pos;
    }
    bool close() {
        const bool ok = std::fflush(f) == 0 && !std::ferror(f);
        const bool closed = std::fclose(f) == 0;
        f = nullptr;
        return ok && closed;
    }
};

inline bool exists(const std::string& path) {
    struct stat sb;
    return stat(path.c_str(), &sb) == 0 && S_ISREG(sb.st_mode);
}

// Header of one integer: the sign (splitting files only) and the byte count.
inline bool put_header(File& f, bool with_sign, int sign, size_t count) {
    if (with_sign && !f.put(&sign, sizeof(int))) return false;
    return f.put(&count, sizeof(size_t));
}

// Reads a header; false when the file ends early or the count exceeds what the file holds.
inline bool get_header(File& f, bool with_sign, int& sign, size_t& count) {
    sign = 1;
    if (with_sign && !f.get(&sign, sizeof(int))) return false;
    if (!f.get(&count, sizeof(size_t))) return false;
    return (uint64_t)count <= f.remaining();
}

// Writes a magnitude held in host memory (n limbs, top limb nonzero or n == 0).
inline bool put_limbs(File& f, const uint64_t* x, size_t n) {
    const size_t count = byte_count(n, n ? x[n - 1] : 0);
    return f.put(x, count);
}

// Reads `count` bytes into limbs x[0 .. ceil(count / 8)) (the last limb zero-padded) and
// returns the length without leading zero limbs.
inline bool get_limbs(File& f, uint64_t* x, size_t count, size_t& n) {
    const size_t nl = (count + 7) / 8;
    if (nl) x[nl - 1] = 0;
    if (!f.get(x, count)) return false;
    n = nl;
    while (n && x[n - 1] == 0) --n;
    return true;
}

}  // namespace ckpt
}  // namespace pg
