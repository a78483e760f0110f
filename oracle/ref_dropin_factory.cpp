// ORACLE -- test infrastructure only (see ref_dropin.cpp). Makes the library's pi::B200Multiplier
// for the reference's BinarySplitting / PiEngine; this translation unit sees the library's
// pi::Multiplier declaration, which is the reference's (src/arithmetic/multiplier.h:16-41)
// member for member, so the object is used through the reference's declaration unchanged.
#include <cstddef>

#include "b200_multiplier.h"

namespace refb {
pi::Multiplier* make_b200_multiplier(size_t threshold, int device) { return new pi::B200Multiplier(threshold, device); }
unsigned long long b200_gpu_calls(pi::Multiplier* m) {
    auto* b = dynamic_cast<pi::B200Multiplier*>(m);
    return b ? (unsigned long long)b->stats().gpu_calls.load() : 0ull;
}
}  // namespace refb
