// Instantiations of the pass kernels for the wide configuration (64-bit coefficients over five
// primes, modarith.cuh), compiled apart from the 32-bit ones in ntt_engine.cu.
#include "pass_launch.cuh"

namespace pg {

cudaError_t launch_pass_wide(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                             const TwiddleTables& tw, cudaStream_t st) {
    return launch_pass_np<kWidePrimes>(plan, pass, inverse, src, fuse, prm, tw, st);
}

cudaError_t allow_big_tiles_wide() { return allow_big_tiles_np<kWidePrimes>(); }

}  // namespace pg
