// Pass launches: the kernel instantiation for a pass (layout, sub-transform length, direction,
// source, fusion) and its launch; templated on the prime count NP so that the 32-bit configuration
// (NP = 3, ntt_engine.cu) and the wide one (NP = 5, ntt_wide.cu) compile in separate units.
#pragma once
#include <cuda_runtime.h>

#include "ntt_engine.cuh"
#include "ntt_pass.cuh"

namespace pg {

// Dynamic shared memory of a pass: the tile, plus the four-step row factors of a strided tile or
// the per-row sources of a contiguous one (RowSrc, 16 bytes a row).
template <Layout LAY, int LOGN>
constexpr size_t pass_smem() {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    return ((size_t)4 << LOGE) + (LAY == Layout::Strided ? ((size_t)8 << LOGN) : ((size_t)16 << (LOGE - LOGN)));
}

template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE, int NP>
static cudaError_t run_pass(const PassParams& prm, const TwiddleTables& tw, cudaStream_t st) {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    constexpr int NT = pass_threads(LOGE);
    uint64_t tiles;
    if constexpr (LAY == Layout::Strided) {
        tiles = (uint64_t)prm.njobs << (prm.logL - LOGE);
    } else {
        const uint64_t rows = (uint64_t)prm.njobs << (prm.logL - LOGN);
        const uint64_t per = 1ull << (LOGE - LOGN);
        tiles = (rows + per - 1) / per;
    }
    auto kern = ntt_pass_kernel<LAY, LOGN, LOGE, NT, INV, SRC, FUSE, NP>;
    constexpr size_t smem = pass_smem<LAY, LOGN>();
    dim3 grid((unsigned)tiles, NP);
    kern<<<grid, NT, smem, st>>>(prm, tw);
    return cudaGetLastError();
}

// Kernels whose tiles need more than the default 48 KB of dynamic shared memory opt in on the
// current device; done for every such kernel when a context's tables are built, so that no
// attribute is set in the middle of a stream capture.
template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE, int NP>
static cudaError_t allow_smem() {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    constexpr size_t smem = pass_smem<LAY, LOGN>();
    if constexpr (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(ntt_pass_kernel<LAY, LOGN, LOGE, pass_threads(LOGE), INV, SRC, FUSE, NP>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The first forward pass reads limbs: as 32-bit coefficients (NP = 3) or 64-bit ones (NP = 5).
template <int NP>
constexpr Source limb_source() { return NP == kWidePrimes ? Source::Limbs64 : Source::Limbs; }

template <int NP, int N>
static cudaError_t contig_pass(bool inverse, Source src, Fuse fuse, const PassParams& prm, const TwiddleTables& tw,
                               cudaStream_t st) {
    constexpr Source LS = limb_source<NP>();
    if (inverse && fuse == Fuse::Combine) {
        if constexpr (NP == kNumPrimes) return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::Combine, NP>(prm, tw, st);
        return cudaErrorInvalidValue;  // the splitting's merges run in the 32-bit configuration
    }
    if (inverse) return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::None, NP>(prm, tw, st);
    if (src == LS) {
        if (fuse == Fuse::None) return run_pass<Layout::Contig, N, false, LS, Fuse::None, NP>(prm, tw, st);
        if (fuse == Fuse::MulInverse) return run_pass<Layout::Contig, N, false, LS, Fuse::MulInverse, NP>(prm, tw, st);
        return run_pass<Layout::Contig, N, false, LS, Fuse::SqrInverse, NP>(prm, tw, st);
    }
    if (src != Source::Residues) return cudaErrorInvalidValue;
    if (fuse == Fuse::None) return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::None, NP>(prm, tw, st);
    if (fuse == Fuse::MulInverse) return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse, NP>(prm, tw, st);
    return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse, NP>(prm, tw, st);
}

template <int NP, int N>
static cudaError_t strided_pass(bool inverse, Source src, const PassParams& prm, const TwiddleTables& tw,
                                cudaStream_t st) {
    constexpr Source LS = limb_source<NP>();
    if (inverse) return run_pass<Layout::Strided, N, true, Source::Residues, Fuse::None, NP>(prm, tw, st);
    if (src == LS) return run_pass<Layout::Strided, N, false, LS, Fuse::None, NP>(prm, tw, st);
    if (src != Source::Residues) return cudaErrorInvalidValue;
    return run_pass<Layout::Strided, N, false, Source::Residues, Fuse::None, NP>(prm, tw, st);
}

template <int NP, int N>
static cudaError_t allow_smem_contig() {
    constexpr Source LS = limb_source<NP>();
    cudaError_t e = cudaSuccess;
    if constexpr (NP == kNumPrimes) e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::Combine, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::MulInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::SqrInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse, NP>();
    return e;
}

template <int NP, int N>
static cudaError_t allow_smem_strided() {
    constexpr Source LS = limb_source<NP>();
    cudaError_t e = allow_smem<Layout::Strided, N, true, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, LS, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, Source::Residues, Fuse::None, NP>();
    return e;
}

template <int NP>
static cudaError_t allow_big_tiles_np() {
    cudaError_t e = allow_smem_contig<NP, 14>();
    if (e == cudaSuccess) e = allow_smem_strided<NP, 11>();
    if (e == cudaSuccess) e = allow_smem_strided<NP, 12>();
    return e;
}

// Launch pass `pass` of `plan` in the configuration with NP primes.
template <int NP>
static cudaError_t launch_pass_np(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm0,
                                  const TwiddleTables& tw, cudaStream_t st) {
    const int logN = plan.logN[pass];
    const bool contig = (pass == plan.npass - 1);
    PassParams prm = prm0;
    if (!contig) {
        prm.rowB = row_table(tw, plan.logN[pass] + plan.logS[pass], logN, inverse ? 1 : 0);
        if (!prm.rowB) return cudaErrorInvalidValue;  // no four-step table for this split
    }
    if (contig) {
        if (inverse && (src != Source::Residues || (fuse != Fuse::None && fuse != Fuse::Combine)))
            return cudaErrorInvalidValue;
        switch (logN) {
            case 6: return contig_pass<NP, 6>(inverse, src, fuse, prm, tw, st);
            case 7: return contig_pass<NP, 7>(inverse, src, fuse, prm, tw, st);
            case 8: return contig_pass<NP, 8>(inverse, src, fuse, prm, tw, st);
            case 9: return contig_pass<NP, 9>(inverse, src, fuse, prm, tw, st);
            case 10: return contig_pass<NP, 10>(inverse, src, fuse, prm, tw, st);
            case 11: return contig_pass<NP, 11>(inverse, src, fuse, prm, tw, st);
            case 12: return contig_pass<NP, 12>(inverse, src, fuse, prm, tw, st);
            case 13: return contig_pass<NP, 13>(inverse, src, fuse, prm, tw, st);
            case 14: return contig_pass<NP, 14>(inverse, src, fuse, prm, tw, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (logN) {
        case 5: return strided_pass<NP, 5>(inverse, src, prm, tw, st);
        case 6: return strided_pass<NP, 6>(inverse, src, prm, tw, st);
        case 7: return strided_pass<NP, 7>(inverse, src, prm, tw, st);
        case 8: return strided_pass<NP, 8>(inverse, src, prm, tw, st);
        case 9: return strided_pass<NP, 9>(inverse, src, prm, tw, st);
        case 10: return strided_pass<NP, 10>(inverse, src, prm, tw, st);
        case 11: return strided_pass<NP, 11>(inverse, src, prm, tw, st);
        case 12: return strided_pass<NP, 12>(inverse, src, prm, tw, st);
        default: return cudaErrorInvalidValue;
    }
}

// Defined in ntt_wide.cu (the NP = 5 instantiations).
cudaError_t launch_pass_wide(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                             const TwiddleTables& tw, cudaStream_t st);
cudaError_t allow_big_tiles_wide();

}  // namespace pg
