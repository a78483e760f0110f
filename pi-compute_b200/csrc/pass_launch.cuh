// Pass launches: the kernel instantiation for a pass (layout, sub-transform length, direction,
// source, fusion) and its launch; templated on the prime count NP so that the 32-bit configuration
// (NP = 3, ntt_engine.cu) and the wide one (NP = 5, ntt_wide.cu) compile in separate units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "ntt_engine.cuh"
#include "ntt_pass.cuh"

namespace pg {

// Dynamic shared memory of a pass: the tile, plus the four-step row factors of a strided tile or
// the per-row sources of a contiguous one (RowSrc, 16 bytes a row), plus a TMA tile's barrier.
template <Layout LAY, int LOGN, bool TMA = false>
constexpr size_t pass_smem() {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    return ((size_t)4 << LOGE) + (LAY == Layout::Strided ? ((size_t)8 << LOGN) : ((size_t)16 << (LOGE - LOGN))) +
           (TMA ? 16 : 0);
}

// Whether a strided pass of sub-transform length 2^LOGN can load its tiles by TMA: rows of at
// least 32 words (one 128-byte swizzle line).
template <int LOGN>
constexpr bool strided_tma_ok() { return tile_log(true, LOGN) - LOGN >= 5; }

// TMA tile loads are used unless PG_TMA is set to 0 (read at every launch; the cp.async copies
// remain for the passes TMA does not serve and for comparison).
inline bool tma_requested() {
    const char* e = std::getenv("PG_TMA");
    return !e || std::strtol(e, nullptr, 10) != 0;
}

// cuTensorMapEncodeTiled from the driver (through the runtime, so no driver library is linked).
using TmapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline TmapEncodeFn tmap_encoder() {
    static const TmapEncodeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (TmapEncodeFn) nullptr;
        }
        return reinterpret_cast<TmapEncodeFn>(f);
    }();
    return fn;
}

// The tensor map of a pass's residues for TMA tile loads (128-byte swizzle, 32-word lines):
//   contiguous: [job][prime][line][32 words]; boxes of 256 lines, or of E / L whole arrays when a
//               tile spans several jobs;
//   strided:    [job * NP + prime][block of N' = N S][row m < N][column chunk < S / 32][32 words];
//               boxes of (C / 32 chunks) x min(N, 256) rows.
// Job j's prime-p array must sit at data + (j NP + p) L (one job, or job_stride = NP L).
template <Layout LAY, int LOGN, int NP>
static bool make_tmap(CUtensorMap* m, const PassParams& P) {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    const TmapEncodeFn enc = tmap_encoder();
    if (!enc) return false;
    const uint64_t L = P.L;
    const uint64_t js = P.njobs == 1 ? (uint64_t)NP * L : P.job_stride;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r;
    if constexpr (LAY == Layout::Contig) {
        const cuuint64_t dims[4] = {32, L / 32, (cuuint64_t)NP, P.njobs};
        const cuuint64_t strides[3] = {128, L * 4, js * 4};
        cuuint32_t box[4] = {32, 256, 1, 1};
        if (P.logL < LOGE) {
            box[1] = (cuuint32_t)(L / 32);
            box[3] = (cuuint32_t)((1ull << LOGE) / L);
        }
        r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, P.data, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        if (js != (uint64_t)NP * L) return false;
        const uint64_t S = 1ull << P.logS, N = 1ull << LOGN, C = 1ull << (LOGE - LOGN);
        const cuuint64_t dims[5] = {32, S / 32, N, L / (N * S), (cuuint64_t)P.njobs * NP};
        const cuuint64_t strides[4] = {128, S * 4, N * S * 4, L * 4};
        const cuuint32_t box[5] = {32, (cuuint32_t)(C / 32), (cuuint32_t)(N < 256 ? N : 256), 1, 1};
        r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 5, P.data, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    return r == CUDA_SUCCESS;
}

template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE, int NP, bool TMA = false>
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
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    if constexpr (TMA) {
        if (!make_tmap<LAY, LOGN, NP>(&tmap, prm)) return cudaErrorInvalidValue;
    }
    auto kern = ntt_pass_kernel<LAY, LOGN, LOGE, NT, INV, SRC, FUSE, NP, TMA>;
    constexpr size_t smem = pass_smem<LAY, LOGN, TMA>();
    if (tiles * NP > 0x7fffffffull) return cudaErrorInvalidValue;
    kern<<<(unsigned)(tiles * NP), NT, smem, st>>>(prm, tw, tmap);
    return cudaGetLastError();
}

// Kernels whose tiles need more than the default 48 KB of dynamic shared memory opt in on the
// current device; done for every such kernel when a context's tables are built, so that no
// attribute is set in the middle of a stream capture.
template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE, int NP, bool TMA = false>
static cudaError_t allow_smem() {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    constexpr size_t smem = pass_smem<LAY, LOGN, TMA>();
    if constexpr (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(ntt_pass_kernel<LAY, LOGN, LOGE, pass_threads(LOGE), INV, SRC, FUSE, NP, TMA>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The first forward pass reads limbs: as 32-bit coefficients (NP = 3) or 64-bit ones (NP = 5).
template <int NP>
constexpr Source limb_source() { return NP == kWidePrimes ? Source::Limbs64 : Source::Limbs; }

template <int NP, int N>
static cudaError_t contig_pass(bool inverse, Source src, Fuse fuse, const PassParams& prm, const TwiddleTables& tw,
                               cudaStream_t st, bool tma) {
    constexpr Source LS = limb_source<NP>();
    if (inverse && fuse == Fuse::Combine)
        return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::Combine, NP>(prm, tw, st);
    if (tma && src == Source::Residues) {
        if (inverse) return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::None, NP, true>(prm, tw, st);
        if (fuse == Fuse::None)
            return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::None, NP, true>(prm, tw, st);
        if (fuse == Fuse::MulInverse)
            return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse, NP, true>(prm, tw, st);
        return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse, NP, true>(prm, tw, st);
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
                                cudaStream_t st, bool tma) {
    constexpr Source LS = limb_source<NP>();
    if constexpr (strided_tma_ok<N>()) {
        if (tma && src == Source::Residues) {
            if (inverse) return run_pass<Layout::Strided, N, true, Source::Residues, Fuse::None, NP, true>(prm, tw, st);
            return run_pass<Layout::Strided, N, false, Source::Residues, Fuse::None, NP, true>(prm, tw, st);
        }
    }
    if (inverse) return run_pass<Layout::Strided, N, true, Source::Residues, Fuse::None, NP>(prm, tw, st);
    if (src == LS) return run_pass<Layout::Strided, N, false, LS, Fuse::None, NP>(prm, tw, st);
    if (src != Source::Residues) return cudaErrorInvalidValue;
    return run_pass<Layout::Strided, N, false, Source::Residues, Fuse::None, NP>(prm, tw, st);
}

template <int NP, int N>
static cudaError_t allow_smem_contig() {
    constexpr Source LS = limb_source<NP>();
    cudaError_t e = cudaSuccess;
    e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::Combine, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::MulInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, LS, Fuse::SqrInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::None, NP, true>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::None, NP, true>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse, NP, true>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse, NP, true>();
    return e;
}

template <int NP, int N>
static cudaError_t allow_smem_strided() {
    constexpr Source LS = limb_source<NP>();
    cudaError_t e = allow_smem<Layout::Strided, N, true, Source::Residues, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, LS, Fuse::None, NP>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, Source::Residues, Fuse::None, NP>();
    if constexpr (strided_tma_ok<N>()) {
        if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, true, Source::Residues, Fuse::None, NP, true>();
        if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, Source::Residues, Fuse::None, NP, true>();
    }
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
    // TMA tiles: residues in the uniform job layout, 16-byte aligned
    const bool tma = tma_requested() && src == Source::Residues && fuse != Fuse::Combine && !prm.comb3 &&
                     (prm.njobs == 1 || prm.job_stride == (uint64_t)NP * prm.L) &&
                     ((uintptr_t)prm.data & 15) == 0;
    if (contig) {
        if (inverse && (src != Source::Residues || (fuse != Fuse::None && fuse != Fuse::Combine)))
            return cudaErrorInvalidValue;
        switch (logN) {
            case 6: return contig_pass<NP, 6>(inverse, src, fuse, prm, tw, st, tma);
            case 7: return contig_pass<NP, 7>(inverse, src, fuse, prm, tw, st, tma);
            case 8: return contig_pass<NP, 8>(inverse, src, fuse, prm, tw, st, tma);
            case 9: return contig_pass<NP, 9>(inverse, src, fuse, prm, tw, st, tma);
            case 10: return contig_pass<NP, 10>(inverse, src, fuse, prm, tw, st, tma);
            case 11: return contig_pass<NP, 11>(inverse, src, fuse, prm, tw, st, tma);
            case 12: return contig_pass<NP, 12>(inverse, src, fuse, prm, tw, st, tma);
            case 13: return contig_pass<NP, 13>(inverse, src, fuse, prm, tw, st, tma);
            case 14: return contig_pass<NP, 14>(inverse, src, fuse, prm, tw, st, tma);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (logN) {
        case 5: return strided_pass<NP, 5>(inverse, src, prm, tw, st, tma);
        case 6: return strided_pass<NP, 6>(inverse, src, prm, tw, st, tma);
        case 7: return strided_pass<NP, 7>(inverse, src, prm, tw, st, tma);
        case 8: return strided_pass<NP, 8>(inverse, src, prm, tw, st, tma);
        case 9: return strided_pass<NP, 9>(inverse, src, prm, tw, st, tma);
        case 10: return strided_pass<NP, 10>(inverse, src, prm, tw, st, tma);
        case 11: return strided_pass<NP, 11>(inverse, src, prm, tw, st, tma);
        case 12: return strided_pass<NP, 12>(inverse, src, prm, tw, st, tma);
        default: return cudaErrorInvalidValue;
    }
}

// Defined in ntt_wide.cu (the NP = 5 instantiations).
cudaError_t launch_pass_wide(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                             const TwiddleTables& tw, cudaStream_t st);
cudaError_t allow_big_tiles_wide();

}  // namespace pg
