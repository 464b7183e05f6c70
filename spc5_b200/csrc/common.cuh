// common.cuh -- shared definitions of the sm_100a beta(r,VS) kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

#include "spc5cuda.h"

namespace spc5cuda {

// Layout of SPC5Mat<T> (src/spc5.hpp:31-42, 145-148): VS = 512 / (8 sizeof T)
// columns per block, uint8 masks for double, uint16 masks for float.
template <class T>
struct Layout;
template <>
struct Layout<double> {
    static constexpr int VS = 8;
    static constexpr int MASK_BYTES = 1;
};
template <>
struct Layout<float> {
    static constexpr int VS = 16;
    static constexpr int MASK_BYTES = 2;
};

// Header stride of one block: int32 column + R masks (spc5.hpp:215-216).
template <class T, int R>
struct Header {
    static constexpr int STRIDE = 4 + R * Layout<T>::MASK_BYTES;
    static constexpr int MASK_BYTES_TOTAL = R * Layout<T>::MASK_BYTES;
    // 32-bit words that hold the mask bytes once the record is shifted to
    // byte 0 (the column occupies word 0).
    static constexpr int MASK_WORDS = (MASK_BYTES_TOTAL + 3) / 4;
    // aligned 32-bit words that cover one record: every one of them holds at
    // least one byte of the record, so none reads past the array.
    static constexpr int LOAD_WORDS = (STRIDE % 4 == 0) ? STRIDE / 4 : 2;
};

// Thrown inside the host layer, turned into a status code at the C ABI.
struct Error : std::runtime_error {
    spc5cuda_status status;
    Error(spc5cuda_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw Error(e == cudaErrorMemoryAllocation ? SPC5CUDA_ERR_NOMEM : SPC5CUDA_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define SPC5_CUDA(call) ::spc5cuda::check_cuda((call), #call)

inline int div_up(long a, long b) { return int((a + b - 1) / b); }

// Number of SMs of the current device (cached per device).
int sm_count();

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

// Decode the packed header of block b: returns the column and the mask bytes
// as little-endian 32-bit words (mask byte j in bits 8*(j%4) of mw[j/4]).
// Loads are aligned 32-bit words that each contain at least one byte of the
// record (the array base must be 4-byte aligned).
template <class T, int R>
__device__ __forceinline__ int load_header(const uint8_t* __restrict__ hdr, long b,
                                           uint32_t (&mw)[Header<T, R>::MASK_WORDS]) {
    using H = Header<T, R>;
    const long off = b * H::STRIDE;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(hdr) + (off >> 2);
    uint32_t lw[H::LOAD_WORDS + 1];
#pragma unroll
    for (int k = 0; k < H::LOAD_WORDS; ++k) lw[k] = __ldg(w + k);
    lw[H::LOAD_WORDS] = 0u;
    if constexpr (H::STRIDE % 4 == 0) {
#pragma unroll
        for (int k = 0; k < H::MASK_WORDS; ++k) mw[k] = lw[1 + k];
        return int(lw[0]);
    } else {
        const unsigned sh = unsigned(off & 3) * 8u;
        // the record ends inside this word: clear the next record's bytes
        mw[0] = __funnelshift_r(lw[1], lw[2], sh) & ((1u << (8 * H::MASK_BYTES_TOTAL)) - 1u);
        return int(__funnelshift_r(lw[0], lw[1], sh));
    }
}

// Mask of sub-row i from the decoded words.
template <class T, int R>
__device__ __forceinline__ uint32_t mask_of(const uint32_t (&mw)[Header<T, R>::MASK_WORDS], int i) {
    constexpr int MB = Layout<T>::MASK_BYTES;
    const int byte = i * MB;
    const uint32_t word = mw[byte >> 2];
    return (word >> ((byte & 3) * 8)) & (MB == 1 ? 0xFFu : 0xFFFFu);
}

// L2 cache policies: the matrix is streamed once per SpMV and should not
// push x out of L2; x is gathered many times and should stay.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 16-byte global -> shared asynchronous copy (L2 only) with an L2 policy.
__device__ __forceinline__ void cp_async16_hint(uint32_t saddr, const void* gptr, uint64_t pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gptr),
                 "l"(pol)
                 : "memory");
}

// Read-only load of an x element with an L2 policy.
__device__ __forceinline__ double ld_x(const double* p, uint64_t pol) {
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_x(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

}  // namespace spc5cuda
