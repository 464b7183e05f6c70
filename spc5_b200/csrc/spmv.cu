// spmv.cu -- beta(r,VS) SpMV kernels, y += A x.
//
// Mapping: one group of VS lanes (8 for f64, 16 for f32 / mixed) owns one
// block-row; lane c owns column c of every block of that block-row, with
// one accumulator per sub-row.  This is the lane structure of the reference
// AVX-512 kernels (core_SPC5_{r}rVc_Spmv_{double,float}, src/spc5.hpp:
// 2309-2715): per block the lane loads x[col + c] once and, for every sub-row
// whose mask has bit c, the value at the sub-row's compact offset plus
// popcount(mask & lanes-below-c) (the expand-load), then a fused
// multiply-add into that sub-row's accumulator.  Blocks are visited in
// order, so every (sub-row, lane) accumulator is the same FMA chain as the
// reference's vector lane; the row sum is the butterfly over lane distance
// VS/2 ... 1, which is the _mm512_reduce_add_{pd,ps} tree.  A lane whose bit
// is clear skips the FMA: the reference adds fma(0, x, acc) there, which
// leaves acc unchanged for finite x (acc is never -0.0 in round-to-nearest
// when it starts at +0.0), so y is bit-identical for finite x.
//
// The value offset of a block-row is not stored in the format; valptr holds
// it (from the CSR row pointer at conversion time, or a header pass).
#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

namespace {

constexpr int SPMV_THREADS = 256;

// Accumulator type A, value type V, x type X, y type Y.
template <class Layout_T, int R, class V, class X, class A, class Y>
__global__ void __launch_bounds__(SPMV_THREADS)
    k_spmv_groups(int nrows, int nbr, const int* __restrict__ brptr,
                  const uint8_t* __restrict__ headers, const V* __restrict__ values,
                  const int* __restrict__ valptr, const X* __restrict__ x, Y* __restrict__ y) {
    constexpr int VS = Layout<Layout_T>::VS;
    using H = Header<Layout_T, R>;
    const int lane = threadIdx.x & 31;
    const int c = lane & (VS - 1);
    const unsigned gmask = (VS == 32 ? 0xffffffffu : ((1u << VS) - 1u)) << (lane & ~(VS - 1));
    const uint32_t below = (1u << c) - 1u;
    const long group = (long(blockIdx.x) * blockDim.x + threadIdx.x) / VS;
    const long ngroups = (long(gridDim.x) * blockDim.x) / VS;
    for (long br = group; br < nbr; br += ngroups) {
        const int b1 = __ldg(brptr + br + 1);
        int b = __ldg(brptr + br);
        long v = __ldg(valptr + br);
        A acc[R];
#pragma unroll
        for (int i = 0; i < R; ++i) acc[i] = A(0);
        for (; b < b1; ++b) {
            uint32_t mw[H::MASK_WORDS];
            const int col = load_header<Layout_T, R>(headers, b, mw);
            uint32_t any = 0;
#pragma unroll
            for (int k = 0; k < H::MASK_WORDS; ++k) any |= mw[k];
            // fold every sub-row's mask onto the VS lane bits
            uint32_t lanes = 0;
#pragma unroll
            for (int i = 0; i < R; ++i) lanes |= mask_of<Layout_T, R>(mw, i);
            (void)any;
            A xv = A(0);
            if ((lanes >> c) & 1u) xv = A(__ldg(x + col + c));
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const uint32_t m = mask_of<Layout_T, R>(mw, i);
                if ((m >> c) & 1u) {
                    const A e = A(__ldg(values + v + __popc(m & below)));
                    acc[i] = fma(e, xv, acc[i]);
                }
                v += __popc(m);
            }
        }
        // _mm512_reduce_add tree: lane distance VS/2, ..., 1
#pragma unroll
        for (int i = 0; i < R; ++i) {
#pragma unroll
            for (int d = VS / 2; d >= 1; d >>= 1) acc[i] += __shfl_xor_sync(gmask, acc[i], d, VS);
        }
        A s = acc[0];
#pragma unroll
        for (int i = 1; i < R; ++i)
            if (c == i) s = acc[i];
        const long row = br * R + c;
        if (c < R && row < nrows) y[row] += Y(s);
    }
}

template <class Layout_T, class V, class X, class A, class Y>
void launch_groups(const BetaView& m, const X* x, Y* y, cudaStream_t s) {
    if (m.nbr <= 0) return;
    constexpr int VS = Layout<Layout_T>::VS;
    const long groups_needed = m.nbr;
    const int per_cta = SPMV_THREADS / VS;
    const int max_ctas = sm_count() * (2048 / SPMV_THREADS) * 4;
    const int ctas = int(std::max(1L, std::min<long>((groups_needed + per_cta - 1) / per_cta, max_ctas)));
    const V* vals = static_cast<const V*>(m.values);
    switch (m.r) {
        case 1:
            k_spmv_groups<Layout_T, 1, V, X, A, Y><<<ctas, SPMV_THREADS, 0, s>>>(
                m.nrows, m.nbr, m.brptr, m.headers, vals, m.valptr, x, y);
            break;
        case 2:
            k_spmv_groups<Layout_T, 2, V, X, A, Y><<<ctas, SPMV_THREADS, 0, s>>>(
                m.nrows, m.nbr, m.brptr, m.headers, vals, m.valptr, x, y);
            break;
        case 4:
            k_spmv_groups<Layout_T, 4, V, X, A, Y><<<ctas, SPMV_THREADS, 0, s>>>(
                m.nrows, m.nbr, m.brptr, m.headers, vals, m.valptr, x, y);
            break;
        case 8:
            k_spmv_groups<Layout_T, 8, V, X, A, Y><<<ctas, SPMV_THREADS, 0, s>>>(
                m.nrows, m.nbr, m.brptr, m.headers, vals, m.valptr, x, y);
            break;
        default:
            throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    }
    SPC5_CUDA(cudaGetLastError());
}

}  // namespace

void launch_spmv_f64(const BetaView& m, const double* x, double* y, cudaStream_t s) {
    launch_groups<double, double, double, double, double>(m, x, y, s);
}

void launch_spmv_f32(const BetaView& m, const float* x, float* y, cudaStream_t s) {
    launch_groups<float, float, float, float, float>(m, x, y, s);
}

void launch_spmv_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    launch_groups<float, float, float, double, double>(m, x, y, s);
}

}  // namespace spc5cuda
