// spmv_rows.cu -- thread-per-sub-row beta(r,VS) SpMV, y += A x, for
// matrices whose block-rows are short (every block-row's headers and values
// fit one per-warp staging buffer: stencils, Poisson, banded and FEM-like
// matrices).
//
// Work split: warp w owns the contiguous block-rows [wstart[w], wstart[w+1])
// (balanced by blocks).  It walks them in chunks of at most 32 / L
// block-rows (L lanes per block-row, L >= r): the chunk's packed headers and
// values are copied into the warp's shared-memory buffer with coalesced
// 16-byte cp.async (rows_stage.cuh), then the L lanes of each block-row work
// on it from shared memory.  With L = r >= 2 lane s owns sub-row s and all VS
// columns; otherwise lane q owns the columns q + L k of every sub-row.
// Either way a lane holds r * VS / L accumulators in registers, a block
// costs it one header decode and predicated multiply-adds, and the row sums
// need at most log2(L) shuffles per block-row.  The sorted plan (plan.cu)
// also runs this kernel on segments of block-rows too large to stage.
//
// Arithmetic (bit-identical to the reference kernels core_SPC5_{r}rVc_Spmv_*,
// src/spc5.hpp:2309-2715): accumulator c of sub-row s receives
// fma(value, x[col + c], acc[c]) for every block in order whose mask s has
// bit c, reading the values at the sub-row's compact offset in the block
// (the masks of the sub-rows below s, then popcount of the bits below c) --
// the expand-load of the vector kernel.  The row sum is the
// _mm512_reduce_add tree over the accumulators (distance VS/2, then VS/4,
// ..., 1) and y[row] += sum.  Clear bits skip the FMA, which leaves the
// accumulator unchanged for finite x (it starts at +0.0 and never becomes
// -0.0), so y is bit-identical for finite x.
#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"
#include "rows_stage.cuh"

namespace spc5cuda {

namespace {

using rows::FULL;
constexpr int ROWS_THREADS = rows::THREADS;
constexpr int ROWS_WARPS = rows::WARPS;
constexpr int ROWS_CTAS_PER_SM = 16;

template <class LT, int R, class V, int L>
using RowGeo = rows::Geo<LT, R, V, L>;

// The blocks [b, b_stop) of a staged chunk for the lane that owns sub-row q
// of its block-row and all VS columns (acc[c / CPL][c % CPL] is column c).
// Its values in a block are contiguous: after those of the sub-rows below q,
// one per set bit of its mask, in column order.
template <class LT, int R, class V, class X, class A, int CPL>
__device__ __forceinline__ void rows_subrow_blocks(const uint32_t* hw, long h_al, const V* vbuf,
                                                   const X* __restrict__ x, int q, int& b, int b_stop, int& v,
                                                   uint64_t pol_x, A (&acc)[R][CPL]) {
    constexpr int VS = Layout<LT>::VS, MB = Layout<LT>::MASK_BYTES;
    constexpr int MW = Header<LT, R>::MASK_WORDS, STRIDE = Header<LT, R>::STRIDE;
    constexpr int FPW = 4 / MB, BITS = 8 * MB;
    constexpr uint32_t FMASK = MB == 1 ? 0xFFu : 0xFFFFu;
    // blocks per step (their x loads are issued together): 4 at r = 8 for
    // double blocks, else 16 / VS (measured on B200: 4 blocks lifted the
    // power-law r = 8 SpMV by 10% and slowed r = 2 by 9%)
    constexpr int UT = (R == 8 && VS == 8) ? 4 : (16 / VS > 1 ? 16 / VS : 1);
    const int wq = q / FPW;
    const unsigned sh = unsigned(q % FPW) * BITS;
    uint32_t lowmask[MW];  // mask bits of the sub-rows below q
#pragma unroll
    for (int w = 0; w < MW; ++w) lowmask[w] = w < wq ? 0xFFFFFFFFu : (w == wq ? (1u << sh) - 1u : 0u);
    while (__any_sync(FULL, b < b_stop)) {
        int col[UT];
        uint32_t mw[UT][MW];
        uint32_t mi[UT];
#pragma unroll
        for (int u = 0; u < UT; ++u) {
            col[u] = 0;
#pragma unroll
            for (int w = 0; w < MW; ++w) mw[u][w] = 0u;
            if (b + u < b_stop) col[u] = rows::decode_staged<LT, R>(hw, long(b + u) * STRIDE - h_al, mw[u]);
            uint32_t word = mw[u][0];
#pragma unroll
            for (int w = 1; w < MW; ++w) word = w == wq ? mw[u][w] : word;
            mi[u] = (word >> sh) & FMASK;
        }
        X xk[UT][VS];
#pragma unroll
        for (int u = 0; u < UT; ++u) {
            const X* xp = x + col[u];
#pragma unroll
            for (int c = 0; c < VS; ++c) xk[u][c] = ((mi[u] >> c) & 1u) ? ld_x(xp + c, pol_x) : X(0);
        }
#pragma unroll
        for (int u = 0; u < UT; ++u) {
            int pre = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < MW; ++w) {
                pre += __popc(mw[u][w] & lowmask[w]);
                tot += __popc(mw[u][w]);
            }
            int idx = v + pre;
#pragma unroll
            for (int c = 0; c < VS; ++c) {
                if ((mi[u] >> c) & 1u) {
                    acc[c / CPL][c % CPL] = fma(A(vbuf[idx]), A(xk[u][c]), acc[c / CPL][c % CPL]);
                    ++idx;
                }
            }
            v += tot;
        }
        b += UT;
    }
}

// SEG: the block-rows are segments of long block-rows (the length-sorted
// plan's largest ones), laid out so that chunk k of warp w holds segment k of
// each of the block-rows w * 32 / L + slot (nseg of them, ng = min(32 / L,
// nseg - w * 32 / L) in warp w): a lane keeps its accumulators from chunk to
// chunk and adds its row sum to y after the last one (perm[w * 32 / L +
// slot] is the block-row of y).  The FMA chain of every (sub-row, column) is
// the block-row's own, in block order.
template <class LT, int R, class V, class X, class A, class Y, int L, bool SEG>
__global__ void __launch_bounds__(ROWS_THREADS)
    k_rows(int nrows, const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
           const V* __restrict__ values, const int* __restrict__ valptr,
           const int* __restrict__ wstart, int nwarps, const int* __restrict__ perm, int nseg,
           const X* __restrict__ x, Y* __restrict__ y, const int* __restrict__ run_if, int run_if_value) {
    // a launch gated on a device word (see BetaView::run_if)
    if (run_if && __ldg(run_if) != run_if_value) return;
    using G = RowGeo<LT, R, V, L>;
    constexpr int VS = G::VS, MB = G::MB, MW = G::MW, SPW = G::SPW;
    constexpr int FPW = 4 / MB;  // mask fields per 32-bit word
    constexpr int BITS = 8 * MB;
    constexpr uint32_t FMASK = MB == 1 ? 0xFFu : 0xFFFFu;
    constexpr bool Y_ATOMIC = sizeof(Y) == 8;  // red.add.f64 is y + s rounded once
    constexpr int CPL = VS / L;  // columns per lane
    // L = r >= 2: lane q owns sub-row q for all VS columns instead (the same
    // R * CPL = VS accumulators, held per column: acc[c / CPL][c % CPL]).  A
    // column lane pays the offset arithmetic of every mask field per block; a
    // sub-row lane finds its values contiguous, after the masks below its own.
    // Not in the segmented part at r = 4, where the column lanes' x loads of 8
    // blocks per step hide the gathers better (measured on B200).
    constexpr bool TRANS = R >= 2 && L == R && !(R == 4 && SEG);
    extern __shared__ __align__(16) unsigned char smem[];

    const int lane = threadIdx.x & 31;
    const int wi = threadIdx.x >> 5;
    const int warp = blockIdx.x * ROWS_WARPS + wi;
    const int slot = lane / L;  // block-row of the chunk
    const int q = lane % L;     // column class: this lane owns columns c = q + L k

    int r_begin = 0, r_stop = 0;
    if (warp < nwarps) {
        r_begin = __ldg(wstart + warp);
        r_stop = __ldg(wstart + warp + 1);
    }
    const uint64_t pol_x = l2_evict_last_policy();

    A acc[R][CPL];
    auto zero = [&]() {
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int k = 0; k < CPL; ++k) acc[i][k] = A(0);
    };
    // ---- row sums: the _mm512_reduce_add tree (distance VS/2, ..., 1).
    // Levels of distance >= L pair columns of the same class inside the
    // lane; the last log2(L) levels pair the lanes of the block-row.  Then
    // y[brow * R + q] += sum of sub-row q (warp-uniform call).
    auto flush = [&](bool mine, int brow) {
        A res = A(0);
        if constexpr (TRANS) {
            // the whole tree inside the lane: column c in acc[c / CPL][c % CPL]
#pragma unroll
            for (int d = VS / 2; d >= 1; d >>= 1) {
#pragma unroll
                for (int c = 0; c < d; ++c)
                    acc[c / CPL][c % CPL] = acc[c / CPL][c % CPL] + acc[(c + d) / CPL][(c + d) % CPL];
            }
            res = acc[0][0];
        } else {
#pragma unroll
            for (int i = 0; i < R; ++i) {
#pragma unroll
                for (int d = CPL / 2; d >= 1; d >>= 1) {
#pragma unroll
                    for (int k = 0; k < d; ++k) acc[i][k] = acc[i][k] + acc[i][k + d];
                }
                A sum = acc[i][0];
#pragma unroll
                for (int d = L / 2; d >= 1; d >>= 1) sum = sum + __shfl_xor_sync(FULL, sum, d);
                if (i == q) res = sum;
            }
        }
        if (mine && q < R) {
            const long yrow = long(brow) * R + q;
            if (yrow < nrows) {
                if constexpr (Y_ATOMIC) atomicAdd(y + yrow, Y(res));
                else y[yrow] = y[yrow] + Y(res);
            }
        }
    };

    // ---- the blocks of block-row r0 + slot of a staged chunk
    auto compute = [&](const rows::Chunk& ch, const uint32_t* hw, const V* vbuf) {
        // blocks per step: the x loads of all of them are issued before the
        // FMAs, which still run block by block (the chain order is kept)
        constexpr int U = (16 / CPL) < 1 ? 1 : ((16 / CPL) > 8 ? 8 : 16 / CPL);
        const int src = slot > 0 ? slot - 1 : 0;
        const int b_prev = __shfl_sync(FULL, ch.b_hi, src);
        const int v_prev = __shfl_sync(FULL, ch.v_hi, src);
        const int b_mine = __shfl_sync(FULL, ch.b_hi, slot);
        const bool mine = slot < ch.nrow;
        int b = mine ? (slot > 0 ? b_prev : ch.b_lo) : 0;
        const int b_stop = mine ? b_mine : 0;
        int v = (mine ? (slot > 0 ? v_prev : ch.v_lo) : 0) - ch.v_al;  // buffer index of the block's values

        if constexpr (!SEG) zero();
        if constexpr (TRANS) {
            rows_subrow_blocks<LT, R, V, X, A, CPL>(hw, ch.h_al, vbuf, x, q, b, b_stop, v, pol_x, acc);
        } else {
            while (__any_sync(FULL, b < b_stop)) {
                int col[U];
                uint32_t mw[U][MW];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    col[u] = 0;
#pragma unroll
                    for (int w = 0; w < MW; ++w) mw[u][w] = 0u;
                    if (b + u < b_stop) col[u] = rows::decode_staged<LT, R>(hw, long(b + u) * G::STRIDE - ch.h_al, mw[u]);
                }
                // x of this lane's columns where some sub-row has a value
                X xk[U][CPL];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t uni = rows::mask_union<LT, R>(mw[u]);
                    const X* xp = x + col[u] + q;
#pragma unroll
                    for (int k = 0; k < CPL; ++k)
                        xk[u][k] = ((uni >> (q + L * k)) & 1u) ? ld_x(xp + L * k, pol_x) : X(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    uint32_t pre[MW];
                    const int tot = rows::subrow_prefix<LT, R>(mw[u], pre);
#pragma unroll
                    for (int k = 0; k < CPL; ++k) {
                        const int c = q + L * k;
                        const uint32_t below = (1u << c) - 1u;
#pragma unroll
                        for (int w = 0; w < MW; ++w) {
                            // field i: buffer offset of sub-row i's value in column c
                            const uint32_t off = rows::column_offsets<LT, R>(mw[u][w], pre[w], below);
#pragma unroll
                            for (int f = 0; f < FPW; ++f) {
                                const int i = w * FPW + f;
                                if (i < R && ((mw[u][w] >> (f * BITS + c)) & 1u)) {
                                    const int idx = v + int((off >> (f * BITS)) & FMASK);
                                    acc[i][k] = fma(A(vbuf[idx]), A(xk[u][k]), acc[i][k]);
                                }
                            }
                        }
                    }
                    v += tot;
                }
                b += U;
            }
        }
        if constexpr (!SEG) flush(mine, mine ? (perm ? __ldg(perm + ch.r0 + slot) : ch.r0 + slot) : 0);
    };

    unsigned char* wbuf = smem + wi * G::BUF_BYTES;
    if constexpr (SEG) {
        if (warp >= nwarps) return;  // warp-uniform
        const int ng = min(SPW, nseg - warp * SPW);
        zero();
        rows::walk<LT, R, V, L>(brptr, headers, values, valptr, r_begin, r_stop, wbuf, compute, ng);
        flush(slot < ng, slot < ng ? __ldg(perm + warp * SPW + slot) : 0);
    } else {
        rows::walk<LT, R, V, L>(brptr, headers, values, valptr, r_begin, r_stop, wbuf, compute);
    }
}

template <class K>
void set_smem(K kernel, int bytes) {
    SPC5_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// Calls f(std::integral_constant<int, R>, std::integral_constant<int, L>)
// for a supported (r, lanes-per-block-row) pair: L >= r, L in {1, 2, 4, 8}.
template <class F>
void dispatch_rl(int r, int lanes, F&& f) {
    using std::integral_constant;
    const int L = lanes ? lanes : r;
    switch (r) {
        case 1:
            switch (L) {
                case 1: f(integral_constant<int, 1>{}, integral_constant<int, 1>{}); return;
                case 2: f(integral_constant<int, 1>{}, integral_constant<int, 2>{}); return;
                case 4: f(integral_constant<int, 1>{}, integral_constant<int, 4>{}); return;
                case 8: f(integral_constant<int, 1>{}, integral_constant<int, 8>{}); return;
            }
            break;
        case 2:
            switch (L) {
                case 2: f(integral_constant<int, 2>{}, integral_constant<int, 2>{}); return;
                case 4: f(integral_constant<int, 2>{}, integral_constant<int, 4>{}); return;
                case 8: f(integral_constant<int, 2>{}, integral_constant<int, 8>{}); return;
            }
            break;
        case 4:
            switch (L) {
                case 4: f(integral_constant<int, 4>{}, integral_constant<int, 4>{}); return;
                case 8: f(integral_constant<int, 4>{}, integral_constant<int, 8>{}); return;
            }
            break;
        case 8:
            if (L == 8) {
                f(integral_constant<int, 8>{}, integral_constant<int, 8>{});
                return;
            }
            break;
    }
    throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8 and lanes >= r");
}

template <class LT, class V, class X, class A, class Y>
int rows_occupancy(int r, int lanes) {
    int n = 0;
    dispatch_rl(r, lanes, [&](auto RC, auto LC) {
        constexpr int R_ = decltype(RC)::value, L_ = decltype(LC)::value;
        using G = RowGeo<LT, R_, V, L_>;
        auto kern = k_rows<LT, R_, V, X, A, Y, L_, false>;
        set_smem(kern, G::SMEM);
        SPC5_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, ROWS_THREADS, G::SMEM));
    });
    return std::max(1, std::min(n, ROWS_CTAS_PER_SM));
}

template <class LT, class V, class X, class A, class Y>
void launch_rows_impl(const BetaView& m, const X* x, Y* y, cudaStream_t s) {
    if (m.nbr <= 0 || m.nwarps <= 0) return;
    const V* vals = static_cast<const V*>(m.values);
    const int ctas = (m.nwarps + ROWS_WARPS - 1) / ROWS_WARPS;
    dispatch_rl(m.r, m.lanes, [&](auto RC, auto LC) {
        constexpr int R_ = decltype(RC)::value, L_ = decltype(LC)::value;
        using G = RowGeo<LT, R_, V, L_>;
        auto kern = m.nseg > 0 ? k_rows<LT, R_, V, X, A, Y, L_, true> : k_rows<LT, R_, V, X, A, Y, L_, false>;
        set_smem(kern, G::SMEM);
        kern<<<ctas, ROWS_THREADS, G::SMEM, s>>>(m.nrows, m.brptr, m.headers, vals, m.valptr, m.wstart,
                                                 m.nwarps, m.perm, m.nseg, x, y, m.run_if, m.run_if_value);
    });
    SPC5_CUDA(cudaGetLastError());
}

// flag[0] = 1 when a block-row of maxes[0] blocks and maxes[1] values fits
// the staging buffers (the test of rows_fit, on the device), else 0.
__global__ void k_fit_flag(const int* __restrict__ maxes, int stride, int vbytes, int hb, int vb,
                           int* __restrict__ flag) {
    const long hneed = long(maxes[0]) * stride + 32;
    const long vneed = (long(maxes[1]) + 2 * (16 / vbytes)) * vbytes;
    flag[0] = (hneed <= hb && vneed <= vb) ? 1 : 0;
}

// Largest block count and value count of any block-row.
__global__ void k_blockrow_max(int nbr, const int* __restrict__ brptr, const int* __restrict__ valptr,
                               int* __restrict__ out) {
    int mb = 0, mv = 0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        mb = max(mb, brptr[i + 1] - brptr[i]);
        mv = max(mv, valptr[i + 1] - valptr[i]);
    }
    for (int d = 16; d >= 1; d >>= 1) {
        mb = max(mb, __shfl_xor_sync(FULL, mb, d));
        mv = max(mv, __shfl_xor_sync(FULL, mv, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, mb);
        atomicMax(out + 1, mv);
    }
}

}  // namespace

int rows_warps(int vt, int r, int lanes) {
    // cached per (device, value type, r, lanes): the drop-in symbols ask on
    // every call
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, int> cache;
    int dev = 0;
    SPC5_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, vt, r, lanes);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    int per_sm;
    if (vt == SPC5CUDA_F64) {
        per_sm = rows_occupancy<double, double, double, double, double>(r, lanes);
    } else if (vt == SPC5CUDA_F32_V8) {
        per_sm = rows_occupancy<double, float, float, double, double>(r, lanes);
    } else {
        per_sm = std::min(rows_occupancy<float, float, float, float, float>(r, lanes),
                          rows_occupancy<float, float, float, double, double>(r, lanes));
    }
    const int n = sm_count() * per_sm * ROWS_WARPS;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = n;
    return n;
}

// Staging buffer sizes of RowGeo (every instantiation).
constexpr int ROWS_HB = rows::HB;
constexpr int ROWS_VB = rows::VB;

bool rows_fit(int vt, int r, int max_blocks, int max_values) {
    // every block-row alone must fit the staging buffers, alignment included
    const int stride = 4 + r * (vt == SPC5CUDA_F32 ? 2 : 1);
    const int vbytes = vt == SPC5CUDA_F64 ? 8 : 4;
    const long hneed = long(max_blocks) * stride + 32;
    const long vneed = (long(max_values) + 2 * (16 / vbytes)) * vbytes;
    return hneed <= ROWS_HB && vneed <= ROWS_VB;
}

long rows_lane_units(int vt, int r, int nblocks, int nvalues) {
    // a block-row of this size fits `lanes` lanes' share of a chunk (32 / lanes
    // block-rows per chunk) when the result is <= lanes * ROWS_UNIT
    const long stride = 4 + r * (vt == SPC5CUDA_F32 ? 2 : 1);
    const long vbytes = vt == SPC5CUDA_F64 ? 8 : 4;
    return std::max(long(nblocks) * stride * (ROWS_VB - 32), long(nvalues) * vbytes * (ROWS_HB - 32));
}

long rows_unit() { return long(ROWS_HB - 32) * long(ROWS_VB - 32) / 32; }

int rows_hb() { return ROWS_HB; }
int rows_vb() { return ROWS_VB; }

void blockrow_max(int nbr, const int* brptr, const int* valptr, int* max_blocks, int* max_values,
                  cudaStream_t s) {
    int* d = nullptr;
    SPC5_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d), 2 * sizeof(int), s));
    SPC5_CUDA(cudaMemsetAsync(d, 0, 2 * sizeof(int), s));
    if (nbr > 0) {
        const int threads = 256;
        const int blocks = std::max(1, std::min(div_up(nbr, threads), sm_count() * 4));
        k_blockrow_max<<<blocks, threads, 0, s>>>(nbr, brptr, valptr, d);
        SPC5_CUDA(cudaGetLastError());
    }
    int h[2] = {0, 0};
    SPC5_CUDA(cudaMemcpyAsync(h, d, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaFreeAsync(d, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    *max_blocks = h[0];
    *max_values = h[1];
}

void launch_rows_fit_flag(int vt, int r, int nbr, const int* brptr, const int* valptr, int* work,
                          cudaStream_t s) {
    SPC5_CUDA(cudaMemsetAsync(work, 0, 3 * sizeof(int), s));
    if (nbr > 0) {
        const int threads = 256;
        const int blocks = std::max(1, std::min(div_up(nbr, threads), sm_count() * 4));
        k_blockrow_max<<<blocks, threads, 0, s>>>(nbr, brptr, valptr, work + 1);
        SPC5_CUDA(cudaGetLastError());
    }
    const int stride = 4 + r * (vt == SPC5CUDA_F32 ? 2 : 1);
    const int vbytes = vt == SPC5CUDA_F64 ? 8 : 4;
    k_fit_flag<<<1, 1, 0, s>>>(work + 1, stride, vbytes, ROWS_HB, ROWS_VB, work);
    SPC5_CUDA(cudaGetLastError());
}

void launch_rows_f64(const BetaView& m, const double* x, double* y, cudaStream_t s) {
    launch_rows_impl<double, double, double, double, double>(m, x, y, s);
}

void launch_rows_f32(const BetaView& m, const float* x, float* y, cudaStream_t s) {
    launch_rows_impl<float, float, float, float, float>(m, x, y, s);
}

void launch_rows_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    launch_rows_impl<float, float, float, double, double>(m, x, y, s);
}

void launch_rows_mixed8(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    launch_rows_impl<double, float, float, double, double>(m, x, y, s);
}

}  // namespace spc5cuda
