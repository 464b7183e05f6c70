// spmm_rows.cu -- staged multi-RHS SpMM, Y += A X, for matrices whose every
// block-row fits the row kernels' staging buffers (rows_stage.cuh).
//
// A warp walks its block-rows in chunks staged into shared memory; each
// block-row of a chunk is served by L lanes (mm_lanes), and lane q owns the
// columns q + L k of every block for all R sub-rows and KC right-hand sides
// (R * VS / L * KC accumulators, at most 32).  Per block a lane decodes the
// staged header once, loads its KC x values per column (only where some
// sub-row has a value in that column: blocks at the right edge may reach
// past the last column), reads each of its values once from shared memory
// and issues KC multiply-adds with it.  The sorted plan's parts run here too
// (the block-row permutation, and the segments of its largest block-rows).
//
// Arithmetic per right-hand side j is the SpMV's (src/spc5.hpp:2309-2715):
// accumulator (i, j) of column c receives fma(value, x[col + c][j], acc) for
// every block in order whose mask i has bit c; the row sum is the
// _mm512_reduce_add tree over the VS columns (XOR distances VS/2, ..., 1: in
// the lane, then across the L lanes); then
// Y[row][j] += sum (one rounding: red.add.f64 for double Y, load-add-store for
// float Y, exactly as the SpMV kernels).  Column j of the result is therefore
// bit-identical to an SpMV with column j of X.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "rows_stage.cuh"

namespace spc5cuda {

namespace {

using rows::FULL;

// Lanes per block-row of the staged SpMM: one column per lane for double
// blocks (8 columns); for float blocks (16 columns) two per lane, except at
// r = 8 where one column per lane keeps four right-hand sides per pass.  The
// segmented part of a sorted plan keeps the plan's lanes (seg_lanes).
template <class LT, int R, bool SEG>
constexpr int mm_lanes() {
    if constexpr (SEG) return seg_lanes(R);
    return (Layout<LT>::VS == 16 && R == 8) ? 16 : 8;
}

// Y += A X over block-rows [r_begin, r_stop) of one matrix for right-hand
// sides [0, KC) of xm / ym (already offset to the pass's first one); perm
// (if not null) maps a block-row of these arrays to its block-row of Y.  SEG:
// the block-rows are the interleaved segments of ng long block-rows (chunk k
// holds segment k of each, as the segmented row kernel reads them), whose
// block-rows of Y are perm[seg_base + slot]; a lane keeps its accumulators
// over all chunks and Y is updated once, after the last.
template <class LT, int R, int KC, class V, class X, class A, class Y, bool SEG>
__device__ __forceinline__ void mm_range(int nrows, const int* __restrict__ brptr,
                                         const uint8_t* __restrict__ headers, const V* __restrict__ values,
                                         const int* __restrict__ valptr, int r_begin, int r_stop,
                                         const int* __restrict__ perm, int ng, int seg_base,
                                         const X* __restrict__ xm, long ldx, long xcs, Y* __restrict__ ym,
                                         long ldy, long ycs, unsigned char* wbuf) {
    constexpr int VS = Layout<LT>::VS;
    constexpr int L = mm_lanes<LT, R, SEG>();  // lanes per block-row
    constexpr int CPL = VS / L;                // columns per lane: q + L k
    constexpr int LOGL = L == 16 ? 4 : (L == 8 ? 3 : (L == 4 ? 2 : (L == 2 ? 1 : 0)));
    using G = rows::Geo<LT, R, V, L, rows::MM_HB, rows::MM_VB>;
    constexpr int MB = G::MB, MW = G::MW;
    constexpr int FPW = 4 / MB;  // mask fields per 32-bit word
    constexpr int BITS = 8 * MB;
    constexpr uint32_t FMASK = MB == 1 ? 0xFFu : 0xFFFFu;
    constexpr bool Y_ATOMIC = sizeof(Y) == 8;
    static_assert(R * CPL * KC <= 32, "accumulators");
    // blocks per step: their x loads are issued before the FMAs, which still
    // run block by block (the chain order is kept)
    constexpr int XW = CPL * KC;  // x values of one block
    constexpr int U = XW >= 8 ? 1 : 8 / XW;
    const int lane = threadIdx.x & 31;
    const int slot = lane / L;  // block-row of the chunk
    const int q = lane % L;     // this lane's columns: q + L k
    const uint64_t pol_x = l2_evict_last_policy();

    A acc[R][CPL][KC];
    auto zero = [&]() {
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int k = 0; k < CPL; ++k)
#pragma unroll
                for (int j = 0; j < KC; ++j) acc[i][k][j] = A(0);
    };

    // ---- row sums: the _mm512_reduce_add tree (distance VS/2, ..., 1).
    // Levels of distance >= L pair columns of one lane.  The last log2(L)
    // levels pair the lanes of the block-row as a reduce-scatter of the
    // N = R KC sums: at distance d the lane with bit d set keeps the odd
    // entries and its partner the even ones, each adding the partner's
    // copy (the same pairs as the tree, so the same bits), until one sum
    // per entry is left; then the plain butterfly.  Lane q ends with the
    // entries t L + rev(q) (rev: q's log2(L) bits reversed), or, when
    // N < L, entry rev(q) mod N in the lanes whose low bits are zero.
    // Entries are ordered so that one store covers neighbouring
    // addresses: (i, j) at i KC + j for row-major Y (ycs == 1), at j R + i
    // otherwise (the R rows of consecutive block-rows are adjacent).  Then
    // Y[brow R + i][j] += sum (warp-uniform call).
    auto flush = [&](bool mine, int brow) {
        constexpr int N = R * KC;
#pragma unroll
        for (int i = 0; i < R; ++i) {
#pragma unroll
            for (int j = 0; j < KC; ++j) {
#pragma unroll
                for (int d = CPL / 2; d >= 1; d >>= 1) {
#pragma unroll
                    for (int k = 0; k < d; ++k) acc[i][k][j] = acc[i][k][j] + acc[i][k + d][j];
                }
            }
        }
        const bool row_major = ycs == 1;
        A sv[N];
#pragma unroll
        for (int e = 0; e < N; ++e) sv[e] = row_major ? acc[e / KC][0][e % KC] : acc[e % R][0][e / R];
#pragma unroll
        for (int lev = 0; lev < LOGL; ++lev) {
            const int d = L >> (lev + 1);
            const int n = N >> lev;  // entries still held
            const bool hi = (q & d) != 0;
            if (n >= 2) {
#pragma unroll
                for (int t = 0; t < n / 2; ++t) {
                    const A keep = hi ? sv[2 * t + 1] : sv[2 * t];
                    const A send = hi ? sv[2 * t] : sv[2 * t + 1];
                    sv[t] = keep + __shfl_xor_sync(FULL, send, d);
                }
            } else {
                sv[0] = sv[0] + __shfl_xor_sync(FULL, sv[0], d);
            }
        }
        const int rq = LOGL ? int(__brev(unsigned(q)) >> (32 - LOGL)) : 0;
        constexpr int PER = N >= L ? N / L : 1;
        const bool writer = mine && (N >= L || (q & (L / N - 1)) == 0);
        const long row0 = long(brow) * R;
#pragma unroll
        for (int t = 0; t < PER; ++t) {
            const int e = N >= L ? t * L + rq : (rq & (N - 1));
            const int i = row_major ? e / KC : e % R;
            const int j = row_major ? e % KC : e / R;
            const long yrow = row0 + i;
            if (writer && yrow < nrows) {
                Y* dst = ym + yrow * ldy + long(j) * ycs;
                if constexpr (Y_ATOMIC) atomicAdd(dst, Y(sv[t]));
                else *dst = *dst + Y(sv[t]);
            }
        }
    };

    auto compute = [&](const rows::Chunk& ch, const uint32_t* hw, const V* vbuf) {
        const int src = slot > 0 ? slot - 1 : 0;
        const int b_prev = __shfl_sync(FULL, ch.b_hi, src);
        const int v_prev = __shfl_sync(FULL, ch.v_hi, src);
        const int b_mine = __shfl_sync(FULL, ch.b_hi, slot);
        const bool mine = slot < ch.nrow;
        int b = mine ? (slot > 0 ? b_prev : ch.b_lo) : 0;
        const int b_stop = mine ? b_mine : 0;
        int v = (mine ? (slot > 0 ? v_prev : ch.v_lo) : 0) - ch.v_al;

        if constexpr (!SEG) zero();
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
            X xk[U][CPL][KC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t uni = rows::mask_union<LT, R>(mw[u]);
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    const bool has = (uni >> (q + L * k)) & 1u;
                    const X* xr = xm + long(col[u] + q + L * k) * ldx;
#pragma unroll
                    for (int j = 0; j < KC; ++j) xk[u][k][j] = has ? ld_x(xr + long(j) * xcs, pol_x) : X(0);
                }
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
                        const uint32_t off = rows::column_offsets<LT, R>(mw[u][w], pre[w], below);
#pragma unroll
                        for (int f = 0; f < FPW; ++f) {
                            const int i = w * FPW + f;
                            if (i < R && ((mw[u][w] >> (f * BITS + c)) & 1u)) {
                                const A e = A(vbuf[v + int((off >> (f * BITS)) & FMASK)]);
#pragma unroll
                                for (int j = 0; j < KC; ++j) acc[i][k][j] = fma(e, A(xk[u][k][j]), acc[i][k][j]);
                            }
                        }
                    }
                }
                v += tot;
            }
            b += U;
        }
        if constexpr (!SEG) flush(mine, mine ? (perm ? __ldg(perm + ch.r0 + slot) : ch.r0 + slot) : 0);
    };
    if constexpr (SEG) {
        zero();
        rows::walk<LT, R, V, L, rows::MM_HB, rows::MM_VB>(brptr, headers, values, valptr, r_begin, r_stop, wbuf,
                                                          compute, ng);
        flush(slot < ng, slot < ng ? __ldg(perm + seg_base + slot) : 0);
    } else {
        rows::walk<LT, R, V, L, rows::MM_HB, rows::MM_VB>(brptr, headers, values, valptr, r_begin, r_stop, wbuf,
                                                          compute);
    }
}

// One matrix: warp w owns block-rows [wstart[w], wstart[w + 1]).  SEG: warp
// w owns the segments of long block-rows w * 32 / L + slot (nseg in all).
template <class LT, int R, int KC, class V, class X, class A, class Y, bool SEG>
__global__ void __launch_bounds__(rows::THREADS)
    k_spmm_rows(int nrows, const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
                const V* __restrict__ values, const int* __restrict__ valptr, const int* __restrict__ wstart,
                int nwarps, const int* __restrict__ perm, int nseg, const X* __restrict__ xm, long ldx, long xcs,
                Y* __restrict__ ym, long ldy, long ycs) {
    constexpr int L = mm_lanes<LT, R, SEG>();
    using G = rows::Geo<LT, R, V, L, rows::MM_HB, rows::MM_VB>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int wi = threadIdx.x >> 5;
    const int warp = blockIdx.x * rows::WARPS + wi;
    if (warp >= nwarps) return;  // warp-uniform
    const int r_begin = __ldg(wstart + warp), r_stop = __ldg(wstart + warp + 1);
    const int ng = SEG ? min(G::SPW, nseg - warp * G::SPW) : 0;
    mm_range<LT, R, KC, V, X, A, Y, SEG>(nrows, brptr, headers, values, valptr, r_begin, r_stop, perm, ng,
                                         warp * G::SPW, xm, ldx, xcs, ym, ldy, ycs, smem + wi * G::BUF_BYTES);
}

// Batched: warps walk the job list with the grid's warp count as stride; job
// j is block-rows [r_begin, r_end) of mats[j.mat] for right-hand sides
// [kofs, kofs + KC).  X and Y of a batch are row-major (xcs = ycs = 1).
template <class LT, int R, int KC, class V, class X, class A, class Y>
__global__ void __launch_bounds__(rows::THREADS)
    k_spmm_rows_batch(const BatchMat* __restrict__ mats, const BatchJob* __restrict__ jobs, int njobs) {
    using G = rows::Geo<LT, R, V, mm_lanes<LT, R, false>(), rows::MM_HB, rows::MM_VB>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int wi = threadIdx.x >> 5;
    const int nw = gridDim.x * rows::WARPS;
    for (int j = blockIdx.x * rows::WARPS + wi; j < njobs; j += nw) {  // warp-uniform
        const BatchJob job = jobs[j];
        const BatchMat& m = mats[job.mat];
        mm_range<LT, R, KC, V, X, A, Y, false>(m.nrows, m.brptr, m.headers, static_cast<const V*>(m.values),
                                               m.valptr, job.r_begin, job.r_end, nullptr, 0, 0,
                                               static_cast<const X*>(m.x) + job.kofs, m.ldx, 1L,
                                               static_cast<Y*>(m.y) + job.kofs, m.ldy, 1L,
                                               smem + wi * G::BUF_BYTES);
    }
}

template <class K>
void set_smem(K kernel, int bytes) {
    SPC5_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// Calls f(integral_constant<R>, integral_constant<KC>) for r in {1, 2, 4, 8}
// and kc a power of two up to mm_kc_limit of the kernel's lanes.
template <class LT, bool SEG, class F>
void dispatch_rkc(int r, int kc, F&& f) {
    using std::integral_constant;
    auto with_r = [&](auto RC) {
        constexpr int R_ = decltype(RC)::value;
        constexpr int KMAX = mm_kc_limit(Layout<LT>::VS, R_, mm_lanes<LT, R_, SEG>());
        switch (kc) {
            case 1: f(RC, integral_constant<int, 1>{}); return true;
            case 2: if constexpr (KMAX >= 2) { f(RC, integral_constant<int, 2>{}); return true; } break;
            case 4: if constexpr (KMAX >= 4) { f(RC, integral_constant<int, 4>{}); return true; } break;
            case 8: if constexpr (KMAX >= 8) { f(RC, integral_constant<int, 8>{}); return true; } break;
            case 16: if constexpr (KMAX >= 16) { f(RC, integral_constant<int, 16>{}); return true; } break;
        }
        return false;
    };
    bool done = false;
    switch (r) {
        case 1: done = with_r(integral_constant<int, 1>{}); break;
        case 2: done = with_r(integral_constant<int, 2>{}); break;
        case 4: done = with_r(integral_constant<int, 4>{}); break;
        case 8: done = with_r(integral_constant<int, 8>{}); break;
    }
    if (!done) throw Error(SPC5CUDA_ERR_INVALID, "unsupported (r, right-hand sides per pass)");
}

template <class LT, bool SEG, class V, class X, class A, class Y>
void spmm_rows_run(const BetaView& m, int k, const X* x, long ldx, long xcs, Y* y, long ldy, long ycs,
                   cudaStream_t s) {
    const int ctas = (m.nwarps + rows::WARPS - 1) / rows::WARPS;
    const V* vals = static_cast<const V*>(m.values);
    for (int k0 = 0; k0 < k;) {
        const int kc = spmm_rows_kc(Layout<LT>::VS, m.r, k - k0, SEG);
        dispatch_rkc<LT, SEG>(m.r, kc, [&](auto RC, auto KCC) {
            constexpr int R_ = decltype(RC)::value, KC_ = decltype(KCC)::value;
            constexpr int SMEM = rows::Geo<LT, R_, V, mm_lanes<LT, R_, SEG>(), rows::MM_HB, rows::MM_VB>::SMEM;
            auto kern = k_spmm_rows<LT, R_, KC_, V, X, A, Y, SEG>;
            set_smem(kern, SMEM);
            kern<<<ctas, rows::THREADS, SMEM, s>>>(m.nrows, m.brptr, m.headers, vals, m.valptr, m.wstart,
                                                   m.nwarps, m.perm, m.nseg, x + long(k0) * xcs, ldx, xcs,
                                                   y + long(k0) * ycs, ldy, ycs);
        });
        k0 += kc;
    }
}

template <class LT, class V, class X, class A, class Y>
void spmm_rows_impl(const BetaView& m, int k, const X* x, long ldx, long xcs, Y* y, long ldy, long ycs,
                    cudaStream_t s) {
    if (m.nbr <= 0 || k <= 0 || m.nwarps <= 0) return;
    if (m.nseg > 0) {
        if (m.lanes != seg_lanes(m.r)) throw Error(SPC5CUDA_ERR_INVALID, "segment lanes");
        spmm_rows_run<LT, true, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s);
    } else {
        spmm_rows_run<LT, false, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s);
    }
    SPC5_CUDA(cudaGetLastError());
}

template <class LT, class V, class X, class A, class Y>
void batch_rows_impl(int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs, int ctas,
                     cudaStream_t s) {
    dispatch_rkc<LT, false>(r, kc, [&](auto RC, auto KCC) {
        constexpr int R_ = decltype(RC)::value, KC_ = decltype(KCC)::value;
        constexpr int SMEM = rows::Geo<LT, R_, V, mm_lanes<LT, R_, false>(), rows::MM_HB, rows::MM_VB>::SMEM;
        auto kern = k_spmm_rows_batch<LT, R_, KC_, V, X, A, Y>;
        set_smem(kern, SMEM);
        int per_sm = 0;
        SPC5_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, rows::THREADS, SMEM));
        const int grid = std::max(1, std::min(ctas, sm_count() * std::max(1, per_sm)));
        kern<<<grid, rows::THREADS, SMEM, s>>>(mats, jobs, njobs);
    });
}

}  // namespace

int spmm_rows_kc(int vs, int r, int k, bool seg) {
    const int lanes = seg ? seg_lanes(r) : ((vs == 16 && r == 8) ? 16 : 8);
    const int kmax = mm_kc_limit(vs, r, lanes);
    int kc = 1;
    while (kc * 2 <= k && kc * 2 <= kmax) kc *= 2;
    return kc;
}

void launch_spmm_rows_f64(const BetaView& m, int k, const double* x, long ldx, long xcs, double* y, long ldy,
                          long ycs, cudaStream_t s) {
    spmm_rows_impl<double, double, double, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_rows_f32(const BetaView& m, int k, const float* x, long ldx, long xcs, float* y, long ldy,
                          long ycs, cudaStream_t s) {
    spmm_rows_impl<float, float, float, float, float>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_rows_mixed(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y, long ldy,
                            long ycs, cudaStream_t s) {
    spmm_rows_impl<float, float, float, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_rows_mixed8(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y, long ldy,
                             long ycs, cudaStream_t s) {
    spmm_rows_impl<double, float, float, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_batch_rows(int kind, int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs,
                       cudaStream_t s) {
    if (njobs <= 0) return;
    const int ctas = div_up(njobs, rows::WARPS);
    if (kind == 0)
        batch_rows_impl<double, double, double, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    else if (kind == 1)
        batch_rows_impl<float, float, float, float, float>(r, kc, mats, jobs, njobs, ctas, s);
    else if (kind == 2)
        batch_rows_impl<float, float, float, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    else
        batch_rows_impl<double, float, float, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    SPC5_CUDA(cudaGetLastError());
}

}  // namespace spc5cuda
