// spmm.cu -- multi-RHS SpMM on the beta(r,VS) format, Y += A X, k <= 16.
//
// Every right-hand side goes through exactly the arithmetic of the SpMV
// kernel (spmv.cu): lane c of a VS-lane group owns column c of every block of
// a block-row, one accumulator per (sub-row, right-hand side), blocks in order,
// then the _mm512_reduce_add tree over the VS lanes and y += sum.  Column j of
// the result is therefore bit-identical to an SpMV with column j of X, which
// is what lets the request loop coalesce independent requests into one
// launch and still return each request's solo result.
//
// X and Y are row-major with leading dimensions ldx, ldy (KC consecutive
// right-hand sides of one matrix row are contiguous), so the x gather of a
// lane is one vector load per block.  KC right-hand sides are handled per pass;
// larger k runs ceil(k / KC) passes over the matrix.
#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

namespace {

// Y += A X over block-rows [r_begin, r_end) of one matrix, for the VS-lane
// group this lane belongs to (has == false: the group idles).  Warp-uniform
// control flow: every lane of the warp executes the same collective
// operations, whatever its group's range.
template <class LT, int R, int KC, class V, class X, class A, class Y>
__device__ __forceinline__ void spmm_range(bool has, int nrows, const int* __restrict__ brptr,
                                           const uint8_t* __restrict__ headers,
                                           const V* __restrict__ values, int r_begin, int r_end,
                                           int v_begin, const X* __restrict__ xm, long ldx,
                                           long xcs, Y* __restrict__ ym, long ldy, long ycs) {
    constexpr int VS = Layout<LT>::VS;
    using H = Header<LT, R>;
    constexpr int MW = H::MASK_WORDS;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int c = lane & (VS - 1);
    const uint32_t below = (1u << c) - 1u;
    if (!has) r_end = r_begin;
    int b = has ? __ldg(brptr + r_begin) : 0;
    const int b_stop = has ? __ldg(brptr + r_end) : 0;
    int v = v_begin;
    int row = r_begin;
    int rend = has ? __ldg(brptr + r_begin + 1) : 0x7fffffff;

    A acc[R][KC];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int q = 0; q < KC; ++q) acc[i][q] = A(0);

    // warp-uniform flush of every group whose block-row ends at block pos
    auto flush_while = [&](bool active, int pos) {
        for (;;) {
            const bool need = active && row < r_end && pos == rend;
            if (!__any_sync(FULL, need)) break;
#pragma unroll
            for (int i = 0; i < R; ++i) {
#pragma unroll
                for (int q = 0; q < KC; ++q) {
                    A s = acc[i][q];
#pragma unroll
                    for (int d = VS / 2; d >= 1; d >>= 1) s += __shfl_xor_sync(FULL, s, d, VS);
                    const int yrow = row * R + i;
                    if (need && ((i * KC + q) % VS) == c && yrow < nrows) {
                        Y* dst = ym + long(yrow) * ldy + long(q) * ycs;
                        if constexpr (sizeof(Y) == 8) atomicAdd(dst, Y(s));
                        else *dst = *dst + Y(s);
                    }
                }
            }
            if (need) {
#pragma unroll
                for (int i = 0; i < R; ++i)
#pragma unroll
                    for (int q = 0; q < KC; ++q) acc[i][q] = A(0);
                ++row;
                rend = row < r_end ? __ldg(brptr + row + 1) : 0x7fffffff;
            }
        }
    };

    while (__any_sync(FULL, b < b_stop)) {
        const int n = b < b_stop ? min(VS, b_stop - b) : 0;
        uint32_t mw[MW];
        int col = 0;
#pragma unroll
        for (int q = 0; q < MW; ++q) mw[q] = 0u;
        if (c < n) col = load_header<LT, R>(headers, long(b + c), mw);
        int tot = 0;
#pragma unroll
        for (int q = 0; q < MW; ++q) tot += __popc(mw[q]);
        int incl = tot;
#pragma unroll
        for (int d = 1; d < VS; d <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, d, VS);
            if (c >= d) incl += t;
        }
        const int voff = v + incl - tot;
        for (int j = 0; j < VS; ++j) {
            if (!__any_sync(FULL, j < n)) break;
            const bool act = j < n;
            uint32_t bm[MW];
#pragma unroll
            for (int q = 0; q < MW; ++q) bm[q] = __shfl_sync(FULL, mw[q], j, VS);
            const int bcol = __shfl_sync(FULL, col, j, VS);
            const int bv = __shfl_sync(FULL, voff, j, VS);
            flush_while(act, b + j);
            if (!act) continue;
            uint32_t lanes = 0;
#pragma unroll
            for (int i = 0; i < R; ++i) lanes |= mask_of<LT, R>(bm, i);
            if (!((lanes >> c) & 1u)) continue;
            A xk[KC];
            const X* xr = xm + long(bcol + c) * ldx;
#pragma unroll
            for (int q = 0; q < KC; ++q) xk[q] = A(__ldg(xr + long(q) * xcs));
            int pre = bv;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const uint32_t m = mask_of<LT, R>(bm, i);
                if ((m >> c) & 1u) {
                    const A e = A(__ldg(values + pre + __popc(m & below)));
#pragma unroll
                    for (int q = 0; q < KC; ++q) acc[i][q] = fma(e, xk[q], acc[i][q]);
                }
                pre += __popc(m);
            }
        }
        const int wtot = __shfl_sync(FULL, incl, VS - 1, VS);
        if (n > 0) {
            v += wtot;
            b += n;
        }
    }
    for (;;) {
        const bool need = row < r_end;
        if (!__any_sync(FULL, need)) break;
        flush_while(need, need ? rend : -1);
    }
}

template <class LT, int R, int KC, class V, class X, class A, class Y>
__global__ void __launch_bounds__(128)
    k_spmm(int nrows, const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
           const V* __restrict__ values, const int* __restrict__ valptr,
           const int* __restrict__ gstart, int ngroups, const X* __restrict__ xm, long ldx,
           long xcs, Y* __restrict__ ym, long ldy, long ycs) {
    constexpr int VS = Layout<LT>::VS;
    const int group = int((long(blockIdx.x) * blockDim.x + threadIdx.x) / VS);
    int r_begin = 0, r_end = 0;
    if (group < ngroups) {
        r_begin = __ldg(gstart + group);
        r_end = __ldg(gstart + group + 1);
    }
    if (!__any_sync(0xffffffffu, r_begin < r_end)) return;
    const bool has = r_begin < r_end;
    const int v_begin = has ? __ldg(valptr + r_begin) : 0;
    spmm_range<LT, R, KC, V, X, A, Y>(has, nrows, brptr, headers, values, r_begin, r_end, v_begin,
                                      xm, ldx, xcs, ym, ldy, ycs);
}

// Batched launch: job j is block-rows [r_begin, r_end) of matrix mats[j.mat]
// for right-hand sides [kofs, kofs + KC).  Groups walk the job list with the
// grid's group count as stride; each job is about the same number of blocks.
template <class LT, int R, int KC, class V, class X, class A, class Y>
__global__ void __launch_bounds__(128)
    k_spmm_batch(const BatchMat* __restrict__ mats, const BatchJob* __restrict__ jobs, int njobs) {
    constexpr int VS = Layout<LT>::VS;
    const int group = int((long(blockIdx.x) * blockDim.x + threadIdx.x) / VS);
    const int ngroups = int((long(gridDim.x) * blockDim.x) / VS);
    for (int base = 0; base < njobs; base += ngroups) {
        const int j = base + group;
        const bool has = j < njobs;
        BatchJob job{0, 0, 0, 0};
        BatchMat m{};
        if (has) {
            job = jobs[j];
            m = mats[job.mat];
        }
        const int v_begin = has ? __ldg(m.valptr + job.r_begin) : 0;
        spmm_range<LT, R, KC, V, X, A, Y>(
            has, m.nrows, m.brptr, m.headers, static_cast<const V*>(m.values), job.r_begin, job.r_end,
            v_begin, static_cast<const X*>(m.x) + long(job.kofs) * m.xcs, m.ldx, m.xcs,
            static_cast<Y*>(m.y) + long(job.kofs) * m.ycs, m.ldy, m.ycs);
    }
}

// KC right-hand sides per pass, bounded so that R * KC accumulators stay in
// registers.
template <int R>
constexpr int kc_max() {
    return R >= 8 ? 4 : (R >= 4 ? 8 : 16);
}

template <class LT, int R, int KC, class V, class X, class A, class Y>
void launch_kc(const BetaView& m, const X* x, long ldx, long xcs, Y* y, long ldy, long ycs,
               cudaStream_t s) {
    constexpr int VS = Layout<LT>::VS;
    const int threads = 128;
    const int ctas = int((long(m.ngroups) * VS + threads - 1) / threads);
    k_spmm<LT, R, KC, V, X, A, Y><<<ctas, threads, 0, s>>>(m.nrows, m.brptr, m.headers,
                                                            static_cast<const V*>(m.values), m.valptr,
                                                            m.gstart, m.ngroups, x, ldx, xcs, y, ldy,
                                                            ycs);
}

template <class LT, int R, class V, class X, class A, class Y>
void launch_r(const BetaView& m, int k, const X* x, long ldx, long xcs, Y* y, long ldy, long ycs,
              cudaStream_t s) {
    constexpr int KMAX = kc_max<R>();
    int k0 = 0;
    while (k0 < k) {
        const int rem = k - k0;
        const X* xs = x + long(k0) * xcs;
        Y* ys = y + long(k0) * ycs;
        if (rem >= KMAX) {
            launch_kc<LT, R, KMAX, V, X, A, Y>(m, xs, ldx, xcs, ys, ldy, ycs, s);
            k0 += KMAX;
        } else if (rem >= 8 && KMAX >= 8) {
            launch_kc<LT, R, (KMAX >= 8 ? 8 : 1), V, X, A, Y>(m, xs, ldx, xcs, ys, ldy, ycs, s);
            k0 += 8;
        } else if (rem >= 4) {
            launch_kc<LT, R, 4, V, X, A, Y>(m, xs, ldx, xcs, ys, ldy, ycs, s);
            k0 += 4;
        } else if (rem >= 2) {
            launch_kc<LT, R, 2, V, X, A, Y>(m, xs, ldx, xcs, ys, ldy, ycs, s);
            k0 += 2;
        } else {
            launch_kc<LT, R, 1, V, X, A, Y>(m, xs, ldx, xcs, ys, ldy, ycs, s);
            k0 += 1;
        }
    }
    SPC5_CUDA(cudaGetLastError());
}

template <class LT, class V, class X, class A, class Y>
void launch_spmm_impl(const BetaView& m, int k, const X* x, long ldx, long xcs, Y* y, long ldy,
                      long ycs, cudaStream_t s) {
    if (m.nbr <= 0 || k <= 0) return;
    switch (m.r) {
        case 1: launch_r<LT, 1, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s); break;
        case 2: launch_r<LT, 2, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s); break;
        case 4: launch_r<LT, 4, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s); break;
        case 8: launch_r<LT, 8, V, X, A, Y>(m, k, x, ldx, xcs, y, ldy, ycs, s); break;
        default: throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    }
}

}  // namespace

void launch_spmm_f64(const BetaView& m, int k, const double* x, long ldx, long xcs, double* y,
                     long ldy, long ycs, cudaStream_t s) {
    if (m.wstart) return launch_spmm_rows_f64(m, k, x, ldx, xcs, y, ldy, ycs, s);
    launch_spmm_impl<double, double, double, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_f32(const BetaView& m, int k, const float* x, long ldx, long xcs, float* y,
                     long ldy, long ycs, cudaStream_t s) {
    if (m.wstart) return launch_spmm_rows_f32(m, k, x, ldx, xcs, y, ldy, ycs, s);
    launch_spmm_impl<float, float, float, float, float>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_mixed(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                       long ldy, long ycs, cudaStream_t s) {
    if (m.wstart) return launch_spmm_rows_mixed(m, k, x, ldx, xcs, y, ldy, ycs, s);
    launch_spmm_impl<float, float, float, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

void launch_spmm_mixed8(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                        long ldy, long ycs, cudaStream_t s) {
    if (m.wstart) return launch_spmm_rows_mixed8(m, k, x, ldx, xcs, y, ldy, ycs, s);
    launch_spmm_impl<double, float, float, double, double>(m, k, x, ldx, xcs, y, ldy, ycs, s);
}

int batch_kc(int r, int k) {
    const int kmax = r >= 8 ? 4 : (r >= 4 ? 8 : 16);
    int kc = 1;
    while (kc * 2 <= k && kc * 2 <= kmax) kc *= 2;
    return kc;
}

namespace {

template <class LT, int R, class V, class X, class A, class Y>
void batch_r(int kc, const BatchMat* mats, const BatchJob* jobs, int njobs, int ctas, cudaStream_t s) {
#define SPC5_BATCH(KC_)                                                                      \
    k_spmm_batch<LT, R, KC_, V, X, A, Y><<<ctas, 128, 0, s>>>(mats, jobs, njobs);
    switch (kc) {
        case 1: SPC5_BATCH(1); break;
        case 2: SPC5_BATCH(2); break;
        case 4: SPC5_BATCH(4); break;
        case 8:
            if constexpr (R <= 4) { SPC5_BATCH(8); } else throw Error(SPC5CUDA_ERR_INVALID, "kc");
            break;
        case 16:
            if constexpr (R <= 2) { SPC5_BATCH(16); } else throw Error(SPC5CUDA_ERR_INVALID, "kc");
            break;
        default: throw Error(SPC5CUDA_ERR_INVALID, "kc must be 1, 2, 4, 8 or 16");
    }
#undef SPC5_BATCH
}

template <class LT, class V, class X, class A, class Y>
void batch_impl(int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs, int ctas,
                cudaStream_t s) {
    switch (r) {
        case 1: batch_r<LT, 1, V, X, A, Y>(kc, mats, jobs, njobs, ctas, s); break;
        case 2: batch_r<LT, 2, V, X, A, Y>(kc, mats, jobs, njobs, ctas, s); break;
        case 4: batch_r<LT, 4, V, X, A, Y>(kc, mats, jobs, njobs, ctas, s); break;
        case 8: batch_r<LT, 8, V, X, A, Y>(kc, mats, jobs, njobs, ctas, s); break;
        default: throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    }
}

}  // namespace

void launch_batch(int kind, int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs,
                  int ctas, cudaStream_t s) {
    if (njobs <= 0) return;
    if (kind == 0)
        batch_impl<double, double, double, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    else if (kind == 1)
        batch_impl<float, float, float, float, float>(r, kc, mats, jobs, njobs, ctas, s);
    else if (kind == 2)
        batch_impl<float, float, float, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    else
        batch_impl<double, float, float, double, double>(r, kc, mats, jobs, njobs, ctas, s);
    SPC5_CUDA(cudaGetLastError());
}

}  // namespace spc5cuda
