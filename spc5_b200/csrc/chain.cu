// chain.cu -- the largest block-rows of the length-sorted plan as exact
// multiply-add chains.
//
// In the reference kernels (core_SPC5_{r}rVc_Spmv_*, src/spc5.hpp:2309-2715)
// every (sub-row s, column c) of a block-row owns one accumulator, which
// receives fma(value, x[col + c], acc) for each block in order whose mask s
// has bit c; the row sum is the _mm512_reduce_add tree over the VS
// accumulators of the sub-row.  Those chains are independent of one another,
// so a block-row of thousands of blocks need not be walked block by block:
// the plan stores, for each chain, its values and x indices in chain order,
// and one lane runs one chain with no header decode and no empty column
// slots.  The chains are sorted by length class (lengths within about 1/8 of
// one another; chains of one class stay in chain-id order, so neighbouring
// lanes often run neighbouring columns of one sub-row) and
// cut into slices of 32 (one warp each, the longest first); entry j of the
// slice's lane l is at slice_off[slice] + 32 j + l, so a warp's value and
// index loads are coalesced and its lanes finish together.  Empty chains are
// not stored: a bit mask per sub-row marks its non-empty ones.  A second
// launch adds each sub-row's VS chain results (+0 for the empty ones, the
// reference's untouched accumulators) with the reduce tree into y.  Every
// chain runs the reference's multiply-adds in the reference's order: y is
// bit-identical for finite x.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "common.cuh"
#include "handle.h"
#include "kernels.h"

namespace spc5cuda {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;

// The SpMV chain kernel runs 8 entries per step.  For short chains (fewer
// than 16 entries on average: the part of a large r) it is compiled for 4
// resident CTAs per SM, so that more chains are in flight; long chains (small
// r) keep the registers for the next step's loads.  Measured on B200,
// power-law N = 4M, with the chain part for the block-rows above 8 lanes
// (r = 1 then ran chains too): r = 8 645 against 669 us, r = 1 540 against
// 576 us.
constexpr int CHAIN_U = 8;
constexpr int CHAIN_SHORT = 16;

__device__ __forceinline__ int hdr_col(const uint8_t* __restrict__ h) {
    return int(uint32_t(h[0]) | (uint32_t(h[1]) << 8) | (uint32_t(h[2]) << 16) | (uint32_t(h[3]) << 24));
}

// Mask of sub-row s of a packed header (mask bytes MB per sub-row).
template <int MB>
__device__ __forceinline__ uint32_t hdr_mask(const uint8_t* __restrict__ h, int s) {
    if constexpr (MB == 1) return h[4 + s];
    else return uint32_t(h[4 + 2 * s]) | (uint32_t(h[5 + 2 * s]) << 8);
}

// ---- build --------------------------------------------------------------

// Length class of a chain of n entries: n itself below 8, then four classes
// per octave (monotone in n; one class spans at most 1/8 of its lengths).
__device__ __forceinline__ int length_class(int n) {
    if (n < 8) return n;
    const int b = 31 - __clz(n);
    return 8 + 4 * (b - 3) + ((n >> (b - 2)) & 3);
}

// clen[(i r + s) VS + c] = blocks of block-row i whose mask s has bit c,
// ckey the same chain's length class; cmask[i r + s] bit c: that chain is
// not empty; *nonempty += their number.
template <int VS, int MB>
__global__ void k_chain_len(int nlong, int r, const int* __restrict__ brptr, const uint8_t* __restrict__ hdr,
                            int* __restrict__ clen, int* __restrict__ ckey, uint32_t* __restrict__ cmask,
                            int* __restrict__ nonempty) {
    const int stride = 4 + r * MB;
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < long(nlong) * r;
         t += long(gridDim.x) * blockDim.x) {
        const int i = int(t / r), s = int(t % r);
        int cnt[VS];
#pragma unroll
        for (int c = 0; c < VS; ++c) cnt[c] = 0;
        for (long b = brptr[i]; b < brptr[i + 1]; ++b) {
            const uint32_t m = hdr_mask<MB>(hdr + b * stride, s);
#pragma unroll
            for (int c = 0; c < VS; ++c) cnt[c] += int((m >> c) & 1u);
        }
        uint32_t mask = 0u;
#pragma unroll
        for (int c = 0; c < VS; ++c) {
            clen[t * VS + c] = cnt[c];
            ckey[t * VS + c] = length_class(cnt[c]);
            mask |= cnt[c] > 0 ? (1u << c) : 0u;
        }
        cmask[t] = mask;
        if (mask) atomicAdd(nonempty, __popc(mask));
    }
}

__global__ void k_chain_pos(long nchains, const int* __restrict__ corder, int* __restrict__ pos) {
    for (long p = long(blockIdx.x) * blockDim.x + threadIdx.x; p < nchains; p += long(gridDim.x) * blockDim.x)
        pos[corder[p]] = int(p);
}

// width[g] = 32 x the longest chain of slice g; width[nslices] = 0.
__global__ void k_slice_width(long nchains, int nslices, const int* __restrict__ slen, long* __restrict__ width) {
    for (long g = long(blockIdx.x) * blockDim.x + threadIdx.x; g <= nslices; g += long(gridDim.x) * blockDim.x) {
        int most = 0;
        for (long p = g * 32; p < min(nchains, g * 32 + 32); ++p) most = max(most, slen[p]);
        width[g] = 32L * most;
    }
}

// slen[p] = clen[order[p]] for the sorted positions p < n.
__global__ void k_gather_len(long n, const int* __restrict__ order, const int* __restrict__ clen,
                             int* __restrict__ slen) {
    for (long p = long(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += long(gridDim.x) * blockDim.x)
        slen[p] = clen[order[p]];
}

// Walks block-row i's blocks for sub-row s and calls f(entry, value offset,
// x index) for each of its values in block order: the value's offset in the
// block-row (from v0) and its chain entry.
template <int VS, int MB, class F>
__device__ __forceinline__ void walk_subrow(int r, int i, int s, const int* __restrict__ brptr,
                                            const uint8_t* __restrict__ hdr, const int* __restrict__ pos,
                                            const long* __restrict__ slice_off, long v0, F&& f) {
    const int stride = 4 + r * MB;
    const long t = long(i) * r + s;
    int p[VS], j[VS];
#pragma unroll
    for (int c = 0; c < VS; ++c) {
        p[c] = pos[t * VS + c];
        j[c] = 0;
    }
    long v = v0;
    for (long b = brptr[i]; b < brptr[i + 1]; ++b) {
        const uint8_t* h = hdr + b * stride;
        const int col = hdr_col(h);
        int below = 0, tot = 0;
        for (int q = 0; q < r; ++q) {
            const int pc = __popc(hdr_mask<MB>(h, q));
            below += q < s ? pc : 0;
            tot += pc;
        }
        const uint32_t m = hdr_mask<MB>(h, s);
        int k = 0;
#pragma unroll
        for (int c = 0; c < VS; ++c) {
            if ((m >> c) & 1u) {
                const long e = slice_off[p[c] >> 5] + 32L * j[c] + (p[c] & 31);
                f(e, v + below + k, col + c);
                ++k;
                ++j[c];
            }
        }
        v += tot;
    }
}

// The chain entries of every value of the sorted block-rows [0, nlong).
template <class V, int VS, int MB>
__global__ void k_chain_fill(int nlong, int r, const int* __restrict__ brptr, const int* __restrict__ valptr,
                             const uint8_t* __restrict__ hdr, const V* __restrict__ vals,
                             const int* __restrict__ pos, const long* __restrict__ slice_off, V* __restrict__ cval,
                             int* __restrict__ ccol) {
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < long(nlong) * r;
         t += long(gridDim.x) * blockDim.x) {
        const int i = int(t / r), s = int(t % r);
        walk_subrow<VS, MB>(r, i, s, brptr, hdr, pos, slice_off, valptr[i], [&](long e, long v, int x) {
            cval[e] = vals[v];
            ccol[e] = x;
        });
    }
}

// The reverse: the values of the sorted block-rows [0, nlong) back at their
// places in the reference order (block-row perm[i] at ref_valptr).
template <class V, int VS, int MB>
__global__ void k_chain_unfill(int nlong, int r, const int* __restrict__ brptr, const int* __restrict__ perm,
                               const int* __restrict__ ref_valptr, const uint8_t* __restrict__ hdr,
                               const int* __restrict__ pos, const long* __restrict__ slice_off,
                               const V* __restrict__ cval, V* __restrict__ vals) {
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < long(nlong) * r;
         t += long(gridDim.x) * blockDim.x) {
        const int i = int(t / r), s = int(t % r);
        walk_subrow<VS, MB>(r, i, s, brptr, hdr, pos, slice_off, ref_valptr[perm[i]],
                            [&](long e, long v, int) { vals[v] = cval[e]; });
    }
}

__global__ void k_sub_i32(long n, int* __restrict__ a, const int* __restrict__ base_at) {
    const int base = *base_at;
    for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += long(gridDim.x) * blockDim.x)
        a[k] -= base;
}

int grid_of(long n, int threads) { return std::max(1, std::min(div_up(n, threads), sm_count() * 8)); }

template <class T>
T* ptr(const Owned& o) { return static_cast<T*>(o.p); }

// ---- SpMV ---------------------------------------------------------------

// U entries of a chain: value and x index of entries j0 .. j0 + U - 1
// (those below len), streamed once.
template <class V, int U>
__device__ __forceinline__ void load_entries(const V* __restrict__ vp, const int* __restrict__ cp, int j0, int len,
                                             V (&v)[U], int (&col)[U]) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        v[u] = V(0);
        col[u] = 0;
        if (j0 + u < len) {
            v[u] = __ldcs(vp + 32L * (j0 + u));
            col[u] = __ldcs(cp + 32L * (j0 + u));
        }
    }
}

// One warp per slice, one lane per chain: acc_out[chain] = the chain's
// multiply-adds from +0 in entry order.  U entries per step; the next
// step's values and indices load while this step's x gathers are in flight.
template <class V, class X, class A, int U, int MINB>
__global__ void __launch_bounds__(256, MINB) k_chain_spmv(long nchains, int nslices, const int* __restrict__ slen,
                                                    const int* __restrict__ corder,
                                                    const long* __restrict__ slice_off, const V* __restrict__ cval,
                                                    const int* __restrict__ ccol, const X* __restrict__ x,
                                                    A* __restrict__ acc_out) {
    const int lane = threadIdx.x & 31;
    const long g = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (g >= nslices) return;  // warp-uniform
    const long p = g * 32 + lane;
    const bool live = p < nchains;
    const int len = live ? __ldg(slen + p) : 0;
    const int width = __reduce_max_sync(FULL, len);
    const long base = __ldg(slice_off + g) + lane;
    const V* vp = cval + base;
    const int* cp = ccol + base;
    const uint64_t pol = l2_evict_last_policy();
    A acc = A(0);
    V v[U];
    int col[U];
    load_entries<V, U>(vp, cp, 0, len, v, col);
    for (int j0 = 0; j0 < width; j0 += U) {
        X xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) xv[u] = (j0 + u < len) ? ld_x(x + col[u], pol) : X(0);
        V vn[U];
        int cn[U];
        load_entries<V, U>(vp, cp, j0 + U, len, vn, cn);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (j0 + u < len) acc = fma(A(v[u]), A(xv[u]), acc);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            v[u] = vn[u];
            col[u] = cn[u];
        }
    }
    if (live) acc_out[__ldg(corder + p)] = acc;
}

// y[perm[i] r + s] += the reduce tree (distance VS/2, ..., 1) over the VS
// chain results of sub-row s of block-row i.
template <class A, class Y, int VS>
__global__ void k_chain_rows(int nlong, int r, int nrows, const int* __restrict__ perm,
                             const uint32_t* __restrict__ cmask, const A* __restrict__ acc, Y* __restrict__ y) {
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < long(nlong) * r;
         t += long(gridDim.x) * blockDim.x) {
        const int i = int(t / r), s = int(t % r);
        const uint32_t mask = __ldg(cmask + t);
        A a[VS];
#pragma unroll
        for (int c = 0; c < VS; ++c) a[c] = ((mask >> c) & 1u) ? acc[t * VS + c] : A(0);
#pragma unroll
        for (int d = VS / 2; d >= 1; d >>= 1) {
#pragma unroll
            for (int c = 0; c < d; ++c) a[c] = a[c] + a[c + d];
        }
        const long row = long(__ldg(perm + i)) * r + s;
        if (row < nrows) y[row] = y[row] + Y(a[0]);
    }
}

// ---- SpMM ---------------------------------------------------------------

// As k_chain_spmv for the kc <= KC right-hand sides q of X (element (row,
// q) at x[row ldx + q xcs]): acc_out[chain KC + q].
template <class V, class X, class A, int KC, int U>
__global__ void __launch_bounds__(256) k_chain_spmm(long nchains, int nslices, const int* __restrict__ slen,
                                                    const int* __restrict__ corder,
                                                    const long* __restrict__ slice_off, const V* __restrict__ cval,
                                                    const int* __restrict__ ccol, int kc, const X* __restrict__ x,
                                                    long ldx, long xcs, A* __restrict__ acc_out) {
    const int lane = threadIdx.x & 31;
    const long g = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (g >= nslices) return;  // warp-uniform
    const long p = g * 32 + lane;
    const bool live = p < nchains;
    const int len = live ? __ldg(slen + p) : 0;
    const int width = __reduce_max_sync(FULL, len);
    const long base = __ldg(slice_off + g) + lane;
    const V* vp = cval + base;
    const int* cp = ccol + base;
    const uint64_t pol = l2_evict_last_policy();
    A acc[KC];
#pragma unroll
    for (int q = 0; q < KC; ++q) acc[q] = A(0);
    for (int j0 = 0; j0 < width; j0 += U) {
        V v[U];
        int col[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            v[u] = V(0);
            col[u] = 0;
            if (j0 + u < len) {
                v[u] = __ldcs(vp + 32L * (j0 + u));
                col[u] = __ldcs(cp + 32L * (j0 + u));
            }
        }
        X xv[U][KC];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const X* xr = x + long(col[u]) * ldx;
#pragma unroll
            for (int q = 0; q < KC; ++q) xv[u][q] = (j0 + u < len && q < kc) ? ld_x(xr + q * xcs, pol) : X(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (j0 + u < len) {
#pragma unroll
                for (int q = 0; q < KC; ++q)
                    if (q < kc) acc[q] = fma(A(v[u]), A(xv[u][q]), acc[q]);
            }
        }
    }
    if (live) {
        const long c = __ldg(corder + p);
#pragma unroll
        for (int q = 0; q < KC; ++q)
            if (q < kc) acc_out[c * KC + q] = acc[q];
    }
}

template <class A, class Y, int VS, int KC>
__global__ void k_chain_rows_mm(int nlong, int r, int nrows, int kc, const int* __restrict__ perm,
                                const uint32_t* __restrict__ cmask, const A* __restrict__ acc, Y* __restrict__ y,
                                long ldy, long ycs) {
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < long(nlong) * r * kc;
         t += long(gridDim.x) * blockDim.x) {
        const int q = int(t % kc);
        const long sr = t / kc;
        const int i = int(sr / r), s = int(sr % r);
        const uint32_t mask = __ldg(cmask + sr);
        A a[VS];
#pragma unroll
        for (int c = 0; c < VS; ++c) a[c] = ((mask >> c) & 1u) ? acc[(sr * VS + c) * KC + q] : A(0);
#pragma unroll
        for (int d = VS / 2; d >= 1; d >>= 1) {
#pragma unroll
            for (int c = 0; c < d; ++c) a[c] = a[c] + a[c + d];
        }
        const long row = long(__ldg(perm + i)) * r + s;
        if (row < nrows) {
            Y* yp = y + row * ldy + q * ycs;
            *yp = *yp + Y(a[0]);
        }
    }
}

template <class V, class X, class A, class Y, int VS>
void chain_spmv(const spc5cuda_mat* m, const SpmvPart& part, const X* x, Y* y, cudaStream_t s) {
    const int* perm = m->plan->perm.as<int>();
    PoolBuf acc(sizeof(A) * size_t(part.nseg) * size_t(m->r) * VS, s);  // indexed by chain id
    const int threads = 256;
    const int blocks = std::max(1, div_up(long(part.nslices) * 32, threads));
    auto kern = part.entries < CHAIN_SHORT * part.nchains ? k_chain_spmv<V, X, A, CHAIN_U, 4>
                                                          : k_chain_spmv<V, X, A, CHAIN_U, 1>;
    kern<<<blocks, threads, 0, s>>>(part.nchains, part.nslices, ptr<int>(part.slen), ptr<int>(part.corder),
                                    ptr<long>(part.slice_off), ptr<V>(part.cval), ptr<int>(part.ccol), x,
                                    acc.as<A>());
    SPC5_CUDA(cudaGetLastError());
    k_chain_rows<A, Y, VS><<<grid_of(long(part.nseg) * m->r, threads), threads, 0, s>>>(
        part.nseg, m->r, m->nrows, perm, ptr<uint32_t>(part.cmask), acc.as<A>(), y);
    SPC5_CUDA(cudaGetLastError());
}

template <class V, class X, class A, class Y, int VS, int KC, int U>
void chain_spmm_pass(const spc5cuda_mat* m, const SpmvPart& part, int kc, const X* x, long ldx, long xcs, Y* y,
                     long ldy, long ycs, A* acc, cudaStream_t s) {
    const int threads = 256;
    const int blocks = std::max(1, div_up(long(part.nslices) * 32, threads));
    k_chain_spmm<V, X, A, KC, U><<<blocks, threads, 0, s>>>(part.nchains, part.nslices, ptr<int>(part.slen),
                                                            ptr<int>(part.corder), ptr<long>(part.slice_off),
                                                            ptr<V>(part.cval), ptr<int>(part.ccol), kc, x, ldx,
                                                            xcs, acc);
    SPC5_CUDA(cudaGetLastError());
    k_chain_rows_mm<A, Y, VS, KC><<<grid_of(long(part.nseg) * m->r * kc, threads), threads, 0, s>>>(
        part.nseg, m->r, m->nrows, kc, m->plan->perm.as<int>(), ptr<uint32_t>(part.cmask), acc, y, ldy, ycs);
    SPC5_CUDA(cudaGetLastError());
}

template <class V, class X, class A, class Y, int VS>
void chain_spmm(const spc5cuda_mat* m, const SpmvPart& part, int k, const X* x, long ldx, long xcs, Y* y, long ldy,
                long ycs, cudaStream_t s) {
    constexpr int KC = 8;
    PoolBuf acc(sizeof(A) * size_t(part.nseg) * size_t(m->r) * VS * KC, s);  // indexed by chain id
    for (int q0 = 0; q0 < k; q0 += KC) {
        const int kc = std::min(KC, k - q0);
        if (kc <= 2)
            chain_spmm_pass<V, X, A, Y, VS, KC, 4>(m, part, kc, x + long(q0) * xcs, ldx, xcs, y + long(q0) * ycs, ldy,
                                                   ycs, acc.as<A>(), s);
        else
            chain_spmm_pass<V, X, A, Y, VS, KC, 2>(m, part, kc, x + long(q0) * xcs, ldx, xcs, y + long(q0) * ycs, ldy,
                                                   ycs, acc.as<A>(), s);
    }
}

template <class V, int VS, int MB>
void build_chains_t(spc5cuda_mat* m, SortedPlan* plan, SpmvPart& part, cudaStream_t s) {
    const int r = m->r;
    const int nlong = part.nseg;
    const long nids = long(nlong) * r * VS;  // chain ids, empty chains included
    const int* sbrptr = plan->sbrptr.as<int>();
    const uint8_t* shdr = plan->sheaders.as<uint8_t>();
    // ---- lengths, sorted (longest first, stable): the non-empty chains are
    // the first `nchains`
    DevBuf clen(sizeof(int) * size_t(nids), s), ids(sizeof(int) * size_t(nids), s);
    DevBuf ckey(sizeof(int) * size_t(nids), s), skey(sizeof(int) * size_t(nids), s);
    DevBuf order(sizeof(int) * size_t(nids), s);
    DevBuf nonempty(sizeof(int), s);
    SPC5_CUDA(cudaMemsetAsync(nonempty.p, 0, sizeof(int), s));
    part.cmask.alloc(sizeof(uint32_t) * size_t(long(nlong) * r));
    k_chain_len<VS, MB><<<grid_of(long(nlong) * r, 128), 128, 0, s>>>(
        nlong, r, sbrptr, shdr, clen.as<int>(), ckey.as<int>(), ptr<uint32_t>(part.cmask), nonempty.as<int>());
    SPC5_CUDA(cudaGetLastError());
    launch_iota(nids, ids.as<int>(), s);
    size_t temp = 0;
    SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, temp, ckey.as<int>(), skey.as<int>(), ids.as<int>(),
                                                        order.as<int>(), nids, 0, 32, s));
    {
        DevBuf tmp(temp, s);
        SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, temp, ckey.as<int>(), skey.as<int>(),
                                                            ids.as<int>(), order.as<int>(), nids, 0, 32, s));
    }
    int ne = 0;
    SPC5_CUDA(cudaMemcpyAsync(&ne, nonempty.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    const long nchains = ne;
    part.nchains = nchains;
    part.nslices = int((nchains + 31) / 32);
    part.slen.alloc(sizeof(int) * size_t(std::max(nchains, 1L)));
    part.corder.alloc(sizeof(int) * size_t(std::max(nchains, 1L)));
    if (nchains > 0) {
        SPC5_CUDA(cudaMemcpyAsync(part.corder.p, order.p, sizeof(int) * size_t(nchains), cudaMemcpyDeviceToDevice,
                                  s));
        k_gather_len<<<grid_of(nchains, 256), 256, 0, s>>>(nchains, order.as<int>(), clen.as<int>(),
                                                           ptr<int>(part.slen));
        SPC5_CUDA(cudaGetLastError());
    }
    // ---- slices: offsets of 32 x the longest chain of each
    DevBuf width(sizeof(long) * size_t(part.nslices + 1), s);
    part.slice_off.alloc(sizeof(long) * size_t(part.nslices + 1));
    k_slice_width<<<grid_of(part.nslices + 1L, 256), 256, 0, s>>>(nchains, part.nslices, ptr<int>(part.slen),
                                                                  width.as<long>());
    SPC5_CUDA(cudaGetLastError());
    temp = 0;
    SPC5_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, width.as<long>(), ptr<long>(part.slice_off),
                                            part.nslices + 1, s));
    {
        DevBuf tmp(temp, s);
        SPC5_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, temp, width.as<long>(), ptr<long>(part.slice_off),
                                                part.nslices + 1, s));
    }
    long entries = 0;
    SPC5_CUDA(cudaMemcpyAsync(&entries, ptr<long>(part.slice_off) + part.nslices, sizeof(long),
                              cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    // ---- the entries (padding slots stay unread); pos: sorted position of
    // each non-empty chain id
    DevBuf pos(sizeof(int) * size_t(std::max(nids, 1L)), s);
    k_chain_pos<<<grid_of(nchains, 256), 256, 0, s>>>(nchains, ptr<int>(part.corder), pos.as<int>());
    SPC5_CUDA(cudaGetLastError());
    int nvals = 0;
    SPC5_CUDA(cudaMemcpyAsync(&nvals, plan->svalptr.as<int>() + nlong, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    part.entries = nvals;  // the chain part's values (the svalptr prefix)
    part.cval.alloc(sizeof(V) * size_t(std::max(entries, 4L)));
    part.ccol.alloc(sizeof(int) * size_t(std::max(entries, 4L)));
    k_chain_fill<V, VS, MB><<<grid_of(long(nlong) * r, 128), 128, 0, s>>>(
        nlong, r, sbrptr, plan->svalptr.as<int>(), shdr, plan->svalues.as<V>(), pos.as<int>(),
        ptr<long>(part.slice_off), ptr<V>(part.cval), ptr<int>(part.ccol));
    SPC5_CUDA(cudaGetLastError());
    // ---- the sorted copy keeps the values of the other block-rows only
    int vbase = 0;
    SPC5_CUDA(cudaMemcpyAsync(&vbase, plan->svalptr.as<int>() + nlong, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    const long rest = m->nnz - vbase;
    Owned tail;
    tail.alloc(sizeof(V) * size_t(std::max(rest + 8, 4L)));
    if (rest > 0)
        SPC5_CUDA(cudaMemcpyAsync(tail.p, plan->svalues.as<V>() + vbase, sizeof(V) * size_t(rest),
                                  cudaMemcpyDeviceToDevice, s));
    const int nbr = m->nbr();
    DevBuf base(sizeof(int), s);
    SPC5_CUDA(cudaMemcpyAsync(base.p, plan->svalptr.as<int>() + nlong, sizeof(int), cudaMemcpyDeviceToDevice, s));
    k_sub_i32<<<grid_of(nbr + 1L, 256), 256, 0, s>>>(nbr + 1L, plan->svalptr.as<int>(), base.as<int>());
    SPC5_CUDA(cudaGetLastError());
    SPC5_CUDA(cudaStreamSynchronize(s));
    plan->svalues = std::move(tail);
}

template <class V, int VS, int MB>
void unchain_t(const spc5cuda_mat* m, const SpmvPart& part, void* values, cudaStream_t s) {
    const SortedPlan& p = *m->plan;
    const long nchains = part.nchains;
    DevBuf pos(sizeof(int) * size_t(std::max(long(part.nseg) * m->r * VS, 1L)), s);
    k_chain_pos<<<grid_of(nchains, 256), 256, 0, s>>>(nchains, ptr<int>(part.corder), pos.as<int>());
    SPC5_CUDA(cudaGetLastError());
    k_chain_unfill<V, VS, MB><<<grid_of(long(part.nseg) * m->r, 128), 128, 0, s>>>(
        part.nseg, m->r, p.sbrptr.as<int>(), p.perm.as<int>(), m->valptr.as<int>(), p.sheaders.as<uint8_t>(),
        pos.as<int>(), ptr<long>(part.slice_off), ptr<V>(part.cval), static_cast<V*>(values));
    SPC5_CUDA(cudaGetLastError());
    SPC5_CUDA(cudaStreamSynchronize(s));  // pos is freed on return
}

__global__ void k_iota(long n, int* __restrict__ a) {
    for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += long(gridDim.x) * blockDim.x)
        a[k] = int(k);
}

}  // namespace

void launch_iota(long n, int* a, cudaStream_t s) {
    if (n <= 0) return;
    k_iota<<<grid_of(n, 256), 256, 0, s>>>(n, a);
    SPC5_CUDA(cudaGetLastError());
}

void build_chains(spc5cuda_mat* m, SortedPlan* plan, SpmvPart& part, cudaStream_t s) {
    switch (m->value_type) {
        case SPC5CUDA_F64: build_chains_t<double, 8, 1>(m, plan, part, s); break;
        case SPC5CUDA_F32: build_chains_t<float, 16, 2>(m, plan, part, s); break;
        default: build_chains_t<float, 8, 1>(m, plan, part, s); break;
    }
}

void unchain_values(const spc5cuda_mat* m, const SpmvPart& part, void* values, cudaStream_t s) {
    switch (m->value_type) {
        case SPC5CUDA_F64: unchain_t<double, 8, 1>(m, part, values, s); break;
        case SPC5CUDA_F32: unchain_t<float, 16, 2>(m, part, values, s); break;
        default: unchain_t<float, 8, 1>(m, part, values, s); break;
    }
}

void chain_part_spmv(const spc5cuda_mat* m, const SpmvPart& part, const void* x, void* y, bool mixed,
                     cudaStream_t s) {
    if (m->value_type == SPC5CUDA_F64)
        chain_spmv<double, double, double, double, 8>(m, part, static_cast<const double*>(x),
                                                      static_cast<double*>(y), s);
    else if (m->value_type == SPC5CUDA_F32_V8)
        chain_spmv<float, float, double, double, 8>(m, part, static_cast<const float*>(x), static_cast<double*>(y),
                                                    s);
    else if (mixed)
        chain_spmv<float, float, double, double, 16>(m, part, static_cast<const float*>(x),
                                                     static_cast<double*>(y), s);
    else
        chain_spmv<float, float, float, float, 16>(m, part, static_cast<const float*>(x), static_cast<float*>(y), s);
}

void chain_part_spmm(const spc5cuda_mat* m, const SpmvPart& part, int k, const void* x, long ldx, long xcs, void* y,
                     long ldy, long ycs, bool mixed, cudaStream_t s) {
    if (m->value_type == SPC5CUDA_F64)
        chain_spmm<double, double, double, double, 8>(m, part, k, static_cast<const double*>(x), ldx, xcs,
                                                      static_cast<double*>(y), ldy, ycs, s);
    else if (m->value_type == SPC5CUDA_F32_V8)
        chain_spmm<float, float, double, double, 8>(m, part, k, static_cast<const float*>(x), ldx, xcs,
                                                    static_cast<double*>(y), ldy, ycs, s);
    else if (mixed)
        chain_spmm<float, float, double, double, 16>(m, part, k, static_cast<const float*>(x), ldx, xcs,
                                                     static_cast<double*>(y), ldy, ycs, s);
    else
        chain_spmm<float, float, float, float, 16>(m, part, k, static_cast<const float*>(x), ldx, xcs,
                                                   static_cast<float*>(y), ldy, ycs, s);
}

}  // namespace spc5cuda
