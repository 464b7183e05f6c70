// spmv.cu -- beta(r,VS) SpMV kernels, y += A x.
//
// Arithmetic (bit-identical to the reference): one group of VS lanes (8 for
// f64, 16 for f32 / mixed) owns a block-row at a time; lane c owns column c
// of every block, with one accumulator per sub-row.  This is the lane
// structure of the reference AVX-512 kernels (core_SPC5_{r}rVc_Spmv_{double,
// float}, src/spc5.hpp:2309-2715): for every sub-row whose mask has bit c the
// lane fetches the value at the sub-row's compact offset plus
// popcount(mask & lanes-below-c) (the expand-load) and does a fused
// multiply-add with x[col + c] into that sub-row's accumulator.  Blocks are
// visited in order, so every (sub-row, lane) accumulator is the same FMA
// chain as the reference's vector lane; the row sum is the butterfly over
// lane distance VS/2 ... 1, which is the _mm512_reduce_add_{pd,ps} tree, and
// y[row] += sum.  A lane whose bit is clear skips the FMA: the reference adds
// fma(0, x, acc) there, which leaves acc unchanged for finite x (acc starts
// at +0.0 and is never -0.0 in round-to-nearest), so y is bit-identical for
// finite x.
//
// Work split (replaces the OpenMP ThreadInterval split, spc5.hpp:346-427):
// every group gets one contiguous range of block-rows holding about
// nblocks / groups blocks (gstart[], built on the device).  A group streams
// its range in chunks of VS blocks: lane j loads the packed header of block
// j of the chunk (consecutive records, one coalesced access), the group
// scans the per-block value counts to get each block's value offset, and the
// next chunk's headers and row ends are loaded before the current chunk is
// processed.  Values and headers are read once (streaming loads, evict
// first); x goes through L1/L2.
#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

namespace {

constexpr int SPMV_CTAS_PER_SM = 16;

template <int VS>
__device__ __forceinline__ unsigned group_mask(int lane) {
    return (VS == 32 ? 0xffffffffu : ((1u << VS) - 1u)) << (lane & ~(VS - 1));
}

// Streaming 32-bit load of header words (read once).
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p) { return __ldcs(p); }

template <class V>
__device__ __forceinline__ V ld_stream(const V* p) {
    return __ldcs(p);
}

// Header of block b decoded from aligned 32-bit words (each word holds at
// least one byte of the record, so none reads past the array).
template <class LT, int R>
__device__ __forceinline__ int load_header_stream(const uint8_t* __restrict__ hdr, long b,
                                                  uint32_t (&mw)[Header<LT, R>::MASK_WORDS]) {
    using H = Header<LT, R>;
    const long off = b * H::STRIDE;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(hdr) + (off >> 2);
    uint32_t lw[H::LOAD_WORDS + 1];
#pragma unroll
    for (int k = 0; k < H::LOAD_WORDS; ++k) lw[k] = ld_stream_u32(w + k);
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

// Asynchronous 16-byte global -> shared copy (cached in L2 only).
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* gptr) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gptr) : "memory");
}

// Asynchronous 4- or 8-byte global -> shared copy (cached in L1: x is reused).
template <int BYTES>
__device__ __forceinline__ void cp_async_small(uint32_t saddr, const void* gptr) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(saddr), "l"(gptr), "n"(BYTES)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Waits until at most one committed group of this thread is still in flight.
__device__ __forceinline__ void cp_async_wait_prev() {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Byte-wise population count of a 32-bit word (SWAR).
__device__ __forceinline__ uint32_t popc_bytes(uint32_t w) {
    w = w - ((w >> 1) & 0x55555555u);
    w = (w & 0x33333333u) + ((w >> 2) & 0x33333333u);
    return (w + (w >> 4)) & 0x0F0F0F0Fu;
}

// OR of the r masks of one block folded onto the VS lane bits.
template <class LT, int R>
__device__ __forceinline__ uint32_t lanes_of(const uint32_t (&mw)[Header<LT, R>::MASK_WORDS]) {
    uint32_t w = 0;
#pragma unroll
    for (int q = 0; q < Header<LT, R>::MASK_WORDS; ++q) w |= mw[q];
    if constexpr (Layout<LT>::MASK_BYTES == 1) {
        w |= w >> 16;
        w |= w >> 8;
        return w & 0xFFu;
    } else {
        w |= w >> 16;
        return w & 0xFFFFu;
    }
}

// Geometry of the kernel: a group of VS lanes (lane c = column c of every
// block) owns one block-row stream; GPW groups per warp run in lockstep.
template <class LT, int R, class V, class X, class A>
struct Geo {
    static constexpr int VS = Layout<LT>::VS;
    static constexpr int THREADS = 128;
    static constexpr int GPW = 32 / VS;                      // groups per warp
    static constexpr int GPC = THREADS / VS;                 // groups per CTA
    static constexpr int EPU = 16 / int(sizeof(V));          // values per 16-byte unit
    static constexpr int CAP = 1024 / int(sizeof(V));        // staged values per window
    static constexpr int VBUF = CAP + 2 * EPU;               // + alignment slack
    static constexpr int VBYTES = VBUF * int(sizeof(V));
    static constexpr int XBYTES = VS * VS * int(sizeof(X));  // x of one window: [block][column]
    static constexpr int BUF_BYTES = (VBYTES + XBYTES + 15) / 16 * 16;
    static constexpr int RED_BYTES = R > 1 ? (R * VS * int(sizeof(A)) + 15) / 16 * 16 : 0;
    static constexpr int GROUP_BYTES = 2 * BUF_BYTES + RED_BYTES;  // double-buffered windows
    static constexpr int SMEM = GPC * GROUP_BYTES;
    static constexpr int MW = Header<LT, R>::MASK_WORDS;
    static constexpr int PW = (R + 3) / 4;                   // packed sub-row prefixes
    static_assert(CAP >= VS * R, "a block must fit one window");
};

// One window of a group: lane j describes block j of the window (j < n).
template <class LT, int R>
struct Win {
    static constexpr int MW = Header<LT, R>::MASK_WORDS;
    static constexpr int PW = (R + 3) / 4;
    uint32_t mw[MW];
    uint32_t pre[PW];  // exclusive prefix of the sub-row value counts, one byte per sub-row
    int voff;          // staging-buffer index of the block's first value
    int n;             // blocks in the window (group-uniform)
};

// Headers of up to VS blocks starting at block p: lane j holds block p + j.
template <class LT, int R>
struct Raw {
    uint32_t mw[Header<LT, R>::MASK_WORDS];
    int col;
    bool ok;
};

template <class LT, int R>
__device__ __forceinline__ void load_raw(Raw<LT, R>& rw, const uint8_t* __restrict__ headers, int p,
                                         int b_stop, int j) {
    rw.ok = p + j < b_stop;
    rw.col = 0;
#pragma unroll
    for (int q = 0; q < Header<LT, R>::MASK_WORDS; ++q) rw.mw[q] = 0u;
    if (rw.ok) rw.col = load_header_stream<LT, R>(headers, long(p + j), rw.mw);
}

template <class LT, int R, class V, class X, class A, class Y>
__global__ void __launch_bounds__(128)
    k_spmv(int nrows, const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
           const V* __restrict__ values, const int* __restrict__ valptr,
           const int* __restrict__ gstart, int ngroups, const X* __restrict__ x,
           Y* __restrict__ y) {
    using G = Geo<LT, R, V, X, A>;
    constexpr int VS = G::VS, MW = G::MW, PW = G::PW;
    constexpr int MB = Layout<LT>::MASK_BYTES;
    constexpr bool Y_ATOMIC = sizeof(Y) == 8;  // red.add.f64 is y + s rounded once
    constexpr unsigned FULL = 0xffffffffu;
    constexpr unsigned VSMASK = (VS == 32) ? FULL : ((1u << VS) - 1u);
    extern __shared__ __align__(16) unsigned char smem[];

    const int lane = threadIdx.x & 31;
    const int c = lane & (VS - 1);
    const int gbase_lane = lane & ~(VS - 1);
    const uint32_t below = (1u << c) - 1u;
    const int gi = threadIdx.x / VS;
    const int group = blockIdx.x * G::GPC + gi;
    const uint32_t sgroup = uint32_t(__cvta_generic_to_shared(smem)) + uint32_t(gi * G::GROUP_BYTES);
    unsigned char* pgroup = smem + gi * G::GROUP_BYTES;
    A* red = reinterpret_cast<A*>(pgroup + 2 * G::BUF_BYTES);

    int r_begin = 0, r_end = 0;
    if (group < ngroups) {
        r_begin = __ldg(gstart + group);
        r_end = __ldg(gstart + group + 1);
    }
    if (!__any_sync(FULL, r_begin < r_end)) return;
    const bool has = r_begin < r_end;
    const int b_stop = has ? __ldg(brptr + r_end) : 0;
    int p = has ? __ldg(brptr + r_begin) : 0;  // first block of the next window to stage
    int v_next = has ? __ldg(valptr + r_begin) : 0;

    // row bookkeeping: current block-row row = rbase + k, rend = its end block
    int row = r_begin, rbase = r_begin, k = 0;
    int ends = (has && rbase + 1 + c <= r_end) ? __ldg(brptr + rbase + 1 + c) : 0x7fffffff;
    int ends_nxt = (has && rbase + 1 + VS + c <= r_end) ? __ldg(brptr + rbase + 1 + VS + c) : 0x7fffffff;
    int rend = __shfl_sync(FULL, ends, 0, VS);
    Y ycur = Y(0);
    if (!Y_ATOMIC && has && c < R && row * R + c < nrows) ycur = y[row * R + c];

    A acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = A(0);

    // Flush every group whose current block-row ends at block position pos,
    // repeating for empty block-rows; warp-uniform control flow.  The row sum
    // is the _mm512_reduce_add tree over the VS lane accumulators: distance
    // VS/2 first, then VS/4, ..., 1.
    auto flush_while = [&](bool active, int pos) {
        for (;;) {
            const bool need = active && row < r_end && pos == rend;
            if (!__any_sync(FULL, need)) break;
            A s = A(0);
            if constexpr (R == 1) {
                s = acc[0];
#pragma unroll
                for (int d = VS / 2; d >= 1; d >>= 1) s += __shfl_xor_sync(FULL, s, d, VS);
            } else {
                if (need) {
#pragma unroll
                    for (int i = 0; i < R; ++i) red[i * VS + c] = acc[i];
                }
                __syncwarp();
                if (need && c < R) {
                    A a[VS];
#pragma unroll
                    for (int e = 0; e < VS; ++e) a[e] = red[c * VS + e];
#pragma unroll
                    for (int d = VS / 2; d >= 1; d >>= 1) {
#pragma unroll
                        for (int e = 0; e < d; ++e) a[e] = a[e] + a[e + d];
                    }
                    s = a[0];
                }
                __syncwarp();
            }
            if (need) {
                const int yrow = row * R + c;
                if (c < R && yrow < nrows) {
                    if constexpr (Y_ATOMIC) atomicAdd(y + yrow, Y(s));
                    else y[yrow] = ycur + Y(s);
                }
#pragma unroll
                for (int i = 0; i < R; ++i) acc[i] = A(0);
                ++row;
                if (++k == VS) {
                    k = 0;
                    rbase += VS;
                    ends = ends_nxt;
                    ends_nxt = (rbase + 1 + VS + c <= r_end) ? __ldg(brptr + rbase + 1 + VS + c) : 0x7fffffff;
                }
                if constexpr (!Y_ATOMIC) {
                    const int ynext = row * R + c;
                    if (c < R && row < r_end && ynext < nrows) ycur = y[ynext];
                }
            }
            rend = __shfl_sync(FULL, ends, k, VS);
        }
    };

    // ---- stage one window: headers rw (blocks p ...) -> win; values and x into buffer bi
    auto stage = [&](const Raw<LT, R>& rw, Win<LT, R>& win, int bi) {
        int tot = 0;
#pragma unroll
        for (int q = 0; q < MW; ++q) tot += __popc(rw.mw[q]);
        if (!rw.ok) tot = 0;
        int incl = tot;
#pragma unroll
        for (int d = 1; d < VS; d <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, d, VS);
            if (c >= d) incl += t;
        }
        const int n = __popc((__ballot_sync(FULL, rw.ok && incl <= G::CAP) >> gbase_lane) & VSMASK);
        const int tv = __shfl_sync(FULL, incl, (n > 0 ? n : 1) - 1, VS);
        const int s0 = v_next & ~(G::EPU - 1);
        const int shift = v_next - s0;
        win.n = n;
#pragma unroll
        for (int q = 0; q < MW; ++q) win.mw[q] = rw.mw[q];
        win.voff = shift + incl - tot;
        {
            uint32_t run = 0;
#pragma unroll
            for (int q = 0; q < PW; ++q) win.pre[q] = 0u;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                win.pre[i >> 2] |= run << ((i & 3) * 8);
                run += __popc(mask_of<LT, R>(rw.mw, i));
            }
        }
        const uint32_t vb = sgroup + uint32_t(bi * G::BUF_BYTES);
        if (n > 0) {
            const int units = (shift + tv + G::EPU - 1) / G::EPU;
            const V* src = values + s0;
            for (int u = c; u < units; u += VS) cp_async16(vb + uint32_t(u) * 16u, src + u * G::EPU);
        }
        // x: lane c copies column c of every block that holds a value there
        {
            const uint32_t lor = lanes_of<LT, R>(rw.mw);
            const uint32_t xb = vb + uint32_t(G::VBYTES) + uint32_t(c) * uint32_t(sizeof(X));
#pragma unroll
            for (int j = 0; j < VS; ++j) {
                const int cj = __shfl_sync(FULL, rw.col, j, VS);
                const uint32_t lj = __shfl_sync(FULL, lor, j, VS);
                if (j < n && ((lj >> c) & 1u))
                    cp_async_small<int(sizeof(X))>(xb + uint32_t(j * VS) * uint32_t(sizeof(X)), x + (cj + c));
            }
        }
        cp_async_commit();
        v_next += (n > 0) ? tv : 0;
        p += n;
    };

    // ---- prologue: stage window 0, load the headers of window 1
    Raw<LT, R> raw;
    load_raw<LT, R>(raw, headers, p, b_stop, c);
    Win<LT, R> cur;
    int wstart = p;  // first block of the current window
    stage(raw, cur, 0);
    load_raw<LT, R>(raw, headers, p, b_stop, c);
    int bi = 0;

    while (__any_sync(FULL, cur.n > 0)) {
        Win<LT, R> nxt;
        const int nstart = p;
        stage(raw, nxt, bi ^ 1);
        load_raw<LT, R>(raw, headers, p, b_stop, c);

        // block positions of this window where a block-row of some group ends
        // (known row ends: ends of rows rbase+1 .. rbase+VS, ends_nxt beyond);
        // positions past the last known end are checked individually.
        uint32_t rmask;
        {
            const int rel = ends - wstart;
            uint32_t mine = (rel >= 0 && rel < VS) ? (1u << rel) : 0u;
            const int last = __shfl_sync(FULL, ends_nxt, VS - 1, VS);
            const int lrel = last - wstart;
            if (c == 0 && lrel < VS) mine |= VSMASK << (lrel < 0 ? 0 : lrel);
            const int rel2 = ends_nxt - wstart;
            if (rel2 >= 0 && rel2 < VS) mine |= 1u << rel2;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) mine |= __shfl_xor_sync(FULL, mine, d);
            rmask = mine;
        }
        cp_async_wait_prev();
        __syncwarp();

        const V* vbuf = reinterpret_cast<const V*>(pgroup + bi * G::BUF_BYTES);
        const X* xbuf = reinterpret_cast<const X*>(pgroup + bi * G::BUF_BYTES + G::VBYTES);
#pragma unroll
        for (int j = 0; j < VS; ++j) {
            if (!__any_sync(FULL, j < cur.n)) break;
            const bool act = j < cur.n;
            uint32_t bm[MW];
#pragma unroll
            for (int q = 0; q < MW; ++q) bm[q] = __shfl_sync(FULL, cur.mw[q], j, VS);
            uint32_t bp[PW];
#pragma unroll
            for (int q = 0; q < PW; ++q) bp[q] = __shfl_sync(FULL, cur.pre[q], j, VS);
            const int voff = __shfl_sync(FULL, cur.voff, j, VS);
            if ((rmask >> j) & 1u) flush_while(act, wstart + j);
            if (act) {
                const A xv = A(xbuf[j * VS + c]);
                if constexpr (MB == 1 && R >= 2) {
#pragma unroll
                    for (int q = 0; q < MW; ++q) {
                        const uint32_t Q = bp[q] + popc_bytes(bm[q] & (below * 0x01010101u));
#pragma unroll
                        for (int ii = 0; ii < 4; ++ii) {
                            const int i = q * 4 + ii;
                            if (i < R && ((bm[q] >> (ii * 8 + c)) & 1u))
                                acc[i] = fma(A(vbuf[voff + int((Q >> (ii * 8)) & 0xFFu)]), xv, acc[i]);
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < R; ++i) {
                        const uint32_t m = mask_of<LT, R>(bm, i);
                        if ((m >> c) & 1u) {
                            const int idx = voff + int((bp[i >> 2] >> ((i & 3) * 8)) & 0xFFu) + __popc(m & below);
                            acc[i] = fma(A(vbuf[idx]), xv, acc[i]);
                        }
                    }
                }
            }
        }
        __syncwarp();
        cur = nxt;
        wstart = nstart;
        bi ^= 1;
    }
    cp_async_wait_all();
    // the last block-row of every range and any empty block-rows after it
    for (;;) {
        const bool need = row < r_end;
        if (!__any_sync(FULL, need)) break;
        flush_while(need, need ? rend : -1);
    }
}

// gstart[g] = first block-row whose first block lies in group g's share
// [g * nblocks / G, (g+1) * nblocks / G); gstart[G] = nbr.
__global__ void k_partition(int nbr, const int* __restrict__ brptr, int ngroups,
                            int* __restrict__ gstart) {
    const long nblocks = brptr[nbr];
    for (long rr = long(blockIdx.x) * blockDim.x + threadIdx.x; rr <= nbr;
         rr += long(gridDim.x) * blockDim.x) {
        // bucket of block-row rr (nbr -> G); groups in (bucket(rr-1), bucket(rr)] start at rr
        auto bucket = [&](long q) -> long {
            if (q >= nbr) return ngroups;
            if (nblocks == 0) return 0;
            const long bk = (long(brptr[q]) * ngroups) / nblocks;
            return bk < ngroups ? bk : ngroups - 1;
        };
        const long hi = bucket(rr);
        const long lo = rr == 0 ? -1 : bucket(rr - 1);
        for (long g = lo + 1; g <= hi && g <= ngroups; ++g) gstart[g] = int(rr);
    }
}

template <class K>
void set_smem(K kernel, int bytes) {
    SPC5_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

template <class LT, class V, class X, class A, class Y>
void launch_impl(const BetaView& m, const X* x, Y* y, cudaStream_t s) {
    if (m.nbr <= 0) return;
    const V* vals = static_cast<const V*>(m.values);
#define SPC5_LAUNCH(R_)                                                                          \
    {                                                                                            \
        using G = Geo<LT, R_, V, X, A>;                                                          \
        const int ctas = (m.ngroups + G::GPC - 1) / G::GPC;                                      \
        auto kern = k_spmv<LT, R_, V, X, A, Y>;                                                  \
        set_smem(kern, G::SMEM);                                                                 \
        kern<<<ctas, G::THREADS, G::SMEM, s>>>(m.nrows, m.brptr, m.headers, vals, m.valptr,      \
                                               m.gstart, m.ngroups, x, y);                       \
    }
    switch (m.r) {
        case 1: SPC5_LAUNCH(1); break;
        case 2: SPC5_LAUNCH(2); break;
        case 4: SPC5_LAUNCH(4); break;
        case 8: SPC5_LAUNCH(8); break;
        default: throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    }
#undef SPC5_LAUNCH
    SPC5_CUDA(cudaGetLastError());
}

}  // namespace

namespace {

template <class LT, class V, class X, class A, class Y>
int occupancy(int r) {
    int n = 0;
#define SPC5_OCC(R_)                                                                             \
    {                                                                                            \
        using G = Geo<LT, R_, V, X, A>;                                                          \
        auto kern = k_spmv<LT, R_, V, X, A, Y>;                                                  \
        set_smem(kern, G::SMEM);                                                                 \
        SPC5_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, G::THREADS, G::SMEM)); \
    }
    switch (r) {
        case 1: SPC5_OCC(1); break;
        case 2: SPC5_OCC(2); break;
        case 4: SPC5_OCC(4); break;
        case 8: SPC5_OCC(8); break;
        default: throw Error(SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    }
#undef SPC5_OCC
    return n;
}

}  // namespace

namespace {

template <class LT, class V>
int groups_per_cta(int) {
    return Geo<LT, 1, V, V, V>::GPC;
}

}  // namespace

int spmv_groups(int vs, int r) {
    // one wave of resident CTAs: the static partition then has no tail
    int per_sm, gpc;
    if (vs == 8) {
        per_sm = occupancy<double, double, double, double, double>(r);
        gpc = groups_per_cta<double, double>(r);
    } else {
        per_sm = std::min(occupancy<float, float, float, float, float>(r),
                          occupancy<float, float, float, double, double>(r));
        gpc = groups_per_cta<float, float>(r);
    }
    per_sm = std::max(1, std::min(per_sm, SPMV_CTAS_PER_SM));
    return sm_count() * per_sm * gpc;
}

void launch_partition(int nbr, const int* brptr, int ngroups, int* gstart, cudaStream_t s) {
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(long(nbr) + 1, threads), sm_count() * 8));
    k_partition<<<blocks, threads, 0, s>>>(nbr, brptr, ngroups, gstart);
    SPC5_CUDA(cudaGetLastError());
}

void launch_spmv_f64(const BetaView& m, const double* x, double* y, cudaStream_t s) {
    launch_impl<double, double, double, double, double>(m, x, y, s);
}

void launch_spmv_f32(const BetaView& m, const float* x, float* y, cudaStream_t s) {
    launch_impl<float, float, float, float, float>(m, x, y, s);
}

void launch_spmv_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    launch_impl<float, float, float, double, double>(m, x, y, s);
}

}  // namespace spc5cuda
