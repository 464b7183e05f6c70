// rows_stage.cuh -- the staged walk over a warp's block-rows shared by the
// thread-per-sub-row SpMV (spmv_rows.cu) and SpMM (spmm_rows.cu) kernels.
//
// A warp owns a contiguous range of block-rows and walks it in chunks of at
// most 32 / L block-rows (L lanes per block-row).  The chunk's packed headers
// and values are copied into the warp's shared-memory buffer with coalesced
// 16-byte cp.async (matrix data streamed with an L2 evict-first policy, the
// data after the chunk prefetched into L2), then the caller's compute step
// reads every block of the chunk from shared memory.  The helpers below
// decode a staged header and locate the value of (sub-row, column) in a block
// -- the expand-load offsets of the reference vector kernels.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace spc5cuda {
namespace rows {

constexpr int THREADS = 128;
constexpr int WARPS = THREADS / 32;
// One warp's staging buffer: 7.5 KB, so that 7 CTAs of 4 warps fit an SM
// (measured on B200: 10 KB buffers, 5 per SM, were 3% slower on the
// power-law matrix and 10% on the 27-point stencil; 5 KB chunks were too
// small for the stencil).
constexpr int HB = 1536;  // header bytes of one warp's staging buffer
constexpr int VB = 6144;  // value bytes of one warp's staging buffer
// The multi-RHS kernels are limited by registers to 4 CTAs per SM, so they
// stage larger chunks (every block-row or segment cut for the buffers above
// fits these).
constexpr int MM_HB = 2048;
constexpr int MM_VB = 8192;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Bulk prefetch of [p, p + bytes) into L2 (p 16-byte aligned, bytes a
// multiple of 16); no data is returned.
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes) {
    if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

template <class LT, int R, class V, int L, int HB_ = HB, int VB_ = VB>
struct Geo {
    static constexpr int VS = Layout<LT>::VS;
    static constexpr int MB = Layout<LT>::MASK_BYTES;
    static constexpr int STRIDE = Header<LT, R>::STRIDE;
    static constexpr int MW = Header<LT, R>::MASK_WORDS;
    static constexpr int LOAD_WORDS = Header<LT, R>::LOAD_WORDS;
    static_assert(L >= R && L <= Layout<LT>::VS && 32 % L == 0, "lanes per block-row");
    static constexpr int SPW = 32 / L;  // block-rows per chunk (L lanes each)
    static constexpr int EPU = 16 / int(sizeof(V));
    static constexpr int BUF_BYTES = HB_ + VB_;
    static constexpr int SMEM = WARPS * BUF_BYTES;
};

// One chunk of a warp's range: block-rows r0 .. r0 + nrow - 1, small enough
// for one staging buffer.  Lane k < nrow holds the end block and end value of
// block-row r0 + k.
struct Chunk {
    int r0, nrow;
    int b_lo, v_lo;  // first block and first value of the chunk
    long h_al;       // 16-byte aligned start of the chunk's header bytes
    int v_al;        // start of the chunk's values, rounded down to 16 bytes
    int b_hi, v_hi;  // this lane's block-row end (lane < nrow)
    int hunits, vunits;
};

// Walks block-rows [r_begin, r_stop) of one matrix (warp-uniform bounds):
// stage a chunk into wbuf, load the next chunk's bounds while the copies fly,
// call compute(chunk, staged header words, staged values), repeat.  A chunk
// holds at most `cap` (<= 32 / L) block-rows: as many as fit the buffer.  The
// caller guarantees that every block-row alone fits the buffer.
template <class LT, int R, class V, int L, int HB_ = HB, int VB_ = VB, class F>
__device__ __forceinline__ void walk(const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
                                     const V* __restrict__ values, const int* __restrict__ valptr,
                                     int r_begin, int r_stop, unsigned char* wbuf, F&& compute,
                                     int cap = 32 / L) {
    using G = Geo<LT, R, V, L>;
    constexpr int S = G::STRIDE, EPU = G::EPU;
    if (r_begin >= r_stop) return;
    const int lane = threadIdx.x & 31;
    const uint32_t s_h = uint32_t(__cvta_generic_to_shared(wbuf));
    const uint32_t s_v = s_h + uint32_t(HB_);
    const uint32_t* hw = reinterpret_cast<const uint32_t*>(wbuf);
    const V* vbuf = reinterpret_cast<const V*>(wbuf + HB_);
    const uint64_t pol_stream = l2_evict_first_policy();
    // end of this range's header bytes and values: prefetches stay inside
    const long h_stop = (long(__ldg(brptr + r_stop)) * S + 15) & ~15L;
    const long v_stop = (long(__ldg(valptr + r_stop)) + EPU - 1) & ~long(EPU - 1);

    // bounds() issues the loads of the block-row ends (lane k: block-row
    // r0 + k), finish() decides how many block-rows fit the buffer.
    struct Bounds {
        int r0, b_lo, v_lo, b_hi, v_hi;
        bool cand;
    };
    auto bounds = [&](int r0, int b_lo, int v_lo) {
        Bounds bd;
        bd.r0 = r0;
        bd.b_lo = b_lo;
        bd.v_lo = v_lo;
        bd.cand = lane < cap && r0 + lane < r_stop;
        bd.b_hi = bd.cand ? __ldg(brptr + r0 + lane + 1) : 0;
        bd.v_hi = bd.cand ? __ldg(valptr + r0 + lane + 1) : 0;
        return bd;
    };
    auto finish = [&](const Bounds& bd) {
        Chunk ch;
        ch.r0 = bd.r0;
        ch.b_lo = bd.b_lo;
        ch.v_lo = bd.v_lo;
        ch.b_hi = bd.b_hi;
        ch.v_hi = bd.v_hi;
        ch.h_al = (long(ch.b_lo) * S) & ~15L;
        ch.v_al = ch.v_lo & ~(EPU - 1);
        bool fits = false;
        if (bd.cand) {
            const long hneed = ((long(ch.b_hi) * S + 15) & ~15L) - ch.h_al;
            const long vneed = long((ch.v_hi + EPU - 1) & ~(EPU - 1)) - ch.v_al;
            fits = hneed <= HB_ && vneed * long(sizeof(V)) <= VB_;
        }
        // the ends grow with the lane, so the fitting lanes are a prefix
        ch.nrow = __popc(__ballot_sync(FULL, fits));
        const int last = ch.nrow > 0 ? ch.nrow - 1 : 0;
        const int b_end = __shfl_sync(FULL, ch.b_hi, last);
        const int v_end = __shfl_sync(FULL, ch.v_hi, last);
        ch.hunits = 0;
        ch.vunits = 0;
        if (ch.nrow > 0) {
            ch.hunits = int((((long(b_end) * S + 15) & ~15L) - ch.h_al) >> 4);
            ch.vunits = (v_end - ch.v_al + EPU - 1) / EPU;
        }
        return ch;
    };
    // copy a chunk's headers and values into the buffer (one commit group)
    auto stage = [&](const Chunk& ch) {
        const uint8_t* hsrc = headers + ch.h_al;
        for (int u = lane; u < ch.hunits; u += 32) cp_async16_hint(s_h + 16u * uint32_t(u), hsrc + 16L * u, pol_stream);
        const V* vsrc = values + ch.v_al;
        for (int u = lane; u < ch.vunits; u += 32) cp_async16_hint(s_v + 16u * uint32_t(u), vsrc + long(u) * EPU, pol_stream);
        cp_async_commit();
        // warm L2 with the data after this chunk (the next one is about as
        // large), clipped to this range
        if (lane == 0 && ch.nrow > 0 && ch.r0 + ch.nrow < r_stop) {
            const long h0 = ch.h_al + 16L * ch.hunits;
            const long hn = std::min(16L * ch.hunits, h_stop - h0);
            if (hn > 0) l2_prefetch(headers + h0, uint32_t(hn));
            const long v0 = long(ch.v_al) + long(ch.vunits) * EPU;
            const long vn = std::min(long(ch.vunits) * EPU, v_stop - v0);
            if (vn > 0) l2_prefetch(values + v0, uint32_t(vn * long(sizeof(V))));
        }
    };

    Chunk cur = finish(bounds(r_begin, __ldg(brptr + r_begin), __ldg(valptr + r_begin)));
    while (cur.nrow > 0) {  // warp-uniform
        stage(cur);
        const int last = cur.nrow - 1;
        const int r_next = cur.r0 + cur.nrow;
        const Bounds nb = bounds(r_next, __shfl_sync(FULL, cur.b_hi, last), __shfl_sync(FULL, cur.v_hi, last));
        cp_async_wait_all();
        __syncwarp();
        compute(cur, hw, vbuf);
        __syncwarp();  // the next chunk overwrites the buffer
        cur = r_next < r_stop ? finish(nb) : Chunk{r_next, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    }
    cp_async_wait_all();
}

// Header of block bb from a chunk's staged records (off = bb * stride minus
// the chunk's aligned header start): the column and the mask words (mask of
// sub-row i in field i % (4 / mask bytes) of word i / (4 / mask bytes)).
template <class LT, int R>
__device__ __forceinline__ int decode_staged(const uint32_t* hw, long off,
                                             uint32_t (&mw)[Header<LT, R>::MASK_WORDS]) {
    using H = Header<LT, R>;
    uint32_t lw[H::LOAD_WORDS + 1];
#pragma unroll
    for (int w = 0; w < H::LOAD_WORDS; ++w) lw[w] = hw[(off >> 2) + w];
    lw[H::LOAD_WORDS] = 0u;
    if constexpr (H::STRIDE % 4 == 0) {
#pragma unroll
        for (int w = 0; w < H::MASK_WORDS; ++w) mw[w] = lw[1 + w];
        return int(lw[0]);
    } else {
        const unsigned sh = unsigned(off & 3) * 8u;
        mw[0] = __funnelshift_r(lw[1], lw[2], sh) & ((1u << (8 * H::MASK_BYTES_TOTAL)) - 1u);
        return int(__funnelshift_r(lw[0], lw[1], sh));
    }
}

// Union of the sub-row masks (bit c: some sub-row has a value in column c).
template <class LT, int R>
__device__ __forceinline__ uint32_t mask_union(const uint32_t (&mw)[Header<LT, R>::MASK_WORDS]) {
    uint32_t uni = 0;
#pragma unroll
    for (int w = 0; w < Header<LT, R>::MASK_WORDS; ++w) uni |= mw[w];
    if constexpr (Layout<LT>::MASK_BYTES == 1) return (uni | (uni >> 16)) | ((uni | (uni >> 16)) >> 8);
    else return uni | (uni >> 16);
}

// Per mask word: exclusive prefix of the sub-row value counts, one field per
// sub-row (pre); returns the block's value count.
template <class LT, int R>
__device__ __forceinline__ int subrow_prefix(const uint32_t (&mw)[Header<LT, R>::MASK_WORDS],
                                             uint32_t (&pre)[Header<LT, R>::MASK_WORDS]) {
    uint32_t carry = 0;
#pragma unroll
    for (int w = 0; w < Header<LT, R>::MASK_WORDS; ++w) {
        uint32_t cnt = mw[w] - ((mw[w] >> 1) & 0x55555555u);
        cnt = (cnt & 0x33333333u) + ((cnt >> 2) & 0x33333333u);
        cnt = (cnt + (cnt >> 4)) & 0x0F0F0F0Fu;
        if constexpr (Layout<LT>::MASK_BYTES == 1) {
            pre[w] = cnt * 0x01010100u + carry * 0x01010101u;
            carry += (cnt * 0x01010101u) >> 24;
        } else {
            cnt = (cnt + (cnt >> 8)) & 0x001F001Fu;
            pre[w] = (cnt << 16) + carry * 0x00010001u;
            carry += (cnt + (cnt >> 16)) & 0xFFFFu;
        }
    }
    return int(carry);
}

// Field f of the result: offset, from the block's first value, of the value
// of sub-row (w * fields per word + f) in the column whose lower columns are
// `below`, for mask word w with prefix pre_w.
template <class LT, int R>
__device__ __forceinline__ uint32_t column_offsets(uint32_t mw_w, uint32_t pre_w, uint32_t below) {
    if constexpr (R == 1) {
        return uint32_t(__popc(mw_w & below));
    } else if constexpr (Layout<LT>::MASK_BYTES == 1) {
        uint32_t t = mw_w & (below * 0x01010101u);
        t = t - ((t >> 1) & 0x55555555u);
        t = (t & 0x33333333u) + ((t >> 2) & 0x33333333u);
        return pre_w + ((t + (t >> 4)) & 0x0F0F0F0Fu);
    } else {
        uint32_t t = mw_w & (below * 0x00010001u);
        t = t - ((t >> 1) & 0x55555555u);
        t = (t & 0x33333333u) + ((t >> 2) & 0x33333333u);
        t = (t + (t >> 4)) & 0x0F0F0F0Fu;
        return pre_w + ((t + (t >> 8)) & 0x001F001Fu);
    }
}

}  // namespace rows
}  // namespace spc5cuda
