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
// its range in windows of up to VS blocks:
//   * lane j loads the packed header of block j of the window two windows
//     ahead (consecutive records, one coalesced access);
//   * one window ahead, the group scans the per-block value counts, packs
//     each block's mask with the staging-buffer offsets of its sub-rows into
//     one broadcast word, and copies the window's values into shared memory
//     with 16-byte cp.async (double-buffered);
//   * for the current window, every lane first issues its x loads for all
//     blocks (x[col + c] where any sub-row has bit c; L1/L2-cached, so the
//     loads of a whole window are in flight together), then runs the FMAs.
// When a block-row ends, each lane stores its accumulators to a per-group
// slot in shared memory; the slots of a window are reduced together at its
// end, one lane per (block-row, sub-row), with the same tree.
#include <climits>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

namespace {

constexpr int SPMV_CTAS_PER_SM = 16;
constexpr unsigned FULL = 0xffffffffu;

// Streaming 32-bit load of header words (read once).
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p) { return __ldcs(p); }

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

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Waits until at most one committed group of this thread is still in flight.
__device__ __forceinline__ void cp_async_wait_prev() {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Mask words hold one field per sub-row: a byte (f64, VS = 8) or a half-word
// (f32, VS = 16).  Fields<MB> does per-field arithmetic on whole words.
template <int MB>
struct Fields;

template <>
struct Fields<1> {
    static constexpr uint32_t REP = 0x01010101u;  // one in every field
    static constexpr int BITS = 8;
    static constexpr int PER_WORD = 4;
    // population count of every byte (SWAR)
    __device__ static __forceinline__ uint32_t popc(uint32_t w) {
        w = w - ((w >> 1) & 0x55555555u);
        w = (w & 0x33333333u) + ((w >> 2) & 0x33333333u);
        return (w + (w >> 4)) & 0x0F0F0F0Fu;
    }
    // exclusive prefix of the fields (field k = sum of fields below k)
    __device__ static __forceinline__ uint32_t prefix(uint32_t f) { return f * 0x01010100u; }
    __device__ static __forceinline__ uint32_t sum(uint32_t f) { return (f * 0x01010101u) >> 24; }
    __device__ static __forceinline__ uint32_t get(uint32_t q, int k) { return (q >> (8 * k)) & 0xFFu; }
    // OR of the fields
    __device__ static __forceinline__ uint32_t fold(uint32_t w) {
        w |= w >> 16;
        w |= w >> 8;
        return w & 0xFFu;
    }
};

template <>
struct Fields<2> {
    static constexpr uint32_t REP = 0x00010001u;
    static constexpr int BITS = 16;
    static constexpr int PER_WORD = 2;
    __device__ static __forceinline__ uint32_t popc(uint32_t w) {
        w = w - ((w >> 1) & 0x55555555u);
        w = (w & 0x33333333u) + ((w >> 2) & 0x33333333u);
        w = (w + (w >> 4)) & 0x0F0F0F0Fu;
        return (w + (w >> 8)) & 0x001F001Fu;
    }
    __device__ static __forceinline__ uint32_t prefix(uint32_t f) { return f << 16; }
    __device__ static __forceinline__ uint32_t sum(uint32_t f) { return (f + (f >> 16)) & 0xFFFFu; }
    __device__ static __forceinline__ uint32_t get(uint32_t q, int k) { return (q >> (16 * k)) & 0xFFFFu; }
    __device__ static __forceinline__ uint32_t fold(uint32_t w) { return (w | (w >> 16)) & 0xFFFFu; }
};

// Geometry of the kernel: a group of VS lanes (lane c = column c of every
// block) owns one block-row stream; GPW groups per warp run in lockstep.
template <class LT, int R, class V, class A>
struct Geo {
    static constexpr int VS = Layout<LT>::VS;
    static constexpr int MB = Layout<LT>::MASK_BYTES;
    static constexpr int THREADS = 128;
    static constexpr int GPW = 32 / VS;                      // groups per warp
    static constexpr int GPC = THREADS / VS;                 // groups per CTA
    static constexpr int EPU = 16 / int(sizeof(V));          // values per 16-byte unit
    static constexpr int MW = Header<LT, R>::MASK_WORDS;
    // masks of one block fit in 16 bits: one broadcast word carries the masks
    // (low half) and the buffer offsets of the sub-rows (high half)
    static constexpr bool PACKED = R * MB <= 2;
    static constexpr int NW = PACKED ? 1 : 2 * MW;           // broadcast words per block
    // staged values per window: a full window of 8-column f64 blocks at
    // r = 1, else the densest window of a 27-point stencil (12 values per
    // block) -- denser windows are shortened
    static constexpr int CAP = (VS == 8) ? (R == 1 ? 64 : 96) : 256;
    static constexpr int VBUF = ((CAP + 2 * EPU) * int(sizeof(V)) + 15) / 16 * 16;
    // flushed block-rows per reduction batch: MAXS * R = VS items, one per lane
    static constexpr int MAXS = VS / R > 0 ? VS / R : 1;
    static constexpr int SLOT_BYTES = MAXS * R * VS * int(sizeof(A));
    static constexpr int GROUP_BYTES = 2 * VBUF + SLOT_BYTES;
    static constexpr int SMEM = GPC * GROUP_BYTES;
    static_assert(CAP >= VS * R, "a block must fit one window");
    static_assert(CAP + 2 * EPU + (R - 1) * VS + VS <= (MB == 1 ? 256 : 65536),
                  "buffer offsets must fit one mask field");
    static_assert(MAXS * R == VS, "one reduction item per lane");
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

// One staged window of a group: lane j describes block j (j < n).
template <int NW>
struct Win {
    uint32_t w[NW];  // broadcast words: masks and buffer offsets of the sub-rows
    int col;
    int n;       // blocks in the window (group-uniform)
    int wstart;  // first block of the window (group-uniform)
};

template <class LT, int R, class V, class X, class A, class Y>
__global__ void __launch_bounds__(128)
    k_spmv(int nrows, const int* __restrict__ brptr, const uint8_t* __restrict__ headers,
           const V* __restrict__ values, const int* __restrict__ valptr,
           const int* __restrict__ gstart, int ngroups, const int* __restrict__ perm,
           const X* __restrict__ x, Y* __restrict__ y, const int* __restrict__ run_if, int run_if_value) {
    // a launch gated on a device word: the drop-in symbols enqueue the row
    // kernel and this one, and exactly one of them does the work
    if (run_if && __ldg(run_if) != run_if_value) return;
    using G = Geo<LT, R, V, A>;
    using F = Fields<G::MB>;
    constexpr int VS = G::VS, MW = G::MW, NW = G::NW, PW = F::PER_WORD;
    constexpr bool Y_ATOMIC = sizeof(Y) == 8;  // red.add.f64 is y + s rounded once
    constexpr uint32_t VSMASK = (1u << VS) - 1u;
    // keep the broadcast words of a window in registers between the x pass
    // and the FMA pass when they are few, else shuffle them again
    constexpr bool KEEP = NW * VS <= 8;
    extern __shared__ __align__(16) unsigned char smem[];

    const int lane = threadIdx.x & 31;
    const int c = lane & (VS - 1);
    const int gshift = lane & ~(VS - 1);  // bit offset of this group in warp bitmaps
    const uint32_t below = (1u << c) - 1u;
    const int gi = threadIdx.x / VS;
    const int group = blockIdx.x * G::GPC + gi;
    unsigned char* gbase = smem + gi * G::GROUP_BYTES;
    const uint32_t sgbase = uint32_t(__cvta_generic_to_shared(gbase));
    A* slots = reinterpret_cast<A*>(gbase + 2 * G::VBUF);

    int r_begin = 0, r_end = 0;
    if (group < ngroups) {
        r_begin = __ldg(gstart + group);
        r_end = __ldg(gstart + group + 1);
    }
    if (!__any_sync(FULL, r_begin < r_end)) return;
    const uint64_t pol_stream = l2_evict_first_policy();  // values: read once
    const uint64_t pol_x = l2_evict_last_policy();        // x: gathered many times
    const bool has = r_begin < r_end;
    const int b_stop = has ? __ldg(brptr + r_end) : 0;
    int p = has ? __ldg(brptr + r_begin) : 0;  // first block of the next window to stage
    int v_next = has ? __ldg(valptr + r_begin) : 0;

    // Row bookkeeping (group-uniform except ends / ends_nxt): block-row `row`
    // is the next to flush; lane c holds the end (exclusive block index) of
    // block-rows rbase + c (ends) and rbase + VS + c (ends_nxt); row = rbase + k.
    int row = r_begin, rbase = r_begin, k = 0;
    int ends = (has && rbase + c < r_end) ? __ldg(brptr + rbase + 1 + c) : INT_MAX;
    int ends_nxt = (has && rbase + VS + c < r_end) ? __ldg(brptr + rbase + 1 + VS + c) : INT_MAX;
    int rend = __shfl_sync(FULL, ends, 0, VS);
    int ns = 0;    // slots holding flushed block-rows
    int srow = 0;  // block-row of slot 0

    A acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i) acc[i] = A(0);

    // Reduce the flushed block-rows held in the slots: lane t takes item t =
    // (slot t / R, sub-row t % R) and sums its VS lane values with the
    // _mm512_reduce_add tree (distance VS/2 first, then VS/4, ..., 1).
    auto reduce_batch = [&](bool doit) {
        __syncwarp();
        if (doit && c < ns * R) {
            A a[VS];
            const A* sp = slots + c * VS;
            if constexpr (sizeof(A) == 8) {
#pragma unroll
                for (int e = 0; e < VS; e += 2) {
                    const double2 t = *reinterpret_cast<const double2*>(sp + e);
                    a[e] = A(t.x);
                    a[e + 1] = A(t.y);
                }
            } else {
#pragma unroll
                for (int e = 0; e < VS; e += 4) {
                    const float4 t = *reinterpret_cast<const float4*>(sp + e);
                    a[e] = A(t.x);
                    a[e + 1] = A(t.y);
                    a[e + 2] = A(t.z);
                    a[e + 3] = A(t.w);
                }
            }
#pragma unroll
            for (int d = VS / 2; d >= 1; d >>= 1) {
#pragma unroll
                for (int e = 0; e < d; ++e) a[e] = a[e] + a[e + d];
            }
            const int brow = perm ? __ldg(perm + srow + c / R) : srow + c / R;
            const long yrow = long(brow) * R + (c % R);
            if (yrow < nrows) {
                if constexpr (Y_ATOMIC) atomicAdd(y + yrow, Y(a[0]));
                else y[yrow] = y[yrow] + Y(a[0]);
            }
        }
        if (doit) ns = 0;
        __syncwarp();
    };

    // Flush every group whose current block-row ends at block b (the rows
    // that end before block b is processed), repeating for empty block-rows;
    // warp-uniform control flow.
    auto flush_exact = [&](int b, bool active) {
        for (;;) {
            const bool fl = active && row < r_end && rend == b;
            if (!__any_sync(FULL, fl)) break;
            if (fl) {
                if (ns == 0) srow = row;
                A* sp = slots + ns * (R * VS) + c;
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    sp[i * VS] = acc[i];
                    acc[i] = A(0);
                }
                ++ns;
                ++row;
                if (++k == VS) {
                    k = 0;
                    rbase += VS;
                    ends = ends_nxt;
                    ends_nxt = (rbase + VS + c < r_end) ? __ldg(brptr + rbase + 1 + VS + c) : INT_MAX;
                }
            }
            rend = __shfl_sync(FULL, ends, k, VS);
            if (__any_sync(FULL, ns == G::MAXS)) reduce_batch(ns == G::MAXS);
        }
    };

    // ---- stage one window: headers rw (blocks p ...) -> win; values into buffer bi
    auto stage = [&](const Raw<LT, R>& rw, Win<NW>& win, int bi) {
        uint32_t cnt[MW];
        int tot = 0;
#pragma unroll
        for (int q = 0; q < MW; ++q) {
            cnt[q] = F::popc(rw.mw[q]);
            tot += int(F::sum(cnt[q]));
        }
        if (!rw.ok) tot = 0;
        int incl = tot;
#pragma unroll
        for (int d = 1; d < VS; d <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, d, VS);
            if (c >= d) incl += t;
        }
        const int n = __popc((__ballot_sync(FULL, rw.ok && incl <= G::CAP) >> gshift) & VSMASK);
        const int tv = __shfl_sync(FULL, incl, (n > 0 ? n : 1) - 1, VS);
        const int s0 = v_next & ~(G::EPU - 1);
        const int shift = v_next - s0;
        const uint32_t voff = uint32_t(shift + incl - tot);  // buffer index of the block's first value
        win.n = n;
        win.wstart = p;
        win.col = rw.col;
        if constexpr (G::PACKED) {
            const uint32_t base = (voff * F::REP + F::prefix(cnt[0])) & 0xFFFFu;
            win.w[0] = rw.mw[0] | (base << 16);
        } else {
            uint32_t carry = 0;
#pragma unroll
            for (int q = 0; q < MW; ++q) {
                win.w[q] = rw.mw[q];
                win.w[MW + q] = (voff + carry) * F::REP + F::prefix(cnt[q]);
                carry += F::sum(cnt[q]);
            }
        }
        if (n > 0) {
            const uint32_t vb = sgbase + uint32_t(bi * G::VBUF);
            const int units = (shift + tv + G::EPU - 1) / G::EPU;
            const V* src = values + s0;
            for (int u = c; u < units; u += VS) cp_async16_hint(vb + uint32_t(u) * 16u, src + u * G::EPU, pol_stream);
        }
        cp_async_commit();
        v_next += (n > 0) ? tv : 0;
        p += n;
    };

    // masks (q-th word) and buffer offsets (q-th word) of a broadcast block
    auto mask_word = [&](const uint32_t (&w)[NW], int q) -> uint32_t {
        if constexpr (G::PACKED) return w[0] & 0xFFFFu;
        else return w[q];
    };
    auto base_word = [&](const uint32_t (&w)[NW], int q) -> uint32_t {
        if constexpr (G::PACKED) return w[0] >> 16;
        else return w[MW + q];
    };

    // ---- prologue: stage window 0, load the headers of window 1
    Raw<LT, R> raw;
    load_raw<LT, R>(raw, headers, p, b_stop, c);
    Win<NW> cur;
    stage(raw, cur, 0);
    load_raw<LT, R>(raw, headers, p, b_stop, c);
    int bi = 0;

    while (__any_sync(FULL, cur.n > 0)) {
        // ---- x pass: every lane loads x[col + c] of every block of the window
        // in which some sub-row has bit c
        X xv[VS];
        uint32_t keep[KEEP ? VS : 1][NW];
#pragma unroll
        for (int j = 0; j < VS; ++j) {
            if (!__any_sync(FULL, j < cur.n)) break;
            const int cj = __shfl_sync(FULL, cur.col, j, VS);
            uint32_t wj[NW];
#pragma unroll
            for (int q = 0; q < NW; ++q) wj[q] = __shfl_sync(FULL, cur.w[q], j, VS);
            uint32_t lanes = 0;
#pragma unroll
            for (int q = 0; q < MW; ++q) lanes |= F::fold(mask_word(wj, q));
            xv[j] = X(0);
            if (j < cur.n && ((lanes >> c) & 1u)) xv[j] = ld_x(x + (cj + c), pol_x);
            if constexpr (KEEP) {
#pragma unroll
                for (int q = 0; q < NW; ++q) keep[j][q] = wj[q];
            }
        }

        // ---- stage the next window, load the headers of the one after it
        Win<NW> nxt;
        stage(raw, nxt, bi ^ 1);
        load_raw<LT, R>(raw, headers, p, b_stop, c);

        // ---- block positions of this window where a block-row of some group
        // may end (known ends of rows row .. rbase + 2 VS - 1; past the last
        // known end every position is checked)
        uint32_t rmask;
        {
            uint32_t mine = 0;
            const int rel = ends - cur.wstart;
            if (c >= k && rel >= 0 && rel < cur.n) mine |= 1u << rel;
            const int rel2 = ends_nxt - cur.wstart;
            if (rel2 >= 0 && rel2 < cur.n) mine |= 1u << rel2;
            const int last = __shfl_sync(FULL, ends_nxt, VS - 1, VS);
            const int lrel = last - cur.wstart;
            if (c == 0 && lrel < cur.n) mine |= VSMASK << (lrel < 0 ? 0 : lrel);
            rmask = __reduce_or_sync(FULL, mine) & VSMASK;
        }
        cp_async_wait_prev();
        __syncwarp();

        // ---- FMA pass
        const V* vbuf = reinterpret_cast<const V*>(gbase + bi * G::VBUF);
#pragma unroll
        for (int j = 0; j < VS; ++j) {
            if (!__any_sync(FULL, j < cur.n)) break;
            const bool act = j < cur.n;
            if ((rmask >> j) & 1u) flush_exact(cur.wstart + j, act);
            uint32_t wj[NW];
            if constexpr (KEEP) {
#pragma unroll
                for (int q = 0; q < NW; ++q) wj[q] = keep[j][q];
            } else {
#pragma unroll
                for (int q = 0; q < NW; ++q) wj[q] = __shfl_sync(FULL, cur.w[q], j, VS);
            }
            if (act) {
                const A xa = A(xv[j]);
#pragma unroll
                for (int q = 0; q < MW; ++q) {
                    const uint32_t m = mask_word(wj, q);
                    uint32_t qoff;
                    if constexpr (R == 1) qoff = base_word(wj, q) + uint32_t(__popc(m & below));
                    else qoff = base_word(wj, q) + F::popc(m & (below * F::REP));
#pragma unroll
                    for (int f = 0; f < PW; ++f) {
                        const int i = q * PW + f;
                        if (i < R && ((m >> (f * F::BITS + c)) & 1u))
                            acc[i] = fma(A(vbuf[F::get(qoff, f)]), xa, acc[i]);
                    }
                }
            }
        }
        // the block-rows flushed in this window
        if (__any_sync(FULL, ns > 0)) reduce_batch(ns > 0);
        __syncwarp();
        cur = nxt;
        bi ^= 1;
    }
    cp_async_wait_all();
    // the last block-row of every range and any empty block-rows after it
    flush_exact(b_stop, has);
    if (__any_sync(FULL, ns > 0)) reduce_batch(ns > 0);
}

// gstart[g] = first block-row of [a, b) whose first block lies in group g's
// share [g * n / G, (g+1) * n / G) of the range's n blocks; gstart[G] = b.
__global__ void k_partition(int a, int b, const int* __restrict__ brptr, int ngroups,
                            int* __restrict__ gstart) {
    const long base = brptr[a];
    const long nblocks = long(brptr[b]) - base;
    for (long rr = a + long(blockIdx.x) * blockDim.x + threadIdx.x; rr <= b;
         rr += long(gridDim.x) * blockDim.x) {
        // bucket of block-row rr (b -> G); groups in (bucket(rr-1), bucket(rr)] start at rr
        auto bucket = [&](long q) -> long {
            if (q >= b) return ngroups;
            if (nblocks == 0) return 0;
            const long bk = ((long(brptr[q]) - base) * ngroups) / nblocks;
            return bk < ngroups ? bk : ngroups - 1;
        };
        const long hi = bucket(rr);
        const long lo = rr == a ? -1 : bucket(rr - 1);
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
        using G = Geo<LT, R_, V, A>;                                                          \
        const int ctas = (m.ngroups + G::GPC - 1) / G::GPC;                                      \
        auto kern = k_spmv<LT, R_, V, X, A, Y>;                                                  \
        set_smem(kern, G::SMEM);                                                                 \
        kern<<<ctas, G::THREADS, G::SMEM, s>>>(m.nrows, m.brptr, m.headers, vals, m.valptr,      \
                                               m.gstart, m.ngroups, m.perm, x, y, m.run_if,      \
                                               m.run_if_value);                                  \
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
        using G = Geo<LT, R_, V, A>;                                                          \
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
    return Geo<LT, 1, V, V>::GPC;
}

}  // namespace

int spmv_groups(int vs, int r) {
    // one wave of resident CTAs: the static partition then has no tail;
    // cached per (device, VS, r) (the drop-in symbols ask on every call)
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, int> cache;
    int dev = 0;
    SPC5_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, vs, r);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
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
    const int n = sm_count() * per_sm * gpc;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = n;
    return n;
}

void launch_partition(int nbr, const int* brptr, int ngroups, int* gstart, cudaStream_t s) {
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(long(nbr) + 1, threads), sm_count() * 8));
    k_partition<<<blocks, threads, 0, s>>>(0, nbr, brptr, ngroups, gstart);
    SPC5_CUDA(cudaGetLastError());
}

void launch_partition_range(int a, int b, const int* brptr, int ngroups, int* gstart, cudaStream_t s) {
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(long(b - a) + 1, threads), sm_count() * 8));
    k_partition<<<blocks, threads, 0, s>>>(a, b, brptr, ngroups, gstart);
    SPC5_CUDA(cudaGetLastError());
}

void launch_spmv_f64(const BetaView& m, const double* x, double* y, cudaStream_t s) {
    if (m.wstart) launch_rows_f64(m, x, y, s);
    else launch_impl<double, double, double, double, double>(m, x, y, s);
}

void launch_spmv_f32(const BetaView& m, const float* x, float* y, cudaStream_t s) {
    if (m.wstart) launch_rows_f32(m, x, y, s);
    else launch_impl<float, float, float, float, float>(m, x, y, s);
}

void launch_spmv_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    if (m.wstart) launch_rows_mixed(m, x, y, s);
    else launch_impl<float, float, float, double, double>(m, x, y, s);
}

void launch_spmv_mixed8(const BetaView& m, const float* x, double* y, cudaStream_t s) {
    if (m.wstart) launch_rows_mixed8(m, x, y, s);
    else launch_impl<double, float, float, double, double>(m, x, y, s);
}

}  // namespace spc5cuda
