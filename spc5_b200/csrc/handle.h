// handle.h -- host-side internals shared by the C ABI translation units:
// device buffers, status plumbing and the matrix handle (spc5cuda_mat).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

// Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(size_t n, cudaStream_t st) : bytes(n), s(st) {
        if (n) SPC5_CUDA(cudaMallocAsync(&p, n, st));
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// The library's stream-ordered memory pool on the current device (capi.cu),
// and per-call scratch from it.
cudaMemPool_t scratch_pool();
struct PoolBuf {
    void* p = nullptr;
    cudaStream_t s;
    PoolBuf(size_t n, cudaStream_t st) : s(st) {
        SPC5_CUDA(cudaMallocFromPoolAsync(&p, n < 16 ? size_t(16) : n, scratch_pool(), st));
    }
    ~PoolBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    template <class U>
    U* as() const { return static_cast<U*>(p); }
};

// Persistent device buffer owned by a matrix handle.
struct Owned {
    void* p = nullptr;
    size_t bytes = 0;
    void alloc(size_t n) {
        release();
        if (n) SPC5_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    Owned() = default;
    Owned(const Owned&) = delete;
    Owned& operator=(const Owned&) = delete;
    Owned(Owned&& o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    Owned& operator=(Owned&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~Owned() { release(); }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

inline int format_to_r(int format) {
    switch (format) {
        case SPC5CUDA_FORMAT_1rVc_WT: return 1;
        case SPC5CUDA_FORMAT_2rVc: return 2;
        case SPC5CUDA_FORMAT_4rVc: return 4;
        case SPC5CUDA_FORMAT_8rVc: return 8;
        default: return 0;
    }
}

inline int r_to_format(int r) {
    switch (r) {
        case 1: return SPC5CUDA_FORMAT_1rVc_WT;
        case 2: return SPC5CUDA_FORMAT_2rVc;
        case 4: return SPC5CUDA_FORMAT_4rVc;
        case 8: return SPC5CUDA_FORMAT_8rVc;
        default: return SPC5CUDA_UNDEFINED_FORMAT;
    }
}

// F64 and F32_V8 use the 8-column layout (uint8 masks), F32 the 16-column one.
inline bool valid_value_type(int value_type) {
    return value_type == SPC5CUDA_F64 || value_type == SPC5CUDA_F32 || value_type == SPC5CUDA_F32_V8;
}
inline int vs_of(int value_type) { return value_type == SPC5CUDA_F32 ? 16 : 8; }
inline int mask_bytes_of(int value_type) { return value_type == SPC5CUDA_F32 ? 2 : 1; }
inline int value_bytes_of(int value_type) { return value_type == SPC5CUDA_F64 ? 8 : 4; }

template <class F>
inline spc5cuda_status guarded(F&& f) {
    try {
        f();
        return SPC5CUDA_OK;
    } catch (const Error& e) {
        return e.status;
    } catch (const std::bad_alloc&) {
        return SPC5CUDA_ERR_NOMEM;
    } catch (...) {
        return SPC5CUDA_ERR_INVALID;
    }
}

inline void require(bool cond, spc5cuda_status s, const char* what) {
    if (!cond) throw Error(s, what);
}


// One part of the length-sorted plan: sorted block-rows [a, b), run by the
// row kernel with `lanes` lanes per block-row (split: one range per warp), or
// by the group kernel when lanes == 0 (split: one range per group); split
// holds nsplit + 1 block-row starts.  The part of the block-rows too large
// to stage (nseg = b - a > 0, a = 0) is either the chain part (chains: the
// multiply-add chains below; two launches) or segmented: cut into segments
// that are, interleaved per warp; vbrptr / vvalptr are the segments' block
// and value offsets and split their per-warp ranges.
struct SpmvPart {
    int lanes = 0;
    int a = 0, b = 0;
    int nseg = 0;
    bool chains = false;
    Owned split;
    int nsplit = 0;
    Owned vbrptr, vvalptr;
    // the chain part (chain.cu): one multiply-add chain per (block-row,
    // sub-row, column) of the nseg largest block-rows, chain id
    // (i * r + s) * VS + c.  The nchains non-empty ones, sorted by length
    // (slen, corder: chain ids), cut into slices of 32 chains, entry j of the
    // slice's lane l at slice_off[slice] + 32 j + l (cval: value, ccol: x
    // index); cmask[i * r + s] bit c: chain c of that sub-row is not empty.
    long nchains = 0;
    long entries = 0;  // values in the chains
    int nslices = 0;
    Owned slen, corder, slice_off, cval, ccol, cmask;
};

// A copy of the matrix with its block-rows sorted by size (plan.cu).  Its
// parts write disjoint rows of y, so an SpMV forks them onto two streams of
// the plan and joins them back to the caller's stream.
struct SortedPlan {
    Owned sbrptr, sheaders, svalues, svalptr, perm;
    std::vector<SpmvPart> parts;
    bool in_order = false;  // run the parts one after another on the caller's stream
    cudaStream_t aux[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    std::mutex mu;  // one fork/join at a time (the events are shared)
    SortedPlan() = default;
    SortedPlan(const SortedPlan&) = delete;
    SortedPlan& operator=(const SortedPlan&) = delete;
    ~SortedPlan() {
        for (auto& st : aux)
            if (st) cudaStreamDestroy(st);
        if (fork) cudaEventDestroy(fork);
        for (auto& e : join)
            if (e) cudaEventDestroy(e);
    }
    long bytes() const {
        long n = long(sbrptr.bytes + sheaders.bytes + svalues.bytes + svalptr.bytes + perm.bytes);
        for (const auto& p : parts)
            n += long(p.split.bytes + p.vbrptr.bytes + p.vvalptr.bytes + p.slen.bytes + p.corder.bytes +
                      p.slice_off.bytes + p.cval.bytes + p.ccol.bytes + p.cmask.bytes);
        return n;
    }
};

// The length-sorted plan of a converted matrix (plan.cu; synchronises s),
// and the view of one of its parts.
void build_sorted_plan(spc5cuda_mat* m, cudaStream_t s);
BetaView plan_view(const spc5cuda_mat* m, const SpmvPart& part);
// The reference-order headers and values of a handle whose plan holds the
// only copy, written to device buffers of m->headers / m->values size.
void rebuild_original(const spc5cuda_mat* m, uint8_t* headers, void* values, cudaStream_t s);
// The chain part (chain.cu): built from the sorted copy's block-rows
// [0, part.nseg), whose values it then drops from the copy (synchronises s);
// its values back in the reference order; y += A x and Y += A X over it.
void build_chains(spc5cuda_mat* m, SortedPlan* plan, SpmvPart& part, cudaStream_t s);
void unchain_values(const spc5cuda_mat* m, const SpmvPart& part, void* values, cudaStream_t s);
void chain_part_spmv(const spc5cuda_mat* m, const SpmvPart& part, const void* x, void* y, bool mixed,
                     cudaStream_t s);
void chain_part_spmm(const spc5cuda_mat* m, const SpmvPart& part, int k, const void* x, long ldx, long xcs, void* y,
                     long ldy, long ycs, bool mixed, cudaStream_t s);
void launch_iota(long n, int* a, cudaStream_t s);
// y += A x through the plan (x, y of the handle's types; mixed: F32 or
// F32_V8 handle, float x, double y).  fork: run the parts concurrently on the
// plan's two streams and join them back to s (one such call at a time per
// handle); otherwise one after another on s, so that calls on different
// streams (the request loop's slots) overlap without sharing plan streams.
void plan_spmv(const spc5cuda_mat* m, const void* x, void* y, bool mixed, cudaStream_t s, bool fork = true);
// Y += A X through the plan with the staged SpMM (element (row i, rhs q) of
// X at x[i * ldx + q * xcs], likewise Y).
void plan_spmm(const spc5cuda_mat* m, int k, const void* x, long ldx, long xcs, void* y, long ldy, long ycs,
               bool mixed, cudaStream_t s, bool fork = true);

}  // namespace spc5cuda

// The device-resident SPC5Mat<T> (src/spc5.hpp:44-62).
struct spc5cuda_mat {
    using Owned = spc5cuda::Owned;
    using BetaView = spc5cuda::BetaView;
    int value_type = SPC5CUDA_F64;
    int format = SPC5CUDA_UNDEFINED_FORMAT;
    int r = 0;
    int nrows = 0, ncols = 0;
    long nnz = 0;
    long nblocks = 0;
    Owned rowptr;   // CSR row pointer (nrows+1); dropped after conversion
    Owned colidx;   // CSR column indices; dropped after conversion
    Owned values;   // nnz values (CSR order, then beta order)
    Owned brptr;    // rowsSize after conversion: ceil(nrows/r)+1 block offsets
    Owned headers;  // blocksColumnIndexesWithMasks
    Owned valptr;   // ceil(nrows/r)+1 value offsets (not in the reference format)
    Owned gstart;   // ngroups+1 block-row starts of the per-group ranges
    int ngroups = 0;
    Owned wstart;   // nwarps+1 block-row starts of the thread-per-sub-row kernel's warps
    int nwarps = 0;
    int kernel = SPC5CUDA_KERNEL_AUTO;  // SpMV kernel choice (spc5cuda_mat_set_kernel)
    bool rows_ok = false;               // every block-row fits the row kernel's buffers
    std::unique_ptr<spc5cuda::SortedPlan> plan;  // length-sorted copy (irregular matrices)
    // the plan holds the only copy of headers and values (set when the plan
    // is built and serves SpMV): the reference order is rebuilt on demand
    bool original_dropped = false;

    int nbr() const { return r ? spc5cuda::div_up(nrows, r) : 0; }
    BetaView view() const {
        BetaView v;
        v.r = r;
        v.nrows = nrows;
        v.nbr = nbr();
        v.brptr = brptr.as<int>();
        v.headers = headers.as<uint8_t>();
        v.values = values.p;
        v.valptr = valptr.as<int>();
        v.gstart = gstart.as<int>();
        v.ngroups = ngroups;
        if (use_rows()) {
            v.wstart = wstart.as<int>();
            v.nwarps = nwarps;
        }
        return v;
    }
    // The view of the SpMM kernels: the per-warp ranges of the staged kernel
    // whenever every block-row fits its buffers, unless the group kernel was
    // requested.
    BetaView spmm_view() const {
        BetaView v = view();
        v.wstart = nullptr;
        v.nwarps = 0;
        if (rows_ok && nwarps > 0 && kernel != SPC5CUDA_KERNEL_GROUPS) {
            v.wstart = wstart.as<int>();
            v.nwarps = nwarps;
        }
        return v;
    }
    // The thread-per-sub-row kernel runs when every block-row fits its
    // staging buffers, on request or by default (it is faster than the group
    // kernel on the B200 for every r).
    bool use_rows() const {
        if (!rows_ok || nwarps <= 0) return false;
        return kernel == SPC5CUDA_KERNEL_ROWS || kernel == SPC5CUDA_KERNEL_AUTO;
    }
    // The length-sorted plan runs on request, or by default when some
    // block-row is too large for the row kernel (irregular matrices).
    bool use_plan() const {
        if (!plan) return false;
        return kernel == SPC5CUDA_KERNEL_SORTED || (kernel == SPC5CUDA_KERNEL_AUTO && !rows_ok);
    }
    bool wants_plan() const {
        return kernel == SPC5CUDA_KERNEL_SORTED || (kernel == SPC5CUDA_KERNEL_AUTO && !rows_ok);
    }
    size_t header_bytes() const {
        return size_t(nblocks) * size_t(4 + r * spc5cuda::mask_bytes_of(value_type));
    }
    size_t value_bytes() const { return size_t(nnz) * size_t(spc5cuda::value_bytes_of(value_type)); }
    // Bring the reference-order headers and values back into the handle
    // (synchronises s); a no-op unless the plan holds the only copy.
    void restore_original(cudaStream_t s) {
        if (!original_dropped) return;
        Owned h, v;
        h.alloc(std::max<size_t>(header_bytes(), 16));
        v.alloc(std::max<size_t>(value_bytes(), 16));
        spc5cuda::rebuild_original(this, h.as<uint8_t>(), v.p, s);
        SPC5_CUDA(cudaStreamSynchronize(s));
        headers = std::move(h);
        values = std::move(v);
        original_dropped = false;
    }
    long device_bytes() const {
        return long(rowptr.bytes + colidx.bytes + values.bytes + brptr.bytes + headers.bytes +
                    valptr.bytes + gstart.bytes + wstart.bytes) + (plan ? plan->bytes() : 0L);
    }
    // The per-group block-row ranges for the current device.
    // The per-group block-row ranges for the current device, and the per-warp
    // ranges of the thread-per-sub-row kernel when every block-row fits it.
    void build_partition(cudaStream_t s) {
        const int vs = spc5cuda::vs_of(value_type);
        ngroups = spc5cuda::spmv_groups(vs, r);
        gstart.alloc(sizeof(int) * size_t(ngroups + 1));
        spc5cuda::launch_partition(nbr(), brptr.as<int>(), ngroups, gstart.as<int>(), s);
        int max_blocks = 0, max_values = 0;
        spc5cuda::blockrow_max(nbr(), brptr.as<int>(), valptr.as<int>(), &max_blocks, &max_values, s);
        rows_ok = spc5cuda::rows_fit(value_type, r, max_blocks, max_values);
        if (rows_ok) {
            nwarps = spc5cuda::rows_warps(value_type, r);
            wstart.alloc(sizeof(int) * size_t(nwarps + 1));
            spc5cuda::launch_partition(nbr(), brptr.as<int>(), nwarps, wstart.as<int>(), s);
        } else {
            nwarps = 0;
            wstart.release();
        }
        restore_original(s);  // the plan may hold the only copy
        plan.reset();
        if (wants_plan()) spc5cuda::build_sorted_plan(this, s);
    }
};


namespace spc5cuda {

// Block counts per block-row of a CSR handle for rows-per-block r, scanned
// into brptr_out (ceil(nrows/r)+1 ints); returns the total (synchronises s).
long count_blocks(const spc5cuda_mat* m, int r, int* brptr_out, cudaStream_t s);

// Value offsets of every block-row from the header masks.
void valptr_from_headers(int mask_bytes, int r, int nbr, const int* brptr, const uint8_t* headers,
                         int* valptr, cudaStream_t s);

}  // namespace spc5cuda
