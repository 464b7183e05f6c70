// convert.cu -- CSR -> beta(r,VS) conversion on the device, plus the scans
// and per-block-row offsets the SpMV kernels use.
//
// The conversion is the reference's greedy (core_CSR_to_SPC5_rVc,
// src/spc5.hpp:165-228; CSR_to_SPC5_1rVc 455-488) run as two passes over
// independent block-rows:
//   pass 1  counts[br]  = blocks of block-row br         (k_blockrow_counts)
//   scan    brptr       = exclusive scan of the counts   (== rowsSize after
//                                                         conversion, 220-227)
//   pass 2  headers + values of block-row br at brptr[br] and at the CSR
//           value offset rowptr[br*r]                    (k_emit)
// Inside a block-row the greedy is a sequential chain (the next block starts
// at the smallest unconsumed column of the r sub-rows), so one thread walks
// one block-row; block-rows are independent and run in parallel.  Values are
// copied bit for bit, so the arrays equal the reference's exactly.
#include <climits>

#include "common.cuh"
#include "kernels.h"

namespace spc5cuda {

// ---------------------------------------------------------------------------
// exclusive scan (int32), three phases: tile sums, scan of tile sums, tiles
// ---------------------------------------------------------------------------

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int warp_inclusive_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_sums[32];
    __shared__ int block_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int inc = warp_inclusive_scan(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < nwarps ? warp_sums[lane] : 0;
        const int wi = warp_inclusive_scan(w);
        if (lane < nwarps) warp_sums[lane] = wi - w;
        if (lane == 31) block_total = wi;
    }
    __syncthreads();
    const int res = inc - v + warp_sums[warp];
    if (total) *total = block_total;
    __syncthreads();
    return res;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(const int* __restrict__ in, long n,
                                                            int* __restrict__ sums) {
    const long base = long(blockIdx.x) * SCAN_TILE;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long i = base + long(k) * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    int total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One CTA scans the tile sums in place (exclusive) and writes the grand
// total to sums[ntiles].
__global__ void __launch_bounds__(1024) k_scan_sums(int* __restrict__ sums, long ntiles) {
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long b = 0; b < ntiles; b += blockDim.x) {
        const long i = b + threadIdx.x;
        const int v = i < ntiles ? sums[i] : 0;
        int total;
        const int ex = block_exclusive_scan(v, &total);
        const int c = carry;
        if (i < ntiles) sums[i] = c + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const int* in, int* out, long n,
                                                             const int* __restrict__ sums,
                                                             long ntiles) {
    const long base = long(blockIdx.x) * SCAN_TILE;
    // thread t owns items [base + t*ITEMS, +ITEMS): blocked arrangement
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long i = base + long(threadIdx.x) * SCAN_ITEMS + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    int running = block_exclusive_scan(s, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long i = base + long(threadIdx.x) * SCAN_ITEMS + k;
        if (i < n) out[i] = running;
        running += v[k];
    }
    if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) out[n] = sums[ntiles];
}

}  // namespace

long scan_tmp_ints(long n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

void exclusive_scan_i32(const int* in, int* out, long n, int* tmp, cudaStream_t s) {
    if (n <= 0) {
        SPC5_CUDA(cudaMemsetAsync(out, 0, sizeof(int), s));
        return;
    }
    const long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    k_tile_sums<<<unsigned(ntiles), SCAN_THREADS, 0, s>>>(in, n, tmp);
    k_scan_sums<<<1, 1024, 0, s>>>(tmp, ntiles);
    k_scan_tiles<<<unsigned(ntiles), SCAN_THREADS, 0, s>>>(in, out, n, tmp, ntiles);
    SPC5_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// CSR validation
// ---------------------------------------------------------------------------

namespace {

__global__ void k_validate_csr(int nrows, int ncols, long nnz, const int* __restrict__ rowptr,
                               const int* __restrict__ colidx, int* __restrict__ flag) {
    const long stride = long(gridDim.x) * blockDim.x;
    const long tid = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (tid == 0 && (rowptr[0] != 0 || long(rowptr[nrows]) != nnz)) atomicMax(flag, 1);
    for (long i = tid; i < nrows; i += stride) {
        const int a = rowptr[i], b = rowptr[i + 1];
        if (b < a || a < 0 || long(b) > nnz) {
            atomicMax(flag, 1);
            continue;
        }
        int prev = -1;
        for (int k = a; k < b; ++k) {
            const int c = colidx[k];
            if (c < 0 || c >= ncols) {
                atomicMax(flag, 2);
                break;
            }
            if (c <= prev) {
                atomicMax(flag, 3);
                break;
            }
            prev = c;
        }
    }
}

}  // namespace

void launch_validate_csr(int nrows, int ncols, long nnz, const int* rowptr, const int* colidx,
                         int* d_flag, cudaStream_t s) {
    SPC5_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
    const int threads = 256;
    const int blocks = nrows > 0 ? std::min(div_up(nrows, threads), sm_count() * 8) : 1;
    k_validate_csr<<<blocks, threads, 0, s>>>(nrows, ncols, nnz, rowptr, colidx, d_flag);
    SPC5_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// the greedy (spc5.hpp:186-218), one thread per block-row
// ---------------------------------------------------------------------------

namespace {

template <int VS, int R>
__global__ void __launch_bounds__(256) k_blockrow_counts(int nrows, int nbr,
                                                         const int* __restrict__ rowptr,
                                                         const int* __restrict__ colidx,
                                                         int* __restrict__ counts) {
    for (long br = long(blockIdx.x) * blockDim.x + threadIdx.x; br < nbr;
         br += long(gridDim.x) * blockDim.x) {
        const long row0 = br * R;
        int head[R], end[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const bool ok = row0 + i < nrows;
            head[i] = ok ? rowptr[row0 + i] : 0;
            end[i] = ok ? rowptr[row0 + i + 1] : 0;
        }
        int cnt = 0;
        for (;;) {
            bool have = false;
            int idx = INT_MAX;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if (head[i] < end[i]) {
                    have = true;
                    idx = min(idx, __ldg(colidx + head[i]));
                }
            }
            if (!have) break;
            ++cnt;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                // columns inside a row ascend, so col >= idx: col < idx + VS
                // is col - idx < VS without the int overflow of idx + VS
                while (head[i] < end[i] && __ldg(colidx + head[i]) - idx < VS) ++head[i];
            }
        }
        counts[br] = cnt;
    }
}

template <int VS, int R, class V>
__global__ void __launch_bounds__(256) k_emit(int nrows, int nbr, const int* __restrict__ rowptr,
                                              const int* __restrict__ colidx,
                                              const V* __restrict__ vin,
                                              const int* __restrict__ brptr,
                                              uint8_t* __restrict__ headers, V* __restrict__ vout) {
    constexpr int MB = VS == 8 ? 1 : 2;
    constexpr int STRIDE = 4 + R * MB;
    for (long br = long(blockIdx.x) * blockDim.x + threadIdx.x; br < nbr;
         br += long(gridDim.x) * blockDim.x) {
        const long row0 = br * R;
        int head[R], end[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const bool ok = row0 + i < nrows;
            head[i] = ok ? rowptr[row0 + i] : 0;
            end[i] = ok ? rowptr[row0 + i + 1] : 0;
        }
        long vo = rowptr[row0];
        uint8_t* h = headers + long(brptr[br]) * STRIDE;
        for (;;) {
            bool have = false;
            int idx = INT_MAX;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if (head[i] < end[i]) {
                    have = true;
                    idx = min(idx, __ldg(colidx + head[i]));
                }
            }
            if (!have) break;
            h[0] = uint8_t(idx);
            h[1] = uint8_t(idx >> 8);
            h[2] = uint8_t(idx >> 16);
            h[3] = uint8_t(idx >> 24);
#pragma unroll
            for (int i = 0; i < R; ++i) {
                uint32_t m = 0;
                while (head[i] < end[i]) {
                    const int d = __ldg(colidx + head[i]) - idx;
                    if (d >= VS) break;
                    vout[vo++] = vin[head[i]];
                    m |= 1u << d;
                    ++head[i];
                }
                h[4 + i * MB] = uint8_t(m);
                if (MB == 2) h[5 + i * MB] = uint8_t(m >> 8);
            }
            h += STRIDE;
        }
    }
}

__global__ void k_valptr_from_csr(int r, int nrows, int nbr, const int* __restrict__ rowptr,
                                  int* __restrict__ valptr) {
    for (long br = long(blockIdx.x) * blockDim.x + threadIdx.x; br <= nbr;
         br += long(gridDim.x) * blockDim.x) {
        const long row = br * r < nrows ? br * r : nrows;
        valptr[br] = rowptr[row];
    }
}

template <int MB>
__global__ void __launch_bounds__(256) k_value_counts(int r, int nbr, const int* __restrict__ brptr,
                                                      const uint8_t* __restrict__ headers,
                                                      int* __restrict__ counts) {
    const int stride = 4 + r * MB;
    for (long br = long(blockIdx.x) * blockDim.x + threadIdx.x; br < nbr;
         br += long(gridDim.x) * blockDim.x) {
        int s = 0;
        for (long b = brptr[br]; b < brptr[br + 1]; ++b) {
            const uint8_t* h = headers + b * stride + 4;
            for (int k = 0; k < r * MB; ++k) s += __popc(uint32_t(h[k]));
        }
        counts[br] = s;
    }
}

template <int VS, int R>
void counts_r(int nrows, const int* rowptr, const int* colidx, int* counts, cudaStream_t s) {
    const int nbr = div_up(nrows, R);
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(nbr, threads), sm_count() * 16));
    k_blockrow_counts<VS, R><<<blocks, threads, 0, s>>>(nrows, nbr, rowptr, colidx, counts);
}

template <int VS, int R, class V>
void emit_r(int nrows, const int* rowptr, const int* colidx, const void* vin, const int* brptr,
            uint8_t* headers, void* vout, cudaStream_t s) {
    const int nbr = div_up(nrows, R);
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(nbr, threads), sm_count() * 16));
    k_emit<VS, R, V><<<blocks, threads, 0, s>>>(nrows, nbr, rowptr, colidx,
                                               static_cast<const V*>(vin), brptr, headers,
                                               static_cast<V*>(vout));
}

}  // namespace

void launch_blockrow_counts(int vs, int r, int nrows, const int* rowptr, const int* colidx,
                            int* counts, cudaStream_t s) {
    if (nrows <= 0) return;
#define SPC5_COUNTS(VS_, R_) \
    if (vs == VS_ && r == R_) { counts_r<VS_, R_>(nrows, rowptr, colidx, counts, s); }
    SPC5_COUNTS(8, 1) else SPC5_COUNTS(8, 2) else SPC5_COUNTS(8, 4) else SPC5_COUNTS(8, 8)
    else SPC5_COUNTS(16, 1) else SPC5_COUNTS(16, 2) else SPC5_COUNTS(16, 4) else SPC5_COUNTS(16, 8)
    else throw Error(SPC5CUDA_ERR_FORMAT, "unsupported (VS, r)");
#undef SPC5_COUNTS
    SPC5_CUDA(cudaGetLastError());
}

void launch_emit(int vs, int r, int nrows, const int* rowptr, const int* colidx, const void* vin,
                 int value_bytes, const int* brptr, uint8_t* headers, void* vout, cudaStream_t s) {
    if (nrows <= 0) return;
    if (value_bytes == 8) {
#define SPC5_EMIT(VS_, R_) \
    if (vs == VS_ && r == R_) { emit_r<VS_, R_, double>(nrows, rowptr, colidx, vin, brptr, headers, vout, s); }
        SPC5_EMIT(8, 1) else SPC5_EMIT(8, 2) else SPC5_EMIT(8, 4) else SPC5_EMIT(8, 8)
        else SPC5_EMIT(16, 1) else SPC5_EMIT(16, 2) else SPC5_EMIT(16, 4) else SPC5_EMIT(16, 8)
        else throw Error(SPC5CUDA_ERR_FORMAT, "unsupported (VS, r)");
#undef SPC5_EMIT
    } else if (value_bytes == 4) {
#define SPC5_EMIT(VS_, R_) \
    if (vs == VS_ && r == R_) { emit_r<VS_, R_, float>(nrows, rowptr, colidx, vin, brptr, headers, vout, s); }
        SPC5_EMIT(8, 1) else SPC5_EMIT(8, 2) else SPC5_EMIT(8, 4) else SPC5_EMIT(8, 8)
        else SPC5_EMIT(16, 1) else SPC5_EMIT(16, 2) else SPC5_EMIT(16, 4) else SPC5_EMIT(16, 8)
        else throw Error(SPC5CUDA_ERR_FORMAT, "unsupported (VS, r)");
#undef SPC5_EMIT
    } else {
        throw Error(SPC5CUDA_ERR_INVALID, "value size must be 4 or 8");
    }
    SPC5_CUDA(cudaGetLastError());
}

void launch_valptr_from_csr(int r, int nrows, const int* rowptr, int* valptr, cudaStream_t s) {
    const int nbr = div_up(nrows, r);
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(long(nbr) + 1, threads), sm_count() * 16));
    k_valptr_from_csr<<<blocks, threads, 0, s>>>(r, nrows, nbr, rowptr, valptr);
    SPC5_CUDA(cudaGetLastError());
}

void launch_blockrow_value_counts(int mask_bytes, int r, int nbr, const int* brptr,
                                  const uint8_t* headers, int* counts, cudaStream_t s) {
    if (nbr <= 0) return;
    const int threads = 256;
    const int blocks = std::max(1, std::min(div_up(nbr, threads), sm_count() * 16));
    if (mask_bytes == 1)
        k_value_counts<1><<<blocks, threads, 0, s>>>(r, nbr, brptr, headers, counts);
    else
        k_value_counts<2><<<blocks, threads, 0, s>>>(r, nbr, brptr, headers, counts);
    SPC5_CUDA(cudaGetLastError());
}

}  // namespace spc5cuda
