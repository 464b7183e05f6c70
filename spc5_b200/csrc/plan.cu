// plan.cu -- the length-sorted SpMV plan of a matrix with irregular block-rows.
//
// Power-law and other irregular matrices mix block-rows of one block with
// block-rows of hundreds; no single work split suits both.  The plan keeps a
// copy of the matrix with its block-rows sorted by size (largest first) --
// every block-row keeps its own blocks and values in their order, so every
// accumulator sees the same FMA chain and y is bit-identical -- plus perm[i],
// the block-row of y that sorted block-row i belongs to.  The sorted order is
// cut into parts, each run by the kernel that suits its block-rows:
//   * block-rows too large for the row kernel's chunks (above the class of
//     L = 8 lanes), at r = 2, 4, 8: the chain part (chain.cu), one lane per
//     (sub-row, column) multiply-add chain, chains sorted by length;
//   * the same at r = 1: cut into segments of at most L/32 of a
//     chunk's buffers (greedy, in block order), the segments of 32 / L
//     neighbouring block-rows interleaved so that a chunk holds segment k of
//     each of them; the row kernel (L lanes per block-row) then stages them
//     like short block-rows while every lane keeps its block-row's
//     accumulators from chunk to chunk;
//   * the rest: the row kernel with L = 8, 4, 2 or 1 lanes per block-row,
//     the smallest L whose chunk of 32 / L block-rows fits the staging
//     buffers.  Block-rows of one chunk have about the same size, so no lane
//     waits for a much longer neighbour.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

#include "handle.h"

namespace spc5cuda {

namespace {

// key[i] = size of block-row i in row-kernel lane units (rows_lane_units),
// idx[i] = i.
__global__ void k_row_keys(int nbr, const int* __restrict__ brptr, const int* __restrict__ valptr,
                           long kb, long kv, unsigned long long* __restrict__ keys, int* __restrict__ idx) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const long nb = brptr[i + 1] - brptr[i];
        const long nv = valptr[i + 1] - valptr[i];
        keys[i] = static_cast<unsigned long long>(max(nb * kb, nv * kv));
        idx[i] = int(i);
    }
}

// Block and value counts of the sorted block-rows.
__global__ void k_sorted_counts(int nbr, const int* __restrict__ perm, const int* __restrict__ brptr,
                                const int* __restrict__ valptr, int* __restrict__ snb, int* __restrict__ snv) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const int p = perm[i];
        snb[i] = brptr[p + 1] - brptr[p];
        snv[i] = valptr[p + 1] - valptr[p];
    }
}

// The reference order back from the sorted copy: sorted block-row i goes to
// block-row perm[i]'s offsets (one warp per block-row); headers of the
// block-rows [a, nbr), values of [vfrom, nbr) (the others are in the chain
// part or in segments).
template <class V>
__global__ void k_unsorted_copy(int a, int vfrom, int nbr, const int* __restrict__ perm,
                                const int* __restrict__ sbrptr,
                                const int* __restrict__ svalptr, const int* __restrict__ brptr,
                                const int* __restrict__ valptr, int stride, const uint8_t* __restrict__ shdr,
                                uint8_t* __restrict__ hdr, const V* __restrict__ svals, V* __restrict__ vals) {
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * blockDim.x / 32;
    for (long i = a + (long(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < nbr; i += warps) {
        const int p = perm[i];
        const long h0 = long(sbrptr[i]) * stride, hn = long(sbrptr[i + 1]) * stride - h0;
        const long d0 = long(brptr[p]) * stride;
        for (long k = lane; k < hn; k += 32) hdr[d0 + k] = shdr[h0 + k];
        if (i < vfrom) continue;
        const long v0 = svalptr[i], vn = long(svalptr[i + 1]) - v0;
        const long w0 = valptr[p];
        for (long k = lane; k < vn; k += 32) vals[w0 + k] = svals[v0 + k];
    }
}

// The same for the segmented block-rows [0, nlong): block-row i is warp
// g = i / spw, slot s = i % spw of the segment layout; its segment k is
// segment row split[g] + k n_g + s (n_g = its warp's block-rows), and its
// segments, in order, are its blocks and values in order.
template <class V>
__global__ void k_unsegmented_copy(int nlong, int spw, const int* __restrict__ perm, const int* __restrict__ split,
                                   const int* __restrict__ vbrptr, const int* __restrict__ vvalptr,
                                   const int* __restrict__ brptr, const int* __restrict__ valptr, int stride,
                                   const uint8_t* __restrict__ shdr, uint8_t* __restrict__ hdr,
                                   const V* __restrict__ svals, V* __restrict__ vals) {
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * blockDim.x / 32;
    for (long i = (long(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < nlong; i += warps) {
        const int g = int(i) / spw, s = int(i) % spw;
        const int n = min(spw, nlong - g * spw);
        const int rows = split[g + 1] - split[g];
        const int p = perm[i];
        long hb = long(brptr[p]) * stride, vb = valptr[p];
        for (int k = 0; k * n < rows; ++k) {
            const int j = split[g] + k * n + s;
            const long h0 = long(vbrptr[j]) * stride, hn = long(vbrptr[j + 1]) * stride - h0;
            for (long t = lane; t < hn; t += 32) hdr[hb + t] = shdr[h0 + t];
            hb += hn;
            const long v0 = vvalptr[j], vn = long(vvalptr[j + 1]) - v0;
            for (long t = lane; t < vn; t += 32) vals[vb + t] = svals[v0 + t];
            vb += vn;
        }
    }
}

// Copy block-row perm[i] to sorted position i: one warp per block-row.
template <class V>
__global__ void k_sorted_copy(int nbr, const int* __restrict__ perm, const int* __restrict__ brptr,
                              const int* __restrict__ valptr, const int* __restrict__ sbrptr,
                              const int* __restrict__ svalptr, int stride, const uint8_t* __restrict__ hdr,
                              uint8_t* __restrict__ shdr, const V* __restrict__ vals, V* __restrict__ svals) {
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * blockDim.x / 32;
    for (long i = (long(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < nbr; i += warps) {
        const int p = perm[i];
        const long h0 = long(brptr[p]) * stride, hn = long(brptr[p + 1]) * stride - h0;
        const long d0 = long(sbrptr[i]) * stride;
        for (long k = lane; k < hn; k += 32) shdr[d0 + k] = hdr[h0 + k];
        const long v0 = valptr[p], vn = long(valptr[p + 1]) - v0;
        const long w0 = svalptr[i];
        for (long k = lane; k < vn; k += 32) svals[w0 + k] = vals[v0 + k];
    }
}

// counts[j] = number of sorted keys above thr[j] (keys descend).
__global__ void k_class_counts(int nbr, const unsigned long long* __restrict__ skeys,
                               unsigned long long t0, unsigned long long t1, unsigned long long t2,
                               unsigned long long t3, int* __restrict__ counts) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const unsigned long long k = skeys[i];
        const unsigned long long nk = i + 1 < nbr ? skeys[i + 1] : 0ull;
        // the last index above each threshold marks the count
        if (k > t0 && nk <= t0) counts[0] = int(i + 1);
        if (k > t1 && nk <= t1) counts[1] = int(i + 1);
        if (k > t2 && nk <= t2) counts[2] = int(i + 1);
        if (k > t3 && nk <= t3) counts[3] = int(i + 1);
    }
}

// Values of block b (popcount of its mask bytes).
__device__ __forceinline__ int block_values(const uint8_t* __restrict__ hdr, long b, int stride) {
    int n = 0;
    for (int k = 4; k < stride; ++k) n += __popc(unsigned(hdr[b * stride + k]));
    return n;
}

// Greedy cut of blocks [b0, b1) (first value v0) into segments of at most
// bmax blocks and vmax values, in block order: emit(k, first block, blocks,
// first value, values) for segment k.
template <class F>
__device__ void cut_segments(int b0, int b1, int v0, const uint8_t* __restrict__ hdr, int stride, int bmax,
                             int vmax, F&& emit) {
    int k = 0, sb = b0, sv = v0, nb = 0, nv = 0;
    for (int b = b0; b < b1; ++b) {
        const int pc = block_values(hdr, b, stride);
        if (nb > 0 && (nb + 1 > bmax || nv + pc > vmax)) {
            emit(k++, sb, nb, sv, nv);
            sb = b;
            sv += nv;
            nb = 0;
            nv = 0;
        }
        ++nb;
        nv += pc;
    }
    if (nb > 0) emit(k, sb, nb, sv, nv);
}

// nseg_of[i] = segments of sorted block-row i < nlong.
__global__ void k_seg_count(int nlong, const int* __restrict__ sbrptr, const int* __restrict__ svalptr,
                            const uint8_t* __restrict__ hdr, int stride, int bmax, int vmax,
                            int* __restrict__ nseg_of) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nlong; i += long(gridDim.x) * blockDim.x) {
        int n = 0;
        cut_segments(sbrptr[i], sbrptr[i + 1], svalptr[i], hdr, stride, bmax, vmax,
                     [&](int, int, int, int, int) { ++n; });
        nseg_of[i] = n;
    }
}

// Segment rows of warp g: (most segments of its block-rows) x (its block-rows).
__global__ void k_seg_warp_rows(int nlong, int spw, int nw, const int* __restrict__ nseg_of,
                                int* __restrict__ vrows) {
    for (long g = long(blockIdx.x) * blockDim.x + threadIdx.x; g < nw; g += long(gridDim.x) * blockDim.x) {
        const int a = int(g) * spw, n = min(spw, nlong - a);
        int most = 0;
        for (int s = 0; s < n; ++s) most = max(most, nseg_of[a + s]);
        vrows[g] = most * n;
    }
}

// Segment k of block-row i (warp g = i / spw, slot s = i % spw) is segment
// row wbase[g] + k n_g + s: its block and value counts (vnb, vnv, zero for
// the rows of block-rows with fewer segments) and where it starts in the
// sorted copy (vsb, vsv).
__global__ void k_seg_fill(int nlong, int spw, const int* __restrict__ sbrptr, const int* __restrict__ svalptr,
                           const uint8_t* __restrict__ hdr, int stride, int bmax, int vmax,
                           const int* __restrict__ wbase, int* __restrict__ vnb, int* __restrict__ vnv,
                           int* __restrict__ vsb, int* __restrict__ vsv) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nlong; i += long(gridDim.x) * blockDim.x) {
        const int g = int(i) / spw, s = int(i) % spw;
        const int n = min(spw, nlong - g * spw);
        const int base = wbase[g];
        cut_segments(sbrptr[i], sbrptr[i + 1], svalptr[i], hdr, stride, bmax, vmax,
                     [&](int k, int sb, int nb, int sv, int nv) {
                         const long v = base + long(k) * n + s;
                         vnb[v] = nb;
                         vnv[v] = nv;
                         vsb[v] = sb;
                         vsv[v] = sv;
                     });
    }
}

// Copy every segment row to its place (one warp per segment row).
template <class V>
__global__ void k_seg_copy(int nv, const int* __restrict__ vsb, const int* __restrict__ vsv,
                           const int* __restrict__ vbrptr, const int* __restrict__ vvalptr, int stride,
                           const uint8_t* __restrict__ hdr, uint8_t* __restrict__ thdr, const V* __restrict__ vals,
                           V* __restrict__ tvals) {
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * blockDim.x / 32;
    for (long v = (long(blockIdx.x) * blockDim.x + threadIdx.x) / 32; v < nv; v += warps) {
        const long nb = vbrptr[v + 1] - vbrptr[v];
        if (nb == 0) continue;
        const long h0 = long(vsb[v]) * stride, d0 = long(vbrptr[v]) * stride, hn = nb * stride;
        for (long k = lane; k < hn; k += 32) thdr[d0 + k] = hdr[h0 + k];
        const long w0 = vsv[v], e0 = vvalptr[v], en = long(vvalptr[v + 1]) - e0;
        for (long k = lane; k < en; k += 32) tvals[e0 + k] = vals[w0 + k];
    }
}

int grid_for(long n, int threads) { return std::max(1, std::min(div_up(n, threads), sm_count() * 8)); }

}  // namespace

namespace {

// Cuts the part's block-rows (sorted positions [0, nseg)) into segments of
// at most 1/32 of a chunk's buffers per lane, rewrites that region of the
// sorted copy in the interleaved segment order and builds the part's segment
// offsets and per-warp ranges (synchronises s).
void build_segments(const spc5cuda_mat* m, SortedPlan* plan, SpmvPart& part, int stride, int vbytes,
                    cudaStream_t s) {
    const int nlong = part.nseg;
    const int L = part.lanes;
    const int spw = 32 / L;
    // the budget of a block-row that L lanes stage in one chunk
    const int bmax = int(L * (rows_hb() - 32) / 32 / stride);
    const int vmax = int(L * (rows_vb() - 32) / 32 / vbytes);
    const int nw = (nlong + spw - 1) / spw;
    const int* sbrptr = plan->sbrptr.as<int>();
    const int* svalptr = plan->svalptr.as<int>();
    DevBuf nseg_of(sizeof(int) * size_t(nlong), s), vrows(sizeof(int) * size_t(nw), s);
    k_seg_count<<<grid_for(nlong, 128), 128, 0, s>>>(nlong, sbrptr, svalptr, plan->sheaders.as<uint8_t>(), stride,
                                                     bmax, vmax, nseg_of.as<int>());
    SPC5_CUDA(cudaGetLastError());
    k_seg_warp_rows<<<grid_for(nw, 128), 128, 0, s>>>(nlong, spw, nw, nseg_of.as<int>(), vrows.as<int>());
    SPC5_CUDA(cudaGetLastError());
    part.split.alloc(sizeof(int) * size_t(nw + 1));
    part.nsplit = nw;
    {
        DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nw)), s);
        exclusive_scan_i32(vrows.as<int>(), part.split.as<int>(), nw, tmp.as<int>(), s);
    }
    int nv = 0;
    SPC5_CUDA(cudaMemcpyAsync(&nv, part.split.as<int>() + nw, sizeof(int), cudaMemcpyDeviceToHost, s));
    int ends[2] = {0, 0};  // blocks and values of the part
    SPC5_CUDA(cudaMemcpyAsync(&ends[0], sbrptr + nlong, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaMemcpyAsync(&ends[1], svalptr + nlong, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    DevBuf vnb(sizeof(int) * size_t(nv), s), vnv(sizeof(int) * size_t(nv), s);
    DevBuf vsb(sizeof(int) * size_t(nv), s), vsv(sizeof(int) * size_t(nv), s);
    SPC5_CUDA(cudaMemsetAsync(vnb.p, 0, vnb.bytes, s));
    SPC5_CUDA(cudaMemsetAsync(vnv.p, 0, vnv.bytes, s));
    k_seg_fill<<<grid_for(nlong, 128), 128, 0, s>>>(nlong, spw, sbrptr, svalptr, plan->sheaders.as<uint8_t>(),
                                                    stride, bmax, vmax, part.split.as<int>(), vnb.as<int>(),
                                                    vnv.as<int>(), vsb.as<int>(), vsv.as<int>());
    SPC5_CUDA(cudaGetLastError());
    part.vbrptr.alloc(sizeof(int) * size_t(nv + 1));
    part.vvalptr.alloc(sizeof(int) * size_t(nv + 1));
    {
        DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nv)), s);
        exclusive_scan_i32(vnb.as<int>(), part.vbrptr.as<int>(), nv, tmp.as<int>(), s);
        exclusive_scan_i32(vnv.as<int>(), part.vvalptr.as<int>(), nv, tmp.as<int>(), s);
    }
    // the segments hold exactly the part's blocks and values: rewrite that
    // region of the sorted copy in segment order
    const size_t hbytes = size_t(ends[0]) * size_t(stride), vbytes_all = size_t(ends[1]) * size_t(vbytes);
    DevBuf th(std::max<size_t>(16, hbytes), s), tv(std::max<size_t>(16, vbytes_all), s);
    const int blocks = std::max(1, std::min(div_up(long(nv) * 32, 256), sm_count() * 16));
    if (m->value_type == SPC5CUDA_F64)
        k_seg_copy<double><<<blocks, 256, 0, s>>>(nv, vsb.as<int>(), vsv.as<int>(), part.vbrptr.as<int>(),
                                                  part.vvalptr.as<int>(), stride, plan->sheaders.as<uint8_t>(),
                                                  th.as<uint8_t>(), plan->svalues.as<double>(), tv.as<double>());
    else
        k_seg_copy<float><<<blocks, 256, 0, s>>>(nv, vsb.as<int>(), vsv.as<int>(), part.vbrptr.as<int>(),
                                                 part.vvalptr.as<int>(), stride, plan->sheaders.as<uint8_t>(),
                                                 th.as<uint8_t>(), plan->svalues.as<float>(), tv.as<float>());
    SPC5_CUDA(cudaGetLastError());
    if (hbytes) SPC5_CUDA(cudaMemcpyAsync(plan->sheaders.p, th.p, hbytes, cudaMemcpyDeviceToDevice, s));
    if (vbytes_all) SPC5_CUDA(cudaMemcpyAsync(plan->svalues.p, tv.p, vbytes_all, cudaMemcpyDeviceToDevice, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void build_sorted_plan(spc5cuda_mat* m, cudaStream_t s) {
    const int nbr = m->nbr();
    const int vs = vs_of(m->value_type);
    const int r = m->r;
    const int stride = 4 + r * mask_bytes_of(m->value_type);
    const int vbytes = value_bytes_of(m->value_type);
    auto plan = std::make_unique<SortedPlan>();
    if (nbr <= 0) {
        m->plan = std::move(plan);
        return;
    }
    // ---- sort the block-rows by size, largest first (stable)
    DevBuf keys(sizeof(unsigned long long) * size_t(nbr), s), skeys(sizeof(unsigned long long) * size_t(nbr), s);
    DevBuf idx(sizeof(int) * size_t(nbr), s);
    plan->perm.alloc(sizeof(int) * size_t(nbr));
    const long kb = rows_lane_units(m->value_type, r, 1, 0), kv = rows_lane_units(m->value_type, r, 0, 1);
    k_row_keys<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, m->brptr.as<int>(), m->valptr.as<int>(), kb, kv,
                                                  keys.as<unsigned long long>(), idx.as<int>());
    SPC5_CUDA(cudaGetLastError());
    size_t temp = 0;
    SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, temp, keys.as<unsigned long long>(),
                                                        skeys.as<unsigned long long>(), idx.as<int>(),
                                                        plan->perm.as<int>(), nbr, 0, 64, s));
    {
        DevBuf tmp(temp, s);
        SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, temp, keys.as<unsigned long long>(),
                                                            skeys.as<unsigned long long>(), idx.as<int>(),
                                                            plan->perm.as<int>(), nbr, 0, 64, s));
    }
    // ---- sorted block-row and value offsets, then the copy
    plan->sbrptr.alloc(sizeof(int) * size_t(nbr + 1));
    plan->svalptr.alloc(sizeof(int) * size_t(nbr + 1));
    {
        DevBuf snb(sizeof(int) * size_t(nbr), s), snv(sizeof(int) * size_t(nbr), s);
        k_sorted_counts<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, plan->perm.as<int>(), m->brptr.as<int>(),
                                                           m->valptr.as<int>(), snb.as<int>(), snv.as<int>());
        SPC5_CUDA(cudaGetLastError());
        DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nbr)), s);
        exclusive_scan_i32(snb.as<int>(), plan->sbrptr.as<int>(), nbr, tmp.as<int>(), s);
        exclusive_scan_i32(snv.as<int>(), plan->svalptr.as<int>(), nbr, tmp.as<int>(), s);
    }
    plan->sheaders.alloc(size_t(std::max(16L, m->nblocks * long(stride) + 16)));
    plan->svalues.alloc(size_t(std::max(16L, (m->nnz + 8) * long(vbytes))));
    {
        const int threads = 256;
        const int blocks = std::max(1, std::min(div_up(long(nbr) * 32, threads), sm_count() * 16));
        if (m->value_type == SPC5CUDA_F64)
            k_sorted_copy<double><<<blocks, threads, 0, s>>>(
                nbr, plan->perm.as<int>(), m->brptr.as<int>(), m->valptr.as<int>(), plan->sbrptr.as<int>(),
                plan->svalptr.as<int>(), stride, m->headers.as<uint8_t>(), plan->sheaders.as<uint8_t>(),
                m->values.as<double>(), plan->svalues.as<double>());
        else
            k_sorted_copy<float><<<blocks, threads, 0, s>>>(
                nbr, plan->perm.as<int>(), m->brptr.as<int>(), m->valptr.as<int>(), plan->sbrptr.as<int>(),
                plan->svalptr.as<int>(), stride, m->headers.as<uint8_t>(), plan->sheaders.as<uint8_t>(),
                m->values.as<float>(), plan->svalues.as<float>());
        SPC5_CUDA(cudaGetLastError());
    }
    // ---- parts: sizes above 8, 4, 2, 1 lane units
    int counts[4] = {0, 0, 0, 0};
    {
        DevBuf dc(4 * sizeof(int), s);
        SPC5_CUDA(cudaMemsetAsync(dc.p, 0, 4 * sizeof(int), s));
        const unsigned long long u = static_cast<unsigned long long>(rows_unit());
        k_class_counts<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, skeys.as<unsigned long long>(), 8 * u, 4 * u,
                                                          2 * u, u, dc.as<int>());
        SPC5_CUDA(cudaGetLastError());
        SPC5_CUDA(cudaMemcpyAsync(counts, dc.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
        SPC5_CUDA(cudaStreamSynchronize(s));
    }
    // counts[j]: block-rows above the limit of L = 8 >> j lanes; every
    // boundary is at least the previous one (sizes descend)
    // the chain part for r >= 2, the segmented part at r = 1, measured on B200
    // (power-law N = 4M, FP64 / mixed us per SpMV): chains at r = 2 497 / 519
    // against segments 568 / 608, r = 4 519 / 560 against 651 / 785, r = 8
    // 564 / 761 against 940 / 784; segments at r = 1 475 / 369 against chains
    // 527 / 576.  The chain part takes the block-rows above the limit of
    // 8 >> chain_class[r] lanes (the smaller ones run faster as chains than on
    // the row kernel too): r = 2 above 2 lanes (408 / 405 us, against 501 /
    // 518 above 8 and 548 / 508 with every block-row in chains), r = 4 above 4
    // lanes (459 / 487 against 517 / 575), r = 8 above 2 lanes (548 / 509
    // against 563 / 679)
    static constexpr int chain_class[9] = {0, 0, 2, 0, 1, 0, 0, 0, 2};
    const int nbig = r >= 2 ? counts[chain_class[r]] : counts[0];
    int lo = nbig;
    if (nbig > 0) {
        SpmvPart big;
        big.a = 0;
        big.b = nbig;
        big.nseg = nbig;
        big.chains = r >= 2;
        big.lanes = big.chains ? 0 : seg_lanes(r);
        plan->parts.push_back(std::move(big));
    }
    const int lanes_of[4] = {8, 4, 2, 1};
    for (int j = 0; j < 4; ++j) {
        const int L = lanes_of[j];
        if (L < r) break;
        // block-rows of this part: above the next smaller class's limit (or
        // all the rest when the next class is below r)
        const bool last = j == 3 || lanes_of[j + 1] < r;
        const int hi = last ? nbr : std::max(lo, counts[j + 1]);
        if (hi > lo) plan->parts.push_back({L, lo, hi});
        lo = hi;
        if (last) break;
    }
    // ---- a balanced split of every part
    for (auto& part : plan->parts) {
        const int rows = part.b - part.a;
        if (part.chains) {
            build_chains(m, plan.get(), part, s);
            // the chain part and the row kernel's parts contend for the
            // SMs' load pipes: one after the other they run faster than
            // concurrently (power-law N = 4M, r = 8, B200: FP64 563 against
            // 688 us, mixed 8-column layout 679 against 759 us)
            plan->in_order = true;
            continue;
        }
        if (part.nseg > 0) {
            build_segments(m, plan.get(), part, stride, vbytes, s);
            continue;
        }
        if (part.lanes == 0) {
            part.nsplit = std::max(1, std::min(spmv_groups(vs, r), rows));
        } else {
            const int per_chunk = 32 / part.lanes;
            part.nsplit = std::max(1, std::min(rows_warps(m->value_type, r, part.lanes), (rows + per_chunk - 1) / per_chunk));
        }
        part.split.alloc(sizeof(int) * size_t(part.nsplit + 1));
        launch_partition_range(part.a, part.b, plan->sbrptr.as<int>(), part.nsplit, part.split.as<int>(), s);
    }
    for (auto& st : plan->aux) SPC5_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    SPC5_CUDA(cudaEventCreateWithFlags(&plan->fork, cudaEventDisableTiming));
    for (auto& e : plan->join) SPC5_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SPC5_CUDA(cudaStreamSynchronize(s));
    m->plan = std::move(plan);
    // the sorted copy serves every SpMV now: the reference-order headers and
    // values are rebuilt from it when a call needs them (restore_original)
    if (m->use_plan()) {
        m->headers.release();
        m->values.release();
        m->original_dropped = true;
    }
}

void rebuild_original(const spc5cuda_mat* m, uint8_t* headers, void* values, cudaStream_t s) {
    const SortedPlan& p = *m->plan;
    const int nbr = m->nbr();
    const int stride = 4 + m->r * mask_bytes_of(m->value_type);
    const bool f64 = m->value_type == SPC5CUDA_F64;
    const int threads = 256;
    const SpmvPart* big = nullptr;
    for (const auto& part : p.parts)
        if (part.nseg > 0) big = &part;
    const int nlong = big ? big->nseg : 0;
    // headers of the chain part are in plain sorted order, those of the
    // segmented part in segment order (below)
    const int a = big && !big->chains ? nlong : 0;
    if (nbr > a) {
        const int blocks = std::max(1, std::min(div_up(long(nbr - a) * 32, threads), sm_count() * 16));
        if (f64)
            k_unsorted_copy<double><<<blocks, threads, 0, s>>>(
                a, nlong, nbr, p.perm.as<int>(), p.sbrptr.as<int>(), p.svalptr.as<int>(), m->brptr.as<int>(),
                m->valptr.as<int>(), stride, p.sheaders.as<uint8_t>(), headers, p.svalues.as<double>(),
                static_cast<double*>(values));
        else
            k_unsorted_copy<float><<<blocks, threads, 0, s>>>(
                a, nlong, nbr, p.perm.as<int>(), p.sbrptr.as<int>(), p.svalptr.as<int>(), m->brptr.as<int>(),
                m->valptr.as<int>(), stride, p.sheaders.as<uint8_t>(), headers, p.svalues.as<float>(),
                static_cast<float*>(values));
        SPC5_CUDA(cudaGetLastError());
    }
    if (big && big->chains) {
        unchain_values(m, *big, values, s);
    } else if (big) {
        const int spw = 32 / big->lanes;
        const int blocks = std::max(1, std::min(div_up(long(nlong) * 32, threads), sm_count() * 16));
        if (f64)
            k_unsegmented_copy<double><<<blocks, threads, 0, s>>>(
                nlong, spw, p.perm.as<int>(), big->split.as<int>(), big->vbrptr.as<int>(), big->vvalptr.as<int>(),
                m->brptr.as<int>(), m->valptr.as<int>(), stride, p.sheaders.as<uint8_t>(), headers,
                p.svalues.as<double>(), static_cast<double*>(values));
        else
            k_unsegmented_copy<float><<<blocks, threads, 0, s>>>(
                nlong, spw, p.perm.as<int>(), big->split.as<int>(), big->vbrptr.as<int>(), big->vvalptr.as<int>(),
                m->brptr.as<int>(), m->valptr.as<int>(), stride, p.sheaders.as<uint8_t>(), headers,
                p.svalues.as<float>(), static_cast<float*>(values));
        SPC5_CUDA(cudaGetLastError());
    }
}

BetaView plan_view(const spc5cuda_mat* m, const SpmvPart& part) {
    const SortedPlan& p = *m->plan;
    BetaView v;
    v.r = m->r;
    v.nrows = m->nrows;
    v.nbr = m->nbr();
    v.brptr = p.sbrptr.as<int>();
    v.headers = p.sheaders.as<uint8_t>();
    v.values = p.svalues.p;
    v.valptr = p.svalptr.as<int>();
    v.perm = p.perm.as<int>();
    if (part.nseg > 0) {
        v.brptr = part.vbrptr.as<int>();
        v.valptr = part.vvalptr.as<int>();
        v.nseg = part.nseg;
    }
    if (part.lanes == 0) {
        v.gstart = part.split.as<int>();
        v.ngroups = part.nsplit;
    } else {
        v.wstart = part.split.as<int>();
        v.nwarps = part.nsplit;
        v.lanes = part.lanes;
    }
    return v;
}

namespace {

// Runs launch(part, stream) for every part of the plan: the parts write
// disjoint rows of y, so the part of the largest block-rows runs on one plan
// stream, the smaller row-kernel parts on the other, the largest of those on
// the caller's stream; all start after the work already queued on s and s
// waits for all of them.  Without fork, or for a plan whose parts run
// faster in order (in_order), they run one after another on s.
template <class F>
void run_parts(const spc5cuda_mat* m, cudaStream_t s, bool fork, F&& launch) {
    SortedPlan& p = *m->plan;
    if (!fork || p.in_order) {
        // the parts one after another on the caller's stream: no shared plan
        // streams, so calls on different streams overlap freely
        for (const auto& part : p.parts) launch(part, s);
        return;
    }
    std::lock_guard<std::mutex> lk(p.mu);
    SPC5_CUDA(cudaEventRecord(p.fork, s));
    for (auto st : p.aux) SPC5_CUDA(cudaStreamWaitEvent(st, p.fork, 0));
    int biggest = -1;
    long most = -1;
    for (size_t i = 0; i < p.parts.size(); ++i) {
        const long blocks = (p.parts[i].lanes && !p.parts[i].nseg) ? long(p.parts[i].b - p.parts[i].a) : -1;
        if (blocks > most) most = blocks, biggest = int(i);
    }
    for (size_t i = 0; i < p.parts.size(); ++i) {
        const auto& part = p.parts[i];
        cudaStream_t st = (part.lanes == 0 || part.nseg) ? p.aux[0] : (int(i) == biggest ? s : p.aux[1]);
        launch(part, st);
    }
    for (int k = 0; k < 2; ++k) {
        SPC5_CUDA(cudaEventRecord(p.join[k], p.aux[k]));
        SPC5_CUDA(cudaStreamWaitEvent(s, p.join[k], 0));
    }
}

}  // namespace

void plan_spmv(const spc5cuda_mat* m, const void* x, void* y, bool mixed, cudaStream_t s, bool fork) {
    // the launchers pick the row kernel when the view has warp ranges
    run_parts(m, s, fork, [&](const SpmvPart& part, cudaStream_t st) {
        if (part.chains) {
            chain_part_spmv(m, part, x, y, mixed, st);
            return;
        }
        const BetaView v = plan_view(m, part);
        if (m->value_type == SPC5CUDA_F64)
            launch_spmv_f64(v, static_cast<const double*>(x), static_cast<double*>(y), st);
        else if (m->value_type == SPC5CUDA_F32_V8)
            launch_spmv_mixed8(v, static_cast<const float*>(x), static_cast<double*>(y), st);
        else if (mixed)
            launch_spmv_mixed(v, static_cast<const float*>(x), static_cast<double*>(y), st);
        else
            launch_spmv_f32(v, static_cast<const float*>(x), static_cast<float*>(y), st);
    });
}

void plan_spmm(const spc5cuda_mat* m, int k, const void* x, long ldx, long xcs, void* y, long ldy, long ycs,
               bool mixed, cudaStream_t s, bool fork) {
    run_parts(m, s, fork, [&](const SpmvPart& part, cudaStream_t st) {
        if (part.chains) {
            chain_part_spmm(m, part, k, x, ldx, xcs, y, ldy, ycs, mixed, st);
            return;
        }
        const BetaView v = plan_view(m, part);
        if (!v.wstart) throw Error(SPC5CUDA_ERR_INVALID, "plan part without warp ranges");
        if (m->value_type == SPC5CUDA_F64)
            launch_spmm_rows_f64(v, k, static_cast<const double*>(x), ldx, xcs, static_cast<double*>(y), ldy, ycs,
                                 st);
        else if (m->value_type == SPC5CUDA_F32_V8)
            launch_spmm_rows_mixed8(v, k, static_cast<const float*>(x), ldx, xcs, static_cast<double*>(y), ldy,
                                    ycs, st);
        else if (mixed)
            launch_spmm_rows_mixed(v, k, static_cast<const float*>(x), ldx, xcs, static_cast<double*>(y), ldy, ycs,
                                   st);
        else
            launch_spmm_rows_f32(v, k, static_cast<const float*>(x), ldx, xcs, static_cast<float*>(y), ldy, ycs,
                                 st);
    });
}

}  // namespace spc5cuda
