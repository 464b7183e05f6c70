// coo.cu -- COO -> CSR on the device, and beta(r,VS) -> COO decode.
//
// COO -> CSR follows COO_sorted_to_CSR / COO_unsorted_to_CSR (src/spc5.hpp:
// 77-114): unsorted triplets are sorted by (row, column) -- a radix sort of
// the 64-bit key row * ncols + column (CUB, a stable sort like the
// reference's std::sort comparator on distinct keys) -- then rows are
// counted into rowptr[i + 1] and scanned.
//
// The decode is the corrected form of core_SPC5_rVc_iterate (spc5.hpp:
// 255-273; the reference indexes the masks by block-row instead of sub-row,
// line 263): one thread per block-row walks its blocks and emits
// (row, column, value) in storage order.
#include <cub/device/device_radix_sort.cuh>

#include "handle.h"

namespace spc5cuda {
namespace {

template <int MB>
__global__ void k_decode(int r, int nrows, int nbr, const int* __restrict__ brptr,
                         const uint8_t* __restrict__ headers, const int* __restrict__ valptr,
                         const void* __restrict__ values, int value_bytes, int* __restrict__ rows,
                         int* __restrict__ cols, void* __restrict__ vout) {
    constexpr int VS = MB == 1 ? 8 : 16;
    const int stride = 4 + r * MB;
    for (long br = long(blockIdx.x) * blockDim.x + threadIdx.x; br < nbr;
         br += long(gridDim.x) * blockDim.x) {
        int v = valptr[br];
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const uint8_t* h = headers + long(b) * stride;
            const int col = int(uint32_t(h[0]) | (uint32_t(h[1]) << 8) | (uint32_t(h[2]) << 16) |
                                (uint32_t(h[3]) << 24));
            for (int i = 0; i < r; ++i) {
                uint32_t m = h[4 + i * MB];
                if (MB == 2) m |= uint32_t(h[5 + i * MB]) << 8;
                for (int c = 0; c < VS; ++c) {
                    if ((m >> c) & 1u) {
                        rows[v] = int(br) * r + i;
                        cols[v] = col + c;
                        if (value_bytes == 8)
                            static_cast<double*>(vout)[v] = static_cast<const double*>(values)[v];
                        else
                            static_cast<float*>(vout)[v] = static_cast<const float*>(values)[v];
                        ++v;
                    }
                }
            }
        }
    }
}

__global__ void k_keys(long nnz, long ncols, const int* __restrict__ rows,
                       const int* __restrict__ cols, unsigned long long* __restrict__ keys,
                       int* __restrict__ idx) {
    for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz;
         k += long(gridDim.x) * blockDim.x) {
        keys[k] = (unsigned long long)(rows[k]) * (unsigned long long)(ncols) +
                  (unsigned long long)(cols[k]);
        idx[k] = int(k);
    }
}

template <class T>
__global__ void k_gather(long nnz, long ncols, const unsigned long long* __restrict__ keys,
                         const int* __restrict__ perm, const T* __restrict__ vin,
                         int* __restrict__ rows_out, int* __restrict__ cols_out,
                         T* __restrict__ vout) {
    for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz;
         k += long(gridDim.x) * blockDim.x) {
        rows_out[k] = int(keys[k] / (unsigned long long)ncols);
        cols_out[k] = int(keys[k] % (unsigned long long)ncols);
        vout[k] = vin[perm[k]];
    }
}

// rowptr[i + 1] = number of entries of row i (rows in range), rowptr[0] = 0;
// entries with a row outside [0, nrows) raise *flag.
__global__ void k_row_counts(long nnz, int nrows, const int* __restrict__ rows,
                             int* __restrict__ counts, int* __restrict__ flag) {
    for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz;
         k += long(gridDim.x) * blockDim.x) {
        const int rw = rows[k];
        if (rw < 0 || rw >= nrows) atomicMax(flag, 1);
        else atomicAdd(counts + rw, 1);
    }
}

int grid_for(long n) { return int(std::max(1L, std::min((n + 255) / 256, long(sm_count()) * 16))); }

}  // namespace
}  // namespace spc5cuda

using namespace spc5cuda;

extern "C" {

spc5cuda_status spc5cuda_decode_coo(const spc5cuda_mat* m, int* rows, int* cols, void* values,
                                    void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        if (m->nnz == 0 || m->nrows == 0) return;
        require(rows && cols && values, SPC5CUDA_ERR_INVALID, "null output");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int nbr = m->nbr();
        const uint8_t* hdr = m->headers.as<uint8_t>();
        const void* vals = m->values.p;
        const bool rebuild = m->original_dropped;  // the sorted copy holds the only one
        DevBuf th(rebuild ? std::max<size_t>(16, m->header_bytes()) : 0, s);
        DevBuf tv(rebuild ? std::max<size_t>(16, m->value_bytes()) : 0, s);
        if (rebuild) {
            rebuild_original(m, th.as<uint8_t>(), tv.p, s);
            hdr = th.as<uint8_t>();
            vals = tv.p;
        }
        if (mask_bytes_of(m->value_type) == 1)
            k_decode<1><<<grid_for(nbr), 256, 0, s>>>(m->r, m->nrows, nbr, m->brptr.as<int>(), hdr,
                                                      m->valptr.as<int>(), vals, value_bytes_of(m->value_type),
                                                      rows, cols, values);
        else
            k_decode<2><<<grid_for(nbr), 256, 0, s>>>(m->r, m->nrows, nbr, m->brptr.as<int>(), hdr,
                                                      m->valptr.as<int>(), vals, value_bytes_of(m->value_type),
                                                      rows, cols, values);
        SPC5_CUDA(cudaGetLastError());
    });
}

spc5cuda_status spc5cuda_mat_create_coo(spc5cuda_mat** out, int value_type, int nrows, int ncols,
                                        long nnz, const int* rows, const int* cols,
                                        const void* values, int on_device, int sorted,
                                        void* stream) {
    return guarded([&] {
        require(out != nullptr, SPC5CUDA_ERR_INVALID, "null out");
        *out = nullptr;
        require(valid_value_type(value_type), SPC5CUDA_ERR_INVALID,
                "value type");
        require(nrows >= 0 && ncols >= 0 && nnz >= 0 && nnz < (1L << 31), SPC5CUDA_ERR_INVALID,
                "sizes");
        require(nnz == 0 || (rows && cols && values), SPC5CUDA_ERR_INVALID, "null array");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t vb = size_t(value_bytes_of(value_type));
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        DevBuf r_in(sizeof(int) * size_t(nnz) + 4, s), c_in(sizeof(int) * size_t(nnz) + 4, s),
            v_in(vb * size_t(nnz) + 8, s);
        if (nnz) {
            SPC5_CUDA(cudaMemcpyAsync(r_in.p, rows, sizeof(int) * size_t(nnz), kind, s));
            SPC5_CUDA(cudaMemcpyAsync(c_in.p, cols, sizeof(int) * size_t(nnz), kind, s));
            SPC5_CUDA(cudaMemcpyAsync(v_in.p, values, vb * size_t(nnz), kind, s));
        }
        DevBuf r_s(sizeof(int) * size_t(nnz) + 4, s), c_s(sizeof(int) * size_t(nnz) + 4, s),
            v_s(vb * size_t(nnz) + 8, s);
        const int* rsrc = r_in.as<int>();
        const int* csrc = c_in.as<int>();
        const void* vsrc = v_in.p;
        if (!sorted && nnz > 1) {
            // COO_unsorted_to_CSR: sort by (row, column)
            DevBuf keys(sizeof(unsigned long long) * size_t(nnz), s),
                keys2(sizeof(unsigned long long) * size_t(nnz), s), idx(sizeof(int) * size_t(nnz), s),
                idx2(sizeof(int) * size_t(nnz), s);
            k_keys<<<grid_for(nnz), 256, 0, s>>>(nnz, ncols, r_in.as<int>(), c_in.as<int>(),
                                                 keys.as<unsigned long long>(), idx.as<int>());
            size_t temp = 0;
            SPC5_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.as<unsigned long long>(),
                                                      keys2.as<unsigned long long>(), idx.as<int>(),
                                                      idx2.as<int>(), int(nnz), 0, 64, s));
            DevBuf tmp(temp + 16, s);
            SPC5_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, temp, keys.as<unsigned long long>(),
                                                      keys2.as<unsigned long long>(), idx.as<int>(),
                                                      idx2.as<int>(), int(nnz), 0, 64, s));
            if (vb == 8)
                k_gather<double><<<grid_for(nnz), 256, 0, s>>>(
                    nnz, ncols, keys2.as<unsigned long long>(), idx2.as<int>(), v_in.as<double>(),
                    r_s.as<int>(), c_s.as<int>(), v_s.as<double>());
            else
                k_gather<float><<<grid_for(nnz), 256, 0, s>>>(
                    nnz, ncols, keys2.as<unsigned long long>(), idx2.as<int>(), v_in.as<float>(),
                    r_s.as<int>(), c_s.as<int>(), v_s.as<float>());
            SPC5_CUDA(cudaGetLastError());
            rsrc = r_s.as<int>();
            csrc = c_s.as<int>();
            vsrc = v_s.p;
            SPC5_CUDA(cudaStreamSynchronize(s));
        }
        // COO_sorted_to_CSR: histogram of rows, then exclusive scan
        DevBuf counts(sizeof(int) * size_t(nrows + 1), s), flag(sizeof(int), s),
            scan_tmp(sizeof(int) * size_t(scan_tmp_ints(nrows) + 1), s);
        SPC5_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * size_t(nrows + 1), s));
        SPC5_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
        if (nnz)
            k_row_counts<<<grid_for(nnz), 256, 0, s>>>(nnz, nrows, rsrc, counts.as<int>(),
                                                       flag.as<int>());
        int bad = 0;
        SPC5_CUDA(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        SPC5_CUDA(cudaStreamSynchronize(s));
        require(bad == 0, SPC5CUDA_ERR_INVALID, "row index out of range");
        exclusive_scan_i32(counts.as<int>(), counts.as<int>(), nrows, scan_tmp.as<int>(), s);
        SPC5_CUDA(cudaStreamSynchronize(s));
        // the CSR handle copies and validates (sorted, unique, in-range columns)
        const spc5cuda_status st = spc5cuda_mat_create_csr(out, value_type, nrows, ncols, nnz,
                                                           counts.as<int>(), csrc, vsrc, 1, stream);
        if (st != SPC5CUDA_OK) throw Error(st, "COO -> CSR");
    });
}

}  // extern "C"
