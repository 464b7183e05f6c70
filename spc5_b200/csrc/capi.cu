// capi.cu -- the C ABI (include/spc5cuda.h): matrix handles, device
// conversion, drop-in kernels.  Every entry point catches the internal
// spc5cuda::Error and returns a status code; nothing throws across the ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "handle.h"

namespace spc5cuda {

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    SPC5_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) dev = 0;
    if (cached[dev] == 0) {
        int n = 0;
        SPC5_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        cached[dev] = n > 0 ? n : 1;
    }
    return cached[dev];
}

namespace {

thread_local spc5cuda_status g_last_error = SPC5CUDA_OK;
thread_local cudaStream_t g_stream = nullptr;

}  // namespace
}  // namespace spc5cuda

using namespace spc5cuda;

namespace {

void copy_in(Owned& dst, const void* src, size_t bytes, int on_device, cudaStream_t s) {
    dst.alloc(bytes);
    if (bytes)
        SPC5_CUDA(cudaMemcpyAsync(dst.p, src, bytes,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
}

// Runs the validation kernel and turns its flag into a status.
void validate_csr(const spc5cuda_mat* m, cudaStream_t s) {
    DevBuf flag(sizeof(int), s);
    launch_validate_csr(m->nrows, m->ncols, m->nnz, m->rowptr.as<int>(), m->colidx.as<int>(),
                        flag.as<int>(), s);
    int h = 0;
    SPC5_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    if (h != 0) throw Error(SPC5CUDA_ERR_INVALID, "malformed CSR");
}

}  // namespace

long spc5cuda::count_blocks(const spc5cuda_mat* m, int r, int* brptr_out, cudaStream_t s) {
    const long nbr = div_up(m->nrows, r);
    DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nbr) + 1), s);
    launch_blockrow_counts(vs_of(m->value_type), r, m->nrows, m->rowptr.as<int>(),
                           m->colidx.as<int>(), brptr_out, s);
    exclusive_scan_i32(brptr_out, brptr_out, nbr, tmp.as<int>(), s);
    int total = 0;
    SPC5_CUDA(cudaMemcpyAsync(&total, brptr_out + nbr, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPC5_CUDA(cudaStreamSynchronize(s));
    return total;
}

void spc5cuda::valptr_from_headers(int mask_bytes, int r, int nbr, const int* brptr, const uint8_t* headers,
                         int* valptr, cudaStream_t s) {
    DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nbr) + 1), s);
    launch_blockrow_value_counts(mask_bytes, r, nbr, brptr, headers, valptr, s);
    exclusive_scan_i32(valptr, valptr, nbr, tmp.as<int>(), s);
}

// The library's own stream-ordered memory pool on the current device: the
// per-call scratch of the drop-in symbols and of the plan's chain part comes
// from it, and it keeps freed memory for the next call (release threshold:
// never), so repeated calls do not go back to the driver.  One pool per
// device for the process lifetime.
cudaMemPool_t spc5cuda::scratch_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    SPC5_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, SPC5CUDA_ERR_UNSUPPORTED, "device index");
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        SPC5_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t keep = UINT64_MAX;
        SPC5_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

namespace {

// core_SPC5_{r}rVc_Spmv_{double,float} over device arrays without a handle.
// Per call, all on the stream and without a host round trip: the value
// offsets of the block-rows (one pass over the headers), the largest
// block-row, the per-group and per-warp splits; then the row kernel and the
// group kernel are both enqueued, gated on a device word: the row kernel runs
// when every block-row fits its staging buffers, the group kernel otherwise.
// Both give the reference's bits.
template <class T>
void core_spmv(int r, long nbRows, const int* rowsSizes, const unsigned char* headers,
               const T* values, const T* x, T* y, cudaStream_t s) {
    require(r == 1 || r == 2 || r == 4 || r == 8, SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
    require(nbRows >= 0 && nbRows < (1L << 31), SPC5CUDA_ERR_INVALID, "nbRows out of range");
    if (nbRows == 0) return;
    // headers / values may be null only for a matrix without blocks
    require(rowsSizes && x && y, SPC5CUDA_ERR_INVALID, "null pointer");
    require(aligned(headers, 4) && aligned(values, 16) && aligned(rowsSizes, 4),
            SPC5CUDA_ERR_INVALID, "misaligned array (headers 4 bytes, values 16 bytes)");
    constexpr int vt = sizeof(T) == 8 ? SPC5CUDA_F64 : SPC5CUDA_F32;
    const int nbr = div_up(nbRows, r);
    const int ngroups = spmv_groups(vs_of(vt), r);
    const int nwarps = rows_warps(vt, r);
    PoolBuf valptr(sizeof(int) * size_t(nbr + 1), s);
    PoolBuf gstart(sizeof(int) * size_t(ngroups + 1), s);
    PoolBuf wstart(sizeof(int) * size_t(nwarps + 1), s);
    PoolBuf work(sizeof(int) * 4, s);
    {
        PoolBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nbr) + 1), s);
        launch_blockrow_value_counts(mask_bytes_of(vt), r, nbr, rowsSizes, headers, valptr.as<int>(), s);
        exclusive_scan_i32(valptr.as<int>(), valptr.as<int>(), nbr, tmp.as<int>(), s);
    }
    launch_partition(nbr, rowsSizes, ngroups, gstart.as<int>(), s);
    launch_partition(nbr, rowsSizes, nwarps, wstart.as<int>(), s);
    launch_rows_fit_flag(vt, r, nbr, rowsSizes, valptr.as<int>(), work.as<int>(), s);
    BetaView v;
    v.r = r;
    v.nrows = int(nbRows);
    v.nbr = nbr;
    v.brptr = rowsSizes;
    v.headers = headers;
    v.values = values;
    v.valptr = valptr.as<int>();
    v.gstart = gstart.as<int>();
    v.ngroups = ngroups;
    v.run_if = work.as<int>();
    BetaView vr = v;
    vr.wstart = wstart.as<int>();
    vr.nwarps = nwarps;
    v.run_if_value = 0;   // group kernel: some block-row does not fit
    vr.run_if_value = 1;  // row kernel: every block-row fits
    if constexpr (sizeof(T) == 8) {
        launch_spmv_f64(vr, x, y, s);
        launch_spmv_f64(v, x, y, s);
    } else {
        launch_spmv_f32(vr, x, y, s);
        launch_spmv_f32(v, x, y, s);
    }
}

}  // namespace

extern "C" {

const char* spc5cuda_status_string(spc5cuda_status s) {
    switch (s) {
        case SPC5CUDA_OK: return "ok";
        case SPC5CUDA_ERR_INVALID: return "invalid argument";
        case SPC5CUDA_ERR_CUDA: return "CUDA error";
        case SPC5CUDA_ERR_NOMEM: return "out of device memory";
        case SPC5CUDA_ERR_FORMAT: return "unknown format or wrong matrix state";
        case SPC5CUDA_ERR_UNSUPPORTED: return "unsupported";
        case SPC5CUDA_ERR_TIMEOUT: return "device wait timed out";
        case SPC5CUDA_ERR_DEVICE: return "device reported a data error";
        default: return "unknown status";
    }
}

spc5cuda_status spc5cuda_get_last_error(void) { return g_last_error; }

void spc5cuda_set_stream(void* stream) { g_stream = static_cast<cudaStream_t>(stream); }

spc5cuda_status spc5cuda_core_spmv_f64(int r, long nbRows, const int* rowsSizes,
                                       const unsigned char* headers, const double* values,
                                       const double* x, double* y, void* stream) {
    return guarded([&] {
        core_spmv<double>(r, nbRows, rowsSizes, headers, values, x, y,
                          static_cast<cudaStream_t>(stream));
    });
}

spc5cuda_status spc5cuda_core_spmv_f32(int r, long nbRows, const int* rowsSizes,
                                       const unsigned char* headers, const float* values,
                                       const float* x, float* y, void* stream) {
    return guarded([&] {
        core_spmv<float>(r, nbRows, rowsSizes, headers, values, x, y,
                         static_cast<cudaStream_t>(stream));
    });
}

#define SPC5_DROPIN(R_, NAME_, T_, FN_)                                                       \
    void NAME_(const long int nbRows, const int* rowsSizes,                                   \
               const unsigned char* blocksColumnIndexesWithMasks, const T_* values,           \
               const T_* x, T_* y) {                                                          \
        g_last_error =                                                                        \
            FN_(R_, nbRows, rowsSizes, blocksColumnIndexesWithMasks, values, x, y, g_stream); \
    }

SPC5_DROPIN(1, core_SPC5_1rVc_Spmv_double, double, spc5cuda_core_spmv_f64)
SPC5_DROPIN(2, core_SPC5_2rVc_Spmv_double, double, spc5cuda_core_spmv_f64)
SPC5_DROPIN(4, core_SPC5_4rVc_Spmv_double, double, spc5cuda_core_spmv_f64)
SPC5_DROPIN(8, core_SPC5_8rVc_Spmv_double, double, spc5cuda_core_spmv_f64)
SPC5_DROPIN(1, core_SPC5_1rVc_Spmv_float, float, spc5cuda_core_spmv_f32)
SPC5_DROPIN(2, core_SPC5_2rVc_Spmv_float, float, spc5cuda_core_spmv_f32)
SPC5_DROPIN(4, core_SPC5_4rVc_Spmv_float, float, spc5cuda_core_spmv_f32)
SPC5_DROPIN(8, core_SPC5_8rVc_Spmv_float, float, spc5cuda_core_spmv_f32)
#undef SPC5_DROPIN

spc5cuda_status spc5cuda_mat_create_csr(spc5cuda_mat** out, int value_type, int nrows, int ncols,
                                        long nnz, const int* rowptr, const int* colidx,
                                        const void* values, int on_device, void* stream) {
    return guarded([&] {
        require(out != nullptr, SPC5CUDA_ERR_INVALID, "null out");
        *out = nullptr;
        require(valid_value_type(value_type), SPC5CUDA_ERR_INVALID,
                "value type");
        require(nrows >= 0 && ncols >= 0 && nnz >= 0 && nnz < (1L << 31), SPC5CUDA_ERR_INVALID,
                "sizes");
        require(rowptr != nullptr && (nnz == 0 || (colidx && values)), SPC5CUDA_ERR_INVALID,
                "null array");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        auto* m = new spc5cuda_mat();
        try {
            m->value_type = value_type;
            m->format = SPC5CUDA_FORMAT_CSR;
            m->nrows = nrows;
            m->ncols = ncols;
            m->nnz = nnz;
            copy_in(m->rowptr, rowptr, sizeof(int) * size_t(nrows + 1), on_device, s);
            copy_in(m->colidx, colidx, sizeof(int) * size_t(nnz), on_device, s);
            copy_in(m->values, values, size_t(value_bytes_of(value_type)) * size_t(nnz),
                    on_device, s);
            validate_csr(m, s);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

spc5cuda_status spc5cuda_mat_create_beta(spc5cuda_mat** out, int value_type, int r, int nrows,
                                         int ncols, long nnz, long nblocks, const int* rowsSize,
                                         const unsigned char* headers, const void* values,
                                         int on_device, void* stream) {
    return guarded([&] {
        require(out != nullptr, SPC5CUDA_ERR_INVALID, "null out");
        *out = nullptr;
        require(valid_value_type(value_type), SPC5CUDA_ERR_INVALID,
                "value type");
        require(r_to_format(r) != SPC5CUDA_UNDEFINED_FORMAT, SPC5CUDA_ERR_FORMAT, "r");
        require(nrows >= 0 && ncols >= 0 && nnz >= 0 && nnz < (1L << 31) && nblocks >= 0 &&
                    nblocks < (1L << 31),
                SPC5CUDA_ERR_INVALID, "sizes");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        auto* m = new spc5cuda_mat();
        try {
            m->value_type = value_type;
            m->format = r_to_format(r);
            m->r = r;
            m->nrows = nrows;
            m->ncols = ncols;
            m->nnz = nnz;
            m->nblocks = nblocks;
            const int nbr = div_up(nrows, r);
            const size_t stride = 4 + size_t(r) * mask_bytes_of(value_type);
            copy_in(m->brptr, rowsSize, sizeof(int) * size_t(nbr + 1), on_device, s);
            copy_in(m->headers, headers, stride * size_t(nblocks), on_device, s);
            copy_in(m->values, values, size_t(value_bytes_of(value_type)) * size_t(nnz), on_device,
                    s);
            m->valptr.alloc(sizeof(int) * size_t(nbr + 1));
            if (nbr > 0) {
                valptr_from_headers(mask_bytes_of(value_type), r, nbr, m->brptr.as<int>(),
                                    m->headers.as<uint8_t>(), m->valptr.as<int>(), s);
            } else {
                SPC5_CUDA(cudaMemsetAsync(m->valptr.p, 0, sizeof(int), s));
            }
            m->build_partition(s);
            SPC5_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

spc5cuda_status spc5cuda_mat_destroy(spc5cuda_mat* mat) {
    return guarded([&] { delete mat; });
}

spc5cuda_status spc5cuda_mat_info(const spc5cuda_mat* m, spc5cuda_info* out) {
    return guarded([&] {
        require(m && out, SPC5CUDA_ERR_INVALID, "null");
        out->value_type = m->value_type;
        out->format = m->format;
        out->r = m->r;
        out->vs = vs_of(m->value_type);
        out->nrows = m->nrows;
        out->ncols = m->ncols;
        out->nnz = m->nnz;
        out->nblocks = m->nblocks;
        out->header_bytes = m->nblocks * (4 + long(m->r) * mask_bytes_of(m->value_type));
        out->device_bytes = m->device_bytes();
    });
}

spc5cuda_status spc5cuda_mat_set_kernel(spc5cuda_mat* m, int kernel) {
    return guarded([&] {
        require(m, SPC5CUDA_ERR_INVALID, "null");
        require(kernel == SPC5CUDA_KERNEL_AUTO || kernel == SPC5CUDA_KERNEL_GROUPS ||
                    kernel == SPC5CUDA_KERNEL_ROWS || kernel == SPC5CUDA_KERNEL_SORTED,
                SPC5CUDA_ERR_INVALID, "unknown kernel");
        if (kernel == SPC5CUDA_KERNEL_ROWS && m->r != 0)
            require(m->rows_ok, SPC5CUDA_ERR_UNSUPPORTED, "a block-row exceeds the row kernel's buffers");
        m->kernel = kernel;
        if (m->r != 0 && m->wants_plan() && !m->plan) build_sorted_plan(m, nullptr);
        // the group and row kernels run on the handle's own arrays: bring
        // them back from the sorted copy if it held the only one, then
        // release the copy
        if (m->plan && !m->use_plan()) {
            m->restore_original(nullptr);
            SPC5_CUDA(cudaDeviceSynchronize());  // no SpMV may still read the copy
            m->plan.reset();
        }
    });
}

spc5cuda_status spc5cuda_mat_spmv_launches(const spc5cuda_mat* m, int* launches) {
    return guarded([&] {
        require(m && launches, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        if (m->nrows == 0) *launches = 0;
        else if (m->use_plan()) {
            *launches = 0;
            for (const auto& part : m->plan->parts) *launches += part.chains ? 2 : 1;
        }
        else *launches = 1;
    });
}

spc5cuda_status spc5cuda_mat_kernel(const spc5cuda_mat* m, int* kernel) {
    return guarded([&] {
        require(m && kernel, SPC5CUDA_ERR_INVALID, "null");
        if (m->r == 0) *kernel = SPC5CUDA_KERNEL_AUTO;
        else if (m->use_plan()) *kernel = SPC5CUDA_KERNEL_SORTED;
        else *kernel = m->use_rows() ? SPC5CUDA_KERNEL_ROWS : SPC5CUDA_KERNEL_GROUPS;
    });
}

spc5cuda_status spc5cuda_block_count(const spc5cuda_mat* m, int r, long* nblocks, void* stream) {
    return guarded([&] {
        require(m && nblocks, SPC5CUDA_ERR_INVALID, "null");
        require(m->format == SPC5CUDA_FORMAT_CSR, SPC5CUDA_ERR_FORMAT, "block count needs CSR");
        require(r_to_format(r) != SPC5CUDA_UNDEFINED_FORMAT, SPC5CUDA_ERR_FORMAT, "r");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        DevBuf counts(sizeof(int) * size_t(div_up(m->nrows, r) + 1), s);
        *nblocks = count_blocks(m, r, counts.as<int>(), s);
    });
}

spc5cuda_status spc5cuda_convert(spc5cuda_mat* m, int format, void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->format == SPC5CUDA_FORMAT_CSR, SPC5CUDA_ERR_FORMAT, "matrix is not CSR");
        const int r = format_to_r(format);
        require(r != 0, SPC5CUDA_ERR_FORMAT, "CSR_to_SPC5 : Unknown format type");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int nbr = div_up(m->nrows, r);
        Owned brptr;
        brptr.alloc(sizeof(int) * size_t(nbr + 1));
        const long nb = m->nrows > 0 ? count_blocks(m, r, brptr.as<int>(), s) : 0;
        if (m->nrows == 0) SPC5_CUDA(cudaMemsetAsync(brptr.p, 0, sizeof(int), s));
        const size_t stride = 4 + size_t(r) * mask_bytes_of(m->value_type);
        Owned headers, values, valptr;
        headers.alloc(stride * size_t(nb));
        values.alloc(size_t(value_bytes_of(m->value_type)) * size_t(m->nnz));
        valptr.alloc(sizeof(int) * size_t(nbr + 1));
        launch_emit(vs_of(m->value_type), r, m->nrows, m->rowptr.as<int>(), m->colidx.as<int>(),
                    m->values.p, value_bytes_of(m->value_type), brptr.as<int>(),
                    headers.as<uint8_t>(), values.p, s);
        launch_valptr_from_csr(r, m->nrows, m->rowptr.as<int>(), valptr.as<int>(), s);
        SPC5_CUDA(cudaStreamSynchronize(s));
        std::swap(m->brptr.p, brptr.p);
        std::swap(m->brptr.bytes, brptr.bytes);
        std::swap(m->headers.p, headers.p);
        std::swap(m->headers.bytes, headers.bytes);
        std::swap(m->values.p, values.p);
        std::swap(m->values.bytes, values.bytes);
        std::swap(m->valptr.p, valptr.p);
        std::swap(m->valptr.bytes, valptr.bytes);
        m->rowptr.release();
        m->colidx.release();
        m->r = r;
        m->format = format;
        m->nblocks = nb;
        m->build_partition(s);
        SPC5_CUDA(cudaStreamSynchronize(s));
    });
}

spc5cuda_status spc5cuda_get_arrays(const spc5cuda_mat* m, int* rowsSize, unsigned char* headers,
                                    void* values, int to_host, void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        if (rowsSize)
            SPC5_CUDA(cudaMemcpyAsync(rowsSize, m->brptr.p, m->brptr.bytes, kind, s));
        const void* hsrc = m->headers.p;
        const void* vsrc = m->values.p;
        // the sorted copy holds the only one: the reference order, rebuilt
        const bool rebuild = m->original_dropped && (headers || values);
        DevBuf th(rebuild ? std::max<size_t>(16, m->header_bytes()) : 0, s);
        DevBuf tv(rebuild ? std::max<size_t>(16, m->value_bytes()) : 0, s);
        if (rebuild) {
            rebuild_original(m, th.as<uint8_t>(), tv.p, s);
            hsrc = th.p;
            vsrc = tv.p;
        }
        if (headers && m->header_bytes())
            SPC5_CUDA(cudaMemcpyAsync(headers, hsrc, m->header_bytes(), kind, s));
        if (values && m->value_bytes())
            SPC5_CUDA(cudaMemcpyAsync(values, vsrc, m->value_bytes(), kind, s));
        if (to_host) SPC5_CUDA(cudaStreamSynchronize(s));
    });
}

spc5cuda_status spc5cuda_spmv(const spc5cuda_mat* m, const void* x, void* y, void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "SPC5_Spmv : Unknown format type");
        if (m->nrows == 0) return;
        require(x && y, SPC5CUDA_ERR_INVALID, "null vector");
        require(m->value_type != SPC5CUDA_F32_V8, SPC5CUDA_ERR_FORMAT,
                "an F32_V8 matrix takes the mixed-precision calls only");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (m->use_plan()) {
            plan_spmv(m, x, y, false, s);
        } else if (m->value_type == SPC5CUDA_F64) {
            launch_spmv_f64(m->view(), static_cast<const double*>(x), static_cast<double*>(y), s);
        } else {
            launch_spmv_f32(m->view(), static_cast<const float*>(x), static_cast<float*>(y), s);
        }
    });
}

spc5cuda_status spc5cuda_spmv_mixed(const spc5cuda_mat* m, const float* x, double* y,
                                    void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        require(m->value_type == SPC5CUDA_F32 || m->value_type == SPC5CUDA_F32_V8, SPC5CUDA_ERR_FORMAT,
                "mixed precision needs an F32 or F32_V8 matrix");
        if (m->nrows == 0) return;
        require(x && y, SPC5CUDA_ERR_INVALID, "null vector");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (m->use_plan()) {
            plan_spmv(m, x, y, true, s);
        } else if (m->value_type == SPC5CUDA_F32_V8) {
            launch_spmv_mixed8(m->view(), x, y, s);
        } else {
            launch_spmv_mixed(m->view(), x, y, s);
        }
    });
}

spc5cuda_status spc5cuda_spmm(const spc5cuda_mat* m, int k, const void* X, long ldx, void* Y,
                              long ldy, void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        require(k >= 0 && ldx >= k && ldy >= k, SPC5CUDA_ERR_INVALID, "k / leading dimensions");
        if (m->nrows == 0 || k == 0) return;
        require(X && Y, SPC5CUDA_ERR_INVALID, "null block of vectors");
        require(m->value_type != SPC5CUDA_F32_V8, SPC5CUDA_ERR_FORMAT,
                "an F32_V8 matrix takes the mixed-precision calls only");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (m->use_plan())
            plan_spmm(m, k, X, ldx, 1, Y, ldy, 1, false, s);
        else if (m->value_type == SPC5CUDA_F64)
            launch_spmm_f64(m->spmm_view(), k, static_cast<const double*>(X), ldx, 1,
                            static_cast<double*>(Y), ldy, 1, s);
        else
            launch_spmm_f32(m->spmm_view(), k, static_cast<const float*>(X), ldx, 1,
                            static_cast<float*>(Y), ldy, 1, s);
    });
}

spc5cuda_status spc5cuda_spmm_mixed(const spc5cuda_mat* m, int k, const float* X, long ldx,
                                    double* Y, long ldy, void* stream) {
    return guarded([&] {
        require(m != nullptr, SPC5CUDA_ERR_INVALID, "null");
        require(m->r != 0, SPC5CUDA_ERR_FORMAT, "matrix is not converted");
        require(m->value_type == SPC5CUDA_F32 || m->value_type == SPC5CUDA_F32_V8, SPC5CUDA_ERR_FORMAT,
                "mixed precision needs an F32 or F32_V8 matrix");
        require(k >= 0 && ldx >= k && ldy >= k, SPC5CUDA_ERR_INVALID, "k / leading dimensions");
        if (m->nrows == 0 || k == 0) return;
        require(X && Y, SPC5CUDA_ERR_INVALID, "null block of vectors");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (m->use_plan())
            plan_spmm(m, k, X, ldx, 1, Y, ldy, 1, true, s);
        else if (m->value_type == SPC5CUDA_F32_V8)
            launch_spmm_mixed8(m->spmm_view(), k, X, ldx, 1, Y, ldy, 1, s);
        else
            launch_spmm_mixed(m->spmm_view(), k, X, ldx, 1, Y, ldy, 1, s);
    });
}

}  // extern "C"
