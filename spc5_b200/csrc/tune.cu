// tune.cu -- format selection: the reference's polynomial model on device
// block counts, and the B200 autotuner (cost model or measured trial runs).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "handle.h"

namespace spc5cuda {

namespace {

// Algorithmic bytes of one y += A x in beta(r,VS) (values, headers, block-row
// pointer, x once, y read and written).
double spmv_bytes(const spc5cuda_mat* m, int r, long nblocks) {
    const double sv = value_bytes_of(m->value_type);
    const double mb = mask_bytes_of(m->value_type);
    const double nbr = double(div_up(m->nrows, r));
    return double(m->nnz) * sv + double(nblocks) * (4.0 + r * mb) + 4.0 * (nbr + 1.0) +
           double(m->ncols) * sv + 2.0 * double(m->nrows) * sv;
}

// B200 cost model of the SpMV kernel (spmv.cu): the kernel is bounded by
// whichever is slower, streaming its algorithmic bytes at the sustained
// fraction of HBM bandwidth it reaches, or issuing its per-block work.  The
// per-block costs are SpMV times measured on a B200 (148 SMs, 1.965 GHz)
// divided by the block count, on a 27-point stencil and a power-law matrix;
// the f32 layout has twice the lanes per block.
constexpr double kHbmBytesPerUs = 6.0e6;                            // ~6.0 TB/s
constexpr double kBlockUsF64[4] = {35e-6, 42e-6, 48e-6, 56e-6};     // r = 1, 2, 4, 8
constexpr double kBlockUsF32[4] = {50e-6, 58e-6, 66e-6, 78e-6};

int r_index(int r) { return r == 1 ? 0 : (r == 2 ? 1 : (r == 4 ? 2 : 3)); }

double model_us(const spc5cuda_mat* m, int r, long nblocks) {
    const double t_mem = spmv_bytes(m, r, nblocks) / kHbmBytesPerUs;
    const double per = m->value_type == SPC5CUDA_F64 ? kBlockUsF64[r_index(r)] : kBlockUsF32[r_index(r)];
    const double t_issue = double(nblocks) * per;
    return std::max(t_mem, t_issue);
}

// Converts the CSR handle to r into temporary arrays and times the SpMV
// kernel (1 warm-up, 3 timed launches); returns microseconds per SpMV.
double measure_us(const spc5cuda_mat* m, int r, cudaStream_t s) {
    const int nbr = div_up(m->nrows, r);
    const int vs = vs_of(m->value_type);
    const size_t vb = size_t(value_bytes_of(m->value_type));
    DevBuf brptr(sizeof(int) * size_t(nbr + 1), s);
    const long nb = count_blocks(m, r, brptr.as<int>(), s);
    const size_t stride = 4 + size_t(r) * mask_bytes_of(m->value_type);
    DevBuf headers(stride * size_t(nb) + 16, s);
    DevBuf values(vb * size_t(m->nnz) + 16, s);
    DevBuf valptr(sizeof(int) * size_t(nbr + 1), s);
    const int ngroups = spmv_groups(vs, r);
    DevBuf gstart(sizeof(int) * size_t(ngroups + 1), s);
    DevBuf x(vb * size_t(m->ncols) + 16, s);
    const size_t yb = m->value_type == SPC5CUDA_F32_V8 ? 8 : vb;  // F32_V8: FP64 y
    DevBuf y(yb * size_t(m->nrows) + 16, s);
    launch_emit(vs, r, m->nrows, m->rowptr.as<int>(), m->colidx.as<int>(), m->values.p, int(vb),
                brptr.as<int>(), headers.as<uint8_t>(), values.p, s);
    launch_valptr_from_csr(r, m->nrows, m->rowptr.as<int>(), valptr.as<int>(), s);
    launch_partition(nbr, brptr.as<int>(), ngroups, gstart.as<int>(), s);
    SPC5_CUDA(cudaMemsetAsync(x.p, 0, vb * size_t(m->ncols) + 16, s));
    SPC5_CUDA(cudaMemsetAsync(y.p, 0, yb * size_t(m->nrows) + 16, s));
    BetaView v;
    v.r = r;
    v.nrows = m->nrows;
    v.nbr = nbr;
    v.brptr = brptr.as<int>();
    v.headers = headers.as<uint8_t>();
    v.values = values.p;
    v.valptr = valptr.as<int>();
    v.gstart = gstart.as<int>();
    v.ngroups = ngroups;
    auto run = [&] {
        if (m->value_type == SPC5CUDA_F64)
            launch_spmv_f64(v, x.as<double>(), y.as<double>(), s);
        else if (m->value_type == SPC5CUDA_F32_V8)
            launch_spmv_mixed8(v, x.as<float>(), y.as<double>(), s);
        else
            launch_spmv_f32(v, x.as<float>(), y.as<float>(), s);
    };
    cudaEvent_t e0, e1;
    SPC5_CUDA(cudaEventCreate(&e0));
    SPC5_CUDA(cudaEventCreate(&e1));
    run();
    SPC5_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < 3; ++i) run();
    SPC5_CUDA(cudaEventRecord(e1, s));
    SPC5_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SPC5_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return double(ms) * 1000.0 / 3.0;
}

}  // namespace

}  // namespace spc5cuda

using namespace spc5cuda;

extern "C" {

spc5cuda_status spc5cuda_find_best(const spc5cuda_mat* m, int* r_out, double* estimate,
                                   void* stream) {
    return guarded([&] {
        require(m && r_out && estimate, SPC5CUDA_ERR_INVALID, "null");
        require(m->format == SPC5CUDA_FORMAT_CSR, SPC5CUDA_ERR_FORMAT, "find_best needs CSR");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // SPC5_find_best (spc5.hpp:1151-1223): cubic in the average number of
        // values per block, per format (r = 1, 2, 4) and precision.
        static const double cd[3][4] = {{2.186490e-03, -7.931533e-02, 8.719444e-01, 3.712380e-01},
                                        {9.822706e-04, -4.500002e-02, 6.714119e-01, 2.413985e-01},
                                        {1.320496e-04, -1.222130e-02, 3.520409e-01, 3.603195e-01}};
        static const double cf[3][4] = {{-4.039852e-03, 7.997606e-02, 6.892119e-02, 1.508645e+00},
                                        {-9.195940e-04, 4.442050e-03, 5.273045e-01, 1.101610e+00},
                                        {-4.464933e-05, 1.867266e-03, 1.520910e-01, 1.186131e+00}};
        static const int rs[3] = {1, 2, 4};
        int best = 0;
        double best_speed = 0.0;
        for (int f = 0; f < 3; ++f) {
            DevBuf tmp(sizeof(int) * size_t(div_up(m->nrows, rs[f]) + 1), s);
            const long nb = m->nrows > 0 ? count_blocks(m, rs[f], tmp.as<int>(), s) : 0;
            // the double model for the 8-column layouts (F64, F32_V8)
            const double* c = m->value_type == SPC5CUDA_F32 ? cf[f] : cd[f];
            const double avg = double(m->nnz) / double(nb);
            const double speed = c[0] * (avg * avg * avg) + c[1] * (avg * avg) + c[2] * avg + c[3];
            if (speed > best_speed) {
                best_speed = speed;
                best = rs[f];
            }
        }
        *r_out = best;
        *estimate = best_speed;
    });
}

spc5cuda_status spc5cuda_autotune(const spc5cuda_mat* m, int mode, spc5cuda_tune* out,
                                  void* stream) {
    return guarded([&] {
        require(m && out, SPC5CUDA_ERR_INVALID, "null");
        require(m->format == SPC5CUDA_FORMAT_CSR, SPC5CUDA_ERR_FORMAT, "autotune needs CSR");
        require(mode == SPC5CUDA_TUNE_MODEL || mode == SPC5CUDA_TUNE_MEASURE,
                SPC5CUDA_ERR_INVALID, "mode");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        static const int rs[4] = {1, 2, 4, 8};
        int best = 1;
        double best_us = 0.0;
        for (int f = 0; f < 4; ++f) {
            const int r = rs[f];
            DevBuf tmp(sizeof(int) * size_t(div_up(m->nrows, r) + 1), s);
            const long nb = m->nrows > 0 ? count_blocks(m, r, tmp.as<int>(), s) : 0;
            out->blocks[f] = nb;
            const double us = mode == SPC5CUDA_TUNE_MODEL
                                  ? model_us(m, r, nb)
                                  : (m->nrows > 0 ? measure_us(m, r, s) : 0.0);
            out->est_us[f] = us;
            if (f == 0 || us < best_us) {
                best_us = us;
                best = r;
            }
        }
        out->r = best;
    });
}

}  // extern "C"
