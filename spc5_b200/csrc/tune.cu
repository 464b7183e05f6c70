// tune.cu -- format selection: the reference's polynomial model on device
// block counts, and the B200 autotuner (cost model or measured trial runs).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>

#include "handle.h"

namespace spc5cuda {

namespace {

// B200 cost model of one SpMV through a converted handle's default kernel
// choice (spc5_b200/tune_fit.py fits it from timings on a B200, 148 SMs at
// 1.965 GHz): for value type, r and regime (0: the row kernel, every
// block-row fits its staging buffers; 1: the length-sorted plan),
//     t_us = t0 + nnz * (d0 + d1 / a + d2 / a^2),  a = nnz / blocks_r,
// the time per value keyed by the average number of values per block, as the
// reference's SPC5_find_best model is (src/spc5.hpp:1157-1212).
// Value type (F64, F32, F32_V8) x r (1, 2, 4, 8) x regime: {t0, d0, d1, d2}.
// The sorted-plan rows were refitted after the plan's chain part (r = 2, 4,
// 8) on the plan-regime calibration matrices alone (power-law and random,
// tune_fit.plan_calibration_set), keeping the row-kernel t0.
constexpr double kModel[3][4][2][4] = {
    {
        {{1.027079e+01, -2.714134e-07, 9.285081e-06, 1.994012e-06}, {1.027079e+01, 1.113738e-05, 0.000000e+00, 0.000000e+00}},
        {{1.046586e+01, 6.170896e-07, 9.230068e-06, 9.138698e-06}, {1.046586e+01, 1.212031e-05, 0.000000e+00, 0.000000e+00}},
        {{1.004610e+01, 1.547721e-06, 1.189384e-05, 2.402879e-05}, {1.004610e+01, 8.274836e-06, 0.000000e+00, 0.000000e+00}},
        {{1.004540e+01, 6.250567e-07, 5.782892e-05, -8.901463e-05}, {1.004540e+01, 7.059285e-06, 0.000000e+00, 0.000000e+00}},
    },
    {
        {{1.009044e+01, 2.953275e-07, 6.279096e-06, 1.099184e-05}, {1.009044e+01, 9.763137e-06, 0.000000e+00, 0.000000e+00}},
        {{1.008880e+01, 1.137428e-06, 1.740009e-06, 3.621405e-05}, {1.008880e+01, 1.172209e-05, 0.000000e+00, 0.000000e+00}},
        {{1.020511e+01, 1.170424e-06, 1.023505e-05, 1.026359e-04}, {1.020511e+01, 6.684552e-06, 0.000000e+00, 0.000000e+00}},
        {{1.034971e+01, -4.723864e-07, 8.071517e-05, -1.176461e-04}, {1.034971e+01, 5.902880e-06, 0.000000e+00, 0.000000e+00}},
    },
    {
        {{9.690487e+00, -8.483423e-07, 1.129287e-05, 5.480109e-06}, {9.690487e+00, 1.023616e-05, 0.000000e+00, 0.000000e+00}},
        {{9.904177e+00, 1.562250e-07, 1.131417e-05, 1.759617e-05}, {9.904177e+00, 1.203661e-05, 0.000000e+00, 0.000000e+00}},
        {{1.008765e+01, 1.592180e-07, 2.480687e-05, 2.707475e-05}, {1.008765e+01, 7.725355e-06, 0.000000e+00, 0.000000e+00}},
        {{1.044845e+01, -1.152926e-06, 8.811726e-05, -7.893453e-05}, {1.044845e+01, 6.381369e-06, 0.000000e+00, 0.000000e+00}},
    },
};

int r_index(int r) { return r == 1 ? 0 : (r == 2 ? 1 : (r == 4 ? 2 : 3)); }

double model_us(const spc5cuda_mat* m, int r, long nblocks, int regime) {
    if (m->nnz == 0 || nblocks == 0) return 0.0;
    const double* c = kModel[m->value_type][r_index(r)][regime];
    const double a = double(m->nnz) / double(nblocks);
    const double per_value = std::max(c[1] + c[2] / a + c[3] / (a * a), 1e-7);
    return c[0] + double(m->nnz) * per_value;
}

// 1 when some block-row of the CSR handle at rows-per-block r is too large for
// the row kernel's buffers (the handle would then run the sorted plan): the
// block counts are brptr (scanned), the value counts come from rowptr.
int plan_regime(const spc5cuda_mat* m, int r, const int* brptr, cudaStream_t s) {
    const int nbr = div_up(m->nrows, r);
    DevBuf valptr(sizeof(int) * size_t(nbr + 1), s);
    launch_valptr_from_csr(r, m->nrows, m->rowptr.as<int>(), valptr.as<int>(), s);
    int max_blocks = 0, max_values = 0;
    blockrow_max(nbr, brptr, valptr.as<int>(), &max_blocks, &max_values, s);
    return rows_fit(m->value_type, r, max_blocks, max_values) ? 0 : 1;
}

// A trial run: a temporary handle holding a copy of the CSR matrix is
// converted to r the usual way (its default kernel choice: the row kernel or
// the length-sorted plan) and its SpMV is timed (2 warm-up calls, which also
// load its kernels and size the library's scratch pool, then 5 timed calls);
// returns microseconds per SpMV.
double measure_us(const spc5cuda_mat* m, int r, cudaStream_t s) {
    spc5cuda_mat* t = nullptr;
    auto ok = [](spc5cuda_status st) {
        if (st != SPC5CUDA_OK) throw Error(st, "autotune trial run");
    };
    ok(spc5cuda_mat_create_csr(&t, m->value_type, m->nrows, m->ncols, m->nnz, m->rowptr.as<int>(),
                               m->colidx.as<int>(), m->values.p, 1, s));
    std::unique_ptr<spc5cuda_mat, spc5cuda_status (*)(spc5cuda_mat*)> guard(t, spc5cuda_mat_destroy);
    ok(spc5cuda_convert(t, r_to_format(r), s));
    const size_t xb = size_t(value_bytes_of(m->value_type));
    const size_t yb = m->value_type == SPC5CUDA_F32 ? 4 : 8;  // F32_V8: FP64 y
    DevBuf x(xb * size_t(m->ncols) + 16, s), y(yb * size_t(m->nrows) + 16, s);
    SPC5_CUDA(cudaMemsetAsync(x.p, 0, xb * size_t(m->ncols) + 16, s));
    SPC5_CUDA(cudaMemsetAsync(y.p, 0, yb * size_t(m->nrows) + 16, s));
    auto run = [&] {
        if (m->value_type == SPC5CUDA_F32_V8)
            ok(spc5cuda_spmv_mixed(t, x.as<float>(), y.as<double>(), s));
        else
            ok(spc5cuda_spmv(t, x.p, y.p, s));
    };
    cudaEvent_t e0, e1;
    SPC5_CUDA(cudaEventCreate(&e0));
    SPC5_CUDA(cudaEventCreate(&e1));
    run();
    run();
    SPC5_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < 5; ++i) run();
    SPC5_CUDA(cudaEventRecord(e1, s));
    SPC5_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SPC5_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return double(ms) * 1000.0 / 5.0;
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
            double us = 0.0;
            if (m->nrows > 0) {
                us = mode == SPC5CUDA_TUNE_MODEL ? model_us(m, r, nb, plan_regime(m, r, tmp.as<int>(), s))
                                                 : measure_us(m, r, s);
            }
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
