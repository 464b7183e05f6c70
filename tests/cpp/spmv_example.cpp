// A C++ host program driving the library through include/spc5cuda.hpp the
// way the reference's driver drives spc5.hpp (examples/load_mm_and_compare.cpp):
// build CSR, pick a format, convert, run 16 accumulating SpMVs, check.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "spc5cuda.hpp"

int main() {
    const int g = 64, n = g * g;  // 5-point Poisson
    std::vector<int> rowptr(1, 0), colidx;
    std::vector<double> values;
    for (int i = 0; i < n; ++i) {
        const int iy = i / g, ix = i % g;
        const int cand[5] = {i - g, i - 1, i, i + 1, i + g};
        const bool ok[5] = {iy > 0, ix > 0, true, ix < g - 1, iy < g - 1};
        for (int k = 0; k < 5; ++k)
            if (ok[k]) {
                colidx.push_back(cand[k]);
                values.push_back(k == 2 ? 4.0 : -1.0);
            }
        rowptr.push_back(int(colidx.size()));
    }
    auto mat = spc5cuda::CSR_from_host<double>(n, n, rowptr, colidx, values);
    const auto best = spc5cuda::SPC5_find_best(mat);
    const auto tune = spc5cuda::autotune(mat);
    spc5cuda::CSR_to_SPC5(mat, spc5cuda::format_of_r(tune.r));
    std::vector<double> x(n), y(n, 0.0), ref(n, 0.0);
    for (int i = 0; i < n; ++i) x[i] = double(i % 98);  // the reference driver's x
    double *dx, *dy;
    cudaMalloc(&dx, n * sizeof(double));
    cudaMalloc(&dy, n * sizeof(double));
    cudaMemcpy(dx, x.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(dy, 0, n * sizeof(double));
    for (int loop = 0; loop < 16; ++loop) spc5cuda::SPC5_Spmv(mat, dx, dy);
    cudaMemcpy(y.data(), dy, n * sizeof(double), cudaMemcpyDeviceToHost);
    double maxdiff = 0.0;
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s += x[colidx[k]] * values[k];
        ref[i] = 16.0 * s;
        maxdiff = std::fmax(maxdiff, std::fabs(ref[i] - y[i]));
    }
    std::printf("find_best r=%d (%.3f), autotune r=%d, blocks=%ld, max |diff|=%g\n", best.first,
                best.second, tune.r, mat.numberOfBlocks(), maxdiff);
    cudaFree(dx);
    cudaFree(dy);
    return maxdiff < 1e-9 ? 0 : 1;
}
