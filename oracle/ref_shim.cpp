// ref_shim.cpp -- C entry points around the UNMODIFIED reference header.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit includes src/spc5.hpp of
// berenger-eu/spc5 from where it lies (the include path is given by
// oracle/Makefile) and exposes its conversion, block counter, kernels,
// OpenMP path and format-selection model through plain C functions, so the
// tests can pin the oracle restatement against the reference itself and
// bench.py can time the reference's own AVX-512 OpenMP SpMV as the CPU
// baseline.  Nothing of the reference is copied here; every call below goes
// to the reference's own code.
//
// spc5.hpp defines non-inline extern "C" kernels, so it is included in this
// one translation unit only; -DNDEBUG is required (spc5.hpp:1017 does not
// compile with assertions on).
#include "spc5.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

template <class T>
struct RefMat {
    SPC5Mat<T> mat;
    int r = 0;
#ifdef _OPENMP
    std::vector<ThreadInterval<T>> split;
#endif
};

template <class T>
RefMat<T>* make_csr(int nrows, int ncols, int nnz, const int* rowptr, const int* colidx,
                    const T* values) {
    auto* m = new RefMat<T>();
    m->mat.format = SPC5_MATRIX_TYPE::FORMAT_CSR;
    m->mat.numberOfRows = nrows;
    m->mat.numberOfColumns = ncols;
    m->mat.numberOfNNZ = nnz;
    m->mat.values.reset(new T[nnz > 0 ? nnz : 1]);
    m->mat.rowsSize.reset(new int[nrows + 1]);
    m->mat.valuesColumnIndexes.reset(new int[nnz > 0 ? nnz : 1]);
    std::memcpy(m->mat.values.get(), values, sizeof(T) * size_t(nnz));
    std::memcpy(m->mat.rowsSize.get(), rowptr, sizeof(int) * size_t(nrows + 1));
    std::memcpy(m->mat.valuesColumnIndexes.get(), colidx, sizeof(int) * size_t(nnz));
    return m;
}

SPC5_MATRIX_TYPE type_of(int r) {
    switch (r) {
        case 1: return SPC5_MATRIX_TYPE::FORMAT_1rVc_WT;
        case 2: return SPC5_MATRIX_TYPE::FORMAT_2rVc;
        case 4: return SPC5_MATRIX_TYPE::FORMAT_4rVc;
        case 8: return SPC5_MATRIX_TYPE::FORMAT_8rVc;
        default: return SPC5_MATRIX_TYPE::UNDEFINED_FORMAT;
    }
}

template <class T>
int block_count(const SPC5Mat<T>& csr, int r) {
    switch (r) {
        case 1: return SPC5_1rVc_block_count<T>(csr);
        case 2: return SPC5_2rVc_block_count<T>(csr);
        case 4: return SPC5_4rVc_block_count<T>(csr);
        case 8: return SPC5_8rVc_block_count<T>(csr);
        default: return -1;
    }
}

template <class T>
int convert(RefMat<T>* m, int r) {
    const SPC5_MATRIX_TYPE t = type_of(r);
    if (t == SPC5_MATRIX_TYPE::UNDEFINED_FORMAT) return -1;
    try {
        CSR_to_SPC5<T>(&m->mat, t);
    } catch (...) {
        return -2;
    }
    m->r = r;
    return m->mat.numberOfBlocks;
}

template <class T>
void get(const RefMat<T>* m, int* rowptr, unsigned char* headers, T* values) {
    const int nbr = (m->mat.numberOfRows + m->r - 1) / m->r;
    const int stride = 4 + m->r * int(sizeof(typename SPC5Mat_Mask<T>::type));
    std::memcpy(rowptr, m->mat.rowsSize.get(), sizeof(int) * size_t(nbr + 1));
    std::memcpy(headers, m->mat.blocksColumnIndexesWithMasks.get(),
                size_t(m->mat.numberOfBlocks) * size_t(stride));
    std::memcpy(values, m->mat.values.get(), sizeof(T) * size_t(m->mat.numberOfNNZ));
}

}  // namespace

extern "C" {

int ref_has_openmp(void) {
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---- f64 ---------------------------------------------------------------
void* ref_f64_create(int nrows, int ncols, int nnz, const int* rowptr, const int* colidx,
                     const double* values) {
    return make_csr<double>(nrows, ncols, nnz, rowptr, colidx, values);
}
void ref_f64_destroy(void* h) { delete static_cast<RefMat<double>*>(h); }
int ref_f64_block_count(void* h, int r) {
    return block_count<double>(static_cast<RefMat<double>*>(h)->mat, r);
}
int ref_f64_convert(void* h, int r) { return convert<double>(static_cast<RefMat<double>*>(h), r); }
void ref_f64_get(void* h, int* rowptr, unsigned char* headers, double* values) {
    get<double>(static_cast<RefMat<double>*>(h), rowptr, headers, values);
}
// SPC5_Spmv<double> -> core_SPC5_{r}rVc_Spmv_double (spc5.hpp:1090-1118)
void ref_f64_spmv(void* h, const double* x, double* y) {
    SPC5_Spmv<double>(static_cast<RefMat<double>*>(h)->mat, x, y);
}
// CSR_Spmv_scalar (spc5.hpp:116-127); call before convert
void ref_f64_csr_spmv(void* h, const double* x, double* y) {
    CSR_Spmv_scalar<double>(static_cast<RefMat<double>*>(h)->mat, x, y);
}
// SPC5_find_best<double> (spc5.hpp:1151-1223); call before convert
int ref_f64_find_best(void* h, double* estimate) {
    auto best = SPC5_find_best<double>(static_cast<RefMat<double>*>(h)->mat);
    *estimate = best.second;
    switch (best.first) {
        case SPC5_MATRIX_TYPE::FORMAT_1rVc_WT: return 1;
        case SPC5_MATRIX_TYPE::FORMAT_2rVc: return 2;
        case SPC5_MATRIX_TYPE::FORMAT_4rVc: return 4;
        case SPC5_MATRIX_TYPE::FORMAT_8rVc: return 8;
        default: return 0;
    }
}

#ifdef _OPENMP
// SPC5_split_omp (spc5.hpp:1307-1336) with an explicit thread count
int ref_f64_split(void* h, int nthreads) {
    auto* m = static_cast<RefMat<double>*>(h);
    switch (m->r) {
        case 1: m->split = SPC5_1rVc_split_omp<double>(m->mat, nthreads); break;
        case 2: m->split = SPC5_2rVc_split_omp<double>(m->mat, nthreads); break;
        case 4: m->split = SPC5_4rVc_split_omp<double>(m->mat, nthreads); break;
        case 8: m->split = SPC5_8rVc_split_omp<double>(m->mat, nthreads); break;
        default: return -1;
    }
    return int(m->split.size());
}
// One SPC5_Spmv_omp call (spc5.hpp:1338-1367); requires ref_f64_split
void ref_f64_spmv_omp(void* h, const double* x, double* y) {
    auto* m = static_cast<RefMat<double>*>(h);
    SPC5_Spmv_omp<double>(m->mat, x, y, m->split);
}
// loops calls of SPC5_Spmv_omp, wall-clock seconds of the whole loop
double ref_f64_time_spmv_omp(void* h, const double* x, double* y, int loops) {
    auto* m = static_cast<RefMat<double>*>(h);
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < loops; ++i) SPC5_Spmv_omp<double>(m->mat, x, y, m->split);
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}
#endif

// ---- f32 ---------------------------------------------------------------
void* ref_f32_create(int nrows, int ncols, int nnz, const int* rowptr, const int* colidx,
                     const float* values) {
    return make_csr<float>(nrows, ncols, nnz, rowptr, colidx, values);
}
void ref_f32_destroy(void* h) { delete static_cast<RefMat<float>*>(h); }
int ref_f32_block_count(void* h, int r) {
    return block_count<float>(static_cast<RefMat<float>*>(h)->mat, r);
}
int ref_f32_convert(void* h, int r) { return convert<float>(static_cast<RefMat<float>*>(h), r); }
void ref_f32_get(void* h, int* rowptr, unsigned char* headers, float* values) {
    get<float>(static_cast<RefMat<float>*>(h), rowptr, headers, values);
}
void ref_f32_spmv(void* h, const float* x, float* y) {
    SPC5_Spmv<float>(static_cast<RefMat<float>*>(h)->mat, x, y);
}
int ref_f32_find_best(void* h, double* estimate) {
    auto best = SPC5_find_best<float>(static_cast<RefMat<float>*>(h)->mat);
    *estimate = best.second;
    switch (best.first) {
        case SPC5_MATRIX_TYPE::FORMAT_1rVc_WT: return 1;
        case SPC5_MATRIX_TYPE::FORMAT_2rVc: return 2;
        case SPC5_MATRIX_TYPE::FORMAT_4rVc: return 4;
        default: return 0;
    }
}
#ifdef _OPENMP
int ref_f32_split(void* h, int nthreads) {
    auto* m = static_cast<RefMat<float>*>(h);
    switch (m->r) {
        case 1: m->split = SPC5_1rVc_split_omp<float>(m->mat, nthreads); break;
        case 2: m->split = SPC5_2rVc_split_omp<float>(m->mat, nthreads); break;
        case 4: m->split = SPC5_4rVc_split_omp<float>(m->mat, nthreads); break;
        case 8: m->split = SPC5_8rVc_split_omp<float>(m->mat, nthreads); break;
        default: return -1;
    }
    return int(m->split.size());
}
double ref_f32_time_spmv_omp(void* h, const float* x, float* y, int loops) {
    auto* m = static_cast<RefMat<float>*>(h);
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < loops; ++i) SPC5_Spmv_omp<float>(m->mat, x, y, m->split);
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}
#endif

}  // extern "C"
