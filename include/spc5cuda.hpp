// spc5cuda.hpp -- header-only C++ wrapper over the C ABI (spc5cuda.h),
// mirroring the calling pattern of the reference's C++ API
// (src/spc5.hpp): build a CSR matrix, CSR_to_SPC5 it, SPC5_Spmv into y.
// Errors become spc5cuda::error exceptions on this side of the ABI (the
// reference throws std::invalid_argument for an unknown format,
// spc5.hpp:1014).  All vectors are device pointers.
#ifndef SPC5CUDA_HPP
#define SPC5CUDA_HPP

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "spc5cuda.h"

namespace spc5cuda {

struct error : std::runtime_error {
    spc5cuda_status status;
    error(spc5cuda_status s, const std::string& what)
        : std::runtime_error(what + ": " + spc5cuda_status_string(s)), status(s) {}
};

inline void check(spc5cuda_status s, const char* what) {
    if (s != SPC5CUDA_OK) throw error(s, what);
}

template <class T>
struct value_type_of;
template <>
struct value_type_of<double> {
    static constexpr int id = SPC5CUDA_F64;
};
template <>
struct value_type_of<float> {
    static constexpr int id = SPC5CUDA_F32;
};

// Device-resident counterpart of SPC5Mat<T> (spc5.hpp:44-62), owning its handle.
template <class T>
class SPC5Mat {
  public:
    SPC5Mat() = default;
    explicit SPC5Mat(spc5cuda_mat* h) : h_(h) {}
    SPC5Mat(const SPC5Mat&) = delete;
    SPC5Mat& operator=(const SPC5Mat&) = delete;
    SPC5Mat(SPC5Mat&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    SPC5Mat& operator=(SPC5Mat&& o) noexcept {
        if (this != &o) {
            reset();
            h_ = std::exchange(o.h_, nullptr);
        }
        return *this;
    }
    ~SPC5Mat() { reset(); }

    spc5cuda_mat* handle() const { return h_; }
    spc5cuda_info info() const {
        spc5cuda_info i{};
        check(spc5cuda_mat_info(h_, &i), "spc5cuda_mat_info");
        return i;
    }
    int numberOfRows() const { return info().nrows; }
    int numberOfColumns() const { return info().ncols; }
    long numberOfNNZ() const { return info().nnz; }
    long numberOfBlocks() const { return info().nblocks; }
    int format() const { return info().format; }

  private:
    void reset() {
        if (h_) spc5cuda_mat_destroy(h_);
        h_ = nullptr;
    }
    spc5cuda_mat* h_ = nullptr;
};

// CSR (host arrays) -> device SPC5Mat in FORMAT_CSR (COO_sorted_to_CSR's output).
template <class T>
SPC5Mat<T> CSR_from_host(int nrows, int ncols, const std::vector<int>& rowptr,
                         const std::vector<int>& colidx, const std::vector<T>& values,
                         void* stream = nullptr) {
    spc5cuda_mat* h = nullptr;
    check(spc5cuda_mat_create_csr(&h, value_type_of<T>::id, nrows, ncols, long(values.size()),
                                  rowptr.data(), colidx.data(), values.data(), 0, stream),
          "spc5cuda_mat_create_csr");
    return SPC5Mat<T>(h);
}

// CSR_to_SPC5 (spc5.hpp:989-1018), on the device.
template <class T>
void CSR_to_SPC5(SPC5Mat<T>& mat, int format, void* stream = nullptr) {
    check(spc5cuda_convert(mat.handle(), format, stream), "CSR_to_SPC5");
}

// SPC5_{r}rVc_block_count (spc5.hpp:510-513 ...); returns the count.
template <class T>
long SPC5_block_count(const SPC5Mat<T>& mat, int r, void* stream = nullptr) {
    long n = 0;
    check(spc5cuda_block_count(mat.handle(), r, &n, stream), "SPC5_block_count");
    return n;
}

// SPC5_Spmv (spc5.hpp:1090-1118): y += A x, device vectors.
template <class T>
void SPC5_Spmv(const SPC5Mat<T>& mat, const T* x, T* y, void* stream = nullptr) {
    check(spc5cuda_spmv(mat.handle(), x, y, stream), "SPC5_Spmv");
}

// Mixed precision: float matrix and x, double y.
inline void SPC5_Spmv_mixed(const SPC5Mat<float>& mat, const float* x, double* y,
                            void* stream = nullptr) {
    check(spc5cuda_spmv_mixed(mat.handle(), x, y, stream), "SPC5_Spmv_mixed");
}

// Y += A X for k right-hand sides, row-major X (ncols x k) and Y (nrows x k).
template <class T>
void SPC5_Spmm(const SPC5Mat<T>& mat, int k, const T* X, long ldx, T* Y, long ldy,
               void* stream = nullptr) {
    check(spc5cuda_spmm(mat.handle(), k, X, ldx, Y, ldy, stream), "SPC5_Spmm");
}

// The reference's speed model (spc5.hpp:1151-1223) on device block counts.
template <class T>
std::pair<int, double> SPC5_find_best(const SPC5Mat<T>& csr, void* stream = nullptr) {
    int r = 0;
    double est = 0.0;
    check(spc5cuda_find_best(csr.handle(), &r, &est, stream), "SPC5_find_best");
    return {r, est};
}

// The B200 autotuner: the best r for a CSR matrix.
template <class T>
spc5cuda_tune autotune(const SPC5Mat<T>& csr, int mode = SPC5CUDA_TUNE_MODEL,
                       void* stream = nullptr) {
    spc5cuda_tune t{};
    check(spc5cuda_autotune(csr.handle(), mode, &t, stream), "autotune");
    return t;
}

inline int format_of_r(int r) {
    switch (r) {
        case 1: return SPC5CUDA_FORMAT_1rVc_WT;
        case 2: return SPC5CUDA_FORMAT_2rVc;
        case 4: return SPC5CUDA_FORMAT_4rVc;
        case 8: return SPC5CUDA_FORMAT_8rVc;
        default: throw error(SPC5CUDA_ERR_FORMAT, "format_of_r");
    }
}

}  // namespace spc5cuda

#endif  // SPC5CUDA_HPP
