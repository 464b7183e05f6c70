// kernels.h -- host-side launchers of the sm_100a kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spc5cuda {

// ---- scan ---------------------------------------------------------------
// out[0..n] = exclusive prefix sum of in[0..n), out[n] = total.  tmp must
// hold scan_tmp_ints(n) ints.  in and out may alias.
long scan_tmp_ints(long n);
void exclusive_scan_i32(const int* in, int* out, long n, int* tmp, cudaStream_t s);

// ---- CSR checks and conversion (convert.cu) -------------------------------
// Writes 0 to *d_flag when the CSR is well formed (monotone rowptr starting
// at 0, columns in [0, ncols), strictly increasing inside a row), else an
// error code (1 rowptr, 2 column range, 3 order/duplicate).
void launch_validate_csr(int nrows, int ncols, long nnz, const int* rowptr, const int* colidx,
                         int* d_flag, cudaStream_t s);

// counts[br] = blocks of block-row br for rows-per-block r and VS columns.
void launch_blockrow_counts(int vs, int r, int nrows, const int* rowptr, const int* colidx,
                            int* counts, cudaStream_t s);

// Emits headers and reordered values of every block-row (brptr = exclusive
// scan of the counts).  value_bytes is 8 or 4.
void launch_emit(int vs, int r, int nrows, const int* rowptr, const int* colidx,
                 const void* vin, int value_bytes, const int* brptr, uint8_t* headers,
                 void* vout, cudaStream_t s);

// valptr[br] = rowptr[min(br*r, nrows)] for br in [0, nbr].
void launch_valptr_from_csr(int r, int nrows, const int* rowptr, int* valptr, cudaStream_t s);

// counts[br] = number of values of block-row br, from the header masks.
void launch_blockrow_value_counts(int mask_bytes, int r, int nbr, const int* brptr,
                                  const uint8_t* headers, int* counts, cudaStream_t s);

// ---- SpMV (spmv.cu) ------------------------------------------------------
struct BetaView {
    int r = 0;
    int nrows = 0;
    int nbr = 0;                    // ceil(nrows / r)
    const int* brptr = nullptr;     // nbr + 1 block offsets
    const uint8_t* headers = nullptr;
    const void* values = nullptr;
    const int* valptr = nullptr;    // nbr + 1 value offsets
    const int* gstart = nullptr;    // ngroups + 1 block-row starts of the group ranges
    int ngroups = 0;
    // thread-per-sub-row kernel (short block-rows): nwarps + 1 block-row
    // starts of the per-warp ranges; null selects the group kernel
    const int* wstart = nullptr;
    int nwarps = 0;
    int lanes = 0;               // row kernel: lanes per block-row (0: r)
    // row kernel: > 0 when these arrays hold the segments of nseg long
    // block-rows, interleaved per warp (the sorted plan's largest part)
    int nseg = 0;
    // block-row of y for each block-row of these arrays (null: the same);
    // set when the arrays are a reordered copy of the matrix
    const int* perm = nullptr;
    // when set, the launch does its work only if *run_if == run_if_value (a
    // device word written by an earlier kernel on the same stream)
    const int* run_if = nullptr;
    int run_if_value = 0;
};

// Number of VS-lane groups the SpMV kernels launch on the current device
// for rows-per-block r: one wave of resident CTAs.
int spmv_groups(int vs, int r);

// gstart[0..ngroups] = block-row ranges holding ~nblocks/ngroups blocks each.
void launch_partition(int nbr, const int* brptr, int ngroups, int* gstart, cudaStream_t s);
// The same over block-rows [a, b): gstart[0] = a, gstart[ngroups] = b.
void launch_partition_range(int a, int b, const int* brptr, int ngroups, int* gstart, cudaStream_t s);

void launch_spmv_f64(const BetaView& m, const double* x, double* y, cudaStream_t s);

// Thread-per-sub-row kernel (spmv_rows.cu): resident warps on this device,
// whether block-rows of at most max_blocks blocks / max_values values fit its
// staging buffers, and the largest block-row of a converted matrix
// (synchronises s).
// (vt: the handle's value type, SPC5CUDA_F64 / F32 / F32_V8.)
int rows_warps(int vt, int r, int lanes = 0);
bool rows_fit(int vt, int r, int max_blocks, int max_values);
// Size of a block-row in units of one lane's share of a row-kernel chunk:
// the block-row fits a chunk of 32 / L block-rows with L lanes each when
// rows_lane_units(...) <= L * rows_unit().
long rows_lane_units(int vt, int r, int nblocks, int nvalues);
long rows_unit();
// Lanes per block-row of the segmented part of a sorted plan (the largest
// block-rows), measured on B200 on the N = 4M power-law matrix: more lanes
// give longer segments and more warps, fewer give more block-rows per warp
// instruction.
constexpr int seg_lanes(int r) { return r == 1 ? 4 : (r == 2 ? 8 : r); }
// Header and value bytes of one warp's staging buffer.
int rows_hb();
int rows_vb();
void blockrow_max(int nbr, const int* brptr, const int* valptr, int* max_blocks, int* max_values,
                  cudaStream_t s);
// The same test on the device, without a host round trip: work[0] = 1 when
// every block-row fits the row kernel's buffers, else 0 (work holds 3 ints;
// work[1], work[2] receive the largest block and value counts).
void launch_rows_fit_flag(int vt, int r, int nbr, const int* brptr, const int* valptr, int* work,
                          cudaStream_t s);
void launch_rows_f64(const BetaView& m, const double* x, double* y, cudaStream_t s);
void launch_rows_f32(const BetaView& m, const float* x, float* y, cudaStream_t s);
void launch_rows_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s);
// Float values in the 8-column layout (F32_V8), float x, FP64 accumulation and y.
void launch_rows_mixed8(const BetaView& m, const float* x, double* y, cudaStream_t s);
void launch_spmv_f32(const BetaView& m, const float* x, float* y, cudaStream_t s);
void launch_spmv_mixed(const BetaView& m, const float* x, double* y, cudaStream_t s);
void launch_spmv_mixed8(const BetaView& m, const float* x, double* y, cudaStream_t s);

// ---- SpMM (spmm.cu): Y += A X.  Element (row i, right-hand side q) of X
// is x[i * ldx + q * xcs] (row-major: xcs = 1; column-major: ldx = 1,
// xcs = leading dimension), likewise Y with ldy, ycs.
void launch_spmm_f64(const BetaView& m, int k, const double* x, long ldx, long xcs, double* y,
                     long ldy, long ycs, cudaStream_t s);
void launch_spmm_f32(const BetaView& m, int k, const float* x, long ldx, long xcs, float* y,
                     long ldy, long ycs, cudaStream_t s);
void launch_spmm_mixed(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                       long ldy, long ycs, cudaStream_t s);
void launch_spmm_mixed8(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                        long ldy, long ycs, cudaStream_t s);

// ---- staged SpMM (spmm_rows.cu) over the per-warp ranges m.wstart /
// m.nwarps of a matrix whose block-rows fit the row kernels' buffers; same
// arguments and results as launch_spmm_*.
void launch_spmm_rows_f64(const BetaView& m, int k, const double* x, long ldx, long xcs, double* y,
                          long ldy, long ycs, cudaStream_t s);
void launch_spmm_rows_f32(const BetaView& m, int k, const float* x, long ldx, long xcs, float* y,
                          long ldy, long ycs, cudaStream_t s);
void launch_spmm_rows_mixed(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                            long ldy, long ycs, cudaStream_t s);
void launch_spmm_rows_mixed8(const BetaView& m, int k, const float* x, long ldx, long xcs, double* y,
                             long ldy, long ycs, cudaStream_t s);

// ---- batched SpMM (spmm.cu): many matrices, one launch per (r, kc) class
struct BatchMat {
    const int* brptr;
    const uint8_t* headers;
    const void* values;
    const int* valptr;
    const void* x;  // row-major ncols x k (ldx)
    long ldx;
    void* y;        // row-major nrows x k (ldy)
    long ldy;
    long xcs;       // stride between right-hand sides (1: row-major)
    long ycs;
    int nrows;
    int pad;
};
struct BatchJob {
    int mat;      // index into the BatchMat array
    int r_begin;  // block-row range
    int r_end;
    int kofs;     // first right-hand side of this pass
};
// right-hand sides per pass for rows-per-block r and k right-hand sides
int batch_kc(int r, int k);
// kind 0 = f64, 1 = f32, 2 = mixed (f32 values and x, f64 y), 3 = mixed in the
// 8-column layout (F32_V8 matrices)
void launch_batch(int kind, int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs,
                  int ctas, cudaStream_t s);
// Right-hand sides per pass of the staged SpMM for VS columns per block,
// rows-per-block r and k right-hand sides left (seg: the segmented part of a
// sorted plan, run with seg_lanes(r) lanes per block-row).
int spmm_rows_kc(int vs, int r, int k, bool seg = false);
// Most right-hand sides per pass of the staged SpMM with `lanes` lanes per
// block-row: r x (vs / lanes columns per lane) x kc accumulators stay at
// most 32, kc at most 16.
constexpr int mm_kc_limit(int vs, int r, int lanes) {
    return 32 / (r * (vs / lanes)) > 16 ? 16 : 32 / (r * (vs / lanes));
}
// The same for matrices whose block-rows fit the row kernels' buffers
// (spmm_rows.cu): one warp per job at a time; kc from spmm_rows_kc.
void launch_batch_rows(int kind, int r, int kc, const BatchMat* mats, const BatchJob* jobs, int njobs,
                       cudaStream_t s);

}  // namespace spc5cuda
