/*
 * spc5cuda.h -- C ABI of the B200 (sm_100a) implementation of SPC5's
 * beta(r,VS) hot path: CSR -> beta(r,VS) conversion and y += A x.
 *
 * The arrays are byte-for-byte the reference's SPC5Mat arrays
 * (src/spc5.hpp:44-62): after conversion rowsSize holds the block-row
 * pointer (ceil(nrows/r)+1 ints), the headers are packed
 * {int32 first column, r masks} records of 4 + r*sizeof(mask) bytes (mask =
 * uint8 for double, VS = 8; uint16 for float, VS = 16), and the values are in
 * block order (sub-row 0 of a block, then sub-row 1, ...).
 *
 * All pointers passed to the compute entry points are DEVICE pointers
 * (cudaMalloc, cudaMallocAsync or torch allocations) with at least 16-byte
 * alignment for the header and value arrays; work is enqueued on the given
 * stream (NULL = legacy default stream) and is asynchronous unless stated.
 * No entry point falls back to the CPU.
 *
 * Results: the FP64 and FP32 kernels compute every row in the order of the
 * reference's AVX-512 kernels (spc5.hpp:2309-2715, default non-MHSUM build),
 * so y matches the reference bit for bit for finite x.  Unlike the
 * reference, x is read only at columns present in the matrix (no
 * SPC5_VEC_PADDING_X needed) and only rows < nbRows of y are written (no
 * SPC5_VEC_PADDING_Y needed); padded buffers work as well.
 */
#ifndef SPC5CUDA_H
#define SPC5CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SPC5CUDA_API __attribute__((visibility("default")))
#else
#define SPC5CUDA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Format ids: the numbering of SPC5_MATRIX_TYPE (spc5.hpp:17-24). */
enum spc5cuda_format {
    SPC5CUDA_UNDEFINED_FORMAT = 0,
    SPC5CUDA_FORMAT_CSR = 1,
    SPC5CUDA_FORMAT_1rVc_WT = 2,
    SPC5CUDA_FORMAT_2rVc = 3,
    SPC5CUDA_FORMAT_4rVc = 4,
    SPC5CUDA_FORMAT_8rVc = 5
};

/* Value types of a matrix: SPC5Mat<double> (VS = 8) or SPC5Mat<float> (VS = 16).
 * SPC5CUDA_F32_V8 (no counterpart in the reference) stores float values in
 * the 8-column layout of SPC5Mat<double> (uint8 masks, headers identical to
 * the double conversion of the same pattern); it serves the mixed-precision
 * calls (float x, FP64 accumulation and y) with half the value bytes of F64. */
enum spc5cuda_value_type { SPC5CUDA_F64 = 0, SPC5CUDA_F32 = 1, SPC5CUDA_F32_V8 = 2 };

/* Status codes (the reference throws std::invalid_argument for an unknown
 * format, spc5.hpp:1014; errors never cross this ABI as exceptions). */
typedef int spc5cuda_status;
#define SPC5CUDA_OK 0
#define SPC5CUDA_ERR_INVALID 1     /* bad argument, size or alignment      */
#define SPC5CUDA_ERR_CUDA 2        /* a CUDA runtime call failed           */
#define SPC5CUDA_ERR_NOMEM 3       /* device allocation failed             */
#define SPC5CUDA_ERR_FORMAT 4      /* unknown format / wrong matrix state  */
#define SPC5CUDA_ERR_UNSUPPORTED 5 /* valid request this build cannot run  */
#define SPC5CUDA_ERR_TIMEOUT 6     /* a bounded device wait gave up        */
#define SPC5CUDA_ERR_DEVICE 7      /* a kernel reported a data error       */

SPC5CUDA_API const char* spc5cuda_status_string(spc5cuda_status s);

/* Status of the last void drop-in call (core_SPC5_*) on this host thread. */
SPC5CUDA_API spc5cuda_status spc5cuda_get_last_error(void);

/* Stream used by the void drop-in entry points on this host thread
 * (default NULL = legacy default stream). */
SPC5CUDA_API void spc5cuda_set_stream(void* stream);

/* ------------------------------------------------------------------------
 * Drop-in kernels.  Same names, argument order and meaning as the
 * reference's extern "C" kernels, over device pointers:
 *   core_SPC5_1rVc_Spmv_{double,float}  spc5.hpp:516-523
 *   core_SPC5_2rVc_Spmv_{double,float}  spc5.hpp:641-648
 *   core_SPC5_4rVc_Spmv_{double,float}  spc5.hpp:769-776
 *   core_SPC5_8rVc_Spmv_{double,float}  spc5.hpp:895-902
 * y[0..nbRows) += A x.  The value offset of every block-row is not stored
 * in the format, so each call first derives it from the headers (one extra
 * pass over the header array), tests on the device whether every block-row
 * fits the row kernel's staging buffers, and runs the row kernel if so, else
 * the group kernel (both enqueued, each gated on that device flag: no host
 * round trip).  Scratch (block-row offsets and work splits) comes from a
 * stream-ordered memory pool the library keeps per device.  The handle API
 * below keeps the offsets resident and adds the length-sorted plan for
 * irregular matrices.  Errors: spc5cuda_get_last_error().
 * ---------------------------------------------------------------------- */
SPC5CUDA_API void core_SPC5_1rVc_Spmv_double(const long int nbRows, const int* rowsSizes,
                                const unsigned char* blocksColumnIndexesWithMasks,
                                const double* values, const double* x, double* y);
SPC5CUDA_API void core_SPC5_2rVc_Spmv_double(const long int nbRows, const int* rowsSizes,
                                const unsigned char* blocksColumnIndexesWithMasks,
                                const double* values, const double* x, double* y);
SPC5CUDA_API void core_SPC5_4rVc_Spmv_double(const long int nbRows, const int* rowsSizes,
                                const unsigned char* blocksColumnIndexesWithMasks,
                                const double* values, const double* x, double* y);
SPC5CUDA_API void core_SPC5_8rVc_Spmv_double(const long int nbRows, const int* rowsSizes,
                                const unsigned char* blocksColumnIndexesWithMasks,
                                const double* values, const double* x, double* y);
SPC5CUDA_API void core_SPC5_1rVc_Spmv_float(const long int nbRows, const int* rowsSizes,
                               const unsigned char* blocksColumnIndexesWithMasks,
                               const float* values, const float* x, float* y);
SPC5CUDA_API void core_SPC5_2rVc_Spmv_float(const long int nbRows, const int* rowsSizes,
                               const unsigned char* blocksColumnIndexesWithMasks,
                               const float* values, const float* x, float* y);
SPC5CUDA_API void core_SPC5_4rVc_Spmv_float(const long int nbRows, const int* rowsSizes,
                               const unsigned char* blocksColumnIndexesWithMasks,
                               const float* values, const float* x, float* y);
SPC5CUDA_API void core_SPC5_8rVc_Spmv_float(const long int nbRows, const int* rowsSizes,
                               const unsigned char* blocksColumnIndexesWithMasks,
                               const float* values, const float* x, float* y);

/* The same drop-in with an explicit r, stream and status (r in {1,2,4,8}). */
SPC5CUDA_API spc5cuda_status spc5cuda_core_spmv_f64(int r, long nbRows, const int* rowsSizes,
                                       const unsigned char* headers, const double* values,
                                       const double* x, double* y, void* stream);
SPC5CUDA_API spc5cuda_status spc5cuda_core_spmv_f32(int r, long nbRows, const int* rowsSizes,
                                       const unsigned char* headers, const float* values,
                                       const float* x, float* y, void* stream);

/* FP64 drop-in that allocates nothing (no counterpart in the reference).
 * For callers that may not allocate device memory during the call -- an
 * application that fixes its memory budget at start-up, a real-time loop
 * that must stay out of the allocator, or a host whose memory pool belongs
 * to another framework.  Same arguments and result as
 * spc5cuda_core_spmv_f64; the per-call scratch lives in one file-scope
 * device array of ~4.5 MB that every GPU loading the library keeps until the
 * process exits.  Limit: ceil(nbRows / r) <= 1,048,576 block-rows, else
 * SPC5CUDA_ERR_INVALID.  The first call on a device looks up the array's
 * address with that device current, so make it before any stream capture;
 * the address is kept for the process, so do not call this entry point on a
 * device after cudaDeviceReset of that device.  All calls share the array: calls that overlap on the GPU (other streams or
 * threads without ordering) race; order them on one stream. */
SPC5CUDA_API spc5cuda_status spc5cuda_core_spmv_f64_noalloc(int r, long nbRows,
                                                            const int* rowsSizes,
                                                            const unsigned char* headers,
                                                            const double* values,
                                                            const double* x, double* y,
                                                            void* stream);

/* ------------------------------------------------------------------------
 * Matrix handle: the device-resident counterpart of SPC5Mat<T>
 * (spc5.hpp:44-62) plus the precomputed partition that replaces the OpenMP
 * ThreadInterval split (spc5.hpp:331-427).
 * ---------------------------------------------------------------------- */
typedef struct spc5cuda_mat spc5cuda_mat;

typedef struct spc5cuda_info {
    int value_type;   /* SPC5CUDA_F64 / SPC5CUDA_F32                        */
    int format;       /* spc5cuda_format                                    */
    int r;            /* rows per block (0 while CSR)                       */
    int vs;           /* columns per block: 8 (f64) or 16 (f32)             */
    int nrows, ncols;
    long nnz;
    long nblocks;     /* numberOfBlocks (0 while CSR)                       */
    long header_bytes;/* nblocks * (4 + r * mask bytes)                     */
    long device_bytes;/* bytes of device memory held by the handle          */
} spc5cuda_info;

/* CSR -> handle (the reference builds CSR with COO_sorted_to_CSR,
 * spc5.hpp:77-104).  Column indices must be sorted inside each row (the
 * greedy conversion assumes it, like the reference).  values are of the
 * handle's value type.  on_device != 0: the three arrays are device
 * pointers; else host pointers (copied).  The call synchronises stream. */
SPC5CUDA_API spc5cuda_status spc5cuda_mat_create_csr(spc5cuda_mat** out, int value_type, int nrows,
                                        int ncols, long nnz, const int* rowptr,
                                        const int* colidx, const void* values, int on_device,
                                        void* stream);

/* Already-converted beta arrays -> handle (e.g. from a host SPC5Mat after
 * CSR_to_SPC5).  rowsSize holds ceil(nrows/r)+1 ints. */
SPC5CUDA_API spc5cuda_status spc5cuda_mat_create_beta(spc5cuda_mat** out, int value_type, int r, int nrows,
                                         int ncols, long nnz, long nblocks, const int* rowsSize,
                                         const unsigned char* headers, const void* values,
                                         int on_device, void* stream);

SPC5CUDA_API spc5cuda_status spc5cuda_mat_destroy(spc5cuda_mat* mat);
SPC5CUDA_API spc5cuda_status spc5cuda_mat_info(const spc5cuda_mat* mat, spc5cuda_info* out);

/* SpMV kernel selection (no counterpart in the reference, which has one
 * kernel per r and instruction set).  Both kernels give the same bits.
 *   AUTO   -- the thread-per-sub-row kernel when every block-row fits its
 *             per-warp staging buffers (stencils, Poisson, banded); the
 *             length-sorted plan (below) when some block-row does not;
 *   GROUPS -- always the group kernel (one group of VS lanes per block-row
 *             stream);
 *   ROWS   -- the thread-per-sub-row kernel; SPC5CUDA_ERR_UNSUPPORTED on a
 *             converted matrix with a block-row that does not fit;
 *   SORTED -- the length-sorted plan: the handle holds its headers and
 *             values with the block-rows sorted by size (the largest ones
 *             as multiply-add chains at r = 2, 4, 8, in segments at r = 1)
 *             instead of in the reference order, and SpMV runs each size
 *             class with the kernel and lanes per block-row that suit it.
 *             AUTO uses it when some block-row does not fit the row kernel
 *             (power-law and other irregular matrices).
 * spc5cuda_mat_kernel reports the kernel SpMV uses now (GROUPS, ROWS or
 * SORTED; AUTO before conversion).  Selecting SORTED (or AUTO, where it picks
 * the plan) on a converted matrix builds the plan and releases the
 * reference-order arrays; selecting GROUPS or ROWS rebuilds them from the
 * plan and releases the plan.  Both synchronise the device.
 * spc5cuda_get_arrays and spc5cuda_decode_coo return the reference order
 * whichever form the handle holds; spc5cuda_batch_create rebuilds it into the
 * handle (which then holds both). */
#define SPC5CUDA_KERNEL_AUTO 0
#define SPC5CUDA_KERNEL_GROUPS 1
#define SPC5CUDA_KERNEL_ROWS 2
#define SPC5CUDA_KERNEL_SORTED 3
SPC5CUDA_API spc5cuda_status spc5cuda_mat_set_kernel(spc5cuda_mat* mat, int kernel);
SPC5CUDA_API spc5cuda_status spc5cuda_mat_kernel(const spc5cuda_mat* mat, int* kernel);
/* Kernel launches one spc5cuda_spmv of a converted handle makes now (one
 * per part of the length-sorted plan, else 1; 0 for an empty matrix). */
SPC5CUDA_API spc5cuda_status spc5cuda_mat_spmv_launches(const spc5cuda_mat* mat, int* launches);

/* SPC5_{r}rVc_block_count (spc5.hpp:510-513, 635-638, 764-767, 890-893):
 * number of blocks the conversion to r would produce.  CSR handles only.
 * Synchronises stream. */
SPC5CUDA_API spc5cuda_status spc5cuda_block_count(const spc5cuda_mat* mat, int r, long* nblocks, void* stream);

/* CSR_to_SPC5 (spc5.hpp:989-1018) on the device: converts a CSR handle in
 * place to format (2..5); the arrays equal the reference's bit for bit.
 * Synchronises stream (the block count sizes the header allocation). */
SPC5CUDA_API spc5cuda_status spc5cuda_convert(spc5cuda_mat* mat, int format, void* stream);

/* Copy the converted arrays out (SPC5Mat::rowsSize / blocksColumnIndexesWithMasks
 * / values).  to_host != 0: host destinations, synchronous. */
SPC5CUDA_API spc5cuda_status spc5cuda_get_arrays(const spc5cuda_mat* mat, int* rowsSize,
                                    unsigned char* headers, void* values, int to_host,
                                    void* stream);

/* SPC5_Spmv (spc5.hpp:1090-1118): y += A x, device x (ncols) and y (nrows)
 * of the handle's value type. */
SPC5CUDA_API spc5cuda_status spc5cuda_spmv(const spc5cuda_mat* mat, const void* x, void* y, void* stream);

/* Mixed precision (no counterpart in the reference): an F32 or F32_V8
 * handle, float x, double y; FP64 per-lane accumulation and FP64 row
 * reduction.  On an F32_V8 handle each chain is the FP64 kernel's chain on
 * the float values and float x widened to double (their product is exact in
 * FP64), so y equals spc5cuda_spmv on the F64 matrix of the rounded values
 * and x.  spc5cuda_spmv and spc5cuda_spmm reject F32_V8 handles
 * (SPC5CUDA_ERR_FORMAT): only the mixed calls take them. */
SPC5CUDA_API spc5cuda_status spc5cuda_spmv_mixed(const spc5cuda_mat* mat, const float* x, double* y,
                                    void* stream);

/* Multi-RHS SpMM (no counterpart in the reference): Y += A X for k
 * right-hand sides.  X is row-major ncols x k with leading dimension
 * ldx >= k (the k values of one matrix column are contiguous), Y row-major
 * nrows x k with ldy >= k.  Column j of Y is bit-identical to spc5cuda_spmv
 * with column j of X.  The kernel follows the handle's choice (see
 * spc5cuda_mat_set_kernel): through the length-sorted plan when the handle
 * has one; the staged SpMM when every block-row fits the row kernels'
 * buffers; the group SpMM for SPC5CUDA_KERNEL_GROUPS.  Up to 16 right-hand
 * sides run in one pass over the matrix (fewer at larger r: at most 32
 * accumulators per lane); larger k runs several passes. */
SPC5CUDA_API spc5cuda_status spc5cuda_spmm(const spc5cuda_mat* mat, int k, const void* X,
                                           long ldx, void* Y, long ldy, void* stream);
SPC5CUDA_API spc5cuda_status spc5cuda_spmm_mixed(const spc5cuda_mat* mat, int k, const float* X,
                                                 long ldx, double* Y, long ldy, void* stream);

/* COO triplets -> CSR handle on the device, following COO_sorted_to_CSR /
 * COO_unsorted_to_CSR (spc5.hpp:77-114): sorted == 0 sorts by (row, column)
 * first.  Duplicate (row, column) entries are rejected (SPC5CUDA_ERR_INVALID):
 * the beta conversion needs unique columns per row.  Synchronises stream. */
SPC5CUDA_API spc5cuda_status spc5cuda_mat_create_coo(spc5cuda_mat** out, int value_type,
                                                     int nrows, int ncols, long nnz,
                                                     const int* rows, const int* cols,
                                                     const void* values, int on_device, int sorted,
                                                     void* stream);

/* Converted matrix -> COO triplets in storage order (block by block, sub-row,
 * column), the corrected core_SPC5_rVc_iterate (spc5.hpp:255-273; the
 * reference reads the masks at the block-row index, line 263).  Device
 * outputs of nnz entries each. */
SPC5CUDA_API spc5cuda_status spc5cuda_decode_coo(const spc5cuda_mat* mat, int* rows, int* cols,
                                                 void* values, void* stream);

/* ------------------------------------------------------------------------
 * Format selection.
 * ---------------------------------------------------------------------- */

/* SPC5_find_best (spc5.hpp:1151-1223): the reference's cubic model in the
 * average values per block, evaluated for r = 1, 2, 4 on block counts taken
 * on the device.  CSR handles only.  Writes r (0 if no estimate is > 0). */
SPC5CUDA_API spc5cuda_status spc5cuda_find_best(const spc5cuda_mat* mat, int* r,
                                                double* estimate, void* stream);

#define SPC5CUDA_TUNE_MODEL 0   /* B200 cost model on device block counts   */
#define SPC5CUDA_TUNE_MEASURE 1 /* trial conversion + timed SpMV per r      */

typedef struct spc5cuda_tune {
    int r;            /* chosen rows per block                             */
    int pad;
    long blocks[4];   /* block counts for r = 1, 2, 4, 8                   */
    double est_us[4]; /* modelled or measured SpMV microseconds per r      */
} spc5cuda_tune;

/* The project's autotuner (replaces SPC5_find_best on this hardware):
 * picks r in {1, 2, 4, 8} for a CSR handle. */
SPC5CUDA_API spc5cuda_status spc5cuda_autotune(const spc5cuda_mat* mat, int mode,
                                               spc5cuda_tune* out, void* stream);

/* ------------------------------------------------------------------------
 * Batched launch (no counterpart in the reference): n converted matrices of
 * one value type, k[i] right-hand sides each, row-major device blocks X[i]
 * (ncols_i x k[i], ldx[i]) and Y[i] (nrows_i x k[i], ldy[i]), Y[i] += A_i X[i].
 * create() builds the job tables and captures one CUDA graph (synchronises
 * stream); launch() replays it on stream.  The X / Y pointers are fixed at
 * creation.  Results per column equal spc5cuda_spmv bit for bit.
 * ---------------------------------------------------------------------- */
typedef struct spc5cuda_batch spc5cuda_batch;
SPC5CUDA_API spc5cuda_status spc5cuda_batch_create(spc5cuda_batch** out, int n,
                                                   spc5cuda_mat* const* mats, const int* k,
                                                   void* const* X, const long* ldx,
                                                   void* const* Y, const long* ldy, int mixed,
                                                   void* stream);
SPC5CUDA_API spc5cuda_status spc5cuda_batch_launch(spc5cuda_batch* batch, void* stream);
SPC5CUDA_API spc5cuda_status spc5cuda_batch_info(const spc5cuda_batch* batch, int* nclasses,
                                                 long* njobs);
SPC5CUDA_API spc5cuda_status spc5cuda_batch_destroy(spc5cuda_batch* batch);

/* ------------------------------------------------------------------------
 * Request loop (no counterpart in the reference): resident matrices,
 * admission by HBM footprint, same-matrix requests coalesced into
 * multi-RHS launches (k <= max_k), up to `slots` launches in flight
 * (continuous batching), latency percentiles.  A request computes
 * y = A_id x for DEVICE vectors x (ncols) and y (nrows) that stay valid until
 * the request completes.  Each result is bit-identical to a solo SpMV.
 * ---------------------------------------------------------------------- */
typedef struct spc5cuda_server spc5cuda_server;

typedef struct spc5cuda_server_config {
    int slots;        /* concurrent launches (streams), 1..64             */
    int max_k;        /* requests coalesced per launch, 1..16             */
    long hbm_budget;  /* bytes for resident matrices + staging buffers    */
    int mixed;        /* 0: F64 matrices, double x/y; 1: F32 or F32_V8
                         matrices, float x, double y (FP64 accumulation)  */
    int plan_serial;  /* 0 (default): a sorted-plan matrix forks its parts
                         onto the plan's own two streams (measured faster:
                         15.5k against 13.7k req/s at saturation on the
                         serving bench); 1: the parts run in order on the
                         slot's stream, so launches of one matrix in
                         different slots share no plan stream             */
} spc5cuda_server_config;

typedef struct spc5cuda_server_stats {
    long completed;      /* requests completed since the last reset          */
    long launches;       /* SpMM launches                                    */
    double mean_k;       /* requests per launch                              */
    double p50_us;       /* submit -> completion latency percentiles         */
    double p99_us;
    double max_us;
    double req_per_s;    /* completed / (last completion - first submit)     */
    long resident_bytes; /* device bytes of the registered matrices          */
    int matrices;
    int pad;
} spc5cuda_server_stats;

SPC5CUDA_API spc5cuda_status spc5cuda_server_create(spc5cuda_server** out,
                                                    const spc5cuda_server_config* cfg);
/* Registers a converted matrix (the handle stays owned by the caller and
 * must outlive the server).  SPC5CUDA_ERR_NOMEM when the resident bytes
 * plus staging would exceed the HBM budget.  Only while no request is in
 * flight. */
SPC5CUDA_API spc5cuda_status spc5cuda_server_add_matrix(spc5cuda_server* srv, spc5cuda_mat* mat,
                                                        int* id);
SPC5CUDA_API spc5cuda_status spc5cuda_server_submit(spc5cuda_server* srv, int id, const void* x,
                                                    void* y, long* request);
/* Blocks until the request completes (SPC5CUDA_ERR_TIMEOUT after timeout_s);
 * latency_us may be NULL.  A request can be waited on once. */
SPC5CUDA_API spc5cuda_status spc5cuda_server_wait(spc5cuda_server* srv, long request,
                                                  double timeout_s, double* latency_us);
SPC5CUDA_API spc5cuda_status spc5cuda_server_drain(spc5cuda_server* srv, double timeout_s);
SPC5CUDA_API spc5cuda_status spc5cuda_server_get_stats(spc5cuda_server* srv,
                                                   spc5cuda_server_stats* out, int reset);
SPC5CUDA_API spc5cuda_status spc5cuda_server_destroy(spc5cuda_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* SPC5CUDA_H */
