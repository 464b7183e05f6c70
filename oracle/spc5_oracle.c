/*
 * spc5_oracle.c -- CPU restatement of SPC5's beta(r,VS) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product library (spc5_b200) never links or calls
 * it, and it is never the thing that is measured as the GPU result.
 *
 * Every function restates one algorithm of the reference header
 * src/spc5.hpp (berenger-eu/spc5) and cites the lines it follows.  Parity of
 * this restatement is pinned against the reference itself, compiled from its
 * own sources into oracle/_ref/ (see oracle/Makefile and
 * tests/test_oracle_vs_reference.py), and against the committed golden
 * fixtures in tests/golden/.
 *
 * Layout (spc5.hpp:17-62, 145-148):
 *   f64: VS = 8 columns per block, one uint8 mask per sub-row
 *   f32: VS = 16 columns per block, one uint16 mask per sub-row
 *   header of one block = int32 first column, then r masks, packed (no
 *   alignment), so the block stride is 4 + r * sizeof(mask) bytes.
 *   rowsSize[0..ceil(n/r)] = block-row pointer (in blocks).
 *   values = the nnz values in block order; inside a block, every value of
 *   sub-row 0 (ascending column), then sub-row 1, and so on.
 *
 * Floating-point order of the SpMV restatements follows the AVX-512 kernels
 * (spc5.hpp:2309-2715, non-MHSUM build): one fused multiply-add accumulator
 * per (sub-row, column-in-block) lane, blocks in order, then the
 * _mm512_reduce_add_{pd,ps} tree, which is a butterfly over lane distance
 * VS/2, ..., 2, 1, then y[row] += sum.
 *
 * Build: cc -O2 -ffp-contract=off -fPIC -shared (oracle/Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

/* ---------------------------------------------------------------------- */
/* header access                                                            */
/* ---------------------------------------------------------------------- */

static int rd_i32(const uint8_t* p) {
    int v;
    memcpy(&v, p, 4);
    return v;
}

static unsigned rd_mask(const uint8_t* p, int mask_bytes) {
    if (mask_bytes == 1) return p[0];
    return (unsigned)p[0] | ((unsigned)p[1] << 8);
}

static void wr_mask(uint8_t* p, int mask_bytes, unsigned m) {
    p[0] = (uint8_t)(m & 0xFFu);
    if (mask_bytes == 2) p[1] = (uint8_t)((m >> 8) & 0xFFu);
}

/* ---------------------------------------------------------------------- */
/* CSR -> beta(r,VS) conversion                                             */
/* ---------------------------------------------------------------------- */

/*
 * Greedy per block-row, restating core_CSR_to_SPC5_rVc<T,r> (spc5.hpp:165-228);
 * for r = 1 this is the same output as CSR_to_SPC5_1rVc (spc5.hpp:455-488).
 *   - heads[i] = first unconsumed entry of sub-row i            (176-182)
 *   - idxCol = min over sub-rows of the column at the head       (186-199)
 *   - every sub-row consumes entries with column < idxCol + VS,
 *     appending the value and setting bit (col - idxCol)          (202-213)
 *   - header = int idxCol then r masks                            (215-216)
 *   - rowsSize[blockrow] = blocks before it                       (220-227)
 *
 * value_size is 8 (double) or 4 (float); vs is 8 or 16; mask_bytes 1 or 2.
 * out_blockrowptr must hold ceil(nrows/r)+1 ints, out_headers
 * nblocks*(4+r*mask_bytes) bytes (use oracle_block_count first), out_values
 * nnz values.  Returns the number of blocks.
 */
long oracle_csr_to_beta(int r, int vs, int mask_bytes, int value_size,
                        int nrows, const int* rowptr, const int* colidx,
                        const void* values, int* out_blockrowptr,
                        uint8_t* out_headers, void* out_values) {
    const int stride = 4 + r * mask_bytes;
    long nblocks = 0;
    long out_val = 0;
    int heads[8];
    unsigned masks[8];
    const uint8_t* vin = (const uint8_t*)values;
    uint8_t* vout = (uint8_t*)out_values;
    for (int row0 = 0; row0 < nrows; row0 += r) {
        out_blockrowptr[row0 / r] = (int)nblocks;
        for (int i = 0; i < r; ++i) heads[i] = (row0 + i < nrows) ? rowptr[row0 + i] : 0;
        for (;;) {
            int have = 0;
            int idx_col = INT_MAX;
            for (int i = 0; i < r; ++i) {
                if (row0 + i < nrows && heads[i] < rowptr[row0 + i + 1]) {
                    have = 1;
                    if (colidx[heads[i]] < idx_col) idx_col = colidx[heads[i]];
                }
            }
            if (!have) break;
            for (int i = 0; i < r; ++i) {
                masks[i] = 0;
                if (row0 + i >= nrows) continue;
                while (heads[i] < rowptr[row0 + i + 1] &&
                       colidx[heads[i]] < idx_col + vs) {
                    memcpy(vout + (size_t)out_val * value_size,
                           vin + (size_t)heads[i] * value_size, (size_t)value_size);
                    out_val += 1;
                    masks[i] |= 1u << (colidx[heads[i]] - idx_col);
                    heads[i] += 1;
                }
            }
            uint8_t* h = out_headers + (size_t)nblocks * stride;
            memcpy(h, &idx_col, 4);
            for (int i = 0; i < r; ++i) wr_mask(h + 4 + i * mask_bytes, mask_bytes, masks[i]);
            nblocks += 1;
        }
    }
    out_blockrowptr[(nrows + r - 1) / r] = (int)nblocks;
    return nblocks;
}

/*
 * Block count of the same greedy, restating core_SPC5_block_count<T,r,VS>
 * (spc5.hpp:276-317).
 */
long oracle_block_count(int r, int vs, int nrows, const int* rowptr, const int* colidx) {
    long nblocks = 0;
    int heads[8];
    for (int row0 = 0; row0 < nrows; row0 += r) {
        for (int i = 0; i < r; ++i) heads[i] = (row0 + i < nrows) ? rowptr[row0 + i] : 0;
        for (;;) {
            int have = 0;
            int idx_col = INT_MAX;
            for (int i = 0; i < r; ++i) {
                if (row0 + i < nrows && heads[i] < rowptr[row0 + i + 1]) {
                    have = 1;
                    if (colidx[heads[i]] < idx_col) idx_col = colidx[heads[i]];
                }
            }
            if (!have) break;
            nblocks += 1;
            for (int i = 0; i < r; ++i) {
                if (row0 + i >= nrows) continue;
                while (heads[i] < rowptr[row0 + i + 1] && colidx[heads[i]] < idx_col + vs)
                    heads[i] += 1;
            }
        }
    }
    return nblocks;
}

/*
 * Per-block-row block counts (the first pass of a two-pass conversion); the
 * same greedy as oracle_block_count, split by block-row.
 */
void oracle_blockrow_counts(int r, int vs, int nrows, const int* rowptr,
                            const int* colidx, int* out_counts) {
    int heads[8];
    for (int row0 = 0; row0 < nrows; row0 += r) {
        int cnt = 0;
        for (int i = 0; i < r; ++i) heads[i] = (row0 + i < nrows) ? rowptr[row0 + i] : 0;
        for (;;) {
            int have = 0;
            int idx_col = INT_MAX;
            for (int i = 0; i < r; ++i) {
                if (row0 + i < nrows && heads[i] < rowptr[row0 + i + 1]) {
                    have = 1;
                    if (colidx[heads[i]] < idx_col) idx_col = colidx[heads[i]];
                }
            }
            if (!have) break;
            cnt += 1;
            for (int i = 0; i < r; ++i) {
                if (row0 + i >= nrows) continue;
                while (heads[i] < rowptr[row0 + i + 1] && colidx[heads[i]] < idx_col + vs)
                    heads[i] += 1;
            }
        }
        out_counts[row0 / r] = cnt;
    }
}

/* ---------------------------------------------------------------------- */
/* beta(r,VS) SpMV, y += A x                                                */
/* ---------------------------------------------------------------------- */

/*
 * FP64, restating core_SPC5_{1,2,4,8}rVc_Spmv_double (spc5.hpp:2309-2336,
 * 2368-2403, 2446-2495, 2554-2632):
 *   acc[i][c] = fma(expand(mask_i, values)[c], x[col + c], acc[i][c])
 *   values += popcount(mask_i)                   (per sub-row, in order)
 *   y[row + i] += reduce_add(acc[i])             ((a0+a4)+(a2+a6))+((a1+a5)+(a3+a7))
 * x is read at every lane of the window like _mm512_loadu_pd, so x must be
 * readable up to ncols + 7 (SPC5_VEC_PADDING_X, spc5.hpp:26-29).  Only rows
 * < nrows are written (the reference also writes the r-1 padding rows of the
 * last block-row with +0.0 sums).
 */
void oracle_beta_spmv_f64(int r, int nrows, const int* brptr, const uint8_t* headers,
                          const double* values, const double* x, double* y) {
    const int stride = 4 + r;
    double acc[8][8];
    const double* v = values;
    const uint8_t* h = headers;
    for (int row0 = 0, br = 0; row0 < nrows; row0 += r, ++br) {
        memset(acc, 0, sizeof(acc));
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const int col = rd_i32(h);
            for (int i = 0; i < r; ++i) {
                const unsigned m = h[4 + i];
                int k = 0;
                for (int c = 0; c < 8; ++c) {
                    const double e = ((m >> c) & 1u) ? v[k++] : 0.0;
                    acc[i][c] = fma(e, x[col + c], acc[i][c]);
                }
                v += k;
            }
            h += stride;
        }
        for (int i = 0; i < r && row0 + i < nrows; ++i) {
            const double* a = acc[i];
            const double s = ((a[0] + a[4]) + (a[2] + a[6])) + ((a[1] + a[5]) + (a[3] + a[7]));
            y[row0 + i] += s;
        }
    }
}

/*
 * FP32, restating core_SPC5_{1,2,4,8}rVc_Spmv_float (spc5.hpp:2338-2365,
 * 2407-2442, 2500-2549, 2637-2715) with the _mm512_reduce_add_ps tree
 * (lane distance 8, 4, 2, 1).
 */
static float tree16f(const float* a) {
    float t3[8], t6[4], t8[2];
    for (int i = 0; i < 8; ++i) t3[i] = a[i + 8] + a[i];
    for (int i = 0; i < 4; ++i) t6[i] = t3[i + 4] + t3[i];
    t8[0] = t6[0] + t6[2];
    t8[1] = t6[1] + t6[3];
    return t8[0] + t8[1];
}

void oracle_beta_spmv_f32(int r, int nrows, const int* brptr, const uint8_t* headers,
                          const float* values, const float* x, float* y) {
    const int stride = 4 + 2 * r;
    float acc[8][16];
    const float* v = values;
    const uint8_t* h = headers;
    for (int row0 = 0, br = 0; row0 < nrows; row0 += r, ++br) {
        memset(acc, 0, sizeof(acc));
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const int col = rd_i32(h);
            for (int i = 0; i < r; ++i) {
                const unsigned m = rd_mask(h + 4 + 2 * i, 2);
                int k = 0;
                for (int c = 0; c < 16; ++c) {
                    const float e = ((m >> c) & 1u) ? v[k++] : 0.0f;
                    acc[i][c] = fmaf(e, x[col + c], acc[i][c]);
                }
                v += k;
            }
            h += stride;
        }
        for (int i = 0; i < r && row0 + i < nrows; ++i) y[row0 + i] += tree16f(acc[i]);
    }
}

/*
 * Mixed precision (no counterpart in the reference): the f32 layout
 * (VS = 16, uint16 masks, FP32 values and x) with FP64 lane accumulators,
 * FP64 tree reduction (lane distance 8, 4, 2, 1) and FP64 y.  The product of
 * two floats is exact in double, so fma((double)v, (double)x, acc) rounds
 * once per term.  This is the definition the CUDA mixed kernel follows.
 */
static double tree16d(const double* a) {
    double t3[8], t6[4], t8[2];
    for (int i = 0; i < 8; ++i) t3[i] = a[i + 8] + a[i];
    for (int i = 0; i < 4; ++i) t6[i] = t3[i + 4] + t3[i];
    t8[0] = t6[0] + t6[2];
    t8[1] = t6[1] + t6[3];
    return t8[0] + t8[1];
}

void oracle_beta_spmv_mixed(int r, int nrows, const int* brptr, const uint8_t* headers,
                            const float* values, const float* x, double* y) {
    const int stride = 4 + 2 * r;
    double acc[8][16];
    const float* v = values;
    const uint8_t* h = headers;
    for (int row0 = 0, br = 0; row0 < nrows; row0 += r, ++br) {
        memset(acc, 0, sizeof(acc));
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const int col = rd_i32(h);
            for (int i = 0; i < r; ++i) {
                const unsigned m = rd_mask(h + 4 + 2 * i, 2);
                int k = 0;
                for (int c = 0; c < 16; ++c) {
                    if ((m >> c) & 1u) {
                        acc[i][c] = fma((double)v[k], (double)x[col + c], acc[i][c]);
                        k++;
                    }
                }
                v += k;
            }
            h += stride;
        }
        for (int i = 0; i < r && row0 + i < nrows; ++i) y[row0 + i] += tree16d(acc[i]);
    }
}

/*
 * The same FP64 product regrouped as multiply-add chains, the form in which
 * the CUDA path runs the largest block-rows of irregular matrices: the
 * accumulator of (sub-row i, column c) in oracle_beta_spmv_f64 above
 * (spc5.hpp:2309-2632) only changes at the blocks whose mask i has bit c,
 * so its chain is the list of those values and x indices in block order;
 * each chain is evaluated from +0.0 on its own, then the reduce_add tree of
 * the 8 chain results of a sub-row is added to y.  The reference's
 * fma(0, x, acc) at a clear bit leaves acc unchanged for finite x (acc starts
 * at +0.0 and never becomes -0.0 in round-to-nearest), so for finite x this
 * equals oracle_beta_spmv_f64 bit for bit.  Returns 0, or -1 when out of
 * memory.
 */
int oracle_beta_spmv_f64_chains(int r, int nrows, const int* brptr, const uint8_t* headers,
                                const double* values, const double* x, double* y) {
    const int stride = 4 + r;
    const int nbr = (nrows + r - 1) / r;
    long cap = 0;
    for (int br = 0; br < nbr; ++br) {
        const long nb = brptr[br + 1] - brptr[br];
        if (nb > cap) cap = nb;
    }
    /* chain (i, c) of a block-row holds at most one entry per block */
    double* cval = (double*)malloc(sizeof(double) * (size_t)(64 * (cap > 0 ? cap : 1)));
    int* ccol = (int*)malloc(sizeof(int) * (size_t)(64 * (cap > 0 ? cap : 1)));
    if (!cval || !ccol) {
        free(cval);
        free(ccol);
        return -1;
    }
    const double* v = values;
    for (int br = 0; br < nbr; ++br) {
        int len[8][8];
        memset(len, 0, sizeof(len));
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const uint8_t* h = headers + (long)b * stride;
            const int col = rd_i32(h);
            for (int i = 0; i < r; ++i) {
                const unsigned m = h[4 + i];
                for (int c = 0; c < 8; ++c) {
                    if ((m >> c) & 1u) {
                        const long e = (long)(i * 8 + c) * cap + len[i][c]++;
                        cval[e] = *v++;
                        ccol[e] = col + c;
                    }
                }
            }
        }
        const int row0 = br * r;
        for (int i = 0; i < r && row0 + i < nrows; ++i) {
            double a[8];
            for (int c = 0; c < 8; ++c) {
                double acc = 0.0;
                const long e0 = (long)(i * 8 + c) * cap;
                for (int j = 0; j < len[i][c]; ++j) acc = fma(cval[e0 + j], x[ccol[e0 + j]], acc);
                a[c] = acc;
            }
            y[row0 + i] += ((a[0] + a[4]) + (a[2] + a[6])) + ((a[1] + a[5]) + (a[3] + a[7]));
        }
    }
    free(cval);
    free(ccol);
    return 0;
}

/*
 * Multi-RHS (SpMM) FP64 restatement: column j of X (leading dimension ldx)
 * goes through exactly the FP64 SpMV order above, so every column of
 * the result equals an independent SpMV of that column.
 */
void oracle_beta_spmm_f64(int r, int nrows, const int* brptr, const uint8_t* headers,
                          const double* values, int k, const double* X, long ldx,
                          double* Y, long ldy) {
    for (int j = 0; j < k; ++j)
        oracle_beta_spmv_f64(r, nrows, brptr, headers, values, X + (size_t)j * ldx,
                             Y + (size_t)j * ldy);
}

/* ---------------------------------------------------------------------- */
/* CSR oracle and decode                                                    */
/* ---------------------------------------------------------------------- */

/*
 * FP64 CSR SpMV, restating CSR_Spmv_scalar (spc5.hpp:116-127): sequential
 * sum per row in storage order, then y[row] += sum.  Also returns, per row,
 * sum |a_ij x_j| in absrow (may be NULL), the scale used by the
 * componentwise error metric of the tests.
 */
void oracle_csr_spmv_f64(int nrows, const int* rowptr, const int* colidx,
                         const double* values, const double* x, double* y,
                         double* absrow) {
    for (int i = 0; i < nrows; ++i) {
        double s = 0.0, a = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const double p = x[colidx[k]] * values[k];
            s += p;
            a += fabs(p);
        }
        y[i] += s;
        if (absrow) absrow[i] = a;
    }
}

/*
 * Decode beta(r,VS) back to COO triplets (row, col, value) in storage order:
 * the corrected form of core_SPC5_rVc_iterate (spc5.hpp:255-273), whose
 * mask lookup indexes by block-row instead of sub-row (line 263).  Returns
 * the number of triplets written (= nnz).
 */
long oracle_beta_to_coo(int r, int vs, int mask_bytes, int value_size, int nrows,
                        const int* brptr, const uint8_t* headers, const void* values,
                        int* out_rows, int* out_cols, void* out_values) {
    const int stride = 4 + r * mask_bytes;
    long k = 0;
    const uint8_t* vin = (const uint8_t*)values;
    uint8_t* vout = (uint8_t*)out_values;
    for (int row0 = 0, br = 0; row0 < nrows; row0 += r, ++br) {
        for (int b = brptr[br]; b < brptr[br + 1]; ++b) {
            const uint8_t* h = headers + (size_t)b * stride;
            const int col = rd_i32(h);
            for (int i = 0; i < r; ++i) {
                const unsigned m = rd_mask(h + 4 + i * mask_bytes, mask_bytes);
                for (int c = 0; c < vs; ++c) {
                    if ((m >> c) & 1u) {
                        out_rows[k] = row0 + i;
                        out_cols[k] = col + c;
                        memcpy(vout + (size_t)k * value_size, vin + (size_t)k * value_size,
                               (size_t)value_size);
                        k += 1;
                    }
                }
            }
        }
    }
    return k;
}

/* ---------------------------------------------------------------------- */
/* COO -> CSR and the format-selection model                                */
/* ---------------------------------------------------------------------- */

/*
 * COO (sorted by row then column) to CSR, restating COO_sorted_to_CSR
 * (spc5.hpp:77-104): histogram of rows into rowptr[i+1], then prefix sum.
 * Unsorted input is first sorted by (i, j) in COO_unsorted_to_CSR
 * (spc5.hpp:107-114); the test side does that sort.
 */
void oracle_coo_sorted_to_csr(int nrows, long nnz, const int* rows, int* rowptr) {
    for (int i = 0; i <= nrows; ++i) rowptr[i] = 0;
    for (long k = 0; k < nnz; ++k) rowptr[rows[k] + 1] += 1;
    for (int i = 2; i <= nrows; ++i) rowptr[i] += rowptr[i - 1];
}

/*
 * The reference's speed model, SPC5_find_best<T> (spc5.hpp:1151-1223): a
 * cubic polynomial in the average number of values per block, per format
 * and precision, evaluated for r = 1, 2, 4 only (8rVc is never considered);
 * the format with the largest estimate wins.  blocks[0..2] are the block
 * counts for r = 1, 2, 4.  Returns r (1, 2 or 4; 0 when no estimate is > 0)
 * and writes the estimate.
 */
int oracle_find_best(int is_double, long nnz, const long blocks[3], double* estimate) {
    static const double cd[3][4] = {
        {2.186490e-03, -7.931533e-02, 8.719444e-01, 3.712380e-01},
        {9.822706e-04, -4.500002e-02, 6.714119e-01, 2.413985e-01},
        {1.320496e-04, -1.222130e-02, 3.520409e-01, 3.603195e-01}};
    static const double cf[3][4] = {
        {-4.039852e-03, 7.997606e-02, 6.892119e-02, 1.508645e+00},
        {-9.195940e-04, 4.442050e-03, 5.273045e-01, 1.101610e+00},
        {-4.464933e-05, 1.867266e-03, 1.520910e-01, 1.186131e+00}};
    static const int rs[3] = {1, 2, 4};
    int best = 0;
    double best_speed = 0.0;
    for (int f = 0; f < 3; ++f) {
        const double* c = is_double ? cd[f] : cf[f];
        const double avg = (double)nnz / (double)blocks[f];
        const double s = c[0] * (avg * avg * avg) + c[1] * (avg * avg) + c[2] * avg + c[3];
        if (s > best_speed) {
            best_speed = s;
            best = rs[f];
        }
    }
    *estimate = best_speed;
    return best;
}

/*
 * Block-balanced split of block-rows over threads, restating the serial
 * scan of core_SPC5_rVc_threadsplit (spc5.hpp:346-387): a thread boundary is
 * placed before block-row R when the target (t+1)*blocks/threads is closer
 * to the blocks before R than to the blocks up to R.  Writes the first row
 * and the first value of each thread (nthreads entries each).
 */
void oracle_threadsplit(int r, int vs, int mask_bytes, int nrows, const int* brptr,
                        const uint8_t* headers, int nthreads, int* start_row,
                        int* nrows_out, long* value_offset) {
    const int stride = 4 + r * mask_bytes;
    const long nblocks = brptr[(nrows + r - 1) / r];
    const double per = (double)nblocks / (double)nthreads;
    int t = 0;
    long val = 0;
    start_row[0] = 0;
    value_offset[0] = 0;
    for (int row0 = 0; row0 < nrows; row0 += r) {
        const int br = row0 / r;
        if (t != nthreads - 1 && row0 &&
            fabs((double)(t + 1) * per - brptr[br]) < fabs((double)(t + 1) * per - brptr[br + 1])) {
            nrows_out[t] = row0 - start_row[t];
            t += 1;
            start_row[t] = row0;
            value_offset[t] = val;
        }
        for (int b = brptr[br]; b < brptr[br + 1]; ++b)
            for (int i = 0; i < r; ++i)
                val += __builtin_popcount(rd_mask(headers + (size_t)b * stride + 4 + i * mask_bytes,
                                                  mask_bytes));
    }
    nrows_out[t] = nrows - start_row[t];
    t += 1;
    for (; t < nthreads; ++t) {
        start_row[t] = nrows;
        value_offset[t] = val;
        nrows_out[t] = 0;
    }
    (void)vs;
}
