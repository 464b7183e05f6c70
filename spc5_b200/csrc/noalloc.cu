// noalloc.cu -- a drop-in SpMV entry point that allocates no device memory.
//
// Why: the ordinary drop-in (core_SPC5_{r}rVc_Spmv_double) needs scratch on
// every call -- the value offset of each block-row, a scan buffer and the
// per-group ranges -- and takes it from cudaMallocAsync.  Some callers cannot
// allocate at that point: code running inside a memory-budgeted host
// application that forbids allocations after start-up, real-time loops that
// must not enter the allocator, or hosts whose pool is owned by another
// framework.  spc5cuda_core_spmv_f64_noalloc does the same computation with
// its scratch in one fixed, file-scope device array instead, so the call
// itself never allocates or frees.
//
// Limits and rules (also in include/spc5cuda.h):
//   * at most kMaxBlockRows = 1,048,576 block-rows (ceil(nbRows / r)); larger
//     matrices are rejected with SPC5CUDA_ERR_INVALID;
//   * the array costs ~4.5 MB on every GPU that loads the library, for the
//     life of the process;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   * every call shares the one array, so calls whose work overlaps on the GPU
//     (different streams, or different host threads, without ordering between
//     them) race and give wrong results; order them on one stream.  Every
//     scratch word a call reads is written earlier by that same call, so
//     nothing left over from the previous call is ever used.
#include <cuda_runtime.h>

#include <mutex>

#include "handle.h"

namespace spc5cuda {
namespace {

constexpr int kMaxBlockRows = 1 << 20;
constexpr int kMaxGroups = 1 << 16;
constexpr int kScanInts = kMaxBlockRows / 2048 + 2;  // >= scan_tmp_ints(kMaxBlockRows)
constexpr int kValptrOff = 0;
constexpr int kScanOff = kValptrOff + kMaxBlockRows + 1;
constexpr int kGstartOff = kScanOff + kScanInts;
constexpr int kScratchInts = kGstartOff + kMaxGroups + 1;

__device__ __align__(256) int g_noalloc_scratch[kScratchInts];

std::mutex g_scratch_mu;
int* g_scratch_addr[64] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device with that device current).
int* scratch_address() {
    int dev = 0;
    SPC5_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, SPC5CUDA_ERR_UNSUPPORTED, "device index");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        SPC5_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_addr[dev] = static_cast<int*>(p);
    }
    return g_scratch_addr[dev];
}

}  // namespace
}  // namespace spc5cuda

using namespace spc5cuda;

extern "C" {

spc5cuda_status spc5cuda_core_spmv_f64_noalloc(int r, long nbRows, const int* rowsSizes,
                                               const unsigned char* headers, const double* values,
                                               const double* x, double* y, void* stream) {
    return guarded([&] {
        require(r == 1 || r == 2 || r == 4 || r == 8, SPC5CUDA_ERR_FORMAT, "r must be 1, 2, 4 or 8");
        require(nbRows >= 0 && nbRows < (1L << 31), SPC5CUDA_ERR_INVALID, "nbRows out of range");
        if (nbRows == 0) return;
        require(rowsSizes && x && y, SPC5CUDA_ERR_INVALID, "null pointer");
        require(aligned(headers, 4) && aligned(values, 16) && aligned(rowsSizes, 4),
                SPC5CUDA_ERR_INVALID, "misaligned array (headers 4 bytes, values 16 bytes)");
        const int nbr = div_up(nbRows, r);
        require(nbr <= kMaxBlockRows, SPC5CUDA_ERR_INVALID,
                "spc5cuda_core_spmv_f64_noalloc: more than 1,048,576 block-rows");
        const int ngroups = spmv_groups(8, r);
        require(ngroups <= kMaxGroups, SPC5CUDA_ERR_UNSUPPORTED, "too many SpMV groups on this GPU");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int* base = scratch_address();
        int* valptr = base + kValptrOff;
        int* scan_tmp = base + kScanOff;
        int* gstart = base + kGstartOff;
        // value offset of every block-row: per-block-row popcounts, then scan
        launch_blockrow_value_counts(1, r, nbr, rowsSizes, headers, valptr, s);
        exclusive_scan_i32(valptr, valptr, nbr, scan_tmp, s);
        launch_partition(nbr, rowsSizes, ngroups, gstart, s);
        BetaView v;
        v.r = r;
        v.nrows = int(nbRows);
        v.nbr = nbr;
        v.brptr = rowsSizes;
        v.headers = headers;
        v.values = values;
        v.valptr = valptr;
        v.gstart = gstart;
        v.ngroups = ngroups;
        launch_spmv_f64(v, x, y, s);
    });
}

}  // extern "C"
