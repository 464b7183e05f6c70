// plan.cu -- the length-sorted SpMV plan of a matrix with irregular block-rows.
//
// Power-law and other irregular matrices mix block-rows of one block with
// block-rows of hundreds; no single work split suits both.  The plan keeps a
// copy of the matrix with its block-rows sorted by size (largest first) --
// every block-row keeps its own blocks and values in their order, so every
// accumulator sees the same FMA chain and y is bit-identical -- plus perm[i],
// the block-row of y that sorted block-row i belongs to.  The sorted order is
// cut into parts, each run by the kernel that suits its block-rows:
//   * block-rows too large for the row kernel's chunks: the group kernel, on
//     a balanced split of the part (neighbouring block-rows now have about
//     the same size, so the groups of a warp stay in step and rarely end a
//     row inside a window);
//   * the rest: the row kernel with L = 8, 4, 2 or 1 lanes per block-row,
//     the smallest L whose chunk of 32 / L block-rows fits the staging
//     buffers.  Block-rows of one chunk have about the same size, so no lane
//     waits for a much longer neighbour.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

#include "handle.h"

namespace spc5cuda {

namespace {

// key[i] = size of block-row i in row-kernel lane units (rows_lane_units),
// idx[i] = i.
__global__ void k_row_keys(int nbr, const int* __restrict__ brptr, const int* __restrict__ valptr,
                           long kb, long kv, unsigned long long* __restrict__ keys, int* __restrict__ idx) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const long nb = brptr[i + 1] - brptr[i];
        const long nv = valptr[i + 1] - valptr[i];
        keys[i] = static_cast<unsigned long long>(max(nb * kb, nv * kv));
        idx[i] = int(i);
    }
}

// Block and value counts of the sorted block-rows.
__global__ void k_sorted_counts(int nbr, const int* __restrict__ perm, const int* __restrict__ brptr,
                                const int* __restrict__ valptr, int* __restrict__ snb, int* __restrict__ snv) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const int p = perm[i];
        snb[i] = brptr[p + 1] - brptr[p];
        snv[i] = valptr[p + 1] - valptr[p];
    }
}

// Copy block-row perm[i] to sorted position i: one warp per block-row.
template <class V>
__global__ void k_sorted_copy(int nbr, const int* __restrict__ perm, const int* __restrict__ brptr,
                              const int* __restrict__ valptr, const int* __restrict__ sbrptr,
                              const int* __restrict__ svalptr, int stride, const uint8_t* __restrict__ hdr,
                              uint8_t* __restrict__ shdr, const V* __restrict__ vals, V* __restrict__ svals) {
    const int lane = threadIdx.x & 31;
    const long warps = long(gridDim.x) * blockDim.x / 32;
    for (long i = (long(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < nbr; i += warps) {
        const int p = perm[i];
        const long h0 = long(brptr[p]) * stride, hn = long(brptr[p + 1]) * stride - h0;
        const long d0 = long(sbrptr[i]) * stride;
        for (long k = lane; k < hn; k += 32) shdr[d0 + k] = hdr[h0 + k];
        const long v0 = valptr[p], vn = long(valptr[p + 1]) - v0;
        const long w0 = svalptr[i];
        for (long k = lane; k < vn; k += 32) svals[w0 + k] = vals[v0 + k];
    }
}

// counts[j] = number of sorted keys above thr[j] (keys descend).
__global__ void k_class_counts(int nbr, const unsigned long long* __restrict__ skeys,
                               unsigned long long t0, unsigned long long t1, unsigned long long t2,
                               unsigned long long t3, int* __restrict__ counts) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbr; i += long(gridDim.x) * blockDim.x) {
        const unsigned long long k = skeys[i];
        const unsigned long long nk = i + 1 < nbr ? skeys[i + 1] : 0ull;
        // the last index above each threshold marks the count
        if (k > t0 && nk <= t0) counts[0] = int(i + 1);
        if (k > t1 && nk <= t1) counts[1] = int(i + 1);
        if (k > t2 && nk <= t2) counts[2] = int(i + 1);
        if (k > t3 && nk <= t3) counts[3] = int(i + 1);
    }
}

int grid_for(long n, int threads) { return std::max(1, std::min(div_up(n, threads), sm_count() * 8)); }

}  // namespace

void build_sorted_plan(spc5cuda_mat* m, cudaStream_t s) {
    const int nbr = m->nbr();
    const int vs = vs_of(m->value_type);
    const int r = m->r;
    const int stride = 4 + r * mask_bytes_of(m->value_type);
    const int vbytes = value_bytes_of(m->value_type);
    auto plan = std::make_unique<SortedPlan>();
    if (nbr <= 0) {
        m->plan = std::move(plan);
        return;
    }
    // ---- sort the block-rows by size, largest first (stable)
    DevBuf keys(sizeof(unsigned long long) * size_t(nbr), s), skeys(sizeof(unsigned long long) * size_t(nbr), s);
    DevBuf idx(sizeof(int) * size_t(nbr), s);
    plan->perm.alloc(sizeof(int) * size_t(nbr));
    const long kb = rows_lane_units(vs, r, 1, 0), kv = rows_lane_units(vs, r, 0, 1);
    k_row_keys<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, m->brptr.as<int>(), m->valptr.as<int>(), kb, kv,
                                                  keys.as<unsigned long long>(), idx.as<int>());
    SPC5_CUDA(cudaGetLastError());
    size_t temp = 0;
    SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, temp, keys.as<unsigned long long>(),
                                                        skeys.as<unsigned long long>(), idx.as<int>(),
                                                        plan->perm.as<int>(), nbr, 0, 64, s));
    {
        DevBuf tmp(temp, s);
        SPC5_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, temp, keys.as<unsigned long long>(),
                                                            skeys.as<unsigned long long>(), idx.as<int>(),
                                                            plan->perm.as<int>(), nbr, 0, 64, s));
    }
    // ---- sorted block-row and value offsets, then the copy
    plan->sbrptr.alloc(sizeof(int) * size_t(nbr + 1));
    plan->svalptr.alloc(sizeof(int) * size_t(nbr + 1));
    {
        DevBuf snb(sizeof(int) * size_t(nbr), s), snv(sizeof(int) * size_t(nbr), s);
        k_sorted_counts<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, plan->perm.as<int>(), m->brptr.as<int>(),
                                                           m->valptr.as<int>(), snb.as<int>(), snv.as<int>());
        SPC5_CUDA(cudaGetLastError());
        DevBuf tmp(sizeof(int) * size_t(scan_tmp_ints(nbr)), s);
        exclusive_scan_i32(snb.as<int>(), plan->sbrptr.as<int>(), nbr, tmp.as<int>(), s);
        exclusive_scan_i32(snv.as<int>(), plan->svalptr.as<int>(), nbr, tmp.as<int>(), s);
    }
    plan->sheaders.alloc(size_t(std::max(16L, m->nblocks * long(stride) + 16)));
    plan->svalues.alloc(size_t(std::max(16L, (m->nnz + 8) * long(vbytes))));
    {
        const int threads = 256;
        const int blocks = std::max(1, std::min(div_up(long(nbr) * 32, threads), sm_count() * 16));
        if (m->value_type == SPC5CUDA_F64)
            k_sorted_copy<double><<<blocks, threads, 0, s>>>(
                nbr, plan->perm.as<int>(), m->brptr.as<int>(), m->valptr.as<int>(), plan->sbrptr.as<int>(),
                plan->svalptr.as<int>(), stride, m->headers.as<uint8_t>(), plan->sheaders.as<uint8_t>(),
                m->values.as<double>(), plan->svalues.as<double>());
        else
            k_sorted_copy<float><<<blocks, threads, 0, s>>>(
                nbr, plan->perm.as<int>(), m->brptr.as<int>(), m->valptr.as<int>(), plan->sbrptr.as<int>(),
                plan->svalptr.as<int>(), stride, m->headers.as<uint8_t>(), plan->sheaders.as<uint8_t>(),
                m->values.as<float>(), plan->svalues.as<float>());
        SPC5_CUDA(cudaGetLastError());
    }
    // ---- parts: sizes above 8, 4, 2, 1 lane units
    int counts[4] = {0, 0, 0, 0};
    {
        DevBuf dc(4 * sizeof(int), s);
        SPC5_CUDA(cudaMemsetAsync(dc.p, 0, 4 * sizeof(int), s));
        const unsigned long long u = static_cast<unsigned long long>(rows_unit());
        k_class_counts<<<grid_for(nbr, 256), 256, 0, s>>>(nbr, skeys.as<unsigned long long>(), 8 * u, 4 * u,
                                                          2 * u, u, dc.as<int>());
        SPC5_CUDA(cudaGetLastError());
        SPC5_CUDA(cudaMemcpyAsync(counts, dc.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
        SPC5_CUDA(cudaStreamSynchronize(s));
    }
    // counts[j]: block-rows above the limit of L = 8 >> j lanes; every
    // boundary is at least the previous one (sizes descend)
    const int above8 = counts[0];
    int lo = above8;
    if (above8 > 0) plan->parts.push_back({0, 0, above8});
    const int lanes_of[4] = {8, 4, 2, 1};
    for (int j = 0; j < 4; ++j) {
        const int L = lanes_of[j];
        if (L < r) break;
        // block-rows of this part: above the next smaller class's limit (or
        // all the rest when the next class is below r)
        const bool last = j == 3 || lanes_of[j + 1] < r;
        const int hi = last ? nbr : std::max(lo, counts[j + 1]);
        if (hi > lo) plan->parts.push_back({L, lo, hi});
        lo = hi;
        if (last) break;
    }
    // ---- a balanced split of every part
    for (auto& part : plan->parts) {
        const int rows = part.b - part.a;
        if (part.lanes == 0) {
            part.nsplit = std::max(1, std::min(spmv_groups(vs, r), rows));
        } else {
            const int per_chunk = 32 / part.lanes;
            part.nsplit = std::max(1, std::min(rows_warps(vs, r, part.lanes), (rows + per_chunk - 1) / per_chunk));
        }
        part.split.alloc(sizeof(int) * size_t(part.nsplit + 1));
        launch_partition_range(part.a, part.b, plan->sbrptr.as<int>(), part.nsplit, part.split.as<int>(), s);
    }
    for (auto& st : plan->aux) SPC5_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    SPC5_CUDA(cudaEventCreateWithFlags(&plan->fork, cudaEventDisableTiming));
    for (auto& e : plan->join) SPC5_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SPC5_CUDA(cudaStreamSynchronize(s));
    m->plan = std::move(plan);
}

BetaView plan_view(const spc5cuda_mat* m, const SpmvPart& part) {
    const SortedPlan& p = *m->plan;
    BetaView v;
    v.r = m->r;
    v.nrows = m->nrows;
    v.nbr = m->nbr();
    v.brptr = p.sbrptr.as<int>();
    v.headers = p.sheaders.as<uint8_t>();
    v.values = p.svalues.p;
    v.valptr = p.svalptr.as<int>();
    v.perm = p.perm.as<int>();
    if (part.lanes == 0) {
        v.gstart = part.split.as<int>();
        v.ngroups = part.nsplit;
    } else {
        v.wstart = part.split.as<int>();
        v.nwarps = part.nsplit;
        v.lanes = part.lanes;
    }
    return v;
}

void plan_spmv(const spc5cuda_mat* m, const void* x, void* y, bool mixed, cudaStream_t s) {
    SortedPlan& p = *m->plan;
    // the parts write disjoint rows of y: the group-kernel part runs on one
    // plan stream, the smaller row-kernel parts on the other, the largest
    // row-kernel part on the caller's stream; all start after the work
    // already queued on s and s waits for all of them
    std::lock_guard<std::mutex> lk(p.mu);
    SPC5_CUDA(cudaEventRecord(p.fork, s));
    for (auto st : p.aux) SPC5_CUDA(cudaStreamWaitEvent(st, p.fork, 0));
    int biggest = -1;
    long most = -1;
    for (size_t i = 0; i < p.parts.size(); ++i) {
        const long blocks = p.parts[i].lanes ? long(p.parts[i].b - p.parts[i].a) : -1;
        if (blocks > most) most = blocks, biggest = int(i);
    }
    for (size_t i = 0; i < p.parts.size(); ++i) {
        const auto& part = p.parts[i];
        cudaStream_t st = part.lanes == 0 ? p.aux[0] : (int(i) == biggest ? s : p.aux[1]);
        // the launchers pick the row kernel when the view has warp ranges
        const BetaView v = plan_view(m, part);
        if (m->value_type == SPC5CUDA_F64)
            launch_spmv_f64(v, static_cast<const double*>(x), static_cast<double*>(y), st);
        else if (mixed)
            launch_spmv_mixed(v, static_cast<const float*>(x), static_cast<double*>(y), st);
        else
            launch_spmv_f32(v, static_cast<const float*>(x), static_cast<float*>(y), st);
    }
    for (int k = 0; k < 2; ++k) {
        SPC5_CUDA(cudaEventRecord(p.join[k], p.aux[k]));
        SPC5_CUDA(cudaStreamWaitEvent(s, p.join[k], 0));
    }
}

}  // namespace spc5cuda
