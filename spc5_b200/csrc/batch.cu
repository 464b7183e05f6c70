// batch.cu -- many matrices of uneven sizes, each with its own k right-hand
// sides, in one CUDA graph.
//
// Every matrix is cut into jobs of about kJobBlocks blocks along block-row
// boundaries; each pass of kc right-hand sides (kc a power of two, at most
// the register budget of its r) is a separate job.  Jobs are grouped by
// (value kind, r, kc, kernel): one launch of the batched SpMM kernel per class
// walks its job list with a fixed grid.  Matrices whose every block-row fits
// the row kernels' staging buffers (and that did not ask for the group
// kernel) run the staged SpMM, one warp per job; the others the group SpMM.
// The class launches are captured as parallel branches of one graph, so small
// matrices of different classes share the GPU; spc5cuda_batch_launch replays
// the graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "handle.h"

namespace spc5cuda {
namespace {
constexpr int kJobBlocks = 2048;
}  // namespace
}  // namespace spc5cuda

using namespace spc5cuda;

struct spc5cuda_batch {
    Owned mats;                          // BatchMat[n]
    std::vector<Owned> jobs;             // BatchJob[] per class
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int nclasses = 0;
    long njobs = 0;
    ~spc5cuda_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

extern "C" {

spc5cuda_status spc5cuda_batch_create(spc5cuda_batch** out, int n, spc5cuda_mat* const* mats,
                                      const int* k, void* const* X, const long* ldx,
                                      void* const* Y, const long* ldy, int mixed, void* stream) {
    return guarded([&] {
        require(out != nullptr && n >= 0, SPC5CUDA_ERR_INVALID, "args");
        *out = nullptr;
        require(n == 0 || (mats && k && X && ldx && Y && ldy), SPC5CUDA_ERR_INVALID, "null");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        auto* bt = new spc5cuda_batch();
        try {
            std::vector<BatchMat> hm(static_cast<size_t>(n));
            // class (kind, r, kc, staged) -> jobs
            std::map<std::tuple<int, int, int, bool>, std::vector<BatchJob>> classes;
            for (int i = 0; i < n; ++i) {
                const spc5cuda_mat* m = mats[i];
                require(m && m->r != 0, SPC5CUDA_ERR_FORMAT, "batch matrices must be converted");
                require(k[i] >= 0 && ldx[i] >= k[i] && ldy[i] >= k[i], SPC5CUDA_ERR_INVALID, "k");
                const int kind = mixed ? (m->value_type == SPC5CUDA_F32_V8 ? 3 : 2)
                                       : (m->value_type == SPC5CUDA_F64 ? 0 : 1);
                require(mixed ? (m->value_type == SPC5CUDA_F32 || m->value_type == SPC5CUDA_F32_V8)
                              : m->value_type != SPC5CUDA_F32_V8,
                        SPC5CUDA_ERR_FORMAT, "mixed batches need F32 or F32_V8 matrices, the others F64 or F32");
                // batch graphs read the reference order: a handle whose
                // sorted copy held the only one keeps both from here on
                const_cast<spc5cuda_mat*>(m)->restore_original(s);
                BatchMat& b = hm[size_t(i)];
                b.brptr = m->brptr.as<int>();
                b.headers = m->headers.as<uint8_t>();
                b.values = m->values.p;
                b.valptr = m->valptr.as<int>();
                b.x = X[i];
                b.ldx = ldx[i];
                b.y = Y[i];
                b.ldy = ldy[i];
                b.xcs = 1;
                b.ycs = 1;
                b.nrows = m->nrows;
                b.pad = 0;
                if (m->nrows == 0 || k[i] == 0) continue;
                // block-row cuts every ~kJobBlocks blocks
                const int nbr = m->nbr();
                std::vector<int> bp(size_t(nbr) + 1);
                SPC5_CUDA(cudaMemcpyAsync(bp.data(), m->brptr.p, sizeof(int) * bp.size(),
                                          cudaMemcpyDeviceToHost, s));
                SPC5_CUDA(cudaStreamSynchronize(s));
                std::vector<std::pair<int, int>> pieces;
                int start = 0;
                for (int rr = 1; rr <= nbr; ++rr) {
                    if (rr == nbr || bp[size_t(rr)] - bp[size_t(start)] >= kJobBlocks) {
                        pieces.emplace_back(start, rr);
                        start = rr;
                    }
                }
                int kofs = 0;
                while (kofs < k[i]) {
                    const bool staged = m->spmm_view().wstart != nullptr;
                    const int kc = staged ? spmm_rows_kc(vs_of(m->value_type), m->r, k[i] - kofs)
                                          : batch_kc(m->r, k[i] - kofs);
                    auto& list = classes[std::make_tuple(kind, m->r, kc, staged)];
                    for (auto& pc : pieces) list.push_back(BatchJob{i, pc.first, pc.second, kofs});
                    kofs += kc;
                }
            }
            bt->mats.alloc(sizeof(BatchMat) * std::max<size_t>(1, hm.size()));
            if (n > 0)
                SPC5_CUDA(cudaMemcpyAsync(bt->mats.p, hm.data(), sizeof(BatchMat) * hm.size(),
                                          cudaMemcpyHostToDevice, s));
            for (auto& kv : classes) {
                bt->jobs.emplace_back();
                Owned& o = bt->jobs.back();
                o.alloc(sizeof(BatchJob) * kv.second.size());
                SPC5_CUDA(cudaMemcpyAsync(o.p, kv.second.data(), sizeof(BatchJob) * kv.second.size(),
                                          cudaMemcpyHostToDevice, s));
                bt->njobs += long(kv.second.size());
            }
            SPC5_CUDA(cudaStreamSynchronize(s));
            bt->nclasses = int(classes.size());

            // capture: one branch per class, forked from and joined into a
            // private capture stream
            cudaStream_t cap;
            SPC5_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            std::vector<cudaStream_t> br(classes.size());
            std::vector<cudaEvent_t> done(classes.size());
            cudaEvent_t fork;
            SPC5_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
            for (size_t c = 0; c < br.size(); ++c) {
                SPC5_CUDA(cudaStreamCreateWithFlags(&br[c], cudaStreamNonBlocking));
                SPC5_CUDA(cudaEventCreateWithFlags(&done[c], cudaEventDisableTiming));
            }
            SPC5_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            SPC5_CUDA(cudaEventRecord(fork, cap));
            size_t c = 0;
            const int sms = sm_count();
            for (auto& kv : classes) {
                const int kind = std::get<0>(kv.first), r = std::get<1>(kv.first), kc = std::get<2>(kv.first);
                const bool staged = std::get<3>(kv.first);
                const int vs = (kind == 0 || kind == 3) ? 8 : 16;
                const int njobs = int(kv.second.size());
                const int ctas = std::max(1, std::min(div_up(long(njobs) * vs, 128), sms * 16));
                SPC5_CUDA(cudaStreamWaitEvent(br[c], fork, 0));
                if (staged)
                    launch_batch_rows(kind, r, kc, bt->mats.as<BatchMat>(), bt->jobs[c].as<BatchJob>(), njobs,
                                      br[c]);
                else
                    launch_batch(kind, r, kc, bt->mats.as<BatchMat>(), bt->jobs[c].as<BatchJob>(), njobs,
                                 ctas, br[c]);
                SPC5_CUDA(cudaEventRecord(done[c], br[c]));
                SPC5_CUDA(cudaStreamWaitEvent(cap, done[c], 0));
                ++c;
            }
            SPC5_CUDA(cudaStreamEndCapture(cap, &bt->graph));
            SPC5_CUDA(cudaGraphInstantiate(&bt->exec, bt->graph, 0));
            for (size_t q = 0; q < br.size(); ++q) {
                cudaStreamDestroy(br[q]);
                cudaEventDestroy(done[q]);
            }
            cudaEventDestroy(fork);
            cudaStreamDestroy(cap);
        } catch (...) {
            delete bt;
            throw;
        }
        *out = bt;
    });
}

spc5cuda_status spc5cuda_batch_launch(spc5cuda_batch* bt, void* stream) {
    return guarded([&] {
        require(bt != nullptr, SPC5CUDA_ERR_INVALID, "null");
        if (bt->exec) SPC5_CUDA(cudaGraphLaunch(bt->exec, static_cast<cudaStream_t>(stream)));
    });
}

spc5cuda_status spc5cuda_batch_info(const spc5cuda_batch* bt, int* nclasses, long* njobs) {
    return guarded([&] {
        require(bt != nullptr, SPC5CUDA_ERR_INVALID, "null");
        if (nclasses) *nclasses = bt->nclasses;
        if (njobs) *njobs = bt->njobs;
    });
}

spc5cuda_status spc5cuda_batch_destroy(spc5cuda_batch* bt) {
    return guarded([&] { delete bt; });
}

}  // extern "C"
