// Batched step of many independent grids (include/dragon_batch.h): one
// persistent kernel per step over a device work queue (batch_kernel.cuh), the
// per-step launches captured in a CUDA graph, and an autotuner over the launch
// shape. Members of a batch share one precision: the FP64 batch runs the
// kernel instantiated here; a mixed FP32/FP64 batch runs the one in
// batch_mixed.cu and its prologues in k_batch_prologue below. Every member
// follows its own single-grid advance: exactly in FP64, and in mixed
// precision exactly for 1D members and to FP32 rounding for 2D MHD members.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dragon_batch.h"
#include "batch_kernel.cuh"
#include "handle.h"

void dragon_gpu_set_error_message(const char* msg);

using namespace dgpu;
using namespace dgpu_rt;
using namespace dgpu_batch;

namespace {

int fail(int code, const std::string& msg) {
    dragon_gpu_set_error_message(msg.c_str());
    return code;
}

#define CKB(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return fail(DRAGON_GPU_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
    } while (0)

// The prologues of a mixed batch's members for one step: one CTA per member
// at a time (the step kernel then finds phase 0 complete).
__global__ void __launch_bounds__(kThreads) k_batch_prologue(const BatchInst* __restrict__ insts, int n,
                                                           unsigned* ctr) {
    if (*(const volatile unsigned*)&ctr[kCtrActive] == 0) return;
    for (int m = blockIdx.x; m < n; m += gridDim.x) {
        const BatchInst& I = insts[m];
        prologue_item(I, ldv(&I.ctl->cur), &ctr[kCtrActive]);
        __syncthreads();
    }
}

__global__ void k_batch_summary(const BatchInst* __restrict__ insts, int n, Summary* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const StepCtl* c = insts[i].ctl;
    out[i] = Summary{ldv(&c->err), ldv(&c->done), ldv(&c->steps_done), ldv(&c->cur)};
}

// Built solver combinations: 1D hydro {HLLC, exact} x 2D MHD {HLLD} x tile
// {126, 254} cells (the tile's half states, TS + 2 cells, fill 128 or 256
// threads of the CTA's round).
StepKernel pick_kernel(int s1d, int tile) {
    const bool exact = s1d == RS_EXACT;
    if (tile == 126)
        return exact ? k_batch_step<false, RS_EXACT, RS_HLLD, 126> : k_batch_step<false, RS_HLLC, RS_HLLD, 126>;
    return exact ? k_batch_step<false, RS_EXACT, RS_HLLD, 254> : k_batch_step<false, RS_HLLC, RS_HLLD, 254>;
}

}  // namespace

struct dragon_batch {
    std::vector<dragon_grid*> members;
    dragon_batch_tuning tune{254, 0, 0, 32, 8, 1};
    int s1d = -1;
    int prec = -1;  // the members' precision (0 FP64, 1 mixed)
    cudaStream_t stream = nullptr;
    BatchInst* d_insts = nullptr;
    WorkItem* d_items = nullptr;
    int nitems = 0;
    unsigned* d_ctr = nullptr;
    size_t ctr_words = 0;
    Summary* d_sum = nullptr;
    Summary* h_sum = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool dirty = true;
    int grid_ctas = 0;
    // a mixed batch's 2D MHD members (by increasing fuse_first) and the CTAs of their fused launch
    int* d_fmembers = nullptr;
    int n_fmembers = 0;
    int fuse_ctas = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

void release_device(dragon_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    for (void* p : {(void*)b->d_insts, (void*)b->d_items, (void*)b->d_ctr, (void*)b->d_sum, (void*)b->d_fmembers})
        if (p) cudaFree(p);
    b->d_fmembers = nullptr;
    b->n_fmembers = 0;
    b->fuse_ctas = 0;
    if (b->h_sum) cudaFreeHost(b->h_sum);
    b->d_insts = nullptr;
    b->d_items = nullptr;
    b->d_ctr = nullptr;
    b->d_sum = nullptr;
    b->h_sum = nullptr;
}

int tiles_along(int n, int t) { return (n + t - 1) / t; }

BatchInst make_inst(dragon_grid* h, int tile, int group, bool mixed) {
    BatchInst I;
    std::memset(&I, 0, sizeof(I));
    I.kind = h->dim == 1 ? K1D : KMHD2D;
    I.G = h->cg;
    I.FG = h->fg;
    I.w[0] = h->w[0];
    I.w[1] = h->w[1];
    I.B[0] = h->B[0];
    I.B[1] = h->B[1];
    I.S = h->mhd_s;
    I.ctl = h->ctl;
    I.bcs = h->dbcs;
    I.sa = step_args(h, 0);
    PrologueArgs& pa = I.pa;
    pa.dx = h->d[0];
    pa.dy = h->d[1];
    pa.dz = h->d[2];
    pa.cfl_coeff = h->cfg.cfl_coeff;
    pa.tol = h->cfg.timestep_tol;
    pa.cfl = h->cfg.cfl;
    pa.bookkeeping = 1;
    pa.apply_bc = 1;
    pa.compute_dt = 1;
    pa.nbc = h->nbc;
    pa.bc_first = 0;
    pa.stall_cta = -1;
    I.ntiles[0] = mixed ? 0 : 1;  // a mixed batch runs its prologues in k_batch_prologue
    I.ntj[0] = 1;
    I.group = group < 1 ? 1 : group;
    if (I.kind == K1D) {
        I.last_phase = 1;
        I.ntiles[1] = tiles_along(h->n[0] + 2 * h->g, mixed ? kMx1dTile : tile);
        I.ntj[1] = 1;
        return I;
    }
    const int nx = h->n[0], ny = h->n[1];
    I.frame = mhd2d_frame_points(h->cg.n[0], h->cg.n[1], h->cg.g);
    if (mixed) {
        // the fused step, in the batch's fused launch: segments of up to 128
        // rows (a multiple of the 8 rows an iteration advances; each segment
        // refills the rings once)
        I.last_phase = 0;
        I.fuse_strips = tiles_along(ny, kFuseTJ);
        I.fuse_seg_rows = std::min(128, tiles_along(nx, kFuseR) * kFuseR);
        I.fuse_ctas = I.fuse_strips * tiles_along(nx, I.fuse_seg_rows);
        return I;
    }
    I.last_phase = 8;
    I.ntiles[1] = (int)std::max<long long>(1, (I.frame + kCopyChunk - 1) / kCopyChunk);
    I.ntj[1] = 1;
    // the seven sweeps of the single-grid step and their cell ranges
    const int ext[7] = {4, 4, 3, 2, 2, 1, 0};
    for (int k = 0; k < 7; k++) {
        const int ni = nx + ext[k], nj = ny + ext[k];
        I.ntj[2 + k] = tiles_along(nj, kTileJ);
        I.rtiles[2 + k] = I.ntj[2 + k] * tiles_along(ni, kTileI);
        I.ntiles[2 + k] = tiles_along(I.rtiles[2 + k], I.group);
    }
    return I;
}

std::vector<WorkItem> make_queue(const std::vector<BatchInst>& insts, int order, int wave) {
    std::vector<int> idx(insts.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = (int)i;
    auto cells = [&](int i) {
        const BatchInst& I = insts[i];
        return (long long)I.G.n[0] * I.G.n[1] * (I.kind == KMHD2D ? 8 : 1);
    };
    if (order == 2) std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cells(a) > cells(b); });
    std::vector<WorkItem> q;
    auto emit = [&](int i, int p) {
        for (int t = 0; t < insts[i].ntiles[p]; t++) q.push_back(WorkItem{i, p, t, 0});
    };
    auto emit_kind_phase = [&](int kind, int p) {
        for (int i : idx)
            if (insts[i].kind == kind && p <= insts[i].last_phase) emit(i, p);
    };
    if (order == 1) {
        for (int p = 0; p < kPhases; p++) emit_kind_phase(K1D, p);
        for (int p = 0; p < kPhases; p++) emit_kind_phase(KMHD2D, p);
        return q;
    }
    if (order == 3) {
        // wavefront: diagonal t holds phase p of MHD group t - p, so a group's
        // phases follow one another one diagonal apart; every item of a
        // member's phase p - 1 sits on an earlier diagonal than its phase p
        for (int p = 0; p < kPhases; p++) emit_kind_phase(K1D, p);
        std::vector<std::vector<int>> groups;
        for (int i : idx) {
            if (insts[i].kind != KMHD2D) continue;
            if (groups.empty() || (int)groups.back().size() >= wave) groups.emplace_back();
            groups.back().push_back(i);
        }
        const int ng = (int)groups.size();
        for (int t = 0; t < ng + kPhases - 1; t++)
            for (int p = kPhases - 1; p >= 0; p--) {
                const int g = t - p;
                if (g < 0 || g >= ng) continue;
                for (int i : groups[g])
                    if (p <= insts[i].last_phase) emit(i, p);
            }
        return q;
    }
    // phase-major; the 1D steps sit after the MHD copies so that they fill
    // the gaps of the MHD phase chain
    for (int i : idx) emit(i, 0);
    emit_kind_phase(KMHD2D, 1);
    emit_kind_phase(K1D, 1);
    for (int p = 2; p < kPhases; p++) emit_kind_phase(KMHD2D, p);
    return q;
}

// (Re)builds the device descriptors, the queue and the CUDA graph of
// tune.graph_steps steps.
int build(dragon_batch* b) {
    release_device(b);
    const int n = (int)b->members.size();
    std::vector<BatchInst> insts;
    insts.reserve(n);
    const bool mixed = b->prec == 1;
    for (dragon_grid* h : b->members) insts.push_back(make_inst(h, b->tune.tile_1d, b->tune.mhd_tiles, mixed));
    std::vector<int> fmembers;  // a mixed batch's 2D MHD members, in the fused launch's CTA order
    if (mixed) {
        int first = 0;
        for (int i = 0; i < n; i++) {
            if (insts[i].kind != KMHD2D) continue;
            insts[i].fuse_first = first;
            first += insts[i].fuse_ctas;
            fmembers.push_back(i);
        }
        b->fuse_ctas = first;
        b->n_fmembers = (int)fmembers.size();
    }
    const std::vector<WorkItem> q = make_queue(insts, b->tune.order, std::max(1, b->tune.wave));
    b->nitems = (int)q.size();
    b->ctr_words = kCtrDone + (size_t)kPhases * n;
    CKB(cudaMalloc(&b->d_insts, sizeof(BatchInst) * n));
    CKB(cudaMalloc(&b->d_items, sizeof(WorkItem) * std::max<size_t>(1, q.size())));
    CKB(cudaMalloc(&b->d_ctr, sizeof(unsigned) * b->ctr_words));
    CKB(cudaMalloc(&b->d_sum, sizeof(Summary) * n));
    CKB(cudaMallocHost(&b->h_sum, sizeof(Summary) * n));
    CKB(cudaMemcpyAsync(b->d_insts, insts.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, b->stream));
    if (!q.empty())
        CKB(cudaMemcpyAsync(b->d_items, q.data(), sizeof(WorkItem) * q.size(), cudaMemcpyHostToDevice, b->stream));
    if (!fmembers.empty()) {
        CKB(cudaMalloc(&b->d_fmembers, sizeof(int) * fmembers.size()));
        CKB(cudaMemcpyAsync(b->d_fmembers, fmembers.data(), sizeof(int) * fmembers.size(), cudaMemcpyHostToDevice,
                            b->stream));
    }
    CKB(cudaMemsetAsync(b->d_ctr, 0, sizeof(unsigned) * b->ctr_words, b->stream));
    CKB(cudaStreamSynchronize(b->stream));

    const StepKernel kern = mixed ? pick_kernel_mx(b->s1d, b->tune.tile_1d) : pick_kernel(b->s1d, b->tune.tile_1d);
    int dev = 0, sms = 0, occ = 0;
    CKB(cudaGetDevice(&dev));
    CKB(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CKB(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0));
    if (occ < 1) return fail(DRAGON_GPU_ECUDA, "batched step kernel cannot be resident");
    int per_sm = b->tune.ctas_per_sm > 0 ? std::min(b->tune.ctas_per_sm, occ) : occ;
    b->grid_ctas = std::max(1, std::min(per_sm * sms, b->nitems));

    CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < b->tune.graph_steps; k++) {
        cudaMemsetAsync(b->d_ctr + kCtrHead, 0, sizeof(unsigned) * (b->ctr_words - kCtrHead), b->stream);
        if (mixed) k_batch_prologue<<<std::min(n, sms * 8), kThreads, 0, b->stream>>>(b->d_insts, n, b->d_ctr);
        if (b->nitems > 0) kern<<<b->grid_ctas, kThreads, 0, b->stream>>>(b->d_insts, b->d_items, b->nitems, b->d_ctr);
        if (b->fuse_ctas > 0 &&
            launch_fused_mhd(b->d_insts, b->d_fmembers, b->n_fmembers, b->fuse_ctas, b->d_ctr, b->stream)) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            return fail(DRAGON_GPU_ECUDA, "fused MHD launch of the batch failed");
        }
    }
    k_batch_summary<<<(n + 255) / 256, 256, 0, b->stream>>>(b->d_insts, n, b->d_sum);
    cudaMemcpyAsync(b->h_sum, b->d_sum, sizeof(Summary) * n, cudaMemcpyDeviceToHost, b->stream);
    cudaError_t ec = cudaStreamEndCapture(b->stream, &b->graph);
    if (ec != cudaSuccess) return fail(DRAGON_GPU_ECUDA, std::string("graph capture failed: ") + cudaGetErrorString(ec));
    CKB(cudaGraphInstantiate(&b->gexec, b->graph, 0));
    b->dirty = false;
    return 0;
}

// The reference's catch block (CFL.cpp:194-209) for one member whose step
// failed inside the batch: halve t1 and retry the same step on the same
// ghosts with the member's own kernels.
int retry_member(dragon_grid* h, int* retries) {
    int rc = pull_ctl(h);
    if (rc) return rc;
    StepCtl& C = *h->hctl;
    const int c = C.cur;
    const int stage = (int)(C.err_key >> 56);
    if (stage == ST_CFL_ZERO) return fail(DRAGON_GPU_ECFL, stage_name(stage));
    if (stage == ST_BARRIER) return fail(DRAGON_GPU_ECUDA, stage_name(stage));
    double t1 = C.t1;
    for (;;) {
        (*retries)++;
        t1 *= 0.5;
        if (t1 < h->cfg.timestep_tol)
            return fail(DRAGON_GPU_EDT, std::string("Timestep has fallen below minimum after: ") + stage_name(stage));
        C.t1 = t1;
        C.err = 0;
        C.err_key = ~0ull;
        if ((rc = push_ctl(h))) return rc;
        if ((rc = zero_slot(h, c ^ 1))) return rc;
        if ((rc = launch_step(h, c))) return rc;
        if ((rc = pull_ctl(h))) return rc;
        if (!C.err) break;
    }
    C.cur = c ^ 1;  // the retried step is committed; the next prologue accounts it
    return push_ctl(h);
}

int advance(dragon_batch* b, int nsteps, dragon_batch_stats* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    const int n = (int)b->members.size();
    if (n == 0 || nsteps == 0) return 0;
    int rc;
    // members' pending work, then each member's control block for this advance
    for (dragon_grid* h : b->members) CKB(cudaStreamSynchronize(h->stream));
    for (dragon_grid* h : b->members) {
        if (!h->imax_valid) {
            if ((rc = zero_slot(h, h->cur))) return rc;
            if ((rc = launch_interior_cfl(h, h->cur, h->cur))) return rc;
        }
        reset_ctl(h, INFINITY, nsteps, 1);
        h->hctl->cur = h->cur;
        if ((rc = push_ctl(h))) return rc;
    }
    for (dragon_grid* h : b->members) CKB(cudaStreamSynchronize(h->stream));
    if (b->dirty && (rc = build(b))) return rc;
    CKB(cudaMemsetAsync(b->d_ctr + kCtrTimeouts, 0, sizeof(unsigned), b->stream));
    {
        const unsigned active = (unsigned)n;
        CKB(cudaMemcpyAsync(b->d_ctr + kCtrActive, &active, sizeof(unsigned), cudaMemcpyHostToDevice, b->stream));
        CKB(cudaStreamSynchronize(b->stream));
    }
    int retries = 0, replays = 0;
    float ms_total = 0.f;
    const int max_replays = (nsteps + 1) / b->tune.graph_steps + 2;
    for (int budget = max_replays;;) {
        CKB(cudaEventRecord(b->ev0, b->stream));
        CKB(cudaGraphLaunch(b->gexec, b->stream));
        CKB(cudaEventRecord(b->ev1, b->stream));
        CKB(cudaStreamSynchronize(b->stream));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        ms_total += ms;
        replays++;
        bool all_done = true, failed = false;
        for (int i = 0; i < n; i++) {
            if (b->h_sum[i].err) {
                failed = true;
                if ((rc = retry_member(b->members[i], &retries))) return rc;
                b->h_sum[i].done = 0;
            }
            all_done &= b->h_sum[i].done != 0;
        }
        if (all_done) break;
        // a retried member is one step behind: allow the replays it needs
        if (failed) budget += 1;
        if (--budget <= 0) return fail(DRAGON_GPU_ESTEP, "batched advance did not finish its steps");
    }
    unsigned timeouts = 0;
    CKB(cudaMemcpy(&timeouts, b->d_ctr + kCtrTimeouts, sizeof(unsigned), cudaMemcpyDeviceToHost));
    for (dragon_grid* h : b->members) {
        if ((rc = pull_ctl(h))) return rc;
        add_newton(h, *h->hctl);
        h->cur = h->hctl->cur;
        h->imax_valid = true;
    }
    if (st) {
        st->steps = nsteps;
        st->retries = retries;
        st->graph_replays = replays;
        st->work_items = b->nitems;
        st->spin_timeouts = timeouts;
        st->replay_ms = ms_total;
    }
    if (timeouts) return fail(DRAGON_GPU_ECUDA, "batched step: a dependency wait gave up");
    return 0;
}

}  // namespace

extern "C" {

int dragon_gpu_batch_create(dragon_batch** out) {
    if (!out) return fail(DRAGON_GPU_EINVAL, "null argument");
    dragon_batch* b = new dragon_batch();
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        dragon_gpu_batch_destroy(b);
        return fail(DRAGON_GPU_ECUDA, "batch stream / events");
    }
    *out = b;
    return 0;
}

int dragon_gpu_batch_destroy(dragon_batch* b) {
    if (!b) return 0;
    if (b->stream) cudaStreamSynchronize(b->stream);
    release_device(b);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return 0;
}

int dragon_gpu_batch_add_instance(dragon_batch* b, dragon_grid* h, int* index) {
    if (!b || !h) return fail(DRAGON_GPU_EINVAL, "null argument");
    if (h->cfg.precision != 0 && h->cfg.precision != 1) return fail(DRAGON_GPU_EINVAL, "unknown precision");
    if (b->prec >= 0 && b->prec != h->cfg.precision)
        return fail(DRAGON_GPU_EUNSUPPORTED, "batched members share one precision (FP64 or mixed)");
    if (!h->user_entries.empty())
        return fail(DRAGON_GPU_EUNSUPPORTED, "batched members run built-in boundary elements only (no user fills)");
    if (h->dim == 1 && !h->mhd) {
        if (h->solver != RS_HLLC && h->solver != RS_EXACT)
            return fail(DRAGON_GPU_EUNSUPPORTED, "batched 1D members use HLLC / HLLX or the exact solver");
        if (h->cfg.exact_guess != GUESS_MEAN && h->solver == RS_EXACT)
            return fail(DRAGON_GPU_EUNSUPPORTED, "batched members use the reference's star-pressure guess");
        if (b->s1d >= 0 && b->s1d != h->solver) return fail(DRAGON_GPU_EUNSUPPORTED, "batched 1D members share one solver");
        b->s1d = h->solver;
    } else if (h->dim == 2 && h->mhd) {
        if (h->solver != RS_HLLD) return fail(DRAGON_GPU_EUNSUPPORTED, "batched 2D MHD members use HLLD / HLLX");
    } else {
        return fail(DRAGON_GPU_EUNSUPPORTED, "batches hold 1D hydro and 2D MHD grids");
    }
    for (dragon_grid* m : b->members)
        if (m == h) return fail(DRAGON_GPU_EINVAL, "grid is already in the batch");
    if (index) *index = (int)b->members.size();
    b->prec = h->cfg.precision;
    b->members.push_back(h);
    b->dirty = true;
    return 0;
}

int dragon_gpu_batch_size(const dragon_batch* b) { return b ? (int)b->members.size() : 0; }

int dragon_gpu_batch_set_tuning(dragon_batch* b, const dragon_batch_tuning* t) {
    if (!b || !t) return fail(DRAGON_GPU_EINVAL, "null argument");
    if ((t->tile_1d != 126 && t->tile_1d != 254) || t->ctas_per_sm < 0 || t->ctas_per_sm > 8 || t->order < 0 ||
        t->order > 3 || t->graph_steps < 1 || t->graph_steps > 1024 ||
        !(t->mhd_tiles == 0 || t->mhd_tiles == 1 || t->mhd_tiles == 2 || t->mhd_tiles == 4 || t->mhd_tiles == 8) ||
        t->wave < 0 || t->wave > 64)
        return fail(DRAGON_GPU_EINVAL, "invalid batch tuning");
    b->tune = *t;
    if (b->tune.mhd_tiles == 0) b->tune.mhd_tiles = 1;
    if (b->tune.wave == 0) b->tune.wave = 1;
    b->dirty = true;
    return 0;
}

int dragon_gpu_batch_get_tuning(const dragon_batch* b, dragon_batch_tuning* t) {
    if (!b || !t) return fail(DRAGON_GPU_EINVAL, "null argument");
    *t = b->tune;
    return 0;
}

int dragon_gpu_batch_advance_steps(dragon_batch* b, int nsteps, dragon_batch_stats* st) {
    if (!b || nsteps < 0) return fail(DRAGON_GPU_EINVAL, "invalid argument");
    if (b->s1d < 0) b->s1d = RS_HLLC;
    return advance(b, nsteps, st);
}

int dragon_gpu_batch_autotune(dragon_batch* b, int steps, dragon_batch_tuning* best, double* best_ms) {
    if (!b || steps < 1) return fail(DRAGON_GPU_EINVAL, "invalid argument");
    if (b->members.empty()) return fail(DRAGON_GPU_EINVAL, "empty batch");
    if (b->s1d < 0) b->s1d = RS_HLLC;
    // snapshot every member's state (current buffer, counters) to restore after each candidate
    struct Snap {
        double* w = nullptr;
        double* B = nullptr;
        size_t wn = 0, bn = 0;
        int cur = 0;
        dragon_newton_stats ntot{};
    };
    std::vector<Snap> snaps(b->members.size());
    auto free_snaps = [&]() {
        for (Snap& s : snaps) {
            if (s.w) cudaFree(s.w);
            if (s.B) cudaFree(s.B);
        }
    };
    for (size_t i = 0; i < b->members.size(); i++) {
        dragon_grid* h = b->members[i];
        Snap& s = snaps[i];
        CKB(cudaStreamSynchronize(h->stream));
        s.cur = h->cur;
        s.ntot = h->ntot;
        s.wn = (size_t)h->nf * h->cg.plane;
        s.bn = h->B[0] ? (size_t)3 * h->fg.plane : 0;
        if (cudaMalloc(&s.w, sizeof(double) * s.wn) != cudaSuccess ||
            (s.bn && cudaMalloc(&s.B, sizeof(double) * s.bn) != cudaSuccess)) {
            free_snaps();
            return fail(DRAGON_GPU_ECUDA, "autotune snapshot allocation failed");
        }
        cudaMemcpyAsync(s.w, h->w[h->cur], sizeof(double) * s.wn, cudaMemcpyDeviceToDevice, b->stream);
        if (s.bn) cudaMemcpyAsync(s.B, h->B[h->cur], sizeof(double) * s.bn, cudaMemcpyDeviceToDevice, b->stream);
    }
    CKB(cudaStreamSynchronize(b->stream));
    auto restore = [&]() -> int {
        for (size_t i = 0; i < b->members.size(); i++) {
            dragon_grid* h = b->members[i];
            Snap& s = snaps[i];
            h->cur = s.cur;
            h->ntot = s.ntot;
            h->imax_valid = false;
            CKB(cudaMemcpyAsync(h->w[h->cur], s.w, sizeof(double) * s.wn, cudaMemcpyDeviceToDevice, b->stream));
            if (s.bn) CKB(cudaMemcpyAsync(h->B[h->cur], s.B, sizeof(double) * s.bn, cudaMemcpyDeviceToDevice, b->stream));
        }
        CKB(cudaStreamSynchronize(b->stream));
        return 0;
    };
    const dragon_batch_tuning keep = b->tune;
    dragon_batch_tuning win = keep;
    double win_ms = INFINITY;
    int rc = 0;
    auto trial = [&](const dragon_batch_tuning& t) -> int {
        b->tune = t;
        b->dirty = true;
        dragon_batch_stats s{};
        int r = advance(b, steps, &s);
        if (r) return r;
        if ((r = restore())) return r;
        if (s.replay_ms < win_ms) {
            win_ms = s.replay_ms;
            win = t;
        }
        return 0;
    };
    // launch shape and queue order with one MHD tile per item, then the MHD
    // tiles per item for the best of those, then the wavefront order
    for (int tile : {126, 254})
        for (int per_sm : {1, 2, 4, 8})
            for (int order : {0, 1, 2})
                if (!rc) rc = trial(dragon_batch_tuning{tile, per_sm, order, steps, 1, 1});
    const dragon_batch_tuning base = win;
    bool any_mhd = false;
    for (dragon_grid* h : b->members) any_mhd |= h->dim == 2;
    if (any_mhd) {
        for (int group : {2, 4, 8})
            if (!rc) {
                dragon_batch_tuning t = base;
                t.mhd_tiles = group;
                rc = trial(t);
            }
        // the wavefront order over MHD groups of a few sizes, with the best shape so far
        const dragon_batch_tuning shaped = win;
        for (int wave : {1, 4, 16})
            if (!rc) {
                dragon_batch_tuning t = shaped;
                t.order = 3;
                t.wave = wave;
                rc = trial(t);
            }
    }
    free_snaps();
    win.graph_steps = keep.graph_steps;
    b->tune = win;
    b->dirty = true;
    if (rc) return rc;
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms / steps;
    return 0;
}

}  // extern "C"
