// The persistent batched-step kernel (include/dragon_batch.h), shared by the
// FP64 batch (batch.cu, compiled without contraction like the single-grid
// FP64 kernels: every member runs exactly the arithmetic of its own
// single-grid step) and the mixed FP32/FP64 batch (batch_mixed.cu, compiled
// like the single-grid mixed kernels: 1D members run their single-grid
// arithmetic exactly; in the 2D MHD phase bodies, inlined into this kernel,
// the compiler may fuse other FP32 multiply-adds than in the single-grid
// kernels, so those members agree with their own mixed advance to FP32
// rounding).
//
// Work items of one member and one step, in dependency order:
//   phase 0      the prologue: step bookkeeping, ghost fill, CFL dt (one item;
//                a mixed batch runs the prologues in a kernel of their own,
//                k_batch_prologue in batch.cu, so that they keep the FP64
//                arithmetic of the single-grid prologue)
//   1D hydro     phase 1: step tiles of tile_1d cells (mixed: kMx1dTile cells,
//                the single-grid mixed sweep's tiling)
//   2D MHD       phase 1: copy of the ghost frame of the state and face B into
//                the output buffers (mhd2d_copy_frame),
//                phases 2-8: the seven phases of the single-grid step, one
//                or more 32 x 8 cell tiles per item (FP64 batches; a mixed
//                batch steps its 2D MHD members with the fused one-kernel
//                step of step_mhd_fused.cuh in a launch of its own,
//                k_batch_fused_mhd in batch_mixed.cu)
// A CTA takes the next item from a global counter, waits until every item of
// the member's previous phase has finished, runs it and counts it done. The
// queue lists a member's phases in order, so every item a CTA can wait for was
// taken earlier by a CTA that is running and never waits on a later item: the
// waits always end (each is bounded anyway, and a wait that gives up is
// counted and reported). The CTA that finishes a member's last item of the
// step flips the member's current buffer unless the step failed or was not
// taken.
#pragma once

#include <cuda_runtime.h>

#include "boundary.cuh"
#include "step1d_mixed.cuh"
#include "step_hydro.cuh"
#include "step_mhd.cuh"
#include "step_mhd_mixed.cuh"
#include "step_mhd_fused.cuh"

namespace dgpu_batch {

using namespace dgpu;

constexpr int kPhases = 9;
constexpr int kThreads = 256;
constexpr int kCopyChunk = kThreads * 16;     // ghost-frame points per copy item
constexpr long long kSpinLimit = 1LL << 24;   // polls of a dependency wait (each >= 64 ns)
enum Kind : int { K1D = 0, KMHD2D = 1 };

struct BatchInst {
    int kind;
    int last_phase;
    int ntiles[kPhases];     // work items of each phase (a mixed batch: none in phase 0)
    int rtiles[kPhases];     // 32 x 8 tiles of each 2D MHD phase
    int group;               // MHD tiles per work item
    int ntj[kPhases];        // MHD phases: tiles along j
    Geo G, FG;
    double* w[2];
    double* B[2];
    MhdScratch S;            // the mixed 2D MHD step reads it as FP32 planes
    StepCtl* ctl;
    const BCEntry* bcs;
    StepArgs sa;
    PrologueArgs pa;
    long long frame;         // ghost-frame points copied by phase 1 (MHD, mhd2d_frame_points)
    // a mixed batch's 2D MHD member runs the fused one-kernel step instead of
    // phases 1-8: its strips, rows per segment, CTAs and first CTA in the
    // batch's fused launch (k_batch_fused_mhd)
    int fuse_strips, fuse_seg_rows, fuse_ctas, fuse_first;
};

struct WorkItem {
    int inst, phase, tile, pad;
};

// What the host needs after a replay, per member.
struct Summary {
    int err, done, steps_done, cur;
};

// counters: [0] dependency waits that gave up and [1] members that have not
// finished the advance (both kept across the launches of an advance), [2] queue
// head, [3 + kPhases * m + p] finished items of member m, phase p (reset per step)
constexpr int kCtrTimeouts = 0, kCtrActive = 1, kCtrHead = 2, kCtrDone = 3;

using StepKernel = void (*)(const BatchInst*, const WorkItem*, int, unsigned*);

__device__ __forceinline__ int ldv(const int* p) { return *(const volatile int*)p; }

__device__ __forceinline__ void wait_count(const unsigned* counter, unsigned target, unsigned* timeouts) {
    long long polls = 0;
    while (*(const volatile unsigned*)counter < target) {
        if (++polls > kSpinLimit) {
            atomicAdd(timeouts, 1u);
            break;
        }
        __nanosleep(64);
    }
    __threadfence();
}

// A member's prologue for the step that reads buffer cur; counts the member
// off `active` when this prologue finds its steps complete.
__device__ __forceinline__ void prologue_item(const BatchInst& I, int cur, unsigned* active) {
    __shared__ int s_was_done;
    if (threadIdx.x == 0) s_was_done = ldv(&I.ctl->done);
    PrologueArgs pa = I.pa;
    pa.slot_in = cur;
    pa.slot_out = cur ^ 1;
    if (I.kind == K1D) prologue_body<false>(I.G, I.FG, I.w[cur], nullptr, I.bcs, I.ctl, pa);
    else prologue_body<true>(I.G, I.FG, I.w[cur], I.B[cur], I.bcs, I.ctl, pa);
    __syncthreads();
    if (threadIdx.x == 0 && !s_was_done && ldv(&I.ctl->done)) atomicSub(active, 1u);
}

template <bool MIXED, int S1D, int SMHD, int TS>
__device__ __forceinline__ void run_item(const BatchInst& I, const WorkItem& wi, int cur, unsigned* active) {
    if constexpr (!MIXED) {
        if (wi.phase == 0) {
            prologue_item(I, cur, active);
            return;
        }
    }
    StepArgs sa = I.sa;
    sa.slot_out = cur ^ 1;
    if (I.kind == K1D) {
        if constexpr (MIXED) step1d_tile_mx<S1D, kMx1dTile>(I.G, I.w[cur], I.w[cur ^ 1], I.ctl, sa, wi.tile);
        else step1d_tile<false, S1D, TS>(I.G, I.w[cur], I.w[cur ^ 1], I.ctl, sa, wi.tile);
        return;
    }
    if (wi.phase == 1) {
        if (ldv(&I.ctl->err) | ldv(&I.ctl->done)) return;
        const long long base = (long long)wi.tile * kCopyChunk;
        const long long end = base + kCopyChunk < I.frame ? base + kCopyChunk : I.frame;
        mhd2d_copy_frame(I.G, I.FG, I.w[cur], I.w[cur ^ 1], I.B[cur], I.B[cur ^ 1], base, end, threadIdx.x, blockDim.x);
        return;
    }
    const int nbx = I.ntj[wi.phase];
    if constexpr (MIXED) {
        const MhdScratchF SF{(float*)I.S.hs, (float*)I.S.fx, (float*)I.S.fy, (float*)I.S.er,
                             (float*)I.S.e0, (float*)I.S.eh, I.S.plane};
        const Mhd2DMixedArgs A{I.G, I.FG, I.w[cur], I.w[cur ^ 1], I.B[cur], I.B[cur ^ 1], SF, I.ctl, sa};
        for (int k = 0; k < I.group; k++) {
            const int tile = wi.tile * I.group + k;
            if (tile >= I.rtiles[wi.phase]) break;  // uniform across the CTA
            if (k) __syncthreads();                 // the previous tile's shared words are read
            const Tile2 T{tile % nbx, tile / nbx, (int)(threadIdx.x % kTileJ), (int)(threadIdx.x / kTileJ)};
            switch (wi.phase) {
                case 2: mx_halfstates(A, T); break;
                case 3: mx_fluxes<SMHD, false>(A, T); break;
                case 4: mx_edges<false>(A, T); break;
                case 5: mx_half(A, T); break;
                case 6: mx_fluxes<SMHD, true>(A, T); break;
                case 7: mx_edges<true>(A, T); break;
                default: mx_update(A, T); break;
            }
        }
    } else {
        const Mhd2DArgs A{I.G, I.FG, I.w[cur], I.w[cur ^ 1], I.B[cur], I.B[cur ^ 1], I.S, I.ctl, sa};
        for (int k = 0; k < I.group; k++) {
            const int tile = wi.tile * I.group + k;
            if (tile >= I.rtiles[wi.phase]) break;  // uniform across the CTA
            if (k) __syncthreads();                 // the previous tile's shared words are read
            const Tile2 T{tile % nbx, tile / nbx, (int)(threadIdx.x % kTileJ), (int)(threadIdx.x / kTileJ)};
            switch (wi.phase) {
                case 2: mhd2d_halfstates(A, T); break;
                case 3: mhd2d_prelim<SMHD>(A, T); break;
                case 4: mhd2d_e0(A, T); break;
                case 5: mhd2d_half(A, T); break;
                case 6: mhd2d_final_flux<SMHD>(A, T); break;
                case 7: mhd2d_efinal(A, T); break;
                default: mhd2d_update(A, T); break;
            }
        }
    }
}

// Resident CTAs per SM the kernel is built for: two for FP64 (128 registers);
// three for the lighter mixed bodies (85 registers, some spilled), which on the
// batch of 2048 1D hydro and 256 2D MHD grids ran 10 % faster than two (1.69e9
// against 1.54e9 cell-updates/s) and faster than four (1.55e9).
template <bool MIXED>
constexpr int kBatchCtasPerSm = MIXED ? 3 : 2;

template <bool MIXED, int S1D, int SMHD, int TS>
__global__ void __launch_bounds__(kThreads, kBatchCtasPerSm<MIXED>) k_batch_step(const BatchInst* __restrict__ insts,
                                                         const WorkItem* __restrict__ items, int nitems,
                                                         unsigned* ctr) {
    __shared__ int s_item;
    // every member has finished its steps (a launch after the last one a graph
    // replay needs): nothing to take from the queue
    if (*(const volatile unsigned*)&ctr[kCtrActive] == 0) return;
    for (;;) {
        __syncthreads();  // the previous item's users of shared memory are done
        if (threadIdx.x == 0) s_item = (int)atomicAdd(&ctr[kCtrHead], 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) return;
        const WorkItem wi = items[it];
        const BatchInst& I = insts[wi.inst];
        unsigned* done = ctr + kCtrDone + (size_t)kPhases * wi.inst;
        // a member that has finished its steps (or failed this one) has nothing
        // left to do in this launch: its items only count themselves, without
        // waiting for the phase before them
        if (wi.phase > 0 && threadIdx.x == 0 && !(ldv(&I.ctl->done) | ldv(&I.ctl->err)))
            wait_count(done + wi.phase - 1, (unsigned)I.ntiles[wi.phase - 1], &ctr[kCtrTimeouts]);
        __syncthreads();
        const int cur = ldv(&I.ctl->cur);
        run_item<MIXED, S1D, SMHD, TS>(I, wi, cur, &ctr[kCtrActive]);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(done + wi.phase, 1u);
            if (wi.phase == I.last_phase && prev + 1 == (unsigned)I.ntiles[wi.phase]) {
                StepCtl* c = I.ctl;
                if (!ldv(&c->err) && !ldv(&c->done)) *(volatile int*)&c->cur = cur ^ 1;
            }
        }
    }
}

// The mixed batch's step kernel for a 1D solver and tile size (batch_mixed.cu).
StepKernel pick_kernel_mx(int s1d, int tile);

// A mixed batch's fused 2D MHD launch (batch_mixed.cu): `ctas` CTAs over the
// members listed in `members` (by increasing fuse_first).
int launch_fused_mhd(const BatchInst* insts, const int* members, int nm, int ctas, unsigned* ctr, cudaStream_t st);
size_t fused_mhd_smem();

}  // namespace dgpu_batch
