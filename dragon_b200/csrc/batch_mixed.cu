// The mixed FP32/FP64 batched step: k_batch_step (batch_kernel.cuh) over the
// mixed 1D tile bodies (step1d_mixed.cuh), and the fused 2D MHD step
// (step_mhd_fused.cuh) of the MHD members in one launch of its own. Compiled with FMA
// contraction and fast single-precision division / square root, like the
// single-grid mixed kernels, so every member runs the arithmetic of its own
// single-grid mixed step.
#include "batch_kernel.cuh"

namespace dgpu_batch {

// Built solver combinations: 1D hydro {HLLC, exact} x 2D MHD {HLLD}. The 1D
// members run kMx1dTile-cell tiles whatever tile_1d says (the tiling is part
// of the mixed arithmetic), so both tile settings give the same kernel.
StepKernel pick_kernel_mx(int s1d, int /*tile*/) {
    return s1d == RS_EXACT ? k_batch_step<true, RS_EXACT, RS_HLLD, kMx1dTile>
                           : k_batch_step<true, RS_HLLC, RS_HLLD, kMx1dTile>;
}

namespace {

// The fused one-kernel step (step_mhd_fused.cuh) of every 2D MHD member of a
// mixed batch, in one launch: CTA b steps strip / segment b - fuse_first of
// the member whose CTA range holds b. The CTA that finishes a member's last
// CTA flips the member's current buffer unless the step failed or was not
// taken, as the persistent kernel does for its members' last phase.
__global__ void __launch_bounds__(kFuseNT, 2) k_batch_fused_mhd(const BatchInst* __restrict__ insts,
                                                              const int* __restrict__ members, int nm,
                                                              unsigned* ctr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& S = *reinterpret_cast<FusedMhdSmem<kFuseTJ, kFuseR>*>(smem_raw);
    if (*(const volatile unsigned*)&ctr[kCtrActive] == 0) return;
    int lo = 0, hi = nm - 1;  // the last member whose first CTA is <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (insts[members[mid]].fuse_first <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const int m = members[lo];
    const BatchInst& I = insts[m];
    const int local = (int)blockIdx.x - I.fuse_first;
    const int cur = ldv(&I.ctl->cur);
    StepArgs sa = I.sa;
    sa.slot_out = cur ^ 1;
    mhd2d_fused_body<RS_HLLD, kFuseTJ, kFuseR, kFuseNT>(I.G, I.FG, I.w[cur], I.w[cur ^ 1], I.B[cur], I.B[cur ^ 1],
                                                         I.ctl, sa, I.fuse_seg_rows, local % I.fuse_strips,
                                                         local / I.fuse_strips, local, I.fuse_ctas, S);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(ctr + kCtrDone + (size_t)kPhases * m + (kPhases - 1), 1u);
        if (prev + 1 == (unsigned)I.fuse_ctas) {
            StepCtl* c = I.ctl;
            if (!ldv(&c->err) && !ldv(&c->done)) *(volatile int*)&c->cur = cur ^ 1;
        }
    }
}

}  // namespace

size_t fused_mhd_smem() { return sizeof(FusedMhdSmem<kFuseTJ, kFuseR>); }

int launch_fused_mhd(const BatchInst* insts, const int* members, int nm, int ctas, unsigned* ctr, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_batch_fused_mhd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fused_mhd_smem()) != cudaSuccess)
            return 1;
        attr = true;
    }
    k_batch_fused_mhd<<<ctas, kFuseNT, fused_mhd_smem(), st>>>(insts, members, nm, ctr);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace dgpu_batch
