// Single-grid mixed FP32/FP64 2D MHD step: the fused one-kernel step of
// step_mhd_fused.cuh (the batched step runs the seven phase bodies of
// step_mhd_mixed.cuh as work items instead). Compiled with FMA contraction
// and fast single-precision division / square root.
#include <algorithm>

#include "launchers.h"
#include "step_mhd_fused.cuh"

namespace dgpu {

namespace {

// One fused launch: a strip of columns per blockIdx.x, a segment of rows per
// blockIdx.y. Segments are sized so the CTAs fill the device's resident
// slots about once (each segment costs one ring-filling iteration extra).
template <int SOLVER>
int launch_fused(const Geo& G, const Geo& FG, const double* w, double* wout, const double* B, double* Bout,
                 StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    auto kern = k_mhd2d_fused_mixed<SOLVER, kFuseTJ, kFuseR, kFuseNT>;
    const size_t smem = sizeof(FusedMhdSmem<kFuseTJ, kFuseR>);
    static int slots = 0;
    if (slots == 0) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
        int dev = 0, sms = 0, occ = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kFuseNT, smem) != cudaSuccess || occ < 1)
            return 1;
        slots = occ * sms;
    }
    const int nx = G.n[0], ny = G.n[1];
    const int strips = (ny + kFuseTJ - 1) / kFuseTJ;
    const int segs_wanted = std::max(1, slots / strips);
    int seg = (nx + segs_wanted - 1) / segs_wanted;
    seg = std::max(4 * kFuseR, (seg + kFuseR - 1) / kFuseR * kFuseR);
    const dim3 grid(strips, (nx + seg - 1) / seg);
    kern<<<grid, kFuseNT, smem, st>>>(G, FG, w, wout, B, Bout, ctl, sa, seg);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

int launch_step2d_mhd_mixed(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                            double* Bout, const MhdScratchF&, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return launch_fused<RS_HLL>(G, FG, w, wout, B, Bout, ctl, sa, st);
        case RS_HLLE: return launch_fused<RS_HLLE>(G, FG, w, wout, B, Bout, ctl, sa, st);
        default: return launch_fused<RS_HLLD>(G, FG, w, wout, B, Bout, ctl, sa, st);
    }
}

}  // namespace dgpu
