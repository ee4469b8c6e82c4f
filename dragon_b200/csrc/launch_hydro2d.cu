// FP64 fused 2D CTU hydro launchers (every hydro solver).
#include "launchers.h"
#include "step_hydro.cuh"

namespace dgpu {

// Tiles of 19 x 22 cells, 512 threads, one CTA per SM (126 registers): each
// phase's items (half states 504, predictor faces 963, corrections 918, final
// faces 877, updates 418) fill their last round of threads nearly full, where
// 8 x 32 tiles on 256 threads left rounds of 40 to 124 items in four phases,
// and the two-cell halo is recomputed on fewer cells per output cell.
// Measured on the 1024^2 shear layer: 0.486 ms per step against 0.534 ms for
// 8 x 32 (23 x 18: 0.488, 16 x 26: 0.509, 16 x 32 on 512 threads: 0.549);
// results bit-identical.
constexpr int k2dTI = 19, k2dTJ = 22, k2dNT = 512;

template <int S>
static int go(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, const CUtensorMap* map,
              cudaStream_t st) {
    auto kern = k_step2d_hydro<S, k2dTI, k2dTJ, k2dNT>;
    const size_t smem = sizeof(Smem2DH<k2dTI, k2dTJ>);
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
        attr_set = true;
    }
    dim3 grid((G.n[1] + k2dTJ - 1) / k2dTJ, (G.n[0] + k2dTI - 1) / k2dTI);
    kern<<<grid, k2dNT, smem, st>>>(G, win, wout, ctl, sa, *map);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int step2d_tile_box(int mixed, int box[3]) {
    box[0] = (mixed ? kMx2dTJ : k2dTJ) + 6;
    box[1] = (mixed ? kMx2dTI : k2dTI) + 4;
    box[2] = 5;
    return 0;
}

int launch_step2d_hydro(int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa,
                        const CUtensorMap* map, cudaStream_t st) {
    switch (solver) {
        case RS_HLLC: return go<RS_HLLC>(G, win, wout, ctl, sa, map, st);
        case RS_HLL: return go<RS_HLL>(G, win, wout, ctl, sa, map, st);
        case RS_HLLE: return go<RS_HLLE>(G, win, wout, ctl, sa, map, st);
        case RS_ROE: return go<RS_ROE>(G, win, wout, ctl, sa, map, st);
        default: return go<RS_EXACT>(G, win, wout, ctl, sa, map, st);
    }
}

}  // namespace dgpu
