// FP64 fused 2D CTU hydro launchers (every hydro solver).
#include "launchers.h"
#include "step_hydro.cuh"

namespace dgpu {

constexpr int k2dTI = 8, k2dTJ = 32, k2dNT = 256;

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
    box[0] = k2dTJ + 6;
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
