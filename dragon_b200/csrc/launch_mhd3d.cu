// 3D MHD CTU + CT launchers (HLLD, HLL, HLLE).
#include "launchers.h"
#include "step_mhd3d.cuh"

namespace dgpu {

int launch_step3d_mhd(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                      double* Bout, const Mhd3DScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return launch_step3d_mhd_t<RS_HLL>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        case RS_HLLE: return launch_step3d_mhd_t<RS_HLLE>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        default: return launch_step3d_mhd_t<RS_HLLD>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
    }
}

}  // namespace dgpu
