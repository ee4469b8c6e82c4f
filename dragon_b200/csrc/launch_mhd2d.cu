// 2D MHD CTU + CT launchers (HLLD, HLL, HLLE) and the face->cell B initialiser.
#include "launchers.h"
#include "step_mhd.cuh"

namespace dgpu {

int launch_step2d_mhd(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                      double* Bout, const MhdScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return launch_step2d_mhd_t<RS_HLL>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        case RS_HLLE: return launch_step2d_mhd_t<RS_HLLE>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        default: return launch_step2d_mhd_t<RS_HLLD>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
    }
}

int launch_init_body_fields(const Geo& G, const Geo& FG, double* w, const double* B, cudaStream_t s) {
    return launch_init_body_fields_t(G, FG, w, B, s);
}

}  // namespace dgpu
