// 3D CTU hydro launchers (every hydro solver).
#include "launchers.h"
#include "step3d.cuh"

namespace dgpu {

int launch_step3d_hydro(int solver, const Geo& G, const double* w, double* wout, const Hydro3DScratch& S,
                        StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLLC: return launch_step3d_hydro_t<RS_HLLC>(G, w, wout, S, ctl, sa, st);
        case RS_HLL: return launch_step3d_hydro_t<RS_HLL>(G, w, wout, S, ctl, sa, st);
        case RS_HLLE: return launch_step3d_hydro_t<RS_HLLE>(G, w, wout, S, ctl, sa, st);
        case RS_ROE: return launch_step3d_hydro_t<RS_ROE>(G, w, wout, S, ctl, sa, st);
        default: return launch_step3d_hydro_t<RS_EXACT>(G, w, wout, S, ctl, sa, st,
                                                         sa.exact_guess == GUESS_LEARNED && sa.mlp != nullptr);
    }
}

}  // namespace dgpu
