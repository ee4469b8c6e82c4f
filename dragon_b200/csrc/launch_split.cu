// Strang-split sweep launchers (2D / 3D, every hydro solver, every axis).
#include "launchers.h"
#include "step_split.cuh"

namespace dgpu {

template <int S, int DIM>
static int go(int axis, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, double f,
              cudaStream_t st) {
    if (axis == 0) return launch_sweep_t<S, DIM, 0>(G, win, wout, ctl, sa, f, st);
    if constexpr (DIM == 2) return launch_sweep_t<S, DIM, 1>(G, win, wout, ctl, sa, f, st);
    else {
        if (axis == 1) return launch_sweep_t<S, DIM, 1>(G, win, wout, ctl, sa, f, st);
        return launch_sweep_t<S, DIM, 2>(G, win, wout, ctl, sa, f, st);
    }
}

template <int S>
static int go_dim(int axis, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, double f,
                  cudaStream_t st) {
    return G.dim == 2 ? go<S, 2>(axis, G, win, wout, ctl, sa, f, st) : go<S, 3>(axis, G, win, wout, ctl, sa, f, st);
}

int launch_sweep(int solver, int axis, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa,
                 double factor, cudaStream_t st) {
    switch (solver) {
        case RS_HLLC: return go_dim<RS_HLLC>(axis, G, win, wout, ctl, sa, factor, st);
        case RS_HLL: return go_dim<RS_HLL>(axis, G, win, wout, ctl, sa, factor, st);
        case RS_HLLE: return go_dim<RS_HLLE>(axis, G, win, wout, ctl, sa, factor, st);
        case RS_ROE: return go_dim<RS_ROE>(axis, G, win, wout, ctl, sa, factor, st);
        default: return go_dim<RS_EXACT>(axis, G, win, wout, ctl, sa, factor, st);
    }
}

}  // namespace dgpu
