// 1D sweep launchers (hydro and MHD, every solver).
#include "launchers.h"
#include "step_hydro.cuh"

namespace dgpu {

constexpr int k1dTS = 128;

template <bool MHD, int S>
static int go(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    const int np = G.n[0] + 2 * G.g;
    k_step1d<MHD, S, k1dTS><<<(np + k1dTS - 1) / k1dTS, k1dTS, 0, st>>>(G, win, wout, ctl, sa);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int launch_step1d(bool mhd, int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                  const StepArgs& sa, cudaStream_t st) {
    if (mhd) {
        switch (solver) {
            case RS_HLL: return go<true, RS_HLL>(G, win, wout, ctl, sa, st);
            case RS_HLLE: return go<true, RS_HLLE>(G, win, wout, ctl, sa, st);
            default: return go<true, RS_HLLD>(G, win, wout, ctl, sa, st);
        }
    }
    switch (solver) {
        case RS_HLLC: return go<false, RS_HLLC>(G, win, wout, ctl, sa, st);
        case RS_HLL: return go<false, RS_HLL>(G, win, wout, ctl, sa, st);
        case RS_HLLE: return go<false, RS_HLLE>(G, win, wout, ctl, sa, st);
        case RS_ROE: return go<false, RS_ROE>(G, win, wout, ctl, sa, st);
        default: return go<false, RS_EXACT>(G, win, wout, ctl, sa, st);
    }
}

}  // namespace dgpu
