// 1D sweep launchers (hydro and MHD, every solver).
#include "launchers.h"
#include "step_hydro.cuh"

namespace dgpu {

// Tiles of TS = NT - 2 cells on NT threads: the half states (TS + 2 cells)
// and the faces (TS + 1) of a tile fit one round of the CTA's threads, where
// tiles of 128 cells on 128 threads ran each of those phases in two rounds,
// the second holding one or two items. Hydro: 254 cells on 256 threads; MHD
// (eight fields in static shared memory, at most 48 KB): 126 on 128.
template <bool MHD>
struct Tile1D {
    static constexpr int NT = MHD ? 128 : 256, TS = NT - 2;
};

template <bool MHD, int S>
static int go(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    const int np = G.n[0] + 2 * G.g;
    constexpr int TS = Tile1D<MHD>::TS, NT = Tile1D<MHD>::NT;
    k_step1d<MHD, S, TS, NT><<<(np + TS - 1) / TS, NT, 0, st>>>(G, win, wout, ctl, sa);
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
