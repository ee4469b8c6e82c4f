// Single-grid mixed FP32/FP64 1D sweeps: step1d_tile_mx (hydro) and
// step1d_tile_mx_mhd (MHD) of step1d_mixed.cuh, one tile per CTA. Compiled with FMA contraction and
// fast single-precision division / square root.
#include "launchers.h"
#include "step1d_mixed.cuh"

namespace dgpu {

namespace {

template <int SOLVER, int TS, int NT>
__global__ void __launch_bounds__(NT)
k_step1d_mx(Geo G, const double* __restrict__ win, double* __restrict__ wout, StepCtl* ctl, StepArgs sa) {
    step1d_tile_mx<SOLVER, TS>(G, win, wout, ctl, sa, blockIdx.x);
}

// The 1D MHD sweep, mixed precision: 126-cell tiles on 128 threads (eight
// FP32 fields in static shared memory), as the FP64 MHD sweep.
template <int SOLVER, int TS, int NT>
__global__ void __launch_bounds__(NT)
k_step1d_mx_mhd(Geo G, const double* __restrict__ win, double* __restrict__ wout, StepCtl* ctl, StepArgs sa) {
    step1d_tile_mx_mhd<SOLVER, TS>(G, win, wout, ctl, sa, blockIdx.x);
}

template <int S>
int go_mhd(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    constexpr int TS = 126, NT = 128;
    const int np = G.n[0] + 2 * G.g;
    k_step1d_mx_mhd<S, TS, NT><<<(np + TS - 1) / TS, NT, 0, st>>>(G, win, wout, ctl, sa);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

template <int S>
int go(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    const int np = G.n[0] + 2 * G.g;
    k_step1d_mx<S, kMx1dTile, kMx1dThreads><<<(np + kMx1dTile - 1) / kMx1dTile, kMx1dThreads, 0, st>>>(G, win, wout,
                                                                                                    ctl, sa);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

int launch_step1d_mixed(bool mhd, int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                        const StepArgs& sa, cudaStream_t st) {
    if (mhd) {
        switch (solver) {
            case RS_HLL: return go_mhd<RS_HLL>(G, win, wout, ctl, sa, st);
            case RS_HLLE: return go_mhd<RS_HLLE>(G, win, wout, ctl, sa, st);
            default: return go_mhd<RS_HLLD>(G, win, wout, ctl, sa, st);
        }
    }
    switch (solver) {
        case RS_HLLC: return go<RS_HLLC>(G, win, wout, ctl, sa, st);
        case RS_HLL: return go<RS_HLL>(G, win, wout, ctl, sa, st);
        case RS_HLLE: return go<RS_HLLE>(G, win, wout, ctl, sa, st);
        case RS_ROE: return go<RS_ROE>(G, win, wout, ctl, sa, st);
        default: return go<RS_EXACT>(G, win, wout, ctl, sa, st);
    }
}

}  // namespace dgpu
