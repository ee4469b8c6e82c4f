// Single-grid mixed FP32/FP64 2D MHD step: the seven phase bodies of
// step_mhd_mixed.cuh, one 32 x 8 tile per CTA. Compiled with FMA contraction
// and fast single-precision division / square root.
#include "launchers.h"
#include "step_mhd_mixed.cuh"

namespace dgpu {

namespace {

__global__ void k_mx_halfstates(Mhd2DMixedArgs A) { mx_halfstates(A, launch_tile()); }
template <int SOLVER, bool FINAL>
__global__ void __launch_bounds__(256, 3) k_mx_fluxes(Mhd2DMixedArgs A) { mx_fluxes<SOLVER, FINAL>(A, launch_tile()); }
template <bool FINAL>
__global__ void k_mx_edges(Mhd2DMixedArgs A) { mx_edges<FINAL>(A, launch_tile()); }
__global__ void k_mx_half(Mhd2DMixedArgs A) { mx_half(A, launch_tile()); }
__global__ void k_mx_update(Mhd2DMixedArgs A) { mx_update(A, launch_tile()); }

template <int SOLVER>
int launch_mx(const Geo& G, const Geo& FG, const double* w, double* wout, const double* B, double* Bout,
              const MhdScratchF& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    Mhd2DMixedArgs A{G, FG, w, wout, B, Bout, S, ctl, sa};
    const dim3 blk(kTileJ, kTileI);
    auto grid_for = [&](int ni, int nj) { return dim3((nj + kTileJ - 1) / kTileJ, (ni + kTileI - 1) / kTileI); };
    const int nx = G.n[0], ny = G.n[1];
    if (launch_mhd2d_copy_frame(G, FG, w, wout, B, Bout, st)) return 1;
    k_mx_halfstates<<<grid_for(nx + 4, ny + 4), blk, 0, st>>>(A);
    k_mx_fluxes<SOLVER, false><<<grid_for(nx + 4, ny + 4), blk, 0, st>>>(A);
    k_mx_edges<false><<<grid_for(nx + 3, ny + 3), blk, 0, st>>>(A);
    k_mx_half<<<grid_for(nx + 2, ny + 2), blk, 0, st>>>(A);
    k_mx_fluxes<SOLVER, true><<<grid_for(nx + 2, ny + 2), blk, 0, st>>>(A);
    k_mx_edges<true><<<grid_for(nx + 1, ny + 1), blk, 0, st>>>(A);
    k_mx_update<<<grid_for(nx, ny), blk, 0, st>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

int launch_step2d_mhd_mixed(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                            double* Bout, const MhdScratchF& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return launch_mx<RS_HLL>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        case RS_HLLE: return launch_mx<RS_HLLE>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        default: return launch_mx<RS_HLLD>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
    }
}

}  // namespace dgpu
