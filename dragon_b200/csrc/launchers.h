// Host-side launchers of the step kernels, one translation unit per kernel
// family so the library builds in parallel. Each returns 0 on a clean launch.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "grid.cuh"

namespace dgpu {

struct MhdScratch;
struct MhdScratchF;
struct Hydro3DScratch;
struct Mhd3DScratch;

int launch_step1d(bool mhd, int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                  const StepArgs& sa, cudaStream_t st);
// Mixed FP32/FP64 1D sweep, hydro or MHD (step1d_mixed.cu).
int launch_step1d_mixed(bool mhd, int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                        const StepArgs& sa, cudaStream_t st);
// The fused 2D hydro steps load each tile with one TMA copy through `map`, a
// tensor map of the input buffer with the box step2d_tile_box gives (columns,
// rows, fields) for the FP64 (mixed = 0) or the mixed kernel.
constexpr int kMx2dTI = 16, kMx2dTJ = 32;
int step2d_tile_box(int mixed, int box[3]);
int launch_step2d_hydro(int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa,
                        const CUtensorMap* map, cudaStream_t st);
int launch_step2d_hydro_mixed(int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                              const StepArgs& sa, const CUtensorMap* map, cudaStream_t st);
int launch_step2d_mhd(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                      double* Bout, const MhdScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st);
int launch_step2d_mhd_mixed(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                            double* Bout, const MhdScratchF& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st);
// One Strang-split sweep (Godunov::sweep along every line of an axis), dt = factor * t1.
int launch_sweep(int solver, int axis, const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa,
                 double factor, cudaStream_t st);
int launch_init_body_fields(const Geo& G, const Geo& FG, double* w, const double* B, cudaStream_t s);
int launch_step3d_hydro(int solver, const Geo& G, const double* w, double* wout, const Hydro3DScratch& S,
                        StepCtl* ctl, const StepArgs& sa, cudaStream_t st);
// Mixed FP32/FP64 3D hydro step (step3d_mixed.cu): FP32 intermediates in S's planes.
int launch_step3d_hydro_mixed(int solver, const Geo& G, const double* w, double* wout, const Hydro3DScratch& S,
                              StepCtl* ctl, const StepArgs& sa, cudaStream_t st);
// Mixed FP32/FP64 3D MHD step (step3d_mhd_mixed.cu): FP32 half states and fluxes in S's planes.
int launch_step3d_mhd_mixed(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                            double* Bout, const Mhd3DScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st);
int launch_step3d_mhd(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                      double* Bout, const Mhd3DScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st);

}  // namespace dgpu
