// Device intermediates of the multi-kernel steps (allocated per grid handle).
#pragma once

namespace dgpu {

// 2D MHD step, all on the face geometry (n+1 per axis, same ghosts), which
// covers every cell, face and edge index the step uses.
struct MhdScratch {
    double* hs;   // 4 x 8 planes: xL, xR, yL, yR half states (primitive)
    double* fx;   // 8 planes: predictor, then final x-face fluxes
    double* fy;   // 8 planes: predictor, then final y-face fluxes
    double* er;   // 3 planes: body E of w
    double* e0;   // 3 planes: predictor corner E, then final corner E
    double* eh;   // 3 planes: body E of the half-step cells
    long long plane;
    static constexpr int kPlanes = 32 + 8 + 8 + 3 + 3 + 3;
};
constexpr int kMhd2DKernels = 7;

// The same intermediates in FP32 (mixed-precision 2D MHD step); they live in
// the same allocation, which is sized for the FP64 form.
struct MhdScratchF {
    float* hs;
    float* fx;
    float* fy;
    float* er;
    float* e0;
    float* eh;
    long long plane;
};

// 3D hydro step, on the cell geometry.
struct Hydro3DScratch {
    double* hs;    // 6 x 5 planes: xL, xR, yL, yR, zL, zR
    double* pf;    // 3 x 5 planes: predictor F_X, F_Y, F_Z; then final fluxes
    double* cf;    // 6 x 5 planes: F_Xz, F_Yz, F_Xy, F_Zy, F_Yx, F_Zx
    long long plane;
    static constexpr int kPlanes = 30 + 15 + 30;
};
constexpr int kHydro3DKernels = 5;

// 3D MHD step, on the face geometry.
struct Mhd3DScratch {
    double* hs;   // 6 x 8 planes: xL, xR, yL, yR, zL, zR half states (primitive)
    double* fx;   // 8 planes each: predictor, then final fluxes
    double* fy;
    double* fz;
    double* er;   // 3 planes: body E of w
    double* e0;   // 3 planes: predictor edge E, then final edge E
    double* eh;   // 3 planes: body E of the half-step cells
    long long plane;
    static constexpr int kPlanes = 48 + 24 + 9;
};
constexpr int kMhd3DKernels = 7;

}  // namespace dgpu
