// The mixed FP32/FP64 batched step: k_batch_step (batch_kernel.cuh) over the
// mixed tile bodies (step1d_mixed.cuh, step_mhd_mixed.cuh). Compiled with FMA
// contraction and fast single-precision division / square root, like the
// single-grid mixed kernels, so every member runs the arithmetic of its own
// single-grid mixed step.
#include "batch_kernel.cuh"

namespace dgpu_batch {

// Built solver combinations: 1D hydro {HLLC, exact} x 2D MHD {HLLD}. The 1D
// members run kMx1dTile-cell tiles whatever tile_1d says (the tiling is part
// of the mixed arithmetic), so both tile settings give the same kernel.
StepKernel pick_kernel_mx(int s1d, int /*tile*/) {
    return s1d == RS_EXACT ? k_batch_step<true, RS_EXACT, RS_HLLD, kMx1dTile>
                           : k_batch_step<true, RS_HLLC, RS_HLLD, kMx1dTile>;
}

}  // namespace dgpu_batch
