// Tile loads of the 2D state through the Tensor Memory Accelerator.
//
// A CTA's tile with its halo (all five hydro field planes) is one
// cp.async.bulk.tensor copy from this GPU's own memory into shared memory,
// issued by one thread and completed on an mbarrier the whole CTA waits on.
// The tensor map (encoded on the host, stage_tmap in runtime.cu) describes a
// state buffer as a 3D tensor: padded columns (innermost), padded rows, field
// planes. Boxes start on an even padded column (16-byte aligned for FP64),
// so a tile whose first column is odd loads one extra column and is indexed
// from an offset of one. Coordinates past the padded array read zeros.
// No cluster multicast is used: every copy reads this GPU's memory into the
// issuing CTA's shared memory.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "grid.cuh"

namespace dgpu {

constexpr long long kTmaWaitPolls = 1LL << 24;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// True once phase `parity` of the barrier completed; gives up after
// kTmaWaitPolls polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (long long k = 0; k < kTmaWaitPolls; k++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One 3D tile copy global -> shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Loads the five field planes of padded rows [row0, row0 + rows) and padded
// columns [col0, col0 + cols) (cols even, col0 even) into dst[5][rows][cols]
// (FP64), on the CTA's mbarrier *bar (initialised here, phase 0). Every thread
// of the CTA calls it; returns false (after recording ST_TILE_LOAD) when the
// copy did not complete within the wait limit.
__device__ __forceinline__ bool load_state_tile(double* dst, const CUtensorMap* map, int col0, int row0, unsigned bytes,
                                                uint64_t* bar, StepCtl* ctl) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, bytes);
        tma_load_3d(dst, map, col0, row0, 0, bar);
    }
    __syncthreads();
    const bool ok = mbar_wait(bar, 0);
    if (!ok) {
        record_error(ctl, ST_TILE_LOAD, 0);
        mbar_wait(bar, 0);  // give a late copy one more wait before the CTA may leave
    }
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

}  // namespace dgpu
