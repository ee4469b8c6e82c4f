// CFL time step over a caller-owned device state without any allocation.
//
// Some callers cannot allocate device memory once their run has started: a
// host application that hands every byte of GPU memory to its own pool at
// start-up and forbids allocations afterwards, or a time-stepping loop where
// the implicit device-wide synchronisation of cudaMalloc/cudaFree would stall
// other streams. This entry point serves them: the caller passes the state
// (already on the device) and receives the time step; the only working memory
// is a fixed array compiled into this library.
//
// The working memory is `g_cfl_scratch` below: kCflNoallocMaxParts partial
// maxima plus two result words (~128 KB). Every GPU that loads this library
// keeps one copy of it until the process exits. All calls on a device share
// that copy, and it keeps whatever the previous call left in it, so each call
// rewrites every slot it reads before reading it. Calls whose work overlaps on
// the GPU (for example issued on two different streams without ordering)
// race on the array and may return each other's result; callers must
// serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/dragon_gpu.h"
#include "grid.cuh"

using namespace dgpu;

void dragon_gpu_set_error_message(const char* msg);  // runtime.cu

namespace {

constexpr int kCflNoallocMaxParts = 16384;
constexpr int kResultSlot = kCflNoallocMaxParts;  // [dt, max speed]

// Fixed device working memory: one partial maximum per row (2D), plane (3D)
// or chunk of 1024 cells (1D), then the two result words.
static __device__ __align__(256) double g_cfl_scratch[kCflNoallocMaxParts + 2];

// Device address of g_cfl_scratch per device, resolved once per device with
// that device current. The array's name in host code is only a stand-in for
// the symbol, never a usable device pointer.
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int fail_na(int code, const std::string& m) {
    dragon_gpu_set_error_message(m.c_str());
    return code;
}

int scratch_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail_na(DRAGON_GPU_ECUDA, "cfl_time_noalloc: no usable current CUDA device");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
        if (e != cudaSuccess || !p)
            return fail_na(DRAGON_GPU_ECUDA, std::string("cfl_time_noalloc: cudaGetSymbolAddress failed: ") +
                                                 cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return 0;
}

// One CTA per part: the maximum CFL signal speed over its share of the box
// [-1, n+1)^dim (interior plus one ghost layer, CFL.cpp:88-137), written to
// scratch[part]. Same per-cell speeds and NaN-skipping max as the handle path.
template <bool MHD>
__global__ void k_cfl_parts_noalloc(Geo G, const double* __restrict__ w, int cfl, double dx, double dy, double dz,
                                    double* __restrict__ scratch) {
    __shared__ double red[32];
    const int part = blockIdx.x;
    double m = 0.0;
    if (G.dim == 1) {
        const int lo = part * 1024 - 1, hi = min(lo + 1024, G.n[0] + 1);
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x)
            m = speed_max(m, cfl_speed_1d<MHD>(load_prim<MHD>(w, G.plane, gidx1(G, i))));
    } else if (G.dim == 2) {
        const int i = part - 1;
        for (int j = -1 + (int)threadIdx.x; j < G.n[1] + 1; j += blockDim.x)
            m = speed_max(m, cfl_speed<MHD>(load_prim<MHD>(w, G.plane, gidx2(G, i, j)), cfl, dx, dy, 0.0));
    } else {
        const int i = part - 1;
        const int ey = G.n[1] + 2, ez = G.n[2] + 2;
        for (int t = threadIdx.x; t < ey * ez; t += blockDim.x) {
            const int j = t / ez - 1, k = t % ez - 1;
            m = speed_max(m, cfl_speed<MHD>(load_prim<MHD>(w, G.plane, gidx3(G, i, j, k)), cfl, dx, dy, dz));
        }
    }
    m = block_max(m, red);
    if (threadIdx.x == 0) scratch[part] = m;
}

// Reduces the parts and writes [dt, max speed] into the result slots.
__global__ void k_cfl_finish_noalloc(int nparts, int dim, double cfl_coeff, double dx, double* __restrict__ scratch) {
    __shared__ double red[32];
    double m = 0.0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) m = speed_max(m, scratch[p]);
    m = block_max(m, red);
    if (threadIdx.x == 0) {
        scratch[kResultSlot + 1] = m;
        scratch[kResultSlot] = (m > 0) ? ((dim == 1) ? cfl_coeff * dx / m : cfl_coeff / m) : 0.0;
    }
}

}  // namespace

extern "C" int dragon_gpu_cfl_time_noalloc(int dim, int nx, int ny, int nz, int ghosts, int mhd, const double* d_prim,
                                           long long plane_stride, long long pitch, double dx, double dy, double dz,
                                           int cfl, double cfl_coeff, void* stream, double* dt_out) {
    if (!d_prim || !dt_out || dim < 1 || dim > 3 || nx < 1 || (dim >= 2 && ny < 1) || (dim == 3 && nz < 1) ||
        ghosts < 1)
        return fail_na(DRAGON_GPU_EINVAL, "cfl_time_noalloc: invalid arguments");
    const int n[3] = {nx, dim >= 2 ? ny : 1, dim == 3 ? nz : 1};
    long long nparts = (dim == 1) ? ((long long)nx + 2 + 1023) / 1024 : (long long)nx + 2;
    if (nparts > kCflNoallocMaxParts)
        return fail_na(DRAGON_GPU_EINVAL,
                       "cfl_time_noalloc: grid too large for the fixed working memory (at most " +
                           std::to_string(kCflNoallocMaxParts - 2) + " cells along x for 2D/3D grids, " +
                           std::to_string((long long)kCflNoallocMaxParts * 1024 - 2) + " cells for 1D grids)");
    Geo G;
    G.dim = dim;
    G.g = ghosts;
    for (int a = 0; a < 3; a++) {
        G.n[a] = n[a];
        G.ext[a] = a < dim ? n[a] + 2 * ghosts : 1;
    }
    if (dim == 1) {
        G.pitch = 1;
        G.pitch2 = 1;
    } else {
        G.pitch = pitch;
        G.pitch2 = (dim == 3) ? (long long)G.ext[1] * pitch : pitch;
    }
    G.plane = plane_stride;
    if (dim >= 2 && pitch < G.ext[dim - 1]) return fail_na(DRAGON_GPU_EINVAL, "cfl_time_noalloc: pitch too small");
    if (plane_stride < (long long)G.ext[0] * G.pitch2)
        return fail_na(DRAGON_GPU_EINVAL, "cfl_time_noalloc: plane stride too small");

    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mhd) k_cfl_parts_noalloc<true><<<(int)nparts, 256, 0, s>>>(G, d_prim, cfl, dx, dy, dz, scratch);
    else k_cfl_parts_noalloc<false><<<(int)nparts, 256, 0, s>>>(G, d_prim, cfl, dx, dy, dz, scratch);
    k_cfl_finish_noalloc<<<1, 1024, 0, s>>>((int)nparts, dim, cfl_coeff, dx, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_na(DRAGON_GPU_ECUDA, std::string("cfl_time_noalloc: launch: ") + cudaGetErrorString(e));
    double res[2] = {0.0, 0.0};
    e = cudaMemcpyAsync(res, scratch + kResultSlot, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_na(DRAGON_GPU_ECUDA, std::string("cfl_time_noalloc: ") + cudaGetErrorString(e));
    if (!(res[1] > 0)) return fail_na(DRAGON_GPU_ECFL, "CFL timestep failed: max signal speed is zero");
    *dt_out = res[0];
    return 0;
}
