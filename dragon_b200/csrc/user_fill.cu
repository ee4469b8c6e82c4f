// User ghost-fill elements compiled for the device.
//
// The reference lets a problem subclass GhostFill and fill ghost cells in its
// own apply(Grid&) (GhostFill.hpp:16-30; the Jet inflow of
// Examples/CollidingFlows/Jets/Jets.hpp:12-39 and Jet.cpp is the shipped
// example). Here the user writes that fill as a CUDA device function over one
// ghost cell; dragon_gpu_user_fill_create compiles it with NVRTC into a kernel
// that visits the ghost cells of the element's faces, and the grid launches
// that kernel at the element's place in the boundary list, inside the device
// advance loop: no state crosses the host link and the host does not wait.
//
// The user function:
//
//     __device__ void NAME(const dragon_fill_ctx& c, int i, int j, int k);
//
// is called once per ghost cell (i, j, k) (interior coordinates, ghosts
// negative or >= n) of every face in the binding's fill mask, with c.axis and
// c.side naming the face. For one face, the ghost layers of a transverse point
// are visited by one thread from the face outward (layer 1, 2, ... g), so a
// fill may read the layer it wrote just before; different transverse points
// and the two faces of an axis run in parallel, and the axes run one after
// another (x, then y, then z). A fill may read any cell and face B and writes
// only the ghost cell it is called for (and face B of that cell).
//
// NVRTC (libnvrtc.so.12) and the driver's module API are loaded at run time;
// without NVRTC, creating a fill fails with its reason and nothing else
// changes.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dragon_gpu.h"
#include "handle.h"

using namespace dgpu;

void dragon_gpu_set_error_message(const char* msg);  // runtime.cu

struct dragon_user_fill {
    std::string function;
    std::string log;
    std::vector<char> cubin;
    std::mutex mu;
    std::map<CUcontext, std::pair<CUmodule, CUfunction>> loaded;  // per context
};

namespace {

int fail_uf(int code, const std::string& m) {
    dragon_gpu_set_error_message(m.c_str());
    return code;
}

// ---- NVRTC, loaded on first use -------------------------------------------
struct NvrtcApi {
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*log_size)(nvrtcProgram, size_t*);
    nvrtcResult (*log)(nvrtcProgram, char*);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
    nvrtcResult (*cubin)(nvrtcProgram, char*);
    nvrtcResult (*destroy)(nvrtcProgram*);
    const char* (*err)(nvrtcResult);
    bool ok = false;
    std::string why;
};

const NvrtcApi& nvrtc() {
    static NvrtcApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        std::vector<std::string> names = {"libnvrtc.so.12", "libnvrtc.so"};
        if (const char* home = std::getenv("CUDA_HOME")) names.push_back(std::string(home) + "/lib64/libnvrtc.so.12");
        names.push_back("/usr/local/cuda/lib64/libnvrtc.so.12");
        void* so = nullptr;
        for (const auto& n : names)
            if ((so = dlopen(n.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
        if (!so) {
            api.why = "NVRTC (libnvrtc.so.12) could not be loaded";
            return;
        }
        auto sym = [&](const char* n) { return dlsym(so, n); };
        api.create = reinterpret_cast<decltype(api.create)>(sym("nvrtcCreateProgram"));
        api.compile = reinterpret_cast<decltype(api.compile)>(sym("nvrtcCompileProgram"));
        api.log_size = reinterpret_cast<decltype(api.log_size)>(sym("nvrtcGetProgramLogSize"));
        api.log = reinterpret_cast<decltype(api.log)>(sym("nvrtcGetProgramLog"));
        api.cubin_size = reinterpret_cast<decltype(api.cubin_size)>(sym("nvrtcGetCUBINSize"));
        api.cubin = reinterpret_cast<decltype(api.cubin)>(sym("nvrtcGetCUBIN"));
        api.destroy = reinterpret_cast<decltype(api.destroy)>(sym("nvrtcDestroyProgram"));
        api.err = reinterpret_cast<decltype(api.err)>(sym("nvrtcGetErrorString"));
        api.ok = api.create && api.compile && api.log_size && api.log && api.cubin_size && api.cubin && api.destroy &&
                 api.err;
        if (!api.ok) api.why = "NVRTC is missing an entry point";
    });
    return api;
}

// ---- the driver's module API, through the runtime's entry-point query ------
struct DriverApi {
    CUresult (*load)(CUmodule*, const void*) = nullptr;
    CUresult (*get)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                       void**, void**) = nullptr;
    CUresult (*ctx)(CUcontext*) = nullptr;
    bool ok = false;
};

const DriverApi& driver() {
    static DriverApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char* n) -> void* {
            void* p = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint(n, &p, cudaEnableDefault, &q) != cudaSuccess ||
                q != cudaDriverEntryPointSuccess)
                return nullptr;
            return p;
        };
        api.load = reinterpret_cast<decltype(api.load)>(get("cuModuleLoadData"));
        api.get = reinterpret_cast<decltype(api.get)>(get("cuModuleGetFunction"));
        api.launch = reinterpret_cast<decltype(api.launch)>(get("cuLaunchKernel"));
        api.ctx = reinterpret_cast<decltype(api.ctx)>(get("cuCtxGetCurrent"));
        api.ok = api.load && api.get && api.launch && api.ctx;
    });
    return api;
}

// ---- the program NVRTC compiles ---------------------------------------------
// The context a fill sees: the state arrays and geometry of the grid, the
// binding's parameters, and the face being filled. Its layout is the host's
// FillCtx below, member for member.
const char* kPrelude = R"(
#define DRAGON_RHO 0
#define DRAGON_P 1
#define DRAGON_VX 2
#define DRAGON_VY 3
#define DRAGON_VZ 4
#define DRAGON_BX 5
#define DRAGON_BY 6
#define DRAGON_BZ 7
struct dragon_fill_ctx {
    double* w;                            /* primitive planes: w[f * plane + cell(i, j, k)] */
    double* B;                            /* face B planes (MHD, 2D / 3D), else null */
    long long plane, pitch, pitch2;       /* cells: elements per plane, per row, per x layer */
    long long fplane, fpitch, fpitch2;    /* faces: the same on the face grid (n + 1 per axis) */
    const double* params;                 /* the binding's parameters */
    double d[3];                          /* dx, dy, dz */
    int dim, n[3], g, nf, nparams;
    int axis, side;                       /* the face being filled: axis 0..2, side 0 low / 1 high */
    int off[3];                           /* global index of cell (0, 0, 0): a slab's place in a distributed grid */
    __device__ long long cell(int i, int j, int k) const {
        return dim == 1 ? (long long)(i + g)
             : dim == 2 ? (long long)(i + g) * pitch + (j + g)
                        : (long long)(i + g) * pitch2 + (long long)(j + g) * pitch + (k + g);
    }
    __device__ long long face(int i, int j, int k) const {
        return dim == 2 ? (long long)(i + g) * fpitch + (j + g)
                        : (long long)(i + g) * fpitch2 + (long long)(j + g) * fpitch + (k + g);
    }
    __device__ double get(int f, int i, int j, int k) const { return w[f * plane + cell(i, j, k)]; }
    __device__ void set(int f, int i, int j, int k, double v) const { w[f * plane + cell(i, j, k)] = v; }
    __device__ double getB(int c, int i, int j, int k) const { return B[c * fplane + face(i, j, k)]; }
    __device__ void setB(int c, int i, int j, int k, double v) const { B[c * fplane + face(i, j, k)] = v; }
};
#line 1 "user_fill"
)";

// The kernel around the user's function: one thread per (side, transverse
// point) of one axis, the ghost layers from the face outward.
std::string wrapper(const std::string& fn) {
    return R"(
extern "C" __global__ void __launch_bounds__(256) dragon_fill_kernel(dragon_fill_ctx c, const int* err, const int* done,
                                                                    int axis, int sides, int corners) {
    if ((*(const volatile int*)err) | (*(const volatile int*)done)) return;
    int ta[2] = {-1, -1}, t0[2] = {0, 0}, tn[2] = {1, 1}, nt = 0;
    for (int b = 0; b < c.dim; b++) {
        if (b == axis) continue;
        ta[nt] = b;
        t0[nt] = corners ? -c.g : 0;
        tn[nt] = corners ? c.n[b] + c.g : c.n[b];
        nt++;
    }
    const long long s0 = tn[0] - t0[0], s1 = tn[1] - t0[1], per = s0 * s1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * per;
         t += (long long)gridDim.x * blockDim.x) {
        const int side = (int)(t / per);
        if (!((sides >> side) & 1)) continue;
        const long long r = t - side * per;
        int q[3] = {0, 0, 0};
        if (nt > 0) q[ta[0]] = t0[0] + (int)(r / s1);
        if (nt > 1) q[ta[1]] = t0[1] + (int)(r % s1);
        dragon_fill_ctx cc = c;
        cc.axis = axis;
        cc.side = side;
        for (int gl = 1; gl <= c.g; gl++) {
            q[axis] = side == 0 ? -gl : c.n[axis] - 1 + gl;
            )" + fn + R"((cc, q[0], q[1], q[2]);
        }
    }
}
)";
}

// Host mirror of dragon_fill_ctx.
struct FillCtx {
    double* w;
    double* B;
    long long plane, pitch, pitch2;
    long long fplane, fpitch, fpitch2;
    const double* params;
    double d[3];
    int dim, n[3], g, nf, nparams;
    int axis, side;
    int off[3];
};

bool valid_identifier(const char* s) {
    if (!s || !*s || !(std::isalpha((unsigned char)s[0]) || s[0] == '_')) return false;
    for (const char* p = s; *p; p++)
        if (!(std::isalnum((unsigned char)*p) || *p == '_')) return false;
    return true;
}

// The kernel of a fill in the current context, loaded on first use there.
int fill_function(dragon_user_fill* f, CUfunction* out) {
    const DriverApi& D = driver();
    if (!D.ok) return fail_uf(DRAGON_GPU_ECUDA, "the driver's module API is not available");
    CUcontext ctx = nullptr;
    if (D.ctx(&ctx) != CUDA_SUCCESS || !ctx) {
        cudaFree(nullptr);  // makes the device's primary context current
        if (D.ctx(&ctx) != CUDA_SUCCESS || !ctx) return fail_uf(DRAGON_GPU_ECUDA, "no CUDA context for the user fill");
    }
    std::lock_guard<std::mutex> lk(f->mu);
    auto it = f->loaded.find(ctx);
    if (it != f->loaded.end()) {
        *out = it->second.second;
        return 0;
    }
    CUmodule m = nullptr;
    CUfunction fn = nullptr;
    if (D.load(&m, f->cubin.data()) != CUDA_SUCCESS) return fail_uf(DRAGON_GPU_ECUDA, "loading the user fill module failed");
    if (D.get(&fn, m, "dragon_fill_kernel") != CUDA_SUCCESS)
        return fail_uf(DRAGON_GPU_ECUDA, "the user fill module has no fill kernel");
    f->loaded[ctx] = {m, fn};
    *out = fn;
    return 0;
}

}  // namespace

int dragon_gpu_user_fill_create(const char* source, const char* function, dragon_user_fill** out) {
    if (!source || !out || !valid_identifier(function))
        return fail_uf(DRAGON_GPU_EINVAL, "user fill: source, a function name (an identifier) and an output are required");
    *out = nullptr;
    const NvrtcApi& N = nvrtc();
    if (!N.ok) return fail_uf(DRAGON_GPU_ECUDA, N.why);
    const std::string prog_src = std::string(kPrelude) + source + "\n" + wrapper(function);
    nvrtcProgram prog;
    nvrtcResult r = N.create(&prog, prog_src.c_str(), "dragon_user_fill.cu", 0, nullptr, nullptr);
    if (r != NVRTC_SUCCESS) return fail_uf(DRAGON_GPU_ECUDA, std::string("nvrtcCreateProgram: ") + N.err(r));
    // the same arithmetic rules as the library's FP64 kernels: no contraction,
    // IEEE division and square root
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false", "--prec-div=true",
                          "--prec-sqrt=true", "-lineinfo"};
    r = N.compile(prog, 6, opts);
    auto* f = new dragon_user_fill();
    f->function = function;
    size_t ls = 0;
    if (N.log_size(prog, &ls) == NVRTC_SUCCESS && ls > 1) {
        f->log.resize(ls);
        N.log(prog, &f->log[0]);
        f->log.resize(std::strlen(f->log.c_str()));
    }
    if (r != NVRTC_SUCCESS) {
        const std::string msg = "user fill did not compile:\n" + f->log;
        N.destroy(&prog);
        delete f;
        return fail_uf(DRAGON_GPU_EINVAL, msg);
    }
    size_t cs = 0;
    if (N.cubin_size(prog, &cs) != NVRTC_SUCCESS || cs == 0) {
        N.destroy(&prog);
        delete f;
        return fail_uf(DRAGON_GPU_ECUDA, "nvrtcGetCUBINSize failed");
    }
    f->cubin.resize(cs);
    N.cubin(prog, f->cubin.data());
    N.destroy(&prog);
    *out = f;
    return 0;
}

int dragon_gpu_user_fill_destroy(dragon_user_fill* f) {
    // Modules stay loaded until their context ends: a grid created later in
    // the same context may still be launching them from its stream.
    delete f;
    return 0;
}

const char* dragon_gpu_user_fill_log(const dragon_user_fill* f) { return f ? f->log.c_str() : ""; }

int dragon_gpu_set_user_fill(dragon_grid* h, int entry, dragon_user_fill* f, int fill_faces, int corners,
                             const double* params, int nparams) {
    if (!h) return fail_uf(DRAGON_GPU_EINVAL, "null handle");
    if (h->adv.pending) return fail_uf(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!f || nparams < 0 || (nparams > 0 && !params))
        return fail_uf(DRAGON_GPU_EINVAL, "user fill: a compiled fill and its parameters are required");
    if (entry < 0 || entry >= h->caller_entries)
        return fail_uf(DRAGON_GPU_EINVAL, "user fill: entry index outside the boundary list");
    const int dev = h->nbc - h->caller_entries + entry;
    if (std::find(h->user_entries.begin(), h->user_entries.end(), dev) == h->user_entries.end())
        return fail_uf(DRAGON_GPU_EINVAL, "user fill: the boundary entry is not of the user type");
    UserFillBinding& b = h->ufill[dev];
    if (b.dparams) {
        cudaStreamSynchronize(h->stream);
        cudaFree(b.dparams);
        b.dparams = nullptr;
    }
    b.fill = f;
    b.fill_faces = fill_faces & ((1 << (2 * h->dim)) - 1);
    b.corners = corners ? 1 : 0;
    b.nparams = nparams;
    if (nparams > 0) {
        if (cudaMalloc(&b.dparams, sizeof(double) * nparams) != cudaSuccess)
            return fail_uf(DRAGON_GPU_ECUDA, "user fill: parameter allocation failed");
        if (cudaMemcpy(b.dparams, params, sizeof(double) * nparams, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail_uf(DRAGON_GPU_ECUDA, "user fill: parameter upload failed");
    }
    return 0;
}

namespace dgpu_rt {

void clear_user_fills(dragon_grid* h) {
    bool any = false;
    for (auto& b : h->ufill) any |= b.dparams != nullptr;
    if (any) cudaStreamSynchronize(h->stream);
    for (auto& b : h->ufill)
        if (b.dparams) cudaFree(b.dparams);
    h->ufill.clear();
}

int launch_user_fill(dragon_grid* h, int c, int entry, double* w_buf) {
    const UserFillBinding& b = h->ufill[entry];
    if (!b.fill) return fail_uf(DRAGON_GPU_EINVAL, "a user boundary entry has no fill bound (dragon_gpu_set_user_fill)");
    CUfunction fn = nullptr;
    int rc = fill_function(b.fill, &fn);
    if (rc) return rc;
    FillCtx x{};
    x.w = w_buf ? w_buf : h->w[c];
    x.B = (h->mhd && h->dim >= 2) ? h->B[c] : nullptr;
    x.plane = h->cg.plane;
    x.pitch = h->cg.pitch;
    x.pitch2 = h->cg.pitch2;
    x.fplane = h->fg.plane;
    x.fpitch = h->fg.pitch;
    x.fpitch2 = h->fg.pitch2;
    x.params = b.dparams;
    for (int a = 0; a < 3; a++) {
        x.d[a] = h->d[a];
        x.n[a] = h->n[a];
    }
    x.dim = h->dim;
    x.g = h->g;
    x.nf = h->nf;
    x.nparams = b.nparams;
    for (int a = 0; a < 3; a++) x.off[a] = h->origin[a];
    const int* err = &h->ctl->err;
    const int* done = &h->ctl->done;
    int corners = b.corners;
    for (int axis = 0; axis < h->dim; axis++) {
        int sides = (b.fill_faces >> (2 * axis)) & 3;
        if (!sides) continue;
        long long per = 1;
        for (int t = 0; t < h->dim; t++)
            if (t != axis) per *= corners ? h->n[t] + 2 * h->g : h->n[t];
        const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((2 * per + 255) / 256, 148 * 8));
        void* args[] = {&x, &err, &done, &axis, &sides, &corners};
        if (driver().launch(fn, blocks, 1, 1, 256, 1, 1, 0, (CUstream)h->stream, args, nullptr) != CUDA_SUCCESS)
            return fail_uf(DRAGON_GPU_ECUDA, "user fill launch failed");
        h->launches++;
    }
    return 0;
}

}  // namespace dgpu_rt
