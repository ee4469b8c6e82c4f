// Output and restart from device buffers: DRAGONHOARD::writeToFile and
// DRAGONHOARD::loadFromFile (DRAGONHOARD/HDF5Output.cpp:103-528,
// HDF5Restart.cpp:61-377) behind the C ABI of include/dragon_gpu.h.
//
// A snapshot is one or two launches on the grid's stream: k_hoard_pack turns
// the SoA state planes (last index fastest) into the file's datasets
// (x fastest, HDF5Output.cpp:308) through 32 x 32 shared-memory tiles, so the
// loads and the stores are both coalesced, computing E and the momenta on the
// way; the face-B planes go through the same kernel. The packed buffer is
// downloaded on a copy stream into pinned memory while later steps run, and a
// host thread lays out the HDF5 file and deflates its chunks on every core
// (hoard_file.cu). Two staging slots let one file be written while the next
// snapshot is taken.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <thread>

#include <sys/resource.h>
#include <sys/syscall.h>
#include <unistd.h>
#include <vector>

#include "fluid.cuh"
#include "handle.h"
#include "hoard_file.h"

using namespace dgpu;

void dragon_gpu_set_error_message(const char* msg);  // runtime.cu

namespace {

int fail_h(int code, const std::string& m) {
    dragon_gpu_set_error_message(m.c_str());
    return code;
}

#define HK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) return fail_h(DRAGON_GPU_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// What one dataset holds, computed per cell from its primitive state.
enum PackKind { PK_FIELD = 0, PK_ENERGY = 1, PK_MOM = 2 };
constexpr int kMaxItems = 12;
struct PackItem {
    int kind;
    int arg;  // field (PK_FIELD) or momentum component (PK_MOM)
    int f32;  // stored as float
    long long off;  // byte offset of the dataset in the staging buffer
};
struct PackList {
    PackItem it[kMaxItems];
    int n;
};

// w[f] for a run-time f without indexing the register array dynamically.
template <int NF>
__device__ __forceinline__ double pick(const double (&w)[NF], int f) {
    double r = w[0];
#pragma unroll
    for (int q = 1; q < NF; q++)
        if (f == q) r = w[q];
    return r;
}

template <int NF, bool MHD>
__device__ __forceinline__ double pack_value(const double (&w)[NF], const PackItem& it) {
    if constexpr (NF >= 5) {
        if (it.kind == PK_MOM) return pick(w, 2 + it.arg) * w[0];  // ConservativeState(w): mom = v * rho
        if (it.kind == PK_ENERGY) {
            Prim<double> p;
            p.rho = w[0];
            p.p = w[1];
            p.vx = w[2];
            p.vy = w[3];
            p.vz = w[4];
            if constexpr (MHD && NF >= 8) {
                p.Bx = w[5];
                p.By = w[6];
                p.Bz = w[7];
            } else {
                p.Bx = p.By = p.Bz = 0;
            }
            return energy<MHD>(p);  // PrimitiveState::energy (FluidElement.cpp:53-59)
        }
    }
    return pick(w, it.arg);
}

__device__ __forceinline__ void store(char* dst, const PackItem& it, long long e, double v) {
    if (it.f32) reinterpret_cast<float*>(dst + it.off)[e] = (float)v;
    else reinterpret_cast<double*>(dst + it.off)[e] = v;
}

// 2D / 3D: the state is row-major with the last axis fastest (address
// (x+sh)*Pi + (m+sh)*Pm + (l+sh), m the middle axis of 3D), the file is x
// fastest (((l*NM + m)*NX + x). A 32 x 8 block loads a 32 (x) x 32 (l) tile
// along l, computes one dataset into shared memory at a time and stores it
// along x.
template <int NF, bool MHD>
__global__ void __launch_bounds__(256)
k_hoard_pack(const double* __restrict__ src, long long plane, long long Pi, long long Pm, int sh, int NX, int NM, int NL,
             PackList L, char* __restrict__ dst) {
    __shared__ double tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int l0 = blockIdx.x * 32, x0 = blockIdx.y * 32, m = blockIdx.z;
    double v[4][NF];
    bool in[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int x = x0 + ty + 8 * r, l = l0 + tx;
        in[r] = x < NX && l < NL;
        const long long a = (long long)(x + sh) * Pi + (long long)(m + sh) * Pm + (l + sh);
#pragma unroll
        for (int f = 0; f < NF; f++) v[r][f] = in[r] ? __ldg(src + f * plane + a) : 0.0;
    }
    for (int d = 0; d < L.n; d++) {
        const PackItem it = L.it[d];
#pragma unroll
        for (int r = 0; r < 4; r++) tile[ty + 8 * r][tx] = in[r] ? pack_value<NF, MHD>(v[r], it) : 0.0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int x = x0 + tx, l = l0 + ty + 8 * r;
            if (x < NX && l < NL) store(dst, it, ((long long)l * NM + m) * NX + x, tile[tx][ty + 8 * r]);
        }
        __syncthreads();
    }
}

// 1D: the state and the file are both x fastest.
template <int NF, bool MHD>
__global__ void __launch_bounds__(256)
k_hoard_pack1d(const double* __restrict__ src, long long plane, int sh, int NX, PackList L, char* __restrict__ dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= NX) return;
    double v[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) v[f] = __ldg(src + f * plane + x + sh);
    for (int d = 0; d < L.n; d++) store(dst, L.it[d], x, pack_value<NF, MHD>(v, L.it[d]));
}

// One dataset of a file: its key, shape (slowest first), element type and
// where it sits in the staging buffer.
struct PlanDs {
    std::string path;
    int rank;
    uint64_t dims[3];
    int type;
    size_t off, bytes;
    bool face;
    PackItem item;
};

struct Plan {
    std::vector<PlanDs> ds;
    std::vector<hoard::Attr> attrs;
    size_t total = 0;
    int ext[3] = {1, 1, 1};  // cells written per axis (x, y, z)
    int sh = 0;              // device index shift: g without ghosts, 0 with them
};

// What the file layout depends on: the grid's dimension, extents, ghost
// width (of the padded arrays), spacing and physics.
struct Shape {
    int dim;
    int n[3];
    int g;
    double d[3];
    bool mhd;
};

Shape shape_of(const dragon_grid* h) {
    return Shape{h->dim, {h->n[0], h->n[1], h->n[2]}, h->g, {h->d[0], h->d[1], h->d[2]}, h->mhd};
}

int make_plan(const Shape& h_, double t, int cycle, const dragon_hoard_opts& o, Plan* P) {
    const Shape* h = &h_;
    const int opt = o.write_option, red = o.redundant;
    // HDF5Output.cpp:21-30: which representations the option writes
    const bool prims = opt & 1;
    const bool consv = opt & 4;
    const bool redundants = red != 0;
    const bool write_e = (opt & 2) && (consv || redundants);
    if (!(prims || consv))
        return fail_h(DRAGON_GPU_EINVAL, "write option does not write a sufficient description of the fluid");
    if (red < 0 || red > 2) return fail_h(DRAGON_GPU_EINVAL, "redundant-values option must be 0, 1 or 2");
    if (o.compression > 9) return fail_h(DRAGON_GPU_EINVAL, "compression level must be at most 9 (deflate)");
    const int dim = h->dim;
    const int ng = o.ghosts ? h->g : 0;
    P->sh = h->g - ng;
    for (int a = 0; a < dim; a++) P->ext[a] = h->n[a] + 2 * ng;
    auto attr_i = [&](const char* k, int v) { P->attrs.push_back({k, hoard::kI32, v, 0.0}); };
    auto attr_d = [&](const char* k, double v) { P->attrs.push_back({k, hoard::kF64, 0, v}); };
    attr_i("format_version", 1);
    attr_i("write_option", opt);
    attr_i("dim", dim);
    attr_i("MHD", h->mhd ? 1 : 0);
    attr_i("ng", ng);
    const char* nk[3] = {"nx", "ny", "nz"};
    const char* dk[3] = {"dx", "dy", "dz"};
    for (int a = 0; a < dim; a++) attr_i(nk[a], h->n[a]);
    for (int a = 0; a < dim; a++) attr_d(dk[a], h->d[a]);
    attr_i("cycle", cycle);
    attr_d("time", t);

    auto add = [&](const std::string& path, bool face, int type, int kind, int arg) {
        PlanDs d{};
        d.path = path;
        d.rank = dim;
        for (int a = 0; a < dim; a++) d.dims[dim - 1 - a] = uint64_t(P->ext[a] + (face ? 1 : 0));
        d.type = type;
        uint64_t n = 1;
        for (int a = 0; a < dim; a++) n *= d.dims[a];
        d.bytes = n * (type == hoard::kF64 ? 8 : 4);
        d.off = P->total;
        P->total += (d.bytes + 255) / 256 * 256;
        d.face = face;
        d.item = PackItem{kind, arg, type == hoard::kF32 ? 1 : 0, (long long)d.off};
        P->ds.push_back(d);
    };
    const int F64 = hoard::kF64, F32 = hoard::kF32;
    add("/fluid/rho", false, F64, PK_FIELD, 0);
    if (prims) {
        add("/fluid/v/x", false, F64, PK_FIELD, 2);
        add("/fluid/v/y", false, F64, PK_FIELD, 3);
        add("/fluid/v/z", false, F64, PK_FIELD, 4);
        add("/fluid/p", false, F64, PK_FIELD, 1);
    }
    if (write_e) {
        add("/fluid/E", false, (consv || red == 2) ? F64 : F32, PK_ENERGY, 0);
        if (consv) {
            add("/fluid/momentum/x", false, F64, PK_MOM, 0);
            add("/fluid/momentum/y", false, F64, PK_MOM, 1);
            add("/fluid/momentum/z", false, F64, PK_MOM, 2);
        }
    }
    if (h->mhd) {
        if (dim == 1) {  // 1D: cell B, always double (HDF5Output.cpp:149-151)
            add("/fluid/B/x", false, F64, PK_FIELD, 5);
            add("/fluid/B/y", false, F64, PK_FIELD, 6);
            add("/fluid/B/z", false, F64, PK_FIELD, 7);
        } else {
            if (redundants) {
                const int bt = red == 2 ? F64 : F32;
                add("/fluid/B/x", false, bt, PK_FIELD, 5);
                add("/fluid/B/y", false, bt, PK_FIELD, 6);
                add("/fluid/B/z", false, bt, PK_FIELD, 7);
            }
            add("/fluid/Bf/x", true, F64, PK_FIELD, 0);
            add("/fluid/Bf/y", true, F64, PK_FIELD, 1);
            add("/fluid/Bf/z", true, F64, PK_FIELD, 2);
        }
    }
    return 0;
}

template <int NF, bool MHD>
int launch_pack(const dragon_grid* h, const Geo& G, const double* src, const PackList& L, int sh, const int* ext,
                int face, char* dst, cudaStream_t st) {
    const int NX = ext[0] + face;
    if (h->dim == 1) {
        k_hoard_pack1d<NF, MHD><<<(NX + 255) / 256, 256, 0, st>>>(src, G.plane, sh, NX, L, dst);
    } else {
        const int NM = h->dim == 3 ? ext[1] + face : 1;
        const int NL = ext[h->dim - 1] + face;
        const long long Pi = h->dim == 3 ? G.pitch2 : G.pitch;
        const long long Pm = h->dim == 3 ? G.pitch : 0;
        dim3 grid((NL + 31) / 32, (NX + 31) / 32, NM);
        k_hoard_pack<NF, MHD><<<grid, dim3(32, 8), 0, st>>>(src, G.plane, Pi, Pm, sh, NX, NM, NL, L, dst);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Enqueues the pack of the current state into dst on the grid's stream;
// returns the number of launches, or -1.
int enqueue_pack(dragon_grid* h, const Plan& P, char* dst) {
    PackList cells{}, faces{};
    for (const auto& d : P.ds) {
        PackList& L = d.face ? faces : cells;
        L.it[L.n++] = d.item;
    }
    const int c = h->cur;
    int launches = 0;
    int rc = 0;
    if (cells.n) {
        rc |= h->mhd ? launch_pack<8, true>(h, h->cg, h->w[c], cells, P.sh, P.ext, 0, dst, h->stream)
                     : launch_pack<5, false>(h, h->cg, h->w[c], cells, P.sh, P.ext, 0, dst, h->stream);
        launches++;
    }
    if (faces.n) {
        rc |= launch_pack<3, false>(h, h->fg, h->B[c], faces, P.sh, P.ext, 1, dst, h->stream);
        launches++;
    }
    return rc ? -1 : launches;
}

}  // namespace

// Per-grid snapshot state: two staging slots (device buffer, pinned host
// buffer, copy event, writer thread) and the copy stream.
struct HoardSlot {
    char* dbuf = nullptr;
    size_t dcap = 0;
    char* hbuf = nullptr;
    size_t hcap = 0;
    cudaEvent_t copied = nullptr;
    std::thread writer;
    int rc = 0;
    std::string err;
};
struct HoardState {
    HoardSlot slot[2];
    int next = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t packed = nullptr;
};

namespace {

int join_slot(HoardSlot& s, std::string* err) {
    if (s.writer.joinable()) s.writer.join();
    const int rc = s.rc;
    if (rc && err && err->empty()) *err = s.err;
    s.rc = 0;
    s.err.clear();
    return rc;
}

int ensure_state(dragon_grid* h) {
    if (h->hoard) return 0;
    auto* S = new HoardState();
    h->hoard = S;
    HK(cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking));
    HK(cudaEventCreateWithFlags(&S->packed, cudaEventDisableTiming));
    for (auto& s : S->slot) HK(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
    return 0;
}

// background: the caller keeps stepping while the file is written, so the
// writer and its deflate threads run at a lower scheduling priority than the
// thread that drives the steps.
int snapshot(dragon_grid* h, double t, int cycle, const char* path, const dragon_hoard_opts* opts, int* slot_used,
             bool background) {
    if (!h || !path) return fail_h(DRAGON_GPU_EINVAL, "null argument");
    if (h->adv.pending) return fail_h(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    dragon_hoard_opts o;
    if (opts) o = *opts;
    else dragon_gpu_hoard_default_opts(&o);
    Plan P;
    if (int rc = make_plan(shape_of(h), t, cycle, o, &P)) return rc;
    if (int rc = ensure_state(h)) return rc;
    HoardState* S = h->hoard;
    const int k = S->next;
    HoardSlot& s = S->slot[k];
    std::string prev;
    const int prc = join_slot(s, &prev);
    if (s.dcap < P.total) {
        if (s.dbuf) cudaFree(s.dbuf);
        s.dbuf = nullptr;
        s.dcap = 0;
        HK(cudaMalloc(&s.dbuf, P.total));
        s.dcap = P.total;
    }
    if (s.hcap < P.total) {
        if (s.hbuf) cudaFreeHost(s.hbuf);
        s.hbuf = nullptr;
        s.hcap = 0;
        HK(cudaHostAlloc(&s.hbuf, P.total, cudaHostAllocDefault));
        s.hcap = P.total;
    }
    const int nl = enqueue_pack(h, P, s.dbuf);
    if (nl < 0) return fail_h(DRAGON_GPU_ECUDA, std::string("pack launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    h->launches += nl;
    HK(cudaEventRecord(S->packed, h->stream));
    HK(cudaStreamWaitEvent(S->copy, S->packed, 0));
    HK(cudaMemcpyAsync(s.hbuf, s.dbuf, P.total, cudaMemcpyDeviceToHost, S->copy));
    HK(cudaEventRecord(s.copied, S->copy));
    int dev = 0;
    HK(cudaGetDevice(&dev));
    const std::string file(path);
    const int level = o.compression, threads = o.threads;
    HoardSlot* sp = &s;
    s.writer = std::thread([sp, P = std::move(P), file, level, threads, dev, background]() {
        // threads created by this one (the deflate pool) inherit its nice value
        if (background) setpriority(PRIO_PROCESS, id_t(syscall(SYS_gettid)), 10);
        cudaSetDevice(dev);
        const cudaError_t e = cudaEventSynchronize(sp->copied);
        if (e != cudaSuccess) {
            sp->rc = DRAGON_GPU_ECUDA;
            sp->err = std::string("snapshot download failed: ") + cudaGetErrorString(e);
            return;
        }
        std::vector<hoard::Dataset> ds;
        for (const auto& d : P.ds) {
            hoard::Dataset x;
            x.path = d.path;
            x.rank = d.rank;
            for (int a = 0; a < 3; a++) x.dims[a] = d.dims[a];
            x.type = d.type;
            x.data = sp->hbuf + d.off;
            ds.push_back(x);
        }
        std::string err;
        if (hoard::write_file(file, P.attrs, ds, level, threads, &err)) {
            sp->rc = DRAGON_GPU_EINVAL;
            sp->err = err;
        }
    });
    S->next ^= 1;
    if (slot_used) *slot_used = k;
    if (prc) return fail_h(prc, "an earlier snapshot failed: " + prev);
    return 0;
}

}  // namespace

namespace {

// The datasets of plan P from host arrays in the reference's layout (prim:
// the padded cells, nf values each; faceB: the padded faces, 3 values each),
// the same values k_hoard_pack computes, into out (P.total bytes).
void host_pack(const Shape& S, const Plan& P, const double* prim, const double* faceB, char* out) {
    const int nf = S.mhd ? 8 : 5, dim = S.dim, g = S.g;
    for (const auto& ds : P.ds) {
        const int fc = ds.face ? 1 : 0;
        int X[3] = {1, 1, 1};  // padded extents of the source array
        for (int a = 0; a < dim; a++) X[a] = S.n[a] + fc + 2 * g;
        const int NX = P.ext[0] + fc, NY = dim > 1 ? P.ext[1] + fc : 1, NZ = dim > 2 ? P.ext[2] + fc : 1;
        const PackItem& it = ds.item;
        long long e = 0;
        for (int z = 0; z < NZ; z++)
            for (int y = 0; y < NY; y++)
                for (int x = 0; x < NX; x++, e++) {
                    const size_t c = (size_t(x + P.sh) * X[1] + (dim > 1 ? y + P.sh : 0)) * X[2] + (dim > 2 ? z + P.sh : 0);
                    double v;
                    if (ds.face) {
                        v = faceB[c * 3 + it.arg];
                    } else {
                        const double* w = prim + c * nf;
                        if (it.kind == PK_MOM) {
                            v = w[2 + it.arg] * w[0];
                        } else if (it.kind == PK_ENERGY) {
                            Prim<double> q{w[0], w[1], w[2], w[3], w[4], 0, 0, 0};
                            if (S.mhd) {
                                q.Bx = w[5];
                                q.By = w[6];
                                q.Bz = w[7];
                            }
                            v = S.mhd ? energy<true>(q) : energy<false>(q);
                        } else {
                            v = w[it.arg];
                        }
                    }
                    if (it.f32) reinterpret_cast<float*>(out + it.off)[e] = (float)v;
                    else reinterpret_cast<double*>(out + it.off)[e] = v;
                }
    }
}

// Restart of host arrays in the reference's layout (W: the padded cells, nf
// values each; FB: the padded faces, 3 values each, MHD 2D / 3D): checks the
// file against the shape and overwrites the cells and faces of the file's
// range as HDF5Restart.cpp:61-377 does; the others keep their values.
int load_into(const Shape& S, const char* path, double* W, double* FB, double* t, int* cycle, double* d_out) {
    const int nf = S.mhd ? 8 : 5;
    hoard::File F;
    std::string err;
    if (!F.open(path, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    auto geti = [&](const char* k, int* v) {
        double x;
        if (!F.attr(k, &x, &err)) return false;
        *v = int(x);
        return true;
    };
    auto getd = [&](const char* k, double* v) { return F.attr(k, v, &err); };
    int fmt, dim, mhd, ng, wopt, cyc;
    if (!geti("format_version", &fmt)) return fail_h(DRAGON_GPU_EINVAL, err);
    if (fmt > 1) return fail_h(DRAGON_GPU_EINVAL, "Please update to the latest version of DRAGON to read this file");
    if (!geti("dim", &dim)) return fail_h(DRAGON_GPU_EINVAL, err);
    if (dim != S.dim)
        return fail_h(DRAGON_GPU_EINVAL, "Expected " + std::to_string(S.dim) + (S.dim == 1 ? " dimension" : " dimensions") +
                                             " but got " + std::to_string(dim));
    if (!geti("MHD", &mhd)) return fail_h(DRAGON_GPU_EINVAL, err);
    if (mhd && !S.mhd) return fail_h(DRAGON_GPU_EINVAL, "File was saved using MHD. Please enable MHD in Config.h");
    const char* nk[3] = {"nx", "ny", "nz"};
    const char* dk[3] = {"dx", "dy", "dz"};
    int n[3] = {1, 1, 1};
    double d[3] = {0, 0, 0};
    for (int a = 0; a < dim; a++)
        if (!geti(nk[a], &n[a])) return fail_h(DRAGON_GPU_EINVAL, err);
    for (int a = 0; a < dim; a++)
        if (n[a] != S.n[a]) return fail_h(DRAGON_GPU_EINVAL, "File size does not match the grid size");
    if (!geti("ng", &ng)) return fail_h(DRAGON_GPU_EINVAL, err);
    ng = std::min(ng, S.g);
    for (int a = 0; a < dim; a++)
        if (!getd(dk[a], &d[a])) return fail_h(DRAGON_GPU_EINVAL, err);
    double tt;
    if (!getd("time", &tt) || !geti("cycle", &cyc) || !geti("write_option", &wopt)) return fail_h(DRAGON_GPU_EINVAL, err);

    // the file's range: cells i in [-ng, n + ng) per axis, flattened x fastest
    int E[3] = {1, 1, 1};
    for (int a = 0; a < dim; a++) E[a] = n[a] + 2 * ng;
    const size_t cells = size_t(E[0]) * E[1] * E[2];
    const size_t faces = size_t(E[0] + 1) * (dim > 1 ? E[1] + 1 : 1) * (dim > 2 ? E[2] + 1 : 1);
    auto need = [&](const char* key, size_t count, std::vector<double>* v, bool zero_if_missing) {
        if (!F.has(key)) {
            if (zero_if_missing) {
                v->assign(count, 0.0);
                return true;
            }
            err = std::string("no dataset ") + key;
            return false;
        }
        if (!F.read(key, v, &err)) return false;
        if (v->size() < count) {
            err = std::string(key) + " is smaller than the grid range it loads";
            return false;
        }
        return true;
    };
    std::vector<double> rho, p, vx, vy, vz, Eg, px, py, pz, bx, by, bz, fx, fy, fz;
    if (!need("/fluid/rho", cells, &rho, false)) return fail_h(DRAGON_GPU_EINVAL, err);
    const bool cellB = S.mhd && mhd;
    if (cellB) {
        // HDF5Restart.cpp: 1D requires cell B; 2D / 3D read zeros where it is absent
        const bool zmiss = dim > 1;
        if (!need("/fluid/B/x", cells, &bx, zmiss) || !need("/fluid/B/y", cells, &by, zmiss) ||
            !need("/fluid/B/z", cells, &bz, zmiss))
            return fail_h(DRAGON_GPU_EINVAL, err);
        if (dim > 1 && (!need("/fluid/Bf/x", faces, &fx, true) || !need("/fluid/Bf/y", faces, &fy, true) ||
                        !need("/fluid/Bf/z", faces, &fz, true)))
            return fail_h(DRAGON_GPU_EINVAL, err);
    }
    const bool from_prim = wopt & 1;
    if (from_prim) {
        if (!need("/fluid/p", cells, &p, false) || !need("/fluid/v/x", cells, &vx, false) ||
            !need("/fluid/v/y", cells, &vy, false) || !need("/fluid/v/z", cells, &vz, false))
            return fail_h(DRAGON_GPU_EINVAL, err);
    } else {
        if (!need("/fluid/E", cells, &Eg, false) || !need("/fluid/momentum/x", cells, &px, false) ||
            !need("/fluid/momentum/y", cells, &py, false) || !need("/fluid/momentum/z", cells, &pz, false))
            return fail_h(DRAGON_GPU_EINVAL, err);
    }

    const bool has_faces = S.mhd && dim > 1;
    const int g = S.g;
    int X[3] = {1, 1, 1}, XF[3] = {1, 1, 1};
    for (int a = 0; a < dim; a++) {
        X[a] = S.n[a] + 2 * g;
        XF[a] = S.n[a] + 1 + 2 * g;
    }
    auto cell_at = [&](int i, int j, int k) {
        return ((size_t(i + g) * X[1] + (dim > 1 ? j + g : 0)) * X[2] + (dim > 2 ? k + g : 0)) * nf;
    };
    const int jlo = dim > 1 ? -ng : 0, jhi = dim > 1 ? n[1] + ng : 1;
    const int klo = dim > 2 ? -ng : 0, khi = dim > 2 ? n[2] + ng : 1;
    for (int k = klo; k < khi; k++)
        for (int j = jlo; j < jhi; j++)
            for (int i = -ng; i < n[0] + ng; i++) {
                const size_t f = (size_t(k - klo) * E[1] + (j - jlo)) * E[0] + (i + ng);
                double* w = W + cell_at(i, j, k);
                w[0] = rho[f];
                if (S.mhd) {
                    w[5] = cellB ? bx[f] : 0.0;
                    w[6] = cellB ? by[f] : 0.0;
                    w[7] = cellB ? bz[f] : 0.0;
                }
                if (from_prim) {
                    w[1] = p[f];
                    w[2] = vx[f];
                    w[3] = vy[f];
                    w[4] = vz[f];
                } else {
                    Cons<double> U;
                    U.rho = w[0];
                    U.mx = px[f];
                    U.my = py[f];
                    U.mz = pz[f];
                    U.E = Eg[f];
                    U.Bx = S.mhd ? w[5] : 0.0;
                    U.By = S.mhd ? w[6] : 0.0;
                    U.Bz = S.mhd ? w[7] : 0.0;
                    const Prim<double> q = S.mhd ? to_prim<true>(U) : to_prim<false>(U);
                    w[1] = q.p;
                    w[2] = q.vx;
                    w[3] = q.vy;
                    w[4] = q.vz;
                }
            }
    if (has_faces) {
        const int kfhi = dim > 2 ? n[2] + ng : 0;
        for (int k = klo; k <= kfhi; k++)
            for (int j = -ng; j <= n[1] + ng; j++)
                for (int i = -ng; i <= n[0] + ng; i++) {
                    const size_t f = (size_t(k - klo) * (E[1] + 1) + (j + ng)) * (E[0] + 1) + (i + ng);
                    const size_t at = ((size_t(i + g) * XF[1] + (j + g)) * XF[2] + (dim > 2 ? k + g : 0)) * 3;
                    FB[at + 0] = cellB ? fx[f] : 0.0;
                    FB[at + 1] = cellB ? fy[f] : 0.0;
                    FB[at + 2] = cellB ? fz[f] : 0.0;
                }
    }
    for (int a = 0; a < 3; a++) d_out[a] = a < dim ? d[a] : 0.0;
    *t = tt;
    *cycle = cyc;
    return 0;
}

}  // namespace

namespace dgpu_rt {
void hoard_release(dragon_grid* h) {
    HoardState* S = h->hoard;
    if (!S) return;
    for (auto& s : S->slot) {
        join_slot(s, nullptr);
        if (s.dbuf) cudaFree(s.dbuf);
        if (s.hbuf) cudaFreeHost(s.hbuf);
        if (s.copied) cudaEventDestroy(s.copied);
    }
    if (S->packed) cudaEventDestroy(S->packed);
    if (S->copy) cudaStreamDestroy(S->copy);
    delete S;
    h->hoard = nullptr;
}
}  // namespace dgpu_rt

extern "C" {

void dragon_gpu_hoard_default_opts(dragon_hoard_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->write_option = 3;  // HDF5_WRITE_PRIMITIVE_AND_ENERGY
    o->redundant = 1;     // HDF5_WRITE_FLOAT
    o->compression = 4;   // HDF5_COMPRESSION_LEVEL
    o->ghosts = 0;
    o->threads = 0;
}

int dragon_hoard_write_host(const char* path, int dim, int mhd, const int* n3, int ghosts, const double* d3, double t,
                            int cycle, const double* prim, const double* faceB, const dragon_hoard_opts* opts) {
    if (!path || !n3 || !d3 || !prim || dim < 1 || dim > 3 || ghosts < 0 || (mhd && dim > 1 && !faceB))
        return fail_h(DRAGON_GPU_EINVAL, "invalid argument");
    Shape S{dim, {n3[0], dim > 1 ? n3[1] : 1, dim > 2 ? n3[2] : 1}, ghosts,
            {d3[0], dim > 1 ? d3[1] : 0.0, dim > 2 ? d3[2] : 0.0}, mhd != 0};
    for (int a = 0; a < dim; a++)
        if (S.n[a] < 1) return fail_h(DRAGON_GPU_EINVAL, "invalid extents");
    dragon_hoard_opts o;
    if (opts) o = *opts;
    else dragon_gpu_hoard_default_opts(&o);
    Plan P;
    if (int rc = make_plan(S, t, cycle, o, &P)) return rc;
    std::vector<char> buf(P.total);
    host_pack(S, P, prim, faceB, buf.data());
    std::vector<hoard::Dataset> ds;
    for (const auto& d : P.ds) {
        hoard::Dataset x;
        x.path = d.path;
        x.rank = d.rank;
        for (int a = 0; a < 3; a++) x.dims[a] = d.dims[a];
        x.type = d.type;
        x.data = buf.data() + d.off;
        ds.push_back(x);
    }
    std::string err;
    if (hoard::write_file(path, P.attrs, ds, o.compression, o.threads, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    return 0;
}

int dragon_gpu_hoard_write_async(dragon_grid* h, double t, int cycle, const char* path, const dragon_hoard_opts* o) {
    return snapshot(h, t, cycle, path, o, nullptr, true);
}

int dragon_gpu_hoard_write(dragon_grid* h, double t, int cycle, const char* path, const dragon_hoard_opts* o) {
    int k = 0;
    if (int rc = snapshot(h, t, cycle, path, o, &k, false)) return rc;
    std::string err;
    const int rc = join_slot(h->hoard->slot[k], &err);
    return rc ? fail_h(rc, err) : 0;
}

int dragon_gpu_hoard_wait(dragon_grid* h) {
    if (!h) return fail_h(DRAGON_GPU_EINVAL, "null grid");
    if (!h->hoard) return 0;
    std::string err;
    int rc = 0;
    for (int i = 0; i < 2; i++) {
        // oldest first
        const int r = join_slot(h->hoard->slot[(h->hoard->next + i) & 1], &err);
        if (!rc) rc = r;
    }
    return rc ? fail_h(rc, err) : 0;
}

int dragon_gpu_hoard_load(dragon_grid* h, const char* path, double* t, int* cycle) {
    if (!h || !path || !t || !cycle) return fail_h(DRAGON_GPU_EINVAL, "null argument");
    if (h->adv.pending) return fail_h(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    // the grid's own files still being written are complete first (a restart
    // may name one of them); their status stays for dragon_gpu_hoard_wait
    if (h->hoard)
        for (auto& s : h->hoard->slot)
            if (s.writer.joinable()) s.writer.join();
    // current state (reference order, dense padded): cells outside the file's
    // range keep their values
    std::vector<double> W(dragon_gpu_prim_count(h)), FB(dragon_gpu_faceB_count(h));
    if (int rc = dragon_gpu_download_prim(h, W.data())) return rc;
    if (!FB.empty())
        if (int rc = dragon_gpu_download_faceB(h, FB.data())) return rc;
    double d[3];
    if (int rc = load_into(shape_of(h), path, W.data(), FB.empty() ? nullptr : FB.data(), t, cycle, d)) return rc;
    for (int a = 0; a < h->dim; a++) h->d[a] = d[a];
    if (int rc = dragon_gpu_upload_prim(h, W.data())) return rc;
    if (!FB.empty())
        if (int rc = dragon_gpu_upload_faceB(h, FB.data())) return rc;
    return 0;
}

int dragon_hoard_load_host(const char* path, int dim, int mhd, const int* n3, int ghosts, double* prim, double* faceB,
                           double* t, int* cycle, double* d3) {
    if (!path || !n3 || !prim || !t || !cycle || !d3 || dim < 1 || dim > 3 || ghosts < 0 || (mhd && dim > 1 && !faceB))
        return fail_h(DRAGON_GPU_EINVAL, "invalid argument");
    Shape S{dim, {n3[0], dim > 1 ? n3[1] : 1, dim > 2 ? n3[2] : 1}, ghosts, {0, 0, 0}, mhd != 0};
    for (int a = 0; a < dim; a++)
        if (S.n[a] < 1) return fail_h(DRAGON_GPU_EINVAL, "invalid extents");
    return load_into(S, path, prim, faceB, t, cycle, d3);
}

int dragon_h5_write(const char* file, const dragon_h5_attr* attrs, int nattrs, const dragon_h5_dataset* dsets,
                    int ndsets, int level, int threads) {
    if (!file || nattrs < 0 || ndsets < 0 || (nattrs && !attrs) || (ndsets && !dsets))
        return fail_h(DRAGON_GPU_EINVAL, "invalid argument");
    std::vector<hoard::Attr> A;
    for (int i = 0; i < nattrs; i++) {
        if (!attrs[i].name || (attrs[i].type != DRAGON_H5_I32 && attrs[i].type != DRAGON_H5_F64))
            return fail_h(DRAGON_GPU_EINVAL, "attributes are named int32 or double scalars");
        A.push_back({attrs[i].name, attrs[i].type == DRAGON_H5_I32 ? hoard::kI32 : hoard::kF64, attrs[i].ivalue,
                     attrs[i].dvalue});
    }
    std::vector<hoard::Dataset> D;
    for (int i = 0; i < ndsets; i++) {
        const auto& s = dsets[i];
        if (!s.path || !s.data || s.rank < 1 || s.rank > 3 || (s.type != DRAGON_H5_F64 && s.type != DRAGON_H5_F32))
            return fail_h(DRAGON_GPU_EINVAL, "datasets are named float or double arrays of rank 1 to 3");
        hoard::Dataset x;
        x.path = s.path;
        x.rank = s.rank;
        for (int a = 0; a < s.rank; a++) {
            if (s.dims[a] <= 0) return fail_h(DRAGON_GPU_EINVAL, "dataset dimensions must be positive");
            x.dims[a] = uint64_t(s.dims[a]);
        }
        x.type = s.type == DRAGON_H5_F64 ? hoard::kF64 : hoard::kF32;
        x.data = s.data;
        D.push_back(x);
    }
    std::string err;
    if (hoard::write_file(file, A, D, level, threads, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    return 0;
}

int dragon_h5_read_attr(const char* file, const char* name, double* value) {
    if (!file || !name || !value) return fail_h(DRAGON_GPU_EINVAL, "null argument");
    hoard::File F;
    std::string err;
    if (!F.open(file, &err) || !F.attr(name, value, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    return 0;
}

int dragon_h5_dataset_shape(const char* file, const char* path, int* rank, long long* dims3) {
    if (!file || !path || !rank || !dims3) return fail_h(DRAGON_GPU_EINVAL, "null argument");
    hoard::File F;
    std::string err;
    std::vector<uint64_t> dims;
    if (!F.open(file, &err) || !F.shape(path, &dims, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    if (dims.size() > 3) return fail_h(DRAGON_GPU_EINVAL, "dataset rank above 3");
    *rank = int(dims.size());
    for (int a = 0; a < 3; a++) dims3[a] = a < int(dims.size()) ? (long long)dims[a] : 0;
    return 0;
}

int dragon_h5_read(const char* file, const char* path, double* out, long long capacity) {
    if (!file || !path || !out) return fail_h(DRAGON_GPU_EINVAL, "null argument");
    hoard::File F;
    std::string err;
    std::vector<double> v;
    if (!F.open(file, &err) || !F.read(path, &v, &err)) return fail_h(DRAGON_GPU_EINVAL, err);
    if ((long long)v.size() > capacity) return fail_h(DRAGON_GPU_EINVAL, "output buffer too small");
    std::copy(v.begin(), v.end(), out);
    return 0;
}

}  // extern "C"
