// Host runtime behind include/dragon_gpu.h: grid handles, host<->device
// transfers in the reference's AoS order, the boundary program, and the
// device-resident advance loop (Grid::advance_unsplit, CFL.cpp:188-213).
//
// The advance loop enqueues batches of (prologue, step) kernel pairs without
// host synchronisation. The prologue does the previous step's bookkeeping
// (dt -= t1), the ghost fill and the CFL dt; the step kernel reads t1 from the
// control block. A failed step raises the device error word, after which every
// later kernel of the batch returns at once, so the failed step's input buffer
// is still intact; the host then halves dt and retries exactly like the
// reference's catch block (CFL.cpp:194-209).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dragon_gpu.h"
#include "../../include/dragon_learned.h"
#include "boundary.cuh"
#include "handle.h"
#include "launchers.h"
#include "mlp.cuh"
#include "recon.cuh"
#include "riemann.cuh"
#include "scratch.h"

using namespace dgpu;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return fail(DRAGON_GPU_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
    } while (0)

constexpr int kBatch = 64;

long long round_up(long long a, long long b) { return (a + b - 1) / b * b; }

Geo make_geo(int dim, const int* n, int g) {
    Geo G;
    G.dim = dim;
    G.g = g;
    for (int a = 0; a < 3; a++) {
        G.n[a] = a < dim ? n[a] : 1;
        G.ext[a] = a < dim ? n[a] + 2 * g : 1;
    }
    if (dim == 1) {
        G.pitch = 1;
        G.pitch2 = 1;
        G.plane = round_up(G.ext[0], 32);
    } else if (dim == 2) {
        G.pitch = round_up(G.ext[1], 32);
        G.pitch2 = G.pitch;
        G.plane = (long long)G.ext[0] * G.pitch;
    } else {
        G.pitch = round_up(G.ext[2], 32);
        G.pitch2 = (long long)G.ext[1] * G.pitch;
        G.plane = (long long)G.ext[0] * G.pitch2;
    }
    return G;
}

// AoS (reference order, dense padded) <-> SoA (device planes).
__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, Geo G, int nf) {
    const long long ey = G.ext[1], ez = G.ext[2];
    const long long total = (long long)G.ext[0] * ey * ez;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long k = t % ez, j = (t / ez) % ey, i = t / (ey * ez);
        long long m;
        if (G.dim == 1) m = i;
        else if (G.dim == 2) m = i * G.pitch + j;
        else m = i * G.pitch2 + j * G.pitch + k;
        for (int f = 0; f < nf; f++) soa[f * G.plane + m] = aos[t * nf + f];
    }
}
__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, Geo G, int nf) {
    const long long ey = G.ext[1], ez = G.ext[2];
    const long long total = (long long)G.ext[0] * ey * ez;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long k = t % ez, j = (t / ez) % ey, i = t / (ey * ez);
        long long m;
        if (G.dim == 1) m = i;
        else if (G.dim == 2) m = i * G.pitch + j;
        else m = i * G.pitch2 + j * G.pitch + k;
        for (int f = 0; f < nf; f++) aos[t * nf + f] = soa[f * G.plane + m];
    }
}

// Copies `layers` whole layers along `axis` starting at padded position
// `first`, every field, between the state and a contiguous buffer ordered
// field, layer, transverse (the last axis fastest). Transverse axes cover
// padded positions [t0, t0 + tn).
__global__ void k_halo(Geo G, double* __restrict__ w, double* __restrict__ buf, int axis, int first, int layers, int nf,
                       int t0, int tn0, int tn1, int unpack) {
    int tax[2] = {0, 0}, nt = 0;
    for (int b = 0; b < G.dim; b++)
        if (b != axis) tax[nt++] = b;
    const long long sec = (long long)tn0 * tn1;
    const long long per_field = (long long)layers * sec;
    const long long total = per_field * nf;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per_field);
        const long long r = t % per_field;
        int q[3] = {0, 0, 0};
        q[axis] = first + (int)(r / sec);
        const long long tr = r % sec;
        if (nt > 0) q[tax[0]] = t0 + (int)(tr / tn1);
        if (nt > 1) q[tax[1]] = t0 + (int)(tr % tn1);
        long long m;
        if (G.dim == 1) m = q[0];
        else if (G.dim == 2) m = (long long)q[0] * G.pitch + q[1];
        else m = (long long)q[0] * G.pitch2 + (long long)q[1] * G.pitch + q[2];
        if (unpack) w[f * G.plane + m] = buf[t];
        else buf[t] = w[f * G.plane + m];
    }
}

int solver_id(const dragon_config& c) {
    if (c.mhd) {
        if (c.riemann == RS_HLL) return RS_HLL;
        if (c.riemann == RS_HLLE) return RS_HLLE;
        return RS_HLLD;
    }
    switch (c.riemann) {
        case RS_HLLX:
        case RS_HLLC: return RS_HLLC;
        case RS_HLL: return RS_HLL;
        case RS_HLLE: return RS_HLLE;
        case RS_ROE: return RS_ROE;
        default: return RS_EXACT;  // Flux.cpp:20-34 runtime switch default
    }
}

}  // namespace

// Lets the library's other translation units report a failure through
// dragon_gpu_last_error().
void dragon_gpu_set_error_message(const char* msg) { g_last_error = msg; }

// Packed network of a trainer (learned.cu).
const MlpNet* dragon_mlp_packed_net(dragon_mlp* m);


namespace dgpu_rt {

size_t dense_count(const Geo& G) { return (size_t)G.ext[0] * G.ext[1] * G.ext[2]; }

StepArgs step_args(const dragon_grid* h, int slot_out) {
    StepArgs a;
    a.dx = h->d[0];
    a.dy = h->d[1];
    a.dz = h->d[2];
    a.limiter = h->cfg.limiter;
    a.cfl = h->cfg.cfl;
    a.exact_max_iters = h->cfg.exact_max_iters;
    a.exact_tol = h->cfg.exact_tol;
    a.ct_energy = h->cfg.ct_energy;
    a.slot_out = slot_out;
    a.forced = 0;
    a.exact_guess = h->cfg.exact_guess;
    a.guess_err = h->cfg.perfect_guess_err_exp > 0 ? std::pow(10.0, -h->cfg.perfect_guess_err_exp) : 0.0;
    a.nlog = NewtonLog{h->nlog_rows, h->nlog_count, h->nlog_cap, h->nlog_stride};
    a.mlp = h->mlp_dev;
    return a;
}

cudaEvent_t take_event(dragon_grid* h) {
    if (!h->ev_pool.empty()) {
        cudaEvent_t e = h->ev_pool.back();
        h->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Folds finished step-kernel timings into the running total.
void collect_profile(dragon_grid* h) {
    for (auto& p : h->ev_pending) {
        float ms = 0;
        if (cudaEventSynchronize(p.second) == cudaSuccess && cudaEventElapsedTime(&ms, p.first, p.second) == cudaSuccess) {
            h->prof_ms += ms;
            h->prof_n += 1;
        }
        h->ev_pool.push_back(p.first);
        h->ev_pool.push_back(p.second);
    }
    h->ev_pending.clear();
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// The tensor map of state buffer b for the fused 2D hydro kernel (mixed or
// FP64): the five field planes as a 3D FP64 tensor (padded columns, padded
// rows, fields) with the kernel's tile box; encoded on first use, the buffers
// live as long as the handle.
static int state_tile_map(dragon_grid* h, int mixed, int b, const CUtensorMap** out) {
    if (!h->tmap_ok[mixed][b]) {
        auto encode = tensor_map_encoder();
        if (!encode) return fail(DRAGON_GPU_ECUDA, "cuTensorMapEncodeTiled is not available");
        int box[3];
        step2d_tile_box(mixed, box);
        const cuuint64_t dims[3] = {(cuuint64_t)h->cg.ext[1], (cuuint64_t)h->cg.ext[0], 5};
        const cuuint64_t strides[2] = {(cuuint64_t)h->cg.pitch * sizeof(double), (cuuint64_t)h->cg.plane * sizeof(double)};
        const cuuint32_t boxd[3] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2]};
        const cuuint32_t elem[3] = {1, 1, 1};
        const CUresult r = encode(&h->tmap[mixed][b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, h->w[b], dims, strides, boxd,
                                  elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(DRAGON_GPU_ECUDA, "cuTensorMapEncodeTiled failed for the state tile");
        h->tmap_ok[mixed][b] = true;
    }
    *out = &h->tmap[mixed][b];
    return 0;
}

int launch_step(dragon_grid* h, int c) {
    const StepArgs sa = step_args(h, c ^ 1);
    if (sa.exact_guess == GUESS_LEARNED && h->solver == RS_EXACT && !sa.mlp)
        return fail(DRAGON_GPU_EINVAL, "exact_guess = learned needs a network (dragon_gpu_grid_set_mlp)");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (h->prof) {
        e0 = take_event(h);
        e1 = take_event(h);
        cudaEventRecord(e0, h->stream);
    }
    int rc = 0, nk = 1;
    if (h->dim == 1) {
        rc = (h->cfg.precision == 1)
                 ? launch_step1d_mixed(h->mhd, h->solver, h->cg, h->w[c], h->w[c ^ 1], h->ctl, sa, h->stream)
                 : launch_step1d(h->mhd, h->solver, h->cg, h->w[c], h->w[c ^ 1], h->ctl, sa, h->stream);
    } else if (h->mhd) {
        if (h->dim == 3) {
            rc = (h->cfg.precision == 1)
                     ? launch_step3d_mhd_mixed(h->solver, h->cg, h->fg, h->w[c], h->w[c ^ 1], h->B[c], h->B[c ^ 1],
                                               h->m3_s, h->ctl, sa, h->stream)
                     : launch_step3d_mhd(h->solver, h->cg, h->fg, h->w[c], h->w[c ^ 1], h->B[c], h->B[c ^ 1], h->m3_s,
                                         h->ctl, sa, h->stream);
            nk = kMhd3DKernels;
        } else if (h->cfg.precision == 1) {
            const MhdScratchF SF{(float*)h->mhd_s.hs, (float*)h->mhd_s.fx, (float*)h->mhd_s.fy, (float*)h->mhd_s.er,
                                 (float*)h->mhd_s.e0, (float*)h->mhd_s.eh, h->mhd_s.plane};
            rc = launch_step2d_mhd_mixed(h->solver, h->cg, h->fg, h->w[c], h->w[c ^ 1], h->B[c], h->B[c ^ 1], SF,
                                         h->ctl, sa, h->stream);
        } else {
            rc = launch_step2d_mhd(h->solver, h->cg, h->fg, h->w[c], h->w[c ^ 1], h->B[c], h->B[c ^ 1], h->mhd_s,
                                   h->ctl, sa, h->stream);
        }
        // 2D: the ghost-frame copy, then seven phase kernels (FP64) or the fused kernel (mixed)
        if (h->dim == 2) nk = h->cfg.precision == 1 ? 1 : kMhd2DKernels;
    } else if (h->dim == 2) {
        const int mixed = h->cfg.precision == 1 ? 1 : 0;
        const CUtensorMap* map = nullptr;
        if ((rc = state_tile_map(h, mixed, c, &map))) return rc;
        rc = mixed ? launch_step2d_hydro_mixed(h->solver, h->cg, h->w[c], h->w[c ^ 1], h->ctl, sa, map, h->stream)
                   : launch_step2d_hydro(h->solver, h->cg, h->w[c], h->w[c ^ 1], h->ctl, sa, map, h->stream);
    } else {
        rc = (h->cfg.precision == 1)
                 ? launch_step3d_hydro_mixed(h->solver, h->cg, h->w[c], h->w[c ^ 1], h->h3_s, h->ctl, sa, h->stream)
                 : launch_step3d_hydro(h->solver, h->cg, h->w[c], h->w[c ^ 1], h->h3_s, h->ctl, sa, h->stream);
        nk = kHydro3DKernels;
    }
    if (rc) return fail(DRAGON_GPU_ECUDA, std::string("step launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    if (h->prof) {
        cudaEventRecord(e1, h->stream);
        h->ev_pending.push_back({e0, e1});
    }
    h->launches += nk;
    return 0;
}

// w_buf overrides the state buffer (the Strang-split sweeps fill ghosts of their intermediate buffers).
static int launch_prologue_range(dragon_grid* h, int c, int bookkeeping, int apply_bc, int compute_dt, int slot_in,
                                 int slot_out, double* w_buf, int bc_first, int bc_count) {
    double* W = w_buf ? w_buf : h->w[c];
    if (bc_count < 0) bc_count = h->nbc - bc_first;
    PrologueArgs pa;
    pa.dx = h->d[0];
    pa.dy = h->d[1];
    pa.dz = h->d[2];
    pa.cfl_coeff = h->cfg.cfl_coeff;
    pa.tol = h->cfg.timestep_tol;
    pa.cfl = h->cfg.cfl;
    pa.slot_in = slot_in;
    pa.slot_out = slot_out;
    pa.bookkeeping = bookkeeping;
    pa.apply_bc = apply_bc;
    pa.compute_dt = compute_dt;
    pa.nbc = bc_count;
    pa.bc_first = bc_first;
    pa.stall_cta = h->dbg_stall_cta;
    auto one_cta = [&](const PrologueArgs& a) {
        if (h->mhd) k_prologue<true><<<1, 1024, 0, h->stream>>>(h->cg, h->fg, W, h->B[c], h->dbcs, h->ctl, a);
        else k_prologue<false><<<1, 1024, 0, h->stream>>>(h->cg, h->fg, W, h->B[c], h->dbcs, h->ctl, a);
        h->launches++;
    };
    if (h->dim == 1 || !apply_bc || bc_count == 0) {
        one_cta(pa);
        CK(cudaGetLastError());
        return 0;
    }
    long long ext_max = 1;  // largest transverse section of a pass, padded
    for (int a = 0; a < h->dim; a++) {
        long long sec = 1;
        for (int b = 0; b < h->dim; b++)
            if (b != a) sec *= (h->fg.ext[b]);
        ext_max = std::max(ext_max, sec);
    }
    const long long items = 2 * ext_max * h->g;
    const int blocks = (int)std::max<long long>(1, std::min<long long>((items + 255) / 256, 148 * 8));
    // 2D / 3D: one cooperative launch (bookkeeping, every ghost-fill pass over
    // the whole grid, the ring CFL and dt, grid barriers between them) where the
    // device can hold its CTAs at once
    int& cap = h->coop_cap[h->mhd ? 1 : 0];
    const void* coop = h->mhd ? (const void*)k_prologue_coop<true> : (const void*)k_prologue_coop<false>;
    if (cap == 0) {
        int dev = 0, sms = 0, occ = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, coop, 256, 0));
        int coop_ok = 0;
        CK(cudaDeviceGetAttribute(&coop_ok, cudaDevAttrCooperativeLaunch, dev));
        cap = (coop_ok && occ > 0) ? occ * sms : -1;
    }
    if (cap > 0 && !h->dbg_no_coop) {
        Geo g0 = h->cg, g1 = h->fg;
        double* wp = W;
        double* bp = h->B[c];
        const BCEntry* ep = h->dbcs;
        StepCtl* cp = h->ctl;
        PrologueArgs ap = pa;
        void* args[] = {&g0, &g1, &wp, &bp, &ep, &cp, &ap};
        CK(cudaLaunchCooperativeKernel(coop, std::min(blocks, cap), 256, args, 0, h->stream));
        h->launches++;
        return 0;
    }
    // no cooperative launch: bookkeeping on one CTA, every ghost-fill pass over
    // a whole grid, then the ring CFL and dt on one CTA (the ghost layers of a
    // large grid are far too much work for one CTA)
    PrologueArgs head = pa;
    head.apply_bc = 0;
    head.compute_dt = 0;
    one_cta(head);
    for (int e = bc_first; e < bc_first + bc_count; e++) {
        for (int a = 0; a < h->dim; a++) {
            if (h->mhd) k_bc_pass<true><<<blocks, 256, 0, h->stream>>>(h->cg, h->fg, W, h->B[c], h->dbcs, h->ctl, e, a, 0);
            else k_bc_pass<false><<<blocks, 256, 0, h->stream>>>(h->cg, h->fg, W, h->B[c], h->dbcs, h->ctl, e, a, 0);
            h->launches++;
        }
        if (h->mhd) {
            for (int a = 0; a < h->dim; a++) {
                k_bc_pass<true><<<blocks, 256, 0, h->stream>>>(h->cg, h->fg, W, h->B[c], h->dbcs, h->ctl, e, a, 1);
                h->launches++;
            }
        }
    }
    if (compute_dt) {
        PrologueArgs tail = pa;
        tail.bookkeeping = 0;
        tail.apply_bc = 0;
        one_cta(tail);
    }
    CK(cudaGetLastError());
    return 0;
}

// The prologue over entries [bc_first, bc_first + bc_count) of the compiled
// list (all of them by default). A user fill compiled for the device splits
// it: the prologue of the entries before it (with the bookkeeping), the fill's
// kernel, then the rest, the last part computing dt; everything stays in the
// stream, so the device advance loop runs on without the host.
int launch_prologue(dragon_grid* h, int c, int bookkeeping, int apply_bc, int compute_dt, int slot_in, int slot_out,
                    double* w_buf = nullptr, int bc_first = 0, int bc_count = -1) {
    if (bc_count < 0) bc_count = h->nbc - bc_first;
    if (!apply_bc || h->user_entries.empty())
        return launch_prologue_range(h, c, bookkeeping, apply_bc, compute_dt, slot_in, slot_out, w_buf, bc_first,
                                     bc_count);
    int seg = bc_first, head = 1, rc;
    for (int u : h->user_entries) {
        if (u < bc_first || u >= bc_first + bc_count) continue;
        if (u > seg || (head && bookkeeping))
            if ((rc = launch_prologue_range(h, c, head ? bookkeeping : 0, 1, 0, slot_in, slot_out, w_buf, seg, u - seg)))
                return rc;
        if ((rc = launch_user_fill(h, c, u, w_buf))) return rc;
        seg = u + 1;
        head = 0;
    }
    const int rest = bc_first + bc_count - seg;
    if (rest > 0 || compute_dt || (head && bookkeeping))
        return launch_prologue_range(h, c, head ? bookkeeping : 0, 1, compute_dt, slot_in, slot_out, w_buf, seg, rest);
    return 0;
}

int launch_interior_cfl(dragon_grid* h, int c, int slot) {
    const long long total = (long long)h->n[0] * h->n[1] * h->n[2];
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
    if (blocks < 1) blocks = 1;
    if (h->mhd) k_interior_cfl<true><<<blocks, 256, 0, h->stream>>>(h->cg, h->w[c], h->ctl, slot, h->cfg.cfl, h->d[0], h->d[1], h->d[2]);
    else k_interior_cfl<false><<<blocks, 256, 0, h->stream>>>(h->cg, h->w[c], h->ctl, slot, h->cfg.cfl, h->d[0], h->d[1], h->d[2]);
    CK(cudaGetLastError());
    h->launches++;
    return 0;
}

// Grid2D/3D::split_step (Splitting.cpp:118-217) reading buffer c, writing
// c ^ 1: the Strang sequence of sweeps for sweep counter value `order`
// (2D: XYX / YXY alternating; 3D: the six cyclic and anticyclic orders),
// each sweep after a ghost fill of its input (advanceX/Y/Z apply the boundary
// first). Intermediates alternate between c ^ 1 and a third buffer, so buffer
// c stays intact for a retry. The interior CFL maximum of the result is
// accumulated into slot c ^ 1 for the next step's dt. 1D grids take the
// unsplit step (Grid1D::split_step calls unsplit_step).
int launch_split_step(dragon_grid* h, int c, long long order) {
    if (h->dim == 1) return launch_step(h, c);
    if (!h->wsplit) {
        CK(cudaMalloc(&h->wsplit, sizeof(double) * h->nf * h->cg.plane));
        CK(cudaMemsetAsync(h->wsplit, 0, sizeof(double) * h->nf * h->cg.plane, h->stream));
    }
    struct Sweep { int axis; double f; };
    Sweep seq[5];
    int ns = 3;
    if (h->dim == 2) {
        const int a = (order % 2 == 0) ? 0 : 1, b = 1 - a;
        seq[0] = {a, 0.5}; seq[1] = {b, 1.0}; seq[2] = {a, 0.5};
    } else {
        static const int orders[6][3] = {{0, 1, 2}, {2, 0, 1}, {1, 2, 0}, {2, 1, 0}, {0, 2, 1}, {1, 0, 2}};
        const int* o = orders[order % 6];
        ns = 5;
        seq[0] = {o[0], 0.5}; seq[1] = {o[1], 0.5}; seq[2] = {o[2], 1.0}; seq[3] = {o[1], 0.5}; seq[4] = {o[0], 0.5};
    }
    const StepArgs sa = step_args(h, c ^ 1);
    double* in = h->w[c];
    double* out = h->w[c ^ 1];
    for (int k = 0; k < ns; k++) {
        int rc = launch_prologue(h, c, 0, 1, 0, 2, 2, in);
        if (rc) return rc;
        if (launch_sweep(h->solver, seq[k].axis, h->cg, in, out, h->ctl, sa, seq[k].f, h->stream))
            return fail(DRAGON_GPU_ECUDA, std::string("sweep launch failed: ") + cudaGetErrorString(cudaGetLastError()));
        h->launches++;
        in = out;
        out = (out == h->w[c ^ 1]) ? h->wsplit : h->w[c ^ 1];
    }
    return launch_interior_cfl(h, c ^ 1, c ^ 1);
}

// The step the current mode takes: unsplit, or split with the sweep order of
// advance-local step k.
int launch_any_step(dragon_grid* h, int c, long long k) {
    return h->split_mode ? launch_split_step(h, c, h->sweep_step + k) : launch_step(h, c);
}

// Writes the control block's header (everything before vmax) from the host mirror.
int push_ctl(dragon_grid* h) {
    CK(cudaMemcpyAsync(h->ctl, h->hctl, offsetof(StepCtl, vmax), cudaMemcpyHostToDevice, h->stream));
    return 0;
}
int pull_ctl(dragon_grid* h) {
    CK(cudaMemcpyAsync(h->hctl, h->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}
int zero_slot(dragon_grid* h, int slot) {
    CK(cudaMemsetAsync(&h->ctl->vmax[slot], 0, sizeof(unsigned long long), h->stream));
    return 0;
}

void reset_ctl(dragon_grid* h, double remaining, int max_steps, int check_cfl) {
    StepCtl& c = *h->hctl;
    unsigned long long keep[3] = {c.vmax[0], c.vmax[1], c.vmax[2]};
    std::memset(&c, 0, sizeof(StepCtl));
    c.remaining = remaining;
    c.err_key = ~0ull;
    c.max_steps = max_steps;
    c.check_cfl = check_cfl;
    for (int i = 0; i < 3; i++) c.vmax[i] = keep[i];
}

void fill_failure(const StepCtl& c, dragon_step_status* st, int code) {
    if (!st) return;
    st->code = code;
    st->stage = (c.err_key == ~0ull) ? 0 : (int)(c.err_key >> 56);
    st->cell = (c.err_key == ~0ull) ? -1 : (long long)(c.err_key & 0x00FFFFFFFFFFFFFFull);
    st->dt = c.t1;
}

// Adds a control block's exact-solver counters to the grid's running totals.
void add_newton(dragon_grid* h, const StepCtl& c) {
    h->ntot.exact_calls += c.exact_calls;
    h->ntot.newton_iters += c.newton_iters;
    h->ntot.trrs += c.trrs;
    h->ntot.cap_hits += c.cap_hits;
    h->ntot.guess_rejects += c.guess_rejects;
    h->ntot.judge_reruns += c.judge_reruns;
    h->ntot.pivots_exact += c.pivots_exact;
}

void fill_stats(dragon_grid* h, const StepCtl& c, dragon_advance_stats* st) {
    add_newton(h, c);
    if (!st) return;
    st->pivots_exact += c.pivots_exact;
    st->hlld_to_hlle += c.hlld_to_hlle;
    st->newton_iters += c.newton_iters;
    st->exact_calls += c.exact_calls;
    st->trrs += c.trrs;
    st->muscl_first_order += c.muscl_first_order;
}

const char* stage_name(int s) {
    switch (s) {
        case ST_PRELIM_FLUX: return "Riemann Solution to physical inputs is unphysical (predictor flux)";
        case ST_FINAL_FLUX: return "Riemann Solution to physical inputs is unphysical";
        case ST_NAN: return "NaN state would be produced";
        case ST_UNPHYSICAL: return "Unphysical state would be produced";
        case ST_CFL_ZERO: return "CFL timestep failed: max signal speed is zero";
        case ST_BARRIER: return "ghost fill failed: a grid barrier gave up waiting";
        case ST_TILE_LOAD: return "step failed: a tile load did not complete";
        default: return "step failed";
    }
}

// Shared advance loop. remaining/max_steps select advance(interval) or a step count.
// One batch of up to kBatch steps of the advance in flight: for step k the
// prologue (bookkeeping, ghost fill, CFL dt) reads buffer cur0 ^ (k & 1) and
// the step writes the other buffer.
static int enqueue_batch(dragon_grid* h) {
    AdvanceState& A = h->adv;
    int nb = kBatch;
    if (A.max_steps > 0) nb = (int)std::min<long long>(kBatch, (long long)A.max_steps + 1 - A.k);
    if (nb < 1) nb = 1;
    int rc;
    for (int b = 0; b < nb; b++) {
        const int c = A.cur0 ^ (int)((A.k + b) & 1);
        // with a step budget, the slot after the last step only accounts it;
        // advance_finish does that on the host (account_last_step)
        if (A.max_steps > 0 && A.k + b >= A.max_steps) continue;
        if ((rc = launch_prologue(h, c, 1, 1, 1, c, c ^ 1))) return rc;
        if ((rc = launch_any_step(h, c, A.k + b))) return rc;
    }
    A.k += nb;
    return 0;
}

// The bookkeeping of the prologue that would follow a step budget's last
// step (prologue_bookkeeping), done on the host mirror once that step has run:
// one launch fewer per budgeted advance. The device copy of the control block
// is not read again before the next advance rewrites it.
static bool account_last_step(dragon_grid* h, StepCtl& C) {
    if (C.have_prev) {
        C.remaining -= C.t1;
        C.elapsed += C.t1;
        C.steps_done += 1;
    }
    C.have_prev = 1;
    if (!(C.remaining > h->cfg.timestep_tol) || (C.max_steps > 0 && C.steps_done >= C.max_steps)) C.done = 1;
    return C.done != 0;
}

int advance_begin(dragon_grid* h, double remaining, int max_steps, int check_cfl) {
    if (h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight: call dragon_gpu_advance_wait");
    h->can_rollback = false;
    AdvanceState& A = h->adv;
    A = AdvanceState{};
    A.cur0 = h->cur;
    A.remaining = remaining;
    A.max_steps = max_steps;
    reset_ctl(h, remaining, max_steps, check_cfl);
    int rc = push_ctl(h);
    if (rc) return rc;
    if (!h->imax_valid) {
        if ((rc = zero_slot(h, A.cur0))) return rc;
        if ((rc = launch_interior_cfl(h, A.cur0, A.cur0))) return rc;
    }
    A.pending = true;
    rc = enqueue_batch(h);
    if (rc) A.pending = false;
    return rc;
}

// Reads the control block after each batch: on a failed step halves t1 and
// retries it on the same ghosts (CFL.cpp:198-208), otherwise enqueues the next
// batch until the advance is done.
int advance_finish(dragon_grid* h, dragon_advance_stats* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    AdvanceState& A = h->adv;
    if (!A.pending) return fail(DRAGON_GPU_EINVAL, "no advance in flight");
    A.pending = false;
    const int cur0 = A.cur0;
    int rc;
    for (;;) {
        if ((rc = pull_ctl(h))) return rc;
        StepCtl& C = *h->hctl;
        if (C.err) {
            const long long ks = C.steps_done;  // index of the failed step
            const int c = cur0 ^ (int)(ks & 1);
            h->cur = c;
            h->imax_valid = true;
            const int stage = (int)(C.err_key >> 56);
            fill_stats(h, C, st);
            if (st) { st->steps = (int)ks; fill_failure(C, &st->failure, DRAGON_GPU_ESTEP); }
            if (stage == ST_CFL_ZERO) {
                if (st) st->failure.code = DRAGON_GPU_ECFL;
                if (h->split_mode) h->sweep_step += ks;
                return fail(DRAGON_GPU_ECFL, stage_name(stage));
            }
            if (stage == ST_BARRIER || stage == ST_TILE_LOAD) {  // not a physics failure: no retry
                if (st) st->failure.code = DRAGON_GPU_ECUDA;
                if (h->split_mode) h->sweep_step += ks;
                h->imax_valid = false;
                return fail(DRAGON_GPU_ECUDA, stage_name(stage));
            }
            // CFL.cpp:198-208: halve t1 and retry the same step on the same ghosts.
            double t1 = C.t1;
            for (;;) {
                A.retries++;
                t1 *= 0.5;
                if (t1 < h->cfg.timestep_tol) {
                    if (st) { st->retries = A.retries; st->failure.code = DRAGON_GPU_EDT; }
                    if (h->split_mode) h->sweep_step += ks;
                    return fail(DRAGON_GPU_EDT, std::string("Timestep has fallen below minimum after: ") + stage_name(stage));
                }
                C.t1 = t1;
                C.err = 0;
                C.err_key = ~0ull;
                C.pivots_exact = C.hlld_to_hlle = C.newton_iters = C.exact_calls = C.trrs = C.muscl_first_order = 0;
                C.cap_hits = C.guess_rejects = C.judge_reruns = 0;
                if ((rc = push_ctl(h))) return rc;
                if ((rc = zero_slot(h, c ^ 1))) return rc;
                if ((rc = launch_any_step(h, c, ks))) return rc;
                if ((rc = pull_ctl(h))) return rc;
                if (!C.err) break;
                fill_stats(h, C, st);
            }
            // success: the next prologue accounts the retried step; step k reads
            // buffer cur0 ^ (k & 1) == c ^ 1
            A.k = ks + 1;
            if ((rc = enqueue_batch(h))) return rc;
            continue;
        }
        if (!C.done && A.max_steps > 0 && A.k > A.max_steps && !account_last_step(h, C))
            return fail(DRAGON_GPU_ESTEP, "step budget consumed but the advance did not finish");
        if (C.done) {
            h->cur = cur0 ^ (int)(C.steps_done & 1);
            h->imax_valid = true;
            if (h->split_mode) h->sweep_step += C.steps_done;
            fill_stats(h, C, st);
            if (st) {
                st->steps = C.steps_done;
                st->retries = A.retries;
                st->last_dt = C.t1;
                // the interval consumed (Grid::advance's own bookkeeping), or for a
                // step budget without an interval the sum of the steps' dt
                st->time_advanced = std::isfinite(A.remaining) ? (A.remaining - C.remaining) : C.elapsed;
            }
            return 0;
        }
        if ((rc = enqueue_batch(h))) return rc;
    }
}

int advance_impl(dragon_grid* h, double remaining, int max_steps, int check_cfl, dragon_advance_stats* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    int rc = advance_begin(h, remaining, max_steps, check_cfl);
    if (rc) return rc;
    return advance_finish(h, st);
}

}  // namespace dgpu_rt

using namespace dgpu_rt;

extern "C" {

const char* dragon_gpu_last_error(void) { return g_last_error.c_str(); }

void dragon_gpu_default_config(dragon_config* c, int mhd) {
    std::memset(c, 0, sizeof(*c));
    c->mhd = mhd ? 1 : 0;
    c->riemann = RS_HLLX;
    c->limiter = LIM_MC;
    c->cfl = 1;
    c->ct_energy = 2;
    c->exact_max_iters = 6;
    c->exact_tol = 1e-12;
    c->cfl_coeff = 0.3;
    c->timestep_tol = 1e-14;
    c->precision = 0;
}

int dragon_gpu_grid_create(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts,
                           const dragon_config* cfg, dragon_grid** out) {
    if (!out || dim < 1 || dim > 3 || nx < 1 || (dim >= 2 && ny < 1) || (dim >= 3 && nz < 1))
        return fail(DRAGON_GPU_EINVAL, "invalid grid extents");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count < 1)
        return fail(DRAGON_GPU_ECUDA, "no CUDA device available");
    dragon_grid* h = new dragon_grid();
    if (cfg) h->cfg = *cfg;
    else dragon_gpu_default_config(&h->cfg, 0);
    h->mhd = h->cfg.mhd != 0;
    h->nf = h->mhd ? 8 : 5;
    h->dim = dim;
    h->n[0] = nx;
    h->n[1] = dim >= 2 ? ny : 1;
    h->n[2] = dim >= 3 ? nz : 1;
    h->d[0] = dx;
    h->d[1] = dim >= 2 ? dy : 0.0;
    h->d[2] = dim >= 3 ? dz : 0.0;
    // validGhosts (Splitting.cpp:23-31): MHD + CTU needs 3, MUSCL-Hancock 2
    const int gmin = (h->mhd && dim >= 2) ? 3 : 2;
    h->g = ghosts > gmin ? ghosts : gmin;
    if (h->mhd && dim == 1) h->g = ghosts > 3 ? ghosts : 3;
    h->solver = solver_id(h->cfg);
    if (h->cfg.exact_guess < GUESS_MEAN || h->cfg.exact_guess > GUESS_PERFECT) {
        delete h;
        return fail(DRAGON_GPU_EINVAL, "exact_guess must be 0 (mean), 1 (analytic), 2 (learned) or 3 (perfect)");
    }
    if (h->cfg.exact_guess == GUESS_LEARNED && !(dim == 3 && !h->mhd)) {
        delete h;
        return fail(DRAGON_GPU_EUNSUPPORTED, "the learned star-pressure guess is built for 3D hydro grids");
    }
    if (h->cfg.precision != 0 && h->cfg.exact_guess == GUESS_LEARNED) {
        delete h;
        return fail(DRAGON_GPU_EUNSUPPORTED, "the learned star-pressure guess runs on the FP64 3D step");
    }
    h->cg = make_geo(dim, h->n, h->g);
    int nfc[3] = {h->n[0] + 1, h->n[1] + 1, h->n[2] + 1};
    h->fg = make_geo(dim, nfc, h->g);
    auto cleanup = [&](int code) {
        dragon_gpu_grid_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(DRAGON_GPU_ECUDA, "cudaStreamCreate failed"));
    for (int b = 0; b < 2; b++) {
        if (cudaMalloc(&h->w[b], sizeof(double) * h->nf * h->cg.plane) != cudaSuccess)
            return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc state failed"));
        cudaMemsetAsync(h->w[b], 0, sizeof(double) * h->nf * h->cg.plane, h->stream);
        if (h->mhd && dim >= 2) {
            if (cudaMalloc(&h->B[b], sizeof(double) * 3 * h->fg.plane) != cudaSuccess)
                return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc faceB failed"));
            cudaMemsetAsync(h->B[b], 0, sizeof(double) * 3 * h->fg.plane, h->stream);
        }
    }
    if (h->mhd && dim == 2) {
        const long long P = h->fg.plane;
        if (cudaMalloc(&h->mhd_buf, sizeof(double) * MhdScratch::kPlanes * P) != cudaSuccess)
            return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc MHD intermediates failed"));
        h->mhd_s.hs = h->mhd_buf;
        h->mhd_s.fx = h->mhd_buf + 32 * P;
        h->mhd_s.fy = h->mhd_buf + 40 * P;
        h->mhd_s.er = h->mhd_buf + 48 * P;
        h->mhd_s.e0 = h->mhd_buf + 51 * P;
        h->mhd_s.eh = h->mhd_buf + 54 * P;
        h->mhd_s.plane = P;
    }
    if (h->mhd && dim == 3) {
        const long long P = h->fg.plane;
        if (cudaMalloc(&h->m3_buf, sizeof(double) * Mhd3DScratch::kPlanes * P) != cudaSuccess)
            return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc 3D MHD intermediates failed"));
        h->m3_s.hs = h->m3_buf;
        h->m3_s.fx = h->m3_buf + 48 * P;
        h->m3_s.fy = h->m3_buf + 56 * P;
        h->m3_s.fz = h->m3_buf + 64 * P;
        h->m3_s.er = h->m3_buf + 72 * P;
        h->m3_s.e0 = h->m3_buf + 75 * P;
        h->m3_s.eh = h->m3_buf + 78 * P;
        h->m3_s.plane = P;
    }
    if (!h->mhd && dim == 3) {
        const long long P = h->cg.plane;
        if (cudaMalloc(&h->h3_buf, sizeof(double) * Hydro3DScratch::kPlanes * P) != cudaSuccess)
            return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc 3D intermediates failed"));
        h->h3_s.hs = h->h3_buf;
        h->h3_s.pf = h->h3_buf + 30 * P;
        h->h3_s.cf = h->h3_buf + 45 * P;
        h->h3_s.plane = P;
    }
    if (cudaMalloc(&h->ctl, sizeof(StepCtl)) != cudaSuccess) return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc ctl failed"));
    cudaMemsetAsync(h->ctl, 0, sizeof(StepCtl), h->stream);
    if (cudaMallocHost(&h->hctl, sizeof(StepCtl)) != cudaSuccess) return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMallocHost failed"));
    std::memset(h->hctl, 0, sizeof(StepCtl));
    h->stage_elems = std::max(dense_count(h->cg) * h->nf, (h->mhd && dim >= 2) ? dense_count(h->fg) * 3 : (size_t)0);
    if (cudaMalloc(&h->stage, sizeof(double) * h->stage_elems) != cudaSuccess)
        return cleanup(fail(DRAGON_GPU_ECUDA, "cudaMalloc staging failed"));
    // default boundary: empty list = implicit Outflow on every face
    int rc = dragon_gpu_set_boundary(h, nullptr, 0);
    if (rc) return cleanup(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return cleanup(fail(DRAGON_GPU_ECUDA, "init sync failed"));
    *out = h;
    return 0;
}

int dragon_gpu_grid_destroy(dragon_grid* h) {
    if (!h) return 0;
    if (h->stream) cudaStreamSynchronize(h->stream);
    hoard_release(h);
    collect_profile(h);
    clear_user_fills(h);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    for (int b = 0; b < 2; b++) {
        if (h->w[b]) cudaFree(h->w[b]);
        if (h->B[b]) cudaFree(h->B[b]);
    }
    if (h->ctl) cudaFree(h->ctl);
    if (h->mhd_buf) cudaFree(h->mhd_buf);
    if (h->h3_buf) cudaFree(h->h3_buf);
    if (h->m3_buf) cudaFree(h->m3_buf);
    if (h->wsplit) cudaFree(h->wsplit);
    if (h->hctl) cudaFreeHost(h->hctl);
    if (h->dbcs) cudaFree(h->dbcs);
    if (h->stage) cudaFree(h->stage);
    if (h->nlog_rows) cudaFree(h->nlog_rows);
    if (h->nlog_count) cudaFree(h->nlog_count);
    if (h->mlp_dev) cudaFree(h->mlp_dev);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

int dragon_gpu_grid_info(const dragon_grid* h, int* dim, int* n3, int* ghosts, int* nfields) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (dim) *dim = h->dim;
    if (n3) { n3[0] = h->n[0]; n3[1] = h->n[1]; n3[2] = h->n[2]; }
    if (ghosts) *ghosts = h->g;
    if (nfields) *nfields = h->nf;
    return 0;
}

size_t dragon_gpu_prim_count(const dragon_grid* h) { return h ? dense_count(h->cg) * h->nf : 0; }
size_t dragon_gpu_faceB_count(const dragon_grid* h) {
    return (h && h->mhd && h->dim >= 2) ? dense_count(h->fg) * 3 : 0;
}

static int transfer(dragon_grid* h, bool up, bool faces, double* host) {
    if (!h || !host) return fail(DRAGON_GPU_EINVAL, "null argument");
    if (h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (faces && !(h->mhd && h->dim >= 2)) return fail(DRAGON_GPU_EINVAL, "grid has no face-centred B");
    const Geo& G = faces ? h->fg : h->cg;
    const int nf = faces ? 3 : h->nf;
    double* dev = faces ? h->B[h->cur] : h->w[h->cur];
    const size_t cnt = dense_count(G) * nf;
    const int blocks = (int)std::min<size_t>((dense_count(G) + 255) / 256, 148 * 16);
    if (up) {
        CK(cudaMemcpyAsync(h->stage, host, cnt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        k_aos_to_soa<<<blocks, 256, 0, h->stream>>>(h->stage, dev, G, nf);
        CK(cudaGetLastError());
        h->launches++;
        h->imax_valid = false;
        h->can_rollback = false;
    } else {
        k_soa_to_aos<<<blocks, 256, 0, h->stream>>>(dev, h->stage, G, nf);
        CK(cudaGetLastError());
        h->launches++;
        CK(cudaMemcpyAsync(host, h->stage, cnt * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int dragon_gpu_upload_prim(dragon_grid* h, const double* host) { return transfer(h, true, false, const_cast<double*>(host)); }
int dragon_gpu_download_prim(dragon_grid* h, double* host) { return transfer(h, false, false, host); }
int dragon_gpu_upload_faceB(dragon_grid* h, const double* host) { return transfer(h, true, true, const_cast<double*>(host)); }
int dragon_gpu_download_faceB(dragon_grid* h, double* host) { return transfer(h, false, true, host); }

int dragon_gpu_set_boundary(dragon_grid* h, const dragon_bc_desc* list, int n) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h || n < 0 || (n > 0 && !list)) return fail(DRAGON_GPU_EINVAL, "invalid boundary list");
    std::vector<BCEntry> v;
    // implicit Outflow over every face no entry covers (BoundaryList.hpp:97-104)
    int uncovered = FX_NEG | FX_POS | FY_NEG | FY_POS | FZ_NEG | FZ_POS;
    std::vector<BCEntry> user;
    std::vector<int> device_fill;  // caller indices of user fills compiled for the device
    for (int i = 0; i < n; i++) {
        BCEntry e{};
        e.type = list[i].type;
        if (e.type == DRAGON_BC_USER) {
            // the device list carries it as Ignore (its faces count as covered);
            // the prologue launches its bound fill at this place
            e.type = BC_IGNORE;
            device_fill.push_back(i);
        }
        if (e.type < BC_OUTFLOW || e.type > BC_IGNORE) return fail(DRAGON_GPU_EINVAL, "unknown boundary type");
        e.faces = list[i].faces & 63;
        if (e.type == BC_PERIODIC) {
            // Periodic.cpp:14-15: a periodic axis always covers both faces
            int f = 0;
            if (e.faces & (FX_NEG | FX_POS)) f |= FX_NEG | FX_POS;
            if (e.faces & (FY_NEG | FY_POS)) f |= FY_NEG | FY_POS;
            if (e.faces & (FZ_NEG | FZ_POS)) f |= FZ_NEG | FZ_POS;
            e.faces = f;
        }
        e.corners = list[i].corners ? 1 : 0;
        for (int k = 0; k < 8; k++) e.state[k] = list[i].state[k];
        uncovered &= ~e.faces;
        user.push_back(e);
    }
    if (uncovered) {
        BCEntry imp{};
        imp.type = BC_OUTFLOW;
        imp.faces = uncovered;
        imp.corners = 1;
        v.push_back(imp);
    }
    for (auto& e : user) v.push_back(e);
    if (h->dbcs) { cudaStreamSynchronize(h->stream); cudaFree(h->dbcs); h->dbcs = nullptr; }
    h->nbc = (int)v.size();
    h->hbcs = v;
    clear_user_fills(h);
    h->caller_entries = n;
    h->user_entries.clear();
    for (int i : device_fill) h->user_entries.push_back(h->nbc - n + i);
    h->ufill.assign(h->nbc, UserFillBinding{});
    if (h->nbc) {
        CK(cudaMalloc(&h->dbcs, sizeof(BCEntry) * v.size()));
        CK(cudaMemcpyAsync(h->dbcs, v.data(), sizeof(BCEntry) * v.size(), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return 0;
}

int dragon_gpu_apply_boundary(dragon_grid* h) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    reset_ctl(h, 0.0, 0, 0);
    int rc = push_ctl(h);
    if (rc) return rc;
    if ((rc = launch_prologue(h, h->cur, 0, 1, 0, 2, 2))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int dragon_gpu_boundary_entries(const dragon_grid* h) { return h ? h->nbc : 0; }

int dragon_gpu_set_origin(dragon_grid* h, int i0, int j0, int k0) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null grid");
    h->origin[0] = i0;
    h->origin[1] = h->dim > 1 ? j0 : 0;
    h->origin[2] = h->dim > 2 ? k0 : 0;
    return 0;
}

int dragon_gpu_apply_boundary_range(dragon_grid* h, int first, int count) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h || first < 0 || count < 0 || first + count > h->nbc) return fail(DRAGON_GPU_EINVAL, "entry range out of bounds");
    if (count == 0) return 0;
    reset_ctl(h, 0.0, 0, 0);
    int rc = push_ctl(h);
    if (rc) return rc;
    if ((rc = launch_prologue(h, h->cur, 0, 1, 0, 2, 2, nullptr, first, count))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int dragon_gpu_cfl_time(dragon_grid* h, double* dt_out) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h || !dt_out) return fail(DRAGON_GPU_EINVAL, "null argument");
    reset_ctl(h, INFINITY, 0, 1);
    int rc = push_ctl(h);
    if (rc) return rc;
    if ((rc = zero_slot(h, 2))) return rc;
    if ((rc = launch_interior_cfl(h, h->cur, 2))) return rc;
    if ((rc = launch_prologue(h, h->cur, 0, 0, 1, 2, 2))) return rc;
    if ((rc = pull_ctl(h))) return rc;
    if (h->hctl->err) return fail(DRAGON_GPU_ECFL, stage_name(ST_CFL_ZERO));
    *dt_out = h->hctl->t1;
    return 0;
}

int dragon_gpu_unsplit_step(dragon_grid* h, double dt, dragon_step_status* st) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (st) std::memset(st, 0, sizeof(*st));
    reset_ctl(h, 0.0, 0, 0);
    h->hctl->t1 = dt;
    int rc = push_ctl(h);
    if (rc) return rc;
    const int c = h->cur;
    if ((rc = zero_slot(h, c ^ 1))) return rc;
    if ((rc = launch_step(h, c))) return rc;
    if ((rc = pull_ctl(h))) return rc;
    add_newton(h, *h->hctl);
    if (h->hctl->err) {
        fill_failure(*h->hctl, st, DRAGON_GPU_ESTEP);
        return fail(DRAGON_GPU_ESTEP, stage_name((int)(h->hctl->err_key >> 56)));
    }
    h->cur = c ^ 1;
    h->imax_valid = true;
    h->can_rollback = true;
    if (st) st->dt = dt;
    return 0;
}

int dragon_gpu_step_rollback(dragon_grid* h) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (!h->can_rollback) return fail(DRAGON_GPU_EINVAL, "no committed unsplit_step to undo");
    CK(cudaStreamSynchronize(h->stream));
    h->cur ^= 1;
    h->imax_valid = false;
    h->can_rollback = false;
    return 0;
}

// Geometry, base pointer and field count of the cell state or face-centred B.
static int halo_target(dragon_grid* h, int faces, Geo* G, double** base, int* nf) {
    if (faces) {
        if (!h->mhd || h->dim < 2) return fail(DRAGON_GPU_EINVAL, "grid has no face-centred B");
        *G = h->fg;
        *base = h->B[h->cur];
        *nf = 3;
    } else {
        *G = h->cg;
        *base = h->w[h->cur];
        *nf = h->nf;
    }
    return 0;
}

// Transverse extent (padded positions) of a halo along `axis`.
static void halo_transverse(const Geo& G, int dim, int axis, int corners, int* t0, int tn[2]) {
    tn[0] = tn[1] = 1;
    *t0 = corners ? 0 : G.g;
    int k = 0;
    for (int b = 0; b < dim; b++)
        if (b != axis) tn[k++] = corners ? G.ext[b] : G.n[b];
}

int dragon_gpu_halo_size(const dragon_grid* h, int axis, int layers, int faces, int corners, long long* count) {
    if (!h || axis < 0 || axis >= h->dim || layers < 1 || !count) return fail(DRAGON_GPU_EINVAL, "invalid halo arguments");
    Geo G;
    double* base;
    int nf;
    int rc = halo_target(const_cast<dragon_grid*>(h), faces, &G, &base, &nf);
    if (rc) return rc;
    if (layers > G.ext[axis]) return fail(DRAGON_GPU_EINVAL, "more layers than the padded extent");
    int t0, tn[2];
    halo_transverse(G, h->dim, axis, corners, &t0, tn);
    *count = (long long)nf * layers * tn[0] * tn[1];
    return 0;
}

static int halo_copy(dragon_grid* h, int axis, int first, int layers, int faces, int corners, double* buf, int on_device,
                     bool pack) {
    long long count = 0;
    int rc = dragon_gpu_halo_size(h, axis, layers, faces, corners, &count);
    if (rc) return rc;
    Geo G;
    double* base;
    int nf;
    halo_target(h, faces, &G, &base, &nf);
    if (first < -G.g || first + layers > G.n[axis] + G.g) return fail(DRAGON_GPU_EINVAL, "halo layers outside the padded grid");
    if (!buf) return fail(DRAGON_GPU_EINVAL, "null buffer");
    int t0, tn[2];
    halo_transverse(G, h->dim, axis, corners, &t0, tn);
    double* dev = buf;
    if (!on_device) {
        // the staging buffer holds a whole padded grid, so any set of layers fits
        if ((size_t)count > h->stage_elems) return fail(DRAGON_GPU_EINVAL, "halo larger than the staging buffer");
        dev = h->stage;
    }
    if (!pack && !on_device) CK(cudaMemcpyAsync(dev, buf, sizeof(double) * count, cudaMemcpyHostToDevice, h->stream));
    const int blocks = (int)std::min<long long>((count + 255) / 256, 148 * 16);
    k_halo<<<std::max(blocks, 1), 256, 0, h->stream>>>(G, base, dev, axis, first + G.g, layers, nf, t0, tn[0], tn[1],
                                                       pack ? 0 : 1);
    CK(cudaGetLastError());
    h->launches++;
    if (pack && !on_device) CK(cudaMemcpyAsync(buf, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (!pack) {
        h->imax_valid = false;
        h->can_rollback = false;
    }
    return 0;
}

int dragon_gpu_halo_pack(dragon_grid* h, int axis, int first, int layers, int faces, int corners, double* buf,
                         int buf_on_device) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    return halo_copy(h, axis, first, layers, faces, corners, buf, buf_on_device, true);
}

int dragon_gpu_halo_unpack(dragon_grid* h, int axis, int first, int layers, int faces, int corners, const double* buf,
                           int buf_on_device) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    return halo_copy(h, axis, first, layers, faces, corners, const_cast<double*>(buf), buf_on_device, false);
}

int dragon_gpu_advance(dragon_grid* h, double interval, int check_cfl, dragon_advance_stats* st) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    return advance_impl(h, interval, 0, check_cfl ? 1 : 0, st);
}

int dragon_gpu_advance_steps(dragon_grid* h, int nsteps, dragon_advance_stats* st) {
    if (!h || nsteps < 0) return fail(DRAGON_GPU_EINVAL, "invalid argument");
    if (nsteps == 0) { if (st) std::memset(st, 0, sizeof(*st)); return 0; }
    return advance_impl(h, INFINITY, nsteps, 1, st);
}

int dragon_gpu_advance_steps_async(dragon_grid* h, int nsteps) {
    if (!h || nsteps < 1) return fail(DRAGON_GPU_EINVAL, "invalid argument");
    if (h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an advance is already in flight");
    return advance_begin(h, INFINITY, nsteps, 1);
}

int dragon_gpu_advance_wait(dragon_grid* h, dragon_advance_stats* st) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    return advance_finish(h, st);
}

static int split_unsupported(const dragon_grid* h) {
    if (h->mhd && h->dim >= 2) return fail(DRAGON_GPU_EUNSUPPORTED, "the Strang-split path is built for hydro grids");
    if (h->cfg.precision != 0) return fail(DRAGON_GPU_EUNSUPPORTED, "the Strang-split path runs in FP64");
    return 0;
}

int dragon_gpu_split_step(dragon_grid* h, double dt, dragon_step_status* st) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    int rc = split_unsupported(h);
    if (rc) return rc;
    if (st) std::memset(st, 0, sizeof(*st));
    reset_ctl(h, 0.0, 0, 0);
    h->hctl->t1 = dt;
    if ((rc = push_ctl(h))) return rc;
    const int c = h->cur;
    if ((rc = zero_slot(h, c ^ 1))) return rc;
    if ((rc = launch_split_step(h, c, h->sweep_step))) return rc;
    if ((rc = pull_ctl(h))) return rc;
    add_newton(h, *h->hctl);
    if (h->hctl->err) {
        fill_failure(*h->hctl, st, DRAGON_GPU_ESTEP);
        return fail(DRAGON_GPU_ESTEP, stage_name((int)(h->hctl->err_key >> 56)));
    }
    h->cur = c ^ 1;
    h->imax_valid = true;
    if (h->dim >= 2) h->sweep_step++;
    if (st) st->dt = dt;
    return 0;
}

int dragon_gpu_advance_split(dragon_grid* h, double interval, int check_cfl, dragon_advance_stats* st) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    int rc = split_unsupported(h);
    if (rc) return rc;
    h->split_mode = h->dim >= 2;
    rc = advance_impl(h, interval, 0, check_cfl ? 1 : 0, st);
    h->split_mode = false;
    return rc;
}

void* dragon_gpu_stream(dragon_grid* h) { return h ? (void*)h->stream : nullptr; }

int dragon_gpu_device_state(dragon_grid* h, double** prim, long long* plane, long long* pitch) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (prim) *prim = h->w[h->cur];
    if (plane) *plane = h->cg.plane;
    if (pitch) *pitch = h->cg.pitch;
    return 0;
}

unsigned long long dragon_gpu_launch_count(const dragon_grid* h) { return h ? h->launches : 0; }

int dragon_gpu_debug_set(dragon_grid* h, int key, int value) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    switch (key) {
        case DRAGON_GPU_DEBUG_STALL_CTA: h->dbg_stall_cta = value < 0 ? -1 : value; return 0;
        case DRAGON_GPU_DEBUG_NO_COOP: h->dbg_no_coop = value != 0; return 0;
        default: return fail(DRAGON_GPU_EINVAL, "unknown debug key");
    }
}

int dragon_gpu_profile_enable(dragon_grid* h, int on) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    collect_profile(h);
    h->prof = on != 0;
    return 0;
}

int dragon_gpu_profile_read(dragon_grid* h, double* ms_total, long long* launches, int reset) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    collect_profile(h);
    if (ms_total) *ms_total = h->prof_ms;
    if (launches) *launches = h->prof_n;
    if (reset) { h->prof_ms = 0; h->prof_n = 0; }
    return 0;
}

int dragon_gpu_initialize_B_fields(dragon_grid* h) {
    if (h && h->adv.pending) return fail(DRAGON_GPU_EINVAL, "an asynchronous advance is in flight");
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (!(h->mhd && h->dim >= 2)) return fail(DRAGON_GPU_EINVAL, "grid has no face-centred B");
    int rc = dragon_gpu_apply_boundary(h);
    if (rc) return rc;
    rc = launch_init_body_fields(h->cg, h->fg, h->w[h->cur], h->B[h->cur], h->stream);
    if (rc) return fail(DRAGON_GPU_ECUDA, "initialize_B_fields launch failed");
    h->launches++;
    h->imax_valid = false;
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int dragon_gpu_newton_stats(dragon_grid* h, dragon_newton_stats* out, int reset) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    if (out) {
        *out = h->ntot;
        if (h->nlog_count) {
            unsigned long long seen = 0;
            CK(cudaMemcpyAsync(&seen, h->nlog_count, sizeof(seen), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            out->log_seen = seen;
            const unsigned long long kept = (seen + h->nlog_stride - 1) / h->nlog_stride;
            out->log_stored = kept < (unsigned long long)h->nlog_cap ? kept : (unsigned long long)h->nlog_cap;
        }
    }
    if (reset) h->ntot = dragon_newton_stats{};
    return 0;
}

int dragon_gpu_newton_log_enable(dragon_grid* h, long long capacity, int stride) {
    if (!h || capacity < 0 || stride < 1) return fail(DRAGON_GPU_EINVAL, "invalid log arguments");
    CK(cudaStreamSynchronize(h->stream));
    if (h->nlog_rows) cudaFree(h->nlog_rows);
    if (h->nlog_count) cudaFree(h->nlog_count);
    h->nlog_rows = nullptr;
    h->nlog_count = nullptr;
    h->nlog_cap = 0;
    h->nlog_stride = 1;
    if (capacity == 0) return 0;
    CK(cudaMalloc(&h->nlog_rows, sizeof(double) * kNewtonLogCols * capacity));
    CK(cudaMalloc(&h->nlog_count, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(h->nlog_count, 0, sizeof(unsigned long long), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->nlog_cap = capacity;
    h->nlog_stride = stride;
    return 0;
}

static long long nlog_stored(dragon_grid* h, int* rc) {
    *rc = 0;
    if (!h->nlog_count) return 0;
    unsigned long long seen = 0;
    if (cudaMemcpyAsync(&seen, h->nlog_count, sizeof(seen), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        *rc = fail(DRAGON_GPU_ECUDA, "reading the log counter failed");
        return 0;
    }
    const unsigned long long kept = (seen + h->nlog_stride - 1) / h->nlog_stride;
    return kept < (unsigned long long)h->nlog_cap ? (long long)kept : h->nlog_cap;
}

int dragon_gpu_newton_log_read(dragon_grid* h, double* host_rows, long long max_rows, long long* n_out) {
    if (!h || max_rows < 0 || (max_rows > 0 && !host_rows)) return fail(DRAGON_GPU_EINVAL, "invalid arguments");
    int rc;
    long long n = nlog_stored(h, &rc);
    if (rc) return rc;
    if (n > max_rows) n = max_rows;
    if (n > 0) {
        CK(cudaMemcpyAsync(host_rows, h->nlog_rows, sizeof(double) * kNewtonLogCols * n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (n_out) *n_out = n;
    return 0;
}

int dragon_gpu_newton_log_device(dragon_grid* h, const double** rows, long long* n_stored) {
    if (!h) return fail(DRAGON_GPU_EINVAL, "null handle");
    int rc;
    const long long n = nlog_stored(h, &rc);
    if (rc) return rc;
    if (rows) *rows = h->nlog_rows;
    if (n_stored) *n_stored = n;
    return 0;
}

int dragon_gpu_grid_set_mlp(dragon_grid* h, const dragon_mlp* m) {
    if (!h || !m) return fail(DRAGON_GPU_EINVAL, "null argument");
    const MlpNet* net = dragon_mlp_packed_net(const_cast<dragon_mlp*>(m));
    if (!net) return fail(DRAGON_GPU_ECUDA, "packing the network failed");
    if (!h->mlp_dev) CK(cudaMalloc(&h->mlp_dev, sizeof(MlpNet)));
    CK(cudaMemcpyAsync(h->mlp_dev, net, sizeof(MlpNet), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

}  // extern "C"
