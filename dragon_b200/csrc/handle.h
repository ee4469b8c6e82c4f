// Internal: the grid handle behind dragon_grid* and the runtime helpers the
// batched step (batch.cu) shares with the single-grid runtime (runtime.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "../../include/dragon_gpu.h"
#include "../../include/dragon_learned.h"
#include "boundary.cuh"
#include "scratch.h"

namespace dgpu {
struct MlpNet;
}
struct dragon_user_fill;
struct HoardState;

// A user ghost fill bound to one entry of a grid's boundary list
// (dragon_gpu_set_user_fill): the compiled fill, the faces whose ghost cells it
// visits, whether it visits their corners, and its parameters on the device.
struct UserFillBinding {
    dragon_user_fill* fill = nullptr;
    int fill_faces = 0;
    int corners = 1;
    double* dparams = nullptr;
    int nparams = 0;
};

// The device advance loop between its first batch and its completion
// (dragon_gpu_advance_steps_async / dragon_gpu_advance_wait).
struct AdvanceState {
    bool pending = false;
    int cur0 = 0;         // buffer step 0 reads
    long long k = 0;      // advance-local index of the next step to enqueue
    int retries = 0;
    double remaining = 0;
    int max_steps = 0;
};

struct dragon_grid {
    int dim = 0;
    int n[3] = {1, 1, 1};
    int g = 0;
    double d[3] = {0, 0, 0};
    int nf = 5;
    bool mhd = false;
    dragon_config cfg{};
    int solver = dgpu::RS_HLLC;
    dgpu::Geo cg{}, fg{};
    double* w[2] = {nullptr, nullptr};
    double* B[2] = {nullptr, nullptr};
    int cur = 0;
    dgpu::StepCtl* ctl = nullptr;
    dgpu::StepCtl* hctl = nullptr;
    dgpu::BCEntry* dbcs = nullptr;
    int nbc = 0;
    std::vector<dgpu::BCEntry> hbcs;
    double* stage = nullptr;
    size_t stage_elems = 0;
    cudaStream_t stream = nullptr;
    bool imax_valid = false;
    unsigned long long launches = 0;
    // intermediates of the 2D MHD step
    dgpu::MhdScratch mhd_s{};
    double* mhd_buf = nullptr;
    // intermediates of the 3D hydro step
    dgpu::Hydro3DScratch h3_s{};
    // the last unsplit_step committed (a sharded step may still be undone)
    bool can_rollback = false;
    // Strang-split path: third state buffer and the sweep-order counter (Grid::sweep_step)
    double* wsplit = nullptr;
    long long sweep_step = 0;
    bool split_mode = false;
    // intermediates of the 3D MHD step
    dgpu::Mhd3DScratch m3_s{};
    double* m3_buf = nullptr;
    double* h3_buf = nullptr;
    // step-kernel timing (dragon_gpu_profile_*)
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending;
    double prof_ms = 0;
    long long prof_n = 0;
    // exact solver: converged-solve log, learned-guess network, counters
    double* nlog_rows = nullptr;
    unsigned long long* nlog_count = nullptr;
    long long nlog_cap = 0;
    int nlog_stride = 1;
    dgpu::MlpNet* mlp_dev = nullptr;
    dragon_newton_stats ntot{};
    AdvanceState adv{};
    // CTAs of the cooperative prologue that fit on the device (hydro, MHD); 0: not yet known, -1: none
    int coop_cap[2] = {0, 0};
    // test hooks (dragon_gpu_debug_set): CTA of the cooperative prologue that
    // returns before its first grid barrier (-1: none); take the prologue path
    // of devices without cooperative launch
    int dbg_stall_cta = -1;
    bool dbg_no_coop = false;
    // user ghost fills: entries of the compiled list that are device user
    // fills (in list order), their bindings (indexed by entry), and the length
    // of the caller's list (the compiled list may start with an implicit Outflow)
    std::vector<int> user_entries;
    std::vector<UserFillBinding> ufill;
    int caller_entries = 0;
    // TMA tensor maps of the two state buffers for the fused 2D hydro kernels
    // (FP64, mixed), encoded on first use
    CUtensorMap tmap[2][2];
    bool tmap_ok[2][2] = {{false, false}, {false, false}};
    // output snapshots in flight (hoard.cu), created on first use
    HoardState* hoard = nullptr;
    // global index of cell (0, 0, 0) as user fills see it (dragon_gpu_set_origin)
    int origin[3] = {0, 0, 0};
};

namespace dgpu_rt {

// Step arguments for a step that reads buffer c and accumulates its CFL max into slot_out.
dgpu::StepArgs step_args(const dragon_grid* h, int slot_out);
// Enqueues the step kernels reading buffer c, writing c ^ 1 (the unsplit step).
int launch_step(dragon_grid* h, int c);
// Enqueues the interior CFL maximum of buffer c into vmax[slot].
int launch_interior_cfl(dragon_grid* h, int c, int slot);
// Host mirror of the control block <-> device (header only / all, synchronising).
int push_ctl(dragon_grid* h);
int pull_ctl(dragon_grid* h);
int zero_slot(dragon_grid* h, int slot);
void reset_ctl(dragon_grid* h, double remaining, int max_steps, int check_cfl);
void add_newton(dragon_grid* h, const dgpu::StepCtl& c);
const char* stage_name(int s);
// Enqueues the bound user fill of compiled boundary entry `entry` on state
// buffer c (w_buf overrides the cell array); skipped on the device once the
// advance is done or failed (user_fill.cu).
int launch_user_fill(dragon_grid* h, int c, int entry, double* w_buf);
// Releases a handle's user-fill bindings (their device parameters).
void clear_user_fills(dragon_grid* h);
// Waits for a handle's output snapshots and frees their buffers (hoard.cu).
void hoard_release(dragon_grid* h);

}  // namespace dgpu_rt
