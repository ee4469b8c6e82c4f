/*
 * dragon_gpu.h — C ABI of the B200 unsplit Godunov update for DRAGON grids.
 *
 * One handle is one grid (DRAGON's Grid1D / Grid2D / Grid3D) resident in GPU
 * memory. The entry points replace, one for one, the calls DRAGON's pthread
 * subgrid path makes on a grid; each declaration names the reference
 * interface it stands in for (paths are relative to the DRAGON source tree).
 *
 * Conventions
 *   - Every function returns 0 on success or a DRAGON_GPU_E* code; the message
 *     of the last failure on the calling thread is dragon_gpu_last_error().
 *   - Host arrays use the reference's own memory order: the ghost-padded array
 *     of ExtendedArray{1,2,3}D (Hydro/ExtendedArray/ExtendedArray.hpp:75,125;
 *     last index fastest, ghosts included), NF doubles per cell in the order
 *     of PrimitiveState (FluidElement/FluidElement.hpp:34-43):
 *     rho, p, vx, vy, vz, and for MHD Bx, By, Bz (NF = 5 or 8).
 *   - Face-centred B (MHD, 2D/3D) uses the (n+1)-per-dimension padded face
 *     arrays of Grid2D/Grid3D (Hydro/Grid.hpp:65,107) with 3 doubles per face.
 *   - A handle is used by one host thread at a time; distinct handles may run
 *     concurrently (each owns a CUDA stream).
 */
#ifndef DRAGON_GPU_H
#define DRAGON_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DRAGON_GPU_OK 0
#define DRAGON_GPU_EINVAL 1       /* bad argument */
#define DRAGON_GPU_ECUDA 2        /* CUDA runtime failure */
#define DRAGON_GPU_ESTEP 3        /* step produced an unphysical / non-finite state or no physical flux */
#define DRAGON_GPU_ECFL 4         /* CFL limit failed: max signal speed is zero */
#define DRAGON_GPU_EDT 5          /* retried step fell below Timestep_Tolerance */
#define DRAGON_GPU_EUNSUPPORTED 6 /* configuration not built */

/* Runtime form of DRAGON/Config.h's switches (Config.h:26-90). Ids equal the
 * reference's macro values: RIEMANN_EXACT 0, HLL 1, HLLC 2, HLLD 3, HLLE 4,
 * HLLX 5, ROE 6; LIMITER_MINMOD 0, MC 1, VANLEER 2, SUPERBEE 3, VANALBADA 4;
 * CFL_MAX 0, CFL_ADD 1, p > 1 for the p-norm; CT_CONSV_TOTAL_E 0, THERMAL 1,
 * BETA_GATED 2. */
typedef struct dragon_config {
    int mhd;              /* 0 hydro, 1 MHD (the reference's #define MHD) */
    int riemann;          /* RIEMANN_DEFAULT */
    int limiter;          /* MUSCL_DEFAULT_LIMITER */
    int cfl;              /* CFL_CALCULATION */
    int ct_energy;        /* CT_ENERGY_CONSV */
    int exact_max_iters;  /* ExactRiemann_MaxIters (6) */
    double exact_tol;     /* ExactRiemann_Tolerance (1e-12) */
    double cfl_coeff;     /* CFL_coeff (0.3) */
    double timestep_tol;  /* Timestep_Tolerance (1e-14) */
    int precision;        /* 0: FP64 throughout (bit-faithful), 1: mixed FP32/FP64 */
    int exact_guess;      /* start of the exact solver's Newton iteration: 0 the reference's
                             (pL + pR) / 2 (Exact.cpp:47), 1 adaptive PVRS / two-rarefaction /
                             two-shock, 2 learned (dragon_learned.h; 3D grids), 3 a measurement
                             arm: the converged star pressure of an uncounted first solve */
    int perfect_guess_err_exp; /* exact_guess 3: the start is that pressure times (1 +- 10^-e)
                             for e > 0 (+ where pL >= pR), exactly it for e <= 0 */
    int reserved[5];
} dragon_config;

/* Fills the reference's shipped defaults for the given physics mode. */
void dragon_gpu_default_config(dragon_config* cfg, int mhd);

/* Boundary list entry (DRAGON/Boundary/Boundary.hpp:158-229). type: 0 Outflow,
 * 1 Outflow::Gated, 2 Fixed, 3 Reflective, 4 Periodic, 5 Ignore, 6 a user
 * GhostFill compiled for the device (DRAGON_BC_USER; bind its fill with
 * dragon_gpu_set_user_fill). faces is the bit mask of Boundary::face_mask
 * (X- 1, X+ 2, Y- 4, Y+ 8, Z- 16, Z+ 32); state is Fixed's primitive state
 * (NF values). */
#define DRAGON_BC_USER 6
typedef struct dragon_bc_desc {
    int type;
    int faces;
    int corners;
    int reserved;
    double state[8];
} dragon_bc_desc;

typedef struct dragon_step_status {
    int code;              /* DRAGON_GPU_OK or DRAGON_GPU_ESTEP / ECFL */
    int stage;             /* 1 predictor flux, 2 final flux, 3 non-finite, 4 unphysical, 5 CFL */
    long long cell;        /* linear padded index of the first failing cell/face */
    double dt;             /* dt of the (last) attempt */
} dragon_step_status;

typedef struct dragon_advance_stats {
    int steps;                      /* successful steps */
    int retries;                    /* halvings after a failed step (CFL.cpp:198-208) */
    double last_dt;
    double time_advanced;
    unsigned long long pivots_exact;      /* verify_and_fallback pivots to the exact solver */
    unsigned long long hlld_to_hlle;      /* HLLD star states replaced by HLLE */
    unsigned long long newton_iters;      /* exact solver Newton iterations */
    unsigned long long exact_calls;       /* exact solver star-pressure solves */
    unsigned long long trrs;              /* two-rarefaction closed forms */
    unsigned long long muscl_first_order; /* MUSCL first-order fallbacks */
    dragon_step_status failure;           /* last failure seen (code 0 if none) */
} dragon_advance_stats;

typedef struct dragon_grid dragon_grid;

/* Grid1D(size, dx, ghosts) / Grid2D(nx, ny, dx, dy, ghosts) /
 * Grid3D(nx, ny, nz, dx, dy, dz, ghosts) (Hydro/Grid.hpp:46,70,112;
 * Hydro/Godunov/Splitting.cpp:23-61): ghosts are raised to the minimum the
 * scheme needs (2 hydro, 3 MHD) exactly like validGhosts. Unused extents are
 * ignored. Replaces DistGrid{1,2,3}D's constructors (Refinement/DistGrid.cpp:41-111). */
int dragon_gpu_grid_create(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts,
                           const dragon_config* cfg, dragon_grid** out);
int dragon_gpu_grid_destroy(dragon_grid* g);
/* getGhosts() / getSize*() (Hydro/Grid.hpp:54,79,121) */
int dragon_gpu_grid_info(const dragon_grid* g, int* dim, int* n3, int* ghosts, int* nfields);
/* Number of doubles in the padded primitive array and in the padded face-B array. */
size_t dragon_gpu_prim_count(const dragon_grid* g);
size_t dragon_gpu_faceB_count(const dragon_grid* g);

/* Bulk access standing in for operator[] over the whole padded array
 * (Hydro/Grid.hpp:52-53,77-78,119-120) and _B() (Hydro/Grid.hpp:83,125);
 * the transfers DistGrid::pushToChildren / loadFromChildren do
 * (Refinement/DistGrid.cpp:115-289). Synchronous with respect to the host. */
int dragon_gpu_upload_prim(dragon_grid* g, const double* host);
int dragon_gpu_download_prim(dragon_grid* g, double* host);
int dragon_gpu_upload_faceB(dragon_grid* g, const double* host);
int dragon_gpu_download_faceB(dragon_grid* g, double* host);

/* grid.boundary = ... (Hydro/Grid.hpp:35; Boundary/BoundaryList.hpp:22-105). */
int dragon_gpu_set_boundary(dragon_grid* g, const dragon_bc_desc* list, int n);
/* boundary.apply(grid) (Boundary/BoundaryList.hpp:79-93) */
int dragon_gpu_apply_boundary(dragon_grid* g);
/* Entries of the compiled list (the implicit Outflow first when some face is
 * uncovered, then the caller's entries in order), and one contiguous range of
 * them applied alone: a host that owns custom GhostFill elements (passed here
 * as Ignore entries covering their faces) runs its own fills between ranges,
 * in list order (BoundaryList.hpp:79-93). */
int dragon_gpu_boundary_entries(const dragon_grid* g);
int dragon_gpu_apply_boundary_range(dragon_grid* g, int first, int count);

/* A user GhostFill element (Boundary/GhostFill.hpp:16-30; the Jet of
 * Examples/CollidingFlows/Jets/Jets.hpp:12-39 is the reference's example)
 * written as a CUDA device function and compiled for the device with NVRTC:
 *
 *     __device__ void NAME(const dragon_fill_ctx& c, int i, int j, int k);
 *
 * is called once per ghost cell (i, j, k) of the faces it is bound to fill
 * (interior coordinates: ghosts are negative or >= n), with c.axis / c.side
 * the face. dragon_fill_ctx gives the padded state: c.get(f, i, j, k) /
 * c.set(f, i, j, k, v) on primitive field f (DRAGON_RHO, DRAGON_P,
 * DRAGON_VX..VZ, DRAGON_BX..BZ), c.getB / c.setB on face B (MHD 2D / 3D),
 * c.n[3], c.g, c.d[3], c.dim, c.params[0 .. c.nparams) and c.off[3], the
 * global index of the grid's cell (0, 0, 0) (non-zero for the slab of a
 * distributed grid: dragon_gpu_set_origin; a global x position is
 * (c.off[0] + i + 0.5) * c.d[0]). One thread walks
 * the ghost layers of a transverse point of one face outward (layer 1 first),
 * transverse points and the two faces of an axis run in parallel, the axes
 * one after another; a fill writes only the ghost cell (and its face B) it is
 * called for. Compiled without FMA contraction, with IEEE division and square
 * root, like the library's FP64 kernels. A failed compile returns
 * DRAGON_GPU_EINVAL with NVRTC's log as the error message; without NVRTC,
 * DRAGON_GPU_ECUDA. A fill may be bound to any number of grids. */
typedef struct dragon_user_fill dragon_user_fill;
int dragon_gpu_user_fill_create(const char* source, const char* function, dragon_user_fill** out);
int dragon_gpu_user_fill_destroy(dragon_user_fill* f);
/* NVRTC's log of the compile (warnings), "" if none. */
const char* dragon_gpu_user_fill_log(const dragon_user_fill* f);
/* Binds fill f to entry `entry` (an index into the list last passed to
 * dragon_gpu_set_boundary, whose type must be DRAGON_BC_USER): it fills the
 * ghost cells of fill_faces (a face mask; the reference's Jet fills its jet
 * face while its GhostFill faces mask is 0), with their corner ghosts when
 * corners != 0, reading params (copied to the device). The grid runs it at
 * the entry's place in BoundaryList::apply order (BoundaryList.hpp:79-93) in
 * every ghost fill and inside the device advance loop, with no host
 * round trip. dragon_gpu_set_boundary drops the bindings. f must stay alive
 * while it is bound: destroy it only after the grids it is bound to are
 * destroyed or have had their boundary list set again. */
int dragon_gpu_set_user_fill(dragon_grid* g, int entry, dragon_user_fill* f, int fill_faces, int corners,
                             const double* params, int nparams);
/* The global index of the grid's cell (0, 0, 0), as user fills see it in
 * dragon_fill_ctx::off: a DistGrid child's offset in its parent
 * (Refinement/DistGrid.cpp:41-111 computes it per child); 0 for a whole grid. */
int dragon_gpu_set_origin(dragon_grid* g, int i0, int j0, int k0);
/* Grid::initialize_B_fields (MHD/B_fields.cpp:117-149) */
int dragon_gpu_initialize_B_fields(dragon_grid* g);

/* CFL::cfl_time (Hydro/CFL/CFL.cpp:88-137) on the current ghosts. */
int dragon_gpu_cfl_time(dragon_grid* g, double* dt_out);
/* Grid::unsplit_step(dt) (Hydro/Godunov/Unsplit.cpp:28-206, Splitting.cpp:100-115):
 * one step with the caller's dt on the current ghosts; on failure nothing is
 * committed and st describes the failure (the reference throws). */
int dragon_gpu_unsplit_step(dragon_grid* g, double dt, dragon_step_status* st);
/* Grid::advance(dt, check_cfl) (Hydro/CFL/CFL.cpp:151-213): the whole
 * sub-cycling loop — ghost fill, CFL dt, step, halve-and-retry on failure —
 * runs on the device; DistGrid's thread fan-out and all-or-nothing commit
 * (Refinement/DistGrid.cpp:292-304, DRAGONWING/Multithreading/pthread_parallel.cpp:84-152)
 * become one kernel sequence with a device error word. */
int dragon_gpu_advance(dragon_grid* g, double interval, int check_cfl, dragon_advance_stats* st);
/* advance by a fixed number of CFL-limited steps (the interval is unbounded). */
int dragon_gpu_advance_steps(dragon_grid* g, int nsteps, dragon_advance_stats* st);
/* dragon_gpu_advance_steps in two halves: _async enqueues the first batch of
 * steps on the handle's stream and returns without waiting for the device;
 * _wait reads the outcome, runs any retry and further batches, and fills st.
 * Between the two the handle takes no other call. */
int dragon_gpu_advance_steps_async(dragon_grid* g, int nsteps);
int dragon_gpu_advance_wait(dragon_grid* g, dragon_advance_stats* st);
/* Grid::split_step(dt) (Hydro/Godunov/Splitting.cpp:118-217): the Strang
 * sequence of one-dimensional Godunov sweeps, the order alternating with the
 * grid's sweep counter (2D: XYX / YXY; 3D: the six cyclic and anticyclic
 * orders); 1D grids take the unsplit step, as the reference does. Hydro grids,
 * FP64. No commit on failure. */
int dragon_gpu_split_step(dragon_grid* g, double dt, dragon_step_status* st);
/* Grid::advance_split(dt, check_cfl) (Hydro/CFL/CFL.cpp:160-184): the advance
 * loop around split_step. */
int dragon_gpu_advance_split(dragon_grid* g, double interval, int check_cfl, dragon_advance_stats* st);

/* A grid split across devices (the role of DistGrid's children,
 * Refinement/DistGrid.cpp:58-346): copies of whole layers along `axis`
 * between the current state and a contiguous buffer, for the halo exchange.
 * The layers are [first, first + layers) in interior coordinates (ghost
 * layers negative or >= n); the transverse axes span the padded extent when
 * `corners` is set, else their interior (a GhostFill's corner flag,
 * Boundary/GhostFill.hpp:28). faces = 0 selects the cell-centred fields,
 * faces = 1 the face-centred B (n + 1 positions per axis, 3 components; MHD
 * 2D/3D). buf holds halo_size doubles ordered field, layer, transverse (last
 * axis fastest), in device memory when buf_on_device, else host memory. */
int dragon_gpu_halo_size(const dragon_grid* g, int axis, int layers, int faces, int corners, long long* count);
int dragon_gpu_halo_pack(dragon_grid* g, int axis, int first, int layers, int faces, int corners, double* buf,
                         int buf_on_device);
int dragon_gpu_halo_unpack(dragon_grid* g, int axis, int first, int layers, int faces, int corners, const double* buf,
                           int buf_on_device);
/* Undoes the last unsplit_step if nothing touched the grid since (its input
 * buffer is intact): the all-or-nothing commit of a step taken by several
 * devices together (DistGrid.cpp:292-304). */
int dragon_gpu_step_rollback(dragon_grid* g);

/* The CUDA stream the handle's kernels run on (cudaStream_t). */
void* dragon_gpu_stream(dragon_grid* g);
/* Device pointer to the current primitive planes (SoA, NF planes of
 * dragon_gpu_plane_stride doubles; layout described in the design notes). */
int dragon_gpu_device_state(dragon_grid* g, double** prim, long long* plane_stride, long long* pitch);
/* Number of kernels this handle has launched since creation. */
unsigned long long dragon_gpu_launch_count(const dragon_grid* g);
/* Step-kernel timing: when enabled, CUDA events bracket every step-kernel
 * launch on the handle's stream; read returns the summed milliseconds and the
 * number of timed launches since the last reset (no reference counterpart:
 * measurement hook for the roofline). */
int dragon_gpu_profile_enable(dragon_grid* g, int on);
int dragon_gpu_profile_read(dragon_grid* g, double* ms_total, long long* launches, int reset);

/* Test hooks (no reference counterpart). DRAGON_GPU_DEBUG_STALL_CTA: CTA
 * `value` of every following cooperative ghost-fill launch (2D / 3D grids)
 * returns before its first grid barrier, so the others' bounded barrier wait
 * runs out and the advance fails with DRAGON_GPU_ECUDA; value < 0 turns it
 * off. DRAGON_GPU_DEBUG_NO_COOP: value != 0 makes the ghost fill take the
 * path of devices without cooperative launch (one launch per pass). */
#define DRAGON_GPU_DEBUG_STALL_CTA 1
#define DRAGON_GPU_DEBUG_NO_COOP 2
int dragon_gpu_debug_set(dragon_grid* g, int key, int value);

/* CFL time step of a state the caller already holds on the device, without
 * allocating anything (no counterpart in the reference: it serves callers
 * that may not allocate device memory after start-up, such as applications
 * that hand all GPU memory to their own pool, or loops that cannot afford the
 * device-wide synchronisation of cudaMalloc/cudaFree). The state uses this
 * library's layout: NF planes of plane_stride doubles, each a ghost-padded
 * array with rows of `pitch` doubles (the last index contiguous), as
 * dragon_gpu_device_state reports it. The result equals dragon_gpu_cfl_time's
 * for the same state and configuration (cfl = CFL_CALCULATION, cfl_coeff =
 * CFL_coeff). stream is a cudaStream_t (NULL for the default stream); the
 * call returns once dt_out is written.
 * Limits: working memory is one fixed ~128 KB array inside the library, kept
 * on every GPU that loads it until the process exits; grids may have at most
 * 16382 cells along x (2D/3D) or 16777214 cells (1D), larger ones are
 * rejected with DRAGON_GPU_EINVAL. The first call on each device looks up the
 * array's device address, so make it before any CUDA stream capture. All
 * calls share the array: calls that overlap on the GPU race, so serialise
 * them. */
int dragon_gpu_cfl_time_noalloc(int dim, int nx, int ny, int nz, int ghosts, int mhd, const double* d_prim,
                                long long plane_stride, long long pitch, double dx, double dy, double dz, int cfl,
                                double cfl_coeff, void* stream, double* dt_out);

/* ---- Output and restart from device buffers ------------------------------
 * Replaces DRAGONHOARD::writeToFile and DRAGONHOARD::loadFromFile
 * (DRAGONHOARD/DragonHoard.hpp:16-33; HDF5Output.cpp:103-528,
 * HDF5Restart.cpp:61-377). A file holds the reference's layout and keys
 * (HDF5_Attrs.hpp:14-59): int and double attributes format_version (1),
 * write_option, dim, MHD, ng, nx[, ny, nz], dx[, dy, dz], cycle, time on the
 * root group, and datasets /fluid/rho, /fluid/v/{x,y,z}, /fluid/p, /fluid/E,
 * /fluid/momentum/{x,y,z}, /fluid/B/{x,y,z}, /fluid/Bf/{x,y,z} as the options
 * select them, flattened x fastest (HDF5Output.cpp:308) with dimensions
 * {nz, ny, nx}. Files are HDF5 (superblock 0, chunked + deflate or
 * contiguous), written without the HDF5 library. */
typedef struct {
    int write_option; /* HDF5_WRITE_OPTION (DRAGONHOARD_Config.h:24-28): 1 primitive, 3 primitive + energy,
                         6 conservative, 7 both; default 3 */
    int redundant;    /* HDF5_REDUNDANT_VALS_OPTION (:31-35): 0 omit, 1 float, 2 double; default 1 */
    int compression;  /* HDF5_COMPRESSION_LEVEL (:22): deflate level (1-9) of chunked datasets; <= 0 writes
                         them contiguous and uncompressed; default 4 */
    int ghosts;       /* WRITE_GHOSTS_TO_FILE (:32): nonzero writes the ghost layers too; default 0 */
    int threads;      /* host threads that compress chunks; 0: every core */
    int reserved[3];
} dragon_hoard_opts;

void dragon_gpu_hoard_default_opts(dragon_hoard_opts* o);
/* Writes the grid's current state to `path` (the full file name) and returns
 * when the file is complete. */
int dragon_gpu_hoard_write(dragon_grid* g, double t, int cycle, const char* path, const dragon_hoard_opts* o);
/* Snapshots the current state on the grid's stream and returns: the device
 * packs the datasets into one of two staging buffers, a copy stream downloads
 * it while later steps run, and a host thread writes the file. A third call
 * waits for the oldest snapshot's file first; if that file failed, the call
 * returns its failure (this call's snapshot is taken all the same). Later
 * steps and boundary calls do not change a snapshot already taken. */
int dragon_gpu_hoard_write_async(dragon_grid* g, double t, int cycle, const char* path, const dragon_hoard_opts* o);
/* Waits for every file of g in flight; returns the first failure among them. */
int dragon_gpu_hoard_wait(dragon_grid* g);
/* Restart (HDF5Restart.cpp:61-377), after the grid's own files in flight are
 * complete: checks format_version <= 1, dim, MHD
 * and the extents against the grid, then loads dx/dy/dz (the grid's spacing
 * becomes the file's), the cells and (MHD 2D / 3D) face B of the file's
 * range: primitive values when write_option has bit 1, else rho, momentum and
 * E converted to primitive values. Returns *t and *cycle. */
int dragon_gpu_hoard_load(dragon_grid* g, const char* path, double* t, int* cycle);

/* The same file from, and the same restart into, host arrays in this
 * header's host layout (prim: the padded cells with NF values each; faceB:
 * the padded faces with 3 values each, MHD 2D / 3D, else may be NULL) of a
 * grid of `dim` dimensions, extents n3 and `ghosts` ghost layers: what a
 * host-side grid, or the gathered slabs of a distributed grid, writes and
 * restarts from. dragon_hoard_load_host returns the file's spacing in d3. */
int dragon_hoard_write_host(const char* path, int dim, int mhd, const int* n3, int ghosts, const double* d3, double t,
                            int cycle, const double* prim, const double* faceB, const dragon_hoard_opts* o);
int dragon_hoard_load_host(const char* path, int dim, int mhd, const int* n3, int ghosts, double* prim, double* faceB,
                           double* t, int* cycle, double* d3);

/* The HDF5 subset itself, on host arrays (no device involved). */
#define DRAGON_H5_F64 0
#define DRAGON_H5_F32 1
#define DRAGON_H5_I32 2
typedef struct {
    const char* path;  /* absolute, e.g. "/fluid/v/x"; parent groups are created */
    int rank;          /* 1 to 3 */
    long long dims[3]; /* slowest first */
    int type;          /* DRAGON_H5_F64 or DRAGON_H5_F32 */
    const void* data;  /* row-major */
} dragon_h5_dataset;
typedef struct {
    const char* name;
    int type; /* DRAGON_H5_I32 or DRAGON_H5_F64 */
    int ivalue;
    double dvalue;
} dragon_h5_attr;
int dragon_h5_write(const char* file, const dragon_h5_attr* attrs, int nattrs, const dragon_h5_dataset* dsets,
                    int ndsets, int level, int threads);
int dragon_h5_read_attr(const char* file, const char* name, double* value);
/* rank 0 for a scalar; dims3 receives up to three dimensions, slowest first. */
int dragon_h5_dataset_shape(const char* file, const char* path, int* rank, long long* dims3);
/* Reads a dataset converted to double; capacity is out's length in elements. */
int dragon_h5_read(const char* file, const char* path, double* out, long long capacity);

const char* dragon_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DRAGON_GPU_H */
