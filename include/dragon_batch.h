/*
 * dragon_batch.h — many independent DRAGON grids advanced together.
 *
 * The reference advances each Grid on its own (Grid::advance, Hydro/CFL/CFL.cpp:151-213)
 * and runs independent problems one after another or on separate threads.
 * A batch groups existing grid handles (dragon_gpu.h) of uneven sizes, each
 * keeping its own configuration, boundary list, CFL dt, step count and
 * halve-and-retry on failure, and advances all of them with one persistent
 * kernel per step: CTAs take work items from a device queue (each grid's
 * ghost fill + CFL dt, then its step tiles in dependency order), and the
 * per-step launches are captured in a CUDA graph. After
 * dragon_gpu_batch_advance_steps every FP64 grid holds exactly the state its
 * own dragon_gpu_advance_steps would have produced (mixed members: below).
 *
 * Supported members: 1D hydro grids (HLLC / HLLX or the exact solver) and 2D
 * MHD grids (HLLD / HLLX); all 1D members share one solver, and all members
 * one precision: FP64 (dragon_config.precision 0) or mixed FP32/FP64 (1). A
 * mixed batch's 1D members end exactly where their own mixed advance ends, its
 * 2D MHD members to FP32 rounding of it (the compiler may fuse FP32
 * multiply-adds differently in the batched kernel). No counterpart in the
 * reference (its batch is a loop over grids).
 */
#ifndef DRAGON_BATCH_H
#define DRAGON_BATCH_H

#include "dragon_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dragon_batch dragon_batch;

/* Launch shape of the batched step, chosen by dragon_gpu_batch_autotune or
 * set by the caller. */
typedef struct dragon_batch_tuning {
    int tile_1d;      /* cells per 1D work item: 126 or 254 (FP64 batches; mixed: always 254) */
    int ctas_per_sm;  /* resident CTAs of the persistent kernel per SM (1..8, capped by occupancy) */
    int order;        /* queue order: 0 phase-major (all grids' phase k before phase k+1, 1D tiles after
                         the first MHD phase), 1 1D grids first, 2 largest grids first within each phase,
                         3 wavefront: 1D grids first, then the 2D MHD grids in groups of `wave`, group g's
                         phase k queued with group g+1's phase k-1 (a group's intermediates are reused
                         while they are still in L2) */
    int graph_steps;  /* steps captured per CUDA graph */
    int mhd_tiles;    /* 32 x 8 tiles of a 2D MHD phase per work item: 1, 2, 4 or 8 (0 reads as 1; default 8) */
    int wave;         /* order 3: 2D MHD grids per wavefront group, 1..64 (0 reads as 1) */
} dragon_batch_tuning;

typedef struct dragon_batch_stats {
    int steps;                 /* steps every member advanced */
    int retries;               /* halvings after failed member steps */
    int graph_replays;
    long long work_items;      /* per step */
    unsigned long long spin_timeouts; /* dependency waits that gave up (0 on a healthy run) */
    double replay_ms;          /* device time of the graph replays (CUDA events) */
} dragon_batch_stats;

int dragon_gpu_batch_create(dragon_batch** out);
/* Members stay owned by the caller and must outlive the batch. */
int dragon_gpu_batch_destroy(dragon_batch* b);
/* Adds a grid; index receives its position in the batch. */
int dragon_gpu_batch_add_instance(dragon_batch* b, dragon_grid* g, int* index);
int dragon_gpu_batch_size(const dragon_batch* b);
int dragon_gpu_batch_set_tuning(dragon_batch* b, const dragon_batch_tuning* t);
int dragon_gpu_batch_get_tuning(const dragon_batch* b, dragon_batch_tuning* t);
/* Times every candidate launch shape for steps_per_candidate steps on the
 * members' current states (restored afterwards) and keeps the fastest. */
int dragon_gpu_batch_autotune(dragon_batch* b, int steps_per_candidate, dragon_batch_tuning* best, double* best_ms);
/* Every member takes nsteps CFL-limited steps (dragon_gpu_advance_steps). */
int dragon_gpu_batch_advance_steps(dragon_batch* b, int nsteps, dragon_batch_stats* st);

#ifdef __cplusplus
}
#endif

#endif /* DRAGON_BATCH_H */
