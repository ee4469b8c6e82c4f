// Ghost fills (DRAGON/Boundary) and the per-step prologue.
//
// A boundary list is compiled on the host into BCEntry records in application
// order: the implicit Outflow over uncovered faces first, then the user's
// entries (BoundaryList.hpp:79-104). Each entry is applied axis by axis (X, Y,
// Z) exactly as the reference's GhostFill::apply loops run, because later
// axes read corner ghosts written by earlier ones; within one axis the two
// sides touch disjoint cells and run in parallel. MHD face-B ghosts follow the
// cell ghosts of the same entry (Outflow.cpp:78-117, Reflective.cpp:99-137,
// Periodic.cpp:311-331, Fixed.cpp:372-406).
#pragma once

#include "grid.cuh"

namespace dgpu {

enum BCType : int { BC_OUTFLOW = 0, BC_OUTFLOW_GATED = 1, BC_FIXED = 2, BC_REFLECTIVE = 3, BC_PERIODIC = 4, BC_IGNORE = 5 };
// Face bits (Boundary.hpp:139-149)
constexpr int FX_NEG = 1, FX_POS = 2, FY_NEG = 4, FY_POS = 8, FZ_NEG = 16, FZ_POS = 32;

struct BCEntry {
    int type;
    int faces;
    int corners;
    int pad;
    double state[8];   // Fixed: primitive state rho, p, vx, vy, vz, Bx, By, Bz
};

struct PrologueArgs {
    double dx, dy, dz;
    double cfl_coeff;
    double tol;
    int cfl;
    int slot_in;        // interior max written by the previous step (or the initial CFL pass)
    int slot_out;       // slot the coming step accumulates into (zeroed here)
    int bookkeeping;    // account for the previous step (advance loop)
    int apply_bc;       // fill ghosts
    int compute_dt;     // compute t1 from the CFL limit
    int nbc;            // entries to apply
    int bc_first;       // first entry to apply
    int stall_cta;      // test hook: this CTA of k_prologue_coop returns before its first barrier (-1: none)
};

// ---------------------------------------------------------------------------
// Cell ghosts of one entry along one axis. The axis index a in 0..dim-1; the
// remaining axes are transverse. Strided over (side, transverse point, ghost
// layer) by the calling threads: tid of nthreads (one CTA in the prologue, a
// whole grid in k_bc_pass).
template <bool MHD>
__device__ void bc_cells_axis(const Geo& G, double* __restrict__ w, const BCEntry& e, int a, long long tid,
                              long long nthreads) {
    const int dim = G.dim, ng = G.g;
    const int na = G.n[a];
    const bool negOn = e.faces & (1 << (2 * a)), posOn = e.faces & (1 << (2 * a + 1));
    const bool periodic = e.type == BC_PERIODIC;
    if (e.type == BC_IGNORE) return;
    if (!negOn && !posOn) return;
    // transverse ranges
    int t0[2] = {0, 0}, tn[2] = {1, 1};
    int ta[2] = {-1, -1};
    int nt = 0;
    for (int b = 0; b < dim; b++) {
        if (b == a) continue;
        ta[nt] = b;
        // 1D grids have no corners; 2D/3D extend transverse ranges into ghosts when corners are on.
        t0[nt] = e.corners ? -ng : 0;
        tn[nt] = e.corners ? G.n[b] + ng : G.n[b];
        nt++;
    }
    const long long span0 = tn[0] - t0[0], span1 = tn[1] - t0[1];
    const long long per_side = span0 * span1 * ng;
    const long long total = 2 * per_side;
    for (long long t = tid; t < total; t += nthreads) {
        const int side = (int)(t / per_side);  // 0 negative, 1 positive
        long long r = t - side * per_side;
        const int gl = (int)(r % ng) + 1;
        r /= ng;
        const int c1 = (int)(r % span1) + t0[1];
        const int c0 = (int)(r / span1) + t0[0];
        if (side == 0 && !negOn) continue;
        if (side == 1 && !posOn) continue;
        int dst[3] = {0, 0, 0}, src[3] = {0, 0, 0};
        if (nt > 0) { dst[ta[0]] = src[ta[0]] = c0; }
        if (nt > 1) { dst[ta[1]] = src[ta[1]] = c1; }
        int sa;
        if (side == 0) {
            dst[a] = -gl;
            if (e.type == BC_REFLECTIVE) sa = gl - 1;
            else if (periodic) sa = na - gl;
            else sa = 0;
        } else {
            dst[a] = na - 1 + gl;
            if (e.type == BC_REFLECTIVE) sa = na - gl;
            else if (periodic) sa = gl - 1;
            else sa = na - 1;
        }
        src[a] = sa;
        long long md, ms;
        if (dim == 1) { md = gidx1(G, dst[0]); ms = gidx1(G, src[0]); }
        else if (dim == 2) { md = gidx2(G, dst[0], dst[1]); ms = gidx2(G, src[0], src[1]); }
        else { md = gidx3(G, dst[0], dst[1], dst[2]); ms = gidx3(G, src[0], src[1], src[2]); }
        Prim<double> v;
        if (e.type == BC_FIXED) {
            v = Prim<double>{e.state[0], e.state[1], e.state[2], e.state[3], e.state[4],
                             e.state[5], e.state[6], e.state[7]};
        } else {
            v = load_prim<MHD>(w, G.plane, ms);
        }
        double* vel = (a == 0) ? &v.vx : (a == 1 ? &v.vy : &v.vz);
        if (e.type == BC_OUTFLOW_GATED) {
            // Outflow.cpp:26,33,50,58: kill inflow through the face
            if (side == 0 && *vel > 0) *vel = 0;
            if (side == 1 && *vel < 0) *vel = 0;
        } else if (e.type == BC_REFLECTIVE) {
            *vel *= -1;
            if constexpr (MHD) {
                v.Bx *= -1; v.By *= -1; v.Bz *= -1;
                double* bn = (a == 0) ? &v.Bx : (a == 1 ? &v.By : &v.Bz);
                *bn *= -1;
            }
        }
        store_prim<MHD>(w, G.plane, md, v);
    }
}

// Face-B ghosts of one entry along one axis. FG is the face geometry (n+1 per
// axis); n_cells the cell extents. One thread per (side, transverse point)
// runs the sequential ghost-layer recurrence.
__device__ inline void bc_faces_axis(const Geo& FG, const int* ncell, double* __restrict__ B, const BCEntry& e, int a,
                                     long long tid, long long nthreads) {
    const int dim = FG.dim, ng = FG.g;
    const int na = ncell[a];
    const bool negOn = e.faces & (1 << (2 * a)), posOn = e.faces & (1 << (2 * a + 1));
    if (e.type == BC_IGNORE) return;
    if (!negOn && !posOn) return;
    int t0[2] = {0, 0}, tn[2] = {0, 0};
    int ta[2] = {-1, -1};
    int nt = 0;
    for (int b = 0; b < dim; b++) {
        if (b == a) continue;
        ta[nt] = b;
        t0[nt] = e.corners ? -ng : 0;
        tn[nt] = e.corners ? ncell[b] + ng : ncell[b];   // inclusive bound
        nt++;
    }
    const long long span0 = tn[0] - t0[0] + 1, span1 = (nt > 1) ? (tn[1] - t0[1] + 1) : 1;
    const long long per_side = span0 * span1;
    const long long plane = FG.plane;
    auto idx = [&](int ia, int c0, int c1) -> long long {
        int q[3] = {0, 0, 0};
        q[a] = ia;
        q[ta[0]] = c0;
        if (nt > 1) q[ta[1]] = c1;
        if (dim == 2) return gidx2(FG, q[0], q[1]);
        return gidx3(FG, q[0], q[1], q[2]);
    };
    const int tr0 = (a == 0) ? 1 : 0;          // first transverse component
    const int tr1 = (a == 2) ? 1 : 2;          // second transverse component
    for (long long t = tid; t < 2 * per_side; t += nthreads) {
        const int side = (int)(t / per_side);
        long long r = t - side * per_side;
        const int c1 = (int)(r % span1) + t0[1];
        const int c0 = (int)(r / span1) + t0[0];
        if (side == 0 && !negOn) continue;
        if (side == 1 && !posOn) continue;
        if (e.type == BC_OUTFLOW || e.type == BC_OUTFLOW_GATED) {
            if (side == 0) {
                for (int gl = 1; gl <= ng; gl++) {
                    long long d = idx(-gl, c0, c1), s0 = idx(0, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = B[c * plane + s0];
                    B[a * plane + d] = 2 * B[a * plane + idx(-gl + 1, c0, c1)] - B[a * plane + idx(-gl + 2, c0, c1)];
                }
            } else {
                long long bn = idx(na, c0, c1), bm = idx(na - 1, c0, c1);
                B[tr0 * plane + bn] = B[tr0 * plane + bm];
                B[tr1 * plane + bn] = B[tr1 * plane + bm];
                for (int gl = 1; gl <= ng; gl++) {
                    long long d = idx(na + gl, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = B[c * plane + bn];
                    B[a * plane + d] = 2 * B[a * plane + idx(na + gl - 1, c0, c1)] - B[a * plane + idx(na + gl - 2, c0, c1)];
                }
            }
        } else if (e.type == BC_REFLECTIVE) {
            if (side == 0) {
                for (int gl = 1; gl <= ng; gl++) {
                    long long d = idx(-gl, c0, c1), s = idx(gl - 1, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = B[c * plane + s] * -1;
                    B[a * plane + d] = B[a * plane + idx(gl, c0, c1)];
                }
            } else {
                long long bn = idx(na, c0, c1), bm = idx(na - 1, c0, c1);
                for (int c = 0; c < 3; c++) B[c * plane + bn] = B[c * plane + bm] * -1;
                for (int gl = 1; gl <= ng; gl++) {
                    long long d = idx(na + gl, c0, c1), s = idx(na - gl - 1, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = B[c * plane + s] * -1;
                    B[a * plane + d] = B[a * plane + idx(na - gl, c0, c1)];
                }
            }
        } else if (e.type == BC_PERIODIC) {
            for (int gl = 1; gl <= ng; gl++) {
                long long d, s;
                if (side == 0) { d = idx(-gl, c0, c1); s = idx(na - gl, c0, c1); }
                else { d = idx(na - 1 + gl, c0, c1); s = idx(gl - 1, c0, c1); }
                for (int c = 0; c < 3; c++) B[c * plane + d] = B[c * plane + s];
            }
        } else if (e.type == BC_FIXED) {
            if (side == 0) {
                B[a * plane + idx(0, c0, c1)] = e.state[5 + a];
                for (int gl = 1; gl <= ng; gl++) {
                    long long d = idx(-gl, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = e.state[5 + c];
                }
            } else {
                for (int gl = 0; gl < ng; gl++) {
                    long long d = idx(na + gl, c0, c1);
                    for (int c = 0; c < 3; c++) B[c * plane + d] = e.state[5 + c];
                }
            }
        }
    }
}

// Step bookkeeping of the previous step (CFL.cpp:188-213), by one thread:
// returns non-zero when this step is not taken (failed or finished advance).
__device__ __forceinline__ int prologue_bookkeeping(StepCtl* ctl, const PrologueArgs& pa) {
    if (ctl->err) return 1;
    if (ctl->done) return 1;
    if (pa.bookkeeping) {
        if (ctl->have_prev) {
            ctl->remaining -= ctl->t1;
            ctl->elapsed += ctl->t1;
            ctl->steps_done += 1;
        }
        ctl->have_prev = 1;
        if (!(ctl->remaining > pa.tol) || (ctl->max_steps > 0 && ctl->steps_done >= ctl->max_steps)) {
            ctl->done = 1;
            return 1;
        }
    }
    return 0;
}

// Whether the bookkeeping ends the advance, computed from the control block
// without writing it (the same operations as prologue_bookkeeping): a prior
// step's dt is taken off the interval first, so remaining - t1 is the value
// the bookkeeping compares.
__device__ __forceinline__ int bookkeeping_done(const StepCtl* ctl, const PrologueArgs& pa) {
    const volatile StepCtl* c = ctl;
    if (c->done) return 1;
    if (!pa.bookkeeping) return 0;
    const bool prev = c->have_prev != 0;
    const double rem = prev ? c->remaining - c->t1 : c->remaining;
    const int steps = prev ? c->steps_done + 1 : c->steps_done;
    return (!(rem > pa.tol) || (c->max_steps > 0 && steps >= c->max_steps)) ? 1 : 0;
}

// Max CFL signal speed over the one-cell ghost ring (CFL.cpp:91,110,125:
// ng = min(1, ghosts)) of a 2D / 3D grid, ring points t0, t0 + stride, ...
template <bool MHD>
__device__ __forceinline__ double ring_speed_max(const Geo& G, const double* __restrict__ w, const PrologueArgs& pa,
                                                 long long t0, long long stride) {
    double m = 0.0;
    if (G.dim == 2) {
        const int nx = G.n[0], ny = G.n[1];
        const long long rows = 2LL * (ny + 2), total = rows + 2LL * nx;
        for (long long r = t0; r < total; r += stride) {
            int i, j;
            if (r < ny + 2) { i = -1; j = (int)r - 1; }
            else if (r < rows) { i = nx; j = (int)(r - (ny + 2)) - 1; }
            else {
                long long q = r - rows;
                if (q < nx) { i = (int)q; j = -1; }
                else { i = (int)(q - nx); j = ny; }
            }
            Prim<double> W = load_prim<MHD>(w, G.plane, gidx2(G, i, j));
            m = speed_max(m, cfl_speed<MHD>(W, pa.cfl, pa.dx, pa.dy, 0.0));
        }
    } else {
        const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
        const long long ey = ny + 2, ez = nz + 2;
        // ring = two i-slabs, then two j-strips per interior i, then two k-cells per interior (i,j)
        const long long nA = 2 * ey * ez, nB = (long long)nx * 2 * ez, nC = (long long)nx * ny * 2;
        for (long long r = t0; r < nA + nB + nC; r += stride) {
            int i, j, k;
            if (r < nA) {
                i = (r < ey * ez) ? -1 : nx;
                long long q = r % (ey * ez);
                j = (int)(q / ez) - 1;
                k = (int)(q % ez) - 1;
            } else if (r < nA + nB) {
                long long q = r - nA;
                i = (int)(q / (2 * ez));
                long long s = q % (2 * ez);
                j = (s < ez) ? -1 : ny;
                k = (int)(s % ez) - 1;
            } else {
                long long q = r - nA - nB;
                i = (int)(q / (2LL * ny));
                long long s = q % (2LL * ny);
                j = (int)(s >> 1);
                k = (s & 1) ? nz : -1;
            }
            Prim<double> W = load_prim<MHD>(w, G.plane, gidx3(G, i, j, k));
            m = speed_max(m, cfl_speed<MHD>(W, pa.cfl, pa.dx, pa.dy, pa.dz));
        }
    }
    return m;
}

// This step's dt from the ring max m and the interior max of the previous
// step's epilogue (CFL.cpp:98-137, 196), by one thread.
__device__ __forceinline__ void prologue_set_dt(const Geo& G, StepCtl* ctl, const PrologueArgs& pa, double m) {
    double inner = __longlong_as_double((long long)ctl->vmax[pa.slot_in]);
    double maxs = speed_max(inner, m);
    ctl->max_speed = maxs;
    ctl->vmax[pa.slot_out] = 0ull;
    if (ctl->check_cfl) {
        if (maxs <= 0) {
            record_error(ctl, ST_CFL_ZERO, 0);
        } else {
            double cfl_dt = (G.dim == 1) ? pa.cfl_coeff * pa.dx / maxs : pa.cfl_coeff / maxs;
            ctl->t1 = smin(ctl->remaining, cfl_dt);
        }
    } else {
        ctl->t1 = ctl->remaining;
    }
}

// Per-step prologue, one CTA: step bookkeeping of the previous step, ghost
// fill, CFL over the ghost ring combined with the interior max the previous
// step's epilogue produced, and this step's dt (CFL.cpp:188-213).
// The body runs on one CTA of any size (a multiple of 32 threads); k_prologue
// launches it alone, the batched step runs it as one work item.
template <bool MHD>
__device__ __forceinline__ void prologue_body(const Geo& G, const Geo& FG, double* __restrict__ w,
                                              double* __restrict__ B, const BCEntry* __restrict__ bcs, StepCtl* ctl,
                                              const PrologueArgs& pa) {
    __shared__ int s_skip;
    __shared__ double s_red[32];
    if (threadIdx.x == 0) s_skip = prologue_bookkeeping(ctl, pa);
    __syncthreads();
    if (s_skip) return;

    if (pa.apply_bc) {
        for (int e = pa.bc_first; e < pa.bc_first + pa.nbc; e++) {
            const BCEntry be = bcs[e];
            for (int a = 0; a < G.dim; a++) {
                bc_cells_axis<MHD>(G, w, be, a, threadIdx.x, blockDim.x);
                __syncthreads();
            }
            if constexpr (MHD) {
                if (G.dim >= 2) {
                    for (int a = 0; a < G.dim; a++) {
                        bc_faces_axis(FG, G.n, B, be, a, threadIdx.x, blockDim.x);
                        __syncthreads();
                    }
                }
            }
        }
    }

    if (!pa.compute_dt) return;
    double m = 0.0;
    if (G.dim == 1) {
        if (threadIdx.x < 2) {
            int i = threadIdx.x == 0 ? -1 : G.n[0];
            Prim<double> W = load_prim<MHD>(w, G.plane, gidx1(G, i));
            m = cfl_speed_1d<MHD>(W);
        }
    } else {
        m = ring_speed_max<MHD>(G, w, pa, threadIdx.x, blockDim.x);
    }
    m = block_max(m, s_red);
    if (threadIdx.x == 0) prologue_set_dt(G, ctl, pa, m);
}

template <bool MHD>
__global__ void __launch_bounds__(1024) k_prologue(Geo G, Geo FG, double* __restrict__ w, double* __restrict__ B,
                                                   const BCEntry* __restrict__ bcs, StepCtl* ctl, PrologueArgs pa) {
    prologue_body<MHD>(G, FG, w, B, bcs, ctl, pa);
}

// Grid-wide barrier of a cooperative launch (every CTA resident). Bounded: a
// wait that gives up records ST_BARRIER and returns false. A waiting CTA also
// gives up as soon as another CTA has recorded a failure (the only failure the
// prologue records before its last barrier is a barrier that gave up), so one
// missing CTA costs one wait limit, not one per remaining barrier.
constexpr long long kGridBarrierPolls = 1LL << 22;  // >= 32 ns each
__device__ __forceinline__ bool grid_barrier(StepCtl* ctl) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = &ctl->bar_gen;
        const unsigned g0 = *gen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(&ctl->bar_arrive, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->bar_arrive, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            long long polls = 0;
            while (*gen == g0) {
                if (*(const volatile int*)&ctl->err) {
                    ok = 0;
                    break;
                }
                if (++polls > kGridBarrierPolls) {
                    ok = 0;
                    record_error(ctl, ST_BARRIER, 0);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// The prologue of a 2D / 3D grid as one cooperative launch: bookkeeping (CTA
// 0), then every ghost-fill pass over the whole grid in the reference's order
// (entry by entry, cells axis by axis, then faces axis by axis), then the
// ring CFL max (a block max per CTA, an atomic max across them) and dt (CTA
// 0), with a grid barrier between the stages. The same work as the one-CTA
// prologue_body, spread over the grid.
template <bool MHD>
__global__ void __launch_bounds__(256) k_prologue_coop(Geo G, Geo FG, double* __restrict__ w, double* __restrict__ B,
                                                      const BCEntry* __restrict__ bcs, StepCtl* ctl, PrologueArgs pa) {
    __shared__ int s_skip;
    __shared__ double s_red[32];
    // Every CTA reads the control block and decides alone: a failure recorded
    // by an earlier launch of this advance (a flux, state or barrier failure
    // of the batch the host has not read yet) or an advance the bookkeeping
    // ends (bookkeeping_done) returns before any barrier. Nothing writes the
    // control block until every CTA has read it, so all CTAs decide alike:
    // CTA 0 writes the bookkeeping after the first grid barrier, or, when the
    // advance is done, the last CTA to decide writes it.
    if (threadIdx.x == 0) {
        s_skip = *(const volatile int*)&ctl->err ? 1 : bookkeeping_done(ctl, pa) ? 2 : 0;
        if (blockIdx.x == pa.stall_cta) s_skip = 1;
    }
    __syncthreads();
    if (s_skip == 1) return;
    if (s_skip == 2) {
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(&ctl->bar_arrive, 1u) == gridDim.x - 1) {
                atomicExch(&ctl->bar_arrive, 0u);
                prologue_bookkeeping(ctl, pa);
            }
        }
        return;
    }
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    if (lead) ctl->ring_bits = 0ull;
    bool booked = false;
    auto book = [&] {
        if (lead && !booked) prologue_bookkeeping(ctl, pa);
        booked = true;
    };
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    // An entry fills its cells axis by axis, then its faces axis by axis. Cell
    // passes read and write only cells, face passes only faces, so the cell
    // and face passes of one axis share a stage: each array still sees its
    // passes in the reference's order, with one barrier per axis.
    if (pa.apply_bc) {
        for (int e = pa.bc_first; e < pa.bc_first + pa.nbc; e++) {
            const BCEntry be = bcs[e];
            for (int a = 0; a < G.dim; a++) {
                bc_cells_axis<MHD>(G, w, be, a, tid, nt);
                if constexpr (MHD) {
                    if (G.dim >= 2) bc_faces_axis(FG, G.n, B, be, a, tid, nt);
                }
                if (!grid_barrier(ctl)) return;
                book();
            }
        }
    }
    // The host launches this kernel only with a ghost-fill stage, so the
    // bookkeeping was written after the first stage's barrier.
    if (!pa.compute_dt) return;
    double m = ring_speed_max<MHD>(G, w, pa, tid, nt);
    m = block_max(m, s_red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->ring_bits, m);
    if (!grid_barrier(ctl)) return;
    book();
    if (lead) prologue_set_dt(G, ctl, pa, __longlong_as_double((long long)*(volatile unsigned long long*)&ctl->ring_bits));
}

// One ghost-fill pass (entry, axis; cells or faces) spread over a whole grid,
// for grids whose ghost layers are too large for the one-CTA prologue. The
// passes run as separate launches in the prologue's order (entry by entry,
// cells axis by axis, then faces axis by axis), so each sees the corners the
// earlier ones wrote. Skipped once the step is done or failed.
template <bool MHD>
__global__ void k_bc_pass(Geo G, Geo FG, double* __restrict__ w, double* __restrict__ B,
                          const BCEntry* __restrict__ bcs, StepCtl* ctl, int entry, int axis, int faces) {
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_skip = *(const volatile int*)&ctl->err | *(const volatile int*)&ctl->done;
    __syncthreads();
    if (s_skip) return;
    const BCEntry be = bcs[entry];
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, n = (long long)gridDim.x * blockDim.x;
    if (faces) bc_faces_axis(FG, G.n, B, be, axis, tid, n);
    else bc_cells_axis<MHD>(G, w, be, axis, tid, n);
}

// Interior CFL maximum over all interior cells (multi-CTA), accumulated into
// ctl->vmax[slot]. Used before the first step of an advance and by cfl_time.
template <bool MHD>
__global__ void k_interior_cfl(Geo G, const double* __restrict__ w, StepCtl* ctl, int slot, int cfl, double dx,
                               double dy, double dz) {
    __shared__ double s_red[32];
    const long long nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const long long total = nx * ny * nz;
    double m = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        long long mi;
        if (G.dim == 1) mi = gidx1(G, (int)t);
        else if (G.dim == 2) mi = gidx2(G, (int)(t / ny), (int)(t % ny));
        else mi = gidx3(G, (int)(t / (ny * nz)), (int)((t / nz) % ny), (int)(t % nz));
        Prim<double> W = load_prim<MHD>(w, G.plane, mi);
        m = speed_max(m, grid_cfl_speed<MHD>(W, G.dim, cfl, dx, dy, dz));
    }
    m = block_max(m, s_red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[slot], m);
}

}  // namespace dgpu
