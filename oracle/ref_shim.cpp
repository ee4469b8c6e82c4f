// C-ABI shim around the DRAGON reference, compiled together with the
// reference's own sources into oracle/_ref/libdragon_ref_{hydro,mhd,mhd_rt}.so.
//
// Test infrastructure only: the parity tests and the CPU baseline call the
// reference through these entry points. Nothing here computes physics; every
// call goes to the reference's public API (Grid1D/2D/3D, DistGrid*, the
// Boundary types, CFL::cfl_time, TVD::*, Riemann::*).
//
// Flat layouts used by every entry point:
//   * primitive cells: AoS, NF doubles per cell in the order
//     rho, p, vx, vy, vz[, Bx, By, Bz] (PrimitiveState, FluidElement.hpp:34-43),
//     cells in the reference's padded order (ExtendedArray.hpp:75,125:
//     last index fastest, ghosts included);
//   * face B: AoS of 3 doubles over the (n+1)-per-dimension padded arrays
//     (Grid.hpp:65,107; Splitting.cpp:277-293).
#include "Grid.hpp"
#include "DistGrid.hpp"
#include "CFL.hpp"
#include "TVD.hpp"
#include "Riemann.hpp"
#include "Boundary.hpp"
#include "DragonWing.hpp"
#include "Config.h"

#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>

namespace {

#ifdef MHD
constexpr int NF = 8;
#else
constexpr int NF = 5;
#endif

void to_prim(const double* a, PrimitiveState& w) {
    w.rho = a[0]; w.p = a[1]; w.v = {a[2], a[3], a[4]};
#ifdef MHD
    w.B = {a[5], a[6], a[7]};
#endif
}
void from_prim(const PrimitiveState& w, double* a) {
    a[0] = w.rho; a[1] = w.p; a[2] = w.v.x; a[3] = w.v.y; a[4] = w.v.z;
#ifdef MHD
    a[5] = w.B.x; a[6] = w.B.y; a[7] = w.B.z;
#endif
}
void to_cons(const double* a, ConservativeState& u) {
    u.rho = a[0]; u.E = a[1]; u.mom = {a[2], a[3], a[4]};
#ifdef MHD
    u.B = {a[5], a[6], a[7]};
#endif
}
void from_cons(const ConservativeState& u, double* a) {
    a[0] = u.rho; a[1] = u.E; a[2] = u.mom.x; a[3] = u.mom.y; a[4] = u.mom.z;
#ifdef MHD
    a[5] = u.B.x; a[6] = u.B.y; a[7] = u.B.z;
#endif
}

void put_msg(char* msg, int len, const char* s) {
    if (!msg || len <= 0) return;
    std::strncpy(msg, s, len - 1);
    msg[len - 1] = 0;
}

struct Handle {
    int dim;
    bool dist;
    std::unique_ptr<Grid> grid;
    Boundary::BoundaryList pending;
};

Grid1D* g1(Handle* h) { return static_cast<Grid1D*>(h->grid.get()); }
Grid2D* g2(Handle* h) { return static_cast<Grid2D*>(h->grid.get()); }
Grid3D* g3(Handle* h) { return static_cast<Grid3D*>(h->grid.get()); }

// A serial grid must not see a stale thread count left by a DistGrid step
// (pthread_parallel.cpp:51-59 keeps nthreads until the next initialize).
void serial_mode(Handle* h) {
    if (!h->dist) DRAGONWING::initialize(0);
}

}  // namespace

extern "C" {

int ref_is_mhd(void) {
#ifdef MHD
    return 1;
#else
    return 0;
#endif
}
int ref_nfields(void) { return NF; }

// Runtime switches (DRAGON/Config.h:97-110) and DistGrid's core_count.
void ref_config(int riemann, int limiter, int cfl, int ct_energy, int core_count) {
    CONFIG::riemann_choice = riemann;
    CONFIG::limiter_choice = limiter;
    CONFIG::cfl_choice = cfl;
#if defined(MHD) && CT_ENERGY_CONSV == CHOOSE_RUNTIME
    CONFIG::CT_energy_choice = ct_energy;
#else
    (void)ct_energy;
#endif
    if (core_count > 0) CONFIG::core_count = core_count;
}
int ref_ct_runtime(void) {
#if CT_ENERGY_CONSV == CHOOSE_RUNTIME
    return 1;
#else
    return 0;
#endif
}

void* ref_grid_new(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts,
                   int dist) {
    auto* h = new Handle();
    h->dim = dim;
    h->dist = dist != 0;
    if (dim == 1) {
        if (dist) h->grid = std::make_unique<DistGrid1D>(nx, dx, ghosts);
        else h->grid = std::make_unique<Grid1D>(nx, dx, ghosts);
    } else if (dim == 2) {
        if (dist) h->grid = std::make_unique<DistGrid2D>(nx, ny, dx, dy, ghosts);
        else h->grid = std::make_unique<Grid2D>(nx, ny, dx, dy, ghosts);
    } else {
        if (dist) h->grid = std::make_unique<DistGrid3D>(nx, ny, nz, dx, dy, dz, ghosts);
        else h->grid = std::make_unique<Grid3D>(nx, ny, nz, dx, dy, dz, ghosts);
    }
    return h;
}
void ref_grid_free(void* p) { delete static_cast<Handle*>(p); }

int ref_grid_ghosts(void* p) {
    auto* h = static_cast<Handle*>(p);
    if (h->dim == 1) return g1(h)->getGhosts();
    if (h->dim == 2) return g2(h)->getGhosts();
    return g3(h)->getGhosts();
}

// Copies the whole padded primitive array out of / into the grid.
void ref_grid_get_prim(void* p, double* out) {
    auto* h = static_cast<Handle*>(p);
    if (h->dim == 1) {
        Grid1D& g = *g1(h);
        const int n = g.getSize(), ng = g.getGhosts();
        for (int i = -ng; i < n + ng; i++) from_prim(g[i], out + (size_t)(i + ng) * NF);
    } else if (h->dim == 2) {
        Grid2D& g = *g2(h);
        const int nx = g.getSizeX(), ny = g.getSizeY(), ng = g.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++, m++) from_prim(g[i, j], out + m * NF);
    } else {
        Grid3D& g = *g3(h);
        const int nx = g.getSizeX(), ny = g.getSizeY(), nz = g.getSizeZ(), ng = g.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++)
                for (int k = -ng; k < nz + ng; k++, m++) from_prim(g[i, j, k], out + m * NF);
    }
}
void ref_grid_set_prim(void* p, const double* in) {
    auto* h = static_cast<Handle*>(p);
    if (h->dim == 1) {
        Grid1D& g = *g1(h);
        const int n = g.getSize(), ng = g.getGhosts();
        for (int i = -ng; i < n + ng; i++) to_prim(in + (size_t)(i + ng) * NF, g[i]);
    } else if (h->dim == 2) {
        Grid2D& g = *g2(h);
        const int nx = g.getSizeX(), ny = g.getSizeY(), ng = g.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++, m++) to_prim(in + m * NF, g[i, j]);
    } else {
        Grid3D& g = *g3(h);
        const int nx = g.getSizeX(), ny = g.getSizeY(), nz = g.getSizeZ(), ng = g.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++)
                for (int k = -ng; k < nz + ng; k++, m++) to_prim(in + m * NF, g[i, j, k]);
    }
}

#ifdef MHD
void ref_grid_get_faceB(void* p, double* out) {
    auto* h = static_cast<Handle*>(p);
    if (h->dim == 2) {
        auto& B = g2(h)->_B();
        const int nx = B.getSizeX(), ny = B.getSizeY(), ng = B.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++, m++) {
                out[3 * m] = B[i, j].x; out[3 * m + 1] = B[i, j].y; out[3 * m + 2] = B[i, j].z;
            }
    } else if (h->dim == 3) {
        auto& B = g3(h)->_B();
        const int nx = B.getSizeX(), ny = B.getSizeY(), nz = B.getSizeZ(), ng = B.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++)
                for (int k = -ng; k < nz + ng; k++, m++) {
                    out[3 * m] = B[i, j, k].x; out[3 * m + 1] = B[i, j, k].y; out[3 * m + 2] = B[i, j, k].z;
                }
    }
}
void ref_grid_set_faceB(void* p, const double* in) {
    auto* h = static_cast<Handle*>(p);
    if (h->dim == 2) {
        auto& B = g2(h)->_B();
        const int nx = B.getSizeX(), ny = B.getSizeY(), ng = B.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++, m++) B[i, j] = vec3{in[3 * m], in[3 * m + 1], in[3 * m + 2]};
    } else if (h->dim == 3) {
        auto& B = g3(h)->_B();
        const int nx = B.getSizeX(), ny = B.getSizeY(), nz = B.getSizeZ(), ng = B.getGhosts();
        size_t m = 0;
        for (int i = -ng; i < nx + ng; i++)
            for (int j = -ng; j < ny + ng; j++)
                for (int k = -ng; k < nz + ng; k++, m++)
                    B[i, j, k] = vec3{in[3 * m], in[3 * m + 1], in[3 * m + 2]};
    }
}
int ref_initialize_B_fields(void* p, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    try {
        h->grid->initialize_B_fields();
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}
#endif

// Boundary list construction, mirroring `grid.boundary = A + B + ...`
// (Boundary.hpp:129-134, BoundaryList.hpp:26-44). type: 0 Outflow,
// 1 Outflow::Gated, 2 Fixed, 3 Reflective, 4 Periodic, 5 Ignore.
void ref_boundary_clear(void* p) {
    auto* h = static_cast<Handle*>(p);
    h->pending.clear();
    h->grid->boundary = Boundary::BoundaryList();
}
int ref_boundary_add(void* p, int type, int faces, int corners, const double* fixed_state) {
    auto* h = static_cast<Handle*>(p);
    const bool c = corners != 0;
    switch (type) {
        case 0: h->pending.append(Boundary::Outflow(faces, c, false)); break;
        case 1: h->pending.append(Boundary::Outflow::Gated(faces, c)); break;
        case 2: {
            PrimitiveState s;
            to_prim(fixed_state, s);
            h->pending.append(Boundary::Fixed(s, faces, c));
            break;
        }
        case 3: h->pending.append(Boundary::Reflective(faces, c)); break;
        case 4: h->pending.append(Boundary::Periodic(faces, c)); break;
        case 5: h->pending.append(Boundary::Ignore(faces, c)); break;
        default: return 1;
    }
    return 0;
}
// Moves the list built so far into grid.boundary.
void ref_boundary_commit(void* p) {
    auto* h = static_cast<Handle*>(p);
    h->grid->boundary = std::move(h->pending);
    h->pending = Boundary::BoundaryList();
}
void ref_boundary_apply(void* p) {
    auto* h = static_cast<Handle*>(p);
    h->grid->boundary.apply(*h->grid);
}
int ref_face_mask(const char* s) { return Boundary::face_mask(std::string(s)); }

int ref_cfl_time(void* p, double* out, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    try {
        *out = CFL::cfl_time(*h->grid);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

// One Grid::unsplit_step (Unsplit.cpp:28-206, Splitting.cpp:100-115); a
// thrown std::runtime_error becomes status 1 with its message.
int ref_unsplit_step(void* p, double dt, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    serial_mode(h);
    try {
        h->grid->unsplit_step(dt);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

// Grid::advance (CFL.cpp:151-213). The reference exits the process when a
// retried step drops below Timestep_Tolerance; callers keep inputs physical.
int ref_advance(void* p, double dt, int check_cfl, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    serial_mode(h);
    try {
        h->grid->advance(dt, check_cfl != 0);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

int ref_split_step(void* p, double dt, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    serial_mode(h);
    try {
        h->grid->split_step(dt);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

int ref_advance_split(void* p, double dt, int check_cfl, char* msg, int len) {
    auto* h = static_cast<Handle*>(p);
    serial_mode(h);
    try {
        h->grid->advance_split(dt, check_cfl != 0);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

// --- unit-level entry points (pure functions of the reference) ---------------

int ref_limiter(int kind, double a, double b, double* out) {
    switch (kind) {
        case LIMITER_MINMOD: *out = TVD::minmod(a, b); break;
        case LIMITER_MC: *out = TVD::MC(a, b); break;
        case LIMITER_VANLEER: *out = TVD::vanLeer(a, b); break;
        case LIMITER_SUPERBEE: *out = TVD::superbee(a, b); break;
        case LIMITER_VANALBADA: *out = TVD::vanAlbada(a, b); break;
        default: return 1;
    }
    return 0;
}

void ref_muscl(const double* wl, const double* wc, const double* wr, double dt_dL, const double* dB,
               double* outL, double* outR) {
    PrimitiveState WL, WC, WR, L, R;
    to_prim(wl, WL); to_prim(wc, WC); to_prim(wr, WR);
    vec3 db{dB[0], dB[1], dB[2]};
    TVD::MUSCL(WL, L, WC, R, WR, dt_dL, db);
    from_prim(L, outL);
    from_prim(R, outR);
}

void ref_prim_to_cons(const double* w, double* u) {
    PrimitiveState W; to_prim(w, W);
    from_cons(ConservativeState(W), u);
}
void ref_cons_to_prim(const double* u, double* w) {
    ConservativeState U; to_cons(u, U);
    from_prim(PrimitiveState(U), w);
}
void ref_prim_flux(const double* w, double* f) {
    PrimitiveState W; to_prim(w, W);
    from_cons(W.flux(), f);
}

// solver: -1 = the configured dispatch with the physicality pivot
// (Riemann::flux_X/Y/Z, Flux.cpp:17-115); otherwise one solver directly:
// 0 exact, 1 HLL, 2 HLLC, 3 HLLD, 4 HLLE, 6 Roe. dim selects X/Y/Z swapping
// for the dispatch form.
int ref_riemann_flux(int solver, const double* l, const double* r, double dt_dx, int dim, double* out,
                     char* msg, int len) {
    PrimitiveState L, R;
    to_prim(l, L); to_prim(r, R);
    try {
        Riemann rp(L, R);
        ConservativeState F;
        switch (solver) {
            case -1:
                F = dim == 0 ? rp.flux_X(dt_dx) : (dim == 1 ? rp.flux_Y(dt_dx) : rp.flux_Z(dt_dx));
                break;
#ifndef MHD
            case 0: F = rp.exact().flux(); break;
            case 2: F = rp.HLLC(); break;
            case 6: F = rp.Roe(); break;
#else
            case 3: F = rp.HLLD(); break;
#endif
            case 1: F = rp.HLL(); break;
            case 4: F = rp.HLLE(); break;
            default: put_msg(msg, len, "unknown solver"); return 2;
        }
        from_cons(F, out);
    } catch (const std::exception& e) {
        put_msg(msg, len, e.what());
        return 1;
    }
    return 0;
}

#ifndef MHD
// Exact star state (Exact.cpp:47-93) for a given Newton guess (<= 0 selects
// the reference's default mean guess): sL/sR as primitive states.
void ref_exact_star(const double* l, const double* r, double pGuess, double* sl, double* sr) {
    PrimitiveState L, R;
    to_prim(l, L); to_prim(r, R);
    Riemann rp(L, R);
    RiemannSolution s = pGuess > 0 ? rp.exact(pGuess) : rp.exact();
    from_prim(s.sL, sl);
    from_prim(s.sR, sr);
}
void ref_exact_sample(const double* l, const double* r, double x_t, double* out) {
    PrimitiveState L, R;
    to_prim(l, L); to_prim(r, R);
    RiemannSolution s = Riemann(L, R).exact();
    from_prim(s.sample(x_t), out);
}
#endif

double ref_cfl_speed(const double* w, double dx, double dy, double dz) {
    PrimitiveState W; to_prim(w, W);
    return CFL::cfl_speed(W, dx, dy, dz);
}

}  // extern "C"
