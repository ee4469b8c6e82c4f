// The reference-side binding: DRAGON's own Grid2D / Grid3D with their
// unsplit_step overridden by the C ABI of include/dragon_gpu.h, as a
// maintainer who keeps the reference's Grid classes would write it (the
// snippet in INTEGRATION.md, with the MHD face fields and a 3D form).
//
// Everything else stays the reference's: Grid::advance / advance_unsplit
// (DRAGON/Hydro/CFL/CFL.cpp:151-213) fills the ghosts with the reference's
// BoundaryList, takes CFL::cfl_time on the host arrays and calls the virtual
// unsplit_step; the override uploads the padded arrays, steps on the GPU and
// downloads them. A failed device step becomes std::runtime_error, so the
// reference's catch-and-halve loop (CFL.cpp:194-209) retries it.
//
// Compile with the reference's include paths and Config.h; link
// libdragon_gpu.so.
#pragma once

#include <stdexcept>

#include "Config.h"
#include "Grid.hpp"
#include "dragon_gpu.h"

namespace refside {

inline void ck(int rc) {
    if (rc) throw std::runtime_error(dragon_gpu_last_error());
}

// DRAGON's switches as the C ABI's runtime configuration. The shipped
// Config.h defines RIEMANN_DEFAULT / MUSCL_DEFAULT_LIMITER / CFL_CALCULATION
// as constants; a build whose Config.h chooses them at run time
// (CHOOSE_RUNTIME) reads CONFIG::riemann_choice and friends instead.
inline dragon_config config_from_reference() {
    dragon_config c;
#ifdef MHD
    dragon_gpu_default_config(&c, 1);
#else
    dragon_gpu_default_config(&c, 0);
#endif
#if RIEMANN_DEFAULT == CHOOSE_RUNTIME
    c.riemann = CONFIG::riemann_choice;
#else
    c.riemann = RIEMANN_DEFAULT;
#endif
#if MUSCL_DEFAULT_LIMITER == CHOOSE_RUNTIME
    c.limiter = CONFIG::limiter_choice;
#else
    c.limiter = MUSCL_DEFAULT_LIMITER;
#endif
#if CFL_CALCULATION == CHOOSE_RUNTIME
    c.cfl = CONFIG::cfl_choice;
#else
    c.cfl = CFL_CALCULATION;
#endif
    c.exact_max_iters = CONFIG::ExactRiemann_MaxIters;
    c.exact_tol = CONFIG::ExactRiemann_Tolerance;
    c.cfl_coeff = CONFIG::CFL_coeff;
    c.timestep_tol = CONFIG::Timestep_Tolerance;
    return c;
}

struct GPUGrid2D : public Grid2D {
    dragon_grid* h = nullptr;
    long calls = 0, failures = 0;  // unsplit_step calls and the ones that threw

    GPUGrid2D(int nx, int ny, double dx, double dy, int ghosts = 1) : Grid2D(nx, ny, dx, dy, ghosts) {
        dragon_config c = config_from_reference();
        ck(dragon_gpu_grid_create(2, nx, ny, 1, dx, dy, 0, getGhosts(), &c, &h));
    }
    ~GPUGrid2D() override { dragon_gpu_grid_destroy(h); }

    void unsplit_step(double dt) override {
        const int g = getGhosts();
        calls++;
        ck(dragon_gpu_upload_prim(h, &w[-g, -g].rho));
#ifdef MHD
        ck(dragon_gpu_upload_faceB(h, &B[-g, -g].x));
#endif
        dragon_step_status st;
        if (dragon_gpu_unsplit_step(h, dt, &st)) {
            failures++;
            throw std::runtime_error(dragon_gpu_last_error());
        }
        ck(dragon_gpu_download_prim(h, &w[-g, -g].rho));
#ifdef MHD
        ck(dragon_gpu_download_faceB(h, &B[-g, -g].x));
#endif
    }
    const PrimitiveState* cells() { return &w[-getGhosts(), -getGhosts()]; }
#ifdef MHD
    const vec3* faces() { return &B[-getGhosts(), -getGhosts()]; }
#endif
};

struct GPUGrid3D : public Grid3D {
    dragon_grid* h = nullptr;
    long calls = 0, failures = 0;

    GPUGrid3D(int nx, int ny, int nz, double dx, double dy, double dz, int ghosts = 2)
        : Grid3D(nx, ny, nz, dx, dy, dz, ghosts) {
        dragon_config c = config_from_reference();
        ck(dragon_gpu_grid_create(3, nx, ny, nz, dx, dy, dz, getGhosts(), &c, &h));
    }
    ~GPUGrid3D() override { dragon_gpu_grid_destroy(h); }

    void unsplit_step(double dt) override {
        const int g = getGhosts();
        calls++;
        ck(dragon_gpu_upload_prim(h, &w[-g, -g, -g].rho));
#ifdef MHD
        ck(dragon_gpu_upload_faceB(h, &B[-g, -g, -g].x));
#endif
        dragon_step_status st;
        if (dragon_gpu_unsplit_step(h, dt, &st)) {
            failures++;
            throw std::runtime_error(dragon_gpu_last_error());
        }
        ck(dragon_gpu_download_prim(h, &w[-g, -g, -g].rho));
#ifdef MHD
        ck(dragon_gpu_download_faceB(h, &B[-g, -g, -g].x));
#endif
    }
    const PrimitiveState* cells() { return &w[-getGhosts(), -getGhosts(), -getGhosts()]; }
#ifdef MHD
    const vec3* faces() { return &B[-getGhosts(), -getGhosts(), -getGhosts()]; }
#endif
};

// The plain reference grids with read access to their padded arrays.
struct RefGrid2D : public Grid2D {
    using Grid2D::Grid2D;
    const PrimitiveState* cells() { return &w[-getGhosts(), -getGhosts()]; }
#ifdef MHD
    const vec3* faces() { return &B[-getGhosts(), -getGhosts()]; }
#endif
};
struct RefGrid3D : public Grid3D {
    using Grid3D::Grid3D;
    const PrimitiveState* cells() { return &w[-getGhosts(), -getGhosts(), -getGhosts()]; }
#ifdef MHD
    const vec3* faces() { return &B[-getGhosts(), -getGhosts(), -getGhosts()]; }
#endif
};

}  // namespace refside
