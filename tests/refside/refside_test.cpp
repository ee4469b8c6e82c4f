// Drives DRAGON's own Grid::advance through the reference-side binding
// (gpugrid.hpp) and through the plain reference grid on the same initial
// state, then compares the padded arrays bit for bit.
//
//   refside_hydro kh2d | walls2d | retry2d | blast3d
//   refside_mhd   ot2d | blast3d_mhd
//
// Prints one line "<case> bitwise calls=<n> failures=<n> mismatches=<n>" and
// exits 0 when every cell (and face) matches, 1 otherwise.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "Boundary.hpp"
#include "DragonWing.hpp"
#include "gpugrid.hpp"

using refside::GPUGrid2D;
using refside::GPUGrid3D;
using refside::RefGrid2D;
using refside::RefGrid3D;

namespace {

#ifdef MHD
constexpr int NF = 8;
#else
constexpr int NF = 5;
#endif

// Deterministic noise in [-1, 1) (splitmix64 of the cell index).
double noise(uint64_t k) {
    uint64_t z = k + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) / (double)(1ull << 52) - 1.0;
}

long mismatches(const PrimitiveState* a, const PrimitiveState* b, long cells) {
    long bad = 0;
    const double* x = &a->rho;
    const double* y = &b->rho;
    for (long k = 0; k < cells * NF; k++)
        if (std::memcmp(&x[k], &y[k], sizeof(double)) != 0) bad++;
    return bad;
}

#ifdef MHD
long mismatches(const vec3* a, const vec3* b, long faces) {
    long bad = 0;
    for (long k = 0; k < faces; k++)
        if (std::memcmp(&a[k], &b[k], sizeof(vec3)) != 0) bad++;
    return bad;
}
#endif

int report(const char* name, long calls, long failures, long bad) {
    std::printf("%s %s calls=%ld failures=%ld mismatches=%ld\n", name, bad ? "DIFFERENT" : "bitwise", calls, failures,
                bad);
    return bad ? 1 : 0;
}

template <class G>
void shear_layer(G& g, int nx, int ny) {
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            const double y = (j + 0.5) / ny;
            PrimitiveState s;
            const bool in = std::abs(y - 0.5) < 0.25;
            s.rho = in ? 2.0 : 1.0;
            s.p = 2.5;
            s.v = vec3(in ? 0.5 : -0.5, 0.01 * noise((uint64_t)i * ny + j), 0.0);
            g[i, j] = s;
        }
}

#ifndef MHD
int run_kh2d(bool walls) {
    const int nx = 64, ny = 48;
    CONFIG::riemann_choice = RIEMANN_HLLC;
    CONFIG::limiter_choice = walls ? LIMITER_MC : LIMITER_VANLEER;
    RefGrid2D R(nx, ny, 1.0 / nx, 1.0 / ny, 2);
    GPUGrid2D G(nx, ny, 1.0 / nx, 1.0 / ny, 2);
    shear_layer(R, nx, ny);
    shear_layer(G, nx, ny);
    if (walls) {
        // the example list of the reference's documentation
        R.boundary = Boundary::Reflective("X") + Boundary::Periodic("YZ");
        G.boundary = Boundary::Reflective("X") + Boundary::Periodic("YZ");
    } else {
        R.boundary = Boundary::Periodic();
        G.boundary = Boundary::Periodic();
    }
    R.advance(0.05);
    G.advance(0.05);
    const int g = R.getGhosts();
    return report(walls ? "walls2d" : "kh2d", G.calls, G.failures,
                  mismatches(G.cells(), R.cells(), (long)(nx + 2 * g) * (ny + 2 * g)));
}

// A converging flow at Mach ~2000 advanced with a fixed dt (no CFL limit):
// the first attempts fail, and the reference's advance halves dt and retries
// them through the binding.
int run_retry2d() {
    const int n = 16;
    CONFIG::riemann_choice = RIEMANN_HLLC;
    CONFIG::limiter_choice = LIMITER_MC;
    RefGrid2D R(n, n, 1.0 / n, 1.0 / n, 2);
    GPUGrid2D G(n, n, 1.0 / n, 1.0 / n, 2);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            PrimitiveState s;
            s.rho = 1.0;
            s.p = 1e-3;
            s.v = vec3(i < 8 ? 50.0 : -50.0, 0.0, 0.0);
            R[i, j] = s;
            G[i, j] = s;
        }
    R.advance(0.01, false);
    G.advance(0.01, false);
    const int g = R.getGhosts();
    return report("retry2d", G.calls, G.failures, mismatches(G.cells(), R.cells(), (long)(n + 2 * g) * (n + 2 * g)));
}

int run_blast3d() {
    const int n = 24;
    const double d = 1.0 / n;
    CONFIG::riemann_choice = RIEMANN_HLLC;
    CONFIG::limiter_choice = LIMITER_MC;
    RefGrid3D R(n, n, n, d, d, d, 2);
    GPUGrid3D G(n, n, n, d, d, d, 2);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                const double x = (i + 0.5) * d - 0.5, y = (j + 0.5) * d - 0.5, z = (k + 0.5) * d - 0.5;
                PrimitiveState s;
                s.rho = 1.0;
                s.p = (x * x + y * y + z * z < 0.01) ? 10.0 : 0.1;
                R[i, j, k] = s;
                G[i, j, k] = s;
            }
    R.boundary = Boundary::Reflective("Z") + Boundary::Periodic("XY");
    G.boundary = Boundary::Reflective("Z") + Boundary::Periodic("XY");
    R.advance(0.01);
    G.advance(0.01);
    const int g = R.getGhosts();
    return report("blast3d", G.calls, G.failures,
                  mismatches(G.cells(), R.cells(), (long)(n + 2 * g) * (n + 2 * g) * (n + 2 * g)));
}
#else
// Orszag-Tang in DRAGON's Gaussian units with face-centred B set through
// _B() and the cell fields from initialize_B_fields (MHDGodunov_Tests.cpp:126-132).
int run_ot2d() {
    const int n = 48;
    const double d = 1.0 / n, pi = 3.14159265358979323846, B0 = 1.0 / std::sqrt(4.0 * pi);
    CONFIG::riemann_choice = RIEMANN_HLLX;
    CONFIG::limiter_choice = LIMITER_MC;
    RefGrid2D R(n, n, d, d, 3);
    GPUGrid2D G(n, n, d, d, 3);
    for (Grid2D* X : {(Grid2D*)&R, (Grid2D*)&G}) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const double x = (i + 0.5) * d, y = (j + 0.5) * d;
                PrimitiveState s;
                s.rho = 25.0 / (36.0 * pi);
                s.p = 5.0 / (12.0 * pi);
                s.v = vec3(-std::sin(2 * pi * y), std::sin(2 * pi * x), 0.0);
                (*X)[i, j] = s;
            }
        for (int i = 0; i <= n; i++)
            for (int j = 0; j <= n; j++) {
                X->_B()[i, j].x = -B0 * std::sin(2 * pi * (j + 0.5) * d);
                X->_B()[i, j].y = B0 * std::sin(4 * pi * (i + 0.5) * d);
            }
        X->boundary = Boundary::Periodic();
        X->boundary.apply(*X);
        X->initialize_B_fields();
    }
    R.advance(0.05);
    G.advance(0.05);
    const int g = R.getGhosts();
    const long bad = mismatches(G.cells(), R.cells(), (long)(n + 2 * g) * (n + 2 * g)) +
                     mismatches(G.faces(), R.faces(), (long)(n + 1 + 2 * g) * (n + 1 + 2 * g));
    return report("ot2d", G.calls, G.failures, bad);
}

int run_blast3d_mhd() {
    const int n = 16;
    const double d = 1.0 / n, b = 1.0 / std::sqrt(2.0);
    CONFIG::riemann_choice = RIEMANN_HLLX;
    CONFIG::limiter_choice = LIMITER_MC;
    RefGrid3D R(n, n, n, d, d, d, 3);
    GPUGrid3D G(n, n, n, d, d, d, 3);
    for (Grid3D* X : {(Grid3D*)&R, (Grid3D*)&G}) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    const double x = (i + 0.5) * d - 0.5, y = (j + 0.5) * d - 0.5, z = (k + 0.5) * d - 0.5;
                    PrimitiveState s;
                    s.rho = 1.0;
                    s.p = (x * x + y * y + z * z < 0.01) ? 10.0 : 0.1;
                    (*X)[i, j, k] = s;
                }
        for (int i = 0; i <= n; i++)
            for (int j = 0; j <= n; j++)
                for (int k = 0; k <= n; k++) X->_B()[i, j, k] = vec3(b, b, 0.0);
        X->boundary = Boundary::Outflow();
        X->boundary.apply(*X);
        X->initialize_B_fields();
    }
    R.advance(0.01);
    G.advance(0.01);
    const int g = R.getGhosts();
    const long bad = mismatches(G.cells(), R.cells(), (long)(n + 2 * g) * (n + 2 * g) * (n + 2 * g)) +
                     mismatches(G.faces(), R.faces(), (long)(n + 1 + 2 * g) * (n + 1 + 2 * g) * (n + 1 + 2 * g));
    return report("blast3d_mhd", G.calls, G.failures, bad);
}
#endif

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <case>\n", argv[0]);
        return 2;
    }
    DRAGONWING::initialize(0);
    CONFIG::cfl_choice = CFL_ADD;
    const std::string c = argv[1];
    try {
#ifndef MHD
        if (c == "kh2d") return run_kh2d(false);
        if (c == "walls2d") return run_kh2d(true);
        if (c == "retry2d") return run_retry2d();
        if (c == "blast3d") return run_blast3d();
#else
        if (c == "ot2d") return run_ot2d();
        if (c == "blast3d_mhd") return run_blast3d_mhd();
#endif
    } catch (const std::exception& e) {
        std::printf("%s error: %s\n", c.c_str(), e.what());
        return 1;
    }
    std::fprintf(stderr, "unknown case %s\n", c.c_str());
    return 2;
}
