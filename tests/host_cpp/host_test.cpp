// Test driver of the C++23 host API (include/dragon/dragon.hpp), written the
// way code against the reference is: Grid2D, grid[i, j], grid.boundary =
// Boundary::Reflective("X") + Boundary::Periodic("YZ"), grid.advance(dt).
//
//   host_test boundary                 boundary composition, no GPU needed
//   host_test run <case> <dir>         runs <case> from <dir>/<case>.in.bin,
//                                      writes <dir>/<case>.out.bin
//
// Input / output files hold the padded cell array (PrimitiveState layout, last
// index fastest, ghosts included), then for MHD the padded face-B array; the
// test compares the output with the oracle.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "dragon/dragon.hpp"
#include "dragon/hoard.hpp"

using namespace dragon;

static int failures = 0;
#define CHECK(c)                                                                 \
    do {                                                                         \
        if (!(c)) {                                                              \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #c); \
            failures++;                                                          \
        }                                                                        \
    } while (0)

// A user boundary element, the reference's Jet pattern (Jets.hpp:12-39): the
// X- ghost cells, corners included, take a fixed inflow state on the host.
struct Inflow : GhostFill {
    PrimitiveState s;
    explicit Inflow(PrimitiveState st) : GhostFill(Boundary::X_negative, true), s(st) {}
    void apply(Grid1D& g) override {
        for (int gl = 1; gl <= g.getGhosts(); gl++) g[-gl] = s;
    }
    void apply(Grid2D& g) override {
        const int ng = g.getGhosts();
        for (int j = -ng; j < g.getSizeY() + ng; j++)
            for (int gl = 1; gl <= ng; gl++) g[-gl, j] = s;
    }
    void apply(Grid3D& g) override {
        const int ng = g.getGhosts();
        for (int j = -ng; j < g.getSizeY() + ng; j++)
            for (int k = -ng; k < g.getSizeZ() + ng; k++)
                for (int gl = 1; gl <= ng; gl++) g[-gl, j, k] = s;
    }
};

static int test_boundary() {
    using namespace Boundary;
    CHECK(face_mask("X") == X);
    CHECK(face_mask("Y-") == Y_negative);
    CHECK(face_mask("XZ+") == (X | Z_positive));
    CHECK(face_mask("LRUD") == (X | Y));
    CHECK(face_mask("x+y") == (X_positive | Y));

    BoundaryList a = Reflective("X") + Periodic("YZ");
    CHECK(a.size() == 2);
    auto d = a.descriptors();
    CHECK(d[0].type == 3 && d[0].faces == X && d[0].corners == 1);
    CHECK(d[1].type == 4 && d[1].faces == (Y | Z));
    CHECK(a.uncovered_faces() == 0);

    // Periodic pairs faces; Outflow::Gated; Fixed carries its state; order kept
    PrimitiveState s;
    s.rho = 2.0;
    s.p = 3.0;
    s.v = vec3(0.5, 0, 0);
    BoundaryList b = Outflow::Gated("Y-", false) + Periodic("X+") + Fixed(s, "Z");
    auto e = b.descriptors();
    CHECK(e.size() == 3);
    CHECK(e[0].type == 1 && e[0].faces == Y_negative && e[0].corners == 0);
    CHECK(e[1].type == 4 && e[1].faces == X);
    CHECK(e[2].type == 2 && e[2].state[0] == 2.0 && e[2].state[1] == 3.0 && e[2].state[2] == 0.5);
    CHECK(b.uncovered_faces() == Y_positive);
    CHECK(!b.has_user_elements());

    // List + List, Element + List (prepend), +=
    BoundaryList c = Ignore("X") + (Reflective("Y") + Outflow("Z"));
    CHECK(c.descriptors()[0].type == 5 && c.descriptors()[1].type == 3 && c.descriptors()[2].type == 0);
    c += Periodic("X");
    CHECK(c.size() == 4 && c.descriptors()[3].type == 4);
    BoundaryList u = Reflective("Y") + Inflow(s);
    CHECK(u.has_user_elements());
    CHECK(u.descriptors()[1].type == 5 && u.descriptors()[1].faces == X_negative);
    CHECK(u.uncovered_faces() == (X_positive | Z));

    // assignment from an element replaces the list
    BoundaryList g;
    g = Periodic();
    CHECK(g.size() == 1 && g.descriptors()[0].faces == (X | Y | Z));
    return failures;
}

static std::vector<double> read_all(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open " + path);
    const auto n = (size_t)f.tellg();
    std::vector<double> v(n / sizeof(double));
    f.seekg(0);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)n);
    return v;
}

static void write_all(const std::string& path, const std::vector<double>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

constexpr int NF = sizeof(PrimitiveState) / sizeof(double);

static PrimitiveState state_at(const std::vector<double>& a, size_t k) {
    const double* q = &a[k * NF];
    PrimitiveState s;
    s.rho = q[0];
    s.p = q[1];
    s.v = vec3(q[2], q[3], q[4]);
#ifdef MHD
    s.B = vec3(q[5], q[6], q[7]);
#endif
    return s;
}

static void put_state(std::vector<double>& a, const PrimitiveState& s) {
    const double* p = &s.rho;
    a.insert(a.end(), p, p + NF);
}

static int run_case(const std::string& name, const std::string& dir) {
    const std::vector<double> in = read_all(dir + "/" + name + ".in.bin");
    std::vector<double> out;
    Config cfg;
    if (name == "sod1d") {
        const int n = 512, g = 2;
        cfg.riemann = 2;  // HLLC
        cfg.limiter = 0;  // minmod
        Grid1D grid(n, 1.0 / n, g, cfg);
        for (int i = -g; i < n + g; i++) grid[i] = state_at(in, (size_t)(i + g));
        grid.advance(0.2);  // implicit Outflow on every face
        std::printf("steps %d last_dt %.17g\n", grid.last_advance().steps, grid.last_advance().last_dt);
        for (int i = -g; i < n + g; i++) put_state(out, grid[i]);
    } else if (name == "kh2d" || name == "kh2d_walls" || name == "kh2d_inflow" || name == "kh2d_device_inflow") {
        const int nx = 64, ny = 48, g = 2;
        cfg.riemann = 2;
        cfg.limiter = 2;  // van Leer
        Grid2D grid(nx, ny, 1.0 / nx, 1.0 / ny, g, cfg);
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) grid[i, j] = state_at(in, (size_t)((i + g) * (ny + 2 * g) + (j + g)));
        if (name == "kh2d") {
            grid.boundary = Boundary::Periodic();
            grid.advance_steps(5);
        } else if (name == "kh2d_walls") {
            grid.boundary = Boundary::Reflective("X") + Boundary::Periodic("YZ");
            grid.advance(0.02);
        } else if (name == "kh2d_inflow") {
            PrimitiveState jet;
            jet.rho = 3.0;
            jet.p = 2.5;
            jet.v = vec3(0.8, 0.0, 0.0);
            grid.boundary = Boundary::Periodic("Y") + Inflow(jet);
            grid.advance(0.02);
        } else {
            // the same inflow as a fill compiled for the device
            const char* src = R"(
__device__ void inflow(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nparams; f++) c.set(f, i, j, k, c.params[f]);
})";
            grid.boundary = Boundary::Periodic("Y") +
                            Boundary::DeviceFill(src, "inflow", Boundary::X_negative, Boundary::X_negative,
                                                 {3.0, 2.5, 0.8, 0.0, 0.0});
            grid.advance(0.02);
        }
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) put_state(out, grid[i, j]);
#ifdef MHD
    } else if (name == "ot2d") {
        const int n = 32, g = 3;
        cfg.riemann = 5;  // HLLD
        Grid2D grid(n, n, 1.0 / n, 1.0 / n, g, cfg);
        const size_t ncell = (size_t)(n + 2 * g) * (n + 2 * g);
        for (int i = -g; i < n + g; i++)
            for (int j = -g; j < n + g; j++) grid[i, j] = state_at(in, (size_t)((i + g) * (n + 2 * g) + (j + g)));
        auto& B = grid._B();
        for (int i = -g; i <= n + g; i++)
            for (int j = -g; j <= n + g; j++) {
                const size_t k = ncell * NF + 3 * (size_t)((i + g) * (n + 1 + 2 * g) + (j + g));
                B[i, j] = vec3(in[k], in[k + 1], in[k + 2]);
            }
        grid.boundary = Boundary::Periodic();
        grid.initialize_B_fields();
        grid.advance_steps(5);
        for (int i = -g; i < n + g; i++)
            for (int j = -g; j < n + g; j++) put_state(out, grid[i, j]);
        for (int i = -g; i <= n + g; i++)
            for (int j = -g; j <= n + g; j++) {
                const vec3 b = B[i, j];
                out.push_back(b.x);
                out.push_back(b.y);
                out.push_back(b.z);
            }
#endif
    } else if (name == "hoard2d") {
        // DRAGONHOARD from C++: run 3 steps, write a frame, restart a fresh
        // grid (spacing 0) from the newest frame, run 3 more steps on both
        const int nx = 64, ny = 48, g = 2;
        cfg.riemann = 2;
        cfg.limiter = 2;
        Grid2D grid(nx, ny, 1.0 / nx, 1.0 / ny, g, cfg);
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) grid[i, j] = state_at(in, (size_t)((i + g) * (ny + 2 * g) + (j + g)));
        grid.boundary = Boundary::Periodic();
        grid.advance_steps(3);
        DRAGONHOARD::output_dir = dir + "/frames";
        DRAGONHOARD::verifyOutputDirectory();
        DRAGONHOARD::options.write_option = 1;
        DRAGONHOARD::writeToFileAsync(grid, 0.25, 2, DRAGONHOARD::output_base_name + "_" + DRAGONHOARD::cycle_string(2));
        DRAGONHOARD::writeToFile(grid, 0.5, 3, DRAGONHOARD::output_base_name + "_" + DRAGONHOARD::cycle_string(3));
        DRAGONHOARD::waitForFiles(grid);
        DRAGONHOARD::restart_frame = -1;
        const std::string file = DRAGONHOARD::restartFileName();
        Grid2D again(nx, ny, 0.0, 0.0, g, cfg);
        double t = 0;
        int cycle = 0;
        DRAGONHOARD::loadFromFile(again, t, cycle, file);
        std::printf("file %s t %.17g cycle %d dx %.17g dy %.17g\n", file.c_str(), t, cycle, again.dx, again.dy);
        again.boundary = Boundary::Periodic();
        grid.advance_steps(3);
        again.advance_steps(3);
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) put_state(out, grid[i, j]);
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) put_state(out, again[i, j]);
    } else if (name == "blast3d") {
        const int n = 16, g = 2;
        cfg.riemann = 2;
        Grid3D grid(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, g, cfg);
        const int e = n + 2 * g;
        for (int i = -g; i < n + g; i++)
            for (int j = -g; j < n + g; j++)
                for (int k = -g; k < n + g; k++) grid[i, j, k] = state_at(in, (size_t)(((i + g) * e + (j + g)) * e + (k + g)));
        grid.advance_steps(3);
        for (int i = -g; i < n + g; i++)
            for (int j = -g; j < n + g; j++)
                for (int k = -g; k < n + g; k++) put_state(out, grid[i, j, k]);
    } else {
        std::fprintf(stderr, "unknown case %s\n", name.c_str());
        return 2;
    }
    write_all(dir + "/" + name + ".out.bin", out);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 2 && std::string(argv[1]) == "boundary") {
        const int f = test_boundary();
        std::printf(f ? "FAILED %d\n" : "ok\n", f);
        return f ? 1 : 0;
    }
    if (argc >= 4 && std::string(argv[1]) == "run") {
        try {
            return run_case(argv[2], argv[3]);
        } catch (const std::exception& e) {
            std::fprintf(stderr, "error: %s\n", e.what());
            return 3;
        }
    }
    std::fprintf(stderr, "usage: host_test boundary | run <case> <dir>\n");
    return 2;
}
