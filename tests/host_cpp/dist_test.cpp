// Test driver of the C++ DistGrid (include/dragon/dist.hpp) on one GPU.
//
//   dist_test threads <P> <case>   P ranks as threads, each with its own slab
//                                  on the visible GPU, exchanging through host
//                                  memory (their kernels never wait on one
//                                  another); the gathered result must equal
//                                  the serial grid's bit for bit
//   dist_test nccl1 <case>         one rank over a one-GPU NCCL communicator
//
// Cases: kh (periodic shear layer), walls (Outflow Y without corner ghosts +
// Reflective X), blast3d (3D, implicit Outflow), ot (Orszag-Tang, MHD build).
#include <cuda_runtime.h>
#include <nccl.h>

#include <barrier>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "dragon/dist.hpp"

using namespace dragon;

// Ranks as threads of one process: transfers go through host mailboxes.
struct Shared {
    int P;
    std::barrier<> bar;
    std::vector<std::vector<double>> box;  // box[src * P + dst]
    std::vector<double> red;
    explicit Shared(int p) : P(p), bar(p), box((size_t)p * p), red(p) {}
};

class ThreadComm : public SlabComm {
public:
    ThreadComm(Shared& s, int r) : s_(s), r_(r) {}
    int rank() const override { return r_; }
    int size() const override { return s_.P; }
    void exchange(const std::vector<SlabTransfer>& t, void* stream) override {
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        for (const SlabTransfer& x : t) {
            auto& b = s_.box[(size_t)r_ * s_.P + x.peer];
            b.resize(x.send_count);
            cudaMemcpy(b.data(), x.send, sizeof(double) * x.send_count, cudaMemcpyDeviceToHost);
        }
        s_.bar.arrive_and_wait();
        bool sizes_ok = true;
        for (const SlabTransfer& x : t) {
            const auto& b = s_.box[(size_t)x.peer * s_.P + r_];
            if (b.size() != x.recv_count) {
                sizes_ok = false;
                continue;
            }
            cudaMemcpy(x.recv, b.data(), sizeof(double) * x.recv_count, cudaMemcpyHostToDevice);
        }
        s_.bar.arrive_and_wait();
        if (!sizes_ok) throw std::runtime_error("a received halo has the wrong size");
    }
    double allreduce_min(double v) override {
        s_.red[r_] = v;
        s_.bar.arrive_and_wait();
        double m = s_.red[0];
        for (double x : s_.red) m = std::fmin(m, x);
        s_.bar.arrive_and_wait();
        return m;
    }

private:
    Shared& s_;
    int r_;
};

struct Case {
    int dim, n[3], g;
    double d[3];
    Config cfg;
    int steps;
    std::vector<PrimitiveState> w;
    std::vector<vec3> B;
};

static size_t cells(const Case& c) {
    size_t k = 1;
    for (int a = 0; a < c.dim; a++) k *= (size_t)(c.n[a] + 2 * c.g);
    return k;
}

static Case make_case(const std::string& name) {
    Case c{};
    std::mt19937_64 rng(1234);
    std::uniform_real_distribution<double> u(-0.01, 0.01);
    if (name == "kh" || name == "walls" || name == "fills") {
        c.dim = 2;
        c.n[0] = 40;
        c.n[1] = 24;
        c.n[2] = 1;
        c.g = 2;
        c.d[0] = 1.0 / 40;
        c.d[1] = 1.0 / 24;
        c.cfg.riemann = 2;
        c.cfg.limiter = 2;
        c.steps = 4;
        c.w.resize(cells(c));
        const int ey = c.n[1] + 2 * c.g;
        for (int i = -c.g; i < c.n[0] + c.g; i++)
            for (int j = -c.g; j < c.n[1] + c.g; j++) {
                // every cell, ghosts included, holds a physical state (a corner an
                // element leaves alone keeps it)
                const int jj = std::min(std::max(j, 0), c.n[1] - 1);
                const double y = (jj + 0.5) * c.d[1];
                PrimitiveState& s = c.w[(size_t)(i + c.g) * ey + (j + c.g)];
                const bool inner = std::fabs(y - 0.5) < 0.25;
                s.rho = inner ? 2.0 : 1.0;
                s.p = 2.5;
                s.v = vec3(inner ? 0.5 : -0.5, u(rng), 0.0);
            }
    } else if (name == "blast3d") {
        c.dim = 3;
        c.n[0] = 12;
        c.n[1] = 10;
        c.n[2] = 8;
        c.g = 2;
        for (int a = 0; a < 3; a++) c.d[a] = 1.0 / 12;
        c.cfg.riemann = 2;
        c.steps = 2;
        c.w.resize(cells(c));
        for (int i = 0; i < c.n[0]; i++)
            for (int j = 0; j < c.n[1]; j++)
                for (int k = 0; k < c.n[2]; k++) {
                    const double x = (i + 0.5) / 12 - 0.5, y = (j + 0.5) / 12 - 5.0 / 12, z = (k + 0.5) / 12 - 4.0 / 12;
                    PrimitiveState& s = c.w[((size_t)(i + 2) * 14 + (j + 2)) * 12 + (k + 2)];
                    s.rho = 1.0;
                    s.p = x * x + y * y + z * z < 0.04 ? 10.0 : 0.1;
                }
#ifdef MHD
    } else if (name == "ot") {
        const int n = 24, g = 3;
        c.dim = 2;
        c.n[0] = c.n[1] = n;
        c.n[2] = 1;
        c.g = g;
        c.d[0] = c.d[1] = 1.0 / n;
        c.cfg.riemann = 5;
        c.steps = 3;
        c.w.resize(cells(c));
        const double pi = 3.14159265358979323846, B0 = 1.0 / std::sqrt(4 * pi);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const double x = (i + 0.5) / n, y = (j + 0.5) / n;
                PrimitiveState& s = c.w[(size_t)(i + g) * (n + 2 * g) + (j + g)];
                s.rho = 25.0 / (36.0 * pi);
                s.p = 5.0 / (12.0 * pi);
                s.v = vec3(-std::sin(2 * pi * y), std::sin(2 * pi * x), 0.0);
            }
        c.B.resize((size_t)(n + 1 + 2 * g) * (n + 1 + 2 * g));
        for (int i = 0; i <= n; i++)
            for (int j = 0; j <= n; j++) {
                const double xf = (double)i / n, yc = (j + 0.5) / n, xc = (i + 0.5) / n, yf = (double)j / n;
                (void)yf;
                c.B[(size_t)(i + g) * (n + 1 + 2 * g) + (j + g)] =
                    vec3(-B0 * std::sin(2 * pi * yc), B0 * std::sin(4 * pi * xc), 0.0);
                (void)xf;
            }
#endif
    } else {
        std::fprintf(stderr, "unknown case %s\n", name.c_str());
        std::exit(2);
    }
    return c;
}

// Device user fills (NVRTC): the y faces take the nearest interior row with vy
// from the global x position (c.off[0]: the slab's place), X- is a jet.
static const char* kYFill = R"(
__device__ void yfill(const dragon_fill_ctx& c, int i, int j, int k) {
    const int js = c.side == 0 ? 0 : c.n[1] - 1;
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, i, js, k));
    const double x = (c.off[0] + i + 0.5) * c.d[0];
    c.set(DRAGON_VY, i, j, k, c.params[0] * x * (1.0 - x));
})";
static const char* kJet = R"(
__device__ void jet(const dragon_fill_ctx& c, int i, int j, int k) {
    for (int f = 0; f < c.nf; f++) c.set(f, i, j, k, c.get(f, 0, j, k));
    if (fabs((j + 0.5) * c.d[1] - 0.5) < 0.2) {
        c.set(DRAGON_RHO, i, j, k, 2.0);
        c.set(DRAGON_P, i, j, k, 3.0);
        c.set(DRAGON_VX, i, j, k, 1.5);
    }
})";

static void set_boundary(Boundary::BoundaryList& b, const std::string& name) {
    if (name == "kh" || name == "ot") b = Boundary::Periodic();
    else if (name == "walls") b = Boundary::Outflow("Y", false) + Boundary::Reflective("X");
    else if (name == "fills")
        b = Boundary::DeviceFill(kYFill, "yfill", Boundary::Y, Boundary::Y, {0.4}) +
            Boundary::DeviceFill(kJet, "jet", Boundary::X_negative, Boundary::X_negative) + Boundary::Outflow("X+");
}

// The serial grid's run through the same C++ API (Grid::advance_steps).
static void serial(const std::string& name, const Case& c, std::vector<PrimitiveState>& w, std::vector<vec3>& B) {
    std::unique_ptr<Grid> G;
    if (c.dim == 2) G = std::make_unique<Grid2D>(c.n[0], c.n[1], c.d[0], c.d[1], c.g, c.cfg);
    else G = std::make_unique<Grid3D>(c.n[0], c.n[1], c.n[2], c.d[0], c.d[1], c.d[2], c.g, c.cfg);
    dragon_grid* h = G->handle();
    if (dragon_gpu_upload_prim(h, &c.w[0].rho)) std::abort();
    if (!c.B.empty() && dragon_gpu_upload_faceB(h, &c.B[0].x)) std::abort();
    set_boundary(G->boundary, name);
    if (!c.B.empty()) {
        // the host mirror is stale: push the boundary and initialise on the device directly
        std::vector<dragon_bc_desc> d = G->boundary.descriptors();
        if (dragon_gpu_set_boundary(h, d.data(), (int)d.size()) || dragon_gpu_initialize_B_fields(h)) std::abort();
    }
    std::vector<dragon_bc_desc> d = G->boundary.descriptors();
    if (dragon_gpu_set_boundary(h, d.data(), (int)d.size())) std::abort();
    for (size_t k = 0; k < G->boundary.size(); k++)
        if (const auto* df = dynamic_cast<const Boundary::DeviceFill*>(&G->boundary[k]))
            if (dragon_gpu_set_user_fill(h, (int)k, df->compiled(), df->fill_faces, df->get_corners() ? 1 : 0,
                                         df->params.empty() ? nullptr : df->params.data(), (int)df->params.size()))
                std::abort();
    dragon_advance_stats st;
    if (dragon_gpu_advance_steps(h, c.steps, &st)) {
        std::fprintf(stderr, "serial: %s\n", dragon_gpu_last_error());
        std::abort();
    }
    w.resize(c.w.size());
    if (dragon_gpu_download_prim(h, &w[0].rho)) std::abort();
    if (!c.B.empty()) {
        B.resize(c.B.size());
        if (dragon_gpu_download_faceB(h, &B[0].x)) std::abort();
    }
}

static std::unique_ptr<DistGrid> make_dist(const Case& c, SlabComm& comm) {
    if (c.dim == 2) return std::make_unique<DistGrid2D>(c.n[0], c.n[1], c.d[0], c.d[1], c.g, comm, c.cfg);
    return std::make_unique<DistGrid3D>(c.n[0], c.n[1], c.n[2], c.d[0], c.d[1], c.d[2], c.g, comm, c.cfg);
}

static void run_rank(const std::string& name, const Case& c, SlabComm& comm, std::vector<PrimitiveState>& out,
                     std::vector<vec3>& outB, std::string& err) {
    try {
        auto D = make_dist(c, comm);
        D->scatter(c.w.data(), c.B.empty() ? nullptr : c.B.data());
        set_boundary(D->boundary, name);
        if (!c.B.empty()) D->initialize_B_fields();
        D->advance_steps(c.steps);
        D->gather(out.data(), outB.empty() ? nullptr : outB.data());
    } catch (const std::exception& e) {
        err = e.what();
    }
}

static int compare(const char* what, const std::vector<PrimitiveState>& a, const std::vector<PrimitiveState>& b,
                   const std::vector<vec3>& A, const std::vector<vec3>& B) {
    if (std::memcmp(a.data(), b.data(), sizeof(PrimitiveState) * a.size()) != 0) {
        std::fprintf(stderr, "%s: cells differ from the serial grid\n", what);
        return 1;
    }
    if (!A.empty() && std::memcmp(A.data(), B.data(), sizeof(vec3) * A.size()) != 0) {
        std::fprintf(stderr, "%s: face B differs from the serial grid\n", what);
        return 1;
    }
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: dist_test threads <P> <case> | nccl1 <case>\n");
        return 2;
    }
    const std::string mode = argv[1];
    const std::string name = mode == "threads" ? argv[3] : argv[2];
    const Case c = make_case(name);
    std::vector<PrimitiveState> ws;
    std::vector<vec3> Bs;
    serial(name, c, ws, Bs);
    std::vector<PrimitiveState> out(c.w.size());
    std::vector<vec3> outB(c.B.size());
    if (mode == "threads") {
        const int P = std::atoi(argv[2]);
        Shared sh(P);
        std::vector<std::thread> th;
        std::vector<std::string> errs(P);
        std::vector<std::unique_ptr<ThreadComm>> comms;
        for (int r = 0; r < P; r++) comms.push_back(std::make_unique<ThreadComm>(sh, r));
        for (int r = 0; r < P; r++)
            th.emplace_back([&, r] { run_rank(name, c, *comms[r], out, outB, errs[r]); });
        for (auto& t : th) t.join();
        for (int r = 0; r < P; r++)
            if (!errs[r].empty()) {
                std::fprintf(stderr, "rank %d: %s\n", r, errs[r].c_str());
                return 3;
            }
    } else if (mode == "nccl1") {
        ncclComm_t comm;
        int dev = 0;
        if (ncclCommInitAll(&comm, 1, &dev) != ncclSuccess) {
            std::fprintf(stderr, "ncclCommInitAll failed\n");
            return 3;
        }
        {
            auto sc = make_nccl_comm(comm);
            std::string err;
            run_rank(name, c, *sc, out, outB, err);
            if (!err.empty()) {
                std::fprintf(stderr, "nccl rank: %s\n", err.c_str());
                return 3;
            }
        }
        ncclCommDestroy(comm);
    } else {
        return 2;
    }
    if (compare(name.c_str(), out, ws, outB, Bs)) return 1;
    std::printf("ok %s %s\n", mode.c_str(), name.c_str());
    return 0;
}
