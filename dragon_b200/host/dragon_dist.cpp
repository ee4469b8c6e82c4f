// DistGrid over several GPUs for C++ hosts (include/dragon/dist.hpp): x slabs,
// halo exchange through a SlabComm, global CFL minimum, all-or-nothing commit.
// Built as libdragon_dist.so (hydro) and libdragon_dist_mhd.so (with MHD).
#include "../../include/dragon/dist.hpp"

#include <cuda_runtime.h>
#include <nccl.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

namespace dragon {

namespace {

constexpr int kAllFaces = 63;
constexpr int kNF = kMHD ? 8 : 5;

// A step that failed on some slab: the advance loop halves dt and retries.
struct SlabStepFailed : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void nccl_check(ncclResult_t r, const char* what) {
    if (r != ncclSuccess) throw std::runtime_error(std::string(what) + ": " + ncclGetErrorString(r));
}

class NcclComm : public SlabComm {
public:
    explicit NcclComm(ncclComm_t c) : comm_(c) {
        nccl_check(ncclCommUserRank(comm_, &rank_), "ncclCommUserRank");
        nccl_check(ncclCommCount(comm_, &size_), "ncclCommCount");
        cuda_check(cudaMalloc(&scalar_, sizeof(double)), "cudaMalloc");
    }
    ~NcclComm() override { cudaFree(scalar_); }
    int rank() const override { return rank_; }
    int size() const override { return size_; }
    void exchange(const std::vector<SlabTransfer>& t, void* stream) override {
        if (t.empty()) return;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        nccl_check(ncclGroupStart(), "ncclGroupStart");
        for (const SlabTransfer& x : t) {
            nccl_check(ncclSend(x.send, x.send_count, ncclDouble, x.peer, comm_, s), "ncclSend");
            nccl_check(ncclRecv(x.recv, x.recv_count, ncclDouble, x.peer, comm_, s), "ncclRecv");
        }
        nccl_check(ncclGroupEnd(), "ncclGroupEnd");
    }
    double allreduce_min(double v) override {
        cuda_check(cudaMemcpy(scalar_, &v, sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
        nccl_check(ncclAllReduce(scalar_, scalar_, 1, ncclDouble, ncclMin, comm_, nullptr), "ncclAllReduce");
        cuda_check(cudaMemcpy(&v, scalar_, sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
        return v;
    }

private:
    ncclComm_t comm_;
    int rank_ = 0, size_ = 1;
    double* scalar_ = nullptr;
};

}  // namespace

std::unique_ptr<SlabComm> make_nccl_comm(ncclComm_t comm) { return std::make_unique<NcclComm>(comm); }

size_t dist_child_size(int n, int parts, int i) { return (size_t)(n / parts + (i < n % parts ? 1 : 0)); }

DistGrid::DistGrid(int dim, const int* n, const double* d, int ghosts, SlabComm& comm, const Config& cfg)
    : dim_(dim), cfg_(cfg), comm_(comm) {
    parts_ = comm.size();
    rank_ = comm.rank();
    for (int a = 0; a < dim; a++) N_[a] = n[a];
    // validGhosts (DistGrid.cpp:27-39) for the unsplit scheme
    g_ = std::max(ghosts, kMHD ? 3 : 2);
    size_t smallest = dist_child_size(N_[0], parts_, parts_ - 1);
    if ((int)smallest < g_)
        throw std::invalid_argument("slabs of " + std::to_string(smallest) + " cells are thinner than the ghost width");
    off_ = 0;
    for (int r = 0; r < rank_; r++) off_ += (int)dist_child_size(N_[0], parts_, r);
    n_[0] = (int)dist_child_size(N_[0], parts_, rank_);
    n_[1] = N_[1];
    n_[2] = N_[2];
    const dragon_config c = cfg.to_c();
    check(dragon_gpu_grid_create(dim, n_[0], dim > 1 ? n_[1] : 1, dim > 2 ? n_[2] : 1, d[0], dim > 1 ? d[1] : 0,
                                 dim > 2 ? d[2] : 0, g_, &c, &h_));
    int dd = 0, nn[3], gg = 0, nf = 0;
    dragon_gpu_grid_info(h_, &dd, nn, &gg, &nf);
    if (gg != g_ || nf != kNF) throw std::logic_error("slab grid does not match the distributed grid");
    faces_ = kMHD && dim >= 2;
    // user fills see global coordinates (dragon_fill_ctx::off)
    check(dragon_gpu_set_origin(h_, off_, 0, 0));
    program();
}

DistGrid::~DistGrid() {
    if (dbuf_) cudaFree(dbuf_);
    if (h_) dragon_gpu_grid_destroy(h_);
}

void DistGrid::check(int rc) const {
    if (rc == 0) return;
    const char* msg = dragon_gpu_last_error();
    if (rc == DRAGON_GPU_EINVAL || rc == DRAGON_GPU_EUNSUPPORTED) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// The slab's boundary list: the global list in order after the implicit Outflow
// over the globally uncovered faces, each element masked to the global faces
// this slab touches; an element periodic in x leaves an Ignore placeholder
// where the first and last slab exchange their layers; a final Ignore over
// every face keeps the device from adding an Outflow between slabs.
void DistGrid::program() {
    int own = kAllFaces & ~Boundary::X;
    if (rank_ == 0) own |= Boundary::X_negative;
    if (rank_ == parts_ - 1) own |= Boundary::X_positive;
    if (boundary.has_user_elements())
        throw std::logic_error("boundary elements with a host apply() are not supported on a DistGrid");
    std::vector<dragon_bc_desc> e;
    // device user fills by entry, each filling the global faces this slab touches
    std::vector<std::tuple<const void*, int, std::vector<double>>> fills;
    std::vector<std::pair<int, const Boundary::DeviceFill*>> fill_at;
    auto entry = [](int type, int faces, int corners, const double* st) {
        dragon_bc_desc d;
        std::memset(&d, 0, sizeof(d));
        d.type = type;
        d.faces = faces;
        d.corners = corners;
        if (st) std::memcpy(d.state, st, sizeof(double) * kNF);
        return d;
    };
    const int unc = boundary.uncovered_faces() & kAllFaces;
    if (unc & own) e.push_back(entry(0, unc & own, 1, nullptr));
    wrap_at_ = -1;
    for (size_t k = 0; k < boundary.size(); k++) {
        const GhostFill& el = boundary[k];
        const int f = el.get_faces() & kAllFaces;
        if (el.device_type() == 4 && (f & Boundary::X)) {
            if (wrap_at_ >= 0) throw std::logic_error("more than one element periodic in x");
            wrap_at_ = (int)e.size();
            wrap_corners_ = el.get_corners() ? 1 : 0;
            e.push_back(entry(5, 0, 1, nullptr));
            const int rest = f & ~Boundary::X;
            if (rest && dim_ > 1) e.push_back(entry(4, rest, wrap_corners_, nullptr));
        } else if (el.device_type() == DRAGON_BC_USER) {
            const auto* df = dynamic_cast<const Boundary::DeviceFill*>(&el);
            if (!df) throw std::logic_error("a user boundary entry that is not a Boundary::DeviceFill");
            fill_at.push_back({(int)e.size(), df});
            fills.emplace_back(df->compiled(), df->fill_faces & own, df->params);
            e.push_back(entry(DRAGON_BC_USER, f & own, el.get_corners() ? 1 : 0, nullptr));
        } else {
            e.push_back(entry(el.device_type(), f & own, el.get_corners() ? 1 : 0, el.device_state()));
        }
    }
    e.push_back(entry(5, kAllFaces, 1, nullptr));
    entries_ = e;
    if (pushed_.size() == e.size() && std::memcmp(pushed_.data(), e.data(), sizeof(dragon_bc_desc) * e.size()) == 0 &&
        pushed_fills_ == fills)
        return;
    check(dragon_gpu_set_boundary(h_, e.data(), (int)e.size()));
    if (dragon_gpu_boundary_entries(h_) != (int)e.size()) throw std::logic_error("device list differs from the slab list");
    for (size_t q = 0; q < fill_at.size(); q++) {
        const auto* df = fill_at[q].second;
        const auto& pr = std::get<2>(fills[q]);
        check(dragon_gpu_set_user_fill(h_, fill_at[q].first, df->compiled(), std::get<1>(fills[q]),
                                       df->get_corners() ? 1 : 0, pr.empty() ? nullptr : pr.data(), (int)pr.size()));
    }
    pushed_ = e;
    pushed_fills_ = fills;
}

// Layers sent to / received from the neighbour across `side` (0 low x, 1 high
// x): between slabs the high neighbour's faces [0, g] land on [nl, nl + g]
// (the shared face takes the higher slab's value, DistGrid.cpp:222-250); the
// periodic wrap moves g layers of faces (Periodic.cpp:55-62).
DistGrid::Msg DistGrid::message(int side, bool send, bool wrap, int corners) const {
    const int g = g_, nl = n_[0], high_faces = wrap ? g : g + 1;
    Msg m;
    if (send) {
        if (side == 0) m = {0, g, 0, high_faces, 0, 0};
        else m = {nl - g, g, nl - g, g, 0, 0};
    } else {
        if (side == 0) m = {-g, g, -g, g, 0, 0};
        else m = {nl, g, nl, high_faces, 0, 0};
    }
    long long c = 0;
    check(dragon_gpu_halo_size(h_, 0, m.cn, 0, corners, &c));
    m.nc = (size_t)c;
    if (faces_) {
        check(dragon_gpu_halo_size(h_, 0, m.fn, 1, corners, &c));
        m.nf = (size_t)c;
    }
    return m;
}

void DistGrid::exchange(const std::vector<std::pair<int, int>>& sides_peers, bool wrap, int corners) {
    std::vector<Msg> sm, rm;
    size_t total = 0;
    for (auto [side, peer] : sides_peers) {
        (void)peer;
        sm.push_back(message(side, true, wrap, corners));
        rm.push_back(message(side, false, wrap, corners));
        total += sm.back().nc + sm.back().nf + rm.back().nc + rm.back().nf;
    }
    if (total > dbuf_count_) {
        if (dbuf_) cudaFree(dbuf_);
        dbuf_ = nullptr;
        cuda_check(cudaMalloc(&dbuf_, sizeof(double) * total), "cudaMalloc");
        dbuf_count_ = total;
    }
    std::vector<SlabTransfer> t;
    std::vector<double*> recv_at;
    size_t off = 0;
    for (size_t k = 0; k < sides_peers.size(); k++) {
        double* s = dbuf_ + off;
        off += sm[k].nc + sm[k].nf;
        double* r = dbuf_ + off;
        off += rm[k].nc + rm[k].nf;
        check(dragon_gpu_halo_pack(h_, 0, sm[k].c0, sm[k].cn, 0, corners, s, 1));
        if (sm[k].nf) check(dragon_gpu_halo_pack(h_, 0, sm[k].f0, sm[k].fn, 1, corners, s + sm[k].nc, 1));
        t.push_back(SlabTransfer{sides_peers[k].second, s, sm[k].nc + sm[k].nf, r, rm[k].nc + rm[k].nf});
        recv_at.push_back(r);
    }
    comm_.exchange(t, dragon_gpu_stream(h_));
    for (size_t k = 0; k < sides_peers.size(); k++) {
        check(dragon_gpu_halo_unpack(h_, 0, rm[k].c0, rm[k].cn, 0, corners, recv_at[k], 1));
        if (rm[k].nf) check(dragon_gpu_halo_unpack(h_, 0, rm[k].f0, rm[k].fn, 1, corners, recv_at[k] + rm[k].nc, 1));
    }
}

void DistGrid::apply_range(int first, int count) {
    if (count > 0) check(dragon_gpu_apply_boundary_range(h_, first, count));
}

void DistGrid::apply_boundary() {
    program();
    const int n = (int)entries_.size();
    if (wrap_at_ < 0) {
        apply_range(0, n);
    } else {
        apply_range(0, wrap_at_);
        if (parts_ == 1) {
            // one slab periodic in x wraps onto itself
            const Msg lo_s = message(1, true, true, wrap_corners_), hi_s = message(0, true, true, wrap_corners_);
            const Msg lo_r = message(0, false, true, wrap_corners_), hi_r = message(1, false, true, wrap_corners_);
            const size_t total = lo_s.nc + lo_s.nf + hi_s.nc + hi_s.nf;
            if (total > dbuf_count_) {
                if (dbuf_) cudaFree(dbuf_);
                dbuf_ = nullptr;
                cuda_check(cudaMalloc(&dbuf_, sizeof(double) * total), "cudaMalloc");
                dbuf_count_ = total;
            }
            double* a = dbuf_;
            double* b = dbuf_ + lo_s.nc + lo_s.nf;
            const int c = wrap_corners_;
            check(dragon_gpu_halo_pack(h_, 0, lo_s.c0, lo_s.cn, 0, c, a, 1));
            if (lo_s.nf) check(dragon_gpu_halo_pack(h_, 0, lo_s.f0, lo_s.fn, 1, c, a + lo_s.nc, 1));
            check(dragon_gpu_halo_pack(h_, 0, hi_s.c0, hi_s.cn, 0, c, b, 1));
            if (hi_s.nf) check(dragon_gpu_halo_pack(h_, 0, hi_s.f0, hi_s.fn, 1, c, b + hi_s.nc, 1));
            check(dragon_gpu_halo_unpack(h_, 0, lo_r.c0, lo_r.cn, 0, c, a, 1));
            if (lo_r.nf) check(dragon_gpu_halo_unpack(h_, 0, lo_r.f0, lo_r.fn, 1, c, a + lo_r.nc, 1));
            check(dragon_gpu_halo_unpack(h_, 0, hi_r.c0, hi_r.cn, 0, c, b, 1));
            if (hi_r.nf) check(dragon_gpu_halo_unpack(h_, 0, hi_r.f0, hi_r.fn, 1, c, b + hi_r.nc, 1));
            comm_.exchange({}, dragon_gpu_stream(h_));
        } else if (rank_ == 0) {
            exchange({{0, parts_ - 1}}, true, wrap_corners_);
        } else if (rank_ == parts_ - 1) {
            exchange({{1, 0}}, true, wrap_corners_);
        } else {
            comm_.exchange({}, dragon_gpu_stream(h_));
        }
        apply_range(wrap_at_ + 1, n - wrap_at_ - 1);
    }
    std::vector<std::pair<int, int>> pairs;
    if (rank_ > 0) pairs.push_back({0, rank_ - 1});
    if (rank_ < parts_ - 1) pairs.push_back({1, rank_ + 1});
    if (pairs.empty()) comm_.exchange({}, dragon_gpu_stream(h_));
    else exchange(pairs, false, 1);
}

double DistGrid::cfl_time() {
    double dt = 0;
    const int rc = dragon_gpu_cfl_time(h_, &dt);
    if (rc == DRAGON_GPU_ECFL) dt = std::numeric_limits<double>::infinity();
    else check(rc);
    dt = comm_.allreduce_min(dt);
    if (std::isinf(dt)) throw std::runtime_error("CFL timestep failed: max signal speed is zero");
    return dt;
}

bool DistGrid::try_step(double dt) {
    dragon_step_status st;
    const int rc = dragon_gpu_unsplit_step(h_, dt, &st);
    if (rc == DRAGON_GPU_ESTEP) return false;
    check(rc);
    return true;
}

void DistGrid::unsplit_step(double dt) {
    const bool ok = try_step(dt);
    if (comm_.allreduce_min(ok ? 1.0 : 0.0) < 1.0) {
        if (ok) check(dragon_gpu_step_rollback(h_));
        throw SlabStepFailed("a slab of the distributed grid failed its step");
    }
}

double DistGrid::step_with_retry(double t1) {
    for (;;) {
        try {
            unsplit_step(t1);
            return t1;
        } catch (const SlabStepFailed&) {
            retries_++;
            t1 *= 0.5;
            if (t1 < cfg_.timestep_tol) throw std::runtime_error("Timestep has fallen below minimum");
        }
    }
}

void DistGrid::advance(double dt, bool check_cfl) {
    while (dt > cfg_.timestep_tol) {
        apply_boundary();
        double t1 = check_cfl ? std::min(dt, cfl_time()) : dt;
        t1 = step_with_retry(t1);
        dt -= t1;
        steps_++;
    }
}

void DistGrid::advance_steps(int nsteps) {
    for (int s = 0; s < nsteps; s++) {
        apply_boundary();
        step_with_retry(cfl_time());
        steps_++;
    }
}

void DistGrid::initialize_B_fields() {
    if (!faces_) throw std::invalid_argument("grid has no face-centred B");
    apply_boundary();
    check(dragon_gpu_initialize_B_fields(h_));
}

void DistGrid::scatter(const PrimitiveState* global, const vec3* global_B) {
    const size_t row = (size_t)(dim_ > 1 ? N_[1] + 2 * g_ : 1) * (dim_ > 2 ? N_[2] + 2 * g_ : 1);
    check(dragon_gpu_upload_prim(h_, &global[(size_t)off_ * row].rho));
    if (faces_) {
        if (!global_B) throw std::invalid_argument("an MHD grid needs its face-centred B");
        const size_t frow = (size_t)(N_[1] + 1 + 2 * g_) * (dim_ > 2 ? N_[2] + 1 + 2 * g_ : 1);
        check(dragon_gpu_upload_faceB(h_, &global_B[(size_t)off_ * frow].x));
    }
}

void DistGrid::gather(PrimitiveState* global, vec3* global_B) const {
    const size_t row = (size_t)(dim_ > 1 ? N_[1] + 2 * g_ : 1) * (dim_ > 2 ? N_[2] + 2 * g_ : 1);
    const int nl = n_[0], g = g_;
    std::vector<PrimitiveState> w((size_t)(nl + 2 * g) * row);
    check(dragon_gpu_download_prim(h_, &w[0].rho));
    const int lo = rank_ == 0 ? 0 : g, hi = rank_ == parts_ - 1 ? nl + 2 * g : g + nl;
    std::copy(w.begin() + (size_t)lo * row, w.begin() + (size_t)hi * row, global + (size_t)(off_ + lo) * row);
    if (faces_ && global_B) {
        const size_t frow = (size_t)(N_[1] + 1 + 2 * g) * (dim_ > 2 ? N_[2] + 1 + 2 * g : 1);
        std::vector<vec3> B((size_t)(nl + 1 + 2 * g) * frow);
        check(dragon_gpu_download_faceB(h_, &B[0].x));
        const int fhi = rank_ == parts_ - 1 ? nl + 1 + 2 * g : g + nl;
        std::copy(B.begin() + (size_t)lo * frow, B.begin() + (size_t)fhi * frow, global_B + (size_t)(off_ + lo) * frow);
    }
}

DistGrid1D::DistGrid1D(int nx, double dx, int ghosts, SlabComm& comm, const Config& cfg)
    : DistGrid(1, std::array<int, 3>{nx, 1, 1}.data(), std::array<double, 3>{dx, 0, 0}.data(), ghosts, comm, cfg) {}
DistGrid2D::DistGrid2D(int nx, int ny, double dx, double dy, int ghosts, SlabComm& comm, const Config& cfg)
    : DistGrid(2, std::array<int, 3>{nx, ny, 1}.data(), std::array<double, 3>{dx, dy, 0}.data(), ghosts, comm, cfg) {}
DistGrid3D::DistGrid3D(int nx, int ny, int nz, double dx, double dy, double dz, int ghosts, SlabComm& comm,
                       const Config& cfg)
    : DistGrid(3, std::array<int, 3>{nx, ny, nz}.data(), std::array<double, 3>{dx, dy, dz}.data(), ghosts, comm, cfg) {}

}  // namespace dragon
