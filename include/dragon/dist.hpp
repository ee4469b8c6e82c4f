// DistGrid1D / DistGrid2D / DistGrid3D over several GPUs for C++ hosts: the
// reference's DistGrid (DRAGON/Refinement/DistGrid.hpp:17-86,
// DistGrid.cpp:21-360) with its children on GPUs instead of pthreads.
//
// One rank per GPU (a process, or a thread with its own device current). The
// x axis is cut into slabs sized by computeChildSize (DistGrid.cpp:21-25), each
// with validGhosts' width (:27-39); rank r holds slab r on its GPU. One step:
//   1. the slab's part of the boundary list fills its ghosts on the device (an
//      element periodic in x becomes an exchange between the first and last
//      slab, at its place in the list);
//   2. halo exchange with the x neighbours: ghost-width layers of cells, and of
//      face-centred B for MHD, packed on the device into one buffer per peer;
//   3. every slab's CFL time, all-reduced to the minimum (CFL_coeff / max_speed
//      is monotone in max_speed, so this is the serial grid's CFL time);
//   4. every slab steps; an all-reduce of the success flags commits all slabs
//      or none (dragon_gpu_step_rollback) and the step is retried at half dt.
// The result is the serial grid's, bit for bit.
//
// The transport is a SlabComm: make_nccl_comm() wraps an NCCL communicator
// (device buffers, ncclSend / ncclRecv / ncclAllReduce on the slab's stream);
// a caller can supply any other. Link libdragon_dist.so (MHD:
// libdragon_dist_mhd.so), which needs libnccl and libcudart.
#pragma once

#include <memory>
#include <tuple>
#include <vector>

#include "dragon.hpp"

typedef struct ncclComm* ncclComm_t;

namespace dragon {

// One send to and one receive from `peer`, in device memory of the calling
// rank's GPU (the two sizes differ for face-centred B: the shared face travels
// one way only).
struct SlabTransfer {
    int peer;
    const double* send;
    size_t send_count;
    double* recv;
    size_t recv_count;
};

class SlabComm {
public:
    virtual ~SlabComm() = default;
    virtual int rank() const = 0;
    virtual int size() const = 0;
    // Collective: every rank calls it for every exchange phase, possibly with
    // no transfers. `stream` is the slab's CUDA stream (cudaStream_t); the
    // send buffers are ready on it, and the receive buffers must be complete
    // on it when the call returns.
    virtual void exchange(const std::vector<SlabTransfer>& transfers, void* stream) = 0;
    // Collective minimum of one double.
    virtual double allreduce_min(double v) = 0;
};

// NCCL transport over an existing communicator (not owned).
std::unique_ptr<SlabComm> make_nccl_comm(ncclComm_t comm);

size_t dist_child_size(int n, int parts, int i);  // computeChildSize

class DistGrid {
public:
    DistGrid(const DistGrid&) = delete;
    DistGrid& operator=(const DistGrid&) = delete;
    virtual ~DistGrid();

    Boundary::BoundaryList boundary = Boundary::BoundaryList();

    // pushToChildren (DistGrid.cpp:115-204): this rank's slab of a padded
    // global array in the reference's order (every rank passes the same array;
    // B: the padded face array, MHD 2D / 3D).
    void scatter(const PrimitiveState* global, const vec3* global_B = nullptr);
    // loadFromChildren (DistGrid.cpp:208-289) for this rank's part: writes the
    // slab's interior x layers (the outer slabs also their x ghosts) into the
    // padded global array. Every rank writes its part; a caller that wants the
    // whole array on one rank gathers the parts itself.
    void gather(PrimitiveState* global, vec3* global_B = nullptr) const;

    void apply_boundary();
    double cfl_time();
    // DistGrid<T>::step (DistGrid.cpp:292-304): all slabs or none; throws
    // std::runtime_error when a slab failed (nothing committed).
    void unsplit_step(double dt);
    // Grid::advance_unsplit (CFL.cpp:188-213) over the slabs.
    void advance(double dt, bool check_cfl = true);
    // nsteps CFL-limited steps.
    void advance_steps(int nsteps);
    void initialize_B_fields();

    int ghosts() const { return g_; }
    int offset() const { return off_; }        // first global x cell of this slab
    int slab_size() const { return n_[0]; }    // x cells of this slab
    dragon_grid* handle() const { return h_; }
    int steps() const { return steps_; }
    int retries() const { return retries_; }

protected:
    DistGrid(int dim, const int* n, const double* d, int ghosts, SlabComm& comm, const Config& cfg);

private:
    struct Msg { int c0, cn, f0, fn; size_t nc, nf; };
    void program();
    Msg message(int side, bool send, bool wrap, int corners) const;
    void exchange(const std::vector<std::pair<int, int>>& sides_peers, bool wrap, int corners);
    void apply_range(int first, int count);
    void check(int rc) const;
    bool try_step(double dt);
    double step_with_retry(double t1);

    int dim_;
    int N_[3] = {1, 1, 1}, n_[3] = {1, 1, 1};
    int g_ = 0, off_ = 0, parts_ = 1, rank_ = 0;
    bool faces_ = false;
    Config cfg_;
    SlabComm& comm_;
    dragon_grid* h_ = nullptr;
    std::vector<dragon_bc_desc> entries_;
    int wrap_at_ = -1, wrap_corners_ = 1;
    std::vector<dragon_bc_desc> pushed_;
    // device user fills bound with the pushed list: (fill, faces filled on this slab, params) per entry
    std::vector<std::tuple<const void*, int, std::vector<double>>> pushed_fills_;
    double* dbuf_ = nullptr;  // device send / receive buffers
    size_t dbuf_count_ = 0;
    int steps_ = 0, retries_ = 0;
};

class DistGrid1D : public DistGrid {
public:
    DistGrid1D(int nx, double dx, int ghosts, SlabComm& comm, const Config& cfg = default_config());
};
class DistGrid2D : public DistGrid {
public:
    DistGrid2D(int nx, int ny, double dx, double dy, int ghosts, SlabComm& comm, const Config& cfg = default_config());
};
class DistGrid3D : public DistGrid {
public:
    DistGrid3D(int nx, int ny, int nz, double dx, double dy, double dz, int ghosts, SlabComm& comm,
               const Config& cfg = default_config());
};

}  // namespace dragon
