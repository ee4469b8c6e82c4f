// dragon_b200 C++23 host API: DRAGON's user-facing Grid / Boundary /
// PrimitiveState interface (DRAGON/Hydro/Grid.hpp:19-144,
// DRAGON/Boundary/Boundary.hpp:19-132, DRAGON/Boundary/BoundaryList.hpp:15-128,
// DRAGON/Boundary/GhostFill.hpp:16-30, DRAGON/FluidElement/FluidElement.hpp:18-68)
// with the state resident on the GPU behind the C ABI of dragon_gpu.h.
//
// Code written against the reference compiles against this header after
// `using namespace dragon;`:
//
//     Grid2D grid(nx, ny, 1.0 / nx, 1.0 / ny);
//     grid.boundary = Boundary::Reflective("X") + Boundary::Periodic("YZ");
//     grid[i, j] = w;                 // host mirror, uploaded before the next device call
//     grid.advance(dt);               // the whole advance loop runs on the device
//
// Physics is chosen like the reference: define MHD (or include the
// reference's Config.h, which does) before this header for MHD grids, and link
// libdragon_host_mhd.so instead of libdragon_host.so. The reference's
// compile-time switches (RIEMANN_DEFAULT, MUSCL_DEFAULT_LIMITER,
// CFL_CALCULATION, CT_ENERGY_CONSV and the CONFIG:: constants) become the
// runtime dragon::Config that grids are built with; when the reference's
// Config.h was included first its values are taken over (Config::from_reference).
//
// The host mirror of a grid is the padded array in the reference's memory
// order (last index fastest, ghosts included, PrimitiveState layout), synced
// lazily: mutable access marks it newer than the device (uploaded before the
// next device call), a device call marks the device newer (downloaded on the
// next access). A reference returned by operator[] is valid until the next
// device call on the grid.
#pragma once

#include <cmath>
#include <concepts>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "../dragon_gpu.h"

namespace dragon {

#ifdef MHD
inline constexpr bool kMHD = true;
#else
inline constexpr bool kMHD = false;
#endif

// ---------------------------------------------------------------------------
// FluidElement (FluidElement.hpp:18-68)

struct vec3 {
    double x, y, z;
    vec3(double x_ = 0, double y_ = 0, double z_ = 0) : x(x_), y(y_), z(z_) {}
    vec3 swappedXY() const { return {y, x, z}; }
    vec3 swappedXZ() const { return {z, y, x}; }
    vec3 swappedYZ() const { return {x, z, y}; }
    void swapXY() { std::swap(x, y); }
    void swapXZ() { std::swap(x, z); }
    void swapYZ() { std::swap(y, z); }
};

struct PrimitiveState {
    double rho, p;
    vec3 v;
#ifdef MHD
    vec3 B;
#endif
    PrimitiveState() : rho(0), p(0) {}

    // Ideal gas, gamma = 5/3 (Constants.h:18); Gaussian-unit magnetic energy.
    double energy() const;
    double enthalpy() const;
    double cs() const;
    bool isPhysical() const;
};
static_assert(sizeof(vec3) == 3 * sizeof(double));
static_assert(sizeof(PrimitiveState) == (kMHD ? 8 : 5) * sizeof(double),
              "PrimitiveState must match the C ABI's per-cell field layout");

// ---------------------------------------------------------------------------
// Config.h's switches at run time

struct Config {
    int riemann = 5;          // RIEMANN_HLLX
    int limiter = 1;          // LIMITER_MC
    int cfl = 1;              // CFL_ADD
    int ct_energy = 2;        // CT_CONSV_BETA_GATED
    int exact_max_iters = 6;  // ExactRiemann_MaxIters
    double exact_tol = 1e-12; // ExactRiemann_Tolerance
    double cfl_coeff = 0.3;   // CFL_coeff
    double timestep_tol = 1e-14;  // Timestep_Tolerance
    int precision = 0;        // 0 FP64 (bit-faithful), 1 mixed FP32/FP64
    int exact_guess = 0;      // 0 the reference's mean guess, 1 adaptive, 2 learned

    dragon_config to_c() const;
    // The reference's Config.h values when it was included before this header.
    static Config from_reference();
};

// Process-wide defaults the grid constructors use (Config.h is global in the
// reference too).
Config& default_config();

inline Config Config::from_reference() {
    Config c;
#ifdef Config_h
#if defined(RIEMANN_DEFAULT) && RIEMANN_DEFAULT >= 0
    c.riemann = RIEMANN_DEFAULT;
#endif
#if defined(MUSCL_DEFAULT_LIMITER) && MUSCL_DEFAULT_LIMITER >= 0
    c.limiter = MUSCL_DEFAULT_LIMITER;
#endif
#if defined(CFL_CALCULATION) && CFL_CALCULATION >= 0
    c.cfl = CFL_CALCULATION;
#endif
#if defined(CT_ENERGY_CONSV) && CT_ENERGY_CONSV >= 0
    c.ct_energy = CT_ENERGY_CONSV;
#endif
    c.exact_max_iters = CONFIG::ExactRiemann_MaxIters;
    c.exact_tol = CONFIG::ExactRiemann_Tolerance;
    c.cfl_coeff = CONFIG::CFL_coeff;
    c.timestep_tol = CONFIG::Timestep_Tolerance;
#endif
    return c;
}

class Grid;
class Grid1D;
class Grid2D;
class Grid3D;

// ---------------------------------------------------------------------------
// Boundary (GhostFill.hpp, Boundary.hpp, BoundaryList.hpp)

class GhostFill {
public:
    virtual ~GhostFill() = default;
    int get_faces() const { return faces; }
    bool get_corners() const { return corners; }

    // Fill the ghost cells of `grid`. Built-in elements run on the device. A
    // user element (the reference's Jet pattern, Jets.hpp:12-39) overrides
    // these and fills through grid[i, j] on the host mirror; a grid whose list
    // holds one runs its advance loop from the host.
    virtual void apply(Grid1D& grid);
    virtual void apply(Grid2D& grid);
    virtual void apply(Grid3D& grid);
    void apply(Grid& grid);

    // Device entry type (dragon_bc_desc::type) of a built-in element, -1 for a
    // user element.
    virtual int device_type() const { return -1; }
    virtual const double* device_state() const { return nullptr; }

protected:
    int faces;
    bool corners;
    explicit GhostFill(int faces_, bool corner_ghosts) : faces(faces_), corners(corner_ghosts) {}
    // A built-in element applied on its own, on the device.
    void apply_device(Grid& grid) const;
};

namespace Boundary {

class BoundaryList;
template <class T>
concept BoundaryElement = !std::derived_from<std::decay_t<T>, BoundaryList> && std::derived_from<std::decay_t<T>, GhostFill>;

constexpr int X_negative = 1 << 0;
constexpr int X_positive = 1 << 1;
constexpr int X = X_negative | X_positive;
constexpr int Y_negative = 1 << 2;
constexpr int Y_positive = 1 << 3;
constexpr int Y = Y_negative | Y_positive;
constexpr int Z_negative = 1 << 4;
constexpr int Z_positive = 1 << 5;
constexpr int Z = Z_negative | Z_positive;

// GhostFill.cpp:14-48: "X", "Y-", "XZ+", and L / R / U / D.
int face_mask(std::string s);

class Outflow : public GhostFill {
public:
    Outflow(std::string faces, bool corner_ghosts = true, bool gated = false)
        : Outflow(face_mask(std::move(faces)), corner_ghosts, gated) {}
    Outflow(int faces = X | Y | Z, bool corner_ghosts = true, bool gated_ = false)
        : GhostFill(faces, corner_ghosts), gated(gated_) {}
    static Outflow Gated(std::string faces, bool corner_ghosts = true) { return Outflow(std::move(faces), corner_ghosts, true); }
    static Outflow Gated(int faces = X | Y | Z, bool corner_ghosts = true) { return Outflow(faces, corner_ghosts, true); }
    int device_type() const override { return gated ? 1 : 0; }
    bool gated;
};

class Fixed : public GhostFill {
public:
    Fixed(PrimitiveState s, std::string faces, bool corner_ghosts = true)
        : Fixed(s, face_mask(std::move(faces)), corner_ghosts) {}
    Fixed(PrimitiveState s, int faces = X | Y | Z, bool corner_ghosts = true) : GhostFill(faces, corner_ghosts), state(s) {}
    int device_type() const override { return 2; }
    const double* device_state() const override { return &state.rho; }

protected:
    PrimitiveState state;
};

class Reflective : public GhostFill {
public:
    Reflective(std::string faces, bool corner_ghosts = true) : Reflective(face_mask(std::move(faces)), corner_ghosts) {}
    Reflective(int faces = X | Y | Z, bool corner_ghosts = true) : GhostFill(faces, corner_ghosts) {}
    int device_type() const override { return 3; }
};

class Periodic : public GhostFill {
public:
    // Periodic.cpp:14-15: either face of an axis selects both.
    Periodic(std::string faces, bool corner_ghosts = true) : Periodic(face_mask(std::move(faces)), corner_ghosts) {}
    Periodic(int faces = X | Y | Z, bool corner_ghosts = true)
        : GhostFill(((faces & X) ? X : 0) | ((faces & Y) ? Y : 0) | ((faces & Z) ? Z : 0), corner_ghosts) {}
    int device_type() const override { return 4; }
};

class Ignore : public GhostFill {
public:
    Ignore(std::string faces, bool corner_ghosts = true) : Ignore(face_mask(std::move(faces)), corner_ghosts) {}
    Ignore(int faces = X | Y | Z, bool corner_ghosts = true) : GhostFill(faces, corner_ghosts) {}
    int device_type() const override { return 5; }
};

// A user element compiled for the device (dragon_gpu_user_fill_create):
// `source` defines __device__ void <function>(const dragon_fill_ctx& c, int i,
// int j, int k), called for every ghost cell of `fill_faces` (the contract is
// in dragon_gpu.h). It runs at its place in the list inside the device
// advance loop, with no host round trip; `faces` keeps its BoundaryList
// meaning (the reference's Jet claims none, GhostFill(0, true)). Throws
// std::runtime_error with NVRTC's log when the source does not compile.
class DeviceFill : public GhostFill {
public:
    DeviceFill(const std::string& source, const std::string& function, int faces, int fill_faces,
               std::vector<double> params = {}, bool corner_ghosts = true);
    DeviceFill(const std::string& source, const std::string& function, std::string faces, std::string fill_faces,
               std::vector<double> params = {}, bool corner_ghosts = true)
        : DeviceFill(source, function, face_mask(std::move(faces)), face_mask(std::move(fill_faces)),
                     std::move(params), corner_ghosts) {}
    int device_type() const override { return DRAGON_BC_USER; }
    dragon_user_fill* compiled() const { return fill_.get(); }
    int fill_faces;
    std::vector<double> params;

private:
    std::shared_ptr<dragon_user_fill> fill_;
};

// Elements applied in order after an implicit Outflow over every face no
// element covers (BoundaryList.hpp:79-104). Move-only, like the reference's.
class BoundaryList : public GhostFill {
public:
    using GhostFill::apply;

    template <BoundaryElement... Bs>
    BoundaryList(Bs&&... bs) : GhostFill(X | Y | Z, true) {
        (append(std::forward<Bs>(bs)), ...);
    }
    BoundaryList(const BoundaryList&) = delete;
    BoundaryList(BoundaryList&&) noexcept = default;
    BoundaryList& operator=(BoundaryList&&) noexcept = default;
    template <BoundaryElement B>
    BoundaryList& operator=(B&& b) {
        clear();
        append(std::forward<B>(b));
        return *this;
    }

    template <BoundaryElement B>
    void append(B&& b) {
        elements.push_back(std::make_unique<std::decay_t<B>>(std::forward<B>(b)));
    }
    void append(BoundaryList&& bs) {
        for (auto& b : bs.elements) elements.push_back(std::move(b));
        bs.elements.clear();
    }
    template <BoundaryElement B>
    void prepend(B&& b) {
        elements.insert(elements.begin(), std::make_unique<std::decay_t<B>>(std::forward<B>(b)));
    }
    void prepend(BoundaryList&& bs) {
        bs.append(std::move(*this));
        elements = std::move(bs.elements);
    }
    void clear() { elements.clear(); }

    void apply(Grid1D& grid) override;
    void apply(Grid2D& grid) override;
    void apply(Grid3D& grid) override;

    size_t size() const { return elements.size(); }
    const GhostFill& operator[](size_t k) const { return *elements[k]; }
    GhostFill& operator[](size_t k) { return *elements[k]; }
    bool has_user_elements() const;
    // The faces no element covers (the implicit Outflow's, BoundaryList.hpp:97-104).
    int uncovered_faces() const;
    // The device list: one descriptor per element, in order (user elements as
    // Ignore entries over their faces); the device prepends the implicit Outflow.
    std::vector<dragon_bc_desc> descriptors() const;

private:
    std::vector<std::unique_ptr<GhostFill>> elements;
};

template <BoundaryElement A, BoundaryElement B>
BoundaryList operator+(A&& a, B&& b) {
    BoundaryList r;
    r.append(std::forward<A>(a));
    r.append(std::forward<B>(b));
    return r;
}
template <BoundaryElement B>
BoundaryList& operator+=(BoundaryList& lhs, B&& rhs) {
    lhs.append(std::forward<B>(rhs));
    return lhs;
}
template <BoundaryElement B>
BoundaryList operator+(BoundaryList lhs, B&& rhs) {
    lhs += std::forward<B>(rhs);
    return lhs;
}
template <BoundaryElement A>
BoundaryList operator+(A&& lhs, BoundaryList rhs) {
    rhs.prepend(std::forward<A>(lhs));
    return rhs;
}
inline BoundaryList& operator+=(BoundaryList& lhs, BoundaryList rhs) {
    lhs.append(std::move(rhs));
    return lhs;
}
inline BoundaryList operator+(BoundaryList lhs, BoundaryList rhs) {
    lhs += std::move(rhs);
    return lhs;
}

}  // namespace Boundary

// ---------------------------------------------------------------------------
// Grids (Grid.hpp:19-144)

// Statistics of the last device advance (solver pivots, Newton iterations...).
using AdvanceStats = dragon_advance_stats;

class Grid {
public:
    Grid(const Grid&) = delete;
    Grid& operator=(const Grid&) = delete;
    virtual ~Grid();

    // Grid::advance / advance_split / advance_unsplit (CFL.cpp:151-213): the
    // loop runs on the device; with user boundary elements it runs from the
    // host with the same steps. Throws std::runtime_error where the reference
    // throws, and where it exits (the retried step fell below the tolerance).
    void advance(double dt, bool check_cfl = true);
    void advance_split(double dt, bool check_cfl = true);
    void advance_unsplit(double dt, bool check_cfl = true);
    // nsteps CFL-limited unsplit steps, each the reference's advance(cfl_time()).
    void advance_steps(int nsteps);

    // Grid::split_step / unsplit_step (Splitting.cpp:118-299, Unsplit.cpp:28-206):
    // commit nothing and throw std::runtime_error when the step fails.
    virtual void split_step(double dt);
    virtual void unsplit_step(double dt);
    // Grid::on_step_fail (Unsplit.cpp:21-23): true = halve dt and retry. Called
    // by the host-driven loop (grids with user boundary elements).
    virtual bool on_step_fail(const std::exception& e);
    // Grid::initialize_B_fields (B_fields.cpp:117-149), MHD 2D / 3D.
    virtual void initialize_B_fields();

    // CFL::cfl_time (CFL.cpp:88-137) on the current ghosts.
    double cfl_time();
    // boundary.apply(*this) with the grid's list.
    void apply_boundary();

    Boundary::BoundaryList boundary = Boundary::BoundaryList();

    // GPU side
    dragon_grid* handle() const { return h_; }
    const Config& config() const { return cfg_; }
    const AdvanceStats& last_advance() const { return stats_; }
    void upload();    // host mirror -> device now
    void download();  // device -> host mirror now
    // For callers of the C ABI on handle(): make the device state current
    // (host-side edits uploaded first), and record that the device state
    // changed behind the host mirror (it refreshes on its next access).
    void sync_device() { to_device(); }
    void device_changed() { dev_newer_ = true; }
    int getGhosts() const { return g_; }

protected:
    Grid(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts, const Config& cfg);
    PrimitiveState& cell(long long k);
    const PrimitiveState& cell(long long k) const;
    vec3& face(long long k);
    long long index(int i, int j, int k) const;
    long long face_index(int i, int j, int k) const;
    void to_device();
    void host_current() const;
    void push_boundary();
    void apply_boundary_host();
    void advance_host(double dt, bool check_cfl, bool split);
    void step_call(bool split, double dt);
    [[noreturn]] void raise(int rc) const;

    int dim_ = 0, n_[3] = {1, 1, 1}, g_ = 0, nf_ = 0;
    Config cfg_;
    dragon_grid* h_ = nullptr;
    mutable std::vector<PrimitiveState> w_;
    mutable std::vector<vec3> B_;
    mutable bool dev_newer_ = false;
    bool host_newer_ = true;
    std::vector<dragon_bc_desc> pushed_;
    // device fills bound with the pushed list: (fill, fill faces, params) per entry
    std::vector<std::tuple<const void*, int, std::vector<double>>> pushed_fills_;
    bool pushed_valid_ = false;
    AdvanceStats stats_{};

    friend class GhostFill;
    friend class Boundary::BoundaryList;
};

class Grid1D : public Grid {
public:
    double dx;
    Grid1D(int size, double dx_, int ghosts = 1, const Config& cfg = default_config());
    PrimitiveState& operator[](int k) { return cell(index(k, 0, 0)); }
    const PrimitiveState& operator[](int k) const { return cell(index(k, 0, 0)); }
    int getSize() const { return n_[0]; }
};

class Grid2D : public Grid {
public:
    double dx, dy;
    Grid2D(int nx, int ny, double dx_, double dy_, int ghosts = 1, const Config& cfg = default_config());
    PrimitiveState& operator[](int i, int j) { return cell(index(i, j, 0)); }
    const PrimitiveState& operator[](int i, int j) const { return cell(index(i, j, 0)); }
    int getSizeX() const { return n_[0]; }
    int getSizeY() const { return n_[1]; }
#ifdef MHD
    // Face-centred B, n + 1 positions per axis with the same ghosts (Grid.hpp:83).
    struct FaceB {
        Grid2D* g;
        vec3& operator[](int i, int j) { return g->face(g->face_index(i, j, 0)); }
    };
    FaceB& _B() { return faceB_; }

private:
    FaceB faceB_{this};
#endif
};

class Grid3D : public Grid {
public:
    double dx, dy, dz;
    Grid3D(int nx, int ny, int nz, double dx_, double dy_, double dz_, int ghosts = 2, const Config& cfg = default_config());
    PrimitiveState& operator[](int i, int j, int k) { return cell(index(i, j, k)); }
    const PrimitiveState& operator[](int i, int j, int k) const { return cell(index(i, j, k)); }
    int getSizeX() const { return n_[0]; }
    int getSizeY() const { return n_[1]; }
    int getSizeZ() const { return n_[2]; }
#ifdef MHD
    struct FaceB {
        Grid3D* g;
        vec3& operator[](int i, int j, int k) { return g->face(g->face_index(i, j, k)); }
    };
    FaceB& _B() { return faceB_; }

private:
    FaceB faceB_{this};
#endif
};

}  // namespace dragon
