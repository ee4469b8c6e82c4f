// C++23 host layer over the C ABI (include/dragon/dragon.hpp): the reference's
// Grid / Boundary API with the state on the GPU. Built twice, like the
// reference's MHD switch: libdragon_host.so (hydro) and, with -DMHD,
// libdragon_host_mhd.so.
#include "../../include/dragon/dragon.hpp"
#include "../../include/dragon/hoard.hpp"

#include <cctype>
#include <filesystem>
#include <cstring>
#include <iostream>

namespace dragon {

namespace {
constexpr double kGamma = 5.0 / 3.0;
constexpr double k1_8pi = 1.0 / (8.0 * 3.14159265358979323846);
constexpr int kNF = kMHD ? 8 : 5;
}  // namespace

// ---------------------------------------------------------------------------
// FluidElement (FluidElement.cpp:53-96)

double PrimitiveState::energy() const {
    double e = p / (kGamma - 1.0) + 0.5 * rho * (v.x * v.x + v.y * v.y + v.z * v.z);
#ifdef MHD
    e += (B.x * B.x + B.y * B.y + B.z * B.z) * k1_8pi;
#endif
    return e;
}

double PrimitiveState::enthalpy() const {
    double h = energy() + p;
#ifdef MHD
    h += (B.x * B.x + B.y * B.y + B.z * B.z) * k1_8pi;
#endif
    return h / rho;
}

double PrimitiveState::cs() const { return std::sqrt(kGamma * p / rho); }

bool PrimitiveState::isPhysical() const {
    bool ok = std::isfinite(rho) && std::isfinite(p) && std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) &&
              rho > 0 && p > 0;
#ifdef MHD
    ok = ok && std::isfinite(B.x) && std::isfinite(B.y) && std::isfinite(B.z);
#endif
    return ok;
}

// ---------------------------------------------------------------------------
// Config

dragon_config Config::to_c() const {
    dragon_config c;
    dragon_gpu_default_config(&c, kMHD ? 1 : 0);
    c.riemann = riemann;
    c.limiter = limiter;
    c.cfl = cfl;
    c.ct_energy = ct_energy;
    c.exact_max_iters = exact_max_iters;
    c.exact_tol = exact_tol;
    c.cfl_coeff = cfl_coeff;
    c.timestep_tol = timestep_tol;
    c.precision = precision;
    c.exact_guess = exact_guess;
    return c;
}

Config& default_config() {
    static Config c;
    return c;
}

// ---------------------------------------------------------------------------
// Boundary

namespace Boundary {

int face_mask(std::string s) {
    int mask = 0;
    s += ' ';
    for (size_t k = 0; k + 1 < s.size(); k++) {
        const char c = (char)std::toupper((unsigned char)s[k]);
        const char nx = s[k + 1];
        auto pick = [&](int neg, int pos) { mask |= nx == '+' ? pos : nx == '-' ? neg : (neg | pos); };
        switch (c) {
            case 'X': pick(X_negative, X_positive); break;
            case 'Y': pick(Y_negative, Y_positive); break;
            case 'Z': pick(Z_negative, Z_positive); break;
            case 'L': mask |= X_negative; break;
            case 'R': mask |= X_positive; break;
            case 'U': mask |= Y_positive; break;
            case 'D': mask |= Y_negative; break;
            default: break;
        }
    }
    return mask;
}

bool BoundaryList::has_user_elements() const {
    for (auto& e : elements)
        if (e->device_type() < 0) return true;
    return false;
}

int BoundaryList::uncovered_faces() const {
    int unc = X | Y | Z;
    for (auto& e : elements) unc &= ~e->get_faces();
    return unc;
}

DeviceFill::DeviceFill(const std::string& source, const std::string& function, int faces, int fill_faces_,
                       std::vector<double> params_, bool corner_ghosts)
    : GhostFill(faces, corner_ghosts), fill_faces(fill_faces_), params(std::move(params_)) {
    dragon_user_fill* f = nullptr;
    if (dragon_gpu_user_fill_create(source.c_str(), function.c_str(), &f)) throw std::runtime_error(dragon_gpu_last_error());
    fill_.reset(f, [](dragon_user_fill* p) { dragon_gpu_user_fill_destroy(p); });
}

std::vector<dragon_bc_desc> BoundaryList::descriptors() const {
    std::vector<dragon_bc_desc> out;
    out.reserve(elements.size());
    for (auto& e : elements) {
        dragon_bc_desc d;
        std::memset(&d, 0, sizeof(d));
        const int t = e->device_type();
        d.type = t < 0 ? 5 : t;  // a user element only covers its faces on the device
        d.faces = e->get_faces();
        d.corners = e->get_corners() ? 1 : 0;
        if (const double* s = e->device_state()) std::memcpy(d.state, s, sizeof(double) * kNF);
        out.push_back(d);
    }
    return out;
}

void BoundaryList::apply(Grid1D& grid) { static_cast<Grid&>(grid).apply_boundary(); }
void BoundaryList::apply(Grid2D& grid) { static_cast<Grid&>(grid).apply_boundary(); }
void BoundaryList::apply(Grid3D& grid) { static_cast<Grid&>(grid).apply_boundary(); }

}  // namespace Boundary

// A built-in element applied on its own: the grid's device list is swapped for
// this element plus an Ignore over every face (so no implicit Outflow runs);
// the grid's own list goes back to the device before its next use.
void GhostFill::apply_device(Grid& g) const {
    if (device_type() < 0)
        throw std::logic_error("a user GhostFill must override apply() for every grid dimension it is used with");
    dragon_bc_desc d[2];
    std::memset(d, 0, sizeof(d));
    d[0].type = device_type();
    d[0].faces = get_faces();
    d[0].corners = get_corners() ? 1 : 0;
    if (const double* s = device_state()) std::memcpy(d[0].state, s, sizeof(double) * kNF);
    d[1].type = 5;
    d[1].faces = 63;
    d[1].corners = 1;
    if (g.host_newer_) g.upload();
    g.pushed_valid_ = false;
    int rc = dragon_gpu_set_boundary(g.h_, d, 2);
    if (!rc) rc = dragon_gpu_apply_boundary(g.h_);
    if (rc) g.raise(rc);
    g.dev_newer_ = true;
}

void GhostFill::apply(Grid1D& grid) { apply_device(grid); }
void GhostFill::apply(Grid2D& grid) { apply_device(grid); }
void GhostFill::apply(Grid3D& grid) { apply_device(grid); }
void GhostFill::apply(Grid& grid) {
    if (auto* g1 = dynamic_cast<Grid1D*>(&grid)) return apply(*g1);
    if (auto* g2 = dynamic_cast<Grid2D*>(&grid)) return apply(*g2);
    if (auto* g3 = dynamic_cast<Grid3D*>(&grid)) return apply(*g3);
}

// ---------------------------------------------------------------------------
// Grid

Grid::Grid(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts, const Config& cfg)
    : dim_(dim), cfg_(cfg) {
    const dragon_config c = cfg.to_c();
    if (int rc = dragon_gpu_grid_create(dim, nx, ny, nz, dx, dy, dz, ghosts, &c, &h_)) raise(rc);
    int d = 0, nf = 0;
    dragon_gpu_grid_info(h_, &d, n_, &g_, &nf);
    nf_ = nf;
    if (nf_ != kNF) {
        dragon_gpu_grid_destroy(h_);
        h_ = nullptr;
        throw std::logic_error(kMHD ? "an MHD build (MHD defined) needs libdragon_host_mhd" : "a hydro build needs libdragon_host");
    }
    w_.assign(dragon_gpu_prim_count(h_) / kNF, PrimitiveState());
    if (kMHD && dim >= 2) B_.assign(dragon_gpu_faceB_count(h_) / 3, vec3());
}

Grid::~Grid() {
    if (h_) dragon_gpu_grid_destroy(h_);
}

void Grid::raise(int rc) const {
    const char* msg = dragon_gpu_last_error();
    if (rc == DRAGON_GPU_EINVAL || rc == DRAGON_GPU_EUNSUPPORTED) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

long long Grid::index(int i, int j, int k) const {
    const long long e1 = n_[1] + 2 * g_, e2 = n_[2] + 2 * g_;
    if (dim_ == 1) return i + g_;
    if (dim_ == 2) return (long long)(i + g_) * e1 + (j + g_);
    return ((long long)(i + g_) * e1 + (j + g_)) * e2 + (k + g_);
}

long long Grid::face_index(int i, int j, int k) const {
    const long long e1 = n_[1] + 1 + 2 * g_, e2 = n_[2] + 1 + 2 * g_;
    if (dim_ == 2) return (long long)(i + g_) * e1 + (j + g_);
    return ((long long)(i + g_) * e1 + (j + g_)) * e2 + (k + g_);
}

void Grid::host_current() const {
    if (!dev_newer_) return;
    if (int rc = dragon_gpu_download_prim(h_, &w_[0].rho)) raise(rc);
    if (!B_.empty())
        if (int rc = dragon_gpu_download_faceB(h_, &B_[0].x)) raise(rc);
    dev_newer_ = false;
}

PrimitiveState& Grid::cell(long long k) {
    host_current();
    host_newer_ = true;
    return w_[k];
}
const PrimitiveState& Grid::cell(long long k) const {
    host_current();
    return w_[k];
}
vec3& Grid::face(long long k) {
    host_current();
    host_newer_ = true;
    return B_[k];
}

void Grid::upload() {
    host_current();
    if (int rc = dragon_gpu_upload_prim(h_, &w_[0].rho)) raise(rc);
    if (!B_.empty())
        if (int rc = dragon_gpu_upload_faceB(h_, &B_[0].x)) raise(rc);
    host_newer_ = false;
}

void Grid::download() {
    dev_newer_ = true;
    host_current();
}

void Grid::to_device() {
    if (host_newer_) upload();
    push_boundary();
}

void Grid::push_boundary() {
    const std::vector<dragon_bc_desc> d = boundary.descriptors();
    std::vector<std::tuple<const void*, int, std::vector<double>>> fills;
    for (size_t k = 0; k < boundary.size(); k++)
        if (auto* f = dynamic_cast<const Boundary::DeviceFill*>(&boundary[k]))
            fills.emplace_back(f->compiled(), f->fill_faces, f->params);
    if (pushed_valid_ && d.size() == pushed_.size() &&
        (d.empty() || std::memcmp(d.data(), pushed_.data(), sizeof(dragon_bc_desc) * d.size()) == 0) &&
        fills == pushed_fills_)
        return;
    pushed_valid_ = false;
    if (int rc = dragon_gpu_set_boundary(h_, d.data(), (int)d.size())) raise(rc);
    // bind each device fill to its entry (dragon_gpu_set_boundary dropped the old bindings)
    for (size_t k = 0; k < boundary.size(); k++)
        if (auto* f = dynamic_cast<const Boundary::DeviceFill*>(&boundary[k]))
            if (int rc = dragon_gpu_set_user_fill(h_, (int)k, f->compiled(), f->fill_faces, f->get_corners() ? 1 : 0,
                                                  f->params.data(), (int)f->params.size()))
                raise(rc);
    pushed_ = d;
    pushed_fills_ = std::move(fills);
    pushed_valid_ = true;
}

void Grid::apply_boundary() {
    to_device();
    if (!boundary.has_user_elements()) {
        if (int rc = dragon_gpu_apply_boundary(h_)) raise(rc);
        dev_newer_ = true;
        return;
    }
    apply_boundary_host();
}

// BoundaryList::apply with user elements (BoundaryList.hpp:79-93): runs of
// built-in entries on the device (the implicit Outflow first), each user
// element's apply() on the host mirror between them.
void Grid::apply_boundary_host() {
    to_device();
    const int n = (int)boundary.size();
    const int off = dragon_gpu_boundary_entries(h_) - n;  // 1 when the device prepended the implicit Outflow
    int start = 0;
    for (int k = 0; k <= n; k++) {
        const bool user = k < n && boundary[k].device_type() < 0;
        if (k < n && !user) continue;
        const int stop = off + k;
        if (stop > start) {
            to_device();
            if (int rc = dragon_gpu_apply_boundary_range(h_, start, stop - start)) raise(rc);
            dev_newer_ = true;
        }
        if (user) {
            GhostFill& e = boundary[k];
            if (dim_ == 1) e.apply(static_cast<Grid1D&>(*this));
            else if (dim_ == 2) e.apply(static_cast<Grid2D&>(*this));
            else e.apply(static_cast<Grid3D&>(*this));
        }
        start = off + k + 1;
    }
}

double Grid::cfl_time() {
    to_device();
    double dt = 0;
    if (int rc = dragon_gpu_cfl_time(h_, &dt)) raise(rc);
    return dt;
}

void Grid::step_call(bool split, double dt) {
    to_device();
    dragon_step_status st;
    const int rc = split ? dragon_gpu_split_step(h_, dt, &st) : dragon_gpu_unsplit_step(h_, dt, &st);
    if (rc) raise(rc);
    dev_newer_ = true;
}

void Grid::unsplit_step(double dt) { step_call(false, dt); }
void Grid::split_step(double dt) { step_call(true, dt); }

bool Grid::on_step_fail(const std::exception&) { return true; }

void Grid::initialize_B_fields() {
    to_device();
    if (int rc = dragon_gpu_initialize_B_fields(h_)) raise(rc);
    dev_newer_ = true;
}

// Grid::advance_unsplit / advance_split (CFL.cpp:160-213) from the host.
void Grid::advance_host(double dt, bool check_cfl, bool split) {
    std::memset(&stats_, 0, sizeof(stats_));
    const double tol = cfg_.timestep_tol;
    while (dt > tol) {
        apply_boundary_host();
        double t1 = check_cfl ? std::min(dt, cfl_time()) : dt;
        for (;;) {
            try {
                if (split) split_step(t1);
                else unsplit_step(t1);
                break;
            } catch (const std::exception& e) {
                if (on_step_fail(e)) std::cout << "\t" << e.what() << "\n";
                else return;
            }
            stats_.retries++;
            t1 *= 0.5;
            if (t1 < tol) throw std::runtime_error("Timestep has fallen below minimum");
        }
        dt -= t1;
        stats_.steps++;
        stats_.last_dt = t1;
        stats_.time_advanced += t1;
    }
}

void Grid::advance(double dt, bool check_cfl) {
#if defined(Config_h) && !defined(DIMENSION_UNSPLIT)
    advance_split(dt, check_cfl);
#else
    advance_unsplit(dt, check_cfl);
#endif
}

void Grid::advance_unsplit(double dt, bool check_cfl) {
    if (boundary.has_user_elements()) return advance_host(dt, check_cfl, false);
    to_device();
    const int rc = dragon_gpu_advance(h_, dt, check_cfl ? 1 : 0, &stats_);
    dev_newer_ = true;
    if (rc) raise(rc);
}

void Grid::advance_split(double dt, bool check_cfl) {
    if (boundary.has_user_elements()) return advance_host(dt, check_cfl, true);
    to_device();
    const int rc = dragon_gpu_advance_split(h_, dt, check_cfl ? 1 : 0, &stats_);
    dev_newer_ = true;
    if (rc) raise(rc);
}

void Grid::advance_steps(int nsteps) {
    if (boundary.has_user_elements()) {
        for (int s = 0; s < nsteps; s++) {
            apply_boundary_host();
            advance_host(cfl_time(), true, false);
        }
        return;
    }
    to_device();
    const int rc = dragon_gpu_advance_steps(h_, nsteps, &stats_);
    dev_newer_ = true;
    if (rc) raise(rc);
}

Grid1D::Grid1D(int size, double dx_, int ghosts, const Config& cfg)
    : Grid(1, size, 1, 1, dx_, 0, 0, ghosts, cfg), dx(dx_) {}
Grid2D::Grid2D(int nx, int ny, double dx_, double dy_, int ghosts, const Config& cfg)
    : Grid(2, nx, ny, 1, dx_, dy_, 0, ghosts, cfg), dx(dx_), dy(dy_) {}
Grid3D::Grid3D(int nx, int ny, int nz, double dx_, double dy_, double dz_, int ghosts, const Config& cfg)
    : Grid(3, nx, ny, nz, dx_, dy_, dz_, ghosts, cfg), dx(dx_), dy(dy_), dz(dz_) {}

}  // namespace dragon

// ---------------------------------------------------------------------------
// DRAGONHOARD (DragonHoard.hpp:16-33) over dragon_gpu_hoard_*

namespace DRAGONHOARD {
namespace {

dragon_hoard_opts c_opts() {
    dragon_hoard_opts o;
    dragon_gpu_hoard_default_opts(&o);
    o.write_option = options.write_option;
    o.redundant = options.redundant_vals;
    o.compression = options.compression_level;
    o.ghosts = options.write_ghosts ? 1 : 0;
    o.threads = options.threads;
    return o;
}

std::string with_ext(const std::string& f) {
    const std::string ext = ".h5";
    if (f.size() > ext.size() && f.compare(f.size() - ext.size(), ext.size(), ext) == 0) return f;
    return f + ext;
}

void write(dragon::Grid& grid, double t, int cycle, const std::string& filename, bool wait) {
    grid.sync_device();
    const dragon_hoard_opts o = c_opts();
    const std::string path = output_dir + "/" + filename + ".h5";
    const int rc = wait ? dragon_gpu_hoard_write(grid.handle(), t, cycle, path.c_str(), &o)
                        : dragon_gpu_hoard_write_async(grid.handle(), t, cycle, path.c_str(), &o);
    if (rc) throw std::runtime_error(dragon_gpu_last_error());
}

}  // namespace

void writeToFile(dragon::Grid& grid, double t, int cycle, const std::string& filename) {
    write(grid, t, cycle, filename, true);
}

void writeToFileAsync(dragon::Grid& grid, double t, int cycle, const std::string& filename) {
    write(grid, t, cycle, filename, false);
}

void waitForFiles(dragon::Grid& grid) {
    if (dragon_gpu_hoard_wait(grid.handle())) throw std::runtime_error(dragon_gpu_last_error());
}

void loadFromFile(dragon::Grid& grid, double& t, int& cycle, const std::string& filename) {
    grid.sync_device();
    const std::string path = output_dir + "/" + with_ext(filename);
    if (dragon_gpu_hoard_load(grid.handle(), path.c_str(), &t, &cycle)) throw std::runtime_error(dragon_gpu_last_error());
    grid.device_changed();
    double d[3] = {0, 0, 0};
    const char* keys[3] = {"dx", "dy", "dz"};
    for (int a = 0; a < 3; a++) dragon_h5_read_attr(path.c_str(), keys[a], &d[a]);
    if (auto* g = dynamic_cast<dragon::Grid3D*>(&grid)) {
        g->dx = d[0];
        g->dy = d[1];
        g->dz = d[2];
    } else if (auto* g2 = dynamic_cast<dragon::Grid2D*>(&grid)) {
        g2->dx = d[0];
        g2->dy = d[1];
    } else if (auto* g1 = dynamic_cast<dragon::Grid1D*>(&grid)) {
        g1->dx = d[0];
    }
}

void verifyOutputDirectory() {
    const std::filesystem::path dir = output_dir;
    if (std::filesystem::exists(dir)) {
        if (!std::filesystem::is_directory(dir)) throw std::runtime_error(dir.string() + " exists but is not a directory");
    } else {
        std::filesystem::create_directories(dir);
    }
}

std::string restartFileName() {
    std::string best;
    int best_n = -1;
    for (const auto& e : std::filesystem::directory_iterator(output_dir)) {
        if (!e.is_regular_file()) continue;
        const std::string s = e.path().filename().string();
        const size_t dot = s.rfind('.');
        if ((dot == std::string::npos ? std::string() : s.substr(dot)) != ".h5") continue;
        const size_t end = s.find('.');
        const size_t pos = s.rfind('_', end);
        if (pos == std::string::npos || pos + 1 >= end) continue;
        bool digits = true;
        for (size_t i = pos + 1; i < end; i++) digits = digits && std::isdigit(static_cast<unsigned char>(s[i]));
        if (!digits) continue;
        const int n = std::stoi(s.substr(pos + 1, end - pos - 1));
        if (restart_frame >= 0) {
            if (n == restart_frame) return s;
        } else if (n > best_n) {
            best = s;
            best_n = n;
        }
    }
    return best;
}

std::string cycle_string(int n) {
    const char* z = n < 10 ? "0000" : n < 100 ? "000" : n < 1000 ? "00" : n < 10000 ? "0" : "";
    return z + std::to_string(n);
}

}  // namespace DRAGONHOARD
