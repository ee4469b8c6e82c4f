/*
 * dragon_oracle.h — CPU restatement of DRAGON's unsplit Godunov update.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle: a plain-C restatement
 * of the reference's algorithm (DRAGON/FluidElement, Hydro/Reconstruction,
 * Hydro/Riemann, Hydro/Godunov, Hydro/CFL, Boundary, MHD), written in the
 * reference's loop structure and operand order. It is pinned bit for bit
 * against the reference itself (oracle/_ref, tests/test_oracle_port.py) and
 * against the reference's golden vectors. Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may call it; the product never does.
 *
 * Built twice (like the reference): liboracle_hydro.so and, with -DORACLE_MHD,
 * liboracle_mhd.so. Arrays use the reference's padded AoS order: NF doubles per
 * cell (rho, p, vx, vy, vz[, Bx, By, Bz]), last index fastest; face B arrays
 * have n+1 cells per axis and 3 doubles per face.
 */
#ifndef DRAGON_ORACLE_H
#define DRAGON_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Runtime switches, ids as in DRAGON/Config.h. */
void ora_set_options(int riemann, int limiter, int cfl, int ct_energy, int exact_max_iters, double exact_tol,
                     double cfl_coeff, double timestep_tol);
int ora_nfields(void);

typedef struct ora_grid ora_grid;
ora_grid* ora_grid_new(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts);
void ora_grid_free(ora_grid* g);
int ora_grid_ghosts(const ora_grid* g);
void ora_grid_set_prim(ora_grid* g, const double* a);
void ora_grid_get_prim(const ora_grid* g, double* a);
void ora_grid_set_faceB(ora_grid* g, const double* a);
void ora_grid_get_faceB(const ora_grid* g, double* a);

/* Boundary list: type 0 Outflow, 1 Outflow::Gated, 2 Fixed, 3 Reflective,
 * 4 Periodic, 5 Ignore; faces = Boundary::face_mask bits. */
void ora_boundary_clear(ora_grid* g);
int ora_boundary_add(ora_grid* g, int type, int faces, int corners, const double* state);
void ora_boundary_apply(ora_grid* g);
int ora_initialize_B_fields(ora_grid* g);

/* Status codes: 0 ok, 1 step failed (the reference throws), 2 CFL zero speed,
 * 3 dt below Timestep_Tolerance (the reference exits). */
int ora_cfl_time(ora_grid* g, double* dt);
int ora_unsplit_step(ora_grid* g, double dt);
int ora_advance(ora_grid* g, double dt, int check_cfl, int* steps, int* retries);

/* Unit-level pieces. */
double ora_limiter(int kind, double a, double b);
void ora_muscl(const double* wl, const double* wc, const double* wr, double dt_dL, const double* dB, double* L,
               double* R);
int ora_riemann_flux(int solver, const double* l, const double* r, double dt_dx, int axis, double* out);
void ora_exact_star(const double* l, const double* r, double pGuess, double* sl, double* sr, int* iters);
/* Records every Newton-branch exact solve into buf (8 doubles per row:
 * rhoL, vxL, pL, rhoR, vxR, pR, p*, iterations, negated when the iteration
 * cap rather than the tolerance ended the solve; x-normal frame) until cap rows;
 * stop returns the number of solves seen (may exceed cap). Hydro build only. */
void ora_exact_log_start(double* buf, long cap);
long ora_exact_log_stop(void);

#ifdef __cplusplus
}
#endif
#endif
