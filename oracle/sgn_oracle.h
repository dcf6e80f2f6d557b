/*
 * sgn_oracle.h -- CPU oracle for the 2D hyperbolic-SGN flux-reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU kernels are compared
 * against; no product code links or calls it. Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it.
 *
 * Two libraries implement this same C interface:
 *   liboracle.so        sgn_oracle.c, a plain-C restatement of the reference
 *                       algorithm (each function cites the reference lines it follows)
 *   _ref/libsgnref.so   ref_shim.cpp, a thin wrapper over the reference's own
 *                       sources compiled from their original location (Makefile)
 * Parity of the restatement is pinned against the compiled reference and against
 * the golden fixtures under tests/golden/.
 *
 * Boundary conditions: OR_BC_PERIODIC is the reference's only mode
 * (src/core/mesh2d.h:36-45). OR_BC_WALL is a reflective wall (mirror ghost state)
 * that the reference lacks; the restatement implements it with ghost states and the
 * reference shim implements it by mirror doubling (periodic reference on the
 * doubled domain, first quadrant extracted), which is operation-for-operation the
 * same computation.
 *
 * State layout (the reference's, src/solver/sgn2d.h:22-27): variable-major,
 * U[v * Nd + e * 25 + a + 5 b], e = ex + Nx ey, Nd = 25 Nx Ny nodes per field.
 */
#ifndef SGN_ORACLE_H
#define SGN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_BC_PERIODIC = 0, OR_BC_WALL = 1 };
/* solution points (PointSet, src/core/fr_operators.h) */
enum { OR_POINTS_GLL = 0, OR_POINTS_GAUSS = 1 };

typedef struct or_ctx or_ctx;

/* Solver set-up (mirrors SGN2D::SGN2D, src/solver/sgn2d.cpp:30-84). Returns NULL on
 * invalid arguments (the reference throws std::invalid_argument). */
or_ctx* or_create(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                  double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                  const double* bathy_par, int n_par);
/* The same with the solution point set: Gauss points need a flat bottom (bathy_kind
 * OR_BATHY_NONE, H = 0), as SGN2D requires (sgn2d.cpp:46-47); their face traces are
 * interpolated with lL / lR, and a wall mirrors the element's own face trace. */
or_ctx* or_create_points(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                         double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                         const double* bathy_par, int n_par, int points);
void or_destroy(or_ctx* s);
long or_ndof(const or_ctx* s); /* nodes per field, SGN2D::nDof */

/* FR tables (FROperators1D accessors, src/core/fr_operators.h:68-89). Sizes:
 * nodes/lL/lR/gLp/gRp/qw: P+1, D: (P+1)^2 row-major. */
void or_tables(const or_ctx* s, double* nodes, double* D, double* lL, double* lR,
               double* gLp, double* gRp, double* qw);
/* Bathymetry arrays (SGN2D accessors, sgn2d.h:94-98): Hnod/Hx/Hy: Nd, HfaceX/HfaceY:
 * ne*np. HfaceXEnd (Ny*np) and HfaceYEnd (Nx*np) hold the depth on the right and top
 * domain edges, used only by walls; any pointer may be NULL. */
void or_bathymetry(const or_ctx* s, double* Hnod, double* Hx, double* Hy, double* HfaceX,
                   double* HfaceY, double* HfaceXEnd, double* HfaceYEnd);
/* [restatement only] Replaces the bathymetry arrays (same sizes as or_bathymetry; NULL
 * keeps an array). The tests perturb the depth statics directly through it when they
 * check the adjoint of the right-hand side by finite differences. */
void or_set_bathymetry(or_ctx* s, const double* Hnod, const double* Hx, const double* Hy,
                       const double* HfaceX, const double* HfaceY, const double* HfaceXEnd,
                       const double* HfaceYEnd);
void or_node_coords(const or_ctx* s, double* x, double* y); /* sgn2d.cpp:89-102 */

int or_rhs(const or_ctx* s, const double* U, double* dU);     /* sgn2d.cpp:125-290 */
double or_max_wave_speed(const or_ctx* s, const double* U);   /* sgn2d.cpp:295-305 */
double or_cfl_time_step(const or_ctx* s, const double* U, double cfl); /* :310-314 */
double or_mass(const or_ctx* s, const double* U);             /* sgn2d.cpp:319-329 */
double or_energy(const or_ctx* s, const double* U);           /* sgn2d.cpp:334-348 */

/* Integrators (src/solver/rk.cpp) with f = the rhs above. */
void or_rk4_step(const or_ctx* s, double t, double dt, double* U); /* rk.cpp:23-38 */
void or_bs3_step(const or_ctx* s, double t, double dt, double* U); /* rk.cpp:41-54 */

/* Adaptive BS3(2) (rk.cpp:67-164). opts = {atol, rtol, dtMin, dtMax, safety, facMin,
 * facMax, stopAfter}; stopAfter > 0 (restatement only) ends the run after that many
 * accepted steps; stats = {accepted, rejected, rhsEvals, tReached, dtLast, maxNormLast,
 * aborted}. If log != NULL, attempt k writes {t, dt, errNorm, accepted} to
 * log[4k..4k+3] for k < max_log. Returns the number of attempts. */
long or_integrate_adaptive(const or_ctx* s, double* U, double t0, double tEnd,
                           double dt0, const double* opts, double* stats, double* log,
                           long max_log);

#ifdef __cplusplus
}
#endif

#endif /* SGN_ORACLE_H */
