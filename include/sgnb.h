/*
 * sgnb.h -- C ABI of the B200 (sm_100a) implementation of the 2D hyperbolic-SGN
 * flux-reconstruction right-hand side and its adaptive Bogacki-Shampine 3(2) loop.
 *
 * Plain C: pointers, sizes and status codes only. Every entry point names the
 * interface of the reference project (gsalanglada/sgn-hyperbolic-gpu) that it
 * replaces. A header-only C++ wrapper with the reference's member signatures is in
 * sgnb.hpp.
 *
 * State layout (unchanged from the reference, src/solver/sgn2d.h:22-27):
 * variable-major doubles U[v * Nd + e * 25 + a + 5 b], v in (h, hu, hv, hw, hp),
 * element e = ex + Nx ey, node (a, b) of the 5 x 5 grid of solution points (GLL, or
 * Gauss-Legendre with point_set), Nd = 25 Nx Ny.
 *
 * Errors: every function returns an sgnb_status; nothing aborts the process
 * (the reference aborts on CUDA errors, src/cuda/sgn2d_cuda.cu:29-37).
 * sgnb_last_error() gives a message for the last failure on a context.
 * Threading: a context belongs to one host thread at a time; its work runs on its
 * own CUDA stream on the device chosen at creation.
 */
#ifndef SGNB_H
#define SGNB_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SGNB_OK = 0,
  SGNB_ERR_INVALID = 1,      /* bad argument or size (reference: std::invalid_argument) */
  SGNB_ERR_UNSUPPORTED = 2,  /* valid for the reference, not built here (P != 4, ...) */
  SGNB_ERR_CUDA = 3,         /* CUDA runtime error; the message names the call */
  SGNB_ERR_NAN = 4,          /* non-finite embedded error: the run stopped */
  SGNB_ERR_DTMIN = 5,        /* step size fell below dtMin (reference stats.aborted) */
  SGNB_ERR_TIMEOUT = 6,      /* a bounded device wait gave up */
  SGNB_ERR_NOMEM = 7,        /* device allocation failed */
  SGNB_ERR_NO_DEVICE = 8     /* no CUDA device visible */
} sgnb_status;

enum { SGNB_BC_PERIODIC = 0, SGNB_BC_WALL = 1 };

/* Solution points (PointSet, src/core/fr_operators.h:51). Gauss-Legendre points need a
 * flat bottom (SGNB_BATHY_NONE: H = 0), as SGN2D requires (sgn2d.cpp:46-47); their face
 * traces are interpolated with lL / lR, and a wall mirrors the element's own trace. */
enum { SGNB_POINTS_GLL = 0, SGNB_POINTS_GAUSS = 1 };

/* Arithmetic modes. */
enum {
  SGNB_FP64_EXACT = 0, /* reference operation order, no FMA: bit-identical to the CPU */
  SGNB_FP64_FAST = 1,  /* FMA + reciprocals: within 1e-13 relative per field */
  SGNB_MIXED = 2       /* FP32 deviations from the lake at rest, FP64 hydrostatic balance,
                          FP64 state / RK accumulation / error / controller, FP32 stage
                          derivatives (an addition to the reference, which is FP64 only) */
};

/* Built-in still-depth profiles H(x, y); SGNB_BATHY_ARRAYS takes precomputed arrays.
 * Parameter vectors are documented in sgnb_setup.cpp. */
enum {
  SGNB_BATHY_NONE = 0,      /* H = 0 (the reference's empty stillDepth, sgn2d.h:55) */
  SGNB_BATHY_CONST = 1,     /* p0 */
  SGNB_BATHY_GAUSS = 2,     /* p0 - p1 exp(-((x-p2)^2 + (y-p3)^2) / p4) */
  SGNB_BATHY_SHOAL = 3,     /* elliptic shoal on a plane */
  SGNB_BATHY_GAUSS_SUM = 4, /* plane minus a sum of Gaussian bumps */
  SGNB_BATHY_CELLS = 5,     /* bilinear interpolant of a grid of cell means */
  SGNB_BATHY_ARRAYS = 100   /* Hnod .. HfaceYEnd given by the caller */
};

/* Construction parameters; mirrors the arguments of
 * SGN2D(int P, int Nx, int Ny, double Lx, double Ly, const sgn2d::Params&,
 *       std::function<double(double,double)> stillDepth, PointSet)
 * (src/solver/sgn2d.h:57-59) plus the sgn2d::Params fields (src/physics/sgn_flux2d.h:57-62).
 * Call sgnb_desc_init() first. */
typedef struct {
  int P, Nx, Ny;             /* only P = 4 is built; Nx, Ny >= 2 */
  double Lx, Ly;
  double g, c, gamma, nManning; /* nManning >= 0: Manning friction (0 = off) */
  int bc_x, bc_y;            /* SGNB_BC_*; walls are an addition to the reference */
  int precision;             /* SGNB_FP64_EXACT, SGNB_FP64_FAST or SGNB_MIXED */
  int device;                /* CUDA device ordinal */
  /* FR tables of FROperators1D (src/core/fr_operators.h:68-89); all NULL = built here */
  const double *nodes, *D, *lL, *lR, *gLp, *gRp, *qw;
  int bathy_kind;            /* SGNB_BATHY_* */
  const double* bathy_par;
  int n_bathy_par;
  /* SGNB_BATHY_ARRAYS: the SGN2D accessors stillDepthNodal/GradX/GradY/FaceX/FaceY
   * (sgn2d.h:94-98; Nd, Nd, Nd, 5 Nx Ny, 5 Nx Ny doubles) and, for walls, the depth on
   * the right edge (5 Ny, sampled at x = Nx hx) and top edge (5 Nx, at y = Ny hy). */
  const double *Hnod, *Hx, *Hy, *HfaceX, *HfaceY, *HfaceXEnd, *HfaceYEnd;
  /* Slab of a larger mesh (x decomposition, as the reference's multi-GPU solver splits
   * it, src/parallel/slab1d.h:55-72): the full mesh has Nx_global elements over Lx and
   * this context owns the Nx columns from ex_offset on; node coordinates, bathymetry and
   * face depths are the full mesh's. Nx_global = 0: the context is the whole mesh. */
  int Nx_global, ex_offset;
  /* SGNB_POINTS_*, the PointSet argument of SGN2D (sgn2d.h:57-59); caller-given tables
   * whose lL / lR are not unit rows are Gauss points whatever this says. Gauss points
   * run in the FP64 modes on whole meshes (not batched, no adjoint). */
  int point_set;
} sgnb_desc;

/* AdaptiveRKOptions (src/solver/rk.h:53-61). */
typedef struct {
  double atol, rtol, dtMin, dtMax, safety, facMin, facMax;
} sgnb_rk_opts;

/* AdaptiveRKStats (src/solver/rk.h:64-72) plus the attempt count, a status and the
 * number of kernels the call launched. */
typedef struct {
  long long accepted, rejected, rhsEvals, attempts;
  double tReached, dtLast, maxNormLast;
  int aborted;   /* 1: dt < dtMin (as the reference); 2: non-finite error */
  int status;    /* sgnb_status of the run */
  long long kernel_launches; /* device kernels launched, including no-op tail launches */
} sgnb_rk_stats;

typedef struct sgnb_ctx sgnb_ctx;

/* Defaults: P 4, Nx = Ny = 2, Lx = Ly = 1, Params{g 9.81, c 0, gamma 1.5, n 0},
 * periodic, FP64 exact, device 0, tables built here, H = 0. */
void sgnb_desc_init(sgnb_desc* d);
/* Defaults of AdaptiveRKOptions (src/solver/rk.h:53-61). */
void sgnb_rk_opts_init(sgnb_rk_opts* o);

/* Replaces SGN2DCuda::SGN2DCuda(const SGN2D&) (src/cuda/sgn2d_cuda.h:33): allocates the
 * device state and uploads tables and bathymetry. */
int sgnb_create(const sgnb_desc* d, sgnb_ctx** out);
/* Replaces SGN2DCuda::~SGN2DCuda (src/cuda/sgn2d_cuda.h:34). NULL is allowed. */
int sgnb_destroy(sgnb_ctx* ctx);

/* SGN2D::nDof (src/solver/sgn2d.h:64): nodes per field. State size is 5 * this. */
long long sgnb_ndof(const sgnb_ctx* ctx);

/* SGN2DCuda::upload / download (src/cuda/sgn2d_cuda.h:41-42): host <-> device state. */
int sgnb_upload(sgnb_ctx* ctx, const double* U_host);
int sgnb_download(sgnb_ctx* ctx, double* U_host);

/* SGN2DCuda::rhsOnce (src/cuda/sgn2d_cuda.h:43): dU = R(uploaded state), to the host. */
int sgnb_rhs_once(sgnb_ctx* ctx, double* dU_host);
/* SGN2D::rhs (src/solver/sgn2d.h:78): dU = R(U) for host arrays; the uploaded state is
 * left untouched. */
int sgnb_rhs_host(sgnb_ctx* ctx, const double* U_host, double* dU_host);
/* SGN2DCuda::rhsDevice (src/cuda/sgn2d_cuda.h:51), public here: dU = R(U) for device
 * arrays on a caller stream (cudaStream_t, NULL = the context stream). Asynchronous. */
int sgnb_rhs_device(sgnb_ctx* ctx, const double* U_dev, double* dU_dev, void* stream);

/* SGN2DCuda::integrateAdaptive (src/cuda/sgn2d_cuda.h:46-47), the device-resident form
 * of integrateAdaptive (src/solver/rk.h:78-80): integrates the uploaded state in place.
 * opts NULL = defaults. Returns SGNB_OK also when stats->aborted is set (as the
 * reference returns normally with stats.aborted). */
int sgnb_integrate_adaptive(sgnb_ctx* ctx, double t0, double tEnd, double dt0,
                            const sgnb_rk_opts* opts, sgnb_rk_stats* stats);
/* The same device-resident loop run for a fixed number of accepted steps instead of to
 * an end time (tEnd = infinity, stop after nsteps accepted): the form the benchmark uses
 * for "N adaptive steps". Built on integrateAdaptive (src/solver/rk.h:78-80); the
 * reference has no step-count stop. */
int sgnb_integrate_steps(sgnb_ctx* ctx, double t0, double dt0, long long nsteps,
                         const sgnb_rk_opts* opts, sgnb_rk_stats* stats);
/* n consecutive bs3Step (src/solver/rk.h:50) steps of the uploaded state with the
 * given step sizes, starting at t0: the frozen-dt replay of an accepted sequence. */
int sgnb_bs3_steps(sgnb_ctx* ctx, double t0, const double* dts, long long n);
/* n consecutive rk4Step (src/solver/rk.h:42, classical RK4, src/solver/rk.cpp:23-38) steps
 * of the uploaded state with the given step sizes, starting at t0 (the right-hand side
 * does not depend on t). FP64 modes; SGNB_ERR_UNSUPPORTED in the mixed mode. Like the
 * reference it checks nothing: a non-finite state stays in the buffer. */
int sgnb_rk4_steps(sgnb_ctx* ctx, double t0, const double* dts, long long n);

/* Attempt log of the last sgnb_integrate_adaptive / sgnb_bs3_steps call: per attempt
 * (t, dt, errNorm, accepted as 1.0 / 0.0), up to 65536 attempts. Copies min(cap, n)
 * rows into out and sets *n to the number recorded. No reference counterpart (the
 * reference keeps only AdaptiveRKStats); it exposes the controller's dt sequence. */
int sgnb_attempt_log(sgnb_ctx* ctx, double* out, long long cap, long long* n);

/* Profiling hook, no reference counterpart: launches `count` copies of one fused stage
 * kernel of a BS3(2) attempt (stage 2: k2 = R(u + dt/2 k1); 3: k3 = R(u + 3dt/4 k2);
 * 4: the end-point stage with uNew, k4 and the error partials) on the uploaded state with
 * step dt, on `stream` (NULL = context stream), asynchronously. It overwrites only the
 * stage buffers, so the uploaded state is unchanged; run an integration first so that
 * k1 is defined. */
int sgnb_launch_stage(sgnb_ctx* ctx, int stage, double dt, int count, void* stream);

/* SGN2D::maxWaveSpeed / cflTimeStep / mass / energy (src/solver/sgn2d.h:85-90) of the
 * uploaded state, reduced on the device. */
int sgnb_max_wave_speed(sgnb_ctx* ctx, double* out);
int sgnb_cfl_time_step(sgnb_ctx* ctx, double cfl, double* out);
int sgnb_mass(sgnb_ctx* ctx, double* out);
int sgnb_energy(sgnb_ctx* ctx, double* out);

/* Allocation-free variant of sgnb_max_wave_speed / sgnb_mass / sgnb_energy, without a
 * context; no counterpart in the reference. For callers that cannot allocate device
 * memory (a framework that owns all of it through its own pool, or a fixed-budget loop
 * that must not call cudaMalloc between steps): it allocates nothing and keeps its
 * per-block partials in a library-owned 128 KB __device__ array instead.
 * what = 0 largest wave speed, 1 mass, 2 energy of the state U_dev (device, the layout
 * above, 25 Nx Ny nodes per field); Hnod_dev (device, nodal still depth) is read only
 * for the energy. The result is written to out_dev[0] (device) asynchronously on
 * `stream` (NULL = the legacy default stream) on the current device.
 * Limit: 25 Nx Ny <= 67,108,864 nodes per field, else SGNB_ERR_INVALID.
 * Every call looks the array's device address up on the current device (so a device
 * reset between calls leaves nothing stale); the first call on a device also loads the
 * library's device code there, so make that first call before any stream capture. All
 * calls on a device share the array: calls that overlap on the GPU race. */
int sgnb_diag_noalloc(int what, int Nx, int Ny, double Lx, double Ly, double g, double c,
                      double gamma, const double* U_dev, const double* Hnod_dev,
                      double* out_dev, void* stream);

/* Host-side set-up queries (no device work). */
/* SGN2D::nodeCoords (src/solver/sgn2d.h:70). */
int sgnb_node_coords(const sgnb_ctx* ctx, double* x, double* y);
/* Device pointers of the state buffer that holds u and of the context stream, for
 * callers that manage device memory themselves. */
int sgnb_state_device_ptr(sgnb_ctx* ctx, double** U_dev, void** stream);

/* FROperators1D tables for degree P (src/core/fr_operators.cpp:134-200), computed on
 * the host without a device. Sizes P+1, (P+1)^2 for D. */
int sgnb_fr_tables(int P, double* nodes, double* D, double* lL, double* lR, double* gLp,
                   double* gRp, double* qw);
/* The same for a point set (SGNB_POINTS_*): FROperators1D(P, pointSet). */
int sgnb_fr_tables_points(int P, int point_set, double* nodes, double* D, double* lL,
                          double* lR, double* gLp, double* gRp, double* qw);
/* The bathymetry arrays sgnb_create would upload for d (SGN2D ctor,
 * src/solver/sgn2d.cpp:30-84), on the host without a device. Any pointer may be NULL. */
int sgnb_setup_bathymetry(const sgnb_desc* d, double* Hnod, double* Hx, double* Hy,
                          double* HfaceX, double* HfaceY, double* HfaceXEnd,
                          double* HfaceYEnd);

/* The fast mode's reciprocal (fn 0: 1/x) and square root (fn 1) elementwise over n
 * doubles of device memory (x in, y out) on `stream` (NULL: the legacy default stream),
 * synchronised: the fast arithmetic mode's own Newton-Raphson forms, exposed so that
 * tests can compare them with the IEEE results. */
int sgnb_fast_math(int fn, const double* x, double* y, long long n, void* stream);

/* The checked build (libsgnb_checked.so, compiled with -DSGNB_CHECKED) range-checks every
 * global access of the fused FP64 and mixed-precision kernels and of the adjoint's
 * kernels against its buffer; an out-of-range index is
 * counted and the access skipped. The count on `device` since the last reset (reset != 0
 * zeroes it after reading). SGNB_ERR_UNSUPPORTED in the normal build. */
int sgnb_checked_oob(int device, long long* count, int reset);

/* Slab decomposition (the reference's multi-GPU solver, src/cuda/sgn2d_cuda_mpi.cu:148-161,
 * 487-537: x slabs, one halo exchange per right-hand side, one reduction of the error norm
 * per step). A slab is a context created with Nx_global / ex_offset; its neighbours'
 * traces across the slab edges come from ghost arrays [5 fields][Ny][5 nodes] that the
 * caller fills with the neighbours' packed edges before every stage; the caller gathers
 * every slab's error partials and runs each slab's controller on all of them, so that
 * every slab takes the same decision.
 *   sgnb_set_ghosts   device ghost arrays of the left / right edge (NULL: the edge
 *                     follows bc_x: a wall, or the periodic wrap of a single slab)
 *   sgnb_slab_pack    this slab's edge nodes for the neighbours: stage 0 = the input
 *                     `in` of a right-hand side (NULL: the current state), 2 / 3 = the
 *                     intermediate stages of the running attempt, 4 = its end-point
 *                     candidate; sendL / sendR are [5][Ny][5] device arrays
 *   sgnb_slab_begin   the controller from t0 with dt0 until tEnd (HUGE_VAL: none) or
 *                     nsteps accepted steps (0: none), whichever comes first (dts != NULL:
 *                     nsteps frozen step sizes, the bs3Step replay)
 *   sgnb_slab_launch  stage 1 (FSAL head k1 = R(u)), 2, 3, 4 (end point, error partials)
 *   sgnb_slab_partials / sgnb_slab_control / sgnb_slab_status: this slab's partials
 *                     (3 doubles per tile), the controller on the gathered partials of all
 *                     slabs (n_total = 5 x the nodes of the whole mesh), the controller
 *                     state (synchronises).
 * The right-hand side of a slab is sgnb_rhs_device after its ghosts hold the neighbours'
 * packed inputs. FP64 modes; `stream` NULL = the context's stream. */
int sgnb_set_ghosts(sgnb_ctx* ctx, const double* ghostL, const double* ghostR);
int sgnb_slab_pack(sgnb_ctx* ctx, int stage, const double* in, double* sendL, double* sendR,
                   void* stream);
int sgnb_slab_begin(sgnb_ctx* ctx, double t0, double tEnd, double dt0, long long nsteps,
                    const double* dts, const sgnb_rk_opts* opts);
int sgnb_slab_launch(sgnb_ctx* ctx, int stage, void* stream);
int sgnb_slab_partials(sgnb_ctx* ctx, double** partials, int* nblk);
int sgnb_slab_control(sgnb_ctx* ctx, const double* partials, int nblk, long long n_total,
                      void* stream);
int sgnb_slab_status(sgnb_ctx* ctx, sgnb_rk_stats* st, int* done, void* stream);
/* Fused edge exchange (the slab form of the multi-GPU solver's RHS epilogue writing the
 * halo line into the peer's ghost buffer): one stage launch with this stage's ghost inputs
 * (ghostL / ghostR, NULL at a wall), whose slab-edge tiles of stages 2 and 3 also store
 * the next stage's edge inputs straight into the neighbours' ghost arrays for that stage
 * (edgeL: the left neighbour's right ghost, edgeR: the right neighbour's left ghost; on
 * another device, peer memory that this device can address). Stage 1 and 4 write no edges;
 * the caller packs stage 0 and 2 (sgnb_slab_pack, with the neighbours' ghost arrays as
 * the send buffers) and orders each launch after the neighbours' launches that fill its
 * ghosts. */
int sgnb_slab_stage(sgnb_ctx* ctx, int stage, const double* ghostL, const double* ghostR,
                    double* edgeL, double* edgeR, void* stream);
/* Lets kernels on `device` address the memory of `peer` (NVLink / NVSwitch peer access;
 * a repeated call is a no-op; device == peer is a no-op). */
int sgnb_enable_peer_access(int device, int peer);
/* The controller on the error partials of all nslab (<= 32) slabs, read in place in slab
 * order (partials[k]: device pointer, peer memory allowed; nblk[k] blocks): no gather. */
int sgnb_slab_control_all(sgnb_ctx* ctx, const double* const* partials, const int* nblk,
                          int nslab, long long n_total, void* stream);

/* Device-side sampling for the reference's applications, which download the whole state
 * at every sample time and scan it on the host (apps/shoal_focus_mpi.cu:195-205,
 * apps/tsunami_margin_mpi.cu:184-198). sgnb_eta_max: the largest eta = h - H of the
 * current state over the nodes inside [x0, x1] x [y0, y1] (bounds inclusive; +-HUGE_VAL for
 * none) and the node holding it (smallest index on ties; -1 and -HUGE_VAL when the
 * window holds no node). sgnb_sample_eta: eta at n nodes (gauges). sgnb_nearest_node: the
 * node closest to (x, y) (smallest index on ties), as the applications place gauges. */
int sgnb_eta_max(sgnb_ctx* ctx, double x0, double x1, double y0, double y1, double* eta_max,
                 long long* node);
int sgnb_sample_eta(sgnb_ctx* ctx, const long long* nodes, int n, double* eta);
int sgnb_nearest_node(const sgnb_ctx* ctx, double x, double y, long long* node);
/* Element means of eta = h - H, u, v, p and H of the current state (out: 5 * Nx * Ny,
 * field-major, element ex + Nx ey), formed on the device as the reference's VTK writer
 * forms them (src/io/vtk2d.h:38-44), and that writer's legacy-VTK frame
 * (STRUCTURED_POINTS, ASCII, src/io/vtk2d.h:30-83) from them: only 5 Nx Ny values cross
 * to the host instead of the state. */
int sgnb_element_means(sgnb_ctx* ctx, double* out);
int sgnb_write_vtk(sgnb_ctx* ctx, const char* path);

/* Batched sweep (no reference counterpart; the reference runs one instance per
 * SGN2DCuda): n independent instances (their own mesh size, parameters, bathymetry and
 * state) advanced together, one launch per RK stage over all instances' tiles, each
 * instance with its own adaptive controller; the attempts run as a device-side loop (a
 * CUDA graph whose WHILE conditional node repeats one attempt of every still-running
 * instance until all are done). All
 * instances of a batch run in one arithmetic mode: SGNB_FP64_FAST (tile shapes 8x4, 16x2,
 * 4x8) or SGNB_MIXED (8x4 tiles). Instance i is an ordinary context
 * (sgnb_batch_instance) for upload / download / diagnostics between runs. */
typedef struct sgnb_batch sgnb_batch;
int sgnb_batch_create(const sgnb_desc* descs, int n, sgnb_batch** out);
int sgnb_batch_destroy(sgnb_batch* b);
int sgnb_batch_size(const sgnb_batch* b);
/* The batch's CUDA stream (cudaStream_t): its launches run there, for callers that time or
 * order work around them. */
int sgnb_batch_stream(const sgnb_batch* b, void** stream);
sgnb_ctx* sgnb_batch_instance(sgnb_batch* b, int i);
/* nsteps accepted steps for every instance, starting from dt0[i]; stats[n]. */
int sgnb_batch_integrate_steps(sgnb_batch* b, const double* dt0, long long nsteps,
                               const sgnb_rk_opts* opts, sgnb_rk_stats* stats);
/* Launch configuration: tile shape (0: 8x4, 1: 16x2, 2: 4x8 elements) and the grid:
 * blocks == 0 launches one CTA per tile of the work list, blocks > 0 that many persistent
 * CTAs looping over it (default: 8x4, one CTA per tile; sgnb_batch_autotune picks one). */
int sgnb_batch_set_config(sgnb_batch* b, int shape, int blocks);
int sgnb_batch_get_config(const sgnb_batch* b, int* shape, int* blocks);
/* Autotuner: times one adaptive attempt (three stage launches, reps times) for every tile
 * shape and grid (one CTA per tile, persistent grids of 1..4 CTAs per SM) at step sizes
 * dt0[i], keeps the fastest (sgnb_batch_get_config reports it). ms_out (optional, 15
 * entries, shape-major) receives the measured ms per attempt (-1 for shapes a mixed batch
 * does not use). The instances' states are left unchanged. */
int sgnb_batch_autotune(sgnb_batch* b, const double* dt0, int reps, double* ms_out);
const char* sgnb_batch_last_error(const sgnb_batch* b);

/* Adjoint (no reference counterpart). A frozen-dt BS3(2) trajectory of a context
 * (SGNB_FP64_FAST or SGNB_FP64_EXACT) parameterised by the bathymetry as Nx * Ny element
 * means (mapped to the depth statics by the bilinear cell interpolant, SGNB_BATHY_CELLS
 * with Mx = Nx, My = Ny) and the initial free surface eta0 (Nd nodal values;
 * h0 = H + eta0, zero velocity, w = p = 0). sgnb_adj_forward replaces the context's
 * bathymetry, runs nsteps steps of sizes dts, records eta = h - H at the gauge nodes
 * after every step (eta_out[n * ngauges + g], n = 0 .. nsteps-1 for the states after
 * steps 1 .. nsteps) and keeps the state every checkpoint_every steps; the context then
 * holds the final state. sgnb_adj_vjp takes the cotangent of those records and returns
 * the gradients with respect to the element means and eta0 (checkpoint-and-recompute,
 * hand-written VJP kernels of every right-hand-side phase and of the RK update). */
typedef struct sgnb_adj sgnb_adj;
int sgnb_adj_create(sgnb_ctx* ctx, long long nsteps, const double* dts, int ngauges,
                    const long long* gauge_nodes, int checkpoint_every, sgnb_adj** out);
int sgnb_adj_destroy(sgnb_adj* a);
int sgnb_adj_forward(sgnb_adj* a, const double* means, const double* eta0, double* eta_out);
int sgnb_adj_vjp(sgnb_adj* a, const double* eta_bar, double* grad_means, double* grad_eta0);
/* VJP of the right-hand side at a host state U: Ubar = (dR/dU)^T Rbar and the cotangents
 * of the context's depth statics (any of those pointers may be NULL; sizes as in
 * sgnb_desc's arrays). */
int sgnb_rhs_vjp(sgnb_ctx* ctx, const double* U, const double* Rbar, double* Ubar,
                 double* Hnod_bar, double* Hx_bar, double* Hy_bar, double* HfaceX_bar,
                 double* HfaceY_bar, double* HfaceXEnd_bar, double* HfaceYEnd_bar);

const char* sgnb_status_string(int status);
/* Message of the last failure on ctx (or of the last failed sgnb_create when NULL). */
const char* sgnb_last_error(const sgnb_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SGNB_H */
