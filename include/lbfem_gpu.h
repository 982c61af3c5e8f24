/*
 * lbfem_gpu.h -- C ABI of the B200 (sm_100a) implementation of the
 * per-time-step hot path of lbm-fem: the matrix-free Taylor-Galerkin streaming
 * operator, the consistent (Jacobi-PCG) or lumped mass solve and the nodal BGK
 * collision, for the Lee-Lin predictor-corrector and the Bardow-Karlin-Gusev
 * collide-then-stream schemes.
 *
 * Conventions
 *  - Plain C types only; no CUDA or torch types cross this boundary.
 *  - Every function returns an int status (LBFEM_OK = 0). No exception crosses
 *    the ABI; the message of the last failure is lbfem_gpu_last_error(ctx).
 *  - Host buffers belong to the caller; device memory belongs to the context.
 *  - Population vectors are structure-of-arrays: block a (population a,
 *    a = 0..8, D2Q9 numbering of include/lbfem/d2q9.h:18-22) occupies
 *    [a*n_dofs, (a+1)*n_dofs) and is indexed by the caller's DoF numbers.
 *    Increment / right-hand-side vectors of the moving populations have 8
 *    blocks (block a-1 holds population a), as in include/lbfem/streaming.h.
 *  - One host thread per context; calls are ordered on the context's stream.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * the lbm-fem sources).
 */
#ifndef LBFEM_GPU_H
#define LBFEM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  LBFEM_OK = 0,
  LBFEM_ERR_ARG = 1,            /* bad argument (AssertThrow / ExcMessage in the reference) */
  LBFEM_ERR_NO_CONVERGENCE = 2, /* CG hit its iteration cap: SolverControl::NoConvergence, mass.h:38-43 */
  LBFEM_ERR_NONFINITE = 3,      /* NaN or Inf met in a residual norm */
  LBFEM_ERR_CUDA = 4,           /* a CUDA runtime call failed */
  LBFEM_ERR_UNSUPPORTED = 5,    /* option or mesh the implementation does not handle */
  LBFEM_ERR_TIMEOUT = 6,        /* a bounded device-side wait gave up */
  LBFEM_ERR_STATE = 7           /* call out of order (e.g. step before set_time_step) */
};

enum { LBFEM_SCHEME_LEELIN = 0, LBFEM_SCHEME_BARDOW = 1 };             /* schemes.h:379,406 */
enum { LBFEM_MASS_CG = 0, LBFEM_MASS_LUMPED = 1, LBFEM_MASS_RICHARDSON = 2 }; /* mass.h:26-31 */
enum { LBFEM_STREAMING_TG2 = 0, LBFEM_STREAMING_TG3 = 1, LBFEM_STREAMING_TG3_SPLIT = 2 }; /* streaming.h:25-30 */
enum { LBFEM_PRECISION_FP64 = 0, LBFEM_PRECISION_MIXED = 1 };
enum { LBFEM_ADVECTION_TAYLOR_GALERKIN = 0, LBFEM_ADVECTION_LEELIN = 1 }; /* advection.h:211,256 */

/*
 * The discretisation, exported once from the host-side mesh builder (deal.II's
 * Discretization::reinit, discretization.h:78-144, in the reference).
 *
 * The mesh is the tensor-product box the reference builds: n_cells_x x
 * n_cells_y axis-parallel cells with vertex coordinates vertex_x[0..n_cells_x]
 * and vertex_y[0..n_cells_y] (uniform, tanh-stretched or any increasing
 * sequence), FE_Q(degree) on Gauss-Lobatto support points.
 *
 * Structured node (i, j), 0 <= i <= degree*n_cells_x, 0 <= j <= degree*n_cells_y,
 * is the support point at vertex_x[i/degree] + (i%degree-th Gauss-Lobatto point)
 * and likewise in y. In a periodic direction the last node column (row) is the
 * periodic image of the first: its DoF is constrained to the first one, as
 * make_periodicity_constraints does (discretization.h:110-112).
 *
 * dof_index[j*(degree*n_cells_x+1) + i] is the caller's DoF number of node
 * (i, j); NULL means the structured numbering itself (n_dofs must then be
 * (degree*n_cells_x+1)*(degree*n_cells_y+1)). Every DoF must appear once.
 *
 * Walls (discretization.h:63-67, Walls): the DoF of each wall node and the
 * velocity (2 doubles) of its wall. Wall nodes must lie on a non-periodic side
 * of the box.
 */
typedef struct lbfem_mesh_desc {
  int32_t degree;                /* p = 1..4 */
  int32_t n_cells_x, n_cells_y;  /* >= 2 in a periodic direction, >= 1 otherwise */
  int32_t periodic_x, periodic_y;
  const double *vertex_x;        /* n_cells_x + 1 increasing coordinates */
  const double *vertex_y;        /* n_cells_y + 1 increasing coordinates */
  int64_t n_dofs;
  const int64_t *dof_index;      /* NULL or (p*nx+1)*(p*ny+1) entries */
  int64_t n_walls;
  const int64_t *wall_dof;       /* n_walls caller DoF numbers */
  const double *wall_velocity;   /* 2*n_walls */
  /*
   * NULL, or the mapped vertices of a general quadrilateral mesh (the
   * reference's --distort, TaylorGreenVortex::transform_mesh,
   * test_cases.h:52-63): vertex (i, j), 0 <= i <= n_cells_x, 0 <= j <= n_cells_y,
   * at (vertex_xy[2 k], vertex_xy[2 k + 1]), k = j (n_cells_x + 1) + i. Each cell is
   * the bilinear image of the unit square through its four vertices (MappingQ1),
   * its support points the images of the Gauss-Lobatto points. vertex_x /
   * vertex_y still give the box's extent (first and last entries). Supported:
   * FP64, TG2, either scheme, consistent or lumped mass, no walls.
   */
  const double *vertex_xy;
} lbfem_mesh_desc;

/*
 * Settings of the scheme and of its streaming step (StreamingSettings,
 * MassSettings: streaming.h:32-36, mass.h:33-48).
 */
typedef struct lbfem_params {
  int32_t scheme;                /* LBFEM_SCHEME_* */
  int32_t mass;                  /* LBFEM_MASS_* */
  int32_t richardson;            /* passes of LBFEM_MASS_RICHARDSON after the lumped start (reference default 2) */
  int32_t streaming;             /* LBFEM_STREAMING_*; TG3 and TG3_SPLIT need Bardow, CG and FP64 */
  int32_t precision;             /* LBFEM_PRECISION_* */
  int32_t cg_max_iterations;     /* reference default 200 */
  double cg_tolerance;           /* relative to |r|, reference default 1e-8 */
  int32_t remove_wall_mass_flux; /* -1: scheme default (Bardow 1, Lee-Lin 0), advection.h:182-199 */
  int32_t device;                /* CUDA device ordinal */
  /*
   * LBFEM_PRECISION_MIXED only: the relative CG tolerance of the mass solve is
   * max(cg_tolerance, mixed_tolerance); 0 selects LBFEM_MIXED_TOLERANCE. The
   * right-hand side of the mixed path comes from FP32 arithmetic, so it is
   * resolved to about 1e-7 of its norm on coarse meshes and to about
   * 1e-7 / (2 pi h) on node spacing h; a tolerance far below that solves
   * rounding noise. No counterpart in the reference (FP64 only).
   */
  double mixed_tolerance;
} lbfem_params;

/* Default relative CG tolerance of the mixed-precision mass solve. */
#define LBFEM_MIXED_TOLERANCE 1e-6

typedef struct lbfem_gpu_ctx lbfem_gpu_ctx;

/* Fills *params with the reference defaults (Bardow, CG, 1e-8, 200 its, TG2, FP64). */
void lbfem_gpu_default_params(lbfem_params *params);

/* Human-readable text of a status code. */
const char *lbfem_gpu_status_string(int status);

/* The message of the last failure on ctx ("" if none). */
const char *lbfem_gpu_last_error(const lbfem_gpu_ctx *ctx);

/* Number of CUDA devices visible (0 without a GPU); never fails. */
int lbfem_gpu_device_count(void);

/*
 * The reference element matrix op (0 mass, 1 derivative int l_a l_b', 2
 * stiffness) of FE_Q(degree) on [0, 1], row-major (degree + 1)^2 entries: in
 * FP64 (ref64) and as the FP32 kernels use it (ref32; either may be null). The
 * FP32 derivative and stiffness rows sum exactly to zero, as the FP64 rows do
 * in exact arithmetic. Needs no GPU. The reference's counterpart is deal.II's
 * FE_Q shape data behind FEEvaluation (advection.h:100-121).
 */
int lbfem_gpu_reference_matrix(int32_t degree, int32_t op, double *ref64, float *ref32);

/*
 * Creates a context: exports the discretisation to flat device arrays and
 * builds the operators (Discretization::reinit + Scheme constructor,
 * discretization.h:78-144, schemes.h:85-90,111-116, streaming.h:41-60).
 * A mesh of 2^31 or more nodes is refused with LBFEM_ERR_UNSUPPORTED (the
 * kernels index a population array with 32-bit indices).
 */
int lbfem_gpu_create(const lbfem_mesh_desc *mesh, const lbfem_params *params, lbfem_gpu_ctx **ctx);
int lbfem_gpu_destroy(lbfem_gpu_ctx *ctx);

/* Scheme::set_time_step (schemes.h:40-44): dt fixed, lambda = nu / c_s^2. */
int lbfem_gpu_set_time_step(lbfem_gpu_ctx *ctx, double dt, double lambda);

/*
 * Scheme::set_initial_populations (schemes.h:51-59, Bardow: 129-141): loads the
 * physical populations f (host, 9 blocks) and applies the scheme's initial
 * transform (Bardow: g = f + dt/(2 lambda) (f - feq(f))). Resets the CG
 * extrapolation history. Needs the time step.
 */
int lbfem_gpu_set_initial_populations(lbfem_gpu_ctx *ctx, const double *f);

/* Raw copies of the scheme's populations Scheme::f (schemes.h:63), 9 blocks, host. */
int lbfem_gpu_set_populations(lbfem_gpu_ctx *ctx, const double *f);
int lbfem_gpu_get_populations(lbfem_gpu_ctx *ctx, double *f);

/*
 * Raw checkpoints of Scheme::f in the reference's format (io.h:137-165,
 * write_checkpoint / read_checkpoint): the file name.rank holds the 9 blocks
 * of n_dofs FP64 values one after the other, in the caller's DoF numbering. It
 * is written to name.rank.tmp and renamed, never leaving a torn file. A file
 * of another size is rejected (LBFEM_ERR_ARG). Valid for the same mesh and
 * numbering; Bardow's transformed populations also assume the same dt.
 */
int lbfem_gpu_write_checkpoint(lbfem_gpu_ctx *ctx, const char *name, int32_t rank);
int lbfem_gpu_read_checkpoint(lbfem_gpu_ctx *ctx, const char *name, int32_t rank);

/* Scheme::step (LeeLin schemes.h:92-98, Bardow schemes.h:118-124), n_steps times, device-resident. */
int lbfem_gpu_step(lbfem_gpu_ctx *ctx, int32_t n_steps);

/*
 * The host-buffer form of the same call: f (host, 9 blocks, caller numbering)
 * is uploaded, n_steps steps are taken, and f is downloaded again.
 */
int lbfem_gpu_step_host(lbfem_gpu_ctx *ctx, double *f, int32_t n_steps);

/* Waits for all work queued on ctx; returns the first deferred device-side failure. */
int lbfem_gpu_synchronize(lbfem_gpu_ctx *ctx);

/*
 * AdvectionOperator::apply (advection.h:49-58) with TaylorGalerkinAdvection
 * (kind = LBFEM_ADVECTION_TAYLOR_GALERKIN, advection.h:219-241) or
 * LeeLinAdvection (kind = LBFEM_ADVECTION_LEELIN, feq required, advection.h:263-289):
 * rhs (8 blocks) <- r_alpha of f (and feq), lattice velocities e (9 x 2,
 * Directions), time step {dt, lambda}. remove_wall_mass_flux: -1 = default of
 * the kind (1 for Taylor-Galerkin as Bardow builds it, 0 for Lee-Lin).
 * Host buffers. Constrained (periodic image) entries of rhs are zero.
 */
int lbfem_gpu_advection(lbfem_gpu_ctx *ctx, const double *f, const double *feq, const double *e, double dt,
                        double lambda, int32_t kind, int32_t remove_wall_mass_flux, double *rhs);

/*
 * MassSolver::solve (mass.h:185-213): x <- A^{-1} r with A = M + tg3 K_e(e),
 * K_e = int (e.grad N)(e.grad N^T) (StreamingMatrix, mass.h:57-129; e: 2 values,
 * needed when tg3_coefficient != 0, which CG supports and iterated lumping does
 * not: LBFEM_ERR_UNSUPPORTED). One block of n_dofs values.
 * CG starts from x (input) and stops at |r - A x| <= cg_tolerance |r|;
 * lumped and Richardson (x = M_L^{-1} r, then `richardson` passes
 * x += M_L^{-1} (r - M x)) overwrite x. Returns LBFEM_ERR_NO_CONVERGENCE when
 * the iteration cap is hit (x then holds the last iterate). Host buffers.
 */
int lbfem_gpu_mass_solve(lbfem_gpu_ctx *ctx, double *x, const double *r, const double *e, double tg3_coefficient);

/*
 * compute_stream_function (io.h:31-95): psi with u = -dpsi/dy, v = dpsi/dx from
 * (grad phi, grad psi) = (dphi/dx, v) - (dphi/dy, u), psi = 0 on every side of
 * the box, Jacobi-PCG to 1e-12 |b| (at most 10000 iterations). velocity: u then
 * v, two blocks of n_dofs (periodic images carry their source's value); psi:
 * n_dofs. Host buffers; uses the context's solver scratch (call between steps).
 */
int lbfem_gpu_stream_function(lbfem_gpu_ctx *ctx, const double *velocity, double *psi);

/* y <- M x, the MassOperator vmult (discretization.h:51), constrained rows the identity. Host buffers. */
int lbfem_gpu_mass_vmult(lbfem_gpu_ctx *ctx, double *y, const double *x);

/* CG iterations of all solves so far (MassSolver::cg_iterations, mass.h:215). */
int lbfem_gpu_cg_iterations(const lbfem_gpu_ctx *ctx, int64_t *iterations);

/* collide_bgk (collision.h:152-168): g (9 blocks, in place) <- BGK collision with rate omega. Host buffers. */
int lbfem_gpu_collide_bgk(lbfem_gpu_ctx *ctx, double *g, double omega);

/* compute_equilibrium (collision.h:105-113): feq (9 blocks) <- equilibrium of f, wall velocity imposed. */
int lbfem_gpu_compute_equilibrium(lbfem_gpu_ctx *ctx, const double *f, double *feq);

/* predictor_corrector (collision.h:119-145): f (9 blocks, in place), feq (9), incr (8), theta = dt/lambda. */
int lbfem_gpu_predictor_corrector(lbfem_gpu_ctx *ctx, double *f, const double *feq, const double *incr,
                                  double theta);

/*
 * Device-pointer forms of the operators, for a caller that keeps the vectors
 * in device memory (a shim whose deal.II vectors have device mirrors) and
 * swaps only the operators of Scheme::step: no host copy per call. Vectors are
 * DEVICE pointers with the same block layout and the caller's DoF numbering
 * (permuted on the device when the context has a dof_index; with the
 * structured numbering the kernels work on the caller's buffers in place).
 * The small parameter arrays (e: 9 x 2 or 2 doubles) stay on the host.
 *
 * `stream` is the caller's cudaStream_t passed as a pointer (NULL: the legacy
 * default stream). The call's device work is ordered after the work queued on
 * `stream` before the call, and the work queued on `stream` after the call
 * waits for it (events; the host does not wait). The exceptions are
 * lbfem_gpu_mass_solve_dev with consistent mass, whose Jacobi-PCG reads its
 * state back once per iteration and returns when the solve is done, and
 * lbfem_gpu_step_stream, which reads the step's status as lbfem_gpu_step does.
 */
/* AdvectionOperator::apply (advection.h:49-58, 219-241, 263-289): as lbfem_gpu_advection. */
int lbfem_gpu_advection_dev(lbfem_gpu_ctx *ctx, const double *f, const double *feq, const double *e, double dt,
                            double lambda, int32_t kind, int32_t remove_wall_mass_flux, double *rhs, void *stream);
/* MassSolver::solve (mass.h:185-213): as lbfem_gpu_mass_solve, x and r device vectors. */
int lbfem_gpu_mass_solve_dev(lbfem_gpu_ctx *ctx, double *x, const double *r, const double *e, double tg3_coefficient,
                             void *stream);
/* collide_bgk (collision.h:152-168): as lbfem_gpu_collide_bgk, g a device vector. */
int lbfem_gpu_collide_bgk_dev(lbfem_gpu_ctx *ctx, double *g, double omega, void *stream);
/* compute_equilibrium (collision.h:105-113): as lbfem_gpu_compute_equilibrium. */
int lbfem_gpu_compute_equilibrium_dev(lbfem_gpu_ctx *ctx, const double *f, double *feq, void *stream);
/* predictor_corrector (collision.h:119-145): as lbfem_gpu_predictor_corrector. */
int lbfem_gpu_predictor_corrector_dev(lbfem_gpu_ctx *ctx, double *f, const double *feq, const double *incr,
                                      double theta, void *stream);
/* Scheme::f (schemes.h:63) to and from a device vector of 9 blocks. */
int lbfem_gpu_set_populations_dev(lbfem_gpu_ctx *ctx, const double *f, void *stream);
int lbfem_gpu_get_populations_dev(lbfem_gpu_ctx *ctx, double *f, void *stream);
/* Scheme::step (schemes.h:92-98, 118-124) n_steps times, ordered on the caller's stream. */
int lbfem_gpu_step_stream(lbfem_gpu_ctx *ctx, int32_t n_steps, void *stream);

/*
 * One y-strip of a mesh decomposed over several contexts (one per rank), as
 * the reference distributes its triangulation and vectors over MPI ranks
 * (discretization.h:71-75) with a ghost exchange inside every operator
 * application (MatrixFree::loop, advection.h:151-175) and an MPI sum in every
 * CG dot product (mass.h:204-211).
 *
 * The context is created on the rank's local mesh: the cells of its strip
 * plus one ghost cell layer below (when it has a neighbour below) and the
 * ghost node row above (when it has a neighbour above), non-periodic in y,
 * with the walls of those rows. The rank owns the node rows
 * [ghost_below, n_rows - ghost_above) of the local mesh; the others are
 * copies of the neighbours' owned rows (ghost_below = degree rows, the
 * ghost cell layer; ghost_above = 1 row, the neighbour's first owned row).
 * For a periodic y axis the last rank's ghost row above holds the first
 * rank's row 0 (the periodic image row is not kept separately).
 *
 * comm(user, op, count) is the caller's collective, called by
 * lbfem_gpu_step (and the operator entries) with the context's stream idle:
 *  - LBFEM_COMM_EXCHANGE: send_below holds 1 row and send_above `degree` rows
 *    (count bytes per row), to the neighbour below / above; fill recv_below
 *    with `degree` rows from the neighbour below and recv_above with 1 row from
 *    the neighbour above. Sides without a neighbour are skipped.
 *  - LBFEM_COMM_ALLREDUCE: sum the first count doubles of sums over the ranks,
 *    in place.
 * Every rank makes the same calls in the same order. comm returns 0 on
 * success; anything else fails the step with LBFEM_ERR_ARG. The buffers are
 * device memory, at least lbfem_gpu_strip_buffer_bytes each (sums: 64
 * doubles), and stay valid while the context lives. In strip mode steps run
 * host-driven (no step graphs), CG and conservation sums count the owned rows,
 * and lbfem_gpu_stream_function is refused. No counterpart in the reference
 * beyond the MPI decomposition named above.
 */
enum { LBFEM_COMM_EXCHANGE = 0, LBFEM_COMM_ALLREDUCE = 1 };
typedef int (*lbfem_comm_fn)(void *user, int32_t op, int64_t count);
typedef struct lbfem_strip_desc {
  int32_t ghost_below;          /* degree (neighbour below) or 0 */
  int32_t ghost_above;          /* 1 (neighbour above) or 0 */
  /* y-widths of the neighbours' cells that share the local mesh's bottom and
   * top node rows (0 where there is none): the mass diagonals of those rows
   * get the missing cell's share, so that the Jacobi factors of the ghost
   * rows equal the owner's */
  double cell_below, cell_above;
  lbfem_comm_fn comm;
  void *user;
  void *send_below, *send_above, *recv_below, *recv_above;
  double *sums;
} lbfem_strip_desc;
/* Bytes each exchange buffer of lbfem_strip_desc needs on this context. */
int lbfem_gpu_strip_buffer_bytes(const lbfem_gpu_ctx *ctx, int64_t *bytes);
int lbfem_gpu_set_strip(lbfem_gpu_ctx *ctx, const lbfem_strip_desc *strip);

/* Discretization::node_weight (discretization.h:164-169): the lumped mass diagonal, n_dofs values (1 on periodic images). */
int lbfem_gpu_node_weight(lbfem_gpu_ctx *ctx, double *w);

/* The Jacobi diagonal of the mass matrix (MassOperator::compute_diagonal), n_dofs values (1 on periodic images). */
int lbfem_gpu_jacobi_diagonal(lbfem_gpu_ctx *ctx, double *d);

/*
 * Moments of the current populations at every DoF (D2Q9::moments, d2q9.h:30-41):
 * rho, ux, uy (host, n_dofs each; any may be NULL). Periodic images carry the
 * value of their source node.
 */
int lbfem_gpu_moments(lbfem_gpu_ctx *ctx, double *rho, double *ux, double *uy);

/*
 * FP64 conservation sums over the independent nodes with the lumped-mass
 * weights w (cgdbe.cc:353-368): out[0] = sum w, out[1] = sum w rho,
 * out[2] = sum w rho ux, out[3] = sum w rho uy, out[4] = sum w |u|^2.
 */
int lbfem_gpu_conservation(lbfem_gpu_ctx *ctx, double out[5]);

/* Page-locked host memory for fast host<->device copies (NULL on failure). */
void *lbfem_gpu_host_alloc(size_t bytes);
void lbfem_gpu_host_free(void *ptr);

/*
 * Device-side timing on the context's stream: lbfem_gpu_event_record(ctx, k)
 * records event k (0..15); lbfem_gpu_event_elapsed(ctx, a, b, &ms) waits for b
 * and returns the time between a and b in milliseconds.
 */
int lbfem_gpu_event_record(lbfem_gpu_ctx *ctx, int32_t slot);
int lbfem_gpu_event_elapsed(lbfem_gpu_ctx *ctx, int32_t a, int32_t b, float *ms);

/*
 * The streaming right-hand side of the scheme on the device-resident
 * populations, into the context's own rhs buffer (no host copies): the kernel
 * that lbfem_gpu_step launches first (Bardow: collide + advection fused and
 * the collided populations written back; Lee-Lin: advection with the nodal
 * equilibria computed on the fly). For timing and profiling of that kernel.
 */
int lbfem_gpu_advection_resident(lbfem_gpu_ctx *ctx);

/*
 * One refinement round of the mixed-precision mass solve (the window
 * correction with its FP64 residual, k_window_correct) for all 8 systems, on the
 * resident right-hand side and solution, into scratch buffers (the solution
 * history is not touched). For timing and profiling of that kernel; mixed
 * precision with consistent mass only.
 */
int lbfem_gpu_solve_round_resident(lbfem_gpu_ctx *ctx);

/*
 * The streaming kernel's tile, chosen at run time: before a mixed-precision
 * context's first step, each compiled tile shape of its degree (cells per CTA and
 * per thread's x / y segment) is timed on the context's own buffers, and the
 * fastest is kept (cached per device, degree, scheme and grid for the process;
 * LBFEM_TUNE=0 in the environment keeps the default). shape: -1 not yet tuned,
 * 0 the default shape, 1 the alternative (8 x-pass warps), 2 the small one
 * (shared memory and registers for 3 CTAs per SM); ms: the three shapes' times
 * per launch (3 floats). No counterpart in the reference.
 */
int lbfem_gpu_tuning(const lbfem_gpu_ctx *ctx, int32_t *shape, float *ms);

/* Statistics of the last lbfem_gpu_step call: CG iterations per solve (mean) and kernel launches. */
int lbfem_gpu_last_step_stats(const lbfem_gpu_ctx *ctx, double *cg_iterations_per_solve, int64_t *kernel_launches);

/*
 * Batched stepping of independent instances (contexts of any mesh, degree,
 * scheme and precision on one device). lbfem_gpu_batch_step advances every
 * instance by n_steps steps; each step of all instances is one CUDA graph
 * launch. The mixed-precision instances with consistent mass and TG2
 * streaming on Cartesian whole meshes are stepped by grouped kernels: each
 * kernel of the step runs over the tiles of all these instances (of one
 * degree), and the solve loops while any of them is active. Every other
 * instance is an independent branch of the graph running its own step graph.
 * Small instances thus share launches or run side by side on the GPU. Results
 * are bitwise those of lbfem_gpu_step on each context (LBFEM_BATCH_GROUP=0 in
 * the environment at batch creation makes every instance a branch). A solver failure in any instance is returned
 * (the lowest instance index, its message in lbfem_gpu_batch_last_error); that
 * instance stays as before its failing step, the others complete all steps.
 * The contexts must have their time step set and must not be stepped through
 * another call while a batch call runs. No counterpart in the reference (one
 * instance per run, cgdbe.cc).
 */
typedef struct lbfem_gpu_batch lbfem_gpu_batch;
int lbfem_gpu_batch_create(lbfem_gpu_ctx *const *ctxs, int32_t n_ctxs, lbfem_gpu_batch **batch);
int lbfem_gpu_batch_step(lbfem_gpu_batch *batch, int32_t n_steps);
const char *lbfem_gpu_batch_last_error(const lbfem_gpu_batch *batch);
/* Device time (CUDA events on the batch stream) of the graph launches of the last batch_step call, in ms. */
int lbfem_gpu_batch_last_ms(const lbfem_gpu_batch *batch, float *ms);
/* Kernels launched by the last batch_step call, all instances and the grouped launches. */
int lbfem_gpu_batch_last_launches(const lbfem_gpu_batch *batch, int64_t *launches);
int lbfem_gpu_batch_destroy(lbfem_gpu_batch *batch);

/*
 * The mass solve of lbfem_gpu_mass_solve (consistent mass, Jacobi-PCG) for
 * callers that cannot allocate device memory at the time of the call: a host
 * framework that owns every device allocation and hands out only its own
 * buffers, or a solver embedded in a code whose memory pool is sized once at
 * start-up. It has no counterpart in the reference.
 *
 * x (in: start, out: solution) and r are DEVICE pointers to n_dofs doubles in
 * the structured numbering (the context must have been created without
 * dof_index). The CG work buffers are not the context's: they live in one
 * fixed file-scope device array of the library (about 3.8 MiB, held by every
 * GPU that loads the library until the process exits), so the call allocates
 * nothing. Limits: at most 131072 nodes; larger meshes are rejected with
 * LBFEM_ERR_ARG. (The array also bounds the tiles at 4096, which no mesh of at
 * most 131072 nodes reaches: the most is 2731, Q1 with one cell across.)
 *
 * The call runs eagerly on the context's own stream and is host-synchronous:
 * it reads the solver state back to the host once per CG iteration and
 * returns when the solve has finished. It therefore cannot itself be recorded
 * into a CUDA graph. The solve reads x and r on the context's stream, which is
 * not ordered with the caller's streams: the caller must have finished
 * writing x and r before the call (for example with cudaStreamSynchronize on
 * the stream that wrote them). The first call on a device looks up the
 * array's device address. All calls share the array, so calls that overlap on
 * the GPU (from several threads or contexts) race, and a call must not overlap
 * any other call on the same context. Iterations are not added to
 * lbfem_gpu_cg_iterations.
 */
int lbfem_gpu_mass_solve_noalloc(lbfem_gpu_ctx *ctx, double *x, const double *r);

/*
 * The sum-factorisation contraction of the streaming right-hand side's x pass
 * (the FEEvaluation gradient / integrate pair it replaces is advection.h:100-121),
 * alone on a rows x (degree * cells + 1) grid of two fields, on CUDA cores
 * (tensor = 0) or tensor cores (tensor = 1: TF32 mma.sync with a three-term
 * split for FP32, DMMA for FP64), degree 2 or 3. Times `reps` launches with CUDA
 * events on the default stream (ms: per launch) and returns a checksum of the
 * outputs for comparing the two forms. A measurement for the choice between
 * CUDA and tensor cores; the steps do not use it. No counterpart in the reference.
 */
int lbfem_gpu_contraction_study(int32_t device, int32_t degree, int32_t fp64, int32_t tensor, int32_t rows,
                                int32_t cells, int32_t reps, float *ms, double *checksum);

#ifdef __cplusplus
}
#endif

#endif /* LBFEM_GPU_H */
