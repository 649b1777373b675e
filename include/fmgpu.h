/*
 * fmgpu.h -- C-ABI of libfmgpu.so, the B200 (sm_100a) multigrid solve path
 * behind Femlisp's Lisp-level iteration API.
 *
 * Style follows Femlisp's foreign interface (interface/superlu.c:51-88,
 * interface/umfpack.c:44-77, bound by src/alien/superlu.lisp:57-75 through
 * fl.port:def-function, src/basic/port.lisp:442-547): plain C functions of
 * ints, longs, doubles and pointers that return an int status
 * (0 = FMG_OK, negative = error).  Handles are opaque.  Host arrays passed in
 * are read or written during the call only and never retained.  A context
 * serialises all its work on one CUDA stream and must be used from one host
 * thread at a time.  Device faults are returned as status codes, never as
 * aborts; fmg_last_error() gives the message of the last failure.
 *
 * Grids are Femlisp's uniformly refined hierarchical meshes of the unit
 * n-cube (src/mesh/meshgen.lisp:180-183: level l has n0*2^l cells per
 * direction) with a Lagrange Q1/Q2 ansatz space (lagrange.lisp:176-202).
 * Nodes are numbered lexicographically, x fastest; a level matrix is stored by
 * stencil slot (slot s = sum_k (o_k + order) (2 order + 1)^k for the node
 * offset o), the structured form of Femlisp's key-indexed <sparse-matrix>
 * (src/matlisp/sparse-matrix.lisp:49,703-840).
 */
#ifndef FMGPU_H
#define FMGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define FMG_OK 0
#define FMG_ERR_ARG (-1)        /* invalid argument or size */
#define FMG_ERR_CUDA (-2)       /* CUDA runtime error (message in fmg_last_error) */
#define FMG_ERR_STATE (-3)      /* call out of order (e.g. solve before assemble) */
#define FMG_ERR_NOMEM (-4)      /* device allocation failed */
#define FMG_ERR_NUMERIC (-5)    /* NaN/Inf met in a residual norm */
#define FMG_ERR_UNSUPPORTED (-6)
#define FMG_ERR_IO (-7)         /* bad or corrupted file */

/* ------------------------------------------------------ coefficient kinds */
#define FMG_K_CONST 0           /* scalar diffusion k, n = 1 (default 1.0) */
#define FMG_K_CELL 1            /* k per top-level cell, n = cells; coarse levels
                                   sample it at their own Gauss points */
#define FMG_F_CONST 2           /* constant source, n = 1 (default 1.0) */
#define FMG_F_IP 3              /* source at the Gauss points of every top-level
                                   cell, n = cells * (order+1)^dim */
#define FMG_LAMBDA_MU_CELL 4    /* elasticity (ncomp 3): the Lame constants
                                   lambda = mu = E per top-level cell, n = cells
                                   (isotropic-elasticity-tensor, elasticity.lisp:71-88);
                                   coarse levels sample E at their Gauss points */
#define FMG_F_VEC 5             /* elasticity: constant force vector, n = ncomp */

/* ------------------------------------------------------------ iteration */
#define FMG_JACOBI 0            /* <jacobi> :damp (linit.lisp:220-250) */
#define FMG_SOR 1               /* <sor> :omega, colour ordering (linit.lisp:288-323) */
#define FMG_SSC 2               /* (geometric-ssc) :omega, vertex-centred blocks (geoblock.lisp:37-158,
                                   blockit.lisp:118-204); scalar grids */
#define FMG_PSC 3               /* (geometric-psc) :damp, the same blocks, corrections from one residual
                                   added (blockit.lisp:118-204); scalar grids */

#define FMG_METHOD_MG 0         /* <linear-solver> :iteration <geometric-cs> */
#define FMG_METHOD_CG_MG 1      /* <cg> :preconditioner <geometric-cs> */
#define FMG_METHOD_CG 2         /* <cg> without preconditioner */

#define FMG_MULTIPLICATIVE 0    /* :combination (multigrid.lisp:67-70) */
#define FMG_ADDITIVE 1

typedef struct fmg_ctx fmg_ctx;
typedef struct fmg_grid fmg_grid;
typedef struct fmg_vec fmg_vec;

/* Solver configuration: the initargs of <geometric-cs> (multigrid.lisp:55-70,
   geomg.lisp:148-155), <cg> (krylow.lisp:67-70) and the success/failure
   forms of <linear-solver> (iterate.lisp:105-123). */
typedef struct {
  int method;          /* FMG_METHOD_* */
  int smoother;        /* FMG_JACOBI, FMG_SOR, FMG_SSC or FMG_PSC */
  double damp;         /* :damp of <jacobi>, :omega of <sor> */
  int pre_steps, post_steps, gamma;
  int compat_alias;    /* 1: the preconditioner is called as (iterate q w w),
                          rhs and residual aliased (krylow.lisp:120) */
  double coarse_damp;  /* :damp of the <lu> coarse-grid iteration (1.0) */
  double rtol;         /* success if :reduction < rtol (<= 0: off) */
  double atol;         /* success if :defnorm < atol (<= 0: off) */
  int maxsteps;        /* failure if :step > maxsteps */
  int combination;     /* FMG_MULTIPLICATIVE or FMG_ADDITIVE */
  int fmg;             /* 1: the iterator's cycle is the F-cycle (:fmg t,
                          f-cycle, multigrid.lisp:290-297): the residual
                          restricted to the base level, then from the base up a
                          cycle on each level and a prolongation to the next;
                          fmg_solve and fmg_vcycle only */
} fmg_solve_cfg;

/* ------------------------------------------------------------- context */
/* Opens device `device` (load-foreign-library, port.lisp:360-379, plus the
   state the Lisp side keeps).  */
int fmg_init(int device, fmg_ctx** ctx);
/* Grids keep their context alive and vectors their grid: destroying a handle
   that still has dependants defers its release to the last dependant. */
int fmg_finalize(fmg_ctx* ctx);
/* Copies the message of the last failure (NUL-terminated) into buf. */
int fmg_last_error(fmg_ctx* ctx, char* buf, int len);
int fmg_synchronize(fmg_ctx* ctx);
/* The CUDA stream (cudaStream_t) all work of ctx is queued on. */
int fmg_get_stream(fmg_ctx* ctx, void** stream);
/* Number of kernels this library has launched in this process (diagnostics;
   no counterpart in the reference). */
int fmg_launch_count(long long* out);

/* ---------------------------------------------------------------- grids */
/* A level hierarchy base_level..top_level of the uniformly refined unit
   n-cube (uniformly-refined-hierarchical-mesh, meshgen.lisp:180-183) with
   Lagrange order `order` (lagrange-fe, lagrange.lisp:176-202) and `ncomp`
   components: 1 (the cdr problem) or 3 with dim 3 (linear elasticity,
   elasticity-model-problem, elasticity.lisp:112-123: vectors hold 3 values
   per node, node-major; level matrices 3 x 3 blocks per stencil slot, layout
   [slot][k][l][node]; the Jacobi smoother inverts the 3 x 3 diagonal blocks;
   CG / MG with Jacobi only).  dirichlet_mask bit 2k / 2k+1 marks the face
   x_k = 0 / 1 as essential boundary, all components of its nodes (the
   :external-boundary constraint coefficient, cdr.lisp:184-185). */
int fmg_grid_create(fmg_ctx* ctx, int dim, int order, int ncomp, int n0, int top_level,
                    int base_level, int dirichlet_mask, fmg_grid** grid);
/* A hierarchy of algebraic levels 0 .. nlevels-1 (0 the coarsest, sizes[l]
   unknowns each) without geometry, for the matrices Femlisp forms on
   unstructured or adaptively refined meshes (multilevel-decomposition,
   geomg.lisp:109-142; constraints.lisp:58-151): the level matrices come
   through fmg_set_matrix (compressed rows or the columns of
   sparse-matrix->ccs over the caller's numbering), the interpolation between
   each level and the one below through fmg_set_interpolation, the top-level
   rhs through fmg_set_rhs.  Once every matrix and interpolation is in place
   the base level's LU is formed and fmg_solve / fmg_vcycle / the level
   operators run the same iteration as on structured grids (Jacobi smoother;
   the base level at most 1024 unknowns).  Rows sum in column order, so a
   structured level handed over this way gives its structured results bit
   for bit.  Geometry-bound calls (fmg_assemble*, fmg_set_coefficient,
   fmg_get_matrix, SOR/SSC/PSC, the mixed solve, the damping network) return
   FMG_ERR_UNSUPPORTED. */
int fmg_grid_create_algebraic(fmg_ctx* ctx, int nlevels, const long* sizes, fmg_grid** grid);
/* The interpolation I from level fine_level - 1 to fine_level (nfine x
   ncoarse; FMG_CSR or FMG_CCS): prolongate xf += I xc, restrict rc = I^T rf
   (multigrid.lisp:202-252); constrained fine rows and coarse columns empty
   (constrained-interpolation-matrix, constraints.lisp:58-72). */
int fmg_set_interpolation(fmg_grid* grid, int fine_level, int layout, const int* start, const int* index,
                          const double* values, long nfine, long ncoarse);
int fmg_grid_destroy(fmg_grid* grid);
long fmg_grid_nnodes(const fmg_grid* grid, int level);
int fmg_grid_nslots(const fmg_grid* grid);

/* Coefficients of the cdr model problem (cdr-model-problem, cdr.lisp:153-204):
   diffusion k and source f, sampled by the host (Lisp coefficient closures
   cannot run on the device). */
int fmg_set_coefficient(fmg_grid* grid, int kind, const double* host, long n);

/* Cell-wise Lagrange stiffness assembly of every level, with the Dirichlet
   rows turned into identity rows, and the dense LU of the base level:
   assemble-interior (fedisc.lisp:108-206) for the top level (:surface) and
   for each coarse level (:refined, geomg.lisp:109-142), eliminate-constraints
   + m+! P (constraints.lisp:323-411, fedisc.lisp:244-253, geomg.lisp:128-137),
   and getrf! of the <lu> coarse-grid iteration (linit.lisp:137-151). */
int fmg_assemble(fmg_grid* grid);
/* fmg_assemble with the coarse levels chosen like multilevel-decomposition
   (geomg.lisp:109-142): FMG_ASSEMBLE_REDISCRETIZE assembles every level
   (assemble-interior :refined); FMG_ASSEMBLE_GALERKIN assembles the top
   level and forms each coarser one as the Galerkin product I^T A_{l+1} I with
   the constrained interpolation (:galerkin-p t, geomg.lisp:122-123; every
   structured form: scalar Q1/Q2 and 3 x 3 node blocks, each entry summed in
   a fixed order, so the levels are deterministic; FMG_ERR_UNSUPPORTED on an
   algebraic grid). */
#define FMG_ASSEMBLE_REDISCRETIZE 0
#define FMG_ASSEMBLE_GALERKIN 1
int fmg_assemble_levels(fmg_grid* grid, int mode);
/* Upload a level matrix assembled elsewhere: the parity path for matrices
   Femlisp builds itself (assemble-interior with any coefficient functions,
   fedisc.lisp:108-206; Galerkin products, geomg.lisp:122-123), handed over
   in the compressed-column form of sparse-matrix->ccs (sparselu.lisp:226-263,
   the form interface/superlu.c:51-88 takes) or as compressed rows.  Rows and
   columns use the grid's numbering: node-major (dof = node * ncomp + comp),
   nodes lexicographic with x fastest; n is the number of rows.  start has
   n + 1 offsets, index / values start[n] entries; duplicate entries add up.
   Every entry must lie in the level's Lagrange stencil (|offset| <= order per
   direction; for Q2 also the element coupling), else FMG_ERR_ARG, except for
   explicit zeros, which are dropped.  Dirichlet rows are taken as given.  A
   hierarchy is complete, and solvable, once every level base..top has a
   matrix (uploaded, or from an earlier assembly); the base level's LU is then
   formed.  A grid with an uploaded matrix applies its mixed form through the
   stored FP32 matrix, not matrix-free from the coefficients.  On an
   algebraic grid (fmg_grid_create_algebraic) any pattern is accepted: the
   matrix is kept as compressed rows (columns ascending, duplicates summed,
   explicit zeros dropped) with its diagonal for the Jacobi smoother. */
#define FMG_CSR 0
#define FMG_CCS 1
int fmg_set_matrix(fmg_grid* grid, int level, int layout, const int* start, const int* index,
                   const double* values, long n);
/* Top-level right-hand side (the rhs of an uploaded system); n = nodes * ncomp. */
int fmg_set_rhs(fmg_grid* grid, const double* host, long n);
/* Level matrix to the host, layout [slot][node] (debug / parity). */
int fmg_get_matrix(fmg_grid* grid, int level, double* host);
/* Top-level right-hand side (the assembled rhs of discretize-globally,
   fedisc.lisp:307-316). */
int fmg_get_rhs(fmg_grid* grid, double* host);
/* Per-node Jacobi/SOR damping on a level (NULL resets to the scalar :damp). */
int fmg_set_node_damping(fmg_grid* grid, int level, const double* host, long n);

/* -------------------------------------------------------------- vectors */
/* A device vector on a level (make-domain-vector-for, sparse-vector.lisp:53-58). */
int fmg_vec_create(fmg_grid* grid, int level, fmg_vec** vec);
int fmg_vec_destroy(fmg_vec* vec);
int fmg_vec_set(fmg_vec* vec, const double* host, long n);
int fmg_vec_get(const fmg_vec* vec, double* host, long n);
/* fill! / x<-0 (vector.lisp:224) */
int fmg_vec_fill(fmg_vec* vec, double value);
/* copy! (vector.lisp:304-312, sparse-vector.lisp:248-258) */
int fmg_copy(const fmg_vec* x, fmg_vec* y);
/* axpy! y := y + alpha x (vector.lisp:321-326) */
int fmg_axpy(double alpha, const fmg_vec* x, fmg_vec* y);
/* dot (sparse-vector.lisp:260-264), deterministic chunked reduction */
int fmg_dot(const fmg_vec* x, const fmg_vec* y, double* out);
/* l2-norm (vector.lisp:328-331) */
int fmg_l2_norm(const fmg_vec* x, double* out);

/* ------------------------------------------------------------ operators */
/* gemm! 1.0 A x 0.0 y on level `level` (sparse-matrix.lisp:392-405) */
int fmg_matvec(fmg_grid* grid, int level, const fmg_vec* x, fmg_vec* y);
/* gemm! 1.0 A x 0.0 y on the top level, or with b non-null compute-residual
   y := b - A x (sparse-matrix.lisp:392-405, linit.lisp:73-80), applied
   matrix-free from the cell coefficients as fmg_solve_mixed applies its top
   level: fp32 = 0, FP64 in the difference form of that solve's CG operator;
   fp32 = 1, FP32 arithmetic on x, b and the coefficients rounded to FP32 (the
   V-cycle's top level), the result widened; fp32 = 2 (b must be NULL), FP64
   arithmetic on x rounded to FP32 (the CG operator a = A p of that solve,
   whose search direction is FP32).  3D scalar Q1 grids with
   FMG_K_CELL coefficients only (FMG_ERR_UNSUPPORTED otherwise); y must differ
   from x and b.  Waits for the result. */
int fmg_matvec_mf(fmg_grid* grid, int fp32, const fmg_vec* x, const fmg_vec* b, fmg_vec* y);
/* compute-residual r := b - A x (linit.lisp:73-80); b may be r */
int fmg_residual(fmg_grid* grid, int level, const fmg_vec* x, const fmg_vec* b, fmg_vec* r);
/* restrict: rc := I^T rf with the constrained interpolation
   (multigrid.lisp:202-212, constraints.lisp:58-72) */
int fmg_restrict(fmg_grid* grid, int fine_level, const fmg_vec* rf, fmg_vec* rc);
/* prolongate: xf := xf + I xc (multigrid.lisp:237-239) */
int fmg_prolongate(fmg_grid* grid, int coarse_level, const fmg_vec* xc, fmg_vec* xf);
/* one <jacobi> step: r := D^-1 r, x := x + damp r (linit.lisp:220-250) */
int fmg_jacobi(fmg_grid* grid, int level, double damp, fmg_vec* x, fmg_vec* r);
/* one multicolour <sor> sweep (linit.lisp:288-323); b may be r */
int fmg_sor(fmg_grid* grid, int level, double omega, fmg_vec* x, const fmg_vec* b, fmg_vec* r);
/* one (geometric-ssc) sweep (blockit.lisp:118-204) over the vertex-centred
   blocks of geoblock.lisp:72-158 -- on the structured grid the 3^d box of
   nodes around each even node (Q2), the node alone (Q1), Dirichlet members
   other than the vertex left out: per block r_B := b_B - (A x)_B, the dense
   local system solved by LU with partial pivoting, x_B += omega c.  Blocks in
   colour order (vertex index mod 2 per direction), lexicographic within a
   colour; b may be r (the alias inside <cg>). */
int fmg_ssc(fmg_grid* grid, int level, double omega, fmg_vec* x, const fmg_vec* b, fmg_vec* r);
/* one (geometric-psc) sweep: every vertex block of fmg_ssc solves its local
   system with the residual r as given (r is read, not written), and the
   corrections are added in increasing vertex order, x_B += damp c_B
   (overlapping blocks sum theirs) */
int fmg_psc(fmg_grid* grid, int level, double damp, fmg_vec* x, const fmg_vec* r);
/* the <lu> coarse-grid iteration on the base level: r := A^-1 r,
   x := x + damp r (linit.lisp:156-161) */
int fmg_coarse_solve(fmg_grid* grid, double damp, fmg_vec* x, fmg_vec* r);

/* ------------------------------------------------------------- solvers */
/* One application of the <geometric-cs> iterator (multigrid.lisp:366-386) on
   the top level.  Passing the same vector as b and r reproduces the alias of
   the <cg> preconditioner call (krylow.lisp:120). */
int fmg_vcycle(fmg_grid* grid, const fmg_solve_cfg* cfg, fmg_vec* x, fmg_vec* b, fmg_vec* r);
/* The <linear-solver> loop (iterate.lisp:239-250, solve.lisp:139-164,
   linsolve.lisp:58-73) on the assembled top-level system, starting from x.
   hist receives :defnorm per step (hist_len >= maxsteps + 2), *nsteps the
   last step index, *status 0 = success, 1 = failure (maxsteps). */
int fmg_solve(fmg_grid* grid, const fmg_solve_cfg* cfg, fmg_vec* x, double* hist, int hist_len,
              int* nsteps, int* status);
/* The <cg> iterator (make-iterator, krylow.lisp:72-132) one call at a time,
   for a host whose own <linear-solver> loop drives it (linsolve.lisp:58-73).
   fmg_cg_start is the iterator's initialize: restart from the residual r
   (up to date, :residual-before t): w := r, p := M(w) with the cycle of cfg
   (method CG+MG; plain CG: p := r), alpha := (p, r).  fmg_cg_step is its
   iterate: a := A p, lam := alpha / (a, p), x += lam p, r -= lam a,
   q := M(r), alpha' := (q, r), p := (alpha'/alpha) p + q; r stays up to
   date (:residual-after t) and *defnorm (may be NULL) receives ||r||.  The
   search direction and the cycle's vectors stay in the grid between calls;
   the arithmetic is fmg_solve's, step for step. */
int fmg_cg_start(fmg_grid* grid, const fmg_solve_cfg* cfg, const fmg_vec* r);
int fmg_cg_step(fmg_grid* grid, fmg_vec* x, fmg_vec* r, double* defnorm);

/* ------------------------------------------------------ mixed precision */
/* No counterpart in the reference.  Mixed-precision variant of fmg_solve for
   <cg> + <geometric-cs> with Jacobi smoothing: flexible CG in FP64 (FP64
   operator, recursive FP64 residual, FP64 solution update) preconditioned by
   one V-cycle per step that smooths, restricts and prolongates in FP32 with
   BF16 coarse right-hand sides and residuals, the coarsest dense solve staying
   in FP64.  When the recursive residual meets the tolerance the true residual
   is recomputed with the assembled FP64 matrix, and CG restarts from it if it
   does not.  With matrix_free set, a 3D Q1 problem with a cell-wise
   coefficient applies its top-level operator (FP64 and FP32) from the cell
   coefficients instead of the stored matrix.  hist receives the true residual
   at the start and at every restart check and the recursive residual after
   each CG iteration; *nouter counts restart checks, *ninner CG iterations.
   With judge > 0 and per-node damping installed (fmg_net_apply or
   fmg_set_node_damping), the plain cycle (scalar :damp) judges the learned
   one inside the solve: on each of the first `judge` CG steps after every
   (re)start both cycles are applied to the same residual r, and each
   direction z is scored by the energy decrease (z, r)^2 / (z, A z) a step
   along it gives; if the plain cycle's is larger the node damping is dropped
   for the rest of the solve, which restarts from the true residual with the
   plain cycle (fmg_learned_status counts the revert and reports the last
   judged step's two figures). */
typedef struct {
  double inner_rtol;   /* reserved, 0 */
  int max_inner;       /* reserved, 0 */
  int max_outer;       /* restart checks allowed (default 20) */
  int matrix_free;     /* 1: matrix-free top level where available */
  int judge;           /* CG steps after each (re)start judged against the plain cycle (0: none) */
} fmg_mixed_cfg;

int fmg_solve_mixed(fmg_grid* grid, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mcfg, fmg_vec* x,
                    double* hist, int hist_len, int* nouter, int* ninner, int* status);

/* ------------------------------------------------------ damping network */
/* No counterpart in the reference: the learned part of the smoother.  A
   3-layer 3^d convolution net on the node grid of a level (16 input channels:
   per adjacent cell the centred log coefficient and a presence bit; 32 hidden
   channels; BF16 weights and activations, FP32 accumulation on the tensor
   cores) predicts each node's Jacobi damping in [omega_min, omega_max]
   (0.1, 1.3).  The prediction becomes the level's node damping, i.e. it
   replaces the scalar damp of <jacobi> (linit.lisp:220-250) node by node in
   the FP64 and the mixed-precision cycles.  Scalar Q1 grids, d = 2 or 3. */
typedef struct fmg_net fmg_net;

/* parameters: He-uniform weights from seed, output bias for omega = 0.6 */
int fmg_net_create(fmg_ctx* ctx, int dim, unsigned long long seed, fmg_net** out);
int fmg_net_destroy(fmg_net* net);
/* flat FP32 parameter vector: W1[taps][32][16], b1[32], W2[taps][32][32],
   b2[32], W3[taps][32], b3[1]; tap = (dx+1) + 3(dy+1) + 9(dz+1) */
long fmg_net_nparams(const fmg_net* net);
int fmg_net_get_params(fmg_net* net, float* host, long n);
int fmg_net_set_params(fmg_net* net, const float* host, long n);
/* accumulated gradient of the training loss (same layout) */
int fmg_net_get_grads(fmg_net* net, float* host, long n);
int fmg_net_zero_grads(fmg_net* net);
/* one Adam step with the accumulated gradients, which are then cleared */
int fmg_net_adam(fmg_net* net, double lr, double beta1, double beta2, double eps);
/* versioned weight file with a checksum; a damaged file fails with FMG_ERR_IO */
int fmg_net_save(fmg_net* net, const char* path);
int fmg_net_load(fmg_ctx* ctx, const char* path, fmg_net** out);
/* forward pass on one level (base < level <= top): installs the node damping
   of that level and copies it to omega (N values) when omega is not NULL */
int fmg_net_damping(fmg_net* net, fmg_grid* grid, int level, double* omega);
/* forward pass on every level above the base (installs the damping) */
int fmg_net_apply(fmg_net* net, fmg_grid* grid);
/* backward pass from dL/domega (N host values) of the level of the last
   fmg_net_damping call; gradients are added to the accumulator */
int fmg_net_backward(fmg_net* net, fmg_grid* grid, int level, const double* gomega);
/* Training loss of one error sample e0 on the top level: the A-norm error
   contraction |S C S e0|_A^2 / |e0|_A^2 of one V(1,1) cycle with the level's
   current node damping (S the damped Jacobi sweep, C the coarse-grid
   correction of the cycle below), and its gradient with respect to that
   damping (N values, when gomega is not NULL).  FP64. */
int fmg_learn_loss(fmg_grid* grid, const fmg_solve_cfg* cfg, const fmg_vec* e0, double* loss, double* gomega);
/* The loss of fmg_learn_loss with the node damping of every level (levels
   without node damping use cfg->damp), differentiated through the whole
   V-cycle: dL/domega of `level` (N of that level values) when gomega is not
   NULL.  FP64. */
int fmg_learn_loss_levels(fmg_grid* grid, const fmg_solve_cfg* cfg, const fmg_vec* e0, int level, double* loss,
                          double* gomega);
/* One training step: forward on every level above the base (the net's
   damping everywhere, as at inference), nsamples errors generated by the
   multigrid (random, then max_cycles V-cycles of A e = 0 with the current
   damping), mean loss -> *loss, and its gradient with respect to the damping
   of every level (through the whole cycle) back through the net of each
   level into the gradient accumulator. */
int fmg_learn_step(fmg_net* net, fmg_grid* grid, const fmg_solve_cfg* cfg, int nsamples,
                   unsigned long long seed, int max_cycles, double* loss);

/* The judge (no counterpart in the reference): the plain <geometric-cs>
   cycle (scalar cfg->damp) judges the cycle with the installed node damping
   the way it will be used.  cfg->method CG+MG: 6 CG steps with each on the
   same manufactured problem (random x*, b = A x*, x0 = 0), rho = per-step
   A-norm error contraction (what CG minimises).  MG: each cycle 8 times on
   A e = 0 from the same random vector, rho = the last cycle's A-norm
   contraction.  The node damping stays only if rho_learned <= 0.98
   rho_plain, else it is removed and the plain cycle is used (*accepted = 0).
   During solves: fmg_solve's MG iteration drops the node damping when the
   mean residual reduction of the last 3 cycles is worse than rho_plain (0.9
   when the judge has not run) or a cycle grows the residual 1.5x; in CG runs
   (fmg_solve CG+MG, fmg_solve_mixed), whose residual norms need not fall
   monotonically, only divergence (100x the run's initial residual) drops it,
   and CG restarts from the current residual with the plain cycle. */
int fmg_learned_judge(fmg_grid* grid, const fmg_solve_cfg* cfg, double* rho_plain, double* rho_learned,
                      int* accepted);
/* fmg_learned_judge for the mixed-precision solve: the CG probe takes its 6
   steps with fmg_solve_mixed (the FP32/BF16 cycle, with and without the node
   damping) instead of fmg_solve, so the damping is judged with the cycle that
   fmg_solve_mixed runs, at about a third of the FP64 probe's cost.
   cfg->method must be FMG_METHOD_CG_MG; mcfg as for fmg_solve_mixed
   (max_outer is ignored). */
int fmg_learned_judge_mixed(fmg_grid* grid, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mcfg,
                            double* rho_plain, double* rho_learned, int* accepted);
/* active: learned damping installed and accepted; reverts: mixed solves whose
   runtime judge fell back to the plain cycle */
int fmg_learned_status(const fmg_grid* grid, int* active, double* rho_plain, double* rho_learned, int* reverts);

/* ---------------------------------------------------------------- batches */
/* No counterpart in the reference, which solves one system per solve call:
   a batch of nbatch independent problems with the geometry of `like` (a 1D
   or 2D scalar Q1 hierarchy, base level <= 1024 unknowns), kept in shared
   buffers and solved together -- every kernel launch covers all problems,
   every reduction and CG scalar is per problem.  The result is a grid
   handle; fmg_vec_create on it makes batched vectors of nbatch x N values
   (problem k's values at k*N on the host side), fmg_grid_destroy releases
   it.  Entry points that work on a single problem refuse a batch. */
int fmg_batch_create(fmg_grid* like, int nbatch, fmg_grid** batch);
/* Problem `index` from an assembled grid of the batch's geometry: its level
   matrices, top-level rhs, coarse-level inverse and node damping (assembled
   and damped as for fmg_solve on that grid: fmg_assemble, fmg_net_apply,
   fmg_set_node_damping).  Node damping must be present on a level for every
   problem of the batch or for none.  The batch is solvable once every
   problem is loaded. */
int fmg_batch_load(fmg_grid* batch, int index, fmg_grid* src);
/* fmg_solve (solve.lisp:139-164 with <cg> krylow.lisp:72-132 or the MG
   iteration) of every problem at once, from x: CG + MG, MG or CG with the
   Jacobi smoother, multiplicative cycles, no f-cycle, compat_alias 0.  Each
   problem stops at its own tolerance (or after maxsteps) and keeps its
   iterate; steps[k], status[k] and hist[k*hist_len ..] (hist may be NULL)
   are those fmg_solve reports for problem k on its own grid, and so are the
   iterates, bit for bit.  The runtime judge of learned damping is not run:
   each problem uses the damping it was loaded with. */
int fmg_batch_solve(fmg_grid* batch, const fmg_solve_cfg* cfg, fmg_vec* x, double* hist, int hist_len, int* steps,
                    int* status);

/* No counterpart in the reference: a measurement hook for the mixed solve's
   top-level kernels.  Runs `reps` back-to-back launches of one of them on the
   grid's own mixed-solve buffers, as an earlier fmg_solve_mixed on this grid
   with the matrix-free top level left them (FMG_ERR_STATE otherwise), on the
   context's stream without waiting, so that a caller can time them with
   events on that stream.  The launches overwrite scratch vectors of the mixed
   solve only; the next solve starts afresh. */
#define FMG_MXK_RESIDUAL 1   /* FP32 r = b - A x, matrix-free */
#define FMG_MXK_SMOOTH 2     /* FP32 y = x + w (b - A x) / d with the flexible CG's two FP64 dot products */
#define FMG_MXK_MATVEC64 3   /* FP64 a = A p of the FP32 search direction, with (a, p) */
#define FMG_MXK_RESTRICT 4   /* the top-level residual restricted to the level below (BF16 rhs, x zeroed) */
#define FMG_MXK_PROLONG 5    /* the level below's correction prolongated and added to the top level */
#define FMG_MXK_PRESMOOTH 6  /* the top-level pre-smoothing from zero, y = w b / d */
int fmg_mixed_top_kernel(fmg_grid* grid, int kind, int reps);

/* No counterpart in the reference: a self-test of the device-side give-up
   path of the library's bounded waits (the mbarrier waits of the tensor-core
   kernels, which otherwise give up only after 2^24 polls or 2 s).  One CTA
   initialises an mbarrier and waits on it with the limits given (max_polls
   polls in [1, 2^24], max_ns nanoseconds of global time in [1, 2e9]); no MMA
   or bulk copy is in flight.  arrive = 1: a thread arrives first, the wait
   completes, FMG_OK.  arrive = 0: nothing arrives, the wait gives up, the
   kernel records its error word and returns, and the call reports
   FMG_ERR_CUDA with the message of a timed-out wait (fmg_last_error); the
   context stays usable. */
int fmg_wait_selftest(fmg_ctx* ctx, int arrive, int max_polls, long long max_ns);

/* ------------------------------------------------- allocation-free variant */
/* No counterpart in the reference.  The dot product of fmg_dot for callers
   that cannot allocate device memory: hosts whose device memory is already
   owned by their own pool allocator, and latency-critical loops that must not
   take the implicit device synchronisation of cudaMalloc/cudaFree.  x, y
   (n doubles) and out (1 double) are device pointers supplied by the caller;
   the result is written to *out on the context's stream (no host sync).  The
   reduction scratch is a fixed ~256 KB array inside the library, held by every
   GPU that loads it until exit.  n <= FMG_NOALLOC_MAX_N, else FMG_ERR_ARG.
   The first call on a device looks up the scratch address and should come
   before any stream capture.  Each call makes the context's device current
   while it runs and restores the caller's current device before returning.
   All calls share the scratch: calls that overlap on the GPU race. */
#define FMG_NOALLOC_MAX_N 134217728L
int fmg_dot_noalloc(fmg_ctx* ctx, const double* x, const double* y, long n, double* out);

#ifdef __cplusplus
}
#endif
#endif /* FMGPU_H */
