/*
 * fmg_oracle.h -- CPU restatement of Femlisp's multigrid solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the GPU path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product (gnu_femlisp_b200/, libfmgpu.so) never links it.
 *
 * What it restates (reference paths relative to the Femlisp source root):
 *   assembly      src/discretization/fedisc.lisp:73-206 (assemble-interior,
 *                 assemble-cell), ellsys-fe.lisp:68-218 (discretize-locally),
 *                 fe.lisp:235-244,502-535 (quadrature rule, cell geometry),
 *                 quadrature.lisp:143-215 (Gauss rule), lagrange.lisp:41-152
 *   constraints   constraints.lisp:58-72,323-411, fedisc.lisp:239-253,
 *                 geomg.lisp:128-137 (Dirichlet rows become identity rows)
 *   transfers     sparseas.lisp:232-272, fetransfer.lisp:73-195 (nodal
 *                 interpolation, constrained rows/columns removed)
 *   iteration     linit.lisp:73-323 (compute-residual, product-iterator,
 *                 <lu>, <jacobi>, <sor>), multigrid.lisp:173-393 (lmgc,
 *                 smooth, restrict, prolongate, make-iterator),
 *                 krylow.lisp:72-132 (<cg>, including the rhs/residual alias
 *                 of the preconditioner call), solve.lisp:139-164,
 *                 linsolve.lisp:58-73, iterate.lisp:239-250 (solver loop).
 *
 * Parity is pinned by the reference's own known answers (mg-cdr.lisp:85-87
 * convergence rate 0.39407..., ellsys-fe.lisp:249-256 exact nodal value
 * 0.125, sparseas.lisp:401-448 P*I = Id and quadratic reproduction); the
 * reference ships no golden vectors and no Lisp runs here.
 *
 * Canonical arithmetic (the GPU FP64 path follows the same operation order,
 * which is what makes bitwise agreement possible):
 *   - every multiply-add written as fma() is a fused multiply-add; all other
 *     operations are single IEEE operations (build with -ffp-contract=off);
 *   - row sums: acc = 0; for slot s ascending: acc = fma(a_s, x_{i+off_s}, acc);
 *   - reductions (dot, l2 norm): "DR4096" -- chunks of 4096 elements;
 *     256 lanes per chunk, lane t owns chunk positions 2t+512m+u (m = 0..7,
 *     u = 0..1) and accumulates them in (m,u) order with fma; the 256 lane
 *     sums are folded per 32-lane group (halving 16,8,4,2,1) and the 8 group
 *     sums folded by halving 4,2,1; the chunk sums are then folded the same
 *     way (lane t sums chunks t, t+256, ... with plain adds).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* coefficient kinds (shared numbering with include/fmgpu.h) */
enum { ORA_K_CONST = 0, ORA_K_CELL = 1, ORA_F_CONST = 2, ORA_F_IP = 3, ORA_LAMBDA_MU_CELL = 4, ORA_F_VEC = 5 };

/* smoother kinds */
enum { ORA_JACOBI = 0, ORA_SOR = 1, ORA_SSC = 2, ORA_PSC = 3 };

/* iteration methods of the solver loop */
enum { ORA_METHOD_MG = 0, ORA_METHOD_CG_MG = 1, ORA_METHOD_CG = 2 };

typedef struct {
  int method;          /* ORA_METHOD_* */
  int smoother;        /* ORA_JACOBI, ORA_SOR, ORA_SSC or ORA_PSC (geometric-ssc / -psc, vertex blocks) */
  double damp;         /* <jacobi> :damp or <sor> :omega */
  int pre_steps, post_steps, gamma;
  int compat_alias;    /* 1: CG calls the preconditioner as (iterate q w w) */
  double coarse_damp;  /* <lu> :damp (1.0) */
  double rtol;         /* success if reduction < rtol (<=0: off) */
  double atol;         /* success if defnorm < atol (<=0: off) */
  int maxsteps;        /* failure if step > maxsteps */
  int combination;     /* 0 :multiplicative, 1 :additive (multigrid.lisp:55-70) */
  int fmg;             /* 1: f-cycle (multigrid.lisp:290-297) */
} ora_solve_cfg;

void* ora_create(int dim, int order, int ncomp, int n0, int top_level, int base_level,
                 int dirichlet_mask);
void ora_destroy(void* h);
int ora_set_coefficient(void* h, int kind, const double* vals, long n);
int ora_assemble(void* h);
/* mode 0: every level re-discretised (ora_assemble); 1: levels below the top
   as Galerkin products I^T A_{l+1} I (geomg.lisp:122-123), Q1 scalar only */
int ora_assemble_levels(void* h, int mode);
int ora_set_node_damping(void* h, int level, const double* w, long n);

long ora_nnodes(void* h, int level);
int ora_nslots(void* h);
int ora_set_matrix(void* h, int level, const double* a);   /* level matrix in the ora_get_matrix layout */
int ora_set_rhs(void* h, const double* b);                 /* top-level rhs */
/* algebraic hierarchies: levels 0 .. nlevels-1, compressed rows (columns ascending) */
void* ora_create_algebraic(int nlevels, const long* sizes);
int ora_set_csr_matrix(void* h, int level, const long* start, const int* index, const double* value);
int ora_set_interpolation(void* h, int fine_level, const long* start, const int* index, const double* value);
int ora_finish_levels(void* h);                            /* coarse inverse once every level is set */
int ora_get_matrix(void* h, int level, double* out);      /* [slot][k][l][node] (nc x nc blocks) */
int ora_get_rhs(void* h, double* out);
int ora_get_coarse_inverse(void* h, double* out);           /* n*n row-major */

int ora_matvec(void* h, int level, const double* x, double* y);
int ora_residual(void* h, int level, const double* x, const double* b, double* r);
int ora_restrict(void* h, int fine_level, const double* rf, double* rc);
int ora_prolongate(void* h, int coarse_level, const double* xc, double* xf, int constrained);
int ora_inject(void* h, int coarse_level, const double* xf, double* xc);
int ora_jacobi(void* h, int level, double damp, double* x, double* r);
int ora_sor(void* h, int level, double omega, double* x, const double* b, double* r);
int ora_psc(void* h, int level, double damp, double* x, const double* r);
int ora_ssc(void* h, int level, double omega, double* x, const double* b, double* r);
int ora_coarse_solve(void* h, double damp, double* x, double* r);
double ora_dot(const double* x, const double* y, long n);
double ora_dot_par(const double* x, const double* y, long n);   /* same result, OpenMP chunks */

/* one application of the multigrid iterator (multigrid.lisp:366-386);
   pass b == r to get the aliasing of the CG preconditioner call */
int ora_vcycle(void* h, const ora_solve_cfg* cfg, double* x, double* b, double* r);

/* the full solver loop; x is the solution (in/out, start 0), hist receives
   the defnorm per step (len >= maxsteps+2). returns 0 on success, 1 on
   failure (maxsteps), <0 on error */
int ora_solve(void* h, const ora_solve_cfg* cfg, double* x, double* hist, int hist_len,
              int* nsteps);

/* The 3D Q1 operator of a cell-wise coefficient applied matrix-free, in the
   operation order of the GPU's matrix-free top level (the operator of its
   mixed-precision solve; no counterpart in the reference, which always
   assembles): per node, from the 8 cell coefficients k and the neighbour
   values x (zero at Dirichlet nodes and outside the grid),
     wc[sy][sx] = k[0][sy][sx] + k[1][sy][sx],  K = (wc00 + wc01) + (wc10 + wc11),
     12 face-diagonal and 8 body-diagonal terms in a fixed order, each
     s = fma(w, x_i - x_j, s) (FP64) or s = fma(w, x_j, s), s = fma(4K, x_i, -s) (FP32),
     (A x)_i = (h/12) s; Dirichlet rows are identity rows.
   It equals assemble-interior's matrix (fedisc.lisp:108-206) times x up to
   rounding.  fp32 = 1: k, x, b and h/12 rounded to FP32 and FP32
   arithmetic; fp32 = 2: x rounded to FP32, FP64 arithmetic.  b == NULL: y = A x, else y = b - A x.  M nodes a side,
   k: (M-1)^3 cells, x fastest. */
void ora_mf_apply(int M, int dmask, const double* k, int fp32, const double* x, const double* b, double* y);

int ora_num_threads(void);
void ora_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
