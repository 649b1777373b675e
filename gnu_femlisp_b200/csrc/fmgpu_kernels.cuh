// fmgpu_kernels.cuh -- launch interface of the FP64 kernels.
#pragma once

#include "fmgpu_internal.cuh"

namespace fmg {

// what a kernel needs to know about one level
// compressed rows of a sparse matrix on the device (columns ascending in a row)
struct CsrView {
  const long long* start = nullptr;  // rows + 1 offsets
  const int* index = nullptr;
  const double* value = nullptr;
};

struct LevelView {
  const double* A;      // [slot][Np], or [slot][k][l][Np] for nc = 3
  long long N, Np, M;   // nodes, padded stride, nodes per direction
  int dim, order, dmask, center;
  const double* omega;  // per-node damping or nullptr
  int nc = 1;           // components per node (1, or 3 for elasticity)
  int nb = 1;           // problems of a batched level (scalar Q1, 1D/2D): vectors Np apart, matrices slots x Np
  // algebraic levels (no geometry): the matrix in compressed rows, its
  // diagonal, and the interpolation from the level below, I (rows of this
  // level) and I^T (rows of the level below); A, M and dim are then unused
  bool csr = false;
  CsrView a, p, pt;
  const double* diag = nullptr;
  // algebraic levels: a colouring of the matrix graph for the SOR/SSC sweeps
  // (rows of one colour couple to none of each other): the rows grouped by
  // colour (device) and the colour offsets (host), ncol + 1 of them
  const int* crow = nullptr;
  const long long* coff = nullptr;
  int ncol = 0;
};

// arguments of the assembly kernel of one level
struct AsmArgs {
  long long N, Np, M, n;        // nodes, padded stride, nodes/direction, cells/direction
  int dmask, nl, nq;
  int nc = 1;                   // components (3: elasticity, Kbar/Ctab = Ebar/Etab)
  double* A;                    // out: [slot][Np]
  double* rhs;                  // out (top level only) or nullptr
  const double* Kbar;           // [a][b]: sum over Gauss points
  const double* Ctab;           // [q][a][b]
  const double* Phi;            // [q][a]
  const double* kcell;          // top level: k per cell, or nullptr
  const double* kq;             // coarse level: k per cell and Gauss point, or nullptr
  const double* fip;            // source per cell and Gauss point, or nullptr
  double kconst, fconst;
  double fvec[3] = {0.0, 0.0, 0.0};  // nc = 3: constant force per component
  int fvec_on = 0;
};

// FP32 copy of a Q2 level in the full slot layout (structural zeros
// included) from its sliced storage, [slot][block entry][Np]
void launch_level_to_f32(const LevelView& L, int nslots, float* out, cudaStream_t st);
// host-side: the node's position in slot s of a Q2 level's sliced storage
// (colour-major for scalar levels), or -1 when the slot is a structural zero
// of that node
long long q2_slot_pos(int dim, long long M, long long i, int s, bool colour_major);
// FP32 mixed cycle of the vector form (3 x 3 blocks, FP32 copies of the level
// matrices in the same layout): residual r = b - A x, first Jacobi step from a
// zero guess, fused residual + Jacobi step, transfers (restriction writes the
// coarse rhs and zeroes the coarse solution)
void vec32_spmv(int order, const float* A, long long N, long long Np, long long M, const float* x, const float* b,
                float* y, cudaStream_t st);
void vec32_jacobi0(const float* A, long long N, long long Np, int center, float damp, const double* omega,
                   const float* b, float* x, cudaStream_t st);
void vec32_jacobi_res(int order, const float* A, long long N, long long Np, long long M, double damp,
                      const double* omega, const float* x, const float* b, float* xout, cudaStream_t st);
// diagonal-block operations of the recorded cycle (vector form); mode 0:
// y = B^-1 x, 1: y = w B^-1 x, 2: y += w B^-1 x (w per node)
void launch_bdiag3(const LevelView& L, int mode, const double* w, const double* x, double* y, cudaStream_t st);
void launch_xpwv3(const double* x, const double* w, const double* v, double* y, long long N, cudaStream_t st);
void launch_acc_prod3(double* acc, const double* a, const double* b, long long N, cudaStream_t st);
void vec32_restrict(int order, long long MC, long long MF, int dmask, const float* rf, float* bc, float* xc,
                    cudaStream_t st);
void vec32_prolong(int order, long long MF, long long MC, int dmask, const float* xc, float* xf, cudaStream_t st);
// y = f x between precisions; mode 0: f = 1, 1: f = 1/sqrt(sc[slot]), 2: f = sqrt(sc[slot])
void vec_to32(const double* x, const double* sc, int slot, int mode, float* y, long long n, cudaStream_t st);
void vec_to64(const float* x, const double* sc, int slot, int mode, double* y, long long n, cudaStream_t st);
void vec_f64_to_f32(const double* x, float* y, long long n, cudaStream_t st);
// sc[S_RATIO] = first ? 0 : -sc[S_TMP] / sc[S_BETA] (FCG(1) beta)
void launch_fcg_beta(double* sc, bool first, cudaStream_t st);
// A_C := I^T A_F I for a scalar Q1 level below F (constrained interpolation)
void launch_galerkin(const LevelView& F, const LevelView& Cl, double* AC, cudaStream_t st);
void launch_spmv(const LevelView& L, const double* x, const double* b, double* y, const double* dv,
                 const Reduce* R, cudaStream_t st);
void launch_jacobi(const LevelView& L, double damp, double* x, double* r, bool write_r, cudaStream_t st);
void launch_jacobi_res(const LevelView& L, double damp, const double* x, const double* b, double* xout,
                       double* r, bool write_r, const double* dv, const Reduce* R, cudaStream_t st);
void launch_sor(const LevelView& L, double omega, double* x, const double* b, double* r, cudaStream_t st);
// <geometric-ssc>: the number of vertex blocks of a Q2 level (0 for Q1, whose
// blocks are single nodes), the block size 3^dim, the LU factors of every
// block (F: blocks x size^2 doubles, P: blocks x size bytes), and one sweep
// with them (b may be r)
long long ssc_blocks(const LevelView& L);
int ssc_block_size(int dim);
void launch_ssc_factor(const LevelView& L, double* F, unsigned char* P, cudaStream_t st);
void launch_ssc(const LevelView& L, double omega, double* x, const double* b, double* r, const double* F,
                const unsigned char* P, cudaStream_t st);
// one <geometric-psc> sweep with the residual r (not written): block
// corrections into C (blocks x size doubles, Q2), added to x in block order
void launch_psc(const LevelView& L, double damp, double* x, const double* r, const double* F,
                const unsigned char* P, double* C, cudaStream_t st);
void launch_restrict(const LevelView& F, const LevelView& C, const double* rf, double* rc, double* rhsc,
                     double* solc, cudaStream_t st);
void launch_prolong(const LevelView& C, const LevelView& F, const double* xc, double* xf, cudaStream_t st);
// nb problems of a batched base level: inverses n x n apart, vectors vs apart
void launch_coarse_solve(const double* AinvT, int n, double damp, double* x, double* r, cudaStream_t st,
                         int nb = 1, long long vs = 0);
void launch_lu(double* A, int n, int* piv, double* X, double* XT, cudaStream_t st);
void launch_fill(double* x, long long n, double v, cudaStream_t st);
void launch_copy(const double* x, double* y, long long n, cudaStream_t st);
void launch_axpy(double alpha, const double* sc, int aslot, const double* x, double* y, long long n,
                 cudaStream_t st);
void launch_dot(const double* x, const double* y, long long n, const Reduce& R, cudaStream_t st);
// per problem of nb batched vectors (vs apart): each problem's dot in its own reduction
void launch_dot_b(const double* x, const double* y, long long n, long long vs, int nb, const Reduce& R,
                  cudaStream_t st);
void launch_cg_update(const double* sc, double* x, const double* p, double* r, const double* a, double* w,
                      double* w2, double* q, long long n, const Reduce& R, cudaStream_t st);
void launch_p_update(const double* sc, double* p, const double* q, long long n, cudaStream_t st);
// batched CG updates: per-problem scalars (S_COUNT apart); problems whose
// frozen[] entry is non-zero keep x, r and p
void launch_cg_update_b(const double* sc, double* x, const double* p, double* r, const double* a, double* w,
                        double* w2, double* q, long long n, long long vs, int nb, const double* frozen,
                        const Reduce& R, cudaStream_t st);
void launch_p_update_b(const double* sc, double* p, const double* q, long long n, long long vs, int nb,
                       const double* frozen, cudaStream_t st);
void launch_sample_kq(int dim, long long ncells_l, long long n_l, long long n_top, double ratio, int np,
                      const double* xi, const double* kcell, double* kq, cudaStream_t st);
// kbar_h / ctab_h: host copies of a.Kbar / a.Ctab (null: the generic kernel)
// whether launch_assemble can form a level's rhs and matrix in separate passes
// (a.A or a.rhs null): the unrolled 3D scalar Q1 kernel
bool assemble_splits(int dim, int order, int nc, const AsmArgs& a);
void launch_assemble(int dim, int order, const AsmArgs& a, const double* kbar_h, const double* ctab_h,
                     cudaStream_t st);
void launch_densify(const LevelView& L, double* Dm, cudaStream_t st);

}  // namespace fmg
