// fmgpu.cu -- host runtime of libfmgpu.so: handles, assembly driver, the
// multigrid iterator and the <linear-solver>/<cg> loop, and the C-ABI.
//
// The multigrid iterator replays Femlisp's bookkeeping exactly
// (multigrid.lisp:173-393, linit.lisp:73-323): per level a residual-p flag
// decides when compute-residual runs, the product-iterator recomputes the
// residual after each Jacobi step, restrict zeroes the coarse solution and
// copies the restricted residual into the coarse rhs, and the top level uses
// the caller's vectors without copying -- so passing the same vector as rhs
// and residual reproduces the alias of the <cg> preconditioner call.
// Kernel fusion is applied only where it leaves every observable value
// unchanged: compute-residual is fused into the Jacobi step that consumes it,
// and the residual writes of a smoother are skipped when nothing can read them
// before they are recomputed (distinct rhs and residual vectors).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <algorithm>
#include <string>
#include <utility>

#include "fmgpu_kernels.cuh"
#include "fmgpu_learn.cuh"
#include "fmgpu_mixed.cuh"

using namespace fmg;

struct fmg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  double* host_scal = nullptr;  // pinned copy of a grid's scalar slots
  std::string err;
  int grids = 0;                // live grids and nets: the context outlives them
  bool closed = false;          // fmg_finalize called while grids were alive
};

namespace {

struct Lvl {
  long long n = 0, M = 0, N = 0, Np = 0;
  double h = 0;
  double* A = nullptr;
  double* omega = nullptr;
  double* sol[2] = {nullptr, nullptr};
  double* rhs = nullptr;
  double* res = nullptr;
  double* Kbar = nullptr;
  double* Ctab = nullptr;
  double* Phi = nullptr;
  std::vector<double> Kbar_h, Ctab_h;  // host copies of the element tables
  // algebraic levels: the matrix, the interpolation from the level below and
  // its transpose in compressed rows, and the matrix diagonal (device)
  struct Csr {
    long long* start = nullptr;
    int* index = nullptr;
    double* value = nullptr;
  } ca, cp, cpt;
  double* diag = nullptr;
  // the colouring of an algebraic level's matrix graph (SOR/SSC sweeps):
  // rows grouped by colour, ascending inside a colour, and colour offsets
  std::vector<long long> coff;
  int* crow = nullptr;
};

}  // namespace

struct fmg_grid {
  fmg_ctx* ctx = nullptr;
  int dim = 0, order = 0, nc = 1, n0 = 1, top = 0, base = 0, dmask = 0;
  int nslots = 0, center = 0, nl = 0, nq = 0, np = 0;
  std::vector<Lvl> lev;
  int kkind = FMG_K_CONST;
  double kconst = 1.0;
  int fkind = FMG_F_CONST;
  double fconst = 1.0;
  double fvec[3] = {0.0, 0.0, 0.0};  // FMG_F_VEC
  double xi_h[3] = {0, 0, 0};
  double* xi_d = nullptr;
  double* kcell_d = nullptr;
  double* fip_d = nullptr;
  double* rhs = nullptr;       // assembled top-level rhs
  double* ainvT = nullptr;     // base-level inverse, transposed
  int nbase = 0;
  double* scal = nullptr;      // S_COUNT scalar slots
  double* part = nullptr;      // reduction partials
  unsigned* counter = nullptr;
  // top-level work vectors of the solvers
  double *p = nullptr, *a = nullptr, *w = nullptr, *w2 = nullptr, *q = nullptr, *r = nullptr,
         *xs = nullptr, *xs2 = nullptr;
  bool assembled = false;
  bool assembled_once = false;
  std::vector<char> have;      // levels whose matrix is in place
  bool uploaded = false;       // some level matrix came from fmg_set_matrix
  bool algebraic = false;      // levels without geometry: matrices and interpolations from the host
  std::vector<char> haveP;     // algebraic: levels whose interpolation from the level below is in place
  bool top_deferred = false;   // the top level's matrix is formed on first use (its rhs is in place)
  // <geometric-ssc>: LU factors of the vertex blocks per level, formed once per assembly
  std::vector<double*> sscF;
  std::vector<unsigned char*> sscP;
  std::vector<double*> sscC;   // <geometric-psc>: the blocks' corrections
  std::vector<long long> sscEpoch;
  bool ssc_unprepared = false; // a sweep found no factors (and was not run)
  long long epoch = 0;         // incremented by every assembly
  struct MixedState* mx = nullptr;
  struct MixedVec* mxv = nullptr;  // mixed solve state of the vector (elasticity) form
  bool x_zero = false;             // the judge's probe: the next solve starts from x = 0 (r = b, no matvec)
  double* kq = nullptr;        // Gauss-point coefficient samples of a coarse level
  double *lu = nullptr, *lux = nullptr;  // coarse LU factors and inverse workspace
  int* piv = nullptr;
  // multigrid state (multigrid.lisp:101-116)
  std::vector<double*> solp, sparep, rhsp, resp;
  std::vector<int> rp;
  int cur = 0;
  double* lt[10] = {};         // top-level vectors of the damping-network training loss
  std::vector<std::vector<double*>> lvv;  // per-level vectors of the recorded linear V-cycle
  bool learned = false;        // per-node damping installed by a damping network
  double rho_plain = 0.0;      // judge: slow-mode contraction of the plain cycle (0: not measured)
  double rho_learned = 0.0;    //        and of the learned cycle
  int reverts = 0;             // mixed solves whose runtime judge fell back to the plain cycle
  // <cg> iterator run step by step (fmg_cg_start / fmg_cg_step): alpha of the
  // last restart or step, and the configuration it was started with
  double cg_alpha = 0.0;
  bool cg_started = false;
  fmg_solve_cfg cg_cfg{};
  // a batch (fmg_batch_create): nb problems of one geometry at fixed strides
  // in every buffer; each is loaded from an assembled grid (fmg_batch_load)
  int nb = 1;
  std::vector<char> loaded;
  double* frozen = nullptr;    // per problem: non-zero once its solve has stopped
  std::vector<void*> allocs;
  int vecs = 0;                // live vectors: the grid outlives them
  bool destroyed = false;      // fmg_grid_destroy called while vectors were alive
};

struct fmg_vec {
  fmg_grid* g = nullptr;
  int level = 0;
  long long n = 0;
  double* d = nullptr;
};

// device data of the mixed-precision solve, built from an assembly
struct MixedState {
  long long epoch = -1;             // assembly it was converted from
  bool top32 = false;               // the top level's FP32 copy is of that assembly
  bool mf = false;                  // top level applied matrix-free
  std::vector<Lev32> lv;            // per level (FP32 matrices)
  std::vector<float*> A32, om32, x0, x1;
  std::vector<__nv_bfloat16*> bc, rc;  // coarse rhs and residual (BF16)
  float* k32 = nullptr;             // top-level cell coefficients (FP32)
  float *rtop = nullptr, *r = nullptr, *q = nullptr, *qs = nullptr;  // FP32 top-level vectors
  float *zp = nullptr, *zs = nullptr;  // the in-solve judge: the plain cycle's result and its spare
  float* p32 = nullptr;             // FP32 search direction of the flexible CG
  double *r64 = nullptr, *a64 = nullptr;  // FP64 residual and A p of the mixed solve (layout lay)
  double* x64 = nullptr;            // the solve's iterate in layout lay (copied from and back to the caller's)
  VLay lay;                         // layout of the top-level vectors above (rtop excepted):
                                    // padded with the matrix-free top level, natural otherwise
  long long cap = 0;                // elements each top-level vector holds
  float* wd = nullptr;              // top level: damping / diagonal per node (matrix-free smoothing)
  const float* wd_om = nullptr;     // the node damping and scalar damping wd was formed with
  float wd_w = 0.f;
  bool wd_ok = false;
  double* sc = nullptr;
  double* part = nullptr;
  unsigned* counter = nullptr;
  double* host = nullptr;           // pinned copy of sc
  // CUDA graphs of one flexible-CG step, keyed by every pointer and value the
  // captured kernels bake in (the V-cycle's ping-pong buffers alternate)
  struct StepGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
    float *q = nullptr, *qs = nullptr;
    std::vector<float*> x0, x1;
  };
  std::vector<StepGraph> graphs;
  bool graphs_off = false;          // a capture failed: launch eagerly from then on
};

// the top level's matrix where its assembly was deferred (defined below,
// among the entry points)
extern "C" {
static int ensure_top(fmg_grid* g);
}

// ------------------------------------------------------------------ errors
namespace {

int set_err(fmg_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

int cuda_err(fmg_ctx* c, cudaError_t e, const char* what) {
  return set_err(c, FMG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// return a non-zero status
#define FMG_RC(expr)                   \
  do {                                 \
    const int rc_ = (expr);            \
    if (rc_) return rc_;               \
  } while (0)
#define FMG_CK(ctx, call)                                   \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_err((ctx), e_, #call); \
  } while (0)

int launched(fmg_ctx* c, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(c, e, what);
  return FMG_OK;
}

long long pad64(long long n) { return (n + 63) / 64 * 64; }

int dalloc(fmg_grid* g, double** p, long long n) {
  void* q = nullptr;
  size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(double);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(g->ctx, FMG_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(q, 0, bytes, g->ctx->stream);
  if (e != cudaSuccess) return cuda_err(g->ctx, e, "cudaMemsetAsync");
  g->allocs.push_back(q);
  *p = (double*)q;
  return FMG_OK;
}

void dfree(fmg_grid* g, void* p) {
  if (!p) return;
  for (auto it = g->allocs.begin(); it != g->allocs.end(); ++it)
    if (*it == p) { g->allocs.erase(it); break; }
  cudaFree(p);
}

// ------------------------------------------------------------ FE tables
// Gauss rule with order+1 points per direction on [0,1] (fe.lisp:235-244,
// quadrature.lisp:202-215): xi = (1 - t)/2 for the Gauss-Legendre nodes t in
// ascending order, weights w_GL/2.
void gauss1d(int order, int* np, double* xi, double* w) {
  if (order == 1) {
    const double t = std::sqrt(1.0 / 3.0);
    const double ts[2] = {-t, t};
    *np = 2;
    for (int k = 0; k < 2; ++k) { xi[k] = 0.5 * (1.0 - ts[k]); w[k] = 0.5; }
  } else {
    const double t = std::sqrt(0.6);
    const double ts[3] = {-t, 0.0, t};
    const double wg[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    *np = 3;
    for (int k = 0; k < 3; ++k) { xi[k] = 0.5 * (1.0 - ts[k]); w[k] = 0.5 * wg[k]; }
  }
}

// 1D Lagrange basis on the uniform nodes 0, 1/p, .., 1 (lagrange.lisp:41-51)
double lag(int order, int a, double s) {
  if (order == 1) return a == 0 ? 1.0 - s : s;
  if (a == 0) return 2.0 * (s - 0.5) * (s - 1.0);
  if (a == 1) return 4.0 * s * (1.0 - s);
  return 2.0 * s * (s - 0.5);
}
double dlag(int order, int a, double s) {
  if (order == 1) return a == 0 ? -1.0 : 1.0;
  if (a == 0) return 4.0 * s - 3.0;
  if (a == 1) return 4.0 - 8.0 * s;
  return 4.0 * s - 1.0;
}

// Element tables of one level (cell width h): the integration weight at q is
// W_q h^d (fe-cell-geometry, fe.lisp:502-535) and the physical gradient is the
// reference gradient times 1/h; C[q][a][b] = W_q h^d grad phi_a . grad phi_b,
// Kbar = sum_q C[q], Phi[q][a] = W_q h^d phi_a (ellsys-fe.lisp:120-127,183-190).
void make_tables(int dim, int order, double h, std::vector<double>& C, std::vector<double>& Kbar,
                 std::vector<double>& Phi, int* nl_out, int* nq_out) {
  int np;
  double xi[3], w[3];
  gauss1d(order, &np, xi, w);
  const int p1 = order + 1;
  int nl = 1, nq = 1;
  for (int k = 0; k < dim; ++k) { nl *= p1; nq *= np; }
  double vol = 1.0;
  for (int k = 0; k < dim; ++k) vol = vol * h;
  const double invh = 1.0 / h;
  C.assign((size_t)nq * nl * nl, 0.0);
  Kbar.assign((size_t)nl * nl, 0.0);
  Phi.assign((size_t)nq * nl, 0.0);
  std::vector<double> G((size_t)nl * 3), phi(nl);
  for (int q = 0; q < nq; ++q) {
    const int qi[3] = {q % np, (q / np) % np, q / (np * np)};
    double W = 1.0;
    for (int k = 0; k < dim; ++k) W = W * w[qi[k]];
    const double Wv = W * vol;
    for (int a = 0; a < nl; ++a) {
      const int ai[3] = {a % p1, (a / p1) % p1, a / (p1 * p1)};
      double v = 1.0;
      for (int k = 0; k < dim; ++k) v = v * lag(order, ai[k], xi[qi[k]]);
      phi[a] = v;
      for (int kd = 0; kd < dim; ++kd) {
        double gg = 1.0;
        for (int k = 0; k < dim; ++k)
          gg = gg * (k == kd ? dlag(order, ai[k], xi[qi[k]]) : lag(order, ai[k], xi[qi[k]]));
        G[a * 3 + kd] = gg * invh;
      }
    }
    for (int a = 0; a < nl; ++a) {
      Phi[(size_t)q * nl + a] = Wv * phi[a];
      for (int b = 0; b < nl; ++b) {
        double gg = G[a * 3] * G[b * 3];
        for (int kd = 1; kd < dim; ++kd) gg = std::fma(G[a * 3 + kd], G[b * 3 + kd], gg);
        C[((size_t)q * nl + a) * nl + b] = Wv * gg;
      }
    }
  }
  for (int q = 0; q < nq; ++q)
    for (int ab = 0; ab < nl * nl; ++ab) Kbar[ab] = Kbar[ab] + C[(size_t)q * nl * nl + ab];
  *nl_out = nl;
  *nq_out = nq;
}

// Elastic tables of one level, lambda = mu = E (isotropic-elasticity-tensor,
// elasticity.lisp:71-88, in the A-term of ellsys-fe.lisp:120-127), per unit E:
//   Etab[q][a][b][k][l] = W_q h^d (G_ak G_bl + G_al G_bk + d_kl G_a . G_b),
// t = fma(G_al, G_bk, G_ak G_bl), t = t + G_a . G_b on the diagonal, the dot
// as an fma chain over the directions; Ebar = sum_q Etab[q].
void make_elastic_tables(int dim, int order, double h, std::vector<double>& E, std::vector<double>& Ebar) {
  int np;
  double xi[3], w[3];
  gauss1d(order, &np, xi, w);
  const int p1 = order + 1;
  int nl = 1, nq = 1;
  for (int k = 0; k < dim; ++k) { nl *= p1; nq *= np; }
  double vol = 1.0;
  for (int k = 0; k < dim; ++k) vol = vol * h;
  const double invh = 1.0 / h;
  const size_t per_q = (size_t)nl * nl * dim * dim;
  E.assign(per_q * nq, 0.0);
  Ebar.assign(per_q, 0.0);
  std::vector<double> G((size_t)nl * 3);
  for (int q = 0; q < nq; ++q) {
    const int qi[3] = {q % np, (q / np) % np, q / (np * np)};
    double W = 1.0;
    for (int k = 0; k < dim; ++k) W = W * w[qi[k]];
    const double Wv = W * vol;
    for (int a = 0; a < nl; ++a) {
      const int ai[3] = {a % p1, (a / p1) % p1, a / (p1 * p1)};
      for (int kd = 0; kd < dim; ++kd) {
        double gg = 1.0;
        for (int k = 0; k < dim; ++k)
          gg = gg * (k == kd ? dlag(order, ai[k], xi[qi[k]]) : lag(order, ai[k], xi[qi[k]]));
        G[a * 3 + kd] = gg * invh;
      }
    }
    for (int a = 0; a < nl; ++a)
      for (int b = 0; b < nl; ++b) {
        double gg = G[a * 3] * G[b * 3];
        for (int kd = 1; kd < dim; ++kd) gg = std::fma(G[a * 3 + kd], G[b * 3 + kd], gg);
        for (int k = 0; k < dim; ++k)
          for (int l = 0; l < dim; ++l) {
            double t = std::fma(G[a * 3 + l], G[b * 3 + k], G[a * 3 + k] * G[b * 3 + l]);
            if (k == l) t = t + gg;
            E[(size_t)q * per_q + (((size_t)a * nl + b) * dim + k) * dim + l] = Wv * t;
          }
      }
  }
  for (int q = 0; q < nq; ++q)
    for (size_t e = 0; e < per_q; ++e) Ebar[e] = Ebar[e] + E[(size_t)q * per_q + e];
}

int upload(fmg_grid* g, double** dst, const std::vector<double>& v) {
  int rc = dalloc(g, dst, (long long)v.size());
  if (rc) return rc;
  FMG_CK(g->ctx, cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 g->ctx->stream));
  return FMG_OK;
}

LevelView view(const fmg_grid* g, int l) {
  const Lvl& L = g->lev[l];
  LevelView v;
  v.A = L.A; v.N = L.N; v.Np = L.Np; v.M = L.M;
  v.dim = g->dim; v.order = g->order; v.dmask = g->dmask; v.center = g->center;
  v.omega = L.omega;
  v.nc = g->nc;
  v.nb = g->nb;
  if (g->algebraic) {
    v.csr = true;
    v.a = CsrView{L.ca.start, L.ca.index, L.ca.value};
    v.p = CsrView{L.cp.start, L.cp.index, L.cp.value};
    v.pt = CsrView{L.cpt.start, L.cpt.index, L.cpt.value};
    v.diag = L.diag;
    v.crow = L.crow;
    v.coff = L.coff.data();
    v.ncol = L.coff.empty() ? 0 : (int)L.coff.size() - 1;
  }
  return v;
}

Reduce reducer(fmg_grid* g, int epi, int slot) {
  Reduce R;
  R.part = g->part; R.counter = g->counter; R.scal = g->scal; R.epi = epi; R.slot = slot;
  return R;
}

// ------------------------------------------------------- multigrid iterator
struct MG {
  fmg_grid* g;
  const fmg_solve_cfg& c;
  bool literal;          // keep every residual write (fmg_vcycle on user vectors)
  cudaStream_t st;

  bool alias(int l) const { return g->rhsp[l] == g->resp[l]; }

  void residual(int l) {
    launch_spmv(view(g, l), g->solp[l], g->rhsp[l], g->resp[l], nullptr, nullptr, st);
  }
  void ensure_res() {  // ensure-mg-residual (multigrid.lisp:173-177)
    const int l = g->cur;
    if (!g->rp[l]) { residual(l); g->rp[l] = 1; }
  }
  // one <jacobi> step; with need_res the preceding compute-residual is fused in
  void jacobi_step(int l, bool need_res) {
    const bool write_r = literal || alias(l);
    if (need_res) {
      launch_jacobi_res(view(g, l), c.damp, g->solp[l], g->rhsp[l], g->sparep[l], g->resp[l], write_r,
                        nullptr, nullptr, st);
      std::swap(g->solp[l], g->sparep[l]);
    } else {
      launch_jacobi(view(g, l), c.damp, g->solp[l], g->resp[l], write_r, st);
    }
  }
  void smooth(int steps) {  // smooth (multigrid.lisp:179-189) + product-iterator (linit.lisp:94-120)
    if (steps <= 0) return;
    const int l = g->cur;
    if (c.smoother == FMG_JACOBI) {
      bool need = !g->rp[l];  // residual-before: ensure-mg-residual
      for (int s = 0; s < steps; ++s) {
        jacobi_step(l, need);
        need = true;          // the product-iterator recomputes after every step
      }
      if (steps > 1 && (literal || alias(l))) residual(l);
    } else if (c.smoother == FMG_SSC) {
      // residual-before t, residual-after nil (blockit.lisp:118-204): the
      // block sweep reads b and x only, so the residuals of ensure-mg-residual
      // and of the product-iterator matter only where they are seen (a
      // user's r) or where r is b (the alias inside <cg>)
      const bool keep = literal || alias(l);
      const bool ready = g->order == 1 || ((int)g->sscF.size() > l && g->sscF[l] && g->sscEpoch[l] == g->epoch);
      if (!ready) { g->ssc_unprepared = true; g->rp[l] = 0; return; }
      if (keep) ensure_res();
      for (int s = 0; s < steps; ++s) {
        launch_ssc(view(g, l), c.damp, g->solp[l], g->rhsp[l], g->resp[l], g->order == 2 ? g->sscF[l] : nullptr,
                   g->order == 2 ? g->sscP[l] : nullptr, st);
        if (steps > 1 && keep) residual(l);
      }
    } else if (c.smoother == FMG_PSC) {
      // residual-before t, residual-after nil, r read and not written
      // (blockit.lisp:118-204): the residual before every step, as for <jacobi>
      const bool ready = g->order == 1 || ((int)g->sscF.size() > l && g->sscF[l] && g->sscEpoch[l] == g->epoch);
      if (!ready) { g->ssc_unprepared = true; g->rp[l] = 0; return; }
      bool need = !g->rp[l];
      for (int s = 0; s < steps; ++s) {
        if (need) residual(l);
        launch_psc(view(g, l), c.damp, g->solp[l], g->resp[l], g->order == 2 ? g->sscF[l] : nullptr,
                   g->order == 2 ? g->sscP[l] : nullptr, g->order == 2 ? g->sscC[l] : nullptr, st);
        need = true;
      }
      if (steps > 1 && (literal || alias(l))) residual(l);
    } else {
      for (int s = 0; s < steps; ++s) launch_sor(view(g, l), c.damp, g->solp[l], g->rhsp[l], g->resp[l], st);
    }
    g->rp[l] = 0;
  }
  void restrict_() {  // restrict + :after methods (multigrid.lisp:202-224)
    const int l = g->cur;
    ensure_res();
    launch_restrict(view(g, l), view(g, l - 1), g->resp[l], g->resp[l - 1], g->rhsp[l - 1], g->solp[l - 1], st);
    g->cur = l - 1;
    g->rp[l - 1] = 1;
  }
  void prolongate() {  // multigrid.lisp:237-252
    const int l = g->cur;
    launch_prolong(view(g, l), view(g, l + 1), g->solp[l], g->solp[l + 1], st);
    g->cur = l + 1;
    g->rp[l + 1] = 0;
  }
  void lmgc() {  // multigrid.lisp:254-288
    const int l = g->cur;
    if (l == g->base) {
      launch_coarse_solve(g->ainvT, g->nbase, c.coarse_damp, g->solp[l], g->resp[l], st, g->nb, g->lev[l].Np);
      g->rp[l] = 0;
      return;
    }
    if (c.combination == FMG_MULTIPLICATIVE) {
      smooth(c.pre_steps);
      restrict_();
    } else {
      restrict_();
      g->cur += 1;
      smooth(c.pre_steps);
      g->cur -= 1;
    }
    const int gam = c.gamma == 0 ? 0 : (g->cur == g->base ? 1 : c.gamma);
    for (int i = gam; i >= 1; --i) {
      lmgc();
      if (i != 1) ensure_res();
    }
    if (c.combination == FMG_MULTIPLICATIVE) {
      prolongate();
      smooth(c.post_steps);
    } else {
      g->cur += 1;
      smooth(c.post_steps);
      g->cur -= 1;
      prolongate();
    }
  }
  // f-cycle (multigrid.lisp:290-297): restrict from the top to the base
  // level, then from the base up a cycle on each level and, below the top,
  // the prolongation of its solution to the level above
  void fcycle() {
    const int top = g->cur;
    for (int l = top; l > g->base; --l) restrict_();
    for (int l = g->base; l <= top; ++l) {
      lmgc();
      if (l != top) prolongate();
    }
  }
  // the iterate closure of the multigrid iterator (multigrid.lisp:366-386);
  // *x may be swapped with *spare (ping-pong of fused Jacobi steps)
  void iterate(double** x, double** spare, double* b, double* r) {
    const int top = g->top;
    g->solp[top] = *x; g->sparep[top] = *spare;
    g->rhsp[top] = b; g->resp[top] = r;
    g->rp[top] = 1;
    g->cur = top;
    if (c.fmg) fcycle();
    else lmgc();
    *x = g->solp[top];
    *spare = g->sparep[top];
  }
};

// the LU factors of the vertex blocks of level l (scalar Q2) for the SSC
// sweeps, formed once per assembly
int ssc_prepare(fmg_grid* g, int l) {
  if ((int)g->sscF.size() != g->top + 1) {
    g->sscF.assign(g->top + 1, nullptr);
    g->sscP.assign(g->top + 1, nullptr);
    g->sscC.assign(g->top + 1, nullptr);
    g->sscEpoch.assign(g->top + 1, -1);
  }
  if (l == g->top) FMG_RC(ensure_top(g));
  const LevelView v = view(g, l);
  const long long nb = ssc_blocks(v);
  if (nb == 0 || g->sscEpoch[l] == g->epoch) return FMG_OK;
  const int bs = ssc_block_size(g->dim);
  int rc;
  if (!g->sscF[l]) {
    double* p = nullptr;
    if ((rc = dalloc(g, &g->sscF[l], nb * bs * bs)) || (rc = dalloc(g, &p, (nb * bs + 7) / 8)) ||
        (rc = dalloc(g, &g->sscC[l], nb * bs)))
      return rc;
    g->sscP[l] = (unsigned char*)p;
  }
  launch_ssc_factor(v, g->sscF[l], g->sscP[l], g->ctx->stream);
  if ((rc = launched(g->ctx, "ssc factor"))) return rc;
  g->sscEpoch[l] = g->epoch;
  return FMG_OK;
}

int check_cfg(fmg_grid* g, const fmg_solve_cfg* c) {
  if (!c) return set_err(g->ctx, FMG_ERR_ARG, "null configuration");
  if (g->algebraic && c->smoother == FMG_PSC)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "algebraic grids: Jacobi, SOR and one-unknown SSC");
  if (g->nc != 1 && c->smoother != FMG_JACOBI)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "3-component grids: the (block) Jacobi smoother only");
  if (c->smoother != FMG_JACOBI && c->smoother != FMG_SOR && c->smoother != FMG_SSC && c->smoother != FMG_PSC)
    return set_err(g->ctx, FMG_ERR_ARG, "unknown smoother %d", c->smoother);
  if (c->pre_steps < 0 || c->post_steps < 0 || c->gamma < 0 || c->gamma > 4)
    return set_err(g->ctx, FMG_ERR_ARG, "bad cycle parameters");
  if (c->combination != FMG_MULTIPLICATIVE && c->combination != FMG_ADDITIVE)
    return set_err(g->ctx, FMG_ERR_ARG, "bad combination");
  if (c->method < FMG_METHOD_MG || c->method > FMG_METHOD_CG)
    return set_err(g->ctx, FMG_ERR_ARG, "bad method");
  if (c->fmg != 0 && c->fmg != 1) return set_err(g->ctx, FMG_ERR_ARG, "fmg is 0 or 1");
  g->ssc_unprepared = false;
  if (c->smoother == FMG_SSC || c->smoother == FMG_PSC) {  // block factors of every smoothed level
    for (int l = g->base + 1; l <= g->top; ++l) {
      const int rc = ssc_prepare(g, l);
      if (rc) return rc;
    }
  }
  return FMG_OK;
}

int vec_check(const fmg_vec* v, const fmg_grid* g, int level) {
  if (!v || v->g != g || v->level != level) return FMG_ERR_ARG;
  return FMG_OK;
}

// copies the grid scalars to the host and waits
int read_scalars(fmg_grid* g) {
  fmg_ctx* c = g->ctx;
  FMG_CK(c, cudaMemcpyAsync(c->host_scal, g->scal, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  if (c->host_scal[S_MFERR] != 0.0) {  // a matrix-free kernel gave up on a copy: its results are void
    FMG_CK(c, cudaMemsetAsync(g->scal + S_MFERR, 0, sizeof(double), c->stream));
    if (g->mx) FMG_CK(c, cudaMemsetAsync(g->mx->counter, 0, sizeof(unsigned), c->stream));
    return set_err(c, FMG_ERR_CUDA, "a bounded wait of the matrix-free operator timed out (the kernel gave up)");
  }
  return FMG_OK;
}

}  // namespace

// =================================================================== C-ABI
extern "C" {

int fmg_init(int device, fmg_ctx** out) {
  if (!out) return FMG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || device < 0 || device >= ndev) return FMG_ERR_CUDA;
  fmg_ctx* c = new (std::nothrow) fmg_ctx();
  if (!c) return FMG_ERR_NOMEM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost((void**)&c->host_scal, S_COUNT * sizeof(double)) != cudaSuccess) {
    delete c;
    return FMG_ERR_CUDA;
  }
  *out = c;
  return FMG_OK;
}

static void ctx_release(fmg_ctx* c) {
  cudaStreamSynchronize(c->stream);
  cudaFreeHost(c->host_scal);
  cudaStreamDestroy(c->stream);
  delete c;
}

// Releases the context; if grids of it are still alive the release happens
// when the last of them is destroyed.
int fmg_finalize(fmg_ctx* c) {
  if (!c || c->closed) return FMG_ERR_ARG;
  c->closed = true;
  if (c->grids == 0) ctx_release(c);
  return FMG_OK;
}

int fmg_last_error(fmg_ctx* c, char* buf, int len) {
  if (!c || !buf || len <= 0) return FMG_ERR_ARG;
  snprintf(buf, (size_t)len, "%s", c->err.c_str());
  return FMG_OK;
}

int fmg_synchronize(fmg_ctx* c) {
  if (!c) return FMG_ERR_ARG;
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  return FMG_OK;
}

int fmg_launch_count(long long* out) {
  if (!out) return FMG_ERR_ARG;
  *out = g_launches.load(std::memory_order_relaxed);
  return FMG_OK;
}

int fmg_get_stream(fmg_ctx* c, void** stream) {
  if (!c || !stream) return FMG_ERR_ARG;
  *stream = (void*)c->stream;
  return FMG_OK;
}

int fmg_grid_create(fmg_ctx* c, int dim, int order, int ncomp, int n0, int top_level, int base_level,
                    int dirichlet_mask, fmg_grid** out) {
  if (!c || !out) return FMG_ERR_ARG;
  *out = nullptr;
  if (dim < 1 || dim > 3 || order < 1 || order > 2 || n0 < 1 || base_level < 0 || base_level > top_level ||
      top_level >= kMaxLevels)
    return set_err(c, FMG_ERR_ARG, "unsupported grid (dim %d order %d levels %d..%d)", dim, order, base_level,
                   top_level);
  if (ncomp != 1 && !(ncomp == 3 && dim == 3))
    return set_err(c, FMG_ERR_UNSUPPORTED, "ncomp %d: scalar problems and 3D elasticity (3) are built", ncomp);
  fmg_grid* g = new (std::nothrow) fmg_grid();
  if (!g) return FMG_ERR_NOMEM;
  g->ctx = c;
  c->grids += 1;
  g->dim = dim; g->order = order; g->nc = ncomp; g->n0 = n0;
  g->top = top_level; g->base = base_level; g->dmask = dirichlet_mask;
  int w = 2 * order + 1;
  g->nslots = 1;
  for (int k = 0; k < dim; ++k) g->nslots *= w;
  g->center = (g->nslots - 1) / 2;
  g->lev.resize(top_level + 1);
  for (int l = 0; l <= top_level; ++l) {
    Lvl& L = g->lev[l];
    L.n = (long long)n0 << l;
    L.M = order * L.n + 1;
    L.N = 1;
    for (int k = 0; k < dim; ++k) L.N *= L.M;
    L.Np = pad64(L.N);
    L.h = 1.0 / (double)L.n;
  }
  double wq[3];
  gauss1d(order, &g->np, g->xi_h, wq);
  g->nl = 1; g->nq = 1;
  for (int k = 0; k < dim; ++k) { g->nl *= order + 1; g->nq *= g->np; }
  *out = g;
  return FMG_OK;
}

static int ensure_buffers(fmg_grid* g);
static int finish_levels(fmg_grid* g);
static bool host_csr(long nrows, long ncols, int layout, const int* start, const int* index, const double* values,
                     std::vector<long long>& rs, std::vector<int>& ci, std::vector<double>& cv, std::string& err);
static int upload_csr(fmg_grid* g, Lvl::Csr& d, const std::vector<long long>& rs, const std::vector<int>& ci,
                      const std::vector<double>& cv);
static bool hierarchy_complete(const fmg_grid* g);

// A hierarchy of algebraic levels 0 .. nlevels-1 (0 the coarsest) with the
// given numbers of unknowns: no geometry, the level matrices and the
// interpolations between the levels come from the host (fmg_set_matrix,
// fmg_set_interpolation) -- the matrices Femlisp forms on an unstructured or
// adaptively refined mesh (multilevel-decomposition, geomg.lisp:109-142, with
// the constrained interpolation of constraints.lisp:58-72).
int fmg_grid_create_algebraic(fmg_ctx* c, int nlevels, const long* sizes, fmg_grid** out) {
  if (!c || !out || !sizes) return FMG_ERR_ARG;
  *out = nullptr;
  if (nlevels < 1 || nlevels > kMaxLevels) return set_err(c, FMG_ERR_ARG, "nlevels %d out of range", nlevels);
  for (int l = 0; l < nlevels; ++l)
    if (sizes[l] < 1 || sizes[l] > (1L << 31) - 1) return set_err(c, FMG_ERR_ARG, "level %d: %ld unknowns", l, sizes[l]);
  fmg_grid* g = new (std::nothrow) fmg_grid();
  if (!g) return FMG_ERR_NOMEM;
  g->ctx = c;
  c->grids += 1;
  g->algebraic = true;
  g->dim = 0; g->order = 1; g->nc = 1; g->n0 = 1;
  g->top = nlevels - 1; g->base = 0; g->dmask = 0;
  g->nslots = 1; g->center = 0;
  g->lev.resize(nlevels);
  for (int l = 0; l < nlevels; ++l) {
    Lvl& L = g->lev[l];
    L.N = sizes[l];
    L.Np = pad64(L.N);
    L.n = 0; L.M = 0; L.h = 0.0;
  }
  *out = g;
  return FMG_OK;
}

// The interpolation I from level fine_level - 1 to fine_level of an algebraic
// grid (nfine x ncoarse, compressed rows or columns): prolongate xf += I xc,
// restrict rc = I^T rf (multigrid.lisp:202-252).  Rows of constrained fine
// unknowns and columns of constrained coarse ones are empty, as in Femlisp's
// constrained interpolation.
int fmg_set_interpolation(fmg_grid* g, int fine_level, int layout, const int* start, const int* index,
                          const double* values, long nfine, long ncoarse) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !start) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  if (!g->algebraic) return set_err(c, FMG_ERR_UNSUPPORTED, "interpolations are built in on structured grids");
  if (fine_level <= g->base || fine_level > g->top) return set_err(c, FMG_ERR_ARG, "level %d has no level below", fine_level);
  if (layout != FMG_CSR && layout != FMG_CCS) return set_err(c, FMG_ERR_ARG, "unknown matrix layout %d", layout);
  Lvl& F = g->lev[fine_level];
  if (nfine != F.N || ncoarse != g->lev[fine_level - 1].N)
    return set_err(c, FMG_ERR_ARG, "interpolation to level %d is %lld x %lld, got %ld x %ld", fine_level, F.N,
                   g->lev[fine_level - 1].N, nfine, ncoarse);
  int rc;
  FMG_CK(c, cudaSetDevice(c->device));
  if ((rc = ensure_buffers(g))) return rc;
  std::vector<long long> rs, rst;
  std::vector<int> ci, cit;
  std::vector<double> cv, cvt;
  std::string err;
  if (!host_csr(nfine, ncoarse, layout, start, index, values, rs, ci, cv, err) ||
      !host_csr(ncoarse, nfine, layout == FMG_CSR ? FMG_CCS : FMG_CSR, start, index, values, rst, cit, cvt, err))
    return set_err(c, FMG_ERR_ARG, "%s", err.c_str());
  if ((rc = upload_csr(g, F.cp, rs, ci, cv)) || (rc = upload_csr(g, F.cpt, rst, cit, cvt))) return rc;
  g->assembled = false;
  if ((int)g->haveP.size() != g->top + 1) g->haveP.assign(g->top + 1, 0);
  g->haveP[fine_level] = 1;
  return hierarchy_complete(g) ? finish_levels(g) : FMG_OK;
}

static void mixed_vec_delete(MixedVec* m);

static void grid_release(fmg_grid* g) {
  fmg_ctx* c = g->ctx;
  cudaStreamSynchronize(c->stream);
  for (void* p : g->allocs) cudaFree(p);
  if (g->mx && g->mx->host) cudaFreeHost(g->mx->host);
  if (g->mx)
    for (auto& e : g->mx->graphs) cudaGraphExecDestroy(e.exec);
  delete g->mx;
  mixed_vec_delete(g->mxv);
  delete g;
  c->grids -= 1;
  if (c->closed && c->grids == 0) ctx_release(c);
}

// Releases the grid; if vectors of it are still alive the release happens
// when the last of them is destroyed.
int fmg_grid_destroy(fmg_grid* g) {
  if (!g || g->destroyed) return FMG_ERR_ARG;
  g->destroyed = true;
  if (g->vecs == 0) grid_release(g);
  return FMG_OK;
}

long fmg_grid_nnodes(const fmg_grid* g, int level) {
  if (!g || level < 0 || level > g->top) return -1;
  return (long)g->lev[level].N;
}

int fmg_grid_nslots(const fmg_grid* g) { return g ? g->nslots : -1; }

int fmg_set_coefficient(fmg_grid* g, int kind, const double* host, long n) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (g && g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on an algebraic grid", __func__);
  if (!g || !host) return FMG_ERR_ARG;
  long long ncell = 1;
  for (int k = 0; k < g->dim; ++k) ncell *= g->lev[g->top].n;
  switch (kind) {
    case FMG_K_CONST:
      if (n != 1) return set_err(g->ctx, FMG_ERR_ARG, "K_CONST wants 1 value");
      g->kkind = kind; g->kconst = host[0]; break;
    case FMG_K_CELL: {  // straight to the device (read during the call only)
      if (n != ncell) return set_err(g->ctx, FMG_ERR_ARG, "K_CELL wants %lld values, got %ld", ncell, n);
      int rc;
      if (!g->kcell_d && (rc = dalloc(g, &g->kcell_d, ncell))) return rc;
      FMG_CK(g->ctx, cudaMemcpyAsync(g->kcell_d, host, ncell * sizeof(double), cudaMemcpyHostToDevice, g->ctx->stream));
      FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
      g->kkind = kind;
      break;
    }
    case FMG_F_CONST:
      if (n != 1) return set_err(g->ctx, FMG_ERR_ARG, "F_CONST wants 1 value");
      g->fkind = kind; g->fconst = host[0]; break;
    case FMG_LAMBDA_MU_CELL: {  // elasticity: lambda = mu = E per top-level cell
      if (g->nc != 3) return set_err(g->ctx, FMG_ERR_ARG, "LAMBDA_MU_CELL is for 3-component grids");
      if (n != ncell) return set_err(g->ctx, FMG_ERR_ARG, "LAMBDA_MU_CELL wants %lld values, got %ld", ncell, n);
      int rc;
      if (!g->kcell_d && (rc = dalloc(g, &g->kcell_d, ncell))) return rc;
      FMG_CK(g->ctx, cudaMemcpyAsync(g->kcell_d, host, ncell * sizeof(double), cudaMemcpyHostToDevice, g->ctx->stream));
      FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
      g->kkind = FMG_K_CELL;
      break;
    }
    case FMG_F_VEC:
      if (g->nc != 3 || n != 3) return set_err(g->ctx, FMG_ERR_ARG, "F_VEC wants 3 values on a 3-component grid");
      g->fkind = kind;
      for (int k = 0; k < 3; ++k) g->fvec[k] = host[k];
      break;
    case FMG_F_IP: {
      if (g->nc != 1) return set_err(g->ctx, FMG_ERR_ARG, "F_IP is for scalar grids");
      if (n != ncell * g->nq) return set_err(g->ctx, FMG_ERR_ARG, "F_IP wants %lld values", ncell * g->nq);
      int rc;
      if (!g->fip_d && (rc = dalloc(g, &g->fip_d, ncell * g->nq))) return rc;
      FMG_CK(g->ctx, cudaMemcpyAsync(g->fip_d, host, ncell * g->nq * sizeof(double), cudaMemcpyHostToDevice,
                                     g->ctx->stream));
      FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
      g->fkind = kind;
      break;
    }
    default: return set_err(g->ctx, FMG_ERR_ARG, "unknown coefficient kind %d", kind);
  }
  g->assembled = false;
  return FMG_OK;
}

// device buffers of a hierarchy, allocated by the first assembly and reused
// by later ones (only the coefficient data change between assemblies)
// the device buffers of an algebraic hierarchy (level vectors, coarse LU,
// solver vectors); the matrices and interpolations arrive separately
static int ensure_buffers_alg(fmg_grid* g) {
  int rc;
  const Lvl& T = g->lev[g->top];
  if ((rc = dalloc(g, &g->rhs, T.Np))) return rc;
  const long long nb = g->lev[g->base].N;
  if (nb > 1024)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "base level has %lld unknowns; the dense coarse solve takes <= 1024",
                   nb);
  g->nbase = (int)nb;
  const long long nn = nb * nb;
  if ((rc = dalloc(g, &g->lu, nn)) || (rc = dalloc(g, &g->lux, nn)) || (rc = dalloc(g, &g->ainvT, nn)) ||
      (rc = dalloc(g, (double**)&g->piv, nb)))
    return rc;
  for (int l = g->base; l < g->top; ++l) {
    Lvl& L = g->lev[l];
    if ((rc = dalloc(g, &L.sol[0], L.Np)) || (rc = dalloc(g, &L.sol[1], L.Np)) || (rc = dalloc(g, &L.rhs, L.Np)) ||
        (rc = dalloc(g, &L.res, L.Np)))
      return rc;
  }
  if ((rc = dalloc(g, &g->scal, S_COUNT))) return rc;
  if ((rc = dalloc(g, &g->part, nchunks(T.Np) + 1))) return rc;
  if ((rc = dalloc(g, (double**)&g->counter, 1))) return rc;
  double** tv[] = {&g->p, &g->a, &g->w, &g->w2, &g->q, &g->r, &g->xs, &g->xs2};
  for (double** v : tv)
    if ((rc = dalloc(g, v, T.Np))) return rc;
  g->assembled_once = true;
  return FMG_OK;
}

static int ensure_buffers(fmg_grid* g) {
  if (g->assembled_once) return FMG_OK;
  if (g->algebraic) return ensure_buffers_alg(g);
  int rc;
  const Lvl& T = g->lev[g->top];
  long long ncell_top = 1, ncell_kq = 0;
  for (int k = 0; k < g->dim; ++k) ncell_top *= T.n;
  if (g->top > g->base) ncell_kq = ncell_top >> g->dim;  // largest coarse level
  std::vector<double> xiv(g->xi_h, g->xi_h + g->np);
  if ((rc = upload(g, &g->xi_d, xiv))) return rc;
  const int nc = g->nc;
  if ((rc = dalloc(g, &g->rhs, T.Np * nc))) return rc;
  if ((rc = dalloc(g, &g->kq, ncell_kq * g->nq))) return rc;
  for (int l = g->top; l >= g->base; --l) {
    Lvl& L = g->lev[l];
    std::vector<double> C, Kbar, Phi;
    int nl, nq;
    make_tables(g->dim, g->order, L.h, C, Kbar, Phi, &nl, &nq);
    if (nc == 3) make_elastic_tables(g->dim, g->order, L.h, C, Kbar);  // Kbar := Ebar, C := Etab
    if ((rc = upload(g, &L.Kbar, Kbar)) || (rc = upload(g, &L.Ctab, C)) || (rc = upload(g, &L.Phi, Phi)))
      return rc;
    L.Kbar_h = Kbar;
    L.Ctab_h = C;
    if ((rc = dalloc(g, &L.A, (long long)g->nslots * nc * nc * L.Np))) return rc;
  }
  const Lvl& B = g->lev[g->base];
  const long long nb = B.N * nc;
  if ((nc == 1 && nb > 1024) || nb > 2048)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED,
                   "base level has %lld unknowns; the dense coarse solve takes <= %d", nb, nc == 1 ? 1024 : 2048);
  g->nbase = (int)nb;
  const long long nn = nb * nb;
  if ((rc = dalloc(g, &g->lu, nn)) || (rc = dalloc(g, &g->lux, nn)) || (rc = dalloc(g, &g->ainvT, nn)) ||
      (rc = dalloc(g, (double**)&g->piv, nb)))
    return rc;
  for (int l = g->base; l < g->top; ++l) {
    Lvl& L = g->lev[l];
    const long long nv = L.Np * nc;
    if ((rc = dalloc(g, &L.sol[0], nv)) || (rc = dalloc(g, &L.sol[1], nv)) || (rc = dalloc(g, &L.rhs, nv)) ||
        (rc = dalloc(g, &L.res, nv)))
      return rc;
  }
  if ((rc = dalloc(g, &g->scal, S_COUNT))) return rc;
  // reduction partials: the longest top-level vector (the mixed solve's padded ones in 3D)
  long long nred = T.Np * nc;
  if (g->dim == 3) nred = std::max(nred, padded_lay((int)T.M, g->dmask).total);
  if ((rc = dalloc(g, &g->part, nchunks(nred) + 1))) return rc;
  if ((rc = dalloc(g, (double**)&g->counter, 1))) return rc;
  double** tv[] = {&g->p, &g->a, &g->w, &g->w2, &g->q, &g->r, &g->xs, &g->xs2};
  for (double** v : tv)
    if ((rc = dalloc(g, v, T.Np * nc))) return rc;
  g->assembled_once = true;
  return FMG_OK;
}

int fmg_assemble(fmg_grid* g) { return fmg_assemble_levels(g, FMG_ASSEMBLE_REDISCRETIZE); }

static int finish_levels(fmg_grid* g);
static AsmArgs asm_args(fmg_grid* g, int l, bool sample);
static int ensure_top(fmg_grid* g);

int fmg_assemble_levels(fmg_grid* g, int mode) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g) return FMG_ERR_ARG;
  if (g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on an algebraic grid", __func__);
  fmg_ctx* c = g->ctx;
  if (mode != FMG_ASSEMBLE_REDISCRETIZE && mode != FMG_ASSEMBLE_GALERKIN)
    return set_err(c, FMG_ERR_ARG, "unknown assembly mode %d", mode);
  cudaStream_t st = c->stream;
  int rc;
  FMG_CK(c, cudaSetDevice(c->device));
  g->assembled = false;
  if ((rc = ensure_buffers(g))) return rc;
  const long long n_top = g->lev[g->top].n;
  for (int l = g->top; l >= g->base; --l) {
    Lvl& L = g->lev[l];
    if (mode == FMG_ASSEMBLE_GALERKIN && l < g->top) {  // I^T A_{l+1} I (geomg.lisp:122-123)
      launch_galerkin(view(g, l + 1), view(g, l), L.A, st);
      if ((rc = launched(c, "galerkin"))) return rc;
      continue;
    }
    long long ncells = 1;
    for (int k = 0; k < g->dim; ++k) ncells *= L.n;
    const bool sample = (l < g->top && g->kkind == FMG_K_CELL);
    if (sample) {
      launch_sample_kq(g->dim, ncells, L.n, n_top, std::ldexp(1.0, g->top - l), g->np, g->xi_d, g->kcell_d, g->kq,
                       st);
      if ((rc = launched(c, "sample_kq"))) return rc;
    }
    AsmArgs a = asm_args(g, l, sample);
    // the top level's matrix of the unrolled Q1 path waits for its first
    // use (the mixed solve applies that level from the cell coefficients and
    // never reads it); its rhs is formed now
    // (not where the top level is the base: the coarse LU reads it right away)
    const bool defer = l == g->top && l > g->base && mode == FMG_ASSEMBLE_REDISCRETIZE &&
                       assemble_splits(g->dim, g->order, g->nc, a);
    if (defer) a.A = nullptr;
    launch_assemble(g->dim, g->order, a, L.Kbar_h.data(), L.Ctab_h.data(), st);
    if ((rc = launched(c, "assemble"))) return rc;
    if (l == g->top) g->top_deferred = defer;
  }
  g->have.assign(g->top + 1, 1);
  g->uploaded = false;
  return finish_levels(g);
}

// The arguments of level l's assembly (the rhs on the top level; sample:
// the coarse level's coefficient samples are in g->kq).
static AsmArgs asm_args(fmg_grid* g, int l, bool sample) {
  const Lvl& L = g->lev[l];
  AsmArgs a;
  a.N = L.N; a.Np = L.Np; a.M = L.M; a.n = L.n;
  a.dmask = g->dmask; a.nl = g->nl; a.nq = g->nq;
  a.A = L.A;
  a.rhs = (l == g->top) ? g->rhs : nullptr;
  a.Kbar = L.Kbar; a.Ctab = L.Ctab; a.Phi = L.Phi;
  a.kcell = (l == g->top && g->kkind == FMG_K_CELL) ? g->kcell_d : nullptr;
  a.kq = sample ? g->kq : nullptr;
  a.fip = g->fkind == FMG_F_IP ? g->fip_d : nullptr;
  a.kconst = g->kconst; a.fconst = g->fconst;
  a.nc = g->nc;
  a.fvec_on = g->fkind == FMG_F_VEC ? 1 : 0;
  for (int k = 0; k < 3; ++k) a.fvec[k] = g->fvec[k];
  return a;
}

// The top level's matrix where its assembly was deferred (see above).
static int ensure_top(fmg_grid* g) {
  if (!g->top_deferred) return FMG_OK;
  Lvl& L = g->lev[g->top];
  AsmArgs a = asm_args(g, g->top, false);
  a.rhs = nullptr;
  launch_assemble(g->dim, g->order, a, L.Kbar_h.data(), L.Ctab_h.data(), g->ctx->stream);
  g->top_deferred = false;
  return launched(g->ctx, "assemble (top level)");
}

// The coarse LU and the multigrid state of a hierarchy whose level matrices
// are all in place (assembled, formed, or uploaded).
static int finish_levels(fmg_grid* g) {
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  int rc;
  // dense LU of the base level and its explicit inverse
  const Lvl& B = g->lev[g->base];
  const long long nb = B.N * g->nc;
  FMG_CK(c, cudaMemsetAsync(g->lu, 0, (size_t)nb * nb * sizeof(double), st));
  launch_densify(view(g, g->base), g->lu, st);
  launch_lu(g->lu, (int)nb, g->piv, g->lux, g->ainvT, st);
  if ((rc = launched(c, "coarse LU"))) return rc;
  // multigrid state
  const int nlev = g->top + 1;
  g->solp.assign(nlev, nullptr); g->sparep.assign(nlev, nullptr);
  g->rhsp.assign(nlev, nullptr); g->resp.assign(nlev, nullptr);
  g->rp.assign(nlev, 0);
  for (int l = g->base; l < g->top; ++l) {
    g->solp[l] = g->lev[l].sol[0]; g->sparep[l] = g->lev[l].sol[1];
    g->rhsp[l] = g->lev[l].rhs; g->resp[l] = g->lev[l].res;
  }
  FMG_CK(c, cudaStreamSynchronize(st));
  g->assembled = true;
  g->epoch += 1;
  return FMG_OK;
}

// A level matrix given as compressed rows (CSR) or columns (CCS, the form of
// sparse-matrix->ccs, sparselu.lisp:226-263) over the grid's numbering
// (node-major, lexicographic nodes, x fastest), scattered into the stencil-slot
// storage on the host and copied to the device in one piece.
// Compressed rows (columns ascending, duplicates summed, exact zeros dropped)
// of an nrows x ncols matrix given as compressed rows or columns; false (and
// the message) on a malformed input.
static bool host_csr(long nrows, long ncols, int layout, const int* start, const int* index, const double* values,
                     std::vector<long long>& rs, std::vector<int>& ci, std::vector<double>& cv, std::string& err) {
  const long nlines = layout == FMG_CSR ? nrows : ncols, nother = layout == FMG_CSR ? ncols : nrows;
  if (start[0] != 0) { err = "start[0] must be 0"; return false; }
  std::vector<std::vector<std::pair<int, double>>> rows((size_t)nrows);
  for (long a = 0; a < nlines; ++a) {
    if (start[a + 1] < start[a]) { err = "start decreases at " + std::to_string(a); return false; }
    for (int e = start[a]; e < start[a + 1]; ++e) {
      const long b = index[e];
      if (b < 0 || b >= nother) { err = "index out of range at entry " + std::to_string(e); return false; }
      if (values[e] == 0.0) continue;
      const long row = layout == FMG_CSR ? a : b, col = layout == FMG_CSR ? b : a;
      rows[(size_t)row].push_back({(int)col, values[e]});
    }
  }
  rs.assign((size_t)nrows + 1, 0);
  ci.clear();
  cv.clear();
  for (long i = 0; i < nrows; ++i) {
    auto& r = rows[(size_t)i];
    std::stable_sort(r.begin(), r.end(), [](const std::pair<int, double>& x, const std::pair<int, double>& y) {
      return x.first < y.first;
    });
    for (size_t k = 0; k < r.size(); ++k) {
      if (!ci.empty() && (long long)ci.size() > rs[(size_t)i] && ci.back() == r[k].first) cv.back() += r[k].second;
      else { ci.push_back(r[k].first); cv.push_back(r[k].second); }
    }
    rs[(size_t)i + 1] = (long long)ci.size();
  }
  return true;
}

static int upload_csr(fmg_grid* g, Lvl::Csr& d, const std::vector<long long>& rs, const std::vector<int>& ci,
                      const std::vector<double>& cv) {
  dfree(g, d.start); dfree(g, d.index); dfree(g, d.value);
  d = Lvl::Csr{};
  int rc;
  if ((rc = dalloc(g, (double**)&d.start, (long long)rs.size())) ||
      (rc = dalloc(g, (double**)&d.index, ((long long)ci.size() + 1) / 2)) ||
      (rc = dalloc(g, &d.value, (long long)cv.size())))
    return rc;
  cudaStream_t st = g->ctx->stream;
  FMG_CK(g->ctx, cudaMemcpyAsync(d.start, rs.data(), rs.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
  if (!ci.empty()) {
    FMG_CK(g->ctx, cudaMemcpyAsync(d.index, ci.data(), ci.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    FMG_CK(g->ctx, cudaMemcpyAsync(d.value, cv.data(), cv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  FMG_CK(g->ctx, cudaStreamSynchronize(st));
  return FMG_OK;
}

// every level matrix in place and, on an algebraic grid, every interpolation
static bool hierarchy_complete(const fmg_grid* g) {
  for (int m = g->base; m <= g->top; ++m) {
    if ((int)g->have.size() <= m || !g->have[m]) return false;
    if (g->algebraic && m > g->base && ((int)g->haveP.size() <= m || !g->haveP[m])) return false;
  }
  return true;
}

// Greedy colouring of the graph of a level matrix (i ~ j when a_ij or a_ji is
// stored, i != j): rows in ascending order take the smallest colour none of
// their coloured neighbours has.  Rows of one colour then couple to none of
// each other, so an SOR sweep over the colours in order, the rows of a
// colour in any order, is Femlisp's <sor> with the rows ordered by colour
// (the :compare ordering of linit.lisp:288-323).  Returns the rows grouped
// by colour and the colour offsets.
static void greedy_colouring(long n, const std::vector<long long>& rs, const std::vector<int>& ci,
                             std::vector<int>& rows, std::vector<long long>& off) {
  std::vector<long long> ts((size_t)n + 1, 0);  // the transpose's structure
  for (long i = 0; i < n; ++i)
    for (long long e = rs[(size_t)i]; e < rs[(size_t)i + 1]; ++e) ts[(size_t)ci[(size_t)e] + 1] += 1;
  for (long i = 0; i < n; ++i) ts[(size_t)i + 1] += ts[(size_t)i];
  std::vector<int> ti((size_t)ts[(size_t)n]);
  std::vector<long long> fill(ts.begin(), ts.end() - 1);
  for (long i = 0; i < n; ++i)
    for (long long e = rs[(size_t)i]; e < rs[(size_t)i + 1]; ++e) ti[(size_t)fill[(size_t)ci[(size_t)e]]++] = (int)i;
  std::vector<int> col((size_t)n, -1), mark;
  int ncol = 0;
  for (long i = 0; i < n; ++i) {
    auto see = [&](int j) {
      if (j == i || col[(size_t)j] < 0) return;
      if ((size_t)col[(size_t)j] >= mark.size()) mark.resize((size_t)col[(size_t)j] + 1, -1);
      mark[(size_t)col[(size_t)j]] = (int)i;
    };
    for (long long e = rs[(size_t)i]; e < rs[(size_t)i + 1]; ++e) see(ci[(size_t)e]);
    for (long long e = ts[(size_t)i]; e < ts[(size_t)i + 1]; ++e) see(ti[(size_t)e]);
    int c = 0;
    while ((size_t)c < mark.size() && mark[(size_t)c] == i) ++c;
    col[(size_t)i] = c;
    ncol = std::max(ncol, c + 1);
  }
  off.assign((size_t)ncol + 1, 0);
  for (long i = 0; i < n; ++i) off[(size_t)col[(size_t)i] + 1] += 1;
  for (int c = 0; c < ncol; ++c) off[(size_t)c + 1] += off[(size_t)c];
  rows.assign((size_t)n, 0);
  std::vector<long long> pos(off.begin(), off.end() - 1);
  for (long i = 0; i < n; ++i) rows[(size_t)pos[(size_t)col[(size_t)i]]++] = (int)i;
}

// fmg_set_matrix on an algebraic grid: the level matrix as compressed rows,
// its diagonal and the colouring of its graph
static int set_matrix_alg(fmg_grid* g, int level, int layout, const int* start, const int* index,
                          const double* values, long n) {
  Lvl& L = g->lev[level];
  if (n != L.N) return set_err(g->ctx, FMG_ERR_ARG, "level %d has %lld rows, got %ld", level, L.N, n);
  std::vector<long long> rs;
  std::vector<int> ci;
  std::vector<double> cv;
  std::string err;
  if (!host_csr(n, n, layout, start, index, values, rs, ci, cv, err))
    return set_err(g->ctx, FMG_ERR_ARG, "%s", err.c_str());
  std::vector<double> dg((size_t)n, 0.0);
  for (long i = 0; i < n; ++i)
    for (long long e = rs[(size_t)i]; e < rs[(size_t)i + 1]; ++e)
      if (ci[(size_t)e] == i) dg[(size_t)i] = cv[(size_t)e];
  int rc;
  if ((rc = upload_csr(g, L.ca, rs, ci, cv))) return rc;
  dfree(g, L.diag);
  L.diag = nullptr;
  if ((rc = upload(g, &L.diag, dg))) return rc;
  std::vector<int> crow;
  greedy_colouring(n, rs, ci, crow, L.coff);
  dfree(g, L.crow);
  L.crow = nullptr;
  if ((rc = dalloc(g, (double**)&L.crow, ((long long)n + 1) / 2))) return rc;
  FMG_CK(g->ctx, cudaMemcpyAsync(L.crow, crow.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, g->ctx->stream));
  FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
  g->assembled = false;
  if ((int)g->have.size() != g->top + 1) g->have.assign(g->top + 1, 0);
  g->have[level] = 1;
  g->uploaded = true;
  return hierarchy_complete(g) ? finish_levels(g) : FMG_OK;
}

int fmg_set_matrix(fmg_grid* g, int level, int layout, const int* start, const int* index, const double* values,
                   long n) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !start || (!index && n > 0) || (!values && n > 0)) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  if (level < g->base || level > g->top) return set_err(c, FMG_ERR_ARG, "level %d out of range", level);
  if (layout != FMG_CSR && layout != FMG_CCS) return set_err(c, FMG_ERR_ARG, "unknown matrix layout %d", layout);
  const Lvl& L = g->lev[level];
  const int nc = g->nc, dim = g->dim, ord = g->order, w = 2 * ord + 1;
  if (n != L.N * nc) return set_err(c, FMG_ERR_ARG, "level %d has %lld rows, got %ld", level, L.N * nc, n);
  if (start[0] != 0) return set_err(c, FMG_ERR_ARG, "start[0] must be 0");
  for (long a = 0; a < n; ++a)
    if (start[a + 1] < start[a]) return set_err(c, FMG_ERR_ARG, "start decreases at %ld", a);
  int rc;
  FMG_CK(c, cudaSetDevice(c->device));
  if ((rc = ensure_buffers(g))) return rc;
  if (g->algebraic) return set_matrix_alg(g, level, layout, start, index, values, n);
  const long long M = L.M, Np = L.Np;
  std::vector<double> H((size_t)g->nslots * nc * nc * Np, 0.0);
  for (long a = 0; a < n; ++a) {
    for (int e = start[a]; e < start[a + 1]; ++e) {
      const long b = index[e];
      if (b < 0 || b >= n) return set_err(c, FMG_ERR_ARG, "index %ld out of range at entry %d", b, e);
      const long row = layout == FMG_CSR ? a : b, col = layout == FMG_CSR ? b : a;
      const long long i = row / nc, j = col / nc;
      const int k = (int)(row % nc), l = (int)(col % nc);
      long long ti = i, tj = j;
      int s = 0, wk = 1;
      bool in = true;
      for (int d = 0; d < dim; ++d) {
        const long long o = tj % M - ti % M;
        if (o < -ord || o > ord) in = false;
        s += (int)(o + ord) * wk;
        wk *= w;
        ti /= M; tj /= M;
      }
      const long long p = !in ? -1 : ord == 2 ? q2_slot_pos(dim, M, i, s, nc == 1) : i;
      if (p < 0) {
        if (values[e] != 0.0)
          return set_err(c, FMG_ERR_ARG, "entry (%ld,%ld) lies outside the Q%d stencil of the level", row, col, ord);
        continue;
      }
      H[((size_t)s * nc * nc + (size_t)k * nc + l) * Np + p] += values[e];
    }
  }
  g->assembled = false;
  FMG_CK(c, cudaMemcpyAsync(L.A, H.data(), H.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  if ((int)g->have.size() != g->top + 1) g->have.assign(g->top + 1, 0);
  g->have[level] = 1;
  g->uploaded = true;
  if (level == g->top) g->top_deferred = false;
  return hierarchy_complete(g) ? finish_levels(g) : FMG_OK;  // complete with the last level
}

int fmg_set_rhs(fmg_grid* g, const double* host, long n) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !host) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  const Lvl& T = g->lev[g->top];
  if (n != T.N * g->nc) return set_err(c, FMG_ERR_ARG, "rhs wants %lld values, got %ld", T.N * g->nc, n);
  int rc;
  FMG_CK(c, cudaSetDevice(c->device));
  if ((rc = ensure_buffers(g))) return rc;
  FMG_CK(c, cudaMemcpyAsync(g->rhs, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  return FMG_OK;
}

int fmg_get_matrix(fmg_grid* g, int level, double* host) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !host) return FMG_ERR_ARG;
  if (g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on an algebraic grid", __func__);
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  if (level < g->base || level > g->top) return set_err(g->ctx, FMG_ERR_ARG, "level %d out of range", level);
  if (level == g->top) FMG_RC(ensure_top(g));
  const Lvl& L = g->lev[level];
  const size_t rows = (size_t)g->nslots * g->nc * g->nc;
  FMG_CK(g->ctx, cudaMemcpy2DAsync(host, L.N * sizeof(double), L.A, L.Np * sizeof(double), L.N * sizeof(double),
                                   rows, cudaMemcpyDeviceToHost, g->ctx->stream));
  FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
  if (g->order == 2) {  // sliced storage -> one entry per node and slot, structural zeros included
    std::vector<double> raw((size_t)L.N);
    const int nblk = g->nc * g->nc;
    for (size_t row = 0; row < rows; ++row) {
      double* h = host + row * L.N;
      std::copy(h, h + L.N, raw.begin());
      const int s = (int)(row / nblk);
      for (long long i = 0; i < L.N; ++i) {
        const long long p = q2_slot_pos(g->dim, L.M, i, s, g->nc == 1);
        h[i] = p >= 0 ? raw[(size_t)p] : 0.0;
      }
    }
  }
  return FMG_OK;
}

int fmg_get_rhs(fmg_grid* g, double* host) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !host) return FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  const Lvl& T = g->lev[g->top];
  FMG_CK(g->ctx, cudaMemcpyAsync(host, g->rhs, T.N * g->nc * sizeof(double), cudaMemcpyDeviceToHost,
                                 g->ctx->stream));
  FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
  return FMG_OK;
}

int fmg_set_node_damping(fmg_grid* g, int level, const double* host, long n) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g) return FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  if (level <= g->base || level > g->top) return set_err(g->ctx, FMG_ERR_ARG, "level %d has no smoother", level);
  Lvl& L = g->lev[level];
  g->learned = false;  // damping set by hand: no judge
  if (!host) {
    if (L.omega) { cudaStreamSynchronize(g->ctx->stream); dfree(g, L.omega); }
    L.omega = nullptr;
    return FMG_OK;
  }
  if (n != L.N) return set_err(g->ctx, FMG_ERR_ARG, "damping wants %lld values", L.N);
  int rc;
  if (!L.omega && (rc = dalloc(g, &L.omega, L.Np))) return rc;
  FMG_CK(g->ctx, cudaMemcpyAsync(L.omega, host, L.N * sizeof(double), cudaMemcpyHostToDevice, g->ctx->stream));
  return FMG_OK;
}

int fmg_vec_create(fmg_grid* g, int level, fmg_vec** out) {
  if (!g || !out || level < 0 || level > g->top) return FMG_ERR_ARG;
  fmg_vec* v = new (std::nothrow) fmg_vec();
  if (!v) return FMG_ERR_NOMEM;
  v->g = g; v->level = level; v->n = g->lev[level].N * g->nc * g->nb;
  g->vecs += 1;
  const long long np = g->nb > 1 ? g->lev[level].Np * g->nb : pad64(v->n);  // a batch: problems Np apart
  cudaError_t e = cudaMalloc((void**)&v->d, np * sizeof(double));
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete v;
    g->vecs -= 1;
    return set_err(g->ctx, FMG_ERR_NOMEM, "vector allocation failed");
  }
  FMG_CK(g->ctx, cudaMemsetAsync(v->d, 0, np * sizeof(double), g->ctx->stream));
  *out = v;
  return FMG_OK;
}

int fmg_vec_destroy(fmg_vec* v) {
  if (!v) return FMG_ERR_ARG;
  fmg_grid* g = v->g;
  cudaStreamSynchronize(g->ctx->stream);
  cudaFree(v->d);
  delete v;
  g->vecs -= 1;
  if (g->destroyed && g->vecs == 0) grid_release(g);
  return FMG_OK;
}

int fmg_vec_set(fmg_vec* v, const double* host, long n) {
  if (!v || !host || n != v->n) return FMG_ERR_ARG;
  if (v->g->nb > 1) {  // host: the problems one after another; device: Np apart
    const Lvl& L = v->g->lev[v->level];
    FMG_CK(v->g->ctx, cudaMemcpy2DAsync(v->d, L.Np * sizeof(double), host, L.N * sizeof(double),
                                        L.N * sizeof(double), v->g->nb, cudaMemcpyHostToDevice, v->g->ctx->stream));
    FMG_CK(v->g->ctx, cudaStreamSynchronize(v->g->ctx->stream));
    return FMG_OK;
  }
  FMG_CK(v->g->ctx, cudaMemcpyAsync(v->d, host, n * sizeof(double), cudaMemcpyHostToDevice, v->g->ctx->stream));
  FMG_CK(v->g->ctx, cudaStreamSynchronize(v->g->ctx->stream));
  return FMG_OK;
}

int fmg_vec_get(const fmg_vec* v, double* host, long n) {
  if (!v || !host || n != v->n) return FMG_ERR_ARG;
  if (v->g->nb > 1) {
    const Lvl& L = v->g->lev[v->level];
    FMG_CK(v->g->ctx, cudaMemcpy2DAsync(host, L.N * sizeof(double), v->d, L.Np * sizeof(double),
                                        L.N * sizeof(double), v->g->nb, cudaMemcpyDeviceToHost, v->g->ctx->stream));
    FMG_CK(v->g->ctx, cudaStreamSynchronize(v->g->ctx->stream));
    return FMG_OK;
  }
  FMG_CK(v->g->ctx, cudaMemcpyAsync(host, v->d, n * sizeof(double), cudaMemcpyDeviceToHost, v->g->ctx->stream));
  FMG_CK(v->g->ctx, cudaStreamSynchronize(v->g->ctx->stream));
  return FMG_OK;
}

// the device length of a vector (a batch's problems sit Np apart)
static long long vec_len(const fmg_vec* v) {
  return v->g->nb > 1 ? v->g->lev[v->level].Np * v->g->nb : v->n;
}

int fmg_vec_fill(fmg_vec* v, double value) {
  if (!v) return FMG_ERR_ARG;
  launch_fill(v->d, vec_len(v), value, v->g->ctx->stream);
  return launched(v->g->ctx, "fill");
}

int fmg_copy(const fmg_vec* x, fmg_vec* y) {
  if (!x || !y || x->n != y->n) return FMG_ERR_ARG;
  launch_copy(x->d, y->d, vec_len(x), x->g->ctx->stream);
  return launched(x->g->ctx, "copy");
}

int fmg_axpy(double alpha, const fmg_vec* x, fmg_vec* y) {
  if (!x || !y || x->n != y->n) return FMG_ERR_ARG;
  launch_axpy(alpha, nullptr, -1, x->d, y->d, vec_len(x), x->g->ctx->stream);
  return launched(x->g->ctx, "axpy");
}

int fmg_dot(const fmg_vec* x, const fmg_vec* y, double* out) {
  if (!x || !y || !out || x->n != y->n) return FMG_ERR_ARG;
  fmg_grid* g = x->g;
  if (g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "fmg_dot: not on a batch");
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  launch_dot(x->d, y->d, x->n, reducer(g, EPI_STORE, S_DOT), g->ctx->stream);
  int rc = launched(g->ctx, "dot");
  if (rc) return rc;
  if ((rc = read_scalars(g))) return rc;
  *out = g->ctx->host_scal[S_DOT];
  return FMG_OK;
}

int fmg_l2_norm(const fmg_vec* x, double* out) {
  int rc = fmg_dot(x, x, out);
  if (rc) return rc;
  *out = std::sqrt(*out);
  return FMG_OK;
}

int fmg_matvec(fmg_grid* g, int level, const fmg_vec* x, fmg_vec* y) {
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, level) || vec_check(y, g, level) || x == y) return FMG_ERR_ARG;
  if (level == g->top) FMG_RC(ensure_top(g));
  launch_spmv(view(g, level), x->d, nullptr, y->d, nullptr, nullptr, g->ctx->stream);
  return launched(g->ctx, "matvec");
}

int fmg_residual(fmg_grid* g, int level, const fmg_vec* x, const fmg_vec* b, fmg_vec* r) {
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, level) || vec_check(b, g, level) || vec_check(r, g, level) || x == r) return FMG_ERR_ARG;
  if (level == g->top) FMG_RC(ensure_top(g));
  launch_spmv(view(g, level), x->d, b->d, r->d, nullptr, nullptr, g->ctx->stream);
  return launched(g->ctx, "residual");
}

int fmg_restrict(fmg_grid* g, int fine_level, const fmg_vec* rf, fmg_vec* rc) {
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (fine_level <= g->base || vec_check(rf, g, fine_level) || vec_check(rc, g, fine_level - 1)) return FMG_ERR_ARG;
  const Lvl& C = g->lev[fine_level - 1];
  // the coarse rhs/sol side outputs of the fused kernel go to level scratch
  launch_restrict(view(g, fine_level), view(g, fine_level - 1), rf->d, rc->d, C.rhs, C.sol[1], g->ctx->stream);
  return launched(g->ctx, "restrict");
}

int fmg_prolongate(fmg_grid* g, int coarse_level, const fmg_vec* xc, fmg_vec* xf) {
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (coarse_level < g->base || coarse_level >= g->top || vec_check(xc, g, coarse_level) ||
      vec_check(xf, g, coarse_level + 1))
    return FMG_ERR_ARG;
  launch_prolong(view(g, coarse_level), view(g, coarse_level + 1), xc->d, xf->d, g->ctx->stream);
  return launched(g->ctx, "prolongate");
}

int fmg_jacobi(fmg_grid* g, int level, double damp, fmg_vec* x, fmg_vec* r) {
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, level) || vec_check(r, g, level)) return FMG_ERR_ARG;
  if (level == g->top) FMG_RC(ensure_top(g));
  launch_jacobi(view(g, level), damp, x->d, r->d, true, g->ctx->stream);
  return launched(g->ctx, "jacobi");
}

int fmg_sor(fmg_grid* g, int level, double omega, fmg_vec* x, const fmg_vec* b, fmg_vec* r) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (g && g->nc != 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "SOR: scalar grids");
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, level) || vec_check(b, g, level) || vec_check(r, g, level)) return FMG_ERR_ARG;
  if (level == g->top) FMG_RC(ensure_top(g));
  launch_sor(view(g, level), omega, x->d, b->d, r->d, g->ctx->stream);
  return launched(g->ctx, "sor");
}

int fmg_ssc(fmg_grid* g, int level, double omega, fmg_vec* x, const fmg_vec* b, fmg_vec* r) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (g->nc != 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "geometric SSC: scalar grids");
  if (vec_check(x, g, level) || vec_check(b, g, level) || vec_check(r, g, level) || x == b || x == r)
    return FMG_ERR_ARG;
  int rc = ssc_prepare(g, level);  // forms a deferred top level first
  if (rc) return rc;
  launch_ssc(view(g, level), omega, x->d, b->d, r->d, g->order == 2 ? g->sscF[level] : nullptr,
             g->order == 2 ? g->sscP[level] : nullptr, g->ctx->stream);
  return launched(g->ctx, "ssc");
}

int fmg_psc(fmg_grid* g, int level, double damp, fmg_vec* x, const fmg_vec* r) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (g && g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on an algebraic grid", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (g->nc != 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "geometric PSC: scalar grids");
  if (vec_check(x, g, level) || vec_check(r, g, level) || x == r) return FMG_ERR_ARG;
  int rc = ssc_prepare(g, level);  // forms a deferred top level first
  if (rc) return rc;
  if (level == g->top && g->order == 1) FMG_RC(ensure_top(g));
  launch_psc(view(g, level), damp, x->d, r->d, g->order == 2 ? g->sscF[level] : nullptr,
             g->order == 2 ? g->sscP[level] : nullptr, g->order == 2 ? g->sscC[level] : nullptr, g->ctx->stream);
  return launched(g->ctx, "psc");
}

int fmg_coarse_solve(fmg_grid* g, double damp, fmg_vec* x, fmg_vec* r) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, g->base) || vec_check(r, g, g->base)) return FMG_ERR_ARG;
  launch_coarse_solve(g->ainvT, g->nbase, damp, x->d, r->d, g->ctx->stream);
  return launched(g->ctx, "coarse solve");
}

int fmg_vcycle(fmg_grid* g, const fmg_solve_cfg* cfg, fmg_vec* x, fmg_vec* b, fmg_vec* r) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  FMG_RC(ensure_top(g));
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (vec_check(x, g, g->top) || vec_check(b, g, g->top) || vec_check(r, g, g->top) || x == b || x == r)
    return FMG_ERR_ARG;
  MG mg{g, *cfg, true, g->ctx->stream};
  double* xp = x->d;
  double* sp = g->xs;
  mg.iterate(&xp, &sp, b->d, r->d);
  if (xp != x->d) launch_copy(xp, x->d, x->n, g->ctx->stream);
  if (g->ssc_unprepared) return set_err(g->ctx, FMG_ERR_STATE, "SSC factors missing");
  return launched(g->ctx, "vcycle");
}

int fmg_solve(fmg_grid* g, const fmg_solve_cfg* cfg, fmg_vec* xv, double* hist, int hist_len, int* nsteps,
              int* status) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  FMG_RC(ensure_top(g));
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (vec_check(xv, g, g->top) || !nsteps || !status) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const fmg_solve_cfg& cf = *cfg;
  const LevelView T = view(g, g->top);
  const long long n = T.N * g->nc;
  const double* b = g->rhs;
  double* x = xv->d;
  double* xspare = g->xs2;
  MG mg{g, cf, false, st};
  double defnorm = 0.0, initial = -1.0, alpha = 0.0, prev = 0.0;
  bool rp = false, initialized = false;
  *status = 1;
  // the plain cycle judges learned cycles as in fmg_solve_mixed; on a revert
  // the node damping is hidden for the rest of this solve and restored after
  bool judge_active = g->learned && cf.smoother == FMG_JACOBI && cf.method != FMG_METHOD_CG;
  const int judged_from = cf.method == FMG_METHOD_MG ? 1 : 2;  // a CG run's first step may grow
  double win[3] = {0.0, 0.0, 0.0};
  std::vector<double*> hidden;
  // CG vectors start at zero (make-domain-vector-for)
  launch_fill(g->p, n, 0.0, st);
  for (int step = 0;; ++step) {
    if (!rp) {  // intermediate :before -> ensure-residual (problem.lisp:109-116)
      if (step == 0 && g->x_zero) launch_copy(b, g->r, n, st);  // x = 0: r = b exactly
      else launch_spmv(T, x, b, g->r, nullptr, nullptr, st);
      launch_dot(g->r, g->r, n, reducer(g, EPI_STORE, S_RR), st);
      if ((rc = launched(c, "residual"))) return rc;
      rp = true;
    }
    if ((rc = read_scalars(g))) return rc;
    defnorm = std::sqrt(c->host_scal[S_RR]);
    if (initialized) alpha = c->host_scal[S_ALPHA];
    if (!std::isfinite(defnorm)) {
      *nsteps = step;
      return set_err(c, FMG_ERR_NUMERIC, "defnorm is %g at step %d", defnorm, step);
    }
    if (initial < 0) initial = defnorm;
    const double reduction = initial == 0.0 ? 0.0 : defnorm / initial;
    if (hist && step < hist_len) hist[step] = defnorm;
    *nsteps = step;
    if (judge_active && step >= judged_from && prev > 0.0) {
      // MG: the mean reduction of the last 3 cycles against the plain cycle's
      // contraction, or a cycle growing the residual 1.5x; CG: residual norms
      // are not monotone, so only divergence (100x the initial residual) counts
      bool drop;
      if (cf.method == FMG_METHOD_MG) {
        const double rho = defnorm / prev;
        win[step % 3] = rho;
        const double bound = g->rho_plain > 0 ? g->rho_plain : 0.9;
        drop = rho > 1.5 || (step >= judged_from + 2 && std::cbrt(win[0] * win[1] * win[2]) > bound);
      } else {
        drop = defnorm > 100.0 * initial;
      }
      if (drop) {
        for (Lvl& L : g->lev) { hidden.push_back(L.omega); L.omega = nullptr; }
        judge_active = false;
        g->reverts += 1;
        initialized = false;  // CG restarts from the current residual with the plain cycle
      }
    }
    prev = defnorm;
    if ((cf.rtol > 0 && reduction < cf.rtol) || (cf.atol > 0 && defnorm < cf.atol)) { *status = 0; break; }
    if (step > cf.maxsteps) { *status = 1; break; }
    if (cf.method == FMG_METHOD_MG) {
      mg.iterate(&x, &xspare, const_cast<double*>(b), g->r);
      rp = false;
      continue;
    }
    // <cg> (krylow.lisp:72-132)
    if (!initialized) {  // restart: w := r; M(p <- w, w); alpha = (p, r)
      if (cf.method == FMG_METHOD_CG_MG) {
        if (cf.compat_alias) {
          launch_copy(g->r, g->w, n, st);
          mg.iterate(&g->p, &g->xs, g->w, g->w);
        } else {
          launch_copy(g->r, g->w2, n, st);
          mg.iterate(&g->p, &g->xs, g->r, g->w2);
        }
      } else {
        launch_copy(g->r, g->p, n, st);
      }
      launch_dot(g->p, g->r, n, reducer(g, EPI_STORE, S_ALPHA), st);
      if ((rc = launched(c, "restart"))) return rc;
      if ((rc = read_scalars(g))) return rc;
      alpha = c->host_scal[S_ALPHA];
      initialized = true;
    }
    if (alpha != 0.0) {  // krylow.lisp:106-127
      const bool pre = cf.method == FMG_METHOD_CG_MG;
      const Reduce Rl = reducer(g, EPI_CG_LAMBDA, 0);
      launch_spmv(T, g->p, nullptr, g->a, g->p, &Rl, st);  // a = A p; beta = (a,p); lam = alpha/beta
      const Reduce Rr = reducer(g, EPI_STORE, S_RR);
      // x += lam p; r -= lam a; (r,r) for the next :defnorm; w := r; q := 0
      if (pre && cf.compat_alias)
        launch_cg_update(g->scal, x, g->p, g->r, g->a, g->w, nullptr, g->q, n, Rr, st);
      else if (pre)
        launch_cg_update(g->scal, x, g->p, g->r, g->a, nullptr, g->w2, g->q, n, Rr, st);
      else
        launch_cg_update(g->scal, x, g->p, g->r, g->a, g->q, nullptr, nullptr, n, Rr, st);  // q := (copy r)
      if (pre) {
        if (cf.compat_alias) mg.iterate(&g->q, &g->xs, g->w, g->w);
        else mg.iterate(&g->q, &g->xs, g->r, g->w2);
      }
      launch_dot(g->q, g->r, n, reducer(g, EPI_CG_ALPHA, 0), st);  // new alpha, ratio
      launch_p_update(g->scal, g->p, g->q, n, st);                     // p := ratio p + q
      if ((rc = launched(c, "cg step"))) return rc;
    }
    rp = true;  // residual-after t
  }
  if (x != xv->d) launch_copy(x, xv->d, n, st);
  if (!hidden.empty())
    for (size_t l = 0; l < g->lev.size(); ++l) g->lev[l].omega = hidden[l];
  FMG_CK(c, cudaStreamSynchronize(st));
  if (g->ssc_unprepared) return set_err(c, FMG_ERR_STATE, "SSC factors missing");
  return launched(c, "solve");
}

// <cg>'s iterator one call at a time (krylow.lisp:72-132), for a host whose
// own solver loop drives it (linsolve.lisp:58-73): fmg_cg_start is the
// iterator's initialize (restart: w := r, p := M(w), alpha := (p, r)),
// fmg_cg_step its iterate (a := A p, lam := alpha / (a, p), x += lam p,
// r -= lam a, q := M(r), alpha' := (q, r), p := (alpha'/alpha) p + q).  The
// search direction and the preconditioner's vectors stay in the grid between
// calls; x and r are the caller's vectors (r up to date at the start,
// :residual-before t; kept up to date by every step, :residual-after t).
int fmg_cg_start(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_vec* rv) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  FMG_RC(ensure_top(g));
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (vec_check(rv, g, g->top)) return FMG_ERR_ARG;
  if (cfg->method == FMG_METHOD_MG) return set_err(g->ctx, FMG_ERR_ARG, "fmg_cg_start: a CG method");
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const long long n = g->lev[g->top].N * g->nc;
  MG mg{g, *cfg, false, st};
  double* r = rv->d;
  if (cfg->method == FMG_METHOD_CG_MG) {
    launch_fill(g->p, n, 0.0, st);  // the preconditioner starts from x = 0 (make-domain-vector-for)
    if (cfg->compat_alias) {
      launch_copy(r, g->w, n, st);
      mg.iterate(&g->p, &g->xs, g->w, g->w);
    } else {
      launch_copy(r, g->w2, n, st);
      mg.iterate(&g->p, &g->xs, r, g->w2);
    }
  } else {
    launch_copy(r, g->p, n, st);
  }
  launch_dot(g->p, r, n, reducer(g, EPI_STORE, S_ALPHA), st);
  if ((rc = launched(c, "cg start"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  g->cg_alpha = c->host_scal[S_ALPHA];
  g->cg_cfg = *cfg;
  g->cg_started = true;
  return FMG_OK;
}

int fmg_cg_step(fmg_grid* g, fmg_vec* xv, fmg_vec* rv, double* defnorm) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (!g->cg_started) return set_err(g->ctx, FMG_ERR_STATE, "fmg_cg_step before fmg_cg_start");
  if (vec_check(xv, g, g->top) || vec_check(rv, g, g->top) || xv == rv) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const fmg_solve_cfg& cf = g->cg_cfg;
  const LevelView T = view(g, g->top);
  const long long n = T.N * g->nc;
  double *x = xv->d, *r = rv->d;
  MG mg{g, cf, false, st};
  int rc;
  if (g->cg_alpha != 0.0) {  // krylow.lisp:106-127, as in fmg_solve
    const bool pre = cf.method == FMG_METHOD_CG_MG;
    const Reduce Rl = reducer(g, EPI_CG_LAMBDA, 0);
    launch_spmv(T, g->p, nullptr, g->a, g->p, &Rl, st);
    const Reduce Rr = reducer(g, EPI_STORE, S_RR);
    if (pre && cf.compat_alias)
      launch_cg_update(g->scal, x, g->p, r, g->a, g->w, nullptr, g->q, n, Rr, st);
    else if (pre)
      launch_cg_update(g->scal, x, g->p, r, g->a, nullptr, g->w2, g->q, n, Rr, st);
    else
      launch_cg_update(g->scal, x, g->p, r, g->a, g->q, nullptr, nullptr, n, Rr, st);
    if (pre) {
      if (cf.compat_alias) mg.iterate(&g->q, &g->xs, g->w, g->w);
      else mg.iterate(&g->q, &g->xs, r, g->w2);
    }
    launch_dot(g->q, r, n, reducer(g, EPI_CG_ALPHA, 0), st);
    launch_p_update(g->scal, g->p, g->q, n, st);
  } else {  // nothing to do: the residual norm is reported as it stands
    launch_dot(r, r, n, reducer(g, EPI_STORE, S_RR), st);
  }
  if ((rc = launched(c, "cg step"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  if (g->cg_alpha != 0.0) g->cg_alpha = c->host_scal[S_ALPHA];
  const double dn = std::sqrt(c->host_scal[S_RR]);
  if (!std::isfinite(dn)) return set_err(c, FMG_ERR_NUMERIC, "defnorm is %g", dn);
  if (defnorm) *defnorm = dn;
  return FMG_OK;
}


// ================================================================ batches
// A batch holds nb independent problems of one geometry (a 1D or 2D scalar
// Q1 hierarchy) in shared buffers, each problem at a fixed stride: the
// multigrid iterator and CG run all of them in the same launches, the
// kernels taking the problem from a grid coordinate, every reduction and
// every CG scalar per problem.  The arithmetic per problem is that of
// fmg_solve on the problem's own grid.
int fmg_batch_create(fmg_grid* like, int nbatch, fmg_grid** out) {
  if (!like || !out || nbatch < 1) return FMG_ERR_ARG;
  *out = nullptr;
  fmg_ctx* c = like->ctx;
  if (like->nb > 1 || like->algebraic || like->nc != 1 || like->order != 1 || like->dim > 2)
    return set_err(c, FMG_ERR_UNSUPPORTED, "fmg_batch_create: 1D or 2D scalar Q1 grids");
  const long long nb_base = like->lev[like->base].N;
  if (nb_base > 1024)
    return set_err(c, FMG_ERR_UNSUPPORTED, "fmg_batch_create: base level has %lld unknowns (<= 1024)", nb_base);
  fmg_grid* g = new (std::nothrow) fmg_grid();
  if (!g) return FMG_ERR_NOMEM;
  g->ctx = c;
  c->grids += 1;
  g->dim = like->dim; g->order = like->order; g->nc = 1; g->n0 = like->n0;
  g->top = like->top; g->base = like->base; g->dmask = like->dmask;
  g->nslots = like->nslots; g->center = like->center;
  g->lev.resize(like->lev.size());
  for (size_t l = 0; l < like->lev.size(); ++l) {
    Lvl& L = g->lev[l];
    const Lvl& S = like->lev[l];
    L.n = S.n; L.M = S.M; L.N = S.N; L.Np = S.Np; L.h = S.h;
  }
  g->nb = nbatch;
  g->loaded.assign(nbatch, 0);
  g->nbase = (int)nb_base;
  int rc = FMG_OK;
  FMG_CK(c, cudaSetDevice(c->device));
  const long long B = nbatch;
  const Lvl& T = g->lev[g->top];
  for (int l = g->base; l <= g->top && !rc; ++l) {
    Lvl& L = g->lev[l];
    rc = dalloc(g, &L.A, (long long)g->nslots * L.Np * B);
    if (l < g->top) {
      if (!rc) rc = dalloc(g, &L.sol[0], L.Np * B);
      if (!rc) rc = dalloc(g, &L.sol[1], L.Np * B);
      if (!rc) rc = dalloc(g, &L.rhs, L.Np * B);
      if (!rc) rc = dalloc(g, &L.res, L.Np * B);
    }
  }
  if (!rc) rc = dalloc(g, &g->rhs, T.Np * B);
  if (!rc) rc = dalloc(g, &g->ainvT, nb_base * nb_base * B);
  if (!rc) rc = dalloc(g, &g->scal, S_COUNT * B);
  if (!rc) rc = dalloc(g, &g->part, (nchunks(T.Np) + 1) * B);
  if (!rc) rc = dalloc(g, (double**)&g->counter, (B + 1) / 2);
  if (!rc) rc = dalloc(g, &g->frozen, B);
  double** tv[] = {&g->p, &g->a, &g->w, &g->w2, &g->q, &g->r, &g->xs, &g->xs2};
  for (double** v : tv)
    if (!rc) rc = dalloc(g, v, T.Np * B);
  if (rc) {
    grid_release(g);
    return rc;
  }
  const int nlev = g->top + 1;
  g->solp.assign(nlev, nullptr); g->sparep.assign(nlev, nullptr);
  g->rhsp.assign(nlev, nullptr); g->resp.assign(nlev, nullptr);
  g->rp.assign(nlev, 0);
  for (int l = g->base; l < g->top; ++l) {
    g->solp[l] = g->lev[l].sol[0]; g->sparep[l] = g->lev[l].sol[1];
    g->rhsp[l] = g->lev[l].rhs; g->resp[l] = g->lev[l].res;
  }
  g->assembled_once = true;
  *out = g;
  return launched(c, "batch create");
}

// Problem `index` of the batch from an assembled grid of the same geometry:
// its level matrices, top-level rhs, coarse inverse and node damping.  Node
// damping must be present on a level for every problem or for none.
int fmg_batch_load(fmg_grid* g, int index, fmg_grid* src) {
  if (!g || !src || g->nb < 2 || index < 0 || index >= g->nb) return FMG_ERR_ARG;
  fmg_ctx* c = g->ctx;
  if (src->ctx != c || src->nb > 1 || src->algebraic || src->dim != g->dim || src->order != g->order ||
      src->nc != 1 || src->n0 != g->n0 || src->top != g->top || src->base != g->base || src->dmask != g->dmask)
    return set_err(c, FMG_ERR_ARG, "fmg_batch_load: the source grid's geometry differs from the batch's");
  if (!src->assembled) return set_err(c, FMG_ERR_STATE, "fmg_batch_load: the source grid is not assembled");
  FMG_RC(ensure_top(src));
  cudaStream_t st = c->stream;
  int rc;
  for (int l = g->base; l <= g->top; ++l) {
    Lvl& L = g->lev[l];
    const Lvl& S = src->lev[l];
    const size_t mb = (size_t)g->nslots * L.Np * sizeof(double);
    FMG_CK(c, cudaMemcpyAsync(L.A + (size_t)index * g->nslots * L.Np, S.A, mb, cudaMemcpyDeviceToDevice, st));
    const bool had = L.omega != nullptr;
    bool first = true;
    for (int k = 0; k < g->nb; ++k) first = first && (!g->loaded[k] || k == index);
    if ((S.omega != nullptr) != had && !first)
      return set_err(c, FMG_ERR_STATE, "fmg_batch_load: node damping on level %d for some problems only", l);
    if (S.omega && !had && (rc = dalloc(g, &L.omega, L.Np * g->nb))) return rc;
    if (!S.omega && had) L.omega = nullptr;  // the first problem loaded again, now without damping
    if (S.omega)
      FMG_CK(c, cudaMemcpyAsync(L.omega + (size_t)index * L.Np, S.omega, (size_t)L.N * sizeof(double),
                                cudaMemcpyDeviceToDevice, st));
  }
  const Lvl& T = g->lev[g->top];
  FMG_CK(c, cudaMemcpyAsync(g->rhs + (size_t)index * T.Np, src->rhs, (size_t)T.N * sizeof(double),
                            cudaMemcpyDeviceToDevice, st));
  const size_t nn = (size_t)g->nbase * g->nbase;
  FMG_CK(c, cudaMemcpyAsync(g->ainvT + index * nn, src->ainvT, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
  g->loaded[index] = 1;
  bool all = true;
  for (char k : g->loaded) all = all && k;
  g->assembled = all;
  return launched(c, "batch load");
}

// fmg_solve of every problem of the batch at once (CG + MG, MG or CG; the
// Jacobi smoother, multiplicative cycles, the clean preconditioner call):
// each problem stops at its own tolerance or maxsteps and keeps its iterate
// from then on; steps, status and the defnorm histories (hist: hist_len
// entries per problem) are per problem.  The judge of learned damping is not
// run: each problem uses the node damping it was loaded with.
int fmg_batch_solve(fmg_grid* g, const fmg_solve_cfg* cfg, fmg_vec* xv, double* hist, int hist_len, int* steps,
                    int* status) {
  if (!g || g->nb < 2) return g ? set_err(g->ctx, FMG_ERR_ARG, "fmg_batch_solve: not a batch") : FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "fmg_batch_solve: problems not loaded");
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (vec_check(xv, g, g->top) || !steps || !status) return FMG_ERR_ARG;
  const fmg_solve_cfg& cf = *cfg;
  if (cf.smoother != FMG_JACOBI || cf.combination != FMG_MULTIPLICATIVE || cf.fmg || cf.compat_alias)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED,
                   "fmg_batch_solve: Jacobi, multiplicative cycles, no f-cycle, the clean preconditioner call");
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const int nb = g->nb;
  const Lvl& T = g->lev[g->top];
  const LevelView TV = view(g, g->top);
  const long long n = T.N, vs = T.Np, nall = vs * nb;
  const double* b = g->rhs;
  // CG updates x in place (a stopped problem's iterate stays frozen); the MG
  // iteration moves every problem, so it runs on two internal vectors and a
  // problem's iterate is copied to x when it stops
  const bool mgit = cf.method == FMG_METHOD_MG;
  double* x = mgit ? g->a : xv->d;
  double* xspare = mgit ? g->q : g->xs2;
  MG mg{g, cf, false, st};
  std::vector<double> hs((size_t)S_COUNT * nb), initial(nb, -1.0), fz(nb, 0.0);
  std::vector<char> done(nb, 0);
  for (int k = 0; k < nb; ++k) { steps[k] = 0; status[k] = 1; }
  auto read_all = [&]() -> int {
    FMG_CK(c, cudaMemcpyAsync(hs.data(), g->scal, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    FMG_CK(c, cudaStreamSynchronize(st));
    return FMG_OK;
  };
  auto reducer_b = [&](int epi, int slot) { return reducer(g, epi, slot); };
  launch_fill(g->p, nall, 0.0, st);
  launch_fill(g->frozen, nb, 0.0, st);
  if (mgit) launch_copy(xv->d, x, nall, st);
  bool initialized = false;
  for (int step = 0;; ++step) {
    if (step == 0) {
      launch_spmv(TV, x, b, g->r, nullptr, nullptr, st);
      launch_dot_b(g->r, g->r, n, vs, nb, reducer_b(EPI_STORE, S_RR), st);
      if ((rc = launched(c, "batch residual"))) return rc;
    }
    if ((rc = read_all())) return rc;
    bool changed = false, all = true;
    for (int k = 0; k < nb; ++k) {
      if (done[k]) continue;
      const double dn = std::sqrt(hs[(size_t)k * S_COUNT + S_RR]);
      if (!std::isfinite(dn)) return set_err(c, FMG_ERR_NUMERIC, "problem %d: defnorm is %g at step %d", k, dn, step);
      if (initial[k] < 0) initial[k] = dn;
      if (hist && step < hist_len) hist[(size_t)k * hist_len + step] = dn;
      steps[k] = step;
      const double red = initial[k] == 0.0 ? 0.0 : dn / initial[k];
      const bool conv = (cf.rtol > 0 && red < cf.rtol) || (cf.atol > 0 && dn < cf.atol);
      if (conv || step > cf.maxsteps) {
        status[k] = conv ? 0 : 1;
        done[k] = 1;
        fz[k] = 1.0;
        changed = true;
        if (mgit)  // the iterate of this step is the problem's result
          FMG_CK(c, cudaMemcpyAsync(xv->d + (size_t)k * vs, x + (size_t)k * vs, n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st));
      }
      all = all && done[k];
    }
    if (all) break;
    if (changed) FMG_CK(c, cudaMemcpyAsync(g->frozen, fz.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
    if (mgit) {
      mg.iterate(&x, &xspare, const_cast<double*>(b), g->r);
      launch_spmv(TV, x, b, g->r, nullptr, nullptr, st);
      launch_dot_b(g->r, g->r, n, vs, nb, reducer_b(EPI_STORE, S_RR), st);
      if ((rc = launched(c, "batch mg step"))) return rc;
      continue;
    }
    const bool pre = cf.method == FMG_METHOD_CG_MG;
    if (!initialized) {  // w := r; p := M(w) (or r); alpha := (p, r)
      if (pre) {
        launch_copy(g->r, g->w2, nall, st);
        mg.iterate(&g->p, &g->xs, g->r, g->w2);
      } else {
        launch_copy(g->r, g->p, nall, st);
      }
      launch_dot_b(g->p, g->r, n, vs, nb, reducer_b(EPI_STORE, S_ALPHA), st);
      initialized = true;
    }
    const Reduce Rl = reducer_b(EPI_CG_LAMBDA, 0);
    launch_spmv(TV, g->p, nullptr, g->a, g->p, &Rl, st);  // a = A p; lam = alpha / (a, p)
    const Reduce Rr = reducer_b(EPI_STORE, S_RR);
    if (pre) launch_cg_update_b(g->scal, x, g->p, g->r, g->a, nullptr, g->w2, g->q, n, vs, nb, g->frozen, Rr, st);
    else launch_cg_update_b(g->scal, x, g->p, g->r, g->a, g->q, nullptr, nullptr, n, vs, nb, g->frozen, Rr, st);
    if (pre) mg.iterate(&g->q, &g->xs, g->r, g->w2);
    launch_dot_b(g->q, g->r, n, vs, nb, reducer_b(EPI_CG_ALPHA, 0), st);
    launch_p_update_b(g->scal, g->p, g->q, n, vs, nb, g->frozen, st);
    if ((rc = launched(c, "batch cg step"))) return rc;
  }
  FMG_CK(c, cudaStreamSynchronize(st));
  return launched(c, "batch solve");
}

}  // extern "C"

// the give-up path of the bounded device waits, run alone
extern "C" int fmg_wait_selftest(fmg_ctx* c, int arrive, int max_polls, long long max_ns) {
  if (!c) return FMG_ERR_ARG;
  if (max_polls < 1 || max_polls > (1 << 24) || max_ns < 1 || max_ns > 2000000000ll)
    return set_err(c, FMG_ERR_ARG, "fmg_wait_selftest: polls in [1, 2^24], ns in [1, 2e9]");
  const char* msg = nullptr;
  const int rc = wait_selftest(arrive != 0, max_polls, max_ns, c->stream, &msg);
  return rc == FMG_OK ? FMG_OK : set_err(c, rc, "%s", msg);
}

// context accessors for the allocation-free entry point (fmgpu_noalloc.cu)
namespace fmg {
int ctx_device(const fmg_ctx* c) { return c->device; }
cudaStream_t ctx_stream(const fmg_ctx* c) { return c->stream; }
int ctx_error(fmg_ctx* c, int code, const char* msg) {
  c->err = msg;
  return code;
}
}  // namespace fmg

// ============================================================ mixed solve
// FP64 iterative refinement around an FP32 flexible CG whose preconditioner is
// one V-cycle in FP32 (smoothing, restriction, prolongation), with BF16
// coarse right-hand sides and residuals and the coarsest dense solve in FP64.
// The outer residual r = b - A x and the update x += e use the assembled FP64
// top-level matrix, so the reported :defnorm is the true FP64 residual.
namespace {

int mx_alloc_f(fmg_grid* g, float** p, long long n) { return dalloc(g, (double**)p, (n + 1) / 2); }

// the mixed solve applies its top level matrix-free (3D scalar Q1 with cell
// coefficients, the matrix not uploaded) when asked to
bool mixed_top_mf(const fmg_grid* g, bool want_mf) {
  return want_mf && g->dim == 3 && g->order == 1 && g->nc == 1 && !g->uploaded && g->kkind == FMG_K_CELL;
}

// the FP64 matrix-free operator of the top level
MFArgs64 mf64_args(const fmg_grid* g, double damp) {
  const Lvl& L = g->lev[g->top];
  MFArgs64 m;
  m.k = g->kcell_d; m.omega = nullptr; m.N = L.N; m.M = (int)L.M; m.n = (int)L.n; m.dmask = g->dmask;
  m.hs = L.h / 12.0; m.w = damp;
  m.err = g->scal + S_MFERR;
  m.xl = m.ol = m.yl = natural_lay((int)L.M, 3);
  return m;
}

int mixed_prepare(fmg_grid* g, bool want_mf) {
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  int rc;
  if (!g->mx) g->mx = new MixedState();
  MixedState& X = *g->mx;
  const int nl = g->top + 1;
  // the matrix-free top level rebuilds A from the coefficients: not for uploaded matrices
  const bool mf = mixed_top_mf(g, want_mf);
  if (X.lv.empty()) {  // first use: allocate
    X.lv.assign(nl, Lev32{});
    X.A32.assign(nl, nullptr); X.om32.assign(nl, nullptr);
    X.x0.assign(nl, nullptr); X.x1.assign(nl, nullptr);
    X.bc.assign(nl, nullptr); X.rc.assign(nl, nullptr);
    for (int l = g->base; l <= g->top; ++l) {
      const Lvl& L = g->lev[l];
      if ((rc = mx_alloc_f(g, &X.A32[l], (long long)g->nslots * L.Np)) || (rc = mx_alloc_f(g, &X.x0[l], L.Np)) ||
          (rc = mx_alloc_f(g, &X.x1[l], L.Np)) || (rc = mx_alloc_f(g, &X.om32[l], L.Np)))
        return rc;
      if ((rc = dalloc(g, (double**)&X.bc[l], (L.Np + 3) / 4)) || (rc = dalloc(g, (double**)&X.rc[l], (L.Np + 3) / 4)))
        return rc;
    }
    const Lvl& T = g->lev[g->top];
    long long ncell = 1;
    for (int k = 0; k < g->dim; ++k) ncell *= T.n;
    // top-level vectors: room for the padded layout where the grid has one
    X.cap = T.Np;
    if (g->dim == 3) X.cap = std::max(X.cap, (padded_lay((int)T.M, g->dmask).total + 63) / 64 * 64);
    float** tv[] = {&X.rtop, &X.r, &X.q, &X.qs, &X.p32, &X.wd, &X.zp, &X.zs};
    for (float** v : tv)
      if ((rc = mx_alloc_f(g, v, X.cap))) return rc;
    if ((rc = dalloc(g, &X.r64, X.cap)) || (rc = dalloc(g, &X.a64, X.cap)) || (rc = dalloc(g, &X.x64, X.cap)))
      return rc;
    if ((rc = mx_alloc_f(g, &X.k32, ncell))) return rc;
    const long long nparts =
        std::max({(long long)nchunks(X.cap), mx_top_blocks((int)T.M), X.cap / kBlock + 1}) + 1;
    if ((rc = dalloc(g, &X.sc, M_COUNT)) || (rc = dalloc(g, &X.part, 2 * nparts)) ||
        (rc = dalloc(g, (double**)&X.counter, 1)))
      return rc;
    if (!X.host) FMG_CK(c, cudaMallocHost((void**)&X.host, M_COUNT * sizeof(double)));
  }
  auto to32 = [&](int l) {
    const Lvl& L = g->lev[l];
    if (g->order == 2) launch_level_to_f32(view(g, l), g->nslots, X.A32[l], st);  // sliced -> full slots
    else mx_f64_to_f32(L.A, X.A32[l], (long long)g->nslots * L.Np, st);
  };
  if (X.epoch != g->epoch) {  // convert the current assembly (the top level only where it is stored)
    for (int l = g->base; l < g->top; ++l) to32(l);
    if (g->kkind == FMG_K_CELL) {
      long long ncell = 1;
      for (int k = 0; k < g->dim; ++k) ncell *= g->lev[g->top].n;
      mx_f64_to_f32(g->kcell_d, X.k32, ncell, st);
    }
    X.epoch = g->epoch;
    X.top32 = false;
  }
  if (!mf && !X.top32) {
    FMG_RC(ensure_top(g));
    to32(g->top);
    X.top32 = true;
  }
  for (int l = g->base; l <= g->top; ++l) {  // per-node damping may change between solves
    const Lvl& L = g->lev[l];
    if (L.omega) mx_f64_to_f32(L.omega, X.om32[l], L.N, st);
    Lev32& V = X.lv[l];
    V.A = X.A32[l]; V.om = L.omega ? X.om32[l] : nullptr;
    V.N = L.N; V.Np = L.Np; V.M = L.M; V.dim = g->dim; V.order = g->order; V.dmask = g->dmask;
  }
  const VLay lay = mf ? padded_lay((int)g->lev[g->top].M, g->dmask)
                     : natural_lay((int)g->lev[g->top].M, g->dim);
  if (lay.front != X.lay.front || lay.py != X.lay.py || lay.pz != X.lay.pz || lay.total != X.lay.total) {
    // a new layout: the padding of every top-level vector starts (and stays) zero
    float* fv[] = {X.r, X.q, X.qs, X.p32, X.wd, X.zp, X.zs};
    for (float* v : fv) FMG_CK(c, cudaMemsetAsync(v, 0, X.cap * sizeof(float), st));
    FMG_CK(c, cudaMemsetAsync(X.r64, 0, X.cap * sizeof(double), st));
    FMG_CK(c, cudaMemsetAsync(X.a64, 0, X.cap * sizeof(double), st));
    FMG_CK(c, cudaMemsetAsync(X.x64, 0, X.cap * sizeof(double), st));
    X.lay = lay;
    X.wd_ok = false;
  }
  X.mf = mf;
  return launched(c, "mixed prepare");
}

struct MixedMG {
  fmg_grid* g;
  MixedState& X;
  const fmg_solve_cfg& c;
  cudaStream_t st;

  bool top_mf() const { return X.mf && g->kkind == FMG_K_CELL; }
  MFArgs mf_args() const {
    const Lvl& T = g->lev[g->top];
    MFArgs a;
    a.k = X.k32;
    a.omega = X.lv[g->top].om;
    a.N = T.N; a.M = (int)T.M; a.n = (int)T.n; a.dmask = g->dmask;
    a.hs = (float)(T.h / 12.0);
    a.w = (float)c.damp;
    const bool wd = X.wd_ok && X.wd_om == a.omega && X.wd_w == a.w;
    a.wd = wd ? X.wd : nullptr;
    a.err = g->scal + S_MFERR;
    a.xl = a.ol = a.yl = X.lay;
    return a;
  }
  // damping / diagonal of the top level for the damping now in use (once per
  // solve, and again after a revert to the plain damping)
  void prepare_wd() {
    X.wd_ok = false;
    if (!top_mf()) return;
    const MFArgs a = mf_args();
    mx_top_wd(a, X.wd, st);
    X.wd_om = a.omega;
    X.wd_w = a.w;
    X.wd_ok = true;
  }
  // one FP32 operator application on level l (modes of k_mf_q1 / k_st32)
  void apply(int l, int mode, const float* x, const void* b, bool b_bf16, void* y, bool y_bf16, const double* v,
             const double* v2, const Reduce2* R) {
    Lev32 L = X.lv[l];
    L.w = (float)c.damp;
    if (l == g->top && top_mf() && !b_bf16 && !y_bf16) {
      MFArgs a = mf_args();
      if (a.omega && (mode == 2 || mode == 3) && !a.wd) {  // the padded smoothing takes its damping over d formed
        prepare_wd();
        a = mf_args();
      }
      if (mode <= 1) a.yl = natural_lay(a.M, 3);  // A x and residuals come out in the natural layout (rtop)
      mx_top_apply(mode, a, x, (const float*)b, (float*)y, v, v2, R, st);
    } else {
      mx_level_apply(mode, L, x, b, b_bf16, y, y_bf16, v, v2, R, st);
    }
  }
  // V-cycle on level l from x = 0 for rhs b (FP32 on the top level, BF16
  // below); the result is left in X.x0[l] (top: *xq); with R the last top-level
  // smoothing step also reduces (x, v) and (x, v2)
  void vcycle(int l, const void* b, float** xq, float** xs, const double* v, const double* v2, const Reduce2* R) {
    const bool top = (l == g->top);
    const bool bbf = !top;
    float*& x = top ? *xq : X.x0[l];
    float*& xn = top ? *xs : X.x1[l];
    if (l == g->base) {
      mx_coarse(g->ainvT, g->nbase, (const __nv_bfloat16*)b, x, st);
      return;
    }
    if (c.pre_steps >= 1) {  // pre-smoothing from x = 0
      apply(l, 3, nullptr, b, bbf, x, false, nullptr, nullptr, nullptr);
      for (int s = 1; s < c.pre_steps; ++s) {
        apply(l, 2, x, b, bbf, xn, false, nullptr, nullptr, nullptr);
        std::swap(x, xn);
      }
    } else {
      launch_fill((double*)x, ((top ? X.lay.total : X.lv[l].Np) + 1) / 2, 0.0, st);
    }
    void* r = top ? (void*)X.rtop : (void*)X.rc[l];  // residual and restriction
    apply(l, 1, x, b, bbf, r, !top, nullptr, nullptr, nullptr);
    mx_restrict(X.lv[l], X.lv[l - 1], r, !top, X.bc[l - 1], X.x0[l - 1], st);
    vcycle(l - 1, X.bc[l - 1], nullptr, nullptr, nullptr, nullptr, nullptr);
    mx_prolong(X.lv[l - 1], X.lv[l], X.x0[l - 1], x, st, top ? &X.lay : nullptr);
    for (int s = 0; s < c.post_steps; ++s) {
      const bool last = top && R && s == c.post_steps - 1;
      apply(l, 2, x, b, bbf, xn, false, last ? v : nullptr, last ? v2 : nullptr, last ? R : nullptr);
      std::swap(x, xn);
    }
  }
  // FP64 a = A p for the FP32 search direction p, with (a, p) -> lam = rho / (a, p)
  void matvec64(const float* p, double* a, const Reduce2& Rl) {
    const LevelView T = view(g, g->top);
    if (top_mf()) {
      MFArgs64 m = mf64_args(g, c.damp);
      m.xl = X.lay;                    // p: a top-level FP32 vector
      if (a == X.a64) m.yl = X.lay;    // the CG's A p; elsewhere (the judge's scratch) natural
      mx_top_apply64(m, p, a, p, &Rl, st);
    } else {  // stored FP64 matrix: widen p first
      mx_f32_to_f64(p, g->xs2, T.N, st);
      launch_spmv(T, g->xs2, nullptr, a, nullptr, nullptr, st);
      mx_dot2_64(a, p, nullptr, T.N, Rl, st);
    }
  }

};

Reduce2 red2(MixedState& X, int epi, int s0, int s1) {
  Reduce2 R;
  R.part = X.part; R.counter = X.counter; R.scal = X.sc; R.epi = epi; R.slot0 = s0; R.slot1 = s1;
  return R;
}

int mx_read(fmg_grid* g) {
  MixedState& X = *g->mx;
  FMG_CK(g->ctx, cudaMemcpyAsync(X.host, X.sc, M_COUNT * sizeof(double), cudaMemcpyDeviceToHost, g->ctx->stream));
  FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
  return FMG_OK;
}

int mx_set_scalar(fmg_grid* g, int slot, double v) {
  MixedState& X = *g->mx;
  X.host[slot] = v;
  FMG_CK(g->ctx, cudaMemcpyAsync(X.sc + slot, X.host + slot, sizeof(double), cudaMemcpyHostToDevice, g->ctx->stream));
  return FMG_OK;
}

// key of one CG step: the vectors it reads and writes, the level buffers in
// their current ping-pong state, the node damping in use and the cycle's
// scalar parameters
std::vector<uint64_t> step_key(const fmg_grid* g, const MixedState& X, const fmg_solve_cfg& c, const double* x) {
  std::vector<uint64_t> k;
  auto P = [&](const void* v) { k.push_back((uint64_t)(uintptr_t)v); };
  P(x); P(X.q); P(X.qs); P(X.r); P(X.rtop);
  for (size_t l = 0; l < X.lv.size(); ++l) { P(X.x0[l]); P(X.x1[l]); P(X.lv[l].om); }
  uint64_t d;
  std::memcpy(&d, &c.damp, sizeof d);
  k.push_back(d);
  k.push_back((uint64_t)c.pre_steps << 32 | (uint32_t)c.post_steps);
  k.push_back((uint64_t)(X.mf ? 1 : 0) << 8 | (uint64_t)g->kkind | (uint64_t)(X.wd_ok ? 1 : 0) << 16);
  P(X.wd_om);
  return k;
}

// Runs one CG step through a cached CUDA graph (captured on first use): the
// ~30 launches of a step then cost one graph launch.  body() must queue the
// whole step, the scalar copy to the host included, and nothing that waits.
template <class Body>
int run_step_graph(fmg_grid* g, const fmg_solve_cfg& c, const double* x, Body body) {
  MixedState& X = *g->mx;
  fmg_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  if (X.graphs_off) {
    body();
    return launched(ctx, "mixed step");
  }
  const std::vector<uint64_t> key = step_key(g, X, c, x);
  MixedState::StepGraph* e = nullptr;
  for (auto& ge : X.graphs)
    if (ge.key == key) e = &ge;
  if (!e) {
    const float *q0 = X.q, *qs0 = X.qs;
    const std::vector<float*> x00 = X.x0, x10 = X.x1;
    const long long l0 = g_launches.load(std::memory_order_relaxed);
    cudaGraph_t gr = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      body();
      ok = cudaStreamEndCapture(st, &gr) == cudaSuccess && gr;
      ok = ok && cudaGraphInstantiate(&ex, gr, 0) == cudaSuccess;
      if (gr) cudaGraphDestroy(gr);
    }
    const long long nl = g_launches.load(std::memory_order_relaxed) - l0;
    g_launches.fetch_sub(nl, std::memory_order_relaxed);  // queued in the graph, not launched yet
    if (!ok) {  // run this step eagerly from the state before the capture
      cudaGetLastError();
      X.q = const_cast<float*>(q0); X.qs = const_cast<float*>(qs0);
      X.x0 = x00; X.x1 = x10;
      X.graphs_off = true;
      body();
      return launched(ctx, "mixed step");
    }
    if (X.graphs.size() >= 4) {
      cudaGraphExecDestroy(X.graphs.front().exec);
      X.graphs.erase(X.graphs.begin());
    }
    MixedState::StepGraph ng;
    ng.key = key; ng.exec = ex; ng.launches = nl;
    ng.q = X.q; ng.qs = X.qs; ng.x0 = X.x0; ng.x1 = X.x1;  // state after the step
    X.graphs.push_back(std::move(ng));
    e = &X.graphs.back();
  }
  FMG_CK(ctx, cudaGraphLaunch(e->exec, st));
  g_launches.fetch_add(e->launches, std::memory_order_relaxed);
  X.q = e->q; X.qs = e->qs; X.x0 = e->x0; X.x1 = e->x1;
  return FMG_OK;
}

}  // namespace

// Flexible CG in FP64 (recursive FP64 residual, FP64 solution update, FP64
// operator) preconditioned by one FP32/BF16 V-cycle per step.  The FP32
// residual handed to the V-cycle is scaled to unit norm by the previous
// step's residual norm; the preconditioned vector is scaled back in FP64.
// When the recursive residual meets the tolerance the true residual is
// recomputed with the assembled FP64 matrix and reported; if it does not meet
// the tolerance, CG restarts from it.
// ------------------------------------------------ mixed solve, vector form
// FP64 flexible CG (FCG(1): rho = (z, r), beta = -(z, a)/(p, a) of the last
// step, p = z + beta p, lam = rho / (a, p)) with FP64 x, r, p and a = A p on
// the assembled FP64 blocks; its preconditioner is one V(pre, post) cycle in
// FP32 -- 3 x 3 block Jacobi on FP32 copies of the level matrices, FP32
// transfers -- with the base level's dense solve in FP64.  The residual is
// handed to the cycle scaled to unit norm and its result scaled back.  At
// convergence of the recursive residual the true FP64 residual is checked,
// and CG restarts from it if it has not converged.
struct MixedVec {
  long long epoch = -1;
  std::vector<float*> A32, x, xs, b, r;  // per level
  double *b64 = nullptr, *x64 = nullptr;  // base level in FP64
  double* z = nullptr;                    // preconditioned residual, FP64
};

static void mixed_vec_delete(MixedVec* m) { delete m; }

static int mixed_vec_prepare(fmg_grid* g) {
  if (!g->mxv) g->mxv = new MixedVec();
  MixedVec& V = *g->mxv;
  cudaStream_t st = g->ctx->stream;
  int rc;
  const int nl = g->top + 1;
  if (V.A32.empty()) {
    V.A32.assign(nl, nullptr); V.x.assign(nl, nullptr); V.xs.assign(nl, nullptr);
    V.b.assign(nl, nullptr); V.r.assign(nl, nullptr);
    for (int l = g->base; l <= g->top; ++l) {
      const Lvl& L = g->lev[l];
      const long long nv = 3 * L.Np;
      if ((rc = mx_alloc_f(g, &V.A32[l], (long long)g->nslots * 9 * L.Np)) || (rc = mx_alloc_f(g, &V.x[l], nv)) ||
          (rc = mx_alloc_f(g, &V.xs[l], nv)) || (rc = mx_alloc_f(g, &V.b[l], nv)) || (rc = mx_alloc_f(g, &V.r[l], nv)))
        return rc;
    }
    if ((rc = dalloc(g, &V.b64, g->nbase)) || (rc = dalloc(g, &V.x64, g->nbase)) ||
        (rc = dalloc(g, &V.z, 3 * g->lev[g->top].Np)))
      return rc;
  }
  if (V.epoch != g->epoch) {  // FP32 copies of the current assembly (same layout)
    for (int l = g->base; l <= g->top; ++l) {
      const Lvl& L = g->lev[l];
      vec_f64_to_f32(L.A, V.A32[l], (long long)g->nslots * 9 * L.Np, st);
    }
    V.epoch = g->epoch;
  }
  return launched(g->ctx, "mixed prepare (vector form)");
}

// V.x[l] := V_l V.b[l] in FP32 from a zero guess (correction scheme)
static void vcycle32_vec(fmg_grid* g, const fmg_solve_cfg& cf, int l, cudaStream_t st) {
  MixedVec& V = *g->mxv;
  const Lvl& L = g->lev[l];
  const long long n = 3 * L.N;
  if (l == g->base) {
    vec_to64(V.b[l], nullptr, 0, 0, V.b64, n, st);
    launch_fill(V.x64, n, 0.0, st);
    launch_coarse_solve(g->ainvT, g->nbase, cf.coarse_damp, V.x64, V.b64, st);
    vec_to32(V.x64, nullptr, 0, 0, V.x[l], n, st);
    return;
  }
  float *x = V.x[l], *xs = V.xs[l];
  if (cf.pre_steps > 0) {
    vec32_jacobi0(V.A32[l], L.N, L.Np, g->center, (float)cf.damp, L.omega, V.b[l], x, st);
    for (int s = 1; s < cf.pre_steps; ++s) {
      vec32_jacobi_res(g->order, V.A32[l], L.N, L.Np, L.M, cf.damp, L.omega, x, V.b[l], xs, st);
      std::swap(x, xs);
    }
  } else {
    cudaMemsetAsync(x, 0, (size_t)n * sizeof(float), st);
  }
  vec32_spmv(g->order, V.A32[l], L.N, L.Np, L.M, x, V.b[l], V.r[l], st);  // r = b - A x
  const Lvl& C = g->lev[l - 1];
  vec32_restrict(g->order, C.M, L.M, g->dmask, V.r[l], V.b[l - 1], V.x[l - 1], st);
  vcycle32_vec(g, cf, l - 1, st);
  vec32_prolong(g->order, L.M, C.M, g->dmask, V.x[l - 1], x, st);
  for (int s = 0; s < cf.post_steps; ++s) {
    vec32_jacobi_res(g->order, V.A32[l], L.N, L.Np, L.M, cf.damp, L.omega, x, V.b[l], xs, st);
    std::swap(x, xs);
  }
  if (x != V.x[l]) cudaMemcpyAsync(V.x[l], x, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

static int solve_mixed_vec(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mcfg, fmg_vec* xv,
                           double* hist, int hist_len, int* nouter, int* ninner, int* status) {
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const fmg_solve_cfg& cf = *cfg;
  if (cf.method != FMG_METHOD_CG_MG)
    return set_err(c, FMG_ERR_UNSUPPORTED, "mixed solve: CG preconditioned by the multigrid cycle");
  int rc;
  if ((rc = mixed_vec_prepare(g))) return rc;
  MixedVec& V = *g->mxv;
  const int top = g->top;
  const LevelView T = view(g, top);
  const long long n = 3 * T.N;
  double *x = xv->d, *r = g->r, *p = g->p, *a = g->a, *z = V.z;
  const double* b = g->rhs;
  const int max_restart = mcfg->max_outer > 0 ? mcfg->max_outer : 20;
  double initial = -1.0;
  int step = 0, iters = 0;
  *status = 1;
  *nouter = 0;
  *ninner = 0;
  // learned damping, judged as it runs: only divergence (100x the restart's
  // residual) drops it -- hidden for the rest of the solve, restored after --
  // and CG restarts from the true residual with the plain cycle
  bool judge_active = g->learned;
  std::vector<double*> hidden;
  for (int restart = 0; restart <= max_restart; ++restart) {
    if (restart == 0 && g->x_zero) launch_copy(b, r, n, st);  // x = 0: r = b exactly
    else launch_spmv(T, x, b, r, nullptr, nullptr, st);      // true FP64 residual
    launch_dot(r, r, n, reducer(g, EPI_STORE, S_RR), st);
    if ((rc = read_scalars(g))) return rc;
    const double dn = std::sqrt(c->host_scal[S_RR]);
    if (!std::isfinite(dn)) return set_err(c, FMG_ERR_NUMERIC, "defnorm is %g", dn);
    if (initial < 0) initial = dn;
    if (hist && step < hist_len) hist[step] = dn;
    *nouter = restart;
    *ninner = iters;
    if ((cf.rtol > 0 && (initial == 0.0 || dn / initial < cf.rtol)) || (cf.atol > 0 && dn < cf.atol)) {
      *status = 0;
      break;
    }
    if (restart == max_restart || iters > cf.maxsteps) break;
    launch_fill(p, n, 0.0, st);
    bool first = true, converged = false;
    while (iters <= cf.maxsteps) {
      vec_to32(r, g->scal, S_RR, 1, V.b[top], n, st);  // r / |r|
      vcycle32_vec(g, cf, top, st);
      vec_to64(V.x[top], g->scal, S_RR, 2, z, n, st);  // z = |r| V(r / |r|)
      launch_dot(z, r, n, reducer(g, EPI_STORE, S_ALPHA), st);           // rho
      if (!first) launch_dot(z, a, n, reducer(g, EPI_STORE, S_TMP), st);  // (z, a) of the last a
      launch_fcg_beta(g->scal, first, st);
      launch_p_update(g->scal, p, z, n, st);                             // p = beta p + z
      const Reduce Rl = reducer(g, EPI_CG_LAMBDA, 0);
      launch_spmv(T, p, nullptr, a, p, &Rl, st);                         // a = A p; (a, p); lam
      const Reduce Rr = reducer(g, EPI_STORE, S_RR);
      launch_cg_update(g->scal, x, p, r, a, nullptr, nullptr, nullptr, n, Rr, st);  // x, r; (r, r)
      if ((rc = launched(c, "mixed step (vector form)"))) return rc;
      if ((rc = read_scalars(g))) return rc;
      first = false;
      ++iters;
      ++step;
      const double rn = std::sqrt(c->host_scal[S_RR]);
      if (!std::isfinite(rn)) return set_err(c, FMG_ERR_NUMERIC, "residual is %g at step %d", rn, step);
      if (hist && step < hist_len) hist[step] = rn;
      if ((cf.rtol > 0 && rn / initial < cf.rtol) || (cf.atol > 0 && rn < cf.atol)) { converged = true; break; }
      if (judge_active && rn > 100.0 * dn) {
        for (Lvl& Lh : g->lev) { hidden.push_back(Lh.omega); Lh.omega = nullptr; }
        judge_active = false;
        g->reverts += 1;
        break;
      }
    }
    if (!converged && iters > cf.maxsteps) {
      *ninner = iters;
      break;
    }
    ++step;  // the true-residual check takes one history slot
  }
  FMG_CK(c, cudaStreamSynchronize(st));
  if (!hidden.empty())
    for (size_t l = 0; l < g->lev.size(); ++l) g->lev[l].omega = hidden[l];
  return launched(c, "solve_mixed (vector form)");
}

extern "C" int fmg_solve_mixed(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mcfg, fmg_vec* xv,
                               double* hist, int hist_len, int* nouter, int* ninner, int* status) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (!mcfg || vec_check(xv, g, g->top) || !nouter || !ninner || !status) return FMG_ERR_ARG;
  if (g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "mixed solve: structured grids");
  if (cfg->fmg) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "mixed solve: V/W cycles (fmg = 0)");
  if (cfg->smoother != FMG_JACOBI || cfg->combination != FMG_MULTIPLICATIVE || cfg->gamma != 1 ||
      g->base >= g->top || cfg->post_steps < 1)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED,
                   "mixed solve: Jacobi V(pre,post>=1) cycles with gamma 1 and at least two levels");
  if (g->nc == 3) return solve_mixed_vec(g, cfg, mcfg, xv, hist, hist_len, nouter, ninner, status);
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  if ((rc = mixed_prepare(g, mcfg->matrix_free != 0))) return rc;
  MixedState& X = *g->mx;
  MixedMG mg{g, X, *cfg, st};
  mg.prepare_wd();
  const LevelView T = view(g, g->top);
  const long long n = T.N;
  const double* b = g->rhs;
  // the CG's vectors: padded with the matrix-free top level (its kernels take
  // them by tensor copy; the iterate is copied in here and back at the end),
  // the solvers' natural ones otherwise
  double* x = xv->d;
  if (X.mf) {
    mx_f64_copy_lay(xv->d, X.x64, X.lay, (int)T.M, st);
    x = X.x64;
  }
  double *r = X.mf ? X.r64 : g->r, *a = X.mf ? X.a64 : g->a;
  const long long nv = X.mf ? X.lay.total : n;  // elements of the top-level vectors, padding included
  float* p = X.p32;
  *status = 1;
  *nouter = 0;
  *ninner = 0;
  const int max_restart = mcfg->max_outer > 0 ? mcfg->max_outer : 20;
  bool judge_active = g->learned, revert_restart = false;
  // the in-solve judge: some level carries node damping and judged steps are asked for
  bool shadow = false;
  if (mcfg->judge > 0)
    for (const auto& V : X.lv) shadow = shadow || V.om != nullptr;
  if (shadow && !g->w) return set_err(c, FMG_ERR_STATE, "solve_mixed: work vectors missing");
  double initial = -1.0;
  int step = 0, iters = 0;  // history slots, CG iterations
  for (int restart = 0; restart <= max_restart; ++restart) {
    // true FP64 residual (x = 0: r = b exactly), from the cell coefficients
    // where the top level is matrix-free, else with the assembled matrix
    if (restart == 0 && g->x_zero) {
      if (X.mf) mx_f64_copy_lay(b, r, X.lay, (int)T.M, st);
      else launch_copy(b, r, n, st);
    } else if (mg.top_mf()) {
      MFArgs64 m = mf64_args(g, cfg->damp);
      m.xl = m.yl = X.lay;  // x and r padded, b the grid's natural rhs
      mx_top_residual64(m, x, b, r, st);
    } else {
      launch_spmv(T, x, b, r, nullptr, nullptr, st);
    }
    launch_dot(r, r, nv, reducer(g, EPI_STORE, S_RR), st);
    if ((rc = read_scalars(g))) return rc;
    const double dn = std::sqrt(c->host_scal[S_RR]);
    if (!std::isfinite(dn)) return set_err(c, FMG_ERR_NUMERIC, "defnorm is %g", dn);
    if (initial < 0) initial = dn;
    if (hist && step < hist_len) hist[step] = dn;
    *nouter = restart;
    *ninner = iters;
    if ((cfg->rtol > 0 && (initial == 0.0 || dn / initial < cfg->rtol)) || (cfg->atol > 0 && dn < cfg->atol)) {
      *status = 0;
      break;
    }
    if (restart == max_restart || iters > cfg->maxsteps) break;
    // start: r32 = r / |r|, z = M r, p = z
    if ((rc = mx_set_scalar(g, M_SCALE, dn > 0 ? 1.0 / dn : 1.0))) return rc;
    if ((rc = mx_set_scalar(g, M_SUSED, dn > 0 ? 1.0 / dn : 1.0))) return rc;
    if ((rc = mx_set_scalar(g, M_SINV, dn > 0 ? dn : 1.0))) return rc;
    mx_scale_to32(r, X.sc, M_SCALE, X.r, X.mf ? nv : T.Np, st);
    {
      const Reduce2 Rr = red2(X, EPI2_RHO, 0, 0);
      mg.vcycle(g->top, X.r, &X.q, &X.qs, r, nullptr, &Rr);
      mx_fcg64_p(X.sc, p, X.q, nv, true, st);
    }
    bool converged = false;
    const int it0 = iters;
    revert_restart = false;
    // one CG step after the first: z = M r with (z, r) and (z, a), p = z/s + beta p,
    // a = A p with (a, p), x += lam p, r -= lam a with (r, r), scalars to the host
    auto step_body = [&]() {
      const Reduce2 Rf = red2(X, EPI2_FCG, 0, 0);
      mg.vcycle(g->top, X.r, &X.q, &X.qs, r, a, &Rf);
      mx_fcg64_p(X.sc, p, X.q, nv, false, st);
      mg.matvec64(p, a, red2(X, EPI2_LAMBDA, 0, 0));
      mx_fcg64_update(X.sc, x, p, r, a, X.r, X.mf ? nv : T.Np, red2(X, EPI2_UPDATE, 0, 0), st);
      cudaMemcpyAsync(X.host, X.sc, M_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st);
    };
    while (iters <= cfg->maxsteps) {
      if (iters == it0) {
        mg.matvec64(p, a, red2(X, EPI2_LAMBDA, 0, 0));
        mx_fcg64_update(X.sc, x, p, r, a, X.r, X.mf ? nv : T.Np, red2(X, EPI2_UPDATE, 0, 0), st);
        if ((rc = launched(c, "mixed step"))) return rc;
        if ((rc = mx_read(g))) return rc;
      } else if (shadow && iters - it0 <= mcfg->judge) {
        // a judged step: the learned cycle (the step's own, with its FCG dots)
        // and the plain cycle on the same residual, each direction scored by
        // the energy decrease (z, r)^2 / (z, A z) of a step along it
        // (z, r) of each comes from its cycle's fused reduction: the learned
        // one's as rho = (z, r) / s (s the residual's scale), the plain one's raw
        const Reduce2 Rf = red2(X, EPI2_FCG, 0, 0);
        mg.vcycle(g->top, X.r, &X.q, &X.qs, r, a, &Rf);
        mg.matvec64(X.q, g->w, red2(X, EPI2_STORE, M_ZAL, M_TMP));
        std::vector<const float*> om(X.lv.size());
        for (size_t l = 0; l < X.lv.size(); ++l) { om[l] = X.lv[l].om; X.lv[l].om = nullptr; }
        const Reduce2 Rp = red2(X, EPI2_STORE, M_ZRP, M_TMP);
        mg.vcycle(g->top, X.r, &X.zp, &X.zs, r, nullptr, &Rp);
        for (size_t l = 0; l < X.lv.size(); ++l) X.lv[l].om = om[l];
        mg.matvec64(X.zp, g->w, red2(X, EPI2_STORE, M_ZAP, M_TMP));
        if ((rc = launched(c, "judged step"))) return rc;
        if ((rc = mx_read(g))) return rc;
        const double zrl = X.host[M_ALPHA] * X.host[M_SUSED];
        const double el = zrl * zrl / X.host[M_ZAL];
        const double ep = X.host[M_ZRP] * X.host[M_ZRP] / X.host[M_ZAP];
        g->rho_learned = el;
        g->rho_plain = ep;
        if (!(el >= ep)) {  // the plain cycle does better (or the learned figure is not finite)
          for (auto& V : X.lv) V.om = nullptr;
          mg.prepare_wd();
          judge_active = false;
          shadow = false;
          g->reverts += 1;
          revert_restart = true;
          break;
        }
        mx_fcg64_p(X.sc, p, X.q, nv, false, st);
        mg.matvec64(p, a, red2(X, EPI2_LAMBDA, 0, 0));
        mx_fcg64_update(X.sc, x, p, r, a, X.r, X.mf ? nv : T.Np, red2(X, EPI2_UPDATE, 0, 0), st);
        if ((rc = launched(c, "mixed step"))) return rc;
        if ((rc = mx_read(g))) return rc;
      } else {
        if ((rc = run_step_graph(g, *cfg, x, step_body))) return rc;
        FMG_CK(c, cudaStreamSynchronize(st));
      }
      ++step;
      ++iters;
      const double rn = std::sqrt(X.host[M_RR]);
      if (!std::isfinite(rn)) return set_err(c, FMG_ERR_NUMERIC, "residual is %g at step %d", rn, step);
      if (hist && step < hist_len) hist[step] = rn;
      // the learned cycles as they run: CG residual norms are not monotone
      // (they may grow for several steps under strong coefficient jumps), so
      // only divergence -- 100x the run's initial true residual -- drops the
      // node damping; the flexible CG then restarts from the true residual
      if (judge_active && iters > it0 && rn > 100.0 * dn) {
        for (auto& V : X.lv) V.om = nullptr;  // plain damping for the rest of the solve
        mg.prepare_wd();
        judge_active = false;
        g->reverts += 1;
        revert_restart = true;
      }
      if ((cfg->rtol > 0 && rn / initial < cfg->rtol) || (cfg->atol > 0 && rn < cfg->atol)) { converged = true; break; }
      if (revert_restart) break;
    }
    if (!converged && iters > cfg->maxsteps) {
      *ninner = iters;
      break;
    }
    ++step;  // the true-residual check occupies one history slot
  }
  if (X.mf) mx_f64_from_lay(X.x64, X.lay, xv->d, (int)T.M, st);
  FMG_CK(c, cudaStreamSynchronize(st));
  return launched(c, "solve_mixed");
}


// The measurement hook over the mixed solve's top-level kernels: `reps`
// launches of one of them on the buffers the last matrix-free mixed solve of
// this grid left (FP32 cycle vectors, the FP32 search direction, the FP64
// residual and a = A p), with the damping it formed the per-node
// damping/diagonal for.  Nothing waits; the caller times the stream.
extern "C" int fmg_matvec_mf(fmg_grid* g, int fp32, const fmg_vec* x, const fmg_vec* b, fmg_vec* y) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !g->assembled) return g ? set_err(g->ctx, FMG_ERR_STATE, "not assembled") : FMG_ERR_ARG;
  if (vec_check(x, g, g->top) || vec_check(y, g, g->top) || x == y || (b && (vec_check(b, g, g->top) || b == y)))
    return FMG_ERR_ARG;
  if (!mixed_top_mf(g, true) || g->algebraic)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED,
                   "matvec_mf: 3D scalar Q1 grids with cell-wise coefficients (no uploaded matrices)");
  if (fp32 < 0 || fp32 > 2 || (fp32 == 2 && b)) return FMG_ERR_ARG;
  cudaStream_t st = g->ctx->stream;
  if (fp32 == 0) {
    const MFArgs64 a = mf64_args(g, 0.0);
    if (b) mx_top_residual64(a, x->d, b->d, y->d, st);
    else mx_top_apply64x(a, x->d, y->d, st);
  } else if (fp32 == 2) {  // the CG operator of the mixed solve: FP64 A of an FP32 direction
    int rc = mixed_prepare(g, true);
    if (rc) return rc;
    MixedState& X = *g->mx;
    mx_f64_to_f32_lay(x->d, X.q, X.lay, (int)g->lev[g->top].M, st);
    MFArgs64 m = mf64_args(g, 0.0);
    m.xl = X.lay;
    mx_top_apply64(m, X.q, y->d, X.q, nullptr, st);
  } else {
    int rc = mixed_prepare(g, true);
    if (rc) return rc;
    MixedState& X = *g->mx;
    const long long n = g->lev[g->top].N;
    fmg_solve_cfg c{};
    c.damp = 1.0;
    MixedMG mg{g, X, c, st};
    const int M = (int)g->lev[g->top].M;
    mx_f64_to_f32_lay(x->d, X.q, X.lay, M, st);
    if (b) mx_f64_to_f32_lay(b->d, X.r, X.lay, M, st);
    MFArgs a = mg.mf_args();
    a.yl = natural_lay(M, 3);
    mx_top_apply(b ? 1 : 0, a, X.q, b ? X.r : nullptr, X.qs, nullptr, nullptr, nullptr, st);
    mx_f32_to_f64(X.qs, y->d, n, st);
  }
  FMG_RC(launched(g->ctx, "matvec_mf"));
  return read_scalars(g);  // reports a kernel that gave up waiting for a copy
}

extern "C" int fmg_mixed_top_kernel(fmg_grid* g, int kind, int reps) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g) return FMG_ERR_ARG;
  if (!g->mx || !g->mx->mf || !g->mx->wd_ok || !g->mx->r64 || !g->mx->a64)
    return set_err(g->ctx, FMG_ERR_STATE, "fmg_mixed_top_kernel: no matrix-free mixed solve has run on this grid");
  if (reps < 1 || kind < FMG_MXK_RESIDUAL || kind > FMG_MXK_PRESMOOTH)
    return set_err(g->ctx, FMG_ERR_ARG, "fmg_mixed_top_kernel: kind %d, reps %d", kind, reps);
  MixedState& X = *g->mx;
  fmg_solve_cfg c{};
  c.damp = (double)X.wd_w;
  c.pre_steps = c.post_steps = c.gamma = 1;
  MixedMG mg{g, X, c, g->ctx->stream};
  const Reduce2 R = red2(X, EPI2_STORE, M_TMP, M_TMP);
  for (int k = 0; k < reps; ++k) {
    if (kind == FMG_MXK_RESIDUAL) mg.apply(g->top, 1, X.q, X.r, false, X.rtop, false, nullptr, nullptr, nullptr);
    else if (kind == FMG_MXK_SMOOTH) mg.apply(g->top, 2, X.q, X.r, false, X.qs, false, X.r64, X.a64, &R);
    else if (kind == FMG_MXK_MATVEC64) mg.matvec64(X.p32, X.a64, R);
    else if (kind == FMG_MXK_RESTRICT)
      mx_restrict(X.lv[g->top], X.lv[g->top - 1], X.rtop, false, X.bc[g->top - 1], X.x0[g->top - 1], g->ctx->stream);
    else if (kind == FMG_MXK_PROLONG)
      mx_prolong(X.lv[g->top - 1], X.lv[g->top], X.x0[g->top - 1], X.q, g->ctx->stream, &X.lay);
    else mg.apply(g->top, 3, nullptr, X.r, false, X.q, false, nullptr, nullptr, nullptr);
  }
  return launched(g->ctx, "mixed_top_kernel");
}

// ========================================================= learned damping
// The damping network predicts per-node Jacobi damping for every level above
// the base from the coefficient field; the values become the level's node
// damping (the same storage fmg_set_node_damping writes), used by the FP64
// and the mixed-precision cycles alike.  Training minimises the A-norm error
// contraction of one V-cycle,
//   L = |e3|_A^2 / |e0|_A^2,  e1 = S e0,  e2 = C e1,  e3 = S e2,
//   S = I - diag(w) D^-1 A (one damped Jacobi sweep),
//   C = I - P M R A (coarse-grid correction, M the V-cycle of the level below),
// on errors e0 that the multigrid itself produces (random vectors after k
// cycles of A e = 0 with the current damping).  With M symmetric (Jacobi pre- and post-smoothing
// with equal damping, exact coarsest solve) and R = P^T the gradient is
//   g3 = 2 A e3 / |e0|_A^2
//   dL/dw += -g3 .* (D^-1 A e2)
//   g2 = g3 - A D^-1 (w .* g3)          (S^T g3)
//   g1 = g2 - A P M R g2                (C^T g2)
//   dL/dw += -g1 .* (D^-1 A e0)
namespace {

constexpr int S_LOSS = 10, S_E0 = 11, S_E3 = 12;  // grid scalar slots used by the training loss

unsigned long long splitmix(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// He-uniform weights, zero hidden biases, output bias giving omega = 0.6
void net_init_params(std::vector<float>& p, const NetLayout& L, float omin, float omax, unsigned long long seed) {
  p.assign((size_t)L.n, 0.f);
  unsigned long long s = seed ^ 0x5DEECE66Dull;
  auto uni = [&](float a) { return a * (float)((double)(splitmix(s) >> 11) * (2.0 / 9007199254740992.0) - 1.0); };
  const int nin = 2 << L.dim;  // features actually present in the 16 input channels
  const float a1 = std::sqrt(6.f / (float)(L.taps * nin)), a2 = std::sqrt(6.f / (float)(L.taps * kNetHid));
  for (long long i = 0; i < (long long)L.taps * kNetHid * kNetIn; ++i) p[L.w1 + i] = uni(a1);
  for (long long i = 0; i < (long long)L.taps * kNetHid * kNetHid; ++i) p[L.w2 + i] = uni(a2);
  for (long long i = 0; i < (long long)L.taps * kNetHid; ++i) p[L.w3 + i] = 0.1f * uni(a2);
  const double f = (0.6 - omin) / (omax - omin);
  p[L.b3] = (float)std::log(f / (1.0 - f));
}

int net_upload(fmg_net* net, const float* host) {
  fmg_ctx* c = net->ctx;
  FMG_CK(c, cudaMemcpyAsync(net->P, host, (size_t)net->lay.n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  net->weights_stale = true;
  return FMG_OK;
}

void net_release(fmg_net* net) {
  fmg_ctx* c = net->ctx;
  cudaStreamSynchronize(c->stream);
  net_free_all(net);
  delete net;
  c->grids -= 1;
  if (c->closed && c->grids == 0) ctx_release(c);
}

int net_grid_check(fmg_net* net, fmg_grid* g) {
  if (!net || !g) return FMG_ERR_ARG;
  if (g->ctx != net->ctx) return set_err(g->ctx, FMG_ERR_ARG, "net and grid belong to different contexts");
  if (g->dim != net->dim) return set_err(g->ctx, FMG_ERR_ARG, "net is %dD, grid %dD", net->dim, g->dim);
  if (!((g->order == 1 && g->nc == 1) || (g->order == 2 && g->nc == 3 && g->dim == 3)))
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "damping network: scalar Q1 levels or 3D Q2 elasticity");
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  return FMG_OK;
}

// features + forward pass on level l; writes the level's node damping.
// with_mean: first (re)compute the mean log k over the top level's cells,
// which every level's features are centred by
int net_level_forward(fmg_net* net, fmg_grid* g, int l, bool with_mean) {
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  int rc;
  Lvl& L = g->lev[l];
  const Lvl& T = g->lev[g->top];
  if ((rc = net_reserve(net, act_geom(g->dim, (int)T.M, 1)))) return set_err(c, rc, "damping network: no memory");
  if (!L.omega && (rc = dalloc(g, &L.omega, L.Np))) return rc;
  long long ncell_top = 1;
  for (int k = 0; k < g->dim; ++k) ncell_top *= T.n;
  const bool kc = g->kkind == FMG_K_CELL;
  if (with_mean) {
    if (kc) {
      if ((rc = launch_logmean(net, g->kcell_d, ncell_top, net->stat, st)))
        return set_err(c, rc, "damping network: no memory");
    } else {
      net->lraw_n = 0;
      launch_set_scalar(net->stat, std::log(g->kconst), st);
    }
  }
  const ActGeom ag = act_geom(g->dim, (int)L.M, 1);
  if ((rc = launch_features(net, ag, (int)L.n, g->order, T.n, std::ldexp(1.0, g->top - l), g->np, g->xi_d,
                            kc ? g->kcell_d : nullptr, g->kconst, net->stat, st)))
    return set_err(c, rc, "damping network: no memory");
  if ((rc = net_forward(net, ag, L.omega, st))) return set_err(c, rc, "damping network forward failed");
  return launched(c, "damping network forward");
}

int net_finish(fmg_net* net) {
  const char* msg = nullptr;
  int rc = net_check_error(net, net->ctx->stream, &msg);
  if (rc) return set_err(net->ctx, rc, "%s", msg);
  return FMG_OK;
}

int learn_vectors(fmg_grid* g) {
  if (g->lt[0]) return FMG_OK;
  int rc;
  for (double*& v : g->lt)
    if ((rc = dalloc(g, &v, g->lev[g->top].Np * g->nc))) return rc;
  return FMG_OK;
}

// M R y on the level below the top (result in that level's solution vector)
void coarse_apply(fmg_grid* g, const fmg_solve_cfg& cf, const double* y, cudaStream_t st) {
  const int t = g->top;
  launch_restrict(view(g, t), view(g, t - 1), y, g->resp[t - 1], g->rhsp[t - 1], g->solp[t - 1], st);
  g->cur = t - 1;
  g->rp[t - 1] = 1;
  MG mg{g, cf, false, st};
  mg.lmgc();
  g->cur = t;
}

// loss of one error sample and its gradient with respect to the top-level
// damping w (device); scal[S_LOSS] (+)= L * weight, gw (+)= weight * dL/dw
void learn_loss_grad(fmg_grid* g, const fmg_solve_cfg& cf, const double* e0, const double* w, double* gw,
                     double weight, bool first, cudaStream_t st) {
  const LevelView T = view(g, g->top);
  const long long n = T.N, Np = T.Np;
  const double* A = T.A;
  const int ce = g->center;
  double *u = g->lt[0], *v0 = g->lt[1], *e1 = g->lt[2], *e2 = g->lt[3], *v2 = g->lt[4], *e3 = g->lt[5],
         *g3 = g->lt[6], *t = g->lt[7], *g2 = g->lt[8], *q = g->lt[9];
  launch_spmv(T, e0, nullptr, u, nullptr, nullptr, st);                     // u = A e0
  launch_dot(e0, u, n, reducer(g, EPI_STORE, S_E0), st);                    // |e0|_A^2
  launch_dinv(A, ce, Np, u, v0, n, st);                                     // v0 = D^-1 A e0
  launch_sub_wv(e0, w, v0, e1, n, st);                                      // e1 = S e0
  launch_spmv(T, e1, nullptr, u, nullptr, nullptr, st);                     // u = A e1
  coarse_apply(g, cf, u, st);
  launch_fill(q, n, 0.0, st);
  launch_prolong(view(g, g->top - 1), T, g->solp[g->top - 1], q, st);      // q = P M R A e1
  launch_sub_wv(e1, nullptr, q, e2, n, st);                                 // e2 = C e1
  launch_spmv(T, e2, nullptr, u, nullptr, nullptr, st);
  launch_dinv(A, ce, Np, u, v2, n, st);                                     // v2 = D^-1 A e2
  launch_sub_wv(e2, w, v2, e3, n, st);                                      // e3 = S e2
  launch_spmv(T, e3, nullptr, u, nullptr, nullptr, st);                     // u = A e3
  launch_dot(e3, u, n, reducer(g, EPI_STORE, S_E3), st);
  launch_ratio_acc(g->scal, S_LOSS, S_E3, S_E0, weight, first, st);
  launch_scale_by(u, 2.0 * weight, g->scal, S_E0, g3, n, st);               // g3
  launch_gomega(g3, v2, gw, !first, n, st);                                 // post-smoother term
  launch_wg_dinv(A, ce, Np, w, g3, t, n, st);                               // t = w g3 / d
  launch_spmv(T, t, g3, g2, nullptr, nullptr, st);                          // g2 = g3 - A t
  coarse_apply(g, cf, g2, st);
  launch_fill(q, n, 0.0, st);
  launch_prolong(view(g, g->top - 1), T, g->solp[g->top - 1], q, st);      // q = P M R g2
  launch_spmv(T, q, g2, t, nullptr, nullptr, st);                           // g1 = g2 - A q
  launch_gomega(t, v0, gw, true, n, st);                                    // pre-smoother term
}

// ---- the V-cycle with the damping of every level differentiated
// The error propagator of the V(1,1) Jacobi cycle is E e0 = e0 - V(A e0),
// with V the cycle applied to a right-hand side from a zero guess:
//   x1 = w .* D^-1 f,  c = V_below(R (f - A x1)),  x2 = x1 + P c,
//   x3 = x2 + w .* D^-1 (f - A x2)            (base level: x = A^-1 f)
// LinV records what its adjoint needs (D^-1 f, D^-1 r2 per level) and runs
// the reverse pass, accumulating dL/dw of every level; it is the same linear
// operator as the multigrid iterator's cycle, written without its residual
// bookkeeping.
enum { LV_F = 0, LV_DF, LV_DR2, LV_X, LV_T1, LV_T2, LV_T3, LV_W, LV_WBAR, LV_COUNT };

int linv_vectors(fmg_grid* g) {
  if (!g->lvv.empty()) return FMG_OK;
  g->lvv.assign(g->lev.size(), std::vector<double*>(LV_COUNT, nullptr));
  int rc;
  for (int l = g->base; l <= g->top; ++l)
    for (int v = 0; v < LV_COUNT; ++v)
      if ((rc = dalloc(g, &g->lvv[l][v], g->lev[l].Np * g->nc))) return rc;
  return FMG_OK;
}

struct LinV {
  fmg_grid* g;
  cudaStream_t st;
  const double* w(int l) const { return g->lev[l].omega ? g->lev[l].omega : g->lvv[l][LV_W]; }
  // x = V_l(f)
  void fwd(int l, const double* f, double* x) {
    std::vector<double*>& V = g->lvv[l];
    const LevelView L = view(g, l);
    const long long n = L.N, nv = L.N * g->nc;
    const bool vec = g->nc == 3;  // D = the 3 x 3 diagonal blocks
    if (l == g->base) {
      launch_copy(f, V[LV_T1], nv, st);
      launch_fill(x, nv, 0.0, st);
      launch_coarse_solve(g->ainvT, g->nbase, 1.0, x, V[LV_T1], st);
      return;
    }
    std::vector<double*>& C = g->lvv[l - 1];
    const LevelView Lc = view(g, l - 1);
    if (vec) {
      launch_bdiag3(L, 0, nullptr, f, V[LV_DF], st);  // D^-1 f
      launch_bdiag3(L, 1, w(l), f, V[LV_X], st);      // x1
    } else {
      launch_dinv(L.A, L.center, L.Np, f, V[LV_DF], n, st);          // D^-1 f
      launch_wg_dinv(L.A, L.center, L.Np, w(l), f, V[LV_X], n, st);  // x1
    }
    launch_spmv(L, V[LV_X], f, V[LV_T1], nullptr, nullptr, st);    // r1 = f - A x1
    launch_restrict(L, Lc, V[LV_T1], C[LV_F], C[LV_T2], C[LV_X], st);
    fwd(l - 1, C[LV_F], C[LV_X]);
    launch_prolong(Lc, L, C[LV_X], V[LV_X], st);                    // x2 = x1 + P c
    launch_spmv(L, V[LV_X], f, V[LV_T1], nullptr, nullptr, st);    // r2 = f - A x2
    if (vec) {
      launch_bdiag3(L, 0, nullptr, V[LV_T1], V[LV_DR2], st);       // D^-1 r2
      launch_xpwv3(V[LV_X], w(l), V[LV_DR2], x, n, st);            // x3
    } else {
      launch_dinv(L.A, L.center, L.Np, V[LV_T1], V[LV_DR2], n, st);  // D^-1 r2
      launch_xpwv(V[LV_X], w(l), V[LV_DR2], x, n, st);               // x3
    }
  }
  // given xbar = dL/dx3 (destroyed), fbar = dL/df; dL/dw added to LV_WBAR
  void bwd(int l, double* xbar, double* fbar) {
    std::vector<double*>& V = g->lvv[l];
    const LevelView L = view(g, l);
    const long long n = L.N, nv = L.N * g->nc;
    const bool vec = g->nc == 3;  // D symmetric 3 x 3 blocks: the adjoint uses the same solves
    if (l == g->base) {  // A symmetric: fbar = A^-1 xbar
      launch_fill(fbar, nv, 0.0, st);
      launch_coarse_solve(g->ainvT, g->nbase, 1.0, fbar, xbar, st);
      return;
    }
    std::vector<double*>& C = g->lvv[l - 1];
    const LevelView Lc = view(g, l - 1);
    if (vec) {
      launch_acc_prod3(V[LV_WBAR], xbar, V[LV_DR2], n, st);
      launch_bdiag3(L, 1, w(l), xbar, V[LV_T1], st);
    } else {
      launch_acc_prod(V[LV_WBAR], xbar, V[LV_DR2], n, st);                 // x3 = x2 + w D^-1 r2
      launch_wg_dinv(L.A, L.center, L.Np, w(l), xbar, V[LV_T1], n, st);    // r2bar
    }
    launch_copy(V[LV_T1], fbar, nv, st);                                 // r2 = f - A x2
    launch_spmv(L, V[LV_T1], xbar, V[LV_T2], nullptr, nullptr, st);      // x2bar = xbar - A r2bar
    launch_restrict(L, Lc, V[LV_T2], C[LV_F], C[LV_T2], C[LV_X], st);    // cbar = R x2bar
    bwd(l - 1, C[LV_F], C[LV_X]);                                        // fcbar
    launch_fill(V[LV_T1], nv, 0.0, st);
    launch_prolong(Lc, L, C[LV_X], V[LV_T1], st);                        // r1bar = P fcbar
    launch_add(V[LV_T1], fbar, nv, st);                                  // r1 = f - A x1
    launch_spmv(L, V[LV_T1], V[LV_T2], V[LV_T3], nullptr, nullptr, st);  // x1bar = x2bar - A r1bar
    if (vec) {
      launch_acc_prod3(V[LV_WBAR], V[LV_T3], V[LV_DF], n, st);
      launch_bdiag3(L, 2, w(l), V[LV_T3], fbar, st);
    } else {
      launch_acc_prod(V[LV_WBAR], V[LV_T3], V[LV_DF], n, st);              // x1 = w D^-1 f
      launch_wg_dinv_acc(L.A, L.center, L.Np, w(l), V[LV_T3], fbar, n, st);
    }
  }
};

// loss of one error sample e0 with the damping of every level, dL/dw of every
// level added (times weight) to the levels' LV_WBAR; scal[S_LOSS] (+)= L * weight
void learn_loss_grad_levels(fmg_grid* g, const fmg_solve_cfg& cf, const double* e0, double weight, bool first,
                            cudaStream_t st) {
  LinV lv{g, st};
  const int t = g->top;
  const LevelView T = view(g, t);
  const long long n = T.N * g->nc;  // vector length
  std::vector<double*>& V = g->lvv[t];
  for (int l = g->base + 1; l <= t; ++l)
    if (!g->lev[l].omega) launch_fill(g->lvv[l][LV_W], g->lev[l].N, cf.damp, st);
  launch_spmv(T, e0, nullptr, V[LV_F], nullptr, nullptr, st);        // f = A e0
  launch_dot(e0, V[LV_F], n, reducer(g, EPI_STORE, S_E0), st);
  double* x3 = g->lt[4];
  lv.fwd(t, V[LV_F], x3);
  double *e3 = g->lt[5], *u3 = g->lt[0], *xbar = g->lt[6], *fbar = g->lt[7];
  launch_sub_wv(e0, nullptr, x3, e3, n, st);                           // e3 = e0 - V(A e0)
  launch_spmv(T, e3, nullptr, u3, nullptr, nullptr, st);
  launch_dot(e3, u3, n, reducer(g, EPI_STORE, S_E3), st);
  launch_ratio_acc(g->scal, S_LOSS, S_E3, S_E0, weight, first, st);
  launch_scale_by(u3, -2.0 * weight, g->scal, S_E0, xbar, n, st);      // dL/dx3 = -2 A e3 / |e0|_A^2
  lv.bwd(t, xbar, fbar);
}

int learn_cfg_check(fmg_grid* g, const fmg_solve_cfg* cf) {
  if (g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "training: structured grids");
  int rc = check_cfg(g, cf);
  if (rc) return rc;
  if (cf->smoother != FMG_JACOBI || cf->combination != FMG_MULTIPLICATIVE || cf->pre_steps != 1 ||
      cf->post_steps != 1 || cf->gamma != 1 || g->top <= g->base || cf->fmg ||
      !((g->nc == 1 && g->order == 1) || (g->nc == 3 && g->order == 2 && g->dim == 3)))
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED,
                   "training loss: Jacobi V(1,1), scalar Q1 or 3D Q2 elasticity, at least two levels");
  return g->assembled ? ensure_top(g) : FMG_OK;  // the FP64 cycles read the top level's matrix
}

}  // namespace

extern "C" {

int fmg_net_create(fmg_ctx* c, int dim, unsigned long long seed, fmg_net** out) {
  if (!c || !out || c->closed) return FMG_ERR_ARG;
  *out = nullptr;
  if (dim != 2 && dim != 3) return set_err(c, FMG_ERR_UNSUPPORTED, "damping network: dim %d (2 or 3)", dim);
  FMG_CK(c, cudaSetDevice(c->device));
  fmg_net* net = new (std::nothrow) fmg_net();
  if (!net) return FMG_ERR_NOMEM;
  net->ctx = c;
  net->dim = dim;
  net->lay = net_layout(dim);
  net->seed = seed;
  net->omega_min = 0.1f;
  net->omega_max = 1.3f;
  c->grids += 1;
  const NetLayout& L = net->lay;
  const size_t T = (size_t)L.taps, nb = sizeof(__nv_bfloat16);
  int rc = FMG_OK;
  if ((rc = net_alloc(net, (void**)&net->P, L.n * sizeof(float))) ||
      (rc = net_alloc(net, (void**)&net->G, L.n * sizeof(float))) ||
      (rc = net_alloc(net, (void**)&net->Mo, L.n * sizeof(float))) ||
      (rc = net_alloc(net, (void**)&net->Vo, L.n * sizeof(float))) ||
      (rc = net_alloc(net, (void**)&net->wf1, T * kNetHid * kNetIn * nb)) ||
      (rc = net_alloc(net, (void**)&net->wf2, T * kNetHid * kNetHid * nb)) ||
      (rc = net_alloc(net, (void**)&net->wf3, T * kNetOut * kNetHid * nb)) ||
      (rc = net_alloc(net, (void**)&net->wb2, T * kNetHid * kNetHid * nb)) ||
      (rc = net_alloc(net, (void**)&net->wb3, T * kNetHid * kNetOut * nb)) ||
      (rc = net_alloc(net, (void**)&net->stat, (8 + kLogSumBlocks) * sizeof(double))) ||
      (rc = net_alloc(net, (void**)&net->err, sizeof(unsigned)))) {
    net_release(net);
    return set_err(c, rc, "damping network: device allocation failed");
  }
  std::vector<float> p;
  net_init_params(p, L, net->omega_min, net->omega_max, seed);
  if ((rc = net_upload(net, p.data()))) {
    net_release(net);
    return rc;
  }
  *out = net;
  return FMG_OK;
}

int fmg_net_destroy(fmg_net* net) {
  if (!net) return FMG_ERR_ARG;
  net_release(net);
  return FMG_OK;
}

long fmg_net_nparams(const fmg_net* net) { return net ? (long)net->lay.n : -1; }

int fmg_net_get_params(fmg_net* net, float* host, long n) {
  if (!net || !host || n != (long)net->lay.n) return FMG_ERR_ARG;
  fmg_ctx* c = net->ctx;
  FMG_CK(c, cudaMemcpyAsync(host, net->P, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  return FMG_OK;
}

int fmg_net_set_params(fmg_net* net, const float* host, long n) {
  if (!net || !host || n != (long)net->lay.n) return FMG_ERR_ARG;
  for (long i = 0; i < n; ++i)
    if (!std::isfinite(host[i])) return set_err(net->ctx, FMG_ERR_NUMERIC, "parameter %ld is not finite", i);
  return net_upload(net, host);
}

int fmg_net_get_grads(fmg_net* net, float* host, long n) {
  if (!net || !host || n != (long)net->lay.n) return FMG_ERR_ARG;
  fmg_ctx* c = net->ctx;
  FMG_CK(c, cudaMemcpyAsync(host, net->G, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  FMG_CK(c, cudaStreamSynchronize(c->stream));
  return FMG_OK;
}

int fmg_net_zero_grads(fmg_net* net) {
  if (!net) return FMG_ERR_ARG;
  FMG_CK(net->ctx, cudaMemsetAsync(net->G, 0, (size_t)net->lay.n * sizeof(float), net->ctx->stream));
  return FMG_OK;
}

int fmg_net_adam(fmg_net* net, double lr, double beta1, double beta2, double eps) {
  if (!net || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0)) return FMG_ERR_ARG;
  launch_adam(net, (float)lr, (float)beta1, (float)beta2, (float)eps, net->ctx->stream);
  return launched(net->ctx, "adam");
}

int fmg_net_damping(fmg_net* net, fmg_grid* g, int level, double* host_omega) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  int rc = net_grid_check(net, g);
  if (rc) return rc;
  if (level <= g->base || level > g->top) return set_err(g->ctx, FMG_ERR_ARG, "level %d has no smoother", level);
  if ((rc = net_level_forward(net, g, level, true))) return rc;
  if ((rc = net_finish(net))) return rc;
  const Lvl& L = g->lev[level];
  if (host_omega) {
    FMG_CK(g->ctx, cudaMemcpyAsync(host_omega, L.omega, L.N * sizeof(double), cudaMemcpyDeviceToHost, g->ctx->stream));
    FMG_CK(g->ctx, cudaStreamSynchronize(g->ctx->stream));
  }
  return FMG_OK;
}

int fmg_net_apply(fmg_net* net, fmg_grid* g) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  int rc = net_grid_check(net, g);
  if (rc) return rc;
  for (int l = g->top; l > g->base; --l)
    if ((rc = net_level_forward(net, g, l, l == g->top))) return rc;
  if ((rc = net_finish(net))) return rc;
  g->learned = true;
  return FMG_OK;
}

int fmg_net_backward(fmg_net* net, fmg_grid* g, int level, const double* host_gomega) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  int rc = net_grid_check(net, g);
  if (rc) return rc;
  if (!host_gomega || level <= g->base || level > g->top) return FMG_ERR_ARG;
  const Lvl& L = g->lev[level];
  const ActGeom ag = act_geom(g->dim, (int)L.M, 1);
  if (!net->have_forward || net->geom.Mx != ag.Mx || net->geom.Mz != ag.Mz || !L.omega)
    return set_err(g->ctx, FMG_ERR_STATE, "backward needs the forward pass of this level (fmg_net_damping)");
  if ((rc = learn_vectors(g))) return rc;
  FMG_CK(g->ctx, cudaMemcpyAsync(g->lt[0], host_gomega, L.N * sizeof(double), cudaMemcpyHostToDevice, g->ctx->stream));
  if ((rc = net_backward(net, g->lt[0], L.omega, g->ctx->stream))) return set_err(g->ctx, rc, "backward failed");
  if ((rc = launched(g->ctx, "damping network backward"))) return rc;
  return net_finish(net);
}

int fmg_learn_loss(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_vec* e0, double* loss, double* host_gomega) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !loss) return FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  int rc = learn_cfg_check(g, cfg);
  if (rc) return rc;
  if (g->nc != 1)  // the top-level form; fmg_learn_loss_levels covers the vector form
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "fmg_learn_loss: scalar grids (use fmg_learn_loss_levels)");
  if (vec_check(e0, g, g->top)) return FMG_ERR_ARG;
  if ((rc = learn_vectors(g))) return rc;
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const Lvl& T = g->lev[g->top];
  // gradient into xs2, damping from the level (or the scalar damping in xs)
  const double* w = T.omega;
  if (!w) {
    launch_fill(g->xs, T.N, cfg->damp, st);
    w = g->xs;
  }
  learn_loss_grad(g, *cfg, e0->d, w, g->xs2, 1.0, true, st);
  if ((rc = launched(c, "learn loss"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  *loss = c->host_scal[S_LOSS];
  if (host_gomega) {
    FMG_CK(c, cudaMemcpyAsync(host_gomega, g->xs2, T.N * sizeof(double), cudaMemcpyDeviceToHost, st));
    FMG_CK(c, cudaStreamSynchronize(st));
  }
  return FMG_OK;
}

// The loss of fmg_learn_loss with the damping of every level differentiated
// through the recorded V-cycle; the gradient with respect to `level`'s node
// damping is returned (N of that level values).
int fmg_learn_loss_levels(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_vec* e0, int level, double* loss,
                          double* host_gomega) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!g || !loss) return FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  int rc = learn_cfg_check(g, cfg);
  if (rc) return rc;
  if (vec_check(e0, g, g->top) || level <= g->base || level > g->top) return FMG_ERR_ARG;
  if ((rc = learn_vectors(g)) || (rc = linv_vectors(g))) return rc;
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  for (int l = g->base + 1; l <= g->top; ++l) launch_fill(g->lvv[l][LV_WBAR], g->lev[l].N, 0.0, st);
  learn_loss_grad_levels(g, *cfg, e0->d, 1.0, true, st);
  if ((rc = launched(c, "learn loss (levels)"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  *loss = c->host_scal[S_LOSS];
  if (host_gomega) {
    FMG_CK(c, cudaMemcpyAsync(host_gomega, g->lvv[level][LV_WBAR], g->lev[level].N * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    FMG_CK(c, cudaStreamSynchronize(st));
  }
  return FMG_OK;
}

// One training step on one grid: forward pass on every level (the net's
// damping everywhere, as at inference), nsamples
// error samples made by the multigrid itself (a random vector after
// max_cycles V-cycles of A e = 0 with the current damping: power iterations
// that turn toward the slowest modes of the cycle), the mean loss and its
// gradient, and the backward pass; gradients are added to the net's
// accumulator (fmg_net_adam applies and clears them).  For CG the rate is set
// by the largest eigenvalue mu of the cycle's error propagator E (symmetric
// and positive semidefinite in the A inner product); on its eigenvector the
// loss is mu^2 and the gradient that of mu^2.
int fmg_learn_step(fmg_net* net, fmg_grid* g, const fmg_solve_cfg* cfg, int nsamples, unsigned long long seed,
                   int max_cycles, double* loss) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  int rc = net_grid_check(net, g);
  if (rc) return rc;
  if ((rc = learn_cfg_check(g, cfg))) return rc;
  if (nsamples < 1 || max_cycles < 0 || !loss) return FMG_ERR_ARG;
  if ((rc = learn_vectors(g)) || (rc = linv_vectors(g))) return rc;
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  for (int l = g->base + 1; l <= g->top; ++l) {
    if ((rc = net_level_forward(net, g, l, l == g->base + 1))) return rc;
    launch_fill(g->lvv[l][LV_WBAR], g->lev[l].N, 0.0, st);
  }
  Lvl& T = g->lev[g->top];
  const long long n = T.N * g->nc;
  double* e = g->xs;
  double* spare = g->w2;
  for (int s = 0; s < nsamples; ++s) {
    launch_rand_fill(e, g->dim, T.M, g->dmask, seed * 1000003ull + (unsigned long long)s, st, g->nc);
    if (max_cycles > 0) {  // power iterations of the current (learned) cycle: A e = 0
      MG mg{g, *cfg, false, st};
      launch_fill(g->q, n, 0.0, st);  // b = 0
      for (int k = 0; k < max_cycles; ++k) {
        launch_spmv(view(g, g->top), e, g->q, g->r, nullptr, nullptr, st);  // r = 0 - A e
        mg.iterate(&e, &spare, g->q, g->r);
      }
    }
    learn_loss_grad_levels(g, *cfg, e, 1.0 / nsamples, s == 0, st);
  }
  if ((rc = launched(c, "learn step"))) return rc;
  // backward through the net of every level (its forward pass recomputed)
  for (int l = g->base + 1; l <= g->top; ++l) {
    if ((rc = net_level_forward(net, g, l, false))) return rc;
    if ((rc = net_backward(net, g->lvv[l][LV_WBAR], g->lev[l].omega, st))) return set_err(c, rc, "backward failed");
  }
  if ((rc = launched(c, "learn backward"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  *loss = c->host_scal[S_LOSS];
  if ((rc = net_finish(net))) return rc;
  if (!std::isfinite(*loss)) return set_err(c, FMG_ERR_NUMERIC, "training loss is %g", *loss);
  return FMG_OK;
}

}  // extern "C"

// ------------------------------------------------ the judge
namespace {

// A-norm contraction |e_k|_A / |e_{k-1}|_A of the FP64 cycle with the damping
// currently installed, after k cycles of A e = 0 from a seeded random vector
int cycle_contraction(fmg_grid* g, const fmg_solve_cfg& cf, int k, unsigned long long seed, double* rho) {
  fmg_ctx* c = g->ctx;
  cudaStream_t st = c->stream;
  const Lvl& T = g->lev[g->top];
  const long long n = T.N * g->nc;
  double* e = g->xs;
  double* spare = g->w2;
  launch_rand_fill(e, g->dim, T.M, g->dmask, seed, st, g->nc);
  launch_fill(g->q, n, 0.0, st);
  MG mg{g, cf, false, st};
  for (int it = 0; it < k; ++it) {
    if (it == k - 1) {
      launch_spmv(view(g, g->top), e, nullptr, g->a, nullptr, nullptr, st);
      launch_dot(e, g->a, n, reducer(g, EPI_STORE, S_E0), st);
    }
    launch_spmv(view(g, g->top), e, g->q, g->r, nullptr, nullptr, st);
    mg.iterate(&e, &spare, g->q, g->r);
  }
  launch_spmv(view(g, g->top), e, nullptr, g->a, nullptr, nullptr, st);
  launch_dot(e, g->a, n, reducer(g, EPI_STORE, S_E3), st);
  int rc;
  if ((rc = launched(c, "judge"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  const double e0 = c->host_scal[S_E0], e1 = c->host_scal[S_E3];
  *rho = (e0 > 0 && std::isfinite(e1)) ? std::sqrt(e1 / e0) : INFINITY;
  return FMG_OK;
}

}  // namespace

extern "C" int fmg_solve(fmg_grid* g, const fmg_solve_cfg* cfg, fmg_vec* xv, double* hist, int hist_len,
                         int* nsteps, int* status);

namespace {

// A-norm error contraction per step of k steps of CG preconditioned by the
// cycle with the damping currently installed, on a manufactured problem:
// x* random (Dirichlet nodes zero), b = A x*, x0 = 0; CG minimises the A-norm
// error, so (|x* - x_k|_A / |x*|_A)^(1/k) ranks preconditioners for CG where
// residual norms (not monotone under strong coefficient jumps) do not
// (mc non-null: the steps are those of fmg_solve_mixed with the mixed cycle)
int cg_probe(fmg_grid* g, const fmg_solve_cfg& cf, const fmg_mixed_cfg* mc, int k, unsigned long long seed,
             double* rho) {
  fmg_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const Lvl& T = g->lev[g->top];
  const LevelView TV = view(g, g->top);
  const long long n = T.N * g->nc;
  double *xs = g->lt[9], *b = g->lt[7], *e = g->lt[6];
  launch_rand_fill(xs, g->dim, T.M, g->dmask, seed, st, g->nc);
  int rc0;
  if (mc && mixed_top_mf(g, mc->matrix_free != 0)) {  // the operator the mixed solve applies
    mx_top_apply64x(mf64_args(g, cf.damp), xs, b, st);
  } else {
    if ((rc0 = ensure_top(g))) return rc0;
    launch_spmv(TV, xs, nullptr, b, nullptr, nullptr, st);
  }
  launch_dot(xs, b, n, reducer(g, EPI_STORE, S_E0), st);
  fmg_solve_cfg c = cf;
  c.rtol = 0.0;
  c.atol = 0.0;
  c.maxsteps = k - 1;  // steps 0 .. k
  fmg_vec x;
  x.g = g;
  x.level = g->top;
  x.n = n;
  x.d = g->lt[8];
  launch_fill(x.d, n, 0.0, st);
  double* rhs = g->rhs;
  const bool learned = g->learned;
  g->rhs = b;
  g->learned = false;
  g->x_zero = true;
  int ns = 0, status = 0, nouter = 0, rc;
  if (mc) {
    fmg_mixed_cfg m = *mc;
    m.max_outer = 1;
    rc = fmg_solve_mixed(g, &c, &m, &x, nullptr, 0, &nouter, &ns, &status);
  } else {
    rc = fmg_solve(g, &c, &x, nullptr, 0, &ns, &status);
  }
  g->rhs = rhs;
  g->learned = learned;
  g->x_zero = false;
  if (rc) return rc;
  // |e_k|_A^2 = e_k . A e_k with A e_k = b - A x_k, the solve's FP64 residual
  // (the matrix-free mixed solve leaves it padded: brought to g->r first)
  launch_sub_wv(xs, nullptr, x.d, e, n, st);
  if (mc && g->mx && g->mx->mf) mx_f64_from_lay(g->mx->r64, g->mx->lay, g->r, (int)T.M, st);
  launch_dot(e, g->r, n, reducer(g, EPI_STORE, S_E3), st);
  if ((rc = launched(ctx, "judge probe"))) return rc;
  if ((rc = read_scalars(g))) return rc;
  const double e0 = ctx->host_scal[S_E0], ek = ctx->host_scal[S_E3];
  *rho = (e0 > 0 && std::isfinite(ek) && ns > 0) ? std::pow(ek / e0, 0.5 / ns) : INFINITY;
  return FMG_OK;
}

}  // namespace

namespace {

// The plain <geometric-cs> (scalar :damp) judges the learned damping the way
// the cycle will be used.  As a CG preconditioner (cfg->method CG+MG): 6 CG
// steps with each on the same manufactured problem, the per-step A-norm error
// contractions compared.  As the iteration (MG): both cycles run 8 times on
// A e = 0 from the same random vector, the last-cycle A-norm contractions
// compared.  The learned damping stays installed only if its figure is at
// least 2 % below the plain cycle's; otherwise it is removed (the fallback).
// The plain cycle's figure is also the bound of the judge inside fmg_solve's
// MG iteration.  mc non-null: the CG steps are fmg_solve_mixed's (the FP32 /
// BF16 cycle with the same damping) -- the cycle the mixed solve will use,
// at a third of the FP64 cycle's cost.
constexpr double kJudgeMargin = 0.98;
int learned_judge(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mc, double* rho_plain,
                  double* rho_learned, int* accepted) {
  if (!g || !accepted) return FMG_ERR_ARG;
  if (!g->assembled) return set_err(g->ctx, FMG_ERR_STATE, "not assembled");
  if (g->algebraic) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "judge: structured grids");
  int rc = check_cfg(g, cfg);
  if (rc) return rc;
  if (cfg->smoother != FMG_JACOBI || g->top <= g->base)
    return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "judge: Jacobi cycles with at least two levels");
  const bool cg = cfg->method == FMG_METHOD_CG_MG;
  if (mc && !cg) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "mixed judge: the CG+MG method only");
  bool any = false;
  for (int l = g->base + 1; l <= g->top; ++l) any = any || g->lev[l].omega;
  if (!any) return set_err(g->ctx, FMG_ERR_STATE, "no node damping installed");
  if (!(mc && mixed_top_mf(g, mc->matrix_free != 0)) && (rc = ensure_top(g))) return rc;
  if ((rc = learn_vectors(g))) return rc;
  auto figure = [&](double* rho) {
    return cg ? cg_probe(g, *cfg, mc, 6, 0x4A554447ull, rho) : cycle_contraction(g, *cfg, 8, 0x4A554447ull, rho);
  };
  std::vector<double*> saved(g->lev.size());
  for (size_t l = 0; l < g->lev.size(); ++l) { saved[l] = g->lev[l].omega; g->lev[l].omega = nullptr; }
  double rp = 0, rl = 0;
  rc = figure(&rp);
  for (size_t l = 0; l < g->lev.size(); ++l) g->lev[l].omega = saved[l];
  if (rc || (rc = figure(&rl))) return rc;
  g->rho_plain = rp;
  g->rho_learned = rl;
  const bool ok = rl <= kJudgeMargin * rp;
  if (!ok) {  // fall back to the plain cycle
    cudaStreamSynchronize(g->ctx->stream);
    for (int l = g->base + 1; l <= g->top; ++l) {
      dfree(g, g->lev[l].omega);
      g->lev[l].omega = nullptr;
    }
  }
  g->learned = ok;
  if (rho_plain) *rho_plain = rp;
  if (rho_learned) *rho_learned = rl;
  *accepted = ok ? 1 : 0;
  return FMG_OK;
}

}  // namespace

extern "C" {

int fmg_learned_judge(fmg_grid* g, const fmg_solve_cfg* cfg, double* rho_plain, double* rho_learned, int* accepted) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  return learned_judge(g, cfg, nullptr, rho_plain, rho_learned, accepted);
}

int fmg_learned_judge_mixed(fmg_grid* g, const fmg_solve_cfg* cfg, const fmg_mixed_cfg* mcfg, double* rho_plain,
                            double* rho_learned, int* accepted) {
  if (g && g->nb > 1) return set_err(g->ctx, FMG_ERR_UNSUPPORTED, "%s: not on a batch", __func__);
  if (!mcfg) return FMG_ERR_ARG;
  return learned_judge(g, cfg, mcfg, rho_plain, rho_learned, accepted);
}

int fmg_learned_status(const fmg_grid* g, int* active, double* rho_plain, double* rho_learned, int* reverts) {
  if (!g) return FMG_ERR_ARG;
  if (active) *active = g->learned ? 1 : 0;
  if (rho_plain) *rho_plain = g->rho_plain;
  if (rho_learned) *rho_learned = g->rho_learned;
  if (reverts) *reverts = g->reverts;
  return FMG_OK;
}

}  // extern "C"

// ------------------------------------------------ weight files
// Layout (little endian): "FMGDNET1", u32 version (1), u32 dim, u64 nparams,
// f32 omega_min, f32 omega_max, u64 seed, u64 optimiser steps, f32 params[],
// then the FNV-1a 64 hash of every preceding byte.
namespace {

constexpr char kNetMagic[8] = {'F', 'M', 'G', 'D', 'N', 'E', 'T', '1'};

uint64_t fnv1a(const unsigned char* p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) { h ^= p[i]; h *= 1099511628211ull; }
  return h;
}

template <typename T>
void put(std::vector<unsigned char>& b, const T& v) {
  const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
  b.insert(b.end(), p, p + sizeof(T));
}

template <typename T>
T get(const unsigned char* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}

}  // namespace

extern "C" {

int fmg_net_save(fmg_net* net, const char* path) {
  if (!net || !path) return FMG_ERR_ARG;
  std::vector<float> p((size_t)net->lay.n);
  int rc = fmg_net_get_params(net, p.data(), (long)p.size());
  if (rc) return rc;
  std::vector<unsigned char> b(kNetMagic, kNetMagic + 8);
  put<uint32_t>(b, 1u);
  put<uint32_t>(b, (uint32_t)net->dim);
  put<uint64_t>(b, (uint64_t)net->lay.n);
  put<float>(b, net->omega_min);
  put<float>(b, net->omega_max);
  put<uint64_t>(b, (uint64_t)net->seed);
  put<uint64_t>(b, (uint64_t)net->adam_t);
  const unsigned char* pp = reinterpret_cast<const unsigned char*>(p.data());
  b.insert(b.end(), pp, pp + p.size() * sizeof(float));
  put<uint64_t>(b, fnv1a(b.data(), b.size()));
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_err(net->ctx, FMG_ERR_IO, "cannot write %s", path);
  const size_t w = std::fwrite(b.data(), 1, b.size(), f);
  const int cl = std::fclose(f);
  if (w != b.size() || cl != 0) return set_err(net->ctx, FMG_ERR_IO, "short write to %s", path);
  return FMG_OK;
}

int fmg_net_load(fmg_ctx* c, const char* path, fmg_net** out) {
  if (!c || !path || !out) return FMG_ERR_ARG;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_err(c, FMG_ERR_IO, "cannot read %s", path);
  std::vector<unsigned char> b;
  unsigned char buf[65536];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) {
    b.insert(b.end(), buf, buf + k);
    if (b.size() > ((size_t)64 << 20)) break;
  }
  std::fclose(f);
  const size_t head = 8 + 4 + 4 + 8 + 4 + 4 + 8 + 8;
  if (b.size() < head + 8 || std::memcmp(b.data(), kNetMagic, 8) != 0)
    return set_err(c, FMG_ERR_IO, "%s: not a damping-network file", path);
  if (get<uint64_t>(b.data() + b.size() - 8) != fnv1a(b.data(), b.size() - 8))
    return set_err(c, FMG_ERR_IO, "%s: checksum mismatch (corrupted file)", path);
  const uint32_t ver = get<uint32_t>(b.data() + 8), dim = get<uint32_t>(b.data() + 12);
  const uint64_t n = get<uint64_t>(b.data() + 16);
  if (ver != 1 || (dim != 2 && dim != 3) || n != (uint64_t)net_layout((int)dim).n ||
      b.size() != head + n * sizeof(float) + 8)
    return set_err(c, FMG_ERR_IO, "%s: unsupported version, dimension or size", path);
  const float omin = get<float>(b.data() + 24), omax = get<float>(b.data() + 28);
  if (!(omin > 0.f) || !(omax > omin) || !(omax < 2.f))
    return set_err(c, FMG_ERR_IO, "%s: bad damping range", path);
  fmg_net* net = nullptr;
  int rc = fmg_net_create(c, (int)dim, get<uint64_t>(b.data() + 32), &net);
  if (rc) return rc;
  net->omega_min = omin;
  net->omega_max = omax;
  net->adam_t = (long long)get<uint64_t>(b.data() + 40);
  std::vector<float> p((size_t)n);
  std::memcpy(p.data(), b.data() + head, n * sizeof(float));
  if ((rc = fmg_net_set_params(net, p.data(), (long)n))) {
    fmg_net_destroy(net);
    return rc == FMG_ERR_NUMERIC ? set_err(c, FMG_ERR_IO, "%s: parameters are not finite", path) : rc;
  }
  *out = net;
  return FMG_OK;
}

}  // extern "C"
