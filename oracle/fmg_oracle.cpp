// fmg_oracle.cpp -- CPU restatement of Femlisp's multigrid solve path.
//
// TEST INFRASTRUCTURE ONLY (the checker of the GPU path; see fmg_oracle.h for
// the list of reference files restated and for the canonical arithmetic).
// Build with -ffp-contract=off: every fused multiply-add is an explicit fma().
//
// Structured restatement: Femlisp keys matrix blocks by mesh cells in hash
// tables (sparse-matrix.lisp:703-840).  On a uniformly refined n-cube the
// key <-> index map is fixed (lexicographic node numbering, x fastest), and a
// level matrix is stored by stencil slot: slot s holds A(i, i+off_s) for every
// node i, with zeros where the reference has no block (outside the grid,
// eliminated Dirichlet columns, structurally absent Q2 couplings).
#include "fmg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- reductions
constexpr int DR_LANES = 256, DR_VEC = 2, DR_CHUNK = 4096, DR_M = DR_CHUNK / (DR_LANES * DR_VEC);

// 256 lane sums -> one value: halving 16,8,4,2,1 inside each 32-lane group,
// then halving 4,2,1 over the 8 group sums (the order of a warp butterfly
// followed by a butterfly over the warp sums).
double dr_fold256(double* v) {
  double g[8];
  for (int w = 0; w < 8; ++w) {
    double a[32];
    for (int l = 0; l < 32; ++l) a[l] = v[32 * w + l];
    for (int half = 16; half >= 1; half >>= 1)
      for (int l = 0; l < half; ++l) a[l] = a[l] + a[l + half];
    g[w] = a[0];
  }
  for (int half = 4; half >= 1; half >>= 1)
    for (int l = 0; l < half; ++l) g[l] = g[l] + g[l + half];
  return g[0];
}

double dr_chunk(const double* x, const double* y, long n, long c) {
  double lane[DR_LANES];
  long base = c * DR_CHUNK;
  for (int t = 0; t < DR_LANES; ++t) {
    double acc = 0.0;
    for (int m = 0; m < DR_M; ++m)
      for (int u = 0; u < DR_VEC; ++u) {
        long i = base + DR_VEC * t + (long)DR_LANES * DR_VEC * m + u;
        if (i < n) acc = std::fma(x[i], y[i], acc);
      }
    lane[t] = acc;
  }
  return dr_fold256(lane);
}

double dr_final(const double* part, long P) {
  double lane[DR_LANES];
  for (int t = 0; t < DR_LANES; ++t) {
    double acc = 0.0;
    for (long k = t; k < P; k += DR_LANES) acc = acc + part[k];
    lane[t] = acc;
  }
  return dr_fold256(lane);
}

double dr_dot(const double* x, const double* y, long n, bool par) {
  long P = (n + DR_CHUNK - 1) / DR_CHUNK;
  if (P == 0) return 0.0;
  std::vector<double> part(P);
  if (par) {
#pragma omp parallel for schedule(static)
    for (long c = 0; c < P; ++c) part[c] = dr_chunk(x, y, n, c);
  } else {
    for (long c = 0; c < P; ++c) part[c] = dr_chunk(x, y, n, c);
  }
  return dr_final(part.data(), P);
}

// ---------------------------------------------------------------- FE tables
// Gauss rule with order+1 points per direction on [0,1]
// (fe.lisp:235-244, quadrature.lisp:202-215): xi = (1 - t)/2 for the
// Gauss-Legendre nodes t in ascending order, weight = w_GL / 2.
struct Rule1D {
  int np = 0;
  double xi[3], w[3];
};

Rule1D gauss1d(int order) {
  Rule1D r;
  if (order == 1) {
    double t = std::sqrt(1.0 / 3.0);
    double ts[2] = {-t, t};
    r.np = 2;
    for (int k = 0; k < 2; ++k) { r.xi[k] = 0.5 * (1.0 - ts[k]); r.w[k] = 0.5; }
  } else {
    double t = std::sqrt(0.6);
    double ts[3] = {-t, 0.0, t};
    double wg[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    r.np = 3;
    for (int k = 0; k < 3; ++k) { r.xi[k] = 0.5 * (1.0 - ts[k]); r.w[k] = 0.5 * wg[k]; }
  }
  return r;
}

// 1D Lagrange basis with uniform nodes 0, 1/p, .., 1 (lagrange.lisp:41-51)
double lag1d(int order, int a, double s) {
  if (order == 1) return a == 0 ? 1.0 - s : s;
  if (a == 0) return 2.0 * (s - 0.5) * (s - 1.0);
  if (a == 1) return 4.0 * s * (1.0 - s);
  return 2.0 * s * (s - 0.5);
}
double dlag1d(int order, int a, double s) {
  if (order == 1) return a == 0 ? -1.0 : 1.0;
  if (a == 0) return 4.0 * s - 3.0;
  if (a == 1) return 4.0 - 8.0 * s;
  return 4.0 * s - 1.0;
}

struct Tables {
  int dim = 0, order = 0, nl = 0, nq = 0;
  Rule1D r;
  std::vector<double> C;     // [q][a][b]: (W_q vol) * grad phi_a . grad phi_b
  std::vector<double> Kbar;  // [a][b]: sum_q C
  std::vector<double> Phi;   // [q][a]: (W_q vol) * phi_a
  std::vector<double> G;     // [q][a][3]: grad phi_a at point q
  std::vector<double> Wv;    // [q]: W_q vol
};

Tables make_tables(int dim, int order, double h) {
  Tables T;
  T.dim = dim; T.order = order;
  T.r = gauss1d(order);
  int p1 = order + 1;
  T.nl = 1; T.nq = 1;
  for (int k = 0; k < dim; ++k) { T.nl *= p1; T.nq *= T.r.np; }
  double vol = 1.0;
  for (int k = 0; k < dim; ++k) vol = vol * h;
  double invh = 1.0 / h;
  T.C.assign((size_t)T.nq * T.nl * T.nl, 0.0);
  T.Kbar.assign((size_t)T.nl * T.nl, 0.0);
  T.Phi.assign((size_t)T.nq * T.nl, 0.0);
  for (int q = 0; q < T.nq; ++q) {
    int qi[3] = {q % T.r.np, (q / T.r.np) % T.r.np, q / (T.r.np * T.r.np)};
    double W = 1.0;
    for (int k = 0; k < dim; ++k) W = W * T.r.w[qi[k]];
    double Wv = W * vol;
    std::vector<double> G((size_t)T.nl * 3, 0.0), phi(T.nl);
    for (int a = 0; a < T.nl; ++a) {
      int ai[3] = {a % p1, (a / p1) % p1, a / (p1 * p1)};
      double v = 1.0;
      for (int k = 0; k < dim; ++k) v = v * lag1d(order, ai[k], T.r.xi[qi[k]]);
      phi[a] = v;
      for (int kd = 0; kd < dim; ++kd) {
        double g = 1.0;
        for (int k = 0; k < dim; ++k)
          g = g * (k == kd ? dlag1d(order, ai[k], T.r.xi[qi[k]]) : lag1d(order, ai[k], T.r.xi[qi[k]]));
        G[a * 3 + kd] = g * invh;
      }
    }
    T.Wv.push_back(Wv);
    T.G.insert(T.G.end(), G.begin(), G.end());
    for (int a = 0; a < T.nl; ++a) {
      T.Phi[(size_t)q * T.nl + a] = Wv * phi[a];
      for (int b = 0; b < T.nl; ++b) {
        double g = G[a * 3] * G[b * 3];
        for (int kd = 1; kd < dim; ++kd) g = std::fma(G[a * 3 + kd], G[b * 3 + kd], g);
        T.C[((size_t)q * T.nl + a) * T.nl + b] = Wv * g;
      }
    }
  }
  for (int q = 0; q < T.nq; ++q)
    for (int ab = 0; ab < T.nl * T.nl; ++ab) T.Kbar[ab] = T.Kbar[ab] + T.C[(size_t)q * T.nl * T.nl + ab];
  return T;
}

// Isotropic elasticity with lambda = mu = E (isotropic-elasticity-tensor,
// elasticity.lisp:71-88: A^{kl}_{ij} = lambda d_ik d_jl + mu (d_ij d_kl +
// d_kj d_il)) in the A-term of discretize-locally (ellsys-fe.lisp:120-127,
// block (k,l) += w (G D^{kl}) G^T), per unit E at point q:
//   E_q[a][b][k][l] = (W_q vol) (G_ak G_bl + G_al G_bk + d_kl G_a . G_b)
// formed as t = fma(G_al, G_bk, G_ak * G_bl), t = t + G_a . G_b when k = l,
// with G_a . G_b = fma chain over the directions; Ebar = sum_q E_q.
struct ElasticTables {
  std::vector<double> E;     // [q][a][b][k][l]
  std::vector<double> Ebar;  // [a][b][k][l]
};

ElasticTables make_elastic_tables(const Tables& T) {
  ElasticTables X;
  const int nl = T.nl, nq = T.nq, d = T.dim;
  const size_t per_q = (size_t)nl * nl * d * d;
  X.E.assign(per_q * nq, 0.0);
  X.Ebar.assign(per_q, 0.0);
  for (int q = 0; q < nq; ++q) {
    const double* G = &T.G[(size_t)q * nl * 3];
    for (int a = 0; a < nl; ++a)
      for (int b = 0; b < nl; ++b) {
        double gg = G[a * 3] * G[b * 3];
        for (int kd = 1; kd < d; ++kd) gg = std::fma(G[a * 3 + kd], G[b * 3 + kd], gg);
        for (int k = 0; k < d; ++k)
          for (int l = 0; l < d; ++l) {
            double t = std::fma(G[a * 3 + l], G[b * 3 + k], G[a * 3 + k] * G[b * 3 + l]);
            if (k == l) t = t + gg;
            X.E[(size_t)q * per_q + (((size_t)a * nl + b) * d + k) * d + l] = T.Wv[q] * t;
          }
      }
  }
  for (int q = 0; q < nq; ++q)
    for (size_t e = 0; e < per_q; ++e) X.Ebar[e] = X.Ebar[e] + X.E[(size_t)q * per_q + e];
  return X;
}

// ---------------------------------------------------------------- hierarchy
// compressed rows, columns ascending
struct Csr {
  std::vector<long> start;
  std::vector<int> index;
  std::vector<double> value;
};

struct Level {
  long n = 0, M = 0, N = 0;
  double h = 0;
  std::vector<double> A;        // [slot][node][nc][nc]
  std::vector<double> omega;    // optional per-node damping (size N)
  // algebraic levels: the matrix, its diagonal, the interpolation from the
  // level below (rows of this level) and its transpose (rows of the level below)
  Csr a, p, pt;
  std::vector<double> dg;
  std::vector<int> colour;      // algebraic levels: the greedy colouring of the matrix graph
  int ncol = 0;
};

struct Hier {
  int dim, order, nc, n0, top, base, dmask;
  int span;                     // stencil half width (= order)
  int nslots;
  int kkind = ORA_K_CONST;
  double kconst = 1.0;
  std::vector<double> kcell;    // top-level cells
  int fkind = ORA_F_CONST;
  double fconst = 1.0;
  double fvec[3] = {0.0, 0.0, 0.0};  // ORA_F_VEC: constant force per component
  std::vector<double> fip;      // top-level cells x nq
  std::vector<Level> lev;
  std::vector<double> rhs;
  std::vector<double> ainv;     // base-level inverse, row-major
  long nbase = 0;
  bool assembled = false;
  bool algebraic = false;       // levels without geometry (matrices and interpolations given)

  // V-cycle state (multigrid.lisp:101-116)
  std::vector<double*> sol, rhsv, res;
  std::vector<int> rp;
  std::vector<std::vector<double>> store;
  int cur = 0;
};

inline void coords(const Hier& H, long M, long i, long c[3]) {
  c[0] = i % M; c[1] = H.dim > 1 ? (i / M) % M : 0; c[2] = H.dim > 2 ? i / (M * M) : 0;
}

inline bool is_dirichlet(const Hier& H, long M, const long c[3]) {
  for (int k = 0; k < H.dim; ++k) {
    if (c[k] == 0 && (H.dmask >> (2 * k) & 1)) return true;
    if (c[k] == M - 1 && (H.dmask >> (2 * k + 1) & 1)) return true;
  }
  return false;
}

inline int slot_of(const Hier& H, const long o[3]) {
  int w = 2 * H.span + 1, s = 0, mul = 1;
  for (int k = 0; k < H.dim; ++k) { s += (int)(o[k] + H.span) * mul; mul *= w; }
  return s;
}

inline void slot_offset(const Hier& H, int s, long o[3]) {
  int w = 2 * H.span + 1;
  o[0] = o[1] = o[2] = 0;
  for (int k = 0; k < H.dim; ++k) { o[k] = s % w - H.span; s /= w; }
}

long vec_len(const Hier& H, int l) { return H.lev[l].N * H.nc; }

// coefficient at Gauss point q of cell c on level l (re-discretisation:
// coarse levels evaluate the coefficient at their own integration points,
// ellsys-fe.lisp:102-121, pde-problem.lisp:212-247)
double k_at(const Hier& H, int l, const Tables& T, const long cc[3], int q) {
  if (H.kkind == ORA_K_CONST) return H.kconst;
  long nt = H.lev[H.top].n;
  double r = std::ldexp(1.0, H.top - l);
  int np = T.r.np;
  int qi[3] = {q % np, (q / np) % np, q / (np * np)};
  long f[3] = {0, 0, 0};
  for (int k = 0; k < H.dim; ++k) f[k] = (long)std::floor(((double)cc[k] + T.r.xi[qi[k]]) * r);
  long idx = f[0] + nt * (f[1] + nt * f[2]);
  return H.kcell[idx];
}

int assemble_level_vec(Hier& H, int l);

int assemble_level(Hier& H, int l) {
  Level& L = H.lev[l];
  Tables T = make_tables(H.dim, H.order, L.h);
  const int p = H.order, p1 = p + 1, nl = T.nl, nq = T.nq, nc = H.nc;
  if (nc != 1) return assemble_level_vec(H, l);
  L.A.assign((size_t)H.nslots * L.N, 0.0);
  const bool top = (l == H.top);
  const bool cellconst = (H.kkind == ORA_K_CONST) || top;
  if (top) H.rhs.assign(L.N, 0.0);
  const long n = L.n, M = L.M;
  const int center = [&] { long z[3] = {0, 0, 0}; return slot_of(H, z); }();
#pragma omp parallel for schedule(static)
  for (long i = 0; i < L.N; ++i) {
    long ci[3];
    coords(H, M, i, ci);
    if (is_dirichlet(H, M, ci)) {
      L.A[(size_t)center * L.N + i] = 1.0;
      continue;
    }
    // adjacent cells per direction, ascending
    // cells c with p*c <= i <= p*c + p, clipped to the grid
    long lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < H.dim; ++k) {
      lo[k] = ci[k] >= p ? (ci[k] - 1) / p : 0;
      hi[k] = std::min(n - 1, ci[k] / p);
    }
    double acc_b = 0.0;
    for (long cz = lo[2]; cz <= hi[2]; ++cz)
      for (long cy = lo[1]; cy <= hi[1]; ++cy)
        for (long cx = lo[0]; cx <= hi[0]; ++cx) {
          long cc[3] = {cx, cy, cz};
          long cidx = cx + n * (cy + n * cz);
          int ai[3] = {0, 0, 0};
          for (int k = 0; k < H.dim; ++k) ai[k] = (int)(ci[k] - p * cc[k]);
          int a = ai[0] + p1 * (ai[1] + p1 * ai[2]);
          double kc = 0.0;
          double kq[27];
          if (cellconst) kc = (H.kkind == ORA_K_CONST) ? H.kconst : H.kcell[cidx];
          else
            for (int q = 0; q < nq; ++q) kq[q] = k_at(H, l, T, cc, q);
          for (int b = 0; b < nl; ++b) {
            int bi[3] = {b % p1, (b / p1) % p1, b / (p1 * p1)};
            long cj[3] = {0, 0, 0}, o[3] = {0, 0, 0};
            for (int k = 0; k < H.dim; ++k) { cj[k] = p * cc[k] + bi[k]; o[k] = cj[k] - ci[k]; }
            if (is_dirichlet(H, M, cj)) continue;  // S*A*S: constrained column removed
            double v;
            if (cellconst) v = kc * T.Kbar[(size_t)a * nl + b];
            else {
              v = 0.0;
              for (int q = 0; q < nq; ++q) v = std::fma(kq[q], T.C[((size_t)q * nl + a) * nl + b], v);
            }
            int s = slot_of(H, o);
            double& dst = L.A[(size_t)s * L.N + i];
            dst = dst + v;
          }
          if (top) {
            double bl = 0.0;
            for (int q = 0; q < nq; ++q) {
              double f = (H.fkind == ORA_F_CONST) ? H.fconst : H.fip[(size_t)cidx * nq + q];
              bl = std::fma(f, T.Phi[(size_t)q * nl + a], bl);
            }
            acc_b = acc_b + bl;
          }
        }
    if (top) H.rhs[i] = acc_b;
  }
  return 0;
}

// the vector (nc = dim) elasticity form of assemble_level: the same gather,
// each node pair contributing an nc x nc block; layout [slot][k][l][node],
// the rhs [node][k]
int assemble_level_vec(Hier& H, int l) {
  Level& L = H.lev[l];
  Tables T = make_tables(H.dim, H.order, L.h);
  ElasticTables X = make_elastic_tables(T);
  const int p = H.order, p1 = p + 1, nl = T.nl, nq = T.nq, nc = H.nc;
  if (nc != H.dim) return -2;
  L.A.assign((size_t)H.nslots * nc * nc * L.N, 0.0);
  const bool top = (l == H.top);
  const bool cellconst = (H.kkind == ORA_K_CONST) || top;
  if (top) H.rhs.assign((size_t)L.N * nc, 0.0);
  const long n = L.n, M = L.M, N = L.N;
  const int center = [&] { long z[3] = {0, 0, 0}; return slot_of(H, z); }();
  auto at = [&](int s, int k, int m, long i) -> double& { return L.A[(((size_t)s * nc + k) * nc + m) * N + i]; };
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) {
    long ci[3];
    coords(H, M, i, ci);
    if (is_dirichlet(H, M, ci)) {
      for (int k = 0; k < nc; ++k) at(center, k, k, i) = 1.0;
      continue;
    }
    long lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < H.dim; ++k) {
      lo[k] = ci[k] >= p ? (ci[k] - 1) / p : 0;
      hi[k] = std::min(n - 1, ci[k] / p);
    }
    double acc_b[3] = {0.0, 0.0, 0.0};
    for (long cz = lo[2]; cz <= hi[2]; ++cz)
      for (long cy = lo[1]; cy <= hi[1]; ++cy)
        for (long cx = lo[0]; cx <= hi[0]; ++cx) {
          long cc[3] = {cx, cy, cz};
          long cidx = cx + n * (cy + n * cz);
          int ai[3] = {0, 0, 0};
          for (int k = 0; k < H.dim; ++k) ai[k] = (int)(ci[k] - p * cc[k]);
          int a = ai[0] + p1 * (ai[1] + p1 * ai[2]);
          double kc = 0.0;
          double kq[27];
          if (cellconst) kc = (H.kkind == ORA_K_CONST) ? H.kconst : H.kcell[cidx];
          else
            for (int q = 0; q < nq; ++q) kq[q] = k_at(H, l, T, cc, q);
          for (int b = 0; b < nl; ++b) {
            int bi[3] = {b % p1, (b / p1) % p1, b / (p1 * p1)};
            long cj[3] = {0, 0, 0}, o[3] = {0, 0, 0};
            for (int k = 0; k < H.dim; ++k) { cj[k] = p * cc[k] + bi[k]; o[k] = cj[k] - ci[k]; }
            if (is_dirichlet(H, M, cj)) continue;
            int s = slot_of(H, o);
            for (int k = 0; k < nc; ++k)
              for (int m = 0; m < nc; ++m) {
                const size_t e = (((size_t)a * nl + b) * nc + k) * nc + m;
                double v;
                if (cellconst) v = kc * X.Ebar[e];
                else {
                  v = 0.0;
                  for (int q = 0; q < nq; ++q) v = std::fma(kq[q], X.E[(size_t)q * nl * nl * nc * nc + e], v);
                }
                double& dst = at(s, k, m, i);
                dst = dst + v;
              }
          }
          if (top) {
            for (int k = 0; k < nc; ++k) {
              double bl = 0.0;
              for (int q = 0; q < nq; ++q) {
                double f = (H.fkind == ORA_F_VEC) ? H.fvec[k] : H.fconst;
                bl = std::fma(f, T.Phi[(size_t)q * nl + a], bl);
              }
              acc_b[k] = acc_b[k] + bl;
            }
          }
        }
    if (top)
      for (int k = 0; k < nc; ++k) H.rhs[(size_t)i * nc + k] = acc_b[k];
  }
  return 0;
}

// dense LU with partial pivoting and explicit inverse of the base level
// (replaces the sparse LDU of sparselu.lisp:61-216; both are exact solves)
void build_coarse_inverse(Hier& H) {
  Level& L = H.lev[H.base];
  const int nc = H.nc;
  long n = L.N * nc;
  H.nbase = n;
  std::vector<double> A((size_t)n * n, 0.0);
  if (H.algebraic)
    for (long i = 0; i < L.N; ++i)
      for (long e = L.a.start[i]; e < L.a.start[i + 1]; ++e) A[(size_t)i * n + L.a.index[e]] = L.a.value[e];
  for (long i = 0; i < (H.algebraic ? 0 : L.N); ++i)
    for (int s = 0; s < H.nslots; ++s) {
      long o[3];
      slot_offset(H, s, o);
      long ci[3];
      coords(H, L.M, i, ci);
      long cj[3] = {ci[0] + o[0], ci[1] + o[1], ci[2] + o[2]};
      bool in = true;
      for (int k = 0; k < H.dim; ++k) if (cj[k] < 0 || cj[k] >= L.M) in = false;
      if (!in) continue;
      long j = cj[0] + L.M * (cj[1] + L.M * cj[2]);
      for (int k = 0; k < nc; ++k)
        for (int m = 0; m < nc; ++m)
          A[(size_t)(i * nc + k) * n + (j * nc + m)] = L.A[(((size_t)s * nc + k) * nc + m) * L.N + i];
    }
  std::vector<long> piv(n);
  for (long k = 0; k < n; ++k) {
    long pk = k;
    double mx = std::fabs(A[(size_t)k * n + k]);
    for (long i = k + 1; i < n; ++i) {
      double v = std::fabs(A[(size_t)i * n + k]);
      if (v > mx) { mx = v; pk = i; }
    }
    piv[k] = pk;
    if (pk != k)
      for (long j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)pk * n + j]);
    double d = A[(size_t)k * n + k];
    for (long i = k + 1; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)i * n + k] / d;
    for (long i = k + 1; i < n; ++i) {
      double lik = A[(size_t)i * n + k];
      for (long j = k + 1; j < n; ++j) A[(size_t)i * n + j] = std::fma(-lik, A[(size_t)k * n + j], A[(size_t)i * n + j]);
    }
  }
  H.ainv.assign((size_t)n * n, 0.0);
  std::vector<double> b(n);
  for (long col = 0; col < n; ++col) {
    std::fill(b.begin(), b.end(), 0.0);
    b[col] = 1.0;
    for (long k = 0; k < n; ++k) if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (long k = 0; k < n; ++k)
      for (long i = k + 1; i < n; ++i) b[i] = std::fma(-A[(size_t)i * n + k], b[k], b[i]);
    for (long k = n - 1; k >= 0; --k) {
      b[k] = b[k] / A[(size_t)k * n + k];
      for (long i = 0; i < k; ++i) b[i] = std::fma(-A[(size_t)i * n + k], b[k], b[i]);
    }
    for (long i = 0; i < n; ++i) H.ainv[(size_t)i * n + col] = b[i];
  }
}

// ---------------------------------------------------------------- kernels
inline double row_sum(const Hier& H, const Level& L, long i, const double* x) {
  if (H.algebraic) {  // stored entries, columns ascending
    double acc = 0.0;
    for (long e = L.a.start[i]; e < L.a.start[i + 1]; ++e) acc = std::fma(L.a.value[e], x[L.a.index[e]], acc);
    return acc;
  }
  long ci[3];
  coords(H, L.M, i, ci);
  double acc = 0.0;
  for (int s = 0; s < H.nslots; ++s) {
    long o[3];
    slot_offset(H, s, o);
    bool in = true;
    long cj[3];
    for (int k = 0; k < 3; ++k) {
      cj[k] = ci[k] + o[k];
      if (k < H.dim && (cj[k] < 0 || cj[k] >= L.M)) in = false;
    }
    if (!in) continue;
    long j = cj[0] + L.M * (cj[1] + L.M * cj[2]);
    acc = std::fma(L.A[(size_t)s * L.N + i], x[j], acc);
  }
  return acc;
}

// row (i, k) of a block (nc > 1) level: slots ascending, the nc columns of
// each block ascending: acc = fma(A[s][k][m][i], x[j nc + m], acc)
inline double row_sum_vec(const Hier& H, const Level& L, long i, int k, const double* x) {
  const int nc = H.nc;
  long ci[3];
  coords(H, L.M, i, ci);
  double acc = 0.0;
  for (int s = 0; s < H.nslots; ++s) {
    long o[3];
    slot_offset(H, s, o);
    bool in = true;
    long cj[3];
    for (int kk = 0; kk < 3; ++kk) {
      cj[kk] = ci[kk] + o[kk];
      if (kk < H.dim && (cj[kk] < 0 || cj[kk] >= L.M)) in = false;
    }
    if (!in) continue;
    long j = cj[0] + L.M * (cj[1] + L.M * cj[2]);
    for (int m = 0; m < nc; ++m)
      acc = std::fma(L.A[(((size_t)s * nc + k) * nc + m) * L.N + i], x[j * nc + m], acc);
  }
  return acc;
}

// gemm! 1.0 A x 0.0 y (sparse-matrix.lisp:392-405)
void matvec(const Hier& H, int l, const double* x, double* y) {
  const Level& L = H.lev[l];
  const int nc = H.nc;
  if (nc > 1) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < L.N; ++i)
      for (int k = 0; k < nc; ++k) y[i * nc + k] = row_sum_vec(H, L, i, k, x);
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < L.N; ++i) y[i] = row_sum(H, L, i, x);
}

// compute-residual r := b - A x (linit.lisp:73-80); b may alias r
void residual(const Hier& H, int l, const double* x, const double* b, double* r) {
  const Level& L = H.lev[l];
  const int nc = H.nc;
  if (nc > 1) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < L.N; ++i) {
      double sv[3];
      for (int k = 0; k < nc; ++k) sv[k] = row_sum_vec(H, L, i, k, x);
      for (int k = 0; k < nc; ++k) r[i * nc + k] = b[i * nc + k] - sv[k];
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < L.N; ++i) {
    double s = row_sum(H, L, i, x);
    r[i] = b[i] - s;
  }
}

// t := B^-1 r for one 3 x 3 (nc x nc) diagonal block: LU with partial
// pivoting (first largest |entry| of the column, LAPACK dgetrf semantics)
// and substitution, the operation order fixed as written
void block_solve(const double* Bm, int nc, const double* r, double* t) {
  double M[3][3], b[3];
  for (int k = 0; k < nc; ++k) {
    b[k] = r[k];
    for (int m = 0; m < nc; ++m) M[k][m] = Bm[k * nc + m];
  }
  for (int c = 0; c < nc; ++c) {
    int pr = c;
    double mx = std::fabs(M[c][c]);
    for (int rr = c + 1; rr < nc; ++rr)
      if (std::fabs(M[rr][c]) > mx) { mx = std::fabs(M[rr][c]); pr = rr; }
    if (pr != c) {
      for (int m = 0; m < nc; ++m) std::swap(M[c][m], M[pr][m]);
      std::swap(b[c], b[pr]);
    }
    for (int rr = c + 1; rr < nc; ++rr) {
      const double f = M[rr][c] / M[c][c];
      for (int m = c + 1; m < nc; ++m) M[rr][m] = std::fma(-f, M[c][m], M[rr][m]);
      b[rr] = std::fma(-f, b[c], b[rr]);
    }
  }
  for (int c = nc - 1; c >= 0; --c) {
    double sacc = b[c];
    for (int m = c + 1; m < nc; ++m) sacc = std::fma(-M[c][m], t[m], sacc);
    t[c] = sacc / M[c][c];
  }
}

inline double diag(const Hier& H, const Level& L, long i) {
  if (H.algebraic) return L.dg[i];
  long z[3] = {0, 0, 0};
  return L.A[(size_t)slot_of(H, z) * L.N + i];
}

// <jacobi> on a sparse matrix (linit.lisp:220-250): r_k := A_kk^-1 r_k
// (gesv! overwrites the residual block), x_k += damp * r_k
void jacobi(const Hier& H, int l, double damp, double* x, double* r) {
  const Level& L = H.lev[l];
  const double* w = L.omega.empty() ? nullptr : L.omega.data();
  const int nc = H.nc;
  if (nc > 1) {  // 3 x 3 blocks (linit.lisp:234: gesv! on the diagonal block)
    long z[3] = {0, 0, 0};
    const int center = slot_of(H, z);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < L.N; ++i) {
      double Bm[9], t[3];
      for (int k = 0; k < nc; ++k)
        for (int m = 0; m < nc; ++m) Bm[k * nc + m] = L.A[(((size_t)center * nc + k) * nc + m) * L.N + i];
      block_solve(Bm, nc, r + i * nc, t);
      const double om = w ? w[i] : damp;
      for (int k = 0; k < nc; ++k) {
        r[i * nc + k] = t[k];
        x[i * nc + k] = std::fma(om, t[k], x[i * nc + k]);
      }
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < L.N; ++i) {
    double t = r[i] / diag(H, L, i);
    r[i] = t;
    x[i] = std::fma(w ? w[i] : damp, t, x[i]);
  }
}

int colour_of(const Hier& H, const long c[3]) {
  int p1 = H.order + 1, col = 0, mul = 1;
  for (int k = 0; k < H.dim; ++k) { col += (int)(c[k] % p1) * mul; mul *= p1; }
  return col;
}

// <sor> on a sparse matrix (linit.lisp:288-323), rows ordered by colour
// class (the :compare slot, linit.lisp:260-263,293-295).  Rows of one colour
// do not couple, so the order inside a colour does not matter.
// SOR (ssc = false: r := the scaled correction, linit.lisp:288-323) or the
// one-unknown-block SSC sweep (r := the residual, blockit.lisp:131-138) of
// an algebraic level: colours in order, the row sum over the stored entries
// in their (column-ascending) order
void sor_alg(const Hier& H, int l, double omega, double* x, const double* b, double* r, bool ssc) {
  const Level& L = H.lev[l];
  const double* w = (L.omega.empty() || ssc) ? nullptr : L.omega.data();
  for (int col = 0; col < L.ncol; ++col) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < L.N; ++i) {
      if (L.colour[i] != col) continue;
      double s = 0.0;
      for (long e = L.a.start[i]; e < L.a.start[i + 1]; ++e) s = std::fma(L.a.value[e], x[L.a.index[e]], s);
      const double rr = b[i] - s;
      const double t = rr / L.dg[i];
      r[i] = ssc ? rr : t;
      x[i] = std::fma(w ? w[i] : omega, t, x[i]);
    }
  }
}

void sor(const Hier& H, int l, double omega, double* x, const double* b, double* r) {
  if (H.algebraic) {
    sor_alg(H, l, omega, x, b, r, false);
    return;
  }
  const Level& L = H.lev[l];
  int ncol = 1;
  for (int k = 0; k < H.dim; ++k) ncol *= H.order + 1;
  const double* w = L.omega.empty() ? nullptr : L.omega.data();
  for (int col = 0; col < ncol; ++col) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < L.N; ++i) {
      long ci[3];
      coords(H, L.M, i, ci);
      if (colour_of(H, ci) != col) continue;
      double s = row_sum(H, L, i, x);
      double ri = b[i] - s;
      double t = ri / diag(H, L, i);
      r[i] = t;
      x[i] = std::fma(w ? w[i] : omega, t, x[i]);
    }
  }
}

// <geometric-ssc> with vertex-centred blocks (geoblock.lisp:37-158,
// blockit.lisp:118-204), one sweep.  The block of a vertex is the vertex and
// every non-Dirichlet degree of freedom whose subcell contains it
// (find-vertex-centered-block, geoblock.lisp:72-100): on the structured grid
// the 3^d box of nodes around an even node for Q2, the node alone for Q1.
// For each block in turn: r_k := b_k - sum_j A_kj x_j on its rows (b may be r,
// the alias inside <cg>), the local system A_BB c = r_B solved by LU with
// partial pivoting, x_B += omega c (blockit.lisp:131-180).
// Order: vertices by colour (vertex index mod 2 per direction, colours
// ascending), lexicographic inside a colour; blocks of one colour neither
// share nodes nor read each other's unknowns, so they run in any order.
// The block is kept as the full box: members outside the domain or
// Dirichlet (other than the vertex) become identity rows and zero columns,
// which leaves every pivot choice and every operation on the real rows as in
// the compact block.  LU: right-looking, row interchanges to the first
// position holding the largest magnitude, multipliers scaled by the pivot's
// reciprocal, no fused multiply-adds (the dgetf2 + dgetrs sequence of gesv!).
//
// VBlock / vertex_block: the vertex block's members (the full 3^d box, real
// members marked); vertex_block_solve: c = A_BB^-1 rr by the LU above, rr the
// members' right-hand side on entry (zero for the padded ones), c on return.
struct VBlock {
  int NB;
  long node[27];
  bool real[27];
  long cn[27][3];
};

void vertex_block(const Hier& H, const Level& L, const long v[3], VBlock& B) {
  const int D = H.dim;
  B.NB = H.order == 2 ? (D == 1 ? 3 : D == 2 ? 9 : 27) : 1;
  const int centre = B.NB / 2;
  for (int u = 0; u < B.NB; ++u) {
    int t = u;
    bool in = true;
    for (int k = 0; k < 3; ++k) {
      const long d = (k < D && B.NB > 1) ? (t % 3) - 1 : 0;
      if (k < D && B.NB > 1) t /= 3;
      B.cn[u][k] = v[k] + d;
      if (k < D && (B.cn[u][k] < 0 || B.cn[u][k] >= L.M)) in = false;
    }
    B.real[u] = in && (u == centre || !is_dirichlet(H, L.M, B.cn[u]));
    B.node[u] = in ? B.cn[u][0] + L.M * (B.cn[u][1] + L.M * B.cn[u][2]) : -1;
  }
}

void vertex_block_solve(const Hier& H, const Level& L, const VBlock& B, double* rr) {
  const int NB = B.NB, D = H.dim;
  double a[27][27];
  for (int t = 0; t < NB; ++t) {
    if (!B.real[t]) {
      for (int u = 0; u < NB; ++u) a[t][u] = u == t ? 1.0 : 0.0;
      continue;
    }
    const long i = B.node[t];
    for (int u = 0; u < NB; ++u) {
      if (!B.real[u]) { a[t][u] = 0.0; continue; }
      long o[3] = {0, 0, 0};
      bool near = true;
      for (int k = 0; k < D; ++k) {
        o[k] = B.cn[u][k] - B.cn[t][k];
        if (o[k] < -H.span || o[k] > H.span) near = false;
      }
      a[t][u] = near ? L.A[(size_t)slot_of(H, o) * L.N + i] : 0.0;
    }
  }
  for (int k = 0; k < NB; ++k) {
    int p = k;
    double amax = std::fabs(a[k][k]);
    for (int i = k + 1; i < NB; ++i)
      if (std::fabs(a[i][k]) > amax) { amax = std::fabs(a[i][k]); p = i; }
    if (p != k) {
      for (int j = 0; j < NB; ++j) std::swap(a[k][j], a[p][j]);
      std::swap(rr[k], rr[p]);
    }
    const double rcp = 1.0 / a[k][k];
    for (int i = k + 1; i < NB; ++i) {
      const double m = a[i][k] * rcp;
      a[i][k] = m;
      for (int j = k + 1; j < NB; ++j) a[i][j] = a[i][j] - m * a[k][j];
      rr[i] = rr[i] - m * rr[k];
    }
  }
  for (int k = NB - 1; k >= 0; --k) {
    rr[k] = rr[k] / a[k][k];
    for (int i = 0; i < k; ++i) rr[i] = rr[i] - rr[k] * a[i][k];
  }
}

// <geometric-psc> (geoblock.lisp:43-45, blockit.lisp:118-204 without the
// per-block residual update): every vertex block solves A_BB c_B = r_B with
// the residual r as it was before the sweep (r is not written), and the
// corrections are added in block order, x_B += damp c_B -- overlapping blocks
// sum their corrections (the block loop reads x_B after the earlier blocks
// wrote it).  Order: vertices lexicographic.
void psc(const Hier& H, int l, double damp, double* x, const double* r) {
  const Level& L = H.lev[l];
  const int D = H.dim;
  const long nv = H.order == 2 ? (L.M + 1) / 2 : L.M;
  long nvert = 1;
  for (int k = 0; k < D; ++k) nvert *= nv;
  for (long q = 0; q < nvert; ++q) {
    const long v[3] = {(q % nv) * H.order, D > 1 ? ((q / nv) % nv) * H.order : 0, D > 2 ? (q / (nv * nv)) * H.order : 0};
    VBlock B;
    vertex_block(H, L, v, B);
    double rr[27];
    for (int t = 0; t < B.NB; ++t) rr[t] = B.real[t] ? r[B.node[t]] : 0.0;
    vertex_block_solve(H, L, B, rr);
    for (int u = 0; u < B.NB; ++u)
      if (B.real[u]) x[B.node[u]] = std::fma(damp, rr[u], x[B.node[u]]);
  }
}

void ssc_block(const Hier& H, const Level& L, const long v[3], double omega, double* x, const double* b,
               double* r) {
  VBlock B;
  vertex_block(H, L, v, B);
  double rr[27];
  for (int t = 0; t < B.NB; ++t) {
    rr[t] = 0.0;
    if (!B.real[t]) continue;
    const long i = B.node[t];
    rr[t] = b[i] - row_sum(H, L, i, x);
    r[i] = rr[t];
  }
  vertex_block_solve(H, L, B, rr);
  for (int u = 0; u < B.NB; ++u)
    if (B.real[u]) x[B.node[u]] = std::fma(omega, rr[u], x[B.node[u]]);
}

void ssc(const Hier& H, int l, double omega, double* x, const double* b, double* r) {
  if (H.algebraic) {
    sor_alg(H, l, omega, x, b, r, true);
    return;
  }
  const Level& L = H.lev[l];
  const int D = H.dim;
  const long nv = H.order == 2 ? (L.M + 1) / 2 : L.M;  // vertices per direction
  long nvert = 1;
  for (int k = 0; k < D; ++k) nvert *= nv;
  for (int col = 0; col < (1 << D); ++col) {
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nvert; ++q) {
      long a[3] = {q % nv, D > 1 ? (q / nv) % nv : 0, D > 2 ? q / (nv * nv) : 0};
      int c = 0;
      for (int k = 0; k < D; ++k) c |= (int)(a[k] & 1) << k;
      if (c != col) continue;
      long v[3];
      for (int k = 0; k < 3; ++k) v[k] = a[k] * H.order;
      ssc_block(H, L, v, omega, x, b, r);
    }
  }
}

// 1D interpolation stencils (fetransfer.lisp:73-195 evaluated for uniform
// Lagrange Q1/Q2): coarse node J <-> fine node 2J.
int restrict_stencil1d(int order, long J, long* off, double* w) {
  if (order == 1) { off[0] = -1; off[1] = 0; off[2] = 1; w[0] = 0.5; w[1] = 1.0; w[2] = 0.5; return 3; }
  if (J % 2 == 0) {
    long o[5] = {-3, -1, 0, 1, 3};
    double ww[5] = {-0.125, 0.375, 1.0, 0.375, -0.125};
    for (int k = 0; k < 5; ++k) { off[k] = o[k]; w[k] = ww[k]; }
    return 5;
  }
  off[0] = -1; off[1] = 0; off[2] = 1; w[0] = 0.75; w[1] = 1.0; w[2] = 0.75;
  return 3;
}

// coarse nodes contributing to fine node I (ascending J)
int prolong_stencil1d(int order, long I, long* J, double* w) {
  if (I % 2 == 0) { J[0] = I / 2; w[0] = 1.0; return 1; }
  if (order == 1) { J[0] = (I - 1) / 2; J[1] = (I + 1) / 2; w[0] = 0.5; w[1] = 0.5; return 2; }
  long c = I / 4;
  double s = (double)(I - 4 * c) / 4.0;
  J[0] = 2 * c; J[1] = 2 * c + 1; J[2] = 2 * c + 2;
  w[0] = 2.0 * (s - 0.5) * (s - 1.0);
  w[1] = 4.0 * s * (1.0 - s);
  w[2] = 2.0 * s * (s - 0.5);
  return 3;
}

// res_{l-1} := I^T res_l (multigrid.lisp:202-212, gemm! ... :tn) with the
// constrained interpolation (constraints.lisp:58-72)
void restrict_(const Hier& H, int lf, const double* rf, double* rc) {
  const Level& F = H.lev[lf];
  const Level& C = H.lev[lf - 1];
  if (H.algebraic) {  // rc = I^T rf, fine entries ascending
    for (long J = 0; J < C.N; ++J) {
      double acc = 0.0;
      for (long e = F.pt.start[J]; e < F.pt.start[J + 1]; ++e) acc = std::fma(F.pt.value[e], rf[F.pt.index[e]], acc);
      rc[J] = acc;
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (long J = 0; J < C.N; ++J) {
    long cJ[3];
    coords(H, C.M, J, cJ);
    const int nc = H.nc;
    if (is_dirichlet(H, C.M, cJ)) { for (int c = 0; c < nc; ++c) rc[J * nc + c] = 0.0; continue; }
    long off[3][5] = {{0}, {0}, {0}};
    double w[3][5] = {{1.0}, {1.0}, {1.0}};
    int cnt[3] = {1, 1, 1};
    for (int k = 0; k < H.dim; ++k) cnt[k] = restrict_stencil1d(H.order, cJ[k], off[k], w[k]);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int x = 0; x < cnt[0]; ++x) {
          long fi[3] = {2 * cJ[0] + off[0][x], 2 * cJ[1] + off[1][y], 2 * cJ[2] + off[2][z]};
          bool in = true;
          for (int k = 0; k < H.dim; ++k) if (fi[k] < 0 || fi[k] >= F.M) in = false;
          if (!in) continue;
          if (is_dirichlet(H, F.M, fi)) continue;
          double ww = w[0][x];
          if (H.dim > 1) ww = ww * w[1][y];
          if (H.dim > 2) ww = ww * w[2][z];
          long i = fi[0] + F.M * (fi[1] + F.M * fi[2]);
          for (int c = 0; c < nc; ++c) acc[c] = std::fma(ww, rf[i * nc + c], acc[c]);
        }
    for (int c = 0; c < nc; ++c) rc[J * nc + c] = acc[c];
  }
}

// sol_{l+1} += I sol_l (multigrid.lisp:237-239, gemm! ... :nn)
void prolongate(const Hier& H, int lc, const double* xc, double* xf, bool constrained) {
  const Level& C = H.lev[lc];
  const Level& F = H.lev[lc + 1];
  if (H.algebraic) {  // xf += I xc, coarse entries ascending; empty (constrained) rows untouched
    for (long i = 0; i < F.N; ++i) {
      if (F.p.start[i] == F.p.start[i + 1]) continue;
      double acc = 0.0;
      for (long e = F.p.start[i]; e < F.p.start[i + 1]; ++e) acc = std::fma(F.p.value[e], xc[F.p.index[e]], acc);
      xf[i] = xf[i] + acc;
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < F.N; ++i) {
    long fi[3];
    coords(H, F.M, i, fi);
    if (constrained && is_dirichlet(H, F.M, fi)) continue;
    long J[3][3] = {{0}, {0}, {0}};
    double w[3][3] = {{1.0}, {1.0}, {1.0}};
    int cnt[3] = {1, 1, 1};
    for (int k = 0; k < H.dim; ++k) cnt[k] = prolong_stencil1d(H.order, fi[k], J[k], w[k]);
    const int nc = H.nc;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int x = 0; x < cnt[0]; ++x) {
          long cj[3] = {J[0][x], J[1][y], J[2][z]};
          if (constrained && is_dirichlet(H, C.M, cj)) continue;
          double ww = w[0][x];
          if (H.dim > 1) ww = ww * w[1][y];
          if (H.dim > 2) ww = ww * w[2][z];
          long j = cj[0] + C.M * (cj[1] + C.M * cj[2]);
          for (int c = 0; c < nc; ++c) acc[c] = std::fma(ww, xc[j * nc + c], acc[c]);
        }
    for (int c = 0; c < nc; ++c) xf[i * nc + c] = xf[i * nc + c] + acc[c];
  }
}

// Galerkin coarse operator (multilevel-decomposition with :galerkin-p t,
// geomg.lisp:109-142; galerkin-product, amg.lisp:247-285): A_l = I^T A_{l+1} I
// with the constrained interpolation (constraints.lisp:58-72: rows of fine
// Dirichlet nodes and columns of coarse Dirichlet nodes removed), identity
// blocks at coarse Dirichlet nodes.  For nested Lagrange spaces every nonzero
// term couples two nodes of one coarse cell, so the product has the level's
// own stencil (Q2: an odd-coordinate node's +-2 entries come out exactly
// zero, and terms reaching beyond the stencil multiply structural zeros).  Order, as galerkin-product associates it ((R_kl A_lm) P_mn, block
// products componentwise, the interpolation acting on each component):
// per coarse row I, fine i over the restriction stencil of I (z, y, x
// ascending), fine slots ascending, coarse J over the interpolation stencil of
// j (z, y, x ascending), block entries (k, m) row-major:
// acc[J - I][k][m] = fma(w_iI * a_ij[k][m], w_jJ, acc[J - I][k][m]).
int galerkin_level(Hier& H, int l) {
  const int nc = H.nc;
  Level& C = H.lev[l];
  const Level& F = H.lev[l + 1];
  C.A.assign((size_t)H.nslots * nc * nc * C.N, 0.0);
  const int center = [&] { long z[3] = {0, 0, 0}; return slot_of(H, z); }();
  auto at = [&](const Level& L, int s, int k, int m, long i) { return (((size_t)s * nc + k) * nc + m) * L.N + i; };
#pragma omp parallel for schedule(dynamic, 16)
  for (long I = 0; I < C.N; ++I) {
    long cI[3];
    coords(H, C.M, I, cI);
    if (is_dirichlet(H, C.M, cI)) {
      for (int k = 0; k < nc; ++k) C.A[at(C, center, k, k, I)] = 1.0;
      continue;
    }
    std::vector<double> acc((size_t)H.nslots * nc * nc, 0.0);
    long off[3][5] = {{0}, {0}, {0}};
    double w[3][5] = {{1.0}, {1.0}, {1.0}};
    int cnt[3] = {1, 1, 1};
    for (int k = 0; k < H.dim; ++k) cnt[k] = restrict_stencil1d(H.order, cI[k], off[k], w[k]);
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int x = 0; x < cnt[0]; ++x) {
          long fi[3] = {2 * cI[0] + off[0][x], 2 * cI[1] + off[1][y], 2 * cI[2] + off[2][z]};
          bool in = true;
          for (int k = 0; k < H.dim; ++k) if (fi[k] < 0 || fi[k] >= F.M) in = false;
          if (!in || is_dirichlet(H, F.M, fi)) continue;
          double wi = w[0][x];
          if (H.dim > 1) wi = wi * w[1][y];
          if (H.dim > 2) wi = wi * w[2][z];
          const long i = fi[0] + F.M * (fi[1] + F.M * fi[2]);
          for (int s = 0; s < H.nslots; ++s) {
            long o[3];
            slot_offset(H, s, o);
            long fj[3] = {fi[0] + o[0], fi[1] + o[1], fi[2] + o[2]};
            bool inj = true;
            for (int k = 0; k < H.dim; ++k) if (fj[k] < 0 || fj[k] >= F.M) inj = false;
            if (!inj || is_dirichlet(H, F.M, fj)) continue;
            double wa[9];
            for (int e = 0; e < nc * nc; ++e) wa[e] = wi * F.A[at(F, s, e / nc, e % nc, i)];
            long J[3][3] = {{0}, {0}, {0}};
            double wj[3][3] = {{1.0}, {1.0}, {1.0}};
            int cj[3] = {1, 1, 1};
            for (int k = 0; k < H.dim; ++k) cj[k] = prolong_stencil1d(H.order, fj[k], J[k], wj[k]);
            for (int zz = 0; zz < cj[2]; ++zz)
              for (int yy = 0; yy < cj[1]; ++yy)
                for (int xx = 0; xx < cj[0]; ++xx) {
                  long cJ[3] = {J[0][xx], J[1][yy], J[2][zz]};
                  if (is_dirichlet(H, C.M, cJ)) continue;
                  double ww = wj[0][xx];
                  if (H.dim > 1) ww = ww * wj[1][yy];
                  if (H.dim > 2) ww = ww * wj[2][zz];
                  long d[3] = {cJ[0] - cI[0], cJ[1] - cI[1], cJ[2] - cI[2]};
                  // a coarse node beyond the stencil: the term multiplies a
                  // structural zero (Q2: an odd-coordinate fine node has no
                  // +-2 coupling) and adds nothing
                  bool far = false;
                  for (int k = 0; k < H.dim; ++k) far = far || d[k] < -H.span || d[k] > H.span;
                  if (far) continue;
                  const int S = slot_of(H, d);
                  for (int e = 0; e < nc * nc; ++e)
                    acc[(size_t)S * nc * nc + e] = std::fma(wa[e], ww, acc[(size_t)S * nc * nc + e]);
                }
          }
        }
    for (int S = 0; S < H.nslots; ++S)
      for (int e = 0; e < nc * nc; ++e) C.A[at(C, S, e / nc, e % nc, I)] = acc[(size_t)S * nc * nc + e];
  }
  return 0;
}

// <lu> coarse-grid iterator (linit.lisp:137-162): r := A^-1 r; x += damp r
void coarse_solve(const Hier& H, double damp, double* x, double* r) {
  long n = H.nbase;
  std::vector<double> t(n);
  for (long i = 0; i < n; ++i) {
    double acc = 0.0;
    for (long j = 0; j < n; ++j) acc = std::fma(H.ainv[(size_t)i * n + j], r[j], acc);
    t[i] = acc;
  }
  for (long i = 0; i < n; ++i) { r[i] = t[i]; x[i] = std::fma(damp, t[i], x[i]); }
}

// ---------------------------------------------------------------- multigrid
// One smoother step (the base iterator) and its flags (linit.lisp:220-323,
// blockit.lisp:118-204): <jacobi> and the block iterations residual-before t,
// <sor> residual-before nil; all residual-after nil.
bool smoother_residual_before(const ora_solve_cfg& c) { return c.smoother != ORA_SOR; }

void smoother_step(Hier& H, const ora_solve_cfg& c, int l, double* x, double* b, double* r) {
  if (c.smoother == ORA_JACOBI) jacobi(H, l, c.damp, x, r);
  else if (c.smoother == ORA_SSC) ssc(H, l, c.damp, x, b, r);
  else if (c.smoother == ORA_PSC) psc(H, l, c.damp, x, r);
  else sor(H, l, c.damp, x, b, r);
}

// product-iterator (linit.lisp:94-120): after every step the residual is
// recomputed when residual-before and not residual-after
void smoother_product(Hier& H, const ora_solve_cfg& c, int l, int steps, double* x, double* b,
                      double* r) {
  if (steps == 1) { smoother_step(H, c, l, x, b, r); return; }
  for (int s = 0; s < steps; ++s) {
    smoother_step(H, c, l, x, b, r);
    if (smoother_residual_before(c)) residual(H, l, x, b, r);
  }
}

void ensure_mg_residual(Hier& H) {  // multigrid.lisp:173-177
  int l = H.cur;
  if (!H.rp[l]) {
    residual(H, l, H.sol[l], H.rhsv[l], H.res[l]);
    H.rp[l] = 1;
  }
}

void smooth(Hier& H, const ora_solve_cfg& c, int steps) {  // multigrid.lisp:179-189
  if (steps <= 0) return;
  if (smoother_residual_before(c)) ensure_mg_residual(H);
  int l = H.cur;
  smoother_product(H, c, l, steps, H.sol[l], H.rhsv[l], H.res[l]);
  H.rp[l] = 0;
}

void mg_restrict(Hier& H) {  // multigrid.lisp:202-224
  int l = H.cur;
  ensure_mg_residual(H);
  restrict_(H, l, H.res[l], H.res[l - 1]);
  H.cur = l - 1;
  H.rp[l - 1] = 0;
  long n = vec_len(H, l - 1);
  std::fill(H.sol[l - 1], H.sol[l - 1] + n, 0.0);
  std::copy(H.res[l - 1], H.res[l - 1] + n, H.rhsv[l - 1]);
  H.rp[l - 1] = 1;
}

void mg_prolongate(Hier& H) {  // multigrid.lisp:237-252
  int l = H.cur;
  prolongate(H, l, H.sol[l], H.sol[l + 1], true);
  H.cur = l + 1;
  H.rp[l + 1] = 0;
}

void lmgc(Hier& H, const ora_solve_cfg& c) {  // multigrid.lisp:254-288
  int l = H.cur;
  if (l == H.base) {
    coarse_solve(H, c.coarse_damp, H.sol[l], H.res[l]);
    H.rp[l] = 0;
    return;
  }
  if (c.combination == 0) {
    smooth(H, c, c.pre_steps);
    mg_restrict(H);
  } else {  // :additive -- smoothing on level l after the restriction
    mg_restrict(H);
    H.cur += 1;
    smooth(H, c, c.pre_steps);
    H.cur -= 1;
  }
  int g = c.gamma == 0 ? 0 : (H.cur == H.base ? 1 : c.gamma);
  for (int i = g; i >= 1; --i) {
    lmgc(H, c);
    if (i != 1) ensure_mg_residual(H);
  }
  if (c.combination == 0) {
    mg_prolongate(H);
    smooth(H, c, c.post_steps);
  } else {
    H.cur += 1;
    smooth(H, c, c.post_steps);
    H.cur -= 1;
    mg_prolongate(H);
  }
}

// the multigrid iterator's iterate function (multigrid.lisp:366-386): the
// top-level sol/rhs/res are the caller's vectors, with no copy
// f-cycle (multigrid.lisp:290-297): restrict from the top to the base level,
// then from the base up a cycle on each level and, below the top, the
// prolongation of its solution to the level above
void f_cycle(Hier& H, const ora_solve_cfg& c) {
  const int top = H.cur;
  for (int l = top; l > H.base; --l) mg_restrict(H);
  for (int l = H.base; l <= top; ++l) {
    lmgc(H, c);
    if (l != top) mg_prolongate(H);
  }
}

void mg_iterate(Hier& H, const ora_solve_cfg& c, double* x, double* b, double* r) {
  int top = H.top;
  H.sol[top] = x; H.rhsv[top] = b; H.res[top] = r;
  H.rp[top] = 1;
  H.cur = top;
  if (c.fmg) f_cycle(H, c);
  else lmgc(H, c);
}

void ensure_state(Hier& H) {
  int nl = H.top + 1;
  if ((int)H.sol.size() == nl) return;
  H.sol.assign(nl, nullptr); H.rhsv.assign(nl, nullptr); H.res.assign(nl, nullptr);
  H.rp.assign(nl, 0);
  H.store.assign(3 * nl, {});
  for (int l = H.base; l < H.top; ++l) {
    long n = vec_len(H, l);
    H.store[3 * l].assign(n, 0.0); H.store[3 * l + 1].assign(n, 0.0); H.store[3 * l + 2].assign(n, 0.0);
    H.sol[l] = H.store[3 * l].data(); H.rhsv[l] = H.store[3 * l + 1].data(); H.res[l] = H.store[3 * l + 2].data();
  }
}

}  // namespace

// ==================================================================== C API
extern "C" {

void* ora_create(int dim, int order, int ncomp, int n0, int top_level, int base_level,
                 int dirichlet_mask) {
  if (dim < 1 || dim > 3 || order < 1 || order > 2 || (ncomp != 1 && ncomp != dim) || n0 < 1 ||
      base_level < 0 || base_level > top_level || top_level > 12)
    return nullptr;
  Hier* H = new Hier();
  H->dim = dim; H->order = order; H->nc = ncomp; H->n0 = n0;
  H->top = top_level; H->base = base_level; H->dmask = dirichlet_mask;
  H->span = order;
  H->nslots = 1;
  for (int k = 0; k < dim; ++k) H->nslots *= 2 * order + 1;
  H->lev.resize(top_level + 1);
  for (int l = 0; l <= top_level; ++l) {
    Level& L = H->lev[l];
    L.n = (long)n0 << l;
    L.M = order * L.n + 1;
    L.N = 1;
    for (int k = 0; k < dim; ++k) L.N *= L.M;
    L.h = 1.0 / (double)L.n;
  }
  return H;
}

void ora_destroy(void* h) { delete (Hier*)h; }

int ora_set_coefficient(void* h, int kind, const double* vals, long n) {
  Hier& H = *(Hier*)h;
  long nt = H.lev[H.top].n, ncell = 1;
  for (int k = 0; k < H.dim; ++k) ncell *= nt;
  Tables T = make_tables(H.dim, H.order, 1.0);
  switch (kind) {
    case ORA_K_CONST: if (n != 1) return -1; H.kkind = kind; H.kconst = vals[0]; break;
    case ORA_K_CELL: if (n != ncell) return -1; H.kkind = kind; H.kcell.assign(vals, vals + n); break;
    case ORA_F_CONST: if (n != 1) return -1; H.fkind = kind; H.fconst = vals[0]; break;
    case ORA_F_IP: if (n != ncell * T.nq || H.nc != 1) return -1; H.fkind = kind; H.fip.assign(vals, vals + n); break;
    case ORA_LAMBDA_MU_CELL:  // lambda = mu = E per top-level cell (nc = dim)
      if (n != ncell || H.nc == 1) return -1;
      H.kkind = ORA_K_CELL;
      H.kcell.assign(vals, vals + n);
      break;
    case ORA_F_VEC: if (n != H.nc) return -1; H.fkind = kind; for (int k = 0; k < n; ++k) H.fvec[k] = vals[k]; break;
    default: return -1;
  }
  H.assembled = false;
  return 0;
}

int ora_assemble_levels(void* h, int mode) {
  Hier& H = *(Hier*)h;
  if (mode != 0 && mode != 1) return -1;
  for (int l = H.top; l >= H.base; --l) {
    int rc = (mode == 1 && l < H.top) ? galerkin_level(H, l) : assemble_level(H, l);
    if (rc) return rc;
  }
  build_coarse_inverse(H);
  H.assembled = true;
  ensure_state(H);
  return 0;
}

// Level matrices handed over from outside (the counterpart of fmg_set_matrix):
// the slot layout of ora_get_matrix; ora_finish_levels then forms the coarse
// inverse once every level is in place.
int ora_set_matrix(void* h, int level, const double* a) {
  Hier& H = *(Hier*)h;
  if (level < H.base || level > H.top) return -1;
  Level& L = H.lev[level];
  L.A.assign(a, a + (size_t)H.nslots * H.nc * H.nc * L.N);
  H.assembled = false;
  return 0;
}

// Algebraic hierarchies (the counterpart of fmg_grid_create_algebraic):
// levels 0 .. nlevels-1 of the given sizes, matrices and interpolations as
// compressed rows with columns ascending.
void* ora_create_algebraic(int nlevels, const long* sizes) {
  if (nlevels < 1 || nlevels > 16) return nullptr;
  Hier* H = new Hier();
  H->algebraic = true;
  H->dim = 0; H->order = 1; H->nc = 1; H->n0 = 1;
  H->top = nlevels - 1; H->base = 0; H->dmask = 0;
  H->span = 1; H->nslots = 1;
  H->lev.resize(nlevels);
  for (int l = 0; l < nlevels; ++l) H->lev[l].N = sizes[l];
  return H;
}

int ora_set_csr_matrix(void* h, int level, const long* start, const int* index, const double* value) {
  Hier& H = *(Hier*)h;
  if (!H.algebraic || level < H.base || level > H.top) return -1;
  Level& L = H.lev[level];
  L.a.start.assign(start, start + L.N + 1);
  L.a.index.assign(index, index + start[L.N]);
  L.a.value.assign(value, value + start[L.N]);
  L.dg.assign(L.N, 0.0);
  for (long i = 0; i < L.N; ++i)
    for (long e = start[i]; e < start[i + 1]; ++e)
      if (index[e] == i) L.dg[i] = value[e];
  // the colouring of the SOR/SSC sweeps: rows in ascending order take the
  // smallest colour none of their coloured neighbours (a_ij or a_ji stored,
  // j != i) has -- Femlisp's <sor> with the rows ordered by colour
  // (linit.lisp:288-323, the :compare ordering)
  std::vector<std::vector<int>> nbr(L.N);
  for (long i = 0; i < L.N; ++i)
    for (long e = start[i]; e < start[i + 1]; ++e)
      if (index[e] != i) {
        nbr[i].push_back(index[e]);
        nbr[index[e]].push_back((int)i);
      }
  L.colour.assign(L.N, -1);
  L.ncol = 0;
  for (long i = 0; i < L.N; ++i) {
    std::vector<char> used(nbr[i].size() + 1, 0);
    for (int j : nbr[i])
      if (L.colour[j] >= 0 && (size_t)L.colour[j] < used.size()) used[L.colour[j]] = 1;
    int c = 0;
    while (used[c]) ++c;
    L.colour[i] = c;
    L.ncol = std::max(L.ncol, c + 1);
  }
  H.assembled = false;
  return 0;
}


int ora_set_interpolation(void* h, int fine_level, const long* start, const int* index, const double* value) {
  Hier& H = *(Hier*)h;
  if (!H.algebraic || fine_level <= H.base || fine_level > H.top) return -1;
  Level& F = H.lev[fine_level];
  const long NC = H.lev[fine_level - 1].N;
  F.p.start.assign(start, start + F.N + 1);
  F.p.index.assign(index, index + start[F.N]);
  F.p.value.assign(value, value + start[F.N]);
  std::vector<std::vector<std::pair<int, double>>> cols(NC);
  for (long i = 0; i < F.N; ++i)
    for (long e = start[i]; e < start[i + 1]; ++e) cols[index[e]].push_back({(int)i, value[e]});
  F.pt = Csr{};
  F.pt.start.assign(1, 0);
  for (long J = 0; J < NC; ++J) {
    for (auto& q : cols[J]) { F.pt.index.push_back(q.first); F.pt.value.push_back(q.second); }
    F.pt.start.push_back((long)F.pt.index.size());
  }
  H.assembled = false;
  return 0;
}

int ora_set_rhs(void* h, const double* b) {
  Hier& H = *(Hier*)h;
  H.rhs.assign(b, b + (size_t)H.lev[H.top].N * H.nc);
  return 0;
}

int ora_finish_levels(void* h) {
  Hier& H = *(Hier*)h;
  for (int l = H.base; l <= H.top; ++l) {
    const Level& L = H.lev[l];
    if (H.algebraic ? (L.a.start.size() != (size_t)L.N + 1 || (l > H.base && L.p.start.size() != (size_t)L.N + 1))
                    : L.A.size() != (size_t)H.nslots * H.nc * H.nc * L.N)
      return -1;
  }
  if (H.rhs.size() != (size_t)H.lev[H.top].N * H.nc) H.rhs.assign((size_t)H.lev[H.top].N * H.nc, 0.0);
  build_coarse_inverse(H);
  H.assembled = true;
  ensure_state(H);
  return 0;
}

int ora_assemble(void* h) {
  Hier& H = *(Hier*)h;
  for (int l = H.top; l >= H.base; --l) {
    int rc = assemble_level(H, l);
    if (rc) return rc;
  }
  build_coarse_inverse(H);
  H.assembled = true;
  ensure_state(H);
  return 0;
}

int ora_set_node_damping(void* h, int level, const double* w, long n) {
  Hier& H = *(Hier*)h;
  if (level < 0 || level > H.top || n != H.lev[level].N) return -1;
  if (w) H.lev[level].omega.assign(w, w + n); else H.lev[level].omega.clear();
  return 0;
}

long ora_nnodes(void* h, int level) { return ((Hier*)h)->lev[level].N; }
int ora_nslots(void* h) { return ((Hier*)h)->nslots; }

int ora_get_matrix(void* h, int level, double* out) {
  Hier& H = *(Hier*)h;
  if (!H.assembled || level < H.base || level > H.top) return -1;
  std::copy(H.lev[level].A.begin(), H.lev[level].A.end(), out);
  return 0;
}

int ora_get_rhs(void* h, double* out) {
  Hier& H = *(Hier*)h;
  if (!H.assembled) return -1;
  std::copy(H.rhs.begin(), H.rhs.end(), out);
  return 0;
}

int ora_get_coarse_inverse(void* h, double* out) {
  Hier& H = *(Hier*)h;
  if (!H.assembled) return -1;
  std::copy(H.ainv.begin(), H.ainv.end(), out);
  return 0;
}

int ora_matvec(void* h, int level, const double* x, double* y) { matvec(*(Hier*)h, level, x, y); return 0; }
int ora_residual(void* h, int level, const double* x, const double* b, double* r) {
  residual(*(Hier*)h, level, x, b, r);
  return 0;
}
int ora_restrict(void* h, int fine_level, const double* rf, double* rc) {
  restrict_(*(Hier*)h, fine_level, rf, rc);
  return 0;
}
int ora_prolongate(void* h, int coarse_level, const double* xc, double* xf, int constrained) {
  prolongate(*(Hier*)h, coarse_level, xc, xf, constrained != 0);
  return 0;
}
// projection (injection) of fine nodal values onto the coarse nodes
int ora_inject(void* h, int coarse_level, const double* xf, double* xc) {
  Hier& H = *(Hier*)h;
  const Level& C = H.lev[coarse_level];
  const Level& F = H.lev[coarse_level + 1];
  for (long J = 0; J < C.N; ++J) {
    long c[3];
    coords(H, C.M, J, c);
    xc[J] = xf[2 * c[0] + F.M * (2 * c[1] + F.M * 2 * c[2])];
  }
  return 0;
}
int ora_jacobi(void* h, int level, double damp, double* x, double* r) {
  jacobi(*(Hier*)h, level, damp, x, r);
  return 0;
}
int ora_sor(void* h, int level, double omega, double* x, const double* b, double* r) {
  if (((Hier*)h)->nc != 1) return -2;
  sor(*(Hier*)h, level, omega, x, b, r);
  return 0;
}
int ora_psc(void* h, int level, double damp, double* x, const double* r) {
  if (((Hier*)h)->nc != 1) return -2;
  psc(*(Hier*)h, level, damp, x, r);
  return 0;
}
int ora_ssc(void* h, int level, double omega, double* x, const double* b, double* r) {
  if (((Hier*)h)->nc != 1) return -2;
  ssc(*(Hier*)h, level, omega, x, b, r);
  return 0;
}
int ora_coarse_solve(void* h, double damp, double* x, double* r) {
  coarse_solve(*(Hier*)h, damp, x, r);
  return 0;
}
double ora_dot(const double* x, const double* y, long n) { return dr_dot(x, y, n, false); }
double ora_dot_par(const double* x, const double* y, long n) { return dr_dot(x, y, n, true); }

extern "C++" {
namespace {
template <typename T>
void mf_apply(int M, int dm, const double* kc, const double* xd, const double* bd, double* y, bool x32) {
  const int n = M - 1;
  const long long MM = (long long)M * M, N = MM * M;
  const T hs = (T)((1.0 / n) / 12.0);
  auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
  auto xv = [&](long long i) { return x32 ? (T)(float)xd[i] : (T)xd[i]; };
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {
    const int ix = (int)(i % M), iy = (int)((i / M) % M), iz = (int)(i / MM);
    T ax;
    if (dirf(ix, 1, 2) || dirf(iy, 4, 8) || dirf(iz, 16, 32)) {
      ax = xv(i);
    } else {
      T k[2][2][2];
      for (int cz = 0; cz < 2; ++cz)
        for (int cy = 0; cy < 2; ++cy)
          for (int cx = 0; cx < 2; ++cx) {
            const int ex = ix - 1 + cx, ey = iy - 1 + cy, ez = iz - 1 + cz;
            const bool in = ex >= 0 && ex < n && ey >= 0 && ey < n && ez >= 0 && ez < n;
            k[cz][cy][cx] = in ? (T)kc[ex + (long long)n * (ey + (long long)n * ez)] : T(0);
          }
      auto X = [&](int dx, int dy, int dz) -> T {
        const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
        const bool in = jx >= 0 && jx < M && jy >= 0 && jy < M && jz >= 0 && jz < M && !dirf(jx, 1, 2) &&
                        !dirf(jy, 4, 8) && !dirf(jz, 16, 32);
        return in ? xv((long long)jz * MM + (long long)jy * M + jx) : T(0);
      };
      constexpr bool DIFF = sizeof(T) == 8;
      const T wc[2][2] = {{k[0][0][0] + k[1][0][0], k[0][0][1] + k[1][0][1]},
                          {k[0][1][0] + k[1][1][0], k[0][1][1] + k[1][1][1]}};
      const T ksum = (wc[0][0] + wc[0][1]) + (wc[1][0] + wc[1][1]);
      const T xc = X(0, 0, 0);
      // three partial sums: the node's own plane, the plane below, the plane above
      T sp[3] = {T(0), T(0), T(0)};
      auto term = [&](int a, T w, T xj) { sp[a] = DIFF ? std::fma(w, xc - xj, sp[a]) : std::fma(w, xj, sp[a]); };
      for (int sy = 0; sy < 2; ++sy)
        for (int sx = 0; sx < 2; ++sx) term(0, wc[sy][sx], X(2 * sx - 1, 2 * sy - 1, 0));
      for (int cz = 0; cz < 2; ++cz) {
        const int dz = 2 * cz - 1;
        for (int sx = 0; sx < 2; ++sx) term(1 + cz, k[cz][0][sx] + k[cz][1][sx], X(2 * sx - 1, 0, dz));
        for (int sy = 0; sy < 2; ++sy) term(1 + cz, k[cz][sy][0] + k[cz][sy][1], X(0, 2 * sy - 1, dz));
        for (int sy = 0; sy < 2; ++sy)
          for (int sx = 0; sx < 2; ++sx) term(1 + cz, k[cz][sy][sx], X(2 * sx - 1, 2 * sy - 1, dz));
      }
      T s = sp[0] + (sp[1] + sp[2]);
      if (!DIFF) s = std::fma(T(4) * ksum, xc, -s);
      ax = hs * s;
    }
    y[i] = (double)(bd ? (T)bd[i] - ax : ax);
  }
}
}  // namespace
}  // extern "C++"

void ora_mf_apply(int M, int dmask, const double* k, int fp32, const double* x, const double* b, double* y) {
  if (fp32 == 1) mf_apply<float>(M, dmask, k, x, b, y, false);
  else mf_apply<double>(M, dmask, k, x, b, y, fp32 == 2);
}

int ora_vcycle(void* h, const ora_solve_cfg* cfg, double* x, double* b, double* r) {
  Hier& H = *(Hier*)h;
  if (!H.assembled) return -1;
  mg_iterate(H, *cfg, x, b, r);
  return 0;
}

// <linear-solver> loop (iterate.lisp:239-250, solve.lisp:139-155,
// linsolve.lisp:58-73) around <cg> (krylow.lisp:72-132) or the bare
// multigrid iterator
int ora_solve(void* h, const ora_solve_cfg* cfg, double* x, double* hist, int hist_len, int* nsteps) {
  Hier& H = *(Hier*)h;
  if (!H.assembled) return -1;
  if (H.nc != 1 && cfg->smoother != ORA_JACOBI) return -2;
  if (H.algebraic && cfg->smoother == ORA_PSC) return -2;
  const ora_solve_cfg& c = *cfg;
  const int top = H.top;
  const long n = vec_len(H, top);
  std::vector<double> r(n, 0.0), p(n, 0.0), a(n, 0.0), w(n, 0.0), w2(n, 0.0), q(n, 0.0);
  std::vector<double> bcopy(H.rhs);  // the problem's rhs is never written
  bool rp = false, initialized = false;
  double defnorm = 0.0, initial = -1.0, alpha = 0.0;
  const bool par = true;
  auto precond = [&](double* sol, double* rr) {
    // (copy! r w) then (iterate sol w w) -- or a separate residual vector
    std::copy(rr, rr + n, w.begin());
    if (c.compat_alias) mg_iterate(H, c, sol, w.data(), w.data());
    else {
      std::copy(rr, rr + n, w2.begin());
      mg_iterate(H, c, sol, w.data(), w2.data());
    }
  };
  for (int step = 0;; ++step) {
    if (!rp) { residual(H, top, x, bcopy.data(), r.data()); rp = true; }
    defnorm = std::sqrt(dr_dot(r.data(), r.data(), n, par));
    if (initial < 0) initial = defnorm;
    double reduction = (initial == 0.0) ? 0.0 : defnorm / initial;
    if (step < hist_len) hist[step] = defnorm;
    *nsteps = step;
    if ((c.rtol > 0 && reduction < c.rtol) || (c.atol > 0 && defnorm < c.atol)) return 0;
    if (step > c.maxsteps) return 1;
    if (c.method == ORA_METHOD_MG) {
      mg_iterate(H, c, x, bcopy.data(), r.data());
      rp = false;
      continue;
    }
    // <cg>
    if (!initialized) {  // restart (krylow.lisp:88-96)
      if (c.method == ORA_METHOD_CG_MG) precond(p.data(), r.data());
      else std::copy(r.begin(), r.end(), p.begin());
      alpha = dr_dot(p.data(), r.data(), n, par);
      initialized = true;
    }
    if (alpha != 0.0) {  // krylow.lisp:106-127
      matvec(H, top, p.data(), a.data());
      double beta = dr_dot(a.data(), p.data(), n, par);
      double lam = alpha / beta;
      for (long i = 0; i < n; ++i) x[i] = std::fma(lam, p[i], x[i]);
      for (long i = 0; i < n; ++i) r[i] = std::fma(-lam, a[i], r[i]);
      if (c.method == ORA_METHOD_CG_MG) {
        std::fill(q.begin(), q.end(), 0.0);
        precond(q.data(), r.data());
      } else {
        std::copy(r.begin(), r.end(), q.begin());
      }
      double new_alpha = dr_dot(q.data(), r.data(), n, par);
      double s = new_alpha / alpha;
      for (long i = 0; i < n; ++i) p[i] = s * p[i];
      for (long i = 0; i < n; ++i) p[i] = p[i] + q[i];
      alpha = new_alpha;
    }
    rp = true;
  }
}

int ora_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// the OpenMP thread count of the following calls (the 1-thread timing of the
// CPU baseline); the results do not depend on it (fixed loop orders)
void ora_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
