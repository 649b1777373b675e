// kernels_fp64.cu -- the FP64 kernels of the multigrid solve path (sm_100a).
//
// Layout in HBM: a level matrix is stored by stencil slot (structure of
// arrays): A[s * Np + i] = A(i, i + off_s), Np = node count rounded up to a
// multiple of 64 so that every slot array starts on a 512-byte boundary.
// Column indices are implicit (off_s = ox + M oy + M^2 oz), so the matvec
// streams only matrix values: 128-bit loads of two consecutive rows per
// thread, coalesced across the warp.  Entries outside the grid, in eliminated
// Dirichlet columns and structurally absent Q2 couplings are stored as zeros,
// which lets neighbour indices be clamped to the vector instead of tested.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include "fmgpu_kernels.cuh"

namespace fmg {

std::atomic<long long> g_launches{0};

template <int D, int P>
struct St {
  static constexpr int W = 2 * P + 1;
  static constexpr int NS = D == 1 ? W : (D == 2 ? W * W : W * W * W);
  static constexpr int CENTER = (NS - 1) / 2;
};

template <int D, int P>
__device__ __forceinline__ long long slot_off(int s, long long M) {
  constexpr int W = 2 * P + 1;
  long long o = (long long)(s % W - P);
  if (D > 1) o += M * (long long)((s / W) % W - P);
  if (D > 2) o += M * M * (long long)((s / (W * W)) % W - P);
  return o;
}

__device__ __forceinline__ void node_coords(long long i, long long M, int dim, long long c[3]) {
  c[0] = i % M;
  c[1] = dim > 1 ? (i / M) % M : 0;
  c[2] = dim > 2 ? i / (M * M) : 0;
}

// node_coords in 32-bit arithmetic (levels of fewer than 2^31 nodes)
__device__ __forceinline__ void node_coords32(long long i, long long M, int dim, long long c[3]) {
  const unsigned u = (unsigned)i, m = (unsigned)M;
  const unsigned q = u / m;
  c[0] = u - q * m;
  c[1] = dim > 1 ? q % m : 0;
  c[2] = dim > 2 ? q / m : 0;
}

__device__ __forceinline__ bool node_dirichlet(const long long c[3], long long M, int dim, int dmask) {
  for (int k = 0; k < dim; ++k) {
    if (c[k] == 0 && ((dmask >> (2 * k)) & 1)) return true;
    if (c[k] == M - 1 && ((dmask >> (2 * k + 1)) & 1)) return true;
  }
  return false;
}

// --------------------------------------------------- Q2 sliced storage
// A Q2 node couples at offset +-2 along direction k only when its coordinate k
// is even (a cell vertex); an odd coordinate (an edge / face / cell midpoint)
// couples within +-1.  Slot s of a Q2 level therefore stores only the nodes
// that admit it: those even along every direction where |offset_k| = 2 (the
// slot's pattern r, bit k).  They sit at the front of the slot's array, in
// lexicographic order of the coordinates halved along the restricted
// directions, so a level holds exactly its structural nonzeros (boundary and
// Dirichlet zeros aside) and a Q2 sweep streams no structural zero.  Q1
// levels and the centre slot (pattern 0) keep one entry per node.
template <int D>
__host__ __device__ __forceinline__ int q2_pattern(int s) {
  int r = 0;
  for (int k = 0; k < D; ++k) {
    const int o = s % 5 - 2;
    if (o == 2 || o == -2) r |= 1 << k;
    s /= 5;
  }
  return r;
}

// a node's index in the slot arrays of every pattern, and which patterns it admits
template <int D>
struct Q2Rows {
  long long idx[1 << D];
  unsigned valid;  // bit r: the node is stored in pattern-r slots
};

template <int D>
__host__ __device__ __forceinline__ void q2_rows(const long long c[3], long long M, Q2Rows<D>& q) {
  const long long H = (M + 1) / 2;
  q.valid = 0;
  for (int r = 0; r < (1 << D); ++r) {
    bool ok = true;
    long long id = 0, mul = 1;
    for (int k = 0; k < D; ++k) {
      const bool rk = (r >> k) & 1;
      if (rk && (c[k] & 1)) ok = false;
      id += (rk ? c[k] / 2 : c[k]) * mul;
      mul *= rk ? H : M;
    }
    q.idx[r] = id;
    if (ok) q.valid |= 1u << r;
  }
}

// Visits the stored slots of Q2 node c in ascending slot order (the order of
// every row sum): f(slot, neighbour offset, position in the slot's array).
// The z and y offsets are loops, the 5 x offsets unrolled; the row's index
// in a slot array depends only on which directions the slot restricts.
template <int D, typename F>
__device__ __forceinline__ void q2_row(const long long c[3], long long M, F&& f) {
  const long long H = (M + 1) / 2;
  const bool ex = !(c[0] & 1), ey = D > 1 && !(c[1] & 1), ez = D > 2 && !(c[2] & 1);
  for (int sz = 0; sz < (D > 2 ? 5 : 1); ++sz) {
    const int oz = D > 2 ? sz - 2 : 0;
    const bool rz = oz == 2 || oz == -2;
    if (rz && !ez) continue;
    for (int sy = 0; sy < (D > 1 ? 5 : 1); ++sy) {
      const int oy = D > 1 ? sy - 2 : 0;
      const bool ry = oy == 2 || oy == -2;
      if (ry && !ey) continue;
      const long long yz = (ry ? c[1] / 2 : c[1]) + (ry ? H : M) * (rz ? c[2] / 2 : c[2]);
      const long long p0 = c[0] + M * yz, p1 = c[0] / 2 + H * yz;
      const long long obase = (long long)oy * M + (long long)oz * M * M;
#pragma unroll
      for (int sx = 0; sx < 5; ++sx) {
        const int ox = sx - 2;
        const bool rx = ox == 2 || ox == -2;
        if (rx && !ex) continue;
        f(sx + 5 * (sy + 5 * sz), obase + ox, rx ? p1 : p0);
      }
    }
  }
}

// Scalar Q2 levels go one step further: rows are grouped by colour class
// (coordinates mod 3 -- the classes of the multicolour <sor>), classes in
// ascending order, and inside a class a slot array holds the rows that admit
// the slot in lexicographic order of their place in the class grid.  Along a
// direction the class's coordinates are d, d+3, d+6, .. (d = coordinate mod 3),
// or, where the slot restricts the direction to even coordinates, x0(d),
// x0(d)+6, .. with x0 = 0, 4, 2 for d = 0, 1, 2.  A colour sweep then streams
// one contiguous block of every slot array.  off[r][colour] is where the
// class's block starts in the arrays of pattern-r slots.
struct Q2Layout {
  long long off[8][27];
};

__host__ __device__ __forceinline__ int q2c_x0(int d) { return d == 0 ? 0 : (d == 1 ? 4 : 2); }
// rows of class digit d along one direction (M coordinates), restricted or not
__host__ __device__ __forceinline__ long long q2c_ext(long long M, int d, bool r) {
  if (!r) return (M - d + 2) / 3;
  const int x0 = q2c_x0(d);
  return x0 < M ? (M - x0 + 5) / 6 : 0;
}
// place of coordinate c (digit d = c mod 3) in its class grid along one direction
__host__ __device__ __forceinline__ long long q2c_j(long long c, int d, bool r) {
  return r ? (c - q2c_x0(d)) / 6 : (c - d) / 3;
}

Q2Layout q2_layout(int D, long long M) {
  Q2Layout L{};
  int ncol = 1;
  for (int k = 0; k < D; ++k) ncol *= 3;
  for (int r = 0; r < (1 << D); ++r) {
    long long acc = 0;
    for (int col = 0; col < ncol; ++col) {
      L.off[r][col] = acc;
      long long cnt = 1;
      int t = col;
      for (int k = 0; k < D; ++k) {
        cnt *= q2c_ext(M, t % 3, (r >> k) & 1);
        t /= 3;
      }
      acc += cnt;
    }
  }
  return L;
}

// storage position of node c in the arrays of pattern-r slots (the node must
// be even along the restricted directions)
template <int D>
__host__ __device__ __forceinline__ long long q2c_pos(const Q2Layout& L, const long long c[3], long long M, int r) {
  int col = 0, m3 = 1;
  long long p = 0, mul = 1;
  for (int k = 0; k < D; ++k) {
    const int d = (int)(c[k] % 3);
    const bool rk = (r >> k) & 1;
    col += d * m3;
    m3 *= 3;
    p += q2c_j(c[k], d, rk) * mul;
    mul *= q2c_ext(M, d, rk);
  }
  return L.off[r][col] + p;
}

// q2_row for the colour-major layout of scalar Q2 levels
template <int D, typename F>
__device__ __forceinline__ void q2c_row(const Q2Layout& L, const long long c[3], long long M, F&& f) {
  int col = 0, m3 = 1;
  long long j[3][2] = {{0, 0}, {0, 0}, {0, 0}}, e[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  bool ev[3] = {false, false, false};
  for (int k = 0; k < D; ++k) {
    const int d = (int)(c[k] % 3);
    col += d * m3;
    m3 *= 3;
    ev[k] = !(c[k] & 1);
    for (int rk = 0; rk < 2; ++rk) {
      j[k][rk] = q2c_j(c[k], d, rk);
      e[k][rk] = q2c_ext(M, d, rk);
    }
  }
  for (int sz = 0; sz < (D > 2 ? 5 : 1); ++sz) {
    const int oz = D > 2 ? sz - 2 : 0;
    const int rz = (oz == 2 || oz == -2) ? 1 : 0;
    if (rz && !ev[2]) continue;
    for (int sy = 0; sy < (D > 1 ? 5 : 1); ++sy) {
      const int oy = D > 1 ? sy - 2 : 0;
      const int ry = (oy == 2 || oy == -2) ? 1 : 0;
      if (ry && !ev[1]) continue;
      const long long yz = j[1][ry] + e[1][ry] * j[2][rz];
      const long long b0 = L.off[(ry << 1) | (rz << 2)][col] + j[0][0] + e[0][0] * yz;
      const long long b1 = L.off[1 | (ry << 1) | (rz << 2)][col] + j[0][1] + e[0][1] * yz;
      const long long obase = (long long)oy * M + (long long)oz * M * M;
#pragma unroll
      for (int sx = 0; sx < 5; ++sx) {
        const int ox = sx - 2;
        const bool rx = ox == 2 || ox == -2;
        if (rx && !ev[0]) continue;
        f(sx + 5 * (sy + 5 * sz), obase + ox, rx ? b1 : b0);
      }
    }
  }
}

// A node's position in the slot arrays of every pattern (32-bit: levels have
// fewer than 2^31 nodes) and the patterns it admits, in the colour-major
// layout of scalar Q2 levels (colour) or the natural sliced one (vector
// levels); visited with every slot unrolled, so the pattern of a slot is a
// compile-time constant and the loads can be issued ahead.
template <int D>
struct Q2Base {
  int p[1 << D];
  unsigned valid;
};

// CLAMP: keep every position in bounds (callers that load unstored slots too)
template <int D, bool COLOUR, bool CLAMP = false>
__device__ __forceinline__ void q2_base(const Q2Layout& lay, const long long c[3], long long M, Q2Base<D>& b) {
  long long nmax_l = 1;
  for (int k = 0; k < D; ++k) nmax_l *= M;
  const int nmax = (int)nmax_l;
  // per direction, unrestricted (0) and restricted (1): place and extent in
  // 32-bit arithmetic with constant divisors
  const int Mi = (int)M;
  int j[3][2] = {{0, 0}, {0, 0}, {0, 0}}, e[3][2] = {{1, 1}, {1, 1}, {1, 1}};
  int col = 0, m3 = 1;
  unsigned odd = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const int ck = (int)c[k];
    if (ck & 1) odd |= 1u << k;
    if (COLOUR) {
      const int d = ck % 3, x0 = q2c_x0(d);
      col += d * m3;
      m3 *= 3;
      j[k][0] = (ck - d) / 3;
      j[k][1] = (ck - x0) / 6;
      e[k][0] = (Mi - d + 2) / 3;
      e[k][1] = x0 < Mi ? (Mi - x0 + 5) / 6 : 0;
    } else {
      j[k][0] = ck;
      j[k][1] = ck >> 1;
      e[k][0] = Mi;
      e[k][1] = (Mi + 1) >> 1;
    }
  }
  b.valid = 0;
#pragma unroll
  for (int r = 0; r < (1 << D); ++r) {
    if (!(r & odd)) b.valid |= 1u << r;
    const int rx = r & 1, ry = (r >> 1) & 1, rz = (r >> 2) & 1;
    const int p = j[0][rx] + e[0][rx] * (j[1][ry] + e[1][ry] * j[2][rz]);
    const int q = COLOUR ? (int)lay.off[r][col] + p : p;
    b.p[r] = (CLAMP && q >= nmax) ? nmax - 1 : q;
  }
}

// Visits every slot (structural zeros too): f(slot, neighbour offset,
// position, stored).  A position is in bounds even where the slot is not
// stored for the node (the halved coordinate of an odd one), so callers load
// unconditionally and use 0 where !stored -- the structural zero the full
// layout would hold, in the same place of the row sum -- which lets the
// loads be issued ahead.
// ALL = false visits only the stored slots (the streaming kernels); ALL =
// true every slot, for the latency-bound colour sweeps of the SOR.
template <int D, bool ALL, typename F>
__device__ __forceinline__ void q2_visit(const Q2Base<D>& b, long long M, F&& f) {
  constexpr int NS = D == 1 ? 5 : (D == 2 ? 25 : 125);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int r = q2_pattern<D>(s);
    const bool st = ((b.valid >> r) & 1) != 0;
    if (ALL || st) f(s, slot_off<D, 2>(s, M), (long long)b.p[r], st);
  }
}

// ------------------------------------------------------------ batches
// A batched level holds nb independent problems of the same geometry, each
// at a fixed stride (vectors: the padded length Np; matrices: slots x Np).
// The 1D-grid kernels take the problem from blockIdx.y, the transfer kernels
// (1D/2D levels) from blockIdx.z; with one problem the offsets are zero.  A
// reduction then runs per problem: its partials, counter and scalar slots
// move with the problem.
__device__ __forceinline__ Reduce batch_reduce(Reduce R, unsigned bq) {
  R.part += (long long)bq * gridDim.x;
  R.counter += bq;
  R.scal += (long long)bq * S_COUNT;
  return R;
}

// ----------------------------------------------------------------- matvec
// y = A x (RES = false) or r = b - A x (RES = true, b may alias r); with DOT
// the chunk reduction of (y, dv) is fused in (DR4096 order).
template <int D, int P, bool RES, bool DOT>
__global__ void __launch_bounds__(kBlock)
k_spmv(const double* __restrict__ A, long long N, long long Np, long long M,
       const double* __restrict__ x, const double* b, double* y, const double* __restrict__ dv,
       Reduce R) {
  constexpr int NS = St<D, P>::NS;
  __shared__ double smem[8];
  const long long bq = blockIdx.y;  // problem of a batched level
  A += bq * NS * Np;
  x += bq * Np;
  y += bq * Np;
  if (RES) b += bq * Np;
  if (DOT) {
    dv += bq * Np;
    R = batch_reduce(R, (unsigned)bq);
  }
  const long long base = (long long)blockIdx.x * kChunk + 2 * threadIdx.x;
  double acc = 0.0;
#pragma unroll 1
  for (int m = 0; m < kPairsPerThread; ++m) {
    const long long i0 = base + 512LL * m;
    if (i0 >= N) break;
    const bool two = i0 + 1 < N;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const long long o = slot_off<D, P>(s, M);
      const double2 a = __ldg(reinterpret_cast<const double2*>(A + (long long)s * Np + i0));
      const double x0 = __ldg(x + clampi(i0 + o, N));
      const double x1 = __ldg(x + clampi(i0 + 1 + o, N));
      s0 = fma(a.x, x0, s0);
      s1 = fma(a.y, x1, s1);
    }
    double y0 = s0, y1 = s1;
    if (RES) {
      y0 = b[i0] - s0;
      if (two) y1 = b[i0 + 1] - s1;
    }
    y[i0] = y0;
    if (two) y[i0 + 1] = y1;
    if (DOT) {
      acc = fma(y0, dv[i0], acc);
      if (two) acc = fma(y1, dv[i0 + 1], acc);
    }
  }
  if (DOT) dr_finish(acc, R, smem);
}

// k_jacobi on a scalar Q2 level (the diagonal sits at the node's colour-major place)
template <int D>
__global__ void __launch_bounds__(kBlock)
k_jacobi_q2(const double* __restrict__ A, long long N, long long Np, long long M, double damp,
            const double* __restrict__ omega, double* x, double* r, int write_r, const __grid_constant__ Q2Layout lay) {
  constexpr int C = St<D, 2>::CENTER;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  long long c[3];
  node_coords32(i, M, D, c);
  const double t = r[i] / A[(long long)C * Np + q2c_pos<D>(lay, c, M, 0)];
  if (write_r) r[i] = t;
  x[i] = fma(omega ? omega[i] : damp, t, x[i]);
}

// ------------------------------------- Q2 rows by colour class and parity
// The row kernels of scalar Q2 levels give each block rows of one colour
// class and one parity pattern (bit k: coordinate k odd).  All rows of a
// warp then admit the same slots, so a row is a compile-time list of its
// stored slots -- no per-slot test, no divergence -- and a thread issues a
// whole z-plane of the stencil (up to 25 coefficient and 25 neighbour loads)
// before the plane's first multiply-add; the row sum still runs in slot
// order, skipping only structural zeros.  Along direction k the class (digit
// d = c mod 3) holds c = d + 3 j, j = 0 .. n-1; its rows of parity p are
// j = j0, j0 + 2, .. with j0 = (p + d) & 1.  Inside a class the coefficient
// arrays are contiguous, so a warp's loads of one slot stay within a few
// sectors.
constexpr int kQ2T = 128;  // threads per block
// matvec and Jacobi residual in 3D: four blocks per SM (at most 128
// registers: the batched loads of a stencil plane fit without spills, 16
// warps per SM instead of 12; the SOR sweep measured slower so)
template <int D>
constexpr int kQ2MinBlocks = D == 3 ? 4 : 1;

struct Q2Sub {
  int d[3], j0[3], n[3];  // class digit, first place and row count along each direction
  long long cnt;          // rows of the (class, parity) subgrid
};

template <int D>
__host__ __device__ __forceinline__ void q2_sub(int M, int colour, int pat, Q2Sub& s) {
  s.cnt = 1;
  int t = colour;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k < D) {
      const int d = t % 3, nk = (M - d + 2) / 3, j0 = (((pat >> k) & 1) + d) & 1;
      t /= 3;
      s.d[k] = d;
      s.j0[k] = j0;
      s.n[k] = nk > j0 ? (nk - j0 + 1) / 2 : 0;
    } else {
      s.d[k] = 0;
      s.j0[k] = 0;
      s.n[k] = 1;
    }
    s.cnt *= s.n[k];
  }
}

// blocks a class takes: its parity subgrids one after another
template <int D>
__host__ __device__ __forceinline__ long long q2_class_blocks(int M, int colour) {
  long long nb = 0;
  for (int pat = 0; pat < (1 << D); ++pat) {
    Q2Sub s;
    q2_sub<D>(M, colour, pat, s);
    nb += (s.cnt + kQ2T - 1) / kQ2T;
  }
  return nb;
}

// block blk of a class: its parity pattern, subgrid and this thread's row u
// in it; false when the thread has no row
template <int D>
__device__ __forceinline__ bool q2_block(int M, int colour, long long blk, int& pat, Q2Sub& s, long long& u) {
  for (pat = 0; pat < (1 << D); ++pat) {
    q2_sub<D>(M, colour, pat, s);
    const long long nb = (s.cnt + kQ2T - 1) / kQ2T;
    if (blk < nb) {
      u = blk * kQ2T + threadIdx.x;
      return u < s.cnt;
    }
    blk -= nb;
  }
  return false;
}

// a row's coordinates, node index and its positions in the arrays of every
// slot pattern (colour-major layout; patterns it does not admit are never read)
template <int D>
__device__ __forceinline__ long long q2_place(const Q2Layout& lay, int M, int colour, const Q2Sub& s, long long u,
                                              int c[3], int (&p)[1 << D]) {
  const unsigned uu = (unsigned)u;
  const unsigned q = D > 1 ? uu / (unsigned)s.n[0] : 0u;
  const int uk[3] = {(int)(D > 1 ? uu - q * (unsigned)s.n[0] : uu), D > 2 ? (int)(q % (unsigned)s.n[1]) : (int)q,
                     D > 2 ? (int)(q / (unsigned)s.n[1]) : 0};
  int j[3][2], e[3][2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k < D) {
      const int jj = s.j0[k] + 2 * uk[k], d = s.d[k], x0 = q2c_x0(d);
      c[k] = d + 3 * jj;
      j[k][0] = jj;
      e[k][0] = (M - d + 2) / 3;
      j[k][1] = (c[k] - x0) / 6;
      e[k][1] = x0 < M ? (M - x0 + 5) / 6 : 0;
    } else {
      c[k] = 0;
      j[k][0] = j[k][1] = 0;
      e[k][0] = e[k][1] = 1;
    }
  }
#pragma unroll
  for (int r = 0; r < (1 << D); ++r) {
    const int rx = r & 1, ry = (r >> 1) & 1, rz = (r >> 2) & 1;
    p[r] = (int)lay.off[r][colour] + j[0][rx] + e[0][rx] * (j[1][ry] + e[1][ry] * j[2][rz]);
  }
  return (long long)c[0] + (long long)M * (c[1] + (long long)M * c[2]);
}

// sum over the row's stored slots, in slot order, of A(i, s) x(i + off_s).
// PAT: the row's parity pattern.  Neighbour coordinates are clamped into the
// grid per direction (a slot reaching outside holds a zero).  XL: how x is
// read -- 0 plain loads (x is written by the kernel), 1 the read-only path
template <int D, int PAT, int XL>
__device__ __forceinline__ double q2_row_sum(const double* __restrict__ A, long long Np, const double* x, int M,
                                             const int c[3], const int (&p)[1 << D]) {
  int cl[3][5];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 0; o < 5; ++o) cl[k][o] = k < D ? min(max(c[k] + o - 2, 0), M - 1) : 0;
  constexpr int NZ = D > 2 ? 5 : 1, NY = D > 1 ? 5 : 1;
  double s = 0.0;
#pragma unroll
  for (int sz = 0; sz < NZ; ++sz) {
    const bool rz = D > 2 && (sz == 0 || sz == 4);
    if (rz && (PAT & 4)) continue;
    // the loads of a plane's rows 0-2, their multiply-adds, then rows 3-4
    // (at most 30 doubles in flight: the 3D kernels fit four or five blocks
    // per SM without spills); the sum stays in slot order
    double av[15], xv[15];
    int q = 0;
#pragma unroll
    for (int sy = 0; sy < NY; ++sy) {
      const bool ry = D > 1 && (sy == 0 || sy == 4);
      if (!(ry && (PAT & 2))) {
        const double* xl = x + (long long)M * (cl[1][sy] + (long long)M * cl[2][sz]);
#pragma unroll
        for (int sx = 0; sx < 5; ++sx) {
          const bool rx = sx == 0 || sx == 4;
          if (rx && (PAT & 1)) continue;
          const int slot = sx + 5 * (sy + 5 * sz);
          const int r = (rx ? 1 : 0) | (ry ? 2 : 0) | (rz ? 4 : 0);
          av[q] = __ldg(A + (long long)slot * Np + p[r]);
          xv[q] = XL == 1 ? __ldg(xl + cl[0][sx]) : xl[cl[0][sx]];
          ++q;
        }
      }
      if (sy == 2 || sy == NY - 1) {
#pragma unroll
        for (int k = 0; k < q; ++k) s = fma(av[k], xv[k], s);
        q = 0;
      }
    }
  }
  return s;
}

// calls f(integral_constant<int, pat>) for the runtime pattern pat
template <int D, typename F>
__device__ __forceinline__ void q2_pat_dispatch(int pat, F&& f) {
  switch (pat) {
    case 0: f(std::integral_constant<int, 0>{}); break;
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: if constexpr (D > 1) f(std::integral_constant<int, 2>{}); break;
    case 3: if constexpr (D > 1) f(std::integral_constant<int, 3>{}); break;
    case 4: if constexpr (D > 2) f(std::integral_constant<int, 4>{}); break;
    case 5: if constexpr (D > 2) f(std::integral_constant<int, 5>{}); break;
    case 6: if constexpr (D > 2) f(std::integral_constant<int, 6>{}); break;
    default: if constexpr (D > 2) f(std::integral_constant<int, 7>{}); break;
  }
}

// the rows of block blk of colour class `colour` in the multicolour <sor>
// sweep of a scalar Q2 level (linit.lisp:288-323): r = (b - A x)/d, x += w r
template <int D, int XL>
__device__ __forceinline__ void sor_q2_block(const double* __restrict__ A, long long Np, int M, int colour,
                                             long long blk, double omega_s, const double* __restrict__ omega,
                                             double* x, const double* b, double* r, const Q2Layout& lay) {
  int pat;
  Q2Sub sub;
  long long u;
  if (!q2_block<D>(M, colour, blk, pat, sub, u)) return;
  int c[3], p[1 << D];
  const long long i = q2_place<D>(lay, M, colour, sub, u, c, p);
  constexpr int C = St<D, 2>::CENTER;
  // the row's own operands first, so that their loads overlap the stencil's
  const double d = __ldg(A + (long long)C * Np + p[0]);
  const double bi = b[i], xi = x[i], wi = omega ? __ldg(omega + i) : omega_s;
  double s = 0.0;
  q2_pat_dispatch<D>(pat, [&](auto P) { s = q2_row_sum<D, decltype(P)::value, XL>(A, Np, x, M, c, p); });
  const double tt = (bi - s) / d;
  r[i] = tt;
  x[i] = fma(wi, tt, xi);
}

// one colour of the sweep per launch
template <int D>
__global__ void __launch_bounds__(kQ2T)
k_sor_q2(const double* __restrict__ A, long long Np, int M, int colour, double omega_s,
         const double* __restrict__ omega, double* x, const double* b, double* r,
         const __grid_constant__ Q2Layout lay) {
  sor_q2_block<D, 0>(A, Np, M, colour, blockIdx.x, omega_s, omega, x, b, r, lay);
}

// y = A x or r = b - A x on a scalar Q2 level, rows by class (blockIdx.y) and parity
template <int D, bool RES>
__global__ void __launch_bounds__(kQ2T, kQ2MinBlocks<D>)
k_spmv_q2c(const double* __restrict__ A, long long Np, int M, const double* __restrict__ x, const double* b,
           double* y, const __grid_constant__ Q2Layout lay) {
  int pat;
  Q2Sub sub;
  long long u;
  const int colour = (int)blockIdx.y;
  if (!q2_block<D>(M, colour, blockIdx.x, pat, sub, u)) return;
  int c[3], p[1 << D];
  const long long i = q2_place<D>(lay, M, colour, sub, u, c, p);
  double s = 0.0;
  q2_pat_dispatch<D>(pat, [&](auto P) { s = q2_row_sum<D, decltype(P)::value, 1>(A, Np, x, M, c, p); });
  y[i] = RES ? b[i] - s : s;
}

// k_jacobi_res on a scalar Q2 level, rows by class and parity
template <int D>
__global__ void __launch_bounds__(kQ2T, kQ2MinBlocks<D>)
k_jacobi_res_q2c(const double* __restrict__ A, long long Np, int M, double damp, const double* __restrict__ omega,
                 const double* __restrict__ x, const double* b, double* __restrict__ xout, double* r, int write_r,
                 const __grid_constant__ Q2Layout lay) {
  int pat;
  Q2Sub sub;
  long long u;
  const int colour = (int)blockIdx.y;
  if (!q2_block<D>(M, colour, blockIdx.x, pat, sub, u)) return;
  int c[3], p[1 << D];
  const long long i = q2_place<D>(lay, M, colour, sub, u, c, p);
  constexpr int C = St<D, 2>::CENTER;
  const double d = __ldg(A + (long long)C * Np + p[0]);
  double s = 0.0;
  q2_pat_dispatch<D>(pat, [&](auto P) { s = q2_row_sum<D, decltype(P)::value, 1>(A, Np, x, M, c, p); });
  const double t = (b[i] - s) / d;
  if (write_r) r[i] = t;
  xout[i] = fma(omega ? omega[i] : damp, t, x[i]);
}

// ------------------------------------------------------------- smoothers
// <jacobi> step with an up-to-date residual: t = r/d, x += w t, r := t
__global__ void __launch_bounds__(kBlock)
k_jacobi(const double* __restrict__ Dg, long long N, double damp, const double* __restrict__ omega,
         double* x, double* r, int write_r, long long vs = 0, long long as = 0) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const long long bq = blockIdx.y;  // problem of a batched level: vector stride vs, matrix stride as
  Dg += bq * as;
  x += bq * vs;
  r += bq * vs;
  if (omega) omega += bq * vs;
  const double t = r[i] / Dg[i];
  if (write_r) r[i] = t;
  const double w = omega ? omega[i] : damp;
  x[i] = fma(w, t, x[i]);
}

// compute-residual fused with the following <jacobi> step:
// t = (b - A x)/d, xout = x + w t, r := t; optional fused (xout, dv) reduction
template <int D, int P, bool DOT>
__global__ void __launch_bounds__(kBlock)
k_jacobi_res(const double* __restrict__ A, long long N, long long Np, long long M, double damp,
             const double* __restrict__ omega, const double* __restrict__ x, const double* b,
             double* __restrict__ xout, double* r, int write_r, const double* __restrict__ dv,
             Reduce R) {
  constexpr int NS = St<D, P>::NS;
  constexpr int C = St<D, P>::CENTER;
  __shared__ double smem[8];
  const long long bq = blockIdx.y;  // problem of a batched level
  A += bq * NS * Np;
  x += bq * Np;
  b += bq * Np;
  xout += bq * Np;
  r += bq * Np;
  if (omega) omega += bq * Np;
  if (DOT) {
    dv += bq * Np;
    R = batch_reduce(R, (unsigned)bq);
  }
  const long long base = (long long)blockIdx.x * kChunk + 2 * threadIdx.x;
  double acc = 0.0;
#pragma unroll 1
  for (int m = 0; m < kPairsPerThread; ++m) {
    const long long i0 = base + 512LL * m;
    if (i0 >= N) break;
    const bool two = i0 + 1 < N;
    double s0 = 0.0, s1 = 0.0, d0 = 1.0, d1 = 1.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const long long o = slot_off<D, P>(s, M);
      const double2 a = __ldg(reinterpret_cast<const double2*>(A + (long long)s * Np + i0));
      if (s == C) { d0 = a.x; d1 = a.y; }
      const double x0 = __ldg(x + clampi(i0 + o, N));
      const double x1 = __ldg(x + clampi(i0 + 1 + o, N));
      s0 = fma(a.x, x0, s0);
      s1 = fma(a.y, x1, s1);
    }
    {
      const double t = (b[i0] - s0) / d0;
      if (write_r) r[i0] = t;
      const double xn = fma(omega ? omega[i0] : damp, t, x[i0]);
      xout[i0] = xn;
      if (DOT) acc = fma(xn, dv[i0], acc);
    }
    if (two) {
      const double t = (b[i0 + 1] - s1) / d1;
      if (write_r) r[i0 + 1] = t;
      const double xn = fma(omega ? omega[i0 + 1] : damp, t, x[i0 + 1]);
      xout[i0 + 1] = xn;
      if (DOT) acc = fma(xn, dv[i0 + 1], acc);
    }
  }
  if (DOT) dr_finish(acc, R, smem);
}

// one colour of the multicolour <sor> sweep on a Q1 level (P = 1): rows with
// (i_k mod (P+1)) = col_k (scalar Q2 levels: k_sor_q2).
// SSC: the <geometric-ssc> sweep of a Q1 level, whose vertex blocks hold one
// node -- the same update, with r keeping the unscaled residual
// (blockit.lisp:131-138) instead of the <sor> correction (linit.lisp:312-322)
template <int D, int P, bool SSC = false>
__global__ void __launch_bounds__(kBlock)
k_sor_colour(const double* __restrict__ A, long long N, long long Np, long long M, int colour,
             double omega_s, const double* __restrict__ omega, double* x, const double* b, double* r) {
  constexpr int NS = St<D, P>::NS;
  constexpr int C = St<D, P>::CENTER;
  constexpr int Q = P + 1;
  const int cx = colour % Q, cy = (colour / Q) % Q, cz = colour / (Q * Q);
  const long long nx = (M - cx + Q - 1) / Q;
  const long long ny = D > 1 ? (M - cy + Q - 1) / Q : 1;
  const long long nz = D > 2 ? (M - cz + Q - 1) / Q : 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny * nz) return;
  const unsigned tu = (unsigned)t, nxu = (unsigned)nx, nyu = (unsigned)ny;
  const unsigned tq = tu / nxu;
  const long long jx = tu - tq * nxu, jy = tq % nyu, jz = tq / nyu;
  const long long i = (cx + Q * jx) + M * ((D > 1 ? cy + Q * jy : 0) + M * (D > 2 ? cz + Q * jz : 0));
  double s = 0.0, d = 1.0;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const long long o = slot_off<D, P>(k, M);
    const double a = A[(long long)k * Np + i];
    if (k == C) d = a;
    s = fma(a, x[clampi(i + o, N)], s);
  }
  const double rr = b[i] - s;
  const double tt = rr / d;
  r[i] = SSC ? rr : tt;
  x[i] = fma(omega ? omega[i] : omega_s, tt, x[i]);
}

// Step K of the warp's LU factorisation of a vertex block (rows in lanes):
// the pivot is the first position holding the largest magnitude, the lane at
// position K and the pivot's lane exchange positions (the rows stay put), the
// rows below keep their multiplier in column K.  The recursion keeps every
// index a compile-time constant, so the row stays in registers.
template <int NB, int K>
__device__ __forceinline__ void ssc_lu_step(double (&a)[NB], int& pos, int lane) {
  if constexpr (K < NB) {
    constexpr unsigned FULL = 0xffffffffu;
    double val = (lane < NB && pos >= K) ? fabs(a[K]) : -1.0;
    int key = pos, ln = lane;
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
      const double ov = __shfl_xor_sync(FULL, val, m);
      const int ok = __shfl_xor_sync(FULL, key, m);
      const int ol = __shfl_xor_sync(FULL, ln, m);
      if (ov > val || (ov == val && ok < key)) { val = ov; key = ok; ln = ol; }
    }
    if (pos == K) pos = key;  // row interchange
    if (lane == ln) pos = K;
    const double piv = __shfl_sync(FULL, a[K], ln);
    const double rcp = 1.0 / piv;
    const bool below = lane < NB && pos > K;
    const double mlt = a[K] * rcp;
#pragma unroll
    for (int j = K + 1; j < NB; ++j) {
      const double pj = __shfl_sync(FULL, a[j], ln);
      if (below) a[j] = a[j] - mlt * pj;
    }
    if (below) a[K] = mlt;
    ssc_lu_step<NB, K + 1>(a, pos, lane);
  }
}

// Column K of the forward substitution with the stored unit lower factor:
// the row at position K is final, the rows below subtract their multiplier
// times it (the operations, in order, of carrying the right-hand side
// through the elimination).
template <int NB, int K>
__device__ __forceinline__ void ssc_fwd_step(const double (&a)[NB], double& rr, int pos, int lane) {
  if constexpr (K < NB) {
    constexpr unsigned FULL = 0xffffffffu;
    const unsigned who = __ballot_sync(FULL, lane < NB && pos == K);
    const double rk = __shfl_sync(FULL, rr, __ffs(who) - 1);
    if (lane < NB && pos > K) rr = rr - a[K] * rk;
    ssc_fwd_step<NB, K + 1>(a, rr, pos, lane);
  }
}

// Column K of the backward substitution: the lane at position K divides,
// the rows above subtract; the lane of member K keeps the solution.
template <int NB, int K>
__device__ __forceinline__ void ssc_back_step(const double (&a)[NB], double& rr, int pos, int lane, double& corr) {
  if constexpr (K >= 0) {
    constexpr unsigned FULL = 0xffffffffu;
    const unsigned who = __ballot_sync(FULL, lane < NB && pos == K);
    const int kl = __ffs(who) - 1;
    const double xk = __shfl_sync(FULL, rr / a[K], kl);
    if (lane < NB && pos < K) rr = rr - xk * a[K];
    if (lane == K) corr = xk;
    ssc_back_step<NB, K - 1>(a, rr, pos, lane, corr);
  }
}

// Member `lane` of the vertex block of vertex v (2 x vertex index): its node
// coordinates and offsets, whether it is in the domain, and whether it is a
// member of the block (the vertex itself, or a non-Dirichlet node).
template <int D>
struct SscMember {
  int dm[3], c[3];
  bool real;
};

template <int D>
__device__ __forceinline__ SscMember<D> ssc_member(const int v[3], int lane, int Mi, int dmask) {
  constexpr int NB = D == 1 ? 3 : (D == 2 ? 9 : 27);
  SscMember<D> m;
  bool in = lane < NB, dir = false;
#pragma unroll
  for (int k = 0; k < 3; ++k) { m.dm[k] = 0; m.c[k] = v[k]; }
#pragma unroll
  for (int k = 0, q = lane; k < D; ++k, q /= 3) {
    m.dm[k] = q % 3 - 1;
    m.c[k] = v[k] + m.dm[k];
    in = in && m.c[k] >= 0 && m.c[k] < Mi;
    dir = dir || (m.c[k] == 0 && ((dmask >> (2 * k)) & 1)) || (m.c[k] == Mi - 1 && ((dmask >> (2 * k + 1)) & 1));
  }
  m.real = in && (lane == NB / 2 || !dir);
  return m;
}

// The LU factors of every vertex block of a scalar Q2 level (all colours in
// one launch), for the <geometric-ssc> sweeps: the local matrix A_BB
// (blockit.lisp:150-153) gathered by the member lanes -- every entry lies in
// a pattern-0 slot: a row that is odd along a direction meets the box only
// within +-1 there -- members outside the domain, and Dirichlet members
// other than the vertex, as identity rows with zero columns (the pivots and
// the arithmetic of the real rows are those of the compact block), then
// factored as by gesv! (right-looking, partial pivoting).  The factors depend
// on the matrix only, so a sweep that reuses them repeats exactly the
// operations of factoring afresh.  Layout: F[block][k][member], the row's
// final position in P[block][member]; block = lexicographic vertex index.
template <int D>
__global__ void __launch_bounds__(128)
k_ssc_factor_q2(const double* __restrict__ A, long long Np, long long M, int dmask, double* F, unsigned char* P,
                const __grid_constant__ Q2Layout lay) {
  constexpr int NB = D == 1 ? 3 : (D == 2 ? 9 : 27);
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // uniform per warp
  const int Mi = (int)M;
  const int nv = (Mi + 1) / 2;
  const long long nblk = D == 1 ? nv : (D == 2 ? (long long)nv * nv : (long long)nv * nv * nv);
  if (w >= nblk) return;  // the whole warp leaves together
  const int wi = (int)w;
  const int v[3] = {2 * (wi % nv), D > 1 ? 2 * ((wi / nv) % nv) : 0, D > 2 ? 2 * (wi / (nv * nv)) : 0};
  const SscMember<D> mb = ssc_member<D>(v, lane, Mi, dmask);
  const unsigned realmask = __ballot_sync(FULL, mb.real);
  double a[NB];
  if (mb.real) {
    const long long cl[3] = {mb.c[0], mb.c[1], mb.c[2]};
    Q2Base<D> qb;
    q2_base<D, true, true>(lay, cl, M, qb);
    const long long p0 = qb.p[0];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      bool near = true;
      int sl = 0;
#pragma unroll
      for (int k = 0, q = u, m5 = 1; k < D; ++k, q /= 3, m5 *= 5) {
        const int o = (q % 3 - 1) - mb.dm[k];
        near = near && o >= -1 && o <= 1;
        sl += (o + 2) * m5;
      }
      a[u] = (near && ((realmask >> u) & 1)) ? A[(long long)sl * Np + p0] : 0.0;
    }
  } else {
#pragma unroll
    for (int u = 0; u < NB; ++u) a[u] = (u == lane) ? 1.0 : 0.0;
  }
  int pos = lane;  // lanes >= NB are never candidates
  ssc_lu_step<NB, 0>(a, pos, lane);
  if (lane < NB) {
    double* f = F + w * NB * NB + lane;
#pragma unroll
    for (int k = 0; k < NB; ++k) f[k * NB] = a[k];
    P[w * NB + lane] = (unsigned char)pos;
  }
}

// One colour of the <geometric-ssc> sweep on a scalar Q2 level
// (blockit.lisp:118-204 with the vertex-centred blocks of geoblock.lisp:72-158):
// a warp per vertex block, lane t holding member t of the 3^D box around the
// vertex (x fastest).  Each member lane forms its row's residual r = b - A x
// (b may alias r: the alias inside <cg>), then the warp solves A_BB c = r_B
// with the stored factors (forward in position order, backward column by
// column) and x_B += omega c.  Blocks of one colour (vertex index mod 2 per
// direction) share no node and read no unknown another one writes.
template <int D>
__global__ void __launch_bounds__(128, 6)
k_ssc_q2(const double* __restrict__ A, long long N, long long Np, long long M, int dmask, int colour,
         double omega, double* x, const double* b, double* r, const double* __restrict__ F,
         const unsigned char* __restrict__ P, const __grid_constant__ Q2Layout lay) {
  constexpr int NB = D == 1 ? 3 : (D == 2 ? 9 : 27);
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // uniform per warp
  const int Mi = (int)M;
  const int nv = (Mi + 1) / 2;  // vertices per direction
  const int bx = colour & 1, by = (colour >> 1) & 1, bz = (colour >> 2) & 1;
  const int ex = (nv - bx + 1) / 2, ey = D > 1 ? (nv - by + 1) / 2 : 1, ez = D > 2 ? (nv - bz + 1) / 2 : 1;
  if (w >= (long long)ex * ey * ez) return;  // the whole warp leaves together
  const int wi = (int)w;
  const int jx = wi % ex, jq = wi / ex, jy = jq % ey, jz = jq / ey;
  const int ax = bx + 2 * jx, ay = D > 1 ? by + 2 * jy : 0, az = D > 2 ? bz + 2 * jz : 0;
  const int v[3] = {2 * ax, 2 * ay, 2 * az};
  const long long blk = ax + (long long)nv * (ay + (long long)nv * az);
  const SscMember<D> mb = ssc_member<D>(v, lane, Mi, dmask);
  // the unknowns the block's rows read: the 7^D nodes within 3 of the
  // vertex, staged in shared memory (0 outside the domain, where the rows'
  // stored coefficients are 0 as well)
  constexpr int W7 = D == 1 ? 7 : (D == 2 ? 49 : 343);
  __shared__ double xs_all[4][W7];
  double* xs = xs_all[threadIdx.x >> 5];
  for (int e = lane; e < W7; e += 32) {
    const int lx = e % 7, ly = (e / 7) % 7, lz = e / 49;
    const int gx = v[0] + lx - 3, gy = D > 1 ? v[1] + ly - 3 : 0, gz = D > 2 ? v[2] + lz - 3 : 0;
    const bool inside = gx >= 0 && gx < Mi && (D < 2 || (gy >= 0 && gy < Mi)) && (D < 3 || (gz >= 0 && gz < Mi));
    xs[e] = inside ? x[gx + M * ((long long)gy + M * (long long)gz)] : 0.0;
  }
  __syncwarp();
  const long long i = mb.real ? (long long)mb.c[0] + M * ((long long)mb.c[1] + M * (long long)mb.c[2]) : 0;
  double rr = 0.0;
  if (mb.real) {
    const long long cl[3] = {mb.c[0], mb.c[1], mb.c[2]};
    Q2Base<D> qb;
    q2_base<D, true, true>(lay, cl, M, qb);
    const int lc = (mb.dm[0] + 3) + 7 * (D > 1 ? mb.dm[1] + 3 : 0) + 49 * (D > 2 ? mb.dm[2] + 3 : 0);
    double s = 0.0;
    q2_visit<D, true>(qb, M, [&](int k, long long, long long p, bool st) {
      double av = A[(long long)k * Np + p];
      av = st ? av : 0.0;
      const int lo = (k % 5 - 2) + (D > 1 ? 7 * ((k / 5) % 5 - 2) : 0) + (D > 2 ? 49 * (k / 25 - 2) : 0);
      s = fma(av, xs[lc + lo], s);
    });
    rr = b[i] - s;
    r[i] = rr;
  }
  double a[NB];
  int pos = lane;
  if (lane < NB) {
    const double* f = F + blk * NB * NB + lane;
#pragma unroll
    for (int k = 0; k < NB; ++k) a[k] = __ldg(f + k * NB);
    pos = P[blk * NB + lane];
  } else {
#pragma unroll
    for (int k = 0; k < NB; ++k) a[k] = 0.0;
  }
  ssc_fwd_step<NB, 0>(a, rr, pos, lane);
  double corr = 0.0;
  ssc_back_step<NB, NB - 1>(a, rr, pos, lane, corr);
  if (mb.real) x[i] = fma(omega, corr, x[i]);
}

// <geometric-psc> on a scalar Q1 level: one-node blocks, x_i += damp r_i /
// a_ii (the 1 x 1 LU divides by the pivot), r unchanged
template <int D>
__global__ void __launch_bounds__(kBlock)
k_psc_q1(const double* __restrict__ A, long long N, long long Np, double damp, double* x, const double* r) {
  constexpr int C = St<D, 1>::CENTER;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  x[i] = fma(damp, r[i] / A[(long long)C * Np + i], x[i]);
}

// <geometric-psc> on a scalar Q2 level, first pass: every vertex block (warp
// per block, all blocks in one launch) solves A_BB c = r_B with the stored
// factors and the residual as it stands (r is read, not written); member t's
// correction goes to C[block][t] (zero for padded members).
template <int D>
__global__ void __launch_bounds__(128, 6)
k_psc_block_q2(long long M, int dmask, const double* __restrict__ r, const double* __restrict__ F,
               const unsigned char* __restrict__ P, double* __restrict__ C) {
  constexpr int NB = D == 1 ? 3 : (D == 2 ? 9 : 27);
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // uniform per warp
  const int Mi = (int)M;
  const int nv = (Mi + 1) / 2;
  const long long nblk = D == 1 ? nv : (D == 2 ? (long long)nv * nv : (long long)nv * nv * nv);
  if (w >= nblk) return;  // the whole warp leaves together
  const int wi = (int)w;
  const int v[3] = {2 * (wi % nv), D > 1 ? 2 * ((wi / nv) % nv) : 0, D > 2 ? 2 * (wi / (nv * nv)) : 0};
  const SscMember<D> mb = ssc_member<D>(v, lane, Mi, dmask);
  double rr = mb.real ? r[(long long)mb.c[0] + M * ((long long)mb.c[1] + M * (long long)mb.c[2])] : 0.0;
  double a[NB];
  int pos = lane;
  if (lane < NB) {
    const double* f = F + w * NB * NB + lane;
#pragma unroll
    for (int k = 0; k < NB; ++k) a[k] = __ldg(f + k * NB);
    pos = P[w * NB + lane];
  } else {
#pragma unroll
    for (int k = 0; k < NB; ++k) a[k] = 0.0;
  }
  ssc_fwd_step<NB, 0>(a, rr, pos, lane);
  double corr = 0.0;
  ssc_back_step<NB, NB - 1>(a, rr, pos, lane, corr);
  if (lane < NB) C[w * NB + lane] = corr;
}

// second pass: node i adds, in increasing vertex order, damp times its
// correction from each block holding it as a member (the vertices within 1
// of it along every direction; a Dirichlet node belongs to its own block only)
template <int D>
__global__ void __launch_bounds__(kBlock)
k_psc_gather_q2(long long N, long long M, int dmask, double damp, const double* __restrict__ C, double* x) {
  constexpr int NB = D == 1 ? 3 : (D == 2 ? 9 : 27);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int Mi = (int)M, nv = (Mi + 1) / 2;
  int c[3] = {(int)(i % M), D > 1 ? (int)((i / M) % M) : 0, D > 2 ? (int)(i / (M * M)) : 0};
  bool dir = false;
#pragma unroll
  for (int k = 0; k < D; ++k)
    dir = dir || (c[k] == 0 && ((dmask >> (2 * k)) & 1)) || (c[k] == Mi - 1 && ((dmask >> (2 * k + 1)) & 1));
  // candidate vertex coordinates per direction, ascending
  int vc[3][2], nvc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    nvc[k] = 1;
    vc[k][0] = vc[k][1] = 0;
    if (k >= D) continue;
    if (c[k] & 1) {
      nvc[k] = 2;
      vc[k][0] = c[k] - 1;
      vc[k][1] = c[k] + 1;
    } else {
      vc[k][0] = c[k];
    }
  }
  double xi = x[i];
  for (int iz = 0; iz < nvc[2]; ++iz)
    for (int iy = 0; iy < nvc[1]; ++iy)
      for (int ix = 0; ix < nvc[0]; ++ix) {
        const int vx = vc[0][ix], vy = vc[1][iy], vz = vc[2][iz];
        const bool own = vx == c[0] && (D < 2 || vy == c[1]) && (D < 3 || vz == c[2]);  // i is the vertex
        if (dir && !own) continue;
        const long long blk = (vx >> 1) + (long long)nv * ((vy >> 1) + (long long)nv * (vz >> 1));
        int t = c[0] - vx + 1;
        if (D > 1) t += 3 * (c[1] - vy + 1);
        if (D > 2) t += 9 * (c[2] - vz + 1);
        xi = fma(damp, C[blk * NB + t], xi);
      }
  x[i] = xi;
}

// ------------------------------------------------------ algebraic levels
// Compressed-row forms of the level operators (matrices handed over by the
// host, e.g. from sparse-matrix->ccs on an unstructured or adaptive mesh).
// Each row sums its entries in stored (column-ascending) order with fma, the
// order in which the stencil forms sum their slots, so a structured level
// given as compressed rows yields the structured results bit for bit.

// y = A x, or r = b - A x (b may alias r)
__global__ void __launch_bounds__(kBlock)
k_csr_spmv(long long N, CsrView a, const double* __restrict__ x, const double* b, double* y, int res) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = 0.0;
  for (long long e = a.start[i]; e < a.start[i + 1]; ++e) s = fma(a.value[e], __ldg(x + a.index[e]), s);
  y[i] = res ? b[i] - s : s;
}

// compute-residual fused with the following <jacobi> step (as k_jacobi_res)
__global__ void __launch_bounds__(kBlock)
k_csr_jacobi_res(long long N, CsrView a, const double* __restrict__ diag, double damp,
                 const double* __restrict__ omega, const double* __restrict__ x, const double* b,
                 double* __restrict__ xout, double* r, int write_r) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = 0.0;
  for (long long e = a.start[i]; e < a.start[i + 1]; ++e) s = fma(a.value[e], __ldg(x + a.index[e]), s);
  const double t = (b[i] - s) / diag[i];
  if (write_r) r[i] = t;
  xout[i] = fma(omega ? omega[i] : damp, t, x[i]);
}

// one colour of the SOR (SSC = false: r := the scaled correction, the
// <sor> of linit.lisp:288-323) or point-block SSC sweep (r := the residual,
// blockit.lisp:131-138) of an algebraic level: rows of the colour in any
// order (they couple to none of each other), the row sum over the stored
// entries, columns ascending
__global__ void __launch_bounds__(kBlock)
k_csr_sor(const int* __restrict__ rows, long long cnt, CsrView a, const double* __restrict__ diag, double omega_s,
          const double* __restrict__ omega, double* x, const double* b, double* r, int ssc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const long long i = rows[t];
  double s = 0.0;
  for (long long e = a.start[i]; e < a.start[i + 1]; ++e) s = fma(a.value[e], x[a.index[e]], s);
  const double rr = b[i] - s;
  const double tt = rr / diag[i];
  r[i] = ssc ? rr : tt;
  x[i] = fma(omega ? omega[i] : omega_s, tt, x[i]);
}

// rc = I^T rf row by row of I^T (fine entries ascending); the coarse rhs
// takes rc, the coarse solution 0 (the :after methods of restrict)
__global__ void __launch_bounds__(kBlock)
k_csr_restrict(long long NC, CsrView pt, const double* __restrict__ rf, double* rc, double* rhsc, double* solc) {
  const long long J = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (J >= NC) return;
  double s = 0.0;
  for (long long e = pt.start[J]; e < pt.start[J + 1]; ++e) s = fma(pt.value[e], __ldg(rf + pt.index[e]), s);
  rc[J] = s;
  if (rhsc) rhsc[J] = s;
  if (solc) solc[J] = 0.0;
}

// xf += I xc (coarse entries ascending)
__global__ void __launch_bounds__(kBlock)
k_csr_prolong(long long NF, CsrView p, const double* __restrict__ xc, double* xf) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NF || p.start[i] == p.start[i + 1]) return;  // constrained rows keep their value
  double s = 0.0;
  for (long long e = p.start[i]; e < p.start[i + 1]; ++e) s = fma(p.value[e], __ldg(xc + p.index[e]), s);
  xf[i] = xf[i] + s;
}

// the level matrix as a dense row-major n x n array (zeros written beforehand)
__global__ void __launch_bounds__(kBlock) k_csr_densify(long long N, CsrView a, double* Dm) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (long long e = a.start[i]; e < a.start[i + 1]; ++e) Dm[i * N + a.index[e]] = a.value[e];
}

// -------------------------------------------------------------- transfers
template <int P>
__device__ __forceinline__ int restrict_1d(long long J, long long* off, double* w) {
  if (P == 1) { off[0] = -1; off[1] = 0; off[2] = 1; w[0] = 0.5; w[1] = 1.0; w[2] = 0.5; return 3; }
  if ((J & 1) == 0) {
    off[0] = -3; off[1] = -1; off[2] = 0; off[3] = 1; off[4] = 3;
    w[0] = -0.125; w[1] = 0.375; w[2] = 1.0; w[3] = 0.375; w[4] = -0.125;
    return 5;
  }
  off[0] = -1; off[1] = 0; off[2] = 1; w[0] = 0.75; w[1] = 1.0; w[2] = 0.75;
  return 3;
}

template <int P>
__device__ __forceinline__ int prolong_1d(long long I, long long* J, double* w) {
  if ((I & 1) == 0) { J[0] = I / 2; w[0] = 1.0; return 1; }
  if (P == 1) { J[0] = (I - 1) / 2; J[1] = (I + 1) / 2; w[0] = 0.5; w[1] = 0.5; return 2; }
  const long long c = I / 4;
  const double s = (double)(I - 4 * c) / 4.0;
  J[0] = 2 * c; J[1] = 2 * c + 1; J[2] = 2 * c + 2;
  w[0] = 2.0 * (s - 0.5) * (s - 1.0);
  w[1] = 4.0 * s * (1.0 - s);
  w[2] = 2.0 * s * (s - 0.5);
  return 3;
}

// Launch shape of the transfer kernels: blocks (32, 8) over x and y, one z
// plane per blockIdx.z, 32-bit node coordinates (levels have < 2^31 nodes).
__device__ __forceinline__ bool face_dir(int c, int M, int k, int dmask) {
  return (c == 0 && ((dmask >> (2 * k)) & 1)) || (c == M - 1 && ((dmask >> (2 * k + 1)) & 1));
}

// rc := I^T rf (constrained), rhs_c := rc, sol_c := 0 (restrict + its :after
// methods for the correction scheme, multigrid.lisp:202-224)
template <int D, int P>
__global__ void __launch_bounds__(kBlock)
k_restrict(int MC, int MF, int dmask, const double* __restrict__ rf, double* __restrict__ rc,
           double* __restrict__ rhsc, double* __restrict__ solc, long long fs = 0, long long cs = 0) {
  if (D == 1 && threadIdx.y != 0) return;
  if (D < 3) {  // problem of a batched level: fine stride fs, coarse stride cs
    const long long bq = blockIdx.z;
    rf += bq * fs;
    rc += bq * cs;
    rhsc += bq * cs;
    solc += bq * cs;
  }
  const int cJ[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (cJ[0] >= MC || cJ[1] >= MC) return;
  const long long J = cJ[0] + (long long)MC * (cJ[1] + (long long)MC * cJ[2]);
  bool dj = false;
  for (int k = 0; k < D; ++k) dj = dj || face_dir(cJ[k], MC, k, dmask);
  double acc = 0.0;
  if (!dj) {
    long long off[3][5] = {{0}, {0}, {0}};
    double w[3][5] = {{1.0}, {1.0}, {1.0}};
    int cnt[3] = {1, 1, 1};
    for (int k = 0; k < D; ++k) cnt[k] = restrict_1d<P>(cJ[k], off[k], w[k]);
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int xx = 0; xx < cnt[0]; ++xx) {
          const int fi[3] = {2 * cJ[0] + (int)off[0][xx], 2 * cJ[1] + (int)off[1][y], 2 * cJ[2] + (int)off[2][z]};
          bool skip = false;
          for (int k = 0; k < D; ++k) skip = skip || fi[k] < 0 || fi[k] >= MF || face_dir(fi[k], MF, k, dmask);
          if (skip) continue;
          double ww = w[0][xx];
          if (D > 1) ww = ww * w[1][y];
          if (D > 2) ww = ww * w[2][z];
          acc = fma(ww, rf[fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2])], acc);
        }
  }
  rc[J] = acc;
  rhsc[J] = acc;
  solc[J] = 0.0;
}

// xf := xf + I xc (constrained) (prolongate, multigrid.lisp:237-239)
template <int D, int P>
__global__ void __launch_bounds__(kBlock)
k_prolong(int MF, int MC, int dmask, const double* __restrict__ xc, double* __restrict__ xf, long long fs = 0,
          long long cs = 0) {
  if (D == 1 && threadIdx.y != 0) return;
  if (D < 3) {  // problem of a batched level
    const long long bq = blockIdx.z;
    xc += bq * cs;
    xf += bq * fs;
  }
  const int fi[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (fi[0] >= MF || fi[1] >= MF) return;
  for (int k = 0; k < D; ++k)
    if (face_dir(fi[k], MF, k, dmask)) return;
  const long long i = fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2]);
  long long J[3][3] = {{0}, {0}, {0}};
  double w[3][3] = {{1.0}, {1.0}, {1.0}};
  int cnt[3] = {1, 1, 1};
  for (int k = 0; k < D; ++k) cnt[k] = prolong_1d<P>(fi[k], J[k], w[k]);
  double acc = 0.0;
  for (int z = 0; z < cnt[2]; ++z)
    for (int y = 0; y < cnt[1]; ++y)
      for (int xx = 0; xx < cnt[0]; ++xx) {
        const int cj[3] = {(int)J[0][xx], (int)J[1][y], (int)J[2][z]};
        bool dj = false;
        for (int k = 0; k < D; ++k) dj = dj || face_dir(cj[k], MC, k, dmask);
        if (dj) continue;
        double ww = w[0][xx];
        if (D > 1) ww = ww * w[1][y];
        if (D > 2) ww = ww * w[2][z];
        acc = fma(ww, xc[cj[0] + (long long)MC * (cj[1] + (long long)MC * cj[2])], acc);
      }
  xf[i] = xf[i] + acc;
}

// -------------------------------------------------------------- coarse LU
// The dense LU with partial pivoting of the base level and its explicit
// inverse (the <lu> coarse-grid iteration; the oracle's dense LU).  Every
// form below performs, for every element, the operations of the unblocked
// right-looking loop in the same order -- pivot: the first row holding the
// largest magnitude among the rows not yet eliminated; multiplier: column
// entry / pivot; update: a_ij = fma(-l_ik, a_kj, a_ij) for k ascending;
// inverse: the interchanges, then per column the unit-lower forward and the
// upper backward substitution (x_k = b_k / u_kk, then b_i = fma(-u_ik, x_k,
// b_i) for the rows above) -- so factors, pivots and inverse are the same bit
// for bit whichever form runs.
//
// Blocked form for matrices beyond shared memory: panels of kLuB columns,
// rows interchanged through a logical permutation (physical rows stay put).
constexpr int kLuB = 32;

// the panel k0..k1-1: per column the pivot (the first logical row holding the
// largest magnitude), the interchange, and the updates of the panel's later
// columns; the multipliers (column / pivot) are stored one step later, and
// the panel's last column's after the loop
__global__ void __launch_bounds__(1024) k_lu_panel(double* A, int n, int k0, int k1, int* piv, int* perm) {
  __shared__ double bv[32];
  __shared__ int bi[32];
  const int tid = threadIdx.x, nt = blockDim.x;
  double dprev = 1.0;
  for (int k = k0; k < k1; ++k) {
    double best = -1.0;
    int besti = n;
    for (int i = k + tid; i < n; i += nt) {
      const double v = fabs(A[(long long)perm[i] * n + k]);
      if (v > best || (v == best && i < besti)) { best = v; besti = i; }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
      if (ov > best || (ov == best && oi < besti)) { best = ov; besti = oi; }
    }
    if ((tid & 31) == 0) { bv[tid >> 5] = best; bi[tid >> 5] = besti; }
    __syncthreads();
    if (tid == 0) {
      double b = bv[0];
      int ib = bi[0];
      for (int w = 1; w < (nt + 31) / 32; ++w)
        if (bv[w] > b || (bv[w] == b && bi[w] < ib)) { b = bv[w]; ib = bi[w]; }
      piv[k] = ib;
      const int t = perm[k];
      perm[k] = perm[ib];
      perm[ib] = t;
    }
    __syncthreads();
    const long long pr = perm[k];
    const double d = A[pr * n + k];
    const int m = n - k - 1, w = k1 - k - 1;
    const long long mw = (long long)m * w, nprev = k > k0 ? n - k : 0;  // previous column: logical rows k ..
    for (long long idx = tid; idx < mw + nprev; idx += nt) {
      if (idx < mw) {
        const int i = k + 1 + (int)(idx / w), j = k + 1 + (int)(idx % w);
        const long long ri = perm[i];
        const double l = A[ri * n + k] / d;
        A[ri * n + j] = fma(-l, A[pr * n + j], A[ri * n + j]);
      } else {
        const long long ri = perm[k + (int)(idx - mw)];
        A[ri * n + k - 1] = A[ri * n + k - 1] / dprev;
      }
    }
    dprev = d;
    __syncthreads();
  }
  for (int i = k1 + tid; i < n; i += nt) {  // the panel's last column, logical rows k1 ..
    const long long ri = perm[i];
    A[ri * n + k1 - 1] = A[ri * n + k1 - 1] / dprev;
  }
}

// the panel's rows right of the panel: column j (one thread) takes the
// panel's elimination steps in order
__global__ void k_lu_urows(double* A, int n, int k0, int k1, const int* __restrict__ perm) {
  const int j = k1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int k = k0; k < k1; ++k) {
    const double ukj = A[(long long)perm[k] * n + j];
    for (int i = k + 1; i < k1; ++i) {
      const long long ri = perm[i];
      A[ri * n + j] = fma(-A[ri * n + k], ukj, A[ri * n + j]);
    }
  }
}

// the trailing rows and columns: each element takes the panel's steps in order
__global__ void __launch_bounds__(256) k_lu_trail(double* A, int n, int k0, int k1, const int* __restrict__ perm) {
  const int j = k1 + blockIdx.x * 32 + threadIdx.x;
  const int i = k1 + blockIdx.y * 8 + threadIdx.y;
  if (i >= n || j >= n) return;
  const long long ri = perm[i];
  double a = A[ri * n + j];
  for (int k = k0; k < k1; ++k) a = fma(-A[ri * n + k], A[(long long)perm[k] * n + j], a);
  A[ri * n + j] = a;
}

__global__ void k_lu_permute(const double* __restrict__ A, int n, const int* __restrict__ perm, double* X) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const long long i = t / n, j = t % n;
  X[t] = A[(long long)perm[i] * n + j];
}

__global__ void k_iota(int* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

// The inverse with one CTA per column of X reading the factors transposed
// (LT[k][i] = LU[i][k], coalesced over the rows)
__global__ void __launch_bounds__(256) k_lu_inverse_colT(const double* __restrict__ LT, const int* __restrict__ piv,
                                                         int n, double* X) {
  extern __shared__ double S[];
  double* xv = S;
  double* out = S + n;
  const int tid = threadIdx.x, nt = blockDim.x, j = blockIdx.x;
  for (int i = tid; i < n; i += nt) xv[i] = (i == j) ? 1.0 : 0.0;
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < n; ++k) {
      const int p = piv[k];
      if (p != k) { const double t = xv[k]; xv[k] = xv[p]; xv[p] = t; }
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double bk = xv[k];
    const double* col = LT + (long long)k * n;
    for (int i = k + 1 + tid; i < n; i += nt) xv[i] = fma(-col[i], bk, xv[i]);
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const double* col = LT + (long long)k * n;
    const double bk = xv[k] / col[k];
    if (tid == 0) out[k] = bk;
    for (int i = tid; i < k; i += nt) xv[i] = fma(-col[i], bk, xv[i]);
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) X[(long long)i * n + j] = out[i];
}



// The factorisation on a shared-memory copy of A (n x n doubles fit in one
// CTA), two block barriers per column: warp 0 finds the pivot and
// interchanges logical rows through a permutation; every thread then updates
// the trailing submatrix, forming the multiplier it needs as the quotient the
// column will hold, and scales the previous column (which no later step reads
// before that).
__global__ void __launch_bounds__(1024) k_lu_factor_smem2(double* A, int n, int* piv) {
  extern __shared__ double S[];
  int* perm = reinterpret_cast<int*>(S + (size_t)n * n);
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
  for (int idx = tid; idx < n * n; idx += nt) S[idx] = A[idx];
  for (int i = tid; i < n; i += nt) perm[i] = i;
  __syncthreads();
  double dprev = 1.0;
  for (int k = 0; k < n; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int besti = n;
      for (int i = k + lane; i < n; i += 32) {
        const double v = fabs(S[perm[i] * n + k]);
        if (v > best || (v == best && i < besti)) { best = v; besti = i; }
      }
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
        if (ov > best || (ov == best && oi < besti)) { best = ov; besti = oi; }
      }
      if (lane == 0) {
        piv[k] = besti;
        const int t = perm[k];
        perm[k] = perm[besti];
        perm[besti] = t;
      }
    }
    __syncthreads();
    const int pr = perm[k];
    const double d = S[pr * n + k];
    const int m = n - k - 1;
    const int mm = m * m, nprev = k > 0 ? n - k : 0;  // previous column: logical rows k .. n-1
    for (int idx = tid; idx < mm + nprev; idx += nt) {
      if (idx < mm) {
        const int i = k + 1 + idx / m, j = k + 1 + idx % m;
        const int ri = perm[i];
        const double l = S[ri * n + k] / d;
        S[ri * n + j] = fma(-l, S[pr * n + j], S[ri * n + j]);
      } else {
        const int ri = perm[k + (idx - mm)];
        S[ri * n + k - 1] = S[ri * n + k - 1] / dprev;
      }
    }
    dprev = d;
    __syncthreads();
  }
  for (int idx = tid; idx < n * n; idx += nt) A[idx] = S[perm[idx / n] * n + idx % n];
}

// The inverse with the factors in shared memory and one CTA per column of X:
// the threads share the rows, a block barrier per elimination column.
__global__ void __launch_bounds__(256) k_lu_inverse_col(const double* __restrict__ LU, const int* __restrict__ piv,
                                                        int n, double* X) {
  extern __shared__ double S[];
  double* L = S;              // n x n
  double* xv = S + n * n;     // the column, forward
  double* out = xv + n;       // the column, backward
  const int tid = threadIdx.x, nt = blockDim.x, j = blockIdx.x;
  for (int idx = tid; idx < n * n; idx += nt) L[idx] = LU[idx];
  for (int i = tid; i < n; i += nt) xv[i] = (i == j) ? 1.0 : 0.0;
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < n; ++k) {
      const int p = piv[k];
      if (p != k) { const double t = xv[k]; xv[k] = xv[p]; xv[p] = t; }
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double bk = xv[k];
    for (int i = k + 1 + tid; i < n; i += nt) xv[i] = fma(-L[i * n + k], bk, xv[i]);
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const double bk = xv[k] / L[k * n + k];
    if (tid == 0) out[k] = bk;
    for (int i = tid; i < k; i += nt) xv[i] = fma(-L[i * n + k], bk, xv[i]);
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) X[(long long)i * n + j] = out[i];
}



__global__ void k_transpose(const double* __restrict__ X, int n, double* __restrict__ XT) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const long long i = t / n, j = t % n;
  XT[j * n + i] = X[i * n + j];
}

// row i of A^-1 r: sum_j (A^-1)^T[j][i] rs[j] in ascending j, sixteen
// coefficients loaded before their multiply-adds (one memory wait per
// sixteen terms instead of one per term)
__device__ __forceinline__ double coarse_row(const double* __restrict__ AinvT, int n, int i, const double* rs) {
  double acc = 0.0;
  int j = 0;
  for (; j + 16 <= n; j += 16) {
    double a[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = __ldg(AinvT + (long long)(j + q) * n + i);
#pragma unroll
    for (int q = 0; q < 16; ++q) acc = fma(a[q], rs[j + q], acc);
  }
  for (; j < n; ++j) acc = fma(__ldg(AinvT + (long long)j * n + i), rs[j], acc);
  return acc;
}

// <lu> coarse-grid iterator: r := A^-1 r, x := x + damp r (one block, n <= 1024)
__global__ void __launch_bounds__(1024)
k_coarse_solve(const double* __restrict__ AinvT, int n, double damp, double* x, double* r, long long vs = 0) {
  __shared__ double rs[1024];
  const long long bq = blockIdx.x;  // one CTA per problem of a batched base level
  AinvT += bq * n * n;
  x += bq * vs;
  r += bq * vs;
  const int i = threadIdx.x;
  if (i < n) rs[i] = r[i];
  __syncthreads();
  if (i >= n) return;
  const double acc = coarse_row(AinvT, n, i, rs);
  r[i] = acc;
  x[i] = fma(damp, acc, x[i]);
}

// the same for n > 1024 unknowns (block bases of the vector form): one CTA,
// rows strided over its threads, the residual staged in shared memory
__global__ void __launch_bounds__(1024)
k_coarse_solve_big(const double* __restrict__ AinvT, int n, double damp, double* x, double* r) {
  extern __shared__ double rsb[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) rsb[i] = r[i];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double acc = coarse_row(AinvT, n, i, rsb);
    r[i] = acc;
    x[i] = fma(damp, acc, x[i]);
  }
}

// ------------------------------------------------------------ vector ops
__global__ void k_fill(double* x, long long n, double v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

__global__ void k_copy(const double* __restrict__ x, double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i];
}

// axpy!: y := y + alpha x (alpha from a device slot when aslot >= 0)
__global__ void k_axpy(double alpha, const double* __restrict__ sc, int aslot, const double* __restrict__ x,
                       double* y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = aslot >= 0 ? sc[aslot] : alpha;
  y[i] = fma(a, x[i], y[i]);
}

// DR4096 dot product (x, y)
__global__ void __launch_bounds__(kBlock)
k_dot(const double* __restrict__ x, const double* __restrict__ y, long long n, Reduce R, long long vs = 0) {
  __shared__ double smem[8];
  const long long bq = blockIdx.y;  // problem of a batched vector (stride vs)
  x += bq * vs;
  y += bq * vs;
  R = batch_reduce(R, (unsigned)bq);
  const long long base = (long long)blockIdx.x * kChunk + 2 * threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int m = 0; m < kPairsPerThread; ++m) {
    const long long i0 = base + 512LL * m;
    if (i0 < n) acc = fma(x[i0], y[i0], acc);
    if (i0 + 1 < n) acc = fma(x[i0 + 1], y[i0 + 1], acc);
  }
  dr_finish(acc, R, smem);
}

// CG update (krylow.lisp:117-121): x += lam p; r -= lam a; fused (r,r);
// then w := r and (optionally) w2 := r, q := 0 for the preconditioner call
__global__ void __launch_bounds__(kBlock)
k_cg_update(const double* __restrict__ sc, double* __restrict__ x, const double* __restrict__ p,
            double* __restrict__ r, const double* __restrict__ a, double* __restrict__ w,
            double* __restrict__ w2, double* __restrict__ q, long long n, Reduce R, long long vs = 0,
            const double* __restrict__ frozen = nullptr) {
  __shared__ double smem[8];
  const long long bq = blockIdx.y;  // problem of a batched vector (stride vs); frozen: it has converged
  sc += bq * S_COUNT;
  x += bq * vs;
  p += bq * vs;
  r += bq * vs;
  a += bq * vs;
  if (w) w += bq * vs;
  if (w2) w2 += bq * vs;
  if (q) q += bq * vs;
  R = batch_reduce(R, (unsigned)bq);
  const bool fz = frozen && frozen[bq] != 0.0;
  const double lam = sc[S_LAM], nlam = sc[S_NEGLAM];
  const long long base = (long long)blockIdx.x * kChunk + 2 * threadIdx.x;
  double acc = 0.0;
#pragma unroll 2
  for (int m = 0; m < kPairsPerThread; ++m) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long i = base + 512LL * m + u;
      if (i < n) {
        const double rn = fz ? r[i] : fma(nlam, a[i], r[i]);
        if (!fz) {
          x[i] = fma(lam, p[i], x[i]);
          r[i] = rn;
        }
        acc = fma(rn, rn, acc);
        if (w) w[i] = rn;
        if (w2) w2[i] = rn;
        if (q) q[i] = 0.0;
      }
    }
  }
  dr_finish(acc, R, smem);
}

// p := (new_alpha/alpha) p (scal!), then p := p + q (m+!)
__global__ void k_p_update(const double* __restrict__ sc, double* __restrict__ p, const double* __restrict__ q,
                           long long n, long long vs = 0, const double* __restrict__ frozen = nullptr) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long bq = blockIdx.y;  // problem of a batched vector; frozen problems keep p
  if (frozen && frozen[bq] != 0.0) return;
  sc += bq * S_COUNT;
  p += bq * vs;
  q += bq * vs;
  const double t = sc[S_RATIO] * p[i];
  p[i] = t + q[i];
}

// -------------------------------------------------------------- assembly
// Gauss-point samples of a cell-wise coefficient for a coarse level:
// kq[c * nq + q] = kcell[top cell containing the q-th Gauss point of c]
template <int D>
__global__ void k_sample_kq(long long ncells_l, long long n_l, long long n_top, double ratio, int np,
                            const double* __restrict__ xi, const double* __restrict__ kcell,
                            double* __restrict__ kq) {
  int nq = 1;
  for (int k = 0; k < D; ++k) nq *= np;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncells_l * nq) return;
  const long long c = t / nq;
  const int q = (int)(t % nq);
  const long long cc[3] = {c % n_l, D > 1 ? (c / n_l) % n_l : 0, D > 2 ? c / (n_l * n_l) : 0};
  const int qi[3] = {q % np, (q / np) % np, q / (np * np)};
  long long f[3] = {0, 0, 0};
  for (int k = 0; k < D; ++k) f[k] = (long long)floor(((double)cc[k] + xi[qi[k]]) * ratio);
  kq[t] = kcell[f[0] + n_top * (f[1] + n_top * f[2])];
}

// Stiffness entries by gather: for node i and slot s with neighbour j, the
// sum over the cells containing both nodes, in increasing cell index, of the
// local matrix entry (assemble-interior + global-local-matrix-operation,
// fedisc.lisp:73-206, sparseif.lisp:308-385).  Dirichlet rows become identity
// rows and Dirichlet columns are dropped (S A S + P).  On the top level the
// right-hand side is gathered the same way.
template <int D, int P>
__global__ void __launch_bounds__(kBlock)
k_assemble(AsmArgs g, const __grid_constant__ Q2Layout lay) {
  constexpr int NS = St<D, P>::NS;
  constexpr int C = St<D, P>::CENTER;
  constexpr int W = 2 * P + 1;
  constexpr int P1 = P + 1;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  long long ci[3];
  node_coords(i, g.M, D, ci);
  // the storage position of slot s of this node (-1: not stored, a structural zero)
  auto pos = [&](int s) -> long long {
    if (P != 2) return (long long)s * g.Np + i;
    const int r = q2_pattern<D>(s);
    for (int k = 0; k < D; ++k)
      if (((r >> k) & 1) && (ci[k] & 1)) return -1;
    return (long long)s * g.Np + q2c_pos<D>(lay, ci, g.M, r);
  };
  if (node_dirichlet(ci, g.M, D, g.dmask)) {
    for (int s = 0; s < NS; ++s) {
      const long long p = pos(s);
      if (p >= 0) g.A[p] = (s == C) ? 1.0 : 0.0;
    }
    if (g.rhs) g.rhs[i] = 0.0;
    return;
  }
  const int nl = g.nl, nq = g.nq;
  for (int s = 0; s < NS; ++s) {
    if (pos(s) < 0) continue;
    long long o[3] = {s % W - P, D > 1 ? (s / W) % W - P : 0, D > 2 ? (s / (W * W)) % W - P : 0};
    long long cj[3], lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool ok = true;
    for (int k = 0; k < 3; ++k) cj[k] = ci[k] + o[k];
    for (int k = 0; k < D; ++k) {
      if (cj[k] < 0 || cj[k] >= g.M) ok = false;
      const long long mx = ci[k] > cj[k] ? ci[k] : cj[k];
      const long long mn = ci[k] < cj[k] ? ci[k] : cj[k];
      lo[k] = mx >= P ? (mx - 1) / P : 0;
      hi[k] = mn / P;
      if (hi[k] > g.n - 1) hi[k] = g.n - 1;
    }
    double v = 0.0;
    if (ok && !node_dirichlet(cj, g.M, D, g.dmask)) {
      for (long long cz = lo[2]; cz <= hi[2]; ++cz)
        for (long long cy = lo[1]; cy <= hi[1]; ++cy)
          for (long long cx = lo[0]; cx <= hi[0]; ++cx) {
            const long long cc[3] = {cx, cy, cz};
            const long long cidx = cx + g.n * (cy + g.n * cz);
            int a = 0, b = 0, mul = 1;
            for (int k = 0; k < D; ++k) {
              a += (int)(ci[k] - P * cc[k]) * mul;
              b += (int)(cj[k] - P * cc[k]) * mul;
              mul *= P1;
            }
            double e;
            if (g.kq == nullptr) {
              const double kc = g.kcell ? g.kcell[cidx] : g.kconst;
              e = kc * g.Kbar[a * nl + b];
            } else {
              e = 0.0;
              for (int q = 0; q < nq; ++q)
                e = fma(g.kq[cidx * nq + q], g.Ctab[((long long)q * nl + a) * nl + b], e);
            }
            v = v + e;
          }
    }
    g.A[pos(s)] = v;
  }
  if (g.rhs) {
    long long lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < D; ++k) {
      lo[k] = ci[k] >= P ? (ci[k] - 1) / P : 0;
      hi[k] = ci[k] / P;
      if (hi[k] > g.n - 1) hi[k] = g.n - 1;
    }
    double acc = 0.0;
    for (long long cz = lo[2]; cz <= hi[2]; ++cz)
      for (long long cy = lo[1]; cy <= hi[1]; ++cy)
        for (long long cx = lo[0]; cx <= hi[0]; ++cx) {
          const long long cc[3] = {cx, cy, cz};
          const long long cidx = cx + g.n * (cy + g.n * cz);
          int a = 0, mul = 1;
          for (int k = 0; k < D; ++k) { a += (int)(ci[k] - P * cc[k]) * mul; mul *= P1; }
          double bl = 0.0;
          for (int q = 0; q < nq; ++q) {
            const double f = g.fip ? g.fip[cidx * nq + q] : g.fconst;
            bl = fma(f, g.Phi[q * nl + a], bl);
          }
          acc = acc + bl;
        }
    g.rhs[i] = acc;
  }
}

// k_assemble for 3D Q1 with the cell loops unrolled at compile time.  Node i
// is corner a = (1-bx) + 2 (1-by) + 4 (1-bz) of its adjacent cell ci - 1 + b
// (b = bx + 2 by + 4 bz), and neighbour j = i + o is corner a + ox + 2 oy +
// 4 oz of that cell when every 1 - b_k + o_k is 0 or 1.  The cells are walked
// in increasing b -- increasing cell index, the order k_assemble sums in --
// each adding its contribution to the 8 slots it touches, and every entry is
// formed with the same operations (e = k Kbar[a][b'], or e = sum_q fma(kq,
// Ctab, e); v = v + e), so the two kernels agree bit for bit.  The element
// tables travel as a kernel parameter (constant bank): operands of the FMAs
// without loads.  KQ: a coarse level's coefficient samples at the 8 Gauss
// points of each cell.
struct Q1Tab {
  double K[64];   // Kbar[a][b]
  double C[512];  // Ctab[q][a][b]
};

template <bool KQ>
__global__ void __launch_bounds__(kBlock)
k_assemble_q1_3d(AsmArgs g, const __grid_constant__ Q1Tab tab) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int M = (int)g.M, n = (int)g.n;
  const int ix = (int)(i % M), iy = (int)((i / M) % M), iz = (int)(i / ((long long)M * M));
  const long long ci[3] = {ix, iy, iz};
  if (node_dirichlet(ci, g.M, 3, g.dmask)) {
    if (g.A) {
#pragma unroll
      for (int s = 0; s < 27; ++s) g.A[(long long)s * g.Np + i] = (s == 13) ? 1.0 : 0.0;
    }
    if (g.rhs) g.rhs[i] = 0.0;
    return;
  }
  double v[27];
#pragma unroll
  for (int s = 0; s < 27; ++s) v[s] = 0.0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    if (!g.A) break;  // the right-hand side alone
    const int cx = ix - 1 + (b & 1), cy = iy - 1 + ((b >> 1) & 1), cz = iz - 1 + (b >> 2);
    if (cx < 0 || cx >= n || cy < 0 || cy >= n || cz < 0 || cz >= n) continue;
    const long long cidx = cx + (long long)n * (cy + (long long)n * cz);
    const int ax = 1 - (b & 1), ay = 1 - ((b >> 1) & 1), az = 1 - (b >> 2);
    const int a = ax + 2 * ay + 4 * az;
    double kq[KQ ? 8 : 1];
    if (KQ) {
#pragma unroll
      for (int q = 0; q < 8; ++q) kq[q] = __ldg(g.kq + cidx * 8 + q);
    } else {
      kq[0] = g.kcell ? __ldg(g.kcell + cidx) : g.kconst;
    }
#pragma unroll
    for (int bb = 0; bb < 8; ++bb) {  // neighbour corner: slot o = corner bb - corner a
      const int ox = (bb & 1) - ax, oy = ((bb >> 1) & 1) - ay, oz = (bb >> 2) - az;
      const int s = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
      double e;
      if (KQ) {
        e = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) e = fma(kq[q], tab.C[(q * 8 + a) * 8 + bb], e);
      } else {
        e = kq[0] * tab.K[a * 8 + bb];
      }
      v[s] = v[s] + e;
    }
  }
  if (g.A) {
#pragma unroll
    for (int s = 0; s < 27; ++s) {
      const int ox = s % 3 - 1, oy = (s / 3) % 3 - 1, oz = s / 9 - 1;
      const long long cj[3] = {ix + ox, iy + oy, iz + oz};
      const bool ok = cj[0] >= 0 && cj[0] < g.M && cj[1] >= 0 && cj[1] < g.M && cj[2] >= 0 && cj[2] < g.M &&
                      !node_dirichlet(cj, g.M, 3, g.dmask);
      g.A[(long long)s * g.Np + i] = ok ? v[s] : 0.0;
    }
  }
  if (g.rhs) {
    double acc = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int cx = ix - 1 + (b & 1), cy = iy - 1 + ((b >> 1) & 1), cz = iz - 1 + (b >> 2);
      if (cx < 0 || cx >= n || cy < 0 || cy >= n || cz < 0 || cz >= n) continue;
      const long long cidx = cx + (long long)n * (cy + (long long)n * cz);
      const int a = (1 - (b & 1)) + 2 * (1 - ((b >> 1) & 1)) + 4 * (1 - (b >> 2));
      double bl = 0.0;
      for (int q = 0; q < g.nq; ++q) {
        const double f = g.fip ? g.fip[cidx * g.nq + q] : g.fconst;
        bl = fma(f, g.Phi[q * g.nl + a], bl);
      }
      acc = acc + bl;
    }
    g.rhs[i] = acc;
  }
}

// ====================================================== vector form (nc = 3)
// Elasticity with 3 x 3 nodal blocks: vectors [node][3], level matrices
// [slot][k][l][Np] (block row component k, column component l).  Every
// kernel follows the scalar one with the component loops innermost, in the
// order the oracle uses.

// t := B^-1 r for one diagonal block: LU with partial pivoting (the first
// largest |entry| of the column, LAPACK dgetrf semantics) and substitution
// -- the gesv! of <jacobi> on a 3 x 3 block (linit.lisp:234)
template <typename T>
__device__ __forceinline__ void block_solve3(const T* B, const T* r, T* t) {
  T M[3][3], b[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    b[k] = r[k];
#pragma unroll
    for (int m = 0; m < 3; ++m) M[k][m] = B[k * 3 + m];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    int pr = c;
    T mx = fabs(M[c][c]);
#pragma unroll
    for (int rr = c + 1; rr < 3; ++rr)
      if (fabs(M[rr][c]) > mx) { mx = fabs(M[rr][c]); pr = rr; }
    if (pr != c) {
#pragma unroll
      for (int rr = c + 1; rr < 3; ++rr)
        if (rr == pr) {
#pragma unroll
          for (int m = 0; m < 3; ++m) { const T tt = M[c][m]; M[c][m] = M[rr][m]; M[rr][m] = tt; }
          const T tb = b[c]; b[c] = b[rr]; b[rr] = tb;
        }
    }
#pragma unroll
    for (int rr = c + 1; rr < 3; ++rr) {
      const T f = M[rr][c] / M[c][c];
#pragma unroll
      for (int m = c + 1; m < 3; ++m) M[rr][m] = fma(-f, M[c][m], M[rr][m]);
      b[rr] = fma(-f, b[c], b[rr]);
    }
  }
#pragma unroll
  for (int c = 2; c >= 0; --c) {
    T sacc = b[c];
#pragma unroll
    for (int m = c + 1; m < 3; ++m) sacc = fma(-M[c][m], t[m], sacc);
    t[c] = sacc / M[c][c];
  }
}

// the three block-row sums of node i: slots ascending, columns ascending
template <int P, typename T>
__device__ __forceinline__ void row_sums3(const T* __restrict__ A, long long N, long long Np, long long M,
                                          const T* __restrict__ x, long long i, T* s, T* dblk) {
  constexpr int NS = St<3, P>::NS;
  constexpr int C = St<3, P>::CENTER;
  s[0] = s[1] = s[2] = T(0);
  auto blk = [&](int sl, long long o, long long p, bool) {
    const long long j = clampi(i + o, N);
    const T xj[3] = {__ldg(x + 3 * j), __ldg(x + 3 * j + 1), __ldg(x + 3 * j + 2)};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const T a = __ldg(A + ((long long)(sl * 3 + k) * 3 + m) * Np + p);
        if (dblk && sl == C) dblk[k * 3 + m] = a;
        s[k] = fma(a, xj[m], s[k]);
      }
  };
  if constexpr (P == 2) {  // sliced storage
    long long c[3];
    node_coords32(i, M, 3, c);
    Q2Base<3> qb;
    q2_base<3, false>(Q2Layout{}, c, M, qb);
    q2_visit<3, false>(qb, M, blk);
  } else {
#pragma unroll 3
    for (int sl = 0; sl < NS; ++sl) blk(sl, slot_off<3, P>(sl, M), i, true);
  }
}

// y = A x or r = b - A x (b may alias r)
template <int P, bool RES, typename T = double>
__global__ void __launch_bounds__(kBlock)
k_spmv3(const T* __restrict__ A, long long N, long long Np, long long M, const T* __restrict__ x,
        const T* b, T* y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T s[3];
  row_sums3<P, T>(A, N, Np, M, x, i, s, (T*)nullptr);
#pragma unroll
  for (int k = 0; k < 3; ++k) y[3 * i + k] = RES ? b[3 * i + k] - s[k] : s[k];
}

// <jacobi> on 3 x 3 blocks with an up-to-date residual: t = B^-1 r_i, x_i += w t, r_i := t
__global__ void __launch_bounds__(kBlock)
k_jacobi3(const double* __restrict__ A, long long N, long long Np, int center, double damp,
          const double* __restrict__ omega, double* x, double* r, int write_r) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double B[9], t[3];
#pragma unroll
  for (int e = 0; e < 9; ++e) B[e] = A[((long long)center * 9 + e) * Np + i];
  const double rr[3] = {r[3 * i], r[3 * i + 1], r[3 * i + 2]};
  block_solve3<double>(B, rr, t);
  const double w = omega ? omega[i] : damp;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (write_r) r[3 * i + k] = t[k];
    x[3 * i + k] = fma(w, t[k], x[3 * i + k]);
  }
}

// compute-residual fused with the following block <jacobi> step:
// r_i = b_i - (A x)_i, t = B^-1 r_i, xout_i = x_i + w t, r_i := t
template <int P, typename T = double>
__global__ void __launch_bounds__(kBlock)
k_jacobi_res3(const T* __restrict__ A, long long N, long long Np, long long M, double damp,
              const double* __restrict__ omega, const T* __restrict__ x, const T* b,
              T* __restrict__ xout, T* r, int write_r) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T s[3], B[9], t[3];
  row_sums3<P, T>(A, N, Np, M, x, i, s, B);
  const T rr[3] = {b[3 * i] - s[0], b[3 * i + 1] - s[1], b[3 * i + 2] - s[2]};
  block_solve3<T>(B, rr, t);
  const T w = omega ? (T)omega[i] : (T)damp;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (write_r) r[3 * i + k] = t[k];
    xout[3 * i + k] = fma(w, t[k], x[3 * i + k]);
  }
}

// rc := I^T rf per component (constrained), rhs_c := rc, sol_c := 0
template <int P, typename T = double>
__global__ void __launch_bounds__(kBlock)
k_restrict3(int MC, int MF, int dmask, const T* __restrict__ rf, T* __restrict__ rc,
            T* __restrict__ rhsc, T* __restrict__ solc) {
  const int cJ[3] = {(int)(blockIdx.x * 32 + threadIdx.x), (int)(blockIdx.y * 8 + threadIdx.y), (int)blockIdx.z};
  if (cJ[0] >= MC || cJ[1] >= MC) return;
  const long long J = cJ[0] + (long long)MC * (cJ[1] + (long long)MC * cJ[2]);
  bool dj = false;
  for (int k = 0; k < 3; ++k) dj = dj || face_dir(cJ[k], MC, k, dmask);
  T acc[3] = {T(0), T(0), T(0)};
  if (!dj) {
    long long off[3][5] = {{0}, {0}, {0}};
    double w[3][5] = {{1.0}, {1.0}, {1.0}};
    int cnt[3];
    for (int k = 0; k < 3; ++k) cnt[k] = restrict_1d<P>(cJ[k], off[k], w[k]);
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int xx = 0; xx < cnt[0]; ++xx) {
          const int fi[3] = {2 * cJ[0] + (int)off[0][xx], 2 * cJ[1] + (int)off[1][y], 2 * cJ[2] + (int)off[2][z]};
          bool skip = false;
          for (int k = 0; k < 3; ++k) skip = skip || fi[k] < 0 || fi[k] >= MF || face_dir(fi[k], MF, k, dmask);
          if (skip) continue;
          const T ww = (T)(w[0][xx] * w[1][y] * w[2][z]);
          const long long f = fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2]);
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[c] = fma(ww, rf[3 * f + c], acc[c]);
        }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    rc[3 * J + c] = acc[c];
    rhsc[3 * J + c] = acc[c];
    solc[3 * J + c] = T(0);
  }
}

// xf := xf + I xc per component (constrained)
template <int P, typename T = double>
__global__ void __launch_bounds__(kBlock)
k_prolong3(int MF, int MC, int dmask, const T* __restrict__ xc, T* __restrict__ xf) {
  const int fi[3] = {(int)(blockIdx.x * 32 + threadIdx.x), (int)(blockIdx.y * 8 + threadIdx.y), (int)blockIdx.z};
  if (fi[0] >= MF || fi[1] >= MF) return;
  for (int k = 0; k < 3; ++k)
    if (face_dir(fi[k], MF, k, dmask)) return;
  const long long i = fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2]);
  long long J[3][3] = {{0}, {0}, {0}};
  double w[3][3] = {{1.0}, {1.0}, {1.0}};
  int cnt[3];
  for (int k = 0; k < 3; ++k) cnt[k] = prolong_1d<P>(fi[k], J[k], w[k]);
  T acc[3] = {T(0), T(0), T(0)};
  for (int z = 0; z < cnt[2]; ++z)
    for (int y = 0; y < cnt[1]; ++y)
      for (int xx = 0; xx < cnt[0]; ++xx) {
        const int cj[3] = {(int)J[0][xx], (int)J[1][y], (int)J[2][z]};
        bool dj = false;
        for (int k = 0; k < 3; ++k) dj = dj || face_dir(cj[k], MC, k, dmask);
        if (dj) continue;
        const T ww = (T)(w[0][xx] * w[1][y] * w[2][z]);
        const long long j = cj[0] + (long long)MC * (cj[1] + (long long)MC * cj[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] = fma(ww, xc[3 * j + c], acc[c]);
      }
#pragma unroll
  for (int c = 0; c < 3; ++c) xf[3 * i + c] = xf[3 * i + c] + acc[c];
}

// Elasticity stiffness by gather (the vector form of k_assemble): for node i,
// slot s and block entry (k, l), the sum over the cells containing both nodes,
// in increasing cell index, of E_c Ebar[a][b][k][l] (top level, E per cell)
// or sum_q fma(E(x_q), Etab[q][a][b][k][l], .) (coarse levels, E sampled at
// the cell's Gauss points); Dirichlet nodes get identity blocks, Dirichlet
// columns are dropped.  a.Kbar = Ebar, a.Ctab = Etab, a.fvec the force.
template <int P>
__global__ void __launch_bounds__(kBlock)
k_assemble3(AsmArgs g) {
  constexpr int NS = St<3, P>::NS;
  constexpr int C = St<3, P>::CENTER;
  constexpr int W = 2 * P + 1;
  constexpr int P1 = P + 1;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  long long ci[3];
  node_coords(i, g.M, 3, ci);
  const int nl = g.nl, nq = g.nq;
  Q2Rows<3> q2;
  if (P == 2) q2_rows<3>(ci, g.M, q2);
  auto pos = [&](int s) -> long long {  // the node's entry in slot s (-1: a structural zero, not stored)
    if (P != 2) return i;
    const int r = q2_pattern<3>(s);
    return ((q2.valid >> r) & 1) ? q2.idx[r] : -1;
  };
  if (node_dirichlet(ci, g.M, 3, g.dmask)) {
    for (int s = 0; s < NS; ++s) {
      const long long p = pos(s);
      if (p < 0) continue;
      for (int e = 0; e < 9; ++e) g.A[((long long)s * 9 + e) * g.Np + p] = (s == C && e % 4 == 0) ? 1.0 : 0.0;
    }
    if (g.rhs)
      for (int k = 0; k < 3; ++k) g.rhs[3 * i + k] = 0.0;
    return;
  }
  for (int s = 0; s < NS; ++s) {
    const long long ps = pos(s);
    if (ps < 0) continue;
    const long long o[3] = {s % W - P, (s / W) % W - P, s / (W * W) - P};
    long long cj[3], lo[3], hi[3];
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
      cj[k] = ci[k] + o[k];
      if (cj[k] < 0 || cj[k] >= g.M) ok = false;
      const long long mx = ci[k] > cj[k] ? ci[k] : cj[k];
      const long long mn = ci[k] < cj[k] ? ci[k] : cj[k];
      lo[k] = mx >= P ? (mx - 1) / P : 0;
      hi[k] = mn / P;
      if (hi[k] > g.n - 1) hi[k] = g.n - 1;
    }
    double v[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) v[e] = 0.0;
    if (ok && !node_dirichlet(cj, g.M, 3, g.dmask)) {
      for (long long cz = lo[2]; cz <= hi[2]; ++cz)
        for (long long cy = lo[1]; cy <= hi[1]; ++cy)
          for (long long cx = lo[0]; cx <= hi[0]; ++cx) {
            const long long cc[3] = {cx, cy, cz};
            const long long cidx = cx + g.n * (cy + g.n * cz);
            int a = 0, b = 0, mul = 1;
            for (int k = 0; k < 3; ++k) {
              a += (int)(ci[k] - P * cc[k]) * mul;
              b += (int)(cj[k] - P * cc[k]) * mul;
              mul *= P1;
            }
            const long long ab = ((long long)a * nl + b) * 9;
            if (g.kq == nullptr) {
              const double kc = g.kcell ? g.kcell[cidx] : g.kconst;
#pragma unroll
              for (int e = 0; e < 9; ++e) v[e] = v[e] + kc * __ldg(g.Kbar + ab + e);
            } else {
#pragma unroll
              for (int e = 0; e < 9; ++e) {
                double ee = 0.0;
                for (int q = 0; q < nq; ++q)
                  ee = fma(__ldg(g.kq + cidx * nq + q), __ldg(g.Ctab + (long long)q * nl * nl * 9 + ab + e), ee);
                v[e] = v[e] + ee;
              }
            }
          }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) g.A[((long long)s * 9 + e) * g.Np + ps] = v[e];
  }
  if (g.rhs) {
    long long lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
      lo[k] = ci[k] >= P ? (ci[k] - 1) / P : 0;
      hi[k] = ci[k] / P;
      if (hi[k] > g.n - 1) hi[k] = g.n - 1;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long cz = lo[2]; cz <= hi[2]; ++cz)
      for (long long cy = lo[1]; cy <= hi[1]; ++cy)
        for (long long cx = lo[0]; cx <= hi[0]; ++cx) {
          const long long cc[3] = {cx, cy, cz};
          int a = 0, mul = 1;
          for (int k = 0; k < 3; ++k) { a += (int)(ci[k] - P * cc[k]) * mul; mul *= P1; }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            double bl = 0.0;
            const double f = g.fvec_on ? g.fvec[k] : g.fconst;
            for (int q = 0; q < nq; ++q) bl = fma(f, g.Phi[q * nl + a], bl);
            acc[k] = acc[k] + bl;
          }
        }
    for (int k = 0; k < 3; ++k) g.rhs[3 * i + k] = acc[k];
  }
}

// dense (3N x 3N) copy of a small block level matrix, for the coarse LU
template <int P>
__global__ void k_densify3(const double* __restrict__ A, long long N, long long Np, long long M,
                           double* __restrict__ Dm) {
  constexpr int NS = St<3, P>::NS;
  constexpr int W = 2 * P + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * NS) return;
  const long long i = t / NS;
  const int s = (int)(t % NS);
  long long ci[3];
  node_coords(i, M, 3, ci);
  const long long o[3] = {s % W - P, (s / W) % W - P, s / (W * W) - P};
  long long cj[3];
  for (int k = 0; k < 3; ++k) {
    cj[k] = ci[k] + o[k];
    if (cj[k] < 0 || cj[k] >= M) return;
  }
  const long long j = cj[0] + M * (cj[1] + M * cj[2]);
  const long long n = 3 * N;
  long long p = i;
  if constexpr (P == 2) {  // sliced storage
    Q2Rows<3> q;
    q2_rows<3>(ci, M, q);
    const int r = q2_pattern<3>(s);
    if (!((q.valid >> r) & 1)) return;
    p = q.idx[r];
  }
  for (int k = 0; k < 3; ++k)
    for (int m = 0; m < 3; ++m) Dm[(3 * i + k) * n + 3 * j + m] = A[((long long)s * 9 + k * 3 + m) * Np + p];
}

// The full slot layout of a level (structural zeros included) in FP32 -- the
// layout the stored-level kernels of the mixed cycle read -- from a Q2
// level's sliced storage; one thread per (slot, node)
template <int D>
__global__ void k_expand_q2_f32(const double* __restrict__ A, long long N, long long Np, long long M, int nslots,
                                float* __restrict__ out, const __grid_constant__ Q2Layout lay) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nslots * N) return;
  const int s = (int)(t / N);
  const long long i = t - (long long)s * N;
  long long c[3];
  node_coords(i, M, D, c);
  const int r = q2_pattern<D>(s);
  bool ok = true;
  for (int k = 0; k < D; ++k)
    if (((r >> k) & 1) && (c[k] & 1)) ok = false;
  out[(long long)s * Np + i] = ok ? (float)A[(long long)s * Np + q2c_pos<D>(lay, c, M, r)] : 0.f;
}

// Galerkin coarse operator A_C = I^T A_F I of a structured level -- scalar
// Q1/Q2 and 3 x 3 node blocks -- with the constrained interpolation (fine
// Dirichlet rows and coarse Dirichlet columns removed; identity blocks at
// coarse Dirichlet nodes).  One thread per (coarse slot S, coarse row I): it
// walks the oracle's order -- fine i over the restriction stencil of I
// (z, y, x), fine slots ascending, the coarse J = I + off_S looked up in j's
// interpolation stencil -- and keeps the terms that land on S, so each entry
// sums the oracle's terms in the oracle's order:
// acc[k][m] = fma(w_iI * a_ij[k][m], w_jJ, acc[k][m]).  Fine entries a level
// does not store (Q2: an odd-coordinate node's +-2 slots) are structural
// zeros and are skipped.
template <int D, int P>
__device__ __forceinline__ long long gal_pos(const Q2Layout& lay, const long long c[3], long long M, int s, int nc) {
  if (P == 1) return c[0] + M * (c[1] + M * c[2]);
  const int r = q2_pattern<D>(s);
  for (int k = 0; k < D; ++k)
    if (((r >> k) & 1) && (c[k] & 1)) return -1;
  if (nc == 1) return q2c_pos<D>(lay, c, M, r);  // scalar Q2: colour-major
  const long long H = (M + 1) / 2;              // node blocks: lexicographic, halved where restricted
  long long id = 0, mul = 1;
  for (int k = 0; k < D; ++k) {
    const bool rk = (r >> k) & 1;
    id += (rk ? c[k] / 2 : c[k]) * mul;
    mul *= rk ? H : M;
  }
  return id;
}

template <int D, int P, int NC>
__global__ void __launch_bounds__(kBlock)
k_galerkin(const double* __restrict__ AF, long long NpF, int MF, double* __restrict__ AC, long long NCN,
           long long NpC, int MC, int dmask, Q2Layout layF, Q2Layout layC) {
  constexpr int W = 2 * P + 1;
  constexpr int NS = D == 1 ? W : (D == 2 ? W * W : W * W * W);
  constexpr int CEN = (NS - 1) / 2;
  constexpr int NE = NC * NC;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)NS * NCN) return;
  const int S = (int)(t / NCN);
  const long long I = t - (long long)S * NCN;
  long long cI[3];
  node_coords(I, MC, D, cI);
  const long long pI = gal_pos<D, P>(layC, cI, MC, S, NC);
  if (pI < 0) return;  // an entry the coarse level does not store
  double acc[NE];
#pragma unroll
  for (int e = 0; e < NE; ++e) acc[e] = 0.0;
  if (node_dirichlet(cI, MC, D, dmask)) {
#pragma unroll
    for (int e = 0; e < NE; ++e) AC[((long long)S * NE + e) * NpC + pI] = (S == CEN && e % (NC + 1) == 0) ? 1.0 : 0.0;
    return;
  }
  const int oS[3] = {S % W - P, D > 1 ? (S / W) % W - P : 0, D > 2 ? S / (W * W) - P : 0};
  long long cJ[3] = {0, 0, 0};
  bool okJ = true;
  for (int k = 0; k < D; ++k) {
    cJ[k] = cI[k] + oS[k];
    okJ = okJ && cJ[k] >= 0 && cJ[k] < MC;
  }
  if (okJ && !node_dirichlet(cJ, MC, D, dmask)) {
    long long off[3][5] = {{0}, {0}, {0}};
    double w[3][5] = {{1.0}, {1.0}, {1.0}};
    int cnt[3] = {1, 1, 1};
    for (int k = 0; k < D; ++k) cnt[k] = restrict_1d<P>(cI[k], off[k], w[k]);
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y)
        for (int x = 0; x < cnt[0]; ++x) {
          const long long fi[3] = {2 * cI[0] + off[0][x], D > 1 ? 2 * cI[1] + off[1][y] : 0,
                                   D > 2 ? 2 * cI[2] + off[2][z] : 0};
          bool skip = false;
          for (int k = 0; k < D; ++k) skip = skip || fi[k] < 0 || fi[k] >= MF || face_dir((int)fi[k], MF, k, dmask);
          if (skip) continue;
          double wi = w[0][x];
          if (D > 1) wi = wi * w[1][y];
          if (D > 2) wi = wi * w[2][z];
          for (int oz = (D > 2 ? -P : 0); oz <= (D > 2 ? P : 0); ++oz)
            for (int oy = (D > 1 ? -P : 0); oy <= (D > 1 ? P : 0); ++oy)
              for (int ox = -P; ox <= P; ++ox) {
                const int o[3] = {ox, oy, oz};
                long long fj[3] = {0, 0, 0};
                double wj[3] = {1.0, 1.0, 1.0};
                bool hit = true;
                for (int k = 0; k < D && hit; ++k) {
                  fj[k] = fi[k] + o[k];
                  if (fj[k] < 0 || fj[k] >= MF || face_dir((int)fj[k], MF, k, dmask)) { hit = false; break; }
                  long long Jk[3];
                  double wk[3];
                  const int nk = prolong_1d<P>(fj[k], Jk, wk);
                  bool found = false;
                  for (int q = 0; q < nk; ++q)
                    if (Jk[q] == cJ[k]) { wj[k] = wk[q]; found = true; }
                  hit = found;
                }
                if (!hit) continue;
                const int sf = (ox + P) + W * ((D > 1 ? oy : 0) + (D > 1 ? P : 0)) +
                               W * W * ((D > 2 ? oz : 0) + (D > 2 ? P : 0));
                const long long pF = gal_pos<D, P>(layF, fi, MF, sf, NC);
                if (pF < 0) continue;  // a structural zero
                double ww = wj[0];
                if (D > 1) ww = ww * wj[1];
                if (D > 2) ww = ww * wj[2];
#pragma unroll
                for (int e = 0; e < NE; ++e)
                  acc[e] = fma(wi * AF[((long long)sf * NE + e) * NpF + pF], ww, acc[e]);
              }
        }
  }
#pragma unroll
  for (int e = 0; e < NE; ++e) AC[((long long)S * NE + e) * NpC + pI] = acc[e];
}

// ---- diagonal-block operations of the recorded cycle (vector form)
// mode 0: y_i = B_i^-1 x_i; 1: y_i = w_i B_i^-1 x_i; 2: y_i += w_i B_i^-1 x_i
// (B_i the 3 x 3 diagonal block, symmetric, so the same solve serves the adjoint)
__global__ void __launch_bounds__(kBlock)
k_bdiag3(const double* __restrict__ A, long long N, long long Np, int center, int mode,
         const double* __restrict__ w, const double* __restrict__ x, double* __restrict__ y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double B[9], t[3];
#pragma unroll
  for (int e = 0; e < 9; ++e) B[e] = A[((long long)center * 9 + e) * Np + i];
  const double xx[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  block_solve3<double>(B, xx, t);
  const double wi = mode == 0 ? 1.0 : w[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = mode == 0 ? t[k] : wi * t[k];
    y[3 * i + k] = mode == 2 ? y[3 * i + k] + v : v;
  }
}

// y = x + w .* v with w per node (y may be x)
__global__ void k_xpwv3(const double* x, const double* __restrict__ w, const double* __restrict__ v, double* y,
                        long long N) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) y[3 * i + k] = x[3 * i + k] + w[i] * v[3 * i + k];
}

// acc_i += sum_k a_ik b_ik (per-node dot of two vectors)
__global__ void k_acc_prod3(double* __restrict__ acc, const double* __restrict__ a, const double* __restrict__ b,
                            long long N) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = a[3 * i] * b[3 * i];
  s = fma(a[3 * i + 1], b[3 * i + 1], s);
  s = fma(a[3 * i + 2], b[3 * i + 2], s);
  acc[i] += s;
}

// ---- FP32 forms for the mixed cycle of the vector form
// first smoothing step from a zero guess: x = w B^-1 b
template <typename T>
__global__ void __launch_bounds__(kBlock)
k_jacobi0_3(const T* __restrict__ A, long long N, long long Np, int center, float damp,
            const double* __restrict__ omega, const T* __restrict__ b, T* __restrict__ x) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T B[9], t[3];
#pragma unroll
  for (int e = 0; e < 9; ++e) B[e] = A[((long long)center * 9 + e) * Np + i];
  const T bb[3] = {b[3 * i], b[3 * i + 1], b[3 * i + 2]};
  block_solve3<T>(B, bb, t);
  const T w = omega ? (T)omega[i] : (T)damp;
#pragma unroll
  for (int k = 0; k < 3; ++k) x[3 * i + k] = w * t[k];
}

// y = f x with f from a grid scalar: mode 0: 1, mode 1: 1/sqrt(sc[slot]), mode 2: sqrt(sc[slot])
template <typename TI, typename TO>
__global__ void k_vscale(const TI* __restrict__ x, const double* __restrict__ sc, int slot, int mode,
                         TO* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f = 1.0;
  if (mode) {
    const double v = sc[slot];
    f = v > 0.0 ? (mode == 1 ? 1.0 / sqrt(v) : sqrt(v)) : 1.0;
  }
  y[i] = (TO)((double)x[i] * f);
}

// the FCG(1) coefficient beta = -(z, a) / (p, a) of the previous step (0 on a restart)
__global__ void k_fcg_beta(double* sc, int first) {
  sc[S_RATIO] = first ? 0.0 : -sc[S_TMP] / sc[S_BETA];
}

// ---------------------------------------------------------- dispatchers
#define FMG_DISPATCH(D_, P_, ...)                                             \
  do {                                                                        \
    if ((D_) == 1 && (P_) == 1) { constexpr int D = 1, P = 1; __VA_ARGS__; }  \
    else if ((D_) == 2 && (P_) == 1) { constexpr int D = 2, P = 1; __VA_ARGS__; } \
    else if ((D_) == 3 && (P_) == 1) { constexpr int D = 3, P = 1; __VA_ARGS__; } \
    else if ((D_) == 1 && (P_) == 2) { constexpr int D = 1, P = 2; __VA_ARGS__; } \
    else if ((D_) == 2 && (P_) == 2) { constexpr int D = 2, P = 2; __VA_ARGS__; } \
    else { constexpr int D = 3, P = 2; __VA_ARGS__; }                         \
  } while (0)

#define Q1_DISPATCH(D_, ...)                                              \
  do {                                                                    \
    if ((D_) == 1) { constexpr int D = 1; __VA_ARGS__; }                  \
    else if ((D_) == 2) { constexpr int D = 2; __VA_ARGS__; }             \
    else { constexpr int D = 3; __VA_ARGS__; }                            \
  } while (0)
#define Q2_DISPATCH Q1_DISPATCH

static inline unsigned grid1(long long n, int bs = kBlock) { return (unsigned)((n + bs - 1) / bs); }

// the row kernels of scalar Q2 levels over every class: blockIdx.y the class,
// blockIdx.x the blocks of its parity subgrids (the largest class's count)
template <int D>
static dim3 q2_grid(int M) {
  int ncol = 1;
  for (int k = 0; k < D; ++k) ncol *= 3;
  long long nb = 1;
  for (int col = 0; col < ncol; ++col) nb = std::max(nb, q2_class_blocks<D>(M, col));
  return dim3((unsigned)nb, (unsigned)ncol);
}

void launch_spmv(const LevelView& L, const double* x, const double* b, double* y, const double* dv,
                 const Reduce* R, cudaStream_t st) {
  if (L.csr) {  // the reduction as a separate DR4096 pass
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_csr_spmv<<<grid1(L.N), kBlock, 0, st>>>(L.N, L.a, x, b, y, b ? 1 : 0);
    if (dv) launch_dot(y, dv, L.N, *R, st);
    return;
  }
  if (L.nc == 3) {  // 3 x 3 blocks: the reduction, if any, as a separate DR4096 pass
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (L.order == 2) {
      if (b) k_spmv3<2, true><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y);
      else k_spmv3<2, false><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y);
    } else {
      if (b) k_spmv3<1, true><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y);
      else k_spmv3<1, false><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y);
    }
    if (dv) launch_dot(y, dv, 3 * L.N, *R, st);
    return;
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (L.order == 2) {  // rows by colour class and parity, the reduction as a separate DR4096 pass
    const Q2Layout lay = q2_layout(L.dim, L.M);
    Q2_DISPATCH(L.dim, {
      const dim3 g = q2_grid<D>((int)L.M);
      if (b) k_spmv_q2c<D, true><<<g, kQ2T, 0, st>>>(L.A, L.Np, (int)L.M, x, b, y, lay);
      else k_spmv_q2c<D, false><<<g, kQ2T, 0, st>>>(L.A, L.Np, (int)L.M, x, b, y, lay);
    });
    if (dv) launch_dot(y, dv, L.N, *R, st);
    return;
  }
  const dim3 g(nchunks(L.N), (unsigned)L.nb);
  Reduce r0 = R ? *R : Reduce{};
  Q1_DISPATCH(L.dim, {
    if (b && dv) k_spmv<D, 1, true, true><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y, dv, r0);
    else if (b) k_spmv<D, 1, true, false><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y, dv, r0);
    else if (dv) k_spmv<D, 1, false, true><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y, dv, r0);
    else k_spmv<D, 1, false, false><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, x, b, y, dv, r0);
  });
}

void launch_jacobi(const LevelView& L, double damp, double* x, double* r, bool write_r, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (L.csr) {
    k_jacobi<<<grid1(L.N), kBlock, 0, st>>>(L.diag, L.N, damp, L.omega, x, r, write_r ? 1 : 0);
    return;
  }
  if (L.nc == 3) {
    k_jacobi3<<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.center, damp, L.omega, x, r, write_r ? 1 : 0);
    return;
  }
  if (L.order == 2) {  // colour-major sliced storage
    const Q2Layout lay = q2_layout(L.dim, L.M);
    Q2_DISPATCH(L.dim, {
      k_jacobi_q2<D><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, damp, L.omega, x, r, write_r ? 1 : 0, lay);
    });
    return;
  }
  const double* Dg = L.A + (long long)L.center * L.Np;
  long long ns = 1;
  for (int k = 0; k < L.dim; ++k) ns *= 3;
  k_jacobi<<<dim3(grid1(L.N), (unsigned)L.nb), kBlock, 0, st>>>(Dg, L.N, damp, L.omega, x, r, write_r ? 1 : 0,
                                                                L.Np, ns * L.Np);
}

void launch_jacobi_res(const LevelView& L, double damp, const double* x, const double* b, double* xout,
                       double* r, bool write_r, const double* dv, const Reduce* R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (L.csr) {
    k_csr_jacobi_res<<<grid1(L.N), kBlock, 0, st>>>(L.N, L.a, L.diag, damp, L.omega, x, b, xout, r,
                                                      write_r ? 1 : 0);
    if (dv) launch_dot(xout, dv, L.N, *R, st);
    return;
  }
  if (L.nc == 3) {
    if (L.order == 2)
      k_jacobi_res3<2><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, damp, L.omega, x, b, xout, r,
                                                        write_r ? 1 : 0);
    else
      k_jacobi_res3<1><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, damp, L.omega, x, b, xout, r,
                                                        write_r ? 1 : 0);
    if (dv) launch_dot(xout, dv, 3 * L.N, *R, st);
    return;
  }
  if (L.order == 2) {  // rows by colour class and parity
    const Q2Layout lay = q2_layout(L.dim, L.M);
    Q2_DISPATCH(L.dim, {
      k_jacobi_res_q2c<D><<<q2_grid<D>((int)L.M), kQ2T, 0, st>>>(L.A, L.Np, (int)L.M, damp, L.omega, x, b, xout, r,
                                                                 write_r ? 1 : 0, lay);
    });
    if (dv) launch_dot(xout, dv, L.N, *R, st);
    return;
  }
  const dim3 g(nchunks(L.N), (unsigned)L.nb);
  Reduce r0 = R ? *R : Reduce{};
  Q1_DISPATCH(L.dim, {
    if (dv) k_jacobi_res<D, 1, true><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, damp, L.omega, x, b, xout, r,
                                                             write_r ? 1 : 0, dv, r0);
    else k_jacobi_res<D, 1, false><<<g, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, damp, L.omega, x, b, xout, r,
                                                         write_r ? 1 : 0, dv, r0);
  });
}

static void launch_csr_sor(const LevelView& L, double omega, const double* om, double* x, const double* b, double* r,
                           bool ssc, cudaStream_t st) {
  g_launches.fetch_add(L.ncol, std::memory_order_relaxed);
  for (int c = 0; c < L.ncol; ++c) {
    const long long cnt = L.coff[c + 1] - L.coff[c];
    if (cnt > 0)
      k_csr_sor<<<grid1(cnt), kBlock, 0, st>>>(L.crow + L.coff[c], cnt, L.a, L.diag, omega, om, x, b, r, ssc ? 1 : 0);
  }
}

void launch_sor(const LevelView& L, double omega, double* x, const double* b, double* r, cudaStream_t st) {
  if (L.csr) {
    launch_csr_sor(L, omega, L.omega, x, b, r, false, st);
    return;
  }
  const Q2Layout lay = q2_layout(L.dim, L.M);
  int Q = L.order + 1, ncol = 1;
  for (int k = 0; k < L.dim; ++k) ncol *= Q;
  g_launches.fetch_add(ncol, std::memory_order_relaxed);
  for (int col = 0; col < ncol; ++col) {
    const int cx = col % Q, cy = (col / Q) % Q, cz = col / (Q * Q);
    long long cnt = (L.M - cx + Q - 1) / Q;
    if (L.dim > 1) cnt *= (L.M - cy + Q - 1) / Q;
    if (L.dim > 2) cnt *= (L.M - cz + Q - 1) / Q;
    if (L.order == 2) {
      Q2_DISPATCH(L.dim, {
        const unsigned nb = (unsigned)q2_class_blocks<D>((int)L.M, col);
        if (nb) k_sor_q2<D><<<nb, kQ2T, 0, st>>>(L.A, L.Np, (int)L.M, col, omega, L.omega, x, b, r, lay);
      });
    } else {
      Q1_DISPATCH(L.dim, {
        k_sor_colour<D, 1><<<grid1(cnt), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, col, omega, L.omega, x, b, r);
      });
    }
  }
}

long long ssc_blocks(const LevelView& L) {
  if (L.order != 2) return 0;
  long long nv = (L.M + 1) / 2, n = 1;
  for (int k = 0; k < L.dim; ++k) n *= nv;
  return n;
}

int ssc_block_size(int dim) { return dim == 1 ? 3 : (dim == 2 ? 9 : 27); }

void launch_ssc_factor(const LevelView& L, double* F, unsigned char* P, cudaStream_t st) {
  if (L.order != 2) return;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const Q2Layout lay = q2_layout(L.dim, L.M);
  const unsigned grid = (unsigned)((ssc_blocks(L) * 32 + 127) / 128);
  Q2_DISPATCH(L.dim, { k_ssc_factor_q2<D><<<grid, 128, 0, st>>>(L.A, L.Np, L.M, L.dmask, F, P, lay); });
}

void launch_ssc(const LevelView& L, double omega, double* x, const double* b, double* r, const double* F,
                const unsigned char* P, cudaStream_t st) {
  if (L.csr) {  // an algebraic level: one-unknown blocks over its colouring
    launch_csr_sor(L, omega, nullptr, x, b, r, true, st);
    return;
  }
  const int ncol = 1 << L.dim;
  g_launches.fetch_add(ncol, std::memory_order_relaxed);
  if (L.order == 1) {  // one-node blocks: the colour sweep of the SOR with the SSC residual
    for (int col = 0; col < ncol; ++col) {
      const int cx = col & 1, cy = (col >> 1) & 1, cz = (col >> 2) & 1;
      long long cnt = (L.M - cx + 1) / 2;
      if (L.dim > 1) cnt *= (L.M - cy + 1) / 2;
      if (L.dim > 2) cnt *= (L.M - cz + 1) / 2;
      Q1_DISPATCH(L.dim, {
        k_sor_colour<D, 1, true><<<grid1(cnt), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, col, omega, nullptr, x, b, r);
      });
    }
    return;
  }
  const Q2Layout lay = q2_layout(L.dim, L.M);
  const long long nv = (L.M + 1) / 2;
  for (int col = 0; col < ncol; ++col) {
    long long cnt = (nv - (col & 1) + 1) / 2;
    if (L.dim > 1) cnt *= (nv - ((col >> 1) & 1) + 1) / 2;
    if (L.dim > 2) cnt *= (nv - ((col >> 2) & 1) + 1) / 2;
    const unsigned grid = (unsigned)((cnt * 32 + 127) / 128);
    Q2_DISPATCH(L.dim, {
      k_ssc_q2<D><<<grid, 128, 0, st>>>(L.A, L.N, L.Np, L.M, L.dmask, col, omega, x, b, r, F, P, lay);
    });
  }
}

void launch_psc(const LevelView& L, double damp, double* x, const double* r, const double* F,
                const unsigned char* P, double* C, cudaStream_t st) {
  if (L.order == 1) {  // one-node blocks: x_i += damp r_i / a_ii, r unchanged
    g_launches.fetch_add(1, std::memory_order_relaxed);
    Q1_DISPATCH(L.dim, { k_psc_q1<D><<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, damp, x, r); });
    return;
  }
  g_launches.fetch_add(2, std::memory_order_relaxed);
  const unsigned grid = (unsigned)((ssc_blocks(L) * 32 + 127) / 128);
  Q2_DISPATCH(L.dim, {
    k_psc_block_q2<D><<<grid, 128, 0, st>>>(L.M, L.dmask, r, F, P, C);
    k_psc_gather_q2<D><<<grid1(L.N), kBlock, 0, st>>>(L.N, L.M, L.dmask, damp, C, x);
  });
}

static inline dim3 xfer_grid(long long M, int dim) {
  return dim3((unsigned)((M + 31) / 32), (unsigned)(dim > 1 ? (M + 7) / 8 : 1), (unsigned)(dim > 2 ? M : 1));
}

void launch_restrict(const LevelView& F, const LevelView& Cl, const double* rf, double* rc, double* rhsc,
                     double* solc, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (F.csr) {
    k_csr_restrict<<<grid1(Cl.N), kBlock, 0, st>>>(Cl.N, F.pt, rf, rc, rhsc, solc);
    return;
  }
  if (F.nc == 3) {
    if (F.order == 2)
      k_restrict3<2><<<xfer_grid(Cl.M, 3), dim3(32, 8), 0, st>>>((int)Cl.M, (int)F.M, F.dmask, rf, rc, rhsc, solc);
    else
      k_restrict3<1><<<xfer_grid(Cl.M, 3), dim3(32, 8), 0, st>>>((int)Cl.M, (int)F.M, F.dmask, rf, rc, rhsc, solc);
    return;
  }
  FMG_DISPATCH(F.dim, F.order, {
    dim3 gr = xfer_grid(Cl.M, D);
    if (D < 3) gr.z = (unsigned)F.nb;  // the problems of a batched level
    k_restrict<D, P><<<gr, dim3(32, 8), 0, st>>>((int)Cl.M, (int)F.M, F.dmask, rf, rc, rhsc, solc, F.Np, Cl.Np);
  });
}

void launch_prolong(const LevelView& Cl, const LevelView& F, const double* xc, double* xf, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (F.csr) {
    k_csr_prolong<<<grid1(F.N), kBlock, 0, st>>>(F.N, F.p, xc, xf);
    return;
  }
  if (F.nc == 3) {
    if (F.order == 2)
      k_prolong3<2><<<xfer_grid(F.M, 3), dim3(32, 8), 0, st>>>((int)F.M, (int)Cl.M, F.dmask, xc, xf);
    else
      k_prolong3<1><<<xfer_grid(F.M, 3), dim3(32, 8), 0, st>>>((int)F.M, (int)Cl.M, F.dmask, xc, xf);
    return;
  }
  FMG_DISPATCH(F.dim, F.order, {
    dim3 gr = xfer_grid(F.M, D);
    if (D < 3) gr.z = (unsigned)F.nb;
    k_prolong<D, P><<<gr, dim3(32, 8), 0, st>>>((int)F.M, (int)Cl.M, F.dmask, xc, xf, F.Np, Cl.Np);
  });
}

void launch_coarse_solve(const double* AinvT, int n, double damp, double* x, double* r, cudaStream_t st, int nb,
                         long long vs) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (n <= 1024) {
    k_coarse_solve<<<(unsigned)nb, 1024, 0, st>>>(AinvT, n, damp, x, r, vs);
  } else {
    static bool init = false;
    if (!init) {
      cudaFuncSetAttribute(k_coarse_solve_big, cudaFuncAttributeMaxDynamicSharedMemorySize, 48 * 1024 * 4);
      init = true;
    }
    k_coarse_solve_big<<<1, 1024, (size_t)n * sizeof(double), st>>>(AinvT, n, damp, x, r);
  }
}

void launch_lu(double* A, int n, int* piv, double* X, double* XT, cudaStream_t st) {
  g_launches.fetch_add(3, std::memory_order_relaxed);
  const size_t f_smem = (size_t)n * n * sizeof(double), i_smem = f_smem + (size_t)n * 32 * sizeof(double);
  constexpr size_t kMaxSmem = 200 * 1024;
  if (i_smem <= kMaxSmem) {  // the factors fit in shared memory (n <= 144)
    static bool init = false;
    if (!init) {
      cudaFuncSetAttribute(k_lu_factor_smem2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
      cudaFuncSetAttribute(k_lu_inverse_col, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
      init = true;
    }
    k_lu_factor_smem2<<<1, 1024, f_smem + (size_t)n * sizeof(int), st>>>(A, n, piv);
    k_lu_inverse_col<<<n, 256, f_smem + 2 * (size_t)n * sizeof(double), st>>>(A, piv, n, X);
  } else {  // blocked in global memory (L2-resident); perm lives in XT until the end
    int* perm = reinterpret_cast<int*>(XT);
    k_iota<<<grid1(n), kBlock, 0, st>>>(perm, n);
    for (int k0 = 0; k0 < n; k0 += kLuB) {
      const int k1 = std::min(n, k0 + kLuB);
      k_lu_panel<<<1, 1024, 0, st>>>(A, n, k0, k1, piv, perm);
      if (k1 < n) {
        k_lu_urows<<<grid1(n - k1, 128), 128, 0, st>>>(A, n, k0, k1, perm);
        k_lu_trail<<<dim3((unsigned)((n - k1 + 31) / 32), (unsigned)((n - k1 + 7) / 8)), dim3(32, 8), 0, st>>>(
            A, n, k0, k1, perm);
      }
      g_launches.fetch_add(3, std::memory_order_relaxed);
    }
    k_lu_permute<<<grid1((long long)n * n), kBlock, 0, st>>>(A, n, perm, X);   // X: the factors, rows interchanged
    k_transpose<<<grid1((long long)n * n), kBlock, 0, st>>>(X, n, A);         // A: the factors transposed
    k_lu_inverse_colT<<<n, 256, 2 * (size_t)n * sizeof(double), st>>>(A, piv, n, X);
    g_launches.fetch_add(4, std::memory_order_relaxed);
  }
  k_transpose<<<grid1((long long)n * n), kBlock, 0, st>>>(X, n, XT);
}

void launch_fill(double* x, long long n, double v, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (n > 0) k_fill<<<grid1(n), kBlock, 0, st>>>(x, n, v);
}
void launch_copy(const double* x, double* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (n > 0) k_copy<<<grid1(n), kBlock, 0, st>>>(x, y, n);
}
void launch_axpy(double alpha, const double* sc, int aslot, const double* x, double* y, long long n,
                 cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (n > 0) k_axpy<<<grid1(n), kBlock, 0, st>>>(alpha, sc, aslot, x, y, n);
}
void launch_dot(const double* x, const double* y, long long n, const Reduce& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dot<<<nchunks(n), kBlock, 0, st>>>(x, y, n, R);
}
void launch_dot_b(const double* x, const double* y, long long n, long long vs, int nb, const Reduce& R,
                  cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dot<<<dim3(nchunks(n), (unsigned)nb), kBlock, 0, st>>>(x, y, n, R, vs);
}
void launch_cg_update(const double* sc, double* x, const double* p, double* r, const double* a, double* w,
                      double* w2, double* q, long long n, const Reduce& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cg_update<<<nchunks(n), kBlock, 0, st>>>(sc, x, p, r, a, w, w2, q, n, R);
}
void launch_p_update(const double* sc, double* p, const double* q, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_p_update<<<grid1(n), kBlock, 0, st>>>(sc, p, q, n);
}
void launch_cg_update_b(const double* sc, double* x, const double* p, double* r, const double* a, double* w,
                        double* w2, double* q, long long n, long long vs, int nb, const double* frozen,
                        const Reduce& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cg_update<<<dim3(nchunks(n), (unsigned)nb), kBlock, 0, st>>>(sc, x, p, r, a, w, w2, q, n, R, vs, frozen);
}
void launch_p_update_b(const double* sc, double* p, const double* q, long long n, long long vs, int nb,
                       const double* frozen, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_p_update<<<dim3(grid1(n), (unsigned)nb), kBlock, 0, st>>>(sc, p, q, n, vs, frozen);
}

void launch_sample_kq(int dim, long long ncells_l, long long n_l, long long n_top, double ratio, int np,
                      const double* xi, const double* kcell, double* kq, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  long long nq = 1;
  for (int k = 0; k < dim; ++k) nq *= np;
  const unsigned g = grid1(ncells_l * nq);
  if (dim == 1) k_sample_kq<1><<<g, kBlock, 0, st>>>(ncells_l, n_l, n_top, ratio, np, xi, kcell, kq);
  else if (dim == 2) k_sample_kq<2><<<g, kBlock, 0, st>>>(ncells_l, n_l, n_top, ratio, np, xi, kcell, kq);
  else k_sample_kq<3><<<g, kBlock, 0, st>>>(ncells_l, n_l, n_top, ratio, np, xi, kcell, kq);
}

bool assemble_splits(int dim, int order, int nc, const AsmArgs& a) {
  return nc == 1 && dim == 3 && order == 1 && a.nl == 8 && a.nq == 8 && a.M < (1 << 20);
}

void launch_assemble(int dim, int order, const AsmArgs& a, const double* kbar_h, const double* ctab_h,
                     cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (a.nc == 3) {  // elasticity: a.Kbar / a.Ctab hold the elastic tables
    if (order == 2) k_assemble3<2><<<grid1(a.N), kBlock, 0, st>>>(a);
    else k_assemble3<1><<<grid1(a.N), kBlock, 0, st>>>(a);
    return;
  }
  if (dim == 3 && order == 1 && a.nl == 8 && a.nq == 8 && kbar_h && ctab_h && a.M < (1 << 20)) {
    Q1Tab tab;
    std::memcpy(tab.K, kbar_h, sizeof tab.K);
    std::memcpy(tab.C, ctab_h, sizeof tab.C);
    if (a.kq) k_assemble_q1_3d<true><<<grid1(a.N), kBlock, 0, st>>>(a, tab);
    else k_assemble_q1_3d<false><<<grid1(a.N), kBlock, 0, st>>>(a, tab);
    return;
  }
  const Q2Layout lay = q2_layout(dim, a.M);
  FMG_DISPATCH(dim, order, { k_assemble<D, P><<<grid1(a.N), kBlock, 0, st>>>(a, lay); });
}

}  // namespace fmg

namespace fmg {

// dense row-major copy of a (small) level matrix, for the coarse LU
template <int D, int P>
__global__ void k_densify(const double* __restrict__ A, long long N, long long Np, long long M,
                          double* __restrict__ Dm, const __grid_constant__ Q2Layout lay) {
  constexpr int NS = St<D, P>::NS;
  constexpr int W = 2 * P + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * NS) return;
  const long long i = t / NS;
  const int s = (int)(t % NS);
  long long ci[3];
  node_coords(i, M, D, ci);
  const long long o[3] = {s % W - P, D > 1 ? (s / W) % W - P : 0, D > 2 ? (s / (W * W)) % W - P : 0};
  long long cj[3];
  for (int k = 0; k < 3; ++k) cj[k] = ci[k] + o[k];
  for (int k = 0; k < D; ++k) if (cj[k] < 0 || cj[k] >= M) return;
  const long long j = cj[0] + M * (cj[1] + M * cj[2]);
  long long p = i;
  if constexpr (P == 2) {  // colour-major sliced storage
    const int r = q2_pattern<D>(s);
    for (int k = 0; k < D; ++k)
      if (((r >> k) & 1) && (ci[k] & 1)) return;
    p = q2c_pos<D>(lay, ci, M, r);
  }
  Dm[i * N + j] = A[(long long)s * Np + p];
}

void launch_level_to_f32(const LevelView& L, int nslots, float* out, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const long long n = (long long)nslots * L.N;
  const Q2Layout lay = q2_layout(L.dim, L.M);
  Q1_DISPATCH(L.dim, { k_expand_q2_f32<D><<<grid1(n), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, nslots, out, lay); });
}

void launch_galerkin(const LevelView& F, const LevelView& Cl, double* AC, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const Q2Layout lf = q2_layout(F.dim, F.M), lc = q2_layout(Cl.dim, Cl.M);
  const int ns = F.order == 1 ? (F.dim == 1 ? 3 : F.dim == 2 ? 9 : 27) : (F.dim == 1 ? 5 : F.dim == 2 ? 25 : 125);
  const unsigned g = grid1((long long)ns * Cl.N);
  const int mf = (int)F.M, mc = (int)Cl.M;
  if (F.nc == 3) {
    if (F.order == 2) k_galerkin<3, 2, 3><<<g, kBlock, 0, st>>>(F.A, F.Np, mf, AC, Cl.N, Cl.Np, mc, F.dmask, lf, lc);
    else k_galerkin<3, 1, 3><<<g, kBlock, 0, st>>>(F.A, F.Np, mf, AC, Cl.N, Cl.Np, mc, F.dmask, lf, lc);
    return;
  }
  if (F.order == 2) {
    Q1_DISPATCH(F.dim, { k_galerkin<D, 2, 1><<<g, kBlock, 0, st>>>(F.A, F.Np, mf, AC, Cl.N, Cl.Np, mc, F.dmask, lf, lc); });
  } else {
    Q1_DISPATCH(F.dim, { k_galerkin<D, 1, 1><<<g, kBlock, 0, st>>>(F.A, F.Np, mf, AC, Cl.N, Cl.Np, mc, F.dmask, lf, lc); });
  }
}

void launch_bdiag3(const LevelView& L, int mode, const double* w, const double* x, double* y, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_bdiag3<<<grid1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.center, mode, w, x, y);
}
void launch_xpwv3(const double* x, const double* w, const double* v, double* y, long long N, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_xpwv3<<<grid1(N), kBlock, 0, st>>>(x, w, v, y, N);
}
void launch_acc_prod3(double* acc, const double* a, const double* b, long long N, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_acc_prod3<<<grid1(N), kBlock, 0, st>>>(acc, a, b, N);
}

void vec32_spmv(int order, const float* A, long long N, long long Np, long long M, const float* x, const float* b,
                float* y, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (order == 2) k_spmv3<2, true, float><<<grid1(N), kBlock, 0, st>>>(A, N, Np, M, x, b, y);
  else k_spmv3<1, true, float><<<grid1(N), kBlock, 0, st>>>(A, N, Np, M, x, b, y);
}
void vec32_jacobi0(const float* A, long long N, long long Np, int center, float damp, const double* omega,
                   const float* b, float* x, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_jacobi0_3<float><<<grid1(N), kBlock, 0, st>>>(A, N, Np, center, damp, omega, b, x);
}
void vec32_jacobi_res(int order, const float* A, long long N, long long Np, long long M, double damp,
                      const double* omega, const float* x, const float* b, float* xout, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (order == 2)
    k_jacobi_res3<2, float><<<grid1(N), kBlock, 0, st>>>(A, N, Np, M, damp, omega, x, b, xout, (float*)nullptr, 0);
  else
    k_jacobi_res3<1, float><<<grid1(N), kBlock, 0, st>>>(A, N, Np, M, damp, omega, x, b, xout, (float*)nullptr, 0);
}
void vec32_restrict(int order, long long MC, long long MF, int dmask, const float* rf, float* bc, float* xc,
                    cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (order == 2)
    k_restrict3<2, float><<<xfer_grid(MC, 3), dim3(32, 8), 0, st>>>((int)MC, (int)MF, dmask, rf, bc, bc, xc);
  else
    k_restrict3<1, float><<<xfer_grid(MC, 3), dim3(32, 8), 0, st>>>((int)MC, (int)MF, dmask, rf, bc, bc, xc);
}
void vec32_prolong(int order, long long MF, long long MC, int dmask, const float* xc, float* xf, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (order == 2) k_prolong3<2, float><<<xfer_grid(MF, 3), dim3(32, 8), 0, st>>>((int)MF, (int)MC, dmask, xc, xf);
  else k_prolong3<1, float><<<xfer_grid(MF, 3), dim3(32, 8), 0, st>>>((int)MF, (int)MC, dmask, xc, xf);
}
void vec_to32(const double* x, const double* sc, int slot, int mode, float* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_vscale<double, float><<<grid1(n), kBlock, 0, st>>>(x, sc, slot, mode, y, n);
}
void vec_to64(const float* x, const double* sc, int slot, int mode, double* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_vscale<float, double><<<grid1(n), kBlock, 0, st>>>(x, sc, slot, mode, y, n);
}
void vec_f64_to_f32(const double* x, float* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_vscale<double, float><<<grid1(n), kBlock, 0, st>>>(x, nullptr, 0, 0, y, n);
}
void launch_fcg_beta(double* sc, bool first, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fcg_beta<<<1, 1, 0, st>>>(sc, first ? 1 : 0);
}

long long q2_slot_pos(int dim, long long M, long long i, int s, bool colour_major) {
  const long long c[3] = {i % M, dim > 1 ? (i / M) % M : 0, dim > 2 ? i / (M * M) : 0};
  if (colour_major) {
    const Q2Layout lay = q2_layout(dim, M);
    int r = 0, t = s;
    for (int k = 0; k < dim; ++k) {
      const int o = t % 5 - 2;
      if (o == 2 || o == -2) {
        if (c[k] & 1) return -1;
        r |= 1 << k;
      }
      t /= 5;
    }
    if (dim == 3) return q2c_pos<3>(lay, c, M, r);
    if (dim == 2) return q2c_pos<2>(lay, c, M, r);
    return q2c_pos<1>(lay, c, M, r);
  }
  if (dim == 3) {
    Q2Rows<3> q;
    q2_rows<3>(c, M, q);
    const int r = q2_pattern<3>(s);
    return ((q.valid >> r) & 1) ? q.idx[r] : -1;
  }
  if (dim == 2) {
    Q2Rows<2> q;
    q2_rows<2>(c, M, q);
    const int r = q2_pattern<2>(s);
    return ((q.valid >> r) & 1) ? q.idx[r] : -1;
  }
  Q2Rows<1> q;
  q2_rows<1>(c, M, q);
  const int r = q2_pattern<1>(s);
  return ((q.valid >> r) & 1) ? q.idx[r] : -1;
}

void launch_densify(const LevelView& L, double* Dm, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (L.csr) {
    k_csr_densify<<<grid1(L.N), kBlock, 0, st>>>(L.N, L.a, Dm);
    return;
  }
  if (L.nc == 3) {
    if (L.order == 2) k_densify3<2><<<grid1(L.N * St<3, 2>::NS), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, Dm);
    else k_densify3<1><<<grid1(L.N * St<3, 1>::NS), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, Dm);
    return;
  }
  const Q2Layout lay = q2_layout(L.dim, L.M);
  FMG_DISPATCH(L.dim, L.order, {
    constexpr int NS = St<D, P>::NS;
    k_densify<D, P><<<grid1(L.N * NS), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, Dm, lay);
  });
}

}  // namespace fmg
