// mixed.cu -- kernels of the mixed-precision solve (FP32 V-cycle, BF16 coarse
// right-hand sides and residuals, FP64 iterative refinement).
//
// The top level of a 3D Q1 hierarchy with a cell-wise coefficient is applied
// matrix-free: for node i and each of its 8 cells c,
//   (A x)_i = h/12 * sum_c k_c (4 x_i - x_e1 - x_e2 - x_e3 - x_v)
// where e1..e3 and v are the nodes of c that differ from i in two and three
// coordinates (the unit-cube Q1 stiffness has 1/3 on the diagonal, 0 between
// face neighbours, -1/12 between edge and vertex neighbours; this is the
// assembled operator K = sum_c k_c h K_ref of assemble-interior).  A row then
// reads 27 neighbour values (L1-resident) and 8 cell coefficients instead of
// 27 stored matrix entries: about 12 B/row of HBM traffic instead of 116.
// Coarse levels use the assembled matrices converted to FP32.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <type_traits>

#include "fmgpu_mixed.cuh"
#include "umma.cuh"

namespace fmg {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ float ldv(const float* p, long long i) { return p[i]; }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p, long long i) { return __bfloat162float(p[i]); }
__device__ __forceinline__ void stv(float* p, long long i, float v) { p[i] = v; }
__device__ __forceinline__ void stv(__nv_bfloat16* p, long long i, float v) { p[i] = __float2bfloat16_rn(v); }

__device__ __forceinline__ bool dir_node(int ix, int iy, int iz, int M, int dmask) {
  return (ix == 0 && (dmask & 1)) || (ix == M - 1 && (dmask & 2)) || (iy == 0 && (dmask & 4)) ||
         (iy == M - 1 && (dmask & 8)) || (iz == 0 && (dmask & 16)) || (iz == M - 1 && (dmask & 32));
}

__device__ __forceinline__ void epi2_apply(const Reduce2& R, double t0, double t1) {
  double* sc = R.scal;
  switch (R.epi) {
    case EPI2_LAMBDA: {  // (a, p); lam = rho / (a, p)
      sc[M_PA] = t0;
      sc[M_LAM] = sc[M_ALPHA] / t0;
      break;
    }
    case EPI2_RHO: {     // z = q / s: rho = (z, r)
      sc[M_ALPHA] = t0 / sc[M_SUSED];
      break;
    }
    case EPI2_FCG: {     // rho = (z, r); beta = -(z, a) / (p, a)
      const double su = sc[M_SUSED];
      sc[M_ALPHA] = t0 / su;
      sc[M_BETA] = -(t1 / su) / sc[M_PA];
      break;
    }
    case EPI2_UPDATE: {  // (r, r); the scale of the next FP32 residual
      sc[M_RR] = t0;
      sc[M_SUSED] = sc[M_SCALE];
      sc[M_SINV] = 1.0 / sc[M_SCALE];
      sc[M_SCALE] = t0 > 0.0 ? 1.0 / sqrt(t0) : 1.0;
      break;
    }
    default:
      sc[R.slot0] = t0; sc[R.slot1] = t1;
  }
}

// two fixed-order reductions finished by the last block (same tree as
// dr_finish); the epilogue is applied to the two sums
__device__ __forceinline__ void dr_finish2(double v0, double v1, const Reduce2& R, double* smem) {
  __shared__ bool is_last;
  double s0 = dr_fold256(v0, smem);
  double s1 = dr_fold256(v1, smem);
  if (threadIdx.x == 0) {
    R.part[2 * blockIdx.x] = s0;
    R.part[2 * blockIdx.x + 1] = s1;
    __threadfence();
    unsigned done = atomicAdd(R.counter, 1u);
    is_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double a0 = 0.0, a1 = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += kBlock) {
    a0 = a0 + __ldcg(R.part + 2 * k);
    a1 = a1 + __ldcg(R.part + 2 * k + 1);
  }
  double t0 = dr_fold256(a0, smem);
  double t1 = dr_fold256(a1, smem);
  if (threadIdx.x == 0) {
    epi2_apply(R, t0, t1);
    *R.counter = 0u;
  }
}

// ------------------------------------------------- matrix-free top level
// The Q1 row of a node from the coefficients k[cz][cy][cx] of its 8 cells
// (index 0: the cell on the lower side of the node along that axis) and the
// values X(dx, dy, dz) of its neighbours, zero where eliminated: the diagonal
// d = 4 hs K (K the sum of the 8 cells) and ax = (A x)_i, evaluated as 4 K x_i
// minus, over the 12 face diagonals, the sum of the two cells sharing each
// times its value, minus, over the 8 body diagonals, the one cell times its
// value (the Q1 stiffness has weight zero between axis neighbours).  FP64
// (DIFF): the row as sum_j w_j (x_i - x_j) -- the weights sum to 4 K, and the
// differences of a smooth iterate are small, so the true residual's rounding
// is far below that of 4 K x_i - sum_j w_j x_j.
template <typename T, bool HX, bool DIFF, typename XF>
__device__ __forceinline__ void mf_row(const T (&k)[2][2][2], const XF& X, T hs, T& ax, T& d, T& xc) {
  const T wc[2][2] = {{k[0][0][0] + k[1][0][0], k[0][0][1] + k[1][0][1]},
                      {k[0][1][0] + k[1][1][0], k[0][1][1] + k[1][1][1]}};
  const T ksum = (wc[0][0] + wc[0][1]) + (wc[1][0] + wc[1][1]);
  T sacc = T(0);
  xc = T(0);
  if (HX) {
    xc = X(0, 0, 0);
    // three independent sums (the plane's own 4 terms, then 8 for each of the
    // planes below and above) so that the multiply-add chains overlap
    T sp[3] = {T(0), T(0), T(0)};
    auto term = [&](int a, T w, T xj) { sp[a] = DIFF ? fma(w, xc - xj, sp[a]) : fma(w, xj, sp[a]); };
#pragma unroll
    for (int sy = 0; sy < 2; ++sy)
#pragma unroll
      for (int sx = 0; sx < 2; ++sx) term(0, wc[sy][sx], X(2 * sx - 1, 2 * sy - 1, 0));
#pragma unroll
    for (int cz = 0; cz < 2; ++cz) {
      const int dz = 2 * cz - 1;
#pragma unroll
      for (int sx = 0; sx < 2; ++sx)  // face diagonals (sx, 0, sz): cells (sx, *, sz)
        term(1 + cz, k[cz][0][sx] + k[cz][1][sx], X(2 * sx - 1, 0, dz));
#pragma unroll
      for (int sy = 0; sy < 2; ++sy)  // face diagonals (0, sy, sz): cells (*, sy, sz)
        term(1 + cz, k[cz][sy][0] + k[cz][sy][1], X(0, 2 * sy - 1, dz));
#pragma unroll
      for (int sy = 0; sy < 2; ++sy)
#pragma unroll
        for (int sx = 0; sx < 2; ++sx)  // body diagonals
          term(1 + cz, k[cz][sy][sx], X(2 * sx - 1, 2 * sy - 1, dz));
    }
    sacc = sp[0] + (sp[1] + sp[2]);
    if (!DIFF) sacc = fma(T(4) * ksum, xc, -sacc);
  }
  d = T(4) * hs * ksum;
  ax = hs * sacc;
}

// mode 0: A x; 1: b - A x; 2: x + w (b - A x)/d; 3: w b/d (w over d formed
// beforehand when use_wd)
template <int MODE, typename T>
__device__ __forceinline__ T mf_out(T ax, T d, T xc, T bb, T o, bool use_wd) {
  if (MODE == 0) return ax;
  if (MODE == 1) return bb - ax;
  if (MODE == 2) return use_wd ? fma(o, bb - ax, xc) : fma(o, (bb - ax) / d, xc);
  return use_wd ? o * bb : o * (bb / d);
}

constexpr int kFX = 32, kFY = 16, kFZ = 32;   // tile: nodes along x, y; planes per CTA
constexpr int kFRows = kFY + 2;               // x rows of a plane (y0-1 .. y0+16)
constexpr int kFCRows = kFY + 1;              // cell rows of a plane (y0-1 .. y0+15)
constexpr int kFPW = kFX + 2;                 // packed row: x0-1 .. x0+32
constexpr int kXW = 40;                       // tensor-copy halo row: 40 FP32 from the 16-byte boundary at or below x0-1
constexpr int kOW = 36;                       // operand box row: 36 elements from tensor x0 (node x0 - front)
constexpr int kFThreads = 256;
constexpr int kFaceNodes = 1024;              // nodes per face CTA

// the cell tile of a plane as one TMA box: cells x0-1-COFF .. x0-1-COFF+CW-1
// (the box starts on a 16-byte boundary), rows y0-1 .. y0+15
template <typename T>
struct CellBox {
  static constexpr int CW = sizeof(T) == 4 ? 36 : 34;       // cells per row
  static constexpr int COFF = sizeof(T) == 4 ? 3 : 1;       // where cell x0-1 sits in a row
  static constexpr uint32_t CTX = kFCRows * CW * sizeof(T);  // bytes per box
};

struct MftGeo {
  int nbx, nby, nbz, nmain;   // tiled box: nbx x nby x nbz tiles from the origin
  int nface;                  // face CTAs (they come first in the grid)
  long long X1, Y1, Z1;       // the tiled box's extents in nodes
  int ax, ay, az;             // the tiled CTAs write [ax, X1) x [ay, Y1) x [az, Z1) (1: the face at 0 is left out)
  long long F;                // nodes outside what the tiled CTAs write
};

// the u-th coordinate outside [a, b) along an axis of M nodes
__device__ __forceinline__ int outside(long long u, long long a, long long b) { return (int)(u < a ? u : u + (b - a)); }

// node (ix, iy, iz) of the f-th node the face CTAs own: the planes z outside
// [az, Z1), then the rows y outside [ay, Y1) of the planes inside, then the
// columns x outside [ax, X1) of the rows inside
__device__ __forceinline__ void face_node(long long f, const MftGeo& q, int M, int& ix, int& iy, int& iz) {
  const long long MM = (long long)M * M;
  const long long nz = q.Z1 - q.az, ny = q.Y1 - q.ay, nx = q.X1 - q.ax;
  const long long s1 = MM * (M - nz);
  if (f < s1) {
    iz = outside(f / MM, q.az, q.Z1);
    const long long r = f % MM;
    iy = (int)(r / M);
    ix = (int)(r % M);
    return;
  }
  f -= s1;
  const long long a2 = (long long)M * (M - ny), s2 = a2 * nz;
  if (f < s2) {
    iz = (int)(q.az + f / a2);
    const long long r = f % a2;
    iy = outside(r / M, q.ay, q.Y1);
    ix = (int)(r % M);
    return;
  }
  f -= s2;
  const long long cx = M - nx, a3 = cx * ny;
  iz = (int)(q.az + f / a3);
  const long long r = f % a3;
  iy = (int)(q.ay + r / cx);
  ix = outside(r % cx, q.ax, q.X1);
}

template <typename T, typename TV, typename TX, int MODE, bool RED>
__device__ __forceinline__ void mf_face_cta(const MFArgsT<T>& g, const MftGeo& geo, int fb, const TX* __restrict__ x,
                                            const T* __restrict__ b, T* __restrict__ y, const TV* __restrict__ v,
                                            const TV* __restrict__ v2, double& acc0, double& acc1) {
  constexpr bool HX = MODE != 3;
  constexpr bool HB = MODE != 0;
  constexpr bool DIFF = sizeof(T) == 8;
  constexpr bool HO = MODE == 2 || MODE == 3;
  const int M = g.M, n = g.n, dm = g.dmask;
  const long long MM = (long long)M * M;
  auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
  const bool uwd = g.wd != nullptr;
  const long long f0 = (long long)fb * kFaceNodes;
#pragma unroll 1
  for (int q = 0; q < kFaceNodes / kFThreads; ++q) {
    const long long f = f0 + threadIdx.x + (long long)q * kFThreads;
    if (f >= geo.F) break;
    int ix, iy, iz;
    face_node(f, geo, M, ix, iy, iz);
    const long long in = (long long)iz * MM + (long long)iy * M + ix;  // natural (omega)
    const long long io = g.ol.at(ix, iy, iz);                          // operands
    T ax, d, xc;
    if (dirf(ix, 1, 2) || dirf(iy, 4, 8) || dirf(iz, 16, 32)) {
      xc = HX ? (T)x[g.xl.at(ix, iy, iz)] : T(0);
      ax = xc;
      d = T(1);
    } else {
      T k[2][2][2];
#pragma unroll
      for (int cz = 0; cz < 2; ++cz)
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
          for (int cx = 0; cx < 2; ++cx) {
            const int ex = ix - 1 + cx, ey = iy - 1 + cy, ez = iz - 1 + cz;
            const bool in = ex >= 0 && ex < n && ey >= 0 && ey < n && ez >= 0 && ez < n;
            k[cz][cy][cx] = in ? __ldg(g.k + ex + (long long)n * (ey + (long long)n * ez)) : T(0);
          }
      auto X = [&](int dx, int dy, int dz) -> T {
        const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
        const bool in = jx >= 0 && jx < M && jy >= 0 && jy < M && jz >= 0 && jz < M && !dirf(jx, 1, 2) &&
                        !dirf(jy, 4, 8) && !dirf(jz, 16, 32);
        return in ? (T)x[g.xl.at(jx, jy, jz)] : T(0);
      };
      mf_row<T, HX, DIFF>(k, X, g.hs, ax, d, xc);
    }
    const T bb = HB ? __ldg(b + io) : T(0);
    const T o = (HO && uwd) ? __ldg(g.wd + io) : ((HO && g.omega) ? __ldg(g.omega + in) : g.w);
    const T out = mf_out<MODE>(ax, d, xc, bb, o, uwd);
    y[g.yl.at(ix, iy, iz)] = out;
    if (RED) {
      constexpr bool VX = sizeof(T) == 8;  // the FP64 operator reduces (A p, p): the vector is x itself
      acc0 = fma((double)out, VX ? (double)xc : (double)v[io], acc0);
      if (v2) acc1 = fma((double)out, (double)v2[io], acc1);
    }
  }
}

// The operator as one launch over two kinds of CTA.  Tiled CTAs own a 32 x 16
// column of nodes (thread (lx, ly): the y-adjacent nodes 2ly, 2ly+1) and
// march z through 32 planes.  Face CTAs (first in the grid) evaluate, from
// global memory, the nodes outside the tiled box -- the faces x, y or z = 2^L
// where the box stops short of the grid, the whole grid when it is below 32
// cells a side -- and the Dirichlet faces x, y, z = 0 inside it (identity
// rows), 1024 nodes each.  FP32 arithmetic, or FP64 in difference form with
// each x value widened once as it enters the registers.
// A stage of a tiled CTA's shared-memory ring (6 slots, 5 for the smoothing
// mode) holds what one step reads: the x halo of the plane above, the 17 x 36
// cell tile (one TMA box) and the per-node operands of the step's own plane
// (b, the damping, the FP64 reduction vectors).  An FP32 x and the FP32
// modes' operands are kept padded, so each comes as one TMA box per stage:
// the 18 x 40 halo from the 16-byte boundary at or below node x0 - 1 of a map
// that leaves out the Dirichlet faces (they and the outside read as zero),
// and 16 x 36 operand boxes from node x0 - front.  An FP64 x (the true
// residual of FP64 vectors) comes by cp.async per element (18 x 34, the
// eliminated and outside entries zero-filled at the copy), its operands by a
// cp.async per node and thread.  All copies of a stage complete on its full
// mbarrier (the TMA's expect-tx arrival, plus 256 cp.async arrivals where
// there are any); each warp releases a stage on its empty mbarrier once it has
// read it, and a slot is refilled only after all 8 warps have released it, so
// warps drift apart by a few steps and no block barrier is needed.  Stages are
// requested two or three steps before they are read.
// A thread keeps the x values and cells its two nodes read in registers as it
// marches z, reading each plane once (the loop runs three steps per turn so
// register roles rotate at compile time).
constexpr int kCRing = 6;   // ring slots (5 where six stages would not leave room for two CTAs per SM)
constexpr int kPX = kFPW;   // packed x row: x0-1 .. x0+32

template <typename T, typename TV, typename TX, int MODE, bool RED>
struct MfcLayout {
  static constexpr bool HB = MODE != 0, HO = MODE == 2 || MODE == 3, HX = MODE != 3;
  static constexpr bool XT = sizeof(TX) == 4;        // an FP32 x halo comes by tensor copy (padded x)
  static constexpr bool OT = sizeof(T) == 4;         // so do the FP32 modes' operands (padded)
  static constexpr bool VX = RED && sizeof(T) == 8;  // the FP64 operator reduces (A p, p): v is x
  static constexpr bool HV = RED && !VX;             // reduction vectors to load
  static constexpr int up(int b) { return (b + 127) / 128 * 128; }
  static constexpr int XR = XT ? kXW : kPX;          // halo row
  static constexpr int XS = HX ? up(kFRows * XR * (int)sizeof(TX)) : 0;  // x halo
  static constexpr int CS = up(kFCRows * CellBox<T>::CW * (int)sizeof(T));  // cell box (TMA)
  static constexpr int OPN = OT ? kFY * kOW : 2 * kFThreads;  // operand elements of a stage
  static constexpr int OB = HB ? up(OPN * (int)sizeof(T)) : 0;  // b of the step's plane
  static constexpr int OO = HO ? up(OPN * (int)sizeof(T)) : 0;  // damping
  static constexpr int OV = HV ? up(OPN * (int)sizeof(TV)) : 0;  // reduction vectors
  static constexpr int SB = XS + CS + OB + OO + 2 * OV;
  static constexpr int NR = SB * kCRing > 100 * 1024 ? kCRing - 1 : kCRing;  // ring slots: two CTAs per SM
  static constexpr int LOOK = NR - 1;  // stage j is requested at step j - LOOK and read at step j - 2
  static constexpr int SMEM = NR * SB + 2 * NR * 8 + 128;
  // every copy of a stage is a tensor copy: its full barrier takes one arrival
  static constexpr bool ALLT = (!HX || XT) && (OT || !(HB || HO || HV));
};

__device__ __forceinline__ void cpa(void* dst, const void* src, bool ok, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
// one arrival on the mbarrier once this thread's earlier cp.async copies have landed
__device__ __forceinline__ void cpa_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(umma::smem_u32(bar)) : "memory");
}

// OPT: 1 per-node damping present (g.wd or g.omega), 2 a second reduction
// vector, 4 the damping already divided by the diagonal (g.wd)
template <typename T, typename TV, typename TX, int MODE, bool RED, int OPT>
__global__ void __launch_bounds__(kFThreads, (sizeof(T) == 4 && MODE != 2) ? 3 : 2)
k_mfc(MFArgsT<T> g, const __grid_constant__ CUtensorMap tk_cells, const __grid_constant__ CUtensorMap tm_x,
      const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_o,
      const __grid_constant__ CUtensorMap tm_v, const __grid_constant__ CUtensorMap tm_v2, MftGeo geo,
      const TX* __restrict__ x, const T* __restrict__ b, T* __restrict__ y, const TV* __restrict__ v,
      const TV* __restrict__ v2, Reduce2 R) {
  typedef MfcLayout<T, TV, TX, MODE, RED> L;
  typedef CellBox<T> LC;
  constexpr bool DIFF = sizeof(T) == 8;  // the FP64 operator in difference form
  constexpr bool HX = L::HX, HB = L::HB, HO = L::HO;
  constexpr bool OM = HO && (OPT & 1), V2 = RED && (OPT & 2), UWD = HO && (OPT & 4);
  extern __shared__ __align__(128) unsigned char sm_dyn[];
  __shared__ double red[8];
  unsigned char* sm = sm_dyn + ((128u - (umma::smem_u32(sm_dyn) & 127u)) & 127u);
  const int tid = threadIdx.x;
  double acc0 = 0.0, acc1 = 0.0;
  if ((int)blockIdx.x >= geo.nface) {
    const int M = g.M, dm = g.dmask;
    auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
    const T* om_src = UWD ? g.wd : g.omega;  // per-node damping source (OM)
    const T hs = g.hs;
    const int bid = (int)blockIdx.x - geo.nface;
    const int bx = bid % geo.nbx, by = (bid / geo.nbx) % geo.nby, bz = bid / (geo.nbx * geo.nby);
    const int x0 = bx * kFX, y0 = by * kFY, z0 = bz * kFZ;
    const int lx = tid & 31, ly = tid >> 5;
    constexpr int NR = L::NR, LOOK = L::LOOK;
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + NR * L::SB);
    uint64_t* empty = full + NR;
    if (tid == 0)
      for (int s = 0; s < NR; ++s) {
        umma::mbar_init_count(&full[s], L::ALLT ? 1 : kFThreads + 1);
        umma::mbar_init_count(&empty[s], kFThreads / 32);
      }
    __syncthreads();
    // tensor-copy halo: its box starts on the 16-byte boundary at or below
    // node x0 - 1 of the map, which leaves out the Dirichlet faces (so that
    // they, like the outside, read as zero); node x0 - 1 sits at column xoff
    const int lox = dm & 1, loy = (dm >> 2) & 1, loz = (dm >> 4) & 1;
    const int xoff = (3 - lox) & 3;
    const int fr = g.ol.front;  // operand boxes start at tensor x0: node x0 + c at column c + front
    const int last = kFZ + 1;
    // this thread's share of the x halo: elements tid, tid+256, tid+512 of 18 x 34
    int hoff[3];
    bool hok[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = tid + q * kFThreads;
      const int r = e / kPX, jj = e - r * kPX;
      const int xx = x0 - 1 + jj, yy = y0 - 1 + r;
      hok[q] = e < kFRows * kPX && xx >= 0 && xx < M && yy >= 0 && yy < M && !dirf(xx, 1, 2) && !dirf(yy, 4, 8);
      hoff[q] = hok[q] ? (int)(g.xl.front + xx + (long long)g.xl.py * yy) : 0;
    }
    const int ix = x0 + lx, iy0 = y0 + 2 * ly;
    bool ok = true;  // every wait of this warp so far completed; after one gives up, the rest wait 1 ms at most
    auto wait = [&](uint64_t* bar, uint32_t parity) {
      bool w = umma::mbar_test(bar, parity);
      if (!w) w = ok ? umma::mbar_wait(bar, parity) : umma::mbar_wait_for(bar, parity, 1 << 16, 1000000ull);
      ok = __all_sync(0xffffffffu, w) && ok;
    };
    // stage j: x plane z0-1+j, cell plane z0-2+j, operands of plane z0-2+j, in
    // ring slot j % NR; the issue and read streams count slots and phases
    int is = 0, rs = 0;          // slot of the next stage to request / to read
    uint32_t ip = 0u, rp = 0u;   // its phase parity
    auto issue = [&](int j) {
      const int s = is;
      if (j >= NR) wait(&empty[s], ip ^ 1u);  // all warps released the slot's previous stage
      unsigned char* st = sm + s * L::SB;
      const int zo = z0 - 2 + j;  // the operands' plane
      const bool ops = zo >= z0 && (HB || HO || L::HV);
      if (tid == 0) {
        uint32_t tx = LC::CTX;
        if (HX && L::XT) tx += kFRows * kXW * (uint32_t)sizeof(TX);
        if (L::OT && ops)
          tx += (uint32_t)L::OPN * ((HB ? (uint32_t)sizeof(T) : 0u) + (OM ? (uint32_t)sizeof(T) : 0u) +
                                    (L::HV ? (uint32_t)sizeof(TV) : 0u) + (V2 ? (uint32_t)sizeof(TV) : 0u));
        umma::fence_async_smem();
        umma::mbar_arrive_expect_tx(&full[s], tx);
        umma::tma_load_3d(st + L::XS, &tk_cells, &full[s], x0 - 1 - LC::COFF, y0 - 1, z0 - 2 + j);
        if (HX && L::XT) umma::tma_load_3d(st, &tm_x, &full[s], x0 - 1 - xoff - lox, y0 - 1 - loy, z0 - 1 + j - loz);
        if (L::OT && ops) {
          unsigned char* op = st + L::XS + L::CS;
          if (HB) umma::tma_load_3d(op, &tm_b, &full[s], x0, y0, zo);
          if (OM) umma::tma_load_3d(op + L::OB, &tm_o, &full[s], x0, y0, zo);
          if (L::HV) umma::tma_load_3d(op + L::OB + L::OO, &tm_v, &full[s], x0, y0, zo);
          if (V2) umma::tma_load_3d(op + L::OB + L::OO + L::OV, &tm_v2, &full[s], x0, y0, zo);
        }
      }
      if (HX && !L::XT) {
        const int z = z0 - 1 + j;
        const bool zok = z >= 0 && z < M && !dirf(z, 16, 32);
        const TX* pl = x + (zok ? (long long)z * g.xl.pz : 0ll);
        TX* xs = reinterpret_cast<TX*>(st);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int e = tid + q * kFThreads;
          if (q < 2 || e < kFRows * kPX) cpa(xs + e, pl + hoff[q], zok && hok[q], (int)sizeof(TX));
        }
      }
      if (!L::OT && ops) {
        unsigned char* op = st + L::XS + L::CS;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const long long i = g.ol.at(ix, iy0 + r, zo);
          const int k = r * kFThreads + tid;
          if (HB) cpa(reinterpret_cast<T*>(op) + k, b + i, true, (int)sizeof(T));
          if (OM) cpa(reinterpret_cast<T*>(op + L::OB) + k, om_src + i, true, (int)sizeof(T));
          if (L::HV) cpa(reinterpret_cast<TV*>(op + L::OB + L::OO) + k, v + i, true, (int)sizeof(TV));
          if (V2) cpa(reinterpret_cast<TV*>(op + L::OB + L::OO + L::OV) + k, v2 + i, true, (int)sizeof(TV));
        }
      }
      if (!L::ALLT) cpa_arrive(&full[s]);
      if (++is == NR) {
        is = 0;
        ip ^= 1u;
      }
    };
    auto consume = [&](T (&xv)[4][3], T (&kv)[3][2], bool want_k) {  // the next stage in the read stream
      wait(&full[rs], rp);
      const unsigned char* st = sm + rs * L::SB;
      if (HX) {
        const TX* xs = reinterpret_cast<const TX*>(st) + (L::XT ? xoff : 0);
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int c = 0; c < 3; ++c) xv[k][c] = (T)xs[(2 * ly + k) * L::XR + lx + c];
      }
      if (want_k) {
        const T* cs = reinterpret_cast<const T*>(st + L::XS);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 2; ++c) kv[r][c] = cs[(2 * ly + r) * LC::CW + lx + c + LC::COFF];
      }
    };
    auto release = [&]() {  // the stage just read; the read stream moves on
      __syncwarp();
      if (lx == 0) umma::mbar_arrive(&empty[rs]);
      if (++rs == NR) {
        rs = 0;
        rp ^= 1u;
      }
    };
    T xr[3][4][3], kr[3][3][2];
    for (int j = 0; j < LOOK && j <= last; ++j) issue(j);
    consume(xr[0], kr[1], false);  // stage 0: x plane z0-1 (its cell plane is not read)
    release();
    consume(xr[1], kr[0], true);   // stage 1: x plane z0, cell plane z0-1
    release();
    const bool dirx = dirf(ix, 1, 2);
    const bool diry0 = dirf(iy0, 4, 8), diry1 = dirf(iy0 + 1, 4, 8);
    // step t (plane z0+t): x planes iz-1, iz, iz+1 in xr[t%3], xr[(t+1)%3],
    // xr[(t+2)%3] (the last one read now), cell planes iz-1, iz in kr[t%2],
    // kr[(t+1)%2] (the last one read now); the operands come with stage t+2
    auto step = [&](auto Qc, int t) {
      constexpr int Q = decltype(Qc)::value;
      constexpr int PM = Q % 3, P0 = (Q + 1) % 3, PP = (Q + 2) % 3, CM = Q % 3, C0 = (Q + 1) % 3;
      if (t + LOOK <= last) issue(t + LOOK);
      consume(xr[PP], kr[C0], true);  // stage t+2
      const unsigned char* op = sm + rs * L::SB + L::XS + L::CS;
      T bb[2], oo[2];
      TV vv[2], vv2[2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int k = L::OT ? (2 * ly + r) * kOW + lx + fr : r * kFThreads + tid;
        bb[r] = HB ? reinterpret_cast<const T*>(op)[k] : T(0);
        oo[r] = OM ? reinterpret_cast<const T*>(op + L::OB)[k] : g.w;
        vv[r] = L::HV ? reinterpret_cast<const TV*>(op + L::OB + L::OO)[k] : TV(0);
        vv2[r] = V2 ? reinterpret_cast<const TV*>(op + L::OB + L::OO + L::OV)[k] : TV(0);
      }
      release();
      const int iz = z0 + t;
      const bool dirz = dirf(iz, 16, 32);
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        T k[2][2][2];
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
          for (int cx = 0; cx < 2; ++cx) {
            k[0][cy][cx] = kr[CM][r + cy][cx];
            k[1][cy][cx] = kr[C0][r + cy][cx];
          }
        auto X = [&](int dx, int dy, int dz) -> T {
          return xr[dz < 0 ? PM : (dz > 0 ? PP : P0)][r + 1 + dy][1 + dx];
        };
        T ax, d, xc;
        mf_row<T, HX, DIFF>(k, X, hs, ax, d, xc);
        const T out = mf_out<MODE>(ax, d, xc, bb[r], oo[r], UWD);
        if (!(dirz || dirx || (r ? diry1 : diry0))) {  // identity rows: the face CTAs
          y[g.yl.at(ix, iy0 + r, iz)] = out;
          if (RED) {
            acc0 = fma((double)out, L::VX ? (double)xc : (double)vv[r], acc0);
            if (V2) acc1 = fma((double)out, (double)vv2[r], acc1);
          }
        }
      }
    };
    typedef std::integral_constant<int, 0> Q0;
    typedef std::integral_constant<int, 1> Q1;
    typedef std::integral_constant<int, 2> Q2;
    typedef std::integral_constant<int, 3> Q3;
    typedef std::integral_constant<int, 4> Q4;
    typedef std::integral_constant<int, 5> Q5;
    int t = 0;
#pragma unroll 1
    for (; t + 3 <= kFZ; t += 3) {
      step(Q0{}, t);
      step(Q1{}, t + 1);
      step(Q2{}, t + 2);
    }
    if constexpr (kFZ % 3 > 0) step(Q0{}, t);
    if constexpr (kFZ % 3 > 1) step(Q1{}, t + 1);
    // every stage requested has been waited for; a wait that gave up voids the results
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (__syncthreads_or(!ok) && tid == 0 && g.err) *g.err = 1.0;
  } else {
    mf_face_cta<T, TV, TX, MODE, RED>(g, geo, (int)blockIdx.x, x, b, y, v, v2, acc0, acc1);
  }
  if (RED) dr_finish2(acc0, acc1, R, red);
}

// ------------------------------------------------------ stored FP32 levels
template <int D, int P>
struct St32 {
  static constexpr int W = 2 * P + 1;
  static constexpr int NS = D == 1 ? W : (D == 2 ? W * W : W * W * W);
  static constexpr int CENTER = (NS - 1) / 2;
};

template <int D, int P>
__device__ __forceinline__ long long soff(int s, long long M) {
  constexpr int W = 2 * P + 1;
  long long o = (long long)(s % W - P);
  if (D > 1) o += M * (long long)((s / W) % W - P);
  if (D > 2) o += M * M * (long long)((s / (W * W)) % W - P);
  return o;
}

// mode 0: y = A x; 1: y = b - A x; 2: y = x + w (b - Ax)/d; 3: y = w b/d
// RPT consecutive rows per thread: with four, a slot's four coefficients come
// as one 16-byte load (the slot arrays are 256-byte aligned, Np a multiple of
// 64) and the neighbour values through L1 -- for the large levels, which are
// bandwidth-bound; one row per thread on the small, latency-bound ones (and
// on the 125-slot 3D Q2 rows, whose four-row form would spill).  Each row
// sums in slot order either way.
template <int D, int P, int MODE, typename TB, typename TY, bool RED, int RPT>
__global__ void __launch_bounds__(kBlock)
k_st32(const float* __restrict__ A, long long N, long long Np, long long M, float w, const float* __restrict__ om,
       const float* __restrict__ x, const TB* __restrict__ b, TY* __restrict__ y, const double* __restrict__ v,
       const double* __restrict__ v2, Reduce2 R) {
  constexpr int NS = St32<D, P>::NS;
  constexpr int C = St32<D, P>::CENTER;
  static_assert(RPT == 1 || RPT == 4, "one or four rows per thread");
  __shared__ double smem[8];
  double acc0 = 0.0, acc1 = 0.0;
  const long long i0 = ((long long)blockIdx.x * kBlock + threadIdx.x) * RPT;
  if (i0 < N) {
    float s[RPT], d[RPT], xc[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) s[r] = xc[r] = 0.f;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      if (MODE == 3 && k != C) continue;
      float a[RPT];
      if constexpr (RPT == 4) {
        const float4 a4 = __ldg(reinterpret_cast<const float4*>(A + (long long)k * Np + i0));
        a[0] = a4.x; a[1] = a4.y; a[2] = a4.z; a[3] = a4.w;
      } else {
#pragma unroll
        for (int r = 0; r < RPT; ++r) a[r] = __ldg(A + (long long)k * Np + i0 + r);
      }
      if (k == C) {
#pragma unroll
        for (int r = 0; r < RPT; ++r) d[r] = a[r];
      }
      if (MODE == 3) continue;
      const long long o = soff<D, P>(k, M);
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const float xv = __ldg(x + clampi(i0 + r + o, N));
        s[r] = fmaf(a[r], xv, s[r]);
        if (k == C) xc[r] = xv;
      }
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const long long i = i0 + r;
      if (i < N) {
        float out;
        if (MODE == 0) out = s[r];
        else if (MODE == 1) out = ldv(b, i) - s[r];
        else if (MODE == 2) out = fmaf(om ? om[i] : w, (ldv(b, i) - s[r]) / d[r], xc[r]);
        else out = (om ? om[i] : w) * (ldv(b, i) / d[r]);
        stv(y, i, out);
        if (RED) {
          acc0 = fma((double)out, (double)v[i], acc0);
          if (v2) acc1 = fma((double)out, (double)v2[i], acc1);
        }
      }
    }
  }
  if (RED) dr_finish2(acc0, acc1, R, smem);
}

__device__ __forceinline__ bool fdir(int c, int M, int k, int dmask) {
  return (c == 0 && ((dmask >> (2 * k)) & 1)) || (c == M - 1 && ((dmask >> (2 * k + 1)) & 1));
}

// Q1 restriction: three fine nodes per direction with weights 1/2, 1, 1/2,
// fixed-size loops in registers
template <int D, typename TR>
__device__ __forceinline__ void restrict_q1_node(int MC, int MF, int dmask, const TR* __restrict__ rf,
                                                 __nv_bfloat16* __restrict__ bc, float* __restrict__ xc, int c0,
                                                 int c1, int c2) {
  const int cJ[3] = {c0, c1, c2};
  const long long J = cJ[0] + (long long)MC * (cJ[1] + (long long)MC * cJ[2]);
  if (D == 3 && cJ[0] >= 1 && cJ[0] <= MC - 2 && cJ[1] >= 1 && cJ[1] <= MC - 2 && cJ[2] >= 1 && cJ[2] <= MC - 2) {
    // interior coarse node: its 27 fine neighbours lie inside and off every
    // face; weights 1/2, 1, 1/2 applied one direction at a time
    const long long MF2 = (long long)MF * MF;
    const TR* p0 = rf + (2 * cJ[0] - 1) + (long long)MF * (2 * cJ[1] - 1) + MF2 * (2 * cJ[2] - 1);
    float t[3];
#pragma unroll
    for (int z = 0; z < 3; ++z) {
      float u[3];
#pragma unroll
      for (int y = 0; y < 3; ++y) {
        const TR* q = p0 + (long long)MF * y + MF2 * z;
        u[y] = fmaf(.5f, ldv(q, 0) + ldv(q, 2), ldv(q, 1));
      }
      t[z] = fmaf(.5f, u[0] + u[2], u[1]);
    }
    bc[J] = __float2bfloat16_rn(fmaf(.5f, t[0] + t[2], t[1]));
    xc[J] = 0.f;
    return;
  }
  bool dj = false;
#pragma unroll
  for (int k = 0; k < D; ++k) dj = dj || fdir(cJ[k], MC, k, dmask);
  float acc = 0.f;
  if (!dj) {
    float w[3][3];
    int f[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        if (k >= D) { f[k][t] = 0; w[k][t] = t == 1 ? 1.f : 0.f; continue; }
        const int fc = 2 * cJ[k] + t - 1;
        const bool ok = fc >= 0 && fc < MF && !fdir(fc, MF, k, dmask);
        f[k][t] = ok ? fc : 0;
        w[k][t] = ok ? (t == 1 ? 1.f : .5f) : 0.f;
      }
#pragma unroll
    for (int z = 0; z < 3; ++z)
#pragma unroll
      for (int y = 0; y < 3; ++y) {
        const long long row = (long long)MF * (f[1][y] + (long long)MF * f[2][z]);
        const float wyz = w[1][y] * w[2][z];
#pragma unroll
        for (int xx = 0; xx < 3; ++xx) acc = fmaf(w[0][xx] * wyz, ldv(rf, row + f[0][xx]), acc);
      }
  }
  bc[J] = __float2bfloat16_rn(acc);
  xc[J] = 0.f;
}

template <int D, typename TR>
__global__ void __launch_bounds__(kBlock)
k_restrict_q1(int MC, int MF, int dmask, const TR* __restrict__ rf, __nv_bfloat16* __restrict__ bc,
              float* __restrict__ xc) {
  if (D == 1 && threadIdx.y != 0) return;
  const int c0 = (int)(blockIdx.x * 32 + threadIdx.x), c1 = D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0;
  if (c0 >= MC || c1 >= MC) return;
  restrict_q1_node<D, TR>(MC, MF, dmask, rf, bc, xc, c0, c1, D > 2 ? (int)blockIdx.z : 0);
}

// 3D Q1 restriction by 2 x 2 coarse nodes (J0 .. J0+1, K0 .. K0+1 at one I)
// per thread, blocks (32, 8) over I and J0 / 2, blockIdx.z = K0 / 2: when all
// four are interior their 5 x 5 fine rows are summed over x once and shared
// (75 loads for four nodes instead of 108), each node then combined over y
// and z exactly as k_restrict_q1's interior form does; otherwise each node
// takes k_restrict_q1's per-node form
template <typename TR>
__global__ void __launch_bounds__(kBlock)
k_restrict_q1b(int MC, int MF, int dmask, const TR* __restrict__ rf, __nv_bfloat16* __restrict__ bc,
               float* __restrict__ xc) {
  const int I = blockIdx.x * 32 + threadIdx.x, J0 = 2 * (blockIdx.y * 8 + threadIdx.y), K0 = 2 * blockIdx.z;
  if (I >= MC || J0 >= MC) return;
  if (I >= 1 && I <= MC - 2 && J0 >= 1 && J0 + 1 <= MC - 2 && K0 >= 1 && K0 + 1 <= MC - 2) {
    const long long MF2 = (long long)MF * MF;
    const TR* p0 = rf + (2 * I - 1) + (long long)MF * (2 * J0 - 1) + MF2 * (2 * K0 - 1);
    float u[5][5];
#pragma unroll
    for (int z = 0; z < 5; ++z)
#pragma unroll
      for (int y = 0; y < 5; ++y) {
        const TR* q = p0 + (long long)MF * y + MF2 * z;
        u[z][y] = fmaf(.5f, ldv(q, 0) + ldv(q, 2), ldv(q, 1));
      }
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
        float t[3];
#pragma unroll
        for (int z = 0; z < 3; ++z) {
          const float* w = u[2 * dz + z] + 2 * dy;
          t[z] = fmaf(.5f, w[0] + w[2], w[1]);
        }
        const long long J = I + (long long)MC * ((J0 + dy) + (long long)MC * (K0 + dz));
        bc[J] = __float2bfloat16_rn(fmaf(.5f, t[0] + t[2], t[1]));
        xc[J] = 0.f;
      }
    return;
  }
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
      if (J0 + dy < MC && K0 + dz < MC) restrict_q1_node<3, TR>(MC, MF, dmask, rf, bc, xc, I, J0 + dy, K0 + dz);
}

// restriction of a residual (FP32 or BF16) into the coarse rhs (BF16), coarse
// solution zeroed; blocks (32, 8) over x, y and one z plane per blockIdx.z
template <int D, int P, typename TR>
__global__ void __launch_bounds__(kBlock)
k_restrict_mx(int MC, int MF, int dmask, const TR* __restrict__ rf, __nv_bfloat16* __restrict__ bc,
              float* __restrict__ xc) {
  if (D == 1 && threadIdx.y != 0) return;
  const int cJ[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (cJ[0] >= MC || cJ[1] >= MC) return;
  const long long J = cJ[0] + (long long)MC * (cJ[1] + (long long)MC * cJ[2]);
  bool dj = false;
  for (int k = 0; k < D; ++k) dj = dj || fdir(cJ[k], MC, k, dmask);
  float acc = 0.f;
  if (!dj) {
    int off[3][5] = {{0}, {0}, {0}};
    float wt[3][5] = {{1.f}, {1.f}, {1.f}};
    int cnt[3] = {1, 1, 1};
#pragma unroll
    for (int k = 0; k < D; ++k) {
      if (P == 1) { off[k][0] = -1; off[k][1] = 0; off[k][2] = 1; wt[k][0] = .5f; wt[k][1] = 1.f; wt[k][2] = .5f; cnt[k] = 3; }
      else if ((cJ[k] & 1) == 0) {
        const int o[5] = {-3, -1, 0, 1, 3};
        const float ww[5] = {-.125f, .375f, 1.f, .375f, -.125f};
        for (int t = 0; t < 5; ++t) { off[k][t] = o[t]; wt[k][t] = ww[t]; }
        cnt[k] = 5;
      } else { off[k][0] = -1; off[k][1] = 0; off[k][2] = 1; wt[k][0] = .75f; wt[k][1] = 1.f; wt[k][2] = .75f; cnt[k] = 3; }
      // zero the weights of fine nodes outside the grid or on Dirichlet faces
      for (int t = 0; t < cnt[k]; ++t) {
        const int f = 2 * cJ[k] + off[k][t];
        if (f < 0 || f >= MF || fdir(f, MF, k, dmask)) { wt[k][t] = 0.f; off[k][t] = -2 * cJ[k]; }
      }
    }
    for (int z = 0; z < cnt[2]; ++z)
      for (int y = 0; y < cnt[1]; ++y) {
        const long long row = (long long)MF * ((2 * cJ[1] + off[1][y]) + (long long)MF * (2 * cJ[2] + off[2][z]));
        const float wyz = wt[1][y] * wt[2][z];
        for (int xx = 0; xx < cnt[0]; ++xx)
          acc = fmaf(wt[0][xx] * wyz, ldv(rf, row + 2 * cJ[0] + off[0][xx]), acc);
      }
  }
  bc[J] = __float2bfloat16_rn(acc);
  xc[J] = 0.f;
}

// xf += I xc (FP32), same launch shape.  Per direction a fine node has one
// coarse parent (even index) or two (odd); both cases use two slots with the
// second weight zero, so the loops are fixed-size and stay in registers.
template <int D>
__global__ void __launch_bounds__(kBlock)
k_prolong_q1(int MF, int MC, int dmask, const float* __restrict__ xc, float* __restrict__ xf) {
  if (D == 1 && threadIdx.y != 0) return;
  const int fi[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (fi[0] >= MF || fi[1] >= MF) return;
  bool dirf = false;
#pragma unroll
  for (int k = 0; k < D; ++k) dirf = dirf || fdir(fi[k], MF, k, dmask);
  if (dirf) return;
  int J0[3], J1[3];
  float w0[3], w1[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k >= D) { J0[k] = J1[k] = 0; w0[k] = 1.f; w1[k] = 0.f; continue; }
    const int I = fi[k];
    const bool odd = I & 1;
    J0[k] = I >> 1;
    J1[k] = odd ? J0[k] + 1 : J0[k];
    w0[k] = odd ? .5f : 1.f;
    w1[k] = odd ? .5f : 0.f;
    if (fdir(J0[k], MC, k, dmask)) w0[k] = 0.f;
    if (fdir(J1[k], MC, k, dmask)) w1[k] = 0.f;
  }
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = c >> 2;
    const float ww = (bx ? w1[0] : w0[0]) * (by ? w1[1] : w0[1]) * (bz ? w1[2] : w0[2]);
    const long long j = (bx ? J1[0] : J0[0]) + (long long)MC * ((by ? J1[1] : J0[1]) + (long long)MC * (bz ? J1[2] : J0[2]));
    acc = fmaf(ww, __ldg(xc + j), acc);
  }
  const long long i = fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2]);
  xf[i] += acc;
}

// 3D Q1 prolongation by coarse node (xf in layout fl): thread (I, J, K) updates the fine nodes
// (2I+a, 2J+b, 2K+c), a, b, c in {0, 1}, from the 8 coarse values at
// I..I+1, J..J+1, K..K+1, loaded once (coarse Dirichlet values read as
// zero, which is what a zero weight gives there).  Cells whose fine nodes are
// all off the faces interpolate one direction at a time; the others sum each
// fine node with the weights and in the order of k_prolong_q1.
__global__ void __launch_bounds__(kBlock)
k_prolong_q1c(int MF, int MC, int dmask, const float* __restrict__ xc, float* __restrict__ xf, VLay fl) {
  const int I = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y, K = blockIdx.z;
  if (I >= MC || J >= MC) return;
  const long long MC2 = (long long)MC * MC;
  if (I >= 1 && I <= MC - 2 && J >= 1 && J <= MC - 2 && K >= 1 && K <= MC - 2) {
    // the eight fine nodes lie inside and off every face (only the coarse
    // neighbours I + 1, J + 1, K + 1 can sit on a face): interpolate one
    // direction at a time (weights 1 and 1/2, 1/2), read all eight fine
    // values, then write them
    const float* c0 = xc + K * MC2 + (long long)J * MC + I;
    const bool hx = I + 1 < MC - 1 || !(dmask & 2), hy = J + 1 < MC - 1 || !(dmask & 8),
               hz = K + 1 < MC - 1 || !(dmask & 32);
    float e[2][2][2];
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
        const bool ok = (dz == 0 || hz) && (dy == 0 || hy);
        const float* q = c0 + MC2 * dz + (long long)MC * dy;
        const float v0 = ok ? __ldg(q) : 0.f, v1 = ok && hx ? __ldg(q + 1) : 0.f;
        e[dz][dy][0] = v0;
        e[dz][dy][1] = .5f * (v0 + v1);
      }
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int a = 0; a < 2; ++a) e[dz][1][a] = .5f * (e[dz][0][a] + e[dz][1][a]);
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) e[1][b][a] = .5f * (e[0][b][a] + e[1][b][a]);
    float* o = xf + fl.at(2 * I, 2 * J, 2 * K);
    const long long py = fl.py, pz = fl.pz;
    float old[2][2][2];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int a = 0; a < 2; ++a) old[c][b][a] = o[a + py * b + pz * c];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int a = 0; a < 2; ++a) o[a + py * b + pz * c] = old[c][b][a] + e[c][b][a];
    return;
  }
  float v[2][2][2];
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const int ci = I + dx, cj = J + dy, ck = K + dz;
        const bool ok = ci < MC && cj < MC && ck < MC && !fdir(ci, MC, 0, dmask) && !fdir(cj, MC, 1, dmask) &&
                        !fdir(ck, MC, 2, dmask);
        v[dz][dy][dx] = ok ? __ldg(xc + ck * MC2 + (long long)cj * MC + ci) : 0.f;
      }
  // the eight fine values are read before any is written (the compiler
  // cannot tell that the eight layout offsets differ), so their loads overlap
  bool fok[2][2][2];
  long long fo[2][2][2];
  float old[2][2][2];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int fx = 2 * I + a, fy = 2 * J + b, fz = 2 * K + c;
        fok[c][b][a] = fx < MF && fy < MF && fz < MF && !fdir(fx, MF, 0, dmask) && !fdir(fy, MF, 1, dmask) &&
                       !fdir(fz, MF, 2, dmask);
        fo[c][b][a] = fl.at(fx, fy, fz);
        old[c][b][a] = fok[c][b][a] ? xf[fo[c][b][a]] : 0.f;
      }
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const float wz0 = c ? .5f : 1.f, wz1 = c ? .5f : 0.f;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wy0 = b ? .5f : 1.f, wy1 = b ? .5f : 0.f;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        if (!fok[c][b][a]) continue;
        const float wx0 = a ? .5f : 1.f, wx1 = a ? .5f : 0.f;
        float acc = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int bx = q & 1, by = (q >> 1) & 1, bz = q >> 2;
          const float ww = (bx ? wx1 : wx0) * (by ? wy1 : wy0) * (bz ? wz1 : wz0);
          // even fine index: the second coarse node is the first one, weight 0
          acc = fmaf(ww, v[c ? bz : 0][b ? by : 0][a ? bx : 0], acc);
        }
        xf[fo[c][b][a]] = old[c][b][a] + acc;
      }
    }
  }
}

// 3D Q1 prolongation into a padded layout (rows of py = 4k elements, planes
// of pz = py M, the array 16-byte aligned): thread (m, J, K) updates the
// entries at row offsets 4m .. 4m + 3 of the fine rows (2J + b, 2K + c),
// b, c in {0, 1}, one 16-byte load and store per row, all loads before the
// stores; pads, Dirichlet nodes and nodes outside the grid get a zero
// correction.  The four coarse rows (J..J+1, K..K+1) are read on the three
// columns the four fine x need and interpolated over y, z, then x (coarse
// Dirichlet values read as zero).
__global__ void __launch_bounds__(kBlock)
k_prolong_q1v(int MF, int MC, int dmask, const float* __restrict__ xc, float* __restrict__ xf, VLay fl) {
  const unsigned q = (unsigned)fl.py >> 2;
  const unsigned idx = blockIdx.x * kBlock + threadIdx.x;
  if (idx >= q * (unsigned)MC) return;
  const int J = (int)(idx / q), m = (int)(idx - (unsigned)J * q), K = blockIdx.y;
  const int x0 = 4 * m - fl.front;
  const int c0 = x0 >> 1;  // floor(x0 / 2), x0 >= -3
  bool okc[3], oky[2], okz[2];
#pragma unroll
  for (int t = 0; t < 3; ++t) okc[t] = c0 + t >= 0 && c0 + t < MC && !fdir(c0 + t, MC, 0, dmask);
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    oky[d] = J + d < MC && !fdir(J + d, MC, 1, dmask);
    okz[d] = K + d < MC && !fdir(K + d, MC, 2, dmask);
  }
  const long long MC2 = (long long)MC * MC;
  float R[2][2][3];
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const float* row = xc + (K + dz) * MC2 + (long long)(J + dy) * MC + c0;
#pragma unroll
      for (int t = 0; t < 3; ++t) R[dz][dy][t] = okz[dz] && oky[dy] && okc[t] ? __ldg(row + t) : 0.f;
    }
  // over y, then z: R[c][b][t] becomes the value on fine row (2J + b, 2K + c)
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int t = 0; t < 3; ++t) R[dz][1][t] = .5f * (R[dz][0][t] + R[dz][1][t]);
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int t = 0; t < 3; ++t) R[1][b][t] = .5f * (R[0][b][t] + R[1][b][t]);
  bool okx[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) okx[l] = x0 + l >= 0 && x0 + l < MF && !fdir(x0 + l, MF, 0, dmask);
  bool okr[2][2];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int fy = 2 * J + b, fz = 2 * K + c;
      okr[c][b] = fy < MF && fz < MF && !fdir(fy, MF, 1, dmask) && !fdir(fz, MF, 2, dmask);
    }
  float4* o = reinterpret_cast<float4*>(xf + (long long)fl.py * (2 * J) + fl.pz * (2 * K) + 4 * m);
  const long long qy = q, qz = fl.pz >> 2;  // row and plane strides in float4
  float4 v[2][2];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
      if (okr[c][b]) v[c][b] = o[qy * b + qz * c];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (!okr[c][b]) continue;
      const float* r = R[c][b];
      float e[4];
      if (x0 & 1) {  // x0 = 2 c0 + 1
        e[0] = .5f * (r[0] + r[1]); e[1] = r[1]; e[2] = .5f * (r[1] + r[2]); e[3] = r[2];
      } else {
        e[0] = r[0]; e[1] = .5f * (r[0] + r[1]); e[2] = r[1]; e[3] = .5f * (r[1] + r[2]);
      }
      float4 w = v[c][b];
      w.x += okx[0] ? e[0] : 0.f;
      w.y += okx[1] ? e[1] : 0.f;
      w.z += okx[2] ? e[2] : 0.f;
      w.w += okx[3] ? e[3] : 0.f;
      o[qy * b + qz * c] = w;
    }
}

// Q2 (and any order): generic stencil with runtime lengths
template <int D, int P>
__global__ void __launch_bounds__(kBlock)
k_prolong_mx(int MF, int MC, int dmask, const float* __restrict__ xc, float* __restrict__ xf) {
  if (D == 1 && threadIdx.y != 0) return;
  const int fi[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (fi[0] >= MF || fi[1] >= MF) return;
  for (int k = 0; k < D; ++k)
    if (fdir(fi[k], MF, k, dmask)) return;
  const long long i = fi[0] + (long long)MF * (fi[1] + (long long)MF * fi[2]);
  int J[3][3] = {{0}, {0}, {0}};
  float wt[3][3] = {{1.f}, {1.f}, {1.f}};
  int cnt[3] = {1, 1, 1};
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const int I = fi[k];
    if ((I & 1) == 0) { J[k][0] = I / 2; wt[k][0] = 1.f; cnt[k] = 1; }
    else if (P == 1) { J[k][0] = (I - 1) / 2; J[k][1] = (I + 1) / 2; wt[k][0] = wt[k][1] = .5f; cnt[k] = 2; }
    else {
      const int c = I / 4;
      const bool q1 = (I - 4 * c) == 1;
      J[k][0] = 2 * c; J[k][1] = 2 * c + 1; J[k][2] = 2 * c + 2;
      wt[k][0] = q1 ? .375f : -.125f; wt[k][1] = .75f; wt[k][2] = q1 ? -.125f : .375f;
      cnt[k] = 3;
    }
    for (int t = 0; t < cnt[k]; ++t)
      if (fdir(J[k][t], MC, k, dmask)) wt[k][t] = 0.f;
  }
  float acc = 0.f;
  for (int z = 0; z < cnt[2]; ++z)
    for (int y = 0; y < cnt[1]; ++y) {
      const long long row = (long long)MC * (J[1][y] + (long long)MC * J[2][z]);
      const float wyz = wt[1][y] * wt[2][z];
      for (int xx = 0; xx < cnt[0]; ++xx) acc = fmaf(wt[0][xx] * wyz, xc[row + J[0][xx]], acc);
    }
  xf[i] += acc;
}

// coarsest level in FP64: x = A^-1 b (b BF16 -> FP64, x FP32), n <= 1024;
// eight threads per row (each a strided eighth of the columns, then a
// shuffle sum), 128 rows at a time, so the coefficient loads of all rows
// are in flight together
__global__ void __launch_bounds__(1024)
k_coarse_mx(const double* __restrict__ AinvT, int n, const __nv_bfloat16* __restrict__ b, float* __restrict__ x) {
  __shared__ double rs[1024];
  for (int i = threadIdx.x; i < n; i += 1024) rs[i] = (double)__bfloat162float(b[i]);
  __syncthreads();
  const int l8 = threadIdx.x & 7;
  for (int base = (threadIdx.x >> 5) * 4; base < n; base += 128) {  // warp-uniform: rows base .. base+3
    const int i = base + ((threadIdx.x >> 3) & 3);
    double acc = 0.0;
    if (i < n) {
#pragma unroll 4
      for (int j = l8; j < n; j += 8) acc = fma(__ldg(AinvT + (long long)j * n + i), rs[j], acc);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    if (i < n && l8 == 0) x[i] = (float)acc;
  }
}

// ------------------------------------------------------------ vector ops
__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// r32 = r64 / sqrt(sc[s_rr]); e32 = 0
__global__ void k_scale_in(const double* __restrict__ r, const double* __restrict__ sc, int s_rr, float* __restrict__ r32,
                           float* __restrict__ e32, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double inv = 1.0 / sqrt(sc[s_rr]);
  r32[i] = (float)(r[i] * inv);
  e32[i] = 0.f;
}

// x64 += sqrt(sc[s_rr]) * e32
__global__ void k_scale_out(const float* __restrict__ e32, const double* __restrict__ sc, int s_rr, double* __restrict__ x,
                            long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = fma(sqrt(sc[s_rr]), (double)e32[i], x[i]);
}

// FP64 flexible-CG update: x += lam p; r -= lam a; (r, r); and the FP32
// copy of the new residual scaled by the current scale slot; all five in one
// layout (natural or padded), two entries per thread and pass, 16-byte
// accesses; the padding is zero in p and a and stays zero in x and r.  A
// fixed grid of kUpdBlocks blocks strides over the vectors, so the last
// block's sum of the per-block partials is short and the sum's order does
// not depend on the GPU.
constexpr int kUpdBlocks = 1184;  // eight per SM of a B200
__global__ void __launch_bounds__(kBlock)
k_fcg64_update(double* sc, double* __restrict__ x, const float* __restrict__ p, double* __restrict__ r,
               const double* __restrict__ a, float* __restrict__ r32, long long n, Reduce2 R) {
  __shared__ double smem[8];
  const double lam = sc[M_LAM], s = sc[M_SCALE];
  double acc = 0.0;
  const long long stride = (long long)gridDim.x * kBlock * 2;
  for (long long i0 = ((long long)blockIdx.x * kBlock + threadIdx.x) * 2; i0 < n; i0 += stride) {
    // n is the padded length (even); padding entries are zero
    const float2 pf = *reinterpret_cast<const float2*>(p + i0);
    const double2 pv = make_double2((double)pf.x, (double)pf.y);
    const double2 av = *reinterpret_cast<const double2*>(a + i0);
    double2 xv = *reinterpret_cast<double2*>(x + i0);
    double2 rv = *reinterpret_cast<double2*>(r + i0);
    xv.x = fma(lam, pv.x, xv.x); xv.y = fma(lam, pv.y, xv.y);
    rv.x = fma(-lam, av.x, rv.x); rv.y = fma(-lam, av.y, rv.y);
    *reinterpret_cast<double2*>(x + i0) = xv;
    *reinterpret_cast<double2*>(r + i0) = rv;
    *reinterpret_cast<float2*>(r32 + i0) = make_float2((float)(rv.x * s), (float)(rv.y * s));
    acc = fma(rv.x, rv.x, acc);
    acc = fma(rv.y, rv.y, acc);
  }
  dr_finish2(acc, 0.0, R, smem);
}

// p = q / s + beta p  (first: p = q / s), s the scale of the FP32 residual,
// computed in FP64 and stored in FP32: the search direction only has to be
// the same vector in a = A p and in x += lam p, which it is
__global__ void k_fcg64_p(const double* __restrict__ sc, float* __restrict__ p, const float* __restrict__ q,
                          long long n, int first) {
  const long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i0 >= n) return;
  const double inv = sc[M_SINV], beta = sc[M_BETA];  // 1 / scale of the FP32 residual
  if (i0 + 4 <= n && (((uintptr_t)(p + i0) | (uintptr_t)(q + i0)) & 15) == 0) {
    const float4 qv = *reinterpret_cast<const float4*>(q + i0);
    float4 pv = *reinterpret_cast<float4*>(p + i0);
    const double z0 = (double)qv.x * inv, z1 = (double)qv.y * inv, z2 = (double)qv.z * inv, z3 = (double)qv.w * inv;
    pv.x = (float)(first ? z0 : fma(beta, (double)pv.x, z0));
    pv.y = (float)(first ? z1 : fma(beta, (double)pv.y, z1));
    pv.z = (float)(first ? z2 : fma(beta, (double)pv.z, z2));
    pv.w = (float)(first ? z3 : fma(beta, (double)pv.w, z3));
    *reinterpret_cast<float4*>(p + i0) = pv;
  } else {
    for (long long i = i0; i < n && i < i0 + 4; ++i) {
      const double z = (double)q[i] * inv;
      p[i] = (float)(first ? z : fma(beta, (double)p[i], z));
    }
  }
}

__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

// r32 = r * sc[slot]
__global__ void k_scale_to32(const double* __restrict__ r, const double* __restrict__ sc, int slot,
                             float* __restrict__ r32, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r32[i] = (float)(r[i] * sc[slot]);
}

// two FP64 dot products (x, y) and (x, y2) with the epilogue of R
__global__ void __launch_bounds__(kBlock)
k_dot2_64(const double* __restrict__ xv, const float* __restrict__ yv, const double* __restrict__ y2,
          long long n, Reduce2 R) {
  __shared__ double smem[8];
  const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
  double a0 = 0.0, a1 = 0.0;
  if (i < n) {
    a0 = xv[i] * (double)yv[i];
    if (y2) a1 = xv[i] * y2[i];
  }
  dr_finish2(a0, a1, R, smem);
}

// ---------------------------------------------------------- dispatchers
#define MX_DISPATCH(D_, P_, ...)                                              \
  do {                                                                        \
    if ((D_) == 1 && (P_) == 1) { constexpr int D = 1, P = 1; __VA_ARGS__; }  \
    else if ((D_) == 2 && (P_) == 1) { constexpr int D = 2, P = 1; __VA_ARGS__; } \
    else if ((D_) == 3 && (P_) == 1) { constexpr int D = 3, P = 1; __VA_ARGS__; } \
    else if ((D_) == 1 && (P_) == 2) { constexpr int D = 1, P = 2; __VA_ARGS__; } \
    else if ((D_) == 2 && (P_) == 2) { constexpr int D = 2, P = 2; __VA_ARGS__; } \
    else { constexpr int D = 3, P = 2; __VA_ARGS__; }                         \
  } while (0)

static inline unsigned g1(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// the tiled box (whole 32 x 16 x 32 tiles from the origin) and the nodes left
// to the face CTAs: outside the box, and its Dirichlet faces x, y, z = 0
static MftGeo mft_geo(int M, int dmask) {
  MftGeo q{};
  const int n = M - 1;
  q.nbx = n / kFX;
  q.nby = n / kFY;
  q.nbz = n / kFZ;
  if (q.nbx == 0 || q.nby == 0 || q.nbz == 0) q.nbx = q.nby = q.nbz = 0;
  q.nmain = q.nbx * q.nby * q.nbz;
  q.X1 = (long long)q.nbx * kFX;
  q.Y1 = (long long)q.nby * kFY;
  q.Z1 = (long long)q.nbz * kFZ;
  if (q.nmain > 0) {
    q.ax = (dmask & 1) ? 1 : 0;
    q.ay = (dmask & 4) ? 1 : 0;
    q.az = (dmask & 16) ? 1 : 0;
  }
  q.F = (long long)M * M * M - (q.X1 - q.ax) * (q.Y1 - q.ay) * (q.Z1 - q.az);
  q.nface = (int)((q.F + kFaceNodes - 1) / kFaceNodes);
  return q;
}

static unsigned mft_blocks(const MftGeo& q) { return (unsigned)(q.nmain + q.nface); }

static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

template <typename E>
static CUtensorMapDataType tm_type() {
  return sizeof(E) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
}

// the cells as n x n x n, boxes of one plane's cell tile; cells outside
// read as zero
template <typename T>
static bool cell_map(const T* k, int n, CUtensorMap* tk) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return false;
  const cuuint32_t one[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides[2] = {(cuuint64_t)n * sizeof(T), (cuuint64_t)n * n * sizeof(T)};
  const cuuint32_t box[3] = {(cuuint32_t)CellBox<T>::CW, (cuuint32_t)kFCRows, 1};
  return enc(tk, tm_type<T>(), 3, const_cast<T*>(k), dims, strides, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

VLay natural_lay(int M, int dim) {
  VLay L;
  L.front = 0;
  L.py = M;
  L.pz = (long long)M * M;
  L.total = dim == 3 ? L.pz * M : (dim == 2 ? L.pz : M);
  return L;
}

VLay padded_lay(int M, int dmask) {
  VLay L;
  L.front = (4 - (dmask & 1)) & 3;
  L.py = (L.front + M + 3) / 4 * 4;
  L.pz = (long long)L.py * M;
  L.total = L.pz * M;
  return L;
}

// an FP32 x in layout L as the halo source: the nodes off the Dirichlet
// faces, boxes of 40 x 18 from a 16-byte boundary (the map's origin, node
// (l_x, l_y, l_z), sits on one by the choice of front)
static bool halo_map(const float* x, const VLay& L, int M, int dmask, CUtensorMap* tm) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return false;
  const int lo[3] = {dmask & 1, (dmask >> 2) & 1, (dmask >> 4) & 1};
  const int hi[3] = {(dmask >> 1) & 1, (dmask >> 3) & 1, (dmask >> 5) & 1};
  const float* base = x + L.at(lo[0], lo[1], lo[2]);
  if (((uintptr_t)base & 15) || ((L.py * 4) & 15) || ((L.pz * 4) & 15)) return false;
  const cuuint32_t one[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {(cuuint64_t)(M - lo[0] - hi[0]), (cuuint64_t)(M - lo[1] - hi[1]),
                              (cuuint64_t)(M - lo[2] - hi[2])};
  const cuuint64_t strides[2] = {(cuuint64_t)L.py * 4, (cuuint64_t)L.pz * 4};
  const cuuint32_t box[3] = {(cuuint32_t)kXW, (cuuint32_t)kFRows, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, one,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// a per-node operand in layout L: the whole padded array (py x M x M),
// boxes of 36 x 16 from tensor x0 (node x0 - front)
template <typename E>
static bool op_map(const E* p, const VLay& L, int M, CUtensorMap* tm) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return false;
  if (((uintptr_t)p & 15) || ((L.py * sizeof(E)) & 15) || ((L.pz * sizeof(E)) & 15)) return false;
  const cuuint32_t one[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {(cuuint64_t)L.py, (cuuint64_t)M, (cuuint64_t)M};
  const cuuint64_t strides[2] = {(cuuint64_t)L.py * sizeof(E), (cuuint64_t)L.pz * sizeof(E)};
  const cuuint32_t box[3] = {(cuuint32_t)kOW, (cuuint32_t)kFY, 1};
  return enc(tm, tm_type<E>(), 3, const_cast<E*>(p), dims, strides, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, typename TV, typename TX, int MODE, bool RED>
static void mft_launch(const MFArgsT<T>& g, const TX* x, const T* b, T* y, const TV* v, const TV* v2,
                       const Reduce2& R, cudaStream_t st) {
  typedef MfcLayout<T, TV, TX, MODE, RED> L;
  MftGeo q = mft_geo(g.M, g.dmask);
  CUtensorMap tk{}, tx{}, tb{}, to{}, tv{}, tv2{};
  // every map needs a 16-byte aligned base and pitch, the operand boxes the
  // operand layout's front at most 4; without them every node goes to the
  // face CTAs
  const T* om = g.wd ? g.wd : g.omega;
  constexpr bool HO = MODE == 2 || MODE == 3;
  bool maps = q.nmain > 0 && cell_map<T>(g.k, g.n, &tk);
  if (maps && L::HX && L::XT) maps = halo_map(reinterpret_cast<const float*>(x), g.xl, g.M, g.dmask, &tx);
  if (maps && L::OT) {
    maps = g.ol.front <= 4 && (!L::HB || op_map<T>(b, g.ol, g.M, &tb)) &&
           (!(HO && om) || (g.wd && op_map<T>(g.wd, g.ol, g.M, &to))) && (!L::HV || op_map<TV>(v, g.ol, g.M, &tv)) &&
           (!(L::HV && v2) || op_map<TV>(v2, g.ol, g.M, &tv2));
  }
  if (!maps) {
    q = MftGeo{};
    q.F = g.N;
    q.nface = (int)((q.F + kFaceNodes - 1) / kFaceNodes);
  }
  int dev = 0;
  cudaGetDevice(&dev);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const int opt = (HO && (g.wd || g.omega) ? 1 : 0) | (RED && v2 ? 2 : 0) | (HO && g.wd ? 4 : 0);
  auto go = [&](auto oc) {
    constexpr int OPT = decltype(oc)::value;
    auto kern = k_mfc<T, TV, TX, MODE, RED, OPT>;
    constexpr int smem = L::SMEM;
    static unsigned attr = 0;  // devices the shared-memory size was raised on
    if (dev < 32 && !((attr >> dev) & 1u)) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      attr |= 1u << dev;
    }
    kern<<<mft_blocks(q), kFThreads, smem, st>>>(g, tk, tx, tb, to, tv, tv2, q, x, b, y, v, v2, R);
  };
  switch (opt) {
    case 1: if constexpr (HO) go(std::integral_constant<int, 1>{}); break;
    case 2: if constexpr (RED) go(std::integral_constant<int, 2>{}); break;
    case 3: if constexpr (HO && RED) go(std::integral_constant<int, 3>{}); break;
    case 5: if constexpr (HO) go(std::integral_constant<int, 5>{}); break;
    case 7: if constexpr (HO && RED) go(std::integral_constant<int, 7>{}); break;
    default: go(std::integral_constant<int, 0>{});
  }
}

template <typename T, typename TV, typename TX>
static void mf_launch(int mode, const MFArgsT<T>& g, const TX* x, const T* b, T* y, const TV* v, const TV* v2,
                      const Reduce2* R, cudaStream_t st) {
  const Reduce2 r0 = R ? *R : Reduce2{};
  if constexpr (sizeof(T) == 8) {  // the FP64 operator: a = A p, or the true residual of FP64 vectors
    if (mode == 1) mft_launch<T, TV, TX, 1, false>(g, x, b, y, v, v2, r0, st);
    else if (R) mft_launch<T, TV, TX, 0, true>(g, x, b, y, v, v2, r0, st);
    else mft_launch<T, TV, TX, 0, false>(g, x, b, y, v, v2, r0, st);
  } else if (R) {
    switch (mode) {
      case 0: mft_launch<T, TV, TX, 0, true>(g, x, b, y, v, v2, r0, st); break;
      case 1: mft_launch<T, TV, TX, 1, true>(g, x, b, y, v, v2, r0, st); break;
      case 2: mft_launch<T, TV, TX, 2, true>(g, x, b, y, v, v2, r0, st); break;
      default: mft_launch<T, TV, TX, 3, true>(g, x, b, y, v, v2, r0, st);
    }
  } else {
    switch (mode) {
      case 0: mft_launch<T, TV, TX, 0, false>(g, x, b, y, v, v2, r0, st); break;
      case 1: mft_launch<T, TV, TX, 1, false>(g, x, b, y, v, v2, r0, st); break;
      case 2: mft_launch<T, TV, TX, 2, false>(g, x, b, y, v, v2, r0, st); break;
      default: mft_launch<T, TV, TX, 3, false>(g, x, b, y, v, v2, r0, st);
    }
  }
}

// pre-smoothing from zero with the damping over the diagonal formed: y = wd b,
// four nodes per thread (16-byte accesses when all three vectors allow them)
__global__ void __launch_bounds__(kBlock) k_wd_scale(const float* __restrict__ wd, const float* __restrict__ b,
                                                     float* __restrict__ y, long long n) {
  const long long i0 = ((long long)blockIdx.x * kBlock + threadIdx.x) * 4;
  if (i0 >= n) return;
  if (i0 + 4 <= n && (((uintptr_t)wd | (uintptr_t)b | (uintptr_t)y) & 15) == 0) {
    const float4 w = __ldg(reinterpret_cast<const float4*>(wd + i0));
    const float4 v = __ldg(reinterpret_cast<const float4*>(b + i0));
    *reinterpret_cast<float4*>(y + i0) = make_float4(w.x * v.x, w.y * v.y, w.z * v.z, w.w * v.w);
  } else {
    for (long long i = i0; i < n && i < i0 + 4; ++i) y[i] = __ldg(wd + i) * __ldg(b + i);
  }
}

// kernels over every node of an M^3 grid launched as dim3(g1(M^2), M): node
// (ix, iy) of plane blockIdx.y with one 32-bit division (M^2 < 2^32), i its
// natural index
__device__ __forceinline__ bool plane_node(int M, int& ix, int& iy, int& iz, long long& i) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x, mu = (unsigned)M;
  if (q >= mu * mu) return false;
  iy = (int)(q / mu);
  ix = (int)(q - (unsigned)iy * mu);
  iz = (int)blockIdx.y;
  i = (long long)iz * ((long long)M * M) + q;
  return true;
}

// wd (layout g.ol) = damping / diagonal of the matrix-free top level, the diagonal formed
// as in the matrix-free operator (4 hs times the sum of the node's 8 cell coefficients, summed
// in the same order; cells outside the grid count zero); Dirichlet nodes
// (identity rows) get the damping itself
__global__ void __launch_bounds__(kBlock) k_mf_wd(MFArgs g, float* __restrict__ wd) {
  const int M = g.M, n = g.n, dm = g.dmask;
  int ix, iy, iz;
  long long i;
  if (!plane_node(M, ix, iy, iz, i)) return;
  auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
  const float om = g.omega ? __ldg(g.omega + i) : g.w;
  const long long o = g.ol.at(ix, iy, iz);
  if (dirf(ix, 1, 2) || dirf(iy, 4, 8) || dirf(iz, 16, 32)) {
    wd[o] = om;
    return;
  }
  float k[2][2][2];
  if (ix >= 1 && ix <= n - 1 && iy >= 1 && iy <= n - 1 && iz >= 1 && iz <= n - 1) {
    // interior node: its 8 cells exist, one base address and fixed strides
    const long long nn = (long long)n * n;
    const float* c0 = g.k + (ix - 1) + (long long)n * (iy - 1) + nn * (iz - 1);
#pragma unroll
    for (int cz = 0; cz < 2; ++cz)
#pragma unroll
      for (int cy = 0; cy < 2; ++cy)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) k[cz][cy][cx] = __ldg(c0 + cx + (long long)n * cy + nn * cz);
  } else {
#pragma unroll
    for (int cz = 0; cz < 2; ++cz)
#pragma unroll
      for (int cy = 0; cy < 2; ++cy)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int x = ix - 1 + cx, y = iy - 1 + cy, z = iz - 1 + cz;
          const bool in = x >= 0 && x < n && y >= 0 && y < n && z >= 0 && z < n;
          k[cz][cy][cx] = in ? __ldg(g.k + x + (long long)n * (y + (long long)n * z)) : 0.f;
        }
  }
  const float wc[2][2] = {{k[0][0][0] + k[1][0][0], k[0][0][1] + k[1][0][1]},
                          {k[0][1][0] + k[1][1][0], k[0][1][1] + k[1][1][1]}};
  const float ksum = (wc[0][0] + wc[0][1]) + (wc[1][0] + wc[1][1]);
  wd[o] = om / (4.f * g.hs * ksum);
}

void mx_top_wd(const MFArgs& g, float* wd, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_mf_wd<<<dim3(g1((long long)g.M * g.M), (unsigned)g.M), kBlock, 0, st>>>(g, wd);
}

void mx_top_apply(int mode, const MFArgs& g, const float* x, const float* b, float* y, const double* v,
                  const double* v2, const Reduce2* R, cudaStream_t st) {
  if (mode == 3 && g.wd && !R) {  // a stream of two reads and a write over the arrays (padding included)
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const long long n = g.ol.total;
    k_wd_scale<<<g1((n + 3) / 4), kBlock, 0, st>>>(g.wd, b, y, n);
    return;
  }
  mf_launch<float, double, float>(mode, g, x, b, y, v, v2, R, st);
}

void mx_top_apply64(const MFArgs64& g, const float* x, double* y, const float* v, const Reduce2* R,
                    cudaStream_t st) {
  mf_launch<double, float, float>(0, g, x, nullptr, y, v, nullptr, R, st);
}

void mx_top_apply64x(const MFArgs64& g, const double* x, double* y, cudaStream_t st) {
  mf_launch<double, double, double>(0, g, x, nullptr, y, nullptr, nullptr, nullptr, st);
}

void mx_top_residual64(const MFArgs64& g, const double* x, const double* b, double* r, cudaStream_t st) {
  mf_launch<double, double, double>(1, g, x, b, r, nullptr, nullptr, nullptr, st);
}

long long mx_top_blocks(int M) { return mft_blocks(mft_geo(M, 63)); }  // the most face CTAs any mask gives

// levels from this many rows on take four rows per thread
constexpr long long kSt32Wide = 1ll << 20;

template <int D, int P, int MODE, typename TB, typename TY, bool RED>
void st32_launch(const Lev32& L, const float* x, const void* b, void* y, const double* v, const double* v2,
                 const Reduce2& r0, cudaStream_t st) {
  constexpr int W = (D == 3 && P == 2) ? 1 : 4;
  if (W == 4 && L.N >= kSt32Wide)
    k_st32<D, P, MODE, TB, TY, RED, W><<<g1((L.N + W - 1) / W), kBlock, 0, st>>>(
        L.A, L.N, L.Np, L.M, L.w, L.om, x, (const TB*)b, (TY*)y, v, v2, r0);
  else
    k_st32<D, P, MODE, TB, TY, RED, 1><<<g1(L.N), kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x,
                                                                    (const TB*)b, (TY*)y, v, v2, r0);
}

void mx_level_apply(int mode, const Lev32& L, const float* x, const void* b, bool b_bf16, void* y, bool y_bf16,
                    const double* v, const double* v2, const Reduce2* R, cudaStream_t st) {
  Reduce2 r0 = R ? *R : Reduce2{};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  typedef __nv_bfloat16 bf;
  MX_DISPATCH(L.dim, L.order, {
    if (R) {  // reductions only on FP32 vectors
      if (mode == 0) st32_launch<D, P, 0, float, float, true>(L, x, b, y, v, v2, r0, st);
      else if (mode == 2) st32_launch<D, P, 2, float, float, true>(L, x, b, y, v, v2, r0, st);
      else st32_launch<D, P, 1, float, float, true>(L, x, b, y, v, v2, r0, st);
    } else if (mode == 0) {
      st32_launch<D, P, 0, float, float, false>(L, x, b, y, v, v2, r0, st);
    } else if (mode == 1) {
      if (b_bf16 && y_bf16) st32_launch<D, P, 1, bf, bf, false>(L, x, b, y, v, v2, r0, st);
      else if (b_bf16) st32_launch<D, P, 1, bf, float, false>(L, x, b, y, v, v2, r0, st);
      else if (y_bf16) st32_launch<D, P, 1, float, bf, false>(L, x, b, y, v, v2, r0, st);
      else st32_launch<D, P, 1, float, float, false>(L, x, b, y, v, v2, r0, st);
    } else if (mode == 2) {
      if (b_bf16) st32_launch<D, P, 2, bf, float, false>(L, x, b, y, v, v2, r0, st);
      else st32_launch<D, P, 2, float, float, false>(L, x, b, y, v, v2, r0, st);
    } else {
      if (b_bf16) st32_launch<D, P, 3, bf, float, false>(L, x, b, y, v, v2, r0, st);
      else st32_launch<D, P, 3, float, float, false>(L, x, b, y, v, v2, r0, st);
    }
  });
}

static inline dim3 xgrid(long long M, int dim) {
  return dim3((unsigned)((M + 31) / 32), (unsigned)(dim > 1 ? (M + 7) / 8 : 1), (unsigned)(dim > 2 ? M : 1));
}

void mx_restrict(const Lev32& F, const Lev32& C, const void* rf, bool rf_bf16, __nv_bfloat16* bc, float* xc,
                 cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const dim3 gr = xgrid(C.M, F.dim), bl(32, 8);
  if (F.order == 1) {
    typedef __nv_bfloat16 bf;
    if (F.dim == 3 && C.N >= (1ll << 20)) {  // large levels: 2 x 2 coarse nodes per thread
      const dim3 g2((unsigned)((C.M + 31) / 32), (unsigned)((C.M + 15) / 16), (unsigned)((C.M + 1) / 2));
      if (rf_bf16) k_restrict_q1b<bf><<<g2, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const bf*)rf, bc, xc);
      else k_restrict_q1b<float><<<g2, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const float*)rf, bc, xc);
    } else if (F.dim == 3) {  // small levels are latency-bound: one coarse node per thread
      if (rf_bf16) k_restrict_q1<3, bf><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const bf*)rf, bc, xc);
      else k_restrict_q1<3, float><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const float*)rf, bc, xc);
    } else if (F.dim == 2) {
      if (rf_bf16) k_restrict_q1<2, bf><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const bf*)rf, bc, xc);
      else k_restrict_q1<2, float><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const float*)rf, bc, xc);
    } else {
      if (rf_bf16) k_restrict_q1<1, bf><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const bf*)rf, bc, xc);
      else k_restrict_q1<1, float><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const float*)rf, bc, xc);
    }
    return;
  }
  MX_DISPATCH(F.dim, F.order, {
    if (rf_bf16) k_restrict_mx<D, P, __nv_bfloat16><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const __nv_bfloat16*)rf, bc, xc);
    else k_restrict_mx<D, P, float><<<gr, bl, 0, st>>>((int)C.M, (int)F.M, F.dmask, (const float*)rf, bc, xc);
  });
}

void mx_prolong(const Lev32& C, const Lev32& F, const float* xc, float* xf, cudaStream_t st, const VLay* xfl) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const dim3 gr = xgrid(F.M, F.dim), bl(32, 8);
  if (F.order == 1) {
    if (F.dim == 3 && xfl && xfl->py % 4 == 0 && xfl->pz % 4 == 0 && ((uintptr_t)xf & 15) == 0)
      k_prolong_q1v<<<dim3((unsigned)((xfl->py / 4 * C.M + kBlock - 1) / kBlock), (unsigned)C.M), kBlock, 0, st>>>(
          (int)F.M, (int)C.M, F.dmask, xc, xf, *xfl);
    else if (F.dim == 3)
      k_prolong_q1c<<<dim3((unsigned)((C.M + 31) / 32), (unsigned)((C.M + 7) / 8), (unsigned)C.M), bl, 0, st>>>(
          (int)F.M, (int)C.M, F.dmask, xc, xf, xfl ? *xfl : natural_lay((int)F.M, 3));
    else if (F.dim == 2) k_prolong_q1<2><<<gr, bl, 0, st>>>((int)F.M, (int)C.M, F.dmask, xc, xf);
    else k_prolong_q1<1><<<gr, bl, 0, st>>>((int)F.M, (int)C.M, F.dmask, xc, xf);
    return;
  }
  MX_DISPATCH(F.dim, F.order, { k_prolong_mx<D, P><<<gr, bl, 0, st>>>((int)F.M, (int)C.M, F.dmask, xc, xf); });
}

void mx_coarse(const double* AinvT, int n, const __nv_bfloat16* b, float* x, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_coarse_mx<<<1, 1024, 0, st>>>(AinvT, n, b, x);
}

void mx_f64_to_f32(const double* a, float* b, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_f64_to_f32<<<g1(n), kBlock, 0, st>>>(a, b, n);
}

void mx_fcg64_update(double* sc, double* x, const float* p, double* r, const double* a, float* r32, long long np,
                     const Reduce2& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const long long nb = std::min<long long>(g1(np / 2), kUpdBlocks);
  k_fcg64_update<<<(unsigned)std::max<long long>(nb, 1), kBlock, 0, st>>>(sc, x, p, r, a, r32, np, R);
}

// b (layout bl) = a (natural), 3D, M nodes a side: FP64 to FP32, and FP64
// copied (grids of plane_node)

__global__ void k_f64_to_f32_lay(const double* __restrict__ a, float* __restrict__ b, VLay bl, int M) {
  int ix, iy, iz;
  long long i;
  if (!plane_node(M, ix, iy, iz, i)) return;
  b[bl.at(ix, iy, iz)] = (float)a[i];
}

__global__ void k_f64_copy_lay(const double* __restrict__ a, double* __restrict__ b, VLay bl, int M) {
  int ix, iy, iz;
  long long i;
  if (!plane_node(M, ix, iy, iz, i)) return;
  b[bl.at(ix, iy, iz)] = a[i];
}

// b (natural) = a (layout al), FP64, 3D
__global__ void k_f64_from_lay(const double* __restrict__ a, VLay al, double* __restrict__ b, int M) {
  int ix, iy, iz;
  long long i;
  if (!plane_node(M, ix, iy, iz, i)) return;
  b[i] = a[al.at(ix, iy, iz)];
}

void mx_f64_from_lay(const double* a, const VLay& al, double* b, int M, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_f64_from_lay<<<dim3(g1((long long)M * M), (unsigned)M), kBlock, 0, st>>>(a, al, b, M);
}

void mx_f64_to_f32_lay(const double* a, float* b, const VLay& bl, int M, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_f64_to_f32_lay<<<dim3(g1((long long)M * M), (unsigned)M), kBlock, 0, st>>>(a, b, bl, M);
}

void mx_f64_copy_lay(const double* a, double* b, const VLay& bl, int M, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_f64_copy_lay<<<dim3(g1((long long)M * M), (unsigned)M), kBlock, 0, st>>>(a, b, bl, M);
}

void mx_f32_to_f64(const float* a, double* b, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_f32_to_f64<<<g1(n), kBlock, 0, st>>>(a, b, n);
}

void mx_fcg64_p(const double* sc, float* p, const float* q, long long n, bool first, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fcg64_p<<<g1((n + 3) / 4), kBlock, 0, st>>>(sc, p, q, n, first ? 1 : 0);
}

void mx_scale_to32(const double* r, const double* sc, int slot, float* r32, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_scale_to32<<<g1(n), kBlock, 0, st>>>(r, sc, slot, r32, n);
}

void mx_dot2_64(const double* x, const float* y, const double* y2, long long n, const Reduce2& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dot2_64<<<g1(n), kBlock, 0, st>>>(x, y, y2, n, R);
}

}  // namespace fmg
