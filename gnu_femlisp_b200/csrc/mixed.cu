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
#include <cuda_bf16.h>

#include "fmgpu_mixed.cuh"

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
// The reductions of the z-marching kernels run over a 3D grid of blocks.
__device__ __forceinline__ void dr_finish2_grid(double v0, double v1, const Reduce2& R, double* smem) {
  __shared__ bool is_last;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  double s0 = dr_fold256(v0, smem);
  double s1 = dr_fold256(v1, smem);
  if (threadIdx.x + threadIdx.y == 0) {
    R.part[2 * bid] = s0;
    R.part[2 * bid + 1] = s1;
    __threadfence();
    unsigned done = atomicAdd(R.counter, 1u);
    is_last = (done == nb - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  const unsigned t = threadIdx.x + blockDim.x * threadIdx.y;
  double a0 = 0.0, a1 = 0.0;
  for (unsigned k = t; k < nb; k += kBlock) {
    a0 = a0 + __ldcg(R.part + 2 * k);
    a1 = a1 + __ldcg(R.part + 2 * k + 1);
  }
  double t0 = dr_fold256(a0, smem);
  double t1 = dr_fold256(a1, smem);
  if (t == 0) {
    epi2_apply(R, t0, t1);
    *R.counter = 0u;
  }
}

// Matrix-free top-level operator, 2.5D blocking: a CTA owns a 32 x 16 column
// of nodes (256 threads, thread (lx, ly) computes the y-adjacent nodes 2ly and
// 2ly+1) and marches z through ZS planes.  The (32+2) x (16+2) halo of each x
// plane and the 33 x 17 cells of each cell plane are copied into a 5-stage
// shared-memory ring by cp.async (4/8-byte copies, masked entries zero-filled:
// Dirichlet nodes and nodes outside the grid read as zero -- eliminated
// columns -- and cells outside the grid as zero coefficient), two stages ahead
// of the plane being computed.  Stage s holds x plane s+1 and cell plane s;
// plane iz reads the x planes of stages iz-2 .. iz and the cell planes of
// stages iz-1, iz.  The per-node operands (b, omega, v, v2) are register-
// prefetched one plane ahead, and ring slots advance by increments.  The row
// is evaluated in factored form: 4 K x_i minus, over the 12 face diagonals,
// the sum of the two cells sharing each times its value, minus, over the 8
// body diagonals, the one cell times its value (axis neighbours have weight
// zero in the Q1 stiffness).
constexpr int kMX = 32;                            // nodes along x of a CTA
constexpr int kHX = kMX + 2, kCX = kMX + 1;        // halo / cell tile along x
constexpr int kMFThreads = 256;
constexpr int kStages = 5;

__device__ __forceinline__ void cpa(void* dst, const void* src, bool ok, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int kMY4 = 16;
constexpr int kHY4 = kMY4 + 2, kCY4 = kMY4 + 1;
constexpr int kNH4 = kHX * kHY4, kNC4 = kCX * kCY4;  // 612, 561

template <typename T, typename TV, typename TX, int ZS, int MODE, bool RED>
__global__ void __launch_bounds__(kMFThreads)
k_mf4(MFArgsT<T> g, const TX* __restrict__ x, const T* __restrict__ b, T* __restrict__ y,
      const TV* __restrict__ v, const TV* __restrict__ v2, Reduce2 R) {
  constexpr bool HX = MODE != 3;
  constexpr bool HB = MODE != 0;
  constexpr bool DIFF = sizeof(T) == 8;  // the FP64 operator in difference form
  constexpr bool HO = MODE == 2 || MODE == 3;
  __shared__ TX xs[kStages][HX ? kNH4 : 1];
  __shared__ T ks[kStages][kNC4];
  __shared__ double smem[8];
  const int tid = threadIdx.x, lx = tid & (kMX - 1), ly = tid / kMX;
  const int x0 = blockIdx.x * kMX, y0 = blockIdx.y * kMY4, z0 = blockIdx.z * ZS;
  const int M = g.M, n = g.n, dm = g.dmask;
  const long long MM = (long long)M * M, nn = (long long)n * n;
  const int ix = x0 + lx, iy0 = y0 + 2 * ly;
  auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
  int hoff[3], coff[3];
  bool hok[3], cok[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int e = tid + q * kMFThreads;
    const int jx = x0 - 1 + e % kHX, jy = y0 - 1 + e / kHX;
    hok[q] = e < kNH4 && jx >= 0 && jx < M && jy >= 0 && jy < M && !dirf(jx, 1, 2) && !dirf(jy, 4, 8);
    hoff[q] = hok[q] ? jy * M + jx : 0;
    const int cx = x0 - 1 + e % kCX, cy = y0 - 1 + e / kCX;
    cok[q] = e < kNC4 && cx >= 0 && cx < n && cy >= 0 && cy < n;
    coff[q] = cok[q] ? cy * n + cx : 0;
  }
  const bool own0 = ix < M && iy0 < M, own1 = ix < M && iy0 + 1 < M;
  const long long col0 = own0 ? (long long)iy0 * M + ix : 0;
  const long long col1 = own1 ? (long long)(iy0 + 1) * M + ix : 0;
  const bool omv = g.omega != nullptr;
  const int zend = min(z0 + ZS, M);
  auto issue = [&](int st, int sl) {  // x plane st+1 and cell plane st into slot sl
    if (HX) {
      const int jz = st + 1;
      const bool vz = jz >= 0 && jz < M && !dirf(jz, 16, 32);
      const TX* pl = x + (long long)(vz ? jz : 0) * MM;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int e = tid + q * kMFThreads;
        if (e < kNH4) cpa(&xs[sl][e], pl + hoff[q], vz && hok[q], (int)sizeof(TX));
      }
    }
    const bool vz = st >= 0 && st < n;
    const T* pl = g.k + (long long)(vz ? st : 0) * nn;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = tid + q * kMFThreads;
      if (e < kNC4) cpa(&ks[sl][e], pl + coff[q], vz && cok[q], (int)sizeof(T));
    }
    cpa_commit();
  };
  struct Ops { T b[2], o[2]; TV v[2], v2[2]; };
  auto ldops = [&](int jz, Ops& o) {  // per-node operands of a plane (two nodes)
    const bool in = jz < zend;
    const long long zb = (long long)jz * MM;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const bool ok = in && (r ? own1 : own0);
      const long long i = zb + (r ? col1 : col0);
      o.b[r] = (HB && ok) ? __ldg(b + i) : T(0);
      o.o[r] = (HO && g.wd && ok) ? __ldg(g.wd + i) : ((HO && omv && ok) ? __ldg(g.omega + i) : g.w);
      o.v[r] = (RED && ok) ? __ldg(v + i) : TV(0);
      o.v2[r] = (RED && ok && v2) ? __ldg(v2 + i) : TV(0);
    }
  };
  issue(z0 - 2, 0);
  issue(z0 - 1, 1);
  issue(z0, 2);
  issue(z0 + 1, 3);
  int s2 = 0, s1 = 1, s0 = 2, si = 4;  // slots of stages iz-2, iz-1, iz and of the next issue
  Ops cur, nxt;
  ldops(z0, cur);
  double acc0 = 0.0, acc1 = 0.0;
  const bool dirx = dirf(ix, 1, 2);
  const T hs = g.hs;
#pragma unroll 1
  for (int iz = z0; iz < zend; ++iz) {
    issue(iz + 2, si);
    ldops(iz + 1, nxt);
    cpa_wait<2>();
    __syncthreads();
    const bool dirz = dirf(iz, 16, 32);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (!(r ? own1 : own0)) continue;
      const int iy = iy0 + r;
      const long long i = (long long)iz * MM + (r ? col1 : col0);
      const bool dir = dirz || dirx || dirf(iy, 4, 8);
      T ax = T(0), d = T(1), xc = T(0);
      if (dir) {
        if (HX) { xc = (T)x[i]; ax = xc; }
      } else {
        T k[2][2][2];  // k[cz][cy][cx]: cz 0 cell plane iz-1 (slot s1), 1 cell plane iz (slot s0)
#pragma unroll
        for (int cz = 0; cz < 2; ++cz)
#pragma unroll
          for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cx = 0; cx < 2; ++cx) k[cz][cy][cx] = ks[cz ? s0 : s1][(2 * ly + r + cy) * kCX + lx + cx];
        const T wc[2][2] = {{k[0][0][0] + k[1][0][0], k[0][0][1] + k[1][0][1]},
                            {k[0][1][0] + k[1][1][0], k[0][1][1] + k[1][1][1]}};
        const T ksum = (wc[0][0] + wc[0][1]) + (wc[1][0] + wc[1][1]);
        T sacc = T(0);
        if (HX) {
          const int h = (2 * ly + r + 1) * kHX + lx + 1;
          const TX* X1 = xs[s1];  // x plane iz
          xc = (T)X1[h];
          // FP64: the row as sum_j w_j (x_i - x_j) -- the weights sum to 4 K,
          // and the differences of a smooth iterate are small, so the true
          // residual's rounding is far below that of 4 K x_i - sum_j w_j x_j
          auto term = [&](T w, T xj) { sacc = DIFF ? fma(w, xc - xj, sacc) : fma(w, xj, sacc); };
#pragma unroll
          for (int sy = 0; sy < 2; ++sy)
#pragma unroll
            for (int sx = 0; sx < 2; ++sx) term(wc[sy][sx], (T)X1[h + (2 * sy - 1) * kHX + 2 * sx - 1]);
#pragma unroll
          for (int cz = 0; cz < 2; ++cz) {
            const TX* Xz = xs[cz ? s0 : s2];  // x plane iz+1 / iz-1
#pragma unroll
            for (int sx = 0; sx < 2; ++sx)   // face diagonals (sx, 0, sz): cells (sx, *, sz)
              term(k[cz][0][sx] + k[cz][1][sx], (T)Xz[h + 2 * sx - 1]);
#pragma unroll
            for (int sy = 0; sy < 2; ++sy)   // face diagonals (0, sy, sz): cells (*, sy, sz)
              term(k[cz][sy][0] + k[cz][sy][1], (T)Xz[h + (2 * sy - 1) * kHX]);
#pragma unroll
            for (int sy = 0; sy < 2; ++sy)
#pragma unroll
              for (int sx = 0; sx < 2; ++sx)  // body diagonals
                term(k[cz][sy][sx], (T)Xz[h + (2 * sy - 1) * kHX + 2 * sx - 1]);
          }
          if (!DIFF) sacc = fma(T(4) * ksum, xc, -sacc);
        }
        d = T(4) * hs * ksum;
        ax = hs * sacc;
      }
      T out;
      if (MODE == 0) out = ax;
      else if (MODE == 1) out = cur.b[r] - ax;
      else if (MODE == 2) out = g.wd ? fma(cur.o[r], cur.b[r] - ax, xc) : fma(cur.o[r], (cur.b[r] - ax) / d, xc);
      else out = g.wd ? cur.o[r] * cur.b[r] : cur.o[r] * (cur.b[r] / d);
      y[i] = out;
      if (RED) {
        acc0 = fma((double)out, (double)cur.v[r], acc0);
        if (v2) acc1 = fma((double)out, (double)cur.v2[r], acc1);
      }
    }
    cur = nxt;
    __syncthreads();  // slot s2 is refilled by the next issue
    si = s2;
    s2 = s1;
    s1 = s0;
    s0 = s0 + 1 == kStages ? 0 : s0 + 1;
  }
  cpa_wait<0>();
  if (RED) dr_finish2_grid(acc0, acc1, R, smem);
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
// One row per thread (the 27 loads of a row are its only latency chain).
template <int D, int P, int MODE, typename TB, typename TY, bool RED>
__global__ void __launch_bounds__(kBlock)
k_st32(const float* __restrict__ A, long long N, long long Np, long long M, float w, const float* __restrict__ om,
       const float* __restrict__ x, const TB* __restrict__ b, TY* __restrict__ y, const double* __restrict__ v,
       const double* __restrict__ v2, Reduce2 R) {
  constexpr int NS = St32<D, P>::NS;
  constexpr int C = St32<D, P>::CENTER;
  __shared__ double smem[8];
  double acc0 = 0.0, acc1 = 0.0;
  const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
  if (i < N) {
    float a[NS], xv[NS];
    if (MODE != 3) {
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        a[k] = __ldg(A + (long long)k * Np + i);
        xv[k] = __ldg(x + clampi(i + soff<D, P>(k, M), N));
      }
    }
    const float d = MODE != 3 ? a[C] : __ldg(A + (long long)C * Np + i);
    float s = 0.f;
    if (MODE != 3) {
#pragma unroll
      for (int k = 0; k < NS; ++k) s = fmaf(a[k], xv[k], s);
    }
    float out;
    if (MODE == 0) out = s;
    else if (MODE == 1) out = ldv(b, i) - s;
    else if (MODE == 2) out = fmaf(om ? om[i] : w, (ldv(b, i) - s) / d, xv[C]);
    else out = (om ? om[i] : w) * (ldv(b, i) / d);
    stv(y, i, out);
    if (RED) {
      acc0 = fma((double)out, (double)v[i], acc0);
      if (v2) acc1 = fma((double)out, (double)v2[i], acc1);
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
__global__ void __launch_bounds__(kBlock)
k_restrict_q1(int MC, int MF, int dmask, const TR* __restrict__ rf, __nv_bfloat16* __restrict__ bc,
              float* __restrict__ xc) {
  if (D == 1 && threadIdx.y != 0) return;
  const int cJ[3] = {(int)(blockIdx.x * 32 + threadIdx.x), D > 1 ? (int)(blockIdx.y * 8 + threadIdx.y) : 0,
                     D > 2 ? (int)blockIdx.z : 0};
  if (cJ[0] >= MC || cJ[1] >= MC) return;
  const long long J = cJ[0] + (long long)MC * (cJ[1] + (long long)MC * cJ[2]);
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

// 3D Q1 prolongation by coarse node: thread (I, J, K) updates the fine nodes
// (2I+a, 2J+b, 2K+c), a, b, c in {0, 1}, from the 8 coarse values at
// I..I+1, J..J+1, K..K+1, loaded once; each fine node is summed with the
// weights and in the order of k_prolong_q1 (coarse Dirichlet values read as
// zero, which is what a zero weight gives there).
__global__ void __launch_bounds__(kBlock)
k_prolong_q1c(int MF, int MC, int dmask, const float* __restrict__ xc, float* __restrict__ xf) {
  const int I = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y, K = blockIdx.z;
  if (I >= MC || J >= MC) return;
  const long long MC2 = (long long)MC * MC, MF2 = (long long)MF * MF;
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
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int fz = 2 * K + c;
    if (fz >= MF || fdir(fz, MF, 2, dmask)) continue;
    const float wz0 = c ? .5f : 1.f, wz1 = c ? .5f : 0.f;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int fy = 2 * J + b;
      if (fy >= MF || fdir(fy, MF, 1, dmask)) continue;
      const float wy0 = b ? .5f : 1.f, wy1 = b ? .5f : 0.f;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int fx = 2 * I + a;
        if (fx >= MF || fdir(fx, MF, 0, dmask)) continue;
        const float wx0 = a ? .5f : 1.f, wx1 = a ? .5f : 0.f;
        float acc = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int bx = q & 1, by = (q >> 1) & 1, bz = q >> 2;
          const float ww = (bx ? wx1 : wx0) * (by ? wy1 : wy0) * (bz ? wz1 : wz0);
          // even fine index: the second coarse node is the first one, weight 0
          acc = fmaf(ww, v[c ? bz : 0][b ? by : 0][a ? bx : 0], acc);
        }
        float* o = xf + fz * MF2 + (long long)fy * MF + fx;
        *o += acc;
      }
    }
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

// coarsest level in FP64: x = A^-1 b (b BF16 -> FP64, x FP32)
__global__ void __launch_bounds__(1024)
k_coarse_mx(const double* __restrict__ AinvT, int n, const __nv_bfloat16* __restrict__ b, float* __restrict__ x) {
  __shared__ double rs[1024];
  const int i = threadIdx.x;
  if (i < n) rs[i] = (double)__bfloat162float(b[i]);
  __syncthreads();
  if (i >= n) return;
  double acc = 0.0;
  for (int j = 0; j < n; ++j) acc = fma(AinvT[(long long)j * n + i], rs[j], acc);
  x[i] = (float)acc;
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
// copy of the new residual scaled by the current scale slot
__global__ void __launch_bounds__(kBlock)
k_fcg64_update(double* sc, double* __restrict__ x, const float* __restrict__ p, double* __restrict__ r,
               const double* __restrict__ a, float* __restrict__ r32, long long n, Reduce2 R) {
  __shared__ double smem[8];
  const double lam = sc[M_LAM], s = sc[M_SCALE];
  double acc = 0.0;
  const long long i0 = ((long long)blockIdx.x * kBlock + threadIdx.x) * 2;
  if (i0 < n) {  // n is the padded length (even); padding entries are zero
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

constexpr int kZS2 = 32;  // planes per CTA of k_mf2

static dim3 mf2_grid(int M) {
  return dim3((unsigned)((M + kMX - 1) / kMX), (unsigned)((M + kMY4 - 1) / kMY4), (unsigned)((M + kZS2 - 1) / kZS2));
}

template <typename T, typename TV, typename TX>
static void mf_launch(int mode, const MFArgsT<T>& g, const TX* x, const T* b, T* y, const TV* v, const TV* v2,
                      const Reduce2* R, cudaStream_t st) {
  const dim3 grid = mf2_grid(g.M);
  Reduce2 r0 = R ? *R : Reduce2{};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if constexpr (sizeof(T) == 8) {  // the FP64 operator is only applied (mode 0)
    if (R) k_mf4<T, TV, TX, kZS2, 0, true><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0);
    else k_mf4<T, TV, TX, kZS2, 0, false><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0);
  } else if (R) {
    switch (mode) {
      case 0: k_mf4<T, TV, TX, kZS2, 0, true><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 1: k_mf4<T, TV, TX, kZS2, 1, true><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 2: k_mf4<T, TV, TX, kZS2, 2, true><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      default: k_mf4<T, TV, TX, kZS2, 3, true><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0);
    }
  } else {
    switch (mode) {
      case 0: k_mf4<T, TV, TX, kZS2, 0, false><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 1: k_mf4<T, TV, TX, kZS2, 1, false><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 2: k_mf4<T, TV, TX, kZS2, 2, false><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0); break;
      default: k_mf4<T, TV, TX, kZS2, 3, false><<<grid, kMFThreads, 0, st>>>(g, x, b, y, v, v2, r0);
    }
  }
}

// pre-smoothing from zero with the damping over the diagonal formed: y = wd b
__global__ void __launch_bounds__(kBlock) k_wd_scale(const float* __restrict__ wd, const float* __restrict__ b,
                                                     float* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
  if (i < n) y[i] = __ldg(wd + i) * __ldg(b + i);
}

// wd = damping / diagonal of the matrix-free top level, the diagonal formed
// as in k_mf4 (4 hs times the sum of the node's 8 cell coefficients, summed
// in the same order; cells outside the grid count zero); Dirichlet nodes
// (identity rows) get the damping itself
__global__ void __launch_bounds__(kBlock) k_mf_wd(MFArgs g, float* __restrict__ wd) {
  const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
  if (i >= g.N) return;
  const int M = g.M, n = g.n, dm = g.dmask;
  const int ix = (int)(i % M), iy = (int)((i / M) % M), iz = (int)(i / ((long long)M * M));
  auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
  const float om = g.omega ? __ldg(g.omega + i) : g.w;
  if (dirf(ix, 1, 2) || dirf(iy, 4, 8) || dirf(iz, 16, 32)) {
    wd[i] = om;
    return;
  }
  float k[2][2][2];
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
  const float wc[2][2] = {{k[0][0][0] + k[1][0][0], k[0][0][1] + k[1][0][1]},
                          {k[0][1][0] + k[1][1][0], k[0][1][1] + k[1][1][1]}};
  const float ksum = (wc[0][0] + wc[0][1]) + (wc[1][0] + wc[1][1]);
  wd[i] = om / (4.f * g.hs * ksum);
}

void mx_top_wd(const MFArgs& g, float* wd, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_mf_wd<<<g1(g.N), kBlock, 0, st>>>(g, wd);
}

void mx_top_apply(int mode, const MFArgs& g, const float* x, const float* b, float* y, const double* v,
                  const double* v2, const Reduce2* R, cudaStream_t st) {
  if (mode == 3 && g.wd && !R) {  // a stream of two reads and a write
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_wd_scale<<<g1(g.N), kBlock, 0, st>>>(g.wd, b, y, g.N);
    return;
  }
  mf_launch<float, double, float>(mode, g, x, b, y, v, v2, R, st);
}

void mx_top_apply64(const MFArgs64& g, const float* x, double* y, const float* v, const Reduce2* R,
                    cudaStream_t st) {
  mf_launch<double, float, float>(0, g, x, nullptr, y, v, nullptr, R, st);
}

void mx_top_apply64x(const MFArgs64& g, const double* x, double* y, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_mf4<double, double, double, kZS2, 0, false><<<mf2_grid(g.M), kMFThreads, 0, st>>>(g, x, nullptr, y, nullptr,
                                                                                     nullptr, Reduce2{});
}

void mx_top_residual64(const MFArgs64& g, const double* x, const double* b, double* r, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_mf4<double, double, double, kZS2, 1, false><<<mf2_grid(g.M), kMFThreads, 0, st>>>(g, x, b, r, nullptr, nullptr,
                                                                                     Reduce2{});
}

long long mx_top_blocks(int M) {
  const dim3 gr = mf2_grid(M);
  return (long long)gr.x * gr.y * gr.z;
}

void mx_level_apply(int mode, const Lev32& L, const float* x, const void* b, bool b_bf16, void* y, bool y_bf16,
                    const double* v, const double* v2, const Reduce2* R, cudaStream_t st) {
  const unsigned grid = g1(L.N);
  Reduce2 r0 = R ? *R : Reduce2{};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  typedef __nv_bfloat16 bf;
  MX_DISPATCH(L.dim, L.order, {
    if (R) {  // reductions only on FP32 vectors
      if (mode == 0) k_st32<D, P, 0, float, float, true><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
      else if (mode == 2) k_st32<D, P, 2, float, float, true><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
      else k_st32<D, P, 1, float, float, true><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
    } else if (mode == 0) {
      k_st32<D, P, 0, float, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
    } else if (mode == 1) {
      if (b_bf16 && y_bf16) k_st32<D, P, 1, bf, bf, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const bf*)b, (bf*)y, v, v2, r0);
      else if (b_bf16) k_st32<D, P, 1, bf, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const bf*)b, (float*)y, v, v2, r0);
      else if (y_bf16) k_st32<D, P, 1, float, bf, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (bf*)y, v, v2, r0);
      else k_st32<D, P, 1, float, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
    } else if (mode == 2) {
      if (b_bf16) k_st32<D, P, 2, bf, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const bf*)b, (float*)y, v, v2, r0);
      else k_st32<D, P, 2, float, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
    } else {
      if (b_bf16) k_st32<D, P, 3, bf, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const bf*)b, (float*)y, v, v2, r0);
      else k_st32<D, P, 3, float, float, false><<<grid, kBlock, 0, st>>>(L.A, L.N, L.Np, L.M, L.w, L.om, x, (const float*)b, (float*)y, v, v2, r0);
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
    if (F.dim == 3) {
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

void mx_prolong(const Lev32& C, const Lev32& F, const float* xc, float* xf, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const dim3 gr = xgrid(F.M, F.dim), bl(32, 8);
  if (F.order == 1) {
    if (F.dim == 3)
      k_prolong_q1c<<<dim3((unsigned)((C.M + 31) / 32), (unsigned)((C.M + 7) / 8), (unsigned)C.M), bl, 0, st>>>(
          (int)F.M, (int)C.M, F.dmask, xc, xf);
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
  k_fcg64_update<<<g1(np / 2), kBlock, 0, st>>>(sc, x, p, r, a, r32, np, R);
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
