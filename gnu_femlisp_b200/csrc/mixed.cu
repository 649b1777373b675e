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

// Register-blocked stencil: a thread owns NX consecutive nodes along x of
// one (y, z-segment) column block and marches z over ZS planes, keeping the
// x values of three planes (rows y-1, y, y+1, positions x-1 .. x+NX) and the
// coefficients of two cell planes (rows y-1, y, cells x-1 .. x+NX-1) in
// registers.  Each new plane costs 3 (NX+2) loads of x and 2 (NX+1) loads of
// k, shared by NX nodes; validity is separable per direction (inside the grid
// and off the Dirichlet faces), so eliminated columns read as zero.
// mode 0: y = A x; 1: y = b - A x; 2: y = x + w (b - A x)/d; 3: y = w b / d
// (x = 0).  With RED, (y, v) and (y, v2) are accumulated in FP64.
template <typename T, typename TV, int NX, int ZS, int MODE, bool RED>
__global__ void __launch_bounds__(kBlock, 2)
k_mf_q1(MFArgsT<T> g, const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ y,
        const TV* __restrict__ v, const TV* __restrict__ v2, Reduce2 R) {
  __shared__ double smem[8];
  const int M = g.M, n = g.n, dm = g.dmask;
  const int ngx = (M + NX - 1) / NX;
  const long long t = (long long)blockIdx.x * kBlock + threadIdx.x;
  const int xg = (int)(t % ngx), iy = (int)(t / ngx);
  const int ix0 = xg * NX, z0 = blockIdx.y * ZS;
  double acc0 = 0.0, acc1 = 0.0;
  if (iy < M) {
    const long long MM = (long long)M * M;
    auto dirf = [&](int c, int lo, int hi) { return (c == 0 && (dm & lo)) || (c == M - 1 && (dm & hi)); };
    T W[3][3][NX + 2];   // [plane][row][x]
    T K[2][2][NX + 1];   // [cell plane][cell row][cell x]
    // boundary columns: clamped addresses, validity recomputed per load
    // (inside the grid, off the Dirichlet faces; cells inside the grid)
    auto ldplane = [&](int jz, T (*dst)[NX + 2]) {
      const bool vz = jz >= 0 && jz < M && !dirf(jz, 16, 32);
      const long long zb = (long long)min(max(jz, 0), M - 1) * MM;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int jy = iy - 1 + r;
        const bool vr = vz && jy >= 0 && jy < M && !dirf(jy, 4, 8);
        const T* row = x + zb + (long long)min(max(jy, 0), M - 1) * M;
#pragma unroll
        for (int j = 0; j < NX + 2; ++j) {
          const int jx = ix0 - 1 + j;
          const bool ok = vr && jx >= 0 && jx < M && !dirf(jx, 1, 2);
          const T xv = __ldg(row + min(max(jx, 0), M - 1));
          dst[r][j] = ok ? xv : T(0);
        }
      }
    };
    auto ldcells = [&](int cz, T (*dst)[NX + 1]) {
      const bool vz = cz >= 0 && cz < n;
      const long long zb = (long long)min(max(cz, 0), n - 1) * n * n;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int cy = iy - 1 + r;
        const bool vr = vz && cy >= 0 && cy < n;
        const T* row = g.k + zb + (long long)min(max(cy, 0), n - 1) * n;
#pragma unroll
        for (int j = 0; j < NX + 1; ++j) {
          const int cx = ix0 - 1 + j;
          const T kv = __ldg(row + min(max(cx, 0), n - 1));
          dst[r][j] = (vr && cx >= 0 && cx < n) ? kv : T(0);
        }
      }
    };
    // interior columns (every x and y neighbour position in 1 .. M-2) load
    // without clamps or masks; a plane is then valid or zero as a whole
    const bool fast = ix0 >= 2 && ix0 + NX <= M - 2 && iy >= 2 && iy <= M - 3;
    const T* xcol = x + (long long)(iy - 1) * M + (ix0 - 1);
    const T* kcol = g.k + (long long)(iy - 1) * n + (ix0 - 1);
    auto ldplane_fast = [&](int jz, T (*dst)[NX + 2]) {
      const bool vz = jz >= 0 && jz < M && !dirf(jz, 16, 32);
      if (vz) {
        const T* p0 = xcol + (long long)jz * MM;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int j = 0; j < NX + 2; ++j) dst[r][j] = __ldg(p0 + r * M + j);
      } else {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int j = 0; j < NX + 2; ++j) dst[r][j] = T(0);
      }
    };
    auto ldcells_fast = [&](int cz, T (*dst)[NX + 1]) {
      if (cz >= 0 && cz < n) {
        const T* p0 = kcol + (long long)cz * n * n;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int j = 0; j < NX + 1; ++j) dst[r][j] = __ldg(p0 + r * n + j);
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int j = 0; j < NX + 1; ++j) dst[r][j] = T(0);
      }
    };
    if (fast) {
      if (MODE != 3) { ldplane_fast(z0 - 1, W[0]); ldplane_fast(z0, W[1]); }
      ldcells_fast(z0 - 1, K[0]);
    } else {
      if (MODE != 3) { ldplane(z0 - 1, W[0]); ldplane(z0, W[1]); }
      ldcells(z0 - 1, K[0]);
    }
    const bool diry = dirf(iy, 4, 8);
    const T hs = g.hs;
#pragma unroll 1
    for (int kz = 0; kz < ZS; ++kz) {
      const int iz = z0 + kz;
      if (iz < M) {
        if (fast) {
          if (MODE != 3) ldplane_fast(iz + 1, W[2]);
          ldcells_fast(iz, K[1]);
        } else {
          if (MODE != 3) ldplane(iz + 1, W[2]);
          ldcells(iz, K[1]);
        }
        const bool dirz = dirf(iz, 16, 32);
        const long long rowi = (long long)iz * MM + (long long)iy * M;
#pragma unroll
        for (int j = 0; j < NX; ++j) {
          const int ix = ix0 + j;
          if (ix < M) {
            const long long i = rowi + ix;
            const bool dir = diry || dirz || dirf(ix, 1, 2);
            T ax = T(0), d = T(1), xc = T(0);
            if (dir) {
              if (MODE != 3) { xc = x[i]; ax = xc; }
            } else {
              T ks = T(0), sacc = T(0);
              xc = MODE != 3 ? W[1][1][j + 1] : T(0);
#pragma unroll
              for (int c = 0; c < 8; ++c) {
                const int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
                const T kc = K[cz][cy][j + cx];
                ks += kc;
                if (MODE != 3) {
                  const int px = j + 1 + (2 * cx - 1), py = 1 + (2 * cy - 1), pz = 1 + (2 * cz - 1);
                  const T e = T(4) * xc - W[1][py][px] - W[pz][1][px] - W[pz][py][j + 1] - W[pz][py][px];
                  sacc = fma(kc, e, sacc);
                }
              }
              d = T(4) * hs * ks;
              ax = hs * sacc;
            }
            T out;
            if (MODE == 0) out = ax;
            else if (MODE == 1) out = b[i] - ax;
            else if (MODE == 2) out = fma(g.omega ? g.omega[i] : g.w, (b[i] - ax) / d, xc);
            else out = (g.omega ? g.omega[i] : g.w) * (b[i] / d);
            y[i] = out;
            if (RED) {
              acc0 = fma((double)out, (double)v[i], acc0);
              if (v2) acc1 = fma((double)out, (double)v2[i], acc1);
            }
          }
        }
        if (MODE != 3) {
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int j = 0; j < NX + 2; ++j) { W[0][r][j] = W[1][r][j]; W[1][r][j] = W[2][r][j]; }
        }
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int j = 0; j < NX + 1; ++j) K[0][r][j] = K[1][r][j];
      }
    }
  }
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
k_fcg64_update(double* sc, double* __restrict__ x, const double* __restrict__ p, double* __restrict__ r,
               const double* __restrict__ a, float* __restrict__ r32, long long n, Reduce2 R) {
  __shared__ double smem[8];
  const double lam = sc[M_LAM], s = sc[M_SCALE];
  double acc = 0.0;
  const long long i0 = ((long long)blockIdx.x * kBlock + threadIdx.x) * 2;
  if (i0 < n) {  // n is the padded length (even); padding entries are zero
    const double2 pv = *reinterpret_cast<const double2*>(p + i0);
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

// p = q / s + beta p  (first: p = q / s), s the scale of the FP32 residual
__global__ void k_fcg64_p(const double* __restrict__ sc, double* __restrict__ p, const float* __restrict__ q,
                          long long n, int first) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double z = (double)q[i] / sc[M_SUSED];
  p[i] = first ? z : fma(sc[M_BETA], p[i], z);
}

// r32 = r * sc[slot]
__global__ void k_scale_to32(const double* __restrict__ r, const double* __restrict__ sc, int slot,
                             float* __restrict__ r32, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r32[i] = (float)(r[i] * sc[slot]);
}

// two FP64 dot products (x, y) and (x, y2) with the epilogue of R
__global__ void __launch_bounds__(kBlock)
k_dot2_64(const double* __restrict__ xv, const double* __restrict__ yv, const double* __restrict__ y2,
          long long n, Reduce2 R) {
  __shared__ double smem[8];
  const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
  double a0 = 0.0, a1 = 0.0;
  if (i < n) {
    a0 = xv[i] * yv[i];
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

constexpr int kNX32 = 4, kNX64 = 1, kZS = 8;

template <typename T, typename TV, int NX>
static unsigned mf_blocks_x(int M) {
  const long long cols = (long long)((M + NX - 1) / NX) * M;
  return (unsigned)((cols + kBlock - 1) / kBlock);
}

template <typename T, typename TV, int NX>
static void mf_launch(int mode, const MFArgsT<T>& g, const T* x, const T* b, T* y, const TV* v, const TV* v2,
                      const Reduce2* R, cudaStream_t st) {
  const dim3 grid(mf_blocks_x<T, TV, NX>(g.M), (g.M + kZS - 1) / kZS);
  Reduce2 r0 = R ? *R : Reduce2{};
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (R) {
    switch (mode) {
      case 0: k_mf_q1<T, TV, NX, kZS, 0, true><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 1: k_mf_q1<T, TV, NX, kZS, 1, true><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 2: k_mf_q1<T, TV, NX, kZS, 2, true><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      default: k_mf_q1<T, TV, NX, kZS, 3, true><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0);
    }
  } else {
    switch (mode) {
      case 0: k_mf_q1<T, TV, NX, kZS, 0, false><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 1: k_mf_q1<T, TV, NX, kZS, 1, false><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      case 2: k_mf_q1<T, TV, NX, kZS, 2, false><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0); break;
      default: k_mf_q1<T, TV, NX, kZS, 3, false><<<grid, kBlock, 0, st>>>(g, x, b, y, v, v2, r0);
    }
  }
}

void mx_top_apply(int mode, const MFArgs& g, const float* x, const float* b, float* y, const double* v,
                  const double* v2, const Reduce2* R, cudaStream_t st) {
  mf_launch<float, double, kNX32>(mode, g, x, b, y, v, v2, R, st);
}

void mx_top_apply64(const MFArgs64& g, const double* x, double* y, const double* v, const Reduce2* R,
                    cudaStream_t st) {
  mf_launch<double, double, kNX64>(0, g, x, nullptr, y, v, nullptr, R, st);
}

long long mx_top_blocks(int M) {
  const long long a = (long long)mf_blocks_x<float, double, kNX32>(M) * ((M + kZS - 1) / kZS);
  const long long b = (long long)mf_blocks_x<double, double, kNX64>(M) * ((M + kZS - 1) / kZS);
  return a > b ? a : b;
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
    if (F.dim == 3) k_prolong_q1<3><<<gr, bl, 0, st>>>((int)F.M, (int)C.M, F.dmask, xc, xf);
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

void mx_fcg64_update(double* sc, double* x, const double* p, double* r, const double* a, float* r32, long long np,
                     const Reduce2& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fcg64_update<<<g1(np / 2), kBlock, 0, st>>>(sc, x, p, r, a, r32, np, R);
}

void mx_fcg64_p(const double* sc, double* p, const float* q, long long n, bool first, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fcg64_p<<<g1(n), kBlock, 0, st>>>(sc, p, q, n, first ? 1 : 0);
}

void mx_scale_to32(const double* r, const double* sc, int slot, float* r32, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_scale_to32<<<g1(n), kBlock, 0, st>>>(r, sc, slot, r32, n);
}

void mx_dot2_64(const double* x, const double* y, const double* y2, long long n, const Reduce2& R, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dot2_64<<<g1(n), kBlock, 0, st>>>(x, y, y2, n, R);
}

}  // namespace fmg
