// fmgpu_mixed.cuh -- launch interface of the mixed-precision kernels.
#pragma once

#include <cuda_bf16.h>

#include "fmgpu_internal.cuh"

namespace fmg {

// scalar slots of the mixed solve (FP64)
enum MScal { M_ALPHA = 0, M_PA, M_LAM, M_BETA, M_QA, M_RR, M_SCALE, M_SUSED, M_TMP, M_SINV,
             M_ZAL, M_ZRP, M_ZAP,  // the in-solve judge: (z, A z) of the learned cycle, (z, r) and (z, A z) of the plain one
             M_COUNT = 16 };
enum Epi2 { EPI2_STORE = 0, EPI2_LAMBDA = 1, EPI2_FCG = 2, EPI2_RHO = 3, EPI2_UPDATE = 4 };

struct Reduce2 {
  double* part;        // 2 partials per chunk
  unsigned* counter;
  double* scal;
  int epi, slot0, slot1;
};

// Where a top-level vector keeps node (ix, iy, iz): at front + ix + py iy +
// pz iz.  Natural: front 0, py = M, pz = M^2.  Padded (the FP32 vectors and
// the FP64 residual and A p of the matrix-free mixed solve): rows of py = 4k
// elements and front = (4 - l) % 4, l = 1 when the face x = 0 is Dirichlet,
// so that the row start of the first node off that face sits on a 16-byte
// boundary -- a plane's tile of such a vector is one tensor copy.  The
// padding stays zero.
struct VLay {
  int front = 0, py = 0;
  long long pz = 0, total = 0;  // total: elements of the array (pads included)
  __host__ __device__ __forceinline__ long long at(int ix, int iy, int iz) const {
    return front + ix + (long long)py * iy + pz * iz;
  }
};
VLay natural_lay(int M, int dim);
VLay padded_lay(int M, int dmask);

// matrix-free 3D Q1 top level
template <typename T>
struct MFArgsT {
  const T* k;          // coefficient per cell (n^3)
  const T* omega;      // per-node damping or nullptr (natural layout)
  long long N;
  int M, n, dmask;
  T hs;                // h / 12
  T w;                 // scalar damping
  const T* wd = nullptr;  // per-node damping / diagonal (mx_top_wd), or nullptr: formed in the kernel
  double* err = nullptr;  // set to 1 by a CTA whose bounded wait for a copy ran out
  // layouts of x, of the per-node operands (b, wd, the reduction vectors) and
  // of the output y.  An FP32 x comes by tensor copy and must be padded, so
  // must the operands of the FP32 modes; FP64 x and operands are natural.
  VLay xl, ol, yl;
};
typedef MFArgsT<float> MFArgs;
typedef MFArgsT<double> MFArgs64;

// one level with an FP32 copy of its assembled matrix
struct Lev32 {
  const float* A;      // [slot][Np]
  const float* om;     // per-node damping or nullptr
  long long N, Np, M;
  int dim, order, dmask;
  float w;
};

void mx_top_apply(int mode, const MFArgs& g, const float* x, const float* b, float* y, const double* v,
                  const double* v2, const Reduce2* R, cudaStream_t st);
// FP64 y = A x on the top level for an FP32 x, with (y, v) reduced (epilogue of R)
void mx_top_apply64(const MFArgs64& g, const float* x, double* y, const float* v, const Reduce2* R,
                    cudaStream_t st);
// the FP64 operator of FP64 vectors: y = A x (the probe's right-hand side)
// and r = b - A x (the true residual of the mixed solve), from the cell
// coefficients like the FP64 CG operator
void mx_top_apply64x(const MFArgs64& g, const double* x, double* y, cudaStream_t st);
void mx_top_residual64(const MFArgs64& g, const double* x, const double* b, double* r, cudaStream_t st);
long long mx_top_blocks(int M);  // blocks of the matrix-free kernel (reduction partials)
// wd = damping / diagonal per top-level node (Dirichlet nodes: the damping)
// for the smoothing modes of mx_top_apply
void mx_top_wd(const MFArgs& g, float* wd, cudaStream_t st);  // wd in g.ol
void mx_level_apply(int mode, const Lev32& L, const float* x, const void* b, bool b_bf16, void* y, bool y_bf16,
                    const double* v, const double* v2, const Reduce2* R, cudaStream_t st);
void mx_restrict(const Lev32& F, const Lev32& C, const void* rf, bool rf_bf16, __nv_bfloat16* bc, float* xc,
                 cudaStream_t st);
void mx_prolong(const Lev32& C, const Lev32& F, const float* xc, float* xf, cudaStream_t st,
                const VLay* xfl = nullptr);  // xfl: the layout of xf (natural if null)
void mx_coarse(const double* AinvT, int n, const __nv_bfloat16* b, float* x, cudaStream_t st);
void mx_f64_to_f32(const double* a, float* b, long long n, cudaStream_t st);
// b (layout bl) = a (natural, M nodes a side, 3D)
void mx_f64_to_f32_lay(const double* a, float* b, const VLay& bl, int M, cudaStream_t st);
void mx_f64_copy_lay(const double* a, double* b, const VLay& bl, int M, cudaStream_t st);
// b (natural) = a (layout al), FP64, 3D
void mx_f64_from_lay(const double* a, const VLay& al, double* b, int M, cudaStream_t st);
// FP64 flexible CG: x += lam p, r -= lam a, (r,r), r32 = r * scale, all five
// in one layout of np elements (even; padding zero)
void mx_fcg64_update(double* sc, double* x, const float* p, double* r, const double* a, float* r32, long long np,
                     const Reduce2& R, cudaStream_t st);
// p = q / s + beta p (FP32 search direction)
void mx_fcg64_p(const double* sc, float* p, const float* q, long long n, bool first, cudaStream_t st);
void mx_f32_to_f64(const float* a, double* b, long long n, cudaStream_t st);
void mx_scale_to32(const double* r, const double* sc, int slot, float* r32, long long n, cudaStream_t st);
void mx_dot2_64(const double* x, const float* y, const double* y2, long long n, const Reduce2& R, cudaStream_t st);

}  // namespace fmg
