// fmgpu_learn.cuh -- the damping network: parameter layout, activation
// geometry, the net handle and the launch interface of its kernels.
//
// Net (D = 2 or 3, 3^D taps, 'same' convolutions with zero padding):
//   X0  16 channels per node: for each of the 2^D cells around the node its
//       centred log coefficient and a presence bit (rest zero)
//   H1 = relu(conv(X0; W1) + b1)       32 channels
//   H2 = relu(conv(H1; W2) + b2)       32 channels
//   z  = conv(H2; W3) + b3             1 channel
//   omega = omega_min + (omega_max - omega_min) * sigmoid(z)
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "fmgpu_internal.cuh"

struct fmg_ctx;

namespace fmg {

constexpr int kNetIn = 16;    // input channels (padded)
constexpr int kNetHid = 32;   // hidden channels
constexpr int kNetOut = 16;   // output channels of the last GEMM (channel 0 used)
constexpr int kLogSumBlocks = 1184;  // blocks of the mean-log-k reduction (8 per SM of a B200)

// offsets of the flat FP32 parameter vector
struct NetLayout {
  int dim = 0, taps = 0;
  long long w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, n = 0;
};
NetLayout net_layout(int dim);

// node grid of one level (or a batch of 2D problems stacked in z), padded by
// one zero ghost node on each side in x, y (and z for D = 3)
struct ActGeom {
  int D = 0, Mx = 0, My = 0, Mz = 0;  // interior nodes (2D: Mz = planes)
  int Px = 0, Py = 0, Pz = 0;         // padded extents
  long long npad() const { return (long long)Px * Py * Pz; }
  long long nodes() const { return (long long)Mx * My * Mz; }
};
ActGeom act_geom(int D, int M, int planes);

}  // namespace fmg

struct fmg_net {
  fmg_ctx* ctx = nullptr;
  int dim = 0;
  fmg::NetLayout lay;
  float omega_min = 0.2f, omega_max = 1.0f;
  unsigned long long seed = 0;
  float* P = nullptr;          // parameters (FP32, flat layout)
  float* G = nullptr;          // accumulated gradients
  float* Mo = nullptr;         // Adam moments
  float* Vo = nullptr;
  long long adam_t = 0;
  __nv_bfloat16* wf1 = nullptr;  // [taps][32][16]
  __nv_bfloat16* wf2 = nullptr;  // [taps][32][32]
  __nv_bfloat16* wf3 = nullptr;  // [taps][16][32], row 0 = W3
  __nv_bfloat16* wb2 = nullptr;  // backward: [taps][32 ci][32 co] = W2[flip][co][ci]
  __nv_bfloat16* wb3 = nullptr;  // backward: [taps][32 ci][16 co], column 0 = W3[flip][ci]
  bool weights_stale = true;     // BF16 copies out of date
  // activations of the last forward pass (grown on demand)
  long long cap = 0;
  __nv_bfloat16 *X0 = nullptr, *H1 = nullptr, *H2 = nullptr, *dZ = nullptr, *dP2 = nullptr, *dP1 = nullptr;
  fmg::ActGeom geom;           // geometry of the last forward pass
  bool have_forward = false;
  float* part = nullptr;       // weight-gradient partials
  long long part_cap = 0;
  double* stat = nullptr;      // [0] mean log k, from [8] the kLogSumBlocks partials of its sum
  float* fc = nullptr;         // cell feature values of the level being featurised
  long long fc_cap = 0;
  double* lraw = nullptr;      // log k of every top-level cell, taken with the mean
  long long lraw_cap = 0, lraw_n = 0;  // capacity; cells it holds now (0: none)
  unsigned* err = nullptr;     // device error word (bounded waits that ran out)
  std::vector<void*> allocs;
};

namespace fmg {

// device allocations of a net (zeroed)
int net_alloc(fmg_net* net, void** p, size_t bytes);
void net_free_all(fmg_net* net);
int net_reserve(fmg_net* net, const ActGeom& g);  // activation buffers for g
void net_refresh_weights(fmg_net* net, cudaStream_t st);

// mean of log k over n cells -> *out (device), deterministic
int launch_logmean(fmg_net* net, const double* k, long long n, double* out, cudaStream_t st);
// features of level nodes (Q1): cells of n_l per direction, coefficient of
// the top level (n_top cells per direction) sampled at np Gauss points xi
// per direction of each level cell (ratio = n_top / n_l); kconst used when
// kcell is null
// (written to net->X0; the level's cell log-coefficients go to net->lk first)
// sub = 2 for Q2 node grids: a node's 2^D adjacent half-cells, each in a cell
int launch_features(fmg_net* net, const ActGeom& g, int n_l, int sub, long long n_top, double ratio, int np,
                    const double* xi, const double* kcell, double kconst, const double* mean, cudaStream_t st);
// the three forward convolutions; omega (level order, FP64) written when non-null
int net_forward(fmg_net* net, const ActGeom& g, double* omega, cudaStream_t st);
// backward from dL/domega (level order) through the net of the last forward
// pass; gradients added to net->G
int net_backward(fmg_net* net, const double* gomega, const double* omega, cudaStream_t st);
void launch_adam(fmg_net* net, float lr, float b1, float b2, float eps, cudaStream_t st);
int net_check_error(fmg_net* net, cudaStream_t st, const char** msg);
// one CTA waits on an mbarrier with the given limits (arrive: a thread arrives
// first); FMG_ERR_CUDA with *msg set when the wait gave up
int wait_selftest(int arrive, int max_polls, long long max_ns, cudaStream_t st, const char** msg);

// FP64 helpers of the training loss (level vectors of length n)
// nc values per node (vector form), nodes on the Dirichlet faces zero
void launch_rand_fill(double* e, int D, long long M, int dmask, unsigned long long seed, cudaStream_t st, int nc = 1);
// v = u / diag(A)   (diag: slot `center` of the stencil storage)
void launch_dinv(const double* A, int center, long long Np, const double* u, double* v, long long n, cudaStream_t st);
// y = x - w .* v
void launch_sub_wv(const double* x, const double* w, const double* v, double* y, long long n, cudaStream_t st);
// g_omega (+)= -g .* v
void launch_gomega(const double* g, const double* v, double* gw, bool accumulate, long long n, cudaStream_t st);
// t = w .* g / diag(A)
void launch_wg_dinv(const double* A, int center, long long Np, const double* w, const double* g, double* t,
                    long long n, cudaStream_t st);
// scal[dst] (+)= factor * scal[num] / scal[den]
void launch_ratio_acc(double* scal, int dst, int num, int den, double factor, bool first, cudaStream_t st);
void launch_set_scalar(double* p, double v, cudaStream_t st);
// y = x + w .* v (y may be x); acc += a .* b; y += w .* x / diag(A); y += x
void launch_xpwv(const double* x, const double* w, const double* v, double* y, long long n, cudaStream_t st);
void launch_acc_prod(double* acc, const double* a, const double* b, long long n, cudaStream_t st);
void launch_wg_dinv_acc(const double* A, int center, long long Np, const double* w, const double* x, double* y,
                        long long n, cudaStream_t st);
void launch_add(const double* x, double* y, long long n, cudaStream_t st);
// y = s * x / scal[slot]
void launch_scale_by(const double* x, double s, const double* scal, int slot, double* y, long long n,
                     cudaStream_t st);

}  // namespace fmg
