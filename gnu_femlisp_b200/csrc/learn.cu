// learn.cu -- kernels and handle of the damping network (the learned part of
// the smoother: per-node Jacobi damping predicted from the coefficient field).
//
// Every convolution of the net -- the three forward layers and the two
// data-gradient layers of the backward pass -- is one implicit GEMM on the
// 5th-generation tensor cores.  A CTA owns 8 x 16 output nodes of one plane
// (the 128 rows of one tcgen05.mma), stages the (8+2) x (16+2) x 3 halo of
// its input activations in shared memory in the no-swizzle K-major layout,
// and for each of the 3^D taps issues MMAs whose A operand is that halo
// shifted by the tap -- a different start address of the same shared memory,
// no copy -- against the tap's weights, accumulating the 128 x Cout tile in
// tensor memory.  The CTA is persistent: it stages the weights once and walks
// its tiles; two CTAs share an SM so one stages while the other multiplies.
//
// The weight gradients are tensor-core GEMMs as well: for each tap,
// dW[co][ci] = sum over nodes of G[node][co] X[node + tap][ci], the node
// dimension being K.  The staged gradient tile and the staged input halo are
// read MN-major (their 8 channels are the contiguous 16 bytes), M = 64 with
// the gradient channels zero-padded, 8 taps accumulating side by side in
// tensor memory across all tiles of a CTA; per-CTA partials are then summed
// in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "fmgpu_learn.cuh"
#include "umma.cuh"

namespace fmg {

NetLayout net_layout(int dim) {
  NetLayout L;
  L.dim = dim;
  L.taps = dim == 3 ? 27 : 9;
  long long o = 0;
  L.w1 = o; o += (long long)L.taps * kNetHid * kNetIn;
  L.b1 = o; o += kNetHid;
  L.w2 = o; o += (long long)L.taps * kNetHid * kNetHid;
  L.b2 = o; o += kNetHid;
  L.w3 = o; o += (long long)L.taps * kNetHid;
  L.b3 = o; o += 1;
  L.n = o;
  return L;
}

ActGeom act_geom(int D, int M, int planes) {
  ActGeom g;
  g.D = D;
  g.Mx = M; g.My = M; g.Mz = D == 3 ? M : planes;
  g.Px = M + 2; g.Py = M + 2; g.Pz = D == 3 ? M + 2 : planes;
  return g;
}

namespace {

typedef __nv_bfloat16 bf16;

constexpr int kThreads = 128;                  // 4 warps: one per tensor-memory lane quadrant
constexpr int TX = 8, TY = 16;                 // output tile (x fastest): 128 MMA rows
constexpr int HX = TX + 2, HY = TY + 2;        // halo tile
constexpr int kRowB = 16;                      // one 8-channel chunk of one node
constexpr int kHyB = HX * kRowB;               // 160: halo y-row stride
constexpr int kPlaneB = HY * kHyB;             // 2880: halo plane stride

template <int D>
struct Tp {
  static constexpr int TAPS = D == 3 ? 27 : 9;
  static constexpr int ZH = D == 3 ? 3 : 1;    // halo planes
  static constexpr int CHB = ZH * kPlaneB;     // bytes of one 8-channel chunk of the halo
  static constexpr int ROWS = HX * HY * ZH;    // halo nodes
};

struct TileGeo {
  int Mx, My, Mz, Px, Py, Pz, ntx, nty;
  long long ntiles;
};

TileGeo tile_geo(const ActGeom& g) {
  TileGeo t;
  t.Mx = g.Mx; t.My = g.My; t.Mz = g.Mz; t.Px = g.Px; t.Py = g.Py; t.Pz = g.Pz;
  t.ntx = (g.Mx + TX - 1) / TX;
  t.nty = (g.My + TY - 1) / TY;
  t.ntiles = (long long)t.ntx * t.nty * g.Mz;
  return t;
}

__device__ __forceinline__ void tile_xyz(const TileGeo& t, long long id, int& tx, int& ty, int& tz) {
  tx = (int)(id % t.ntx);
  const long long r = id / t.ntx;
  ty = (int)(r % t.nty);
  tz = (int)(r / t.nty);
}

// tap = (dx+1) + 3 (dy+1) [+ 9 (dz+1)]: byte offset of the shifted window in the halo
template <int D>
__device__ __forceinline__ uint32_t tap_off(int tap) {
  const int dx = tap % 3, dy = (tap / 3) % 3, dz = D == 3 ? tap / 9 : 0;
  return (uint32_t)(dz * kPlaneB + dy * kHyB + dx * kRowB);
}

// padded index of interior node (ix, iy) of plane tz
template <int D>
__device__ __forceinline__ long long pad_index(const TileGeo& t, int ix, int iy, int tz) {
  const int pz = D == 3 ? tz + 1 : tz;
  return ((long long)pz * t.Py + iy + 1) * t.Px + ix + 1;
}

// 16-byte asynchronous copy global -> shared, zero-filled when !ok
__device__ __forceinline__ void cp16(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(ok ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// halo of input activations [npad][C] -> shared memory, chunk c of halo node
// r = hx + HX (hy + HY hz) at byte c*CHB + 16 r (zeros outside the array);
// asynchronous copies, so all of a thread's copies are in flight at once
// (the caller waits with cp_wait_all before the barrier)
template <int D, int C>
__device__ __forceinline__ void stage_halo(uint8_t* hs, const bf16* __restrict__ in, const TileGeo& t, int tx,
                                           int ty, int tz) {
  constexpr int ROWS = Tp<D>::ROWS, CHB = Tp<D>::CHB;
  for (int idx = threadIdx.x; idx < (C / 8) * ROWS; idx += kThreads) {
    const int c = idx / ROWS, r = idx - c * ROWS;
    const int hx = r % HX, hy = (r / HX) % HY, hz = r / (HX * HY);
    const int px = tx * TX + hx, py = ty * TY + hy, pz = tz + hz;
    const bool ok = px < t.Px && py < t.Py && pz < t.Pz;
    const long long node = ok ? ((long long)pz * t.Py + py) * t.Px + px : 0;
    cp16(hs + c * CHB + r * kRowB, reinterpret_cast<const uint4*>(in + node * C) + c, ok);
  }
}

// weights [taps][COUT][CIN] -> per tap a K-major COUT x CIN tile (asynchronous)
template <int TAPS, int CIN, int COUT>
__device__ __forceinline__ void stage_weights(uint8_t* ws, const bf16* __restrict__ w) {
  constexpr int CH = CIN / 8;
  for (int idx = threadIdx.x; idx < TAPS * COUT * CH; idx += kThreads) {
    const int c = idx % CH, co = (idx / CH) % COUT, tap = idx / (CH * COUT);
    cp16(ws + tap * (COUT * CIN * 2) + umma::kmajor_offset(co, c * 8, CIN),
         reinterpret_cast<const uint4*>(w + ((long long)tap * COUT + co) * CIN) + c, true);
  }
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

enum ConvEpi { EPI_RELU = 0, EPI_OMEGA = 1, EPI_MASK = 2 };

struct ConvArgs {
  TileGeo t;
  const bf16* in;     // [npad][CIN]
  const bf16* w;      // [taps][COUT][CIN]
  const float* bias;  // EPI_RELU: COUT values; EPI_OMEGA: 1
  const bf16* mask;   // EPI_MASK: activation [npad][COUT] whose relu is differentiated
  bf16* out;          // [npad][COUT]
  double* omega;      // EPI_OMEGA: level order
  float omin, omax;
  unsigned* err;
};

// epilogue of output node (ix, iy) of plane tz: v = its COUT accumulators
template <int D, int COUT, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, const float* v, int ix, int iy, int tz) {
  if (ix < a.t.Mx && iy < a.t.My) {
    const long long p = pad_index<D>(a.t, ix, iy, tz);
    if constexpr (EPI == EPI_RELU) {
      uint32_t pk[COUT / 2];
#pragma unroll
      for (int c = 0; c < COUT; c += 2)
        pk[c / 2] = pack2(fmaxf(v[c] + __ldg(a.bias + c), 0.f), fmaxf(v[c + 1] + __ldg(a.bias + c + 1), 0.f));
      uint4* o = reinterpret_cast<uint4*>(a.out + p * COUT);
#pragma unroll
      for (int q = 0; q < COUT / 8; ++q) o[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
    } else if constexpr (EPI == EPI_OMEGA) {
      const float z = v[0] + __ldg(a.bias);
      const float s = 1.f / (1.f + __expf(-z));
      const long long i = ((long long)tz * a.t.My + iy) * a.t.Mx + ix;
      a.omega[i] = (double)(a.omin + (a.omax - a.omin) * s);
    } else {  // EPI_MASK
      const uint4* m = reinterpret_cast<const uint4*>(a.mask + p * COUT);
      uint4* o = reinterpret_cast<uint4*>(a.out + p * COUT);
#pragma unroll
      for (int q = 0; q < COUT / 8; ++q) {
        uint4 mm = __ldg(m + q);
        const bf16* mh = reinterpret_cast<const bf16*>(&mm);
        uint32_t pk[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const float g0 = __bfloat162float(mh[e]) > 0.f ? v[8 * q + e] : 0.f;
          const float g1 = __bfloat162float(mh[e + 1]) > 0.f ? v[8 * q + e + 1] : 0.f;
          pk[e / 2] = pack2(g0, g1);
        }
        o[q] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      }
    }
  }
}

template <int D, int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kThreads) k_conv(ConvArgs a) {
  constexpr int TAPS = Tp<D>::TAPS, CHB = Tp<D>::CHB;
  constexpr int WTAP = COUT * CIN * 2;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, COUT, false, false);
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* ws = smem;
  uint8_t* hs = smem + TAPS * WTAP;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  stage_weights<TAPS, CIN, COUT>(ws, a.w);
  cp_wait_all();
  if (warp == 0) umma::tmem_alloc(&tslot, 32);
  if (tid == 0) umma::mbar_init(&bar);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const uint32_t hb = umma::smem_u32(hs), wb = umma::smem_u32(ws);
  uint32_t phase = 0;
  bool failed = false;
  for (long long id = blockIdx.x; id < a.t.ntiles; id += gridDim.x) {
    int tx, ty, tz;
    tile_xyz(a.t, id, tx, ty, tz);
    stage_halo<D, CIN>(hs, a.in, a.t, tx, ty, tz);
    cp_wait_all();
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after();
      uint32_t acc = 0;
      for (int tap = 0; tap < TAPS; ++tap) {
        const uint32_t aoff = tap_off<D>(tap);
#pragma unroll
        for (int kh = 0; kh < CIN / 16; ++kh) {
          // A: rows = 8 x-nodes (16 B apart) x 16 y-rows (kHyB apart), K chunks CHB apart
          const uint64_t ad = umma::make_desc(hb + aoff + 2 * kh * CHB, CHB, kHyB);
          // B: the tap's COUT x CIN weights, K chunks 128 B apart, 8-row groups (CIN/8)*128 apart
          const uint64_t bd = umma::make_desc(wb + tap * WTAP + kh * 256, 128, (CIN / 8) * 128);
          umma::mma_bf16(tmem, ad, bd, IDESC, acc);
          acc = 1;
        }
      }
      umma::mma_commit(&bar);
    }
    const bool ok = umma::mbar_wait(&bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) { failed = true; break; }
    umma::fence_after();
    float v[COUT];
    umma::tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16), v);
    const int r = warp * 32 + lane;
    conv_epilogue<D, COUT, EPI>(a, v, tx * TX + (r & 7), ty * TY + (r >> 3), tz);
    umma::fence_before();  // the loads above precede the next tile's MMAs (barrier at the loop top)
  }
  if (failed) {
    if (tid == 0) atomicOr(a.err, 1u);
    umma::mbar_wait(&bar, phase ^ 1u);  // bounded: let the tile's MMAs drain before freeing
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after();
    umma::tmem_dealloc(tmem, 32);
  }
}

// ---- 3D convolution marching along z
// A CTA owns the 8 x 16 column (tx, ty) over kSeg output planes z0 .. z0+S-1
// and walks the input planes P = z0 .. z0+S+1 (padded plane numbers) once
// each.  Input plane P feeds output planes P, P-1, P-2 through the weight
// slices dz = 0, 1, 2, so one MMA per (xy tap, K step) multiplies the plane's
// shifted halo (A, M = 128 nodes) by the three slices side by side (B, N =
// 3 COUT rows) into three accumulators: output z's COUT columns sit at
// col(z) = COUT (kSeg - 1 - (z - z0)), descending in z, so the slices dz of
// plane P land at col(P - dz) = col(P) + dz COUT, one contiguous N range.
// Slices whose output plane lies outside the segment are dropped from the
// ends of that range.  An output plane's first product (plane P = z, dz = 0,
// first tap) is issued on its own with accumulate off.
//   Per input plane the A tile is read 9 (CIN / 16) + 1 times instead of
// 27 (CIN / 16) times, which is what bounds the single-plane form (an
// M = 128, N = COUT MMA reads 4 KB of A from shared memory per K step).
// Pipeline: the halo planes sit in a ring of kRing slots; plane P + 2 is
// loaded (cp.async) while plane P is multiplied, and output plane P - 3 is
// read out of tensor memory and stored while the MMAs of plane P run (two
// mbarriers, one per plane parity, each with at most one commit pending).
constexpr int kSeg = 8;    // output planes per work item
constexpr int kRing = 4;   // halo plane slots
constexpr int kSlotB = (kPlaneB + 127) / 128 * 128;  // 2944: ring slots 128-byte aligned (TMA destinations)

template <int CIN, int COUT>
struct Z3 {
  static constexpr int CHB = kRing * kSlotB;       // one 8-channel chunk of the ring
  static constexpr int RING = (CIN / 8) * CHB;
  static constexpr int WTAP = 3 * COUT * CIN * 2;  // one xy tap: the dz = 0, 1, 2 slices, K-major
  static constexpr int WBYTES = 9 * WTAP;
  static constexpr int SMEM = WBYTES + RING;
  static constexpr uint32_t TCOLS = kSeg * COUT;   // 128 or 256 tensor-memory columns
};

// weights [27 taps][COUT][CIN] (tap = dx + 3 dy + 9 dz) -> per xy tap t a
// K-major (3 COUT) x CIN tile whose row dz COUT + co holds tap t + 9 dz
// (defined after the thread count of the kernel that stages them)

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Warp roles: warp 4's first lane is the producer -- it issues, per input
// plane, CIN/8 tiled TMA copies of the (8 channels) x 10 x 18 box of the
// activation tensor [z][y][x][C] (viewed as 5D: 8 channels, C/8 chunks, x, y,
// z; nodes beyond the array read as zeros) into the plane's ring slot,
// completing on that slot's mbarrier, waits for the plane (bounded) and
// issues its MMAs, committing them to the plane's mbarrier mb[k] (k the
// plane's index in the work item).  Warps 0-3 (one tensor-memory lane
// quadrant each) only run the epilogue: output plane j of the item is
// complete once the MMAs of input plane j + 2 are, so they wait mb[j + 2] and
// read the plane's accumulators, while the producer's copies and MMAs for the
// planes after it go on.  The producer refills a ring slot once the MMAs of
// the plane that read it are done (mb[k - 2]).  One block barrier per work
// item orders the epilogue's tensor-memory reads before the next item's MMAs
// (which reuse the columns); before it the producer waits every commit of
// the item, so each mbarrier's phases complete strictly in turn.
constexpr int kZThreads = 160;

template <int CIN, int COUT>
__device__ __forceinline__ void stage_weights_z3(uint8_t* ws, const bf16* __restrict__ w) {
  constexpr int CH = CIN / 8, R = 3 * COUT;
  for (int idx = threadIdx.x; idx < 9 * R * CH; idx += kZThreads) {
    const int c = idx % CH, row = (idx / CH) % R, t = idx / (CH * R);
    const int dz = row / COUT, co = row - dz * COUT;
    cp16(ws + t * Z3<CIN, COUT>::WTAP + umma::kmajor_offset(row, c * 8, CIN),
         reinterpret_cast<const uint4*>(w + ((long long)(t + 9 * dz) * COUT + co) * CIN) + c, true);
  }
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kZThreads) k_conv3z(ConvArgs a, const __grid_constant__ CUtensorMap tin) {
  using Z = Z3<CIN, COUT>;
  constexpr uint32_t kPlaneTx = (CIN / 8) * kPlaneB;  // bytes of one plane's copies
  constexpr int NP = kSeg + 2;                        // input planes of a full work item
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* ws = smem;
  uint8_t* hs = smem + Z::WBYTES;
  __shared__ __align__(8) uint64_t mb[NP];
  __shared__ __align__(8) uint64_t full[kRing];
  __shared__ uint32_t tslot;
  __shared__ int halo_timeout;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool producer = warp == 4 && lane == 0;
  const TileGeo& t = a.t;
  const int nseg = (t.Mz + kSeg - 1) / kSeg;
  const long long items = (long long)t.ntx * t.nty * nseg;

  stage_weights_z3<CIN, COUT>(ws, a.w);
  cp_commit();
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  umma::fence_async_smem();  // the staged weights -> the tensor core's proxy
  if (warp == 0) umma::tmem_alloc(&tslot, Z::TCOLS);
  if (tid == 0) {
    for (int i = 0; i < NP; ++i) umma::mbar_init(&mb[i]);
    for (int i = 0; i < kRing; ++i) umma::mbar_init(&full[i]);
    halo_timeout = 0;
  }
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const uint32_t hb = umma::smem_u32(hs), wb = umma::smem_u32(ws);
  uint32_t mphase = 0u;  // bit k: parity of the phase of mb[k] this item's commit completes (every thread)
  uint32_t fphase = 0u;  // producer, bit s: parity of full[s]'s next phase
  uint32_t fpend = 0u;   // producer, bit s: a plane load on full[s] not yet waited for
  bool failed = false;
  int tx = 0, ty = 0;
  auto load_plane = [&](int P) {  // the producer
    const int sl = P % kRing;
    umma::mbar_arrive_expect_tx(&full[sl], kPlaneTx);
    uint8_t* dst = hs + sl * kSlotB;
    for (int c = 0; c < CIN / 8; ++c) umma::tma_load_5d(dst + c * Z::CHB, &tin, &full[sl], 0, c, tx * TX, ty * TY, P);
    fpend |= 1u << sl;
  };
  for (long long id = blockIdx.x; id < items; id += gridDim.x) {
    tx = (int)(id % t.ntx);
    const long long rest = id / t.ntx;
    ty = (int)(rest % t.nty);
    const int z0 = (int)(rest / t.nty) * kSeg;
    const int S = min(kSeg, t.Mz - z0);
    const int nplanes = S + 2;  // padded input planes z0 .. z0+S+1
    if (producer) {
      load_plane(z0);
      load_plane(z0 + 1);
      for (int k = 0; k < nplanes; ++k) {
        const int P = z0 + k;
        if (k + 2 < nplanes) {
          // the slot of plane P + 2 was last read by the MMAs of plane P - 2
          // (of this item; those of the item before are all done by now)
          if (k >= 2 && !umma::mbar_wait(&mb[k - 2], (mphase >> (k - 2)) & 1u)) failed = true;
          load_plane(P + 2);
        }
        const int sl = P % kRing;
        const bool landed = umma::mbar_wait(&full[sl], (fphase >> sl) & 1u);
        if (landed) {
          fphase ^= 1u << sl;
          fpend &= ~(1u << sl);
        } else {
          halo_timeout = 1;
        }
        umma::fence_after();
        if (landed && !failed) {
          const int dlo = max(0, P - (z0 + S - 1)), dhi = min(2, P - z0);
          const uint32_t dcol = tmem + (uint32_t)(COUT * (kSeg - 1 - (P - dlo - z0)));
          const uint32_t aslot = hb + (uint32_t)(sl * kSlotB);
          const uint32_t idesc = umma::idesc_bf16(128, (dhi - dlo + 1) * COUT, false, false);
          const uint32_t brow = (uint32_t)(dlo * (COUT / 8) * (CIN / 8) * 128);  // row dlo COUT of the B tile
          bool first = dlo == 0;  // this plane opens output plane P
          for (int tap = 0; tap < 9; ++tap) {
            const uint32_t aoff = (uint32_t)((tap / 3) * kHyB + (tap % 3) * kRowB);
#pragma unroll
            for (int kh = 0; kh < CIN / 16; ++kh) {
              // A: 8 x-nodes 16 B apart x 16 y-rows kHyB apart, K chunks CHB apart
              const uint64_t ad = umma::make_desc(aslot + aoff + 2 * kh * Z::CHB, Z::CHB, kHyB);
              const uint32_t wt = wb + tap * Z::WTAP + kh * 256;
              if (first) {
                // output P alone (slice dz = 0, N = COUT) with accumulate off, then the other slices
                umma::mma_bf16(dcol, ad, umma::make_desc(wt, 128, (CIN / 8) * 128),
                               umma::idesc_bf16(128, COUT, false, false), 0u);
                if (dhi > 0)
                  umma::mma_bf16(dcol + COUT, ad,
                                 umma::make_desc(wt + (COUT / 8) * (CIN / 8) * 128, 128, (CIN / 8) * 128),
                                 umma::idesc_bf16(128, dhi * COUT, false, false), 1u);
                first = false;
              } else {
                umma::mma_bf16(dcol, ad, umma::make_desc(wt + brow, 128, (CIN / 8) * 128), idesc, 1u);
              }
            }
          }
        }
        umma::mma_commit(&mb[k]);  // also when nothing was issued: every commit is waited for
      }
      // every commit of the item done before the block barrier: each mbarrier
      // then completes its phases strictly in turn
      for (int k = 0; k < nplanes; ++k)
        if (!umma::mbar_wait(&mb[k], (mphase >> k) & 1u)) failed = true;
    } else if (warp < 4) {
      for (int j = 0; j < S; ++j) {
        if (!umma::mbar_wait(&mb[j + 2], (mphase >> (j + 2)) & 1u)) failed = true;
        umma::fence_after();
        if (!failed) {
          float v[COUT];
          umma::tmem_ld<COUT>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(COUT * (kSeg - 1 - j)), v);
          const int r = warp * 32 + lane;
          conv_epilogue<3, COUT, EPI>(a, v, tx * TX + (r & 7), ty * TY + (r >> 3), z0 + j);
        }
      }
    }
    mphase ^= (1u << nplanes) - 1u;
    umma::fence_before();  // the tensor-memory reads above precede the next item's MMAs
    const bool stop = __syncthreads_or(failed || halo_timeout != 0);
    umma::fence_after();
    if (stop) {
      failed = true;
      break;
    }
  }
  if (failed) {
    if (tid == 0) atomicOr(a.err, 1u);
    if (producer)  // bounded: no copy may still be landing when the CTA exits
      for (int sl = 0; sl < kRing; ++sl)
        if ((fpend >> sl) & 1u) umma::mbar_wait(&full[sl], (fphase >> sl) & 1u);
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after();
    umma::tmem_dealloc(tmem, Z::TCOLS);
  }
}

struct WgradArgs {
  TileGeo t;
  const bf16* g;   // [npad][CG] gradient at the layer's output
  const bf16* x;   // [npad][CX] the layer's input
  float* part;     // [gridDim.x][TAPS][CG][CX]
  unsigned* err;
};

constexpr int kWgTaps = 8;  // taps per CTA: one block of tensor-memory columns each

template <int D, int CG, int CX>
__global__ void __launch_bounds__(kThreads) k_wgrad(WgradArgs a) {
  constexpr int TAPS = Tp<D>::TAPS, CHB = Tp<D>::CHB;
  constexpr int GCH = TY * 128;  // one 8-channel chunk of the gradient tile (16 y-rows of 8 nodes)
  constexpr uint32_t IDESC = umma::idesc_bf16(64, CX, true, true);
  constexpr uint32_t TCOLS = kWgTaps * CX;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* gs = smem;            // 8 chunks (M = 64); chunks >= CG/8 stay zero
  uint8_t* hs = smem + 8 * GCH;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tap0 = blockIdx.y * kWgTaps;
  const int nt = min(kWgTaps, TAPS - tap0);

  for (int i = tid; i < (8 - CG / 8) * GCH / 16; i += kThreads)
    reinterpret_cast<uint4*>(gs + (CG / 8) * GCH)[i] = make_uint4(0u, 0u, 0u, 0u);
  if (warp == 0) umma::tmem_alloc(&tslot, TCOLS);
  if (tid == 0) umma::mbar_init(&bar);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const uint32_t gb = umma::smem_u32(gs), hb = umma::smem_u32(hs);
  uint32_t phase = 0;
  bool failed = false, any = false;
  for (long long id = blockIdx.x; id < a.t.ntiles; id += gridDim.x) {
    int tx, ty, tz;
    tile_xyz(a.t, id, tx, ty, tz);
    for (int idx = tid; idx < (CG / 8) * 128; idx += kThreads) {
      const int c = idx >> 7, r = idx & 127, x = r & 7, y = r >> 3;
      const int ix = tx * TX + x, iy = ty * TY + y;
      const bool ok = ix < a.t.Mx && iy < a.t.My;
      const long long p = ok ? pad_index<D>(a.t, ix, iy, tz) : 0;
      cp16(gs + c * GCH + y * 128 + x * 16, reinterpret_cast<const uint4*>(a.g + p * CG) + c, ok);
    }
    stage_halo<D, CX>(hs, a.x, a.t, tx, ty, tz);
    cp_wait_all();
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after();
      for (int j = 0; j < nt; ++j) {
        const uint32_t boff = tap_off<D>(tap0 + j);
#pragma unroll
        for (int kk = 0; kk < TY / 2; ++kk) {  // K = 16 nodes: y-rows 2kk, 2kk+1
          // A = G^T (M = channels, MN-major): K groups (y-rows) 128 B apart, channel chunks GCH apart
          const uint64_t ad = umma::make_desc(gb + kk * 256, 128, GCH);
          // B = shifted halo (N = channels, MN-major): K groups kHyB apart, channel chunks CHB apart
          const uint64_t bd = umma::make_desc(hb + boff + 2 * kk * kHyB, kHyB, CHB);
          umma::mma_bf16(tmem + j * CX, ad, bd, IDESC, (any || kk > 0) ? 1u : 0u);
        }
      }
      umma::mma_commit(&bar);
    }
    const bool ok = umma::mbar_wait(&bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) { failed = true; break; }
    any = true;
  }
  if (failed) {
    if (tid == 0) atomicOr(a.err, 1u);
    umma::mbar_wait(&bar, phase ^ 1u);
  } else {
    umma::fence_after();
    float* dst = a.part + (long long)blockIdx.x * TAPS * CG * CX;
    if (warp < 2) {  // M = 64: row m lives in lane (m % 16) + 32 (m / 16)
      const int m = warp * 16 + lane;
      for (int j = 0; j < nt; ++j) {
        float v[CX];
        umma::tmem_ld<CX>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * CX), v);
        if (lane < 16 && m < CG) {
          float* o = dst + ((long long)(tap0 + j) * CG + m) * CX;
#pragma unroll
          for (int c = 0; c < CX; ++c) o[c] = any ? v[c] : 0.f;
        }
      }
    }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after();
    umma::tmem_dealloc(tmem, TCOLS);
  }
}

// out[tap][co][ci] += sum over s of part[s][tap][co][ci], co < nco, fixed order
__global__ void k_wgrad_reduce(const float* __restrict__ part, int S, int taps, int CG, int CX, int nco,
                               float* __restrict__ out) {
  const long long n = (long long)taps * nco * CX;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(k % CX);
    const long long r = k / CX;
    const int co = (int)(r % nco), tap = (int)(r / nco);
    float s = 0.f;
    for (int q = 0; q < S; ++q) s += part[(((long long)q * taps + tap) * CG + co) * CX + ci];
    out[k] += s;
  }
}

// zero the ghost layer of an activation buffer laid out for t (buffers are
// shared between levels, so the ghost nodes of a smaller level may hold data)
template <int D>
__global__ void k_zero_ghosts(TileGeo t, int chunks, uint4* __restrict__ buf) {
  // ghost nodes only: the two z faces (3D), then the ring of every other plane
  const long long face = (long long)t.Px * t.Py;
  const long long g1 = D == 3 ? 2 * face : 0;
  const int ring = 2 * t.Px + 2 * (t.Py - 2);
  const long long nghost = g1 + (long long)(D == 3 ? t.Pz - 2 : t.Pz) * ring;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < nghost * chunks;
       g += (long long)gridDim.x * blockDim.x) {
    const long long node = g / chunks;
    const int c = (int)(g - node * chunks);
    long long p;
    if (node < g1) {
      p = (node >= face ? (long long)(t.Pz - 1) * face : 0) + node % face;
    } else {
      const long long r0 = node - g1;
      const long long pz = r0 / ring + (D == 3 ? 1 : 0);
      const int r = (int)(r0 % ring);
      int x, y;
      if (r < t.Px) { x = r; y = 0; }
      else if (r < 2 * t.Px) { x = r - t.Px; y = t.Py - 1; }
      else { const int r2 = r - 2 * t.Px; y = 1 + (r2 >> 1); x = (r2 & 1) ? t.Px - 1 : 0; }
      p = pz * face + (long long)y * t.Px + x;
    }
    buf[p * chunks + c] = make_uint4(0u, 0u, 0u, 0u);
  }
}

template <int D>
void zero_ghosts(const TileGeo& t, int C, bf16* buf, cudaStream_t st) {
  const long long face = (long long)t.Px * t.Py;
  const long long n = ((D == 3 ? 2 * face : 0) + (long long)(D == 3 ? t.Pz - 2 : t.Pz) * (2 * t.Px + 2 * (t.Py - 2))) *
                      (C / 8);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_zero_ghosts<D><<<(unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8192)), 256, 0, st>>>(
      t, C / 8, reinterpret_cast<uint4*>(buf));
}

// per-block channel sums of [npad][C] -> part[block][C]
template <int C>
__global__ void __launch_bounds__(256) k_colsum(const bf16* __restrict__ g, long long npad, float* __restrict__ part) {
  constexpr int J = 256 / C;
  __shared__ float s[256];
  const int c = threadIdx.x % C, j = threadIdx.x / C;
  float acc = 0.f;
  for (long long p = (long long)blockIdx.x * J + j; p < npad; p += (long long)gridDim.x * J)
    acc += __bfloat162float(g[p * C + c]);
  s[threadIdx.x] = acc;
  __syncthreads();
  if (j == 0) {
    float t = 0.f;
    for (int q = 0; q < J; ++q) t += s[q * C + c];
    part[(long long)blockIdx.x * C + c] = t;
  }
}

__global__ void k_colsum_final(const float* __restrict__ part, int nb, int C, int nout, float* __restrict__ out) {
  const int c = threadIdx.x;
  if (c >= nout) return;
  float t = 0.f;
  for (int b = 0; b < nb; ++b) t += part[(long long)b * C + c];
  out[c] += t;
}

// dZ (16 channels, channel 0 used) from dL/domega: dL/dz = g (w - wmin)(wmax - w)/(wmax - wmin)
template <int D>
__global__ void k_dz(TileGeo t, const double* __restrict__ gw, const double* __restrict__ w, float omin, float omax,
                     bf16* __restrict__ dz) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)t.Mx * t.My * t.Mz) return;
  const int ix = (int)(i % t.Mx), iy = (int)((i / t.Mx) % t.My), iz = (int)(i / ((long long)t.Mx * t.My));
  const double om = w[i];
  const float d = (float)(gw[i] * (om - omin) * (omax - om) / (double)(omax - omin));
  uint4* o = reinterpret_cast<uint4*>(dz + pad_index<D>(t, ix, iy, iz) * kNetOut);
  o[0] = make_uint4(pack2(d, 0.f), 0u, 0u, 0u);
  o[1] = make_uint4(0u, 0u, 0u, 0u);
}

// FP32 parameters -> BF16 forward weights and flipped/transposed backward weights
__global__ void k_net_weights(const float* __restrict__ P, NetLayout L, bf16* wf1, bf16* wf2, bf16* wf3, bf16* wb2,
                              bf16* wb3) {
  const long long T = L.taps;
  const long long n1 = T * kNetHid * kNetIn, n2 = T * kNetHid * kNetHid, n3 = T * kNetOut * kNetHid;
  const long long nb2 = n2, nb3 = T * kNetHid * kNetOut;
  const long long tot = n1 + n2 + n3 + nb2 + nb3;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
    long long q = k;
    if (q < n1) { wf1[q] = __float2bfloat16_rn(P[L.w1 + q]); continue; }
    q -= n1;
    if (q < n2) { wf2[q] = __float2bfloat16_rn(P[L.w2 + q]); continue; }
    q -= n2;
    if (q < n3) {  // [tap][co 16][ci 32]
      const int ci = (int)(q % kNetHid), co = (int)((q / kNetHid) % kNetOut), tap = (int)(q / (kNetHid * kNetOut));
      wf3[q] = __float2bfloat16_rn(co == 0 ? P[L.w3 + (long long)tap * kNetHid + ci] : 0.f);
      continue;
    }
    q -= n3;
    if (q < nb2) {  // [tap][o = ci of W2][i = co of W2] = W2[flip][co][ci]
      const int i = (int)(q % kNetHid), o = (int)((q / kNetHid) % kNetHid), tap = (int)(q / (kNetHid * kNetHid));
      const long long ft = T - 1 - tap;
      wb2[q] = __float2bfloat16_rn(P[L.w2 + (ft * kNetHid + i) * kNetHid + o]);
      continue;
    }
    q -= nb2;
    {  // [tap][o = ci of W3 (32)][i (16)]: i = 0 carries W3[flip][ci]
      const int i = (int)(q % kNetOut), o = (int)((q / kNetOut) % kNetHid), tap = (int)(q / (kNetOut * kNetHid));
      const long long ft = T - 1 - tap;
      wb3[q] = __float2bfloat16_rn(i == 0 ? P[L.w3 + ft * kNetHid + o] : 0.f);
    }
  }
}

__global__ void k_adam(float* __restrict__ P, float* __restrict__ G, float* __restrict__ Mo, float* __restrict__ Vo,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = b1 * Mo[i] + (1.f - b1) * g;
  const float v = b2 * Vo[i] + (1.f - b2) * g * g;
  Mo[i] = m;
  Vo[i] = v;
  P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  G[i] = 0.f;
}

// raw[i] = log k[i] and a deterministic sum of them: per-block partials (a
// fixed grid of eight blocks per SM of a B200, so the FP64 logarithms of all
// SMs overlap) then one block
__global__ void __launch_bounds__(kBlock) k_logsum(const double* __restrict__ k, long long n, double* __restrict__ raw,
                                                   double* __restrict__ part) {
  __shared__ double sm[8];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock) {
    const double l = log(k[i]);
    raw[i] = l;
    acc += l;
  }
  const double s = dr_fold256(acc, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kBlock) k_logmean_final(const double* __restrict__ part, int nb, long long n,
                                                          double* __restrict__ out) {
  __shared__ double sm[8];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nb; b += kBlock) acc += part[b];
  const double s = dr_fold256(acc, sm);
  if (threadIdx.x == 0) *out = s / (double)n;
}

__global__ void k_set_scalar(double* p, double v) { *p = v; }

__global__ void k_ratio_acc(double* scal, int dst, int num, int den, double factor, int first) {
  const double r = factor * scal[num] / scal[den];
  scal[dst] = first ? r : scal[dst] + r;
}

// a cell's input to the network: its mean log-coefficient lk, centred by the
// top level's mean log k, halved and clamped to [-8, 8]
__device__ __forceinline__ float cell_feature(double lk, double mu) {
  return (float)fmin(fmax((lk - mu) * 0.5, -8.0), 8.0);
}

// log-coefficient of every cell of one Q1 level: the mean of log k over the
// cell's np^D Gauss points xi, k being the top level's cell coefficient
// (ratio = n_top / n_l fine cells per level cell and direction).  Consecutive
// points in one fine cell reuse its logarithm (the same value the sum would
// add again), so the top level costs one log per cell; with lraw (log k of
// every top-level cell, taken with the mean) no level takes a logarithm.
// Written: the cell's feature value (cell_feature), once per cell rather than
// once per adjacent node.
template <int D>
__global__ void k_cell_logk(int n_l, long long n_top, double ratio, int np, const double* __restrict__ xi,
                            const double* __restrict__ kcell, const double* __restrict__ lraw,
                            const double* __restrict__ mean, float* __restrict__ fc) {
  long long nc = n_l;
  for (int k = 1; k < D; ++k) nc *= n_l;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const unsigned cu = (unsigned)c, nu = (unsigned)n_l;  // nc < 2^32 (checked by the launcher)
  const int cc[3] = {(int)(cu % nu), (int)((cu / nu) % nu), D == 3 ? (int)(cu / (nu * nu)) : 0};
  int nq = 1;
  for (int k = 0; k < D; ++k) nq *= np;
  if (ratio == 1.0) {  // every Gauss point lies in the cell itself (0 < xi < 1)
    const double l1 = lraw ? lraw[c] : log(kcell[c]);
    double s1 = 0.0;
    for (int q = 0; q < nq; ++q) s1 += l1;
    fc[c] = cell_feature(s1 / nq, *mean);
    return;
  }
  double s = 0.0, lv = 0.0;
  long long last = -1;
  for (int q = 0; q < nq; ++q) {
    const int qi[3] = {q % np, (q / np) % np, q / (np * np)};
    long long fi[3] = {0, 0, 0};
    for (int k = 0; k < D; ++k) fi[k] = (long long)floor(((double)cc[k] + xi[qi[k]]) * ratio);
    const long long idx = fi[0] + n_top * (fi[1] + n_top * fi[2]);
    if (idx != last) {
      lv = lraw ? __ldg(lraw + idx) : log(kcell[idx]);
      last = idx;
    }
    s += lv;
  }
  fc[c] = cell_feature(s / nq, *mean);
}

// node features of one Q1 level from the level's cell feature values fc
// (null: every cell the value of the constant log kconst); blockIdx.y is the
// node plane
template <int D>
__global__ void k_features(TileGeo t, int n_l, int sub, const float* __restrict__ fc, double kconst,
                           const double* __restrict__ mean, bf16* __restrict__ X0) {
  const unsigned iu = blockIdx.x * blockDim.x + threadIdx.x, mx = (unsigned)t.Mx;
  if (iu >= mx * (unsigned)t.My) return;
  const int iy = (int)(iu / mx), ix = (int)(iu - (unsigned)iy * mx), iz = D == 3 ? (int)blockIdx.y : 0;
  const int node[3] = {ix, iy, iz};
  constexpr int NC = 1 << D;
  const float fconst = fc ? 0.f : cell_feature(log(kconst), *mean);
  float f[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) f[c] = 0.f;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    int cc[3] = {0, 0, 0};
    bool in = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {  // adjacent cell (sub = 2: half-cell of a Q2 node, then its cell)
      const int h = node[k] - 1 + ((c >> k) & 1);
      in = in && h >= 0 && h < n_l * sub;
      cc[k] = sub == 1 ? h : (sub == 2 ? h >> 1 : h / sub);  // h >= 0 wherever cc is used
    }
    if (!in) continue;
    f[c] = fc ? __ldg(fc + cc[0] + (long long)n_l * (cc[1] + (long long)n_l * cc[2])) : fconst;
    f[NC + c] = 1.f;
  }
  uint4* o = reinterpret_cast<uint4*>(X0 + pad_index<D>(t, ix, iy, iz) * kNetIn);
  o[0] = make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
  o[1] = make_uint4(pack2(f[8], f[9]), pack2(f[10], f[11]), pack2(f[12], f[13]), pack2(f[14], f[15]));
}

// ----------------------------------------------------- FP64 loss helpers
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_rand_fill(double* e, int D, long long M, int dmask, int nc, unsigned long long seed) {
  long long N = M;
  for (int k = 1; k < D; ++k) N *= M;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // entry nc i + component
  if (t >= N * nc) return;
  const long long i = t / nc;
  const long long c[3] = {i % M, D > 1 ? (i / M) % M : 0, D > 2 ? i / (M * M) : 0};
  bool dir = false;
  for (int k = 0; k < D; ++k) {
    if (c[k] == 0 && ((dmask >> (2 * k)) & 1)) dir = true;
    if (c[k] == M - 1 && ((dmask >> (2 * k + 1)) & 1)) dir = true;
  }
  const unsigned long long h = mix64(seed * 0x100000001B3ull ^ (unsigned long long)t);
  e[t] = dir ? 0.0 : (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

__global__ void k_dinv(const double* __restrict__ A, long long Np, const double* __restrict__ u, double* __restrict__ v,
                       long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = u[i] / A[i];
}

__global__ void k_sub_wv(const double* __restrict__ x, const double* __restrict__ w, const double* __restrict__ v,
                         double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] - (w ? w[i] * v[i] : v[i]);
}

__global__ void k_gomega(const double* __restrict__ g, const double* __restrict__ v, double* __restrict__ gw,
                         int accumulate, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) gw[i] = (accumulate ? gw[i] : 0.0) - g[i] * v[i];
}

__global__ void k_wg_dinv(const double* __restrict__ A, const double* __restrict__ w, const double* __restrict__ g,
                          double* __restrict__ t, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) t[i] = w[i] * g[i] / A[i];
}

__global__ void k_scale_by(const double* __restrict__ x, double s, const double* __restrict__ scal, int slot,
                           double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = s * x[i] / scal[slot];
}

// y = x + w .* v  (y may be x)
__global__ void k_xpwv(const double* x, const double* __restrict__ w, const double* __restrict__ v, double* y,
                       long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] + w[i] * v[i];
}

// acc += a .* b
__global__ void k_acc_prod(double* __restrict__ acc, const double* __restrict__ a, const double* __restrict__ b,
                           long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] += a[i] * b[i];
}

// y += w .* x / diag(A)
__global__ void k_wg_dinv_acc(const double* __restrict__ A, const double* __restrict__ w, const double* __restrict__ x,
                              double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += w[i] * x[i] / A[i];
}

__global__ void k_add(const double* __restrict__ x, double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

inline unsigned blocks_for(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// the activation tensor [Pz][Py][Px][C] (BF16) as the 5D TMA view (8
// channels, C/8 chunks, x, y, z) with a box of one chunk over the 10 x 18 halo
// of one plane; nodes beyond the array are read as zeros
bool act_tensor_map(const bf16* base, int C, const TileGeo& t, CUtensorMap* out) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[5] = {8, (cuuint64_t)(C / 8), (cuuint64_t)t.Px, (cuuint64_t)t.Py, (cuuint64_t)t.Pz};
  const cuuint64_t strides[4] = {16, (cuuint64_t)C * 2, (cuuint64_t)t.Px * C * 2, (cuuint64_t)t.Py * t.Px * C * 2};
  const cuuint32_t box[5] = {8, 1, (cuuint32_t)HX, (cuuint32_t)HY, 1};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return encode(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(base), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int D, int CIN, int COUT, int EPI>
int conv(const ConvArgs& a, cudaStream_t st) {
  if constexpr (D == 3) {
    constexpr size_t smem = Z3<CIN, COUT>::SMEM;
    static bool init3 = false;
    if (!init3) {
      cudaFuncSetAttribute(k_conv3z<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      init3 = true;
    }
    CUtensorMap tin;
    if (!act_tensor_map(a.in, CIN, a.t, &tin)) return FMG_ERR_CUDA;
    const long long items = (long long)a.t.ntx * a.t.nty * ((a.t.Mz + kSeg - 1) / kSeg);
    const long long grid = std::min<long long>(items, 2LL * sm_count());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_conv3z<CIN, COUT, EPI><<<(unsigned)std::max<long long>(grid, 1), kZThreads, smem, st>>>(a, tin);
  } else {
    constexpr size_t smem = (size_t)Tp<D>::TAPS * COUT * CIN * 2 + (size_t)(CIN / 8) * Tp<D>::CHB;
    static bool init = false;
    if (!init) {
      cudaFuncSetAttribute(k_conv<D, CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      init = true;
    }
    const long long grid = std::min<long long>(a.t.ntiles, 2LL * sm_count());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_conv<D, CIN, COUT, EPI><<<(unsigned)std::max<long long>(grid, 1), kThreads, smem, st>>>(a);
  }
  return FMG_OK;
}

template <int D, int CG, int CX>
int wgrad(fmg_net* net, const TileGeo& t, const bf16* g, const bf16* x, long long w_off, int nco, cudaStream_t st) {
  constexpr int TAPS = Tp<D>::TAPS;
  constexpr size_t smem = (size_t)8 * TY * 128 + (size_t)(CX / 8) * Tp<D>::CHB;
  static bool init = false;
  if (!init) {
    cudaFuncSetAttribute(k_wgrad<D, CG, CX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    init = true;
  }
  const int groups = (TAPS + kWgTaps - 1) / kWgTaps;
  const long long S = std::max<long long>(1, std::min<long long>(t.ntiles, (2LL * sm_count()) / groups));
  const long long need = std::max<long long>(S * TAPS * CG * CX, 256LL * kNetHid);  // colsum partials too
  if (need > net->part_cap) {
    if (net->part) { cudaStreamSynchronize(st); cudaFree(net->part); net->part = nullptr; net->part_cap = 0; }
    if (cudaMalloc(&net->part, (size_t)need * sizeof(float)) != cudaSuccess) { cudaGetLastError(); return FMG_ERR_NOMEM; }
    net->part_cap = need;
  }
  WgradArgs a;
  a.t = t; a.g = g; a.x = x; a.part = net->part; a.err = net->err;
  g_launches.fetch_add(2, std::memory_order_relaxed);
  k_wgrad<D, CG, CX><<<dim3((unsigned)S, (unsigned)groups), kThreads, smem, st>>>(a);
  const long long nout = (long long)TAPS * nco * CX;
  k_wgrad_reduce<<<blocks_for(nout), 256, 0, st>>>(net->part, (int)S, TAPS, CG, CX, nco, net->G + w_off);
  return FMG_OK;
}

template <int C>
void colsum(fmg_net* net, const bf16* g, long long npad, long long b_off, int nout, cudaStream_t st) {
  const int nb = 256;
  // the partials use the head of the weight-gradient scratch (reserved by wgrad first)
  g_launches.fetch_add(2, std::memory_order_relaxed);
  k_colsum<C><<<nb, 256, 0, st>>>(g, npad, net->part);
  k_colsum_final<<<1, 32, 0, st>>>(net->part, nb, C, nout, net->G + b_off);
}

template <int D>
int forward_d(fmg_net* net, const ActGeom& g, double* omega, cudaStream_t st) {
  const TileGeo t = tile_geo(g);
  const NetLayout& L = net->lay;
  zero_ghosts<D>(t, kNetIn, net->X0, st);
  zero_ghosts<D>(t, kNetHid, net->H1, st);
  zero_ghosts<D>(t, kNetHid, net->H2, st);
  ConvArgs a{};
  a.t = t; a.err = net->err; a.omin = net->omega_min; a.omax = net->omega_max;
  int rc;
  a.in = net->X0; a.w = net->wf1; a.bias = net->P + L.b1; a.out = net->H1;
  if ((rc = conv<D, kNetIn, kNetHid, EPI_RELU>(a, st))) return rc;
  a.in = net->H1; a.w = net->wf2; a.bias = net->P + L.b2; a.out = net->H2;
  if ((rc = conv<D, kNetHid, kNetHid, EPI_RELU>(a, st))) return rc;
  if (omega) {
    a.in = net->H2; a.w = net->wf3; a.bias = net->P + L.b3; a.out = nullptr; a.omega = omega;
    if ((rc = conv<D, kNetHid, kNetOut, EPI_OMEGA>(a, st))) return rc;
  }
  return FMG_OK;
}

template <int D>
int backward_d(fmg_net* net, const double* gomega, const double* omega, cudaStream_t st) {
  const ActGeom& g = net->geom;
  const TileGeo t = tile_geo(g);
  const NetLayout& L = net->lay;
  const long long npad = g.npad();
  int rc;
  zero_ghosts<D>(t, kNetOut, net->dZ, st);
  zero_ghosts<D>(t, kNetHid, net->dP2, st);
  zero_ghosts<D>(t, kNetHid, net->dP1, st);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dz<D><<<blocks_for(g.nodes()), 256, 0, st>>>(t, gomega, omega, net->omega_min, net->omega_max, net->dZ);
  // layer 3: dW3 = sum dZ (x) H2_shift, db3 = sum dZ
  if ((rc = wgrad<D, kNetOut, kNetHid>(net, t, net->dZ, net->H2, L.w3, 1, st))) return rc;
  colsum<kNetOut>(net, net->dZ, npad, L.b3, 1, st);
  ConvArgs a{};
  a.t = t; a.err = net->err;
  a.in = net->dZ; a.w = net->wb3; a.mask = net->H2; a.out = net->dP2;
  if ((rc = conv<D, kNetOut, kNetHid, EPI_MASK>(a, st))) return rc;
  // layer 2
  if ((rc = wgrad<D, kNetHid, kNetHid>(net, t, net->dP2, net->H1, L.w2, kNetHid, st))) return rc;
  colsum<kNetHid>(net, net->dP2, npad, L.b2, kNetHid, st);
  a.in = net->dP2; a.w = net->wb2; a.mask = net->H1; a.out = net->dP1;
  if ((rc = conv<D, kNetHid, kNetHid, EPI_MASK>(a, st))) return rc;
  // layer 1
  if ((rc = wgrad<D, kNetHid, kNetIn>(net, t, net->dP1, net->X0, L.w1, kNetHid, st))) return rc;
  colsum<kNetHid>(net, net->dP1, npad, L.b1, kNetHid, st);
  return FMG_OK;
}

}  // namespace

int net_alloc(fmg_net* net, void** p, size_t bytes) {
  void* q = nullptr;
  if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) {
    cudaGetLastError();
    return FMG_ERR_NOMEM;
  }
  if (cudaMemset(q, 0, bytes ? bytes : 16) != cudaSuccess) {
    cudaFree(q);
    return FMG_ERR_CUDA;
  }
  net->allocs.push_back(q);
  *p = q;
  return FMG_OK;
}

static void net_free(fmg_net* net, void* p) {
  if (!p) return;
  for (auto it = net->allocs.begin(); it != net->allocs.end(); ++it)
    if (*it == p) { net->allocs.erase(it); break; }
  cudaFree(p);
}

void net_free_all(fmg_net* net) {
  for (void* p : net->allocs) cudaFree(p);
  net->allocs.clear();
  if (net->part) cudaFree(net->part);
  net->part = nullptr;
  net->part_cap = 0;
}

int net_reserve(fmg_net* net, const ActGeom& g) {
  const long long need = g.npad();
  if (need <= net->cap) {
    return FMG_OK;
  }
  bf16** bufs[] = {&net->X0, &net->H1, &net->H2, &net->dZ, &net->dP2, &net->dP1};
  const int ch[] = {kNetIn, kNetHid, kNetHid, kNetOut, kNetHid, kNetHid};
  cudaDeviceSynchronize();
  for (int b = 0; b < 6; ++b) {
    net_free(net, *bufs[b]);
    *bufs[b] = nullptr;
  }
  net->cap = 0;
  for (int b = 0; b < 6; ++b) {
    int rc = net_alloc(net, (void**)bufs[b], (size_t)need * ch[b] * sizeof(bf16));
    if (rc) return rc;
  }
  net->cap = need;
  return FMG_OK;
}

void net_refresh_weights(fmg_net* net, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_net_weights<<<256, 256, 0, st>>>(net->P, net->lay, net->wf1, net->wf2, net->wf3, net->wb2, net->wb3);
  net->weights_stale = false;
}

// the mean log k over the n top-level cells into out (= net->stat, its
// partials after it), the logs themselves kept in net->lraw for the levels'
// cell means
int launch_logmean(fmg_net* net, const double* k, long long n, double* out, cudaStream_t st) {
  const int nb = kLogSumBlocks;  // fixed, so the sum's order does not depend on the GPU
  net->lraw_n = 0;
  if (n > net->lraw_cap) {
    cudaStreamSynchronize(st);
    net_free(net, net->lraw);
    net->lraw = nullptr;
    net->lraw_cap = 0;
    if (int rc = net_alloc(net, (void**)&net->lraw, (size_t)n * sizeof(double))) return rc;
    net->lraw_cap = n;
  }
  g_launches.fetch_add(2, std::memory_order_relaxed);
  k_logsum<<<nb, kBlock, 0, st>>>(k, n, net->lraw, out + 8);
  k_logmean_final<<<1, kBlock, 0, st>>>(out + 8, nb, n, out);
  net->lraw_n = n;
  return FMG_OK;
}

int launch_features(fmg_net* net, const ActGeom& g, int n_l, int sub, long long n_top, double ratio, int np,
                    const double* xi, const double* kcell, double kconst, const double* mean, cudaStream_t st) {
  const TileGeo t = tile_geo(g);
  long long ncell = n_l;
  for (int k = 1; k < g.D; ++k) ncell *= n_l;
  if (kcell && ncell > net->fc_cap) {
    cudaStreamSynchronize(st);
    net_free(net, net->fc);
    net->fc = nullptr;
    net->fc_cap = 0;
    if (int rc = net_alloc(net, (void**)&net->fc, (size_t)ncell * sizeof(float))) return rc;
    net->fc_cap = ncell;
  }
  const float* fc = kcell ? net->fc : nullptr;
  long long ntop = n_top;
  for (int k = 1; k < g.D; ++k) ntop *= n_top;
  const double* lraw = net->lraw_n == ntop ? net->lraw : nullptr;  // logs of this top level
  if (ncell >= (1LL << 32) || g.nodes() >= (1LL << 32) || g.Mz > 65535) return FMG_ERR_UNSUPPORTED;
  g_launches.fetch_add(kcell ? 2 : 1, std::memory_order_relaxed);
  const dim3 fg(blocks_for((long long)g.Mx * g.My), g.D == 3 ? (unsigned)g.Mz : 1u);  // node planes in y
  if (g.D == 3) {
    if (kcell) k_cell_logk<3><<<blocks_for(ncell), 256, 0, st>>>(n_l, n_top, ratio, np, xi, kcell, lraw, mean, net->fc);
    k_features<3><<<fg, 256, 0, st>>>(t, n_l, sub, fc, kconst, mean, net->X0);
  } else {
    if (kcell) k_cell_logk<2><<<blocks_for(ncell), 256, 0, st>>>(n_l, n_top, ratio, np, xi, kcell, lraw, mean, net->fc);
    k_features<2><<<fg, 256, 0, st>>>(t, n_l, sub, fc, kconst, mean, net->X0);
  }
  return FMG_OK;
}

int net_forward(fmg_net* net, const ActGeom& g, double* omega, cudaStream_t st) {
  if (net->weights_stale) net_refresh_weights(net, st);
  int rc = g.D == 3 ? forward_d<3>(net, g, omega, st) : forward_d<2>(net, g, omega, st);
  if (rc) return rc;
  net->geom = g;
  net->have_forward = true;
  return FMG_OK;
}

int net_backward(fmg_net* net, const double* gomega, const double* omega, cudaStream_t st) {
  if (!net->have_forward) return FMG_ERR_STATE;
  if (net->weights_stale) net_refresh_weights(net, st);
  return net->geom.D == 3 ? backward_d<3>(net, gomega, omega, st) : backward_d<2>(net, gomega, omega, st);
}

void launch_adam(fmg_net* net, float lr, float b1, float b2, float eps, cudaStream_t st) {
  net->adam_t += 1;
  const float c1 = 1.f - powf(b1, (float)net->adam_t), c2 = 1.f - powf(b2, (float)net->adam_t);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_adam<<<blocks_for(net->lay.n), 256, 0, st>>>(net->P, net->G, net->Mo, net->Vo, net->lay.n, lr, b1, b2, eps, c1, c2);
  net->weights_stale = true;
}

int net_check_error(fmg_net* net, cudaStream_t st, const char** msg) {
  unsigned h = 0;
  if (cudaMemcpyAsync(&h, net->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    *msg = "CUDA error in the damping network";
    return FMG_ERR_CUDA;
  }
  if (h) {
    cudaMemsetAsync(net->err, 0, sizeof(unsigned), st);
    *msg = "a tensor-core wait of the damping network timed out";
    return FMG_ERR_CUDA;
  }
  return FMG_OK;
}

// The give-up path of the bounded waits, run alone: one CTA initialises an
// mbarrier, optionally arrives on it, and waits with the given limits; a wait
// that runs out records the error word, as the tensor-core kernels do, and the
// kernel returns.  Nothing else (no MMA, no bulk copy) is in flight.
__global__ void k_wait_selftest(unsigned* err, int arrive, int max_polls, unsigned long long max_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) umma::mbar_init(&bar);
  __syncthreads();
  if (arrive && threadIdx.x == 0) umma::mbar_arrive(&bar);
  __syncthreads();
  const bool ok = umma::mbar_wait_for(&bar, 0u, max_polls, max_ns);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, 1u);
}

int wait_selftest(int arrive, int max_polls, long long max_ns, cudaStream_t st, const char** msg) {
  unsigned* err = nullptr;
  unsigned h = 0;
  *msg = "CUDA error in the wait self-test";
  if (cudaMalloc((void**)&err, sizeof(unsigned)) != cudaSuccess) return FMG_ERR_CUDA;
  int rc = FMG_OK;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess) rc = FMG_ERR_CUDA;
  if (rc == FMG_OK) {
    k_wait_selftest<<<1, 128, 0, st>>>(err, arrive, max_polls, (unsigned long long)max_ns);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = FMG_ERR_CUDA;
  }
  cudaFree(err);
  if (rc == FMG_OK && h) {
    *msg = "a bounded device wait timed out (the kernel gave up, recorded its error word and returned)";
    rc = FMG_ERR_CUDA;
  }
  return rc;
}

void launch_rand_fill(double* e, int D, long long M, int dmask, unsigned long long seed, cudaStream_t st, int nc) {
  long long N = M;
  for (int k = 1; k < D; ++k) N *= M;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_rand_fill<<<blocks_for(N * nc), 256, 0, st>>>(e, D, M, dmask, nc, seed);
}

void launch_dinv(const double* A, int center, long long Np, const double* u, double* v, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_dinv<<<blocks_for(n), 256, 0, st>>>(A + (long long)center * Np, Np, u, v, n);
}

void launch_sub_wv(const double* x, const double* w, const double* v, double* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_sub_wv<<<blocks_for(n), 256, 0, st>>>(x, w, v, y, n);
}

void launch_gomega(const double* g, const double* v, double* gw, bool accumulate, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_gomega<<<blocks_for(n), 256, 0, st>>>(g, v, gw, accumulate ? 1 : 0, n);
}

void launch_wg_dinv(const double* A, int center, long long Np, const double* w, const double* g, double* t,
                    long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_wg_dinv<<<blocks_for(n), 256, 0, st>>>(A + (long long)center * Np, w, g, t, n);
}

void launch_scale_by(const double* x, double s, const double* scal, int slot, double* y, long long n,
                     cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_scale_by<<<blocks_for(n), 256, 0, st>>>(x, s, scal, slot, y, n);
}

void launch_ratio_acc(double* scal, int dst, int num, int den, double factor, bool first, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_ratio_acc<<<1, 1, 0, st>>>(scal, dst, num, den, factor, first ? 1 : 0);
}

void launch_xpwv(const double* x, const double* w, const double* v, double* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_xpwv<<<blocks_for(n), 256, 0, st>>>(x, w, v, y, n);
}

void launch_acc_prod(double* acc, const double* a, const double* b, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_acc_prod<<<blocks_for(n), 256, 0, st>>>(acc, a, b, n);
}

void launch_wg_dinv_acc(const double* A, int center, long long Np, const double* w, const double* x, double* y,
                        long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_wg_dinv_acc<<<blocks_for(n), 256, 0, st>>>(A + (long long)center * Np, w, x, y, n);
}

void launch_add(const double* x, double* y, long long n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_add<<<blocks_for(n), 256, 0, st>>>(x, y, n);
}

void launch_set_scalar(double* p, double v, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_set_scalar<<<1, 1, 0, st>>>(p, v);
}

}  // namespace fmg
