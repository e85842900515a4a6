// wx3d_mlp.cu -- learned surrogate for the hydrogen-rate + cooling_h update.
//
// A 4 -> 64 -> 64 -> 2 MLP with SiLU activations maps
//   (log10 n_H dt/yr, log10 T, x_HII, log10 dt/yr)
//      ->  (delta x_HII / SCALE_X, log10(cooling factor) / SCALE_C)
// for one step of updateNeutralFraction (hrate.f90:82-142) followed by
// apply_cooling_h_neq (cooling_h.f90:154-252); the cooling factor is the
// ratio of the pressures after and before the step, so the new state is
// P1 = cf * P0 and n_HI = n_H (1 - x1), as the plain step writes it.
//
// Operands are BF16, products accumulate in FP32 in tensor memory: the two
// hidden layers, and every product of the backward pass, are tcgen05.mma
// (kind::f16, M=128) issued by one thread, with operands in shared memory in
// the canonical no-swizzle core-matrix layout and the accumulator in TMEM,
// read back with tcgen05.ld.  In the forward pass the inputs, W1, the first
// hidden layer and W2 are split into a BF16 head and a BF16 tail
// (a = hi + lo, lo = bf16(a - hi)) and each layer sums the three products
// hi*hi + lo*hi + hi*lo, which carries about 16 significant bits instead of
// 8.  The 64 -> 2 output layer is an FP32 dot product on the CUDA cores.
//
// Operand layout.  A matrix of R rows and C columns (bf16) is stored as a
// grid of 8x8 "core matrices" of 128 bytes: element (r, c) lives at byte
//     ((r/8) * (C/8) + c/8) * 128 + (r%8) * 16 + (c%8) * 2.
// Read with K = columns (K-major) the descriptor strides are LBO = 128 (next
// 8 columns) and SBO = C/8*128 (next 8 rows).  The same bytes read with
// K = rows (MN-major, the transposed matrix) have SBO = 128 (next 8 of the
// M/N columns) and LBO = C/8*128 (next 8 of the K rows).  The backward pass
// uses that second view for the weight gradients, which contract over the
// batch, so no transposed copies are needed.  M is always 128: weight
// gradients (64 rows) run with the activation buffers padded to 128
// columns, and column 64 of the padding holds ones, so row 64 of each
// weight-gradient accumulator is the bias gradient.
//
// Every wait on an mbarrier has an iteration limit; on timeout the kernel
// records an error, still frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/wx3d.h"
#include "wx3d_internal.h"
#include "wx3d_rates.cuh"

namespace wx {
namespace mlp {

constexpr int NIN = 4, NH = 64, NOUT = 2;
constexpr int TILE = 128;                      // samples per MMA tile (M)
// parameter vector: W1[4][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2]
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NIN * NH, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH * NOUT, NPARAM = OFF_B3 + NOUT;

// Packed bf16 operand images of the weights (core-matrix layout):
//   W1B  [N=64 ][K=16]  (n,k) = hi(W1[k][n]) k<4, 0 at k=4, hi(W1[k-5][n])
//                       for 5<=k<9, lo(W1[k-9][n]) for 9<=k<13: B of layer 1,
//                       against input rows (hi(x), 1, lo(x), hi(x))
//   W2B  [N=64 ][K=64]  (n,k) = hi(W2[k][n]),     B of layer 2
//   W2L  [N=64 ][K=64]  (n,k) = lo(W2[k][n]),     B of layer 2 (tail)
//   W3R  [N=64 ][K=16]  (n,k) = W3[n][k]   (k<2), B of dH2 = dY W3^T
//   W2R  [N=64 ][K=64]  (n,k) = W2[n][k],         B of dH1 = dZ2 W2^T
constexpr int PK_W1B = 0, PK_W2B = PK_W1B + 64 * 16, PK_W2L = PK_W2B + 64 * 64, PK_W3R = PK_W2L + 64 * 64,
              PK_W2R = PK_W3R + 64 * 16, PK_N = PK_W2R + 64 * 64;   // bf16 elements
constexpr int PK_INF = PK_W3R;                                      // forward-only prefix

__host__ __device__ constexpr int cm_off(int r, int c, int C) {  // element offset in a core-matrix grid
  return (((r >> 3) * (C >> 3) + (c >> 3)) << 6) + ((r & 7) << 3) + (c & 7);
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier primitives (sm_100a)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;
}

// Instruction descriptor: kind::f16, BF16 x BF16 -> F32, both K-major unless
// the *_mn flags ask for MN-major, M x N.
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  const uint32_t z = 0;  // disable-output-lane mask: no lane disabled
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase with the given parity; returns false after
// `limit` unsuccessful tries (the kernel then records an error and returns).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 22) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMEM allocation by one full warp; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM address of (lane = this warp's first lane, column col).
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int col) {
  return base + ((uint32_t)((threadIdx.x >> 5) * 32) << 16) + (uint32_t)col;
}

// Writes 8 consecutive bf16 values of row r starting at column c (c % 8 == 0).
__device__ __forceinline__ void put8(__nv_bfloat16* m, int r, int c, int C, const float* v) {
  __align__(16) __nv_bfloat162 q[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) q[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4*>(m + cm_off(r, c, C)) = *reinterpret_cast<const uint4*>(q);
}

// Writes 8 consecutive values of row r (c % 8 == 0) as their bf16 head into
// hi and their bf16 tail into lo (lo may have another column count CL).
__device__ __forceinline__ void put8_split(__nv_bfloat16* hi, int C, __nv_bfloat16* lo, int CL, int r, int c,
                                           const float* v) {
  __align__(16) __nv_bfloat162 qh[4], ql[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    qh[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    const float2 f = __bfloat1622float2(qh[i]);
    ql[i] = __floats2bfloat162_rn(v[2 * i] - f.x, v[2 * i + 1] - f.y);
  }
  *reinterpret_cast<uint4*>(hi + cm_off(r, c, C)) = *reinterpret_cast<const uint4*>(qh);
  *reinterpret_cast<uint4*>(lo + cm_off(r, c, CL)) = *reinterpret_cast<const uint4*>(ql);
}

// SiLU(z) = z sigma(z) with sigma(z) = (1 + tanh(z/2)) / 2: one tanh.approx
// (a single SFU operation, relative error about 2^-11) per activation.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_approx(h), h);
}
__device__ __forceinline__ float dsilu(float z) {
  const float s = fmaf(0.5f, tanh_approx(0.5f * z), 0.5f);
  return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------------------
// Normalisation of the surrogate's inputs and outputs (the trust box).
struct Box {
  static constexpr double LN_LO = -3.0, LN_HI = 4.0;    // log10 n_H  [cm^-3]
  static constexpr double LT_LO = 2.0, LT_HI = 8.0;     // log10 T    [K]
  static constexpr double LD_LO = -2.0, LD_HI = 3.0;    // log10 dt   [yr]
  static constexpr double SCALE_X = 0.125;              // output 0 = delta x_HII / SCALE_X
  static constexpr double SCALE_C = 0.30102999566398120;  // output 1 = log10(cf) / log10(2)
};

// Network inputs in [-1, 1]: log10(n_H dt/yr) over [-5, 7] (the rates of
// hrate.f90 and the losses of cooling_h.f90 depend on n_H and dt only
// through their product), log10 T, x_HII and log10 dt/yr.
template <class F>
__host__ __device__ inline void normalise(F lgn, F lgT, F x, F lgdt, float* in) {
  constexpr double ND_LO = Box::LN_LO + Box::LD_LO, ND_HI = Box::LN_HI + Box::LD_HI;
  in[0] = (float)((lgn + lgdt - F(0.5 * (ND_LO + ND_HI))) * F(2.0 / (ND_HI - ND_LO)));
  in[1] = (float)((lgT - F(0.5 * (Box::LT_LO + Box::LT_HI))) * F(2.0 / (Box::LT_HI - Box::LT_LO)));
  in[2] = (float)(F(2) * x - F(1));
  in[3] = (float)((lgdt - F(0.5 * (Box::LD_LO + Box::LD_HI))) * F(2.0 / (Box::LD_HI - Box::LD_LO)));
}

// One plain FP64 step of hrate then cooling_h for a cell at rest with H
// density dh, neutral fraction y0 and temperature T0 (EOS_H_RATE:
// P = T k dh (2-y) / p_sc).  Returns y1 and the cooling factor P1/P0.
__device__ inline void plain_h_update(double dh, double y0, double T0, double dts, const PhysParams& ph, double* y1o,
                                      double* cfo) {
  double u[6], p[6];
  p[0] = dh * ph.mu0;
  p[1] = p[2] = p[3] = 0.0;
  p[4] = T0 * KB * dh * (2.0 - y0) / ph.p_sc;
  p[5] = dh * y0;
  prim2flow<6, false>(p, u, ph.cv);
  const double p4 = p[4];
  double ml = 0.0;
  h_cool_step<5>(u, p, dts, ph, &ml);
  *y1o = p[5] / (p[0] / ph.mu0);
  *cfo = p[4] / p4;
}

// ---------------------------------------------------------------------------
// Sample generator: log-uniform n, T, dt; uniform x_HII; targets from the
// plain FP64 integrator.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t seed, uint64_t i, int k) {
  return (double)(mix64(seed ^ mix64(i * 8 + k)) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void sample_kernel(PhysParams ph, long long n, unsigned long long seed, float* __restrict__ in,
                              float* __restrict__ out, double* __restrict__ raw) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double lgn = Box::LN_LO + (Box::LN_HI - Box::LN_LO) * u01(seed, i, 0);
    const double lgT = Box::LT_LO + (Box::LT_HI - Box::LT_LO) * u01(seed, i, 1);
    const double x = u01(seed, i, 2);
    const double lgd = Box::LD_LO + (Box::LD_HI - Box::LD_LO) * u01(seed, i, 3);
    const double dh = pow(10.0, lgn), T0 = pow(10.0, lgT), dts = pow(10.0, lgd) * 3.155673600e+7;
    double y1, cf;
    plain_h_update(dh, 1.0 - x, T0, dts, ph, &y1, &cf);
    normalise(lgn, lgT, x, lgd, in + 4 * i);
    out[2 * i] = (float)(((1.0 - y1) - x) / Box::SCALE_X);
    out[2 * i + 1] = (float)(log10(cf) / Box::SCALE_C);
    if (raw) {
      raw[4 * i] = dh; raw[4 * i + 1] = T0; raw[4 * i + 2] = x; raw[4 * i + 3] = dts;
    }
  }
}

// ---------------------------------------------------------------------------
// Shared memory.  FwdSmem is the training kernel's forward image (hidden
// activations padded to 128 columns for the weight-gradient MMAs); InfSmem
// is the inference image (64-column hidden layer 1, no layer-2 buffer: the
// 64 -> 2 output layer runs on the CUDA cores in FP32).

struct __align__(128) FwdSmem {
  __nv_bfloat16 x[TILE * 16];     // [128][16]  inputs hi(x), 1 (dW1 bias row), lo(x), hi(x)
  __nv_bfloat16 h1[TILE * 128];   // [128][128] hi(SiLU(z1)), cols 64.. = (1, 0, ...)
  __nv_bfloat16 h1lo[TILE * 64];  // [128][64]  lo(SiLU(z1))
  __nv_bfloat16 h2[TILE * 128];   // [128][128] SiLU(z2), cols 64.. = (1, 0, ...)
  __nv_bfloat16 w[PK_N];          // packed weights
  float b1[NH], b2[NH], w3[NH * NOUT], b3[16];
  uint64_t bar;
  uint32_t tmem;
  int err;
};

struct __align__(128) InfSmem {
  // The inputs are dead once the layer-1 MMA has completed, before the
  // first hidden layer is written, and the next tile's inputs are written
  // after the layer-2 MMA has completed: the two share their bytes.
  union {
    __nv_bfloat16 x[TILE * 16];   // [128][16]  inputs hi(x), 1, lo(x), hi(x)
    __nv_bfloat16 h1[TILE * 64];  // [128][64]  hi(SiLU(z1))
  };
  __nv_bfloat16 h1lo[TILE * 64];  // [128][64]  lo(SiLU(z1))
  __nv_bfloat16 w[PK_INF];        // W1B, W2B, W2L
  float b1[NH], b2[NH], w3[NH * NOUT], b3[16];
  int queue[2 * TILE];            // fallback cells of the fused source kernel
  int qn;
  uint64_t bar;
  uint32_t tmem;
  int err;
};
// Inference CTAs allocate 128 TMEM columns; the dynamic shared memory of an
// inference launch is padded so that at most four CTAs share an SM (five
// would need more than the 228 KB of an SM) and their allocations
// (4 x 128 of 512 columns) never wait on each other.
constexpr size_t INF_SMEM = 56 * 1024;
static_assert(sizeof(InfSmem) <= INF_SMEM && 5 * (INF_SMEM + 1024) > 228 * 1024, "inference shared memory");

struct __align__(128) BwdSmem {
  __nv_bfloat16 dy[TILE * 16];    // [128][16]  output gradient (cols 0,1)
  __nv_bfloat16 dz2[TILE * 64];   // [128][64]
  __nv_bfloat16 dz1[TILE * 128];  // [128][128] cols 64.. zero (M padding of dW1^T)
};

// Loads the first nw packed weights and the FP32 biases and output layer.
template <class S>
__device__ void load_weights(S& s, const __nv_bfloat16* __restrict__ pk, const float* __restrict__ prm, int nw) {
  const uint4* src = reinterpret_cast<const uint4*>(pk);
  uint4* dst = reinterpret_cast<uint4*>(s.w);
  for (int i = threadIdx.x; i < nw / 8; i += blockDim.x) dst[i] = src[i];
  for (int i = threadIdx.x; i < NH; i += blockDim.x) {
    s.b1[i] = prm[OFF_B1 + i];
    s.b2[i] = prm[OFF_B2 + i];
  }
  for (int i = threadIdx.x; i < NH * NOUT; i += blockDim.x) s.w3[i] = prm[OFF_W3 + i];
  if (threadIdx.x < 16) s.b3[threadIdx.x] = threadIdx.x < NOUT ? prm[OFF_B3 + threadIdx.x] : 0.f;
}

// Writes the padding columns 64..127 of an activation row: 1 at column 64.
__device__ __forceinline__ void pad_row(__nv_bfloat16* m, int r) {
  float v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = 0.f;
  v[0] = 1.f;
  put8(m, r, 64, 128, v);
  v[0] = 0.f;
#pragma unroll
  for (int c = 72; c < 128; c += 8) put8(m, r, c, 128, v);
}

// Forward pass of one tile whose inputs are already in s.x.  Layers 1 and 2
// are tcgen05 MMAs into TMEM columns [0,64) (z1) and [64,128) (z2), layer 2
// as the 12 K-steps hi(h1) hi(W2) + lo(h1) hi(W2) + hi(h1) lo(W2); the
// output layer is an FP32 dot product of this thread's SiLU(z2) row with
// W3.  HC is the column count of s.h1; KEEP stores SiLU(z2) (bf16) in h2s
// for the weight gradients.  On return y[0..1] holds this thread's outputs
// and z1/z2 stay in TMEM.  Returns false (uniformly) on timeout.
template <int HC, bool KEEP, class S>
__device__ bool forward_tile(S& s, __nv_bfloat16* h2s, uint32_t& phase, float* y) {
  const int t = threadIdx.x;
  const uint32_t tb = s.tmem;
  const uint32_t xa = smem_u32(s.x), h1a = smem_u32(s.h1), h1l = smem_u32(s.h1lo), wa = smem_u32(s.w);
  // layer 1: [128 x 16] x W1B -> z1 (the three products are K columns)
  fence_async_smem();
  fence_before();
  __syncthreads();
  if (t == 0) {
    fence_after();
    mma_bf16(tb + 0, sdesc(xa, 128, 256), sdesc(wa + 2 * PK_W1B, 128, 256), idesc(128, 64, 0, 0), 0);
    mma_commit(&s.bar);
  }
  if (!__syncthreads_and(mbar_wait(&s.bar, phase))) return false;
  phase ^= 1;
  fence_after();
  {
    float z[64];
#pragma unroll
    for (int q = 0; q < 4; ++q) tmem_ld16(tmem_addr(tb, 16 * q), z + 16 * q);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      float h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) h[i] = silu(z[8 * q + i] + s.b1[8 * q + i]);
      put8_split(s.h1, HC, s.h1lo, 64, t, 8 * q, h);
    }
  }
  // layer 2: [128 x 64] x (W2B + W2L) -> z2
  fence_async_smem();
  fence_before();
  __syncthreads();
  if (t == 0) {
    fence_after();
#pragma unroll
    for (int j = 0; j < 4; ++j)
      mma_bf16(tb + 64, sdesc(h1a + 256 * j, 128, (HC / 8) * 128), sdesc(wa + 2 * PK_W2B + 256 * j, 128, 8 * 128),
               idesc(128, 64, 0, 0), j > 0);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      mma_bf16(tb + 64, sdesc(h1l + 256 * j, 128, 8 * 128), sdesc(wa + 2 * PK_W2B + 256 * j, 128, 8 * 128),
               idesc(128, 64, 0, 0), 1);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      mma_bf16(tb + 64, sdesc(h1a + 256 * j, 128, (HC / 8) * 128), sdesc(wa + 2 * PK_W2L + 256 * j, 128, 8 * 128),
               idesc(128, 64, 0, 0), 1);
    mma_commit(&s.bar);
  }
  if (!__syncthreads_and(mbar_wait(&s.bar, phase))) return false;
  phase ^= 1;
  fence_after();
  {
    float z[64];
#pragma unroll
    for (int q = 0; q < 4; ++q) tmem_ld16(tmem_addr(tb, 64 + 16 * q), z + 16 * q);
    tmem_wait_ld();
    float y0 = s.b3[0], y1 = s.b3[1];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      float h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int j = 8 * q + i;
        h[i] = silu(z[j] + s.b2[j]);
        y0 = fmaf(h[i], s.w3[2 * j], y0);
        y1 = fmaf(h[i], s.w3[2 * j + 1], y1);
      }
      if (KEEP) put8(h2s, t, 8 * q, 128, h);
    }
    y[0] = y0;
    y[1] = y1;
  }
  fence_before();
  return true;
}

// Input row r: hi(x) (cols 0-3), 1 (col 4), lo(x) (5-8), hi(x) (9-12), 0.
template <class S>
__device__ __forceinline__ void put_inputs(S& s, int r, const float* in4, bool valid) {
  float v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = 0.f;
  if (valid) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float hi = __bfloat162float(__float2bfloat16_rn(in4[i]));
      v[i] = hi;
      v[5 + i] = in4[i] - hi;
      v[9 + i] = hi;
    }
    v[4] = 1.f;
  }
  put8(s.x, r, 0, 16, v);
  put8(s.x, r, 8, 16, v + 8);
}

// Inference over n samples: out[i] = MLP(in[i]).  128 threads per CTA.
__global__ void __launch_bounds__(TILE, 4) forward_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                           long long n, const __nv_bfloat16* __restrict__ pk,
                                                           const float* __restrict__ prm, int* err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  InfSmem& s = *reinterpret_cast<InfSmem*>(smraw);
  const int t = threadIdx.x;
  load_weights(s, pk, prm, PK_INF);
  if (t == 0) { mbar_init(&s.bar, 1); s.err = 0; }
  if (t < 32) tmem_alloc(&s.tmem, 128);
  fence_before();
  __syncthreads();
  fence_after();
  uint32_t phase = 0;
  const long long ntiles = (n + TILE - 1) / TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long i = tile * TILE + t;
    const bool valid = i < n;
    float in4[4] = {0, 0, 0, 0};
    if (valid) {
      const float4 q = reinterpret_cast<const float4*>(in)[i];
      in4[0] = q.x; in4[1] = q.y; in4[2] = q.z; in4[3] = q.w;
    }
    put_inputs(s, t, in4, valid);
    float y[2];
    if (!forward_tile<64, false>(s, nullptr, phase, y)) { s.err = 1; break; }
    if (valid) { out[2 * i] = y[0]; out[2 * i + 1] = y[1]; }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (t < 32) tmem_free(s.tmem, 128);
  if (t == 0 && s.err) atomicAdd(err, 1);
}

// ---------------------------------------------------------------------------
// Training: forward, loss gradient, backward and weight gradients for
// `tiles` consecutive tiles per CTA; the weight gradients accumulate in TMEM
// across the CTA's tiles and are added to the global FP32 gradient at the end.
//
// TMEM columns: [0,64) z1, [64,128) z2, [128,160) free,
// [160,224) dH2 then dH1, [256,272) dW3 (rows = hidden2, row 64 = db3),
// [288,352) dW2 (rows = hidden1, row 64 = db2), [352,368) dW1^T
// (rows = hidden1, column 4 = db1).  512 columns.
__global__ void __launch_bounds__(TILE) train_kernel(const float* __restrict__ in, const float* __restrict__ tgt,
                                                      long long n, long long first_tile, int tiles, float gscale,
                                                      const __nv_bfloat16* __restrict__ pk,
                                                      const float* __restrict__ prm, float* __restrict__ grad,
                                                      float* __restrict__ loss, int* err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  FwdSmem& s = *reinterpret_cast<FwdSmem*>(smraw);
  BwdSmem& b = *reinterpret_cast<BwdSmem*>(smraw + ((sizeof(FwdSmem) + 127) / 128) * 128);
  const int t = threadIdx.x;
  load_weights(s, pk, prm, PK_N);
  if (t == 0) { mbar_init(&s.bar, 1); s.err = 0; }
  if (t < 32) tmem_alloc(&s.tmem, 512);
  pad_row(s.h1, t);
  pad_row(s.h2, t);
  {
    float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 64; c < 128; c += 8) put8(b.dz1, t, c, 128, z);
    put8(b.dy, t, 8, 16, z);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tb = s.tmem;
  const uint32_t xa = smem_u32(s.x), h1a = smem_u32(s.h1), h2a = smem_u32(s.h2), wa = smem_u32(s.w);
  const uint32_t dya = smem_u32(b.dy), dz2a = smem_u32(b.dz2), dz1a = smem_u32(b.dz1);
  uint32_t phase = 0;
  float lsum = 0.f;
  bool ok = true;
  const long long ntiles = (n + TILE - 1) / TILE;
  for (int k = 0; k < tiles && ok; ++k) {
    const long long tile = first_tile + (long long)blockIdx.x * tiles + k;
    if (tile >= ntiles) break;
    const long long i = tile * TILE + t;
    const bool valid = i < n;
    float in4[4] = {0, 0, 0, 0}, tg[2] = {0, 0};
    if (valid) {
      const float4 q = reinterpret_cast<const float4*>(in)[i];
      in4[0] = q.x; in4[1] = q.y; in4[2] = q.z; in4[3] = q.w;
      tg[0] = tgt[2 * i];
      tg[1] = tgt[2 * i + 1];
    }
    put_inputs(s, t, in4, valid);
    float y[2];
    if (!forward_tile<128, true>(s, s.h2, phase, y)) { ok = false; break; }
    // loss = sum (y - t)^2 * gscale ; dL/dy = 2 (y - t) * gscale
    float dy[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (valid) {
      const float e0 = y[0] - tg[0], e1 = y[1] - tg[1];
      lsum += e0 * e0 + e1 * e1;
      dy[0] = 2.f * e0 * gscale;
      dy[1] = 2.f * e1 * gscale;
    }
    put8(b.dy, t, 0, 16, dy);
    // dH2 = dY W3^T  [128x16]x[64x16]^T -> TMEM 160
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (t == 0) {
      fence_after();
      mma_bf16(tb + 160, sdesc(dya, 128, 256), sdesc(wa + 2 * PK_W3R, 128, 256), idesc(128, 64, 0, 0), 0);
      mma_commit(&s.bar);
    }
    if (!__syncthreads_and(mbar_wait(&s.bar, phase))) { ok = false; break; }
    phase ^= 1;
    fence_after();
    {
      float g[64], z[64];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem_addr(tb, 160 + 16 * q), g + 16 * q);
        tmem_ld16(tmem_addr(tb, 64 + 16 * q), z + 16 * q);
      }
      tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float d[8];
#pragma unroll
        for (int i2 = 0; i2 < 8; ++i2) d[i2] = valid ? g[8 * q + i2] * dsilu(z[8 * q + i2] + s.b2[8 * q + i2]) : 0.f;
        put8(b.dz2, t, 8 * q, 64, d);
      }
    }
    // dH1 = dZ2 W2^T -> TMEM 160 ; dW3 += H2^T dY ; dW2 += H1^T dZ2
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (t == 0) {
      fence_after();
#pragma unroll
      for (int j = 0; j < 4; ++j)
        mma_bf16(tb + 160, sdesc(dz2a + 256 * j, 128, 8 * 128), sdesc(wa + 2 * PK_W2R + 256 * j, 128, 8 * 128),
                 idesc(128, 64, 0, 0), j > 0);
      // weight gradients contract over the batch (K = 128 = 8 steps of 16):
      // A = activations viewed MN-major (rows = 128 padded units),
      // B = gradients viewed MN-major.
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t acc = (k > 0 || j > 0) ? 1u : 0u;
        // batch rows 16j..16j+15 are row-blocks 2j, 2j+1 of each buffer
        mma_bf16(tb + 256, sdesc(h2a + 2 * j * (16 * 128), 16 * 128, 128),
                 sdesc(dya + 2 * j * (2 * 128), 2 * 128, 128), idesc(128, 16, 1, 1), acc);
        mma_bf16(tb + 288, sdesc(h1a + 2 * j * (16 * 128), 16 * 128, 128),
                 sdesc(dz2a + 2 * j * (8 * 128), 8 * 128, 128), idesc(128, 64, 1, 1), acc);
      }
      mma_commit(&s.bar);
    }
    if (!__syncthreads_and(mbar_wait(&s.bar, phase))) { ok = false; break; }
    phase ^= 1;
    fence_after();
    {
      float g[64], z[64];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem_addr(tb, 160 + 16 * q), g + 16 * q);
        tmem_ld16(tmem_addr(tb, 0 + 16 * q), z + 16 * q);
      }
      tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float d[8];
#pragma unroll
        for (int i2 = 0; i2 < 8; ++i2) d[i2] = valid ? g[8 * q + i2] * dsilu(z[8 * q + i2] + s.b1[8 * q + i2]) : 0.f;
        put8(b.dz1, t, 8 * q, 128, d);
      }
    }
    // dW1^T += dZ1^T X  (rows = hidden1, N = 16 inputs; column 4 = db1)
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (t == 0) {
      fence_after();
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t acc = (k > 0 || j > 0) ? 1u : 0u;
        mma_bf16(tb + 352, sdesc(dz1a + 2 * j * (16 * 128), 16 * 128, 128),
                 sdesc(xa + 2 * j * (2 * 128), 2 * 128, 128), idesc(128, 16, 1, 1), acc);
      }
      mma_commit(&s.bar);
    }
    if (!__syncthreads_and(mbar_wait(&s.bar, phase))) { ok = false; break; }
    phase ^= 1;
    fence_after();
  }
  // flush the accumulated weight gradients: lanes (= rows) 0..63 hold the
  // hidden units, lane 64 the bias row.  The TMEM loads are warp-collective,
  // so every thread issues them and only the owners of a row add it.
  ok = __syncthreads_and(ok);
  const int row = t;
  const long long first = first_tile + (long long)blockIdx.x * tiles;
  if (ok && first < ntiles) {
    float g[64], g3[16], g1[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) tmem_ld16(tmem_addr(tb, 288 + 16 * q), g + 16 * q);
    tmem_ld16(tmem_addr(tb, 256), g3);
    tmem_ld16(tmem_addr(tb, 352), g1);
    tmem_wait_ld();
    if (row < 64) {
      // dW2: row = hidden1 unit j, columns = hidden2 units -> W2[j][.]
      for (int i2 = 0; i2 < 64; ++i2) atomicAdd(&grad[OFF_W2 + row * NH + i2], g[i2]);
      atomicAdd(&grad[OFF_W3 + row * NOUT + 0], g3[0]);
      atomicAdd(&grad[OFF_W3 + row * NOUT + 1], g3[1]);
      for (int i2 = 0; i2 < NIN; ++i2) atomicAdd(&grad[OFF_W1 + i2 * NH + row], g1[i2]);
      atomicAdd(&grad[OFF_B1 + row], g1[4]);
    } else if (row == 64) {
      for (int i2 = 0; i2 < 64; ++i2) atomicAdd(&grad[OFF_B2 + i2], g[i2]);
      atomicAdd(&grad[OFF_B3 + 0], g3[0]);
      atomicAdd(&grad[OFF_B3 + 1], g3[1]);
    }
  }
  // loss: warp reduce then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0 && loss) atomicAdd(loss, lsum * gscale);
  if (!ok && t == 0) s.err = 1;
  fence_before();
  __syncthreads();
  fence_after();
  if (t < 32) tmem_free(s.tmem, 512);
  if (t == 0 && s.err) atomicAdd(err, 1);
}

// Adam on the FP32 master parameters, then repacks the bf16 operand images.
__global__ void adam_kernel(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    prm[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// Row and column of element o of a core-matrix image with C columns.
__device__ __forceinline__ void cm_rc(int o, int C, int* r, int* c) {
  const int cb = o >> 6, w = o & 63;
  *r = (cb / (C >> 3)) * 8 + (w >> 3);
  *c = (cb % (C >> 3)) * 8 + (w & 7);
}

__device__ __forceinline__ float bf16_hi(float a) { return __bfloat162float(__float2bfloat16_rn(a)); }

__global__ void pack_kernel(const float* __restrict__ prm, __nv_bfloat16* __restrict__ pk) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < PK_N; e += gridDim.x * blockDim.x) {
    float v = 0.f;
    int n, k;
    if (e < PK_W2B) {  // W1B [64][16]
      cm_rc(e - PK_W1B, 16, &n, &k);
      if (k < NIN) v = prm[OFF_W1 + k * NH + n];
      else if (k >= 5 && k < 5 + NIN) v = prm[OFF_W1 + (k - 5) * NH + n];
      else if (k >= 9 && k < 9 + NIN) {
        const float a = prm[OFF_W1 + (k - 9) * NH + n];
        v = a - bf16_hi(a);
      }
    } else if (e < PK_W2L) {  // W2B [64][64]: (n,k) = hi(W2[k][n])
      cm_rc(e - PK_W2B, 64, &n, &k);
      v = prm[OFF_W2 + k * NH + n];
    } else if (e < PK_W3R) {  // W2L [64][64]: (n,k) = lo(W2[k][n])
      cm_rc(e - PK_W2L, 64, &n, &k);
      const float a = prm[OFF_W2 + k * NH + n];
      v = a - bf16_hi(a);
    } else if (e < PK_W2R) {  // W3R [64][16]: (n,k) = W3[n][k]
      cm_rc(e - PK_W3R, 16, &n, &k);
      v = k < NOUT ? prm[OFF_W3 + n * NOUT + k] : 0.f;
    } else {  // W2R [64][64]: (n,k) = W2[n][k]
      cm_rc(e - PK_W2R, 64, &n, &k);
      v = prm[OFF_W2 + n * NH + k];
    }
    pk[e] = __float2bfloat16_rn(v);
  }
}

// ---------------------------------------------------------------------------
// Fused source step with the surrogate: updatePrims, then for every cell
// either the MLP's (delta x_HII, delta log10 T) -- when the cell lies in the
// trust box and in a trusted bin of the table -- or the plain FP64
// hrate + cooling_h step, then the CFL minimum.  Tiles of 128 cells of one
// block; the MMA work of a tile is uniform, the fallback is per cell.
struct SurrParams {
  double* __restrict__ u;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int nwork;
  DevCtl* ctl;
  PhysParams ph;
  const __nv_bfloat16* __restrict__ pk;
  const float* __restrict__ prm;
  const uint8_t* __restrict__ trust;
  int do_dt;
  int* err;
  const double* __restrict__ cool_lt;
  const double* __restrict__ cool_lc;
  int ncool;
  int nZ;
};

// Plain FP64 step of one cell (the fallback), with its store and its CFL
// contribution: hrate + cooling_h, or hrate then table cooling, as the plain
// source step does them (hrate.f90:101-140, then cooling_h.f90:175-246 or
// cooling.f90:303-369 / cooling_schure.f90:134-228).
template <int NEQ>
__device__ __forceinline__ void fallback_cell(const SurrParams& P, int id, double dts, double& dtl, double& mloss) {
  const int slot = id >> 12, c = id & (BCELLS - 1);
  const size_t o = ((size_t)slot * NEQ) * BCELLS + c;
  const PhysParams& ph = P.ph;
  double u[NEQ], p[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e) u[e] = P.u[o + (size_t)e * BCELLS];
  flow2prim<NEQ, false>(u, p, ph.inv_cv);
  if (ph.cooling == WX_COOL_H) {
    h_cool_step<5>(u, p, dts, ph, &mloss);
  } else {
    const double T = calc_temp<5>(p, ph);
    const double dh = p[0] / ph.mu0;
    const double y0 = p[5] / dh;
    const double y1 = h_rate_y1(T, dh, y0, dts);
    p[5] = p[0] * y1 / ph.mu0;
    u[5] = p[5];
    table_cooling<NEQ, 5>(u, p, dts, ph, P.cool_lt, P.cool_lc, P.ncool, P.nZ, mloss);
  }
  P.u[o + 4 * (size_t)BCELLS] = u[4];
  P.u[o + 5 * (size_t)BCELLS] = u[5];
  if (P.do_dt) dtl = dmin(dtl, cell_dt<NEQ, false>(p, P.blocks[slot], P.ph.gamma));
}

// Cells that fall back are queued in shared memory (id = slot * 4096 + cell)
// and integrated 128 at a time, so a warp runs the plain integrator only
// for a full set of fallback cells, not for each of its tiles that holds
// one.
template <int NEQ>
__global__ void __launch_bounds__(TILE, 4) surrogate_source_kernel(SurrParams P) {
  extern __shared__ __align__(128) unsigned char smraw[];
  InfSmem& s = *reinterpret_cast<InfSmem*>(smraw);
  int* queue = s.queue;
  int& qn = s.qn;
  const int t = threadIdx.x, lane = t & 31;
  const PhysParams& ph = P.ph;
  load_weights(s, P.pk, P.prm, PK_INF);
  if (t == 0) { mbar_init(&s.bar, 1); s.err = 0; qn = 0; }
  if (t < 32) tmem_alloc(&s.tmem, 128);
  fence_before();
  __syncthreads();
  fence_after();
  uint32_t phase = 0;
  const double dts = P.ctl->dt * ph.t_sc;
  const float lgd = log10f((float)(dts / 3.155673600e+7));
  const bool dt_in = lgd >= (float)Box::LD_LO && lgd <= (float)Box::LD_HI;
  const double inv_mu0 = 1.0 / ph.mu0;
  const double cf_min = 1.0 - ph.cooling_limit;
  double dtl = 1.0e300, mloss = 0.0;
  unsigned nsur = 0, nplain = 0;
  const long long ntiles = (long long)P.nwork * (BCELLS / TILE);
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int slot = P.work[tile / (BCELLS / TILE)];
    const int c = (int)(tile % (BCELLS / TILE)) * TILE + t;
    if (!dt_in) {  // dt outside the training box (the same for every thread): plain step, no queue
      fallback_cell<NEQ>(P, (slot << 12) | c, dts, dtl, mloss);
      ++nplain;
      continue;
    }
    const size_t o = ((size_t)slot * NEQ) * BCELLS + c;
    double u[NEQ], p[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) u[e] = P.u[o + (size_t)e * BCELLS];
    flow2prim<NEQ, false>(u, p, ph.inv_cv);
    // gate: inside the training box and in a trusted bin (FP32 logs)
    const double dh = p[0] * inv_mu0;
    const double y0 = p[5] / dh;
    const double T0 = calc_temp<5>(p, ph);
    const float lgn = log10f((float)dh), lgT = log10f((float)T0), x0 = (float)(1.0 - y0);
    bool use = dt_in && lgn >= (float)Box::LN_LO && lgn <= (float)Box::LN_HI && lgT >= (float)Box::LT_LO &&
               lgT <= (float)Box::LT_HI && x0 >= 0.f && x0 <= 1.f;
    if (use) {
      const int bn = min(TRUST_ND - 1, max(0, (int)floorf((lgn + lgd - (float)TRUST_ND_LO) * (float)(1.0 / TRUST_ND_W))));
      const int bt = min(TRUST_T - 1, max(0, (int)floorf((lgT - (float)TRUST_T_LO) * (float)(1.0 / TRUST_T_W))));
      const int bx = min(TRUST_X - 1, (int)(x0 * TRUST_X));
      use = P.trust[(bn * TRUST_T + bt) * TRUST_X + bx] != 0;
    }
    // queue the fallback cells (warp-aggregated)
    {
      const unsigned fb = __ballot_sync(0xffffffffu, !use);
      int base = 0;
      if (lane == 0 && fb) base = atomicAdd(&qn, __popc(fb));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (!use) queue[base + __popc(fb & ((1u << lane) - 1u))] = (slot << 12) | c;
    }
    if (__syncthreads_or(use)) {  // the tile's MMAs run only if some cell uses them
      float in4[4];
      normalise(lgn, lgT, x0, lgd, in4);
      put_inputs(s, t, in4, use);
      float y[2];
      if (!forward_tile<64, false>(s, nullptr, phase, y)) { s.err = 1; break; }
      if (use) {
        double y1 = 1.0 - ((double)x0 + (double)y[0] * Box::SCALE_X);
        y1 = dmin(y1, 1.0 - 1.e-4);
        y1 = dmax(y1, 0.0);
        if (ph.cooling == WX_COOL_H) {  // both outputs: x_HII and the cooling factor
          const double cf = (double)exp10f(y[1] * (float)Box::SCALE_C);
          mloss = dmax(mloss, 1.0 - cf);
          p[4] *= dmin(1.0, dmax(cf, cf_min));
          p[5] = p[0] * y1 * inv_mu0;
          const double EK = 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
          u[4] = EK + ph.cv * p[4];
        } else {  // x_HII from the network (the hrate update), then the plain table cooling
          p[5] = p[0] * y1 / ph.mu0;
          u[5] = p[5];
          table_cooling<NEQ, 5>(u, p, dts, ph, P.cool_lt, P.cool_lc, P.ncool, P.nZ, mloss);
        }
        P.u[o + 4 * (size_t)BCELLS] = u[4];
        P.u[o + 5 * (size_t)BCELLS] = p[5];
        if (P.do_dt) dtl = dmin(dtl, cell_dt<NEQ, false>(p, P.blocks[slot], ph.gamma));
        ++nsur;
      }
    }
    __syncthreads();
    const int q = qn;
    if (q >= TILE) {  // a full set: one queued cell per thread
      fallback_cell<NEQ>(P, queue[q - TILE + t], dts, dtl, mloss);
      ++nplain;
      __syncthreads();
      if (t == 0) qn = q - TILE;
      __syncthreads();
    }
  }
  {  // the remainder of the queue
    __syncthreads();
    const int q = qn;
    if (t < q) {
      fallback_cell<NEQ>(P, queue[t], dts, dtl, mloss);
      ++nplain;
    }
  }
  if (P.do_dt) {
    double v = dtl;
    for (int k = 16; k > 0; k >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, k));
    if (lane == 0) atomic_min_pos(&P.ctl->dtmin_bits, v);
  }
  double mm = mloss;
  for (int k = 16; k > 0; k >>= 1) mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, k));
  if (lane == 0 && mm > 0.0) atomic_max_pos(&P.ctl->maxloss_bits, mm);
  nsur = __reduce_add_sync(0xffffffffu, nsur);
  nplain = __reduce_add_sync(0xffffffffu, nplain);
  if (lane == 0) {
    if (nsur) atomicAdd(&P.ctl->sur[0], (unsigned long long)nsur);
    if (nplain) atomicAdd(&P.ctl->sur[1], (unsigned long long)nplain);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (t < 32) tmem_free(s.tmem, 128);
  if (t == 0 && s.err) atomicAdd(P.err, 1);
}

// Waits, with the kernels' bounded wait, on an mbarrier that nothing
// arrives at, and records the timeout the way the MLP kernels do: the test
// of the error path that a lost MMA completion would take.
__global__ void wait_timeout_probe_kernel(int limit, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const bool ok = __syncthreads_and(mbar_wait(&bar, 0, limit));
  if (!ok && threadIdx.x == 0) atomicAdd(err, 1);
}

}  // namespace mlp
}  // namespace wx

// =============================================================================
// C-ABI

using namespace wx;
using namespace wx::mlp;

struct wx_mlp {
  float* prm = nullptr;           // FP32 master parameters [NPARAM]
  float* m = nullptr;             // Adam moments
  float* v = nullptr;
  float* grad = nullptr;          // FP32 gradient accumulator
  __nv_bfloat16* pk = nullptr;    // packed bf16 operand images
  float* loss = nullptr;          // device scalar
  int* err = nullptr;             // device error counter (timeouts)
  long long step = 0;
  int nsm = 148;
};

namespace wx {

cudaError_t launch_surrogate_source(const SurrLaunch& L, cudaStream_t s) {
  SurrParams P{L.u,      L.blocks,  L.work,    L.nwork,      L.ctl,       L.ph,     L.mlp->pk, L.mlp->prm,
               L.trust,  L.do_dt,   L.mlp->err, L.cool_lt,   L.cool_lc,   L.ncool,  L.nZ};
  const long long ntiles = (long long)L.nwork * (BCELLS / TILE);
  if (ntiles == 0) return cudaSuccess;  // no local block
  const int grid = (int)std::min<long long>(ntiles, 4LL * L.nsm);
  if (L.neq == 6) {
    cudaFuncSetAttribute(surrogate_source_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM);
    surrogate_source_kernel<6><<<grid, TILE, INF_SMEM, s>>>(P);
  } else if (L.neq == 7) {
    cudaFuncSetAttribute(surrogate_source_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM);
    surrogate_source_kernel<7><<<grid, TILE, INF_SMEM, s>>>(P);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace wx

namespace {

PhysParams phys_from(const wx_config& f) {
  PhysParams p{};
  p.gamma = f.gamma;
  p.cv = 1.0 / (f.gamma - 1.0);
  p.inv_cv = 1.0 / p.cv;
  p.cfl = f.cfl;
  p.eta = f.visc_eta;
  p.mu0 = f.mu0; p.mui = f.mui; p.ion_thres = f.ion_thres;
  p.d_sc = f.d_sc;
  p.p_sc = f.d_sc * (f.v_sc * f.v_sc);
  p.e_sc = p.p_sc;
  p.t_sc = f.l_sc / f.v_sc;
  p.dtout = f.dtout;
  p.cooling_limit = f.cooling_limit;
  p.limiter = f.limiter_type;
  p.eight_wave = f.eight_wave;
  for (int i = 0; i < 6; ++i) p.bc[i] = f.bc[i];
  p.eos = WX_EOS_H_RATE;
  p.cooling = WX_COOL_H;
  p.fp = 5;
  p.npassive = 1;
  return p;
}

int mlp_check(wx_mlp* w) {
  int e = 0;
  if (cudaMemcpy(&e, w->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return WX_ERR_CUDA;
  return e ? WX_ERR_TIMEOUT : WX_OK;
}

size_t train_smem() { return ((sizeof(FwdSmem) + 127) / 128) * 128 + sizeof(BwdSmem); }

}  // namespace

extern "C" {

int wx3d_mlp_create(uint64_t seed, wx_mlp** out) {
  if (!out) return WX_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WX_ERR_NO_DEVICE;
  wx_mlp* w = new wx_mlp();
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&w->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaMalloc(&w->prm, NPARAM * 4) || cudaMalloc(&w->m, NPARAM * 4) || cudaMalloc(&w->v, NPARAM * 4) ||
      cudaMalloc(&w->grad, NPARAM * 4) || cudaMalloc(&w->pk, PK_N * 2) || cudaMalloc(&w->loss, 4) ||
      cudaMalloc(&w->err, 4)) {
    delete w;
    return WX_ERR_CUDA;
  }
  // Glorot-uniform weights, zero biases, from a 64-bit LCG
  std::vector<float> h(NPARAM, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((st >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  const float a1 = std::sqrt(6.f / (NIN + NH)), a2 = std::sqrt(6.f / (NH + NH)), a3 = std::sqrt(6.f / (NH + NOUT));
  for (int i = 0; i < NIN * NH; ++i) h[OFF_W1 + i] = a1 * uni();
  for (int i = 0; i < NH * NH; ++i) h[OFF_W2 + i] = a2 * uni();
  for (int i = 0; i < NH * NOUT; ++i) h[OFF_W3 + i] = a3 * uni();
  cudaMemcpy(w->prm, h.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemset(w->m, 0, NPARAM * 4);
  cudaMemset(w->v, 0, NPARAM * 4);
  cudaMemset(w->err, 0, 4);
  pack_kernel<<<(PK_N + 255) / 256, 256>>>(w->prm, w->pk);
  if (cudaDeviceSynchronize() != cudaSuccess) { delete w; return WX_ERR_CUDA; }
  cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM);
  cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
  *out = w;
  return WX_OK;
}

int wx3d_mlp_destroy(wx_mlp* w) {
  if (!w) return WX_ERR_INVALID_ARG;
  cudaFree(w->prm); cudaFree(w->m); cudaFree(w->v); cudaFree(w->grad); cudaFree(w->pk);
  cudaFree(w->loss); cudaFree(w->err);
  delete w;
  return WX_OK;
}

int wx3d_mlp_nparams(void) { return NPARAM; }

int wx3d_mlp_get_params(wx_mlp* w, float* host) {
  if (!w || !host) return WX_ERR_INVALID_ARG;
  return cudaMemcpy(host, w->prm, NPARAM * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? WX_OK : WX_ERR_CUDA;
}

int wx3d_mlp_set_params(wx_mlp* w, const float* host) {
  if (!w || !host) return WX_ERR_INVALID_ARG;
  if (cudaMemcpy(w->prm, host, NPARAM * 4, cudaMemcpyHostToDevice) != cudaSuccess) return WX_ERR_CUDA;
  pack_kernel<<<(PK_N + 255) / 256, 256>>>(w->prm, w->pk);
  return cudaDeviceSynchronize() == cudaSuccess ? WX_OK : WX_ERR_CUDA;
}

// Training / evaluation samples from the plain FP64 integrator.  d_in
// [n][4] normalised inputs, d_tgt [n][2] targets (delta x_HII / 0.125,
// log10(P1/P0) / log10 2), d_raw [n][4] (n_H, T, x_HII, dt in s) or NULL.
int wx3d_mlp_samples(const wx_config* cfg, int64_t n, uint64_t seed, float* d_in, float* d_tgt, double* d_raw,
                     void* stream) {
  if (!cfg || n <= 0 || !d_in || !d_tgt) return WX_ERR_INVALID_ARG;
  const PhysParams ph = phys_from(*cfg);
  sample_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(ph, n, seed, d_in, d_tgt, d_raw);
  if (cudaGetLastError() != cudaSuccess) return WX_ERR_CUDA;
  return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? WX_OK : WX_ERR_CUDA;
}

// Inference with the tcgen05 forward kernel.
int wx3d_check_wait_timeout(int32_t limit) {
  if (limit < 1 || limit > (1 << 22)) return WX_ERR_INVALID_ARG;
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return WX_ERR_CUDA;
  int e = 0;
  cudaError_t ce = cudaMemset(err, 0, sizeof(int));
  if (ce == cudaSuccess) {
    wait_timeout_probe_kernel<<<1, 128>>>(limit, err);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  if (ce == cudaSuccess) ce = cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(err);
  if (ce != cudaSuccess) return WX_ERR_CUDA;
  return e ? WX_ERR_TIMEOUT : WX_OK;
}

int wx3d_mlp_forward(wx_mlp* w, int64_t n, const float* d_in, float* d_out, void* stream) {
  if (!w || n <= 0 || !d_in || !d_out) return WX_ERR_INVALID_ARG;
  const long long ntiles = (n + TILE - 1) / TILE;
  const int grid = (int)std::min<long long>(ntiles, 4LL * w->nsm);
  cudaMemsetAsync(w->err, 0, 4, (cudaStream_t)stream);
  forward_kernel<<<grid, TILE, INF_SMEM, (cudaStream_t)stream>>>(d_in, d_out, n, w->pk, w->prm, w->err);
  if (cudaGetLastError() != cudaSuccess) return WX_ERR_CUDA;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return WX_ERR_CUDA;
  return mlp_check(w);
}

// Mean-squared-error loss and its gradient over all n samples (one pass of
// the tcgen05 training kernel, no parameter update).  grad_host [NPARAM].
int wx3d_mlp_gradient(wx_mlp* w, int64_t n, const float* d_in, const float* d_tgt, float* loss, float* grad_host) {
  if (!w || n <= 0 || !d_in || !d_tgt) return WX_ERR_INVALID_ARG;
  const long long ntiles = (n + TILE - 1) / TILE;
  const int ncta = (int)std::min<long long>(ntiles, w->nsm);
  const int tiles = (int)((ntiles + ncta - 1) / ncta);
  cudaMemset(w->grad, 0, NPARAM * 4);
  cudaMemset(w->loss, 0, 4);
  cudaMemset(w->err, 0, 4);
  train_kernel<<<ncta, TILE, train_smem()>>>(d_in, d_tgt, n, 0, tiles, 1.0f / (float)n, w->pk, w->prm, w->grad,
                                             w->loss, w->err);
  if (cudaGetLastError() != cudaSuccess) return WX_ERR_CUDA;
  if (cudaDeviceSynchronize() != cudaSuccess) return WX_ERR_CUDA;
  int rc = mlp_check(w);
  if (rc) return rc;
  if (loss) cudaMemcpy(loss, w->loss, 4, cudaMemcpyDeviceToHost);
  if (grad_host) cudaMemcpy(grad_host, w->grad, NPARAM * 4, cudaMemcpyDeviceToHost);
  return WX_OK;
}

// Adam training over n samples for `epochs` passes in minibatches of
// `batch` samples (rounded to 128); loss_per_epoch (host, may be NULL)
// receives the mean training loss of each epoch.
int wx3d_mlp_train(wx_mlp* w, int64_t n, const float* d_in, const float* d_tgt, int32_t epochs, int32_t batch,
                   float lr, float* loss_per_epoch) {
  if (!w || n <= 0 || !d_in || !d_tgt || epochs <= 0 || batch <= 0) return WX_ERR_INVALID_ARG;
  const long long ntiles = (n + TILE - 1) / TILE;
  const long long btiles = std::max<long long>(1, batch / TILE);
  const int ncta = (int)std::min<long long>(btiles, w->nsm);
  const int tiles = (int)((btiles + ncta - 1) / ncta);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  cudaMemset(w->err, 0, 4);
  for (int ep = 0; ep < epochs; ++ep) {
    cudaMemset(w->loss, 0, 4);
    long long nb = 0;
    for (long long t0 = 0; t0 < ntiles; t0 += (long long)ncta * tiles, ++nb) {
      const long long cnt = std::min<long long>((long long)ncta * tiles, ntiles - t0) * TILE;
      const long long m = std::min<long long>(cnt, n - t0 * TILE);
      cudaMemsetAsync(w->grad, 0, NPARAM * 4);
      train_kernel<<<ncta, TILE, train_smem()>>>(d_in, d_tgt, n, t0, tiles, 1.0f / (float)m, w->pk, w->prm, w->grad,
                                                 w->loss, w->err);
      ++w->step;
      const float c1 = 1.f / (1.f - std::pow(b1, (float)w->step));
      const float c2 = 1.f / (1.f - std::pow(b2, (float)w->step));
      adam_kernel<<<(NPARAM + 255) / 256, 256>>>(w->prm, w->grad, w->m, w->v, lr, b1, b2, eps, c1, c2);
      pack_kernel<<<(PK_N + 255) / 256, 256>>>(w->prm, w->pk);
    }
    if (cudaGetLastError() != cudaSuccess) return WX_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return WX_ERR_CUDA;
    int rc = mlp_check(w);
    if (rc) return rc;
    if (loss_per_epoch) {
      float l = 0.f;
      cudaMemcpy(&l, w->loss, 4, cudaMemcpyDeviceToHost);
      loss_per_epoch[ep] = l / (float)nb;
    }
  }
  return WX_OK;
}

}  // extern "C"
