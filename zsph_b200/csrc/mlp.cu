// Learned-corrector network on the fifth-generation tensor cores (sm_100a).
//
// MLP 32 -> 128 -> 128 -> 4, SiLU, bf16 operands, fp32 accumulation in TMEM.
// One CTA of 128 threads owns one 128-row tile at a time: thread t <-> tile
// row t <-> TMEM lane t.  Thread 0 issues tcgen05.mma from shared-memory
// operands (layout: umma.cuh) and commits to one mbarrier; every thread then
// reads its row of the accumulator with tcgen05.ld, applies bias and SiLU and
// writes the next layer's bf16 operand row back to shared memory.
//
// Modes of the one kernel:
//   kPredict  standardized outputs per row -> global memory
//   kCorrect  learned corrector epilogue: acceleration and drho/dt of the
//             corrector stage = predictor-stage values + de-standardized
//             network output, then the time_int.cu:50-92 correction in place
//   kTrain    forward + backward of the weighted squared error; the weight
//             gradients accumulate in TMEM across all tiles of the CTA
//             (dW = G^T H with G and H read MN-major from the same buffers
//             the forward pass wrote K-major) and leave as one partial row
//             per CTA, reduced deterministically by the Adam kernel.
// SiLU(z) = z * s(z), s(z) = 0.5 tanh(z/2) + 0.5 with the MUFU tanh; its
// derivative s (1 + z (1 - s)) is kept as bf16 for the backward pass.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "integrate.cuh"
#include "umma.cuh"
#include "zsph_internal.cuh"

namespace zsph {
namespace {

using namespace umma;

constexpr int kIn = ZSPH_MLP_IN, kHid = ZSPH_MLP_HID, kOut = ZSPH_MLP_OUT, kOutPad = 16;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kOut * kHid, kNParam = kOffB3 + kOut;
constexpr int kNPartial = ZSPH_MLP_NPARTIAL;
static_assert(kNParam == ZSPH_MLP_NPARAM, "parameter layout");
static_assert(kNPartial >= kNParam + 1 && kNPartial % 4 == 0, "partial row layout");

enum { kPredict = 0, kCorrect = 1, kTrain = 2 };

// Shared-memory map (bytes).  Inference reuses the layer-1 activation buffer
// for layer 2 and needs no backward buffers: 88 KB, two CTAs per SM.
template <int MODE> struct Smem {
  static constexpr bool TR = MODE == kTrain;
  static constexpr uint32_t X = 0;                                 // 128 x 32
  static constexpr uint32_t H1 = X + 8192;                         // 128 x 128
  static constexpr uint32_t H2 = TR ? H1 + 32768 : H1;             // 128 x 128
  static constexpr uint32_t S1 = H2 + 32768;                       // silu'(z1), then G1
  static constexpr uint32_t S2 = TR ? S1 + 32768 : S1;             // silu'(z2), then G2
  static constexpr uint32_t G3 = TR ? S2 + 32768 : S2;             // 128 x 16
  static constexpr uint32_t ONES = TR ? G3 + 4096 : G3;            // 128 x 16, column 0 = 1
  static constexpr uint32_t W1 = TR ? ONES + 4096 : ONES;          // 128 x 32
  static constexpr uint32_t W2 = W1 + 8192;                        // 128 x 128
  static constexpr uint32_t W3 = W2 + 32768;                       // 16 x 128
  static constexpr uint32_t B = W3 + 4096;                         // b1, b2, b3 (fp32)
  static constexpr uint32_t CTRL = B + 1088;                       // mbarrier, tmem address, reductions
  static constexpr uint32_t BYTES = CTRL + 256;
  // dynamic shared memory requested: more than BYTES so that every operand
  // span an MMA can address (start + 15 blocks at either byte offset) lies
  // inside the allocation; inference still fits two CTAs per SM
  static constexpr uint32_t ALLOC = TR ? 227 * 1024 : 113 * 1024;
  static constexpr uint32_t NCOLS = TR ? 512 : 256;                // TMEM columns
};
static_assert(Smem<kTrain>::BYTES <= 227 * 1024, "train shared memory");
static_assert(Smem<kCorrect>::BYTES <= Smem<kCorrect>::ALLOC && Smem<kTrain>::BYTES <= Smem<kTrain>::ALLOC, "");
static_assert(2 * (Smem<kCorrect>::ALLOC + 1024) <= 228 * 1024, "two inference CTAs per SM");

// TMEM column map (fp32 columns; lane = tile row, or output unit for dW)
constexpr uint32_t cZ1 = 0;     // z1, later dH2
constexpr uint32_t cZ2 = 128;   // z2, later dH1
constexpr uint32_t cDW2 = 256;  // dW2 [out][in]
constexpr uint32_t cDW1 = 384;  // dW1 [out][in]
constexpr uint32_t cZ3 = 416;   // z3 (train); inference puts z3 at cZ1
constexpr uint32_t cDW3 = 432;  // dW3^T [in][out]
constexpr uint32_t cDB1 = 448;  // db1 in column 0
constexpr uint32_t cDB2 = 464;  // db2 in column 0

constexpr uint32_t kId128x128KK = idesc_bf16(128, 128, 0, 0);
constexpr uint32_t kId128x16KK = idesc_bf16(128, 16, 0, 0);
constexpr uint32_t kId128x16MM = idesc_bf16(128, 16, 1, 1);
constexpr uint32_t kId128x128KM = idesc_bf16(128, 128, 0, 1);
constexpr uint32_t kId128x128MM = idesc_bf16(128, 128, 1, 1);
constexpr uint32_t kId128x32MM = idesc_bf16(128, 32, 1, 1);

struct Net {
  const __nv_bfloat16* w1;   // [128][32]
  const __nv_bfloat16* w2;   // [128][128]
  const __nv_bfloat16* w3p;  // [16][128], rows 4..15 zero
  const float* b1;
  const float* b2;
  const float* b3;
};

struct MlpArgs {
  Net net;
  const uint4* x;       // feature tiles, 512 uint4 each
  int ntiles;           // tiles to visit
  const int* tile_ids;  // tile indirection (training batches), or null
  int nrows;            // valid rows (predict / correct)
  float4* out;          // predict: standardized outputs
  const float4* y;      // train: standardized targets per row
  const float* wrow;    // train: loss weight per row
  float inv_wsum;
  float* partial;       // train: [gridDim.x][kNPartial]
  int* flags;
  // correct
  KParams kp;
  zsph_ptc_t ptc;  // state after the predictor (n+1/2 plus tmp_* = n), corrected in place
  float4* acc;          // predictor-stage (acc, drho/dt) in, corrector-stage out
  const float4* dprev;  // D: predictor-stage value minus the previous corrector value
  float4 oa, ob;        // residual = yhat * oa + ob (de-standardized, dimensional)
};

__device__ __forceinline__ float tanh_mufu(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(uint32_t u) {
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xFFFF0000u));
}

// row-major bf16 [R][C] in global memory -> core-matrix buffer
__device__ void load_operand(unsigned char* dst, const __nv_bfloat16* src, int R, int C) {
  const int per_row = C / 8;
  for (int k = threadIdx.x; k < R * per_row; k += blockDim.x) {
    const int r = k / per_row, cb = k - r * per_row;
    *reinterpret_cast<uint4*>(dst + core_off(R, r, cb * 8)) =
        *reinterpret_cast<const uint4*>(src + (size_t)r * C + cb * 8);
  }
}

// z = acc + bias -> h = silu(z) (and s = silu'(z) when training), bf16 rows
template <bool TR>
__device__ __forceinline__ void hidden_rows(uint32_t taddr, const float* bias, unsigned char* sH, unsigned char* sS,
                                            int row) {
#pragma unroll 1
  for (int c0 = 0; c0 < kHid; c0 += 32) {
    float v[32];
    tmem_ld32(taddr + c0, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t h[4], s[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = q * 8 + 2 * e;
        const float z0 = v[j] + bias[c0 + j], z1 = v[j + 1] + bias[c0 + j + 1];
        const float s0 = fmaf(0.5f, tanh_mufu(0.5f * z0), 0.5f), s1 = fmaf(0.5f, tanh_mufu(0.5f * z1), 0.5f);
        h[e] = pack_bf16(z0 * s0, z1 * s1);
        if (TR) s[e] = pack_bf16(s0 * fmaf(z0, 1.0f - s0, 1.0f), s1 * fmaf(z1, 1.0f - s1, 1.0f));
      }
      const uint32_t off = core_off(128, row, c0 + q * 8);
      *reinterpret_cast<uint4*>(sH + off) = make_uint4(h[0], h[1], h[2], h[3]);
      if (TR) *reinterpret_cast<uint4*>(sS + off) = make_uint4(s[0], s[1], s[2], s[3]);
    }
  }
}

// G = dH (TMEM) * silu' (bf16 in sS), written over sS
__device__ __forceinline__ void grad_rows(uint32_t taddr, unsigned char* sS, int row) {
#pragma unroll 1
  for (int c0 = 0; c0 < kHid; c0 += 32) {
    float v[32];
    tmem_ld32(taddr + c0, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint4* p = reinterpret_cast<uint4*>(sS + core_off(128, row, c0 + q * 8));
      const uint4 s = *p;
      const uint32_t sv[4] = {s.x, s.y, s.z, s.w};
      uint32_t g[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 d = unpack_bf16(sv[e]);
        const int j = q * 8 + 2 * e;
        g[e] = pack_bf16(v[j] * d.x, v[j + 1] * d.y);
      }
      *p = make_uint4(g[0], g[1], g[2], g[3]);
    }
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int MODE>
__global__ void __launch_bounds__(128, 1) k_mlp(MlpArgs a) {
  using L = Smem<MODE>;
  constexpr bool TR = L::TR;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* sX = sm + L::X;
  unsigned char* sH1 = sm + L::H1;
  unsigned char* sH2 = sm + L::H2;
  unsigned char* sS1 = sm + L::S1;
  unsigned char* sS2 = sm + L::S2;
  unsigned char* sG3 = sm + L::G3;
  unsigned char* sOnes = sm + L::ONES;
  unsigned char* sW1 = sm + L::W1;
  unsigned char* sW2 = sm + L::W2;
  unsigned char* sW3 = sm + L::W3;
  float* sB1 = reinterpret_cast<float*>(sm + L::B);
  float* sB2 = sB1 + kHid;
  float* sB3 = sB2 + kHid;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::CTRL);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + L::CTRL + 8);
  float* s_red = reinterpret_cast<float*>(sm + L::CTRL + 16);  // [4 warps][8]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tmem_alloc(s_tmem, L::NCOLS);
    tmem_relinquish();
  }
  if (tid == 0) mbar_init(bar, 1);
  load_operand(sW1, a.net.w1, kHid, kIn);
  load_operand(sW2, a.net.w2, kHid, kHid);
  load_operand(sW3, a.net.w3p, kOutPad, kHid);
  for (int k = tid; k < kHid; k += 128) {
    sB1[k] = a.net.b1[k];
    sB2[k] = a.net.b2[k];
  }
  if (tid < kOut) sB3[tid] = a.net.b3[tid];
  if (TR) {
    // ones operand [128 rows][16]: column 0 = 1.0 (bf16 0x3F80)
    *reinterpret_cast<uint4*>(sOnes + core_off(128, tid, 0)) = make_uint4(0x3F80u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(sOnes + core_off(128, tid, 8)) = make_uint4(0u, 0u, 0u, 0u);
  }
  fence_proxy_async();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tb = *s_tmem;
  const uint32_t lrow = (uint32_t)(warp * 32) << 16;  // this warp's TMEM lanes

  uint32_t phase = 0;
  bool failed = false;
  bool first = true;  // no tile accumulated into the dW columns yet
  float r_db3[kOut] = {0.f, 0.f, 0.f, 0.f}, r_loss = 0.f;

  // bounded wait for the MMAs committed last; false (on every thread) if it timed out
  auto wait_mma = [&]() -> bool {
    const bool ok = mbar_wait(bar, phase);
    if (__syncthreads_or(ok ? 0 : 1)) return false;
    phase ^= 1u;
    fence_after();
    return true;
  };

  for (int it = blockIdx.x; it < a.ntiles; it += gridDim.x) {
    const int tile = a.tile_ids ? a.tile_ids[it] : it;
    const int row = tile * 128 + tid;
    const uint4* src = a.x + (size_t)tile * 512;
#pragma unroll
    for (int k = 0; k < 4; ++k) reinterpret_cast<uint4*>(sX)[tid + 128 * k] = src[tid + 128 * k];
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      mma(tb + cZ1, kmaj(sX, 128, 0), kmaj(sW1, 128, 0), kId128x128KK, false);
      mma(tb + cZ1, kmaj(sX, 128, 1), kmaj(sW1, 128, 1), kId128x128KK, true);
      commit(bar);
    }
    if (!wait_mma()) { failed = true; break; }
    hidden_rows<TR>(tb + lrow + cZ1, sB1, sH1, sS1, tid);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
#pragma unroll
      for (int k = 0; k < 8; ++k) mma(tb + cZ2, kmaj(sH1, 128, k), kmaj(sW2, 128, k), kId128x128KK, k > 0);
      commit(bar);
    }
    if (!wait_mma()) { failed = true; break; }
    hidden_rows<TR>(tb + lrow + cZ2, sB2, sH2, sS2, tid);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    const uint32_t cz3 = TR ? cZ3 : cZ1;
    if (tid == 0) {
      fence_after();
#pragma unroll
      for (int k = 0; k < 8; ++k) mma(tb + cz3, kmaj(sH2, 128, k), kmaj(sW3, kOutPad, k), kId128x16KK, k > 0);
      commit(bar);
    }
    if (!wait_mma()) { failed = true; break; }
    float z3[16];
    tmem_ld16(tb + lrow + cz3, z3);
    float yh[kOut];
#pragma unroll
    for (int k = 0; k < kOut; ++k) yh[k] = z3[k] + sB3[k];

    if (MODE == kPredict) {
      if (row < a.nrows) a.out[row] = make_float4(yh[0], yh[1], yh[2], yh[3]);
    } else if (MODE == kCorrect) {
      if (row < a.nrows && a.ptc.type[row] == 1) {
        // corrector stage = linear extrapolation a_n + D + learned residual
        float4 acc = a.acc[row];
        const float4 d = a.dprev[row];
        acc.x += d.x + fmaf(yh[0], a.oa.x, a.ob.x);
        acc.y += d.y + fmaf(yh[1], a.oa.y, a.ob.y);
        acc.z += d.z + fmaf(yh[2], a.oa.z, a.ob.z);
        acc.w += d.w + fmaf(yh[3], a.oa.w, a.ob.w);
        a.acc[row] = acc;
        if (!isfinite(acc.x + acc.y + acc.z + acc.w)) atomicOr(a.flags, ZSPH_FLAG_NAN);
        integrate_one<2>(a.kp, a.ptc, a.ptc, row, acc);
      }
    } else {
      // d loss / d yhat, loss and db3 partial sums (fp32, per thread)
      const float4 yt = a.y[row];
      const float w = a.wrow[row];
      const float yv[kOut] = {yt.x, yt.y, yt.z, yt.w};
      float g[kOut];
#pragma unroll
      for (int k = 0; k < kOut; ++k) {
        const float d = yh[k] - yv[k];
        r_loss = fmaf(w * d, d, r_loss);
        g[k] = 2.0f * w * d * a.inv_wsum;
        r_db3[k] += g[k];
      }
      *reinterpret_cast<uint4*>(sG3 + core_off(128, tid, 0)) =
          make_uint4(pack_bf16(g[0], g[1]), pack_bf16(g[2], g[3]), 0u, 0u);
      *reinterpret_cast<uint4*>(sG3 + core_off(128, tid, 8)) = make_uint4(0u, 0u, 0u, 0u);
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        // dW3^T[in][out] += H2^T G3 ; dH2 = G3 W3
#pragma unroll
        for (int k = 0; k < 8; ++k)
          mma(tb + cDW3, mnmaj(sH2, 128, k), mnmaj(sG3, 128, k), kId128x16MM, !(first && k == 0));
        mma(tb + cZ1, kmaj(sG3, 128, 0), mnmaj(sW3, kOutPad, 0), kId128x128KM, false);
        commit(bar);
      }
      if (!wait_mma()) { failed = true; break; }
      grad_rows(tb + lrow + cZ1, sS2, tid);  // G2
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        // dW2[out][in] += G2^T H1 ; db2 += G2^T 1 ; dH1 = G2 W2
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          mma(tb + cDW2, mnmaj(sS2, 128, k), mnmaj(sH1, 128, k), kId128x128MM, !(first && k == 0));
          mma(tb + cDB2, mnmaj(sS2, 128, k), mnmaj(sOnes, 128, k), kId128x16MM, !(first && k == 0));
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) mma(tb + cZ2, kmaj(sS2, 128, k), mnmaj(sW2, 128, k), kId128x128KM, k > 0);
        commit(bar);
      }
      if (!wait_mma()) { failed = true; break; }
      grad_rows(tb + lrow + cZ2, sS1, tid);  // G1
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        // dW1[out][in] += G1^T X ; db1 += G1^T 1
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          mma(tb + cDW1, mnmaj(sS1, 128, k), mnmaj(sX, 128, k), kId128x32MM, !(first && k == 0));
          mma(tb + cDB1, mnmaj(sS1, 128, k), mnmaj(sOnes, 128, k), kId128x16MM, !(first && k == 0));
        }
        commit(bar);
      }
      if (!wait_mma()) { failed = true; break; }
      first = false;
    }
    fence_before();
    __syncthreads();  // TMEM columns and operand buffers free for the next tile
  }

  if (TR && !failed) {
    float* P = a.partial + (size_t)blockIdx.x * kNPartial;
    if (first) {
      for (int k = tid; k < kNPartial; k += 128) P[k] = 0.f;
    } else {
      float v[32];
#pragma unroll 1
      for (int c0 = 0; c0 < kHid; c0 += 32) {
        tmem_ld32(tb + lrow + cDW2 + c0, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) P[kOffW2 + tid * kHid + c0 + j] = v[j];
      }
      tmem_ld32(tb + lrow + cDW1, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) P[kOffW1 + tid * kIn + j] = v[j];
      float u[16];
      tmem_ld16(tb + lrow + cDW3, u);
#pragma unroll
      for (int k = 0; k < kOut; ++k) P[kOffW3 + k * kHid + tid] = u[k];
      tmem_ld16(tb + lrow + cDB1, u);
      P[kOffB1 + tid] = u[0];
      tmem_ld16(tb + lrow + cDB2, u);
      P[kOffB2 + tid] = u[0];
    }
    // db3 and the loss: warp sums, then warps in order
#pragma unroll
    for (int k = 0; k < kOut; ++k) r_db3[k] = warp_sum(r_db3[k]);
    r_loss = warp_sum(r_loss);
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < kOut; ++k) s_red[warp * 8 + k] = r_db3[k];
      s_red[warp * 8 + 4] = r_loss;
    }
    __syncthreads();
    if (tid < kOut + 1) {
      float s = 0.f;
      for (int w = 0; w < 4; ++w) s += s_red[w * 8 + tid];
      P[tid < kOut ? kOffB3 + tid : kNParam] = s;
    }
    if (tid >= kOut + 1 && tid < kNPartial - kNParam + kOut) P[kNParam + 1 + (tid - kOut - 1)] = 0.f;
  }

  fence_before();
  __syncthreads();
  if (failed) {
    // report, let the MMAs in flight land (bounded), then release TMEM
    if (tid == 0) atomicOr(a.flags, ZSPH_FLAG_TIMEOUT);
    mbar_wait(bar, phase);
    __syncthreads();
  }
  if (warp == 0) tmem_dealloc(tb, L::NCOLS);
}

// Adam (fp32, no weight decay) with a deterministic reduction of the
// partial rows; every operation rounds separately (no contraction) so a
// float32 host restatement reproduces it bit for bit.
__global__ void k_adam(float* w, float* m1, float* m2, const float* partial, int nparts, float lr, float b1, float b2,
                       float eps, float bc1, float bc2, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3p) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kNParam) return;
  float g = 0.f;
  for (int c = 0; c < nparts; ++c) g = __fadd_rn(g, partial[(size_t)c * kNPartial + k]);
  const float m = __fadd_rn(__fmul_rn(b1, m1[k]), __fmul_rn(__fsub_rn(1.0f, b1), g));
  const float v = __fadd_rn(__fmul_rn(b2, m2[k]), __fmul_rn(__fsub_rn(1.0f, b2), __fmul_rn(g, g)));
  m1[k] = m;
  m2[k] = v;
  const float step = __fdiv_rn(__fmul_rn(lr, __fdiv_rn(m, bc1)), __fadd_rn(__fsqrt_rn(__fdiv_rn(v, bc2)), eps));
  const float wk = __fsub_rn(w[k], step);
  w[k] = wk;
  if (k < kOffB1) w1[k - kOffW1] = __float2bfloat16_rn(wk);
  else if (k >= kOffW2 && k < kOffB2) w2[k - kOffW2] = __float2bfloat16_rn(wk);
  else if (k >= kOffW3 && k < kOffB3) w3p[k - kOffW3] = __float2bfloat16_rn(wk);
}

// fp32 master -> bf16 weights (rows 4..15 of w3p stay zero)
__global__ void k_refresh(const float* w, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3p) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kNParam) return;
  if (k < kOffB1) w1[k - kOffW1] = __float2bfloat16_rn(w[k]);
  else if (k >= kOffW2 && k < kOffB2) w2[k - kOffW2] = __float2bfloat16_rn(w[k]);
  else if (k >= kOffW3 && k < kOffB3) w3p[k - kOffW3] = __float2bfloat16_rn(w[k]);
}

struct PackArgs {
  float mean[kIn], inv_std[kIn];
};

// rows [n][32] fp32 -> standardized bf16 tiles; one thread per 8-feature chunk
__global__ void k_pack_rows(const float* rows, int n, PackArgs pa, unsigned char* tiles, int ntiles) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = k >> 2, cb = k & 3;
  if (r >= ntiles * 128) return;
  uint32_t u[4] = {0u, 0u, 0u, 0u};
  if (r < n) {
    const float4 a = reinterpret_cast<const float4*>(rows)[(size_t)r * 8 + cb * 2];
    const float4 b = reinterpret_cast<const float4*>(rows)[(size_t)r * 8 + cb * 2 + 1];
    const float x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int c = cb * 8 + 2 * e;
      u[e] = pack_bf16((x[2 * e] - pa.mean[c]) * pa.inv_std[c], (x[2 * e + 1] - pa.mean[c + 1]) * pa.inv_std[c + 1]);
    }
  }
  *reinterpret_cast<uint4*>(tiles + (size_t)(r >> 7) * 8192 + core_off(128, r & 127, cb * 8)) =
      make_uint4(u[0], u[1], u[2], u[3]);
}

// The kernels' dynamic shared-memory opt-in and the SM count belong to one
// device context: they are set up on the first launch in each context of
// each device (the current one), and again after the context changes
// (cudaDeviceReset, for example).  A process may use several devices.
constexpr int kMaxDevices = 64;
struct DevInit {
  unsigned long long ctx = 0;  // current_context_id() when set up
  int sms = 0;
  bool done = false;
};
std::mutex g_init_mu;
DevInit g_init[kMaxDevices];

// Sets up the current device's context if needed; *sms receives its SM count.
cudaError_t init_mlp_kernels(int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_init_mu);
  DevInit& d = g_init[dev];
  const unsigned long long ctx = current_context_id();
  if (!d.done || ctx == 0 || ctx != d.ctx) {
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (!e) e = cudaFuncSetAttribute(k_mlp<kPredict>, cudaFuncAttributeMaxDynamicSharedMemorySize, Smem<kPredict>::ALLOC);
    if (!e) e = cudaFuncSetAttribute(k_mlp<kCorrect>, cudaFuncAttributeMaxDynamicSharedMemorySize, Smem<kCorrect>::ALLOC);
    if (!e) e = cudaFuncSetAttribute(k_mlp<kTrain>, cudaFuncAttributeMaxDynamicSharedMemorySize, Smem<kTrain>::ALLOC);
    if (e) {
      d.done = false;
      return e;
    }
    d.sms = n;
    d.ctx = current_context_id();
    d.done = true;
  }
  *sms = d.sms;
  return cudaSuccess;
}

int fail(int code, const std::string& msg) {
  record_library_error(msg);
  return code;
}
int fail_cuda(cudaError_t e, const char* what) {
  return fail(ZSPH_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// splitmix64
uint64_t mix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__nv_bfloat16* bf(void* p) { return static_cast<__nv_bfloat16*>(p); }

}  // namespace
}  // namespace zsph

namespace zsph {

int mlp_sm_count() {
  int sms = 0;
  return init_mlp_kernels(&sms) ? 0 : sms;
}

Net mlp_net(const Mlp& m) {
  return Net{bf(m.w1), bf(m.w2), bf(m.w3p), m.w + kOffB1, m.w + kOffB2, m.w + kOffB3};
}

// learned-corrector epilogue over the state after the predictor (learn.cu)
cudaError_t launch_mlp_correct(const Mlp& m, const KParams& kp, const void* tiles, const zsph_ptc_t& ptc,
                               float4* acc, const float4* dprev, float4 oa, float4 ob, int* flags, cudaStream_t st) {
  int sms = 0;
  cudaError_t e = init_mlp_kernels(&sms);
  if (e) return e;
  MlpArgs a{};
  a.net = mlp_net(m);
  a.x = static_cast<const uint4*>(tiles);
  a.ntiles = (kp.n + 127) / 128;
  a.nrows = kp.n;
  a.flags = flags;
  a.kp = kp;
  a.ptc = ptc;
  a.acc = acc;
  a.dprev = dprev;
  a.oa = oa;
  a.ob = ob;
  const int grid = std::min(a.ntiles, 2 * sms);
  k_mlp<kCorrect><<<grid, 128, Smem<kCorrect>::ALLOC, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const Mlp& m, const void* tiles, int n, float* out, int* flags,
                               cudaStream_t st) {
  int sms = 0;
  cudaError_t e = init_mlp_kernels(&sms);
  if (e) return e;
  MlpArgs a{};
  a.net = mlp_net(m);
  a.x = static_cast<const uint4*>(tiles);
  a.ntiles = (n + 127) / 128;
  a.nrows = n;
  a.out = reinterpret_cast<float4*>(out);
  a.flags = flags;
  const int grid = std::min(a.ntiles, 2 * sms);
  if (grid > 0) k_mlp<kPredict><<<grid, 128, Smem<kPredict>::ALLOC, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const Mlp& m, const void* tiles, const float* y, const float* w, const int* ids,
                            int ntiles, float inv_wsum, float* partial, int* nparts, int* flags, cudaStream_t st) {
  int sms = 0;
  cudaError_t e = init_mlp_kernels(&sms);
  if (e) return e;
  MlpArgs a{};
  a.net = mlp_net(m);
  a.x = static_cast<const uint4*>(tiles);
  a.ntiles = ntiles;
  a.tile_ids = ids;
  a.y = reinterpret_cast<const float4*>(y);
  a.wrow = w;
  a.inv_wsum = inv_wsum;
  a.partial = partial;
  a.flags = flags;
  const int grid = std::max(1, std::min(ntiles, sms));
  k_mlp<kTrain><<<grid, 128, Smem<kTrain>::ALLOC, st>>>(a);
  *nparts = grid;
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(Mlp& m, const float* partial, int nparts, float lr, float b1, float b2, float eps,
                            cudaStream_t st) {
  m.step += 1;
  const float bc1 = (float)(1.0 - std::pow((double)b1, (double)m.step));
  const float bc2 = (float)(1.0 - std::pow((double)b2, (double)m.step));
  k_adam<<<(kNParam + 255) / 256, 256, 0, st>>>(m.w, m.m1, m.m2, partial, nparts, lr, b1, b2, eps, bc1, bc2, bf(m.w1),
                                                bf(m.w2), bf(m.w3p));
  return cudaGetLastError();
}

cudaError_t launch_mlp_pack(const float* rows, int n, const float* mean, const float* inv_std, void* tiles,
                            cudaStream_t st) {
  PackArgs pa;
  for (int c = 0; c < kIn; ++c) {
    pa.mean[c] = mean ? mean[c] : 0.f;
    pa.inv_std[c] = inv_std ? inv_std[c] : 1.f;
  }
  const int ntiles = (n + 127) / 128;
  const int threads = ntiles * 128 * 4;
  if (threads > 0)
    k_pack_rows<<<(threads + 255) / 256, 256, 0, st>>>(rows, n, pa, static_cast<unsigned char*>(tiles), ntiles);
  return cudaGetLastError();
}

}  // namespace zsph

using namespace zsph;

extern "C" {

int zsph_mlp_create(unsigned long long seed, zsph_mlp_t** out) {
  if (!out) return fail(ZSPH_EINVAL, "zsph_mlp_create: out is NULL");
  *out = nullptr;
  auto* m = new zsph_mlp();
  cudaError_t e = cudaMalloc(&m->w, sizeof(float) * kNParam * 3);
  if (!e) e = cudaMalloc(&m->w1, sizeof(__nv_bfloat16) * (kHid * kIn + kHid * kHid + kOutPad * kHid));
  if (e) {
    cudaFree(m->w);
    delete m;
    return fail(ZSPH_ENOMEM, std::string("zsph_mlp_create: ") + cudaGetErrorString(e));
  }
  m->m1 = m->w + kNParam;
  m->m2 = m->w + 2 * kNParam;
  m->w2 = bf(m->w1) + kHid * kIn;
  m->w3p = bf(m->w2) + kHid * kHid;
  for (int k = 0; k < kFeat; ++k) {
    m->in_mean[k] = 0.f;
    m->in_inv_std[k] = 1.f;
  }
  for (int k = 0; k < kOut; ++k) {
    m->out_mean[k] = 0.f;
    m->out_std[k] = 1.f;
  }
  std::vector<float> h(kNParam, 0.f);
  uint64_t s = seed;
  auto uni = [&](float bound) { return (float)(((mix64(s) >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * bound; };
  for (int k = 0; k < kHid * kIn; ++k) h[kOffW1 + k] = uni(1.0f / std::sqrt((float)kIn));
  for (int k = 0; k < kHid * kHid; ++k) h[kOffW2 + k] = uni(1.0f / std::sqrt((float)kHid));
  for (int k = 0; k < kOut * kHid; ++k) h[kOffW3 + k] = uni(1.0f / std::sqrt((float)kHid));
  e = cudaMemset(m->w, 0, sizeof(float) * kNParam * 3);
  if (!e) e = cudaMemset(m->w1, 0, sizeof(__nv_bfloat16) * (kHid * kIn + kHid * kHid + kOutPad * kHid));
  if (!e) e = cudaMemcpy(m->w, h.data(), sizeof(float) * kNParam, cudaMemcpyHostToDevice);
  if (!e) {
    k_refresh<<<(kNParam + 255) / 256, 256>>>(m->w, bf(m->w1), bf(m->w2), bf(m->w3p));
    e = cudaDeviceSynchronize();
  }
  if (e) {
    zsph_mlp_destroy(m);
    return fail_cuda(e, "zsph_mlp_create");
  }
  *out = m;
  return ZSPH_OK;
}

int zsph_mlp_destroy(zsph_mlp_t* m) {
  if (!m) return ZSPH_OK;
  cudaFree(m->w);
  cudaFree(m->w1);
  delete m;
  return ZSPH_OK;
}

int zsph_mlp_set_params(zsph_mlp_t* m, const float* params) {
  if (!m || !params) return fail(ZSPH_EINVAL, "zsph_mlp_set_params: bad argument");
  cudaError_t e = cudaMemcpy(m->w, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice);
  if (!e) {
    k_refresh<<<(kNParam + 255) / 256, 256>>>(m->w, bf(m->w1), bf(m->w2), bf(m->w3p));
    e = cudaDeviceSynchronize();
  }
  return e ? fail_cuda(e, "zsph_mlp_set_params") : ZSPH_OK;
}

int zsph_mlp_get_params(zsph_mlp_t* m, float* params) {
  if (!m || !params) return fail(ZSPH_EINVAL, "zsph_mlp_get_params: bad argument");
  cudaError_t e = cudaMemcpy(params, m->w, sizeof(float) * kNParam, cudaMemcpyDeviceToHost);
  return e ? fail_cuda(e, "zsph_mlp_get_params") : ZSPH_OK;
}

int zsph_mlp_set_moments(zsph_mlp_t* m, const float* m1, const float* m2, int step) {
  if (!m || !m1 || !m2 || step < 0) return fail(ZSPH_EINVAL, "zsph_mlp_set_moments: bad argument");
  cudaError_t e = cudaMemcpy(m->m1, m1, sizeof(float) * kNParam, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(m->m2, m2, sizeof(float) * kNParam, cudaMemcpyHostToDevice);
  m->step = step;
  return e ? fail_cuda(e, "zsph_mlp_set_moments") : ZSPH_OK;
}

int zsph_mlp_get_moments(zsph_mlp_t* m, float* m1, float* m2, int* step) {
  if (!m) return fail(ZSPH_EINVAL, "zsph_mlp_get_moments: bad argument");
  cudaError_t e = cudaSuccess;
  if (m1) e = cudaMemcpy(m1, m->m1, sizeof(float) * kNParam, cudaMemcpyDeviceToHost);
  if (!e && m2) e = cudaMemcpy(m2, m->m2, sizeof(float) * kNParam, cudaMemcpyDeviceToHost);
  if (step) *step = m->step;
  return e ? fail_cuda(e, "zsph_mlp_get_moments") : ZSPH_OK;
}

int zsph_mlp_set_norm(zsph_mlp_t* m, const float* in_mean, const float* in_inv_std, const float* out_mean,
                      const float* out_std) {
  if (!m || !in_mean || !in_inv_std || !out_mean || !out_std) return fail(ZSPH_EINVAL, "zsph_mlp_set_norm: bad argument");
  std::memcpy(m->in_mean, in_mean, sizeof m->in_mean);
  std::memcpy(m->in_inv_std, in_inv_std, sizeof m->in_inv_std);
  std::memcpy(m->out_mean, out_mean, sizeof m->out_mean);
  std::memcpy(m->out_std, out_std, sizeof m->out_std);
  return ZSPH_OK;
}

int zsph_mlp_get_norm(zsph_mlp_t* m, float* in_mean, float* in_inv_std, float* out_mean, float* out_std) {
  if (!m) return fail(ZSPH_EINVAL, "zsph_mlp_get_norm: bad argument");
  if (in_mean) std::memcpy(in_mean, m->in_mean, sizeof m->in_mean);
  if (in_inv_std) std::memcpy(in_inv_std, m->in_inv_std, sizeof m->in_inv_std);
  if (out_mean) std::memcpy(out_mean, m->out_mean, sizeof m->out_mean);
  if (out_std) std::memcpy(out_std, m->out_std, sizeof m->out_std);
  return ZSPH_OK;
}

int zsph_mlp_pack(const float* rows, int n, const float* mean, const float* inv_std, void* tiles, void* stream) {
  if (n < 0 || (n > 0 && (!rows || !tiles))) return fail(ZSPH_EINVAL, "zsph_mlp_pack: bad argument");
  if ((reinterpret_cast<uintptr_t>(rows) | reinterpret_cast<uintptr_t>(tiles)) & 15)
    return fail(ZSPH_EINVAL, "zsph_mlp_pack: rows and tiles must be 16-byte aligned");
  cudaError_t e = launch_mlp_pack(rows, n, mean, inv_std, tiles, static_cast<cudaStream_t>(stream));
  return e ? fail_cuda(e, "zsph_mlp_pack") : ZSPH_OK;
}

int zsph_mlp_forward(zsph_mlp_t* m, const void* tiles, int n, float* out, void* stream) {
  if (!m || n < 0 || (n > 0 && (!tiles || !out))) return fail(ZSPH_EINVAL, "zsph_mlp_forward: bad argument");
  if ((reinterpret_cast<uintptr_t>(tiles) | reinterpret_cast<uintptr_t>(out)) & 15)
    return fail(ZSPH_EINVAL, "zsph_mlp_forward: tiles and out must be 16-byte aligned");
  int* flags = nullptr;
  cudaError_t e = cudaMalloc(&flags, sizeof(int));
  if (!e) e = cudaMemset(flags, 0, sizeof(int));
  if (!e) e = launch_mlp_forward(*m, tiles, n, out, flags, static_cast<cudaStream_t>(stream));
  int f = 0;
  if (!e) e = cudaMemcpyAsync(&f, flags, sizeof(int), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream));
  if (!e) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  cudaFree(flags);
  if (e) return fail_cuda(e, "zsph_mlp_forward");
  return (f & ZSPH_FLAG_TIMEOUT) ? fail(ZSPH_ETIMEOUT, "zsph_mlp_forward: tensor-core wait timed out") : ZSPH_OK;
}

int zsph_mlp_grad(zsph_mlp_t* m, const void* tiles, const float* y, const float* w, const int* tile_ids, int ntiles,
                  float inv_wsum, float* partial, int* nparts, void* stream) {
  if (!m || !tiles || !y || !w || !partial || !nparts || ntiles < 0)
    return fail(ZSPH_EINVAL, "zsph_mlp_grad: bad argument");
  if ((reinterpret_cast<uintptr_t>(tiles) | reinterpret_cast<uintptr_t>(y)) & 15)
    return fail(ZSPH_EINVAL, "zsph_mlp_grad: tiles and y must be 16-byte aligned");
  int* flags = nullptr;
  cudaError_t e = cudaMalloc(&flags, sizeof(int));
  if (!e) e = cudaMemset(flags, 0, sizeof(int));
  if (!e)
    e = launch_mlp_grad(*m, tiles, y, w, tile_ids, ntiles, inv_wsum, partial, nparts, flags,
                        static_cast<cudaStream_t>(stream));
  int f = 0;
  if (!e) e = cudaMemcpyAsync(&f, flags, sizeof(int), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream));
  if (!e) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  cudaFree(flags);
  if (e) return fail_cuda(e, "zsph_mlp_grad");
  return (f & ZSPH_FLAG_TIMEOUT) ? fail(ZSPH_ETIMEOUT, "zsph_mlp_grad: tensor-core wait timed out") : ZSPH_OK;
}

int zsph_mlp_adam(zsph_mlp_t* m, const float* partial, int nparts, float lr, float beta1, float beta2, float eps,
                  void* stream) {
  if (!m || !partial || nparts <= 0) return fail(ZSPH_EINVAL, "zsph_mlp_adam: bad argument");
  cudaError_t e = launch_mlp_adam(*m, partial, nparts, lr, beta1, beta2, eps, static_cast<cudaStream_t>(stream));
  return e ? fail_cuda(e, "zsph_mlp_adam") : ZSPH_OK;
}

}  // extern "C"
