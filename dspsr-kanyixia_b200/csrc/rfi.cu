// rfi.cu -- a learned RFI-mask proposer in front of SpectralKurtosis.
//
// The reference zaps a (block, channel) of M samples when the spectral
// kurtosis estimator of either polarisation leaves [lower, upper]
// (SpectralKurtosis::detect_skfb, Signal/General/SpectralKurtosis.C:1105-1222).
// This proposer reads features of the same blocks -- the SK sums S1, S2 that
// SpectralKurtosis::compute forms (SpectralKurtosis.C:674-798) -- and
// proposes the mask with a small network trained on masks the SK stage itself
// produced.  Where its confidence is below a threshold the SK decision is
// used instead, and against SK its misses and false zaps are counted.
//
// Features of (block b, channel c), eight floats, all scaled by 16 (about
// one standard deviation of a Gaussian block at M = 1024) and clamped:
//   0, 1  log power of each polarisation, less the block's mean over channels
//   2, 3  V - 1 of each polarisation (the SK estimator, Nita & Gary 2010b eq. 8)
//   4, 5  the same for block b - 1 (0 at the first block)
//   6, 7  the same for block b + 1 (0 at the last block)
// Network, a 1-D convolution across channels of one block (3937 weights):
//   conv 8 -> 32, 3 taps, dilation 1, ReLU
//   conv 32 -> 32, 3 taps, dilation 2, ReLU
//   dot 32 -> 1 (logit), sigmoid = probability of "zap"
// Training (FP32 master weights, CUDA cores): forward, weighted binary
// cross-entropy, backward and Adam, one kernel each.  Inference: the two
// convolutions as BF16 GEMMs on the tensor cores (tcgen05.mma, FP32
// accumulation in tensor memory; im2col rows built in shared memory), bias,
// ReLU and the head in FP32, one block of 512 channels per CTA.

#include "dspsr_b200.h"
#include "context.h"
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <random>
#include <vector>

namespace b200 {

using namespace tc;

namespace {

constexpr int NF = 8, NH = 32, KT = 3;
constexpr int P_W1 = 0;
constexpr int P_B1 = P_W1 + NH * NF * KT;   // 768
constexpr int P_W2 = P_B1 + NH;             // 800
constexpr int P_B2 = P_W2 + NH * NH * KT;   // 3872
constexpr int P_W3 = P_B2 + NH;             // 3904
constexpr int P_B3 = P_W3 + NH;             // 3936
constexpr int NPARAM = P_B3 + 1;            // 3937
constexpr float FSCALE = 16.f;
constexpr int MAXCH = 512;                  // channels per block the inference kernel holds

// --------------------------------------------------------------------------
// features
// --------------------------------------------------------------------------

__device__ __forceinline__ float sk_v (float S1, float S2, float Mp, float Nd)
{
  if (Mp < 2.f || S1 <= 0.f) return 1.f;
  const float M_fac = (Mp * Nd + 1.f) / (Mp - 1.f);
  return M_fac * (Mp * (S2 / (S1 * S1)) - 1.f);
}

__device__ __forceinline__ float clampf (float x, float lo, float hi)
{
  return fminf (fmaxf (x, lo), hi);
}

// one CTA per block b; sums[((b*nchan + c)*npol + p)*2 + {0,1}] = (S1, S2)
__global__ void k_rfi_features (const float* __restrict__ sums, const unsigned* __restrict__ counts,
                                const uint64_t npart, const unsigned nchan, const unsigned npol,
                                const unsigned M, const unsigned Nd, float* __restrict__ X)
{
  const uint64_t b = blockIdx.x;
  __shared__ float s_red[32];
  float lsum = 0.f;
  auto power = [&] (uint64_t bb, unsigned c, unsigned p) {
    return sums[((bb * nchan + c) * npol + min (p, npol - 1)) * 2];
  };
  auto mprime = [&] (uint64_t bb, unsigned c) {
    return counts ? float (counts[bb * nchan + c]) : float (M);
  };
  for (unsigned c = threadIdx.x; c < nchan; c += blockDim.x)
    lsum += logf (fmaxf (power (b, c, 0), 1e-30f) / fmaxf (mprime (b, c), 1.f));
  for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync (0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = lsum;
  __syncthreads ();
  if (threadIdx.x < 32)
  {
    float v = threadIdx.x < (blockDim.x + 31) / 32 ? s_red[threadIdx.x] : 0.f;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync (0xffffffffu, v, o);
    if (threadIdx.x == 0) s_red[0] = v / float (nchan);
  }
  __syncthreads ();
  const float lmean = s_red[0];
  for (unsigned c = threadIdx.x; c < nchan; c += blockDim.x)
  {
    float f[NF];
    const float Mp = mprime (b, c);
    for (unsigned p = 0; p < 2; p++)
    {
      const uint64_t i0 = ((b * nchan + c) * npol + min (p, npol - 1)) * 2;
      f[p] = clampf (FSCALE * (logf (fmaxf (sums[i0], 1e-30f) / fmaxf (Mp, 1.f)) - lmean),
                     -64.f, 64.f);
      f[2 + p] = clampf (FSCALE * (sk_v (sums[i0], sums[i0 + 1], Mp, float (Nd)) - 1.f), -16.f,
                         64.f);
      float prev = 0.f, next = 0.f;
      if (b > 0)
      {
        const uint64_t j = (((b - 1) * nchan + c) * npol + min (p, npol - 1)) * 2;
        prev = clampf (FSCALE * (sk_v (sums[j], sums[j + 1], mprime (b - 1, c), float (Nd)) - 1.f),
                       -16.f, 64.f);
      }
      if (b + 1 < npart)
      {
        const uint64_t j = (((b + 1) * nchan + c) * npol + min (p, npol - 1)) * 2;
        next = clampf (FSCALE * (sk_v (sums[j], sums[j + 1], mprime (b + 1, c), float (Nd)) - 1.f),
                       -16.f, 64.f);
      }
      f[4 + p] = prev;
      f[6 + p] = next;
    }
    float4* dst = reinterpret_cast<float4*> (X + (b * nchan + c) * NF);
    dst[0] = make_float4 (f[0], f[1], f[2], f[3]);
    dst[1] = make_float4 (f[4], f[5], f[6], f[7]);
  }
}

// --------------------------------------------------------------------------
// training (FP32)
// --------------------------------------------------------------------------

// out[row][o] = act(b[o] + sum_{t,i} W[o][i][t] in[row + DIL (t-1)][i]) within the block
template <int CIN, int COUT, int DIL, bool RELU>
__global__ void k_conv_fwd (const float* __restrict__ in, const float* __restrict__ W,
                            const float* __restrict__ bias, float* __restrict__ out,
                            const unsigned nchan, const uint64_t nrows)
{
  __shared__ float sW[COUT * CIN * KT + COUT];
  for (int i = threadIdx.x; i < COUT * CIN * KT; i += blockDim.x) sW[i] = W[i];
  for (int i = threadIdx.x; i < COUT; i += blockDim.x) sW[COUT * CIN * KT + i] = bias[i];
  __syncthreads ();
  const uint64_t row = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int c = int (row % nchan);
  float acc[COUT];
#pragma unroll
  for (int o = 0; o < COUT; o++) acc[o] = sW[COUT * CIN * KT + o];
#pragma unroll
  for (int t = 0; t < KT; t++)
  {
    const int cc = c + DIL * (t - 1);
    if (cc < 0 || cc >= int (nchan)) continue;
    const float* x = in + (row + cc - c) * CIN;
#pragma unroll 4
    for (int i = 0; i < CIN; i++)
    {
      const float xi = x[i];
#pragma unroll
      for (int o = 0; o < COUT; o++) acc[o] = fmaf (sW[(o * CIN + i) * KT + t], xi, acc[o]);
    }
  }
#pragma unroll
  for (int o = 0; o < COUT; o++) out[row * COUT + o] = RELU ? fmaxf (acc[o], 0.f) : acc[o];
}

// logit, weighted BCE loss, dLoss/dA2 (through the ReLU) and the head's gradient
__global__ void k_rfi_head (const float* __restrict__ A2, const float* __restrict__ P,
                            const uint8_t* __restrict__ y, const uint64_t nrows, const float wpos,
                            const float inv_n, float* __restrict__ dA2, float* __restrict__ G,
                            float* __restrict__ loss)
{
  const uint64_t row = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const bool live = row < nrows;
  float a[NH];
  float z = P[P_B3];
#pragma unroll
  for (int o = 0; o < NH; o++)
  {
    a[o] = live ? A2[row * NH + o] : 0.f;
    z = fmaf (P[P_W3 + o], a[o], z);
  }
  const float yy = live && y[row] ? 1.f : 0.f;
  const float w = yy > 0.f ? wpos : 1.f;
  // log(1 + e^z) - y z, computed stably
  const float sp = fmaxf (z, 0.f) + log1pf (expf (-fabsf (z)));
  const float l = live ? w * (sp - yy * z) : 0.f;
  const float p = 1.f / (1.f + expf (-z));
  const float dz = live ? w * (p - yy) * inv_n : 0.f;
  if (live)
#pragma unroll
    for (int o = 0; o < NH; o++) dA2[row * NH + o] = a[o] > 0.f ? dz * P[P_W3 + o] : 0.f;
  // warp sums of the head's gradients and of the loss, one atomic per warp
  float gl = l, gb = dz;
  for (int s = 16; s; s >>= 1)
  {
    gl += __shfl_xor_sync (0xffffffffu, gl, s);
    gb += __shfl_xor_sync (0xffffffffu, gb, s);
  }
#pragma unroll
  for (int o = 0; o < NH; o++)
  {
    float g = dz * a[o];
    for (int s = 16; s; s >>= 1) g += __shfl_xor_sync (0xffffffffu, g, s);
    if ((threadIdx.x & 31) == 0) atomicAdd (G + P_W3 + o, g);
  }
  if ((threadIdx.x & 31) == 0)
  {
    atomicAdd (G + P_B3, gb);
    atomicAdd (loss, gl);
  }
}

// dW[o][i][t] += sum_rows dOut[row][o] in[row + DIL (t-1)][i]; db[o] += sum dOut[row][o].
// grid (row chunks, COUT)
template <int CIN, int COUT, int DIL>
__global__ void k_conv_bwd_w (const float* __restrict__ dOut, const float* __restrict__ in,
                              const unsigned nchan, const uint64_t nrows, float* __restrict__ gW,
                              float* __restrict__ gb)
{
  constexpr int NW = CIN * KT;
  __shared__ float s_acc[NW + 1];
  for (int i = threadIdx.x; i <= NW; i += blockDim.x) s_acc[i] = 0.f;
  __syncthreads ();
  const int o = blockIdx.y;
  float acc[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) acc[k] = 0.f;
  float bacc = 0.f;
  for (uint64_t row = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x; row < nrows;
       row += uint64_t (gridDim.x) * blockDim.x)
  {
    const float g = dOut[row * COUT + o];
    if (g == 0.f) continue;
    bacc += g;
    const int c = int (row % nchan);
#pragma unroll
    for (int t = 0; t < KT; t++)
    {
      const int cc = c + DIL * (t - 1);
      if (cc < 0 || cc >= int (nchan)) continue;
      const float* x = in + (row + cc - c) * CIN;
#pragma unroll
      for (int i = 0; i < CIN; i++) acc[i * KT + t] = fmaf (g, x[i], acc[i * KT + t]);
    }
  }
#pragma unroll
  for (int k = 0; k < NW; k++)
  {
    float v = acc[k];
    for (int s = 16; s; s >>= 1) v += __shfl_xor_sync (0xffffffffu, v, s);
    if ((threadIdx.x & 31) == 0) atomicAdd (s_acc + k, v);
  }
  for (int s = 16; s; s >>= 1) bacc += __shfl_xor_sync (0xffffffffu, bacc, s);
  if ((threadIdx.x & 31) == 0) atomicAdd (s_acc + NW, bacc);
  __syncthreads ();
  for (int k = threadIdx.x; k < NW; k += blockDim.x) atomicAdd (gW + o * NW + k, s_acc[k]);
  if (threadIdx.x == 0) atomicAdd (gb + o, s_acc[NW]);
}

// dIn[row][i] = relu'(in) * sum_{t,o} dOut[row - DIL (t-1)][o] W[o][i][t]
template <int CIN, int COUT, int DIL>
__global__ void k_conv_bwd_x (const float* __restrict__ dOut, const float* __restrict__ W,
                              const float* __restrict__ in, const unsigned nchan,
                              const uint64_t nrows, float* __restrict__ dIn)
{
  __shared__ float sW[COUT * CIN * KT];
  for (int i = threadIdx.x; i < COUT * CIN * KT; i += blockDim.x) sW[i] = W[i];
  __syncthreads ();
  const uint64_t row = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int c = int (row % nchan);
  float acc[CIN];
#pragma unroll
  for (int i = 0; i < CIN; i++) acc[i] = 0.f;
#pragma unroll
  for (int t = 0; t < KT; t++)
  {
    const int co = c - DIL * (t - 1);   // the output whose tap t reads this row
    if (co < 0 || co >= int (nchan)) continue;
    const float* g = dOut + (row + co - c) * COUT;
#pragma unroll 4
    for (int o = 0; o < COUT; o++)
    {
      const float go = g[o];
#pragma unroll
      for (int i = 0; i < CIN; i++) acc[i] = fmaf (go, sW[(o * CIN + i) * KT + t], acc[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < CIN; i++) dIn[row * CIN + i] = in[row * CIN + i] > 0.f ? acc[i] : 0.f;
}

__global__ void k_adam (float* __restrict__ P, float* __restrict__ G, float* __restrict__ m,
                        float* __restrict__ v, const int n, const float lr, const float c1,
                        const float c2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float mi = 0.9f * m[i] + 0.1f * g;
  const float vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi * c1) / (sqrtf (vi * c2) + 1e-8f);
  G[i] = 0.f;
}

// --------------------------------------------------------------------------
// inference on the tensor cores
// --------------------------------------------------------------------------

// operand layout: K-major, no swizzle, element (r, k) at (k/8)*LBO + r*16 + (k%8)*2
constexpr unsigned INF_ROWS = MAXCH;          // 4 tiles of 128
constexpr unsigned A_LBO = INF_ROWS * 16;     // 8192
constexpr unsigned K1 = 32;                   // 8 features x 3 taps, padded
constexpr unsigned K2 = NH * KT;              // 96
constexpr unsigned A_BYTES = (K2 / 8) * A_LBO;             // 98304
constexpr unsigned ACT_BYTES = INF_ROWS * NH * 2;          // 32768, row-major BF16
constexpr unsigned B_LBO = NH * 16;                        // 512: N = 32 rows
constexpr unsigned B1_BYTES = (K1 / 8) * B_LBO;            // 2048
constexpr unsigned B2_BYTES = (K2 / 8) * B_LBO;            // 6144
constexpr unsigned IMG_BYTES = B1_BYTES + B2_BYTES;
constexpr unsigned INF_SMEM = A_BYTES + ACT_BYTES + IMG_BYTES + 16;
constexpr unsigned INF_TMEM_COLS = 128;

// the FP32 weights as the BF16 B operands of both convolutions
__global__ void k_rfi_pack (const float* __restrict__ P, uint8_t* __restrict__ img)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < NH * int (K1))
  {
    const int o = idx / K1, k = idx % K1;
    const int t = k / NF, f = k % NF;
    const float w = t < KT ? P[P_W1 + (o * NF + f) * KT + t] : 0.f;
    *reinterpret_cast<__nv_bfloat16*> (img + (k / 8) * B_LBO + o * 16 + (k % 8) * 2) =
        __float2bfloat16_rn (w);
  }
  else if (idx < NH * int (K1 + K2))
  {
    const int j = idx - NH * K1;
    const int o = j / K2, k = j % K2;
    const int t = k / NH, i = k % NH;
    *reinterpret_cast<__nv_bfloat16*> (img + B1_BYTES + (k / 8) * B_LBO + o * 16 + (k % 8) * 2) =
        __float2bfloat16_rn (P[P_W2 + (o * NH + i) * KT + t]);
  }
}

__device__ __forceinline__ uint32_t pack_bf2 (float a, float b)
{
  __nv_bfloat162 p;
  p.x = __float2bfloat16_rn (a);
  p.y = __float2bfloat16_rn (b);
  return *reinterpret_cast<uint32_t*> (&p);
}

// issue one convolution's MMAs: 4 row tiles, N = 32, K in steps of 16
template <unsigned K>
__device__ __forceinline__ void issue_conv (uint32_t tmem, uint32_t a, uint32_t b)
{
  constexpr uint32_t ID = idesc_bf16 (128, NH);
#pragma unroll
  for (unsigned t = 0; t < 4; t++)
#pragma unroll
    for (unsigned ks = 0; ks < K / 16; ks++)
      mma_bf16 (tmem + t * NH, sdesc (a + t * 2048 + ks * 2 * A_LBO, A_LBO, 128),
                sdesc (b + ks * 2 * B_LBO, B_LBO, 128), ID, ks ? 1u : 0u);
}

__global__ void __launch_bounds__ (MAXCH, 1)
k_rfi_infer (const float* __restrict__ X, const uint4* __restrict__ img, const float* __restrict__ P,
             const uint8_t* __restrict__ sk_mask, const uint64_t npart, const unsigned nchan,
             const float lo, const float hi, float* __restrict__ prob, uint8_t* __restrict__ mask,
             unsigned long long* __restrict__ nfall, int* __restrict__ err)
{
  extern __shared__ __align__ (1024) unsigned char sm[];
  unsigned char* A = sm;
  unsigned char* act = sm + A_BYTES;
  unsigned char* Bimg = act + ACT_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*> (Bimg + IMG_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*> (bar + 1);
  const unsigned tid = threadIdx.x, w = tid >> 5;
  const int c = int (tid);
  const bool live = tid < nchan;

  for (unsigned i = tid; i < IMG_BYTES / 16; i += MAXCH)
    reinterpret_cast<uint4*> (Bimg)[i] = __ldg (img + i);
  if (tid == 0) bar_init (bar, 1);
  if (w == 0) tmem_alloc (tslot, INF_TMEM_COLS);
  fence_async_smem ();
  fence_before ();
  __syncthreads ();
  fence_after ();
  const uint32_t tmem = *tslot;
  const uint32_t a_s = saddr (A), b1_s = saddr (Bimg), b2_s = b1_s + B1_BYTES;
  const uint32_t tlane = tmem + ((32u * (w & 3)) << 16) + (w >> 2) * NH;
  float b1[NH], b2[NH], w3[NH];
#pragma unroll
  for (int o = 0; o < NH; o++)
  {
    b1[o] = P[P_B1 + o];
    b2[o] = P[P_B2 + o];
    w3[o] = P[P_W3 + o];
  }
  const float b3 = P[P_B3];
  unsigned parity = 0;
  bool failed = false;
  auto run = [&] (auto ktag, uint32_t bsm) -> bool {
    constexpr unsigned K = decltype (ktag)::value;
    fence_async_smem ();
    fence_before ();
    __syncthreads ();
    if (tid == 0)
    {
      fence_after ();
      issue_conv<K> (tmem, a_s, bsm);
      mma_commit (bar);
    }
    const bool ok = bar_wait (bar, parity);
    parity ^= 1;
    if (__syncthreads_or (!ok)) return false;
    fence_after ();
    return true;
  };

  for (uint64_t b = blockIdx.x; b < npart; b += gridDim.x)
  {
    // layer 1 im2col: chunk t = the 8 features of channel c + t - 1, chunk 3 = 0
#pragma unroll
    for (int t = 0; t < 4; t++)
    {
      const int cc = c + t - 1;
      uint4 q = make_uint4 (0, 0, 0, 0);
      if (t < KT && live && cc >= 0 && cc < int (nchan))
      {
        const float4* x = reinterpret_cast<const float4*> (X + (b * nchan + cc) * NF);
        const float4 u = __ldg (x), v = __ldg (x + 1);
        q = make_uint4 (pack_bf2 (u.x, u.y), pack_bf2 (u.z, u.w), pack_bf2 (v.x, v.y),
                        pack_bf2 (v.z, v.w));
      }
      *reinterpret_cast<uint4*> (A + t * A_LBO + tid * 16) = q;
    }
    if (!run (std::integral_constant<unsigned, K1> {}, b1_s)) { failed = true; break; }
    float v[32];
    tmem_ld32 (tlane, v);
    // bias, ReLU, BF16 activations of this channel (row-major, 64 bytes)
    {
      uint4* dst = reinterpret_cast<uint4*> (act + tid * 64);
#pragma unroll
      for (int j = 0; j < 4; j++)
      {
        float h[8];
#pragma unroll
        for (int e = 0; e < 8; e++) h[e] = fmaxf (v[8 * j + e] + b1[8 * j + e], 0.f);
        dst[j] = make_uint4 (pack_bf2 (h[0], h[1]), pack_bf2 (h[2], h[3]), pack_bf2 (h[4], h[5]),
                             pack_bf2 (h[6], h[7]));
      }
    }
    fence_before ();
    __syncthreads ();
    // layer 2 im2col: taps at c - 2, c, c + 2 (32 activations = four chunks each)
#pragma unroll
    for (int t = 0; t < KT; t++)
    {
      const int cc = c + 2 * (t - 1);
      const bool ok = live && cc >= 0 && cc < int (nchan);
      const uint4* srcp = reinterpret_cast<const uint4*> (act + (ok ? cc : 0) * 64);
#pragma unroll
      for (int j = 0; j < 4; j++)
        *reinterpret_cast<uint4*> (A + (4 * t + j) * A_LBO + tid * 16) =
            ok ? srcp[j] : make_uint4 (0, 0, 0, 0);
    }
    if (!run (std::integral_constant<unsigned, K2> {}, b2_s)) { failed = true; break; }
    tmem_ld32 (tlane, v);
    fence_before ();
    float z = b3;
#pragma unroll
    for (int o = 0; o < NH; o++) z = fmaf (w3[o], fmaxf (v[o] + b2[o], 0.f), z);
    const float p = 1.f / (1.f + expf (-z));
    if (live)
    {
      const uint64_t idx = b * nchan + c;
      if (prob) prob[idx] = p;
      uint8_t zap;
      if (p >= hi) zap = 1;
      else if (p <= lo) zap = 0;
      else
      {
        zap = sk_mask ? sk_mask[idx] : uint8_t (p >= 0.5f);
        if (nfall) atomicAdd (nfall, 1ull);
      }
      if (mask) mask[idx] = zap;
    }
  }
  if (failed && tid == 0)
  {
    atomicExch (err, 1);
    bar_wait (bar, parity ^ 1);
  }
  fence_before ();
  __syncthreads ();
  fence_after ();
  if (w == 0) tmem_free (tmem, INF_TMEM_COLS);
}

} // namespace
} // namespace b200

using namespace b200;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

struct dspsr_b200_rfi_proposer
{
  dspsr_b200_context* ctx = nullptr;
  unsigned nchan = 0, M = 0, Nd = 1;
  uint64_t max_npart = 0, have_npart = 0;
  unsigned max_batch_rows = 0;
  float *X = nullptr, *P = nullptr, *G = nullptr, *m = nullptr, *v = nullptr;
  float *A1 = nullptr, *A2 = nullptr, *dA1 = nullptr, *dA2 = nullptr, *loss = nullptr;
  uint8_t* img = nullptr;
  int* err = nullptr;
  unsigned long long* nfall = nullptr;
  int adam_t = 0;
  std::mt19937_64 rng;
  bool packed = false;

  ~dspsr_b200_rfi_proposer ()
  {
    for (void* p : {(void*) X, (void*) P, (void*) G, (void*) m, (void*) v, (void*) A1, (void*) A2,
                    (void*) dA1, (void*) dA2, (void*) loss, (void*) img, (void*) err,
                    (void*) nfall})
      if (p) cudaFree (p);
  }
};

void b200::rfi_proposer_shape (const dspsr_b200_rfi_proposer* r, dspsr_b200_context** ctx,
                               unsigned* nchan, unsigned* M)
{
  *ctx = r->ctx;
  *nchan = r->nchan;
  *M = r->M;
}

namespace {

int rfail (dspsr_b200_context* ctx, int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start (ap, fmt);
  vsnprintf (buf, sizeof (buf), fmt, ap);
  va_end (ap);
  if (ctx) ctx->error = buf;
  return code;
}

#define RFI_CHECK(ctx, call, where)                                                   \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess)                                                            \
      return rfail ((ctx), DSPSR_B200_ECUDA, "%s: %s", (where), cudaGetErrorString (_e)); \
  } while (0)

// He-style initialisation from a seeded generator, biases zero, head bias at
// the log-odds of a rare class
std::vector<float> init_params (uint64_t seed)
{
  std::mt19937_64 g (seed);
  std::normal_distribution<double> n01 (0.0, 1.0);
  std::vector<float> p (NPARAM, 0.f);
  const double s1 = std::sqrt (2.0 / (NF * KT)), s2 = std::sqrt (2.0 / (NH * KT)),
               s3 = std::sqrt (1.0 / NH);
  for (int i = 0; i < NH * NF * KT; i++) p[P_W1 + i] = float (s1 * n01 (g));
  for (int i = 0; i < NH * NH * KT; i++) p[P_W2 + i] = float (s2 * n01 (g));
  for (int i = 0; i < NH; i++) p[P_W3 + i] = float (s3 * n01 (g));
  p[P_B3] = -3.f;
  return p;
}

int pack (dspsr_b200_rfi_proposer* r)
{
  k_rfi_pack<<<(NH * (K1 + K2) + 255) / 256, 256, 0, r->ctx->stream>>> (r->P, r->img);
  RFI_CHECK (r->ctx, cudaGetLastError (), "rfi pack");
  r->packed = true;
  return DSPSR_B200_OK;
}

} // namespace

extern "C" {

int dspsr_b200_rfi_proposer_create (dspsr_b200_context* ctx, unsigned nchan, unsigned M,
                                    unsigned Nd, uint64_t max_npart, unsigned max_batch_blocks,
                                    uint64_t seed, dspsr_b200_rfi_proposer** out)
{
  if (!ctx || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  if (nchan < 1 || nchan > MAXCH || M < 2 || Nd < 1 || max_npart < 1 || max_batch_blocks < 1)
    return rfail (ctx, DSPSR_B200_EINVAL,
                  "rfi proposer: nchan=%u must be in [1, %d], M >= 2, Nd >= 1, npart >= 1", nchan,
                  MAXCH);
  auto* r = new dspsr_b200_rfi_proposer;
  r->ctx = ctx;
  r->nchan = nchan;
  r->M = M;
  r->Nd = Nd;
  r->max_npart = max_npart;
  r->max_batch_rows = max_batch_blocks * nchan;
  r->rng.seed (seed);
  const uint64_t rows = uint64_t (r->max_batch_rows);
  cudaError_t e = cudaSuccess;
  auto alloc = [&] (auto** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc (reinterpret_cast<void**> (p), bytes);
  };
  alloc (&r->X, max_npart * nchan * NF * sizeof (float));
  alloc (&r->P, NPARAM * sizeof (float));
  alloc (&r->G, NPARAM * sizeof (float));
  alloc (&r->m, NPARAM * sizeof (float));
  alloc (&r->v, NPARAM * sizeof (float));
  alloc (&r->A1, rows * NH * sizeof (float));
  alloc (&r->A2, rows * NH * sizeof (float));
  alloc (&r->dA1, rows * NH * sizeof (float));
  alloc (&r->dA2, rows * NH * sizeof (float));
  alloc (&r->loss, sizeof (float));
  alloc (&r->img, IMG_BYTES);
  alloc (&r->err, sizeof (int));
  alloc (&r->nfall, sizeof (unsigned long long));
  if (e != cudaSuccess)
  {
    delete r;
    return rfail (ctx, DSPSR_B200_ECUDA, "rfi proposer: cudaMalloc: %s", cudaGetErrorString (e));
  }
  std::vector<float> p = init_params (seed);
  std::vector<float> zero (NPARAM, 0.f);
  e = cudaMemcpy (r->P, p.data (), NPARAM * sizeof (float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy (r->G, zero.data (), NPARAM * sizeof (float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy (r->m, zero.data (), NPARAM * sizeof (float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy (r->v, zero.data (), NPARAM * sizeof (float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset (r->err, 0, sizeof (int));
  if (e == cudaSuccess) e = cudaFuncSetAttribute (k_rfi_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  int (INF_SMEM));
  if (e != cudaSuccess)
  {
    delete r;
    return rfail (ctx, DSPSR_B200_ECUDA, "rfi proposer: set-up: %s", cudaGetErrorString (e));
  }
  *out = r;
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_destroy (dspsr_b200_rfi_proposer* r)
{
  if (!r) return DSPSR_B200_EINVAL;
  cudaStreamSynchronize (r->ctx->stream);
  delete r;
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_features (dspsr_b200_rfi_proposer* r, const float* d_sums,
                                      const uint32_t* d_counts, uint64_t npart, unsigned npol)
{
  if (!r || !d_sums || npol < 1 || npol > 2) return DSPSR_B200_EINVAL;
  if (npart < 1 || npart > r->max_npart)
    return rfail (r->ctx, DSPSR_B200_EINVAL, "rfi proposer: npart=%llu outside [1, %llu]",
                  (unsigned long long) npart, (unsigned long long) r->max_npart);
  k_rfi_features<<<unsigned (npart), 256, 0, r->ctx->stream>>> (
      d_sums, d_counts, npart, r->nchan, npol, r->M, r->Nd, r->X);
  RFI_CHECK (r->ctx, cudaGetLastError (), "rfi features");
  r->have_npart = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_train (dspsr_b200_rfi_proposer* r, const uint8_t* d_labels,
                                   unsigned steps, unsigned batch_blocks, float lr,
                                   float pos_weight, float* mean_loss)
{
  if (!r || !d_labels || batch_blocks < 1 || lr <= 0.f || pos_weight <= 0.f) return DSPSR_B200_EINVAL;
  const uint64_t npart = r->have_npart;
  if (npart == 0) return rfail (r->ctx, DSPSR_B200_ESTATE, "rfi proposer: no features yet");
  const uint64_t bb = std::min<uint64_t> (batch_blocks, npart);
  const uint64_t rows = bb * r->nchan;
  if (rows > r->max_batch_rows)
    return rfail (r->ctx, DSPSR_B200_EINVAL, "rfi proposer: batch of %llu blocks > the maximum",
                  (unsigned long long) bb);
  cudaStream_t st = r->ctx->stream;
  const unsigned nb = unsigned ((rows + 255) / 256);
  RFI_CHECK (r->ctx, cudaMemsetAsync (r->loss, 0, sizeof (float), st), "rfi loss");
  for (unsigned s = 0; s < steps; s++)
  {
    const uint64_t b0 = npart > bb ? r->rng () % (npart - bb + 1) : 0;
    const float* x = r->X + b0 * r->nchan * NF;
    const uint8_t* y = d_labels + b0 * r->nchan;
    k_conv_fwd<NF, NH, 1, true><<<nb, 256, 0, st>>> (x, r->P + P_W1, r->P + P_B1, r->A1, r->nchan, rows);
    k_conv_fwd<NH, NH, 2, true><<<nb, 256, 0, st>>> (r->A1, r->P + P_W2, r->P + P_B2, r->A2, r->nchan, rows);
    k_rfi_head<<<nb, 256, 0, st>>> (r->A2, r->P, y, rows, pos_weight, 1.f / float (rows), r->dA2,
                                    r->G, r->loss);
    const dim3 gw (std::min<unsigned> (nb, 64), NH);
    k_conv_bwd_w<NH, NH, 2><<<gw, 256, 0, st>>> (r->dA2, r->A1, r->nchan, rows, r->G + P_W2, r->G + P_B2);
    k_conv_bwd_x<NH, NH, 2><<<nb, 256, 0, st>>> (r->dA2, r->P + P_W2, r->A1, r->nchan, rows, r->dA1);
    k_conv_bwd_w<NF, NH, 1><<<gw, 256, 0, st>>> (r->dA1, x, r->nchan, rows, r->G + P_W1, r->G + P_B1);
    r->adam_t++;
    const float c1 = float (1.0 / (1.0 - std::pow (0.9, r->adam_t)));
    const float c2 = float (1.0 / (1.0 - std::pow (0.999, r->adam_t)));
    k_adam<<<(NPARAM + 255) / 256, 256, 0, st>>> (r->P, r->G, r->m, r->v, NPARAM, lr, c1, c2);
  }
  RFI_CHECK (r->ctx, cudaGetLastError (), "rfi train");
  r->packed = false;
  if (mean_loss)
  {
    float h = 0.f;
    RFI_CHECK (r->ctx, cudaMemcpyAsync (&h, r->loss, sizeof (float), cudaMemcpyDeviceToHost, st),
               "rfi loss read");
    RFI_CHECK (r->ctx, cudaStreamSynchronize (st), "rfi loss sync");
    *mean_loss = steps ? h / (float (steps) * float (rows)) : 0.f;
  }
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_infer (dspsr_b200_rfi_proposer* r, const uint8_t* d_sk_mask,
                                   float confidence, uint8_t* d_mask, float* d_prob,
                                   uint64_t* n_fallback)
{
  if (!r || confidence < 0.5f || confidence > 1.f) return DSPSR_B200_EINVAL;
  const uint64_t npart = r->have_npart;
  if (npart == 0) return rfail (r->ctx, DSPSR_B200_ESTATE, "rfi proposer: no features yet");
  cudaStream_t st = r->ctx->stream;
  if (!r->packed)
  {
    const int rc = pack (r);
    if (rc) return rc;
  }
  RFI_CHECK (r->ctx, cudaMemsetAsync (r->nfall, 0, sizeof (unsigned long long), st), "rfi count");
  int nsm = 148;
  cudaDeviceGetAttribute (&nsm, cudaDevAttrMultiProcessorCount, r->ctx->device);
  const unsigned grid = unsigned (std::min<uint64_t> (npart, uint64_t (nsm)));
  k_rfi_infer<<<grid, MAXCH, INF_SMEM, st>>> (r->X, reinterpret_cast<const uint4*> (r->img), r->P,
                                              d_sk_mask, npart, r->nchan, 1.f - confidence,
                                              confidence, d_prob, d_mask, r->nfall, r->err);
  RFI_CHECK (r->ctx, cudaGetLastError (), "rfi infer");
  if (n_fallback)
  {
    unsigned long long h = 0;
    int e = 0;
    RFI_CHECK (r->ctx, cudaMemcpyAsync (&h, r->nfall, sizeof (h), cudaMemcpyDeviceToHost, st),
               "rfi count read");
    RFI_CHECK (r->ctx, cudaMemcpyAsync (&e, r->err, sizeof (e), cudaMemcpyDeviceToHost, st),
               "rfi status read");
    RFI_CHECK (r->ctx, cudaStreamSynchronize (st), "rfi infer sync");
    if (e) return rfail (r->ctx, DSPSR_B200_ESTATE, "rfi proposer: a device-side wait timed out");
    *n_fallback = h;
  }
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_get_params (dspsr_b200_rfi_proposer* r, float* params, unsigned* n)
{
  if (!r || !n) return DSPSR_B200_EINVAL;
  if (params)
  {
    RFI_CHECK (r->ctx, cudaStreamSynchronize (r->ctx->stream), "rfi sync");
    RFI_CHECK (r->ctx, cudaMemcpy (params, r->P, NPARAM * sizeof (float), cudaMemcpyDeviceToHost),
               "rfi params read");
  }
  *n = NPARAM;
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_set_params (dspsr_b200_rfi_proposer* r, const float* params,
                                        unsigned n)
{
  if (!r || !params || n != NPARAM) return DSPSR_B200_EINVAL;
  RFI_CHECK (r->ctx, cudaStreamSynchronize (r->ctx->stream), "rfi sync");
  RFI_CHECK (r->ctx, cudaMemcpy (r->P, params, NPARAM * sizeof (float), cudaMemcpyHostToDevice),
             "rfi params write");
  r->packed = false;
  return DSPSR_B200_OK;
}

int dspsr_b200_rfi_proposer_get_features (dspsr_b200_rfi_proposer* r, float* features)
{
  if (!r || !features) return DSPSR_B200_EINVAL;
  RFI_CHECK (r->ctx, cudaStreamSynchronize (r->ctx->stream), "rfi sync");
  RFI_CHECK (r->ctx, cudaMemcpy (features, r->X, r->have_npart * r->nchan * NF * sizeof (float),
                                 cudaMemcpyDeviceToHost),
             "rfi features read");
  return DSPSR_B200_OK;
}

} // extern "C"
