// tc_fft.cu -- the convolution row (8192-point forward FFT, x H, inverse FFT)
// with every DFT stage on the tensor cores.
//
// It replaces the cuFFT C2C plans of the reference's convolution engine
// (Signal/General/ConvolutionCUDA.cu:370-413, the batched forward and
// backward plans around the response multiply) for the row half of the
// four-step split, as a drop-in for k_rows32<8192, true>: the same row of
// the scratch in (natural order), the same row out, the response row of
// (channel, k1) in between.
//
// Decomposition, 8192 = 16 x 16 x 32 (indices: n = n_a + 512 n_b,
// n_a = n_d + 32 n_c; spectrum k = k_b + 16 k_c + 256 k_d):
//   F1  for each n_a:        DFT16 over n_b        x w8192^(n_a k_b)
//   F2  for each (k_b, n_d): DFT16 over n_c        x w512^(n_d k_c)
//   F3  for each (k_b, k_c): DFT32 over n_d        -> X[k]  (digit-permuted)
//   x H[k], conjugate
//   I1  for each (k_b, k_c): DFT32 over k_d        x w512^(n_d k_c)
//   I2  for each (k_b, n_d): DFT16 over k_c        x w8192^(n_a k_b)
//   I3  for each n_a:        DFT16 over k_b        -> conjugate = y[n] (natural)
// The inverse runs on conjugated data, where it uses the forward DFT matrices
// and forward twiddles, so the spectrum never needs reordering.
//
// Each stage is one GEMM D[rows x 2R] = A[rows x 2R] . B[2R x 2R]: a data row
// is one radix-R group as 2R reals (re, im interleaved), B is the R-point
// DFT as a real 2R x 2R block.  Operands are BF16 split into NS terms
// (x = x0 + x1 [+ x2], each term the BF16 rounding of what the previous ones
// left), and the MMAs form the products whose order is below the last term
// kept: NS = 2 -> x0 w0 + x0 w1 + x1 w0 (about 16 significant bits), NS = 3 ->
// also x0 w2 + x2 w0 + x1 w1 (about 24 bits, i.e. FP32 accuracy).  The DFT
// terms are stacked along N, so each data term is one MMA against all the
// DFT terms it pairs with (read once per stage, not once per product).  The
// sums accumulate in FP32 in tensor memory (tcgen05.mma kind::f16, M = 128,
// N = 32 ... 192, one elected thread issues; tcgen05.commit arrives on an
// mbarrier the block waits on, bounded).  Each thread then reads its row of
// the accumulator (tcgen05.ld 32x32b), applies the twiddles in FP32, splits
// again and writes the next stage's operand rows in shared memory.  Twiddles
// (two FP64-rounded tables in shared memory, w^e = T_hi[e/64] T_lo[e%64]) and
// the response are FP32; the DFT blocks are split from FP64 values.
//
// Operand layout in shared memory: K-major without swizzle; element (r, k) of
// a rows x K BF16 matrix at (k/8)*LBO + r*16 + (k%8)*2 (8-row core matrices
// of 128 bytes, contiguous: SBO = 128).  LBO is padded (16 or 32 bytes past a
// multiple of 128) so that the stores of each stage spread over the banks.

#include "kernels.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace b200 {

using namespace tc;

namespace {

constexpr int TC_THREADS = 512;
constexpr unsigned TC_N = 8192;

constexpr unsigned LBO16 = 512 * 16 + 32;    // R = 16 stages: 512 rows, K = 32
constexpr unsigned LBO32 = 256 * 16 + 16;    // R = 32 stages: 256 rows, K = 64
constexpr unsigned A_SPLIT_BYTES = 4 * LBO16;          // = 8 * LBO32 = 32896
static_assert (4 * LBO16 == 8 * LBO32, "both stage layouts fill one operand buffer");
static_assert (A_SPLIT_BYTES % 128 == 0, "operand buffers stay 128-byte aligned");
// The B operand of an R-point stage stacks the NS terms of the DFT block
// along N: rows [s 2R, (s + 1) 2R) hold term s (N = NS 2R rows, K = 2R).  A
// product of data term s with terms 0 .. NS-1-s is then one MMA of N = (NS -
// s) 2R that reads its A operand once; it accumulates into column groups s ..
// NS-1 of the tile's NS 2R accumulator columns, and group g ends up holding
// the sum of all products x_s w_j with s + j = g.  The epilogue adds the
// groups.
constexpr unsigned B16_BYTES = 4 * 32 * 16, B32_BYTES = 8 * 64 * 16;   // per term
template <int NS> __host__ __device__ constexpr unsigned b_lbo (int R) { return NS * 2 * R * 16; }
template <int NS> __host__ __device__ constexpr unsigned tmem_cols () { return NS == 2 ? 256 : 512; }

// twiddles w8192^e = T_hi[e >> 6] T_lo[e & 63] from two small tables
constexpr unsigned TW_HI = 128, TW_LO = 64;
constexpr unsigned TW_BYTES = (TW_HI + TW_LO) * 8;

// two operand buffers (a stage reads one while its epilogue writes the
// other), the DFT terms, four mbarriers (one per row tile) and the tensor-
// memory address
template <int NS>
constexpr unsigned tc_smem_bytes ()
{
  return NS * (2 * A_SPLIT_BYTES + B16_BYTES + B32_BYTES) + 64 + TW_BYTES;
}

__device__ __forceinline__ float2 cmulf (float2 a, float2 b)
{
  return make_float2 (a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// the NS-term BF16 split of one complex value, as (re, im) pairs
template <int NS>
__device__ __forceinline__ void split_c (float2 z, uint32_t* out)
{
  float r = z.x, i = z.y;
#pragma unroll
  for (int s = 0; s < NS; s++)
  {
    const __nv_bfloat16 hr = __float2bfloat16_rn (r), hi = __float2bfloat16_rn (i);
    __nv_bfloat162 p;
    p.x = hr;
    p.y = hi;
    out[s] = *reinterpret_cast<uint32_t*> (&p);
    r -= __bfloat162float (hr);
    i -= __bfloat162float (hi);
  }
}

// complex element kc of row r of an operand split (LBO layout above)
__device__ __forceinline__ unsigned aoff (unsigned r, unsigned kc, unsigned lbo)
{
  return (kc >> 2) * lbo + r * 16 + (kc & 3) * 4;
}

template <int NS>
__device__ __forceinline__ void put_c (unsigned char* A, unsigned off, float2 z)
{
  uint32_t s[NS];
  split_c<NS> (z, s);
#pragma unroll
  for (int i = 0; i < NS; i++)
    *reinterpret_cast<uint32_t*> (A + i * A_SPLIT_BYTES + off) = s[i];
}

// four consecutive complex elements 4j..4j+3 of row r: one 16-byte store per split
template <int NS>
__device__ __forceinline__ void put_c4 (unsigned char* A, unsigned r, unsigned j, unsigned lbo,
                                        const float2* z)
{
  uint32_t s[4][NS];
#pragma unroll
  for (int q = 0; q < 4; q++) split_c<NS> (z[q], s[q]);
#pragma unroll
  for (int i = 0; i < NS; i++)
    *reinterpret_cast<uint4*> (A + i * A_SPLIT_BYTES + j * lbo + r * 16) =
        make_uint4 (s[0][i], s[1][i], s[2][i], s[3][i]);
}

// One stage's MMAs, issued by one thread: R = 16 -> 4 row tiles, R = 32 -> 2
// row tiles; K = 2R in steps of 16; per tile and step one MMA per data term
// (N = (NS - s) 2R, see b_lbo).  Each tile's MMAs are committed to that
// tile's mbarrier, so its epilogue can start while later tiles compute.
template <int NS, int R>
__device__ __forceinline__ void issue_stage (uint32_t tmem, uint32_t a_base, uint32_t b_base,
                                             uint64_t* bars)
{
  constexpr unsigned NT = R == 16 ? 4 : 2;
  constexpr unsigned G = 2 * R;                 // one column group
  constexpr unsigned KS = 2 * R / 16;
  constexpr unsigned LBO = R == 16 ? LBO16 : LBO32;
  constexpr unsigned BLBO = b_lbo<NS> (R);
#pragma unroll
  for (unsigned t = 0; t < NT; t++)
  {
#pragma unroll
    for (unsigned ks = 0; ks < KS; ks++)
#pragma unroll
      for (int sp = 0; sp < NS; sp++)
      {
        const uint32_t a = a_base + sp * A_SPLIT_BYTES + t * 2048 + ks * 2 * LBO;
        const uint32_t b = b_base + ks * 2 * BLBO;
        mma_bf16 (tmem + t * NS * G + sp * G, sdesc (a, LBO, 128), sdesc (b, BLBO, 128),
                  idesc_bf16 (128, (NS - sp) * G), (ks | sp) ? 1u : 0u);
      }
    mma_commit (bars + t);
  }
}

// this thread's 32 accumulator columns of the stage: the NS column groups
// (stride apart) added
template <int NS>
__device__ __forceinline__ void tmem_sum (uint32_t taddr, uint32_t stride, float* v)
{
  tmem_ld32 (taddr, v);
#pragma unroll
  for (int g = 1; g < NS; g++)
  {
    float u[32];
    tmem_ld32 (taddr + g * stride, u);
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] += u[i];
  }
}

} // namespace

// rows of the scratch (natural order) -> forward FFT, x H, inverse FFT -> in place
template <int NS>
__global__ void __launch_bounds__ (TC_THREADS, 1)
k_rows_mma (float2* __restrict__ scratch, const float2* __restrict__ tw,
            const uint4* __restrict__ dft, const float2* __restrict__ H, const unsigned n1,
            const unsigned nchan, const unsigned npol, const unsigned nrows,
            int* __restrict__ err)
{
  extern __shared__ __align__ (1024) unsigned char sm[];
  unsigned char* Abuf[2] = {sm, sm + NS * A_SPLIT_BYTES};   // NS operand terms each
  unsigned char* B16 = sm + 2 * NS * A_SPLIT_BYTES;         // NS terms of the DFT16 block
  unsigned char* B32 = B16 + NS * B16_BYTES;                // NS terms of the DFT32 block
  uint64_t* bars = reinterpret_cast<uint64_t*> (B32 + NS * B32_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*> (bars + 4);
  float2* tw_hi = reinterpret_cast<float2*> (reinterpret_cast<unsigned char*> (bars) + 64);
  float2* tw_lo = tw_hi + TW_HI;
  const unsigned tid = threadIdx.x, w = tid >> 5, l = tid & 31;

  // the DFT blocks (already in the operand layout) and the twiddle tables
  // into shared memory
  {
    constexpr unsigned NV = NS * (B16_BYTES + B32_BYTES) / 16;
    uint4* dst = reinterpret_cast<uint4*> (B16);
    for (unsigned i = tid; i < NV; i += TC_THREADS) dst[i] = __ldg (dft + i);
    if (tid < TW_HI) tw_hi[tid] = __ldg (tw + 64 * tid);
    else if (tid < TW_HI + TW_LO) tw_lo[tid - TW_HI] = __ldg (tw + (tid - TW_HI));
  }
  // y w8192^e
  auto twiddle = [&] (float2 y, unsigned e) {
    e &= 8191;
    return cmulf (cmulf (y, tw_hi[e >> 6]), tw_lo[e & 63]);
  };
  if (tid < 4) bar_init (bars + tid, 1);
  if (w == 0) tmem_alloc (tslot, tmem_cols<NS> ());
  fence_async_smem ();
  fence_before ();
  __syncthreads ();
  fence_after ();
  const uint32_t tmem = *tslot;
  const uint32_t b16 = saddr (B16), b32 = saddr (B32);
  // this thread's accumulator lanes: warp w reads lanes 32 (w % 4) ... + 31
  const uint32_t tlane = tmem + ((32u * (w & 3)) << 16);
  unsigned phase = 0;          // bit t: the parity the next wait on bars[t] expects
  bool lost = false;           // this thread's wait gave up
  bool failed = false;         // some thread's did (block-uniform)
  int last_bar = -1;           // thread 0: the barrier of the last commit, and its parity
  unsigned last_parity = 0;

  // one stage on operand buffer `cur`: all operands are in place (barrier,
  // with the block-uniform check of the last waits), thread 0 issues tile by
  // tile, each thread waits (bounded) for its own tile only
  auto run_stage = [&] (auto rtag, int cur) -> bool {
    constexpr int R = decltype (rtag)::value;
    constexpr unsigned NT = R == 16 ? 4 : 2;
    fence_async_smem ();
    fence_before ();
    if (__syncthreads_or (lost)) return false;
    if (tid == 0)
    {
      fence_after ();
      issue_stage<NS, R> (tmem, saddr (Abuf[cur]), R == 16 ? b16 : b32, bars);
      last_bar = int (NT - 1);
      last_parity = (phase >> (NT - 1)) & 1;
    }
    const unsigned t = R == 16 ? (w >> 2) : ((w >> 2) & 1);
    lost = !bar_wait (bars + t, (phase >> t) & 1);
    phase ^= (1u << NT) - 1;
    fence_after ();
    return true;
  };
  using R16 = std::integral_constant<int, 16>;
  using R32 = std::integral_constant<int, 32>;

  for (unsigned row = blockIdx.x; row < nrows; row += gridDim.x)
  {
    float2* g = scratch + uint64_t (row) * TC_N;
    const unsigned k1 = row % n1;
    const unsigned c = (row / n1 / npol) % nchan;
    const float2* h = H + (uint64_t (c) * n1 + k1) * TC_N;
    float v[32];

    // F1 operand (buffer 0): row n_a = tid holds x[n_a + 512 n_b], n_b = 0..15
    {
      float2 z[16];
#pragma unroll
      for (int nb = 0; nb < 16; nb++) z[nb] = g[tid + 512 * nb];
#pragma unroll
      for (int j = 0; j < 4; j++) put_c4<NS> (Abuf[0], tid, j, LBO16, z + 4 * j);
    }
    if (!run_stage (R16 {}, 0)) { failed = true; break; }
    // F1 epilogue: Y1[n_a][k_b] x w8192^(n_a k_b) -> F2 rows 32 k_b + n_d, K = n_c
    tmem_sum<NS> (tlane + (w >> 2) * NS * 32, 32, v);
    {
      const unsigned na = tid, nd = l, nc = w;
#pragma unroll
      for (int kb = 0; kb < 16; kb++)
      {
        const float2 y = twiddle (make_float2 (v[2 * kb], v[2 * kb + 1]), na * kb);
        put_c<NS> (Abuf[1], aoff (32 * kb + nd, nc, LBO16), y);
      }
    }
    if (!run_stage (R16 {}, 1)) { failed = true; break; }
    // F2 epilogue: row (k_b = w, n_d = l), Y2[k_c] x w512^(n_d k_c) -> F3 rows k_b + 16 k_c, K = n_d
    tmem_sum<NS> (tlane + (w >> 2) * NS * 32, 32, v);
    {
      const unsigned kb = w, nd = l;
#pragma unroll
      for (int kc = 0; kc < 16; kc++)
      {
        const float2 y = twiddle (make_float2 (v[2 * kc], v[2 * kc + 1]), 16 * nd * kc);
        put_c<NS> (Abuf[0], aoff (kb + 16 * kc, nd, LBO32), y);
      }
    }
    if (!run_stage (R32 {}, 0)) { failed = true; break; }
    // F3 epilogue: row r3 = k_b + 16 k_c (tile m, quarter q), half hh of k_d:
    // X[r3 + 256 k_d] x H, conjugated -> I1 operand, own row, K = k_d
    const unsigned m = (w >> 2) & 1, hh = w >> 3;
    const unsigned r3 = 128 * m + 32 * (w & 3) + l;
    tmem_sum<NS> (tlane + m * NS * 64 + hh * 32, 64, v);
    {
      float2 z[16];
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        const unsigned kd = 16 * hh + j;
        const float2 x = make_float2 (v[2 * j], v[2 * j + 1]);
        const float2 f = __ldg (h + r3 + 256 * kd);
        // Response::operate (Response.C:662-726), then the conjugate
        z[j] = make_float2 (x.x * f.x - x.y * f.y, -(x.x * f.y + x.y * f.x));
      }
#pragma unroll
      for (int j = 0; j < 4; j++) put_c4<NS> (Abuf[1], r3, 4 * hh + j, LBO32, z + 4 * j);
    }
    if (!run_stage (R32 {}, 1)) { failed = true; break; }
    // I1 epilogue: row r3, U1[n_d] (n_d in this half) x w512^(n_d k_c)
    // -> I2 rows k_b + 16 n_d, K = k_c
    tmem_sum<NS> (tlane + m * NS * 64 + hh * 32, 64, v);
    {
      const unsigned kb = r3 & 15, kc = r3 >> 4;
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        const unsigned nd = 16 * hh + j;
        const float2 y = twiddle (make_float2 (v[2 * j], v[2 * j + 1]), 16 * nd * kc);
        put_c<NS> (Abuf[0], aoff (kb + 16 * nd, kc, LBO16), y);
      }
    }
    if (!run_stage (R16 {}, 0)) { failed = true; break; }
    // I2 epilogue: row r5 = tid = k_b + 16 n_d, U2[n_c] x w8192^(n_a k_b),
    // n_a = n_d + 32 n_c -> I3 rows n_a, K = k_b
    tmem_sum<NS> (tlane + (w >> 2) * NS * 32, 32, v);
    {
      const unsigned kb = tid & 15, nd = tid >> 4;
#pragma unroll
      for (int nc = 0; nc < 16; nc++)
      {
        const unsigned na = nd + 32 * nc;
        const float2 y = twiddle (make_float2 (v[2 * nc], v[2 * nc + 1]), na * kb);
        put_c<NS> (Abuf[1], aoff (na, kb, LBO16), y);
      }
    }
    if (!run_stage (R16 {}, 1)) { failed = true; break; }
    // I3 epilogue: row n_a = tid, y[n_a + 512 n_b] = conjugate.  The next
    // row's F1 operand goes to buffer 0, which no MMA reads any more: every
    // thread passed its I2 wait before the I3 stage began.
    tmem_sum<NS> (tlane + (w >> 2) * NS * 32, 32, v);
#pragma unroll
    for (int nb = 0; nb < 16; nb++) g[tid + 512 * nb] = make_float2 (v[2 * nb], -v[2 * nb + 1]);
  }
  fence_before ();
  if (__syncthreads_or (lost)) failed = true;
  if (failed && tid == 0)
  {
    atomicExch (err, 1);
    // the last commit covers every MMA issued before it: let them finish
    if (last_bar >= 0) bar_wait (bars + last_bar, last_parity);
  }
  __syncthreads ();
  fence_after ();
  if (w == 0) tmem_free (tmem, tmem_cols<NS> ());
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

namespace {

uint16_t bf16_bits (double x)
{
  // round to nearest even from the float value (x is within float range)
  const float f = float (x);
  uint32_t u;
  std::memcpy (&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
  return uint16_t (u);
}

double bf16_value (uint16_t b)
{
  const uint32_t u = uint32_t (b) << 16;
  float f;
  std::memcpy (&f, &u, 4);
  return f;
}

// Real block B[K][N] of the R-point DFT (W[n][k] = exp(-2 pi i n k / R)),
// stored K-major (row N, column K) in the operand layout, split into ns terms.
void put_dft_block (unsigned R, unsigned ns, uint8_t* out)
{
  const unsigned lbo = ns * 2 * R * 16;
  const unsigned K = 2 * R;
  for (unsigned kn = 0; kn < K; kn++)      // B row index (input real index)
    for (unsigned nn = 0; nn < K; nn++)    // B column index (output real index)
    {
      const unsigned n = kn / 2, k = nn / 2;
      const double a = -2.0 * M_PI * double ((uint64_t (n) * k) % R) / double (R);
      const double wr = std::cos (a), wi = std::sin (a);
      double val;
      if (kn % 2 == 0) val = nn % 2 == 0 ? wr : wi;
      else val = nn % 2 == 0 ? -wi : wr;
      double rem = val;
      for (unsigned s = 0; s < ns; s++)
      {
        const uint16_t b = bf16_bits (rem);
        rem -= bf16_value (b);
        // element (row s 2R + nn, column kn) of the K-major (ns 2R) x K matrix
        const unsigned off = (kn / 8) * lbo + (s * 2 * R + nn) * 16 + (kn % 8) * 2;
        std::memcpy (out + off, &b, 2);
      }
    }
}

} // namespace

void make_tc_dft_image (unsigned ns, std::vector<uint8_t>& img)
{
  img.assign (ns * (B16_BYTES + B32_BYTES), 0);
  put_dft_block (16, ns, img.data ());
  put_dft_block (32, ns, img.data () + ns * B16_BYTES);
}

template <int NS>
static cudaError_t launch_rows_mma_t (unsigned nrows, float2* scratch, const ConvTables& tb,
                                      unsigned n1, const ConvShape& sh, cudaStream_t st)
{
  constexpr unsigned smem = tc_smem_bytes<NS> ();
  static_assert (smem <= 227u * 1024u, "tensor-core row kernel shared memory");
  cudaError_t e = cudaFuncSetAttribute (k_rows_mma<NS>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
  if (e != cudaSuccess) return e;
  const unsigned grid = std::min<unsigned> (nrows, unsigned (tb.nsm));
  k_rows_mma<NS><<<grid, TC_THREADS, smem, st>>> (scratch, tb.tw2,
                                                  static_cast<const uint4*> (tb.tc_dft), tb.H, n1,
                                                  sh.nchan, sh.npol, nrows, tb.err);
  return cudaGetLastError ();
}

cudaError_t launch_rows_mma (unsigned nrows, float2* scratch, const ConvTables& tb, unsigned n1,
                             const ConvShape& sh, cudaStream_t st)
{
  if (sh.n2 != TC_N || !tb.tc_dft) return cudaErrorInvalidValue;
  if (tb.tc_splits == 2) return launch_rows_mma_t<2> (nrows, scratch, tb, n1, sh, st);
  if (tb.tc_splits == 3) return launch_rows_mma_t<3> (nrows, scratch, tb, n1, sh, st);
  return cudaErrorInvalidValue;
}

} // namespace b200
