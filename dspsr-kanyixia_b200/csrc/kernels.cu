// kernels.cu -- sm_100a kernels of the B200 baseband hot path.
//
// Overlap-save coherent dedispersion (Signal/General/Convolution.C:724-803 is
// the CPU algorithm; CUDA::ConvolutionEngine runs it as cuFFT + 3 kernels per
// batch) is restructured here as a four-step FFT of length N = n1 * n2:
//
//   K1 (columns)  unpack the int8/int16/float input on load, n1-point DFTs in
//                 registers across the n1 chunks of n2 samples, store rows k1.
//   K2 (rows)     twiddle w_N^{k1 n2}, n2-point Stockham FFT in shared memory,
//                 multiply by the response (stored in four-step order), inverse
//                 n2-point FFT, conjugate twiddle -- one read and one write.
//   K3 (columns)  inverse n1-point DFTs in registers, overlap discard, and then
//                 either write the voltages (Engine::perform) or detect and
//                 fold in the same pass (warp-segmented reduction by bin).
//
// For n1 == 1 a single kernel does load, FFT, multiply, inverse FFT and the
// epilogue entirely in shared memory: one HBM round trip per part.
//
// FFT sign conventions are FFTW's (forward -1, backward +1, unnormalised); the
// 1/sqrt(N) normaliser is folded into the response, as Convolution::prepare
// does (Convolution.C:401-414).

#include "kernels.cuh"
#include "fft_core.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

namespace b200 {

namespace {

constexpr unsigned FULL = 0xffffffffu;

std::atomic<uint64_t> g_launches {0};

struct ClockScope
{
  const KernelClock* c;
  int kind;
  cudaStream_t st;
  ClockScope (const KernelClock* c_, int k, cudaStream_t s) : c (c_), kind (k), st (s)
  {
    g_launches++;
    if (c) c->mark (c->self, kind, 0, st);
  }
  ~ClockScope ()
  {
    if (c) c->mark (c->self, kind, 1, st);
  }
};

// --------------------------------------------------------------------------
// input fetch (unpack fused into the load)
// --------------------------------------------------------------------------

template <int KIND>
__device__ __forceinline__ float2 fetch (const InputView& in, const float* s_lut,
                                         unsigned c, unsigned p, uint64_t t)
{
  const void* base = in.main;
  uint64_t span = in.main_span;
  if (t < in.npre)
    base = in.pre, span = in.pre_span;
  else
    t -= in.npre;
  if constexpr (KIND == IN_INT8)
  {
    const uint8_t* b = static_cast<const uint8_t*> (base)
                       + ((t * in.nchan + c) * in.npol + p) * 2;
    const unsigned short w = __ldg (reinterpret_cast<const unsigned short*> (b));
    return make_float2 (s_lut[w & 0xff], s_lut[w >> 8]);
  }
  else if constexpr (KIND == IN_INT16)
  {
    const int16_t* q = static_cast<const int16_t*> (base)
                       + ((t * in.nchan + c) * in.npol + p) * 2;
    const unsigned w = __ldg (reinterpret_cast<const unsigned*> (q));
    short re = short (w & 0xffff), im = short (w >> 16);
    if (in.offset_binary)
    {
      re = short (re ^ 0x8000);
      im = short (im ^ 0x8000);
    }
    // SixteenBitUnpacker.C:69: float(x) + 0.5 (the double 0.5 rounds to float)
    return make_float2 (__fadd_rn (float (re), 0.5f), __fadd_rn (float (im), 0.5f));
  }
  else
  {
    const float2* f = static_cast<const float2*> (base);
    return __ldg (f + (uint64_t (c) * in.npol + p) * span + t);
  }
}

__device__ __forceinline__ void load_lut (const InputView& in, const float* lut, float* s_lut)
{
  if (in.kind == IN_INT8)
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
      s_lut[i] = lut[i];
}

// --------------------------------------------------------------------------
// detection (Detection.C:253-301 Intensity/PPQQ order, cross_detect.ic:38-41,
// stokes_detect.ic:40-43); explicit _rn arithmetic so that no product is
// fused into an FMA and every value rounds as the reference's CPU code does.
// --------------------------------------------------------------------------

__device__ __forceinline__ void detect_values (int state, unsigned npol, float2 p, float2 q,
                                               float* o)
{
  if (state == 0)
  {
    float v = __fmul_rn (p.x, p.x);
    v = __fadd_rn (v, __fmul_rn (p.y, p.y));
    if (npol == 2)
    {
      v = __fadd_rn (v, __fmul_rn (q.x, q.x));
      v = __fadd_rn (v, __fmul_rn (q.y, q.y));
    }
    o[0] = v;
    return;
  }
  const float pp = __fadd_rn (__fmul_rn (p.x, p.x), __fmul_rn (p.y, p.y));
  const float qq = __fadd_rn (__fmul_rn (q.x, q.x), __fmul_rn (q.y, q.y));
  if (state == 1)
  {
    o[0] = pp;
    o[1] = qq;
    return;
  }
  const float re = __fadd_rn (__fmul_rn (p.x, q.x), __fmul_rn (p.y, q.y));
  const float im = __fsub_rn (__fmul_rn (p.x, q.y), __fmul_rn (p.y, q.x));
  if (state == 2)
  {
    o[0] = pp;
    o[1] = qq;
    o[2] = re;
    o[3] = im;
    return;
  }
  o[0] = __fadd_rn (pp, qq);
  o[1] = __fsub_rn (pp, qq);
  o[2] = __fmul_rn (2.0f, re);
  o[3] = __fmul_rn (2.0f, im);
}

// --------------------------------------------------------------------------
// fold
// --------------------------------------------------------------------------

// Index of the plan segment holding sample t (segments are sorted by start).
__device__ __forceinline__ int seg_search (const FoldSegment* __restrict__ segs, int nseg,
                                           uint64_t t)
{
  int lo = 0, hi = nseg - 1;
  while (lo < hi)
  {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg (&segs[mid].start) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Exact bin of plan sample t in segment s (see host_rules.cpp for the algebra):
// y = (m0 + j*dm) * g in integer arithmetic, then one rounded multiply by nbin.
__device__ __forceinline__ unsigned seg_bin (const FoldSegment* __restrict__ segs, int s,
                                             uint64_t t, unsigned nbin)
{
  const uint64_t start = __ldg (&segs[s].start);
  const int64_t m0 = __ldg (&segs[s].m0);
  const int64_t dm = __ldg (&segs[s].dm);
  const double g = __ldg (&segs[s].g);
  const double y = __dmul_rn (double (m0 + int64_t (t - start) * dm), g);
  return __double2uint_rz (__dmul_rn (y, double (nbin)));
}

__device__ __forceinline__ unsigned fold_bin (const FoldSegment* __restrict__ segs, int nseg,
                                              uint64_t t, unsigned nbin)
{
  return seg_bin (segs, seg_search (segs, nseg, t), t, nbin);
}

// Profile columns of a warp whose active lanes hold increasing sample
// indices: one binary search by the first active lane, then each lane steps
// forward over the (few) segment boundaries between it and that lane.  The
// column is the segment's base plus the bin; NO_COLUMN for skipped samples
// and bins outside [0, nbin).  All 32 lanes call this.
constexpr unsigned NO_COLUMN = 0xffffffffu;
__device__ __forceinline__ unsigned warp_fold_bin (const FoldSegment* __restrict__ segs,
                                                   int nseg, bool ok, uint64_t t, unsigned nbin)
{
  const unsigned act = __ballot_sync (FULL, ok);
  if (!act) return NO_COLUMN;
  const int leader = __ffs (act) - 1;
  int s = 0;
  if ((threadIdx.x & 31) == leader) s = seg_search (segs, nseg, t);
  s = __shfl_sync (FULL, s, leader);
  if (!ok) return NO_COLUMN;
  while (s + 1 < nseg && __ldg (&segs[s + 1].start) <= t) s++;
  const unsigned base = __ldg (&segs[s].base);
  const unsigned bin = seg_bin (segs, s, t, nbin);
  return (base == FOLD_SKIP || bin >= nbin) ? NO_COLUMN : base + bin;
}

// All 32 lanes call this together.  Lanes holding consecutive time samples
// with equal bins form runs; each run is summed by a segmented shuffle
// reduction and added to the profile by its first lane with one atomic.
template <int NOUT, bool HITS>
__device__ __forceinline__ void warp_fold_t (bool ok, unsigned bin, const float* v,
                                             float* prof, unsigned nbin, unsigned* hits)
{
  const int lane = threadIdx.x & 31;
  const unsigned key = ok ? bin : 0xffffffffu;
  const unsigned prev = __shfl_up_sync (FULL, key, 1);
  const bool head = (lane == 0) || (prev != key);
  const unsigned hm = __ballot_sync (FULL, head);
  const int rid = __popc (hm & (FULL >> (31 - lane)));
  float acc[NOUT];
#pragma unroll
  for (int k = 0; k < NOUT; k++) acc[k] = ok ? v[k] : 0.0f;
  int cnt = ok ? 1 : 0;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
  {
    const int orid = __shfl_down_sync (FULL, rid, off);
    const bool take = (lane + off < 32) && (orid == rid);
#pragma unroll
    for (int k = 0; k < NOUT; k++)
    {
      const float o = __shfl_down_sync (FULL, acc[k], off);
      if (take) acc[k] += o;
    }
    if constexpr (HITS)
    {
      const int oc = __shfl_down_sync (FULL, cnt, off);
      if (take) cnt += oc;
    }
  }
  if (head && ok)
  {
#pragma unroll
    for (int k = 0; k < NOUT; k++)
      atomicAdd (prof + uint64_t (k) * nbin + bin, acc[k]);
    if constexpr (HITS) atomicAdd (hits + bin, unsigned (cnt));
  }
}

// Only the warps that count hits (one channel's) reduce the counts; hits is
// the same pointer in every lane, so the choice is warp-uniform.
template <int NOUT>
__device__ __forceinline__ void warp_fold (bool ok, unsigned bin, const float* v,
                                           float* prof, unsigned nbin, unsigned* hits)
{
  if (hits)
    warp_fold_t<NOUT, true> (ok, bin, v, prof, nbin, hits);
  else
    warp_fold_t<NOUT, false> (ok, bin, v, prof, nbin, hits);
}

template <int NOUT>
__device__ __forceinline__ void emit_fold (const FoldView& fv, unsigned c, unsigned npol, bool ok,
                                           uint64_t t, float2 p, float2 q)
{
  // a warp whose samples all fall in the overlap discard has nothing to add
  // (all 32 lanes are here, so the vote and the return are warp-uniform)
  if (!__any_sync (FULL, ok)) return;
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  unsigned bin = fv.cols ? (ok ? __ldg (fv.cols + t) : NO_COLUMN)
                         : warp_fold_bin (fv.segs, fv.nseg, ok, t, fv.nbin);
  if (ok)
  {
    detect_values (fv.state, npol, p, q, v);
    ok = bin < fv.stride;
  }
  warp_fold<NOUT> (ok, bin, v, fv.profiles + uint64_t (c) * NOUT * fv.stride, fv.stride,
                   c == 0 ? fv.hits : nullptr);
}

// --------------------------------------------------------------------------
// shared-memory Stockham FFT
// --------------------------------------------------------------------------

template <int N, int T, int D, int P>
__device__ __forceinline__ void smem_pass (float2* s, float2* v, const float2* tw)
{
  if constexpr (P < stockham_npass (N))
  {
    constexpr int R = stockham_radix (N, P);
    constexpr int Ns = stockham_ns (N, P);
    StockhamPass<N, R, T, D>::load (threadIdx.x, s, v);
    __syncthreads ();
    StockhamPass<N, R, T, D>::compute_store (threadIdx.x, Ns, v, s, tw);
    __syncthreads ();
    smem_pass<N, T, D, P + 1> (s, v, tw);
  }
}

// N-point FFT of s[spad(0..N-1)] in place; the caller has synchronised after
// writing s.  Returns synchronised.
template <int N, int T, int D>
__device__ __forceinline__ void smem_fft (float2* s, const float2* tw)
{
  float2 v[N / T];
  smem_pass<N, T, D, 0> (s, v, tw);
}

// --------------------------------------------------------------------------
// K1: forward column DFTs with the unpack fused into the load
// --------------------------------------------------------------------------

// columns per 128-thread block: one thread per column, two at n1 = 32
template <int N1>
constexpr unsigned fwd_cols_per_block ()
{
  return N1 == 32 ? 64u : 128u;
}

template <int N1, int KIND>
__global__ void __launch_bounds__ (128, 2)
k_fwd_cols (const InputView in, const float* __restrict__ lut, const uint64_t nkeep,
            const uint64_t part0, const unsigned n2, const float2* __restrict__ tw4,
            float2* __restrict__ scratch, const float* __restrict__ apod)
{
  __shared__ float s_lut[256];
  load_lut (in, lut, s_lut);
  __syncthreads ();
  const unsigned b = blockIdx.y;
  const unsigned c = blockIdx.z;
  const uint64_t N = uint64_t (N1) * n2;
  if constexpr (N1 == 32)
  {
    // Two threads per column (a 32-point DFT in one thread's registers
    // spills): thread h of the pair takes rows 2m + h, a 16-point DFT of
    // them gives E (h = 0) or O (h = 1), thread 1 applies w32^j, and one
    // exchange gives X[j] = E[j] + w32^j O[j] to thread 0 and
    // X[j + 16] = E[j] - w32^j O[j] to thread 1.
    const unsigned h = threadIdx.x & 1;
    const unsigned i2 = blockIdx.x * 64 + (threadIdx.x >> 1);
    const uint64_t t0 = (part0 + b) * nkeep + i2;
    for (unsigned p = 0; p < in.npol; p++)
    {
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; m++)
        v[m] = fetch<KIND> (in, s_lut, c, p, t0 + uint64_t (2 * m + h) * n2);
      if (apod)
      {
        // Apodization::operate on the part before the forward FFT (Convolution.C:739-743)
#pragma unroll
        for (int m = 0; m < 16; m++)
        {
          const float w = __ldg (apod + uint64_t (2 * m + h) * n2 + i2);
          v[m] = make_float2 (__fmul_rn (v[m].x, w), __fmul_rn (v[m].y, w));
        }
      }
      RegDFT<16, -1>::run (v);
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        const float2 mine = h ? tw_mul<32, -1> (j, v[j]) : v[j];
        const float2 other = make_float2 (__shfl_xor_sync (0xffffffffu, mine.x, 1),
                                          __shfl_xor_sync (0xffffffffu, mine.y, 1));
        // thread 0: E + O'; thread 1: E - O' (E is the partner's value)
        v[j] = h ? csub (other, mine) : cadd (mine, other);
      }
      const unsigned k0 = 16 * h;
      float2* dst = scratch + ((uint64_t (b) * in.nchan + c) * in.npol + p) * N + i2;
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        const unsigned k1 = k0 + j;
        float2 y = v[j];
        // four-step twiddle w_N^{k1 n2} (row k1 of the [n1][n2] table)
        if (k1) y = cmul (y, __ldg (tw4 + uint64_t (k1) * n2 + i2));
        dst[uint64_t (k1) * n2] = y;
      }
    }
    return;
  }
  const unsigned i2 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t t0 = (part0 + b) * nkeep + i2;
  for (unsigned p = 0; p < in.npol; p++)
  {
    float2 v[N1];
#pragma unroll
    for (int k = 0; k < N1; k++)
      v[k] = fetch<KIND> (in, s_lut, c, p, t0 + uint64_t (k) * n2);
    if (apod)
    {
      // Apodization::operate on the part before the forward FFT (Convolution.C:739-743)
#pragma unroll
      for (int k = 0; k < N1; k++)
      {
        const float w = __ldg (apod + uint64_t (k) * n2 + i2);
        v[k] = make_float2 (__fmul_rn (v[k].x, w), __fmul_rn (v[k].y, w));
      }
    }
    RegDFT<N1, -1>::run (v);
    // four-step twiddle w_N^{k1 n2} (row k1 of the [n1][n2] table; coalesced)
#pragma unroll
    for (int k = 1; k < N1; k++)
      v[k] = cmul (v[k], __ldg (tw4 + uint64_t (k) * n2 + i2));
    float2* dst = scratch + ((uint64_t (b) * in.nchan + c) * in.npol + p) * N + i2;
#pragma unroll
    for (int k = 0; k < N1; k++)
      dst[uint64_t (k) * n2] = v[k];
  }
}

// --------------------------------------------------------------------------
// K1 with the filterbank in front (Filterbank with freq_res 1 and 64 channels,
// FilterbankEngineCPU.C:379-535, then the first four-step pass of each
// channel's convolution), for raw TFPD input of one channel and two
// polarisations and n1 = 8.  The filterbank's own output never reaches
// memory: a warp takes one column i2 of one part and computes, for the eight
// filterbank samples t0 + j*n2 of that column, all 64 channels of both
// polarisations, then each channel's 8-point column DFT.
//
// Lane (j, q), j = lane/4, q = lane%4, reads raw samples s = q + 4m (m < 16)
// of filterbank sample j: a 16-point DFT over m and the twiddle w64^(q ka)
// give Y[q][ka] (ka < 16).  One transpose through the warp's shared buffer
// hands lane 2 ka + pol the 32 values Y[q][ka] of every (q, j): 4-point DFTs
// over q give channels c = ka + 16 kb (kb < 4) of each filterbank sample,
// and 8-point DFTs over j the four channels' column DFTs, all in registers
// (64-point DFT as 16 x 4, X[ka + 16 kb] = sum_q w4^(q kb) w64^(q ka)
// Y[q][ka]).  The block's four warps (four consecutive
// columns) stage their outputs in shared memory and write each scratch row
// in runs of one 32-byte sector (blocks of two or eight warps measured
// slower).  The transpose's rows are 34 float2 apart, so its stores (one row,
// 32 lanes) and 16-byte loads (32 rows) are free of bank conflicts.  The staging is column-major with the even and odd rows in two
// halves (row -> row/2 + (row odd) FBC_SODD, column stride FBC_SP = 2 mod 16):
// the 16 rows a half-warp stores (two apart) and the 4 x 4 (row, column)
// pairs it loads for the write-out then fall in 16 distinct bank pairs.
// --------------------------------------------------------------------------

constexpr int FBC_THREADS = 128;
constexpr int FBC_COLS = FBC_THREADS / 32;      // columns per block, one per warp
constexpr int FBC_XROW = 34;                    // exchange row stride (float2; 16-byte reads)
constexpr int FBC_XSTRIDE = 32 * FBC_XROW;      // float2 per warp exchange buffer
constexpr int FBC_SODD = 520;                   // staging offset of the odd rows (8 mod 16)
constexpr int FBC_SP = 1042;                    // staging column stride (2 mod 16)
constexpr size_t FBC_SMEM =
    (size_t (FBC_SP) * FBC_COLS > size_t (FBC_COLS) * FBC_XSTRIDE ? size_t (FBC_SP) * FBC_COLS
                                                                  : size_t (FBC_COLS) * FBC_XSTRIDE)
    * sizeof (float2);

__host__ __device__ constexpr int fbc_stage (int row, int col)
{
  return col * FBC_SP + (row >> 1) + (row & 1) * FBC_SODD;
}

// (float(x) + 0.5f) * scale for the two's-complement byte x, bit for bit:
// 2^22 + (x + 128) has its last mantissa bit worth 0.5, so subtracting
// 2^22 + 127.5 leaves x + 0.5 exactly; no int -> float conversion
__device__ __forceinline__ float unpack_affine (unsigned byte, float scale)
{
  const float big = __int_as_float (0x4a800000u | (((byte & 0xffu) ^ 0x80u) << 1));
  return __fmul_rn (__fsub_rn (big, 4194431.5f), scale);
}

// The 8-bit table of the fused filterbank pass is one 1 KB copy in shared
// memory.  Eight interleaved copies (lane l reading copy l % 8, so a warp's
// random lookups spread over all banks) measured 10 % slower on the C2 pass:
// the 8 KB table costs more in occupancy than the bank conflicts it removes.

template <int KIND, bool AFFINE>
__device__ __forceinline__ void fetch_raw2 (const InputView& in, const float* s_lut, uint64_t r,
                                            float2& p0, float2& p1)
{
  const void* base = in.main;
  const uint64_t npre = in.npre * 64;
  if (r < npre)
    base = in.pre;
  else
    r -= npre;
  if constexpr (KIND == IN_INT8)
  {
    const unsigned w = __ldg (static_cast<const unsigned*> (base) + r);
    if constexpr (AFFINE)
    {
      const float sc = in.lut_scale;
      p0 = make_float2 (unpack_affine (w, sc), unpack_affine (w >> 8, sc));
      p1 = make_float2 (unpack_affine (w >> 16, sc), unpack_affine (w >> 24, sc));
    }
    else
    {
      p0 = make_float2 (s_lut[w & 0xff], s_lut[(w >> 8) & 0xff]);
      p1 = make_float2 (s_lut[(w >> 16) & 0xff], s_lut[w >> 24]);
    }
  }
  else
  {
    const uint2 w = __ldg (static_cast<const uint2*> (base) + r);
    short a = short (w.x & 0xffff), b = short (w.x >> 16);
    short c = short (w.y & 0xffff), d = short (w.y >> 16);
    if (in.offset_binary)
    {
      a = short (a ^ 0x8000);
      b = short (b ^ 0x8000);
      c = short (c ^ 0x8000);
      d = short (d ^ 0x8000);
    }
    p0 = make_float2 (__fadd_rn (float (a), 0.5f), __fadd_rn (float (b), 0.5f));
    p1 = make_float2 (__fadd_rn (float (c), 0.5f), __fadd_rn (float (d), 0.5f));
  }
}

template <int KIND, bool AFFINE>
__global__ void __launch_bounds__ (FBC_THREADS, 768 / FBC_THREADS)
k_fwd_cols_fb64 (const InputView in, const float* __restrict__ lut, const uint64_t nkeep,
                 const uint64_t part0, const unsigned n2, const float2* __restrict__ tw4,
                 float2* __restrict__ scratch)
{
  extern __shared__ __align__ (16) float2 s_fbc[];
  __shared__ float s_lut[AFFINE ? 1 : 256];
  __shared__ float2 s_tw64[64];
  if (!AFFINE && in.kind == IN_INT8)
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
      s_lut[i] = lut[i];
  if (threadIdx.x < 64)
    s_tw64[threadIdx.x] = make_float2 (cos64 (int (threadIdx.x)), -sin64 (int (threadIdx.x)));
  __syncthreads ();
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned j = lane >> 2, q = lane & 3;
  const unsigned i0 = blockIdx.x * FBC_COLS;
  const unsigned i2 = i0 + warp;
  const unsigned b = blockIdx.y;
  const uint64_t N = 8ull * n2;
  float2* xb = s_fbc + warp * FBC_XSTRIDE;

  // raw samples q + 4m of filterbank sample t, both polarisations
  const uint64_t t = (part0 + b) * nkeep + i2 + uint64_t (j) * n2;
  float2 x0[16], x1[16];
#pragma unroll
  for (int m = 0; m < 16; m++)
    fetch_raw2<KIND, AFFINE> (in, s_lut, t * 64 + q + 4 * m, x0[m], x1[m]);
  RegDFT<16, -1>::run (x0);
  RegDFT<16, -1>::run (x1);
  // twiddle w64^(q ka); lane (j, q) then hands Y[q][ka] of both
  // polarisations to lane 2 ka + pol through the warp's buffer (row 2 ka + pol,
  // column 4 j + q, rows FBC_XROW float2 apart)
#pragma unroll
  for (int ka = 0; ka < 16; ka++)
  {
    const float2 w = s_tw64[(q * ka) & 63];
    xb[(2 * ka) * FBC_XROW + lane] = cmul (x0[ka], w);
    xb[(2 * ka + 1) * FBC_XROW + lane] = cmul (x1[ka], w);
  }
  __syncwarp ();
  // lane 2 ka + pol reads its row in 16-byte pairs: z[jj][qq] = Y[qq][ka] of
  // filterbank sample jj
  float2 z[8][4];
#pragma unroll
  for (int jj = 0; jj < 8; jj++)
#pragma unroll
    for (int qq = 0; qq < 4; qq += 2)
    {
      const float4 t = *reinterpret_cast<const float4*> (xb + lane * FBC_XROW + 4 * jj + qq);
      z[jj][qq] = make_float2 (t.x, t.y);
      z[jj][qq + 1] = make_float2 (t.z, t.w);
    }
  // 4-point DFTs over q: z[jj][kb] = channel ka + 16 kb of filterbank sample jj
#pragma unroll
  for (int jj = 0; jj < 8; jj++) RegDFT<4, -1>::run (z[jj]);
  // the column DFTs over the eight filterbank samples, per channel
  float2 col[4][8];
#pragma unroll
  for (int kb = 0; kb < 4; kb++)
  {
#pragma unroll
    for (int jj = 0; jj < 8; jj++) col[kb][jj] = z[jj][kb];
    RegDFT<8, -1>::run (col[kb]);
  }
  // four-step twiddle w_N^(k1 n2) of column i2, and the filterbank
  // normaliser 1/sqrt(64) (exact)
  float2 tw[8];
  tw[0] = make_float2 (1.f, 0.f);
#pragma unroll
  for (int k1 = 1; k1 < 8; k1++) tw[k1] = __ldg (tw4 + uint64_t (k1) * n2 + i2);
  __syncthreads ();                    // every warp is done with its exchange buffer
  // channel c = ka + 16 kb, pol of lane 2 ka + pol; staging row
  // k1*128 + c*2 + pol, column = warp
  {
    const unsigned ka = lane >> 1, pol = lane & 1;
#pragma unroll
    for (int kb = 0; kb < 4; kb++)
    {
      const unsigned c = ka + 16 * kb;
#pragma unroll
      for (int k1 = 0; k1 < 8; k1++)
      {
        float2 o = k1 ? cmul (col[kb][k1], tw[k1]) : col[kb][k1];
        o = make_float2 (__fmul_rn (o.x, 0.125f), __fmul_rn (o.y, 0.125f));
        s_fbc[fbc_stage (k1 * 128 + c * 2 + pol, warp)] = o;
      }
    }
  }
  __syncthreads ();
  // scratch row ((b*64 + c)*2 + pol)*N + k1*n2, columns i0 .. i0+FBC_COLS-1
#pragma unroll 4
  for (unsigned idx = threadIdx.x; idx < 1024 * FBC_COLS; idx += FBC_THREADS)
  {
    const unsigned row = idx / FBC_COLS, w = idx % FBC_COLS;
    const unsigned k1 = row >> 7, c = (row & 127) >> 1, pol = row & 1;
    scratch[((uint64_t (b) * 64 + c) * 2 + pol) * N + uint64_t (k1) * n2 + i0 + w] =
        s_fbc[fbc_stage (row, w)];
  }
}

// --------------------------------------------------------------------------
// K2 (persistent): the rows.  Row r holds n2 contiguous values,
// r = ((b*nchan + c)*npol + p)*n1 + k1.
// --------------------------------------------------------------------------

template <int N, int D, int P, bool PI, bool PO>
__device__ __forceinline__ void tpass (const float2* src, float2* dst, float2* v,
                                       const float2* tab)
{
  if constexpr (P < stockham_npass (N))
  {
    constexpr int T = stockham_threads (N);
    constexpr int R = stockham_radix (N, P);
    constexpr int Ns = stockham_ns (N, P);
    StockhamPassT<N, R, T, D, PI, PO>::load (threadIdx.x, src, v);
    __syncthreads ();
    StockhamPassT<N, R, T, D, PI, PO>::compute_store (
        threadIdx.x, Ns, v, dst, P ? tab + pass_table_offset (N, P) : nullptr);
    __syncthreads ();
  }
}

// read-only load kept in L1 ahead of other lines (reused by later rows)
__device__ __forceinline__ float2 ldg_evict_last (const float2* p)
{
  float2 v;
  asm volatile ("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];"
                : "=f"(v.x), "=f"(v.y)
                : "l"(p));
  return v;
}

// L2 prefetch of a global range (16-byte aligned, multiple of 16 bytes)
__device__ __forceinline__ void prefetch_l2 (const void* p, unsigned bytes)
{
  asm volatile ("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <int N2>
constexpr size_t rows32_smem_bytes ()
{
  return size_t (spad_size (N2) + Row32<N2>::TABN) * sizeof (float2);
}

// CTAs of k_rows32 resident per SM: at 8192 shared memory (one padded row +
// 10 KB of twiddles) and 128 registers per thread allow two; at 4096 three
// (four would cap the registers at 128, where the 4096-point schedule spills).
// A 30 KB pass-2 table shared by a thread's two butterflies (fewer
// instructions) measured slower: 208 KB of shared memory per SM leaves too
// little L1 for the rows' global loads.  So did one CTA per SM running two
// row groups with named barriers on alternate rows of one run (sharing one
// response row in L1): 1.91 against 1.78 ms per C2 step.
template <int N2>
constexpr unsigned rows32_ctas_per_sm ()
{
  return N2 == 8192 ? 2u : 3u;
}

// The convolution row (CONV: forward FFT, x H, inverse FFT; otherwise the
// inverse FFT alone, for the inverse filterbank's stitched spectra) with 32
// points per thread in three radix passes each way (Row32): pass 0 reads the
// row straight from the scratch in natural order, the forward pass 2, the
// response multiply and the inverse pass 0 run in registers, the last pass
// writes the row back in natural order.  One padded row of shared memory per
// CTA, used in place; several CTAs per SM overlap one another's
// barrier-separated phases.  The next row (and its response) is prefetched
// into L2 while this one is transformed.
template <int N2, bool CONV>
__global__ void __launch_bounds__ (Row32<N2>::T, rows32_ctas_per_sm<N2> ())
k_rows32 (float2* scratch, const float2* __restrict__ H, const unsigned n1,
          const unsigned nchan, const unsigned npol, const unsigned nrows, const unsigned inner)
{
  using RS = Row32<N2>;
  constexpr unsigned ROW_BYTES = N2 * sizeof (float2);
  constexpr unsigned CHUNK = 16384;
  extern __shared__ __align__ (16) float2 s_row32[];
  float2* work = s_row32;
  float2* tab1 = work + spad_size (N2);
  float2* th = tab1 + RS::TAB1;
  float2* tl = th + RS::TABH;
  const int tid = threadIdx.x;
  for (int i = tid; i < RS::TABN; i += RS::T) tab1[i] = RS::table_entry (i);

  // Rows are walked with their response row (channel, k1) outermost and the
  // parts and polarisations innermost (inner = parts x polarisations), and
  // each CTA takes a contiguous run of that order: the rows of one response
  // row follow each other on one SM, which keeps the response in its L1
  // (loaded evict-last, the streamed rows evict-first).
  const auto row_of = [=] (unsigned idx, unsigned& hrow) {
    hrow = idx / inner;                             // c * n1 + k1
    const unsigned bp = idx % inner;
    return ((bp / npol) * nchan * n1 + hrow / n1 * n1) * npol + (bp % npol) * n1 + hrow % n1;
  };
  float2 v[32];
  const unsigned run = (nrows + gridDim.x - 1) / gridDim.x;
  const unsigned idx_end = min (nrows, (blockIdx.x + 1) * run);
  for (unsigned idx = blockIdx.x * run; idx < idx_end; idx++)
  {
    unsigned hrow = 0;
    const unsigned row = CONV ? row_of (idx, hrow) : idx;
    float2* grow = scratch + uint64_t (row) * N2;
    const unsigned next = idx + 1;
    if (tid == 0 && next < idx_end)
    {
      unsigned nh = 0;
      const unsigned nrow = CONV ? row_of (next, nh) : next;
      const char* nr = reinterpret_cast<const char*> (scratch + uint64_t (nrow) * N2);
      for (unsigned o = 0; o < ROW_BYTES; o += CHUNK) prefetch_l2 (nr + o, CHUNK);
      if (CONV && nh != hrow)
      {
        const char* hp = reinterpret_cast<const char*> (H + uint64_t (nh) * N2);
        for (unsigned o = 0; o < ROW_BYTES; o += CHUNK) prefetch_l2 (hp + o, CHUNK);
      }
    }
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++) v[16 * b + r] = __ldcs (grow + tid + b * RS::T + r * RS::NS2);
    __syncthreads ();     // the previous row's last shared-memory reads are done
    if constexpr (CONV)
    {
      RS::template p0_compute_store<-1> (tid, v, work);
      __syncthreads ();
      RS::p1_load (tid, work, v);
      __syncthreads ();
      RS::template p1_compute_store<-1> (tid, v, work, tab1);
      __syncthreads ();
      RS::p2_load (tid, work, v);
      __syncthreads ();
      RS::template p2_compute<-1> (tid, v, th, tl);
      // Response::operate (Response.C:662-726): (f_r d_r - f_i d_i, f_i d_r + f_r d_i)
      const float2* h = H + uint64_t (hrow) * N2;
#pragma unroll
      for (int b = 0; b < 2; b++)
#pragma unroll
        for (int r = 0; r < 16; r++)
        {
          const float2 d = v[16 * b + r];
          const float2 f = ldg_evict_last (h + tid + b * RS::T + r * RS::NS2);
          v[16 * b + r] = make_float2 (d.x * f.x - d.y * f.y, d.x * f.y + d.y * f.x);
        }
    }
    RS::template p0_compute_store<+1> (tid, v, work);
    __syncthreads ();
    RS::p1_load (tid, work, v);
    __syncthreads ();
    RS::template p1_compute_store<+1> (tid, v, work, tab1);
    __syncthreads ();
    RS::p2_load (tid, work, v);
    RS::template p2_compute<+1> (tid, v, th, tl);
    RS::p2_store (tid, v, grow);
  }
}

// --------------------------------------------------------------------------
// K3: inverse column DFTs, overlap discard, voltage out or detect + fold
// --------------------------------------------------------------------------

// One column of an inverse four-step pass: N1 values stride apart, the
// conjugate twiddles tw[k*tw_stride], then the N1-point inverse DFT.
template <int N1>
__device__ __forceinline__ void inv_column (const float2* __restrict__ src, uint64_t stride,
                                            const float2* __restrict__ tw, unsigned tw_stride,
                                            float2* v)
{
#pragma unroll
  for (int k = 0; k < N1; k++)
    v[k] = src[uint64_t (k) * stride];
#pragma unroll
  for (int k = 1; k < N1; k++)
    v[k] = cmulc (v[k], __ldg (tw + uint64_t (k) * tw_stride));
  RegDFT<N1, +1>::run (v);
}

// Two polarisations of 16 or 32 values each do not fit in registers beside
// the DFT's temporaries: the first waits in shared memory (one slot per
// thread, so no barrier) while the second is transformed.
template <int N1, int NPOL>
__host__ __device__ constexpr bool stage_first_pol () { return NPOL == 2 && N1 >= 16; }

template <int N1, int NPOL, int MODE, int NOUT>
__global__ void __launch_bounds__ (128, N1 >= 32 ? 3 : 4)
k_inv_cols (const float2* __restrict__ scratch, const unsigned n2, const unsigned nchan,
            const uint64_t nkeep, const unsigned nfilt_pos, const uint64_t part0,
            const float2* __restrict__ tw4, const FoldView fv, const VoltView vv)
{
  const unsigned b = blockIdx.y;
  const unsigned c = blockIdx.z;
  const uint64_t N = uint64_t (N1) * n2;
  const uint64_t tbase0 = (part0 + b) * nkeep;
  if constexpr (N1 == 32)
  {
    // Two threads per column (16 columns per warp): thread h = lane & 1 of a
    // pair takes rows 2m + h, a 16-point inverse DFT of them gives E (h = 0)
    // or O (h = 1), thread 1 applies w32^j, one exchange leaves
    // X[j] = E[j] + w32^j O[j] with thread 0 and X[j + 16] = E[j] - w32^j O[j]
    // with thread 1; a second shuffle moves them so that lanes 0..15 hold
    // X[j] of the warp's 16 columns and lanes 16..31 X[j + 16] (runs of
    // consecutive samples for the fold).
    const unsigned lane = threadIdx.x & 31;
    const unsigned h = lane & 1;
    const unsigned colw = blockIdx.x * 64 + (threadIdx.x >> 5) * 16;
    const unsigned i2 = colw + (lane >> 1);
    float2 v[NPOL][16];
#pragma unroll
    for (int m = 0; m < 16; m++)
    {
      const unsigned k = 2 * m + h;
      const float2 w = __ldg (tw4 + uint64_t (k) * n2 + i2);
#pragma unroll
      for (int p = 0; p < NPOL; p++)
      {
        const float2 x = scratch[((uint64_t (b) * nchan + c) * NPOL + p) * N + uint64_t (k) * n2 + i2];
        v[p][m] = k ? cmulc (x, w) : x;
      }
    }
    const int srcl = lane < 16 ? 2 * int (lane) : 2 * (int (lane) - 16) + 1;
#pragma unroll
    for (int p = 0; p < NPOL; p++)
    {
      RegDFT<16, +1>::run (v[p]);
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        const float2 mine = h ? tw_mul<32, +1> (j, v[p][j]) : v[p][j];
        const float2 other = make_float2 (__shfl_xor_sync (FULL, mine.x, 1),
                                          __shfl_xor_sync (FULL, mine.y, 1));
        const float2 x = h ? csub (other, mine) : cadd (mine, other);
        v[p][j] = make_float2 (__shfl_sync (FULL, x.x, srcl), __shfl_sync (FULL, x.y, srcl));
      }
    }
    const unsigned ocol = colw + (lane & 15), koff = 16 * (lane >> 4);
#pragma unroll
    for (int j = 0; j < 16; j++)
    {
      const uint64_t tl = uint64_t (koff + j) * n2 + ocol;
      const bool ok = tl >= nfilt_pos && tl < nfilt_pos + nkeep;
      const uint64_t t = tbase0 + (tl - nfilt_pos);
      if constexpr (MODE == OUT_VOLTAGE)
      {
        if (ok)
        {
#pragma unroll
          for (int p = 0; p < NPOL; p++)
            vv.out[(uint64_t (c) * NPOL + p) * vv.span + t] = v[p][j];
        }
      }
      else
        emit_fold<NOUT> (fv, c, NPOL, ok, t, v[0][j], v[NPOL - 1][j]);
    }
    return;
  }
  const unsigned i2 = blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (stage_first_pol<N1, NPOL> ())

  {
    __shared__ float2 s0[N1 * 128];
    const float2* src = scratch + (uint64_t (b) * nchan + c) * 2 * N + i2;
    {
      float2 v[N1];
      inv_column<N1> (src, n2, tw4 + i2, n2, v);
#pragma unroll
      for (int k = 0; k < N1; k++) s0[k * 128 + threadIdx.x] = v[k];
    }
    float2 q[N1];
    inv_column<N1> (src + N, n2, tw4 + i2, n2, q);
#pragma unroll (N1 >= 32 ? 2 : N1)
    for (int k = 0; k < N1; k++)
    {
      const uint64_t tl = uint64_t (k) * n2 + i2;
      const bool ok = tl >= nfilt_pos && tl < nfilt_pos + nkeep;
      const uint64_t t = tbase0 + (tl - nfilt_pos);
      const float2 p = s0[k * 128 + threadIdx.x];
      if constexpr (MODE == OUT_VOLTAGE)
      {
        if (ok)
        {
          vv.out[(uint64_t (c) * 2) * vv.span + t] = p;
          vv.out[(uint64_t (c) * 2 + 1) * vv.span + t] = q[k];
        }
      }
      else
        emit_fold<NOUT> (fv, c, 2, ok, t, p, q[k]);
    }
    return;
  }
  float2 w[N1];
#pragma unroll
  for (int k = 1; k < N1; k++)
    w[k] = __ldg (tw4 + uint64_t (k) * n2 + i2);
  float2 v[NPOL][N1];
#pragma unroll
  for (int p = 0; p < NPOL; p++)
  {
    const float2* src = scratch + ((uint64_t (b) * nchan + c) * NPOL + p) * N + i2;
#pragma unroll
    for (int k = 0; k < N1; k++)
      v[p][k] = src[uint64_t (k) * n2];
    // conjugate four-step twiddle, then the inverse n1-point DFT
#pragma unroll
    for (int k = 1; k < N1; k++)
      v[p][k] = cmulc (v[p][k], w[k]);
    RegDFT<N1, +1>::run (v[p]);
  }
  const uint64_t tbase = (part0 + b) * nkeep;
#pragma unroll
  for (int k = 0; k < N1; k++)
  {
    const uint64_t tl = uint64_t (k) * n2 + i2;
    const bool ok = tl >= nfilt_pos && tl < nfilt_pos + nkeep;
    const uint64_t t = tbase + (tl - nfilt_pos);
    if constexpr (MODE == OUT_VOLTAGE)
    {
      if (ok)
      {
#pragma unroll
        for (int p = 0; p < NPOL; p++)
          vv.out[(uint64_t (c) * NPOL + p) * vv.span + t] = v[p][k];
      }
    }
    else
      emit_fold<NOUT> (fv, c, NPOL, ok, t, v[0][k], v[NPOL - 1][k]);
  }
}

// --------------------------------------------------------------------------
// single-kernel path (n1 == 1): everything in shared memory
// --------------------------------------------------------------------------

template <int N, int T, int KIND, int MODE, int NOUT>
__global__ void __launch_bounds__ (T, 512 / T)
k_fused (const InputView in, const float* __restrict__ lut, const float2* __restrict__ tw,
         const float2* __restrict__ H, const uint64_t nkeep, const unsigned nfilt_pos,
         const uint64_t part0, const FoldView fv, const VoltView vv,
         const float* __restrict__ apod)
{
  extern __shared__ float2 s[];
  __shared__ float s_lut[256];
  constexpr int SP = spad_size (N);
  const unsigned b = blockIdx.x;
  const unsigned c = blockIdx.y;
  const uint64_t part = part0 + b;
  const unsigned npol = in.npol;
  load_lut (in, lut, s_lut);
  __syncthreads ();
  for (unsigned p = 0; p < npol; p++)
    for (int i = threadIdx.x; i < N; i += T)
    {
      float2 x = fetch<KIND> (in, s_lut, c, p, part * nkeep + i);
      if (apod)
      {
        const float w = __ldg (apod + i);
        x = make_float2 (__fmul_rn (x.x, w), __fmul_rn (x.y, w));
      }
      s[p * SP + spad (i)] = x;
    }
  __syncthreads ();
  const float2* h = H + uint64_t (c) * N;
  for (unsigned p = 0; p < npol; p++)
  {
    float2* sp = s + p * SP;
    smem_fft<N, T, -1> (sp, tw);
    for (int i = threadIdx.x; i < N; i += T)
    {
      const float2 d = sp[spad (i)];
      const float2 f = __ldg (h + i);
      sp[spad (i)] = make_float2 (d.x * f.x - d.y * f.y, d.x * f.y + d.y * f.x);
    }
    __syncthreads ();
    smem_fft<N, T, +1> (sp, tw);
  }
  const uint64_t tbase = part * nkeep;
  const unsigned rounds = unsigned ((nkeep + T - 1) / T);
  for (unsigned r = 0; r < rounds; r++)
  {
    const uint64_t j = uint64_t (r) * T + threadIdx.x;
    const bool ok = j < nkeep;
    const int tl = ok ? int (nfilt_pos + j) : 0;
    const float2 pv = s[spad (tl)];
    const float2 qv = npol > 1 ? s[SP + spad (tl)] : make_float2 (0.f, 0.f);
    if (MODE == OUT_VOLTAGE)
    {
      if (ok)
      {
        vv.out[(uint64_t (c) * npol) * vv.span + tbase + j] = pv;
        if (npol > 1) vv.out[(uint64_t (c) * npol + 1) * vv.span + tbase + j] = qv;
      }
    }
    else
      emit_fold<NOUT> (fv, c, npol, ok, tbase + j, pv, qv);
  }
}

// --------------------------------------------------------------------------
// inverse filterbank (InverseFilterbankEngineCPU.C:309-779 restructured)
// --------------------------------------------------------------------------

// Stockham FFT of N points run by a group of T = N/16 threads (tid within the
// group) on the group's own shared-memory array; every group of the CTA runs
// the same passes, so the CTA-wide barriers line up.
// Twiddles come from the per-pass tables (pass_table_offset layout) that the
// caller holds in shared memory.
template <int N, int T, int D, int P>
__device__ __forceinline__ void group_fft_pass (float2* s, float2* v, const float2* tab, int tid)
{
  if constexpr (P < stockham_npass (N))
  {
    constexpr int R = stockham_radix (N, P);
    constexpr int Ns = stockham_ns (N, P);
    StockhamPassT<N, R, T, D, true, true>::load (tid, s, v);
    __syncthreads ();
    StockhamPassT<N, R, T, D, true, true>::compute_store (
        tid, Ns, v, s, P ? tab + pass_table_offset (N, P) : nullptr);
    __syncthreads ();
    group_fft_pass<N, T, D, P + 1> (s, v, tab, tid);
  }
}

// A CTA of IFB_THREADS threads transforms F = 8192/LIN (channel, pol) slots of
// one part: CG = F/npol consecutive fine channels, both pols.  The input tile
// is read so that consecutive threads touch consecutive bytes (for TFPD input
// the slots of one time sample are contiguous; for FPT input the samples of
// one slot are), unpacked and windowed (Apodization::operate) into shared
// memory; each group of LIN/16 threads runs the forward FFT of its slot; then
// the kept bins of both halves -- stitch_one's placement, precomputed per
// channel on the host -- times the response and the spectral window go to the
// output channel's spectrum in four-step order (bin k at row k mod n1, column
// k div n1) for the row kernel.
constexpr int IFB_THREADS = 512;

template <int LIN, int KIND>
__global__ void __launch_bounds__ (IFB_THREADS)
k_ifb_stitch (const InputView in, const IfbShape sh, const IfbTables tb, const uint64_t part0,
              float2* __restrict__ scratch)
{
  constexpr int TF = stockham_threads (LIN);     // threads per transform
  constexpr int F = IFB_THREADS / TF;             // slots per CTA
  // slot stride: the padded transform plus 32 bytes, so that the slots of one
  // time sample written together fall on different banks
  constexpr int SP = spad_size (LIN) + 4;
  constexpr int TABN = pass_tables_size (LIN);
  extern __shared__ float2 s_ifb[];               // [F][SP], then the pass tables
  float2* s_tab = s_ifb + F * SP;
  __shared__ float s_lut[256];
  const unsigned npol = sh.npol;
  const unsigned cg = F / npol;                   // channels per CTA
  const unsigned c0 = blockIdx.x * cg;
  const unsigned b = blockIdx.y;
  load_lut (in, tb.lut, s_lut);
  for (int i = threadIdx.x; i < TABN; i += IFB_THREADS) s_tab[i] = __ldg (tb.ptab_lin + i);
  __syncthreads ();
  const uint64_t t0 = (part0 + b) * sh.in_step;
  // all PER loads of a thread are issued before any is used
  constexpr int PER = F * LIN / IFB_THREADS;
  const unsigned nslot = min (unsigned (F), (sh.nin - c0) * npol);   // live slots
  const uint64_t row = uint64_t (sh.nin) * npol;                       // TFPD values per sample
  uint32_t word[PER];
  float2 fv[KIND == IN_FLOAT ? PER : 1];
#pragma unroll
  for (int k = 0; k < PER; k++)
  {
    const unsigned e = threadIdx.x + k * IFB_THREADS;
    if constexpr (KIND == IN_FLOAT)
    {
      const unsigned slot = e / LIN, t = e % LIN;
      fv[k] = slot < nslot ? __ldg (static_cast<const float2*> (in.main)
                                    + (uint64_t (c0) * npol + slot) * in.main_span + t0 + t)
                           : make_float2 (0.f, 0.f);
    }
    else
    {
      const unsigned slot = e % F, t = e / F;
      const uint64_t idx = (t0 + t) * row + uint64_t (c0) * npol + slot;
      if constexpr (KIND == IN_INT16)
        word[k] = slot < nslot ? __ldg (static_cast<const uint32_t*> (in.main) + idx) : 0u;
      else
        word[k] = slot < nslot ? __ldg (static_cast<const unsigned short*> (in.main) + idx) : 0u;
    }
  }
#pragma unroll
  for (int k = 0; k < PER; k++)
  {
    const unsigned e = threadIdx.x + k * IFB_THREADS;
    unsigned slot, t;
    float2 x;
    if constexpr (KIND == IN_FLOAT)
    {
      slot = e / LIN;
      t = e % LIN;
      x = fv[k];
    }
    else
    {
      slot = e % F;
      t = e / F;
      if constexpr (KIND == IN_INT16)
      {
        short re = short (word[k] & 0xffff), im = short (word[k] >> 16);
        if (in.offset_binary)
        {
          re = short (re ^ 0x8000);
          im = short (im ^ 0x8000);
        }
        // SixteenBitUnpacker.C:69: float(x) + 0.5
        x = make_float2 (__fadd_rn (float (re), 0.5f), __fadd_rn (float (im), 0.5f));
      }
      else
        x = make_float2 (s_lut[word[k] & 0xff], s_lut[word[k] >> 8]);
      if (slot >= nslot) x = make_float2 (0.f, 0.f);
    }
    if (tb.temporal)
    {
      const float w = __ldg (tb.temporal + t);
      x = make_float2 (__fmul_rn (x.x, w), __fmul_rn (x.y, w));
    }
    s_ifb[slot * SP + spad (t)] = x;
  }
  __syncthreads ();
  const unsigned group = threadIdx.x / TF, tid = threadIdx.x % TF;
  float2* s = s_ifb + group * SP;
  {
    float2 v[LIN / TF];
    group_fft_pass<LIN, TF, -1, 0> (s, v, s_tab, tid);
  }
  const unsigned c = c0 + group / npol, p = group % npol;
  if (c >= sh.nin) return;
  const int4 m = __ldg (tb.map + c);
  const unsigned keep2 = sh.keep / 2;
  const unsigned skip2 = (LIN - sh.keep) / 2;
  const unsigned src_neg = sh.dual_sideband ? LIN - keep2 : skip2;
  const unsigned src_pos = sh.dual_sideband ? 0 : skip2 + keep2;
  if (keep2 % sh.n1 == 0)
  {
    // n1 divides keep/2, so every half starts on a multiple of n1 and its
    // bins fill per_row consecutive columns of each four-step row: threads
    // walk them row by row, consecutive threads writing consecutive columns.
    const unsigned per_row = keep2 / sh.n1;
    const bool pow2 = (per_row & (per_row - 1)) == 0;
    const unsigned lg = __ffs (per_row) - 1;
    for (int h = 0; h < 2; h++)
    {
      const int o = h ? m.z : m.x;
      const int offz = h ? m.w : m.y;
      const unsigned off = unsigned (offz & (IFB_ZERO - 1));
      const unsigned src0 = h ? src_pos : src_neg;
      float2* dst = scratch + ((uint64_t (b) * sh.nout + o) * sh.npol + p) * sh.lout + off / sh.n1;
      for (unsigned r = tid; r < keep2; r += TF)
      {
        const unsigned a = pow2 ? r >> lg : r / per_row;
        const unsigned q = r - a * per_row;
        const unsigned j = q * sh.n1 + a;
        float2 y = (offz & IFB_ZERO) ? make_float2 (0.f, 0.f) : s[spad (src0 + j)];
        if (tb.response)
        {
          const float2 f = __ldg (tb.response + uint64_t (o) * sh.lout + off + j);
          y = make_float2 (__fsub_rn (__fmul_rn (f.x, y.x), __fmul_rn (f.y, y.y)),
                           __fadd_rn (__fmul_rn (f.y, y.x), __fmul_rn (f.x, y.y)));
        }
        if (tb.spectral)
        {
          const float w = __ldg (tb.spectral + off + j);
          y = make_float2 (__fmul_rn (y.x, w), __fmul_rn (y.y, w));
        }
        dst[uint64_t (a) * sh.n2 + q] = y;
      }
    }
    return;
  }
  for (unsigned i = tid; i < sh.keep; i += TF)
  {
    const bool neg = i < keep2;
    const unsigned j = neg ? i : i - keep2;
    const int o = neg ? m.x : m.z;
    const int off = neg ? m.y : m.w;
    const unsigned k = unsigned (off & (IFB_ZERO - 1)) + j;
    float2 y = (off & IFB_ZERO) ? make_float2 (0.f, 0.f) : s[spad ((neg ? src_neg : src_pos) + j)];
    if (tb.response)
    {
      // Response::operate: (f_r d_r - f_i d_i, f_i d_r + f_r d_i)
      const float2 f = __ldg (tb.response + uint64_t (o) * sh.lout + k);
      y = make_float2 (__fsub_rn (__fmul_rn (f.x, y.x), __fmul_rn (f.y, y.y)),
                       __fadd_rn (__fmul_rn (f.y, y.x), __fmul_rn (f.x, y.y)));
    }
    if (tb.spectral)
    {
      const float w = __ldg (tb.spectral + k);
      y = make_float2 (__fmul_rn (y.x, w), __fmul_rn (y.y, w));
    }
    float2* dst = scratch + ((uint64_t (b) * sh.nout + o) * sh.npol + p) * sh.lout;
    dst[uint64_t (k % sh.n1) * sh.n2 + k / sh.n1] = y;
  }
}

// Inverse column DFTs of the lout-point transforms (after the row kernel):
// conjugate four-step twiddle, n1-point inverse DFT in registers (n1 may
// carry a factor 3), output discard, voltages out.  Pols one after another.
template <int N1>
__global__ void __launch_bounds__ (128)
k_ifb_cols (const float2* __restrict__ scratch, const IfbShape sh, const float2* __restrict__ tw4,
            const uint64_t part0, const VoltView vv)
{
  const unsigned i2 = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned b = blockIdx.y;
  const unsigned o = blockIdx.z;
  const uint64_t N = uint64_t (N1) * sh.n2;
  const uint64_t tbase = (part0 + b) * sh.out_step;
  for (unsigned p = 0; p < sh.npol; p++)
  {
    const float2* src = scratch + ((uint64_t (b) * sh.nout + o) * sh.npol + p) * N + i2;
    float2 v[N1];
#pragma unroll
    for (int k = 0; k < N1; k++) v[k] = src[uint64_t (k) * sh.n2];
#pragma unroll
    for (int k = 1; k < N1; k++) v[k] = cmulc (v[k], __ldg (tw4 + uint64_t (k) * sh.n2 + i2));
    RegDFTm<N1, +1>::run (v);
    float2* dst = vv.out + (uint64_t (o) * sh.npol + p) * vv.span + tbase;
#pragma unroll
    for (int k = 0; k < N1; k++)
    {
      const uint64_t tl = uint64_t (k) * sh.n2 + i2;
      if (tl >= sh.out_discard_pos && tl < sh.out_discard_pos + sh.out_step)
        dst[tl - sh.out_discard_pos] = v[k];
    }
  }
}

// --------------------------------------------------------------------------
// Filterbank with a response ("During")
// --------------------------------------------------------------------------

// Barrier of a group of TS consecutive threads that exchange data only among
// themselves: a warp barrier when the group lies inside one warp (TS divides
// 32), else the block's.
template <int TS>
__device__ __forceinline__ void group_sync ()
{
  static_assert (TS <= 32 ? 32 % TS == 0 : TS % 32 == 0, "groups must tile the warps");
  if constexpr (TS <= 32)
    __syncwarp ();
  else
    __syncthreads ();
}

// One radix pass of an N-point transform run by the stockham_threads(N)
// threads of one group (lane = index in the group), both sides in the padded
// layout relative to the group's base, or the output unpadded (PO false).
// Every thread of the block calls it.  Its barriers cover the group only, so
// a caller that reads or writes the groups' buffers across groups puts a
// block barrier between that and the passes.
template <int N, int D, int P, bool PO>
__device__ __forceinline__ void gpass (int lane, const float2* src, float2* dst, float2* v,
                                       const float2* tab)
{
  if constexpr (P < stockham_npass (N))
  {
    constexpr int T = stockham_threads (N);
    constexpr int R = stockham_radix (N, P);
    constexpr int Ns = stockham_ns (N, P);
    StockhamPassT<N, R, T, D, true, PO>::load (lane, src, v);
    group_sync<T> ();
    StockhamPassT<N, R, T, D, true, PO>::compute_store (
        lane, Ns, v, dst, P ? tab + pass_table_offset (N, P) : nullptr);
    group_sync<T> ();
  }
}

constexpr int DUR_N2 = 8192;

template <int SEG>
constexpr size_t during_rows_smem ()
{
  return size_t (spad_size (DUR_N2) + Row32<DUR_N2>::TABN + pass_tables_size (SEG))
         * sizeof (float2);
}

// Rows of the big transform (persistent CTAs, one row at a time, two per SM):
// the forward n2-point FFT with 32 points per thread in three passes
// (Row32), the response of each output channel on its segment multiplied in
// registers (Response::operate over nchan_subband channels from
// input_ichan*nchan_subband, FilterbankEngineCPU.C:480-484), then the
// seg-point inverse FFT of every segment, written back in place: each group
// of seg/16 threads takes two segments.  Row r of the scratch is row
// k1 = r mod n1 of (part, input channel, pol).
template <int SEG>
__global__ void __launch_bounds__ (Row32<DUR_N2>::T, 2)
k_rows_during (float2* __restrict__ scratch, const float2* __restrict__ ptab_seg,
               const float2* __restrict__ H, const unsigned n1, const unsigned nsub,
               const unsigned npol, const unsigned nchan_in, const unsigned nrows,
               const unsigned inner)
{
  constexpr int N2 = DUR_N2;
  using RS = Row32<N2>;
  constexpr int T = RS::T;
  constexpr int TABS = pass_tables_size (SEG);
  constexpr int TS = stockham_threads (SEG);
  constexpr int NPS = stockham_npass (SEG);
  constexpr int NG = T / TS;                      // segment groups
  constexpr unsigned ROW_BYTES = N2 * sizeof (float2);
  constexpr unsigned CHUNK = 16384;
  static_assert (NPS == 2 || NPS == 3, "segment transforms of 64 .. 4096 points");
  static_assert (T % TS == 0 && (N2 / SEG) == 2 * NG, "each group takes two segments");
  extern __shared__ __align__ (16) float2 s_dur[];
  float2* work = s_dur;
  float2* tab1 = work + spad_size (N2);
  float2* th = tab1 + RS::TAB1;
  float2* tl = th + RS::TABH;
  float2* tabs = tab1 + RS::TABN;
  const int tid = threadIdx.x;
  for (int i = tid; i < RS::TABN; i += T) tab1[i] = RS::table_entry (i);
  for (int i = tid; i < TABS; i += T) tabs[i] = __ldg (ptab_seg + i);
  const int g = tid / TS, lane = tid % TS;
  // As in k_rows32: rows walked with their response rows (input channel,
  // k1) outermost, parts and polarisations innermost (inner of them), each
  // CTA a contiguous run, the response kept in L1 (evict-last loads) and the
  // scratch rows streamed (evict-first).
  const auto row_of = [=] (unsigned idx, unsigned& hrow) {
    hrow = idx / inner;                             // cin * n1 + k1
    const unsigned bp = idx % inner;
    return ((bp / npol) * nchan_in * n1 + hrow / n1 * n1) * npol + (bp % npol) * n1 + hrow % n1;
  };
  float2 v[32];
  const unsigned run = (nrows + gridDim.x - 1) / gridDim.x;
  const unsigned idx_end = min (nrows, (blockIdx.x + 1) * run);
  for (unsigned idx = blockIdx.x * run; idx < idx_end; idx++)
  {
    unsigned hrow = 0;
    const unsigned row = row_of (idx, hrow);
    const unsigned k1 = hrow % n1;
    const unsigned cin = hrow / n1;
    float2* grow = scratch + uint64_t (row) * N2;
    if (tid == 0 && idx + 1 < idx_end)
    {
      unsigned nh = 0;
      const char* nr = reinterpret_cast<const char*> (scratch + uint64_t (row_of (idx + 1, nh)) * N2);
      for (unsigned o = 0; o < ROW_BYTES; o += CHUNK) prefetch_l2 (nr + o, CHUNK);
    }
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++) v[16 * b + r] = __ldcs (grow + tid + b * T + r * RS::NS2);
    __syncthreads ();     // the previous row's segment passes are done
    RS::template p0_compute_store<-1> (tid, v, work);
    __syncthreads ();
    RS::p1_load (tid, work, v);
    __syncthreads ();
    RS::template p1_compute_store<-1> (tid, v, work, tab1);
    __syncthreads ();
    RS::p2_load (tid, work, v);
    __syncthreads ();
    RS::template p2_compute<-1> (tid, v, th, tl);
    // position i = cs*SEG + f2 of row k1 is bin k1 + n1*f2 of output channel
    // cin*nsub + cs: (f_r d_r - f_i d_i, f_i d_r + f_r d_i), Response.C:662-726
    const float2* hc = H + (uint64_t (cin) * nsub * n1 + k1) * SEG;
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++)
      {
        const int i = tid + b * T + r * RS::NS2;
        const unsigned cs = unsigned (i) / SEG, f2 = unsigned (i) % SEG;
        const float2 f = ldg_evict_last (hc + uint64_t (cs) * n1 * SEG + f2);
        const float2 d = v[16 * b + r];
        work[spad (i)] = make_float2 (d.x * f.x - d.y * f.y, d.x * f.y + d.y * f.x);
      }
    __syncthreads ();
    // spad(s*SEG + i) = spad(s*SEG) + spad(i) because SEG is a multiple of 16
#pragma unroll
    for (int s2 = 0; s2 < 2; s2++)
    {
      const int sg = g + s2 * NG;
      float2* wseg = work + spad (sg * SEG);
      float2* gseg = grow + sg * SEG;
      if constexpr (NPS == 2)
      {
        gpass<SEG, +1, 0, true> (lane, wseg, wseg, v, tabs);
        gpass<SEG, +1, 1, false> (lane, wseg, gseg, v, tabs);
      }
      else
      {
        gpass<SEG, +1, 0, true> (lane, wseg, wseg, v, tabs);
        gpass<SEG, +1, 1, true> (lane, wseg, wseg, v, tabs);
        gpass<SEG, +1, 2, false> (lane, wseg, gseg, v, tabs);
      }
    }
  }
}

// Inverse column DFTs of the freq_res-point transforms: thread i2 holds
// sample t2 = i2 mod seg of output channel cin*nsub + i2/seg; conjugate
// twiddle exp(+2 pi i k1 t2 / freq_res), n1-point inverse DFT giving samples
// t2 + seg*t1, then the discard of nfilt_pos / nfilt_neg
// (FilterbankEngineCPU.C:516-523) and voltages out, or detection + fold.
// seg >= 64, so the 32 lanes of a warp share one output channel.
template <int N1, int NPOL, int MODE, int NOUT>
__global__ void __launch_bounds__ (128, N1 >= 32 ? 3 : 4)
k_inv_cols_during (const float2* __restrict__ scratch, const DuringShape sh, const uint64_t part0,
                   const float2* __restrict__ twd, const FoldView fv, const VoltView vv)
{
  const unsigned i2 = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned b = blockIdx.y;
  const unsigned cin = blockIdx.z;
  const uint64_t N = uint64_t (N1) * sh.n2;
  const unsigned cs = i2 / sh.seg, t2 = i2 % sh.seg;
  const unsigned c = cin * sh.nsub + cs;
  if constexpr (stage_first_pol<N1, NPOL> ())
  {
    __shared__ float2 s0[N1 * 128];
    const float2* src = scratch + (uint64_t (b) * sh.nchan_in + cin) * 2 * N + i2;
    {
      float2 v[N1];
      inv_column<N1> (src, sh.n2, twd + t2, sh.seg, v);
#pragma unroll
      for (int k = 0; k < N1; k++) s0[k * 128 + threadIdx.x] = v[k];
    }
    float2 q[N1];
    inv_column<N1> (src + N, sh.n2, twd + t2, sh.seg, q);
    const uint64_t tb = (part0 + b) * sh.nkeep;
#pragma unroll (N1 >= 32 ? 2 : N1)
    for (int k = 0; k < N1; k++)
    {
      const uint64_t tl = uint64_t (k) * sh.seg + t2;
      const bool ok = tl >= sh.nfilt_pos && tl < sh.nfilt_pos + sh.nkeep;
      const uint64_t t = tb + (tl - sh.nfilt_pos);
      const float2 p = s0[k * 128 + threadIdx.x];
      if constexpr (MODE == OUT_VOLTAGE)
      {
        if (ok)
        {
          vv.out[(uint64_t (c) * 2) * vv.span + t] = p;
          vv.out[(uint64_t (c) * 2 + 1) * vv.span + t] = q[k];
        }
      }
      else
        emit_fold<NOUT> (fv, c, 2, ok, t, p, q[k]);
    }
    return;
  }
  float2 w[N1];
#pragma unroll
  for (int k = 1; k < N1; k++)
    w[k] = __ldg (twd + uint64_t (k) * sh.seg + t2);
  float2 v[NPOL][N1];
#pragma unroll
  for (int p = 0; p < NPOL; p++)
  {
    const float2* src = scratch + ((uint64_t (b) * sh.nchan_in + cin) * NPOL + p) * N + i2;
#pragma unroll
    for (int k = 0; k < N1; k++)
      v[p][k] = src[uint64_t (k) * sh.n2];
#pragma unroll
    for (int k = 1; k < N1; k++)
      v[p][k] = cmulc (v[p][k], w[k]);
    RegDFT<N1, +1>::run (v[p]);
  }
  const uint64_t tbase = (part0 + b) * sh.nkeep;
#pragma unroll
  for (int k = 0; k < N1; k++)
  {
    const uint64_t tl = uint64_t (k) * sh.seg + t2;
    const bool ok = tl >= sh.nfilt_pos && tl < sh.nfilt_pos + sh.nkeep;
    const uint64_t t = tbase + (tl - sh.nfilt_pos);
    if constexpr (MODE == OUT_VOLTAGE)
    {
      if (ok)
      {
#pragma unroll
        for (int p = 0; p < NPOL; p++)
          vv.out[(uint64_t (c) * NPOL + p) * vv.span + t] = v[p][k];
      }
    }
    else
      emit_fold<NOUT> (fv, c, NPOL, ok, t, v[0][k], v[NPOL - 1][k]);
  }
}

// Column passes of N1 = 64 .. 512 points (big transforms of up to 2^22 =
// 512 x 8192 points): a CTA of N1 threads takes COLW = 16 adjacent columns,
// loads them row by row (16 consecutive samples per row) into shared memory,
// one column per group of N1/16 threads, and runs the N1-point Stockham
// transforms there (per-pass tables in shared memory).  Column stride
// spad_size(N1) + 1 keeps the 16 columns of a row on different banks.
constexpr int COLW = 16;

// Buffer stride: with 16 columns per CTA (a half-warp touches one row) 1 mod
// 16 float2 keeps the columns on distinct bank pairs; with 8 (a half-warp
// touches two adjacent rows, k even and k + 1) 2 mod 16 does.
template <int N1, int CW = COLW>
B200_CE int colbig_stride () { return spad_size (N1) + (CW >= 16 ? 1 : 2); }

template <int N1, int NPOL>
constexpr size_t colbig_smem ()
{
  return size_t (NPOL * COLW * colbig_stride<N1> () + pass_tables_size (N1)) * sizeof (float2);
}

// columns per CTA of the inverse pass: 8 for 512-point columns, so that both
// polarisations (72 KB) leave room for a second CTA on the SM
template <int N1>
B200_CE int inv_colw () { return N1 >= 512 ? 8 : COLW; }

template <int N1, int NPOL>
constexpr size_t colbig_inv_smem ()
{
  return size_t (NPOL * inv_colw<N1> () * colbig_stride<N1, inv_colw<N1> ()> ()
                 + pass_tables_size (N1))
         * sizeof (float2);
}

// the N1-point transform (direction D) of every column in col[]
template <int N1, int D, int SP = colbig_stride<N1> ()>
__device__ __forceinline__ void colbig_fft (float2* col, const float2* tab)
{
  constexpr int TS = stockham_threads (N1);
  const int g = threadIdx.x / TS, lane = threadIdx.x % TS;
  float2* base = col + g * SP;
  float2 v[16];
  gpass<N1, D, 0, true> (lane, base, base, v, tab);
  gpass<N1, D, 1, true> (lane, base, base, v, tab);
  gpass<N1, D, 2, true> (lane, base, base, v, tab);
}

// Forward: unpack (and window) on load, N1-point DFTs down the columns, the
// four-step twiddle w_N^{k1 i2}, rows of the scratch out.
template <int N1, int KIND>
__global__ void __launch_bounds__ (N1, 1024 / N1)
k_fwd_cols_big (const InputView in, const float* __restrict__ lut, const uint64_t step,
                const uint64_t part0, const unsigned n2, const float2* __restrict__ tw4,
                const float2* __restrict__ ptab_col, float2* __restrict__ scratch,
                const float* __restrict__ apod)
{
  static_assert (stockham_npass (N1) <= 3, "column transforms of at most three passes");
  constexpr int T = N1;
  constexpr int SP = colbig_stride<N1> ();
  constexpr int TAB = pass_tables_size (N1);
  extern __shared__ __align__ (16) float2 s_cb[];
  float2* col = s_cb;
  float2* tab = s_cb + COLW * SP;
  __shared__ float s_lut[256];
  load_lut (in, lut, s_lut);
  for (int i = threadIdx.x; i < TAB; i += T) tab[i] = __ldg (ptab_col + i);
  const unsigned c0 = blockIdx.x * COLW;
  const unsigned b = blockIdx.y;
  const unsigned c = blockIdx.z;
  const uint64_t N = uint64_t (N1) * n2;
  const uint64_t t0 = (part0 + b) * step + c0;
  // thread (kk, j) takes rows k = kk + m KSTEP of column c0 + j
  constexpr int KSTEP = T / COLW;
  const int j = threadIdx.x % COLW, kk = threadIdx.x / COLW;
  // The block's window t0 + k n2 + j lies in one segment of the input (the
  // carried prefix or the main block) except in the parts that straddle the
  // prefix's end; there each sample takes the general fetch.
  const bool one_seg = t0 >= in.npre || t0 + uint64_t (N1 - 1) * n2 + (COLW - 1) < in.npre;
  const bool in_pre = t0 < in.npre;
  const uint64_t ts = in_pre ? t0 : t0 - in.npre;
  const float* ap = apod ? apod + uint64_t (kk) * n2 + c0 + j : nullptr;
  const uint64_t rstep = uint64_t (KSTEP) * n2;
  for (unsigned p = 0; p < in.npol; p++)
  {
    __syncthreads ();
    const auto put = [&] (int k, float2 x) {
      if (ap)
      {
        const float w = __ldg (ap + uint64_t (k - kk) * n2);
        x = make_float2 (__fmul_rn (x.x, w), __fmul_rn (x.y, w));
      }
      col[j * SP + spad (k)] = x;
    };
    if (one_seg && KIND == IN_FLOAT)
    {
      const float2* f = static_cast<const float2*> (in_pre ? in.pre : in.main)
                        + (uint64_t (c) * in.npol + p) * (in_pre ? in.pre_span : in.main_span)
                        + ts + uint64_t (kk) * n2 + j;
      for (int k = kk; k < N1; k += KSTEP, f += rstep) put (k, __ldg (f));
    }
    else if (one_seg)
    {
      // one complex sample per (t, c, p): 2 bytes (int8) or 4 (int16)
      const uint64_t cs = uint64_t (in.nchan) * in.npol;
      const uint64_t i0 = (ts + uint64_t (kk) * n2 + j) * cs + c * in.npol + p;
      const uint64_t istep = rstep * cs;
      if constexpr (KIND == IN_INT8)
      {
        const unsigned short* q = static_cast<const unsigned short*> (in_pre ? in.pre : in.main) + i0;
        for (int k = kk; k < N1; k += KSTEP, q += istep)
        {
          const unsigned short w = __ldg (q);
          put (k, make_float2 (s_lut[w & 0xff], s_lut[w >> 8]));
        }
      }
      else
      {
        const unsigned* q = static_cast<const unsigned*> (in_pre ? in.pre : in.main) + i0;
        for (int k = kk; k < N1; k += KSTEP, q += istep)
        {
          const unsigned w = __ldg (q);
          short re = short (w & 0xffff), im = short (w >> 16);
          if (in.offset_binary)
          {
            re = short (re ^ 0x8000);
            im = short (im ^ 0x8000);
          }
          // SixteenBitUnpacker.C:69: float(x) + 0.5
          put (k, make_float2 (__fadd_rn (float (re), 0.5f), __fadd_rn (float (im), 0.5f)));
        }
      }
    }
    else
      for (int k = kk; k < N1; k += KSTEP)
        put (k, fetch<KIND> (in, s_lut, c, p, t0 + uint64_t (k) * n2 + j));
    __syncthreads ();
    colbig_fft<N1, -1> (col, tab);
    __syncthreads ();                  // the output below reads across columns' groups
    float2* dst = scratch + ((uint64_t (b) * in.nchan + c) * in.npol + p) * N + c0 + j
                  + uint64_t (kk) * n2;
    const float2* tw = tw4 + uint64_t (kk) * n2 + c0 + j;
    for (int k1 = kk; k1 < N1; k1 += KSTEP, dst += rstep, tw += rstep)
    {
      float2 y = col[j * SP + spad (k1)];
      if (k1) y = cmul (y, __ldg (tw));
      *dst = y;
    }
  }
}

// Inverse columns of the During filterbank for N1 = 64 .. 512: the 16
// columns of a CTA lie in one output channel's segment (seg >= 64); both
// polarisations are loaded with the conjugate twiddle exp(+2 pi i k1 t2 /
// freq_res), transformed, and read back in time order (16 consecutive
// samples per row) for the discard and the voltages or detection + fold.
template <int N1, int NPOL, int MODE, int NOUT>
__global__ void __launch_bounds__ (inv_colw<N1> () * stockham_threads (N1), 1024 / N1)
k_inv_cols_during_big (const float2* __restrict__ scratch, const DuringShape sh,
                       const uint64_t part0, const float2* __restrict__ twd,
                       const float2* __restrict__ ptab_col, const FoldView fv, const VoltView vv)
{
  constexpr int CW = inv_colw<N1> ();
  constexpr int T = CW * stockham_threads (N1);
  constexpr int SP = colbig_stride<N1, CW> ();
  constexpr int TAB = pass_tables_size (N1);
  extern __shared__ __align__ (16) float2 s_cb[];
  float2* tab = s_cb + NPOL * CW * SP;
  for (int i = threadIdx.x; i < TAB; i += T) tab[i] = __ldg (ptab_col + i);
  const unsigned c0 = blockIdx.x * CW;
  const unsigned b = blockIdx.y;
  const unsigned cin = blockIdx.z;
  const uint64_t N = uint64_t (N1) * sh.n2;
  const unsigned cs = c0 / sh.seg, t20 = c0 % sh.seg;
  const unsigned c = cin * sh.nsub + cs;
  // thread (kk, j) takes rows k1 = kk + m KSTEP of column c0 + j
  constexpr int KSTEP = T / CW;
  const int j = threadIdx.x % CW, kk = threadIdx.x / CW;
#pragma unroll
  for (int p = 0; p < NPOL; p++)
  {
    const float2* src = scratch + ((uint64_t (b) * sh.nchan_in + cin) * NPOL + p) * N + c0 + j
                        + uint64_t (kk) * sh.n2;
    const float2* tw = twd + uint64_t (kk) * sh.seg + t20 + j;
    float2* col = s_cb + p * CW * SP + j * SP;
    const uint64_t sstep = uint64_t (KSTEP) * sh.n2, tstep = uint64_t (KSTEP) * sh.seg;
    for (int k1 = kk; k1 < N1; k1 += KSTEP, src += sstep, tw += tstep)
    {
      float2 x = *src;
      if (k1) x = cmulc (x, __ldg (tw));
      col[spad (k1)] = x;
    }
  }
  __syncthreads ();
#pragma unroll
  for (int p = 0; p < NPOL; p++)
    colbig_fft<N1, +1, SP> (s_cb + p * CW * SP, tab);
  __syncthreads ();                    // the fold below reads across columns' groups
  const uint64_t tbase = (part0 + b) * sh.nkeep;
  const float2* c0p = s_cb;
  const float2* c1p = s_cb + (NPOL - 1) * CW * SP;
  for (int e = threadIdx.x; e < CW * N1; e += T)
  {
    const int j = e % CW, t1 = e / CW;
    const uint64_t tl = uint64_t (t1) * sh.seg + t20 + j;
    const bool ok = tl >= sh.nfilt_pos && tl < sh.nfilt_pos + sh.nkeep;
    const uint64_t t = tbase + (tl - sh.nfilt_pos);
    const float2 pv = c0p[j * SP + spad (t1)];
    const float2 qv = c1p[j * SP + spad (t1)];
    if constexpr (MODE == OUT_VOLTAGE)
    {
      if (ok)
      {
        vv.out[(uint64_t (c) * NPOL) * vv.span + t] = pv;
        if (NPOL == 2) vv.out[(uint64_t (c) * NPOL + 1) * vv.span + t] = qv;
      }
    }
    else
      emit_fold<NOUT> (fv, c, NPOL, ok, t, pv, qv);
  }
}

// --------------------------------------------------------------------------
// response construction
// --------------------------------------------------------------------------

// Dedispersion::build_compute (Dedispersion.C:166-186) on the grid of the
// restated PlasmaResponse::build: channel ichan centred at chan_freq, bin ipt
// at freq = ipt*binwidth - chanwidth/2 (natural order).  FFT-order index k
// maps to ipt = k + N/2 (mod N) when the halves are swapped
// (Response::doswap, Response.C:998-1050).  Written in four-step order
// H[c][k1][k2] for k = k1 + n1*k2.
__global__ void k_build_chirp (float2* __restrict__ H, const double* __restrict__ chan_freq,
                               const double* __restrict__ coeff, const double* __restrict__ frac_us,
                               const unsigned nfft, const unsigned n1, const unsigned n2,
                               const double binwidth, const double half_chanwidth,
                               const int swap_halves, const int chirp_mode, const float scale)
{
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (idx >= nfft) return;
  const unsigned k1 = unsigned (idx / n2), k2 = unsigned (idx % n2);
  const unsigned k = k1 + n1 * k2;
  const unsigned ipt = swap_halves ? (k + nfft / 2) % nfft : k;
  const double cf = chan_freq[c];
  const double freq = __dsub_rn (__dmul_rn (double (ipt), binwidth), half_chanwidth);
  const double num = __dmul_rn (coeff[c], __dmul_rn (freq, freq));
  double phase = __ddiv_rn (num, __dadd_rn (cf, freq));
  if (frac_us)
  {
    // Dedispersion::build_compute (Dedispersion.C:176-179): the phase of the
    // channel's fractional-sample inter-channel delay
    const double minus_two_pi = -6.283185307179586476925286766559;
    phase = __dadd_rn (phase, __dmul_rn (__dmul_rn (minus_two_pi, freq), frac_us[c]));
  }
  float re, im;
  if (chirp_mode == 0)
  {
    // Dedispersion.C:104-111: phases stored as float, then polar(1.0f, phase)
    const float ph = __double2float_rn (phase);
    sincosf (ph, &im, &re);
  }
  else
  {
    const double two_pi = 6.283185307179586476925286766559;
    const double red = __dsub_rn (phase, __dmul_rn (two_pi, rint (__ddiv_rn (phase, two_pi))));
    double s, co;
    sincos (red, &s, &co);
    re = __double2float_rn (co);
    im = __double2float_rn (s);
  }
  H[uint64_t (c) * nfft + idx] = make_float2 (__fmul_rn (re, scale), __fmul_rn (im, scale));
}

__global__ void k_permute (float2* __restrict__ dst, const float2* __restrict__ src,
                           const unsigned n1, const unsigned n2, const int inverse)
{
  const uint64_t N = uint64_t (n1) * n2;
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (idx >= N) return;
  const unsigned k1 = unsigned (idx / n2), k2 = unsigned (idx % n2);
  const uint64_t k = k1 + uint64_t (n1) * k2;
  if (inverse)
    dst[c * N + k] = src[c * N + idx];
  else
    dst[c * N + idx] = src[c * N + k];
}

// --------------------------------------------------------------------------
// standalone engines
// --------------------------------------------------------------------------

// FFT filterbank without convolution (Filterbank with freq_res = 1,
// FilterbankEngineCPU.C:379-535): every block of NSUB input samples becomes one
// sample in each of NSUB output channels, channel k = FFT bin k scaled by the
// normaliser 1/sqrt(NSUB) (Filterbank.C:171-180).  The unpack is fused into
// the load; one thread transforms one block of one polarisation in registers.
template <int NSUB, int KIND>
__global__ void __launch_bounds__ (128)
k_filterbank (const InputView in, const float* __restrict__ lut, const uint64_t nblk,
              const float scale, float2* __restrict__ out, const uint64_t out_span)
{
  __shared__ float s_lut[256];
  load_lut (in, lut, s_lut);
  __syncthreads ();
  const uint64_t blk = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned p = blockIdx.y;
  const unsigned cin = blockIdx.z;
  if (blk >= nblk) return;
  float2 v[NSUB];
#pragma unroll
  for (int k = 0; k < NSUB; k++)
    v[k] = fetch<KIND> (in, s_lut, cin, p, blk * NSUB + k);
  RegDFT<NSUB, -1>::run (v);
  float2* o = out + (uint64_t (cin) * NSUB * in.npol + p) * out_span + blk;
#pragma unroll
  for (int k = 0; k < NSUB; k++)
    o[uint64_t (k) * in.npol * out_span] = make_float2 (__fmul_rn (scale, v[k].x),
                                                         __fmul_rn (scale, v[k].y));
}

// The same filterbank for NSUB = 128 .. 4096 with the transforms in shared
// memory: a CTA of FB_THREADS threads takes F = 8192/NSUB (block, pol) slots of
// one input channel, reads their samples in address order (coalesced), runs
// one NSUB-point FFT per group of NSUB/16 threads (per-pass twiddle tables in
// shared memory), and writes the bins channel by channel, consecutive threads
// on consecutive output samples.
constexpr int FB_THREADS = 512;

template <int NSUB, int KIND>
__global__ void __launch_bounds__ (FB_THREADS)
k_filterbank_smem (const InputView in, const float* __restrict__ lut, const float2* __restrict__ ptab,
                   const uint64_t nblk, const float scale, float2* __restrict__ out,
                   const uint64_t out_span)
{
  constexpr int TF = stockham_threads (NSUB);
  constexpr int F = FB_THREADS / TF;
  // odd slot stride (in float2): the output loop reads one bin of consecutive
  // slots, which then fall on different banks
  constexpr int SP = spad_size (NSUB) + 1;
  constexpr int TABN = pass_tables_size (NSUB);
  extern __shared__ float2 s_fb[];                 // [F][SP], then the pass tables
  float2* s_tab = s_fb + F * SP;
  __shared__ float s_lut[256];
  const unsigned npol = in.npol;
  const unsigned bpc = F / npol;                    // blocks per CTA
  const uint64_t blk0 = uint64_t (blockIdx.x) * bpc;
  const unsigned cin = blockIdx.y;
  const unsigned nb = unsigned (min (uint64_t (bpc), nblk - blk0));
  load_lut (in, lut, s_lut);
  for (int i = threadIdx.x; i < TABN; i += FB_THREADS) s_tab[i] = __ldg (ptab + i);
  __syncthreads ();
  const uint64_t t0 = blk0 * NSUB;
  // element e in address order: TFPD (t, pol) pairs, FPT (pol, t); all PER
  // loads of a thread are issued before any is used
  constexpr int PER = F * NSUB / FB_THREADS;
  constexpr unsigned HALF = F * NSUB / 2;          // samples per pol when npol == 2
  const bool two = npol == 2;
  const uint64_t rowv = uint64_t (in.nchan) * npol;  // TFPD values per time sample
  uint32_t word[PER];
  float2 fv[KIND == IN_FLOAT ? PER : 1];
#pragma unroll
  for (int k = 0; k < PER; k++)
  {
    const unsigned e = threadIdx.x + k * FB_THREADS;
    if constexpr (KIND == IN_FLOAT)
    {
      const unsigned p = two ? e / HALF : 0, t = two ? e % HALF : e;
      fv[k] = t / NSUB < nb ? __ldg (static_cast<const float2*> (in.main)
                                     + (uint64_t (cin) * npol + p) * in.main_span + t0 + t)
                            : make_float2 (0.f, 0.f);
    }
    else
    {
      const unsigned p = two ? (e & 1) : 0, t = two ? e >> 1 : e;
      const uint64_t idx = (t0 + t) * rowv + uint64_t (cin) * npol + p;
      if constexpr (KIND == IN_INT16)
        word[k] = t / NSUB < nb ? __ldg (static_cast<const uint32_t*> (in.main) + idx) : 0u;
      else
        word[k] = t / NSUB < nb ? __ldg (static_cast<const unsigned short*> (in.main) + idx) : 0u;
    }
  }
#pragma unroll
  for (int k = 0; k < PER; k++)
  {
    const unsigned e = threadIdx.x + k * FB_THREADS;
    unsigned p, t;
    float2 x;
    if constexpr (KIND == IN_FLOAT)
    {
      p = two ? e / HALF : 0;
      t = two ? e % HALF : e;
      x = fv[k];
    }
    else
    {
      p = two ? (e & 1) : 0;
      t = two ? e >> 1 : e;
      if constexpr (KIND == IN_INT16)
      {
        short re = short (word[k] & 0xffff), im = short (word[k] >> 16);
        if (in.offset_binary)
        {
          re = short (re ^ 0x8000);
          im = short (im ^ 0x8000);
        }
        // SixteenBitUnpacker.C:69: float(x) + 0.5
        x = make_float2 (__fadd_rn (float (re), 0.5f), __fadd_rn (float (im), 0.5f));
      }
      else
        x = make_float2 (s_lut[word[k] & 0xff], s_lut[word[k] >> 8]);
    }
    const unsigned blk = t / NSUB, i = t % NSUB;
    if (blk >= nb) x = make_float2 (0.f, 0.f);
    s_fb[(blk * npol + p) * SP + spad (i)] = x;
  }
  __syncthreads ();
  const unsigned group = threadIdx.x / TF, tid = threadIdx.x % TF;
  {
    float2 v[NSUB / TF];
    group_fft_pass<NSUB, TF, -1, 0> (s_fb + group * SP, v, s_tab, tid);
  }
  // bins out: channel cin*NSUB + k of pol p, sample blk0 + blk
  for (unsigned e = threadIdx.x; e < unsigned (F * NSUB); e += FB_THREADS)
  {
    const unsigned blk = e % bpc, rest = e / bpc;
    const unsigned p = rest % npol, k = rest / npol;
    if (blk >= nb || k >= NSUB) continue;
    const float2 y = s_fb[(blk * npol + p) * SP + spad (k)];
    out[((uint64_t (cin) * NSUB + k) * npol + p) * out_span + blk0 + blk] =
        make_float2 (__fmul_rn (scale, y.x), __fmul_rn (scale, y.y));
  }
}

// SpectralKurtosis::transformation for one resolution with noverlap = 1:
// compute (SpectralKurtosis.C:674-798), detect_skfb (:1105-1222) and mask
// (:1465-1566).  A CTA takes up to U consecutive M-sample blocks of one
// channel:
//
//   1. all threads stream the blocks in (16-byte loads, both pols in flight
//      together), square-law detect them in float as the reference does and
//      keep sqld per (block, pol) in shared memory; out of place the voltages
//      are written through to the output at the same time;
//   2. warp 0 forms the reference's two sequential double sums per (block,
//      pol) -- S1 of sqld, S2 of sqld*sqld -- one lane per sum, 4U lanes in
//      all, so that each conversion to double serves 4U values.  The
//      additions run in the reference's order: the sums (and hence the mask)
//      equal the CPU's bit for bit.  Many CTAs per SM keep the loads of some
//      in flight while others add;
//   3. the SK estimator of each block is tested and zapped blocks of the
//      output are overwritten with zeros (in place, only they are written).
//
// Uncounted samples (sqld == 0 with zero_is_valid unset) add +0.0, which
// leaves a sum of non-negative terms unchanged exactly; they are counted by a
// shared atomic as they are met.  Shared memory holds U * npol columns of
// Ms floats, Ms = M rounded up to a multiple of 4 plus 4 (so that the
// columns read together fall on different banks).
constexpr int SK_THREADS = 128;

__host__ __device__ inline unsigned sk_column (unsigned M) { return ((M + 3) & ~3u) + 4; }

template <int U>
__global__ void __launch_bounds__ (SK_THREADS, 12)
k_sk (const float2* __restrict__ in, const uint64_t in_span, float2* out, const uint64_t out_span,
      const uint64_t npart, const unsigned nchan, const unsigned npol, const unsigned M,
      const int zero_is_valid, const unsigned Nd, const float lower,
      const float upper, float* __restrict__ sums, unsigned* __restrict__ counts,
      uint8_t* __restrict__ mask, unsigned long long* __restrict__ nzap)
{
  extern __shared__ __align__ (16) float s_sqld[];   // [unit][pol][Ms]
  __shared__ double s_sum[U][2][2];
  __shared__ unsigned s_zero[U];
  __shared__ int s_zap[U];
  const uint64_t part0 = uint64_t (blockIdx.x) * U;
  const unsigned c = blockIdx.y;
  const unsigned nu = unsigned (min (uint64_t (U), npart - part0));
  const unsigned Ms = sk_column (M);
  const unsigned n4 = M / 2;                      // float4 (two samples) per (block, pol)
  // out == nullptr: statistics only (SpectralKurtosis::compute), nothing written back
  const bool through = out && !(out == in && out_span == in_span);
  const bool two = npol == 2;
  if (threadIdx.x < U) s_zero[threadIdx.x] = 0;
  // both pols of the CTA's blocks are contiguous runs of nu*M samples
  const float4* src0 = reinterpret_cast<const float4*> (in + uint64_t (c) * npol * in_span
                                                        + part0 * M);
  const float4* src1 = src0 + (two ? in_span / 2 : 0);
  float4* dst0 = reinterpret_cast<float4*> (out + uint64_t (c) * npol * out_span + part0 * M);
  float4* dst1 = dst0 + (two ? out_span / 2 : 0);
  __syncthreads ();
  const unsigned total = nu * n4;
#pragma unroll 4
  for (unsigned f = threadIdx.x; f < total; f += SK_THREADS)
  {
    const unsigned u = f / n4, i = f - u * n4;
    const float4 a = __ldcs (src0 + f);
    float4 b = a;
    if (two) b = __ldcs (src1 + f);
    if (through)
    {
      __stcs (dst0 + f, a);
      if (two) __stcs (dst1 + f, b);
    }
    const float a0 = __fadd_rn (__fmul_rn (a.x, a.x), __fmul_rn (a.y, a.y));
    const float a1 = __fadd_rn (__fmul_rn (a.z, a.z), __fmul_rn (a.w, a.w));
    float2* q0 = reinterpret_cast<float2*> (s_sqld + (u * npol) * Ms);
    q0[i] = make_float2 (a0, a1);
    // Mprime counts pol 0, as detect_skfb reads it
    if (!zero_is_valid && (a0 == 0.0f || a1 == 0.0f))
      atomicAdd (&s_zero[u], unsigned (a0 == 0.0f) + unsigned (a1 == 0.0f));
    if (two)
    {
      float2* q1 = reinterpret_cast<float2*> (s_sqld + (u * npol + 1) * Ms);
      q1[i] = make_float2 (__fadd_rn (__fmul_rn (b.x, b.x), __fmul_rn (b.y, b.y)),
                           __fadd_rn (__fmul_rn (b.z, b.z), __fmul_rn (b.w, b.w)));
    }
  }
  __syncthreads ();
  if (threadIdx.x < 4 * U)
  {
    // lane = unit*4 + pol*2 + (S2 ? 1 : 0)
    const unsigned u = threadIdx.x >> 2, p = (threadIdx.x >> 1) & 1;
    const bool sq = threadIdx.x & 1;
    const bool live = u < nu && p < npol;
    const float* xf = s_sqld + (live ? u * npol + p : 0) * Ms;
    const float4* x = reinterpret_cast<const float4*> (xf);
    const unsigned nq = M / 4;
    double acc = 0.0;
    unsigned i = 0;
    if (nq >= 4)
    {
      float4 q[4];
#pragma unroll
      for (int k = 0; k < 4; k++) q[k] = x[k];
      for (i = 4; i + 4 <= nq; i += 4)
      {
        double t[16];
#pragma unroll
        for (int k = 0; k < 4; k++)
        {
          t[4 * k] = double (sq ? __fmul_rn (q[k].x, q[k].x) : q[k].x);
          t[4 * k + 1] = double (sq ? __fmul_rn (q[k].y, q[k].y) : q[k].y);
          t[4 * k + 2] = double (sq ? __fmul_rn (q[k].z, q[k].z) : q[k].z);
          t[4 * k + 3] = double (sq ? __fmul_rn (q[k].w, q[k].w) : q[k].w);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) q[k] = x[i + k];
#pragma unroll
        for (int k = 0; k < 16; k++) acc = __dadd_rn (acc, t[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; k++)
      {
        acc = __dadd_rn (acc, double (sq ? __fmul_rn (q[k].x, q[k].x) : q[k].x));
        acc = __dadd_rn (acc, double (sq ? __fmul_rn (q[k].y, q[k].y) : q[k].y));
        acc = __dadd_rn (acc, double (sq ? __fmul_rn (q[k].z, q[k].z) : q[k].z));
        acc = __dadd_rn (acc, double (sq ? __fmul_rn (q[k].w, q[k].w) : q[k].w));
      }
    }
    for (unsigned jj = 4 * i; jj < M; jj++)
      acc = __dadd_rn (acc, double (sq ? __fmul_rn (xf[jj], xf[jj]) : xf[jj]));
    if (live) s_sum[u][p][sq] = acc;
  }
  __syncthreads ();
  if (threadIdx.x < nu)
  {
    const unsigned u = threadIdx.x;
    const uint64_t unit = (part0 + u) * nchan + c;
    const unsigned Mprime = M - s_zero[u];
    bool zap = false;
    if (Mprime > 0)
    {
      zap = true;
      if (Mprime > 2)
      {
        // Equation (8) of Nita & Gary (2010b), as detect_skfb evaluates it in float
        const float M_fac = __fdiv_rn (float (Mprime * Nd + 1), float (Mprime - 1));
        zap = false;
        for (unsigned p = 0; p < npol; p++)
        {
          const float S1 = __double2float_rn (s_sum[u][p][0]);
          const float S2 = __double2float_rn (s_sum[u][p][1]);
          const float r = __fdiv_rn (S2, __fmul_rn (S1, S1));
          const float V = __fmul_rn (M_fac, __fsub_rn (__fmul_rn (float (Mprime), r), 1.0f));
          if (V > upper || V < lower) zap = true;
        }
      }
    }
    if (sums)
      for (unsigned p = 0; p < npol; p++)
      {
        sums[2 * (unit * npol + p)] = __double2float_rn (s_sum[u][p][0]);
        sums[2 * (unit * npol + p) + 1] = __double2float_rn (s_sum[u][p][1]);
      }
    if (counts) counts[unit] = Mprime;
    if (mask) mask[unit] = zap ? 1 : 0;
    if (zap && nzap) atomicAdd (nzap, 1ull);
    s_zap[u] = zap;
  }
  __syncthreads ();
  // zero the zapped blocks; each thread overwrites exactly the float4s it wrote through
  if (!out) return;
  const float4 zero = make_float4 (0.f, 0.f, 0.f, 0.f);
  for (unsigned f = threadIdx.x; f < total; f += SK_THREADS)
    if (s_zap[f / n4])
    {
      __stcs (dst0 + f, zero);
      if (two) __stcs (dst1 + f, zero);
    }
}

__global__ void k_unpack8 (const uint8_t* __restrict__ in, const uint64_t ndat,
                           const unsigned nchan, const unsigned npol, const unsigned ndim,
                           const float* __restrict__ lut, float* __restrict__ out,
                           const uint64_t span)
{
  __shared__ float s_lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) s_lut[i] = lut[i];
  __syncthreads ();
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat) return;
  const uint8_t* src = in + (t * nchan + c) * npol * ndim;
  for (unsigned p = 0; p < npol; p++)
    for (unsigned d = 0; d < ndim; d++)
      out[(uint64_t (c) * npol + p) * span + t * ndim + d] = s_lut[src[p * ndim + d]];
}

__global__ void k_unpack16 (const int16_t* __restrict__ in, const uint64_t ndat,
                            const unsigned nchan, const unsigned npol, const unsigned ndim,
                            const int offset_binary, float* __restrict__ out,
                            const uint64_t span)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat) return;
  const int16_t* src = in + (t * nchan + c) * npol * ndim;
  for (unsigned p = 0; p < npol; p++)
    for (unsigned d = 0; d < ndim; d++)
    {
      short v = src[p * ndim + d];
      if (offset_binary) v = short (v ^ 0x8000);
      out[(uint64_t (c) * npol + p) * span + t * ndim + d] = __fadd_rn (float (v), 0.5f);
    }
}

__global__ void k_detect (const float2* __restrict__ in, const uint64_t in_span,
                          const uint64_t ndat, const int state, float* __restrict__ out,
                          const uint64_t out_span)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat) return;
  const float2 p = in[(uint64_t (c) * 2) * in_span + t];
  const float2 q = in[(uint64_t (c) * 2 + 1) * in_span + t];
  float v[4];
  detect_values (state, 2, p, q, v);
  const int nout = detect_nout (state);
  for (int k = 0; k < nout; k++)
    out[(uint64_t (c) * nout + k) * out_span + t] = v[k];
}

// Fold::Engine::fold on detected FPT floats (ndim 1): one warp covers 32
// consecutive samples of one (chan, pol).
__global__ void k_fold (const float* __restrict__ in, const uint64_t in_span,
                        const uint64_t ndat, const unsigned npol, const FoldView fv)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  bool ok = t < ndat;
  const unsigned bin = warp_fold_bin (fv.segs, fv.nseg, ok, t, fv.nbin);
  ok = ok && bin < fv.stride;
  for (unsigned p = 0; p < npol; p++)
  {
    float v = ok ? in[(uint64_t (c) * npol + p) * in_span + t] : 0.f;
    warp_fold<1> (ok, bin, &v, fv.profiles + (uint64_t (c) * npol + p) * fv.stride, fv.stride,
                  (c == 0 && p == 0) ? fv.hits : nullptr);
  }
}

// SampleDelay::transformation (SampleDelay.C:247-298) fused with detection and
// the fold: output sample t of channel c is voltage t + applied[c] of that
// channel (rows [chan][pol] of span values).
template <int NOUT>
__global__ void k_delay_fold (const float2* __restrict__ v, const uint64_t span,
                              const int* __restrict__ applied, const uint64_t ndat,
                              const unsigned npol, const FoldView fv)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  const bool ok = t < ndat;
  float2 p = make_float2 (0.f, 0.f), q = make_float2 (0.f, 0.f);
  if (ok)
  {
    const uint64_t i = t + uint64_t (__ldg (applied + c));
    p = v[(uint64_t (c) * npol) * span + i];
    if (npol == 2) q = v[(uint64_t (c) * npol + 1) * span + i];
  }
  emit_fold<NOUT> (fv, c, npol, ok, t, p, q);
}

// SpectralKurtosis::detect_skfb (SpectralKurtosis.C:1105-1222) from sums
// already formed: per (part, chan), Mprime = counts (M when counts is null);
// none counted leaves the mask as it is, one or two zap, otherwise the
// estimator of each polarisation is tested in float as the reference does.
// Zapped cells are set to 1 (others are left alone, as the reference leaves
// them to reset_mask).
__global__ void k_sk_detect (const float* __restrict__ sums, const unsigned* __restrict__ counts,
                             const uint64_t ncell, const unsigned npol, const unsigned M,
                             const unsigned Nd, const float lower, const float upper,
                             uint8_t* __restrict__ mask, unsigned long long* __restrict__ nzap)
{
  const uint64_t unit = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (unit >= ncell) return;
  const unsigned Mprime = counts ? counts[unit] : M;
  if (Mprime == 0) return;
  bool zap = true;
  if (Mprime > 2)
  {
    const float M_fac = __fdiv_rn (float (Mprime * Nd + 1), float (Mprime - 1));
    zap = false;
    for (unsigned p = 0; p < npol; p++)
    {
      const float S1 = sums[2 * (unit * npol + p)];
      const float S2 = sums[2 * (unit * npol + p) + 1];
      const float r = __fdiv_rn (S2, __fmul_rn (S1, S1));
      const float V = __fmul_rn (M_fac, __fsub_rn (__fmul_rn (float (Mprime), r), 1.0f));
      if (V > upper || V < lower) zap = true;
    }
  }
  if (zap)
  {
    mask[unit] = 1;
    if (nzap) atomicAdd (nzap, 1ull);
  }
}

// SpectralKurtosis::compute (SpectralKurtosis.C:674-798) for blocks of M
// samples every `stride` samples (Resolution::prepare with noverlap =
// M / stride, :251-281): one thread per (block, chan, pol, S1 or S2) adds the
// block's values in order in double, as the reference does; S2 adds the
// float square of each sqld.  counts (pol 0's S1 thread) as the reference's
// sum weights.  Blocks overlap, so each sample is read noverlap times; the
// non-overlapping case has its own faster kernel (k_sk).
__global__ void k_sk_sums_strided (const float2* __restrict__ in, const uint64_t span,
                                   const uint64_t nblk, const uint64_t stride,
                                   const unsigned nchan, const unsigned npol, const unsigned M,
                                   const int zero_is_valid, float* __restrict__ sums,
                                   unsigned* __restrict__ counts)
{
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t total = nblk * nchan * npol * 2;
  if (idx >= total) return;
  const unsigned sq = unsigned (idx & 1);
  const unsigned p = unsigned ((idx >> 1) % npol);
  const uint64_t bc = (idx >> 1) / npol;
  const unsigned c = unsigned (bc % nchan);
  const uint64_t b = bc / nchan;
  const float2* x = in + (uint64_t (c) * npol + p) * span + b * stride;
  double acc = 0.0;
  unsigned n = 0;
  for (unsigned i = 0; i < M; i++)
  {
    const float2 v = x[i];
    const float d = __fadd_rn (__fmul_rn (v.x, v.x), __fmul_rn (v.y, v.y));
    if (zero_is_valid || d != 0.0f)
    {
      acc = __dadd_rn (acc, double (sq ? __fmul_rn (d, d) : d));
      n++;
    }
  }
  const uint64_t unit = b * nchan + c;
  sums[2 * (unit * npol + p) + sq] = __double2float_rn (acc);
  if (counts && p == 0 && sq == 0) counts[unit] = n;
}

// SpectralKurtosis::tscrunch_sums (SpectralKurtosis.C:917-986): coarse part q
// takes the fine parts q*offset + isum*offset, isum < nsum, adding the float
// sums and the counts in that order (the reference's indexing, kept as it is)
__global__ void k_sk_tscrunch (const float* __restrict__ sums, const unsigned* __restrict__ counts,
                               const uint64_t npart, const unsigned nchan, const unsigned npol,
                               const unsigned nsum, const unsigned offset,
                               float* __restrict__ osums, unsigned* __restrict__ ocounts)
{
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t per = uint64_t (nchan) * npol * 2;
  if (idx >= npart * per) return;
  const uint64_t q = idx / per, e = idx % per;
  float acc = sums[(q * offset) * per + e];
  for (unsigned isum = 1; isum < nsum; isum++)
    acc = __fadd_rn (acc, sums[(q * offset + uint64_t (isum) * offset) * per + e]);
  osums[idx] = acc;
  // the counts: one per (part, chan), from the threads of pol 0's S1
  if (e % (npol * 2) == 0)
  {
    const unsigned c = unsigned (e / (npol * 2));
    unsigned n = counts ? counts[(q * offset) * nchan + c] : 0;
    for (unsigned isum = 1; isum < nsum && counts; isum++)
      n += counts[(q * offset + uint64_t (isum) * offset) * nchan + c];
    if (ocounts) ocounts[q * nchan + c] = n;
  }
}

// SpectralKurtosis::detect_skfb (SpectralKurtosis.C:1105-1222) at one
// resolution: thresholds from a table of (count, lower, upper) sorted by
// count (get_limits of each count present); a zapped coarse cell flags nflag
// fine cells, flag_step fine parts apart, starting at q * flag_offset.
__global__ void k_sk_detect_skfb (const float* __restrict__ sums, const unsigned* __restrict__ counts,
                                  const uint64_t npart, const unsigned nchan, const unsigned npol,
                                  const unsigned Nd, const unsigned* __restrict__ lim_count,
                                  const float2* __restrict__ lim, const unsigned nlim,
                                  const unsigned nflag, const unsigned flag_step,
                                  const unsigned flag_offset, uint8_t* __restrict__ mask,
                                  unsigned long long* __restrict__ nzap)
{
  const uint64_t unit = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (unit >= npart * nchan) return;
  const unsigned Mprime = counts[unit];
  if (Mprime == 0) return;
  bool zap = true;
  if (Mprime > 2)
  {
    unsigned lo = 0, hi = nlim;
    while (lo + 1 < hi)
    {
      const unsigned mid = (lo + hi) / 2;
      if (lim_count[mid] <= Mprime) lo = mid; else hi = mid;
    }
    const float2 L = lim[lo];       // (lower, upper); the table holds every count present
    const float M_fac = __fdiv_rn (float (Mprime * Nd + 1), float (Mprime - 1));
    zap = false;
    for (unsigned p = 0; p < npol; p++)
    {
      const float S1 = sums[2 * (unit * npol + p)];
      const float S2 = sums[2 * (unit * npol + p) + 1];
      const float r = __fdiv_rn (S2, __fmul_rn (S1, S1));
      const float V = __fmul_rn (M_fac, __fsub_rn (__fmul_rn (float (Mprime), r), 1.0f));
      if (V > L.y || V < L.x) zap = true;
    }
  }
  if (!zap) return;
  if (nzap) atomicAdd (nzap, 1ull);
  const uint64_t q = unit / nchan;
  const unsigned c = unsigned (unit % nchan);
  for (unsigned f = 0; f < nflag; f++)
    mask[(q * flag_offset + uint64_t (f) * flag_step) * nchan + c] = 1;
}

// SpectralKurtosis::mask with overlapping blocks (SpectralKurtosis.C:1465-
// 1566): the reference copies (or zeroes) part after part, M samples each,
// parts `offset` apart, so a sample keeps the decision of the last part that
// covers it: part min(t / offset, npart - 1), mask row part + nskip; the
// input is read from idat_start on.
__global__ void k_sk_mask_overlap (const uint8_t* __restrict__ mask, const float2* __restrict__ in,
                                   const uint64_t in_span, float2* __restrict__ out,
                                   const uint64_t out_span, const uint64_t ndat_out,
                                   const unsigned nchan, const unsigned npol,
                                   const unsigned offset, const uint64_t npart,
                                   const uint64_t nskip, const uint64_t idat_start)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat_out) return;
  const uint64_t part = min (t / offset, npart - 1);
  const bool zap = __ldg (mask + (part + nskip) * nchan + c) != 0;
  for (unsigned p = 0; p < npol; p++)
  {
    const uint64_t r = uint64_t (c) * npol + p;
    out[r * out_span + t] = zap ? make_float2 (0.f, 0.f) : in[r * in_span + idat_start + t];
  }
}

// SpectralKurtosis::mask (SpectralKurtosis.C:1465-1566): out = in, with the
// blocks whose mask is set zeroed (in place when out == in: only those are
// written).
__global__ void k_sk_mask (const uint8_t* __restrict__ mask, const float2* in, const uint64_t in_span,
                           float2* out, const uint64_t out_span, const uint64_t ndat,
                           const unsigned nchan, const unsigned npol, const unsigned M)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat) return;
  const bool zap = __ldg (mask + (t / M) * nchan + c) != 0;
  const bool inplace = in == out && in_span == out_span;
  for (unsigned p = 0; p < npol; p++)
  {
    const uint64_t r = uint64_t (c) * npol + p;
    if (zap) out[r * out_span + t] = make_float2 (0.f, 0.f);
    else if (!inplace) out[r * out_span + t] = in[r * in_span + t];
  }
}

// Convolution's zero-DM output (Convolution.C:175-193, 789-796) for the
// pipeline: input sample first + t of every (chan, pol), unpacked, into
// out[(c*npol + p)*span + t]
template <int KIND>
__global__ void k_zero_dm (const InputView in, const float* __restrict__ lut, const uint64_t first,
                           const uint64_t n, float2* __restrict__ out, const uint64_t span)
{
  __shared__ float s_lut[256];
  if constexpr (KIND == IN_INT8) load_lut (in, lut, s_lut);
  __syncthreads ();
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const unsigned row = blockIdx.y, c = row / in.npol, p = row % in.npol;
  out[uint64_t (row) * span + t] = fetch<KIND> (in, s_lut, c, p, first + t);
}

// SpectralKurtosis::mask (SpectralKurtosis.C:1465-1566) applied to other
// voltages than the statistics came from (the dedispersed ones, when the
// statistics are of the zero-DM input): block t / M of channel c is zeroed
// in every polarisation where mask[(t / M) * nchan + c] is set.
__global__ void k_sk_apply (const uint8_t* __restrict__ mask, float2* __restrict__ v,
                            const uint64_t span, const uint64_t ndat, const unsigned nchan,
                            const unsigned npol, const unsigned M)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  if (t >= ndat || !__ldg (mask + (t / M) * nchan + c)) return;
  for (unsigned p = 0; p < npol; p++) v[(uint64_t (c) * npol + p) * span + t] = make_float2 (0.f, 0.f);
}

// Detection and Fold::fold of data with zeroed samples (Fold.C:895-930,
// zeroed_samples): every sample is added to its bin, and a hit is counted
// for each channel whose first detected value of the first polarisation is
// non-zero -- into the one hits array shared by all channels.
template <int NOUT>
__global__ void k_zeroed_fold (const float2* __restrict__ v, const uint64_t span,
                               const uint64_t ndat, const unsigned npol, const FoldView fv)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned c = blockIdx.y;
  bool ok = t < ndat;
  if (!__any_sync (FULL, ok)) return;
  float2 p = make_float2 (0.f, 0.f), q = make_float2 (0.f, 0.f);
  if (ok)
  {
    p = v[(uint64_t (c) * npol) * span + t];
    if (npol == 2) q = v[(uint64_t (c) * npol + 1) * span + t];
  }
  float d[4] = {0.f, 0.f, 0.f, 0.f};
  const unsigned bin = fv.cols ? (ok ? __ldg (fv.cols + t) : NO_COLUMN)
                               : warp_fold_bin (fv.segs, fv.nseg, ok, t, fv.nbin);
  if (ok)
  {
    detect_values (fv.state, npol, p, q, d);
    // a zeroed sample adds nothing to the profile and counts no hit
    ok = bin < fv.stride && d[0] != 0.f;
  }
  warp_fold<NOUT> (ok, bin, d, fv.profiles + uint64_t (c) * NOUT * fv.stride, fv.stride, fv.hits);
}

// one thread per sample: the column warp_fold_bin would give it
// A warp takes COLPLAN_GROUPS consecutive groups of 32 samples: one binary
// search for the first sample, then each lane steps forward over the
// segment boundaries from where the previous group's last lane ended.
constexpr int COLPLAN_GROUPS = 32;

__global__ void k_colplan (const FoldSegment* __restrict__ segs, const int nseg,
                           const uint64_t ndat, const unsigned nbin, unsigned* __restrict__ cols)
{
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (uint64_t (blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32) * 32
                      * COLPLAN_GROUPS;
  if (w0 >= ndat) return;             // whole warps
  int s = 0;
  if (lane == 0) s = seg_search (segs, nseg, w0);
  s = __shfl_sync (FULL, s, 0);
  for (int g = 0; g < COLPLAN_GROUPS; g++)
  {
    const uint64_t t = w0 + uint64_t (g) * 32 + lane;
    int sl = s;
    while (sl + 1 < nseg && __ldg (&segs[sl + 1].start) <= t) sl++;
    if (t < ndat)
    {
      const unsigned base = __ldg (&segs[sl].base);
      const unsigned bin = seg_bin (segs, sl, t, nbin);
      cols[t] = (base == FOLD_SKIP || bin >= nbin) ? NO_COLUMN : base + bin;
    }
    s = __shfl_sync (FULL, sl, 31);
  }
}

__global__ void k_binplan (const FoldSegment* __restrict__ segs, const int nseg,
                           const uint64_t ndat, const unsigned nbin, uint32_t* __restrict__ out)
{
  const uint64_t t = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ndat) return;
  out[t] = fold_bin (segs, nseg, t, nbin);
}

// --------------------------------------------------------------------------
// launch helpers
// --------------------------------------------------------------------------

template <int N1, int NPOL, int MODE, int NOUT>
void launch_inv (const ConvShape& sh, dim3 grid, float2* scratch, uint64_t part0,
                 const ConvTables& tb, const FoldView& fv, const VoltView& vv, cudaStream_t st)
{
  if (N1 == 32) grid.x = sh.n2 / 64;        // two threads per column
  k_inv_cols<N1, NPOL, MODE, NOUT><<<grid, 128, 0, st>>> (scratch, sh.n2, sh.nchan, sh.nkeep,
                                                          sh.nfilt_pos, part0, tb.tw4, fv, vv);
}

template <int N2>
void launch_rows (unsigned nrows, float2* scratch, const ConvTables& tb, unsigned n1,
                  const ConvShape& sh, cudaStream_t st)
{
  if (N2 == 8192 && tb.tc_splits)
  {
    launch_rows_mma (nrows, scratch, tb, n1, sh, st);
    return;
  }
  // persistent: as many CTAs as are resident at once
  const unsigned grid = std::min<unsigned> (nrows, rows_ctas_per_sm (N2) * unsigned (tb.nsm));
  k_rows32<N2, true><<<grid, Row32<N2>::T, rows32_smem_bytes<N2> (), st>>> (
      scratch, tb.H, n1, sh.nchan, sh.npol, nrows, nrows / (n1 * sh.nchan));
}

template <int N1>
cudaError_t run_fourstep_n1 (const ConvShape& sh, const ConvTables& tb, const InputView& in,
                             uint64_t part0, unsigned nbatch, float2* scratch, int mode,
                             const FoldView& fv, const VoltView& vv, cudaStream_t st,
                             const KernelClock* clk)
{
  const dim3 gcol (sh.n2 / 128, nbatch, sh.nchan);
  const dim3 gfwd (sh.n2 / fwd_cols_per_block<N1> (), nbatch, sh.nchan);
  if (in.fb_nsub)
  {
    // the 64-channel filterbank inside the column pass
    if (N1 != 8 || in.fb_nsub != 64 || sh.nchan != 64 || in.nchan != 1 || in.npol != 2
        || sh.npol != 2 || tb.apod || (in.kind != IN_INT8 && in.kind != IN_INT16))
      return cudaErrorInvalidValue;
    ClockScope cs (clk, KK_FWD_COLS, st);
    const dim3 g (sh.n2 / FBC_COLS, nbatch);
    if (in.kind == IN_INT8 && in.lut_scale != 0.f)
      k_fwd_cols_fb64<IN_INT8, true><<<g, FBC_THREADS, FBC_SMEM, st>>> (in, tb.lut, sh.nkeep, part0,
                                                                         sh.n2, tb.tw4, scratch);
    else if (in.kind == IN_INT8)
      k_fwd_cols_fb64<IN_INT8, false><<<g, FBC_THREADS, FBC_SMEM, st>>> (in, tb.lut, sh.nkeep, part0,
                                                                          sh.n2, tb.tw4, scratch);
    else
      k_fwd_cols_fb64<IN_INT16, false><<<g, FBC_THREADS, FBC_SMEM, st>>> (in, tb.lut, sh.nkeep,
                                                                           part0, sh.n2, tb.tw4,
                                                                           scratch);
  }
  else
  {
  ClockScope cs (clk, KK_FWD_COLS, st);
  if (in.kind == IN_INT8)
    k_fwd_cols<N1, IN_INT8><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.nkeep, part0, sh.n2, tb.tw4,
                                                   scratch, tb.apod);
  else if (in.kind == IN_INT16)
    k_fwd_cols<N1, IN_INT16><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.nkeep, part0, sh.n2, tb.tw4,
                                                    scratch, tb.apod);
  else
    k_fwd_cols<N1, IN_FLOAT><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.nkeep, part0, sh.n2, tb.tw4,
                                                    scratch, tb.apod);
  }
  const unsigned nrows = N1 * nbatch * sh.nchan * sh.npol;
  {
  ClockScope cs (clk, KK_ROWS, st);
  if (sh.n2 == 8192)
    launch_rows<8192> (nrows, scratch, tb, N1, sh, st);
  else if (sh.n2 == 4096)
    launch_rows<4096> (nrows, scratch, tb, N1, sh, st);
  else
    return cudaErrorInvalidValue;
  }
  ClockScope cs (clk, KK_INV_COLS, st);
  if (sh.npol == 2)
  {
    if (mode == OUT_VOLTAGE)
      launch_inv<N1, 2, OUT_VOLTAGE, 1> (sh, gcol, scratch, part0, tb, fv, vv, st);
    else if (fv.nout == 1)
      launch_inv<N1, 2, OUT_FOLD, 1> (sh, gcol, scratch, part0, tb, fv, vv, st);
    else if (fv.nout == 2)
      launch_inv<N1, 2, OUT_FOLD, 2> (sh, gcol, scratch, part0, tb, fv, vv, st);
    else
      launch_inv<N1, 2, OUT_FOLD, 4> (sh, gcol, scratch, part0, tb, fv, vv, st);
  }
  else
  {
    if (mode == OUT_VOLTAGE)
      launch_inv<N1, 1, OUT_VOLTAGE, 1> (sh, gcol, scratch, part0, tb, fv, vv, st);
    else
      launch_inv<N1, 1, OUT_FOLD, 1> (sh, gcol, scratch, part0, tb, fv, vv, st);
  }
  return cudaGetLastError ();
}

// The fused kernel's shared-memory opt-in (sized for two polarisations), once
// per device and instantiation; later calls only test a bit, so that calls
// made inside a stream capture set nothing up.
template <int N, int KIND, int MODE, int NOUT>
cudaError_t fused_setup ()
{
  static std::atomic<unsigned> done {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice (&dev);
  if (e != cudaSuccess) return e;
  const unsigned bit = dev < 32 ? 1u << dev : 0u;    // devices past 32: set every time
  if (bit && (done.load () & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute (k_fused<N, stockham_threads (N), KIND, MODE, NOUT>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            int (2 * spad_size (N) * sizeof (float2)));
  if (e == cudaSuccess) done.fetch_or (bit);
  return e;
}

template <int N, int KIND, int MODE, int NOUT>
cudaError_t run_fused_t (const ConvShape& sh, const ConvTables& tb, const InputView& in,
                         uint64_t part0, unsigned nbatch, const FoldView& fv,
                         const VoltView& vv, cudaStream_t st, const KernelClock* clk)
{
  constexpr int T = stockham_threads (N);
  const size_t smem = size_t (in.npol) * spad_size (N) * sizeof (float2);
  auto kern = k_fused<N, T, KIND, MODE, NOUT>;
  cudaError_t err = fused_setup<N, KIND, MODE, NOUT> ();
  if (err != cudaSuccess) return err;
  ClockScope cs (clk, KK_FUSED, st);
  kern<<<dim3 (nbatch, sh.nchan), T, smem, st>>> (in, tb.lut, tb.tw2, tb.H, sh.nkeep,
                                                  sh.nfilt_pos, part0, fv, vv, tb.apod);
  return cudaGetLastError ();
}

template <int N, int KIND>
cudaError_t run_fused_k (const ConvShape& sh, const ConvTables& tb, const InputView& in,
                         uint64_t part0, unsigned nbatch, int mode, const FoldView& fv,
                         const VoltView& vv, cudaStream_t st, const KernelClock* clk)
{
  if (mode == OUT_VOLTAGE)
    return run_fused_t<N, KIND, OUT_VOLTAGE, 1> (sh, tb, in, part0, nbatch, fv, vv, st, clk);
  if (fv.nout == 1)
    return run_fused_t<N, KIND, OUT_FOLD, 1> (sh, tb, in, part0, nbatch, fv, vv, st, clk);
  if (fv.nout == 2)
    return run_fused_t<N, KIND, OUT_FOLD, 2> (sh, tb, in, part0, nbatch, fv, vv, st, clk);
  return run_fused_t<N, KIND, OUT_FOLD, 4> (sh, tb, in, part0, nbatch, fv, vv, st, clk);
}

template <int N>
cudaError_t run_fused (const ConvShape& sh, const ConvTables& tb, const InputView& in,
                       uint64_t part0, unsigned nbatch, int mode, const FoldView& fv,
                       const VoltView& vv, cudaStream_t st, const KernelClock* clk)
{
  if (in.kind == IN_INT8)
    return run_fused_k<N, IN_INT8> (sh, tb, in, part0, nbatch, mode, fv, vv, st, clk);
  if (in.kind == IN_INT16)
    return run_fused_k<N, IN_INT16> (sh, tb, in, part0, nbatch, mode, fv, vv, st, clk);
  return run_fused_k<N, IN_FLOAT> (sh, tb, in, part0, nbatch, mode, fv, vv, st, clk);
}

template <int LIN, int KIND>
void launch_ifb_stitch (const IfbShape& sh, const IfbTables& tb, const InputView& in,
                        uint64_t part0, unsigned nbatch, float2* scratch, cudaStream_t st)
{
  constexpr int F = IFB_THREADS / stockham_threads (LIN);
  const size_t smem = (size_t (F) * (spad_size (LIN) + 4) + pass_tables_size (LIN)) * sizeof (float2);
  auto kern = k_ifb_stitch<LIN, KIND>;
  cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
  const unsigned cg = F / sh.npol;
  kern<<<dim3 ((sh.nin + cg - 1) / cg, nbatch), IFB_THREADS, smem, st>>> (in, sh, tb, part0,
                                                                         scratch);
}

template <int LIN>
void launch_ifb_stitch_k (const IfbShape& sh, const IfbTables& tb, const InputView& in,
                          uint64_t part0, unsigned nbatch, float2* scratch, cudaStream_t st)
{
  if (in.kind == IN_INT8)
    launch_ifb_stitch<LIN, IN_INT8> (sh, tb, in, part0, nbatch, scratch, st);
  else if (in.kind == IN_INT16)
    launch_ifb_stitch<LIN, IN_INT16> (sh, tb, in, part0, nbatch, scratch, st);
  else
    launch_ifb_stitch<LIN, IN_FLOAT> (sh, tb, in, part0, nbatch, scratch, st);
}

template <int N1>
void launch_ifb_cols (const IfbShape& sh, const IfbTables& tb, uint64_t part0, unsigned nbatch,
                      const float2* scratch, const VoltView& vv, cudaStream_t st)
{
  k_ifb_cols<N1><<<dim3 (sh.n2 / 128, nbatch, sh.nout), 128, 0, st>>> (scratch, sh, tb.tw4, part0,
                                                                       vv);
}

template <int N2>
void launch_rows_inv (unsigned nrows, float2* scratch, const IfbTables& tb, unsigned n1,
                      unsigned npol, cudaStream_t st)
{
  const unsigned grid = std::min<unsigned> (nrows, rows_ctas_per_sm (N2) * unsigned (tb.nsm));
  k_rows32<N2, false><<<grid, Row32<N2>::T, rows32_smem_bytes<N2> (), st>>> (
      scratch, nullptr, n1, 1, npol, nrows, nrows / n1);
}

template <int N2, bool CONV>
cudaError_t set_rows_smem ()
{
  return cudaFuncSetAttribute (k_rows32<N2, CONV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int (rows32_smem_bytes<N2> ()));
}

} // namespace

uint64_t kernel_launches () { return g_launches.load (); }

unsigned rows_ctas_per_sm (unsigned n2)
{
  return n2 == 8192 ? rows32_ctas_per_sm<8192> () : rows32_ctas_per_sm<4096> ();
}

unsigned pass_tables_count (unsigned n)
{
  switch (n)
  {
    case 64: return pass_tables_size (64);
    case 128: return pass_tables_size (128);
    case 256: return pass_tables_size (256);
    case 512: return pass_tables_size (512);
    case 1024: return pass_tables_size (1024);
    case 2048: return pass_tables_size (2048);
    case 4096: return pass_tables_size (4096);
    case 8192: return pass_tables_size (8192);
    default: return 0;
  }
}

// w_{Ns R}^{a r} rounded once from double precision, [r-1][a] per pass
void make_pass_tables (unsigned n, float2* out, unsigned capacity)
{
  const int N = int (n);
  for (int p = 1; p < stockham_npass (N); p++)
  {
    const int Ns = stockham_ns (N, p), R = stockham_radix (N, p);
    const int off = pass_table_offset (N, p);
    for (int r = 1; r < R; r++)
      for (int a = 0; a < Ns; a++)
      {
        const unsigned idx = unsigned (off + (r - 1) * Ns + a);
        if (idx >= capacity) return;
        const double ang = -2.0 * 3.14159265358979323846 * double (a) * r / (double (Ns) * R);
        out[idx] = make_float2 (float (cos (ang)), float (sin (ang)));
      }
  }
}

// The four-step kernels' shared-memory opt-in, once per device (the current
// one); later calls only test a bit.
cudaError_t convolution_kernel_setup ()
{
  static std::atomic<unsigned> attr_done {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice (&dev);
  if (e != cudaSuccess) return e;
  const unsigned bit = dev < 32 ? 1u << dev : 0u;    // devices past 32: set every time
  if (bit && (attr_done.load () & bit)) return cudaSuccess;
  e = set_rows_smem<8192, true> ();
  if (e == cudaSuccess) e = set_rows_smem<4096, true> ();
  // the single-kernel transforms of the float voltage path (the no-alloc
  // entry point's)
  if (e == cudaSuccess) e = fused_setup<4096, IN_FLOAT, OUT_VOLTAGE, 1> ();
  if (e == cudaSuccess) e = fused_setup<8192, IN_FLOAT, OUT_VOLTAGE, 1> ();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute (k_fwd_cols_fb64<IN_INT8, false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (FBC_SMEM));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute (k_fwd_cols_fb64<IN_INT8, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (FBC_SMEM));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute (k_fwd_cols_fb64<IN_INT16, false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (FBC_SMEM));
  if (e == cudaSuccess) attr_done.fetch_or (bit);
  return e;
}

cudaError_t launch_convolution (const ConvShape& sh, const ConvTables& tb, const InputView& in,
                                uint64_t part0, unsigned nbatch, float2* scratch, int mode,
                                const FoldView& fv, const VoltView& vv, cudaStream_t st,
                                const KernelClock* clk)
{
  if (nbatch == 0) return cudaSuccess;
  if (sh.n1 == 1)
  {
    switch (sh.nfft)
    {
      case 4096: return run_fused<4096> (sh, tb, in, part0, nbatch, mode, fv, vv, st, clk);
      case 8192: return run_fused<8192> (sh, tb, in, part0, nbatch, mode, fv, vv, st, clk);
      default: return cudaErrorInvalidValue;
    }
  }
  {
    const cudaError_t e = convolution_kernel_setup ();
    if (e != cudaSuccess) return e;
  }
  switch (sh.n1)
  {
    case 2: return run_fourstep_n1<2> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 4: return run_fourstep_n1<4> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 8: return run_fourstep_n1<8> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 16: return run_fourstep_n1<16> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 32: return run_fourstep_n1<32> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    default: return cudaErrorInvalidValue;
  }
}

namespace {

template <int SEG>
cudaError_t launch_rows_during (unsigned nrows, float2* scratch, const DuringShape& sh,
                                const DuringTables& tb, cudaStream_t st)
{
  constexpr size_t smem = during_rows_smem<SEG> ();
  static_assert (smem <= 227u * 1024u, "row kernel shared memory");
  cudaError_t e = cudaFuncSetAttribute (k_rows_during<SEG>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
  if (e != cudaSuccess) return e;
  // persistent: two CTAs per SM
  const unsigned grid = std::min<unsigned> (nrows, 2 * unsigned (tb.nsm));
  k_rows_during<SEG><<<grid, Row32<DUR_N2>::T, smem, st>>> (
      scratch, tb.ptab_seg, tb.H, sh.n1, sh.nsub, sh.npol, sh.nchan_in, nrows,
      nrows / (sh.n1 * sh.nchan_in));
  return cudaSuccess;
}

template <int N1, int NPOL, int MODE, int NOUT>
void launch_inv_during (const DuringShape& sh, dim3 grid, const float2* scratch, uint64_t part0,
                        const DuringTables& tb, const FoldView& fv, const VoltView& vv,
                        cudaStream_t st)
{
  k_inv_cols_during<N1, NPOL, MODE, NOUT><<<grid, 128, 0, st>>> (scratch, sh, part0, tb.twd, fv,
                                                                 vv);
}

template <int N1, int NPOL>
void launch_inv_during_m (const DuringShape& sh, dim3 grid, const float2* scratch,
                          uint64_t part0, const DuringTables& tb, int mode, const FoldView& fv,
                          const VoltView& vv, cudaStream_t st)
{
  if (mode == OUT_VOLTAGE)
    launch_inv_during<N1, NPOL, OUT_VOLTAGE, 1> (sh, grid, scratch, part0, tb, fv, vv, st);
  else if (NPOL == 1 || fv.nout == 1)
    launch_inv_during<N1, NPOL, OUT_FOLD, 1> (sh, grid, scratch, part0, tb, fv, vv, st);
  else if (fv.nout == 2)
    launch_inv_during<N1, NPOL, OUT_FOLD, 2> (sh, grid, scratch, part0, tb, fv, vv, st);
  else
    launch_inv_during<N1, NPOL, OUT_FOLD, 4> (sh, grid, scratch, part0, tb, fv, vv, st);
}

template <int N1>
cudaError_t run_during_n1 (const DuringShape& sh, const DuringTables& tb, const InputView& in,
                           uint64_t part0, unsigned nbatch, float2* scratch, int mode,
                           const FoldView& fv, const VoltView& vv, cudaStream_t st,
                           const KernelClock* clk)
{
  const dim3 gcol (sh.n2 / 128, nbatch, sh.nchan_in);
  const dim3 gfwd (sh.n2 / fwd_cols_per_block<N1> (), nbatch, sh.nchan_in);
  {
    ClockScope cs (clk, KK_FWD_COLS, st);
    if (in.kind == IN_INT8)
      k_fwd_cols<N1, IN_INT8><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.in_step, part0, sh.n2, tb.tw4,
                                                     scratch, tb.apod);
    else if (in.kind == IN_INT16)
      k_fwd_cols<N1, IN_INT16><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.in_step, part0, sh.n2,
                                                      tb.tw4, scratch, tb.apod);
    else
      k_fwd_cols<N1, IN_FLOAT><<<gfwd, 128, 0, st>>> (in, tb.lut, sh.in_step, part0, sh.n2,
                                                      tb.tw4, scratch, tb.apod);
  }
  const unsigned nrows = N1 * nbatch * sh.nchan_in * sh.npol;
  cudaError_t e = cudaSuccess;
  {
    ClockScope cs (clk, KK_ROWS, st);
    switch (sh.seg)
    {
      case 64: e = launch_rows_during<64> (nrows, scratch, sh, tb, st); break;
      case 128: e = launch_rows_during<128> (nrows, scratch, sh, tb, st); break;
      case 256: e = launch_rows_during<256> (nrows, scratch, sh, tb, st); break;
      case 512: e = launch_rows_during<512> (nrows, scratch, sh, tb, st); break;
      case 1024: e = launch_rows_during<1024> (nrows, scratch, sh, tb, st); break;
      case 2048: e = launch_rows_during<2048> (nrows, scratch, sh, tb, st); break;
      case 4096: e = launch_rows_during<4096> (nrows, scratch, sh, tb, st); break;
      default: return cudaErrorInvalidValue;
    }
  }
  if (e != cudaSuccess) return e;
  ClockScope cs (clk, KK_INV_COLS, st);
  if (sh.npol == 2)
    launch_inv_during_m<N1, 2> (sh, gcol, scratch, part0, tb, mode, fv, vv, st);
  else
    launch_inv_during_m<N1, 1> (sh, gcol, scratch, part0, tb, mode, fv, vv, st);
  return cudaGetLastError ();
}

template <int N1, int NPOL>
void launch_inv_during_big (const DuringShape& sh, dim3 grid, const float2* scratch,
                            uint64_t part0, const DuringTables& tb, int mode, const FoldView& fv,
                            const VoltView& vv, cudaStream_t st)
{
  constexpr size_t smem = colbig_inv_smem<N1, NPOL> ();
  constexpr int T = inv_colw<N1> () * stockham_threads (N1);
  grid.x = sh.n2 / inv_colw<N1> ();
  if (mode == OUT_VOLTAGE)
  {
    auto k = k_inv_cols_during_big<N1, NPOL, OUT_VOLTAGE, 1>;
    cudaFuncSetAttribute (k, cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
    k<<<grid, T, smem, st>>> (scratch, sh, part0, tb.twd, tb.ptab_col, fv, vv);
    return;
  }
  auto k = NPOL == 1 || fv.nout == 1 ? k_inv_cols_during_big<N1, NPOL, OUT_FOLD, 1>
         : fv.nout == 2 ? k_inv_cols_during_big<N1, NPOL, OUT_FOLD, 2>
                        : k_inv_cols_during_big<N1, NPOL, OUT_FOLD, 4>;
  cudaFuncSetAttribute (k, cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
  k<<<grid, T, smem, st>>> (scratch, sh, part0, tb.twd, tb.ptab_col, fv, vv);
}

template <int N1>
cudaError_t run_during_big (const DuringShape& sh, const DuringTables& tb, const InputView& in,
                            uint64_t part0, unsigned nbatch, float2* scratch, int mode,
                            const FoldView& fv, const VoltView& vv, cudaStream_t st,
                            const KernelClock* clk)
{
  static_assert (colbig_inv_smem<N1, 2> () <= 227u * 1024u, "column kernel shared memory");
  const dim3 gcol (sh.n2 / COLW, nbatch, sh.nchan_in);
  {
    ClockScope cs (clk, KK_FWD_COLS, st);
    constexpr size_t smem = colbig_smem<N1, 1> ();
    if (in.kind == IN_INT8)
    {
      cudaFuncSetAttribute (k_fwd_cols_big<N1, IN_INT8>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
      k_fwd_cols_big<N1, IN_INT8><<<gcol, N1, smem, st>>> (in, tb.lut, sh.in_step, part0, sh.n2,
                                                          tb.tw4, tb.ptab_col, scratch, tb.apod);
    }
    else if (in.kind == IN_INT16)
    {
      cudaFuncSetAttribute (k_fwd_cols_big<N1, IN_INT16>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
      k_fwd_cols_big<N1, IN_INT16><<<gcol, N1, smem, st>>> (in, tb.lut, sh.in_step, part0, sh.n2,
                                                           tb.tw4, tb.ptab_col, scratch, tb.apod);
    }
    else
    {
      cudaFuncSetAttribute (k_fwd_cols_big<N1, IN_FLOAT>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
      k_fwd_cols_big<N1, IN_FLOAT><<<gcol, N1, smem, st>>> (in, tb.lut, sh.in_step, part0, sh.n2,
                                                           tb.tw4, tb.ptab_col, scratch, tb.apod);
    }
  }
  const unsigned nrows = N1 * nbatch * sh.nchan_in * sh.npol;
  cudaError_t e = cudaSuccess;
  {
    ClockScope cs (clk, KK_ROWS, st);
    switch (sh.seg)
    {
      case 64: e = launch_rows_during<64> (nrows, scratch, sh, tb, st); break;
      case 128: e = launch_rows_during<128> (nrows, scratch, sh, tb, st); break;
      case 256: e = launch_rows_during<256> (nrows, scratch, sh, tb, st); break;
      case 512: e = launch_rows_during<512> (nrows, scratch, sh, tb, st); break;
      case 1024: e = launch_rows_during<1024> (nrows, scratch, sh, tb, st); break;
      case 2048: e = launch_rows_during<2048> (nrows, scratch, sh, tb, st); break;
      case 4096: e = launch_rows_during<4096> (nrows, scratch, sh, tb, st); break;
      default: return cudaErrorInvalidValue;
    }
  }
  if (e != cudaSuccess) return e;
  ClockScope cs (clk, KK_INV_COLS, st);
  if (sh.npol == 2)
    launch_inv_during_big<N1, 2> (sh, gcol, scratch, part0, tb, mode, fv, vv, st);
  else
    launch_inv_during_big<N1, 1> (sh, gcol, scratch, part0, tb, mode, fv, vv, st);
  return cudaGetLastError ();
}

} // namespace

namespace {
__global__ void k_window_response (float2* __restrict__ out, const float2* __restrict__ in,
                                   const float* __restrict__ w, const uint64_t n,
                                   const unsigned n1, const unsigned seg)
{
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const uint64_t fr = uint64_t (n1) * seg;
  const unsigned r = unsigned (idx % fr);
  const unsigned f = r / seg + n1 * (r % seg);
  const float2 h = in[idx];
  const float x = __ldg (w + f);
  out[idx] = make_float2 (__fmul_rn (h.x, x), __fmul_rn (h.y, x));
}
} // namespace

cudaError_t launch_window_response (float2* out, const float2* in, const float* window,
                                    unsigned nchan, unsigned n1, unsigned seg, cudaStream_t st)
{
  const uint64_t n = uint64_t (nchan) * n1 * seg;
  g_launches++;
  k_window_response<<<unsigned ((n + 255) / 256), 256, 0, st>>> (out, in, window, n, n1, seg);
  return cudaGetLastError ();
}

bool during_supported (unsigned nsub, unsigned freq_res)
{
  if (nsub < 2 || nsub > 128 || (nsub & (nsub - 1))) return false;
  const uint64_t n = uint64_t (nsub) * freq_res;
  return freq_res && (freq_res & (freq_res - 1)) == 0 && n >= 2 * DUR_N2 && n <= 512 * DUR_N2;
}

cudaError_t launch_filterbank_during (const DuringShape& sh, const DuringTables& tb,
                                      const InputView& in, uint64_t part0, unsigned nbatch,
                                      float2* scratch, int mode, const FoldView& fv,
                                      const VoltView& vv, cudaStream_t st,
                                      const KernelClock* clk)
{
  if (nbatch == 0) return cudaSuccess;
  if (!during_supported (sh.nsub, sh.freq_res) || sh.n2 != unsigned (DUR_N2)
      || uint64_t (sh.n1) * sh.n2 != uint64_t (sh.nsub) * sh.freq_res || sh.seg * sh.nsub != sh.n2
      || sh.npol < 1 || sh.npol > 2 || in.fb_nsub)
    return cudaErrorInvalidValue;
  switch (sh.n1)
  {
    case 2: return run_during_n1<2> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 4: return run_during_n1<4> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 8: return run_during_n1<8> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 16: return run_during_n1<16> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 32: return run_during_n1<32> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 64: return run_during_big<64> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 128:
      return run_during_big<128> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 256:
      return run_during_big<256> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    case 512:
      return run_during_big<512> (sh, tb, in, part0, nbatch, scratch, mode, fv, vv, st, clk);
    default: return cudaErrorInvalidValue;
  }
}

bool ifb_supported_lin (unsigned lin)
{
  return lin == 64 || lin == 128 || lin == 256 || lin == 512 || lin == 1024 || lin == 2048 ||
         lin == 4096;
}

cudaError_t launch_inverse_filterbank (const IfbShape& sh, const IfbTables& tb,
                                       const InputView& in, uint64_t part0, unsigned nbatch,
                                       float2* scratch, const VoltView& vv, cudaStream_t st,
                                       const KernelClock* clk)
{
  if (nbatch == 0) return cudaSuccess;
  if (sh.n2 != 8192 && sh.n2 != 4096) return cudaErrorInvalidValue;
  static unsigned attr_done = 0;
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 32 && !(attr_done & (1u << dev)))
  {
    cudaError_t e = set_rows_smem<8192, false> ();
    if (e == cudaSuccess) e = set_rows_smem<4096, false> ();
    if (e != cudaSuccess) return e;
    attr_done |= 1u << dev;
  }
  {
    ClockScope cs (clk, KK_FWD_COLS, st);
    switch (sh.lin)
    {
      case 64: launch_ifb_stitch_k<64> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 128: launch_ifb_stitch_k<128> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 256: launch_ifb_stitch_k<256> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 512: launch_ifb_stitch_k<512> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 1024: launch_ifb_stitch_k<1024> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 2048: launch_ifb_stitch_k<2048> (sh, tb, in, part0, nbatch, scratch, st); break;
      case 4096: launch_ifb_stitch_k<4096> (sh, tb, in, part0, nbatch, scratch, st); break;
      default: return cudaErrorInvalidValue;
    }
  }
  const unsigned nrows = sh.n1 * nbatch * sh.nout * sh.npol;
  {
    ClockScope cs (clk, KK_ROWS, st);
    if (sh.n2 == 8192)
      launch_rows_inv<8192> (nrows, scratch, tb, sh.n1, sh.npol, st);
    else
      launch_rows_inv<4096> (nrows, scratch, tb, sh.n1, sh.npol, st);
  }
  ClockScope cs (clk, KK_INV_COLS, st);
  switch (sh.n1)
  {
    case 2: launch_ifb_cols<2> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 3: launch_ifb_cols<3> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 4: launch_ifb_cols<4> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 6: launch_ifb_cols<6> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 8: launch_ifb_cols<8> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 12: launch_ifb_cols<12> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 16: launch_ifb_cols<16> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 24: launch_ifb_cols<24> (sh, tb, part0, nbatch, scratch, vv, st); break;
    case 32: launch_ifb_cols<32> (sh, tb, part0, nbatch, scratch, vv, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError ();
}

cudaError_t launch_build_chirp (float2* H, const double* d_chan_freq, const double* d_coeff,
                                const double* d_frac_us, unsigned nchan, unsigned nfft,
                                unsigned n1, unsigned n2, double binwidth, double half_chanwidth,
                                int swap_halves, int chirp_mode, float scale, cudaStream_t st)
{
  const dim3 grid ((nfft + 255) / 256, nchan);
  g_launches++;
  k_build_chirp<<<grid, 256, 0, st>>> (H, d_chan_freq, d_coeff, d_frac_us, nfft, n1, n2,
                                        binwidth, half_chanwidth, swap_halves, chirp_mode, scale);
  return cudaGetLastError ();
}

cudaError_t launch_permute_response (float2* H, const float2* src, unsigned nchan, unsigned n1,
                                     unsigned n2, cudaStream_t st)
{
  const uint64_t N = uint64_t (n1) * n2;
  g_launches++;
  k_permute<<<dim3 (unsigned ((N + 255) / 256), nchan), 256, 0, st>>> (H, src, n1, n2, 0);
  return cudaGetLastError ();
}

cudaError_t launch_unpermute_response (float2* dst, const float2* H, unsigned nchan, unsigned n1,
                                       unsigned n2, cudaStream_t st)
{
  const uint64_t N = uint64_t (n1) * n2;
  g_launches++;
  k_permute<<<dim3 (unsigned ((N + 255) / 256), nchan), 256, 0, st>>> (dst, H, n1, n2, 1);
  return cudaGetLastError ();
}

namespace {
template <int NSUB>
cudaError_t run_filterbank (const InputView& in, const float* d_lut, uint64_t nblk, float scale,
                            float2* out, uint64_t out_span, cudaStream_t st,
                            const KernelClock* clk)
{
  const dim3 grid (unsigned ((nblk + 127) / 128), in.npol, in.nchan);
  ClockScope cs (clk, KK_FILTERBANK, st);
  if (in.kind == IN_INT8)
    k_filterbank<NSUB, IN_INT8><<<grid, 128, 0, st>>> (in, d_lut, nblk, scale, out, out_span);
  else if (in.kind == IN_INT16)
    k_filterbank<NSUB, IN_INT16><<<grid, 128, 0, st>>> (in, d_lut, nblk, scale, out, out_span);
  else
    k_filterbank<NSUB, IN_FLOAT><<<grid, 128, 0, st>>> (in, d_lut, nblk, scale, out, out_span);
  return cudaGetLastError ();
}
template <int NSUB>
cudaError_t run_filterbank_smem (const InputView& in, const float* d_lut, const float2* ptab,
                                 uint64_t nblk, float scale, float2* out, uint64_t out_span,
                                 cudaStream_t st, const KernelClock* clk)
{
  constexpr int F = FB_THREADS / stockham_threads (NSUB);
  const unsigned bpc = F / in.npol;
  const size_t smem = (size_t (F) * (spad_size (NSUB) + 1) + pass_tables_size (NSUB)) *
                      sizeof (float2);
  const dim3 grid (unsigned ((nblk + bpc - 1) / bpc), in.nchan);
  ClockScope cs (clk, KK_FILTERBANK, st);
  cudaError_t e;
  if (in.kind == IN_INT8)
  {
    e = cudaFuncSetAttribute (k_filterbank_smem<NSUB, IN_INT8>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
    if (e == cudaSuccess)
      k_filterbank_smem<NSUB, IN_INT8><<<grid, FB_THREADS, smem, st>>> (in, d_lut, ptab, nblk,
                                                                        scale, out, out_span);
  }
  else if (in.kind == IN_INT16)
  {
    e = cudaFuncSetAttribute (k_filterbank_smem<NSUB, IN_INT16>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
    if (e == cudaSuccess)
      k_filterbank_smem<NSUB, IN_INT16><<<grid, FB_THREADS, smem, st>>> (in, d_lut, ptab, nblk,
                                                                         scale, out, out_span);
  }
  else
  {
    e = cudaFuncSetAttribute (k_filterbank_smem<NSUB, IN_FLOAT>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, int (smem));
    if (e == cudaSuccess)
      k_filterbank_smem<NSUB, IN_FLOAT><<<grid, FB_THREADS, smem, st>>> (in, d_lut, ptab, nblk,
                                                                         scale, out, out_span);
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError ();
}
} // namespace

cudaError_t launch_filterbank (const InputView& in, const float* d_lut, unsigned nsub,
                               uint64_t nblk, float scale, float2* out, uint64_t out_span,
                               cudaStream_t st, const KernelClock* clk, const float2* ptab)
{
  if (nblk == 0) return cudaSuccess;
  // up to 64 channels the one-thread-per-block register transform is faster
  if (nsub >= 128)
  {
    if (!ptab) return cudaErrorInvalidValue;
    switch (nsub)
    {
      case 128: return run_filterbank_smem<128> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      case 256: return run_filterbank_smem<256> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      case 512: return run_filterbank_smem<512> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      case 1024: return run_filterbank_smem<1024> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      case 2048: return run_filterbank_smem<2048> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      case 4096: return run_filterbank_smem<4096> (in, d_lut, ptab, nblk, scale, out, out_span, st, clk);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (nsub)
  {
    case 4: return run_filterbank<4> (in, d_lut, nblk, scale, out, out_span, st, clk);
    case 8: return run_filterbank<8> (in, d_lut, nblk, scale, out, out_span, st, clk);
    case 16: return run_filterbank<16> (in, d_lut, nblk, scale, out, out_span, st, clk);
    case 32: return run_filterbank<32> (in, d_lut, nblk, scale, out, out_span, st, clk);
    case 64: return run_filterbank<64> (in, d_lut, nblk, scale, out, out_span, st, clk);
    default: return cudaErrorInvalidValue;
  }
}

size_t sk_smem_bytes (unsigned npol, unsigned M, unsigned units)
{
  return size_t (units) * npol * sk_column (M) * sizeof (float);
}

cudaError_t launch_sk (const float2* in, uint64_t in_span, float2* out, uint64_t out_span,
                       uint64_t npart, unsigned nchan, unsigned npol, unsigned M,
                       int zero_is_valid, unsigned Nd, float lower, float upper, float* sums,
                       unsigned* counts, uint8_t* mask, unsigned long long* nzap, cudaStream_t st)
{
  if (npart == 0) return cudaSuccess;
  // two blocks per CTA while they fit in a modest footprint, else one
  const unsigned units = sk_smem_bytes (npol, M, 2) <= (48u << 10) ? 2 : 1;
  const size_t smem = sk_smem_bytes (npol, M, units);
  if (smem > SK_SMEM_MAX) return cudaErrorInvalidValue;
  const uint64_t nblk = (npart + units - 1) / units;
  if (nblk > 0x7fffffffull || nchan > 65535) return cudaErrorInvalidValue;
  auto kern = units == 2 ? k_sk<2> : k_sk<1>;
  cudaError_t e = cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int (smem));
  if (e != cudaSuccess) return e;
  g_launches++;
  kern<<<dim3 (unsigned (nblk), nchan), SK_THREADS, smem, st>>> (
      in, in_span, out, out_span, npart, nchan, npol, M, zero_is_valid, Nd, lower, upper, sums,
      counts, mask, nzap);
  return cudaGetLastError ();
}

cudaError_t launch_unpack8 (const uint8_t* in, uint64_t ndat, unsigned nchan, unsigned npol,
                            unsigned ndim, const float* d_lut, float* out, uint64_t span,
                            cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_unpack8<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (
      in, ndat, nchan, npol, ndim, d_lut, out, span);
  return cudaGetLastError ();
}

cudaError_t launch_unpack16 (const int16_t* in, uint64_t ndat, unsigned nchan, unsigned npol,
                             unsigned ndim, int offset_binary, float* out, uint64_t span,
                             cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_unpack16<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (
      in, ndat, nchan, npol, ndim, offset_binary, out, span);
  return cudaGetLastError ();
}

cudaError_t launch_detect (const float2* in, uint64_t in_span, uint64_t ndat, unsigned nchan,
                           int state, float* out, uint64_t out_span, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_detect<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (in, in_span, ndat,
                                                                          state, out, out_span);
  return cudaGetLastError ();
}

cudaError_t launch_fold (const float* in, uint64_t in_span, uint64_t ndat, unsigned nchan,
                         unsigned npol, const FoldView& fv, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_fold<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (in, in_span, ndat, npol,
                                                                        fv);
  return cudaGetLastError ();
}

cudaError_t launch_colplan (const FoldSegment* segs, int nseg, uint64_t ndat, unsigned nbin,
                            unsigned* cols, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  const uint64_t per_block = uint64_t (256) * COLPLAN_GROUPS;
  k_colplan<<<unsigned ((ndat + per_block - 1) / per_block), 256, 0, st>>> (segs, nseg, ndat,
                                                                           nbin, cols);
  return cudaGetLastError ();
}

cudaError_t launch_delay_fold (const float2* v, uint64_t span, const int* applied, uint64_t ndat,
                               unsigned nchan, unsigned npol, const FoldView& fv, cudaStream_t st,
                               const KernelClock* clk)
{
  if (ndat == 0) return cudaSuccess;
  const dim3 grid (unsigned ((ndat + 255) / 256), nchan);
  ClockScope cs (clk, KK_INV_COLS, st);
  if (fv.nout == 1)
    k_delay_fold<1><<<grid, 256, 0, st>>> (v, span, applied, ndat, npol, fv);
  else if (fv.nout == 2)
    k_delay_fold<2><<<grid, 256, 0, st>>> (v, span, applied, ndat, npol, fv);
  else
    k_delay_fold<4><<<grid, 256, 0, st>>> (v, span, applied, ndat, npol, fv);
  return cudaGetLastError ();
}

cudaError_t launch_sk_sums_strided (const float2* in, uint64_t span, uint64_t nblk,
                                   uint64_t stride, unsigned nchan, unsigned npol, unsigned M,
                                   int zero_is_valid, float* sums, unsigned* counts,
                                   cudaStream_t st)
{
  const uint64_t total = nblk * nchan * npol * 2;
  if (total == 0) return cudaSuccess;
  g_launches++;
  k_sk_sums_strided<<<unsigned ((total + 127) / 128), 128, 0, st>>> (
      in, span, nblk, stride, nchan, npol, M, zero_is_valid, sums, counts);
  return cudaGetLastError ();
}

cudaError_t launch_sk_tscrunch (const float* sums, const unsigned* counts, uint64_t npart,
                                unsigned nchan, unsigned npol, unsigned nsum, unsigned offset,
                                float* osums, unsigned* ocounts, cudaStream_t st)
{
  const uint64_t total = npart * nchan * npol * 2;
  if (total == 0) return cudaSuccess;
  g_launches++;
  k_sk_tscrunch<<<unsigned ((total + 255) / 256), 256, 0, st>>> (sums, counts, npart, nchan, npol,
                                                                 nsum, offset, osums, ocounts);
  return cudaGetLastError ();
}

cudaError_t launch_sk_detect_skfb (const float* sums, const unsigned* counts, uint64_t npart,
                                   unsigned nchan, unsigned npol, unsigned Nd,
                                   const unsigned* lim_count, const float2* lim, unsigned nlim,
                                   unsigned nflag, unsigned flag_step, unsigned flag_offset,
                                   uint8_t* mask, unsigned long long* nzap, cudaStream_t st)
{
  const uint64_t total = npart * nchan;
  if (total == 0) return cudaSuccess;
  g_launches++;
  k_sk_detect_skfb<<<unsigned ((total + 255) / 256), 256, 0, st>>> (
      sums, counts, npart, nchan, npol, Nd, lim_count, lim, nlim, nflag, flag_step, flag_offset,
      mask, nzap);
  return cudaGetLastError ();
}

cudaError_t launch_sk_mask_overlap (const uint8_t* mask, const float2* in, uint64_t in_span,
                                    float2* out, uint64_t out_span, uint64_t ndat_out,
                                    unsigned nchan, unsigned npol, unsigned offset,
                                    uint64_t npart, uint64_t nskip, uint64_t idat_start,
                                    cudaStream_t st)
{
  if (ndat_out == 0 || npart == 0) return cudaSuccess;
  g_launches++;
  k_sk_mask_overlap<<<dim3 (unsigned ((ndat_out + 255) / 256), nchan), 256, 0, st>>> (
      mask, in, in_span, out, out_span, ndat_out, nchan, npol, offset, npart, nskip, idat_start);
  return cudaGetLastError ();
}

cudaError_t launch_sk_detect (const float* sums, const unsigned* counts, uint64_t npart,
                              unsigned nchan, unsigned npol, unsigned M, unsigned Nd, float lower,
                              float upper, uint8_t* mask, unsigned long long* nzap, cudaStream_t st)
{
  const uint64_t ncell = npart * nchan;
  if (ncell == 0) return cudaSuccess;
  g_launches++;
  k_sk_detect<<<unsigned ((ncell + 255) / 256), 256, 0, st>>> (sums, counts, ncell, npol, M, Nd,
                                                              lower, upper, mask, nzap);
  return cudaGetLastError ();
}

cudaError_t launch_sk_mask (const uint8_t* mask, const float2* in, uint64_t in_span, float2* out,
                            uint64_t out_span, uint64_t ndat, unsigned nchan, unsigned npol,
                            unsigned M, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_sk_mask<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (
      mask, in, in_span, out, out_span, ndat, nchan, npol, M);
  return cudaGetLastError ();
}

cudaError_t launch_zero_dm (const InputView& in, const float* lut, uint64_t first, uint64_t n,
                            float2* out, uint64_t span, cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  g_launches++;
  const dim3 grid (unsigned ((n + 255) / 256), in.nchan * in.npol);
  if (in.kind == IN_INT8)
    k_zero_dm<IN_INT8><<<grid, 256, 0, st>>> (in, lut, first, n, out, span);
  else if (in.kind == IN_INT16)
    k_zero_dm<IN_INT16><<<grid, 256, 0, st>>> (in, lut, first, n, out, span);
  else
    k_zero_dm<IN_FLOAT><<<grid, 256, 0, st>>> (in, lut, first, n, out, span);
  return cudaGetLastError ();
}

cudaError_t launch_sk_apply (const uint8_t* mask, float2* v, uint64_t span, uint64_t ndat,
                             unsigned nchan, unsigned npol, unsigned M, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_sk_apply<<<dim3 (unsigned ((ndat + 255) / 256), nchan), 256, 0, st>>> (mask, v, span, ndat,
                                                                            nchan, npol, M);
  return cudaGetLastError ();
}

cudaError_t launch_zeroed_fold (const float2* v, uint64_t span, uint64_t ndat, unsigned nchan,
                                unsigned npol, const FoldView& fv, cudaStream_t st,
                                const KernelClock* clk)
{
  if (ndat == 0) return cudaSuccess;
  const dim3 grid (unsigned ((ndat + 255) / 256), nchan);
  ClockScope cs (clk, KK_INV_COLS, st);
  if (fv.nout == 1)
    k_zeroed_fold<1><<<grid, 256, 0, st>>> (v, span, ndat, npol, fv);
  else if (fv.nout == 2)
    k_zeroed_fold<2><<<grid, 256, 0, st>>> (v, span, ndat, npol, fv);
  else
    k_zeroed_fold<4><<<grid, 256, 0, st>>> (v, span, ndat, npol, fv);
  return cudaGetLastError ();
}

cudaError_t launch_binplan (const FoldSegment* segs, int nseg, uint64_t ndat, unsigned nbin,
                            uint32_t* out, cudaStream_t st)
{
  if (ndat == 0) return cudaSuccess;
  g_launches++;
  k_binplan<<<unsigned ((ndat + 255) / 256), 256, 0, st>>> (segs, nseg, ndat, nbin, out);
  return cudaGetLastError ();
}

} // namespace b200
