// fft_core.cuh -- FFT building blocks for the B200 convolution kernels.
//
// Everything here is __host__ __device__ so that the index arithmetic of the
// shared-memory Stockham passes can be exercised on the CPU (one "thread" at a
// time, phase by phase) as well as on the GPU.
//
// Conventions follow the reference's FTransform (FFTW): forward transforms use
// exp(-2 pi i nk/N) (D = -1), backward transforms exp(+2 pi i nk/N) (D = +1),
// both unnormalised.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define B200_HD __host__ __device__ __forceinline__
#define B200_CE __host__ __device__ constexpr

namespace b200 {

B200_HD float2 cadd (float2 a, float2 b) { return make_float2 (a.x + b.x, a.y + b.y); }
B200_HD float2 csub (float2 a, float2 b) { return make_float2 (a.x - b.x, a.y - b.y); }
B200_HD float2 cmul (float2 a, float2 b)
{
  return make_float2 (a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
B200_HD float2 cmulc (float2 a, float2 b)
{
  return make_float2 (a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
B200_HD float2 cscale (float2 a, float s) { return make_float2 (a.x * s, a.y * s); }

// cos(2 pi j / 64) for j = 0..16, correctly rounded decimal expansions.
B200_CE float quarter_cos64 (int j)
{
  return j == 0 ? 1.0f
       : j == 1 ? 0.99518472667219692873f
       : j == 2 ? 0.98078528040323043058f
       : j == 3 ? 0.95694033573220882438f
       : j == 4 ? 0.92387953251128673848f
       : j == 5 ? 0.88192126434835504956f
       : j == 6 ? 0.83146961230254523567f
       : j == 7 ? 0.77301045336273699338f
       : j == 8 ? 0.70710678118654752440f
       : j == 9 ? 0.63439328416364548779f
       : j == 10 ? 0.55557023301960222474f
       : j == 11 ? 0.47139673682599764856f
       : j == 12 ? 0.38268343236508977173f
       : j == 13 ? 0.29028467725446236764f
       : j == 14 ? 0.19509032201612826785f
       : j == 15 ? 0.09801714032956060199f
       : 0.0f;
}

// cos and sin of 2 pi j / 64 for any integer j (reduced to the first quadrant)
B200_CE float cos64 (int j)
{
  return (j & 63) <= 16 ? quarter_cos64 (j & 63)
       : (j & 63) <= 32 ? -quarter_cos64 (32 - (j & 63))
       : (j & 63) <= 48 ? -quarter_cos64 ((j & 63) - 32)
       : quarter_cos64 (64 - (j & 63));
}
B200_CE float sin64 (int j) { return cos64 (j - 16); }

// v * w_R^k with w_R = exp(D 2 pi i / R); k is a compile-time constant after
// unrolling, so the special cases cost nothing.
template <int R, int D>
B200_HD float2 tw_mul (int k, float2 v)
{
  const int j = (k * 64 / R) & 63;     // angle in units of 2 pi / 64
  if (j == 0) return v;
  if (j == 16) return D < 0 ? make_float2 (v.y, -v.x) : make_float2 (-v.y, v.x);
  if (j == 32) return make_float2 (-v.x, -v.y);
  if (j == 48) return D < 0 ? make_float2 (-v.y, v.x) : make_float2 (v.y, -v.x);
  const float c = cos64 (j);
  const float s = D < 0 ? -sin64 (j) : sin64 (j);
  if (j == 8 || j == 24 || j == 40 || j == 56)
  {
    // |c| == |s| == sqrt(1/2): (v.x c - v.y s, v.x s + v.y c)
    const float h = quarter_cos64 (8);
    const float a = (c > 0 ? v.x : -v.x);
    const float b = (s > 0 ? v.y : -v.y);
    const float e = (s > 0 ? v.x : -v.x);
    const float f = (c > 0 ? v.y : -v.y);
    return make_float2 ((a - b) * h, (e + f) * h);
  }
  return make_float2 (v.x * c - v.y * s, v.x * s + v.y * c);
}

// In-register DFT of size R (power of two, R <= 64), natural order in and out.
// Recursive radix-2 decimation in time, fully unrolled.
template <int R, int D>
struct RegDFT
{
  B200_HD static void run (float2* v)
  {
    float2 e[R / 2], o[R / 2];
#pragma unroll
    for (int i = 0; i < R / 2; i++)
    {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    RegDFT<R / 2, D>::run (e);
    RegDFT<R / 2, D>::run (o);
#pragma unroll
    for (int k = 0; k < R / 2; k++)
    {
      const float2 t = tw_mul<R, D> (k, o[k]);
      v[k] = cadd (e[k], t);
      v[k + R / 2] = csub (e[k], t);
    }
  }
};

template <int D>
struct RegDFT<2, D>
{
  B200_HD static void run (float2* v)
  {
    const float2 a = v[0], b = v[1];
    v[0] = cadd (a, b);
    v[1] = csub (a, b);
  }
};

template <int D>
struct RegDFT<1, D>
{
  B200_HD static void run (float2*) {}
};

// cos(2 pi j / 96) for j = 0..24 (decimal expansions to 22 digits), for the
// twiddles of transforms whose length has a factor 3.
B200_CE float quarter_cos96 (int j)
{
  return j == 0 ? 1.0f
       : j == 1 ? 0.9978589232386035067380f
       : j == 2 ? 0.9914448613738104111445f
       : j == 3 ? 0.9807852804032304491261f
       : j == 4 ? 0.9659258262890682867497f
       : j == 5 ? 0.9469301294951056642558f
       : j == 6 ? 0.9238795325112867561281f
       : j == 7 ? 0.8968727415326883038941f
       : j == 8 ? 0.8660254037844386467637f
       : j == 9 ? 0.8314696123025452370787f
       : j == 10 ? 0.7933533402912351645797f
       : j == 11 ? 0.7518398074789773964075f
       : j == 12 ? 0.7071067811865475244008f
       : j == 13 ? 0.6593458151000688684251f
       : j == 14 ? 0.6087614290087206394160f
       : j == 15 ? 0.5555702330196022247428f
       : j == 16 ? 0.5f
       : j == 17 ? 0.4422886902190012819952f
       : j == 18 ? 0.3826834323650897717284f
       : j == 19 ? 0.3214394653031615807010f
       : j == 20 ? 0.2588190451025207623488f
       : j == 21 ? 0.1950903220161282678482f
       : j == 22 ? 0.1305261922200515915484f
       : j == 23 ? 0.0654031292301430668153f
       : 0.0f;
}

B200_CE float cos96 (int j)
{
  const int m = ((j % 96) + 96) % 96;
  return m <= 24 ? quarter_cos96 (m)
       : m <= 48 ? -quarter_cos96 (48 - m)
       : m <= 72 ? -quarter_cos96 (m - 48)
       : quarter_cos96 (96 - m);
}
B200_CE float sin96 (int j) { return cos96 (j - 24); }

// v * w_R^k, w_R = exp(D 2 pi i / R), for R dividing 96
template <int R, int D>
B200_HD float2 tw_mul96 (int k, float2 v)
{
  const int j = (k * (96 / R)) % 96;
  if (j == 0) return v;
  if (j == 24) return D < 0 ? make_float2 (v.y, -v.x) : make_float2 (-v.y, v.x);
  if (j == 48) return make_float2 (-v.x, -v.y);
  if (j == 72) return D < 0 ? make_float2 (-v.y, v.x) : make_float2 (v.y, -v.x);
  const float c = cos96 (j);
  const float s = D < 0 ? -sin96 (j) : sin96 (j);
  return make_float2 (v.x * c - v.y * s, v.x * s + v.y * c);
}

// In-register DFT of size R = 2^a or 3 * 2^a (R <= 96), natural order in and
// out.  A factor 3 is split off first (decimation in time: three interleaved
// sub-sequences of length R/3, twiddled, then 3-point butterflies); powers of
// two go to RegDFT.
template <int R, int D>
struct RegDFTm
{
  B200_HD static void run (float2* v)
  {
    if constexpr (R % 3 != 0)
      RegDFT<R, D>::run (v);
    else
    {
      constexpr int M = R / 3;
      float2 e[3][M];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int m = 0; m < M; m++) e[r][m] = v[3 * m + r];
#pragma unroll
      for (int r = 0; r < 3; r++) RegDFT<M, D>::run (e[r]);
      // sin(2 pi / 3)
      const float h = 0.8660254037844386467637f;
#pragma unroll
      for (int k = 0; k < M; k++)
      {
        const float2 a = e[0][k];
        const float2 b = tw_mul96<R, D> (k, e[1][k]);
        const float2 c = tw_mul96<R, D> (2 * k, e[2][k]);
        const float2 s = cadd (b, c);
        const float2 d = csub (b, c);
        const float2 m = make_float2 (a.x - 0.5f * s.x, a.y - 0.5f * s.y);
        // D * i * h * d
        const float2 r = D < 0 ? make_float2 (h * d.y, -h * d.x) : make_float2 (-h * d.y, h * d.x);
        v[k] = cadd (a, s);
        v[k + M] = cadd (m, r);
        v[k + 2 * M] = csub (m, r);
      }
    }
  }
};

// Shared-memory index padding: one float2 of padding per 16 entries keeps the
// strided Stockham stores of the early passes off a single bank.
B200_HD int spad (int i) { return i + (i >> 4); }
B200_CE int spad_size (int n) { return n + (n >> 4); }

// Stockham pass schedule for an N-point transform run by T = N/16 threads:
// every pass leaves each thread exactly 16 complex values in registers.
// Returns the radix of pass p (0 when there is no such pass).
B200_CE int stockham_radix (int N, int p)
{
  return N == 16384 ? (p < 3 ? 16 : p == 3 ? 4 : 0)
       : N == 8192 ? (p < 3 ? 16 : p == 3 ? 2 : 0)
       : N == 4096 ? (p < 3 ? 16 : 0)
       : N == 2048 ? (p < 2 ? 16 : p == 2 ? 8 : 0)
       : N == 1024 ? (p < 2 ? 16 : p == 2 ? 4 : 0)
       : N == 512 ? (p < 2 ? 16 : p == 2 ? 2 : 0)
       : N == 256 ? (p < 2 ? 16 : 0)
       : N == 128 ? (p < 1 ? 16 : p == 1 ? 8 : 0)
       : N == 64 ? (p < 1 ? 16 : p == 1 ? 4 : 0)
       : 0;
}

B200_CE int stockham_npass (int N)
{
  return stockham_radix (N, 0) == 0 ? 0
       : stockham_radix (N, 1) == 0 ? 1
       : stockham_radix (N, 2) == 0 ? 2
       : stockham_radix (N, 3) == 0 ? 3 : 4;
}

// product of the radices of passes before p
B200_CE int stockham_ns (int N, int p)
{
  return p == 0 ? 1 : stockham_ns (N, p - 1) * stockham_radix (N, p - 1);
}

// threads of an N-point transform
B200_CE int stockham_threads (int N) { return N / 16; }

// One radix-R Stockham pass (Govindaraju et al., SC08, "High performance
// discrete Fourier transforms on graphics processors"): butterfly j reads
// x[j + r N/R], applies w_{Ns R}^{(j mod Ns) r}, performs an R-point DFT and
// writes x'[(j div Ns) Ns R + (j mod Ns) + r Ns].  Output is in natural order
// after the last pass.  tw[m] = exp(-2 pi i m / N) (FP64-computed, rounded).
template <int N, int R, int T, int D>
struct StockhamPass
{
  static constexpr int NB = N / R;      // butterflies in this pass
  static constexpr int BPT = NB / T;    // butterflies per thread
  static_assert (BPT >= 1 && BPT * T == NB, "thread count does not tile the pass");

  B200_HD static void load (int tid, const float2* s, float2* v)
  {
#pragma unroll
    for (int b = 0; b < BPT; b++)
    {
      const int j = tid + b * T;
#pragma unroll
      for (int r = 0; r < R; r++)
        v[b * R + r] = s[spad (j + r * NB)];
    }
  }

  B200_HD static void compute_store (int tid, int Ns, float2* v, float2* s, const float2* tw)
  {
#pragma unroll
    for (int b = 0; b < BPT; b++)
    {
      const int j = tid + b * T;
      const int a = j & (Ns - 1);
      float2* x = v + b * R;
      if (Ns > 1)
      {
        const int step = N / (Ns * R);
#pragma unroll
        for (int r = 1; r < R; r++)
        {
          const float2 w = tw[a * r * step];
          x[r] = D < 0 ? cmul (x[r], w) : cmulc (x[r], w);
        }
      }
      RegDFT<R, D>::run (x);
      const int idxD = (j - a) * R + a;
#pragma unroll
      for (int r = 0; r < R; r++)
        s[spad (idxD + r * Ns)] = x[r];
    }
  }
};

// Per-pass twiddle tables: pass p >= 1 of an N-point schedule uses
// w_{Ns R}^{a r} for a < Ns, 1 <= r < R, stored [r-1][a] (a fastest) so that
// lanes holding consecutive butterflies read consecutive entries.
B200_CE int pass_table_size (int N, int p)
{
  return p == 0 ? 0 : stockham_ns (N, p) * (stockham_radix (N, p) - 1);
}
B200_CE int pass_table_offset (int N, int p)
{
  return p <= 1 ? 0 : pass_table_offset (N, p - 1) + pass_table_size (N, p - 1);
}
B200_CE int pass_tables_size (int N)
{
  return pass_table_offset (N, stockham_npass (N) - 1)
         + pass_table_size (N, stockham_npass (N) - 1);
}

// The same radix-R pass with its twiddles from a per-pass table and with the
// source / destination layouts chosen by the caller: PADI/PADO select the
// padded shared-memory layout (spad) for input/output; an unpadded side may
// be a staging buffer or global memory.
template <int N, int R, int T, int D, bool PADI, bool PADO>
struct StockhamPassT
{
  static constexpr int NB = N / R;
  static constexpr int BPT = NB / T;
  static_assert (BPT >= 1 && BPT * T == NB, "thread count does not tile the pass");

  B200_HD static void load (int tid, const float2* s, float2* v)
  {
#pragma unroll
    for (int b = 0; b < BPT; b++)
    {
      const int j = tid + b * T;
#pragma unroll
      for (int r = 0; r < R; r++)
        v[b * R + r] = s[PADI ? spad (j + r * NB) : j + r * NB];
    }
  }

  // twp: this pass's table ([r-1][a], Ns entries per r) or null when Ns == 1
  B200_HD static void compute_store (int tid, int Ns, float2* v, float2* s, const float2* twp)
  {
#pragma unroll
    for (int b = 0; b < BPT; b++)
    {
      const int j = tid + b * T;
      const int a = j & (Ns - 1);
      float2* x = v + b * R;
      if (Ns > 1)
      {
#pragma unroll
        for (int r = 1; r < R; r++)
        {
          const float2 w = twp[(r - 1) * Ns + a];
          x[r] = D < 0 ? cmul (x[r], w) : cmulc (x[r], w);
        }
      }
      RegDFT<R, D>::run (x);
      const int idxD = (j - a) * R + a;
#pragma unroll
      for (int r = 0; r < R; r++)
        s[PADO ? spad (idxD + r * Ns) : idxD + r * Ns] = x[r];
    }
  }
};

// Rows of N2 = 4096 or 8192 points run by T = N2 / 32 threads holding 32
// values each, in three passes: radix 16 (Ns 1), radix N2 / 256 (Ns 16),
// radix 16 (Ns N2 / 16).  The last pass leaves in thread tid the values
// X[j + r N2/16] (j = tid + b T, b < 2, r < 16), exactly what the first pass
// of a following transform needs in that thread, so a response multiply and
// the next transform's first pass follow in registers.  Pass 0 reads its
// input in natural order from anywhere (global memory); passes 1 and 2 go
// through one padded shared-memory row.  Twiddles: pass 1 from a table
// w_{16 R1}^{a r} [r-1][a]; pass 2 (a < N2/16) as the product of
// w_N2^{32 ah r} [r-1][ah] and w_N2^{al r} [r-1][al], a = 32 ah + al.
template <int N2>
struct Row32
{
  static_assert (N2 == 4096 || N2 == 8192, "Row32 covers 4096- and 8192-point rows");
  static constexpr int T = N2 / 32;        // threads
  static constexpr int R1 = N2 / 256;      // radix of pass 1
  static constexpr int B1 = 256 / T;       // butterflies per thread in pass 1
  static constexpr int NS2 = N2 / 16;      // Ns of pass 2 (and the stride of pass 0's inputs)
  static constexpr int AH = NS2 / 32;      // high digits of a pass-2 twiddle index
  static constexpr int TAB1 = (R1 - 1) * 16;
  static constexpr int TABH = 15 * AH;
  static constexpr int TABL = 15 * 32;
  static constexpr int TABN = TAB1 + TABH + TABL;

  // entry i of the concatenated tables (pass 1, pass-2 high, pass-2 low), as
  // w^m = exp(-2 pi i m / n) rounded from double
  B200_HD static float2 table_entry (int i)
  {
    int m, n;
    if (i < TAB1)
    {
      m = (i % 16) * (i / 16 + 1);
      n = 16 * R1;
    }
    else if (i < TAB1 + TABH)
    {
      i -= TAB1;
      m = 32 * (i % AH) * (i / AH + 1);
      n = N2;
    }
    else
    {
      i -= TAB1 + TABH;
      m = (i % 32) * (i / 32 + 1);
      n = N2;
    }
    m %= n;
    double sn, cs;
#ifdef __CUDA_ARCH__
    sincospi (2.0 * double (m) / double (n), &sn, &cs);
#else
    const double ang = 2.0 * 3.14159265358979323846 * double (m) / double (n);
    sn = sin (ang);
    cs = cos (ang);
#endif
    return make_float2 (float (cs), float (-sn));
  }

  // pass 0 input: v[16 b + r] = x[j + r NS2]
  B200_HD static void p0_load (int tid, const float2* x, float2* v)
  {
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++) v[16 * b + r] = x[tid + b * T + r * NS2];
  }

  // pass 0 (or the first pass of a transform whose input the previous pass 2
  // left in registers): 16-point DFTs, outputs to s[j 16 + r]
  template <int D>
  B200_HD static void p0_compute_store (int tid, float2* v, float2* s)
  {
#pragma unroll
    for (int b = 0; b < 2; b++)
    {
      const int j = tid + b * T;
      RegDFT<16, D>::run (v + 16 * b);
#pragma unroll
      for (int r = 0; r < 16; r++) s[spad (j * 16 + r)] = v[16 * b + r];
    }
  }

  B200_HD static void p1_load (int tid, const float2* s, float2* v)
  {
#pragma unroll
    for (int b = 0; b < B1; b++)
#pragma unroll
      for (int r = 0; r < R1; r++) v[b * R1 + r] = s[spad (tid + b * T + r * 256)];
  }

  template <int D>
  B200_HD static void p1_compute_store (int tid, float2* v, float2* s, const float2* tab1)
  {
#pragma unroll
    for (int b = 0; b < B1; b++)
    {
      const int j = tid + b * T;
      const int a = j & 15;
      float2* x = v + b * R1;
#pragma unroll
      for (int r = 1; r < R1; r++)
      {
        const float2 w = tab1[(r - 1) * 16 + a];
        x[r] = D < 0 ? cmul (x[r], w) : cmulc (x[r], w);
      }
      RegDFT<R1, D>::run (x);
      const int o = (j - a) * R1 + a;
#pragma unroll
      for (int r = 0; r < R1; r++) s[spad (o + r * 16)] = x[r];
    }
  }

  B200_HD static void p2_load (int tid, const float2* s, float2* v)
  {
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++) v[16 * b + r] = s[spad (tid + b * T + r * NS2)];
  }

  // pass 2 in registers: afterwards v[16 b + r] = X[j + r NS2]
  template <int D>
  B200_HD static void p2_compute (int tid, float2* v, const float2* th, const float2* tl)
  {
#pragma unroll
    for (int b = 0; b < 2; b++)
    {
      const int a = tid + b * T;            // < NS2: j itself
      const int ah = a >> 5, al = a & 31;
      float2* x = v + 16 * b;
#pragma unroll
      for (int r = 1; r < 16; r++)
      {
        const float2 w = cmul (th[(r - 1) * AH + ah], tl[(r - 1) * 32 + al]);
        x[r] = D < 0 ? cmul (x[r], w) : cmulc (x[r], w);
      }
      RegDFT<16, D>::run (x);
    }
  }

  // natural-order output of pass 2
  B200_HD static void p2_store (int tid, const float2* v, float2* x)
  {
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int r = 0; r < 16; r++) x[tid + b * T + r * NS2] = v[16 * b + r];
  }
};

} // namespace b200
