// CPU run of the Row32 pass schedule (fft_core.cuh), one thread at a time
// and phase by phase as the row kernel's barriers order them: the forward
// transform, the response multiply in registers, the inverse transform.
// Checks against an FP64 DFT and that every shared-memory access of a
// half-warp (eight-byte words) falls in 16 distinct bank pairs.
#include "fft_core.cuh"

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

using namespace b200;
typedef std::complex<double> cd;

static std::vector<cd> dft (const std::vector<cd>& x, int sign)
{
  const int n = int (x.size ());
  std::vector<cd> w (n), y (n);
  for (int m = 0; m < n; m++)
    w[m] = std::polar (1.0, sign * 2.0 * 3.14159265358979323846 * m / n);
  for (int k = 0; k < n; k++)
  {
    cd acc = 0;
    for (int t = 0; t < n; t++) acc += x[t] * w[(int64_t (k) * t) % n];
    y[k] = acc;
  }
  return y;
}

// shared-memory indices one pass touches, per thread, in access order
struct Trace
{
  std::vector<std::vector<int>> idx;
  explicit Trace (int T) : idx (T) {}
};

static int conflicts (const Trace& tr)
{
  int bad = 0;
  const int T = int (tr.idx.size ());
  for (int w = 0; w < T; w += 32)
    for (size_t k = 0; k < tr.idx[w].size (); k++)
      for (int h = 0; h < 32; h += 16)
      {
        unsigned seen = 0;
        for (int l = 0; l < 16; l++)
        {
          const unsigned bank = unsigned (tr.idx[w + h + l][k]) & 15u;
          if (seen & (1u << bank)) bad++;
          seen |= 1u << bank;
        }
      }
  return bad;
}

// a shared-memory row that records the indices each thread touches
struct SRow
{
  std::vector<float2> data;
  Trace* tr = nullptr;
  int tid = 0;
};

template <int N2>
static int run ()
{
  typedef Row32<N2> RS;
  constexpr int T = RS::T;
  std::mt19937_64 rng (N2);
  std::normal_distribution<double> g;
  std::vector<float2> x (N2), h (N2), y (N2);
  std::vector<cd> xd (N2), hd (N2);
  for (int i = 0; i < N2; i++)
  {
    x[i] = make_float2 (float (g (rng)), float (g (rng)));
    const double ph = 6.283185307179586 * double (int64_t (i) * i % 977) / 977.0;
    h[i] = make_float2 (float (cos (ph)), float (sin (ph)));
    xd[i] = cd (x[i].x, x[i].y);
    hd[i] = cd (h[i].x, h[i].y);
  }
  std::vector<float2> tab (RS::TABN);
  for (int i = 0; i < RS::TABN; i++) tab[i] = RS::table_entry (i);
  const float2* tab1 = tab.data ();
  const float2* th = tab1 + RS::TAB1;
  const float2* tl = th + RS::TABH;

  std::vector<float2> s (spad_size (N2));
  std::vector<std::vector<float2>> v (T, std::vector<float2> (32));
  int bad = 0;

  // shared-memory index traces: recompute the same addresses as the passes
  auto trace_p0_store = [&] {
    Trace tr (T);
    for (int t = 0; t < T; t++)
      for (int b = 0; b < 2; b++)
        for (int r = 0; r < 16; r++) tr.idx[t].push_back (spad ((t + b * T) * 16 + r));
    return conflicts (tr);
  };
  auto trace_p1 = [&] {
    Trace ld (T), st (T);
    for (int t = 0; t < T; t++)
      for (int b = 0; b < RS::B1; b++)
      {
        const int j = t + b * T, a = j & 15;
        for (int r = 0; r < RS::R1; r++)
        {
          ld.idx[t].push_back (spad (j + r * 256));
          st.idx[t].push_back (spad ((j - a) * RS::R1 + a + r * 16));
        }
      }
    return conflicts (ld) + conflicts (st);
  };
  auto trace_p2 = [&] {
    Trace ld (T);
    for (int t = 0; t < T; t++)
      for (int b = 0; b < 2; b++)
        for (int r = 0; r < 16; r++) ld.idx[t].push_back (spad (t + b * T + r * RS::NS2));
    return conflicts (ld);
  };
  bad += trace_p0_store () + trace_p1 () + trace_p2 ();

  // forward
  for (int t = 0; t < T; t++) RS::p0_load (t, x.data (), v[t].data ());
  for (int t = 0; t < T; t++) RS::template p0_compute_store<-1> (t, v[t].data (), s.data ());
  for (int t = 0; t < T; t++) RS::p1_load (t, s.data (), v[t].data ());
  for (int t = 0; t < T; t++) RS::template p1_compute_store<-1> (t, v[t].data (), s.data (), tab1);
  for (int t = 0; t < T; t++) RS::p2_load (t, s.data (), v[t].data ());
  std::vector<float2> X (N2);
  for (int t = 0; t < T; t++)
  {
    RS::template p2_compute<-1> (t, v[t].data (), th, tl);
    RS::p2_store (t, v[t].data (), X.data ());
  }
  // response multiply in registers, then the inverse
  for (int t = 0; t < T; t++)
    for (int b = 0; b < 2; b++)
      for (int r = 0; r < 16; r++)
      {
        float2& d = v[t][16 * b + r];
        d = cmul (d, h[t + b * T + r * RS::NS2]);
      }
  for (int t = 0; t < T; t++) RS::template p0_compute_store<+1> (t, v[t].data (), s.data ());
  for (int t = 0; t < T; t++) RS::p1_load (t, s.data (), v[t].data ());
  for (int t = 0; t < T; t++) RS::template p1_compute_store<+1> (t, v[t].data (), s.data (), tab1);
  for (int t = 0; t < T; t++) RS::p2_load (t, s.data (), v[t].data ());
  for (int t = 0; t < T; t++)
  {
    RS::template p2_compute<+1> (t, v[t].data (), th, tl);
    RS::p2_store (t, v[t].data (), y.data ());
  }

  const std::vector<cd> Xd = dft (xd, -1);
  std::vector<cd> Yd (N2);
  for (int i = 0; i < N2; i++) Yd[i] = Xd[i] * hd[i];
  const std::vector<cd> yd = dft (Yd, +1);
  double e1 = 0, n1 = 0, e2 = 0, n2 = 0;
  for (int i = 0; i < N2; i++)
  {
    e1 += std::norm (cd (X[i].x, X[i].y) - Xd[i]);
    n1 += std::norm (Xd[i]);
    e2 += std::norm (cd (y[i].x, y[i].y) - yd[i]);
    n2 += std::norm (yd[i]);
  }
  const double r1 = sqrt (e1 / n1), r2 = sqrt (e2 / n2);
  printf ("row32 N2=%d forward_rel_rms=%.3e conv_rel_rms=%.3e bank_conflicts=%d\n", N2, r1, r2,
          bad);
  return (r1 < 1e-6 && r2 < 1e-6 && bad == 0) ? 0 : 1;
}

int main ()
{
  int rc = run<4096> ();
  rc |= run<8192> ();
  return rc;
}
