// host_rules.cpp -- host-side bookkeeping of the B200 engine: the dispersion
// smearing rule, FFT-length choice, 8-bit lookup table, fold phase and the
// exact fold-bin plan.
//
// Compiled with -ffp-contract=off: every double operation here must round
// exactly as the reference's x86-64 build does, because the fold-bin plan has
// to reproduce the reference's sequential recurrence bit for bit.

#include "host_rules.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <complex>
#include <cstdint>
#include <vector>

namespace b200 {

// Dedispersion.C:32 -- DM (pc/cm^3) = 2.41e-4 D (s MHz^2)
static const double dm_dispersion = 2.41e-4;

// Dedispersion::delay_time (Dedispersion.C:136-140)
static double delay_time (double dm, double freq)
{
  const double dispersion = dm / dm_dispersion;
  return dispersion * 1.0 / (freq * freq);
}

// PlasmaResponse::smearing_time(half) and smearing_samples
// (PlasmaResponse.C:161-250): the worst (lowest) channel, optionally one half
// of it, plus the default 10% buffer (a float, PlasmaResponse.C:20).
unsigned smearing_samples (double centre_frequency, double bandwidth, double dm,
                           unsigned nchan, int half)
{
  const double abs_bw = std::fabs (bandwidth);
  double ch_abs_bw = abs_bw / double (nchan);
  double lower_ch_cfreq = centre_frequency - (abs_bw - ch_abs_bw) / 2.0;
  if (half)
  {
    ch_abs_bw /= 2.0;
    lower_ch_cfreq += double (half) * ch_abs_bw;
  }
  const double lo = lower_ch_cfreq - std::fabs (0.5 * ch_abs_bw);
  const double hi = lower_ch_cfreq + std::fabs (0.5 * ch_abs_bw);
  double tsmear = delay_time (dm, lo) - delay_time (dm, hi);
  const double sampling_rate = std::fabs (bandwidth) / double (nchan) * 1e6;
  const float smearing_buffer = 0.1f;
  tsmear *= (1.0 + smearing_buffer);
  return unsigned (std::ceil (tsmear * sampling_rate));
}

// Observation::get_centre_frequency (Observation.C:521-534): the base frequency
// is the centre of channel 0 (its lower edge when the channels are DC-centred);
// swapped channel orders are undone first (get_unswapped_ichan, :495-518).
double channel_centre (double cf, double bw, unsigned nchan, unsigned ichan, bool swap,
                       bool dc_centred)
{
  const unsigned ch = swap ? (ichan + nchan / 2) % nchan : ichan;
  const double base = dc_centred ? cf - 0.5 * bw : cf - 0.5 * bw + 0.5 * bw / double (nchan);
  return base + double (ch) * bw / double (nchan);
}

// Response::get_minimum_ndat (Response.C:529-545): the smallest power of two
// strictly greater than impulse_pos + impulse_neg.
unsigned minimum_ndat (unsigned impulse_pos, unsigned impulse_neg)
{
  const double tot = double (impulse_pos) + double (impulse_neg);
  if (tot == 0) return 0;
  unsigned m = unsigned (std::pow (2.0, std::ceil (std::log (tot) / std::log (2.0))));
  while (m <= tot) m *= 2;
  return m;
}

// optimal_fft_length (optimize_fft.c:64-135): double the FFT from the minimum
// while N log N / (N - nbad) keeps decreasing.
int64_t optimal_fft_length (uint64_t nbad, uint64_t nfft_max, unsigned factor)
{
  if (!nbad) return -1;
  uint64_t nfft = factor;
  while (nbad > nfft) nfft *= 2;
  if (nfft_max && nfft_max < nfft) return -1;
  double cost = double (nfft) * std::log (double (nfft)) / double (nfft - nbad);
  while (nfft_max == 0 || nfft * 2 < nfft_max)
  {
    const double prev = cost;
    nfft *= 2;
    cost = double (nfft) * std::log (double (nfft)) / double (nfft - nbad);
    if (cost > prev) { nfft /= 2; break; }
  }
  return int64_t (nfft);
}

// BitTable::generate_unique_values for 8 bits (BitTable.C:172-225): 256
// uniformly spaced output levels scaled to unit variance for a quantiser whose
// input thresholds are spaced by `spacing` (in units of sigma).
void bittable8 (double spacing, bool twos_complement, float* lut, double* scale_out)
{
  float values[256];
  const double out_spacing = 1.0 / 256.0;
  const double out_middle = 255.0 / 2.0;
  const unsigned offset = twos_complement ? 128u : 0u;
  double cum = 0.0, var = 0.0;
  for (unsigned i = 0; i < 256; i++)
  {
    const double level = (double (i) - out_middle) * out_spacing;
    values[(i + offset) % 256] = float (level);
    if (i < 128)
    {
      const double threshold = double (int (i + 1) - 128) * spacing;
      const double c = 0.5 * (1.0 + std::erf (threshold / std::sqrt (2.0)));
      var += level * level * (c - cum);
      cum = c;
    }
  }
  var *= 2.0;
  double scale = 1.0 / std::sqrt (var);
  for (unsigned i = 0; i < 256; i++)
    values[i] = float (double (values[i]) * scale);
  scale *= out_spacing;
  for (unsigned i = 0; i < 256; i++) lut[i] = values[i];
  if (scale_out) *scale_out = scale;
}

void interchannel_delays (double cf, double dm, double rate, const double* freq, unsigned nchan,
                          InterchannelDelays* o)
{
  const double dispersion = dm / 2.41e-4;   // Dedispersion::dm_dispersion
  o->delay.assign (nchan, 0);
  o->frac.assign (nchan, 0.0);
  o->applied.assign (nchan, 0);
  for (unsigned c = 0; c < nchan; c++)
  {
    const double time_delay = dispersion * (1.0 / (cf * cf) - 1.0 / (freq[c] * freq[c]));
    const double sample_delay = time_delay * rate;
    o->delay[c] = int64_t (std::floor (sample_delay + 0.5));
    o->frac[c] = sample_delay - double (o->delay[c]);
  }
  // get_delay_range over all channels (DedispersionSampleDelay.C:130-140):
  // the delay at the mean of the end channels' centres
  const double f = (freq[0] + freq[nchan - 1]) / 2;
  const double d = dispersion * (1.0 / (cf * cf) - 1.0 / (f * f));
  o->span_centre = int64_t (std::floor (d * rate + 0.5));
  o->zero_delay = 0;
  for (unsigned c = 0; c < nchan; c++)
    o->zero_delay = std::max (o->zero_delay, o->delay[c] - o->span_centre);
  o->total_delay = 0;
  for (unsigned c = 0; c < nchan; c++)
  {
    const int64_t zd = o->span_centre + o->zero_delay;
    if (zd - o->delay[c] > int64_t (o->total_delay)) o->total_delay = uint64_t (zd - o->delay[c]);
    // SampleDelay::transformation (SampleDelay.C:277-285)
    o->applied[c] = o->zero_delay ? zd - o->delay[c] : o->delay[c];
  }
}

float affine_lut_scale (const float* lut)
{
  // entry 0 is x = 0: 0.5f * s, so s = 2 * lut[0] exactly
  const float s = 2.0f * lut[0];
  if (!(s > 0.0f) || !std::isfinite (s)) return 0.0f;
  for (int b = 0; b < 256; b++)
  {
    const float x = float (int8_t (uint8_t (b)));
    const float v = (x + 0.5f) * s;
    if (std::memcmp (&v, &lut[b], sizeof (float)) != 0) return 0.0f;
  }
  return s;
}

// Fold::get_phi with a constant period (Fold.C:685-693, 975-979):
//   t   = start + (idat_start + 0.5) / rate          (MJD + seconds)
//   phi = fmod((t - epoch) in seconds, P) / P - reference_phase
// An MJD is (day, second of day, fraction of a second); whole seconds of the
// offset are carried into the integer part before differencing.
double fold_phi (int64_t start_day, int64_t start_sec, double start_frac,
                 int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                 uint64_t idat_start, double rate, double period, double reference_phase)
{
  const double offset = (double (idat_start) + 0.5) / rate;
  const double whole = std::floor (offset);
  double frac = start_frac + (offset - whole);
  int64_t sec = start_sec + int64_t (whole);
  if (frac >= 1.0) { frac -= 1.0; sec += 1; }
  const int64_t day = start_day + sec / 86400;
  sec = sec % 86400;
  const double seconds = double ((day - epoch_day) * 86400 + (sec - epoch_sec))
                         + (frac - epoch_frac);
  return std::fmod (seconds, period) / period - reference_phase;
}

// InverseFilterbankEngineCPU::build_fine_channel_plan (InverseFilterbankEngineCPU.C:378-425):
// when one output channel combines several coarse channels, the input channel
// that lands at stitched position i.  The stitched order rolls the band by half
// a coarse channel, swaps the two halves of the band and the two halves of
// every coarse channel; the plan is the inverse of that re-ordering.
std::vector<unsigned> ifb_fine_channel_plan (unsigned nchan, unsigned per_coarse)
{
  std::vector<unsigned> order (nchan);
  for (unsigned i = 0; i < nchan; i++) order[i] = (i + nchan - per_coarse / 2) % nchan;
  std::vector<unsigned> tmp (order);
  for (unsigned i = 0; i < nchan; i++) order[i] = tmp[(i + nchan / 2) % nchan];
  for (unsigned start = 0; start < nchan; start += per_coarse)
    for (unsigned i = 0; i < per_coarse / 2; i++)
      std::swap (order[start + i], order[start + i + per_coarse / 2]);
  std::vector<unsigned> plan (nchan);
  for (unsigned i = 0; i < nchan; i++) plan[order[i]] = i;
  return plan;
}

// Apodization::build (Apodization.C:60-146) and swap (:168-178); the
// arithmetic keeps the reference's float and double steps.
int apodization (int type, unsigned ndat, unsigned t_start, unsigned t_end, bool swap,
                 float* w)
{
  if (ndat == 0) return -1;
  switch (type)
  {
    case 0:   // top hat
      for (unsigned i = 0; i < ndat; i++) w[i] = 1.0f;
      break;
    case 1:   // Hanning
    {
      const double denom = ndat - 1.0;
      for (unsigned i = 0; i < ndat; i++)
        w[i] = float (0.5 * (1 - std::cos (2.0 * M_PI * double (i) / denom)));
      break;
    }
    case 2:   // Welch
    {
      const float centre = 0.5 * (ndat - 1);
      const float denominator = 0.5 * (ndat + 1);
      for (unsigned i = 0; i < ndat; i++)
      {
        const float q = (float (i) - centre) / denominator;
        w[i] = float (1.0 - q * q);
      }
      break;
    }
    case 3:   // Bartlett
    {
      const float centre = 0.5 * (ndat - 1);
      const float denominator = 0.5 * (ndat - 1);
      for (unsigned i = 0; i < ndat; i++)
        w[i] = float (1.0 - std::fabs ((float (i) - centre) / denominator));
      break;
    }
    case 4:   // Tukey
    {
      const float ds = 2 * t_start, de = 2 * t_end;
      for (unsigned i = 0; i < ndat; i++)
      {
        if (i < t_start)
          w[i] = float (0.5 * (1 - std::cos (2.0 * M_PI * float (i) / ds)));
        else if (i + 1 > ndat - t_end)
          w[i] = float (0.5 * (1 - std::cos (2.0 * M_PI * float (ndat - i - 1) / de)));
        else
          w[i] = 1.0f;
      }
      break;
    }
    default:
      return -1;
  }
  if (swap)
    for (unsigned i = 0; i < ndat / 2; i++) std::swap (w[i], w[i + ndat / 2]);
  return 0;
}

// ---------------------------------------------------------------------------
// Spectral-kurtosis thresholds: SKLimits::calc_limits
// (Signal/Statistics/SKLimits.C:136-229) with the Pearson type IV / VI
// densities of PearsonIV.C / PearsonVI.C (Nita & Gary 2010a,b; Nagahara
// 1999).  The cumulative distributions are integrated by adaptive Gauss-Kronrod
// quadrature (the reference uses Romberg on the midpoint rule) with the same
// split of the real line: the tails beyond -1 and +1 through t = -1/u and
// t = 1/u, the middle directly.  The inversion is the reference's
// Newton-Raphson on log CF / log CCF (NewtonRaphson.h).
// ---------------------------------------------------------------------------

namespace {

struct SKPdf
{
  bool vi = false;
  // Pearson IV
  double m = 0, nu = 0, a = 0, lamda = 0;
  // Pearson VI
  double alpha = 0, beta = 0, delta = 0;
  double logk = 0;
  double operator() (double x) const
  {
    if (vi)
    {
      x -= delta;
      return x >= 0 ? std::exp (logk + (alpha - 1) * std::log (x) - (alpha + beta) * std::log1p (x))
                    : 0.0;
    }
    const double a1 = (x - lamda) / a;
    return std::exp (logk - m * std::log1p (a1 * a1) - nu * std::atan (a1));
  }
};

// log |Gamma(x+iy) / Gamma(x)|^2 for x > 0 (Nagahara 1999, Eq. 27).  The
// argument is raised to X = x+n >= 16 by Gamma(z+1) = z Gamma(z), which
// contributes -sum_k log(1 + y^2/(x+k)^2); at X the Stirling series of
// log Gamma (Bernoulli terms to w^-9, error below 1e-16 for |w| >= 16) is
// differenced between w = X+iy and X analytically, so nothing cancels.
double log_gamma_ratio2 (double x, double y)
{
  double acc = 0;
  while (x < 16)
  {
    const double t = y / x;
    acc -= std::log1p (t * t);
    x += 1;
  }
  // Re[(w - 1/2) log w - w] - [(X - 1/2) log X - X]
  const double lead = (x - 0.5) * 0.5 * std::log1p ((y / x) * (y / x)) - y * std::atan2 (y, x);
  // Re S(w) - S(X) with S(w) = 1/(12w) - 1/(360w^3) + 1/(1260w^5) - 1/(1680w^7) + 1/(1188w^9)
  static const double coef[5] = {1.0 / 12, -1.0 / 360, 1.0 / 1260, -1.0 / 1680, 1.0 / 1188};
  const std::complex<double> w (x, y), w2inv = 1.0 / (w * w);
  std::complex<double> pw = 1.0 / w;
  double px = 1.0 / x, sw = 0, sx = 0;
  for (int k = 0; k < 5; k++)
  {
    sw += coef[k] * pw.real ();
    sx += coef[k] * px;
    pw *= w2inv;
    px /= x * x;
  }
  return acc + 2 * (lead + sw - sx);
}

// 7-point Gauss / 15-point Kronrod pair on [a, b] (abscissae and weights of
// Kronrod 1965 as tabulated in QUADPACK); returns the Kronrod estimate and
// |Kronrod - Gauss| as its error.
template <typename F>
double gauss_kronrod15 (const F& f, double a, double b, double* err)
{
  static const double xk[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                               0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                               0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                               0.207784955007898467600689403773245, 0.0};
  static const double wk[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                               0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                               0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                               0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
  static const double wg[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                               0.381830050505118944950369775488975, 0.417959183673469387755102040816327};
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  const double fc = f (c);
  double rk = wk[7] * fc, rg = wg[3] * fc;
  for (int i = 0; i < 7; i++)
  {
    const double s = f (c - h * xk[i]) + f (c + h * xk[i]);
    rk += wk[i] * s;
    if (i & 1) rg += wg[i / 2] * s;
  }
  *err = std::fabs ((rk - rg) * h);
  return rk * h;
}

// Globally adaptive quadrature: bisect the sub-interval with the largest
// error estimate until the summed error is below 1e-13 of the integral (or
// 4000 sub-intervals); an optional break point (a kink of the density) is
// made an interval end from the start.
template <typename F>
double integrate (const F& f, double a, double b, double kink = NAN)
{
  if (a == b) return 0;
  struct Piece { double a, b, v, e; };
  std::vector<Piece> pieces;
  auto add = [&] (double lo, double hi) {
    Piece q {lo, hi, 0, 0};
    q.v = gauss_kronrod15 (f, lo, hi, &q.e);
    pieces.push_back (q);
  };
  if (kink > std::fmin (a, b) && kink < std::fmax (a, b))
  {
    add (a, kink);
    add (kink, b);
  }
  else
    add (a, b);
  for (int iter = 0; iter < 4000; iter++)
  {
    double total = 0, error = 0;
    size_t worst = 0;
    for (size_t i = 0; i < pieces.size (); i++)
    {
      total += pieces[i].v;
      error += pieces[i].e;
      if (pieces[i].e > pieces[worst].e) worst = i;
    }
    if (error <= 1e-13 * std::fabs (total) || error < 1e-300) return total;
    const Piece w = pieces[worst];
    const double m = 0.5 * (w.a + w.b);
    if (!(m > std::fmin (w.a, w.b) && m < std::fmax (w.a, w.b))) return total;
    pieces[worst] = pieces.back ();
    pieces.pop_back ();
    add (w.a, m);
    add (m, w.b);
  }
  double total = 0;
  for (const Piece& q : pieces) total += q.v;
  return total;
}

struct SKCdf
{
  const SKPdf& p;
  // tail integrands through t = -1/u and t = 1/u; zero at u = 0
  double left_tail (double u) const { return u > 0 ? p (-1.0 / u) / (u * u) : 0.0; }
  double right_tail (double u) const { return u > 0 ? p (1.0 / u) / (u * u) : 0.0; }
  // the Pearson VI density starts at x = delta
  double kink_x () const { return p.vi ? p.delta : NAN; }
  double kink_u (double sign) const
  {
    return p.vi && sign * p.delta > 1 ? sign / p.delta : NAN;
  }
  double cf (double x) const
  {
    auto lt = [this] (double u) { return left_tail (u); };
    if (x < -1) return integrate (lt, 0.0, -1.0 / x, kink_u (-1));
    return integrate (lt, 0.0, 1.0, kink_u (-1)) + integrate (p, -1.0, x, kink_x ());
  }
  double ccf (double x) const
  {
    auto rt = [this] (double u) { return right_tail (u); };
    if (x > 1) return integrate (rt, 0.0, 1.0 / x, kink_u (1));
    return integrate (rt, 0.0, 1.0, kink_u (1)) + integrate (p, x, 1.0, kink_x ());
  }
};

// NewtonRaphson.h: x -= (f(x)-y)/f'(x), clamped to [lo, hi], until dx^2 <= (x 1e-12)^2
template <typename F, typename D>
bool newton (const F& f, const D& df, double y, double& x, double lo, double hi)
{
  for (unsigned i = 0; i < 100; i++)
  {
    const double dx = (f (x) - y) / df (x);
    x -= dx;
    if (lo != hi)
    {
      if (x < lo) x = lo;
      if (x > hi) x = hi;
    }
    if (dx * dx <= (x * 1e-12) * (x * 1e-12)) return true;
  }
  return false;
}

// inverse error function by Newton iteration on erf (to double precision)
double inverse_erf (double y)
{
  if (!(y > -1 && y < 1)) return y > 0 ? INFINITY : -INFINITY;
  double x = 0;
  for (int i = 0; i < 100; i++)
  {
    const double dx = (std::erf (x) - y) / (2.0 / std::sqrt (M_PI) * std::exp (-x * x));
    x -= dx;
    if (std::fabs (dx) <= 1e-16 * std::fabs (x)) break;
  }
  return x;
}

} // namespace

int sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest, float* lower, float* upper)
{
  const double fwer = 1.0 - std::erf (double (std_devs) / std::sqrt (2.0));
  if (M < 2 || !(fwer > 0) || Nd == 0 || ntest == 0) return -1;
  const double pcer = 1.0 - std::pow (1 - fwer, 1.0 / ntest);
  const double target = pcer / 2.0;
  const double psd = inverse_erf (1.0 - pcer) * std::sqrt (2.0);
  if (M >= 32768)
  {
    const double factor = std::sqrt (4.0 / double (M)) * psd;
    *lower = float (1.0f - factor);
    *upper = float (1.0f + factor);
    return 0;
  }
  const double Md = M, N = Nd;
  // SKLimits::parametersIV / parametersVI
  double mu2, beta1, beta2;
  double vmu2 = 0, vmu3 = 0, vmu4 = 0;
  {
    const double b = Md / (Md - 1);
    const double lg = std::lgamma (Md * N + 2);
    vmu2 = 2 * N * (N + 1) * Md * b * std::exp (lg - std::lgamma (Md * N + 4));
    vmu3 = 8 * N * (N + 1) * Md * b * b * std::exp (lg - std::lgamma (Md * N + 6))
           * ((N + 4) * Md * N - 5 * N - 2);
    vmu4 = 12 * N * (N + 1) * Md * b * b * b * std::exp (lg - std::lgamma (Md * N + 8))
           * ((Md * Md * Md + 3 * Md * Md) * std::pow (N, 4)
              + (Md * Md * Md + 68 * Md * Md - 93 * Md) * std::pow (N, 3)
              + (125 * Md * Md - 245 * Md + 84) * N * N + (48 - 32 * Md) * N + 24);
  }
  if (Nd == 1)
  {
    mu2 = (4 * Md * Md) / ((Md - 1) * (Md + 2) * (Md + 3));
    beta1 = (4 * (Md + 2) * (Md + 3) * (5 * Md - 7) * (5 * Md - 7))
            / ((Md - 1) * (Md + 4) * (Md + 4) * (Md + 5) * (Md + 5));
    beta2 = 3 * (Md + 2) * (Md + 3) * (Md * Md * Md + 98 * Md * Md - 185 * Md + 78)
            / ((Md - 1) * (Md + 4) * (Md + 5) * (Md + 6) * (Md + 7));
  }
  else
  {
    mu2 = vmu2;
    beta1 = vmu3 * vmu3 / (vmu2 * vmu2 * vmu2);
    beta2 = vmu4 / (vmu2 * vmu2);
  }
  const double kappa = beta1 * (beta2 + 3) * (beta2 + 3)
                       / (4 * (4 * beta2 - 3 * beta1) * (2 * beta2 - 3 * beta1 - 6));
  if (kappa < 0) return -2;   // Pearson type I: not implemented in the reference either
  SKPdf pdf;
  if (kappa > 1)
  {
    // PearsonVI::prepare with Equation (14) of Nita & Gary (2010b)
    pdf.vi = true;
    const double sq = std::sqrt (16 * std::pow (vmu2, 4) + (4 * vmu2 + 1) * vmu3 * vmu3);
    pdf.alpha = std::pow (vmu3, -3)
                * (32 * std::pow (vmu2, 5) - 4 * vmu3 * std::pow (vmu2, 3)
                   + 8 * vmu3 * vmu3 * vmu2 * vmu2 + vmu3 * vmu3 * vmu2 - std::pow (vmu3, 3)
                   + (8 * std::pow (vmu2, 3) - vmu3 * vmu2 + vmu3 * vmu3) * sq);
    pdf.beta = 3 + 2 * vmu2 * std::pow (vmu3, -2) * (4 * vmu2 * vmu2 + sq);
    pdf.delta = (pdf.beta - pdf.alpha - 1) / (pdf.beta - 1);
    pdf.logk = std::lgamma (pdf.alpha + pdf.beta) - std::lgamma (pdf.alpha) - std::lgamma (pdf.beta);
  }
  else
  {
    // PearsonIV::prepare, Equation (57) of Nita & Gary (2010a)
    const double r = (6 * (beta2 - beta1 - 1)) / (2 * beta2 - 3 * beta1 - 6);
    pdf.m = (r + 2) / 2;
    pdf.nu = -(r * (r - 2) * std::sqrt (beta1)) / std::sqrt (16 * (r - 1) - beta1 * (r - 2) * (r - 2));
    pdf.a = 0.25 * std::sqrt (mu2 * ((16 * (r - 1)) - (beta1 * (r - 2) * (r - 2))));
    pdf.lamda = 1.0 - 0.25 * (r - 2) * std::sqrt (mu2) * std::sqrt (beta1);
    const double log_beta = std::lgamma (pdf.m - 0.5) + 0.5 * std::log (M_PI) - std::lgamma (pdf.m);
    pdf.logk = log_gamma_ratio2 (pdf.m, 0.5 * pdf.nu) - std::log (pdf.a) - log_beta;
  }
  SKCdf cdf {pdf};
  const double sym = std::sqrt (mu2) * psd;
  const double lo = 1 - 2 * sym, hi = 1 + 2 * sym;
  double xl = 1 - sym;
  {
    double x = xl;
    auto f = [&] (double v) { return std::log (cdf.cf (v)); };
    auto df = [&] (double v) { return pdf (v) / cdf.cf (v); };
    if (newton (f, df, std::log (target), x, lo, hi)) xl = x;
  }
  double xu = 1 + sym;
  {
    double x = xu;
    auto f = [&] (double v) { return std::log (cdf.ccf (v)); };
    auto df = [&] (double v) { return -pdf (v) / cdf.ccf (v); };
    if (newton (f, df, std::log (target), x, lo, hi)) xu = x;
  }
  *lower = float (xl);
  *upper = float (xu);
  return 0;
}

// ---------------------------------------------------------------------------
// Exact fold-bin plan.
//
// The reference folds with the sequential FP64 recurrence (Fold.C:815-818)
//     phi -= floor(phi);  ibin = unsigned(phi*nbin);  phi += phase_per_sample;
// The subtraction of floor() is exact, so only the addition rounds.  While
// y = frac(phi) stays inside one binade [2^(e-1), 2^e) every representable y
// is a multiple of the binade's ulp G = 2^(e-53), and fl(y + p) = y + dm*G
// with dm = p/G rounded to the nearest integer -- a constant -- unless p/G
// lies exactly half-way (a tie, whose direction then depends on the parity of
// y/G).  So the recurrence is a chain of exact arithmetic progressions, one
// per binade visited per turn, joined by single steps computed with the same
// double operation the reference performs.  A plan segment stores
// (start, m0, dm, G) and sample start+j has y = (m0 + j*dm) * G exactly; the
// GPU evaluates that in integer arithmetic and forms ibin = unsigned(y*nbin)
// with one correctly rounded multiply, so its bins equal the reference's.
// Ties, y == 0 and subnormal y fall back to one-sample segments.
// ---------------------------------------------------------------------------

static void single (std::vector<FoldSegment>& out, uint64_t k, double y)
{
  FoldSegment s;
  s.start = k;
  s.dm = 0;
  if (y == 0.0)
  {
    s.m0 = 0;
    s.g = 1.0;
  }
  else
  {
    int e = 0;
    std::frexp (y, &e);
    s.g = std::ldexp (1.0, e - 53);
    s.m0 = int64_t (y / s.g);
  }
  out.push_back (s);
}

int64_t build_fold_plan (double phi, double p, uint64_t ndat, std::vector<FoldSegment>* out,
                         double* x_end)
{
  std::vector<FoldSegment> local;
  std::vector<FoldSegment>& segs = out ? *out : local;
  segs.clear ();
  const int64_t top = int64_t (1) << 53;
  double x = phi;
  uint64_t k = 0;
  while (k < ndat)
  {
    const double y = x - std::floor (x);
    int e = 0;
    if (y > 0.0 && y < 1.0)
      std::frexp (y, &e);
    // normal y in (0,1) with a usable increment
    if (!(y > 0.0 && y < 1.0) || e < -1000 || !(p > 0.0))
    {
      single (segs, k, y);
      x = y + p;
      k++;
      continue;
    }
    const double g = std::ldexp (1.0, e - 53);
    const double r = p / g;            // exact: scaling by a power of two
    if (r >= 4.0e18)
    {
      single (segs, k, y);
      x = y + p;
      k++;
      continue;
    }
    const double q = std::floor (r);
    const double f = r - q;            // exact
    if (f == 0.5)
    {
      single (segs, k, y);             // round-half-even tie: step singly
      x = y + p;
      k++;
      continue;
    }
    const int64_t dm = int64_t (q) + (f > 0.5 ? 1 : 0);
    const int64_t m0 = int64_t (y / g);
    uint64_t len;
    if (dm == 0)
      len = ndat - k;                  // y + p rounds back to y forever
    else
      len = uint64_t ((top - 1 - m0) / dm) + 1;
    if (len > ndat - k) len = ndat - k;
    FoldSegment s;
    s.start = k;
    s.m0 = m0;
    s.dm = dm;
    s.g = g;
    segs.push_back (s);
    const double ylast = double (m0 + int64_t (len - 1) * dm) * g;
    x = ylast + p;                     // the reference's own rounding step
    k += len;
  }
  if (x_end) *x_end = x;
  return int64_t (segs.size ());
}

// Archiver::set(Pulsar::Profile*) (Archiver.C:852-984): the amplitude of bin
// ibin is the folded sum over (scale * hits) in double, stored as float;
// unhit bins take the double mean of the hit bins (Archiver.C:944-971);
// a non-finite sum zeroes the profile and marks the channel corrupted, which
// sets the channel's weight to 0 (Archiver.C:776-783).
int archive_profiles (const float* sums, const uint32_t* hits, bool zeroed,
                      unsigned nchan, unsigned npol, unsigned nbin, double scale,
                      uint64_t ndat_total, bool unload_zero_hits, float* amps, float* weights,
                      unsigned* corrupted)
{
  if (!sums || !hits || !amps || !weights || nchan == 0 || npol == 0 || nbin == 0)
    return -1;
  if (scale == 0 || !std::isfinite (scale)) return -1;
  if (zeroed && ndat_total == 0) return -1;
  unsigned bad = 0;
  for (unsigned ic = 0; ic < nchan; ic++)
  {
    const uint32_t* h = hits + (zeroed ? uint64_t (ic) * nbin : 0);
    bool chan_corrupt = false;
    float chan_weight = 1.0f;
    for (unsigned ip = 0; ip < npol; ip++)
    {
      const float* from = sums + (uint64_t (ic) * npol + ip) * nbin;
      float* into = amps + (uint64_t (ic) * npol + ip) * nbin;
      unsigned zeroes = 0, not_finite = 0;
      uint32_t hits_sum = 0;
      for (unsigned ib = 0; ib < nbin; ib++)
      {
        hits_sum += h[ib];
        if (h[ib] == 0)
        {
          zeroes++;
          into[ib] = 0.0f;
        }
        else if (!std::isfinite (from[ib]))
          not_finite++;
        else
          into[ib] = float (double (from[ib]) / (scale * double (h[ib])));
      }
      if (not_finite)
      {
        for (unsigned ib = 0; ib < nbin; ib++) into[ib] = 0.0f;
        chan_corrupt = true;
        bad++;
      }
      if (zeroes)
      {
        if (!unload_zero_hits) return -2;
        double sum = 0.0;
        unsigned count = 0;
        for (unsigned ib = 0; ib < nbin; ib++)
          if (h[ib] != 0)
          {
            sum += into[ib];
            count++;
          }
        if (count == 0) count = 1;
        const double mean = sum / count;
        for (unsigned ib = 0; ib < nbin; ib++)
          if (h[ib] == 0) into[ib] = float (mean);
      }
      if (zeroed) chan_weight = float (hits_sum) / float (ndat_total);
    }
    weights[ic] = chan_corrupt ? 0.0f : chan_weight;
  }
  if (corrupted) *corrupted = bad;
  return 0;
}

} // namespace b200
