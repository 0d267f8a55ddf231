// host_rules.cpp -- host-side bookkeeping of the B200 engine: the dispersion
// smearing rule, FFT-length choice, 8-bit lookup table, fold phase and the
// exact fold-bin plan.
//
// Compiled with -ffp-contract=off: every double operation here must round
// exactly as the reference's x86-64 build does, because the fold-bin plan has
// to reproduce the reference's sequential recurrence bit for bit.

#include "host_rules.h"

#include <cmath>
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

int64_t build_fold_plan (double phi, double p, uint64_t ndat, std::vector<FoldSegment>* out)
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
  return int64_t (segs.size ());
}

} // namespace b200
