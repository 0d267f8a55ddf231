// oracle.cpp -- CPU restatement of the DSPSR baseband hot path.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker / timed CPU baseline.  The
// product library never links or calls it.
//
// Each function names the reference source it restates (paths relative to the
// DSPSR tree).  Built by oracle/Makefile with -ffp-contract=off so that every
// float operation rounds exactly as written, as the reference's x86-64 build
// (SSE2, no FMA contraction) does.

#include "../oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <memory>
#include <algorithm>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// FFT with FFTW's conventions (FTransform::fcc1d forward sign -1, bcc1d
// backward sign +1, both unnormalised).  Radix-2 decimation in time; twiddles
// are computed in double and rounded once to T.
// ---------------------------------------------------------------------------

template <typename T>
struct Plan
{
  int n = 0, log2n = 0;
  std::vector<uint32_t> rev;
  std::vector<std::complex<T>> tw;   // tw[k] = exp(-2 pi i k / n), k < n/2
};

std::mutex plan_mutex;

template <typename T>
const Plan<T>& get_plan (int n)
{
  static std::map<int, std::unique_ptr<Plan<T>>> plans;
  std::lock_guard<std::mutex> lock (plan_mutex);
  auto it = plans.find (n);
  if (it != plans.end ())
    return *it->second;
  auto p = std::make_unique<Plan<T>> ();
  p->n = n;
  int lg = 0;
  while ((1 << lg) < n) lg++;
  p->log2n = lg;
  p->rev.resize (n);
  for (int i = 0; i < n; i++)
  {
    uint32_t r = 0;
    for (int b = 0; b < lg; b++)
      if (i & (1 << b)) r |= 1u << (lg - 1 - b);
    p->rev[i] = r;
  }
  p->tw.resize (std::max (1, n / 2));
  for (int k = 0; k < n / 2; k++)
  {
    double a = -2.0 * M_PI * double (k) / double (n);
    p->tw[k] = std::complex<T> (T (std::cos (a)), T (std::sin (a)));
  }
  auto& ref = *p;
  plans[n] = std::move (p);
  return ref;
}

template <typename T>
void fft (int n, int sign, const std::complex<T>* in, std::complex<T>* out)
{
  const Plan<T>& p = get_plan<T> (n);
  if (in == out)
  {
    std::vector<std::complex<T>> tmp (in, in + n);
    for (int i = 0; i < n; i++) out[p.rev[i]] = tmp[i];
  }
  else
    for (int i = 0; i < n; i++) out[p.rev[i]] = in[i];

  for (int len = 2; len <= n; len <<= 1)
  {
    const int half = len >> 1;
    const int tstep = n / len;
    for (int i = 0; i < n; i += len)
    {
      for (int j = 0; j < half; j++)
      {
        std::complex<T> w = p.tw[j * tstep];
        if (sign > 0) w = std::conj (w);
        const std::complex<T> a = out[i + j];
        const std::complex<T> b0 = out[i + j + half];
        // explicit real arithmetic: no library complex-multiply NaN handling
        const T br = w.real () * b0.real () - w.imag () * b0.imag ();
        const T bi = w.real () * b0.imag () + w.imag () * b0.real ();
        out[i + j] = std::complex<T> (a.real () + br, a.imag () + bi);
        out[i + j + half] = std::complex<T> (a.real () - br, a.imag () - bi);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Observation / PlasmaResponse helpers
// ---------------------------------------------------------------------------

// Dedispersion.C:32 -- DM (pc/cm^3) = 2.41e-4 D (s MHz^2)
const double dm_dispersion = 2.41e-4;

template <typename T> inline T sqr (T x) { return x * x; }

// Dedispersion.C:136-140
double delay_time (double dm, double freq)
{
  double dispersion = dm / dm_dispersion;
  return dispersion * 1.0 / sqr (freq);
}

// Observation.C:521-534 (no channel swapping): centre of channel ichan
double channel_centre (double cf, double bw, unsigned nchan, unsigned ichan, bool dc_centred)
{
  double base = dc_centred ? cf - 0.5 * bw : cf - 0.5 * bw + 0.5 * bw / double (nchan);
  return base + double (ichan) * bw / double (nchan);
}

// Response.C:998-1050 doswap on a single-pol complex buffer of nchan*ndat
template <typename T>
void doswap (std::complex<T>* buf, unsigned nchan, unsigned ndat, unsigned divisions)
{
  // half_npts counts complex values here (the reference counts floats)
  const uint64_t half = uint64_t (ndat) * nchan / (2 * divisions);
  for (unsigned d = 0; d < divisions; d++)
  {
    std::complex<T>* p1 = buf + uint64_t (d) * 2 * half;
    std::complex<T>* p2 = p1 + half;
    for (uint64_t i = 0; i < half; i++) std::swap (p1[i], p2[i]);
  }
}

// Response.C:325-400 swap_as_needed, for the states this path meets
template <typename T>
void swap_as_needed (std::complex<T>* buf, unsigned nchan, unsigned ndat,
                     int input_nchan, int dual_sideband, int dc_centred)
{
  if (input_nchan == 1)
  {
    if (dual_sideband > 0)
      doswap (buf, nchan, ndat, 1);
    unsigned subswap = std::abs (dual_sideband);
    if (subswap > 1)
      doswap (buf, nchan, ndat, subswap);
  }
  else
  {
    if (dc_centred)
    {
      // Response::rotate(-ndat/2) within each channel
      for (unsigned c = 0; c < nchan; c++)
        std::rotate (buf + uint64_t (c) * ndat, buf + uint64_t (c) * ndat + ndat / 2,
                     buf + uint64_t (c + 1) * ndat);
    }
    if (dual_sideband && unsigned (input_nchan) == nchan)
      doswap (buf, nchan, ndat, nchan);
  }
}

// Restatement of the missing PlasmaResponse::build template (called at
// Dedispersion.C:128) with Dedispersion::build_compute (Dedispersion.C:166-186)
// and interchannel_fractional_sample_delay = 0 (no SampleDelay).
// Channel centres follow Observation.C:521-534; within a channel the ndat
// frequency bins run low to high from -chanwidth/2, spanning the channel.
void dedispersion_phases (double cf, double bw, double dm, unsigned nchan,
                          unsigned ndat, bool dc_centred, std::vector<double>& phase)
{
  const double chanwidth = bw / double (nchan);
  const double binwidth = chanwidth / double (ndat);
  const double sign = bw / std::fabs (bw);
  const double dispersion_per_MHz = 1e6 * dm / dm_dispersion;
  phase.resize (uint64_t (nchan) * ndat);
  for (unsigned ichan = 0; ichan < nchan; ichan++)
  {
    const double chan_freq = channel_centre (cf, bw, nchan, ichan, dc_centred);
    const double coeff = -sign * 2 * M_PI * dispersion_per_MHz / sqr (chan_freq);
    for (unsigned ipt = 0; ipt < ndat; ipt++)
    {
      const double freq = double (ipt) * binwidth - 0.5 * chanwidth;
      const double delay_phase = -2.0 * M_PI * freq * 0.0;
      phase[uint64_t (ichan) * ndat + ipt] = coeff * sqr (freq) / (chan_freq + freq) + delay_phase;
    }
  }
}

template <typename T>
uint64_t convolve (const T* in, uint64_t ndat, uint64_t in_span, int nchan, int npol,
                   const T* response, unsigned nfft, unsigned nfilt_pos, unsigned nfilt_neg,
                   T* out, uint64_t out_span, int nthreads, const T* window = nullptr)
{
  typedef std::complex<T> C;
  const uint64_t nsamp_overlap = nfilt_pos + nfilt_neg;
  const uint64_t nsamp_step = nfft - nsamp_overlap;
  uint64_t npart = 0;
  if (ndat >= nfft)
    npart = (ndat - nsamp_overlap) / nsamp_step;   // Convolution.C:486-487
  const int64_t ntask = int64_t (nchan) * npol * npart;
  (void) nthreads;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    std::vector<C> spectrum (nfft), complex_time (nfft), windowed (window ? nfft : 0);
#pragma omp for schedule(static)
    for (int64_t task = 0; task < ntask; task++)
    {
      const uint64_t ipart = uint64_t (task) % npart;
      const int ipol = int ((uint64_t (task) / npart) % npol);
      const int ichan = int (uint64_t (task) / npart / npol);
      const C* ptr = reinterpret_cast<const C*> (in) + (uint64_t (ichan) * npol + ipol) * in_span
                     + ipart * nsamp_step;
      if (window)
      {
        // Apodization::operate on the part (Convolution.C:739-743)
        for (unsigned i = 0; i < nfft; i++)
          windowed[i] = C (ptr[i].real () * window[i], ptr[i].imag () * window[i]);
        ptr = windowed.data ();
      }
      fft<T> (nfft, -1, ptr, spectrum.data ());
      // Response::operate (Response.C:662-726)
      const C* f = reinterpret_cast<const C*> (response) + uint64_t (ichan) * nfft;
      for (unsigned k = 0; k < nfft; k++)
      {
        const T d_r = spectrum[k].real (), d_i = spectrum[k].imag ();
        const T f_r = f[k].real (), f_i = f[k].imag ();
        spectrum[k] = C (f_r * d_r - f_i * d_i, f_i * d_r + f_r * d_i);
      }
      fft<T> (nfft, +1, spectrum.data (), complex_time.data ());
      C* o = reinterpret_cast<C*> (out) + (uint64_t (ichan) * npol + ipol) * out_span
             + ipart * nsamp_step;
      std::memcpy (o, complex_time.data () + nfilt_pos, nsamp_step * sizeof (C));
    }
  }
  return npart;
}

template <typename T>
int detect (const T* in, uint64_t ndat, uint64_t in_span, int nchan, int state,
            T* out, uint64_t out_span)
{
  const int nout = state == 0 ? 1 : state == 1 ? 2 : 4;
  for (int c = 0; c < nchan; c++)
  {
    const T* p = in + 2 * (uint64_t (c) * 2 + 0) * in_span;
    const T* q = in + 2 * (uint64_t (c) * 2 + 1) * in_span;
    T* o[4];
    for (int k = 0; k < nout; k++) o[k] = out + (uint64_t (c) * nout + k) * out_span;
    for (uint64_t j = 0; j < ndat; j++)
    {
      const T p_r = p[2 * j], p_i = p[2 * j + 1], q_r = q[2 * j], q_i = q[2 * j + 1];
      if (state == 0)
      {
        // Detection.C:253-301 (FPT, Intensity): accumulation in this order
        T v = p_r * p_r;
        v += p_i * p_i;
        v += q_r * q_r;
        v += q_i * q_i;
        o[0][j] = v;
      }
      else if (state == 1)
      {
        T v = p_r * p_r; v += p_i * p_i; o[0][j] = v;
        T w = q_r * q_r; w += q_i * q_i; o[1][j] = w;
      }
      else if (state == 2)
      {
        // cross_detect.ic:38-41
        o[0][j] = p_r * p_r + p_i * p_i;
        o[1][j] = q_r * q_r + q_i * q_i;
        o[2][j] = p_r * q_r + p_i * q_i;
        o[3][j] = p_r * q_i - p_i * q_r;
      }
      else
      {
        // stokes_detect.ic:40-43
        const T pp = p_r * p_r + p_i * p_i;
        const T qq = q_r * q_r + q_i * q_i;
        o[0][j] = pp + qq;
        o[1][j] = pp - qq;
        o[2][j] = T (2.0 * (p_r * q_r + p_i * q_i));
        o[3][j] = T (2.0 * (p_r * q_i - p_i * q_r));
      }
    }
  }
  return nout;
}

template <typename T>
void fold_accumulate (const T* in, uint64_t ndat, uint64_t in_span, int nchan, int npol,
                      int ndim, const uint32_t* binplan, unsigned nbin, T* profiles,
                      uint32_t* hits)
{
  // Fold.C:893-931 (FPT); hits counted once per sample (Fold.C:829-835)
  for (uint64_t idat = 0; idat < ndat; idat++)
    if (binplan[idat] < nbin) hits[binplan[idat]]++;
  for (int c = 0; c < nchan; c++)
    for (int p = 0; p < npol; p++)
    {
      const T* timep = in + (uint64_t (c) * npol + p) * in_span;
      T* phasep = profiles + (uint64_t (c) * npol + p) * nbin * ndim;
      for (uint64_t idat = 0; idat < ndat; idat++)
      {
        if (binplan[idat] != nbin)
        {
          T* ph = phasep + uint64_t (binplan[idat]) * ndim;
          for (int d = 0; d < ndim; d++) ph[d] += timep[d];
        }
        timep += ndim;
      }
    }
}

} // namespace

extern "C" {

void orc_fft_f32 (int n, int sign, const float* in, float* out)
{
  fft<float> (n, sign, reinterpret_cast<const std::complex<float>*> (in),
              reinterpret_cast<std::complex<float>*> (out));
}

void orc_fft_f64 (int n, int sign, const double* in, double* out)
{
  fft<double> (n, sign, reinterpret_cast<const std::complex<double>*> (in),
               reinterpret_cast<std::complex<double>*> (out));
}

// BitTable.C:172-225 with nbit = 8, zero_is_a_threshold = true.
// NormalDistribution::cumulative_distribution(x) = (1 + erf(x/sqrt 2)) / 2.
void orc_bittable8 (double input_spacing, int twos_complement, float* lut, double* scale_out)
{
  const unsigned unique_values = 256;
  float values[256];
  const double output_spacing = 1.0 / double (unique_values);
  const double output_middle = double (unique_values - 1) / 2.0;
  const unsigned input_middle = unique_values / 2;
  const unsigned input_offset = twos_complement ? unique_values / 2 : 0;
  double cumulative_probability = 0.0, variance = 0.0;
  for (unsigned i = 0; i < unique_values; i++)
  {
    double output = (double (i) - output_middle) * output_spacing;
    values[(i + input_offset) % unique_values] = output;
    if (i < input_middle)
    {
      double threshold = double (int (i + 1) - int (input_middle)) * input_spacing;
      double cumulative = 0.5 * (1.0 + std::erf (threshold / std::sqrt (2.0)));
      double interval = cumulative - cumulative_probability;
      cumulative_probability = cumulative;
      variance += output * output * interval;
    }
  }
  variance *= 2.0;
  double scale = 1.0 / std::sqrt (variance);
  for (unsigned i = 0; i < unique_values; i++)
    values[i] *= scale;
  scale *= output_spacing;
  // BitTable::generate with values_per_byte = 1, no bit reversal: table[b] = values[b]
  for (unsigned b = 0; b < 256; b++) lut[b] = values[b];
  if (scale_out) *scale_out = scale;
}

// BitUnpacker.C:97-138 with EightBitUnpacker::unpack_bits (EightBitUnpacker.C:25-49)
void orc_unpack8 (const uint8_t* in, uint64_t ndat, int nchan, int npol, int ndim,
                  const float* lut, float* out, uint64_t out_span)
{
  const unsigned nskip = npol * nchan * ndim;
  unsigned offset = 0;
  for (int c = 0; c < nchan; c++)
    for (int p = 0; p < npol; p++)
      for (int d = 0; d < ndim; d++)
      {
        const uint8_t* from = in + offset;
        float* into = out + (uint64_t (c) * npol + p) * out_span + d;
        for (uint64_t idat = 0; idat < ndat; idat++)
        {
          *into = lut[*from];
          from += nskip;
          into += ndim;
        }
        offset++;
      }
}

// SixteenBitUnpacker.C:23-79
void orc_unpack16 (const int16_t* in, uint64_t ndat, int nchan, int npol, int ndim,
                   int offset_binary, float* out, uint64_t out_span)
{
  const unsigned nskip = npol * nchan * ndim;
  unsigned offset = 0;
  for (int c = 0; c < nchan; c++)
    for (int p = 0; p < npol; p++)
      for (int d = 0; d < ndim; d++)
      {
        const int16_t* from = in + offset;
        float* into = out + (uint64_t (c) * npol + p) * out_span + d;
        for (uint64_t idat = 0; idat < ndat; idat++)
        {
          int16_t v = *from;
          if (offset_binary) v = int16_t (v ^ 0x8000);
          *into = float (v) + 0.5;
          from += nskip;
          into += ndim;
        }
        offset++;
      }
}

// PlasmaResponse.C:161-250 (smearing_time(half), smearing_samples) with the
// default 10% smearing buffer and all channels supported.
unsigned orc_smearing_samples (double centre_frequency, double bandwidth, double dm,
                               unsigned nchan, int half)
{
  double abs_bw = std::fabs (bandwidth);
  double ch_abs_bw = abs_bw / double (nchan);
  double lower_ch_cfreq = centre_frequency - (abs_bw - ch_abs_bw) / 2.0;
  if (half)
  {
    ch_abs_bw /= 2.0;
    lower_ch_cfreq += double (half) * ch_abs_bw;
  }
  // smearing_time (cfreq, bw) = delay_time (cfreq - |bw/2|, cfreq + |bw/2|)
  double f1 = lower_ch_cfreq - std::fabs (0.5 * ch_abs_bw);
  double f2 = lower_ch_cfreq + std::fabs (0.5 * ch_abs_bw);
  double tsmear = delay_time (dm, f1) - delay_time (dm, f2);
  double sampling_rate = std::fabs (bandwidth) / double (nchan) * 1e6;
  tsmear *= (1.0 + double (0.1f));   // smearing_buffer is a float (PlasmaResponse.C:20)
  return unsigned (std::ceil (tsmear * sampling_rate));
}

// Response.C:529-545
unsigned orc_minimum_ndat (unsigned impulse_pos, unsigned impulse_neg)
{
  double impulse_tot = impulse_pos + impulse_neg;
  if (impulse_tot == 0) return 0;
  unsigned min = unsigned (std::pow (2.0, std::ceil (std::log (impulse_tot) / std::log (2.0))));
  while (min <= impulse_tot) min *= 2;
  return min;
}

// optimize_fft.c:64-135
int64_t orc_optimal_fft_length (uint64_t nbadperfft, uint64_t nfft_max, unsigned factor)
{
  if (!nbadperfft) return -1;
  uint64_t nfft_min = factor;
  while (nbadperfft > nfft_min) nfft_min *= 2;
  if (nfft_max && nfft_max < nfft_min) return -1;
  uint64_t nfft = nfft_min;
  double order_fft = (double) nfft * std::log ((double) nfft);
  double timescale = order_fft / (double) (nfft - nbadperfft);
  while (nfft_max == 0 || nfft * 2 < nfft_max)
  {
    double prev_timescale = timescale;
    nfft *= 2;
    order_fft = (double) nfft * std::log ((double) nfft);
    timescale = order_fft / (double) (nfft - nbadperfft);
    if (timescale > prev_timescale) { nfft /= 2; break; }
  }
  return (int64_t) nfft;
}

void orc_dedispersion_response (double cf, double bw, double dm, unsigned nchan,
                                unsigned ndat, int input_nchan, int dual_sideband,
                                int dc_centred, int mode, unsigned norm_nfft, float* out)
{
  std::vector<double> phase;
  dedispersion_phases (cf, bw, dm, nchan, ndat, dc_centred != 0 && input_nchan > 1, phase);
  std::complex<float>* h = reinterpret_cast<std::complex<float>*> (out);
  const uint64_t npt = uint64_t (nchan) * ndat;
  for (uint64_t i = 0; i < npt; i++)
  {
    if (mode == 0)
    {
      // Dedispersion.C:104-111: vector<float> phases, polar(float(1.0), phase)
      const float ph = float (phase[i]);
      h[i] = std::complex<float> (std::cos (ph), std::sin (ph));
    }
    else
    {
      // double phase, reduced modulo 2 pi in double, one rounding to float
      const double ph = phase[i] - 2.0 * M_PI * std::nearbyint (phase[i] / (2.0 * M_PI));
      h[i] = std::complex<float> (float (std::cos (ph)), float (std::sin (ph)));
    }
  }
  swap_as_needed (h, nchan, ndat, input_nchan, dual_sideband, dc_centred);
  // ScalarFilter (ScalarFilter.C:29-40) appended by Convolution::prepare_normalizer
  const float s = float (1.0 / std::sqrt (double (norm_nfft)));
  for (uint64_t i = 0; i < npt; i++)
    h[i] = std::complex<float> (h[i].real () * s, h[i].imag () * s);
}

void orc_dedispersion_response_f64 (double cf, double bw, double dm, unsigned nchan,
                                    unsigned ndat, int input_nchan, int dual_sideband,
                                    int dc_centred, unsigned norm_nfft, double* out)
{
  std::vector<double> phase;
  dedispersion_phases (cf, bw, dm, nchan, ndat, dc_centred != 0 && input_nchan > 1, phase);
  std::complex<double>* h = reinterpret_cast<std::complex<double>*> (out);
  const uint64_t npt = uint64_t (nchan) * ndat;
  const double s = 1.0 / std::sqrt (double (norm_nfft));
  for (uint64_t i = 0; i < npt; i++)
    h[i] = std::complex<double> (std::cos (phase[i]) * s, std::sin (phase[i]) * s);
  swap_as_needed (h, nchan, ndat, input_nchan, dual_sideband, dc_centred);
}

// TestResponse.cpp:30-165 with Apodization::Tukey (Apodization.C:123-146)
void orc_tukey_response (unsigned impulse_neg, unsigned impulse_pos, unsigned ndat,
                         float* spectral_out, float* temporal_out)
{
  const unsigned size = impulse_neg + impulse_pos;
  std::vector<float> amp (size);
  {
    float denom_start = 2 * impulse_neg;
    float denom_end = 2 * impulse_pos;
    for (unsigned idat = 0; idat < size; idat++)
    {
      if (idat < impulse_neg)
        amp[idat] = 0.5 * (1 - std::cos (2.0 * M_PI * float (idat) / denom_start));
      else if (idat + 1 > size - impulse_pos)
        amp[idat] = 0.5 * (1 - std::cos (2.0 * M_PI * float (size - idat - 1) / denom_end));
      else
        amp[idat] = 1.0;
    }
  }
  std::vector<std::complex<float>> temporal (size);
  std::complex<double> sum_temporal = 0.0;
  std::vector<float> correction (size);
  double sum_correction = 0.0;
  for (unsigned idat = 0; idat < size; idat++)
  {
    double phase = 2.0 * M_PI * double (idat) / double (size);
    temporal[idat] = amp[idat] * std::complex<float> (std::cos (phase), std::sin (phase));
    sum_temporal += std::complex<double> (temporal[idat]);
    correction[idat] = std::sin (0.5 * phase);
    sum_correction += correction[idat];
  }
  auto mean_offset = sum_temporal / sum_correction;
  for (unsigned idat = 0; idat < size; idat++)
  {
    std::complex<double> t = std::complex<double> (temporal[idat]) - mean_offset * double (correction[idat]);
    temporal[idat] = std::complex<float> (t);
  }
  std::vector<std::complex<float>> padded (ndat, 0.0f);
  for (unsigned idat = 0; idat < impulse_pos; idat++)
    padded[idat] = temporal[idat + impulse_neg];
  const unsigned offset = ndat - impulse_neg;
  for (unsigned idat = 0; idat < impulse_neg; idat++)
    padded[idat + offset] = temporal[idat];
  std::complex<float>* spectral = reinterpret_cast<std::complex<float>*> (spectral_out);
  fft<float> (ndat, -1, padded.data (), spectral);
  float scalefac = 1.0 / std::sqrt (ndat);
  for (unsigned idat = 0; idat < ndat; idat++)
    spectral[idat] *= scalefac;
  std::memcpy (temporal_out, temporal.data (), size * sizeof (std::complex<float>));
}

double orc_channel_centre (double cf, double bw, unsigned nchan, unsigned ichan, int swap,
                           int dc_centred)
{
  // Observation::get_unswapped_ichan (Observation.C:495-518), swap only
  unsigned ch = ichan;
  if (swap) ch = (ch + nchan / 2) % nchan;
  return channel_centre (cf, bw, nchan, ch, dc_centred != 0);
}

} // extern "C"

namespace {
template <typename T>
void response_channels (const double* chan_freq, unsigned nchan, double bw, double dm,
                        unsigned ndat, int mode, unsigned norm_nfft, std::complex<T>* h,
                        const double* frac_delay_us = nullptr, bool swap_halves = true,
                        double norm = 0.0)
{
  const double chanwidth = bw / double (nchan);
  const double binwidth = chanwidth / double (ndat);
  const double sign = bw / std::fabs (bw);
  const double dispersion_per_MHz = 1e6 * dm / dm_dispersion;
  const double nrm = norm > 0 ? norm : double (norm_nfft);
  const T s = sizeof (T) == 4 ? T (float (1.0 / std::sqrt (nrm))) : T (1.0 / std::sqrt (nrm));
  for (unsigned c = 0; c < nchan; c++)
  {
    const double f0 = chan_freq[c];
    const double coeff = -sign * 2 * M_PI * dispersion_per_MHz / sqr (f0);
    // Dedispersion::build_setup / build_compute (Dedispersion.C:141-187): the
    // fractional-sample inter-channel delay, microseconds
    const double fd = frac_delay_us ? frac_delay_us[c] : 0.0;
    for (unsigned k = 0; k < ndat; k++)
    {
      // FFT-order bin k holds natural bin (k + ndat/2) mod ndat when each
      // channel is swapped; the filterbank's response keeps natural order
      const unsigned ipt = swap_halves ? (k + ndat / 2) % ndat : k;
      const double freq = double (ipt) * binwidth - 0.5 * chanwidth;
      const double phase = coeff * sqr (freq) / (f0 + freq) + (-2.0 * M_PI * freq * fd);
      std::complex<T>& o = h[uint64_t (c) * ndat + k];
      if (sizeof (T) == 8)
        o = std::complex<T> (T (std::cos (phase) * s), T (std::sin (phase) * s));
      else if (mode == 0)
      {
        const float ph = float (phase);
        o = std::complex<T> (T (std::cos (ph) * float (s)), T (std::sin (ph) * float (s)));
      }
      else
      {
        const double ph = phase - 2.0 * M_PI * std::nearbyint (phase / (2.0 * M_PI));
        o = std::complex<T> (T (float (std::cos (ph)) * float (s)),
                             T (float (std::sin (ph)) * float (s)));
      }
    }
  }
}

template <typename T>
uint64_t filterbank (const T* in, uint64_t ndat, uint64_t in_span, int nchan_in, int npol,
                     unsigned nsub, T* out, uint64_t out_span)
{
  typedef std::complex<T> C;
  const uint64_t npart = ndat / nsub;
  // Filterbank::prepare_normalizer(1/sqrt(nsamp_fft * freq_res)), freq_res = 1,
  // applied as a complex<float> product with (s, 0) by Response::operate
  const T s = T (1.0 / std::sqrt (double (nsub)));
  std::vector<C> spec (nsub);
  for (int ic = 0; ic < nchan_in; ic++)
    for (uint64_t ipart = 0; ipart < npart; ipart++)
      for (int p = 0; p < npol; p++)
      {
        const C* x = reinterpret_cast<const C*> (in) + (uint64_t (ic) * npol + p) * in_span
                     + ipart * nsub;
        fft<T> (int (nsub), -1, x, spec.data ());
        for (unsigned k = 0; k < nsub; k++)
        {
          const T d_r = spec[k].real (), d_i = spec[k].imag ();
          C* o = reinterpret_cast<C*> (out) + ((uint64_t (ic) * nsub + k) * npol + p) * out_span;
          o[ipart] = C (s * d_r - T (0) * d_i, T (0) * d_r + s * d_i);
        }
      }
  return npart;
}
// Filterbank with a response, the "During" form (-F nchan:D):
// Filterbank::do_prepare (Filterbank.C:98-198) sizes nsamp_fft = nsub *
// freq_res (complex input), nsamp_overlap = nfilt_tot * nsub and nsamp_step =
// nsamp_fft - nsamp_overlap; Filterbank::resize_output (Filterbank.C:398-420)
// npart = (ndat - nsamp_overlap) / nsamp_step; FilterbankEngineCPU::perform
// (FilterbankEngineCPU.C:379-535): forward FFT of each part, Response::operate
// over the nsub channels of the input channel (Response.C:662-726), then per
// output channel a backward FFT of freq_res points and the nkeep samples from
// nfilt_pos.  response: [nchan_in*nsub][freq_res] complex, normaliser applied.
template <typename T>
uint64_t filterbank_during (const T* in, uint64_t ndat, uint64_t in_span, int nchan_in, int npol,
                            unsigned nsub, unsigned freq_res, unsigned nfilt_pos,
                            unsigned nfilt_neg, const T* response, T* out, uint64_t out_span,
                            const float* temporal = nullptr, const float* spectral = nullptr)
{
  typedef std::complex<T> C;
  const uint64_t nsamp_fft = uint64_t (nsub) * freq_res;
  const unsigned nfilt_tot = nfilt_pos + nfilt_neg;
  const uint64_t overlap = uint64_t (nfilt_tot) * nsub;
  const uint64_t step = nsamp_fft - overlap;
  const uint64_t npart = ndat > overlap ? (ndat - overlap) / step : 0;
  const unsigned nkeep = freq_res - nfilt_tot;
  const C* resp = reinterpret_cast<const C*> (response);
  std::vector<C> spec (nsamp_fft), tmp (freq_res), win;
  for (int ic = 0; ic < nchan_in; ic++)
    for (uint64_t ipart = 0; ipart < npart; ipart++)
      for (int p = 0; p < npol; p++)
      {
        const C* x = reinterpret_cast<const C*> (in) + (uint64_t (ic) * npol + p) * in_span
                     + ipart * step;
        if (temporal)
        {
          // Apodization::operate before the forward FFT (FilterbankEngineCPU.C:447-449)
          win.resize (nsamp_fft);
          for (uint64_t k = 0; k < nsamp_fft; k++)
            win[k] = C (x[k].real () * T (temporal[k]), x[k].imag () * T (temporal[k]));
          x = win.data ();
        }
        fft<T> (int (nsamp_fft), -1, x, spec.data ());
        const C* h = resp + uint64_t (ic) * nsamp_fft;
        for (uint64_t k = 0; k < nsamp_fft; k++)
        {
          const T d_r = spec[k].real (), d_i = spec[k].imag ();
          const T f_r = h[k].real (), f_i = h[k].imag ();
          spec[k] = C (f_r * d_r - f_i * d_i, f_i * d_r + f_r * d_i);
        }
        for (unsigned cs = 0; cs < nsub; cs++)
        {
          C* chan = spec.data () + uint64_t (cs) * freq_res;
          if (spectral)
            // Apodization::operate on the channel's spectrum (FilterbankEngineCPU.C:507-509)
            for (unsigned f = 0; f < freq_res; f++)
              chan[f] = C (chan[f].real () * T (spectral[f]), chan[f].imag () * T (spectral[f]));
          fft<T> (int (freq_res), +1, chan, tmp.data ());
          C* o = reinterpret_cast<C*> (out) + ((uint64_t (ic) * nsub + cs) * npol + p) * out_span
                 + ipart * nkeep;
          for (unsigned i = 0; i < nkeep; i++) o[i] = tmp[nfilt_pos + i];
        }
      }
  return npart;
}

} // namespace

extern "C" {

void orc_dedispersion_response_channels (const double* chan_freq, unsigned nchan, double bw,
                                         double dm, unsigned ndat, int mode, unsigned norm_nfft,
                                         float* out)
{
  response_channels<float> (chan_freq, nchan, bw, dm, ndat, mode, norm_nfft,
                            reinterpret_cast<std::complex<float>*> (out));
}

void orc_dedispersion_response_channels_delay (const double* chan_freq, unsigned nchan,
                                               double bw, double dm, unsigned ndat, int mode,
                                               unsigned norm_nfft, const double* frac_delay_us,
                                               float* out)
{
  response_channels<float> (chan_freq, nchan, bw, dm, ndat, mode, norm_nfft,
                            reinterpret_cast<std::complex<float>*> (out), frac_delay_us);
}

// The response of the filterbank with a response: channels centred at
// chan_freq, each in natural frequency order (no per-channel swap), scaled by
// 1/sqrt(norm) with norm = nsamp_fft * freq_res.
void orc_dedispersion_response_during (const double* chan_freq, unsigned nchan, double bw,
                                       double dm, unsigned ndat, int mode, double norm,
                                       float* out)
{
  response_channels<float> (chan_freq, nchan, bw, dm, ndat, mode, 1,
                            reinterpret_cast<std::complex<float>*> (out), nullptr, false, norm);
}

void orc_dedispersion_response_during_f64 (const double* chan_freq, unsigned nchan, double bw,
                                           double dm, unsigned ndat, double norm, double* out)
{
  response_channels<double> (chan_freq, nchan, bw, dm, ndat, 1, 1,
                             reinterpret_cast<std::complex<double>*> (out), nullptr, false, norm);
}

uint64_t orc_filterbank_during_f32 (const float* in, uint64_t ndat, uint64_t in_span,
                                    int nchan_in, int npol, unsigned nsub, unsigned freq_res,
                                    unsigned nfilt_pos, unsigned nfilt_neg, const float* response,
                                    float* out, uint64_t out_span, const float* temporal,
                                    const float* spectral)
{
  return filterbank_during<float> (in, ndat, in_span, nchan_in, npol, nsub, freq_res, nfilt_pos,
                                   nfilt_neg, response, out, out_span, temporal, spectral);
}

uint64_t orc_filterbank_during_f64 (const double* in, uint64_t ndat, uint64_t in_span,
                                    int nchan_in, int npol, unsigned nsub, unsigned freq_res,
                                    unsigned nfilt_pos, unsigned nfilt_neg, const double* response,
                                    double* out, uint64_t out_span, const float* temporal,
                                    const float* spectral)
{
  return filterbank_during<double> (in, ndat, in_span, nchan_in, npol, nsub, freq_res, nfilt_pos,
                                    nfilt_neg, response, out, out_span, temporal, spectral);
}

void orc_dedispersion_response_channels_f64 (const double* chan_freq, unsigned nchan, double bw,
                                             double dm, unsigned ndat, unsigned norm_nfft,
                                             double* out)
{
  response_channels<double> (chan_freq, nchan, bw, dm, ndat, 1, norm_nfft,
                             reinterpret_cast<std::complex<double>*> (out));
}

uint64_t orc_filterbank_f32 (const float* in, uint64_t ndat, uint64_t in_span, int nchan_in,
                             int npol, unsigned nsub, float* out, uint64_t out_span)
{
  return filterbank<float> (in, ndat, in_span, nchan_in, npol, nsub, out, out_span);
}

uint64_t orc_filterbank_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan_in,
                             int npol, unsigned nsub, double* out, uint64_t out_span)
{
  return filterbank<double> (in, ndat, in_span, nchan_in, npol, nsub, out, out_span);
}

uint64_t orc_convolve_f32 (const float* in, uint64_t ndat, uint64_t in_span, int nchan,
                           int npol, const float* response, unsigned nfft, unsigned nfilt_pos,
                           unsigned nfilt_neg, float* out, uint64_t out_span, int nthreads)
{
  return convolve<float> (in, ndat, in_span, nchan, npol, response, nfft, nfilt_pos,
                          nfilt_neg, out, out_span, nthreads);
}

uint64_t orc_convolve_window_f32 (const float* in, uint64_t ndat, uint64_t in_span, int nchan,
                                  int npol, const float* response, unsigned nfft,
                                  unsigned nfilt_pos, unsigned nfilt_neg, float* out,
                                  uint64_t out_span, int nthreads, const float* window)
{
  return convolve<float> (in, ndat, in_span, nchan, npol, response, nfft, nfilt_pos,
                          nfilt_neg, out, out_span, nthreads, window);
}

// Apodization::build (Apodization.C:60-146): window types 0 top hat, 1
// Hanning, 2 Welch, 3 Bartlett, 4 Tukey; swap exchanges halves (:168-178)
int orc_apodization (int type, unsigned ndat, unsigned transition_start,
                     unsigned transition_end, int swap, float* buffer)
{
  if (!ndat) return -1;
  for (unsigned idat = 0; idat < ndat; idat++)
  {
    if (type == 0)
      buffer[idat] = 1.0;
    else if (type == 1)
    {
      double denom = ndat - 1.0;
      buffer[idat] = 0.5 * (1 - cos (2.0 * M_PI * double (idat) / denom));
    }
    else if (type == 2)
    {
      float centre = 0.5 * (ndat - 1);
      float denominator = 0.5 * (ndat + 1);
      float tosquare = (float (idat) - centre) / denominator;
      buffer[idat] = 1.0 - tosquare * tosquare;
    }
    else if (type == 3)
    {
      float centre = 0.5 * (ndat - 1);
      float denominator = 0.5 * (ndat - 1);
      buffer[idat] = 1.0 - fabs ((float (idat) - centre) / denominator);
    }
    else if (type == 4)
    {
      float denom_start = 2 * transition_start;
      float denom_end = 2 * transition_end;
      if (idat < transition_start)
        buffer[idat] = 0.5 * (1 - cos (2.0 * M_PI * float (idat) / denom_start));
      else if (idat + 1 > ndat - transition_end)
        buffer[idat] = 0.5 * (1 - cos (2.0 * M_PI * float (ndat - idat - 1) / denom_end));
      else
        buffer[idat] = 1.0;
    }
    else
      return -1;
  }
  if (swap)
    for (unsigned i = 0; i < ndat / 2; i++) std::swap (buffer[i], buffer[i + ndat / 2]);
  return 0;
}

uint64_t orc_convolve_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan,
                           int npol, const double* response, unsigned nfft, unsigned nfilt_pos,
                           unsigned nfilt_neg, double* out, uint64_t out_span, int nthreads)
{
  return convolve<double> (in, ndat, in_span, nchan, npol, response, nfft, nfilt_pos,
                           nfilt_neg, out, out_span, nthreads);
}

int orc_detect (const float* in, uint64_t ndat, uint64_t in_span, int nchan, int state,
                float* out, uint64_t out_span)
{
  return detect<float> (in, ndat, in_span, nchan, state, out, out_span);
}

int orc_detect_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan, int state,
                    double* out, uint64_t out_span)
{
  return detect<double> (in, ndat, in_span, nchan, state, out, out_span);
}

// Fold.C:685-693 and 975-979: phi = fmod((t - epoch).in_seconds(), P)/P - ref_phase,
// t = start_time + (idat_start + 0.5)/rate.  The MJD is (day, second, fraction of a
// second); the difference in seconds is formed from the integer parts first.
double orc_fold_phi (int64_t start_day, int64_t start_sec, double start_frac,
                     int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                     uint64_t idat_start, double rate, double period, double reference_phase)
{
  double mid_idat_start = double (idat_start) + 0.5;
  double add = mid_idat_start / rate;
  // MJD + seconds: carry whole seconds into the integer part
  double whole = std::floor (add);
  double frac = start_frac + (add - whole);
  int64_t sec = start_sec + int64_t (whole);
  if (frac >= 1.0) { frac -= 1.0; sec += 1; }
  int64_t day = start_day + sec / 86400;
  sec = sec % 86400;
  double seconds = double ((day - epoch_day) * 86400 + (sec - epoch_sec)) + (frac - epoch_frac);
  return std::fmod (seconds, period) / period - reference_phase;
}

// Fold.C:790-837, the sequential FP64 recurrence
void orc_fold_binplan (double phi, double phase_per_sample, uint64_t ndat, unsigned nbin,
                       uint32_t* binplan)
{
  const double double_nbin = double (nbin);
  for (uint64_t idat = 0; idat < ndat; idat++)
  {
    phi -= std::floor (phi);
    double double_ibin = phi * double_nbin;
    unsigned ibin = unsigned (double_ibin);
    phi += phase_per_sample;
    binplan[idat] = ibin;
  }
}

void orc_fold_accumulate (const float* in, uint64_t ndat, uint64_t in_span, int nchan,
                          int npol, int ndim, const uint32_t* binplan, unsigned nbin,
                          float* profiles, uint32_t* hits)
{
  fold_accumulate<float> (in, ndat, in_span, nchan, npol, ndim, binplan, nbin, profiles, hits);
}

void orc_fold_accumulate_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan,
                              int npol, int ndim, const uint32_t* binplan, unsigned nbin,
                              double* profiles, uint32_t* hits)
{
  fold_accumulate<double> (in, ndat, in_span, nchan, npol, ndim, binplan, nbin, profiles, hits);
}

// SpectralKurtosis::compute (SpectralKurtosis.C:674-798), FPT, noverlap = 1:
// square-law detect each sample in float, accumulate S1 and S2 in double,
// store them as float.
uint64_t orc_sk_compute (const float* in, uint64_t ndat, uint64_t in_span, int nchan, int npol,
                         unsigned M, int zero_is_valid, float* sums, uint32_t* counts)
{
  const uint64_t npart = ndat / M;   // Resolution::prepare with noverlap = 1
  // every (part, chan) is independent; threads only split the outer loop
#pragma omp parallel for schedule(static)
  for (int64_t ipart = 0; ipart < int64_t (npart); ipart++)
    for (int ichan = 0; ichan < nchan; ichan++)
      for (int ipol = 0; ipol < npol; ipol++)
      {
        const float* indat = in + 2 * ((uint64_t (ichan) * npol + ipol) * in_span + ipart * M);
        double S1_sum = 0, S2_sum = 0;
        unsigned count = 0;
        for (unsigned i = 0; i < M; i++)
        {
          const float re = indat[2 * i];
          const float im = indat[2 * i + 1];
          const float sqld = (re * re) + (im * im);
          if (zero_is_valid || sqld != 0)
          {
            S1_sum += sqld;
            S2_sum += sqld * sqld;
            count++;
          }
        }
        const uint64_t o = (ipart * nchan + ichan) * npol + ipol;
        sums[2 * o] = float (S1_sum);
        sums[2 * o + 1] = float (S2_sum);
        if (ipol == 0) counts[ipart * nchan + ichan] = count;
      }
  return npart;
}

// SpectralKurtosis::detect_skfb (SpectralKurtosis.C:1105-1222), one resolution
uint64_t orc_sk_detect (const float* sums, const uint32_t* counts, uint64_t npart, int nchan,
                        int npol, unsigned Nd, float lower, float upper, uint8_t* mask)
{
  uint64_t zapped = 0;
  for (uint64_t ipart = 0; ipart < npart; ipart++)
    for (int ichan = 0; ichan < nchan; ichan++)
    {
      const unsigned Mprime = counts[ipart * nchan + ichan];
      uint8_t& out = mask[ipart * nchan + ichan];
      out = 0;
      if (Mprime == 0) continue;
      bool zap = true;
      if (Mprime > 2)
      {
        const float M_fac = (float) (Mprime * Nd + 1) / (Mprime - 1);
        zap = false;
        for (int ipol = 0; ipol < npol; ipol++)
        {
          const uint64_t o = (ipart * nchan + ichan) * npol + ipol;
          const float S1_sum = sums[2 * o];
          const float S2_sum = sums[2 * o + 1];
          const float V = M_fac * (Mprime * (S2_sum / (S1_sum * S1_sum)) - 1);
          if (V > upper || V < lower) zap = true;
        }
      }
      if (zap)
      {
        out = 1;
        zapped++;
      }
    }
  return zapped;
}

// SpectralKurtosis::mask (SpectralKurtosis.C:1465-1566), one resolution
void orc_sk_mask (const float* in, uint64_t in_span, float* out, uint64_t out_span,
                  const uint8_t* mask, uint64_t npart, int nchan, int npol, unsigned M)
{
#pragma omp parallel for schedule(static)
  for (int ichan = 0; ichan < nchan; ichan++)
    for (int ipol = 0; ipol < npol; ipol++)
    {
      const float* indat = in + 2 * (uint64_t (ichan) * npol + ipol) * in_span;
      float* outdat = out + 2 * (uint64_t (ichan) * npol + ipol) * out_span;
      for (uint64_t ipart = 0; ipart < npart; ipart++)
      {
        const bool z = mask[ipart * nchan + ichan] != 0;
        for (unsigned j = 0; j < 2 * M; j++)
          outdat[j] = z ? 0.0f : indat[j];
        indat += 2 * M;
        outdat += 2 * M;
      }
    }
}

} // extern "C"

namespace {

// Pearson IV / VI densities of the SK estimator (PearsonIV.C:37-134,
// PearsonVI.C:22-95)
struct SkDensity
{
  bool type6 = false;
  double m = 0, nu = 0, a = 0, lamda = 0, alpha = 0, beta = 0, delta = 0, logk = 0;
  double operator() (double x) const
  {
    if (type6)
    {
      x -= delta;
      if (x < 0) return 0;
      return std::exp (logk + (alpha - 1) * std::log (x) - (alpha + beta) * std::log (1 + x));
    }
    const double t = (x - lamda) / a;
    return std::exp (logk - m * std::log (1 + t * t) - nu * std::atan (t));
  }
};

// log |Gamma(x+iy)/Gamma(x)|^2 from the product prod_k (1 + y^2/(x+k)^2)^-1:
// the logs are summed for k < K with x+K >= max(1e5, 1e3 |y|), and the rest
// by Euler-Maclaurin on f(t) = y^2/(x+t)^2 - y^4/(2(x+t)^4) from D = x+K:
// y^2/D + f(D)/2 + y^2/(6D^3) - y^4/(6D^3).
double sk_log_gamma_ratio2 (double x, double y)
{
  const double y2 = y * y;
  const double dmax = std::max (1e5, 1e3 * std::fabs (y));
  double s = 0, d = x;
  for (; d < dmax; d += 1) s += std::log1p (y2 / (d * d));
  const double D = d;
  s += y2 / D + 0.5 * (y2 / (D * D)) + (y2 - y2 * y2) / (6 * D * D * D);
  return -s;
}

// Romberg integration (Romberg.h:63-104): stage j of the extended midpoint
// (step / 3) or trapezoid (step / 2) rule, polynomial extrapolation of the
// last five stages to step 0, absolute tolerance 1e-12.
template <typename F>
double sk_romberg (const F& f, double a, double b, bool midpoint)
{
  const int K = 5, JMAX = 18;
  const double ratio = midpoint ? 9.0 : 4.0;
  double h[JMAX + 1], s[JMAX];
  double stage = 0;
  h[0] = 1;
  for (int j = 0; j < JMAX; j++)
  {
    if (midpoint)
    {
      if (j == 0)
        stage = (b - a) * f (0.5 * (a + b));
      else
      {
        const double n = std::pow (3.0, j - 1);   // new points: 2 * 3^(j-1)
        const double del = (b - a) / (3 * n);
        double x = a + 0.5 * del, sum = 0;
        for (uint64_t i = 0; i < uint64_t (n); i++)
        {
          sum += f (x);
          x += 2 * del;
          sum += f (x);
          x += del;
        }
        stage = (stage + (b - a) * sum / n) / 3;
      }
    }
    else
    {
      if (j == 0)
        stage = 0.5 * (b - a) * (f (a) + f (b));
      else
      {
        const double n = std::pow (2.0, j - 1);
        const double del = (b - a) / n;
        double x = a + 0.5 * del, sum = 0;
        for (uint64_t i = 0; i < uint64_t (n); i++, x += del) sum += f (x);
        stage = 0.5 * (stage + (b - a) * sum / n);
      }
    }
    s[j] = stage;
    if (j >= K)
    {
      // Neville's algorithm at step 0 through (h, s) of stages j-K..j-1
      double p[K];
      for (int i = 0; i < K; i++) p[i] = s[j - K + i];
      double last = 0;
      for (int m = 1; m < K; m++)
        for (int i = 0; i < K - m; i++)
        {
          const double hi = h[j - K + i], hm = h[j - K + i + m];
          const double np = (hm * p[i] - hi * p[i + 1]) / (hm - hi);
          if (i == 0) last = np - p[0];
          p[i] = np;
        }
      if (std::fabs (last) <= double (1.0e-12f)) return p[0];
    }
    h[j + 1] = h[j] / ratio;
  }
  return s[JMAX - 1];
}

struct SkCumulative
{
  const SkDensity& pdf;
  // CumulativeDistribution.C:10-24: the tail beyond -1 (or +1) through u = 1/x
  double cf (double x) const
  {
    auto tail = [this] (double u) { return u == 0 ? 0.0 : pdf (-1.0 / u) / (u * u); };
    if (x < -1) return sk_romberg (tail, 0.0, -1.0 / x, true);
    return sk_romberg (tail, 0.0, 1.0, true) + sk_romberg (pdf, -1.0, x, false);
  }
  double ccf (double x) const
  {
    auto tail = [this] (double u) { return u == 0 ? 0.0 : pdf (1.0 / u) / (u * u); };
    if (x > 1) return sk_romberg (tail, 0.0, 1.0 / x, true);
    return sk_romberg (tail, 0.0, 1.0, true) + sk_romberg (pdf, x, 1.0, false);
  }
};

} // namespace

extern "C" {

// SKLimits::calc_limits (SKLimits.C:136-229) with SKLimits::parametersIV/VI
// (:71-134), NewtonRaphson.h (100 iterations, 1e-12 relative, clamped to
// 1 +- 2 sym).  The inverse error function is found by bisection.
int orc_sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest, float* lower,
                   float* upper)
{
  const double fwer = 1.0 - erf ((float) std_devs / sqrt (2));
  if (M < 2 || fwer <= 0 || ntest == 0 || Nd == 0) return -1;
  const double pcer = 1.0 - pow (1 - fwer, 1.0 / ntest);
  const double target = pcer / 2.0;
  // ierf(1 - pcer) by bisection on erf
  double lo_e = 0, hi_e = 10;
  for (int i = 0; i < 200; i++)
  {
    const double mid = 0.5 * (lo_e + hi_e);
    if (erf (mid) < 1.0 - pcer) lo_e = mid; else hi_e = mid;
  }
  const double psd = 0.5 * (lo_e + hi_e) * sqrt (2);
  if (M >= 32768)
  {
    const double factor = sqrt (4.0 / (double) M) * psd;
    *lower = (float) (1.0f - factor);
    *upper = (float) (1.0f + factor);
    return 0;
  }
  const double Mx = M, N = Nd;
  const double b = Mx / (Mx - 1);
  const double lg = lgamma (Mx * N + 2);
  const double mu2_6 = 2 * N * (N + 1) * Mx * b * exp (lg - lgamma (Mx * N + 4));
  const double mu3_6 = 8 * N * (N + 1) * Mx * b * b * exp (lg - lgamma (Mx * N + 6))
                       * ((N + 4) * Mx * N - 5 * N - 2);
  const double mu4_6 = 12 * N * (N + 1) * Mx * b * b * b * exp (lg - lgamma (Mx * N + 8))
      * ((Mx * Mx * Mx + 3 * Mx * Mx) * N * N * N * N
         + (Mx * Mx * Mx + 68 * Mx * Mx - 93 * Mx) * N * N * N
         + (125 * Mx * Mx - 245 * Mx + 84) * N * N + (48 - 32 * Mx) * N + 24);
  double mu2, beta1, beta2;
  if (Nd == 1)
  {
    mu2 = (4 * Mx * Mx) / ((Mx - 1) * (Mx + 2) * (Mx + 3));
    beta1 = 4 * (Mx + 2) * (Mx + 3) * (5 * Mx - 7) * (5 * Mx - 7)
            / ((Mx - 1) * (Mx + 4) * (Mx + 4) * (Mx + 5) * (Mx + 5));
    beta2 = 3 * (Mx + 2) * (Mx + 3) * (Mx * Mx * Mx + 98 * Mx * Mx - 185 * Mx + 78)
            / ((Mx - 1) * (Mx + 4) * (Mx + 5) * (Mx + 6) * (Mx + 7));
  }
  else
  {
    mu2 = mu2_6;
    beta1 = mu3_6 * mu3_6 / (mu2_6 * mu2_6 * mu2_6);
    beta2 = mu4_6 / (mu2_6 * mu2_6);
  }
  const double kappa = beta1 * (beta2 + 3) * (beta2 + 3)
                       / (4 * (4 * beta2 - 3 * beta1) * (2 * beta2 - 3 * beta1 - 6));
  if (kappa < 0) return -2;
  SkDensity pdf;
  if (kappa > 1)
  {
    pdf.type6 = true;
    const double root = sqrt (16 * pow (mu2_6, 4) + (4 * mu2_6 + 1) * mu3_6 * mu3_6);
    pdf.alpha = (32 * pow (mu2_6, 5) - 4 * mu3_6 * pow (mu2_6, 3)
                 + 8 * mu3_6 * mu3_6 * mu2_6 * mu2_6 + mu3_6 * mu3_6 * mu2_6 - pow (mu3_6, 3)
                 + (8 * pow (mu2_6, 3) - mu3_6 * mu2_6 + mu3_6 * mu3_6) * root)
                / pow (mu3_6, 3);
    pdf.beta = 3 + 2 * mu2_6 / (mu3_6 * mu3_6) * (4 * mu2_6 * mu2_6 + root);
    pdf.delta = (pdf.beta - pdf.alpha - 1) / (pdf.beta - 1);
    pdf.logk = lgamma (pdf.alpha + pdf.beta) - lgamma (pdf.alpha) - lgamma (pdf.beta);
  }
  else
  {
    const double r = 6 * (beta2 - beta1 - 1) / (2 * beta2 - 3 * beta1 - 6);
    pdf.m = (r + 2) / 2;
    pdf.nu = -r * (r - 2) * sqrt (beta1) / sqrt (16 * (r - 1) - beta1 * (r - 2) * (r - 2));
    pdf.a = 0.25 * sqrt (mu2 * (16 * (r - 1) - beta1 * (r - 2) * (r - 2)));
    pdf.lamda = 1 - 0.25 * (r - 2) * sqrt (mu2) * sqrt (beta1);
    pdf.logk = sk_log_gamma_ratio2 (pdf.m, 0.5 * pdf.nu) - log (pdf.a)
               - (lgamma (pdf.m - 0.5) + 0.5 * log (M_PI) - lgamma (pdf.m));
  }
  const SkCumulative cdf {pdf};
  const double sym = sqrt (mu2) * psd;
  const double xmin = 1 - 2 * sym, xmax = 1 + 2 * sym;
  for (int side = 0; side < 2; side++)
  {
    double x = side == 0 ? 1 - sym : 1 + sym;
    const double guess = x;
    bool ok = false;
    for (unsigned it = 0; it < 100 && !ok; it++)
    {
      const double c = side == 0 ? cdf.cf (x) : cdf.ccf (x);
      const double dlog = (side == 0 ? pdf (x) : -pdf (x)) / c;
      const double dx = (log (c) - log (target)) / dlog;
      x -= dx;
      if (x < xmin) x = xmin;
      if (x > xmax) x = xmax;
      ok = dx * dx <= (x * 1e-12) * (x * 1e-12);
    }
    const double t = ok ? x : guess;
    if (side == 0) *lower = (float) t; else *upper = (float) t;
  }
  return 0;
}

} // extern "C"

namespace {

// FFT of any length 2^a 3^b (FFTW conventions, unnormalised): recursive
// decimation in time by 2 or 3, twiddles from double; plain DFT otherwise.
// Power-of-two lengths go to the radix-2 routine above.
template <typename T>
void fft_any (int n, int sign, const std::complex<T>* in, std::complex<T>* out)
{
  typedef std::complex<T> C;
  if ((n & (n - 1)) == 0)
  {
    fft<T> (n, sign, in, out);
    return;
  }
  const int r = n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n;
  if (r == n)
  {
    for (int k = 0; k < n; k++)
    {
      std::complex<double> acc (0, 0);
      for (int j = 0; j < n; j++)
      {
        const double a = sign * 2.0 * M_PI * double ((int64_t (j) * k) % n) / double (n);
        acc += std::complex<double> (in[j].real (), in[j].imag ()) *
               std::complex<double> (std::cos (a), std::sin (a));
      }
      out[k] = C (T (acc.real ()), T (acc.imag ()));
    }
    return;
  }
  const int m = n / r;
  std::vector<C> sub (n), res (n);
  for (int q = 0; q < r; q++)
  {
    for (int j = 0; j < m; j++) sub[q * m + j] = in[j * r + q];
    fft_any<T> (m, sign, sub.data () + q * m, res.data () + q * m);
  }
  for (int k = 0; k < m; k++)
  {
    C t[3];
    for (int q = 0; q < r; q++)
    {
      const double a = sign * 2.0 * M_PI * double (int64_t (q) * k) / double (n);
      const C w (T (std::cos (a)), T (std::sin (a)));
      const C v = res[q * m + k];
      t[q] = C (v.real () * w.real () - v.imag () * w.imag (),
                v.real () * w.imag () + v.imag () * w.real ());
    }
    for (int p = 0; p < r; p++)
    {
      C acc = t[0];
      for (int q = 1; q < r; q++)
      {
        const double a = sign * 2.0 * M_PI * double ((p * q) % r) / double (r);
        const C w (T (std::cos (a)), T (std::sin (a)));
        acc += C (t[q].real () * w.real () - t[q].imag () * w.imag (),
                  t[q].real () * w.imag () + t[q].imag () * w.real ());
      }
      out[p * m + k] = acc;
    }
  }
}

// InverseFilterbankEngineCPU::build_fine_channel_plan (InverseFilterbankEngineCPU.C:378-425):
// input channel feeding stitched position ichan when several coarse channels
// are combined into one output channel.
std::vector<unsigned> ifb_fine_channel_plan (unsigned input_nchan, unsigned fine_per_coarse)
{
  std::vector<unsigned> idx (input_nchan), plan (input_nchan);
  const unsigned half_band = input_nchan / 2, half_coarse = fine_per_coarse / 2;
  for (unsigned i = 0; i < input_nchan; i++) idx[i] = (i + input_nchan - half_coarse) % input_nchan;
  for (unsigned i = 0; i < half_band; i++) std::swap (idx[i], idx[i + half_band]);
  for (unsigned ic = 0; ic < input_nchan / fine_per_coarse; ic++)
    for (unsigned i = ic * fine_per_coarse; i < ic * fine_per_coarse + half_coarse; i++)
      std::swap (idx[i], idx[i + half_coarse]);
  for (unsigned i = 0; i < input_nchan; i++) plan[idx[i]] = i;
  return plan;
}

// InverseFilterbankEngineCPU::perform (InverseFilterbankEngineCPU.C:309-366)
// with stitch / stitch_one (:443-616), filter (:620-700) and invert (:703-779)
// for complex (analytic) FPT input.
template <typename T>
int64_t inverse_filterbank (const orc_ifb_config* cfg, const T* in, uint64_t ndat,
                            uint64_t in_span, const T* response, const T* temporal,
                            const T* spectral, T* out, uint64_t out_span)
{
  typedef std::complex<T> C;
  const unsigned nin = cfg->input_nchan, nout = cfg->output_nchan, pfb = cfg->pfb_nchan;
  const unsigned Lin = cfg->input_fft_length;
  if (!nin || !nout || !pfb || nin % nout || nin % pfb || !cfg->os_num || !cfg->os_den) return -1;
  if ((uint64_t (Lin) * cfg->os_den) % cfg->os_num) return -1;
  const unsigned keep = unsigned (uint64_t (Lin) * cfg->os_den / cfg->os_num);  // Rational::normalize
  if ((Lin - keep) % 2 || keep % 2) return -1;
  const unsigned fine_per_out = nin / nout;
  const unsigned Lout = fine_per_out * keep;
  // output_to_input of the output discards (InverseFilterbank.C:285-288)
  auto to_input = [&] (uint64_t n) -> int64_t {
    const uint64_t a = n * nout * cfg->os_num, b = uint64_t (nin) * cfg->os_den;
    return a % b ? -1 : int64_t (a / b);
  };
  const int64_t in_pos = to_input (cfg->output_discard_pos), in_neg = to_input (cfg->output_discard_neg);
  if (in_pos < 0 || in_neg < 0) return -1;
  const uint64_t in_step = Lin - uint64_t (in_pos + in_neg);
  const uint64_t out_step = Lout - uint64_t (cfg->output_discard_pos + cfg->output_discard_neg);
  const unsigned coarse = nin / pfb;
  unsigned coarse_per_out = 1, out_per_coarse = 1, steps = coarse, out_per_step = 1;
  std::vector<unsigned> plan;
  if (fine_per_out > pfb)
  {
    if (fine_per_out % pfb) return -1;
    coarse_per_out = fine_per_out / pfb;
    steps = coarse / coarse_per_out;
    plan = ifb_fine_channel_plan (nin, pfb);
  }
  else if (fine_per_out < pfb)
  {
    if (pfb % fine_per_out) return -1;
    out_per_coarse = pfb / fine_per_out;
    steps = nout / out_per_coarse;
    out_per_step = out_per_coarse;
  }
  const bool shift = cfg->pfb_dc_chan != 0;
  const unsigned keep2 = keep / 2;
  uint64_t npart = 0;
  if (ndat > uint64_t (in_pos + in_neg)) npart = (ndat - (in_pos + in_neg)) / in_step;
  const unsigned spec_len = out_per_step * Lout;   // stitched spectrum of one step
  // (pol, part) pairs are independent: threads take whole pairs
  const int64_t ntask = int64_t (cfg->npol) * int64_t (npart);
#pragma omp parallel
  {
  std::vector<C> time (Lin), fine (Lin), spec (spec_len), tout (Lout);
#pragma omp for schedule(dynamic, 1)
  for (int64_t task = 0; task < ntask; task++)
  {
    const unsigned ipol = unsigned (task / int64_t (npart));
    const uint64_t ipart = uint64_t (task % int64_t (npart));
      for (unsigned istep = 0; istep < steps; istep++)
      {
        const unsigned fine_offset = istep * coarse_per_out * pfb;
        const unsigned out_offset = istep * out_per_coarse;
        std::fill (spec.begin (), spec.end (), C (0, 0));
        // stitch
        for (unsigned icoarse = 0; icoarse < coarse_per_out; icoarse++)
        {
          const unsigned start = fine_offset + icoarse * pfb;
          const uint64_t soff = uint64_t (icoarse) * keep * pfb;
          for (unsigned ich = 0; ich < pfb; ich++)
          {
            unsigned jch = ich + start;
            if (coarse_per_out > 1) jch = plan[jch];
            const C* src = reinterpret_cast<const C*> (in) + (uint64_t (jch) * cfg->npol + ipol) * in_span
                           + ipart * in_step;
            for (unsigned i = 0; i < Lin; i++)
              time[i] = temporal ? C (src[i].real () * temporal[i], src[i].imag () * temporal[i])
                                 : src[i];
            fft<T> (int (Lin), -1, time.data (), fine.data ());
            uint64_t neg, pos;
            if (shift)
            {
              if (ich == 0)
              {
                neg = uint64_t (keep) * pfb - keep2;
                pos = 0;
              }
              else
              {
                neg = uint64_t (keep) * ich - keep2;
                pos = neg + keep2;
              }
            }
            else
            {
              neg = uint64_t (keep) * ich;
              pos = neg + keep2;
            }
            const C* pneg = fine.data () + (Lin - keep2);
            const C* ppos = fine.data ();
            if (!cfg->dual_sideband)
            {
              pneg = fine.data () + (Lin - keep) / 2;
              ppos = pneg + keep2;
            }
            for (unsigned j = 0; j < keep2; j++)
            {
              spec[soff + neg + j] = pneg[j];
              spec[soff + pos + j] = ppos[j];
            }
          }
        }
        // filter
        if (!cfg->pfb_all_chan && cfg->pfb_dc_chan)
          for (unsigned j = 0; j < keep2; j++) spec[spec_len - keep2 + j] = C (0, 0);
        for (unsigned io = 0; io < out_per_step; io++)
        {
          C* s = spec.data () + uint64_t (io) * Lout;
          if (response)
          {
            // Response::operate: (f_r d_r - f_i d_i, f_i d_r + f_r d_i)
            const C* f = reinterpret_cast<const C*> (response) + uint64_t (out_offset + io) * Lout;
            for (unsigned k = 0; k < Lout; k++)
            {
              const T d_r = s[k].real (), d_i = s[k].imag ();
              const T f_r = f[k].real (), f_i = f[k].imag ();
              s[k] = C (f_r * d_r - f_i * d_i, f_i * d_r + f_r * d_i);
            }
          }
          if (spectral)
            for (unsigned k = 0; k < Lout; k++)
              s[k] = C (s[k].real () * spectral[k], s[k].imag () * spectral[k]);
          // invert
          fft_any<T> (int (Lout), +1, s, tout.data ());
          C* dst = reinterpret_cast<C*> (out) + (uint64_t (out_offset + io) * cfg->npol + ipol) * out_span
                   + ipart * out_step;
          for (uint64_t t = 0; t < out_step; t++) dst[t] = tout[cfg->output_discard_pos + t];
        }
      }
  }
  }
  return int64_t (npart);
}

} // namespace

extern "C" {

int64_t orc_inverse_filterbank_f32 (const orc_ifb_config* cfg, const float* in, uint64_t ndat,
                                    uint64_t in_span, const float* response, const float* temporal,
                                    const float* spectral, float* out, uint64_t out_span)
{
  return inverse_filterbank<float> (cfg, in, ndat, in_span, response, temporal, spectral, out,
                                    out_span);
}

int64_t orc_inverse_filterbank_f64 (const orc_ifb_config* cfg, const double* in, uint64_t ndat,
                                    uint64_t in_span, const double* response,
                                    const double* temporal, const double* spectral, double* out,
                                    uint64_t out_span)
{
  return inverse_filterbank<double> (cfg, in, ndat, in_span, response, temporal, spectral, out,
                                     out_span);
}

uint64_t orc_pipeline_c1 (const uint8_t* in, uint64_t ndat, const float* lut,
                          const float* response, unsigned nfft, unsigned nfilt_pos,
                          unsigned nfilt_neg, double phi, double phase_per_sample,
                          unsigned nbin, float* profile, uint32_t* hits, int nthreads)
{
  typedef std::complex<float> C;
  const uint64_t nsamp_overlap = nfilt_pos + nfilt_neg;
  const uint64_t nsamp_step = nfft - nsamp_overlap;
  if (ndat < nfft) return 0;
  const uint64_t npart = (ndat - nsamp_overlap) / nsamp_step;
  const uint64_t nout = npart * nsamp_step;
  std::vector<uint32_t> binplan (nout);
  orc_fold_binplan (phi, phase_per_sample, nout, nbin, binplan.data ());
  for (uint64_t i = 0; i < nout; i++) hits[binplan[i]]++;
  const int nt = nthreads > 0 ? nthreads : 1;
  std::vector<std::vector<float>> partial (nt, std::vector<float> (nbin, 0.0f));
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num ();
#endif
    std::vector<C> win (nfft), spec (nfft), tim[2] = {std::vector<C> (nfft), std::vector<C> (nfft)};
    float* prof = partial[tid].data ();
#pragma omp for schedule(dynamic, 1)
    for (int64_t ipart = 0; ipart < int64_t (npart); ipart++)
    {
      for (int ipol = 0; ipol < 2; ipol++)
      {
        const uint8_t* b = in + uint64_t (ipart) * nsamp_step * 4 + 2 * ipol;
        for (unsigned j = 0; j < nfft; j++)
          win[j] = C (lut[b[4 * j]], lut[b[4 * j + 1]]);
        fft<float> (nfft, -1, win.data (), spec.data ());
        const C* f = reinterpret_cast<const C*> (response);
        for (unsigned k = 0; k < nfft; k++)
        {
          const float d_r = spec[k].real (), d_i = spec[k].imag ();
          const float f_r = f[k].real (), f_i = f[k].imag ();
          spec[k] = C (f_r * d_r - f_i * d_i, f_i * d_r + f_r * d_i);
        }
        fft<float> (nfft, +1, spec.data (), tim[ipol].data ());
      }
      const uint64_t t0 = uint64_t (ipart) * nsamp_step;
      for (uint64_t j = 0; j < nsamp_step; j++)
      {
        const C p = tim[0][nfilt_pos + j], q = tim[1][nfilt_pos + j];
        float v = p.real () * p.real ();
        v += p.imag () * p.imag ();
        v += q.real () * q.real ();
        v += q.imag () * q.imag ();
        prof[binplan[t0 + j]] += v;
      }
    }
  }
  for (int t = 0; t < nt; t++)
    for (unsigned b = 0; b < nbin; b++) profile[b] += partial[t][b];
  return nout;
}

} // extern "C"
