// host_rules.h -- host-side rules of the B200 engine (see host_rules.cpp)
#pragma once

#include <cstdint>
#include <vector>

namespace b200 {

// One arithmetic segment of the exact fold-bin plan: sample start+j (j below
// the next segment's start) has frac(phi) = (m0 + j*dm) * g exactly, and
// folds into profile column base + bin (base = sub-integration slot * nbin;
// FOLD_SKIP: the samples are not folded).
struct FoldSegment
{
  uint64_t start;
  int64_t m0;
  int64_t dm;
  double g;
  uint32_t base = 0;
  uint32_t pad = 0;
};
constexpr uint32_t FOLD_SKIP = 0xffffffffu;

unsigned smearing_samples (double centre_frequency, double bandwidth, double dm,
                           unsigned nchan, int half);
unsigned minimum_ndat (unsigned impulse_pos, unsigned impulse_neg);
// Observation::get_centre_frequency(ichan) with get_unswapped_ichan (swap only)
double channel_centre (double centre_frequency, double bandwidth, unsigned nchan,
                       unsigned ichan, bool swap, bool dc_centred);
int64_t optimal_fft_length (uint64_t nbad, uint64_t nfft_max, unsigned factor);
void bittable8 (double spacing, bool twos_complement, float* lut, double* scale);
// s when every entry of a two's-complement 8-bit table equals
// (float(int8 x) + 0.5f) * s in float arithmetic (BitTable's tables do), so
// that a kernel may compute the value instead of looking it up; else 0
float affine_lut_scale (const float* lut256);
double fold_phi (int64_t start_day, int64_t start_sec, double start_frac,
                 int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                 uint64_t idat_start, double rate, double period, double reference_phase);
// SKLimits::calc_limits: lower/upper thresholds of the SK estimator for M
// samples (Nd integrated), std_devs sigma, ntest tests.  0 on success, -1 for
// invalid arguments, -2 where a Pearson type I density would be needed.
int sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest, float* lower,
               float* upper);
// InverseFilterbank fine-channel plan for combined coarse channels
std::vector<unsigned> ifb_fine_channel_plan (unsigned nchan, unsigned per_coarse);
// Apodization::build: type 0 top hat, 1 Hanning, 2 Welch, 3 Bartlett, 4 Tukey
// (transitions t_start, t_end); swap exchanges the halves.  0 on success.
int apodization (int type, unsigned ndat, unsigned t_start, unsigned t_end, bool swap,
                 float* window);
// Inter-channel dispersion delays (DedispersionPipe -K): the integer sample
// delay of each channel and its fractional remainder
// (Dedispersion::SampleDelay::get_sample_delay, DedispersionSampleDelay.C:
// 82-100), and SampleDelay::build's relative delays (SampleDelay.C:65-141):
// zero_delay, total_delay and the delay applied to each channel.
struct InterchannelDelays
{
  std::vector<int64_t> delay;      // floor(sample delay + 0.5)
  std::vector<double> frac;        // sample delay - delay, in samples
  std::vector<int64_t> applied;    // output sample t of channel c reads input t + applied[c]
  int64_t span_centre = 0;
  int64_t zero_delay = 0;
  uint64_t total_delay = 0;
};
void interchannel_delays (double centre_frequency, double dm, double rate, const double* freq,
                          unsigned nchan, InterchannelDelays* out);

// Archiver::set(Pulsar::Profile*, ...) (Signal/Pulsar/Archiver.C:852-984) with
// Archiver::set(Integration*, ...) (:740-792) for the profiles of one
// sub-integration: sums [nchan][npol][nbin], hits [nbin], or [nchan][nbin]
// when the data were zeroed per channel (PhaseSeries::get_zeroed_data).  amps
// get sum / (scale * hits); bins without hits are 0, or with
// unload_zero_hits the mean of the hit bins; a profile holding a non-finite
// sum is zeroed and its channel's weight set to 0; the weights [nchan] are
// otherwise 1, or hits_sum / ndat_total for zeroed data.  Returns 0, -1 for
// invalid arguments (a scale of 0 or not finite), -2 for bins without hits
// when unload_zero_hits is false; *corrupted counts zeroed profiles.
int archive_profiles (const float* sums, const uint32_t* hits, bool zeroed_data,
                      unsigned nchan, unsigned npol, unsigned nbin, double scale,
                      uint64_t ndat_total, bool unload_zero_hits, float* amps, float* weights,
                      unsigned* corrupted);

// Returns the number of segments; fills *out when non-null.  *x_end, when
// non-null, receives the recurrence's phase after the last sample: the phi
// with which the sequence goes on for the samples that follow.
int64_t build_fold_plan (double phi, double phase_per_sample, uint64_t ndat,
                         std::vector<FoldSegment>* out, double* x_end = nullptr);

} // namespace b200
