/*
 * oracle.h -- CPU restatement of the DSPSR baseband hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference arm of bench.py use it, and only as the checker or as the timed
 * CPU baseline.
 *
 * Every function restates the reference algorithm cited beside it (paths are
 * relative to the DSPSR source tree).  The reference itself cannot be built
 * here (its Signal/General/dsp headers, PSRCHIVE and FFTW are absent), so the
 * oracle carries its own FFT with FFTW's conventions (unnormalised; forward
 * sign -1, backward sign +1).
 *
 * Parity pins:
 *   - the Tukey impulse-response known-answer test restated from
 *     Signal/General/tests/ConvolutionTest.cpp:148-308 (RMS error < 5e-8);
 *   - the zero-DM passthrough of test/Convolution/test_Convolution.cpp;
 *   - the closed-form detection tests of test/Detection/test_Detection.cpp;
 *   - the fold bin recurrence (Signal/Pulsar/Fold.C:815-818) is the reference
 *     loop itself, run literally.
 * Unpinned: the 8-bit BitTable scale (needs PSRCHIVE's JenetAnderson98), the
 * missing PlasmaResponse::build template (restated from its call site and the
 * channel-frequency rule), PSRCHIVE's MJD arithmetic.
 */
#ifndef DSPSR_ORACLE_H
#define DSPSR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FFT (FTransform::fcc1d / bcc1d conventions) ---------------------- */
/* sign = -1 forward, +1 backward; unnormalised; in/out interleaved complex */
void orc_fft_f32 (int n, int sign, const float* in, float* out);
void orc_fft_f64 (int n, int sign, const double* in, double* out);

/* ---- unpack (Kernel/Classes/BitTable.C:172-225, EightBitUnpacker.C:25-49,
        BitUnpacker.C:97-138, SixteenBitUnpacker.C:23-79) ------------------ */
/* 8-bit lookup table; spacing = JenetAnderson98 optimal input spacing */
void orc_bittable8 (double spacing, int twos_complement, float* lut256, double* scale);
/* TFPD bytes -> FPT floats; out[(ichan*npol+ipol)*out_span + idat*ndim + idim] */
void orc_unpack8 (const uint8_t* in, uint64_t ndat, int nchan, int npol, int ndim,
                  const float* lut256, float* out, uint64_t out_span);
void orc_unpack16 (const int16_t* in, uint64_t ndat, int nchan, int npol, int ndim,
                   int offset_binary, float* out, uint64_t out_span);

/* ---- dispersion response (Signal/General/Dedispersion.C:84-186,
        PlasmaResponse.C:91-269, Response.C:325-420,529-621,998-1050,
        Kernel/Classes/Observation.C:521-534, optimize_fft.c:64-135) ------ */
unsigned orc_smearing_samples (double centre_freq, double bandwidth, double dm,
                               unsigned nchan, int half);
unsigned orc_minimum_ndat (unsigned impulse_pos, unsigned impulse_neg);
int64_t  orc_optimal_fft_length (uint64_t nbadperfft, uint64_t nfft_max, unsigned factor);
/* Response in FFT order, nchan*ndat complex values, normaliser 1/sqrt(norm_nfft)
   applied (Convolution.C:401-414).  mode 0: phase cast to float before
   polar() (Dedispersion.C:104-111); mode 1: FP64 phase range-reduced in FP64. */
void orc_dedispersion_response (double centre_freq, double bandwidth, double dm,
                                unsigned nchan, unsigned ndat, int input_nchan,
                                int dual_sideband, int dc_centred, int mode,
                                unsigned norm_nfft, float* out);
/* exact double-precision response (the FP64 oracle) */
void orc_dedispersion_response_f64 (double centre_freq, double bandwidth, double dm,
                                    unsigned nchan, unsigned ndat, int input_nchan,
                                    int dual_sideband, int dc_centred,
                                    unsigned norm_nfft, double* out);
/* Tukey-window test response (Signal/General/testutils/TestResponse.cpp:30-165,
   Apodization.C:123-146); spectral: ndat complex (FFT order, scaled 1/sqrt(ndat));
   temporal: impulse_neg+impulse_pos complex */
void orc_tukey_response (unsigned impulse_neg, unsigned impulse_pos, unsigned ndat,
                         float* spectral, float* temporal);

/* Observation::get_centre_frequency(ichan) with get_unswapped_ichan
   (Kernel/Classes/Observation.C:495-534) */
double orc_channel_centre (double centre_freq, double bandwidth, unsigned nchan,
                           unsigned ichan, int swap, int dc_centred);
/* Response for channels with explicit centre frequencies (what
   PlasmaResponse::configure stores in frequency_input, PlasmaResponse.C:73-80),
   each channel complex-sampled with its DC at FFT bin 0: the within-channel
   bins are half-swapped into FFT order.  mode as above; f64 variant writes
   double complex. */
void orc_dedispersion_response_channels (const double* chan_freq, unsigned nchan,
                                         double bandwidth, double dm, unsigned ndat,
                                         int mode, unsigned norm_nfft, float* out);
/* the same with the fractional inter-channel delay of each channel in
   microseconds (Dedispersion.C:141-187) */
void orc_dedispersion_response_channels_delay (const double* chan_freq, unsigned nchan,
                                               double bw, double dm, unsigned ndat, int mode,
                                               unsigned norm_nfft, const double* frac_delay_us,
                                               float* out);
void orc_dedispersion_response_channels_f64 (const double* chan_freq, unsigned nchan,
                                             double bandwidth, double dm, unsigned ndat,
                                             unsigned norm_nfft, double* out);

/* ---- FFT filterbank without convolution (freq_res = 1):
        Filterbank::do_prepare / prepare_output (Filterbank.C:75-380) and
        FilterbankEngineCPU::perform (FilterbankEngineCPU.C:379-535) --------- */
/* in: complex FPT, nchan_in spans of npol; out: nchan_in*nchan_sub channels of
   ndat/nchan_sub samples, channel k of subband s = FFT bin k of each block of
   nchan_sub samples, scaled by 1/sqrt(nchan_sub).  Returns output ndat. */
uint64_t orc_filterbank_f32 (const float* in, uint64_t ndat, uint64_t in_span, int nchan_in,
                             int npol, unsigned nchan_sub, float* out, uint64_t out_span);
uint64_t orc_filterbank_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan_in,
                             int npol, unsigned nchan_sub, double* out, uint64_t out_span);

/* ---- filterbank with a response ("During", -F nchan:D): Filterbank.C:98-198,
        398-420 and FilterbankEngineCPU.C:379-535 ------------------------------ */
/* response: [nchan_in*nsub][freq_res] complex as Response holds it; out:
   (chan*npol + pol)*out_span, npart*(freq_res - nfilt) samples each.
   Returns npart. */
/* temporal (nsub*freq_res) and spectral (freq_res) windows may be NULL */
uint64_t orc_filterbank_during_f32 (const float* in, uint64_t ndat, uint64_t in_span,
                                    int nchan_in, int npol, unsigned nsub, unsigned freq_res,
                                    unsigned nfilt_pos, unsigned nfilt_neg, const float* response,
                                    float* out, uint64_t out_span, const float* temporal,
                                    const float* spectral);
uint64_t orc_filterbank_during_f64 (const double* in, uint64_t ndat, uint64_t in_span,
                                    int nchan_in, int npol, unsigned nsub, unsigned freq_res,
                                    unsigned nfilt_pos, unsigned nfilt_neg, const double* response,
                                    double* out, uint64_t out_span, const float* temporal,
                                    const float* spectral);
/* its dedispersion response: channels centred at chan_freq, natural frequency
   order within each channel, scaled by 1/sqrt(norm), norm = nsamp_fft*freq_res */
void orc_dedispersion_response_during (const double* chan_freq, unsigned nchan, double bw,
                                       double dm, unsigned ndat, int mode, double norm,
                                       float* out);
void orc_dedispersion_response_during_f64 (const double* chan_freq, unsigned nchan, double bw,
                                           double dm, unsigned ndat, double norm, double* out);

/* ---- overlap-save convolution (Signal/General/Convolution.C:316-813) ----- */
/* in/out FPT: (ichan*npol+ipol)*span complex values; response nchan*nfft complex
   (one filter for all polns).  Returns npart.  out holds npart*(nfft-nfilt) values. */
uint64_t orc_convolve_f32 (const float* in, uint64_t ndat, uint64_t in_span,
                           int nchan, int npol, const float* response,
                           unsigned nfft, unsigned nfilt_pos, unsigned nfilt_neg,
                           float* out, uint64_t out_span, int nthreads);
uint64_t orc_convolve_f64 (const double* in, uint64_t ndat, uint64_t in_span,
                           int nchan, int npol, const double* response,
                           unsigned nfft, unsigned nfilt_pos, unsigned nfilt_neg,
                           double* out, uint64_t out_span, int nthreads);

/* ---- detection (Signal/General/Detection.C:225-630, stokes_detect.ic,
        cross_detect.ic) -------------------------------------------------- */
/* state: 0 Intensity (1 out pol), 1 PPQQ (2), 2 Coherence (4: PP,QQ,Re p*q,Im p*q),
   3 Stokes (4: I,Q,U,V).  in: 2 pols complex FPT; out: FPT floats. */
int orc_detect (const float* in, uint64_t ndat, uint64_t in_span, int nchan,
                int state, float* out, uint64_t out_span);
int orc_detect_f64 (const double* in, uint64_t ndat, uint64_t in_span, int nchan,
                    int state, double* out, uint64_t out_span);

/* ---- fold (Signal/Pulsar/Fold.C:662-990) -------------------------------- */
/* phase of the first sample midpoint, constant period (Fold.C:975-979) */
double orc_fold_phi (int64_t start_day, int64_t start_sec, double start_frac,
                     int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                     uint64_t idat_start, double rate, double period,
                     double reference_phase);
/* the literal sequential recurrence, Fold.C:790-837 */
void orc_fold_binplan (double phi, double phase_per_sample, uint64_t ndat,
                       unsigned nbin, uint32_t* binplan);
/* accumulate FPT data (nchan*npol spans, ndim per sample) into profiles
   [ichan][ipol][ibin*ndim+idim]; hits[ibin] += 1 per sample (Fold.C:893-931) */
void orc_fold_accumulate (const float* in, uint64_t ndat, uint64_t in_span,
                          int nchan, int npol, int ndim, const uint32_t* binplan,
                          unsigned nbin, float* profiles, uint32_t* hits);
void orc_fold_accumulate_f64 (const double* in, uint64_t ndat, uint64_t in_span,
                              int nchan, int npol, int ndim, const uint32_t* binplan,
                              unsigned nbin, double* profiles, uint32_t* hits);

/* ---- SpectralKurtosis, one resolution, noverlap = 1
        (Signal/General/SpectralKurtosis.C:251-281, 674-798, 1105-1222, 1465-1566) */
/* complex FPT input; sums[(ipart*nchan + ichan)*npol + ipol][2] = (S1, S2) as
   float from double accumulation; counts[ipart*nchan + ichan]. Returns npart. */
uint64_t orc_sk_compute (const float* in, uint64_t ndat, uint64_t in_span, int nchan, int npol,
                         unsigned M, int zero_is_valid, float* sums, uint32_t* counts);
/* mask[ipart*nchan + ichan] = 1 where any pol's SK estimator lies outside
   [lower, upper] (or fewer than 3 samples counted); returns zapped count */
uint64_t orc_sk_detect (const float* sums, const uint32_t* counts, uint64_t npart, int nchan,
                        int npol, unsigned Nd, float lower, float upper, uint8_t* mask);
/* out = in, with every masked M-sample block of every pol set to zero */
void orc_sk_mask (const float* in, uint64_t in_span, float* out, uint64_t out_span,
                  const uint8_t* mask, uint64_t npart, int nchan, int npol, unsigned M);
/* SKLimits::calc_limits (Signal/Statistics/SKLimits.C:136-229): lower and
   upper SK thresholds for M samples of Nd integrated intensities, std_devs
   sigma, ntest tests; Romberg-integrated Pearson IV / VI CDFs. 0 on success. */
int orc_sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest, float* lower,
                   float* upper);

/* ---- InverseFilterbank (Signal/General/InverseFilterbank.C:129-454,
        InverseFilterbankEngineCPU.C:46-792), complex FPT input ---------------- */
typedef struct orc_ifb_config
{
  unsigned input_nchan;        /* fine channels */
  unsigned output_nchan;       /* divides input_nchan */
  unsigned pfb_nchan;          /* fine channels per coarse (PFB) channel */
  unsigned npol;
  unsigned input_fft_length;   /* forward FFT per fine channel */
  unsigned os_num, os_den;     /* oversampling factor, e.g. 4/3 */
  unsigned output_discard_pos, output_discard_neg;
  int pfb_dc_chan, pfb_all_chan, dual_sideband;
} orc_ifb_config;
/* in [input_nchan][npol][in_span] complex; out [output_nchan][npol][out_span]
   complex; response [output_nchan][Lout] complex, temporal [Lin] and
   spectral [Lout] real windows, each optional (null).  Lout =
   (input_nchan/output_nchan) * Lin*os_den/os_num.  Returns npart, or -1 for
   an invalid configuration. */
int64_t orc_inverse_filterbank_f32 (const orc_ifb_config* cfg, const float* in, uint64_t ndat,
                                    uint64_t in_span, const float* response,
                                    const float* temporal, const float* spectral, float* out,
                                    uint64_t out_span);
int64_t orc_inverse_filterbank_f64 (const orc_ifb_config* cfg, const double* in, uint64_t ndat,
                                    uint64_t in_span, const double* response,
                                    const double* temporal, const double* spectral, double* out,
                                    uint64_t out_span);

/* overlap-save as orc_convolve_f32 with the temporal apodization window
   (nfft floats) applied to every part before its forward FFT */
uint64_t orc_convolve_window_f32 (const float* in, uint64_t ndat, uint64_t in_span, int nchan,
                                  int npol, const float* response, unsigned nfft,
                                  unsigned nfilt_pos, unsigned nfilt_neg, float* out,
                                  uint64_t out_span, int nthreads, const float* window);
/* Apodization::build (Signal/General/Apodization.C:60-178): 0 top hat,
   1 Hanning, 2 Welch, 3 Bartlett, 4 Tukey; swap exchanges the halves */
int orc_apodization (int type, unsigned ndat, unsigned transition_start,
                     unsigned transition_end, int swap, float* window);

/* ---- the whole single-channel path, for the timed CPU baseline ----------- */
/* int8 TFPD (nchan=1, npol=2, ndim=2) -> unpack -> convolve -> Intensity ->
   fold.  Returns the number of output samples folded per pol. */
uint64_t orc_pipeline_c1 (const uint8_t* in, uint64_t ndat, const float* lut256,
                          const float* response, unsigned nfft, unsigned nfilt_pos,
                          unsigned nfilt_neg, double phi, double phase_per_sample,
                          unsigned nbin, float* profile, uint32_t* hits, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
