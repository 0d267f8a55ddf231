/*
 * dspsr_b200.h -- C ABI of libdspsr_b200.so, the B200 (sm_100a) engine for
 * DSPSR's baseband hot path: unpack -> overlap-save coherent dedispersion ->
 * detection -> fold.
 *
 * Plain C types only: device pointers are untyped or float pointers, sizes
 * are uint64_t, streams are passed as an untyped pointer (a cudaStream_t).  Every call returns an int
 * status (DSPSR_B200_OK == 0); the message of the last failure on a context is
 * returned by dspsr_b200_last_error().  No exception crosses this boundary.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the DSPSR source tree).  The reference's CUDA engines are
 * CUDA::ConvolutionEngine, CUDA::DetectionEngine, CUDA::FoldEngine and the
 * generic_8bit_unpack kernel; their host classes (dsp::Convolution,
 * dsp::Detection, dsp::Fold, dsp::GenericEightBitUnpacker) keep all
 * bookkeeping and hand the engine raw device pointers, strides and counts,
 * which is exactly what these functions take.
 */
#ifndef DSPSR_B200_H
#define DSPSR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSPSR_B200_OK        0
#define DSPSR_B200_EINVAL    1   /* InvalidParam in the reference's Error codes */
#define DSPSR_B200_ESTATE    2   /* InvalidState */
#define DSPSR_B200_ECUDA     3   /* FailedCall (CUDA runtime) */
#define DSPSR_B200_ENOMEM    4
#define DSPSR_B200_ENODEV    5   /* no CUDA device: the library never falls back to the CPU */
#define DSPSR_B200_ETOOBIG   6   /* the sizes need more than the fixed scratch of
                                    dspsr_b200_convolution_perform_noalloc */

/* Signal::State values accepted by detection and the fused path
   (Signal/General/Detection.C:225-630) */
#define DSPSR_B200_INTENSITY 0   /* PP+QQ, one output polarisation */
#define DSPSR_B200_PPQQ      1   /* PP, QQ */
#define DSPSR_B200_COHERENCE 2   /* PP, QQ, Re[p*q], Im[p*q] (cross_detect.ic:38-41) */
#define DSPSR_B200_STOKES    3   /* I, Q, U, V (stokes_detect.ic:40-43) */

/* input sample encodings */
#define DSPSR_B200_INT8_TFPD   0 /* 8-bit two's complement, BitTable lookup */
#define DSPSR_B200_INT16_TFPD  1 /* 16-bit, float(x)+0.5 (SixteenBitUnpacker.C:54-79) */
#define DSPSR_B200_FLOAT_FPT   2 /* complex float, one span per (chan, pol) */

/* arithmetic of the convolution's row FFTs (the n2 = 8192 half of the
   four-step split, nfft >= 16384) */
#define DSPSR_B200_FFT_FP32   0  /* FP32 Stockham passes on the CUDA cores */
#define DSPSR_B200_FFT_BF16X3 3  /* DFT16/DFT32 stages as tensor-core GEMMs, operands
                                    split into three BF16 terms (six products,
                                    FP32 accumulation: FP32-level accuracy) */
#define DSPSR_B200_FFT_BF16X2 2  /* the same with two BF16 terms (three products,
                                    about 16 significant bits per stage) */

/* dispersion response evaluation */
#define DSPSR_B200_CHIRP_REFERENCE 0 /* phase rounded to float before sin/cos,
                                        as Dedispersion.C:104-111 does */
#define DSPSR_B200_CHIRP_FP64      1 /* phase reduced mod 2pi in FP64, then
                                        rounded once to float */

typedef struct dspsr_b200_context dspsr_b200_context;
typedef struct dspsr_b200_convolution dspsr_b200_convolution;
typedef struct dspsr_b200_fold dspsr_b200_fold;
typedef struct dspsr_b200_pipeline dspsr_b200_pipeline;
typedef struct dspsr_b200_inverse_filterbank dspsr_b200_inverse_filterbank;

/* ---------------------------------------------------------------------- */
/* Library and context                                                     */
/* ---------------------------------------------------------------------- */

/* library version, major*10000 + minor*100 + patch */
int dspsr_b200_version (void);

/* Replaces the CUDA::DeviceMemory(stream) + engine construction done in
   SingleThread::construct (Signal/General/SingleThread.C:294-344): binds a
   device and a stream (NULL = legacy default stream). */
int dspsr_b200_context_create (int device, void* stream, dspsr_b200_context** ctx);
int dspsr_b200_context_destroy (dspsr_b200_context* ctx);
int dspsr_b200_context_set_stream (dspsr_b200_context* ctx, void* stream);
const char* dspsr_b200_last_error (const dspsr_b200_context* ctx);
/* blocks until all work queued on the context's stream is done */
int dspsr_b200_synchronize (dspsr_b200_context* ctx);

/* ---------------------------------------------------------------------- */
/* Host-side rules (no GPU needed)                                         */
/* ---------------------------------------------------------------------- */

/* PlasmaResponse::smearing_samples (Signal/General/PlasmaResponse.C:210-250);
   half = -1, 0, +1 */
unsigned dspsr_b200_smearing_samples (double centre_freq_mhz, double bandwidth_mhz,
                                      double dm, unsigned nchan, int half);
/* Response::get_minimum_ndat (Signal/General/Response.C:529-545) */
unsigned dspsr_b200_minimum_ndat (unsigned impulse_pos, unsigned impulse_neg);
/* optimal_fft_length (Signal/General/optimize_fft.c:64-135) */
int64_t dspsr_b200_optimal_fft_length (uint64_t nbadperfft, uint64_t nfft_max,
                                       unsigned factor);
/* BitTable::generate for nbit = 8 (Kernel/Classes/BitTable.C:104-225);
   spacing = the JenetAnderson98 optimal input spacing for 8 bits */
int dspsr_b200_bittable8 (double spacing, int twos_complement, float* lut256,
                          double* scale);
/* Fold::get_phi for a constant folding period (Signal/Pulsar/Fold.C:685-693,
   975-979); MJDs are (day, second, fraction of a second) */
double dspsr_b200_fold_phi (int64_t start_day, int64_t start_sec, double start_frac,
                            int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                            uint64_t idat_start, double rate, double period,
                            double reference_phase);
/* SKLimits::calc_limits (Signal/Statistics/SKLimits.C:136-229) as
   SpectralKurtosis::get_limits calls it (SpectralKurtosis.C:989-1007): the
   float thresholds of the SK estimator for M intensities of Nd integrated
   samples, std_devs sigma, ntest tests (the number of polarisations).
   DSPSR_B200_EINVAL for M < 2, Nd = 0, ntest = 0 or std_devs giving no error
   rate; DSPSR_B200_ESTATE where the moments call for a Pearson type I density
   (which the reference does not implement either). */
int dspsr_b200_sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest,
                          float* lower, float* upper);
/* Apodization::build (Signal/General/Apodization.C:60-146) and swap
   (:168-178): the window of ndat points, type DSPSR_B200_APOD_*; Tukey uses
   transition_start / transition_end.  swap_halves exchanges the two halves
   (spectral windows of dual-sideband data). */
#define DSPSR_B200_APOD_TOPHAT   0
#define DSPSR_B200_APOD_HANNING  1
#define DSPSR_B200_APOD_WELCH    2
#define DSPSR_B200_APOD_BARTLETT 3
#define DSPSR_B200_APOD_TUKEY    4
int dspsr_b200_apodization (int type, unsigned ndat, unsigned transition_start,
                            unsigned transition_end, int swap_halves, float* window);
/* Inter-channel dispersion delays for channels centred at freq_mhz[nchan],
   sampled at rate_hz, relative to the band centre centre_freq_mhz:
   Dedispersion::SampleDelay (DedispersionSampleDelay.C:26-140) gives delay[c]
   (the nearest whole-sample delay) and frac[c] (the remainder, samples);
   SampleDelay::build (SampleDelay.C:65-141) gives zero_delay, total_delay and
   applied[c], the shift SampleDelay::transformation (:247-298) applies:
   output sample t of channel c = input sample t + applied[c]. */
int dspsr_b200_interchannel_delays (double centre_freq_mhz, double dm, double rate_hz,
                                    const double* freq_mhz, unsigned nchan, int64_t* delay,
                                    double* frac, int64_t* applied, int64_t* zero_delay,
                                    uint64_t* total_delay);
/* The profile arithmetic of the PhaseSeries -> archive unloader:
   Archiver::set(Pulsar::Profile*) (Signal/Pulsar/Archiver.C:852-984) and the
   channel weights of Archiver::set(Integration*) (:740-792), for one
   sub-integration.  sums [nchan][npol][nbin] as the fold left them; hits
   [nbin], or [nchan][nbin] when zeroed_data (PhaseSeries::get_zeroed_data);
   scale = PhaseSeries::get_scale; ndat_total = get_ndat_total (zeroed data
   only).  amps [nchan][npol][nbin] = sum / (scale * hits); unhit bins: an
   error (DSPSR_B200_ESTATE, the reference's InvalidParam throw) unless
   unload_zero_hits, then the mean of the hit bins; a profile with a
   non-finite sum is zeroed and its channel's weight set to 0.  weights
   [nchan]: 1, or hits_sum / ndat_total for zeroed data.  *corrupted (may
   be NULL) counts the zeroed profiles.  Host only. */
int dspsr_b200_archive_profiles (const float* sums, const uint32_t* hits, int zeroed_data,
                                 unsigned nchan, unsigned npol, unsigned nbin, double scale,
                                 uint64_t ndat_total, int unload_zero_hits, float* amps,
                                 float* weights, unsigned* corrupted);
/* Number of arithmetic segments the exact fold-bin plan needs for a block
   (see dspsr_b200_fold_set_bins); lets a caller size buffers. */
int64_t dspsr_b200_fold_plan_count (double phi, double phase_per_sample,
                                    uint64_t ndat);

/* ---------------------------------------------------------------------- */
/* Unpacker (GenericEightBitUnpacker::unpack_on_gpu,                       */
/* Kernel/Classes/GenericEightBitUnpacker.C:92-131, and generic_8bit_unpack,*/
/* Kernel/Classes/GenericEightBitUnpackerCUDA.cu:47-100)                    */
/* ---------------------------------------------------------------------- */

/* TFPD bytes (ndim values per (t, chan, pol)) -> FPT floats:
   out[(ichan*npol + ipol)*out_span + idat*ndim + idim] = lut256[byte] */
int dspsr_b200_unpack8 (dspsr_b200_context* ctx, const void* d_in, uint64_t ndat,
                        unsigned nchan, unsigned npol, unsigned ndim,
                        const float* lut256, float* d_out, uint64_t out_span);
/* SixteenBitUnpacker::unpack (Kernel/Classes/SixteenBitUnpacker.C:23-79) */
int dspsr_b200_unpack16 (dspsr_b200_context* ctx, const void* d_in, uint64_t ndat,
                         unsigned nchan, unsigned npol, unsigned ndim,
                         int offset_binary, float* d_out, uint64_t out_span);

/* ---------------------------------------------------------------------- */
/* Convolution::Engine (CUDA::ConvolutionEngine,                            */
/* Signal/General/ConvolutionCUDA.cu:174-774; callers Convolution.C:446-452,*/
/* 656-667, 690-698)                                                        */
/* ---------------------------------------------------------------------- */

/* Engine::prepare(Convolution*): sizes from Convolution::prepare
   (Convolution.C:316-465).  nfft must be a power of two in [4096, 262144]. */
int dspsr_b200_convolution_create (dspsr_b200_context* ctx, unsigned nchan,
                                   unsigned npol, unsigned nfft, unsigned nfilt_pos,
                                   unsigned nfilt_neg, dspsr_b200_convolution** conv);
int dspsr_b200_convolution_destroy (dspsr_b200_convolution* conv);
/* Engine::copy_response(const Response*): nchan*nfft complex floats
   (interleaved re,im) in FFT order, normaliser already applied; host memory. */
int dspsr_b200_convolution_copy_response (dspsr_b200_convolution* conv,
                                          const float* response);
/* Builds the Dedispersion response on the GPU in FP64 (Dedispersion.C:84-186
   with the PlasmaResponse::build grid, Response::swap_as_needed
   Response.C:325-400 and the 1/sqrt(norm_nfft) normaliser of
   Convolution::prepare_normalizer Convolution.C:300-313,401-414). */
int dspsr_b200_convolution_set_dedispersion (dspsr_b200_convolution* conv,
                                             double centre_freq_mhz, double bandwidth_mhz,
                                             double dm, int input_nchan, int dual_sideband,
                                             int dc_centred, int chirp_mode,
                                             unsigned norm_nfft);
/* The same response for channels whose centre frequencies the caller supplies
   (the values PlasmaResponse::configure stores in frequency_input from
   Observation::get_centre_frequency(ichan), PlasmaResponse.C:73-80), each
   channel complex-sampled with DC at its FFT bin 0 (the per-channel
   Response::doswap of Response.C:375-387); bandwidth is the whole band's. */
int dspsr_b200_convolution_set_dedispersion_channels (dspsr_b200_convolution* conv,
                                                      const double* chan_freq_mhz,
                                                      double bandwidth_mhz, double dm,
                                                      int chirp_mode, unsigned norm_nfft);
/* The same overlap-save convolution without allocating anything.  This entry
   point has no counterpart in the reference: it exists for callers that
   cannot call cudaMalloc while they run -- real-time processes that fix all
   memory at start-up so that no allocation stalls a block, and hosts whose
   device memory is owned by another allocator that does not let a library
   allocate behind its back.  It takes no context or engine object: stream (a
   cudaStream_t, NULL for the legacy default stream), the complex FPT input
   (in_span complex samples per (chan, pol)), the response (nchan*nfft complex
   floats in FFT order, in device memory, normaliser applied), and the output;
   sizes as for dspsr_b200_convolution_create.  Its tables and FFT scratch
   live in one static device array of DSPSR_B200_NOALLOC_SCRATCH_BYTES that
   every GPU loading the library keeps until exit; shapes needing more
   (roughly nchan*(npol+1)*nfft*8 bytes plus nfft*8 for FFTs above 8192
   points) return DSPSR_B200_ETOOBIG.  The array's address and the kernels'
   shared-memory opt-in are set up by the first call made on each device,
   whatever its shape (make that call before any stream capture).  All calls
   share the one array and leave their contents in it: calls whose work
   overlaps on the GPU race.  d_status (device memory, may be NULL) is set to
   0 in stream order at the start of the call; a kernel with a bounded
   device-side wait would set it to 1 when the wait gave up (the output then
   not valid), but the FP32 kernels this call runs have none, so it reads 0
   once the stream has passed the call.  Returns the
   launch status; *npart as for dspsr_b200_convolution_perform. */
#define DSPSR_B200_NOALLOC_SCRATCH_BYTES (32ull << 20)
int dspsr_b200_convolution_perform_noalloc (void* stream, const float* d_in, uint64_t in_span,
                                            uint64_t ndat, unsigned nchan, unsigned npol,
                                            unsigned nfft, unsigned nfilt_pos,
                                            unsigned nfilt_neg, const float* d_response,
                                            float* d_out, uint64_t out_span, uint64_t* npart,
                                            int* d_status);
/* Blocks until the engine's queued work is done and returns DSPSR_B200_ESTATE
   if one of its device-side waits gave up (the tensor-core rows' mbarrier
   waits, each bounded to about a second; the FP32 kernels have none),
   DSPSR_B200_OK otherwise. */
int dspsr_b200_convolution_status (dspsr_b200_convolution* conv);
/* copies the response (FFT order) back to host memory, nchan*nfft complex */
int dspsr_b200_convolution_get_response (dspsr_b200_convolution* conv, float* response);
/* Convolution::set_temporal_apodization (Convolution.C:144-147, 222-250,
   applied at :739-743): a window of nfft floats (dspsr_b200_apodization, e.g.
   Tukey with transitions nfilt_pos / nfilt_neg) multiplied into every part
   before its forward FFT; NULL removes it. */
int dspsr_b200_convolution_set_temporal_apodization (dspsr_b200_convolution* conv,
                                                     const float* window);
/* The row FFTs' arithmetic, DSPSR_B200_FFT_FP32 (default), _BF16X3 or
   _BF16X2.  The tensor-core forms replace the cuFFT C2C plans of the
   reference's engine (ConvolutionCUDA.cu:370-413) for the rows of the
   four-step split; they need nfft >= 16384 (EINVAL otherwise). */
int dspsr_b200_convolution_set_fft_precision (dspsr_b200_convolution* conv, int mode);
/* Engine::perform(input, output, npart): complex FPT in (span in complex
   samples per (chan, pol)), complex FPT out; returns npart
   = (ndat - nfilt_pos - nfilt_neg)/(nfft - nfilt_pos - nfilt_neg). */
int dspsr_b200_convolution_perform (dspsr_b200_convolution* conv, const float* d_in,
                                    uint64_t in_span, uint64_t ndat, float* d_out,
                                    uint64_t out_span, uint64_t* npart);
/* Engine::perform(input, output, zero_DM_output, npart) (Convolution.C:690-698,
   789-796): as dspsr_b200_convolution_perform, and the zero-DM output -- the
   undispersed input samples aligned with the output, nfilt_pos after the
   start of each part -- copied to d_zero_dm (complex FPT spans of
   zero_dm_span samples). */
int dspsr_b200_convolution_perform_zero_dm (dspsr_b200_convolution* conv, const float* d_in,
                                            uint64_t in_span, uint64_t ndat, float* d_out,
                                            uint64_t out_span, float* d_zero_dm,
                                            uint64_t zero_dm_span, uint64_t* npart);

/* ---------------------------------------------------------------------- */
/* Filterbank::Engine without convolution (freq_res = 1): CUDA::FilterbankEngine*/
/* (Signal/General/FilterbankEngineCUDA.cu:353-480), FilterbankEngineCPU     */
/* (FilterbankEngineCPU.C:379-535); callers Filterbank.C:454-570            */
/* ---------------------------------------------------------------------- */

/* Every block of nsub input samples of each (input channel, pol) becomes one
   sample in nsub output channels: out channel cin*nsub + k = FFT bin k scaled
   by 1/sqrt(nsub) (Filterbank::prepare_normalizer).  Input as input_kind
   (TFPD int8/int16 or complex-float FPT with in_span); the unpack is fused.
   Output complex-float FPT, (chan*npol + pol)*out_span.  nsub a power of two
   in [4, 4096].
   Returns ndat/nsub output samples; a trailing partial block is ignored. */
int dspsr_b200_filterbank (dspsr_b200_context* ctx, int input_kind, const void* d_in,
                           uint64_t ndat, uint64_t in_span, unsigned nchan_in, unsigned npol,
                           unsigned nsub, const float* lut256, int offset_binary,
                           float* d_out, uint64_t out_span, uint64_t* ndat_out);

/* ---------------------------------------------------------------------- */
/* InverseFilterbank::Engine (InverseFilterbankEngineCPU.C:46-792,          */
/* InverseFilterbankEngineCUDA.cu:58-529; caller InverseFilterbank.C:129-454) */
/* ---------------------------------------------------------------------- */

/* Shape of InverseFilterbank::make_preparations (InverseFilterbank.C:225-330):
   input_nchan fine channels (pfb_nchan per coarse PFB channel), output_nchan
   dividing input_nchan; each fine channel is transformed in
   input_fft_length-point FFTs of which Lin*os_den/os_num bins are kept and
   stitched; output FFT length Lout = (input_nchan/output_nchan) * kept bins,
   which must be n1 * 4096 or n1 * 8192 with n1 in {2,3,4,6,8,12,16,24,32}.
   Output discards are given (from the response); the input discards follow
   by output_to_input (InverseFilterbank.C:128-142).  scratch_bytes bounds the
   device scratch (0 = 512 MiB). */
typedef struct dspsr_b200_ifb_config
{
  unsigned input_nchan;
  unsigned output_nchan;
  unsigned pfb_nchan;
  unsigned npol;
  unsigned input_fft_length;
  unsigned os_num, os_den;
  unsigned output_discard_pos, output_discard_neg;
  int pfb_dc_chan;          /* channel 0 of the PFB is centred on DC */
  int pfb_all_chan;         /* all PFB channels present (else the last half channel is zeroed) */
  int dual_sideband;
  uint64_t scratch_bytes;
} dspsr_b200_ifb_config;

/* Engine::setup (InverseFilterbankEngineCPU.C:46-278) */
int dspsr_b200_inverse_filterbank_create (dspsr_b200_context* ctx,
                                          const dspsr_b200_ifb_config* cfg,
                                          dspsr_b200_inverse_filterbank** ifb);
int dspsr_b200_inverse_filterbank_destroy (dspsr_b200_inverse_filterbank* ifb);
/* info[10] = {kept bins, Lout, input step, output step, input discard pos,
   input discard neg, n1, n2, parts per batch, input FFT length} */
int dspsr_b200_inverse_filterbank_info (dspsr_b200_inverse_filterbank* ifb, uint64_t* info);
/* the response applied by filter() (Response::operate, e.g. the deripple of
   InverseFilterbankResponse::build or a dedispersion response): host complex
   [output_nchan][Lout] interleaved re/im; NULL removes it */
int dspsr_b200_inverse_filterbank_copy_response (dspsr_b200_inverse_filterbank* ifb,
                                                 const float* response);
/* temporal window of input_fft_length points applied before each forward FFT
   and spectral window of Lout points applied after the response (either may
   be NULL), as set_temporal_apodization / set_spectral_apodization do */
int dspsr_b200_inverse_filterbank_set_apodization (dspsr_b200_inverse_filterbank* ifb,
                                                   const float* temporal, const float* spectral);
/* Engine::perform (InverseFilterbankEngineCPU.C:309-366): npart =
   (ndat - input discards) / input step parts; output FPT complex
   [output_nchan][npol] spans of out_span complex samples, npart * output step
   written per span.  Input as dspsr_b200_filterbank takes it (int8 / int16
   TFPD or complex-float FPT with in_span). */
int dspsr_b200_inverse_filterbank_perform (dspsr_b200_inverse_filterbank* ifb, int input_kind,
                                           const void* d_in, uint64_t ndat, uint64_t in_span,
                                           const float* lut256, int offset_binary, float* d_out,
                                           uint64_t out_span, uint64_t* npart);
/* Blocks until the engine's queued work is done; DSPSR_B200_ESTATE would
   report a device-side wait that gave up, but the inverse filterbank's
   kernels have none, so it returns DSPSR_B200_OK (kept for callers that
   check every engine the same way). */
int dspsr_b200_inverse_filterbank_status (dspsr_b200_inverse_filterbank* ifb);

/* ---------------------------------------------------------------------- */
/* Filterbank::Engine with a response: the "During" filterbank (-F N:D;     */
/* Filterbank::do_prepare with a response, Filterbank.C:98-198;             */
/* FilterbankEngineCPU::perform, FilterbankEngineCPU.C:379-535;             */
/* CUDA::FilterbankEngine::perform, FilterbankEngineCUDA.cu:353-480)        */
/* ---------------------------------------------------------------------- */

/* Each part of nsamp_fft = nsub * freq_res input samples of every input
   channel is transformed forward, multiplied by the response of its nsub
   output channels (channel cin*nsub + k takes bins [k*freq_res,
   (k+1)*freq_res) of the FFT-order spectrum), and each output channel is
   transformed back in freq_res points, of which nkeep = freq_res - nfilt_pos
   - nfilt_neg from nfilt_pos are kept.  Parts start nsamp_step = nsub * nkeep
   input samples apart; npart = (ndat - nsub*(nfilt_pos+nfilt_neg)) /
   nsamp_step (Filterbank::resize_output, Filterbank.C:398-420).  Supported:
   nsub a power of two in [2, 128], freq_res a power of two, nsub * freq_res
   in [16384, 4194304]. */
typedef struct dspsr_b200_filterbank_during dspsr_b200_filterbank_during;
typedef struct dspsr_b200_fbd_config
{
  unsigned input_nchan;
  unsigned npol;
  unsigned nsub;            /* output channels per input channel (nchan_subband) */
  unsigned freq_res;        /* points per output channel: the response's ndat */
  unsigned nfilt_pos, nfilt_neg;
  uint64_t scratch_bytes;   /* device scratch bound, 0 = 512 MiB */
} dspsr_b200_fbd_config;

/* Engine::setup (FilterbankEngineCUDA.cu:62-150) */
int dspsr_b200_filterbank_during_create (dspsr_b200_context* ctx,
                                         const dspsr_b200_fbd_config* cfg,
                                         dspsr_b200_filterbank_during** fbd);
int dspsr_b200_filterbank_during_destroy (dspsr_b200_filterbank_during* fbd);
/* info[6] = {nsamp_fft, nsamp_step, nsamp_overlap, nkeep, n1, parts per batch} */
int dspsr_b200_filterbank_during_info (dspsr_b200_filterbank_during* fbd, uint64_t* info);
/* Engine::copy_response: host complex [input_nchan*nsub][freq_res] as
   Response holds it after swap_as_needed, normaliser 1/sqrt(nsamp_fft *
   freq_res) applied (Filterbank.C:171-186). */
int dspsr_b200_filterbank_during_copy_response (dspsr_b200_filterbank_during* fbd,
                                                const float* response);
/* Builds that response on the GPU in FP64: Dedispersion prepared for the
   output channels (Response::prepare(input, nchan), Filterbank.C:101-110;
   Dedispersion.C:84-186), each channel in natural frequency order, then the
   whole response swapped (Response::doswap, Response.C:998-1050) when the
   input is one dual-sideband channel or a swapped multi-channel band
   (Response::swap_as_needed, Response.C:325-400), and the normaliser. */
int dspsr_b200_filterbank_during_set_dedispersion (dspsr_b200_filterbank_during* fbd,
                                                   double centre_freq_mhz,
                                                   double bandwidth_mhz, double dm,
                                                   int swapped, int chirp_mode);
/* Filterbank::set_temporal_apodization / set_spectral_apodization
   (Filterbank.C:201-207, applied at FilterbankEngineCPU.C:447-449, 507-509):
   a window of nsub*freq_res floats multiplied into each part before the
   forward FFT, and one of freq_res floats multiplied into each output
   channel's spectrum before its inverse FFT (held folded into the response);
   NULL removes either. */
int dspsr_b200_filterbank_during_set_apodization (dspsr_b200_filterbank_during* fbd,
                                                  const float* temporal, const float* spectral);
/* copies the response back: [input_nchan*nsub][freq_res] complex, FFT order */
int dspsr_b200_filterbank_during_get_response (dspsr_b200_filterbank_during* fbd,
                                               float* response);
/* Engine::perform (FilterbankEngineCPU.C:379-535): input as
   dspsr_b200_filterbank takes it (int8 / int16 TFPD or complex-float FPT with
   in_span); output complex-float FPT, (chan*npol + pol)*out_span with
   npart * nkeep samples written per span. */
int dspsr_b200_filterbank_during_perform (dspsr_b200_filterbank_during* fbd, int input_kind,
                                          const void* d_in, uint64_t ndat, uint64_t in_span,
                                          const float* lut256, int offset_binary, float* d_out,
                                          uint64_t out_span, uint64_t* npart);
/* The same filterbank with Detection::Engine and Fold::Engine fused into its
   last pass (the filterbank's output never reaches memory): the channels are
   detected to state (Detection.C:225-577) and folded by fold, whose plan
   (dspsr_b200_fold_set_bins) must cover exactly npart * nkeep output samples
   and whose nchan / npol must be input_nchan*nsub / the state's products. */
int dspsr_b200_filterbank_during_perform_fold (dspsr_b200_filterbank_during* fbd,
                                               int input_kind, const void* d_in, uint64_t ndat,
                                               uint64_t in_span, const float* lut256,
                                               int offset_binary, dspsr_b200_fold* fold,
                                               int state, uint64_t* npart);

/* ---------------------------------------------------------------------- */
/* Detection::Engine (CUDA::DetectionEngine, Signal/General/DetectionCUDA.cu;*/
/* callers Detection.C:237-242, 483-489)                                    */
/* ---------------------------------------------------------------------- */

/* square_law / polarimetry on dual-pol complex FPT input; output FPT floats,
   (ichan*nout + k)*out_span, nout = 1, 2, 4, 4 for the four states. */
int dspsr_b200_detect (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span,
                       uint64_t ndat, unsigned nchan, int state, float* d_out,
                       uint64_t out_span);

/* ---------------------------------------------------------------------- */
/* SpectralKurtosis::Engine compute / detect_ft / mask for one resolution  */
/* with noverlap 1 (CUDA::SpectralKurtosisEngine,                           */
/* Signal/General/SpectralKurtosisCUDA.cu:45-99; host loop                  */
/* SpectralKurtosis.C:542-671, 674-798, 1105-1222, 1465-1566)               */
/* ---------------------------------------------------------------------- */

/* Complex FPT input (span in complex samples), npart = ndat / M blocks of M
   samples per channel.  Per (block, channel): S1 and S2 of every pol summed
   as the reference does, the SK estimator of each pol tested against
   [lower, upper] (a block with 1 or 2 counted samples is zapped, one with
   none is not), and the block of every pol copied to d_out with zapped
   blocks set to zero.  d_out may equal d_in (same span): only zapped blocks
   are then written.  Optional device outputs (null to skip):
   d_sums[(ipart*nchan + ichan)*npol + ipol][2] = (S1, S2) as float,
   d_counts[ipart*nchan + ichan] = samples counted (zero_is_valid = 0 skips
   zero samples), d_mask[ipart*nchan + ichan] = 1 where zapped, *d_zapped
   (device uint64) += zapped blocks.  npol is 1 or 2; M and the spans are
   even; d_in and d_out are 16-byte aligned; npol*4*(M + 8) bytes at most
   224 KiB, i.e. M <= 28664 for two pols. */
int dspsr_b200_sk (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span,
                   uint64_t ndat, unsigned nchan, unsigned npol, unsigned M, int zero_is_valid,
                   unsigned Nd, float lower, float upper, float* d_out, uint64_t out_span,
                   float* d_sums, uint32_t* d_counts, uint8_t* d_mask, uint64_t* d_zapped,
                   uint64_t* npart_out);

/* The same engine step by step, as SpectralKurtosis::transformation drives
   it (SpectralKurtosis.C:542-671; CUDA::SpectralKurtosisEngine,
   SpectralKurtosisCUDA.cu:45-99).  Layouts as for dspsr_b200_sk. */
/* Engine::compute (SpectralKurtosis.C:674-798): S1, S2 (d_sums, float) and
   the counted samples (d_counts, optional) of every (part, chan, pol); the
   input is not written.  noverlap > 1 (Resolution::prepare, :251-281): blocks
   of M samples every M / noverlap samples, npart = (ndat - (M - M/noverlap))
   / (M / noverlap). */
int dspsr_b200_sk_compute (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span,
                           uint64_t ndat, unsigned nchan, unsigned npol, unsigned M,
                           unsigned noverlap, int zero_is_valid, float* d_sums,
                           uint32_t* d_counts, uint64_t* npart);
/* Engine::detect_ft (detect_skfb, SpectralKurtosis.C:1105-1222) with the
   thresholds given: d_mask[part][chan] set to 1 where zapped (others left as
   they are); d_counts NULL means M counted everywhere; *d_zapped (device,
   optional) += zapped cells. */
int dspsr_b200_sk_detect_ft (dspsr_b200_context* ctx, const float* d_sums,
                             const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                             unsigned npol, unsigned M, unsigned Nd, float lower, float upper,
                             uint8_t* d_mask, uint64_t* d_zapped);
/* Engine::detect_tscr (SpectralKurtosis.C:1012-1098): each channel's sums
   over all parts tested against the limits for its total count (SKLimits of
   that count, std_devs, npol tests); every part of a zapped channel is set in
   d_mask.  Synchronises; *nzapped_chan = channels zapped. */
int dspsr_b200_sk_detect_tscr (dspsr_b200_context* ctx, const float* d_sums,
                               const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                               unsigned npol, unsigned M, unsigned Nd, float std_devs,
                               uint8_t* d_mask, uint32_t* nzapped_chan);
/* Several resolutions (SpectralKurtosis::detect, SpectralKurtosis.C:830-
   915).  tscrunch_sums (:917-986): coarse part q of npart_to sums the fine
   parts q*offset + i*offset, i < nsum (nsum = M_coarse / M_fine, offset =
   the ratio of the two resolutions' block strides -- the reference's own
   indexing), sums and counts; the fine sums hold npart_from parts. */
int dspsr_b200_sk_tscrunch (dspsr_b200_context* ctx, const float* d_sums,
                            const uint32_t* d_counts, uint64_t npart_from, uint64_t npart_to,
                            unsigned nchan, unsigned npol, unsigned nsum, unsigned offset,
                            float* d_sums_out, uint32_t* d_counts_out);
/* detect_skfb at one resolution (:1105-1222): each (part, chan) is tested
   against SKLimits(count, std_devs) with Nd and npol tests (get_limits,
   :988-1008); a zapped cell sets nflag cells of the finest mask, flag_step
   fine parts apart, from fine part q * flag_offset (nflag = M / M_finest,
   flag_step = the finest noverlap, flag_offset = nflag * flag_step /
   noverlap; all 1 at the finest resolution).  Synchronises. */
int dspsr_b200_sk_detect_skfb (dspsr_b200_context* ctx, const float* d_sums,
                               const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                               unsigned npol, unsigned Nd, float std_devs, unsigned nflag,
                               unsigned flag_step, unsigned flag_offset, uint8_t* d_mask,
                               uint64_t mask_npart, uint64_t* d_zapped);
/* mask (:1465-1566) with overlapping blocks: npart parts of M samples,
   offset apart, from input sample idat_start, mask rows from part nskip; a
   sample takes the decision of the last part that covers it, as the
   reference's part-after-part copy leaves it.  Out of place; writes
   (npart - 1) * offset + M samples per span. */
int dspsr_b200_sk_mask_overlap (dspsr_b200_context* ctx, const uint8_t* d_mask,
                                const float* d_in, uint64_t in_span, float* d_out,
                                uint64_t out_span, unsigned nchan, unsigned npol, unsigned M,
                                unsigned offset, uint64_t npart, uint64_t nskip,
                                uint64_t idat_start);
/* Engine::reset_mask and count_mask (synchronises) */
int dspsr_b200_sk_reset_mask (dspsr_b200_context* ctx, uint8_t* d_mask, uint64_t npart,
                              unsigned nchan);
int dspsr_b200_sk_count_mask (dspsr_b200_context* ctx, const uint8_t* d_mask, uint64_t npart,
                              unsigned nchan, uint64_t* nzapped);
/* Engine::mask (SpectralKurtosis.C:1465-1566): the ndat/M whole blocks of
   d_in copied to d_out with the masked blocks zeroed (d_out == d_in: in
   place, only those blocks written). */
int dspsr_b200_sk_mask (dspsr_b200_context* ctx, const uint8_t* d_mask, const float* d_in,
                        uint64_t in_span, float* d_out, uint64_t out_span, uint64_t ndat,
                        unsigned nchan, unsigned npol, unsigned M);

/* ---------------------------------------------------------------------- */
/* Learned RFI-mask proposer in front of SpectralKurtosis.  It has no       */
/* counterpart in the reference; it proposes the mask that                  */
/* SpectralKurtosis::detect_skfb (SpectralKurtosis.C:1105-1222) would set,  */
/* from features of the SK sums (SpectralKurtosis::compute, :674-798), and   */
/* defers to the SK mask where it is not confident.                         */
/* ---------------------------------------------------------------------- */

typedef struct dspsr_b200_rfi_proposer dspsr_b200_rfi_proposer;
/* nchan in [1, 512] channels per block of M samples (Nd integrated
   samples each), features for up to max_npart blocks, training batches of
   up to max_batch_blocks blocks; weights initialised from seed. */
int dspsr_b200_rfi_proposer_create (dspsr_b200_context* ctx, unsigned nchan, unsigned M,
                                    unsigned Nd, uint64_t max_npart, unsigned max_batch_blocks,
                                    uint64_t seed, dspsr_b200_rfi_proposer** proposer);
int dspsr_b200_rfi_proposer_destroy (dspsr_b200_rfi_proposer* proposer);
/* Features of npart blocks from the SK sums of dspsr_b200_sk (d_sums laid
   out [part][chan][pol][S1, S2], d_counts [part][chan] or NULL for M each). */
int dspsr_b200_rfi_proposer_features (dspsr_b200_rfi_proposer* proposer, const float* d_sums,
                                      const uint32_t* d_counts, uint64_t npart, unsigned npol);
/* steps of Adam (learning rate lr) on random runs of batch_blocks blocks of
   the current features, labels d_labels[part][chan] (1 = zapped, e.g. the
   mask of dspsr_b200_sk); zapped examples weigh pos_weight in the binary
   cross-entropy.  *mean_loss (optional) = mean loss per example. */
int dspsr_b200_rfi_proposer_train (dspsr_b200_rfi_proposer* proposer, const uint8_t* d_labels,
                                   unsigned steps, unsigned batch_blocks, float lr,
                                   float pos_weight, float* mean_loss);
/* The proposal for the current features on the tensor cores: probability
   p of "zap" per (part, chan) into d_prob (optional); d_mask[part][chan] =
   1 where p >= confidence, 0 where p <= 1 - confidence, else d_sk_mask's
   value (the SK fallback; p >= 0.5 when d_sk_mask is NULL).  *n_fallback
   (optional, synchronises) = the number of fallbacks.  confidence in
   [0.5, 1]. */
int dspsr_b200_rfi_proposer_infer (dspsr_b200_rfi_proposer* proposer, const uint8_t* d_sk_mask,
                                   float confidence, uint8_t* d_mask, float* d_prob,
                                   uint64_t* n_fallback);
/* the FP32 weights (host memory): *n = their count (params may be NULL) */
int dspsr_b200_rfi_proposer_get_params (dspsr_b200_rfi_proposer* proposer, float* params,
                                        unsigned* n);
int dspsr_b200_rfi_proposer_set_params (dspsr_b200_rfi_proposer* proposer, const float* params,
                                        unsigned n);
/* the current features, [part][chan][8] floats, into host memory */
int dspsr_b200_rfi_proposer_get_features (dspsr_b200_rfi_proposer* proposer, float* features);

/* ---------------------------------------------------------------------- */
/* Fold::Engine (CUDA::FoldEngine, Signal/Pulsar/FoldCUDA.cu:78-704;        */
/* callers Fold.C:760-887, 1011-1035)                                       */
/* ---------------------------------------------------------------------- */

int dspsr_b200_fold_create (dspsr_b200_context* ctx, unsigned nbin, unsigned nchan,
                            unsigned npol, dspsr_b200_fold** fold);
int dspsr_b200_fold_destroy (dspsr_b200_fold* fold);
/* Engine::set_bins(phi, phase_per_sample, ndat, idat_start) with
   use_set_bins = true (Fold.C:763-778): builds the bin plan of the sequential
   FP64 recurrence of Fold.C:815-818 exactly, as arithmetic segments, on the
   host in O(segments), and uploads it.  Returns ndat_folded. */
int dspsr_b200_fold_set_bins (dspsr_b200_fold* fold, double phi, double phase_per_sample,
                              uint64_t ndat, uint64_t idat_start, uint64_t* ndat_folded);
/* Engine::fold(): accumulate float FPT input (ndim 1) into the profiles */
int dspsr_b200_fold_fold (dspsr_b200_fold* fold, const float* d_in, uint64_t in_span);
/* writes the per-sample bin indices of the current plan (for parity checks) */
int dspsr_b200_fold_binplan (dspsr_b200_fold* fold, uint32_t* d_binplan);
/* Engine::synch(PhaseSeries*): profiles [chan][pol][bin] floats and hits[bin]
   into host memory */
int dspsr_b200_fold_get_profiles (dspsr_b200_fold* fold, float* profiles, uint32_t* hits);
int dspsr_b200_fold_reset (dspsr_b200_fold* fold);

/* ---------------------------------------------------------------------- */
/* Fused path: the SingleThread::run hot loop (SingleThread.C:687-736) over  */
/* Unpacker -> Convolution -> Detection -> Fold for one block, with the     */
/* InputBuffering overlap carry (InputBuffering.C:66-174), in one pass      */
/* through HBM per FFT.                                                      */
/* ---------------------------------------------------------------------- */

typedef struct
{
  /* observation */
  double centre_freq_mhz;   /* centre frequency of the band */
  double bandwidth_mhz;     /* signed bandwidth of the band */
  double dm;                /* dispersion measure, pc/cm^3 */
  unsigned nchan;           /* input channels (complex-sampled) */
  unsigned npol;            /* 1 or 2 */
  int input_kind;           /* DSPSR_B200_INT8_TFPD, _INT16_TFPD or _FLOAT_FPT */
  float lut[256];           /* 8-bit lookup table (BitTable) when INT8 */
  int offset_binary;        /* 16-bit encoding */
  int dual_sideband;        /* Observation::get_dual_sideband */
  int dc_centred;
  /* convolution */
  unsigned nfft;            /* FFT length per part (power of two) */
  unsigned nfilt_pos, nfilt_neg;
  int chirp_mode;           /* DSPSR_B200_CHIRP_REFERENCE or _FP64 */
  /* detection */
  int state;                /* DSPSR_B200_INTENSITY ... _STOKES */
  /* fold */
  unsigned nbin;
  double period_s;          /* constant folding period */
  double reference_phase;
  int64_t epoch_day, epoch_sec; double epoch_frac;   /* reference epoch MJD */
  int64_t start_day, start_sec; double start_frac;   /* MJD of input sample 0 */
  /* tuning: maximum scratch bytes for in-flight FFT parts (0 = default) */
  uint64_t scratch_bytes;
  /* FFT filterbank stage in front of the dedispersion (Filterbank with
     freq_res = 1, Filterbank.C:75-570): channels per input channel, 0 or 1 =
     none, else a power of two in [4, 4096]; blocks must then be multiples
     of it */
  unsigned filterbank_nchan;
  /* sub-integrations (Subint<Fold> with TimeDivide, Signal/Pulsar/dsp/
     Subint.h:206-332, TimeDivide.C): both zero = one integration, read by
     _get_profiles; otherwise each division is folded into its own profiles
     and handed out when closed (_set_unloader, or _pop_subint) */
  double subint_seconds;    /* TimeDivide::set_seconds (division length) */
  double subint_turns;      /* TimeDivide::set_turns, of period_s */
  int64_t subint_epoch_day, subint_epoch_sec;   /* TimeDivide::set_reference_epoch; */
  double subint_epoch_frac;                     /* all zero = none */
  unsigned subint_slots;    /* divisions held on the device at once (0 = 4); one
                               block may touch at most this many */
  /* tuning: 0 = compute a 64-channel filterbank of one dual-polarisation
     int8/int16 channel inside the convolution's first FFT pass where the
     FFT split allows it (its output then never goes through memory);
     -1 = always run the filterbank as a stage of its own */
  int fused_filterbank;
  /* DedispersionPipe's inter-channel dedispersion (-K, DedispersionPipe.C:
     435-470): each channel's response takes the fractional-sample remainder of
     its dispersion delay (Dedispersion.C:141-187) and a SampleDelay stage
     (SampleDelay.C:65-304) shifts the channels by whole samples before
     detection, so the channels' profiles line up; 0 = off */
  int interchannel;
  /* the convolution's row FFTs: DSPSR_B200_FFT_FP32 (0), _BF16X3 or _BF16X2
     (dspsr_b200_convolution_set_fft_precision) */
  int fft_precision;
  /* SpectralKurtosis between the convolution and detection, as LoadToFold
     sets it up with coherent dedispersion (LoadToFold1.C:310-351): sk_M > 0
     = blocks of sk_M samples (even, one resolution, noverlap 1), statistics
     of the convolution's zero-DM output, the mask applied to the dedispersed
     voltages, thresholds SKLimits(sk_M, 1, sk_std_devs (0 = 3), npol); the
     fold then counts a hit for every channel's non-zeroed sample (Fold.C:
     895-930, zeroed data).  Not with interchannel; a filterbank stage runs
     on its own (fused_filterbank is ignored). */
  unsigned sk_M;
  float sk_std_devs;
  /* tuning: the four-step split's row length, 8192 (0 = default) or 4096
     (nfft from 8192 to 131072, n1 = nfft / 4096 columns; the tensor-core rows
     need 8192) */
  unsigned row_length;
} dspsr_b200_pipeline_config;

int dspsr_b200_pipeline_create (dspsr_b200_context* ctx,
                                const dspsr_b200_pipeline_config* config,
                                dspsr_b200_pipeline** pipe);
int dspsr_b200_pipeline_destroy (dspsr_b200_pipeline* pipe);
/* The RFI-mask proposer (dspsr_b200_rfi_proposer_*, created on the same
   context, for the pipeline's channels and sk_M, with max_npart at least the
   SK blocks of one call) in front of the SK stage: each block's SK sums feed
   it, and its mask -- SK's own decision where it is less confident than
   `confidence` -- zeroes the dedispersed voltages.  NULL detaches it. */
int dspsr_b200_pipeline_set_rfi_proposer (dspsr_b200_pipeline* pipe,
                                          dspsr_b200_rfi_proposer* proposer, float confidence);
/* SpectralKurtosis of the pipeline so far: (block, channel) cells zapped
   and tested (SpectralKurtosis::Count; SK's own decisions); synchronises */
int dspsr_b200_pipeline_sk_counts (dspsr_b200_pipeline* pipe, uint64_t* zapped,
                                   uint64_t* tested);
/* Processes one block of ndat new input samples (device memory, layout given
   by input_kind; for FLOAT_FPT in_span is the complex-sample span per
   (chan, pol), otherwise ignored).  Samples that do not complete an FFT part
   are carried into the next call.  Returns the output samples folded. */
int dspsr_b200_pipeline_run (dspsr_b200_pipeline* pipe, const void* d_in, uint64_t ndat,
                             uint64_t in_span, uint64_t* ndat_folded);
/* Same, from host memory: the pipeline copies the block to the device on its
   stream (pinned host memory gives an asynchronous copy). */
int dspsr_b200_pipeline_run_host (dspsr_b200_pipeline* pipe, const void* h_in,
                                  uint64_t ndat, uint64_t* ndat_folded);
/* profiles [chan][nout][nbin] and hits[nbin] into host memory */
int dspsr_b200_pipeline_get_profiles (dspsr_b200_pipeline* pipe, float* profiles,
                                      uint32_t* hits);
/* The same without waiting (PhaseSeries read back while the next block is
   already on its way): queues the copies behind the blocks run so far and
   returns; dspsr_b200_pipeline_wait_profiles waits for the latest such copy
   and reports a timed-out device wait up to that point.  Give pinned host
   memory (cudaHostAlloc) for copies that overlap; keep the buffers untouched
   until the wait returns. */
int dspsr_b200_pipeline_get_profiles_async (dspsr_b200_pipeline* pipe, float* profiles,
                                            uint32_t* hits);
int dspsr_b200_pipeline_wait_profiles (dspsr_b200_pipeline* pipe);
int dspsr_b200_pipeline_reset (dspsr_b200_pipeline* pipe);
/* Per-kernel timing: when enabled, CUDA events are recorded on the context's
   stream around every kernel of the convolution path (column pass, row pass,
   inverse column pass with detect+fold, single-kernel path). */
int dspsr_b200_pipeline_profile (dspsr_b200_pipeline* pipe, int enable);
/* Milliseconds and launch counts per kernel kind since the last call
   (ms[5], launches[5]: columns, rows, inverse columns, single-kernel,
   filterbank). */
int dspsr_b200_pipeline_kernel_times (dspsr_b200_pipeline* pipe, double* ms,
                                      uint64_t* launches);
/* Kernels launched by this library since it was loaded. */
uint64_t dspsr_b200_kernel_launches (void);
/* shape of the plan: nfft, nkeep, FFT split n1 x n2, parts per batch */
int dspsr_b200_pipeline_info (dspsr_b200_pipeline* pipe, uint64_t* info8);

/* ---------------------------------------------------------------------- */
/* Sub-integrations                                                        */
/* ---------------------------------------------------------------------- */

#define DSPSR_B200_SUBINT_FOLD           0   /* fold a range of the block */
#define DSPSR_B200_SUBINT_CLOSE_PARTIAL  1   /* Subint::unload_partial */
#define DSPSR_B200_SUBINT_CLOSE_COMPLETE 2   /* Subint::transformation's unload */

/* one step of Subint<Fold>::transformation for a block (Subint.h:258-332) */
typedef struct
{
  int kind;                          /* DSPSR_B200_SUBINT_* */
  int end_reached;                   /* FOLD: the range ends its division */
  uint64_t idat_start, ndat;         /* FOLD: samples of the block */
  uint64_t division;                 /* FOLD: TimeDivide::get_division */
  int64_t lower_day, lower_sec;      /* FOLD: the division's start ... */
  double lower_frac;
  int64_t upper_day, upper_sec;      /* ... and end, rounded to whole samples */
  double upper_frac;
} dspsr_b200_subint_action;

typedef struct dspsr_b200_time_divide dspsr_b200_time_divide;

/* TimeDivide with a division length in seconds, or in turns of a constant
   period (TimeDivide.C:40-537 without a Pulsar::Predictor), driven by the
   per-block loop of Subint<Fold>.  Host only. */
int dspsr_b200_time_divide_create (double seconds, double turns, double period_s,
                                   int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                                   dspsr_b200_time_divide** td);
/* The actions for one block of ndat samples at rate (Hz) starting at the MJD
   (start_day, start_sec, start_frac): up to cap into actions, *n = count. */
int dspsr_b200_time_divide_block (dspsr_b200_time_divide* td, int64_t start_day,
                                  int64_t start_sec, double start_frac, uint64_t ndat,
                                  double rate, dspsr_b200_subint_action* actions, uint64_t cap,
                                  uint64_t* n);
int dspsr_b200_time_divide_destroy (dspsr_b200_time_divide* td);

/* A closed sub-integration of the pipeline (the PhaseSeries handed to
   PhaseSeriesUnloader::unload / partial) */
typedef struct
{
  uint64_t division;             /* TimeDivide division index */
  uint64_t ndat_folded;          /* output samples folded into it */
  uint64_t first_sample;         /* global output index of the first of them */
  int64_t lower_day, lower_sec;  /* division start */
  double lower_frac;
  int64_t upper_day, upper_sec;  /* division end */
  double upper_frac;
  double integration_length;     /* ndat_folded / rate, seconds */
  int complete;                  /* its end was reached (else the data stopped) */
} dspsr_b200_subint;

/* PhaseSeriesUnloader::unload: called in division order on the calling
   thread with profiles [chan][nout][nbin] and hits[nbin] in host memory valid
   for the call.  A closed division's copy to the host is queued behind the
   block's kernels and its callback runs in the first later _run, _run_host,
   _run_dada, _set_unloader, _reset or _finish call that finds the copy done;
   _finish delivers all that remain. */
typedef void (*dspsr_b200_unload_fn) (void* user, const dspsr_b200_subint* subint,
                                      const float* profiles, const uint32_t* hits);
int dspsr_b200_pipeline_set_unloader (dspsr_b200_pipeline* pipe, dspsr_b200_unload_fn fn,
                                      void* user);
/* closed sub-integrations waiting (when no unloader is set) */
int dspsr_b200_pipeline_subints_ready (dspsr_b200_pipeline* pipe, uint64_t* n);
/* the oldest closed sub-integration into host memory; ESTATE when none */
int dspsr_b200_pipeline_pop_subint (dspsr_b200_pipeline* pipe, dspsr_b200_subint* subint,
                                    float* profiles, uint32_t* hits);
/* Subint::finish (Subint.h:345-362): closes the open division (partial) */
int dspsr_b200_pipeline_finish (dspsr_b200_pipeline* pipe);

/* ---------------------------------------------------------------------- */
/* DADA file source (host only, no GPU needed except for _pipeline_run_dada) */
/* ---------------------------------------------------------------------- */

typedef struct dspsr_b200_dada_file dspsr_b200_dada_file;

/* The observation parameters DADAFile::open_file (Kernel/Classes/DADAFile.C:
   48-68) loads through ASCIIObservation::load (ASCIIObservation.C:88-410)
   and File::open (File.C:175-190, fstat_file_ndat :366-390). */
typedef struct
{
  uint64_t header_bytes;     /* bytes before the first sample (HDR_SIZE; 0 with
                                an adjacent header file that defines none) */
  uint64_t ndat;             /* NDAT when the header gives it, else file_ndat */
  uint64_t file_ndat;        /* samples the file holds after the header */
  uint64_t bits_per_sample;  /* nbit * npol * nchan * ndim */
  uint64_t obs_offset;       /* OBS_OFFSET (or OFFSET) in bytes */
  int64_t picoseconds;       /* PICOSECONDS, 0 when absent */
  int64_t start_day, start_sec;  /* MJD of sample 0: UTC_START + PICOSECONDS */
  double start_frac;             /* + the samples in OBS_OFFSET; 0 for TBD */
  double centre_freq_mhz;    /* FREQ */
  double bandwidth_mhz;      /* BW */
  double tsamp_us;           /* TSAMP, microseconds */
  double rate_hz;            /* 1 / (TSAMP * 1e-6) */
  double hdr_version;        /* HDR_VERSION, 0 when absent */
  unsigned nchan, npol, nbit, ndim;   /* defaults 1, 1, 2, 1 when absent */
  int dual_sideband;         /* DSB: 1, 0, or -1 when absent */
  int adjacent_header;       /* the header came from an adjacent .hdr file */
  char telescope[64], receiver[64], source[64], mode[64];
  char instrument[64], utc_start[64], state[64], basis[64];
} dspsr_b200_dada_info;

/* Message of the calling thread's last failed host-only call (the DADA and
   header calls below, which have no context). */
const char* dspsr_b200_host_error (void);

/* ascii_header_get with a "%s" code (Kernel/Classes/ascii_header.c:34-56,
   117-142): copies the whitespace-delimited value after KEYWORD (a keyword
   at the start of the header, or after a newline or backslash and followed
   by a blank) into value (at most value_cap-1 bytes).  Returns 1, or -1 when
   the keyword or its value is absent. */
int dspsr_b200_ascii_header_get (const char* header, const char* keyword, char* value,
                                 uint64_t value_cap);
/* ascii_header_set (ascii_header.c:58-115): replaces the keyword's value in
   place, or inserts the line before "DATA\n" or at the end.  header_cap is the
   size of the buffer; ETOOBIG when the result would not fit. */
int dspsr_b200_ascii_header_set (char* header, uint64_t header_cap, const char* keyword,
                                 const char* value);
/* ASCIIObservation::load over a NUL-terminated header; header_bytes goes to
   info->header_bytes and file_ndat stays 0.  EINVAL names the first missing
   required keyword (TELESCOPE SOURCE FREQ BW NPOL NBIT TSAMP UTC_START
   OBS_OFFSET) or the invalid NDIM. */
int dspsr_b200_dada_parse (const char* header, uint64_t header_bytes, dspsr_b200_dada_info* info);
/* DADAFile::open_file + File::open: DADAHeader::load_header (DADAHeader.C:
   56-139; HDR_SIZE grows the read until the whole header is in, an absent
   HDR_SIZE sends it to the adjacent .hdr file), then the parse above and the
   sample count from the file size when NDAT is absent. */
int dspsr_b200_dada_open (const char* filename, dspsr_b200_dada_file** file,
                          dspsr_b200_dada_info* info);
/* DADAFile::is_valid (DADAFile.C:32-43, DADAHeader::valid :146-174): 1 when
   the header loads and defines HDR_VERSION and INSTRUMENT, else 0. */
int dspsr_b200_dada_is_valid (const char* filename);
/* the loaded header text (NUL-terminated) and its buffer size */
int dspsr_b200_dada_header (const dspsr_b200_dada_file* file, const char** text, uint64_t* size);
/* File::load_bytes (File.C:248-300): nsamp samples from sample start_sample
   into host memory dst, stopping at the end of the data (NDAT or the file);
   *nread = samples read.  Sample boundaries must fall on whole bytes. */
int dspsr_b200_dada_read (dspsr_b200_dada_file* file, uint64_t start_sample, uint64_t nsamp,
                          void* dst, uint64_t* nread);
int dspsr_b200_dada_close (dspsr_b200_dada_file* file);

/* The file-driven SingleThread loop: nsamp samples (0 = to the end of the
   data) from start_sample, in blocks of block_ndat, through two pinned host
   buffers: the read of one block overlaps the upload and kernels of the block
   before.  The file must match the pipeline: NCHAN, NPOL, NDIM 2 and NBIT 8
   (INT8_TFPD) or 16 (INT16_TFPD).  With a filterbank stage block_ndat must be
   a multiple of its channel count and a short last block is cut to one.
   *ndat_read = samples passed to the pipeline, *ndat_folded = output samples
   folded.  Returns after queueing the last block, like _pipeline_run_host. */
int dspsr_b200_pipeline_run_dada (dspsr_b200_pipeline* pipe, dspsr_b200_dada_file* file,
                                  uint64_t start_sample, uint64_t nsamp, uint64_t block_ndat,
                                  uint64_t* ndat_read, uint64_t* ndat_folded);

#ifdef __cplusplus
}
#endif

#endif
