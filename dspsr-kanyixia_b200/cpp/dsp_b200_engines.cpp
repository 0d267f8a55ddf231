// dsp_b200_engines.cpp -- C++ engines over the C ABI (see dsp_b200_engines.h)

#include "dsp_b200_engines.h"

#include <string>

namespace b200 {

namespace {
std::string message (dspsr_b200_context* ctx, const char* where)
{
  std::string m = where;
  if (ctx)
  {
    m += ": ";
    m += dspsr_b200_last_error (ctx);
  }
  return m;
}
} // namespace

Context::Context (int device, void* stream)
{
  const int rc = dspsr_b200_context_create (device, stream, &ctx);
  if (rc)
    throw Error (rc, rc == DSPSR_B200_ENODEV ? "Context: no CUDA device"
                                             : "Context: dspsr_b200_context_create failed");
}

Context::~Context ()
{
  if (ctx) dspsr_b200_context_destroy (ctx);
}

void Context::check (int rc, const char* where) const
{
  if (rc) throw Error (rc, message (ctx, where));
}

void Context::synchronize () { check (dspsr_b200_synchronize (ctx), "synchronize"); }

// ---- convolution ------------------------------------------------------------

ConvolutionEngine::~ConvolutionEngine ()
{
  if (conv) dspsr_b200_convolution_destroy (conv);
}

void ConvolutionEngine::prepare (unsigned nchan, unsigned npol, unsigned nfft,
                                 unsigned nfilt_pos, unsigned nfilt_neg)
{
  if (conv) dspsr_b200_convolution_destroy (conv);
  conv = nullptr;
  ctx.check (dspsr_b200_convolution_create (ctx.handle (), nchan, npol, nfft, nfilt_pos,
                                            nfilt_neg, &conv),
             "ConvolutionEngine::prepare");
}

void ConvolutionEngine::copy_response (const float* response)
{
  ctx.check (dspsr_b200_convolution_copy_response (conv, response),
             "ConvolutionEngine::copy_response");
}

void ConvolutionEngine::set_dedispersion (double cf, double bw, double dm, int input_nchan,
                                          int dual_sideband, int chirp_mode)
{
  ctx.check (dspsr_b200_convolution_set_dedispersion (conv, cf, bw, dm, input_nchan,
                                                      dual_sideband, 0, chirp_mode, 0),
             "ConvolutionEngine::set_dedispersion");
}

uint64_t ConvolutionEngine::perform (const TimeSeriesView& in, TimeSeriesView& out)
{
  if (in.ndim != 2 || out.ndim != 2)
    throw Error (DSPSR_B200_ESTATE, "ConvolutionEngine::perform: complex data required");
  uint64_t npart = 0;
  ctx.check (dspsr_b200_convolution_perform (conv, in.base, in.span_floats / 2, in.ndat,
                                             out.base, out.span_floats / 2, &npart),
             "ConvolutionEngine::perform");
  return npart;
}

// ---- filterbank ---------------------------------------------------------------

uint64_t FilterbankEngine::perform (const TimeSeriesView& in, TimeSeriesView& out)
{
  if (out.nchan != in.nchan * nsub)
    throw Error (DSPSR_B200_ESTATE, "FilterbankEngine::perform: output nchan mismatch");
  uint64_t n = 0;
  ctx.check (dspsr_b200_filterbank (ctx.handle (), DSPSR_B200_FLOAT_FPT, in.base, in.ndat,
                                    in.span_floats / 2, in.nchan, in.npol, nsub, nullptr, 0,
                                    out.base, out.span_floats / 2, &n),
             "FilterbankEngine::perform");
  out.ndat = n;
  return n;
}

// ---- filterbank with a response --------------------------------------------

FilterbankDuringEngine::~FilterbankDuringEngine ()
{
  if (fbd) dspsr_b200_filterbank_during_destroy (fbd);
}

void FilterbankDuringEngine::setup (unsigned input_nchan, unsigned npol, unsigned nchan_subband,
                                    unsigned freq_res, unsigned nfilt_pos, unsigned nfilt_neg)
{
  if (fbd) dspsr_b200_filterbank_during_destroy (fbd);
  fbd = nullptr;
  dspsr_b200_fbd_config cfg {};
  cfg.input_nchan = input_nchan;
  cfg.npol = npol;
  cfg.nsub = nchan_subband;
  cfg.freq_res = freq_res;
  cfg.nfilt_pos = nfilt_pos;
  cfg.nfilt_neg = nfilt_neg;
  ctx.check (dspsr_b200_filterbank_during_create (ctx.handle (), &cfg, &fbd),
             "FilterbankDuringEngine::setup");
  nsub = nchan_subband;
  keep = freq_res - nfilt_pos - nfilt_neg;
}

void FilterbankDuringEngine::copy_response (const float* response)
{
  ctx.check (dspsr_b200_filterbank_during_copy_response (fbd, response),
             "FilterbankDuringEngine::copy_response");
}

void FilterbankDuringEngine::set_dedispersion (double cf, double bw, double dm, bool swapped,
                                               int chirp_mode)
{
  ctx.check (dspsr_b200_filterbank_during_set_dedispersion (fbd, cf, bw, dm, swapped ? 1 : 0,
                                                            chirp_mode),
             "FilterbankDuringEngine::set_dedispersion");
}

uint64_t FilterbankDuringEngine::perform (const TimeSeriesView& in, TimeSeriesView& out)
{
  if (out.nchan != in.nchan * nsub)
    throw Error (DSPSR_B200_ESTATE, "FilterbankDuringEngine::perform: output nchan mismatch");
  uint64_t npart = 0;
  ctx.check (dspsr_b200_filterbank_during_perform (fbd, DSPSR_B200_FLOAT_FPT, in.base, in.ndat,
                                                   in.span_floats / 2, nullptr, 0, out.base,
                                                   out.span_floats / 2, &npart),
             "FilterbankDuringEngine::perform");
  out.ndat = npart * keep;
  return npart;
}

// ---- detection -------------------------------------------------------------

void DetectionEngine::square_law (const TimeSeriesView& in, TimeSeriesView& out)
{
  ctx.check (dspsr_b200_detect (ctx.handle (), in.base, in.span_floats / 2, in.ndat, in.nchan,
                                DSPSR_B200_INTENSITY, out.base, out.span_floats),
             "DetectionEngine::square_law");
}

void DetectionEngine::polarimetry (unsigned ndim, const TimeSeriesView& in, TimeSeriesView& out,
                                   int state)
{
  (void) ndim;   // output is FPT with one float per product (ndim 1)
  ctx.check (dspsr_b200_detect (ctx.handle (), in.base, in.span_floats / 2, in.ndat, in.nchan,
                                state, out.base, out.span_floats),
             "DetectionEngine::polarimetry");
}

// ---- fold -------------------------------------------------------------------

FoldEngine::~FoldEngine ()
{
  if (fold_) dspsr_b200_fold_destroy (fold_);
}

void FoldEngine::ensure (unsigned nc, unsigned np)
{
  if (fold_ && nc == nchan && np == npol) return;
  if (fold_) dspsr_b200_fold_destroy (fold_);
  fold_ = nullptr;
  nchan = nc;
  npol = np;
  ctx.check (dspsr_b200_fold_create (ctx.handle (), nbin, nchan, npol, &fold_),
             "FoldEngine::setup");
}

void FoldEngine::setup (unsigned nc, unsigned np) { ensure (nc, np); }

void FoldEngine::set_nbin (unsigned n)
{
  if (n != nbin && fold_)
  {
    dspsr_b200_fold_destroy (fold_);
    fold_ = nullptr;
  }
  nbin = n;
}

void FoldEngine::set_ndat (uint64_t n, uint64_t idat_start)
{
  (void) idat_start;
  ndat = n;
}

uint64_t FoldEngine::set_bins (double phi, double pps, uint64_t n, uint64_t idat_start)
{
  if (!fold_) ensure (nchan ? nchan : 1, npol ? npol : 1);
  ctx.check (dspsr_b200_fold_set_bins (fold_, phi, pps, n, idat_start, &ndat_folded),
             "FoldEngine::set_bins");
  hits_valid = false;
  return ndat_folded;
}

unsigned FoldEngine::get_bin_hits (unsigned ibin)
{
  if (!hits_valid)
  {
    std::vector<float> p;
    synch (p, hits_cache);
  }
  return ibin < hits_cache.size () ? hits_cache[ibin] : 0;
}

void FoldEngine::fold (const TimeSeriesView& in)
{
  ensure (in.nchan, in.npol);
  ctx.check (dspsr_b200_fold_fold (fold_, in.base, in.span_floats), "FoldEngine::fold");
  hits_valid = false;
}

void FoldEngine::synch (std::vector<float>& profiles, std::vector<uint32_t>& hits)
{
  profiles.assign (uint64_t (nchan) * npol * nbin, 0.f);
  hits.assign (nbin, 0u);
  ctx.check (dspsr_b200_fold_get_profiles (fold_, profiles.data (), hits.data ()),
             "FoldEngine::synch");
  hits_cache = hits;
  hits_valid = true;
}

// ---- unpack -----------------------------------------------------------------

void unpack8 (Context& ctx, const void* d_bytes, const float lut256[256], TimeSeriesView& out)
{
  ctx.check (dspsr_b200_unpack8 (ctx.handle (), d_bytes, out.ndat, out.nchan, out.npol,
                                 out.ndim, lut256, out.base, out.span_floats),
             "unpack8");
}

// ---- spectral kurtosis ------------------------------------------------------

uint64_t SpectralKurtosisEngine::compute (const TimeSeriesView& in, SKSums& sums, unsigned M,
                                          bool zero_is_valid)
{
  if (in.ndim != 2)
    throw Error (DSPSR_B200_ESTATE, "SpectralKurtosisEngine::compute: complex data required");
  uint64_t npart = 0;
  ctx.check (dspsr_b200_sk_compute (ctx.handle (), in.base, in.span_floats / 2, in.ndat, in.nchan,
                                    in.npol, M, 1, zero_is_valid ? 1 : 0, sums.sums, sums.counts,
                                    &npart),
             "SpectralKurtosisEngine::compute");
  sums.npart = npart;
  sums.nchan = in.nchan;
  sums.npol = in.npol;
  sums.M = M;
  return npart;
}

void SpectralKurtosisEngine::detect_ft (const SKSums& s, uint8_t* mask, float upper, float lower)
{
  ctx.check (dspsr_b200_sk_detect_ft (ctx.handle (), s.sums, s.counts, s.npart, s.nchan, s.npol,
                                      s.M, nd, lower, upper, mask, nullptr),
             "SpectralKurtosisEngine::detect_ft");
}

unsigned SpectralKurtosisEngine::detect_tscr (const SKSums& s, uint8_t* mask, float std_devs)
{
  uint32_t n = 0;
  ctx.check (dspsr_b200_sk_detect_tscr (ctx.handle (), s.sums, s.counts, s.npart, s.nchan, s.npol,
                                        s.M, nd, std_devs, mask, &n),
             "SpectralKurtosisEngine::detect_tscr");
  return n;
}

void SpectralKurtosisEngine::reset_mask (uint8_t* mask, uint64_t npart, unsigned nchan)
{
  ctx.check (dspsr_b200_sk_reset_mask (ctx.handle (), mask, npart, nchan),
             "SpectralKurtosisEngine::reset_mask");
}

uint64_t SpectralKurtosisEngine::count_mask (const uint8_t* mask, uint64_t npart, unsigned nchan)
{
  uint64_t n = 0;
  ctx.check (dspsr_b200_sk_count_mask (ctx.handle (), mask, npart, nchan, &n),
             "SpectralKurtosisEngine::count_mask");
  return n;
}

void SpectralKurtosisEngine::mask (const uint8_t* mask, const TimeSeriesView& in,
                                   TimeSeriesView& out, unsigned M)
{
  ctx.check (dspsr_b200_sk_mask (ctx.handle (), mask, in.base, in.span_floats / 2, out.base,
                                 out.span_floats / 2, in.ndat, in.nchan, in.npol, M),
             "SpectralKurtosisEngine::mask");
  out.ndat = (in.ndat / M) * M;
}

// ---- inverse filterbank -----------------------------------------------------

InverseFilterbankEngine::~InverseFilterbankEngine ()
{
  if (ifb) dspsr_b200_inverse_filterbank_destroy (ifb);
}

void InverseFilterbankEngine::setup (const dspsr_b200_ifb_config& cfg)
{
  if (ifb) dspsr_b200_inverse_filterbank_destroy (ifb);
  ifb = nullptr;
  ctx.check (dspsr_b200_inverse_filterbank_create (ctx.handle (), &cfg, &ifb),
             "InverseFilterbankEngine::setup");
}

void InverseFilterbankEngine::set_response (const float* response)
{
  ctx.check (dspsr_b200_inverse_filterbank_copy_response (ifb, response),
             "InverseFilterbankEngine::set_response");
}

void InverseFilterbankEngine::set_apodization (const float* temporal, const float* spectral)
{
  ctx.check (dspsr_b200_inverse_filterbank_set_apodization (ifb, temporal, spectral),
             "InverseFilterbankEngine::set_apodization");
}

uint64_t InverseFilterbankEngine::perform (const TimeSeriesView& in, TimeSeriesView& out)
{
  if (in.ndim != 2 || out.ndim != 2)
    throw Error (DSPSR_B200_ESTATE, "InverseFilterbankEngine::perform: complex data required");
  uint64_t npart = 0;
  ctx.check (dspsr_b200_inverse_filterbank_perform (ifb, DSPSR_B200_FLOAT_FPT, in.base, in.ndat,
                                                    in.span_floats / 2, nullptr, 0, out.base,
                                                    out.span_floats / 2, &npart),
             "InverseFilterbankEngine::perform");
  const std::vector<uint64_t> i = info ();
  out.ndat = npart * i[3];
  return npart;
}

std::vector<uint64_t> InverseFilterbankEngine::info ()
{
  std::vector<uint64_t> v (10, 0);
  ctx.check (dspsr_b200_inverse_filterbank_info (ifb, v.data ()), "InverseFilterbankEngine::info");
  return v;
}

// ---- unpackers --------------------------------------------------------------

void Unpacker::set_table (const float lut256[256])
{
  for (int i = 0; i < 256; i++) lut[i] = lut256[i];
  have_lut = true;
}

void Unpacker::unpack (const void* d_words, TimeSeriesView& out)
{
  if (kind == EightBit)
  {
    if (!have_lut) throw Error (DSPSR_B200_ESTATE, "Unpacker::unpack: no 8-bit table set");
    ctx.check (dspsr_b200_unpack8 (ctx.handle (), d_words, out.ndat, out.nchan, out.npol,
                                   out.ndim, lut, out.base, out.span_floats),
               "Unpacker::unpack (8-bit)");
  }
  else
    ctx.check (dspsr_b200_unpack16 (ctx.handle (), d_words, out.ndat, out.nchan, out.npol,
                                    out.ndim, offset_binary ? 1 : 0, out.base, out.span_floats),
               "Unpacker::unpack (16-bit)");
}

} // namespace b200
