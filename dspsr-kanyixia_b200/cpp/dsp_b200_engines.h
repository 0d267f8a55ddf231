// dsp_b200_engines.h -- C++ engines with the shapes of DSPSR's CUDA engines,
// implemented over the C ABI of libdspsr_b200.so (include/dspsr_b200.h).
//
// DSPSR's operations (dsp::Convolution, dsp::Detection, dsp::Fold,
// dsp::Filterbank, dsp::GenericEightBitUnpacker) keep all bookkeeping and
// call a pluggable Engine with raw device pointers, strides and counts.  The
// classes here have the method names and argument meanings of those engines
// (recovered from their call sites, because the reference's Signal/General
// headers are not part of the snapshot):
//
//   Convolution::Engine  prepare / copy_response / perform      Convolution.C:446-452, 656-698
//   Filterbank::Engine   setup / perform                        Filterbank.C:245-256, 549-565
//   Detection::Engine    square_law / polarimetry               Detection.C:237-242, 483-489
//   Fold::Engine         set_nbin / set_ndat / set_bins / fold  Fold.C:760-887, 1011-1035
//                        get_bin_hits / synch
//   SpectralKurtosis::Engine  setup / compute / detect_ft /     SpectralKurtosisCUDA.cu:28-104
//                        detect_tscr / reset_mask / count_mask / mask
//   InverseFilterbank::Engine setup / perform                   InverseFilterbank.C:215-228, 441-449
//   Unpacker             matches / unpack / set_device          Unpacker.h:57-103
//
// A TimeSeriesView carries what those call sites read from a dsp::TimeSeries
// (get_datptr(0,0), get_nfloat_span(), get_ndat(), get_nchan(), get_npol()).
// Every failure throws b200::Error carrying the C ABI's status and message,
// as the reference throws its Error (InvalidParam / InvalidState / FailedCall).
#pragma once

#include "dspsr_b200.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace b200 {

class Error : public std::runtime_error
{
public:
  Error (int code, const std::string& what) : std::runtime_error (what), code (code) {}
  int code;
};

// The fields of a dsp::TimeSeries that the engines use.  FPT order: the data
// of (chan, pol) start at base + (chan*npol + pol) * span_floats.
struct TimeSeriesView
{
  float* base = nullptr;        // get_datptr (0, 0), device memory
  uint64_t span_floats = 0;     // get_nfloat_span ()
  uint64_t ndat = 0;            // get_ndat ()
  unsigned nchan = 1;
  unsigned npol = 1;
  unsigned ndim = 2;            // 2 = complex (Signal::Analytic)
};

// One device + stream (CUDA::DeviceMemory(stream) in SingleThread::construct)
class Context
{
public:
  explicit Context (int device = 0, void* stream = nullptr);
  ~Context ();
  Context (const Context&) = delete;
  Context& operator= (const Context&) = delete;
  dspsr_b200_context* handle () const { return ctx; }
  void check (int rc, const char* where) const;
  void synchronize ();
private:
  dspsr_b200_context* ctx = nullptr;
};

// CUDA::ConvolutionEngine
class ConvolutionEngine
{
public:
  explicit ConvolutionEngine (Context& ctx) : ctx (ctx) {}
  ~ConvolutionEngine ();
  // Engine::prepare(Convolution*): the sizes Convolution::prepare computed
  void prepare (unsigned nchan, unsigned npol, unsigned nfft, unsigned nfilt_pos,
                unsigned nfilt_neg);
  // Engine::copy_response(const Response*): nchan*nfft complex floats, FFT order
  void copy_response (const float* response);
  // Dedispersion built on the device (FP64 phase); chirp_mode as in the C ABI
  void set_dedispersion (double centre_freq, double bandwidth, double dm, int input_nchan,
                         int dual_sideband, int chirp_mode = DSPSR_B200_CHIRP_REFERENCE);
  // Engine::perform(input, output, npart); returns npart
  uint64_t perform (const TimeSeriesView& input, TimeSeriesView& output);
private:
  Context& ctx;
  dspsr_b200_convolution* conv = nullptr;
};

// CUDA::FilterbankEngine for freq_res = 1 (no "During" convolution)
class FilterbankEngine
{
public:
  FilterbankEngine (Context& ctx, unsigned nchan_subband) : ctx (ctx), nsub (nchan_subband) {}
  // Engine::perform(in, out, npart, in_step, out_step) with in_step = nsub and
  // out_step = 1 per part; returns the output samples per channel
  uint64_t perform (const TimeSeriesView& input, TimeSeriesView& output);
private:
  Context& ctx;
  unsigned nsub;
};

// CUDA::FilterbankEngine with a response (the "During" filterbank, -F N:D):
// one nsub*freq_res-point FFT per part, the response, freq_res-point inverse
// FFTs per output channel (FilterbankEngineCPU.C:379-535)
class FilterbankDuringEngine
{
public:
  explicit FilterbankDuringEngine (Context& ctx) : ctx (ctx) {}
  ~FilterbankDuringEngine ();
  // Engine::setup(Filterbank*): the sizes Filterbank::do_prepare computed
  void setup (unsigned input_nchan, unsigned npol, unsigned nchan_subband, unsigned freq_res,
              unsigned nfilt_pos, unsigned nfilt_neg);
  // Engine::copy_response: [input_nchan*nchan_subband][freq_res] complex floats
  void copy_response (const float* response);
  void set_dedispersion (double centre_freq, double bandwidth, double dm, bool swapped = true,
                         int chirp_mode = DSPSR_B200_CHIRP_REFERENCE);
  // Engine::perform(in, out, npart, in_step, out_step); returns npart
  uint64_t perform (const TimeSeriesView& input, TimeSeriesView& output);
  uint64_t nkeep () const { return keep; }
private:
  Context& ctx;
  dspsr_b200_filterbank_during* fbd = nullptr;
  unsigned nsub = 0;
  uint64_t keep = 0;
};

// CUDA::DetectionEngine
class DetectionEngine
{
public:
  explicit DetectionEngine (Context& ctx) : ctx (ctx) {}
  void square_law (const TimeSeriesView& input, TimeSeriesView& output);           // Intensity
  void polarimetry (unsigned ndim, const TimeSeriesView& input, TimeSeriesView& output,
                    int state = DSPSR_B200_COHERENCE);
private:
  Context& ctx;
};

// CUDA::FoldEngine with use_set_bins = true
class FoldEngine
{
public:
  explicit FoldEngine (Context& ctx) : ctx (ctx) {}
  ~FoldEngine ();
  const bool use_set_bins = true;
  // Engine::setup (Fold.C:1011-1035): the input's channels and polarisations
  void setup (unsigned nchan, unsigned npol);
  void set_nbin (unsigned nbin);
  void set_ndat (uint64_t ndat, uint64_t idat_start);
  // Engine::set_bins(phi, phase_per_sample, ndat, idat_start): returns ndat_folded
  uint64_t set_bins (double phi, double phase_per_sample, uint64_t ndat, uint64_t idat_start);
  unsigned get_bin_hits (unsigned ibin);
  void fold (const TimeSeriesView& input);
  // Engine::synch(PhaseSeries*): profiles [chan][pol][bin] and hits
  void synch (std::vector<float>& profiles, std::vector<uint32_t>& hits);
  uint64_t get_ndat_folded () const { return ndat_folded; }
private:
  void ensure (unsigned nchan, unsigned npol);
  Context& ctx;
  dspsr_b200_fold* fold_ = nullptr;
  unsigned nbin = 0, nchan = 0, npol = 0;
  uint64_t ndat = 0, ndat_folded = 0;
  std::vector<uint32_t> hits_cache;
  bool hits_valid = false;
};

// GenericEightBitUnpacker::unpack_on_gpu: TFPD bytes on the device -> FPT
void unpack8 (Context& ctx, const void* d_bytes, const float lut256[256],
              TimeSeriesView& output);

// The block layout of the SK engine's sums and mask: S1, S2 per
// (part, chan, pol) as floats, counts and mask per (part, chan)
struct SKSums
{
  float* sums = nullptr;        // [npart][nchan][npol][2], device
  uint32_t* counts = nullptr;   // [npart][nchan], device (may be null: M counted)
  uint64_t npart = 0;
  unsigned nchan = 0, npol = 0, M = 0;
};

// CUDA::SpectralKurtosisEngine: the engine steps SpectralKurtosis::
// transformation drives one after another (compute, detect_ft or detect_tscr,
// count_mask, mask), each on the device
class SpectralKurtosisEngine
{
public:
  explicit SpectralKurtosisEngine (Context& ctx) : ctx (ctx) {}
  // Engine::setup: the integrated samples per value (SpectralKurtosis's Nd)
  void setup (unsigned Nd = 1) { nd = Nd; }
  // Engine::compute(input, sums, sums_tscr, M): returns npart = ndat / M
  uint64_t compute (const TimeSeriesView& input, SKSums& sums, unsigned M,
                    bool zero_is_valid = true);
  // Engine::detect_ft(sums, mask, upper, lower)
  void detect_ft (const SKSums& sums, uint8_t* mask, float upper, float lower);
  // Engine::detect_tscr: each channel over all parts; returns channels zapped
  unsigned detect_tscr (const SKSums& sums, uint8_t* mask, float std_devs);
  void reset_mask (uint8_t* mask, uint64_t npart, unsigned nchan);
  uint64_t count_mask (const uint8_t* mask, uint64_t npart, unsigned nchan);
  // Engine::mask(mask, input, output, M)
  void mask (const uint8_t* mask, const TimeSeriesView& input, TimeSeriesView& output,
             unsigned M);
private:
  Context& ctx;
  unsigned nd = 1;
};

// InverseFilterbank's engine (InverseFilterbankEngineCPU.C:46-792 on the
// device): setup with the configuration InverseFilterbank::make_preparations
// derives, the response and apodizations, perform
class InverseFilterbankEngine
{
public:
  explicit InverseFilterbankEngine (Context& ctx) : ctx (ctx) {}
  ~InverseFilterbankEngine ();
  void setup (const dspsr_b200_ifb_config& config);
  void set_response (const float* response);      // host, [output_nchan][Lout] complex
  void set_apodization (const float* temporal, const float* spectral);
  // Engine::perform(in, out, npart): complex FPT in and out; returns npart
  uint64_t perform (const TimeSeriesView& input, TimeSeriesView& output);
  // {kept bins, Lout, input step, output step, ...} as dspsr_b200_inverse_filterbank_info
  std::vector<uint64_t> info ();
private:
  Context& ctx;
  dspsr_b200_inverse_filterbank* ifb = nullptr;
};

// dsp::Unpacker on the device: GenericEightBitUnpacker (BitTable lookup) and
// SixteenBitUnpacker (float(x) + 0.5, optional offset binary)
class Unpacker
{
public:
  enum Kind { EightBit, SixteenBit };
  Unpacker (Context& ctx, Kind kind) : ctx (ctx), kind (kind) {}
  // Unpacker::matches(const Observation*): NBIT of the data
  bool matches (unsigned nbit) const { return nbit == (kind == EightBit ? 8u : 16u); }
  // Unpacker::get_device_supported / set_device: always the device here
  bool get_device_supported () const { return true; }
  void set_table (const float lut256[256]);        // 8-bit: the BitTable values
  void set_offset_binary (bool on) { offset_binary = on; }
  // Unpacker::unpack: TFPD words on the device -> FPT
  void unpack (const void* d_words, TimeSeriesView& output);
private:
  Context& ctx;
  Kind kind;
  float lut[256] = {};
  bool have_lut = false, offset_binary = false;
};

} // namespace b200
