// kernels.cuh -- launch interface of the B200 hot-path kernels
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>
#include <stdint.h>

#include "host_rules.h"

namespace b200 {

enum InputKind { IN_INT8 = 0, IN_INT16 = 1, IN_FLOAT = 2 };
enum OutMode { OUT_VOLTAGE = 0, OUT_FOLD = 1 };

// Where complex sample t of (chan, pol) lives: a carried prefix of npre
// samples followed by the main block, both in the same layout.
struct InputView
{
  int kind;
  const void* pre;
  const void* main;
  uint64_t npre;
  uint64_t pre_span;     // FPT span (complex samples) of the prefix
  uint64_t main_span;    // FPT span of the main block
  unsigned nchan, npol;
  int offset_binary;     // int16 encoding
  // 64: the input is raw TFPD (one input channel, two polarisations) and the
  // convolution's 64 channels come from a 64-point filterbank computed inside
  // the forward column pass; times (and npre) then count filterbank samples
  // of 64 raw samples, npre_raw = 64 * npre.  0: the input holds the
  // convolution's channels.
  unsigned fb_nsub = 0;
  // nonzero: the 8-bit table equals (float(x) + 0.5f) * lut_scale for every
  // two's-complement x (BitTable's tables do), and the filterbank column pass
  // computes the values instead of looking them up in shared memory
  float lut_scale = 0.f;
};

// Fold / detection epilogue
struct FoldView
{
  const FoldSegment* segs;
  int nseg;
  float* profiles;       // [chan][nout][stride]
  unsigned* hits;        // [stride]
  unsigned nbin;
  unsigned stride;       // profile columns: nbin times the sub-integration slots
  // when set: the profile column of every sample of the block (or NO_COLUMN),
  // computed once for all channels instead of from segs in every channel
  const unsigned* cols = nullptr;
  int state;
  int nout;
};

// Voltage epilogue (Convolution::Engine::perform output)
struct VoltView
{
  float2* out;
  uint64_t span;
};

// Overlap-save plan of one FFT shape
struct ConvShape
{
  unsigned nchan, npol;
  unsigned nfft, n1, n2;     // nfft = n1 * n2; n1 == 1 -> single-kernel path
  unsigned nfilt_pos, nfilt_neg;
  uint64_t nkeep;            // nfft - nfilt_pos - nfilt_neg
};

struct ConvTables
{
  const float2* tw2 = nullptr;   // n2-point table exp(-2 pi i m / n2)
  const float2* tw4 = nullptr;   // [n1][n2] exp(-2 pi i k1 n2 / nfft), null when n1 == 1
  const float2* H = nullptr;     // [nchan][n1][n2] response in four-step order
  const float* lut = nullptr;    // 8-bit lookup table (device), 256 floats
  int* err = nullptr;            // device flag: set when a bounded wait (tensor-core rows) gave up
  int nsm = 0;                   // multiprocessors of the device
  const float* apod = nullptr;   // temporal window [nfft] applied to each part, or null
  // tensor-core row FFT: the DFT16/DFT32 operand image (make_tc_dft_image)
  // and its number of BF16 terms (2 or 3); 0 = the FP32 row kernel
  const void* tc_dft = nullptr;
  int tc_splits = 0;
};

// The DFT16 and DFT32 blocks of the tensor-core row kernel in its shared
// memory operand layout, split into ns BF16 terms (bytes for a device copy).
void make_tc_dft_image (unsigned ns, std::vector<uint8_t>& img);

// The convolution rows (n2 = 8192) on the tensor cores: k_rows_mma.
cudaError_t launch_rows_mma (unsigned nrows, float2* scratch, const ConvTables& tables,
                             unsigned n1, const ConvShape& shape, cudaStream_t stream);

// Per-pass Stockham twiddle tables of an n-point transform, as the row
// kernel reads them (fft_core.cuh pass_table_offset layout).
void make_pass_tables (unsigned n, float2* out, unsigned capacity);
unsigned pass_tables_count (unsigned n);

// Kernels of the convolution path, for per-kernel timing.
enum KernelKind
{
  KK_FWD_COLS = 0, KK_ROWS = 1, KK_INV_COLS = 2, KK_FUSED = 3, KK_FILTERBANK = 4, KK_COUNT = 5
};

// Optional per-kernel clock: mark(self, kind, 0|1, stream) is called right
// before (0) and after (1) each kernel launch of the convolution path.
struct KernelClock
{
  void (*mark) (void* self, int kind, int phase, cudaStream_t stream);
  void* self;
};

// Number of kernels this library has launched since it was loaded.
uint64_t kernel_launches ();

// CTAs of the FP32 convolution row kernel resident per SM for n2-point rows
// (the persistent grid is this times the SM count)
unsigned rows_ctas_per_sm (unsigned n2);

// SpectralKurtosis engine steps on their own: the test of sums already formed
// (detect_skfb) and the mask applied to voltages (out == in: in place).
cudaError_t launch_sk_detect (const float* sums, const unsigned* counts, uint64_t npart,
                              unsigned nchan, unsigned npol, unsigned M, unsigned Nd, float lower,
                              float upper, uint8_t* mask, unsigned long long* nzap,
                              cudaStream_t stream);
cudaError_t launch_sk_mask (const uint8_t* mask, const float2* in, uint64_t in_span, float2* out,
                            uint64_t out_span, uint64_t ndat, unsigned nchan, unsigned npol,
                            unsigned M, cudaStream_t stream);

// SpectralKurtosis with overlapping blocks and several resolutions (engine
// steps): sums of blocks of M every `stride` samples, the reference's
// tscrunch of sums, detect_skfb with per-count limits flagging fine cells,
// and the mask of overlapping blocks.
cudaError_t launch_sk_sums_strided (const float2* in, uint64_t span, uint64_t nblk,
                                   uint64_t stride, unsigned nchan, unsigned npol, unsigned M,
                                   int zero_is_valid, float* sums, unsigned* counts,
                                   cudaStream_t stream);
cudaError_t launch_sk_tscrunch (const float* sums, const unsigned* counts, uint64_t npart,
                                unsigned nchan, unsigned npol, unsigned nsum, unsigned offset,
                                float* osums, unsigned* ocounts, cudaStream_t stream);
cudaError_t launch_sk_detect_skfb (const float* sums, const unsigned* counts, uint64_t npart,
                                   unsigned nchan, unsigned npol, unsigned Nd,
                                   const unsigned* lim_count, const float2* lim, unsigned nlim,
                                   unsigned nflag, unsigned flag_step, unsigned flag_offset,
                                   uint8_t* mask, unsigned long long* nzap, cudaStream_t stream);
cudaError_t launch_sk_mask_overlap (const uint8_t* mask, const float2* in, uint64_t in_span,
                                    float2* out, uint64_t out_span, uint64_t ndat_out,
                                    unsigned nchan, unsigned npol, unsigned offset,
                                    uint64_t npart, uint64_t nskip, uint64_t idat_start,
                                    cudaStream_t stream);

// SpectralKurtosis as a stage of the pipeline: the zero-DM input of n
// output samples starting at input sample `first` (unpacked, FPT rows of
// span), the mask of its blocks applied to other voltages, and detection +
// fold of zeroed data (hits counted per non-zeroed channel sample).
cudaError_t launch_zero_dm (const InputView& in, const float* lut, uint64_t first, uint64_t n,
                            float2* out, uint64_t span, cudaStream_t stream);
cudaError_t launch_sk_apply (const uint8_t* mask, float2* v, uint64_t span, uint64_t ndat,
                             unsigned nchan, unsigned npol, unsigned M, cudaStream_t stream);
cudaError_t launch_zeroed_fold (const float2* v, uint64_t span, uint64_t ndat, unsigned nchan,
                                unsigned npol, const FoldView& fold, cudaStream_t stream,
                                const KernelClock* clock = nullptr);

// Per-device set-up of the four-step convolution kernels (their shared-memory
// opt-in) on the current device; launch_convolution calls it itself.
cudaError_t convolution_kernel_setup ();

// Runs parts [part0, part0 + nbatch) of one block.  scratch holds
// nbatch*nchan*npol*nfft complex values (unused when n1 == 1).
cudaError_t launch_convolution (const ConvShape& shape, const ConvTables& tables,
                                const InputView& in, uint64_t part0, unsigned nbatch,
                                float2* scratch, int mode, const FoldView& fold,
                                const VoltView& volt, cudaStream_t stream,
                                const KernelClock* clock = nullptr);

// Builds the dispersion response directly in four-step order on the device.
// chan_freq/coeff per response channel computed on the host in double.
cudaError_t launch_build_chirp (float2* H, const double* d_chan_freq, const double* d_coeff,
                                const double* d_frac_us, unsigned nchan, unsigned nfft,
                                unsigned n1, unsigned n2, double binwidth, double half_chanwidth,
                                int swap_halves, int chirp_mode, float scale, cudaStream_t st);
// Reorders an FFT-order response [nchan][nfft] into four-step order.
cudaError_t launch_permute_response (float2* H, const float2* src, unsigned nchan,
                                     unsigned n1, unsigned n2, cudaStream_t stream);
// Inverse of launch_permute_response.
cudaError_t launch_unpermute_response (float2* dst, const float2* H, unsigned nchan,
                                       unsigned n1, unsigned n2, cudaStream_t stream);

// FFT filterbank, freq_res = 1: nsub a power of two in [4, 4096]; nblk blocks
// of nsub input samples per (input channel, pol); output FPT with channel
// cin*nsub + k, span out_span.  nsub >= 128 runs the transforms in shared
// memory and needs the per-pass tables of the nsub-point FFT (ptab).
cudaError_t launch_filterbank (const InputView& in, const float* d_lut, unsigned nsub,
                               uint64_t nblk, float scale, float2* out, uint64_t out_span,
                               cudaStream_t stream, const KernelClock* clock = nullptr,
                               const float2* ptab = nullptr);

// InverseFilterbank: per part, forward FFT of lin samples of every fine
// channel, the kept bins stitched into the spectra of the output channels
// (lout = n1 * n2 bins each, n2 in {4096, 8192}), times the response and the
// spectral window, then the inverse lout-point FFT with the output discard.
struct IfbShape
{
  unsigned nin, nout, npol;
  unsigned lin, keep, lout, n1, n2;
  uint64_t in_step, out_step;
  unsigned out_discard_pos;
  int dual_sideband;
};

struct IfbTables
{
  // per input channel: (output channel of the negative half, its first bin,
  // output channel of the positive half, its first bin); bit 30 of a first
  // bin marks a half that is zeroed instead
  const int4* map;
  const float2* ptab_lin;    // per-pass Stockham tables of the lin-point transform
  const float2* tw4;         // [n1][n2] four-step table of the lout-point transform
  const float2* response;    // [nout][lout] or null
  const float* temporal;     // [lin] or null
  const float* spectral;     // [lout] or null
  const float* lut;          // 8-bit table for int8 input
  int* err;
  int nsm;
};

constexpr int IFB_ZERO = 1 << 30;

// Parts [part0, part0 + nbatch); scratch holds nbatch*nout*npol*lout values.
cudaError_t launch_inverse_filterbank (const IfbShape& shape, const IfbTables& tables,
                                       const InputView& in, uint64_t part0, unsigned nbatch,
                                       float2* scratch, const VoltView& out, cudaStream_t stream,
                                       const KernelClock* clock = nullptr);
bool ifb_supported_lin (unsigned lin);

// Filterbank with a response (the "During" form, -F nchan:D:
// FilterbankEngineCPU.C:379-535 with Response::operate over the channels of
// the big spectrum): per part one nsub*freq_res-point forward FFT of every
// input channel, split as n1 x n2 (n2 = 8192); the response; then one inverse
// FFT of freq_res = n1*seg points per output channel, seg = n2/nsub.  In the
// four-step order of the big spectrum output channel cs of an input channel is
// the contiguous range [cs*seg, (cs+1)*seg) of every row, so its inverse
// transform is itself a four-step transform: seg-point inverse FFTs inside the
// row kernel, then n1-point inverse DFTs across the rows.
struct DuringShape
{
  unsigned nchan_in, npol, nsub;
  unsigned n1, n2, seg;          // nsub * freq_res = n1 * n2 (n1 <= 512), seg = n2 / nsub
  unsigned freq_res, nfilt_pos, nfilt_neg;
  uint64_t nkeep;                // freq_res - nfilt_pos - nfilt_neg
  uint64_t in_step;              // nsub * nkeep input samples between parts
};

struct DuringTables
{
  const float2* tw4;       // [n1][n2] exp(-2 pi i k1 m / (n1 n2))
  const float2* ptab_seg;  // per-pass tables of the seg-point FFT
  const float2* twd;       // [n1][seg] exp(-2 pi i k1 t2 / freq_res)
  const float2* ptab_col;  // per-pass tables of the n1-point FFT (n1 >= 64)
  const float2* H;         // [nchan_in*nsub][n1][seg]: bin k1 + n1*f2 of each channel
  const float* lut;        // 8-bit table for int8 input
  int nsm;
  const float* apod;       // temporal window of n1*n2 points, or null
};

bool during_supported (unsigned nsub, unsigned freq_res);
// out = in x window[f] for every bin f = k1 + n1*f2 of the [nchan][n1][seg]
// response layout (Apodization::operate on each channel's spectrum,
// FilterbankEngineCPU.C:507-509, folded into the response)
cudaError_t launch_window_response (float2* out, const float2* in, const float* window,
                                    unsigned nchan, unsigned n1, unsigned seg,
                                    cudaStream_t stream);
// Parts [part0, part0 + nbatch); scratch holds nbatch*nchan_in*npol*n1*n2
// values.  mode OUT_VOLTAGE writes the output channels (chan*npol + pol)*span;
// OUT_FOLD detects and folds them (fold.nout products).
cudaError_t launch_filterbank_during (const DuringShape& shape, const DuringTables& tables,
                                      const InputView& in, uint64_t part0, unsigned nbatch,
                                      float2* scratch, int mode, const FoldView& fold,
                                      const VoltView& out, cudaStream_t stream,
                                      const KernelClock* clock = nullptr);

// SpectralKurtosis (one resolution, noverlap 1): statistics, test and masked
// copy (out may equal in: then only zapped blocks are written; out null:
// statistics, counts and mask only, nothing written back).  sums
// [npart][nchan][npol][2], counts and mask [npart][nchan] are optional.
// in/out spans are complex samples; M and the spans must be even, npol 1 or 2,
// and sk_smem_bytes(npol, M, 1) at most SK_SMEM_MAX.
constexpr size_t SK_SMEM_MAX = 224u << 10;
size_t sk_smem_bytes (unsigned npol, unsigned M, unsigned units);
cudaError_t launch_sk (const float2* in, uint64_t in_span, float2* out, uint64_t out_span,
                       uint64_t npart, unsigned nchan, unsigned npol, unsigned M,
                       int zero_is_valid, unsigned Nd, float lower, float upper, float* sums,
                       unsigned* counts, uint8_t* mask, unsigned long long* nzap,
                       cudaStream_t stream);

cudaError_t launch_unpack8 (const uint8_t* in, uint64_t ndat, unsigned nchan, unsigned npol,
                            unsigned ndim, const float* d_lut, float* out, uint64_t span,
                            cudaStream_t stream);
cudaError_t launch_unpack16 (const int16_t* in, uint64_t ndat, unsigned nchan, unsigned npol,
                             unsigned ndim, int offset_binary, float* out, uint64_t span,
                             cudaStream_t stream);
cudaError_t launch_detect (const float2* in, uint64_t in_span, uint64_t ndat, unsigned nchan,
                           int state, float* out, uint64_t out_span, cudaStream_t stream);
cudaError_t launch_fold (const float* in, uint64_t in_span, uint64_t ndat, unsigned nchan,
                         unsigned npol, const FoldView& fold, cudaStream_t stream);
cudaError_t launch_binplan (const FoldSegment* segs, int nseg, uint64_t ndat, unsigned nbin,
                            uint32_t* out, cudaStream_t stream);
// the profile column (segment base + bin, or 0xffffffff) of samples 0..ndat-1
cudaError_t launch_colplan (const FoldSegment* segs, int nseg, uint64_t ndat, unsigned nbin,
                            unsigned* cols, cudaStream_t st);
// SampleDelay + detection + fold over voltages [chan][pol] (span values a row)
cudaError_t launch_delay_fold (const float2* v, uint64_t span, const int* applied, uint64_t ndat,
                               unsigned nchan, unsigned npol, const FoldView& fv, cudaStream_t st,
                               const KernelClock* clk);

// number of detected output polarisations for a detection state
__host__ __device__ inline int detect_nout (int state) { return state == 0 ? 1 : state == 1 ? 2 : 4; }

} // namespace b200
