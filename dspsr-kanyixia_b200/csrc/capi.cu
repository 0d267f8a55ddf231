// capi.cu -- the C ABI of libdspsr_b200.so (declared in include/dspsr_b200.h):
// contexts, the engine objects that stand in for DSPSR's CUDA engines, and
// the fused unpack -> convolve -> detect -> fold pipeline.

#include "dspsr_b200.h"
#include "kernels.cuh"
#include "host_rules.h"
#include "dada.h"
#include "subint.h"

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <cstdint>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <new>
#include <string>
#include <vector>

using namespace b200;

#include "context.h"

namespace {

int fail (dspsr_b200_context* ctx, int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start (ap, fmt);
  vsnprintf (buf, sizeof (buf), fmt, ap);
  va_end (ap);
  if (ctx) ctx->error = buf;
  return code;
}

int cuda_fail (dspsr_b200_context* ctx, cudaError_t err, const char* where)
{
  return fail (ctx, DSPSR_B200_ECUDA, "%s: %s", where, cudaGetErrorString (err));
}

#define B200_CHECK(ctx, call, where)                                  \
  do {                                                                \
    cudaError_t _e = (call);                                          \
    if (_e != cudaSuccess) return cuda_fail ((ctx), _e, (where));     \
  } while (0)

bool is_pow2 (uint64_t x) { return x && !(x & (x - 1)); }

// Per-pass Stockham tables of an n-point transform uploaded into a device
// buffer (the shared-memory filterbank's twiddles).
cudaError_t upload_pass_tables (unsigned n, float2** dst, size_t* cap)
{
  const unsigned cnt = pass_tables_count (n);
  std::vector<float2> t (std::max (cnt, 1u), make_float2 (0.f, 0.f));
  make_pass_tables (n, t.data (), cnt);
  if (*cap < t.size ())
  {
    if (*dst) cudaFree (*dst);
    *dst = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc (dst, t.size () * sizeof (float2));
    if (e != cudaSuccess) return e;
    *cap = t.size ();
  }
  return cudaMemcpy (*dst, t.data (), t.size () * sizeof (float2), cudaMemcpyHostToDevice);
}


// Device buffer owned by an engine object.
template <typename T>
struct DevBuf
{
  T* ptr = nullptr;
  size_t n = 0;
  cudaError_t reserve (size_t count)
  {
    if (count <= n) return cudaSuccess;
    release ();
    cudaError_t e = cudaMalloc (&ptr, count * sizeof (T));
    if (e == cudaSuccess) n = count; else ptr = nullptr;
    return e;
  }
  void release ()
  {
    if (ptr) cudaFree (ptr);
    ptr = nullptr;
    n = 0;
  }
};

// Twiddle tables rounded once from double precision.
std::vector<float2> make_tw2 (unsigned n)
{
  std::vector<float2> t (n);
  for (unsigned m = 0; m < n; m++)
  {
    const double a = -2.0 * M_PI * double (m) / double (n);
    t[m] = make_float2 (float (std::cos (a)), float (std::sin (a)));
  }
  return t;
}

std::vector<float2> make_tw4 (unsigned n1, unsigned n2)
{
  const uint64_t N = uint64_t (n1) * n2;
  std::vector<float2> t (N);
  for (unsigned k1 = 0; k1 < n1; k1++)
    for (unsigned i = 0; i < n2; i++)
    {
      const uint64_t m = (uint64_t (k1) * i) % N;
      const double a = -2.0 * M_PI * double (m) / double (N);
      t[uint64_t (k1) * n2 + i] = make_float2 (float (std::cos (a)), float (std::sin (a)));
    }
  return t;
}

} // namespace

// ---------------------------------------------------------------------------
// convolution engine
// ---------------------------------------------------------------------------

struct dspsr_b200_convolution
{
  dspsr_b200_context* ctx = nullptr;
  ConvShape shape {};
  DevBuf<float2> tw2, tw4, H, tmp, scratch;
  DevBuf<double> chan_par;
  DevBuf<float> lut, apod;
  DevBuf<int> err;
  DevBuf<uint8_t> tc_dft;
  int tc_splits = 0;
  int nsm = 148;
  bool have_response = false, have_apod = false;
  unsigned max_batch = 1;

  int set_fft_precision (int mode);

  // row_len: the four-step row length, 8192 (0 = default) or 4096 (nfft
  // from 8192 to 131072: then n1 = nfft / 4096 columns)
  int init (dspsr_b200_context* c, unsigned nchan, unsigned npol, unsigned nfft,
            unsigned pos, unsigned neg, uint64_t scratch_bytes, unsigned row_len = 0);
  ConvTables tables () const
  {
    ConvTables t;
    t.tw2 = tw2.ptr;
    t.tw4 = tw4.ptr;
    t.H = H.ptr;
    t.lut = lut.ptr;
    t.err = err.ptr;
    t.nsm = nsm;
    t.apod = have_apod ? apod.ptr : nullptr;
    t.tc_dft = tc_dft.ptr;
    t.tc_splits = tc_splits;
    return t;
  }
  void release ()
  {
    tc_dft.release ();
    apod.release ();
    tw2.release ();
    tw4.release ();
    H.release ();
    tmp.release ();
    scratch.release ();
    chan_par.release ();
    lut.release ();
    err.release ();
  }
  // ESTATE when a bounded device wait of the row kernel gave up
  int status ()
  {
    if (!err.ptr) return DSPSR_B200_OK;
    int h = 0;
    B200_CHECK (ctx, cudaMemcpyAsync (&h, err.ptr, sizeof (int), cudaMemcpyDeviceToHost,
                                      ctx->stream), "read device status");
    B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "device status sync");
    if (h) return fail (ctx, DSPSR_B200_ESTATE, "a device-side wait timed out");
    return DSPSR_B200_OK;
  }
};

int dspsr_b200_convolution::init (dspsr_b200_context* c, unsigned nchan, unsigned npol,
                                  unsigned nfft, unsigned pos, unsigned neg,
                                  uint64_t scratch_bytes, unsigned row_len)
{
  ctx = c;
  if (nchan == 0 || npol == 0 || npol > 2)
    return fail (ctx, DSPSR_B200_EINVAL, "convolution: invalid nchan=%u npol=%u", nchan, npol);
  if (!is_pow2 (nfft) || nfft < 4096 || nfft > 262144)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "convolution: nfft=%u must be a power of two in [4096, 262144]", nfft);
  // Convolution::prepare (Convolution.C:456-459): the FFT must exceed the overlap
  if (uint64_t (pos) + neg >= nfft)
    return fail (ctx, DSPSR_B200_EINVAL, "convolution: nfft=%u <= nfilt=%u", nfft, pos + neg);
  shape.nchan = nchan;
  shape.npol = npol;
  shape.nfft = nfft;
  shape.nfilt_pos = pos;
  shape.nfilt_neg = neg;
  shape.nkeep = nfft - pos - neg;
  if (row_len != 0 && row_len != 4096 && row_len != 8192)
    return fail (ctx, DSPSR_B200_EINVAL, "convolution: row length %u is not 4096 or 8192",
                 row_len);
  if (row_len == 4096 && nfft >= 8192)
  {
    if (nfft > 131072)
      return fail (ctx, DSPSR_B200_EINVAL,
                   "convolution: 4096-point rows need nfft <= 131072 (nfft=%u)", nfft);
    shape.n2 = 4096;
    shape.n1 = nfft / 4096;
  }
  else if (nfft <= 8192)
  {
    shape.n1 = 1;
    shape.n2 = nfft;
  }
  else
  {
    shape.n2 = 8192;
    shape.n1 = nfft / 8192;
  }
  B200_CHECK (ctx, tw2.reserve (shape.n2), "cudaMalloc tw2");
  std::vector<float2> t2 = make_tw2 (shape.n2);
  B200_CHECK (ctx, cudaMemcpy (tw2.ptr, t2.data (), t2.size () * sizeof (float2),
                               cudaMemcpyHostToDevice), "copy tw2");
  if (shape.n1 > 1)
  {
    B200_CHECK (ctx, tw4.reserve (nfft), "cudaMalloc tw4");
    std::vector<float2> t4 = make_tw4 (shape.n1, shape.n2);
    B200_CHECK (ctx, cudaMemcpy (tw4.ptr, t4.data (), t4.size () * sizeof (float2),
                                 cudaMemcpyHostToDevice), "copy tw4");
    B200_CHECK (ctx, err.reserve (1), "cudaMalloc status flag");
    B200_CHECK (ctx, cudaMemset (err.ptr, 0, sizeof (int)), "clear status flag");
    int dev = 0;
    B200_CHECK (ctx, cudaGetDevice (&dev), "cudaGetDevice");
    B200_CHECK (ctx, cudaDeviceGetAttribute (&nsm, cudaDevAttrMultiProcessorCount, dev),
                "multiprocessor count");
    // Parts in flight: the scratch stays near the L2 size unless told
    // otherwise, and the batch is chosen so that its rows spread evenly over
    // the persistent row kernel's CTAs.
    const uint64_t per_part = uint64_t (nchan) * npol * nfft * sizeof (float2);
    const uint64_t budget = scratch_bytes ? scratch_bytes : (uint64_t (512) << 20);
    const uint64_t bmax = std::max<uint64_t> (1, std::min<uint64_t> (65535, budget / per_part));
    const uint64_t rows_per_part = uint64_t (shape.n1) * nchan * npol;
    // (a multiple of the SM count, so also even for the tensor-core rows'
    // one CTA per SM)
    const uint64_t ctas = uint64_t (nsm) * b200::rows_ctas_per_sm (shape.n2);
    max_batch = unsigned (bmax);
    for (uint64_t b = bmax; b >= std::max<uint64_t> (1, bmax / 2); b--)
      if ((b * rows_per_part) % ctas == 0)
      {
        max_batch = unsigned (b);
        break;
      }
    B200_CHECK (ctx, scratch.reserve (uint64_t (max_batch) * nchan * npol * nfft),
                "cudaMalloc scratch");
  }
  else
    max_batch = 65535;
  B200_CHECK (ctx, H.reserve (uint64_t (nchan) * nfft), "cudaMalloc response");
  B200_CHECK (ctx, lut.reserve (256), "cudaMalloc lut");
  return DSPSR_B200_OK;
}

namespace {

// Dedispersion response for channels centred at freq[c] (MHz), channel width
// bw/nchan, each channel complex-sampled with DC at FFT bin 0 when swap_halves
// (Response::doswap per channel).  Per channel the coefficient of
// Dedispersion::build_compute (Dedispersion.C:168-173) is formed on the host
// in double; the GPU evaluates the phase of every bin in FP64.
int build_response (dspsr_b200_convolution* c, const double* freq, double bw, double dm,
                    int swap_halves, int chirp_mode, unsigned norm_nfft,
                    const double* frac_us = nullptr)
{
  dspsr_b200_context* ctx = c->ctx;
  const ConvShape& sh = c->shape;
  const unsigned nchan = sh.nchan;
  std::vector<double> par (3 * nchan, 0.0);
  const double sign = bw / std::fabs (bw);
  const double dispersion_per_MHz = 1e6 * dm / 2.41e-4;
  for (unsigned ic = 0; ic < nchan; ic++)
  {
    par[ic] = freq[ic];
    par[nchan + ic] = -sign * 2 * M_PI * dispersion_per_MHz / (freq[ic] * freq[ic]);
    if (frac_us) par[2 * nchan + ic] = frac_us[ic];
  }
  const double chanwidth = bw / double (nchan);
  const double binwidth = chanwidth / double (sh.nfft);
  const float scale = float (1.0 / std::sqrt (double (norm_nfft ? norm_nfft : sh.nfft)));
  B200_CHECK (ctx, c->chan_par.reserve (3 * nchan), "cudaMalloc channel table");
  B200_CHECK (ctx, cudaMemcpyAsync (c->chan_par.ptr, par.data (), par.size () * sizeof (double),
                                    cudaMemcpyHostToDevice, ctx->stream), "upload channels");
  B200_CHECK (ctx, launch_build_chirp (c->H.ptr, c->chan_par.ptr, c->chan_par.ptr + nchan,
                                       frac_us ? c->chan_par.ptr + 2 * nchan : nullptr, nchan,
                                       sh.nfft, sh.n1, sh.n2, binwidth, 0.5 * chanwidth,
                                       swap_halves, chirp_mode, scale, ctx->stream),
              "build chirp");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "set_dedispersion sync");
  c->have_response = true;
  return DSPSR_B200_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// fold engine
// ---------------------------------------------------------------------------

struct dspsr_b200_fold
{
  dspsr_b200_context* ctx = nullptr;
  unsigned nbin = 0, nchan = 0, npol = 0;
  DevBuf<float> profiles;
  DevBuf<unsigned> hits;
  // Ring of plan buffers: the host builds block b+1's plan while the GPU still
  // folds earlier blocks; it waits only when all NRING slots are in flight.
  static constexpr int NRING = 8;
  static constexpr size_t INITIAL_SEGMENTS = 16384;
  DevBuf<FoldSegment> d_segs[NRING];
  // the column of each sample is computed once per block (k_colplan: one
  // segment search per 1024 samples) instead of by a search per warp in every
  // channel's epilogue; with one channel it still pays (C1: 0.867 -> 0.827 ms
  // per block)
  bool use_cols = false;
  DevBuf<unsigned> d_cols[NRING];
  uint64_t cols_cap = 0;
  FoldSegment* h_segs[NRING] = {};
  size_t h_cap[NRING] = {};
  cudaEvent_t done[NRING] = {};
  int cur = 0;
  int nseg = 0;
  uint64_t ndat = 0;
  std::vector<FoldSegment> plan;

  unsigned slots = 1;                 // sub-integrations held side by side
  int init (dspsr_b200_context* c, unsigned nb, unsigned nc, unsigned np, unsigned ns = 1)
  {
    ctx = c;
    nbin = nb;
    nchan = nc;
    npol = np;
    slots = ns;
    if (nbin == 0 || nchan == 0 || npol == 0 || slots == 0
        || uint64_t (nbin) * slots >= FOLD_SKIP)
      return fail (ctx, DSPSR_B200_EINVAL, "fold: invalid nbin=%u nchan=%u npol=%u slots=%u",
                   nbin, nchan, npol, slots);
    B200_CHECK (ctx, profiles.reserve (uint64_t (nchan) * npol * nbin * slots),
                "cudaMalloc profiles");
    B200_CHECK (ctx, hits.reserve (uint64_t (nbin) * slots), "cudaMalloc hits");
    for (int i = 0; i < NRING; i++)
    {
      B200_CHECK (ctx, cudaEventCreateWithFlags (&done[i], cudaEventDisableTiming),
                  "cudaEventCreate");
      B200_CHECK (ctx, cudaMallocHost (&h_segs[i], INITIAL_SEGMENTS * sizeof (FoldSegment)),
                  "cudaMallocHost plan");
      h_cap[i] = INITIAL_SEGMENTS;
      B200_CHECK (ctx, d_segs[i].reserve (INITIAL_SEGMENTS), "cudaMalloc plan");
    }
    plan.reserve (INITIAL_SEGMENTS);
    return reset ();
  }
  int reset ()
  {
    B200_CHECK (ctx, cudaMemsetAsync (profiles.ptr, 0,
                                      uint64_t (nchan) * npol * nbin * slots * sizeof (float),
                                      ctx->stream), "memset profiles");
    B200_CHECK (ctx, cudaMemsetAsync (hits.ptr, 0, uint64_t (nbin) * slots * sizeof (unsigned),
                                      ctx->stream), "memset hits");
    return DSPSR_B200_OK;
  }
  // zeroes one sub-integration slot
  int reset_slot (unsigned k)
  {
    const size_t pitch = size_t (nbin) * slots * sizeof (float);
    B200_CHECK (ctx, cudaMemset2DAsync (profiles.ptr + size_t (k) * nbin, pitch, 0,
                                        nbin * sizeof (float), size_t (nchan) * npol, ctx->stream),
                "memset slot");
    B200_CHECK (ctx, cudaMemsetAsync (hits.ptr + size_t (k) * nbin, 0, nbin * sizeof (unsigned),
                                      ctx->stream), "memset slot hits");
    return DSPSR_B200_OK;
  }
  // copies one slot to host memory ([chan*npol][nbin] and [nbin]) on the stream
  int download_slot (unsigned k, float* h_prof, uint32_t* h_hits)
  {
    const size_t pitch = size_t (nbin) * slots * sizeof (float);
    if (h_prof)
      B200_CHECK (ctx, cudaMemcpy2DAsync (h_prof, nbin * sizeof (float),
                                          profiles.ptr + size_t (k) * nbin, pitch,
                                          nbin * sizeof (float), size_t (nchan) * npol,
                                          cudaMemcpyDeviceToHost, ctx->stream), "download slot");
    if (h_hits)
      B200_CHECK (ctx, cudaMemcpyAsync (h_hits, hits.ptr + size_t (k) * nbin,
                                        nbin * sizeof (unsigned), cudaMemcpyDeviceToHost,
                                        ctx->stream), "download slot hits");
    return DSPSR_B200_OK;
  }
  // installs a plan built by the caller (segments over ndat samples)
  // Plans go to the device on `up` when set (the stream that carries the
  // block's own upload), else on the context's stream: an upload from host
  // memory queued on the compute stream waits behind whatever host copies
  // another stream has already given the copy engine.
  cudaStream_t up = nullptr;
  cudaEvent_t plan_ev = nullptr;
  int set_plan (std::vector<FoldSegment>& segs, uint64_t n)
  {
    plan.swap (segs);
    return upload_plan (n);
  }
  // builds the exact plan on the host and uploads it on the context's stream
  int set_bins (double phi, double pps, uint64_t n, double* x_end = nullptr)
  {
    build_fold_plan (phi, pps, n, &plan, x_end);
    return upload_plan (n);
  }
  int upload_plan (uint64_t n)
  {
    ndat = n;
    nseg = int (plan.size ());
    cur = (cur + 1) % NRING;
    // the slot about to be overwritten was last read by work queued before `done[cur]`
    B200_CHECK (ctx, cudaEventSynchronize (done[cur]), "cudaEventSynchronize");
    if (h_cap[cur] < plan.size ())
    {
      if (h_segs[cur]) cudaFreeHost (h_segs[cur]);
      h_segs[cur] = nullptr;
      h_cap[cur] = 0;
      const size_t cap = plan.size () * 2 + 64;
      B200_CHECK (ctx, cudaMallocHost (&h_segs[cur], cap * sizeof (FoldSegment)),
                  "cudaMallocHost plan");
      h_cap[cur] = cap;
    }
    B200_CHECK (ctx, d_segs[cur].reserve (std::max<size_t> (plan.size (), 1)),
                "cudaMalloc plan");
    std::memcpy (h_segs[cur], plan.data (), plan.size () * sizeof (FoldSegment));
    if (!plan.empty ())
    {
      B200_CHECK (ctx, cudaMemcpyAsync (d_segs[cur].ptr, h_segs[cur],
                                        plan.size () * sizeof (FoldSegment),
                                        cudaMemcpyHostToDevice, up ? up : ctx->stream),
                  "upload plan");
      if (up)
      {
        if (!plan_ev)
          B200_CHECK (ctx, cudaEventCreateWithFlags (&plan_ev, cudaEventDisableTiming),
                      "cudaEventCreate");
        B200_CHECK (ctx, cudaEventRecord (plan_ev, up), "record plan upload");
        B200_CHECK (ctx, cudaStreamWaitEvent (ctx->stream, plan_ev, 0), "wait plan upload");
      }
    }
    if (use_cols && n && !plan.empty ())
    {
      // every ring slot grows at once, with headroom, so that steady blocks
      // allocate nothing (an allocation would wait for the device)
      if (n > cols_cap)
      {
        cols_cap = n + n / 4;
        for (int i = 0; i < NRING; i++)
        {
          d_cols[i].release ();
          B200_CHECK (ctx, d_cols[i].reserve (cols_cap), "cudaMalloc fold columns");
        }
      }
      B200_CHECK (ctx, launch_colplan (d_segs[cur].ptr, nseg, n, nbin, d_cols[cur].ptr,
                                       ctx->stream), "fold columns");
    }
    return DSPSR_B200_OK;
  }
  // marks the end of the work that reads the current plan buffer
  int release_plan ()
  {
    B200_CHECK (ctx, cudaEventRecord (done[cur], ctx->stream), "cudaEventRecord");
    return DSPSR_B200_OK;
  }
  FoldView view (int state, int nout, unsigned nchan_prof)
  {
    (void) nchan_prof;
    FoldView v;
    v.segs = d_segs[cur].ptr;
    v.nseg = nseg;
    v.profiles = profiles.ptr;
    v.hits = hits.ptr;
    v.nbin = nbin;
    v.stride = nbin * slots;
    v.cols = use_cols && ndat && nseg ? d_cols[cur].ptr : nullptr;
    v.state = state;
    v.nout = nout;
    return v;
  }
  void release ()
  {
    profiles.release ();
    hits.release ();
    if (plan_ev) cudaEventDestroy (plan_ev);
    plan_ev = nullptr;
    for (int i = 0; i < NRING; i++)
    {
      d_segs[i].release ();
      d_cols[i].release ();
      cols_cap = 0;
      if (h_segs[i]) cudaFreeHost (h_segs[i]);
      h_segs[i] = nullptr;
      if (done[i]) cudaEventDestroy (done[i]);
      done[i] = nullptr;
    }
  }
};

// ---------------------------------------------------------------------------
// fused pipeline
// ---------------------------------------------------------------------------

// Per-kernel CUDA-event clock of the pipeline (KernelClock hook).
struct PipeClock
{
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<int> kind;              // kind of each (start, stop) pair
  cudaEvent_t take ()
  {
    if (used == pool.size ())
    {
      cudaEvent_t e = nullptr;
      cudaEventCreate (&e);
      pool.push_back (e);
    }
    return pool[used++];
  }
  static void mark (void* self, int k, int phase, cudaStream_t st)
  {
    PipeClock* c = static_cast<PipeClock*> (self);
    cudaEventRecord (c->take (), st);
    if (phase == 0) c->kind.push_back (k);
  }
  void clear ()
  {
    used = 0;
    kind.clear ();
  }
  ~PipeClock ()
  {
    for (cudaEvent_t e : pool) cudaEventDestroy (e);
  }
};

struct dspsr_b200_pipeline
{
  dspsr_b200_context* ctx = nullptr;
  PipeClock clock;
  dspsr_b200_pipeline_config cfg {};
  dspsr_b200_convolution conv;
  dspsr_b200_fold fold;
  int nout = 1;
  uint64_t bytes_per_sample = 0;   // TFPD bytes per time sample (all chans, pols)
  DevBuf<uint8_t> carry[2];         // carried input (TFPD bytes or FPT floats)
  uint64_t carry_span = 0;          // FPT: complex samples per (chan, pol) row
  uint64_t ncarry = 0;
  int cur_carry = 0;
  uint64_t in0 = 0;                 // global input index of the first sample of the block
  DevBuf<uint8_t> staging[2];       // host->device staging for run_host (double buffer)
  cudaStream_t copy_stream = nullptr;   // run_host uploads, overlapping the kernels
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  bool consumed_pending[2] = {false, false};
  double rate = 0;                  // complex sampling rate of the convolved channels
  unsigned fb_nsub = 0;             // filterbank channels per input channel (0: none)
  bool fb_fused = false;            // filterbank computed inside the column pass
  float lut_scale = 0.f;            // the 8-bit table as (x + 0.5) * scale, or 0
  // inter-channel dedispersion: SampleDelay between the convolution and the
  // fold, its voltages in sd_buf[sd_cur] (rows [chan][pol], sd_span values)
  bool sd_on = false;
  InterchannelDelays sd;
  DevBuf<int> sd_applied;
  DevBuf<float2> sd_buf[2];
  uint64_t sd_span = 0;
  int sd_cur = 0;
  uint64_t sd_ncarry = 0;           // voltages carried per row
  uint64_t sd_out0 = 0;             // SampleDelay output samples before this block
  // SpectralKurtosis between the convolution and detection (LoadToFold1.C:
  // 310-351 with the zero-DM input): dedispersed voltages in sk_v[sk_cur],
  // zero-DM voltages in sk_z[sk_cur] (rows [chan][pol], sk_span values), the
  // last len % M of them carried into the next block
  bool sk_on = false;
  unsigned sk_M = 0;
  float sk_lower = 0.f, sk_upper = 0.f;
  DevBuf<float2> sk_v[2], sk_z[2];
  DevBuf<uint8_t> sk_mask;
  DevBuf<unsigned long long> sk_zapped;
  uint64_t sk_span = 0;
  int sk_cur = 0;
  uint64_t sk_ncarry = 0;
  uint64_t sk_out0 = 0;             // SpectralKurtosis output samples before this block
  uint64_t sk_tested = 0;           // (block, channel) cells tested
  // an RFI-mask proposer in front of the SK stage: its mask replaces SK's
  // where it is confident, SK's own decision is the fallback
  dspsr_b200_rfi_proposer* sk_proposer = nullptr;
  float sk_confidence = 0.9f;
  DevBuf<float> sk_sums;
  DevBuf<uint32_t> sk_counts;
  DevBuf<uint8_t> sk_pmask;
  DevBuf<float2> fbbuf;             // filterbank output, FPT
  float2* fb_tab = nullptr;         // pass tables of the filterbank FFT (fb_nsub >= 128)
  size_t fb_tab_cap = 0;
  // run_host folds a block in pieces: the first piece that folds starts the
  // block's phase with Fold::get_phase, later pieces go on with the block's
  // own phase recurrence, exactly as one fold of the whole block would
  bool in_pieces = false, phase_continue = false;
  double phase_next = 0;
  // sub-integrations (Subint<Fold>): each division folds into its own slot of
  // the fold's profiles; closed slots wait in sub_ready for the unloader or
  // pop_subint, then are zeroed and reused
  bool sub_on = false;
  b200::SubintPlanner planner;
  b200::SubintPlanner planner_init;            // the configured, unstarted divider
  std::vector<b200::SubintAction> sub_actions;
  struct SubSlot
  {
    bool used = false;
    dspsr_b200_subint info {};
  };
  std::vector<SubSlot> sub_slots;
  int sub_cur = -1;
  std::deque<int> sub_ready;
  dspsr_b200_unload_fn unload_fn = nullptr;
  void* unload_user = nullptr;
  // unloads in flight: the slot's copy into page-locked memory was queued,
  // the callback runs once its event has completed
  struct PendingUnload
  {
    dspsr_b200_subint info;
    float* prof;
    uint32_t* hits;
    cudaEvent_t ev;
  };
  std::deque<PendingUnload> sub_pending;
  std::vector<PendingUnload> sub_spare;      // host buffers and events for reuse
  void* pinned[2] = {nullptr, nullptr};   // run_dada: file blocks in page-locked memory
  uint64_t pinned_bytes = 0;
  cudaEvent_t host_free[2] = {nullptr, nullptr};   // uploads of pinned[b] done
  cudaEvent_t snap_ev = nullptr;    // the last asynchronous profile snapshot landed
  int* snap_err = nullptr;          // pinned copy of the row kernel's wait flag at the snapshot
  bool host_free_pending[2] = {false, false};
};

namespace {

// Subint<Fold>::transformation over one block's nout output samples
// (Subint.h:258-332): the divider splits the block into ranges, each range
// folds with its own phase (Fold::fold at its idat_start, Fold.C:685-693)
// into the slot of its division, and a closed division joins sub_ready.
// Samples outside every range are not folded.
void subint_close (dspsr_b200_pipeline* pl)
{
  if (pl->sub_cur < 0) return;
  auto& slot = pl->sub_slots[pl->sub_cur];
  if (slot.info.ndat_folded > 0)
    pl->sub_ready.push_back (pl->sub_cur);
  else
    slot.used = false;                 // nothing folded: still zero
  pl->sub_cur = -1;
}

// out_base: global index of the fold input's first sample; time_base: the
// input sample whose time that is (the convolution shifts its output by
// nfilt_pos samples, Convolution.C:611, and SampleDelay by zero_delay more,
// SampleDelay.C:221)
int pipeline_subint_plan (dspsr_b200_pipeline* pl, uint64_t out_base, uint64_t time_base,
                          uint64_t nout, double pps)
{
  dspsr_b200_context* ctx = pl->ctx;
  const auto& cfg = pl->cfg;
  b200::Mjd start0;
  start0.day = cfg.start_day;
  start0.sec = cfg.start_sec;
  start0.frac = cfg.start_frac;
  const b200::Mjd start = b200::mjd_add (start0, double (time_base) / pl->rate);
  b200::SubintPlanner trial = pl->planner;
  const char* err = nullptr;
  if (!trial.block (start, nout, pl->rate, &pl->sub_actions, &err))
    return fail (ctx, DSPSR_B200_ESTATE, "pipeline sub-integrations: %s", err);
  // every division the block opens needs a free slot now
  unsigned need = 0, nfree = 0;
  bool open = pl->sub_cur >= 0;
  for (const auto& a : pl->sub_actions)
  {
    if (a.kind != b200::SubintAction::FOLD) { open = false; continue; }
    if (!open) { need++; open = true; }
  }
  for (const auto& sl : pl->sub_slots) nfree += sl.used ? 0 : 1;
  if (need > nfree)
    return fail (ctx, DSPSR_B200_ESTATE,
                 "pipeline: the block opens %u sub-integrations and %u of %zu slots are free "
                 "(pop closed sub-integrations, set an unloader, raise subint_slots or pass "
                 "shorter blocks)", need, nfree, pl->sub_slots.size ());
  pl->planner = trial;

  std::vector<FoldSegment> plan, part;
  uint64_t cursor = 0;
  auto skip = [&plan] (uint64_t at) {
    FoldSegment g;
    g.start = at;
    g.m0 = 0;
    g.dm = 0;
    g.g = 1.0;
    g.base = FOLD_SKIP;
    plan.push_back (g);
  };
  for (const auto& a : pl->sub_actions)
  {
    if (a.kind != b200::SubintAction::FOLD)
    {
      subint_close (pl);
      continue;
    }
    if (pl->sub_cur < 0)
    {
      int k = 0;
      while (pl->sub_slots[k].used) k++;
      auto& sl = pl->sub_slots[k];
      sl.used = true;
      sl.info = dspsr_b200_subint {};
      sl.info.division = a.division;
      sl.info.first_sample = out_base + a.idat_start;
      sl.info.lower_day = a.lower.day;
      sl.info.lower_sec = a.lower.sec;
      sl.info.lower_frac = a.lower.frac;
      sl.info.upper_day = a.upper.day;
      sl.info.upper_sec = a.upper.sec;
      sl.info.upper_frac = a.upper.frac;
      pl->sub_cur = k;
    }
    auto& sl = pl->sub_slots[pl->sub_cur];
    sl.info.ndat_folded += a.ndat;
    sl.info.integration_length = double (sl.info.ndat_folded) / pl->rate;
    sl.info.complete = a.end_reached ? 1 : 0;
    if (a.idat_start > cursor) skip (cursor);
    const double phi = fold_phi (cfg.start_day, cfg.start_sec, cfg.start_frac, cfg.epoch_day,
                                 cfg.epoch_sec, cfg.epoch_frac, time_base + a.idat_start,
                                 pl->rate, cfg.period_s, cfg.reference_phase);
    build_fold_plan (phi, pps, a.ndat, &part);
    const uint32_t base = uint32_t (pl->sub_cur) * pl->fold.nbin;
    for (FoldSegment g : part)
    {
      g.start += a.idat_start;
      g.base = base;
      plan.push_back (g);
    }
    cursor = a.idat_start + a.ndat;
  }
  if (cursor < nout || plan.empty ()) skip (cursor);
  return pl->fold.set_plan (plan, nout);
}

// hands closed sub-integration slot k to the caller's buffers (or to the
// pipeline's own, for the unloader), then zeroes and frees the slot
int subint_take (dspsr_b200_pipeline* pl, int k, dspsr_b200_subint* info, float* prof,
                 uint32_t* hits)
{
  dspsr_b200_context* ctx = pl->ctx;
  int rc = pl->fold.download_slot (unsigned (k), prof, hits);
  if (rc) return rc;
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "download sub-integration");
  if (info) *info = pl->sub_slots[k].info;
  rc = pl->fold.reset_slot (unsigned (k));
  if (rc) return rc;
  pl->sub_slots[k].used = false;
  return DSPSR_B200_OK;
}

// PhaseSeriesUnloader::unload for every closed sub-integration, in order.
// Each closed slot is copied to page-locked memory and zeroed on the stream
// (the slot is free again at once: later folds into it queue behind the
// copy); the callback runs when the copy has landed -- now if wait, else at
// the first call that finds it done.
int subint_drain (dspsr_b200_pipeline* pl, bool wait)
{
  if (!pl->unload_fn) return DSPSR_B200_OK;
  dspsr_b200_context* ctx = pl->ctx;
  const size_t nprof = size_t (pl->fold.nchan) * pl->fold.npol * pl->fold.nbin;
  while (!pl->sub_ready.empty ())
  {
    const int k = pl->sub_ready.front ();
    pl->sub_ready.pop_front ();
    dspsr_b200_pipeline::PendingUnload u {};
    if (!pl->sub_spare.empty ())
    {
      u = pl->sub_spare.back ();
      pl->sub_spare.pop_back ();
    }
    else
    {
      B200_CHECK (ctx, cudaMallocHost (&u.prof, nprof * sizeof (float)), "cudaMallocHost unload");
      B200_CHECK (ctx, cudaMallocHost (&u.hits, pl->fold.nbin * sizeof (uint32_t)),
                  "cudaMallocHost unload");
      B200_CHECK (ctx, cudaEventCreateWithFlags (&u.ev, cudaEventDisableTiming), "create event");
    }
    u.info = pl->sub_slots[k].info;
    int rc = pl->fold.download_slot (unsigned (k), u.prof, u.hits);
    if (!rc) rc = pl->fold.reset_slot (unsigned (k));
    if (rc)
    {
      pl->sub_spare.push_back (u);
      return rc;
    }
    B200_CHECK (ctx, cudaEventRecord (u.ev, ctx->stream), "record unload");
    pl->sub_slots[k].used = false;
    pl->sub_pending.push_back (u);
  }
  while (!pl->sub_pending.empty ())
  {
    auto& u = pl->sub_pending.front ();
    if (wait)
      B200_CHECK (ctx, cudaEventSynchronize (u.ev), "wait unload");
    else
    {
      const cudaError_t e = cudaEventQuery (u.ev);
      if (e == cudaErrorNotReady) break;
      B200_CHECK (ctx, e, "unload copy");
    }
    pl->unload_fn (pl->unload_user, &u.info, u.prof, u.hits);
    pl->sub_spare.push_back (u);
    pl->sub_pending.pop_front ();
  }
  return DSPSR_B200_OK;
}

// The fold plan of nout fold-input samples starting at global index out_base,
// whose first sample has the time of input sample time_base: one range with
// the block's phase (continued across the pieces of one host block), or the
// sub-integration ranges.
int pipeline_fold_plan (dspsr_b200_pipeline* pl, uint64_t out_base, uint64_t time_base,
                        uint64_t nout)
{
  const auto& cfg = pl->cfg;
  const double sampling_interval = 1.0 / pl->rate;
  const double pps = sampling_interval / cfg.period_s;   // Fold.C:754-756
  if (pl->sub_on) return pipeline_subint_plan (pl, out_base, time_base, nout, pps);
  const double phi = pl->phase_continue
                   ? pl->phase_next
                   : fold_phi (cfg.start_day, cfg.start_sec, cfg.start_frac, cfg.epoch_day,
                               cfg.epoch_sec, cfg.epoch_frac, time_base, pl->rate, cfg.period_s,
                               cfg.reference_phase);
  const int rc = pl->fold.set_bins (phi, pps, nout, &pl->phase_next);
  if (rc) return rc;
  pl->phase_continue = pl->in_pieces;
  return DSPSR_B200_OK;
}

// SampleDelay with its InputBuffering (SampleDelay.C:166-298) between the
// convolution and the fold: the block's voltages land after the carried ones,
// output sample t of channel c is voltage t + applied[c], and the last
// total_delay voltages of every (chan, pol) carry over.  *folded = outputs.
int pipeline_sd_block (dspsr_b200_pipeline* pl, const InputView& in, uint64_t npart,
                       uint64_t nout, const KernelClock* clk, uint64_t* folded)
{
  dspsr_b200_context* ctx = pl->ctx;
  const ConvShape& sh = pl->conv.shape;
  const auto& cfg = pl->cfg;
  const uint64_t rows = uint64_t (sh.nchan) * cfg.npol;
  const uint64_t len = pl->sd_ncarry + nout;
  if (len > pl->sd_span)
  {
    const uint64_t span = len + len / 4;
    DevBuf<float2> nb[2];
    for (int i = 0; i < 2; i++)
      B200_CHECK (ctx, nb[i].reserve (rows * span), "cudaMalloc sample delay");
    if (pl->sd_ncarry)
      B200_CHECK (ctx, cudaMemcpy2DAsync (nb[0].ptr, span * sizeof (float2),
                                          pl->sd_buf[pl->sd_cur].ptr, pl->sd_span * sizeof (float2),
                                          pl->sd_ncarry * sizeof (float2), rows,
                                          cudaMemcpyDeviceToDevice, ctx->stream),
                  "sample delay carry");
    B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sample delay resize");
    for (int i = 0; i < 2; i++)
    {
      pl->sd_buf[i].release ();
      std::swap (pl->sd_buf[i], nb[i]);
    }
    pl->sd_span = span;
    pl->sd_cur = 0;
  }
  float2* cur = pl->sd_buf[pl->sd_cur].ptr;
  FoldView fv0 {};
  VoltView vv {cur + pl->sd_ncarry, pl->sd_span};
  const ConvTables tb = pl->conv.tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += pl->conv.max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (pl->conv.max_batch, npart - p0));
    B200_CHECK (ctx, launch_convolution (sh, tb, in, p0, nb, pl->conv.scratch.ptr, OUT_VOLTAGE,
                                         fv0, vv, ctx->stream, clk), "convolution kernels");
  }
  const uint64_t total = pl->sd.total_delay;
  const uint64_t out_n = len > total ? len - total : 0;
  if (out_n)
  {
    const uint64_t time_base = pl->sd_out0 + sh.nfilt_pos + uint64_t (pl->sd.zero_delay);
    int rc = pipeline_fold_plan (pl, pl->sd_out0, time_base, out_n);
    if (rc) return rc;
    const FoldView fv = pl->fold.view (cfg.state, pl->nout, cfg.nchan);
    B200_CHECK (ctx, launch_delay_fold (cur, pl->sd_span, pl->sd_applied.ptr, out_n, sh.nchan,
                                        cfg.npol, fv, ctx->stream, clk), "sample delay fold");
    rc = pl->fold.release_plan ();
    if (rc) return rc;
    if (pl->sub_on)
    {
      rc = subint_drain (pl, false);
      if (rc) return rc;
    }
  }
  const uint64_t keep = len - out_n;
  if (keep)
    B200_CHECK (ctx, cudaMemcpy2DAsync (pl->sd_buf[pl->sd_cur ^ 1].ptr, pl->sd_span * sizeof (float2),
                                        cur + out_n, pl->sd_span * sizeof (float2),
                                        keep * sizeof (float2), rows, cudaMemcpyDeviceToDevice,
                                        ctx->stream), "sample delay carry");
  pl->sd_cur ^= 1;
  pl->sd_ncarry = keep;
  pl->sd_out0 += out_n;
  *folded = out_n;
  return DSPSR_B200_OK;
}

// One block through SpectralKurtosis (SpectralKurtosis::transformation with
// one resolution, noverlap 1, the zero-DM input: compute on the zero-DM
// voltages, detect_skfb, mask of the dedispersed voltages; SpectralKurtosis.C
// 542-671) and the fold of zeroed data (Fold.C:895-930).  The SK blocks of M
// samples run from the start of the stream; the samples after the last whole
// block are carried (the zero-DM InputBuffering of SpectralKurtosis.C:43).
int pipeline_sk_block (dspsr_b200_pipeline* pl, const InputView& in, uint64_t npart,
                       uint64_t nout, const KernelClock* clk, uint64_t* folded)
{
  dspsr_b200_context* ctx = pl->ctx;
  const ConvShape& sh = pl->conv.shape;
  const auto& cfg = pl->cfg;
  const uint64_t rows = uint64_t (sh.nchan) * cfg.npol;
  const uint64_t len = pl->sk_ncarry + nout;
  const unsigned M = pl->sk_M;
  if (len > pl->sk_span)
  {
    // rows of an even number of samples keep every row 16-byte aligned
    const uint64_t span = (len + len / 4 + 1) & ~uint64_t (1);
    DevBuf<float2> nv[2], nz[2];
    for (int i = 0; i < 2; i++)
    {
      B200_CHECK (ctx, nv[i].reserve (rows * span), "cudaMalloc sk voltages");
      B200_CHECK (ctx, nz[i].reserve (rows * span), "cudaMalloc sk zero-DM");
    }
    if (pl->sk_ncarry)
    {
      B200_CHECK (ctx, cudaMemcpy2DAsync (nv[0].ptr, span * sizeof (float2),
                                          pl->sk_v[pl->sk_cur].ptr, pl->sk_span * sizeof (float2),
                                          pl->sk_ncarry * sizeof (float2), rows,
                                          cudaMemcpyDeviceToDevice, ctx->stream), "sk carry");
      B200_CHECK (ctx, cudaMemcpy2DAsync (nz[0].ptr, span * sizeof (float2),
                                          pl->sk_z[pl->sk_cur].ptr, pl->sk_span * sizeof (float2),
                                          pl->sk_ncarry * sizeof (float2), rows,
                                          cudaMemcpyDeviceToDevice, ctx->stream), "sk carry");
    }
    B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sk resize");
    for (int i = 0; i < 2; i++)
    {
      pl->sk_v[i].release ();
      pl->sk_z[i].release ();
      std::swap (pl->sk_v[i], nv[i]);
      std::swap (pl->sk_z[i], nz[i]);
    }
    pl->sk_span = span;
    pl->sk_cur = 0;
  }
  float2* v = pl->sk_v[pl->sk_cur].ptr;
  float2* z = pl->sk_z[pl->sk_cur].ptr;
  FoldView fv0 {};
  VoltView vv {v + pl->sk_ncarry, pl->sk_span};
  const ConvTables tb = pl->conv.tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += pl->conv.max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (pl->conv.max_batch, npart - p0));
    B200_CHECK (ctx, launch_convolution (sh, tb, in, p0, nb, pl->conv.scratch.ptr, OUT_VOLTAGE,
                                         fv0, vv, ctx->stream, clk), "convolution kernels");
  }
  // the zero-DM output: the input samples aligned with the output
  // (Convolution.C:789-796), nfilt_pos after the start of the block
  B200_CHECK (ctx, launch_zero_dm (in, tb.lut, sh.nfilt_pos, nout, z + pl->sk_ncarry,
                                   pl->sk_span, ctx->stream), "zero-DM output");
  const uint64_t nblk = len / M;
  const uint64_t out_n = nblk * M;
  if (nblk)
  {
    B200_CHECK (ctx, pl->sk_mask.reserve (nblk * sh.nchan), "cudaMalloc sk mask");
    // statistics and test of the zero-DM blocks (the kernel masks them in
    // place too, which nothing reads), then the mask of the dedispersed ones
    const uint8_t* mask = pl->sk_mask.ptr;
    if (pl->sk_proposer)
    {
      // the SK sums feed the proposer; SK's mask is its fallback
      B200_CHECK (ctx, pl->sk_sums.reserve (nblk * sh.nchan * cfg.npol * 2), "cudaMalloc sk sums");
      B200_CHECK (ctx, pl->sk_counts.reserve (nblk * sh.nchan), "cudaMalloc sk counts");
      B200_CHECK (ctx, pl->sk_pmask.reserve (nblk * sh.nchan), "cudaMalloc proposer mask");
      B200_CHECK (ctx, launch_sk (z, pl->sk_span, z, pl->sk_span, nblk, sh.nchan, cfg.npol, M, 1,
                                  1, pl->sk_lower, pl->sk_upper, pl->sk_sums.ptr,
                                  pl->sk_counts.ptr, pl->sk_mask.ptr, pl->sk_zapped.ptr,
                                  ctx->stream), "spectral kurtosis");
      int rc = dspsr_b200_rfi_proposer_features (pl->sk_proposer, pl->sk_sums.ptr,
                                                 pl->sk_counts.ptr, nblk, cfg.npol);
      if (!rc)
        rc = dspsr_b200_rfi_proposer_infer (pl->sk_proposer, pl->sk_mask.ptr, pl->sk_confidence,
                                            pl->sk_pmask.ptr, nullptr, nullptr);
      if (rc) return fail (ctx, rc, "pipeline: rfi proposer: %s", ctx->error.c_str ());
      mask = pl->sk_pmask.ptr;
    }
    else
      B200_CHECK (ctx, launch_sk (z, pl->sk_span, z, pl->sk_span, nblk, sh.nchan, cfg.npol, M, 1,
                                  1, pl->sk_lower, pl->sk_upper, nullptr, nullptr,
                                  pl->sk_mask.ptr, pl->sk_zapped.ptr, ctx->stream),
                  "spectral kurtosis");
    B200_CHECK (ctx, launch_sk_apply (mask, v, pl->sk_span, out_n, sh.nchan, cfg.npol, M,
                                      ctx->stream), "sk mask");
    pl->sk_tested += nblk * sh.nchan;
    int rc = pipeline_fold_plan (pl, pl->sk_out0, pl->sk_out0 + sh.nfilt_pos, out_n);
    if (rc) return rc;
    const FoldView fv = pl->fold.view (cfg.state, pl->nout, cfg.nchan);
    B200_CHECK (ctx, launch_zeroed_fold (v, pl->sk_span, out_n, sh.nchan, cfg.npol, fv,
                                         ctx->stream, clk), "zeroed fold");
    rc = pl->fold.release_plan ();
    if (rc) return rc;
    if (pl->sub_on)
    {
      rc = subint_drain (pl, false);
      if (rc) return rc;
    }
  }
  const uint64_t keep = len - out_n;
  if (keep)
  {
    B200_CHECK (ctx, cudaMemcpy2DAsync (pl->sk_v[pl->sk_cur ^ 1].ptr, pl->sk_span * sizeof (float2),
                                        v + out_n, pl->sk_span * sizeof (float2),
                                        keep * sizeof (float2), rows, cudaMemcpyDeviceToDevice,
                                        ctx->stream), "sk carry");
    B200_CHECK (ctx, cudaMemcpy2DAsync (pl->sk_z[pl->sk_cur ^ 1].ptr, pl->sk_span * sizeof (float2),
                                        z + out_n, pl->sk_span * sizeof (float2),
                                        keep * sizeof (float2), rows, cudaMemcpyDeviceToDevice,
                                        ctx->stream), "sk carry");
  }
  pl->sk_cur ^= 1;
  pl->sk_ncarry = keep;
  pl->sk_out0 += out_n;
  *folded = out_n;
  return DSPSR_B200_OK;
}

int pipeline_block (dspsr_b200_pipeline* pl, const void* d_in, uint64_t ndat_new,
                    uint64_t in_span, uint64_t* ndat_folded)
{
  dspsr_b200_context* ctx = pl->ctx;
  const ConvShape& sh = pl->conv.shape;
  const auto& cfg = pl->cfg;
  const uint64_t nfilt = uint64_t (sh.nfilt_pos) + sh.nfilt_neg;
  const uint64_t ndat = pl->ncarry + ndat_new;
  // after a filterbank stage the convolution reads complex-float channels,
  // unless the filterbank runs inside the column pass: then the block and the
  // carry stay raw TFPD, counted in filterbank samples of fb_nsub raw samples
  const bool fbraw = pl->fb_fused;
  const bool fpt = !fbraw && (pl->fb_nsub > 1 || cfg.input_kind == DSPSR_B200_FLOAT_FPT);
  if (ndat_folded) *ndat_folded = 0;

  InputView in;
  in.kind = fpt ? IN_FLOAT : cfg.input_kind == DSPSR_B200_INT8_TFPD ? IN_INT8 : IN_INT16;
  in.pre = pl->carry[pl->cur_carry].ptr;
  in.main = d_in;
  in.npre = pl->ncarry;
  in.pre_span = pl->carry_span;
  in.main_span = fpt ? in_span : 0;
  in.nchan = fbraw ? cfg.nchan : sh.nchan;
  in.npol = cfg.npol;
  in.offset_binary = cfg.offset_binary;
  in.fb_nsub = fbraw ? pl->fb_nsub : 0;
  in.lut_scale = fbraw ? pl->lut_scale : 0.f;

  uint64_t npart = 0;
  if (ndat >= sh.nfft) npart = (ndat - nfilt) / sh.nkeep;   // Convolution.C:486-487
  const uint64_t nout = npart * sh.nkeep;

  uint64_t nfolded = nout;
  if (npart > 0 && pl->sd_on)
  {
    KernelClock kc {&PipeClock::mark, &pl->clock};
    int rc = pipeline_sd_block (pl, in, npart, nout, pl->clock.on ? &kc : nullptr, &nfolded);
    if (rc) return rc;
  }
  else if (npart > 0 && pl->sk_on)
  {
    KernelClock kc {&PipeClock::mark, &pl->clock};
    int rc = pipeline_sk_block (pl, in, npart, nout, pl->clock.on ? &kc : nullptr, &nfolded);
    if (rc) return rc;
  }
  else if (npart > 0)
  {
    // Fold::fold (Fold.C:685-693): phase of the first output sample's midpoint;
    // the output starts nfilt_pos samples after the input (Convolution.C:599)
    int rc = pipeline_fold_plan (pl, pl->in0, pl->in0 + sh.nfilt_pos, nout);
    if (rc) return rc;
    FoldView fv = pl->fold.view (cfg.state, pl->nout, cfg.nchan);
    VoltView vv {nullptr, 0};
    const ConvTables tb = pl->conv.tables ();
    KernelClock kc {&PipeClock::mark, &pl->clock};
    const KernelClock* clk = pl->clock.on ? &kc : nullptr;
    for (uint64_t p0 = 0; p0 < npart; p0 += pl->conv.max_batch)
    {
      const unsigned nb = unsigned (std::min<uint64_t> (pl->conv.max_batch, npart - p0));
      B200_CHECK (ctx, launch_convolution (sh, tb, in, p0, nb, pl->conv.scratch.ptr, OUT_FOLD, fv,
                                           vv, ctx->stream, clk), "convolution kernels");
    }
    rc = pl->fold.release_plan ();
    if (rc) return rc;
    if (pl->sub_on)
    {
      rc = subint_drain (pl, false);
      if (rc) return rc;
    }
  }

  // InputBuffering (InputBuffering.C:66-174): samples [nout, ndat) carry over
  const uint64_t keep = ndat - nout;
  const int next = pl->cur_carry ^ 1;
  if (!fpt)
  {
    const uint64_t bps = pl->bytes_per_sample * (fbraw ? pl->fb_nsub : 1);
    B200_CHECK (ctx, pl->carry[next].reserve (std::max<uint64_t> (keep * bps, 16)),
                "cudaMalloc carry");
    uint64_t done = 0;
    if (nout < pl->ncarry)
    {
      const uint64_t n = pl->ncarry - nout;
      B200_CHECK (ctx, cudaMemcpyAsync (pl->carry[next].ptr, pl->carry[pl->cur_carry].ptr + nout * bps,
                                        n * bps, cudaMemcpyDeviceToDevice, ctx->stream),
                  "carry copy");
      done = n;
    }
    if (keep > done)
    {
      const uint64_t from = nout + done - pl->ncarry;
      B200_CHECK (ctx, cudaMemcpyAsync (pl->carry[next].ptr + done * bps,
                                        static_cast<const uint8_t*> (d_in) + from * bps,
                                        (keep - done) * bps, cudaMemcpyDeviceToDevice,
                                        ctx->stream), "carry copy");
    }
  }
  else
  {
    const uint64_t rows = uint64_t (sh.nchan) * cfg.npol;
    const uint64_t span = std::max<uint64_t> (keep, 1);
    B200_CHECK (ctx, pl->carry[next].reserve (rows * span * sizeof (float2)), "cudaMalloc carry");
    uint64_t done = 0;
    if (nout < pl->ncarry)
    {
      const uint64_t n = pl->ncarry - nout;
      B200_CHECK (ctx, cudaMemcpy2DAsync (pl->carry[next].ptr, span * sizeof (float2),
                                          pl->carry[pl->cur_carry].ptr + nout * sizeof (float2),
                                          pl->carry_span * sizeof (float2), n * sizeof (float2),
                                          rows, cudaMemcpyDeviceToDevice, ctx->stream),
                  "carry copy");
      done = n;
    }
    if (keep > done)
    {
      const uint64_t from = nout + done - pl->ncarry;
      B200_CHECK (ctx, cudaMemcpy2DAsync (pl->carry[next].ptr + done * sizeof (float2),
                                          span * sizeof (float2),
                                          static_cast<const uint8_t*> (d_in) + from * sizeof (float2),
                                          in_span * sizeof (float2), (keep - done) * sizeof (float2),
                                          rows, cudaMemcpyDeviceToDevice, ctx->stream),
                  "carry copy");
    }
    pl->carry_span = span;
  }
  pl->cur_carry = next;
  pl->ncarry = keep;
  pl->in0 += nout;
  if (ndat_folded) *ndat_folded = nfolded;
  return DSPSR_B200_OK;
}

// A block of the operation chain: with a filterbank stage the raw input is
// first channelised (Filterbank, freq_res = 1) into complex-float channels,
// which then feed the overlap-save stage.  Blocks are whole filterbank
// transforms (ndat a multiple of the channel count).
int pipeline_input (dspsr_b200_pipeline* pl, const void* d_in, uint64_t ndat, uint64_t in_span,
                    uint64_t* ndat_folded)
{
  if (!pl->fb_nsub) return pipeline_block (pl, d_in, ndat, in_span, ndat_folded);
  dspsr_b200_context* ctx = pl->ctx;
  const auto& cfg = pl->cfg;
  if (ndat % pl->fb_nsub)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: block of %llu samples is not a multiple of "
                 "the %u filterbank channels", (unsigned long long) ndat, pl->fb_nsub);
  if (pl->fb_fused)
    return pipeline_block (pl, d_in, ndat / pl->fb_nsub, 0, ndat_folded);
  const uint64_t nb = ndat / pl->fb_nsub;
  const uint64_t rows = uint64_t (pl->conv.shape.nchan) * cfg.npol;
  B200_CHECK (ctx, pl->fbbuf.reserve (std::max<uint64_t> (rows * nb, 1)), "cudaMalloc filterbank");
  InputView in {};
  in.kind = cfg.input_kind;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = cfg.nchan;
  in.npol = cfg.npol;
  in.offset_binary = cfg.offset_binary;
  const float scale = float (1.0 / std::sqrt (double (pl->fb_nsub)));
  KernelClock kc {&PipeClock::mark, &pl->clock};
  B200_CHECK (ctx, launch_filterbank (in, pl->conv.lut.ptr, pl->fb_nsub, nb, scale, pl->fbbuf.ptr,
                                      nb, ctx->stream, pl->clock.on ? &kc : nullptr, pl->fb_tab),
              "filterbank");
  return pipeline_block (pl, pl->fbbuf.ptr, nb, nb, ndat_folded);
}

} // namespace

// ---------------------------------------------------------------------------
// exported functions
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// inverse filterbank engine
// ---------------------------------------------------------------------------

struct dspsr_b200_inverse_filterbank
{
  dspsr_b200_context* ctx = nullptr;
  IfbShape shape {};
  unsigned in_discard_pos = 0, in_discard_neg = 0;
  DevBuf<int4> map;
  DevBuf<float2> tw_lin, tw4, response, scratch;
  DevBuf<float> temporal, spectral;
  DevBuf<int> err;
  bool have_response = false, have_temporal = false, have_spectral = false;
  int nsm = 148;
  unsigned max_batch = 1;

  int init (dspsr_b200_context* c, const dspsr_b200_ifb_config& cfg);
  IfbTables tables () const
  {
    IfbTables t;
    t.map = map.ptr;
    t.ptab_lin = tw_lin.ptr;
    t.tw4 = tw4.ptr;
    t.response = have_response ? response.ptr : nullptr;
    t.temporal = have_temporal ? temporal.ptr : nullptr;
    t.spectral = have_spectral ? spectral.ptr : nullptr;
    t.lut = ctx->d_lut;
    t.err = err.ptr;
    t.nsm = nsm;
    return t;
  }
  void release ()
  {
    map.release ();
    tw_lin.release ();
    tw4.release ();
    response.release ();
    scratch.release ();
    temporal.release ();
    spectral.release ();
    err.release ();
  }
};

namespace {

// The stitching of InverseFilterbankEngineCPU::perform / stitch / stitch_one /
// filter (InverseFilterbankEngineCPU.C:309-366, 443-616, 620-650), evaluated
// once on the host: where each fine channel's two kept halves land in the
// output channels' spectra, and which half the DC-channel rule zeroes.
// Returns an empty message on success.
std::string ifb_build_map (const dspsr_b200_ifb_config& cfg, unsigned keep, unsigned lout,
                           std::vector<int4>& map)
{
  const unsigned nin = cfg.input_nchan, nout = cfg.output_nchan, pfb = cfg.pfb_nchan;
  const unsigned fine_per_out = nin / nout, coarse = nin / pfb;
  unsigned coarse_per_out = 1, out_per_coarse = 1, steps = coarse, out_per_step = 1;
  std::vector<unsigned> plan;
  if (fine_per_out > pfb)
  {
    if (fine_per_out % pfb) return "output channels do not hold whole coarse channels";
    coarse_per_out = fine_per_out / pfb;
    steps = coarse / coarse_per_out;
    plan = ifb_fine_channel_plan (nin, pfb);
  }
  else if (fine_per_out < pfb)
  {
    if (pfb % fine_per_out) return "coarse channels do not split into whole output channels";
    out_per_coarse = pfb / fine_per_out;
    steps = nout / out_per_coarse;
    out_per_step = out_per_coarse;
  }
  const unsigned keep2 = keep / 2;
  const uint64_t spec_len = uint64_t (out_per_step) * lout;
  map.assign (nin, make_int4 (-1, -1, -1, -1));
  for (unsigned istep = 0; istep < steps; istep++)
  {
    const unsigned fine_offset = istep * coarse_per_out * pfb;
    const unsigned out_offset = istep * out_per_coarse;
    std::vector<char> covered (spec_len / keep2, 0);
    for (unsigned icoarse = 0; icoarse < coarse_per_out; icoarse++)
    {
      const uint64_t soff = uint64_t (icoarse) * keep * pfb;
      for (unsigned ich = 0; ich < pfb; ich++)
      {
        unsigned jch = fine_offset + icoarse * pfb + ich;
        if (coarse_per_out > 1) jch = plan[jch];
        uint64_t neg, pos;
        if (cfg.pfb_dc_chan)
        {
          neg = ich == 0 ? uint64_t (keep) * pfb - keep2 : uint64_t (keep) * ich - keep2;
          pos = ich == 0 ? 0 : neg + keep2;
        }
        else
        {
          neg = uint64_t (keep) * ich;
          pos = neg + keep2;
        }
        neg += soff;
        pos += soff;
        if (map[jch].x >= 0) return "an input channel is stitched twice";
        for (uint64_t at : {neg, pos})
        {
          if (at % keep2 || at >= spec_len || covered[at / keep2]) return "stitched halves overlap";
          covered[at / keep2] = 1;
        }
        map[jch] = make_int4 (int (out_offset + neg / lout), int (neg % lout),
                              int (out_offset + pos / lout), int (pos % lout));
      }
    }
    for (char c : covered)
      if (!c) return "stitched spectrum has gaps";
    // filter: without every PFB channel, the last half channel is zeroed
    if (!cfg.pfb_all_chan && cfg.pfb_dc_chan)
    {
      const uint64_t z = spec_len - keep2;
      const int zo = int (out_offset + z / lout), zk = int (z % lout);
      for (int4& m : map)
      {
        if (m.x == zo && m.y == zk) m.y |= IFB_ZERO;
        if (m.z == zo && m.w == zk) m.w |= IFB_ZERO;
      }
    }
  }
  return std::string ();
}

} // namespace

int dspsr_b200_inverse_filterbank::init (dspsr_b200_context* c, const dspsr_b200_ifb_config& cfg)
{
  ctx = c;
  const unsigned nin = cfg.input_nchan, nout = cfg.output_nchan, pfb = cfg.pfb_nchan;
  if (!nin || !nout || !pfb || nin % nout || nin % pfb || cfg.npol == 0 || cfg.npol > 2 ||
      nin > 65535)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "inverse filterbank: invalid channels (in %u, out %u, pfb %u, npol %u)", nin,
                 nout, pfb, cfg.npol);
  const unsigned lin = cfg.input_fft_length;
  if (!ifb_supported_lin (lin))
    return fail (ctx, DSPSR_B200_EINVAL,
                 "inverse filterbank: input FFT length %u not a power of two in [64, 4096]", lin);
  // Rational::normalize (Rational.C:83-90): the kept bins of each fine channel
  if (!cfg.os_num || !cfg.os_den || (uint64_t (lin) * cfg.os_den) % cfg.os_num)
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: %u * %u/%u is not an integer", lin,
                 cfg.os_den, cfg.os_num);
  const unsigned keep = unsigned (uint64_t (lin) * cfg.os_den / cfg.os_num);
  if (keep == 0 || keep > lin || keep % 2 || (lin - keep) % 2)
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: kept bins %u must be even", keep);
  const unsigned lout = nin / nout * keep;
  // output_to_input (InverseFilterbank.C:128-142) of the output discards
  const uint64_t num = uint64_t (nout) * cfg.os_num, den = uint64_t (nin) * cfg.os_den;
  if ((uint64_t (cfg.output_discard_pos) * num) % den ||
      (uint64_t (cfg.output_discard_neg) * num) % den)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "inverse filterbank: output discards do not map to whole input samples");
  in_discard_pos = unsigned (uint64_t (cfg.output_discard_pos) * num / den);
  in_discard_neg = unsigned (uint64_t (cfg.output_discard_neg) * num / den);
  if (uint64_t (cfg.output_discard_pos) + cfg.output_discard_neg >= lout ||
      uint64_t (in_discard_pos) + in_discard_neg >= lin)
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: discards exceed the FFT length");
  unsigned n2 = 0, n1 = 0;
  for (unsigned cand : {8192u, 4096u})
  {
    if (lout % cand) continue;
    const unsigned r = lout / cand;
    if (r == 2 || r == 3 || r == 4 || r == 6 || r == 8 || r == 12 || r == 16 || r == 24 ||
        r == 32)
    {
      n2 = cand;
      n1 = r;
      break;
    }
  }
  if (!n2)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "inverse filterbank: output FFT length %u is not n1 x 4096 or n1 x 8192 with "
                 "n1 in {2,3,4,6,8,12,16,24,32}", lout);
  std::vector<int4> m;
  const std::string why = ifb_build_map (cfg, keep, lout, m);
  if (!why.empty ()) return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: %s", why.c_str ());
  shape.nin = nin;
  shape.nout = nout;
  shape.npol = cfg.npol;
  shape.lin = lin;
  shape.keep = keep;
  shape.lout = lout;
  shape.n1 = n1;
  shape.n2 = n2;
  shape.in_step = lin - in_discard_pos - in_discard_neg;
  shape.out_step = lout - cfg.output_discard_pos - cfg.output_discard_neg;
  shape.out_discard_pos = cfg.output_discard_pos;
  shape.dual_sideband = cfg.dual_sideband;
  B200_CHECK (ctx, map.reserve (nin), "cudaMalloc stitch map");
  B200_CHECK (ctx, cudaMemcpy (map.ptr, m.data (), nin * sizeof (int4), cudaMemcpyHostToDevice),
              "copy stitch map");
  const unsigned ntab_lin = pass_tables_count (lin);
  std::vector<float2> t (std::max (ntab_lin, 1u), make_float2 (0.f, 0.f));
  make_pass_tables (lin, t.data (), ntab_lin);
  B200_CHECK (ctx, tw_lin.reserve (t.size ()), "cudaMalloc twiddles");
  B200_CHECK (ctx, cudaMemcpy (tw_lin.ptr, t.data (), t.size () * sizeof (float2),
                               cudaMemcpyHostToDevice), "copy twiddles");
  t = make_tw4 (n1, n2);
  B200_CHECK (ctx, tw4.reserve (lout), "cudaMalloc four-step twiddles");
  B200_CHECK (ctx, cudaMemcpy (tw4.ptr, t.data (), lout * sizeof (float2),
                               cudaMemcpyHostToDevice), "copy four-step twiddles");
  B200_CHECK (ctx, err.reserve (1), "cudaMalloc status flag");
  B200_CHECK (ctx, cudaMemset (err.ptr, 0, sizeof (int)), "clear status flag");
  int dev = 0;
  B200_CHECK (ctx, cudaGetDevice (&dev), "cudaGetDevice");
  B200_CHECK (ctx, cudaDeviceGetAttribute (&nsm, cudaDevAttrMultiProcessorCount, dev),
              "multiprocessor count");
  const uint64_t per_part = uint64_t (nout) * cfg.npol * lout * sizeof (float2);
  const uint64_t budget = cfg.scratch_bytes ? cfg.scratch_bytes : (uint64_t (512) << 20);
  max_batch = unsigned (std::max<uint64_t> (1, std::min<uint64_t> (65535, budget / per_part)));
  B200_CHECK (ctx, scratch.reserve (size_t (max_batch) * nout * cfg.npol * lout),
              "cudaMalloc scratch");
  return DSPSR_B200_OK;
}

extern "C" {

int dspsr_b200_inverse_filterbank_create (dspsr_b200_context* ctx,
                                          const dspsr_b200_ifb_config* cfg,
                                          dspsr_b200_inverse_filterbank** out)
{
  if (!ctx || !cfg || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  dspsr_b200_inverse_filterbank* f = new (std::nothrow) dspsr_b200_inverse_filterbank;
  if (!f) return fail (ctx, DSPSR_B200_ENOMEM, "inverse filterbank: out of host memory");
  const int rc = f->init (ctx, *cfg);
  if (rc)
  {
    f->release ();
    delete f;
    return rc;
  }
  *out = f;
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_destroy (dspsr_b200_inverse_filterbank* f)
{
  if (!f) return DSPSR_B200_EINVAL;
  cudaStreamSynchronize (f->ctx->stream);
  f->release ();
  delete f;
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_info (dspsr_b200_inverse_filterbank* f, uint64_t* info)
{
  if (!f || !info) return DSPSR_B200_EINVAL;
  const IfbShape& s = f->shape;
  const uint64_t v[10] = {s.keep, s.lout, s.in_step, s.out_step, f->in_discard_pos,
                          f->in_discard_neg, s.n1, s.n2, f->max_batch, s.lin};
  for (int i = 0; i < 10; i++) info[i] = v[i];
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_copy_response (dspsr_b200_inverse_filterbank* f,
                                                 const float* response)
{
  if (!f) return DSPSR_B200_EINVAL;
  if (!response)
  {
    f->have_response = false;
    return DSPSR_B200_OK;
  }
  const size_t n = size_t (f->shape.nout) * f->shape.lout;
  B200_CHECK (f->ctx, f->response.reserve (n), "cudaMalloc response");
  B200_CHECK (f->ctx, cudaMemcpy (f->response.ptr, response, n * sizeof (float2),
                                  cudaMemcpyHostToDevice), "copy response");
  f->have_response = true;
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_set_apodization (dspsr_b200_inverse_filterbank* f,
                                                   const float* temporal, const float* spectral)
{
  if (!f) return DSPSR_B200_EINVAL;
  f->have_temporal = f->have_spectral = false;
  if (temporal)
  {
    B200_CHECK (f->ctx, f->temporal.reserve (f->shape.lin), "cudaMalloc temporal window");
    B200_CHECK (f->ctx, cudaMemcpy (f->temporal.ptr, temporal, f->shape.lin * sizeof (float),
                                    cudaMemcpyHostToDevice), "copy temporal window");
    f->have_temporal = true;
  }
  if (spectral)
  {
    B200_CHECK (f->ctx, f->spectral.reserve (f->shape.lout), "cudaMalloc spectral window");
    B200_CHECK (f->ctx, cudaMemcpy (f->spectral.ptr, spectral, f->shape.lout * sizeof (float),
                                    cudaMemcpyHostToDevice), "copy spectral window");
    f->have_spectral = true;
  }
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_perform (dspsr_b200_inverse_filterbank* f, int input_kind,
                                           const void* d_in, uint64_t ndat, uint64_t in_span,
                                           const float* lut256, int offset_binary, float* d_out,
                                           uint64_t out_span, uint64_t* npart_out)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (npart_out) *npart_out = 0;
  if (!d_in || !d_out) return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: null buffer");
  if (input_kind < 0 || input_kind > 2 || (input_kind == DSPSR_B200_INT8_TFPD && !lut256))
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: invalid input kind or missing table");
  if (input_kind == DSPSR_B200_FLOAT_FPT && in_span < ndat)
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: in_span < ndat");
  const IfbShape& s = f->shape;
  const uint64_t disc = uint64_t (f->in_discard_pos) + f->in_discard_neg;
  // InverseFilterbank::resize_output (InverseFilterbank.C:599-634)
  const uint64_t npart = ndat > disc ? (ndat - disc) / s.in_step : 0;
  if (npart && npart * s.in_step + disc > ndat) return fail (ctx, DSPSR_B200_EINVAL, "bad npart");
  if (out_span < npart * s.out_step)
    return fail (ctx, DSPSR_B200_EINVAL, "inverse filterbank: out_span < npart * out_step");
  if (input_kind == DSPSR_B200_INT8_TFPD)
    B200_CHECK (ctx, cudaMemcpyAsync (ctx->d_lut, lut256, 256 * sizeof (float),
                                      cudaMemcpyHostToDevice, ctx->stream), "upload lut");
  InputView in {};
  in.kind = input_kind;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = s.nin;
  in.npol = s.npol;
  in.offset_binary = offset_binary;
  VoltView vv {reinterpret_cast<float2*> (d_out), out_span};
  const IfbTables tb = f->tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += f->max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (f->max_batch, npart - p0));
    B200_CHECK (ctx, launch_inverse_filterbank (s, tb, in, p0, nb, f->scratch.ptr, vv,
                                                ctx->stream), "inverse filterbank kernels");
  }
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_inverse_filterbank_status (dspsr_b200_inverse_filterbank* f)
{
  if (!f) return DSPSR_B200_EINVAL;
  int h = 0;
  B200_CHECK (f->ctx, cudaMemcpyAsync (&h, f->err.ptr, sizeof (int), cudaMemcpyDeviceToHost,
                                       f->ctx->stream), "read device status");
  B200_CHECK (f->ctx, cudaStreamSynchronize (f->ctx->stream), "device status sync");
  if (h) return fail (f->ctx, DSPSR_B200_ESTATE, "a device-side wait timed out");
  return DSPSR_B200_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// filterbank with a response ("During")
// ---------------------------------------------------------------------------

struct dspsr_b200_filterbank_during
{
  dspsr_b200_context* ctx = nullptr;
  DuringShape shape {};
  DevBuf<float2> tw4, ptab_seg, ptab_col, twd, H, Hw, tmp, scratch;
  DevBuf<double> chan_par;
  DevBuf<float> temporal, spectral;
  bool have_response = false, have_temporal = false, have_spectral = false;
  int nsm = 148;
  unsigned max_batch = 1;

  DuringTables tables () const
  {
    DuringTables t;
    t.tw4 = tw4.ptr;
    t.ptab_seg = ptab_seg.ptr;
    t.twd = twd.ptr;
    t.ptab_col = ptab_col.ptr;
    t.H = have_spectral ? Hw.ptr : H.ptr;
    t.lut = ctx->d_lut;
    t.nsm = nsm;
    t.apod = have_temporal ? temporal.ptr : nullptr;
    return t;
  }
  // the response the kernels read: H, times the spectral window when one is set
  cudaError_t window_response ()
  {
    if (!have_spectral || !have_response) return cudaSuccess;
    return launch_window_response (Hw.ptr, H.ptr, spectral.ptr, shape.nchan_in * shape.nsub,
                                   shape.n1, shape.seg, ctx->stream);
  }
  void release ()
  {
    tw4.release ();
    ptab_seg.release ();
    ptab_col.release ();
    twd.release ();
    H.release ();
    Hw.release ();
    temporal.release ();
    spectral.release ();
    tmp.release ();
    scratch.release ();
    chan_par.release ();
  }
  int init (dspsr_b200_context* c, const dspsr_b200_fbd_config& cfg);
};

int dspsr_b200_filterbank_during::init (dspsr_b200_context* c, const dspsr_b200_fbd_config& cfg)
{
  ctx = c;
  if (cfg.input_nchan == 0 || cfg.npol == 0 || cfg.npol > 2)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: invalid channel or polarisation count");
  if (!during_supported (cfg.nsub, cfg.freq_res))
    return fail (ctx, DSPSR_B200_EINVAL,
                 "filterbank during: nsub=%u freq_res=%u unsupported (nsub a power of two in "
                 "[2, 128], freq_res a power of two, nsub*freq_res in [16384, 4194304])",
                 cfg.nsub, cfg.freq_res);
  // Filterbank::do_prepare (Filterbank.C:155-196): nkeep = freq_res - nfilt_tot
  if (uint64_t (cfg.nfilt_pos) + cfg.nfilt_neg >= cfg.freq_res)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: freq_res=%u <= nfilt=%u",
                 cfg.freq_res, cfg.nfilt_pos + cfg.nfilt_neg);
  DuringShape& s = shape;
  s.nchan_in = cfg.input_nchan;
  s.npol = cfg.npol;
  s.nsub = cfg.nsub;
  s.freq_res = cfg.freq_res;
  s.nfilt_pos = cfg.nfilt_pos;
  s.nfilt_neg = cfg.nfilt_neg;
  s.n2 = 8192;
  s.n1 = unsigned (uint64_t (cfg.nsub) * cfg.freq_res / s.n2);
  s.seg = s.n2 / cfg.nsub;
  s.nkeep = cfg.freq_res - cfg.nfilt_pos - cfg.nfilt_neg;
  s.in_step = uint64_t (cfg.nsub) * s.nkeep;
  const uint64_t N = uint64_t (s.n1) * s.n2;
  const std::vector<float2> t4 = make_tw4 (s.n1, s.n2);
  const std::vector<float2> td = make_tw4 (s.n1, s.seg);
  B200_CHECK (ctx, tw4.reserve (t4.size ()), "cudaMalloc tw4");
  B200_CHECK (ctx, cudaMemcpy (tw4.ptr, t4.data (), t4.size () * sizeof (float2),
                               cudaMemcpyHostToDevice), "copy tw4");
  B200_CHECK (ctx, twd.reserve (td.size ()), "cudaMalloc channel twiddles");
  B200_CHECK (ctx, cudaMemcpy (twd.ptr, td.data (), td.size () * sizeof (float2),
                               cudaMemcpyHostToDevice), "copy channel twiddles");
  // pass tables of the segment and (n1 >= 64) column transforms (the row
  // kernel builds its own)
  for (int which = 1; which < 3; which++)
  {
    if (which == 2 && s.n1 < 64) break;
    const unsigned n = which == 2 ? s.n1 : s.seg;
    DevBuf<float2>& dst = which == 2 ? ptab_col : ptab_seg;
    const unsigned cnt = pass_tables_count (n);
    std::vector<float2> pt (std::max (cnt, 1u), make_float2 (0.f, 0.f));
    make_pass_tables (n, pt.data (), cnt);
    B200_CHECK (ctx, dst.reserve (pt.size ()), "cudaMalloc pass tables");
    B200_CHECK (ctx, cudaMemcpy (dst.ptr, pt.data (), pt.size () * sizeof (float2),
                                 cudaMemcpyHostToDevice), "copy pass tables");
  }
  int dev = 0;
  B200_CHECK (ctx, cudaGetDevice (&dev), "cudaGetDevice");
  B200_CHECK (ctx, cudaDeviceGetAttribute (&nsm, cudaDevAttrMultiProcessorCount, dev),
              "multiprocessor count");
  const uint64_t per_part = uint64_t (s.nchan_in) * s.npol * N * sizeof (float2);
  const uint64_t budget = cfg.scratch_bytes ? cfg.scratch_bytes : (uint64_t (512) << 20);
  max_batch = unsigned (std::max<uint64_t> (1, std::min<uint64_t> (65535, budget / per_part)));
  B200_CHECK (ctx, scratch.reserve (uint64_t (max_batch) * s.nchan_in * s.npol * N),
              "cudaMalloc scratch");
  B200_CHECK (ctx, H.reserve (uint64_t (s.nchan_in) * s.nsub * s.freq_res), "cudaMalloc response");
  return DSPSR_B200_OK;
}

extern "C" {

int dspsr_b200_filterbank_during_create (dspsr_b200_context* ctx, const dspsr_b200_fbd_config* cfg,
                                         dspsr_b200_filterbank_during** out)
{
  if (!ctx || !cfg || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  dspsr_b200_filterbank_during* f = new (std::nothrow) dspsr_b200_filterbank_during;
  if (!f) return fail (ctx, DSPSR_B200_ENOMEM, "filterbank during: out of host memory");
  const int rc = f->init (ctx, *cfg);
  if (rc)
  {
    dspsr_b200_filterbank_during_destroy (f);
    return rc;
  }
  *out = f;
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_destroy (dspsr_b200_filterbank_during* f)
{
  if (!f) return DSPSR_B200_EINVAL;
  if (f->ctx) cudaStreamSynchronize (f->ctx->stream);
  f->release ();
  delete f;
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_info (dspsr_b200_filterbank_during* f, uint64_t* info)
{
  if (!f || !info) return DSPSR_B200_EINVAL;
  const DuringShape& s = f->shape;
  info[0] = uint64_t (s.nsub) * s.freq_res;
  info[1] = s.in_step;
  info[2] = uint64_t (s.nsub) * (s.nfilt_pos + s.nfilt_neg);
  info[3] = s.nkeep;
  info[4] = s.n1;
  info[5] = f->max_batch;
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_copy_response (dspsr_b200_filterbank_during* f,
                                                const float* response)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (!response) return fail (ctx, DSPSR_B200_EINVAL, "copy_response: null response");
  const DuringShape& s = f->shape;
  const unsigned nchan = s.nchan_in * s.nsub;
  const uint64_t n = uint64_t (nchan) * s.freq_res;
  B200_CHECK (ctx, f->tmp.reserve (n), "cudaMalloc response staging");
  B200_CHECK (ctx, cudaMemcpyAsync (f->tmp.ptr, response, n * sizeof (float2),
                                    cudaMemcpyHostToDevice, ctx->stream), "upload response");
  // bin k1 + n1*f2 of each channel to [chan][k1][f2]
  B200_CHECK (ctx, launch_permute_response (f->H.ptr, f->tmp.ptr, nchan, s.n1, s.seg, ctx->stream),
              "permute response");
  f->have_response = true;
  B200_CHECK (ctx, f->window_response (), "spectral window");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "copy_response sync");
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_set_dedispersion (dspsr_b200_filterbank_during* f, double cf,
                                                   double bw, double dm, int swapped,
                                                   int chirp_mode)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (bw == 0 || !(cf > 0))
    return fail (ctx, DSPSR_B200_EINVAL, "set_dedispersion: invalid frequency/bandwidth");
  const DuringShape& s = f->shape;
  const unsigned nchan = s.nchan_in * s.nsub;
  // response channel j holds natural channel j, or channel (j + nchan/2) mod
  // nchan after the whole response is swapped (half of nchan*freq_res points
  // is nchan/2 whole channels)
  std::vector<double> par (2 * nchan);
  const double sign = bw / std::fabs (bw);
  const double dispersion_per_MHz = 1e6 * dm / 2.41e-4;
  for (unsigned j = 0; j < nchan; j++)
  {
    const double fr = channel_centre (cf, bw, nchan, j, swapped != 0, false);
    if (!(fr > 0)) return fail (ctx, DSPSR_B200_EINVAL, "set_dedispersion: channel below 0 MHz");
    par[j] = fr;
    par[nchan + j] = -sign * 2 * M_PI * dispersion_per_MHz / (fr * fr);
  }
  const double chanwidth = bw / double (nchan);
  const double binwidth = chanwidth / double (s.freq_res);
  const float scale = float (1.0 / std::sqrt (double (s.nsub) * s.freq_res * double (s.freq_res)));
  B200_CHECK (ctx, f->chan_par.reserve (2 * nchan), "cudaMalloc channel table");
  B200_CHECK (ctx, cudaMemcpyAsync (f->chan_par.ptr, par.data (), par.size () * sizeof (double),
                                    cudaMemcpyHostToDevice, ctx->stream), "upload channels");
  B200_CHECK (ctx, launch_build_chirp (f->H.ptr, f->chan_par.ptr, f->chan_par.ptr + nchan, nullptr,
                                       nchan, s.freq_res, s.n1, s.seg, binwidth, 0.5 * chanwidth,
                                       0, chirp_mode, scale, ctx->stream),
              "build chirp");
  f->have_response = true;
  B200_CHECK (ctx, f->window_response (), "spectral window");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "set_dedispersion sync");
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_set_apodization (dspsr_b200_filterbank_during* f,
                                                   const float* temporal, const float* spectral)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  const DuringShape& s = f->shape;
  const uint64_t nfft = uint64_t (s.nsub) * s.freq_res;
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "set_apodization sync");
  f->have_temporal = false;
  if (temporal)
  {
    B200_CHECK (ctx, f->temporal.reserve (nfft), "cudaMalloc temporal window");
    B200_CHECK (ctx, cudaMemcpy (f->temporal.ptr, temporal, nfft * sizeof (float),
                                 cudaMemcpyHostToDevice), "upload temporal window");
    f->have_temporal = true;
  }
  f->have_spectral = false;
  if (spectral)
  {
    B200_CHECK (ctx, f->spectral.reserve (s.freq_res), "cudaMalloc spectral window");
    B200_CHECK (ctx, cudaMemcpy (f->spectral.ptr, spectral, s.freq_res * sizeof (float),
                                 cudaMemcpyHostToDevice), "upload spectral window");
    B200_CHECK (ctx, f->Hw.reserve (uint64_t (s.nchan_in) * s.nsub * s.freq_res),
                "cudaMalloc windowed response");
    f->have_spectral = true;
    B200_CHECK (ctx, f->window_response (), "spectral window");
    B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "set_apodization sync");
  }
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_get_response (dspsr_b200_filterbank_during* f, float* response)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (!response) return fail (ctx, DSPSR_B200_EINVAL, "get_response: null pointer");
  const DuringShape& s = f->shape;
  const unsigned nchan = s.nchan_in * s.nsub;
  const uint64_t n = uint64_t (nchan) * s.freq_res;
  B200_CHECK (ctx, f->tmp.reserve (n), "cudaMalloc response staging");
  B200_CHECK (ctx, launch_unpermute_response (f->tmp.ptr, f->H.ptr, nchan, s.n1, s.seg,
                                              ctx->stream), "unpermute response");
  B200_CHECK (ctx, cudaMemcpyAsync (response, f->tmp.ptr, n * sizeof (float2),
                                    cudaMemcpyDeviceToHost, ctx->stream), "download response");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "get_response sync");
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_perform (dspsr_b200_filterbank_during* f, int input_kind,
                                          const void* d_in, uint64_t ndat, uint64_t in_span,
                                          const float* lut256, int offset_binary, float* d_out,
                                          uint64_t out_span, uint64_t* npart_out)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (npart_out) *npart_out = 0;
  if (!f->have_response) return fail (ctx, DSPSR_B200_ESTATE, "filterbank during: no response set");
  if (!d_in || !d_out) return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: null buffer");
  if (input_kind < 0 || input_kind > 2 || (input_kind == DSPSR_B200_INT8_TFPD && !lut256))
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: invalid input kind or missing table");
  if (input_kind == DSPSR_B200_FLOAT_FPT && in_span < ndat)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: in_span < ndat");
  const DuringShape& s = f->shape;
  // Filterbank::resize_output (Filterbank.C:398-420)
  const uint64_t overlap = uint64_t (s.nsub) * (s.nfilt_pos + s.nfilt_neg);
  const uint64_t npart = ndat > overlap ? (ndat - overlap) / s.in_step : 0;
  if (out_span < npart * s.nkeep)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: out_span < npart * nkeep");
  if (input_kind == DSPSR_B200_INT8_TFPD)
    B200_CHECK (ctx, cudaMemcpyAsync (ctx->d_lut, lut256, 256 * sizeof (float),
                                      cudaMemcpyHostToDevice, ctx->stream), "upload lut");
  InputView in {};
  in.kind = input_kind;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = s.nchan_in;
  in.npol = s.npol;
  in.offset_binary = offset_binary;
  VoltView vv {reinterpret_cast<float2*> (d_out), out_span};
  FoldView fv {};
  const DuringTables tb = f->tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += f->max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (f->max_batch, npart - p0));
    B200_CHECK (ctx, launch_filterbank_during (s, tb, in, p0, nb, f->scratch.ptr, OUT_VOLTAGE, fv,
                                               vv, ctx->stream), "filterbank during kernels");
  }
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_filterbank_during_perform_fold (dspsr_b200_filterbank_during* f, int input_kind,
                                               const void* d_in, uint64_t ndat, uint64_t in_span,
                                               const float* lut256, int offset_binary,
                                               dspsr_b200_fold* fold, int state,
                                               uint64_t* npart_out)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (npart_out) *npart_out = 0;
  if (!f->have_response) return fail (ctx, DSPSR_B200_ESTATE, "filterbank during: no response set");
  if (!d_in || !fold) return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: null argument");
  if (input_kind < 0 || input_kind > 2 || (input_kind == DSPSR_B200_INT8_TFPD && !lut256))
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: invalid input kind or missing table");
  if (input_kind == DSPSR_B200_FLOAT_FPT && in_span < ndat)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: in_span < ndat");
  const DuringShape& s = f->shape;
  if (state < 0 || state > 3 || (s.npol == 1 && state != DSPSR_B200_INTENSITY))
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank during: detection state %d with %u pol",
                 state, s.npol);
  const int nout = detect_nout (state);
  const uint64_t overlap = uint64_t (s.nsub) * (s.nfilt_pos + s.nfilt_neg);
  const uint64_t npart = ndat > overlap ? (ndat - overlap) / s.in_step : 0;
  if (fold->ctx != ctx || fold->nchan != s.nchan_in * s.nsub || fold->npol != unsigned (nout))
    return fail (ctx, DSPSR_B200_EINVAL,
                 "filterbank during: fold engine of %u channels x %u products, expected %u x %d",
                 fold->nchan, fold->npol, s.nchan_in * s.nsub, nout);
  if (fold->ndat != npart * s.nkeep)
    return fail (ctx, DSPSR_B200_ESTATE,
                 "filterbank during: fold plan covers %llu samples, the parts give %llu",
                 (unsigned long long) fold->ndat, (unsigned long long) (npart * s.nkeep));
  if (input_kind == DSPSR_B200_INT8_TFPD)
    B200_CHECK (ctx, cudaMemcpyAsync (ctx->d_lut, lut256, 256 * sizeof (float),
                                      cudaMemcpyHostToDevice, ctx->stream), "upload lut");
  InputView in {};
  in.kind = input_kind;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = s.nchan_in;
  in.npol = s.npol;
  in.offset_binary = offset_binary;
  VoltView vv {nullptr, 0};
  const FoldView fv = fold->view (state, nout, fold->nchan);
  const DuringTables tb = f->tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += f->max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (f->max_batch, npart - p0));
    B200_CHECK (ctx, launch_filterbank_during (s, tb, in, p0, nb, f->scratch.ptr, OUT_FOLD, fv, vv,
                                               ctx->stream), "filterbank during kernels");
  }
  const int rc = fold->release_plan ();
  if (rc) return rc;
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_archive_profiles (const float* sums, const uint32_t* hits, int zeroed_data,
                                 unsigned nchan, unsigned npol, unsigned nbin, double scale,
                                 uint64_t ndat_total, int unload_zero_hits, float* amps,
                                 float* weights, unsigned* corrupted)
{
  const int rc = archive_profiles (sums, hits, zeroed_data != 0, nchan, npol, nbin, scale,
                                   ndat_total, unload_zero_hits != 0, amps, weights, corrupted);
  return rc == 0 ? DSPSR_B200_OK : rc == -2 ? DSPSR_B200_ESTATE : DSPSR_B200_EINVAL;
}

int dspsr_b200_apodization (int type, unsigned ndat, unsigned transition_start,
                            unsigned transition_end, int swap_halves, float* window)
{
  if (!window) return DSPSR_B200_EINVAL;
  return apodization (type, ndat, transition_start, transition_end, swap_halves != 0, window)
             ? DSPSR_B200_EINVAL : DSPSR_B200_OK;
}

} // extern "C"

extern "C" {

int dspsr_b200_version (void) { return 100; }

int dspsr_b200_context_create (int device, void* stream, dspsr_b200_context** out)
{
  if (!out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount (&ndev) != cudaSuccess || ndev == 0)
    return DSPSR_B200_ENODEV;
  if (device < 0 || device >= ndev) return DSPSR_B200_EINVAL;
  if (cudaSetDevice (device) != cudaSuccess) return DSPSR_B200_ECUDA;
  dspsr_b200_context* ctx = new (std::nothrow) dspsr_b200_context;
  if (!ctx) return DSPSR_B200_ENOMEM;
  ctx->device = device;
  ctx->stream = static_cast<cudaStream_t> (stream);
  if (cudaMalloc (&ctx->d_lut, 256 * sizeof (float)) != cudaSuccess)
  {
    delete ctx;
    return DSPSR_B200_ECUDA;
  }
  *out = ctx;
  return DSPSR_B200_OK;
}

int dspsr_b200_context_destroy (dspsr_b200_context* ctx)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (ctx->d_lut) cudaFree (ctx->d_lut);
  if (ctx->d_fb_tab) cudaFree (ctx->d_fb_tab);
  delete ctx;
  return DSPSR_B200_OK;
}

int dspsr_b200_context_set_stream (dspsr_b200_context* ctx, void* stream)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  ctx->stream = static_cast<cudaStream_t> (stream);
  return DSPSR_B200_OK;
}

const char* dspsr_b200_last_error (const dspsr_b200_context* ctx)
{
  return ctx ? ctx->error.c_str () : "null context";
}

int dspsr_b200_synchronize (dspsr_b200_context* ctx)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "cudaStreamSynchronize");
  return DSPSR_B200_OK;
}

unsigned dspsr_b200_smearing_samples (double cf, double bw, double dm, unsigned nchan, int half)
{
  if (nchan == 0 || !(half == 0 || half == 1 || half == -1)) return 0;
  return smearing_samples (cf, bw, dm, nchan, half);
}

unsigned dspsr_b200_minimum_ndat (unsigned pos, unsigned neg) { return minimum_ndat (pos, neg); }

int64_t dspsr_b200_optimal_fft_length (uint64_t nbad, uint64_t nmax, unsigned factor)
{
  return optimal_fft_length (nbad, nmax, factor);
}

int dspsr_b200_bittable8 (double spacing, int twos_complement, float* lut, double* scale)
{
  if (!lut || !(spacing > 0)) return DSPSR_B200_EINVAL;
  bittable8 (spacing, twos_complement != 0, lut, scale);
  return DSPSR_B200_OK;
}

double dspsr_b200_fold_phi (int64_t sd, int64_t ss, double sf, int64_t ed, int64_t es, double ef,
                            uint64_t idat_start, double rate, double period, double ref_phase)
{
  return fold_phi (sd, ss, sf, ed, es, ef, idat_start, rate, period, ref_phase);
}

int dspsr_b200_interchannel_delays (double cf, double dm, double rate, const double* freq,
                                    unsigned nchan, int64_t* delay, double* frac,
                                    int64_t* applied, int64_t* zero_delay, uint64_t* total_delay)
{
  if (!freq || nchan == 0 || !(rate > 0) || !(cf > 0)) return DSPSR_B200_EINVAL;
  InterchannelDelays d;
  interchannel_delays (cf, dm, rate, freq, nchan, &d);
  for (unsigned c = 0; c < nchan; c++)
  {
    if (delay) delay[c] = d.delay[c];
    if (frac) frac[c] = d.frac[c];
    if (applied) applied[c] = d.applied[c];
  }
  if (zero_delay) *zero_delay = d.zero_delay;
  if (total_delay) *total_delay = d.total_delay;
  return DSPSR_B200_OK;
}

int64_t dspsr_b200_fold_plan_count (double phi, double pps, uint64_t ndat)
{
  return build_fold_plan (phi, pps, ndat, nullptr);
}

int dspsr_b200_sk_limits (unsigned M, unsigned Nd, float std_devs, unsigned ntest, float* lower,
                          float* upper)
{
  if (!lower || !upper) return DSPSR_B200_EINVAL;
  const int rc = sk_limits (M, Nd, std_devs, ntest, lower, upper);
  return rc == 0 ? DSPSR_B200_OK : rc == -2 ? DSPSR_B200_ESTATE : DSPSR_B200_EINVAL;
}

// ---- spectral kurtosis -------------------------------------------------------

int dspsr_b200_sk (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span, uint64_t ndat,
                   unsigned nchan, unsigned npol, unsigned M, int zero_is_valid, unsigned Nd,
                   float lower, float upper, float* d_out, uint64_t out_span, float* d_sums,
                   uint32_t* d_counts, uint8_t* d_mask, uint64_t* d_zapped, uint64_t* npart_out)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (npart_out) *npart_out = 0;
  if (!d_in || !d_out || nchan == 0 || nchan > 65535 || Nd == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: invalid argument");
  if (npol != 1 && npol != 2)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: npol must be 1 or 2 (got %u)", npol);
  if (M < 2 || (M & 1) || (in_span & 1) || (out_span & 1))
    return fail (ctx, DSPSR_B200_EINVAL, "sk: M and the spans must be even (M=%u)", M);
  if ((reinterpret_cast<uintptr_t> (d_in) | reinterpret_cast<uintptr_t> (d_out)) & 15)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: buffers must be 16-byte aligned");
  if (M > (1u << 20) || sk_smem_bytes (npol, M, 1) > SK_SMEM_MAX)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: npol*M = %u exceeds the shared-memory block",
                 npol * M);
  const uint64_t npart = ndat / M;
  if (in_span < npart * M || out_span < npart * M)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: span smaller than the blocks");
  if (npart > 0x7fffffffull) return fail (ctx, DSPSR_B200_EINVAL, "sk: too many blocks");
  if (d_in != d_out)
  {
    // partial overlap of input and output is not supported
    const char* a = reinterpret_cast<const char*> (d_in);
    const char* b = reinterpret_cast<const char*> (d_out);
    const uint64_t na = (uint64_t (nchan) * npol * in_span) * 8;
    const uint64_t nb = (uint64_t (nchan) * npol * out_span) * 8;
    if (a < b + nb && b < a + na)
      return fail (ctx, DSPSR_B200_EINVAL, "sk: input and output overlap without being equal");
  }
  if (d_in == d_out && in_span != out_span)
    return fail (ctx, DSPSR_B200_EINVAL, "sk: in-place masking needs equal spans");
  B200_CHECK (ctx, launch_sk (reinterpret_cast<const float2*> (d_in), in_span,
                              reinterpret_cast<float2*> (d_out), out_span, npart, nchan, npol, M,
                              zero_is_valid, Nd, lower, upper, d_sums, d_counts, d_mask,
                              reinterpret_cast<unsigned long long*> (d_zapped), ctx->stream),
              "spectral kurtosis");
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

// ---- SpectralKurtosis::Engine, step by step --------------------------------
// (CUDA::SpectralKurtosisEngine::compute / detect_ft / detect_tscr /
// reset_mask / count_mask / mask, Signal/General/SpectralKurtosisCUDA.cu:
// 45-99, with the host loops of SpectralKurtosis.C:674-798, 1012-1222,
// 1465-1566)

int dspsr_b200_sk_compute (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span,
                           uint64_t ndat, unsigned nchan, unsigned npol, unsigned M,
                           unsigned noverlap, int zero_is_valid, float* d_sums,
                           uint32_t* d_counts, uint64_t* npart_out)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (npart_out) *npart_out = 0;
  if (!d_in || !d_sums || nchan == 0 || nchan > 65535 || (npol != 1 && npol != 2))
    return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: invalid argument");
  if (noverlap == 0 || M < 2 || M % noverlap)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: noverlap=%u does not divide M=%u",
                 noverlap, M);
  if (noverlap > 1)
  {
    // Resolution::prepare (SpectralKurtosis.C:251-281): blocks of M every
    // M / noverlap samples, the first idat_start = M - M / noverlap
    // samples of the input only completing the first block
    const uint64_t stride = M / noverlap, idat_start = M - stride;
    const uint64_t npart = ndat >= idat_start ? (ndat - idat_start) / stride : 0;
    if (in_span < ndat)
      return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: span smaller than ndat");
    B200_CHECK (ctx, launch_sk_sums_strided (reinterpret_cast<const float2*> (d_in), in_span,
                                             npart, stride, nchan, npol, M, zero_is_valid,
                                             d_sums, d_counts, ctx->stream), "sk compute");
    if (npart_out) *npart_out = npart;
    return DSPSR_B200_OK;
  }
  if (M < 2 || (M & 1) || (in_span & 1) || (reinterpret_cast<uintptr_t> (d_in) & 15))
    return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: M and the span must be even, the input "
                 "16-byte aligned");
  if (M > (1u << 20) || sk_smem_bytes (npol, M, 1) > SK_SMEM_MAX)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: npol*M = %u exceeds the kernel's block",
                 npol * M);
  const uint64_t npart = ndat / M;
  if (in_span < npart * M || npart > 0x7fffffffull)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_compute: span smaller than the blocks");
  B200_CHECK (ctx, launch_sk (reinterpret_cast<const float2*> (d_in), in_span, nullptr, in_span,
                              npart, nchan, npol, M, zero_is_valid, 1, -3.4e38f, 3.4e38f, d_sums,
                              d_counts, nullptr, nullptr, ctx->stream), "sk compute");
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_detect_ft (dspsr_b200_context* ctx, const float* d_sums,
                             const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                             unsigned npol, unsigned M, unsigned Nd, float lower, float upper,
                             uint8_t* d_mask, uint64_t* d_zapped)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_sums || !d_mask || nchan == 0 || (npol != 1 && npol != 2) || Nd == 0 || M < 2)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_detect_ft: invalid argument");
  B200_CHECK (ctx, launch_sk_detect (d_sums, d_counts, npart, nchan, npol, M, Nd, lower, upper,
                                     d_mask, reinterpret_cast<unsigned long long*> (d_zapped),
                                     ctx->stream), "sk detect_ft");
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_detect_tscr (dspsr_b200_context* ctx, const float* d_sums,
                               const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                               unsigned npol, unsigned M, unsigned Nd, float std_devs,
                               uint8_t* d_mask, uint32_t* nzapped_chan)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (nzapped_chan) *nzapped_chan = 0;
  if (!d_sums || !d_mask || nchan == 0 || (npol != 1 && npol != 2) || Nd == 0 || M < 2)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_detect_tscr: invalid argument");
  if (npart == 0) return DSPSR_B200_OK;
  // the time-scrunched sums are small: they are formed on the host as the
  // reference does, in double over the float sums, then tested with the
  // limits for each channel's count (SpectralKurtosis::get_limits)
  std::vector<float> sums (npart * nchan * npol * 2);
  std::vector<uint32_t> counts (npart * nchan, M);
  B200_CHECK (ctx, cudaMemcpyAsync (sums.data (), d_sums, sums.size () * sizeof (float),
                                    cudaMemcpyDeviceToHost, ctx->stream), "sk tscr sums");
  if (d_counts)
    B200_CHECK (ctx, cudaMemcpyAsync (counts.data (), d_counts, counts.size () * sizeof (uint32_t),
                                      cudaMemcpyDeviceToHost, ctx->stream), "sk tscr counts");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sk tscr sync");
  std::map<uint64_t, std::pair<float, float>> limits;
  uint32_t nz = 0;
  for (unsigned c = 0; c < nchan; c++)
  {
    uint64_t count = 0;
    for (uint64_t ip = 0; ip < npart; ip++) count += counts[ip * nchan + c];
    if (count == 0) continue;
    auto it = limits.find (count);
    if (it == limits.end ())
    {
      float lo = 0.f, hi = 0.f;
      const unsigned mc = unsigned (std::min<uint64_t> (count, 0xffffffffull));
      if (sk_limits (mc, Nd, std_devs, npol, &lo, &hi) != 0)
        return fail (ctx, DSPSR_B200_ESTATE, "sk_detect_tscr: no limits for count=%llu",
                     (unsigned long long) count);
      it = limits.emplace (count, std::make_pair (lo, hi)).first;
    }
    const float M_t = float (count);
    // Equation (8) of Nita & Gary (2010b), as detect_tscr evaluates it
    const float M_fac = (M_t * float (Nd) + 1) / (M_t - 1);
    bool zap = false;
    for (unsigned p = 0; p < npol; p++)
    {
      double S1 = 0.0, S2 = 0.0;
      for (uint64_t ip = 0; ip < npart; ip++)
      {
        const uint64_t idx = (ip * nchan + c) * npol + p;
        S1 += sums[idx * 2];
        S2 += sums[idx * 2 + 1];
      }
      const double SK = M_fac * (M_t * (S2 / (S1 * S1)) - 1);
      if (SK > it->second.second || SK < it->second.first) zap = true;
    }
    if (zap)
    {
      nz++;
      B200_CHECK (ctx, cudaMemset2DAsync (d_mask + c, nchan, 1, 1, npart, ctx->stream),
                  "sk tscr mask");
    }
  }
  if (nzapped_chan) *nzapped_chan = nz;
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_tscrunch (dspsr_b200_context* ctx, const float* d_sums,
                            const uint32_t* d_counts, uint64_t npart_from, uint64_t npart_to,
                            unsigned nchan, unsigned npol, unsigned nsum, unsigned offset,
                            float* d_sums_out, uint32_t* d_counts_out)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_sums || !d_counts || !d_sums_out || !d_counts_out || nchan == 0 || nsum == 0
      || offset == 0 || (npol != 1 && npol != 2))
    return fail (ctx, DSPSR_B200_EINVAL, "sk_tscrunch: invalid argument");
  if (npart_to && (npart_to - 1) * offset + uint64_t (nsum - 1) * offset >= npart_from)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_tscrunch: the coarse parts reach past the fine ones");
  B200_CHECK (ctx, launch_sk_tscrunch (d_sums, d_counts, npart_to, nchan, npol, nsum, offset,
                                       d_sums_out, d_counts_out, ctx->stream), "sk tscrunch");
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_detect_skfb (dspsr_b200_context* ctx, const float* d_sums,
                               const uint32_t* d_counts, uint64_t npart, unsigned nchan,
                               unsigned npol, unsigned Nd, float std_devs, unsigned nflag,
                               unsigned flag_step, unsigned flag_offset, uint8_t* d_mask,
                               uint64_t mask_npart, uint64_t* d_zapped)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_sums || !d_counts || !d_mask || nchan == 0 || Nd == 0 || nflag == 0
      || flag_step == 0 || (npol != 1 && npol != 2))
    return fail (ctx, DSPSR_B200_EINVAL, "sk_detect_skfb: invalid argument");
  if (npart == 0) return DSPSR_B200_OK;
  if ((npart - 1) * flag_offset + uint64_t (nflag - 1) * flag_step >= mask_npart)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_detect_skfb: flags reach past the mask");
  // get_limits (SpectralKurtosis.C:988-1008) for every count present
  std::vector<uint32_t> counts (npart * nchan);
  B200_CHECK (ctx, cudaMemcpyAsync (counts.data (), d_counts, counts.size () * sizeof (uint32_t),
                                    cudaMemcpyDeviceToHost, ctx->stream), "sk counts");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sk counts");
  std::vector<uint32_t> uniq (counts);
  std::sort (uniq.begin (), uniq.end ());
  uniq.erase (std::unique (uniq.begin (), uniq.end ()), uniq.end ());
  std::vector<uint32_t> lc;
  std::vector<float2> lim;
  for (uint32_t m : uniq)
  {
    if (m <= 2) continue;
    float lo = 0.f, hi = 0.f;
    if (sk_limits (m, Nd, std_devs, npol, &lo, &hi) != 0)
      return fail (ctx, DSPSR_B200_ESTATE, "sk_detect_skfb: no limits for count %u", m);
    lc.push_back (m);
    lim.push_back (make_float2 (lo, hi));
  }
  if (lc.empty ())
  {
    lc.push_back (0);
    lim.push_back (make_float2 (0.f, 0.f));
  }
  DevBuf<uint32_t> d_lc;
  DevBuf<float2> d_lim;
  B200_CHECK (ctx, d_lc.reserve (lc.size ()), "cudaMalloc sk limits");
  B200_CHECK (ctx, d_lim.reserve (lim.size ()), "cudaMalloc sk limits");
  B200_CHECK (ctx, cudaMemcpy (d_lc.ptr, lc.data (), lc.size () * 4, cudaMemcpyHostToDevice),
              "sk limits");
  B200_CHECK (ctx, cudaMemcpy (d_lim.ptr, lim.data (), lim.size () * 8, cudaMemcpyHostToDevice),
              "sk limits");
  const cudaError_t e = launch_sk_detect_skfb (
      d_sums, d_counts, npart, nchan, npol, Nd, d_lc.ptr, d_lim.ptr, unsigned (lc.size ()), nflag,
      flag_step, flag_offset, d_mask, reinterpret_cast<unsigned long long*> (d_zapped),
      ctx->stream);
  const cudaError_t e2 = cudaStreamSynchronize (ctx->stream);
  d_lc.release ();
  d_lim.release ();
  if (e != cudaSuccess) return cuda_fail (ctx, e, "sk detect_skfb");
  if (e2 != cudaSuccess) return cuda_fail (ctx, e2, "sk detect_skfb");
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_mask_overlap (dspsr_b200_context* ctx, const uint8_t* d_mask,
                                const float* d_in, uint64_t in_span, float* d_out,
                                uint64_t out_span, unsigned nchan, unsigned npol, unsigned M,
                                unsigned offset, uint64_t npart, uint64_t nskip,
                                uint64_t idat_start)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_mask || !d_in || !d_out || d_in == d_out || nchan == 0 || offset == 0 || M == 0
      || (npol != 1 && npol != 2))
    return fail (ctx, DSPSR_B200_EINVAL, "sk_mask_overlap: invalid argument");
  if (npart == 0) return DSPSR_B200_OK;
  const uint64_t nout = (npart - 1) * offset + M;
  if (out_span < nout || in_span < idat_start + nout)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_mask_overlap: spans smaller than the blocks");
  B200_CHECK (ctx, launch_sk_mask_overlap (d_mask, reinterpret_cast<const float2*> (d_in), in_span,
                                           reinterpret_cast<float2*> (d_out), out_span, nout,
                                           nchan, npol, offset, npart, nskip, idat_start,
                                           ctx->stream), "sk mask overlap");
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_reset_mask (dspsr_b200_context* ctx, uint8_t* d_mask, uint64_t npart,
                              unsigned nchan)
{
  if (!ctx || !d_mask) return DSPSR_B200_EINVAL;
  B200_CHECK (ctx, cudaMemsetAsync (d_mask, 0, npart * nchan, ctx->stream), "sk reset mask");
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_count_mask (dspsr_b200_context* ctx, const uint8_t* d_mask, uint64_t npart,
                              unsigned nchan, uint64_t* nzapped)
{
  if (!ctx || !d_mask || !nzapped) return DSPSR_B200_EINVAL;
  std::vector<uint8_t> h (npart * nchan);
  B200_CHECK (ctx, cudaMemcpyAsync (h.data (), d_mask, h.size (), cudaMemcpyDeviceToHost,
                                    ctx->stream), "sk count mask");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sk count mask");
  uint64_t n = 0;
  for (uint8_t v : h) n += v != 0;
  *nzapped = n;
  return DSPSR_B200_OK;
}

int dspsr_b200_sk_mask (dspsr_b200_context* ctx, const uint8_t* d_mask, const float* d_in,
                        uint64_t in_span, float* d_out, uint64_t out_span, uint64_t ndat,
                        unsigned nchan, unsigned npol, unsigned M)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_mask || !d_in || !d_out || nchan == 0 || (npol != 1 && npol != 2) || M == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_mask: invalid argument");
  const uint64_t n = (ndat / M) * M;
  if (in_span < n || out_span < n)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_mask: span smaller than the blocks");
  if (d_in == d_out && in_span != out_span)
    return fail (ctx, DSPSR_B200_EINVAL, "sk_mask: in-place masking needs equal spans");
  B200_CHECK (ctx, launch_sk_mask (d_mask, reinterpret_cast<const float2*> (d_in), in_span,
                                   reinterpret_cast<float2*> (d_out), out_span, n, nchan, npol, M,
                                   ctx->stream), "sk mask");
  return DSPSR_B200_OK;
}

// ---- unpack ----------------------------------------------------------------// ---- unpack ----------------------------------------------------------------

int dspsr_b200_unpack8 (dspsr_b200_context* ctx, const void* d_in, uint64_t ndat,
                        unsigned nchan, unsigned npol, unsigned ndim, const float* lut256,
                        float* d_out, uint64_t out_span)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_in || !d_out || !lut256 || nchan == 0 || npol == 0 || ndim == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "unpack8: invalid argument");
  if (out_span < ndat * ndim)
    return fail (ctx, DSPSR_B200_EINVAL, "unpack8: out_span=%llu < ndat*ndim",
                 (unsigned long long) out_span);
  B200_CHECK (ctx, cudaMemcpyAsync (ctx->d_lut, lut256, 256 * sizeof (float),
                                    cudaMemcpyHostToDevice, ctx->stream), "upload lut");
  B200_CHECK (ctx, launch_unpack8 (static_cast<const uint8_t*> (d_in), ndat, nchan, npol, ndim,
                                   ctx->d_lut, d_out, out_span, ctx->stream), "unpack8");
  // the LUT buffer is reused by the next call: keep this call's upload ordered
  return DSPSR_B200_OK;
}

int dspsr_b200_unpack16 (dspsr_b200_context* ctx, const void* d_in, uint64_t ndat,
                         unsigned nchan, unsigned npol, unsigned ndim, int offset_binary,
                         float* d_out, uint64_t out_span)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_in || !d_out || nchan == 0 || npol == 0 || ndim == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "unpack16: invalid argument");
  if (out_span < ndat * ndim)
    return fail (ctx, DSPSR_B200_EINVAL, "unpack16: out_span too small");
  B200_CHECK (ctx, launch_unpack16 (static_cast<const int16_t*> (d_in), ndat, nchan, npol, ndim,
                                    offset_binary, d_out, out_span, ctx->stream), "unpack16");
  return DSPSR_B200_OK;
}

// ---- convolution -----------------------------------------------------------

int dspsr_b200_convolution_create (dspsr_b200_context* ctx, unsigned nchan, unsigned npol,
                                   unsigned nfft, unsigned pos, unsigned neg,
                                   dspsr_b200_convolution** out)
{
  if (!ctx || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  dspsr_b200_convolution* c = new (std::nothrow) dspsr_b200_convolution;
  if (!c) return fail (ctx, DSPSR_B200_ENOMEM, "convolution: out of host memory");
  int rc = c->init (ctx, nchan, npol, nfft, pos, neg, 0);
  if (rc)
  {
    dspsr_b200_convolution_destroy (c);
    return rc;
  }
  *out = c;
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_destroy (dspsr_b200_convolution* c)
{
  if (!c) return DSPSR_B200_EINVAL;
  if (c->ctx) cudaStreamSynchronize (c->ctx->stream);
  c->release ();
  delete c;
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_status (dspsr_b200_convolution* c)
{
  if (!c) return DSPSR_B200_EINVAL;
  return c->status ();
}

int dspsr_b200_convolution_copy_response (dspsr_b200_convolution* c, const float* response)
{
  if (!c) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = c->ctx;
  if (!response) return fail (ctx, DSPSR_B200_EINVAL, "copy_response: null response");
  const ConvShape& sh = c->shape;
  const uint64_t n = uint64_t (sh.nchan) * sh.nfft;
  B200_CHECK (ctx, c->tmp.reserve (n), "cudaMalloc response staging");
  B200_CHECK (ctx, cudaMemcpyAsync (c->tmp.ptr, response, n * sizeof (float2),
                                    cudaMemcpyHostToDevice, ctx->stream), "upload response");
  B200_CHECK (ctx, launch_permute_response (c->H.ptr, c->tmp.ptr, sh.nchan, sh.n1, sh.n2,
                                            ctx->stream), "permute response");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "copy_response sync");
  c->have_response = true;
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_set_dedispersion (dspsr_b200_convolution* c, double cf, double bw,
                                             double dm, int input_nchan, int dual_sideband,
                                             int dc_centred, int chirp_mode, unsigned norm_nfft)
{
  if (!c) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = c->ctx;
  const ConvShape& sh = c->shape;
  if (bw == 0 || !(cf > 0))
    return fail (ctx, DSPSR_B200_EINVAL, "set_dedispersion: invalid frequency/bandwidth");
  if (dc_centred && input_nchan > 1)
    return fail (ctx, DSPSR_B200_EINVAL, "set_dedispersion: DC-centred channels not supported");
  const unsigned nchan = sh.nchan;
  // Observation::get_centre_frequency(ichan) (Observation.C:521-534)
  std::vector<double> freq (nchan);
  for (unsigned ic = 0; ic < nchan; ic++)
    freq[ic] = channel_centre (cf, bw, nchan, ic, false, false);
  // Response::swap_as_needed (Response.C:325-400) for the supported states
  const int swap = (input_nchan == 1 && nchan == 1 && dual_sideband > 0)
                || (input_nchan > 1 && unsigned (input_nchan) == nchan && dual_sideband != 0);
  return build_response (c, freq.data (), bw, dm, swap, chirp_mode, norm_nfft);
}

int dspsr_b200_convolution_set_dedispersion_channels (dspsr_b200_convolution* c,
                                                      const double* chan_freq, double bw,
                                                      double dm, int chirp_mode,
                                                      unsigned norm_nfft)
{
  if (!c) return DSPSR_B200_EINVAL;
  if (!chan_freq || bw == 0)
    return fail (c->ctx, DSPSR_B200_EINVAL, "set_dedispersion_channels: invalid argument");
  for (unsigned ic = 0; ic < c->shape.nchan; ic++)
    if (!(chan_freq[ic] > 0))
      return fail (c->ctx, DSPSR_B200_EINVAL, "set_dedispersion_channels: bad frequency");
  return build_response (c, chan_freq, bw, dm, 1, chirp_mode, norm_nfft);
}

int dspsr_b200_filterbank (dspsr_b200_context* ctx, int input_kind, const void* d_in,
                           uint64_t ndat, uint64_t in_span, unsigned nchan_in, unsigned npol,
                           unsigned nsub, const float* lut256, int offset_binary, float* d_out,
                           uint64_t out_span, uint64_t* ndat_out)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (ndat_out) *ndat_out = 0;
  if (!d_in || !d_out || nchan_in == 0 || npol == 0 || npol > 2)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank: invalid argument");
  if (input_kind < 0 || input_kind > 2 || (input_kind == DSPSR_B200_INT8_TFPD && !lut256))
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank: invalid input kind or missing table");
  if (!is_pow2 (nsub) || nsub < 4 || nsub > 4096)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank: nsub=%u not a power of two in [4, 4096]",
                 nsub);
  if (nsub >= 128 && ctx->fb_tab_n != nsub)
  {
    size_t cap = ctx->fb_tab_n ? pass_tables_count (ctx->fb_tab_n) : 0;
    B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sync before table upload");
    B200_CHECK (ctx, upload_pass_tables (nsub, &ctx->d_fb_tab, &cap), "filterbank tables");
    ctx->fb_tab_n = nsub;
  }
  if (input_kind == DSPSR_B200_FLOAT_FPT && in_span < ndat)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank: in_span < ndat");
  const uint64_t nblk = ndat / nsub;
  if (out_span < nblk)
    return fail (ctx, DSPSR_B200_EINVAL, "filterbank: out_span < ndat/nsub");
  if (input_kind == DSPSR_B200_INT8_TFPD)
    B200_CHECK (ctx, cudaMemcpyAsync (ctx->d_lut, lut256, 256 * sizeof (float),
                                      cudaMemcpyHostToDevice, ctx->stream), "upload lut");
  InputView in {};
  in.kind = input_kind;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = nchan_in;
  in.npol = npol;
  in.offset_binary = offset_binary;
  const float scale = float (1.0 / std::sqrt (double (nsub)));
  B200_CHECK (ctx, launch_filterbank (in, ctx->d_lut, nsub, nblk, scale,
                                      reinterpret_cast<float2*> (d_out), out_span, ctx->stream,
                                      nullptr, ctx->d_fb_tab), "filterbank");
  if (ndat_out) *ndat_out = nblk;
  return DSPSR_B200_OK;
}

// The row FFTs in FP32 on the CUDA cores, or on the tensor cores with the
// data and DFT operands split into 2 or 3 BF16 terms.
int dspsr_b200_convolution::set_fft_precision (int mode)
{
  if (mode != DSPSR_B200_FFT_FP32 && mode != DSPSR_B200_FFT_BF16X2
      && mode != DSPSR_B200_FFT_BF16X3)
    return fail (ctx, DSPSR_B200_EINVAL, "fft precision: unknown mode %d", mode);
  if (mode == DSPSR_B200_FFT_FP32)
  {
    tc_splits = 0;
    return DSPSR_B200_OK;
  }
  if (shape.n1 < 2 || shape.n2 != 8192)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "fft precision: the tensor-core rows need nfft >= 16384 (nfft=%u)", shape.nfft);
  const unsigned ns = mode == DSPSR_B200_FFT_BF16X2 ? 2 : 3;
  std::vector<uint8_t> img;
  make_tc_dft_image (ns, img);
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "sync before DFT upload");
  B200_CHECK (ctx, tc_dft.reserve (img.size ()), "cudaMalloc DFT operands");
  B200_CHECK (ctx, cudaMemcpy (tc_dft.ptr, img.data (), img.size (), cudaMemcpyHostToDevice),
              "copy DFT operands");
  tc_splits = int (ns);
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_set_fft_precision (dspsr_b200_convolution* c, int mode)
{
  if (!c) return DSPSR_B200_EINVAL;
  return c->set_fft_precision (mode);
}

int dspsr_b200_convolution_set_temporal_apodization (dspsr_b200_convolution* c,
                                                     const float* window)
{
  if (!c) return DSPSR_B200_EINVAL;
  if (!window)
  {
    c->have_apod = false;
    return DSPSR_B200_OK;
  }
  B200_CHECK (c->ctx, cudaStreamSynchronize (c->ctx->stream), "sync before window upload");
  B200_CHECK (c->ctx, c->apod.reserve (c->shape.nfft), "cudaMalloc temporal window");
  B200_CHECK (c->ctx, cudaMemcpy (c->apod.ptr, window, c->shape.nfft * sizeof (float),
                                  cudaMemcpyHostToDevice), "copy temporal window");
  c->have_apod = true;
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_get_response (dspsr_b200_convolution* c, float* response)
{
  if (!c) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = c->ctx;
  if (!response) return fail (ctx, DSPSR_B200_EINVAL, "get_response: null pointer");
  const ConvShape& sh = c->shape;
  const uint64_t n = uint64_t (sh.nchan) * sh.nfft;
  B200_CHECK (ctx, c->tmp.reserve (n), "cudaMalloc response staging");
  B200_CHECK (ctx, launch_unpermute_response (c->tmp.ptr, c->H.ptr, sh.nchan, sh.n1, sh.n2,
                                              ctx->stream), "unpermute response");
  B200_CHECK (ctx, cudaMemcpyAsync (response, c->tmp.ptr, n * sizeof (float2),
                                    cudaMemcpyDeviceToHost, ctx->stream), "download response");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "get_response sync");
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_perform (dspsr_b200_convolution* c, const float* d_in,
                                    uint64_t in_span, uint64_t ndat, float* d_out,
                                    uint64_t out_span, uint64_t* npart_out)
{
  if (!c) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = c->ctx;
  const ConvShape& sh = c->shape;
  if (npart_out) *npart_out = 0;
  if (!c->have_response) return fail (ctx, DSPSR_B200_ESTATE, "perform: no response set");
  if (!d_in || !d_out) return fail (ctx, DSPSR_B200_EINVAL, "perform: null pointer");
  if (in_span < ndat) return fail (ctx, DSPSR_B200_EINVAL, "perform: in_span < ndat");
  uint64_t npart = 0;
  const uint64_t nfilt = uint64_t (sh.nfilt_pos) + sh.nfilt_neg;
  if (ndat >= sh.nfft) npart = (ndat - nfilt) / sh.nkeep;
  if (out_span < npart * sh.nkeep)
    return fail (ctx, DSPSR_B200_EINVAL, "perform: out_span=%llu < npart*nkeep=%llu",
                 (unsigned long long) out_span, (unsigned long long) (npart * sh.nkeep));
  InputView in {};
  in.kind = IN_FLOAT;
  in.pre = nullptr;
  in.main = d_in;
  in.npre = 0;
  in.main_span = in_span;
  in.nchan = sh.nchan;
  in.npol = sh.npol;
  FoldView fv {};
  VoltView vv {reinterpret_cast<float2*> (d_out), out_span};
  const ConvTables tb = c->tables ();
  for (uint64_t p0 = 0; p0 < npart; p0 += c->max_batch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (c->max_batch, npart - p0));
    B200_CHECK (ctx, launch_convolution (sh, tb, in, p0, nb, c->scratch.ptr, OUT_VOLTAGE, fv, vv,
                                         ctx->stream), "convolution kernels");
  }
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}

int dspsr_b200_convolution_perform_zero_dm (dspsr_b200_convolution* c, const float* d_in,
                                            uint64_t in_span, uint64_t ndat, float* d_out,
                                            uint64_t out_span, float* d_zero_dm,
                                            uint64_t zero_dm_span, uint64_t* npart_out)
{
  if (!c) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = c->ctx;
  if (!d_zero_dm) return fail (ctx, DSPSR_B200_EINVAL, "perform_zero_dm: null zero-DM output");
  uint64_t npart = 0;
  const int rc = dspsr_b200_convolution_perform (c, d_in, in_span, ndat, d_out, out_span, &npart);
  if (npart_out) *npart_out = npart;
  if (rc) return rc;
  const ConvShape& sh = c->shape;
  const uint64_t n = npart * sh.nkeep;
  if (zero_dm_span < n)
    return fail (ctx, DSPSR_B200_EINVAL, "perform_zero_dm: zero_dm_span < npart*nkeep");
  if (n)
    // Convolution.C:789-796: the input samples aligned with the output
    B200_CHECK (ctx, cudaMemcpy2DAsync (d_zero_dm, zero_dm_span * sizeof (float2),
                                        d_in + 2 * uint64_t (sh.nfilt_pos),
                                        in_span * sizeof (float2), n * sizeof (float2),
                                        uint64_t (sh.nchan) * sh.npol, cudaMemcpyDeviceToDevice,
                                        ctx->stream), "zero-DM copy");
  return DSPSR_B200_OK;
}

// ---- detection -------------------------------------------------------------

int dspsr_b200_detect (dspsr_b200_context* ctx, const float* d_in, uint64_t in_span,
                       uint64_t ndat, unsigned nchan, int state, float* d_out, uint64_t out_span)
{
  if (!ctx) return DSPSR_B200_EINVAL;
  if (!d_in || !d_out || nchan == 0) return fail (ctx, DSPSR_B200_EINVAL, "detect: invalid argument");
  if (state < 0 || state > 3) return fail (ctx, DSPSR_B200_EINVAL, "detect: invalid state %d", state);
  if (in_span < ndat || out_span < ndat)
    return fail (ctx, DSPSR_B200_EINVAL, "detect: span smaller than ndat");
  B200_CHECK (ctx, launch_detect (reinterpret_cast<const float2*> (d_in), in_span, ndat, nchan,
                                  state, d_out, out_span, ctx->stream), "detect");
  return DSPSR_B200_OK;
}

// ---- fold --------------------------------------------------------------------

int dspsr_b200_fold_create (dspsr_b200_context* ctx, unsigned nbin, unsigned nchan,
                            unsigned npol, dspsr_b200_fold** out)
{
  if (!ctx || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  dspsr_b200_fold* f = new (std::nothrow) dspsr_b200_fold;
  if (!f) return fail (ctx, DSPSR_B200_ENOMEM, "fold: out of host memory");
  int rc = f->init (ctx, nbin, nchan, npol);
  if (rc)
  {
    f->release ();
    delete f;
    return rc;
  }
  // engines that fold many channels from one plan (the filterbank with a
  // response) read each sample's column once per block instead of searching
  // the plan in every channel
  f->use_cols = true;
  *out = f;
  return DSPSR_B200_OK;
}

int dspsr_b200_fold_destroy (dspsr_b200_fold* f)
{
  if (!f) return DSPSR_B200_EINVAL;
  if (f->ctx) cudaStreamSynchronize (f->ctx->stream);
  f->release ();
  delete f;
  return DSPSR_B200_OK;
}

int dspsr_b200_fold_set_bins (dspsr_b200_fold* f, double phi, double pps, uint64_t ndat,
                              uint64_t idat_start, uint64_t* ndat_folded)
{
  if (!f) return DSPSR_B200_EINVAL;
  (void) idat_start;   // the plan is relative to the first folded sample
  int rc = f->set_bins (phi, pps, ndat);
  if (rc) return rc;
  if (ndat_folded) *ndat_folded = ndat;
  return DSPSR_B200_OK;
}

int dspsr_b200_fold_fold (dspsr_b200_fold* f, const float* d_in, uint64_t in_span)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (!d_in) return fail (ctx, DSPSR_B200_EINVAL, "fold: null input");
  if (in_span < f->ndat) return fail (ctx, DSPSR_B200_EINVAL, "fold: in_span < ndat");
  FoldView fv = f->view (0, 1, f->nchan);
  B200_CHECK (ctx, launch_fold (d_in, in_span, f->ndat, f->nchan, f->npol, fv, ctx->stream),
              "fold");
  return f->release_plan ();
}

int dspsr_b200_fold_binplan (dspsr_b200_fold* f, uint32_t* d_binplan)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (!d_binplan) return fail (ctx, DSPSR_B200_EINVAL, "binplan: null output");
  B200_CHECK (ctx, launch_binplan (f->d_segs[f->cur].ptr, f->nseg, f->ndat, f->nbin, d_binplan,
                                   ctx->stream), "binplan");
  return f->release_plan ();
}

int dspsr_b200_fold_get_profiles (dspsr_b200_fold* f, float* profiles, uint32_t* hits)
{
  if (!f) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = f->ctx;
  if (profiles)
    B200_CHECK (ctx, cudaMemcpyAsync (profiles, f->profiles.ptr,
                                      uint64_t (f->nchan) * f->npol * f->nbin * sizeof (float),
                                      cudaMemcpyDeviceToHost, ctx->stream), "download profiles");
  if (hits)
    B200_CHECK (ctx, cudaMemcpyAsync (hits, f->hits.ptr, f->nbin * sizeof (unsigned),
                                      cudaMemcpyDeviceToHost, ctx->stream), "download hits");
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "get_profiles sync");
  return DSPSR_B200_OK;
}

int dspsr_b200_fold_reset (dspsr_b200_fold* f)
{
  if (!f) return DSPSR_B200_EINVAL;
  return f->reset ();
}

// ---- pipeline ----------------------------------------------------------------

int dspsr_b200_pipeline_create (dspsr_b200_context* ctx, const dspsr_b200_pipeline_config* cfg,
                                dspsr_b200_pipeline** out)
{
  if (!ctx || !cfg || !out) return DSPSR_B200_EINVAL;
  *out = nullptr;
  if (cfg->input_kind < 0 || cfg->input_kind > 2)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: invalid input_kind %d", cfg->input_kind);
  if (cfg->state < 0 || cfg->state > 3)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: invalid state %d", cfg->state);
  if (cfg->npol == 1 && cfg->state != DSPSR_B200_INTENSITY)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: state %d needs two polarisations", cfg->state);
  if (!(cfg->period_s > 0) || cfg->nbin == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: folding period and nbin must be positive");
  if (cfg->nchan == 0 || cfg->bandwidth_mhz == 0)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline: invalid nchan/bandwidth");
  dspsr_b200_pipeline* pl = new (std::nothrow) dspsr_b200_pipeline;
  if (!pl) return fail (ctx, DSPSR_B200_ENOMEM, "pipeline: out of host memory");
  pl->ctx = ctx;
  pl->cfg = *cfg;
  pl->nout = detect_nout (cfg->state);
  const uint64_t bytes_per_value = cfg->input_kind == DSPSR_B200_INT16_TFPD ? 2 : 1;
  pl->bytes_per_sample = uint64_t (cfg->nchan) * cfg->npol * 2 * bytes_per_value;
  const unsigned fb = cfg->filterbank_nchan > 1 ? cfg->filterbank_nchan : 0;
  if (fb && (!is_pow2 (fb) || fb < 4 || fb > 4096))
  {
    delete pl;
    return fail (ctx, DSPSR_B200_EINVAL,
                 "pipeline: filterbank_nchan=%u not a power of two in [4, 4096]", fb);
  }
  pl->fb_nsub = fb;
  if (fb >= 128 && upload_pass_tables (fb, &pl->fb_tab, &pl->fb_tab_cap) != cudaSuccess)
  {
    delete pl;
    return fail (ctx, DSPSR_B200_ECUDA, "pipeline: filterbank tables");
  }
  // channels the convolution sees
  const unsigned nchan = fb ? cfg->nchan * fb : cfg->nchan;
  pl->rate = std::fabs (cfg->bandwidth_mhz) / double (nchan) * 1e6;
  int rc = pl->conv.init (ctx, nchan, cfg->npol, cfg->nfft, cfg->nfilt_pos, cfg->nfilt_neg,
                          cfg->scratch_bytes, cfg->row_length);
  if (!rc && cfg->fft_precision != DSPSR_B200_FFT_FP32)
    rc = pl->conv.set_fft_precision (cfg->fft_precision);
  if (!rc && cfg->interchannel)
  {
    // DedispersionPipe::construct_interchan (DedispersionPipe.C:435-470): the
    // response takes each channel's fractional delay (Dedispersion::build,
    // Dedispersion.C:84-97 with build_setup :141-162), SampleDelay the whole
    // samples; channel centres as Observation::get_centre_frequency gives them
    std::vector<double> freq (nchan), frac (nchan);
    for (unsigned ic = 0; ic < nchan; ic++)
      freq[ic] = fb ? channel_centre (cfg->centre_freq_mhz, cfg->bandwidth_mhz, nchan, ic,
                                      cfg->dual_sideband != 0, true)
                    : channel_centre (cfg->centre_freq_mhz, cfg->bandwidth_mhz, nchan, ic,
                                      false, false);
    interchannel_delays (cfg->centre_freq_mhz, cfg->dm, pl->rate, freq.data (), nchan, &pl->sd);
    bool ok = nchan > 1 && !(cfg->dc_centred && !fb);
    std::vector<int> applied (nchan);
    for (unsigned ic = 0; ic < nchan && ok; ic++)
    {
      ok = pl->sd.applied[ic] >= 0 && uint64_t (pl->sd.applied[ic]) <= pl->sd.total_delay;
      applied[ic] = int (pl->sd.applied[ic]);
      frac[ic] = pl->sd.frac[ic] / (cfg->bandwidth_mhz / double (nchan));   // microseconds
    }
    if (!ok)
      rc = fail (ctx, DSPSR_B200_EINVAL,
                 "pipeline: inter-channel dedispersion needs several channels whose delays "
                 "lie within the span SampleDelay buffers");
    else
    {
      const int swap = fb ? 1 : cfg->dual_sideband != 0;
      rc = build_response (&pl->conv, freq.data (), cfg->bandwidth_mhz, cfg->dm, swap,
                           cfg->chirp_mode, cfg->nfft, frac.data ());
    }
    if (!rc)
    {
      cudaError_t e = pl->sd_applied.reserve (nchan);
      if (e == cudaSuccess)
        e = cudaMemcpy (pl->sd_applied.ptr, applied.data (), nchan * sizeof (int),
                        cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = cuda_fail (ctx, e, "upload delays");
    }
    pl->sd_on = !rc;
  }
  else if (!rc && !fb)
    rc = dspsr_b200_convolution_set_dedispersion (&pl->conv, cfg->centre_freq_mhz,
                                                  cfg->bandwidth_mhz, cfg->dm, cfg->nchan,
                                                  cfg->dual_sideband, cfg->dc_centred,
                                                  cfg->chirp_mode, cfg->nfft);
  else if (!rc)
  {
    // Filterbank::prepare_output (Filterbank.C:352-381) with freq_res = 1: the
    // output channels are DC-centred and, for dual-sideband input, swapped
    std::vector<double> freq (nchan);
    for (unsigned ic = 0; ic < nchan; ic++)
      freq[ic] = channel_centre (cfg->centre_freq_mhz, cfg->bandwidth_mhz, nchan, ic,
                                 cfg->dual_sideband != 0, true);
    rc = dspsr_b200_convolution_set_dedispersion_channels (&pl->conv, freq.data (),
                                                           cfg->bandwidth_mhz, cfg->dm,
                                                           cfg->chirp_mode, cfg->nfft);
  }
  if (!rc && cfg->input_kind == DSPSR_B200_INT8_TFPD)
  {
    cudaError_t e = cudaMemcpy (pl->conv.lut.ptr, cfg->lut, 256 * sizeof (float),
                                cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cuda_fail (ctx, e, "upload lut");
    pl->lut_scale = affine_lut_scale (cfg->lut);
  }
  // sub-integrations: Subint<Fold>::prepare hands the divider the folding
  // period for divisions in turns (Subint.h:230-242)
  if (!rc && (cfg->subint_seconds != 0 || cfg->subint_turns != 0))
  {
    if (cfg->subint_seconds < 0 || cfg->subint_turns < 0
        || (cfg->subint_seconds > 0 && cfg->subint_turns > 0))
      rc = fail (ctx, DSPSR_B200_EINVAL,
                 "pipeline: subint_seconds=%g, subint_turns=%g: give one positive length",
                 cfg->subint_seconds, cfg->subint_turns);
    else
    {
      pl->sub_on = true;
      b200::TimeDivide& d = pl->planner_init.divider;
      d.division_seconds = cfg->subint_seconds;
      d.division_turns = cfg->subint_turns;
      d.period = cfg->period_s;
      d.reference_epoch.day = cfg->subint_epoch_day;
      d.reference_epoch.sec = cfg->subint_epoch_sec;
      d.reference_epoch.frac = cfg->subint_epoch_frac;
      pl->planner = pl->planner_init;
      pl->sub_slots.resize (cfg->subint_slots ? cfg->subint_slots : 4);
    }
  }
  if (!rc) rc = pl->fold.init (ctx, cfg->nbin, nchan, pl->nout,
                               pl->sub_on ? unsigned (pl->sub_slots.size ()) : 1);
  pl->fold.use_cols = true;
  // C2's shape -- a 64-channel filterbank of one dual-polarisation int8 or
  // int16 channel with four-step parts of 8 x n2 -- runs the filterbank
  // inside the forward column pass: its output never goes through memory
  pl->fb_fused = !rc && fb == 64 && cfg->nchan == 1 && cfg->npol == 2
                 && cfg->input_kind != DSPSR_B200_FLOAT_FPT && pl->conv.shape.n1 == 8
                 && cfg->fused_filterbank >= 0 && cfg->sk_M == 0;
  // SpectralKurtosis between the convolution and detection: its zero-DM
  // input needs the filterbank's channels in memory
  if (!rc && cfg->sk_M)
  {
    if (cfg->sk_M < 4 || (cfg->sk_M & 1) || sk_smem_bytes (cfg->npol, cfg->sk_M, 1) > SK_SMEM_MAX)
      rc = fail (ctx, DSPSR_B200_EINVAL, "pipeline: sk_M=%u must be even, >= 4 and fit the "
                 "SK kernel's block", cfg->sk_M);
    else if (cfg->interchannel)
      rc = fail (ctx, DSPSR_B200_EINVAL, "pipeline: SpectralKurtosis with inter-channel "
                 "dedispersion is not supported");
    else
    {
      const float sd = cfg->sk_std_devs > 0.f ? cfg->sk_std_devs : 3.f;
      if (sk_limits (cfg->sk_M, 1, sd, cfg->npol, &pl->sk_lower, &pl->sk_upper) != 0)
        rc = fail (ctx, DSPSR_B200_EINVAL, "pipeline: no SK limits for M=%u", cfg->sk_M);
      else if (pl->sk_zapped.reserve (1) != cudaSuccess
               || cudaMemset (pl->sk_zapped.ptr, 0, sizeof (unsigned long long)) != cudaSuccess)
        rc = fail (ctx, DSPSR_B200_ECUDA, "pipeline: sk counter");
      else
      {
        pl->sk_on = true;
        pl->sk_M = cfg->sk_M;
      }
    }
  }
  // the carry never exceeds nfft samples: size both carry buffers once
  for (int i = 0; i < 2 && !rc; i++)
  {
    const bool fpt = !pl->fb_fused && (fb || cfg->input_kind == DSPSR_B200_FLOAT_FPT);
    const uint64_t bytes = fpt ? uint64_t (nchan) * cfg->npol * cfg->nfft * sizeof (float2)
                               : uint64_t (cfg->nfft) * pl->bytes_per_sample
                                     * (pl->fb_fused ? fb : 1);
    cudaError_t e = pl->carry[i].reserve (bytes);
    if (e != cudaSuccess) rc = cuda_fail (ctx, e, "cudaMalloc carry");
  }
  if (rc)
  {
    dspsr_b200_pipeline_destroy (pl);
    return rc;
  }
  *out = pl;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_destroy (dspsr_b200_pipeline* pl)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (pl->ctx) cudaStreamSynchronize (pl->ctx->stream);
  pl->conv.release ();
  pl->fold.release ();
  pl->carry[0].release ();
  pl->carry[1].release ();
  pl->staging[0].release ();
  pl->staging[1].release ();
  if (pl->fb_tab) cudaFree (pl->fb_tab);
  if (pl->copy_stream) cudaStreamSynchronize (pl->copy_stream);
  for (int i = 0; i < 2; i++)
  {
    if (pl->copied[i]) cudaEventDestroy (pl->copied[i]);
    if (pl->consumed[i]) cudaEventDestroy (pl->consumed[i]);
  }
  if (pl->copy_stream) cudaStreamDestroy (pl->copy_stream);
  for (int i = 0; i < 2; i++)
  {
    if (pl->pinned[i]) cudaFreeHost (pl->pinned[i]);
    if (pl->host_free[i]) cudaEventDestroy (pl->host_free[i]);
  }
  if (pl->snap_ev) cudaEventDestroy (pl->snap_ev);
  if (pl->snap_err) cudaFreeHost (pl->snap_err);
  for (auto& u : pl->sub_pending) pl->sub_spare.push_back (u);   // undelivered: dropped
  for (auto& u : pl->sub_spare)
  {
    if (u.prof) cudaFreeHost (u.prof);
    if (u.hits) cudaFreeHost (u.hits);
    if (u.ev) cudaEventDestroy (u.ev);
  }
  pl->fbbuf.release ();
  pl->sd_applied.release ();
  pl->sd_buf[0].release ();
  pl->sd_buf[1].release ();
  for (int i = 0; i < 2; i++)
  {
    pl->sk_v[i].release ();
    pl->sk_z[i].release ();
  }
  pl->sk_mask.release ();
  pl->sk_zapped.release ();
  pl->sk_sums.release ();
  pl->sk_counts.release ();
  pl->sk_pmask.release ();
  delete pl;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_run (dspsr_b200_pipeline* pl, const void* d_in, uint64_t ndat,
                             uint64_t in_span, uint64_t* ndat_folded)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (!d_in && ndat) return fail (pl->ctx, DSPSR_B200_EINVAL, "pipeline_run: null input");
  if (pl->cfg.input_kind == DSPSR_B200_FLOAT_FPT && in_span < ndat)
    return fail (pl->ctx, DSPSR_B200_EINVAL, "pipeline_run: in_span < ndat");
  return pipeline_input (pl, d_in, ndat, in_span, ndat_folded);
}

int dspsr_b200_pipeline_run_host (dspsr_b200_pipeline* pl, const void* h_in, uint64_t ndat,
                                  uint64_t* ndat_folded)
{
  if (!pl) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = pl->ctx;
  if (pl->cfg.input_kind == DSPSR_B200_FLOAT_FPT)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline_run_host: TFPD input only");
  if (!h_in && ndat) return fail (ctx, DSPSR_B200_EINVAL, "pipeline_run_host: null input");
  if (ndat_folded) *ndat_folded = 0;
  if (!pl->copy_stream)
  {
    B200_CHECK (ctx, cudaStreamCreateWithFlags (&pl->copy_stream, cudaStreamNonBlocking),
                "create upload stream");
    for (int i = 0; i < 2; i++)
    {
      B200_CHECK (ctx, cudaEventCreateWithFlags (&pl->copied[i], cudaEventDisableTiming),
                  "create event");
      B200_CHECK (ctx, cudaEventCreateWithFlags (&pl->consumed[i], cudaEventDisableTiming),
                  "create event");
    }
  }
  // The block is uploaded in up to eight pieces on a stream of its own, each
  // into one of two staging buffers, so that the upload of a piece overlaps
  // the kernels of the one before; the carried overlap joins the pieces as it
  // joins blocks.  Pieces are whole filterbank transforms.
  const uint64_t unit = pl->fb_nsub ? pl->fb_nsub : 1;
  const uint64_t min_piece = uint64_t (pl->conv.shape.nfft) * unit * 2;
  // (sub-integrations divide each block as a whole: no pieces)
  const uint64_t npiece = pl->sub_on ? 1
                        : ndat >= 8 * min_piece ? 8
                        : ndat >= 4 * min_piece ? 4
                        : ndat >= 2 * min_piece ? 2 : 1;
  const uint64_t piece = ((ndat + npiece - 1) / npiece + unit - 1) / unit * unit;
  const uint64_t bps = pl->bytes_per_sample;
  uint64_t total = 0;
  // one block: its pieces share one fold phase recurrence
  struct PieceScope
  {
    dspsr_b200_pipeline* p;
    explicit PieceScope (dspsr_b200_pipeline* q) : p (q) { p->in_pieces = true; p->phase_continue = false; }
    ~PieceScope () { p->in_pieces = false; p->phase_continue = false; }
  } scope (pl);
  // the pieces' fold plans follow the pieces on the copy stream
  struct PlanStream
  {
    dspsr_b200_fold* f;
    PlanStream (dspsr_b200_fold* g, cudaStream_t s) : f (g) { f->up = s; }
    ~PlanStream () { f->up = nullptr; }
  } plan_stream (&pl->fold, pl->copy_stream);
  for (uint64_t j = 0, off = 0; off < ndat || (ndat == 0 && j == 0); j++, off += piece)
  {
    const uint64_t n = std::min<uint64_t> (piece, ndat - off);
    const int b = int (j & 1);
    if (pl->consumed_pending[b])
      B200_CHECK (ctx, cudaStreamWaitEvent (pl->copy_stream, pl->consumed[b], 0), "wait staging");
    B200_CHECK (ctx, pl->staging[b].reserve (std::max<uint64_t> (piece * bps, 16)),
                "cudaMalloc staging");
    B200_CHECK (ctx, cudaMemcpyAsync (pl->staging[b].ptr, static_cast<const uint8_t*> (h_in) + off * bps,
                                      n * bps, cudaMemcpyHostToDevice, pl->copy_stream),
                "upload block");
    B200_CHECK (ctx, cudaEventRecord (pl->copied[b], pl->copy_stream), "record upload");
    B200_CHECK (ctx, cudaStreamWaitEvent (ctx->stream, pl->copied[b], 0), "wait upload");
    uint64_t folded = 0;
    const int rc = pipeline_input (pl, pl->staging[b].ptr, n, 0, &folded);
    if (rc) return rc;
    total += folded;
    B200_CHECK (ctx, cudaEventRecord (pl->consumed[b], ctx->stream), "record consumed");
    pl->consumed_pending[b] = true;
    if (ndat == 0) break;
  }
  if (ndat_folded) *ndat_folded = total;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_run_dada (dspsr_b200_pipeline* pl, dspsr_b200_dada_file* file,
                                  uint64_t start_sample, uint64_t nsamp, uint64_t block_ndat,
                                  uint64_t* ndat_read, uint64_t* ndat_folded)
{
  if (!pl) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = pl->ctx;
  if (ndat_read) *ndat_read = 0;
  if (ndat_folded) *ndat_folded = 0;
  if (!file) return fail (ctx, DSPSR_B200_EINVAL, "pipeline_run_dada: null file");
  const dspsr_b200_dada_info& info = dspsr_b200_host::dada_info (file);
  const auto& cfg = pl->cfg;
  const unsigned nbit = cfg.input_kind == DSPSR_B200_INT8_TFPD ? 8
                      : cfg.input_kind == DSPSR_B200_INT16_TFPD ? 16 : 0;
  if (!nbit)
    return fail (ctx, DSPSR_B200_EINVAL, "pipeline_run_dada: TFPD input only");
  // GenericEightBitUnpacker::matches / the 16-bit unpacker: complex TFPD of
  // the pipeline's shape
  if (info.nchan != cfg.nchan || info.npol != cfg.npol || info.ndim != 2 || info.nbit != nbit)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "pipeline_run_dada: file has NCHAN=%u NPOL=%u NDIM=%u NBIT=%u, the pipeline "
                 "takes NCHAN=%u NPOL=%u NDIM=2 NBIT=%u", info.nchan, info.npol, info.ndim,
                 info.nbit, cfg.nchan, cfg.npol, nbit);
  const uint64_t unit = pl->fb_nsub ? pl->fb_nsub : 1;
  if (block_ndat == 0 || block_ndat % unit)
    return fail (ctx, DSPSR_B200_EINVAL,
                 "pipeline_run_dada: block_ndat=%llu must be a positive multiple of %llu",
                 (unsigned long long) block_ndat, (unsigned long long) unit);
  const uint64_t end = std::min (info.ndat, info.file_ndat);
  const uint64_t avail = start_sample < end ? end - start_sample : 0;
  uint64_t total = nsamp ? std::min (nsamp, avail) : avail;
  total -= total % unit;

  const uint64_t bytes = block_ndat * pl->bytes_per_sample;
  if (pl->pinned_bytes < bytes)
  {
    for (int i = 0; i < 2; i++)
    {
      if (pl->host_free_pending[i])
        B200_CHECK (ctx, cudaEventSynchronize (pl->host_free[i]), "wait upload");
      pl->host_free_pending[i] = false;
      if (pl->pinned[i]) cudaFreeHost (pl->pinned[i]);
      pl->pinned[i] = nullptr;
    }
    pl->pinned_bytes = 0;
    for (int i = 0; i < 2; i++)
      B200_CHECK (ctx, cudaHostAlloc (&pl->pinned[i], bytes, cudaHostAllocDefault),
                  "cudaHostAlloc file block");
    pl->pinned_bytes = bytes;
  }
  for (int i = 0; i < 2; i++)
    if (!pl->host_free[i])
      B200_CHECK (ctx, cudaEventCreateWithFlags (&pl->host_free[i], cudaEventDisableTiming),
                  "create event");

  // File::load_bytes into one buffer while the other block's upload and
  // kernels run (the reference's File::load_bytes_device,
  // File.C:280-339, uploads one pinned block at a time)
  uint64_t done = 0, folded = 0;
  int b = 0;
  while (done < total)
  {
    const uint64_t n = std::min (block_ndat, total - done);
    if (pl->host_free_pending[b])
      B200_CHECK (ctx, cudaEventSynchronize (pl->host_free[b]), "wait upload");
    pl->host_free_pending[b] = false;
    uint64_t got = 0;
    int rc = dspsr_b200_dada_read (file, start_sample + done, n, pl->pinned[b], &got);
    if (rc) return fail (ctx, rc, "pipeline_run_dada: %s", dspsr_b200_host_error ());
    if (got != n)
      return fail (ctx, DSPSR_B200_ESTATE, "pipeline_run_dada: read %llu of %llu samples",
                   (unsigned long long) got, (unsigned long long) n);
    uint64_t f = 0;
    rc = dspsr_b200_pipeline_run_host (pl, pl->pinned[b], n, &f);
    if (rc) return rc;
    B200_CHECK (ctx, cudaEventRecord (pl->host_free[b], pl->copy_stream), "record upload");
    pl->host_free_pending[b] = true;
    folded += f;
    done += n;
    b ^= 1;
  }
  if (ndat_read) *ndat_read = done;
  if (ndat_folded) *ndat_folded = folded;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_get_profiles (dspsr_b200_pipeline* pl, float* profiles, uint32_t* hits)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (pl->sub_on)
    return fail (pl->ctx, DSPSR_B200_ESTATE,
                 "pipeline_get_profiles: the pipeline folds sub-integrations; take them with "
                 "pop_subint or an unloader");
  int rc = dspsr_b200_fold_get_profiles (&pl->fold, profiles, hits);
  if (rc) return rc;
  return pl->conv.status ();
}

int dspsr_b200_pipeline_get_profiles_async (dspsr_b200_pipeline* pl, float* profiles,
                                            uint32_t* hits)
{
  if (!pl) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = pl->ctx;
  if (pl->sub_on)
    return fail (ctx, DSPSR_B200_ESTATE,
                 "pipeline_get_profiles_async: the pipeline folds sub-integrations; take them "
                 "with pop_subint or an unloader");
  if (!profiles && !hits) return fail (ctx, DSPSR_B200_EINVAL, "get_profiles_async: no buffer");
  dspsr_b200_fold& f = pl->fold;
  if (!pl->snap_ev)
    B200_CHECK (ctx, cudaEventCreateWithFlags (&pl->snap_ev, cudaEventDisableTiming),
                "cudaEventCreate");
  if (!pl->snap_err)
  {
    B200_CHECK (ctx, cudaHostAlloc (&pl->snap_err, sizeof (int), cudaHostAllocDefault),
                "cudaHostAlloc status");
    *pl->snap_err = 0;
  }
  if (pl->conv.err.ptr)
    B200_CHECK (ctx, cudaMemcpyAsync (pl->snap_err, pl->conv.err.ptr, sizeof (int),
                                      cudaMemcpyDeviceToHost, ctx->stream), "read device status");
  if (profiles)
    B200_CHECK (ctx, cudaMemcpyAsync (profiles, f.profiles.ptr,
                                      uint64_t (f.nchan) * f.npol * f.nbin * sizeof (float),
                                      cudaMemcpyDeviceToHost, ctx->stream), "download profiles");
  if (hits)
    B200_CHECK (ctx, cudaMemcpyAsync (hits, f.hits.ptr, f.nbin * sizeof (unsigned),
                                      cudaMemcpyDeviceToHost, ctx->stream), "download hits");
  B200_CHECK (ctx, cudaEventRecord (pl->snap_ev, ctx->stream), "record snapshot");
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_wait_profiles (dspsr_b200_pipeline* pl)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (pl->snap_ev)
    B200_CHECK (pl->ctx, cudaEventSynchronize (pl->snap_ev), "wait snapshot");
  if (pl->snap_err && *pl->snap_err)
    return fail (pl->ctx, DSPSR_B200_ESTATE, "a device-side wait timed out");
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_set_unloader (dspsr_b200_pipeline* pl, dspsr_b200_unload_fn fn,
                                      void* user)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (pl->sub_on && pl->unload_fn)
  {
    const int rc = subint_drain (pl, true);   // the old unloader takes what it started
    if (rc) return rc;
  }
  pl->unload_fn = fn;
  pl->unload_user = user;
  return pl->sub_on ? subint_drain (pl, true) : DSPSR_B200_OK;
}

int dspsr_b200_pipeline_subints_ready (dspsr_b200_pipeline* pl, uint64_t* n)
{
  if (!pl || !n) return DSPSR_B200_EINVAL;
  *n = pl->sub_ready.size ();
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_pop_subint (dspsr_b200_pipeline* pl, dspsr_b200_subint* subint,
                                    float* profiles, uint32_t* hits)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (!pl->sub_on)
    return fail (pl->ctx, DSPSR_B200_ESTATE, "pop_subint: no sub-integrations configured");
  if (pl->sub_ready.empty ())
    return fail (pl->ctx, DSPSR_B200_ESTATE, "pop_subint: no closed sub-integration");
  const int k = pl->sub_ready.front ();
  pl->sub_ready.pop_front ();
  return subint_take (pl, k, subint, profiles, hits);
}

int dspsr_b200_pipeline_finish (dspsr_b200_pipeline* pl)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (!pl->sub_on) return DSPSR_B200_OK;
  subint_close (pl);
  return subint_drain (pl, true);
}

int dspsr_b200_pipeline_reset (dspsr_b200_pipeline* pl)
{
  if (!pl) return DSPSR_B200_EINVAL;
  pl->ncarry = 0;
  pl->in0 = 0;
  pl->sd_ncarry = 0;
  pl->sd_out0 = 0;
  pl->sk_ncarry = 0;
  pl->sk_out0 = 0;
  if (pl->sub_on)
  {
    const int rc = subint_drain (pl, true);      // unloads already started complete
    if (rc) return rc;
    pl->planner = pl->planner_init;
    for (auto& sl : pl->sub_slots) sl.used = false;
    pl->sub_cur = -1;
    pl->sub_ready.clear ();
  }
  return pl->fold.reset ();
}

int dspsr_b200_pipeline_profile (dspsr_b200_pipeline* pl, int enable)
{
  if (!pl) return DSPSR_B200_EINVAL;
  B200_CHECK (pl->ctx, cudaStreamSynchronize (pl->ctx->stream), "pipeline_profile sync");
  pl->clock.clear ();
  pl->clock.on = enable != 0;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_kernel_times (dspsr_b200_pipeline* pl, double* ms, uint64_t* launches)
{
  if (!pl || !ms || !launches) return DSPSR_B200_EINVAL;
  dspsr_b200_context* ctx = pl->ctx;
  B200_CHECK (ctx, cudaStreamSynchronize (ctx->stream), "kernel_times sync");
  for (int k = 0; k < KK_COUNT; k++)
  {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  for (size_t i = 0; i < pl->clock.kind.size (); i++)
  {
    float t = 0.f;
    B200_CHECK (ctx, cudaEventElapsedTime (&t, pl->clock.pool[2 * i], pl->clock.pool[2 * i + 1]),
                "cudaEventElapsedTime");
    ms[pl->clock.kind[i]] += t;
    launches[pl->clock.kind[i]]++;
  }
  pl->clock.clear ();
  return DSPSR_B200_OK;
}

uint64_t dspsr_b200_kernel_launches (void) { return kernel_launches (); }

int dspsr_b200_pipeline_set_rfi_proposer (dspsr_b200_pipeline* pl,
                                          dspsr_b200_rfi_proposer* proposer, float confidence)
{
  if (!pl) return DSPSR_B200_EINVAL;
  if (!proposer)
  {
    pl->sk_proposer = nullptr;
    return DSPSR_B200_OK;
  }
  if (!pl->sk_on)
    return fail (pl->ctx, DSPSR_B200_ESTATE, "pipeline: the proposer needs the SK stage (sk_M)");
  if (confidence < 0.5f || confidence > 1.f)
    return fail (pl->ctx, DSPSR_B200_EINVAL, "pipeline: confidence %g outside [0.5, 1]",
                 double (confidence));
  dspsr_b200_context* pctx = nullptr;
  unsigned pnchan = 0, pM = 0;
  rfi_proposer_shape (proposer, &pctx, &pnchan, &pM);
  if (pctx != pl->ctx || pnchan != pl->conv.shape.nchan || pM != pl->sk_M)
    return fail (pl->ctx, DSPSR_B200_EINVAL,
                 "pipeline: the proposer (%u channels, blocks of %u%s) does not match the "
                 "pipeline (%u channels, sk_M %u, its own context)", pnchan, pM,
                 pctx != pl->ctx ? ", another context" : "", pl->conv.shape.nchan, pl->sk_M);
  pl->sk_proposer = proposer;
  pl->sk_confidence = confidence;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_sk_counts (dspsr_b200_pipeline* pl, uint64_t* zapped, uint64_t* tested)
{
  if (!pl || !zapped || !tested) return DSPSR_B200_EINVAL;
  *zapped = *tested = 0;
  if (!pl->sk_on) return DSPSR_B200_OK;
  unsigned long long h = 0;
  B200_CHECK (pl->ctx, cudaMemcpyAsync (&h, pl->sk_zapped.ptr, sizeof (h), cudaMemcpyDeviceToHost,
                                        pl->ctx->stream), "sk count");
  B200_CHECK (pl->ctx, cudaStreamSynchronize (pl->ctx->stream), "sk count");
  *zapped = h;
  *tested = pl->sk_tested;
  return DSPSR_B200_OK;
}

int dspsr_b200_pipeline_info (dspsr_b200_pipeline* pl, uint64_t* info)
{
  if (!pl || !info) return DSPSR_B200_EINVAL;
  const ConvShape& sh = pl->conv.shape;
  info[0] = sh.nfft;
  info[1] = sh.nkeep;
  info[2] = sh.n1;
  info[3] = sh.n2;
  info[4] = pl->conv.max_batch;
  info[5] = pl->ncarry;
  info[6] = pl->in0;
  info[7] = uint64_t (pl->fold.nseg);
  return DSPSR_B200_OK;
}

} // extern "C"
