// noalloc.cu -- an overlap-save convolution entry point that allocates no
// memory at all.
//
// Who needs it: callers that must not call cudaMalloc while they run --
// real-time processes that fix every allocation at start-up to keep their
// latency flat, and hosts whose device memory belongs to another allocator (a
// framework's caching pool, an embedding application) that does not let this
// library allocate behind its back.  dspsr_b200_convolution_perform needs an
// engine object whose creation allocates its tables and scratch; this entry
// point instead keeps everything it needs in one fixed array in device memory
// that the library owns from load time.
//
// The array: g_noalloc_scratch below, DSPSR_B200_NOALLOC_SCRATCH_BYTES
// (32 MiB) of static device memory.  Every GPU that loads the library holds it
// until the process exits.  Its device address is taken with
// cudaGetSymbolAddress once per device, together with the kernels' shared-
// memory opt-in, by the first call made with that device current (whatever
// its shape, even one with no whole part), so that first call should come
// before any stream capture.  Every call on a device reuses the same array and
// leaves its contents behind, so calls whose work overlaps on the GPU (two
// streams, two threads) race with each other; serialise them.

#include "dspsr_b200.h"
#include "kernels.cuh"
#include "fft_core.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

using namespace b200;

namespace {

constexpr uint64_t SCRATCH_BYTES = DSPSR_B200_NOALLOC_SCRATCH_BYTES;

// The one static scratch array.  Host code must never hand the symbol itself
// to a kernel: on the host it names a stand-in object, not device memory.
__device__ __align__ (256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[MAX_DEVICES] = {};
int g_nsm[MAX_DEVICES] = {};

constexpr uint64_t align256 (uint64_t x) { return (x + 255) & ~uint64_t (255); }

// Twiddle tables rounded once from double precision, written on the device.
__global__ void k_tw2 (float2* tw2, unsigned n)
{
  const unsigned m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double s, c;
  sincospi (-2.0 * double (m) / double (n), &s, &c);
  tw2[m] = make_float2 (float (c), float (s));
}

__global__ void k_tw4 (float2* tw4, unsigned n1, unsigned n2)
{
  const uint64_t idx = uint64_t (blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t N = uint64_t (n1) * n2;
  if (idx >= N) return;
  const uint64_t k1 = idx / n2, i = idx % n2;
  const uint64_t m = (k1 * i) % N;
  double s, c;
  sincospi (-2.0 * double (m) / double (N), &s, &c);
  tw4[idx] = make_float2 (float (c), float (s));
}

// Device address of the static array for the current device (set-up once per
// device: cudaGetSymbolAddress, checked), plus its multiprocessor count.
cudaError_t scratch_for_device (void** ptr, int* nsm)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice (&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock (g_setup_mutex);
  if (!g_scratch_ptr[dev])
  {
    void* p = nullptr;
    e = cudaGetSymbolAddress (&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaDeviceGetAttribute (&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_nsm[dev] = n;
    g_scratch_ptr[dev] = p;
  }
  *ptr = g_scratch_ptr[dev];
  *nsm = g_nsm[dev];
  return cudaSuccess;
}

} // namespace

extern "C" int dspsr_b200_convolution_perform_noalloc (
    void* stream, const float* d_in, uint64_t in_span, uint64_t ndat, unsigned nchan,
    unsigned npol, unsigned nfft, unsigned nfilt_pos, unsigned nfilt_neg,
    const float* d_response, float* d_out, uint64_t out_span, uint64_t* npart_out,
    int* d_status)
{
  if (npart_out) *npart_out = 0;
  if (!d_in || !d_out || !d_response || nchan == 0 || npol == 0 || npol > 2)
    return DSPSR_B200_EINVAL;
  if (nfft < 4096 || nfft > 262144 || (nfft & (nfft - 1)))
    return DSPSR_B200_EINVAL;
  if (uint64_t (nfilt_pos) + nfilt_neg >= nfft || in_span < ndat) return DSPSR_B200_EINVAL;

  // per-device set-up first, whatever the shape: the array's address, the
  // multiprocessor count and the kernels' shared-memory opt-in
  void* base = nullptr;
  int nsm = 0;
  if (scratch_for_device (&base, &nsm) != cudaSuccess) return DSPSR_B200_ECUDA;
  if (convolution_kernel_setup () != cudaSuccess) return DSPSR_B200_ECUDA;

  ConvShape sh {};
  sh.nchan = nchan;
  sh.npol = npol;
  sh.nfft = nfft;
  sh.nfilt_pos = nfilt_pos;
  sh.nfilt_neg = nfilt_neg;
  sh.nkeep = nfft - nfilt_pos - nfilt_neg;
  sh.n1 = nfft <= 8192 ? 1 : nfft / 8192;
  sh.n2 = nfft <= 8192 ? nfft : 8192;

  uint64_t npart = 0;
  if (ndat >= nfft) npart = (ndat - nfilt_pos - nfilt_neg) / sh.nkeep;
  if (out_span < npart * sh.nkeep) return DSPSR_B200_EINVAL;

  // layout of the static array: status flag, n2-point table, then (four-step
  // only) the [n1][n2] twiddles, the response in four-step order and the FFT
  // scratch of as many parts as fit
  const uint64_t off_tw2 = 256;
  const uint64_t off_tw4 = off_tw2 + align256 (uint64_t (sh.n2) * sizeof (float2));
  uint64_t off_H = off_tw4, off_scratch = off_tw4;
  uint64_t nbatch = 65535;
  if (sh.n1 > 1)
  {
    off_H = off_tw4 + align256 (uint64_t (nfft) * sizeof (float2));
    off_scratch = off_H + align256 (uint64_t (nchan) * nfft * sizeof (float2));
    const uint64_t per_part = uint64_t (nchan) * npol * nfft * sizeof (float2);
    if (off_scratch + per_part > SCRATCH_BYTES) return DSPSR_B200_ETOOBIG;
    // as many parts as fit, reduced (down to half) to a batch whose rows
    // spread evenly over the persistent row kernel's CTAs
    const uint64_t bmax = std::min<uint64_t> (65535, (SCRATCH_BYTES - off_scratch) / per_part);
    const uint64_t rows_per_part = uint64_t (sh.n1) * nchan * npol;
    nbatch = bmax;
    for (uint64_t b = bmax; b >= std::max<uint64_t> (1, bmax / 2); b--)
      if ((b * rows_per_part) % (uint64_t (nsm) * rows_ctas_per_sm (sh.n2)) == 0)
      {
        nbatch = b;
        break;
      }
  }

  cudaStream_t st = static_cast<cudaStream_t> (stream);
  unsigned char* b = static_cast<unsigned char*> (base);
  // the status word: the caller's int when given, else a word of the array;
  // either way it starts every call at zero, and the FP32 kernels this call
  // runs have no device-side waits that could set it
  int* err = d_status ? d_status : reinterpret_cast<int*> (b);
  if (cudaMemsetAsync (err, 0, sizeof (int), st) != cudaSuccess) return DSPSR_B200_ECUDA;
  if (npart == 0) return DSPSR_B200_OK;

  float2* tw2 = reinterpret_cast<float2*> (b + off_tw2);
  float2* tw4 = reinterpret_cast<float2*> (b + off_tw4);
  float2* H = reinterpret_cast<float2*> (b + off_H);
  float2* scratch = reinterpret_cast<float2*> (b + off_scratch);

  // the tables are rewritten for this shape
  k_tw2<<<(sh.n2 + 255) / 256, 256, 0, st>>> (tw2, sh.n2);
  ConvTables tb {};
  tb.tw2 = tw2;
  tb.err = err;
  tb.nsm = nsm;
  tb.lut = nullptr;
  if (sh.n1 > 1)
  {
    k_tw4<<<unsigned ((uint64_t (nfft) + 255) / 256), 256, 0, st>>> (tw4, sh.n1, sh.n2);
    if (launch_permute_response (H, reinterpret_cast<const float2*> (d_response), nchan, sh.n1,
                                 sh.n2, st) != cudaSuccess)
      return DSPSR_B200_ECUDA;
    tb.tw4 = tw4;
    tb.H = H;
  }
  else
    tb.H = reinterpret_cast<const float2*> (d_response);   // FFT order is the kernel's order
  if (cudaGetLastError () != cudaSuccess) return DSPSR_B200_ECUDA;

  InputView in {};
  in.kind = IN_FLOAT;
  in.main = d_in;
  in.main_span = in_span;
  in.nchan = nchan;
  in.npol = npol;
  FoldView fv {};
  VoltView vv {reinterpret_cast<float2*> (d_out), out_span};
  for (uint64_t p0 = 0; p0 < npart; p0 += nbatch)
  {
    const unsigned nb = unsigned (std::min<uint64_t> (nbatch, npart - p0));
    if (launch_convolution (sh, tb, in, p0, nb, scratch, OUT_VOLTAGE, fv, vv, st) != cudaSuccess)
      return DSPSR_B200_ECUDA;
  }
  if (npart_out) *npart_out = npart;
  return DSPSR_B200_OK;
}
