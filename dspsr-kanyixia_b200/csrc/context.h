// context.h -- the library context (one device, one stream, the last error
// message), shared by the translation units that implement the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

struct dspsr_b200_context
{
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  float* d_lut = nullptr;     // scratch LUT for the standalone unpacker
  float2* d_fb_tab = nullptr; // pass tables of the standalone filterbank's FFT
  unsigned fb_tab_n = 0;      // ... for this transform length
};

struct dspsr_b200_rfi_proposer;

namespace b200 {
// the context, channels per block and block length a proposer was made for
void rfi_proposer_shape (const dspsr_b200_rfi_proposer* proposer, dspsr_b200_context** ctx,
                         unsigned* nchan, unsigned* M);
} // namespace b200
