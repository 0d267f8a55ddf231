// engines_main.cpp -- drives the C++ engine classes the way DSPSR's operations
// call their engines (unpack -> convolve -> detect -> fold, and the filterbank
// with a response) and checks them against closed forms: a unit response returns the kept input scaled by
// sqrt(nfft) (the Convolution normaliser of Convolution.C:401-414 left out),
// detection of constant data, and fold bins equal to the reference's
// sequential recurrence (Fold.C:815-818) run here on the host.
#include "dsp_b200_engines.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define CHECK(cond, ...)                       \
  do {                                         \
    if (!(cond))                               \
    {                                          \
      std::printf ("FAIL: " __VA_ARGS__);      \
      std::printf ("\n");                      \
      return 1;                                \
    }                                          \
  } while (0)

int main ()
{
  try
  {
    b200::Context ctx (0, nullptr);
    const unsigned nchan = 1, npol = 2, nfft = 8192, pos = 1000, neg = 700;
    const unsigned nkeep = nfft - pos - neg;
    const uint64_t ndat = nfft + 3 * nkeep;
    // int8 TFPD input: a ramp of byte values
    std::vector<unsigned char> raw (ndat * npol * 2);
    for (size_t i = 0; i < raw.size (); i++) raw[i] = (unsigned char) ((i * 37 + 11) & 0xff);
    float lut[256];
    double scale = 0;
    ctx.check (dspsr_b200_bittable8 (0.0308, 1, lut, &scale), "bittable8");

    void* d_raw = nullptr;
    float *d_x = nullptr, *d_y = nullptr, *d_det = nullptr;
    cudaMalloc (&d_raw, raw.size ());
    cudaMalloc (&d_x, ndat * npol * 2 * sizeof (float));
    cudaMalloc (&d_y, ndat * npol * 2 * sizeof (float));
    cudaMalloc (&d_det, ndat * sizeof (float));
    cudaMemcpy (d_raw, raw.data (), raw.size (), cudaMemcpyHostToDevice);

    // GenericEightBitUnpacker::unpack_on_gpu
    b200::TimeSeriesView x;
    x.base = d_x;
    x.span_floats = ndat * 2;
    x.ndat = ndat;
    x.nchan = nchan;
    x.npol = npol;
    b200::unpack8 (ctx, d_raw, lut, x);

    // Convolution with a unit response: output = kept input * sqrt(nfft)
    b200::ConvolutionEngine conv (ctx);
    conv.prepare (nchan, npol, nfft, pos, neg);
    std::vector<float> unit (nchan * nfft * 2, 0.f);
    for (unsigned k = 0; k < nchan * nfft; k++) unit[2 * k] = 1.0f;
    conv.copy_response (unit.data ());
    b200::TimeSeriesView y = x;
    y.base = d_y;
    // npart = (ndat - nfilt) / nkeep (Convolution.C:486-487) = (nfft + 3 nkeep - nfilt) / nkeep
    const uint64_t npart = conv.perform (x, y);
    CHECK (npart == 4, "npart=%llu", (unsigned long long) npart);
    std::vector<float> hx (ndat * npol * 2), hy (ndat * npol * 2);
    ctx.synchronize ();
    cudaMemcpy (hx.data (), d_x, hx.size () * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy (hy.data (), d_y, hy.size () * 4, cudaMemcpyDeviceToHost);
    double err = 0, ref = 0;
    for (unsigned p = 0; p < npol; p++)
      for (uint64_t j = 0; j < npart * nkeep * 2; j++)
      {
        const double a = hy[p * ndat * 2 + j] / double (nfft);
        const double b = hx[p * ndat * 2 + pos * 2 + j];
        err += (a - b) * (a - b);
        ref += b * b;
      }
    CHECK (std::sqrt (err / ref) < 1e-6, "unit-response passthrough rel err %g",
           std::sqrt (err / ref));

    // Detection::square_law on the unpacked input
    b200::DetectionEngine det (ctx);
    b200::TimeSeriesView d;
    d.base = d_det;
    d.span_floats = ndat;
    d.ndat = ndat;
    d.nchan = nchan;
    d.npol = 1;
    d.ndim = 1;
    det.square_law (x, d);
    std::vector<float> hd (ndat);
    ctx.synchronize ();
    cudaMemcpy (hd.data (), d_det, ndat * 4, cudaMemcpyDeviceToHost);
    for (uint64_t t = 0; t < ndat; t++)
    {
      float v = hx[2 * t] * hx[2 * t];
      v += hx[2 * t + 1] * hx[2 * t + 1];
      v += hx[ndat * 2 + 2 * t] * hx[ndat * 2 + 2 * t];
      v += hx[ndat * 2 + 2 * t + 1] * hx[ndat * 2 + 2 * t + 1];
      CHECK (v == hd[t], "square_law mismatch at %llu", (unsigned long long) t);
    }

    // Fold::Engine with use_set_bins
    b200::FoldEngine fold (ctx);
    const unsigned nbin = 128;
    fold.set_nbin (nbin);
    fold.setup (nchan, 1);
    const double phi = -0.123, pps = 1.0 / 777.7;
    fold.set_ndat (ndat, 0);
    CHECK (fold.set_bins (phi, pps, ndat, 0) == ndat, "set_bins");
    fold.fold (d);
    std::vector<float> prof;
    std::vector<uint32_t> hits;
    fold.synch (prof, hits);
    std::vector<double> rprof (nbin, 0.0);
    std::vector<uint32_t> rhits (nbin, 0);
    double ph = phi;
    for (uint64_t t = 0; t < ndat; t++)
    {
      ph -= std::floor (ph);
      const unsigned ibin = unsigned (ph * double (nbin));
      ph += pps;
      rhits[ibin]++;
      rprof[ibin] += hd[t];
    }
    for (unsigned b = 0; b < nbin; b++)
    {
      CHECK (hits[b] == rhits[b], "hits[%u] %u != %u", b, hits[b], rhits[b]);
      CHECK (std::fabs (prof[b] - rprof[b]) <= 1e-5 * std::fabs (rprof[b]) + 1e-3,
             "profile[%u] %g != %g", b, prof[b], rprof[b]);
    }
    CHECK (fold.get_bin_hits (3) == rhits[3], "get_bin_hits");

    // Filterbank::Engine with a unit response (normaliser 1/sqrt(N F)): a
    // complex exponential at big-FFT bin k0 = c0*F + f0 comes out of output
    // channel c0 as sqrt(nsub) exp(2 pi i f0 t / F) and nowhere else
    {
      const unsigned fsub = 16, fres = 1024, nbig = fsub * fres, c0 = 5, f0 = 37;
      const uint64_t nd = 3 * uint64_t (nbig);
      std::vector<float> hxin (nd * 2);
      for (uint64_t t = 0; t < nd; t++)
      {
        const double a = 2 * M_PI * double ((uint64_t (c0) * fres + f0) * t % nbig) / nbig;
        hxin[2 * t] = float (std::cos (a));
        hxin[2 * t + 1] = float (std::sin (a));
      }
      float *d_in = nullptr, *d_out = nullptr;
      cudaMalloc (&d_in, nd * 2 * sizeof (float));
      cudaMalloc (&d_out, uint64_t (fsub) * nd * 2 * sizeof (float));
      cudaMemcpy (d_in, hxin.data (), nd * 2 * sizeof (float), cudaMemcpyHostToDevice);
      b200::FilterbankDuringEngine fb (ctx);
      fb.setup (1, 1, fsub, fres, 0, 0);
      std::vector<float> resp (uint64_t (fsub) * fres * 2, 0.f);
      const float norm = float (1.0 / std::sqrt (double (nbig) * fres));
      for (uint64_t k = 0; k < uint64_t (fsub) * fres; k++) resp[2 * k] = norm;
      fb.copy_response (resp.data ());
      b200::TimeSeriesView in;
      in.base = d_in;
      in.span_floats = nd * 2;
      in.ndat = nd;
      in.nchan = 1;
      in.npol = 1;
      b200::TimeSeriesView out = in;
      out.base = d_out;
      out.nchan = fsub;
      const uint64_t np = fb.perform (in, out);
      CHECK (np == 3 && out.ndat == 3 * uint64_t (fres), "filterbank during npart=%llu",
             (unsigned long long) np);
      std::vector<float> ho (uint64_t (fsub) * nd * 2);
      ctx.synchronize ();
      cudaMemcpy (ho.data (), d_out, ho.size () * 4, cudaMemcpyDeviceToHost);
      double e2 = 0, r2 = 0, leak = 0;
      const double amp = std::sqrt (double (fsub));
      for (unsigned c = 0; c < fsub; c++)
        for (uint64_t t = 0; t < out.ndat; t++)
        {
          const double re = ho[(c * nd + t) * 2], im = ho[(c * nd + t) * 2 + 1];
          if (c != c0)
          {
            leak += re * re + im * im;
            continue;
          }
          const double a = 2 * M_PI * double ((f0 * (t % fres)) % fres) / fres;
          e2 += (re - amp * std::cos (a)) * (re - amp * std::cos (a))
                + (im - amp * std::sin (a)) * (im - amp * std::sin (a));
          r2 += amp * amp;
        }
      CHECK (std::sqrt (e2 / r2) < 1e-5, "filterbank during tone rel err %g", std::sqrt (e2 / r2));
      CHECK (std::sqrt (leak / r2) < 1e-5, "filterbank during leakage %g", std::sqrt (leak / r2));
      cudaFree (d_in);
      cudaFree (d_out);
    }

    cudaFree (d_raw);
    cudaFree (d_x);
    cudaFree (d_y);
    cudaFree (d_det);
    std::printf ("ALL OK\n");
    return 0;
  }
  catch (b200::Error& e)
  {
    std::printf ("FAIL: b200::Error %d %s\n", e.code, e.what ());
    return 2;
  }
}
