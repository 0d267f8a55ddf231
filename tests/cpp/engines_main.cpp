// engines_main.cpp -- drives the C++ engine classes the way DSPSR's operations
// call their engines (unpack -> convolve -> detect -> fold, and the filterbank
// with a response) and checks them against closed forms: a unit response returns the kept input scaled by
// sqrt(nfft) (the Convolution normaliser of Convolution.C:401-414 left out),
// detection of constant data, and fold bins equal to the reference's
// sequential recurrence (Fold.C:815-818) run here on the host.
#include "dsp_b200_engines.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
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

    // dsp::Unpacker: the 8-bit class equals unpack8; the 16-bit class gives
    // float(x) + 0.5 with offset binary undone (SixteenBitUnpacker.C:54-79)
    {
      b200::Unpacker u8 (ctx, b200::Unpacker::EightBit), u16 (ctx, b200::Unpacker::SixteenBit);
      CHECK (u8.matches (8) && !u8.matches (16) && u16.matches (16), "Unpacker::matches");
      u8.set_table (lut);
      b200::TimeSeriesView y8 = x;
      y8.base = d_y;
      u8.unpack (d_raw, y8);
      std::vector<float> a (ndat * npol * 2), b (ndat * npol * 2);
      ctx.synchronize ();
      cudaMemcpy (a.data (), d_x, a.size () * 4, cudaMemcpyDeviceToHost);
      cudaMemcpy (b.data (), d_y, b.size () * 4, cudaMemcpyDeviceToHost);
      CHECK (a == b, "8-bit Unpacker differs from unpack8");
      const uint64_t n16 = 1000;
      std::vector<uint16_t> w (n16 * 2 * 2);
      for (size_t i = 0; i < w.size (); i++) w[i] = uint16_t (i * 2654435761u);
      void* d_w = nullptr;
      float* d_f = nullptr;
      cudaMalloc (&d_w, w.size () * 2);
      cudaMalloc (&d_f, n16 * 2 * 2 * 4);
      cudaMemcpy (d_w, w.data (), w.size () * 2, cudaMemcpyHostToDevice);
      b200::TimeSeriesView f;
      f.base = d_f;
      f.span_floats = n16 * 2;
      f.ndat = n16;
      f.nchan = 1;
      f.npol = 2;
      u16.set_offset_binary (true);
      u16.unpack (d_w, f);
      std::vector<float> hf (n16 * 2 * 2);
      ctx.synchronize ();
      cudaMemcpy (hf.data (), d_f, hf.size () * 4, cudaMemcpyDeviceToHost);
      for (uint64_t t = 0; t < n16; t++)
        for (unsigned p = 0; p < 2; p++)
          for (unsigned d = 0; d < 2; d++)
          {
            const int16_t v = int16_t (w[(t * 2 + p) * 2 + d] ^ 0x8000);
            CHECK (hf[p * n16 * 2 + t * 2 + d] == float (v) + 0.5f, "16-bit value at %llu",
                   (unsigned long long) t);
          }
      cudaFree (d_w);
      cudaFree (d_f);
    }

    // SpectralKurtosis engine steps: an outlying block is zapped by
    // detect_ft and zeroed by mask; the rest passes unchanged
    {
      const unsigned sc = 4, sp = 2, M = 256;
      const uint64_t sn = 16 * M;
      std::vector<float> v (uint64_t (sc) * sp * sn * 2);
      uint64_t state = 12345;
      auto gauss = [&state] () {
        double u = 0;
        for (int k = 0; k < 12; k++)
        {
          state = state * 6364136223846793005ull + 1442695040888963407ull;
          u += double (state >> 11) / double (1ull << 53);
        }
        return float (u - 6.0);
      };
      for (auto& e : v) e = gauss ();
      // channel 2, block 5: a few huge samples (impulsive RFI)
      for (unsigned p = 0; p < sp; p++)
        for (uint64_t t = 5 * M; t < 5 * M + 8; t++) v[((2 * sp + p) * sn + t) * 2] = 300.f;
      float *d_v = nullptr, *d_o = nullptr, *d_s = nullptr;
      uint32_t* d_c = nullptr;
      uint8_t* d_m = nullptr;
      const uint64_t npart = sn / M;
      cudaMalloc (&d_v, v.size () * 4);
      cudaMalloc (&d_o, v.size () * 4);
      cudaMalloc (&d_s, npart * sc * sp * 2 * 4);
      cudaMalloc (&d_c, npart * sc * 4);
      cudaMalloc (&d_m, npart * sc);
      cudaMemcpy (d_v, v.data (), v.size () * 4, cudaMemcpyHostToDevice);
      b200::TimeSeriesView in;
      in.base = d_v;
      in.span_floats = sn * 2;
      in.ndat = sn;
      in.nchan = sc;
      in.npol = sp;
      b200::TimeSeriesView out = in;
      out.base = d_o;
      b200::SpectralKurtosisEngine sk (ctx);
      sk.setup (1);
      b200::SKSums sums;
      sums.sums = d_s;
      sums.counts = d_c;
      CHECK (sk.compute (in, sums, M) == npart, "SK compute npart");
      float lo = 0, hi = 0;
      ctx.check (dspsr_b200_sk_limits (M, 1, 3.f, sp, &lo, &hi), "sk limits");
      sk.reset_mask (d_m, npart, sc);
      sk.detect_ft (sums, d_m, hi, lo);
      const uint64_t nz = sk.count_mask (d_m, npart, sc);
      std::vector<uint8_t> hm (npart * sc);
      cudaMemcpy (hm.data (), d_m, hm.size (), cudaMemcpyDeviceToHost);
      CHECK (hm[5 * sc + 2] == 1, "SK missed the outlying block");
      CHECK (nz >= 1 && nz <= 4, "SK zapped %llu cells", (unsigned long long) nz);
      sk.mask (d_m, in, out, M);
      std::vector<float> ho (v.size ());
      ctx.synchronize ();
      cudaMemcpy (ho.data (), d_o, ho.size () * 4, cudaMemcpyDeviceToHost);
      for (unsigned c = 0; c < sc; c++)
        for (unsigned p = 0; p < sp; p++)
          for (uint64_t t = 0; t < sn; t++)
          {
            const uint64_t i = ((c * sp + p) * sn + t) * 2;
            const bool z = hm[(t / M) * sc + c] != 0;
            CHECK (z ? (ho[i] == 0.f && ho[i + 1] == 0.f) : (ho[i] == v[i] && ho[i + 1] == v[i + 1]),
                   "SK mask at chan %u sample %llu", c, (unsigned long long) t);
          }
      cudaFree (d_v);
      cudaFree (d_o);
      cudaFree (d_s);
      cudaFree (d_c);
      cudaFree (d_m);
    }

    // InverseFilterbank engine: a tone channelised exactly (fine channel c
    // holds wideband bins c*keep + s, s signed, channel 0 on DC) comes back
    // as L times the tone (256 channels of 64 points, 4/3 oversampled:
    // 48 kept bins, L = 12288)
    {
      const unsigned inch = 256, lin = 64, keep = 48, L = inch * keep, f0 = 1000;
      std::vector<float> xin (uint64_t (inch) * lin * 2, 0.f);
      for (unsigned c = 0; c < inch; c++)
        for (int s = -int (lin) / 2; s < int (lin) / 2; s++)
          if ((int64_t (c) * keep + s + L) % L == f0)
            for (unsigned m = 0; m < lin; m++)
            {
              const double a = 2 * M_PI * double (s) * m / lin;
              xin[(uint64_t (c) * lin + m) * 2] += float (double (L) / lin * std::cos (a));
              xin[(uint64_t (c) * lin + m) * 2 + 1] += float (double (L) / lin * std::sin (a));
            }
      dspsr_b200_ifb_config cfg {};
      cfg.input_nchan = inch;
      cfg.output_nchan = 1;
      cfg.pfb_nchan = inch;
      cfg.npol = 1;
      cfg.input_fft_length = lin;
      cfg.os_num = 4;
      cfg.os_den = 3;
      cfg.pfb_dc_chan = 1;
      cfg.pfb_all_chan = 1;
      cfg.dual_sideband = 1;
      b200::InverseFilterbankEngine ifb (ctx);
      ifb.setup (cfg);
      const std::vector<uint64_t> info = ifb.info ();
      CHECK (info[0] == keep && info[1] == L, "IFB kept %llu Lout %llu",
             (unsigned long long) info[0], (unsigned long long) info[1]);
      float *d_i = nullptr, *d_o = nullptr;
      cudaMalloc (&d_i, xin.size () * 4);
      cudaMalloc (&d_o, uint64_t (L) * 2 * 4);
      cudaMemcpy (d_i, xin.data (), xin.size () * 4, cudaMemcpyHostToDevice);
      b200::TimeSeriesView in;
      in.base = d_i;
      in.span_floats = lin * 2;
      in.ndat = lin;
      in.nchan = inch;
      in.npol = 1;
      b200::TimeSeriesView out;
      out.base = d_o;
      out.span_floats = uint64_t (L) * 2;
      out.nchan = 1;
      out.npol = 1;
      CHECK (ifb.perform (in, out) == 1 && out.ndat == L, "IFB npart / ndat");
      std::vector<float> ho (uint64_t (L) * 2);
      ctx.synchronize ();
      cudaMemcpy (ho.data (), d_o, ho.size () * 4, cudaMemcpyDeviceToHost);
      double e2 = 0, r2 = 0;
      for (unsigned n = 0; n < L; n++)
      {
        const double a = 2 * M_PI * double ((uint64_t (f0) * n) % L) / L;
        const double re = double (L) * std::cos (a), im = double (L) * std::sin (a);
        e2 += (ho[2 * n] - re) * (ho[2 * n] - re) + (ho[2 * n + 1] - im) * (ho[2 * n + 1] - im);
        r2 += re * re + im * im;
      }
      CHECK (std::sqrt (e2 / r2) < 1e-5, "IFB tone rel err %g", std::sqrt (e2 / r2));
      cudaFree (d_i);
      cudaFree (d_o);
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
