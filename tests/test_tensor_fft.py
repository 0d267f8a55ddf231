"""The convolution's row FFTs on the tensor cores (k_rows_mma: DFT16/DFT32
stages as tcgen05 GEMMs with split-BF16 operands) against the FP64 oracle,
through the C ABI.  The reference runs these transforms through cuFFT
(Signal/General/ConvolutionCUDA.cu:370-413); its FP32 CPU path is the
oracle (Convolution.C:724-803)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# three BF16 terms (six products): the voltage bar of the FP32 path
VOLTAGE_RTOL_BF16X3 = 2e-6
# two BF16 terms (three products): about 16 significant bits per stage; the
# measured error of the whole convolution is near 1e-5, bounded here at 3e-5
VOLTAGE_RTOL_BF16X2 = 3e-5
PROFILE_RTOL = 1e-5


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("mode,rtol", [(3, VOLTAGE_RTOL_BF16X3), (2, VOLTAGE_RTOL_BF16X2)])
@pytest.mark.parametrize("nchan,nfft,dm,bw", [(1, 1 << 17, 67.99, 16.0), (4, 1 << 15, 30.0, 64.0),
                                              (2, 1 << 14, 8.0, 32.0)])
def test_tensor_rows_voltages_vs_fp64(ctx, b2, orc, mode, rtol, nchan, nfft, dm, bw):
    rng = np.random.default_rng(nfft + nchan + mode)
    pos = orc.smearing_samples(1400.0, bw, dm, nchan, 1)
    neg = orc.smearing_samples(1400.0, bw, dm, nchan, -1)
    nk = nfft - pos - neg
    ndat = nfft + 3 * nk + 11
    x = (np.round(rng.standard_normal((nchan, 2, ndat)) * 10)
         + 1j * np.round(rng.standard_normal((nchan, 2, ndat)) * 10)).astype(np.complex64)
    h64 = orc.dedispersion_response_f64(1400.0, bw, dm, nchan, nfft, input_nchan=nchan)
    ref = orc.convolve(x.astype(np.complex128), h64, nfft, pos, neg)
    c = b2.Convolution(ctx, nchan, 2, nfft, pos, neg)
    c.set_dedispersion(1400.0, bw, dm, chirp_mode=b2.CHIRP_FP64)
    c.set_fft_precision(mode)
    out = torch.zeros((nchan, 2, 4 * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(dev(x), ndat, ndat, out, 4 * nk) == 4
    ctx.synchronize()
    c.status()
    got = out.cpu().numpy()
    err = rel_rms(got, ref)
    # and the FP32 row kernel on the same input: both near the FP64 answer
    c.set_fft_precision(b2.FFT_FP32)
    out32 = torch.zeros_like(out)
    c.perform(dev(x), ndat, ndat, out32, 4 * nk)
    ctx.synchronize()
    err32 = rel_rms(out32.cpu().numpy(), ref)
    print(f"\nvoltage error vs FP64: nfft={nfft} nchan={nchan} DM={dm}: "
          f"bf16x{mode} {err:.3e}, fp32 {err32:.3e}")
    assert err < rtol, err
    assert err32 < VOLTAGE_RTOL_BF16X3
    c.close()


def test_tensor_rows_c2_shape_vs_fp64(ctx, b2, orc):
    """C2's shape: 64-channel filterbank of 256 MHz, each channel dedispersed
    at DM 500 with 2^16-point FFTs, the rows on the tensor cores (three BF16
    terms): <= 2e-6 relative RMS against the all-FP64 chain."""
    cf, bw, dm, nsub, nfft = 1400.0, 256.0, 500.0, 64, 1 << 16
    pos = orc.smearing_samples(cf, bw, dm, nsub, 1)
    neg = orc.smearing_samples(cf, bw, dm, nsub, -1)
    nk = nfft - pos - neg
    nch = nfft + nk + 5
    ndat = nch * nsub
    rng = np.random.default_rng(64)
    raw = np.clip(np.round(rng.standard_normal(ndat * 4) * 12), -128, 127).astype(np.int8)
    raw = raw.view(np.uint8)
    lut = np.asarray(b2.bittable8()[0], np.float32)
    fbo = torch.zeros((nsub, 2, nch), dtype=torch.complex64, device="cuda")
    assert ctx.filterbank(b2.INT8_TFPD, dev(raw), ndat, 1, 2, nsub, fbo, nch, lut=lut) == nch
    freqs = orc.channel_centres(cf, bw, nsub, swap=True, dc_centred=True)
    c = b2.Convolution(ctx, nsub, 2, nfft, pos, neg)
    c.set_dedispersion_channels(freqs, bw, dm, chirp_mode=b2.CHIRP_FP64)
    c.set_fft_precision(b2.FFT_BF16X3)
    out = torch.zeros((nsub, 2, 2 * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(fbo, nch, nch, out, 2 * nk) == 2
    ctx.synchronize()
    c.status()
    got = out.cpu().numpy()
    c.close()
    x = orc.unpack8(raw, ndat, 1, 2, 2, lut).view(np.complex64).reshape(1, 2, ndat)
    y = orc.filterbank(x.astype(np.complex128), nsub)
    h = orc.dedispersion_response_channels(freqs, bw, dm, nfft, fp64=True)
    ref = orc.convolve(y, h, nfft, pos, neg)
    err = rel_rms(got, ref)
    print(f"\nvoltage error vs FP64 at C2's shape (64 x 2^16, DM 500): bf16x3 {err:.3e}")
    assert err < VOLTAGE_RTOL_BF16X3, err


def test_tensor_rows_rejects_small_ffts(ctx, b2):
    c = b2.Convolution(ctx, 1, 2, 8192, 100, 100)
    with pytest.raises(b2.B200Error):
        c.set_fft_precision(b2.FFT_BF16X3)
    with pytest.raises(b2.B200Error):
        c.set_fft_precision(7)
    c.set_fft_precision(b2.FFT_FP32)
    c.close()


@pytest.mark.parametrize("mode", [3, 2])
def test_tensor_rows_pipeline_profiles(ctx, b2, orc, mode):
    """The fused pipeline (C2's filterbank inside the column pass, tensor-core
    rows, detect + fold in the inverse column pass) against the oracle chain:
    hits bit-exact, profiles within 1e-5 (three terms) or 1e-4 (two)."""
    import test_gpu_pipeline as tp
    cfg = tp.base_cfg(b2, dm=500.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=512,
                      period=5.757e-3)
    rng = np.random.default_rng(5 + mode)
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    blocks = tp.make_blocks(rng, cfg, [(cfg["nfft"] + nk + 321) * 64, (nk - 17) * 64])
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], 1, 2, cfg["nfft"], cfg["pos"],
                       cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                       input_kind=cfg["kind"], lut=cfg["lut"], start_mjd=tp.START,
                       epoch_mjd=tp.EPOCH, filterbank_nchan=64, fft_precision=mode)
    pl = b2.Pipeline(ctx, c)
    tot = 0
    for r in blocks:
        tot += pl.run(torch.from_numpy(r).cuda(), r.size // 4)
    prof, hits = pl.get_profiles()
    pl.close()
    rprof, rhits, rtotal = tp.oracle_chain(orc, b2, blocks, cfg)
    tp.check(prof, hits, tot, rprof, rhits, rtotal, cfg["state"],
             rtol=PROFILE_RTOL if mode == 3 else 1e-4)
