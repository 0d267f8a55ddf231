"""Filterbank with a response (the "During" filterbank, -F nchan:D;
Filterbank.C:98-198, 398-420; FilterbankEngineCPU.C:379-535): the oracle's
restatement pinned on the CPU against an independent numpy evaluation of the
same steps, its response against the dedispersion response of the
convolution path, and the GPU engine against the oracle through the C ABI.

Bars: oracle FP64 equal to numpy to 1e-12 relative RMS; GPU output within
relative RMS DURING_RTOL of the FP32 oracle fed the GPU's own response and of
the FP64 oracle fed the FP64 response; the GPU-built response within 1e-6
relative RMS of the oracle's."""
import numpy as np
import pytest

DURING_RTOL = 5e-6
DURING_RTOL_FP64 = 5e-6


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def numpy_during(x, nsub, freq_res, nfilt, response, temporal=None, spectral=None):
    """The same filterbank straight from its definition with numpy's FFT."""
    nin, npol, ndat = x.shape
    pos, neg = nfilt
    nkeep = freq_res - pos - neg
    n = nsub * freq_res
    step = nsub * nkeep
    npart = (ndat - (pos + neg) * nsub) // step
    out = np.zeros((nin * nsub, npol, npart * nkeep), np.complex128)
    for ic in range(nin):
        h = response[ic * nsub:(ic + 1) * nsub].reshape(-1)
        for ip in range(npart):
            for p in range(npol):
                seg = x[ic, p, ip * step:ip * step + n]
                if temporal is not None:
                    seg = seg * temporal
                spec = np.fft.fft(seg) * h
                for cs in range(nsub):
                    chan = spec[cs * freq_res:(cs + 1) * freq_res]
                    if spectral is not None:
                        chan = chan * spectral
                    y = np.fft.ifft(chan) * freq_res
                    out[ic * nsub + cs, p, ip * nkeep:(ip + 1) * nkeep] = y[pos:pos + nkeep]
    return out


@pytest.mark.parametrize("nin,npol,nsub,freq_res,nfilt", [(1, 2, 8, 64, (5, 9)),
                                                         (2, 1, 4, 128, (0, 0)),
                                                         (1, 2, 16, 32, (7, 0))])
def test_oracle_matches_numpy(orc, nin, npol, nsub, freq_res, nfilt):
    rng = np.random.default_rng(nsub * freq_res + nin)
    nkeep = freq_res - sum(nfilt)
    ndat = 3 * nsub * nkeep + sum(nfilt) * nsub + 11
    x = rng.standard_normal((nin, npol, ndat)) + 1j * rng.standard_normal((nin, npol, ndat))
    h = rng.standard_normal((nin * nsub, freq_res)) + 1j * rng.standard_normal((nin * nsub, freq_res))
    ref = numpy_during(x, nsub, freq_res, nfilt, h)
    got64 = orc.filterbank_during(x, nsub, freq_res, nfilt, h)
    assert got64.shape == ref.shape and ref.shape[2] == 3 * nkeep
    assert rel_rms(got64, ref) < 1e-12
    got32 = orc.filterbank_during(x.astype(np.complex64), nsub, freq_res, nfilt,
                                  h.astype(np.complex64))
    assert rel_rms(got32, ref) < 1e-5


def test_oracle_windows_match_numpy(orc, b2):
    """Filterbank::set_temporal_apodization / set_spectral_apodization: the
    windows multiply each part before the forward FFT and each channel's
    spectrum before its inverse FFT (FilterbankEngineCPU.C:447-449, 507-509)."""
    rng = np.random.default_rng(11)
    nsub, fr, nfilt = 8, 64, (6, 4)
    nkeep = fr - sum(nfilt)
    ndat = 3 * nsub * nkeep + sum(nfilt) * nsub
    x = rng.standard_normal((1, 2, ndat)) + 1j * rng.standard_normal((1, 2, ndat))
    h = rng.standard_normal((nsub, fr)) + 1j * rng.standard_normal((nsub, fr))
    tw = b2.apodization(b2.APOD_TUKEY, nsub * fr, nfilt[0] * nsub, nfilt[1] * nsub)
    sw = b2.apodization(b2.APOD_HANNING, fr)
    ref = numpy_during(x, nsub, fr, nfilt, h, tw.astype(np.float64), sw.astype(np.float64))
    got = orc.filterbank_during(x, nsub, fr, nfilt, h, temporal=tw, spectral=sw)
    assert rel_rms(got, ref) < 1e-12


def test_oracle_response_is_the_unswapped_channel_response(orc):
    """Each channel of the During response is the convolution path's channel
    response (DC at bin 0) rotated back to natural order; the whole swap
    rotates the channels by nchan/2; the normaliser is 1/sqrt(nsamp_fft *
    freq_res)."""
    cf, bw, dm, nchan, fr = 1400.0, -64.0, 30.0, 16, 512
    nfft_big = nchan * fr
    for swapped in (False, True):
        r = orc.dedispersion_response_during(cf, bw, dm, nchan, fr, nfft_big, swapped=swapped,
                                             fp64=True)
        freq = orc.channel_centres(cf, bw, nchan, swap=swapped)
        conv = orc.dedispersion_response_channels(freq, bw, dm, fr, norm_nfft=fr, fp64=True)
        expect = np.roll(conv, fr // 2, axis=1) * np.sqrt(fr) / np.sqrt(float(nfft_big) * fr)
        assert rel_rms(r, expect) < 1e-12
    r0 = orc.dedispersion_response_during(cf, bw, dm, nchan, fr, nfft_big, swapped=False,
                                          fp64=True)
    r1 = orc.dedispersion_response_during(cf, bw, dm, nchan, fr, nfft_big, swapped=True,
                                          fp64=True)
    assert np.array_equal(np.roll(r0, -nchan // 2, axis=0), r1)


def test_oracle_restores_a_dispersed_pulse(orc):
    """Physics check of the restatement: a pulse dispersed by the exact FP64
    inverse of the response over the whole band comes out of the filterbank
    with its power at one time in every channel."""
    cf, bw, dm, nsub, fr = 1400.0, 16.0, 8.0, 8, 1024
    n = nsub * fr
    r = orc.dedispersion_response_during(cf, bw, dm, nsub, fr, n, swapped=True, fp64=True)
    # the response in FFT order of the big transform: its inverse disperses
    big = r.reshape(-1) * np.sqrt(float(n) * fr)
    x = np.zeros(3 * n, np.complex128)
    x[n + n // 2] = 1.0
    spec = np.fft.fft(x[n:2 * n])
    disp = np.fft.ifft(spec * np.conj(big))
    xin = np.zeros((1, 1, 3 * n), np.complex128)
    xin[0, 0, n:2 * n] = disp
    out = orc.filterbank_during(xin, nsub, fr, (0, 0), r)
    power = np.abs(out[:, 0, :]) ** 2
    peaks = np.argmax(power, axis=1)
    assert np.ptp(peaks) <= 1, peaks


# ---------------------------------------------------------------- GPU engine

GPU_CASES = {
    # 16 channels of 1024 points: n1 = 2, 512-point channel transforms
    "dedisp_16x1024_float": dict(nin=1, npol=2, nsub=16, fr=1024, dm=2.0, kind="float",
                                 npart=3),
    # 64 channels of 4096 points (2^18 points, n1 = 32, 128-point segments), int8
    "dedisp_64x4096_int8": dict(nin=1, npol=2, nsub=64, fr=4096, dm=60.0, kind="int8",
                                npart=2),
    # two input channels, one polarisation, a random response, int16
    "random_2in_8x4096_int16": dict(nin=2, npol=1, nsub=8, fr=4096, nfilt=(300, 200),
                                    kind="int16", npart=3),
    # the smallest segments: 128 channels of 128 points
    "random_128x128_float": dict(nin=1, npol=2, nsub=128, fr=128, nfilt=(16, 8), kind="float",
                                 npart=4),
    # two channels of 65536 points (n1 = 16, 4096-point segments)
    "dedisp_2x65536_float": dict(nin=1, npol=1, nsub=2, fr=65536, dm=5.0, kind="float",
                                 npart=2),
    # 2^19 points: 64-point columns in shared memory
    "random_8x65536_float": dict(nin=1, npol=2, nsub=8, fr=65536, nfilt=(900, 1100),
                                 kind="float", npart=2),
    # temporal Tukey and spectral Hanning windows, 2^20 points (128-point columns)
    "windows_16x65536_int16": dict(nin=1, npol=2, nsub=16, fr=65536, nfilt=(2000, 1500),
                                   kind="int16", npart=2, windows=True),
    # the reference's C2 shape with the dedispersion inside the filterbank
    # (-F 64:D at DM 500 over 256 MHz): 2^22 points, 512-point columns
    "dedisp_64x65536_int8_dm500": dict(nin=1, npol=2, nsub=64, fr=65536, dm=500.0, bw=256.0,
                                       kind="int8", npart=2),
}
CF, BW = 1400.0, 64.0


def _input(rng, nin, npol, ndat, kind, b2):
    if kind == "int16":
        raw = rng.integers(-3000, 3000, (ndat, nin, npol, 2)).astype(np.int16)
        x = (raw.astype(np.float32) + 0.5).transpose(1, 2, 0, 3).copy().view(np.complex64)[..., 0]
        return raw.reshape(-1), x, b2.INT16_TFPD, None
    if kind == "int8":
        raw = rng.integers(-128, 128, (ndat, nin, npol, 2)).astype(np.int8).view(np.uint8)
        lut, _ = b2.bittable8()
        x = lut[raw].transpose(1, 2, 0, 3).copy().view(np.complex64)[..., 0]
        return raw.reshape(-1), x, b2.INT8_TFPD, lut
    x = (rng.standard_normal((nin, npol, ndat)) +
         1j * rng.standard_normal((nin, npol, ndat))).astype(np.complex64)
    return x, x, b2.FLOAT_FPT, None


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_during_gpu_matches_oracle(ctx, b2, orc, name):
    torch = pytest.importorskip("torch")
    case = GPU_CASES[name]
    nin, npol, nsub, fr = case["nin"], case["npol"], case["nsub"], case["fr"]
    nchan = nin * nsub
    rng = np.random.default_rng(len(name))
    bw = case.get("bw", BW)
    if "dm" in case:
        half = b2.smearing_samples(CF, bw, case["dm"], nchan, 1)
        nfilt = (half, half)
    else:
        nfilt = case["nfilt"]
    fbd = b2.FilterbankDuring(ctx, nin, npol, nsub, fr, nfilt)
    info = fbd.info
    nkeep = fr - sum(nfilt)
    assert info["nkeep"] == nkeep and info["nsamp_step"] == nsub * nkeep
    assert info["nsamp_fft"] == nsub * fr and info["nsamp_overlap"] == sum(nfilt) * nsub
    if "dm" in case:
        # the FP64-phase chirp against the FP64 response
        fbd.set_dedispersion(CF, bw, case["dm"], swapped=True, chirp_mode=b2.CHIRP_FP64)
        exact = orc.dedispersion_response_during(CF, bw, case["dm"], nchan, fr, nsub * fr,
                                                 swapped=True, fp64=True)
        assert rel_rms(fbd.get_response(), exact) < 1e-6
        # the reference's chirp (phases rounded to float, Dedispersion.C:104-111)
        # against the oracle's; the transforms are then checked with the
        # response the GPU holds, so that the float phases do not hide their error
        fbd.set_dedispersion(CF, bw, case["dm"], swapped=True)
        resp = fbd.get_response()
        ref_resp = orc.dedispersion_response_during(CF, bw, case["dm"], nchan, fr, nsub * fr,
                                                    swapped=True)
        assert rel_rms(resp, ref_resp) < 1e-6, rel_rms(resp, ref_resp)
        resp64 = resp.astype(np.complex128)
    else:
        ph = rng.uniform(0, 2 * np.pi, (nchan, fr))
        resp = (np.exp(1j * ph) * rng.uniform(0.5, 1.5, (nchan, fr))
                / np.sqrt(float(nsub) * fr * fr)).astype(np.complex64)
        fbd.copy_response(resp)
        assert np.array_equal(fbd.get_response(), resp)
        resp64 = resp.astype(np.complex128)
    tw = sw = None
    if case.get("windows"):
        tw = b2.apodization(b2.APOD_TUKEY, nsub * fr, nfilt[0] * nsub, nfilt[1] * nsub)
        sw = b2.apodization(b2.APOD_HANNING, fr)
        fbd.set_apodization(tw, sw)
        # the response read back is the one set, without the spectral window
        assert np.array_equal(fbd.get_response(), resp)
    ndat = case["npart"] * nsub * nkeep + sum(nfilt) * nsub + 7      # a ragged tail
    raw, x, kind, lut = _input(rng, nin, npol, ndat, case["kind"], b2)
    ref = orc.filterbank_during(x, nsub, fr, nfilt, resp, temporal=tw, spectral=sw)
    ref64 = orc.filterbank_during(x.astype(np.complex128), nsub, fr, nfilt, resp64, temporal=tw,
                                  spectral=sw)
    span = case["npart"] * nkeep + 3
    d_out = torch.full((nchan, npol, span, 2), float("nan"), device="cuda")
    if kind == b2.FLOAT_FPT:
        d_in = torch.from_numpy(np.ascontiguousarray(x).view(np.float32)).cuda()
        n = fbd.perform(d_in, ndat, d_out, span)
    else:
        d_in = torch.from_numpy(raw).cuda()
        n = fbd.perform(d_in, ndat, d_out, span, input_kind=kind, lut=lut)
    ctx.synchronize()
    assert n == case["npart"] == fbd.npart(ndat)
    out = d_out.cpu().numpy().view(np.complex64)[..., 0]
    body = out[:, :, :n * nkeep]
    assert np.isnan(out[:, :, n * nkeep:].view(np.float32)).all()
    assert rel_rms(body, ref) < DURING_RTOL, rel_rms(body, ref)
    assert rel_rms(body, ref64) < DURING_RTOL_FP64, rel_rms(body, ref64)
    fbd.close()


@pytest.mark.gpu
def test_during_rejects_unsupported_shapes(ctx, b2):
    for nsub, fr, nfilt in [(256, 1024, (0, 0)),     # segments below 64 points
                            (3, 8192, (0, 0)),       # not a power of two
                            (8, 1024, (0, 0)),       # 8192 points: below the four-step split
                            (128, 65536, (0, 0)),    # 2^23 points
                            (16, 1024, (600, 424))]:  # nothing kept
        with pytest.raises(b2.B200Error):
            b2.FilterbankDuring(ctx, 1, 2, nsub, fr, nfilt)
    fbd = b2.FilterbankDuring(ctx, 1, 2, 16, 1024, (10, 10))
    torch = pytest.importorskip("torch")
    buf = torch.zeros(1 << 16, device="cuda")
    with pytest.raises(b2.B200Error, match="no response"):
        fbd.perform(buf, 1000, buf, 1000)
    fbd.close()


@pytest.mark.gpu
@pytest.mark.parametrize("state,npol,nsub,fr", [(3, 2, 32, 2048), (1, 2, 32, 2048), (0, 1, 32, 2048),
                                                (3, 2, 16, 65536)])
def test_during_fold_matches_its_voltages(ctx, b2, orc, state, npol, nsub, fr):
    """Detection and fold fused into the last pass give the profiles that the
    oracle's Detection and Fold make of the engine's own voltages (checked
    against the oracle above); hits bit-exact."""
    torch = pytest.importorskip("torch")
    dm, npart = 10.0, 3
    half = b2.smearing_samples(CF, BW, dm, nsub, 1)
    fbd = b2.FilterbankDuring(ctx, 1, npol, nsub, fr, (half, half))
    fbd.set_dedispersion(CF, BW, dm)
    nkeep = fbd.info["nkeep"]
    ndat = npart * nsub * nkeep + 2 * half * nsub + 5
    rng = np.random.default_rng(state + 10 * npol)
    x = (rng.standard_normal((1, npol, ndat)) + 1j * rng.standard_normal((1, npol, ndat))
         ).astype(np.complex64)
    d_in = torch.from_numpy(x.view(np.float32)).cuda()
    span = npart * nkeep
    d_v = torch.zeros((nsub, npol, span, 2), device="cuda")
    assert fbd.perform(d_in, ndat, d_v, span) == npart
    ctx.synchronize()
    v = d_v.cpu().numpy().view(np.complex64)[..., 0].astype(np.complex128)
    if npol == 2:
        det = orc.detect(v, state)
    else:
        det = np.abs(v) ** 2
    nout = det.shape[1]
    nbin, phi, pps = 256, 0.3, 1.0 / 1234.5
    plan = orc.fold_binplan(phi, pps, span, nbin)
    rprof, rhits = orc.fold_accumulate(det, plan, nbin)
    f = b2.Fold(ctx, nbin, nsub, nout)
    f.set_bins(phi, pps, span - 1)
    with pytest.raises(b2.B200Error, match="fold plan"):
        fbd.perform_fold(d_in, ndat, f, state)
    f.set_bins(phi, pps, span)
    assert fbd.perform_fold(d_in, ndat, f, state) == npart
    prof, hits = f.get_profiles()
    assert np.array_equal(hits, rhits)
    assert rel_rms(prof, rprof) < 1e-5, rel_rms(prof, rprof)
    f.close()
    fbd.close()
