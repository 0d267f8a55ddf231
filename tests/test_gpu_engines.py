"""GPU parity of the per-operation engines against the CPU oracle, through the
C ABI of libdspsr_b200.so.

Bars: bit-exact for unpacking, detection and fold bin indices; stated
relative tolerances for FFT-convolved voltages and folded profiles."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# relative RMS error of FP32 overlap-save voltages against the FP64 oracle
VOLTAGE_RTOL_FP64 = 2e-6
# and against the FP32 oracle (two independent FP32 FFT round trips)
VOLTAGE_RTOL_FP32 = 3e-6


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


# ---------------------------------------------------------------- unpack

@pytest.mark.parametrize("nchan,npol,ndim,ndat", [(1, 2, 2, 100003), (4, 2, 2, 5000),
                                                  (3, 1, 1, 777), (1, 2, 2, 1)])
def test_unpack8_bit_exact(ctx, b2, orc, nchan, npol, ndim, ndat):
    rng = np.random.default_rng(nchan * 7 + ndat)
    raw = rng.integers(0, 256, ndat * nchan * npol * ndim, dtype=np.uint8)
    lut, _ = b2.bittable8()
    ref = orc.unpack8(raw, ndat, nchan, npol, ndim, lut)
    out = torch.full((nchan, npol, ndat * ndim), np.nan, dtype=torch.float32, device="cuda")
    ctx.unpack8(dev(raw), ndat, nchan, npol, ndim, lut, out, ndat * ndim)
    ctx.synchronize()
    assert out.cpu().numpy().tobytes() == ref.tobytes()


@pytest.mark.parametrize("offset_binary", [False, True])
def test_unpack16_bit_exact(ctx, b2, orc, offset_binary):
    rng = np.random.default_rng(5)
    nchan, npol, ndim, ndat = 3, 2, 2, 4099
    raw = rng.integers(-32768, 32768, ndat * nchan * npol * ndim).astype(np.int16)
    ref = orc.unpack16(raw, ndat, nchan, npol, ndim, offset_binary)
    out = torch.empty((nchan, npol, ndat * ndim), dtype=torch.float32, device="cuda")
    ctx.unpack16(dev(raw), ndat, nchan, npol, ndim, out, ndat * ndim, offset_binary)
    ctx.synchronize()
    assert out.cpu().numpy().tobytes() == ref.tobytes()


def test_unpack8_rejects_short_span(ctx, b2):
    raw = torch.zeros(400, dtype=torch.uint8, device="cuda")
    out = torch.zeros(100, dtype=torch.float32, device="cuda")
    lut, _ = b2.bittable8()
    with pytest.raises(b2.B200Error):
        ctx.unpack8(raw, 100, 1, 2, 2, lut, out, 10)


# ---------------------------------------------------------------- detection

@pytest.mark.parametrize("state", [0, 1, 2, 3])
def test_detect_bit_exact(ctx, b2, orc, state):
    rng = np.random.default_rng(state)
    nchan, ndat = 5, 30011
    x = (rng.standard_normal((nchan, 2, ndat)) + 1j * rng.standard_normal((nchan, 2, ndat))
         ).astype(np.complex64) * 37.0
    ref = orc.detect(x, state)
    nout = ref.shape[1]
    out = torch.empty((nchan, nout, ndat), dtype=torch.float32, device="cuda")
    ctx.detect(dev(x.view(np.float32)), ndat, ndat, nchan, state, out, ndat)
    ctx.synchronize()
    assert out.cpu().numpy().tobytes() == ref.tobytes()


def test_detect_closed_forms(ctx, b2):
    """test_Detection.cpp:113-244 on the GPU engine."""
    nchan, npol, ndat = 8, 2, 100
    f = np.zeros((nchan, npol, ndat), np.float32)
    for c in range(nchan):
        for p in range(npol):
            f[c, p] = c * npol * ndat + p * ndat + np.arange(ndat)
    x = (f + 1j * f).astype(np.complex64)
    out = torch.empty((nchan, 1, ndat), dtype=torch.float32, device="cuda")
    ctx.detect(dev(x.view(np.float32)), ndat, ndat, nchan, b2.INTENSITY, out, ndat)
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy()[:, 0], 2 * f[:, 0] ** 2 + 2 * f[:, 1] ** 2)


# ---------------------------------------------------------------- filterbank

@pytest.mark.parametrize("nsub,kind", [(64, 0), (64, 2), (16, 1), (4, 2), (32, 0), (128, 0),
                                       (256, 1), (1024, 2), (1024, 0), (4096, 1)])
def test_filterbank_matches_oracle(ctx, b2, orc, nsub, kind):
    """Filterbank with freq_res = 1 (FilterbankEngineCPU.C:379-535) through
    dspsr_b200_filterbank, unpack fused for int8/int16 input; 64 channels and
    more run the shared-memory transforms."""
    rng = np.random.default_rng(nsub + kind)
    nchan, npol, ndat = 2, 2, nsub * (3001 if nsub <= 256 else 301) + 7
    lut, _ = b2.bittable8()
    if kind == b2.INT8_TFPD:
        raw = rng.integers(0, 256, ndat * nchan * npol * 2, dtype=np.uint8)
        x = orc.unpack8(raw, ndat, nchan, npol, 2, lut)
        d_in = dev(raw)
    elif kind == b2.INT16_TFPD:
        raw = rng.integers(-3000, 3000, ndat * nchan * npol * 2).astype(np.int16)
        x = orc.unpack16(raw, ndat, nchan, npol, 2)
        d_in = dev(raw)
    else:
        x = rng.standard_normal((nchan, npol, 2 * ndat)).astype(np.float32)
        d_in = dev(x)
    x = x.view(np.complex64).reshape(nchan, npol, ndat)
    ref = orc.filterbank(x, nsub)
    ref64 = orc.filterbank(x.astype(np.complex128), nsub)
    nb = ndat // nsub
    out = torch.zeros((nchan * nsub, npol, nb), dtype=torch.complex64, device="cuda")
    assert ctx.filterbank(kind, d_in, ndat, nchan, npol, nsub, out, nb, in_span=ndat,
                          lut=lut) == nb
    ctx.synchronize()
    got = out.cpu().numpy()
    tol = 3e-7 if nsub <= 64 else 6e-7
    assert rel_rms(got, ref64) < tol, rel_rms(got, ref64)
    assert rel_rms(got, ref) < tol, rel_rms(got, ref)


def test_channel_response_matches_oracle(ctx, b2, orc):
    """Per-channel response of the filterbank's DC-centred, swapped channels."""
    nchan, nfft, bw, dm = 64, 1 << 13, 256.0, 50.0
    freqs = orc.channel_centres(1400.0, bw, nchan, swap=True, dc_centred=True)
    pos = orc.smearing_samples(1400.0, bw, dm, nchan, 1)
    neg = orc.smearing_samples(1400.0, bw, dm, nchan, -1)
    c = b2.Convolution(ctx, nchan, 2, nfft, pos, neg)
    c.set_dedispersion_channels(freqs, bw, dm, chirp_mode=b2.CHIRP_REFERENCE)
    got = c.get_response()
    ref = orc.dedispersion_response_channels(freqs, bw, dm, nfft, mode=0)
    scale = np.float32(1 / np.sqrt(nfft))
    assert np.max(np.abs(got - ref)) < 4 * 2.0 ** -24 * scale
    c.set_dedispersion_channels(freqs, bw, dm, chirp_mode=b2.CHIRP_FP64)
    got = c.get_response()
    ref64 = orc.dedispersion_response_channels(freqs, bw, dm, nfft, fp64=True)
    assert np.max(np.abs(got - ref64)) < 2.0 ** -23 * scale
    c.close()


# ---------------------------------------------------------------- fold

FOLD_CASES = [
    # phi, rate, period, nbin, ndat
    (0.123456789, 16e6, 0.08933, 1024, 1 << 24),      # C1 block
    (-0.3, 4e6, 5.757e-3, 2048, 1 << 22),             # C2 channel block
    (0.1, 781250.0, 1.6e-3, 4096, 1 << 20),           # C5 channel block
    (-1e-20, 1e6, 1e-3, 64, 100000),                  # first sample rounds to phase 1.0
    (0.0, 1.0, 1024.0, 1024, 100000),                 # dyadic phase step
]


@pytest.mark.parametrize("phi,rate,period,nbin,ndat", FOLD_CASES)
def test_fold_bins_bit_exact(ctx, b2, orc, phi, rate, period, nbin, ndat):
    pps = (1.0 / rate) / period
    ref = orc.fold_binplan(phi, pps, ndat, nbin)
    f = b2.Fold(ctx, nbin, 1, 1)
    f.set_bins(phi, pps, ndat)
    out = torch.empty(ndat, dtype=torch.int32, device="cuda")
    f.binplan(out)
    ctx.synchronize()
    got = out.cpu().numpy().view(np.uint32)
    bad = np.flatnonzero(got != ref)
    assert bad.size == 0, (bad[:5], got[bad[:5]], ref[bad[:5]])
    f.close()


def test_fold_accumulate(ctx, b2, orc):
    rng = np.random.default_rng(9)
    nchan, npol, ndat, nbin = 3, 4, 200000, 512
    phi, pps = 0.77, 1.0 / 3001.7
    data = rng.random((nchan, npol, ndat), dtype=np.float32)
    plan = orc.fold_binplan(phi, pps, ndat, nbin)
    rprof, rhits = orc.fold_accumulate(data.astype(np.float64), plan, nbin)
    f = b2.Fold(ctx, nbin, nchan, npol)
    f.set_bins(phi, pps, ndat)
    f.fold(dev(data), ndat)
    prof, hits = f.get_profiles()
    assert np.array_equal(hits, rhits)
    assert np.max(np.abs(prof - rprof) / rprof) < 2e-6
    # a second block accumulates onto the first
    f.set_bins(phi, pps, ndat)
    f.fold(dev(data), ndat)
    prof2, hits2 = f.get_profiles()
    assert np.array_equal(hits2, 2 * rhits)
    assert np.max(np.abs(prof2 - 2 * rprof) / (2 * rprof)) < 2e-6
    f.close()


# ---------------------------------------------------------------- convolution

@pytest.mark.parametrize("nfft,fft", [(4096, 0), (8192, 0), (16384, 0), (1 << 16, 0),
                                      (1 << 17, 0), (1 << 18, 0), (16384, 3), (1 << 16, 3),
                                      (1 << 17, 3), (1 << 18, 3)])
def test_convolution_tukey_known_answer(ctx, b2, orc, nfft, fft):
    """ConvolutionTest.test_operate_tukey (ConvolutionTest.cpp:148-308) on the
    GPU engine, at the reference's FFT length and at the lengths the BASELINE
    configurations use; fft = 3: the rows on the tensor cores (three BF16
    terms), held to the same thresholds."""
    from test_oracle import _tukey_case

    def gpu_convolve(x, r, n, pos, neg):
        if n != nfft:
            # widen the FFT: the test response is rebuilt for the new length
            spec, _ = orc.tukey_response(neg, pos, nfft)
            norm = np.float32(1.0 / np.sqrt(nfft))
            r = (spec.view(np.float32) * norm).view(np.complex64).reshape(1, nfft)
        nchan, npol, ndat = x.shape
        c = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
        c.copy_response(r)
        if fft:
            c.set_fft_precision(fft)
        npart = c.npart(ndat)
        out = torch.zeros((nchan, npol, npart * c.nkeep), dtype=torch.complex64, device="cuda")
        c.perform(dev(x), ndat, ndat, out, npart * c.nkeep)
        ctx.synchronize()
        c.close()
        return out.cpu().numpy()

    if nfft == 4096:
        _tukey_case(orc, gpu_convolve)
    else:
        # same impulses and thresholds, FFT length nfft
        n_neg, n_pos = 128, 256
        spectral, temporal = orc.tukey_response(n_neg, n_pos, nfft)
        n_overlap = n_neg + n_pos
        n_keep = nfft - n_overlap
        n_loop = max(3, (1 << 20) // (2 * n_keep))
        input_ndat = n_keep * 2 * n_loop + n_overlap
        x = np.zeros((1, 2, input_ndat), np.complex64)
        offsets = []
        for iloop in range(n_loop):
            for ipol in range(2):
                off = [n_overlap, nfft - n_pos][ipol] + iloop * 2 * n_keep + iloop + ipol
                offsets.append((ipol, off))
                x[0, ipol, off] = 1.0
        norm = np.float32(1.0 / np.sqrt(nfft))
        r = (spectral.view(np.float32) * norm).view(np.complex64).reshape(1, nfft)
        out = gpu_convolve(x, r, nfft, n_pos, n_neg)
        expect = np.zeros_like(out)
        for ipol, off in offsets:
            expect[0, ipol, off - n_overlap:off] = temporal
        for ipol in range(2):
            t = temporal.astype(np.complex128)
            for p, off in offsets:
                if p != ipol:
                    continue
                seg = out[0, ipol, off - n_overlap:off].astype(np.complex128)
                err = np.sqrt(np.sum(np.abs(seg - t) ** 2) / np.sum(np.abs(t) ** 2) / n_overlap)
                assert err < 5e-8, (nfft, ipol, off, err)
            mask = np.abs(expect[0, ipol]) == 0
            rms = np.sqrt(np.mean(np.abs(out[0, ipol][mask].astype(np.complex128)) ** 2))
            assert rms < 5e-8, (nfft, ipol, rms)


@pytest.mark.parametrize("nfft,nchan,pos,neg", [(4096, 2, 300, 211), (8192, 1, 1000, 1500),
                                                (1 << 14, 3, 2000, 1777), (1 << 17, 1, 28462, 29455)])
def test_convolution_matches_oracle(ctx, b2, orc, nfft, nchan, pos, neg):
    rng = np.random.default_rng(nfft + nchan)
    npol = 2
    nk = nfft - pos - neg
    ndat = nk * 5 + pos + neg + 123
    x = (rng.standard_normal((nchan, npol, ndat)) + 1j * rng.standard_normal((nchan, npol, ndat))
         ).astype(np.complex64)
    h = (rng.standard_normal((nchan, nfft)) + 1j * rng.standard_normal((nchan, nfft))
         ).astype(np.complex64) / np.float32(np.sqrt(nfft))
    ref64 = orc.convolve(x.astype(np.complex128), h.astype(np.complex128), nfft, pos, neg)
    ref32 = orc.convolve(x, h, nfft, pos, neg)
    c = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    c.copy_response(h)
    assert np.array_equal(c.get_response(), h)
    npart = c.npart(ndat)
    assert npart == 5
    out = torch.zeros((nchan, npol, npart * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(dev(x), ndat, ndat, out, npart * nk) == npart
    ctx.synchronize()
    got = out.cpu().numpy()
    assert rel_rms(got, ref64) < VOLTAGE_RTOL_FP64
    assert rel_rms(got, ref32) < VOLTAGE_RTOL_FP32
    c.close()


@pytest.mark.parametrize("nchan,nfft,dm,bw", [(1, 1 << 17, 67.99, 16.0), (4, 1 << 15, 30.0, 64.0),
                                              (2, 1 << 16, 500.0, -8.0)])
def test_dedispersion_response_matches_oracle(ctx, b2, orc, nchan, nfft, dm, bw):
    pos = orc.smearing_samples(1400.0, bw, dm, nchan, 1)
    neg = orc.smearing_samples(1400.0, bw, dm, nchan, -1)
    assume = pos + neg < nfft
    assert assume
    c = b2.Convolution(ctx, nchan, 2, nfft, pos, neg)
    # reference mode: float(phase) then sin/cos in float (Dedispersion.C:104-111)
    c.set_dedispersion(1400.0, bw, dm, chirp_mode=b2.CHIRP_REFERENCE)
    got = c.get_response()
    ref = orc.dedispersion_response(1400.0, bw, dm, nchan, nfft, input_nchan=nchan, mode=0)
    scale = np.float32(1 / np.sqrt(nfft))
    # same float phase on both sides; sinf/cosf differ by at most a few ulp
    assert np.max(np.abs(got - ref)) < 4 * 2.0 ** -24 * scale
    c.set_dedispersion(1400.0, bw, dm, chirp_mode=b2.CHIRP_FP64)
    got = c.get_response()
    ref = orc.dedispersion_response(1400.0, bw, dm, nchan, nfft, input_nchan=nchan, mode=1)
    assert np.max(np.abs(got - ref)) < 2 * 2.0 ** -24 * scale
    ref64 = orc.dedispersion_response_f64(1400.0, bw, dm, nchan, nfft, input_nchan=nchan)
    assert np.max(np.abs(got - ref64)) < 2.0 ** -23 * scale
    c.close()


@pytest.mark.parametrize("nchan,nfft,dm,bw", [(1, 1 << 17, 67.99, 16.0), (1, 8192, 5.0, 16.0),
                                              (4, 1 << 15, 30.0, 64.0)])
def test_dedispersed_voltages_within_2e6_of_fp64(ctx, b2, orc, nchan, nfft, dm, bw):
    """Dedispersed voltages with the FP64-phase chirp against the all-FP64
    oracle (FP64 response and FFT): relative RMS error <= 2e-6."""
    rng = np.random.default_rng(nfft + nchan)
    pos = orc.smearing_samples(1400.0, bw, dm, nchan, 1)
    neg = orc.smearing_samples(1400.0, bw, dm, nchan, -1)
    nk = nfft - pos - neg
    ndat = nfft + 3 * nk
    x = (np.round(rng.standard_normal((nchan, 2, ndat)) * 10)
         + 1j * np.round(rng.standard_normal((nchan, 2, ndat)) * 10)).astype(np.complex64)
    h64 = orc.dedispersion_response_f64(1400.0, bw, dm, nchan, nfft, input_nchan=nchan)
    ref = orc.convolve(x.astype(np.complex128), h64, nfft, pos, neg)
    c = b2.Convolution(ctx, nchan, 2, nfft, pos, neg)
    c.set_dedispersion(1400.0, bw, dm, chirp_mode=b2.CHIRP_FP64)
    out = torch.zeros((nchan, 2, 4 * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(dev(x), ndat, ndat, out, 4 * nk) == 4
    ctx.synchronize()
    got = out.cpu().numpy()
    assert rel_rms(got, ref) < VOLTAGE_RTOL_FP64, rel_rms(got, ref)
    c.close()


def test_convolution_rejects_bad_shapes(ctx, b2):
    with pytest.raises(b2.B200Error):
        b2.Convolution(ctx, 1, 2, 3000, 10, 10)        # not a power of two
    with pytest.raises(b2.B200Error):
        b2.Convolution(ctx, 1, 2, 4096, 3000, 1096)    # no samples kept
    c = b2.Convolution(ctx, 1, 2, 4096, 100, 100)
    x = torch.zeros((1, 2, 5000), dtype=torch.complex64, device="cuda")
    with pytest.raises(b2.B200Error):
        c.perform(x, 5000, 5000, x, 5000)               # no response yet
    c.copy_response(np.ones(4096, np.complex64))
    out = torch.zeros((1, 2, 10), dtype=torch.complex64, device="cuda")
    with pytest.raises(b2.B200Error):
        c.perform(x, 5000, 5000, out, 10)               # output too small
    assert c.perform(x, 5000, 100, out, 10) == 0       # fewer samples than one FFT
    c.close()


@pytest.mark.parametrize("nfft,pos,neg", [(8192, 100, 200), (1 << 15, 0, 0), (1 << 16, 3000, 1000)])
def test_convolution_zero_dm_output_is_input(ctx, b2, orc, nfft, pos, neg):
    """test_Convolution.cpp:151-186: the zero-DM output equals the input,
    sample for sample (here: the input samples aligned with the output)."""
    nchan, npol = 2, 2
    nk = nfft - pos - neg
    ndat = 3 * nk + pos + neg + 17
    rng = np.random.default_rng(nfft)
    x = (rng.standard_normal((nchan, npol, ndat)) +
         1j * rng.standard_normal((nchan, npol, ndat))).astype(np.complex64)
    resp = np.exp(1j * rng.uniform(0, 2 * np.pi, (nchan, nfft))).astype(np.complex64)
    conv = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    conv.copy_response(resp)
    d_in = dev(x.view(np.float32))
    out = torch.zeros((nchan, npol, 3 * nk, 2), device="cuda")
    zdm = torch.full((nchan, npol, 3 * nk + 5, 2), float("nan"), device="cuda")
    out2 = torch.zeros_like(out)
    n = conv.perform_zero_dm(d_in, ndat, ndat, out, 3 * nk, zdm, 3 * nk + 5)
    conv.perform(d_in, ndat, ndat, out2, 3 * nk)
    ctx.synchronize()
    assert n == 3
    z = zdm.cpu().numpy().view(np.complex64)[..., 0]
    assert z[:, :, :3 * nk].tobytes() == x[:, :, pos:pos + 3 * nk].tobytes()
    assert np.isnan(z[:, :, 3 * nk:].view(np.float32)).all()
    assert out.cpu().numpy().tobytes() == out2.cpu().numpy().tobytes()
    conv.close()


def test_c2_shape_voltages_within_2e6_of_fp64(ctx, b2, orc):
    """The C2 shape (256 MHz dual-pol int8 at 1400 MHz, a 64-channel FFT
    filterbank, each 4 MHz channel dedispersed at DM 500 with 2^16-point
    FFTs, FP64-phase chirp): the dedispersed voltages of every channel against
    the all-FP64 oracle chain (FP64 unpack values, filterbank, response and
    FFTs; Filterbank.C:549-565, Convolution.C:724-803): relative RMS error
    <= 2e-6 over all channels and polarisations."""
    cf, bw, dm, nsub, nfft = 1400.0, 256.0, 500.0, 64, 1 << 16
    pos = orc.smearing_samples(cf, bw, dm, nsub, 1)
    neg = orc.smearing_samples(cf, bw, dm, nsub, -1)
    nk = nfft - pos - neg
    npart = 3
    nch = nfft + (npart - 1) * nk + 77            # samples per channel
    ndat = nch * nsub                              # input samples per pol
    rng = np.random.default_rng(500)
    raw = np.clip(np.round(rng.standard_normal(ndat * 4) * 12), -128, 127).astype(np.int8)
    raw = raw.view(np.uint8)
    lut, _ = b2.bittable8()
    lut = np.asarray(lut, np.float32)

    # GPU: filterbank engine, then the convolution engine on its channels
    fbo = torch.zeros((nsub, 2, nch), dtype=torch.complex64, device="cuda")
    n = ctx.filterbank(b2.INT8_TFPD, dev(raw), ndat, 1, 2, nsub, fbo, nch, lut=lut)
    assert n == nch
    freqs = orc.channel_centres(cf, bw, nsub, swap=True, dc_centred=True)
    c = b2.Convolution(ctx, nsub, 2, nfft, pos, neg)
    c.set_dedispersion_channels(freqs, bw, dm, chirp_mode=b2.CHIRP_FP64)
    out = torch.zeros((nsub, 2, npart * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(fbo, nch, nch, out, npart * nk) == npart
    ctx.synchronize()
    c.status()
    got = out.cpu().numpy()
    c.close()

    # FP64 oracle chain on the same bytes
    x = orc.unpack8(raw, ndat, 1, 2, 2, lut).view(np.complex64).reshape(1, 2, ndat)
    y = orc.filterbank(x.astype(np.complex128), nsub)
    h = orc.dedispersion_response_channels(freqs, bw, dm, nfft, fp64=True)
    ref = orc.convolve(y, h, nfft, pos, neg)
    assert ref.shape == got.shape
    err = rel_rms(got, ref)
    assert err < VOLTAGE_RTOL_FP64, err
    # and channel by channel (no channel may hide behind the average)
    per = [rel_rms(got[k], ref[k]) for k in range(nsub)]
    assert max(per) < 2 * VOLTAGE_RTOL_FP64, max(per)
