"""Apodization (Signal/General/Apodization.C): the window builders bit for bit
against the oracle, and the temporal window fused into the convolution's
loads on the GPU against the oracle's windowed overlap-save."""
import numpy as np
import pytest

VOLTAGE_RTOL_FP32 = 3e-6

WINDOWS = [(kind, n, ts, te, sw) for kind in range(5) for n in (2, 17, 1024, 65536)
           for (ts, te) in ((1, 1), (n // 4, n // 8), (n // 2, n // 2)) for sw in (False, True)]


@pytest.mark.parametrize("kind,n,ts,te,sw", WINDOWS)
def test_window_matches_oracle(b2, orc, kind, n, ts, te, sw):
    a = b2.apodization(kind, n, ts, te, sw)
    b = orc.apodization(kind, n, ts, te, sw)
    assert a.tobytes() == b.tobytes()


def test_window_shapes(b2):
    n = 64
    h = b2.apodization(b2.APOD_HANNING, n)
    assert h[0] == 0 and abs(h[n // 2] - 1) < 1e-2 and np.allclose(h, h[::-1], atol=1e-6)
    t = b2.apodization(b2.APOD_TUKEY, n, 8, 8)
    assert t[0] == 0 and t[n - 1] == 0 and np.all(t[8:n - 8] == 1)
    assert np.all(b2.apodization(b2.APOD_TOPHAT, n) == 1)
    s = b2.apodization(b2.APOD_HANNING, n, swap_halves=True)
    assert s.tobytes() == np.concatenate([h[n // 2:], h[:n // 2]]).tobytes()
    with pytest.raises(b2.B200Error):
        b2.apodization(9, n)


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


@pytest.mark.gpu
@pytest.mark.parametrize("nchan,npol,nfft,pos,neg", [(2, 2, 8192, 700, 500), (1, 2, 1 << 16, 9000, 7000)])
def test_convolution_temporal_window(ctx, b2, orc, nchan, npol, nfft, pos, neg):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(nfft)
    nkeep = nfft - pos - neg
    ndat = 3 * nkeep + pos + neg
    x = (rng.standard_normal((nchan, npol, ndat)) +
         1j * rng.standard_normal((nchan, npol, ndat))).astype(np.complex64)
    resp = np.exp(1j * rng.uniform(0, 2 * np.pi, (nchan, nfft))).astype(np.complex64)
    win = b2.apodization(b2.APOD_TUKEY, nfft, pos, neg)
    ref = orc.convolve_window(x, resp, nfft, pos, neg, win)
    conv = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    conv.copy_response(resp)
    conv.set_temporal_apodization(win)
    d_in = torch.from_numpy(x.view(np.float32)).cuda()
    d_out = torch.zeros((nchan, npol, 3 * nkeep, 2), device="cuda")
    n = conv.perform(d_in, ndat, ndat, d_out, 3 * nkeep)
    ctx.synchronize()
    assert n == 3
    out = d_out.cpu().numpy().view(np.complex64)[..., 0]
    assert rel_rms(out, ref) < VOLTAGE_RTOL_FP32, rel_rms(out, ref)
    # removing the window restores the plain convolution
    conv.set_temporal_apodization(None)
    conv.perform(d_in, ndat, ndat, d_out, 3 * nkeep)
    ctx.synchronize()
    out = d_out.cpu().numpy().view(np.complex64)[..., 0]
    assert rel_rms(out, orc.convolve(x, resp, nfft, pos, neg)) < VOLTAGE_RTOL_FP32
    conv.close()
