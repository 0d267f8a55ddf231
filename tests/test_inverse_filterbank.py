"""InverseFilterbank: the oracle's restatement pinned by an exact
channelise -> stitch -> invert round trip (CPU), and the GPU engine against
the oracle through the C ABI.

Bars: round trip to FP32 rounding (relative RMS 1e-5) against the exact
model; GPU output within relative RMS IFB_RTOL of the FP32 oracle and
IFB_RTOL_FP64 of the FP64 oracle."""
import numpy as np
import pytest

IFB_RTOL = 5e-6
IFB_RTOL_FP64 = 5e-6


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def channelise(w, nchan, lin, keep):
    """An exactly invertible oversampled channeliser of one block: fine
    channel c holds the wideband spectrum bins (c*keep + s) mod L for the
    signed fine-FFT bins s in [-lin/2, lin/2), so channel 0 sits on DC."""
    L = w.size
    W = np.fft.fft(w)
    s = np.fft.fftfreq(lin, 1.0 / lin).astype(int)
    out = np.empty((nchan, lin), np.complex128)
    for c in range(nchan):
        out[c] = np.fft.ifft(W[(c * keep + s) % L])
    return out


@pytest.mark.parametrize("nchan,lin,os", [(16, 64, (4, 3)), (8, 256, (8, 7)), (32, 32, (1, 1))])
def test_oracle_round_trip(orc, nchan, lin, os):
    keep = lin * os[1] // os[0]
    L = nchan * keep
    rng = np.random.default_rng(nchan + lin)
    w = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    x = channelise(w, nchan, lin, keep)[:, None, :]
    cfg = dict(input_nchan=nchan, output_nchan=1, pfb_nchan=nchan, npol=1,
               input_fft_length=lin, os_num=os[0], os_den=os[1], output_discard_pos=0,
               output_discard_neg=0, pfb_dc_chan=1, pfb_all_chan=1, dual_sideband=1)
    y = orc.inverse_filterbank(x, cfg)
    assert y.shape == (1, 1, L)
    assert rel_rms(y[0, 0], L * w) < 1e-5
    y64 = orc.inverse_filterbank(x, cfg, fp64=True)
    assert rel_rms(y64[0, 0], L * w) < 1e-12


def test_oracle_split_into_outputs(orc):
    """Splitting a coarse channel into several outputs: each output channel is
    the inverse transform of its own run of fine channels (stitch of the
    whole coarse channel, then one inverse FFT per output)."""
    nchan, lin, keep, nout = 16, 64, 48, 4
    L = nchan * keep
    rng = np.random.default_rng(5)
    w = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    x = channelise(w, nchan, lin, keep)[:, None, :]
    cfg = dict(input_nchan=nchan, output_nchan=nout, pfb_nchan=nchan, npol=1,
               input_fft_length=lin, os_num=4, os_den=3, output_discard_pos=0,
               output_discard_neg=0, pfb_dc_chan=1, pfb_all_chan=1, dual_sideband=1)
    y = orc.inverse_filterbank(x, cfg)
    W = np.fft.fft(w)
    lout = L // nout
    for o in range(nout):
        ref = np.fft.ifft(W[o * lout:(o + 1) * lout]) * lout
        assert rel_rms(y[o, 0], ref) < 1e-5


def test_oracle_rejects_non_integer_shapes(orc):
    cfg = dict(input_nchan=16, output_nchan=1, pfb_nchan=16, npol=1, input_fft_length=66,
               os_num=4, os_den=3, output_discard_pos=0, output_discard_neg=0,
               pfb_dc_chan=1, pfb_all_chan=1, dual_sideband=1)
    with pytest.raises(ValueError):
        orc.inverse_filterbank(np.zeros((16, 1, 132), np.complex64), cfg)
