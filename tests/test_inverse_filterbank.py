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


# ---------------------------------------------------------------- GPU engine

GPU_CASES = {
    # the reference's own test shape (test/test_config.toml [[InverseFilterbank.test_shapes]]):
    # 256 -> 1 channels, 128-point input FFTs, 16/16 input overlap, two parts, os 4/3
    "reference_shape": dict(nin=256, nout=1, pfb=256, npol=1, lin=128, os=(4, 3),
                            disc=(3072, 3072), npart=2, kind="float", dc=1, allc=1, dsb=1),
    "split_int16_windows": dict(nin=64, nout=4, pfb=64, npol=2, lin=1024, os=(4, 3),
                                disc=(1536, 768), npart=3, kind="int16", dc=1, allc=0, dsb=1,
                                response=True, temporal=True, spectral=True),
    "combine_coarse_lsb": dict(nin=32, nout=1, pfb=8, npol=2, lin=1024, os=(4, 3),
                               disc=(96, 192), npart=2, kind="float", dc=1, allc=1, dsb=0,
                               pad=6),
    "c5_shape_int16": dict(nin=256, nout=1, pfb=256, npol=2, lin=1024, os=(4, 3),
                           disc=(6144, 6144), npart=2, kind="int16", dc=1, allc=1, dsb=1),
    "int8_no_dc_shift": dict(nin=16, nout=1, pfb=16, npol=2, lin=2048, os=(4, 3),
                             disc=(0, 0), npart=2, kind="int8", dc=0, allc=1, dsb=1),
}


def _case_input(rng, case, ndat, b2):
    nin, npol = case["nin"], case["npol"]
    if case["kind"] == "int16":
        raw = rng.integers(-3000, 3000, (ndat, nin, npol, 2)).astype(np.int16)
        x = (raw.astype(np.float32) + 0.5).transpose(1, 2, 0, 3).copy().view(np.complex64)[..., 0]
        return raw.reshape(-1), x, b2.INT16_TFPD, None
    if case["kind"] == "int8":
        raw = rng.integers(-128, 128, (ndat, nin, npol, 2)).astype(np.int8).view(np.uint8)
        lut, _ = b2.bittable8()
        x = lut[raw].transpose(1, 2, 0, 3).copy().view(np.complex64)[..., 0]
        return raw.reshape(-1), x, b2.INT8_TFPD, lut
    x = (rng.standard_normal((nin, npol, ndat)) +
         1j * rng.standard_normal((nin, npol, ndat))).astype(np.complex64)
    return x, x, b2.FLOAT_FPT, None


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GPU_CASES))
def test_ifb_gpu_matches_oracle(ctx, b2, orc, name):
    torch = pytest.importorskip("torch")
    case = GPU_CASES[name]
    ifb = b2.InverseFilterbank(ctx, case["nin"], case["nout"], case["pfb"], case["npol"],
                               case["lin"], os=case["os"], output_discard=case["disc"],
                               pfb_dc_chan=case["dc"], pfb_all_chan=case["allc"],
                               dual_sideband=case["dsb"])
    info = ifb.info
    cfg = dict(input_nchan=case["nin"], output_nchan=case["nout"], pfb_nchan=case["pfb"],
               npol=case["npol"], input_fft_length=case["lin"], os_num=case["os"][0],
               os_den=case["os"][1], output_discard_pos=case["disc"][0],
               output_discard_neg=case["disc"][1], pfb_dc_chan=case["dc"],
               pfb_all_chan=case["allc"], dual_sideband=case["dsb"])
    keep, lout, ipos, ineg, in_step, out_step = orc.ifb_sizes(cfg)
    assert (info["keep"], info["lout"], info["in_step"], info["out_step"]) == \
        (keep, lout, in_step, out_step)
    ndat = case["npart"] * in_step + ipos + ineg + 5      # a ragged tail
    rng = np.random.default_rng(len(name))
    raw, x, kind, lut = _case_input(rng, case, ndat, b2)
    resp = temporal = spectral = None
    if case.get("response"):
        ph = rng.uniform(0, 2 * np.pi, (case["nout"], lout))
        resp = (np.exp(1j * ph) * rng.uniform(0.5, 1.5, (case["nout"], lout))).astype(np.complex64)
        ifb.copy_response(resp)
    if case.get("temporal"):
        temporal = b2.apodization(b2.APOD_TUKEY, case["lin"], ipos, ineg)
    if case.get("spectral"):
        spectral = b2.apodization(b2.APOD_HANNING, lout, swap_halves=True)
    ifb.set_apodization(temporal, spectral)
    ref = orc.inverse_filterbank(x, cfg, response=resp, temporal=temporal, spectral=spectral)
    ref64 = orc.inverse_filterbank(x, cfg, response=resp, temporal=temporal, spectral=spectral,
                                   fp64=True)
    span = case["npart"] * out_step + 3
    d_out = torch.full((case["nout"], case["npol"], span, 2), float("nan"), device="cuda")
    if kind == b2.FLOAT_FPT:
        pad = case.get("pad", 0)
        xin = np.zeros((case["nin"], case["npol"], ndat + pad), np.complex64)
        xin[:, :, :ndat] = x
        d_in = torch.from_numpy(xin.view(np.float32)).cuda()
        n = ifb.perform(d_in, ndat, d_out, span, in_span=ndat + pad)
    else:
        d_in = torch.from_numpy(raw).cuda()
        n = ifb.perform(d_in, ndat, d_out, span, input_kind=kind, lut=lut)
    ctx.synchronize()
    ifb.status()
    assert n == case["npart"]
    out = d_out.cpu().numpy().view(np.complex64)[..., 0]
    body = out[:, :, :n * out_step]
    assert np.isnan(out[:, :, n * out_step:].view(np.float32)).all()
    assert rel_rms(body, ref64) < IFB_RTOL_FP64, rel_rms(body, ref64)
    assert rel_rms(body, ref) < IFB_RTOL, rel_rms(body, ref)
    ifb.close()


@pytest.mark.gpu
def test_ifb_rejects_bad_shapes(ctx, b2):
    bad = [
        dict(input_nchan=16, output_nchan=1, pfb_nchan=16, npol=1, input_fft_length=256),  # Lout 3072
        dict(input_nchan=16, output_nchan=1, pfb_nchan=16, npol=1, input_fft_length=100),
        dict(input_nchan=256, output_nchan=1, pfb_nchan=256, npol=1, input_fft_length=128,
             output_discard=(1000, 0)),                                                  # not whole
        dict(input_nchan=256, output_nchan=3, pfb_nchan=256, npol=1, input_fft_length=128),
        dict(input_nchan=256, output_nchan=1, pfb_nchan=256, npol=3, input_fft_length=128),
    ]
    for b in bad:
        with pytest.raises(b2.B200Error) as e:
            b2.InverseFilterbank(ctx, **b)
        assert e.value.code == b2._capi.EINVAL, b
