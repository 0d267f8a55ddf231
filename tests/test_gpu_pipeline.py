"""GPU parity of the fused unpack -> convolve -> detect -> fold pipeline
against the oracle chain, block by block with the overlap carry
(InputBuffering) and the per-block fold phase (Fold::fold, Fold.C:685-693)."""
import zlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# relative error of each folded profile bin against the oracle chain
PROFILE_RTOL = 1e-5
# FP64-chirp pipeline against the all-FP64 oracle chain
PROFILE_RTOL_FP64 = 5e-6

START = (60000, 3600, 0.25)
EPOCH = (59999, 0, 0.0)


def oracle_chain(orc, b2, raw_blocks, cfg, fp64=False):
    """raw_blocks: list of TFPD arrays.  Mirrors SingleThread::run over the
    blocks: unpack, overlap-save, detect, fold with one phase per block."""
    d, nchan = oracle_detected(orc, b2, raw_blocks, cfg, fp64)
    return oracle_fold(orc, b2, raw_blocks, cfg, d, nchan)


def oracle_detected(orc, b2, raw_blocks, cfg, fp64=False):
    """The detected output of the whole stream: (d [chan][nout][t], nchan)."""
    y, nchan = oracle_voltages(orc, b2, raw_blocks, cfg, fp64)
    if cfg["npol"] == 1:
        d = (y.real ** 2 + y.imag ** 2)
        d = d.reshape(nchan, 1, -1)
    else:
        d = orc.detect(y, cfg["state"])
    return d, nchan


def oracle_voltages(orc, b2, raw_blocks, cfg, fp64=False, interchannel=None):
    """The dedispersed voltages of the whole stream: (y [chan][pol][t], nchan).
    interchannel: a dict to receive the inter-channel delays, whose fractional
    parts then enter the response (Dedispersion.C:141-187)."""
    nchan, npol = cfg["nchan"], cfg["npol"]
    kind = cfg["kind"]
    raw = np.concatenate([r.reshape(-1) for r in raw_blocks])
    if kind == b2.INT8_TFPD:
        ndat_tot = raw.size // (nchan * npol * 2)
        x = orc.unpack8(raw, ndat_tot, nchan, npol, 2, cfg["lut"])
    elif kind == b2.INT16_TFPD:
        ndat_tot = raw.size // (nchan * npol * 2)
        x = orc.unpack16(raw, ndat_tot, nchan, npol, 2, False)
    else:
        x = np.concatenate([r for r in raw_blocks], axis=2).view(np.float32)
        ndat_tot = x.shape[2] // 2
    x = x.view(np.complex64).reshape(nchan, npol, ndat_tot)
    nfft, pos, neg = cfg["nfft"], cfg["pos"], cfg["neg"]
    nk = nfft - pos - neg
    fb = cfg.get("fb", 0)
    if interchannel is not None:
        if fb:
            x = orc.filterbank(x, fb)
            nchan *= fb
            freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nchan, swap=True, dc_centred=True)
        else:
            freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nchan)
        rate = abs(cfg["bw"]) / nchan * 1e6
        delays = orc.interchannel_delays(cfg["cf"], cfg["dm"], rate, list(freqs))
        interchannel.update(delays)
        frac_us = delays["frac"] / (cfg["bw"] / nchan)
        h = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], nfft, mode=0,
                                               frac_delay_us=frac_us)
        y = orc.convolve(x, h, nfft, pos, neg)
    elif fb:
        # Filterbank (freq_res = 1): DC-centred, swapped output channels
        x = orc.filterbank(x.astype(np.complex128) if fp64 else x, fb)
        nchan *= fb
        ndat_tot //= fb
        freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nchan, swap=True, dc_centred=True)
        h = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], nfft, mode=0,
                                               fp64=fp64)
        y = orc.convolve(x, h, nfft, pos, neg)
    elif fp64:
        h = orc.dedispersion_response_f64(cfg["cf"], cfg["bw"], cfg["dm"], nchan, nfft,
                                          input_nchan=nchan)
        y = orc.convolve(x.astype(np.complex128), h, nfft, pos, neg)
    else:
        h = orc.dedispersion_response(cfg["cf"], cfg["bw"], cfg["dm"], nchan, nfft,
                                      input_nchan=nchan, mode=0)
        y = orc.convolve(x, h, nfft, pos, neg)
    return y, nchan


def block_outputs(b2, raw_blocks, cfg):
    """(in0, nout) of each block: the parts the overlap carry completes."""
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    fb = cfg.get("fb", 0)
    out, in0, carry = [], 0, 0
    for r in raw_blocks:
        nb = r.shape[-1] // 2 if cfg["kind"] == b2.FLOAT_FPT else r.size // (cfg["nchan"] * cfg["npol"] * 2)
        if fb:
            nb //= fb
        ndat = carry + nb
        npart = (ndat - cfg["pos"] - cfg["neg"]) // nk if ndat >= cfg["nfft"] else 0
        out.append((in0, npart * nk))
        in0 += npart * nk
        carry = ndat - npart * nk
    return out


def oracle_subints(orc, b2, raw_blocks, cfg, td_kw):
    """Subint<Fold> over the blocks: each range folds with its own phase into
    its division; closed divisions with data are returned in order as
    (division, first_sample, ndat_folded, profiles, hits)."""
    d, nchan = oracle_detected(orc, b2, raw_blocks, cfg)
    rate = abs(cfg["bw"]) / nchan * 1e6
    pps = (1.0 / rate) / cfg["period"]
    nbin = cfg["nbin"]
    td = orc.TimeDivideOracle(**td_kw)
    subs, cur = [], None

    def close():
        nonlocal cur
        if cur is not None and cur[2] > 0:
            subs.append(tuple(cur))
        cur = None

    for in0, nout in block_outputs(b2, raw_blocks, cfg):
        if nout == 0:
            continue
        start = orc.mjd_add(START, (in0 + cfg["pos"]) / rate)
        for a in orc.subint_block_actions(td, start, nout, rate):
            if a[0] == "close":
                close()
                continue
            _, i0, n, div = a[:4]
            if cur is None:
                cur = [div, in0 + i0, 0, np.zeros((nchan, d.shape[1], nbin), d.dtype),
                       np.zeros(nbin, np.uint32)]
            phi = orc.fold_phi(START, EPOCH, in0 + cfg["pos"] + i0, rate, cfg["period"])
            plan = orc.fold_binplan(phi, pps, n, nbin)
            orc.fold_accumulate(np.ascontiguousarray(d[:, :, in0 + i0:in0 + i0 + n]), plan, nbin,
                                cur[3], cur[4])
            cur[2] += n
    close()
    return subs


def oracle_fold(orc, b2, raw_blocks, cfg, d, nchan):
    npol = cfg["npol"]
    kind = cfg["kind"]
    nfft, pos, neg = cfg["nfft"], cfg["pos"], cfg["neg"]
    nk = nfft - pos - neg
    fb = cfg.get("fb", 0)
    rate = abs(cfg["bw"]) / nchan * 1e6
    pps = (1.0 / rate) / cfg["period"]
    nbin = cfg["nbin"]
    prof = np.zeros((nchan, d.shape[1], nbin), d.dtype)
    hits = np.zeros(nbin, np.uint32)
    in0, carry = 0, 0
    for r in raw_blocks:
        nb = r.shape[-1] // 2 if kind == b2.FLOAT_FPT else r.size // (cfg["nchan"] * npol * 2)
        if fb:
            nb //= fb
        ndat = carry + nb
        npart = (ndat - pos - neg) // nk if ndat >= nfft else 0
        nout = npart * nk
        if nout:
            phi = orc.fold_phi(START, EPOCH, in0 + pos, rate, cfg["period"])
            plan = orc.fold_binplan(phi, pps, nout, nbin)
            orc.fold_accumulate(np.ascontiguousarray(d[:, :, in0:in0 + nout]), plan, nbin,
                                prof, hits)
        in0 += nout
        carry = ndat - nout
    return prof, hits, in0


def make_blocks(rng, cfg, sizes):
    nchan, npol = cfg["nchan"], cfg["npol"]
    blocks = []
    for n in sizes:
        if cfg["kind"] == b2mod().INT8_TFPD:
            v = np.clip(np.round(rng.standard_normal(n * nchan * npol * 2) * 10), -128, 127)
            blocks.append(v.astype(np.int8).view(np.uint8))
        elif cfg["kind"] == b2mod().INT16_TFPD:
            v = np.round(rng.standard_normal(n * nchan * npol * 2) * 300)
            blocks.append(v.astype(np.int16))
        else:
            v = rng.standard_normal((nchan, npol, 2 * n)).astype(np.float32)
            blocks.append(v)
    return blocks


def b2mod():
    import dspsr_b200
    return dspsr_b200


def run_pipeline(ctx, b2, blocks, cfg, host=False):
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], cfg["nfft"],
                       cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                       input_kind=cfg["kind"], lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                       scratch_bytes=cfg.get("scratch", 0),
                       chirp_mode=cfg.get("chirp", b2.CHIRP_REFERENCE),
                       filterbank_nchan=cfg.get("fb", 0), row_length=cfg.get("row", 0),
                       fft_precision=cfg.get("fft", 0))
    pl = b2.Pipeline(ctx, c)
    total = 0
    for r in blocks:
        if cfg["kind"] == b2.FLOAT_FPT:
            n = r.shape[-1] // 2
            total += pl.run(torch.from_numpy(r).cuda(), n, n)
        elif host:
            n = r.size // (cfg["nchan"] * cfg["npol"] * 2)
            total += pl.run_host(r, n)
        else:
            n = r.size // (cfg["nchan"] * cfg["npol"] * 2)
            total += pl.run(torch.from_numpy(r).cuda(), n)
    prof, hits = pl.get_profiles()
    info = pl.info()
    pl.close()
    return prof, hits, total, info


def base_cfg(b2, **kw):
    cfg = dict(cf=1400.0, bw=16.0, dm=5.0, nchan=1, npol=2, nbin=256, period=0.0123,
               state=b2.INTENSITY, kind=b2.INT8_TFPD, lut=b2.bittable8()[0])
    cfg.update(kw)
    # with a filterbank the smearing is that of its output channels
    nchan_conv = cfg["nchan"] * (cfg.get("fb", 0) or 1)
    pos, neg, nfft = b2.dispersion_plan(cfg["cf"], cfg["bw"], cfg["dm"], nchan_conv,
                                        cfg.get("nfft"))
    cfg.update(pos=pos, neg=neg, nfft=nfft)
    return cfg


def profile_scale(rprof, state):
    """Per-(chan, bin) power scale of a folded profile: the profile itself for
    intensity-like products, the total power PP+QQ (or Stokes I) for the
    signed cross products, whose bins are sums with cancellation."""
    if state in (0, 1):
        return np.abs(rprof)
    if state == 2:
        s = rprof[:, 0:1] + rprof[:, 1:2]
    else:
        s = rprof[:, 0:1]
    return np.broadcast_to(s, rprof.shape)


def check(prof, hits, total, rprof, rhits, rtotal, state, rtol=PROFILE_RTOL):
    assert total == rtotal
    assert np.array_equal(hits, rhits)
    scale = profile_scale(rprof.astype(np.float64), state)
    empty = hits == 0
    assert np.all(prof[..., empty] == 0)
    err = np.abs(prof.astype(np.float64) - rprof)[..., ~empty]
    sc = scale[..., ~empty]
    # a bin whose scale is exactly zero (all of a channel's samples there
    # zeroed) must be exactly zero too
    rel = np.divide(err, sc, out=np.where(err == 0, 0.0, np.inf), where=sc > 0)
    assert np.max(rel) < rtol, float(np.max(rel))


CASES = {
    # single-kernel path (nfft 8192), intensity, int8
    "fused8k_int8": dict(dm=5.0),
    # four-step path at the C1 physics (DM 67.99, 16 MHz, nfft 2^17)
    "c1_fourstep": dict(dm=67.99, nfft=1 << 17, nbin=1024, period=0.08933),
    # coherence products with int16 input, 4 channels, four-step 2^14
    "coherence_int16": dict(dm=5.0, bw=64.0, nchan=4, nfft=1 << 14, state=2, kind=1, nbin=128),
    # full Stokes on float FPT input, small scratch (many batches)
    "stokes_float": dict(dm=3.0, bw=32.0, nchan=2, nfft=1 << 15, state=3, kind=2, nbin=512,
                         scratch=8 << 20),
    # one polarisation, intensity, fused 4096
    "onepol_4096": dict(dm=1.0, npol=1, nfft=4096),
    # C2 shape: 64-channel FFT filterbank of 256 MHz, per-channel dedispersion,
    # full Stokes, single-kernel path (DM 50 -> 8192) and four-step (DM 500 -> 2^16)
    "c2_filterbank_8k": dict(dm=50.0, bw=256.0, fb=64, state=3, nbin=2048, period=5.757e-3),
    "c2_filterbank_64k": dict(dm=500.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=2048,
                              period=5.757e-3),
    # a table that is not (x + 0.5) * scale: looked up, not computed
    "c2_fb64k_table": dict(dm=500.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=2048,
                           period=5.757e-3, lut=(np.asarray(__import__("dspsr_b200").bittable8()[0])
                                                 * (1 + 1e-3 * np.cos(np.arange(256)))).astype(np.float32)),
    # the four-step split with 4096-point rows (n1 = 8 and 32 columns)
    "rows4096_2p15": dict(dm=5.0, bw=64.0, nchan=2, nfft=1 << 15, state=2, nbin=256,
                          row=4096),
    "rows4096_2p17": dict(dm=67.99, nfft=1 << 17, nbin=1024, period=0.08933, row=4096),
    # the largest FFT of the multi-stream workload: 2^18 = 32 x 8192 (the
    # 32-row column passes), full Stokes
    "c3_2p18_stokes": dict(dm=100.0, bw=16.0, nfft=1 << 18, state=3, nbin=512, period=0.05),
    # the rows on the tensor cores (three BF16 terms), four channels
    "tensor_rows_4ch": dict(dm=8.0, bw=32.0, nchan=4, nfft=1 << 15, state=3, nbin=256, fft=3),
    "fused8k_table": dict(dm=5.0, lut=(np.asarray(__import__("dspsr_b200").bittable8()[0])
                                       * (1 + 1e-3 * np.sin(np.arange(256)))).astype(np.float32)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_pipeline_matches_oracle_chain(ctx, b2, orc, name):
    cfg = base_cfg(b2, **CASES[name])
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    # three uneven blocks: the carry spans block boundaries
    sizes = [cfg["nfft"] + 3 * nk + 17, 2 * nk - 5, nk + 1234]
    if cfg.get("fb"):
        # whole filterbank transforms per block; fewer parts for the CPU oracle
        fb = cfg["fb"]
        sizes = [(cfg["nfft"] + nk + 17) * fb, (nk - 5) * fb, (nk // 2 + 1234) * fb]
    blocks = make_blocks(rng, cfg, sizes)
    prof, hits, total, info = run_pipeline(ctx, b2, blocks, cfg)
    rprof, rhits, rtotal = oracle_chain(orc, b2, blocks, cfg)
    check(prof, hits, total, rprof, rhits, rtotal, cfg["state"])
    # the FP64-chirp form against the FP64 oracle chain (FP64 response, FFT,
    # detection and sums).  The reference-mode chirp rounds |phase| ~ 1e4 rad
    # to float, which alone moves profiles by ~1e-5, so it is not compared here.
    prof64, hits64, total64, _ = run_pipeline(ctx, b2, blocks, dict(cfg, chirp=b2.CHIRP_FP64))
    rprof64, rhits64, _ = oracle_chain(orc, b2, blocks, cfg, fp64=True)
    check(prof64, hits64, total64, rprof64, rhits64, rtotal, cfg["state"], rtol=PROFILE_RTOL_FP64)


def test_pipeline_host_input_matches_device_input(ctx, b2):
    cfg = base_cfg(b2, dm=67.99, nfft=1 << 17, nbin=1024, period=0.08933)
    rng = np.random.default_rng(1)
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    blocks = make_blocks(rng, cfg, [cfg["nfft"] + 2 * nk, nk + 99])
    a = run_pipeline(ctx, b2, blocks, cfg)
    b = run_pipeline(ctx, b2, blocks, cfg, host=True)
    assert a[2] == b[2]
    assert np.array_equal(a[1], b[1])
    check(a[0], a[1], a[2], b[0].astype(np.float64), b[1], b[2], cfg["state"], rtol=1e-6)


@pytest.mark.parametrize("nfft_mult", [9, 17])
def test_pipeline_host_upload_in_pieces(ctx, b2, nfft_mult):
    """Large host blocks are uploaded in 2 or 4 pieces that overlap the
    kernels; the carried overlap joins them, so the result equals the
    device-input run."""
    cfg = base_cfg(b2, dm=20.0, nfft=1 << 15, nbin=512, period=0.08933)
    rng = np.random.default_rng(nfft_mult)
    blocks = make_blocks(rng, cfg, [nfft_mult * cfg["nfft"] + 12345, 3 * cfg["nfft"] + 7,
                                    nfft_mult * cfg["nfft"]])
    a = run_pipeline(ctx, b2, blocks, cfg)
    b = run_pipeline(ctx, b2, blocks, cfg, host=True)
    assert a[2] == b[2]
    assert np.array_equal(a[1], b[1])
    check(a[0], a[1], a[2], b[0].astype(np.float64), b[1], b[2], cfg["state"], rtol=1e-6)


def test_pipeline_async_profiles_follow_each_block(ctx, b2):
    """get_profiles_async queued after each host block, and waited for once
    the next block is already queued, gives the profiles a synchronous
    get_profiles gives after the same blocks."""
    cfg = base_cfg(b2, dm=20.0, nfft=1 << 15, nbin=512, period=0.08933)
    rng = np.random.default_rng(5)
    blocks = make_blocks(rng, cfg, [9 * cfg["nfft"] + 333, 5 * cfg["nfft"], 9 * cfg["nfft"],
                                    2 * cfg["nfft"] + 1])

    def pipe():
        c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"],
                           cfg["nfft"], cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"],
                           state=cfg["state"], input_kind=cfg["kind"], lut=cfg["lut"],
                           start_mjd=START, epoch_mjd=EPOCH)
        return b2.Pipeline(ctx, c)

    nsamp = [r.size // (cfg["nchan"] * cfg["npol"] * 2) for r in blocks]
    pl = pipe()
    want = []
    for r, n in zip(blocks, nsamp):
        pl.run_host(r, n)
        want.append(pl.get_profiles())
    pl.close()
    pl = pipe()
    bufs = [pl.profile_buffers(), pl.profile_buffers()]
    got = []
    for i, (r, n) in enumerate(zip(blocks, nsamp)):
        pl.run_host(r, n)
        if i:
            pl.wait_profiles()
            got.append(tuple(x.copy() for x in bufs[(i - 1) % 2]))
        pl.get_profiles_async(*bufs[i % 2])
    pl.wait_profiles()
    got.append(tuple(x.copy() for x in bufs[(len(blocks) - 1) % 2]))
    pl.close()
    for (gp, gh), (wp, wh) in zip(got, want):
        assert np.array_equal(gh, wh)
        assert np.allclose(gp, wp, rtol=1e-6, atol=1e-6 * np.abs(wp).max())


def test_pipeline_short_blocks_only_carry(ctx, b2):
    """Blocks shorter than one FFT fold nothing and are carried forward."""
    cfg = base_cfg(b2, dm=5.0)
    rng = np.random.default_rng(2)
    blocks = make_blocks(rng, cfg, [1000, 2000, 3000])
    prof, hits, total, info = run_pipeline(ctx, b2, blocks, cfg)
    assert total == 0 and hits.sum() == 0
    blocks = make_blocks(rng, cfg, [1000, 2000, 3000, 9000])
    prof, hits, total, info = run_pipeline(ctx, b2, blocks, cfg)
    assert total > 0 and hits.sum() == total


def test_pipeline_restores_dispersed_pulse(ctx, b2):
    """A pulse train dispersed by an independent FP64 inverse chirp (numpy FFT
    of the whole block) is restored: the folded profile peaks at the pulse
    phase with the expected duty cycle."""
    from dspsr_b200 import synth
    cfg = base_cfg(b2, dm=67.99, nfft=1 << 17, nbin=256, period=0.005)
    raw, truth = synth.dispersed_pulse_train(ndat=1 << 21, cf=cfg["cf"], bw=cfg["bw"], dm=cfg["dm"],
                                             period=cfg["period"], duty=0.03, snr=50.0, sigma=10.0,
                                             seed=3, start_mjd=START, epoch_mjd=EPOCH)
    prof, hits, total, info = run_pipeline(ctx, b2, [raw], cfg)
    p = prof[0, 0] / np.maximum(hits, 1)
    on = np.argmax(p)
    assert abs(((on + 0.5) / cfg["nbin"] - truth["phase"] + 0.5) % 1.0 - 0.5) < 0.03
    assert (p.max() - np.median(p)) > 20 * np.std(p[np.abs(np.arange(256) - on) > 30])


def dada_keys(cfg, ndat_hint=None):
    """A header for cfg's observation whose start time is START."""
    keys = {"HDR_VERSION": "1.0", "TELESCOPE": "PKS", "SOURCE": "J0437-4715",
            "INSTRUMENT": "CASPSR", "FREQ": cfg["cf"], "BW": cfg["bw"], "NCHAN": cfg["nchan"],
            "NPOL": cfg["npol"], "NBIT": 8 if cfg["kind"] == 0 else 16, "NDIM": 2,
            "TSAMP": cfg["nchan"] / abs(cfg["bw"]), "UTC_START": "2023-02-25-01:00:00",
            "PICOSECONDS": 250000000000, "OBS_OFFSET": 0}
    return keys


def run_file(ctx, b2, path, cfg, block_ndat, start=0, nsamp=0):
    with b2.DADAFile(path) as f:
        c = f.pipeline_config(cfg["dm"], cfg["nfft"], cfg["pos"], cfg["neg"], cfg["nbin"],
                              cfg["period"], state=cfg["state"], lut=cfg["lut"],
                              epoch_mjd=EPOCH, filterbank_nchan=cfg.get("fb", 0))
        assert (c.start_day, c.start_sec, c.start_frac) == START
        pl = b2.Pipeline(ctx, c)
        nread, nfold = pl.run_dada(f, block_ndat, start, nsamp)
        prof, hits = pl.get_profiles()
        pl.close()
    return prof, hits, nread, nfold


@pytest.mark.parametrize("name,kw,block", [
    ("int8_4chan", dict(dm=20.0, bw=64.0, nchan=4, nfft=1 << 16, nbin=256, period=0.00557),
     2 * (1 << 16) + 123),
    ("int16_coherence", dict(dm=5.0, bw=32.0, nchan=2, nfft=1 << 13, state=2, kind=1, nbin=128),
     50000),
    ("filterbank16", dict(dm=30.0, bw=64.0, fb=16, nfft=1 << 13, state=3, nbin=512,
                          period=0.0041), 16 * 9000),
])
def test_pipeline_reads_dada_file(ctx, b2, orc, tmp_path, name, kw, block):
    """A recorded DADA file through pipeline_run_dada (blocks read into two
    pinned buffers, each read overlapping the previous block's upload and
    kernels): the same profiles as run_host with the same blocks, and the
    oracle chain's within PROFILE_RTOL."""
    cfg = base_cfg(b2, **kw)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    unit = cfg.get("fb", 0) or 1
    ndat = 5 * cfg["nfft"] * unit + 999
    raw = make_blocks(rng, cfg, [ndat])[0]
    path = tmp_path / f"{name}.dada"
    b2.write_dada(path, dada_keys(cfg), raw)
    prof, hits, nread, nfold = run_file(ctx, b2, path, cfg, block)
    used = ndat - ndat % unit
    assert nread == used
    bps = cfg["nchan"] * cfg["npol"] * 2
    flat = raw.reshape(-1)[: used * bps]
    blocks = [flat[i * bps:(i + block) * bps] for i in range(0, used, block)]
    hprof, hhits, htotal, _ = run_pipeline(ctx, b2, blocks, cfg, host=True)
    assert nfold == htotal > 0
    # the fold's float sums are not order-deterministic between runs
    check(prof, hits, nfold, hprof.astype(np.float64), hhits, htotal, cfg["state"], rtol=1e-6)
    rprof, rhits, rtotal = oracle_chain(orc, b2, blocks, cfg)
    check(prof, hits, nfold, rprof, rhits, rtotal, cfg["state"])


def test_pipeline_dada_window_and_rejects(ctx, b2, tmp_path):
    """start_sample / nsamp select a window of the file; a file whose shape
    differs from the pipeline's, or a block that splits a filterbank
    transform, is refused."""
    cfg = base_cfg(b2, dm=5.0, nchan=2, bw=32.0, nfft=1 << 13)
    rng = np.random.default_rng(5)
    ndat = 6 * cfg["nfft"]
    raw = make_blocks(rng, cfg, [ndat])[0]
    path = tmp_path / "w.dada"
    b2.write_dada(path, dada_keys(cfg), raw)
    prof, hits, nread, nfold = run_file(ctx, b2, path, cfg, 10000, start=4000,
                                        nsamp=3 * cfg["nfft"])
    assert nread == 3 * cfg["nfft"]
    bps = cfg["nchan"] * cfg["npol"] * 2
    win = raw.reshape(-1)[4000 * bps:(4000 + nread) * bps]
    blocks = [win[i * bps:(i + 10000) * bps] for i in range(0, nread, 10000)]
    hprof, hhits, htotal, _ = run_pipeline(ctx, b2, blocks, cfg, host=True)
    check(prof, hits, nfold, hprof.astype(np.float64), hhits, htotal, cfg["state"], rtol=1e-6)
    # past the end: nothing read
    assert run_file(ctx, b2, path, cfg, 10000, start=ndat + 5)[2:] == (0, 0)
    # shape mismatch: the pipeline takes 4 channels, the file has 2
    with b2.DADAFile(path) as f:
        c = f.pipeline_config(cfg["dm"], cfg["nfft"], cfg["pos"], cfg["neg"], 64, 0.01)
        c.nchan = 4
        pl = b2.Pipeline(ctx, c)
        with pytest.raises(b2.B200Error, match="NCHAN=2"):
            pl.run_dada(f, 10000)
        pl.close()
        pos, neg, nfft = b2.dispersion_plan(cfg["cf"], cfg["bw"], cfg["dm"], 32, 4096)
        c = f.pipeline_config(cfg["dm"], nfft, pos, neg, 64, 0.01, filterbank_nchan=16)
        pl = b2.Pipeline(ctx, c)
        with pytest.raises(b2.B200Error, match="multiple of 16"):
            pl.run_dada(f, 10008)
        pl.close()


def run_subints(ctx, b2, blocks, cfg, td_kw, slots=0, pop=False, host=False, interchannel=0):
    """The pipeline with sub-integrations: closed divisions as (info, prof, hits)."""
    kw = dict(subint_seconds=td_kw.get("seconds", 0.0), subint_turns=td_kw.get("turns", 0.0),
              subint_slots=slots, interchannel=interchannel)
    if "reference_epoch" in td_kw:
        kw["subint_epoch"] = td_kw["reference_epoch"]
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], cfg["nfft"],
                       cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                       input_kind=cfg["kind"], lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                       filterbank_nchan=cfg.get("fb", 0), **kw)
    pl = b2.Pipeline(ctx, c)
    got = []
    if not pop:
        pl.set_unloader(lambda info, prof, hits: got.append((info, prof, hits)))
    for r in blocks:
        n = r.size // (cfg["nchan"] * cfg["npol"] * 2)
        if host:
            pl.run_host(r, n)
        else:
            pl.run(torch.from_numpy(r).cuda(), n)
        if pop:
            while pl.subints_ready():
                got.append(pl.pop_subint())
    pl.finish()
    while pop and pl.subints_ready():
        got.append(pl.pop_subint())
    with pytest.raises(b2.B200Error, match="sub-integrations"):
        pl.get_profiles()
    pl.close()
    return got


def check_subints(got, want, cfg, rate):
    assert len(got) == len(want) > 1
    for (info, prof, hits), (div, first, n, rprof, rhits) in zip(got, want):
        assert (info["division"], info["first_sample"], info["ndat_folded"]) == (div, first, n)
        assert info["integration_length"] == n / rate
        check(prof, hits, int(hits.sum()), rprof.astype(np.float64), rhits, int(rhits.sum()),
              cfg["state"])


SUBINT_CASES = {
    # seconds: three blocks of ~3.3 ms at 16 MHz over 1 ms divisions, fused path
    "seconds_fused": (dict(dm=5.0, nbin=128, period=0.00123), dict(seconds=0.001), 0),
    # single-pulse mode (one turn per division), four-step path, Stokes, 2 channels
    "turns_fourstep": (dict(dm=3.0, bw=32.0, nchan=2, nfft=1 << 15, state=3, nbin=256,
                            period=0.0009), dict(turns=1.0, period=0.0009), 16),
    # a reference epoch and a 16-channel filterbank in front
    "epoch_filterbank": (dict(dm=30.0, bw=64.0, fb=16, nfft=1 << 13, state=3, nbin=256,
                              period=0.0041), dict(seconds=0.002,
                                                   reference_epoch=(60000, 3599, 0.9993)), 8),
}


@pytest.mark.parametrize("name", list(SUBINT_CASES))
def test_pipeline_subints_match_oracle(ctx, b2, orc, name):
    """Subint<Fold>: every closed division's profiles, hits and sample count
    against the oracle's TimeDivide + fold, delivered through the unloader;
    the same through pop_subint from host input."""
    kw, td_kw, slots = SUBINT_CASES[name]
    cfg = base_cfg(b2, **kw)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    unit = cfg.get("fb", 0) or 1
    sizes = [(cfg["nfft"] + 3 * nk + 17) * unit, (2 * nk - 5) * unit, (nk + 1234) * unit]
    blocks = make_blocks(rng, cfg, sizes)
    td = dict(td_kw)
    if "turns" in td:
        td["period"] = cfg["period"]
    got = run_subints(ctx, b2, blocks, cfg, td, slots=slots)
    want = oracle_subints(orc, b2, blocks, cfg, td)
    rate = abs(cfg["bw"]) / (cfg["nchan"] * unit) * 1e6
    check_subints(got, want, cfg, rate)
    got2 = run_subints(ctx, b2, blocks, cfg, td, slots=slots, pop=True, host=True)
    check_subints(got2, want, cfg, rate)


def test_pipeline_subint_slots_exhausted(ctx, b2):
    """A block that opens more divisions than there are free slots is refused
    before any work is queued, and the pipeline goes on once slots free up."""
    cfg = base_cfg(b2, dm=5.0, nbin=64, period=0.00123)
    rng = np.random.default_rng(3)
    blocks = make_blocks(rng, cfg, [5 * cfg["nfft"]])
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], cfg["nfft"],
                       cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"], lut=cfg["lut"],
                       start_mjd=START, epoch_mjd=EPOCH, subint_seconds=0.0005, subint_slots=2)
    pl = b2.Pipeline(ctx, c)
    n = blocks[0].size // 4
    with pytest.raises(b2.B200Error, match="slots are free"):
        pl.run(torch.from_numpy(blocks[0]).cuda(), n)
    pl.close()
    with pytest.raises(b2.B200Error, match="one positive length"):
        b2.Pipeline(ctx, b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], 1, 2, cfg["nfft"],
                                        cfg["pos"], cfg["neg"], 64, 0.001, subint_seconds=1.0,
                                        subint_turns=1.0))


@pytest.mark.parametrize("kind,perturb", [(0, False), (1, False), (0, True)])
def test_pipeline_fused_filterbank_matches_stage(ctx, b2, orc, kind, perturb):
    """The 64-channel filterbank computed inside the column pass (C2's shape)
    against the filterbank as a stage of its own and against the oracle
    chain, over blocks whose carry crosses parts, from device and host
    memory; perturb: an 8-bit table that is not affine, looked up from the
    pass's replicated shared-memory copies."""
    cfg = base_cfg(b2, dm=500.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=512,
                   period=5.757e-3, kind=kind)
    if perturb:
        cfg["lut"] = (np.asarray(cfg["lut"], np.float32)
                      * (1 + 1e-3 * np.cos(np.arange(256)))).astype(np.float32)
    rng = np.random.default_rng(77 + kind)
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    blocks = make_blocks(rng, cfg, [(cfg["nfft"] + 2 * nk + 321) * 64, (nk - 17) * 64,
                                    (3 * nk + 5) * 64])

    def run(fused, host=False):
        c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], 1, 2, cfg["nfft"], cfg["pos"],
                           cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                           input_kind=kind, lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                           filterbank_nchan=64, fused_filterbank=0 if fused else -1)
        pl = b2.Pipeline(ctx, c)
        tot = 0
        for r in blocks:
            n = r.size // 4
            tot += pl.run_host(r, n) if host else pl.run(torch.from_numpy(r).cuda(), n)
        prof, hits = pl.get_profiles()
        pl.close()
        return prof, hits, tot

    fused = run(True)
    stage = run(False)
    check(fused[0], fused[1], fused[2], stage[0].astype(np.float64), stage[1], stage[2],
          cfg["state"], rtol=2e-6)
    rprof, rhits, rtotal = oracle_chain(orc, b2, blocks, cfg)
    check(fused[0], fused[1], fused[2], rprof, rhits, rtotal, cfg["state"])
    hostrun = run(True, host=True)
    check(hostrun[0], hostrun[1], hostrun[2], fused[0].astype(np.float64), fused[1], fused[2],
          cfg["state"], rtol=2e-6)


def oracle_interchannel_chain(orc, b2, raw_blocks, cfg):
    """DedispersionPipe with -K: the convolution's voltages pass SampleDelay
    (with its InputBuffering of total_delay samples) before detection and the
    fold; the fold's phase is taken at each block's first SampleDelay output,
    zero_delay samples later than the convolution's."""
    delays = {}
    y, nchan = oracle_voltages(orc, b2, raw_blocks, cfg, interchannel=delays)
    rate = abs(cfg["bw"]) / nchan * 1e6
    pps = (1.0 / rate) / cfg["period"]
    nbin = cfg["nbin"]
    nout = 4 if cfg["state"] in (2, 3) else (2 if cfg["state"] == 1 else 1)
    prof = np.zeros((nchan, nout, nbin), np.float32)
    hits = np.zeros(nbin, np.uint32)
    g0, total = 0, 0
    tot = delays["total_delay"]
    for in0, n in block_outputs(b2, raw_blocks, cfg):
        seg = y[:, :, g0:in0 + n]
        out = orc.sample_delay_block(seg, delays["applied"], tot)
        m = out.shape[2]
        if m:
            d = orc.detect(np.ascontiguousarray(out), cfg["state"])
            phi = orc.fold_phi(START, EPOCH, g0 + cfg["pos"] + delays["zero_delay"], rate,
                               cfg["period"])
            plan = orc.fold_binplan(phi, pps, m, nbin)
            orc.fold_accumulate(np.ascontiguousarray(d), plan, nbin, prof, hits)
        g0 += m
        total += m
    return prof, hits, total, delays


@pytest.mark.parametrize("name,kw", [
    # C2's shape: 64-channel filterbank (computed in the column pass), DM 500
    # (DM 5: at C2's DM 500 the channels span 0.39 s, more data than the
    # oracle should chew through here)
    ("c2_fb64", dict(dm=5.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=1024,
                     period=5.757e-3)),
    # eight int16 channels straight from the input, coherence products
    ("nchan8_int16", dict(dm=10.0, bw=64.0, nchan=8, nfft=1 << 14, state=2, kind=1,
                          nbin=256, period=0.0031)),
])
def test_pipeline_interchannel_matches_oracle(ctx, b2, orc, name, kw):
    """-K: fractional delays in the response and SampleDelay's whole-sample
    shifts before the fold, against the oracle chain; the channels' pulse
    then lines up."""
    cfg = base_cfg(b2, **kw)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    unit = cfg.get("fb", 0) or 1
    blocks = make_blocks(rng, cfg, [(cfg["nfft"] + 2 * nk + 77) * unit, (nk - 3) * unit,
                                    (2 * nk + 999) * unit])
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], cfg["nfft"],
                       cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                       input_kind=cfg["kind"], lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                       filterbank_nchan=cfg.get("fb", 0), interchannel=1)
    pl = b2.Pipeline(ctx, c)
    total = 0
    for r in blocks:
        total += pl.run(torch.from_numpy(r).cuda(), r.size // (cfg["nchan"] * cfg["npol"] * 2))
    prof, hits = pl.get_profiles()
    pl.close()
    rprof, rhits, rtotal, delays = oracle_interchannel_chain(orc, b2, blocks, cfg)
    assert delays["total_delay"] > 0
    check(prof, hits, total, rprof, rhits, rtotal, cfg["state"])


def test_pipeline_interchannel_aligns_channels(ctx, b2):
    """A pulse train dispersed across 64 MHz (DM 30: 5.8 ms across the band,
    more than the 5 ms period) through a 16-channel filterbank: without -K
    the channels' profiles peak at phases spread by the inter-channel delays,
    with -K they line up.  (The DC-centred filterbank's channel 8 holds the
    Nyquist bin: half of it is the other band edge, so it is left out.)"""
    from dspsr_b200 import synth
    cf, bw, dm, period, nbin = 1400.0, 64.0, 30.0, 0.005, 256
    raw, truth = synth.dispersed_pulse_train(ndat=1 << 22, cf=cf, bw=bw, dm=dm, period=period,
                                             duty=0.03, snr=30.0, sigma=10.0, seed=11,
                                             start_mjd=START, epoch_mjd=EPOCH)
    pos, neg, nfft = b2.dispersion_plan(cf, bw, dm, 16, 1 << 14)

    def peaks(interchannel):
        c = b2.make_config(cf, bw, dm, 1, 2, nfft, pos, neg, nbin, period, start_mjd=START,
                           epoch_mjd=EPOCH, filterbank_nchan=16, interchannel=interchannel)
        pl = b2.Pipeline(ctx, c)
        pl.run(torch.from_numpy(raw).cuda(), raw.size // 4)
        prof, hits = pl.get_profiles()
        pl.close()
        p = prof[:, 0] / np.maximum(hits, 1)
        return np.delete(np.argmax(p, axis=1), 8)

    def spread(b):
        # circular spread of the peak bins around their circular mean
        ang = 2 * np.pi * b / nbin
        mean = np.angle(np.mean(np.exp(1j * ang)))
        d = np.angle(np.exp(1j * (ang - mean))) * nbin / (2 * np.pi)
        return np.max(np.abs(d))

    # the pulse is 0.03 x 256 = 7.7 bins wide: its peak bin wanders inside it
    assert spread(peaks(0)) > 20
    assert spread(peaks(1)) <= 5


def oracle_interchannel_subints(orc, b2, raw_blocks, cfg, td_kw):
    """-K and sub-integrations together: SampleDelay's outputs of each block
    (starting zero_delay samples after the convolution's) are divided by
    TimeDivide and folded range by range."""
    delays = {}
    y, nchan = oracle_voltages(orc, b2, raw_blocks, cfg, interchannel=delays)
    rate = abs(cfg["bw"]) / nchan * 1e6
    pps = (1.0 / rate) / cfg["period"]
    nbin = cfg["nbin"]
    nout = 4 if cfg["state"] in (2, 3) else (2 if cfg["state"] == 1 else 1)
    td = orc.TimeDivideOracle(**td_kw)
    subs, cur = [], None
    tot, zero = delays["total_delay"], delays["zero_delay"]

    def close():
        nonlocal cur
        if cur is not None and cur[2] > 0:
            subs.append(tuple(cur))
        cur = None

    g0 = 0
    for in0, n in block_outputs(b2, raw_blocks, cfg):
        out = orc.sample_delay_block(y[:, :, g0:in0 + n], delays["applied"], tot)
        m = out.shape[2]
        if m == 0:
            continue
        d = orc.detect(np.ascontiguousarray(out), cfg["state"])
        start = orc.mjd_add(START, (g0 + cfg["pos"] + zero) / rate)
        for a in orc.subint_block_actions(td, start, m, rate):
            if a[0] == "close":
                close()
                continue
            _, i0, k, div = a[:4]
            if cur is None:
                cur = [div, g0 + i0, 0, np.zeros((nchan, nout, nbin), np.float32),
                       np.zeros(nbin, np.uint32)]
            phi = orc.fold_phi(START, EPOCH, g0 + cfg["pos"] + zero + i0, rate, cfg["period"])
            plan = orc.fold_binplan(phi, pps, k, nbin)
            orc.fold_accumulate(np.ascontiguousarray(d[:, :, i0:i0 + k]), plan, nbin, cur[3],
                                cur[4])
            cur[2] += k
        g0 += m
    close()
    return subs


def test_pipeline_interchannel_with_subints(ctx, b2, orc):
    """-K, sub-integrations and host uploads in pieces at once (a 64-channel
    filterbank computed in the column pass): every division against the
    oracle."""
    cfg = base_cfg(b2, dm=5.0, bw=256.0, fb=64, nfft=1 << 16, state=3, nbin=256,
                   period=5.757e-3)
    rng = np.random.default_rng(99)
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    blocks = make_blocks(rng, cfg, [(cfg["nfft"] + 2 * nk + 77) * 64, (nk - 3) * 64,
                                    (2 * nk + 999) * 64])
    td = dict(seconds=0.02)
    got = run_subints(ctx, b2, blocks, cfg, td, slots=8, host=True, interchannel=1)
    want = oracle_interchannel_subints(orc, b2, blocks, cfg, td)
    check_subints(got, want, cfg, abs(cfg["bw"]) / 64 * 1e6)


def oracle_sk_chain(orc, b2, raw_blocks, cfg, M, std_devs=3.0):
    """LoadToFold with coherent dedispersion and SpectralKurtosis
    (LoadToFold1.C:310-351): SK statistics of the zero-DM input (the input
    samples aligned with the convolution's output), the mask applied to the
    dedispersed voltages (SpectralKurtosis.C:1465-1566), detection, and the
    fold of zeroed data (Fold.C:895-930) over the ranges SpectralKurtosis
    hands on per block (whole M-sample blocks, the rest carried)."""
    y, nchan = oracle_voltages(orc, b2, raw_blocks, cfg)
    nchan0, npol = cfg["nchan"], cfg["npol"]
    raw = np.concatenate([r.reshape(-1) for r in raw_blocks])
    if cfg["kind"] == b2.INT8_TFPD:
        ndat_tot = raw.size // (nchan0 * npol * 2)
        x = orc.unpack8(raw, ndat_tot, nchan0, npol, 2, cfg["lut"])
    else:
        ndat_tot = raw.size // (nchan0 * npol * 2)
        x = orc.unpack16(raw, ndat_tot, nchan0, npol, 2, False)
    x = x.view(np.complex64).reshape(nchan0, npol, ndat_tot)
    if cfg.get("fb"):
        x = orc.filterbank(x, cfg["fb"])
    pos = cfg["pos"]
    ntot = y.shape[2]
    zdm = np.ascontiguousarray(x[:, :, pos:pos + ntot])
    lo, hi = orc.sk_limits(M, 1, std_devs, npol)
    nsk = (ntot // M) * M
    sums, counts, mask, masked = orc.sk(zdm, M, lo, hi, ndat=nsk)
    v = y.copy()
    for b in range(nsk // M):
        v[mask[b].astype(bool), :, b * M:(b + 1) * M] = 0
    d = orc.detect(v, cfg["state"])
    rate = abs(cfg["bw"]) / nchan * 1e6
    pps = (1.0 / rate) / cfg["period"]
    nbin = cfg["nbin"]
    prof = np.zeros((nchan, d.shape[1], nbin), d.dtype)
    hits = np.zeros(nbin, np.uint32)
    s0, carry = 0, 0
    for (_, nout) in block_outputs(b2, raw_blocks, cfg):
        ln = carry + nout
        out_n = (ln // M) * M
        if out_n:
            phi = orc.fold_phi(START, EPOCH, s0 + pos, rate, cfg["period"])
            plan = orc.fold_binplan(phi, pps, out_n, nbin)
            orc.fold_accumulate_zeroed(np.ascontiguousarray(d[:, :, s0:s0 + out_n]), plan, nbin,
                                       prof, hits)
        s0 += out_n
        carry = ln - out_n
    return prof, hits, s0, int(mask.sum()), mask.size


@pytest.mark.parametrize("name,kw,M", [
    ("sk_c1_fourstep", dict(dm=67.99, nfft=1 << 17, nbin=1024, period=0.08933), 1024),
    ("sk_stokes_4ch", dict(dm=5.0, bw=64.0, nchan=4, nfft=1 << 14, state=3, nbin=128), 256),
    ("sk_filterbank", dict(dm=50.0, bw=256.0, fb=64, state=3, nbin=512, period=5.757e-3), 128),
])
def test_pipeline_sk_stage_matches_oracle(ctx, b2, orc, name, kw, M):
    """SpectralKurtosis between the convolution and detection, on int8 data
    with RFI bursts: the mask, profiles and hits of the whole chain against
    the oracle chain; hits exact (per non-zeroed channel sample), profiles
    within 1e-5."""
    cfg = base_cfg(b2, **kw)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    fb = cfg.get("fb", 0) or 1
    sizes = [(cfg["nfft"] + 2 * nk + 17) * fb, (nk - 5) * fb, (nk + 1234) * fb]
    blocks = make_blocks(rng, cfg, sizes)
    # impulsive RFI: a few bursts of large values in the raw samples
    for r in blocks:
        v = r.view(np.int8).reshape(-1)
        for _ in range(3):
            t0 = int(rng.integers(0, v.size - 4096))
            v[t0:t0 + int(rng.integers(256, 4096))] = rng.integers(-127, 128, 1)[0]
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], cfg["nfft"],
                       cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"], state=cfg["state"],
                       input_kind=cfg["kind"], lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                       filterbank_nchan=cfg.get("fb", 0), sk_M=M)
    pl = b2.Pipeline(ctx, c)
    tot = 0
    for r in blocks:
        tot += pl.run(torch.from_numpy(r).cuda(), r.size // (cfg["nchan"] * cfg["npol"] * 2))
    prof, hits = pl.get_profiles()
    zapped, tested = pl.sk_counts()
    pl.close()
    rprof, rhits, rtotal, rzap, rtested = oracle_sk_chain(orc, b2, blocks, cfg, M)
    assert tested == rtested and zapped == rzap, (zapped, rzap, tested, rtested)
    assert rzap > 0
    check(prof, hits, tot, rprof, rhits, rtotal, cfg["state"])


def test_pipeline_sk_stage_with_rfi_proposer(ctx, b2):
    """The RFI-mask proposer in front of the pipeline's SK stage: a proposer
    that is never confident (p = 0.5 everywhere) defers every cell to SK, so
    hits equal the SK-only pipeline's exactly and profiles to the rounding of
    the fold's atomic sums (their order differs from run to run); one that is
    sure of RFI everywhere (p ~ 1) zaps every block, so nothing is folded."""
    cfg = base_cfg(b2, dm=5.0, bw=64.0, nchan=4, nfft=1 << 14, state=3, nbin=128)
    rng = np.random.default_rng(31)
    nk = cfg["nfft"] - cfg["pos"] - cfg["neg"]
    blocks = make_blocks(rng, cfg, [cfg["nfft"] + 3 * nk + 17, 2 * nk - 5])
    for r in blocks:
        v = r.view(np.int8).reshape(-1)
        v[1000:5000] = 90                                   # a burst SK flags
    M = 256

    def run(bias=None):
        c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"],
                           cfg["nfft"], cfg["pos"], cfg["neg"], cfg["nbin"], cfg["period"],
                           state=cfg["state"], lut=cfg["lut"], start_mjd=START, epoch_mjd=EPOCH,
                           sk_M=M)
        pl = b2.Pipeline(ctx, c)
        pr = None
        if bias is not None:
            pr = b2.RfiProposer(ctx, cfg["nchan"], M, max_npart=4096)
            p = np.zeros_like(pr.params())
            p[-1] = bias                                     # the head's bias alone
            pr.set_params(p)
            pl.set_rfi_proposer(pr, confidence=0.9)
        tot = 0
        for r in blocks:
            tot += pl.run(torch.from_numpy(r).cuda(), r.size // (cfg["nchan"] * 4))
        prof, hits = pl.get_profiles()
        zap, tested = pl.sk_counts()
        pl.close()
        if pr is not None:
            pr.close()
        return prof, hits, tot, zap

    p0, h0, t0, z0 = run()
    assert z0 > 0
    p1, h1, t1, z1 = run(bias=0.0)
    assert z1 == z0
    # Stokes Q, U, V bins are sums with cancellation: their rounding is
    # measured against the bin's Stokes I
    check(p1, h1, t1, p0, h0, t0, state=cfg["state"], rtol=1e-6)
    p2, h2, t2, _ = run(bias=20.0)
    assert t2 == t0 and h2.sum() == 0 and np.all(p2 == 0)
