"""SpectralKurtosis: SKLimits thresholds (host rule, no GPU) and the fused
compute / detect / mask kernel (GPU) against the CPU oracle.

Bars: thresholds identical as floats to the oracle's independent restatement
(Romberg-integrated there, Gauss-Kronrod here); S1/S2 sums, counts, mask and
masked voltages bit-exact."""
import math

import numpy as np
import pytest


# ---------------------------------------------------------------- thresholds (CPU)

LIMIT_CASES = [(M, Nd, sd, nt) for M in (8, 32, 128, 1000, 1024, 8192, 32767)
               for Nd in (1, 4) for sd in (3.0,) for nt in (1, 2)] + \
              [(128, 1, 2.0, 1), (128, 1, 4.0, 2), (256, 16, 3.0, 1), (64, 2, 5.0, 1)]


@pytest.mark.parametrize("M,Nd,sd,nt", LIMIT_CASES)
def test_sk_limits_match_oracle(b2, orc, M, Nd, sd, nt):
    assert b2.sk_limits(M, Nd, sd, nt) == orc.sk_limits(M, Nd, sd, nt)


@pytest.mark.parametrize("M", [32768, 65536, 1 << 20])
def test_sk_limits_gaussian_branch(b2, M):
    # M >= 32768: 1 -+ sqrt(4/M) * sigma (SKLimits.C:152-160); ntest 1 keeps sigma
    lo, hi = b2.sk_limits(M, 1, 3.0, 1)
    f = math.sqrt(4.0 / M) * 3.0
    assert abs(float(lo) - (1 - f)) <= 1e-7 and abs(float(hi) - (1 + f)) <= 1e-7


def test_sk_limits_invalid(b2):
    for M in (0, 1):
        with pytest.raises(b2.B200Error) as e:
            b2.sk_limits(M)
        assert e.value.code == b2._capi.EINVAL
    # M = 3 needs a Pearson type I density, which the reference rejects too
    with pytest.raises(b2.B200Error) as e:
        b2.sk_limits(3)
    assert e.value.code == b2._capi.ESTATE


@pytest.mark.parametrize("M,Nd", [(128, 1), (1024, 1), (64, 4)])
def test_sk_limits_upper_tail_rate(b2, M, Nd):
    """Monte-Carlo pin: for Gaussian noise the SK estimator exceeds the upper
    threshold with probability pcer/2 (3 sigma, one test: 1.3499e-3).  The
    lower tail is not pinned: the Pearson approximation is loose there."""
    lo, hi = b2.sk_limits(M, Nd, 3.0, 1)
    rng = np.random.default_rng(M + Nd)
    nblk, chunk = 300_000, max(1, 8_000_000 // M)
    over = 0
    for b0 in range(0, nblk, chunk):
        intens = rng.gamma(Nd, 1.0, size=(min(chunk, nblk - b0), M))
        s1 = intens.sum(1)
        s2 = (intens * intens).sum(1)
        v = (M * Nd + 1) / (M - 1) * (M * s2 / (s1 * s1) - 1)
        over += int((v > hi).sum())
    expect = nblk * (1 - math.erf(3 / math.sqrt(2))) / 2
    assert abs(over - expect) < 5 * math.sqrt(expect), (over, expect)


def test_oracle_sk_closed_forms(orc):
    """Constant-power blocks give V = 0 (zapped below any positive lower
    threshold); all-zero blocks count zero samples when zeros are invalid and
    are then left alone; one or two counted samples are always zapped."""
    M, nchan, npol = 64, 3, 2
    x = np.ones((nchan, npol, 4 * M), np.complex64)
    x[1, :, M:2 * M] = 0
    x[2, :, 2 * M:3 * M] = 0
    x[2, :, 2 * M] = 1 + 1j
    lo, hi = orc.sk_limits(M, 1, 3.0, npol)
    sums, counts, mask, out = orc.sk(x, M, lo, hi, zero_is_valid=False)
    assert counts[1, 1] == 0 and mask[1, 1] == 0
    assert counts[2, 2] == 1 and mask[2, 2] == 1
    assert mask[0, 0] == 1           # V = 0 < lower
    np.testing.assert_array_equal(out[2, :, 2 * M:3 * M], 0)
    np.testing.assert_array_equal(out[1, :, M:2 * M], 0)


# ---------------------------------------------------------------- kernel (GPU)

def _voltages(rng, nchan, npol, span, M, zero_blocks=True):
    x = (rng.standard_normal((nchan, npol, span)) +
         1j * rng.standard_normal((nchan, npol, span))).astype(np.complex64)
    nblk = span // M
    if nblk == 0:
        return x
    # RFI: bright bursts, a constant-amplitude tone, zero blocks, sparse blocks
    for k in range(max(1, nblk * nchan // 6)):
        c, b = rng.integers(nchan), rng.integers(nblk)
        kind = k % 4
        seg = slice(b * M, (b + 1) * M)
        if kind == 0:
            x[c, :, seg] *= 6.0
            x[c, :, b * M:b * M + M // 4] *= 4.0
        elif kind == 1:
            t = np.arange(M)
            x[c, 0, seg] = (3 * np.exp(2j * np.pi * 0.1 * t)).astype(np.complex64)
        elif kind == 2 and zero_blocks:
            x[c, :, seg] = 0
        elif kind == 3 and zero_blocks:
            x[c, :, seg] = 0
            x[c, :, b * M + M // 2] = 2 - 1j
    return x


GPU_CASES = [
    # nchan, npol, M, ndat, pad (span = ndat + pad, even), zero_is_valid, Nd, inplace
    (8, 2, 128, 128 * 40 + 37, 7, True, 1, False),
    (8, 2, 128, 128 * 40, 0, False, 1, True),
    (4, 1, 1024, 1024 * 12, 2, True, 1, False),
    (16, 2, 64, 64 * 30 + 5, 9, False, 4, False),
    (3, 2, 25600, 25600 * 3, 0, True, 1, True),     # one block per CTA
    (5, 2, 2, 2 * 301, 4, False, 1, False),
    (4, 2, 130, 130 * 20 + 3, 1, True, 1, False),   # M % 4 == 2: the column tail
    (2, 2, 256, 100, 0, True, 1, False),            # ndat < M: nothing to do
]


@pytest.mark.gpu
@pytest.mark.parametrize("nchan,npol,M,ndat,pad,ziv,Nd,inplace", GPU_CASES)
def test_sk_kernel_bit_exact(ctx, b2, orc, nchan, npol, M, ndat, pad, ziv, Nd, inplace):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(M * 31 + nchan)
    span = ndat + pad
    x = _voltages(rng, nchan, npol, span, M)
    lo, hi = b2.sk_limits(M, Nd, 3.0, npol) if M > 3 else (np.float32(0.5), np.float32(1.5))
    ref_sums, ref_counts, ref_mask, ref_out = orc.sk(x, M, lo, hi, Nd=Nd, zero_is_valid=ziv,
                                                      ndat=ndat)
    npart = ndat // M
    d_in = torch.from_numpy(x.view(np.float32)).cuda()
    d_out = d_in if inplace else torch.full_like(d_in, float("nan"))
    d_sums = torch.zeros(max(1, npart * nchan * npol * 2), dtype=torch.float32, device="cuda")
    d_counts = torch.zeros(max(1, npart * nchan), dtype=torch.int32, device="cuda")
    d_mask = torch.full((max(1, npart * nchan),), 7, dtype=torch.uint8, device="cuda")
    d_zap = torch.zeros(1, dtype=torch.int64, device="cuda")
    n = ctx.sk(d_in, span, ndat, nchan, npol, M, lo, hi, d_out, span, d_sums, d_counts, d_mask,
               d_zap, Nd=Nd, zero_is_valid=ziv)
    ctx.synchronize()
    assert n == npart
    out = d_out.cpu().numpy().view(np.complex64).reshape(nchan, npol, span)
    if npart == 0:
        if not inplace:
            assert np.isnan(out.view(np.float32)).all()
        return
    assert d_sums.cpu().numpy().tobytes() == ref_sums.tobytes()
    assert d_counts.cpu().numpy().astype(np.uint32).tobytes() == ref_counts.tobytes()
    mask = d_mask.cpu().numpy().reshape(npart, nchan)
    np.testing.assert_array_equal(mask, ref_mask)
    assert int(d_zap.item()) == int(ref_mask.sum())
    assert 0 < ref_mask.sum() < ref_mask.size        # the case exercises both outcomes
    body = npart * M
    assert out[:, :, :body].tobytes() == ref_out[:, :, :body].tobytes()
    tail = out[:, :, body:].view(np.float32)
    if inplace:
        assert tail.tobytes() == x[:, :, body:].view(np.float32).tobytes()
    else:
        assert np.isnan(tail).all()


@pytest.mark.gpu
def test_sk_optional_outputs(ctx, b2, orc):
    """The statistics outputs are optional: in-place masking alone."""
    torch = pytest.importorskip("torch")
    nchan, npol, M = 4, 2, 256
    ndat = M * 20
    rng = np.random.default_rng(3)
    x = _voltages(rng, nchan, npol, ndat, M, zero_blocks=False)
    lo, hi = b2.sk_limits(M, 1, 3.0, npol)
    _, _, ref_mask, ref_out = orc.sk(x, M, lo, hi)
    d = torch.from_numpy(x.view(np.float32)).cuda()
    ctx.sk(d, ndat, ndat, nchan, npol, M, lo, hi, d, ndat)
    ctx.synchronize()
    assert d.cpu().numpy().tobytes() == ref_out.view(np.float32).tobytes()


@pytest.mark.gpu
def test_sk_rejects_bad_arguments(ctx, b2):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(2 * 2 * 4096 + 64, dtype=torch.float32, device="cuda")
    out = torch.zeros_like(buf)
    bad = [
        dict(M=127),                                   # odd M
        dict(npol=3),
        dict(in_span=1023),                            # odd span
        dict(M=28672),                                 # 2*4*(28672+4) bytes > 224 KiB
        dict(d_in=buf.data_ptr() + 8),                 # not 16-byte aligned
        dict(d_out=buf.data_ptr() + 64),               # overlaps without being equal
        dict(out_span=2048, d_out=buf.data_ptr()),     # in place with another span
    ]
    for b in bad:
        a = dict(d_in=buf.data_ptr(), in_span=1024, ndat=1024, nchan=2, npol=2, M=128,
                 d_out=out.data_ptr(), out_span=1024)
        a.update(b)
        with pytest.raises(b2.B200Error, match="sk") as e:
            ctx.sk(a["d_in"], a["in_span"], a["ndat"], a["nchan"], a["npol"], a["M"], 0.5, 1.5,
                   a["d_out"], a["out_span"])
        assert e.value.code == b2._capi.EINVAL, b


# ---------------------------------------------------------------- engine steps (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("nchan,npol,M,ndat,zero_is_valid", [(8, 2, 128, 5157, True),
                                                             (4, 1, 1024, 12288, False),
                                                             (16, 2, 64, 1925, True)])
def test_sk_engine_steps_match_oracle(ctx, b2, orc, nchan, npol, M, ndat, zero_is_valid):
    """compute / detect_ft / detect_tscr / reset_mask / count_mask / mask,
    each through the C ABI, against the oracle's restatement of the same step
    and against the fused single-pass engine."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(nchan * M + npol)
    span = ndat + (ndat & 1)
    x = (rng.standard_normal((nchan, npol, span)) + 1j * rng.standard_normal((nchan, npol, span))
         ).astype(np.complex64)
    x[0, :, :M] *= 8.0                                   # an outlying block
    x[nchan - 1, :, 2 * M:3 * M] = 0.0                   # a silent block
    if nchan > 2:
        x[1] += 2.0 * np.exp(2j * np.pi * 0.1 * np.arange(span))   # a tone all along channel 1
    lo, hi = b2.sk_limits(M, 1, 3.0, npol)
    rs, rc, rm, rout = orc.sk(x, M, lo, hi, zero_is_valid=zero_is_valid, ndat=ndat)
    npart = ndat // M
    d = torch.from_numpy(x).cuda()
    sums = torch.zeros((npart, nchan, npol, 2), dtype=torch.float32, device="cuda")
    counts = torch.zeros((npart, nchan), dtype=torch.int32, device="cuda")
    assert ctx.sk_compute(d, span, ndat, nchan, npol, M, sums, counts, zero_is_valid) == npart
    ctx.synchronize()
    assert np.array_equal(sums.cpu().numpy(), rs)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint32), rc)
    assert np.array_equal(d.cpu().numpy(), x), "compute must not write its input"
    mask = torch.full((npart, nchan), 7, dtype=torch.uint8, device="cuda")
    ctx.sk_reset_mask(mask, npart, nchan)
    ctx.sk_detect_ft(sums, counts, npart, nchan, npol, M, lo, hi, mask)
    assert np.array_equal(mask.cpu().numpy(), rm)
    assert ctx.sk_count_mask(mask, npart, nchan) == int(rm.sum())
    # mask out of place and in place: the oracle's masked copy
    out = torch.full_like(d, complex(np.nan, np.nan))
    ctx.sk_mask(mask, d, span, out, span, ndat, nchan, npol, M)
    ctx.sk_mask(mask, d, span, d, span, ndat, nchan, npol, M)
    ctx.synchronize()
    n = npart * M
    assert np.array_equal(out.cpu().numpy()[..., :n], rout[..., :n])
    assert np.array_equal(d.cpu().numpy()[..., :n], rout[..., :n])
    # detect_tscr ORs each zapped channel into every part
    ref_t = orc.sk_detect_tscr(rs, rc, 1, 3.0)
    nz = ctx.sk_detect_tscr(sums, counts, npart, nchan, npol, M, 3.0, mask)
    assert nz == int(ref_t[0].sum())
    assert np.array_equal(mask.cpu().numpy(), rm | ref_t)
    if nchan > 2:
        assert ref_t[0, 1] == 1, "the tone channel is zapped by the time-scrunched test"


@pytest.mark.gpu
@pytest.mark.parametrize("res,zero_is_valid", [([(64, 1), (128, 2), (256, 4)], True),
                                               ([(128, 1), (256, 2)], False),
                                               ([(64, 2)], True)])
def test_sk_resolutions_match_oracle(ctx, b2, orc, res, zero_is_valid):
    """SpectralKurtosis::detect over several resolutions with overlapping
    blocks (SpectralKurtosis.C:251-281, 830-986, 1105-1222, 1465-1566): sums
    of every resolution, the finest mask and the masked voltages through the
    C ABI's engine steps, bit-exact against the oracle's restatement."""
    torch = pytest.importorskip("torch")
    nchan, npol, ndat = 6, 2, 5000
    rng = np.random.default_rng(len(res) * 7 + int(zero_is_valid))
    x = (rng.standard_normal((nchan, npol, ndat)) + 1j * rng.standard_normal((nchan, npol, ndat))
         ).astype(np.complex64)
    x[1, :, 700:760] *= 12.0                        # a burst
    x[3] += 3.0 * np.exp(2j * np.pi * 0.21 * np.arange(ndat))     # a tone
    if not zero_is_valid:
        x[4, :, 1000:1100] = 0                      # dropped samples
    d = torch.from_numpy(x).cuda()
    std_devs = 3.0
    # the reference's order: compute at the finest, then per resolution
    # tscrunch (from the previous one) and detect_skfb into the finest mask
    M0, nov0 = res[0]
    off0, npart0, _, _ = orc.sk_resolution(M0, nov0, ndat)
    rs, rc = orc.sk_compute_overlap(x, M0, nov0, zero_is_valid)
    assert rs.shape[0] == npart0
    gs = torch.zeros((npart0, nchan, npol, 2), dtype=torch.float32, device="cuda")
    gc = torch.zeros((npart0, nchan), dtype=torch.int32, device="cuda")
    assert ctx.sk_compute(d, ndat, ndat, nchan, npol, M0, gs, gc, zero_is_valid, nov0) == npart0
    ctx.synchronize()
    assert np.array_equal(gs.cpu().numpy(), rs)
    assert np.array_equal(gc.cpu().numpy().astype(np.uint32), rc)
    rmask = np.zeros((npart0, nchan), np.uint8)
    gmask = torch.zeros((npart0, nchan), dtype=torch.uint8, device="cuda")
    prev = (M0, nov0, off0, npart0)
    for ires, (M, nov) in enumerate(res):
        off, npart, _, _ = orc.sk_resolution(M, nov, ndat)
        if ires > 0:
            nsum, offset = M // prev[0], off // prev[2]
            rs, rc = orc.sk_tscrunch(rs, rc, npart, nsum, offset)
            gs2 = torch.zeros((npart, nchan, npol, 2), dtype=torch.float32, device="cuda")
            gc2 = torch.zeros((npart, nchan), dtype=torch.int32, device="cuda")
            ctx.sk_tscrunch(gs, gc, prev[3], npart, nchan, npol, nsum, offset, gs2, gc2)
            gs, gc = gs2, gc2
            ctx.synchronize()
            assert np.array_equal(gs.cpu().numpy(), rs), ires
            assert np.array_equal(gc.cpu().numpy().astype(np.uint32), rc), ires
        nflag = M // M0 if ires else 1
        flag_step = nov0 if ires else 1
        flag_offset = nflag * flag_step // nov if ires else 1
        orc.sk_detect_skfb(rs, rc, 1, std_devs, rmask, nflag, flag_step, flag_offset)
        ctx.sk_detect_skfb(gs, gc, npart, nchan, npol, std_devs, gmask, npart0, nflag, flag_step,
                           flag_offset)
        assert np.array_equal(gmask.cpu().numpy(), rmask), ires
        prev = (M, nov, off, npart)
    assert rmask.sum() > 0
    # mask (SpectralKurtosis.C:1465-1566)
    max_M, max_off = res[-1][0], orc.sk_resolution(res[-1][0], res[-1][1], ndat)[0]
    idat_start = max_M - max_off
    nskip = idat_start // off0
    back_out = orc.sk_resolution(res[-1][0], res[-1][1], ndat)[2]
    npart_m = (back_out - M0) // off0 + 1
    ref = orc.sk_mask_overlap(rmask, x, M0, off0, npart_m, nskip, idat_start)
    out = torch.full((nchan, npol, ref.shape[2]), complex(np.nan, np.nan), dtype=torch.complex64,
                     device="cuda")
    ctx.sk_mask_overlap(gmask, d, ndat, out, ref.shape[2], nchan, npol, M0, off0, npart_m, nskip,
                        idat_start)
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
