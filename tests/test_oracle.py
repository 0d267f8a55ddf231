"""Pins the CPU oracle against the reference's own known-answer tests.

The reference cannot be built here (its Signal/General/dsp headers, PSRCHIVE
and FFTW are absent), so these tests restate its test cases and thresholds:
  - Signal/General/tests/ConvolutionTest.cpp:148-308  (Tukey impulse response, 5e-8)
  - test/Detection/test_Detection.cpp:113-244         (closed-form detection)
  - Signal/General/PlasmaResponse.C / Response.C      (smear and FFT-length rules)
  - Signal/Pulsar/Fold.C:815-818                       (bin recurrence)
"""
import numpy as np
import pytest


def test_fft_matches_numpy(orc):
    rng = np.random.default_rng(7)
    for n in (8, 64, 4096, 1 << 17):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        ref = np.fft.fft(x)
        got = orc.fft(x.astype(np.complex128))
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13
        back = orc.fft(x.astype(np.complex128), +1)
        assert np.max(np.abs(back - np.fft.ifft(x) * n)) / n < 1e-13
        got32 = orc.fft(x.astype(np.complex64))
        rel = np.sqrt(np.mean(np.abs(got32 - ref) ** 2) / np.mean(np.abs(ref) ** 2))
        assert rel < 3e-7


def test_smearing_rule_matches_the_workloads_numbers(orc):
    # C1: DM 67.99, 16 MHz at 1400 MHz, one channel
    neg = orc.smearing_samples(1400.0, 16.0, 67.99, 1, -1)
    pos = orc.smearing_samples(1400.0, 16.0, 67.99, 1, 1)
    assert (neg, pos) == (29455, 28462)
    assert orc.minimum_ndat(pos, neg) == 1 << 16
    assert orc.optimal_fft_length(neg + pos) == 1 << 20
    # C2: DM 500, 64 x 4 MHz channels
    neg = orc.smearing_samples(1400.0, 256.0, 500.0, 64, -1)
    pos = orc.smearing_samples(1400.0, 256.0, 500.0, 64, 1)
    assert neg + pos == 35319
    assert orc.minimum_ndat(pos, neg) == 1 << 16


def test_optimal_fft_length_rule(orc):
    # optimize_fft.c: T(N) = N log N / (N - nbad) is minimised over powers of two
    for nbad in (1, 100, 384, 5566, 57917):
        n = orc.optimal_fft_length(nbad)
        cost = lambda m: m * np.log(m) / (m - nbad)
        assert n > nbad
        assert cost(n) <= cost(2 * n)
        if n // 2 > nbad:
            assert cost(n) <= cost(n // 2)
    assert orc.optimal_fft_length(384) == 4096


def _tukey_case(orc, convolve):
    """ConvolutionTest.test_operate_tukey (ConvolutionTest.cpp:148-308), Analytic."""
    n_neg, n_pos = 128, 256
    nfilt = orc.optimal_fft_length(n_neg + n_pos)
    spectral, temporal = orc.tukey_response(n_neg, n_pos, nfilt)
    n_loop = 256 + 13
    n_overlap = n_neg + n_pos
    n_keep = nfilt - n_overlap
    expected_ndat = n_keep * 2 * n_loop
    input_ndat = expected_ndat + n_overlap
    npol = 2
    x = np.zeros((1, npol, input_ndat), np.complex64)
    base = [n_overlap, nfilt - n_pos]
    offsets = np.zeros((n_loop, npol), np.int64)
    for iloop in range(n_loop):
        for ipol in range(npol):
            off = base[ipol] + iloop * 2 * (nfilt - n_overlap) + iloop + ipol
            offsets[iloop, ipol] = off
            x[0, ipol, off] = 1.0
    # Convolution::prepare_normalizer appends a ScalarFilter of 1/sqrt(nfft)
    # (Convolution.C:300-313, 401-414): a complex<float> times float product
    norm = np.float32(1.0 / np.sqrt(nfilt))
    resp = (spectral.view(np.float32) * norm).view(np.complex64)
    out = convolve(x, resp.reshape(1, nfilt), nfilt, n_pos, n_neg)
    assert out.shape[2] == expected_ndat
    for ipol in range(npol):
        res = out[0, ipol].astype(np.complex128)
        base_power, base_count, bidx = 0.0, 0, 0
        for iloop in range(n_loop):
            off = offsets[iloop, ipol] - n_overlap
            seg = res[off:off + n_overlap]
            diff = seg - temporal.astype(np.complex128)
            ratio = np.sum(np.abs(diff) ** 2) / np.sum(np.abs(temporal.astype(np.complex128)) ** 2)
            mean_error = np.sqrt(ratio / n_overlap)
            assert mean_error < 5e-8, (ipol, iloop, mean_error)
            end = out.shape[2] if iloop + 1 == n_loop else offsets[iloop + 1, ipol] - n_overlap
            base_power += np.sum(np.abs(res[bidx:off]) ** 2)
            base_count += off - bidx
            bidx = off + n_overlap
            base_power += np.sum(np.abs(res[bidx:end]) ** 2)
            base_count += end - bidx
            bidx = end
        rms = np.sqrt(base_power / base_count)
        assert rms < 5e-8, (ipol, rms)


def test_tukey_known_answer(orc):
    _tukey_case(orc, lambda x, r, n, pos, neg: orc.convolve(x, r, n, pos, neg))


def test_zero_dm_response_is_passthrough(orc):
    """A unit response (normaliser 1/sqrt(N) folded in) returns the kept input
    samples (the zero-DM identity of test/Convolution/test_Convolution.cpp)."""
    rng = np.random.default_rng(3)
    nfft, pos, neg = 4096, 300, 200
    x = (rng.standard_normal((2, 2, 20000)) + 1j * rng.standard_normal((2, 2, 20000)))
    h = orc.dedispersion_response_f64(1400.0, 16.0, 0.0, 2, nfft, input_nchan=2)
    y = orc.convolve(x.astype(np.complex128), h, nfft, pos, neg)
    nk = nfft - pos - neg
    npart = (20000 - pos - neg) // nk
    ref = x[:, :, pos:pos + npart * nk] * np.sqrt(nfft)
    assert np.max(np.abs(y - ref)) < 1e-9 * np.max(np.abs(ref))


def test_detection_closed_forms(orc):
    """test_Detection.cpp:113-244, Analytic input: re = im = ichan*npol*ndat + ipol*ndat + idat."""
    nchan, npol, ndat = 8, 2, 100
    f = np.zeros((nchan, npol, ndat), np.float32)
    for c in range(nchan):
        for p in range(npol):
            f[c, p] = c * npol * ndat + p * ndat + np.arange(ndat)
    x = (f + 1j * f).astype(np.complex64)
    inten = orc.detect(x, "Intensity")
    assert np.array_equal(inten[:, 0], 2 * f[:, 0] ** 2 + 2 * f[:, 1] ** 2)
    ppqq = orc.detect(x, "PPQQ")
    assert np.array_equal(ppqq, 2 * f ** 2)
    coh = orc.detect(x, "Coherence")
    assert np.array_equal(coh[:, 2], 2 * f[:, 0] * f[:, 1])
    assert np.array_equal(coh[:, 3], np.zeros_like(f[:, 0]))
    st = orc.detect(x, "Stokes")
    assert np.array_equal(st[:, 0], 2 * f[:, 0] ** 2 + 2 * f[:, 1] ** 2)
    assert np.array_equal(st[:, 1], 2 * f[:, 0] ** 2 - 2 * f[:, 1] ** 2)
    assert np.array_equal(st[:, 2], 4 * f[:, 0] * f[:, 1])


def test_fold_binplan_is_the_recurrence(orc):
    phi, p, nbin = -0.25, 1.0 / (16e6 * 0.08933), 1024
    plan = orc.fold_binplan(phi, p, 100000, nbin)
    x = phi
    ref = np.empty(100000, np.uint32)
    for i in range(100000):
        x -= np.floor(x)
        ref[i] = int(x * nbin)
        x += p
    assert np.array_equal(plan, ref)


def test_bittable8_levels(orc):
    lut, scale = orc.bittable8(0.0308)
    # two's complement: byte b holds int8 v, level (v + 0.5) * scale
    v = np.arange(256).astype(np.uint8).view(np.int8).astype(np.float64)
    assert np.allclose(lut, (v + 0.5) * scale, rtol=1e-6, atol=0)
    assert lut[0] > 0 and lut[255] < 0 and lut[127] > 0 and lut[128] < 0


def test_dedispersion_response_unit_modulus(orc):
    h = orc.dedispersion_response(1400.0, 16.0, 67.99, 1, 1 << 14, mode=0)
    assert np.allclose(np.abs(h) * np.sqrt(1 << 14), 1.0, atol=1e-6)
    h64 = orc.dedispersion_response_f64(1400.0, 16.0, 67.99, 1, 1 << 14)
    # the reference's float(phase) cast limits agreement to ~|phase| * 2^-24
    err = np.abs(h[0] - h64[0]) * np.sqrt(1 << 14)
    assert np.max(err) < 0.05
