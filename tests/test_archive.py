"""The profile arithmetic of the PhaseSeries -> archive unloader
(Archiver::set, Signal/Pulsar/Archiver.C:740-792, 852-984), host side,
against the oracle's independent restatement: amplitudes and weights
bit-exact, the reference's error for bins without hits."""
import numpy as np
import pytest


def _case(rng, nchan=4, npol=4, nbin=256, zeroed=False):
    sums = (rng.standard_normal((nchan, npol, nbin)) * 1e4).astype(np.float32)
    if zeroed:
        hits = rng.integers(1, 5000, (nchan, nbin)).astype(np.uint32)
    else:
        hits = rng.integers(1, 5000, nbin).astype(np.uint32)
    return sums, hits


def test_amplitudes_match_oracle(b2, orc):
    rng = np.random.default_rng(1)
    for scale in (1.0, 0.125, 3.7e-3):
        sums, hits = _case(rng)
        amps, w, bad = b2.archive_profiles(sums, hits, scale=scale)
        ra, rw, rbad = orc.archive_profiles(sums, hits, scale=scale)
        assert np.array_equal(amps.view(np.uint32), ra.view(np.uint32))
        assert np.array_equal(w, rw) and bad == rbad == 0
        assert np.all(w == 1.0)


def test_bins_without_hits(b2, orc):
    rng = np.random.default_rng(2)
    sums, hits = _case(rng, nchan=3, npol=2, nbin=64)
    hits[[0, 5, 63]] = 0
    with pytest.raises(b2.B200Error, match="without hits"):
        b2.archive_profiles(sums, hits)
    with pytest.raises(ValueError):
        orc.archive_profiles(sums, hits)
    amps, w, _ = b2.archive_profiles(sums, hits, unload_zero_hits=True)
    ra, rw, _ = orc.archive_profiles(sums, hits, unload_zero_hits=True)
    assert np.array_equal(amps.view(np.uint32), ra.view(np.uint32))
    # the unhit bins hold the mean of the hit bins
    hit = hits != 0
    for ic in range(3):
        for ip in range(2):
            m = np.mean(amps[ic, ip, hit].astype(np.float64))
            assert np.allclose(amps[ic, ip, ~hit], np.float32(m), rtol=1e-6)


def test_non_finite_profile_zeroes_its_channel_weight(b2, orc):
    rng = np.random.default_rng(3)
    sums, hits = _case(rng, nchan=5, npol=4, nbin=128)
    sums[2, 1, 17] = np.nan
    sums[4, 3, 0] = np.inf
    amps, w, bad = b2.archive_profiles(sums, hits)
    ra, rw, rbad = orc.archive_profiles(sums, hits)
    assert bad == rbad == 2
    assert np.array_equal(amps.view(np.uint32), ra.view(np.uint32))
    assert np.array_equal(w, rw)
    assert w[2] == 0 and w[4] == 0 and w[0] == 1
    assert np.all(amps[2, 1] == 0) and np.any(amps[2, 0] != 0)


def test_zeroed_data_weights(b2, orc):
    rng = np.random.default_rng(4)
    sums, hits = _case(rng, nchan=6, npol=2, nbin=100, zeroed=True)
    ndat_total = int(hits.sum(axis=1).max()) + 1234
    amps, w, _ = b2.archive_profiles(sums, hits, zeroed_data=True, ndat_total=ndat_total)
    ra, rw, _ = orc.archive_profiles(sums, hits, zeroed_data=True, ndat_total=ndat_total)
    assert np.array_equal(amps.view(np.uint32), ra.view(np.uint32))
    assert np.array_equal(w.view(np.uint32), rw.view(np.uint32))
    assert np.all((w > 0) & (w < 1))


def test_invalid_arguments(b2):
    sums = np.ones((1, 1, 8), np.float32)
    hits = np.ones(8, np.uint32)
    for scale in (0.0, float("nan"), float("inf")):
        with pytest.raises(b2.B200Error, match="invalid"):
            b2.archive_profiles(sums, hits, scale=scale)
    with pytest.raises(b2.B200Error, match="invalid"):
        b2.archive_profiles(sums, np.ones((1, 8), np.uint32), zeroed_data=True, ndat_total=0)
