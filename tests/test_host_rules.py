"""CPU-side checks of libdspsr_b200.so: it loads, exports every function
include/dspsr_b200.h declares, and its host rules (no GPU needed) agree with
the oracle's restatement of the reference."""
import ctypes
import re

import numpy as np
import pytest


def _declared_functions(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dspsr_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(b2):
    from dspsr_b200 import _capi
    names = _declared_functions(_capi.HEADER_PATH)
    assert len(names) >= 30
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares every one of them too
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)


def test_version(b2):
    assert b2._capi.lib().dspsr_b200_version() >= 100


@pytest.mark.parametrize("cf,bw,dm,nchan", [
    (1400.0, 16.0, 67.99, 1), (1400.0, 256.0, 500.0, 64), (1400.0, -128.0, 2000.0, 32),
    (1400.0, 800.0, 1000.0, 1024), (350.0, 64.0, 10.0, 8)])
def test_smearing_rule_matches_oracle(b2, orc, cf, bw, dm, nchan):
    for half in (-1, 0, 1):
        assert b2.smearing_samples(cf, bw, dm, nchan, half) == \
            orc.smearing_samples(cf, bw, dm, nchan, half)
    pos = orc.smearing_samples(cf, bw, dm, nchan, 1)
    neg = orc.smearing_samples(cf, bw, dm, nchan, -1)
    assert b2.minimum_ndat(pos, neg) == orc.minimum_ndat(pos, neg)
    assert b2.optimal_fft_length(pos + neg) == orc.optimal_fft_length(pos + neg)


def test_bittable_is_bitwise_the_oracle(b2, orc):
    for spacing in (0.0308, 0.05, 0.01):
        for twos in (True, False):
            a, sa = b2.bittable8(spacing, twos)
            b, sb = orc.bittable8(spacing, twos)
            assert a.tobytes() == b.tobytes()
            assert sa == sb


def test_fold_phi_is_bitwise_the_oracle(b2, orc):
    rng = np.random.default_rng(11)
    for _ in range(200):
        start = (60000 + int(rng.integers(0, 100)), int(rng.integers(0, 86400)), float(rng.random()))
        epoch = (59990 + int(rng.integers(0, 5)), int(rng.integers(0, 86400)), float(rng.random()))
        idat = int(rng.integers(0, 1 << 40))
        rate = float(rng.choice([16e6, 4e6, 781250.0]))
        period = float(rng.uniform(1e-3, 1.0))
        a = b2.fold_phi(start, epoch, idat, rate, period, 0.1)
        b = orc.fold_phi(start, epoch, idat, rate, period, 0.1)
        assert a == b


def test_fold_plan_is_compact(b2):
    # C1: 2^24 samples at 16 MHz, P = 89.33 ms: a few hundred segments
    n = b2.fold_plan_count(0.123, (1 / 16e6) / 0.08933, 1 << 24)
    assert 0 < n < 1000


def test_dispersion_plan_rejects_short_fft(b2):
    with pytest.raises(b2.B200Error):
        b2.dispersion_plan(1400.0, 16.0, 67.99, 1, nfft=1 << 15)
    pos, neg, nfft = b2.dispersion_plan(1400.0, 16.0, 67.99, 1)
    assert (pos, neg, nfft) == (28462, 29455, 1 << 16)


def test_context_without_gpu_reports_no_device(b2):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(b2.B200Error) as e:
        b2.Context(0)
    assert e.value.code == b2._capi.ENODEV
