"""Inter-channel dispersion delays (DedispersionPipe -K): the host rule
behind the pipeline's SampleDelay stage and response, against the oracle's
pure-Python restatement of Dedispersion::SampleDelay
(Signal/General/DedispersionSampleDelay.C:26-140) and SampleDelay::build
(Signal/General/SampleDelay.C:65-141)."""
import numpy as np
import pytest


def centres(orc, cf, bw, nchan, fb):
    if fb:
        return np.asarray(orc.channel_centres(cf, bw, nchan, swap=True, dc_centred=True))
    return np.asarray(orc.channel_centres(cf, bw, nchan))


@pytest.mark.parametrize("cf,bw,dm,nchan,fb", [
    (1400.0, 256.0, 500.0, 64, True),       # C2
    (1400.0, -256.0, 500.0, 64, True),      # lower sideband
    (1400.0, 800.0, 1000.0, 1024, True),    # C5's re-channelisation
    (1400.0, 64.0, 40.0, 8, False),
    (820.0, 200.0, -12.5, 32, False),       # negative DM: the lower channels lead
    (1400.0, 64.0, 0.0, 8, False),          # no dispersion: no delay
    (1400.0, 16.0, 67.99, 1, False),
])
def test_delays_match_oracle(b2, orc, cf, bw, dm, nchan, fb):
    freqs = centres(orc, cf, bw, nchan, fb)
    rate = abs(bw) / nchan * 1e6
    p = b2.interchannel_delays(cf, dm, rate, freqs)
    o = orc.interchannel_delays(cf, dm, rate, list(freqs))
    assert np.array_equal(p["delay"], o["delay"])
    assert np.array_equal(p["frac"], o["frac"])
    assert np.array_equal(p["applied"], o["applied"])
    assert (p["zero_delay"], p["total_delay"]) == (o["zero_delay"], o["total_delay"])
    # the fraction is the rounding remainder; the applied shifts stay inside
    # the buffered span
    assert np.all(np.abs(p["frac"]) <= 0.5)
    if nchan > 1 and dm != 0:
        assert p["zero_delay"] > 0 and p["total_delay"] > 0
        assert np.all((p["applied"] >= 0) & (p["applied"] <= p["total_delay"]))
        # delays relative to the band follow 1/f^2
        t = dm / 2.41e-4 * (1 / cf ** 2 - 1 / freqs ** 2) * rate
        assert np.all(np.abs(p["delay"] - t) <= 0.5)
    if dm == 0:
        assert p["total_delay"] == 0 and not p["applied"].any()


def test_sample_delay_block_restates_transformation(orc):
    """output[c][t] = input[c][t + applied[c]] for ndat - total samples."""
    y = np.arange(3 * 2 * 20, dtype=np.float32).reshape(3, 2, 20)
    out = orc.sample_delay_block(y, [0, 3, 5], 5)
    assert out.shape == (3, 2, 15)
    assert np.array_equal(out[1, 1], y[1, 1, 3:18])
    assert orc.sample_delay_block(y[:, :, :4], [0, 3, 5], 5).shape[2] == 0
