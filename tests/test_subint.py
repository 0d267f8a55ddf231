"""Sub-integrations: TimeDivide (Signal/Pulsar/TimeDivide.C) and the block
loop of Subint<Fold> (Signal/Pulsar/dsp/Subint.h:206-362), host side, against
the oracle's independent pure-Python restatement."""
import numpy as np
import pytest


def product_actions(td, start, ndat, rate):
    out = []
    for a in td.block(start, ndat, rate):
        if a["kind"] == 0:
            out.append(("fold", a["idat_start"], a["ndat"], a["division"], bool(a["end_reached"]),
                        (a["lower_day"], a["lower_sec"], a["lower_frac"]),
                        (a["upper_day"], a["upper_sec"], a["upper_frac"])))
        else:
            out.append(("close", "partial" if a["kind"] == 1 else "complete"))
    return out


def run_both(b2, orc, blocks, rate, **kw):
    td = b2.TimeDivide(**kw)
    to = orc.TimeDivideOracle(**kw)
    res = []
    for start, ndat in blocks:
        p = product_actions(td, start, ndat, rate)
        o = orc.subint_block_actions(to, start, ndat, rate)
        assert p == o, (start, ndat)
        res.append(p)
    return res


def contiguous(orc, start, sizes, rate):
    out, t = [], start
    for n in sizes:
        out.append((t, n))
        t = orc.mjd_add(t, n / rate)
    return out


CASES = [
    dict(seconds=10.0),                       # integer seconds: start aligned within the day
    dict(seconds=2.5),
    dict(seconds=0.0137),
    dict(turns=1.0, period=0.005757),         # single-pulse mode
    dict(turns=8.0, period=0.08933),
    dict(turns=0.5, period=0.0016),
    dict(seconds=1.0, reference_epoch=(60000, 3000, 0.5)),
]


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_time_divide_matches_oracle(b2, orc, ci):
    kw = CASES[ci]
    rng = np.random.default_rng(ci)
    for rate in (16e6, 4e6, 1e6 / 3.0):
        span = (kw.get("seconds") or kw["turns"] * kw["period"]) * rate
        sizes = [int(x) for x in rng.integers(max(1, int(span / 7)), int(span * 3) + 2, 12)]
        start = (60000, int(rng.integers(0, 86000)), float(rng.random()))
        run_both(b2, orc, contiguous(orc, start, sizes, rate), rate, **kw)


def test_time_divide_gaps_and_overlaps(b2, orc):
    """Blocks with gaps between them and blocks that restart earlier data
    (as parallel readers produce) take the reference's paths."""
    rate = 4e6
    rng = np.random.default_rng(7)
    t = (60010, 500, 0.125)
    blocks = []
    for i in range(30):
        n = int(rng.integers(1000, 3_000_000))
        blocks.append((t, n))
        step = n / rate + float(rng.choice([0.0, 0.3, -0.2, 1.7]))
        t = orc.mjd_add(t, step)
    for kw in CASES:
        run_both(b2, orc, blocks, rate, **kw)


def test_divisions_tile_contiguous_data(b2, orc):
    """On contiguous data every sample folds exactly once, each closed
    division except the first holds division_ndat samples, and the folds of
    one division are contiguous."""
    rate = 16e6
    res = run_both(b2, orc, contiguous(orc, (60000, 3600, 0.25), [3_000_000] * 20, rate),
                   rate, seconds=0.5)
    per_div = {}
    for acts in res:
        covered = 0
        for a in acts:
            if a[0] == "fold":
                assert a[1] == covered
                covered += a[2]
                per_div[a[3]] = per_div.get(a[3], 0) + a[2]
        assert covered == 3_000_000
    divs = sorted(per_div)
    assert divs == list(range(divs[0], divs[-1] + 1))
    for d in divs[1:-1]:
        assert per_div[d] == 8_000_000


def test_single_pulse_divisions(b2, orc):
    """turns = 1: one division per pulse period, rounded to whole samples."""
    rate, period = 4e6, 0.005757
    res = run_both(b2, orc, contiguous(orc, (60000, 10, 0.0), [100_000] * 10, rate), rate,
                   turns=1.0, period=period)
    folds = [a for acts in res for a in acts if a[0] == "fold"]
    n = {}
    for a in folds:
        n[a[3]] = n.get(a[3], 0) + a[2]
    inner = [n[d] for d in sorted(n)[1:-1]]
    assert all(abs(x - period * rate) <= 1 for x in inner)


def test_time_divide_rejects(b2):
    with pytest.raises(b2.B200Error, match="division length"):
        b2.TimeDivide()
    with pytest.raises(b2.B200Error, match="division length"):
        b2.TimeDivide(turns=1.0)
    td = b2.TimeDivide(seconds=1.0)
    with pytest.raises(b2.B200Error, match="rate"):
        td.block((60000, 0, 0.0), 10, 0.0)
    with pytest.raises(b2.B200Error, match="start time"):
        td.block((0, 0, 0.0), 10, 1e6)
    with pytest.raises(b2.B200Error, match="room for 2"):
        td.block((60000, 0, 0.0), 10_000_000, 1e6, cap=2)
