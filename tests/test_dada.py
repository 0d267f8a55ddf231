"""DADA file source: the ASCII header rules (Kernel/Classes/ascii_header.c),
DADAHeader::load_header / valid (DADAHeader.C:56-174), ASCIIObservation::load
(ASCIIObservation.C:88-410) and File's sample arithmetic (File.C:175-390).

The header get/set rules are pinned against the reference's own
ascii_header.c, compiled from its sources by `make -C oracle ref` into
oracle/_ref/ (skipped where that library was not built)."""
import ctypes
import datetime
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libascii_header_ref.so")

BASE_KEYS = {
    "HDR_VERSION": "1.0", "TELESCOPE": "PKS", "RECEIVER": "MULTI", "INSTRUMENT": "CASPSR",
    "SOURCE": "J0437-4715", "MODE": "PSR", "FREQ": 1382, "BW": -400, "NPOL": 2, "NBIT": 8,
    "NDIM": 2, "NCHAN": 4, "TSAMP": 0.0025, "UTC_START": "2010-04-13-02:05:45",
    "OBS_OFFSET": 0,
}


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built (needs the reference sources: make -C oracle ref)")
    return ctypes.CDLL(REF_LIB)


def ref_get(ref, header, key):
    buf = ctypes.create_string_buffer(8192)
    rc = ref.ascii_header_get(header.encode(), key.encode(), b"%s", buf)
    return buf.value.decode() if rc == 1 else None


def ref_set(ref, header, key, value, size=4096):
    buf = ctypes.create_string_buffer(header.encode(), size)
    assert ref.ascii_header_set(buf, key.encode(), b"%s", str(value).encode()) == 0
    return buf.value.decode()


HEADERS = [
    "HDR_VERSION 1.0\nNCHAN 4\nNPOL 2\n",
    # keyword as the first word, with and without a following blank
    "NCHAN\t16\nXNCHAN 3\n",
    "NCHANS 9\nNCHAN 5\n",
    # keyword inside another word and after a backslash
    "SOURCE_NAME x\nNCHAN_PFB 8\n\\NCHAN 7\n",
    # value on the next line, value missing at the end
    "FREQ\n  1400.5\nBW",
    "BW  \n",
    # comments, tabs and carriage returns
    "TSAMP 0.025 # microseconds\nUTC_START\t2020-01-01-00:00:00\r\nNDIM 2\n",
    # a keyword whose first match is not at a line start
    "COMMENT FREQ is 1 GHz\nFREQ 1000\n",
    # a value longer than the reference's 64-byte scan buffers
    "SOURCE " + "J" * 50 + "\n",
    "",
]
KEYS = ["HDR_VERSION", "NCHAN", "NPOL", "SOURCE", "FREQ", "BW", "TSAMP", "UTC_START", "NDIM",
        "XNCHAN", "NCHAN_PFB", "MISSING", "COMMENT"]


@pytest.mark.parametrize("hi", range(len(HEADERS)))
def test_header_get_matches_reference(b2, ref, hi):
    h = HEADERS[hi]
    for k in KEYS:
        assert b2.ascii_header_get(h, k) == ref_get(ref, h, k), (h, k)


SET_SEQUENCES = [
    ("", [("HDR_SIZE", 4096), ("NCHAN", 4), ("NCHAN", 16), ("FREQ", 1400.25)]),
    ("HDR_VERSION 1.0\nNCHAN 4   # comment kept\nDATA\n", [("NCHAN", 8), ("NPOL", 2),
                                                          ("BW", -64)]),
    ("SOURCE J0437\nTELESCOPE PKS", [("TELESCOPE", "MOST"), ("MODE", "CAL")]),
    ("XNPOL 3\nNPOL\t1\n", [("NPOL", 2), ("XNPOL", 4)]),
]


@pytest.mark.parametrize("si", range(len(SET_SEQUENCES)))
def test_header_set_matches_reference(b2, ref, si):
    h0, ops = SET_SEQUENCES[si]
    a = b = h0
    for k, v in ops:
        a = b2.ascii_header_set(a, k, v)
        b = ref_set(ref, b, k, v)
        assert a == b, (k, v)


def test_header_set_reports_overflow(b2):
    with pytest.raises(b2.B200Error, match="buffer has 64"):
        b2.ascii_header_set("", "SOURCE", "x" * 80, header_size=64)


def mjd_of(utc):
    t = datetime.datetime.strptime(utc, "%Y-%m-%d-%H:%M:%S").replace(
        tzinfo=datetime.timezone.utc)
    s = int(t.timestamp())
    return 40587 + s // 86400, s % 86400


def header_text(b2, keys, size=4096):
    text = b2.ascii_header_set("", "HDR_SIZE", size, size)
    for k, v in keys.items():
        text = b2.ascii_header_set(text, k, v, size)
    return text


def test_parse_fields_and_start_time(b2):
    keys = dict(BASE_KEYS, OBS_OFFSET=16 * 1000, PICOSECONDS=250_000_000_000, DSB=1,
                STATE="Analytic", BASIS="Linear")
    i = b2.dada_parse(header_text(b2, keys))
    assert (i["nchan"], i["npol"], i["nbit"], i["ndim"]) == (4, 2, 8, 2)
    assert i["centre_freq_mhz"] == 1382.0 and i["bandwidth_mhz"] == -400.0
    assert i["tsamp_us"] == 0.0025 and i["rate_hz"] == 1.0 / (0.0025 * 1e-6)
    assert i["bits_per_sample"] == 128 and i["hdr_version"] == 1.0
    assert (i["telescope"], i["receiver"], i["source"], i["mode"], i["instrument"]) == (
        "PKS", "MULTI", "J0437-4715", "PSR", "CASPSR")
    assert (i["state"], i["basis"], i["dual_sideband"]) == ("Analytic", "Linear", 1)
    day, sec = mjd_of("2010-04-13-02:05:45")
    assert (i["start_day"], i["start_sec"]) == (day, sec) == (55299, 7545)
    # PICOSECONDS, then the 1000 samples of OBS_OFFSET at 2.5 ns
    assert i["start_frac"] == pytest.approx(0.25 + 1000 * 0.0025e-6, abs=1e-15)
    assert i["ndat"] == 0 and i["file_ndat"] == 0


def test_parse_defaults(b2):
    keys = {k: v for k, v in BASE_KEYS.items() if k not in ("NCHAN", "NDIM", "RECEIVER",
                                                            "HDR_VERSION", "MODE")}
    keys["UTC_START"] = "TBD"
    i = b2.dada_parse(header_text(b2, keys))
    assert (i["nchan"], i["ndim"], i["receiver"], i["hdr_version"]) == (1, 1, "unknown", 0.0)
    assert (i["start_day"], i["start_sec"], i["start_frac"]) == (0, 0, 0.0)
    assert i["dual_sideband"] == -1 and i["bits_per_sample"] == 16


@pytest.mark.parametrize("key", ["TELESCOPE", "SOURCE", "FREQ", "BW", "NPOL", "NBIT", "TSAMP",
                                 "UTC_START", "OBS_OFFSET"])
def test_parse_required_keys(b2, key):
    keys = {k: v for k, v in BASE_KEYS.items() if k != key}
    with pytest.raises(b2.B200Error, match=f"failed load {key}"):
        b2.dada_parse(header_text(b2, keys))


def test_parse_offset_fallback_and_bad_values(b2):
    keys = {k: v for k, v in BASE_KEYS.items() if k != "OBS_OFFSET"}
    keys["OFFSET"] = 128
    assert b2.dada_parse(header_text(b2, keys))["obs_offset"] == 128
    with pytest.raises(b2.B200Error, match="invalid NDIM=3"):
        b2.dada_parse(header_text(b2, dict(BASE_KEYS, NDIM=3)))
    with pytest.raises(b2.B200Error, match="failed load FREQ"):
        b2.dada_parse(header_text(b2, dict(BASE_KEYS, FREQ="high")))
    with pytest.raises(b2.B200Error, match="strptime"):
        b2.dada_parse(header_text(b2, dict(BASE_KEYS, UTC_START="2010/04/13")))
    with pytest.raises(b2.B200Error, match="BLOCK_DATA_BYTES"):
        b2.dada_parse(header_text(b2, dict(BASE_KEYS, BLOCK_DATA_BYTES=4096,
                                           BLOCK_HEADER_BYTES=64)))


def raw_data(ndat, nchan=4, npol=2, seed=0):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, ndat * nchan * npol * 2, dtype=np.uint8)


def test_open_and_read(b2, tmp_path):
    data = raw_data(1000)
    path = tmp_path / "obs.dada"
    b2.write_dada(path, BASE_KEYS, data)
    with b2.DADAFile(path) as f:
        assert f.info["header_bytes"] == 4096 and f.info["adjacent_header"] == 0
        assert f.ndat == f.info["file_ndat"] == 1000 and f.bytes_per_sample == 16
        assert f.header.startswith("HDR_SIZE")
        assert np.array_equal(f.read(0, 1000), data)
        assert np.array_equal(f.read(123, 77), data[123 * 16:200 * 16])
        # reads stop at the end of the data, past it they return nothing
        assert np.array_equal(f.read(990, 50), data[990 * 16:])
        assert f.read(1000, 10).size == 0 and f.read(5000, 10).size == 0
    assert b2.dada_is_valid(path)


def test_ndat_from_header_and_partial_samples(b2, tmp_path):
    data = raw_data(1000)
    # NDAT below the file size: the data end at NDAT
    p = tmp_path / "short.dada"
    b2.write_dada(p, dict(BASE_KEYS, NDAT=600), data)
    with b2.DADAFile(p) as f:
        assert f.info["ndat"] == 600 and f.info["file_ndat"] == 1000 and f.ndat == 600
        assert f.read(590, 100).size == 10 * 16
    # NDAT above it (a recording cut short): the data end with the file; a
    # trailing partial sample is not a sample
    p = tmp_path / "long.dada"
    b2.write_dada(p, dict(BASE_KEYS, NDAT=10 ** 12), np.concatenate([data, data[:7]]))
    with b2.DADAFile(p) as f:
        assert f.info["ndat"] == 10 ** 12 and f.info["file_ndat"] == 1000 and f.ndat == 1000
        assert np.array_equal(f.read(999, 100), data[999 * 16:])


def test_header_larger_than_default(b2, tmp_path):
    """HDR_SIZE above 4096: DADAHeader::load_header reads again with the
    larger size, so keys past the first 4096 bytes are seen."""
    size = 16384
    text = header_text(b2, {k: v for k, v in BASE_KEYS.items() if k != "SOURCE"}, size)
    for j in range(200):
        text = b2.ascii_header_set(text, f"PAD_{j:03d}", "x" * 20, size)
    assert len(text) > 4096
    text = b2.ascii_header_set(text, "SOURCE", "B1937+21", size)
    data = raw_data(100, seed=1)
    p = tmp_path / "big.dada"
    with open(p, "wb") as f:
        f.write(text.encode() + b"\0" * (size - len(text)))
        f.write(data.tobytes())
    with b2.DADAFile(p) as f:
        assert f.info["header_bytes"] == size and f.info["source"] == "B1937+21"
        assert f.ndat == 100 and np.array_equal(f.read(0, 100), data)


def test_adjacent_header_file(b2, tmp_path):
    """No HDR_SIZE in the data file: the header comes from name.hdr (or
    name.ext.hdr); an HDR_SIZE there is a block to skip in the data file."""
    data = raw_data(500, seed=2)
    text = "\n".join(f"{k} {v}" for k, v in BASE_KEYS.items()) + "\n"
    raw = tmp_path / "obs.raw"
    raw.write_bytes(b"\0" * 8 + data.tobytes())
    # 4096 bytes are needed before the header search, as fread requires
    with pytest.raises(b2.B200Error):
        b2.DADAFile(raw)
    raw.write_bytes(data.tobytes() * 10)
    with pytest.raises(b2.B200Error, match="no adjacent header"):
        b2.DADAFile(raw)
    (tmp_path / "obs.hdr").write_text(text)
    with b2.DADAFile(raw) as f:
        assert f.info["adjacent_header"] == 1 and f.info["header_bytes"] == 0
        assert f.ndat == 5000 and np.array_equal(f.read(0, 500), data)
    os.remove(tmp_path / "obs.hdr")
    (tmp_path / "obs.raw.hdr").write_text(text + "HDR_SIZE 16\n")
    with b2.DADAFile(raw) as f:
        assert f.info["adjacent_header"] == 1 and f.info["header_bytes"] == 16
        assert f.ndat == 4999 and np.array_equal(f.read(0, 10), data[16:16 + 160])


def test_is_valid(b2, tmp_path):
    data = raw_data(10)
    for drop, ok in (("INSTRUMENT", False), ("HDR_VERSION", False), (None, True)):
        keys = {k: v for k, v in BASE_KEYS.items() if k != drop}
        p = tmp_path / f"v_{drop}.dada"
        b2.write_dada(p, keys, data)
        assert b2.dada_is_valid(p) == ok
    (tmp_path / "tiny.dada").write_bytes(b"HDR_SIZE 4096\n")
    assert not b2.dada_is_valid(tmp_path / "tiny.dada")
    assert not b2.dada_is_valid(tmp_path / "absent.dada")


def test_sub_byte_samples(b2, tmp_path):
    """4-bit, one real channel: two samples a byte; reads must start and end
    on bytes."""
    keys = dict(BASE_KEYS, NBIT=4, NPOL=1, NCHAN=1, NDIM=1)
    p = tmp_path / "nib.dada"
    data = np.arange(64, dtype=np.uint8)
    b2.write_dada(p, keys, data)
    with b2.DADAFile(p) as f:
        assert f.info["bits_per_sample"] == 4 and f.ndat == 128
        assert np.array_equal(f.read(2, 10), data[1:6])
        with pytest.raises(b2.B200Error, match="byte"):
            f.read(1, 10)


def test_pipeline_config_from_file(b2, tmp_path):
    p = tmp_path / "cfg.dada"
    b2.write_dada(p, dict(BASE_KEYS, PICOSECONDS=5 * 10 ** 11), raw_data(10))
    with b2.DADAFile(p) as f:
        c = f.pipeline_config(dm=10.0, nfft=8192, nfilt_pos=100, nfilt_neg=100, nbin=64,
                              period=0.005)
        assert (c.centre_freq_mhz, c.bandwidth_mhz, c.nchan, c.npol) == (1382.0, -400.0, 4, 2)
        assert c.input_kind == b2.INT8_TFPD and c.dual_sideband == 1
        assert (c.start_day, c.start_sec, c.start_frac) == (55299, 7545, 0.5)
    b2.write_dada(p, dict(BASE_KEYS, NDIM=1), raw_data(10))
    with b2.DADAFile(p) as f, pytest.raises(b2.B200Error, match="NDIM 2"):
        f.pipeline_config(dm=10.0, nfft=8192, nfilt_pos=100, nfilt_neg=100, nbin=64,
                          period=0.005)
