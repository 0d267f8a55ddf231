"""ctypes loader for the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or as the timed CPU baseline.  The
product library never imports it.  The C++ sources it wraps restate the DSPSR
reference path; each function there cites the reference file:line it follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
i16p = np.ctypeslib.ndpointer(dtype=np.int16, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
c_u64 = ctypes.c_uint64
c_i64 = ctypes.c_int64
c_int = ctypes.c_int
c_uint = ctypes.c_uint
c_dbl = ctypes.c_double

_SIGS = {
    "orc_fft_f32": (None, [c_int, c_int, f32p, f32p]),
    "orc_fft_f64": (None, [c_int, c_int, f64p, f64p]),
    "orc_bittable8": (None, [c_dbl, c_int, f32p, ctypes.POINTER(c_dbl)]),
    "orc_unpack8": (None, [u8p, c_u64, c_int, c_int, c_int, f32p, f32p, c_u64]),
    "orc_unpack16": (None, [i16p, c_u64, c_int, c_int, c_int, c_int, f32p, c_u64]),
    "orc_smearing_samples": (c_uint, [c_dbl, c_dbl, c_dbl, c_uint, c_int]),
    "orc_minimum_ndat": (c_uint, [c_uint, c_uint]),
    "orc_optimal_fft_length": (c_i64, [c_u64, c_u64, c_uint]),
    "orc_dedispersion_response": (None, [c_dbl, c_dbl, c_dbl, c_uint, c_uint, c_int, c_int,
                                         c_int, c_int, c_uint, f32p]),
    "orc_dedispersion_response_f64": (None, [c_dbl, c_dbl, c_dbl, c_uint, c_uint, c_int,
                                             c_int, c_int, c_uint, f64p]),
    "orc_tukey_response": (None, [c_uint, c_uint, c_uint, f32p, f32p]),
    "orc_convolve_f32": (c_u64, [f32p, c_u64, c_u64, c_int, c_int, f32p, c_uint, c_uint,
                                 c_uint, f32p, c_u64, c_int]),
    "orc_convolve_f64": (c_u64, [f64p, c_u64, c_u64, c_int, c_int, f64p, c_uint, c_uint,
                                 c_uint, f64p, c_u64, c_int]),
    "orc_detect": (c_int, [f32p, c_u64, c_u64, c_int, c_int, f32p, c_u64]),
    "orc_detect_f64": (c_int, [f64p, c_u64, c_u64, c_int, c_int, f64p, c_u64]),
    "orc_fold_phi": (c_dbl, [c_i64, c_i64, c_dbl, c_i64, c_i64, c_dbl, c_u64, c_dbl, c_dbl,
                             c_dbl]),
    "orc_fold_binplan": (None, [c_dbl, c_dbl, c_u64, c_uint, u32p]),
    "orc_fold_accumulate": (None, [f32p, c_u64, c_u64, c_int, c_int, c_int, u32p, c_uint,
                                   f32p, u32p]),
    "orc_fold_accumulate_f64": (None, [f64p, c_u64, c_u64, c_int, c_int, c_int, u32p, c_uint,
                                       f64p, u32p]),
    "orc_sk_compute": (c_u64, [f32p, c_u64, c_u64, c_int, c_int, c_uint, c_int, f32p, u32p]),
    "orc_sk_detect": (c_u64, [f32p, u32p, c_u64, c_int, c_int, c_uint, ctypes.c_float,
                              ctypes.c_float, u8p]),
    "orc_sk_mask": (None, [f32p, c_u64, f32p, c_u64, u8p, c_u64, c_int, c_int, c_uint]),
    "orc_sk_limits": (c_int, [c_uint, c_uint, ctypes.c_float, c_uint,
                              ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "orc_inverse_filterbank_f32": (c_i64, [ctypes.c_void_p, f32p, c_u64, c_u64, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, f32p, c_u64]),
    "orc_inverse_filterbank_f64": (c_i64, [ctypes.c_void_p, f64p, c_u64, c_u64, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, f64p, c_u64]),
    "orc_convolve_window_f32": (c_u64, [f32p, c_u64, c_u64, c_int, c_int, f32p, c_uint, c_uint,
                                        c_uint, f32p, c_u64, c_int, f32p]),
    "orc_apodization": (c_int, [c_int, c_uint, c_uint, c_uint, c_int, f32p]),
    "orc_pipeline_c1": (c_u64, [u8p, c_u64, f32p, f32p, c_uint, c_uint, c_uint, c_dbl, c_dbl,
                                c_uint, f32p, u32p, c_int]),
    "orc_channel_centre": (c_dbl, [c_dbl, c_dbl, c_uint, c_uint, c_int, c_int]),
    "orc_dedispersion_response_channels": (None, [f64p, c_uint, c_dbl, c_dbl, c_uint, c_int,
                                                  c_uint, f32p]),
    "orc_dedispersion_response_channels_delay": (None, [f64p, c_uint, c_dbl, c_dbl, c_uint, c_int,
                                                         c_uint, f64p, f32p]),
    "orc_dedispersion_response_channels_f64": (None, [f64p, c_uint, c_dbl, c_dbl, c_uint,
                                                      c_uint, f64p]),
    "orc_filterbank_f32": (c_u64, [f32p, c_u64, c_u64, c_int, c_int, c_uint, f32p, c_u64]),
    "orc_filterbank_f64": (c_u64, [f64p, c_u64, c_u64, c_int, c_int, c_uint, f64p, c_u64]),
    "orc_filterbank_during_f32": (c_u64, [f32p, c_u64, c_u64, c_int, c_int, c_uint, c_uint,
                                          c_uint, c_uint, f32p, f32p, c_u64, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "orc_filterbank_during_f64": (c_u64, [f64p, c_u64, c_u64, c_int, c_int, c_uint, c_uint,
                                          c_uint, c_uint, f64p, f64p, c_u64, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "orc_dedispersion_response_during": (None, [f64p, c_uint, c_dbl, c_dbl, c_uint, c_int, c_dbl,
                                                f32p]),
    "orc_dedispersion_response_during_f64": (None, [f64p, c_uint, c_dbl, c_dbl, c_uint, c_dbl,
                                                    f64p]),
}


def sk(x, M, lower, upper, Nd=1, zero_is_valid=True, ndat=None):
    """x: complex64 (nchan, npol, span); the first ndat (default span) samples
    of each span are used.  Returns sums (npart, nchan, npol, 2), counts
    (npart, nchan), mask (npart, nchan) uint8 and a copy of x whose first
    npart*M samples are masked."""
    nchan, npol, span = x.shape
    ndat = span if ndat is None else ndat
    x = np.ascontiguousarray(x, np.complex64)
    xf = x.view(np.float32).ravel()
    npart = ndat // M
    sums = np.zeros((npart, nchan, npol, 2), np.float32)
    counts = np.zeros((npart, nchan), np.uint32)
    lib().orc_sk_compute(xf, ndat, span, nchan, npol, M, int(zero_is_valid), sums.ravel(),
                         counts.ravel())
    mask = np.zeros((npart, nchan), np.uint8)
    lib().orc_sk_detect(sums.ravel(), counts.ravel(), npart, nchan, npol, Nd, lower, upper,
                        mask.ravel())
    out = x.copy()
    lib().orc_sk_mask(xf, span, out.view(np.float32).ravel(), span, mask.ravel(), npart, nchan,
                      npol, M)
    return sums, counts, mask, out


def sk_detect_tscr(sums, counts, Nd, std_devs):
    """SpectralKurtosis::detect_tscr (Signal/General/SpectralKurtosis.C:
    1012-1098) with noverlap 1: per channel, the count and the double sums of
    the float S1, S2 over all parts; the SK estimator against the limits of
    SKLimits(count, std_devs) with Nd and ntest = npol; a zapped channel is
    flagged in every part.  sums (npart, nchan, npol, 2) float32, counts
    (npart, nchan).  Returns the mask (npart, nchan) uint8 of these flags."""
    npart, nchan, npol, _ = sums.shape
    mask = np.zeros((npart, nchan), np.uint8)
    for c in range(nchan):
        count = int(np.sum(counts[:, c], dtype=np.uint64))
        if count == 0:
            continue
        lo, hi = sk_limits(count, Nd, std_devs, npol)
        M_t = np.float32(count)
        M_fac = np.float32((M_t * np.float32(Nd) + np.float32(1)) / (M_t - np.float32(1)))
        zap = False
        for p in range(npol):
            S1 = 0.0
            S2 = 0.0
            for ip in range(npart):                 # sequential double sums
                S1 += float(sums[ip, c, p, 0])
                S2 += float(sums[ip, c, p, 1])
            SK = float(M_fac) * (float(M_t) * (S2 / (S1 * S1)) - 1)
            if SK > float(hi) or SK < float(lo):
                zap = True
        if zap:
            mask[:, c] = 1
    return mask


def sk_resolution(M, noverlap, ndat):
    """Resolution::prepare (Signal/General/SpectralKurtosis.C:251-281):
    (overlap_offset, npart, output_ndat, idat_start)."""
    off = M // noverlap
    start = M - off
    if ndat < start:
        return off, 0, 0, start
    nblock = (ndat - start) // off
    end = nblock * off
    if end < start:
        return off, 0, 0, start
    return off, nblock, end - start, start


def sk_compute_overlap(x, M, noverlap, zero_is_valid=True, ndat=None):
    """SpectralKurtosis::compute (SpectralKurtosis.C:674-798) for the blocks
    Resolution::prepare gives: block b holds samples b*off ... b*off + M - 1;
    S1 and S2 of each (block, chan, pol) summed in order in double from the
    float sqld (S2 of its float square), the pol-0 count as the weight.
    Returns sums (npart, nchan, npol, 2) float32 and counts (npart, nchan)."""
    nchan, npol, span = x.shape
    ndat = span if ndat is None else ndat
    off, npart, _, _ = sk_resolution(M, noverlap, ndat)
    xr = np.ascontiguousarray(x.real, np.float32)
    xi = np.ascontiguousarray(x.imag, np.float32)
    sqld = xr * xr + xi * xi                              # float32, no contraction
    sums = np.zeros((npart, nchan, npol, 2), np.float32)
    counts = np.zeros((npart, nchan), np.uint32)
    for b in range(npart):
        blk = sqld[:, :, b * off:b * off + M]
        keep = np.ones_like(blk, bool) if zero_is_valid else blk != 0
        v1 = np.where(keep, blk, np.float32(0)).astype(np.float64)
        v2 = np.where(keep, blk * blk, np.float32(0)).astype(np.float64)
        # sequential double sums (adding +0.0 for skipped values changes nothing)
        sums[b, :, :, 0] = np.cumsum(v1, axis=2)[:, :, -1].astype(np.float32)
        sums[b, :, :, 1] = np.cumsum(v2, axis=2)[:, :, -1].astype(np.float32)
        counts[b] = keep[:, 0].sum(axis=1)
    return sums, counts


def sk_tscrunch(sums, counts, npart_to, nsum, offset):
    """SpectralKurtosis::tscrunch_sums (SpectralKurtosis.C:917-986): coarse
    part q adds the fine parts q*offset + i*offset, i < nsum, in that order
    (float sums, integer counts) -- the reference's indexing."""
    out = np.zeros((npart_to,) + sums.shape[1:], np.float32)
    oc = np.zeros((npart_to, counts.shape[1]), np.uint32)
    for q in range(npart_to):
        acc = sums[q * offset].copy()
        cc = counts[q * offset].astype(np.uint64)
        for i in range(1, nsum):
            acc = (acc + sums[q * offset + i * offset]).astype(np.float32)
            cc = cc + counts[q * offset + i * offset]
        out[q] = acc
        oc[q] = cc.astype(np.uint32)
    return out, oc


def sk_detect_skfb(sums, counts, Nd, std_devs, mask, nflag=1, flag_step=1, flag_offset=1):
    """SpectralKurtosis::detect_skfb (SpectralKurtosis.C:1105-1222) at one
    resolution, limits of SKLimits(count, std_devs) per count (get_limits,
    :988-1008) with npol tests; a zapped cell sets nflag fine mask cells from
    fine part q*flag_offset, flag_step apart.  Updates mask in place."""
    npart, nchan, npol, _ = sums.shape
    cache = {}
    for q in range(npart):
        for c in range(nchan):
            mp = int(counts[q, c])
            if mp == 0:
                continue
            zap = True
            if mp > 2:
                if mp not in cache:
                    cache[mp] = sk_limits(mp, Nd, std_devs, npol)
                lo, hi = cache[mp]
                m_fac = np.float32(mp * Nd + 1) / np.float32(mp - 1)
                zap = False
                for p in range(npol):
                    s1, s2 = sums[q, c, p, 0], sums[q, c, p, 1]
                    v = m_fac * (np.float32(mp) * (s2 / (s1 * s1)) - np.float32(1))
                    if v > hi or v < lo:
                        zap = True
            if zap:
                for f in range(nflag):
                    mask[q * flag_offset + f * flag_step, c] = 1
    return mask


def sk_mask_overlap(mask, x, M, offset, npart, nskip, idat_start):
    """SpectralKurtosis::mask (SpectralKurtosis.C:1465-1566): part after part,
    M samples from the input at idat_start + ipart*offset copied (or zeroed
    where mask[ipart + nskip] is set) to the output at ipart*offset."""
    nchan, npol, _ = x.shape
    out = np.zeros((nchan, npol, (npart - 1) * offset + M), x.dtype)
    for c in range(nchan):
        for p in range(npol):
            for ip in range(npart):
                a = ip * offset
                if mask[ip + nskip, c]:
                    out[c, p, a:a + M] = 0
                else:
                    out[c, p, a:a + M] = x[c, p, idat_start + a:idat_start + a + M]
    return out


def sk_limits(M, Nd=1, std_devs=3.0, ntest=1):
    """(lower, upper) float32 thresholds of SKLimits::calc_limits."""
    lo, hi = ctypes.c_float(), ctypes.c_float()
    rc = lib().orc_sk_limits(M, Nd, std_devs, ntest, ctypes.byref(lo), ctypes.byref(hi))
    if rc != 0:
        raise ValueError(f"sk_limits: invalid M={M} Nd={Nd} std_devs={std_devs} (rc {rc})")
    return np.float32(lo.value), np.float32(hi.value)


class IfbConfig(ctypes.Structure):
    """orc_ifb_config (oracle.h)."""
    _fields_ = [("input_nchan", c_uint), ("output_nchan", c_uint), ("pfb_nchan", c_uint),
                ("npol", c_uint), ("input_fft_length", c_uint), ("os_num", c_uint),
                ("os_den", c_uint), ("output_discard_pos", c_uint),
                ("output_discard_neg", c_uint), ("pfb_dc_chan", c_int), ("pfb_all_chan", c_int),
                ("dual_sideband", c_int)]


def ifb_sizes(cfg):
    """(keep, Lout, input_discard_pos, input_discard_neg, in_step, out_step)."""
    keep = cfg["input_fft_length"] * cfg["os_den"] // cfg["os_num"]
    lout = cfg["input_nchan"] // cfg["output_nchan"] * keep
    scale = cfg["output_nchan"] * cfg["os_num"], cfg["input_nchan"] * cfg["os_den"]
    ipos = cfg["output_discard_pos"] * scale[0] // scale[1]
    ineg = cfg["output_discard_neg"] * scale[0] // scale[1]
    return (keep, lout, ipos, ineg, cfg["input_fft_length"] - ipos - ineg,
            lout - cfg["output_discard_pos"] - cfg["output_discard_neg"])


def inverse_filterbank(x, cfg, response=None, temporal=None, spectral=None, fp64=False):
    """x: complex (input_nchan, npol, ndat).  cfg: dict of orc_ifb_config
    fields.  Returns complex (output_nchan, npol, npart*out_step)."""
    nin, npol, ndat = x.shape
    c = IfbConfig(**{k: int(v) for k, v in cfg.items()})
    keep, lout, ipos, ineg, in_step, out_step = ifb_sizes(cfg)
    npart = (ndat - ipos - ineg) // in_step if ndat > ipos + ineg else 0
    cdt, rdt = (np.complex128, np.float64) if fp64 else (np.complex64, np.float32)
    xin = np.ascontiguousarray(x, cdt)
    out = np.zeros((cfg["output_nchan"], npol, max(1, npart * out_step)), cdt)

    def opt(a, dt):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, dt)
        return a, a.ctypes.data
    r, rp = opt(response, cdt)
    t, tp = opt(temporal, rdt)
    sp_, spp = opt(spectral, rdt)
    f = lib().orc_inverse_filterbank_f64 if fp64 else lib().orc_inverse_filterbank_f32
    n = f(ctypes.addressof(c), xin.view(rdt).ravel(), ndat, ndat, rp, tp, spp,
          out.view(rdt).ravel(), out.shape[2])
    if n < 0:
        raise ValueError("inverse_filterbank: invalid configuration")
    assert n == npart
    return out[:, :, :npart * out_step]


def channel_centres(cf, bw, nchan, swap=False, dc_centred=False):
    return np.array([lib().orc_channel_centre(cf, bw, nchan, i, int(swap), int(dc_centred))
                     for i in range(nchan)], np.float64)


def dedispersion_response_channels(chan_freq, bw, dm, ndat, mode=0, norm_nfft=None, fp64=False,
                                   frac_delay_us=None):
    chan_freq = np.ascontiguousarray(chan_freq, np.float64)
    nchan = chan_freq.size
    if frac_delay_us is not None:
        assert not fp64
        out = np.empty(nchan * ndat, np.complex64)
        lib().orc_dedispersion_response_channels_delay(
            chan_freq, nchan, bw, dm, ndat, mode, norm_nfft or ndat,
            np.ascontiguousarray(frac_delay_us, np.float64), out.view(np.float32))
        return out.reshape(nchan, ndat)
    if fp64:
        out = np.empty(nchan * ndat, np.complex128)
        lib().orc_dedispersion_response_channels_f64(chan_freq, nchan, bw, dm, ndat,
                                                     norm_nfft or ndat, out.view(np.float64))
    else:
        out = np.empty(nchan * ndat, np.complex64)
        lib().orc_dedispersion_response_channels(chan_freq, nchan, bw, dm, ndat, mode,
                                                 norm_nfft or ndat, out.view(np.float32))
    return out.reshape(nchan, ndat)


def filterbank(x, nsub):
    """x: complex (nchan_in, npol, ndat) -> (nchan_in*nsub, npol, ndat//nsub)."""
    nchan, npol, ndat = x.shape
    nout = ndat // nsub
    if x.dtype == np.complex64:
        out = np.zeros((nchan * nsub, npol, nout), np.complex64)
        lib().orc_filterbank_f32(np.ascontiguousarray(x).view(np.float32).ravel(), ndat, ndat,
                                 nchan, npol, nsub, out.view(np.float32).ravel(), nout)
    else:
        out = np.zeros((nchan * nsub, npol, nout), np.complex128)
        lib().orc_filterbank_f64(np.ascontiguousarray(x, np.complex128).view(np.float64).ravel(),
                                 ndat, ndat, nchan, npol, nsub, out.view(np.float64).ravel(), nout)
    return out


def dedispersion_response_during(cf, bw, dm, nchan, freq_res, nsamp_fft, swapped=True, mode=0,
                                 fp64=False):
    """The filterbank-with-response (During) dedispersion response,
    [nchan][freq_res] as Response holds it after swap_as_needed: Dedispersion
    prepared for the nchan output channels (Filterbank.C:101-110), each channel
    in natural frequency order, the whole response swapped when the input is
    one dual-sideband channel (Response.C:336-345, 998-1050) -- a rotation by
    nchan/2 whole channels -- and the normaliser 1/sqrt(nsamp_fft*freq_res)
    (Filterbank.C:171-186)."""
    chan_freq = channel_centres(cf, bw, nchan, swap=swapped)
    norm = float(nsamp_fft) * float(freq_res)
    if fp64:
        out = np.empty(nchan * freq_res, np.complex128)
        lib().orc_dedispersion_response_during_f64(chan_freq, nchan, bw, dm, freq_res, norm,
                                                   out.view(np.float64))
    else:
        out = np.empty(nchan * freq_res, np.complex64)
        lib().orc_dedispersion_response_during(chan_freq, nchan, bw, dm, freq_res, mode, norm,
                                               out.view(np.float32))
    return out.reshape(nchan, freq_res)


def filterbank_during(x, nsub, freq_res, nfilt, response, temporal=None, spectral=None):
    """x: complex (nchan_in, npol, ndat); response [nchan_in*nsub][freq_res];
    optional float windows temporal (nsub*freq_res) and spectral (freq_res) ->
    (nchan_in*nsub, npol, npart*(freq_res - nfilt_pos - nfilt_neg))."""
    nchan, npol, ndat = x.shape
    pos, neg = nfilt
    nkeep = freq_res - pos - neg
    overlap = (pos + neg) * nsub
    npart = (ndat - overlap) // (nsub * nkeep) if ndat > overlap else 0
    if x.dtype == np.complex64:
        dt, rdt, f = np.complex64, np.float32, lib().orc_filterbank_during_f32
    else:
        dt, rdt, f = np.complex128, np.float64, lib().orc_filterbank_during_f64
    xin = np.ascontiguousarray(x, dt)
    r = np.ascontiguousarray(response, dt)
    assert r.shape == (nchan * nsub, freq_res)
    out = np.zeros((nchan * nsub, npol, max(npart * nkeep, 1)), dt)
    tw = None if temporal is None else np.ascontiguousarray(temporal, np.float32)
    sw = None if spectral is None else np.ascontiguousarray(spectral, np.float32)
    assert tw is None or tw.size == nsub * freq_res
    assert sw is None or sw.size == freq_res
    n = f(xin.view(rdt).ravel(), ndat, ndat, nchan, npol, nsub, freq_res, pos, neg,
          r.view(rdt).ravel(), out.view(rdt).ravel(), out.shape[2],
          None if tw is None else tw.ctypes.data, None if sw is None else sw.ctypes.data)
    assert n == npart
    return out[:, :, :npart * nkeep]


def build():
    """Compile the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


# ---- thin numpy helpers --------------------------------------------------

def fft(x, sign=-1):
    """Unnormalised complex FFT of a complex64/complex128 vector (FFTW conventions)."""
    x = np.ascontiguousarray(x)
    n = x.shape[0]
    if x.dtype == np.complex64:
        out = np.empty(n, np.complex64)
        lib().orc_fft_f32(n, sign, x.view(np.float32), out.view(np.float32))
    else:
        x = x.astype(np.complex128)
        out = np.empty(n, np.complex128)
        lib().orc_fft_f64(n, sign, x.view(np.float64), out.view(np.float64))
    return out


def bittable8(spacing, twos_complement=True):
    lut = np.empty(256, np.float32)
    scale = c_dbl()
    lib().orc_bittable8(spacing, int(twos_complement), lut, ctypes.byref(scale))
    return lut, scale.value


def unpack8(raw, ndat, nchan, npol, ndim, lut):
    """TFPD uint8 bytes -> FPT float32 array of shape (nchan, npol, ndat*ndim)."""
    out = np.empty((nchan, npol, ndat * ndim), np.float32)
    lib().orc_unpack8(np.ascontiguousarray(raw.view(np.uint8).ravel()), ndat, nchan, npol,
                      ndim, lut, out.reshape(-1), ndat * ndim)
    return out


def unpack16(raw, ndat, nchan, npol, ndim, offset_binary=False):
    out = np.empty((nchan, npol, ndat * ndim), np.float32)
    lib().orc_unpack16(np.ascontiguousarray(raw.view(np.int16).ravel()), ndat, nchan, npol,
                       ndim, int(offset_binary), out.reshape(-1), ndat * ndim)
    return out


def smearing_samples(cf, bw, dm, nchan, half):
    return lib().orc_smearing_samples(cf, bw, dm, nchan, half)


def minimum_ndat(pos, neg):
    return lib().orc_minimum_ndat(pos, neg)


def optimal_fft_length(nbad, nmax=0, factor=1):
    return lib().orc_optimal_fft_length(nbad, nmax, factor)


def dedispersion_response(cf, bw, dm, nchan, ndat, input_nchan=1, dual_sideband=1,
                          dc_centred=0, mode=0, norm_nfft=None):
    out = np.empty(nchan * ndat, np.complex64)
    lib().orc_dedispersion_response(cf, bw, dm, nchan, ndat, input_nchan, dual_sideband,
                                    dc_centred, mode, norm_nfft or ndat, out.view(np.float32))
    return out.reshape(nchan, ndat)


def dedispersion_response_f64(cf, bw, dm, nchan, ndat, input_nchan=1, dual_sideband=1,
                              dc_centred=0, norm_nfft=None):
    out = np.empty(nchan * ndat, np.complex128)
    lib().orc_dedispersion_response_f64(cf, bw, dm, nchan, ndat, input_nchan, dual_sideband,
                                        dc_centred, norm_nfft or ndat, out.view(np.float64))
    return out.reshape(nchan, ndat)


def tukey_response(neg, pos, ndat):
    spec = np.empty(ndat, np.complex64)
    temp = np.empty(neg + pos, np.complex64)
    lib().orc_tukey_response(neg, pos, ndat, spec.view(np.float32), temp.view(np.float32))
    return spec, temp


def convolve(x, response, nfft, nfilt_pos, nfilt_neg, nthreads=8):
    """x: complex (nchan, npol, ndat); response: complex (nchan, nfft).
    Returns the (nchan, npol, npart*nkeep) overlap-save output."""
    nchan, npol, ndat = x.shape
    nkeep = nfft - nfilt_pos - nfilt_neg
    npart = (ndat - nfilt_pos - nfilt_neg) // nkeep if ndat >= nfft else 0
    if x.dtype == np.complex64:
        out = np.zeros((nchan, npol, npart * nkeep), np.complex64)
        r = np.ascontiguousarray(response, np.complex64)
        lib().orc_convolve_f32(np.ascontiguousarray(x).view(np.float32).ravel(), ndat, ndat,
                               nchan, npol, r.view(np.float32).ravel(), nfft, nfilt_pos,
                               nfilt_neg, out.view(np.float32).ravel(), npart * nkeep, nthreads)
    else:
        out = np.zeros((nchan, npol, npart * nkeep), np.complex128)
        r = np.ascontiguousarray(response, np.complex128)
        lib().orc_convolve_f64(np.ascontiguousarray(x, np.complex128).view(np.float64).ravel(),
                               ndat, ndat, nchan, npol, r.view(np.float64).ravel(), nfft,
                               nfilt_pos, nfilt_neg, out.view(np.float64).ravel(),
                               npart * nkeep, nthreads)
    return out


def convolve_window(x, response, nfft, nfilt_pos, nfilt_neg, window, nthreads=8):
    """convolve() with a temporal window (nfft floats) on every part."""
    nchan, npol, ndat = x.shape
    nkeep = nfft - nfilt_pos - nfilt_neg
    npart = (ndat - nfilt_pos - nfilt_neg) // nkeep if ndat >= nfft else 0
    out = np.zeros((nchan, npol, npart * nkeep), np.complex64)
    r = np.ascontiguousarray(response, np.complex64)
    lib().orc_convolve_window_f32(np.ascontiguousarray(x, np.complex64).view(np.float32).ravel(),
                                  ndat, ndat, nchan, npol, r.view(np.float32).ravel(), nfft,
                                  nfilt_pos, nfilt_neg, out.view(np.float32).ravel(),
                                  npart * nkeep, nthreads,
                                  np.ascontiguousarray(window, np.float32))
    return out


def apodization(kind, ndat, transition_start=0, transition_end=0, swap=False):
    w = np.zeros(ndat, np.float32)
    if lib().orc_apodization(kind, ndat, transition_start, transition_end, int(swap), w) != 0:
        raise ValueError("apodization: invalid type or size")
    return w


STATES = {"Intensity": 0, "PPQQ": 1, "Coherence": 2, "Stokes": 3}
NOUT = {0: 1, 1: 2, 2: 4, 3: 4}


def detect(x, state):
    """x: complex (nchan, 2, ndat) -> float (nchan, nout, ndat)."""
    state = STATES.get(state, state)
    nchan, npol, ndat = x.shape
    assert npol == 2
    nout = NOUT[state]
    if x.dtype == np.complex64:
        out = np.empty((nchan, nout, ndat), np.float32)
        lib().orc_detect(np.ascontiguousarray(x).view(np.float32).ravel(), ndat, ndat, nchan,
                         state, out.ravel(), ndat)
    else:
        out = np.empty((nchan, nout, ndat), np.float64)
        lib().orc_detect_f64(np.ascontiguousarray(x, np.complex128).view(np.float64).ravel(),
                             ndat, ndat, nchan, state, out.ravel(), ndat)
    return out


def fold_phi(start_mjd, epoch_mjd, idat_start, rate, period, reference_phase=0.0):
    return lib().orc_fold_phi(start_mjd[0], start_mjd[1], start_mjd[2], epoch_mjd[0],
                              epoch_mjd[1], epoch_mjd[2], idat_start, rate, period,
                              reference_phase)


def fold_binplan(phi, phase_per_sample, ndat, nbin):
    out = np.empty(ndat, np.uint32)
    lib().orc_fold_binplan(phi, phase_per_sample, ndat, nbin, out)
    return out


def fold_accumulate(data, binplan, nbin, profiles=None, hits=None):
    """data: float (nchan, npol, ndat) (ndim 1).  Returns profiles (nchan,npol,nbin), hits."""
    nchan, npol, ndat = data.shape
    f64 = data.dtype == np.float64
    if profiles is None:
        profiles = np.zeros((nchan, npol, nbin), np.float64 if f64 else np.float32)
    if hits is None:
        hits = np.zeros(nbin, np.uint32)
    fn = lib().orc_fold_accumulate_f64 if f64 else lib().orc_fold_accumulate
    fn(np.ascontiguousarray(data).ravel(), ndat, ndat, nchan, npol, 1,
       np.ascontiguousarray(binplan, np.uint32), nbin, profiles.reshape(-1), hits)
    return profiles, hits


def fold_accumulate_zeroed(data, binplan, nbin, profiles, hits):
    """Fold::fold of data with zeroed samples (Signal/Pulsar/Fold.C:895-930,
    zeroed_samples true, one hits array for all channels): every sample is
    added to its bin in sequence (zeroed ones add nothing); a hit is counted
    for each channel sample whose first polarisation's value is non-zero.
    data: float (nchan, npol, ndat); profiles (nchan, npol, nbin) and hits
    (nbin) are updated in place."""
    scratch = np.zeros_like(hits)
    fold_accumulate(data, binplan, nbin, profiles, scratch)
    plan = np.asarray(binplan, np.int64)
    for c in range(data.shape[0]):
        np.add.at(hits, plan[data[c, 0] != 0], 1)
    return profiles, hits


def pipeline_c1(raw, ndat, lut, response, nfft, nfilt_pos, nfilt_neg, phi, pps, nbin,
                nthreads=8):
    prof = np.zeros(nbin, np.float32)
    hits = np.zeros(nbin, np.uint32)
    n = lib().orc_pipeline_c1(np.ascontiguousarray(raw.view(np.uint8).ravel()), ndat, lut,
                              np.ascontiguousarray(response, np.complex64).view(np.float32).ravel(),
                              nfft, nfilt_pos, nfilt_neg, phi, pps, nbin, prof, hits, nthreads)
    return prof, hits, n


# ---------------------------------------------------------------------------
# TimeDivide (Signal/Pulsar/TimeDivide.C) and the block loop of Subint<Fold>
# (Signal/Pulsar/dsp/Subint.h:206-362), pure Python.  MJDs are
# (day, second, fraction) tuples; the arithmetic follows PSRCHIVE's MJD
# (whole days and seconds plus a fraction), which is not in the reference
# tree, so it is restated, not pinned.
# ---------------------------------------------------------------------------

import math


def mjd_add(m, seconds):
    day, sec, frac = m
    f = frac + seconds
    whole = math.floor(f)
    frac = f - whole
    d, s = divmod(sec + int(whole), 86400)
    return (day + d, s, frac)


def mjd_diff(a, b):
    """(a - b).in_seconds()"""
    return float((a[0] - b[0]) * 86400 + (a[1] - b[1])) + (a[2] - b[2])


def _rint(x):
    return int(round(x))          # half to even, as rint / lrint


class TimeDivideOracle:
    """TimeDivide with a length in seconds, or in turns of a constant period."""

    def __init__(self, seconds=0.0, turns=0.0, period=0.0, reference_epoch=(0, 0, 0.0)):
        self.seconds, self.turns, self.period = seconds, turns, period
        self.reference_epoch = tuple(reference_epoch)
        self.start_time = (0, 0, 0.0)
        self.lower = self.upper = self.current_end = (0, 0, 0.0)
        self.is_valid = False
        self.division = 0

    # TimeDivide.C:40-76
    def set_start_time(self, t):
        if self.start_time == tuple(t):
            return
        self.start_time = tuple(t)
        self.is_valid = False
        if self.reference_epoch != (0, 0, 0.0):
            self.start_time = self.reference_epoch
        elif self.seconds and self.seconds == float(int(self.seconds)):
            isec = int(self.seconds)
            day, sec, _ = self.start_time
            self.start_time = (day, (sec // isec) * isec, 0.0)

    # TimeDivide.C:503-537
    def _round_bounds(self, m1, m2, obs_start, rate):
        samples = _rint(mjd_diff(m1, obs_start) * rate)
        self.lower = mjd_add(obs_start, samples / rate)
        self.division_ndat = _rint(mjd_diff(m2, self.lower) * rate)
        self.upper = mjd_add(self.lower, self.division_ndat / rate)

    # TimeDivide.C:349-501 (no predictor)
    def _set_boundaries(self, t, obs_start, rate):
        divide_start = max(self.start_time, t)
        spi = self.seconds if not self.turns else self.period * self.turns
        self.division = int(mjd_diff(divide_start, self.start_time) / spi)
        self._round_bounds(mjd_add(self.start_time, self.division * spi),
                           mjd_add(self.start_time, (self.division + 1) * spi), obs_start, rate)

    # TimeDivide.C:130-333
    def set_bounds(self, start, ndat, rate):
        start = tuple(start)
        end = mjd_add(start, ndat / rate) if ndat else start
        divide_start = max(self.current_end, start) if self.is_valid else start
        self.new_division = self.end_reached = self.in_next = False
        if end < self.lower or self.upper < mjd_add(divide_start, 0.5 / rate):
            self.new_division = True
            self._set_boundaries(mjd_add(divide_start, 0.55 / rate), start, rate)
        divide_start = max(self.lower, divide_start)
        self.idat_start = _rint(mjd_diff(divide_start, start) * rate)
        if self.idat_start >= ndat:
            self.is_valid = False
            return
        divide_end = min(end, self.upper)
        idat_end = _rint(mjd_diff(divide_end, start) * rate)
        assert idat_end > self.idat_start
        if idat_end > ndat:
            idat_end = ndat
        elif idat_end < ndat:
            self.in_next = True
        self.ndat = idat_end - self.idat_start
        if mjd_diff(self.upper, divide_end) * rate < 0.5:
            self.end_reached = True
        self.is_valid = True
        self.current_end = mjd_add(start, idat_end / rate)


def subint_block_actions(td, start, ndat, rate):
    """Subint<Fold>::transformation for one block (Subint.h:258-332): a list
    of ("fold", idat_start, ndat, division, end_reached) and ("close", kind)
    steps, kind "partial" or "complete"."""
    if td.start_time == (0, 0, 0.0):
        td.set_start_time(start)
    out = []
    more, first = True, True
    while more:
        td.set_bounds(start, ndat, rate)
        more = td.in_next
        if first and td.new_division:
            out.append(("close", "partial"))
        if not td.is_valid:
            continue
        out.append(("fold", td.idat_start, td.ndat, td.division, td.end_reached,
                    td.lower, td.upper))
        if not td.end_reached:
            continue
        if first:
            out.append(("close", "partial"))
            first = False
            continue
        out.append(("close", "complete"))
    return out


# ---------------------------------------------------------------------------
# Inter-channel dispersion delays: Dedispersion::SampleDelay
# (Signal/General/DedispersionSampleDelay.C:26-140) and SampleDelay::build /
# transformation (Signal/General/SampleDelay.C:65-298), pure Python.
# ---------------------------------------------------------------------------

def interchannel_delays(cf, dm, rate, chan_freq):
    dispersion = dm / 2.41e-4
    delay, frac = [], []
    for f in chan_freq:
        sample_delay = dispersion * (1.0 / (cf * cf) - 1.0 / (f * f)) * rate
        d = math.floor(sample_delay + 0.5)
        delay.append(int(d))
        frac.append(sample_delay - d)
    fm = (chan_freq[0] + chan_freq[-1]) / 2
    span = int(math.floor(dispersion * (1.0 / (cf * cf) - 1.0 / (fm * fm)) * rate + 0.5))
    zero = max([0] + [d - span for d in delay])
    zd = span + zero
    total = max([0] + [zd - d for d in delay])
    applied = [zd - d if zero else d for d in delay]
    return dict(delay=np.array(delay, np.int64), frac=np.array(frac), applied=np.array(applied),
                zero_delay=zero, total_delay=total)


def sample_delay_block(y, applied, total):
    """SampleDelay::transformation on one block y [chan][pol][t]: output
    [chan][pol][t] = y[chan][pol][t + applied[chan]] for t < ndat - total."""
    n = y.shape[2] - total
    if n <= 0:
        return y[:, :, :0]
    out = np.empty(y.shape[:2] + (n,), y.dtype)
    for c in range(y.shape[0]):
        out[c] = y[c, :, applied[c]:applied[c] + n]
    return out


def archive_profiles(sums, hits, scale=1.0, zeroed_data=False, ndat_total=0,
                     unload_zero_hits=False):
    """Archiver::set(Pulsar::Profile*) (Signal/Pulsar/Archiver.C:852-984) and the
    channel weights of Archiver::set(Integration*) (:740-792), restated with
    Python scalars: amp = float32(float64(sum) / (scale * float64(hits)));
    unhit bins 0, or (unload_zero_hits) the float64 mean of the hit bins; a
    non-finite sum zeroes its profile and the channel's weight; weights 1, or
    float32(hits_sum) / float32(ndat_total) for zeroed data.  Raises
    ValueError where the reference throws for unhit bins."""
    sums = np.asarray(sums, np.float32)
    nchan, npol, nbin = sums.shape
    hits = np.asarray(hits, np.uint32).reshape(nchan if zeroed_data else 1, nbin)
    amps = np.zeros_like(sums)
    weights = np.ones(nchan, np.float32)
    corrupted = 0
    for ic in range(nchan):
        h = hits[ic if zeroed_data else 0]
        bad_chan = False
        w = np.float32(1.0)
        for ip in range(npol):
            src = sums[ic, ip]
            out = amps[ic, ip]
            zeroes = not_finite = 0
            hits_sum = 0
            for ib in range(nbin):
                hits_sum = (hits_sum + int(h[ib])) & 0xffffffff
                if h[ib] == 0:
                    zeroes += 1
                    out[ib] = 0.0
                elif not np.isfinite(src[ib]):
                    not_finite += 1
                else:
                    out[ib] = np.float32(float(src[ib]) / (scale * float(h[ib])))
            if not_finite:
                out[:] = 0.0
                bad_chan = True
                corrupted += 1
            if zeroes:
                if not unload_zero_hits:
                    raise ValueError("bins without hits")
                tot, cnt = 0.0, 0
                for ib in range(nbin):
                    if h[ib] != 0:
                        tot += float(out[ib])
                        cnt += 1
                mean = tot / max(cnt, 1)
                for ib in range(nbin):
                    if h[ib] == 0:
                        out[ib] = np.float32(mean)
            if zeroed_data:
                w = np.float32(np.float32(hits_sum) / np.float32(ndat_total))
        weights[ic] = 0.0 if bad_chan else w
    return amps, weights, corrupted
