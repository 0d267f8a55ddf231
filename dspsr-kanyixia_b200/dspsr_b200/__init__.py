"""Host-side interface to the B200 engine of DSPSR's baseband hot path.

This module mirrors the reference's operation / engine interfaces over the
C ABI of libdspsr_b200.so (include/dspsr_b200.h):

  Unpacker           -> unpack8 / unpack16      (GenericEightBitUnpacker, SixteenBitUnpacker)
  Convolution engine -> Convolution             (CUDA::ConvolutionEngine)
  Filterbank engine  -> FilterbankDuring        (Filterbank with a response, -F N:D)
  InverseFilterbank  -> InverseFilterbank       (InverseFilterbank::Engine)
  Detection engine   -> detect                  (CUDA::DetectionEngine)
  Fold engine        -> Fold                    (CUDA::FoldEngine with use_set_bins)
  SingleThread loop  -> Pipeline                (unpack -> convolve -> detect -> fold)
  DADAFile / header  -> DADAFile, dada_parse, ascii_header_get/_set (file source of the loop)

Device buffers are torch CUDA tensors (torch is only the allocator and stream
provider here); every computation runs in the library's sm_100a kernels.
"""
import ctypes
import os
import weakref

import numpy as np

from . import _capi
from ._capi import (B200Error, PipelineConfig, INTENSITY, PPQQ, COHERENCE, STOKES, INT8_TFPD,
                    INT16_TFPD, FLOAT_FPT, CHIRP_REFERENCE, CHIRP_FP64, FFT_FP32, FFT_BF16X2,
                    FFT_BF16X3)

__all__ = ["Context", "Convolution", "RfiProposer", "InverseFilterbank", "FilterbankDuring", "Fold", "apodization", "Pipeline", "PipelineConfig", "B200Error",
           "smearing_samples", "minimum_ndat", "optimal_fft_length", "bittable8", "fold_phi",
           "sk_limits", "DADAFile", "dada_parse", "dada_is_valid", "ascii_header_get",
           "ascii_header_set", "write_dada", "TimeDivide", "interchannel_delays",
           "fold_plan_count", "archive_profiles", "INTENSITY", "PPQQ", "COHERENCE", "STOKES", "INT8_TFPD",
           "INT16_TFPD", "FLOAT_FPT", "CHIRP_REFERENCE", "CHIRP_FP64", "NOUT",
           "FFT_FP32", "FFT_BF16X2", "FFT_BF16X3"]

NOUT = {INTENSITY: 1, PPQQ: 2, COHERENCE: 4, STOKES: 4}
# Jenet & Anderson (1998) optimal uniform-quantiser input spacing for 8 bits
JA98_SPACING_8BIT = 0.0308


def _ptr(x):
    """Device pointer of a torch tensor (or an int address)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


# ---- host rules ---------------------------------------------------------------

def smearing_samples(centre_freq, bandwidth, dm, nchan, half):
    return _capi.lib().dspsr_b200_smearing_samples(centre_freq, bandwidth, dm, nchan, half)


def minimum_ndat(impulse_pos, impulse_neg):
    return _capi.lib().dspsr_b200_minimum_ndat(impulse_pos, impulse_neg)


def optimal_fft_length(nbad, nfft_max=0, factor=1):
    return _capi.lib().dspsr_b200_optimal_fft_length(nbad, nfft_max, factor)


def bittable8(spacing=JA98_SPACING_8BIT, twos_complement=True):
    lut = np.empty(256, np.float32)
    scale = ctypes.c_double()
    rc = _capi.lib().dspsr_b200_bittable8(spacing, int(twos_complement), _fptr(lut),
                                          ctypes.byref(scale))
    if rc:
        raise B200Error(rc, "bittable8: invalid spacing")
    return lut, scale.value


def sk_limits(M, Nd=1, std_devs=3.0, ntest=1):
    """SKLimits::calc_limits -> (lower, upper) float32 thresholds."""
    lo = np.zeros(1, np.float32)
    hi = np.zeros(1, np.float32)
    rc = _capi.lib().dspsr_b200_sk_limits(M, Nd, std_devs, ntest, _fptr(lo), _fptr(hi))
    if rc != _capi.OK:
        raise B200Error(rc, f"sk_limits: no thresholds for M={M} Nd={Nd} std_devs={std_devs}")
    return lo[0], hi[0]


APOD_TOPHAT, APOD_HANNING, APOD_WELCH, APOD_BARTLETT, APOD_TUKEY = range(5)


def apodization(kind, ndat, transition_start=0, transition_end=0, swap_halves=False):
    """Apodization::build: the float window of ndat points."""
    w = np.zeros(ndat, np.float32)
    rc = _capi.lib().dspsr_b200_apodization(kind, ndat, transition_start, transition_end,
                                           int(swap_halves), _fptr(w))
    if rc != _capi.OK:
        raise B200Error(rc, f"apodization: invalid type {kind} or size {ndat}")
    return w


def archive_profiles(sums, hits, scale=1.0, zeroed_data=False, ndat_total=0,
                     unload_zero_hits=False):
    """Archiver::set for one sub-integration's profiles: sums (nchan, npol,
    nbin), hits (nbin,) or (nchan, nbin) when zeroed_data -> (amps, weights,
    corrupted)."""
    s = np.ascontiguousarray(sums, np.float32)
    nchan, npol, nbin = s.shape
    h = np.ascontiguousarray(hits, np.uint32)
    assert h.size == (nchan * nbin if zeroed_data else nbin)
    amps = np.empty_like(s)
    weights = np.empty(nchan, np.float32)
    bad = ctypes.c_uint()
    rc = _capi.lib().dspsr_b200_archive_profiles(
        _fptr(s), h.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), int(zeroed_data), nchan,
        npol, nbin, scale, ndat_total, int(unload_zero_hits), _fptr(amps), _fptr(weights),
        ctypes.byref(bad))
    if rc:
        raise B200Error(rc, "archive_profiles: " + ("bins without hits" if rc == _capi.ESTATE
                                                    else "invalid argument"))
    return amps, weights, bad.value


def fold_phi(start_mjd, epoch_mjd, idat_start, rate, period, reference_phase=0.0):
    return _capi.lib().dspsr_b200_fold_phi(start_mjd[0], start_mjd[1], start_mjd[2],
                                           epoch_mjd[0], epoch_mjd[1], epoch_mjd[2], idat_start,
                                           rate, period, reference_phase)


def interchannel_delays(centre_freq, dm, rate, chan_freq):
    """Dedispersion::SampleDelay + SampleDelay::build for channels centred at
    chan_freq: dict of delay, frac, applied (arrays), zero_delay, total_delay."""
    f = np.ascontiguousarray(chan_freq, np.float64)
    n = f.size
    delay = np.empty(n, np.int64)
    frac = np.empty(n, np.float64)
    applied = np.empty(n, np.int64)
    zd = ctypes.c_int64()
    td = ctypes.c_uint64()
    P64 = ctypes.POINTER(ctypes.c_int64)
    PD = ctypes.POINTER(ctypes.c_double)
    rc = _capi.lib().dspsr_b200_interchannel_delays(
        centre_freq, dm, rate, f.ctypes.data_as(PD), n, delay.ctypes.data_as(P64),
        frac.ctypes.data_as(PD), applied.ctypes.data_as(P64), ctypes.byref(zd), ctypes.byref(td))
    if rc:
        raise B200Error(rc, "interchannel_delays: invalid argument")
    return dict(delay=delay, frac=frac, applied=applied, zero_delay=zd.value,
                total_delay=td.value)


def kernel_launches():
    """Kernels the library has launched since it was loaded."""
    return _capi.lib().dspsr_b200_kernel_launches()


def fold_plan_count(phi, phase_per_sample, ndat):
    return _capi.lib().dspsr_b200_fold_plan_count(phi, phase_per_sample, ndat)


# ---- context ----------------------------------------------------------------------

class Context:
    """A device and a stream (CUDA::DeviceMemory(stream) in the reference)."""

    def __init__(self, device=0, stream=None):
        self._lib = _capi.lib()
        h = ctypes.c_void_p()
        rc = self._lib.dspsr_b200_context_create(device, stream, ctypes.byref(h))
        if rc:
            raise B200Error(rc, f"context_create(device={device}) failed")
        self.handle = h
        # engines made on this context: released before it
        self._children = weakref.WeakSet()

    def _adopt(self, child):
        self._children.add(child)

    def check(self, rc, what=""):
        if rc:
            msg = self._lib.dspsr_b200_last_error(self.handle)
            raise B200Error(rc, f"{what}: {msg.decode() if msg else ''}")

    def set_stream(self, stream):
        self.check(self._lib.dspsr_b200_context_set_stream(self.handle, stream), "set_stream")

    def synchronize(self):
        self.check(self._lib.dspsr_b200_synchronize(self.handle), "synchronize")

    def close(self):
        if self.handle:
            for child in list(self._children):
                child.close()
            self._lib.dspsr_b200_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- Unpacker ---------------------------------------------------------------
    def unpack8(self, d_in, ndat, nchan, npol, ndim, lut, d_out, out_span):
        lut = np.ascontiguousarray(lut, np.float32)
        self.check(self._lib.dspsr_b200_unpack8(self.handle, _ptr(d_in), ndat, nchan, npol, ndim,
                                                _fptr(lut), _ptr(d_out), out_span), "unpack8")

    def unpack16(self, d_in, ndat, nchan, npol, ndim, d_out, out_span, offset_binary=False):
        self.check(self._lib.dspsr_b200_unpack16(self.handle, _ptr(d_in), ndat, nchan, npol, ndim,
                                                 int(offset_binary), _ptr(d_out), out_span),
                   "unpack16")

    # ---- Filterbank engine (freq_res = 1) -------------------------------------------
    def filterbank(self, input_kind, d_in, ndat, nchan_in, npol, nsub, d_out, out_span,
                   in_span=0, lut=None, offset_binary=False):
        """Returns the output samples per channel (ndat // nsub)."""
        n = ctypes.c_uint64()
        lp = _fptr(np.ascontiguousarray(lut, np.float32)) if lut is not None else None
        self.check(self._lib.dspsr_b200_filterbank(self.handle, input_kind, _ptr(d_in), ndat,
                                                   in_span, nchan_in, npol, nsub, lp,
                                                   int(offset_binary), _ptr(d_out), out_span,
                                                   ctypes.byref(n)), "filterbank")
        return n.value

    # ---- Detection engine ----------------------------------------------------------
    def detect(self, d_in, in_span, ndat, nchan, state, d_out, out_span):
        self.check(self._lib.dspsr_b200_detect(self.handle, _ptr(d_in), in_span, ndat, nchan,
                                               state, _ptr(d_out), out_span), "detect")

    # ---- SpectralKurtosis engine, step by step --------------------------------------
    def sk_compute(self, d_in, in_span, ndat, nchan, npol, M, d_sums, d_counts=None,
                   zero_is_valid=True, noverlap=1):
        n = ctypes.c_uint64()
        self.check(self._lib.dspsr_b200_sk_compute(self.handle, _ptr(d_in), in_span, ndat, nchan,
                                                   npol, M, noverlap, int(zero_is_valid),
                                                   _ptr(d_sums), _ptr(d_counts),
                                                   ctypes.byref(n)), "sk_compute")
        return n.value

    def sk_tscrunch(self, d_sums, d_counts, npart_from, npart_to, nchan, npol, nsum, offset,
                    d_sums_out, d_counts_out):
        self.check(self._lib.dspsr_b200_sk_tscrunch(self.handle, _ptr(d_sums), _ptr(d_counts),
                                                    npart_from, npart_to, nchan, npol, nsum,
                                                    offset, _ptr(d_sums_out), _ptr(d_counts_out)),
                   "sk_tscrunch")

    def sk_detect_skfb(self, d_sums, d_counts, npart, nchan, npol, std_devs, d_mask, mask_npart,
                       nflag=1, flag_step=1, flag_offset=1, Nd=1, d_zapped=None):
        self.check(self._lib.dspsr_b200_sk_detect_skfb(self.handle, _ptr(d_sums), _ptr(d_counts),
                                                       npart, nchan, npol, Nd, std_devs, nflag,
                                                       flag_step, flag_offset, _ptr(d_mask),
                                                       mask_npart, _ptr(d_zapped)),
                   "sk_detect_skfb")

    def sk_mask_overlap(self, d_mask, d_in, in_span, d_out, out_span, nchan, npol, M, offset,
                        npart, nskip, idat_start):
        self.check(self._lib.dspsr_b200_sk_mask_overlap(self.handle, _ptr(d_mask), _ptr(d_in),
                                                        in_span, _ptr(d_out), out_span, nchan,
                                                        npol, M, offset, npart, nskip,
                                                        idat_start), "sk_mask_overlap")

    def sk_detect_ft(self, d_sums, d_counts, npart, nchan, npol, M, lower, upper, d_mask,
                     Nd=1, d_zapped=None):
        self.check(self._lib.dspsr_b200_sk_detect_ft(self.handle, _ptr(d_sums), _ptr(d_counts),
                                                     npart, nchan, npol, M, Nd, lower, upper,
                                                     _ptr(d_mask), _ptr(d_zapped)),
                   "sk_detect_ft")

    def sk_detect_tscr(self, d_sums, d_counts, npart, nchan, npol, M, std_devs, d_mask, Nd=1):
        n = ctypes.c_uint32()
        self.check(self._lib.dspsr_b200_sk_detect_tscr(self.handle, _ptr(d_sums), _ptr(d_counts),
                                                       npart, nchan, npol, M, Nd, std_devs,
                                                       _ptr(d_mask), ctypes.byref(n)),
                   "sk_detect_tscr")
        return n.value

    def sk_reset_mask(self, d_mask, npart, nchan):
        self.check(self._lib.dspsr_b200_sk_reset_mask(self.handle, _ptr(d_mask), npart, nchan),
                   "sk_reset_mask")

    def sk_count_mask(self, d_mask, npart, nchan):
        n = ctypes.c_uint64()
        self.check(self._lib.dspsr_b200_sk_count_mask(self.handle, _ptr(d_mask), npart, nchan,
                                                      ctypes.byref(n)), "sk_count_mask")
        return n.value

    def sk_mask(self, d_mask, d_in, in_span, d_out, out_span, ndat, nchan, npol, M):
        self.check(self._lib.dspsr_b200_sk_mask(self.handle, _ptr(d_mask), _ptr(d_in), in_span,
                                                _ptr(d_out), out_span, ndat, nchan, npol, M),
                   "sk_mask")

    # ---- SpectralKurtosis engine (one resolution, noverlap 1) -----------------------
    def sk(self, d_in, in_span, ndat, nchan, npol, M, lower, upper, d_out, out_span,
           d_sums=None, d_counts=None, d_mask=None, d_zapped=None, Nd=1, zero_is_valid=True):
        """compute + detect_ft + mask in one pass; returns npart = ndat // M."""
        n = ctypes.c_uint64()
        self.check(self._lib.dspsr_b200_sk(self.handle, _ptr(d_in), in_span, ndat, nchan, npol, M,
                                           int(zero_is_valid), Nd, lower, upper, _ptr(d_out),
                                           out_span, _ptr(d_sums), _ptr(d_counts), _ptr(d_mask),
                                           _ptr(d_zapped), ctypes.byref(n)), "sk")
        return n.value


class RfiProposer:
    """The learned RFI-mask proposer in front of SpectralKurtosis: features
    from the SK sums, training on SK masks, tensor-core inference with the SK
    mask as the fallback where it is not confident."""

    NFEAT = 8

    def __init__(self, ctx, nchan, M, Nd=1, max_npart=1024, max_batch_blocks=32, seed=1):
        self.ctx = ctx
        self._lib = ctx._lib
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_rfi_proposer_create(ctx.handle, nchan, M, Nd, max_npart,
                                                           max_batch_blocks, seed,
                                                           ctypes.byref(h)), "rfi_proposer_create")
        self.handle = h
        ctx._adopt(self)
        self.nchan, self.M = nchan, M
        self.npart = 0

    def features(self, d_sums, npart, npol, d_counts=None):
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_features(
            self.handle, _ptr(d_sums), _ptr(d_counts), npart, npol), "rfi_proposer_features")
        self.npart = npart

    def train(self, d_labels, steps, batch_blocks=16, lr=3e-3, pos_weight=4.0):
        loss = ctypes.c_float()
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_train(
            self.handle, _ptr(d_labels), steps, batch_blocks, lr, pos_weight,
            ctypes.byref(loss)), "rfi_proposer_train")
        return loss.value

    def infer(self, d_mask, d_prob=None, d_sk_mask=None, confidence=0.9, count=True):
        """Returns the number of (block, channel) cells that fell back to SK
        (count=False: queued without waiting, returns None)."""
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_infer(
            self.handle, _ptr(d_sk_mask), confidence, _ptr(d_mask), _ptr(d_prob),
            ctypes.byref(n) if count else None), "rfi_proposer_infer")
        return n.value if count else None

    def params(self):
        n = ctypes.c_uint()
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_get_params(self.handle, None,
                                                                    ctypes.byref(n)), "params")
        out = np.empty(n.value, np.float32)
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_get_params(self.handle, _fptr(out),
                                                                    ctypes.byref(n)), "params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_set_params(self.handle, _fptr(p),
                                                                    p.size), "set_params")

    def get_features(self):
        out = np.empty((self.npart, self.nchan, self.NFEAT), np.float32)
        self.ctx.check(self._lib.dspsr_b200_rfi_proposer_get_features(self.handle, _fptr(out)),
                       "get_features")
        return out

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_rfi_proposer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Convolution:
    """Convolution::Engine: overlap-save FFT convolution on complex FPT data."""

    def __init__(self, ctx, nchan, npol, nfft, nfilt_pos, nfilt_neg):
        self.ctx = ctx
        self._lib = ctx._lib
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_convolution_create(ctx.handle, nchan, npol, nfft,
                                                          nfilt_pos, nfilt_neg, ctypes.byref(h)),
                  "convolution_create")
        self.handle = h
        ctx._adopt(self)
        self.nchan, self.npol, self.nfft = nchan, npol, nfft
        self.nfilt_pos, self.nfilt_neg = nfilt_pos, nfilt_neg
        self.nkeep = nfft - nfilt_pos - nfilt_neg

    def copy_response(self, response):
        r = np.ascontiguousarray(response, np.complex64)
        assert r.size == self.nchan * self.nfft
        self.ctx.check(self._lib.dspsr_b200_convolution_copy_response(
            self.handle, _fptr(r.view(np.float32))), "copy_response")

    def set_dedispersion(self, centre_freq, bandwidth, dm, input_nchan=None, dual_sideband=1,
                         dc_centred=0, chirp_mode=CHIRP_REFERENCE, norm_nfft=None):
        self.ctx.check(self._lib.dspsr_b200_convolution_set_dedispersion(
            self.handle, centre_freq, bandwidth, dm,
            self.nchan if input_nchan is None else input_nchan, dual_sideband, dc_centred,
            chirp_mode, norm_nfft or self.nfft), "set_dedispersion")

    def set_dedispersion_channels(self, chan_freq, bandwidth, dm, chirp_mode=CHIRP_REFERENCE,
                                  norm_nfft=None):
        f = np.ascontiguousarray(chan_freq, np.float64)
        assert f.size == self.nchan
        self.ctx.check(self._lib.dspsr_b200_convolution_set_dedispersion_channels(
            self.handle, f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), bandwidth, dm,
            chirp_mode, norm_nfft or self.nfft), "set_dedispersion_channels")

    def set_temporal_apodization(self, window):
        w = None if window is None else np.ascontiguousarray(window, np.float32)
        assert w is None or w.size == self.nfft
        self.ctx.check(self._lib.dspsr_b200_convolution_set_temporal_apodization(
            self.handle, None if w is None else _fptr(w)), "set_temporal_apodization")

    def set_fft_precision(self, mode):
        """FFT_FP32 (default), FFT_BF16X3 or FFT_BF16X2: the row FFTs on the
        CUDA cores or as split-BF16 tensor-core GEMMs (nfft >= 16384)."""
        self.ctx.check(self._lib.dspsr_b200_convolution_set_fft_precision(self.handle, mode),
                       "set_fft_precision")

    def status(self):
        self.ctx.check(self._lib.dspsr_b200_convolution_status(self.handle), "status")

    def get_response(self):
        out = np.empty(self.nchan * self.nfft, np.complex64)
        self.ctx.check(self._lib.dspsr_b200_convolution_get_response(
            self.handle, _fptr(out.view(np.float32))), "get_response")
        return out.reshape(self.nchan, self.nfft)

    def npart(self, ndat):
        if ndat < self.nfft:
            return 0
        return (ndat - self.nfilt_pos - self.nfilt_neg) // self.nkeep

    def perform(self, d_in, in_span, ndat, d_out, out_span):
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_convolution_perform(
            self.handle, _ptr(d_in), in_span, ndat, _ptr(d_out), out_span, ctypes.byref(n)),
            "convolution_perform")
        return n.value

    def perform_zero_dm(self, d_in, in_span, ndat, d_out, out_span, d_zero_dm, zero_dm_span):
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_convolution_perform_zero_dm(
            self.handle, _ptr(d_in), in_span, ndat, _ptr(d_out), out_span, _ptr(d_zero_dm),
            zero_dm_span, ctypes.byref(n)), "convolution_perform_zero_dm")
        return n.value

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_convolution_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class InverseFilterbank:
    """InverseFilterbank::Engine: fine-channel FFTs, stitch, response, inverse FFT."""

    INFO = ("keep", "lout", "in_step", "out_step", "in_discard_pos", "in_discard_neg", "n1",
            "n2", "max_batch", "lin")

    def __init__(self, ctx, input_nchan, output_nchan, pfb_nchan, npol, input_fft_length,
                 os=(4, 3), output_discard=(0, 0), pfb_dc_chan=True, pfb_all_chan=True,
                 dual_sideband=True, scratch_bytes=0):
        self.ctx = ctx
        self._lib = ctx._lib
        cfg = _capi.IfbConfig(input_nchan, output_nchan, pfb_nchan, npol, input_fft_length,
                              os[0], os[1], output_discard[0], output_discard[1],
                              int(pfb_dc_chan), int(pfb_all_chan), int(dual_sideband),
                              scratch_bytes)
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_inverse_filterbank_create(ctx.handle, ctypes.byref(cfg),
                                                                 ctypes.byref(h)),
                  "inverse_filterbank_create")
        self.handle = h
        ctx._adopt(self)
        info = (ctypes.c_uint64 * 10)()
        ctx.check(self._lib.dspsr_b200_inverse_filterbank_info(h, info), "inverse_filterbank_info")
        self.info = dict(zip(self.INFO, list(info)))
        self.nin, self.nout, self.npol = input_nchan, output_nchan, npol

    def copy_response(self, response):
        if response is None:
            self.ctx.check(self._lib.dspsr_b200_inverse_filterbank_copy_response(self.handle, None),
                           "copy_response")
            return
        r = np.ascontiguousarray(response, np.complex64)
        assert r.size == self.nout * self.info["lout"]
        self.ctx.check(self._lib.dspsr_b200_inverse_filterbank_copy_response(
            self.handle, _fptr(r.view(np.float32))), "copy_response")

    def set_apodization(self, temporal=None, spectral=None):
        t = None if temporal is None else np.ascontiguousarray(temporal, np.float32)
        sp = None if spectral is None else np.ascontiguousarray(spectral, np.float32)
        self.ctx.check(self._lib.dspsr_b200_inverse_filterbank_set_apodization(
            self.handle, None if t is None else _fptr(t), None if sp is None else _fptr(sp)),
            "set_apodization")

    def npart(self, ndat):
        d = self.info["in_discard_pos"] + self.info["in_discard_neg"]
        return (ndat - d) // self.info["in_step"] if ndat > d else 0

    def perform(self, d_in, ndat, d_out, out_span, input_kind=FLOAT_FPT, in_span=None, lut=None,
                offset_binary=False):
        n = ctypes.c_uint64()
        lp = _fptr(np.ascontiguousarray(lut, np.float32)) if lut is not None else None
        self.ctx.check(self._lib.dspsr_b200_inverse_filterbank_perform(
            self.handle, input_kind, _ptr(d_in), ndat, ndat if in_span is None else in_span, lp,
            int(offset_binary), _ptr(d_out), out_span, ctypes.byref(n)),
            "inverse_filterbank_perform")
        return n.value

    def status(self):
        self.ctx.check(self._lib.dspsr_b200_inverse_filterbank_status(self.handle), "status")

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_inverse_filterbank_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FilterbankDuring:
    """Filterbank::Engine with a response (the "During" filterbank, -F nchan:D):
    one nsub*freq_res-point FFT per part, the response, then a freq_res-point
    inverse FFT per output channel (FilterbankEngineCPU.C:379-535)."""

    INFO = ("nsamp_fft", "nsamp_step", "nsamp_overlap", "nkeep", "n1", "max_batch")

    def __init__(self, ctx, input_nchan, npol, nsub, freq_res, nfilt=(0, 0), scratch_bytes=0):
        self.ctx = ctx
        self._lib = ctx._lib
        cfg = _capi.FbdConfig(input_nchan, npol, nsub, freq_res, nfilt[0], nfilt[1],
                              scratch_bytes)
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_filterbank_during_create(ctx.handle, ctypes.byref(cfg),
                                                                ctypes.byref(h)),
                  "filterbank_during_create")
        self.handle = h
        ctx._adopt(self)
        info = (ctypes.c_uint64 * 6)()
        ctx.check(self._lib.dspsr_b200_filterbank_during_info(h, info), "filterbank_during_info")
        self.info = dict(zip(self.INFO, list(info)))
        self.nin, self.npol, self.nsub, self.freq_res = input_nchan, npol, nsub, freq_res
        self.nchan = input_nchan * nsub

    def copy_response(self, response):
        r = np.ascontiguousarray(response, np.complex64)
        assert r.size == self.nchan * self.freq_res
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_copy_response(
            self.handle, _fptr(r.view(np.float32))), "copy_response")

    def set_dedispersion(self, centre_freq, bandwidth, dm, swapped=True, chirp_mode=0):
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_set_dedispersion(
            self.handle, centre_freq, bandwidth, dm, int(swapped), chirp_mode), "set_dedispersion")

    def set_apodization(self, temporal=None, spectral=None):
        t = None if temporal is None else np.ascontiguousarray(temporal, np.float32)
        sp = None if spectral is None else np.ascontiguousarray(spectral, np.float32)
        assert t is None or t.size == self.nsub * self.freq_res
        assert sp is None or sp.size == self.freq_res
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_set_apodization(
            self.handle, None if t is None else _fptr(t), None if sp is None else _fptr(sp)),
            "set_apodization")

    def get_response(self):
        out = np.empty(self.nchan * self.freq_res, np.complex64)
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_get_response(
            self.handle, _fptr(out.view(np.float32))), "get_response")
        return out.reshape(self.nchan, self.freq_res)

    def npart(self, ndat):
        o = self.info["nsamp_overlap"]
        return (ndat - o) // self.info["nsamp_step"] if ndat > o else 0

    def perform(self, d_in, ndat, d_out, out_span, input_kind=FLOAT_FPT, in_span=None, lut=None,
                offset_binary=False):
        n = ctypes.c_uint64()
        lp = _fptr(np.ascontiguousarray(lut, np.float32)) if lut is not None else None
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_perform(
            self.handle, input_kind, _ptr(d_in), ndat, ndat if in_span is None else in_span, lp,
            int(offset_binary), _ptr(d_out), out_span, ctypes.byref(n)),
            "filterbank_during_perform")
        return n.value

    def perform_fold(self, d_in, ndat, fold, state, input_kind=FLOAT_FPT, in_span=None, lut=None,
                     offset_binary=False):
        """Filterbank, detection and fold in one pass; fold's plan (set_bins)
        covers npart(ndat) * nkeep output samples."""
        n = ctypes.c_uint64()
        lp = _fptr(np.ascontiguousarray(lut, np.float32)) if lut is not None else None
        self.ctx.check(self._lib.dspsr_b200_filterbank_during_perform_fold(
            self.handle, input_kind, _ptr(d_in), ndat, ndat if in_span is None else in_span, lp,
            int(offset_binary), fold.handle, state, ctypes.byref(n)),
            "filterbank_during_perform_fold")
        return n.value

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_filterbank_during_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Fold:
    """Fold::Engine with use_set_bins: exact bin plan on the host, fold on the GPU."""

    def __init__(self, ctx, nbin, nchan, npol):
        self.ctx = ctx
        self._lib = ctx._lib
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_fold_create(ctx.handle, nbin, nchan, npol, ctypes.byref(h)),
                  "fold_create")
        self.handle = h
        ctx._adopt(self)
        self.nbin, self.nchan, self.npol = nbin, nchan, npol

    def set_bins(self, phi, phase_per_sample, ndat, idat_start=0):
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_fold_set_bins(self.handle, phi, phase_per_sample, ndat,
                                                          idat_start, ctypes.byref(n)), "set_bins")
        return n.value

    def fold(self, d_in, in_span):
        self.ctx.check(self._lib.dspsr_b200_fold_fold(self.handle, _ptr(d_in), in_span), "fold")

    def binplan(self, d_out):
        self.ctx.check(self._lib.dspsr_b200_fold_binplan(self.handle, _ptr(d_out)), "binplan")

    def get_profiles(self):
        prof = np.empty((self.nchan, self.npol, self.nbin), np.float32)
        hits = np.empty(self.nbin, np.uint32)
        self.ctx.check(self._lib.dspsr_b200_fold_get_profiles(
            self.handle, _fptr(prof), hits.ctypes.data_as(_capi.c_u32p)), "get_profiles")
        return prof, hits

    def reset(self):
        self.ctx.check(self._lib.dspsr_b200_fold_reset(self.handle), "fold_reset")

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_fold_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pipeline:
    """The fused SingleThread hot loop: unpack -> convolve -> detect -> fold."""

    def __init__(self, ctx, config):
        self.ctx = ctx
        self._lib = ctx._lib
        self.config = config
        h = ctypes.c_void_p()
        ctx.check(self._lib.dspsr_b200_pipeline_create(ctx.handle, ctypes.byref(config),
                                                       ctypes.byref(h)), "pipeline_create")
        self.handle = h
        ctx._adopt(self)
        self.nout = NOUT[config.state]

    def run(self, d_in, ndat, in_span=0):
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_pipeline_run(self.handle, _ptr(d_in), ndat, in_span,
                                                         ctypes.byref(n)), "pipeline_run")
        return n.value

    def run_host(self, h_in, ndat):
        """h_in: a numpy array (or pinned torch CPU tensor) holding the TFPD block."""
        addr = h_in.ctypes.data if isinstance(h_in, np.ndarray) else h_in.data_ptr()
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_pipeline_run_host(self.handle, addr, ndat,
                                                              ctypes.byref(n)), "pipeline_run_host")
        return n.value

    def run_dada(self, dada, block_ndat, start_sample=0, nsamp=0):
        """Feed a DADAFile through the pipeline in blocks of block_ndat
        (nsamp 0 = to the end of the data); returns (samples read, folded)."""
        nread = ctypes.c_uint64()
        nfold = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_pipeline_run_dada(
            self.handle, dada.handle, start_sample, nsamp, block_ndat, ctypes.byref(nread),
            ctypes.byref(nfold)), "pipeline_run_dada")
        return nread.value, nfold.value

    def set_unloader(self, fn):
        """PhaseSeriesUnloader: fn(info: dict, profiles [chan][nout][nbin], hits [nbin])
        is called for every closed sub-integration (copies of the arrays)."""
        c = self.config
        nchan = c.nchan * (c.filterbank_nchan if c.filterbank_nchan > 1 else 1)
        shape = (nchan, self.nout, c.nbin)

        def tramp(user, info, prof, hits):
            p = np.ctypeslib.as_array(prof, shape=(int(np.prod(shape)),)).reshape(shape).copy()
            h = np.ctypeslib.as_array(hits, shape=(c.nbin,)).copy()
            fn(_struct_dict(info.contents), p, h)

        self._unload = _capi.UNLOAD_FN(tramp) if fn is not None else _capi.UNLOAD_FN()
        self.ctx.check(self._lib.dspsr_b200_pipeline_set_unloader(self.handle, self._unload, None),
                       "set_unloader")

    def subints_ready(self):
        n = ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_pipeline_subints_ready(self.handle, ctypes.byref(n)),
                       "subints_ready")
        return n.value

    def pop_subint(self):
        """The oldest closed sub-integration: (info dict, profiles, hits)."""
        c = self.config
        nchan = c.nchan * (c.filterbank_nchan if c.filterbank_nchan > 1 else 1)
        prof = np.empty((nchan, self.nout, c.nbin), np.float32)
        hits = np.empty(c.nbin, np.uint32)
        info = _capi.Subint()
        self.ctx.check(self._lib.dspsr_b200_pipeline_pop_subint(
            self.handle, ctypes.byref(info), _fptr(prof), hits.ctypes.data_as(_capi.c_u32p)),
            "pop_subint")
        return _struct_dict(info), prof, hits

    def finish(self):
        """Subint::finish: close the open sub-integration."""
        self.ctx.check(self._lib.dspsr_b200_pipeline_finish(self.handle), "pipeline_finish")

    def get_profiles(self):
        c = self.config
        nchan = c.nchan * (c.filterbank_nchan if c.filterbank_nchan > 1 else 1)
        prof = np.empty((nchan, self.nout, c.nbin), np.float32)
        hits = np.empty(c.nbin, np.uint32)
        self.ctx.check(self._lib.dspsr_b200_pipeline_get_profiles(
            self.handle, _fptr(prof), hits.ctypes.data_as(_capi.c_u32p)), "get_profiles")
        return prof, hits

    def profile_buffers(self):
        """Page-locked host arrays (profiles, hits) for get_profiles_async."""
        import torch
        c = self.config
        nchan = c.nchan * (c.filterbank_nchan if c.filterbank_nchan > 1 else 1)
        prof = torch.empty((nchan, self.nout, c.nbin), dtype=torch.float32, pin_memory=True)
        hits = torch.empty(c.nbin, dtype=torch.int32, pin_memory=True)
        return prof.numpy(), hits.numpy().view(np.uint32)

    def get_profiles_async(self, prof, hits):
        """Queue the copy of the profiles and hits so far into prof / hits
        (from profile_buffers) and return; wait_profiles() waits for it."""
        self.ctx.check(self._lib.dspsr_b200_pipeline_get_profiles_async(
            self.handle, _fptr(prof), hits.ctypes.data_as(_capi.c_u32p)), "get_profiles_async")

    def wait_profiles(self):
        self.ctx.check(self._lib.dspsr_b200_pipeline_wait_profiles(self.handle), "wait_profiles")

    def reset(self):
        self.ctx.check(self._lib.dspsr_b200_pipeline_reset(self.handle), "pipeline_reset")

    def profile(self, enable=True):
        self.ctx.check(self._lib.dspsr_b200_pipeline_profile(self.handle, int(enable)),
                       "pipeline_profile")

    KERNELS = ("fwd_cols", "rows", "inv_cols_detect_fold", "fused", "filterbank")

    def kernel_times(self):
        """{kernel: (milliseconds, launches)} since the last call."""
        ms = (ctypes.c_double * 5)()
        n = (ctypes.c_uint64 * 5)()
        self.ctx.check(self._lib.dspsr_b200_pipeline_kernel_times(self.handle, ms, n),
                       "kernel_times")
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNELS)}

    def set_rfi_proposer(self, proposer, confidence=0.9):
        """Put an RfiProposer in front of the SK stage (None detaches it)."""
        self.ctx.check(self._lib.dspsr_b200_pipeline_set_rfi_proposer(
            self.handle, proposer.handle if proposer is not None else None, confidence),
            "set_rfi_proposer")
        self._proposer = proposer

    def sk_counts(self):
        """(zapped, tested) (block, channel) cells of the SpectralKurtosis stage."""
        z, t = ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self._lib.dspsr_b200_pipeline_sk_counts(self.handle, ctypes.byref(z),
                                                               ctypes.byref(t)), "sk_counts")
        return z.value, t.value

    def info(self):
        a = (ctypes.c_uint64 * 8)()
        self.ctx.check(self._lib.dspsr_b200_pipeline_info(self.handle, a), "pipeline_info")
        keys = ["nfft", "nkeep", "n1", "n2", "max_batch", "ncarry", "in0", "nseg"]
        return dict(zip(keys, list(a)))

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_pipeline_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _host_check(rc, what):
    if rc != 0:
        msg = _capi.lib().dspsr_b200_host_error()
        raise B200Error(rc, f"{what}: {msg.decode() if msg else ''}")


def _cstr(text):
    return text.encode() if isinstance(text, str) else bytes(text)


def ascii_header_get(header, keyword):
    """ascii_header_get with a "%s" code (ascii_header.c:117-142): the value
    token after KEYWORD, or None when the keyword or its value is absent."""
    buf = ctypes.create_string_buffer(4096)
    rc = _capi.lib().dspsr_b200_ascii_header_get(_cstr(header), _cstr(keyword), buf, len(buf))
    return buf.value.decode() if rc == 1 else None


def ascii_header_set(header, keyword, value, header_size=4096):
    """ascii_header_set (ascii_header.c:58-115) on a copy of HEADER inside a
    buffer of header_size bytes; returns the new header text."""
    h = _cstr(header)
    buf = ctypes.create_string_buffer(h, max(header_size, len(h) + 1))
    _host_check(_capi.lib().dspsr_b200_ascii_header_set(buf, header_size, _cstr(keyword),
                                                        _cstr(str(value))), "ascii_header_set")
    return buf.value.decode()


def _struct_dict(st):
    return {name: getattr(st, name) for name, _ in st._fields_}


class TimeDivide:
    """TimeDivide + the block loop of Subint<Fold> on the host: the ranges of
    each block that fold into each division, and where divisions close."""

    def __init__(self, seconds=0.0, turns=0.0, period=0.0, reference_epoch=(0, 0, 0.0)):
        self._lib = _capi.lib()
        h = ctypes.c_void_p()
        _host_check(self._lib.dspsr_b200_time_divide_create(seconds, turns, period,
                                                             *reference_epoch, ctypes.byref(h)),
                    "time_divide_create")
        self.handle = h

    def block(self, start_mjd, ndat, rate, cap=4096):
        """Actions for a block of ndat samples at rate starting at start_mjd:
        a list of dicts (kind 0 fold, 1 close partial, 2 close complete)."""
        acts = (_capi.SubintAction * cap)()
        n = ctypes.c_uint64()
        _host_check(self._lib.dspsr_b200_time_divide_block(self.handle, *start_mjd, ndat, rate,
                                                            acts, cap, ctypes.byref(n)),
                    "time_divide_block")
        return [_struct_dict(acts[i]) for i in range(n.value)]

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_time_divide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _info_dict(info):
    d = {}
    for name, _ in _capi.DadaInfo._fields_:
        v = getattr(info, name)
        d[name] = v.decode() if isinstance(v, bytes) else v
    return d


def dada_parse(header, header_bytes=4096):
    """ASCIIObservation::load over a header text: the observation as a dict."""
    info = _capi.DadaInfo()
    _host_check(_capi.lib().dspsr_b200_dada_parse(_cstr(header), header_bytes,
                                                  ctypes.byref(info)), "dada_parse")
    return _info_dict(info)


def dada_is_valid(filename):
    """DADAFile::is_valid: the header loads and names HDR_VERSION and INSTRUMENT."""
    return bool(_capi.lib().dspsr_b200_dada_is_valid(_cstr(os.fspath(filename))))


class DADAFile:
    """A DADA file (DADAFile::open_file, File::open): header, observation
    parameters and whole-sample reads."""

    def __init__(self, filename):
        self._lib = _capi.lib()
        self.filename = os.fspath(filename)
        info = _capi.DadaInfo()
        h = ctypes.c_void_p()
        _host_check(self._lib.dspsr_b200_dada_open(_cstr(self.filename), ctypes.byref(h),
                                                   ctypes.byref(info)), "dada_open")
        self.handle = h
        self.info = _info_dict(info)
        text = ctypes.c_char_p()
        size = ctypes.c_uint64()
        _host_check(self._lib.dspsr_b200_dada_header(self.handle, ctypes.byref(text),
                                                     ctypes.byref(size)), "dada_header")
        self.header = text.value.decode(errors="replace")

    @property
    def ndat(self):
        return min(self.info["ndat"], self.info["file_ndat"])

    @property
    def bytes_per_sample(self):
        return self.info["bits_per_sample"] // 8

    @property
    def dual_sideband(self):
        """Observation::get_dual_sideband: DSB, else true for analytic (NDIM 2) data."""
        dsb = self.info["dual_sideband"]
        return dsb if dsb >= 0 else int(self.info["ndim"] == 2)

    def read(self, start_sample, nsamp):
        """nsamp samples from start_sample as raw bytes (uint8), fewer at the end."""
        out = np.empty(nsamp * self.info["bits_per_sample"] // 8, np.uint8)
        n = ctypes.c_uint64()
        _host_check(self._lib.dspsr_b200_dada_read(self.handle, start_sample, nsamp,
                                                   out.ctypes.data, ctypes.byref(n)), "dada_read")
        return out[: n.value * self.info["bits_per_sample"] // 8]

    def pipeline_config(self, dm, nfft, nfilt_pos, nfilt_neg, nbin, period, **kw):
        """make_config with the file's FREQ, BW, NCHAN, NPOL, NBIT, start time
        and sideband filled in."""
        i = self.info
        if i["ndim"] != 2 or i["nbit"] not in (8, 16):
            raise B200Error(_capi.EINVAL, f"the pipeline takes NDIM 2 with NBIT 8 or 16, the "
                                          f"file has NDIM {i['ndim']} NBIT {i['nbit']}")
        kw.setdefault("input_kind", INT8_TFPD if i["nbit"] == 8 else INT16_TFPD)
        kw.setdefault("start_mjd", (i["start_day"], i["start_sec"], i["start_frac"]))
        kw.setdefault("dual_sideband", self.dual_sideband)
        return make_config(i["centre_freq_mhz"], i["bandwidth_mhz"], dm, i["nchan"], i["npol"],
                           nfft, nfilt_pos, nfilt_neg, nbin, period, **kw)

    def close(self):
        if self.handle:
            self._lib.dspsr_b200_dada_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_dada(filename, keys, data, header_size=4096):
    """Write a DADA file: a header of header_size bytes holding HDR_SIZE and
    KEYS (set in order with ascii_header_set), then the raw bytes of DATA."""
    text = ""
    text = ascii_header_set(text, "HDR_SIZE", header_size, header_size)
    for k, v in keys.items():
        text = ascii_header_set(text, k, v, header_size)
    raw = text.encode()
    with open(filename, "wb") as f:
        f.write(raw + b"\0" * (header_size - len(raw)))
        f.write(np.ascontiguousarray(data).view(np.uint8).tobytes())


def make_config(centre_freq, bandwidth, dm, nchan, npol, nfft, nfilt_pos, nfilt_neg, nbin,
                period, state=INTENSITY, input_kind=INT8_TFPD, lut=None, chirp_mode=CHIRP_REFERENCE,
                start_mjd=(60000, 0, 0.0), epoch_mjd=(60000, 0, 0.0), reference_phase=0.0,
                dual_sideband=1, offset_binary=0, scratch_bytes=0, filterbank_nchan=0,
                subint_seconds=0.0, subint_turns=0.0, subint_slots=0,
                subint_epoch=(0, 0, 0.0), fused_filterbank=0, interchannel=0,
                fft_precision=FFT_FP32, sk_M=0, sk_std_devs=3.0, row_length=0):
    """Fill a PipelineConfig (the fields DedispersionPipe / LoadToFold set up).
    With filterbank_nchan > 1, nchan counts input channels, and nfft and the
    smearing (nfilt_pos, nfilt_neg) refer to the filterbank's output channels."""
    cfg = PipelineConfig()
    cfg.filterbank_nchan = filterbank_nchan
    cfg.centre_freq_mhz = centre_freq
    cfg.bandwidth_mhz = bandwidth
    cfg.dm = dm
    cfg.nchan = nchan
    cfg.npol = npol
    cfg.input_kind = input_kind
    if lut is None:
        lut, _ = bittable8()
    for i in range(256):
        cfg.lut[i] = float(lut[i])
    cfg.offset_binary = offset_binary
    cfg.dual_sideband = dual_sideband
    cfg.dc_centred = 0
    cfg.nfft = nfft
    cfg.nfilt_pos = nfilt_pos
    cfg.nfilt_neg = nfilt_neg
    cfg.chirp_mode = chirp_mode
    cfg.state = state
    cfg.nbin = nbin
    cfg.period_s = period
    cfg.reference_phase = reference_phase
    cfg.epoch_day, cfg.epoch_sec, cfg.epoch_frac = epoch_mjd
    cfg.start_day, cfg.start_sec, cfg.start_frac = start_mjd
    cfg.scratch_bytes = scratch_bytes
    cfg.subint_seconds = subint_seconds
    cfg.subint_turns = subint_turns
    cfg.subint_slots = subint_slots
    cfg.subint_epoch_day, cfg.subint_epoch_sec, cfg.subint_epoch_frac = subint_epoch
    cfg.fused_filterbank = fused_filterbank
    cfg.interchannel = interchannel
    cfg.fft_precision = fft_precision
    cfg.sk_M = sk_M
    cfg.sk_std_devs = sk_std_devs
    cfg.row_length = row_length
    return cfg


def dispersion_plan(centre_freq, bandwidth, dm, nchan, nfft=None):
    """nfilt_pos, nfilt_neg and nfft as PlasmaResponse / Response choose them.

    PlasmaResponse::prepare (PlasmaResponse.C:91-119): impulse_neg is the
    smear of the lower half of the worst channel, impulse_pos of the upper half.
    Without an explicit nfft the minimum legal length is used
    (Response::get_minimum_ndat)."""
    neg = smearing_samples(centre_freq, bandwidth, dm, nchan, -1)
    pos = smearing_samples(centre_freq, bandwidth, dm, nchan, 1)
    nmin = minimum_ndat(pos, neg)
    if nfft is None:
        nfft = nmin
    if nfft < nmin:
        # Response::check_ndat (Response.C:605-621)
        raise B200Error(_capi.EINVAL, f"specified nfft={nfft} < required minimum ndat={nmin}")
    return pos, neg, nfft
