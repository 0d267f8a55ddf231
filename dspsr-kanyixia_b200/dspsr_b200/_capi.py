"""ctypes declarations of libdspsr_b200.so (include/dspsr_b200.h).

The library is built in-tree by dspsr-kanyixia_b200/Makefile into
dspsr-kanyixia_b200/lib/.  Loading fails loudly when it is missing: there is
no CPU fallback for any entry point.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libdspsr_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_ROOT), "include", "dspsr_b200.h")

OK, EINVAL, ESTATE, ECUDA, ENOMEM, ENODEV, ETOOBIG = 0, 1, 2, 3, 4, 5, 6
NOALLOC_SCRATCH_BYTES = 32 << 20
INTENSITY, PPQQ, COHERENCE, STOKES = 0, 1, 2, 3
INT8_TFPD, INT16_TFPD, FLOAT_FPT = 0, 1, 2
CHIRP_REFERENCE, CHIRP_FP64 = 0, 1
FFT_FP32, FFT_BF16X2, FFT_BF16X3 = 0, 2, 3

c_vp = ctypes.c_void_p
c_u64 = ctypes.c_uint64
c_i64 = ctypes.c_int64
c_uint = ctypes.c_uint
c_int = ctypes.c_int
c_dbl = ctypes.c_double
c_fp = ctypes.POINTER(ctypes.c_float)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)


class PipelineConfig(ctypes.Structure):
    """dspsr_b200_pipeline_config"""
    _fields_ = [
        ("centre_freq_mhz", c_dbl),
        ("bandwidth_mhz", c_dbl),
        ("dm", c_dbl),
        ("nchan", c_uint),
        ("npol", c_uint),
        ("input_kind", c_int),
        ("lut", ctypes.c_float * 256),
        ("offset_binary", c_int),
        ("dual_sideband", c_int),
        ("dc_centred", c_int),
        ("nfft", c_uint),
        ("nfilt_pos", c_uint),
        ("nfilt_neg", c_uint),
        ("chirp_mode", c_int),
        ("state", c_int),
        ("nbin", c_uint),
        ("period_s", c_dbl),
        ("reference_phase", c_dbl),
        ("epoch_day", c_i64),
        ("epoch_sec", c_i64),
        ("epoch_frac", c_dbl),
        ("start_day", c_i64),
        ("start_sec", c_i64),
        ("start_frac", c_dbl),
        ("scratch_bytes", c_u64),
        ("filterbank_nchan", c_uint),
        ("subint_seconds", c_dbl),
        ("subint_turns", c_dbl),
        ("subint_epoch_day", c_i64),
        ("subint_epoch_sec", c_i64),
        ("subint_epoch_frac", c_dbl),
        ("subint_slots", c_uint),
        ("fused_filterbank", c_int),
        ("interchannel", c_int),
        ("fft_precision", c_int),
        ("sk_M", c_uint),
        ("sk_std_devs", ctypes.c_float),
        ("row_length", c_uint),
    ]


class SubintAction(ctypes.Structure):
    """dspsr_b200_subint_action"""
    _fields_ = [
        ("kind", c_int),
        ("end_reached", c_int),
        ("idat_start", c_u64),
        ("ndat", c_u64),
        ("division", c_u64),
        ("lower_day", c_i64),
        ("lower_sec", c_i64),
        ("lower_frac", c_dbl),
        ("upper_day", c_i64),
        ("upper_sec", c_i64),
        ("upper_frac", c_dbl),
    ]


class Subint(ctypes.Structure):
    """dspsr_b200_subint"""
    _fields_ = [
        ("division", c_u64),
        ("ndat_folded", c_u64),
        ("first_sample", c_u64),
        ("lower_day", c_i64),
        ("lower_sec", c_i64),
        ("lower_frac", c_dbl),
        ("upper_day", c_i64),
        ("upper_sec", c_i64),
        ("upper_frac", c_dbl),
        ("integration_length", c_dbl),
        ("complete", c_int),
    ]


UNLOAD_FN = ctypes.CFUNCTYPE(None, c_vp, ctypes.POINTER(Subint), ctypes.POINTER(ctypes.c_float),
                             ctypes.POINTER(ctypes.c_uint32))
SUBINT_FOLD, SUBINT_CLOSE_PARTIAL, SUBINT_CLOSE_COMPLETE = 0, 1, 2


class FbdConfig(ctypes.Structure):
    """dspsr_b200_fbd_config"""
    _fields_ = [
        ("input_nchan", c_uint),
        ("npol", c_uint),
        ("nsub", c_uint),
        ("freq_res", c_uint),
        ("nfilt_pos", c_uint),
        ("nfilt_neg", c_uint),
        ("scratch_bytes", ctypes.c_uint64),
    ]


class IfbConfig(ctypes.Structure):
    """dspsr_b200_ifb_config"""
    _fields_ = [
        ("input_nchan", c_uint),
        ("output_nchan", c_uint),
        ("pfb_nchan", c_uint),
        ("npol", c_uint),
        ("input_fft_length", c_uint),
        ("os_num", c_uint),
        ("os_den", c_uint),
        ("output_discard_pos", c_uint),
        ("output_discard_neg", c_uint),
        ("pfb_dc_chan", c_int),
        ("pfb_all_chan", c_int),
        ("dual_sideband", c_int),
        ("scratch_bytes", c_u64),
    ]


class DadaInfo(ctypes.Structure):
    """dspsr_b200_dada_info"""
    _fields_ = [
        ("header_bytes", c_u64),
        ("ndat", c_u64),
        ("file_ndat", c_u64),
        ("bits_per_sample", c_u64),
        ("obs_offset", c_u64),
        ("picoseconds", c_i64),
        ("start_day", c_i64),
        ("start_sec", c_i64),
        ("start_frac", c_dbl),
        ("centre_freq_mhz", c_dbl),
        ("bandwidth_mhz", c_dbl),
        ("tsamp_us", c_dbl),
        ("rate_hz", c_dbl),
        ("hdr_version", c_dbl),
        ("nchan", c_uint),
        ("npol", c_uint),
        ("nbit", c_uint),
        ("ndim", c_uint),
        ("dual_sideband", c_int),
        ("adjacent_header", c_int),
    ] + [(k, ctypes.c_char * 64) for k in ("telescope", "receiver", "source", "mode",
                                            "instrument", "utc_start", "state", "basis")]


SIGNATURES = {
    "dspsr_b200_version": (c_int, []),
    "dspsr_b200_context_create": (c_int, [c_int, c_vp, ctypes.POINTER(c_vp)]),
    "dspsr_b200_context_destroy": (c_int, [c_vp]),
    "dspsr_b200_context_set_stream": (c_int, [c_vp, c_vp]),
    "dspsr_b200_last_error": (ctypes.c_char_p, [c_vp]),
    "dspsr_b200_synchronize": (c_int, [c_vp]),
    "dspsr_b200_smearing_samples": (c_uint, [c_dbl, c_dbl, c_dbl, c_uint, c_int]),
    "dspsr_b200_minimum_ndat": (c_uint, [c_uint, c_uint]),
    "dspsr_b200_optimal_fft_length": (c_i64, [c_u64, c_u64, c_uint]),
    "dspsr_b200_bittable8": (c_int, [c_dbl, c_int, c_fp, ctypes.POINTER(c_dbl)]),
    "dspsr_b200_fold_phi": (c_dbl, [c_i64, c_i64, c_dbl, c_i64, c_i64, c_dbl, c_u64, c_dbl,
                                    c_dbl, c_dbl]),
    "dspsr_b200_fold_plan_count": (c_i64, [c_dbl, c_dbl, c_u64]),
    "dspsr_b200_interchannel_delays": (c_int, [c_dbl, c_dbl, c_dbl, ctypes.POINTER(c_dbl), c_uint,
                                               ctypes.POINTER(c_i64), ctypes.POINTER(c_dbl),
                                               ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                               c_u64p]),
    "dspsr_b200_sk_limits": (c_int, [c_uint, c_uint, ctypes.c_float, c_uint, c_fp, c_fp]),
    "dspsr_b200_unpack8": (c_int, [c_vp, c_vp, c_u64, c_uint, c_uint, c_uint, c_fp, c_vp, c_u64]),
    "dspsr_b200_unpack16": (c_int, [c_vp, c_vp, c_u64, c_uint, c_uint, c_uint, c_int, c_vp,
                                    c_u64]),
    "dspsr_b200_convolution_create": (c_int, [c_vp, c_uint, c_uint, c_uint, c_uint, c_uint,
                                              ctypes.POINTER(c_vp)]),
    "dspsr_b200_convolution_destroy": (c_int, [c_vp]),
    "dspsr_b200_convolution_copy_response": (c_int, [c_vp, c_fp]),
    "dspsr_b200_convolution_set_dedispersion": (c_int, [c_vp, c_dbl, c_dbl, c_dbl, c_int, c_int,
                                                        c_int, c_int, c_uint]),
    "dspsr_b200_convolution_get_response": (c_int, [c_vp, c_fp]),
    "dspsr_b200_convolution_status": (c_int, [c_vp]),
    "dspsr_b200_convolution_set_temporal_apodization": (c_int, [c_vp, c_fp]),
    "dspsr_b200_convolution_set_fft_precision": (c_int, [c_vp, c_int]),
    "dspsr_b200_convolution_perform_noalloc": (c_int, [c_vp, c_vp, c_u64, c_u64, c_uint, c_uint,
                                                       c_uint, c_uint, c_uint, c_vp, c_vp, c_u64,
                                                       c_u64p, c_vp]),
    "dspsr_b200_convolution_set_dedispersion_channels": (c_int, [c_vp, ctypes.POINTER(c_dbl),
                                                                 c_dbl, c_dbl, c_int, c_uint]),
    "dspsr_b200_filterbank": (c_int, [c_vp, c_int, c_vp, c_u64, c_u64, c_uint, c_uint, c_uint,
                                      c_fp, c_int, c_vp, c_u64, c_u64p]),
    "dspsr_b200_convolution_perform": (c_int, [c_vp, c_vp, c_u64, c_u64, c_vp, c_u64, c_u64p]),
    "dspsr_b200_convolution_perform_zero_dm": (c_int, [c_vp, c_vp, c_u64, c_u64, c_vp, c_u64, c_vp,
                                                       c_u64, c_u64p]),
    "dspsr_b200_detect": (c_int, [c_vp, c_vp, c_u64, c_u64, c_uint, c_int, c_vp, c_u64]),
    "dspsr_b200_inverse_filterbank_create": (c_int, [c_vp, ctypes.POINTER(IfbConfig),
                                                     ctypes.POINTER(c_vp)]),
    "dspsr_b200_inverse_filterbank_destroy": (c_int, [c_vp]),
    "dspsr_b200_inverse_filterbank_info": (c_int, [c_vp, c_u64p]),
    "dspsr_b200_inverse_filterbank_copy_response": (c_int, [c_vp, c_fp]),
    "dspsr_b200_inverse_filterbank_set_apodization": (c_int, [c_vp, c_fp, c_fp]),
    "dspsr_b200_inverse_filterbank_perform": (c_int, [c_vp, c_int, c_vp, c_u64, c_u64, c_fp, c_int,
                                                      c_vp, c_u64, c_u64p]),
    "dspsr_b200_inverse_filterbank_status": (c_int, [c_vp]),
    "dspsr_b200_filterbank_during_create": (c_int, [c_vp, ctypes.POINTER(FbdConfig),
                                                    ctypes.POINTER(c_vp)]),
    "dspsr_b200_filterbank_during_destroy": (c_int, [c_vp]),
    "dspsr_b200_filterbank_during_info": (c_int, [c_vp, c_u64p]),
    "dspsr_b200_filterbank_during_copy_response": (c_int, [c_vp, c_fp]),
    "dspsr_b200_filterbank_during_set_dedispersion": (c_int, [c_vp, c_dbl, c_dbl, c_dbl,
                                                              c_int, c_int]),
    "dspsr_b200_filterbank_during_get_response": (c_int, [c_vp, c_fp]),
    "dspsr_b200_filterbank_during_set_apodization": (c_int, [c_vp, c_fp, c_fp]),
    "dspsr_b200_filterbank_during_perform": (c_int, [c_vp, c_int, c_vp, c_u64, c_u64, c_fp, c_int,
                                                     c_vp, c_u64, c_u64p]),
    "dspsr_b200_filterbank_during_perform_fold": (c_int, [c_vp, c_int, c_vp, c_u64, c_u64, c_fp,
                                                          c_int, c_vp, c_int, c_u64p]),
    "dspsr_b200_apodization": (c_int, [c_int, c_uint, c_uint, c_uint, c_int, c_fp]),
    "dspsr_b200_archive_profiles": (c_int, [c_fp, ctypes.POINTER(ctypes.c_uint32), c_int, c_uint,
                                            c_uint, c_uint, c_dbl, c_u64, c_int, c_fp, c_fp,
                                            ctypes.POINTER(c_uint)]),
    "dspsr_b200_sk": (c_int, [c_vp, c_vp, c_u64, c_u64, c_uint, c_uint, c_uint, c_int, c_uint,
                              ctypes.c_float, ctypes.c_float, c_vp, c_u64, c_vp, c_vp, c_vp, c_vp,
                              c_u64p]),
    "dspsr_b200_rfi_proposer_create": (c_int, [c_vp, c_uint, c_uint, c_uint, c_u64, c_uint, c_u64,
                                               ctypes.POINTER(c_vp)]),
    "dspsr_b200_rfi_proposer_destroy": (c_int, [c_vp]),
    "dspsr_b200_sk_compute": (c_int, [c_vp, c_vp, c_u64, c_u64, c_uint, c_uint, c_uint, c_uint,
                                      c_int, c_vp, c_vp, c_u64p]),
    "dspsr_b200_sk_tscrunch": (c_int, [c_vp, c_vp, c_vp, c_u64, c_u64, c_uint, c_uint, c_uint,
                                       c_uint, c_vp, c_vp]),
    "dspsr_b200_sk_detect_skfb": (c_int, [c_vp, c_vp, c_vp, c_u64, c_uint, c_uint, c_uint,
                                          ctypes.c_float, c_uint, c_uint, c_uint, c_vp, c_u64,
                                          c_vp]),
    "dspsr_b200_sk_mask_overlap": (c_int, [c_vp, c_vp, c_vp, c_u64, c_vp, c_u64, c_uint, c_uint,
                                           c_uint, c_uint, c_u64, c_u64, c_u64]),
    "dspsr_b200_sk_detect_ft": (c_int, [c_vp, c_vp, c_vp, c_u64, c_uint, c_uint, c_uint, c_uint,
                                        ctypes.c_float, ctypes.c_float, c_vp, c_vp]),
    "dspsr_b200_sk_detect_tscr": (c_int, [c_vp, c_vp, c_vp, c_u64, c_uint, c_uint, c_uint, c_uint,
                                          ctypes.c_float, c_vp, ctypes.POINTER(ctypes.c_uint32)]),
    "dspsr_b200_sk_reset_mask": (c_int, [c_vp, c_vp, c_u64, c_uint]),
    "dspsr_b200_sk_count_mask": (c_int, [c_vp, c_vp, c_u64, c_uint, c_u64p]),
    "dspsr_b200_sk_mask": (c_int, [c_vp, c_vp, c_vp, c_u64, c_vp, c_u64, c_u64, c_uint, c_uint,
                                   c_uint]),
    "dspsr_b200_pipeline_sk_counts": (c_int, [c_vp, c_u64p, c_u64p]),
    "dspsr_b200_pipeline_set_rfi_proposer": (c_int, [c_vp, c_vp, ctypes.c_float]),
    "dspsr_b200_rfi_proposer_features": (c_int, [c_vp, c_vp, c_vp, c_u64, c_uint]),
    "dspsr_b200_rfi_proposer_train": (c_int, [c_vp, c_vp, c_uint, c_uint, ctypes.c_float,
                                              ctypes.c_float, c_fp]),
    "dspsr_b200_rfi_proposer_infer": (c_int, [c_vp, c_vp, ctypes.c_float, c_vp, c_vp, c_u64p]),
    "dspsr_b200_rfi_proposer_get_params": (c_int, [c_vp, c_fp, ctypes.POINTER(c_uint)]),
    "dspsr_b200_rfi_proposer_set_params": (c_int, [c_vp, c_fp, c_uint]),
    "dspsr_b200_rfi_proposer_get_features": (c_int, [c_vp, c_fp]),
    "dspsr_b200_fold_create": (c_int, [c_vp, c_uint, c_uint, c_uint, ctypes.POINTER(c_vp)]),
    "dspsr_b200_fold_destroy": (c_int, [c_vp]),
    "dspsr_b200_fold_set_bins": (c_int, [c_vp, c_dbl, c_dbl, c_u64, c_u64, c_u64p]),
    "dspsr_b200_fold_fold": (c_int, [c_vp, c_vp, c_u64]),
    "dspsr_b200_fold_binplan": (c_int, [c_vp, c_vp]),
    "dspsr_b200_fold_get_profiles": (c_int, [c_vp, c_fp, c_u32p]),
    "dspsr_b200_fold_reset": (c_int, [c_vp]),
    "dspsr_b200_pipeline_create": (c_int, [c_vp, ctypes.POINTER(PipelineConfig),
                                           ctypes.POINTER(c_vp)]),
    "dspsr_b200_pipeline_destroy": (c_int, [c_vp]),
    "dspsr_b200_pipeline_run": (c_int, [c_vp, c_vp, c_u64, c_u64, c_u64p]),
    "dspsr_b200_pipeline_run_host": (c_int, [c_vp, c_vp, c_u64, c_u64p]),
    "dspsr_b200_pipeline_get_profiles": (c_int, [c_vp, c_fp, c_u32p]),
    "dspsr_b200_pipeline_get_profiles_async": (c_int, [c_vp, c_fp, ctypes.POINTER(ctypes.c_uint32)]),
    "dspsr_b200_pipeline_wait_profiles": (c_int, [c_vp]),
    "dspsr_b200_pipeline_reset": (c_int, [c_vp]),
    "dspsr_b200_pipeline_info": (c_int, [c_vp, c_u64p]),
    "dspsr_b200_pipeline_profile": (c_int, [c_vp, c_int]),
    "dspsr_b200_pipeline_kernel_times": (c_int, [c_vp, ctypes.POINTER(c_dbl), c_u64p]),
    "dspsr_b200_kernel_launches": (c_u64, []),
    "dspsr_b200_host_error": (ctypes.c_char_p, []),
    "dspsr_b200_time_divide_create": (c_int, [c_dbl, c_dbl, c_dbl, c_i64, c_i64, c_dbl,
                                              ctypes.POINTER(c_vp)]),
    "dspsr_b200_time_divide_block": (c_int, [c_vp, c_i64, c_i64, c_dbl, c_u64, c_dbl,
                                             ctypes.POINTER(SubintAction), c_u64, c_u64p]),
    "dspsr_b200_time_divide_destroy": (c_int, [c_vp]),
    "dspsr_b200_pipeline_set_unloader": (c_int, [c_vp, UNLOAD_FN, c_vp]),
    "dspsr_b200_pipeline_subints_ready": (c_int, [c_vp, c_u64p]),
    "dspsr_b200_pipeline_pop_subint": (c_int, [c_vp, ctypes.POINTER(Subint), c_fp, c_u32p]),
    "dspsr_b200_pipeline_finish": (c_int, [c_vp]),
    "dspsr_b200_ascii_header_get": (c_int, [ctypes.c_char_p, ctypes.c_char_p, c_vp, c_u64]),
    "dspsr_b200_ascii_header_set": (c_int, [c_vp, c_u64, ctypes.c_char_p, ctypes.c_char_p]),
    "dspsr_b200_dada_parse": (c_int, [ctypes.c_char_p, c_u64, ctypes.POINTER(DadaInfo)]),
    "dspsr_b200_dada_open": (c_int, [ctypes.c_char_p, ctypes.POINTER(c_vp),
                                     ctypes.POINTER(DadaInfo)]),
    "dspsr_b200_dada_is_valid": (c_int, [ctypes.c_char_p]),
    "dspsr_b200_dada_header": (c_int, [c_vp, ctypes.POINTER(ctypes.c_char_p), c_u64p]),
    "dspsr_b200_dada_read": (c_int, [c_vp, c_u64, c_u64, c_vp, c_u64p]),
    "dspsr_b200_dada_close": (c_int, [c_vp]),
    "dspsr_b200_pipeline_run_dada": (c_int, [c_vp, c_vp, c_u64, c_u64, c_u64, c_u64p, c_u64p]),
}

_lib = None


class B200Error(RuntimeError):
    """A non-zero status from the C ABI (the reference's Error)."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code


def lib():
    """Load libdspsr_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C dspsr-kanyixia_b200` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
