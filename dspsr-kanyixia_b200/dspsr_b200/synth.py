"""Seeded synthetic baseband: Gaussian noise plus a dispersed pulse train.

Stands in for telescope data (no dataset is needed for this path).  The pulse
train is generated in the fold's own phase frame (Fold::get_phi with a
constant period) and dispersed by an FP64 inverse chirp applied to the whole
block in the Fourier domain -- an implementation independent of the
Dedispersion response the pipeline uses, so dedispersion restoring the pulse
is a real check.  Values are quantised to int8 (two's complement) or int16
with saturation, in TFPD order (time, channel, polarisation, re/im).
"""
import numpy as np

DM_DISPERSION = 2.41e-4   # DM (pc/cm^3) = 2.41e-4 D (s MHz^2)


def _phase(ndat, rate, period, start_mjd, epoch_mjd, idat0=0):
    """Pulse phase of each sample midpoint, in the fold's frame."""
    t0 = ((start_mjd[0] - epoch_mjd[0]) * 86400.0 + (start_mjd[1] - epoch_mjd[1])
          + (start_mjd[2] - epoch_mjd[2]))
    t = t0 + (np.arange(ndat, dtype=np.float64) + idat0 + 0.5) / rate
    return np.mod(t / period, 1.0)


def dispersion_phase(nfft, cf, bw, dm):
    """FP64 phase of the dispersion transfer function on an nfft-point FFT grid
    (FFT order) of a complex-sampled band of centre cf and width bw (MHz)."""
    k = np.fft.fftfreq(nfft) * nfft
    f = k * (bw / nfft)          # offset from the band centre, MHz
    d = dm / DM_DISPERSION * 1e6
    return 2 * np.pi * d * f * f / (cf * cf * (cf + f)) * np.sign(bw)


def dispersed_pulse_train(ndat, cf, bw, dm, period, duty=0.03, snr=20.0, sigma=10.0,
                          seed=0, start_mjd=(60000, 0, 0.0), epoch_mjd=(60000, 0, 0.0),
                          pulse_phase=0.3, npol=2, nbit=8, fft=None):
    """One block of ndat complex samples per polarisation, single channel.

    snr: pulse peak power over the noise power per sample.  Returns (raw TFPD
    array, truth dict).  fft: optional (forward, inverse) callables for the
    whole-block transforms (defaults to numpy)."""
    rng = np.random.default_rng(seed)
    rate = abs(bw) * 1e6
    ph = _phase(ndat, rate, period, start_mjd, epoch_mjd)
    on = (np.mod(ph - pulse_phase, 1.0) < duty).astype(np.float64)
    fwd, inv = fft if fft is not None else (np.fft.fft, np.fft.ifft)
    # the inverse of the dedispersion response exp(-i sign 2 pi D f^2/(cf^2 (cf+f)))
    chirp = np.exp(1j * dispersion_phase(ndat, cf, bw, dm))
    out = np.empty((ndat, npol, 2), np.float64)
    amp = np.sqrt(snr) * sigma
    for p in range(npol):
        s = (rng.standard_normal(ndat) + 1j * rng.standard_normal(ndat)) * (amp / np.sqrt(2)) * on
        s = inv(fwd(s) * chirp)
        noise = (rng.standard_normal(ndat) + 1j * rng.standard_normal(ndat)) * (sigma / np.sqrt(2))
        x = s + noise
        out[:, p, 0] = x.real
        out[:, p, 1] = x.imag
    if nbit == 8:
        raw = np.clip(np.round(out), -128, 127).astype(np.int8).view(np.uint8)
    else:
        raw = np.clip(np.round(out), -32768, 32767).astype(np.int16)
    return raw.reshape(-1), {"phase": pulse_phase + duty / 2, "duty": duty, "rate": rate}


def noise_block(ndat, nchan=1, npol=2, sigma=10.0, seed=0, nbit=8):
    """Gaussian noise only, TFPD int8/int16."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(ndat * nchan * npol * 2) * sigma
    if nbit == 8:
        return np.clip(np.round(v), -128, 127).astype(np.int8).view(np.uint8)
    return np.clip(np.round(v), -32768, 32767).astype(np.int16)
