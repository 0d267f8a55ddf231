#!/usr/bin/env python
"""bench.py -- DSPSR baseband hot path on B200: unpack -> overlap-save coherent
dedispersion -> detection -> fold, in complex Msamples/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--config c1|c2|c2d|c2d500|c3|c4|c5|c5ifb]

One step = one block of the workload processed end to end (unpack -> fold),
the InputBuffering overlap carried from block to block.  Inputs are seeded
synthetic baseband (Gaussian noise plus a pulse train dispersed by an FP64
inverse chirp); blocks cycle through four distinct buffers larger than L2.

Multi-GPU: the path has no exchange step (each GPU folds its own stream of
blocks; profiles would be summed once at the end), so N GPUs run N
independent replicas (weak scaling); rank 0 reports the max-over-ranks time.

--impl reference times the reference's CPU algorithm for the same workload
(the C++ CPU restatement in oracle/, all host cores), one bounded sample of
the block per step.
"""
import argparse
import contextlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dspsr-kanyixia_b200"))

START_MJD = (60000, 3600, 0.25)
EPOCH_MJD = (59999, 0, 0.0)

CONFIGS = {
    "c1": dict(
        workload=("single-channel coherent dedispersion: 16 MHz complex baseband at 1400 MHz, "
                  "2 pol int8, DM 67.99, FFT 2^17 (2^15 is below the reference's minimum), "
                  "Intensity, 1024-bin fold, P=89.33 ms, 2^24 samples/pol per block"),
        cf=1400.0, bw=16.0, dm=67.99, nchan=1, npol=2, nfft=1 << 17, nbin=1024,
        period=0.08933, state=0, ndat=1 << 24, duty=0.03, snr=20.0, sigma=10.0, fb=0),
    "c2": dict(
        workload=("filterbank + coherent dedispersion: 256 MHz complex baseband at 1400 MHz, "
                  "2 pol int8, FFT filterbank to 64 x 4 MHz channels, DM 500, per-channel FFT "
                  "2^16, full Stokes, 2048-bin fold, P=5.757 ms, 2^26 samples/pol per block "
                  "(four blocks = the 2^28-sample data set)"),
        cf=1400.0, bw=256.0, dm=500.0, nchan=1, npol=2, nfft=1 << 16, nbin=2048,
        period=5.757e-3, state=3, ndat=1 << 26, duty=0.03, snr=10.0, sigma=12.0, fb=64),
    "c3": dict(
        kind="c3",
        workload=("48 independent streams at once (beams / DM trials): dual-pol int8 complex "
                  "baseband at 1400 MHz, DM ~ U[10, 2000], bandwidth in {16, 32, 64, 128} MHz, "
                  "channels in {1, 8, 32}, FFT 2^12..2^18 per channel (optimal_fft_length), "
                  "Intensity, 512-4096 bins, 2^24 samples/pol per stream per step"),
        nstream=48, cf=1400.0, samples=1 << 24, seed=2024),
    "c4": dict(
        kind="sk",
        workload=("spectral kurtosis RFI excision: 512 channels x 2^20 samples x 2 pol complex "
                  "FP32 voltages (sigma 1) with 20 CW tones (0.5-5 sigma), 1 %-duty broadband "
                  "bursts (1-64 samples, 3-30 sigma) and one drifting chirp; M = 1024, "
                  "3 sigma thresholds (SKLimits), sums + mask + masked copy"),
        nchan=512, npol=2, ndat=1 << 20, M=1024, std_devs=3.0),
    "c5": dict(
        kind="c5",
        workload=("inverse PFB then re-channelised coherent dedispersion: 256 critically "
                  "spaced 4/3-oversampled PFB channels of int16 complex dual-pol voltages "
                  "(seeded Gaussian), 1024-point input FFTs stitched into 196608-point "
                  "spectra (12288-sample discards), FFT filterbank to 1024 channels, DM 1000 "
                  "at 1400 MHz over 800 MHz, per-channel overlap-save, full Stokes, "
                  "4096-bin fold, P=1.6 ms; 1 s of 800 MHz per block (4.17 M samples per "
                  "PFB channel)"),
        nin=256, npol=2, lin=1024, disc=12288, ndat=4166784, cf=1400.0, bw=800.0, dm=1000.0,
        fb=1024, nbin=4096, period=1.6e-3),
    "c5ifb": dict(
        kind="ifb",
        workload=("inverse filterbank stage of C5 alone: 256 PFB channels int16 dual-pol, "
                  "1024-point input FFTs, 196608-point output spectra, 1 s of 800 MHz"),
        nin=256, npol=2, lin=1024, disc=12288, ndat=4166784),
    "c2d": dict(
        kind="fbd",
        workload=("filterbank with the dedispersion inside it (-F 64:D): 256 MHz complex "
                  "baseband at 1400 MHz, 2 pol int8, one 2^18-point FFT per part, the "
                  "response of 64 x 4 MHz channels at DM 25, 64 inverse FFTs of 4096 points, "
                  "full Stokes, 2048-bin fold, P=5.757 ms, 2^26 samples/pol per block"),
        cf=1400.0, bw=256.0, dm=25.0, npol=2, nsub=64, freq_res=4096, nbin=2048,
        period=5.757e-3, state=3, ndat=1 << 26),
    "c2d500": dict(
        kind="fbd",
        workload=("C2 with the dedispersion inside the filterbank (-F 64:D): 256 MHz complex "
                  "baseband at 1400 MHz, 2 pol int8, DM 500, one 2^22-point FFT per part "
                  "(512 x 8192), 64 x 4 MHz channels of 65536 points, full Stokes, 2048-bin "
                  "fold, P=5.757 ms, 2^26 samples/pol per block"),
        cf=1400.0, bw=256.0, dm=500.0, npol=2, nsub=64, freq_res=65536, nbin=2048,
        period=5.757e-3, state=3, ndat=1 << 26),
}

NBLOCKS = 4


def _cpulist(text):
    out = set()
    for part in text.strip().split(","):
        if "-" in part:
            lo, hi = part.split("-")
            out.update(range(int(lo), int(hi) + 1))
        elif part:
            out.add(int(part))
    return out


@contextlib.contextmanager
def near_gpu_memory(local, info=None):
    """Host allocations made inside land in the memory of the NUMA node that
    the GPU is attached to: the thread runs on that node's cores while the
    pages are first touched, so the host-to-device copies of the end-to-end
    figures cross no socket link.  The thread's cores are restored after.
    Without NUMA information (no node, no sysfs) it changes nothing.  `info`
    (a dict) receives the node."""
    old = None
    try:
        import torch
        p = torch.cuda.get_device_properties(local)
        dev = (f"/sys/bus/pci/devices/{p.pci_domain_id:04x}:{p.pci_bus_id:02x}:"
               f"{p.pci_device_id:02x}.0")
        with open(dev + "/numa_node") as f:
            node = int(f.read())
        if node >= 0:
            with open(f"/sys/devices/system/node/node{node}/cpulist") as f:
                cpus = _cpulist(f.read())
            old = os.sched_getaffinity(0)
            os.sched_setaffinity(0, cpus)
            if info is not None:
                info["host_numa_node"] = node
    except Exception:
        pass
    try:
        yield
    finally:
        if old is not None:
            os.sched_setaffinity(0, old)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_init(backend="nccl"):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK).  The
    replicas share nothing but the barriers around the timed region and the
    max over ranks of its duration; "gloo" runs the same plumbing on CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per input sample of a kernel from a committed ncu summary
    (profiles/ncu_traffic.txt lines 'kernel=<config>:<name> bytes_per_sample=<B>',
    each from one ncu capture, dram__bytes_read.sum + dram__bytes_write.sum of a
    launch divided by the input samples that launch covered)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = dict(kv.split("=", 1) for kv in line.split() if "=" in kv)
        if parts.get("kernel") == kernel and "bytes_per_sample" in parts:
            return float(parts["bytes_per_sample"])
    return None


# ---------------------------------------------------------------------------
# synthetic blocks
# ---------------------------------------------------------------------------

FFT_FORMS = {"fp32": 0, "bf16x2": 2, "bf16x3": 3}


def make_blocks(cfg, seed, device):
    """NBLOCKS consecutive int8 TFPD blocks generated on the GPU (torch is the
    synthesis tool here; the product path never uses it)."""
    import torch
    from dspsr_b200 import synth
    ndat, npol = cfg["ndat"], cfg["npol"]
    rate = abs(cfg["bw"]) * 1e6
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    chirp = None
    blocks = []
    for b in range(NBLOCKS):
        ph = torch.from_numpy(synth._phase(ndat, rate, cfg["period"], START_MJD, EPOCH_MJD,
                                           idat0=b * ndat)).to(device)
        on = (torch.remainder(ph - 0.3, 1.0) < cfg["duty"]).to(torch.float64)
        if chirp is None:
            dphi = torch.from_numpy(synth.dispersion_phase(ndat, cfg["cf"], cfg["bw"],
                                                           cfg["dm"])).to(device)
            chirp = torch.polar(torch.ones_like(dphi), dphi)
            del dphi
        out = torch.empty((ndat, npol, 2), dtype=torch.int8, device=device)
        amp = np.sqrt(cfg["snr"]) * cfg["sigma"] / np.sqrt(2)
        for p in range(npol):
            s = torch.complex(torch.randn(ndat, generator=gen, device=device, dtype=torch.float64),
                              torch.randn(ndat, generator=gen, device=device, dtype=torch.float64))
            s = torch.fft.ifft(torch.fft.fft(s * (amp * on)) * chirp)
            n = torch.randn((ndat, 2), generator=gen, device=device, dtype=torch.float64)
            n = n * (cfg["sigma"] / np.sqrt(2))
            n[:, 0] += s.real
            n[:, 1] += s.imag
            out[:, p, :] = torch.clamp(torch.round(n), -128, 127).to(torch.int8)
            del s, n
        blocks.append(out.reshape(-1).view(torch.uint8))
        del ph, on
    del chirp
    # hand the synthesis buffers back so that only the pipeline's memory stays
    torch.cuda.empty_cache()
    torch.cuda.synchronize()
    return blocks


# ---------------------------------------------------------------------------
# CPU: reference arm and cpu_baseline (the oracle restatement of the
# reference's CPU path; test infrastructure, timed here as the CPU baseline)
# ---------------------------------------------------------------------------

def nchan_conv(cfg):
    """Channels the dedispersion sees (after the filterbank, if any)."""
    return cfg["nchan"] * (cfg["fb"] or 1)


def cpu_prepare(cfg):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.lib()
    nc = nchan_conv(cfg)
    pos = orc.smearing_samples(cfg["cf"], cfg["bw"], cfg["dm"], nc, 1)
    neg = orc.smearing_samples(cfg["cf"], cfg["bw"], cfg["dm"], nc, -1)
    lut, _ = orc.bittable8(0.0308)
    if cfg["fb"]:
        freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nc, swap=True, dc_centred=True)
        h = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], cfg["nfft"], mode=0)
    else:
        h = orc.dedispersion_response(cfg["cf"], cfg["bw"], cfg["dm"], 1, cfg["nfft"], mode=0)
    return orc, pos, neg, lut, h


def cpu_sample(cfg, orc, pos, neg, lut, h, nparts, seed=1):
    """Bounded sample: nparts FFT parts (of every channel) of a block, int8 noise."""
    from dspsr_b200 import synth
    nk = cfg["nfft"] - pos - neg
    ndat = (cfg["nfft"] + (nparts - 1) * nk) * (cfg["fb"] or 1)
    raw = synth.noise_block(ndat, cfg["nchan"], cfg["npol"], cfg["sigma"], seed)
    return raw, ndat


def cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads):
    """The reference's CPU chain on one sample: unpack -> (filterbank) ->
    overlap-save -> detection -> fold (oracle/, all host threads in the FFTs)."""
    nc = nchan_conv(cfg)
    rate = abs(cfg["bw"]) / nc * 1e6
    phi = orc.fold_phi(START_MJD, EPOCH_MJD, pos, rate, cfg["period"])
    pps = (1 / rate) / cfg["period"]
    t0 = time.perf_counter()
    if not cfg["fb"]:
        orc.pipeline_c1(raw, ndat, lut, h, cfg["nfft"], pos, neg, phi, pps, cfg["nbin"], threads)
    else:
        x = orc.unpack8(raw, ndat, cfg["nchan"], cfg["npol"], 2, lut)
        x = x.view(np.complex64).reshape(cfg["nchan"], cfg["npol"], ndat)
        y = orc.filterbank(x, cfg["fb"])
        z = orc.convolve(y, h, cfg["nfft"], pos, neg, nthreads=threads)
        d = orc.detect(z, cfg["state"])
        plan = orc.fold_binplan(phi, pps, z.shape[2], cfg["nbin"])
        orc.fold_accumulate(d, plan, cfg["nbin"])
    return time.perf_counter() - t0


def block_parts(cfg, pos, neg):
    """FFT parts (per channel) one block of the workload holds."""
    nk = cfg["nfft"] - pos - neg
    return (cfg["ndat"] // (cfg["fb"] or 1) - pos - neg) // nk


def cpu_baseline(cfg, target_s=15.0):
    """One block of the workload through the CPU restatement, repeated until
    about target_s seconds of CPU work have been timed."""
    orc, pos, neg, lut, h = cpu_prepare(cfg)
    threads = os.cpu_count() or 1
    nparts = block_parts(cfg, pos, neg)
    raw, ndat = cpu_sample(cfg, orc, pos, neg, lut, h, nparts)
    cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads)      # plans, page-in
    total, reps = 0.0, 0
    while total < target_s:
        total += cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads)
        reps += 1
    msps = ndat * cfg["npol"] * reps / total / 1e6
    return {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
            "kind": "port",
            "sample": (f"{nparts} FFT parts per channel ({ndat} input samples/pol, "
                       f"{cfg['npol']} pol) x {reps} through the oracle CPU restatement "
                       f"(self-written FP32 FFT, OpenMP over parts), {total:.1f} s")}


def noalloc_compare(b2, ctx):
    """dspsr_b200_convolution_perform_noalloc beside the engine entry point
    (dspsr_b200_convolution_perform) on one shape that fits the no-alloc
    entry's static 32 MiB array: one channel, two polarisations, C1's FFT
    length and smearing, 2^21 complex float samples per polarisation on the
    device; CUDA events around 10 calls of each after 3 warm-up calls (outside
    the timed region of the line)."""
    import ctypes
    import torch
    nchan, npol, nfft, pos, neg = 1, 2, 1 << 17, 28462, 29455
    nk = nfft - pos - neg
    ndat = 1 << 21
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    x = torch.complex(torch.randn((nchan, npol, ndat), generator=gen, device="cuda"),
                      torch.randn((nchan, npol, ndat), generator=gen, device="cuda"))
    rng = np.random.default_rng(5)
    h = ((rng.standard_normal((nchan, nfft)) + 1j * rng.standard_normal((nchan, nfft)))
         / np.sqrt(nfft)).astype(np.complex64)
    hd = torch.from_numpy(h).cuda()
    conv = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    conv.copy_response(h)
    npart = conv.npart(ndat)
    out_e = torch.empty((nchan, npol, npart * nk), dtype=torch.complex64, device="cuda")
    out_n = torch.empty_like(out_e)
    lib = b2._capi.lib()
    nret = ctypes.c_uint64()

    def engine():
        conv.perform(x, ndat, ndat, out_e, npart * nk)

    def noalloc():
        rc = lib.dspsr_b200_convolution_perform_noalloc(
            None, x.data_ptr(), ndat, ndat, nchan, npol, nfft, pos, neg, hd.data_ptr(),
            out_n.data_ptr(), npart * nk, ctypes.byref(nret), None)
        if rc != 0:
            raise RuntimeError(f"noalloc call failed: {rc}")

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 10

    ms_e, ms_n = timed(engine), timed(noalloc)
    a = out_n.cpu().numpy().astype(np.complex128)
    b = out_e.cpu().numpy().astype(np.complex128)
    conv.close()
    return {"shape": f"{nchan} ch x {npol} pol x {ndat} complex float, nfft {nfft}, "
                     f"{npart} parts", "engine_ms_per_call": round(ms_e, 4),
            "noalloc_ms_per_call": round(ms_n, 4),
            "rel_rms_difference": float(np.sqrt(np.mean(np.abs(a - b) ** 2)
                                                / np.mean(np.abs(b) ** 2)))}


def parity_block(cfg, b2, ctx, pcfg, raw_dev, ndat, pos, neg, nfft, lut):
    """One full block of the timed workload (its first block, a fresh
    pipeline) against the oracle chain on the same bytes: unpack -> (the
    filterbank) -> overlap-save -> detection -> fold with the block's phase
    (Convolution.C:724-803, Fold.C:790-837).  Returns the max relative error of
    the folded profiles (per bin, against the bin's total power) and whether
    the hits are bit-exact."""
    orc = cpu_prepare(cfg)[0]
    pl = b2.Pipeline(ctx, pcfg)
    nout = pl.run(raw_dev, ndat)
    prof, hits = pl.get_profiles()
    pl.close()
    raw = raw_dev.cpu().numpy()
    nc = nchan_conv(cfg)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    x = orc.unpack8(raw, ndat, cfg["nchan"], cfg["npol"], 2, np.asarray(lut, np.float32))
    x = x.view(np.complex64).reshape(cfg["nchan"], cfg["npol"], ndat)
    if cfg["fb"]:
        x = orc.filterbank(x, cfg["fb"])
        freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nc, swap=True, dc_centred=True)
        h = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], nfft, mode=0)
    else:
        h = orc.dedispersion_response(cfg["cf"], cfg["bw"], cfg["dm"], 1, nfft, mode=0)
    y = orc.convolve(x, h, nfft, pos, neg, nthreads=threads)
    del x
    d = orc.detect(y, cfg["state"])
    rate = abs(cfg["bw"]) / nc * 1e6
    phi = orc.fold_phi(START_MJD, EPOCH_MJD, pos, rate, cfg["period"])
    plan = orc.fold_binplan(phi, (1.0 / rate) / cfg["period"], y.shape[2], cfg["nbin"])
    del y
    rprof, rhits = orc.fold_accumulate(d, plan, cfg["nbin"])
    rprof = rprof.astype(np.float64)
    # scale: the bin itself for intensity-like products, else total power
    if cfg["state"] in (0, 1):
        scale = np.abs(rprof)
    else:
        scale = np.broadcast_to(rprof[:, 0:1] if cfg["state"] == 3
                                else rprof[:, 0:1] + rprof[:, 1:2], rprof.shape)
    hit = rhits > 0
    err = float(np.max(np.abs(prof.astype(np.float64) - rprof)[..., hit] / scale[..., hit]))
    ok = bool(np.array_equal(hits, rhits)) and err < 1e-5 and int(nout) == int(d.shape[2])
    return {"block": f"first timed block, {ndat} input samples/pol, fresh pipeline",
            "samples_folded": int(nout), "oracle_samples": int(d.shape[2]),
            "hits_bit_exact": bool(np.array_equal(hits, rhits)),
            "max_profile_rel_err": err, "rtol": 1e-5, "pass": ok,
            "oracle_s": round(time.perf_counter() - t0, 2),
            "oracle": "CPU restatement (FP32, reference-mode chirp)"}


def run_reference(args, cfg, world, rank):
    if rank != 0:
        return
    orc, pos, neg, lut, h = cpu_prepare(cfg)
    threads = os.cpu_count() or 1
    raw, ndat = cpu_sample(cfg, orc, pos, neg, lut, h, threads)
    t1 = cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads)
    budget = 150.0 / max(1, args.steps + args.warmup)
    nparts = max(threads, int(threads * budget / max(t1, 1e-3)))
    nparts = min(nparts, block_parts(cfg, pos, neg))
    raw, ndat = cpu_sample(cfg, orc, pos, neg, lut, h, nparts)
    for _ in range(args.warmup):
        cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads)
    ts = [cpu_run(cfg, orc, pos, neg, lut, h, raw, ndat, threads) for _ in range(args.steps)]
    total = sum(ts)
    msps = ndat * cfg["npol"] * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s unpack->fold", "value": round(msps, 3),
        "unit": "complex Msamples/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian noise, int8)",
        "config": {"workload": cfg["workload"], "sample_parts_per_step": nparts},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
                         "kind": "port",
                         "sample": (f"{nparts} FFT parts per step ({ndat} samples/pol); the "
                                    "reference's own build (DSPSR+PSRCHIVE+FFTW) is not "
                                    "buildable here, so its CPU algorithm runs as the oracle "
                                    "restatement")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_b200(args, cfg, world, rank, local):
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = b2.Context(local)
    nc = nchan_conv(cfg)
    pos, neg, nfft = b2.dispersion_plan(cfg["cf"], cfg["bw"], cfg["dm"], nc, cfg["nfft"])
    nk = nfft - pos - neg
    lut, _ = b2.bittable8()
    if args.lut_perturb:
        # a table that is not (x + 0.5) * scale: the kernels look it up
        lut = (np.asarray(lut, np.float32)
               * (1 + 1e-3 * np.sin(np.arange(256)))).astype(np.float32)
    c = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], nfft, pos,
                       neg, cfg["nbin"], cfg["period"], state=cfg["state"], lut=lut,
                       start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, filterbank_nchan=cfg["fb"],
                       scratch_bytes=args.scratch_mib << 20)
    blocks = make_blocks(cfg, 1234 + rank, device)
    ndat = cfg["ndat"]
    samples_per_step = ndat * cfg["npol"]   # complex samples consumed per step (all pols)
    bytes_per_block = blocks[0].numel()

    # ---- device-resident timed region --------------------------------------
    pl = b2.Pipeline(ctx, c)
    # the clock sampler starts before the warm-up so that nvidia-smi's own
    # start-up (NVML initialisation) is over before the timed region
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for i in range(args.warmup):
        pl.run(blocks[i % NBLOCKS], ndat)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    folded = 0
    for i in range(args.steps):
        folded += pl.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
    ev1.record()
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6

    # the same K steps again with CUDA events around every kernel, for the
    # per-kernel durations of the roofline (the events themselves cost ~10 %,
    # so `value` above is taken without them)
    pl.profile(True)
    for i in range(args.steps):
        pl.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
    ktimes = pl.kernel_times()
    pl.profile(False)
    info = pl.info()
    prof, hits = pl.get_profiles()
    pl.close()

    # the mixed-precision arms: the same workload with the convolution's row
    # FFTs on the tensor cores (split-BF16 DFT GEMMs), timed the same way
    mixed = {}
    forms = [f for f in args.fft.split(",") if f in FFT_FORMS and f != "fp32"]
    if info["n1"] > 1 and forms:
        for form in forms:
            cm = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], nfft,
                                pos, neg, cfg["nbin"], cfg["period"], state=cfg["state"],
                                lut=lut, start_mjd=START_MJD, epoch_mjd=EPOCH_MJD,
                                filterbank_nchan=cfg["fb"], scratch_bytes=args.scratch_mib << 20,
                                fft_precision=FFT_FORMS[form])
            pm = b2.Pipeline(ctx, cm)
            for i in range(args.warmup):
                pm.run(blocks[i % NBLOCKS], ndat)
            torch.cuda.synchronize()
            barrier(world)
            torch.cuda.synchronize()
            m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            m0.record()
            for i in range(args.steps):
                pm.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
            m1.record()
            torch.cuda.synchronize()
            mms = max_over_ranks(m0.elapsed_time(m1), world)
            pm.profile(True)
            for i in range(args.steps):
                pm.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
            mk = pm.kernel_times()
            pm.profile(False)
            mprof, mhits = pm.get_profiles()
            pm.close()
            mval = samples_per_step * args.steps * world / (mms / 1e3) / 1e6
            scale = np.maximum(np.abs(prof[:, :1].astype(np.float64)), 1e-30)
            hit = hits > 0
            mixed[form] = {
                "value": round(mval, 3), "ms_per_step": round(mms / args.steps, 4),
                "ratio_to_fp32": round(mval / value, 4),
                "kernel_ms": {k: round(v[0], 3) for k, v in mk.items() if v[1]},
                "profile_max_rel_diff_vs_fp32": float(np.max(
                    np.abs(mprof.astype(np.float64) - prof)[..., hit]
                    / np.broadcast_to(scale, prof.shape)[..., hit])),
                "hits_equal_fp32": bool(np.array_equal(mhits, hits)),
                "note": ("rows on the tensor cores (tcgen05.mma kind::f16, DFT16/DFT32 "
                         f"stages, {form[-1]} BF16 terms per operand), columns, filterbank, "
                         "detection and fold as in the FP32 arm")}

    # ---- end to end through the public API from pinned host memory ----------
    numa = {}
    with near_gpu_memory(local, numa):
        host = [b.cpu().pin_memory() for b in blocks]
    pl = b2.Pipeline(ctx, c)
    for i in range(args.warmup):
        pl.run_host(host[i % NBLOCKS], ndat)
        pl.get_profiles()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # each step's result (the profiles after its block) comes back
    # asynchronously into page-locked buffers and is waited for once the next
    # block is queued, as a streaming reader of PhaseSeries would
    bufs = [pl.profile_buffers(), pl.profile_buffers()]
    e0.record()
    for i in range(args.steps):
        pl.run_host(host[(args.warmup + i) % NBLOCKS], ndat)
        if i:
            pl.wait_profiles()              # step i-1's result on the host
        pl.get_profiles_async(*bufs[i % 2])
    pl.wait_profiles()                      # the last step's result
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), 1e3 * wall), world)
    p2, h2 = bufs[(args.steps - 1) % 2]
    pl.close()
    e2e = samples_per_step * args.steps * world / (e2e_ms / 1e3) / 1e6
    d2h = p2.nbytes + h2.nbytes

    # ---- optional: sub-integrations, and end to end from a DADA file ---------
    extra = {}
    if args.subint_seconds > 0:
        cs = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], nfft,
                            pos, neg, cfg["nbin"], cfg["period"], state=cfg["state"], lut=lut,
                            start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, filterbank_nchan=cfg["fb"],
                            scratch_bytes=args.scratch_mib << 20,
                            subint_seconds=args.subint_seconds, subint_slots=64)
        pl = b2.Pipeline(ctx, cs)
        nsub = [0]
        pl.set_unloader(lambda info, prof_, hits_: nsub.__setitem__(0, nsub[0] + 1))
        for i in range(args.warmup):
            pl.run(blocks[i % NBLOCKS], ndat)
        torch.cuda.synchronize()
        nsub[0] = 0
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for i in range(args.steps):
            pl.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
        s1.record()
        torch.cuda.synchronize()
        sms = max_over_ranks(s0.elapsed_time(s1), world)
        pl.finish()
        pl.close()
        extra["subint"] = {"seconds": args.subint_seconds, "subints_unloaded": nsub[0],
                           "value": round(samples_per_step * args.steps * world / (sms / 1e3) / 1e6, 3),
                           "ms_per_step": round(sms / args.steps, 4),
                           "note": "device-resident input; every closed sub-integration is "
                                   "copied to the host and handed to the unloader callback"}
    if args.interchannel:
        ck = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nchan"], cfg["npol"], nfft,
                            pos, neg, cfg["nbin"], cfg["period"], state=cfg["state"], lut=lut,
                            start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, filterbank_nchan=cfg["fb"],
                            scratch_bytes=args.scratch_mib << 20, interchannel=1)
        pl = b2.Pipeline(ctx, ck)
        for i in range(args.warmup):
            pl.run(blocks[i % NBLOCKS], ndat)
        torch.cuda.synchronize()
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record()
        kfold = 0
        for i in range(args.steps):
            kfold += pl.run(blocks[(args.warmup + i) % NBLOCKS], ndat)
        k1.record()
        torch.cuda.synchronize()
        kms = max_over_ranks(k0.elapsed_time(k1), world)
        pl.close()
        extra["interchannel"] = {
            "value": round(samples_per_step * args.steps * world / (kms / 1e3) / 1e6, 3),
            "ms_per_step": round(kms / args.steps, 4), "samples_folded": int(kfold),
            "note": "device-resident input; the convolution's voltages go through memory to "
                    "SampleDelay + detect + fold (one extra round trip)"}
    if args.dada:
        import tempfile
        with tempfile.TemporaryDirectory() as tmpd:
            path = os.path.join(tmpd, "c.dada")
            keys = {"HDR_VERSION": "1.0", "TELESCOPE": "synthetic", "SOURCE": "synthetic",
                    "INSTRUMENT": "dspsr_b200", "FREQ": cfg["cf"], "BW": cfg["bw"],
                    "NCHAN": cfg["nchan"], "NPOL": cfg["npol"], "NBIT": 8, "NDIM": 2,
                    "TSAMP": cfg["nchan"] / abs(cfg["bw"]), "UTC_START": "2023-02-25-01:00:00",
                    "OBS_OFFSET": 0}
            with open(path, "wb") as fh:
                text = b""
                hdr = b2.ascii_header_set("", "HDR_SIZE", 4096)
                for k, v in keys.items():
                    hdr = b2.ascii_header_set(hdr, k, v)
                text = hdr.encode()
                fh.write(text + b"\0" * (4096 - len(text)))
                for hb in host:
                    fh.write(hb.numpy().tobytes())
            f = b2.DADAFile(path)
            pl = b2.Pipeline(ctx, f.pipeline_config(cfg["dm"], nfft, pos, neg, cfg["nbin"],
                                                    cfg["period"], state=cfg["state"], lut=lut,
                                                    epoch_mjd=EPOCH_MJD,
                                                    filterbank_nchan=cfg["fb"],
                                                    scratch_bytes=args.scratch_mib << 20))
            # each call streams the whole file (NBLOCKS blocks), so every
            # block's read overlaps the previous block's upload and kernels
            nfile = f.ndat // ndat
            pl.run_dada(f, ndat)
            pl.get_profiles()
            torch.cuda.synchronize()
            barrier(world)
            ncall = max(1, args.steps // nfile)
            d0 = time.perf_counter()
            for i in range(ncall):
                pl.run_dada(f, ndat)
                pd, hd = pl.get_profiles()
            torch.cuda.synchronize()
            dms = max_over_ranks(1e3 * (time.perf_counter() - d0), world) / (ncall * nfile) * args.steps
            pl.close()
            f.close()
            extra["dada_e2e"] = {"value": round(samples_per_step * args.steps * world / (dms / 1e3) / 1e6, 3),
                                 "unit": "complex Msamples/s", "ms_per_step": round(dms / args.steps, 4),
                                 "file_bytes": int(os.path.getsize(path)) if os.path.exists(path) else None,
                                 "block_ndat": ndat,
                                 "note": "pipeline_run_dada over a DADA file of the same blocks "
                                         "(one call per pass over the file, profiles read back "
                                         "after each), read through two pinned buffers; the "
                                         "file was just written, so reads come from the page "
                                         "cache"}

    # ---- roofline of the dominant kernel -----------------------------------
    hbm_peak, bf16_peak, peak_src = measured_peaks()
    name, (kms, kn) = max(ktimes.items(), key=lambda kv: kv[1][0])
    # Algorithmic bytes: the int8 input, 2 bytes per complex sample per pol.
    # Each kernel kind covers all input of the timed region over its kn
    # launches (a batch of FFT parts of every channel, or a whole block).
    samples_per_launch = ndat * args.steps / max(kn, 1)
    alg_bytes = 2.0 * cfg["npol"] * samples_per_launch
    avg_s = kms / 1e3 / max(kn, 1)
    achieved = alg_bytes / avg_s / 1e9
    tb = ncu_traffic(f"{args.config}:{name}")
    # committed summaries give DRAM bytes per input sample of the kernel
    traffic = tb * samples_per_launch if tb else None
    # FP32 view: flops per output sample of the FFT convolution (log2 N radix-2
    # count, both transforms, overlap included) + detection + fold (+ the
    # filterbank's own FFT when there is one)
    import math
    flop_per_sample = (nfft / nk) * (2 * 5 * math.log2(nfft) + 6) + 5
    if cfg["fb"]:
        flop_per_sample += 5 * math.log2(cfg["fb"]) + 2
    fp32_tflops = flop_per_sample * folded * nc * cfg["npol"] / (ms / 1e3) / 1e12
    fp32_peak = 148 * 128 * 2 * (clk["sm_mhz"] or 1965.0) * 1e6 / 1e12

    line = {
        "metric": "complex Msamples/s unpack->fold", "value": round(value, 3),
        "unit": "complex Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian noise + FP64-dispersed pulse train, int8)",
        "config": {"workload": cfg["workload"], "nfft": nfft, "nfilt_pos": pos,
                   "nfilt_neg": neg, "nkeep": nk, "fft_split": [info["n1"], info["n2"]],
                   "filterbank_nchan": cfg["fb"], "nchan_dedispersed": nc,
                   "parts_per_batch": info["max_batch"],
                   "l2": f"inputs larger than L2: {NBLOCKS} distinct {bytes_per_block >> 20} MiB "
                         "blocks cycled",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "kernel_ms": {k: round(v[0], 3) for k, v in ktimes.items() if v[1]},
        "roofline": {"bound": "hbm", "kernel": name, "achieved": round(achieved, 2),
                     "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                     "traffic": traffic, "peak_source": peak_src,
                     "note": "path is FP32-ALU bound (2 B/sample in); see roofline_fp32"},
        "roofline_fp32": {"achieved": round(fp32_tflops, 3), "unit": "TFLOP/s",
                          "peak": round(fp32_peak, 1), "frac": round(fp32_tflops / fp32_peak, 4),
                          "flop_per_sample": round(flop_per_sample, 1),
                          "peak_source": "148 SM x 128 FP32 lanes x 2 x median SM clock"},
        "e2e": {"value": round(e2e, 3), "unit": "complex Msamples/s",
                "h2d_bytes_per_step": int(bytes_per_block), "d2h_bytes_per_step": int(d2h),
                "readback": "each step's profiles copied back asynchronously and waited for "
                            "once the next block is queued", **numa},
        "mixed": mixed or None,
        "check": {"samples_folded": int(folded), "hits_total": int(hits.sum()),
                  "profile_peak_over_median": float(np.max(prof) / max(np.median(prof), 1e-30))},
    }
    line.update(extra)
    if rank == 0 and world == 1 and args.config == "c1":
        line["noalloc"] = noalloc_compare(b2, ctx)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg)
        line["parity"] = parity_block(cfg, b2, ctx, c, blocks[0], ndat, pos, neg, nfft, lut)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


# ---------------------------------------------------------------------------
# SpectralKurtosis workload
# ---------------------------------------------------------------------------

def make_sk_block(cfg, seed, device):
    """Complex FPT voltages [nchan][npol][ndat] with injected RFI, generated on
    the GPU (torch is the synthesis tool here, not the product path)."""
    import torch
    nchan, npol, ndat, M = cfg["nchan"], cfg["npol"], cfg["ndat"], cfg["M"]
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    x = torch.randn((nchan, npol, ndat, 2), generator=gen, device=device) * (1 / np.sqrt(2))
    rng = np.random.default_rng(seed)
    t = torch.arange(ndat, device=device, dtype=torch.float64)
    for _ in range(20):                                   # CW tones
        c = int(rng.integers(nchan))
        amp, f = rng.uniform(0.5, 5.0), rng.uniform(-0.5, 0.5)
        ph = 2 * np.pi * f * t
        for p in range(npol):
            x[c, p, :, 0] += (amp * torch.cos(ph)).float()
            x[c, p, :, 1] += (amp * torch.sin(ph)).float()
    nburst = int(0.01 * ndat / 32.5)                      # 1 % duty, widths 1..64
    for _ in range(nburst):
        w = int(rng.integers(1, 65))
        t0 = int(rng.integers(0, ndat - w))
        x[:, :, t0:t0 + w, :] *= float(rng.uniform(3.0, 30.0))
    nblk = ndat // M                                      # drifting chirp, 3 sigma
    ph = 2 * np.pi * (0.05 * t[:M] + 1e-5 * t[:M] * t[:M])
    for b in range(nblk):
        c = (b * nchan) // nblk
        seg = slice(b * M, (b + 1) * M)
        for p in range(npol):
            x[c, p, seg, 0] += (3 * torch.cos(ph)).float()
            x[c, p, seg, 1] += (3 * torch.sin(ph)).float()
    torch.cuda.synchronize()
    return x.reshape(-1)


def sk_bytes_per_sample(inplace):
    # read 8 B per complex sample; write it back (out of place) or nothing
    return 8.0 if inplace else 16.0


def sk_cpu_sample(cfg):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    M, npol = cfg["M"], cfg["npol"]
    lo, hi = orc.sk_limits(M, 1, cfg["std_devs"], npol)
    # bounded sample: 16 channels of the block, all of their time
    nchan_s = max(1, min(cfg["nchan"], 16))
    rng = np.random.default_rng(7)
    x = (rng.standard_normal((nchan_s, npol, cfg["ndat"])) +
         1j * rng.standard_normal((nchan_s, npol, cfg["ndat"]))).astype(np.complex64)
    return orc, lo, hi, nchan_s, x


def run_reference_sk(args, cfg, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    orc, lo, hi, nchan_s, x = sk_cpu_sample(cfg)
    M, npol = cfg["M"], cfg["npol"]

    def step():
        t0 = time.perf_counter()
        orc.sk(x, M, lo, hi)
        return time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    total = sum(step() for _ in range(args.steps))
    msps = nchan_s * npol * cfg["ndat"] * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s spectral kurtosis",
        "value": round(msps, 3), "unit": "complex Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic (seeded Gaussian complex voltages)",
        "config": {"workload": cfg["workload"], "sample_channels_per_step": nchan_s},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
                         "kind": "port",
                         "sample": (f"{nchan_s} of {cfg['nchan']} channels x {cfg['ndat']} "
                                    f"samples x {npol} pol per step through the oracle "
                                    "restatement of SpectralKurtosis compute/detect/mask "
                                    "(OpenMP over blocks)")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sk(cfg, target_s=12.0):
    threads = os.cpu_count() or 1
    orc, lo, hi, nchan_s, x = sk_cpu_sample(cfg)
    M, npol = cfg["M"], cfg["npol"]
    orc.sk(x, M, lo, hi)
    total, reps = 0.0, 0
    while total < target_s:
        t0 = time.perf_counter()
        orc.sk(x, M, lo, hi)
        total += time.perf_counter() - t0
        reps += 1
    msps = nchan_s * npol * cfg["ndat"] * reps / total / 1e6
    return {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
            "kind": "port",
            "sample": (f"{nchan_s} channels x {cfg['ndat']} samples x {npol} pol x {reps} "
                       f"through the oracle SK restatement (OpenMP over blocks), {total:.1f} s")}


def run_b200_sk(args, cfg, world, rank, local):
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = b2.Context(local)
    nchan, npol, ndat, M = cfg["nchan"], cfg["npol"], cfg["ndat"], cfg["M"]
    lo, hi = b2.sk_limits(M, 1, cfg["std_devs"], npol)
    x = make_sk_block(cfg, 4321 + rank, device)
    npart = ndat // M
    out = torch.empty_like(x)
    sums = torch.empty(npart * nchan * npol * 2, dtype=torch.float32, device=device)
    counts = torch.empty(npart * nchan, dtype=torch.int32, device=device)
    mask = torch.empty(npart * nchan, dtype=torch.uint8, device=device)
    zapped = torch.zeros(1, dtype=torch.int64, device=device)
    samples_per_step = nchan * npol * ndat
    inplace = args.sk_inplace

    def step(src, dst):
        ctx.sk(src, ndat, ndat, nchan, npol, M, lo, hi, dst, ndat, sums, counts, mask, zapped)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    # an in-place step masks its own input; later steps then see masked data,
    # which reads the same bytes (the input exceeds L2 many times per step)
    for _ in range(args.warmup):
        step(x, x if inplace else out)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record()
    for i in range(args.steps):
        step(x, x if inplace else out)
        evs[i + 1].record()
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = evs[0].elapsed_time(evs[-1])
    ms_max = max_over_ranks(ms, world)
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6
    per_launch = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    zap_frac = float(mask.float().mean().item())

    # ---- end to end: pinned host voltages in, masked voltages and mask out --
    numa = {}
    with near_gpu_memory(local, numa):
        hx = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
        hx.copy_(x)
        hout = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
        hout.zero_()
        hmask = torch.empty(mask.shape, dtype=mask.dtype, pin_memory=True)
        hmask.zero_()
    for _ in range(max(1, args.warmup)):
        x.copy_(hx, non_blocking=True)
        step(x, x if inplace else out)
        hout.copy_(x if inplace else out, non_blocking=True)
        hmask.copy_(mask, non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        x.copy_(hx, non_blocking=True)
        step(x, x if inplace else out)
        hout.copy_(x if inplace else out, non_blocking=True)
        hmask.copy_(mask, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), 1e3 * wall), world)
    e2e = samples_per_step * args.steps * world / (e2e_ms / 1e3) / 1e6

    hbm_peak, _, peak_src = measured_peaks()
    bps = sk_bytes_per_sample(inplace)
    avg_s = statistics.mean(per_launch) / 1e3
    achieved = bps * samples_per_step / avg_s / 1e9
    tb = ncu_traffic(f"{args.config}:sk")
    line = {
        "metric": "complex Msamples/s spectral kurtosis", "value": round(value, 3),
        "unit": "complex Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic (seeded Gaussian complex voltages + injected RFI)",
        "config": {"workload": cfg["workload"], "M": M, "thresholds": [float(lo), float(hi)],
                   "in_place": inplace, "zapped_fraction": round(zap_frac, 5),
                   "l2": f"input {x.numel() * 4 >> 30} GiB per step, larger than L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_sk", "achieved": round(achieved, 2),
                     "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                     "traffic": tb * samples_per_step if tb else None,
                     "peak_source": peak_src, "bytes_per_sample": bps},
        "e2e": {"value": round(e2e, 3), "unit": "complex Msamples/s",
                "h2d_bytes_per_step": int(hx.numel() * 4),
                "d2h_bytes_per_step": int(hout.numel() * 4 + hmask.numel())},
    }
    if not args.no_proposer:
        line["proposer"] = sk_proposer(args, cfg, b2, ctx, device, lo, hi, rank, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sk(cfg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def sk_proposer(args, cfg, b2, ctx, device, lo, hi, rank, world):
    """The learned RFI-mask proposer in front of SpectralKurtosis: trained on
    the SK masks of one RFI-injected block, scored against SK on another (miss =
    SK zaps, proposer keeps; false zap = SK keeps, proposer zaps), alone and
    with the SK fallback below the confidence threshold; its throughput is
    that of the feature + tensor-core inference kernels on the SK sums."""
    import torch
    nchan, npol, ndat, M = cfg["nchan"], cfg["npol"], cfg["ndat"], cfg["M"]
    npart = ndat // M
    conf = 0.9

    def sk_of(seed):
        x = make_sk_block(cfg, seed, device)
        sums = torch.empty(npart * nchan * npol * 2, dtype=torch.float32, device=device)
        counts = torch.empty(npart * nchan, dtype=torch.int32, device=device)
        mask = torch.empty(npart * nchan, dtype=torch.uint8, device=device)
        ctx.sk(x, ndat, ndat, nchan, npol, M, lo, hi, x, ndat, sums, counts, mask)
        torch.cuda.synchronize()
        del x
        torch.cuda.empty_cache()
        return sums, counts, mask

    pr = b2.RfiProposer(ctx, nchan, M, max_npart=npart, max_batch_blocks=32, seed=7)
    sums, counts, mask = sk_of(9001 + rank)
    pr.features(sums, npart, npol, counts)
    t0 = time.perf_counter()
    loss0 = pr.train(mask, 20, batch_blocks=32, lr=3e-3)
    loss1 = pr.train(mask, args.proposer_steps, batch_blocks=32, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    sums2, counts2, mask2 = sk_of(9101 + rank)
    alone = torch.empty(npart * nchan, dtype=torch.uint8, device=device)
    fb = torch.empty_like(alone)
    prob = torch.empty(npart * nchan, dtype=torch.float32, device=device)
    # timed: features from the sums + inference with the fallback
    for _ in range(3):
        pr.features(sums2, npart, npol, counts2)
        pr.infer(fb, prob, mask2, confidence=conf)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        pr.features(sums2, npart, npol, counts2)
        pr.infer(fb, prob, mask2, confidence=conf, count=False)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
    nfall = pr.infer(fb, prob, mask2, confidence=conf)
    pr.infer(alone, None, None, confidence=0.5)
    sk = mask2.bool()
    a, f = alone.bool(), fb.bool()
    nsk, nkeep = int(sk.sum()), int((~sk).sum())

    def rates(m):
        return {"miss_rate": round(int((sk & ~m).sum()) / max(nsk, 1), 5),
                "false_zap_rate": round(int((~sk & m).sum()) / max(nkeep, 1), 6)}

    pr.close()
    return {"train": {"steps": 20 + args.proposer_steps, "batch_blocks": 32,
                      "loss_first": round(loss0, 5), "loss_last": round(loss1, 5),
                      "seconds": round(train_s, 2)},
            "sk_zapped_cells": nsk, "cells": int(sk.numel()),
            "alone": rates(a), "with_sk_fallback": dict(rates(f), confidence=conf,
                                                          fallback_cells=int(nfall)),
            "ms_per_block": round(ms, 4),
            "value": round(nchan * npol * ndat / (ms / 1e3) / 1e6, 1),
            "unit": "complex Msamples/s (features + inference on the SK sums)",
            "params": 3937, "weights": "BF16 on the tensor cores, FP32 master copy"}


# ---------------------------------------------------------------------------
# InverseFilterbank workload
# ---------------------------------------------------------------------------

def ifb_cfg_dict(cfg):
    return dict(input_nchan=cfg["nin"], output_nchan=1, pfb_nchan=cfg["nin"], npol=cfg["npol"],
                input_fft_length=cfg["lin"], os_num=4, os_den=3,
                output_discard_pos=cfg["disc"], output_discard_neg=cfg["disc"], pfb_dc_chan=1,
                pfb_all_chan=1, dual_sideband=1)


def run_reference_ifb(args, cfg, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = os.cpu_count() or 1
    c = ifb_cfg_dict(cfg)
    keep, lout, ipos, ineg, in_step, out_step = orc.ifb_sizes(c)
    nparts = 4
    ndat = nparts * in_step + ipos + ineg
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((cfg["nin"], cfg["npol"], ndat)) * 100 +
         1j * rng.standard_normal((cfg["nin"], cfg["npol"], ndat)) * 100).astype(np.complex64)

    def step():
        t0 = time.perf_counter()
        orc.inverse_filterbank(x, c)
        return time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    total = sum(step() for _ in range(args.steps))
    msps = cfg["nin"] * cfg["npol"] * nparts * in_step * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s inverse filterbank",
        "value": round(msps, 3), "unit": "complex Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian complex voltages)",
        "config": {"workload": cfg["workload"], "sample_parts_per_step": nparts},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": 1,
                         "kind": "port",
                         "sample": (f"{nparts} parts of {cfg['nin']} fine channels x "
                                    f"{cfg['npol']} pol through the oracle restatement of "
                                    "InverseFilterbankEngineCPU (single thread, FP32)")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200_ifb(args, cfg, world, rank, local):
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = b2.Context(local)
    ifb = b2.InverseFilterbank(ctx, cfg["nin"], 1, cfg["nin"], cfg["npol"], cfg["lin"],
                               os=(4, 3), output_discard=(cfg["disc"], cfg["disc"]))
    info = ifb.info
    in_step, out_step = info["in_step"], info["out_step"]
    disc_in = info["in_discard_pos"] + info["in_discard_neg"]
    ndat = cfg["ndat"]
    npart = ifb.npart(ndat)
    # int16 TFPD voltages (seeded Gaussian, sigma 100), generated on the GPU
    t_gen = time.perf_counter()
    raw = make_pfb_block(cfg, 99 + rank, device)
    t_gen = time.perf_counter() - t_gen
    out = torch.empty((1, cfg["npol"], npart * out_step, 2), dtype=torch.float32, device=device)
    samples_per_step = cfg["nin"] * cfg["npol"] * npart * in_step

    def step():
        ifb.perform(raw, ndat, out, npart * out_step, input_kind=b2.INT16_TFPD)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record()
    for i in range(args.steps):
        step()
        evs[i + 1].record()
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = evs[0].elapsed_time(evs[-1])
    ms_max = max_over_ranks(ms, world)
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6
    ifb.status()
    hbm_peak, _, peak_src = measured_peaks()
    # algorithmic bytes per step: int16 input once (4 B per complex sample per pol)
    # and the complex-float output once
    alg = raw.numel() * 2 + out.numel() * 4
    achieved = alg / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": "complex Msamples/s inverse filterbank", "value": round(value, 3),
        "unit": "complex Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": ("synthetic: one periodic second of 800 MHz complex baseband (seeded Gaussian "
                 "noise + a 1.6 ms pulsar, 3 % duty, at DM 1000 by an FP64 inverse chirp) "
                 "channelised by a 12-tap-per-channel Kaiser-windowed 4/3-oversampled PFB "
                 f"into 256 int16 channels (generated on the GPU in {t_gen:.1f} s)"),
        "config": {"workload": cfg["workload"], "npart": npart, "input_fft_length": cfg["lin"],
                   "output_fft_length": info["lout"], "fft_split": [info["n1"], info["n2"]],
                   "parts_per_batch": info["max_batch"],
                   "l2": f"input {raw.numel() * 2 >> 20} MiB per step, larger than L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "inverse filterbank (3 kernels)",
                     "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": None,
                     "peak_source": peak_src,
                     "note": "algorithmic bytes: int16 in + complex-float out, once"},
        "e2e": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ifb.close()
    ctx.close()


# ---------------------------------------------------------------------------
# Filterbank with the dedispersion inside it ("During")
# ---------------------------------------------------------------------------

def fbd_sizes(cfg, b2):
    half = b2.smearing_samples(cfg["cf"], cfg["bw"], cfg["dm"], cfg["nsub"], 1)
    return half, cfg["freq_res"] - 2 * half


def run_reference_fbd(args, cfg, world, rank):
    if rank != 0:
        return
    import dspsr_b200 as b2
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    half, nkeep = fbd_sizes(cfg, b2)
    nsub, fr = cfg["nsub"], cfg["freq_res"]
    resp = orc.dedispersion_response_during(cfg["cf"], cfg["bw"], cfg["dm"], nsub, fr, nsub * fr)
    nparts = 2
    ndat = nparts * nsub * nkeep + 2 * half * nsub
    rng = np.random.default_rng(5)
    lut, _ = b2.bittable8()
    raw = rng.integers(0, 256, (cfg["npol"], ndat, 2), dtype=np.uint8)
    nbin = cfg["nbin"]
    pps = (nsub / (cfg["bw"] * 1e6)) / cfg["period"]

    def step():
        t0 = time.perf_counter()
        x = lut[raw].view(np.complex64)[None, :, :, 0]
        v = orc.filterbank_during(x, nsub, fr, (half, half), resp)
        det = orc.detect(v, cfg["state"])
        plan = orc.fold_binplan(0.1, pps, v.shape[2], nbin)
        orc.fold_accumulate(det, plan, nbin)
        return time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    total = sum(step() for _ in range(args.steps))
    msps = cfg["npol"] * nparts * nsub * nkeep * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s filterbank-with-dedispersion -> fold",
        "value": round(msps, 3), "unit": "complex Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform int8 voltages)",
        "config": {"workload": cfg["workload"], "sample_parts_per_step": nparts},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": 1,
                         "kind": "port",
                         "sample": (f"{nparts} parts of {nsub * fr} samples x {cfg['npol']} pol "
                                    "through the oracle restatement of FilterbankEngineCPU with "
                                    "a response, Detection and Fold (single thread, FP32)")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200_fbd(args, cfg, world, rank, local):
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = b2.Context(local)
    half, nkeep = fbd_sizes(cfg, b2)
    nsub, fr, npol = cfg["nsub"], cfg["freq_res"], cfg["npol"]
    fbd = b2.FilterbankDuring(ctx, 1, npol, nsub, fr, (half, half))
    fbd.set_dedispersion(cfg["cf"], cfg["bw"], cfg["dm"])
    ndat = cfg["ndat"]
    npart = fbd.npart(ndat)
    span = npart * nkeep
    nout = b2.NOUT[cfg["state"]]
    fold = b2.Fold(ctx, cfg["nbin"], nsub, nout)
    lut, _ = b2.bittable8()
    gen = torch.Generator(device=device)
    gen.manual_seed(17 + rank)
    # two distinct int8 TFPD blocks, each larger than L2
    raws = [torch.randint(0, 256, (ndat * npol * 2,), dtype=torch.uint8, device=device,
                          generator=gen) for _ in range(2)]
    rate = cfg["bw"] * 1e6 / nsub
    pps = (1.0 / rate) / cfg["period"]
    used = npol * npart * nsub * nkeep

    def step(i):
        fold.set_bins(0.1 + 1e-3 * i, pps, span)
        fbd.perform_fold(raws[i % 2], ndat, fold, cfg["state"], input_kind=b2.INT8_TFPD, lut=lut)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record()
    for i in range(args.steps):
        step(i)
        evs[i + 1].record()
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = evs[0].elapsed_time(evs[-1])
    ms_max = max_over_ranks(ms, world)
    value = used * args.steps * world / (ms_max / 1e3) / 1e6
    hbm_peak, _, peak_src = measured_peaks()
    alg = ndat * npol * 2
    achieved = alg / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": "complex Msamples/s filterbank-with-dedispersion -> fold",
        "value": round(value, 3), "unit": "complex Msamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform int8 voltages)",
        "config": {"workload": cfg["workload"], "npart": npart, "nkeep": nkeep,
                   "nfilt": 2 * half, "fft_split": [fbd.info["n1"], 8192],
                   "parts_per_batch": fbd.info["max_batch"],
                   "l2": (f"two distinct {ndat * npol * 2 >> 20} MiB input blocks alternate"
                          + (", each larger than L2" if ndat * npol * 2 > (126 << 20)
                             else " (profiling size: they fit in L2)")),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "filterbank with response (3 kernels)",
                     "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": None,
                     "peak_source": peak_src,
                     "note": "algorithmic bytes: the int8 input once; FP32-ALU bound like c2"},
        "e2e": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    fold.close()
    fbd.close()
    ctx.close()


# ---------------------------------------------------------------------------
# Multi-stream workload: many independent beams / DM trials at once
# ---------------------------------------------------------------------------

def c3_streams(cfg, b2):
    """The seeded stream list: DM ~ U[10, 2000], bandwidth in {16, 32, 64,
    128} MHz, channels in {1, 8, 32}, redrawn until the reference's minimum
    FFT fits 2^18; FFT length by optimal_fft_length within [2^12, 2^18];
    nbin in {512, 1024, 2048, 4096}; period in [2, 500] ms."""
    rng = np.random.default_rng(cfg["seed"])
    out = []
    while len(out) < cfg["nstream"]:
        dm = float(rng.uniform(10.0, 2000.0))
        bw = float(rng.choice([16.0, 32.0, 64.0, 128.0]))
        nchan = int(rng.choice([1, 8, 32]))
        pos = b2.smearing_samples(cfg["cf"], bw, dm, nchan, 1)
        neg = b2.smearing_samples(cfg["cf"], bw, dm, nchan, -1)
        nmin = b2.minimum_ndat(pos, neg)
        if nmin > (1 << 18):
            continue
        nfft = b2.optimal_fft_length(pos + neg, 1 << 18)
        nfft = int(min(max(nfft if nfft > 0 else nmin, nmin, 1 << 12), 1 << 18))
        ndat = cfg["samples"] // nchan
        if ndat < 2 * nfft:
            continue
        out.append(dict(dm=dm, bw=bw, nchan=nchan, pos=pos, neg=neg, nfft=nfft, ndat=ndat,
                        nbin=int(rng.choice([512, 1024, 2048, 4096])),
                        period=float(rng.uniform(0.002, 0.5))))
    return out


def c3_cpu_sample(cfg, b2, orc, nstream=4):
    """Bounded CPU sample: two FFT parts of each of the first streams through
    the oracle chain unpack -> convolve -> detect -> fold."""
    streams = c3_streams(cfg, b2)[:nstream]
    lut, _ = orc.bittable8(0.0308)
    work = []
    for k, s in enumerate(streams):
        nk = s["nfft"] - s["pos"] - s["neg"]
        ndat = s["nfft"] + nk
        from dspsr_b200 import synth
        raw = synth.noise_block(ndat, s["nchan"], 2, 10.0, 10 + k)
        h = orc.dedispersion_response(cfg["cf"], s["bw"], s["dm"], s["nchan"], s["nfft"],
                                      input_nchan=s["nchan"])
        work.append((s, raw, ndat, h))

    def run(threads):
        t0 = time.perf_counter()
        n = 0
        for s, raw, ndat, h in work:
            x = orc.unpack8(raw, ndat, s["nchan"], 2, 2, lut)
            x = x.view(np.complex64).reshape(s["nchan"], 2, ndat)
            z = orc.convolve(x, h, s["nfft"], s["pos"], s["neg"], nthreads=threads)
            d = orc.detect(z, 0)
            plan = orc.fold_binplan(0.1, 1e-7, z.shape[2], s["nbin"])
            orc.fold_accumulate(d, plan, s["nbin"])
            n += ndat * s["nchan"] * 2
        return time.perf_counter() - t0, n
    return run, len(work)


def run_reference_c3(args, cfg, world, rank):
    if rank != 0:
        return
    import dspsr_b200 as b2
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = os.cpu_count() or 1
    run, ns = c3_cpu_sample(cfg, b2, orc)
    for _ in range(args.warmup):
        run(threads)
    total, n = 0.0, 0
    for _ in range(args.steps):
        t, k = run(threads)
        total += t
        n += k
    msps = n / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s unpack->fold, many streams",
        "value": round(msps, 3), "unit": "complex Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian noise, int8)",
        "config": {"workload": cfg["workload"], "sample_streams": ns},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
                         "kind": "port",
                         "sample": (f"two FFT parts of each of the first {ns} streams through "
                                    "the oracle chain (unpack, overlap-save, detect, fold)")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200_c3(args, cfg, world, rank, local):
    import math
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    streams = c3_streams(cfg, b2)
    lut, _ = b2.bittable8()
    gen = torch.Generator(device=device)
    gen.manual_seed(777 + rank)
    nblk = 2
    for s in streams:
        nbytes = s["ndat"] * s["nchan"] * 2 * 2
        s["blocks"] = [torch.randint(-40, 40, (nbytes,), generator=gen, device=device,
                                     dtype=torch.int8).view(torch.uint8) for _ in range(nblk)]
        s["tstream"] = torch.cuda.Stream(device=device)
        s["ctx"] = b2.Context(local, s["tstream"].cuda_stream)

    def make_pipe(s, plan):
        scratch, row, fft = plan
        c = b2.make_config(cfg["cf"], s["bw"], s["dm"], s["nchan"], 2, s["nfft"], s["pos"],
                           s["neg"], s["nbin"], s["period"], state=b2.INTENSITY, lut=lut,
                           start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, scratch_bytes=scratch,
                           row_length=row, fft_precision=fft)
        return b2.Pipeline(s["ctx"], c)

    def plans(nfft):
        """The autotuner's candidates for one FFT length: the four-step split
        (8192- or 4096-point rows, i.e. nfft/8192 or nfft/4096 columns), the
        rows' arithmetic (FP32 CUDA cores, or the three-term split-BF16
        tensor-core DFT stages, which hold the FP32 error bar) and the
        scratch budget of the FFT batches."""
        out = []
        for sc in (64 << 20, 256 << 20, 1024 << 20):
            if nfft <= 8192:
                out.append((sc, 0, b2.FFT_FP32))
                if nfft == 8192:
                    out.append((sc, 4096, b2.FFT_FP32))
                continue
            out.append((sc, 8192, b2.FFT_FP32))
            if args.c3_tensor:
                out.append((sc, 8192, b2.FFT_BF16X3))
            if nfft <= 131072:
                out.append((sc, 4096, b2.FFT_FP32))
        return out

    # autotuner: per shape class (FFT length, channels) the plan that runs one
    # block fastest, timed alone on the stream
    tuned = {}
    tuned_ms = {}
    t_tune = time.perf_counter()
    for s in streams:
        key = (s["nfft"], s["nchan"])
        if key not in tuned:
            best = None
            for plan in plans(s["nfft"]):
                pl = make_pipe(s, plan)
                for w in range(2):
                    pl.run(s["blocks"][w % nblk], s["ndat"])
                st = s["tstream"]
                times = []
                for rep in range(3):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    pl.run(s["blocks"][rep % nblk], s["ndat"])
                    e1.record(st)
                    e1.synchronize()
                    times.append(e0.elapsed_time(e1))
                ms = statistics.median(times)
                pl.close()
                if best is None or ms < best[0]:
                    best = (ms, plan)
            tuned[key] = best[1]
            tuned_ms[key] = best[0]
        s["plan"] = tuned[key]
        s["scratch"] = tuned[key][0]
        s["pipe"] = make_pipe(s, s["plan"])
    t_tune = time.perf_counter() - t_tune
    torch.cuda.synchronize()
    samples_per_step = sum(s["ndat"] * s["nchan"] * 2 for s in streams)

    def step_sequential(i, default):
        # every pipeline's kernels fill the GPU: one stream after another
        for s in streams:
            s["tstream"].wait_stream(default)
            s["pipe"].run(s["blocks"][i % nblk], s["ndat"])
            default.wait_stream(s["tstream"])

    def step_concurrent(i, default):
        for s in streams:
            s["tstream"].wait_stream(default)
        for s in streams:
            s["pipe"].run(s["blocks"][i % nblk], s["ndat"])
        for s in streams:
            default.wait_stream(s["tstream"])

    default = torch.cuda.current_stream()
    # the schedule is tuned too: two untimed steps of each, the faster kept
    def trial(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(default)
        for i in range(2):
            fn(i, default)
        b.record(default)
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    trial(step_sequential)
    t_seq, t_conc = trial(step_sequential), trial(step_concurrent)
    conc_first = t_conc < t_seq
    # every rank runs the same schedule (rank 0's choice)
    if world > 1:
        import torch.distributed as dist
        flag = torch.tensor([1 if conc_first else 0], device=device)
        dist.broadcast(flag, 0)
        conc_first = bool(flag.item())
    step_fn, other_fn = ((step_concurrent, step_sequential) if conc_first
                         else (step_sequential, step_concurrent))
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for i in range(args.warmup):
        step_fn(i, default)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(default)
    for i in range(args.steps):
        step_fn(args.warmup + i, default)
    ev1.record(default)
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6

    # for comparison: the other schedule, same number of steps
    ev0.record(default)
    for i in range(args.steps):
        other_fn(i, default)
    ev1.record(default)
    torch.cuda.synchronize()
    ms_other = ev0.elapsed_time(ev1)
    other_value = samples_per_step * args.steps / (ms_other / 1e3) / 1e6

    # end to end: pinned host blocks uploaded by each stream's pipeline
    numa = {}
    with near_gpu_memory(local, numa):
        host = [s["blocks"][0].cpu().pin_memory() for s in streams]
    for s, h in zip(streams, host):
        s["pipe"].run_host(h, s["ndat"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(default)
    for i in range(args.steps):
        for s in streams:
            s["tstream"].wait_stream(default)
        for s, h in zip(streams, host):
            s["pipe"].run_host(h, s["ndat"])
        for s in streams:
            default.wait_stream(s["tstream"])
        profs = [s["pipe"].get_profiles() for s in streams]
    e1.record(default)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), 1e3 * wall), world)
    e2e = samples_per_step * args.steps * world / (e2e_ms / 1e3) / 1e6
    d2h = sum(p.nbytes + h_.nbytes for p, h_ in profs)

    flops = 0.0
    for s in streams:
        nk = s["nfft"] - s["pos"] - s["neg"]
        fps = (s["nfft"] / nk) * (2 * 5 * math.log2(s["nfft"]) + 6) + 5
        flops += fps * s["ndat"] * s["nchan"] * 2
    fp32_tflops = flops * args.steps / (ms / 1e3) / 1e12
    fp32_peak = 148 * 128 * 2 * (clk["sm_mhz"] or 1965.0) * 1e6 / 1e12
    hbm_peak, _, peak_src = measured_peaks()
    alg_gbs = 2.0 * samples_per_step * args.steps / (ms / 1e3) / 1e9
    shapes = sorted({(s["nfft"], s["nchan"]) for s in streams})
    line = {
        "metric": "complex Msamples/s unpack->fold, many streams", "value": round(value, 3),
        "unit": "complex Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian noise, int8)",
        "config": {"workload": cfg["workload"], "streams": len(streams),
                   "shape_classes": [list(x) for x in shapes],
                   "tuned": {f"{k[0]}x{k[1]}": {"scratch_mib": v[0] >> 20,
                                                  "row_length": v[1] or min(k[0], 8192),
                                                  "rows": "bf16x3 tensor" if v[2] == 3 else "fp32",
                                                  "block_ms": round(tuned_ms[k], 3),
                                                  "streams": sum(1 for s in streams
                                                                 if (s["nfft"], s["nchan"]) == k)}
                             for k, v in tuned.items()},
                   "autotune_s": round(t_tune, 2),
                   "schedule": ("the 48 pipelines at once, each on its own CUDA stream"
                                if conc_first else "pipelines one after another on the device"),
                   "schedule_trial_ms": {"sequential": round(t_seq / 2, 3),
                                         "concurrent": round(t_conc / 2, 3)},
                   "other_schedule_value": round(other_value, 3),
                   "l2": f"{nblk} distinct blocks per stream ({samples_per_step * 2 >> 20} MiB "
                         "per step), larger than L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": round(alg_gbs, 2),
                     "peak": hbm_peak, "unit": "GB/s", "frac": round(alg_gbs / hbm_peak, 4),
                     "traffic": None, "peak_source": peak_src,
                     "note": "path is FP32-ALU bound (2 B/sample in); see roofline_fp32"},
        "roofline_fp32": {"achieved": round(fp32_tflops, 3), "unit": "TFLOP/s",
                          "peak": round(fp32_peak, 1), "frac": round(fp32_tflops / fp32_peak, 4)},
        "e2e": {"value": round(e2e, 3), "unit": "complex Msamples/s",
                "h2d_bytes_per_step": int(sum(h.numel() for h in host)),
                "d2h_bytes_per_step": int(d2h), **numa},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        run, ns = c3_cpu_sample(cfg, b2, orc)
        threads = os.cpu_count() or 1
        run(threads)
        total, n, reps = 0.0, 0, 0
        while total < 12.0:
            t, k = run(threads)
            total += t
            n += k
            reps += 1
        line["cpu_baseline"] = {"value": round(n / total / 1e6, 3), "unit": "complex Msamples/s",
                                "cores": threads, "kind": "port",
                                "sample": (f"two FFT parts of each of the first {ns} streams x "
                                           f"{reps} through the oracle chain, {total:.1f} s")}
        # parity: the first stream, and the first four-step stream of several
        # channels, one block each through a fresh pipeline with the tuned
        # plan, against the oracle chain
        # the first stream and the first of another shape class (the
        # single-kernel path when there is one)
        first = (streams[0]["nfft"], streams[0]["nchan"])
        others = [i for i, st in enumerate(streams) if (st["nfft"], st["nchan"]) != first]
        fused = [i for i in others if streams[i]["nfft"] <= 8192]
        picks = [0] + (fused or others)[:1]
        line["parity"] = [c3_parity(cfg, b2, orc, streams[i], make_pipe, lut) for i in picks]
    if rank == 0:
        print(json.dumps(line), flush=True)
    for s in streams:
        s["pipe"].close()
        s["ctx"].close()


def c3_parity(cfg, b2, orc, s, make_pipe, lut):
    """One block of stream s through a fresh pipeline (its tuned plan) and
    through the oracle chain unpack -> overlap-save -> intensity -> fold
    (Convolution.C:724-803, Fold.C:790-837): hits bit-exact, profiles within
    1e-5 of each bin."""
    pl = make_pipe(s, s["plan"])
    nout = pl.run(s["blocks"][0], s["ndat"])
    prof, hits = pl.get_profiles()
    pl.close()
    raw = s["blocks"][0].cpu().numpy()
    x = orc.unpack8(raw, s["ndat"], s["nchan"], 2, 2, np.asarray(lut, np.float32))
    x = x.view(np.complex64).reshape(s["nchan"], 2, s["ndat"])
    h = orc.dedispersion_response(cfg["cf"], s["bw"], s["dm"], s["nchan"], s["nfft"],
                                  input_nchan=s["nchan"], mode=0)
    y = orc.convolve(x, h, s["nfft"], s["pos"], s["neg"], nthreads=os.cpu_count() or 1)
    d = orc.detect(y, 0)
    rate = abs(s["bw"]) / s["nchan"] * 1e6
    phi = orc.fold_phi(START_MJD, EPOCH_MJD, s["pos"], rate, s["period"])
    plan = orc.fold_binplan(phi, (1.0 / rate) / s["period"], y.shape[2], s["nbin"])
    rprof, rhits = orc.fold_accumulate(d, plan, s["nbin"])
    hit = rhits > 0
    err = float(np.max(np.abs(prof.astype(np.float64) - rprof)[..., hit]
                       / np.abs(rprof.astype(np.float64))[..., hit]))
    return {"stream": {k: s[k] for k in ("nchan", "nfft", "bw", "dm", "nbin")},
            "plan": {"row_length": s["plan"][1] or min(s["nfft"], 8192),
                     "rows": "bf16x3 tensor" if s["plan"][2] == 3 else "fp32"},
            "samples_folded": int(nout), "oracle_samples": int(y.shape[2]),
            "hits_bit_exact": bool(np.array_equal(hits, rhits)),
            "max_profile_rel_err": err,
            "pass": bool(np.array_equal(hits, rhits)) and err < 1e-5 and nout == y.shape[2]}


def c5_plan(cfg, b2):
    """Re-channelised dedispersion plan of the C5 chain (per output channel)."""
    nc = cfg["fb"]
    pos = b2.smearing_samples(cfg["cf"], cfg["bw"], cfg["dm"], nc, 1)
    neg = b2.smearing_samples(cfg["cf"], cfg["bw"], cfg["dm"], nc, -1)
    nmin = b2.minimum_ndat(pos, neg)
    nfft = b2.optimal_fft_length(pos + neg, 1 << 16)
    nfft = int(min(max(nfft if nfft > 0 else nmin, nmin, 8192), 1 << 16))
    return pos, neg, nfft


def run_reference_c5(args, cfg, world, rank):
    """The chain on the CPU for a bounded sample: inverse filterbank (oracle,
    all threads over parts) -> 1024-channel filterbank -> overlap-save ->
    Stokes -> fold."""
    if rank != 0:
        return
    import dspsr_b200 as b2
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = os.cpu_count() or 1
    c = ifb_cfg_dict(cfg)
    keep, lout, ipos, ineg, in_step, out_step = orc.ifb_sizes(c)
    pos, neg, nfft = c5_plan(cfg, b2)
    nc = cfg["fb"]
    need = (nfft + 16) * nc                     # one FFT part per channel
    nparts = -(-need // out_step)
    ndat = nparts * in_step + ipos + ineg
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((cfg["nin"], cfg["npol"], ndat)) * 100 +
         1j * rng.standard_normal((cfg["nin"], cfg["npol"], ndat)) * 100).astype(np.complex64)
    freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nc, swap=True, dc_centred=True)
    h = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], nfft, mode=0)

    def step():
        t0 = time.perf_counter()
        w = orc.inverse_filterbank(x, c)
        n = (w.shape[2] // nc) * nc
        y = orc.filterbank(w[:, :, :n], nc)
        z = orc.convolve(y, h, nfft, pos, neg, nthreads=threads)
        d = orc.detect(z, 3)
        plan = orc.fold_binplan(0.2, 1e-6, z.shape[2], cfg["nbin"])
        orc.fold_accumulate(d, plan, cfg["nbin"])
        return time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    total = sum(step() for _ in range(args.steps))
    msps = cfg["nin"] * cfg["npol"] * nparts * in_step * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "complex Msamples/s inverse filterbank->fold",
        "value": round(msps, 3), "unit": "complex Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian complex voltages)",
        "config": {"workload": cfg["workload"], "sample_ifb_parts_per_step": nparts},
        "cpu_baseline": {"value": round(msps, 3), "unit": "complex Msamples/s", "cores": threads,
                         "kind": "port",
                         "sample": (f"{nparts} inverse-filterbank parts of {cfg['nin']} "
                                    f"channels x {cfg['npol']} pol (one FFT part per output "
                                    "channel) through the oracle chain")},
        "e2e": {"value": round(msps, 3), "unit": "complex Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def c5_parity(cfg, b2, raw, pos, neg, nfft):
    """A bounded sample of C5's input (the first inverse-filterbank parts,
    enough for one FFT part of every re-channelised output channel) through
    fresh GPU objects and through the oracle chain: InverseFilterbank
    (InverseFilterbankEngineCPU.C:46-792) -> 1024-channel filterbank ->
    overlap-save -> Stokes -> fold.  Hits bit-exact, profiles within 5e-5 of
    Stokes I per bin."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.lib()
    c = ifb_cfg_dict(cfg)
    keep, lout, ipos, ineg, in_step, out_step = orc.ifb_sizes(c)
    nc = cfg["fb"]
    nparts = -(-((nfft + 16) * nc) // out_step)
    ndat = nparts * in_step + ipos + ineg
    nin, npol = cfg["nin"], cfg["npol"]
    sample = raw[:ndat * nin * npol * 2].clone()
    ctx = b2.Context(torch.cuda.current_device())
    ifb = b2.InverseFilterbank(ctx, nin, 1, nin, npol, cfg["lin"], os=(4, 3),
                               output_discard=(cfg["disc"], cfg["disc"]))
    np_ = ifb.npart(ndat)
    nwide = np_ * ifb.info["out_step"]
    wide = torch.empty((1, npol, nwide, 2), dtype=torch.float32, device=sample.device)
    ifb.perform(sample, ndat, wide, nwide, input_kind=b2.INT16_TFPD)
    pcfg = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], 1, npol, nfft, pos, neg, cfg["nbin"],
                          cfg["period"], state=b2.STOKES, input_kind=b2.FLOAT_FPT,
                          start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, filterbank_nchan=nc)
    pipe = b2.Pipeline(ctx, pcfg)
    nout = pipe.run(wide, nwide, nwide)
    prof, hits = pipe.get_profiles()
    pipe.close()
    ifb.close()
    ctx.close()
    t0 = time.perf_counter()
    h16 = sample.cpu().numpy()
    x = orc.unpack16(h16, ndat, nin, npol, 2, False).view(np.complex64).reshape(nin, npol, ndat)
    w = orc.inverse_filterbank(x, c)
    n = (w.shape[2] // nc) * nc
    y = orc.filterbank(w[:, :, :n], nc)
    freqs = orc.channel_centres(cfg["cf"], cfg["bw"], nc, swap=True, dc_centred=True)
    hresp = orc.dedispersion_response_channels(freqs, cfg["bw"], cfg["dm"], nfft, mode=0)
    z = orc.convolve(y, hresp, nfft, pos, neg, nthreads=os.cpu_count() or 1)
    d = orc.detect(z, 3)
    rate = abs(cfg["bw"]) / nc * 1e6
    phi = orc.fold_phi(START_MJD, EPOCH_MJD, pos, rate, cfg["period"])
    plan = orc.fold_binplan(phi, (1.0 / rate) / cfg["period"], z.shape[2], cfg["nbin"])
    rprof, rhits = orc.fold_accumulate(d, plan, cfg["nbin"])
    rprof = rprof.astype(np.float64)
    scale = np.broadcast_to(rprof[:, 0:1], rprof.shape)
    hit = rhits > 0
    err = float(np.max(np.abs(prof.astype(np.float64) - rprof)[..., hit] / scale[..., hit]))
    ok = bool(np.array_equal(hits, rhits)) and err < 5e-5 and nout == z.shape[2]
    return {"sample": f"{np_} inverse-filterbank parts ({ndat} samples per PFB channel)",
            "samples_folded": int(nout), "oracle_samples": int(z.shape[2]),
            "hits_bit_exact": bool(np.array_equal(hits, rhits)), "max_profile_rel_err": err,
            "rtol": 5e-5, "pass": ok, "oracle_s": round(time.perf_counter() - t0, 1)}


def make_pfb_block(cfg, seed, device, taps=12, beta=8.0, duty=0.03, snr=10.0):
    """nin channels of a 4/3-oversampled polyphase filterbank of one second
    of complex baseband at |bw| MHz: seeded Gaussian noise plus a pulsar of
    cfg's period (noise switched on for `duty` of each turn) dispersed at
    cfg's DM by an FP64 inverse chirp over the whole second (the second holds
    a whole number of turns, so the circular chirp is exact).  The prototype
    filter is a Kaiser-windowed sinc of taps * nin points with its cut-off at
    half the channel spacing (pfb_channelise).  Returns int16 TFPD
    [ndat][nin][npol][2], scaled to a noise sigma of about 300.  torch is the
    synthesis tool here (it is not on the product path)."""
    import torch
    from dspsr_b200 import synth
    nin, npol, ndat = cfg["nin"], cfg["npol"], cfg["ndat"]
    L = taps * nin
    nw = int(round(abs(cfg["bw"]) * 1e6))          # one second of wideband samples
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    k = torch.arange(L, device=device, dtype=torch.float64) - (L - 1) / 2
    h = torch.sinc(k / nin) * torch.kaiser_window(L, periodic=False, beta=beta,
                                                   dtype=torch.float64, device=device)
    h = (h / h.sum()).to(torch.float32)
    out = torch.empty((ndat, nin, npol, 2), dtype=torch.int16, device=device)
    rate = abs(cfg["bw"]) * 1e6
    d = cfg["dm"] / synth.DM_DISPERSION * 1e6
    cf, bw = cfg["cf"], cfg["bw"]
    for p in range(npol):
        t = (torch.arange(nw, device=device, dtype=torch.float64) + 0.5) / rate
        on = (torch.remainder(t / cfg["period"] - 0.3, 1.0) < duty).to(torch.float32)
        del t
        x = torch.complex(torch.randn(nw, generator=gen, device=device),
                          torch.randn(nw, generator=gen, device=device)) * (np.sqrt(snr / 2) * on)
        del on
        X = torch.fft.fft(x)
        del x
        chunk = 1 << 26
        for a in range(0, nw, chunk):
            kk = torch.arange(a, min(a + chunk, nw), device=device, dtype=torch.float64)
            kk = torch.where(kk >= (nw + 1) // 2, kk - nw, kk)      # FFT order
            f = kk * (bw / nw)
            ph = torch.remainder(2 * np.pi * d * f * f / (cf * cf * (cf + f)) * np.sign(bw),
                                 2 * np.pi)
            X[a:a + kk.numel()] *= torch.polar(torch.ones_like(ph), ph).to(torch.complex64)
            del kk, f, ph
        x = torch.fft.ifft(X)
        del X
        x += torch.complex(torch.randn(nw, generator=gen, device=device),
                           torch.randn(nw, generator=gen, device=device)) * np.sqrt(0.5)
        for m0, y in pfb_channelise(x, h, nin, taps, ndat):
            n = y.shape[0]
            out[m0:m0 + n, :, p, 0] = torch.clamp(torch.round(y.real * 300 * np.sqrt(nin)),
                                                  -32768, 32767).to(torch.int16)
            out[m0:m0 + n, :, p, 1] = torch.clamp(torch.round(y.imag * 300 * np.sqrt(nin)),
                                                  -32768, 32767).to(torch.int16)
        del x
        torch.cuda.empty_cache()
    torch.cuda.synchronize()
    return out.reshape(-1)


def pfb_channelise(x, h, nin, taps, ndat, mch=1 << 15):
    """The oversampled PFB of a periodic signal x (complex64, one period):
    yields (m0, y[m, c]) chunks, y[m, c] = sum_k h[k] x[(mD - k) mod len(x)]
    exp(-2 pi i c (mD - k) / nin), D = 3 nin / 4: the band around c fs / nin
    shifted to DC, sampled every D samples (channel 0 on DC)."""
    import torch
    nw, D, L = x.numel(), nin * 3 // 4, taps * nin
    device = x.device
    hr = torch.flip(h, [0]).to(torch.complex64)
    c = torch.arange(nin, device=device, dtype=torch.float64)
    # xs[i] = x[(i - (L - 1)) mod nw]; frame m reads xs[mD + j], k = L - 1 - j
    need = (ndat - 1) * D + L
    reps = (need + nw - 1) // nw + 1
    xs = torch.cat([x[nw - (L - 1):]] + [x] * reps)[:need]
    for m0 in range(0, ndat, mch):
        m1 = min(ndat, m0 + mch)
        frames = xs.as_strided((m1 - m0, L), (D, 1), m0 * D)
        # z[r] = sum over k = r (mod nin) of h[k] x[mD - k]; then
        # sum_k h[k] x[mD - k] exp(2 pi i c k / nin) = nin * ifft(z)[c]
        z = (frames * hr).reshape(m1 - m0, taps, nin)
        z = torch.flip(z, [1, 2]).sum(1)
        z = torch.roll(z, shifts=-(nin - 1 - (L - 1) % nin) % nin, dims=1)
        y = torch.fft.ifft(z, dim=1) * nin
        m = torch.arange(m0, m1, device=device, dtype=torch.float64)
        rot = torch.remainder(torch.outer(m * D, c), nin) * (-2 * np.pi / nin)
        yield m0, y * torch.polar(torch.ones_like(rot), rot).to(torch.complex64)
    del xs


def run_b200_c5(args, cfg, world, rank, local):
    import math
    import torch
    import dspsr_b200 as b2
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ctx = b2.Context(local)
    ifb = b2.InverseFilterbank(ctx, cfg["nin"], 1, cfg["nin"], cfg["npol"], cfg["lin"],
                               os=(4, 3), output_discard=(cfg["disc"], cfg["disc"]))
    info = ifb.info
    in_step, out_step = info["in_step"], info["out_step"]
    ndat = cfg["ndat"]
    npart = ifb.npart(ndat)
    nwide = npart * out_step
    pos, neg, nfft = c5_plan(cfg, b2)
    pcfg = b2.make_config(cfg["cf"], cfg["bw"], cfg["dm"], 1, cfg["npol"], nfft, pos, neg,
                          cfg["nbin"], cfg["period"], state=b2.STOKES, input_kind=b2.FLOAT_FPT,
                          start_mjd=START_MJD, epoch_mjd=EPOCH_MJD, filterbank_nchan=cfg["fb"])
    pipe = b2.Pipeline(ctx, pcfg)
    gen = torch.Generator(device=device)
    gen.manual_seed(99 + rank)
    raw = torch.empty((ndat, cfg["nin"], cfg["npol"], 2), dtype=torch.int16, device=device)
    chunk = 1 << 18
    for t0 in range(0, ndat, chunk):
        n = min(chunk, ndat - t0)
        raw[t0:t0 + n] = (torch.randn((n, cfg["nin"], cfg["npol"], 2), generator=gen,
                                      device=device) * 100).round().to(torch.int16)
    raw = raw.reshape(-1)
    wide = torch.empty((1, cfg["npol"], nwide, 2), dtype=torch.float32, device=device)
    samples_per_step = cfg["nin"] * cfg["npol"] * npart * in_step
    default = torch.cuda.current_stream()

    def step(evs=None):
        if evs:
            evs[0].record(default)
        ifb.perform(raw, ndat, wide, nwide, input_kind=b2.INT16_TFPD)
        if evs:
            evs[1].record(default)
        pipe.run(wide, nwide, nwide)
        if evs:
            evs[2].record(default)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(1.0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = b2.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(default)
    for _ in range(args.steps):
        step()
    ev1.record(default)
    torch.cuda.synchronize()
    launches = b2.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6
    # stage split, and the pipeline's kernels
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    pipe.profile(True)
    step(evs)
    torch.cuda.synchronize()
    ktimes = pipe.kernel_times()
    pipe.profile(False)
    ifb_ms = evs[0].elapsed_time(evs[1])
    chain_ms = evs[1].elapsed_time(evs[2])
    prof, hits = pipe.get_profiles()
    ifb.status()
    hbm_peak, _, peak_src = measured_peaks()
    alg = raw.numel() * 2          # int16 input once
    achieved = alg / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": "complex Msamples/s inverse filterbank->fold", "value": round(value, 3),
        "unit": "complex Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian int16 PFB-channel voltages)",
        "config": {"workload": cfg["workload"], "ifb_parts": npart,
                   "ifb_fft": [cfg["lin"], info["lout"]], "rechannels": cfg["fb"],
                   "nfft": nfft, "nfilt_pos": pos, "nfilt_neg": neg,
                   "stage_ms": {"inverse_filterbank": round(ifb_ms, 3),
                                "filterbank_dedisperse_detect_fold": round(chain_ms, 3)},
                   "l2": f"input {raw.numel() * 2 >> 20} MiB per step, larger than L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clk,
        "gpu_launches": int(launches),
        "kernel_ms": {k: round(v[0], 3) for k, v in ktimes.items() if v[1]},
        "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": round(achieved, 2),
                     "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                     "traffic": None, "peak_source": peak_src,
                     "note": "algorithmic bytes: the int16 input once; FFT-bound chain"},
        "e2e": None,
        "parity": c5_parity(cfg, b2, raw, pos, neg, nfft) if rank == 0 and world == 1 else None,
        "check": {"hits_total": int(hits.sum()),
                  # a 1.6 ms turn is 1250 samples of the re-channelised data,
                  # so most of the 4096 bins get no hits: measure the hit ones
                  "bins_hit": int((hits > 0).sum()),
                  "profile_peak_over_median_of_hit_bins": float(
                      np.max((prof[:, 0].sum(0) / np.maximum(hits, 1))[hits > 0])
                      / max(np.median((prof[:, 0].sum(0) / np.maximum(hits, 1))[hits > 0]),
                            1e-30))},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    pipe.close()
    ifb.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lut-perturb", action="store_true",
                    help="c1/c2: an 8-bit table that is not affine, so the kernels look it up")
    ap.add_argument("--c3-tensor", type=int, default=1,
                    help="c3: let the autotuner also try the tensor-core rows (1) or not (0)")
    ap.add_argument("--no-proposer", action="store_true",
                    help="c4: skip the learned RFI-mask proposer")
    ap.add_argument("--proposer-steps", type=int, default=600,
                    help="c4: Adam steps of the proposer's training")
    ap.add_argument("--fft", default="fp32,bf16x3,bf16x2",
                    help="row-FFT arithmetic forms to time (comma list of fp32, bf16x3, "
                         "bf16x2); the first is the line's value, the others go under "
                         "'mixed' with their ratio to it (nfft >= 16384 only)")
    ap.add_argument("--subint-seconds", type=float, default=0.0,
                    help="also time the device-resident run folding sub-integrations of this "
                         "length (TimeDivide), unloaded through the callback (c1/c2)")
    ap.add_argument("--interchannel", action="store_true",
                    help="also time the device-resident run with inter-channel dedispersion "
                         "(-K: fractional delays in the response, SampleDelay before the fold) "
                         "(c1/c2)")
    ap.add_argument("--dada", action="store_true",
                    help="also time end to end from a DADA file holding the blocks "
                         "(pipeline_run_dada; the file is written first, so it is read from "
                         "the page cache) (c1/c2)")
    ap.add_argument("--scratch-mib", type=int, default=0,
                    help="device scratch of the four-step FFT batches (0: the library default)")
    ap.add_argument("--sk-inplace", action="store_true",
                    help="c4: mask the voltages in place (only zapped blocks are written)")
    ap.add_argument("--ndat", type=int, default=0,
                    help="samples per pol per block (default: the workload's); smaller blocks "
                         "are for profiling captures only")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup
    cfg = dict(CONFIGS[args.config])
    if args.ndat:
        cfg["ndat"] = args.ndat
        cfg["workload"] += f" [profiling size: {args.ndat} samples/pol per block]"
    world, rank, local = dist_init()
    try:
        kind = cfg.get("kind", "path")
        if args.impl == "reference":
            {"sk": run_reference_sk, "ifb": run_reference_ifb, "c3": run_reference_c3,
             "c5": run_reference_c5, "fbd": run_reference_fbd}.get(kind, run_reference)(
                 args, cfg, world, rank)
        else:
            {"sk": run_b200_sk, "ifb": run_b200_ifb, "c3": run_b200_c3,
             "c5": run_b200_c5, "fbd": run_b200_fbd}.get(kind, run_b200)(
                 args, cfg, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
