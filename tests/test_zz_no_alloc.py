"""dspsr_b200_convolution_perform_noalloc: the overlap-save convolution for
callers that cannot allocate device memory while they run (a real-time loop
with all memory fixed at start-up, or a host whose device memory belongs to
another allocator).  It keeps its tables and FFT scratch in one static device
array instead of an engine object.

The test calls it through the C ABI and checks its output against the
engine-object entry point (dspsr_b200_convolution_perform) on the same input,
twice in a row, that its status word reads 0 after each call, and that the
second call leaves the device's free memory unchanged; and that a call
captured in a CUDA graph (after one eager call has set the device up)
replays to the same output.  This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# both paths run the same kernels; only the twiddle tables are computed in a
# different place (device FP64 vs host FP64), so the outputs agree to rounding
NOALLOC_RTOL = 1e-6


def rel_rms(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def call_noalloc(b2, x, ndat, nchan, npol, nfft, pos, neg, h_dev, out, status=None, stream=None):
    lib = b2._capi.lib()
    n = ctypes.c_uint64()
    rc = lib.dspsr_b200_convolution_perform_noalloc(
        stream, x.data_ptr(), ndat, ndat, nchan, npol, nfft, pos, neg, h_dev.data_ptr(),
        out.data_ptr(), out.shape[-1], ctypes.byref(n),
        None if status is None else status.data_ptr())
    return rc, n.value


@pytest.mark.parametrize("nchan,nfft,pos,neg", [(1, 1 << 17, 28462, 29455),
                                                (2, 8192, 1000, 1500),
                                                (3, 1 << 14, 2000, 1777)])
def test_noalloc_matches_engine_entry_point(ctx, b2, nchan, nfft, pos, neg):
    rng = np.random.default_rng(nfft + nchan)
    npol = 2
    nk = nfft - pos - neg
    ndat = nfft + 4 * nk + 99
    x = (rng.standard_normal((nchan, npol, ndat)) + 1j * rng.standard_normal((nchan, npol, ndat))
         ).astype(np.complex64)
    h = (rng.standard_normal((nchan, nfft)) + 1j * rng.standard_normal((nchan, nfft))
         ).astype(np.complex64) / np.float32(np.sqrt(nfft))
    xd = torch.from_numpy(x).cuda()
    hd = torch.from_numpy(h).cuda()

    # the existing entry point, with its engine object
    c = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    c.copy_response(h)
    npart = c.npart(ndat)
    ref = torch.zeros((nchan, npol, npart * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(xd, ndat, ndat, ref, npart * nk) == npart
    ctx.synchronize()
    ref = ref.cpu().numpy()
    c.close()

    # a first call with less than one part still sets the device up
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    rc, n = call_noalloc(b2, xd, nfft - 1, nchan, npol, nfft, pos, neg, hd, xd, status)
    torch.cuda.synchronize()
    assert rc == 0 and n == 0
    assert int(status.item()) == 0

    free_after = None
    for call in range(2):
        out = torch.full((nchan, npol, npart * nk), np.nan, dtype=torch.complex64, device="cuda")
        status.fill_(7)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc, n = call_noalloc(b2, xd, ndat, nchan, npol, nfft, pos, neg, hd, out, status)
        torch.cuda.synchronize()
        assert rc == 0, rc
        assert n == npart
        assert int(status.item()) == 0, "a device-side wait gave up"
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_rms(got, ref) < NOALLOC_RTOL, (call, rel_rms(got, ref))
        if call == 1:
            # the second call finds its array set up and allocates nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        free_after = torch.cuda.mem_get_info()[0]
    assert free_after is not None


def test_noalloc_rejects_shapes_beyond_its_scratch(ctx, b2):
    nchan, npol, nfft, pos, neg = 64, 2, 1 << 16, 17576, 17743     # response alone is 32 MiB
    nk = nfft - pos - neg
    ndat = nfft + nk                    # two parts: (ndat - nfilt) / nkeep
    x = torch.zeros((nchan, npol, ndat), dtype=torch.complex64, device="cuda")
    h = torch.zeros((nchan, nfft), dtype=torch.complex64, device="cuda")
    out = torch.zeros((nchan, npol, 2 * nk), dtype=torch.complex64, device="cuda")
    rc, n = call_noalloc(b2, x, ndat, nchan, npol, nfft, pos, neg, h, out)
    assert rc == b2._capi.ETOOBIG and n == 0


@pytest.mark.parametrize("nchan,nfft,pos,neg", [(1, 1 << 17, 28462, 29455),
                                                (2, 8192, 1000, 1500)])
def test_noalloc_captured_in_a_cuda_graph(ctx, b2, nchan, nfft, pos, neg):
    rng = np.random.default_rng(7 * nfft + nchan)
    npol = 2
    nk = nfft - pos - neg
    ndat = nfft + 3 * nk + 5
    x = (rng.standard_normal((nchan, npol, ndat)) + 1j * rng.standard_normal((nchan, npol, ndat))
         ).astype(np.complex64)
    h = (rng.standard_normal((nchan, nfft)) + 1j * rng.standard_normal((nchan, nfft))
         ).astype(np.complex64) / np.float32(np.sqrt(nfft))
    xd = torch.from_numpy(x).cuda()
    hd = torch.from_numpy(h).cuda()
    c = b2.Convolution(ctx, nchan, npol, nfft, pos, neg)
    c.copy_response(h)
    npart = c.npart(ndat)
    ref = torch.zeros((nchan, npol, npart * nk), dtype=torch.complex64, device="cuda")
    assert c.perform(xd, ndat, ndat, ref, npart * nk) == npart
    ctx.synchronize()
    ref = ref.cpu().numpy()
    c.close()

    out = torch.full((nchan, npol, npart * nk), np.nan, dtype=torch.complex64, device="cuda")
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    # one eager call of the shape sets the device up before any capture
    rc, n = call_noalloc(b2, xd, ndat, nchan, npol, nfft, pos, neg, hd, out, status)
    torch.cuda.synchronize()
    assert rc == 0 and n == npart

    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(graph, stream=side):
        rc, n = call_noalloc(b2, xd, ndat, nchan, npol, nfft, pos, neg, hd, out, status,
                             stream=torch.cuda.current_stream().cuda_stream)
    assert rc == 0 and n == npart
    for rep in range(2):
        out.fill_(float("nan"))
        status.fill_(7)
        graph.replay()
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), rep
        assert rel_rms(got, ref) < NOALLOC_RTOL, (rep, rel_rms(got, ref))
    del graph
