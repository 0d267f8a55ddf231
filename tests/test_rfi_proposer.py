"""The learned RFI-mask proposer (csrc/rfi.cu) through the C ABI.

Labels and fallback come from the SpectralKurtosis kernel, which the SK tests
hold bit-exact to the oracle's restatement of SpectralKurtosis::compute and
detect_skfb (SpectralKurtosis.C:674-798, 1105-1222).  Here:
- the features against a numpy evaluation of the same formulas on the same
  sums;
- the tensor-core inference (BF16 operands, FP32 accumulation) against a
  PyTorch FP32 evaluation of the same network with the operands rounded to
  BF16 the same way;
- one Adam step against the sign of PyTorch's autograd gradient;
- training on SK masks of RFI-injected noise: the proposer alone agrees with
  SK on most cells and, with the SK fallback, on more."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

NF, NH = 8, 32


def make_rfi(rng, nchan, npol, nblk, M):
    ndat = nblk * M
    x = (rng.standard_normal((nchan, npol, ndat)) + 1j * rng.standard_normal((nchan, npol, ndat))
         ) / np.sqrt(2)
    t = np.arange(ndat)
    for _ in range(6):                                         # CW tones
        c = rng.integers(nchan)
        x[c] += rng.uniform(0.5, 5.0) * np.exp(2j * np.pi * rng.uniform(-0.5, 0.5) * t)
    for _ in range(int(0.01 * ndat / 32.5)):                   # broadband bursts
        w = int(rng.integers(1, 65))
        t0 = int(rng.integers(0, ndat - w))
        x[:, :, t0:t0 + w] *= rng.uniform(3.0, 30.0)
    for b in range(nblk):                                      # drifting chirp
        c = (b * nchan) // nblk
        tt = np.arange(M)
        x[c, :, b * M:(b + 1) * M] += 3 * np.exp(2j * np.pi * (0.05 * tt + 1e-5 * tt * tt))
    return x.astype(np.complex64)


def run_sk(ctx, b2, x, M):
    nchan, npol, ndat = x.shape
    nblk = ndat // M
    lo, hi = b2.sk_limits(M, 1, 3.0, npol)
    d = torch.from_numpy(x).cuda()
    out = torch.empty_like(d)
    sums = torch.zeros((nblk, nchan, npol, 2), dtype=torch.float32, device="cuda")
    counts = torch.zeros((nblk, nchan), dtype=torch.int32, device="cuda")
    mask = torch.zeros((nblk, nchan), dtype=torch.uint8, device="cuda")
    assert ctx.sk(d, ndat, ndat, nchan, npol, M, lo, hi, out, ndat, sums, counts, mask) == nblk
    ctx.synchronize()
    return sums, counts, mask


def np_features(sums, counts, M):
    s = sums.cpu().numpy().astype(np.float32)
    mp = counts.cpu().numpy().astype(np.float32)
    nblk, nchan, npol, _ = s.shape
    S1, S2 = s[..., 0], s[..., 1]
    mf = (mp * 1 + 1) / (mp - 1)
    V = mf[..., None] * (mp[..., None] * (S2 / (S1 * S1)) - 1)
    lp = np.log(np.maximum(S1, 1e-30) / mp[..., None])
    lmean = lp[..., 0].mean(1, keepdims=True)
    f = np.zeros((nblk, nchan, NF), np.float32)
    f[..., 0:2] = np.clip(16 * (lp - lmean[..., None]), -64, 64)
    vv = np.clip(16 * (V - 1), -16, 64)
    f[..., 2:4] = vv
    f[1:, :, 4:6] = vv[:-1]
    f[:-1, :, 6:8] = vv[1:]
    return f


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float32)


def torch_forward(p, X, emulate_bf16):
    """logits [nblk, nchan] of the network at params p (FP32 flat) on features X."""
    W1 = torch.from_numpy(p[:768].reshape(NH, NF, 3))
    b1 = torch.from_numpy(p[768:800])
    W2 = torch.from_numpy(p[800:3872].reshape(NH, NH, 3))
    b2_ = torch.from_numpy(p[3872:3904])
    W3 = torch.from_numpy(p[3904:3936])
    b3 = float(p[3936])
    x = torch.from_numpy(X).permute(0, 2, 1)           # [nblk, NF, nchan]
    q = bf16 if emulate_bf16 else (lambda t: t)
    h = torch.relu(torch.nn.functional.conv1d(q(x), q(W1), b1, padding=1))
    h = torch.relu(torch.nn.functional.conv1d(q(h), q(W2), b2_, padding=2, dilation=2))
    return torch.einsum("bhc,h->bc", h, W3) + b3


@pytest.fixture(scope="module")
def rfi_case(ctx, b2):
    rng = np.random.default_rng(4)
    M, nchan, nblk = 256, 64, 96
    x = make_rfi(rng, nchan, 2, nblk, M)
    sums, counts, mask = run_sk(ctx, b2, x, M)
    return M, nchan, nblk, sums, counts, mask


def test_proposer_features_match_numpy(ctx, b2, rfi_case):
    M, nchan, nblk, sums, counts, mask = rfi_case
    pr = b2.RfiProposer(ctx, nchan, M, max_npart=nblk)
    pr.features(sums, nblk, 2, counts)
    got = pr.get_features()
    ref = np_features(sums, counts, M)
    assert np.allclose(got, ref, rtol=1e-4, atol=2e-4), float(np.max(np.abs(got - ref)))
    pr.close()


def test_proposer_inference_matches_torch(ctx, b2, rfi_case):
    M, nchan, nblk, sums, counts, mask = rfi_case
    pr = b2.RfiProposer(ctx, nchan, M, max_npart=nblk, seed=11)
    rng = np.random.default_rng(9)
    p = pr.params()
    p = (p + 0.05 * rng.standard_normal(p.size)).astype(np.float32)   # biases non-zero too
    pr.set_params(p)
    pr.features(sums, nblk, 2, counts)
    prob = torch.zeros((nblk, nchan), dtype=torch.float32, device="cuda")
    out = torch.zeros((nblk, nchan), dtype=torch.uint8, device="cuda")
    pr.infer(out, prob, None, confidence=0.5)
    got = prob.cpu().numpy()
    X = pr.get_features()
    z = torch_forward(p, X, emulate_bf16=True).numpy()
    ref = 1 / (1 + np.exp(-z))
    assert np.max(np.abs(got - ref)) < 2e-4, float(np.max(np.abs(got - ref)))
    # and against the plain FP32 network: BF16 operands (8 significant bits)
    # move logits near 0 by up to a few tenths
    z32 = torch_forward(p, X, emulate_bf16=False).numpy()
    assert np.max(np.abs(got - 1 / (1 + np.exp(-z32)))) < 0.1
    assert np.array_equal(out.cpu().numpy(), (got >= 0.5).astype(np.uint8))
    pr.close()


def test_proposer_adam_step_follows_autograd(ctx, b2, rfi_case):
    M, nchan, nblk, sums, counts, mask = rfi_case
    pr = b2.RfiProposer(ctx, nchan, M, max_npart=nblk, max_batch_blocks=nblk, seed=3)
    pr.features(sums, nblk, 2, counts)
    p0 = pr.params()
    lr, wpos = 1e-3, 4.0
    pr.train(mask, 1, batch_blocks=nblk, lr=lr, pos_weight=wpos)
    dp = pr.params() - p0
    # autograd on the same batch (all blocks)
    X = pr.get_features()
    pt = torch.from_numpy(p0.copy()).requires_grad_(True)
    y = torch.from_numpy(mask.cpu().numpy().astype(np.float32))
    W1, b1 = pt[:768].reshape(NH, NF, 3), pt[768:800]
    W2, b2_ = pt[800:3872].reshape(NH, NH, 3), pt[3872:3904]
    W3, b3 = pt[3904:3936], pt[3936]
    x = torch.from_numpy(X).permute(0, 2, 1)
    h = torch.relu(torch.nn.functional.conv1d(x, W1, b1, padding=1))
    h = torch.relu(torch.nn.functional.conv1d(h, W2, b2_, padding=2, dilation=2))
    z = torch.einsum("bhc,h->bc", h, W3) + b3
    w = torch.where(y > 0, torch.tensor(wpos), torch.tensor(1.0))
    loss = (w * torch.nn.functional.binary_cross_entropy_with_logits(z, y, reduction="none")).mean()
    loss.backward()
    g = pt.grad.numpy()
    big = np.abs(g) > 1e-5
    assert big.sum() > 1000
    # Adam's first step moves each weight by lr against the sign of its gradient
    assert np.mean(np.sign(dp[big]) == -np.sign(g[big])) > 0.99
    assert np.allclose(np.abs(dp[big]), lr, rtol=0.05)
    pr.close()


def test_proposer_learns_sk_masks(ctx, b2):
    rng = np.random.default_rng(21)
    M, nchan, nblk = 256, 64, 192
    x = make_rfi(rng, nchan, 2, nblk, M)
    sums, counts, mask = run_sk(ctx, b2, x, M)
    pr = b2.RfiProposer(ctx, nchan, M, max_npart=nblk, max_batch_blocks=32, seed=5)
    pr.features(sums, nblk, 2, counts)
    first = pr.train(mask, 20, batch_blocks=32, lr=3e-3)
    last = pr.train(mask, 400, batch_blocks=32, lr=3e-3)
    assert last < first
    # a held-out RFI block of the same kind
    x2 = make_rfi(np.random.default_rng(22), nchan, 2, 96, M)
    sums2, counts2, mask2 = run_sk(ctx, b2, x2, M)
    pr.features(sums2, 96, 2, counts2)
    alone = torch.zeros((96, nchan), dtype=torch.uint8, device="cuda")
    pr.infer(alone, None, None, confidence=0.5)
    fb = torch.zeros_like(alone)
    nfall = pr.infer(fb, None, mask2, confidence=0.9)
    sk = mask2.cpu().numpy().astype(bool)
    a = alone.cpu().numpy().astype(bool)
    f = fb.cpu().numpy().astype(bool)
    assert sk.sum() > 50
    miss = np.sum(sk & ~a) / sk.sum()
    false_zap = np.sum(~sk & a) / (~sk).sum()
    assert miss < 0.2 and false_zap < 0.02, (miss, false_zap)
    miss_f = np.sum(sk & ~f) / sk.sum()
    assert miss_f <= miss and np.sum(~sk & f) <= np.sum(~sk & a)
    assert 0 < nfall < sk.size
    pr.close()
