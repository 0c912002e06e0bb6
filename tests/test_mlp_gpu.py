"""The learned warm start's network: the library's tensor-core forward and
backward kernels against the numpy oracle (which mirrors the device's BF16
roundings; the tolerance covers FP32 summation order), and training."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import learned as LN, tracer as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    import torch
    tr = T.CudaRayTracer(T.make_triangles(np.zeros((1, 9), np.float32), np.zeros(1, np.int32)))
    n = LN.Network(tr, seed=3)
    yield n, torch
    n.close()
    tr.close()


def _data(torch, n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, LN.INPUTS)).astype(np.float32)
    xt = torch.from_numpy(x).to("cuda").to(torch.bfloat16).contiguous()
    bits = xt.cpu().view(torch.int16).numpy().view(np.uint16)
    t = rng.normal(size=(n, LN.OUTPUTS)).astype(np.float32)
    return xt, bits, torch.from_numpy(t).cuda(), t


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle(net):
    from oracle import mlp_oracle as MO
    n, torch = net
    xt, bits, _, _ = _data(torch, 1000, 1)       # not a multiple of the 128-row tile
    y = n.forward(xt).cpu().numpy()
    want, _, _ = MO.forward(n.params(), bits)
    assert _rel(y, want) < 2e-3


def test_gradient_matches_oracle(net):
    from oracle import mlp_oracle as MO
    n, torch = net
    xt, bits, tt, t = _data(torch, 777, 2)
    g, loss = n.gradient(xt, tt)
    want, want_loss = MO.gradient(n.params(), bits, t)
    assert abs(loss - want_loss) < 1e-3 * want_loss
    gs, ws = LN.split(g), LN.split(want.astype(np.float32))
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        assert _rel(gs[name], ws[name]) < 1e-2, name
    # Two calls give the same gradient but for the atomics' order.
    g2, _ = n.gradient(xt, tt)
    assert _rel(g2, g) < 1e-5


def test_training_fits_a_function(net):
    import torch
    n, _ = net
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(20000, LN.INPUTS)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2], np.abs(x[:, 3]) - 0.5, x[:, 4] ** 2], 1).astype(np.float32)
    xt = torch.from_numpy(x).cuda().to(torch.bfloat16).contiguous()
    tt = torch.from_numpy(t).cuda()
    _, first = n.gradient(xt, tt)
    for step in range(400):
        n.train_step(xt, tt, 3e-3)
    torch.cuda.synchronize()
    last = n.loss()
    assert last < first / 10, (first, last)


def test_tcgen05_forward_at_scale_and_alignment(net):
    """The tcgen05 forward over a million rows (7,813 tiles on 2 CTAs per SM,
    the last tile partial) against the oracle on a spread of rows, and the
    same rows from a 4-byte-aligned (not 16-byte-aligned) input."""
    from oracle import mlp_oracle as MO
    n, torch = net
    rows = 1_000_003
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    xt = torch.randn((rows, LN.INPUTS), device="cuda", generator=g).to(torch.bfloat16).contiguous()
    y = n.forward(xt)
    torch.cuda.synchronize()
    n.status()
    pick = np.unique(np.concatenate([np.arange(0, 300), np.linspace(0, rows - 1, 3000).astype(np.int64),
                                     np.arange(rows - 300, rows)]))
    idx = torch.from_numpy(pick).cuda()
    bits = xt[idx].cpu().view(torch.int16).numpy().view(np.uint16)
    want, _, _ = MO.forward(n.params(), bits)
    got = y[idx].cpu().numpy()
    assert np.isfinite(got).all()
    assert _rel(got, want) < 2e-3
    # A view two elements in: rows start 4 bytes past a 16-byte boundary.
    buf = torch.zeros((4096 * LN.INPUTS + 2,), dtype=torch.bfloat16, device="cuda")
    view = buf[2:].view(4096, LN.INPUTS)
    view.copy_(xt[:4096])
    assert view.data_ptr() % 16 == 4
    y2 = n.forward(view)
    torch.cuda.synchronize()
    assert torch.equal(y2, y[:4096])
