"""CPU checks of the learned bracket's host side: the packed parameter layout, and the
hand-written backward of the CPU reference (the one the device gradient is checked
against) versus torch autograd in plain FP32."""
import numpy as np
import torch


def test_layout_and_init(ht):
    br = ht.bracket
    assert sum(int(np.prod(s)) for _, s in br.LAYOUT) == ht.bracket.HT_BRACKET_NPARAMS == 9928
    p = br.init_params(3)
    o, s = br.OFFSETS["W4"]
    W4 = p[o:o + 512].reshape(s)
    assert np.all(W4[2:] == 0) and np.any(W4[:2] != 0)
    o, s = br.OFFSETS["W1"]
    assert np.all(p[o:o + 1024].reshape(s)[:, 12:] == 0)


def test_reference_backward_matches_autograd(ht):
    br = ht.bracket
    rng = np.random.default_rng(0)
    n = 300
    params = br.init_params(1)
    params[br.OFFSETS["b1"][0]:br.OFFSETS["b4"][0] + 8] = rng.normal(0, 0.1, 64 * 3 + 8)
    F = rng.normal(0, 1, (n, 16)).astype(np.float32)
    F[:, 12:] = 0
    mean = np.zeros(16, np.float32)
    istd = np.ones(16, np.float32)
    t = rng.normal(0, 1, n).astype(np.float32)
    g = br.reference_grad(params, mean, istd, F, t, bf16=False)

    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    W = {k: p[o:o + int(np.prod(s))].view(s) for k, (o, s) in br.OFFSETS.items()}
    X = torch.tensor(F, dtype=torch.float64)
    h = X
    for wn, bn in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        h = torch.clamp(h @ W[wn].T + W[bn], min=0.0)
    Y = h @ W["W4"][:2].T + W["b4"][:2]
    tt = torch.tensor(t, dtype=torch.float64)
    loss = 0.0
    for q, tau in enumerate(br.QUANTILES):
        d = tt - Y[:, q]
        loss = loss + torch.where(d > 0, tau * d, (tau - 1.0) * d).mean()
    loss.backward()
    ref = p.grad.numpy()
    assert np.allclose(g, ref, rtol=1e-4, atol=1e-6 * np.abs(ref).max())
