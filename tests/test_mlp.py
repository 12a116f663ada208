"""The planner MLP: the FP64 oracle pinned by finite differences (CPU), and the CUDA
forward / backward / Adam kernels against the oracle (GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _case(seed, batch):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.2, M.NPARAMS)
    x = rng.normal(0, 1, (batch, M.IN))
    t = rng.normal(0, 1, (batch, M.OUT))
    return p, x, t


def test_oracle_gradient_matches_finite_differences():
    p, x, t = _case(1, 40)
    g = M.grad(p, x, t)
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.choice(M.NPARAMS, 60, replace=False), [M.NPARAMS - 1, M.NPARAMS - 2, 0]])
    h = 1e-6
    for i in idx:
        e = np.zeros(M.NPARAMS)
        e[i] = h
        fd = (M.loss(p + e, x, t) - M.loss(p - e, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), i
    assert M.NPARAMS == 5890


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [1, 31, 32, 33, 1000, 20_000])
def test_cuda_forward_backward_match_fp64_oracle(batch):
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    p, x, t = _case(10 + batch, batch)
    dp = torch.tensor(p, dtype=torch.float32, device="cuda")
    dx = torch.tensor(x, dtype=torch.float32, device="cuda")
    dt = torch.tensor(t, dtype=torch.float32, device="cuda")
    y = torch.empty(batch, 2, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    L.call("mb_mlp_forward", dp.data_ptr(), dx.data_ptr(), batch, y.data_ptr(), st)
    # fp32 kernels against the fp64 oracle evaluated at the fp32-rounded inputs
    p32, x32, t32 = (a.astype(np.float32).astype(np.float64) for a in (p, x, t))
    y_ref, _ = M.forward(p32, x32)
    assert np.allclose(y.cpu().numpy(), y_ref, rtol=1e-4, atol=1e-4)
    g = torch.zeros(M.NPARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    L.call("mb_mlp_backward", dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), batch, g.data_ptr(), loss.data_ptr(), st)
    g_ref = M.grad(p32, x32, t32)
    scale = np.abs(g_ref).max()
    assert np.allclose(g.cpu().numpy(), g_ref, rtol=1e-3, atol=1e-5 * scale)
    assert abs(loss.item() / batch - M.loss(p32, x32, t32)) <= 1e-4 * M.loss(p32, x32, t32) + 1e-6


@pytest.mark.gpu
def test_cuda_adam_and_training_reduce_loss():
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    st = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(4)
    p = rng.normal(0, 0.1, M.NPARAMS)
    g = rng.normal(0, 1, M.NPARAMS)
    m = np.zeros(M.NPARAMS)
    v = np.zeros(M.NPARAMS)
    dp, dg, dm, dv = (torch.tensor(a, dtype=torch.float32, device="cuda") for a in (p, g, m, v))
    for step in (1, 2, 3):
        L.call("mb_mlp_adam", dp.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), M.NPARAMS, 1e-3, 0.9, 0.999,
               1e-8, step, 1e-4, st)
        p, m, v = M.adam(p, g, m, v, step, 1e-3, weight_decay=1e-4)
    assert np.allclose(dp.cpu().numpy(), p, rtol=1e-5, atol=1e-6)
    # a learnable target: the loss falls by an order of magnitude in a few hundred steps
    x = rng.normal(0, 1, (4096, M.IN))
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1], x[:, 2] * x[:, 3] * 0.3], 1)
    dx = torch.tensor(x, dtype=torch.float32, device="cuda")
    dt = torch.tensor(t, dtype=torch.float32, device="cuda")
    dp = torch.tensor(rng.normal(0, 0.1, M.NPARAMS), dtype=torch.float32, device="cuda")
    dm, dv, dg = (torch.zeros(M.NPARAMS, dtype=torch.float32, device="cuda") for _ in range(3))
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    first = None
    for step in range(1, 401):
        dg.zero_()
        loss.zero_()
        L.call("mb_mlp_backward", dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), 4096, dg.data_ptr(), loss.data_ptr(),
               st)
        L.call("mb_mlp_adam", dp.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), M.NPARAMS, 3e-3, 0.9,
               0.999, 1e-8, step, 0.0, st)
        if first is None:
            first = loss.item()
    assert loss.item() < 0.1 * first


def test_host_forward_matches_fp64_oracle():
    """The planner's host forward pass (the serving router's path) against the oracle."""
    from mordred_b200.planner import LearnedPlanner
    p, x, _ = _case(77, 300)
    pl = LearnedPlanner(params=p, device="cpu")
    y = pl.predict_log_host(x)
    y_ref, _ = M.forward(p.astype(np.float32).astype(np.float64), x.astype(np.float32).astype(np.float64))
    assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_host_forward_matches_cuda_forward():
    from mordred_b200.planner import LearnedPlanner
    p, x, _ = _case(78, 500)
    pl = LearnedPlanner(params=p)
    assert np.allclose(pl.predict_log_host(x), pl.predict_log(x), rtol=1e-4, atol=1e-4)
