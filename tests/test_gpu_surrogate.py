"""The gravity surrogate's tensor-core kernels against PyTorch FP32 references
of the same operations on the same BF16-rounded values."""
import ctypes as C

import numpy as np
import pytest

from bqp_b200 import _native as N

pytestmark = pytest.mark.gpu


def _gemm(a_bf16, b_bf16):
    import torch
    m, k = a_bf16.shape
    n = b_bf16.shape[0]
    c = torch.empty((m, n), dtype=torch.float32, device="cuda")
    N.check(N.lib().bqp_gemm_bf16_device(m, n, k, C.c_void_p(a_bf16.data_ptr()), C.c_void_p(b_bf16.data_ptr()),
                                         C.c_void_p(c.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return c


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (256, 512, 256), (1024, 256, 1024)])
def test_tensor_core_gemm_matches_fp32_reference(m, n, k):
    import torch
    g = torch.Generator().manual_seed(m + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T  # FP32 products of the BF16 values
    got = _gemm(a.cuda(), b.cuda()).cpu()
    err = (got - ref).abs().max().item()
    # FP32 accumulation in a different order: a few ulp of the partial sums
    assert err <= 1e-5 * np.sqrt(k) * ref.abs().max().item() + 1e-5, err
    # and not a trivially wrong layout: every element checked, signs too
    assert torch.allclose(got, ref, rtol=1e-4, atol=1e-3)


def _surrogate_ctx(order=20):
    from bqp_b200 import workloads
    cfg = N.default_config()
    cfg.order = order
    return N.Context(workloads.synthetic_field(order), cfg)


def test_surrogate_gradients_match_cpu_restatement():
    """Forward pass and every parameter's gradient of one batch against the
    numpy restatement with the same BF16 roundings (oracle/mlp.py)."""
    from oracle import mlp
    rng = np.random.default_rng(7)
    B = 256
    p = np.zeros(mlp.PARAMS, dtype=np.float32)
    p[mlp.OFF_W0:mlp.OFF_B0] = rng.uniform(-1.2, 1.2, 4 * mlp.H)
    p[mlp.OFF_B0:mlp.OFF_W1] = rng.uniform(-0.1, 0.1, mlp.H)
    p[mlp.OFF_W1:mlp.OFF_B1] = rng.uniform(-0.15, 0.15, 3 * mlp.H * mlp.H)
    p[mlp.OFF_B1:mlp.OFF_W4] = rng.uniform(-0.1, 0.1, 3 * mlp.H)
    p[mlp.OFF_W4:mlp.OFF_B4] = rng.uniform(-0.15, 0.15, 3 * mlp.H)
    x = np.concatenate([rng.normal(size=(B, 3)), rng.uniform(-1, 1, (B, 1))], axis=1).astype(np.float32)
    x[:, :3] /= np.linalg.norm(x[:, :3], axis=1, keepdims=True)
    t = rng.normal(size=(B, 3)).astype(np.float32)
    ctx = _surrogate_ctx()
    loss, g, y = ctx.surrogate_grad(p, x, t)
    oloss, og, oy = mlp.forward_backward(p, x, t)
    # the device's SiLU uses the fast exponential: a hidden activation next to
    # a BF16 rounding boundary can round one ulp (2^-8) the other way
    assert np.linalg.norm(y - oy) <= 2e-3 * np.linalg.norm(oy)
    assert np.abs(y - oy).max() <= 1e-2 * np.abs(oy).max()
    assert abs(loss - oloss) <= 2e-3 * oloss
    # per parameter block: relative L2 error of the gradient
    blocks = [(mlp.OFF_W0, mlp.OFF_B0), (mlp.OFF_B0, mlp.OFF_W1)] + \
             [(mlp.OFF_W1 + l * mlp.H * mlp.H, mlp.OFF_W1 + (l + 1) * mlp.H * mlp.H) for l in range(3)] + \
             [(mlp.OFF_B1, mlp.OFF_W4), (mlp.OFF_W4, mlp.OFF_B4), (mlp.OFF_B4, mlp.PARAMS)]
    for a, b in blocks:
        rel = np.linalg.norm(g[a:b] - og[a:b]) / np.linalg.norm(og[a:b])
        assert rel <= 2e-2, (a, b, rel)


def test_surrogate_learns_the_high_degree_field():
    """Training on the GPU reduces the error of the low-degree field (the
    method without the network) by a large factor on held-out positions."""
    order = 20
    ctx = _surrogate_ctx(order)
    loss = ctx.surrogate_train(samples=1 << 19, epochs=8, batch=4096, lr=2e-3, seed=3)
    assert loss[-1] < 0.25 * loss[0], loss
    rng = np.random.default_rng(11)
    n = 20000
    r = rng.uniform(6600.0, 7550.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = u * r[:, None]
    full = ctx.gravity(pos)[0]
    cfg8 = N.default_config()
    cfg8.order = N.SURROGATE_DEGREE
    from bqp_b200 import workloads
    low = N.Context(workloads.synthetic_field(order), cfg8).gravity(pos)[0]
    surr = ctx.surrogate_infer(pos, add_low=True)
    res = np.linalg.norm(full - low, axis=1)
    err_without = np.sqrt(np.mean(res ** 2))
    err_with = np.sqrt(np.mean(np.linalg.norm(full - surr, axis=1) ** 2))
    assert err_with < 0.5 * err_without, (err_with, err_without)
    # the fused inference kernel and the layer-by-layer kernels agree (the
    # same BF16 roundings; FP32 sums in another order)
    unfused = ctx.surrogate_infer(pos, add_low=True, fused=False)
    assert np.sqrt(np.mean(np.sum((unfused - surr) ** 2, axis=1))) <= 1e-3 * err_without
    # parameters round-trip through the host
    p, sigma = ctx.surrogate_params()
    ctx2 = _surrogate_ctx(order)
    ctx2.surrogate_set_params(p, sigma)
    assert np.allclose(ctx2.surrogate_infer(pos[:1000]), surr[:1000], rtol=0, atol=1e-15)


def test_propagation_with_surrogate_gravity():
    """The stage-synchronous engine's gravity through the trained surrogate
    (exact degrees <= 8 + network): one orbit of LEO rows lands far closer
    to the exact-field propagation than the degree-8 field alone does."""
    from bqp_b200 import workloads
    order = 20
    text = workloads.synthetic_field(order)
    ctx = _surrogate_ctx(order)
    ctx.surrogate_train(samples=1 << 19, epochs=8, batch=4096, lr=2e-3, seed=3)
    n = 512
    states = workloads.leo_states(n, seed=9)

    def run(c, order_, surrogate, check=0.0):
        cfg = N.default_config()
        cfg.order = order_
        cfg.force_flags = N.FORCE_SUN | N.FORCE_MOON
        cfg.eps = 1e-9
        cfg.surrogate = int(surrogate)
        cfg.surrogate_check = check
        c.set_config(cfg)
        out, st, _, ev = c.propagate_final(states, workloads.EPOCH_JD, 5400.0)
        assert (st == 0).all()
        return out, ev

    exact, ev_exact = run(_surrogate_ctx(order), order, False)
    low, _ = run(_surrogate_ctx(order), N.SURROGATE_DEGREE, False)
    sur, ev = run(ctx, order, True)
    d_sur = np.linalg.norm(sur[:, :3] - exact[:, :3], axis=1)
    d_low = np.linalg.norm(low[:, :3] - exact[:, :3], axis=1)
    assert (ev > 0).all()
    assert np.sqrt(np.mean(d_sur ** 2)) < 0.5 * np.sqrt(np.mean(d_low ** 2)), (d_sur.mean(), d_low.mean())

    # the per-step residual check with the exact field as fallback: a
    # threshold no row meets puts every step on the exact field (the exact
    # run's trajectory), one every row meets leaves the surrogate run as it was
    # (the exact kernel's column split follows the launch's rows per CTA, so
    # the fallback rows' sums may differ from the exact run's in the last bits)
    every, ev_every = run(ctx, order, True, check=1e-30)
    assert np.abs(every[:, :3] - exact[:, :3]).max() <= 1e-5, np.abs(every - exact).max()
    assert abs(ev_every.mean() / ev_exact.mean() - 1.0) < 0.01
    none, ev_none = run(ctx, order, True, check=1e30)
    assert np.abs(none - sur).max() <= 1e-9, np.abs(none - sur).max()
    assert (ev_none == ev).all()
    # between them: the median of the network's relative error at the orbits'
    # starting positions sends some rows' steps to the exact field
    full = ctx.gravity(states[:, :3])[0]
    rel = np.linalg.norm(ctx.surrogate_infer(states[:, :3], add_low=True) - full, axis=1) / np.linalg.norm(full, axis=1)
    mixed, _ = run(ctx, order, True, check=float(np.median(rel)))
    d_mixed = np.linalg.norm(mixed[:, :3] - exact[:, :3], axis=1)
    moved = np.linalg.norm(mixed[:, :3] - sur[:, :3], axis=1) > 0
    assert moved.any() and (d_mixed > 1e-9).any()
    assert np.sqrt(np.mean(d_mixed ** 2)) < np.sqrt(np.mean(d_sur ** 2)), (d_mixed.mean(), d_sur.mean())
    print(f"\nsurrogate RMS miss {np.sqrt(np.mean(d_sur ** 2)):.3e} km; with the check at the median relative "
          f"error {np.median(rel):.2e}: {np.sqrt(np.mean(d_mixed ** 2)):.3e} km, {moved.sum()} of {n} rows moved")
    # the check is refused when negative or not finite
    cfg = N.default_config()
    cfg.order = order
    cfg.surrogate = 1
    for bad in (-1.0, float("nan"), float("inf")):
        cfg.surrogate_check = bad
        with pytest.raises(N.NativeError):
            ctx.set_config(cfg)
    # the surrogate form refuses to run untrained
    cfg = N.default_config()
    cfg.order = order
    cfg.surrogate = 1
    fresh = _surrogate_ctx(order)
    fresh.set_config(cfg)
    with pytest.raises(N.NativeError):
        fresh.propagate_final(states[:4], workloads.EPOCH_JD, 60.0)
