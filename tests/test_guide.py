"""The path-guiding MLP: FP64 oracle self-check (CPU) and the tensor-core
kernels against the oracle (GPU): inference, gradients, the Adam step, and
what training buys on a known target distribution."""
import ctypes as C

import numpy as np
import pytest

import mcpt
from helpers import oracle

P = mcpt.GUIDE_PARAM_COUNT
LO = np.array([-1.0, -1.0, -1.0], np.float32)
HI = np.array([1.0, 1.0, 1.0], np.float32)
INV = (np.float32(1.0) / (HI - LO)).astype(np.float32)

# parameter blocks: (name, offset, size)
BLOCKS = [("W1", 0, 64 * 144), ("b1", 9216, 64), ("W2", 9280, 4096), ("b2", 13376, 64), ("W3", 13440, 4096),
          ("b3", 17536, 64), ("W4", 17600, 2560), ("b4", 20160, 40)]


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _params(rng):
    p = np.zeros(P, np.float64)
    for name, off, size in BLOCKS:
        if name.startswith("W"):
            fan_in = 144 if name == "W1" else 64
            gain = 0.3 if name == "W4" else 1.0
            p[off:off + size] = rng.uniform(-1, 1, size) * np.sqrt(6.0 / fan_in) * gain
        else:
            p[off:off + size] = rng.normal(0, 0.05, size)
    return p.astype(np.float32).astype(np.float64)


def _records(rng, n):
    rec = np.zeros((n, 10), np.float32)
    rec[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    rec[:, 3:6] = _unit(rng, n)
    rec[:, 6:9] = _unit(rng, n)
    rec[:, 9] = rng.uniform(0.1, 1.0, n)
    return rec


def _oracle_grad(params, rec, emulate):
    g = np.zeros(P, np.float64)
    loss = C.c_double()
    oracle().orc_guide_loss_grad(params.ctypes.data, rec.ctypes.data, len(rec), LO.ctypes.data, INV.ctypes.data, emulate,
                                 g.ctypes.data, C.byref(loss))
    return g, loss.value


def _oracle_mix(params, queries, emulate):
    out = np.zeros((len(queries), 40), np.float64)
    oracle().orc_guide_forward(params.ctypes.data, queries.ctypes.data, len(queries), LO.ctypes.data, INV.ctypes.data,
                               emulate, out.ctypes.data)
    return out


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    params = _params(rng)
    rec = _records(rng, 12)
    g, loss = _oracle_grad(params, rec, 0)
    assert np.isfinite(loss) and np.all(np.isfinite(g))
    idx = np.concatenate([rng.choice(np.arange(off, off + size), 6, replace=False) for _, off, size in BLOCKS])
    for i in idx:
        h = 1e-6 * max(1.0, abs(params[i]))
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        fd = (_oracle_grad(pp, rec, 0)[1] - _oracle_grad(pm, rec, 0)[1]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_oracle_anchored_gradient_matches_finite_differences():
    """Anchored lobes (every raw mean offset by 1.5 x the direction input):
    the offset is a constant, so the gradient still matches finite
    differences."""
    rng = np.random.default_rng(13)
    params = _params(rng)
    rec = _records(rng, 12)
    for flags in (2, 6):
        g, loss = _oracle_grad(params, rec, flags)
        assert np.isfinite(loss) and np.all(np.isfinite(g))
        assert loss != _oracle_grad(params, rec, 0)[1]
        idx = np.concatenate([rng.choice(np.arange(off, off + size), 3, replace=False) for _, off, size in BLOCKS])
        for i in idx:
            h = 1e-6 * max(1.0, abs(params[i]))
            pp, pm = params.copy(), params.copy()
            pp[i] += h
            pm[i] -= h
            fd = (_oracle_grad(pp, rec, flags)[1] - _oracle_grad(pm, rec, flags)[1]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (flags, i, fd, g[i])


def test_oracle_bf16_mirror_stays_close_to_fp64():
    rng = np.random.default_rng(12)
    params = _params(rng)
    rec = _records(rng, 64)
    g64, l64 = _oracle_grad(params, rec, 0)
    gbf, lbf = _oracle_grad(params, rec, 1)
    assert abs(lbf - l64) < 2e-2 * abs(l64)
    assert np.linalg.norm(gbf - g64) < 0.1 * np.linalg.norm(g64)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = mcpt.Context(0)
    yield c
    c.close()


def _guide(ctx, params=None, **kw):
    g = mcpt.Guide(ctx, LO.tolist(), HI.tolist(), **kw)
    if params is not None:
        g.set_params(params.astype(np.float32))
    return g


def _gpu_grad(ctx, g, rec):
    d_rec = torch.from_numpy(rec).cuda()
    d_g = torch.zeros(P, dtype=torch.float32, device="cuda")
    loss = C.c_double()
    mcpt.check(ctx.lib.mc_guide_gradient(g.handle, d_rec.data_ptr(), len(rec), d_g.data_ptr(), C.byref(loss)))
    return d_g.cpu().numpy().astype(np.float64), loss.value


# (anchor_lobes, direction_input) -> the oracle's anchor flags
ANCHOR_CASES = [(False, 0, 0), (True, 0, 2), (True, 1, 6)]


@pytest.mark.gpu
@pytest.mark.parametrize("anchor,direction,aflags", ANCHOR_CASES)
def test_inference_matches_oracle(ctx, anchor, direction, aflags):
    rng = np.random.default_rng(21)
    params = _params(rng)
    g = _guide(ctx, params, anchor_lobes=anchor, direction_input=direction)
    n = 1000
    q = np.zeros((n, 6), np.float32)
    q[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    q[:, 3:6] = _unit(rng, n)
    out = torch.zeros(n * 40, dtype=torch.float32, device="cuda")
    dq = torch.from_numpy(q).cuda()
    mcpt.check(ctx.lib.mc_guide_infer(g.handle, dq.data_ptr(), n, out.data_ptr()))
    got = out.cpu().numpy().reshape(n, 40).astype(np.float64)
    ref = _oracle_mix(params, q, 1 | aflags)
    np.testing.assert_allclose(got[:, :8].sum(1), 1.0, atol=1e-5)
    # BF16 activations: an FP32-accumulation difference can flip one rounding,
    # so a few elements sit further off than the bulk
    np.testing.assert_allclose(got[:, :8], ref[:, :8], atol=2e-3)
    dm = np.abs(got[:, 8:32] - ref[:, 8:32])
    assert np.quantile(dm, 0.999) < 5e-3 and dm.max() < 3e-2
    np.testing.assert_allclose(got[:, 32:40], ref[:, 32:40], rtol=2e-2)
    # the pure FP64 network is close as well (BF16 is the only approximation)
    ref64 = _oracle_mix(params, q, aflags)
    assert np.abs(got[:, :8] - ref64[:, :8]).max() < 2e-2
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,anchor,direction,aflags", [(100, False, 0, 0), (1000, False, 0, 0), (40000, False, 0, 0),
                                                       (1000, True, 0, 2), (1000, True, 1, 6)])
def test_gradient_matches_oracle(ctx, n, anchor, direction, aflags):
    rng = np.random.default_rng(22 + n)
    params = _params(rng)
    g = _guide(ctx, params, anchor_lobes=anchor, direction_input=direction)
    rec = _records(rng, n)
    got, loss = _gpu_grad(ctx, g, rec)
    ref, rloss = _oracle_grad(params, rec, 1 | aflags)
    assert abs(loss - rloss) < 1e-3 * abs(rloss) + 1e-6
    for name, off, size in BLOCKS:
        a, b = got[off:off + size], ref[off:off + size]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-2, (name, err)
    g.close()


@pytest.mark.gpu
def test_adam_step_follows_the_gradient(ctx):
    rng = np.random.default_rng(23)
    params = _params(rng)
    g = _guide(ctx, params, learning_rate=1e-3, anchor_lobes=False)
    rec = _records(rng, 5000)
    # the step follows the kernel's own gradient (the gradient tests compare
    # that with the oracle; a component near zero can take either sign there)
    grad, _ = _gpu_grad(ctx, g, rec)
    grad /= rec[:, 9].astype(np.float64).sum()
    ref, _ = _oracle_grad(params, rec, 1)
    ref /= rec[:, 9].astype(np.float64).sum()
    assert np.linalg.norm(grad - ref) < 2e-2 * np.linalg.norm(ref)
    d_rec = torch.from_numpy(rec).cuda()
    mcpt.check(ctx.lib.mc_guide_train(g.handle, d_rec.data_ptr(), len(rec)))
    assert g.steps() == 1
    new = g.get_params().astype(np.float64)
    step = new - params
    # first Adam step: -lr * g / (|g| + eps) = -lr * sign(g) where |g| >> eps
    big = np.abs(grad) > 1e-5
    np.testing.assert_allclose(step[big], -1e-3 * np.sign(grad[big]), atol=2e-5)
    g.close()


def _target_records(rng, n):
    """Positions uniform in the box; the next direction drawn from a vMF
    (kappa 20) whose mean points from the position to a fixed point; weight 1."""
    rec = np.zeros((n, 10), np.float32)
    pos = rng.uniform(-1, 1, (n, 3))
    rec[:, 0:3] = pos
    rec[:, 3:6] = _unit(rng, n)
    mu = np.array([0.3, 2.0, -0.2]) - pos
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    kappa = 20.0
    u1, u2 = rng.uniform(size=n), rng.uniform(size=n)
    w = 1.0 + np.log(u1 + (1 - u1) * np.exp(-2 * kappa)) / kappa
    s = np.sqrt(np.maximum(0, 1 - w * w))
    phi = 2 * np.pi * u2
    a = np.where(np.abs(mu[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    t = np.cross(mu, a)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(mu, t)
    d = t * (s * np.cos(phi))[:, None] + b * (s * np.sin(phi))[:, None] + mu * w[:, None]
    rec[:, 6:9] = d
    rec[:, 9] = 1.0
    return rec


@pytest.mark.gpu
def test_training_learns_a_directional_target(ctx):
    """Maximum-likelihood training on samples of a position-dependent vMF: the
    trained mixture assigns the held-out samples far more density than the
    untrained one and than uniform sampling (log(1/4pi) = -2.53)."""
    rng = np.random.default_rng(24)
    g = _guide(ctx, seed=5, learning_rate=3e-3, anchor_lobes=False)
    held = _target_records(rng, 4096)

    def mean_log_q():
        _, loss = _gpu_grad(ctx, g, held)
        return -loss / len(held)

    before = mean_log_q()
    for _ in range(300):
        batch = torch.from_numpy(_target_records(rng, 4096)).cuda()
        mcpt.check(ctx.lib.mc_guide_train(g.handle, batch.data_ptr(), 4096))
    after = mean_log_q()
    assert after > before + 2.0, (before, after)
    assert after > -2.53 + 2.0, after
    g.close()


@pytest.mark.gpu
def test_untrained_anchored_guide_proposes_around_the_normal(ctx):
    """An untrained anchored guide: every lobe's mean lies close to the
    direction input (the normal the renderer feeds it) and kappa starts near
    e, so its first samples stay mostly above the surface; an unanchored
    guide's means point anywhere."""
    rng = np.random.default_rng(25)
    n = 4096
    q = np.zeros((n, 6), np.float32)
    q[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    q[:, 3:6] = _unit(rng, n)
    dq = torch.from_numpy(q).cuda()
    cos = {}
    for anchor in (False, True):
        g = _guide(ctx, seed=9, anchor_lobes=anchor)
        out = torch.zeros(n * 40, dtype=torch.float32, device="cuda")
        mcpt.check(ctx.lib.mc_guide_infer(g.handle, dq.data_ptr(), n, out.data_ptr()))
        m = out.cpu().numpy().reshape(n, 40).astype(np.float64)
        means = m[:, 8:32].reshape(n, 8, 3)
        cos[anchor] = np.einsum("nkj,nj->nk", means, q[:, 3:6].astype(np.float64))
        if anchor:
            kap = m[:, 32:40]
            # log kappa = 1 + the untrained output layer's spread (about 0.13)
            assert abs(np.median(kap) / np.e - 1.0) < 0.1 and kap.min() > np.exp(0.2) and kap.max() < np.exp(1.8)
        g.close()
    assert cos[True].min() > 0.9, cos[True].min()
    assert abs(cos[False].mean()) < 0.2


@pytest.mark.gpu
def test_adam_step_refreshes_the_bf16_operands(ctx):
    """The Adam kernel writes each updated parameter's BF16 operand entries in
    place; they must equal what a full regeneration from the FP32 parameters
    writes: inference after training steps equals, bit for bit, inference
    after the same parameters are set again (which regenerates every entry)."""
    rng = np.random.default_rng(26)
    g = _guide(ctx, seed=11, learning_rate=3e-3, anchor_lobes=True)
    for _ in range(5):
        batch = torch.from_numpy(_target_records(rng, 4096)).cuda()
        mcpt.check(ctx.lib.mc_guide_train(g.handle, batch.data_ptr(), 4096))
    n = 2048
    q = np.zeros((n, 6), np.float32)
    q[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    q[:, 3:6] = _unit(rng, n)
    dq = torch.from_numpy(q).cuda()
    out = [torch.zeros(n * 40, dtype=torch.float32, device="cuda") for _ in range(2)]
    mcpt.check(ctx.lib.mc_guide_infer(g.handle, dq.data_ptr(), n, out[0].data_ptr()))
    g.set_params(g.get_params())
    mcpt.check(ctx.lib.mc_guide_infer(g.handle, dq.data_ptr(), n, out[1].data_ptr()))
    assert out[0].cpu().numpy().tobytes() == out[1].cpu().numpy().tobytes()
    g.close()
