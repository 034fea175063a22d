"""Training of the warm-start network by the tensor-core kernels: gradients
against the CPU FP64 restatement (tests/warmstart_ref.py, the same BF16 rounding
points), determinism, loss decrease under Adam, and the bounded-wait error path."""
import numpy as np
import pytest

import warmstart_ref as ref
from helpers import holes_mask

pytestmark = pytest.mark.gpu


def _batch(nimg, ny, nx, seed, holes=True):
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(nimg, ny * nx, 3))
    m /= np.linalg.norm(m, axis=2, keepdims=True)
    t = rng.normal(size=(nimg, ny * nx, 3)) + np.array([0.0, 0.0, 2.0])
    t /= np.linalg.norm(t, axis=2, keepdims=True)
    mask = None
    if holes:
        mask = np.stack([holes_mask(nx, ny, [(nx // 5, -ny // 6, min(nx, ny) // 5)]) for _ in range(nimg)])
        m[mask == 0] = 0.0
        t[mask == 0] = 0.0
    b = rng.uniform(-0.03, 0.03, size=(nimg, 3))
    b[:, 2] = 0.0
    return m, mask, b, t


def _device(m, mask, b, t, ny, nx):
    import torch

    nimg = m.shape[0]
    soa = lambda a: torch.from_numpy(np.ascontiguousarray(  # noqa: E731
        a.reshape(nimg, ny * nx, 3).transpose(0, 2, 1).astype(np.float32))).cuda()
    dm, dt = soa(m), soa(t)
    dk = torch.from_numpy(mask.astype(np.uint8)).cuda() if mask is not None else None
    db = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    return dm, dk, db, dt


def _ptrs(d):
    dm, dk, db, dt = d
    return dm.data_ptr(), (dk.data_ptr() if dk is not None else 0), db.data_ptr(), dt.data_ptr()


@pytest.mark.parametrize("nimg,ny,nx,holes", [(2, 12, 16, True), (1, 24, 40, False), (3, 32, 32, True)])
def test_gradients_match_fp64_restatement(gpu, nimg, ny, nx, holes):
    params = ref.random_params(5)
    m, mask, b, t = _batch(nimg, ny, nx, 17, holes)
    d = _device(m, mask, b, t, ny, nx)
    tr = gpu.WarmStartTrainer(params, nimg * ny * nx)
    loss, g = tr.gradients(nimg, ny, nx, *_ptrs(d))
    loss_ref, g_ref = ref.loss_and_gradient(params, m, mask, b, t, ny, nx)
    assert loss == pytest.approx(loss_ref, rel=1e-5)
    o = 0
    for ci, co in ref.LAYERS:
        for size in (co * 9 * ci, co):
            a, r = g[o:o + size], g_ref[o:o + size]
            o += size
            scale = np.abs(r).max()
            # BF16 intermediate values: an FP32-vs-FP64 difference can move a rounding by one BF16 ulp
            assert np.abs(a - r).max() <= 2e-2 * scale, (ci, co, size)
            assert np.sqrt(((a - r) ** 2).mean()) <= 3e-3 * scale, (ci, co, size)
    cos = float(g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert cos > 0.9999
    # deterministic: the same minibatch gives the same bits
    loss2, g2 = tr.gradients(nimg, ny, nx, *_ptrs(d))
    assert loss2 == loss and np.array_equal(g2, g)
    tr.close()


def test_pipelined_and_oneshot_convolutions_give_the_same_gradients(gpu, monkeypatch):
    ny, nx = 40, 72
    params = ref.random_params(6)
    m, mask, b, t = _batch(2, ny, nx, 8, True)
    d = _device(m, mask, b, t, ny, nx)
    tr = gpu.WarmStartTrainer(params, 2 * ny * nx)
    l1, g1 = tr.gradients(2, ny, nx, *_ptrs(d))
    monkeypatch.setenv("LLG_B200_CONV_ONESHOT", "1")
    l2, g2 = tr.gradients(2, ny, nx, *_ptrs(d))
    monkeypatch.delenv("LLG_B200_CONV_ONESHOT")
    assert l1 == l2 and np.array_equal(g1, g2)
    tr.close()


def test_adam_steps_reduce_the_loss(gpu):
    ny = nx = 32
    params = ref.random_params(8)
    m, mask, b, t = _batch(4, ny, nx, 3, True)
    d = _device(m, mask, b, t, ny, nx)
    tr = gpu.WarmStartTrainer(params, 4 * ny * nx)
    first = tr.step(4, ny, nx, *_ptrs(d), lr=2e-3)
    for _ in range(60):
        last = tr.step(4, ny, nx, *_ptrs(d), lr=2e-3, read_loss=False)
    tr.sync()
    last, _ = tr.gradients(4, ny, nx, *_ptrs(d))
    assert last < 0.8 * first
    p = tr.params()
    assert p.shape == params.shape and np.all(np.isfinite(p)) and not np.array_equal(p, params)
    # the trained parameters run in the inference network
    net = gpu.WarmStartNet(p)
    out = net.forward(m, mask, b, ny, nx).reshape(4, ny * nx, 3)
    ins = mask.reshape(4, -1) != 0
    cos = (out * t).sum(axis=2)[ins].mean()
    assert 1.0 - cos == pytest.approx(last, abs=2e-2)
    net.close()
    tr.close()


def test_timed_out_wait_reports_and_next_call_is_clean(gpu):
    """A spin limit of zero polls makes the tensor-core waits give up at once: the
    call reports LLG_ERR_TIMEOUT (the kernels still wait, bounded, for their MMAs
    before freeing TMEM); with the limit restored the next call succeeds."""
    ny, nx = 16, 16
    params = ref.random_params(2)
    m, mask, b, t = _batch(1, ny, nx, 4, False)
    d = _device(m, mask, b, t, ny, nx)
    tr = gpu.WarmStartTrainer(params, ny * nx)
    loss0, g0 = tr.gradients(1, ny, nx, *_ptrs(d))
    tr.set_spin_limit(0)
    with pytest.raises(gpu.LLGError) as e:
        tr.gradients(1, ny, nx, *_ptrs(d))
    assert e.value.code == -3
    tr.set_spin_limit(1 << 26)
    loss1, g1 = tr.gradients(1, ny, nx, *_ptrs(d))
    assert loss1 == loss0 and np.array_equal(g1, g0)
    tr.close()
    net = gpu.WarmStartNet(params)
    net.set_spin_limit(0)
    with pytest.raises(gpu.LLGError):
        net.forward(m, None, b, ny, nx)
    net.set_spin_limit(1 << 26)
    out = net.forward(m, None, b, ny, nx)
    assert np.all(np.isfinite(out))
    net.close()
