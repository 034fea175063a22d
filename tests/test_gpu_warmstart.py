"""Learned warm start on the tensor cores against the FP32 PyTorch reference."""
import numpy as np
import pytest

import warmstart_ref as ref
from helpers import case, holes_mask

pytestmark = pytest.mark.gpu


def _inputs(nimg, ny, nx, seed, holes=True):
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(nimg, ny * nx, 3))
    m /= np.linalg.norm(m, axis=2, keepdims=True)
    mask = None
    if holes:
        mask = np.stack([holes_mask(nx, ny, [(nx // 5, ny // 6, min(nx, ny) // 5)]) for _ in range(nimg)])
    b = rng.uniform(-0.03, 0.03, size=(nimg, 3))
    b[:, 2] = 0.0
    return m, mask, b


@pytest.mark.parametrize("nimg,ny,nx,holes", [(2, 32, 48, True), (1, 20, 20, False), (3, 128, 128, True)])
def test_forward_matches_reference(gpu, nimg, ny, nx, holes):
    params = ref.random_params(7)
    net = gpu.WarmStartNet(params)
    m, mask, b = _inputs(nimg, ny, nx, 11, holes)
    out = net.forward(m, mask, b, ny, nx).reshape(nimg, ny * nx, 3)
    exp = ref.forward(params, m, mask, b, ny, nx)
    d = np.abs(out - exp)
    # BF16 hidden activations: accumulation-order differences can move a rounding by one BF16 ulp
    assert d.max() < 3e-2
    assert d.mean() < 2e-3
    if mask is not None:
        assert np.all(out[mask.reshape(nimg, -1) == 0] == 0.0)
        ins = mask.reshape(nimg, -1) != 0
        assert np.allclose(np.linalg.norm(out[ins], axis=1), 1.0, atol=1e-6)
    net.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_warm_start_equals_forward(gpu, prec):
    params = ref.random_params(3)
    net = gpu.WarmStartNet(params)
    ny = nx = 64
    m, mask, b = _inputs(2, ny, nx, 5, True)
    cases = [case(nx, ny, mask=mask[i]) for i in range(2)]
    grids = [gpu.Grid2D(nx, ny, c["dx"], c["dy"], c["dz"]) for c in cases]
    mats = [gpu.Material(c["ms"], c["a_ex"], c["k_u"], c["easy"], c["dmi"], c["demag"]) for c in cases]
    bt = gpu.Batch(grids, mats, prec, masks=[mask[0], mask[1]])
    for i in range(2):
        mi = m[i].copy()
        mi[mask[i] == 0] = 0.0
        bt.set_state(i, mi)
        m[i] = mi
    bt.warm_start(net, b)
    exp = net.forward(m, mask, b, ny, nx).reshape(2, ny * nx, 3)
    for i in range(2):
        got = bt.get_state(i)
        assert np.abs(got - exp[i]).max() < 1e-6
    bt.close()
    net.close()


def test_param_count_and_bad_size(gpu):
    assert gpu.WarmStartNet.param_count() == ref.param_count()
    with pytest.raises(gpu.LLGError):
        gpu.WarmStartNet(np.zeros(ref.param_count() - 1, dtype=np.float32))


def test_trained_warm_start_shortens_relax(gpu):
    """The committed network (trained on relaxed 128x128 holey films) proposes states
    that relax in fewer steps than the random starts they were computed from."""
    import os
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "llg-sim_b200"))
    import workloads as W

    net = gpu.WarmStartNet(np.load(os.path.join(root, "llg-sim_b200", "weights", "warmstart_holey128.npy")))
    films, rx = W.holey_film_batch(6, 128, seed=4321)
    steps = {}
    for learned in (False, True):
        b = gpu.Batch([f.grid(gpu) for f in films], [f.material(gpu) for f in films], gpu.FP32,
                      masks=[f.mask for f in films])
        for i, f in enumerate(films):
            m = gpu.init_random(f.n, 31 + i)
            m[f.mask == 0] = 0.0
            b.set_state(i, m)
        if learned:
            b.warm_start(net, [f.b_ext for f in films])
            for i, f in enumerate(films):
                mi = b.get_state(i)
                assert np.all(mi[f.mask == 0] == 0.0)
                assert np.allclose(np.linalg.norm(mi[f.mask != 0], axis=1), 1.0, atol=1e-6)
        st = gpu.RelaxSettings.default(torque_threshold=1e-3, max_err=rx["max_err"], headroom=rx["headroom"],
                                       dt_min=rx["dt_min"], dt_max=rx["dt_max"], max_accepted_steps=60000)
        reps = b.relax([gpu.LLGParams(W.GAMMA, f.alpha, rx["dt0"], f.b_ext) for f in films], gpu.FULL, st)
        assert all(r.stop_reason == 2 for r in reps)
        steps[learned] = sum(r.accepted_steps for r in reps)
        b.close()
    net.close()
    assert steps[True] < steps[False]


@pytest.mark.parametrize("nimg,ny,nx", [(3, 128, 128), (2, 37, 200), (1, 9, 256)])
def test_pipelined_convolution_gives_the_same_bits(gpu, monkeypatch, nimg, ny, nx):
    """The persistent, halo-staged convolution (images up to 256 cells wide) and the
    one-shot kernel (LLG_B200_CONV_ONESHOT=1) issue the same MMAs on the same
    operands: identical proposals."""
    params = ref.random_params(9)
    net = gpu.WarmStartNet(params)
    m, mask, b = _inputs(nimg, ny, nx, 21, True)
    piped = net.forward(m, mask, b, ny, nx)
    monkeypatch.setenv("LLG_B200_CONV_ONESHOT", "1")
    oneshot = net.forward(m, mask, b, ny, nx)
    monkeypatch.delenv("LLG_B200_CONV_ONESHOT")
    assert np.array_equal(piped, oneshot)
    net.close()
