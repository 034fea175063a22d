"""FP32 PyTorch (CPU) reference of the warm-start network with the same BF16
rounding points as the tensor-core kernels: inputs, weights and hidden
activations rounded to BF16, accumulation in FP32, bias in FP32."""
import numpy as np
import torch

LAYERS = ((7, 32), (32, 32), (32, 32), (32, 32), (32, 32), (32, 3))
FIELD_SCALE = 1.0 / 0.05


def param_count():
    return sum(co * 9 * ci + co for ci, co in LAYERS)


def random_params(seed):
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in LAYERS:
        out.append(rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), size=(co, 3, 3, ci)).reshape(-1))
        out.append(rng.normal(0.0, 0.05, size=co))
    return np.concatenate(out).astype(np.float32)


def unpack(params):
    """Flat vector -> list of (W [cout][cin][3][3] torch layout, b [cout])."""
    p = np.asarray(params, dtype=np.float32)
    layers, o = [], 0
    for ci, co in LAYERS:
        w = p[o:o + co * 9 * ci].reshape(co, 3, 3, ci).transpose(0, 3, 1, 2)
        o += co * 9 * ci
        b = p[o:o + co]
        o += co
        layers.append((torch.from_numpy(np.ascontiguousarray(w)), torch.from_numpy(b.copy())))
    return layers


def bf16(x):
    return x.to(torch.bfloat16).to(torch.float32)


def network_input(m, mask, b_ext, ny, nx):
    """m [nimg, ny*nx, 3], mask [nimg, ny*nx] or None, b_ext [nimg, 3] -> [nimg, 7, ny, nx] (FP32)."""
    m = np.asarray(m, dtype=np.float64).reshape(-1, ny * nx, 3)
    nimg = m.shape[0]
    inside = np.ones((nimg, ny * nx)) if mask is None else (np.asarray(mask).reshape(nimg, -1) != 0).astype(float)
    x = np.zeros((nimg, 7, ny * nx), dtype=np.float32)
    x[:, 0:3] = (m * inside[..., None]).transpose(0, 2, 1).astype(np.float32)
    x[:, 3] = inside
    be = np.asarray(b_ext, dtype=np.float64).reshape(nimg, 3)
    x[:, 4:7] = (be.astype(np.float32) * np.float32(FIELD_SCALE))[..., None]
    return torch.from_numpy(x.reshape(nimg, 7, ny, nx)), inside


def forward(params, m, mask, b_ext, ny, nx):
    layers = unpack(params)
    x, inside = network_input(m, mask, b_ext, ny, nx)
    h = bf16(x)
    for li, (w, b) in enumerate(layers):
        y = torch.nn.functional.conv2d(h, bf16(w), bias=None, padding=1) + b.view(1, -1, 1, 1)
        if li < len(layers) - 1:
            h = bf16(torch.relu(y))
        else:
            h = y
    v = h.reshape(h.shape[0], 3, ny * nx).permute(0, 2, 1).numpy().astype(np.float64)
    n = np.linalg.norm(v, axis=2, keepdims=True)
    out = np.where(n > 0, v / np.where(n > 0, n, 1.0), np.array([0.0, 0.0, 1.0]))
    out = out * inside[..., None]
    return out
