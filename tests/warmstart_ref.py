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


def bf16_64(x):
    """Round FP64 values to BF16 (round to nearest even) and back to FP64."""
    return x.to(torch.float32).to(torch.bfloat16).to(torch.float64)


def loss_and_gradient(params, m0, mask, b_ext, target, ny, nx):
    """CPU FP64 restatement of one training backprop of the tensor-core kernels:
    the same BF16 rounding points (input, weights, hidden activations, the loss
    gradient and every input gradient), every sum in FP64.  m0 / target
    [nimg, ny*nx, 3], mask [nimg, ny*nx] or None, b_ext [nimg, 3].  Returns the
    mean cosine loss over film cells and its gradient in the flat parameter
    layout (W[cout][3][3][cin] then b[cout] per layer)."""
    F = torch.nn.functional
    p = np.asarray(params, dtype=np.float32)
    ws, bs, o = [], [], 0
    for ci, co in LAYERS:
        w = p[o:o + co * 9 * ci].reshape(co, 3, 3, ci).transpose(0, 3, 1, 2)
        o += co * 9 * ci
        ws.append(bf16_64(torch.from_numpy(np.ascontiguousarray(w)).to(torch.float64)))
        bs.append(torch.from_numpy(p[o:o + co].astype(np.float64)))
        o += co
    x, inside = network_input(m0, mask, b_ext, ny, nx)
    nimg = x.shape[0]
    acts = [bf16_64(x.to(torch.float64))]
    for li in range(len(LAYERS)):
        y = F.conv2d(acts[-1], ws[li], padding=1) + bs[li].view(1, -1, 1, 1)
        acts.append(bf16_64(torch.relu(y)) if li < len(LAYERS) - 1 else y)
    v = acts[-1]                                                    # [nimg, 3, ny, nx]
    t = torch.from_numpy(np.asarray(target, dtype=np.float32).reshape(nimg, ny, nx, 3).transpose(0, 3, 1, 2)
                         .astype(np.float64))
    ins = torch.from_numpy(inside.reshape(nimg, 1, ny, nx))
    n = torch.sqrt((v * v).sum(dim=1, keepdim=True))
    u = v / torch.where(n > 0, n, torch.ones_like(n))
    c = (u * t).sum(dim=1, keepdim=True)
    count = float(ins.sum())
    loss = float(((1.0 - torch.where(n > 0, c, torch.zeros_like(c))) * ins).sum()) / count
    g = torch.where(n > 0, -(t - c * u) / torch.where(n > 0, n, torch.ones_like(n)), torch.zeros_like(v)) * ins
    g = bf16_64(g)
    grads = [None] * len(LAYERS)
    for li in range(len(LAYERS) - 1, -1, -1):
        a = acts[li]
        dw = torch.nn.grad.conv2d_weight(a, ws[li].shape, g, padding=1)      # [cout][cin][3][3]
        db = g.sum(dim=(0, 2, 3))
        grads[li] = (dw, db)
        if li > 0:
            gi = F.conv_transpose2d(g, ws[li], padding=1)
            g = bf16_64(gi * (acts[li] > 0))
    out = []
    for (dw, db) in grads:
        out.append(dw.permute(0, 2, 3, 1).reshape(-1).numpy() / count)
        out.append(db.numpy() / count)
    return loss, np.concatenate(out)
