"""Train the learned warm-start network on relaxations computed by this library.

    python llg-sim_b200/warmstart_train.py --films 256 --out <dir>

1. Data: holey 128x128 films (workloads.holey_film_batch: 0-6 circular holes,
   D U[0, 2e-3], 0-30 mT in-plane), random unit m0, relaxed on the GPU with the
   batched device relax (FP32, max |m x B| below 1e-3 T; FP32 field round-off
   puts a floor near 2e-4 T under the tightening stages).
2. Training: the network of conv_tc.cu (six 3x3 convolutions, 32 channels, ReLU)
   in PyTorch with BF16 autocast, loss = mean over film cells of 1 - cos(angle)
   between the normalised output and the relaxed m.
3. Export: the flat FP32 parameter vector in the layout llg_warmstart_create
   takes (per layer W[cout][3][3][cin] then b[cout]) to <out>/warmstart.npy,
   a training log and summary (and the dataset with --save-dataset).

The tensor-core kernels run the exported network; PyTorch is used here only as
the offline training tool.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import llg_b200 as L  # noqa: E402
import workloads as W  # noqa: E402

LAYERS = ((7, 32), (32, 32), (32, 32), (32, 32), (32, 32), (32, 3))
FIELD_SCALE = 1.0 / 0.05


def relax_dataset(n, size, seed, chunk, max_steps, log):
    films, rx = W.holey_film_batch(n, size, seed=seed)
    m0s, masks, bexts, mrel, steps = [], [], [], [], []
    for c0 in range(0, n, chunk):
        part = films[c0:c0 + chunk]
        b = L.Batch([f.grid(L) for f in part], [f.material(L) for f in part], L.FP32, masks=[f.mask for f in part])
        for i, f in enumerate(part):
            m = L.init_random(f.n, seed * 100000 + c0 + i)
            m[f.mask == 0] = 0.0
            b.set_state(i, m)
            m0s.append(m)
            masks.append(f.mask)
            bexts.append(f.b_ext)
        st = L.RelaxSettings.default(torque_threshold=1e-3, max_err=rx["max_err"], headroom=rx["headroom"],
                                     dt_min=rx["dt_min"], dt_max=rx["dt_max"], max_accepted_steps=max_steps)
        P = [L.LLGParams(W.GAMMA, f.alpha, rx["dt0"], f.b_ext) for f in part]
        t0 = time.time()
        reps = b.relax(P, L.FULL, st)
        for i in range(len(part)):
            mrel.append(b.get_state(i))
            steps.append(reps[i].accepted_steps)
        log(f"relaxed films {c0}..{c0 + len(part) - 1} in {time.time() - t0:.1f} s, steps "
            f"{int(np.mean(steps[-len(part):]))} mean / {int(np.max(steps[-len(part):]))} max")
        b.close()
    return (np.stack(m0s), np.stack(masks), np.array(bexts), np.stack(mrel), np.array(steps))


def to_input(m0, mask, bext, size):
    import torch

    n = m0.shape[0]
    inside = (mask != 0).astype(np.float32)
    x = np.zeros((n, 7, size * size), dtype=np.float32)
    x[:, 0:3] = (m0 * inside[..., None]).transpose(0, 2, 1)
    x[:, 3] = inside
    x[:, 4:7] = (bext.astype(np.float32) * np.float32(FIELD_SCALE))[..., None]
    return torch.from_numpy(x.reshape(n, 7, size, size))


def build_model():
    import torch.nn as nn

    mods = []
    for li, (ci, co) in enumerate(LAYERS):
        mods.append(nn.Conv2d(ci, co, 3, padding=1))
        if li < len(LAYERS) - 1:
            mods.append(nn.ReLU())
    return nn.Sequential(*mods)


def export_params(model):
    import torch.nn as nn

    out = []
    for mod in model:
        if isinstance(mod, nn.Conv2d):
            w = mod.weight.detach().float().cpu().numpy()          # [cout][cin][3][3]
            out.append(w.transpose(0, 2, 3, 1).reshape(-1))        # -> [cout][3][3][cin]
            out.append(mod.bias.detach().float().cpu().numpy())
    return np.concatenate(out).astype(np.float32)


def train(data, size, epochs, batch, lr, log, seed=0):
    import torch

    torch.manual_seed(seed)
    m0, mask, bext, mrel, _ = data
    x = to_input(m0, mask, bext, size)
    y = torch.from_numpy(mrel.astype(np.float32).transpose(0, 2, 1).reshape(-1, 3, size, size))
    w = torch.from_numpy((mask != 0).astype(np.float32).reshape(-1, 1, size, size))
    dev = "cuda"
    x, y, w = x.to(dev), y.to(dev), w.to(dev)
    model = build_model().to(dev)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    n = x.shape[0]
    steps = epochs * ((n + batch - 1) // batch)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, device=dev)
        tot = 0.0
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            with torch.autocast("cuda", dtype=torch.bfloat16):
                out = model(x[idx])
            out = out.float()
            out = out / (out.norm(dim=1, keepdim=True) + 1e-12)
            cos = (out * y[idx]).sum(dim=1, keepdim=True)
            loss = ((1.0 - cos) * w[idx]).sum() / w[idx].sum().clamp(min=1.0)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            tot += float(loss) * len(idx)
        hist.append(tot / n)
        log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return model, hist


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--films", type=int, default=256)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--chunk", type=int, default=128)
    ap.add_argument("--max-steps", type=int, default=40000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--out", required=True)
    ap.add_argument("--save-dataset", action="store_true")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    logf = open(os.path.join(args.out, "train_log.txt"), "w")

    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    t0 = time.time()
    data = relax_dataset(args.films, args.size, args.seed, args.chunk, args.max_steps, log)
    if args.save_dataset:
        np.savez_compressed(os.path.join(args.out, "dataset.npz"), m0=data[0].astype(np.float32), mask=data[1],
                            bext=data[2], m_relaxed=data[3].astype(np.float32), steps=data[4])
    log(f"dataset: {args.films} films in {time.time() - t0:.1f} s")
    t1 = time.time()
    model, hist = train(data, args.size, args.epochs, args.batch, args.lr, log)
    params = export_params(model)
    assert params.size == L.WarmStartNet.param_count()
    np.save(os.path.join(args.out, "warmstart.npy"), params)
    log(f"training: {time.time() - t1:.1f} s, final loss {hist[-1]:.5f}")
    json.dump({"films": args.films, "size": args.size, "epochs": args.epochs, "loss": hist,
               "relax_steps_mean": float(np.mean(data[4])), "seconds": time.time() - t0},
              open(os.path.join(args.out, "train_summary.json"), "w"))


if __name__ == "__main__":
    main()
