"""Train the learned warm-start network on relaxations computed by this library,
on the GPU, with this library's own tensor-core kernels.

    python llg-sim_b200/warmstart_train.py --films 20000 --out <dir>

1. Data: holey 128x128 films (workloads.holey_film_batch: 0-6 circular holes of
   radius 8-24 cells, D U[0, 2e-3], 0-30 mT in-plane), random unit m0 (zero in
   the holes), relaxed on the GPU by the batched device relax (FP32, max |m x B|
   below --torque; FP32 field round-off puts a floor near 2e-4 T under the
   tightening stages).  The (m0, mask, B_ext) -> relaxed m pairs stay on the GPU.
2. Training: WarmStartTrainer (train_tc.cu): forward and input-gradient
   convolutions and the weight-gradient kernel on the tensor cores (BF16
   operands, FP32 accumulation), loss = mean over film cells of 1 - cos(angle)
   between the normalised output and the relaxed m, Adam on FP32 master weights
   with a cosine learning-rate decay, minibatches drawn by a seeded permutation.
   PyTorch only holds the device arrays (plumbing); no torch operator runs in
   the training loop.
3. Export: the flat FP32 parameter vector in the layout llg_warmstart_create
   takes (per layer W[cout][3][3][cin] then b[cout]) to <out>/warmstart.npy,
   a log and a summary (train / held-out loss per epoch, relax statistics).
"""
import argparse
import json
import math
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


def init_params(seed):
    """He-normal weights, small biases, in the flat layout of llg_warmstart_create."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in LAYERS:
        out.append(rng.normal(0.0, math.sqrt(2.0 / (9 * ci)), size=(co, 3, 3, ci)).reshape(-1))
        out.append(np.zeros(co))
    return np.concatenate(out).astype(np.float32)


def relax_dataset(n, size, seed, chunk, max_steps, torque, log, budget_s=None):
    """Relaxed films, kept on the GPU as they are produced (torch tensors used as
    device arrays): m0 and m_relaxed FP32 SoA [n][3][size*size], masks uint8
    [n][size*size]; B_ext [n][3] and accepted steps [n] on the host.  Host memory
    holds one film at a time.  With budget_s, no new chunk starts after that many
    seconds (the films done so far are returned)."""
    import torch

    films, rx = W.holey_film_batch(n, size, seed=seed)
    hw = size * size
    dev = "cuda"
    m0 = torch.empty((n, 3, hw), dtype=torch.float32, device=dev)
    mrel = torch.empty((n, 3, hw), dtype=torch.float32, device=dev)
    masks = torch.empty((n, hw), dtype=torch.uint8, device=dev)
    bext = np.empty((n, 3))
    steps = np.empty(n, dtype=np.int64)
    t_start = time.time()
    done = 0
    for c0 in range(0, n, chunk):
        if budget_s is not None and time.time() - t_start > budget_s:
            log(f"dataset budget of {budget_s:.0f} s reached after {done} films")
            break
        part = films[c0:c0 + chunk]
        b = L.Batch([f.grid(L) for f in part], [f.material(L) for f in part], L.FP32, masks=[f.mask for f in part])
        for i, f in enumerate(part):
            m = L.init_random(f.n, seed * 1000003 + c0 + i)
            m[f.mask == 0] = 0.0
            b.set_state(i, m)
            m0[c0 + i] = torch.from_numpy(np.ascontiguousarray(m.T, dtype=np.float32))
            masks[c0 + i] = torch.from_numpy(np.ascontiguousarray(f.mask, dtype=np.uint8))
            bext[c0 + i] = f.b_ext
        st = L.RelaxSettings.default(torque_threshold=torque, max_err=rx["max_err"], headroom=rx["headroom"],
                                     dt_min=rx["dt_min"], dt_max=rx["dt_max"], max_accepted_steps=max_steps)
        P = [L.LLGParams(W.GAMMA, f.alpha, rx["dt0"], f.b_ext) for f in part]
        t0 = time.time()
        reps = b.relax(P, L.FULL, st)
        for i in range(len(part)):
            mrel[c0 + i] = torch.from_numpy(np.ascontiguousarray(b.get_state(i).T, dtype=np.float32))
            steps[c0 + i] = reps[i].accepted_steps
        s = steps[c0:c0 + len(part)]
        log(f"relaxed films {c0}..{c0 + len(part) - 1} in {time.time() - t0:.1f} s, steps {int(s.mean())} mean / "
            f"{int(s.max())} max, {int((s >= max_steps).sum())} at the cap")
        b.close()
        done = c0 + len(part)
    return m0[:done], masks[:done], bext[:done], mrel[:done], steps[:done]


def train(data, size, epochs, batch, lr, log, seed=0, holdout=0.02, params=None):
    import torch

    d_m0, d_k, bext, d_t, _ = data
    n = d_m0.shape[0]
    dev = "cuda"
    d_b = torch.from_numpy(np.ascontiguousarray(bext, dtype=np.float64)).to(dev)
    inside = d_k.sum(dim=1).cpu().numpy().astype(np.float64)   # film cells per film
    rng = np.random.default_rng(seed)
    order = rng.permutation(n)
    n_hold = max(1, int(round(holdout * n))) if n > 8 else 0
    hold, train_idx = order[:n_hold], order[n_hold:]
    hw = size * size
    p0 = init_params(seed + 1) if params is None else params
    tr = L.WarmStartTrainer(p0, batch * hw)
    # minibatch buffers (gathered on the device by index)
    bm0 = torch.empty((batch, 3, hw), dtype=torch.float32, device=dev)
    bt = torch.empty_like(bm0)
    bk = torch.empty((batch, hw), dtype=torch.uint8, device=dev)
    bb = torch.empty((batch, 3), dtype=torch.float64, device=dev)

    def gather(idx):
        ii = torch.from_numpy(np.asarray(idx, dtype=np.int64)).to(dev)
        k = len(idx)
        torch.index_select(d_m0, 0, ii, out=bm0[:k])
        torch.index_select(d_t, 0, ii, out=bt[:k])
        torch.index_select(d_k, 0, ii, out=bk[:k])
        torch.index_select(d_b, 0, ii, out=bb[:k])
        return k, (bm0.data_ptr(), bk.data_ptr(), bb.data_ptr(), bt.data_ptr())

    def held_out_loss():
        if n_hold == 0:
            return None
        tot = cells = 0.0
        for b0 in range(0, n_hold, batch):
            idx = hold[b0:b0 + batch]
            k, ptrs = gather(idx)
            loss, _ = tr.gradients(k, size, size, *ptrs)
            c = float(inside[idx].sum())
            tot += loss * c
            cells += c
        return tot / max(cells, 1.0)

    steps_per_epoch = (len(train_idx) + batch - 1) // batch
    total = epochs * steps_per_epoch
    hist = []
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = rng.permutation(train_idx)
        tot = 0.0
        cnt = 0
        for b0 in range(0, len(perm), batch):
            idx = perm[b0:b0 + batch]
            k, ptrs = gather(idx)
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
            read = (b0 // batch) % 25 == 0
            loss = tr.step(k, size, size, *ptrs, lr=cur, read_loss=read)
            if read:
                tot += loss
                cnt += 1
            step += 1
        tr.sync()
        hl = held_out_loss()
        hist.append({"epoch": ep, "train_loss": tot / max(cnt, 1), "held_out_loss": hl,
                     "seconds": time.time() - t0})
        log(f"epoch {ep}: train loss {hist[-1]['train_loss']:.5f}, held-out loss {hl}, {time.time() - t0:.1f} s")
    params = tr.params()
    tr.close()
    return params, hist, {"train_films": int(len(train_idx)), "held_out_films": int(n_hold), "steps": step}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--films", type=int, default=20000)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--chunk", type=int, default=2048)
    ap.add_argument("--max-steps", type=int, default=30000)
    ap.add_argument("--torque", type=float, default=1e-3)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--init", default=None, help="start from these parameters (.npy) instead of a fresh draw")
    ap.add_argument("--data-budget", type=float, default=None, help="seconds after which no new relax chunk starts")
    ap.add_argument("--drop-capped", action="store_true", help="train only on films that reached the torque")
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    logf = open(os.path.join(args.out, "train_log.txt"), "w")

    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    t0 = time.time()
    data = relax_dataset(args.films, args.size, args.seed, args.chunk, args.max_steps, args.torque, log,
                         args.data_budget)
    t_data = time.time() - t0
    n_rel = len(data[4])
    log(f"dataset: {n_rel} films relaxed in {t_data:.1f} s")
    steps_all = data[4]
    if args.drop_capped:
        import torch

        keep = steps_all < args.max_steps
        kt = torch.from_numpy(np.nonzero(keep)[0]).to("cuda")
        m0, masks, bext, mrel, st = data
        data = (m0[kt], masks[kt], bext[keep], mrel[kt], st[keep])
        log(f"training on {int(keep.sum())} films that reached the torque ({int((~keep).sum())} at the cap dropped)")
    init = np.load(args.init) if args.init else None
    t1 = time.time()
    params, hist, info = train(data, args.size, args.epochs, args.batch, args.lr, log, seed=args.seed, params=init)
    assert params.size == L.WarmStartNet.param_count()
    np.save(os.path.join(args.out, "warmstart.npy"), params)
    log(f"training: {time.time() - t1:.1f} s, final train loss {hist[-1]['train_loss']:.5f}")
    steps = steps_all
    json.dump({"films_requested": args.films, "films": n_rel, "films_trained": int(len(data[4])), "size": args.size, "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
               "torque_threshold": args.torque, "max_steps": args.max_steps, "history": hist, **info,
               "relax_steps_mean": float(steps.mean()), "relax_steps_max": int(steps.max()),
               "relax_at_cap": int((steps >= args.max_steps).sum()), "dataset_seconds": t_data,
               "training_seconds": time.time() - t1, "trainer": "llg_wstrain (tcgen05 forward / input-gradient / "
                                                                 "weight-gradient kernels, Adam on the device)"},
              open(os.path.join(args.out, "train_summary.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
