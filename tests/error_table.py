"""Errors of the GPU path against the FP64 oracle for every benchmark configuration.

For each configuration (c1 .. c5 of the benchmark workloads, restated in
llg-sim_b200/workloads.py) and each GPU precision this measures, through the C
ABI, against the CPU FP64 oracle on the same seeded inputs:

* H_demag at the initial state: max |dB| / max |B_ref| and RMS(dB) / RMS(B_ref);
* m after K integrator steps taken with one dt sequence: the oracle first runs
  the configuration's own controller to collect K accepted step sizes, then the
  oracle and the GPU both replay exactly those steps (max_err set out of reach,
  so every replayed attempt is accepted): max |dm| and RMS |dm|;
* total energy of the final states: |E_gpu - E_ref| / |E_ref|.

Run as a script on a GPU host to print the markdown table (and --json PATH for
the record); the c2 row at full size is also asserted by
tests/test_gpu_c2_parity.py.  Only test code imports the oracle.
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (ROOT, os.path.join(ROOT, "llg-sim_b200"), HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)

GAMMA = 1.76085963023e11
NEVER_REJECT = 1e300


def field_err(b, ref):
    b = np.asarray(b, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    d = b - ref
    return {"max": float(np.abs(d).max() / max(np.abs(ref).max(), 1e-300)),
            "rms": float(np.sqrt((d * d).mean()) / max(np.sqrt((ref * ref).mean()), 1e-300))}


def state_err(m, ref):
    d = np.asarray(m, dtype=np.float64) - np.asarray(ref, dtype=np.float64)
    return {"max": float(np.abs(d).max()), "rms": float(np.sqrt((d * d).sum(axis=1).mean()))}


def oracle_dts(O, osv, m0, po, kind, fmask, ctl, k_acc, max_attempts=400):
    """The configuration's own controller on the oracle: the first k_acc accepted dt."""
    m = m0.copy()
    osv.invalidate()
    dts = []
    step = osv.step_rk45 if kind == "rk45" else osv.step_rk23_relax
    for _ in range(max_attempts):
        _, a, dtu = step(m, po, fmask, *ctl)
        if a:
            dts.append(dtu)
            if len(dts) == k_acc:
                break
    return dts


def replay(L, O, osv, gsv, m0, gamma, alpha, bext, kind, fmask, dts):
    """Both engines take exactly the steps dts (all accepted); returns their final states."""
    m = m0.copy()
    osv.invalidate()
    gsv.set_state(m0)
    po = O.make_params(gamma, alpha, dts[0], bext)
    pg = L.LLGParams(gamma, alpha, dts[0], bext)
    args = (NEVER_REJECT, 0.8, 1e-30, 1.0)
    ostep = osv.step_rk45 if kind == "rk45" else osv.step_rk23_relax
    gstep = gsv.step_rk45 if kind == "rk45" else gsv.step_rk23_relax
    for dt in dts:
        po.dt = dt
        pg.dt = dt
        _, ao, _ = ostep(m, po, fmask, *args)
        _, ag, _ = gstep(pg, fmask, *args)
        assert ao and ag
    return m, gsv.get_state()


def run_config(L, O, name, film, m0, kind, ctl, k_acc, precisions=(0, 1), fmask=2):
    """Errors of one configuration for each GPU precision (0 = FP32, 1 = FP64)."""
    og = O.make_grid(film.nx, film.ny, film.dx, film.dy, film.dz)
    om = O.make_material(film.ms, film.a_ex, film.k_u, film.easy, film.dmi, film.demag)
    osv = O.Solver(og, om, film.mask)
    po = O.make_params(GAMMA, film.alpha, ctl["dt0"], film.b_ext)
    dts = oracle_dts(O, osv, m0, po, kind, fmask,
                     (ctl["max_err"], ctl["headroom"], ctl["dt_min"], ctl["dt_max"]), k_acc)
    b_ref = osv.demag_field(m0)
    out = {"config": name, "cells": film.n, "steps": len(dts), "kind": kind}
    m_ref = None
    for prec in precisions:
        gsv = L.Solver(film.grid(L), film.material(L), prec, film.mask)
        gsv.set_state(m0)
        b = gsv.compute_demag_field()
        m_ref, m_gpu = replay(L, O, osv, gsv, m0, GAMMA, film.alpha, film.b_ext, kind, fmask, dts)
        er = osv.energy(m_ref, film.b_ext)
        eg = gsv.compute_energy(film.b_ext)
        e_ref, e_gpu = er.total(), eg.total()
        terms = {t: {"ref_J": getattr(er, t), "abs_err_J": abs(getattr(eg, t) - getattr(er, t))}
                 for t in ("exchange", "anisotropy", "zeeman", "dmi", "demag")}
        out["fp64" if prec else "fp32"] = {"h_demag": field_err(b, b_ref), "m": state_err(m_gpu, m_ref),
                                           "energy_rel": abs(e_gpu - e_ref) / max(abs(e_ref), 1e-300),
                                           "energy_J": e_ref, "energy_terms": terms}
        gsv.close()
    osv.close()
    return out


def configs(full=True):
    """(name, film, m0, kind, controller, accepted steps) for c1 .. c5."""
    import workloads as W
    import llg_b200 as L

    out = []
    f, rx, run = W.film_128x32_relax_then_field()
    out.append(("c1 relax (RK23) 128x32", f, f.m0, "rk23", dict(rx), 20))
    f1 = W.Film(f.nx, f.ny, f.dx, f.dy, f.dz, f.ms, f.a_ex, demag=True, b_ext=f.b_ext, alpha=run["alpha"])
    out.append(("c1 field run (RK45) 128x32", f1, f.m0, "rk45", dict(run), 20))
    f2, seed, run2 = W.film_1024_dmi() if full else W.film_1024_dmi(256, 256)
    out.append((f"c2 {f2.nx}x{f2.ny} RK45", f2, L.init_random(f2.n, seed), "rk45", dict(run2), 3))
    films, run3 = W.mixed_film_batch(256)
    for want in (96, 192, 128, 256):   # radix-3 lengths and register-FFT lengths
        i, fm = next((i, fm) for i, fm in enumerate(films) if fm.nx == want)
        out.append((f"c3 film {i} {fm.nx}x{fm.ny} RK45", fm,
                    L.init_uniform_with_noise(fm.n, (1.0, 0.0, 0.0), run3["noise"], 1000 + i), "rk45", dict(run3), 10))
    for size, tag in ((128, "c4"), (256, "c5")):
        hf, rx4 = W.holey_film_batch(1, size, seed=77)
        fm = hf[0]
        m = L.init_random(fm.n, 900000)
        m[fm.mask == 0] = 0.0
        out.append((f"{tag} holey {size}x{size} relax (RK23)", fm, m, "rk23", dict(rx4), 10))
    return out


def table(rows):
    head = ("| config | steps | prec | H_demag max | H_demag RMS | m max | m RMS | E rel |\n"
            "|---|---:|---|---:|---:|---:|---:|---:|")
    lines = [head]
    for r in rows:
        for p in ("fp32", "fp64"):
            if p not in r:
                continue
            e = r[p]
            lines.append(f"| {r['config']} | {r['steps']} | {p.upper()} | {e['h_demag']['max']:.2e} | "
                         f"{e['h_demag']['rms']:.2e} | {e['m']['max']:.2e} | {e['m']['rms']:.2e} | "
                         f"{e['energy_rel']:.2e} |")
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--json", default=None)
    ap.add_argument("--small", action="store_true", help="c2 at 256x256 instead of 1024x1024")
    args = ap.parse_args()
    import llg_b200 as L
    import oracle as O

    O.set_threads(os.cpu_count() or 1)
    rows = []
    for name, film, m0, kind, ctl, k in configs(full=not args.small):
        rows.append(run_config(L, O, name, film, m0, kind, ctl, k))
        print(json.dumps(rows[-1]), flush=True)
    print(table(rows))
    if args.json:
        with open(args.json, "w") as fh:
            json.dump(rows, fh, indent=1)


if __name__ == "__main__":
    main()
