"""The benchmark film itself (1024x1024, 2 nm cubes, Ku 8e5, D 3e-3, random m0,
demag on) against the CPU FP64 oracle, through the C ABI: H_demag at the initial
state, and m and the total energy after three RK45 steps that both engines take
with the same step sizes (the oracle's own controller picks them first).

Tolerances are the measured errors with a margin (measured on B200: FP32 H_demag
3.2e-7 max / 2.2e-7 RMS, m 3.3e-7, E 7.0e-8; FP64 1.3e-13 / 1.3e-13, 1.2e-15,
3.4e-15): FP32 carries single-precision round-off of the 2048^2 padded
transforms; FP64 matches to round-off."""
import pytest

from error_table import run_config

pytestmark = pytest.mark.gpu

# (H_demag max, H_demag RMS, m max, E rel) per precision
TOL = {"fp32": (2e-6, 1e-6, 2e-6, 1e-6), "fp64": (1e-11, 1e-11, 1e-13, 1e-12)}


def test_benchmark_film_matches_oracle(orc, gpu):
    import workloads as W

    film, seed, run = W.film_1024_dmi()
    m0 = gpu.init_random(film.n, seed)
    r = run_config(gpu, orc, "c2", film, m0, "rk45", dict(run), 3)
    assert r["steps"] == 3
    for p, (hmax, hrms, mmax, erel) in TOL.items():
        e = r[p]
        assert e["h_demag"]["max"] <= hmax, (p, e)
        assert e["h_demag"]["rms"] <= hrms, (p, e)
        assert e["m"]["max"] <= mmax, (p, e)
        assert e["energy_rel"] <= erel, (p, e)
