"""Host logic of the benchmark record (CPU): both arms carry the same config
object, the per-leg summaries stay short, and the two CPU-baseline threading
variants of the oracle give identical results."""
import json

import numpy as np

import bench


def test_both_arms_share_the_config_object():
    a, b = bench.config_dict(1), bench.config_dict(1)
    assert a == b
    assert a["global_cells"] == a["cells_per_gpu"] == 1024 * 1024
    assert bench.config_dict(4)["global_cells"] == 4 * 1024 * 1024


def test_compact_legs_are_short_and_rounded():
    warm = {"workload": "w" * 500, "weights": "x", "plain": {"wall_s": 23.456789, "fp32_stage_s": 10.0},
            "learned": {"wall_s": 7.123456}, "speedup_total": 3.3333333,
            "films": [{"film": i, "energy_rel_diff": 1e-9, "fallback": False} for i in range(256)]}
    out = bench.compact_legs({"value": 7.123456e8, "ms": 6000.123, "accepted_mean": 1614.2, "rejected": 1},
                             None, warm, None, None, None)
    assert "workload" not in out["warm_start_c5"]
    assert "films" not in out["warm_start_c5"]   # the per-film table goes to --detail only
    assert out["batch_c3"]["value"] == 7.123e8
    assert len(json.dumps(out)) < 400


def test_cpu_variants_give_identical_results(orc):
    nx, ny = 48, 40
    g = orc.make_grid(nx, ny, 2e-9, 2e-9, 2e-9)
    mat = orc.make_material(5.8e5, 1.5e-11, 8e5, (0, 0, 1), 3e-3, True)
    res = []
    for par in (False, True):
        orc.set_parallel_local(par)
        s = orc.Solver(g, mat)
        m = orc.init_random(nx * ny, 1)
        p = orc.make_params(1.76085963023e11, 0.3, 1e-14, (0.0, 0.0, 0.0))
        for _ in range(3):
            s.step_rk45(m, p, 2, 1e-5, 0.8, 1e-18, 1e-11)
        res.append(m.copy())
    orc.set_parallel_local(False)
    assert np.array_equal(res[0], res[1])
    assert set(bench.CPU_VARIANTS) == {"reference-threading", "fully-parallel"}
