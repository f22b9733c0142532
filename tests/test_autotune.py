"""Team-size tuning table (titus_b200.autotune): keys by problem shape and GPU,
records the best measured team, and lookup returns it. The measurement itself
(tune) needs a GPU and is exercised by `python -m titus_b200.autotune`."""
import json

from titus_b200 import autotune


class FakeSettings:
    NCellsX = NCellsY = 128
    r = 60


class FakeSolver:
    settings = FakeSettings()
    N = 484
    q = 16


def test_record_and_lookup(tmp_path):
    path = str(tmp_path / "batched.json")
    sv = FakeSolver()
    assert autotune.lookup(sv, path, gpu_name="B200") is None
    import torch  # noqa: F401  (shape_key asks torch for the GPU name only when none is given)

    tab = {}
    key = autotune.shape_key(sv, "B200")
    assert key == "128x128_N484_q16_cap60|B200"
    tab[key] = {"team_ctas": 2, "spot_iterations_per_s": {"1": 10.0, "2": 12.0}, "probe": "x"}
    with open(path, "w") as f:
        json.dump(tab, f)
    assert autotune.lookup(sv, path, gpu_name="B200") == 2
    assert autotune.lookup(sv, path, gpu_name="H100") is None
