"""The committed record of the learned warm start's held-out evaluation
(pot3d_b200/weights/fno_pfss_127x181x361.json, written by
python -m pot3d_b200.warmstart on one B200): the protocol of the learned
configuration -- 2000 training pairs at 127x181x361 solved to 1e-9, 200
held-out seeds -- and what it recorded for every held-out seed."""
import json
import os

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
WEIGHTS = os.path.join(ROOT, "pot3d_b200", "weights", "fno_pfss_127x181x361")


def test_recorded_held_out_evaluation():
    """The committed 200-seed record of the operator: the C4 protocol (2000
    training pairs solved to 1e-9, 200 held-out seeds) and a gain on every
    held-out seed's iteration count."""
    with open(WEIGHTS + ".json") as fh:
        rec = json.load(fh)
    assert rec["config"]["train"] == 2000 and rec["config"]["test"] == 200
    assert rec["config"]["train_eps"] <= 1e-9
    ev = rec["evaluation"]
    assert ev["cases"] == 200 and len(rec["cases"]) == 200
    assert ev["iteration_ratio"] < 1.0 and ev["fewer_iterations_cases"] == 200
    assert ev["sol_rel_diff_max"] < 1e-7
