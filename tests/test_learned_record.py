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


def test_radial_resampling_weights():
    """The operator runs on other grids with its radial levels (the training
    mesh's) interpolated linearly onto the solver mesh's, in the radius
    normalised between the boundaries: exact for a field linear in that
    coordinate, interior levels interpolated, the outermost extrapolated."""
    import numpy as np
    from pot3d_b200 import host
    from pot3d_b200.fno import radial_weights
    src = host.make_mesh(127, 5, 8)
    for nr, r1 in ((255, 2.5), (511, 2.5), (63, 2.5), (95, 2.7)):
        dst = host.make_mesh(nr, 5, 8, r1=r1)
        idx, w = radial_weights(src.rh, dst.rh, dst.r[0], dst.r[-1])
        assert len(idx) == nr - 2 and idx.min() >= 0 and idx.max() <= 123

        def lin(m):
            s = (m.rh[1:-1] - m.r[0]) / (m.r[-1] - m.r[0])
            return 3.0 * s - 0.25
        o = lin(src)
        got = o[idx] + w * (o[idx + 1] - o[idx])
        assert np.max(np.abs(got - lin(dst))) < 1e-13
        # only levels beyond the source's outermost ones (at the two ends) extrapolate
        inner = np.flatnonzero((w >= 0.0) & (w <= 1.0))
        assert np.all(np.diff(inner) == 1) and inner[0] <= 2 and inner[-1] >= len(w) - 3


def test_recorded_evaluation_on_the_headline_grid():
    """The committed evaluation of the same operator run on the 255x361x721
    grid (python -m pot3d_b200.warmstart --nr 255 --nt 361 --np 721 --test
    20 --evaluate ...): 20 held-out seeds, the radial levels resampled, fewer
    iterations on every seed, guesses within 3% of the solution, and the
    solutions from either start within 1e-7."""
    with open(WEIGHTS + "_at_255x361x721.json") as fh:
        rec = json.load(fh)
    cfg = rec["config"]
    assert (cfg["nr"], cfg["nt"], cfg["np"]) == (255, 361, 721)
    assert cfg["evaluate"].endswith("fno_pfss_127x181x361.npz") and cfg["radial_levels_resampled"]
    assert cfg["test_seed0"] >= 5000 and cfg["test"] == 20  # outside the training seeds 1000-2999
    ev = rec["evaluation"]
    assert ev["cases"] == 20 and len(rec["cases"]) == 20
    assert ev["fewer_iterations_cases"] == 20 and ev["iteration_ratio"] < 0.9
    assert ev["guess_rel_err_max"] < 0.03 and ev["sol_rel_diff_max"] < 1e-7
