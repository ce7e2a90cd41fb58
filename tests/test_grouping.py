"""Grid groups of an ensemble (CPU): runs on one rung of the grid ladder share W and form one group."""
from ggbtddft_b200 import problems as P
from ggbtddft_b200.engine import group_runs


def test_runs_on_one_rung_share_W_and_form_one_group():
    ladder = [P.GridRung(48, 40.0, 11), P.GridRung(64, 50.0, 15)]
    runs = P.argon_ensemble(6, seed=0, n_steps=8, ladder=ladder)
    groups = group_runs(runs)
    assert sorted(i for g in groups for i in g) == list(range(6))
    keys = []
    for g in groups:
        r0 = runs[g[0]]
        assert all(runs[i].W is r0.W and (runs[i].n_r, runs[i].n_l) == (r0.n_r, r0.n_l) for i in g)
        keys.append((r0.n_r, r0.n_l))
    assert len(set(keys)) == len(groups)
    assert set(keys) <= {(48, 12), (64, 16)}


def test_a_run_built_alone_equals_its_twin_in_the_ensemble():
    import numpy as np
    ladder = [P.GridRung(48, 40.0, 11), P.GridRung(64, 50.0, 15)]
    full = P.argon_ensemble(6, seed=0, n_steps=8, ladder=ladder)
    one = P.argon_ensemble(6, seed=0, n_steps=8, ladder=ladder, only=[4])
    assert len(one) == 1
    a, b = full[4], one[0]
    assert (a.n_r, a.n_l, a.name) == (b.n_r, b.n_l, b.name)
    np.testing.assert_array_equal(a.E, b.E)
    np.testing.assert_array_equal(a.x0, b.x0)
    np.testing.assert_array_equal(a.W, b.W)
