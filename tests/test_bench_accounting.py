"""The bench's algorithmic bytes/flops per phase and its DRAM-traffic estimate (CPU)."""
from types import SimpleNamespace

import pytest

import bench


def _run(n_r, l_max, n_orb=9, hartree=True, angular="reference", n_har=4):
    return SimpleNamespace(n_r=n_r, n_l=l_max + 1, n_orb=n_orb, use_hartree=hartree, target_id=1, n_har=n_har,
                           angular=angular)


def test_chain_products_per_half_step():
    assert bench.chain_products(_run(600, 96)) == 5                     # FF, FP, D, P + 1
    assert bench.chain_products(_run(600, 96, n_har=3)) == 4            # FP, D, P + 1
    assert bench.chain_products(_run(600, 96, hartree=False)) == 2      # P + 1
    assert bench.chain_products(_run(600, 96, angular="theta")) == 2   # one phase at the nodes


def test_phase_bytes_and_flops_of_one_int8_group():
    runs = [_run(600, 96) for _ in range(16)]
    tf = bench.phase_traffic(runs, [list(range(16))], "split_int8")
    elems = 600 * 97 * 144
    # W as eight int8 planes, x as 12 B of slices in, complex128 out
    assert tf["radial"]["bytes"] == 8 * 600 * 600 * 97 + (12 + 16) * elems
    assert tf["radial"]["flops"] == 8.0 * 600 * 600 * 97 * 144
    # complex128 in and out; five chain products with all four couplings
    assert tf["angular_first"]["bytes"] == 2 * 16 * elems
    assert tf["angular_second"]["flops"] == 5 * 4.0 * 97 * 97 * 600 * 144


def test_basis_reuse_accounting():
    """split_int8 theta form with basis reuse: the first half runs one product, the second half also
    writes the kept node-basis vectors; other forms and the reference chain are unchanged."""
    runs = [_run(600, 96, angular="theta") for _ in range(16)]
    elems = 600 * 97 * 144
    off = bench.phase_traffic(runs, [list(range(16))], "split_int8")
    on = bench.phase_traffic(runs, [list(range(16))], "split_int8", theta_reuse=True)
    assert off["angular_first"]["flops"] == 2 * 4.0 * 97 * 97 * 600 * 144
    assert on["angular_first"]["flops"] == 1 * 4.0 * 97 * 97 * 600 * 144
    assert on["angular_first"]["bytes"] == off["angular_first"]["bytes"] == 2 * 16 * elems
    assert on["angular_second"]["flops"] == off["angular_second"]["flops"]
    assert on["angular_second"]["bytes"] == 3 * 16 * elems
    assert on["radial"] == off["radial"]
    ref_chain = [_run(600, 96) for _ in range(16)]
    assert (bench.phase_traffic(ref_chain, [list(range(16))], "split_int8", theta_reuse=True) ==
            bench.phase_traffic(ref_chain, [list(range(16))], "split_int8"))
    assert (bench.phase_traffic(runs, [list(range(16))], "fp64", theta_reuse=True) ==
            bench.phase_traffic(runs, [list(range(16))], "fp64"))


def test_traffic_estimate_uses_the_ratio_of_each_groups_kernel():
    runs = [_run(600, 96), _run(600, 96), _run(900, 144)]
    groups = [[0, 1], [2]]
    est = bench.measured_traffic(runs, groups, "split_int8", "angular_second")
    one = bench.phase_traffic(runs, [[0, 1]], "split_int8")["angular_second"]["bytes"]
    two = bench.phase_traffic(runs, [[2]], "split_int8")["angular_second"]["bytes"]
    r1 = bench.MEASURED_TRAFFIC_RATIO[("split_int8", "angular_second", 1)]
    r2 = bench.MEASURED_TRAFFIC_RATIO[("split_int8", "angular_second", 2)]
    assert est == pytest.approx(one * r1 + two * r2)
    # no capture for this form: no estimate
    assert bench.measured_traffic(runs, groups, "fp64", "angular_second") is None


@pytest.mark.parametrize("name,total", [("ar-ens64", 64), ("hhe-ens256", 256), ("ar16-n600", 16), ("he-fp64", 1)])
def test_cpu_sample_covers_every_grid_group_once(name, total):
    """The CPU legs time one run per grid group and weight it by the runs in that group."""
    from ggbtddft_b200 import problems as P
    groups = bench.workload_groups(name)
    assert sum(count for _, count, _ in groups) == total
    if name == "ar-ens64":
        dr = P.argon_draws(64, seed=0)
        assert len(groups) == 5                      # the five ladder rungs
        for idx, count, _ in groups:
            same = [i for i in range(64) if dr.rung[i] == dr.rung[idx]]
            assert len(same) == count and idx == same[0]


def test_step_bound_is_the_sum_of_phase_bounds():
    """Phases run one after another: an HBM-bound radial product and a flop-bound angular chain do
    not overlap, so the step's roofline time adds their bounds."""
    tf = {"radial": dict(bytes=6.45e12, flops=1e12), "angular_first": dict(bytes=1e6, flops=36.6e12),
          "angular_second": dict(bytes=6.45e11, flops=0.0)}
    s = bench.phase_bound_seconds(tf, 6450.0, 36.6)
    assert abs(s - (1.0 + 1.0 + 0.1)) < 1e-12
