"""cmi_run_until_converged: the convergence criterion mean |delta x_H| < tol
with per-instance freezing (no reference counterpart: the reference runs a
fixed number of iterations)."""
import numpy as np
import pytest

from parallelcmacionize_b200 import CMIError, TransportEngine
from parallelcmacionize_b200.problems import lognormal_config, stromgren

pytestmark = pytest.mark.gpu


def _pair():
    a, nA = stromgren(ncell=32, num_subgrid=2, num_photon=400_000)
    b, nB = lognormal_config(ncell=32, num_subgrid=2, num_photon=100_000, num_sources=2,
                             sigma_ln=1.0, seed=5)
    return [a, b], [nA, nB]


def _engine(specs, dens):
    eng = TransportEngine(specs, precision="fp32")
    for i, n in enumerate(dens):
        eng.set_fields(i, n)
    return eng


def test_run_until_converged_freezes_and_matches_fixed_runs():
    specs, dens = _pair()
    tol, max_it, min_it = 0.02, 25, 2
    eng = _engine(specs, dens)
    stats, at = eng.run_until_converged(tol, max_iterations=max_it, min_iterations=min_it,
                                        seed=31)
    x_conv = [eng.get_fields(i)[0] for i in range(2)]
    assert any(a > 0 for a in at)
    assert len(stats) == (max(at) if all(a > 0 for a in at) else max_it)
    for i, a in enumerate(at):
        dx = [s[i]["mean_abs_dx"] for s in stats]
        if a:
            assert dx[a - 1] < tol
            assert all(d >= tol for d in dx[min_it - 1:a - 1])
            for s in stats[a:]:  # frozen
                assert s[i]["packets_emitted"] == 0 and s[i]["mean_abs_dx"] == 0.0
        else:
            assert all(d >= tol for d in dx[min_it - 1:])
        for s in stats[: a or len(stats)]:
            assert s[i]["packets_emitted"] == specs[i].num_photon
            assert s[i]["error_flags"] == 0
    # all instances active again afterwards
    st = eng.run_iterations(1, seed=99)[0]
    assert [s["packets_emitted"] for s in st] == [g.num_photon for g in specs]
    eng.close()

    # freezing one instance does not change the other: each instance's x_H at
    # its convergence equals a plain run of that many iterations (packets are
    # keyed by instance; J sums in a different order -> FP64 rounding)
    for i, a in enumerate(at):
        if not a:
            continue
        e2 = _engine(specs, dens)
        e2.run_iterations(a, seed=31)
        np.testing.assert_allclose(e2.get_fields(i)[0], x_conv[i], rtol=1e-9, atol=1e-15)
        e2.close()


def test_run_until_converged_arguments():
    specs, dens = _pair()
    eng = _engine(specs, dens)
    with pytest.raises(CMIError):
        eng.run_until_converged(0.1, max_iterations=0)
    with pytest.raises(CMIError):
        eng.run_until_converged(0.1, max_iterations=3, min_iterations=4)
    with pytest.raises(CMIError):
        eng.run_until_converged(float("nan"), max_iterations=3)
    # tolerance 0 never converges: runs max_iterations
    stats, at = eng.run_until_converged(0.0, max_iterations=3, min_iterations=1)
    assert len(stats) == 3 and at == [0, 0]
    eng.close()
