"""The multi-GPU replica path of ReplicaRunner on one GPU.

With an all-reduce that leaves J as it is, one rank runs exactly the code a
rank of a multi-GPU job runs (the captured transport graph of
cmi_shoot_packets, the all-reduce ordered on the engine's stream, then
cmi_compute_neutral_fraction for the packets of all ranks); it must trace the
same packets as cmi_run_iterations (identical counts) and give the same
fields to FP64 rounding.
"""
import numpy as np
import pytest
import torch

from parallelcmacionize_b200 import TransportEngine
from parallelcmacionize_b200.distributed import ReplicaRunner
from parallelcmacionize_b200.problems import lognormal_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["mixed", "fp32", "fp64"])
def test_replica_path_equals_run_iterations(precision):
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=200_000, num_sources=2,
                                seed=11)
    with TransportEngine(spec, precision=precision) as a:
        a.set_fields(0, nH)
        sa = [it[0] for it in a.run_iterations(3, seed=42)]
        xa, Ja = a.get_fields(0)
    calls = []

    def identity_allreduce(t, op):
        # runs on the engine's stream (the runner makes it torch's current stream)
        calls.append(torch.cuda.current_stream().cuda_stream)

    with TransportEngine(spec, precision=precision) as b:
        b.set_fields(0, nH)
        runner = ReplicaRunner(b, allreduce=identity_allreduce)
        sb = runner.run(3, seed=42)
        xb, Jb = b.get_fields(0)
        assert calls == [b.stream()] * 3
        # transport-only iterations are replayed from their own captured graph
        assert runner.launches > 0
    # J is merged from the walk's shared tallies with FP64 atomics in an order
    # that varies from run to run: the fields agree to FP64 rounding
    np.testing.assert_allclose(xb, xa, rtol=1e-12, atol=1e-18)
    assert not Ja.any() and not Jb.any()  # reset by the balance
    for p, q in zip(sa, sb):
        for k in ("packets_emitted", "packets_absorbed", "packets_escaped", "cell_crossings",
                  "subgrid_transits"):
            assert p[k] == q[k], k
        assert q["error_flags"] == 0
        assert abs(p["mean_abs_dx"] - q["mean_abs_dx"]) <= 1e-12 * max(p["mean_abs_dx"], 1e-30)
