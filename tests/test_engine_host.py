"""Host-side rules of TransportEngine, with a stand-in for the library (no GPU).

cmi_set_fields_prefetched returns before its side-stream copies are done, so
the wrapper keeps the host arrays it handed over (the prefetched n_H and the
x_H) until a call that waits for those copies returns.
"""
import numpy as np
import pytest

from parallelcmacionize_b200 import TransportEngine
from parallelcmacionize_b200.problems import stromgren


class RecordingLib:
    """Every entry point succeeds and is recorded."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def entry(*args):
            self.calls.append(name)
            return 0
        return entry


def engine_without_device(grid):
    eng = TransportEngine.__new__(TransportEngine)
    eng.grids = [grid]
    eng._L = RecordingLib()
    eng._h = None  # close() does nothing
    return eng


def held(eng):
    return [a for a in getattr(eng, "_in_flight", []) if a is not None]


WAITING_CALLS = {
    "run_iterations": lambda e: e.run_iterations(1),
    "run_until_converged": lambda e: e.run_until_converged(0.01, max_iterations=2),
    "shoot_packets": lambda e: e.shoot_packets(),
    "get_fields": lambda e: e.get_fields(0),
    "synchronize": lambda e: e.synchronize(),
}


@pytest.mark.parametrize("call", sorted(WAITING_CALLS))
def test_prefetched_arrays_held_until_a_waiting_call(call):
    grid, nH = stromgren(ncell=16, num_subgrid=2, num_photon=1000)
    eng = engine_without_device(grid)
    n = nH.copy()
    x = np.full(nH.size, 0.5, dtype=np.float32)  # converted: the wrapper's copy is sent
    eng.prefetch_number_density(0, n)
    eng.set_fields_prefetched(0, x)
    h = held(eng)
    assert any(a is n for a in h)
    sent = [a for a in h if a is not n]
    assert len(sent) == 1 and sent[0].dtype == np.float64 and np.array_equal(sent[0], x)
    # a second step before any waiting call keeps both steps' arrays
    n2 = nH * 2.0
    eng.prefetch_number_density(0, n2)
    eng.set_fields_prefetched(0, sent[0])
    assert len(held(eng)) == 4
    WAITING_CALLS[call](eng)
    assert held(eng) == []
    assert eng._L.calls.count("cmi_set_fields_prefetched") == 2


def test_prefetch_checks_the_array():
    grid, nH = stromgren(ncell=16, num_subgrid=2, num_photon=1000)
    eng = engine_without_device(grid)
    with pytest.raises(ValueError):
        eng.prefetch_number_density(0, nH.astype(np.float32))
    with pytest.raises(ValueError):
        eng.prefetch_number_density(0, nH[::2])
    with pytest.raises(ValueError):
        eng.set_fields_prefetched(0, np.zeros(nH.size + 1))
    assert eng._L.calls == []
