"""Parity of the mixed-precision transport (CMI_TRANSPORT_MIXED) on the GPU.

The mixed walk keeps the reference's FP64 geometry operation for operation
(DensitySubGrid.hpp:1186-1305) and holds the cell opacity, the optical depths
and the tallies in FP32.  Against the reference, on every golden packet set:
the cell sequence and the exit direction are identical, every path length but
the absorbing cell's is bit-identical, and an exiting packet leaves with the
reference's position bit for bit.  The absorbing cell's length carries the
FP32 error of the accumulated optical depth.  Against its own CPU restatement
(cmio_interact_mixed) everything is bit for bit.
"""
import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200 import GridSpec, TransportEngine
from parallelcmacionize_b200.problems import lognormal_config

pytestmark = pytest.mark.gpu

WALK_CASES = ["interior16", "entries8", "edges16", "noncubic"]
# relative error of the absorbing cell's path length: FP32 optical depths
# (measured on the golden sets: 5.6e-5 at most; packets whose FP64 target
# depth is below the FP32 range are left out, their last length is ~0)
FINAL_LENGTH_RTOL = 1e-4


def engine_for(g, precision="mixed"):
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=(1, 1, 1))
    eng = TransportEngine(spec, precision=precision)
    eng.set_fields(0, g["nH"], g["xH"])
    return eng


@pytest.mark.parametrize("case", WALK_CASES)
def test_trace_mixed_matches_reference_geometry(case):
    g = golden(f"walk_{case}.npz")
    eng = engine_for(g)
    sg = O.subgrid(g["box"], g["ncell"])
    kappas = {}
    for i in range(g["photons"].size):
        ph = g["photons"][i]
        ind = int(g["in_dirs"][i])
        out, res, cells, lengths, n = eng.trace_packet(0, 0, ind, ph)
        # the reference's walk (the FP64 oracle equals it bit for bit)
        p = g["photons"][i: i + 1].copy()
        rres, rcells, rlen, rn = O.interact(sg, g["nH"], g["xH"], np.zeros_like(g["nH"]), p, ind,
                                            max_steps=4096)
        assert res == rres == g["result"][i]
        assert n == rn
        assert np.array_equal(cells, rcells)  # cell sequence
        full = n if res != 0 else n - 1       # crossings that are not the absorbing one
        assert lengths[:full].tobytes() == rlen[:full].tobytes()  # path lengths, bit for bit
        if res != 0:
            assert out["position"].tobytes() == g["out"][i]["position"].tobytes()
        elif n > 0 and ph["tau"] > 1e-30:
            assert abs(lengths[-1] - rlen[-1]) <= FINAL_LENGTH_RTOL * abs(rlen[-1])
        # the CPU restatement, bit for bit (cell opacity from the photon's sigma)
        sig = float(ph["sigma"])
        kap = kappas.setdefault(sig, O.kappa32(g["nH"], g["xH"], sig))
        q = O.packets_mixed(g["photons"][i: i + 1], [ind])
        ores, ocells, olen, on = O.interact_mixed(sg, kap, q, max_steps=4096)
        assert (res, n) == (ores, on)
        assert np.array_equal(cells, ocells)
        assert lengths.tobytes() == olen.tobytes()
        assert out["position"].tobytes() == q["pos"][0].tobytes()
        assert np.float32(out["tau"]) == q["tau"][0]
    eng.close()


@pytest.mark.parametrize("case", WALK_CASES)
def test_traverse_buffer_mixed(case):
    """do_photon_traversal with the mixed walk: the reference's grouping into
    the 27 output buffers, and J = sum of (lmin sigma) weight over the walk's
    FP64 lengths."""
    g = golden(f"walk_{case}.npz")
    eng = engine_for(g)
    sg = O.subgrid(g["box"], g["ncell"])
    J_expect = np.zeros_like(g["nH"])
    for d in np.unique(g["in_dirs"]):
        sel = np.nonzero(g["in_dirs"] == d)[0]
        out, counts, done = eng.traverse_buffer(0, 0, int(d), g["photons"][sel])
        assert done == 0
        res = g["result"][sel]
        assert np.array_equal(counts, np.bincount(res, minlength=27))
        # exiting photons carry the reference's positions and directions
        exp_exit = np.concatenate([g["out"][sel][res == k] for k in range(1, 27)])
        got_exit = out[counts[0]:]
        assert got_exit["position"].tobytes() == exp_exit["position"].tobytes()
        assert got_exit["direction"].tobytes() == exp_exit["direction"].tobytes()
        for i in sel:
            ph = g["photons"][i]
            kap = O.kappa32(g["nH"], g["xH"], float(ph["sigma"]))
            q = O.packets_mixed(g["photons"][i: i + 1], [int(d)])
            _, cells, lens, _ = O.interact_mixed(sg, kap, q, max_steps=4096)
            np.add.at(J_expect, cells, lens * float(ph["sigma"]) * float(ph["weight"]))
    _, J = eng.get_fields(0)
    np.testing.assert_allclose(J, J_expect, rtol=1e-12, atol=0)
    # and the reference's J: every crossing but the absorbing one is exact
    np.testing.assert_allclose(J.sum(), g["J"].sum(), rtol=1e-4)
    eng.close()


def test_transport_packets_mixed():
    """The full wavefront on the lattice golden: the reference's fates and
    transits, the CPU restatement's crossings and fixed-point tallies."""
    g = golden("transport.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=tuple(int(v) for v in g["num_subgrid"]))
    eng = TransportEngine(spec, precision="mixed")
    eng.set_fields(0, g["nH"], g["xH"])
    st = eng.transport_packets(0, g["photons"], g["start"])
    assert st["error_flags"] == 0
    assert st["packets_absorbed"] == int(np.sum(g["fate"] == 0))
    assert st["packets_escaped"] == int(np.sum(g["fate"] == 1))
    assert st["subgrid_transits"] == int(g["transits"].sum())
    lat = O.LatticeGrid(g["box"], g["ncell"], g["num_subgrid"])
    kappa = O.kappa32(g["nH"], g["xH"])
    q = O.packets_mixed(g["photons"])
    fixed = np.zeros(g["nH"].size, np.uint64)
    cnt = lat.transport_mixed(kappa, None, q, g["start"], fixed=fixed)
    assert st["cell_crossings"] == cnt["crossings"]
    Jo = np.zeros_like(g["nH"])
    cnt64 = lat.transport(g["nH"], g["xH"], Jo, g["photons"].copy(), g["start"])
    assert cnt["crossings"] == cnt64["crossings"]  # the reference's crossings
    # every escaped packet leaves the box where the reference's does, bit for bit
    esc = g["fate"] == 1
    assert q["pos"][esc].tobytes() == g["final"]["position"][esc].tobytes()
    _, J = eng.get_fields(0)
    np.testing.assert_allclose(J, fixed.astype(np.float64) * lat.fixed_unit() * 6.3e-22,
                               rtol=1e-12, atol=0)
    np.testing.assert_allclose(J.sum(), g["J"].sum(), rtol=1e-6)
    eng.close()


def test_transport_mixed_independent_of_chunking():
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=300_000, num_sources=3)
    ref = None
    for chunk, run, refill in [(128, 0, 0), (32, 0, 0), (64, 1, 0), (256, 8, 0), (128, 0, 1),
                               (128, 0, 32)]:
        eng = TransportEngine(spec, precision="mixed", packets_per_chunk=chunk,
                              max_run_chunks=run, refill_lanes=refill)
        eng.set_fields(0, nH)
        st = [eng.shoot_packets(seed=9, iteration=i)[0] for i in range(2)]
        _, J = eng.get_fields(0)
        eng.close()
        for s in st:
            assert s["error_flags"] == 0, (chunk, run, refill)
            assert s["packets_absorbed"] + s["packets_escaped"] == 300_000
        key = [(s["cell_crossings"], s["packets_absorbed"], s["subgrid_transits"]) for s in st]
        if ref is None:
            ref = (key, J)
            continue
        assert key == ref[0], (chunk, run, refill)
        np.testing.assert_allclose(J, ref[1], rtol=1e-12, atol=0)


def test_iteration_mixed_vs_fp64_same_packets():
    """The same Philox packets through the reference's FP64 walk and the mixed
    walk: the geometry is the same, so only packets whose absorption point
    lies within the FP32 optical-depth error of a cell face can cross a
    different number of cells."""
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=200_000, num_sources=2)
    res = {}
    for prec in ("fp64", "mixed"):
        eng = TransportEngine(spec, precision=prec)
        eng.set_fields(0, nH)
        st = eng.shoot_packets(seed=5, iteration=0)[0]
        _, J = eng.get_fields(0)
        res[prec] = (st, J)
        eng.close()
    (s64, J64), (sm, Jm) = res["fp64"], res["mixed"]
    assert sm["error_flags"] == 0
    assert abs(int(s64["cell_crossings"]) - int(sm["cell_crossings"])) <= 1e-5 * s64["cell_crossings"]
    assert s64["subgrid_transits"] == sm["subgrid_transits"]
    assert s64["packets_escaped"] == sm["packets_escaped"]
    big = J64 > 1e-3 * J64.max()
    rel = np.abs(Jm[big] - J64[big]) / J64[big]
    assert np.median(rel) < 1e-6
    np.testing.assert_allclose(Jm.sum(), J64.sum(), rtol=1e-6)
