"""Parity of the CUDA path (through the C ABI) with the oracle and the reference.

FP64 transport is the reference's arithmetic operation for operation, so its
cell sequences, path lengths, photons and (where the summation order is the
same) J are compared bit for bit.  The FP32 transport is compared bit for bit
with its own CPU restatement (cmio_interact32) and within stated tolerances
with the FP64 reference.
"""
import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200 import (CMIError, GridSpec, PHOTON_DTYPE, TransportEngine,
                                     blocked_to_cube, cube_to_blocked)
from parallelcmacionize_b200.problems import (cell_radii, ionized_radius, lognormal_config,
                                              stromgren, stromgren_profile)

pytestmark = pytest.mark.gpu

PC = 3.086e16
WALK_CASES = ["interior16", "entries8", "edges16", "noncubic"]


def single_subgrid_engine(g, precision="fp64", balance="reference"):
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=(1, 1, 1))
    eng = TransportEngine(spec, precision=precision, balance=balance)
    eng.set_fields(0, g["nH"], g["xH"])
    return eng


@pytest.mark.parametrize("case", WALK_CASES)
def test_trace_fp64_bit_exact(case):
    g = golden(f"walk_{case}.npz")
    eng = single_subgrid_engine(g)
    sg = O.subgrid(g["box"], g["ncell"])
    for i in range(g["photons"].size):
        ph = g["photons"][i]
        out, res, cells, lengths, n = eng.trace_packet(0, 0, int(g["in_dirs"][i]), ph)
        p = g["photons"][i: i + 1].copy()
        ores, ocells, olengths, on = O.interact(sg, g["nH"], g["xH"], np.zeros_like(g["nH"]),
                                                p, int(g["in_dirs"][i]), max_steps=4096)
        assert res == g["result"][i] == ores
        assert n == on
        assert np.array_equal(cells, ocells)            # cell sequence, bit-exact
        assert lengths.tobytes() == olengths.tobytes()  # path lengths, bit-exact
        assert out.tobytes() == g["out"][i].tobytes()   # photon as the reference leaves it
    # one packet per launch: J receives the packets' tallies in reference order
    _, J = eng.get_fields(0)
    assert J.tobytes() == g["J"].tobytes()
    eng.close()


@pytest.mark.parametrize("case", WALK_CASES)
def test_traverse_buffer_fp64(case):
    """do_photon_traversal: grouping into the 27 output buffers, input order kept."""
    g = golden(f"walk_{case}.npz")
    eng = single_subgrid_engine(g)
    J_ref = np.zeros_like(g["nH"])
    for d in np.unique(g["in_dirs"]):
        sel = np.nonzero(g["in_dirs"] == d)[0]
        out, counts, done = eng.traverse_buffer(0, 0, int(d), g["photons"][sel])
        assert done == 0
        res = g["result"][sel]
        expect = np.concatenate([g["out"][sel][res == k] for k in range(27)])
        assert np.array_equal(counts, np.bincount(res, minlength=27))
        assert out.tobytes() == expect.tobytes()
    _, J = eng.get_fields(0)
    np.testing.assert_allclose(J, g["J"], rtol=1e-13, atol=0)
    eng.close()


def test_traverse_buffer_flags():
    """Disabled output buffers (escaped: neighbour outside; absorbed with
    reemission off) are dropped and counted as done (testDensitySubGrid_omp.cpp:1178-1191)."""
    g = golden("walk_entries8.npz")
    eng = single_subgrid_engine(g)
    sel = np.nonzero(g["in_dirs"] == 0)[0]
    enabled = np.ones(27, np.uint8)
    enabled[0] = 0
    enabled[21:] = 0
    out, counts, done = eng.traverse_buffer(0, 0, 0, g["photons"][sel], enabled=enabled)
    res = g["result"][sel]
    assert done == int(np.sum((res == 0) | (res >= 21)))
    assert counts[0] == 0 and np.all(counts[21:] == 0)
    assert int(counts.sum()) + done == sel.size
    eng.close()


@pytest.mark.parametrize("case", ["interior16", "edges16", "noncubic"])
def test_trace_fp32_matches_cpu_spec(case):
    """FP32 walk on the GPU == cmio_interact32 on the host, bit for bit."""
    g = golden(f"walk_{case}.npz")
    eng = single_subgrid_engine(g, precision="fp32")
    sg = O.subgrid(g["box"], g["ncell"])
    kappa = O.kappa32(g["nH"], g["xH"])
    cs = np.array(sg.cell_size, dtype=np.float32)
    for i in range(g["photons"].size):
        if g["photons"]["sigma"][i] != 6.3e-22:
            continue  # the FP32 kappa field folds in the instance cross section
        ph = g["photons"][i]
        out, res, cells, lengths, n = eng.trace_packet(0, 0, 0, ph)
        q = np.zeros(1, O.PACKET32_DTYPE)
        q["pos"] = (ph["position"] - g["box"][:3]) * np.array(sg.inv_cell_size)
        q["dir"] = ph["direction"]
        q["tau"] = ph["tau"]
        ores, ocells, olen, on = O.interact32(g["ncell"], cs, kappa, None, q, max_steps=4096,
                                              inv_cell_size=np.array(sg.inv_cell_size))
        assert res == ores and n == on
        assert np.array_equal(cells, ocells)
        assert np.array_equal(lengths.astype(np.float32), olen)


def test_transport_packets_fp64():
    """Full wavefront (emission bucket, plan, scatter, walk rounds) on given packets."""
    g = golden("transport.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=tuple(int(v) for v in g["num_subgrid"]))
    eng = TransportEngine(spec, precision="fp64")
    eng.set_fields(0, g["nH"], g["xH"])
    st = eng.transport_packets(0, g["photons"], g["start"])
    assert st["packets_absorbed"] == int(np.sum(g["fate"] == 0))
    assert st["packets_escaped"] == int(np.sum(g["fate"] == 1))
    assert st["subgrid_transits"] == int(g["transits"].sum())
    assert st["error_flags"] == 0
    lat = O.LatticeGrid(g["box"], g["ncell"], g["num_subgrid"])
    Jo = np.zeros_like(g["nH"])
    cnt = lat.transport(g["nH"], g["xH"], Jo, g["photons"].copy(), g["start"])
    assert st["cell_crossings"] == cnt["crossings"]
    _, J = eng.get_fields(0)
    np.testing.assert_allclose(J, g["J"], rtol=1e-12, atol=1e-300)
    eng.close()


def test_transport_packets_fp32_matches_cpu_spec():
    g = golden("transport.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=tuple(int(v) for v in g["num_subgrid"]))
    eng = TransportEngine(spec, precision="fp32")
    eng.set_fields(0, g["nH"], g["xH"])
    st = eng.transport_packets(0, g["photons"], g["start"])
    lat = O.LatticeGrid(g["box"], g["ncell"], g["num_subgrid"])
    kappa = O.kappa32(g["nH"], g["xH"])
    q = np.zeros(g["photons"].size, O.PACKET32_DTYPE)
    sub = [lat.subgrid_desc(int(s)) for s in g["start"]]
    for i, s in enumerate(sub):
        q["pos"][i] = (g["photons"]["position"][i] - np.array(s.anchor)) * np.array(s.inv_cell_size)
    q["dir"] = g["photons"]["direction"]
    q["tau"] = g["photons"]["tau"]
    tally = np.zeros(g["nH"].size)
    fixed = np.zeros(g["nH"].size, np.uint64)
    cnt = lat.transport32(kappa, tally, q.copy(), g["start"], fixed=fixed)
    assert st["packets_absorbed"] == cnt["absorbed"]
    assert st["packets_escaped"] == cnt["escaped"]
    assert st["cell_crossings"] == cnt["crossings"]
    _, J = eng.get_fields(0)
    # default tally: exact 64-bit fixed-point sums, merged into FP64 once per
    # subgrid residency -> equal to the oracle's integer sums to FP64 rounding
    np.testing.assert_allclose(J, fixed.astype(np.float64) * lat.fixed_unit() * 6.3e-22,
                               rtol=1e-12, atol=0)
    # the fixed-point rounding: at most half a unit (lref / 2^25) per crossing
    half_unit = 0.5 * lat.fixed_unit() * 6.3e-22
    assert np.all(np.abs(J - tally * 6.3e-22) <= 1e-9 * np.abs(J) + 100 * half_unit)
    # and against the FP64 reference
    np.testing.assert_allclose(J.sum(), g["J"].sum(), rtol=1e-4)
    eng.close()
    # the compensated-FP32 tally variant: FP32 partials + their TwoSum errors
    eng = TransportEngine(spec, precision="fp32", tally="fp32_compensated")
    eng.set_fields(0, g["nH"], g["xH"])
    eng.transport_packets(0, g["photons"], g["start"])
    _, Jc = eng.get_fields(0)
    np.testing.assert_allclose(Jc, tally * 6.3e-22, rtol=1e-9, atol=0)
    eng.close()


def test_transport_fp32_independent_of_chunking():
    """The FP32 walk's packet ring (chunks of 32 .. 1024 packets, claimed up
    to 256 packets ahead of the copies, runs of 1 .. 64 chunks per claim, lanes
    routed and refilled one at a time up to all 32 at once):
    every chunking traces the same packets, so the counts are identical and J
    (exact fixed-point sums, merged into FP64 in varying order) agrees to FP64
    rounding."""
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=400_000, num_sources=3)
    ref = None
    for chunk, run, refill in [(128, 0, 0), (32, 0, 0), (64, 0, 0), (64, 1, 0), (256, 8, 0),
                               (1024, 0, 0), (128, 0, 1), (128, 0, 32), (64, 4, 5)]:
        eng = TransportEngine(spec, precision="fp32", packets_per_chunk=chunk,
                              max_run_chunks=run, refill_lanes=refill)
        eng.set_fields(0, nH)
        st = [eng.shoot_packets(seed=9, iteration=i)[0] for i in range(2)]
        _, J = eng.get_fields(0)
        eng.close()
        for s in st:
            assert s["error_flags"] == 0, (chunk, run, refill)
            assert s["packets_absorbed"] + s["packets_escaped"] == 400_000
        key = [(s["cell_crossings"], s["packets_absorbed"], s["subgrid_transits"]) for s in st]
        if ref is None:
            ref = (key, J)
            continue
        assert key == ref[0], (chunk, run, refill)
        np.testing.assert_allclose(J, ref[1], rtol=1e-12, atol=0)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_multi_tile_plan_matches_single_tile(precision):
    """More than 4096 subgrids in a context: the round plan runs as
    count / offsets / write over several tiles.  Instance 1's packets (Philox
    keyed by the instance index) must be traced identically whether instance 0
    has 4096 subgrids (4160 in all: two plan tiles) or 8 (one tile)."""
    big, nbig = lognormal_config(ncell=128, num_subgrid=16, num_photon=300_000, num_sources=2,
                                 seed=3)
    tiny, ntiny = lognormal_config(ncell=16, num_subgrid=2, num_photon=1000, num_sources=1,
                                   seed=5)
    small, nsmall = lognormal_config(ncell=32, num_subgrid=4, num_photon=100_000, num_sources=2,
                                     seed=4)
    out = []
    for first, nfirst in ((big, nbig), (tiny, ntiny)):
        eng = TransportEngine([first, small], precision=precision)
        eng.set_fields(0, nfirst)
        eng.set_fields(1, nsmall)
        st = [eng.shoot_packets(seed=8, iteration=i) for i in range(2)]
        for s in st:
            for k in s:
                assert k["error_flags"] == 0
                assert k["packets_absorbed"] + k["packets_escaped"] == k["packets_emitted"]
        out.append(([(s[1]["cell_crossings"], s[1]["packets_absorbed"], s[1]["subgrid_transits"])
                     for s in st], eng.get_fields(1)[1]))
        eng.close()
    assert out[0][0] == out[1][0]
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-12, atol=0)


def test_oversized_packet_ring_is_refused():
    """Two 4096-packet chunks (256 KB) do not fit in a CTA's shared memory:
    creation fails with NOT_SUPPORTED and the next context works."""
    spec, nH = lognormal_config(ncell=32, num_subgrid=2, num_photon=10_000, num_sources=1)
    with pytest.raises(CMIError) as e:
        TransportEngine(spec, precision="fp32", packets_per_chunk=4096)
    assert "shared memory" in str(e.value)
    eng = TransportEngine(spec, precision="fp32")
    eng.set_fields(0, nH)
    assert eng.run_iterations(1, seed=1)[0][0]["error_flags"] == 0
    eng.close()


def test_balance_reference_form_bit_exact():
    g = golden("balance.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=(1, 1, 1))
    eng = TransportEngine(spec, precision="fp64", balance="reference")
    eng.set_fields(0, g["nH"], np.full(g["nH"].size, 1e-6))
    eng.set_intensity(0, g["J"])
    eng.compute_neutral_fraction(0, float(g["L"]), int(g["N"]))
    x, J = eng.get_fields(0)
    assert x.tobytes() == g["xH"].tobytes()
    assert np.all(J == 0)
    eng.close()


def test_balance_stable_form():
    g = golden("balance.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=(2, 2, 2))
    eng = TransportEngine(spec, precision="fp32", balance="stable")
    nH = g["nH"]
    eng.set_fields(0, nH, np.full(nH.size, 1e-6), layout="cube")
    eng.set_intensity(0, g["J"], layout="cube")
    eng.compute_neutral_fraction(0, float(g["L"]), int(g["N"]))
    x, _ = eng.get_fields(0, layout="cube")
    sg = O.subgrid(g["box"], g["ncell"])
    xo = np.zeros_like(nH)
    O.compute_neutral_fraction(nH.copy(), xo, g["J"].copy(),
                               O.jfac(float(g["L"]), float(g["N"]), np.array(sg.inv_cell_size)),
                               4e-19, form=1)
    assert x.tobytes() == xo.tobytes()
    eng.close()


def test_layout_round_trip():
    spec = GridSpec(box=(0, 0, 0, 1, 2, 3), ncell=(12, 8, 16), num_subgrid=(3, 2, 4))
    eng = TransportEngine(spec, precision="fp32")
    cube = np.random.default_rng(0).uniform(size=(12, 8, 16))
    eng.set_fields(0, number_density=None, neutral_fraction=cube.reshape(-1), layout="cube")
    x_blocked, _ = eng.get_fields(0, layout="blocked")
    assert np.array_equal(x_blocked, cube_to_blocked(cube, spec.ncell, spec.num_subgrid))
    x_cube, _ = eng.get_fields(0, layout="cube")
    assert np.array_equal(x_cube.reshape(12, 8, 16), cube)
    assert np.array_equal(blocked_to_cube(x_blocked, spec.ncell, spec.num_subgrid), cube)
    eng.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_iteration_conservation(precision):
    """Every emitted packet ends absorbed or escaped; counts are conserved
    (the termination rule of testDensitySubGrid_omp.cpp:2370-2397)."""
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=300_001, num_sources=3)
    eng = TransportEngine(spec, precision=precision)
    eng.set_fields(0, nH)
    stats = eng.run_iterations(3, seed=11)
    for it in stats:
        s = it[0]
        assert s["packets_emitted"] == 300_001
        assert s["packets_absorbed"] + s["packets_escaped"] == s["packets_emitted"]
        assert s["error_flags"] == 0
        assert 1 <= s["rounds"] <= 4 + 4 + 4 - 2 + 3  # straight-line bound + spares
        assert s["cell_crossings"] > s["subgrid_transits"] > 0
    eng.close()


def test_iteration_fp32_vs_fp64_same_packets():
    """Same Philox packets through both precisions: J agrees to FP32 accuracy."""
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=200_000, num_sources=2)
    res = {}
    for prec in ("fp64", "fp32"):
        eng = TransportEngine(spec, precision=prec)
        eng.set_fields(0, nH)
        st = eng.shoot_packets(seed=5, iteration=0)[0]
        _, J = eng.get_fields(0)
        res[prec] = (st, J)
        eng.close()
    s64, J64 = res["fp64"]
    s32, J32 = res["fp32"]
    assert abs(int(s64["cell_crossings"]) - int(s32["cell_crossings"])) <= 2e-4 * s64["cell_crossings"]
    assert abs(int(s64["packets_escaped"]) - int(s32["packets_escaped"])) <= 2e-3 * s64["packets_emitted"] + 5
    big = J64 > 1e-3 * J64.max()
    rel = np.abs(J32[big] - J64[big]) / J64[big]
    assert np.median(rel) < 1e-5
    np.testing.assert_allclose(J32.sum(), J64.sum(), rtol=1e-4)


def test_iteration_matches_oracle_port():
    """GPU FP64 iteration vs the oracle's OpenMP port on the same Philox packets."""
    spec, nH = lognormal_config(ncell=32, num_subgrid=4, num_photon=50_000, num_sources=2,
                                sigma_ln=0.5)
    eng = TransportEngine(spec, precision="fp64", balance="stable")
    eng.set_fields(0, nH)
    st = eng.run_iterations(1, seed=77)[0][0]
    x_gpu, _ = eng.get_fields(0)
    eng.close()
    lat = O.LatticeGrid(spec.box, spec.ncell, spec.num_subgrid)
    src = np.array(spec.sources)
    x = np.full(nH.size, 1e-6)
    J = np.zeros(nH.size)
    cnt = lat.iteration_omp(nH, x, J, src[:, :3], src[:, 3], 50_000, 77, 0, balance_form=1)
    # directions differ from the host's only by the last-ulp of sin/cos
    assert abs(cnt["crossings"] - st["cell_crossings"]) <= 1e-4 * cnt["crossings"] + 10
    assert cnt["absorbed"] + cnt["escaped"] == 50_000
    close = np.isclose(x_gpu, x, rtol=1e-9, atol=1e-15)
    assert close.mean() > 0.999


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_stromgren_radius(precision):
    """64^3 Stromgren sphere, 1e6 packets x 10 iterations: ionized radius within
    1% of the analytic R_S and within 3 sigma of the reference's seed ensemble."""
    spec, nH = stromgren(ncell=64, num_subgrid=8, num_photon=1_000_000)
    eng = TransportEngine(spec, precision=precision)
    eng.set_fields(0, nH)
    stats = eng.run_iterations(10, seed=2024)
    x, _ = eng.get_fields(0, layout="cube")
    eng.close()
    _, _, Rs = stromgren_profile()
    R = ionized_radius(x.reshape(spec.ncell), spec)
    assert abs(R / Rs - 1) < 0.01
    ens = golden("stromgren_ensemble.npz")
    mu, sd = ens["radii"].mean(), ens["radii"].std(ddof=1)
    assert abs(R - mu) < 3 * sd + 1e-4 * mu  # + MC floor of one seed set
    # radial profile against the ensemble, bin by bin
    r = cell_radii(spec).reshape(-1)
    edges = ens["edges"]
    which = np.digitize(r, edges) - 1
    prof = np.array([x[which == b].mean() if np.any(which == b) else np.nan
                     for b in range(len(edges) - 1)])
    m = np.nanmean(ens["profiles"], axis=0)
    s = np.nanstd(ens["profiles"], axis=0, ddof=1)
    ok = np.isfinite(m) & (s > 0)
    z = np.abs(prof[ok] - m[ok]) / s[ok]
    assert np.mean(z > 3) <= 0.1 and np.median(z) < 2.0
    for it in stats:
        assert it[0]["error_flags"] == 0


def test_batched_instances():
    """Several uneven instances in one context (one launch per kernel)."""
    specs = []
    fields = []
    for k, (side, sub) in enumerate([(32, 4), (48, 3), (64, 8)]):
        spec, nH = lognormal_config(ncell=side, num_subgrid=sub, num_photon=5 * side ** 3,
                                    num_sources=1 + k, seed=100 + k)
        specs.append(spec)
        fields.append(nH)
    eng = TransportEngine(specs, precision="fp32")
    for i, nH in enumerate(fields):
        eng.set_fields(i, nH)
    stats = eng.run_iterations(2, seed=3)
    for it in stats:
        for i, s in enumerate(it):
            assert s["packets_emitted"] == specs[i].num_photon
            assert s["packets_absorbed"] + s["packets_escaped"] == s["packets_emitted"]
            assert s["error_flags"] == 0
    for i in range(3):
        x, _ = eng.get_fields(i)
        assert np.all((x > 0) & (x <= 1))
    eng.close()


def test_invalid_arguments():
    spec = GridSpec(box=(0, 0, 0, 1, 1, 1), ncell=(8, 8, 8), num_subgrid=(2, 2, 2))
    eng = TransportEngine(spec, precision="fp64")
    ph = np.zeros(1, PHOTON_DTYPE)
    ph["direction"] = (1, 0, 0)
    ph["tau"] = 1
    with pytest.raises(CMIError) as e:
        eng.trace_packet(0, 8, 0, ph[0])
    assert e.value.code == 1
    with pytest.raises(CMIError):
        eng.trace_packet(0, 0, 27, ph[0])
    with pytest.raises(CMIError):
        eng.set_sources(0, [[2.0, 0.5, 0.5]], [1e48])  # outside the box
    with pytest.raises(CMIError):
        eng.transport_packets(0, ph, [99])
    with pytest.raises(CMIError):
        TransportEngine(GridSpec(box=(0, 0, 0, 1, 1, 1), ncell=(10, 8, 8), num_subgrid=(3, 2, 2)))
    eng.close()


def test_result_files_from_the_engine(tmp_path):
    """write_outputs: the engine's x_H in the reference's .bin and .dat files,
    read back unchanged; the radial profile of a Stromgren run drops across R_S."""
    import os
    from parallelcmacionize_b200.outputs import (radial_profile, read_neutral_fractions_binary,
                                                  read_neutral_fractions_dat, write_outputs)
    spec, nH = stromgren(ncell=32, num_subgrid=4, num_photon=200_000)
    eng = TransportEngine(spec)
    eng.set_fields(0, nH)
    eng.run_iterations(6, seed=3)
    x, _ = eng.get_fields(0, intensity=False)
    paths = write_outputs(eng, 0, prefix=os.path.join(tmp_path, "nf"), nH_blocked=nH)
    eng.close()
    assert np.array_equal(read_neutral_fractions_binary(paths["bin"]), x)
    rec = read_neutral_fractions_dat(paths["dat"])
    assert np.array_equal(rec["xH"], x) and np.array_equal(rec["nH"], nH)
    _, _, Rs = stromgren_profile()
    r, prof = radial_profile(rec, bins=16, r_max=1.5 * Rs)
    assert np.nanmax(prof[r < 0.7 * Rs]) < 0.1 and np.nanmin(prof[r > 1.3 * Rs]) > 0.5


def test_prefetched_density_equals_set_fields():
    """cmi_prefetch_number_density + cmi_set_fields_prefetched load the same
    n_H (the device array, bit for bit) as cmi_set_fields, twice in a row, and
    an iteration from them gives the same x_H (FP64 tally merges in another
    order: within 1e-12)."""
    import torch
    from parallelcmacionize_b200.distributed import _CudaArray
    spec, nH = lognormal_config(ncell=32, num_subgrid=2, num_photon=50_000, num_sources=2)
    x0 = np.full(nH.size, 1e-3)
    res, dev_n = [], []
    for prefetch in (False, True):
        eng = TransportEngine(spec)
        if prefetch:
            pin = torch.from_numpy(nH.copy()).pin_memory()
            eng.prefetch_number_density(0, pin.numpy())
            with pytest.raises(CMIError):  # one pending prefetch per instance
                eng.prefetch_number_density(0, pin.numpy())
            eng.set_fields_prefetched(0, x0)
            with pytest.raises(CMIError):  # consumed
                eng.set_fields_prefetched(0, x0)
            # a second round with another density, then the first again
            pin2 = torch.from_numpy(nH * 2.0).pin_memory()
            eng.prefetch_number_density(0, pin2.numpy())
            eng.set_fields_prefetched(0, x0)
            eng.prefetch_number_density(0, pin.numpy())
            eng.set_fields_prefetched(0, x0)
        else:
            eng.set_fields(0, nH, x0)
        ptr, count = eng.device_field(0, "n")
        dev_n.append(torch.as_tensor(_CudaArray(ptr, count), device="cuda").cpu().numpy())
        eng.run_iterations(1, seed=3)
        res.append(eng.get_fields(0, intensity=False)[0])
        eng.close()
    assert np.array_equal(dev_n[0], dev_n[1])
    np.testing.assert_allclose(res[1], res[0], rtol=1e-12, atol=0)


def test_prefetched_fields_are_awaited():
    """cmi_set_fields_prefetched returns before its side-stream copies are
    done; the entry points that read the fields wait for them: get_fields
    returns the x_H just sent (pinned, 2 MB) bit for bit, device_field the
    n_H, and a second set in a row replaces the first."""
    import torch
    from parallelcmacionize_b200.distributed import _CudaArray
    spec, nH = lognormal_config(ncell=64, num_subgrid=4, num_photon=10_000, num_sources=1)
    with TransportEngine(spec) as eng:
        eng.set_fields(0, np.full(nH.size, 1e8), np.full(nH.size, 1e-6))
        pin_n = torch.from_numpy(nH.copy()).pin_memory()
        for k in range(2):
            pin_x = torch.from_numpy(np.linspace(1e-4, 0.9, nH.size) * (k + 1) / 2).pin_memory()
            eng.prefetch_number_density(0, pin_n.numpy())
            eng.set_fields_prefetched(0, pin_x.numpy())
            x = eng.get_fields(0, intensity=False)[0]
            assert np.array_equal(x, pin_x.numpy())
        ptr, count = eng.device_field(0, "n")
        dev = torch.as_tensor(_CudaArray(ptr, count), device="cuda").cpu().numpy()
        ref = TransportEngine(spec)
        ref.set_fields(0, nH, np.full(nH.size, 1e-6))
        p2, c2 = ref.device_field(0, "n")
        want = torch.as_tensor(_CudaArray(p2, c2), device="cuda").cpu().numpy()
        ref.close()
        assert np.array_equal(dev, want)


@pytest.mark.parametrize("workload", ["lognormal128", "large256"])
def test_full_size_conservation_and_fp32_vs_fp64(workload):
    """At the full benchmark sizes (128^3 with 1e7 packets; 256^3 with 1e8):
    every emitted packet ends absorbed or escaped in both precisions, no
    device flag is raised, and the FP32 walk's J agrees with the FP64 walk's
    (the reference arithmetic) on the same Philox packets from the same x_H
    (median relative difference < 1e-6 over cells with J > 1e-3 max J; sum
    within 1e-6)."""
    from parallelcmacionize_b200.problems import large_config
    if workload == "lognormal128":
        spec, nH = lognormal_config(ncell=128, num_subgrid=8, num_photon=10_000_000,
                                    num_sources=4)
    else:
        spec, nH = large_config()
    x0 = None
    res = {}
    for prec in ("fp32", "fp64"):
        with TransportEngine(spec, precision=prec) as eng:
            eng.set_fields(0, nH)
            if x0 is None:  # a converging field: two plain iterations in FP32
                for it in eng.run_iterations(2, seed=9):
                    s = it[0]
                    assert s["error_flags"] == 0
                    assert s["packets_absorbed"] + s["packets_escaped"] == s["packets_emitted"]
                x0 = eng.get_fields(0, intensity=False)[0]
            eng.set_fields(0, None, x0)
            st = eng.shoot_packets(seed=21, iteration=0)[0]
            assert st["error_flags"] == 0
            assert st["packets_absorbed"] + st["packets_escaped"] == st["packets_emitted"]
            res[prec] = (st, eng.get_fields(0)[1])
    (s32, J32), (s64, J64) = res["fp32"], res["fp64"]
    assert abs(int(s32["cell_crossings"]) - int(s64["cell_crossings"])) <= 1e-5 * s64["cell_crossings"]
    lit = J64 > 1e-3 * J64.max()
    rel = np.abs(J32[lit] - J64[lit]) / J64[lit]
    assert np.median(rel) < 1e-6, np.median(rel)
    assert abs(J32.sum() / J64.sum() - 1) < 1e-6
