"""Emission on the GPU: the reference's ranlxd streams and the per-source split.

* CMI_RNG_RANLUX replays the reference's fill_buffer streams
  (testDensitySubGrid_omp.cpp:529-597, seeded per buffer as described in
  cmacionize_b200.h): k_emit_ranlux's photons equal the oracle's replay
  (the reference generator with correctly rounded sin, cos and log) bit for
  bit, and the reference's own photons (golden file) up to glibc's rare
  last-bit misroundings.
* An iteration with CMI_RNG_RANLUX transports exactly those photons: the
  FP64 wavefront gives the reference walk's counts and J on them.
* Per-source packet numbers follow the reference split
  (testDensitySubGrid_omp.cpp:2199-2208): the truncation (unsigned)(L_i /
  L_tot * N) for every source, plus one packet for num_photon_rem distinct
  sources (distribute, :1650-1677; the draws that pick them are Philox here).
"""
import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200 import GridSpec, TransportEngine
from parallelcmacionize_b200.problems import lognormal_config

pytestmark = pytest.mark.gpu

PC = 3.086e16
BOX = (-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC)


def ulps(a, b):
    return np.abs(np.asarray(a, np.float64).view(np.int64) - np.asarray(b, np.float64).view(np.int64))


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_ranlux_emission_replays_reference_stream(precision):
    g = golden("emission.npz")
    first = 0
    glibc_differ = 0
    for seed, n, src in zip(g["seeds"], g["counts"], g["sources"]):
        ref = g["photons"][first: first + n]
        first += n
        spec = GridSpec(box=BOX, ncell=(16, 16, 16), num_subgrid=(2, 2, 2),
                        sources=[(float(src[0]), float(src[1]), float(src[2]), 4.26e49)],
                        num_photon=int(n))
        with TransportEngine(spec, precision=precision, rng="ranlux") as eng:
            # buffer 0 of iteration 0 draws from ranlxd(seed)
            out = eng.emit_photons(seed=int(seed), iteration=0)
        assert out.size == n
        cr = O.fill_buffer_stream_cr(int(seed), src, int(n))
        assert out.tobytes() == cr.tobytes()  # the replay, bit for bit
        # the reference's own photons (glibc cos, sin, log): one ulp at most
        assert out["position"].tobytes() == ref["position"].tobytes()
        assert out["direction"][:, 2].tobytes() == ref["direction"][:, 2].tobytes()
        d = np.concatenate([ulps(out["direction"][:, 0], ref["direction"][:, 0]),
                            ulps(out["direction"][:, 1], ref["direction"][:, 1]),
                            ulps(out["tau"], ref["tau"])])
        assert d.max() <= 1
        glibc_differ += int(np.count_nonzero(d))
    assert glibc_differ <= 4  # 2 of 1611 draws on this host's glibc


def test_ranlux_buffers_follow_the_seeding_rule():
    """Buffer b of iteration i over all sources draws from ranlxd(seed + b +
    i * buffers): 3 sources with about 450, 200 and 130 packets are 3 + 2 + 1
    or 3 + 1 + 1 buffers, depending on where the remainder packet goes."""
    L = [4.5e48, 2.0e48, 1.3e48]
    pos = [(0.0, 0.0, 0.0), (1.1 * PC, -2.0 * PC, 0.3 * PC), (-3.0 * PC, 3.3 * PC, 4.0 * PC)]
    spec = GridSpec(box=BOX, ncell=(16, 16, 16), num_subgrid=(2, 2, 2),
                    sources=[p + (l,) for p, l in zip(pos, L)], num_photon=780)
    seed, it = 1234, 2
    with TransportEngine(spec, precision="fp64", rng="ranlux") as eng:
        out = eng.emit_photons(seed=seed, iteration=it)
    counts = [int(c) for c in O.split_packets(L, 780, seed=seed, iteration=it)]
    nbuf = sum((c + 199) // 200 for c in counts)
    b = 0
    k = 0
    for s, n in enumerate(counts):
        done = 0
        while done < n:
            m = min(200, n - done)
            exp = O.fill_buffer_stream_cr(seed + b + it * nbuf, pos[s], m)
            assert out[k: k + m].tobytes() == exp.tobytes(), (s, b)
            k += m
            done += m
            b += 1
    assert k == out.size == 780


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ranlux_iteration_transports_the_emitted_photons(precision):
    """The wavefront with CMI_RNG_RANLUX traces exactly the photons
    cmi_emit_photons returns: same counts and J as the oracle's walk of them
    (FP64: the reference's interact arithmetic; mixed: its CPU restatement)."""
    spec, nH = lognormal_config(ncell=32, num_subgrid=4, num_photon=2500, num_sources=3, seed=7)
    with TransportEngine(spec, precision=precision, rng="ranlux") as eng:
        eng.set_fields(0, nH)
        ph = eng.emit_photons(seed=77, iteration=0)
        st = eng.shoot_packets(seed=77, iteration=0)[0]
        _, J = eng.get_fields(0)
    assert st["error_flags"] == 0 and st["packets_emitted"] == ph.size == 2500
    lat = O.LatticeGrid(spec.box, spec.ncell, spec.num_subgrid)
    start = np.array([lat.locate(p) for p in ph["position"]], np.uint32)
    xH = np.full(nH.size, 1e-6)
    if precision == "fp64":
        Jo = np.zeros(nH.size)
        cnt = lat.transport(nH, xH, Jo, ph.copy(), start)
        np.testing.assert_allclose(J, Jo, rtol=1e-12, atol=0)
    else:
        fixed = np.zeros(nH.size, np.uint64)
        cnt = lat.transport_mixed(O.kappa32(nH, xH), None, O.packets_mixed(ph), start,
                                  fixed=fixed)
        np.testing.assert_allclose(J, fixed.astype(np.float64) * lat.fixed_unit() * 6.3e-22,
                                   rtol=1e-12, atol=0)
    assert st["packets_absorbed"] == cnt["absorbed"]
    assert st["packets_escaped"] == cnt["escaped"]
    assert st["cell_crossings"] == cnt["crossings"]
    assert st["subgrid_transits"] == cnt["transits"]


@pytest.mark.parametrize("rng", ["philox", "ranlux"])
def test_per_source_numbers_follow_the_reference_split(rng):
    L = np.array([4.26e48, 1.0e48, 3.3e48, 7.7e47, 2.2e48])
    pos = [(0.0, 0.0, 0.0), (1.0 * PC, 2.0 * PC, -1.0 * PC), (-2.5 * PC, 0.5 * PC, 3.0 * PC),
           (4.0 * PC, -4.0 * PC, 0.2 * PC), (-1.2 * PC, -3.3 * PC, -4.4 * PC)]
    N = 100_003
    spec = GridSpec(box=BOX, ncell=(16, 16, 16), num_subgrid=(2, 2, 2),
                    sources=[p + (l,) for p, l in zip(pos, L)], num_photon=N)
    trunc = np.array([int(l / L.sum() * N) for l in L])  # the reference's truncation
    rem = N - int(trunc.sum())
    assert 0 < rem < L.size
    with TransportEngine(spec, precision="fp64", rng=rng) as eng:
        for it in range(3):
            ph = eng.emit_photons(seed=42, iteration=it)
            counts = np.array([np.sum(np.all(ph["position"] == np.array(p), axis=1))
                               for p in pos])
            assert counts.sum() == N == ph.size
            extra = counts - trunc
            assert set(extra.tolist()) <= {0, 1} and int(extra.sum()) == rem
            # the Philox remainder draws, restated by the oracle
            assert np.array_equal(counts, O.split_packets(L, N, seed=42, iteration=it))
            # the photons come source after source
            assert np.array_equal(np.repeat(np.arange(L.size), counts),
                                  [next(i for i, p in enumerate(pos) if np.array_equal(q, p))
                                   for q in ph["position"]])


def test_philox_emission_matches_the_oracle_draws():
    """Philox emission (production): the packets of the oracle's
    cmio_philox_packet; sin, cos and log come from the CUDA math library on
    the device and from the C library on the host, so they agree to a few ulp."""
    spec, nH = lognormal_config(ncell=32, num_subgrid=4, num_photon=20_000, num_sources=2, seed=3)
    with TransportEngine(spec, precision="mixed") as eng:
        ph = eng.emit_photons(seed=99, iteration=4)
    d, tau = O.philox_packets(99, 4, 0, ph.size)
    assert ulps(ph["direction"], d).max() <= 4
    assert ulps(ph["tau"], tau).max() <= 4
