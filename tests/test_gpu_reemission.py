"""Reemission (reemission_probability; do_reemission,
testDensitySubGrid_omp.cpp:675-702) on the GPU against the oracle's lattice
transport with the same counter-based draws, and the Stromgren radius it
implies: R_S with Q / (1 - p) photons (scripts/plot_neutral_fraction_profile.py:60-82)."""
import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200 import CMIError, GridSpec, TransportEngine
from parallelcmacionize_b200.problems import ionized_radius, stromgren, stromgren_profile

pytestmark = pytest.mark.gpu


def _engine(g, precision, p):
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=tuple(int(v) for v in g["num_subgrid"]),
                    reemission_probability=p)
    eng = TransportEngine(spec, precision=precision)
    eng.set_fields(0, g["nH"], g["xH"])
    return eng


@pytest.mark.parametrize("p", [0.364, 0.9])
def test_reemission_fp64_matches_oracle(p):
    """FP64 walk + reemission on given packets vs the oracle (same Philox draws,
    seed 0 / iteration 0 of a fresh context): counts and J."""
    g = golden("transport.npz")
    eng = _engine(g, "fp64", p)
    st = eng.transport_packets(0, g["photons"], g["start"])
    _, J = eng.get_fields(0)
    eng.close()
    lat = O.LatticeGrid(g["box"], g["ncell"], g["num_subgrid"])
    Jo = np.zeros_like(g["nH"])
    c = lat.transport(g["nH"], g["xH"], Jo, g["photons"].copy(), g["start"],
                      reemission=(p, 0, 0, 0))
    assert c["reemitted"] > 0
    # sincos/log of the direction draws on the device and on the host may
    # differ in the last bit; with a few hundred re-emissions they do not
    assert st["packets_reemitted"] == c["reemitted"]
    assert st["packets_absorbed"] == c["absorbed"]
    assert st["packets_escaped"] == c["escaped"]
    assert st["cell_crossings"] == c["crossings"]
    np.testing.assert_allclose(J, Jo, rtol=1e-12, atol=1e-300)
    # the fraction of absorptions that were re-emitted
    frac = c["reemitted"] / (c["reemitted"] + c["absorbed"])
    n = c["reemitted"] + c["absorbed"]
    assert abs(frac - p) < 4 * np.sqrt(p * (1 - p) / n)


def test_reemission_fp32_matches_oracle():
    g = golden("transport.npz")
    p = 0.5
    eng = _engine(g, "fp32", p)
    st = eng.transport_packets(0, g["photons"], g["start"])
    eng.close()
    lat = O.LatticeGrid(g["box"], g["ncell"], g["num_subgrid"])
    kappa = O.kappa32(g["nH"], g["xH"])
    q = np.zeros(g["photons"].size, O.PACKET32_DTYPE)
    for i, s in enumerate(int(v) for v in g["start"]):
        d = lat.subgrid_desc(s)
        q["pos"][i] = (g["photons"]["position"][i] - np.array(d.anchor)) * np.array(d.inv_cell_size)
    q["dir"] = g["photons"]["direction"]
    q["tau"] = g["photons"]["tau"]
    c = lat.transport32(kappa, None, q, g["start"], reemission=(p, 0, 0, 0))
    assert st["packets_reemitted"] == c["reemitted"] > 0
    assert st["packets_absorbed"] == c["absorbed"]
    assert st["cell_crossings"] == c["crossings"]


def test_reemission_off_is_unchanged():
    g = golden("transport.npz")
    a = _engine(g, "fp32", 0.0)
    sa = a.transport_packets(0, g["photons"], g["start"])
    a.close()
    assert sa["packets_reemitted"] == 0


def test_reemission_probability_validated():
    g = golden("transport.npz")
    eng = _engine(g, "fp32", 0.0)
    for bad in (-0.1, 1.0, float("nan")):
        with pytest.raises(CMIError):
            eng.set_reemission_probability(0, bad)
    eng.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_stromgren_radius_with_reemission(precision):
    """A 2e49 s^-1 source (so that the larger sphere stays inside the box),
    p = 0.364 (the realistic value of params.txt): the ionized radius grows to
    R_S(Q / (1 - p)) within 2%, and the ratio to the p = 0 radius follows
    (1 - p)^(-1/3) within 2%."""
    Q, p = 2.0e49, 0.364
    radii = {}
    for prob in (0.0, p):
        spec, nH = stromgren(ncell=64, num_subgrid=8, num_photon=1_000_000, luminosity=Q)
        spec.reemission_probability = prob
        eng = TransportEngine(spec, precision=precision)
        eng.set_fields(0, nH)
        st = eng.run_iterations(12, seed=77)
        x, _ = eng.get_fields(0, layout="cube")
        eng.close()
        assert all(s[0]["error_flags"] == 0 for s in st)
        s = st[-1][0]
        assert s["packets_absorbed"] + s["packets_escaped"] == s["packets_emitted"]
        if prob:
            assert s["packets_reemitted"] > 0.2 * s["packets_emitted"]
        radii[prob] = ionized_radius(x.reshape(spec.ncell), spec)
    _, _, Rs0 = stromgren_profile(Q=Q)
    _, _, Rsp = stromgren_profile(Q=Q, reemission_probability=p)
    assert abs(radii[0.0] / Rs0 - 1) < 0.02
    assert abs(radii[p] / Rsp - 1) < 0.02
    assert abs(radii[p] / radii[0.0] / (1 - p) ** (-1 / 3) - 1) < 0.02


@pytest.mark.parametrize("precision", ["mixed", "fp32", "fp64"])
def test_stromgren_reemission_within_reference_ensemble(precision):
    """64^3 Stromgren sphere with reemission probability 0.364, 1e6 packets x
    10 iterations: ionized radius within 3 sigma of the reference's own
    8-seed ensemble (its interact + the driver's do_reemission,
    tests/golden/stromgren_reemission_ensemble.npz) and the radial profile
    bin by bin."""
    from parallelcmacionize_b200.problems import cell_radii
    ens = golden("stromgren_reemission_ensemble.npz")
    spec, nH = stromgren(ncell=64, num_subgrid=8, num_photon=int(ens["packets"]))
    spec.reemission_probability = float(ens["probability"])
    eng = TransportEngine(spec, precision=precision, balance="reference")
    eng.set_fields(0, nH)
    stats = eng.run_iterations(int(ens["iterations"]), seed=4048)
    x, _ = eng.get_fields(0, layout="cube")
    eng.close()
    for it in stats:
        assert it[0]["error_flags"] == 0
    R = ionized_radius(x.reshape(spec.ncell), spec)
    mu, sd = ens["radii"].mean(), ens["radii"].std(ddof=1)
    n = ens["radii"].size
    assert abs(R - mu) < 3 * sd * np.sqrt(1 + 1 / n) + 1e-4 * mu
    r = cell_radii(spec).reshape(-1)
    edges = ens["edges"]
    which = np.digitize(r, edges) - 1
    prof = np.array([x[which == b].mean() if np.any(which == b) else np.nan
                     for b in range(len(edges) - 1)])
    m = np.nanmean(ens["profiles"], axis=0)
    s = np.nanstd(ens["profiles"], axis=0, ddof=1)
    ok = np.isfinite(m) & (s > 0)
    z = np.abs(prof[ok] - m[ok]) / (s[ok] * np.sqrt(1 + 1 / n))
    assert np.mean(z > 3) <= 0.1 and np.median(z) < 2.0
