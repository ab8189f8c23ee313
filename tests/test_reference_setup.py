"""The reference driver's initial conditions from Python
(parallelcmacionize_b200.problems.reference_setup, parallelcmacionize_b200.ranlxd)
against the reference's own outputs: its RandomGenerator streams
(tests/golden/rng.npz) and the result file of its random_density run
(tests/golden/outputs_random.npz)."""
import numpy as np
import pytest

from conftest import golden

from parallelcmacionize_b200.outputs import DAT_RECORD
from parallelcmacionize_b200.params import Parameters
from parallelcmacionize_b200.problems import reference_setup
from parallelcmacionize_b200.ranlxd import Ranlxd

PARAMS = """box:
  anchor: [-5. pc, -4. pc, -3. pc]
  sides: [10. pc, 8. pc, 6. pc]
ncell: [8, 8, 4]
num_photon: 1000
number_of_iterations: 1
reemission_probability: 0.
number_of_sources: {sources}
random_density: {random}
num_subgrid: [2, 2, 1]
"""


def test_ranlxd_matches_reference_streams():
    g = golden("rng.npz")
    for seed, ref in zip(g["seeds"], g["streams"]):
        r = Ranlxd(int(seed))
        assert np.array_equal(np.array([r.uniform() for _ in range(ref.size)]), ref), seed


def test_random_density_matches_reference_file():
    g = golden("outputs_random.npz")
    rec = g["dat"].view(DAT_RECORD)
    spec, nH = reference_setup(Parameters.from_text(str(g["params"])), threads=int(g["threads"]))
    assert np.array_equal(nH, rec["nH"])
    assert spec.sources == [(0.0, 0.0, 0.0, 4.26e49)]
    assert spec.num_photon == 20000 and spec.ncell == (16, 16, 8)


@pytest.mark.parametrize("random", [False, True])
def test_random_sources_follow_the_density_draws(random):
    """Source k takes draws 3k..3k+2 after the density's 70 (10 modes x 7),
    seed 42 + threads (threads = 0: the golden seed-42 stream)."""
    stream = golden("rng.npz")
    ref = stream["streams"][list(stream["seeds"]).index(42)]
    p = Parameters.from_text(PARAMS.format(sources=3, random="true" if random else "false"))
    spec, nH = reference_setup(p, threads=0)
    first = 70 if random else 0
    box = p.box
    for k, src in enumerate(spec.sources):
        want = [box[a] + ref[first + 3 * k + a] * box[3 + a] for a in range(3)]
        assert list(src[:3]) == want and src[3] == 4.26e48
    if not random:
        assert np.all(nH == 1e8)
    else:
        assert nH.std() > 0.05 * nH.mean() and np.all(nH >= 0)
