"""cmi_walk_photons (the dust driver's per-photon DensitySubGrid::propagate
and compute_optical_depth) on the GPU against the reference's own results
(tests/golden/dust_walks.npz, from the reference harness): every output
direction and every photon field bit for bit; and the C++ surface's
DensitySubGrid::propagate / compute_optical_depth on one photon."""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden
from parallelcmacionize_b200 import CMIError, GridSpec, TransportEngine

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIELDS = ("position", "direction", "tau", "sigma", "weight", "type")


@pytest.mark.parametrize("case", ["interior16", "entries8", "noncubic"])
@pytest.mark.parametrize("depth", [False, True])
def test_walks_match_reference(case, depth):
    g = golden(f"walk_{case}.npz")
    d = golden("dust_walks.npz")
    ph, dirs = g["photons"], g["in_dirs"]
    if depth:
        ref, res_ref = d[f"{case}_depth_out"], d[f"{case}_depth_res"]
    else:
        keep = d[f"{case}_keep"]
        ph, dirs = ph[keep], dirs[keep]
        ref, res_ref = d[f"{case}_prop_out"], d[f"{case}_prop_res"]
    spec = GridSpec(box=tuple(g["box"]), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=(1, 1, 1))
    with TransportEngine(spec, precision="fp64") as eng:
        eng.set_fields(0, g["nH"], g["xH"])
        out, res = eng.walk_photons(0, 0, ph, dirs, depth=depth)
    assert np.array_equal(res, res_ref)
    for f in FIELDS:
        assert out[f].tobytes() == ref[f].tobytes(), f


def test_walk_arguments():
    g = golden("walk_interior16.npz")
    spec = GridSpec(box=tuple(g["box"]), ncell=(16, 16, 16), num_subgrid=(1, 1, 1))
    with TransportEngine(spec) as eng:
        eng.set_fields(0, g["nH"], g["xH"])
        with pytest.raises(CMIError):
            eng.walk_photons(0, 1, g["photons"][:2], 0)   # no subgrid 1
        with pytest.raises(CMIError):
            eng.walk_photons(0, 0, g["photons"][:2], 27)  # no direction 27


def test_cpp_surface_propagate(tmp_path):
    """DensitySubGrid::propagate and compute_optical_depth of the C++ surface
    on the first photon of the interior case, against the reference."""
    g = golden("walk_interior16.npz")
    d = golden("dust_walks.npz")
    src = tmp_path / "w.cpp"
    p = g["photons"][0]
    nh = ",".join(repr(float(v)) for v in g["nH"])
    xh = ",".join(repr(float(v)) for v in g["xH"])
    box = ",".join(repr(float(v)) for v in g["box"])
    src.write_text(f'''#include <cstdio>
#include "cmacionize/DensityGrid.hpp"
static const double NH[] = {{{nh}}}, XH[] = {{{xh}}};
int main() {{
  const double box[6] = {{{box}}};
  const int n[3] = {{16, 16, 16}}, ns[3] = {{1, 1, 1}};
  DensityGrid grid(box, n, ns);
  DensitySubGrid sg = grid.subgrid(0);
  for (int c = 0; c < 4096; ++c) {{ sg.set_number_density(c, NH[c]); sg.set_neutral_fraction(c, XH[c]); }}
  for (int mode = 0; mode < 2; ++mode) {{
    Photon ph;
    ph.set_position({float(p["position"][0])!r}, {float(p["position"][1])!r}, {float(p["position"][2])!r});
    ph.set_direction({float(p["direction"][0])!r}, {float(p["direction"][1])!r}, {float(p["direction"][2])!r});
    ph.set_target_optical_depth({float(p["tau"])!r});
    ph.set_photoionization_cross_section({float(p["sigma"])!r});
    ph.set_weight({float(p["weight"])!r});
    const int r = mode ? sg.compute_optical_depth(ph, 0) : sg.propagate(ph, 0);
    std::printf("%d %a %a %a %a\\n", r, ph.get_position()[0], ph.get_position()[1],
                ph.get_position()[2], ph.get_target_optical_depth());
  }}
}}
''')
    exe = tmp_path / "w"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", os.path.join(ROOT, "parallelcmacionize_b200"),
                    "-lcmacionize_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "parallelcmacionize_b200")], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True,
                           text=True).stdout.split("\n")
    for line, key in zip(lines, ("prop", "depth")):
        f = line.split()
        ref = d[f"interior16_{key}_out"][0]
        assert int(f[0]) == int(d[f"interior16_{key}_res"][0])
        assert [float.fromhex(v) for v in f[1:4]] == list(ref["position"])
        assert float.fromhex(f[4]) == ref["tau"]
