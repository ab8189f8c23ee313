"""The C++ host surface (include/cmacionize/*.hpp) over the C ABI."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DRIVER = os.path.join(ROOT, "parallelcmacionize_b200", "stromgren_driver")

PARAMS = """## Physical parameters
box:
  anchor: [-5. pc, -5. pc, -5. pc]
  sides: [10. pc, 10. pc, 10. pc]
ncell: [{n}, {n}, {n}]
num_photon: {photons}
number_of_iterations: {iters}
reemission_probability: 0.
number_of_sources: 1
random_density: false
## Algorithm parameters
num_subgrid: [{s}, {s}, {s}]
queue_size_per_thread: 100
memoryspace_size: 50000
number_of_tasks: 500000
MPI_buffer_size: 1000
cost_copy_factor: 10
edge_copy_factor: 0.01
general_queue_size: 100000
"""


def test_headers_compile_against_the_abi(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(
        '#include "cmacionize/DensityGrid.hpp"\n#include "cmacionize/Parameters.hpp"\n'
        '#include <cassert>\n#include <sstream>\n'
        "int main() {\n"
        "  assert(TravelDirections::output_to_input_direction(TRAVELDIRECTION_CORNER_PPN)"
        " == TRAVELDIRECTION_CORNER_NNP);\n"
        "  assert(TravelDirections::get_output_direction(9) == TRAVELDIRECTION_EDGE_X_PN);\n"
        "  RandomGenerator r(42); double u = r.get_uniform_random_double(); assert(u >= 0 && u < 1);\n"
        '  std::istringstream s("box:\\n  anchor: [0 pc, 0 pc, 0 pc]\\n");\n'
        "  Parameters p(s); double a[3]; p.get_physical_vector(\"box:anchor\", a);\n"
        "  PhotonBuffer b; b.grow(3); assert(b.size() == 3);\n"
        "  return 0;\n}\n")
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe)], check=True)
    subprocess.run([str(exe)], check=True)


def test_ranlxd_header_matches_reference_stream(tmp_path):
    """The shared ranlxd header (host + device) reproduces RandomGenerator."""
    from conftest import golden
    g = golden("rng.npz")
    src = tmp_path / "r.cpp"
    src.write_text('#include "cmacionize/RandomGenerator.hpp"\n#include <cstdio>\n#include <cstdlib>\n'
                   "int main(int c, char **v) { RandomGenerator r(atoi(v[1]));\n"
                   "  for (int i = 0; i < 2500; ++i) printf(\"%a\\n\", r.get_uniform_random_double()); }\n")
    exe = tmp_path / "r"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe)], check=True)
    for seed, ref in zip(g["seeds"], g["streams"]):
        out = subprocess.run([str(exe), str(int(seed))], check=True, capture_output=True,
                             text=True).stdout.split()
        assert np.array_equal(np.array([float.fromhex(x) for x in out]), ref)


def test_stromgren_driver_rejects_bad_input(tmp_path):
    """Command-line and params.txt errors end the driver with a message and a
    non-zero status before any device work.  The reference stops on the same
    inputs through cmac_error (a missing key: YAMLDictionary.hpp:562)."""
    if not os.path.exists(DRIVER):
        pytest.fail("stromgren_driver not built (make -C parallelcmacionize_b200/csrc)")
    r = subprocess.run([DRIVER], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([DRIVER, "-t", "1", "-p", str(tmp_path / "absent.txt")],
                       cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "unable to open" in r.stderr
    p = tmp_path / "params.txt"
    p.write_text("box:\n  anchor: [-5. pc, -5. pc, -5. pc]\n")
    r = subprocess.run([DRIVER, "-t", "1", "-p", str(p)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and 'missing parameter "box:sides"' in r.stderr
    assert not (tmp_path / "neutral_fractions.bin").exists()


def _random_case():
    from conftest import golden
    g = golden("outputs_random.npz")
    from parallelcmacionize_b200.outputs import DAT_RECORD
    return g, g["dat"].view(DAT_RECORD)


def test_random_density_header_matches_reference_files(tmp_path):
    """CosineDensityField (the driver's random_density set-up) gives the n_H
    the reference driver wrote to its .dat file, bit for bit, when seeded as
    the reference seeds its host generator (42 + threads)."""
    g, rec = _random_case()
    pc = 3.086e16
    box = [float(v) * pc for v in g["anchor_pc"]] + [float(v) * pc for v in g["sides_pc"]]
    src = tmp_path / "d.cpp"
    src.write_text(
        '#include "cmacionize/RandomDensity.hpp"\n#include <cstdio>\n#include <cstdlib>\n'
        "int main(int c, char **v) {\n"
        "  double box[6]; for (int a = 0; a < 6; ++a) box[a] = strtod(v[1 + a], nullptr);\n"
        "  int ns[3], n[3]; for (int a = 0; a < 3; ++a) { ns[a] = atoi(v[7 + a]);"
        " n[a] = atoi(v[10 + a]) / ns[a]; }\n"
        "  RandomGenerator rng(42 + atoi(v[13])); const CosineDensityField f(rng, box);\n"
        "  for (int s = 0; s < ns[0] * ns[1] * ns[2]; ++s) {\n"
        "    const int si[3] = {s / (ns[1] * ns[2]), (s / ns[2]) % ns[1], s % ns[2]};\n"
        "    double sb[6]; for (int a = 0; a < 3; ++a) { sb[3 + a] = box[3 + a] / ns[a];"
        " sb[a] = box[a] + si[a] * sb[3 + a]; }\n"
        "    for (int q = 0; q < n[0] * n[1] * n[2]; ++q) {\n"
        "      const int i3[3] = {q / (n[1] * n[2]), (q / n[2]) % n[1], q % n[2]};\n"
        "      double m[3]; CosineDensityField::cell_midpoint(sb, n, i3, m);\n"
        '      printf("%a %a %a %a\\n", m[0], m[1], m[2], f(m));\n'
        "    }\n  }\n}\n")
    exe = tmp_path / "d"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    args = [repr(float(b)) for b in box] + [str(int(v)) for v in g["num_subgrid"]] + \
        [str(int(v)) for v in g["ncell"]] + [str(int(g["threads"]))]
    out = subprocess.run([str(exe)] + args, check=True, capture_output=True, text=True).stdout
    got = np.array([[float.fromhex(x) for x in line.split()] for line in out.splitlines()])
    assert got.shape == (rec.size, 4)
    assert np.array_equal(got[:, :3], rec["pos"])
    assert np.array_equal(got[:, 3], rec["nH"])
    # a field with structure, not the uniform 1e8
    assert rec["nH"].std() > 0.05 * rec["nH"].mean()


@pytest.mark.gpu
def test_stromgren_driver_random_density(tmp_path):
    """The driver with random_density: true and the reference's command line
    writes the reference's cell centres and n_H bit for bit; x_H comes from
    a different (device) packet stream and is compared statistically."""
    if not os.path.exists(DRIVER):
        pytest.fail("stromgren_driver not built (make -C parallelcmacionize_b200/csrc)")
    g, rec = _random_case()
    p = tmp_path / "params.txt"
    p.write_text(str(g["params"]))
    r = subprocess.run([DRIVER, "-t", str(int(g["threads"])), "-p", str(p)], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    from parallelcmacionize_b200.outputs import read_neutral_fractions_dat
    ours = read_neutral_fractions_dat(tmp_path / "neutral_fractions.dat")
    assert ours.size == rec.size
    assert np.array_equal(ours["pos"], rec["pos"])
    assert np.array_equal(ours["nH"], rec["nH"])
    assert np.array_equal(ours["hydro"], rec["hydro"])
    x = np.fromfile(tmp_path / "neutral_fractions.bin", dtype=np.float64)
    assert np.array_equal(x, ours["xH"])
    assert np.all((x > 0) & (x <= 1))
    # 2e4 packets over 2048 cells: cell values are noisy, the mean is not
    assert abs(x.mean() - rec["xH"].mean()) < 0.05 * rec["xH"].mean() + 0.01


@pytest.mark.gpu
def test_stromgren_driver_runs(tmp_path):
    """The reference's command line and params.txt, on the GPU path."""
    if not os.path.exists(DRIVER):
        pytest.fail("stromgren_driver not built (make -C parallelcmacionize_b200/csrc)")
    p = tmp_path / "params.txt"
    p.write_text(PARAMS.format(n=32, s=4, photons=200000, iters=6))
    r = subprocess.run([DRIVER, "-t", "1", "-p", str(p)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Total Monte Carlo time" in r.stderr
    x = np.fromfile(tmp_path / "neutral_fractions.bin", dtype=np.float64)
    assert x.size == 32 ** 3
    assert np.all((x > 0) & (x <= 1))
    from parallelcmacionize_b200.engine import blocked_to_cube
    from parallelcmacionize_b200.problems import GridSpec, ionized_radius, stromgren_profile
    spec = GridSpec(box=(-5 * 3.086e16,) * 3 + (10 * 3.086e16,) * 3, ncell=(32,) * 3,
                    num_subgrid=(4,) * 3)
    R = ionized_radius(blocked_to_cube(x, spec.ncell, spec.num_subgrid), spec)
    _, _, Rs = stromgren_profile()
    assert abs(R / Rs - 1) < 0.05  # coarse 32^3 grid
    # the .dat file: the same x_H, n_H = 1e8 (uniform params), and the
    # reference's record layout and cell centres (Python writer, pinned to
    # the reference's own files in tests/test_outputs.py)
    from parallelcmacionize_b200.outputs import neutral_fractions_dat
    dat = np.fromfile(tmp_path / "neutral_fractions.dat", dtype=np.uint8)
    ref = neutral_fractions_dat(spec, x, np.full(x.size, 1e8))
    assert np.array_equal(dat, ref.view(np.uint8))
