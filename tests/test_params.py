"""The params.txt reader (parallelcmacionize_b200/params.py): the keys of the
reference driver (testDensitySubGrid_omp.cpp:948-1013), YAML nesting and
comments (YAMLDictionary.hpp), length units (UnitConverter.hpp), and the
errors on missing or malformed values."""
import pytest

from parallelcmacionize_b200.params import ParameterError, Parameters, parse_yaml_subset

PC = 3.086e16

TEXT = """## Physical parameters
box:
  anchor: [-5. pc, -4 pc, -3.e0 pc]   # a comment
  sides: [10. pc, 8 pc, 6 pc]
ncell: [32, 16, 8]
num_photon: 1e6
number_of_iterations: 10
reemission_probability: 0.364
number_of_sources: 1
random_density: false
## Algorithm parameters
num_subgrid: [4, 2, 1]
queue_size_per_thread: 100
cost_copy_factor: 10
"""


def test_keys_units_and_nesting():
    p = Parameters.from_text(TEXT)
    assert p.box == (-5 * PC, -4 * PC, -3 * PC, 10 * PC, 8 * PC, 6 * PC)
    assert p.ncell == (32, 16, 8) and p.num_subgrid == (4, 2, 1)
    assert p.num_photon == 1_000_000 and p.number_of_iterations == 10
    assert p.reemission_probability == 0.364
    assert p.number_of_sources == 1 and p.random_density is False
    assert p.capacity == {"queue_size_per_thread": 100.0, "cost_copy_factor": 10.0}
    d = parse_yaml_subset(TEXT)
    assert d["box:anchor"].startswith("[-5. pc") and "anchor" not in d


def test_round_trip_through_text():
    p = Parameters.from_text(TEXT)
    q = Parameters.from_text(p.to_text())
    assert (q.box, q.ncell, q.num_subgrid, q.num_photon, q.number_of_iterations,
            q.reemission_probability, q.number_of_sources, q.random_density) == \
        (p.box, p.ncell, p.num_subgrid, p.num_photon, p.number_of_iterations,
         p.reemission_probability, p.number_of_sources, p.random_density)


@pytest.mark.parametrize("value,expected", [("true", True), ("yes", True), ("1", True),
                                            ("false", False), ("no", False), ("0", False)])
def test_booleans(value, expected):
    assert Parameters.from_text(TEXT.replace("random_density: false",
                                             f"random_density: {value}")).random_density is expected


@pytest.mark.parametrize("edit,message", [
    (("number_of_sources: 1\n", ""), "missing parameter"),
    (("random_density: false", "random_density: maybe"), "not a boolean"),
    (("num_photon: 1e6", "num_photon: -5"), "unsigned integer"),
    (("num_photon: 1e6", "num_photon: 2.5"), "unsigned integer"),
    (("sides: [10. pc, 8 pc, 6 pc]", "sides: [10. pc, 8 pc]"), "3 components"),
    (("sides: [10. pc, 8 pc, 6 pc]", "sides: [10. parsec, 8 pc, 6 pc]"), "unknown unit"),
    (("ncell: [32, 16, 8]", "ncell: [30, 16, 8]"), "multiple of num_subgrid"),
    (("ncell: [32, 16, 8]", "ncell 32"), "cannot parse"),
])
def test_errors(edit, message):
    with pytest.raises(ParameterError, match=message):
        Parameters.from_text(TEXT.replace(*edit))


def test_cpp_surface_reads_the_same_values(tmp_path):
    """include/cmacionize/Parameters.hpp (the C++ surface) and this reader
    agree on every plain-method value of the same file, bit for bit."""
    import os
    import subprocess

    from conftest import ROOT
    src = tmp_path / "p.cpp"
    src.write_text(
        '#include "cmacionize/Parameters.hpp"\n#include <cstdio>\n'
        "int main(int c, char **v) {\n"
        "  const PlainMethodParameters p(Parameters::from_file(v[1]));\n"
        '  for (double b : p.box) printf("%a\\n", b);\n'
        '  printf("%a\\n", p.reemission_probability);\n'
        '  for (int a = 0; a < 3; ++a) printf("%d %d\\n", p.ncell[a], p.num_subgrid[a]);\n'
        '  printf("%u %u %u %d\\n", p.num_photon, p.number_of_iterations,'
        " p.number_of_sources, (int)p.random_density);\n}\n")
    exe = tmp_path / "p"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    for text in (TEXT, TEXT.replace("random_density: false", "random_density: yes")
                 .replace("number_of_sources: 1", "number_of_sources: 3")):
        f = tmp_path / "params.txt"
        f.write_text(text)
        out = subprocess.run([str(exe), str(f)], check=True, capture_output=True,
                             text=True).stdout.split("\n")
        p = Parameters.from_text(text)
        assert [float.fromhex(v) for v in out[:6]] == list(p.box)
        assert float.fromhex(out[6]) == p.reemission_probability
        assert [tuple(map(int, out[7 + a].split())) for a in range(3)] == \
            list(zip(p.ncell, p.num_subgrid))
        assert list(map(int, out[10].split())) == [p.num_photon, p.number_of_iterations,
                                                   p.number_of_sources, int(p.random_density)]
