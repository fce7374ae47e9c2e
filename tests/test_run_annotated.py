"""annotated.dat (Annotated::dump, c++/output.hpp:77-125): the lowest `dumpannotated` energies
of every step's computed states (and of the initial subspaces, calc0), extended over a
degenerate cluster at the cut and grouped by degeneracy, "E (Q SS) ... [multiplicity]".
The oracle against the reference's files of every regression case that has one; the run driver's formatter
(nrg_run.annotated_lines) against the oracle on the same cases and on hand-made edge cases;
the device run against the reference."""
import os

import pytest

from nrgljubljana_b200.nrg_run import RunParams, annotated_lines

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
CASES = sorted(c for c in os.listdir(GOLD) if os.path.exists(os.path.join(GOLD, c, "annotated.dat")))
E_RTOL, E_ATOL = 2e-7, 1e-9  # energies printed to 8 significant digits


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def assert_annotated(got_lines, want_text, what):
    want = want_text.split("\n")
    while want and want[-1] == "":
        want.pop()
    got = list(got_lines)
    while got and got[-1] == "":
        got.pop()
    assert len(got) == len(want), f"{what}: {len(got)} lines vs {len(want)}"
    for k, (g, w) in enumerate(zip(got, want)):
        if w == "":
            assert g == "", f"{what} line {k}: {g!r} vs block end"
            continue
        ge, grest = g.split(" ", 1)
        we, wrest = w.split(" ", 1)
        assert grest == wrest, f"{what} line {k}: {g!r} vs {w!r}"
        assert abs(float(ge) - float(we)) <= E_RTOL * abs(float(we)) + E_ATOL, f"{what} line {k}: {g!r} vs {w!r}"


@pytest.fixture(scope="module")
def oracle_annotated(oracle):
    from oracle import nrg_run_cpu
    cache = {}

    def get(case):
        if case not in cache:
            lines = []
            nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, annotated_out=lines)
            cache[case] = lines
        return cache[case]
    return get


def test_cases_present():
    assert len(CASES) >= 18


@pytest.mark.parametrize("case", CASES)
def test_oracle_annotated_matches_reference(oracle_annotated, case):
    assert_annotated(oracle_annotated(case), read(case, "annotated.dat"), case)


def test_formatter_edge_cases():
    p = RunParams.from_param({"dumpannotated": "4"})
    # a cluster at the cut (within grouptol = 1e-6 relative) is dumped whole; equal energies of
    # different subspaces are one group, their labels sorted as strings
    entries = [(0.0, (0, 1)), (0.5, (1, 2)), (0.5, (-1, 2)), (0.7, (10, 1)), (0.7 * (1 + 1e-7), (2, 1)),
               (0.9, (0, 3))]
    assert annotated_lines(entries, p, 1.0, 0.0) == ["0 (0 1) [1]", "0.5 (-1 2) (1 2) [4]",
                                                     "0.7 (10 1) (2 1) [2]", ""]
    p = RunParams.from_param({"dumpannotated": "2", "dumpgroups": "false", "dumpscaled": "false",
                              "dumpprecision": "4"})
    assert annotated_lines([(0.0, (0, 1)), (0.123456, (1, 2)), (2.0, (0, 1))], p, 2.0, 0.0) == \
        ["0 0 1", "0.2469 1 2", ""]


@pytest.mark.parametrize("case", CASES)
def test_formatter_matches_oracle(oracle_annotated, case):
    """The driver's formatter, fed the oracle's eigenvalues step by step, writes the same lines."""
    from oracle import nrg_run_cpu
    blocks = []
    nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, annotated_out=[],
                    annotated_entries=blocks)
    p = RunParams.from_param({k: v for k, v in nrg_run_cpu.parse_param(read(case, "param")).items()
                              if k in RunParams.__dataclass_fields__})
    lines = []
    for entries, scale, etot in blocks:
        lines += annotated_lines(entries, p, scale, etot)
    assert lines == oracle_annotated(case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_annotated(case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert_annotated(res.annotated, read(case, "annotated.dat"), f"{case} (device run)")
