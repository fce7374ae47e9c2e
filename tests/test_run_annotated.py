"""annotated.dat and energies.nrg.
annotated.dat (Annotated::dump, c++/output.hpp:77-125): the lowest `dumpannotated` energies
of every step's computed states (and of the initial subspaces, calc0), extended over a
degenerate cluster at the cut and grouped by degeneracy, "E (Q SS) ... [multiplicity]".
The oracle against the reference's files of every regression case that has one; the run driver's formatter
(nrg_run.annotated_lines) against the oracle on the same cases and on hand-made edge cases;
the device run against the reference. energies.nrg (Output::dump_energies,
c++/output.hpp:157-161, dumpenergies=true): every computed level of every step by subspace,
the oracle and the device run against the reference's file, the formatter on a hand-made step."""
import os

import pytest

from nrgljubljana_b200.nrg_run import RunParams, annotated_lines, energies_block

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


# the device run's file on a subset: every dump option, one and two channels, the largest case
GPU_CASES = ["test17_dumpannotated", "test18_dumpscaled", "test19_dumpabs", "test20_dumpgroups", "test68_grouptol",
             "test56_dsyevr", "test300_QS_ref", "legacy_one_jkondonew"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES)
def test_gpu_annotated(case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert_annotated(res.annotated, read(case, "annotated.dat"), f"{case} (device run)")


ENERGY_CASES = sorted(c for c in os.listdir(GOLD) if os.path.exists(os.path.join(GOLD, c, "energies.nrg")))


def parse_energies(text):
    """[(label, [((Q, SS), [levels])])] of an energies.nrg text."""
    blocks = []
    for line in text.split("\n"):
        if line.startswith("===== Iteration number: "):
            blocks.append((int(line.split(":")[1]), []))
        elif line.startswith("Subspace: "):
            q, ss = line.split()[1:3]
            blocks[-1][1].append(((int(q), int(ss)), None))
        elif line.strip():
            I, _ = blocks[-1][1][-1]
            blocks[-1][1][-1] = (I, [float(x) for x in line.split()])
    return blocks


def assert_energies(got_text, want_text, what):
    got, want = parse_energies(got_text), parse_energies(want_text)
    assert [(lab, [I for I, _ in subs]) for lab, subs in got] == [(lab, [I for I, _ in subs]) for lab, subs in want], what
    for (lab, gs), (_, ws) in zip(got, want):
        for (I, g), (_, w) in zip(gs, ws):
            assert len(g) == len(w) and all(abs(a - b) <= 1e-5 * abs(b) + 1e-9 for a, b in zip(g, w)), (what, lab, I)


def test_energy_cases_present():
    assert ENERGY_CASES == ["test62_dumpenergies"]


@pytest.mark.parametrize("case", ENERGY_CASES)
def test_oracle_energies_match_reference(oracle, case):
    from oracle import nrg_run_cpu
    out = []
    nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, energies_out=out)
    assert_energies("".join(out), read(case, "energies.nrg"), case)


def test_energies_formatter():
    import numpy as np
    text = energies_block(3, {(1, 2): np.array([0.25, 1.0 / 3.0]), (-1, 2): np.array([0.0, 1e-5, 12345678.0])})
    assert text == ("\n===== Iteration number: 3\nSubspace: -1 2\n0 1e-05 1.23457e+07 \n"
                    "Subspace: 1 2\n0.25 0.333333 \n")


@pytest.mark.gpu
@pytest.mark.parametrize("case", ENERGY_CASES)
def test_gpu_energies(case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert_energies("".join(res.energies), read(case, "energies.nrg"), f"{case} (device run)")


SUBSPACE_CASES = sorted(c for c in os.listdir(GOLD) if os.path.exists(os.path.join(GOLD, c, "subspaces.dat")))


def test_subspace_cases_present():
    assert SUBSPACE_CASES == ["test63_dumpsubspaces", "test_dmnrg_only"]


@pytest.mark.parametrize("case", SUBSPACE_CASES)
def test_oracle_subspaces_match_reference(oracle, case):
    """subspaces.dat (Store::dump_subspaces, c++/store.hpp:75-84): per step the number of
    subspaces and each one's kept and computed states, exactly."""
    from oracle import nrg_run_cpu
    out = []
    nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, subspaces_out=out)
    assert "".join(line + "\n" for line in out) == read(case, "subspaces.dat")


@pytest.mark.gpu
@pytest.mark.parametrize("case", SUBSPACE_CASES)
def test_gpu_subspaces(case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert "".join(line + "\n" for line in res.subspaces) == read(case, "subspaces.dat")
