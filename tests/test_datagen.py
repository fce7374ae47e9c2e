"""The data generator (nrgljubljana_b200.datagen) against the reference's own inputs and
outputs: its Wilson chains equal the xi/zeta tables of the reference's data files, its
initial clusters (the Anderson model, the two-channel Kondo model of spin 1/2 and 1) equal
their multiplets and matrix elements (singlet, doublet and triplet operators), and a run on
a regenerated input reproduces the reference's td/custom outputs and DM-NRG spectra."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
SIAM = ["test0_minimal", "test3_disc_z", "test4_disc_c", "test10_keepmin", "test12_Nmax", "test13_strategy_all",
        "test15_safeguard", "test35_betabar", "legacy_simple", "legacy_Himp"]


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def generate(case):
    from nrgljubljana_b200.datagen import siam_qs
    from nrgljubljana_b200.inputs import parse_param, read_data
    kv = parse_param(read(case, "param"))
    ref = read_data(read(case, "data"))
    return ref, siam_qs(float(kv["U"]), float(kv["delta"]), float(kv["Gamma"]), float(kv.get("Lambda", 2)), ref.nmax,
                        float(kv.get("z", 1)), kv.get("discretization", "Z"), ops=list(ref.ops))


@pytest.mark.parametrize("case", ["test0_minimal", "test4_disc_c", "test12_Nmax", "legacy_simple", "legacy_Himp"])
def test_wilson_chain_matches_reference_tables(case):
    from nrgljubljana_b200.datagen import wilson_chain
    from nrgljubljana_b200.inputs import parse_param, read_data
    kv = parse_param(read(case, "param"))
    d = read_data(read(case, "data"))
    xi, zeta = wilson_chain(float(kv.get("Lambda", 2)), d.nmax, float(kv.get("z", 1)), kv.get("discretization", "Z"))
    assert np.max(np.abs(xi - d.xi[0]) / d.xi[0]) <= 2.3e-16  # the printed 20 digits, rounded once
    assert np.all(zeta == 0.0) and np.all(d.zeta[0] == 0.0)  # particle-hole symmetric band


def test_initial_cluster_matches_reference_data():
    from nrgljubljana_b200.inputs import read_data
    ref, txt = generate("legacy_Himp")
    gen = read_data(txt)
    assert [I for I, _ in gen.subspaces] == [I for I, _ in ref.subspaces]
    for (I, e), (_, f) in zip(gen.subspaces, ref.subspaces):
        assert np.max(np.abs(e - f)) < 1e-14
    assert abs(gen.gs_energy - ref.gs_energy) < 1e-14
    assert set(gen.opch[0][0]) == set(ref.opch[0][0])
    for k, m in ref.opch[0][0].items():  # eigenvector signs are free: compare singular values
        sg = np.linalg.svd(gen.opch[0][0][k], compute_uv=False)
        assert np.max(np.abs(sg - np.linalg.svd(m, compute_uv=False))) < 1e-14
    for name, (kind, mats) in ref.ops.items():
        for k, m in mats.items():
            assert np.max(np.abs(np.diag(gen.ops[name][1][k]) - np.diag(m))) < 1e-13, (name, k)


@pytest.mark.parametrize("case", ["test0_minimal", "test4_disc_c", "test15_safeguard", "legacy_simple", "legacy_Himp"])
def test_regenerated_input_reproduces_reference_outputs(oracle, case):
    from oracle import nrg_run_cpu
    from test_nrg_run import REF_ATOL, REF_RTOL, assert_close, ref_rows
    _, txt = generate(case)
    tdf, td, cf, cu = nrg_run_cpu.run(read(case, "param"), txt, threads=os.cpu_count() or 1)
    assert_close(td, ref_rows(case, "td")[1], REF_RTOL, REF_ATOL, f"{case} td")
    assert_close(cu, ref_rows(case, "custom")[1], REF_RTOL, REF_ATOL, f"{case} custom")


@pytest.mark.gpu
@pytest.mark.parametrize("case", SIAM)
def test_gpu_run_on_regenerated_input(case):
    from nrgljubljana_b200.nrg_run import run_files
    from test_nrg_run import REF_ATOL, REF_RTOL, assert_close, ref_rows
    _, txt = generate(case)
    res = run_files(read(case, "param"), txt)
    assert_close(res.td, ref_rows(case, "td")[1], REF_RTOL, REF_ATOL, f"{case} td")
    assert_close(res.custom, ref_rows(case, "custom")[1], REF_RTOL, REF_ATOL, f"{case} custom")


@pytest.mark.parametrize("case", ["test2_algorithms_dmnrg", "test23_DMNRG"])
def test_regenerated_operators_reproduce_reference_spectra(oracle, case):
    """The generator's A_d (d^dag doublet), n_d (singlet) and sigma_d (triplet) blocks: a
    DM-NRG run on the regenerated input gives the reference's three spectra."""
    from oracle import nrg_run_cpu
    from nrgljubljana_b200.datagen import siam_qs
    from nrgljubljana_b200.inputs import parse_param, read_data
    from test_dmnrg import ATOL_REL_TO_MAX, RTOL, SPECTRA, assert_spectrum, ref_spectrum
    kv = parse_param(read(case, "param"))
    ref = read_data(read(case, "data"))
    txt = siam_qs(float(kv["U"]), float(kv["delta"]), float(kv["Gamma"]), float(kv.get("Lambda", 2)), ref.nmax,
                  float(kv.get("z", 1)), kv.get("discretization", "Z"), ops=["n_d", "A_d", "sigma_d"])
    spec = {}
    nrg_run_cpu.run(read(case, "param"), txt, threads=os.cpu_count() or 1, spectra=spec)
    for name in SPECTRA:
        assert_spectrum(spec[name], ref_spectrum(case, name), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


def test_triplet_elements_match_reference_data():
    """sigma_d of the generator against test23_DMNRG's data (singular values per block:
    the eigenvector signs are free)."""
    from nrgljubljana_b200.datagen import siam_qs
    from nrgljubljana_b200.inputs import parse_param, read_data
    kv = parse_param(read("test23_DMNRG", "param"))
    ref = read_data(read("test23_DMNRG", "data"))
    gen = read_data(siam_qs(float(kv["U"]), float(kv["delta"]), float(kv["Gamma"]), float(kv["Lambda"]), ref.nmax,
                            ops=["sigma_d"]))
    kind, mats = ref.ops["sigma_d"]
    assert gen.ops["sigma_d"][0] == kind == "t"
    assert set(gen.ops["sigma_d"][1]) == set(mats)
    for k, m in mats.items():
        sg = np.linalg.svd(gen.ops["sigma_d"][1][k], compute_uv=False)
        assert np.max(np.abs(sg - np.linalg.svd(m, compute_uv=False)), initial=0.0) < 1e-14, k


# two-channel Kondo inputs: (case, impurity spin, operators of the data file)
KONDO = [("test300_QS_ref", 1.0, []), ("test310_QS_ref", 0.5, ["q_f^2"])]


def generate_kondo(case, spin, ops):
    from nrgljubljana_b200.datagen import kondo_qs
    from nrgljubljana_b200.inputs import parse_param, read_data
    kv = parse_param(read(case, "param"))
    ref = read_data(read(case, "data"))
    return ref, kondo_qs([float(kv["Jkondo1"]), float(kv["Jkondo2"])], spin, float(kv["Lambda"]), ref.nmax,
                         float(kv["z"]), kv["discretization"], ops=ops)


@pytest.mark.parametrize("case,spin,ops", KONDO)
def test_kondo_cluster_matches_reference_data(case, spin, ops):
    from nrgljubljana_b200.inputs import read_data
    ref, txt = generate_kondo(case, spin, ops)
    gen = read_data(txt)
    assert gen.channels == ref.channels == 2
    assert [I for I, _ in gen.subspaces] == [I for I, _ in ref.subspaces]
    for (I, e), (_, f) in zip(gen.subspaces, ref.subspaces):
        assert np.max(np.abs(e - f)) < 1e-14
    assert abs(gen.gs_energy - ref.gs_energy) < 1e-14
    for ch in range(2):
        assert set(gen.opch[ch][0]) == set(ref.opch[ch][0])
        for k, m in ref.opch[ch][0].items():
            sg = np.linalg.svd(gen.opch[ch][0][k], compute_uv=False)
            assert np.max(np.abs(sg - np.linalg.svd(m, compute_uv=False))) < 1e-14
    assert np.max(np.abs(gen.xi[1] - ref.xi[1]) / ref.xi[1]) <= 2.3e-16


@pytest.mark.parametrize("case,spin,ops", KONDO)
def test_regenerated_kondo_input_reproduces_reference_outputs(oracle, case, spin, ops):
    from oracle import nrg_run_cpu
    from test_nrg_run import REF_ATOL, REF_RTOL, assert_close, ref_rows
    _, txt = generate_kondo(case, spin, ops)
    tdf, td, cf, cu = nrg_run_cpu.run(read(case, "param"), txt, threads=os.cpu_count() or 1)
    assert_close(td, ref_rows(case, "td")[1], REF_RTOL, REF_ATOL, f"{case} td")
    assert_close(cu, ref_rows(case, "custom")[1], REF_RTOL, REF_ATOL, f"{case} custom")


@pytest.mark.gpu
@pytest.mark.parametrize("case,spin,ops", KONDO)
def test_gpu_run_on_regenerated_kondo_input(case, spin, ops):
    from nrgljubljana_b200.nrg_run import run_files
    from test_nrg_run import REF_ATOL, REF_RTOL, assert_close, ref_rows
    _, txt = generate_kondo(case, spin, ops)
    res = run_files(read(case, "param"), txt)
    assert_close(res.td, ref_rows(case, "td")[1], REF_RTOL, REF_ATOL, f"{case} td")
    assert_close(res.custom, ref_rows(case, "custom")[1], REF_RTOL, REF_ATOL, f"{case} custom")
