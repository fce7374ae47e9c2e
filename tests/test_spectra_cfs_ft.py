"""Complete-Fock-space (CFS) and conventional finite-temperature (FT) spectra of whole runs
against the reference's regression outputs: {spec,corr,spin}_{CFS,CFSgt,CFSls}_dens_*.dat of
test/c++/test2_algorithms_cfs, test2_algorithms_cfsgtls and test_cfs_only, and every
spectrum (DMNRG, FDM, CFS, FT) and the FDM expectation values of test2_algorithms and
test11_T, which run the four algorithms together.
CFS (Algo_CFSgt, Algo_CFSls, c++/algo_CFS.hpp): the DM-NRG density matrices, the operators
recalculated over all states, the last step's kept-kept term with Boltzmann weights over
Z_ft and, at the other steps, the discarded-kept terms with rho, merged whole. FT (Algo_FT,
c++/algo_FT.hpp): kept-kept terms with ((-sign) e^{-E1/T} + e^{-Ep/T}) / Z_ft of the step,
merged with the N/N+2 window. The device run builds both from the FDM pair modes of
nrg_spec_accumulate; `test_cfs_terms_by_fdm_modes` and `test_ft_terms_by_fdm_modes` check
that composition bin by bin with the oracle's direct terms and its FDM pair sums."""
import os

import numpy as np
import pytest

from test_dmnrg import ATOL_REL_TO_MAX, ORA_ATOL_REL_TO_MAX, ORA_RTOL, RTOL, assert_spectrum

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
CFS_CASES = ["test2_algorithms_cfs", "test2_algorithms_cfsgtls", "test_cfs_only",
             "legacy_sigma_trick_siam_qs",  # keep 5000, four spectra with cross pairs A_d-B_d, B_d-A_d
             "legacy_globalop_Q1Q2-QS"]  # two channels: correlators of the global charges Q1, Q2, Qdiff
ALL_CASES = ["test2_algorithms", "test11_T", "test55_gt_ls",  # DMNRG + FDM + CFS + FT (and gt/ls parts)
             "test2_algorithms_finite",  # FT alone
             "legacy_substeps_one_siam_std"]  # DMNRG + FDM + CFS + FT with tdfdm
TAB_RTOL = 2e-9  # customfdm printed to 10 significant digits


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def rows(case, name):
    return np.array([[float(x) for x in line.split()] for line in read(case, name).splitlines()
                     if line.strip() and not line.startswith("#")])


def spectrum_files(case):
    return sorted(f[:-4] for f in os.listdir(os.path.join(GOLD, case))
                  if f.endswith(".dat") and f.startswith(("spec_", "corr_", "spin_")))


@pytest.fixture(scope="module")
def oracle_cfs(oracle):
    from oracle import nrg_run_cpu
    cache = {}

    def get(case):
        if case not in cache:
            spec, fo = {}, {}
            nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, spectra=spec,
                            fdm_out=fo)
            cache[case] = (spec, fo)
        return cache[case]
    return get


def assert_customfdm(got, case, what, name="customfdm"):
    if os.path.exists(os.path.join(GOLD, case, name)):
        want = rows(case, name)[-1]
        got = np.asarray(got, dtype=float)
        # plus 1e-12 of the row's scale: C_fdm = <E^2> - <E>^2 of a degenerate ground state at low
        # T is cancellation noise (1e-23 here) in the reference's sums and in these alike
        atol = 1e-12 * np.abs(want).max()
        assert got.shape == want.shape and np.all(np.abs(got - want) <= TAB_RTOL * np.abs(want) + atol), what


@pytest.mark.parametrize("case", CFS_CASES + ALL_CASES)
def test_oracle_cfs_spectra_match_reference(oracle_cfs, case):
    spec, fo = oracle_cfs(case)
    assert sorted(spec) == spectrum_files(case)
    for name in spectrum_files(case):
        assert_spectrum(spec[name], rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")
    for name in ("customfdm", "tdfdm"):
        if name in fo:
            assert_customfdm(fo[name][1], case, f"{case} {name}", name)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CFS_CASES + ALL_CASES)
def test_gpu_cfs_spectra(oracle_cfs, case):
    """The device run's CFS (and FT, DMNRG, FDM) spectra against the reference and the oracle."""
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    spec, fo = oracle_cfs(case)
    assert sorted(res.spectra) == spectrum_files(case)
    for name in spectrum_files(case):
        got = res.spectra[name]
        assert_spectrum(got, rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name} vs reference")
        assert_spectrum(got, spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} {name} vs oracle")
    for name in ("customfdm", "tdfdm"):
        if getattr(res, name) is not None:
            assert_customfdm(getattr(res, name)[1], case, f"{case} {name}", name)


def fdm_mode_composition(cb, last, Ei, ki, Ej, kj, o1, o2, rho_i, rho_j, factor, sign, T, Zft):
    """The CFS terms of one pair as the device run forms them from the FDM pair modes
    (nrg_run.QSRun._cfs_pairs): at the last step, the FDMgt / FDMls D x D term over the kept
    states (K = 0, the pair cut to the kept states) with wnf = 1/Z_ft; at the other steps, the
    FDMgt K(Ii) x D(Ij) term with op2 rho(Ii) (CFSls) and the FDMls D(Ii) x K(Ij) term with the
    two operators swapped and rho(Ij) (CFSgt), wnf = 0 and the factor times -sign."""
    empty = np.zeros((0, 0))
    if last:
        cb["gt"].fdm_pair("gt", Ei[:ki], 0, Ej[:kj], 0, o1[:kj, :ki], o2[:kj, :ki], empty, factor, sign, T, 1.0 / Zft)
        cb["ls"].fdm_pair("ls", Ei[:ki], 0, Ej[:kj], 0, o1[:kj, :ki], o2[:kj, :ki], empty, factor, sign, T, 1.0 / Zft)
    else:
        cb["ls"].fdm_pair("gt", Ei, ki, Ej, kj, o1, o2, rho_i, -sign * factor, sign, T, 0.0)
        cb["gt"].fdm_pair("ls", Ei, ki, Ej, kj, o2, o1, rho_j, -sign * factor, sign, T, 0.0)


@pytest.mark.parametrize("sign", [1, -1])
@pytest.mark.parametrize("last,keep_all", [(False, False), (True, True), (True, False)])
def test_cfs_terms_by_fdm_modes(oracle, sign, last, keep_all):
    from oracle import nrg_run_cpu
    from oracle.oracle import ChainBinning
    rng = np.random.default_rng(11 + sign + 2 * last + 4 * keep_all)
    ni, nj = 9, 7
    ki, kj = (ni, nj) if keep_all else (4, 3)
    Ei = np.sort(rng.uniform(0.0, 3.0, ni))
    Ej = np.sort(rng.uniform(0.0, 3.0, nj))
    Ei -= Ei[0]
    Ej -= Ej[0]
    o1, o2 = rng.standard_normal((nj, ni)), rng.standard_normal((nj, ni))
    a, b = rng.standard_normal((ki, ki)), rng.standard_normal((kj, kj))
    rho_i, rho_j = a @ a.T, b @ b.T
    T, Zft, f = 0.3, 2.5, 0.7
    direct = {w: ChainBinning(-4, 2, 50) for w in ("gt", "ls")}
    for w, (E, wt) in nrg_run_cpu.cfs_terms(last, Ei, ki, Ej, kj, o1, o2, rho_i, rho_j, sign, T, Zft).items():
        if E.size:
            direct[w].add(E, wt, f)
    comp = {w: ChainBinning(-4, 2, 50) for w in ("gt", "ls")}
    fdm_mode_composition(comp, last, Ei, ki, Ej, kj, o1, o2, rho_i, rho_j, f, sign, T, Zft)
    for w in ("gt", "ls"):
        x = np.concatenate([direct[w].pos_re, direct[w].neg_re])
        y = np.concatenate([comp[w].pos_re, comp[w].neg_re])
        assert np.abs(x).max() > 0.0  # one half may be empty (kept minus discarded energies are < 0)
        assert np.allclose(x, y, rtol=1e-12, atol=1e-13 * np.abs(x).max()), w


def ft_fdm_mode_composition(cb, Ei, ki, Ej, kj, o1, o2, factor, sign, T, Z):
    """FT of one pair as the device run forms it: the FDMgt and the FDMls D x D terms of the
    pair cut to its kept states (K = 0) with wnf = 1/Z_ft, into one bin set."""
    empty = np.zeros((0, 0))
    for mode in ("gt", "ls"):
        cb.fdm_pair(mode, Ei[:ki], 0, Ej[:kj], 0, o1[:kj, :ki], o2[:kj, :ki], empty, factor, sign, T, 1.0 / Z)


@pytest.mark.parametrize("sign", [1, -1])
def test_ft_terms_by_fdm_modes(oracle, sign):
    from oracle import nrg_run_cpu
    from oracle.oracle import ChainBinning
    rng = np.random.default_rng(23 + sign)
    ni, nj, ki, kj = 9, 7, 6, 5
    Ei = np.sort(rng.uniform(0.0, 3.0, ni))
    Ej = np.sort(rng.uniform(0.0, 3.0, nj))
    Ei -= Ei[0]
    Ej -= Ej[0]
    o1, o2 = rng.standard_normal((nj, ni)), rng.standard_normal((nj, ni))
    T, Z, f = 0.3, 2.5, 0.7
    direct = ChainBinning(-4, 2, 50)
    E, wt = nrg_run_cpu.ft_terms(Ei[:ki], Ej[:kj], o1[:kj, :ki], o2[:kj, :ki], sign, T, Z)
    direct.add(E, wt, f)
    comp = ChainBinning(-4, 2, 50)
    ft_fdm_mode_composition(comp, Ei, ki, Ej, kj, o1, o2, f, sign, T, Z)
    x = np.concatenate([direct.pos_re, direct.neg_re])
    y = np.concatenate([comp.pos_re, comp.neg_re])
    assert np.abs(x).max() > 0.0
    assert np.allclose(x, y, rtol=1e-12, atol=1e-13 * np.abs(x).max())
