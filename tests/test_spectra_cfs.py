"""Complete-Fock-space (CFS) spectra of whole runs against the reference's regression outputs
({spec,corr,spin}_{CFS,CFSgt,CFSls}_dens_*.dat of test/c++/test2_algorithms_cfs,
test2_algorithms_cfsgtls and test_cfs_only): the DM-NRG density matrices, the operators of
the spectra recalculated over all states, the last step's kept-kept term with Boltzmann
weights over Z_ft and, at the other steps, the discarded-kept terms with rho (Algo_CFSgt,
Algo_CFSls, c++/algo_CFS.hpp), merged whole, trimmed and broadened. The device run builds
these terms from the FDM pair modes of nrg_spec_accumulate; `test_cfs_terms_by_fdm_modes`
checks that composition term by term with the oracle's own CFS and FDM pair sums."""
import os

import numpy as np
import pytest

from test_dmnrg import ATOL_REL_TO_MAX, ORA_ATOL_REL_TO_MAX, ORA_RTOL, RTOL, assert_spectrum

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
CFS_CASES = ["test2_algorithms_cfs", "test2_algorithms_cfsgtls", "test_cfs_only"]


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def rows(case, name):
    return np.array([[float(x) for x in line.split()] for line in read(case, name).splitlines()
                     if line.strip() and not line.startswith("#")])


def spectrum_files(case):
    return sorted(f[:-4] for f in os.listdir(os.path.join(GOLD, case)) if f.endswith(".dat"))


@pytest.fixture(scope="module")
def oracle_cfs(oracle):
    from oracle import nrg_run_cpu
    cache = {}

    def get(case):
        if case not in cache:
            spec = {}
            nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, spectra=spec)
            cache[case] = spec
        return cache[case]
    return get


@pytest.mark.parametrize("case", CFS_CASES)
def test_oracle_cfs_spectra_match_reference(oracle_cfs, case):
    spec = oracle_cfs(case)
    assert sorted(spec) == spectrum_files(case)
    for name in spectrum_files(case):
        assert_spectrum(spec[name], rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CFS_CASES)
def test_gpu_cfs_spectra(oracle_cfs, case):
    """The device run's CFS, CFSgt and CFSls spectra against the reference and the oracle."""
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    spec = oracle_cfs(case)
    assert sorted(res.spectra) == spectrum_files(case)
    for name in spectrum_files(case):
        got = res.spectra[name]
        assert_spectrum(got, rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name} vs reference")
        assert_spectrum(got, spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} {name} vs oracle")


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
