"""DM-NRG spectra of whole runs against the reference's regression outputs: the spectral
function of a doublet (spec_DMNRG_dens_A_d-A_d.dat), the correlator of a singlet
(corr_DMNRG_dens_n_d-n_d.dat) and the dynamic spin susceptibility of a triplet
(spin_DMNRG_dens_sigma_d-sigma_d.dat) of test/c++/test2_algorithms_dmnrg, test23_DMNRG,
test24_NN1 (N/N+1 patching), test25_NN2avg, test26_NN2even and test27_bins (5 bins per
decade): doublet and triplet recalculation, density-matrix sweep, DM-NRG pair sums into log
bins with the fermionic or bosonic sign, patching, trimming and log-Gaussian broadening."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
DM_CASES = ["test2_algorithms_dmnrg", "test23_DMNRG", "test24_NN1", "test25_NN2avg", "test26_NN2even", "test27_bins",
            "test24_NN1_Nmax=10", "test24_NN1_Nmax=11", "test27_NN2odd", "test30_cosine_band", "test31_flat_band",
            "test32_arbitrary_DOS", "test47_nrgchain", "test48_adapt_tri=old", "test50_ref1", "test52_ref2",
            "test54_ref3", "test33_Delta", "test34_bandrescale", "test49_template1", "test51_template2",
            "test53_template3"]
SPECTRA = ["spec_DMNRG_dens_A_d-A_d", "corr_DMNRG_dens_n_d-n_d", "spin_DMNRG_dens_sigma_d-sigma_d"]
SPEC = SPECTRA[0]
# the refs print 10 significant digits; values far below the peak are compared absolutely
RTOL, ATOL_REL_TO_MAX = 2e-9, 1e-10
# device run against the oracle at full precision
ORA_RTOL, ORA_ATOL_REL_TO_MAX = 1e-9, 1e-11


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def ref_spectrum(case, name=SPEC):
    rows = [[float(x) for x in line.split()] for line in read(case, name + ".dat").splitlines()
            if line.strip() and not line.startswith("#")]
    return np.array(rows)


def assert_spectrum(got, want, rtol, atol_rel, what):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    assert np.max(np.abs(got[:, 0] - want[:, 0]) / np.abs(want[:, 0])) < 1e-9, f"{what}: mesh"
    tol = rtol * np.abs(want[:, 1]) + atol_rel * np.abs(want[:, 1]).max()
    bad = np.abs(got[:, 1] - want[:, 1]) > tol
    assert not bad.any(), f"{what}: E={want[bad][0, 0]} {got[bad][0, 1]!r} vs {want[bad][0, 1]!r}"


@pytest.fixture(scope="module")
def oracle_spectra(oracle):
    from oracle import nrg_run_cpu
    cache = {}

    def get(case):
        if case not in cache:
            spec = {}
            nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1, spectra=spec)
            cache[case] = spec
        return cache[case]
    return get


@pytest.mark.parametrize("case", DM_CASES)
def test_oracle_dmnrg_spectra_match_reference(oracle_spectra, case):
    got = oracle_spectra(case)
    assert sorted(got) == sorted(SPECTRA)
    for name in SPECTRA:
        assert_spectrum(got[name], ref_spectrum(case, name), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", DM_CASES)
def test_gpu_dmnrg_spectra(oracle_spectra, case):
    """The device run (doublet and triplet recalculation, density-matrix sweep as batched
    rotate terms, pair sums binned by nrg_spec_accumulate, broadening by nrg_broaden) against
    the reference's spectra and the oracle's."""
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert sorted(res.spectra) == sorted(SPECTRA)
    for name in SPECTRA:
        got = res.spectra[name]
        assert_spectrum(got, ref_spectrum(case, name), RTOL, ATOL_REL_TO_MAX, f"{case} {name} vs reference")
        assert_spectrum(got, oracle_spectra(case)[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} {name} vs oracle")


# two channels (model.m of the reference's regression tests): doublet recalculation with the
# two-channel tables, N/N+1-type window factor sqrt(Lambda) of two channels
DM2_CASES = ["regr2defaults", "regr2lastall_false", "regr2lastall_true"]


def spectrum_names(case):
    return sorted(f[:-4] for f in os.listdir(os.path.join(GOLD, case))
                  if f.endswith(".dat") and f.startswith(("spec_", "corr_", "spin_")))


@pytest.mark.parametrize("case", DM2_CASES)
def test_oracle_two_channel_dmnrg_spectra(oracle_spectra, case):
    got = oracle_spectra(case)
    assert sorted(got) == spectrum_names(case)
    for name in spectrum_names(case):
        assert_spectrum(got[name], ref_spectrum(case, name), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", DM2_CASES)
def test_gpu_two_channel_dmnrg_spectra(oracle_spectra, case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    assert sorted(res.spectra) == spectrum_names(case)
    for name in spectrum_names(case):
        assert_spectrum(res.spectra[name], ref_spectrum(case, name), RTOL, ATOL_REL_TO_MAX, f"{case} {name} vs reference")
        assert_spectrum(res.spectra[name], oracle_spectra(case)[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX,
                        f"{case} {name} vs oracle")
