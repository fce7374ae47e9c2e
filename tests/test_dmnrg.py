"""DM-NRG spectral functions of whole runs against the reference's regression outputs
(spec_DMNRG_dens_A_d-A_d.dat of test/c++/test2_algorithms_dmnrg, test23_DMNRG and
test27_bins: doublet recalculation, density-matrix sweep, DM-NRG pair sums into log bins,
N/N+2 or N/N+1 patching, trimming and log-Gaussian broadening)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
DM_CASES = ["test2_algorithms_dmnrg", "test23_DMNRG", "test27_bins"]
SPEC = "spec_DMNRG_dens_A_d-A_d.dat"
# the refs print 10 significant digits; values far below the peak are compared absolutely
RTOL, ATOL_REL_TO_MAX = 2e-9, 1e-10
# device run against the oracle at full precision
ORA_RTOL, ORA_ATOL_REL_TO_MAX = 1e-9, 1e-11


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def ref_spectrum(case):
    rows = [[float(x) for x in line.split()] for line in read(case, SPEC).splitlines()
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
def test_oracle_dmnrg_spectrum_matches_reference(oracle_spectra, case):
    assert_spectrum(oracle_spectra(case)["A_d-A_d"], ref_spectrum(case), RTOL, ATOL_REL_TO_MAX, case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", DM_CASES)
def test_gpu_dmnrg_spectrum(oracle_spectra, case):
    """The device run (doublet recalculation, density-matrix sweep as batched rotate
    terms, pair sums binned by nrg_spec_accumulate, broadening by nrg_broaden) against the
    reference's spectrum and the oracle's."""
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    got = res.spectra["A_d-A_d"]
    assert_spectrum(got, ref_spectrum(case), RTOL, ATOL_REL_TO_MAX, f"{case} vs reference")
    assert_spectrum(got, oracle_spectra(case)["A_d-A_d"], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} vs oracle")
