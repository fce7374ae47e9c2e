"""Green's functions on the Matsubara axis -- Algo_FDMmats (c++/algo_FDM.hpp:153-217),
Algo_DMNRGmats (c++/algo_DMNRG.hpp:61-106) and Algo_FTmats (c++/algo_FT.hpp:50-91, with the
initial cluster of docalc0, c++/core.hpp:251-260), saved by GFMatsubara (c++/spectrum.hpp:
212-227) -- against the reference's regression outputs {spec,corr,spin}_*mats_dens_*.dat (rows
w_n, Re G, Im G, printed to 10 significant digits) of test21_mats, test2_algorithms_fdmmats,
legacy_matsubara_test1-qs, test_dmnrg_only, test2_algorithms_finitemats, test65_algorithms_mats
(all six algorithms in one run) and test0_clean, beside the real-frequency spectra of the same
runs: the oracle on the CPU, the device run (the terms of every subspace pair summed over the
Matsubara points by nrg_spec_accumulate_mats) on the GPU against both."""
import os

import numpy as np
import pytest

from test_dmnrg import ATOL_REL_TO_MAX, ORA_ATOL_REL_TO_MAX, ORA_RTOL, RTOL, assert_spectrum

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
CASES = ["test21_mats", "test2_algorithms_fdmmats", "legacy_matsubara_test1-qs", "test_dmnrg_only",
         "test2_algorithms_finitemats", "test65_algorithms_mats", "test0_clean"]
MATS_RTOL = 2e-9   # the reference's 10 printed digits
MATS_ORA_RTOL = 1e-9  # device against the oracle: other eigensolver, other summation order


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def rows(case, name):
    return np.array([[float(x) for x in line.split()] for line in read(case, name).splitlines()
                     if line.strip() and not line.startswith("#")])


def files(case, mats):
    return sorted(f[:-4] for f in os.listdir(os.path.join(GOLD, case))
                  if f.endswith(".dat") and f.startswith(("spec_", "corr_", "spin_")) and ("mats_dens" in f) == mats)


def assert_mats(got, want, rtol, what):
    """Column by column: within rtol of the value, or of the column's largest value for the
    entries that vanish (the imaginary parts of bosonic functions at w_0)."""
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    assert got.shape == want.shape, f"{what}: {got.shape} != {want.shape}"
    scale = np.maximum(np.abs(want).max(axis=0), 1e-300)
    bad = np.abs(got - want) > rtol * np.abs(want) + 1e-12 * scale
    assert not bad.any(), f"{what}: rows {np.nonzero(bad.any(axis=1))[0][:5]}: {got[bad][:3]} vs {want[bad][:3]}"


@pytest.fixture(scope="module")
def oracle_mats(oracle):
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


@pytest.mark.parametrize("case", CASES)
def test_oracle_matsubara_matches_reference(oracle_mats, case):
    spec, _ = oracle_mats(case)
    assert sorted(spec) == sorted(files(case, True) + files(case, False))
    for name in files(case, True):
        assert_mats(spec[name], rows(case, name + ".dat"), MATS_RTOL, f"{case} {name}")
    for name in files(case, False):
        assert_spectrum(spec[name], rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_matsubara(oracle_mats, case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    spec, _ = oracle_mats(case)
    assert sorted(res.spectra) == sorted(files(case, True) + files(case, False))
    for name in files(case, True):
        assert_mats(res.spectra[name], rows(case, name + ".dat"), MATS_RTOL, f"{case} {name} vs reference")
        assert_mats(res.spectra[name], spec[name], MATS_ORA_RTOL, f"{case} {name} vs oracle")
    for name in files(case, False):
        assert_spectrum(res.spectra[name], rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX,
                        f"{case} {name} vs reference")
        assert_spectrum(res.spectra[name], spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} {name} vs oracle")
