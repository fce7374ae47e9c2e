"""Full-density-matrix (FDM) outputs of whole runs against the reference's regression outputs:
the spectra {spec,corr,spin}_{FDM,FDMgt,FDMls}_dens_*.dat, the FDM thermodynamics (tdfdm)
and the FDM expectation values (customfdm) of test/c++/test2_algorithms_fdm,
test2_algorithms_fdmexpv, test2_algorithms_fdmgtls, test60_discard_immediately,
test61_discard_trim, test64_emax, test66_fdmexpvn, legacy_fdmexpv2, legacy_fdmexpv3 and the
two-channel c++sym_all/test314_model=ZERO:
partial statistical sums Z_n^D and weights w_n, the FDM density-matrix sweep with its
discarded-state sectors, the spectra operators recalculated over all states, FDM pair sums
(gt and ls parts) binned per step, trimming and broadening."""
import os

import numpy as np
import pytest

from test_dmnrg import ATOL_REL_TO_MAX, ORA_ATOL_REL_TO_MAX, ORA_RTOL, RTOL, assert_spectrum

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
FDM_CASES = ["test2_algorithms_fdm", "test2_algorithms_fdmexpv", "test2_algorithms_fdmgtls",
             "test60_discard_immediately", "test61_discard_trim", "test64_emax", "test66_fdmexpvn",
             "legacy_fdmexpv2", "legacy_fdmexpv3", "test314_model=ZERO"]
# tdfdm/customfdm: printed to 10 significant digits (20 for the legacy customfdm)
TAB_RTOL = 2e-9


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def rows(case, name):
    return np.array([[float(x) for x in line.split()] for line in read(case, name).splitlines()
                     if line.strip() and not line.startswith("#")])


def spectrum_files(case):
    return sorted(f[:-4] for f in os.listdir(os.path.join(GOLD, case))
                  if f.endswith(".dat") and f.startswith(("spec_", "corr_", "spin_")))


def assert_row(got, want, what):
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    assert got.shape == want.shape, f"{what}: {got.shape} != {want.shape}"
    bad = np.abs(got - want) > TAB_RTOL * np.abs(want) + 1e-300
    assert not bad.any(), f"{what}: {got} vs {want}"


@pytest.fixture(scope="module")
def oracle_fdm(oracle):
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


@pytest.mark.parametrize("case", FDM_CASES)
def test_oracle_fdm_outputs_match_reference(oracle_fdm, case):
    spec, fo = oracle_fdm(case)
    assert sorted(spec) == spectrum_files(case)
    for name in spectrum_files(case):
        assert_spectrum(spec[name], rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name}")
    for name in ("tdfdm", "customfdm"):
        if os.path.exists(os.path.join(GOLD, case, name)):
            assert_row(fo[name][1], rows(case, name)[-1], f"{case} {name}")


@pytest.mark.gpu
@pytest.mark.parametrize("case", FDM_CASES)
def test_gpu_fdm_outputs(oracle_fdm, case):
    """The device run (FDM density-matrix sweep as batched rotate terms with diagonal
    discarded-state sectors, spectra operators over all states, FDM pair sums binned by
    nrg_spec_accumulate, broadening by nrg_broaden) against the reference and the oracle."""
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    spec, fo = oracle_fdm(case)
    assert sorted(res.spectra) == spectrum_files(case)
    for name in spectrum_files(case):
        got = res.spectra[name]
        assert_spectrum(got, rows(case, name + ".dat"), RTOL, ATOL_REL_TO_MAX, f"{case} {name} vs reference")
        assert_spectrum(got, spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{case} {name} vs oracle")
    for name in ("tdfdm", "customfdm"):
        if os.path.exists(os.path.join(GOLD, case, name)):
            got = getattr(res, name)
            assert_row(got[1], rows(case, name)[-1], f"{case} {name} vs reference")
            assert np.allclose(got[1], fo[name][1], rtol=1e-11, atol=0), f"{case} {name} vs oracle"


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["test2_algorithms_fdm", "test314_model=ZERO"])
def test_gpu_fdm_with_eigenvectors_in_host_memory(monkeypatch, case):
    """The same run with every stored step's eigenvectors moved to host memory after each
    step (a headroom no device has) and brought back by the FDM sweep and the spectral pass:
    the FDM thermodynamics are equal and the spectra agree to the binning's round-off."""
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import QSRun, RunParams
    p, d = RunParams.from_param(parse_param(read(case, "param"))), read_data(read(case, "data"))
    base = QSRun(p, d, 0).run()
    monkeypatch.setattr(QSRun, "SPILL_HEADROOM_BYTES", 1 << 60)
    monkeypatch.setattr(QSRun, "SPILL_CHECK_BYTES", 0)
    run = QSRun(p, d, 0)
    res = run.run()
    assert run.spilled_bytes > 0
    assert res.tdfdm == base.tdfdm
    assert sorted(res.spectra) == sorted(base.spectra)
    for name, want in base.spectra.items():
        got = res.spectra[name]
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), name
