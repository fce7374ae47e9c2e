"""Reduced forms of the benchmark's large NRG-run workloads, run on the device and by the
oracle on the same generated inputs:

* the two-channel Kondo FDM run (spin-1/2 impurity, J = 0.2 on both flat channels, Lambda = 3,
  T = 1e-6, FDM dynamic spin susceptibility S_imp-S_imp and the FDM thermodynamics), with keep
  and Nmax cut from 5000 and 50 so that the oracle finishes in well under a minute: the
  forward sweep (two-channel QS Hamiltonian, batched eigensolve with large blocks,
  recalculation of both channels' <||f||> and of the triplet operator), the FDM density
  matrices (c++/dmnrg.hpp:146-217) and the FDM pair sums (c++/algo_FDM.hpp:30-151);
* the Anderson-model DM-NRG run with 10 bins per decade over [1e-10, 1] (keep and Nmax cut
  from 4000 and 60): doublet recalculation, DM-NRG sweep and binning on the coarse grid.

Thermodynamics (td, tdfdm) and spectra agree with the oracle to the tolerances of the other
whole-run tests; the truncation keeps the same states at every step (the block orders of
every step are equal), so no step is compared past a change of the kept multiplets."""
import os

import numpy as np
import pytest

from test_dmnrg import ORA_ATOL_REL_TO_MAX, ORA_RTOL, assert_spectrum

pytestmark = pytest.mark.gpu

TD_RTOL, TD_ATOL = 1e-10, 1e-11  # td of the device run against the oracle (other eigensolver)
TDFDM_RTOL, TDFDM_ATOL = 1e-10, 1e-11

KONDO_PARAM = """[param]
symtype=QS
Lambda=3
keep={keep}
T=1e-6
fdm=true
spect=S_imp-S_imp
"""

ANDERSON_PARAM = """[param]
symtype=QS
model=SIAM
U=1.0
Gamma=0.04
delta=0
band=flat
discretization=Z
Lambda=2
z=1
keep={keep}
T=1e-8
ops=n_d A_d
dmnrg=true
specd=A_d-A_d
bins=10
emin=1e-10
emax=1
"""


def _both(param, data):
    from nrgljubljana_b200.nrg_run import run_files
    from oracle import nrg_run_cpu
    spec, fo = {}, {}
    _, td_cpu, _, _ = nrg_run_cpu.run(param, data, threads=os.cpu_count() or 1, spectra=spec, fdm_out=fo)
    res = run_files(param, data)
    return res, np.array(td_cpu), spec, fo


def _assert_td(got, want):
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    assert got.shape == want.shape
    err = np.abs(got - want) - (TD_RTOL * np.abs(want) + TD_ATOL)
    assert not (err > 0).any(), f"td differs at {np.unravel_index(int(np.argmax(err)), err.shape)}"


def test_two_channel_kondo_fdm_reduced(oracle):
    from nrgljubljana_b200.datagen import kondo_qs
    param = KONDO_PARAM.format(keep=600)
    data = kondo_qs([0.2, 0.2], 0.5, 3.0, 12, ops=["S_imp"])
    res, td_cpu, spec, fo = _both(param, data)
    assert max(res.max_dim_per_step) > 600, "the reduced run must reach the large-block path"
    _assert_td(res.td, td_cpu)
    assert sorted(res.spectra) == sorted(spec) == ["spin_FDM_dens_S_imp-S_imp"]
    name = "spin_FDM_dens_S_imp-S_imp"
    assert_spectrum(res.spectra[name], spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{name} vs oracle")
    assert res.tdfdm[0] == fo["tdfdm"][0]
    # the FDM heat capacity at T = 1e-6 vanishes: round-off noise of order 1e-35 in both runs
    assert np.allclose(res.tdfdm[1], fo["tdfdm"][1], rtol=TDFDM_RTOL, atol=TDFDM_ATOL), (res.tdfdm[1], fo["tdfdm"][1])


def test_anderson_dmnrg_coarse_bins_reduced(oracle):
    from nrgljubljana_b200.datagen import siam_qs
    param = ANDERSON_PARAM.format(keep=1500)
    data = siam_qs(1.0, 0.0, 0.04, 2.0, 30, 1.0, "Z", ops=["n_d", "A_d"])
    res, td_cpu, spec, _ = _both(param, data)
    assert max(res.max_dim_per_step) > 224, "the reduced run must reach the blocked reduction"
    _assert_td(res.td, td_cpu)
    name = "spec_DMNRG_dens_A_d-A_d"
    assert sorted(res.spectra) == sorted(spec) == [name]
    assert_spectrum(res.spectra[name], spec[name], ORA_RTOL, ORA_ATOL_REL_TO_MAX, f"{name} vs oracle")
