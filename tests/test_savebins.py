"""Raw binned spectra (savebins, c++/spectrum.hpp:146-170) and the output options of a run
(broaden, reim, prec_xy, prec_td, width_td, ...): the driver's trim-and-order of the bins
(nrg_run.raw_bins) against a per-bin restatement of Bins::trim (c++/bins.hpp:165-185), the
oracle's raw bins of a reference DM-NRG case against its own broadened spectrum and the
reference's, the binary and text writers, and the parameter reader."""
import os

import numpy as np
import pytest

from nrgljubljana_b200.nrg_run import RunParams, Result, raw_bins, write_bins, write_outputs

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")


def per_bin(e, pos, neg, discard_trim, reim):
    """Bins::trim of each half, then savebins' order: positive bins, then E = -|E|."""
    rows = []
    for sgn, w in ((1.0, pos), (-1.0, neg)):
        for i in range(len(e)):
            if i == len(e) - 1 or abs(w[i]) >= discard_trim * (e[i + 1] - e[i]):
                rows.append((sgn * e[i], w[i], 0.0) if reim else (sgn * e[i], w[i]))
    return np.array(rows)


@pytest.mark.parametrize("reim", [False, True])
def test_raw_bins_trim_and_order(reim):
    rng = np.random.default_rng(5)
    e = np.logspace(-8, 1, 200)
    pos = rng.standard_normal(200) * 10.0 ** rng.uniform(-25, 0, 200)
    neg = rng.standard_normal(200) * 10.0 ** rng.uniform(-25, 0, 200)
    pos[-1] = neg[-1] = 0.0  # the last bin is kept even when empty
    got = raw_bins(pos, neg, e, 1e-16, reim)
    want = per_bin(e, pos, neg, 1e-16, reim)
    assert got.shape == want.shape and np.array_equal(got, want)
    assert got.shape[1] == (3 if reim else 2)
    npos = int(np.sum(got[:, 0] > 0))
    assert np.all(np.diff(got[:npos, 0]) > 0) and np.all(np.diff(-got[npos:, 0]) > 0)


def test_write_bins_round_trip(tmp_path):
    rows = np.array([[1e-3, 0.25, 0.0], [2e-3, -0.5, 0.0], [-1e-3, 0.125, 0.0]])
    path = tmp_path / "spec.bin"
    write_bins(str(path), rows)
    assert path.stat().st_size == rows.size * 8
    assert np.array_equal(np.fromfile(path, dtype=np.float64).reshape(-1, 3), rows)


def test_write_outputs_formats(tmp_path):
    p = RunParams.from_param({"reim": "true", "prec_xy": "6", "prec_td": "8", "width_td": "12", "savebins": "true"})
    res = Result(["T", "C"], [[0.5, 1.0 / 3.0]], ["T"], [[0.5]])
    res.spectra["spec_DMNRG_dens_A_d-A_d"] = np.array([[-1.0, 0.1234567891], [1.0, 0.5]])
    res.bins["spec_DMNRG_dens_A_d-A_d"] = np.array([[1.0, 0.5, 0.0], [-1.0, 0.25, 0.0]])
    write_outputs(str(tmp_path), p, res)
    assert (tmp_path / "spec_DMNRG_dens_A_d-A_d.dat").read_text() == "-1 0.123457 0\n1 0.5 0\n"
    assert np.array_equal(np.fromfile(tmp_path / "spec_DMNRG_dens_A_d-A_d.bin").reshape(-1, 3),
                          res.bins["spec_DMNRG_dens_A_d-A_d"])
    td = (tmp_path / "td").read_text().splitlines()
    assert td[1] == " " + f"{0.5:>12.8g} " + f"{1.0 / 3.0:>12.8g} "


def test_param_reader_accepts_output_keys():
    p = RunParams.from_param({"broaden": "false", "savebins": "true", "reim": "true", "prec_xy": "12",
                              "prec_td": "9", "prec_custom": "7", "width_td": "20", "width_custom": "18",
                              "dmnrg": "true", "specd": "A_d-A_d"})
    assert not p.broaden and p.savebins and p.reim
    assert (p.prec_xy, p.prec_td, p.prec_custom, p.width_td, p.width_custom) == (12, 9, 7, 20, 18)


def test_oracle_raw_bins_reproduce_its_spectrum(oracle):
    """The oracle's savebins rows of test23_DMNRG, broadened with BR_NEW on the mesh of its
    .dat output, give that output back; the .dat also matches the reference's file."""
    from oracle import nrg_run_cpu as O
    from test_dmnrg import ATOL_REL_TO_MAX, RTOL, assert_spectrum
    case = "test23_DMNRG"
    param = open(os.path.join(GOLD, case, "param")).read()
    data = open(os.path.join(GOLD, case, "data")).read()
    spec, bins = {}, {}
    O.run(param, data, threads=os.cpu_count() or 1, spectra=spec, bins_out=bins)
    assert sorted(bins) == sorted(spec)
    kv = O.parse_param(param)
    T = float(kv.get("T", 0.001))
    alpha = float(kv.get("alpha", 0.3))
    omega0 = float(kv.get("omega0", -1.0))
    omega0 = omega0 if omega0 >= 0.0 else float(kv.get("omega0_ratio", 1.0)) * T
    for name, rows in bins.items():
        assert rows.shape[1] == 2
        dat = spec[name]
        got = np.array([sum(w * O._BR_NEW(E, e, alpha, omega0) for e, w in rows) for E in dat[:, 0]])
        assert np.allclose(got, dat[:, 1], rtol=1e-12, atol=1e-14 * np.abs(dat[:, 1]).max()), name
        ref = np.loadtxt(os.path.join(GOLD, case, name + ".dat"))
        assert_spectrum(dat, ref, RTOL, ATOL_REL_TO_MAX, f"{case} {name}")


def test_oracle_broaden_false_writes_no_spectrum(oracle):
    from oracle import nrg_run_cpu as O
    case = "test23_DMNRG"
    param = open(os.path.join(GOLD, case, "param")).read() + "\nbroaden=false\n"
    data = open(os.path.join(GOLD, case, "data")).read()
    spec, bins = {}, {}
    O.run(param, data, threads=os.cpu_count() or 1, spectra=spec, bins_out=bins)
    assert spec == {} and len(bins) > 0
