"""Regenerate the NRG-run fixtures under tests/golden/nrg/ from the reference's regression tests.

Each case directory of the reference's ``test/c++/<case>/`` (or ``test/c++sym_all/<case>/``) holds the run's input (``param``,
``data``) and the outputs the reference produced with a real LAPACK (``ref/td``,
``ref/custom``, printed to 10 significant digits; for DM-NRG cases also the spectral
functions ``ref/{spec,corr,spin}_{DMNRG,FDM,FDMgt,FDMls}_dens_*.dat`` and the FDM outputs
``ref/tdfdm``, ``ref/customfdm``). They are copied here unchanged so that
the tests can run where the reference tree is absent. Usage:

    python tests/golden/make_nrg_fixtures.py /path/to/nrgljubljana
"""
import os
import re
import shutil
import sys

CASES = [
    "test0_minimal", "test0_minimal_Nmax1", "test0_minimal_Nmax2", "test0_minimal_Nmax3",
    "test3_disc_z", "test4_disc_c", "test10_keepmin", "test12_Nmax", "test13_strategy_all",
    "test14_strategy_kept", "test15_safeguard", "test16_safeguardmax", "test35_betabar",
    "test56_dsyevd", "test56_dsyevr", "test200_data_has", "legacy_simple", "legacy_Himp",
    "test2_algorithms_dmnrg", "test23_DMNRG", "test27_bins", "test24_NN1", "test25_NN2avg", "test26_NN2even",
    "c++sym_all/test300_QS_ref", "c++sym_all/test310_QS_ref",
    "test2_algorithms_fdm", "test2_algorithms_fdmexpv", "test2_algorithms_fdmgtls", "test60_discard_immediately",
    "test61_discard_trim", "test64_emax", "test66_fdmexpvn", "legacy_fdmexpv2", "legacy_fdmexpv3",
    "regr2defaults", "regr2lastall_false", "regr2lastall_true", "legacy_one_jkondonew",
    "c++sym_all/test314_model=ZERO",
    "test2_algorithms_cfs", "test2_algorithms_cfsgtls", "test_cfs_only", "test2_algorithms", "test11_T",
    "test0_minimal_Nmax1_td", "test0_minimal_Nmax2_td", "test0_minimal_Nmax3_td", "test17_dumpannotated",
    "test18_dumpscaled", "test19_dumpabs", "test20_dumpgroups", "test24_NN1_Nmax=10", "test24_NN1_Nmax=11",
    "test27_NN2odd", "test2_algorithms_finite", "test30_cosine_band", "test31_flat_band", "test55_gt_ls",
    "test58_dsyev", "test5_disc_y", "test62_dumpenergies", "test67_fixeps", "test68_grouptol", "test8_keep",
    "test9_keepenergy", "legacy_sigma_trick_siam_qs", "legacy_substeps_one_siam_std", "test32_arbitrary_DOS",
    "test47_nrgchain", "test48_adapt_tri=old", "test50_ref1", "test52_ref2", "test54_ref3",
    "test33_Delta", "test34_bandrescale", "test49_template1", "test51_template2", "test53_template3",
    "test63_dumpsubspaces", "c++sym_all/legacy_globalop_Q1Q2-QS",
    "test21_mats", "test2_algorithms_fdmmats", "legacy_matsubara_test1-qs",
    "test_dmnrg_only", "test2_algorithms_finitemats", "test65_algorithms_mats", "test0_clean",
]
# spectra of the DM-NRG, FDM (real frequencies and Matsubara), CFS and FT algorithms, FDM thermodynamics and expectation values,
# and the annotated eigenvalue lists (annotated.dat)
SPECTRUM = re.compile(r"^(spec|corr|spin)_(DMNRG|DMNRGmats|FDM|FDMgt|FDMls|FDMmats|CFS|CFSgt|CFSls|FT|FTmats)_dens_.*\.dat$")


def main(ref_root: str) -> None:
    out_root = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nrg")
    for case in CASES:
        sub, name = case.split("/") if "/" in case else ("c++", case)
        src = os.path.join(ref_root, "test", sub, case.split("/")[-1])
        dst = os.path.join(out_root, name)
        os.makedirs(dst, exist_ok=True)
        extra = [f for f in sorted(os.listdir(os.path.join(src, "ref")))
                 if SPECTRUM.match(f) or f in ("tdfdm", "customfdm", "annotated.dat", "energies.nrg", "subspaces.dat")]
        for name, rel in [("param", "param"), ("data", "data"), ("td", "ref/td"), ("custom", "ref/custom")] + \
                [(f, "ref/" + f) for f in extra]:
            p = os.path.join(src, rel)
            if os.path.exists(p):
                shutil.copyfile(p, os.path.join(dst, name))
    print(f"wrote {len(CASES)} cases to {out_root}")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NRG_REFERENCE")
    if not ref:
        sys.exit(f"usage: {sys.argv[0]} REFERENCE_DIR (or set NRG_REFERENCE): the NRG Ljubljana source tree")
    main(ref)
