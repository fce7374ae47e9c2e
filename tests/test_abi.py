"""CPU checks of the drop-in boundary: the C-ABI library loads, exports every entry point
that include/nrg_b200.h declares, and refuses to run without an sm_100 device."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "nrg_b200.h")).read()
    return sorted(set(re.findall(r"NRG_API\s+(?:const\s+)?\w+\*?\s+(nrg_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from nrgljubljana_b200 import build
    build.build()
    from nrgljubljana_b200 import _lib
    return _lib.load()


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "nrg_diag_batch" in syms and "nrg_gemm3_batch" in syms and "nrg_spec_accumulate" in syms
    from nrgljubljana_b200 import _lib
    assert sorted(_lib.EXPORTS) == syms


def test_library_exports_every_declared_symbol(lib):
    for s in header_symbols():
        assert hasattr(lib, s), s
        assert ctypes.cast(getattr(lib, s), ctypes.c_void_p).value


def test_version(lib):
    assert lib.nrg_version() == 2


def test_no_cpu_fallback_without_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import nrgljubljana_b200 as nb
    with pytest.raises(nb.NRGError) as ei:
        nb.Context()
    assert ei.value.code == -4


def test_bins_grid_matches_oracle(lib, oracle):
    import nrgljubljana_b200 as nb
    for (lo, hi, b) in ((-10.0, 0.0, 10), (-14.0, 2.0, 1000), (-3.0, 1.0, 7)):
        g = nb.BinGrid(lo, hi, b)
        cb = oracle.ChainBinning(lo, hi, b)
        assert g.nbins == cb.nbins
        assert np.array_equal(g.energies(), cb.energies)


def test_diag_argument_errors(lib):
    import ctypes as C
    # null context is rejected before any device work
    n = (C.c_int * 1)(4)
    ptrs = (C.c_void_p * 1)()
    info = (C.c_int * 1)()
    assert lib.nrg_diag_batch(None, 1, n, ptrs, ptrs, ptrs, info, None) == -1


def test_descriptor_layouts_match_the_header(tmp_path):
    """The ctypes structures and numpy record types the host side builds descriptors with
    have the byte layout the C compiler gives the header's structs."""
    import ctypes as C
    import subprocess
    from nrgljubljana_b200._lib import GEMM3_DTYPE, HPIECE_DTYPE, Gemm3, HPiece
    src = tmp_path / "layout.c"
    fields = {"nrg_gemm3": [f[0] for f in Gemm3._fields_], "nrg_hpiece": [f[0] for f in HPiece._fields_]}
    body = ['#include <stdio.h>', '#include <stddef.h>', '#include "nrg_b200.h"', 'int main(void) {']
    for st, names in fields.items():
        body.append(f'printf("%zu\\n", sizeof({st}));')
        body += [f'printf("%zu\\n", offsetof({st}, {n}));' for n in names]
    body.append("return 0; }")
    src.write_text("\n".join(body))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = []
    for S, dt in ((Gemm3, GEMM3_DTYPE), (HPiece, HPIECE_DTYPE)):
        assert dt.itemsize == C.sizeof(S)
        want.append(C.sizeof(S))
        for name, _ in S._fields_:
            assert dt.fields[name][1] == getattr(S, name).offset
            want.append(getattr(S, name).offset)
    assert got == want
