"""The C-ABI library builds, loads and exports every symbol the header
declares.  Loads the library but makes no compute call (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(cyc_\w+)\s*\(", txt, flags=re.M))
    return names


def test_header_declares_the_engine_surface():
    names = declared_symbols()
    for must in ("cyc_engine_compute_gradient_and_hessian", "cyc_engine_update_xbeta",
                 "cyc_engine_compute_remaining_statistics", "cyc_engine_get_log_likelihood",
                 "cyc_fit", "cyc_batch_fit", "cyc_dataset_create"):
        assert must in names


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = ctypes.CDLL(os.path.join(ROOT, "cyclops_b200", "_lib", "libcyclops_b200.so"))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    from cyclops_b200 import _native
    assert declared_symbols() <= set(_native.exported_symbols())


def test_errors_are_status_codes_not_exceptions(cuda_lib):
    """Argument checks happen before any device work."""
    from cyclops_b200 import _native as N
    h = ctypes.c_void_p()
    rc = cuda_lib.cyc_dataset_create(None, 0, ctypes.byref(h))
    assert rc == 1
    assert b"null" in cuda_lib.cyc_last_error()
    assert cuda_lib.cyc_engine_set_weights(None, None, 0) == 1


@pytest.mark.parametrize("where", ["y", "time", "col_val"])
@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_non_finite_data_is_refused_before_device_work(cuda_lib, where, bad):
    """A NaN or infinity in the outcomes, times or covariate values is an
    argument error from cyc_dataset_create (no GPU needed to see it)."""
    import numpy as np
    from cyclops_b200 import _native as N
    K = 6
    arr = {"y": np.array([0, 1, 0, 1, 1, 0], float), "time": np.arange(1.0, K + 1),
           "col_val": np.array([0.5, -1.0, 2.0]), "fmt": np.array([3, 1], np.int32),
           "cp": np.array([0, 0, 3], np.int64), "ci": np.array([0, 2, 5], np.int32),
           "vp": np.array([0, 0, 3], np.int64)}
    arr[where] = arr[where].copy()
    arr[where][1] = bad
    d = N.DataDesc(model=4, K=K, J=2, pid=None, y=arr["y"].ctypes.data, time=arr["time"].ctypes.data,
                   col_format=arr["fmt"].ctypes.data, col_ptr=arr["cp"].ctypes.data,
                   col_idx=arr["ci"].ctypes.data, val_ptr=arr["vp"].ctypes.data,
                   col_val=arr["col_val"].ctypes.data, has_offset=0, has_intercept=1)
    h = ctypes.c_void_p()
    assert cuda_lib.cyc_dataset_create(ctypes.byref(d), 0, ctypes.byref(h)) == 1
    assert b"non-finite" in cuda_lib.cyc_last_error()


# C struct of the header -> its ctypes mirror in cyclops_b200/_native.py
_MIRRORS = {"cyc_data_desc": "DataDesc", "cyc_control": "Control", "cyc_prior": "Prior",
            "cyc_fit_spec": "FitSpec", "cyc_fit_result": "FitResult", "cyc_run_stats": "RunStats"}


def test_struct_mirrors_match_the_header(tmp_path):
    """Size and field offsets of every ABI struct, as a C compiler lays them
    out from include/cyclops_b200.h, equal the ctypes mirrors' (a field
    appended to a struct must be appended to its mirror too)."""
    import shutil
    import subprocess
    from cyclops_b200 import _native as N
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cyclops_b200.h"', "int main(void) {"]
    for cname, pyname in _MIRRORS.items():
        st = getattr(N, pyname)
        lines.append(f'printf("{pyname} size %zu\\n", sizeof({cname}));')
        for field, _ in st._fields_:
            lines.append(f'printf("{pyname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        pyname, field, value = line.split()
        st = getattr(N, pyname)
        want = ctypes.sizeof(st) if field == "size" else getattr(st, field).offset
        assert int(value) == want, (pyname, field, int(value), want)


def test_library_reports_the_header_abi_version(cuda_lib):
    import re
    txt = open(os.path.join(ROOT, "include", "cyclops_b200.h")).read()
    want = int(re.search(r"#define CYC_ABI_VERSION (\d+)", txt).group(1))
    assert cuda_lib.cyc_version() == want
