"""The C ABI library loads and matches include/astroflow_dd.h (no GPU needed)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from astroflow_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "astroflow_dd.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(dd_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        from astroflow_b200.build import build

        build()
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 10
    assert set(names) == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(L, n), n
    assert L.dd_abi_version() == 2


def test_error_path_without_gpu_is_a_status_not_an_exit():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present; covered by the GPU tests")
    except Exception:
        pass
    from astroflow_b200.dedisp import Plan

    with pytest.raises((RuntimeError, ValueError)):
        Plan(dict(tsamp=1e-4, fch1=1000.0, foff=1.0, nbits=8, nchans=64, ndata=1000), 0, 10, 1000,
             1063, 1.0)


def test_struct_layouts_match_c():
    """sizeof/offsetof of the ABI structs seen by a C compiler equal the ctypes mirror."""
    structs = {
        "dd_header": _lib.Header, "dd_iqrm_config": _lib.IqrmConfig, "dd_rfi_config": _lib.RfiConfig,
        "dd_plan_params": _lib.PlanParams, "dd_plan_info": _lib.PlanInfo,
        "dd_run_stats": _lib.RunStats, "dd_batch_info": _lib.BatchInfo,
        "dd_stream_info": _lib.StreamInfo, "dd_single_dm_params": _lib.SingleDmParams,
        "dd_single_dm_info": _lib.SingleDmInfo, "dd_tune_report": _lib.TuneReport,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-o", exe, src], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = dict(line.split() for line in out.strip().splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"
