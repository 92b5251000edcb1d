"""The C-ABI library loads and exports every entry point include/lapw1gpu.h
declares; without a GPU its init reports 'no device' instead of crashing."""
import ctypes as C
import os
import re

import pytest

from hack_wein2k_b200 import build, lapw1gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "lapw1gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lapw1gpu_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = lapw1gpu.load()
    assert lapw1gpu.version().startswith("lapw1gpu")
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = lapw1gpu.load()
    names = header_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(lapw1gpu.EXPORTS) == names


def test_init_without_device_reports_nodevice():
    from tests.conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    lib = lapw1gpu.load()
    h = C.c_void_p()
    rc = lib.lapw1gpu_init(0, C.byref(h))
    assert rc == 6  # LAPW1GPU_ERR_NODEVICE
    assert not h.value


def test_last_error_is_an_empty_string_before_any_cuda_failure():
    """lapw1gpu_last_error names the CUDA call behind a LAPW1GPU_ERR_CUDA;
    in a fresh thread that has had none it is the empty string."""
    import threading
    lib = lapw1gpu.load()
    out = []
    t = threading.Thread(target=lambda: out.append(lib.lapw1gpu_last_error()))
    t.start()
    t.join()
    assert out == [b""]


def test_problem_struct_layout_matches_header():
    """Field order of the ctypes mirror follows the C struct."""
    from hack_wein2k_b200.problem import CProblem
    src = open(os.path.join(ROOT, "include", "lapw1gpu.h")).read()
    body = src[src.index("typedef struct lapw1gpu_problem"):src.index("} lapw1gpu_problem;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";")[:-1]:
        decl = decl.split("{", 1)[-1].strip()
        for part in decl.split(","):
            m = re.search(r"(\w+)\s*(\[\d+\])?\s*$", part.strip())
            if m:
                names.append(m.group(1))
    assert names == [f for f, _ in CProblem._fields_]


def test_hns_noalloc_range_check_runs_on_the_host():
    """The allocation-free HNS entry point rejects an RMT |k+G| beyond
    SPHBES's range before any device work: the check needs no GPU."""
    import dataclasses

    import numpy as np

    from hack_wein2k_b200 import synth
    p = synth.small_case("lo")
    rmt = np.array(p.rmt, dtype=np.float64, copy=True)
    rmt[0] = 25.0 / float(np.max(p.rk[: p.nv]))
    with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
        lapw1gpu.hns_noalloc(dataclasses.replace(p, rmt=rmt), 0x1000, p.n, 0)
    assert e.value.code == 7
