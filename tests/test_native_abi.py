"""libssfft loads and exports every entry point include/ssfft.h declares; host-side
argument validation that needs no GPU."""

import ctypes
import os
import re

import pytest

from materialite_b200 import _native as nat

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "ssfft.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ssfft_\w+)\s*\(", text)))


def test_library_is_built_and_loads():
    assert os.path.isfile(nat.library_path()), "build with python -m materialite_b200.csrc.build"
    nat.load_library()


def test_every_declared_function_is_exported():
    lib = nat.load_library()
    names = declared_functions()
    assert "ssfft_step" in names and "ssfft_create" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(nat.EXPORTED_SYMBOLS)


def config(n=(16, 16, 16), precision=nat.SSFFT_MIXED, mask=(0, 1, 1, 1, 1, 1)):
    cfg = nat.SsfftConfig()
    for d in range(3):
        cfg.n[d] = n[d]
    cfg.precision = precision
    for c in range(6):
        cfg.stress_mask[c] = mask[c]
    return cfg


def estimate(cfg, evp=0, nslip=0):
    lib = nat.load_library()
    out = ctypes.c_size_t()
    rc = lib.ssfft_estimate_bytes(ctypes.byref(cfg), evp, nslip, ctypes.byref(out))
    return rc, out.value


def test_estimate_bytes_scales_with_grid():
    rc, small = estimate(config((32, 32, 32)))
    assert rc == 0
    rc, big = estimate(config((64, 64, 64)))
    assert rc == 0 and big > 4 * small  # grid buffers dominate the fixed reduction space
    rc, evp = estimate(config((64, 64, 64)), 1, 12)
    assert rc == 0 and evp > big


@pytest.mark.parametrize("n,mask,code", [((37, 8, 8), (0,) * 6, -4),      # prime factor 37
                                         ((8, 8, 8), (0, 0.5, 0, 0, 0, 0), -1),
                                         ((0, 8, 8), (0,) * 6, -4)])
def test_config_validation(n, mask, code):
    rc, _ = estimate(config(n, mask=mask))
    assert rc == code
    assert nat.load_library().ssfft_last_error()


@pytest.mark.parametrize("field", ["krylov_floor", "krylov_forcing"])
@pytest.mark.parametrize("value", [-0.1, 1.0, float("nan")])
def test_krylov_stop_option_validation(field, value):
    cfg = config()
    setattr(cfg, field, value)
    rc, _ = estimate(cfg)
    assert rc == -1
    assert field.encode() in nat.load_library().ssfft_last_error()


def test_invalid_precision_rejected():
    rc, _ = estimate(config(precision=7))
    assert rc == -1


# ctypes mirrors of the header's structs, with their C type names
def _struct_mirrors():
    from materialite_b200 import serving as sv
    return {"ssfft_config": nat.SsfftConfig, "ssfft_step_in": nat.SsfftStepIn,
            "ssfft_step_out": nat.SsfftStepOut, "ssfft_rate_schedule": nat.SsfftRateSchedule,
            "ssfft_solve_out": nat.SsfftSolveOut, "ssfft_phase": sv.SsfftPhase,
            "ssfft_request": sv.SsfftRequest, "ssfft_completion": sv.SsfftCompletion}


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Size and every field offset of each ctypes struct equal what a C compiler makes
    of include/ssfft.h (gcc on the host; no GPU)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    mirrors = _struct_mirrors()
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append('  return 0;\n}')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c11", str(src), "-o", str(exe)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n"):
        if row:
            cname, key, val = row.split()
            got[(cname, key)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_voronoi_rejects_bad_arguments_before_touching_the_gpu():
    lib = nat.load_library()
    dims = (ctypes.c_int32 * 3)(4, 4, 4)
    vec = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    seeds = (ctypes.c_double * 3)(0.5, 0.5, 0.5)
    out = (ctypes.c_int32 * 64)()
    assert lib.ssfft_voronoi(dims, vec, vec, vec, seeds, 0, 1, 0, out) == -1  # SSFFT_E_INVALID
    bad = (ctypes.c_int32 * 3)(4, 0, 4)
    assert lib.ssfft_voronoi(bad, vec, vec, vec, seeds, 1, 1, 0, out) == -1  # SSFFT_E_INVALID
    assert b"positive" in lib.ssfft_last_error()
