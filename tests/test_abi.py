"""The C-ABI boundary, checked without a GPU.

* libpentadsolver_b200.so loads and exports every entry point include/*.h
  declares (C names through ctypes, the C++ overloads by their mangled names).
* Sizing functions and argument validation are host logic: they answer
  without touching a device.
"""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

import pentadsolver as ps

REPO = Path(__file__).resolve().parent.parent
INCLUDE = REPO / "include"


def declared_c_functions():
    names = set()
    for h in INCLUDE.glob("*.h*"):
        text = h.read_text()
        # exported declarations carry PENTAD_API; inline wrappers do not
        for m in re.finditer(r"PENTAD_API\s*(?:\n\s*)?[\w\s\*]*?\b(pentadsolver_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_reference_api():
    names = declared_c_functions()
    for ref_name in ("pentadsolver_create", "pentadsolver_destroy",
                     "pentadsolver_D_gpsv_batch", "pentadsolver_S_gpsv_batch",
                     "pentadsolver_D_gpsv_batch_buffer_size_ext",
                     "pentadsolver_S_gpsv_batch_buffer_size_ext",
                     "pentadsolver_kernel_that_ran"):
        assert ref_name in names


def test_library_exports_every_declared_c_symbol():
    lib = ps.lib()
    missing = [n for n in declared_c_functions()
               if n != "pentadsolver_gpsv_batch" and n != "pentadsolver_gpsv_batch_buffer_size_ext"
               and not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(shutil.which("nm") is None, reason="nm not available")
def test_library_exports_cpp_overloads():
    out = subprocess.run(["nm", "-D", "--defined-only", str(ps.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    # pentadsolver_gpsv_batch(void*, const double*x5, double*, const int*, int, int, void*)
    for mangled in ("_Z23pentadsolver_gpsv_batchPvPKdS1_S1_S1_S1_PdPKiiiS_",
                    "_Z23pentadsolver_gpsv_batchPvPKfS1_S1_S1_S1_PfPKiiiS_",
                    "_Z39pentadsolver_gpsv_batch_buffer_size_extPvPKdS1_S1_S1_S1_S1_PKiii",
                    "_Z39pentadsolver_gpsv_batch_buffer_size_extPvPKfS1_S1_S1_S1_S1_PKiii"):
        assert mangled in out


@pytest.mark.parametrize("dims,solvedim", [((256, 256, 256), 0), ((256, 256, 256), 1),
                                           ((64, 32, 16), 2), ((200,), 0), ((8, 8), 1)])
@pytest.mark.parametrize("elem", [8, 4])
def test_buffer_size_covers_global_scratch(dims, solvedim, elem):
    n_total = 1
    for v in dims:
        n_total *= v
    b = ps.buffer_size(list(dims), solvedim, elem)
    # the reference's values (src/cuda/singlenode/pentad_cuda.cu:1554-1577):
    # 9 n n_sys elements along x (its transpose path), 3 n n_sys otherwise
    assert b == (9 if solvedim == 0 else 3) * n_total * elem
    # the reference-named sizing functions agree
    fn = getattr(ps.lib(), f"pentadsolver_{'D' if elem == 8 else 'S'}_gpsv_batch_buffer_size_ext")
    assert fn(None, None, None, None, None, None, None, ps._dims(dims), len(dims), solvedim) == b
    h, dv = ps.ctypes.c_size_t(7), ps.ctypes.c_size_t(0)
    fn2 = getattr(ps.lib(), f"pentadsolver_{'D' if elem == 8 else 'S'}_gpsv_batch_buffer_size_two_buffer")
    fn2(None, None, None, None, None, None, None, ps._dims(dims), len(dims), solvedim,
        ps.ctypes.byref(h), ps.ctypes.byref(dv))
    assert h.value == 0 and dv.value == b


@pytest.mark.parametrize("dims,ndim,solvedim", [
    ((16, 16, 16), 3, 3),      # solvedim out of range
    ((16, 16, 16), 3, -1),
    ((4, 16, 16), 3, 0),       # a line of 4 rows (the reference asserts > 4)
    ((16, 0, 16), 3, 1),       # empty dimension
    ((16,) * 9, 9, 0),         # rank above the maximum
])
def test_invalid_shapes_rejected_on_host(dims, ndim, solvedim):
    out = ps.ctypes.c_size_t(0)
    st = ps.lib().pentadsolver_buffer_size_ex(None, 8, ps._dims(dims), ndim, solvedim,
                                              ps.ctypes.byref(out))
    assert st == ps.INVALID_VALUE
    # the solve entry point rejects the shape before any device work
    st = ps.lib().pentadsolver_D_gpsv_batch_ex(None, 1, 1, 1, 1, 1, 1, ps._dims(dims), ndim,
                                               solvedim, None, 0, None)
    assert st == ps.INVALID_VALUE


def test_null_arrays_rejected():
    st = ps.lib().pentadsolver_D_gpsv_batch_ex(None, None, 1, 1, 1, 1, 1, ps._dims([8, 8]), 2,
                                               0, None, 0, None)
    assert st == ps.INVALID_VALUE


def test_handles_and_selection_on_host():
    with ps.Handle() as h:
        assert h.value
        assert h.kernel_that_ran(0) == "none"
        h.set_algo(1, "naive")
        h.set_algo(2, "thomas-pcr", pcr_lanes=2)
        h.set_algo(0, None)
        with pytest.raises(ps.PentadError):
            h.set_algo(0, "bogus")
        with pytest.raises(ps.PentadError):
            h.set_algo(3, "naive")
        with pytest.raises(ps.PentadError):
            h.set_algo(0, "thomas-pcr", pcr_lanes=3)
    assert ps.kernel_that_ran(5) == "none"


def test_status_strings():
    assert ps.status_string(ps.SUCCESS) == "success"
    assert ps.status_string(ps.ZERO_PIVOT) == "zero pivot"
    assert ps.status_string(ps.INVALID_VALUE) == "invalid value"


def test_headers_compile_as_c_and_cpp(tmp_path):
    cc = shutil.which("gcc")
    cxx = shutil.which("g++")
    if cc is None or cxx is None:
        pytest.skip("no host compiler")
    src = tmp_path / "t.c"
    src.write_text('#include "pentadsolver.hpp"\n#include "pentadsolver_ext.h"\n'
                   "int main(void){return 0;}\n")
    subprocess.run([cc, "-std=c11", "-Wall", "-Werror", f"-I{INCLUDE}", "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", f"-I{INCLUDE}", "-x", "c++", "-c",
                    str(src), "-o", str(tmp_path / "t2.o")], check=True)
    src2 = tmp_path / "t2.c"
    src2.write_text('#include "pentadsolver_cuda.hpp"\nint main(void){return 0;}\n')
    subprocess.run([cc, "-std=c11", "-Wall", "-Werror", f"-I{INCLUDE}", "-c", str(src2), "-o",
                    str(tmp_path / "t3.o")], check=True)
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", f"-I{INCLUDE}", "-x", "c++", "-c",
                    str(src2), "-o", str(tmp_path / "t4.o")], check=True)


def test_adi_graph_refuses_bad_arguments_before_touching_a_device():
    # pentadsolver_adi_create checks its arguments before any device work
    # (NULL out-pointer, element size, missing arrays or buffer, iteration
    # count, a buffer smaller than the x direction's reference size)
    import ctypes

    import pentadsolver as ps

    f = ps._typed("pentadsolver_adi_create",
                  [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 7 +
                  [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.POINTER(ctypes.c_void_p)])
    out = ctypes.c_void_p(None)
    dims = ps._dims([16, 16, 16])
    need = ps.buffer_size([16, 16, 16], 0, 8)
    arrs = [256] * 6
    cases = [
        (8, arrs, 3, 1, 256, need, None),           # no out-pointer
        (2, arrs, 3, 1, 256, need, out),            # element size
        (8, [256] * 5 + [0], 3, 1, 256, need, out),  # missing x
        (8, arrs, 3, 0, 256, need, out),            # no iterations
        (8, arrs, 3, 1, 0, need, out),              # no buffer
        (8, arrs, 3, 1, 256, need - 8, out),        # buffer too small
    ]
    for eb, a, nd, it, buf, nbytes, o in cases:
        st = f(None, eb, *a, dims, nd, it, buf, nbytes, None if o is None else ctypes.byref(o))
        assert st == ps.INVALID_VALUE, (eb, nd, it, buf, nbytes)
        assert not out.value


def test_plan_entry_points_refuse_bad_arguments_on_host():
    # plan execution, description, status and destruction take a NULL plan as
    # invalid; pentadsolver_plan_execute_ex also refuses unknown flag bits
    import ctypes

    import pentadsolver as ps

    exe = ps._typed("pentadsolver_plan_execute", [ctypes.c_void_p, ctypes.c_void_p])
    exe_ex = ps._typed("pentadsolver_plan_execute_ex",
                       [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int])
    destroy = ps._typed("pentadsolver_plan_destroy", [ctypes.c_void_p])
    describe = ps._typed("pentadsolver_plan_describe", [ctypes.c_void_p], ctypes.c_char_p)
    assert exe(None, None) == ps.INVALID_VALUE
    for flags in (0, 1, 2, -1):
        assert exe_ex(None, None, flags) == ps.INVALID_VALUE
    assert destroy(None) == ps.INVALID_VALUE
    assert describe(None) == b"none"
