"""The C ABI boundary, checked without a GPU.

* libcuSZp.so loads and exports every extern "C" function include/cuSZp.h declares;
* a C++ translation unit that takes the address of every function declared in
  include/cuSZp.h and include/cuSZp/*.h (the reference's 36 per-mode C++ entry
  points, TimingGPU, the *_Yafan I/O helpers) links against the library, i.e. the
  mangled names match the reference's declarations;
* the host-only file helpers round-trip data.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "cuszp_b200", "lib", "libcuSZp.so")
CUDA_INC = "/usr/local/cuda/include"


def _extern_c_functions():
    text = open(os.path.join(INC, "cuSZp.h")).read()
    body = text[text.index('extern "C" {'):]
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cuSZp_\w+)\s*\(", body, re.M)
    return sorted(set(names))


def test_library_exports_every_c_symbol():
    lib = ctypes.CDLL(LIB)
    names = _extern_c_functions()
    assert "cuSZp_compress" in names and "cuSZp_decompress" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_entry_points_link(tmp_path):
    """Every declared function (C and C++ linkage) resolves in libcuSZp.so."""
    decls = []
    for fn in ["cuSZp.h"] + sorted("cuSZp/" + f for f in os.listdir(os.path.join(INC, "cuSZp"))):
        text = open(os.path.join(INC, fn)).read()
        decls += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b((?:cuSZp_|read|write|sym|convert)\w+)\s*\(", text, re.M)
    decls = sorted(set(decls))
    assert len([d for d in decls if re.match(r"cuSZp_(de)?compress_[123]D_", d)]) == 36
    src = ['#include <cuSZp.h>', 'volatile const void* sink;', 'int main() {']
    for d in decls:
        src.append(f'  sink = (const void*)&{d};')
    src += ['  TimingGPU t; t.StartCounter(); (void)t;', '  return 0;', '}']
    cpp = tmp_path / "link_all.cpp"
    cpp.write_text("\n".join(src))
    exe = tmp_path / "link_all"
    r = subprocess.run(["g++", "-std=c++17", f"-I{INC}", f"-I{CUDA_INC}", str(cpp), "-o", str(exe),
                        f"-L{os.path.dirname(LIB)}", "-lcuSZp", "-L/usr/local/cuda/lib64", "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_mangled_names_match_reference_signatures():
    """Spot-check the Itanium mangling the reference's headers produce."""
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    for sym in ["_Z27cuSZp_compress_1D_fixed_f32PfPhmPmfP11CUstream_st",
                "_Z29cuSZp_decompress_1D_fixed_f32PfPhmmfP11CUstream_st",
                "_Z27cuSZp_compress_2D_fixed_f64PdPhmPm5uint3dP11CUstream_st",
                "_Z31cuSZp_decompress_3D_outlier_f64PdPhmm5uint3dP11CUstream_st",
                "_ZN9TimingGPU12StartCounterEv", "_ZN9TimingGPU10GetCounterEv"]:
        assert sym in out, sym


def test_file_helpers_roundtrip(tmp_path):
    """The *_Yafan helpers have C++ linkage (as in the reference); bind their mangled names."""
    lib = ctypes.CDLL(LIB)
    write = getattr(lib, "_Z29writeDoubleData_inBytes_YafanPdmPcPi")
    read = getattr(lib, "_Z20readDoubleData_YafanPcPmPi")
    x = np.arange(1000, dtype=np.float64) * 0.5
    path = str(tmp_path / "d.f64").encode()
    st = ctypes.c_int(-1)
    write.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    write(x.ctypes.data, x.size, path, ctypes.byref(st))
    assert st.value == 0
    read.restype = ctypes.POINTER(ctypes.c_double)
    read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
    n = ctypes.c_size_t(0)
    p = read(path, ctypes.byref(n), ctypes.byref(st))
    assert st.value == 0 and n.value == 1000
    y = np.ctypeslib.as_array(p, shape=(1000,)).copy()
    assert np.array_equal(x, y)
    assert open(path.decode(), "rb").read() == x.tobytes()


def test_cli_usage_without_gpu():
    cli = os.path.join(ROOT, "cuszp_b200", "lib", "cuSZp")
    r = subprocess.run([cli, "-h"], capture_output=True, text=True)
    assert r.returncode != 0 and "-eb" in r.stdout
    r = subprocess.run([cli, "-i", "x", "-t", "f16"], capture_output=True, text=True)
    assert "Unsupported data type" in r.stdout


@pytest.mark.parametrize("sym", ["cuSZp_compress", "cuSZp_decompress"])
def test_python_binding_has_reference_signature(sym):
    from cuszp_b200 import pycuSZp
    f = getattr(pycuSZp.lib, sym)
    assert len(f.argtypes) == 10
    assert f.argtypes[6] is pycuSZp.Uint3
