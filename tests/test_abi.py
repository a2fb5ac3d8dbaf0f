"""Host-side checks of the C ABI (no GPU needed): the library loads, exports
every function that include/isdf_c.h declares, and rejects bad arguments
before touching the device."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

import libisdf_b200 as isdf


def _declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(isdf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = isdf.lib()
    names = _declared_functions("isdf_c.h")
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    lib = isdf.lib()
    assert lib.isdf_status_string(0) == b"ok"
    assert b"positive definite" in lib.isdf_status_string(isdf.ISDF_ERR_NOT_SPD)


def test_null_arguments_are_rejected_without_a_device():
    lib = isdf.lib()
    rc = lib.isdf_solve(None, None, 0, 1, 1, 0, 1, 0, 0, None, None, 1, 0, 0, None, None)
    assert rc == isdf.ISDF_ERR_ARG
    assert b"null" in lib.isdf_last_error()


def test_bad_state_window_rejected():
    dom = isdf.Domain(length=(1.0, 1.0, 1.0), num_grid=(4, 4, 4))
    piv = __import__("numpy").zeros(64, dtype="int32")
    with pytest.raises(isdf.IsdfError) as e:
        isdf.ISDF(0x1000, dom, 2, 4, 3, 0, 2, 0, 8, 0x2000, piv, 5)  # nocc - nv1 < 0
    assert e.value.code == isdf.ISDF_ERR_ARG
    with pytest.raises(isdf.IsdfError):
        isdf.ISDF(0x1000, dom, 2, 4, 2, 0, 2, 0, 8, 0x2000, piv, 5, s1="Random")


def test_default_options_match_reference_constants():
    o = isdf._Options()
    isdf.lib().isdf_default_options(ctypes.byref(o))
    assert o.precision == isdf.PRECISION_FP64
    assert o.qrcp_oversample == 1.5 and o.qrcp_seed == 41  # getpoints_QRCP.cpp:82, isdf.cpp:68
    assert o.rand_seed == -1


def test_cxx_header_compiles():
    src = '#include "isdf.hpp"\nint main(){ isdf::Domain d; (void)d; return 0; }\n'
    r = subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                        "-x", "c++", "-"], input=src.encode(), capture_output=True)
    assert r.returncode == 0, r.stderr.decode()


_STRUCTS = [("isdf_domain_t", "_Domain"), ("isdf_options_t", "_Options"),
            ("isdf_report_t", "_Report"), ("isdf_server_config_t", "_ServerConfig"),
            ("isdf_request_t", "_Request"), ("isdf_server_stats_t", "_ServerStats")]


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """The Python binding's ctypes structures have the size and field offsets
    that a C compiler gives the structs of include/isdf_c.h (a mismatch would
    pass garbage across the boundary without any error)."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "isdf_c.h"', 'int main(void) {']
    for c_name, py_name in _STRUCTS:
        cls = getattr(isdf, py_name)
        lines.append(f'  printf("{py_name} size %zu\\n", sizeof({c_name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{py_name} {field} %zu\\n", offsetof({c_name}, {field}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe)], capture_output=True)
    assert r.returncode == 0, r.stderr.decode()
    out = subprocess.run([str(exe)], capture_output=True, check=True).stdout.decode().split("\n")
    c_layout = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for _, py_name in _STRUCTS:
        cls = getattr(isdf, py_name)
        assert c_layout[(py_name, "size")] == ctypes.sizeof(cls), py_name
        for field, _ in cls._fields_:
            assert c_layout[(py_name, field)] == getattr(cls, field).offset, (py_name, field)


def test_cxx_drop_in_caller_links(tmp_path):
    """tests/cxx/drop_in.cpp, a caller written like the reference's example
    driver, compiles against include/isdf.hpp and links to libisdf_b200.so
    (it is run on the GPU by tests/test_cxx_drop_in_gpu.py)."""
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    libdir = os.path.join(ROOT, "libisdf_b200")
    isdf.lib()
    r = subprocess.run(["g++", "-std=c++14", os.path.join(ROOT, "tests", "cxx", "drop_in.cpp"),
                        "-o", str(tmp_path / "drop_in"), "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(cuda, "include"), "-L", libdir, "-l:libisdf_b200.so",
                        "-L", os.path.join(cuda, "lib64"), "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cxx_mpi_caller_links(tmp_path):
    """With mpi.h included first, include/isdf.hpp's ISDF() dispatches an MPI
    communicator of more than one rank to the p-rank solve over NCCL
    (isdf_comm_nccl_unique_id + MPI_Bcast + isdf_comm_create_nccl +
    isdf_solve_sharded): that branch compiles and links (tests/cxx/mpi_stub
    stands in for an MPI installation; several ranks need several GPUs)."""
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    src = tmp_path / "mpi_caller.cpp"
    src.write_text("#include <mpi.h>\n#include \"isdf.hpp\"\n"
                   "int main() { isdf::Domain d; d.comm = MPI_COMM_WORLD;\n"
                   "  if (false) isdf::isdffunc::ISDF(nullptr, d, 1, 2, 1, 1, 1, 1, 4, nullptr,\n"
                   "                                  nullptr, 10);\n"
                   "  return isdf::isdffunc::sharded_comm(d.comm) == nullptr ? 0 : 1; }\n")
    isdf.lib()
    exe = tmp_path / "mpi_caller"
    r = subprocess.run(["g++", "-std=c++14", str(src), "-o", str(exe),
                        "-I", os.path.join(ROOT, "tests", "cxx", "mpi_stub"),
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
                        "-L", os.path.join(ROOT, "libisdf_b200"), "-l:libisdf_b200.so",
                        "-Wl,-rpath," + os.path.join(ROOT, "libisdf_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # at world size 1 no NCCL communicator is made (the one-GPU path runs)
    assert subprocess.run([str(exe)]).returncode == 0


def test_request_footprint_counts_check_and_oversampling():
    """isdf_request_workspace_bytes includes what isdf_workspace_bytes leaves
    out: the check's buffers (they depend on the grid's shape) and the QRCP
    oversampling; invalid requests give 0."""
    dom = isdf.Domain(length=(10.26,) * 3, num_grid=(40, 40, 40))
    base = isdf.request_workspace_bytes(dom, 32, 16, 16, 16, 16, 320)
    assert base == isdf.workspace_bytes(64000, 32, 320)
    assert isdf.request_workspace_bytes(dom, 32, 16, 16, 16, 16, 320, check=True) > base
    q15 = isdf.request_workspace_bytes(dom, 32, 16, 16, 16, 16, 320, s1="QRCP")
    q25 = isdf.request_workspace_bytes(dom, 32, 16, 16, 16, 16, 320, s1="QRCP",
                                       options=isdf.Options(qrcp_oversample=2.5))
    assert q25 > q15 == isdf.workspace_bytes(64000, 32, 320, selector=isdf.SELECT_QRCP)
    bad = isdf.Domain(length=(1.0,) * 3, num_grid=(0, 4, 4))
    assert isdf.request_workspace_bytes(bad, 32, 16, 16, 16, 16, 320) == 0
