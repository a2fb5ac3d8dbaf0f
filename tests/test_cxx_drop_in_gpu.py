"""The C++ drop-in: tests/cxx/drop_in.cpp calls isdf::isdffunc::ISDF the way
the reference's example driver does (examples/si8/readpsi.cpp:219-237), is
compiled against include/isdf.hpp and linked to libisdf_b200.so, and runs the
reference's own Si8 example data (16^3 grid, 35 states, Nv = 16, Nc = 0,
mu = 192, 500 K-means iterations, check on). piv must equal the reference's
(the golden made by the reference's own code), the QRCP overload (mu = 160:
the sketch width IRound(sqrt(1.5 mu)) must fit the 16-state window) must give
the same pivots as the Python binding, and failures must arrive as
std::runtime_error with the library's message."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

import libisdf_b200 as isdf

pytestmark = pytest.mark.gpu

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    exe = tmp_path / "drop_in"
    libdir = os.path.join(ROOT, "libisdf_b200")
    cmd = ["g++", "-std=c++14", "-O1", os.path.join(ROOT, "tests", "cxx", "drop_in.cpp"), "-o",
           str(exe), "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           "-L", libdir, "-l:libisdf_b200.so", f"-Wl,-rpath,{libdir}",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cxx_caller_runs_the_reference_example(torch_cuda, tmp_path):
    isdf.lib()  # the library is built
    g = load_golden("si8_example")
    psi = np.asfortranarray(g["psi"])
    ng, nstate = psi.shape
    n = [int(x) for x in g["ng"]]
    length = float(g["length"][0])
    a = [int(g[k]) for k in ("nocc", "nv1", "nc1", "nv2", "nc2")]
    mu, iters = int(g["rk_requested"]), int(g["iters"])
    (tmp_path / "psi.bin").write_bytes(psi.tobytes(order="F"))
    exe = _build(tmp_path)
    out = tmp_path / "out"
    mu_q = 160
    r = subprocess.run([str(exe), str(tmp_path / "psi.bin"), *map(str, n), repr(length),
                        str(nstate), *map(str, a), str(mu), str(iters), str(mu_q), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    piv_k = np.fromfile(str(out) + ".kmeans.piv", dtype=np.int32)
    assert np.array_equal(piv_k, g["piv"])
    # the QRCP overload against the Python binding on the same inputs
    piv_q = np.fromfile(str(out) + ".qrcp.piv", dtype=np.int32)
    d_psi = torch_cuda.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch_cuda.empty((mu_q, ng), dtype=torch_cuda.float64, device="cuda")
    piv_py = np.zeros(ng, dtype=np.int32)
    isdf.ISDF(d_psi, isdf.Domain(length=(length,) * 3, num_grid=tuple(n)), a[0], nstate, *a[1:],
              mu_q, d_theta, piv_py, iters, s1="QRCP")
    assert np.array_equal(piv_q, piv_py)
    assert "caught: Wrong select points method" in lines
    assert any(l.startswith("caught: mu outside") for l in lines), lines
