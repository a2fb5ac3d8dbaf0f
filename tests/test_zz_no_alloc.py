"""isdf_fit_noalloc: the fit for callers that cannot let the library allocate
device memory (for instance a DFT code that has reserved nearly all of HBM for
its own pool before it calls ISDF, or one that cannot take the device-wide
synchronisation of cudaFree). It must give the same theta as the allocating
isdf_fit and as the oracle on the same inputs, twice in a row (the fixed
scratch array keeps the previous call's contents, so the second call checks
that nothing stale leaks into the result), change the device's free memory by
nothing once the library's own workspace is released, accept a caller's
stream, and reject sizes its 8 MiB array cannot hold.

Named test_zz_* so that pytest collects it last: a run that stops at the first
failure has run every other test before this one."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden
from oracle import fit as ofit

import libisdf_b200 as isdf

pytestmark = pytest.mark.gpu


def _fn():
    f = isdf.lib().isdf_fit_noalloc
    P, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    f.argtypes = [P, LL, I, I, I, I, I, I, I, P, P, P, P]
    f.restype = I
    return f


def _noalloc_fit(torch, d_psi, ng, nstate, a, rk, piv, d_theta, stream=None):
    d_theta.fill_(float("nan"))
    torch.cuda.synchronize()
    info = ctypes.c_int(-1)
    p = np.ascontiguousarray(piv[:rk], dtype=np.int32)
    rc = _fn()(d_psi.data_ptr(), ng, nstate, *a, rk, p.ctypes.data, d_theta.data_ptr(),
               ctypes.addressof(info), stream)
    assert rc == isdf.ISDF_OK, isdf.lib().isdf_last_error()
    assert info.value == 0
    return np.asfortranarray(d_theta.cpu().numpy().T)


def test_noalloc_fit_matches_allocating_fit_twice(torch_cuda):
    torch = torch_cuda
    g = load_golden("small_s1s2")
    psi = g["psi"]
    ng, nstate = psi.shape
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    rk = int(g["rk_eff"])
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_ref = torch.zeros((rk, ng), dtype=torch.float64, device="cuda")
    assert isdf.fit(d_psi, ng, nstate, *a, rk, g["piv"], d_ref) == 0
    th_ref = np.asfortranarray(d_ref.cpu().numpy().T)
    fd_ref = ofit.fitted_densities(th_ref, psi, *a, rk, g["piv"])
    fd_oracle = ofit.fitted_densities(ofit.getbasis(psi, *a, rk, g["piv"]), psi, *a, rk, g["piv"])
    bufs = [torch.empty((rk, ng), dtype=torch.float64, device="cuda") for _ in range(3)]
    stream = torch.cuda.Stream()
    # first call: loads the module that holds the fixed array
    _noalloc_fit(torch, d_psi, ng, nstate, a, rk, g["piv"], bufs[0])
    isdf.lib().isdf_release_workspace()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k, s in enumerate((None, stream.cuda_stream)):
        th = _noalloc_fit(torch, d_psi, ng, nstate, a, rk, g["piv"], bufs[1 + k], s)
        assert np.isfinite(th).all()
        fd = ofit.fitted_densities(th, psi, *a, rk, g["piv"])
        assert ofit.rel(fd, fd_ref) <= 1e-10
        assert ofit.rel(fd, fd_oracle) <= 1e-10
        assert ofit.rel(th, th_ref) <= 1e-10
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "device memory changed across the calls"


def test_noalloc_fit_rejects_sizes_beyond_the_array(torch_cuda):
    torch = torch_cuda
    ng, nstate, rk = 4096, 512, 1024
    d_psi = torch.zeros((nstate, ng), dtype=torch.float64, device="cuda")
    d_theta = torch.zeros((rk, ng), dtype=torch.float64, device="cuda")
    piv = np.arange(rk, dtype=np.int32)
    info = ctypes.c_int(0)
    rc = _fn()(d_psi.data_ptr(), ng, nstate, 256, 256, 256, 256, 256, rk, piv.ctypes.data,
               d_theta.data_ptr(), ctypes.addressof(info), None)
    assert rc == isdf.ISDF_ERR_UNSUPPORTED
    assert b"bytes of scratch" in isdf.lib().isdf_last_error()
