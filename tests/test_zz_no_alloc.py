"""The allocation-free RK4 entry point against the regular one.

nrgpu_bssn_rk4_step_noalloc serves host codes that cannot allocate device
memory themselves (their device memory belongs to another runtime's pool, or
they allocate nothing after start-up); it keeps its scratch in a fixed array
of the library image instead of level-owned buffers.  Called through the C ABI
twice in a row, it must give what nrgpu_bssn_rk4_step gives after each call,
within the 1e-12 relative tolerance of the other parity tests, at every
centred order (the 6th-order run also covers the order ladder near the box
edge), and the device's free memory must not change across a call.  Its
companion nrgpu_bssn_noalloc_status must report a non-finite state.  This file
is collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from baum_b200 import abi, bssn, punctures

pytestmark = pytest.mark.gpu


def _ptrs(t):
    return abi.ptr_array([t.data_ptr() + i * t.stride(0) * 8 for i in range(abi.NVARS)])


def _entry(L):
    f = L.nrgpu_bssn_rk4_step_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Box), C.c_double, C.c_double, C.c_double, C.POINTER(C.c_void_p),
                  C.c_double, C.POINTER(abi.BssnParams), C.c_void_p]
    g = L.nrgpu_bssn_noalloc_status
    g.restype = C.c_int
    g.argtypes = [C.POINTER(C.c_int), C.c_void_p]
    return f, g


def _state():
    lev, u0 = punctures.schwarzschild_c1(n_inner=20, dx=0.5)   # 22^3 = 10648 points
    # a non-zero shift so that advection and every rhs term take part
    x, y, z = lev.coords()
    u0[18] = 0.05 * np.sin(0.7 * x) * np.cos(0.4 * z)
    u0[19] = -0.03 * np.cos(0.5 * y + 0.2 * x)
    u0[20] = 0.02 * np.sin(0.3 * z - 0.6 * y)
    return lev, u0


@pytest.mark.parametrize("order", [2, 4, 6])
def test_noalloc_rk4_matches_regular_entry_point(gpu, order):
    L = abi.lib()
    f, status = _entry(L)
    lev, u0 = _state()
    p = abi.bssn_params(order_centered=order, order_advection=order)
    dt = 0.125
    dl = bssn.DeviceLevel(lev)
    ua = torch.from_numpy(u0.copy()).cuda()
    ub = torch.from_numpy(u0.copy()).cuda()
    stream = torch.cuda.current_stream()
    for call in range(2):
        bssn.evolve_rk_rk4(dl, ua, dt, p, stream)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st = f(C.byref(lev.boxes[0]), lev.dx, lev.dx, lev.dx, _ptrs(ub), dt, C.byref(p),
               C.c_void_p(stream.cuda_stream))
        assert st == 0, L.nrgpu_last_error()
        torch.cuda.synchronize()
        if call == 1:
            # the set-up (and any lazy module load) happened in the first call
            assert torch.cuda.mem_get_info()[0] == free0
        a, b = ua.cpu().numpy(), ub.cpu().numpy()
        err = max(np.abs(a[v] - b[v]).max() / max(np.abs(a[v]).max(), 1e-8) for v in range(abi.NVARS))
        assert err < 1e-12, (order, call, err)
        flag = C.c_int(-1)
        assert status(C.byref(flag), C.c_void_p(stream.cuda_stream)) == 0, L.nrgpu_last_error()
        assert flag.value == 0
    dl.close()


def test_noalloc_status_reports_a_non_finite_state(gpu):
    L = abi.lib()
    f, status = _entry(L)
    lev, u0 = _state()
    p = abi.bssn_params()
    u0[13, 11 + 22 * (11 + 22 * 11)] = np.nan   # K at the centre point (11, 11, 11)
    u = torch.from_numpy(u0).cuda()
    stream = torch.cuda.current_stream()
    flag = C.c_int(-1)
    assert status(C.byref(flag), C.c_void_p(stream.cuda_stream)) == 0   # clears what came before
    st = f(C.byref(lev.boxes[0]), lev.dx, lev.dx, lev.dx, _ptrs(u), 0.125, C.byref(p),
           C.c_void_p(stream.cuda_stream))
    assert st == 0, L.nrgpu_last_error()
    assert status(C.byref(flag), C.c_void_p(stream.cuda_stream)) == 0, L.nrgpu_last_error()
    assert flag.value == 1
    # read and cleared: a second read reports nothing
    assert status(C.byref(flag), C.c_void_p(stream.cuda_stream)) == 0
    assert flag.value == 0


def test_noalloc_rejects_boxes_over_the_limit(gpu):
    L = abi.lib()
    f, _ = _entry(L)
    big = abi.Box(26, 26, 26, 0, -6.25, -6.25, -6.25)   # 17576 > 16384 points
    p = abi.bssn_params()
    dummy = abi.ptr_array([1] * abi.NVARS)   # never dereferenced: the size check comes first
    st = f(C.byref(big), C.c_double(0.5), C.c_double(0.5), C.c_double(0.5), dummy, C.c_double(0.1),
           C.byref(p), C.c_void_p(0))
    assert st == -1
    assert b"exceeds" in L.nrgpu_last_error()
