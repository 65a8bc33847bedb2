"""Host-side mirror of the reference's Z4c evolution callbacks.

Same calling conventions as :mod:`baum_b200.bssn`, for the 25-variable Z4c
list (reference z4.c:234-242, :data:`baum_b200.abi.Z4_VARS`):
``z4_rhs_movpunc_N`` (z4_rhs_movpunc_N.c:23), ``set_boundary``
(boundary.c:25), ``evolve_rhs`` (evolve.c:37), ``evolve_rk_rk4`` (rk.c:220)
followed by ``z4_algcon`` (z4.c:49).
"""
import ctypes as C

from . import abi
from .bssn import DeviceLevel, _ptrs, _stream  # noqa: F401

NV = abi.Z4_NVARS


def z4_rhs_movpunc_N(dl, unew, upre, c, ucur, params, stream=None):
    abi.check(abi.lib().nrgpu_z4_rhs(dl.handle, _ptrs(unew, NV), _ptrs(upre, NV), float(c), _ptrs(ucur, NV),
                                     C.byref(params), _stream(stream)))


def set_boundary(dl, unew, upre, c, ucur, params, stream=None):
    abi.check(abi.lib().nrgpu_z4_boundary(dl.handle, _ptrs(unew, NV), _ptrs(upre, NV), float(c), _ptrs(ucur, NV),
                                          C.byref(params), _stream(stream)))


def evolve_rhs(dl, unew, upre, c, ucur, params, stream=None):
    z4_rhs_movpunc_N(dl, unew, upre, c, ucur, params, stream)
    set_boundary(dl, unew, upre, c, ucur, params, stream)


def evolve_rk_rk4(dl, u, dt, params, stream=None):
    abi.check(abi.lib().nrgpu_z4_rk4_step(dl.handle, _ptrs(u, NV), float(dt), C.byref(params), _stream(stream)))
