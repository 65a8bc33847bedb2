"""Host-side mirror of the reference's BSSN evolution callbacks over the C ABI.

The reference registers ``bssn_rhs_movpunc_N(unew, upre, c, ucur)`` as the
"geometry" rhs (bssn.c:17,325), ``set_boundary`` as the boundary
(boundary.c:25), ``evolve_rk_rk4`` as the integrator (rk.c:220) and
``bssn_algcon`` after each step (bssn.c:86).  The functions here have the
same names, argument meaning and order; a variable list is a float64 tensor
of shape (24, npoints) in the reference's evolve-list order
(:data:`baum_b200.abi.BSSN_VARS`) on the level's CUDA device.  torch provides
device memory and streams only; all arithmetic runs in libnrgpu.so.
"""
import ctypes as C

import torch

from . import abi

NV = abi.NVARS


def _ptrs(t, nv=NV):
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.dim() == 2 and t.shape[0] == nv):
        raise ValueError("a variable list is a contiguous float64 CUDA tensor of shape (%d, npoints)" % nv)
    base = t.data_ptr()
    step = t.stride(0) * 8
    return abi.ptr_array([base + i * step for i in range(nv)])


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class DeviceLevel:
    """Device mirror of a level (``nrgpu_level_create``)."""

    def __init__(self, level, device=0):
        L = abi.lib()
        torch.cuda.set_device(device)
        abi.check(L.nrgpu_init(device))
        self.level = level
        self.npoints = level.npoints
        h = C.c_void_p()
        abi.check(L.nrgpu_level_create(C.byref(level.desc), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            abi.lib().nrgpu_level_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def empty(self, nv=NV):
        return torch.zeros((nv, self.npoints), dtype=torch.float64, device="cuda")

    def set_block(self, bx, by, bz=1):
        """Run the rhs kernels in blocks of bx x by x bz = 128 threads."""
        abi.check(abi.lib().nrgpu_level_block(self.handle, int(bx), int(by), int(bz)))

    def block(self):
        b = (C.c_int * 3)()
        abi.check(abi.lib().nrgpu_level_get_block(self.handle, b))
        return tuple(b)

    def autotune(self, system, params, stream=None):
        """Time the rhs block shapes for this level and keep the fastest;
        returns it as (x, y, z)."""
        b = (C.c_int * 3)()
        abi.check(abi.lib().nrgpu_level_autotune(self.handle, int(system), C.byref(params), _stream(stream), b))
        return tuple(b)

    def queue(self, on=-1):
        """The Z4c interior of all boxes in one persistent launch over a
        queue of tiles (nrgpu_level_queue): on = 1, 0, or -1 to query."""
        r = abi.lib().nrgpu_level_queue(self.handle, int(on))
        if r < 0:
            abi.check(r)
        return int(r)

    def tile(self, on=-1):
        """The staged-tile (TMA) interior rhs: on = 1 (a block per tile), 2
        (persistent), 0 (off); -1 only queries; returns the setting."""
        r = abi.lib().nrgpu_level_tile(self.handle, int(on))
        if r < 0:
            abi.check(r)
        return int(r)

    def nan_flag(self):
        f = C.c_int()
        abi.check(abi.lib().nrgpu_level_nan_flag(self.handle, C.byref(f)))
        return bool(f.value)


def bssn_rhs_movpunc_N(dl, unew, upre, c, ucur, params, stream=None):
    """Inner-point rhs (c == 0) or unew = upre + c*rhs with the algebraic
    fixes (c != 0); mirrors bssn_rhs_movpunc_N (bssn_rhs_movpunc_N.c:27)."""
    abi.check(abi.lib().nrgpu_bssn_rhs(dl.handle, _ptrs(unew), _ptrs(upre), float(c), _ptrs(ucur),
                                       C.byref(params), _stream(stream)))


def set_boundary(dl, unew, upre, c, ucur, params, stream=None):
    """Radiative boundary on PHYBOUND points (set_boundary, boundary.c:25)."""
    abi.check(abi.lib().nrgpu_bssn_boundary(dl.handle, _ptrs(unew), _ptrs(upre), float(c), _ptrs(ucur),
                                            C.byref(params), _stream(stream)))


def evolve_rhs(dl, unew, upre, c, ucur, params, stream=None):
    """rhs then boundary, as evolve_rhs (evolve.c:37) with comp = 0."""
    bssn_rhs_movpunc_N(dl, unew, upre, c, ucur, params, stream)
    set_boundary(dl, unew, upre, c, ucur, params, stream)


def bssn_algcon(dl, u, params, stream=None):
    """det(g~) = 1, tr(A~) = 0 (bssn_algcon, bssn_algcon.c:25)."""
    abi.check(abi.lib().nrgpu_bssn_algcon(dl.handle, _ptrs(u), C.byref(params), _stream(stream)))


def evolve_rk_rk4(dl, u, dt, params, stream=None):
    """One RK4 step in place plus algcon (rk.c:220, bssn.c:86)."""
    abi.check(abi.lib().nrgpu_bssn_rk4_step(dl.handle, _ptrs(u), float(dt), C.byref(params), _stream(stream)))


def evolve_host(dl, host_u, nsteps, dt, params):
    """nsteps RK4 steps of a host state (numpy or CPU tensor (24, npoints),
    or a list of 24 contiguous float64 numpy arrays, one per variable, as
    BAM keeps them), uploaded and downloaded inside the call
    (nrgpu_bssn_evolve_host)."""
    import numpy as np
    if isinstance(host_u, (list, tuple)):
        if len(host_u) != NV or not all(a.dtype == np.float64 and a.flags.c_contiguous for a in host_u):
            raise ValueError("24 contiguous float64 arrays")
        ptrs = abi.ptr_array([a.ctypes.data for a in host_u])
    else:
        if isinstance(host_u, torch.Tensor):
            base, step = host_u.data_ptr(), host_u.stride(0) * 8
        else:
            assert host_u.dtype == np.float64 and host_u.flags.c_contiguous
            base, step = host_u.ctypes.data, host_u.strides[0]
        ptrs = abi.ptr_array([base + i * step for i in range(NV)])
    abi.check(abi.lib().nrgpu_bssn_evolve_host(dl.handle, ptrs, int(nsteps), float(dt), C.byref(params)))
    return host_u
