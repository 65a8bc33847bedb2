"""Puncture tracking on the device: the host-side mirror of the reference's
shift-integration tracker over the C ABI.

``track_moving_puncture_integrate(dl, beta, beta_p, dt, pos)`` follows
track_moving_puncture_integrate (projects/Gauge/moving_punctures_integrate.c:
29-100) with the position test of track_puncture (moving_punctures.c:
189-191): ``beta`` and ``beta_p`` are the level's shift now and one step
earlier (float64 CUDA tensors of shape (3, npoints)), ``pos`` a float64 CUDA
tensor of shape (n, 3) updated in place.  All arithmetic runs in libnrgpu.so
(nrgpu_track_punctures); the positions equal the reference's bit for bit.
``track_moving_puncture_extremum(dl, var, pos)`` is the reference's other
tracker (moving_puncture_track_method = ext), a search for the extremum of
one level variable (nrgpu_track_punctures_extremum).
Inside a mesh-refinement run, :meth:`baum_b200.fmr.Hierarchy.track` tracks
on the finest level during the steps.
"""
import ctypes as C

import torch

from . import abi
from .bssn import _ptrs, _stream


def track_moving_puncture_integrate(dl, beta, beta_p, dt, pos, order=4, fixz=False, stream=None):
    """Advance the punctures at ``pos`` (n x 3, in place) by one step of
    length ``dt``; returns the per-puncture status (bit 0: integrated, bit 1:
    the new position is on the level and was taken) as an int32 tensor."""
    if not (pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous() and pos.dim() == 2
            and pos.shape[1] == 3):
        raise ValueError("pos is a contiguous float64 CUDA tensor of shape (n, 3)")
    status = torch.zeros(pos.shape[0], dtype=torch.int32, device=pos.device)
    abi.check(abi.lib().nrgpu_track_punctures(dl.handle, _ptrs(beta, 3), _ptrs(beta_p, 3), float(dt), int(order),
                                              int(bool(fixz)), pos.shape[0], C.c_void_p(pos.data_ptr()),
                                              C.c_void_p(status.data_ptr()), _stream(stream)))
    return status


def track_moving_puncture_extremum(dl, var, pos, order=4, find_max=False, minmove=0.01, fixz=False, stream=None):
    """Move the punctures at ``pos`` (n x 3, in place) toward the minimum
    (or maximum) of ``var`` (a float64 CUDA tensor of npoints); returns the
    per-puncture status as for track_moving_puncture_integrate."""
    if not (pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous() and pos.dim() == 2
            and pos.shape[1] == 3):
        raise ValueError("pos is a contiguous float64 CUDA tensor of shape (n, 3)")
    if not (var.is_cuda and var.dtype == torch.float64 and var.is_contiguous() and var.numel() == dl.npoints):
        raise ValueError("var is a contiguous float64 CUDA tensor of the level's npoints")
    status = torch.zeros(pos.shape[0], dtype=torch.int32, device=pos.device)
    abi.check(abi.lib().nrgpu_track_punctures_extremum(dl.handle, C.c_void_p(var.data_ptr()), int(bool(find_max)),
                                                       float(minmove), int(order), int(bool(fixz)), pos.shape[0],
                                                       C.c_void_p(pos.data_ptr()), C.c_void_p(status.data_ptr()),
                                                       _stream(stream)))
    return status
