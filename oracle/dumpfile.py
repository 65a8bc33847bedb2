"""Reader of the raw FP64 level dumps written by oracle/harness/nrharness.c
(test infrastructure).  Format documented in that file's header."""
import numpy as np

MAGIC = 0x3147524E


def read(path):
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(48), dtype="<i8")
        if hdr[0] != MAGIC:
            raise ValueError("%s: not a level dump" % path)
        l, nboxes, nvars, npoints, iteration = (int(x) for x in hdr[1:6])
        t, dx, dy, dz, dt = np.frombuffer(f.read(40), dtype="<f8")
        boxes = []
        for _ in range(nboxes):
            bi = np.frombuffer(f.read(32), dtype="<i8")
            bx = np.frombuffer(f.read(24), dtype="<f8")
            boxes.append((int(bi[0]), int(bi[1]), int(bi[2]), int(bi[3]),
                          float(bx[0]), float(bx[1]), float(bx[2])))
        names = [f.read(32).split(b"\0")[0].decode() for _ in range(nvars)]
        boundary = np.frombuffer(f.read(4 * npoints), dtype="<i4").copy()
        data = np.frombuffer(f.read(8 * nvars * npoints), dtype="<f8").reshape(nvars, npoints).copy()
    return dict(level=l, iteration=iteration, time=float(t), dx=float(dx), dy=float(dy),
                dz=float(dz), dt=float(dt), boxes=boxes, names=names, boundary=boundary, data=data)
