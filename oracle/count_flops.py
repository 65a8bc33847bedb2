"""FLOPs per inner point of the CPU restatement of the BSSN and Z4c right-hand
sides (test infrastructure: the algorithmic work behind the roofline).

    python oracle/count_flops.py

Compiles oracle/nr_oracle.c as C++ with -DORACLE_COUNT_FLOPS (the counting
scalar of oracle/flopcount.h: + - * / one FLOP each, log/exp/pow counted
apart) into oracle/_ref/nr_count.so and counts one full-order point of a
smooth state with a non-zero shift, dissipation on.  The restatement follows
the reference's generated code operation by operation, so the counts are the
reference's algorithmic work on that path.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, ".."))
from baum_b200 import abi, synthetic  # noqa: E402

SO = os.path.join(HERE, "_ref", "nr_count.so")


def build():
    os.makedirs(os.path.dirname(SO), exist_ok=True)
    subprocess.run(["g++", "-O1", "-x", "c++", "-DORACLE_COUNT_FLOPS", "-fPIC", "-shared",
                    os.path.join(HERE, "nr_oracle.c"), "-o", SO], check=True)
    return C.CDLL(SO)


def count(L, system, params):
    lev = abi.Level.single_box(16, 0.3)
    x, y, z = lev.coords()
    nv = abi.NVARS if system == "bssn" else abi.Z4_NVARS
    unit = synthetic.BSSN_UNIT if system == "bssn" else synthetic.Z4_UNIT
    u = np.ascontiguousarray(synthetic.fourier_state(x, y, z, nv, unit, 8, 0.05, 16.0, 3))
    ptrs = abi.ptr_array([u.ctypes.data + v * u.strides[0] for v in range(nv)])
    f, t = C.c_longlong(), C.c_longlong()
    fn = L.oracle_count_point if system == "bssn" else L.oracle_count_z4_point
    fn(C.byref(lev.desc), ptrs, 8, 8, 8, C.byref(params), C.byref(f), C.byref(t))
    return f.value, t.value


def main():
    L = build()
    out = {}
    for name, system, params in (
            ("bssn_o4_ko6", "bssn", abi.bssn_params()),
            ("bssn_o6_ko6", "bssn", abi.bssn_params(order_centered=6, order_advection=6)),
            ("z4c_o4_ko6", "z4c", abi.z4_params()),
            ("z4c_o6_ko6", "z4c", abi.z4_params(order_centered=6, order_advection=6))):
        f, t = count(L, system, params)
        out[name] = {"flops": f, "transcendental": t}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
