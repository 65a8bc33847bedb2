"""Benchmark of the BSSN evolution hot path on B200.

Workload (one "step"): one RK4 step of the single Schwarzschild puncture,
BSSN, 1+log withshift + Gamma-driver (eta = 2), 4th-order centred and
lopsided advection, KO6 (dissipation_factor 0.1), radiative boundary, on a
66^3 box (64^3 inner points, dx = 0.25): four fused rhs stages, boundary,
RK updates and the algebraic constraints.  RHS point-updates per step =
4 x 64^3.  Initial data: analytic Brill-Lindquist (synthetic, no files).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs independent replicas, one per GPU (the path does not shard).
Prints one JSON line (rank 0).
"""
import argparse
import ctypes as C
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RHS point-updates/s at <=1e-12 rel err vs plain; V-cycles to 1e-10 residual"
UNIT = "RHS point-updates/s"
N_INNER = 64
DX = 0.25
DT = 0.25 * DX
PTS_PER_RHS = N_INNER ** 3
RHS_PER_STEP = 4
# algorithmic FP64 work of one inner point: operators of the reference's
# generated rhs (bssn_rhs_movpunc_N.c) on its 4th-order + KO6 path
FLOP_PER_POINT = 4973
# DRAM bytes of one RK-stage launch of bssn_rhs_kernel on the 64^3 box, block 32 x 8 x 1
# (dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture, mean of
# the two captured launches, stages 1 and 2: 108.6 MB and 216.5 MB)
RHS_TRAFFIC_BYTES = 162.6e6
CONFIG = {"workload": "bssn_schwarzschild_64^3_rk4", "box": "66^3 (64^3 inner + boundary layer)",
          "dx": DX, "dt": DT, "order": 4, "dissipation": "KO6 eps=0.1", "gauge": "1+log, Gamma-driver eta=2",
          "l2": "flushed (256 MiB write) before every timed step", "parallelism": "replicas"}


def sample_clocks_start():
    if not shutil.which("nvidia-smi"):
        return None
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    idx = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0] or "0"
    p = subprocess.Popen(["nvidia-smi", "-i", idx, "--query-gpu=" + q, "--format=csv,noheader,nounits",
                          "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
    return p, f


def sample_clocks_stop(h):
    if h is None:
        return None
    p, f = h
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    f.seek(0)
    rows = [r.split(",") for r in f.read().strip().splitlines() if r.strip()]
    f.close()
    os.unlink(f.name)
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for r in rows:
        try:
            sm.append(float(r[1]))
            mx.append(float(r[2]))
        except (ValueError, IndexError):
            continue
        for n, v in zip(names, r[5:9]):
            if v.strip().lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm)}


def reference_cpu(steps, warmup, cores=None, nxyz=N_INNER):
    """Time the reference's own CPU evolution (oracle/_ref/bam, built from the
    reference sources) on this host: same workload, all host threads."""
    bam = os.path.join(ROOT, "oracle", "_ref", "bam")
    cores = cores or os.cpu_count() or 1
    if not os.path.exists(bam):
        return None
    par = """physics = adm bssn punctures
mass1 = 1
mass2 = 0
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
bssn_lapse = 1+log withshift
bssn_shift = gamma0 withGadv withBadv withShiftadv
bssn_shiftdriver = 2.0
bssn_shiftgammacoeff = 0.75
grid = box
nxyz = %d
dxyz = %g
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
dissipation_factor = 0.1
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
iterations = %d
boundary = radiative
bampi_timer_on = yes
""" % (nxyz, DX, steps + warmup)
    work = tempfile.mkdtemp(prefix="bamref_")
    try:
        with open(os.path.join(work, "c1.par"), "w") as f:
            f.write(par)
        t0 = time.time()
        r = subprocess.run([bam, "-nt", str(cores), "c1.par"], cwd=work, capture_output=True, text=True)
        wall = time.time() - t0
        if r.returncode:
            return None
        txt = open(os.path.join(work, "c1", "timer.0")).read()
        # level-0 timers printed (and reset) after each top-level iteration
        blocks = re.split(r"Timers after top level iteration (\d+)", txt)
        ev, rh = {}, {}
        for i in range(1, len(blocks), 2):
            it = int(blocks[i])
            m = re.search(r"^ 0 evolve\s+([\d.]+)\s+(\d+)", blocks[i + 1], re.M)
            n = re.search(r"^ 0 bssn_rhs\s+([\d.]+)\s+(\d+)", blocks[i + 1], re.M)
            if m:
                ev[it] = float(m.group(1))
            if n:
                rh[it] = float(n.group(1))
        last = steps + warmup
        t_ev = sum(ev[i] for i in range(warmup + 1, last + 1))
        t_rh = sum(rh[i] for i in range(warmup + 1, last + 1))
        pts = nxyz ** 3 * RHS_PER_STEP * steps
        return {"value": pts / t_ev, "rhs_only_value": pts / t_rh if t_rh > 0 else None, "cores": cores,
                "seconds": t_ev, "wall_s": wall,
                "sample": "%d RK4 steps (after %d warm-up) of the %d^3-inner puncture box, reference "
                          "timer 'evolve' (rhs + boundary + RK updates)" % (steps, warmup, nxyz)}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def reference_cpu_median(steps, warmup, runs=3):
    """reference_cpu run `runs` times: the run with the median rate, and all
    rates."""
    res = [reference_cpu(steps, warmup) for _ in range(runs)]
    if any(r is None for r in res):
        return None
    res.sort(key=lambda r: r["value"])
    med = dict(res[len(res) // 2])
    med["runs"] = [r["value"] for r in res]
    med["sample"] += "; median of %d runs" % runs
    return med


MG_BINARIES_SEED = 2024
# V-cycle cap of the binary-puncture runs: from u = 0 the draws of the
# workload's distribution need more than 2000 cycles on the x in
# [-16.1, 16.1] domain
MG_VCYCLE_NMAX = 6000
MG_PAR = """physics = adm punctures multigrid
mass1 = %.17g
px1 = %.17g
my1 = %.17g
sx1 = %.17g
sy1 = %.17g
sz1 = %.17g
mass2 = %.17g
px2 = %.17g
my2 = %.17g
sx2 = %.17g
sy2 = %.17g
sz2 = %.17g
punctures_solver = multigrid
punctures_tolerance = 1e-10
grid = box
nxyz = %d
dxyz = %.17g
mg_verbose = some
mg_vcycle_nmax = 2000
mg_relax_npre = 3
mg_relax_npost = 3
mg_size_nmin = 4
mg_exact_nmin = 10
mg_exact_nmax = 200
iterations = 0
"""


def mg_binaries(n):
    """The standard binary (m = 0.5 each at x = +-4, P_y = +-0.1,
    S_z = +-0.1), then n - 1 seeded draws of the workload's parameter
    distribution (they are not among the warm start's training draws, which
    use other seeds)."""
    import numpy as np
    from baum_b200 import punctures
    rng = np.random.default_rng(MG_BINARIES_SEED)
    fixed = punctures.Binary([0.5, 0.5], [[4, 0, 0], [-4, 0, 0]], [[0, 0.1, 0], [0, -0.1, 0]],
                             [[0, 0, 0.1], [0, 0, -0.1]])
    return [fixed] + [punctures.Binary.sample(rng) for _ in range(n - 1)]


def reference_mg(binary, nxyz, dx, cores=None):
    """The reference's puncture multigrid (oracle/_ref/bam) on this host:
    V cycles and seconds to the 1e-10 RMS residual."""
    bam = os.path.join(ROOT, "oracle", "_ref", "bam")
    if not os.path.exists(bam):
        return None
    b = binary
    par = MG_PAR % (b.mass[0], b.pos[0][0], b.mom[0][1], b.spin[0][0], b.spin[0][1], b.spin[0][2],
                    b.mass[1], b.pos[1][0], b.mom[1][1], b.spin[1][0], b.spin[1][1], b.spin[1][2], nxyz, dx)
    work = tempfile.mkdtemp(prefix="bammg_")
    try:
        with open(os.path.join(work, "mg.par"), "w") as f:
            f.write(par)
        t0 = time.time()
        r = subprocess.run([bam, "-nt", str(cores or os.cpu_count() or 1), "mg.par"], cwd=work,
                           capture_output=True, text=True)
        wall = time.time() - t0
        m = re.search(r"after (\d+) V-cycles", r.stdout)
        if r.returncode or not m:
            return None
        return {"vcycles": int(m.group(1)), "seconds": wall}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def gpu_mg(m, dx, binaries, warm=False, nmax=2000):
    """V cycles, ms and final RMS residual to 1e-10 for each binary: full-V
    from u = 0 (the reference's default); with warm, also V cycles from
    u = 0 and from the learned warm start (the network's u in FP32 and its
    smoothing sweeps, timed with the solve).  A count of nmax is the cap
    ("capped": the residual stayed above 1e-10)."""
    import torch
    from baum_b200 import abi, punctures, warmstart
    mg = punctures.Multigrid(m, dx, abi.mg_params(vcycle_nmax=nmax))
    mgv = punctures.Multigrid(m, dx, abi.mg_params(vcycle_nmax=nmax, fullV=0)) if warm else None
    net = warmstart.Network.load() if warm else None
    out = []

    def run(solver, a, bb, start):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u = start()
        n, res = solver.solve(a, bb, u)
        torch.cuda.synchronize()
        return {"vcycles": n, "ms": round(1e3 * (time.perf_counter() - t0), 2), "residual": res,
                "capped": bool(res > 1e-10)}

    zeros = lambda: torch.zeros(m ** 3, dtype=torch.float64, device="cuda")  # noqa: E731
    for b in binaries:
        a, bb = mg.coefficients(b)
        mg.solve(a, bb, zeros())  # warm-up: stack, graphs
        row = {"fullV_from_zero": run(mg, a, bb, zeros)}
        if warm:
            mgv.solve(a, bb, zeros())
            row["V_from_zero"] = run(mgv, a, bb, zeros)
            row["V_from_warm_start"] = run(mgv, a, bb, lambda: warmstart.warm_guess(net, mgv, b, m, dx))
            row["V_from_warm_start_tc"] = run(mgv, a, bb,
                                              lambda: warmstart.warm_guess(net, mgv, b, m, dx, path="tc"))
        out.append(row)
    mg.close()
    if warm:
        mgv.close()
        net.close()
    return out


def mlp_inference(m, dx, reps=20):
    """The warm start's network evaluated on the m^3 grid, three ways, timed
    with CUDA events on the launching stream (mean over reps after 3
    warm-ups): BF16 through the training path's kernels (features, four
    mma.sync GEMMs with bias + SiLU, the output layer), FP32 on the CUDA
    cores, and BF16 in one tcgen05 kernel.  Each call (ms_per_call) includes
    the upload of the binary's conditioning vector before its kernels.
    FLOPs per point: 2 (32 x 128 + 3 x 128 x 128 + 128) = 106,752."""
    import torch
    from baum_b200 import warmstart
    net = warmstart.Network.load()
    b = mg_binaries(1)[0]
    u = torch.empty(m ** 3, dtype=torch.float64, device="cuda")
    paths = {"bf16_mma_sync": lambda: net.predict_u(b, m, dx, out=u),
             "fp32_simt": lambda: net.predict_u_fp32(b, m, dx, out=u),
             "bf16_tcgen05": lambda: net.predict_u_tc(b, m, dx, out=u, check=False)}
    flops = 2.0 * (32 * 128 + 3 * 128 * 128 + 128) * m ** 3
    out = {"grid": "%d^3" % m, "flop_per_point": 106752}
    for name, fn in paths.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(reps):
            # each call uploads the conditioning table and synchronises the
            # stream first, so every launch is bracketed by its own events
            fn()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record()
            fn()
            s1.record()
            torch.cuda.synchronize()
            ms += s0.elapsed_time(s1)
        ms /= reps
        out[name] = {"ms_per_call": round(ms, 4), "tflops": round(flops / ms * 1e-9, 2)}
    flag = 0
    try:
        net.predict_u_tc(b, m, dx, out=u)
    except Exception as e:  # a bounded wait ran out
        flag = str(e)
    out["bf16_tcgen05"]["timed_out"] = flag
    net.close()
    return out


from baum_b200.workloads import C5_DX0, C5_SIZES, FMR_DX0, FMR_SIZES  # noqa: E402


# start positions of the tracked punctures in the FMR workload (inside the
# finest level of the nested boxes)
TRACK_START = [[0.3, 0.1, 0.0], [-0.3, -0.1, 0.0]]


def gpu_fmr(steps=2, variants=(("graph", 1, 1), ("launches", 0, 1), ("graph_untuned_32x4", 1, 0),
                                ("graph_tracked", 1, 1, True)), warm=2,
            sizes=None, dx0=None, order=4):
    import torch
    from baum_b200 import abi, fmr, workloads
    sizes = sizes or FMR_SIZES
    dx0 = dx0 or FMR_DX0
    levels, params, dt = workloads.fmr_setup(sizes, dx0, order)
    state = workloads.fmr_state_device
    inner = [int((lev.boundary == 0).sum()) for lev in levels]
    upd_per_coarse = sum(n * 4 * 2 ** l for l, n in enumerate(inner))
    out = {"workload": "%d nested 2:1 levels, Z4c %s order + KO%d, Berger-Oliger, order_RP 4, nbuffer 3, "
                       "box points per side %s, dx0 %.3g, Fourier data 1e-3"
                       % (len(sizes), "4th" if order == 4 else "6th", 6, sizes, dx0),
           "rhs_point_updates_per_coarse_step": upd_per_coarse}
    # parity of the benchmarked grid: one coarse step from the initial data
    # against the oracle's stored state of the same grid
    fixture = os.path.join(ROOT, "tests", "golden", "fmr_c3_oracle.npz")
    if sizes == FMR_SIZES and order == 4 and os.path.exists(fixture):
        H = fmr.Hierarchy(levels, dt, params)
        u = [state(lev) for lev in levels]
        H.advance(u, 1)
        torch.cuda.synchronize()
        H.close()
        e_pts, e_sum = workloads.stored_state_deviation(u, fixture)
        tol = [workloads.level_tolerance(l) for l in range(len(levels))]
        out["parity"] = {"vs": "oracle state after 1 coarse step (tests/golden/fmr_c3_oracle.npz): every "
                               "variable at 512 seeded points per level, per-variable sums",
                         "rel_err_points_per_level": e_pts, "rel_err_sums_per_level": e_sum,
                         "tol_per_level": tol, "tol_sums": 1e-12,
                         "ok": bool(all(e < t for e, t in zip(e_pts, tol)) and max(e_sum) < 1e-12)}
        del u
        torch.cuda.empty_cache()
    # the product configuration (graph + per-level tuned block shapes), then
    # plain launches, then the graph with every level at the 32 x 4 default,
    # then the product configuration tracking two punctures on the finest
    # level (two tracker launches per finest-level step)
    for v in variants:
        key, use_graph, tune = v[:3]
        track = len(v) > 3 and v[3]
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=use_graph, autotune=tune))
        if track:
            H.track(TRACK_START)
        blocks = ["%dx%dx%d" % H.block(l) for l in range(len(levels))]
        u = [state(lev) for lev in levels]
        H.advance(u, 1)   # first coarse step: 2nd-order time interpolation, no graph
        for _ in range(warm - 1):
            H.advance(u, 1)   # graph capture (with use_graph)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        H.advance(u, steps)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        out[key] = {"ms_per_coarse_step": ms, "value": upd_per_coarse / (ms * 1e-3), "blocks": blocks}
        finite = all(bool(torch.isfinite(t).all()) for t in u)
        out[key]["finite"] = finite
        if track:
            pos, st = H.punctures()
            out[key]["punctures"] = pos.tolist()
            out[key]["tracker_status"] = st.tolist()
        H.close()
        del u
        torch.cuda.empty_cache()
    out["value"] = out["graph"]["value"]
    out["unit"] = UNIT
    return out


def gpu_fmr_moving(steps=1, warm=1, order=6, omega=0.3, radius=1.0):
    """The full form's grid with moving boxes: 9 nested 2:1 levels, level 0
    a 192^3-inner box (dx 0.5), levels 1-4 the fixed 136^3 cubes about the
    origin (amr_move_lcube = 4), levels 5-8 a 72^3 box around each of two
    punctures (amr_nxyz = 192 128 128 128 128 64), which follow the forced
    circular motion amr_move_force = 3 (radius 1, angular velocity 0.3;
    Fourier data carry no punctures to track).  Z4c 6th order + KO6.  The
    boxes move where the reference's move_box would (baum_b200/moving.py,
    nrgpu_fmr_regrid); coarse steps run without the CUDA graph."""
    import torch
    from baum_b200 import abi, fmr, moving, workloads
    nxyz = [192, 128, 128, 128, 128, 64]
    sizes = lambda lp: moving.box_size(lp, 192, lcube=4, nxyz_list=nxyz)  # noqa: E731
    pos = moving.circle_positions(radius, omega)
    levels = fmr.nested_levels([194], C5_DX0)
    for lp in range(8):
        h = levels[lp].dx
        boxes, ibox = moving.nested_bboxes(h, sizes(lp), pos(0.0), moving=lp + 1 > 4)
        levels.append(moving.level_of_bboxes(boxes, ibox, h))
    params = [abi.z4_params_from_par(dissfactor=(0.1 if l == 0 else 0.02) / 64, order_centered=order,
                                     order_advection=order) for l in range(9)]
    dt = [0.25 * C5_DX0 / 2 ** l for l in range(9)]
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=1, autotune=1))
    policy = moving.MovingBoxes(H, pos, sizes, lcube=4)
    u = [workloads.fmr_state_device(lev) for lev in levels]
    policy.u = u
    H.set_move(policy.hook)
    for _ in range(warm):
        H.advance(u, 1)
    torch.cuda.synchronize()
    nmoves0 = len(policy.moves)
    upd = sum(int((H.levels[l].boundary == 0).sum()) * 4 * 2 ** l for l in range(9))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    H.advance(u, steps)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    out = {"workload": "9 levels: 194^3 (dx 0.5), 4 fixed 136^3 cubes, 4 levels of two 72^3 puncture boxes on "
                       "a forced circular motion (radius %.3g, omega %.3g), Z4c %s order + KO6" %
                       (radius, omega, "6th" if order == 6 else "4th"),
           "ms_per_coarse_step": ms, "rhs_point_updates_per_coarse_step_at_end": upd,
           "value": upd / (ms * 1e-3), "unit": UNIT,
           "moves_per_coarse_step": (len(policy.moves) - nmoves0) / steps,
           "levels_moved_per_coarse_step": sum(sum(x is not None for x in m[2]) for m in policy.moves[nmoves0:]) /
           steps,
           "boxes_per_level_at_end": [H.levels[l].desc.nboxes for l in range(9)],
           "finite": all(bool(torch.isfinite(t).all()) for t in u)}
    H.set_move(None)
    H.close()
    return out


FMR_REF_PAR = """physics = adm z4 nrharness
adm_data = Minkowski
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = box
amr = bo newfmr
amr_fmr = nestedboxes
amr_lmax = 2
amr_nbuffer = 3
nxyz = %d
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
dissipation_factor = 0.1
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
iterations = %d
mass1 = 1
mass2 = 0
nrharness_dir = .
nrharness_data = fourier
nrharness_amp = 1e-3
nrharness_length = 16
nrharness_flags = yes
"""


def fmr_same_grid(nxyz=48, cores=None):
    """The reference's own 3-level Berger-Oliger Z4c run (oracle/_ref/bam,
    all host threads) against this build on the grid the reference made:
    the GPU reads the reference's level boxes and flags from its dumps.  A
    coarse step's time is the difference of a 3- and a 1-iteration run."""
    import torch
    from baum_b200 import abi, fmr, synthetic
    from oracle import dumpfile
    bam = os.path.join(ROOT, "oracle", "_ref", "bam")
    if not os.path.exists(bam):
        return None
    cores = cores or os.cpu_count() or 1
    walls, work = {}, None
    for its in (1, 3):
        work = tempfile.mkdtemp(prefix="bamfmr_")
        with open(os.path.join(work, "f.par"), "w") as f:
            f.write(FMR_REF_PAR % (nxyz, its))
        t0 = time.time()
        r = subprocess.run([bam, "-nt", str(cores), "f.par"], cwd=work, capture_output=True, text=True)
        walls[its] = time.time() - t0
        if r.returncode:
            shutil.rmtree(work, ignore_errors=True)
            return None
        if its == 1:
            levels = []
            for l in range(3):
                d = dumpfile.read(os.path.join(work, "flags_l%d.bin" % l))
                b = d["boxes"][0]
                levels.append(abi.Level([(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6])], float(d["dx"]),
                                        d["boundary"]))
        shutil.rmtree(work, ignore_errors=True)
    ref_s = (walls[3] - walls[1]) / 2
    inner = [int((lev.boundary == 0).sum()) for lev in levels]
    upd = sum(n * 4 * 2 ** l for l, n in enumerate(inner))
    params = [abi.z4_params_from_par(dissfactor=(0.1 if l == 0 else 0.02) / 64) for l in range(3)]
    dt = [0.25 * lev.desc.dx for lev in levels]
    H = fmr.Hierarchy(levels, dt, params)
    u = []
    for lev in levels:
        x, y, z = (torch.from_numpy(c).cuda() for c in lev.coords())
        u.append(synthetic.fourier_state_device(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 1e-3, 16.0, 1))
    H.advance(u, 2)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    H.advance(u, 4)
    b.record()
    torch.cuda.synchronize()
    gpu_ms = a.elapsed_time(b) / 4
    H.close()
    return {"workload": "reference's 3-level Z4c grid, nxyz %d, dxyz 0.5, boxes per side %s"
                        % (nxyz, [lev.boxes[0].m for lev in levels]),
            "rhs_point_updates_per_coarse_step": upd,
            "gpu": {"ms_per_coarse_step": gpu_ms, "value": upd / (gpu_ms * 1e-3)},
            "reference": {"s_per_coarse_step": ref_s, "value": upd / ref_s, "cores": cores,
                          "timing": "wall time of a 3-iteration minus a 1-iteration run, over 2"}}


# the binary's grid in BAM (Z4c, punctures at x = +-2.75 place one box per
# puncture on each finer level), for the batched-over-plain ratio: the same
# parfile in the reference binary with the B200 module (oracle/_ref/bam_gpu)
# in callback mode (the plain per-box drop-in: BAM's own Berger-Oliger
# recursion, RK4 and restriction/prolongation on the host, every rhs and
# boundary evaluation on the GPU with the level's lists copied over and
# back) and in fmr mode (the whole coarse step of all levels on the device,
# replayed as a CUDA graph); the plain reference on the host cores beside them
BATCH_PAR = """physics = adm z4 punctures nrharness%s
adm_data = Minkowski
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = box
amr = bo newfmr
amr_fmr = nestedboxes
amr_lmax = %d
amr_nbuffer = 3
nxyz = %d
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
dissipation_factor = 0.1
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
iterations = %d
mass1 = 0.5
px1 = 2.75
mass2 = 0.5
px2 = -2.75
punctures_solver = none
nrharness_data = fourier
nrharness_amp = 1e-3
nrharness_length = 16
%s
"""


def batching_ratio(lmax=4, nxyz=48, cores=None, with_reference=True):
    """Seconds per coarse step of the binary grid in the three binaries: the
    wall-time difference of two runs of different lengths over the extra
    coarse steps (1 and 3 for the slow binaries; 2 and 42 for the fmr mode,
    whose coarse step is far shorter than the run-to-run spread of start-up,
    level set-up and autotuning)."""
    bam, bam_gpu = (os.path.join(ROOT, "oracle", "_ref", b) for b in ("bam", "bam_gpu"))
    if not (os.path.exists(bam) and os.path.exists(bam_gpu)):
        return None
    cores = cores or os.cpu_count() or 1
    runs = {"fmr": (bam_gpu, " nrgpu", "nrgpu_mode = fmr\nz4_register_algcon = no", (2, 42)),
            "callback": (bam_gpu, " nrgpu", "nrgpu_mode = callback", (1, 3)),
            "reference": (bam, "", "", (1, 3))}
    if not with_reference:
        del runs["reference"]
    out = {"grid": "BAM binary grid: Z4c, punctures m = 0.5 at x = +-2.75, amr_lmax %d, nxyz %d, dxyz 0.5, "
                   "4th order + KO6, Fourier data 1e-3" % (lmax, nxyz), "cores": cores}
    for key, (binary, phys, extra, lens) in runs.items():
        walls = {}
        for its in lens:
            work = tempfile.mkdtemp(prefix="bambatch_")
            try:
                with open(os.path.join(work, "b.par"), "w") as f:
                    f.write(BATCH_PAR % (phys, lmax, nxyz, its, extra))
                t0 = time.time()
                r = subprocess.run([binary, "-nt", str(cores), "b.par"], cwd=work, capture_output=True, text=True,
                                   timeout=1800)
                walls[its] = time.time() - t0
                if r.returncode:
                    out[key] = {"error": (r.stdout[-400:] + r.stderr[-400:])}
                    break
            finally:
                shutil.rmtree(work, ignore_errors=True)
        if len(walls) == 2:
            out[key] = {"s_per_coarse_step": (walls[lens[1]] - walls[lens[0]]) / (lens[1] - lens[0]),
                        "runs": {str(k): round(v, 2) for k, v in walls.items()}}
    if all("s_per_coarse_step" in out.get(k, {}) for k in ("fmr", "callback")):
        out["batched_over_plain"] = out["callback"]["s_per_coarse_step"] / out["fmr"]["s_per_coarse_step"]
    return out


def oracle_port_cpu():
    """Fallback CPU baseline: the oracle restatement, one RK4 step."""
    from oracle import oracle
    from baum_b200 import abi, punctures
    lev, u = punctures.schwarzschild_c1(N_INNER, DX)
    p = abi.bssn_params()
    t0 = time.time()
    oracle.bssn_evolve(lev, u, DT, 1, p)
    t = time.time() - t0
    return {"value": PTS_PER_RHS * RHS_PER_STEP / t, "cores": os.cpu_count() or 1,
            "sample": "1 RK4 step of the 64^3-inner puncture box (oracle restatement, OpenMP)"}


def count_launches(fn):
    """Kernels of this library launched by fn(): one call under the CUDA
    activity profiler (outside every timed region), counting kernel records
    that are not torch's own (fills, copies) or the runtime's memset/memcpy."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    names = []
    for e in prof.events():
        if e.device_type != torch.autograd.DeviceType.CUDA:
            continue
        n = e.name
        if "at::" in n or "Memcpy" in n or "Memset" in n or "memcpy" in n or "memset" in n:
            continue
        names.append(n)
    short = set()
    for n in names:
        m = re.findall(r"([a-z][a-z0-9_]*_kernel)", n)
        short.add(m[-1] if m else n[:40])
    return len(names), sorted(short)


def max_over_ranks(values, device):
    """Each value's maximum over the ranks of the process group (all-reduce
    MAX; the values themselves when no group of more than one rank is
    initialised)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 20))
    warm = 1
    res = reference_cpu_median(steps, warm)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/bam not built on this host"}))
        return
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * res["seconds"] / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic Brill-Lindquist puncture)", "config": CONFIG,
            "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": res["cores"], "kind": "reference",
                             "sample": res["sample"]},
            "rhs_only_value": res["rhs_only_value"], "runs": res["runs"],
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_ours(args, rank, world):
    import numpy as np
    import torch
    from baum_b200 import abi, build, bssn, punctures

    build.build()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    L = abi.lib()
    lev, u0 = punctures.schwarzschild_c1(N_INNER, DX)
    p = abi.bssn_params()
    dl = bssn.DeviceLevel(lev, dev)
    u = torch.from_numpy(u0).cuda()
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    block = dl.autotune(abi.SYSTEM_BSSN, p, stream)   # the level's rhs block shape

    def step():
        bssn.evolve_rk_rk4(dl, u, DT, p, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clk = sample_clocks_start() if rank == 0 else None
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()
        ev[s][0].record(stream)
        step()
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev)

    # dominant kernel alone: the interior rhs launch, timed with events on
    # the launching stream, L2 flushed before each launch
    r = dl.empty()
    rev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
    bssn.bssn_rhs_movpunc_N(dl, r, u, 0.0, u, p, stream)
    for a, b in rev:
        flush.zero_()
        a.record(stream)
        bssn.bssn_rhs_movpunc_N(dl, r, u, 0.0, u, p, stream)
        b.record(stream)
    torch.cuda.synchronize()
    rhs_ms = sum(a.elapsed_time(b) for a, b in rev) / len(rev)
    clocks = sample_clocks_stop(clk) if rank == 0 else None
    if args.case == "c1-step":
        if rank == 0:
            units = PTS_PER_RHS * RHS_PER_STEP * args.steps * world
            print(json.dumps({"case": "c1-step", "value": units / (ms * 1e-3), "unit": UNIT,
                              "ms_per_step": ms / args.steps, "rhs_launch_ms": rhs_ms,
                              "block": "%dx%dx%d" % block, "clocks": clocks}))
        return

    # this library's kernels in one step, counted by the activity profiler
    per_step, kernel_names = count_launches(step)
    # measured FP64 peak on this GPU (no FP64 entry in the peak list)
    fl, pms = C.c_double(), C.c_float()
    abi.check(L.nrgpu_probe_fp64_peak(4000, C.byref(fl), C.byref(pms)))
    fp64_peak = fl.value / 1e12

    # end to end: host state in pinned memory, one RK4 step per call with the
    # upload and download inside the timed region
    h = torch.from_numpy(u0.copy()).pin_memory()
    bssn.evolve_host(dl, h, 1, DT, p)
    e2e_t = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bssn.evolve_host(dl, h, 1, DT, p)
        e2e_t.append(time.perf_counter() - t0)
    state_bytes = abi.NVARS * lev.npoints * 8

    # the job's times are the slowest rank's (replicas: no data-path exchange)
    ms, e2e_sum = max_over_ranks([ms, sum(e2e_t)], "cuda")
    if rank != 0:
        return
    units = PTS_PER_RHS * RHS_PER_STEP * args.steps * world
    value = units / (ms * 1e-3)
    achieved = FLOP_PER_POINT * PTS_PER_RHS / (rhs_ms * 1e-3) / 1e12
    cpu = reference_cpu_median(10, 1) if world == 1 and not args.no_cpu else None
    if cpu:
        cpu = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "reference",
               "sample": cpu["sample"], "runs": cpu["runs"]}
    elif world == 1 and not args.no_cpu:
        c = oracle_port_cpu()
        cpu = {"value": c["value"], "unit": UNIT, "cores": c["cores"], "kind": "port", "sample": c["sample"]}
    # the multigrid half of the metric: V cycles and ms to the 1e-10 RMS
    # residual on the 129^3-cell binary-puncture grid (dx = 0.25, x in
    # [-16.1, 16.1]): the standard binary and 5 seeded draws of the
    # workload's distribution, full-V from u = 0 as the reference does, V
    # cycles from u = 0 and from the learned warm start; the reference on
    # the same binaries at 66^3 (dx = 0.5, the same domain) for the first two
    from baum_b200 import warmstart
    bins = mg_binaries(6)
    mg130 = gpu_mg(warmstart.C2_M, warmstart.C2_DX, bins, warm=True, nmax=MG_VCYCLE_NMAX)
    mg66 = gpu_mg(66, 0.5, bins[:2])
    ref66 = [reference_mg(b, 64, 0.5) for b in bins[:2]] if not args.no_cpu else [None, None]
    fmr_line = gpu_fmr(2)
    if world == 1 and not args.no_cpu:
        fmr_line["same_grid_reference"] = fmr_same_grid()
        # the batched path against the plain per-box drop-in, both inside BAM
        # (the plain reference on the same grid: bench.py --case batching)
        fmr_line["batched_over_plain"] = batching_ratio(with_reference=False)
    fv = [r["fullV_from_zero"] for r in mg130]
    multigrid = {
        "workload": "binary punctures, Bowen-York, 130^3 points (129^3 cells), dx=0.25 (x in [-16.1, 16.1]), "
                    "tol 1e-10 RMS, cap %d V cycles" % MG_VCYCLE_NMAX,
        "vcycles": [r["vcycles"] for r in fv], "ms": [r["ms"] for r in fv],
        "capped": [r["capped"] for r in fv], "final_residual": [r["residual"] for r in fv],
        "ms_per_vcycle": sum(r["ms"] for r in fv) / max(1, sum(r["vcycles"] for r in fv)),
        "seed": MG_BINARIES_SEED, "per_binary": mg130,
        "warm_start": "network u in FP32 + %d damped Jacobi sweeps (omega %.3g), then V cycles; "
                      "V_from_warm_start_tc: the BF16 u of the tcgen05 kernel + the same sweeps"
                      % (warmstart.NSMOOTH, warmstart.OMEGA),
        "inference": mlp_inference(warmstart.C2_M, warmstart.C2_DX),
        "same_grid_66": [{"gpu_vcycles": g["fullV_from_zero"]["vcycles"], "gpu_ms": g["fullV_from_zero"]["ms"],
                          "gpu_residual": g["fullV_from_zero"]["residual"],
                          "reference_vcycles": r["vcycles"] if r else None,
                          "reference_s": round(r["seconds"], 2) if r else None,
                          "reference_cores": os.cpu_count()} for g, r in zip(mg66, ref66)],
    }
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Brill-Lindquist puncture)",
        "config": CONFIG,
        "roofline": {"bound": "fp64", "kernel": "bssn_rhs_kernel (interior rhs, one launch = 64^3 points)",
                     "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                     "peak_source": "measured FP64 FMA probe on this GPU (nrgpu_probe_fp64_peak)",
                     "flop_per_point": FLOP_PER_POINT, "launch_ms": rhs_ms, "traffic": RHS_TRAFFIC_BYTES,
                     "block": "%dx%dx%d" % block},
        "cpu_baseline": cpu,
        "e2e": {"value": PTS_PER_RHS * RHS_PER_STEP * args.steps * world / e2e_sum, "unit": UNIT,
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "call": "nrgpu_bssn_evolve_host(nsteps=1) from pinned host memory"},
        "gpu_launches": per_step * args.steps,
        "gpu_launches_per_step": {"count": per_step, "kernels": kernel_names,
                                  "how": "one step under the CUDA activity profiler, outside the timed region"},
        "clocks": clocks,
        "multigrid": multigrid,
        "fmr": fmr_line,
    }
    print(json.dumps(line))


def run_c1_kernels(args):
    """The interior rhs of the 64^3 BSSN box in its three forms, each timed
    alone (rhs evaluation, CUDA events, L2 flushed before each launch):
    the per-point kernel with the tuned block shape (64 x 4 x 1), the staged-tile kernel
    one block per tile, and its persistent form.  A shift is set so that
    every term takes part.  For profiling (ncu -k regex:bssn_rhs)."""
    import numpy as np
    import torch
    from baum_b200 import abi, build, bssn, punctures
    build.build()
    torch.cuda.set_device(0)
    lev, u0 = punctures.schwarzschild_c1(N_INNER, DX)
    x, _, _ = lev.coords()
    u0[18] = 0.05 * np.sin(0.3 * x)
    p = abi.bssn_params()
    u = torch.from_numpy(u0).cuda()
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")
    out = {"case": "c1-kernels"}
    ref = None
    for mode in (0, 1, 2):
        dl = bssn.DeviceLevel(lev)
        if mode == 0:
            dl.set_block(64, 4, 1)   # the shape the tuner picks for this box
            out["block"] = "64x4x1"
        else:
            dl.tile(mode)
        r = dl.empty()
        ts = []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            bssn.bssn_rhs_movpunc_N(dl, r, u, 0.0, u, p)
            b.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                ts.append(a.elapsed_time(b))
        ms = float(np.median(ts))
        rh = r.cpu().numpy()
        if ref is None:
            ref = rh
        err = max(float(np.abs(rh[v] - ref[v]).max() / max(np.abs(ref[v]).max(), 1e-8)) for v in range(abi.NVARS))
        out[["per_point", "tile", "tile_persistent"][mode]] = {
            "rhs_ms": ms, "tflops": FLOP_PER_POINT * PTS_PER_RHS / (ms * 1e-3) / 1e12, "rel_err_vs_per_point": err}
        dl.close()
    print(json.dumps(out))


def run_precision_fmr(args):
    """The FP32-stencil option where it is meant to apply: the batched
    7-level Z4c grid with precision 1 (KO sums in FP32) or 2 (KO and centred
    derivative sums in FP32) on the outer levels 0-2 only, the inner levels
    FP64.  After --steps coarse steps (the first with 2nd-order time
    interpolation) from the same data: per level and variable the largest
    difference to the FP64 run relative to the variable's size, the change
    of the Hamiltonian and momentum constraint norms on levels 0-2, and the
    time per coarse step (graph replay, tuned shapes)."""
    import copy
    import numpy as np
    import torch
    from baum_b200 import abi, adm, build, bssn, fmr, workloads
    build.build()
    torch.cuda.set_device(0)
    levels, params, dt = workloads.fmr_setup()
    out = {"case": "precision-fmr", "levels_with_option": [0, 1, 2], "coarse_steps": args.steps}
    ref = None
    for prec in (0, 1, 2):
        pp = [copy.copy(q) for q in params]
        for l in (0, 1, 2):
            pp[l].precision = prec
        H = fmr.Hierarchy(levels, dt, pp)
        u = [workloads.fmr_state_device(lev) for lev in levels]
        H.advance(u, 1)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        H.advance(u, args.steps - 1)
        b.record()
        torch.cuda.synchronize()
        H.close()
        row = {"ms_per_coarse_step": a.elapsed_time(b) / max(1, args.steps - 1)}
        cons = []
        for l in (0, 1, 2):
            dl = bssn.DeviceLevel(levels[l])
            _, _, nrm = adm.computeadmconstraints(dl, u[l], 4)
            cons.append([nrm["ham"][0], max(nrm[k][0] for k in ("momx", "momy", "momz"))])
            dl.close()
        row["constraint_norms_l012"] = cons
        if ref is None:
            ref = u
        else:
            per = []
            for l in range(len(levels)):
                d = (u[l] - ref[l]).abs().amax(dim=1) / ref[l].abs().amax(dim=1).clamp_min(1e-8)
                per.append(d.cpu().numpy().tolist())
            row["rel_err_per_level_per_variable"] = per
            row["max_rel_err_per_level"] = [max(x) for x in per]
            rc = out["precision_0"]["constraint_norms_l012"]
            row["constraint_norm_rel_change_l012"] = [[abs(c[i] - r[i]) / r[i] for i in range(2)]
                                                      for c, r in zip(cons, rc)]
            del u
        out["precision_%d" % prec] = row
        torch.cuda.empty_cache()
    print(json.dumps(out))


def run_z4c160(args):
    """The precision-sweep box as a throughput case: Z4c, 6th order + KO6,
    160^3 inner points (162^3 with the boundary layer), dx 0.15,
    Brill-Lindquist binary m = 0.5 at x = +-5; RK4 steps with the L2 flushed
    before each.  State 0.85 GB, scratch 2.6 GB."""
    import torch
    from baum_b200 import abi, build, punctures, z4
    build.build()
    torch.cuda.set_device(0)
    n, dx = 160, 0.15
    lev = abi.Level.single_box(n + 2, dx)
    u0 = punctures.z4_brill_lindquist_state(lev, [(0.5, 5.0, 0.0, 0.0), (0.5, -5.0, 0.0, 0.0)])
    p = abi.z4_params(order_centered=6, order_advection=6)
    dl = z4.DeviceLevel(lev)
    block = dl.autotune(abi.SYSTEM_Z4C, p)
    u = torch.from_numpy(u0).cuda()
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        z4.evolve_rk_rk4(dl, u, 0.25 * dx, p)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, b in ev:
        flush.zero_()
        a.record()
        z4.evolve_rk_rk4(dl, u, 0.25 * dx, p)
        b.record()
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    pts = n ** 3
    print(json.dumps({"case": "z4c160", "block": "%dx%dx%d" % block, "metric": "RHS point-updates/s",
                      "value": 4 * pts / (ms * 1e-3),
                      "unit": UNIT, "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
                      "dtype": "f64", "config": {"workload": "Z4c 6th order + KO6, 160^3 inner, dx 0.15, "
                                                             "BL binary m=0.5 at x=+-5", "l2": "flushed"},
                      "finite": bool(torch.isfinite(u).all())}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--case", default="c1", choices=["c1", "c1-step", "c1-kernels", "mg", "fmr", "c5", "z4c160",
                                                      "batching", "precision-fmr", "mlp"],
                    help="c1: the benchmark line; c1-step: only the 64^3 BSSN RK4 steps and the rhs "
                         "launches of that line (for profiling); mg: only the 130^3 multigrid solve of the "
                         "first seeded binary (for profiling); fmr: only the 7-level Z4c step, graph replay with tuned "
                         "blocks, --warmup and --steps coarse steps (for profiling); z4c160: the 160^3 Z4c box "
                         "alone; mlp: the warm start network's inference on the 130^3 grid, three kernels")
    ap.add_argument("--lmax", type=int, default=4, help="with --case batching: finest level of the BAM grid")
    ap.add_argument("--nxyz", type=int, default=48, help="with --case batching: coarse points per side")
    ap.add_argument("--mg-cycles", type=int, default=0,
                    help="with --case mg: run exactly this many V cycles from the finest level (profiling)")
    args = ap.parse_args()
    if args.case == "z4c160":
        run_z4c160(args)
        return
    if args.case == "fmr":
        import torch
        from baum_b200 import build
        build.build()
        torch.cuda.set_device(0)
        print(json.dumps({"case": "fmr", **gpu_fmr(args.steps, variants=(("graph", 1, 1),),
                                                     warm=max(args.warmup, 2))}))
        return
    if args.case == "precision-fmr":
        run_precision_fmr(args)
        return
    if args.case == "c1-kernels":
        run_c1_kernels(args)
        return
    if args.case == "mlp":
        import torch
        from baum_b200 import build, warmstart
        build.build()
        torch.cuda.set_device(0)
        print(json.dumps({"case": "mlp", **mlp_inference(warmstart.C2_M, warmstart.C2_DX, reps=args.steps)}))
        return
    if args.case == "batching":
        print(json.dumps({"case": "batching", **(batching_ratio(args.lmax, args.nxyz) or {"unavailable": "bam_gpu"})}))
        return
    if args.case == "c5":
        import torch
        from baum_b200 import build
        build.build()
        torch.cuda.set_device(0)
        r = gpu_fmr(args.steps, variants=(("graph", 1, 1),), warm=max(args.warmup, 2), sizes=C5_SIZES,
                    dx0=C5_DX0, order=6)
        r["note"] = "static boxes (value); moving: the same depth with moving puncture boxes on the finest levels"
        torch.cuda.empty_cache()
        r["moving"] = gpu_fmr_moving(max(1, args.steps), 1)
        print(json.dumps({"case": "c5", **r}))
        return
    if args.case == "mg":
        import torch
        from baum_b200 import build
        build.build()
        torch.cuda.set_device(0)
        if args.mg_cycles:
            # profiling: exactly K V cycles from the finest level (no full-V
            # start, tolerance 0): the first kernels are the 130^3 sweeps
            from baum_b200 import abi, punctures
            mg = punctures.Multigrid(130, 0.25, abi.mg_params(fullV=0, tol=0.0, vcycle_nmax=args.mg_cycles))
            a, bb = mg.coefficients(mg_binaries(1)[0])
            u = torch.zeros(130 ** 3, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            n, res = mg.solve(a, bb, u)
            torch.cuda.synchronize()
            print(json.dumps({"case": "mg", "vcycles": n, "ms": 1e3 * (time.perf_counter() - t0), "residual": res}))
            mg.close()
            return
        from baum_b200 import warmstart
        r = gpu_mg(warmstart.C2_M, warmstart.C2_DX, mg_binaries(1))[0]["fullV_from_zero"]
        print(json.dumps({"case": "mg", "workload": "binary punctures, Bowen-York, 130^3 points, dx=0.25, "
                                                     "tol 1e-10 RMS, full-V", "seed": MG_BINARIES_SEED, **r,
                          "ms_per_vcycle": r["ms"] / max(1, r["vcycles"])}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
