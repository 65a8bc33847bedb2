"""Build the reference CPU code (BAM) as the oracle binary ``oracle/_ref/bam``.

Test infrastructure only: this compiles the checker, never the product.

The reference sources are compiled where they lie (``REF``, read-only), single
rank against ``oracle/mpi_stub/mpi.h`` (no MPI library in the image), with
OpenMP and the reference's own ``-O2`` flags (reference ``MyConfig:27``).
BAM's own make system is not run: the three files it generates from
``MyConfig`` (``Makefile:108-128``: the automatic include, initialize and
finalize lists) are written here into ``oracle/_ref/gen``, listing the modules
this oracle needs plus the dump harness ``oracle/harness/nrharness.c``.

Usage:  python oracle/build_ref.py [--ref PATH] [-j N]
Outputs only into oracle/_ref/ (git-ignored; travels with the tree).
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# module directory -> object list, as in each module's Makefile OBJS line
MODULES = [
    ("src/main/amr", "bam_amr box check flag grid inject move print points regrid shells storage"),
    ("src/utility/AwA", "bam_AwA AwA"),
    ("src/utility/boundary", "bam_boundary boundary excision extrapolate inversion periodic plane "
                             "radiative robin symmetry tube normals"),
    ("src/utility/checkpoint", "bam_checkpoint checkpoint checkpoint_read checkpoint_write wolfio"),
    ("src/utility/elliptic/iterative", "bam_iterative Newton bicgstab cgs gaussseidel jacobi poisson sor utility"),
    ("src/utility/elliptic/multigrid", "bam_multigrid exactsolve fasmg makestack multigrid relax residual "
                                       "restrictprolong solve utility print"),
    ("src/utility/evolve", "bam_evolve evolve icn rk"),
    ("src/utility/interpolate", "bam_interpolate barycentric interpolate interpolate_boxtobox_N "
                                "interpolate_global lagrange WENO linear"),
    ("src/utility/output", "bam_output output output0d output1d output2d output3d outputVTK outputXDMF "
                           "outputShells outputSphere"),
    ("src/utility/NumericUtils", "bam_NumericUtils integral integral3D newton_lnsrch nrutil f_to_minimize "
                                 "fd_jacobian ludcmp lubksb lnsrch_double rtsafe_itsP attenuation "
                                 "Integral_over_sphere Integral_over_volume Integral_over_volume_4 "
                                 "path_integral fact SphericalHarmonics SphericalHarmonics_precomp"),
    ("src/utility/units", "bam_units units"),
    ("src/projects/adm", "bam_adm adm adm_constraints_N adm_data adm_utility"),
    ("src/projects/bssn", "bam_bssn bssn bssn_init bssn_eta bssn_rhs_movpunc_N bssn_algcon "
                          "bssn_rhs_add_source bssn_boundary"),
    ("src/projects/z4", "bam_z4 z4 z4_boundary z4_boundary_box z4_boundary_box_rad z4_boundary_shell "
                        "z4_init z4_algcon z4_rhs_movpunc_N z4_rhs_add_source"),
    ("src/projects/punctures", "bam_punctures ConformalFactor ExtrinsicCurvature FlagRegrid Lapse Mass "
                               "Punctures PuncturesPS PunctureSolve Shift VectorLieFlat VectorLaplaceFlat "
                               "VectorLaplaceFlatGS OutsideBox FullBox FuncsForOutsideBox Sequences "
                               "forMovingPunctures PunctureData_with_given_M_ADM"),
    ("src/projects/Gauge", "bam_Gauge moving_punctures moving_punctures_integrate puncture_properties "
                           "puncture_properties_integrand"),
    ("src/projects/ADM_mass", "bam_ADM_mass ADM_mass adm_mass_integrand adm_mass_integrand_chi adm_pj_integrand"),
    ("src/projects/Invariants", "bam_Invariants Invariants curvature_invariants_N dphi_int2_psi4_N"),
    # bampi and main go last, as in the reference Makefile
    ("src/main/bampi", "bam_bampi bampi copy debug output openmp profile reduce split_box synchronize "
                       "synchronize_fmr timer"),
    ("src/main/main", "bam_main main parameters physics skeleton system tensors utilities variables"),
]
FINAL = {"main", "adm", "evolve"}  # modules with a bam_<name>_final()


def write_generated(ref, gen, extra=()):
    """extra: (name, header) of further modules, initialised last."""
    os.makedirs(gen, exist_ok=True)
    names = [os.path.basename(d) for d, _ in MODULES] + ["nrharness"] + [n for n, _ in extra]
    inc = ["/* module list for the oracle build (written by oracle/build_ref.py) */"]
    for d, _ in MODULES:
        n = os.path.basename(d)
        inc.append('#include "%s/%s/bam_%s.h"' % (ref, d, n))
    inc.append('#include "%s/harness/bam_nrharness.h"' % HERE)
    for _, h in extra:
        inc.append('#include "%s"' % h)
    init = []
    fin = []
    # the reference calls every module initializer except main's in list order
    for n in names:
        if n == "main":
            continue
        init.append("bam_%s();" % n)
        inc.append("void bam_%s();" % n)
    for n in names:
        if n in FINAL:
            fin.append("bam_%s_final();" % n)
            inc.append("void bam_%s_final();" % n)
    # bam_main() is the first initializer in the reference list too
    init.insert(0, "bam_main();")
    inc.append("void bam_main();")
    files = {"bam_automatic_include.h": inc, "bam_automatic_initialize.c": init,
             "bam_automatic_finalize.c": fin}
    for fn, lines in files.items():
        p = os.path.join(gen, fn)
        txt = "\n".join(lines) + "\n"
        if not os.path.exists(p) or open(p).read() != txt:
            open(p, "w").write(txt)


def main():
    ap = argparse.ArgumentParser()
    # the reference tree: --ref, else $BAM_REFERENCE_DIR, else the build
    # container's read-only copy
    ap.add_argument("--ref", default=os.environ.get("BAM_REFERENCE_DIR", "/root/reference"))
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--cc", default="gcc")
    a = ap.parse_args()
    ref = os.path.abspath(a.ref)
    if not os.path.isdir(os.path.join(ref, "src")):
        print("build_ref: reference not found at %s; oracle/_ref not rebuilt" % ref)
        return 0
    gen = os.path.join(OUT, "gen")
    obj = os.path.join(OUT, "obj")
    os.makedirs(obj, exist_ok=True)
    write_generated(ref, gen)
    base = [a.cc, "-O2", "-DOPENMP", "-fopenmp", "-std=gnu99", "-w", "-fcommon",
            "-I" + gen, "-I" + os.path.join(HERE, "mpi_stub"),
            "-I" + os.path.join(ref, "src/main/main"), "-I" + os.path.join(ref, "src/main/amr"),
            "-I" + os.path.join(ref, "src/main/bampi")]
    jobs = []
    for d, objs in MODULES:
        for f in objs.split():
            src = os.path.join(ref, d, f + ".c")
            o = os.path.join(obj, d.replace("/", "_") + "__" + f + ".o")
            jobs.append((src, o, os.path.join(ref, d)))
    jobs.append((os.path.join(HERE, "harness", "nrharness.c"), os.path.join(obj, "harness__nrharness.o"),
                 os.path.join(HERE, "harness")))
    jobs.append((os.path.join(HERE, "mpi_stub", "mpi_stub.c"), os.path.join(obj, "mpi_stub.o"),
                 os.path.join(HERE, "mpi_stub")))
    stub_h = os.path.join(HERE, "mpi_stub", "mpi.h")

    # the generated module lists are included by main.c: a change of the
    # module list rebuilds it
    gen_t = max(os.path.getmtime(os.path.join(gen, f)) for f in os.listdir(gen))

    def compile_one(job):
        src, o, incdir = job
        deps = [os.path.getmtime(src), os.path.getmtime(stub_h)]
        if src.endswith(os.path.join("main", "main", "main.c")):
            deps.append(gen_t)
        if os.path.exists(o) and os.path.getmtime(o) >= max(deps):
            return None
        cmd = base + ["-I" + incdir, "-c", src, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            return "%s\n%s" % (" ".join(cmd), r.stderr[-4000:])
        return None

    with cf.ThreadPoolExecutor(a.j) as ex:
        errs = [e for e in ex.map(compile_one, jobs) if e]
    if errs:
        print("\n".join(errs))
        return 1
    # link through an archive, as the reference does with its per-module
    # static libraries, so objects nobody references are left out
    exe = os.path.join(OUT, "bam")
    lib = os.path.join(OUT, "libbamref.a")
    if os.path.exists(lib):
        os.remove(lib)
    objs = [o for _, o, _ in jobs]
    entry = [o for o in objs if o.endswith("src_main_main__main.o")]
    subprocess.run(["ar", "rcs", lib] + objs, check=True)
    r = subprocess.run([a.cc, "-fopenmp", "-o", exe] + entry +
                       ["-Wl,--start-group", lib, "-Wl,--end-group", "-lm"],
                       capture_output=True, text=True)
    if r.returncode:
        print(r.stderr[-6000:])
        return 1
    print("build_ref: built", exe)
    return build_gpu_variant(ref, a, base, obj, entry, lib)


def build_gpu_variant(ref, a, base, obj, entry, lib):
    """oracle/_ref/bam_gpu: the same reference with the B200 binding module
    (baum_b200/bam/nrgpu_bam.c) linked against baum_b200/libnrgpu.so, the
    drop-in as a maintainer would add it.  Built only when the library is."""
    repo = os.path.dirname(HERE)
    so = os.path.join(repo, "baum_b200", "libnrgpu.so")
    if not os.path.exists(so):
        print("build_ref: baum_b200/libnrgpu.so not built; oracle/_ref/bam_gpu skipped")
        return 0
    gen = os.path.join(OUT, "gen_gpu")
    write_generated(ref, gen, [("nrgpu", os.path.join(repo, "baum_b200", "bam", "bam_nrgpu.h"))])
    bgen = [x if not x.startswith("-I" + os.path.join(OUT, "gen")) else "-I" + gen for x in base]
    main_o = os.path.join(obj, "gpu__main.o")
    bind_o = os.path.join(obj, "gpu__nrgpu_bam.o")
    for src, o, inc in [(os.path.join(ref, "src/main/main/main.c"), main_o, os.path.join(ref, "src/main/main")),
                        (os.path.join(repo, "baum_b200", "bam", "nrgpu_bam.c"), bind_o,
                         os.path.join(ref, "src/projects/bssn"))]:
        r = subprocess.run(bgen + ["-I" + inc, "-DNRGPU_WRAP_MULTIGRID", "-DNRGPU_WRAP_MOVE_BOX", "-c", src, "-o", o],
                           capture_output=True, text=True)
        if r.returncode:
            print(r.stderr[-4000:])
            return 1
    cuda = "/usr/local/cuda/lib64"
    exe = os.path.join(OUT, "bam_gpu")
    # --wrap=multigrid: PickEllipticSolver's pointer to multigrid() lands on
    # the module's __wrap_multigrid (device solve under nrgpu_multigrid = yes);
    # --wrap=move_box: main.c's move_box lands on __wrap_move_box (the device
    # moves the boxes in nrgpu_mode = fmr)
    r = subprocess.run([a.cc, "-fopenmp", "-o", exe, main_o, bind_o, "-Wl,--wrap=multigrid", "-Wl,--wrap=move_box",
                        "-Wl,--start-group", lib, "-Wl,--end-group",
                        "-L" + os.path.dirname(so), "-lnrgpu", "-Wl,-rpath,$ORIGIN/../../baum_b200",
                        "-L" + cuda, "-lcudart", "-Wl,-rpath," + cuda, "-lm"], capture_output=True, text=True)
    if r.returncode:
        print(r.stderr[-6000:])
        return 1
    print("build_ref: built", exe)
    return 0


if __name__ == "__main__":
    sys.exit(main())
