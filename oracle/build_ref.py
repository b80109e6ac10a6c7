#!/usr/bin/env python3
"""Build the reference's own CPU solver code into oracle/_ref/ (test infrastructure).

    python oracle/build_ref.py <reference Source/ directory>
    (or SPH_REFERENCE_SOURCE=<dir> python oracle/build_ref.py)

Recipe, run in the build container only (the reference tree is not present on
the GPU machines; the built libraries travel there instead):

1. Transcode the reference solver sources (GBK / UTF-16LE, CRLF) to UTF-8 in
   oracle/_ref/src/.  Line numbers are unchanged, so file:line citations into
   the reference still hold.
2. Augment the *copy* of SphBase.h with the particle / threshold members that
   the solver sources use but this revision of SphBase.h does not declare
   (DFSPH.cpp, IISph_M.cpp and WcSph.cpp come from a later revision),
   `friend class RefHarness;` / `friend class SphWithIO;` lines, and an
   #ifdef around the real_t typedef.
   Each edit is inserted at a fixed anchor (AUGMENT); nothing else changes.
3. Compile SphBase.cpp + one solver .cpp + oracle/refshim/ref_harness.cpp into
   one shared library per solver (DFSPH.h, IISph.h and IISph_M.h share the
   include guard II_SPH_H_, so each solver needs its own library):
       oracle/_ref/libref_dfsph.so, libref_wcsph.so, libref_pcisph.so,
       libref_iisphm.so; and the surface reconstruction (surface_field.cpp,
       marching_cubes.cpp) into libref_surface.so
   Two precisions: real_t=float (the reference as shipped, SphBase.h:40) and
   real_t=double (the typedef switch the reference itself describes,
   SphBase.h:37-39) -> suffix _f64.  A third DFSPH variant,
   libref_dfsph_capped.so, changes only the loops' bookkeeping (double density
   sum, iteration caps of 100, the divergence goal in relative form) so that
   large scenes terminate under the same goals as the GPU run; see DF_CAP.
   Flags: -O3 -fopenmp, no -march (x86-64 SSE2, so no FMA contraction), which
   is what the parity statements assume.

Nothing is written outside oracle/_ref/.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's Source/ directory: the first argument, else $SPH_REFERENCE_SOURCE
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPH_REFERENCE_SOURCE", "")
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")
SHIM = os.path.join(HERE, "refshim")

FILES = ["SphBase.h", "SphBase.cpp", "Vec23.h", "DFSPH.h", "DFSPH.cpp", "WcSph.h",
         "WcSph.cpp", "PciSph.h", "PciSph.cpp", "IISph_M.h", "IISph_M.cpp", "IISph.h", "IISph.cpp",
         "surface_field.h", "surface_field.cpp", "marching_cubes.h", "marching_cubes.cpp"]

# (anchor line in SphBase.h, text inserted after it).  The anchors are the last
# member of FluidParticle (SphBase.h:117), of BoundaryParticle (SphBase.h:198)
# and of ThresholdsBase (SphBase.h:582).
AUGMENT = [
    ("    real_t VF_divergenceDeviation;\n\n    std::vector<real_t> MT_restVolumeFraction;",
     "    real_t density, density_adv, DFalpha, DFalpha2, DFkappa, DFkappaV, divergenceDeviation;\n"
     "    vec_t DFalpha1, vel_adv, acce_adv, angular_velocity, omega, vorticity, vortical_angular_velocity,\n"
     "        laplacian_angular_velocity, psi, n0Vorticity, n1Vorticity, deltaVorticity, dOmega;\n",
     "before"),
    ("    real_t DF_divergenceDeviation;\n};\n\n//see 9",
     "    vec_t singleVelocity, angular_velocity;\n", "before_close"),
    ("        real_t sum_energy;\n    } m_TH;",
     "        int enable_vortex = 0; real_t nu = 0, nu_t = 0, zeta = 0, alpha = 0;\n", "after_first_line"),
    # the oracle harness class reads private members (mg_NS, ker_* and
    # ker_update_numbers, SphBase.h:680-800)
    ("class SphBase{\n\npublic:\n", "    friend class RefHarness;\n", "after_anchor"),
    # the test harness's updateSolids stand-in (refshim/SphWithIO.h) moves a
    # dynamic solid with SphSolid::updatePaticles(com, transform, v, w), a
    # protected member (SphBase.h:344-346)
    ("class SphSolid : public SphObject  {\npublic:\n", "    friend class SphWithIO;\n", "after_anchor"),
    # the precision switch the reference describes at SphBase.h:37-40
    ("typedef float real_t;\n",
     "#ifdef REF_REAL_DOUBLE\ntypedef double real_t;\n#else\n", "wrap_typedef"),
]

# Vec23.h's mat33(const vec3&, vec3&, vec3&) binds temporaries to non-const
# references (an MSVC extension) where surface_field.cpp scales a matrix
# (Vec23.h:399, 444); the copy takes const references.
VEC_FIX = [
    ("inline mat33( const vec3<_T>& a, vec3<_T>& b, vec3<_T>& c ): U(a), V(b), W(c) { }",
     "inline mat33( const vec3<_T>& a, const vec3<_T>& b, const vec3<_T>& c ): U(a), V(b), W(c) { }"),
]

# DFSPH.cpp's density loop (DFSPH.cpp:225-231, 566, 627-631, 696) sums the
# density in float and has no iteration cap.  The "capped" build changes that
# bookkeeping only: the sum becomes double and the loop stops after
# REF_DF_MAXITER iterations.  Used for CPU-baseline timing of large scenes.
DF_CAP = [
    # divergence goal (DFSPH.cpp:762): absolute 2.5 -> the relative definition
    # mean(Drho/Dt) * dt / rho0 <= REF_DIV_REL, as the GPU configuration uses
    ("\t\treal_t errorRateGoal = 2.5;\n",
     "\t\treal_t errorRateGoal = real_t(REF_DIV_REL * rho0 / m_TH.dt);\n"),
    ("\t\tint maximumIteration = 30;\n\t\tint minimumIteration = 1;",
     "\t\tint maximumIteration = REF_DIV_MAXITER;\n\t\tint minimumIteration = 1;"),
    ("\t\treal_t densitySum = 0;\n\t\tint maximumIteration = 50;",
     "\t\tdouble densitySum = 0;\n\t\tint maximumIteration = 50;"),
    ("\t\twhile (errorRate > errorRateGoal || currentIteration < minimumIteration)\n",
     "\t\twhile ((errorRate > errorRateGoal || currentIteration < minimumIteration) && currentIteration < REF_DF_MAXITER)\n"),
    # iteration counts of both loops, summed for the harness to read
    # (ref_df_iters); inserted on the loops' closing lines, so line numbers
    # stay those of DFSPH.cpp
    ("\t\t} //end of iteration\n",
     "\t\t} { extern int ref_df_iter_count[2]; ref_df_iter_count[0] += currentIteration; } //end of iteration\n"),
    ("\t\t} // end of the iteration\n\n\t\t/* loop particle 4 */",
     "\t\t} { extern int ref_df_iter_count[2]; ref_df_iter_count[1] += currentIteration; } // end of the iteration"
     "\n\n\t\t/* loop particle 4 */"),
]

SOLVERS = {
    "dfsph": ("DFSPH.cpp", "DFSPH.h", "DFSPH", []),
    "dfsph_capped": ("DFSPH_capped.cpp", "DFSPH.h", "DFSPH", ["-DREF_DF_MAXITER=100", "-DREF_DIV_REL=1e-3",
                                                         "-DREF_DIV_MAXITER=100"]),
    "wcsph": ("WcSph.cpp", "WcSph.h", "WcSph", []),
    "pcisph": ("PciSph.cpp", "PciSph.h", "PciSph", ["-DPREDICTION_PCISPH"]),
    "iisphm": ("IISph_M.cpp", "IISph_M.h", "IISph_M", ["-DIISPH"]),
    "iisph": ("IISph.cpp", "IISph.h", "IISph", ["-DIISPH"]),
}


def transcode(name):
    raw = open(os.path.join(REF, name), "rb").read()
    if raw[:2] in (b"\xff\xfe", b"\xfe\xff"):
        text = raw.decode("utf-16")
    else:
        try:
            text = raw.decode("utf-8")
        except UnicodeDecodeError:
            text = raw.decode("gbk", errors="replace")
    return text.replace("\r\n", "\n")


def augment(text):
    for anchor, ins, mode in AUGMENT:
        pos = text.find(anchor)
        if pos < 0:
            raise SystemExit("anchor not found in SphBase.h: %r" % anchor[:40])
        if mode == "before":
            cut = pos + anchor.index("\n\n") + 1
        elif mode == "before_close":
            cut = pos + anchor.index("};")
        elif mode == "after_anchor":
            cut = pos + len(anchor)
        elif mode == "wrap_typedef":
            text = text[:pos] + ins + anchor + "#endif\n" + text[pos + len(anchor):]
            continue
        else:
            cut = pos + anchor.index("\n") + 1
        text = text[:cut] + ins + text[cut:]
    return text


def write_if_changed(dst, t):
    if not os.path.exists(dst) or open(dst).read() != t:
        open(dst, "w").write(t)


def main():
    if not REF or not os.path.isdir(REF):
        print("reference sources not given or not present (%r); keeping prebuilt oracle/_ref" % REF)
        return 0
    os.makedirs(SRC, exist_ok=True)
    for f in FILES:
        t = transcode(f)
        if f == "SphBase.h":
            t = augment(t)
        if f == "Vec23.h":
            for a, b in VEC_FIX:
                if a not in t:
                    raise SystemExit("Vec23.h anchor not found: %r" % a[:40])
                t = t.replace(a, b, 1)
        write_if_changed(os.path.join(SRC, f), t)
        if f == "DFSPH.cpp":
            for old, new in DF_CAP:
                if old not in t:
                    raise SystemExit("DFSPH.cpp anchor not found: %r" % old[:40])
                t = t.replace(old, new, 1)
            write_if_changed(os.path.join(SRC, "DFSPH_capped.cpp"), t)
    jobs = []
    for tag, (cpp, hdr, cls, defs) in SOLVERS.items():
        for real, suffix in (("float", ""), ("double", "_f64")):
            so = os.path.join(OUT, "libref_%s%s.so" % (tag, suffix))
            deps = [os.path.join(SRC, cpp), os.path.join(SRC, "SphBase.cpp"),
                    os.path.join(SHIM, "ref_harness.cpp"), os.path.join(SHIM, "SphWithIO.h"),
                    os.path.join(SRC, "SphBase.h")]
            if os.path.exists(so) and all(os.path.getmtime(so) >= os.path.getmtime(d) for d in deps):
                continue
            cmd = ["g++", "-std=c++17", "-O3", "-fopenmp", "-fPIC", "-shared", "-w",
                   
                   "-DREF_SOLVER_HEADER=\"%s\"" % hdr, "-DREF_SOLVER_CLASS=" + cls,
                   "-DREF_TAG_" + tag, "-I" + SRC, "-I" + SHIM] + defs + [
                   os.path.join(SRC, "SphBase.cpp"), os.path.join(SRC, cpp),
                   os.path.join(SHIM, "ref_harness.cpp"), "-o", so]
            if real == "double":
                cmd.insert(1, "-DREF_REAL_DOUBLE")
            jobs.append((so, cmd))
    # surface reconstruction: surface_field.cpp (TNT / JAMA replaced by the
    # stand-in refshim/jama_svd.h) and marching_cubes.cpp, which declares its
    # tables extern and defines them static (-fpermissive) and calls memcpy
    # without including <cstring>
    for real, suffix in (("float", ""),):
        so = os.path.join(OUT, "libref_surface%s.so" % suffix)
        srcs = [os.path.join(SRC, "surface_field.cpp"), os.path.join(SRC, "marching_cubes.cpp"),
                os.path.join(SHIM, "surface_harness.cpp")]
        deps = srcs + [os.path.join(SRC, "SphBase.h"), os.path.join(SHIM, "jama_svd.h")]
        if not (os.path.exists(so) and all(os.path.getmtime(so) >= os.path.getmtime(d) for d in deps)):
            jobs.append((so, ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-w", "-fpermissive", "-fopenmp",
                              "-include", "cstring", "-I" + SHIM, "-I" + SRC] + srcs + ["-o", so]))
    # the C++ drop-in checks: scene classes derived from each of the
    # reference's solver classes, switched to the GPU through
    # include/sphgpu_solver.hpp (links libsphgpu.so)
    lib = os.path.join(ROOT, "graphics_b200", "libsphgpu.so")
    for tag, cls, cpp, defs in (("dfsph", "DFSPH", "DFSPH.cpp", []), ("iisph", "IISph", "IISph.cpp", ["-DIISPH"]),
                                ("wcsph", "WcSph", "WcSph.cpp", []),
                                ("pcisph", "PciSph", "PciSph.cpp", ["-DPREDICTION_PCISPH"]),
                                ("iisph_m", "IISph_M", "IISph_M.cpp", ["-DIISPH"])):
        if not os.path.exists(lib):
            break
        exe = os.path.join(OUT, "dropin_" + tag)
        deps = [os.path.join(SHIM, "dropin_main.cpp"), os.path.join(ROOT, "include", "sphgpu_solver.hpp"),
                os.path.join(ROOT, "include", "sphgpu.h"), os.path.join(SRC, cpp),
                os.path.join(SRC, "SphBase.cpp"), os.path.join(SRC, "SphBase.h"), os.path.join(SHIM, "SphWithIO.h"),
                lib]
        if not (os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(d) for d in deps)):
            jobs.append((exe, ["g++", "-std=c++17", "-O2", "-fopenmp", "-w", "-DREF_SOLVER_HEADER=\"%s.h\"" % cls,
                               "-DREF_SOLVER_CLASS=" + cls, "-DREF_SPHGPU_SOLVER=SPHGPU_" + tag.upper(),
                               "-I" + SRC, "-I" + SHIM, "-I" + os.path.join(ROOT, "include")] + defs +
                         [os.path.join(SHIM, "dropin_main.cpp"), os.path.join(SRC, "SphBase.cpp"),
                          os.path.join(SRC, cpp), "-L" + os.path.dirname(lib), "-lsphgpu",
                          "-Wl,-rpath,$ORIGIN/../../graphics_b200", "-o", exe]))
    procs = [(so, subprocess.Popen(cmd, stderr=subprocess.PIPE)) for so, cmd in jobs]
    rc = 0
    for so, p in procs:
        _, err = p.communicate()
        if p.returncode:
            sys.stderr.write(err.decode()[-4000:])
            rc = 1
        else:
            print("built", os.path.relpath(so, HERE))
    return rc


if __name__ == "__main__":
    sys.exit(main())
