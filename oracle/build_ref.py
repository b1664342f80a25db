#!/usr/bin/env python3
"""Recipe that compiles the HARM3D reference's own CPU step into oracle/_ref/.

This is test infrastructure: it produces the reference executables that pin
the C oracle (oracle/harm_oracle.c) and the golden fixtures under
tests/golden/.  Nothing in the product (coolharm3d_b200/) links or runs them.

What it does, per configuration:
  1. stages the reference's src/ files into oracle/_ref/<cfg>/src/
     (a git-ignored build folder; reference sources are never committed),
  2. applies the documented compile-time switch edits to the staged
     options.h (each edit is listed in CONFIGS below),
     and the documented parameter edits to the staged init.<setup>.c,
  3. regenerates defs.h from globals.h exactly as the reference makefile
     does (src/makefile, the `egrep "^extern|^#if..." globals.h | sed` rule),
  4. compiles every source of src/makefile:364-373 except corona*.c, plus
     oracle/ref_probe.c (our harness hook), with
       gcc -O3 -fcommon -ffp-contract=off
     step_ch.c is compiled with -Dstep_ch=ref_step_ch so that the reference's
     own main() loop calls the probe's step_ch(), which wraps the real one,
     dumps state and optionally loads an initial state (see ref_probe.c).

Usage:  python oracle/build_ref.py [cfg ...]   (default: all configs)
The reference tree is read from $HARM_REF_SRC, else from a checkout named
`reference` beside this repository (<repo>/../reference/src).
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REPO = os.path.dirname(HERE)
REF_SRC = os.environ.get("HARM_REF_SRC") or os.path.join(os.path.dirname(REPO), "reference", "src")

# src/makefile:364-373, minus corona.c corona2.c (cooling choices 4/5 only)
# and minus the init file (one init.*.c is linked per configuration).
BASE_SRCS = [
    "bounds.c", "coord.c", "diag.c", "dump.c", "fixup.c", "flux_ct.c", "image.c",
    "lu.c", "main.c", "metric.c", "phys.c", "ranc.c", "restart.c", "recon.c",
    "step_ch.c", "u2p_util.c", "utoprim_1d_ee.c", "utoprim_1d_ee2.c",
    "utoprim_1dfix1.c", "utoprim_1dvsq2fix1.c", "utoprim_1d.c",
    "utoprim_2d_fast.c", "harm_mpi.c", "dump_hdf.c", "dump_history.c",
    "dump_stat.c", "dump_stat2.c", "dump_radflux.c", "dump_surface.c",
    "dump_timers.c", "decomp.c", "dump_photosphere.c", "interp_data.c",
]

# Output-only switches turned off in every configuration (no HDF5 in the image).
IO_OFF = {
    "MAKE_HISTORY": "0", "MAKE_HDF5": "0", "MAKE_STAT": "0", "MAKE_RADFLUX": "0",
    "MAKE_PHOTOSPHERE": "0", "MAKE_ASCII": "0", "MAKE_IMAGE": "0",
}

MINK = {
    "METRIC_TYPE_CHOICE": "(METRIC_MINK_CARTESIAN)",
    "COORD_TYPE_CHOICE": "(COORD_IDENTITY)",
    "USE_COOLING_FUNCTION": "(0)",
    "RESCALE_R": "(0)",
}

# name -> (init file, options.h edits, literal edits to the init file; an edit
# given as (file, old, new) applies to another staged source file)
CONFIGS = {
    # Balsara test 1, 1D shock tube: MC + HLLE + para flux-CT, outflow.
    "balsara1": ("init.balsara1.c",
                 dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_OUTFLOW)",
                      RECON_TYPE_CHOICE="(RECON_MC)", FLUX_TYPE_CHOICE="(FLUX_HLLE)"),
                 [("cour = 0.8 ;", "cour = 0.5 ;")]),
    # Same physics with the shipped Courant number, LF flux and minmod slopes,
    # plain Toth flux-CT: exercises the alternative switches of the step.
    "balsara1_lf": ("init.balsara1.c",
                    dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_OUTFLOW)",
                         RECON_TYPE_CHOICE="(RECON_MINMOD)", FLUX_TYPE_CHOICE="(FLUX_LF)",
                         USE_FLUX_CT_PARA="(0)"),
                    []),
    # Periodic linear wave (the reference's 2D slow mode): PPM_MC + HLLE.
    "linwave": ("init.linearwave.c",
                dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_PERIODIC)",
                     RECON_TYPE_CHOICE="(RECON_PPM_MC)", FLUX_TYPE_CHOICE="(FLUX_HLLE)"),
                []),
    # Entropy-equation fix off: the inversion tree without pow(), so every
    # branch of it can be compared bit for bit with a GPU build.
    "balsara1_noee": ("init.balsara1.c",
                      dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_OUTFLOW)", RECON_TYPE_CHOICE="(RECON_MC)",
                           FLUX_TYPE_CHOICE="(FLUX_HLLE)", USE_ENTROPY_EQ="(0)"),
                      [("cour = 0.8 ;", "cour = 0.5 ;")]),
    "linwave_noee": ("init.linearwave.c",
                     dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_PERIODIC)", RECON_TYPE_CHOICE="(RECON_PPM_MC)",
                          FLUX_TYPE_CHOICE="(FLUX_HLLE)", USE_ENTROPY_EQ="(0)"),
                     []),
    # Fishbone-Moncrief torus in Kerr-Schild a=0.9, modified KS (DIAGONAL3)
    # coordinates, SPHERICAL_OUTFLOW3, PPM_MC + HLLE, para flux-CT, RESCALE_R,
    # entropy fix, H/R = 0.1 cooling: the configuration's parameters replace
    # the shipped ones (a 0 -> 0.9, Rout 40 -> 120, phi range pi/2 -> 2 pi,
    # Gamma 4/3 -> 5/3, r_in 10 -> 6, r_pmax 16 -> 12, randfact 0 -> 0.04,
    # USE_COOLING_FUNCTION 5 -> 1, FLUX_LF -> FLUX_HLLE, h_o_r 0.05 -> 0.1),
    # and the stray ';' after init_prim's header (init.torus.c:355) is removed.
    "torus": ("init.torus.c",
              dict(USE_COOLING_FUNCTION="(1)", FLUX_TYPE_CHOICE="(FLUX_HLLE)"),
              [("gam = (4./3.) ;", "gam = (5./3.) ;"),
               ("GridLength[3] = M_PI/2. ;", "GridLength[3] = 2.*M_PI ;"),
               ("  a = 0.;          /* Spin", "  a = 0.9;          /* Spin"),
               ("Rout     = 40.;", "Rout     = 120.;"),
               ("struct of_coord *coords, double *pr);\n{", "struct of_coord *coords, double *pr)\n{"),
               ("rin = 10. ;", "rin = 6. ;"),
               ("rmax = 16. ;", "rmax = 12. ;"),
               ("  randfact = 0.;", "  randfact = 4.e-2;"),
               ("phys.c", "const double h_o_r  = 5.e-2;", "const double h_o_r  = 1.e-1;")]),
    # The torus configuration on the reference's general time-dependent metric
    # path (METRIC_GENERAL_DYNAMIC: geometry at three time levels, METRIC_DIM
    # 3 tables, connection rebuilt every substep by 4th-order differences of
    # gcov plus a time derivative; metric.c:3390-3648, conn.h) with its
    # Minkowski-spherical test spacetime (METRIC_DYNAMIC_MINK_SPHERICAL,
    # options.h:90).  SET_TSHRINK 1: main.c:505-508 refuses to compile the
    # dynamic path without it for every spacetime but the PN ones.
    "torus_dynmink": ("init.torus.c",
                      dict(USE_COOLING_FUNCTION="(1)", FLUX_TYPE_CHOICE="(FLUX_HLLE)",
                           METRIC_TYPE_CHOICE="(METRIC_GENERAL_DYNAMIC)",
                           METRIC_DYNAMIC_TYPE_CHOICE="(METRIC_DYNAMIC_MINK_SPHERICAL)", SET_TSHRINK="(1)"),
                      None),
    # The same torus on the dynamic path with the reference's Kerr-Schild test
    # spacetime (METRIC_DYNAMIC_KS_SPHERICAL, options.h:88): geometry of
    # the three time levels from ks_gcov/gcon/gdet_func, the static analytic
    # connection in place of the finite differences (metric.c:3555-3558).
    "torus_dynks": ("init.torus.c",
                    dict(USE_COOLING_FUNCTION="(1)", FLUX_TYPE_CHOICE="(FLUX_HLLE)",
                         METRIC_TYPE_CHOICE="(METRIC_GENERAL_DYNAMIC)",
                         METRIC_DYNAMIC_TYPE_CHOICE="(METRIC_DYNAMIC_KS_SPHERICAL)", SET_TSHRINK="(1)"),
                    None),
    # The circumbinary-disk setup of the post-Newtonian binary runs
    # (init.nz_pn_bbh_disk.c: De Villiers-Hawley-Krolik disk with q = 1.58
    # around the binary's total mass M = 1 at separation 20M, inner edge 2(a+M),
    # pressure maximum 5(a+M), 1% perturbation of u from ranc() seeded with 1,
    # dipole loop following the density) on the dynamic-metric path.  The PN
    # spacetime bodies are absent from the reference (metric.h:105-171), so
    # the reference's own Minkowski-spherical test spacetime stands in for it.
    # Parameters of the configuration: r over [0.75a, 13a] (Rin 0.05a -> 0.75a,
    # Rout 100a -> 13a), plasma beta 100 -> 10, H/R = 0.1 cooling (h_o_r 0.05
    # -> 0.1).  The shipped file does not compile against this source tree;
    # the four compile fixes, each the evident intent: the two diagnostic
    # arrays sized by N1TOT at file scope (a run-time size here) get a fixed
    # size, the local prototype of init_prim() takes the struct of_coord * of
    # its definition, the diagnostic `rdiskout = x[RR]` reads coords->x[RR],
    # and get_rpmax()'s coords_loc is the struct of_coord that coord_of_r()
    # fills (it was declared struct of_geom).  One behavioural fix: init_prim()
    # moves the stored coordinate coords->x[RR] of each zone to the BL radius
    # in place and moves it back only inside the disk (:494-507), so outside
    # the disk the grid's coordinate arrays stay shifted by M; the reference's
    # run then evaluates its metric there at r + M from the second step on
    # (advance_geometry -> set_general_geometry reads get_coord,
    # metric.c:398-430, 3390-3422) and builds its RESCALE_R and cooling
    # tables from the shifted row (recon.c:1142-1165, phys.c:683-704).  The
    # staged copy saves the coordinate and puts it back in both branches
    # (exactly: (r + M) - M is not always r).
    "pnbbh_dynmink": ("init.nz_pn_bbh_disk.c",
                      dict(USE_COOLING_FUNCTION="(1)", FLUX_TYPE_CHOICE="(FLUX_HLLE)",
                           METRIC_TYPE_CHOICE="(METRIC_GENERAL_DYNAMIC)",
                           METRIC_DYNAMIC_TYPE_CHOICE="(METRIC_DYNAMIC_MINK_SPHERICAL)", SET_TSHRINK="(1)"),
                      [("double height_denom[N1TOT] = {0.};", "double height_denom[4096] = {0.};"),
                       ("double height_numer[N1TOT] = {0.};", "double height_numer[4096] = {0.};"),
                       ("  void init_prim( int i, int j, int k, double *xp, double *pr);",
                        "  void init_prim( int i, int j, int k, struct of_coord *coords, double *pr);"),
                       ("{ rdiskout = x[RR]; }", "{ rdiskout = coords->x[RR]; }"),
                       ("  struct of_geom coords_loc;", "  struct of_coord coords_loc;"),
                       ("Rout     = 100.*initial_bbh_separation;", "Rout     = 13.*initial_bbh_separation;"),
                       ("Rin = 0.05 * (initial_bbh_separation) ;", "Rin = 0.75 * (initial_bbh_separation) ;"),
                       ("beta     = 1.e2 ;", "beta     = 10. ;"),
                       ("  coords->x[RR] += m_bh_tot;  /* Transform to BL coordinates */",
                        "  const double x_rr_grid = coords->x[RR];\n  coords->x[RR] += m_bh_tot;"),
                       ("    coords->x[RR] -= m_bh_tot;  /* Transform back from BL coordinates */",
                        "    coords->x[RR] = x_rr_grid;"),
                       ("  else { \n    PLOOP pr[l] = 0.;\n  }",
                        "  else { \n    PLOOP pr[l] = 0.;\n    coords->x[RR] = x_rr_grid;\n  }"),
                       ("phys.c", "const double h_o_r  = 5.e-2;", "const double h_o_r  = 1.e-1;")]),
    # Advected field loop (Gardiner & Stone 2005), 2D periodic Minkowski:
    # PPM_MC + HLLE + para flux-CT, the shipped parameters.  The setup calls
    # the time-dependent-coordinate macro SET_GEOM_COORD_TIME_FUNCS without
    # including metric.h, where it is defined, so it does not link; the call
    # (a no-op for the static Minkowski grid) is removed.
    "field_loop": ("init.field_loop.c",
                   dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_PERIODIC)",
                        RECON_TYPE_CHOICE="(RECON_PPM_MC)", FLUX_TYPE_CHOICE="(FLUX_HLLE)"),
                   [("SET_GEOM_COORD_TIME_FUNCS(t,1);", "")]),
    # Same setup with van Leer PPM limiter and LF flux.
    "linwave_vl": ("init.linearwave.c",
                   dict(MINK, BC_TYPE_CHOICE="(BC_CARTESIAN_PERIODIC)",
                        RECON_TYPE_CHOICE="(RECON_PPM_VL)", FLUX_TYPE_CHOICE="(FLUX_LF)"),
                   []),
}


# the dynamic-metric tori take the torus configuration's edits of init.torus.c and phys.c
CONFIGS["torus_dynmink"] = CONFIGS["torus_dynmink"][:2] + (CONFIGS["torus"][2],)
CONFIGS["torus_dynks"] = CONFIGS["torus_dynks"][:2] + (CONFIGS["torus"][2],)


def set_define(text, name, value):
    pat = re.compile(r"^(#define\s+%s\s+)(.*)$" % re.escape(name), re.M)
    if not pat.search(text):
        raise SystemExit("build_ref: no '#define %s' in options.h" % name)
    return pat.sub(lambda m: m.group(1) + value, text, count=1)


def stage(cfg):
    init_file, opts, init_edits = CONFIGS[cfg]
    bdir = os.path.join(OUT, cfg)
    sdir = os.path.join(bdir, "src")
    if os.path.isdir(sdir):
        shutil.rmtree(sdir)
    os.makedirs(sdir)
    for f in os.listdir(REF_SRC):
        if f.endswith((".c", ".h")):
            shutil.copy(os.path.join(REF_SRC, f), sdir)
    opt_path = os.path.join(sdir, "options.h")
    text = open(opt_path).read()
    for k, v in dict(IO_OFF, **opts).items():
        text = set_define(text, k, v)
    open(opt_path, "w").write(text)
    for e in init_edits:
        fname, old, new = (init_file,) + tuple(e) if len(e) == 2 else e
        fpath = os.path.join(sdir, fname)
        text = open(fpath).read()
        if old not in text:
            raise SystemExit("build_ref: edit target %r not in %s" % (old, fname))
        open(fpath, "w").write(text.replace(old, new, 1))
    # defs.h: same transform as the reference makefile's defs.h rule.
    defs = []
    for line in open(os.path.join(sdir, "globals.h")):
        if re.match(r"^(extern|#if|#elif|#else|#endif)", line):
            defs.append(re.sub(r"^extern", "", line, count=1))
    open(os.path.join(sdir, "defs.h"), "w").write("".join(defs))
    return bdir, sdir, init_file


def build(cfg, jobs=8):
    bdir, sdir, init_file = stage(cfg)
    odir = os.path.join(bdir, "obj")
    os.makedirs(odir, exist_ok=True)
    cflags = ["-O3", "-fcommon", "-ffp-contract=off", "-w", "-I", sdir]
    srcs = [os.path.join(sdir, s) for s in BASE_SRCS + [init_file]]
    srcs.append(os.path.join(HERE, "ref_probe.c"))
    procs, objs = [], []
    for s in srcs:
        o = os.path.join(odir, os.path.basename(s)[:-2] + ".o")
        extra = ["-Dstep_ch=ref_step_ch"] if os.path.basename(s) == "step_ch.c" else []
        objs.append(o)
        procs.append(subprocess.Popen(["gcc"] + cflags + extra + ["-c", s, "-o", o]))
        if len(procs) >= jobs:
            if procs.pop(0).wait() != 0:
                raise SystemExit("build_ref: compile failed for " + cfg)
    for p in procs:
        if p.wait() != 0:
            raise SystemExit("build_ref: compile failed for " + cfg)
    exe = os.path.join(bdir, "harm3d")
    subprocess.check_call(["gcc", "-o", exe] + objs + ["-lm"])
    return exe


NATIVE_FLAGS = ["-O3", "-march=native", "-fcommon", "-w"]


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def build_native(cfg, jobs=None):
    """The reference's own build for timing on this machine: the sources staged
    in oracle/_ref/<cfg>/src (by build()) compiled with the flags its users
    would use, gcc -O3 -march=native -fcommon, plus the probe, into
    oracle/_ref/<cfg>/harm3d_native; a stamp records the CPU it was built for.
    Needs no reference checkout: the staged sources travel with oracle/_ref.
    Returns the executable, rebuilt only when the CPU differs."""
    bdir = os.path.join(OUT, cfg)
    sdir = os.path.join(bdir, "src")
    exe = os.path.join(bdir, "harm3d_native")
    stamp = exe + ".cpu"
    model = cpu_model()
    if os.path.exists(exe) and os.path.exists(stamp) and open(stamp).read() == model:
        return exe
    if not os.path.isdir(sdir):
        raise RuntimeError("no staged reference sources in %s (run oracle/build_ref.py where the reference is)" % sdir)
    init_file = CONFIGS[cfg][0]
    odir = os.path.join(bdir, "obj_native")
    os.makedirs(odir, exist_ok=True)
    srcs = [os.path.join(sdir, x) for x in BASE_SRCS + [init_file]] + [os.path.join(HERE, "ref_probe.c")]
    jobs = jobs or max(1, os.cpu_count() or 1)
    procs, objs = [], []
    for src in srcs:
        o = os.path.join(odir, os.path.basename(src)[:-2] + ".o")
        extra = ["-Dstep_ch=ref_step_ch"] if os.path.basename(src) == "step_ch.c" else []
        objs.append(o)
        procs.append(subprocess.Popen(["gcc"] + NATIVE_FLAGS + ["-I", sdir] + extra + ["-c", src, "-o", o]))
        if len(procs) >= jobs:
            if procs.pop(0).wait() != 0:
                raise RuntimeError("build_ref: native compile failed for " + cfg)
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("build_ref: native compile failed for " + cfg)
    subprocess.check_call(["gcc", "-o", exe + ".tmp"] + objs + ["-lm"])
    os.replace(exe + ".tmp", exe)
    with open(stamp, "w") as f:
        f.write(model)
    return exe


def main(argv):
    cfgs = argv or sorted(CONFIGS)
    if not os.path.isdir(REF_SRC):
        print("build_ref: reference sources not found at %s; skipping" % REF_SRC)
        return 0
    for c in cfgs:
        print("built", build(c))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
