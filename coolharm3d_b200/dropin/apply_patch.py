#!/usr/bin/env python3
"""Apply the USE_GPU_STEP hooks to a copy of the HARM3D reference's src/.

  python apply_patch.py <src-dir>

Adds hg_driver.c (the driver's side of libharmgpu, beside this script) to
<src-dir> and inserts, each inside `#if USE_GPU_STEP`, five calls:
  step_ch.c  first statement of step_ch():      if (hg_gpu_step()) return;
  main.c     after global_init():               hg_gpu_init();
             after the loop's nstep++:          hg_gpu_sync_host(0);
             before the final restart_write():  hg_gpu_sync_host(1);
  diag.c     dump_ener(), after its flux totals
             are scaled:                         hg_gpu_totals(U_tot, F_tot);
(dump_ener integrates the last substep's conserved variables and boundary
fluxes, which stay on the device: the library sums them there.)
Built without -DUSE_GPU_STEP=1 the sources compile to the unchanged CPU
program.  Build with -DUSE_GPU_STEP=1 -I<repo>/include, add hg_driver.c to
the sources, and link -L<repo>/coolharm3d_b200 -lharmgpu
-Wl,-rpath,<repo>/coolharm3d_b200.  Raises if an anchor line is missing
(another version of the sources); applying twice is refused.
"""
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
MARK = "USE_GPU_STEP hook"


def _insert(text, pattern, block, before=False, last=False):
    """Insert `block` after (or before) the line matching `pattern`."""
    ms = list(re.finditer(pattern, text, re.M))
    if not ms:
        raise RuntimeError("anchor %r not found" % pattern)
    m = ms[-1] if last else ms[0]
    if before:
        pos = text.rfind("\n", 0, m.start()) + 1
    else:
        pos = text.find("\n", m.end()) + 1
    return text[:pos] + block + text[pos:]


def hook(indent, call):
    return "#if USE_GPU_STEP  /* %s */\n%s%s\n#endif\n" % (MARK, indent, call)


def apply(src):
    sc = os.path.join(src, "step_ch.c")
    mc = os.path.join(src, "main.c")
    dc = os.path.join(src, "diag.c")
    s, m, dg = open(sc).read(), open(mc).read(), open(dc).read()
    if MARK in s or MARK in m or MARK in dg:
        raise RuntimeError("already patched: " + src)
    # the first statement of step_ch(): after the line holding its opening brace
    i = s.index("void step_ch(void)")
    j = s.index("{", i)
    k = s.find("\n", j) + 1
    s = s[:k] + hook("  ", "{ extern int hg_gpu_step(void); if (hg_gpu_step()) return; }") + s[k:]
    m = _insert(m, r"^\s*global_init\(\)\s*;", hook("\t", "{ extern void hg_gpu_init(void); hg_gpu_init(); }"))
    m = _insert(m, r"^\s*nstep\+\+\s*;", hook("\t\t", "{ extern void hg_gpu_sync_host(int); hg_gpu_sync_host(0); }"))
    m = _insert(m, r"^\s*restart_write\(\)\s*;", hook("\t", "{ extern void hg_gpu_sync_host(int); hg_gpu_sync_host(1); }"),
                before=True, last=True)
    dg = _insert(dg, r"^\s*PLOOP\s+F_tot\[2\]\[BCUP\]\[l\]\s*\*=",
                 hook("  ", "{ extern void hg_gpu_totals(double *, double *); hg_gpu_totals(U_tot, &F_tot[0][0][0]); }"))
    open(sc, "w").write(s)
    open(mc, "w").write(m)
    open(dc, "w").write(dg)
    shutil.copy(os.path.join(HERE, "hg_driver.c"), os.path.join(src, "hg_driver.c"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    apply(sys.argv[1])
