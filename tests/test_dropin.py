"""The drop-in, compiled for real: the reference's own driver (main.c,
init.balsara1.c, diag.c, restart.c, ...) with the USE_GPU_STEP hooks of
coolharm3d_b200/dropin (apply_patch.py + hg_driver.c) linked against
libharmgpu.so, against the same sources built without the hooks.

Sources: the reference tree staged by oracle/build_ref.py in
oracle/_ref/balsara1/src (Balsara test 1, MC + HLLE, CFL 0.5), with one
test-only edit applied to both builds: the final time 0.4 -> 0.015 (52 steps
on 1024 zones) so the CPU build finishes in seconds.  Both programs run the
whole driver loop; the GPU program's restart files (restart_write(), the
ASCII rdump the driver writes every n_restart steps and at the end) must be
byte for byte the CPU program's, and its energy file (dump_ener every 10
steps: U and boundary-flux integrals summed on the device, M_tot from the
device) must agree to 1e-12 (the sums' order differs)."""
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

import harmtest as ht

REPO = ht.REPO
STAGED = REPO / "oracle" / "_ref" / "balsara1" / "src"
LIBDIR = REPO / "coolharm3d_b200"
sys.path.insert(0, str(REPO / "coolharm3d_b200" / "dropin"))
sys.path.insert(0, str(REPO / "oracle"))

pytestmark = pytest.mark.skipif(not STAGED.is_dir(), reason="reference sources not staged (oracle/build_ref.py)")

CFLAGS = ["-O3", "-fcommon", "-ffp-contract=off", "-w"]
N = (1024, 1, 1)


def build_pair(work):
    """(cpu_exe, gpu_exe) built from one patched copy of the staged sources."""
    import apply_patch
    import build_ref
    src = os.path.join(work, "src")
    shutil.copytree(STAGED, src)
    init = os.path.join(src, "init.balsara1.c")
    text = open(init).read()
    assert "GridLength[0] = 0.4 ;" in text
    open(init, "w").write(text.replace("GridLength[0] = 0.4 ;", "GridLength[0] = 0.015 ;", 1))
    apply_patch.apply(src)
    common = [s for s in build_ref.BASE_SRCS + ["init.balsara1.c"] if s not in ("main.c", "step_ch.c", "diag.c")]
    jobs = []
    for s in common:
        jobs.append((os.path.join(src, s), os.path.join(work, "o_" + s[:-2] + ".o"), []))
    for variant, extra in (("cpu", []), ("gpu", ["-DUSE_GPU_STEP=1", "-I", str(REPO / "include")])):
        for s in ("main.c", "step_ch.c", "diag.c", "hg_driver.c"):
            jobs.append((os.path.join(src, s), os.path.join(work, "%s_%s.o" % (variant, s[:-2])), extra))
    procs = [subprocess.Popen(["gcc"] + CFLAGS + ["-I", src] + extra + ["-c", s, "-o", o]) for s, o, extra in jobs]
    assert all(p.wait() == 0 for p in procs)
    objs_common = [o for s, o, e in jobs[:len(common)]]
    exes = []
    for variant in ("cpu", "gpu"):
        exe = os.path.join(work, "harm3d_" + variant)
        objs = objs_common + [os.path.join(work, "%s_%s.o" % (variant, s))
                              for s in ("main", "step_ch", "diag", "hg_driver")]
        libs = ["-lm"] if variant == "cpu" else ["-L", str(LIBDIR), "-lharmgpu", "-Wl,-rpath," + str(LIBDIR), "-lm"]
        subprocess.check_call(["gcc", "-o", exe] + objs + libs)
        exes.append(exe)
    return exes


def run(exe, cwd):
    os.makedirs(cwd)
    r = subprocess.run([exe, "1", "1", "1"] + [str(x) for x in N], cwd=cwd, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def test_patched_driver_compiles_and_links():
    """Both programs build from the patched sources (no GPU needed to link)."""
    with tempfile.TemporaryDirectory() as td:
        cpu, gpu = build_pair(td)
        assert os.path.exists(cpu) and os.path.exists(gpu)


@pytest.mark.gpu
def test_patched_driver_reproduces_cpu_run():
    with tempfile.TemporaryDirectory() as td:
        cpu, gpu = build_pair(td)
        out_c = run(cpu, os.path.join(td, "run_cpu"))
        out_g = run(gpu, os.path.join(td, "run_gpu"))
        rc, rg = Path(td, "run_cpu"), Path(td, "run_gpu")
        dumps = sorted(p.name for p in rc.glob("rdump*"))
        assert dumps and dumps == sorted(p.name for p in rg.glob("rdump*"))
        for name in dumps:
            assert (rc / name).read_bytes() == (rg / name).read_bytes(), name
        # the driver's step count and zone-cycles line (main.c:117)
        ns = [line for line in out_c.splitlines() if line.startswith("ns,ts")]
        assert ns and ns == [line for line in out_g.splitlines() if line.startswith("ns,ts")]
        ec = np.loadtxt(rc / "KDHARM0_ener.out")
        eg = np.loadtxt(rg / "KDHARM0_ener.out")
        assert ec.shape == eg.shape
        np.testing.assert_allclose(eg, ec, rtol=1e-12, atol=1e-15 * np.abs(ec).max())
