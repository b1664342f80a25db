"""Shared test helpers: state/geometry file I/O, the reference runner and the
C-oracle wrapper.  Test infrastructure only (the product never imports it).

State files ("HGST") and geometry files ("HGGM") are written by
oracle/ref_probe.c; their layout is documented there.  Arrays use the
reference's own index order p[i][j][k][l] (l = primitive variable fastest).
"""
import ctypes
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
REF_DIR = REPO / "oracle" / "_ref"
ORACLE_SO = REPO / "oracle" / "liboracle.so"
NG, NP, NFAIL = 3, 8, 15

# Compile-time switches of each reference configuration (oracle/build_ref.py).
# recon: RECON_TYPE_CHOICE, flux: FLUX_TYPE_CHOICE, ct_para: USE_FLUX_CT_PARA,
# bc: BC_TYPE_CHOICE, metric_dim: METRIC_DIM, ee: USE_ENTROPY_EQ.
CONFIG_SWITCHES = {
    "balsara1": dict(recon=2, flux=1, ct_para=1, bc=0, metric_dim=0, ee=1, cooling=0, rescale=0),
    "balsara1_lf": dict(recon=0, flux=0, ct_para=0, bc=0, metric_dim=0, ee=1, cooling=0, rescale=0),
    "linwave": dict(recon=5, flux=1, ct_para=1, bc=1, metric_dim=0, ee=1, cooling=0, rescale=0),
    "linwave_vl": dict(recon=4, flux=0, ct_para=1, bc=1, metric_dim=0, ee=1, cooling=0, rescale=0),
    "balsara1_noee": dict(recon=2, flux=1, ct_para=1, bc=0, metric_dim=0, ee=0, cooling=0, rescale=0),
    "linwave_noee": dict(recon=5, flux=1, ct_para=1, bc=1, metric_dim=0, ee=0, cooling=0, rescale=0),
    "torus": dict(recon=5, flux=1, ct_para=1, bc=10, metric_dim=2, ee=1, cooling=1, rescale=1),
    "field_loop": dict(recon=5, flux=1, ct_para=1, bc=1, metric_dim=0, ee=1, cooling=0, rescale=0),
    "torus_dynmink": dict(recon=5, flux=1, ct_para=1, bc=10, metric_dim=3, ee=1, cooling=1, rescale=1),
    "pnbbh_dynmink": dict(recon=5, flux=1, ct_para=1, bc=10, metric_dim=3, ee=1, cooling=1, rescale=1),
    "torus_dynks": dict(recon=5, flux=1, ct_para=1, bc=10, metric_dim=3, ee=1, cooling=1, rescale=1),
}
CONFIG_HOR = 0.1  # h_o_r of the torus and disk builds' cooling function (both set to 0.1)

# COORD_DIAGONAL3 parameters of the dynamic-metric configurations'
# set_special_coord() (init.torus.c:245-270, init.nz_pn_bbh_disk.c:333-350)
CONFIG_DYN = {
    "torus_dynmink": dict(R0=0.0, h_slope=0.35, diag3_exponent=7),
    "pnbbh_dynmink": dict(R0=0.0, h_slope=0.0729419909586, diag3_exponent=9),
    "torus_dynks": dict(R0=0.0, h_slope=0.35, diag3_exponent=7, spacetime=0, spin=0.9),  # DYN_KS_SPHERICAL
}


def tot(n):
    return n + 2 * NG


def read_state(path):
    b = Path(path).read_bytes()
    assert b[:4] == b"HGST", path
    o = 4
    ver, n1, n2, n3, ng, np_ = np.frombuffer(b, np.int32, 6, o); o += 24
    t, dt, mtot = np.frombuffer(b, np.float64, 3, o); o += 24
    nstep = int(np.frombuffer(b, np.int32, 1, o)[0]); o += 4
    nfailtot = np.frombuffer(b, np.uint64, NFAIL, o).copy(); o += 8 * NFAIL
    shp = (tot(n1), tot(n2), tot(n3))
    ncell = shp[0] * shp[1] * shp[2]
    p = np.frombuffer(b, np.float64, ncell * NP, o).reshape(shp + (NP,)).copy(); o += 8 * ncell * NP
    out = dict(n=(int(n1), int(n2), int(n3)), t=float(t), dt=float(dt), m_tot=float(mtot), nstep=nstep,
               nfailtot=nfailtot, p=p)
    if len(b) > o:
        out["pflag"] = np.frombuffer(b, np.int32, ncell, o).reshape(shp).copy(); o += 4 * ncell
        out["gamma"] = np.frombuffer(b, np.float64, ncell, o).reshape(shp).copy(); o += 8 * ncell
        out["nfail"] = np.frombuffer(b, np.int32, ncell * NFAIL, o).reshape((NFAIL,) + shp).copy()
    return out


def write_state(path, p, t, dt, nstep=0):
    n = tuple(s - 2 * NG for s in p.shape[:3])
    with open(path, "wb") as f:
        f.write(b"HGST")
        f.write(np.array([1, n[0], n[1], n[2], NG, NP], np.int32).tobytes())
        f.write(np.array([t, dt, 0.0], np.float64).tobytes())
        f.write(np.array([nstep], np.int32).tobytes())
        f.write(np.zeros(NFAIL, np.uint64).tobytes())
        f.write(np.ascontiguousarray(p, np.float64).tobytes())


def read_geom(path, n):
    b = Path(path).read_bytes()
    assert b[:4] == b"HGGM", path
    prm = np.frombuffer(b, np.float64, 14, 4)
    o = 4 + 14 * 8
    ngeom, nconn = (int(x) for x in np.frombuffer(b, np.int32, 2, o)); o += 8
    geom = np.frombuffer(b, np.float64, ngeom * 42, o).reshape(ngeom, 42).copy(); o += ngeom * 42 * 8
    conn = np.frombuffer(b, np.float64, nconn * 64, o).reshape(nconn, 64).copy(); o += nconn * 64 * 8
    shp = (tot(n[0]), tot(n[1]), tot(n[2]))
    cell6 = np.frombuffer(b, np.float64, shp[0] * shp[1] * shp[2] * 6, o).reshape(shp + (6,)).copy()
    o += shp[0] * shp[1] * shp[2] * 6 * 8
    per_i = np.frombuffer(b, np.float64, shp[0] * 3, o).reshape(shp[0], 3).copy()
    return dict(gam=prm[0], cour=prm[1], grid_length=prm[2:6].copy(), startx=prm[6:10].copy(),
                dx=prm[10:14].copy(), geom=geom, conn=conn, cell6=cell6, rface=per_i[:, 0].copy(),
                cool_omega=per_i[:, 1].copy(), cool_temp=per_i[:, 2].copy())


def ref_exe(cfg):
    return REF_DIR / cfg / "harm3d"


def ref_available(cfg):
    return ref_exe(cfg).exists()


def run_ref(cfg, n, steps, load=None, dumps=(), want_geom=False, timeout=600):
    """Run the reference build `cfg` on an n1 x n2 x n3 grid for `steps` steps.

    Returns {"states": {step: state}, "geom": geom-or-None}.  Step 0 is the
    state handed to the first step (after init, or the loaded state)."""
    with tempfile.TemporaryDirectory() as td:
        env = dict(os.environ)
        env["HARM_PROBE_OUT"] = os.path.join(td, "st")
        env["HARM_PROBE_MAXSTEPS"] = str(steps)
        dl = sorted(set(dumps) | {steps})
        env["HARM_PROBE_DUMP"] = ",".join(str(x) for x in dl)
        if want_geom:
            env["HARM_PROBE_GEOM"] = os.path.join(td, "geom.bin")
            if CONFIG_SWITCHES[cfg]["cooling"]:
                env["HARM_PROBE_HOR"] = repr(CONFIG_HOR)
        if load is not None:
            lp = os.path.join(td, "load.bin")
            write_state(lp, load["p"], load["t"], load["dt"])
            env["HARM_PROBE_LOAD"] = lp
        r = subprocess.run([str(ref_exe(cfg)), "1", "1", "1"] + [str(x) for x in n], cwd=td, env=env,
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed: %s\n%s" % (r.returncode, r.stderr[-2000:]))
        states = {s: read_state(os.path.join(td, "st.%d.bin" % s)) for s in dl}
        geom = read_geom(os.path.join(td, "geom.bin"), n) if want_geom else None
    return dict(states=states, geom=geom)


def run_ref_final(cfg, n, load=None, want_geom=False, timeout=3600):
    """Run the reference build `cfg` until its own final time GridLength[0]
    (main.c:64) and return (state at t_final, geometry-or-None)."""
    with tempfile.TemporaryDirectory() as td:
        env = dict(os.environ)
        env["HARM_PROBE_OUT"] = os.path.join(td, "st")
        env["HARM_PROBE_FINAL"] = "1"
        env.pop("HARM_PROBE_MAXSTEPS", None)
        env.pop("HARM_PROBE_DUMP", None)
        if want_geom:
            env["HARM_PROBE_GEOM"] = os.path.join(td, "geom.bin")
        if load is not None:
            lp = os.path.join(td, "load.bin")
            write_state(lp, load["p"], load["t"], load["dt"])
            env["HARM_PROBE_LOAD"] = lp
        r = subprocess.run([str(ref_exe(cfg)), "1", "1", "1"] + [str(x) for x in n], cwd=td, env=env,
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed: %s\n%s" % (r.returncode, r.stderr[-2000:]))
        files = sorted(Path(td).glob("st.*.bin"))
        assert len(files) == 1, files
        state = read_state(files[0])
        geom = read_geom(os.path.join(td, "geom.bin"), n) if want_geom else None
    return state, geom


class OrDesc(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int32), ("n2", ctypes.c_int32), ("n3", ctypes.c_int32),
                ("recon_type", ctypes.c_int32), ("flux_type", ctypes.c_int32),
                ("use_flux_ct_para", ctypes.c_int32), ("bc_type", ctypes.c_int32),
                ("metric_dim", ctypes.c_int32), ("use_entropy_eq", ctypes.c_int32),
                ("cooling", ctypes.c_int32), ("rescale_r", ctypes.c_int32), ("pad0", ctypes.c_int32),
                ("gam", ctypes.c_double), ("cour", ctypes.c_double), ("dx", ctypes.c_double * 4),
                ("startx", ctypes.c_double * 4), ("grid_length", ctypes.c_double * 4),
                ("t", ctypes.c_double)]


_olib = None
_olibs = {}
# The oracle builds (oracle/Makefile): "liboracle.so" with glibc's pow() (the
# reference's own arithmetic), "liboracle_cr.so" with the correctly rounded
# pow() the engine uses, "liboracle_powcmp.so" glibc's pow() counting where
# the two differ.
CR_ORACLE = "liboracle_cr.so"


def ensure_oracle(name="liboracle.so"):
    """Path of an oracle build, made with oracle/Makefile if missing."""
    path = REPO / "oracle" / name
    if not path.exists():
        subprocess.check_call(["make", "-s", "-C", str(REPO / "oracle"), name])
    return path


def oracle_lib(name=None):
    """The oracle library: the one at ORACLE_SO, or the build `name`."""
    global _olib
    if name is not None:
        if name not in _olibs:
            _olibs[name] = _configure(ctypes.CDLL(str(ensure_oracle(name))))
        return _olibs[name]
    if _olib is None:
        if not ORACLE_SO.exists():
            subprocess.check_call(["make", "-s", "-C", str(REPO / "oracle"), "liboracle.so"])
        _olib = _configure(ctypes.CDLL(str(ORACLE_SO)))
    return _olib


def _configure(lib):
    P = ctypes.c_void_p
    lib.or_create.restype = P
    lib.or_create.argtypes = [ctypes.POINTER(OrDesc), P, P, P, P]
    lib.or_destroy.argtypes = [P]
    lib.or_set_prims.argtypes = [P, P, ctypes.c_double, ctypes.c_double]
    for fn in ("or_get_prims", "or_get_pflag", "or_get_gamma", "or_get_nfail", "or_get_nfailtot"):
        getattr(lib, fn).argtypes = [P, P]
    lib.or_get_time.argtypes = [P, P, P, P]
    lib.or_step.argtypes = [P, ctypes.c_int]
    lib.or_fixup_bounds.argtypes = [P]
    lib.or_totals.argtypes = [P, P, P, P]
    lib.or_face_flux.argtypes = [P, ctypes.c_int, P, P]
    lib.or_set_cooling.argtypes = [P, P, P]
    lib.or_ntot.restype = ctypes.c_long
    lib.or_ntot.argtypes = [P]
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Oracle:
    """The C restatement of the reference step (oracle/harm_oracle.c).
    lib: which oracle build (None: ORACLE_SO, glibc's pow(); CR_ORACLE: the
    correctly rounded pow() of the engine)."""

    def __init__(self, n, sw, geomd, lib=None):
        self.lib = oracle_lib(lib)
        d = OrDesc()
        d.n1, d.n2, d.n3 = n
        d.recon_type, d.flux_type, d.use_flux_ct_para = sw["recon"], sw["flux"], sw["ct_para"]
        d.bc_type, d.metric_dim, d.use_entropy_eq = sw["bc"], sw["metric_dim"], sw["ee"]
        d.cooling, d.rescale_r = sw["cooling"], sw["rescale"]
        d.gam, d.cour = geomd["gam"], geomd["cour"]
        for a in range(4):
            d.dx[a] = geomd["dx"][a]
            d.startx[a] = geomd["startx"][a]
            d.grid_length[a] = geomd["grid_length"][a]
        self.n = n
        self.shape = tuple(tot(x) for x in n)
        self._keep = [np.ascontiguousarray(geomd["geom"]), np.ascontiguousarray(geomd["conn"]),
                      np.ascontiguousarray(geomd["cell6"]), geomd.get("rface")]
        self.h = self.lib.or_create(ctypes.byref(d), *(_ptr(x) for x in self._keep))
        if sw["cooling"]:
            om = np.ascontiguousarray(geomd["cool_omega"], np.float64)
            te = np.ascontiguousarray(geomd["cool_temp"], np.float64)
            self.lib.or_set_cooling(self.h, _ptr(om), _ptr(te))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.or_destroy(self.h)
            self.h = None

    def set_state(self, p, t, dt):
        p = np.ascontiguousarray(p, np.float64)
        self.lib.or_set_prims(self.h, _ptr(p), t, dt)

    def step(self, n=1):
        self.lib.or_step(self.h, n)

    # the Engine methods a setup drives (upload / fixup_bounds / download)
    def upload(self, p):
        self.set_state(p, 0.0, 0.0)

    def fixup_bounds(self):
        self.lib.or_fixup_bounds(self.h)

    def totals(self):
        u = np.zeros(8)
        f = np.zeros((3, 2, 8))
        m = ctypes.c_double()
        self.lib.or_totals(self.h, _ptr(u), _ptr(f), ctypes.byref(m))
        return u, f, m.value

    def download(self):
        p = np.empty(self.shape + (NP,))
        self.lib.or_get_prims(self.h, _ptr(p))
        return p

    def face_flux(self, d):
        f = np.empty(self.shape + (NP,))
        m = ctypes.c_double()
        self.lib.or_face_flux(self.h, d, _ptr(f), ctypes.byref(m))
        return f, m.value

    def state(self):
        ncell = self.shape[0] * self.shape[1] * self.shape[2]
        p = np.empty(self.shape + (NP,))
        pf = np.empty(self.shape, np.int32)
        g = np.empty(self.shape)
        nf = np.empty((NFAIL,) + self.shape, np.int32)
        nft = np.empty(NFAIL, np.uint64)
        tt = (ctypes.c_double * 3)()
        self.lib.or_get_prims(self.h, _ptr(p))
        self.lib.or_get_pflag(self.h, _ptr(pf))
        self.lib.or_get_gamma(self.h, _ptr(g))
        self.lib.or_get_nfail(self.h, _ptr(nf))
        self.lib.or_get_nfailtot(self.h, _ptr(nft))
        self.lib.or_get_time(self.h, ctypes.byref(tt, 0), ctypes.byref(tt, 8), ctypes.byref(tt, 16))
        assert ncell == p.shape[0] * p.shape[1] * p.shape[2]
        return dict(p=p, pflag=pf, gamma=g, nfail=nf, nfailtot=nft, t=tt[0], dt=tt[1], m_tot=tt[2])


def interior(a, n):
    """Physical cells of a [N1TOT][N2TOT][N3TOT]... array."""
    return a[NG:NG + n[0], NG:NG + n[1], NG:NG + n[2]]
