"""coolharm3d_b200 -- B200 (sm_100a) engine for HARM3D's step_ch()/advance() path.

The engine is the in-tree shared library libharmgpu.so (C ABI in
include/harmgpu.h).  This module is its Python binding, used by the tests and
bench.py the way the reference's C driver (src/main.c, src/step_ch.c) uses the
library: describe the grid, hand over geometry and primitives, step, read back.

There is no CPU fallback: if libharmgpu.so is missing or no CUDA device is
present, Engine() raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HARMGPU_LIB") or os.path.join(HERE, "libharmgpu.so")
NG, NP, NFAIL, NGEOM = 3, 8, 15, 42

# options.h switch values accepted by the engine
RECON_MINMOD, RECON_VANL, RECON_MC, RECON_PPM_MM, RECON_PPM_VL, RECON_PPM_MC = range(6)
FLUX_LF, FLUX_HLLE = 0, 1
BC_CARTESIAN_OUTFLOW, BC_CARTESIAN_PERIODIC, BC_SPHERICAL_OUTFLOW3 = 0, 1, 10
PREC_FP64, PREC_MIXED, PREC_FP64_FMA = 0, 1, 2

# nfail[] slots (macros.h:243-258)
NFAIL_NAMES = ["FLOOR", "TMAX", "GAMMA_MAX", "GAMMA_CALC", "USE_FULL_INV", "USE_EE", "UTOPRIM",
               "UTOPRIM_EE", "USE_INTERP_PRIM", "USE_INTERP_V", "INTERP_PRIM", "INTERP_V",
               "CUTOUT_PRESSURE", "CUTOUT_GAMMA", "CUTOUT_BC"]


class GridDesc(ctypes.Structure):
    """hg_grid_desc of include/harmgpu.h."""
    _fields_ = [("n1", ctypes.c_int32), ("n2", ctypes.c_int32), ("n3", ctypes.c_int32),
                ("recon_type", ctypes.c_int32), ("flux_type", ctypes.c_int32),
                ("use_flux_ct_para", ctypes.c_int32), ("bc_type", ctypes.c_int32),
                ("metric_dim", ctypes.c_int32), ("use_entropy_eq", ctypes.c_int32),
                ("cooling", ctypes.c_int32), ("rescale_r", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("gam", ctypes.c_double), ("cour", ctypes.c_double), ("dx", ctypes.c_double * 4),
                ("startx", ctypes.c_double * 4), ("grid_length", ctypes.c_double * 4),
                ("t", ctypes.c_double), ("device", ctypes.c_int32), ("reserved", ctypes.c_int32)]


EXPORTS = ["hg_check_mirror", "hg_init", "hg_set_geometry", "hg_set_cell_data", "hg_upload_prims", "hg_download_prims",
           "hg_upload_prims_tree", "hg_download_prims_tree", "hg_set_time", "hg_step", "hg_get_fail_counts",
           "hg_download_pflag", "hg_download_gamma", "hg_download_nfail", "hg_get_diag", "hg_last_step_ms",
           "hg_destroy", "hg_strerror", "hg_build_geometry_minkowski", "hg_profile", "hg_kernel_times", "hg_face_flux", "hg_face_flux_noalloc", "hg_set_cooling_tables",
           "hg_build_geometry_ks_mks", "hg_fixup_bounds", "hg_batch_create", "hg_batch_add", "hg_batch_remove",
           "hg_batch_size", "hg_batch_step", "hg_batch_destroy", "hg_mem_info", "hg_grid_bytes",
           "hg_get_totals", "hg_get_launch_config", "hg_set_launch_config", "hg_autotune",
           "hg_write_rdump", "hg_read_rdump", "hg_fp64_peak", "hg_set_dynamic_metric", "hg_dyn_geometry",
           "hg_dyn_geometry_block", "hg_download_dyn_level"]
KERNEL_CLASSES = ["flux", "emf", "update", "fallback", "bounds", "fixup", "misc", "geometry"]

DYN_KS_SPHERICAL = 0
DYN_MINK_SPHERICAL = 2
DYN_PN_BINARY = 3


class DynMetric(ctypes.Structure):
    """hg_dyn_metric: the spacetime and COORD_DIAGONAL3 parameters of a
    metric_dim 3 (time-dependent metric) grid."""
    _fields_ = [("spacetime", ctypes.c_int32), ("diag3_exponent", ctypes.c_int32), ("R0", ctypes.c_double),
                ("h_slope", ctypes.c_double), ("diag3_factor", ctypes.c_double), ("dt_conn", ctypes.c_double),
                ("m1", ctypes.c_double), ("m2", ctypes.c_double), ("separation", ctypes.c_double),
                ("phase0", ctypes.c_double), ("inspiral", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("spin", ctypes.c_double)]


def dyn_metric(spacetime=DYN_MINK_SPHERICAL, R0=0.0, h_slope=0.35, th_cutout=None, diag3_exponent=7, dt_conn=9.0e-6,
               m1=0.5, m2=0.5, separation=20.0, phase0=0.0, inspiral=1, spin=0.0):
    """The torus setup's coordinates (set_special_coord, init.torus.c:245-270:
    th_cutout = SMALL pi, diag3_factor = 1 - 2 th_cutout/pi - h_slope), the
    driver's dt_conn (main.c:569), for DYN_PN_BINARY the binary and for
    DYN_KS_SPHERICAL the spin."""
    import math
    if th_cutout is None:
        th_cutout = 1e-15 * math.pi
    m = DynMetric()
    m.spacetime, m.diag3_exponent, m.R0, m.h_slope = spacetime, diag3_exponent, R0, h_slope
    m.diag3_factor = 1. - 2 * th_cutout / math.pi - h_slope
    m.dt_conn = dt_conn
    m.m1, m.m2, m.separation, m.phase0, m.inspiral = m1, m2, separation, phase0, inspiral
    m.spin = spin
    return m


def dyn_geometry(desc, m, pos, i, j, k, t=0.0):
    """hg_dyn_geometry: the 42-double struct of_geom the device evaluates, on the host."""
    out = np.zeros(NGEOM)
    _check(load_library().hg_dyn_geometry(ctypes.byref(desc), ctypes.byref(m), pos, i, j, k, t, _ptr(out)),
           "hg_dyn_geometry")
    return out


class LaunchConfig(ctypes.Structure):
    """hg_launch_config: blocks per launch of each kernel class and the
    strip length of the x2/x3 flux kernels."""
    _fields_ = [("grid_flux", ctypes.c_int32), ("grid_flux32", ctypes.c_int32), ("grid_emf", ctypes.c_int32),
                ("grid_update", ctypes.c_int32), ("grid_fixup", ctypes.c_int32), ("grid_bounds", ctypes.c_int32),
                ("strip_faces", ctypes.c_int32), ("strip_x1", ctypes.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def load_library(path=LIB_PATH):
    """Load libharmgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libharmgpu.so not found at %s: run coolharm3d_b200/build.py" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    I = ctypes.c_int
    lib.hg_init.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(P)]
    lib.hg_set_geometry.argtypes = [P, P, ctypes.c_int64, P, ctypes.c_int64]
    lib.hg_set_cell_data.argtypes = [P, P, P]
    for fn in ("hg_upload_prims", "hg_download_prims", "hg_upload_prims_tree", "hg_download_prims_tree",
               "hg_get_fail_counts", "hg_download_pflag", "hg_download_gamma", "hg_download_nfail",
               "hg_last_step_ms"):
        getattr(lib, fn).argtypes = [P, P]
    lib.hg_check_mirror.argtypes = [P, P, P]
    lib.hg_set_time.argtypes = [P, ctypes.c_double, ctypes.c_double]
    lib.hg_step.argtypes = [P, ctypes.c_int32, P, P]
    lib.hg_get_diag.argtypes = [P, P, P]
    lib.hg_destroy.argtypes = [P]
    lib.hg_destroy.restype = None
    lib.hg_strerror.argtypes = [I]
    lib.hg_strerror.restype = ctypes.c_char_p
    lib.hg_build_geometry_minkowski.argtypes = [ctypes.POINTER(GridDesc), P, P]
    lib.hg_profile.argtypes = [P, ctypes.c_int32]
    lib.hg_kernel_times.argtypes = [P, P, P]
    lib.hg_face_flux.argtypes = [P, ctypes.c_int32, P, P]
    lib.hg_set_cooling_tables.argtypes = [P, P, P]
    lib.hg_face_flux_noalloc.argtypes = [ctypes.POINTER(GridDesc), P, P, P, P, ctypes.c_int32, P]
    D = ctypes.c_double
    lib.hg_fixup_bounds.argtypes = [P]
    lib.hg_batch_create.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(P)]
    lib.hg_batch_add.argtypes = [P, P]
    lib.hg_batch_remove.argtypes = [P, P]
    lib.hg_batch_size.argtypes = [P]
    lib.hg_batch_step.argtypes = [P, P, P]
    lib.hg_batch_destroy.argtypes = [P]
    lib.hg_mem_info.argtypes = [ctypes.c_int32, P, P]
    lib.hg_fp64_peak.argtypes = [ctypes.c_int32, P, P]
    lib.hg_set_dynamic_metric.argtypes = [P, P]
    lib.hg_dyn_geometry.argtypes = [ctypes.POINTER(GridDesc), P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_double, P]
    lib.hg_dyn_geometry_block.argtypes = [ctypes.POINTER(GridDesc), P, ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_int32, ctypes.c_int32, P]
    lib.hg_download_dyn_level.argtypes = [P, ctypes.c_int32, P]
    lib.hg_get_totals.argtypes = [P, P, P, P]
    lib.hg_get_launch_config.argtypes = [P, ctypes.POINTER(LaunchConfig)]
    lib.hg_set_launch_config.argtypes = [P, ctypes.POINTER(LaunchConfig)]
    lib.hg_autotune.argtypes = [P, ctypes.c_int32, ctypes.POINTER(LaunchConfig), P, P]
    lib.hg_write_rdump.argtypes = [P, ctypes.c_char_p, ctypes.c_int32, P, ctypes.c_int32]
    lib.hg_read_rdump.argtypes = [P, ctypes.c_char_p, P, P, P]
    lib.hg_grid_bytes.argtypes = [ctypes.POINTER(GridDesc), P]
    lib.hg_build_geometry_ks_mks.argtypes = [ctypes.POINTER(GridDesc), D, D, D, D, ctypes.c_int32, D,
                                             P, P, P, P, P, P]
    for fn in EXPORTS:
        if fn not in ("hg_destroy", "hg_strerror", "hg_batch_destroy"):
            getattr(lib, fn).restype = I
    _lib = lib
    return lib


class HarmGPUError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        msg = load_library().hg_strerror(rc).decode()
        raise HarmGPUError("%s failed: %s (%d)" % (what, msg, rc))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def make_desc(n, gam, cour, dx, startx, grid_length, t=0.0, recon=RECON_PPM_MC, flux=FLUX_HLLE, ct_para=1,
              bc=BC_CARTESIAN_PERIODIC, metric_dim=0, use_ee=1, cooling=0, rescale_r=0, precision=PREC_FP64,
              device=0):
    d = GridDesc()
    d.n1, d.n2, d.n3 = (int(x) for x in n)
    d.recon_type, d.flux_type, d.use_flux_ct_para = recon, flux, ct_para
    d.bc_type, d.metric_dim, d.use_entropy_eq = bc, metric_dim, use_ee
    d.cooling, d.rescale_r, d.precision = cooling, rescale_r, precision
    d.gam, d.cour, d.t, d.device = gam, cour, t, device
    for a in range(4):
        d.dx[a], d.startx[a], d.grid_length[a] = dx[a], startx[a], grid_length[a]
    return d


def ref_shape(n):
    return tuple(int(x) + 2 * NG for x in n)


def minkowski_tables(desc):
    """Geometry and per-cell floor tables of Minkowski space (host builder)."""
    lib = load_library()
    shp = ref_shape((desc.n1, desc.n2, desc.n3))
    geom = np.zeros(NGEOM)
    cell6 = np.zeros(shp + (6,))
    _check(lib.hg_build_geometry_minkowski(ctypes.byref(desc), _ptr(geom), _ptr(cell6)),
           "hg_build_geometry_minkowski")
    return geom, cell6


def ks_mks_tables(desc, a, R0=0.0, h_slope=0.35, th_cutout=1e-15 * np.pi, diag3_exponent=7, h_o_r=0.1):
    """Geometry, connection, per-zone data, FACE1 radii and H/R cooling tables
    of Kerr-Schild space-time in COORD_DIAGONAL3 modified Kerr-Schild
    coordinates (host builder).  diag3_factor = 1 - 2 th_cutout/pi - h_slope,
    as set_special_coord() sets it (init.torus.c:254-269).  Returns a dict with
    geom (5*N1TOT*N2TOT, 42), conn (N1*N2, 64), cell6, rface, cool_omega,
    cool_temp."""
    lib = load_library()
    n1, n2, n3 = desc.n1, desc.n2, desc.n3
    shp = ref_shape((n1, n2, n3))
    out = dict(geom=np.zeros((5 * shp[0] * shp[1], NGEOM)), conn=np.zeros((n1 * n2, 64)),
               cell6=np.zeros(shp + (6,)), rface=np.zeros(shp[0]), cool_omega=np.zeros(shp[0]),
               cool_temp=np.zeros(shp[0]))
    diag3_factor = 1.0 - 2 * th_cutout / np.pi - h_slope
    _check(lib.hg_build_geometry_ks_mks(ctypes.byref(desc), a, R0, h_slope, diag3_factor, diag3_exponent, h_o_r,
                                        *[_ptr(out[k]) for k in ("geom", "conn", "cell6", "rface", "cool_omega",
                                                                 "cool_temp")]),
           "hg_build_geometry_ks_mks")
    return out


def dyn_geometry_block(desc, m, pos, t, i0, ni):
    """hg_dyn_geometry_block: planes i0 .. i0+ni-1 of the struct of_geom the
    device evaluates, (ni, N2TOT, N3TOT, 42), on the host."""
    shp = ref_shape((desc.n1, desc.n2, desc.n3))
    out = np.zeros((ni, shp[1], shp[2], NGEOM))
    _check(load_library().hg_dyn_geometry_block(ctypes.byref(desc), ctypes.byref(m), pos, t, i0, ni, _ptr(out)),
           "hg_dyn_geometry_block")
    return out


class Engine:
    """One device-resident grid (an hg_handle)."""

    def __init__(self, desc):
        self.lib = load_library()
        self.desc = desc
        self.n = (desc.n1, desc.n2, desc.n3)
        self.shape = ref_shape(self.n)
        h = ctypes.c_void_p()
        _check(self.lib.hg_init(ctypes.byref(desc), ctypes.byref(h)), "hg_init")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.hg_destroy(self.h)
            self.h = None

    __del__ = close

    def set_geometry(self, geom, conn=None):
        geom = np.ascontiguousarray(geom, np.float64)
        ng = geom.size // NGEOM
        conn = None if conn is None else np.ascontiguousarray(conn, np.float64)
        nc = 0 if conn is None else conn.size // 64
        _check(self.lib.hg_set_geometry(self.h, _ptr(geom), ng, _ptr(conn), nc), "hg_set_geometry")

    def set_dynamic_metric(self, m):
        """metric_dim 3: the time-dependent metric the device evaluates."""
        _check(self.lib.hg_set_dynamic_metric(self.h, ctypes.byref(m)), "hg_set_dynamic_metric")

    def set_cell_data(self, cell6, rface=None):
        cell6 = np.ascontiguousarray(cell6, np.float64)
        rface = None if rface is None else np.ascontiguousarray(rface, np.float64)
        self._keep = (cell6, rface)
        _check(self.lib.hg_set_cell_data(self.h, _ptr(cell6), _ptr(rface)), "hg_set_cell_data")

    def set_cooling_tables(self, omega, t_target):
        om = np.ascontiguousarray(omega, np.float64)
        tt = np.ascontiguousarray(t_target, np.float64)
        _check(self.lib.hg_set_cooling_tables(self.h, _ptr(om), _ptr(tt)), "hg_set_cooling_tables")

    def upload(self, p):
        p = np.ascontiguousarray(p, np.float64)
        assert p.shape == self.shape + (NP,), p.shape
        _check(self.lib.hg_upload_prims(self.h, _ptr(p)), "hg_upload_prims")

    def check_mirror(self, first=False):
        """Mixed form: stored values where the FP32 copy differs from the
        state rounded to float (0 expected between steps); with first=True
        also the lowest mismatching stored offset (l * S + o), or -1."""
        n, f = ctypes.c_int64(), ctypes.c_int64()
        _check(self.lib.hg_check_mirror(self.h, ctypes.byref(n), ctypes.byref(f)), "hg_check_mirror")
        return (n.value, f.value) if first else n.value

    def download(self, out=None):
        """The primitives in the reference layout; into `out` (a C-contiguous
        float64 array of that shape, e.g. from pinned_array) if given."""
        if out is None:
            out = np.empty(self.shape + (NP,))
        assert out.shape == self.shape + (NP,) and out.dtype == np.float64 and out.flags.c_contiguous
        _check(self.lib.hg_download_prims(self.h, _ptr(out)), "hg_download_prims")
        return out

    def dyn_level(self, level=0):
        """metric_dim 3: time level 0/1/2 (n_beg, n_mid, n_end) of the next
        step as the device evaluated it, (4, N1TOT, N2TOT, N3TOT, 42): the
        positions FACE1..FACE3 and CENT."""
        out = np.empty((4,) + self.shape + (NGEOM,))
        _check(self.lib.hg_download_dyn_level(self.h, level, _ptr(out)), "hg_download_dyn_level")
        return out

    def set_time(self, t, dt):
        _check(self.lib.hg_set_time(self.h, t, dt), "hg_set_time")

    def step(self, n=1):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        _check(self.lib.hg_step(self.h, n, ctypes.byref(t), ctypes.byref(dt)), "hg_step")
        return t.value, dt.value

    def fail_counts(self):
        v = np.zeros(NFAIL, np.uint64)
        _check(self.lib.hg_get_fail_counts(self.h, _ptr(v)), "hg_get_fail_counts")
        return v

    def pflag(self):
        v = np.empty(self.shape, np.int32)
        _check(self.lib.hg_download_pflag(self.h, _ptr(v)), "hg_download_pflag")
        return v

    def gamma(self):
        v = np.empty(self.shape)
        _check(self.lib.hg_download_gamma(self.h, _ptr(v)), "hg_download_gamma")
        return v

    def nfail(self):
        v = np.empty((NFAIL,) + self.shape, np.int32)
        _check(self.lib.hg_download_nfail(self.h, _ptr(v)), "hg_download_nfail")
        return v

    def fixup_bounds(self):
        """Floors and gamma ceiling over the physical zones, then the boundary
        zones, on the resident primitives (the setups' fixup(p); bounds(p,0))."""
        _check(self.lib.hg_fixup_bounds(self.h), "hg_fixup_bounds")

    def face_flux(self, d):
        """(flux of direction d in the reference layout, max char speed)."""
        f = np.empty(self.shape + (NP,))
        m = ctypes.c_double()
        _check(self.lib.hg_face_flux(self.h, d, _ptr(f), ctypes.byref(m)), "hg_face_flux")
        return f, m.value

    def launch_config(self):
        c = LaunchConfig()
        _check(self.lib.hg_get_launch_config(self.h, ctypes.byref(c)), "hg_get_launch_config")
        return c

    def set_launch_config(self, c):
        _check(self.lib.hg_set_launch_config(self.h, ctypes.byref(c)), "hg_set_launch_config")

    def autotune(self, steps=3):
        """Measure launch configurations on the resident state (which is
        restored) and keep the fastest; returns (config, ms before, ms after)."""
        c = LaunchConfig()
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.hg_autotune(self.h, steps, ctypes.byref(c), ctypes.byref(a), ctypes.byref(b)), "hg_autotune")
        return c, a.value, b.value

    def write_rdump(self, path, nstep=0, n_out=None, rdump_cnt=0):
        """restart_write(): the ASCII rdump file of the resident state."""
        no = np.ascontiguousarray(n_out if n_out is not None else np.zeros(11), np.int32)
        _check(self.lib.hg_write_rdump(self.h, str(path).encode(), nstep, _ptr(no), rdump_cnt), "hg_write_rdump")

    def read_rdump(self, path):
        """restart_read(): load an rdump file; returns (nstep, n_out, rdump_cnt)."""
        ns, rc = ctypes.c_int32(), ctypes.c_int32()
        no = np.zeros(11, np.int32)
        _check(self.lib.hg_read_rdump(self.h, str(path).encode(), ctypes.byref(ns), _ptr(no), ctypes.byref(rc)),
               "hg_read_rdump")
        return ns.value, no, rc.value

    def totals(self):
        """(U_tot[8], F_tot[3, 2, 8], max |div B|) of the last step (dump_ener)."""
        u = np.zeros(8)
        f = np.zeros((3, 2, 8))
        m = ctypes.c_double()
        _check(self.lib.hg_get_totals(self.h, _ptr(u), _ptr(f), ctypes.byref(m)), "hg_get_totals")
        return u, f, m.value

    def diag(self):
        m = ctypes.c_double()
        c = (ctypes.c_double * 3)()
        _check(self.lib.hg_get_diag(self.h, ctypes.byref(m), c), "hg_get_diag")
        return m.value, tuple(c)

    def profile(self, enable=True):
        _check(self.lib.hg_profile(self.h, 1 if enable else 0), "hg_profile")

    def kernel_times(self):
        """{class: (total ms, launches)} since the last profile() call."""
        ms = np.zeros(len(KERNEL_CLASSES))
        n = np.zeros(len(KERNEL_CLASSES), np.int64)
        _check(self.lib.hg_kernel_times(self.h, _ptr(ms), _ptr(n)), "hg_kernel_times")
        return {c: (float(ms[i]), int(n[i])) for i, c in enumerate(KERNEL_CLASSES)}

    def last_step_ms(self):
        v = ctypes.c_double()
        _check(self.lib.hg_last_step_ms(self.h, ctypes.byref(v)), "hg_last_step_ms")
        return v.value


def mem_info(device=0):
    """(free, total) bytes of the device."""
    f, t = ctypes.c_uint64(), ctypes.c_uint64()
    _check(load_library().hg_mem_info(device, ctypes.byref(f), ctypes.byref(t)), "hg_mem_info")
    return f.value, t.value


def fp64_peak(device=0):
    """(TFLOP/s, ms) of the device's measured FP64 fused-multiply-add peak."""
    tf, ms = ctypes.c_double(), ctypes.c_double()
    _check(load_library().hg_fp64_peak(device, ctypes.byref(tf), ctypes.byref(ms)), "hg_fp64_peak")
    return tf.value, ms.value


def pinned_array(shape, dtype=np.float64):
    """A numpy array in page-locked host memory (torch's pinned allocator).
    hg_upload_prims / hg_download_prims move such a buffer by one DMA, with
    no staging copy on the host."""
    import torch
    t = torch.empty(int(np.prod(shape)) * np.dtype(dtype).itemsize, dtype=torch.uint8, pin_memory=True)
    return t.numpy().view(dtype).reshape(shape)  # the view's base chain holds the tensor


def grid_bytes(desc):
    """Device bytes hg_init allocates for desc."""
    b = ctypes.c_uint64()
    _check(load_library().hg_grid_bytes(ctypes.byref(desc), ctypes.byref(b)), "hg_grid_bytes")
    return b.value


class Batch:
    """Resident grids of one device advanced together (hg_batch_*): one
    step() advances every member by one of its own steps, its kernels
    overlapping the other members' on the device."""

    def __init__(self, device=0, max_grids=256):
        self.lib = load_library()
        b = ctypes.c_void_p()
        _check(self.lib.hg_batch_create(device, max_grids, ctypes.byref(b)), "hg_batch_create")
        self.b = b
        self.members = []
        self._t = np.zeros(max_grids)
        self._dt = np.zeros(max_grids)

    def add(self, engine):
        _check(self.lib.hg_batch_add(self.b, engine.h), "hg_batch_add")
        self.members.append(engine)

    def remove(self, engine):
        _check(self.lib.hg_batch_remove(self.b, engine.h), "hg_batch_remove")
        self.members.remove(engine)

    def __len__(self):
        return len(self.members)

    def step(self):
        """One step of every member; returns (t, dt) arrays in member order."""
        _check(self.lib.hg_batch_step(self.b, _ptr(self._t), _ptr(self._dt)), "hg_batch_step")
        n = len(self.members)
        return self._t[:n].copy(), self._dt[:n].copy()

    def close(self):
        if getattr(self, "b", None):
            self.lib.hg_batch_destroy(self.b)
            self.b = None
            self.members = []

    __del__ = close
