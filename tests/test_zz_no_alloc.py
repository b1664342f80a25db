"""hg_face_flux_noalloc: the flux entry point for callers that cannot
allocate device memory (inside CUDA-graph capture, under a host memory pool
that owns the device, or in loops that cannot afford cudaMalloc's
synchronisation).  Its only scratch is a static array inside the library.

Checked through the C ABI against the allocating entry point hg_face_flux on
three calls in a row (each reuses the scratch the one before left behind),
covering the HLL and the LF flux and all three directions; both must agree
bit for bit, the tolerance of the FP64 parity tests.  This
file sorts last so that a run stopping at the first failure has run every
other test first."""
import ctypes

import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures

pytestmark = pytest.mark.gpu


def _engine(f):
    sw = f["sw"]
    d = hg.make_desc(f["n"], f["gam"], f["cour"], f["dx"], f["startx"], f["grid_length"], t=f["t0"],
                     recon=sw["recon"], flux=sw["flux"], ct_para=sw["ct_para"], bc=sw["bc"], use_ee=sw["ee"])
    geom, cell6 = hg.minkowski_tables(d)
    e = hg.Engine(d)
    e.set_geometry(geom)
    e.set_cell_data(cell6)
    e.upload(f["p0"])
    return d, geom, e


def test_noalloc_flux_matches_allocating_entry_point_on_consecutive_calls():
    import torch
    lib = hg.load_library()
    # HLL (PPM_MC) along x1 and x2, then LF (PPM_VL) along x3
    calls = [("linwave_noee_stress_10x8x6_s2", 0), ("linwave_12x10x8_s2", 1), ("linwave_vl_stress_8x8x8_s2", 2)]
    stream = torch.cuda.current_stream()
    for name, d in calls:
        f = fixtures.load(name)
        assert f["sw"]["flux"] == (0 if "_vl_" in name else 1)
        desc, geom, e = _engine(f)
        want, want_max = e.face_flux(d)
        prims = torch.from_numpy(np.ascontiguousarray(f["p0"])).cuda()
        flux = torch.zeros_like(prims)
        mx = torch.zeros(1, dtype=torch.float64, device="cuda")
        g = np.ascontiguousarray(geom)
        rc = lib.hg_face_flux_noalloc(ctypes.byref(desc), g.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.c_void_p(prims.data_ptr()), ctypes.c_void_p(flux.data_ptr()),
                                      ctypes.c_void_p(mx.data_ptr()), d, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.hg_strerror(rc)
        torch.cuda.synchronize()
        got = flux.cpu().numpy()
        assert np.array_equal(got, want), (name, d, np.argwhere(got != want)[:4].tolist())
        assert float(mx.cpu()[0]) == want_max
        e.close()


def test_noalloc_flux_rejects_grids_beyond_its_scratch():
    lib = hg.load_library()
    n = (256, 256, 256)
    d = hg.make_desc(n, 4 / 3, 0.4, [1e-5] + [1 / 256.] * 3, [0] + [-3 / 256.] * 3, [1, 1, 1, 1])
    geom = np.zeros(42)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.hg_face_flux_noalloc(ctypes.byref(d), geom.ctypes.data_as(ctypes.c_void_p), dummy, dummy, dummy, 0, None)
    assert rc == -2
