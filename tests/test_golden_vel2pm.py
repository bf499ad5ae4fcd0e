"""Pins of the oracle against the reference's own test data (CPU only).

* tests/os_vel2pm/result/sky.obs.txt of the reference (371 rows, committed as
  tests/golden/os_vel2pm_sky_obs.npz by tests/golden/make_golden.py): its radec
  columns pin gal2other (galequ, gal2other_gpu.cu.h:39-60) to the printed 8
  decimals, its pmlb columns pin vcyl2pm (vel2pm_gpu.cu.h:221-251, defaults
  vel2pm_host.cpp:89-92) to the printed 0.1 mas/yr once the printed vcyl
  (0.1 km/s) rounding is allowed for.
* the known-answer comment of vcyl2pm (vel2pm_gpu.cu.h:223-232): X=8100, Y=100,
  Z=3000, v=(10, 50, -30) must give (12.72 mas/yr, -14.75 mas/yr, -27.34 km/s).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import galfast_b200 as G
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "os_vel2pm_sky_obs.npz")


def vcyl2pm(flavour, par, l, b, X, Y, Z, v):
    L = O.load(flavour)
    n = len(l)
    a = lambda x, t: np.ascontiguousarray(x, dtype=t)
    l, b = a(l, np.float64), a(b, np.float64)
    X, Y, Z = a(X, np.float32), a(Y, np.float32), a(Z, np.float32)
    vx, vy, vz = a(v[:, 0], np.float32), a(v[:, 1], np.float32), a(v[:, 2], np.float32)
    out = np.zeros((n, 3), dtype=np.float32)
    L.or_vcyl2pm(C.addressof(par), n, l.ctypes.data, b.ctypes.data, X.ctypes.data, Y.ctypes.data, Z.ctypes.data,
                 vx.ctypes.data, vy.ctypes.data, vz.ctypes.data, out.ctypes.data)
    return out


def default_par(coordsys=0):
    p = G.Vel2pmConfig()
    p.coordsys = coordsys
    p.vLSR, p.u0, p.v0, p.w0, p.Rg = -220.0, -10.0, -5.3, 7.2, 8000.0
    return p


@pytest.mark.parametrize("flavour", ["p", "l"])
def test_vcyl2pm_known_answer(flavour):
    X, Y, Z = 8100.0, 100.0, 3000.0
    l = math.degrees(math.atan2(-Y, 8000 - X))
    b = math.degrees(math.asin(Z / math.sqrt((8000 - X) ** 2 + Y ** 2 + Z ** 2)))
    pm = vcyl2pm(flavour, default_par(), [l], [b], [X], [Y], [Z], np.array([[10.0, 50.0, -30.0]]))[0]
    assert np.round(pm.astype(np.float64), 2).tolist() == [12.72, -14.75, -27.34]


@pytest.mark.parametrize("flavour", ["p", "l"])
def test_vcyl2pm_golden_rows(flavour):
    g = np.load(GOLD)
    pm = vcyl2pm(flavour, default_par(), g["lb"][:, 0], g["lb"][:, 1], g["XYZ"][:, 0], g["XYZ"][:, 1],
                 g["XYZ"][:, 2], g["vcyl"])
    d = np.abs(pm - g["pmlb"])
    # printed to 0.1 (half-unit 0.05) from velocities printed to 0.1 km/s
    assert d[:, 0].max() < 0.06 and d[:, 1].max() < 0.06
    assert d[:, 2].max() < 0.15
    # mean |error| of uniform rounding to 0.1 is 0.025; v_r also carries the three rounded input velocities
    assert d[:, 0].mean() < 0.03 and d[:, 1].mean() < 0.03 and d[:, 2].mean() < 0.045


@pytest.mark.parametrize("flavour", ["p", "l"])
def test_gal2other_golden_rows(flavour):
    g = np.load(GOLD)
    n = len(g["comp"])
    t = G.HostTable(n, 0)
    t.arrays["lb"][:, :] = g["lb"].T
    t.arrays["hidden"][:] = 0
    t.t.size = n
    O.load(flavour).or_module_gal2other(1, C.addressof(t.t), 0, n)
    radec = t.col("radec").T
    assert np.abs(radec - g["radec"]).max() < 6e-9


def test_vel2pm_module_equatorial_is_rotation_of_galactic():
    """pm_galequ preserves the proper-motion modulus (transform_pm, vel2pm_gpu.cu.h:109-137)."""
    g = np.load(GOLD)
    gal = vcyl2pm("p", default_par(0), g["lb"][:, 0], g["lb"][:, 1], g["XYZ"][:, 0], g["XYZ"][:, 1],
                  g["XYZ"][:, 2], g["vcyl"])
    equ = vcyl2pm("p", default_par(1), g["lb"][:, 0], g["lb"][:, 1], g["XYZ"][:, 0], g["XYZ"][:, 1],
                  g["XYZ"][:, 2], g["vcyl"])
    mg = np.hypot(gal[:, 0], gal[:, 1])
    me = np.hypot(equ[:, 0], equ[:, 1])
    np.testing.assert_allclose(me, mg, rtol=1e-4, atol=1e-4)
    np.testing.assert_array_equal(equ[:, 2], gal[:, 2])
