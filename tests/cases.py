"""Parity cases shared by the golden-fixture generator and the tests.

Each case is a small 3D run whose initial state is fully determined by code
here: markers come from the ranmar placer (oracle/pic_oracle.c:po_place and
the device placer implement the same rule) and fields from a closed-form sum
of modes.  The reference's output for every case is frozen in
tests/golden/<name>.npz by tests/golden/make_golden.py.
"""
import math

import numpy as np

TWO_PI = 2 * math.pi
N_CR = 4 * math.pi ** 2          # critical density in code units (misc_units.c:96-114)

CASES = {
    # Periodic box, warm drifting electrons filling the whole box.
    "periodic_thermal": dict(n=(10, 12, 14), bc_min=(0, 0, 0), bc_max=(0, 0, 0),
                             steps=6, ppc=2, uth=(0.1, 0.1, 0.1), drift=(0.3, -0.2, 0.1),
                             field_amp=0.5, box="full"),
    # Mirror walls, relativistic electrons: reflections and 2-/3-face crossings.
    "mirror_hot": dict(n=(12, 10, 10), bc_min=(1, 1, 1), bc_max=(1, 1, 1),
                       steps=8, ppc=2, uth=(1.5, 1.5, 1.5), drift=(0, 0, 0),
                       field_amp=2.0, box="full"),
    # Mur (open) on x, periodic on y, mirror on z: markers removed at open walls.
    "mur_mixed": dict(n=(14, 10, 12), bc_min=(2, 0, 1), bc_max=(2, 0, 1),
                      steps=8, ppc=2, uth=(1.0, 1.0, 1.0), drift=(0.5, 0, 0),
                      field_amp=1.0, box="full"),
    # All walls Mur, cold slab in the middle, strong fields (field parity).
    "mur_slab": dict(n=(16, 12, 12), bc_min=(2, 2, 2), bc_max=(2, 2, 2),
                     steps=10, ppc=4, uth=(0, 0, 0), drift=(0, 0, 0),
                     field_amp=3.0, box="slab"),
}

H_LAMBDA = 0.05 / TWO_PI          # 0.05 c/omega_p at n = n_cr, in wavelengths


def geometry(case):
    n = case["n"]
    L_um = [v * H_LAMBDA for v in n]          # lambda = 1 micron
    return n, L_um


def place_box(case):
    n = case["n"]
    if case["box"] == "full":
        return (0, 0, 0), tuple(n)
    lo = (n[0] // 2 - 2, 3, 3)
    hi = (n[0] // 2 + 2, n[1] - 3, n[2] - 3)
    return lo, hi


def placer_args(case, h):
    lo, hi = place_box(case)
    return dict(lo=lo, hi=hi, ppc=case["ppc"], rho=-N_CR / case["ppc"], qDivM=-1.0, h=h,
                drift=case["drift"], uth=case["uth"], seed=(1802, 9373), skip=0, id0=1)


def initial_fields(case, h):
    """Closed-form E and H over the checkpoint region [0,n]^3 (AoS, k fastest)."""
    n = case["n"]
    a = case["field_amp"]
    i, j, k = np.meshgrid(np.arange(n[0] + 1), np.arange(n[1] + 1), np.arange(n[2] + 1),
                          indexing="ij")
    x, y, z = i / n[0], j / n[1], k / n[2]
    E = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
    H = np.zeros_like(E)
    E[..., 0] = a * np.sin(TWO_PI * (y + 2 * z)) * np.cos(TWO_PI * x)
    E[..., 1] = a * 0.7 * np.cos(TWO_PI * (x - z)) + 0.1 * a * np.sin(3 * TWO_PI * y)
    E[..., 2] = a * 0.4 * np.sin(TWO_PI * (2 * x + y))
    H[..., 0] = a * 0.3 * np.cos(TWO_PI * (y - z))
    H[..., 1] = a * 0.6 * np.sin(TWO_PI * (x + z)) * np.cos(TWO_PI * y)
    H[..., 2] = a * 0.5 * np.cos(TWO_PI * (x + 2 * y))
    return E, H
