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


# ---------------------------------------------------------------------------
# Runs at the benchmark configurations' sizes and the field-only runs.
# ---------------------------------------------------------------------------
# Cavity resonator (setup/tag_EMResonator.c, deck tests/02_EM-resonator/
# resonator.input): a 30^3 mirror box, 3 microns a side, Courant 0.9, the
# Yee scheme's exact (m, n, l) = (1, 1, 1) eigenmode with Ex polarisation
# and amplitude 5, set up by the reference's own setup.out.
RESONATOR = dict(n=(30, 30, 30), L_um=(3.0, 3.0, 3.0), tau=-0.9, bc=(1, 1, 1), mode=(1, 1, 1),
                 polarisation=0, amplitude=5.0, steps=60)


def resonator_deck():
    from refrun import deck_text
    c = RESONATOR
    text = deck_text(c["n"], c["L_um"], c["tau"], c["bc"], c["bc"])
    text += ("\n[EMResonator]\n@ Yee_2nd_order\tdispersion\n@ %d\tmx\n@ %d\tmy\n@ %d\tmz\n"
             "@ %s\tpolarisation\n@ %.17g\tamplitude\n"
             % (c["mode"] + ("xyz"[c["polarisation"]].join(("E", "")), c["amplitude"])))
    return text


def resonator_omega(h, tau):
    """The mode's frequency from the Yee scheme's dispersion relation,
    omega = (2/tau) asin(tau |D_r| / 2), D_r = (2/h) sin(k h / 2) per axis,
    k = pi m / L with the polarisation's own wave number zeroed
    (setup/tag_EMResonator.c:31-57, 85)."""
    c = RESONATOR
    m = list(c["mode"])
    m[c["polarisation"]] = 0
    k = [math.pi * m[a] / (h[a] * c["n"][a]) for a in range(3)]
    Dr = [2 * math.sin(0.5 * k[a] * h[a]) / h[a] for a in range(3)]
    Dt = math.sqrt(sum(v * v for v in Dr))
    return math.asin(0.5 * tau * Dt) * 2 / tau


# A free pulse leaving an empty box through first-order Mur walls on all
# six faces (core/emCap_Mur.c): h = 0.05, Courant 0.5, E = curl(A z^) of
# a Gaussian A_z placed on the Hz staggering, so that the discrete
# divergence of E is zero and nothing static stays behind; H = 0.
# Checkpoints after 60 steps (the pulse crossing the walls) and 120 steps
# (gone: 0.1 % of the energy left).
MUR_PULSE = dict(n=(32, 28, 24), h=0.05, tau=-0.5, bc=(2, 2, 2), center=(16.0, 14.0, 12.0),
                 width=2.5, amplitude=3.0, period=60, records=2)


def mur_pulse_fields():
    """Initial E, H over the checkpoint region [0, n]^3.  A_z lives at
    (i - 1/2, j - 1/2, k) like Hz; Ex[i,j,k] (at i - 1/2) = dA_z/dy and
    Ey[i,j,k] (at j - 1/2) = -dA_z/dx as forward differences in cells."""
    c = MUR_PULSE
    n = c["n"]
    i, j, k = np.meshgrid(np.arange(n[0] + 2), np.arange(n[1] + 2), np.arange(n[2] + 1),
                          indexing="ij")
    r2 = (i - 0.5 - c["center"][0]) ** 2 + (j - 0.5 - c["center"][1]) ** 2 + (k - c["center"][2]) ** 2
    A = c["amplitude"] * c["width"] * np.exp(-r2 / c["width"] ** 2)
    E = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1, 3))
    E[..., 0] = A[:-1, 1:, :] - A[:-1, :-1, :]
    E[..., 1] = -(A[1:, :-1, :] - A[:-1, :-1, :])
    return E, np.zeros_like(E)


# BASELINE configuration 1 at full size: the 32^3 periodic thermal plasma,
# h = 0.05 c/omega_p, Courant 0.5, electrons at 8 markers per cell placed by
# ranmar (seeds 1802, 9373) with u_th = 0.01 per axis, 200 steps.
THERMAL_C1 = dict(n=(32, 32, 32), tau=-0.5, bc=(0, 0, 0), ppc=8, uth=(0.01, 0.01, 0.01),
                  steps=200, sample_every=64)


def thermal_c1_markers(h):
    import oracle_port
    c = THERMAL_C1
    return oracle_port.place(lo=(0, 0, 0), hi=c["n"], ppc=c["ppc"], rho=-N_CR / c["ppc"], qDivM=-1.0,
                             h=h, uth=c["uth"], seed=(1802, 9373))


# BASELINE configuration 2's grid and foil: 256 x 128 x 128 cells at 20 per
# wavelength, Courant 0.5, Mur on every face, a 30 n_cr foil 10 cells thick
# with 5-cell transverse margins, electrons and protons at 16 markers per
# cell each (4 455 680 markers).  The foil is warm (u_th 0.2 for electrons,
# 0.2 sqrt(m_e/m_p) for protons) so that its currents build fields from rest
# (a cold foil without a laser never moves); 10 steps.
FOIL_C2 = dict(n=(256, 128, 128), h=0.05, tau=-0.5, bc=(2, 2, 2), lo=(120, 5, 5), hi=(130, 123, 123),
               ppc=16, density=30.0, uth_e=0.2, steps=10, sample_every=1024)


def foil_c2_markers(h):
    import oracle_port
    c = FOIL_C2
    each = int(np.prod([b - a for a, b in zip(c["lo"], c["hi"])])) * c["ppc"]
    up = c["uth_e"] / math.sqrt(1836.0)
    e = oracle_port.place(lo=c["lo"], hi=c["hi"], ppc=c["ppc"], rho=-c["density"] * N_CR / c["ppc"],
                          qDivM=-1.0, h=h, uth=(c["uth_e"],) * 3, seed=(1802, 9373), skip=0, id0=1)
    p = oracle_port.place(lo=c["lo"], hi=c["hi"], ppc=c["ppc"], rho=c["density"] * N_CR / c["ppc"],
                          qDivM=1.0 / 1836, h=h, uth=(up,) * 3, seed=(1802, 9373), skip=7 * each,
                          id0=1 + each)
    return np.concatenate([e, p])


def field_sample(n, count, seed, box=None):
    """A fixed set of `count` node indices (i, j, k) of the checkpoint
    region [0, n]^3, or of a box ((lo), (hi)) inside it, from a seeded
    generator: the nodes a golden file stores and a test compares."""
    rng = np.random.default_rng(seed)
    lo, hi = box if box else ((0, 0, 0), n)
    return np.stack([rng.integers(lo[a], hi[a] + 1, size=count) for a in range(3)], axis=1)


def shell_spectrum(F, n):
    """Power spectrum of each component of a periodic field over
    [0, n)^3, summed over shells of integer |k| (k in index units): an
    array (components, shells)."""
    F = np.asarray(F)[:n[0], :n[1], :n[2]]
    k = np.meshgrid(*[np.fft.fftfreq(n[a]) * n[a] for a in range(3)], indexing="ij")
    shell = np.rint(np.sqrt(k[0] ** 2 + k[1] ** 2 + k[2] ** 2)).astype(int).ravel()
    out = []
    for c in range(F.shape[-1]):
        p = np.abs(np.fft.fftn(F[..., c])) ** 2
        out.append(np.bincount(shell, weights=p.ravel()))
    return np.array(out)
