"""Setup tags on the device (row f-4): the restatements the device follows
against the reference's own outputs in tests/golden/setup_tags.npz
([DF:two-stream] and [velocity shift] through setup.out, [DF:uniform]
through oracle/_ref/df_uniform.out), and the C library's rand () the
[DF:uniform] tag draws from."""
import ctypes
import math
import os
import sys

import numpy as np

import refrun

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "setup_tags.npz"))


def libc_rand(n, skip=0):
    """n draws of the C library's rand () from its default seed, after skip."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    for _ in range(skip):
        libc.rand()
    return np.array([libc.rand() for _ in range(n)], dtype=np.int64)


def glibc_rand(n, skip=0):
    """The published additive feedback generator of the GNU C library's
    random(3) with seed 1 (the device's restatement)."""
    r = [1]
    for i in range(1, 31):
        r.append(16807 * r[-1] % 2147483647)
    r += r[0:3]
    out = []
    i = 34
    while len(out) < n + skip:
        r.append((r[i - 3] + r[i - 31]) % (1 << 32))
        if i >= 344:
            out.append(r[i] >> 1)
        i += 1
    return np.array(out[skip:], dtype=np.int64)


def df_uniform(c, n, draws):
    """setup/tag_DF_uniform.c:36-70 over n markers from the draws."""
    rho_crit = 4 * math.pi ** 2          # e n_cr/rho0 is 4 pi^2 at every wavelength
    f = draws.reshape(n, 3) / 2147483647.0
    u = np.array(c["u"]) + (f - 0.5) * np.array(c["du"])
    rho = np.float32(c["rho"] * (rho_crit / make_golden.DF_PPC))
    return u, rho


def test_published_generator_is_the_c_library_rand():
    assert np.array_equal(glibc_rand(2000, 17), libc_rand(2000, 17))


def test_df_uniform_matches_the_reference_tag():
    for q, c in enumerate(make_golden.DF_CASES):
        want = GOLD["df%d" % q]
        n = len(want)
        u, rho = df_uniform(c, n, glibc_rand(3 * n, c["skip"]))
        assert np.array_equal(u, want[:, :3])
        assert np.allclose(want[:, 3], rho, rtol=1e-6)
        assert np.all(want[:, 4] == np.float32(c["qDivM"]))


def two_stream(h, L):
    """setup/tag_twoStream.c:23-103 in its order."""
    N, m, g, qm = make_golden.TS["N"], make_golden.TS["m"], make_golden.TS["gamma"], make_golden.TS["qDivM"]
    rho = g * g / qm
    k = [2 * math.pi * m[a] / L[a] for a in range(3)]
    kabs = math.sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2])
    V = g * math.sqrt(3.0) / (2 * kabs)
    v = [V * k[a] / kabs for a in range(3)]
    rho *= L[0] * L[1] * L[2] / (h[0] * h[1] * h[2] * (N[0] * N[1] * N[2]))
    d = [L[a] / float(N[a]) for a in range(3)]
    out = np.zeros(2 * N[0] * N[1] * N[2], refrun.MARKER_DTYPE)
    q = 0
    for i in range(N[0]):
        for j in range(N[1]):
            for kk in range(N[2]):
                for s in (1.0, -1.0):
                    out[q] = ((i + 0.5) * d[0], (j + 0.5) * d[1], (kk + 0.5) * d[2], s * v[0], s * v[1],
                              s * v[2], rho, qm, q + 1, 0)
                    q += 1
    return out


def markers(key):
    return np.frombuffer(GOLD[key].tobytes(), refrun.MARKER_DTYPE)


def test_two_stream_and_shift_match_setup():
    h, L = GOLD["domain"][:3], GOLD["domain"][3:]
    want = two_stream(h, L)
    got = markers("two_stream0")
    for f in ("x", "y", "z", "vx", "vy", "vz", "rho", "qDivM", "id"):
        assert np.array_equal(got[f], want[f]), f
    shifted = markers("two_stream1")
    for a, f in enumerate(("vx", "vy", "vz")):
        assert np.array_equal(shifted[f], got[f] + make_golden.TS["dv"][a]), f
