"""TF/SF interface (core/em_TFSF.c): the oracle against the reference's
record and play runs in tests/golden/tfsf.npz (made by
tests/golden/make_golden.py make_tfsf)."""
import os
import sys

import numpy as np
import pytest

import oracle_port
import parity
import refrun

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "tfsf.npz"))
BC = (2, 2, 2)


def raw(key):
    return bytes(GOLD[key])


def streams(prefix):
    """(headers (24, 11), frames (k, frame size)) of the 24 face streams."""
    heads, data = [], []
    for k in refrun.TFSF_FACES:
        h, f = refrun.read_tfsf_stream(raw(prefix + k))
        heads.append(h)
        data.append(f)
    return np.array(heads), np.concatenate(data, axis=1)


def box_cfg(mode, frames=0, open_faces=((0, 0, 0), (0, 0, 0))):
    b = make_golden.TFSF_BOX
    return dict(lo=(b[0], b[2], b[4]), hi=(b[1], b[3], b[5]), mode=mode, open=open_faces, frames=frames)


def oracle(markers=None):
    h, tau = tuple(GOLD["h"]), float(GOLD["tau"])
    o = oracle_port.OracleRun(make_golden.TFSF_N, h, tau, BC, BC)
    o.set_fields(np.zeros(o.shape()), np.zeros(o.shape()))
    o.set_markers(markers if markers is not None else np.zeros(0, oracle_port.MARKER_DTYPE))
    return o, h


def defrag(stream):
    """The reference TFSFdefrag (source/TFSFdefrag/main.c:159-283) for one
    recording rank and no filter: the header keeps only the face region,
    every value is 0.0 + the recorded one."""
    head, frames = refrun.read_tfsf_stream(stream)
    out = np.zeros(11, "<i4")
    out[:6] = head[:6]
    return out.tobytes() + (0.0 + frames).astype("<f8").tobytes()


def test_record_streams_match_the_reference():
    o, h = oracle()
    o.set_gauss_spot(**make_golden.tfsf_spot(h))
    o.set_tfsf(**box_cfg(oracle_port.TFSF_REC))
    o.init()
    o.step(make_golden.TFSF_STEPS)
    heads, want = streams("rec/")
    regions = o.tfsf_faces()
    assert np.array_equal(regions, heads[:, :6])
    assert np.all(heads[:, 6:] == [0, 1, 0, 0, 0])           # cpu, barcode = record, wrap
    got = o.tfsf_recorded()
    assert got.shape == want.shape == (make_golden.TFSF_STEPS, want.shape[1])
    assert parity.rel_err(got, want) < 1e-13
    assert np.frombuffer(raw("rec/lastFrameTime.bin"), "<i4")[0] == make_golden.TFSF_STEPS


def test_defrag_restatement_matches_the_reference_merge():
    for k in refrun.TFSF_FACES:
        assert defrag(raw("rec/" + k)) == raw("merged/" + k), k


def merged_frames():
    _, frames = streams("merged/")
    return frames


@pytest.mark.parametrize("mode", [0, 2])
def test_play_matches_the_reference(mode):
    o, h = oracle(make_golden.tfsf_plasma(tuple(GOLD["h"])) if mode == 0 else None)
    frames = merged_frames()
    o.set_tfsf(**box_cfg(mode, frames=len(frames)), frames_data=frames)
    o.init()
    rows = o.step(make_golden.TFSF_STEPS)
    E, H = o.fields()
    wantE = np.frombuffer(raw("play%d/E" % mode), "<f8").reshape(E.shape)
    assert parity.rel_err(E, wantE) < 1e-12
    if mode == 0:
        wantH = np.frombuffer(raw("play0/H"), "<f8").reshape(H.shape)
        assert parity.rel_err(H, wantH) < 1e-12
        d = np.frombuffer(raw("play0/diag"), "<f8").reshape(-1, 10)
        np.testing.assert_allclose(d[:, 1:6], rows[1:, :5], rtol=5e-6, atol=1e-12)


def test_play_rejects_faces_near_walls():
    o, _ = oracle()
    cfg = box_cfg(0, frames=1)
    cfg["hi"] = (13, 8, 8)                  # H face x = 14 > 18 - 5
    with pytest.raises(ValueError):
        o.set_tfsf(**cfg, frames_data=np.zeros((1, 10 ** 4)))
