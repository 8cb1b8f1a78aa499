"""Checkpoint / restart in the reference's raw format (src/io.jl:6-72).

* the file written from the device has the reference's header (magic, n_cons,
  n_global, n_local, coords, t, step, little-endian) followed by the interior
  of Q in Julia order, equal to the solver's state;
* a round trip restores state and clock, and a restart continues bitwise like
  the uninterrupted run;
* a file built here by the reference's layout loads on the device;
* mismatches are refused with the reference's messages.
"""
import struct

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import scenarios

pytestmark = pytest.mark.gpu

MAGIC = 0x434C4553434B5054
HEADER = struct.calcsize("<Q10qdq")   # 104 bytes


def _case():
    return scenarios.two_species_tube((cl.lele_d1_6(), cl.compact_filter(0.45)), 200, 5.0, 0.3)


def test_checkpoint_file_layout(tmp_path):
    d, Q0, tf = _case()
    S = cl.Solver(d)
    S.set_state(Q0)
    S.run(tf, 7)
    S.save_checkpoint(tmp_path / "tube")
    raw = (tmp_path / "tube.r0000.ckpt").read_bytes()
    magic, ncons, g1, g2, g3, l1, l2, l3, c1, c2, c3, t, step = struct.unpack("<Q10qdq", raw[:HEADER])
    assert magic == MAGIC and ncons == 6
    assert (g1, g2, g3) == (200, 1, 1) and (l1, l2, l3) == (200, 1, 1) and (c1, c2, c3) == (0, 0, 0)
    assert t == S.t and step == 7
    data = np.frombuffer(raw[HEADER:], dtype="<f8")
    assert data.size == 6 * 200
    want = S.get_state(layout="interior")
    assert np.array_equal(data.reshape(want.shape), want)


def test_round_trip_and_restart(tmp_path):
    # test/runtests.jl:1866-1878, then a continuation: with artificial
    # properties off the step size depends on the state alone, so the
    # restarted run continues bitwise (with them on, max_rate reads the
    # previous stage's coefficients, which a checkpoint does not hold)
    d = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, cl.lele_d1_6(), cl.compact_filter(0.45),
                       art=cl.ArtParams(enabled=False))
    Q0 = cl.initialize(d, lambda x, y, z: cl.Prim(u=(np.sin(x), 0.0 * y, 0.0 * z), p=1 + 0.1 * np.cos(y),
                                                  rho=1.0 + 0 * x))
    R = cl.Solver(d)
    R.set_state(Q0)
    R.set_clock(0.37, 42, 0.5)
    R.save_checkpoint(tmp_path / "rt")
    R2 = cl.Solver(d)
    R2.load_checkpoint(tmp_path / "rt")
    assert R2.t == 0.37 and R2.steps == 42
    assert np.array_equal(R2.get_state(layout="interior"), R.get_state(layout="interior"))
    A = cl.Solver(d)
    A.set_state(Q0)
    A.run(1e9, 10)
    A.save_checkpoint(tmp_path / "a")
    A.run(1e9, 25)
    B = cl.Solver(d)
    B.load_checkpoint(tmp_path / "a")
    assert B.steps == 10
    B.run(1e9, 25)
    assert B.steps == 25 and B.t == A.t
    assert np.array_equal(A.get_state(), B.get_state())


def test_reference_layout_loads(tmp_path):
    d, Q0, tf = _case()
    S = cl.Solver(d)
    S.set_state(Q0)
    interior = S.get_state(layout="interior")
    rng = np.random.default_rng(5)
    Q = interior * (1 + 1e-3 * rng.standard_normal(interior.shape))
    hdr = struct.pack("<Q10qdq", MAGIC, 6, 200, 1, 1, 200, 1, 1, 0, 0, 0, 0.125, 42)
    (tmp_path / "ref.r0000.ckpt").write_bytes(hdr + Q.astype("<f8").tobytes())
    T = cl.Solver(d)
    T.load_checkpoint(tmp_path / "ref")
    assert T.t == 0.125 and T.steps == 42
    assert np.array_equal(T.get_state(layout="interior"), Q)


def test_mismatches_are_refused(tmp_path):
    d, Q0, tf = _case()
    S = cl.Solver(d)
    S.set_state(Q0)
    S.save_checkpoint(tmp_path / "a")
    raw = (tmp_path / "a.r0000.ckpt").read_bytes()
    cases = {
        "not a CompactLES checkpoint": struct.pack("<Q", 1) + raw[8:],
        "conserved layout mismatch": raw[:8] + struct.pack("<q", 5) + raw[16:],
        "global grid mismatch": raw[:16] + struct.pack("<q", 201) + raw[24:],
        "decomposition mismatch": raw[:40] + struct.pack("<q", 100) + raw[48:],
        "rank layout mismatch": raw[:64] + struct.pack("<q", 1) + raw[72:],
    }
    for msg, blob in cases.items():
        (tmp_path / "bad.r0000.ckpt").write_bytes(blob)
        with pytest.raises(cl.ClesError, match=msg):
            S.load_checkpoint(tmp_path / "bad")
    with pytest.raises(cl.ClesError, match="cannot open"):
        S.load_checkpoint(tmp_path / "missing")
