"""Raw binary state dumps (dndsr_b200/checkpoint.py): bit-exact round trips of (u, uRec) from numpy and torch,
the header's shape checks, and the hand-off of a dumped state to the CPU oracle."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from dndsr_b200.checkpoint import load_state, save_state
from tests.util import oracle_for


def test_round_trip_is_bit_exact(tmp_path):
    rng = np.random.default_rng(0)
    u, uRec = rng.normal(size=(37, 5)), rng.normal(size=(37, 9, 5))
    p = str(tmp_path / "state.bin")
    save_state(p, u, uRec, step=12, t=0.25, note="x")
    a, b, meta = load_state(p)
    assert a.tobytes() == u.tobytes() and b.tobytes() == uRec.tobytes()
    assert meta == {"step": 12, "t": 0.25, "note": "x"}
    save_state(p, torch.tensor(u), torch.tensor(uRec))
    ta, tb, _ = load_state(p, device="cpu")
    assert torch.equal(ta, torch.tensor(u)) and torch.equal(tb, torch.tensor(uRec))


def test_shape_and_format_checks(tmp_path):
    p = str(tmp_path / "s.bin")
    with pytest.raises(ValueError):
        save_state(p, np.zeros((4, 5)), np.zeros((4, 3, 6)))
    with pytest.raises(ValueError):
        save_state(p, np.zeros((4, 5), np.float32), np.zeros((4, 3, 5)))
    save_state(p, np.zeros((4, 5)), np.zeros((4, 3, 5)))
    with open(p, "ab") as fh:
        fh.write(b"\0" * 8)
    with pytest.raises(ValueError):
        load_state(p)


def test_oracle_hand_off(tmp_path):
    m = M.tgv_mesh(4)
    o = oracle_for(m, 2, "HLLEP", 1e-3)
    u = o.init_field(3)
    rng = np.random.default_rng(1)
    uRec = rng.normal(size=(m.n_cell, o.R, 5)) * 1e-3
    p = str(tmp_path / "tgv.bin")
    save_state(p, u, uRec, case="tgv4")
    a, b, _ = load_state(p)
    assert np.array_equal(o.eval_rhs(a, b), o.eval_rhs(u, uRec))
