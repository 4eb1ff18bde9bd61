"""The reference's per-frame load-path schedule (warm_struct / warm_step and the sweep loop of `structural`,
src/lib.rs:1061-1079, 1268-1281) on the GPU, through the C ABI, against the oracle's restatement of the same schedule.

Both sides sweep red-black in FP64; the schedule decides per frame which structures sweep, how many times, with
which relaxation and from which brick-update budget (160,000 for the structural loop, shared in order; 120,000 for
the warm-up), and which structures' joints are live. Per frame the sweep counts, the live joint pass's counts and
largest ratio, every structure's pending warm-up, settle timer and last residual must be identical, and every ten
frames the potentials and the bonds (after fatigue and failures).
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def run_frames(sf, oracle, sc, frames, warm_at=None, active=None):
    ids = sc.structure_ids()
    active = ids if active is None else active
    warm_at = warm_at or {s: 1 for s in ids}
    w = sf.World(sc)
    ow = oracle.OracleWorld(sc)
    totals = [0, 0, 0]
    for f in range(1, frames + 1):
        for s, at in warm_at.items():
            if at == f:
                w.structure_warm(s)
                ow.structure_warm(s)
        rep = w.structure_frame(f, active, dt=DT)
        osw, ows, olive, oj, oover, ofail, ocrush, omr = ow.structure_frame(f, DT, active)
        assert (rep.sweeps, rep.warm_sweeps) == (osw, ows), f
        assert (rep.live, rep.joints, rep.over, rep.failed, rep.crushed) == (olive, oj, oover, ofail, ocrush), f
        assert rep.max_ratio == omr, f
        totals[0] += osw
        totals[1] += ows
        totals[2] += olive
        gw, gs, gt, gr = w.structure_state()
        n = len(gw)
        owarm, osol, oset, ores = ow.structure_state(n)
        np.testing.assert_array_equal(gw, owarm, err_msg=f"frame {f}")
        np.testing.assert_array_equal(gs, osol, err_msg=f"frame {f}")
        np.testing.assert_array_equal(gt, oset, err_msg=f"frame {f}")
        np.testing.assert_array_equal(gr, ores, err_msg=f"frame {f}")
        if f % 10 == 0 or f == frames:
            np.testing.assert_array_equal(w.phi64(), ow.phi64(), err_msg=f"frame {f}")
            b, _, _ = w.bonds()
            ob, _ = ow.bonds()
            np.testing.assert_array_equal(b, ob, err_msg=f"frame {f}")
    w.close()
    return totals


def test_frames_many_structures(sf, oracle):
    """Eight structures of 88-1,364 bricks, warmed at different frames: the warm-up budget carries over from frame
    to frame, the structural loop runs 6 sweeps (then more) for unsettled structures and 1 or 0 once converged."""
    sc = S.structure_lattice(scale=0.05, n_struct=8)
    ids = sc.structure_ids()
    warm_at = {s: 1 + 3 * k for k, s in enumerate(ids)}
    sw, ws, live = run_frames(sf, oracle, sc, 60, warm_at=warm_at)
    assert ws == 560 * len(ids) and sw > 0 and live > 0


def test_frames_frame_and_tower(sf, oracle):
    """The 5-storey frame (3,150 bricks: budget-limited warm-up of 38 sweeps a frame) and the 16-storey tower
    (47,760 bricks: over 15,000, one structural sweep a frame until converged) in one lattice."""
    frame, _ = S.frame5_structure()
    tower, rm = S.tower16_structure()
    tower = tower.without_static(rm)
    # the tower beside the frame: shift it 60 cells along x and give it structure id 1
    xyz = np.concatenate([frame.static_xyz, tower.static_xyz + np.array([60, 0, 0], np.int32)])
    sc = S.Scene(xyz, np.concatenate([frame.static_mat, tower.static_mat]),
                 np.concatenate([frame.static_sid, tower.static_sid + 1]).astype(np.int32),
                 np.concatenate([frame.static_infill, tower.static_infill])).contiguous()
    sw, ws, live = run_frames(sf, oracle, sc, 40)
    assert ws > 0 and sw > 0
