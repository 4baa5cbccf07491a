"""The oracle's restatement of the reference's update schedule, on CPU: the frozen-link
mask of the L_core block faces (src/geometry/GeometryCB.cpp:33-56) after a cumulative
shift, and the shift draws of mpi::shift::random_shift (src/mpi/Shift.cpp:163-172)."""
import numpy as np

import oracle as orc


def test_frozen_mask_count_and_unshifted_faces():
    dims, lcore = (4, 4, 4, 4), 2
    u = orc.hot_philox(dims, 1)
    for shift in ((0, 0, 0, 0), (1, 0, 1, 0)):
        out, fails = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 7, 0, lcore, shift)
        assert fails == 0
        changed = np.any(np.abs(out - u) > 0, axis=(-2, -1))  # (t, z, y, x, mu)
        # per direction: 4 values along mu x 2 of 4 values in each of the 3 other directions
        assert int(changed.sum()) == 4 * 4 * 2 ** 3
        for mu in range(4):
            c = changed[..., mu]
            coords = np.argwhere(c)[:, ::-1]  # (x, y, z, t)
            others = [d for d in range(4) if d != mu]
            assert np.all((coords[:, others] + np.array(shift)[others]) % lcore != 0)


def test_frozen_with_core_equal_to_lattice_is_reference_one_rank():
    # one block of edge L: only the links on the c_d = 0 faces (d != mu) are frozen
    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 2)
    out, _ = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 3, 0, 4, (0, 0, 0, 0))
    changed = np.any(np.abs(out - u) > 0, axis=(-2, -1))
    assert int(changed.sum()) == 4 * 4 * 3 ** 3


def test_shift_sequence_range_and_determinism():
    a = orc.shift_sequence(1234, 4, 50)
    b = orc.shift_sequence(1234, 4, 50)
    assert a.shape == (50, 4) and np.array_equal(a, b)
    assert a.min() >= 0 and a.max() <= 3 and len(np.unique(a)) == 4
    assert not np.array_equal(a, orc.shift_sequence(1235, 4, 50))
