"""Collection of particles by internal electrodes in the CPU oracle: the edge
bit arrays derived from a Dirichlet mask and the crossing rule (a line is
crossed when a drift passes it or ends on it, not when it starts on it)."""
import numpy as np

from oracle import oracle as O


def cathode_mask(m=17, n=17, x=4, top=8):
    mask = np.zeros((n, m), np.uint8)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    mask[0:top + 1, x] = 1  # a vertical electrode from the bottom wall to y = top
    return mask.reshape(-1)


def test_edges_of_a_line_electrode():
    m = n = 17
    vb, hb = O.electrode_bits(cathode_mask(), m, n)
    on = [k for k in range(m * (n - 1)) if (vb[k >> 5] >> (k & 31)) & 1]
    # vertical edges (x = 4, j .. j + 1) for j = 0 .. 7, the first touching the wall
    assert on == [4 * (n - 1) + j for j in range(8)]
    assert not hb.any()


def test_crossing_rule():
    m = n = 17
    vb, hb = O.electrode_bits(cathode_mask(), m, n)
    hit = lambda *p: O.hits_electrode(*p, m, n, vb, hb)
    assert hit(3.9, 2.5, 4.1, 2.6)       # through the electrode
    assert not hit(3.9, 9.5, 4.1, 9.6)   # above its end
    assert hit(4.2, 3.0, 3.95, 3.1)      # moving in -x
    assert not hit(4.0, 3.0, 3.5, 3.0)   # starting on it
    assert hit(3.5, 3.0, 4.0, 3.0)       # ending on it
    assert hit(3.9, 0.5, 4.1, 0.5)       # the segment that meets the wall
    assert not hit(3.2, 2.0, 3.8, 2.5)   # no grid line crossed


def test_drift_counts_walls_and_electrodes_apart():
    m = n = 17
    vb, hb = O.electrode_bits(cathode_mask(), m, n)
    gx = np.array([3.9, 15.9, 3.0, np.nan], np.float32)
    gy = np.array([2.5, 5.0, 12.0, np.nan], np.float32)
    vx = np.array([2e5, 2e5, 1e5, 0.0], np.float32)
    vy = np.zeros(4, np.float32)
    a, c = O.drift_absorb_electrodes_f32(gx, gy, vx, vy, 1e-6, 1e-6, m, n, vb, hb)
    assert (a, c) == (1, 1)
    assert np.isnan(gx[0]) and np.isnan(gx[1]) and gx[2] == np.float32(3.1)
