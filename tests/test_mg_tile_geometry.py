"""The halo geometry of the multigrid's two-level launches, on the CPU.

k_mg_down2 and k_mg_up2 (pic_b200/csrc/multigrid.cu) work two levels in one
CTA over halos that must be wide enough for the CTA's tile to come out as the
separate per-level launches give it.  This test emulates both in FP64 numpy
with the kernels' halo and window formulas (Down2Geom, Up2Geom) and the same
red-black order, restriction and prolongation, and checks every value a tile
stores against the same phases run over the whole grid:
  down: the fine tile's smoothed e, the coarse tile's g and e, and the
        coarser level's restricted g on the tile's nodes;
  up:   the fine tile's corrected and smoothed e.
Grids of 129^2 and 97 x 65 nodes with an electrode on an odd line, tiles at
corners, edges and the interior, one to three sweeps.
"""
import numpy as np
import pytest

TILE = 32


def geometry(S):
    """The tile geometry of the library's multigrid kernels for S sweeps (pic_mg_tile_geometry)."""
    import ctypes

    from pic_b200 import _lib

    out = (ctypes.c_int * _lib.PIC_MG_GEOMETRY_VALUES)()
    _lib.call("pic_mg_tile_geometry", S, out)
    g = list(out)
    assert g[0] == TILE
    return {"down": g[1:3], "up": g[3:6], "up_res": g[6:9], "down2": g[9:13], "up2": g[13:18]}


def test_geometry_is_the_library_s():
    """The kernels' halos are what each phase needs: the down phase one node
    per half-sweep plus two (residual and restriction), the up phase one per
    half-sweep (one more with the residual update), and the two-level launches
    as the emulations below require; these emulations use the library's values."""
    for S in range(1, 9):
        g = geometry(S)
        assert g["down"] == [2 * S + 2, TILE + 2 * (2 * S + 2)]
        assert g["up"][:2] == [2 * S, TILE + 4 * S] and g["up_res"][:2] == [2 * S + 1, TILE + 4 * S + 2]
        assert g["down2"][0] == g["down"][0] and g["down2"][1] == TILE // 2 + 2 * g["down2"][0]


def coarse_mask(mf, fx, fy):
    """pic_mg_create's rule: a coarse node is Dirichlet if its injected fine node
    is, or an internal Dirichlet node lies in its 3 x 3 fine neighbourhood."""
    cx, cy = (fx - 1) // 2 + 1, (fy - 1) // 2 + 1
    inner = np.zeros((fy, fx), bool)
    inner[1:-1, 1:-1] = mf[1:-1, 1:-1] != 0
    mc = np.zeros((cy, cx), np.uint8)
    for J in range(cy):
        for I in range(cx):
            v = mf[2 * J, 2 * I] != 0
            if not v:
                v = inner[max(0, 2 * J - 1):2 * J + 2, max(0, 2 * I - 1):2 * I + 2].any()
            mc[J, I] = 1 if v else 0
    return mc


def dirichlet(m):
    """Edges and mask, as the kernels treat them (outside the grid Dirichlet)."""
    d = m.astype(bool).copy()
    d[0, :] = d[-1, :] = d[:, 0] = d[:, -1] = True
    return d


def half_sweep(e, g, fixed, color, gx, gy, c, omega):
    """One red-black half-sweep over the nodes of global parity `color` that are
    not fixed (gx, gy: the nodes' global coordinates)."""
    sel = ((gx + gy) & 1) == color
    sel[0, :] = sel[-1, :] = sel[:, 0] = sel[:, -1] = False
    sel &= ~fixed
    cx, cy, inv = c
    nb = np.zeros_like(e)
    nb[1:-1, 1:-1] = cx * (e[1:-1, :-2] + e[1:-1, 2:]) + cy * (e[:-2, 1:-1] + e[2:, 1:-1])
    upd = (nb - g) * inv
    e[sel] = e[sel] + omega * (upd[sel] - e[sel])


def sweeps(e, g, fixed, ox, oy, c, omega, S):
    gy, gx = np.mgrid[oy:oy + e.shape[0], ox:ox + e.shape[1]]
    for _ in range(S):
        for color in (0, 1):
            half_sweep(e, g, fixed, color, gx, gy, c, omega)


def residual(e, g, fixed, c):
    cx, cy, _ = c
    r = np.zeros_like(e)
    lap = cx * (e[1:-1, :-2] + e[1:-1, 2:] - 2 * e[1:-1, 1:-1]) + cy * (e[:-2, 1:-1] + e[2:, 1:-1] - 2 * e[1:-1, 1:-1])
    r[1:-1, 1:-1] = g[1:-1, 1:-1] - lap
    r[fixed] = 0.0
    return r


def restrict_at(r, I, J, ox, oy):
    """Full weighting of r (a tile at (ox, oy), fixed nodes already zero) at coarse node (I, J)."""
    y, x = 2 * J - oy, 2 * I - ox
    return (0.25 * r[y, x] + 0.125 * (r[y, x - 1] + r[y, x + 1] + r[y - 1, x] + r[y + 1, x])
            + 0.0625 * (r[y - 1, x - 1] + r[y - 1, x + 1] + r[y + 1, x - 1] + r[y + 1, x + 1]))


def prolong_add(e, fixed, sc, ox, oy, cox, coy):
    """Bilinear prolongation of the coarse window sc (origin (cox, coy)) added on the free nodes of e."""
    H, W = e.shape
    for lj in range(H):
        for li in range(W):
            if fixed[lj, li]:
                continue
            i, j = ox + li, oy + lj
            a, b = (j >> 1) - coy, (i >> 1) - cox
            if not (i & 1) and not (j & 1):
                v = sc[a, b]
            elif (i & 1) and not (j & 1):
                v = 0.5 * (sc[a, b] + sc[a, b + 1])
            elif not (i & 1) and (j & 1):
                v = 0.5 * (sc[a, b] + sc[a + 1, b])
            else:
                v = 0.25 * (sc[a, b] + sc[a, b + 1] + sc[a + 1, b] + sc[a + 1, b + 1])
            e[lj, li] += v


def window(a, fill, oy, ox, h, w):
    """a[oy:oy+h, ox:ox+w] with `fill` outside a."""
    out = np.full((h, w), fill, dtype=a.dtype)
    y0, x0 = max(oy, 0), max(ox, 0)
    y1, x1 = min(oy + h, a.shape[0]), min(ox + w, a.shape[1])
    if y1 > y0 and x1 > x0:
        out[y0 - oy:y1 - oy, x0 - ox:x1 - ox] = a[y0:y1, x0:x1]
    return out


def coeffs(h):
    cx = cy = 1.0 / (h * h)
    return cx, cy, 1.0 / (2 * (cx + cy))


def problem(fx, fy, seed):
    rng = np.random.default_rng(seed)
    mf = np.zeros((fy, fx), np.uint8)
    mf[fy // 3:2 * fy // 3, 2 * (fx // 5) + 1] = 1  # an electrode on an odd column
    mc = coarse_mask(mf, fx, fy)
    cxn, cyn = mc.shape[1], mc.shape[0]
    m2 = coarse_mask(mc, cxn, cyn)
    gF = rng.normal(0, 1, (fy, fx))
    gF[dirichlet(mf)] = 0.0
    return mf, mc, m2, gF


@pytest.mark.parametrize("S", [1, 2, 3])
@pytest.mark.parametrize("shape", [(129, 129), (97, 65)])
def test_two_level_down_tiles_match_the_levels(shape, S):
    fx, fy = shape
    omega, h = 1.15, 1e-3
    cF, cC = coeffs(h), coeffs(2 * h)
    mf, mc, m2, gF = problem(fx, fy, 3 + S)
    dF, dC, d2 = dirichlet(mf), dirichlet(mc), dirichlet(m2)
    # the separate launches, over the whole grid
    eF = np.zeros_like(gF)
    sweeps(eF, gF, dF, 0, 0, cF, omega, S)
    rF = residual(eF, gF, dF, cF)
    rFp = np.pad(rF, 1)  # restriction at the edges reads zeros outside
    gC = np.zeros(mc.shape)
    for J in range(mc.shape[0]):
        for I in range(mc.shape[1]):
            gC[J, I] = 0.0 if dC[J, I] else restrict_at(rFp, I, J, -1, -1)
    eC = np.zeros_like(gC)
    sweeps(eC, gC, dC, 0, 0, cC, omega, S)
    rC = np.pad(residual(eC, gC, dC, cC), 1)
    g2 = np.zeros(m2.shape)
    for J in range(m2.shape[0]):
        for I in range(m2.shape[1]):
            g2[J, I] = 0.0 if d2[J, I] else restrict_at(rC, I, J, -1, -1)
    # the two-level down launch's tile geometry, as the library's kernels use it
    HC, WC, HF, WF = geometry(S)["down2"]
    tiles_x, tiles_y = -(-fx // TILE), -(-fy // TILE)
    for ty, tx in {(0, 0), (tiles_y - 1, tiles_x - 1), (0, tiles_x // 2), (tiles_y // 2, tiles_x // 2)}:
        x0, y0 = tx * TILE, ty * TILE
        ox, oy = x0 - HF, y0 - HF
        fixF = window(dF, True, oy, ox, WF, WF)
        e = np.zeros((WF, WF))
        g = window(gF, 0.0, oy, ox, WF, WF)
        sweeps(e, g, fixF, ox, oy, cF, omega, S)
        core = (slice(HF, HF + TILE), slice(HF, HF + TILE))
        ref = window(eF, 0.0, y0, x0, TILE, TILE)
        inside = window(np.ones_like(eF, bool), False, y0, x0, TILE, TILE)
        np.testing.assert_array_equal(e[core][inside], ref[inside])
        r = residual(e, g, fixF, cF)
        cx0, cy0 = x0 // 2, y0 // 2
        cox, coy = cx0 - HC, cy0 - HC
        fixC = window(dC, True, coy, cox, WC, WC)
        gc = np.zeros((WC, WC))
        for LJ in range(WC):
            for LI in range(WC):
                if not fixC[LJ, LI]:
                    gc[LJ, LI] = restrict_at(r, cox + LI, coy + LJ, ox, oy)
        ccore = (slice(HC, HC + TILE // 2), slice(HC, HC + TILE // 2))
        inC = window(np.ones_like(gC, bool), False, cy0, cx0, TILE // 2, TILE // 2)
        np.testing.assert_array_equal(gc[ccore][inC], window(gC, 0.0, cy0, cx0, TILE // 2, TILE // 2)[inC])
        ec = np.zeros((WC, WC))
        sweeps(ec, gc, fixC, cox, coy, cC, omega, S)
        np.testing.assert_array_equal(ec[ccore][inC], window(eC, 0.0, cy0, cx0, TILE // 2, TILE // 2)[inC])
        rc = residual(ec, gc, fixC, cC)
        for k in range((TILE // 4) ** 2):
            I, J = cx0 // 2 + k % (TILE // 4), cy0 // 2 + k // (TILE // 4)
            if I < m2.shape[1] and J < m2.shape[0] and not d2[J, I]:
                assert restrict_at(rc, I, J, cox, coy) == g2[J, I], (tx, ty, I, J)


@pytest.mark.parametrize("S", [1, 2, 3])
@pytest.mark.parametrize("shape", [(129, 129), (97, 65)])
def test_two_level_up_tiles_match_the_levels(shape, S):
    fx, fy = shape
    omega, h = 1.15, 1e-3
    cF, cC = coeffs(h), coeffs(2 * h)
    mf, mc, m2, gF = problem(fx, fy, 7 + S)
    dF, dC, d2 = dirichlet(mf), dirichlet(mc), dirichlet(m2)
    rng = np.random.default_rng(40 + S)
    # a down-phase state and a correction of the coarsest of the three levels
    eF0 = rng.normal(0, 1, gF.shape)
    eF0[dF] = 0.0
    gC = rng.normal(0, 1, mc.shape)
    gC[dC] = 0.0
    eC0 = rng.normal(0, 1, mc.shape)
    eC0[dC] = 0.0
    e2 = rng.normal(0, 1, m2.shape)
    e2[d2] = 0.0
    # the separate launches, over the whole grid
    eC = eC0.copy()
    prolong_add(eC, dC, np.pad(e2, ((0, 1), (0, 1))), 0, 0, 0, 0)
    sweeps(eC, gC, dC, 0, 0, cC, omega, S)
    eF = eF0.copy()
    prolong_add(eF, dF, np.pad(eC, ((0, 1), (0, 1))), 0, 0, 0, 0)
    sweeps(eF, gF, dF, 0, 0, cF, omega, S)
    # Up2Geom
    HF, WF, CWF, WC, CWC = geometry(S)["up2"]
    tiles_x, tiles_y = -(-fx // TILE), -(-fy // TILE)
    for ty, tx in {(0, 0), (tiles_y - 1, tiles_x - 1), (0, tiles_x // 2), (tiles_y // 2, tiles_x // 2)}:
        x0, y0 = tx * TILE, ty * TILE
        ox, oy = x0 - HF, y0 - HF
        fcx, fcy = ox >> 1, oy >> 1
        cox, coy = fcx - 2 * S, fcy - 2 * S
        c2x, c2y = cox >> 1, coy >> 1
        fixC = window(dC, True, coy, cox, WC, WC)
        ec = np.where(fixC, 0.0, window(eC0, 0.0, coy, cox, WC, WC))
        gc = window(gC, 0.0, coy, cox, WC, WC)
        sc2 = window(e2, 0.0, c2y, c2x, CWC, CWC)
        prolong_add(ec, fixC, sc2, cox, coy, c2x, c2y)
        sweeps(ec, gc, fixC, cox, coy, cC, omega, S)
        fixF = window(dF, True, oy, ox, WF, WF)
        ef = np.where(fixF, 0.0, window(eF0, 0.0, oy, ox, WF, WF))
        gf = window(gF, 0.0, oy, ox, WF, WF)
        prolong_add(ef, fixF, ec, ox, oy, cox, coy)
        sweeps(ef, gf, fixF, ox, oy, cF, omega, S)
        core = (slice(HF, HF + TILE), slice(HF, HF + TILE))
        inside = window(np.ones_like(eF, bool), False, y0, x0, TILE, TILE)
        np.testing.assert_array_equal(ef[core][inside], window(eF, 0.0, y0, x0, TILE, TILE)[inside])
