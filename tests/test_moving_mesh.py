"""Moving mesh and solidification parameters: deck, C ABI and GPU parity.

The oracle's moving mesh (zone shift with the beam, grid rebuild, the in-place
x-then-y remap of the solution fields) and G/R are pinned bit for bit to the
compiled reference by tests/test_oracle.py (golden g_moving towards +x/+y,
live v_moving towards -x/-y, grids compared every step).  Here the CUDA path
runs the same decks: FP64 exact order takes the oracle's outer iterations in
every step, the grid is identical, and every field -- the remapped ones, G and
R included -- is within 1e-8 relative L2.
"""
import numpy as np
import pytest

from conftest import rel_l2

FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl", "hnot", "pp", "grad", "rate")


def test_deck_carries_moving_zones_and_gr(deckdir):
    import amcfd
    import amcfd_decks as D
    p = amcfd.Deck(D.moving_track("mv_parse").write(deckdir)).params
    assert (p.movingmesh, p.xmoveindex, p.ymoveindex, p.solidification) == (1, 1, 1, 1)


def test_create_rejects_a_moving_zone_without_neighbours(deckdir):
    import ctypes as C

    import amcfd
    import amcfd_decks as D
    d = D.moving_track("mv_bad")
    d.moving_mesh = (1, 2)  # the first x zone has no zone before it
    deck = amcfd.Deck(d.write(deckdir))
    h = C.c_void_p()
    assert amcfd.lib().amcfd_create(C.byref(deck.params), None, C.byref(h)) == -1
    amcfd.lib().amcfd_destroy(h)


def _pair(deck, deckdir, **kw):
    import amcfd
    import oracle_py
    d = amcfd.Deck(deck.write(deckdir))
    return amcfd.Solver(d, **kw), oracle_py.Oracle(d.params)


@pytest.mark.gpu
@pytest.mark.parametrize("reverse", [False, True])
def test_moving_mesh_exact_fp64_steps(reverse, deckdir):
    import amcfd
    import amcfd_decks as D
    gpu, orc = _pair(D.moving_track("mv_exact", reverse=reverse), deckdir, order=amcfd.ORDER_EXACT,
                     precision=amcfd.PREC_FP64)
    x0 = gpu.grid("x").copy()
    for s in range(6):
        rg, ro = gpu.step(), orc.step()
        where = f"reverse={reverse} step {s + 1}"
        for k in ("niter", "steadylength", "istat", "iend", "jstat", "jend", "kstat", "jstart"):
            assert rg[k] == ro[k], (where, k, rg[k], ro[k])
        for g in ("x", "y"):
            assert np.array_equal(gpu.grid(g), orc.field(g)), (where, g)
        for f in FIELDS:
            a, b = gpu.get(f), orc.field(f)
            if np.linalg.norm(b) == 0:
                assert np.abs(a).max() < 1e-12, (where, f)
            else:
                assert rel_l2(a, b) < 1e-8, (where, f, rel_l2(a, b))
    assert not np.array_equal(gpu.grid("x"), x0)  # the mesh did move
    assert np.abs(gpu.get("grad")).max() > 0
    gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,order", [(0, 0), (1, 1)])
def test_moving_mesh_graph_replay_bit_identical(prec, order, deckdir):
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.moving_track("mv_graphs", steps=4).write(deckdir))
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=0)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=1)
    for s in range(4):
        ra, rb = a.step(), b.step()
        assert ra["niter"] == rb["niter"], s
        for f in ("temp", "uvel", "grad"):
            assert np.array_equal(a.get(f), b.get(f), equal_nan=True), (s, f)
    a.close()
    b.close()
