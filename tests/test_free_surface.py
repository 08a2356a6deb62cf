"""Energy-balance free surface: deck, C ABI and GPU parity against the oracle.

The oracle's free surface (bisection on the pressure multiplier around the
Jacobi energy balance, then the deformed heights zr and the temperatures on
them) is pinned to the compiled reference by tests/test_oracle.py: golden
g_freesurf (zr and tempr bit for bit, the monitor values as printed) and live
v_freesurf (beam switched off after two steps).  Here the CUDA path computes
the same surface after every step of the golden deck: the bisection takes the
same number of iterations, lambda agrees to 1e-12 relative, fi's extremes and
the fields zr and tempr to 1e-8 relative L2.
"""
import numpy as np
import pytest

from conftest import rel_l2


def test_deck_carries_free_surface_row(deckdir):
    import amcfd
    import amcfd_decks as D
    p = amcfd.Deck(D.free_surface_track("fs_parse").write(deckdir)).params
    assert p.freesurface == 1
    assert (p.fs_lam1, p.fs_lam2, p.fs_surftens, p.fs_maxiterenergy) == (-1e5, 1e5, 1.8, 30.0)
    assert (p.fs_tolenergy, p.fs_maxiterbisect, p.fs_tolbisect, p.fs_urfree) == (1e-6, 40.0, 1e-18, 0.5)


@pytest.mark.gpu
@pytest.mark.parametrize("single_track_off", [False, True])
def test_free_surface_matches_oracle(single_track_off, deckdir):
    import amcfd
    import amcfd_decks as D
    import oracle_py
    dk = D.free_surface_track("fs_gpu", steps=4)
    if single_track_off:
        dk.single_track = (2e-5,) + dk.single_track[1:]
    d = amcfd.Deck(dk.write(deckdir))
    gpu = amcfd.Solver(d, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64)
    orc = oracle_py.Oracle(d.params)
    assert np.array_equal(gpu.get("zr"), orc.field("zr"))  # initial heights: z
    for s in range(4):
        gpu.step()
        orc.step()
        fg, fo = gpu.free_surface(), orc.free_surface()
        where = f"step {s + 1}"
        assert fg["iterations"] == fo["iterations"] and fg["bracketed"] == fo["bracketed"], (where, fg, fo)
        assert abs(fg["lambda"] - fo["lambda"]) <= 1e-12 * abs(fo["lambda"]) + 1e-300, (where, fg, fo)
        assert fg["volume"] == fo["volume"], where
        for k in ("fi_min", "fi_max"):
            assert abs(fg[k] - fo[k]) <= 1e-8 * abs(fo[k]) + 1e-30, (where, k, fg[k], fo[k])
        for f in ("zr", "tempr"):
            assert rel_l2(gpu.get(f), orc.field(f)) < 1e-8, (where, f, rel_l2(gpu.get(f), orc.field(f)))
    gpu.close()
