"""The autotuner: at creation it times the energy assembly with 4, 8 and 16
planes per CTA and the pipelined red-black line solve with its passes 8, 16
and 32 planes apart in its work order (the per-pass sweeps, when they run, with
2, 4 and 8 lines per CTA) on the context's own grid, and keeps the fastest.
The launch shape changes no arithmetic of the sweeps and only the order of the
assembly's FP64 partial sums, so a context pinned to the assembly shape the
tuner chose reproduces the tuned one bit for bit (whatever its sweep stride),
and every shape agrees with the default to rounding."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy")


@pytest.mark.parametrize("prec", [1, 2])
def test_tuned_shapes_are_reported_and_reproducible(prec, tmp_path):
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("tune", nx=40, ny=20, nz=14, steps=3).write(str(tmp_path)))
    a = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, use_graphs=1, autotune=1)
    t = a.tuning()
    assert t["asm_kseg"] in (4, 8, 16) and t["sweep_warps"] in (2, 4, 8), t
    assert all(v > 0 for v in t["asm_ms"].values()), t
    assert t["asm_ms"][t["asm_kseg"]] == min(t["asm_ms"].values())
    assert t["pipe_stride"] in (8, 16, 32), t
    assert t["sweep_ms"][t["pipe_stride"]] == min(t["sweep_ms"].values()) > 0, t
    b = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, use_graphs=1,
                     asm_kseg=t["asm_kseg"], sweep_warps=t["sweep_warps"])
    c = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, use_graphs=1)
    assert b.tuning()["asm_kseg"] == t["asm_kseg"] and b.tuning()["sweep_warps"] == t["sweep_warps"]
    for _ in range(3):
        ra, rb, rc = a.step(), b.step(), c.step()
        assert ra["niter"] == rb["niter"]
    for f in FIELDS:
        x, y, z = a.get(f), b.get(f), c.get(f)
        assert np.array_equal(x, y), f
        if np.linalg.norm(z) > 0:
            assert rel_l2(x, z) < (1e-9 if prec == 2 else 1e-4), (f, rel_l2(x, z))
    for s in (a, b, c):
        s.close()
