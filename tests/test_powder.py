"""Powder-bed mode: deck, layer activation and GPU parity against the oracle.

The oracle's powder branch (effective powder properties, consolidated
fraction, the growing active domain, the push-back of csfrac / solfrac /
mpPhase / mpLiqPhase) is pinned bit for bit to the compiled reference by
tests/test_oracle.py (golden g_powder, live v_powder).  Here the CUDA path
runs the golden deck through the C ABI: FP64 exact order must activate the
same layers at the same steps and take the same outer iterations, with every
field within 1e-8 relative L2 over the whole allocated grid; CUDA-graph replay
across a layer activation is bit-identical to direct launches.
"""
import numpy as np
import pytest

from conftest import rel_l2

POWDER = ("csfrac", "solfrac", "mpPhase", "mpLiqPhase")
FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl", "rho", "diff") + POWDER


def test_deck_adds_the_layers_to_the_last_z_zone(deckdir):
    import amcfd
    import amcfd_decks as D
    d = D.powder_layers("pw_parse", tracks=2, ncvzlayer=3, layerheight=40e-6)
    p = amcfd.Deck(d.write(deckdir)).params
    assert (p.powderbed, p.numlayers, p.ncvzlayer) == (1, 3, 3)
    assert p.layerheight == 40e-6 and p.powderthconb == 5.0
    nz_last = d.z_zones[-1][1]
    assert p.ncvz[p.nzz - 1] == nz_last + 3 * 3
    assert abs(p.zzone[p.nzz - 1] - (d.z_zones[-1][0] + 3 * 40e-6)) < 1e-18


def test_powder_row_needs_eight_values(deckdir):
    import amcfd
    import amcfd_decks as D
    path = D.powder_layers("pw_short").write(deckdir)
    lines = open(path).read().splitlines()
    q = lines.index("*POWDER_BED_MODE") + 2
    lines[q] = " ".join(lines[q].split()[:7])
    open(path, "w").write("\n".join(lines) + "\n")
    with pytest.raises(amcfd.AmcfdError):
        amcfd.Deck(path)


def _pair(deck, deckdir, **kw):
    import amcfd
    import oracle_py
    d = amcfd.Deck(deck.write(deckdir))
    return amcfd.Solver(d, **kw), oracle_py.Oracle(d.params)


@pytest.mark.gpu
def test_powder_exact_fp64_steps(deckdir):
    import amcfd
    import amcfd_decks as D
    gpu, orc = _pair(D.powder_layers("pw_exact"), deckdir, order=amcfd.ORDER_EXACT,
                     precision=amcfd.PREC_FP64)
    assert gpu.shape == orc.shape
    seen = set()
    for s in range(10):
        rg, ro = gpu.step(), orc.step()
        where = f"step {s + 1}"
        for k in ("niter", "nk_active", "trackindx", "istat", "iend", "jstat", "jend", "kstat"):
            assert rg[k] == ro[k], (where, k, rg[k], ro[k])
        assert abs(rg["tpeak"] - ro["tpeak"]) <= 1e-8 * ro["tpeak"], where
        seen.add(rg["nk_active"])
        for f in FIELDS:
            a, b = gpu.get(f), orc.field(f)
            if np.linalg.norm(b) == 0:
                assert np.abs(a).max() < 1e-12, (where, f)
            else:
                assert rel_l2(a, b) < 1e-8, (where, f, rel_l2(a, b))
    assert len(seen) == 2  # a second layer became active on the way
    gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,order", [(0, 0), (1, 1)])
def test_powder_graph_replay_across_activation(prec, order, deckdir):
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.powder_layers("pw_graphs").write(deckdir))
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=0)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=1)
    for s in range(8):
        ra, rb = a.step(), b.step()
        assert ra["niter"] == rb["niter"] and ra["nk_active"] == rb["nk_active"], s
        for f in ("temp", "uvel", "csfrac"):
            assert np.array_equal(a.get(f), b.get(f)), (s, f)
    a.close()
    b.close()


@pytest.mark.gpu
def test_powder_fp32_redblack_close_to_fp64(deckdir):
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.powder_layers("pw_fp32").write(deckdir))
    a = amcfd.Solver(d, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64)
    b = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP32)
    for _ in range(3):
        a.step()
        b.step()
    for f in ("temp", "csfrac"):
        assert rel_l2(b.get(f), a.get(f)) < 1e-3, (f, rel_l2(b.get(f), a.get(f)))
    a.close()
    b.close()
