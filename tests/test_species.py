"""Species equation (ivar 6): deck, C ABI and GPU parity against the oracle.

The oracle's species branch is pinned bit for bit to the compiled reference by
tests/test_oracle.py (golden case g_species, live variant v_species).  Here the
CUDA path runs through the C ABI: FP64 exact order must take the same outer
iterations as the oracle in every step, with avgconcentration and concentration
within 1e-8 relative L2 (the solver parity tolerance); phase by phase the
species coefficients agree to 1e-12 and the solved field to 1e-10; FP32
red-black stays within 1e-3 of FP64.
"""
import numpy as np
import pytest

from conftest import rel_l2

SPECIES = ("avgconcentration", "concentration")


def _deck(name, steps=4, scheme="power_law", species=(1.0, 5e-9, 0.3, 0.7), **kw):
    import amcfd_decks as D
    d = D.small(name, steps=steps, scheme=scheme, **kw)
    d.species = species
    return d


def test_deck_carries_species_row(deckdir):
    import amcfd
    d = amcfd.Deck(_deck("sp_parse", species=(0.5, 2e-9, 0.1, 0.6)).write(deckdir))
    p = d.params
    assert p.species == 1
    assert (p.initconc, p.massdiff, p.kp, p.urfc) == (0.5, 2e-9, 0.1, 0.6)
    assert "avgconcentration" in d.string("scalar_out").split()


def test_species_row_needs_four_values(deckdir):
    import amcfd
    path = _deck("sp_short").write(deckdir)
    text = open(path).read().replace("  1.0 5e-09 0.3 0.7", "  1.0 5e-09 0.3")
    open(path, "w").write(text)
    with pytest.raises(amcfd.AmcfdError):
        amcfd.Deck(path)


def test_report_struct_has_resorc(lib):
    import ctypes

    import amcfd
    assert lib.amcfd_sizeof_report() == ctypes.sizeof(amcfd.AmcfdReport)
    assert lib.amcfd_sizeof_params() == ctypes.sizeof(amcfd.AmcfdParams)
    assert "resorc" in dict(amcfd.AmcfdReport._fields_)


def _pair(deck, deckdir, **kw):
    import amcfd
    import oracle_py
    d = amcfd.Deck(deck.write(deckdir))
    return amcfd.Solver(d, **kw), oracle_py.Oracle(d.params)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["power_law", "upwind"])
def test_species_exact_fp64_steps(scheme, deckdir):
    import amcfd
    gpu, orc = _pair(_deck(f"sp_{scheme}", scheme=scheme), deckdir, order=amcfd.ORDER_EXACT,
                     precision=amcfd.PREC_FP64)
    for s in range(4):
        rg, ro = gpu.step(), orc.step()
        where = f"{scheme} step {s + 1}"
        assert rg["niter"] == ro["niter"], (where, rg["niter"], ro["niter"])
        assert abs(rg["resorc"] - ro["resorc"]) <= 1e-6 * abs(ro["resorc"]) + 1e-12, (where, rg["resorc"], ro["resorc"])
        for f in ("temp", "uvel", "enthalpy") + SPECIES:
            err = rel_l2(gpu.get(f), orc.field(f))
            assert err < 1e-8, (where, f, err)
    c = gpu.get("avgconcentration")
    assert c.max() > 1.5  # the surface condition has raised the melt-pool concentration
    gpu.close()


@pytest.mark.gpu
def test_species_phase_by_phase(deckdir):
    import amcfd
    gpu, orc = _pair(_deck("sp_phases", steps=2), deckdir)
    for step in range(2):
        gpu.run_phase("laser")
        orc.call("begin_step")
        for it in range(2):
            where = f"step {step + 1} iter {it + 1}"
            for ph in ("energy_assemble", "energy_solve", "h2t", "meltpool", "momentum"):
                gpu.run_phase(ph)
            orc.call("energy_assemble")
            orc.call("residual", 5)
            orc.call("props")
            orc.call("block_correct")
            orc.call("solve_entire")
            orc.call("h2t")
            orc.call("meltpool")
            orc.call("momentum")
            # the inputs of the species coefficients, as the momentum phase left them
            pre = {f: rel_l2(gpu.get(f), orc.field(g)) for f, g in
                   (("uvel", "uvel"), ("vvel", "vvel"), ("wvel", "wvel"), ("temp", "temp"), ("rho_next", "rho"))}
            r = gpu.run_phase("species")
            orc.call("species")
            for f in ("an", "as", "ae", "aw", "at", "ab", "ap", "su"):
                a, b = gpu.get(f)[1:-1, 1:-1, 1:-1], orc.field(f)[1:-1, 1:-1, 1:-1]
                if rel_l2(a, b) >= 1e-12:
                    d = np.abs(a - b)
                    q = tuple(int(x) for x in np.unravel_index(np.argmax(d), d.shape))
                    raise AssertionError(f"{where} {f}: rel-L2 {rel_l2(a, b):.3e}, {int((d > 1e-12 * np.abs(b).max()).sum())} "
                                         f"cells differ, largest at interior (k, j, i) {q}: {a[q]!r} vs {b[q]!r}; "
                                         f"inputs before the phase {pre}; report {r}")
            a, b = gpu.get("avgconcentration"), orc.field("avgconcentration")
            assert rel_l2(a, b) < 1e-10, (where, rel_l2(a, b))
            ro = orc.report()
            assert abs(r["resorc"] - ro["resorc"]) <= 1e-7 * abs(ro["resorc"]) + 1e-14, (where, r["resorc"], ro["resorc"])
            gpu.run_phase("converge")
            orc.call("fluxes")
        gpu.run_phase("update")
        orc.call("update_solutions")
        for f in SPECIES:
            assert rel_l2(gpu.get(f), orc.field(f)) < 1e-10, (step, f)
            assert np.array_equal(gpu.get("avgconcentrationnot"), gpu.get("avgconcentration"))
    gpu.close()


@pytest.mark.gpu
def test_species_fp32_redblack_close_to_fp64(deckdir):
    import amcfd
    d = amcfd.Deck(_deck("sp_fp32", steps=3).write(deckdir))
    a = amcfd.Solver(d, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64)
    b = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP32)
    for _ in range(3):
        a.step()
        b.step()
    for f in SPECIES:
        assert rel_l2(b.get(f), a.get(f)) < 1e-3, (f, rel_l2(b.get(f), a.get(f)))
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,order", [(0, 0), (1, 1)])
def test_species_graph_replay_bit_identical(prec, order, deckdir):
    import amcfd
    d = amcfd.Deck(_deck("sp_graphs", steps=3).write(deckdir))
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=0)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=1)
    for s in range(3):
        ra, rb = a.step(), b.step()
        assert ra["niter"] == rb["niter"] and ra["resorc"] == rb["resorc"], s
        for f in SPECIES:
            assert np.array_equal(a.get(f), b.get(f)), (s, f)
    a.close()
    b.close()
