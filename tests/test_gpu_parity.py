"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

FP64, exact sweep order: the GPU reproduces the reference iterates, so every
step must take the same number of outer iterations and the fields must agree
to 1e-8 relative L2 (the residual differences are rounding from the order of
FP64 reductions and fused multiply-adds).  Melt-pool box indices must be
identical and L/D/W agree to 1e-8 relative.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl")
TOL = 1e-8


def _pair(deck, deckdir, **kw):
    import amcfd
    import oracle_py
    path = deck.write(deckdir)
    d = amcfd.Deck(path)
    return d, amcfd.Solver(d, **kw), oracle_py.Oracle(d.params)


def _cmp_fields(gpu, orc, fields=FIELDS, tol=TOL, where=""):
    for f in fields:
        a, b = gpu.get(f), orc.field(f)
        err = rel_l2(a, b)
        if np.linalg.norm(b) == 0:
            assert np.max(np.abs(a)) < 1e-12, (where, f)
        else:
            assert err < tol, (where, f, err)


def _cmp_report(rg, ro, where=""):
    assert rg["niter"] == ro["niter"], (where, rg["niter"], ro["niter"])
    for k in ("istat", "iend", "jstat", "jend", "kstat", "jstart", "powerindicator"):
        assert rg[k] == ro[k], (where, k, rg[k], ro[k])
    for k in ("tpeak", "alen", "depth", "width", "ratio", "heatinlaser"):
        a, b = rg[k], ro[k]
        assert abs(a - b) <= 1e-8 * max(abs(b), 1e-12) + 1e-14, (where, k, a, b)


@pytest.mark.parametrize("variant", ["base", "noflow", "upwind", "toolpath", "cooling", "p150"])
def test_exact_fp64_steps(variant, deckdir):
    import amcfd
    import amcfd_decks as D
    kw = dict(name=variant, steps=4)
    if variant == "noflow":
        kw["fluid_flow"] = False
    elif variant == "upwind":
        kw["scheme"] = "upwind"
    elif variant == "toolpath":
        kw["toolpath"] = True
    elif variant == "cooling":
        kw.update(steps=6, laser_off_after=3)
    elif variant == "p150":
        kw["power"] = 150.0
    deck, gpu, orc = _pair(D.small(**kw), deckdir, order=amcfd.ORDER_EXACT,
                           precision=amcfd.PREC_FP64)
    for s in range(kw["steps"]):
        rg, ro = gpu.step(), orc.step()
        _cmp_report(rg, ro, where=f"{variant} step {s + 1}")
        _cmp_fields(gpu, orc, where=f"{variant} step {s + 1}")
    gpu.close()


def test_exact_fp64_phases(deckdir):
    """Phase by phase through the first two outer iterations of steps 1 and 2."""
    import amcfd
    import amcfd_decks as D
    deck, gpu, orc = _pair(D.small("phases", steps=2), deckdir)
    for step in range(2):
        gpu.run_phase("laser")
        orc.call("begin_step")
        for it in range(2):
            gpu.run_phase("energy_assemble")
            orc.call("energy_assemble")
            orc.call("residual", 5)
            orc.call("props")
            where = f"step {step + 1} iter {it + 1}"
            for f in ("an", "as", "ae", "aw", "at", "ab", "ap", "su"):
                a, b = gpu.get(f)[1:-1, 1:-1, 1:-1], orc.field(f)[1:-1, 1:-1, 1:-1]
                assert rel_l2(a, b) < 1e-12, (where, f, rel_l2(a, b))
            _cmp_fields(gpu, orc, ("enthalpy",), 1e-13, where)
            for f, g in (("diff_next", "diff"), ("rho_next", "rho"), ("vis_next", "vis")):
                assert rel_l2(gpu.get(f), orc.field(g)) < 1e-13, (where, f)
            gpu.run_phase("energy_solve")
            orc.call("block_correct")
            orc.call("solve_entire")
            _cmp_fields(gpu, orc, ("enthalpy",), 1e-10, where + " solve")
            gpu.run_phase("h2t")
            orc.call("h2t")
            _cmp_fields(gpu, orc, ("temp", "fracl"), 1e-10, where + " h2t")
            r = gpu.run_phase("meltpool")
            orc.call("meltpool")
            ro = orc.report()
            for k in ("istat", "iend", "jstat", "jend", "kstat"):
                assert r[k] == ro[k], (where, k)
            assert abs(r["tpeak"] - ro["tpeak"]) < 1e-9 * ro["tpeak"]
            gpu.run_phase("momentum")
            orc.call("momentum")
            _cmp_fields(gpu, orc, ("uvel", "vvel", "wvel", "pressure", "pp"), 1e-9, where + " mom")
            r = gpu.run_phase("converge")
            orc.call("fluxes")
            ro = orc.report()
            for k in ("resorm", "resoru", "resorv", "resorw", "ratio"):
                assert abs(r[k] - ro[k]) <= 1e-7 * abs(ro[k]) + 1e-300, (where, k, r[k], ro[k])
        gpu.run_phase("update")
        orc.call("update_solutions")
        _cmp_fields(gpu, orc, where=f"step {step + 1} end")
    gpu.close()


@pytest.mark.parametrize("flow,tol", [(False, 1e-5), (True, 1e-4)])
def test_redblack_close_to_exact_order(flow, tol, deckdir):
    """The parallel red-black ordering and the exact order are two iterations
    for the same discrete equations; they differ only by what the outer loop
    leaves unconverged (the energy-only loop stops on the heat-balance ratio
    alone).  Observed gaps on this deck: 1.6e-6 (energy only) and 4.8e-6
    (with flow) relative L2 in T after two steps."""
    import amcfd
    import amcfd_decks as D
    dk = D.small("rb", steps=2, maxit=60, fluid_flow=flow)
    dk.tol = 1e-12
    path = dk.write(deckdir)
    d = amcfd.Deck(path)
    ex = amcfd.Solver(d, order=amcfd.ORDER_EXACT)
    rb = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK)
    for _ in range(2):
        ex.step()
        rb.step()
    assert rel_l2(rb.get("temp"), ex.get("temp")) < tol
    assert rel_l2(rb.get("enthalpy"), ex.get("enthalpy")) < tol
    ex.close()
    rb.close()


def test_fp32_close_to_fp64(deckdir):
    import amcfd
    import amcfd_decks as D
    path = D.small("fp32", steps=3).write(deckdir)
    d = amcfd.Deck(path)
    s64 = amcfd.Solver(d, precision=amcfd.PREC_FP64)
    s32 = amcfd.Solver(d, precision=amcfd.PREC_FP32)
    for _ in range(3):
        s64.step()
        s32.step()
    assert rel_l2(s32.get("temp"), s64.get("temp")) < 1e-3
    s64.close()
    s32.close()


@pytest.mark.parametrize("prec,order", [(0, 0), (1, 1)])
def test_graph_replay_bit_identical(prec, order, deckdir):
    """Outer iterations replayed from CUDA graphs give the same bits as direct
    launches (FP64 exact order and FP32 red-black), with and without timing."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("graphs", steps=5, toolpath=True).write(deckdir))
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=0)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=1)
    for s in range(5):
        a.profile(s % 2 == 1)  # alternate timed and untimed iterations on both paths
        b.profile(s % 2 == 1)
        ra, rb = a.step(), b.step()
        ctx = _mismatch_context(s, ra, rb)
        for k in ("niter", "tpeak", "alen", "depth", "width", "resorh", "resorm", "ratio"):
            assert ra[k] == rb[k], (k, ctx)
        for f in FIELDS:
            x, y = a.get(f), b.get(f)
            assert np.array_equal(x, y), _field_mismatch(f, x, y, ctx)
    a.close()
    b.close()


@pytest.mark.parametrize("prec,order,small_box,graphs,box_ctas", [(0, 0, 1, 1, 0), (1, 1, 1, 1, 0), (1, 1, 0, 1, 0),
                                                                  (0, 1, 0, 0, 0), (2, 1, 1, 1, 0), (1, 1, 0, 1, 1),
                                                                  (0, 1, 0, 1, 2)])
def test_overlapped_launches_bit_identical(prec, order, small_box, graphs, box_ctas, deckdir):
    """Launches that overlap the end of the kernel before them (programmatic
    dependent launch, the default) and the momentum box's line solve as one
    cooperative launch with grid barriers between the colour passes give the same
    bits and iteration counts as the serial form (serial_launch: each launch
    starts after the one before it has finished, one launch per colour pass):
    every kernel waits for its predecessor's completion before it reads anything,
    and the cooperative solve repeats the multi-launch arithmetic.  FP64 exact
    order, FP32 red-black and FP32 defect correction; the one-CTA and the
    multi-kernel momentum paths; graphs (the device-driven outer loop) and direct
    launches; and the cooperative solve on 1 and 2 CTAs (box_ctas), where every
    warp takes several lines of a colour and stages them again for each pass."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("pdl", steps=4, power=350.0, toolpath=True).write(deckdir))
    kw = dict(order=order, precision=prec, use_graphs=graphs, small_box=small_box)
    a = amcfd.Solver(d, serial_launch=1, **kw)
    b = amcfd.Solver(d, serial_launch=0, box_ctas=box_ctas, **kw)
    saw_box = False
    for s in range(4):
        ra, rb = a.step(), b.step()
        saw_box |= rb["momentum_cells"] > 0
        ctx = _mismatch_context(s, ra, rb)
        for k in ("niter", "tpeak", "alen", "depth", "width", "resorh", "resorm", "ratio"):
            assert ra[k] == rb[k], (k, ctx)
        for f in FIELDS:
            x, y = a.get(f), b.get(f)
            assert np.array_equal(x, y), _field_mismatch(f, x, y, ctx)
    assert saw_box
    a.close()
    b.close()


def _mismatch_context(step, ra, rb):
    keys = ("niter", "itertot", "resorh", "resorm", "ratio", "tpeak", "momentum_cells")
    return f"step {step + 1}: direct " + str({k: ra[k] for k in keys}) + " graph " + str({k: rb[k] for k in keys})


def _field_mismatch(name, x, y, ctx):
    """Where two fields that should be bit-identical differ: the largest
    difference, the number of differing nodes and the first one as (k, j, i)."""
    diff = x != y
    if not diff.any():
        return f"{name}: equal ({ctx})"
    first = tuple(int(q) for q in np.argwhere(diff)[0])
    return (f"{name}: {int(diff.sum())} nodes differ, max |diff| {float(np.nanmax(np.abs(x - y)))}, "
            f"first (k, j, i) = {first}: {x[first]!r} vs {y[first]!r}; {ctx}")


@pytest.mark.parametrize("prec,order", [(0, 0), (0, 1), (1, 1)])
def test_device_outer_loop_matches_host_loop(prec, order, deckdir):
    """A step launched as one graph (outer iterations chained by conditional
    nodes, convergence tested on the device) gives the same bits and iteration
    counts as one graph per outer iteration with the test on the host, and the
    same launches plus the chain's head kernel once a step.  The deck converges
    before maxit in some steps and not in others (odd and even counts, so the
    property parity of later steps differs), and its melt-pool box is small
    enough for the one-CTA momentum path."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("devloop", steps=8, maxit=11, power=60.0, toolpath=True).write(deckdir))
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=1, host_loop=1)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=1, host_loop=0)
    counts = []
    for s in range(8):
        ra, rb = a.step(), b.step()
        for k in ("niter", "itertot", "tpeak", "alen", "depth", "width", "resorh", "resorm", "ratio",
                  "momentum_cells"):
            assert ra[k] == rb[k], (s, k, ra[k], rb[k])
        for f in FIELDS:
            assert np.array_equal(a.get(f), b.get(f)), (s, f)
        counts.append(rb["niter"])
    assert b.launches == a.launches + 8
    assert min(counts) < 11 and {c % 2 for c in counts} == {0, 1}, counts
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_small_box_momentum_matches_grid_path(prec, deckdir):
    """Red-black runs with the one-CTA momentum chain (small melt-pool box held
    in shared memory) stay within 1e-6 (FP64) / 1e-3 (FP32) relative L2 of the
    same runs with the multi-kernel chain, with the same iteration counts in FP64."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("smallbox", steps=4, power=350.0).write(deckdir))
    a = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, small_box=0)
    b = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, small_box=1)
    tol = 1e-6 if prec == 0 else 1e-3
    saw_box = False
    for s in range(4):
        ra, rb = a.step(), b.step()
        saw_box |= rb["momentum_cells"] > 0
        if prec == 0:
            assert ra["niter"] == rb["niter"], (s, ra["niter"], rb["niter"])
        for f in ("temp", "uvel", "vvel", "wvel", "pressure"):
            x, y = b.get(f), a.get(f)
            if np.linalg.norm(y) > 0:
                assert rel_l2(x, y) < tol, (s, f, rel_l2(x, y))
    assert saw_box
    assert b.launches < a.launches
    a.close()
    b.close()


@pytest.mark.parametrize("prec,order", [(0, 0), (1, 1)])
def test_contexts_of_different_grid_widths_coexist(prec, order, deckdir):
    """Kernel launch limits are per process, shared by all contexts: creating a
    context on a narrow grid after one on a wide grid leaves the wide one's line
    sweeps launchable (the limit is only ever raised), with and without graphs."""
    import amcfd
    import amcfd_decks as D
    wide = amcfd.Deck(D.small("wide", nx=300, ny=14, nz=10, steps=2).write(deckdir + "/wide"))
    narrow = amcfd.Deck(D.small("narrow", nx=20, ny=12, nz=8, steps=2).write(deckdir + "/narrow"))
    for graphs in (0, 1):
        a = amcfd.Solver(wide, order=order, precision=prec, use_graphs=graphs)
        b = amcfd.Solver(narrow, order=order, precision=prec, use_graphs=graphs)
        ra = [a.step() for _ in range(2)]
        b.step()
        c = amcfd.Solver(wide, order=order, precision=prec, use_graphs=graphs)
        rc = [c.step() for _ in range(2)]
        assert [r["niter"] for r in ra] == [r["niter"] for r in rc]
        for f in FIELDS:
            assert np.array_equal(a.get(f), c.get(f)), (graphs, f)
        for s in (a, b, c):
            s.close()
