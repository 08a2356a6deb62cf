"""The CPU oracle against the reference solver.

1. Golden records (tests/golden/*/ref.npz, made by tests/golden/make_golden.py
   from the reference compiled from its own sources): the oracle must reproduce
   them bit for bit -- every step's iteration count and scalars, the fields
   after the first and the last step, and the grid.
2. Live comparison with oracle/_ref/amcfd_ref_dump (only where it was built):
   deck features the golden set does not cover.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN

CASES = ["g_track", "g_toolpath", "g_noflow", "g_cooling", "g_species", "g_powder", "g_moving", "g_freesurf"]
FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl", "pp")
SPECIES_FIELDS = ("avgconcentration", "concentration")
POWDER_FIELDS = ("csfrac", "solfrac", "mpPhase", "mpLiqPhase", "diff", "rho")
MOVING_FIELDS = ("grad", "rate", "hnot")
FREESURF_FIELDS = ("zr", "tempr")


def fs_row(f):
    """The free surface's values as FreeSurfaceManager::execute prints them."""
    return ["%.4e" % f[k] for k in ("lambda", "residual", "fi_min", "fi_max", "volume")] + [str(f["iterations"])]
SCALARS = ("niter", "tpeak", "alen", "depth", "width", "ratio", "resorh", "resorm", "resoru",
           "resorv", "resorw", "heatinlaser", "istat", "iend", "jstat", "jend", "kstat", "jstart",
           "resorc", "nk_active", "trackindx", "steadylength")


def _same(a, b):
    return (a == b) or (np.isnan(a) and np.isnan(b))


@pytest.mark.parametrize("case", CASES)
def test_oracle_bit_exact_on_golden(case, oracle_lib, monkeypatch):
    import amcfd
    import oracle_py
    monkeypatch.chdir(os.path.join(GOLDEN, case))
    deck = amcfd.Deck(f"{case}.k")
    ref = np.load("ref.npz")
    o = oracle_py.Oracle(deck.params)
    for g in ("x", "y", "z", "xu", "yv", "dxpwinv", "dypsinv", "dzpbinv", "fracx", "fracy"):
        assert np.array_equal(o.field(g), ref[f"geom_{g}"]), g
    n = len(ref["s_niter"])
    fields = FIELDS + tuple(f for f in SPECIES_FIELDS + POWDER_FIELDS + MOVING_FIELDS + FREESURF_FIELDS
                            if f"first_{f}" in ref)
    for s in range(n):
        r = o.step()
        if "fs_monitor" in ref:
            assert fs_row(o.free_surface()) == list(ref["fs_monitor"][s]), (case, s)
        for k in SCALARS:
            assert _same(r[k], ref[f"s_{k}"][s]), (case, s, k, r[k], ref[f"s_{k}"][s])
        tag = "first" if s == 0 else "last" if s == n - 1 else None
        if tag:
            for f in fields:
                assert np.array_equal(o.field(f), ref[f"{tag}_{f}"], equal_nan=True), (case, s, f)
            for g in ("x", "y"):  # the grid after the step (moves with a moving mesh)
                if f"{tag}_grid_{g}" in ref:
                    assert np.array_equal(o.field(g), ref[f"{tag}_grid_{g}"]), (case, s, g)


def _variants():
    import amcfd_decks as D
    out = []
    d = D.small("v_evap", steps=3, power=120.0)
    d.evaporation = (6.0e6, 3100.0, 1e-3, 0.056)
    out.append(d)
    d = D.small("v_vol", steps=3, power=100.0)
    d.volumetric = (150.0, 0.4, 60e-6, 50e-6, 2.0)
    out.append(d)
    d = D.small("v_table", steps=4, power=100.0)
    d.heat_table = [(0.0, 150.0, 0.4, 60e-6, 50e-6, 2.0), (2.5e-5, 250.0, 0.4, 80e-6, 40e-6, 2.0),
                    (1.0, 250.0, 0.4, 80e-6, 40e-6, 2.0)]
    out.append(d)
    d = D.small("v_vardt", steps=5)
    d.vardt = [(2e-5, 1e-5, 1.0), (1.0, 5e-6, 1.0)]
    d.finaltime = 4.2e-5
    out.append(d)
    # species with the upwind scheme, a slow diffusivity and a strong partition
    d = D.small("v_species", steps=4, power=250.0, scheme="upwind")
    d.species = (0.5, 2e-9, 0.1, 0.5)
    out.append(d)
    # powder bed with the species equation: three layers of three planes each
    d = D.powder_layers("v_powder", tracks=2, ncvzlayer=3, layerheight=40e-6, track_steps=3, dwell_steps=1)
    d.species = (1.0, 5e-9, 0.3, 0.7)
    out.append(d)
    # moving mesh towards -x and -y (the remap partner is the already-remapped node), with G/R
    out.append(D.moving_track("v_moving", reverse=True, steps=5))
    # free surface on the upwind scheme, beam off after two steps (the volume from lasertime)
    d = D.free_surface_track("v_freesurf", steps=4)
    d.scheme, d.single_track = "upwind", (2e-5,) + d.single_track[1:]
    out.append(d)
    # the 600 x 300 x 120 benchmark deck's toolpath in miniature: a bidirectional
    # raster with the beam off during a dwell between tracks, 12 steps (first
    # track, dwell, start of the second)
    d = D.small("v_raster", steps=12, power=250.0)
    d.single_track = None
    d.toolpath = D.raster_toolpath(0.20e-3, 0.26e-3, 0.18e-3, 60e-6, 2, D._top(d.z_zones), 1.0, 2e-5)
    out.append(d)
    # the exponential scheme: the reference divides 0/0 at zero Peclet number, and
    # the oracle reproduces where the NaNs appear
    out.append(D.small("v_exponential", steps=2, scheme="exponential_law"))
    # the smallest instance of the 64-instance parameter sweep, as the sweep draws it
    sweep = D.config2(steps=2)
    cells = [sum(z[1] for z in q.x_zones) * sum(z[1] for z in q.y_zones) * sum(z[1] for z in q.z_zones)
             for q in sweep]
    out.append(sweep[cells.index(min(cells))])
    # the 120 x 60 x 40 benchmark deck itself, its first two steps
    out.append(D.config0(steps=2))
    # and the 400 x 200 x 100 deck bench.py times, its first step (about 40 s of
    # single-threaded CPU for the two solvers, an 0.9 GB dump)
    out.append(D.config1(steps=1))
    return out


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "amcfd_ref_dump")),
                    reason="reference not built in this checkout (oracle/build_ref.sh)")
@pytest.mark.parametrize("idx", range(13))
def test_oracle_bit_exact_live(idx, tmp_path, oracle_lib):
    import amcfd
    import oracle_py
    from amcfd_dump import read_dump
    deck = _variants()[idx]
    path = deck.write(str(tmp_path))
    out = str(tmp_path / "ref.bin")
    subprocess.check_call([oracle_py.REF_DUMP, path, "--out", out], cwd=str(tmp_path),
                          env=dict(os.environ, OMP_NUM_THREADS="1"), stdout=subprocess.DEVNULL)
    ref = read_dump(out)
    mon = tmp_path / f"{deck.name}_FreeSurfaceMonitor.txt"
    mon = [l.split()[1:] for l in open(mon).read().splitlines()
           if l.startswith("  ") and l.split()[0][:1].isdigit()] if mon.exists() else None
    o = oracle_py.Oracle(amcfd.Deck(path))
    fields = FIELDS + (SPECIES_FIELDS if deck.species is not None else ()) + \
        (POWDER_FIELDS if deck.powder is not None else ()) + (MOVING_FIELDS if deck.solidification else ()) + \
        (FREESURF_FIELDS if deck.free_surface is not None else ())
    for s in ref["steps"]:
        r = o.step()
        assert r["niter"] == s["niter"]
        assert _same(r["tpeak"], s["tpeak"])
        assert _same(r["resorc"], s["resorc"])
        assert r["nk_active"] == s["nk_active"] and r["trackindx"] == s["trackindx"]
        assert r["steadylength"] == s["steadylength"]
        if mon is not None:
            assert fs_row(o.free_surface()) == mon[s["step"] - 1], (deck.name, s["step"])
        assert np.array_equal(o.field("x"), s["grid_x"]) and np.array_equal(o.field("y"), s["grid_y"])
        for f in fields:
            assert np.array_equal(o.field(f), s[f], equal_nan=True), (deck.name, s["step"], f)
