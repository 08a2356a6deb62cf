"""Output path: the files a run writes (.vts/.pvd, _Residuals.txt, the final
geometry) against the ones the compiled reference writes for the same deck.

The reference (oracle/_ref/AM-CFD, built from the reference's sources, one
OpenMP thread) and the GPU solver (FP64, exact sweep order) run the same deck
from directories of their own.  Checked: the .vts XML headers and the .pvd are
byte-identical; the point coordinates are identical; every point array agrees
to 1e-8 relative L2 (the solver parity tolerance), the species fields included
when the deck solves them; the text files agree token
by token, numbers to the precision they are printed with (2 digits, so within
2 % relative).  The cooling-rate lines are left out: the reference computes
them from uninitialised values when the beam row has no molten cell.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

REF_CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "AM-CFD")


def read_vts(path):
    """(header text, [arrays]) of an appended-raw .vts file (Float64 arrays, and the
    UInt8 vtkGhostType array of powder-bed runs, in header order)."""
    data = open(path, "rb").read()
    cut = data.index(b'<AppendedData encoding="raw">_') + len(b'<AppendedData encoding="raw">_')
    head, body = data[:cut].decode(), data[cut:]
    types = ["<f8"] + ["u1" if 'type="UInt8"' in a else "<f8" for a in head.split("<DataArray")[2:]]
    arrays, pos = [], 0
    while body[pos:pos + 4] and not body[pos:].startswith(b"\n</AppendedData>"):
        (n,) = struct.unpack("<i", body[pos:pos + 4])
        arrays.append(np.frombuffer(body[pos + 4:pos + 4 + n], dtype=types[len(arrays)]).astype(np.float64))
        pos += 4 + n
    assert body[pos:] == b"\n</AppendedData> </VTKFile>"
    return head, arrays


def same_tokens(a, b, rtol=2e-2):
    ta, tb = a.split(), b.split()
    if len(ta) != len(tb):
        return False
    for x, y in zip(ta, tb):
        if x == y:
            continue
        try:
            fx, fy = float(x), float(y)
        except ValueError:
            return False
        if not abs(fx - fy) <= rtol * max(abs(fx), abs(fy)) + 1e-12:
            return False
    return True


def text_lines(path):
    return [l for l in open(path).read().splitlines() if "Cooling rate" not in l]


@pytest.mark.skipif(not os.path.exists(REF_CLI), reason="reference binary not built")
@pytest.mark.parametrize("variant", ["plain", "species", "powder", "moving", "freesurf"])
def test_output_files_match_reference(variant, tmp_path, monkeypatch):
    import amcfd
    import amcfd_decks as D
    if variant == "powder":  # csfrac, solfrac and the vtkGhostType array of unbuilt layers
        d = D.powder_layers("outdeck", nx=20, ny=12, nz=8)
    elif variant == "moving":  # points follow the moving grid; grad and rate written
        d = D.moving_track("outdeck", nx=20, ny=12, nz=8, steps=5)
    elif variant == "freesurf":  # points at the deformed heights zr; zr, tempr and the monitor file
        d = D.free_surface_track("outdeck", steps=5)
    else:
        d = D.small("outdeck", nx=20, ny=12, nz=8, steps=5, power=300.0)
    if variant == "species":  # adds avgconcentration and concentration to the written fields
        d.species = (1.0, 5e-9, 0.3, 0.7)
    d.outtime = 2 * d.dt
    d.final_geometry = "outdeck_geom.txt"
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    path = d.write(str(ref_dir), relative=True)
    shutil.copytree(ref_dir, our_dir)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    subprocess.run([REF_CLI, os.path.basename(path)], cwd=ref_dir, env=env, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=300)

    monkeypatch.chdir(our_dir)
    deck = amcfd.Deck(os.path.basename(path))
    s = amcfd.Solver(deck, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64)
    w = amcfd.Writer(s, deck)
    wrote = 0
    t = 0.0
    while t < deck.params.finaltime:
        t = s.step()["timet"]
        wrote += w.step()
    w.finish()
    w.close()
    s.close()
    assert wrote >= 2

    ref_vts = sorted(os.listdir(ref_dir / "out"))
    our_vts = sorted(os.listdir(our_dir / "out"))
    assert ref_vts == our_vts and len(ref_vts) >= 3
    for name in ref_vts:
        ha, aa = read_vts(ref_dir / "out" / name)
        hb, ab = read_vts(our_dir / "out" / name)
        assert ha == hb, name
        assert len(aa) == len(ab)
        assert np.array_equal(aa[0], ab[0]), "coordinates"
        for q, (x, y) in enumerate(zip(aa[1:], ab[1:])):
            if np.linalg.norm(x) == 0:
                assert np.abs(y).max() < 1e-12, (name, q)
            else:
                assert rel_l2(y, x) < 1e-8, (name, q, rel_l2(y, x))
    assert open(ref_dir / "outdeck.pvd").read() == open(our_dir / "outdeck.pvd").read()
    names = ["outdeck_Residuals.txt", "outdeck_geom.txt"]
    if variant == "freesurf":
        names.append("outdeck_FreeSurfaceMonitor.txt")
    for fname in names:
        la, lb = text_lines(ref_dir / fname), text_lines(our_dir / fname)
        assert len(la) == len(lb), fname
        for x, y in zip(la, lb):
            assert same_tokens(x, y), (fname, x, y)
