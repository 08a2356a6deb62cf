"""Generate the golden records of the reference solver (run in the build container).

For each small deck below this script writes the deck, its mesh (and toolpath)
into tests/golden/<name>/ with relative file names, runs the reference solver
compiled from its own sources (oracle/_ref/amcfd_ref_dump, built by
oracle/build_ref.sh) single-threaded in that directory, and stores
<name>/ref.npz: the per-step scalars of every step and the fields after the
first and the last step.  The oracle tests replay the same decks.

usage: python tests/golden/make_golden.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "am-cfd_b200"), os.path.join(ROOT, "oracle")]

import amcfd_decks as D  # noqa: E402
from amcfd_dump import read_dump  # noqa: E402

FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl", "pp")
SPECIES_FIELDS = ("avgconcentration", "concentration")
POWDER_FIELDS = ("csfrac", "solfrac", "mpPhase", "mpLiqPhase", "diff", "rho")
MOVING_FIELDS = ("grad", "rate", "hnot", "grid_x", "grid_y")
FREESURF_FIELDS = ("zr", "tempr")
SCALARS = ("niter", "timet", "resorh", "resorm", "resoru", "resorv", "resorw", "tpeak", "alen",
           "depth", "width", "ratio", "heatinlaser", "istat", "iend", "jstat", "jend", "kstat",
           "jstart", "resorc", "nk_active", "trackindx", "steadylength")


def species_deck():
    d = D.small("g_species", nx=16, ny=10, nz=8, steps=4)
    d.species = (1.0, 5e-9, 0.3, 0.7)
    return d


def decks():
    return [
        D.small("g_track", nx=16, ny=10, nz=8, steps=4),
        D.small("g_toolpath", nx=16, ny=10, nz=8, steps=4, toolpath=True),
        D.small("g_noflow", nx=16, ny=10, nz=8, steps=4, fluid_flow=False),
        D.small("g_cooling", nx=16, ny=10, nz=8, steps=6, laser_off_after=3, scheme="upwind"),
        species_deck(),
        D.powder_layers("g_powder"),
        D.moving_track("g_moving"),
        D.free_surface_track("g_freesurf"),
    ]


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "amcfd_ref_dump")
    if not os.path.exists(exe):
        sys.exit("build the reference first: bash oracle/build_ref.sh")
    for d in decks():
        out = os.path.join(HERE, d.name)
        path = d.write(out, relative=True)
        subprocess.check_call([exe, os.path.basename(path), "--out", "ref.bin"], cwd=out,
                              env=dict(os.environ, OMP_NUM_THREADS="1"), stdout=subprocess.DEVNULL)
        dump = read_dump(os.path.join(out, "ref.bin"))
        os.unlink(os.path.join(out, "ref.bin"))
        steps = dump["steps"]
        rec = {f"s_{k}": np.array([s[k] for s in steps]) for k in SCALARS}
        for tag, s in (("first", steps[0]), ("last", steps[-1])):
            extra = SPECIES_FIELDS + (POWDER_FIELDS if "csfrac" in s else ()) + \
                (MOVING_FIELDS if "grad" in s else ()) + FREESURF_FIELDS
            for f in FIELDS + tuple(f for f in extra if f in s):
                rec[f"{tag}_{f}"] = s[f]
        for g, v in dump["geom"].items():
            rec[f"geom_{g}"] = v
        mon = os.path.join(out, f"{d.name}_FreeSurfaceMonitor.txt")
        if os.path.exists(mon):  # the free surface's monitor values, as printed, one row per step
            rows = [l.split()[1:] for l in open(mon).read().splitlines()
                    if l.startswith("  ") and l.split()[0][:1].isdigit()]
            rec["fs_monitor"] = np.array(rows)
            os.unlink(mon)
        np.savez_compressed(os.path.join(out, "ref.npz"), **rec)
        print(d.name, len(steps), "steps")


if __name__ == "__main__":
    main()
