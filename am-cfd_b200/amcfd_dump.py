"""Reader for the per-step state records written by the reference dump driver
(oracle/ref_driver.cpp) and by the oracle/GPU harness in the same format."""
from __future__ import annotations

import struct
from typing import Dict, List

import numpy as np

FIELDS = ["temp", "uvel", "vvel", "wvel", "pressure", "enthalpy", "fracl", "pp", "diff",
          "rho", "vis", "hnot", "fraclnot"]
SPECIES_FIELDS = ["avgconcentration", "concentration"]
POWDER_FIELDS = ["csfrac", "solfrac", "mpPhase", "mpLiqPhase"]
GEOM = ["x", "y", "z", "xu", "yv", "dxpwinv", "dypsinv", "dzpbinv", "fracx", "fracy"]
SCALARS = ["timet", "resorh", "resorm", "resoru", "resorv", "resorw", "tpeak", "alen",
           "depth", "width", "ratio", "heatinlaser", "ahtoploss", "accul", "heatout",
           "heatvol", "fluxwest", "fluxeast", "fluxtop", "fluxbottom", "fluxnorth",
           "fluxsouth", "beamposx", "beamposy", "scanvel", "resorc"]
INDICES = ["istat", "iend", "jstat", "jend", "kstat", "jstart", "powerindicator", "nk_active", "trackindx",
           "steadylength"]


def read_dump(path: str) -> Dict:
    with open(path, "rb") as f:
        buf = f.read()
    off = 0

    def i32():
        nonlocal off
        v = struct.unpack_from("<i", buf, off)[0]
        off += 4
        return v

    assert buf[:4] == b"AMCR", "not a state dump"
    off = 4
    version = i32()
    assert version == 2, "state dump version"
    ni, nj, nk = i32(), i32(), i32()
    nf, ng = i32(), i32()
    n = ni * nj * nk
    names = []
    for _ in range(nf):  # version 2: the field names
        ln = i32()
        names.append(buf[off:off + ln].decode())
        off += ln
    geom = {}
    for g in range(ng):
        ln = i32()
        geom[GEOM[g]] = np.frombuffer(buf, "<f8", ln, off).copy()
        off += 8 * ln
    steps: List[Dict] = []
    while True:
        s = i32()
        if s < 0:
            break
        rec = {"step": s, "niter": i32(), "itertot": i32()}
        ns = i32()
        sc = np.frombuffer(buf, "<f8", ns, off)
        off += 8 * ns
        rec.update({SCALARS[q]: float(sc[q]) for q in range(ns)})
        nix = i32()
        ix = np.frombuffer(buf, "<i4", nix, off)
        off += 4 * nix
        rec.update({INDICES[q]: int(ix[q]) for q in range(nix)})
        for q in range(nf):
            rec[names[q]] = np.frombuffer(buf, "<f8", n, off).reshape(nk, nj, ni).copy()
            off += 8 * n
        for g, ln in (("x", ni), ("y", nj)):
            rec["grid_" + g] = np.frombuffer(buf, "<f8", ln, off).copy()
            off += 8 * ln
        steps.append(rec)
    return {"version": version, "ni": ni, "nj": nj, "nk": nk, "geom": geom, "steps": steps}
