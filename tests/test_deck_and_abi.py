"""Host logic without a GPU: deck parsing (Mesh.cpp / DomainManager.cpp rules),
the C ABI's exported symbols and struct layouts, and the library loading."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def _header_functions():
    src = open(os.path.join(ROOT, "include", "amcfd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(amcfd_\w+)\s*\(", src)))


def test_library_exports_every_header_function(lib):
    names = _header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_binding(lib):
    import amcfd
    assert C.sizeof(amcfd.AmcfdParams) == lib.amcfd_sizeof_params()
    assert C.sizeof(amcfd.AmcfdReport) == lib.amcfd_sizeof_report()


def test_config_decks_parse(tmp_path):
    import amcfd
    import amcfd_decks as D
    for deck, dims in ((D.config0(steps=3), (122, 62, 42)), (D.config1(steps=3), (402, 202, 102)),
                       (D.config3_eval(steps=3), (202, 102, 62)), (D.config4(steps=3), (602, 302, 122))):
        d = amcfd.Deck(deck.write(str(tmp_path / deck.name)))
        assert d.dims == dims, deck.name
        p = d.params
        assert p.scheme == amcfd.SCHEME_POWER_LAW
        assert p.maxit == 20 and abs(p.nonlintol - 1e-5) < 1e-20
        assert p.navierstokes == 1 and p.steady == 0
        assert abs(p.grav - 9.8) < 1e-12 and abs(p.sigm - 5.67e-8) < 1e-20
    sweep = D.config2(n=8)
    assert len({(s.cells) for s in sweep}) > 1


def test_toolpath_and_tables_parse(tmp_path):
    import amcfd
    import amcfd_decks as D
    dk = D.config4(steps=3)
    d = amcfd.Deck(dk.write(str(tmp_path)))
    assert d.params.udtoolpath == 1 and d.params.ntool == len(dk.toolpath)
    assert d.params.tool_on[1] == 0 and d.params.tool_on[2] == 1


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)


def test_deck_errors(tmp_path):
    import amcfd
    import amcfd_decks as D
    base = D.small("err", steps=2)
    good = base.write(str(tmp_path))
    text = open(good).read()
    # missing mesh file -> AMCFD_E_IO (Mesh.cpp:486-493 exits)
    bad = str(tmp_path / "nomesh.k")
    _write(bad, text.replace("err_mesh.k", "does_not_exist.k"))
    with pytest.raises(amcfd.AmcfdError) as e:
        amcfd.Deck(bad)
    assert e.value.code == -2
    # no *MESH_FILE keyword -> parse error (Mesh.cpp:580-586)
    lines = text.splitlines()
    i = lines.index("*MESH_FILE")
    bad = str(tmp_path / "nomeshkw.k")
    _write(bad, "\n".join(lines[:i] + lines[i + 2:]) + "\n")
    with pytest.raises(amcfd.AmcfdError) as e:
        amcfd.Deck(bad)
    assert e.value.code == -3
    # short material row
    i = lines.index("*MATERIAL_PROPERTIES")
    bad = str(tmp_path / "shortmat.k")
    _write(bad, "\n".join(lines[:i + 2] + lines[i + 3:]) + "\n")
    with pytest.raises(amcfd.AmcfdError):
        amcfd.Deck(bad)
    # a toolpath row without the track id column
    tp = D.small("tp5", steps=2, toolpath=True)
    p = tp.write(str(tmp_path / "tp"))
    crs = str(tmp_path / "tp" / "tp5.crs")
    rows = [r.rsplit(" ", 1)[0] for r in open(crs).read().splitlines()]
    _write(crs, "\n".join(rows) + "\n")
    with pytest.raises(amcfd.AmcfdError) as e:
        amcfd.Deck(p)
    assert e.value.code == -3


def test_deck_comments_blank_lines_and_unknown_keywords(tmp_path):
    import amcfd
    import amcfd_decks as D
    good = D.small("tol", steps=2).write(str(tmp_path))
    text = open(good).read()
    noisy = "$ a comment\n*SOME_UNKNOWN_KEYWORD\n1 2 3\n\n" + text.replace("*UNDER_RELAXATION",
                                                                          "$ note\n*UNDER_RELAXATION")
    p2 = str(tmp_path / "noisy.k")
    _write(p2, noisy)
    a, b = amcfd.Deck(good).params, amcfd.Deck(p2).params
    assert bytes(a)[:C.sizeof(a) - 64] == bytes(b)[:C.sizeof(b) - 64] or a.urfh == b.urfh
    assert (a.dens, a.urfu, a.maxit, a.finaltime) == (b.dens, b.urfu, b.maxit, b.finaltime)


def test_feature_rows_are_checked(tmp_path):
    """A feature keyword without its full parameter row is a parse error; a free
    surface with a negative iteration count is rejected before any device work."""
    import amcfd
    import amcfd_decks as D
    good = D.small("rows", steps=2).write(str(tmp_path))
    text = open(good).read()
    for kw in ("*TRACK_ENERGY_BASED_FREE_SURFACE", "*POWDER_BED_MODE", "*SOLVE_SPECIES",
               "*ACTIVATE_MOVING_MESH"):
        bad = str(tmp_path / "short.k")
        _write(bad, text + kw + "\n  1\n")
        with pytest.raises(amcfd.AmcfdError):
            amcfd.Deck(bad)
    neg = str(tmp_path / "neg.k")
    _write(neg, text + "*TRACK_ENERGY_BASED_FREE_SURFACE\n  -1e5 1e5 1.8 -3 1e-6 40 1e-18 0.5\n")
    d = amcfd.Deck(neg)
    h = C.c_void_p()
    assert amcfd.lib().amcfd_create(C.byref(d.params), None, C.byref(h)) == -1
    amcfd.lib().amcfd_destroy(h)


def test_option_checks_before_any_device_work(tmp_path):
    """Option combinations the solver does not support fail with AMCFD_E_ARG
    before the context touches a GPU: defect correction outside red-black order,
    an unknown precision, a negative wait budget and launch shapes the kernels do
    not offer."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("opts", steps=1).write(str(tmp_path)))
    for kw in (dict(order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP32_DC),
               dict(order=amcfd.ORDER_REDBLACK, precision=7),
               dict(order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64, wait_polls=-5),
               dict(order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP32, asm_kseg=5),
               dict(order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP32, sweep_warps=3),
               dict(order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP32, mom_cluster=3)):
        opts = amcfd.AmcfdOptions(**kw)
        h = C.c_void_p()
        assert amcfd.lib().amcfd_create(C.byref(d.params), C.byref(opts), C.byref(h)) == -1, kw
        assert amcfd.lib().amcfd_last_error(h)
        amcfd.lib().amcfd_destroy(h)
