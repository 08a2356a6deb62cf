"""Mixed-precision defect correction (AMCFD_PREC_FP32_DC) against plain FP64.

The defect-correction mode keeps every field, property, reduction and the
momentum chain in FP64 and moves only the energy line solves, most of the
bytes of an outer iteration, to FP32: the assembly forms the FP64 defect
r = su + sum a_nb h_nb - ap h of the current enthalpy (the same sum the
reference's enhanceConvergenceSpeed accumulates, CFDSolverManager.cpp:2310-2332),
the red-black passes solve A delta = r with FP32 coefficients, and h += delta in
FP64.  The passes are linear, so this is the FP64 red-black iteration with the
rounding moved from h onto its correction: the fields stay at FP64 level.

Checked here: per step the same outer-iteration count as the plain FP64
red-black solve, melt-pool length, depth and width within 1e-6 relative, T and
h within 1e-7 relative L2 of it, f_l within 1e-6 (a
cell at the solidus moves in or out of the mushy band on a tiny change of T),
velocities within 1e-6 of the norm of the whole velocity field (a component
that only starts to move has no scale of its own) and pressure within 1e-6 of
the largest pressure norm of the run (the first step's pressure is only
starting to build up), and T and h at least 10 times closer to it than the
FP32-bulk mode.  Measured on B200: config 0, T 1.5e-11 against 9.2e-8 (FP32)
after the first step, 2.8e-10 against 1.9e-7 after the fourth; the small deck
2.3e-8 against 5.2e-7.  What is left is the FP32 rounding of the corrections,
about 6e-8 of their size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("temp", "enthalpy", "fracl", "uvel", "vvel", "wvel", "pressure")


def _run(d, prec, steps, **kw):
    import amcfd
    s = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, **kw)
    out = []
    for _ in range(steps):
        r = s.step()
        out.append((r, {f: s.get(f) for f in FIELDS}))
    s.close()
    return out


@pytest.mark.parametrize("deck", ["small", "config0"])
def test_defect_correction_matches_fp64(deck, tmp_path):
    import amcfd
    import amcfd_decks as D
    steps = 4
    dk = D.small("dc", steps=steps, power=350.0) if deck == "small" else D.config0(steps=steps)
    d = amcfd.Deck(dk.write(str(tmp_path)))
    ref = _run(d, amcfd.PREC_FP64, steps, use_graphs=1)
    dc = _run(d, amcfd.PREC_FP32_DC, steps, use_graphs=1)
    f32 = _run(d, amcfd.PREC_FP32, steps, use_graphs=1)
    rows = []
    pmax = max(float(np.linalg.norm(f64["pressure"])) for _, f64 in ref)
    for q in range(steps):
        (r64, f64), (rdc, fdc), (r32, ff) = ref[q], dc[q], f32[q]
        vnorm = float(np.sqrt(sum(np.linalg.norm(f64[f]) ** 2 for f in ("uvel", "vvel", "wvel"))))
        e = {}
        for f in FIELDS:
            ref_n = vnorm if f in ("uvel", "vvel", "wvel") else pmax if f == "pressure" else float(np.linalg.norm(f64[f]))
            ref_n = ref_n if ref_n > 0 else 1.0
            e[f] = (float(np.linalg.norm(fdc[f] - f64[f])) / ref_n, float(np.linalg.norm(ff[f] - f64[f])) / ref_n)
        rows.append((q + 1, rdc, r64, e))
        print(f"{deck} step {q + 1} niter dc {rdc['niter']} fp64 {r64['niter']} fp32 {r32['niter']}: " +
              ", ".join(f"{f} dc {a:.2e} fp32 {b:.2e}" for f, (a, b) in e.items()))
    for q, rdc, r64, e in rows:
        assert rdc["niter"] == r64["niter"], (deck, q, rdc["niter"], r64["niter"])
        for k in ("alen", "depth", "width"):  # interpolated at the solidus: 1.5e-7 measured
            assert abs(rdc[k] - r64[k]) <= 1e-6 * max(abs(r64[k]), 1e-9), (deck, q, k, rdc[k], r64[k])
        for f, (e_dc, e_32) in e.items():
            assert e_dc < (1e-7 if f in ("temp", "enthalpy") else 1e-6), (deck, q, f, e_dc)
            if f in ("temp", "enthalpy") and e_32 > 0:
                assert e_dc * 10 < e_32, (deck, q, f, e_dc, e_32)


def test_defect_correction_device_loop_matches_host_loop(tmp_path):
    """The defect-correction launches inside the step graph (outer iterations
    chained on the device) give the bits of the host-driven loop."""
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("dcloop", steps=5, maxit=11, power=60.0, toolpath=True).write(str(tmp_path)))
    a = _run(d, amcfd.PREC_FP32_DC, 5, use_graphs=1, host_loop=1)
    b = _run(d, amcfd.PREC_FP32_DC, 5, use_graphs=1, host_loop=0)
    c = _run(d, amcfd.PREC_FP32_DC, 5, use_graphs=0)
    for q in range(5):
        for other in (b, c):
            assert a[q][0]["niter"] == other[q][0]["niter"]
            for f in FIELDS:
                assert np.array_equal(a[q][1][f], other[q][1][f]), (q + 1, f)


def test_defect_correction_needs_red_black(tmp_path):
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("dcex", steps=1).write(str(tmp_path)))
    with pytest.raises(amcfd.AmcfdError) as e:
        amcfd.Solver(d, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP32_DC)
    assert e.value.code == -1
