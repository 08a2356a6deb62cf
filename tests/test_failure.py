"""Failure detection in the forms that fault no GPU.

The reference has no failure detection: a missing input prints a message and
calls exit(1) (Mesh.cpp:486-493), and a diverging solve runs on with NaN
fields.  Here every device-side wait is bounded and every FP64 reduction is
checked, and the host turns both into error codes:

* a bounded wait that runs out: the exact-order line sweep waits for the
  neighbouring lines of other warps; with a budget of one poll those waits give
  up, the kernel records AMCFD_E_TIMEOUT in the status block and returns, and
  the step fails with that code instead of hanging.  The CUDA context stays
  usable: a new solver in the same process reproduces a clean run bit for bit;
* a non-finite value planted in the enthalpy before a step: the residual
  reduction sees it and the step fails with AMCFD_E_NONFINITE;
* a warm-start prediction that raises the step's initial energy residual is
  rejected (report `fallback` = 1) and the step continues from the state it
  would have had without the network, bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_NONFINITE, E_TIMEOUT = -5, -6
FIELDS = ("temp", "uvel", "vvel", "wvel", "pressure", "enthalpy")


def _deck(tmp, name, **kw):
    import amcfd
    import amcfd_decks as D
    return amcfd.Deck(D.small(name, **kw).write(str(tmp / name)))


@pytest.mark.parametrize("graphs,order,prec", [(0, 0, 0), (1, 0, 0), (1, 1, 1)])
def test_line_wait_budget_runs_out_with_timeout(graphs, order, prec, tmp_path):
    """A line sweep whose waits for neighbouring lines may poll only once fails the
    step with AMCFD_E_TIMEOUT and returns: the exact-order wavefront (FP64) and
    the pipelined red-black passes (FP32)."""
    import amcfd
    d = _deck(tmp_path, "wait", steps=2)
    s = amcfd.Solver(d, order=order, precision=prec, use_graphs=graphs, wait_polls=1)
    with pytest.raises(amcfd.AmcfdError) as e:
        s.step()
    assert e.value.code == E_TIMEOUT, str(e.value)
    assert "device wait gave up" in str(e.value)
    # the context keeps the error: the next step reports it again
    with pytest.raises(amcfd.AmcfdError) as e:
        s.step()
    assert e.value.code == E_TIMEOUT
    s.close()
    # the process's CUDA context is intact: two fresh solvers agree bit for bit
    a = amcfd.Solver(d, order=order, precision=prec, use_graphs=graphs)
    b = amcfd.Solver(d, order=order, precision=prec, use_graphs=0)
    for _ in range(2):
        ra, rb = a.step(), b.step()
        assert ra["niter"] == rb["niter"]
    for f in FIELDS:
        assert np.array_equal(a.get(f), b.get(f)), f
    a.close()
    b.close()


def test_negative_wait_budget_is_rejected(tmp_path):
    import amcfd
    d = _deck(tmp_path, "neg", steps=1)
    with pytest.raises(amcfd.AmcfdError) as e:
        amcfd.Solver(d, wait_polls=-1)
    assert e.value.code == -1


@pytest.mark.parametrize("prec,order,graphs", [(0, 0, 0), (1, 1, 1)])
def test_planted_nan_fails_the_step(prec, order, graphs, tmp_path):
    import amcfd
    d = _deck(tmp_path, "nan", steps=3)
    s = amcfd.Solver(d, order=order, precision=prec, use_graphs=graphs, check_finite=1)
    s.step()
    h = s.get("enthalpy")
    nk, nj, ni = h.shape
    h[nk // 2, nj // 2, ni // 2] = np.nan
    s.set("enthalpy", h)
    with pytest.raises(amcfd.AmcfdError) as e:
        s.step()
    assert e.value.code == E_NONFINITE, str(e.value)
    s.close()


def test_bad_warm_start_prediction_falls_back(tmp_path):
    """An output bias of 50 (an enthalpy increment of about five times the
    liquidus enthalpy everywhere) raises the initial residual: both the full and
    the half increment are rejected every step and the solve is the plain one."""
    import amcfd
    d = _deck(tmp_path, "wsbad", steps=3, nx=32, ny=16, nz=10)
    net = amcfd.Net(seed=5)
    w = net.params()
    w[-16:-14] = 50.0  # last layer: biases of the two outputs used
    net.set_params(w)
    s = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP64)
    plain = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=amcfd.PREC_FP64)
    s.ws_attach(net, amcfd.WS_PREDICT)
    for step in range(3):
        r, rp = s.step(), plain.step()
        assert r["fallback"] == 1, step
        assert r["niter"] == rp["niter"], step
        for f in FIELDS:
            x, y = s.get(f), plain.get(f)
            assert np.array_equal(x, y), (step, f, float(np.max(np.abs(x - y))))
    assert s.ws_stats() == (0, 3)
    s.close()
    plain.close()
    net.close()
