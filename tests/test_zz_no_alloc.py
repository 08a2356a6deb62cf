"""The allocation-free energy residual, checked against the solver's own.

amcfd_energy_residual_noalloc serves callers that cannot let the library
allocate device memory (their own memory pool owns the GPU, or a fixed memory
budget).  They pass device buffers they allocated; the library keeps its scratch
in a fixed device array.  This test hands it the coefficients the solver just
assembled and compares with the residual the solver reported for the same
state, on two calls in a row (two outer iterations, so the second call sees new
data in the shared scratch), and checks the size limit.  The file is named to be
collected last.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # two FP64 sums of the same terms in different orders


def _fn():
    import amcfd
    f = amcfd.lib().amcfd_energy_residual_noalloc
    f.argtypes = [C.c_void_p] * 9 + [C.c_int] * 4 + [C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_energy_residual_noalloc_matches_solver(tmp_path):
    import torch

    import amcfd
    import amcfd_decks as D

    fn = _fn()
    deck = amcfd.Deck(D.small("noalloc", steps=2).write(str(tmp_path)))
    s = amcfd.Solver(deck, order=amcfd.ORDER_EXACT, precision=amcfd.PREC_FP64)
    nk, nj, ni = s.shape
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    s.run_phase("laser")
    for call in range(2):
        rep = s.run_phase("energy_assemble")
        bufs = [torch.from_numpy(s.get(n)).cuda().contiguous()
                for n in ("an", "as", "ae", "aw", "at", "ab", "ap", "su", "enthalpy")]
        rc = fn(*[b.data_ptr() for b in bufs], ni, nj, nk, ni, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got, want = float(out.item()), rep["resorh"]
        assert want > 0
        assert abs(got - want) <= TOL * abs(want), (call, got, want)
        for ph in ("energy_solve", "h2t", "meltpool", "momentum", "converge"):
            s.run_phase(ph)
    # beyond the fixed scratch capacity: rejected before anything is launched
    rc = fn(*[bufs[0].data_ptr()] * 9, ni, nj, 4096 + 3, ni, out.data_ptr(), stream)
    assert rc == -8  # AMCFD_E_CAPACITY
    s.close()
