"""Asynchronous field read-out (amcfd_get_field_async + amcfd_wait_reads): the
field lands in host memory as amcfd_get_field would have copied it at the time of
the call, even though the solver steps on meanwhile, and a synchronous read after
an asynchronous one waits for it."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_async_read_matches_sync_read(prec, deckdir):
    import torch
    import amcfd
    import amcfd_decks as D
    d = amcfd.Deck(D.small("asyncread", steps=4, toolpath=True).write(deckdir))
    s = amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, use_graphs=1)
    n = int(np.prod(s.shape))
    bufs = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    for step in range(3):
        s.step()
        want_t, want_h = s.get("temp"), s.get("enthalpy")
        s.get_into_async("temp", bufs[0].data_ptr())
        s.get_into_async("enthalpy", bufs[1].data_ptr())  # waits on the device for the first copy
        s.step()  # changes both fields while the copies may still run
        s.wait_reads()
        assert np.array_equal(bufs[0].numpy().reshape(s.shape), want_t), step
        assert np.array_equal(bufs[1].numpy().reshape(s.shape), want_h), step
        # a synchronous read right after an asynchronous one
        s.get_into_async("temp", bufs[0].data_ptr())
        now = s.get("temp")
        s.wait_reads()
        assert np.array_equal(bufs[0].numpy().reshape(s.shape), now), step
    s.close()
