"""Host logic of the Python mirror on the CPU, with the library call replaced
by a fake: a batch forgets a bunch's size only after the library has retired
it, so a failed take can be retried."""
import pytest

from haissinskijulia_b200 import Batch, HaissinskiError
from haissinskijulia_b200 import _lib


class _FakeLib:
    def __init__(self, rc):
        self.rc = rc
        self.calls = 0

    def hj_batch_take(self, handle, bid, z, dE, res):
        self.calls += 1
        return self.rc

    def hj_last_error(self, handle):
        return b"fake failure"


class _FakeCtx:
    def __init__(self, lib):
        self._lib = lib
        self.handle = None

    def last_error(self):
        return "fake failure"


def _batch(rc):
    bt = object.__new__(Batch)          # no device: only the host bookkeeping
    bt.ctx = _FakeCtx(_FakeLib(rc))
    bt.handle = None
    bt.sizes = {7: 5}
    return bt


def test_failed_take_keeps_the_bunch():
    bt = _batch(_lib.HJ_ERR_STATE)
    with pytest.raises(HaissinskiError):
        bt.take(7)
    assert bt.sizes == {7: 5}
    with pytest.raises(HaissinskiError):
        bt.take_device(7, 0, 0)
    assert bt.sizes == {7: 5}


def test_successful_take_forgets_the_bunch():
    bt = _batch(_lib.HJ_OK)
    z, dE, r = bt.take(7)
    assert z.shape == (5,) and dE.shape == (5,) and bt.sizes == {}
    assert bt.ctx._lib.calls == 1


def test_unknown_bunch_is_an_argument_error():
    bt = _batch(_lib.HJ_OK)
    with pytest.raises(HaissinskiError) as e:
        bt.take(8)
    assert e.value.status == _lib.HJ_ERR_ARG
    assert bt.ctx._lib.calls == 0
