"""Host logic of the Python mirror on the CPU, with the library calls replaced
by fakes.  A batch forgets a bunch exactly when the library has retired it:
hj_batch_take retires a bunch as soon as its results are read back and only
then reports the bunch's own failure (a non-finite result), while a failure
before the read-back (a CUDA error) leaves the bunch in the batch."""
import pytest

from haissinskijulia_b200 import Batch, HaissinskiError
from haissinskijulia_b200 import _lib


class _FakeLib:
    """hj_batch_take / _many that fail with `rc`, retiring the bunches first
    when `retires` is set (the library's behaviour after the read-back)."""

    def __init__(self, rc, retires, live):
        self.rc = rc
        self.retires = retires
        self.live = set(live)
        self.calls = 0

    def hj_batch_stats(self, handle, out4):
        out4[0] = len(self.live)
        return _lib.HJ_OK

    def _take(self, ids):
        self.calls += 1
        if self.rc == _lib.HJ_OK or self.retires:
            self.live -= set(ids)
        return self.rc

    def hj_batch_take(self, handle, bid, z, dE, res):
        return self._take([bid])

    def hj_batch_take_many(self, handle, k, ids, z, dE, res, corr):
        return self._take([ids[i] for i in range(k)])

    def hj_last_error(self, handle):
        return b"fake failure"


class _FakeCtx:
    def __init__(self, lib):
        self._lib = lib
        self.handle = None

    def last_error(self):
        return "fake failure"


def _batch(rc, retires=False):
    bt = object.__new__(Batch)          # no device: only the host bookkeeping
    bt.ctx = _FakeCtx(_FakeLib(rc, retires, [7, 9]))
    bt.handle = None
    bt.sizes = {7: 5, 9: 3}
    return bt


def test_take_that_fails_before_the_read_back_keeps_the_bunch():
    bt = _batch(_lib.HJ_ERR_CUDA)
    with pytest.raises(HaissinskiError):
        bt.take(7)
    assert bt.sizes == {7: 5, 9: 3}
    with pytest.raises(HaissinskiError):
        bt.take_device(7, 0, 0)
    assert bt.sizes == {7: 5, 9: 3}
    with pytest.raises(HaissinskiError):
        bt.take_many([7, 9])
    assert bt.sizes == {7: 5, 9: 3}


def test_take_of_a_non_finite_bunch_forgets_it():
    bt = _batch(_lib.HJ_ERR_NONFINITE, retires=True)
    with pytest.raises(HaissinskiError) as e:
        bt.take(7)
    assert e.value.status == _lib.HJ_ERR_NONFINITE
    assert bt.sizes == {9: 3}
    with pytest.raises(HaissinskiError) as e:     # the retired bunch is gone for good
        bt.take(7)
    assert e.value.status == _lib.HJ_ERR_ARG


def test_take_device_of_a_non_finite_bunch_forgets_it():
    bt = _batch(_lib.HJ_ERR_NONFINITE, retires=True)
    with pytest.raises(HaissinskiError):
        bt.take_device(9, 0, 0)
    assert bt.sizes == {7: 5}


def test_take_many_with_a_non_finite_bunch_forgets_all():
    bt = _batch(_lib.HJ_ERR_NONFINITE, retires=True)
    with pytest.raises(HaissinskiError):
        bt.take_many([7, 9])
    assert bt.sizes == {}


def test_successful_take_forgets_the_bunch():
    bt = _batch(_lib.HJ_OK)
    z, dE, r = bt.take(7)
    assert z.shape == (5,) and dE.shape == (5,) and bt.sizes == {9: 3}
    assert bt.ctx._lib.calls == 1
    res, corr = bt.take_many([9])
    assert len(res) == 1 and corr is None and bt.sizes == {}


def test_unknown_bunch_is_an_argument_error():
    bt = _batch(_lib.HJ_OK)
    with pytest.raises(HaissinskiError) as e:
        bt.take(8)
    assert e.value.status == _lib.HJ_ERR_ARG
    assert bt.ctx._lib.calls == 0
