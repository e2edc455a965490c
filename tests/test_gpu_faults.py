"""Failure handling on the GPU without a GPU fault: errors are injected on
the host (a device allocation that reports failure) or through a bounded wait
that is left to expire (test_gpu_forces.py, test_gpu_batch.py); every call
returns a status and the context stays usable afterwards."""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
FP64, FP32C = 0, 1


def _inject(k):
    os.environ["NBR_TEST_FAIL_ALLOC"] = str(k)


def _clear():
    os.environ.pop("NBR_TEST_FAIL_ALLOC", None)


@pytest.mark.parametrize("k", [1, 3, 5])
def test_failed_allocation_in_upload_is_reported(nbr, oracle, k):
    with nbr.Context(0) as c:
        c.upload(nbr.plummer(1000, 1))
        _inject(k)  # the k-th of the buffers a larger system needs fails
        try:
            with pytest.raises(nbr.NbrError) as e:
                c.upload(nbr.plummer(5000, 1))
            assert e.value.status == 3  # NBR_ERR_NO_MEMORY
        finally:
            _clear()
        with pytest.raises(nbr.NbrError) as e:
            c.forces(FP64)
        assert e.value.status == 5  # the half-allocated system was dropped
        s = nbr.plummer(5000, 1)
        c.upload(s)
        a = c.forces(FP64, eps2=1e-6)
        ref = oracle.accel(s["x"], s["y"], s["z"], s["m"], eps2=1e-6, extended=True)
        assert rel_err(a, ref).max() <= 1e-12


def test_failed_allocation_in_batch_upload_is_reported(nbr):
    off = np.array([0, 300, 900])
    st = {k: np.concatenate([nbr.plummer(300, 1)[k], nbr.plummer(600, 2)[k]]) for k in nbr.KEYS}
    with nbr.Context(0) as c:
        _inject(2)
        try:
            with pytest.raises(nbr.NbrError) as e:
                c.batch_upload(off, st)
            assert e.value.status == 3
        finally:
            _clear()
        c.batch_upload(off, st)
        a = c.batch_forces(FP32C, eps2=1e-6)
        assert np.all(np.isfinite(a)) and np.abs(a).max() > 0


def test_failed_scratch_allocation_in_run_is_reported(nbr):
    """The split scratch grows on the first evaluation of a larger system."""
    with nbr.Context(0) as c:
        s = nbr.plummer(60000, 3)
        c.upload(s)
        _inject(1)
        try:
            with pytest.raises(nbr.NbrError) as e:
                c.run(FP32C, 0, 2, 1e-3, 2, eps2=1e-6)
            assert e.value.status == 3
        finally:
            _clear()
        st = c.run(FP32C, 0, 2, 1e-3, 2, eps2=1e-6)
        assert st["force_evals"] == 3
        out = c.download()
        assert np.all(np.isfinite(out["x"]))
