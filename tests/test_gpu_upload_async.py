"""orkan_state_upload_async (include/orkan_dev.h): the copy is enqueued on a caller stream
after the library stream's pending work (queued fused gates included), so that work reads
the old contents and the copy's data is what later library work, ordered after it, sees."""
import numpy as np
import pytest
import torch

from oracle import restate as R
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["pure", "tiled", "packed"])
def test_upload_async_orders_after_pending_work(ork5, kind):
    n = 9
    lt = 5
    ork5.set_stream(torch.cuda.current_stream().cuda_stream)
    st = ork5.plus(kind, n)
    for g, qs, th in W.random_circuit(n, 20, seed=12):   # queued (PURE) or enqueued on the library stream
        ork5.gate(st, g, qs, th)
    v = W.gaussian_pure(n, 3)
    full = v if kind == "pure" else np.outer(v, v.conj())
    host = torch.from_numpy(R.to_storage(kind, full, lt)).pin_memory()
    side = torch.cuda.Stream()
    ork5.upload_async(st, host.data_ptr(), side.cuda_stream)
    torch.cuda.current_stream().wait_event(side.record_event())
    assert np.array_equal(ork5.storage(st), host.numpy())
    # later library work sees the uploaded contents
    ork5.gate(st, "h", (0,))
    want = R.apply_gate(kind, full, "h", (0,))
    assert np.abs(ork5.storage(st) - R.to_storage(kind, want, lt)).max() <= 1e-12
    ork5.free(st)
