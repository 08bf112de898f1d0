"""Host staging on the GPU: page-locked huge-page pool chunks and the bounded
copy queue, round trips ordered after work on the caller's stream."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_copy_queue_round_trip(gpu):
    H = gpu.host
    chunk = 4 << 20
    pool = H.HostPool(chunk, chunks_per_block=2, flags=H.HostPool.PIN | H.HostPool.HUGE)
    q = H.CopyQueue(max_in_flight=2)
    try:
        rng = np.random.default_rng(3)
        host = [pool.alloc(chunk) for _ in range(6)]
        vals = [rng.integers(0, 2 ** 62, chunk // 8, dtype=np.int64) for _ in host]
        for p, v in zip(host, vals):
            H.HostPool.view(p, chunk, np.int64)[:] = v
        dev = [torch.empty(chunk // 8, dtype=torch.int64, device="cuda") for _ in host]
        cur = torch.cuda.current_stream()
        for d, p in zip(dev, host):
            q.push(d.data_ptr(), p, chunk, q.H2D, after=cur)
        q.sync()
        for d, v in zip(dev, vals):
            assert (d.cpu().numpy() == v).all()
        # device work queued on the caller's stream, then copies back ordered after it
        for d in dev:
            d.add_(5)
        for d, p in zip(dev, host):
            q.push(p, d.data_ptr(), chunk, q.D2H, after=cur)
        q.sync()
        for p, v in zip(host, vals):
            assert (H.HostPool.view(p, chunk, np.int64) == v + 5).all()
        assert pool.stats() == (3, 6)
    finally:
        q.close()
        pool.close()
