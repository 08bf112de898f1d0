"""Host staging pool (zkp_host_pool_*, the page-locking part needs a GPU and
is tested in test_staging_gpu.py): chunk hand-out, reuse, misuse and
concurrent use, on plain and mmap'ed blocks."""
import threading

import pytest


@pytest.mark.parametrize("flags", [0, 2])
def test_pool_chunks(zkp, flags):
    H = zkp.host
    pool = H.HostPool(1 << 20, chunks_per_block=3, flags=flags)
    try:
        ps = [pool.alloc(1 << 20) for _ in range(7)]
        assert len(set(ps)) == 7
        assert all(p % 4096 == 0 for p in ps)
        assert pool.stats() == (3, 7)  # three blocks of three chunks
        v = H.HostPool.view(ps[3], 1 << 20)
        v[:] = 7
        assert int(v.sum()) == 7 << 20
        pool.free(ps[3])
        assert pool.alloc(100) == ps[3]  # the freed chunk comes back first
        with pytest.raises(ValueError):
            pool.free(ps[0] + 64)  # not a chunk start
        pool.free(ps[0])
        with pytest.raises(ValueError):
            pool.free(ps[0])  # twice
        with pytest.raises(MemoryError):
            pool.alloc((1 << 20) + 1)  # larger than a chunk
    finally:
        pool.close()


def test_pool_threads(zkp):
    H = zkp.host
    pool = H.HostPool(4096, chunks_per_block=16, flags=0)
    got, lock = [], threading.Lock()

    def worker():
        mine = [pool.alloc(4096) for _ in range(50)]
        for p in mine[::2]:
            pool.free(p)
        with lock:
            got.extend(mine[1::2])

    ts = [threading.Thread(target=worker) for _ in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    try:
        assert len(set(got)) == 100
        assert pool.stats()[1] == 100
    finally:
        pool.close()
