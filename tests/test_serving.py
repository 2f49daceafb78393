"""The serving loop (mc_b200_server): block, region and chunk requests batched
behind the HBM decoded-block cache must return exactly what the plain per-call
reads return -- alone, in a mix, after evictions, and for host outputs -- and
what the oracle decodes from the archive file's own blobs."""
import numpy as np
import pytest

from mcb200 import REQ_BLOCK, REQ_CHUNK, REQ_REGION, Server

pytestmark = pytest.mark.gpu
CHUNK = 256 ** 3


@pytest.fixture(scope="module")
def archive(gpu, tmp_path_factory):
    """A 2x2x2-chunk LOD-0 volume at q=6 with one chunk never written and one
    all-air chunk, plus two LOD-1 chunks."""
    import torch
    import volumes
    path = str(tmp_path_factory.mktemp("srv") / "s.mca")
    a = gpu.open(path, 512, 512, 512, 6.0)
    coords, vox = [], []
    for cz in range(2):
        for cy in range(2):
            for cx in range(2):
                if (cz, cy, cx) == (1, 1, 0):
                    continue   # absent
                v = volumes.region(11, (cz * 256, cy * 256, cx * 256), (256, 256, 256), 0.4, device="cuda")
                if (cz, cy, cx) == (0, 1, 1):
                    v.zero_()   # all air
                coords.append((cz, cy, cx))
                vox.append(v.contiguous())
    assert a.append_chunks(0, coords, [v.data_ptr() for v in vox], 6.0, on_device=True) == 0
    l1 = [volumes.region(12, (0, 0, 256 * i), (256, 256, 256), 0.3, device="cuda").contiguous() for i in range(2)]
    assert a.append_chunks(1, [(0, 0, 0), (0, 0, 1)], [v.data_ptr() for v in l1], 3.0, on_device=True) == 0
    torch.cuda.synchronize()
    a.path = path
    yield a
    a.close()


def mixed_requests(rng, n):
    """(kind, lod, z, y, x, dz, dy, dx) tuples: blocks, regions (unaligned, across
    chunk borders, partly outside the volume) and chunks."""
    out = []
    for i in range(n):
        k = i % 10
        if k < 6:
            out.append((REQ_BLOCK, 0, *(int(v) for v in rng.integers(0, 32, 3)), 0, 0, 0))
        elif k < 8:
            z0, y0, x0 = (int(v) for v in rng.integers(-40, 480, 3))
            dz, dy, dx = (int(v) for v in rng.integers(1, 96, 3))
            out.append((REQ_REGION, 0, z0, y0, x0, dz, dy, dx))
        elif k == 8:
            out.append((REQ_CHUNK, 0, *(int(v) for v in rng.integers(0, 2, 3)), 0, 0, 0))
        else:
            out.append((REQ_BLOCK, 1, 0, int(rng.integers(0, 16)), int(rng.integers(0, 32)), 0, 0, 0))
    return out


def expected(a, r):
    kind, lod, z, y, x, dz, dy, dx = r
    if kind == REQ_BLOCK:
        co = a.chunk_offset(lod, z >> 4, y >> 4, x >> 4)
        return a.decode_block(co, z & 15, y & 15, x & 15) if co > 1 else np.zeros(4096, np.uint8)
    if kind == REQ_CHUNK:
        return a.decode_chunk(a.chunk_offset(lod, z, y, x))
    return a.read_region(lod, z, y, x, dz, dy, dx)


def nbytes(r):
    kind, _, _, _, _, dz, dy, dx = r
    return 4096 if kind == REQ_BLOCK else (CHUNK if kind == REQ_CHUNK else dz * dy * dx)


def run(srv, reqs):
    import torch
    outs = [torch.full((nbytes(r),), 0xEE, dtype=torch.uint8, device="cuda") for r in reqs]
    tickets = [srv.submit(Server.request(r[0], r[1], r[2], r[3], r[4], o.data_ptr(), r[5], r[6], r[7]))
               for r, o in zip(reqs, outs)]
    assert all(t >= 0 for t in tickets)
    for t in tickets:
        assert srv.wait(t) == 0
    return [o.cpu().numpy() for o in outs]


def test_mix_matches_plain_reads(archive):
    rng = np.random.default_rng(5)
    reqs = mixed_requests(rng, 60)
    with Server(archive, 256 << 20, 64 << 20) as srv:
        got = run(srv, reqs)
        st = srv.stats()
    for r, g in zip(reqs, got):
        assert np.array_equal(g, expected(archive, r)), r
    assert st["requests"] == len(reqs) and st["misses"] > 0 and st["zero_blocks"] > 0


def test_alone_equals_in_mix(archive):
    rng = np.random.default_rng(6)
    reqs = mixed_requests(rng, 30)
    with Server(archive, 256 << 20, 64 << 20) as srv:
        mixed = run(srv, reqs)
    with Server(archive, 256 << 20, 64 << 20) as srv:
        alone = [run(srv, [r])[0] for r in reqs]
    for r, m, a1 in zip(reqs, mixed, alone):
        assert np.array_equal(m, a1), r


def test_small_cache_evicts(archive):
    """A cache of 6000 blocks (less than two chunks): chunk requests evict
    blocks of earlier requests; repeated blocks hit when still resident."""
    rng = np.random.default_rng(7)
    reqs = mixed_requests(rng, 40) + [(REQ_BLOCK, 0, 3, 4, 5, 0, 0, 0)] * 3
    with Server(archive, 6000 * 4096, 8 << 20) as srv:
        got = run(srv, reqs)
        st = srv.stats()
    for r, g in zip(reqs, got):
        assert np.array_equal(g, expected(archive, r)), r
    assert st["evictions"] > 0 and st["hits"] > 0


def test_region_beyond_a_full_cache_is_refused(archive):
    """A 16 MiB cache (4096 slots) first filled by one chunk: a region over
    that chunk and its neighbour needs both chunks' blocks resident at once,
    more slots than the cache has, so its wait returns -1 rather than waiting
    for a batch that will never come. The neighbour chunk, submitted right
    behind it (often into the same batch), and then the first chunk again are
    served exactly, evicting each other's blocks."""
    import torch
    a_req, b_req = (REQ_CHUNK, 0, 0, 0, 0, 0, 0, 0), (REQ_CHUNK, 0, 0, 0, 1, 0, 0, 0)
    with Server(archive, 16 << 20, 64 << 20) as srv:
        got_a = run(srv, [a_req])[0]
        m_a = srv.stats()["misses"]
        region = torch.empty(256 * 256 * 512, dtype=torch.uint8, device="cuda")
        out_b = torch.full((CHUNK,), 0xEE, dtype=torch.uint8, device="cuda")
        t_r = srv.submit(Server.request(REQ_REGION, 0, 0, 0, 0, region.data_ptr(), 256, 256, 512))
        t_b = srv.submit(Server.request(REQ_CHUNK, 0, 0, 0, 1, out_b.data_ptr()))
        assert t_r >= 0 and t_b >= 0
        assert srv.wait(t_r) == -1
        assert srv.wait(t_b) == 0
        m_b = srv.stats()["misses"] - m_a
        again_a = run(srv, [a_req])[0]
        st = srv.stats()
    assert m_a < 4096 and m_b < 4096 and m_a + m_b > 4096, (m_a, m_b)
    assert st["evictions"] > 0
    want_a = expected(archive, a_req)
    assert np.array_equal(got_a, want_a) and np.array_equal(again_a, want_a)
    assert np.array_equal(out_b.cpu().numpy(), expected(archive, b_req))


def test_host_outputs(archive):
    rng = np.random.default_rng(8)
    reqs = mixed_requests(rng, 20)
    with Server(archive, 64 << 20, 32 << 20, on_device=False) as srv:
        outs = [np.full(nbytes(r), 0xEE, np.uint8) for r in reqs]
        tk = [srv.submit(Server.request(r[0], r[1], r[2], r[3], r[4], o.ctypes.data, r[5], r[6], r[7]))
              for r, o in zip(reqs, outs)]
        for t in tk:
            assert srv.wait(t) == 0
        # a strided region is refused for host outputs
        bad = Server.request(REQ_REGION, 0, 0, 0, 0, outs[0].ctypes.data, 4, 4, 4, sz=100, sy=10)
        assert srv.submit(bad) == -1
    for r, o in zip(reqs, outs):
        assert np.array_equal(o, expected(archive, r)), r


def test_replay_trace(archive):
    """Poisson arrivals through the native replay driver: every request
    completes, latencies are positive, results are exact."""
    import torch
    rng = np.random.default_rng(9)
    reqs = mixed_requests(rng, 200)
    outs = [torch.empty(nbytes(r), dtype=torch.uint8, device="cuda") for r in reqs]
    rq = [Server.request(r[0], r[1], r[2], r[3], r[4], o.data_ptr(), r[5], r[6], r[7]) for r, o in zip(reqs, outs)]
    arrivals = np.cumsum(rng.exponential(20e3, len(reqs))).astype(np.uint64)   # 50k req/s
    with Server(archive, 256 << 20, 64 << 20) as srv:
        rc, lat = srv.replay(rq, arrivals)
        st = srv.stats()
    assert rc == 0 and (lat > 0).all()
    assert st["batches"] > 1
    for i in range(0, len(reqs), 17):
        assert np.array_equal(outs[i].cpu().numpy(), expected(archive, reqs[i])), reqs[i]


def _oracle_volume(oracle, arch, lod, cz, cy, cx, cache):
    """Chunk (lod, cz, cy, cx) decoded by the oracle from the archive file's own
    blob bytes (zeros for an absent or all-air chunk)."""
    import shapes
    key = (lod, cz, cy, cx)
    if key not in cache:
        data = cache.setdefault("data", open(arch.path, "rb").read())
        co = arch.chunk_offset(lod, cz, cy, cx)
        if co <= 1:
            cache[key] = np.zeros((256, 256, 256), np.uint8)
        else:
            cache[key] = oracle.decode_chunk(data[co:co + shapes.blob_len(data, co)]).reshape(256, 256, 256)
    return cache[key]


def _oracle_expected(oracle, arch, r, cache):
    kind, lod, z, y, x, dz, dy, dx = r
    if kind == REQ_BLOCK:
        v = _oracle_volume(oracle, arch, lod, z >> 4, y >> 4, x >> 4, cache)
        bz, by, bx = z & 15, y & 15, x & 15
        return v[bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16].reshape(-1)
    if kind == REQ_CHUNK:
        return _oracle_volume(oracle, arch, lod, z, y, x, cache).reshape(-1)
    out = np.zeros((dz, dy, dx), np.uint8)
    for cz in range(z >> 8, ((z + dz - 1) >> 8) + 1):
        for cy in range(y >> 8, ((y + dy - 1) >> 8) + 1):
            for cx in range(x >> 8, ((x + dx - 1) >> 8) + 1):
                if min(cz, cy, cx) < 0 or max(cz, cy, cx) > 1:
                    continue   # outside the volume: zeros
                v = _oracle_volume(oracle, arch, lod, cz, cy, cx, cache)
                zs, ze = max(z, cz * 256), min(z + dz, cz * 256 + 256)
                ys, ye = max(y, cy * 256), min(y + dy, cy * 256 + 256)
                xs, xe = max(x, cx * 256), min(x + dx, cx * 256 + 256)
                if zs < ze and ys < ye and xs < xe:
                    out[zs - z:ze - z, ys - y:ye - y, xs - x:xe - x] = \
                        v[zs - cz * 256:ze - cz * 256, ys - cy * 256:ye - cy * 256, xs - cx * 256:xe - cx * 256]
    return out.reshape(-1)


def test_served_matches_oracle(archive, oracle):
    """Served results against the oracle's own decode of the archive file's
    blobs (not the library's per-call paths): blocks, regions across chunk
    borders and past the volume, chunks, absent and all-air chunks."""
    rng = np.random.default_rng(10)
    reqs = [r for r in mixed_requests(rng, 60) if r[1] == 0]
    with Server(archive, 256 << 20, 64 << 20) as srv:
        got = run(srv, reqs)
    cache = {}
    for r, g in zip(reqs, got):
        assert np.array_equal(g, _oracle_expected(oracle, archive, r, cache)), r


def test_small_class_reads_large_class_misses(archive):
    """A chunk request (large class) whose blocks are all misses, then block
    requests (small class, another stream) inside that chunk submitted right
    behind it: the block batches find the blocks already assigned to cache
    slots and must wait for the chunk batch's decode before they gather."""
    for trial in range(3):
        reqs = [(REQ_CHUNK, 0, 1, 0, 1, 0, 0, 0)] + \
               [(REQ_BLOCK, 0, 16 + (5 * i) % 16, 3 + i, 16 + (7 * i) % 16, 0, 0, 0) for i in range(12)]
        with Server(archive, 256 << 20, 64 << 20) as srv:
            got = run(srv, reqs)
        for r, g in zip(reqs, got):
            assert np.array_equal(g, expected(archive, r)), (trial, r)

