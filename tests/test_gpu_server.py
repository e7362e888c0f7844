"""The sketch server: on-device Omega generation, results against the oracle, the same
result alone and in a mix of concurrent requests, and HBM-budget admission. No
reference counterpart (the reference's callers run one shgemm() per sketch)."""
import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu


def _rand_a(rng, m, k):
    import torch

    lda = (m + 3) // 4 * 4 + 4
    A = rng.uniform(-1, 1, lda * k).astype(np.float32)
    return A, lda, torch.from_numpy(A).cuda()


def _omega_host(k, n, draw_seed, fp32, scale, dist=0):
    """Omega of one draw, generated on the device by the library and copied back as binary16."""
    import torch

    from shgemm_b200 import server as srv

    if fp32:
        ld = (k + 3) // 4 * 4
        buf = torch.zeros(n * ld, device="cuda", dtype=torch.float32)
    else:
        ld = (k + 7) // 8 * 8
        buf = torch.zeros(n * ld, device="cuda", dtype=torch.float16)
    srv.generate_omega(buf, ld, k, n, dist, draw_seed, scale, fp32)
    torch.cuda.synchronize()
    om = buf.view(n, ld)[:, :k].cpu().numpy()
    return om.astype(np.float16), om


@pytest.mark.parametrize("dist", [0, 1])
def test_generate_omega(cuda_device, dist):
    from shgemm_b200 import server as srv

    k, n = 4096, 64
    scale = n ** -0.5
    h16, _ = _omega_host(k, n, 7, False, scale, dist)
    h16b, _ = _omega_host(k, n, 7, False, scale, dist)
    h32, raw32 = _omega_host(k, n, 7, True, scale, dist)
    other, _ = _omega_host(k, n, 8, False, scale, dist)
    assert np.array_equal(h16.view(np.uint16), h16b.view(np.uint16))        # deterministic
    assert np.array_equal(h16.astype(np.float32), raw32)                     # widened copy is exact
    assert not np.array_equal(h16, other)                                     # seeds differ
    x = h16.astype(np.float64)
    if dist == srv.GAUSSIAN:
        assert abs(x.mean()) < 5 * scale / np.sqrt(x.size)
        assert abs(x.std() / scale - 1) < 0.02
    else:
        assert np.allclose(np.abs(x), np.float16(scale))
        assert abs(np.mean(x > 0) - 0.5) < 0.01


def _mix64(z):
    """splitmix64's finaliser on numpy uint64 (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def test_gaussian_omega_is_box_muller_pairs_of_the_hash(cuda_device):
    """Entries 2i, 2i + 1 of column c are z cos(2 pi u2), z sin(2 pi u2) with z = sqrt(-2 ln u1)
    and u1, u2 from splitmix64(seed * 0x9E3779B97F4A7C15 + c k + 2i + 1): checked through the
    pair's radius and angle, to the binary16 rounding of the stored values (odd k: the last
    entry of a column is a cosine alone)."""
    from shgemm_b200 import server as srv

    k, n, seed, scale = 301, 7, 99, 1.0
    _, om = _omega_host(k, n, seed, True, scale, srv.GAUSSIAN)
    om = om.astype(np.float64)
    with np.errstate(over="ignore"):
        base = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
    for c in range(n):
        r = np.arange(0, k, 2, dtype=np.uint64)
        with np.errstate(over="ignore"):
            x = _mix64(base + np.uint64(c * k) + r + np.uint64(1))
        u1 = ((x >> np.uint64(40)) + np.uint64(1)).astype(np.float64) * 2.0 ** -24
        u2 = ((x >> np.uint64(16)) & np.uint64(0xFFFFFF)).astype(np.float64) * 2.0 ** -24
        z = np.sqrt(-2.0 * np.log(u1))
        z0 = om[c, 0::2]
        np.testing.assert_allclose(z0, scale * z * np.cos(2 * np.pi * u2), rtol=2e-3, atol=2e-3)
        z1 = om[c, 1::2]
        np.testing.assert_allclose(z1, (scale * z * np.sin(2 * np.pi * u2))[:len(z1)], rtol=2e-3, atol=2e-3)


@pytest.mark.parametrize("fp32", [False, True])
def test_omega_batch_matches_single_calls(cuda_device, fp32):
    """One batched launch writes every job exactly as its own generate_omega call would: mixed
    distributions, seeds, scales, ragged and odd k, leading dimensions past k, an empty job."""
    import torch

    from shgemm_b200 import server as srv

    specs = [(300, 17, srv.GAUSSIAN, 5, 0.25), (301, 3, srv.RADEMACHER, 6, 1.0), (64, 64, srv.RADEMACHER_BLOCKS, 7, 0.5),
             (1, 9, srv.GAUSSIAN, 8, 2.0), (0, 4, srv.GAUSSIAN, 9, 1.0), (4097, 2, srv.GAUSSIAN, 10, 0.125)]
    dt = torch.float32 if fp32 else torch.float16
    bufs1, bufs2, jobs = [], [], []
    for (k, cols, dist, seed, scale) in specs:
        ld = k + 8
        b1 = torch.zeros(max(1, cols * ld), device="cuda", dtype=dt)
        b2 = torch.zeros_like(b1)
        srv.generate_omega(b1, ld, k, cols, dist, seed, scale, fp32)
        jobs.append((b2, ld, k, cols, dist, seed, scale))
        bufs1.append(b1)
        bufs2.append(b2)
    srv.generate_omega_batch(jobs, fp32)
    torch.cuda.synchronize()
    for b1, b2 in zip(bufs1, bufs2):
        assert torch.equal(b1.view(torch.int16 if not fp32 else torch.int32),
                           b2.view(torch.int16 if not fp32 else torch.int32))


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_server_result_matches_oracle(cuda_device, tc):
    import torch

    from shgemm_b200 import server as srv

    rng = np.random.default_rng(40 + tc)
    m, n, k, draws, seed = 333, 48, 777, 3, 12345
    A, lda, A_dev = _rand_a(rng, m, k)
    with srv.SketchServer(0, hbm_budget_bytes=1 << 30, compute_type=tc) as s:
        t = s.submit(m, n, k, A_dev, lda, draws=draws, seed=seed)
        assert s.wait(t) == srv.DONE
        st, y, ldy, lat = s.poll(t)
        assert st == srv.DONE and y and ldy == m and lat >= 0
        Y = _view(y, m * n * draws).clone()
        torch.cuda.synchronize()
        s.release(t)
    Y = Y.cpu().numpy()
    for j in range(draws):
        om16, _ = _omega_host(k, n, srv.draw_seed(seed, j), tc == oracle.TF32, n ** -0.5)
        inp = dict(A=A, B=om16.reshape(-1), C=np.zeros(m * n, np.float32), lda=lda, ldb=k, ldc=m)
        gpu = Y[j * m * n:(j + 1) * m * n]
        orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
        ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        K.assert_parity(K.parity_report(gpu, orc, ref, sgc, m, n, m, 0))


def _view(addr, count):
    """A CUDA float32 tensor over `count` floats at device address `addr` (no copy)."""
    import torch

    class _Buf:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (addr, False), "version": 3}

    return torch.as_tensor(_Buf(), device="cuda")


def test_server_same_result_alone_and_in_the_mix(cuda_device):
    """One request's Y is bit-identical whether it runs alone or among concurrent requests."""
    import torch

    from shgemm_b200 import server as srv

    rng = np.random.default_rng(77)
    m, n, k = 1000, 64, 3000
    _, lda, A_dev = _rand_a(rng, m, k)
    others = []
    for i in range(15):
        mo, ko = int(rng.integers(100, 3000)), int(rng.integers(300, 5000))
        _, ldo, Ao = _rand_a(rng, mo, ko)
        others.append((mo, int(rng.choice([32, 64, 128])), ko, Ao, ldo))
    for tc in (oracle.TF32, oracle.FP16):
        with srv.SketchServer(0, hbm_budget_bytes=2 << 30, compute_type=tc, streams=2) as s:
            t = s.submit(m, n, k, A_dev, lda, draws=4, seed=99)
            s.wait(t)
            _, y, _, _ = s.poll(t)
            alone = _view(y, m * n * 4).clone()
            s.release(t)
            tickets = [s.submit(mo, no, ko, Ao, ldo, draws=4, seed=1000 + i)
                       for i, (mo, no, ko, Ao, ldo) in enumerate(others[:8])]
            t = s.submit(m, n, k, A_dev, lda, draws=4, seed=99)
            tickets += [s.submit(mo, no, ko, Ao, ldo, draws=4, seed=2000 + i)
                        for i, (mo, no, ko, Ao, ldo) in enumerate(others[8:])]
            s.drain()
            st, y, _, _ = s.poll(t)
            assert st == srv.DONE
            mixed = _view(y, m * n * 4).clone()
            assert s.stats()["batches"] >= 2
            for q in tickets + [t]:
                s.release(q)
        torch.cuda.synchronize()
        assert torch.equal(alone, mixed), tc


def test_server_admission_respects_budget(cuda_device):
    from shgemm_b200 import server as srv

    rng = np.random.default_rng(3)
    m, n, k, draws = 2048, 128, 4096, 4
    _, lda, A_dev = _rand_a(rng, m, k)
    per_req = lda * k * 4 + k * n * draws * 4 + m * n * draws * 4
    budget = int(per_req * 2.5)
    with srv.SketchServer(0, hbm_budget_bytes=budget, compute_type=oracle.TF32, auto_release=True) as s:
        tickets = [s.submit(m, n, k, A_dev, lda, draws=draws, seed=i) for i in range(12)]
        s.drain()
        st = s.stats()
        assert st["completed"] == 12 and st["failed"] == 0
        assert 0 < st["peak_resident_bytes"] <= budget
        assert st["resident_bytes"] == 0
        assert st["p99_ms"] >= st["p50_ms"] > 0
        assert all(s.poll(t)[0] == srv.DONE for t in tickets)
        # a request that can never fit is refused at submit
        with pytest.raises(Exception):
            s.submit(m, n, k * 4, A_dev, lda, draws=draws)


def test_server_poisson_stream(cuda_device):
    """A short Poisson stream of uneven requests: all complete, latencies recorded."""
    import time

    from shgemm_b200 import server as srv

    rng = np.random.default_rng(11)
    pool_k, pool_m = 4096, 4096
    _, lda, A_dev = _rand_a(rng, pool_m, pool_k)
    with srv.SketchServer(0, hbm_budget_bytes=4 << 30, compute_type=oracle.TF32, auto_release=True) as s:
        t0 = time.perf_counter()
        due = 0.0
        for i in range(120):
            due += rng.exponential(1 / 2000.0)
            while time.perf_counter() - t0 < due:
                pass
            m = int(np.exp(rng.uniform(np.log(256), np.log(pool_m))))
            k = int(np.exp(rng.uniform(np.log(256), np.log(pool_k))))
            n = int(rng.choice([64, 128, 256]))
            s.submit(m, n, k, A_dev, lda, draws=4, seed=i)
        s.drain()
        st = s.stats()
    assert st["completed"] == 120 and st["failed"] == 0
    assert st["batches"] >= 2
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_large_request_runs_in_chunks_and_small_ones_pass_it(cuda_device):
    """A request of ~2.2e12 flops runs as row chunks in successive launches (up to one per
    server stream in flight): a small request submitted right behind it completes first, and
    the large one's rows on both sides of every chunk boundary match the restated reference
    algorithm."""
    import torch

    from shgemm_b200 import server as srv

    m, n, k, draws, seed = 65536, 256, 16384, 4, 77
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    A_dev = torch.randn(k * m, generator=g, device="cuda")  # column-major m x k, lda = m
    small_m, small_k = 1024, 1024
    S_dev = torch.randn(small_k * small_m, generator=g, device="cuda")
    with srv.SketchServer(0, hbm_budget_bytes=16 << 30, compute_type=oracle.TF32) as s:
        tb = s.submit(m, n, k, A_dev, m, draws=draws, seed=seed)
        ts = s.submit(small_m, 64, small_k, S_dev, small_m, draws=draws, seed=seed + 1)
        assert s.wait(ts) == srv.DONE and s.wait(tb) == srv.DONE
        _, _, _, lat_small = s.poll(ts)
        st, y, ldy, lat_big = s.poll(tb)
        assert st == srv.DONE and ldy == m
        assert lat_small < lat_big  # the small request did not wait for all of the large one
        cols = n * draws
        chunk = int(4e11 / (2.0 * cols * k)) // 128 * 128
        rows = sorted({0, 1, m - 1} | {b + d for b in range(chunk, m, chunk) for d in (-1, 0)})
        Y = _view(y, m * cols).view(cols, m)[:, rows].T.contiguous().cpu().numpy()  # len(rows) x cols
        s.release(tb)
        s.release(ts)
    r = len(rows)
    A_rows = A_dev.view(k, m)[:, rows].contiguous().cpu().numpy().reshape(-1)  # r x k column-major, ld = r
    del A_dev, S_dev
    for j in range(draws):
        om16, _ = _omega_host(k, n, srv.draw_seed(seed, j), True, n ** -0.5)
        inp = dict(A=A_rows, B=om16.reshape(-1), C=np.zeros(r * n, np.float32), lda=r, ldb=k, ldc=r)
        gpu = Y[:, j * n:(j + 1) * n].T.reshape(-1).copy()  # r x n column-major
        orc = K.run_oracle(oracle.TF32, 0, 0, r, n, k, 1.0, inp, 0.0, 0, chunk=0)
        ref = K.fp64(0, 0, r, n, k, 1.0, inp, 0.0, 0)
        sgc = K.sgemm(0, 0, r, n, k, 1.0, inp, 0.0, 0)
        K.assert_parity(K.parity_report(gpu, orc, ref, sgc, r, n, r, 0))
