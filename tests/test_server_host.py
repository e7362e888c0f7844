"""The sketch server's host-side rules without a GPU (shgemm_b200/csrc/server_host.hpp):
tests/cpp/server_host_test.cpp checks the arena's first-fit offset allocator against a map
of 256-byte units and prints the row chunks and tile counts of a set of requests, which are
compared here with the rules as the server documents them."""
import math
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHUNK_FLOPS = 4e11


def _chunk_rows(m, row_next, n, draws, k):
    """All rows left, or a multiple of 128 rows near 4e11 flops (2 m n k over the draws), at
    least 128."""
    left = m - row_next
    rows = int(CHUNK_FLOPS / (2.0 * n * draws * k)) // 128 * 128
    return min(max(rows, 128), left)


def _tiles(rows, cols):
    """128-row tiles times column tiles of the smallest power of two in [32, 256] covering
    the columns."""
    bn = 32
    while bn < 256 and bn < cols:
        bn *= 2
    return math.ceil(rows / 128) * math.ceil(cols / bn)


def test_server_host_rules(tmp_path):
    exe = tmp_path / "server_host_test"
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "shgemm_b200", "csrc"), os.path.join(ROOT, "tests", "cpp", "server_host_test.cpp"),
                    "-o", str(exe)], check=True, env=env)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.splitlines()
    assert lines[0] == "allocator ok"
    chunks = [tuple(int(x) for x in ln.split()[1:]) for ln in lines[1:]]
    assert chunks
    by_request = {}
    for (m, n, draws, k, row, rows, units) in chunks:
        assert rows == _chunk_rows(m, row, n, draws, k)
        assert units == _tiles(rows, n * draws)
        by_request.setdefault((m, n, draws, k), []).append((row, rows))
    for (m, n, draws, k), parts in by_request.items():
        starts = [r for r, _ in parts]
        assert starts[0] == 0 and sum(c for _, c in parts) == m
        assert all(c % 128 == 0 for _, c in parts[:-1])  # later chunks start 128-row (512-byte) aligned
        assert starts == sorted(starts)
    # the largest request of the served stream runs in several chunks, the smallest in one
    assert len(by_request[(65536, 256, 4, 16384)]) == 6
    assert len(by_request[(1024, 64, 4, 1024)]) == 1
