"""Multi-rank host logic on CPU (gloo, world size 2): tile sharding, peak-range splits, the
end-of-run catalog gather (MPIExt.jl:1041-1063 mirror), max-over-ranks timing, the bench's
whole-job end-to-end aggregate, and a rank that leaves before the gather.  The per-rank compute is the CPU oracle standing in for the
device collapse, so the test checks the plumbing: a catalog split over ranks and gathered
equals the one-rank catalog record for record."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, GOLDEN, load_package

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, port, timeout_s=30):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _tile(seed=7, n=36):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.arange(1, n + 1),) * 3, indexing="ij")
    d = 0.08 * rng.standard_normal((n, n, n))
    for c in rng.integers(9, n - 8, size=(10, 3)):
        d += 2.5 * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / 10.0)
    d = d.astype(np.float32)
    eta = [(0.3 * rng.standard_normal(d.shape)).astype(np.float32) for _ in range(6)]
    return d, eta


def _catalog(pi, pj, pk, d, eta, alatt=1.0, Rf=3.0):
    sys.path.insert(0, ROOT)
    import oracle
    ht = load_package()
    tab, axes = ht.read_homeltab(os.path.join(GOLDEN, "HomelTab_julia.dat"))
    ct = oracle.CollapseTable(tab, *axes)
    F = oracle.Fields(d, *eta)
    shells = oracle.precompute_shells(5)
    res, _ = oracle.analyse_batch(F, pi, pj, pk, ht.ir2min_of(Rf, alatt), Rf, 1.0, 1.2,
                                  alatt, ct, shells, nbuff=6, kind="cudakernel", nthreads=1)
    n = d.shape[0]
    cen = 0.5 * (n + 1)
    x, y, z = (100.0 + alatt * (np.asarray(v, np.float64) - cen) for v in (pi, pj, pk))
    results = {k: res[k].reshape(len(pi), -1) for k in ("RTHL", "Fbarx", "Sbar", "Sbar2")}
    results = {k: (v[:, 0] if v.shape[1] == 1 else v) for k, v in results.items()}
    return ht.dist.halo_records(x, y, z, results, alatt, D=0.8, coef2=-0.3)


def _peaks():
    sys.path.insert(0, ROOT)
    import oracle
    d, eta = _tile()
    pi, pj, pk, _ = oracle.find_peaks(d, np.zeros(d.shape, np.int8), 6, 0.8)
    return d, eta, np.asarray(pi), np.asarray(pj), np.asarray(pk)


def _worker_split(rank, port, q):
    try:
        dist = _init(rank, port)
        ht = load_package()
        d, eta, pi, pj, pk = _peaks()
        lo, hi = ht.dist.peak_range(len(pi), rank, WORLD)
        local = _catalog(pi[lo:hi], pj[lo:hi], pk[lo:hi], d, eta)
        full = ht.dist.gather_records(local)
        tmax = ht.dist.max_over_ranks(10.0 + rank)
        tot = ht.dist.sum_over_ranks(float(hi - lo))
        q.put((rank, None if full is None else full.tobytes(), tmax, tot, len(pi)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:          # report instead of hanging the parent
        q.put((rank, "ERR " + repr(e), None, None, None))


def _run(target, *extra):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=target, args=(r, port, q) + extra) for r in range(WORLD)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(WORLD):
        r = q.get(timeout=180)
        out[r[0]] = r
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out, [p.exitcode for p in ps]


def test_tiles_round_robin(ht):
    for ntiles in (0, 1, 5, 8, 13):
        for world in (1, 2, 3, 8):
            got = [ht.dist.tiles_for_rank(ntiles, r, world) for r in range(world)]
            flat = sorted(t for g in got for t in g)
            assert flat == list(range(ntiles))
            # mod1(i, n_workers) == w with 1-based tiles and workers
            for r, g in enumerate(got):
                assert all(((t + 1 - 1) % world) + 1 == r + 1 for t in g)
    with pytest.raises(ValueError):
        ht.dist.tiles_for_rank(4, 2, 2)


def test_peak_range_partition(ht):
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            rs = [ht.dist.peak_range(n, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1


def test_halo_records_packing(ht):
    rng = np.random.default_rng(3)
    n = 9
    res = {"RTHL": rng.uniform(0.5, 4, n).astype(np.float32),
           "Fbarx": rng.uniform(1, 3, n).astype(np.float32),
           "Sbar": rng.standard_normal(3 * n).astype(np.float32),
           "Sbar2": rng.standard_normal(3 * n).astype(np.float32)}
    res["RTHL"][[2, 5]] = -1.0
    x, y, z = (rng.uniform(0, 100, n) for _ in range(3))
    alatt, D, c2 = 1.4648, 0.77, -0.25
    got = ht.dist.halo_records(x, y, z, res, alatt, D=D, coef2=c2, ilpt=2)
    rows = []
    for p in range(n):
        if res["RTHL"][p] <= 0:
            continue
        s = res["Sbar"][3 * p:3 * p + 3] * np.float32(D)
        s2 = res["Sbar2"][3 * p:3 * p + 3] * np.float32(c2)
        rows.append([np.float32(x[p]), np.float32(y[p]), np.float32(z[p]), *s,
                     np.float32(float(res["RTHL"][p]) * alatt), *s2, res["Fbarx"][p]])
    assert got.dtype == np.float32 and got.shape == (n - 2, 11)
    np.testing.assert_array_equal(got, np.array(rows, np.float32))
    got1 = ht.dist.halo_records(x, y, z, res, alatt, D=D, coef2=c2, ilpt=1)
    assert np.all(got1[:, 7:10] == 0)


def test_split_catalog_equals_single_rank(ht):
    d, eta, pi, pj, pk = _peaks()
    assert len(pi) >= 4
    whole = _catalog(pi, pj, pk, d, eta)
    out, codes = _run(_worker_split)
    assert codes == [0] * WORLD, out
    assert not isinstance(out[0][1], str), out[0][1]
    got = np.frombuffer(out[0][1], np.float32).reshape(-1, 11)
    assert out[1][1] is None
    np.testing.assert_array_equal(got, whole)
    assert out[0][2] == out[1][2] == 11.0
    assert out[0][3] == out[1][3] == float(len(pi))


def _worker_e2e(rank, port, q):
    try:
        dist = _init(rank, port)
        ht = load_package()
        # rank r: 100 (r + 1) units per step over 4 steps of 10 (r + 1) ms
        mine = {"value": 100.0 * (rank + 1) / (10.0 * (rank + 1) / 1e3), "unit": "u/s",
                "ms_per_step": 10.0 * (rank + 1), "steps": 4,
                "h2d_bytes_per_step": 1000 * (rank + 1), "d2h_bytes_per_step": 7}
        got = ht.dist.aggregate_e2e(mine)
        q.put((rank, got, None, None, None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:
        q.put((rank, "ERR " + repr(e), None, None, None))


def test_e2e_aggregates_over_ranks(ht):
    """The bench's whole-job end-to-end line at N ranks: all ranks' units over the slowest
    rank's time, the copied bytes summed (and the one-rank line unchanged)."""
    one = {"value": 5.0, "ms_per_step": 2.0, "steps": 3, "h2d_bytes_per_step": 1,
           "d2h_bytes_per_step": 2}
    assert ht.dist.aggregate_e2e(one) == one
    out, codes = _run(_worker_e2e)
    assert codes == [0] * WORLD, out
    for r in range(WORLD):
        got = out[r][1]
        assert not isinstance(got, str), got
        assert got["ms_per_step"] == 20.0 and got["ranks"] == WORLD
        assert abs(got["value"] - (100.0 + 200.0) / 0.020) < 1e-9
        assert got["h2d_bytes_per_step"] == 3000 and got["d2h_bytes_per_step"] == 14


def _worker_leaves(rank, port, q):
    """Rank 1 leaves between steps, before the gather; rank 0 must get an error from its
    next collective within the process-group timeout instead of waiting for good."""
    try:
        dist = _init(rank, port, timeout_s=5)
        ht = load_package()
        dist.barrier()                      # one step completed by both ranks
        if rank == 1:
            q.put((rank, "left", None, None, None))
            q.close()
            q.join_thread()                 # flush the message before leaving
            os._exit(0)                     # no collective in flight
        try:
            ht.dist.gather_records(np.zeros((3, 11), np.float32))
            q.put((rank, "no error", None, None, None))
        except Exception as e:
            q.put((rank, "error: " + type(e).__name__, None, None, None))
        q.close()
        q.join_thread()
        os._exit(0)
    except Exception as e:
        q.put((rank, "ERR " + repr(e), None, None, None))


def test_rank_leaving_is_reported(ht):
    out, codes = _run(_worker_leaves)
    assert out[1][1] == "left"
    assert out[0][1].startswith("error"), out[0][1]
