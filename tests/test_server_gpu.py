"""The sort server (sortServer*): requests of mixed sizes, value modes and
bit ranges, from page-locked host memory. Every result must equal the
oracle's, and a request's result must be the same alone and in the mix
(tolerance: exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).pin_memory()


def make_requests(rng, sizes):
    reqs = []
    for i, n in enumerate(sizes):
        keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        keys[::4] &= np.uint32(0x00FFFF00)
        values = np.arange(n, dtype=np.uint32) if i % 2 else None
        end = (16, 24, 32)[i % 3]
        reqs.append((keys, values, end))
    return reqs


def submit_all(server, reqs):
    import torch
    held, tickets = [], []
    for keys, values, end in reqs:
        k = pinned(keys)
        ko = torch.empty_like(k).pin_memory()
        v = pinned(values) if values is not None else None
        vo = torch.empty_like(v).pin_memory() if v is not None else None
        t = server.submit(k.data_ptr(), v.data_ptr() if v is not None else None, keys.size,
                          0, end, ko.data_ptr(), vo.data_ptr() if vo is not None else None)
        held.append((k, ko, v, vo))
        tickets.append(t)
    out = []
    for t, (k, ko, v, vo) in zip(tickets, held):
        st, lat = server.wait(t)
        assert st == 0
        assert lat >= 0
        out.append((ko.numpy().view(np.uint32).copy(),
                    vo.numpy().view(np.uint32).copy() if vo is not None else None))
    return out


def expect(oracle_mod, keys, values, end):
    if values is None:
        k, _ = oracle_mod.sort_stable(keys, [], 0, 0, end)
        return k, None
    k, (v,) = oracle_mod.sort_stable(keys, [values], 1, 0, end)
    return k, v


@pytest.fixture(scope="module")
def server(engine):
    from mgpu_old_b200 import api
    s = api.SortServer(memory_budget=1 << 30, slots=4, coalesce_max=1 << 16)
    yield s
    s.close()


def test_server_results_match_oracle(server, oracle_mod):
    rng = np.random.Generator(np.random.MT19937(1))
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(1), np.log(300_000), 120))]
    reqs = make_requests(rng, sizes)
    out = submit_all(server, reqs)
    for (keys, values, end), (k, v) in zip(reqs, out):
        ek, ev = expect(oracle_mod, keys, values, end)
        assert np.array_equal(k, ek)
        if values is not None:
            assert np.array_equal(v, ev)


def test_same_result_alone_and_in_the_mix(server):
    rng = np.random.Generator(np.random.MT19937(2))
    probes = make_requests(rng, [37, 5000, 70_000, 1_000_000, 3])
    alone = [submit_all(server, [p])[0] for p in probes]
    mix = make_requests(rng, [int(x) for x in rng.integers(1, 200_000, 80)])
    combined = mix[:20] + probes[:2] + mix[20:50] + probes[2:] + mix[50:]
    out = submit_all(server, combined)
    got = out[20:22] + out[52:55]
    for (ak, av), (gk, gv) in zip(alone, got):
        assert np.array_equal(ak, gk)
        assert (av is None and gv is None) or np.array_equal(av, gv)


def test_budget_admission_and_rejection(engine, oracle_mod):
    """With a budget of 4 requests' worth, every request still completes;
    one larger than the whole budget is rejected at submission."""
    from mgpu_old_b200 import api
    budget = 4 * 100_000 * 16
    s = api.SortServer(memory_budget=budget, slots=3, coalesce_max=1 << 12)
    try:
        rng = np.random.Generator(np.random.MT19937(3))
        reqs = make_requests(rng, [100_000] * 12 + [50] * 10)
        out = submit_all(s, reqs)
        for (keys, values, end), (k, v) in zip(reqs, out):
            ek, ev = expect(oracle_mod, keys, values, end)
            assert np.array_equal(k, ek)
            if values is not None:
                assert np.array_equal(v, ev)
        big = pinned(np.zeros(budget, np.uint32))
        with pytest.raises(api.MgpuException) as e:
            s.submit(big.data_ptr(), None, budget, 0, 32, big.data_ptr(), None)
        assert e.value.status == api.SortStatus.CONFIG_NOT_SUPPORTED
    finally:
        s.close()
