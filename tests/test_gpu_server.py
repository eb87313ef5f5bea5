"""The NEST Server on the GPU: a network built, simulated and read through
the reference's /api/<call> routes gives the same raster as the same calls
made directly; networks submitted to the serving routes while others run
give, each, the spikes they give alone (continuous batching changes no
result)."""

import time

import numpy as np
import pytest

from test_server import _req, server  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _build_and_run(call):
    call("ResetKernel", {})
    call("SetKernelStatus", {"params": {"rng_seed": 12}})
    pop = call("Create", {"model": "iaf_psc_exp", "n": 400, "params": {"I_e": 0.0}})
    call("Connect", {"pre": pop, "post": pop, "conn_spec": {"rule": "fixed_indegree", "indegree": 40},
                     "syn_spec": {"weight": 40.0, "delay": 1.5}})
    pg = call("Create", {"model": "poisson_generator", "params": {"rate": 12000.0}})
    call("Connect", {"pre": pg, "post": pop, "syn_spec": {"weight": 40.0, "delay": 1.5}})
    sr = call("Create", {"model": "spike_recorder"})
    call("Connect", {"pre": pop, "post": sr})
    call("Simulate", {"t": 300.0})
    return call("GetStatus", {"nodes": sr, "keys": "events"})


def test_api_routes_equal_direct_calls(server):  # noqa: F811
    def via_http(name, kw):
        st, d = _req(f"{server}/api/{name}", body=kw)
        assert st == 200, d
        return d

    def direct(name, kw):
        import nestgpu
        from nestgpu.server import nestify, serialize

        fn = getattr(nestgpu, name)
        args, kwargs = nestify(fn, [], dict(kw))
        return serialize(fn(*args, **kwargs))

    a = _build_and_run(via_http)
    b = _build_and_run(direct)
    ev_a = a[0] if isinstance(a, list) else a
    ev_b = b[0] if isinstance(b, list) else b
    assert len(ev_a["senders"]) > 200
    oa = np.lexsort((ev_a["senders"], ev_a["times"]))
    ob = np.lexsort((ev_b["senders"], ev_b["times"]))
    np.testing.assert_array_equal(np.asarray(ev_a["senders"])[oa], np.asarray(ev_b["senders"])[ob])
    np.testing.assert_array_equal(np.asarray(ev_a["times"])[oa], np.asarray(ev_b["times"])[ob])


def test_serving_routes_continuous_batching():
    from nestgpu import serving
    from nestgpu.server import NestServer

    srv = NestServer("127.0.0.1", 0, serving_capacity=(100_000, 40_000_000)).start()
    url = f"http://127.0.0.1:{srv.port}"
    try:
        specs = [dict(n=3000, g=4.0, eta=1.6, t_ms=600.0, seed=5), dict(n=5000, g=5.5, eta=1.3, t_ms=300.0, seed=6),
                 dict(n=2000, g=3.5, eta=1.9, t_ms=450.0, seed=7)]
        ids = []
        for sp in specs:
            st, d = _req(url + "/serving/submit", body=sp)
            assert st == 200
            ids.append(d["request"])
            time.sleep(0.05)              # arrivals while the others run
        results = {}
        deadline = time.time() + 120
        while len(results) < len(ids) and time.time() < deadline:
            for rid in ids:
                st, d = _req(f"{url}/serving/result/{rid}?spikes=1")
                assert st == 200
                if d["status"] == "done":
                    results[rid] = d
            time.sleep(0.1)
        assert len(results) == len(ids)
        st, stats = _req(url + "/serving/stats")
        assert stats["done"] == 3 and stats["live"] == 0
    finally:
        srv.stop()
    # each network alone, in a fresh serving engine: identical spikes
    for rid, sp in zip(ids, specs):
        b = serving.OnlineBatcher(capacity_neurons=100_000, capacity_edges=40_000_000)
        try:
            k = b.submit(**sp)
            while b.result(k)["status"] != "done":
                time.sleep(0.05)
            alone = b.result(k, spikes=True)
        finally:
            b.close()
        mix = results[rid]
        assert alone["spikes"] == mix["spikes"] > 100
        o1 = np.lexsort((alone["senders"], alone["times_ms"]))
        o2 = np.lexsort((np.asarray(mix["senders"]), np.asarray(mix["times_ms"])))
        np.testing.assert_array_equal(np.asarray(alone["senders"])[o1], np.asarray(mix["senders"])[o2])
        np.testing.assert_array_equal(np.asarray(alone["times_ms"])[o1], np.asarray(mix["times_ms"])[o2])
