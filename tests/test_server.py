"""The NEST Server routes (nestgpu.server) on the CPU: the reference's
request and response shapes (pynest/nest/server/hl_api_server.py) for calls
that build and inspect a network; Simulate and the serving routes need the
GPU (tests/test_gpu_server.py)."""

import json
import urllib.error
import urllib.request

import pytest


@pytest.fixture
def server():
    from nestgpu.server import NestServer

    srv = NestServer("127.0.0.1", 0).start()
    yield f"http://127.0.0.1:{srv.port}"
    srv.stop()


def _req(url, body=None, form=None):
    data, headers = None, {}
    if body is not None:
        data = json.dumps(body).encode()
        headers["Content-Type"] = "application/json"
    elif form is not None:
        data = form.encode()
        headers["Content-Type"] = "application/x-www-form-urlencoded"
    r = urllib.request.Request(url, data=data, headers=headers, method="POST" if data is not None else "GET")
    try:
        with urllib.request.urlopen(r, timeout=30) as resp:
            return resp.status, json.loads(resp.read())
    except urllib.error.HTTPError as err:
        return err.code, json.loads(err.read())


def test_index_and_call_list(server):
    st, d = _req(server + "/")
    assert st == 200 and d["mpi"] is False and "nest" in d
    st, calls = _req(server + "/api")
    assert st == 200 and {"Create", "Connect", "Simulate", "GetStatus", "GetConnections"} <= set(calls)
    assert calls == sorted(calls)


def test_build_and_inspect_a_network(server):
    assert _req(server + "/api/ResetKernel", body={})[0] == 200
    st, ids = _req(server + "/api/Create", body={"model": "iaf_psc_exp", "n": 3, "params": {"I_e": 376.0}})
    assert st == 200 and ids == [1, 2, 3]
    st, ids2 = _req(server + "/api/Create", form="model=iaf_psc_delta&n=2")   # form arguments
    assert st == 200 and ids2 == [4, 5]
    st, _ = _req(server + "/api/Connect", body={"pre": [1], "post": [2, 3], "syn_spec": {"weight": 20.0,
                                                                                       "delay": 1.5}})
    assert st == 200
    st, vals = _req(server + "/api/GetStatus", body={"nodes": [1, 2], "keys": "I_e"})
    assert st == 200 and vals == [376.0, 376.0]
    st, conns = _req(server + "/api/GetConnections", body={"source": [1]})
    assert st == 200
    assert sorted(conns["target"]) == [2, 3] and conns["weight"] == [20.0, 20.0]
    st, ks = _req(server + "/api/GetKernelStatus", body={"keys": "resolution"})
    assert st == 200 and ks == 0.1


def test_errors_are_reported_as_the_reference_does(server):
    st, d = _req(server + "/api/Create", body={"model": "no_such_model"})
    assert st == 400 and "message" in d and d["lineno"] == -1
    st, d = _req(server + "/api/NoSuchCall", body={})
    assert st == 400
    st, d = _req(server + "/exec", body={"source": "print(1)"})
    assert st == 403 and "disabled" in d["message"]
