"""NEST Server for the engine: the reference's HTTP API
(pynest/nest/server/hl_api_server.py) over this package's PyNEST-compatible
front-end, plus routes that submit networks to the continuous-batching
serving engine.

Routes of the reference, same request and response shapes:

- ``GET /``                 -> ``{"nest": <version>, "mpi": false}`` (hl_api_server.py:180-187)
- ``GET /api``              -> the sorted public call names (:295-298)
- ``GET|POST /api/<call>``  -> ``nestgpu.<call>(*args, **kwargs)``; arguments as the
  reference's ``get_arguments`` reads them (:369-392): a JSON list is the
  positional arguments, a JSON object the keyword arguments (its ``"args"``
  entry the positional ones), else form or query parameters; node-id lists
  in ``nodes``, ``source``, ``target``, ``pre``, ``post`` become
  NodeCollections (``nestify``, :501-513); the result is serialised to JSON
  (NodeCollections as lists of node ids, numpy values as lists and numbers).
  An error is answered with status 400 and ``{"message": "<Error>: <detail>",
  "lineno": -1}`` (:431-463).
- ``/exec``                 -> 403: code execution is off, as the reference's
  default (NEST_SERVER_ENABLE_EXEC_CALL unset, :271-289); this server never
  executes request code.

Serving routes (no counterpart in the reference, which runs one network per
kernel): ``POST /serving/submit`` with a Brunel-type network
(``{"n", "g", "eta", "t_ms", "seed"}``) queues it for the FP32 serving
engine; ``GET /serving/result/<id>`` answers its status and, once done, its
spike count, rate, CV-ISI, latency and (with ``?spikes=1``) its raster;
``GET /serving/stats`` the engine's counters.  Submitted networks are admitted
as pool space frees up and advance with every other live network in the
same slice kernels (serving.OnlineBatcher).

Run:  python -m nestgpu.server [--host 127.0.0.1] [--port 52425]
"""

import argparse
import json
import math
import threading
import time
import traceback
from http.server import BaseHTTPRequestHandler, ThreadingHTTPServer
from urllib.parse import parse_qs, urlparse

import numpy as np

OBJECT_NAMES = ("nodes", "source", "target", "pre", "post")


def serialize(x):
    """JSON-ready form of a call result (the reference's serialize_data)."""
    from .nodes import NodeCollection

    if isinstance(x, NodeCollection):
        return [int(i) for i in x.tolist()]
    if isinstance(x, dict):
        return {str(k): serialize(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [serialize(v) for v in x]
    if isinstance(x, np.ndarray):
        return serialize(x.tolist())
    if isinstance(x, (np.integer,)):
        return int(x)
    if isinstance(x, (np.floating,)):
        return float(x)
    if isinstance(x, np.bool_):
        return bool(x)
    if isinstance(x, float) and not math.isfinite(x):
        return str(x)
    if hasattr(x, "get") and hasattr(x, "source"):  # SynapseCollection
        return serialize(x.get())
    return x


def api_calls():
    import nestgpu

    return sorted(n for n in nestgpu.__all__ if not n.startswith("_"))


def nestify(call, args, kwargs):
    """Node-id lists in the node arguments become NodeCollections."""
    import inspect

    from .nodes import NodeCollection

    try:
        names = list(inspect.signature(call).parameters)
    except (TypeError, ValueError):
        names = []
    args = [NodeCollection(a) if k < len(names) and names[k] in OBJECT_NAMES and isinstance(a, list) else a
            for k, a in enumerate(args)]
    for key in list(kwargs):
        if key in OBJECT_NAMES and isinstance(kwargs[key], list):
            kwargs[key] = NodeCollection(kwargs[key])
    return args, kwargs


class ApiError(Exception):
    def __init__(self, message, status=400):
        super().__init__(message)
        self.status = status


class NestServer:
    """The HTTP server: one front-end kernel (calls serialised by a lock, as
    the reference serves one kernel) and an optional serving engine."""

    def __init__(self, host="127.0.0.1", port=52425, serving_capacity=(2_000_000, 1_200_000_000), device=0):
        self.lock = threading.Lock()
        self.batcher = None
        self.serving_capacity = serving_capacity
        self.device = device
        handler = self._handler()
        self.httpd = ThreadingHTTPServer((host, port), handler)
        self.httpd.daemon_threads = True
        self.port = self.httpd.server_address[1]
        self._thread = None

    # ---- calls
    def call(self, name, args, kwargs):
        import nestgpu

        if name not in api_calls():
            raise ApiError(f"AttributeError: module 'nest' has no attribute '{name}'")
        fn = getattr(nestgpu, name)
        if not callable(fn):
            return serialize(fn)
        args, kwargs = nestify(fn, list(args), dict(kwargs))
        with self.lock:
            try:
                return serialize(fn(*args, **kwargs))
            except Exception as err:  # the reference answers every failure with 400 and its message
                traceback.print_exc()
                detail = err.args[0] if err.args else ""
                raise ApiError(f"{type(err).__name__}: {detail}")

    def serving(self):
        if self.batcher is None:
            from .serving import OnlineBatcher

            self.batcher = OnlineBatcher(capacity_neurons=self.serving_capacity[0],
                                         capacity_edges=self.serving_capacity[1], device=self.device)
        return self.batcher

    # ---- HTTP
    def _handler(self):
        server = self

        class Handler(BaseHTTPRequestHandler):
            def log_message(self, fmt, *a):  # quiet
                pass

            def _send(self, status, obj):
                body = json.dumps(obj).encode()
                self.send_response(status)
                self.send_header("Content-Type", "application/json")
                self.send_header("Content-Length", str(len(body)))
                self.end_headers()
                self.wfile.write(body)

            def _arguments(self):
                """The reference's get_arguments: JSON body, else form, else query."""
                url = urlparse(self.path)
                args, kwargs = [], {}
                n = int(self.headers.get("Content-Length") or 0)
                raw = self.rfile.read(n) if n > 0 else b""
                ctype = (self.headers.get("Content-Type") or "").split(";")[0].strip()
                if raw and ctype == "application/json":
                    data = json.loads(raw)
                    if isinstance(data, str) and data:
                        args = [data]
                    elif isinstance(data, list):
                        args = data
                    elif isinstance(data, dict):
                        kwargs = data
                        if "args" in kwargs:
                            args = kwargs.pop("args")
                    return list(args), kwargs
                form = parse_qs(raw.decode()) if raw else {}
                query = parse_qs(url.query)
                for src in (form, query):
                    if src:
                        if "args" in src:
                            return list(src["args"]), {}
                        return [], {k: v[0] if len(v) == 1 else v for k, v in src.items()}
                return args, kwargs

            def _route(self):
                url = urlparse(self.path)
                parts = [p for p in url.path.split("/") if p]
                try:
                    if not parts:
                        import nestgpu

                        return self._send(200, {"nest": nestgpu.__version__, "mpi": False})
                    if parts[0] == "exec":
                        return self._send(403, {"message": "The route `/exec` has been disabled. Please contact the "
                                                           "server administrator.", "lineno": -1})
                    if parts[0] == "api" and len(parts) == 1:
                        return self._send(200, api_calls())
                    if parts[0] == "api" and len(parts) == 2:
                        args, kwargs = self._arguments()
                        return self._send(200, server.call(parts[1], args, kwargs))
                    if parts[0] == "serving":
                        return self._serving(parts[1:], url)
                    return self._send(404, {"message": f"no route {url.path}", "lineno": -1})
                except ApiError as err:
                    return self._send(err.status, {"message": str(err), "lineno": -1})
                except (ValueError, KeyError, TypeError) as err:
                    return self._send(400, {"message": f"{type(err).__name__}: {err}", "lineno": -1})

            def _serving(self, parts, url):
                if parts == ["submit"]:
                    _, kw = self._arguments()
                    rid = server.serving().submit(n=int(kw["n"]), g=float(kw.get("g", 5.0)),
                                                  eta=float(kw.get("eta", 2.0)), t_ms=float(kw.get("t_ms", 1000.0)),
                                                  seed=int(kw.get("seed", 1)))
                    return self._send(200, {"request": rid})
                if len(parts) == 2 and parts[0] == "result":
                    q = parse_qs(url.query)
                    res = server.serving().result(int(parts[1]), spikes=q.get("spikes", ["0"])[0] in ("1", "true"))
                    if res is None:
                        return self._send(404, {"message": f"no request {parts[1]}", "lineno": -1})
                    return self._send(200, serialize(res))
                if parts == ["stats"]:
                    return self._send(200, serialize(server.serving().stats()))
                return self._send(404, {"message": "no such serving route", "lineno": -1})

            def do_GET(self):
                self._route()

            def do_POST(self):
                self._route()

        return Handler

    def start(self):
        self._thread = threading.Thread(target=self.httpd.serve_forever, daemon=True)
        self._thread.start()
        return self

    def stop(self):
        self.httpd.shutdown()
        self.httpd.server_close()
        if self.batcher is not None:
            self.batcher.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--host", default="127.0.0.1")
    ap.add_argument("--port", type=int, default=52425)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    srv = NestServer(a.host, a.port, device=a.device)
    print(f"NEST Server (nestgpu) on http://{a.host}:{srv.port}", flush=True)
    try:
        srv.httpd.serve_forever()
    except KeyboardInterrupt:
        pass
    finally:
        srv.stop()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
