"""Multi-GPU serving: one render server per device, and a host dispatcher that routes each request to a
device by scene affinity.

The path shards without any exchange: pixels, samples and requests are independent, so a node with N
GPUs serves as N replicas.  Each device keeps its own scene cache (resident scenes under its HBM
budget, least recently used evicted first) and its own request loop (rtc_server_*); nothing crosses
NVLink.  What the dispatcher adds is placement:

  * a scene's first request goes to the device with the least work in flight, which becomes the
    scene's home (the scene is registered there; it uploads on that request);
  * later requests of the scene go to the least-loaded of its homes, so its upload and its BVH stay
    where they are;
  * a scene whose best home carries more than `replicate_at` times the work of the least-loaded device
    (counting the new request) gains that device as another home.  Hot scenes spread over devices;
    cold ones stay on one.

Work in flight is counted in traced paths (width x height x traced samples) and released when the
request's result is collected (poll or wait).  The reference renders one image per call on device 0
(gpu.cu:92-116, 2127); it has no multi-device form.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field

from .scene import MODE_COMPAT, Camera, RenderParams, Scene


@dataclass
class _Ticket:
    device: int
    local: int
    paths: int


@dataclass
class _SceneRecord:
    scene: Scene
    homes: dict = field(default_factory=dict)   # device index -> the scene's id on that device's server


class RenderDispatcher:
    """Routes render requests over one server per device (see the module docstring).

    ``devices``: CUDA device ids (one server each; an id may repeat, e.g. to run two servers on one
    GPU).  ``server_factory(device)`` makes a server; the default is ``RenderServer(device, **server_kw)``.
    A server needs ``add_scene``, ``submit``, ``poll``, ``wait``, ``stats`` and ``close`` with the
    RenderServer signatures.
    """

    def __init__(self, devices=(0,), server_factory=None, replicate_at: float = 2.0, **server_kw):
        if not devices:
            raise ValueError("at least one device")
        if replicate_at < 1.0:
            raise ValueError("replicate_at must be >= 1")
        if server_factory is None:
            from .renderer import RenderServer

            def server_factory(dev):
                return RenderServer(dev, **server_kw)
        self.devices = list(devices)
        self.servers = []
        try:
            for d in self.devices:
                self.servers.append(server_factory(d))
        except Exception:
            self.close()
            raise
        self.replicate_at = float(replicate_at)
        self._mode = server_kw.get("mode", MODE_COMPAT)
        self._lock = threading.Lock()
        self._scenes: dict[int, _SceneRecord] = {}
        self._tickets: dict[int, _Ticket] = {}
        self._next_ticket = 1
        self.load = [0] * len(self.servers)        # traced paths in flight per device
        self.routed = [0] * len(self.servers)      # requests routed per device
        self.replications = 0

    # ---- scenes -------------------------------------------------------------------------------------
    def add_scene(self, scene: Scene) -> int:
        """Registers a scene with the dispatcher (devices register it when they first serve it)."""
        with self._lock:
            sid = len(self._scenes)
            self._scenes[sid] = _SceneRecord(scene)
            return sid

    def homes(self, scene_id: int) -> list:
        """The devices (indices into ``devices``) that hold the scene."""
        with self._lock:
            return sorted(self._scenes[scene_id].homes)

    # ---- requests -----------------------------------------------------------------------------------
    def _paths(self, params: RenderParams) -> int:
        p = RenderParams(**{**params.__dict__, "mode": self._mode})
        return int(params.width) * int(params.height) * p.traced_spp

    def _place(self, rec: _SceneRecord, cost: int) -> int:
        """Device index for a request of `cost` paths (called with the lock held)."""
        least = min(range(len(self.servers)), key=lambda i: (self.load[i], i))
        if not rec.homes:
            return least
        home = min(rec.homes, key=lambda i: (self.load[i], i))
        if least not in rec.homes and self.load[home] + cost > self.replicate_at * (self.load[least] + cost):
            return least
        return home

    def submit(self, scene_id: int, params: RenderParams, camera: Camera | None = None, out=None):
        """Routes and queues a request; returns (ticket, out) like RenderServer.submit."""
        cost = self._paths(params)
        with self._lock:
            if scene_id not in self._scenes:
                raise KeyError(f"unknown scene id {scene_id}")
            rec = self._scenes[scene_id]
            dev = self._place(rec, cost)
            if dev not in rec.homes:
                if rec.homes:
                    self.replications += 1
                rec.homes[dev] = self.servers[dev].add_scene(rec.scene)
            local, out = self.servers[dev].submit(rec.homes[dev], params, camera, out)
            ticket = self._next_ticket
            self._next_ticket += 1
            self._tickets[ticket] = _Ticket(dev, local, cost)
            self.load[dev] += cost
            self.routed[dev] += 1
        return ticket, out

    def _release(self, ticket: int):
        with self._lock:
            t = self._tickets.pop(ticket, None)
            if t is not None:
                self.load[t.device] -= t.paths

    def _ticket(self, ticket: int) -> _Ticket:
        with self._lock:
            if ticket not in self._tickets:
                raise KeyError(f"unknown ticket {ticket}")
            return self._tickets[ticket]

    def poll(self, ticket: int):
        """(done, info); info gains the device index that served the request."""
        t = self._ticket(ticket)
        try:
            done, info = self.servers[t.device].poll(t.local)
        except Exception:
            self._release(ticket)
            raise
        if done:
            self._release(ticket)
        return done, {**info, "device": t.device}

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(out, info) once the request is done; info gains the device index that served it."""
        t = self._ticket(ticket)
        try:
            out, info = self.servers[t.device].wait(t.local, timeout_ms)
        except Exception as e:
            if getattr(e, "status", None) != 5:   # RTC_ERR_TIMEOUT leaves the request in flight
                self._release(ticket)
            raise
        self._release(ticket)
        return out, {**info, "device": t.device}

    def stats(self) -> dict:
        with self._lock:
            load, routed, repl = list(self.load), list(self.routed), self.replications
            scenes = {sid: sorted(r.homes) for sid, r in self._scenes.items()}
        return {"devices": self.devices, "per_device": [s.stats() for s in self.servers], "load_paths": load,
                "routed": routed, "replications": repl, "homes": scenes}

    def close(self):
        for s in getattr(self, "servers", []):
            try:
                s.close()
            except Exception:
                pass
        self.servers = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
