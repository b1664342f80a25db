"""Request serving over the step engine: simulations of different sizes
arrive over time, are admitted while device memory and batch slots allow,
stay resident on the GPU between steps, and advance together -- every
resident grid takes one of its own steps per batched launch -- until each
reaches its final time; new requests join the running batch as slots free
up (continuous batching).  The sequential form runs the same requests one at
a time, each alone with hg_step, in arrival order.

The request stream is seeded: Poisson arrivals, each request a Balsara-1
shock tube (512-4096 zones), an advected field loop (128^2-512^2) or a
linear wave (32^3-128^3), FP64 or mixed precision.  `time_scale` multiplies
every problem's final time (1.0 is the setups' own final time).

Results per request: arrival, start and finish times, time-to-t_final
(finish - arrival), steps taken, the final primitives' checksum, and
optionally the final primitives themselves.
"""
import hashlib
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import PREC_FP64, PREC_MIXED, Batch, Engine, grid_bytes, make_desc, mem_info, setups

KINDS = ("balsara1", "field_loop", "linear_wave")
SIZES = {"balsara1": (512, 1024, 2048, 4096), "field_loop": (128, 256, 512), "linear_wave": (32, 64, 128)}


@dataclass
class Request:
    rid: int
    kind: str
    size: int
    precision: int
    arrival: float
    time_scale: float = 1.0

    def problem_desc(self, device=0):
        """The grid description alone (cheap: no initial data)."""
        n = {"balsara1": (self.size, 1, 1), "field_loop": (self.size, self.size, 1)}.get(self.kind, (self.size,) * 3)
        return make_desc(n, 5.0 / 3.0, 0.4, [1e-5, 1.0, 1.0, 1.0], [0.0] * 4, [1.0] * 4, precision=self.precision,
                         device=device)

    def problem(self, device=0):
        if self.kind == "balsara1":
            prob = setups.balsara1(self.size, precision=self.precision, device=device)
        elif self.kind == "field_loop":
            prob = setups.field_loop((self.size, self.size, 1), precision=self.precision, device=device)
        else:
            prob = setups.linear_wave((self.size,) * 3, precision=self.precision, device=device)
        if self.time_scale != 1.0:
            prob.t_final *= self.time_scale
            prob.desc.grid_length[0] = prob.t_final
        return prob


@dataclass
class Result:
    rid: int
    kind: str
    size: int
    precision: int
    arrival: float
    start: float = 0.0
    finish: float = 0.0
    steps: int = 0
    t: float = 0.0
    zones: int = 0
    checksum: str = ""
    prims: np.ndarray = field(default=None, repr=False)

    @property
    def latency(self):
        return self.finish - self.arrival


def make_stream(n=256, rate=20.0, seed=2026, time_scale=1.0, kinds=KINDS, sizes=None, mixed_fraction=0.5):
    """Seeded request stream: exponential inter-arrival times of mean 1/rate,
    kind uniform over `kinds`, size uniform over the kind's sizes, mixed
    precision with probability mixed_fraction."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = sizes or SIZES
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        kind = kinds[int(rng.integers(len(kinds)))]
        size = int(sizes[kind][int(rng.integers(len(sizes[kind])))])
        prec = PREC_MIXED if rng.random() < mixed_fraction else PREC_FP64
        out.append(Request(rid, kind, size, prec, t, time_scale))
    return out


def _finish(res, eng, keep):
    p = eng.download()
    res.checksum = hashlib.sha256(np.ascontiguousarray(p).tobytes()).hexdigest()[:16]
    if keep:
        res.prims = p


def _prepare(req, device):
    """Host set-up of one request and its resident grid (runs on a worker
    thread: numpy initial data, hg_init, upload, fixup + boundaries)."""
    prob = req.problem(device)
    eng = Engine(prob.desc)
    setups.start(eng, prob)
    return eng, prob


def serve_batched(stream, device=0, max_slots=64, reserve_bytes=2 << 30, keep=False, clock=time.perf_counter,
                  realtime=True, workers=2):
    """Continuous batching.  Requests that have arrived are admitted in
    arrival order while a slot is free and the device keeps reserve_bytes
    free after the new grid; their set-up runs on worker threads while the
    resident grids keep stepping, and they join the batch when ready.  Every
    loop iteration advances all resident grids by one step in one batched
    launch; grids at t_final leave the batch and their results are read back
    on a worker thread.  With realtime False every request counts as arrived
    at the start (a backlog)."""
    from concurrent.futures import ThreadPoolExecutor
    batch = Batch(device, max_slots)
    pool = ThreadPoolExecutor(max_workers=workers)
    pending = deque(sorted(stream, key=lambda r: r.arrival))
    waiting = deque()
    admitting = []  # (request, result, future of (engine, problem))
    active = []     # (engine, request, result)
    finishing = []  # futures of retired grids' read-back
    results = {}

    def retire(eng, res):
        _finish(res, eng, keep)
        res.finish = clock() - t0
        eng.close()
        return res

    t0 = clock()
    try:
        while pending or waiting or admitting or active:
            now = clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.popleft())
            while waiting and len(active) + len(admitting) < max_slots:
                req = waiting[0]
                need = grid_bytes(req.problem_desc(device))
                if (active or admitting) and mem_info(device)[0] < need + reserve_bytes:
                    break
                waiting.popleft()
                res = Result(req.rid, req.kind, req.size, req.precision, req.arrival if realtime else 0.0)
                res.start = clock() - t0
                admitting.append((req, res, pool.submit(_prepare, req, device)))
            still = []
            for req, res, fut in admitting:
                if fut.done():
                    eng, prob = fut.result()
                    res.zones = prob.zones
                    batch.add(eng)
                    active.append((eng, req, res))
                else:
                    still.append((req, res, fut))
            admitting = still
            if not active:
                if admitting:
                    admitting[0][2].result()
                elif pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.01)))
                continue
            t, _ = batch.step()
            done = []
            for m, (eng, req, res) in enumerate(active):
                res.steps += 1
                res.t = float(t[m])
                if t[m] >= eng.desc.grid_length[0]:
                    done.append(m)
            for m in reversed(done):
                eng, req, res = active.pop(m)
                batch.remove(eng)
                finishing.append(pool.submit(retire, eng, res))
        for f in finishing:
            r = f.result()
            results[r.rid] = r
    finally:
        for eng, _, _ in active:
            batch.remove(eng)
            eng.close()
        for _, _, fut in admitting:
            try:
                fut.result()[0].close()
            except Exception:
                pass
        pool.shutdown(wait=True)
        batch.close()
    return [results[r.rid] for r in stream]


def serve_sequential(stream, device=0, keep=False, clock=time.perf_counter, realtime=True):
    """The plain form: one request at a time in arrival order, each stepped
    alone with hg_step(1) until t_final."""
    results = []
    t0 = clock()
    for req in sorted(stream, key=lambda r: r.arrival):
        if realtime:
            while clock() - t0 < req.arrival:
                time.sleep(max(0.0, min(req.arrival - (clock() - t0), 0.01)))
        prob = req.problem(device)
        res = Result(req.rid, req.kind, req.size, req.precision, req.arrival if realtime else 0.0, zones=prob.zones)
        res.start = clock() - t0
        eng = Engine(prob.desc)
        setups.start(eng, prob)
        tf = prob.desc.grid_length[0]
        t = 0.0
        while t < tf:
            t, _ = eng.step(1)
            res.steps += 1
        res.t = t
        _finish(res, eng, keep)
        res.finish = clock() - t0
        eng.close()
        results.append(res)
    order = {r.rid: r for r in results}
    return [order[r.rid] for r in stream]


def summarize(results):
    """Aggregate throughput and latency percentiles of a served stream."""
    lat = np.array([r.latency for r in results])
    span = max(r.finish for r in results) - min(r.arrival for r in results)
    zu = sum(r.zones * r.steps for r in results)
    return {"requests": len(results), "span_s": span, "solves_per_s": len(results) / span,
            "zone_updates_per_s": zu / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "steps": int(sum(r.steps for r in results))}


def _class_key(req):
    return (req.kind, req.size, req.precision)


def measure_classes(stream, device=0, steps=20, copies=8):
    """Per request class (kind, size, precision) of the stream: the CFL
    time step (the setups start from dx[0] = 1e-5, which timestep() grows
    by at most 1.3x per step; stepped until it stops growing, at most 120
    steps), and the zone-update rate of one grid stepped alone (hg_step)
    and of `copies` grids stepped together in one batch (the most the
    device gives that class), each over `steps` steps."""
    out = {}
    for key in sorted({_class_key(r) for r in stream}):
        req = Request(-1, key[0], key[1], key[2], 0.0)
        prob = req.problem(device)
        engs = []
        try:
            for _ in range(copies):
                e = Engine(prob.desc)
                setups.start(e, prob)
                engs.append(e)
            dt = 0.0
            for _ in range(120):
                t, dt_new = engs[0].step(1)
                if dt_new <= dt * 1.0001:
                    dt = dt_new
                    break
                dt = dt_new
            engs[0].step(steps)
            alone = prob.zones * steps / (engs[0].last_step_ms() * 1e-3)
            b = Batch(device, copies)
            for e in engs:
                b.add(e)
            b.step()
            b.step()
            t0 = time.perf_counter()
            for _ in range(steps):
                b.step()
            batched = copies * prob.zones * steps / (time.perf_counter() - t0)
            for e in engs:
                b.remove(e)
            b.close()
        finally:
            for e in engs:
                e.close()
        out[key] = {"dt": dt, "zones": prob.zones, "t_final": prob.t_final, "alone": alone, "batched": batched}
    return out


def stream_bound(stream, classes):
    """How much batching can gain on this stream at most.  Request r needs
    W_r = zones x steps zone-updates (steps = t_final / dt of its class).
    Sequentially it takes W_r / alone_rate; perfectly packed into batches it
    takes at least W_r / batched_rate (its class at full occupancy), so the
    speedup of any batching of the stream is at most
    sum(W_r / alone) / sum(W_r / batched).  Also returns each kind's share of
    the zone-updates and of the sequential time."""
    seq, best = 0.0, 0.0
    share_w, share_t = {}, {}
    for r in stream:
        c = classes[_class_key(r)]
        w = c["zones"] * np.ceil(c["t_final"] * r.time_scale / c["dt"])
        seq += w / c["alone"]
        best += w / c["batched"]
        share_w[r.kind] = share_w.get(r.kind, 0.0) + w
        share_t[r.kind] = share_t.get(r.kind, 0.0) + w / c["alone"]
    tw, tt = sum(share_w.values()), sum(share_t.values())
    return {"max_speedup": seq / best, "sequential_s": seq, "best_batched_s": best,
            "zone_update_share": {k: v / tw for k, v in share_w.items()},
            "sequential_time_share": {k: v / tt for k, v in share_t.items()}}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--time-scale", type=float, default=1.0)
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--mode", choices=["batched", "sequential", "both", "bound"], default="both",
                    help="bound: measure every request class alone and batched, and print the largest speedup "
                         "batching can reach on this stream")
    a = ap.parse_args(argv)
    stream = make_stream(a.requests, a.rate, a.seed, a.time_scale)
    out = {"stream": {"requests": a.requests, "rate_per_s": a.rate, "seed": a.seed, "time_scale": a.time_scale}}
    if a.mode == "bound":
        cls = measure_classes(stream)
        out["classes"] = {"%s/%d/%s" % (k[0], k[1], "mixed" if k[2] == PREC_MIXED else "fp64"): v
                          for k, v in cls.items()}
        out["bound"] = stream_bound(stream, cls)
        print(json.dumps(out))
        return 0
    runs = {}
    if a.mode in ("batched", "both"):
        runs["batched"] = serve_batched(stream, max_slots=a.slots)
        out["batched"] = summarize(runs["batched"])
    if a.mode in ("sequential", "both"):
        runs["sequential"] = serve_sequential(stream)
        out["sequential"] = summarize(runs["sequential"])
    if len(runs) == 2:
        out["same_results"] = all(x.checksum == y.checksum for x, y in zip(runs["batched"], runs["sequential"]))
        out["speedup_solves_per_s"] = out["batched"]["solves_per_s"] / out["sequential"]["solves_per_s"]
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
