"""Launch shapes of a batch chosen by measurement.

The shapes a ``Batch`` launches with change how the work is cut, not what is
computed: every bead's pair force is summed over its neighbour list in
ascending partner id, the persistent grids only change which CTA visits a
tile, a graph of more steps only changes how often the host launches, and the
Verlet skin only changes how often lists are rebuilt (a list holds every
partner within r_cut + skin, so the pair sum is the same).  The trajectory is
therefore the same bit for bit under every candidate, and the tuner is free
to pick the fastest.

``tune`` times a short run of each candidate on copies of the workload's
systems (the caller's state is not touched) and searches one parameter at a
time from the defaults (coordinate descent over ``SPACE``), re-centring on
the best shape after every pass.  Choices are cached in a JSON file keyed by
the workload's signature and the device, so a workload of the same shape
tunes once per device.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import math
import os

import numpy as np

# the candidates of each parameter; the first entry of each is not special,
# the search starts from DEFAULT
SPACE = {
    "block_beads": (64, 128, 256),     # beads per tile = threads per CTA of the bead kernels
    "ctas_per_sm": (0, 2, 4, 8),       # persistent CTAs per SM (0: as many as fit)
    "steps_per_graph": (5, 10, 20),    # steps per captured CUDA graph
    "skin_scale": (0.67, 1.0, 1.5),    # Verlet skin relative to engine.default_skin(r_cut)
    "pair_mode": (0, 1, 2),            # pair forces: list kernel, list walk in the stages, cell-staged kernel
}
DEFAULT = {"block_beads": 128, "ctas_per_sm": 0, "steps_per_graph": 10, "skin_scale": 1.0, "pair_mode": 0}
CACHE = os.path.join(os.path.expanduser("~"), ".cache", "gcr_autotune.json")


def signature(specs, precision, srk_order=2, device_name=""):
    """What the best shape depends on: dimension, precision, SRK order, the
    number of systems and the bead count (to a factor of 2), the mean pair
    cutoff and the device."""
    n = sum(s.n for s in specs)
    rc = float(np.mean([s.params.wca_params[3] for s in specs]))
    key = {"dim": int(specs[0].dim), "precision": precision, "srk_order": int(srk_order), "systems": len(specs),
           "beads_log2": int(round(math.log2(max(n, 1)))), "r_cut": round(rc, 2), "device": device_name}
    return json.dumps(key, sort_keys=True)


def _with_skin(specs, scale):
    from .engine import default_skin
    out = []
    for s in specs:
        sk = s.params.skin if s.params.skin is not None else default_skin(s.params.wca_params[3])
        out.append(dataclasses.replace(s, params=dataclasses.replace(s.params, skin=sk * scale)))
    return out


def search(measure, space=None, start=None, passes=2):
    """Coordinate descent: vary one parameter at a time over its candidates
    with the others fixed at the best shape so far; ``measure(shape)`` returns
    ms per step (inf for a shape that failed).  Returns (best shape, best ms,
    every trial)."""
    space = space or SPACE
    best = dict(start or {k: DEFAULT.get(k, v[0]) for k, v in space.items()})
    seen = {}

    def cost(shape):
        key = json.dumps(shape, sort_keys=True)
        if key not in seen:
            seen[key] = float(measure(dict(shape)))
        return seen[key]

    best_ms = cost(best)
    for _ in range(passes):
        moved = False
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                trial = {**best, name: v}
                ms = cost(trial)
                if ms < best_ms:
                    best, best_ms, moved = trial, ms, True
        if not moved:
            break
    trials = [{**json.loads(k), "ms_per_step": v} for k, v in seen.items()]
    return best, best_ms, trials


def measure_shape(specs, shape, precision="mixed", steps=40, warmup=10, device=None, srk_order=2,
                  couplings=()):
    """ms per step of a Batch of copies of ``specs`` launched with ``shape``
    (CUDA events on the batch's stream; every system under its own adaptive
    dt, as the bench runs them)."""
    import torch
    from .batch import Batch
    from ._lib import GcrError
    sp = _with_skin(specs, shape.get("skin_scale", 1.0))
    try:
        b = Batch(sp, precision=precision, device=device, steps_per_graph=shape["steps_per_graph"],
                  block_beads=shape["block_beads"], ctas_per_sm=shape["ctas_per_sm"], srk_order=srk_order,
                  pair_mode=shape.get("pair_mode", 0))
    except (GcrError, RuntimeError, ValueError):
        return math.inf
    try:
        for members, fixed, cross in couplings:
            b.couple(members, fixed, cross)
        b.set_adaptive(True)
        b.run_checked(warmup)
        b.begin(steps)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(b.engine.stream)
        b.run(steps)
        e1.record(b.engine.stream)
        e1.synchronize()
        if b.overflowed():
            return math.inf
        return e0.elapsed_time(e1) / steps
    finally:
        b.close()


def tune(specs, precision="mixed", steps=40, warmup=10, device=None, srk_order=2, couplings=(), space=None,
         cache=CACHE, refresh=False, passes=2):
    """The fastest launch shape for this workload: a dict with
    ``block_beads``, ``ctas_per_sm``, ``steps_per_graph``, ``skin_scale``,
    ``ms_per_step`` and the ``trials``; taken from the cache when this
    signature was tuned before on this device (unless ``refresh``)."""
    import torch
    dev = torch.device(device or "cuda")
    name = torch.cuda.get_device_name(dev)
    key = signature(specs, precision, srk_order, name)
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as fh:
                table = json.load(fh)
        except (OSError, ValueError):
            table = {}
    h = hashlib.sha1(key.encode()).hexdigest()[:16]
    if not refresh and h in table:
        return table[h]["result"]
    best, best_ms, trials = search(
        lambda shape: measure_shape(specs, shape, precision, steps, warmup, dev, srk_order, couplings),
        space=space, passes=passes)
    result = {**best, "ms_per_step": best_ms, "trials": trials}
    if cache:
        table[h] = {"signature": json.loads(key), "result": result}
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        tmp = cache + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(table, fh, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    return result


def apply(specs, result):
    """The specs with the tuned skin, and the Batch keyword arguments of the
    tuned shape."""
    kw = {"block_beads": result["block_beads"], "ctas_per_sm": result["ctas_per_sm"],
          "steps_per_graph": result["steps_per_graph"], "pair_mode": result.get("pair_mode", 0)}
    return _with_skin(specs, result.get("skin_scale", 1.0)), kw
