"""Shared test helpers: one workload spec -> a GPU Context system and the
matching CPU-oracle system, plus comparison utilities."""
import numpy as np

import oracle_py

QUIRK = {"ref": oracle_py.MODE_REF, "fixed": oracle_py.MODE_FIXED}


def oracle_from_spec(spec, threads=None, fast=False):
    """fast=True: the reference-flags build, for timing only"""
    ctl = dict(spec["control"])
    mode = QUIRK[ctl.pop("quirk", "ref")]
    o = oracle_py.Oracle(threads=threads, mode=mode, fast=fast)
    o.set_types(spec["masses"])
    o.set_pairs(spec["pairs"])
    o.set_state(spec["typ"], spec["pos"], spec["box"], vel=spec.get("vel"), acc=spec.get("acc"))
    o.set_control(**ctl)
    return o


def gpu_from_spec(ctx, spec):
    sid = ctx.add_system(spec["masses"], spec["pairs"], spec["typ"], spec["pos"], spec["box"],
                         vel=spec.get("vel"), acc=spec.get("acc"))
    ctx.set_control(sid, **spec["control"])
    return sid


def pair_multiset(pairs):
    """sorted (i,j) rows with multiplicity, as a structured comparison key"""
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    key = p[:, 0] * (1 << 32) + p[:, 1]
    return np.sort(key)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)
