"""Launch shape of the FP32 batched persistent kernel, and its autotuner.

The shape (threads per block, resident blocks per SM, step pairs per slot
and launch, cell-table ring slots) is a property of a Context and is fixed
at its first FP32 job.  ``tuned_shape()`` returns the shape the autotuner
(``python -m langevindynamicsforpcp_b200.autotune``) committed to
tuning.json next to this file, or None.
"""
from __future__ import annotations

import ctypes as C
import json
import os

from . import _lib as L

TUNING_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def set_fp32_shape(ctx, block=0, blocks_per_sm=0, pair_budget=0, ring_slots=0):
    st = L.lib().ldp_ctx_set_fp32_shape(ctx.handle, block, blocks_per_sm, pair_budget, ring_slots)
    if st != 0:
        raise L.LdpError(st, ctx.last_error())


def get_fp32_shape(ctx) -> dict:
    b, g, r = C.c_int(), C.c_int(), C.c_int()
    pb = C.c_uint64()
    L.lib().ldp_ctx_get_fp32_shape(ctx.handle, C.byref(b), C.byref(g), C.byref(pb), C.byref(r))
    return {"block": b.value, "grid": g.value, "pair_budget": pb.value, "ring_slots": r.value}


def tuned_shape(model: str = "single_over") -> dict | None:
    if not os.path.exists(TUNING_JSON):
        return None
    with open(TUNING_JSON) as f:
        d = json.load(f)
    return d.get("shapes", {}).get(model)


def apply_tuned(ctx, model: str = "single_over") -> dict | None:
    s = tuned_shape(model)
    if s:
        set_fp32_shape(ctx, s["block"], s.get("blocks_per_sm", 0), s["pair_budget"], s.get("ring_slots", 0))
    return s
