"""The checkpoint state mirror of a domain (checkpoint!, checkpoint_payload,
write_checkpoint and the restart, src/io/checkpoint.jl:346-473).

A payload is a self-contained dict: the format tag and version, the mesh
record, the simulation time, copies of the prognostic storage fields (u, v,
w, theta and the pressure, halos included), the scalar parameters of the
CoreSpec, the closure name and its state (the Lagrangian closure's
memories, sgs_state / restore_sgs_state!), the stepper state (the last
accepted dt of an adaptive run), the state of open lateral faces
(open_boundary_checkpoint: the plane buffers and the Orlanski history, as
`Simulation.open_checkpoint` reads them) and free-form extras. `buffers` (the
fields of an earlier payload of the same domain) are refilled in place, so a run that keeps its
last good state (a rollback snapshot) allocates once.

On disk a payload is one .npz file: the arrays plus the rest as a JSON
header. `write_checkpoint` writes `path + ".tmp"` and renames it, so an
interrupted write never leaves a truncated checkpoint under `path`.
`restore` checks the format, the mesh and the parameters against the
domain it fills and returns the time and the stepper state.
"""
from __future__ import annotations

import dataclasses
import json
import os
import time
from typing import Any, Dict, Optional

import numpy as np

CHECKPOINT_FORMAT = "aeolus_b200.checkpoint"
CHECKPOINT_VERSION = 1
FIELDS = ("u", "v", "w", "theta", "p")
CLOSURE_ARRAYS = ("I_LM", "I_MM", "U", "V", "W")


def closure_state(sim) -> Optional[Dict[str, Any]]:
    """checkpoint_state of the run's closure (a copy of sgs_state): the
    Lagrangian closure's memories and its initialised flag, the TKE
    closure's e, None for the closures that keep no state."""
    spec = sim.spec
    kind = closure_state_kind(sim)
    if kind is None:
        return None
    if kind == "tke":
        return {"e": np.array(sim.sgs_state(), dtype=np.float64, copy=True)}
    st = sim.sgs_state()
    out: Dict[str, Any] = {k: np.array(a, dtype=np.float64, copy=True) for k, a in zip(CLOSURE_ARRAYS, st[:5])}
    out["initialised"] = bool(st[5])
    return out


def mesh_record(grid) -> Dict[str, Any]:
    """The mesh of a checkpoint (_mesh_record): sizes, extents, halos, origin,
    the z boundary and the stretched face heights."""
    return {"size": list(grid.size), "extent": [float(x) for x in grid.extent], "halo": list(grid.halo),
            "origin": [float(x) for x in grid.origin], "bc_z": grid.bc_z,
            "zf": None if grid.zf is None else [float(x) for x in grid.zf]}


def parameters(spec) -> Dict[str, Any]:
    """The scalar parameters of a CoreSpec (_parameters): every field that is a
    string, a number or None (the grid and the weight arrays are the mesh's)."""
    out = {}
    for f in dataclasses.fields(spec):
        v = getattr(spec, f.name)
        if v is None or isinstance(v, (str, bool, int, float)):
            out[f.name] = v
    return out


def checkpoint_payload(sim, t: float = 0.0, stepper: Optional[Dict[str, Any]] = None,
                       extra: Optional[Dict[str, Any]] = None, buffers: Optional[Dict[str, np.ndarray]] = None,
                       with_fields: bool = True) -> Dict[str, Any]:
    """The in-memory checkpoint of `sim` (checkpoint_payload,
    src/io/checkpoint.jl:352-398): nothing in it aliases the run."""
    spec = sim.spec
    fields: Dict[str, np.ndarray] = {}
    if with_fields:
        for name in FIELDS:
            b = None if buffers is None else buffers.get(name)
            shape = spec.grid.storage_shape
            if b is not None and b.dtype == np.float64 and b.shape == shape and b.flags.c_contiguous:
                fields[name] = sim.get_field(name, out=b) if _takes_out(sim) else _copy_into(b, sim.get_field(name))
            else:
                fields[name] = np.array(sim.get_field(name), dtype=np.float64, copy=True)
    return {
        "format": CHECKPOINT_FORMAT,
        "version": CHECKPOINT_VERSION,
        "created": time.time(),
        "sim_type": type(sim).__name__,
        "mesh": mesh_record(spec.grid),
        "t": float(t),
        "fields": fields,
        "parameters": parameters(spec),
        "closure_type": spec.sgs if spec.c_s != 0 else "",
        "closure": closure_state(sim),
        "stepper": None if stepper is None else dict(stepper),
        "open": open_state(sim),
        "extra": {} if extra is None else dict(extra),
    }


def _takes_out(sim) -> bool:
    import inspect
    try:
        return "out" in inspect.signature(sim.get_field).parameters
    except (TypeError, ValueError):
        return False


def _copy_into(b: np.ndarray, a: np.ndarray) -> np.ndarray:
    np.copyto(b, a)
    return b


def write_checkpoint(path: str, payload: Dict[str, Any]) -> str:
    """Write a payload to `path` through `path + ".tmp"` and a rename
    (write_checkpoint, src/io/checkpoint.jl:400-417)."""
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    head = {k: v for k, v in payload.items() if k not in ("fields", "closure", "open")}
    head["field_names"] = sorted(payload["fields"])
    arrays = {"field_" + k: v for k, v in payload["fields"].items()}
    cl = payload.get("closure")
    head["closure"] = None if cl is None else {k: v for k, v in cl.items() if not isinstance(v, np.ndarray)}
    if cl is not None:
        head["closure"]["arrays"] = sorted(k for k, v in cl.items() if isinstance(v, np.ndarray))
        arrays.update({"closure_" + k: v for k, v in cl.items() if isinstance(v, np.ndarray)})
    ob = payload.get("open")
    head["open"] = None if ob is None else {k: v for k, v in ob.items() if not isinstance(v, np.ndarray)}
    if ob is not None:
        head["open"]["arrays"] = sorted(k for k, v in ob.items() if isinstance(v, np.ndarray))
        arrays.update({"open_" + k: v for k, v in ob.items() if isinstance(v, np.ndarray)})
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        np.savez(f, header=np.frombuffer(json.dumps(head).encode(), dtype=np.uint8), **arrays)
    os.replace(tmp, path)
    return path


def read_checkpoint(path: str) -> Dict[str, Any]:
    """The payload written by write_checkpoint (no pickled objects are read)."""
    with np.load(path, allow_pickle=False) as z:
        head = json.loads(bytes(z["header"]).decode())
        if head.get("format") != CHECKPOINT_FORMAT:
            raise ValueError(f"{path}: not a checkpoint of this format ({head.get('format')!r})")
        fields = {k: np.array(z["field_" + k]) for k in head.pop("field_names")}
        if head.get("closure") is not None:
            head["closure"].update({k: np.array(z["closure_" + k]) for k in head["closure"].pop("arrays")})
        if head.get("open") is not None:
            head["open"].update({k: np.array(z["open_" + k]) for k in head["open"].pop("arrays")})
    head["fields"] = fields
    return head


def checkpoint(sim, path: str, **kw) -> str:
    """checkpoint!: the payload of `sim` written to `path`."""
    return write_checkpoint(path, checkpoint_payload(sim, **kw))


def restore(sim, payload, check_parameters: bool = True):
    """Fill `sim` from a payload (or a checkpoint path) and return (t,
    stepper). The mesh must be the domain's; with `check_parameters` so must
    every scalar parameter (the closure, the core, the schemes ...)."""
    if isinstance(payload, (str, os.PathLike)):
        payload = read_checkpoint(os.fspath(payload))
    if payload.get("format") != CHECKPOINT_FORMAT:
        raise ValueError(f"not a checkpoint payload ({payload.get('format')!r})")
    if payload.get("version") != CHECKPOINT_VERSION:
        raise ValueError(f"checkpoint version {payload.get('version')} (this build reads {CHECKPOINT_VERSION})")
    mine = mesh_record(sim.spec.grid)
    if payload["mesh"] != mine:
        raise ValueError(f"checkpoint mesh {payload['mesh']} does not match the domain's {mine}")
    if check_parameters:
        p, q = payload["parameters"], parameters(sim.spec)
        diff = sorted(k for k in set(p) | set(q) if p.get(k) != q.get(k))
        if diff:
            raise ValueError(f"checkpoint parameters differ from the domain's: {diff}")
    missing = [n for n in FIELDS if n not in payload["fields"]]
    if missing:
        raise ValueError(f"checkpoint lacks the fields {missing}")
    mine = sim.spec.sgs if sim.spec.c_s != 0 else ""
    if payload.get("closure_type", "") != mine:
        raise ValueError(f"the checkpoint's closure is {payload.get('closure_type')!r}, the domain's {mine!r}")
    cl = payload.get("closure")
    if (cl is None) != (closure_state_kind(sim) is None):
        raise ValueError("the checkpoint's closure state does not fit the domain's closure")
    ob = payload.get("open")
    if (ob is None) != (getattr(sim, "_open", None) is None):
        raise ValueError("the checkpoint's open faces do not fit the domain's")
    for name in FIELDS:
        sim.set_field(name, np.ascontiguousarray(payload["fields"][name], dtype=np.float64))
    if ob is not None:
        sim.restore_open_checkpoint(ob)
    if cl is not None:
        if closure_state_kind(sim) == "tke":
            sim.set_sgs_state(cl["e"])
        else:
            sim.set_sgs_state(tuple(cl[k] for k in CLOSURE_ARRAYS) + (bool(cl["initialised"]),))
    return payload["t"], payload["stepper"]


def open_state(sim) -> Optional[Dict[str, Any]]:
    """The open faces' restart state of `sim` (None: no open face, or a
    domain without them)."""
    f = getattr(sim, "open_checkpoint", None)
    return None if f is None else f()


def closure_state_kind(sim) -> Optional[str]:
    """The kind of state the domain's closure keeps (None: none)."""
    if sim.spec.c_s == 0 or sim.spec.sgs not in ("lagrangian", "tke"):
        return None
    return sim.spec.sgs
