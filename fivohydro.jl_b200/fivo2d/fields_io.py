"""save_fields / load_fields (src/fields_io.jl:70-106): a solver's output saved WITH
what produced it.

The reference writes a JLD2 file; the Julia host keeps doing exactly that (the
binding's `fields_2d(g, U, work::GPUWork2D, model)` returns the reference's
NamedTuple, which its own `save_fields` writes unchanged). This Python host writes
the same record as a NumPy .npz archive, with the reference's schema keys:

    fields        every array of the fields dict, stored as "fields/<name>"
    solver        "FiVo 2+1D" for a 2+1D model
    terms         the integrated Terms switches, name -> bool
    model         a plain-text record of the sectors and term switches
    model_fields  every scalar knob of the model (flattened fivo_params and the
                  keyword knobs), name -> repr
    meta          whatever the caller passed
    created       ISO-8601 time stamp
    fivo_revision git short hash of this tree (+ "-dirty"), or "unknown"

The non-array entries are one JSON document, so the file loads with numpy alone.
"""
from __future__ import annotations

import datetime as _dt
import json
import pathlib
import subprocess

import numpy as np

from . import _abi as A

_ROOT = pathlib.Path(__file__).resolve().parents[2]


def _revision() -> str:
    """_fivo_revision (src/fields_io.jl:37-46)"""
    try:
        rev = subprocess.run(["git", "-C", str(_ROOT), "rev-parse", "--short", "HEAD"], capture_output=True,
                             text=True, check=True, timeout=10).stdout.strip()
        dirty = subprocess.run(["git", "-C", str(_ROOT), "status", "--porcelain", "--untracked-files=no"],
                               capture_output=True, text=True, check=True, timeout=10).stdout.strip()
        return rev + "-dirty" if dirty else rev
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def _terms(model) -> dict:
    return {n: bool(model.params.terms & A.TERM_BIT[n]) for n in A.TERM_NAMES}


def _model_text(model) -> str:
    """the sectors and term switches the model integrates ([x] on, [ ] off)"""
    p = model.params
    mark = lambda b: "[x]" if b else "[ ]"  # noqa: E731
    lines = [f"FiVo 2+1D model, layout {', '.join(model.layout.names)}",
             f"  shear {mark(p.enable_shear)}  bulk {mark(p.enable_bulk)}  charge diffusion {mark(p.enable_diff)}",
             f"  consistent first moment {mark(p.consistent_fm)}  consistent second moment {mark(p.consistent_m2)}",
             "  terms:"]
    lines += [f"    {mark(v)} {k}" for k, v in _terms(model).items()]
    return "\n".join(lines) + "\n"


def _model_fields(model) -> dict:
    """_model_record's scalar fields (src/fields_io.jl:48-66): every scalar of the
    flattened parameters, then the keyword knobs and the EOS"""
    out = {}
    for name, _ in A.FivoParams._fields_:
        v = getattr(model.params, name)
        out[name] = repr(list(v)) if hasattr(v, "__len__") else repr(v)
    for k, v in getattr(model, "knobs", {}).items():
        if isinstance(v, (bool, int, float, str)):
            out[k] = repr(v)
    out["eos"] = type(model.eos).__name__
    for k, v in vars(model.eos).items():
        out["eos." + k] = repr(v)
    return out


def save_fields(path, fields: dict, *, model=None, meta=None, solver: str | None = None):
    """Write `fields` (what fields_2d returned) and the record of the model that made it."""
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    record = dict(solver=solver if solver is not None else ("FiVo 2+1D" if model is not None else "FiVo"),
                  terms=_terms(model) if model is not None else None,
                  model=_model_text(model) if model is not None else "",
                  model_fields=_model_fields(model) if model is not None else {},
                  meta={str(k): v for k, v in (meta or {}).items()},
                  created=_dt.datetime.now().isoformat(timespec="seconds"),
                  fivo_revision=_revision())
    arrays = {f"fields/{k}": np.asarray(v) for k, v in fields.items()}
    with open(path, "wb") as fh:
        np.savez(fh, __record__=np.frombuffer(json.dumps(record, default=repr).encode(), dtype=np.uint8),
                 **arrays)
    return path


def load_fields(path) -> dict:
    """Read a file written by save_fields: dict(fields, solver, terms, model, model_fields,
    meta, created, fivo_revision)."""
    with np.load(path, allow_pickle=False) as z:
        record = json.loads(bytes(z["__record__"]).decode())
        record["fields"] = {k[len("fields/"):]: z[k] for k in z.files if k.startswith("fields/")}
    return record
