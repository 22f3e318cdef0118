"""Run-id and JSON helpers (OOP/run_utils.py:14-47)."""

from __future__ import annotations

import json
import uuid
from dataclasses import asdict, is_dataclass
from datetime import datetime
from pathlib import Path

import numpy as np


def make_run_id(prefix: str) -> str:
    stamp = datetime.now().strftime("%Y%m%d_%H%M%S_%f")
    return f"{prefix}_{stamp}_{uuid.uuid4().hex[:8]}"


def dataclass_to_json_dict(instance) -> dict:
    data = asdict(instance) if is_dataclass(instance) else dict(instance)
    out = {}
    for key, value in data.items():
        if isinstance(value, Path):
            out[key] = str(value)
        elif isinstance(value, (np.integer, np.floating)):
            out[key] = value.item()
        else:
            out[key] = value
    return out


def write_json(path: Path, payload: dict) -> Path:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(payload, indent=2, sort_keys=True))
    return path
