"""Loading helpers for the committed golden fixtures (tests/golden/*.npz)."""
import json
from pathlib import Path

import numpy as np

from qtrk_b200 import abi

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name: str) -> dict:
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        d = {k: z[k] for k in z.files}
    s = abi.QTrkSettings()
    for k, v in json.loads(str(d["settings"])).items():
        setattr(s, k, v)
    d["settings"] = s
    return d
