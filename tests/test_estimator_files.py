"""CPU checks of the shipped estimator network: the built-in copy in the
library equals research_b200/estimator_weights.txt, and the training report
committed beside it records the held-out comparison with HLL."""
import json
from pathlib import Path

import numpy as np

from research_b200 import estimator as E
from research_b200.ocean import MLP_BLOB, lib

PKG = Path(__file__).resolve().parents[1] / "research_b200"


def test_builtin_equals_weights_file():
    blob = np.empty(MLP_BLOB, np.float32)
    assert lib().ocean_mlp_builtin(blob.ctypes.data, MLP_BLOB) == 0
    tok = (PKG / "estimator_weights.txt").read_text().split()
    assert tok[0] == E.TAG and len(tok) == MLP_BLOB + 1
    assert np.array_equal(np.array([float(x) for x in tok[1:]], np.float32), blob)
    assert blob[-1] > 0.0  # calibrated margin


def test_training_report_shows_gain_over_hll():
    r = json.loads((PKG / "estimator_weights.report.json").read_text())
    assert r["matrices"] == 2000 and r["train_rows"] > 1_000_000
    ev = r["eval"]
    assert ev["rows"] == 1 << 21
    assert ev["learned_raw"]["mean_rel_error"] < ev["hll_raw"]["mean_rel_error"]
    assert ev["learned_raw"]["misbinned_pct"] < ev["hll_raw"]["misbinned_pct"]
    assert ev["learned_prealloc"]["est_total"] < ev["hll_prealloc"]["est_total"]
