"""Load the committed golden fixtures (tests/golden/*.npz) as CyclopsData."""
import glob
import json
import os

import numpy as np

from ccd_b200.data import CyclopsData

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def case_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("logistic_l1_", "known_")))


def known_names():
    """Known-answer problems from the reference's R tests (make_known_answers.py)."""
    return sorted(os.path.basename(p)[len("known_"):-4] for p in glob.glob(os.path.join(GOLDEN, "known_*.npz")))


def load_known(name):
    z = np.load(os.path.join(GOLDEN, "known_" + name + ".npz"))
    d = CyclopsData(int(z["model_type"]), z["y"], z["col_start"], z["rows"], z["val_start"], z["vals"],
                    z["fmt"], z["prior_type"], z["prior_var"],
                    time=z["time"] if "time" in z else None,
                    stratum=z["stratum"] if "stratum" in z else None)
    want = {k: z[k] for k in ("beta", "fisher_cols", "pred_est")}
    want.update(loglik=float(z["loglik"]), iterations=int(z["iterations"]), flag=int(z["flag"]))
    for k in ("fixed", "weights", "heldout", "fisher"):  # optional
        want[k] = z[k] if k in z else None
    want["pred_ll"] = float(z["pred_ll"]) if "pred_ll" in z else None
    want["published_2ll"] = float(z["published_2ll"]) if "published_2ll" in z else None
    return d, want


def load_case(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = CyclopsData(int(z["model_type"]), z["y"], z["col_start"], z["rows"], z["val_start"], z["vals"],
                    z["fmt"], z["prior_type"], z["prior_var"],
                    time=z["time"] if "time" in z else None,
                    stratum=z["stratum"] if "stratum" in z else None,
                    offset_col0=bool(int(z["offset_col0"])))
    want = {"conv": int(z["conv"]), "gh0": z["gh0"], "beta": z["beta"], "loglik": float(z["loglik"]),
            "iterations": int(z["iterations"]), "flag": int(z["flag"])}
    # calls on the fitted state (absent from fixtures older than these fields)
    for k in ("fisher", "fisher_cols", "pred_est", "heldout"):
        if k in z:
            want[k] = z[k]
    if "pred_ll" in z:
        want["pred_ll"] = float(z["pred_ll"])
    w = z["weights"] if "weights" in z else None
    return d, w, want


def index():
    with open(os.path.join(GOLDEN, "index.json")) as fh:
        return json.load(fh)
