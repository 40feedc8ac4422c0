"""Brain modules of a connectome's neurons (the labelling rules of flyverse/regions.py:8-31), which
`LIFParams.dt_by_module` keys per-module clocks by: vnc, antennal lobe, mushroom body,
mechanosensory, gustatory, descending, visual projection and optic cells by superclass, class and
type; everything else stays central. The rule table is model data, kept identical so that the
same connectome gets the same clocks."""
from __future__ import annotations

import numpy as np
import pandas as pd

from .connectome import PHOTORECEPTOR_TYPES

MODULES = ("optic", "visual_projection", "antennal_lobe", "mushroom_body", "gustatory",
           "mechanosensory", "central", "descending", "vnc")
SWEET_TYPES = ("GNG232", "GNG132", "GNG175", "GNG229", "GNG215", "GNG108",
               "DNge173", "DNge174", "ANXXX462a", "DNg67")


def labels(c) -> np.ndarray:
    """One module name per neuron; later rules override earlier ones, as in the reference."""
    n = c.neurons
    sc, cl, ty = (n[k].fillna("").astype(str) if k in n else pd.Series([""] * len(n), index=n.index)
                  for k in ("superclass", "class", "type"))
    out = np.full(c.n, "central", dtype=object)
    out[(sc.str.startswith("vnc_") | sc.str.contains("ascending")).to_numpy()] = "vnc"
    out[(cl.isin(["olfactory", "ALLN", "ALPN", "ALIN", "ALON"]) |
         ty.str.match(r"^(ORN_|lLN|v2LN|v3LN|il3LN|l2LN|vLN)")).to_numpy()] = "antennal_lobe"
    out[(cl.isin(["Kenyon_Cell", "MBON", "DAN"]) | ty.str.match(r"^(KC|MBON|APL$|DPM$)")).to_numpy()] = "mushroom_body"
    out[(cl.str.startswith("mechanosensory") | ty.str.match(r"^(JO-|AMMC|WED)")).to_numpy()] = "mechanosensory"
    out[(cl.eq("gustatory") | ty.isin(SWEET_TYPES) | sc.eq("cb_motor")).to_numpy()] = "gustatory"
    out[sc.eq("descending_neuron").to_numpy()] = "descending"
    out[sc.isin(["visual_projection", "visual_projection_tbc", "visual_centrifugal"]).to_numpy()] = "visual_projection"
    out[(sc.eq("ol_intrinsic") | ty.isin(PHOTORECEPTOR_TYPES)).to_numpy()] = "optic"
    if "dataset" in n:
        synthetic = n.dataset.eq("synthetic").to_numpy()
        out[synthetic] = sc.replace("", "synthetic").to_numpy()[synthetic]
    return out


def clock_periods(c, dt: float, dt_by_module: dict) -> np.ndarray:
    """Per-neuron update periods in steps for {module: dt_module} (fly.py:98-107)."""
    lab = labels(c)
    k = np.ones(c.n, np.int64)
    for mod, dt_mod in dt_by_module.items():
        if mod not in set(MODULES) | set(lab):
            raise ValueError(f"unknown module {mod!r} in dt_by_module")
        m = int(round(dt_mod / dt))
        if abs(m * dt - dt_mod) > 1e-9 or m < 1:
            raise ValueError(f"dt_by_module[{mod!r}] = {dt_mod} is not a positive multiple of dt = {dt}")
        k[lab == mod] = m
    return k
