"""The photoreceptor geometry the optic lobe consumes (flyverse/retina.py:59-139, the parts on the
brain-step path): each photoreceptor's connectome row, hex column and spectral sensitivity."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .connectome import PHOTORECEPTOR_TYPES

CHANNELS = ["UV", "B", "G", "R"]
# Relative spectral sensitivity per photoreceptor class over [UV, B, G, R] (retina.py:35-46): a data
# table of the model, kept identical so photoreceptor drive matches the reference.
SENSITIVITY = {
    "R1-R6": [0.50, 0.70, 1.00, 0.05], "R7p": [1.00, 0.05, 0.00, 0.00], "R7y": [1.00, 0.15, 0.00, 0.00],
    "R7d": [1.00, 0.05, 0.00, 0.00], "R7_unclear": [1.00, 0.10, 0.00, 0.00], "R8p": [0.20, 1.00, 0.10, 0.00],
    "R8y": [0.05, 0.30, 1.00, 0.10], "R8d": [1.00, 0.05, 0.00, 0.00], "R8_unclear": [0.12, 0.65, 0.55, 0.05],
    "R7R8_unclear": [0.60, 0.40, 0.30, 0.02],
}


@dataclass
class Retina:
    pr_index: np.ndarray        # connectome row of each photoreceptor
    pr_column: np.ndarray       # column id 0..n_col-1
    pr_sens: np.ndarray         # (n_pr, 4)
    col_side: np.ndarray        # per column
    col_hex: np.ndarray         # (n_col, 2)

    @property
    def n_columns(self) -> int:
        return len(self.col_side)


def build_retina(c) -> Retina:
    """Columns = sorted distinct (side, hex1, hex2) of the photoreceptors (retina.py:123-139)."""
    c.require("optic_columns")
    nrn = c.neurons
    m = nrn.type.isin(PHOTORECEPTOR_TYPES) & nrn.hex1.notna()
    pr = nrn[m]
    keys = list(zip(pr.hex_side, pr.hex1.astype(int), pr.hex2.astype(int)))
    uniq = sorted(set(keys))
    col_of = {k: i for i, k in enumerate(uniq)}
    return Retina(pr_index=np.flatnonzero(m.to_numpy()), pr_column=np.array([col_of[k] for k in keys], dtype=np.int64),
                  pr_sens=np.array([SENSITIVITY[t] for t in pr.type], dtype=np.float32).reshape(-1, 4),
                  col_side=np.array([k[0] for k in uniq]),
                  col_hex=np.array([[k[1], k[2]] for k in uniq], dtype=float).reshape(-1, 2))
