"""Host-side LIF weight construction, one time per brain (scipy, CPU; not on the step path).

Restates the connection rules of flyverse/brain.py so that a brain built here from the same
connectome and LIFParams holds the same float32 W[post, pre] as the reference:
  shaped_weights   brain.py:302-338  receptor sign / gain class, per-transmitter factor, connection
                                     cap, superclass and type path gains, same-type damping
  fan-in scale     brain.py:407-425  (input_norm_ref / total)^alpha clipped to [0.02, 1], row-wise
  unitary size     brain.py:426      x w_syn
The rules are a data contract (the weights must be identical for rasters to be), so the steps are
the reference's; the code is this package's own.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
import re

import numpy as np
import scipy.sparse as sp

DEFAULT_PATH_GAIN = [(r"^descending_neuron$", r"^vnc_", 3.0), (r"^visual_projection$", r"^descending_neuron$", 2.0)]
DEFAULT_TYPE_PATH_GAIN = [(r"^(LC4|LPLC2)$", r"^DNp01$", 3.0)]
DEFAULT_STD_U_BY_TYPE = {r"^ORN_": 0.2, r"^(lLN|v2LN|v3LN|il3LN|l2LN|vLN)": 0.2}
DEFAULT_ADAPT_BY_TYPE: dict = {}
DEFAULT_RECEPTOR_GAIN = {"none": 1.0, "low": 0.5, "mid": 1.0, "high": 1.5}
RECEPTOR_MODELS = (None, "sign", "sign+gain", "full")


def _match(pattern: str, labels: np.ndarray) -> np.ndarray:
    rx = re.compile(pattern)
    cache = {t: bool(rx.match(t)) for t in np.unique(labels)}
    return np.fromiter((cache[t] for t in labels), bool, len(labels))


def receptor_gain(p):
    if p.receptor_model in ("sign+gain", "full"):
        return DEFAULT_RECEPTOR_GAIN if p.receptor_gain is None else p.receptor_gain
    return None


def check_receptor(c, p, receptor):
    if p.receptor_model not in RECEPTOR_MODELS:
        raise ValueError(f"receptor_model must be one of {RECEPTOR_MODELS}")
    if p.receptor_model is None:
        return None
    if receptor is None:
        raise ValueError("receptor_model needs the per-edge receptor lookup: pass receptor= (the reference's "
                         "connectome.receptor_signs(c, ...)), or LIFParams(receptor_model=None) for the "
                         "presynaptic-sign rule")
    if len(receptor.fast_sign) != c.W.nnz:
        raise ValueError("receptor signs are not aligned with this connectome's W")
    return receptor


def _nt_factor(c, by_nt: dict) -> np.ndarray:
    from .connectome import NT_SIGN
    bad = sorted(set(by_nt) - set(NT_SIGN))
    if bad:
        raise ValueError(f"w_syn_by_nt: unknown transmitters {bad}")
    nt = c.neurons.nt.fillna("unknown").to_numpy() if "nt" in c.neurons.columns else np.full(c.n, "unknown")
    f = np.ones(c.n, dtype=np.float32)
    for k, v in by_nt.items():
        v = float(v)
        if not (math.isfinite(v) and v >= 0):
            raise ValueError(f"w_syn_by_nt[{k!r}] must be finite and >= 0")
        f[nt == k] = np.float32(v)
    return f


def _gain_pairs(W: sp.csr_matrix, labels: np.ndarray, rules) -> sp.csr_matrix:
    Wc = W.tocoo()
    for pre_re, post_re, factor in rules:
        pre_m, post_m = _match(pre_re, labels), _match(post_re, labels)
        Wc.data[pre_m[Wc.col] & post_m[Wc.row]] *= np.float32(factor)
    return Wc.tocsr()


def shaped_weights(c, p, receptor=None) -> sp.csr_matrix:
    """Connection rules before the fan-in normalisation (brain.py:302-338)."""
    W = c.W.tocsr().copy()
    receptor = check_receptor(c, p, receptor)
    if receptor is not None:
        W.data = np.abs(W.data) * receptor.fast_factor(receptor_gain(p))
    if p.w_syn_by_nt:
        W.data = W.data * _nt_factor(c, p.w_syn_by_nt)[W.indices]
    if p.conn_cap > 0:
        W.data = np.sign(W.data) * np.minimum(np.abs(W.data), np.float32(p.conn_cap))
    rules = DEFAULT_PATH_GAIN if p.path_gain is None else p.path_gain
    if rules:
        W = _gain_pairs(W, c.neurons.superclass.fillna("").to_numpy(), rules)
    rules = DEFAULT_TYPE_PATH_GAIN if p.type_path_gain is None else p.type_path_gain
    if rules:
        W = _gain_pairs(W, c.neurons.type.fillna("").to_numpy(), rules)
    if p.same_type_gain != 1.0:
        types = c.neurons.type.fillna("").to_numpy()
        Wc = W.tocoo()
        same = (types[Wc.row] == types[Wc.col]) & (types[Wc.row] != "")
        Wc.data[same] *= np.float32(p.same_type_gain)
        W = Wc.tocsr()
    return W


def _norm_key(p):
    recep = None
    if p.receptor_model is not None:
        g = receptor_gain(p)
        recep = (p.receptor_model, p.receptor_net_rule, p.receptor_nt_class_fallback, p.receptor_table,
                 tuple(sorted(g.items())) if g else None)
    return repr((p.conn_cap, DEFAULT_PATH_GAIN if p.path_gain is None else p.path_gain,
                 DEFAULT_TYPE_PATH_GAIN if p.type_path_gain is None else p.type_path_gain,
                 p.same_type_gain, recep) + ((tuple(sorted(p.w_syn_by_nt.items())),) if p.w_syn_by_nt else ()))


def lif_weights(c, p, receptor=None) -> tuple[sp.csr_matrix, np.ndarray | None]:
    """W[post, pre] in mV per transmitted spike and the fan-in scale (brain.py:405-426)."""
    W = shaped_weights(c, p, receptor)
    scale = None
    if p.input_norm_alpha > 0:
        ref = c.reference
        key = _norm_key(p)
        if ref is c:
            tot = np.asarray(abs(W).sum(axis=1)).ravel()
            ref._norm_cache[key] = tot
        else:
            if key not in ref._norm_cache:
                ref._norm_cache[key] = np.asarray(abs(shaped_weights(ref, p)).sum(axis=1)).ravel()
            tot = ref._norm_cache[key][ref.index_of(c.neurons.bodyId)]
        scale = np.clip((p.input_norm_ref / np.maximum(tot, 1.0)) ** p.input_norm_alpha, 0.02, 1.0).astype(np.float32)
        W = (sp.diags(scale) @ W).tocsr()
    W = W.copy()
    W.data = W.data * np.float32(p.w_syn)
    return W, scale


# ------------------------------------------------------------------ the slow receptor tone
# receptor_model "full" (brain.py:100-147, 176-230, 341-359): a slow tone per neuron and class,
# driven by the entries whose receptor row has a slow sign. Class names, defaults and modes are the
# reference's, so the same parameters give the same tone.
GAIN_CLASSES = ["none", "low", "mid", "high"]
SLOW_CLASSES = ["none", "metabotropic_classical", "monoamine"]
SLOW_MODES = ("additive", "gain", "threshold")
DEFAULT_SLOW_GAIN_BY_CLASS = {"metabotropic_classical": 0.0, "monoamine": None}
DEFAULT_SLOW_TAU_BY_CLASS = {"metabotropic_classical": 100.0, "monoamine": None}
SLOW_THRESHOLD_MAX_FRAC = 0.9


@dataclass
class ReceptorSigns:
    """Per stored entry of W (CSR order): the receptor model's fast and slow signs, gain classes
    (int8 codes into GAIN_CLASSES), slow class (codes into SLOW_CLASSES) and synapse counts -- the
    record the reference's connectome.receptor_signs builds (connectome.py:113-170); any object
    with these fields and methods (the reference's own included) can be passed as `receptor=`."""
    fast_sign: np.ndarray
    slow_sign: np.ndarray
    fast_gain: np.ndarray
    slow_gain: np.ndarray
    count: np.ndarray | None = None
    slow_class: np.ndarray | None = None

    def fast_factor(self, gain: dict | None = None) -> np.ndarray:
        f = self.fast_sign.astype(np.float32)
        if gain:
            g = np.array([float(gain.get(k, 1.0)) for k in GAIN_CLASSES], dtype=np.float32)
            f = f * g[self.fast_gain]
        return f

    def slow_factor(self, gain: dict | None = None, slow_class: str | None = None) -> np.ndarray:
        f = self.slow_sign.astype(np.float32)
        if gain:
            g = np.array([float(gain.get(k, 1.0)) for k in GAIN_CLASSES], dtype=np.float32)
            f = f * g[self.slow_gain]
        if slow_class is not None:
            if self.slow_class is None:
                raise ValueError("this receptor record carries no slow-class codes")
            f = f * (self.slow_class == SLOW_CLASSES.index(slow_class)).astype(np.float32)
        return f


@dataclass
class SlowSpec:
    """The resolved slow tone: mode, per-class scale and time constant (non-zero scales only), the
    fast synaptic time constant, and the normalisation of the multiplicative modes (v_th - v_rest)."""
    mode: str
    gain: dict
    tau: dict
    tau_syn: float
    norm_mv: float
    clip: tuple = (0.0, 4.0)

    @property
    def classes(self) -> list:
        return list(self.gain)


def slow_spec(p) -> SlowSpec | None:
    """None unless receptor_model == "full" and some class has a non-zero scale (brain.py:206-225)."""
    if p.receptor_model != "full":
        return None
    if p.slow_mode not in SLOW_MODES:
        raise ValueError(f"slow_mode must be one of {SLOW_MODES}")
    gains = dict(DEFAULT_SLOW_GAIN_BY_CLASS, monoamine=float(p.slow_gain))
    gains.update({k: float(v) for k, v in (p.slow_gain_by_class or {}).items()})
    taus = dict(DEFAULT_SLOW_TAU_BY_CLASS, monoamine=float(p.slow_tau_ms))
    taus.update({k: float(v) for k, v in (p.slow_tau_by_class or {}).items()})
    bad = (set(gains) | set(taus)) - set(SLOW_CLASSES[1:])
    if bad:
        raise ValueError(f"unknown slow classes {sorted(bad)}; use {SLOW_CLASSES[1:]}")
    for k, tau in taus.items():
        if not (math.isfinite(tau) and tau > 0):
            raise ValueError(f"slow tau of class {k!r} must be positive and finite")
    active = {k: g for k, g in gains.items() if g != 0.0}
    if not active:
        return None
    return SlowSpec(p.slow_mode, active, {k: taus[k] for k in active}, float(p.tau_syn), float(p.v_th - p.v_rest),
                    tuple(float(x) for x in p.slow_gain_clip))


def slow_weights(c, p, receptor, spec: SlowSpec, scale: np.ndarray | None) -> dict:
    """{class: csr} slow matrices in mV per transmitted spike (brain.py:341-359, 410-429): per entry
    count x slow sign x gain factor, capped like the fast synapses, entries of other classes
    dropped; then the fan-in scale of the fast weights and w_syn x the class scale."""
    if getattr(receptor, "count", None) is None:
        raise ValueError("the slow tone needs the receptor record's synapse counts")
    out = {}
    for cls in spec.classes:
        S = c.W.tocsr().copy()
        S.data = receptor.count * receptor.slow_factor(receptor_gain(p), slow_class=cls)
        if p.conn_cap > 0:
            S.data = np.sign(S.data) * np.minimum(np.abs(S.data), np.float32(p.conn_cap))
        S.eliminate_zeros()
        if scale is not None:
            S = (sp.diags(scale) @ S).tocsr()
        S = S.copy()
        S.data = S.data * np.float32(p.w_syn * spec.gain[cls])
        out[cls] = S
    return out


def per_type(c, mapping: dict, default: float) -> np.ndarray:
    """(N,) float32 value per neuron from {type regex: value} (re.match), later entries win."""
    out = np.full(c.n, default, dtype=np.float32)
    if mapping:
        types = c.neurons.type.fillna("").to_numpy()
        for pat, val in mapping.items():
            out[_match(pat, types)] = val
    return out


def integer_counts(W: sp.spmatrix, w_syn: float) -> np.ndarray | None:
    """Signed integer synapse counts c with float32(c) * float32(w_syn) == W.data exactly, else None.

    When they exist the LIF runs on the int32 count ring (exact integer sums, g += w_syn * sum)."""
    w = np.float32(w_syn)
    if w == 0:
        return None
    data = np.asarray(W.data, np.float32)
    c = np.round(data / w)
    if not np.all(np.abs(c) < 2**24):
        return None
    if not np.array_equal(c.astype(np.float32) * w, data):
        return None
    return c.astype(np.int32)
