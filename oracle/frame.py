"""ORACLE (test infrastructure): one optic frame on the CPU, the order of flyverse/optic.py:563-604.

photoreceptor stage (optic.py:496-517) in numpy FP32, held inputs and drive through
oracle.spmm, substeps through oracle.optic_run. State is fly-minor [n][B] like the device.
"""
from __future__ import annotations

import numpy as np

from . import optic_run, spmm


def photoreceptor(L, st: dict, rad: np.ndarray, dt_ms: float, p) -> np.ndarray:
    """rad (B, n_col, 4) -> a_pr [n_pr][B]; updates st['I_lp'], st['I_mean'], st['contrast'] (B, n_col*5)."""
    f32 = np.float32
    sens = L.sens.astype(f32)
    r = rad[:, L.pr_column, :].astype(f32)                                  # (B, n_pr, 4)
    ip = r[..., 0] * sens[:, 0]
    for k in (1, 2, 3):
        ip = ip + r[..., k] * sens[:, k]
    avg = L.avg.tocsr()
    I = np.zeros((rad.shape[0], avg.shape[0]), f32)
    for c in range(avg.shape[0]):
        acc = np.zeros(rad.shape[0], f32)
        for e in range(avg.indptr[c], avg.indptr[c + 1]):
            acc = acc + f32(avg.data[e]) * ip[:, avg.indices[e]]
        I[:, c] = acc
    fresh = st["fresh"][:, None]
    lp = np.where(fresh, I, st["I_lp"])
    mean = np.where(fresh, I, st["I_mean"])
    st["fresh"][:] = False
    a_lp, a_ad = float(np.exp(-dt_ms / p.tau_lp_ms)), float(np.exp(-dt_ms / p.tau_adapt_ms))
    lp = f32(a_lp) * lp + f32(1 - a_lp) * I
    mean = f32(a_ad) * mean + f32(1 - a_ad) * lp
    con = np.clip((lp - mean) / (mean + f32(p.eps)), -1.0, p.contrast_clip).astype(f32)
    con = np.where(L.has.reshape(-1)[None], con, f32(0))
    st["I_lp"], st["I_mean"], st["contrast"] = lp.astype(f32), mean.astype(f32), con
    return np.ascontiguousarray(con[:, L.pr_cell].T)                           # [n_pr][B]


def _csr_mv(M, x, alpha):
    """alpha x (M @ x) for x [cols][B], rows summed in CSR order in float32 (the reference's
    sparse product), through the C restatement."""
    M = M.tocsr()
    return spmm(M.indptr, M.indices, M.data, x, x.shape[1], rows=M.shape[0], alpha=alpha)


def stream_signals(hooks, st: dict, dr: np.ndarray, update: bool) -> list:
    """x per hook stream (optic.py:453-472) in FP32: u = dr - G dr, y = u - gain A, x = rectify(y);
    with `update` every adaptation state st["A"][k] then relaxes towards u."""
    f32 = np.float32
    u = dr if hooks.G is None else (dr - _csr_mv(hooks.G, dr, 1.0)).astype(f32)
    xs = []
    for s in hooks.streams:
        k = s["adapt_id"]
        y = u if k < 0 else (u - (f32(hooks.adapt_gain[k]) * st["A"][k]).astype(f32)).astype(f32)
        mode = s["mode"]
        xs.append(y if mode is None else np.maximum(y, f32(0)) if mode == "pos" else
                  np.maximum(-y, f32(0)) if mode == "neg" else np.abs(y))
    if update:
        for k, decay in enumerate(hooks.adapt_decay):
            st["A"][k] = (u + ((st["A"][k] - u) * f32(decay)).astype(f32)).astype(f32)
    return xs


def _hooked_product(rest, blocks, dr, xs):
    """rest @ dr plus every stream block on its signal, added in stream order."""
    acc = _csr_mv(rest, dr, 1.0)
    for W, x in zip(blocks, xs):
        if W is not None:
            acc = (acc + _csr_mv(W, x, 1.0)).astype(np.float32)
    return acc


def ext_substeps(L, st: dict, pr, spk, steps: int, p, slow: dict | None = None, hooks=None) -> None:
    """The substeps with the slow receptor tone and / or the per-stream hooks (optic.py:526-551),
    FP32 in the reference order. slow = {"mode", "norm", "clip", "classes": [(rs, rr, scale, decay)]}
    with state st["g_cls"] [K][m][B], st["g_slow"] [m][B], st["held"] [K][m][B]; hooks: a
    flyb200.optic.StreamHooks with state st["A"] [K_a][m][B]."""
    f32 = np.float32
    b = L.b[:, None].astype(f32)
    a = L.a[:, None].astype(f32)
    for _ in range(steps):
        r = (st["v"] + b).astype(f32)
        if slow is not None and slow["mode"] == "threshold":
            r = (r + np.minimum(st["g_slow"], f32(0.9 * slow["norm"]))).astype(f32)
        dr = (np.clip(r, f32(0), f32(1)) - b).astype(f32)
        if hooks is None:
            rec = _csr_mv(L.M_rr, dr, p.gain_rr)
        else:
            xs = stream_signals(hooks, st, dr, True)
            rec = (f32(p.gain_rr) * _hooked_product(hooks.rest_rr, [s["W_rr"] for s in hooks.streams], dr, xs)).astype(f32)
        ad = (f32(p.adapt_gain) * st["adapt"]).astype(f32)
        if slow is None:
            inp = (((rec + pr).astype(f32) - ad).astype(f32) + spk).astype(f32)
        else:
            tone = np.zeros_like(dr)
            for k, (rs, rr, scale, decay) in enumerate(slow["classes"]):
                target = st["held"][k].copy()
                if rr is not None:
                    target = (target + _csr_mv(rr, dr, p.gain_rr)).astype(f32)
                ts = (target * f32(scale)).astype(f32)
                gk = (ts + (st["g_cls"][k] - ts) * f32(decay)).astype(f32)
                st["g_cls"][k] = gk
                tone = (tone + gk).astype(f32)
            st["g_slow"] = tone
            syn = ((rec + pr).astype(f32) + spk).astype(f32)
            if slow["mode"] == "gain":
                fac = np.clip((f32(1) + tone / f32(slow["norm"])).astype(f32), f32(slow["clip"][0]), f32(slow["clip"][1]))
                inp = ((syn * fac).astype(f32) - ad).astype(f32)
            else:
                inp = (syn - ad).astype(f32)
                if slow["mode"] == "additive":
                    inp = (inp + tone).astype(f32)
        st["v"] = (inp + (st["v"] - inp) * a).astype(f32)
        st["adapt"] = (dr + (st["adapt"] - dr) * f32(L.aad)).astype(f32)


def frame(L, st: dict, rad: np.ndarray, spk_rate: np.ndarray, frame_ms: float, p, slow: dict | None = None,
          hooks=None) -> np.ndarray:
    """Advance one frame in place; returns the drive (B, N) in mV. spk_rate: (B, N) Hz. `slow`: the
    slow receptor tone, `hooks`: the per-stream hooks (see ext_substeps)."""
    B = rad.shape[0]
    a_pr = photoreceptor(L, st, rad, frame_ms, p)
    total = st["pending"] + frame_ms
    steps = int(np.floor((total + 1e-9) / p.dt_ms))
    st["pending"] = max(0.0, total - steps * p.dt_ms)
    rates = np.ascontiguousarray(spk_rate.T.astype(np.float32))                # [N][B]
    if steps:
        M = L.M_rp.tocsr()
        pr = spmm(M.indptr, M.indices, M.data, a_pr, B, rows=M.shape[0], alpha=p.gain_in)
        M = L.M_rs.tocsr()
        spk = spmm(M.indptr, M.indices, M.data, rates, B, rows=M.shape[0], x_index=L.spk_idx, x_div=100.0,
                   x_lo=0.0, x_hi=3.0, alpha=p.gain_fb)
        if slow is None and hooks is None:
            M = L.M_rr.tocsr()
            optic_run(st["v"], st["adapt"], M.indptr, M.indices, M.data, pr, spk, L.a, L.b, p.gain_rr, p.adapt_gain,
                      L.aad, steps)
        else:
            for k, (rs, rr, scale, decay) in enumerate(slow["classes"] if slow is not None else []):
                st["held"][k] = 0.0
                if rs is not None:
                    rs = rs.tocsr()
                    st["held"][k] = spmm(rs.indptr, rs.indices, rs.data, rates, B, rows=rs.shape[0], x_index=L.spk_idx,
                                         x_div=100.0, x_lo=0.0, x_hi=3.0, alpha=p.gain_fb)
            ext_substeps(L, st, pr, spk, steps, p, slow, hooks)
    b = L.b[:, None].astype(np.float32)
    r = (st["v"] + b).astype(np.float32)
    if slow is not None and slow["mode"] == "threshold":
        r = (r + np.minimum(st["g_slow"], np.float32(0.9 * slow["norm"]))).astype(np.float32)
    delta = (np.clip(r, 0.0, 1.0) - b).astype(np.float32)
    st["delta"] = delta
    n = spk_rate.shape[1]
    drive = np.zeros((n, B), np.float32)
    if hooks is None:
        M = L.M_sr.tocsr()
        spmm(M.indptr, M.indices, M.data, delta, B, rows=M.shape[0], y=drive, y_index=L.spk_idx, alpha=p.gain_out_mv,
             y_lo=-p.drive_clip_mv, y_hi=p.drive_clip_mv)
    else:                               # optic.py:485-495, 602
        acc = _hooked_product(hooks.rest_sr, [s["W_sr"] for s in hooks.streams], delta,
                              stream_signals(hooks, st, delta, False))
        drive[L.spk_idx] = np.clip((np.float32(p.gain_out_mv) * acc).astype(np.float32), -p.drive_clip_mv,
                                   p.drive_clip_mv)
    return drive.T
