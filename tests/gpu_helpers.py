"""Run the native LIF entry point on a host-side oracle.LifState, through the C ABI (GPU tests)."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from flyb200 import _abi

LIF_ARRAYS = ("v", "g", "refrac", "adapt", "res", "rate", "counts", "spikes", "drive", "poisson_p")


def native_lif_run(state, out_ptr, out_edge, params, *, n_delay, flags, nsteps, seed=0, uniforms=None,
                   fly_steps=None, raster=False, launch=_abi.LAUNCH_PERSISTENT, block=256, grid=0, fly0=0,
                   device="cuda", items_per_thread=0, with_sync=True, staged=0, defer=False, adapt_jump=None,
                   clocks=None, slow=None):
    """Same contract as oracle.lif_run, executed by flyb_lif_run on the device."""
    dev = torch.device(device)
    n, B = state.n, state.batch
    words = (n * B + 31) // 32
    d = {k: torch.from_numpy(getattr(state, k)).to(dev) for k in LIF_ARRAYS}
    active = torch.from_numpy(state.active).to(dev)
    std_u = torch.from_numpy(state.std_u).to(dev)
    ring = torch.from_numpy(state.ring).to(dev)
    ptr = torch.from_numpy(np.ascontiguousarray(out_ptr, np.int32)).to(dev)
    edge = torch.from_numpy(np.ascontiguousarray(out_edge, np.int32)).to(dev)
    uni = None if uniforms is None else torch.from_numpy(np.ascontiguousarray(uniforms, np.float32)).to(dev)
    fs = None if fly_steps is None else torch.from_numpy(np.ascontiguousarray(fly_steps, np.int32)).to(dev)
    r = torch.zeros(nsteps, words, dtype=torch.int32, device=dev) if raster else None
    events = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    sync = torch.zeros(_abi.LIF_SYNC_WORDS, dtype=torch.int32, device=dev)
    P = np.ascontiguousarray(params, np.float32)
    a = _abi.LifArgs(n=n, batch=B, n_delay=n_delay, ring_slots=state.ring_slots, ring_mode=state.ring_mode,
                     ring_pos=state.ring_pos, flags=flags, nsteps=nsteps, launch=launch, block=block, grid=grid,
                     fly0=fly0, items_per_thread=items_per_thread, staged=staged, step0=state.step, seed=seed, out_ptr=ptr.data_ptr(), out_edge=edge.data_ptr(),
                     v=d["v"].data_ptr(), g=d["g"].data_ptr(), refrac=d["refrac"].data_ptr(),
                     adapt=d["adapt"].data_ptr(), res=d["res"].data_ptr(), rate=d["rate"].data_ptr(),
                     counts=d["counts"].data_ptr(), spikes=d["spikes"].data_ptr(), drive=d["drive"].data_ptr(),
                     poisson_p=d["poisson_p"].data_ptr(), active=active.data_ptr(), std_u=std_u.data_ptr(),
                     params=P.ctypes.data, ring=ring.data_ptr(), uniforms=None if uni is None else uni.data_ptr(),
                     fly_steps=None if fs is None else fs.data_ptr(), raster=None if r is None else r.data_ptr(),
                     events=events.data_ptr(), status=status.data_ptr(), sync=sync.data_ptr() if with_sync else None)
    aj = None if adapt_jump is None else torch.from_numpy(np.ascontiguousarray(adapt_jump, np.float32)).to(dev)
    a.adapt_jump = None if aj is None else aj.data_ptr()
    ck = cc = acc = None
    if clocks is not None:
        ck = torch.from_numpy(np.ascontiguousarray(clocks[0], np.uint8)).to(dev)
        cc = torch.from_numpy(np.ascontiguousarray(clocks[1], np.float32)).to(dev)
        if getattr(state, "clock_acc", None) is None:
            state.clock_acc = np.zeros((n, B), np.int64)
        acc = torch.from_numpy(state.clock_acc).to(dev)
        a.clock_k, a.clock_coef, a.clock_acc = ck.data_ptr(), cc.data_ptr(), acc.data_ptr()
    held = []
    if slow is not None:
        K = len(slow["classes"])
        if getattr(state, "slow_ring", None) is None:
            state.slow_ring = np.zeros((K, state.ring_slots, n, B), np.int64)
            state.slow_g = np.zeros((K, n, B), np.float32)
            state.g_slow = np.zeros((n, B), np.float32)
        srings = torch.from_numpy(state.slow_ring).to(dev)
        sg = torch.from_numpy(state.slow_g).to(dev)
        gs = torch.from_numpy(state.g_slow).to(dev)
        a.slow_classes, a.slow_mode = K, _abi.SLOW_MODE_CODES[slow["mode"]]
        a.slow_norm, a.slow_th_max = slow["norm"], slow["th_max"]
        a.slow_clip_lo, a.slow_clip_hi = slow["clip"]
        for c, (sp_, se_, decay) in enumerate(slow["classes"]):
            tp = torch.from_numpy(np.ascontiguousarray(sp_, np.int32)).to(dev)
            te = torch.from_numpy(np.ascontiguousarray(se_, np.int32)).to(dev)
            held += [tp, te]
            a.slow_out_ptr[c], a.slow_out_edge[c] = tp.data_ptr(), te.data_ptr()
            a.slow_ring[c], a.slow_g[c] = srings[c].data_ptr(), sg[c].data_ptr()
            a.slow_decay[c] = decay
        a.g_slow = gs.data_ptr()
        sacc = None
        if clocks is not None:
            if getattr(state, "slow_clock_acc", None) is None:
                state.slow_clock_acc = np.zeros((K, n, B), np.int64)
            sacc = torch.from_numpy(state.slow_clock_acc).to(dev)
            for c in range(K):
                a.slow_clock_acc[c] = sacc[c].data_ptr()
    if defer:
        a.flags |= _abi.LIF_DEFER_DELIVERY
        cap = int(_abi.lib().flyb_lif_spike_capacity(ct.byref(a)))
        assert cap > 0
        spike_list = torch.empty(cap, 4, dtype=torch.int32, device=dev)
        spike_n = torch.zeros(1, dtype=torch.int32, device=dev)
        a.spike_list, a.spike_n, a.spike_cap = spike_list.data_ptr(), spike_n.data_ptr(), cap
    rc = _abi.lib().flyb_lif_run(ct.byref(a), torch.cuda.current_stream(dev).cuda_stream)
    if rc:
        raise RuntimeError(f"flyb_lif_run: error {rc}")
    torch.cuda.synchronize(dev)
    st = status.cpu().numpy()
    if st[0]:
        raise RuntimeError(f"kernel status {st.tolist()}")
    for k in LIF_ARRAYS:
        getattr(state, k)[...] = d[k].cpu().numpy()
    state.ring[...] = ring.cpu().numpy()
    if acc is not None:
        state.clock_acc[...] = acc.cpu().numpy()
    if slow is not None:
        state.slow_ring[...] = srings.cpu().numpy()
        state.slow_g[...] = sg.cpu().numpy()
        state.g_slow[...] = gs.cpu().numpy()
        if sacc is not None:
            state.slow_clock_acc[...] = sacc.cpu().numpy()
    state.ring_pos = (state.ring_pos + nsteps) % state.ring_slots
    state.step += nsteps
    if fly_steps is not None:
        fly_steps[...] = fs.cpu().numpy()
    return (r.cpu().numpy().view(np.uint32) if raster else None), int(events.item())


def native_lif_run_split(state, out_ptr, out_edge, params, *, split, n_delay, flags, nsteps, seed=0, fly_steps=None,
                         block=256, items_per_thread=0, staged=0, device="cuda", defer=False):
    """oracle.lif_run's contract (raster always on), but every step runs as two neuron ranges,
    [0, split) and [split, n), launched on two streams that overlap, each with
    FLYB_LIF_NO_ADVANCE, then flyb_lif_advance on the joined stream (the device clock keeps the
    step counter, ring slot and raster slot)."""
    dev = torch.device(device)
    n, B = state.n, state.batch
    words = (n * B + 31) // 32
    d = {k: torch.from_numpy(getattr(state, k)).to(dev) for k in LIF_ARRAYS}
    active = torch.from_numpy(state.active).to(dev)
    std_u = torch.from_numpy(state.std_u).to(dev)
    ring = torch.from_numpy(state.ring).to(dev)
    ptr = torch.from_numpy(np.ascontiguousarray(out_ptr, np.int32)).to(dev)
    edge = torch.from_numpy(np.ascontiguousarray(out_edge, np.int32)).to(dev)
    fs = None if fly_steps is None else torch.from_numpy(np.ascontiguousarray(fly_steps, np.int32)).to(dev)
    r = torch.zeros(nsteps, words, dtype=torch.int32, device=dev)
    clock = torch.tensor([state.step, state.ring_pos, 0], dtype=torch.int64, device=dev)
    events = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    P = np.ascontiguousarray(params, np.float32)
    a = _abi.LifArgs(n=n, batch=B, n_delay=n_delay, ring_slots=state.ring_slots, ring_mode=state.ring_mode,
                     ring_pos=0, flags=flags | _abi.LIF_NO_ADVANCE, nsteps=1, launch=_abi.LAUNCH_STEP, block=block,
                     raster_slots=nsteps, raster_pos=0, items_per_thread=items_per_thread, staged=staged, seed=seed,
                     out_ptr=ptr.data_ptr(), out_edge=edge.data_ptr(),
                     v=d["v"].data_ptr(), g=d["g"].data_ptr(), refrac=d["refrac"].data_ptr(),
                     adapt=d["adapt"].data_ptr(), res=d["res"].data_ptr(), rate=d["rate"].data_ptr(),
                     counts=d["counts"].data_ptr(), spikes=d["spikes"].data_ptr(), drive=d["drive"].data_ptr(),
                     poisson_p=d["poisson_p"].data_ptr(), active=active.data_ptr(), std_u=std_u.data_ptr(),
                     params=P.ctypes.data, ring=ring.data_ptr(), fly_steps=None if fs is None else fs.data_ptr(),
                     clock=clock.data_ptr(), raster=r.data_ptr(), events=events.data_ptr(), status=status.data_ptr())
    lib = _abi.lib()
    main = torch.cuda.current_stream(dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    lists = {}
    if defer:
        flags |= _abi.LIF_DEFER_DELIVERY
        a.flags = flags | _abi.LIF_NO_ADVANCE
        for first, count in ((0, split), (split, n - split)):
            a.n_first, a.n_count = first, count
            cap = int(lib.flyb_lif_spike_capacity(ct.byref(a)))
            lists[first] = (torch.empty(cap, 4, dtype=torch.int32, device=dev),
                            torch.zeros(1, dtype=torch.int32, device=dev), cap)
    for _ in range(nsteps):
        for stream, first, count in ((s1, 0, split), (s2, split, n - split)):
            stream.wait_stream(main)
            a.n_first, a.n_count = first, count
            if defer:
                lst = lists[first]
                a.spike_list, a.spike_n, a.spike_cap = lst[0].data_ptr(), lst[1].data_ptr(), lst[2]
            rc = lib.flyb_lif_run(ct.byref(a), stream.cuda_stream)
            if rc:
                torch.cuda.synchronize(dev)
                raise RuntimeError(f"flyb_lif_run: error {rc}")
        main.wait_stream(s1)
        main.wait_stream(s2)
        a.flags = flags & ~_abi.LIF_DEFER_DELIVERY
        rc = lib.flyb_lif_advance(ct.byref(a), main.cuda_stream)
        a.flags = flags | _abi.LIF_NO_ADVANCE
        if rc:
            raise RuntimeError(f"flyb_lif_advance: error {rc}")
    torch.cuda.synchronize(dev)
    st = status.cpu().numpy()
    if st[0]:
        raise RuntimeError(f"kernel status {st.tolist()}")
    for k in LIF_ARRAYS:
        getattr(state, k)[...] = d[k].cpu().numpy()
    state.ring[...] = ring.cpu().numpy()
    state.ring_pos = (state.ring_pos + nsteps) % state.ring_slots
    state.step += nsteps
    if fly_steps is not None:
        fly_steps[...] = fs.cpu().numpy()
    return r.cpu().numpy().view(np.uint32), int(events.item())
