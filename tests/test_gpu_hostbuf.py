"""Host-buffer calls (fft3d_plane_filter) with pageable and with pinned
frames and outputs give the same result as the device-buffer call: a
pageable frame is staged through pinned memory by the calling thread, a
pageable destination gets its result through pinned memory. Several threads
per plane, as a frame-parallel frame server calls the filter."""
import threading

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs

F = 15
CASES = [("bt5_sharpen", dict(sigma=3.0, bt=5, sharpen=0.3)), ("bt3_crop", dict(sigma=2.0, bt=3, l=8, t=4, r=4, b=6)),
         ("kalman", dict(sigma=3.0, bt=0)), ("bt1", dict(sigma=2.5, bt=1))]


def _host(planes, filt, pinned, threads):
    import torch
    p = make_params(**filt)
    descs = plane_descs([a.shape[1:] for a in planes], 8, F)
    outs = []
    for a, d in zip(planes, descs):
        e = engine.PlaneEngine(p, d)
        src = torch.from_numpy(a).pin_memory().numpy() if pinned else a.copy()
        out = torch.empty_like(torch.from_numpy(a)).pin_memory().numpy() if pinned else np.empty_like(a)
        if filt["bt"] == 0:
            threads_here = 1  # Kalman: frames in order
        else:
            threads_here = threads
        counter, lock = [0], threading.Lock()

        def work():
            while True:
                with lock:
                    n = counter[0]
                    counter[0] += 1
                if n >= F:
                    return
                e.filter(n, [src[n + k] if 0 <= n + k < F else None for k in range(-2, 3)], out[n])

        th = [threading.Thread(target=work) for _ in range(threads_here)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        outs.append(out.copy())
        e.close()
    return outs


@pytest.mark.gpu
@pytest.mark.parametrize("name,filt", CASES, ids=[c[0] for c in CASES])
def test_pageable_and_pinned_host_calls_agree(gpu, name, filt):
    planes = synth.make_clip(192, 144, F, noise_sigma=5, seed=95)
    want = engine.filter_clip(planes, **filt)
    for pinned in (False, True):
        got = _host(planes, filt, pinned, threads=4)
        for w, g in zip(want, got):
            assert np.array_equal(w, g), (name, pinned)
