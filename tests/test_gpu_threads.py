"""GPU: launchers called from several host threads at once.

The scorer's launchers fill a parameter block per call and set a per-device
shared-memory limit that follows the band count.  Two host threads that score
different frames concurrently (one of 113 bands, one of 40; FP32 on the FMA
scorer and FP16 on the tensor-core scorer) must each get exactly the maps a
single-thread run gives: the same kernels on the same inputs, so the maps are
compared bit for bit.  The moments launcher (another per-call parameter block)
runs concurrently with the scorer in the same way.
"""
import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(hsi, H, W, B, T, dtype, seed):
    sc = hsi.scene(B, n_targets=T, target_frac=0.01, frame_seed=seed)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype, truth=False)
    targets = hsi.scene_targets(sc)
    tg = torch.from_numpy(targets).cuda()
    nr = torch.from_numpy(hsi.target_norms(targets)).cuda()
    cem = torch.from_numpy((np.random.default_rng(seed).standard_normal((T, B)) * 0.05).astype(np.float32)).cuda()
    return dict(cube=cube, H=H, W=W, B=B, T=T, dtype=dtype, tg=tg, nr=nr, cem=cem)


def _score(hsi, c, stream):
    P = c["H"] * c["W"]
    out = dict(maps=torch.empty((c["T"], P), device="cuda"), best=torch.empty(P, device="cuda"),
               bt=torch.empty(P, dtype=torch.int32, device="cuda"), cbest=torch.empty(P, device="cuda"),
               cbt=torch.empty(P, dtype=torch.int32, device="cuda"))
    f = hsi.make_frame(c["cube"], c["H"], c["W"], c["B"], c["dtype"], sam_targets=c["tg"], sam_norms=c["nr"],
                       sam_maps=out["maps"], sam_best=out["best"], sam_best_target=out["bt"],
                       cem_weights=c["cem"], cem_best=out["cbest"], cem_best_target=out["cbt"], map_stride=P)
    hsi.score_frames([f], stream=stream)
    return out


def _moments(hsi, c, stream):
    with torch.cuda.stream(stream):
        return hsi.scene_moments(c["cube"], c["H"], c["W"], c["B"], dtype=c["dtype"], stream=stream)


def test_two_threads_score_like_one(hsi):
    cases = [_case(hsi, 512, 384, 113, 8, hsi.F32, 0x5EED1001),
             _case(hsi, 256, 640, 40, 4, hsi.F32, 0x5EED1002),
             _case(hsi, 384, 256, 113, 8, hsi.F16, 0x5EED1003),
             _case(hsi, 256, 256, 40, 8, hsi.F16, 0x5EED1004)]
    s0 = torch.cuda.Stream()
    want = [_score(hsi, c, s0) for c in cases]
    want_m = [_moments(hsi, c, s0) for c in cases[:2]]
    torch.cuda.synchronize()

    rounds = 20
    got = [[None] * len(cases) for _ in range(rounds)]
    got_m = [[None] * 2 for _ in range(rounds)]
    errors = []

    def worker(k):
        try:
            s = torch.cuda.Stream()
            for r in range(rounds):
                # thread 0 takes cases 0 and 2, thread 1 cases 1 and 3: different
                # band counts on the same kernels at the same time
                for i in (k, k + 2):
                    got[r][i] = _score(hsi, cases[i], s)
                got_m[r][k] = _moments(hsi, cases[k], s)
            s.synchronize()
        except Exception as e:  # reported in the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    assert not errors, errors
    for r in range(rounds):
        for i, c in enumerate(cases):
            for key in want[i]:
                assert torch.equal(got[r][i][key], want[i][key]), f"round {r}, case {i}: {key} differs"
        for k in range(2):
            assert torch.equal(got_m[r][k], want_m[k]), f"round {r}: moments of case {k} differ"
