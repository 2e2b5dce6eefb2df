"""CUDA-graph capture of device-pointer runs: a replay solves the current contents
of the captured buffers exactly as a direct run does (bit for bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_replay_matches_direct_runs():
    import torch
    from modisp_b200 import _native, workloads
    dev = torch.device("cuda", 0)
    periods = np.geomspace(0.5, 50., 30)
    first = workloads.crustal_batch(64, workloads.SEED + 21)
    second = workloads.crustal_batch(64, workloads.SEED + 22)
    L = max(first["thickness"].shape[1], second["thickness"].shape[1])

    def pad(batch):
        out = {}
        for k, v in batch.items():
            extra = L - v.shape[1]
            if k == "thickness":
                out[k] = np.concatenate([v[:, :-1], np.zeros((v.shape[0], extra)), v[:, -1:]], axis=1)
            else:
                out[k] = np.concatenate([v[:, :-1], np.repeat(v[:, -1:], extra, 1), v[:, -1:]], axis=1)
        return out

    first, second = pad(first), pad(second)
    B, T = 64, periods.size
    o = _native.default_options()
    o.single_precision = 1
    o.group_velocity = 1
    eng = _native.Engine(0, B, L, T, 5, o)
    try:
        x = {k: torch.tensor(first[k], device=dev) for k in ("thickness", "vp", "vs", "rho")}
        per = torch.tensor(periods, device=dev)
        vel = [torch.empty((B, 5, T), dtype=torch.float64, device=dev) for _ in range(2)]
        grp = [torch.empty_like(v) for v in vel]
        i32 = [[torch.empty(s, dtype=torch.int32, device=dev) for s in ((B, T), (B, T), (B, T), (B, 5, T))]
               for _ in range(2)]

        def runs(stream):
            for wave in (0, 1):
                fl, lv, ct, gf = i32[wave]
                eng.run_device(x["thickness"].data_ptr(), x["vp"].data_ptr(), x["vs"].data_ptr(), x["rho"].data_ptr(),
                               B, per.data_ptr(), 0, 1e-10, 1., wave, vel[wave].data_ptr(), fl.data_ptr(),
                               lv.data_ptr(), ct.data_ptr(), grp[wave].data_ptr(), gf.data_ptr(), stream=stream)

        torch.cuda.synchronize()
        eng.graph_begin()
        runs(None)  # recorded, not executed
        eng.graph_end()
        for batch in (first, second, first):
            for k in x:
                x[k].copy_(torch.tensor(batch[k], device=dev))
            torch.cuda.synchronize()
            eng.graph_launch()
            torch.cuda.synchronize()
            replay = [(v.cpu().numpy().copy(), g.cpu().numpy().copy(), i32[w][2].cpu().numpy().copy())
                      for w, (v, g) in enumerate(zip(vel, grp))]
            for wave in (0, 1):
                direct = eng.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, 1e-10, 1.,
                                 wave, group=True)
                np.testing.assert_array_equal(replay[wave][0].view(np.uint64), direct["velocity"].view(np.uint64))
                np.testing.assert_array_equal(replay[wave][1].view(np.uint64), direct["group_velocity"].view(np.uint64))
                np.testing.assert_array_equal(replay[wave][2], direct["counts"])
    finally:
        eng.close()


def test_graph_calls_are_checked():
    from modisp_b200 import _native
    o = _native.default_options()
    eng = _native.Engine(0, 4, 3, 2, 2, o)
    try:
        with pytest.raises(RuntimeError, match="no captured graph"):
            eng.graph_launch()
        with pytest.raises(RuntimeError, match="no graph capture is open"):
            eng.graph_end()
    finally:
        eng.close()


def test_autotuner_on_a_sample(tmp_path, monkeypatch):
    """Every launch shape returns the same roots; the tuner returns one of them."""
    from modisp_b200 import autotune, workloads
    monkeypatch.setenv("MODISP_B200_CACHE", str(tmp_path))
    sample = workloads.crustal_batch(300, workloads.SEED + 41)
    shape = autotune.autotune(sample, np.geomspace(0.5, 50., 30), 5, 0, True)
    assert shape in autotune.CANDIDATES
    assert autotune.cache_path().exists()


def test_chunked_host_run_equals_device_run():
    """The host path solves large batches in pipelined chunks; the results are those
    of one device-pointer run over the whole batch (bit for bit), stats summed."""
    import torch
    from modisp_b200 import _native, workloads
    batch = workloads.crustal_batch(70000, workloads.SEED + 51, nmin=3, nmax=6)
    periods = np.geomspace(1., 40., 6)
    B, L = batch["thickness"].shape
    o = _native.default_options()
    o.single_precision = 1
    o.group_velocity = 1
    eng = _native.Engine(0, B, L, periods.size, 3, o)
    try:
        host = eng.run(batch["thickness"], batch["vp"], batch["vs"], batch["rho"], periods, None, 1e-10, 1., 0,
                       group=True)
        dev = torch.device("cuda", 0)
        x = {k: torch.tensor(batch[k], device=dev) for k in ("thickness", "vp", "vs", "rho")}
        per = torch.tensor(periods, device=dev)
        vel = torch.empty((B, 3, periods.size), dtype=torch.float64, device=dev)
        grp = torch.empty_like(vel)
        gfl = torch.empty((B, 3, periods.size), dtype=torch.int32, device=dev)
        fl, lv, ct = (torch.empty((B, periods.size), dtype=torch.int32, device=dev) for _ in range(3))
        st = torch.zeros(_native.STAT_COUNT, dtype=torch.int64, device=dev)
        eng.run_device(x["thickness"].data_ptr(), x["vp"].data_ptr(), x["vs"].data_ptr(), x["rho"].data_ptr(), B,
                       per.data_ptr(), 0, 1e-10, 1., 0, vel.data_ptr(), fl.data_ptr(), lv.data_ptr(), ct.data_ptr(),
                       grp.data_ptr(), gfl.data_ptr(), stats=st.data_ptr(),
                       stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
    finally:
        eng.close()
    np.testing.assert_array_equal(host["velocity"].view(np.uint64), vel.cpu().numpy().view(np.uint64))
    np.testing.assert_array_equal(host["group_velocity"].view(np.uint64), grp.cpu().numpy().view(np.uint64))
    np.testing.assert_array_equal(host["counts"], ct.cpu().numpy())
    np.testing.assert_array_equal(host["flags"], fl.cpu().numpy().astype(np.uint32))
    stats = st.cpu().numpy()
    assert host["stats"]["roots"] == stats[10] == int(np.isfinite(host["velocity"]).sum())
    assert host["stats"]["traces"] == stats[11] == B * periods.size
