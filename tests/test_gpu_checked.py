"""The bounds-checked build (libhuntian_b200_checked.so, -DHT_CHECKED, loaded with
HT_CHECKED=1): the shell walk's record loads, cell-table ranges, profile rows and mask
writes and the peak scan's output cells are checked before each access, and a failed
check would record status 2 and skip the access instead of trapping.  On the small
periodic-box workload (128^3 box, 36-cell wrap, 30 filters: smoothing, peak scan with the
mask carried, pack and shell walk in PLAIN and BATCHED modes) run in a child process with
the checked build, every check passes (status 0) and every peak, result array and mask is
bit-identical to the normal build's."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
N, L, NBUFF, NF, RMIN, RMAX, SEED = 128, 250.0, 36, 30, 2.0, 40.0, 12345


def run_workload(ht):
    """Peaks, walk results (PLAIN and BATCHED) and the mask of the workload, as numpy."""
    from gpu_helpers import make_box_workload
    W = make_box_workload(ht, N, L, NBUFF, NF, RMIN, RMAX, SEED)
    npk = W["npk"]
    t = W["tile"]
    finder = W["finder"]
    finder.bind_fields(t["delta"], t["etax"], t["etay"], t["etaz"], t["eta2x"], t["eta2y"],
                       t["eta2z"], None)
    out = {f"peak_{c}": W["peaks"][c][:npk].cpu().numpy() for c in ("i", "j", "k", "delta")}
    nt = N + 2 * NBUFF
    for mode in ("plain", "batched"):
        mask = torch.zeros((nt,) * 3, dtype=torch.int8, device="cuda")
        res = finder.analyse(*W["args"], nbuff=NBUFF, mode=mode, mask=mask)
        torch.cuda.synchronize()
        for k, v in res.items():
            out[f"{mode}_{k}"] = v.cpu().numpy()
        out[f"{mode}_mask"] = mask.cpu().numpy()
    out["status"] = np.array([finder.device_status()])
    finder.close()
    return out


def _child(path):
    sys.path.insert(0, HERE)
    from conftest import load_package
    ht = load_package()
    assert ht._lib.LIB_PATH.endswith("libhuntian_b200_checked.so")
    np.savez(path, **run_workload(ht))


def test_checked_build_matches(ht, tmp_path):
    lib = os.path.join(os.path.dirname(HERE), "huntian.jl_b200", "libhuntian_b200_checked.so")
    assert os.path.exists(lib), "build it with: python huntian.jl_b200/build.py --checked"
    path = str(tmp_path / "checked.npz")
    env = dict(os.environ, HT_CHECKED="1")
    code = f"import sys; sys.path.insert(0, {HERE!r}); import test_gpu_checked as t; t._child({path!r})"
    subprocess.run([sys.executable, "-c", code], check=True, env=env, cwd=HERE, timeout=900)
    got = dict(np.load(path))
    want = run_workload(ht)
    assert int(got["status"][0]) == 0 and int(want["status"][0]) == 0
    assert set(got) == set(want)
    for k in want:
        assert np.array_equal(got[k], want[k], equal_nan=want[k].dtype.kind == "f"), k
