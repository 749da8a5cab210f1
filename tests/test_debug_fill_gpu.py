"""Debug fill mode (environment SKGEMM_DEBUG_FILL=1): every scratch buffer of
the library starts as 0xFF bytes, at allocation and again at the start of
each call that uses it (an FP64 NaN, an int8 residue of -1). A kernel that
read scratch it had not written first would change its results. In that
mode the results must equal, bit for bit, those of a normal process: native
and Ozaki GEMM, SYRK, subspace pair, rotation and int8 GEMM (the cases of
tests/test_lanes_pair_gpu.py), a batched plan (fixed configuration) and the
nonlocal projector. The debug results come from a child process (the switch
is read once per process)."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import skgemm

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def plan_and_projector():
    """A batched plan with a fixed configuration and one projector apply."""
    from tests.test_batch_gpu import mixed_batch
    out = []
    items = mixed_batch(41)
    plan = skgemm.Plan([it.item() for it in items], tune=False)
    plan.run()
    plan.status()
    out += [it.dD.cpu().numpy() for it in items]
    plan.close()
    rng = np.random.default_rng(5)
    nd, nb, atoms, images, nrow, ncol = 4096, 64, 6, 2, 100, 8
    nproj = atoms * images
    proj = skgemm.NlocProjector(
        np.full(nproj, nrow), np.full(nproj, ncol), np.repeat(np.arange(1, atoms + 1), images),
        np.append(np.repeat(np.arange(atoms) * ncol, images), atoms * ncol),
        np.concatenate([rng.permutation(nd)[:nrow] for _ in range(nproj)]),
        rng.uniform(-1, 1, nproj * nrow * ncol), rng.uniform(-0.5, 0.5, nproj * ncol), nd)
    psi = torch.from_numpy(rng.uniform(-1, 1, nb * nd)).cuda()
    hpsi = torch.from_numpy(rng.uniform(-1, 1, nb * nd)).cuda()
    proj.apply(nb, 0.01, psi, hpsi, 32)
    skgemm.stream_status()
    proj.close()
    out.append(hpsi.cpu().numpy())
    return out


def all_results():
    from tests.test_lanes_pair_gpu import compute, _flat
    return (_flat(compute(skgemm.PREC_NATIVE)) + _flat(compute(skgemm.PREC_OZAKI_I8)) +
            plan_and_projector())


def test_debug_fill_leaves_results_unchanged(cuda, tmp_path):
    path = str(tmp_path / "debug_fill.npz")
    code = (f"import sys; sys.path[:0] = [{REPO!r}, {os.path.join(REPO, 'stream-k-gemm_b200')!r}]\n"
            "import numpy as np\n"
            "import skgemm\n"
            "from tests.test_debug_fill_gpu import all_results\n"
            "assert skgemm.debug_fill()\n"
            f"np.savez({path!r}, *all_results())\n")
    env = dict(os.environ, SKGEMM_DEBUG_FILL="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(path)
    assert not skgemm.debug_fill()
    got = all_results()
    assert len(got) == len(ref.files)
    for k, a in enumerate(got):
        b = ref[f"arr_{k}"]
        assert a.shape == b.shape, k
        # NaN-equal: outputs that a test leaves as NaN padding stay NaN in both
        assert np.array_equal(a, b, equal_nan=True), k
        assert np.isfinite(b).sum() == np.isfinite(a).sum(), k
