"""The reference arm of bench.py (``--impl reference``) on CPU.

It must time the same workload as the GPU arm (same mesh, clamp set,
pressure faces and ``config``), in the reference's own output form, without
importing the fea_b200 package or mapping its library into the process."""
import json
import os
import subprocess
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_workload_is_the_benchmark_mesh():
    import bench
    for n in (3, 8):
        X, el, clamp, end, faces = bench.workload(n)
        Xr, elr, clampr, facesr = bench.reference_workload(n)
        assert np.array_equal(Xr.numpy(), X) and np.array_equal(elr.numpy(), el)
        assert np.array_equal(clampr.numpy(), clamp) and np.array_equal(facesr.numpy(), faces)


def test_reference_form_coo_is_the_oracle_matrix():
    """The uncoalesced reduced COO of ``Model.stiffness_coo`` (the
    reference's assemble_Stiffness_Matrix form) sums to the oracle's
    coalesced CSR, chunked or not."""
    import bench
    from oracle import fea_oracle as O
    n = 4
    X, el, clamp, faces = bench.reference_workload(n)
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [O.PressureLoad(faces, 0.02)], [(clamp, (0, 1, 2))])
    gc = 1e-3 * torch.randn(int(m.free_mask().sum()), generator=torch.Generator().manual_seed(0),
                            dtype=torch.float64)
    R, (ip, ix, v) = m.assemble(gc)
    pat = [O.element_pattern(el)]
    for chunk in (7, 1 << 14):
        Rr, Ki, Kv = m.stiffness_coo(gc, pat, chunk=chunk)
        assert torch.allclose(Rr, R, rtol=0, atol=1e-15 * float(R.abs().max()))
        A = torch.sparse_coo_tensor(Ki, Kv, (R.shape[0], R.shape[0])).coalesce().to_sparse_csr()
        assert torch.equal(A.crow_indices(), ip) and torch.equal(A.col_indices(), ix)
        assert float((A.values() - v).abs().max()) <= 1e-14 * float(v.abs().max())
    ref = bench.ReferenceAssembly(n)                 # the config it reports: the coalesced system's sizes
    assert (ref.E, ref.N, ref.ndof, ref.nnz) == (el.shape[0], X.shape[0], R.shape[0], int(ip[-1]))


def test_reference_arm_maps_no_fea_b200():
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--n', '4', '--steps', '2', "
            "'--warmup', '1']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'mods': [m for m in sys.modules if m.startswith('fea_b200')], "
            "'so': 'libfea_b200' in maps}))")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    line, probe = json.loads(lines[-2]), json.loads(lines[-1])
    assert probe == {"mods": [], "so": False}
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    import bench
    X, el, clamp, end, faces = bench.workload(4)
    assert line["config"]["workload"] == "c3d8_4cube_jitter_neohookean_assembly"
    assert line["config"]["elements"] == el.shape[0] and line["config"]["nodes"] == X.shape[0]
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert abs(line["ms_per_step"] - el.shape[0] / (line["value"] * 1e9) * 1e3) <= 1e-9 * line["ms_per_step"]
