"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle.

Tolerance: relative L2 error <= 1e-4 on every recorded output (the bound the
FP32 loop must meet against an FP64 restatement of the reference solver).
"""
import numpy as np
import pytest

from cases import CASES, make_case

TOL = 1e-4


def _grid(mod, shape, dx, Nt, dt):
    args = []
    for s in shape:
        args += [s, dx]
    g = (mod.kWaveGrid if hasattr(mod, "kWaveGrid") else mod.KWaveGrid)(*args)
    g.setTime(Nt, dt)
    return g


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_parity(name):
    import kwave_b200 as kw
    from oracle import kspace as oracle
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    run = kw.kspaceFirstOrder2D if dim == 2 else kw.kspaceFirstOrder3D
    gpu = run(_grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)
    ref = oracle.kspace_first_order(_grid(oracle, shape, dx, Nt, dt), med, src, sen, **opts)
    if isinstance(ref, dict):
        assert set(gpu) == set(ref), (sorted(gpu), sorted(ref))
        for k in ref:
            assert gpu[k].shape == ref[k].shape, k
            e = _rel(gpu[k], ref[k])
            assert e <= TOL, "%s: %s rel-L2 %.3e" % (name, k, e)
    else:
        assert gpu.shape == ref.shape
        e = _rel(gpu, ref)
        assert e <= TOL, "%s rel-L2 %.3e" % (name, e)
