"""The oracle's two loop backends agree: NumPy/SciPy FP64 against
torch.float64 on the CPU (the same statements; only the array library
differs).  The torch backend on CUDA is the fast oracle of the full-size GPU
parity tests.  Bound: relative L2 <= 1e-12 on every output."""
import numpy as np
import pytest

from cases import make_case

CASES = ["2d_hetero_abs_nl", "2d_stokes_dirichlet", "2d_nocorr_multi", "2d_u_additive", "2d_u_dirichlet",
         "2d_pml_outside", "3d_p0_u", "3d_multi_signal_additive", "2d_time_reversal", "3d_time_reversal_abs",
         "2d_intensity", "2d_cart_linear", "3d_layered_full_volume", "2d_full_mask_odd"]


def _grid(mod, shape, dx, Nt, dt):
    args = []
    for s in shape:
        args += [s, dx]
    g = mod.KWaveGrid(*args)
    g.setTime(Nt, dt)
    return g


def _rel(a, b):
    d = np.linalg.norm(np.ravel(b))
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / (d if d > 0 else 1.0))


@pytest.mark.parametrize("name", CASES)
def test_torch_backend_matches_numpy(name):
    from oracle import kspace as ks
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    a = ks.kspace_first_order(_grid(ks, shape, dx, Nt, dt), med, src, sen, **opts)
    b = ks.kspace_first_order(_grid(ks, shape, dx, Nt, dt), med, src, sen, Device="cpu", **opts)
    if isinstance(a, dict):
        assert set(a) == set(b)
        for k in a:
            assert b[k].shape == a[k].shape, k
            assert _rel(b[k], a[k]) <= 1e-12, (name, k, _rel(b[k], a[k]))
    else:
        assert b.shape == a.shape
        assert _rel(b, a) <= 1e-12, (name, _rel(b, a))
