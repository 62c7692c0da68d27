"""Adjoint gradient (xfd_adjoint_run behind Simulation::dftPowerObjective) and
saved states (xfd_checkpoint_*).

The objective is J = sum_p |DFT_f Ez(p)|^2 over a patch above a slab holding
a block of per-voxel permittivities; dJ/deps_r per voxel from the discrete
adjoint is checked against central finite differences (h = 1e-4) of J from
plain forward runs -- on the GPU in FP64 (the discrete adjoint is exact, so
they agree to FD truncation), on the oracle (the CPU restatement of the
reference's FP64 path), and for the FP32 form against FP64 differences at
the 1e-3 bar."""
import numpy as np
import pytest

from oracle.reference_model import RefSimulation
from tests.scenes import voxels_objective, voxels_small
from xfdtd_core_b200.host import SceneRun

pytestmark = pytest.mark.gpu
STEPS = 300
H = 1e-4


def _scene(eps=None, steps=STEPS):
    sc = voxels_small(steps=steps)
    vox = [o for o in sc.objects if hasattr(o, "voxel_index")][0]
    if eps is not None:
        vox.eps_r = np.array(eps, dtype=np.float64)
    return sc, vox


def _J_gpu(eps, precision=0):
    sc, _ = _scene(eps)
    ob = voxels_objective()
    r = SceneRun(sc, precision=precision)
    J = r.dft_objective(STEPS, ob["field"], ob["box_s"], ob["box_e"], ob["freq"])
    r.close()
    return J


def _grad_gpu(precision=0, interval=64):
    sc, vox = _scene()
    ob = voxels_objective()
    r = SceneRun(sc, precision=precision)
    J, g = r.dft_objective(STEPS, ob["field"], ob["box_s"], ob["box_e"], ob["freq"], grad=True,
                           checkpoint_interval=interval)
    r.close()
    return J, g, np.array(vox.eps_r)


def _J_oracle(eps):
    sc, _ = _scene(eps)
    ob = voxels_objective()
    orc = RefSimulation(sc)
    s, e = ob["box_s"], ob["box_e"]
    rec = []
    for _ in range(STEPS):
        orc.run(1)
        rec.append(orc.e[ob["field"]][s[0]:e[0], s[1]:e[1], s[2]:e[2]].ravel().copy())
    rec = np.array(rec)
    t = (np.arange(STEPS) + 1) * orc.dt
    F = orc.dt * (rec * np.exp(-2j * np.pi * ob["freq"] * t)[:, None]).sum(axis=0)
    return float(np.sum(np.abs(F) ** 2))


def _sample(shape, k, seed=3):
    rng = np.random.default_rng(seed)
    flat = rng.choice(int(np.prod(shape)), size=k, replace=False)
    return [np.unravel_index(q, shape) for q in flat]


def _fd(eps, idx, J):
    ep, em = eps.copy(), eps.copy()
    ep[idx] += H
    em[idx] -= H
    return (J(ep) - J(em)) / (2 * H)


def test_objective_matches_oracle():
    J, _, eps = _grad_gpu()
    Jf = _J_gpu(eps)
    Jo = _J_oracle(eps)
    assert J > 0
    assert abs(Jf - J) <= 1e-13 * J
    assert abs(Jo - J) <= 1e-12 * J, (J, Jo)


def test_adjoint_fp64_matches_central_differences():
    J, g, eps = _grad_gpu()
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    idx = _sample(eps.shape, 6)
    fd = np.array([_fd(eps, q, _J_gpu) for q in idx])
    ad = np.array([g[q] for q in idx])
    err = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    assert err <= 1e-6, (err, ad, fd)


def test_adjoint_matches_oracle_differences():
    _, g, eps = _grad_gpu()
    idx = _sample(eps.shape, 2, seed=9)
    fd = np.array([_fd(eps, q, _J_oracle) for q in idx])
    ad = np.array([g[q] for q in idx])
    err = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    assert err <= 1e-6, (err, ad, fd)


def test_adjoint_fp32_within_1e3_of_fp64_differences():
    J32, g32, eps = _grad_gpu(precision=1)
    idx = _sample(eps.shape, 6, seed=4)
    fd = np.array([_fd(eps, q, _J_gpu) for q in idx])
    ad = np.array([g32[q] for q in idx])
    err = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    assert err <= 1e-3, (err, ad, fd)


def test_checkpoint_interval_leaves_gradient_unchanged():
    J1, g1, _ = _grad_gpu(interval=7)
    J2, g2, _ = _grad_gpu(interval=STEPS)
    assert J1 == J2
    assert np.linalg.norm(g1 - g2) <= 1e-12 * np.linalg.norm(g2)


def test_adjoint_leaves_forward_state():
    """After the adjoint the engine holds the state of a plain forward run."""
    sc, _ = _scene()
    ob = voxels_objective()
    a = SceneRun(sc)
    a.dft_objective(STEPS, ob["field"], ob["box_s"], ob["box_e"], ob["freq"], grad=True,
                    checkpoint_interval=50)
    a.finish()
    b = SceneRun(_scene()[0])
    b.run()
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_checkpoint_save_load_roundtrip(precision):
    from xfdtd_core_b200 import engine as E
    import ctypes
    sc, _ = _scene(steps=60)
    r = SceneRun(sc, precision=precision)
    L = E.load()
    h = ctypes.c_void_p(r.engine_handle())
    assert L.xfd_checkpoint_step(h, 0) == -1
    r.advance(20)
    assert L.xfd_checkpoint_save(h, 3) == 0
    assert L.xfd_checkpoint_step(h, 3) == 20
    r.advance(20)
    r.finish()
    first = r.fields()
    assert L.xfd_checkpoint_load(h, 3) == 0
    assert L.xfd_current_step(h) == 20
    r.advance(20)
    r.finish()
    for x, y in zip(first, r.fields()):
        assert np.array_equal(x, y)
    assert L.xfd_checkpoint_load(h, 7) != 0
    assert L.xfd_checkpoint_drop(h, 3) == 0
    assert L.xfd_checkpoint_step(h, 3) == -1
    r.close()


def test_checkpoint_load_refused_with_nf2ff():
    """An engine with an NF2FF surface saves states but refuses to load them
    (its running DFT sums cover the steps already taken), and the refused
    load leaves the run untouched: the NF2FF currents after 64 + 40 steps
    (one batch boundary crossed after the save) equal those of a run that
    never tried to load."""
    from xfdtd_core_b200 import engine as E
    import ctypes
    from tests.scenes import dispersive_small
    runs = []
    for try_load in (False, True):
        r = SceneRun(dispersive_small(steps=120), precision=0)
        L = E.load()
        h = ctypes.c_void_p(r.engine_handle())
        r.advance(40)
        assert L.xfd_checkpoint_save(h, 0) == 0
        r.advance(64)
        if try_load:
            st = L.xfd_checkpoint_load(h, 0)
            assert st == 3  # XFD_ERR_UNSUPPORTED
            assert b"NF2FF" in L.xfd_last_error(h)
            assert L.xfd_current_step(h) == 104
        r.finish()
        runs.append((r.fields(), r.nf2ff()))
        r.close()
    for x, y in zip(runs[0][0], runs[1][0]):
        assert np.array_equal(x, y)
    assert np.array_equal(runs[0][1], runs[1][1])


class DftPower:
    """torch.autograd.Function over the adjoint (test harness only): J(eps_r)
    forward, dJ/deps_r from the discrete adjoint on backward."""

    @staticmethod
    def make():
        import torch

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, eps):
                sc, _ = _scene(eps.detach().cpu().numpy())
                ob = voxels_objective()
                r = SceneRun(sc)
                J, g = r.dft_objective(STEPS, ob["field"], ob["box_s"], ob["box_e"], ob["freq"],
                                       grad=True, checkpoint_interval=64)
                r.close()
                ctx.save_for_backward(torch.from_numpy(g))
                return torch.tensor(J, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gJ):
                (g,) = ctx.saved_tensors
                return gJ * g

        return _F


def test_torch_autograd_shim():
    import torch
    _, vox = _scene()
    eps = torch.tensor(np.array(vox.eps_r), dtype=torch.float64, requires_grad=True)
    J = DftPower.make().apply(eps)
    (3.0 * J).backward()
    idx = _sample(tuple(eps.shape), 2, seed=21)
    e0 = np.array(vox.eps_r)
    for q in idx:
        fd = _fd(e0, q, _J_gpu)
        assert abs(eps.grad[q].item() - 3.0 * fd) <= 1e-6 * abs(3.0 * fd)
