"""The differentiable form: the discrete adjoint of the step (reverse Boris
rotation, deposition adjoint as a gather, field-gather adjoint as a
scatter-add, transposed FDTD update), checkpointed and recomputed, against
central finite differences of the forward run.

Tolerances: FP64, 8 steps: 1e-6 relative (measured 2e-8 and below). FP64, 40
steps with 4 checkpoint segments: 1e-5 for psi0 and nb; the Ti/Te loss is
rough at that horizon (cell-crossing decisions of many particles flip), so its
finite-difference quotient itself changes by percents with the step, and the
check is 5e-2. FP32 forward vs FP64 forward adjoint: 1e-5 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BASE = dict(psi0=0.1, nb=0.2, ti_te=5.0)
KEYS = ("psi0", "nb", "ti_te")


def central_fd(eng, rel):
    out = []
    for k in KEYS:
        h = rel * BASE[k]
        p = dict(BASE)
        p[k] += h
        lp = eng.forward(**p)
        p = dict(BASE)
        p[k] -= h
        lm = eng.forward(**p)
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def test_adjoint_matches_finite_differences_fp64(gpu_lib):
    from pbpic_b200.autograd import DiffEngine
    with DiffEngine(32, 16, 8, nsteps=8, checkpoint_every=3, precision="fp64") as e:
        e.forward(**BASE)
        adj = np.array(e.backward())
        fd = central_fd(e, 1e-5)
    assert np.all(np.abs(adj - fd) <= 1e-6 * np.abs(fd)), (adj, fd)


def test_adjoint_over_checkpoint_segments_fp64(gpu_lib):
    from pbpic_b200.autograd import DiffEngine
    with DiffEngine(64, 32, 16, nsteps=40, checkpoint_every=10, precision="fp64") as e:
        e.forward(**BASE)
        adj = np.array(e.backward())
        fd = central_fd(e, 1e-6)
    rel = np.abs(adj - fd) / np.abs(fd)
    assert rel[0] <= 1e-5 and rel[1] <= 1e-5 and rel[2] <= 5e-2, (adj, fd, rel)


def test_fp32_forward_adjoint_matches_fp64(gpu_lib):
    from pbpic_b200.autograd import DiffEngine
    grads = {}
    for prec in ("fp64", "fp32"):
        with DiffEngine(32, 16, 8, nsteps=8, checkpoint_every=3, precision=prec) as e:
            e.forward(**BASE)
            grads[prec] = np.array(e.backward())
    assert np.all(np.abs(grads["fp32"] - grads["fp64"]) <= 1e-5 * np.abs(grads["fp64"]))


def test_autograd_function(gpu_lib):
    import torch

    from pbpic_b200.autograd import DiffEngine, HarrisLoss
    with DiffEngine(32, 16, 8, nsteps=6, checkpoint_every=4, precision="fp64") as e:
        params = torch.tensor([BASE[k] for k in KEYS], dtype=torch.float64, requires_grad=True)
        loss = HarrisLoss.apply(params, e)
        (2.0 * loss).backward()
        ref_loss = e.forward(**BASE)
        ref = np.array(e.backward())
    assert abs(loss.item() - ref_loss) <= 1e-12 * abs(ref_loss)
    assert np.allclose(params.grad.numpy(), 2.0 * ref, rtol=1e-9)


def test_backward_needs_forward(gpu_lib):
    import pbpic_b200
    from pbpic_b200.autograd import DiffEngine
    with DiffEngine(16, 8, 2, nsteps=2, checkpoint_every=1, precision="fp64") as e:
        with pytest.raises(pbpic_b200.PbpicError):
            e.backward()
