"""The learned warm start's neural operator on the GPU: forward loss and
every parameter gradient (tcgen05 GEMMs + support kernels) against a CPU
FP32 autograd restatement (tests/fno_reference.py), and a few Adam steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model_and_batch(seed=0, B=2):
    import torch
    from pot3d_b200 import host
    from pot3d_b200.fno import FNO, grid_from_mesh
    mesh = host.make_mesh(8, 22, 26)
    g = grid_from_mesh(mesh)
    model = FNO(g, seed=seed)
    br0s = []
    for b in range(B):
        tn, pn, fi = host.synthetic_br(10 + b, 6, 2, 22, 26)
        br0s.append(host.br0_from_map(mesh, tn, pn, fi))
    x, sig = model.inputs(br0s)
    rng = np.random.default_rng(seed)
    target = torch.tensor(rng.standard_normal((B, g.nph, g.nth, g.R)), dtype=torch.float32, device="cuda")
    return model, x, target


def test_fno_gradients_match_cpu_autograd(cuda):
    import torch
    from fno_reference import reference_loss_and_grads
    model, x, target = _model_and_batch()
    loss, grad_out = model.loss_and_grad(x, target)
    grads = model.backward(grad_out)
    torch.cuda.synchronize()
    from pot3d_b200.tc import check_errors
    check_errors(cuda)
    l_gpu = float(loss.mean().item())
    l_ref, g_ref = reference_loss_and_grads(model, x, target)
    assert abs(l_gpu - l_ref) <= 2e-2 * abs(l_ref), (l_gpu, l_ref)
    for k, gr in g_ref.items():
        gg = grads[k].detach().cpu().float().view(gr.shape)
        err = torch.linalg.norm(gg - gr) / max(torch.linalg.norm(gr), 1e-20)
        assert err <= 6e-2, (k, float(err))


def test_fno_adam_steps_reduce_loss(cuda):
    model, x, target = _model_and_batch(seed=1)
    losses = []
    for _ in range(30):
        loss, grad_out = model.loss_and_grad(x, target)
        losses.append(float(loss.mean().item()))
        model.adam_step(model.backward(grad_out), lr=3e-3)
    assert losses[-1] < 0.8 * losses[0], losses


def test_fno_inference_equals_training_forward(cuda):
    """The inference path (no activation cache) computes the same output as
    the training path of the same weights, layer by layer."""
    import torch
    model, x, _ = _model_and_batch(seed=2)
    for l in range(model.nl):  # distinct spectral weights per layer
        model.p[f"R{l}"].mul_(1.0 + 0.5 * l)
        model.pb[f"R{l}"] = model.p[f"R{l}"].to(torch.bfloat16).contiguous()
    a = model.forward(x, keep=True).clone()
    b = model.forward(x, keep=False)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_fno_save_load_roundtrip(cuda, tmp_path):
    """A saved operator reloads with the BF16 weights inference uses and
    predicts the same guess; a model for another grid is rejected."""
    import torch
    from pot3d_b200 import host
    from pot3d_b200.fno import FNO, grid_from_mesh
    mesh = host.make_mesh(20, 21, 33)
    g = grid_from_mesh(mesh)
    m = FNO(g, seed=3)
    tn, pn, fi = host.synthetic_br(4, 8, 2, 21, 33)
    x, sig = m.inputs([host.br0_from_map(mesh, tn, pn, fi)])
    p0 = m.predict(x, sig)
    path = str(tmp_path / "m.npz")
    m.save(path)
    m2 = FNO.load(path, g)
    assert torch.equal(m2.predict(x, sig), p0)
    with pytest.raises(ValueError):
        FNO.load(path, grid_from_mesh(host.make_mesh(20, 21, 35)))


def test_predict_is_the_scaled_cropped_output(cuda):
    """The guess kernel writes sigma * output[..., :R] in the solver's packed
    layout, into a caller's buffer when given."""
    import torch
    from pot3d_b200 import host
    from pot3d_b200.fno import FNO, grid_from_mesh
    mesh = host.make_mesh(20, 21, 33)
    g = grid_from_mesh(mesh)
    m = FNO(g, seed=5)
    maps = []
    for sd in (1, 2):
        tn, pn, fi = host.synthetic_br(sd, 8, 2, 21, 33)
        maps.append(host.br0_from_map(mesh, tn, pn, fi))
    x, sig = m.inputs(maps)
    y = m.forward(x).view(2, g.nph, g.nth, -1)[..., :g.R].double()
    ref = (y * torch.tensor(sig, device="cuda").view(2, 1, 1, 1)).reshape(2, -1)
    out = torch.full((2, g.nph * g.nth * g.R), -1.0, dtype=torch.float64, device="cuda")
    got = m.predict(x, sig, out=out)
    assert got.data_ptr() == out.data_ptr()
    assert torch.equal(out, ref)
    with pytest.raises(ValueError):
        m.predict(x, sig, out=torch.empty(5, dtype=torch.float64, device="cuda"))
