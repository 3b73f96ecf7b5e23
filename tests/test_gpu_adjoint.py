"""Per-element soil parameters and the discrete adjoint of the implicit Richards stepper.

* With the same parameters in every element, the element-wise assembly is the
  reference assembly (oracle, VG soil, per-element Ks factor): 1e-12 relative.
* The adjoint gradient of the sensor-misfit loss matches central finite
  differences (step 1e-6 in the log-parameters) to 1e-5 relative, with the
  forward solved tightly (Picard 1e-13, CG 1e-14) so the differences resolve.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import assembly as oasm, soil as osoil  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu
THR, THS = 0.102, 0.368


def cu(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")


def _problem(n=10, steps=8, seed=0, checkpoint_every=3, tight=True):
    from wspm_b200.adjoint import ElementParamRichards
    from wspm_b200.device import DeviceMesh
    pts, tri = mesh.structured_triangles(n, 1.0)
    bc = np.full(len(pts), np.nan)
    bc[np.abs(pts[:, 1] - 1.0) < 1e-12] = -0.1
    dm = DeviceMesh(pts, tri)
    kw = dict(picard_tol=1e-13, krylov_tol=1e-14, adjoint_tol=1e-13) if tight else {}
    prob = ElementParamRichards(dm, THR, THS, bc, 1e-3, steps, checkpoint_every=checkpoint_every, **kw)
    rng = np.random.default_rng(seed)
    base = np.log([0.0922, 3.35, 2.0])
    params = base[None, :] + 0.3 * rng.standard_normal((len(tri), 3))
    target_params = base[None, :] + 0.3 * rng.standard_normal((len(tri), 3))
    sensors = rng.choice(np.where(np.isnan(bc))[0], 6, replace=False)
    h0 = -np.ones(len(pts))
    target = prob.simulate_theta(cu(target_params).view(-1), cu(h0), sensors)
    return prob, params, sensors, h0, target


def test_uniform_element_parameters_reproduce_the_reference_assembly():
    from wspm_b200.adjoint import ElementParamRichards
    from wspm_b200.device import DeviceMesh
    pts, tri = mesh.structured_triangles(16, 1.0)
    rng = np.random.default_rng(1)
    h_m = -rng.uniform(0.05, 2.0, len(pts))
    h_n = h_m - 0.01
    phi = (3.35, THS, THR, 2.0, 0.5, 0.0922)
    bc = np.full(len(pts), np.nan)
    dm = DeviceMesh(pts, tri)
    prob = ElementParamRichards(dm, THR, THS, bc, 3e-3, 1)
    params = np.tile(np.log([1.0, 3.35, 2.0]), (len(tri), 1))
    Ks = np.full(len(tri), 0.0922)
    params[:, 0] = np.log(Ks)
    prob.assemble(cu(params).view(-1), cu(h_m), cu(h_n))
    C, K, th_m = osoil.van_genuchten_model(h_m, phi[:5] + (1.0,))
    th_n = osoil.van_genuchten_model(h_n, phi)[2]
    A_ref, b_ref = oasm.assemble_richards(tri, len(pts), pts, th_m, th_n, h_m, K, C, 3e-3, Ks_elem=Ks)
    A = dm.pattern.to_scipy(prob.vals.cpu().numpy())
    assert np.abs((A - A_ref).toarray()).max() <= 1e-12 * np.abs(A_ref.data).max()
    np.testing.assert_allclose(prob.rhs.cpu().numpy(), b_ref, rtol=0, atol=1e-12 * np.abs(b_ref).max())


def test_adjoint_gradient_matches_central_differences():
    prob, params, sensors, h0, target = _problem()
    p = cu(params).view(-1)
    loss = prob.forward(p, cu(h0), sensors, target)
    grad = prob.backward().cpu().numpy().ravel()
    assert float(loss) > 0 and np.all(np.isfinite(grad))
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(k, grad.size, 3), 3, replace=False) for k in range(3)])
    eps = 1e-6
    scale = np.abs(grad).max()
    for j in idx:
        pp, pm = p.clone(), p.clone()
        pp[j] += eps
        pm[j] -= eps
        fd = (float(prob.forward(pp, cu(h0), sensors, target)) - float(prob.forward(pm, cu(h0), sensors, target))) / (
            2 * eps)
        assert abs(grad[j] - fd) <= 1e-5 * max(abs(fd), 1e-3 * scale), (j, grad[j], fd)


def test_autograd_function_gives_the_adjoint_gradient():
    from wspm_b200.adjoint import ElementRichardsLoss
    prob, params, sensors, h0, target = _problem(steps=4, checkpoint_every=2)
    x = cu(params).requires_grad_(True)
    loss = ElementRichardsLoss.apply(x, prob, cu(h0), sensors, target)
    loss.backward()
    g1 = x.grad.clone()
    prob.forward(cu(params).view(-1), cu(h0), sensors, target)
    g2 = prob.backward()
    torch.testing.assert_close(g1, g2, rtol=0, atol=0)
