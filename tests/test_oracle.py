"""The FP64 oracle pinned against the reference's own tests (CPU only).

Runtime/tests/test_runtime.m holds the only known answers for this path:
exact NCG/projection scalars, the identity filter, FD-vs-adjoint gradient,
loss-only equality and batch invariance.  The golden fixture
tests/golden/reference_kats.json restates those literals; the block-LU
restatement is cross-checked against the sparse LU.
"""
import json
import os

import numpy as np
import pytest

from oracle import helmholtz_fp64 as o

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)


def test_ncg_direction_kats():
    k = kats()["ncg_direction"]
    for case in k:
        d, beta, gz = o.ncg_direction(np.array(case["g"]), np.array(case["z"]), np.array(case["prev_z"]),
                                      case["prev_gz"], np.array(case["previous_direction"]), case["same_frequency"])
        assert abs(beta - case["beta"]) < 1e-14
        if "gz" in case:
            assert gz == case["gz"]
        if "direction" in case:
            assert np.array_equal(d, np.array(case["direction"]))
        assert float(np.sum(np.array(case["g"]) * d)) < 0


def test_projection_kat():
    k = kats()["projection"]
    mask = np.ones((31, 31), bool)
    mask[[*range(5), *range(26, 31)], :] = False
    mask[:, [*range(5), *range(26, 31)]] = False
    init = np.full((31, 31), k["initial"])
    out = o.project_slowness_update(init, -np.ones((31, 31)), k["alpha"], k["max_update_mps"], k["bounds_mps"],
                                    k["step_damping"], mask)
    assert np.all(out[mask] == k["projected"]) and np.array_equal(out[~mask], init[~mask])


def test_ringing_filter_identity_and_lowpass(ref_fixture):
    x = np.arange(-15, 16) * 1e-3
    c = ref_fixture["c_true"]
    assert o.ringing_removal_filt(x, x, c, 1500, 1e5, 0, 4) is c
    filt = o.ringing_removal_filt(x, x, c, 1500, 1e5, .5, 4)
    assert np.all(np.isfinite(filt)) and np.linalg.norm(filt - c) > 0


def test_masked_filtered_direction_descends(ref_fixture):
    """test_runtime.m:170-178: exterior gradient cannot leak into z."""
    mask = ref_fixture["mask"]
    x = np.arange(-15, 16) * 1e-3
    g = np.ones(mask.shape)
    g[~mask] = -1e10
    roi, z = o.roi_gradient(g, mask, x, x, 1500, 1e5, .5, 4)
    g[~mask] = 1e20
    _, z2 = o.roi_gradient(g, mask, x, x, 1500, 1e5, .5, 4)
    assert np.array_equal(z, z2) and np.all(z[~mask] == 0)
    assert np.sum(roi * -z) < 0


def test_linearized_step_length_rules():
    assert o.linearized_step_length(-2.0, 4.0) == 0.5
    assert o.linearized_step_length(3.0, 4.0) == 0.0
    assert o.linearized_step_length(0.0, 0.0) == 0.0
    with pytest.raises(o.WustError):
        o.linearized_step_length(1.0, 0.0)
    with pytest.raises(o.WustError):
        o.linearized_step_length(np.nan, 1.0)


def test_fd_gradient_loss_only_and_batch_invariance(ref_fixture):
    fx = ref_fixture
    init, obs, cfg, direction = fx["initial"], fx["obs"], fx["cfg"], fx["direction"]
    loss, grad, _ = o.wust_oracle(init, obs, 0, cfg)
    loss_only, _, _ = o.wust_oracle(init, obs, 0, cfg, need_gradient=False)
    assert abs(loss_only - loss) <= 1e-6 * loss
    step = 1e-3
    lp, _, _ = o.wust_oracle(1 / (1 / init + step * direction), obs, 0, cfg, need_gradient=False)
    lm, _, _ = o.wust_oracle(1 / (1 / init - step * direction), obs, 0, cfg, need_gradient=False)
    fd = (lp - lm) / (2 * step)
    adj = np.sum(grad * direction)
    assert abs(fd - adj) / max(abs(fd), abs(adj)) < 1e-4
    cfg3 = o.OracleConfig(pml_m=.004, source_batch_size=3)
    l3, g3, _ = o.wust_oracle(init, obs, 0, cfg3)
    assert abs(l3 - loss) / loss < 1e-4
    assert np.linalg.norm(g3 - grad) / np.linalg.norm(grad) < 1e-4


def test_ldr9_derivative(ref_fixture):
    """kwave-ldr9 gradient check (test_runtime.m:123-126)."""
    fx = ref_fixture
    cfg = o.OracleConfig(pml_m=.004, source_batch_size=2, wavenumber="kwave-ldr9",
                         dispersion=dict(time_step_s=2e-8, reference_speed_mps=1700))
    init, obs, direction = fx["initial"], fx["obs"], fx["direction"]
    _, grad, _ = o.wust_oracle(init, obs, 0, cfg)
    step = 1e-3
    lp, _, _ = o.wust_oracle(1 / (1 / init + step * direction), obs, 0, cfg, need_gradient=False)
    lm, _, _ = o.wust_oracle(1 / (1 / init - step * direction), obs, 0, cfg, need_gradient=False)
    fd = (lp - lm) / (2 * step)
    adj = np.sum(grad * direction)
    assert abs(fd - adj) / max(abs(fd), abs(adj)) < 1e-4


def test_block_lu_restatement_matches_sparse_lu(ref_fixture):
    fx = ref_fixture
    s = o.make_solver(fx["c_true"], fx["obs"], 0, fx["cfg"])
    invT = o.block_lu_factor(s.coefs)
    assert np.all(invT[[0, -1], :, :] == 0) and np.all(invT[:, [0, -1], :] == 0)
    src = o.point_sources(fx["tx"], range(3), 31, 31)
    ub = o.block_lu_apply(src, s.coefs, invT, False)
    us = s.solve(src)
    assert np.linalg.norm(ub - us) / np.linalg.norm(us) < 1e-8
    rng = np.random.default_rng(0)
    r = np.zeros((31, 31, 2), complex)
    r[1:-1, 1:-1] = rng.standard_normal((29, 29, 2)) + 1j * rng.standard_normal((29, 29, 2))
    ab = o.block_lu_apply(r, s.coefs, invT, True)
    a_sp = s.solve(r, adjoint=True)
    # interior and the x-border agree; the block solver leaves the y-border at zero
    assert np.linalg.norm((ab - a_sp)[1:-1, :]) / np.linalg.norm(a_sp) < 1e-8
    assert np.all(ab[[0, -1], :-1] == 0)


def test_mass_apply_adjointness(ref_fixture):
    """<M v, w> == <v, M^T w> with the ring handling of HelmholtzSolver.m:211-219."""
    rng = np.random.default_rng(0)
    d, e = 0.18, 0.07
    v = rng.standard_normal((12, 10)) + 1j * rng.standard_normal((12, 10))
    w = rng.standard_normal((12, 10)) + 1j * rng.standard_normal((12, 10))
    lhs = np.vdot(w, o.mass_apply(v, d, e, adjoint=False))
    rhs = np.vdot(o.mass_apply(w, d, e, adjoint=True), v)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_sparse_matrix_structure(ref_fixture):
    fx = ref_fixture
    s = o.make_solver(fx["c_true"], fx["obs"], 0, fx["cfg"], factor=False)
    H = s.H.tocsr()
    ny, nx = 31, 31
    for lin in (0, ny - 1, ny * (nx - 1), 5):          # Dirichlet rows are identity rows
        row = H.getrow(lin)
        assert row.nnz == 1 and row[0, lin] == 1
    assert H.getrow(ny * 5 + 5).nnz == 9
    assert H.nnz == (ny - 2) * (nx - 2) * 9 + (2 * ny + 2 * nx - 4)


def test_stencil_params_against_golden():
    k = kats()["stencil_opt_params"]
    b, d, e = o.stencil_opt_params(*k["args"])
    assert b == 5 / 6
    assert abs(d - k["d"]) < 1e-12 and abs(e - k["e"]) < 1e-12


def test_gauss_newton_product_is_the_curvature_form(ref_fixture):
    """The oracle's Gauss-Newton product Re(J^H J d): its quadratic form is
    directional_curvature.m's curvature and it is symmetric."""
    from oracle import helmholtz_fp64 as o
    fx = ref_fixture
    _, _, state = o.wust_oracle(fx["initial"], fx["obs"], 0, fx["cfg"], retain_state=True)
    mask = fx["obs"].mask[:, :, 0]
    d = fx["direction"]
    e = np.roll(d, 3, axis=1) * fx["mask"]
    hd, kappa = o.gauss_newton_product(state, d, fx["obs"].rx_index, mask)
    he, _ = o.gauss_newton_product(state, e, fx["obs"].rx_index, mask)
    k_ref = o.directional_curvature(state, d, fx["obs"].rx_index, mask)
    assert abs(kappa - k_ref) <= 1e-12 * k_ref
    assert abs(float(np.sum(d * hd)) - k_ref) <= 1e-9 * k_ref
    assert abs(float(np.sum(e * hd)) - float(np.sum(d * he))) <= 1e-9 * abs(float(np.sum(d * hd)))
