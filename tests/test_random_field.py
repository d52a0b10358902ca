"""Strength random field of the limit-load workload (CPU).

The lognormal cohesion / friction-angle fields are drawn by circulant embedding of the
exponential covariance exp(-r / l) on a regular grid and interpolated to the integration
points.  Checked here: the ensemble covariance against the exponential model, independence
of the two fields, determinism under a seed, exact trilinear interpolation of linear
functions, the lognormal transform's mean and coefficient of variation, and the per-point
material of a small random-field slope.
"""
import numpy as np

from slope_stability_octave_b200 import fem, problems


def test_embedding_reproduces_covariance():
    # the padded circulant embedding that the generator uses is non-negative definite, so
    # the coloured noise has exactly the exponential covariance at every lag on the grid
    corr, h = 2.0, 0.5
    _, _, info = fem.gaussian_fields_circulant([0, 0, 0], [10, 5, 5], h, corr, seed=0)
    lam = fem._embedding_eigenvalues(info["embedding"], [h] * 3, corr)
    assert lam.min() >= -1e-12 * lam.max()
    c = np.fft.ifftn(np.maximum(lam, 0.0)).real
    n = info["grid"]
    k = np.arange(n[0])
    assert np.allclose(c[k, 0, 0], np.exp(-k * h / corr), atol=1e-10)
    j = np.arange(n[1])
    assert np.allclose(c[2, j, 3], np.exp(-np.sqrt((2 * h) ** 2 + (j * h) ** 2 + (3 * h) ** 2) / corr), atol=1e-10)


def test_ensemble_covariance_is_exponential():
    corr, h = 2.0, 0.5
    lags = (1, 2, 4)
    acc = {k: [] for k in lags}
    second, cross = [], []
    for seed in range(30):
        F, _, info = fem.gaussian_fields_circulant([0, 0, 0], [20, 5, 5], h, corr, seed=seed)
        assert info["negative_eigen_share"] < 1e-6
        cross.append(np.mean(F[0] * F[1]))
        for f in F:
            second.append(np.mean(f * f))
            for k in lags:
                acc[k].append(np.mean(f[:-k] * f[k:]))
    assert abs(np.mean(second) - 1.0) < 0.06
    assert abs(np.mean(cross)) < 0.06
    for k in lags:
        assert abs(np.mean(acc[k]) - np.exp(-k * h / corr)) < 0.06, k


def test_fields_deterministic_under_seed():
    a, _, _ = fem.gaussian_fields_circulant([0, 0, 0], [6, 3, 2], 0.5, 2.0, seed=5)
    b, _, _ = fem.gaussian_fields_circulant([0, 0, 0], [6, 3, 2], 0.5, 2.0, seed=5)
    c, _, _ = fem.gaussian_fields_circulant([0, 0, 0], [6, 3, 2], 0.5, 2.0, seed=6)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


def test_trilinear_reproduces_linear_functions():
    axes = [np.linspace(0, 4, 9), np.linspace(-1, 2, 7), np.linspace(0, 1, 3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    field = 2 * X - 3 * Y + 0.5 * Z + 1
    pts = np.random.default_rng(0).uniform([0, -1, 0], [4, 2, 1], size=(1000, 3)).T
    got = fem.trilinear(field, axes, pts)
    assert np.allclose(got, 2 * pts[0] - 3 * pts[1] + 0.5 * pts[2] + 1, atol=1e-12)


def test_lognormal_moments():
    g = np.random.default_rng(1).standard_normal(2_000_000)
    x = fem.lognormal_from_gaussian(g, 10.0, 0.3)
    assert abs(x.mean() / 10.0 - 1) < 5e-3
    assert abs(x.std() / x.mean() / 0.3 - 1) < 1e-2
    assert x.min() > 0


def test_random_field_slope_materials():
    P = problems.slope_3d_random_field(1, dims=(15, 10, 15, 10, 10, 2), seed=3)
    m = P.mat
    n = P.weight.size
    for k in ("c0", "phi", "psi", "shear", "bulk", "lame", "gamma"):
        assert m[k].shape == (n,), k
    assert (m["c0"] > 0).all() and (m["phi"] > 0).all() and (m["phi"] < np.pi / 2).all()
    assert np.all(m["psi"] == 0)
    assert 5 < m["c0"].mean() < 15
    assert 30 < np.degrees(m["phi"]).mean() < 40
    # the same seed reproduces the material exactly
    Q = problems.slope_3d_random_field(1, dims=(15, 10, 15, 10, 10, 2), seed=3)
    assert np.array_equal(Q.mat["c0"], m["c0"]) and np.array_equal(Q.mat["phi"], m["phi"])
    # integration points lie inside their elements' bounding boxes
    X = fem.integration_points(P.mesh, P.hat).reshape(3, P.mesh.n_e, -1)
    V = P.mesh.coord[:, P.mesh.elem]
    assert np.all(X >= V.min(axis=1)[:, :, None] - 1e-12) and np.all(X <= V.max(axis=1)[:, :, None] + 1e-12)
