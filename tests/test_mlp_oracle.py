"""The surrogate network's CPU oracle (oracle/mlp.py) pinned by finite differences, and the
library's MLP entry points exported (no GPU needed)."""
import numpy as np
import pytest

from oracle import mlp as M


def small_params(n_in, h, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.7, n_in * h + h + h * h + h + h + 1)


@pytest.mark.parametrize("n_in,h", [(3, 5), (12, 8)])
def test_parameter_gradients_match_finite_differences(n_in, h):
    rng = np.random.default_rng(n_in + h)
    p = small_params(n_in, h, 1)
    x = rng.uniform(-1, 1, (7, n_in))
    t = rng.normal(0, 1, 7)
    loss, g, gx = M.gradients(p, x, t, n_in, h)
    eps = 1e-6
    for i in rng.choice(len(p), 25, replace=False):
        dp = np.zeros_like(p)
        dp[i] = eps
        fd = (M.gradients(p + dp, x, t, n_in, h)[0] - M.gradients(p - dp, x, t, n_in, h)[0]) / (2 * eps)
        assert abs(fd - g[i]) < 1e-6 * max(1.0, abs(fd))
    for b in range(3):
        for k in range(n_in):
            dx = np.zeros_like(x)
            dx[b, k] = eps
            fd = (M.gradients(p, x + dx, t, n_in, h)[0] - M.gradients(p, x - dx, t, n_in, h)[0]) / (2 * eps)
            assert abs(fd - gx[b, k]) < 1e-6 * max(1.0, abs(fd))


def test_input_gradient_matches_finite_differences():
    n_in, h = 4, 6
    rng = np.random.default_rng(3)
    p = small_params(n_in, h, 2)
    x = rng.uniform(-1, 1, (5, n_in))
    g = M.input_gradient(p, x, n_in, h)
    eps = 1e-6
    for k in range(n_in):
        dx = np.zeros_like(x)
        dx[:, k] = eps
        fd = (M.forward(p, x + dx, n_in, h)[0] - M.forward(p, x - dx, n_in, h)[0]) / (2 * eps)
        assert np.abs(fd - g[:, k]).max() < 1e-6


def test_gelu_and_adam_formulas():
    z = np.linspace(-4, 4, 9)
    assert np.allclose(M.gelu(z), z * 0.5 * (1 + np.array([__import__("math").erf(v / np.sqrt(2)) for v in z])))
    p, m, v = M.adam_step(np.ones(3), np.array([1.0, -2.0, 0.0]), np.zeros(3), np.zeros(3), 1, 0.1)
    assert np.allclose(p, [0.9, 1.1, 1.0], atol=1e-6)   # first step moves by lr * sign(g)


def test_init_is_deterministic_and_bounded():
    a = M.init_params(12, 16, 7)
    b = M.init_params(12, 16, 7)
    assert np.array_equal(a, b) and a.dtype == np.float32
    W1 = a[:12 * 16]
    assert np.abs(W1).max() <= np.sqrt(6 / 12) and np.abs(W1).max() > 0.5 * np.sqrt(6 / 12)


def test_mlp_entry_points_exported():
    import ctypes
    import test_abi
    from orkan_b200.build import library_path
    decl = test_abi.declared_functions()
    names = {"orkan_mlp_" + f for f in ("create", "destroy", "param_count", "get_params", "set_params", "forward",
                                        "gradients", "train", "ascend", "launch_count")}
    assert names <= decl
    assert names <= test_abi.exported(library_path(5))
    lib = ctypes.CDLL(library_path(5))
    lib.orkan_mlp_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                     ctypes.c_ulonglong]
    h = ctypes.c_void_p()
    assert lib.orkan_mlp_create(ctypes.byref(h), 0, 16, 8, 1) == 1      # rejected before touching a device
    assert lib.orkan_mlp_create(ctypes.byref(h), 4, 16, 0, 1) == 1
