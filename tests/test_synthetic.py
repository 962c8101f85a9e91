"""CPU tests of the seeded synthetic snapshots (benchmark stand-ins)."""
import numpy as np

from fastimagingpipe_b200 import synthetic


def test_baseline_counts_of_the_benchmark_layouts():
    assert synthetic.baseline_vectors(np.zeros((128, 3))).shape[0] == 8128
    assert synthetic.baseline_vectors(np.zeros((512, 3))).shape[0] == 130816


def test_small_config_shapes_and_determinism():
    a = synthetic.config_small()
    b = synthetic.config_small()
    assert a.num_baselines == 8128 and a.image_size == 512 and a.unit_size == 16
    assert a.vis_re.shape == (3 * 8128,) and a.B.shape == (3 * 8128 * 2,) and a.V.shape == (27,)
    assert np.array_equal(a.vis_re, b.vis_re) and np.array_equal(a.B, b.B)
    c = synthetic.config_small(seed=2)
    assert not np.array_equal(a.vis_re, c.vis_re)


def test_plane_basis_is_orthonormal_and_B_is_the_projection():
    s = synthetic.config_tiny()
    lam = synthetic.C_LIGHT / s.frequency_hz
    for k in range(3):
        V = s.V[9 * k:9 * k + 9].reshape(3, 3).astype(np.float64)
        assert np.allclose(V @ V.T, np.eye(3), atol=1e-6)
        uvw = s.uvw_m[k].astype(np.float64) / lam
        B = s.B[k * s.num_baselines * 2:(k + 1) * s.num_baselines * 2].reshape(-1, 2)
        assert np.allclose(B, uvw @ V[:2].T, rtol=1e-5, atol=1e-2)
        # a coplanar array: the third axis carries (almost) nothing
        assert np.abs(uvw @ V[2]).max() < 1e-3 * np.abs(uvw).max()


def test_dense_core_layout():
    rng = np.random.default_rng(0)
    enu = synthetic.antenna_layout(512, 20000.0, rng, core_fraction=0.5, core_radius_m=1000.0)
    r = np.hypot(enu[:, 0], enu[:, 1])
    assert (r <= 1000.0).sum() >= 256 and r.max() <= 20000.0


def test_flagging_pads_with_zeros():
    s = synthetic.config_tiny(flag_fraction_max=0.3, seed=7)
    f = s.flags
    assert f is not None and f.any()
    nb = s.num_baselines
    for k in range(3):
        fl = f[k]
        assert np.all(s.vis_re[k * nb:(k + 1) * nb][fl] == 0)
        assert np.all(s.B[k * nb * 2:(k + 1) * nb * 2].reshape(-1, 2)[fl] == 0)
