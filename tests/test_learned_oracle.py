"""The learned model's CPU oracle: its analytic root gradient against finite
differences (float64, no GPU)."""
import numpy as np

import learned_oracle as lo


def test_root_gradient_matches_finite_differences():
    import workloads
    for keys in (np.sort(lo.encode_f64(workloads.lognormal_np(4096, 3))),
                 np.sort(lo.encode_i32(workloads.zipf_i32_np(4096, seed=2)))):
        theta = lo.root_init_theta(keys) * (1.0 + 0.1 * np.sin(np.arange(lo.R)))
        _, g = lo.root_loss_grad(keys, theta)
        fd = lo.finite_difference(keys, theta)
        assert np.allclose(g, fd, rtol=1e-4, atol=1e-9)


def test_histogram_start_is_close_to_the_empirical_cdf():
    import workloads
    keys = np.sort(lo.encode_i32(workloads.uniform_i32_np(16384, 1)))
    loss, _ = lo.root_loss_grad(keys, lo.root_init_theta(keys))
    assert loss < 1e-4
