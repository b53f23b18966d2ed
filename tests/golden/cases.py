"""The golden cases: small versions of the benchmark workloads plus cases that
exercise every branch of the step (moving fluid, anisotropic scattering,
moment sources, each metric class, the reference's shipped constants)."""


def golden_cases(W):
    return {
        "flat_beam": W.flat_beam(nx_=20, ny_=20, n_dir=12, steps=15),
        "curved_shell": W.curved_shell(nx_=24, ny_=24, n_dir=16, steps=10),
        "curved_scatter": W.curved_scatter(nx_=24, ny_=24, n_dir=16, n_fourier=9, steps=10),
        "moving_kerr": W.moving_scatter(),
        "moving_schwarzschild": W.moving_scatter(metric_kind=W.SCHWARZSCHILD, seed=12),
        "moving_flat": W.moving_scatter(metric_kind=W.MINKOWSKI, streaming_type=W.FLAT_FIXED, seed=13),
        # the reference as shipped: excision 2.1 M and RK45 tolerance 1e-4
        "shipped_constants": W.curved_shell(nx_=20, ny_=22, n_dir=12, steps=6, rk_tol=1e-4, excision=-1.0),
    }
