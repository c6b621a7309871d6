"""Effective number of looks (reference cuphu/_looks.py:6-88)."""

__all__ = ["get_effective_looks"]


def get_effective_looks(range_looks, azimuth_looks, range_spacing, azimuth_spacing,
                        range_resolution, azimuth_resolution):
    r"""Equivalent number of independent looks for ``unwrap``'s ``nlooks``:
    :math:`n_e = k_r k_a d_r d_a / (\rho_r \rho_a)` (multilook factors times the
    oversampling correction of single-look spacing over resolution)."""
    return (range_looks * azimuth_looks * (range_spacing * azimuth_spacing)
            / (range_resolution * azimuth_resolution))
