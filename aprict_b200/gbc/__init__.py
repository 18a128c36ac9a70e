"""GBC reconstruction pieces (drop-in for ``aprict.gbc``): the expected
weight sums over a cylindrical source locus and the volume-domain cone-beam
ramp filter."""

from . import filters, weightinteg
from .filters import ramp_filter_conebeam
from .weightinteg import backproj_gbc_weight_integ_GPU, backproj_gbc_weight_integ_xygrid_GPU

__all__ = [
    "backproj_gbc_weight_integ_GPU",
    "backproj_gbc_weight_integ_xygrid_GPU",
    "filters",
    "ramp_filter_conebeam",
    "weightinteg",
]
