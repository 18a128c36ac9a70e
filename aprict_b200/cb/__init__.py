"""Cone-beam operators (drop-in for ``aprict.cb``)."""

from . import flatpanel, noop_filter, ramp_filter
from .noop_filter import NoOpFilterer
from .ramp_filter import FBPFilterer, RampFilterer

__all__ = ["FBPFilterer", "NoOpFilterer", "RampFilterer", "flatpanel", "noop_filter", "ramp_filter"]
