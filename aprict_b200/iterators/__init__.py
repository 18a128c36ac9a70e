"""Iterative reconstruction (drop-in for ``aprict.iterators``)."""

from .landweber_vram import Landweber_flatpanel
from .sirt_batch import SIRTBatch
from .sirt_vram import SIRT_flatpanel

__all__ = ["Landweber_flatpanel", "SIRTBatch", "SIRT_flatpanel"]
