"""Cone-beam operators (drop-in for ``aprict.cb``)."""

from . import flatpanel

__all__ = ["flatpanel"]
