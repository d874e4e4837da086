"""Utilities mirroring ``sinv.utils`` (``src/sinv/utils/__init__.py:3``)."""

from . import matrices_utils as matu  # noqa: F401
