"""Validation helpers and constants shared with the reference API."""

from numbers import Number

_EPS = 1e-12  # ksig/utils.py:16


def check_positive_value(scalar: Number, name: str) -> Number:
  """Raises ``ValueError`` unless ``scalar > 0`` (ksig/utils.py:23-35)."""
  if scalar <= 0:
    raise ValueError(f'The parameter \'{name}\' should have a positive value.')
  return scalar
