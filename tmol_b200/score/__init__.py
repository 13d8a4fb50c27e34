"""Scoring terms and their ops.  Importing the package registers the
drop-in ops with torch's dispatcher (``torch.ops.tmol_b200.*``, see
``torch_ops``)."""

from . import torch_ops  # noqa: F401
