"""Calibration harness: gradients of an elevation misfit with respect to the
bottom roughness, the bed elevation and the open-boundary amplitudes, through
the hand-written adjoint of libefdc_xm (efdc_xm_calib_*), exposed to PyTorch
as a torch.autograd.Function.  The solver library itself has no PyTorch
dependency; only this harness uses torch."""
from .problem import CalibProblem, CalibLoss, boundary_groups  # noqa: F401
