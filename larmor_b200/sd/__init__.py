"""Spherical deconvolution on the GPU: MSMT-CSD (and mFOD), with the API of larmor.sd."""

from larmor_b200.sd.csd import CSDModel
from larmor_b200.sd.csd_solver import CSDSolver
from larmor_b200.sd.method import SDMethod
from larmor_b200.sd.model import SDFit, SDModel
from larmor_b200.sd.solvers import DRL, L2NNLS
from larmor_b200.sd.msmt_csd import MSMTCSDModel
from larmor_b200.sd.peaks import Peaks, find_peaks
from larmor_b200.sd.rf import AnisotropicRF, IsotropicRF, ZonalSHRF

__all__ = ["AnisotropicRF", "CSDModel", "CSDSolver", "DRL", "IsotropicRF", "L2NNLS", "MSMTCSDModel", "Peaks", "SDFit", "SDMethod", "SDModel",
           "ZonalSHRF", "find_peaks"]
