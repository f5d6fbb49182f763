"""Spherical deconvolution on the GPU: MSMT-CSD, mFOD, GRL, single-shell CSD and FOD peaks,
with the API of larmor.sd."""

from larmor_b200.sd.csd import CSDModel
from larmor_b200.sd.csd_solver import CSDSolver
from larmor_b200.sd.method import SDMethod
from larmor_b200.sd.model import SDFit, SDModel
from larmor_b200.sd.msmt_csd import MSMTCSDModel
from larmor_b200.sd.peaks import PEAK_RELATIVE_THRESHOLD, SD_MODEL_PEAK_RELATIVE_THRESHOLD, Peaks, find_peaks
from larmor_b200.sd.rf import AnisotropicRF, IsotropicRF, ResponseFunction, ZonalSHRF
from larmor_b200.sd.sh import convert_sh_basis, fit_sh, sh_layout
from larmor_b200.sd.solvers import DRL, L2NNLS, SDSolver

__all__ = ["PEAK_RELATIVE_THRESHOLD", "SD_MODEL_PEAK_RELATIVE_THRESHOLD", "AnisotropicRF", "CSDModel", "CSDSolver",
           "DRL", "IsotropicRF", "L2NNLS", "MSMTCSDModel", "Peaks", "ResponseFunction", "SDFit", "SDMethod", "SDModel",
           "SDSolver", "ZonalSHRF", "convert_sh_basis", "find_peaks", "fit_sh", "sh_layout"]
