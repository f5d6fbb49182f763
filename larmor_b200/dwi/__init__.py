"""DWI models on the GPU: DTI and DKI, with the API of larmor.dwi."""

from larmor_b200.dwi.dki import DKIFit, DKIModel
from larmor_b200.dwi.dti import DTIFit, DTIModel

__all__ = ["DKIFit", "DKIModel", "DTIFit", "DTIModel"]
