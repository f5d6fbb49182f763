"""DWI models on the GPU: DTI and DKI, with the API of larmor.dwi, and the S0 and shell helpers
their inputs use."""

from larmor_b200.dwi.dki import DKIFit, DKIModel
from larmor_b200.dwi.dti import DTIFit, DTIModel
from larmor_b200.dwi.inputs import estimate_s0, mean_b0
from larmor_b200.dwi.shells import shell_mask

__all__ = ["DKIFit", "DKIModel", "DTIFit", "DTIModel", "estimate_s0", "mean_b0", "shell_mask"]
