"""The public names of larmor_b200.sd and larmor_b200.dwi that the reference's packages export
for the fitting path (src/larmor/sd/__init__.py, src/larmor/dwi/__init__.py), and the small
helpers among them, on the CPU."""

from __future__ import annotations

import numpy as np
import pytest

SD_NAMES = ["AnisotropicRF", "CSDModel", "CSDSolver", "DRL", "IsotropicRF", "L2NNLS", "MSMTCSDModel",
            "PEAK_RELATIVE_THRESHOLD", "Peaks", "ResponseFunction", "SDFit", "SDMethod", "SDModel", "SDSolver",
            "SD_MODEL_PEAK_RELATIVE_THRESHOLD", "ZonalSHRF", "convert_sh_basis", "find_peaks", "fit_sh",
            "sh_layout"]
DWI_NAMES = ["DKIFit", "DKIModel", "DTIFit", "DTIModel", "estimate_s0", "mean_b0", "shell_mask"]


@pytest.mark.parametrize(("module", "names"), [("larmor_b200.sd", SD_NAMES), ("larmor_b200.dwi", DWI_NAMES)])
def test_packages_export_the_fitting_names(module, names):
    import importlib

    mod = importlib.import_module(module)
    assert sorted(mod.__all__) == sorted(names)
    assert all(hasattr(mod, name) for name in names)


def test_shell_mask_and_thresholds_are_the_reference_ones():
    """src/larmor/dwi/shells.py:9-25 (strictly within 100 s/mm^2), src/larmor/sd/peaks.py."""
    from larmor_b200.dwi import shell_mask
    from larmor_b200.sd import PEAK_RELATIVE_THRESHOLD, SD_MODEL_PEAK_RELATIVE_THRESHOLD, SDSolver

    bvals = np.array([0.0, 900.0, 1000.0, 1099.9, 1100.0, 2000.0])
    np.testing.assert_array_equal(shell_mask(bvals, 1000.0), [False, False, True, True, False, False])
    np.testing.assert_array_equal(shell_mask(bvals, 1000.0, tol=50.0), [False, False, True, False, False, False])
    assert (PEAK_RELATIVE_THRESHOLD, SD_MODEL_PEAK_RELATIVE_THRESHOLD) == (0.1, 0.2)
    from larmor_b200.sd import DRL, L2NNLS

    assert set(SDSolver.__value__.__args__) == {DRL, L2NNLS}
