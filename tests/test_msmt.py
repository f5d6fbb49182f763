"""The MSMT-CSD problem's matrices against the reference's (tests/golden/msmt.npz, written by the
reference's sd/msmt.py for the responses and three-shell table of tests/sd/test_msmt.py)."""

from __future__ import annotations

import numpy as np
import pytest


def _responses(z):
    from larmor_b200.sd.rf import ZonalSHRF

    return [ZonalSHRF(bvals=z["shells"], coefficients=z[k])
            for k in ("wm_coefficients", "gm_coefficients", "csf_coefficients")]


def test_forward_and_constraint_matrices_are_the_references(msmt_fixture):
    from larmor_b200.sd.msmt import NORM_REG, constraint_matrix, forward_matrix
    from larmor_b200.sd.sphere import DIRS_300

    z = msmt_fixture
    f = forward_matrix(_responses(z), [8, 0, 0], z["bvals"], z["bvecs"])
    np.testing.assert_array_equal(f, z["forward"])
    np.testing.assert_array_equal(constraint_matrix([8, 0, 0], DIRS_300), z["constraints"])
    assert float(np.sqrt(NORM_REG * np.max(np.sum(f**2, axis=0)))) == float(z["ridge"])


def test_b0_rows_see_only_the_isotropic_degree(msmt_fixture):
    from larmor_b200.sd.msmt import forward_matrix

    z = msmt_fixture
    f = forward_matrix(_responses(z), [8, 0, 0], z["bvals"], z["bvecs"])
    b0 = np.linalg.norm(z["bvecs"], axis=1) == 0
    assert b0.any()
    # Columns 1..44 are the WM FOD's l > 0 coefficients.
    assert (f[b0, 1:45] == 0).all() and (f[b0, 0] != 0).all()


def test_a_table_that_cannot_separate_the_tissues_is_refused(msmt_fixture):
    from larmor_b200.sd.msmt import prepare_msmt
    from larmor_b200.sd.sphere import DIRS_300

    z = msmt_fixture
    one_shell = np.abs(z["bvals"] - z["bvals"].max()) < 50
    with pytest.raises(ValueError, match="cannot separate"):
        prepare_msmt(_responses(z), [8, 0, 0], z["bvals"][one_shell], z["bvecs"][one_shell], DIRS_300)
