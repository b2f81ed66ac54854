"""Argument checks of the layer-potential operator that need no GPU."""
import numpy as np
import pytest

from zfmm_b200.operator import Helm2DLayerOperator


def test_double_layer_needs_dipvec():
    z = np.zeros((2, 10), np.complex128)
    with pytest.raises(ValueError, match="dipvec"):
        Helm2DLayerOperator(1e-9, 1.0, z, alpha=1.0, beta=1.0)
