import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def rot_err(qa, qb):
    """Angle (rad) of the rotation between two (w, x, y, z) quaternions, per
    row: 2 atan2(|v|, |w|) of qa* qb, well conditioned near zero (an arccos of
    the dot product turns one float32 rounding into about 7e-4 rad)."""
    import numpy as np
    qa = qa.astype(np.float64)
    qb = qb.astype(np.float64)
    w = qa[:, 0] * qb[:, 0] + np.sum(qa[:, 1:] * qb[:, 1:], axis=1)
    v = qa[:, 0:1] * qb[:, 1:] - qb[:, 0:1] * qa[:, 1:] - np.cross(qa[:, 1:], qb[:, 1:])
    return 2.0 * np.arctan2(np.linalg.norm(v, axis=1), np.abs(w))


def oracle_available():
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liboracle.so")):
        return True
    from oracle import oracle
    return oracle.reference_root() is not None


@pytest.fixture(scope="session")
def oracle_mod():
    if not oracle_available():
        pytest.skip("oracle library not built")
    from oracle import oracle
    return oracle
