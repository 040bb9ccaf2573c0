"""The blackbody table of the render's optical model (blackbody.ts:85-97), oracle side, on CPU."""
import numpy as np

from oracle import fp_oracle


def test_blackbody_table_shape_and_physics():
    t = fp_oracle.blackbody_table()
    assert t.shape == (512, 4) and np.isfinite(t).all()
    kelvin = 500.0 + 9500.0 * np.arange(512) / 511.0
    # Radiance rises with temperature (Stefan-Boltzmann in the visible band); the coolest
    # entries sit at the table's floor of 2^-32 ...
    assert np.all(np.diff(t[:, 3]) >= 0) and t[0, 3] == -32.0
    assert np.all(np.diff(t[t[:, 3] > -32.0, 3]) > 0)
    # ... and is measured from 1800 K.
    i = int(np.argmin(np.abs(kelvin - 1800.0)))
    assert abs(t[i, 3]) < 0.05
    # Each entry is peak-normalised; hot bodies turn from red to blue-white.
    assert np.allclose(t[:, :3].max(axis=1), 1.0, atol=1e-6)
    assert t[0, 0] == 1.0 and t[0, 2] < 0.05
    assert t[-1, 2] == 1.0 and t[-1, 0] < 1.0
