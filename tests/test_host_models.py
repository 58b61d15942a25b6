"""The per-movie host models against the reference's own code (compiled here): the drift walker, the illumination
field and the background fade, bit for bit. Host code only: no GPU."""
import numpy as np
import pytest

from insiliscope_b200.engine import DriftSettings, background_fade_scale, drift_trajectory, illumination_field


@pytest.mark.parametrize("settings", [
    DriftSettings(xy_nm_per_sqrt_sec=10.0, z_nm_per_sqrt_sec=5.0),
    DriftSettings(xy_nm_per_sqrt_sec=5.0, z_nm_per_sqrt_sec=2.0, xy_speed_nm_per_sec=3.0, z_speed_nm_per_sec=1.5,
                  speed_wander_pct=20.0, wander_time_sec=12.0),
    DriftSettings(xy_speed_nm_per_sec=4.0, xy_angle_deg=30.0, z_speed_nm_per_sec=-2.0, z_direction=1,
                  angle_wander_deg=45.0, z_angle_wander_deg=180.0, wander_time_sec=0.0),
    DriftSettings(),
])
@pytest.mark.parametrize("seed", [42, 7, -3])
def test_drift_matches_reference(reference, settings, seed):
    got = drift_trajectory(seed, 300, 0.03, settings)
    want = reference.drift_trajectory(seed, 300, 0.03, settings)
    assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("profile,fwhm", [(0, 50.0), (1, 60.0), (2, 70.0), (1, 5.0)])
@pytest.mark.parametrize("w,h", [(128, 128), (97, 64)])
def test_illumination_field_matches_reference(reference, profile, fwhm, w, h):
    got, mf = illumination_field(w, h, profile, fwhm)
    want, wmf = reference.illumination_field(w, h, profile, fwhm)
    if profile == 0:
        assert got is None and want is None and mf == wmf == 1.0
    else:
        assert got.tobytes() == want.tobytes() and mf == wmf


def test_background_fade(reference):
    for t, d in ((0.0, 30.0), (12.5, 30.0), (100.0, 7.0), (5.0, 0.0)):
        assert background_fade_scale(t, d) == reference.background_fade_scale(t, d)
