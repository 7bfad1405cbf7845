"""CPU checks of the package's host-side set-up code against the reference's
golden files: the PV strip (src/vstrip.rs) and the level replication
(src/swto3d.rs)."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("ng", [18, 32, 64])
def test_pv_strip_golden(sw, ng):
    ref = golden("sta2dfft")["vstrip/qq_init_%d.r8" % ng][1:]
    np.testing.assert_allclose(sw.vstrip.pv_strip(ng), ref, rtol=0, atol=1e-13)


def test_swto3d_golden(sw):
    g = golden("sta2dfft")
    sw2 = g["swto3d/18_2_sw_init.r8"].reshape(3, 18 * 18 + 1)[:, 1:]
    for got, name in zip(sw.swto3d.swto3d_arrays(2, *sw2), ("qq", "dd", "gg")):
        np.testing.assert_array_equal(got, g["swto3d/18_2_%s_init.r8" % name][1:])


def test_parameters_defaults_match_yaml(sw, tmp_path):
    """Parameters defaults equal the reference's parameters.yaml (src/parameters.rs:98-105)."""
    p = tmp_path / "p.yaml"
    p.write_text("""numerical:
  grid_resolution: 32
  vertical_layers: 4
  time_step: 0.03125
  duration: 25.0
  save_interval: 0.25
  max_pressure_difference: 0.000000001
  strip_width: 0.4
  a2: 0.02
  a3: -0.01
physical:
  coriolis_frequency: 12.566370614359173
  gravity_wave_speed: 6.283185307179586
  mean_fluid_depth: 0.4
  damping: 10.0
  nnu: 3.0
environment:
  threads: 0
  output_directory: "./out"
""")
    assert sw.parameters.Parameters.from_yaml(str(p)) == sw.parameters.Parameters()
