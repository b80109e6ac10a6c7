"""The byte model behind bench.py's roofline figures: per fluid particle,
own state in and out plus the 4-byte neighbour index list (neighbour
gathers are cache traffic).  Pins the per-kernel formulas so that a change
to a kernel's compulsory set is made in one place on purpose.  CPU only."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.parametrize("nb", [0.0, 32.14, 48.0])
def test_byte_model_per_kernel(nb):
    from bench import ALG_BYTES
    # sweep A (rho_adv or Drho/Dt, kappa): 40 + 4n
    assert ALG_BYTES["df_density_a"](nb) == pytest.approx(40 + 4 * nb)
    assert ALG_BYTES["df_div_a"](nb) == pytest.approx(40 + 4 * nb)
    # sweep B (v_adv update): 56 + 4n
    assert ALG_BYTES["df_density_b"](nb) == pytest.approx(56 + 4 * nb)
    assert ALG_BYTES["df_div_b"](nb) == pytest.approx(56 + 4 * nb)
    # forces + v_adv: 48 + 4n
    assert ALG_BYTES["df_forces"](nb) == pytest.approx(48 + 4 * nb)
    # list build 20 + 4n, rho/alpha 24 + 4n, fused first divergence sweep 40 + 4n
    assert ALG_BYTES["build_first"](nb) == pytest.approx(44 + 8 * nb)
    assert ALG_BYTES["build_first_div"](nb) == pytest.approx(84 + 12 * nb)
    assert ALG_BYTES["hash"](nb) == 88 and ALG_BYTES["reorder"](nb) == 112


def test_dominant_kernel_figure_at_the_measured_mean():
    from bench import ALG_BYTES
    # 168.6 bytes per particle at the 1 M dam break's 32.14 stored neighbours
    assert round(ALG_BYTES["df_density_a"](32.14), 1) == 168.6
