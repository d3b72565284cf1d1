"""Host-side pieces of the reference interface that need no GPU: the EOS
check, the grid descriptor and the initial data."""
from types import SimpleNamespace

import pytest
import torch

from hlld_ai_b200.physics.eos import hybrid_eos, kernel_gamma
from hlld_ai_b200.physics.grid import Grid2D
from hlld_ai_b200.physics.initial_data2d import PROBLEMS, b_from_potential, initial_prims


def test_kernel_gamma_accepts_any_ideal_gas_hybrid_eos():
    assert kernel_gamma(hybrid_eos(K=0, gamma=5 / 3, gamma_th=5 / 3)) == 5 / 3
    # the reference's hybrid_eos has the same three attributes
    assert kernel_gamma(SimpleNamespace(K=0.0, gamma=4 / 3, gamma_th=4 / 3)) == 4 / 3
    for bad in (SimpleNamespace(K=1.0, gamma=2.0, gamma_th=2.0),
                SimpleNamespace(K=0.0, gamma=2.0, gamma_th=None),
                SimpleNamespace(K=0.0, gamma=2.0, gamma_th=1.5), object()):
        with pytest.raises(NotImplementedError):
            kernel_gamma(bad)


def test_grid_layout_matches_the_reference_shapes():
    g = Grid2D(0.0, 1.0, 10, -1.0, 1.0, 6, ng=3, device="cpu")
    assert g.shape == (16, 12) and (g.nxt, g.nyt) == (16, 12)
    assert g.xf.shape == (17,) and g.yf.shape == (13,)
    assert float(g.x[3]) == 0.05 and float(g.xf[3]) == 0.0 and float(g.yf[9]) == 1.0
    assert g.X.shape == g.shape and float(g.Y[0, 3]) == -1.0 + 0.5 * g.dy
    xc, yc = g.corner_mesh()
    assert xc.shape == (17, 13) and torch.equal(xc[:, 0], g.xf) and torch.equal(yc[0], g.yf)


@pytest.mark.parametrize("problem", sorted(PROBLEMS))
def test_initial_field_is_divergence_free(problem):
    g, eos, prims, Az, spec = initial_prims(problem, 24, 2, "cpu")
    Bxf, Byf = b_from_potential(Az, g.dx, g.dy)
    assert Bxf.shape == (g.nxt + 1, g.nyt) and Byf.shape == (g.nxt, g.nyt + 1)
    scale = max(float(Bxf.abs().max()), float(Byf.abs().max()), 1e-30)
    assert float(g.div_b(Bxf, Byf).abs().max()) < 1e-12 * scale / g.dx
    assert set(prims) == {"rho", "vx", "vy", "vz", "p", "eps", "Bx", "By", "Bz"}
    v2 = prims["vx"] ** 2 + prims["vy"] ** 2 + prims["vz"] ** 2
    assert float(v2.max()) < 1.0 and float(prims["rho"].min()) > 0 and float(prims["p"].min()) > 0
